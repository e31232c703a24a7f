// alphas.cuh -- the alpha_s (gradient-correction) term of the Orsay-Trento functional, core4 = 'OTC'
// (Dynamics_TDDFT/term_alfa.f90:5-117, He_statics/term_alfa.f90, energy.f90 ealphas), binary64.
//
//   falfs   = 1 - denalf/den0s,                 denalf = C2R(fden kalfs)
//   int*alf = C2R(R2C(falfs d*den) kalfs)       (three components)
//   ualphas = [C2R(R2C(grad den . int alf) kalfs)/den0s + div(falfs int alf)] h2o2m4 alphas
//   ealphas = -h2o2m4/2 alphas sum falfs (grad den . int alf) dxyz
// The convolutions run through the pencil FFT passes; this file holds the pointwise stages, the
// divergence (three first-derivative stencil passes) and the energy reduction.
#pragma once
#include "ops.cuh"

namespace he {

// falfs and the three sources falfs * d{x,y,z}den (term_alfa.f90:28-36).
#ifndef HE_KERNEL_TU
__global__ void __launch_bounds__(256) k_alf_src(const double* __restrict__ denalf,
                                                 const double* __restrict__ dx, const double* __restrict__ dy,
                                                 const double* __restrict__ dz, double den0s, long N,
                                                 double* __restrict__ falfs, double* __restrict__ s1,
                                                 double* __restrict__ s2, double* __restrict__ s3) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < N; i += (long)gridDim.x * blockDim.x) {
    const double f = 1.0 - denalf[i] / den0s;
    falfs[i] = f;
    s1[i] = f * dx[i];
    s2[i] = f * dy[i];
    s3[i] = f * dz[i];
  }
}
#endif

// grad den . int alf (term_alfa.f90:65-69).
#ifndef HE_KERNEL_TU
__global__ void __launch_bounds__(256) k_alf_dot(const double* __restrict__ dx, const double* __restrict__ dy,
                                                 const double* __restrict__ dz, const double* __restrict__ ix,
                                                 const double* __restrict__ iy, const double* __restrict__ iz,
                                                 long N, double* __restrict__ out) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < N; i += (long)gridDim.x * blockDim.x)
    out[i] = dx[i] * ix[i] + dy[i] * iy[i] + dz[i] * iz[i];
}
#endif

// falfs * int{x,y,z}alf (term_alfa.f90:87-92).
#ifndef HE_KERNEL_TU
__global__ void __launch_bounds__(256) k_alf_fi(const double* __restrict__ falfs, const double* __restrict__ ix,
                                                const double* __restrict__ iy, const double* __restrict__ iz,
                                                long N, double* __restrict__ s1, double* __restrict__ s2,
                                                double* __restrict__ s3) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < N; i += (long)gridDim.x * blockDim.x) {
    const double f = falfs[i];
    s1[i] = f * ix[i];
    s2[i] = f * iy[i];
    s3[i] = f * iz[i];
  }
}
#endif

// One component of the divergence: out = d f / d axis (derivnD(1,...) of term_alfa.f90:106-108).
template <int AX>
struct OpAxisDeriv {
  static const char* kname() { return "alphas_divergence"; }
  using T = double;
  static constexpr int NV = 0, N8 = 0, N16 = 0;
  const double* s8[1];
  const double2* s16[1];
  double* out;
  HE_D void at(int, int, int, long i, double dx, double dy, double dz, double, const double*,
               const double2*, int, double*) const {
    out[i] = (AX == 0) ? dx : (AX == 1) ? dy : dz;
  }
};

// ualphas = (ua/den0s + d_x s1 + d_y s2 + d_z s3) h2o2m4 alphas (term_alfa.f90:87-113), the
// stencil input being s3; operands ua (raw convolution), d_x s1, d_y s2.
struct OpAlfFinal {
  static const char* kname() { return "alphas_field"; }
  using T = double;
  static constexpr int NV = 0, N8 = 3, N16 = 0;
  const double* s8[N8];
  const double2* s16[1];
  double* out;
  double den0s, h2o2m4, alphas;
  HE_D void at(int, int, int, long i, double, double, double dz, double, const double* v8,
               const double2*, int vs, double*) const {
    const double ua = v8[0] / den0s;
    out[i] = (((ua + v8[vs]) + v8[2 * vs]) + dz) * h2o2m4 * alphas;
  }
};

// sum falfs (dxden intxalf + dyden intyalf + dzden intzalf) (energy.f90:131-135).
#ifndef HE_KERNEL_TU
__global__ void __launch_bounds__(256) k_alf_energy(const double* __restrict__ falfs,
                                                    const double* __restrict__ dx, const double* __restrict__ dy,
                                                    const double* __restrict__ dz, const double* __restrict__ ix,
                                                    const double* __restrict__ iy, const double* __restrict__ iz,
                                                    long N, const ReduceTail rt) {
  double acc[1] = {0.0};
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < N; i += (long)gridDim.x * blockDim.x)
    acc[0] += falfs[i] * (dx[i] * ix[i] + dy[i] * iy[i] + dz[i] * iz[i]);
  block_reduce_store<1>(acc, rt.partials + blockIdx.x);
  reduce_tail<1>(rt, gridDim.x);
}
#endif

}  // namespace he
