// quantum.cuh -- device side of the quantum-impurity path (Dynamics_quantum_impurities), binary64
// and the binary32 variants of the mixed path.
//
// The impurities are wave functions psix_i (nx,ny,nz) with their own Hamiltonians
//   H_i psix_i = timec*(h2o2mx_i lap psix_i - upotx_i psix_i),  h2o2mx_i = h2o2m4*4.002603/m_i,
// coupled to the helium through convolutions with radial kernels (potenimp.f90:1-43):
//   potx4   = sum_i C2R(R2C(|psix_i|^2) uimp_k_i)                  (He sees the impurities)
//   upotx_i = C2R(fden uimp_k_i) + sum_{j!=i} C2R(R2C(|psix_j|^2) uimp_k_k(i,j))
// uimp_k_i is FT_V_spline of the He-X pair potential at |p| (FT_V_spline.f90:14-276,
// potenimpini.f90:116-163).
//
// Kernels here:
//   OpGrad2      stencil consumer: sum |d psi/dx|^2+|d psi/dy|^2+|d psi/dz|^2 (energy.f90:105-109)
//   k_zmix       z pencils: optional forward z transform of one spectrum, then up to two outputs
//                each a sum of up to kMaxTerms (spectrum x real kernel) products, inverse z.
//   k_cnorm2     |psix|^2, k_dot sum a*b, k_moments sum |psix|^2 (1, x, y, z)
//   k_ftv        FT_V_spline's closed-form transform of the cubic pieces, one CTA per momentum
//   k_uimpk      the momentum spline evaluated at pmod over the half spectrum (findi + Horner)
#pragma once
#include "fft_kernels.cuh"
#include "ops.cuh"
#include "setup.cuh"

namespace he {

constexpr int kMaxQImp = 4;
constexpr int kMaxTerms = 4;

// TT = float2: the mixed path's binary32 hi plane, summed in binary64.
template <typename TT>
struct OpGrad2T {
  static const char* kname() { return sizeof(TT) == 8 ? "grad2_reduce_f32" : "grad2_reduce"; }
  using T = TT;
  using R = typename RealOf<TT>::R;
  using Z = typename RealOf<TT>::Z;
  static constexpr int NV = 1, N8 = 0, N16 = 0;
  const R* s8[1];
  const Z* s16[1];
  HE_D void remap(const MemberMap&, int) {}  // no pointers besides the stencil's field
  HE_D static double n2(TT v) { return (double)v.x * (double)v.x + (double)v.y * (double)v.y; }
  HE_D void at(int, int, int, long, TT dx, TT dy, TT dz, TT, const R*, const Z*, int,
               double* acc) const {
    acc[0] += n2(dx) + n2(dy) + n2(dz);
  }
};
using OpGrad2 = OpGrad2T<double2>;

struct ZMixArgs {
  int nxh, ny, nz, tkx;
  LinePlan pl;
  const double2* fwd_in;   // x,y-transformed spectrum to transform along z (null: none)
  double2* fwd_store;      // receives that z spectrum (null: not stored)
  int nout;                // 0, 1 or 2
  double2* out[2];
  int nterm[2];
  const double2* src[2][kMaxTerms];  // full spectra; null = the forward spectrum of fwd_in
  const double* ker[2][kMaxTerms];   // real kernels over the half spectrum
  MemberMap mm;                      // group members (blockIdx.z is the member)
  HE_D void remap(int m) {
    fwd_in = mm(fwd_in, m);
    fwd_store = mm(fwd_store, m);
    for (int o = 0; o < 2; ++o) {
      out[o] = mm(out[o], m);
      for (int t = 0; t < kMaxTerms; ++t) {
        src[o][t] = mm(src[o][t], m);
        ker[o][t] = mm(ker[o][t], m);
      }
    }
  }
};

// Rt = float: the mixed path (binary32 spectra, kernels given as their binary32 copies).
template <int N, int TILE, typename Rt>
HE_D void zmix_body(const ZMixArgs& a) {
  using C = typename Cx<Rt>::T;
  C* smem = smem_as<C>();
  const C* fwd_in = reinterpret_cast<const C*>(a.fwd_in);
  C* fwd_store = reinterpret_cast<C*>(a.fwd_store);
  const int n = (N > 0) ? N : a.nz;
  const int ls = line_stride(n);
  const int TK = (N > 0) ? TILE : a.tkx;
  const int nxh = a.nxh;
  const int tid = threadIdx.x;
  const int nthr = (N > 0) ? tile_threads(TILE) : (int)blockDim.x;  // compile-time when N > 0
  const int kx0 = blockIdx.x * TK;
  const int ky = blockIdx.y;
  C* tw = smem;
  C* P0 = smem + ((a.pl.stw_len + 1) & ~1);
  C* P1 = P0 + TK * ls;
  C* P2 = P1 + TK * ls;
  load_twiddles(tw, a.pl);
  const long plane = (long)nxh * a.ny;
  const long base = (long)nxh * ky;
  C* F = nullptr;
  C *O0 = P0, *O1 = P1, *S = P2;
  if (fwd_in) {
    for (int e = tid; e < TK * n; e += nthr) {
      const int j = e / TK, c = e - j * TK;
      const int kx = kx0 + c;
      P0[c * ls + sw<N>(j)] = (kx < nxh) ? fwd_in[base + kx + plane * j] : Cx<Rt>::make(0, 0);
    }
    __syncthreads();
    F = fft_lines<N>(P0, P1, TK, ls, a.pl, tw, false);
    O0 = (F == P0) ? P1 : P0;
    O1 = P2;
    S = F;
    if (fwd_store) {
      for (int e = tid; e < TK * n; e += nthr) {
        const int j = e / TK, c = e - j * TK;
        const int kx = kx0 + c;
        if (kx < nxh) fwd_store[base + kx + plane * j] = F[c * ls + sw<N>(j)];
      }
    }
  }
  if (a.nout == 0) return;
  // out[o] = sum_t src_t * ker_t, term by term: each term's loads of all the thread's elements
  // are issued together (the element loop unrolls for the compile-time lengths); the running sum
  // stays in the thread's own slots of O0 / O1, added in term order as a register sum would be
  for (int o = 0; o < a.nout; ++o) {
    C* Oo = (o == 0) ? O0 : O1;
#pragma unroll
    for (int e = tid; e < TK * n; e += nthr) {
      const int j = e / TK, c = e - j * TK;
      Oo[c * ls + sw<N>(j)] = Cx<Rt>::make(0, 0);
    }
    for (int t = 0; t < a.nterm[o]; ++t) {
      const C* src = reinterpret_cast<const C*>(a.src[o][t]);
      const Rt* ker = reinterpret_cast<const Rt*>(a.ker[o][t]);
#pragma unroll
      for (int e = tid; e < TK * n; e += nthr) {
        const int j = e / TK, c = e - j * TK;
        const int kx = kx0 + c;
        if (kx >= nxh) continue;
        const int s = c * ls + sw<N>(j);
        const long g = base + kx + plane * j;
        const C v = src ? src[g] : F[s];
        const Rt w = ker[g];
        C acc = Oo[s];
        acc.x += v.x * w;
        acc.y += v.y * w;
        Oo[s] = acc;
      }
    }
  }
  __syncthreads();
  C* R0 = fft_lines<N>(O0, S, TK, ls, a.pl, tw, true);
  for (int e = tid; e < TK * n; e += nthr) {
    const int j = e / TK, c = e - j * TK;
    const int kx = kx0 + c;
    if (kx < nxh) reinterpret_cast<C*>(a.out[0])[base + kx + plane * j] = R0[c * ls + sw<N>(j)];
  }
  if (a.nout < 2) return;
  __syncthreads();
  C* fr = (R0 == O0) ? S : O0;
  C* R1 = fft_lines<N>(O1, fr, TK, ls, a.pl, tw, true);
  for (int e = tid; e < TK * n; e += nthr) {
    const int j = e / TK, c = e - j * TK;
    const int kx = kx0 + c;
    if (kx < nxh) reinterpret_cast<C*>(a.out[1])[base + kx + plane * j] = R1[c * ls + sw<N>(j)];
  }
}

// G: blockIdx.z is the group member, and the arguments are copied with their pointers mapped to
// the member's buffers; otherwise they are read as passed.
template <int N, int TILE, typename Rt, bool G>
__global__ void __launch_bounds__(tile_threads(TILE)) k_zmix(const ZMixArgs a)
#ifdef HE_KERNEL_TU
{
  if constexpr (G) {
    ZMixArgs b = a;
    b.remap(blockIdx.z);
    zmix_body<N, TILE, Rt>(b);
  } else {
    zmix_body<N, TILE, Rt>(a);
  }
}
#else
;
#endif

// ---- pointwise passes (grid-stride, deterministic two-level reductions) -----------------------
#ifndef HE_KERNEL_TU
__global__ void __launch_bounds__(256) k_cnorm2(const double2* __restrict__ f, double* __restrict__ out,
                                                long N, const MemberMap mm) {
  f = mm(f, blockIdx.y);
  out = mm(out, blockIdx.y);
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < N; i += (long)gridDim.x * blockDim.x)
    out[i] = cnorm2(f[i]);
}
#endif

#ifndef HE_KERNEL_TU
__global__ void __launch_bounds__(256) k_dot(const double* __restrict__ a, const double* __restrict__ b,
                                             long N, const ReduceTail rt_in, const MemberMap mm) {
  a = mm(a, blockIdx.y);
  b = mm(b, blockIdx.y);
  const ReduceTail rt = remap(rt_in, mm, blockIdx.y);
  double acc[1] = {0.0};
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < N; i += (long)gridDim.x * blockDim.x)
    acc[0] += a[i] * b[i];
  block_reduce_store<1>(acc, rt.partials + blockIdx.x);
  reduce_tail<1>(rt, gridDim.x);
}
#endif

// The mixed path: |psix|^2 of the compensated pair (hi and lo planes), rounded once to binary32.
#ifndef HE_KERNEL_TU
__global__ void __launch_bounds__(256) k_cnorm2_pair(const float2* __restrict__ hi,
                                                     const float2* __restrict__ lo,
                                                     float* __restrict__ out, long N,
                                                     const MemberMap mm) {
  hi = mm(hi, blockIdx.y);
  lo = mm(lo, blockIdx.y);
  out = mm(out, blockIdx.y);
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < N; i += (long)gridDim.x * blockDim.x) {
    const double re = (double)hi[i].x + (double)lo[i].x, im = (double)hi[i].y + (double)lo[i].y;
    out[i] = (float)(re * re + im * im);
  }
}
#endif

// sum a*b of binary32 fields, summed in binary64 (the mixed path's energy sums).
#ifndef HE_KERNEL_TU
__global__ void __launch_bounds__(256) k_dot_f32(const float* __restrict__ a, const float* __restrict__ b,
                                                 long N, const ReduceTail rt_in, const MemberMap mm) {
  a = mm(a, blockIdx.y);
  b = mm(b, blockIdx.y);
  const ReduceTail rt = remap(rt_in, mm, blockIdx.y);
  double acc[1] = {0.0};
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < N; i += (long)gridDim.x * blockDim.x)
    acc[0] += (double)a[i] * (double)b[i];
  block_reduce_store<1>(acc, rt.partials + blockIdx.x);
  reduce_tail<1>(rt, gridDim.x);
}
#endif

// {sum |f|^2, sum |f|^2 x, sum |f|^2 y, sum |f|^2 z} (DFT4He3d.f90:682-700 of the quantum driver).
// (C = float2: the hi plane of the mixed path's pair, summed in binary64.)
#ifndef HE_KERNEL_TU
template <typename C>
__global__ void __launch_bounds__(256) k_moments(const C* __restrict__ f, int nx, int ny, long N,
                                                 double x0, double y0, double z0, double hx,
                                                 double hy, double hz, const ReduceTail rt_in,
                                                 const MemberMap mm) {
  f = mm(f, blockIdx.y);
  const ReduceTail rt = remap(rt_in, mm, blockIdx.y);
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < N; i += (long)gridDim.x * blockDim.x) {
    const long r = i / nx;
    const int ix = (int)(i - r * nx);
    const int iy = (int)(r % ny), iz = (int)(r / ny);
    const double s = (double)f[i].x * (double)f[i].x + (double)f[i].y * (double)f[i].y;
    acc[0] += s;
    acc[1] += s * (x0 + hx * ix);
    acc[2] += s * (y0 + hy * iy);
    acc[3] += s * (z0 + hz * iz);
  }
  block_reduce_store<4>(acc, rt.partials + blockIdx.x * 4);
  reduce_tail<4>(rt, gridDim.x);
}
#endif

// ---- FT_V_spline --------------------------------------------------------------------------------
struct FtvArgs {
  const double *x, *a, *b, *c, *d;  // cubic spline of V on n nodes: p_j(r) = a + r(b + r(c + r d))
  int n;
  double hp;                        // momentum step H_p; CTA i computes p = i*H_p
  double r0, f0;                    // r_cutoff and f_cutoff (= umax)
  int parabolic;
  double aa, cc;                    // inverted-parabola core fit (FT_V_spline.f90:128-146)
  double* vpp;
};

// Vpp(p) = [core + sum_j closed-form integral of r sin(qr) p_j(r) over [r_j, r_j+1]] * 4 pi / q,
// q = 2 pi p (FT_V_spline.f90:151-225); p = 0 takes the moments r^2 p_j(r) (:164-188).  The
// nodes' sin(q r_j), cos(q r_j) are computed once per node through shared memory.
#ifndef HE_KERNEL_TU
__global__ void __launch_bounds__(256) k_ftv(const FtvArgs A) {
  __shared__ double s_s[257], s_c[257];
  const int tid = threadIdx.x;
  const double p = blockIdx.x * A.hp;
  const double Qpi = 4.0 * kPi;
  double acc[1] = {0.0};
  double tot[1] = {0.0};
  if (p == 0.0) {
    for (int j = tid; j < A.n - 1; j += blockDim.x) {
      const double u = A.x[j], w = A.x[j + 1];
      const double u2 = u * u, w2 = w * w;
      acc[0] += A.a[j] / 3.0 * (w2 * w - u2 * u) + A.b[j] / 4.0 * (w2 * w2 - u2 * u2) +
                A.c[j] / 5.0 * (w2 * w2 * w - u2 * u2 * u) + A.d[j] / 6.0 * (w2 * w2 * w2 - u2 * u2 * u2);
    }
    block_reduce_store<1>(acc, tot);
    if (tid == 0) {
      const double r0 = A.r0;
      const double Vp = A.parabolic ? A.aa * (r0 * r0 * r0 * r0 * r0) * 0.2 + A.cc * (r0 * r0 * r0) / 3.0
                                    : (r0 * r0 * r0) * A.f0 / 3.0;
      A.vpp[blockIdx.x] = (Vp + tot[0]) * Qpi;
    }
    return;
  }
  const double q = 2.0 * kPi * p;
  const double c1oq = 1.0 / q, c1oq2 = c1oq * c1oq, c1oq3 = c1oq2 * c1oq, c1oq4 = c1oq2 * c1oq2,
               c1oq5 = c1oq4 * c1oq;
  for (int base = 0; base < A.n - 1; base += 256) {
    const int j = base + tid;
    if (j < A.n) sincos(q * A.x[j], &s_s[tid], &s_c[tid]);
    if (tid == 0 && base + 256 < A.n) sincos(q * A.x[base + 256], &s_s[256], &s_c[256]);
    __syncthreads();
    if (j < A.n - 1) {
      const double rj = A.x[j], rj1 = A.x[j + 1];
      const double sqrj = s_s[tid], cqrj = s_c[tid], sqrj1 = s_s[tid + 1], cqrj1 = s_c[tid + 1];
      const double a = A.a[j], b = A.b[j], c = A.c[j], d = A.d[j];
      acc[0] += (a + (b + (c + d * rj) * rj) * rj) * rj * c1oq * cqrj -
                (a + (b + (c + d * rj1) * rj1) * rj1) * rj1 * c1oq * cqrj1 +
                (a + (2.0 * b + (3.0 * c + 4.0 * d * rj1) * rj1) * rj1) * c1oq2 * sqrj1 -
                (a + (2.0 * b + (3.0 * c + 4.0 * d * rj) * rj) * rj) * c1oq2 * sqrj +
                (2.0 * b + (6.0 * c + 12.0 * d * rj1) * rj1) * c1oq3 * cqrj1 -
                (2.0 * b + (6.0 * c + 12.0 * d * rj) * rj) * c1oq3 * cqrj +
                (6.0 * c + 24.0 * d * rj) * c1oq4 * sqrj - (6.0 * c + 24.0 * d * rj1) * c1oq4 * sqrj1 +
                24.0 * d * c1oq5 * (cqrj - cqrj1);
    }
    __syncthreads();
  }
  block_reduce_store<1>(acc, tot);
  if (tid == 0) {
    const double r0 = A.r0;
    double sq, cq;
    sincos(q * r0, &sq, &cq);
    const double Vp = A.parabolic
                          ? c1oq * (cq * (6.0 * A.aa * r0 * c1oq2 - A.aa * (r0 * r0 * r0) - A.cc * r0) +
                                    sq * ((3.0 * A.aa * (r0 * r0) + A.cc) * c1oq - 6.0 * A.aa * c1oq3))
                          : A.f0 * c1oq * (sq * c1oq - r0 * cq);
    A.vpp[blockIdx.x] = (Vp + tot[0]) * c1oq * Qpi;
  }
}
#endif

struct UimpkArgs {
  const double *P, *a, *b, *c, *d;  // momentum table (np) and its spline
  int np;
  int nx, ny, nz, nxh;
  double hx, hy, hz;
  double* out;                      // (nxh, ny, nz)
};

// uimp_k(ix,iy,iz) = FT_V_spline(pmod) (potenimpini.f90:136-144): findi's bisection
// (mates.f:4-33) for the piece, then its cubic in p.
#ifndef HE_KERNEL_TU
__global__ void __launch_bounds__(256) k_uimpk(const UimpkArgs A) {
  const long nk = (long)A.nxh * A.ny * A.nz;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < nk; i += (long)gridDim.x * blockDim.x) {
    const long r = i / A.nxh;
    const int ix = (int)(i - r * A.nxh);
    const int iy = (int)(r % A.ny), iz = (int)(r / A.ny);
    const double px = freq_of(ix, A.nx, A.hx), py = freq_of(iy, A.ny, A.hy), pz = freq_of(iz, A.nz, A.hz);
    const double p = sqrt(px * px + py * py + pz * pz);
    int k;
    if (p > A.P[A.np - 1]) k = A.np - 1;
    else if (p < A.P[0]) k = 1;
    else {
      int lo = 1, hi = A.np;
      do {
        const int it = (lo + hi) / 2;
        if (p > A.P[it - 1]) lo = it;
        if (p <= A.P[it - 1]) hi = it;
      } while (hi - lo > 1);
      k = lo;
    }
    --k;
    A.out[i] = A.a[k] + p * (A.b[k] + p * (A.c[k] + p * A.d[k]));
  }
}
#endif

}  // namespace he
