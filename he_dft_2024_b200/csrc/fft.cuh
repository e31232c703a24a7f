// fft.cuh -- shared-memory pencil FFT machinery (binary64) for the R2C/C2R convolutions of the
// mean field.  Replaces the FFTW plans of Dynamics_TDDFT/fft.f90:5-168 and He_statics/fft.f90.
//
// Semantics follow FFTW's dfftw_plan_dft_r2c_3d / dfftw_plan_dft_c2r_3d on column-major
// (nx,ny,nz) arrays: unnormalised forward transform exp(-i...), backward exp(+i...) scaled by
// renor = 1/(nx*ny*nz) afterwards (fft.f90:36,118-168).
//
// A 3-D transform is three pencil passes, each one HBM read and one HBM write of the half
// spectrum: x (contiguous rows, two real rows packed into one complex line), y and z (tiles of
// consecutive kx staged in shared memory).  The k-space kernel multiply is fused into the z pass
// (forward z, multiply, inverse z), and the pointwise prologue/epilogue of poten is fused into
// the x passes.  Lines are transformed by a mixed-radix (8,4,2,3,5) Stockham autosort in shared
// memory (ping-pong buffers), twiddles from a per-length table built on the host in extended
// precision.
#pragma once
#include "common.cuh"

namespace he {

constexpr int kMaxStages = 12;

struct LinePlan {
  int n;                 // line length
  int nst;               // number of radix stages
  int rad[kMaxStages];   // radix of each stage
  const double2* tw;     // device table exp(-2 pi i m / n), m = 0..n-1
};

// Radix-R DFT in registers; inv selects exp(+i).
template <int R>
HE_D void dft(double2* v, bool inv);

template <>
HE_D void dft<2>(double2* v, bool) {
  double2 a = v[0], b = v[1];
  v[0] = cadd(a, b);
  v[1] = csub(a, b);
}

template <>
HE_D void dft<4>(double2* v, bool inv) {
  double2 t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]);
  double2 t2 = cadd(v[1], v[3]), u = csub(v[1], v[3]);
  double2 mu = inv ? cpi(u) : cmi(u);  // exp(-+ i pi/2) * u
  v[0] = cadd(t0, t2);
  v[2] = csub(t0, t2);
  v[1] = cadd(t1, mu);
  v[3] = csub(t1, mu);
}

template <>
HE_D void dft<8>(double2* v, bool inv) {
  const double r = 0.70710678118654752440;  // 1/sqrt(2)
  double2 e[4] = {v[0], v[2], v[4], v[6]};
  double2 o[4] = {v[1], v[3], v[5], v[7]};
  dft<4>(e, inv);
  dft<4>(o, inv);
  // twiddles exp(-+ 2 pi i k / 8), k = 0..3
  double2 w1 = inv ? make_double2(r, r) : make_double2(r, -r);
  double2 o1 = cmul(o[1], w1);
  double2 o2 = inv ? cpi(o[2]) : cmi(o[2]);
  double2 w3 = inv ? make_double2(-r, r) : make_double2(-r, -r);
  double2 o3 = cmul(o[3], w3);
  v[0] = cadd(e[0], o[0]);
  v[4] = csub(e[0], o[0]);
  v[1] = cadd(e[1], o1);
  v[5] = csub(e[1], o1);
  v[2] = cadd(e[2], o2);
  v[6] = csub(e[2], o2);
  v[3] = cadd(e[3], o3);
  v[7] = csub(e[3], o3);
}

template <>
HE_D void dft<3>(double2* v, bool inv) {
  const double c = -0.5, s = 0.86602540378443864676;  // cos, sin of 2 pi / 3
  double2 t = cadd(v[1], v[2]), d = csub(v[1], v[2]);
  double2 m = make_double2(v[0].x + c * t.x, v[0].y + c * t.y);
  double2 sd = cscale(s, d);
  double2 isd = inv ? cpi(sd) : cmi(sd);
  v[0] = cadd(v[0], t);
  v[1] = cadd(m, isd);
  v[2] = csub(m, isd);
}

template <>
HE_D void dft<5>(double2* v, bool inv) {
  const double c1 = 0.30901699437494742410, c2 = -0.80901699437494742410;
  const double s1 = 0.95105651629515357212, s2 = 0.58778525229247312917;
  double2 t1 = cadd(v[1], v[4]), t2 = cadd(v[2], v[3]);
  double2 d1 = csub(v[1], v[4]), d2 = csub(v[2], v[3]);
  double2 a1 = make_double2(v[0].x + c1 * t1.x + c2 * t2.x, v[0].y + c1 * t1.y + c2 * t2.y);
  double2 a2 = make_double2(v[0].x + c2 * t1.x + c1 * t2.x, v[0].y + c2 * t1.y + c1 * t2.y);
  double2 b1 = make_double2(s1 * d1.x + s2 * d2.x, s1 * d1.y + s2 * d2.y);
  double2 b2 = make_double2(s2 * d1.x - s1 * d2.x, s2 * d1.y - s1 * d2.y);
  double2 ib1 = inv ? cpi(b1) : cmi(b1);
  double2 ib2 = inv ? cpi(b2) : cmi(b2);
  v[0] = cadd(v[0], cadd(t1, t2));
  v[1] = cadd(a1, ib1);
  v[4] = csub(a1, ib1);
  v[2] = cadd(a2, ib2);
  v[3] = csub(a2, ib2);
}

// One Stockham stage of radix R over 'nlines' lines (line stride ls) from src to dst.
template <int R>
HE_D void stockham_stage(const double2* __restrict__ src, double2* __restrict__ dst, int nlines,
                         int ls, int n, int ns, const double2* __restrict__ tw, bool inv,
                         int tid, int nthr) {
  const int nr = n / R;
  const int twstep = n / (ns * R);
  const int total = nlines * nr;
  for (int w = tid; w < total; w += nthr) {
    const int line = w / nr;
    const int j = w - line * nr;
    const int k = j % ns;
    const double2* s = src + line * ls;
    double2* d = dst + line * ls;
    double2 v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      double2 x = s[j + r * nr];
      v[r] = (r == 0) ? x : cmul_conj_if(x, tw[r * k * twstep], inv);
    }
    dft<R>(v, inv);
    const int base = (j / ns) * ns * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) d[base + r * ns] = v[r];
  }
}

// Transform 'nlines' lines held in buffer a (b is scratch of the same size).  Returns the buffer
// holding the result.  Ends with __syncthreads().
HE_D double2* fft_lines(double2* a, double2* b, int nlines, int ls, const LinePlan& pl,
                        const double2* tw_smem, bool inv) {
  const int tid = threadIdx.x + blockDim.x * threadIdx.y;
  const int nthr = blockDim.x * blockDim.y;
  double2* src = a;
  double2* dst = b;
  int ns = 1;
  for (int s = 0; s < pl.nst; ++s) {
    const int R = pl.rad[s];
    switch (R) {
      case 8: stockham_stage<8>(src, dst, nlines, ls, pl.n, ns, tw_smem, inv, tid, nthr); break;
      case 4: stockham_stage<4>(src, dst, nlines, ls, pl.n, ns, tw_smem, inv, tid, nthr); break;
      case 2: stockham_stage<2>(src, dst, nlines, ls, pl.n, ns, tw_smem, inv, tid, nthr); break;
      case 3: stockham_stage<3>(src, dst, nlines, ls, pl.n, ns, tw_smem, inv, tid, nthr); break;
      default: stockham_stage<5>(src, dst, nlines, ls, pl.n, ns, tw_smem, inv, tid, nthr); break;
    }
    __syncthreads();
    ns *= R;
    double2* t = src;
    src = dst;
    dst = t;
  }
  return src;
}

HE_D void load_twiddles(double2* tw_smem, const LinePlan& pl) {
  const int tid = threadIdx.x + blockDim.x * threadIdx.y;
  const int nthr = blockDim.x * blockDim.y;
  for (int m = tid; m < pl.n; m += nthr) tw_smem[m] = pl.tw[m];
}

}  // namespace he
