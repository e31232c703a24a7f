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
// memory (ping-pong buffers).
//
// Two instantiations of the line transform: for the common lengths the length N is a template
// parameter, so the per-butterfly index arithmetic uses constant divisors, the stages unroll,
// each stage reads its own twiddle table laid out [r-1][k] (consecutive threads read consecutive
// twiddles), and line storage is swizzled (element i lives at i ^ ((i>>3)&7)) so that both the
// strided and the contiguous side of every stage hit distinct shared-memory banks.  Other
// admissible lengths use the same algorithm with run-time sizes.
#pragma once
#include "common.cuh"

namespace he {

constexpr int kMaxStages = 12;

struct LinePlan {
  int n;                 // line length
  int nst;               // number of radix stages
  int rad[kMaxStages];   // radix of each stage
  const double2* tw;     // device table exp(-2 pi i m / n), m = 0..n-1
  const double2* stw;    // per-stage twiddles [stage][r-1][k], k < ns(stage)
  int stw_len;           // entries in stw
  const double2* tw2;    // register y pass (fft_reg.cuh): W_N^(a k1) at [k1 N2 + a], N entries
  const float2* stwf;    // binary32 copies of stw and tw2 (the mixed-precision chain)
  const float2* tw2f;
};

// Greedy radix choice shared by host and device: 8, then 4, 2, 3, 5.
HE_HD constexpr int radix_of(int m) {
  return (m % 8 == 0) ? 8 : (m % 4 == 0) ? 4 : (m % 2 == 0) ? 2 : (m % 3 == 0) ? 3 : (m % 5 == 0) ? 5 : 1;
}
HE_HD constexpr int radix_at(int n, int s) {
  int m = n;
  for (int st = 0; st < s; ++st) m /= radix_of(m);
  return radix_of(m);
}
HE_HD constexpr int num_stages(int n) {
  int m = n, s = 0;
  while (m > 1 && radix_of(m) > 1) { m /= radix_of(m); ++s; }
  return s;
}
// Offset of stage s's twiddles in the per-stage table: sum over earlier stages of (R-1)*ns.
HE_HD constexpr int stw_offset(int n, int s) {
  int off = 0, ns = 1, m = n;
  for (int st = 0; st < s; ++st) {
    const int R = radix_of(m);
    off += (R - 1) * ns;
    ns *= R;
    m /= R;
  }
  return off;
}
// Line storage swizzle (identity unless N is a multiple of 8).
template <int N>
HE_HD constexpr int sw(int i) {
  if constexpr (N > 0 && N % 8 == 0) return i ^ ((i >> 3) & 7);
  else return i;
}

// Radix-R DFT in registers on double2 or float2 (the mixed-precision chain); inv selects exp(+i).
template <int R, typename C>
HE_D void dft(C* v, bool inv) {
  using Rt = decltype(v[0].x);
  using X = Cx<Rt>;
  if constexpr (R == 2) {
    const C a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  } else if constexpr (R == 4) {
    const C t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]);
    const C t2 = cadd(v[1], v[3]), u = csub(v[1], v[3]);
    const C mu = inv ? cpi(u) : cmi(u);  // exp(-+ i pi/2) * u
    v[0] = cadd(t0, t2);
    v[2] = csub(t0, t2);
    v[1] = cadd(t1, mu);
    v[3] = csub(t1, mu);
  } else if constexpr (R == 8) {
    const Rt r = Rt(0.70710678118654752440);  // 1/sqrt(2)
    C e[4] = {v[0], v[2], v[4], v[6]};
    C o[4] = {v[1], v[3], v[5], v[7]};
    dft<4>(e, inv);
    dft<4>(o, inv);
    // twiddles exp(-+ 2 pi i k / 8), k = 0..3
    const C w1 = inv ? X::make(r, r) : X::make(r, -r);
    const C o1 = cmul(o[1], w1);
    const C o2 = inv ? cpi(o[2]) : cmi(o[2]);
    const C w3 = inv ? X::make(-r, r) : X::make(-r, -r);
    const C o3 = cmul(o[3], w3);
    v[0] = cadd(e[0], o[0]);
    v[4] = csub(e[0], o[0]);
    v[1] = cadd(e[1], o1);
    v[5] = csub(e[1], o1);
    v[2] = cadd(e[2], o2);
    v[6] = csub(e[2], o2);
    v[3] = cadd(e[3], o3);
    v[7] = csub(e[3], o3);
  } else if constexpr (R == 3) {
    const Rt c = Rt(-0.5), sn = Rt(0.86602540378443864676);  // cos, sin of 2 pi / 3
    const C t = cadd(v[1], v[2]), d = csub(v[1], v[2]);
    const C m = X::make(v[0].x + c * t.x, v[0].y + c * t.y);
    const C sd = cscale(sn, d);
    const C isd = inv ? cpi(sd) : cmi(sd);
    v[0] = cadd(v[0], t);
    v[1] = cadd(m, isd);
    v[2] = csub(m, isd);
  } else {
    static_assert(R == 5, "radix");
    const Rt c1 = Rt(0.30901699437494742410), c2 = Rt(-0.80901699437494742410);
    const Rt s1 = Rt(0.95105651629515357212), s2 = Rt(0.58778525229247312917);
    const C t1 = cadd(v[1], v[4]), t2 = cadd(v[2], v[3]);
    const C d1 = csub(v[1], v[4]), d2 = csub(v[2], v[3]);
    const C a1 = X::make(v[0].x + c1 * t1.x + c2 * t2.x, v[0].y + c1 * t1.y + c2 * t2.y);
    const C a2 = X::make(v[0].x + c2 * t1.x + c1 * t2.x, v[0].y + c2 * t1.y + c1 * t2.y);
    const C b1 = X::make(s1 * d1.x + s2 * d2.x, s1 * d1.y + s2 * d2.y);
    const C b2 = X::make(s2 * d1.x - s1 * d2.x, s2 * d1.y - s1 * d2.y);
    const C ib1 = inv ? cpi(b1) : cmi(b1);
    const C ib2 = inv ? cpi(b2) : cmi(b2);
    v[0] = cadd(v[0], cadd(t1, t2));
    v[1] = cadd(a1, ib1);
    v[4] = csub(a1, ib1);
    v[2] = cadd(a2, ib2);
    v[3] = csub(a2, ib2);
  }
}

// ---- compile-time length ------------------------------------------------------------------------
template <int N, int R, int NS, typename C>
HE_D void stage_t(const C* __restrict__ src, C* __restrict__ dst, int nlines, int ls,
                  const C* __restrict__ stw, bool inv, int tid, int nthr) {
  constexpr int NR = N / R;
  const int total = nlines * NR;
  for (int w = tid; w < total; w += nthr) {
    const int line = w / NR;
    const int j = w - line * NR;
    const int k = j % NS;
    const C* s = src + line * ls;
    C* d = dst + line * ls;
    C v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const C x = s[sw<N>(j + r * NR)];
      if constexpr (NS == 1) v[r] = x;
      else v[r] = (r == 0) ? x : cmul_conj_if(x, stw[(r - 1) * NS + k], inv);
    }
    dft<R>(v, inv);
    const int base = (j / NS) * NS * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) d[sw<N>(base + r * NS)] = v[r];
  }
}

template <int N, int S, int NS, typename C>
HE_D C* stages_t(C* src, C* dst, int nlines, int ls, const C* stw, bool inv, int tid, int nthr) {
  if constexpr (S >= num_stages(N)) {
    return src;
  } else {
    constexpr int R = radix_at(N, S);
    stage_t<N, R, NS>(src, dst, nlines, ls, stw + stw_offset(N, S), inv, tid, nthr);
    __syncthreads();
    return stages_t<N, S + 1, NS * R>(dst, src, nlines, ls, stw, inv, tid, nthr);
  }
}

// ---- run-time length ------------------------------------------------------------------------------
template <int R, typename C>
HE_D void stage_rt(const C* __restrict__ src, C* __restrict__ dst, int nlines, int ls,
                   int n, int ns, const C* __restrict__ stw, bool inv, int tid, int nthr) {
  const int nr = n / R;
  const int total = nlines * nr;
  for (int w = tid; w < total; w += nthr) {
    const int line = w / nr;
    const int j = w - line * nr;
    const int k = j % ns;
    const C* s = src + line * ls;
    C* d = dst + line * ls;
    C v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const C x = s[j + r * nr];
      v[r] = (r == 0 || ns == 1) ? x : cmul_conj_if(x, stw[(r - 1) * ns + k], inv);
    }
    dft<R>(v, inv);
    const int base = (j / ns) * ns * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) d[base + r * ns] = v[r];
  }
}

// Transform 'nlines' lines held in buffer a (b is scratch of the same size); N = 0 selects the
// run-time length pl.n.  Returns the buffer holding the result; ends with __syncthreads().
template <int N, typename C>
HE_D C* fft_lines(C* a, C* b, int nlines, int ls, const LinePlan& pl, const C* stw_smem, bool inv) {
  const int tid = threadIdx.x + blockDim.x * threadIdx.y;
  const int nthr = blockDim.x * blockDim.y;
  if constexpr (N > 0) {
    return stages_t<N, 0, 1>(a, b, nlines, ls, stw_smem, inv, tid, nthr);
  } else {
    C* src = a;
    C* dst = b;
    int ns = 1, off = 0;
    for (int s = 0; s < pl.nst; ++s) {
      const int R = pl.rad[s];
      const C* st = stw_smem + off;
      switch (R) {
        case 8: stage_rt<8>(src, dst, nlines, ls, pl.n, ns, st, inv, tid, nthr); break;
        case 4: stage_rt<4>(src, dst, nlines, ls, pl.n, ns, st, inv, tid, nthr); break;
        case 2: stage_rt<2>(src, dst, nlines, ls, pl.n, ns, st, inv, tid, nthr); break;
        case 3: stage_rt<3>(src, dst, nlines, ls, pl.n, ns, st, inv, tid, nthr); break;
        default: stage_rt<5>(src, dst, nlines, ls, pl.n, ns, st, inv, tid, nthr); break;
      }
      __syncthreads();
      off += (R - 1) * ns;
      ns *= R;
      C* t = src;
      src = dst;
      dst = t;
    }
    return src;
  }
}

HE_D void load_twiddles(double2* stw_smem, const LinePlan& pl) {
  const int tid = threadIdx.x + blockDim.x * threadIdx.y;
  const int nthr = blockDim.x * blockDim.y;
  for (int m = tid; m < pl.stw_len; m += nthr) stw_smem[m] = pl.stw[m];
}
HE_D void load_twiddles(float2* stw_smem, const LinePlan& pl) {
  const int tid = threadIdx.x + blockDim.x * threadIdx.y;
  const int nthr = blockDim.x * blockDim.y;
  for (int m = tid; m < pl.stw_len; m += nthr) stw_smem[m] = pl.stwf[m];
}

}  // namespace he
