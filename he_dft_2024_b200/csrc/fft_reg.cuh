// fft_reg.cuh -- y pass of the half spectrum for the common line lengths with the line transform
// held in registers (binary64).  Same result as k_ypass (fft_kernels.cuh): every (kx, z) line of
// the (nx/2+1, ny, nz) array is transformed along y, forward (exp(-i)) or inverse (exp(+i),
// unscaled), in place.
//
// N = N1 * N2, n = a + N2 m, k = k1 + N1 k2:
//   phase A: thread (c, a) loads x[a + N2 m], m < N1, of column kx0 + c straight from HBM/L2
//            (consecutive threads hold consecutive kx: each load instruction reads TK*16
//            contiguous bytes), does the N1-point DFT over m in registers, multiplies by
//            W_N^(a k1) and stores T[k1][a][c] to shared memory;
//   phase B: thread (c, k1) reads T[k1][a][c], a < N2, does the N2-point DFT over a in registers
//            and stores X[k1 + N1 k2] straight to memory.
// One shared-memory exchange per line and no staging copies: the pass is a load, two register
// DFTs and a store per element.  The small DFTs are composed from radix 2, 3, 4, 5 with constant
// twiddles (exact for the quarter turns).
#pragma once
#include "fft_kernels.cuh"

namespace he {

template <int N> struct Split;
template <> struct Split<32> { static constexpr int N1 = 4, N2 = 8; };
template <> struct Split<64> { static constexpr int N1 = 8, N2 = 8; };
template <> struct Split<96> { static constexpr int N1 = 8, N2 = 12; };
template <> struct Split<128> { static constexpr int N1 = 8, N2 = 16; };
template <> struct Split<160> { static constexpr int N1 = 10, N2 = 16; };
template <> struct Split<192> { static constexpr int N1 = 12, N2 = 16; };
template <> struct Split<256> { static constexpr int N1 = 16, N2 = 16; };

// Host-side mirror of Split (0 when n has no register path).
HE_HD constexpr int split_n1(int n) {
  return n == 32 ? 4 : n == 64 ? 8 : n == 96 ? 8 : n == 128 ? 8 : n == 160 ? 10 : n == 192 ? 12 : n == 256 ? 16 : 0;
}

// cos(2 pi j / m), sin(2 pi j / m) for m dividing 16, 12 or 10 (decimal expansions of the
// algebraic values cos(pi/8), cos(pi/6), cos(pi/5), ...).
HE_HD constexpr double c16(int j) {
  switch (((j % 16) + 16) % 16) {
    case 0: return 1.0;
    case 1: case 15: return 0.92387953251128675613;
    case 2: case 14: return 0.70710678118654752440;
    case 3: case 13: return 0.38268343236508977173;
    case 4: case 12: return 0.0;
    case 5: case 11: return -0.38268343236508977173;
    case 6: case 10: return -0.70710678118654752440;
    case 7: case 9: return -0.92387953251128675613;
    default: return -1.0;
  }
}
HE_HD constexpr double c12(int j) {
  switch (((j % 12) + 12) % 12) {
    case 0: return 1.0;
    case 1: case 11: return 0.86602540378443864676;
    case 2: case 10: return 0.5;
    case 3: case 9: return 0.0;
    case 4: case 8: return -0.5;
    case 5: case 7: return -0.86602540378443864676;
    default: return -1.0;
  }
}
HE_HD constexpr double c10(int j) {
  switch (((j % 10) + 10) % 10) {
    case 0: return 1.0;
    case 1: case 9: return 0.80901699437494742410;
    case 2: case 8: return 0.30901699437494742410;
    case 3: case 7: return -0.30901699437494742410;
    case 4: case 6: return -0.80901699437494742410;
    default: return -1.0;
  }
}
HE_HD constexpr double s10(int j) {
  switch (((j % 10) + 10) % 10) {
    case 1: case 4: return 0.58778525229247312917;
    case 2: case 3: return 0.95105651629515357212;
    case 6: case 9: return -0.58778525229247312917;
    case 7: case 8: return -0.95105651629515357212;
    default: return 0.0;
  }
}
HE_HD constexpr double cos2pi(int j, int m) {
  return (16 % m == 0) ? c16(j * (16 / m)) : (12 % m == 0) ? c12(j * (12 / m)) : c10(j * (10 / m));
}
HE_HD constexpr double sin2pi(int j, int m) {
  return (16 % m == 0) ? c16(j * (16 / m) + 12) : (12 % m == 0) ? c12(j * (12 / m) + 9) : s10(j * (10 / m));
}

// x * W_M^E (forward W = exp(-2 pi i E / M); INV conjugates), on double2 or float2.
template <int M, int E, bool INV, typename C>
HE_D C twc(C x) {
  using Rt = decltype(x.x);
  constexpr int e = ((E % M) + M) % M;
  if constexpr (e == 0) return x;
  else if constexpr (2 * e == M) return Cx<Rt>::make(-x.x, -x.y);
  else if constexpr (4 * e == M) return INV ? cpi(x) : cmi(x);
  else if constexpr (4 * e == 3 * M) return INV ? cmi(x) : cpi(x);
  else {
    constexpr double cd = cos2pi(e, M);
    constexpr double sd = INV ? sin2pi(e, M) : -sin2pi(e, M);
    const Rt c = Rt(cd), sn = Rt(sd);
    return Cx<Rt>::make(x.x * c - x.y * sn, x.x * sn + x.y * c);
  }
}

// In-register DFT of length M (natural order in and out) on double2 or float2.
template <int M, bool INV> struct RDft;

template <bool INV> struct RDft<2, INV> {
  template <typename C>
  static HE_D void run(C* v) {
    const C a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  }
};
template <bool INV> struct RDft<3, INV> {
  template <typename C>
  static HE_D void run(C* v) {
    using Rt = decltype(v[0].x);
    const Rt c = Rt(-0.5), sn = Rt(0.86602540378443864676);
    const C t = cadd(v[1], v[2]), d = csub(v[1], v[2]);
    const C m = Cx<Rt>::make(v[0].x + c * t.x, v[0].y + c * t.y);
    const C sd = cscale(sn, d);
    const C isd = INV ? cpi(sd) : cmi(sd);
    v[0] = cadd(v[0], t);
    v[1] = cadd(m, isd);
    v[2] = csub(m, isd);
  }
};
template <bool INV> struct RDft<4, INV> {
  template <typename C>
  static HE_D void run(C* v) {
    const C t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]);
    const C t2 = cadd(v[1], v[3]), u = csub(v[1], v[3]);
    const C mu = INV ? cpi(u) : cmi(u);
    v[0] = cadd(t0, t2);
    v[2] = csub(t0, t2);
    v[1] = cadd(t1, mu);
    v[3] = csub(t1, mu);
  }
};
template <bool INV> struct RDft<5, INV> {
  template <typename C>
  static HE_D void run(C* v) {
    using Rt = decltype(v[0].x);
    using X = Cx<Rt>;
    const Rt c1 = Rt(0.30901699437494742410), c2 = Rt(-0.80901699437494742410);
    const Rt s1 = Rt(0.95105651629515357212), s2 = Rt(0.58778525229247312917);
    const C t1 = cadd(v[1], v[4]), t2 = cadd(v[2], v[3]);
    const C d1 = csub(v[1], v[4]), d2 = csub(v[2], v[3]);
    const C a1 = X::make(v[0].x + c1 * t1.x + c2 * t2.x, v[0].y + c1 * t1.y + c2 * t2.y);
    const C a2 = X::make(v[0].x + c2 * t1.x + c1 * t2.x, v[0].y + c2 * t1.y + c1 * t2.y);
    const C b1 = X::make(s1 * d1.x + s2 * d2.x, s1 * d1.y + s2 * d2.y);
    const C b2 = X::make(s2 * d1.x - s1 * d2.x, s2 * d1.y - s1 * d2.y);
    const C ib1 = INV ? cpi(b1) : cmi(b1);
    const C ib2 = INV ? cpi(b2) : cmi(b2);
    v[0] = cadd(v[0], cadd(t1, t2));
    v[1] = cadd(a1, ib1);
    v[4] = csub(a1, ib1);
    v[2] = cadd(a2, ib2);
    v[3] = csub(a2, ib2);
  }
};

// Composite length A*B with n = a + B m, k = k1 + A k2.
template <int A, int B, bool INV, int AA, int K1, typename C>
HE_D void rdft_tw(const C (&u)[A], C (&t)[A * B]) {
  if constexpr (K1 < A) {
    t[K1 * B + AA] = twc<A * B, AA * K1, INV>(u[K1]);
    rdft_tw<A, B, INV, AA, K1 + 1>(u, t);
  }
}
template <int A, int B, bool INV, int AA = 0, typename C>
HE_D void rdft_rows(const C* v, C (&t)[A * B]) {
  if constexpr (AA < B) {
    C u[A];
#pragma unroll
    for (int m = 0; m < A; ++m) u[m] = v[AA + B * m];
    RDft<A, INV>::run(u);
    rdft_tw<A, B, INV, AA, 0>(u, t);
    rdft_rows<A, B, INV, AA + 1>(v, t);
  }
}
template <int A, int B, bool INV, int K1 = 0, typename C>
HE_D void rdft_cols(C* v, const C (&t)[A * B]) {
  if constexpr (K1 < A) {
    C w[B];
#pragma unroll
    for (int a = 0; a < B; ++a) w[a] = t[K1 * B + a];
    RDft<B, INV>::run(w);
#pragma unroll
    for (int k2 = 0; k2 < B; ++k2) v[K1 + A * k2] = w[k2];
    rdft_cols<A, B, INV, K1 + 1>(v, t);
  }
}
template <int A, int B, bool INV> struct RDftComp {
  template <typename C>
  static HE_D void run(C* v) {
    C t[A * B];
    rdft_rows<A, B, INV>(v, t);
    rdft_cols<A, B, INV>(v, t);
  }
};
template <bool INV> struct RDft<8, INV> : RDftComp<2, 4, INV> {};
template <bool INV> struct RDft<10, INV> : RDftComp<2, 5, INV> {};
template <bool INV> struct RDft<12, INV> : RDftComp<4, 3, INV> {};
template <bool INV> struct RDft<16, INV> : RDftComp<4, 4, INV> {};

// Threads of a y-pass CTA: TK columns x N2.
HE_HD constexpr int yreg_threads(int n, int tk) { return tk * (n / split_n1(n)); }
// Resident CTAs the y pass asks the compiler for: 24 warps per SM where a line's N1 values fit
// without spilling (N1 <= 8; 128: 6 CTAs of 128 threads, 85 registers), no minimum otherwise.
HE_HD constexpr int yreg_min_blocks(int n, int tk) {
  return split_n1(n) <= 8 ? 768 / yreg_threads(n, tk) : 0;
}

template <int N, int TK, bool INV, bool G, typename C>
HE_D void ypass_reg_body(const YZArgs& a, const C* __restrict__ tw2, C* T) {
  using Rt = decltype(T[0].x);
  constexpr int N1 = Split<N>::N1, N2 = Split<N>::N2;
  const int tid = threadIdx.x;
  const int nxh = a.nxh;
  const int kx0 = blockIdx.x * TK;
  // G: blockIdx.z = member x narr + array; otherwise blockIdx.z is the array
  C* arr;
  if constexpr (G) arr = reinterpret_cast<C*>(a.mm(a.arr[blockIdx.z % a.narr], (int)blockIdx.z / a.narr));
  else arr = reinterpret_cast<C*>(a.arr[blockIdx.z]);
  const long base = (long)nxh * N * blockIdx.y;
  {
    const int c = tid % TK, am = tid / TK;  // phase A: column c, a = am
    const int kx = kx0 + c;
    const bool ok = kx < nxh;
    const C* src = arr + base + (ok ? kx : 0) + (long)nxh * am;
    C v[N1];
#pragma unroll
    for (int m = 0; m < N1; ++m) v[m] = ok ? src[(long)nxh * N2 * m] : Cx<Rt>::make(0, 0);
    RDft<N1, INV>::run(v);
#pragma unroll
    for (int k1 = 1; k1 < N1; ++k1) v[k1] = cmul_conj_if(v[k1], __ldg(&tw2[k1 * N2 + am]), INV);
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) T[(k1 * N2 + am) * TK + c] = v[k1];
  }
  __syncthreads();
  if (tid < TK * N1) {
    const int c = tid % TK, k1 = tid / TK;  // phase B: column c, k1
    const int kx = kx0 + c;
    C u[N2];
#pragma unroll
    for (int q = 0; q < N2; ++q) u[q] = T[(k1 * N2 + q) * TK + c];
    RDft<N2, INV>::run(u);
    if (kx < nxh) {
      C* dst = arr + base + kx + (long)nxh * k1;
#pragma unroll
      for (int k2 = 0; k2 < N2; ++k2) dst[(long)nxh * N1 * k2] = u[k2];
    }
  }
}

template <int N, int TK, typename Rt, bool G>
__global__ void __launch_bounds__(yreg_threads(N, TK), yreg_min_blocks(N, TK)) k_ypass_reg(const YZArgs a,
                                                                   const typename Cx<Rt>::T* tw2)
#ifdef HE_KERNEL_TU
{
  pdl_wait_and_trigger();
  using C = typename Cx<Rt>::T;
  C* T = smem_as<C>();
  if (a.inv) ypass_reg_body<N, TK, true, G>(a, tw2, T);
  else ypass_reg_body<N, TK, false, G>(a, tw2, T);
}
#else
;
#endif

// z pass of a convolution with the line transform in registers (N = N1 x N2, TK columns kx):
//   phase A  (thread c, a):  x[kz = a + N2 m] from HBM, DFT_N1 over m, twiddle W_N^(a k1),
//                            exchange through shared memory;
//   phase B  (thread c, k1): DFT_N2 over a -> X[k1 + N1 k2] for all k2 in registers (stored as
//            fden when asked), times the kernel(s), inverse DFT_N2 over k2 -> n2, twiddle
//            W_N^-(n2 k1), exchange;
//   phase A' (thread c, n2): inverse DFT_N1 over k1 -> y[n2 + N2 n1], stored over the input (and
//            into out2).
// The forward spectrum never leaves registers between the two transforms, and a CTA needs one
// (two for two kernels) N x TK exchange buffer instead of three line buffers.
template <int N, int TK, bool G, typename C>
HE_D void zconv_reg_body(const YZArgs& a, int mem, const C* __restrict__ tw2, C* T0, C* T1) {
  using Rt = decltype(T0[0].x);
  using X = Cx<Rt>;
  constexpr bool F32 = sizeof(Rt) == 4;
  constexpr int N1 = Split<N>::N1, N2 = Split<N>::N2;
  const int tid = threadIdx.x;
  const int nxh = a.nxh;
  const int kx0 = blockIdx.x * TK;
  const long plane = (long)nxh * a.ny;
  const long base = (long)nxh * blockIdx.y;
  C* io = reinterpret_cast<C*>(on_member<G>(a.mm, a.io, mem));
  C* out2 = reinterpret_cast<C*>(on_member<G>(a.mm, a.out2, mem));
  C* fden_out = reinterpret_cast<C*>(on_member<G>(a.mm, a.fden_out, mem));
  const double* kern1 = on_member<G>(a.mm, a.k1, mem);
  const double* kern2 = on_member<G>(a.mm, a.k2, mem);
  const float* kern1f = on_member<G>(a.mm, a.k1f, mem);
  const float* kern2f = on_member<G>(a.mm, a.k2f, mem);
  const bool two = F32 ? kern2f != nullptr : kern2 != nullptr;
  {
    const int c = tid % TK, am = tid / TK;
    const int kx = kx0 + c;
    const bool ok = kx < nxh;
    const C* src = io + base + (ok ? kx : 0) + plane * am;
    C v[N1];
#pragma unroll
    for (int m = 0; m < N1; ++m) v[m] = ok ? src[plane * N2 * m] : X::make(0, 0);
    RDft<N1, false>::run(v);
#pragma unroll
    for (int k1 = 1; k1 < N1; ++k1) v[k1] = cmul_conj_if(v[k1], __ldg(&tw2[k1 * N2 + am]), false);
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) T0[(k1 * N2 + am) * TK + c] = v[k1];
  }
  __syncthreads();
  const bool actB = tid < TK * N1;
  const int cB = tid % TK, k1 = tid / TK;
  C u[N2], w[N2];
  if (actB) {
    const int kx = kx0 + cB;
    const bool ok = kx < nxh;
#pragma unroll
    for (int q = 0; q < N2; ++q) u[q] = T0[(k1 * N2 + q) * TK + cB];
    RDft<N2, false>::run(u);
    const long g0 = base + (ok ? kx : 0) + plane * k1;
#pragma unroll
    for (int k2 = 0; k2 < N2; ++k2) {
      const long g = g0 + plane * N1 * k2;
      if (ok && fden_out) fden_out[g] = u[k2];
      if (two) {
        const Rt w2 = ok ? (F32 ? Rt(kern2f[g]) : Rt(kern2[g])) : Rt(0);
        w[k2] = X::make(u[k2].x * w2, u[k2].y * w2);
      }
      const Rt w1 = ok ? (F32 ? Rt(kern1f[g]) : Rt(kern1[g])) : Rt(0);
      u[k2] = X::make(u[k2].x * w1, u[k2].y * w1);
    }
    RDft<N2, true>::run(u);
#pragma unroll
    for (int n2 = 1; n2 < N2; ++n2) u[n2] = cmul_conj_if(u[n2], __ldg(&tw2[k1 * N2 + n2]), true);
    if (two) {
      RDft<N2, true>::run(w);
#pragma unroll
      for (int n2 = 1; n2 < N2; ++n2) w[n2] = cmul_conj_if(w[n2], __ldg(&tw2[k1 * N2 + n2]), true);
    }
  }
  __syncthreads();  // every phase-B thread has read T0
  if (actB) {
#pragma unroll
    for (int n2 = 0; n2 < N2; ++n2) T0[(k1 * N2 + n2) * TK + cB] = u[n2];
    if (two) {
#pragma unroll
      for (int n2 = 0; n2 < N2; ++n2) T1[(k1 * N2 + n2) * TK + cB] = w[n2];
    }
  }
  __syncthreads();
  {
    const int c = tid % TK, n2 = tid / TK;
    const int kx = kx0 + c;
    const bool ok = kx < nxh;
    C v[N1];
#pragma unroll
    for (int q = 0; q < N1; ++q) v[q] = T0[(q * N2 + n2) * TK + c];
    RDft<N1, true>::run(v);
    if (ok) {
      C* dst = io + base + kx + plane * n2;
#pragma unroll
      for (int n1 = 0; n1 < N1; ++n1) dst[plane * N2 * n1] = v[n1];
    }
    if (two) {
#pragma unroll
      for (int q = 0; q < N1; ++q) v[q] = T1[(q * N2 + n2) * TK + c];
      RDft<N1, true>::run(v);
      if (ok) {
        C* dst = out2 + base + kx + plane * n2;
#pragma unroll
        for (int n1 = 0; n1 < N1; ++n1) dst[plane * N2 * n1] = v[n1];
      }
    }
  }
}

template <int N, int TK, typename Rt, bool G>
__global__ void __launch_bounds__(yreg_threads(N, TK)) k_zconv_reg(const YZArgs a,
                                                                   const typename Cx<Rt>::T* tw2)
#ifdef HE_KERNEL_TU
{
  pdl_wait_and_trigger();
  using C = typename Cx<Rt>::T;
  C* T0 = smem_as<C>();
  zconv_reg_body<N, TK, G>(a, G ? (int)blockIdx.z : 0, tw2, T0, T0 + N * TK);  // G: blockIdx.z is the member
}
#else
;
#endif

}  // namespace he
