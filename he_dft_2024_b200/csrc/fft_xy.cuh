// fft_xy.cuh -- the x and y passes of one z-plane fused in shared memory (binary32 chain, square
// x-y planes up to 128 x 128).
//
// In binary32 a whole z-plane of the half spectrum ((nx/2+1) x ny complex, 66.5 KB at 128^2)
// fits in shared memory, so one CTA per plane can run the y transform and the x transform back
// to back and hand the next pass a spectrum that has already been transformed in both
// directions.  The field evaluation then takes 5 launches instead of 9 (the four y passes
// disappear) and the spectra make two trips through L2/HBM fewer per convolution:
//   k_xy_r2c        den plane -> R2C along x -> forward y -> spectrum plane          (x R2C + y)
//   k_xy_c2r2_corr  spectra A, B -> inverse y -> C2R along x -> dencg, delj4; correlation
//                   source -> R2C along x -> forward y -> spectrum             (y + x + y)
//   k_xy_c2r_pot    spectrum -> inverse y -> C2R along x -> pot4 assembly       (y + x)
// Each line transform runs in place in shared memory as two register phases (N = N1 x N2, the
// split and twiddle table of fft_reg.cuh), the exchange written back over the line itself: a
// CTA holds the plane and a small work area, nothing else.  The pointwise prologue/epilogue
// arithmetic is that of k_xpass (binary64 arithmetic on binary32 fields).
#pragma once
#include "fft_reg.cuh"

namespace he {

constexpr int kXYThreads = 512;
constexpr int kXYChunk = 32;  // rows per chunk of the C2R/correlation kernel's x work area

// In-place transform of `nlines` lines of length N held in shared memory (element j of line l at
// base[l * ls + j * es]) by the whole CTA.  Phase A: task (l, a) loads x[a + N2 m], DFT_N1,
// twiddle W_N^(a k1), and after a barrier writes the results over positions k1 N2 + a; phase B:
// task (l, k1) loads positions k1 N2 + q, DFT_N2, and after a barrier writes X[k1 + N1 k2].
// MA and MB bound the phase-A and phase-B tasks per thread.
template <int N, bool INV, int MA, int MB>
HE_D void xy_lines(float2* base, int nlines, int ls, int es, const float2* __restrict__ tw2) {
  constexpr int N1 = Split<N>::N1, N2 = Split<N>::N2;
  const int tid = threadIdx.x, nthr = blockDim.x;
  {
    float2 v[MA][N1];
    const int ta = nlines * N2;
#pragma unroll
    for (int k = 0; k < MA; ++k) {
      const int t = tid + k * nthr;
      if (t < ta) {
        const int l = t / N2, a = t - l * N2;
        const float2* L = base + l * ls;
#pragma unroll
        for (int m = 0; m < N1; ++m) v[k][m] = L[(a + N2 * m) * es];
        RDft<N1, INV>::run(v[k]);
#pragma unroll
        for (int k1 = 1; k1 < N1; ++k1) v[k][k1] = cmul_conj_if(v[k][k1], __ldg(&tw2[k1 * N2 + a]), INV);
      }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < MA; ++k) {
      const int t = tid + k * nthr;
      if (t < ta) {
        const int l = t / N2, a = t - l * N2;
        float2* L = base + l * ls;
#pragma unroll
        for (int k1 = 0; k1 < N1; ++k1) L[(k1 * N2 + a) * es] = v[k][k1];
      }
    }
    __syncthreads();
  }
  {
    float2 u[MB][N2];
    const int tb = nlines * N1;
#pragma unroll
    for (int k = 0; k < MB; ++k) {
      const int t = tid + k * nthr;
      if (t < tb) {
        const int l = t / N1, k1 = t - l * N1;
        const float2* L = base + l * ls;
#pragma unroll
        for (int q = 0; q < N2; ++q) u[k][q] = L[(k1 * N2 + q) * es];
        RDft<N2, INV>::run(u[k]);
      }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < MB; ++k) {
      const int t = tid + k * nthr;
      if (t < tb) {
        const int l = t / N1, k1 = t - l * N1;
        float2* L = base + l * ls;
#pragma unroll
        for (int k2 = 0; k2 < N2; ++k2) L[(k1 + N1 * k2) * es] = u[k][k2];
      }
    }
    __syncthreads();
  }
}

// Task bounds per thread for `lines` lines of length N.
template <int N>
HE_HD constexpr int xy_ma(int lines) { return (lines * Split<N>::N2 + kXYThreads - 1) / kXYThreads; }
template <int N>
HE_HD constexpr int xy_mb(int lines) { return (lines * Split<N>::N1 + kXYThreads - 1) / kXYThreads; }

// Transform of all columns (kx) of a spectrum plane along y (line kx, element ky at kx + ky*NH).
template <int N, bool INV>
HE_D void xy_columns(float2* W, const float2* __restrict__ twy) {
  constexpr int NH = N / 2 + 1;
  xy_lines<N, INV, xy_ma<N>(NH), xy_mb<N>(NH)>(W, NH, 1, NH, twy);
}

// Split of a transformed packed line (rows 2p + i 2p+1) into its two half-spectrum rows, written
// to rowA[k] and rowB[k] (k <= N/2), as split_r2c without the swizzle.
HE_D void xy_split(float2 z, float2 zc_src, float2& A, float2& B) {
  const float2 zc = cconj(zc_src);
  A = make_float2(0.5f * (z.x + zc.x), 0.5f * (z.y + zc.y));
  B = make_float2(0.5f * (z.y - zc.y), -0.5f * (z.x - zc.x));
}

struct XYArgs {
  const float* den;       // R2C input; correlation source and solid penalty input
  const float* dencg_in;  // pot4 assembly inputs
  const float* delj4_in;
  const float* extra;     // potx4 (quantum) or null
  const float* extra2;    // ualphas or null
  float2* specA;          // spectrum in / out
  const float2* specB;
  float* out1;            // dencg (C2R2) or pot4 (C2R_POT)
  float* out2;            // delj4
  const float2* twx;      // W_N^(a k1) tables of the x and y plans (binary32)
  const float2* twy;
  double renor, renor1, cp4, cpp4, a0, a1;
  int lsolid;
  double C, beta, den_m;
};

// den plane -> forward x (R2C, two rows per complex line) -> forward y -> spectrum plane.
template <int N>
__global__ void __launch_bounds__(kXYThreads) k_xy_r2c(const XYArgs a)
#ifdef HE_KERNEL_TU
{
  pdl_wait_and_trigger();
  constexpr int NH = N / 2 + 1, P = 2 * NH, NP = N / 2;
  float2* W = smem_as<float2>();  // NP packed lines of pitch P = rows of pitch NH
  const int tid = threadIdx.x, nthr = blockDim.x;
  const long z = blockIdx.x;
  const float* d = a.den + z * (long)N * N;
  for (int e = tid; e < NP * N; e += nthr) {
    const int p = e / N, x = e - p * N;
    W[p * P + x] = make_float2(d[(2 * p) * N + x], d[(2 * p + 1) * N + x]);
  }
  __syncthreads();
  xy_lines<N, false, xy_ma<N>(NP), xy_mb<N>(NP)>(W, NP, P, 1, a.twx);
  {
    constexpr int TS = NP * NH, MS = (TS + kXYThreads - 1) / kXYThreads;
    float2 A[MS], B[MS];
#pragma unroll
    for (int s = 0; s < MS; ++s) {
      const int t = tid + s * nthr;
      if (t < TS) {
        const int p = t / NH, k = t - p * NH;
        xy_split(W[p * P + k], W[p * P + (N - k) % N], A[s], B[s]);
      }
    }
    __syncthreads();
#pragma unroll
    for (int s = 0; s < MS; ++s) {
      const int t = tid + s * nthr;
      if (t < TS) {
        const int p = t / NH, k = t - p * NH;
        W[p * P + k] = A[s];
        W[p * P + NH + k] = B[s];
      }
    }
    __syncthreads();
  }
  xy_columns<N, false>(W, a.twy);
  float2* o = a.specA + z * (long)NH * N;
  for (int e = tid; e < NH * N; e += nthr) o[e] = W[e];
}
#else
;
#endif

// spectrum plane -> inverse y -> C2R along x (rows 2p, 2p+1 in one line) -> pot4 assembly.
template <int N>
__global__ void __launch_bounds__(kXYThreads) k_xy_c2r_pot(const XYArgs a)
#ifdef HE_KERNEL_TU
{
  pdl_wait_and_trigger();
  constexpr int NH = N / 2 + 1, P = 2 * NH, NP = N / 2;
  float2* W = smem_as<float2>();
  const int tid = threadIdx.x, nthr = blockDim.x;
  const long z = blockIdx.x;
  const float2* src = a.specA + z * (long)NH * N;
  for (int e = tid; e < NH * N; e += nthr) W[e] = src[e];
  __syncthreads();
  xy_columns<N, true>(W, a.twy);
  {
    constexpr int TS = NP * N, MS = (TS + kXYThreads - 1) / kXYThreads;
    float2 Z[MS];
#pragma unroll
    for (int s = 0; s < MS; ++s) {
      const int t = tid + s * nthr;
      if (t < TS) {
        const int p = t / N, k = t - p * N;
        Z[s] = packed_c2r(W + (2 * p) * NH, W + (2 * p + 1) * NH, k, N);
      }
    }
    __syncthreads();
#pragma unroll
    for (int s = 0; s < MS; ++s) {
      const int t = tid + s * nthr;
      if (t < TS) {
        const int p = t / N, k = t - p * N;
        W[p * P + k] = Z[s];
      }
    }
    __syncthreads();
  }
  xy_lines<N, true, xy_ma<N>(NP), xy_mb<N>(NP)>(W, NP, P, 1, a.twx);
  const long g0 = z * (long)N * N;
  for (int e = tid; e < N * N; e += nthr) {
    const int r = e / N, x = e - r * N;
    const long g = g0 + e;
    const float2 zz = W[(r >> 1) * P + x];
    const double sto1 = double((r & 1) ? zz.y : zz.x) * a.renor1;
    const double dc = a.dencg_in[g];
    double pot = double(a.delj4_in[g]) + dc * dc * (a.a0 + a.a1 * dc) + sto1;
    if (a.extra) pot = pot + a.extra[g];
    if (a.extra2) pot = pot + a.extra2[g];
    if (a.lsolid) {
      const double dd = a.den[g];
      const double th = tanhf(float(a.beta) * (float(dd) - float(a.den_m)));
      pot = pot + a.C * (1.0 + th + a.beta * dd * (1.0 - th * th));
    }
    a.out1[g] = float(pot);
  }
}
#else
;
#endif

// spectra A, B -> inverse y -> C2R along x (A + iB per row) -> dencg, delj4; correlation source
// -> R2C along x (two rows per line) -> forward y -> spectrum plane (into specA).  The x work is
// done kXYChunk rows at a time in a work area; each chunk's correlation spectrum rows go over the
// A rows that chunk has consumed.
template <int N>
__global__ void __launch_bounds__(kXYThreads) k_xy_c2r2_corr(const XYArgs a)
#ifdef HE_KERNEL_TU
{
  pdl_wait_and_trigger();
  constexpr int NH = N / 2 + 1, CH = kXYChunk < N ? kXYChunk : N;
  float2* WA = smem_as<float2>();
  float2* WB = WA + NH * N;
  float2* WK = WB + NH * N;  // CH lines of pitch N
  const int tid = threadIdx.x, nthr = blockDim.x;
  const long z = blockIdx.x;
  const float2* sa = a.specA + z * (long)NH * N;
  const float2* sb = a.specB + z * (long)NH * N;
  for (int e = tid; e < NH * N; e += nthr) {
    WA[e] = sa[e];
    WB[e] = sb[e];
  }
  __syncthreads();
  xy_columns<N, true>(WA, a.twy);
  xy_columns<N, true>(WB, a.twy);
  const long g0 = z * (long)N * N;
  for (int r0 = 0; r0 < N; r0 += CH) {
    for (int e = tid; e < CH * N; e += nthr) {
      const int rr = e / N, k = e - rr * N;
      WK[rr * N + k] = packed_c2r(WA + (r0 + rr) * NH, WB + (r0 + rr) * NH, k, N);
    }
    __syncthreads();
    xy_lines<N, true, xy_ma<N>(CH), xy_mb<N>(CH)>(WK, CH, N, 1, a.twx);
    constexpr int TS = CH * N, MS = (TS + kXYThreads - 1) / kXYThreads;
    float cs[MS];
#pragma unroll
    for (int s = 0; s < MS; ++s) {
      const int t = tid + s * nthr;
      if (t < TS) {
        const long g = g0 + (long)r0 * N + t;
        const float2 zz = WK[t];
        const double dcg = double(zz.x) * a.renor1;
        a.out1[g] = float(dcg);
        a.out2[g] = float(double(zz.y) * a.renor);
        cs[s] = float(corr_source(a.den[g], dcg, a.cp4, a.cpp4));
      }
    }
    __syncthreads();
#pragma unroll
    for (int s = 0; s < MS; ++s) {
      const int t = tid + s * nthr;
      if (t < TS) {
        const int rr = t / N, x = t - rr * N;
        reinterpret_cast<float*>(&WK[(rr >> 1) * N + x])[rr & 1] = cs[s];
      }
    }
    __syncthreads();
    xy_lines<N, false, xy_ma<N>(CH / 2), xy_mb<N>(CH / 2)>(WK, CH / 2, N, 1, a.twx);
    for (int e = tid; e < (CH / 2) * NH; e += nthr) {
      const int q = e / NH, k = e - q * NH;
      float2 A, B;
      xy_split(WK[q * N + k], WK[q * N + (N - k) % N], A, B);
      WA[(r0 + 2 * q) * NH + k] = A;
      WA[(r0 + 2 * q + 1) * NH + k] = B;
    }
    __syncthreads();
  }
  xy_columns<N, false>(WA, a.twy);
  float2* o = a.specA + z * (long)NH * N;
  for (int e = tid; e < NH * N; e += nthr) o[e] = WA[e];
}
#else
;
#endif

// Dynamic shared memory of the three kernels.
template <int N>
HE_HD constexpr size_t xy_smem_r2c() { return sizeof(float2) * (size_t)(N / 2) * 2 * (N / 2 + 1); }
template <int N>
HE_HD constexpr size_t xy_smem_pot() { return xy_smem_r2c<N>(); }
template <int N>
HE_HD constexpr size_t xy_smem_corr() {
  return sizeof(float2) * (2 * (size_t)(N / 2 + 1) * N + (size_t)(kXYChunk < N ? kXYChunk : N) * N);
}

}  // namespace he
