// fft_kernels.cuh -- pencil passes of the mean-field convolutions (binary64).
//
// x pass (k_xpass): CTA = RB consecutive rows (y,z) of the grid; rows are contiguous in HBM.
//   R2C: two real rows are packed as one complex line (a + i b), transformed, and split with
//        A[k] = (Z[k] + conj Z[n-k]) / 2, B[k] = -i (Z[k] - conj Z[n-k]) / 2.
//   C2R: two half-spectrum rows are packed as Z = A + i B with Hermitian extension (the imaginary
//        parts of k = 0 and k = n/2 are dropped, as FFTW's c2r does), inverse-transformed, and
//        the real and imaginary parts are the two real rows.
//   The modes fuse poten's pointwise work (Dynamics_TDDFT/poten.f90:131-218):
//     X_R2C_DEN    fden row spectrum of den
//     X_R2C_CORR   spectrum of den*dencg*(cp4+cpp4*dencg)                          (:166-168)
//     X_C2R2       dencg = C2R(A)*renor, delj4 = C2R(B)*renor                      (:142,:154)
//     X_C2R2_CORR  the same, then the R2C of the correlation source into A         (:166-171)
//     X_C2R_POT    sto1 = C2R(A)*renor, penalty, pot4 assembly (+ potx4 of the quantum
//                  impurities when extra is set, + ualphas when extra2 is set)     (:178-218)
//     X_C2R1       out1 = C2R(A)*renor (rows 2p, 2p+1 packed in one line)
// y/z pass (k_ypass, k_zconv): CTA = TKX consecutive kx of one pencil family, staged transposed
//   in shared memory (odd line stride to spread banks).  The z pass does forward z, the k-space
//   multiply by one or two real kernels (wcgk, fvlj4), and the inverse z, and can store the
//   forward spectrum (fden) on the way.
// Every kernel is instantiated for a compile-time line length N (the common grid sizes) and for
// N = 0 (run-time length, other admissible sizes).
#pragma once
#include "fft.cuh"

namespace he {

enum XMode { X_R2C_DEN = 0, X_R2C_CORR = 1, X_C2R2 = 2, X_C2R2_CORR = 3, X_C2R_POT = 4, X_C2R1 = 5 };

// Rows per x-pass CTA and kx columns per y/z-pass CTA for the run-time-length kernels (the
// compile-time kernels take the tile as a template parameter, 16 or 8, picked per context by
// the autotuner; a CTA has 16 threads per tile line).
HE_HD constexpr int tile_rows(int n) { return n <= 256 ? 16 : 8; }
HE_HD constexpr int tile_threads(int tile) { return tile * 16; }
// Line stride in shared memory: the line length rounded up to a multiple of 8, plus one (odd, so
// the transposing gathers of consecutive lines spread over the banks).
HE_HD constexpr int line_stride(int n) { return ((n + 7) / 8) * 8 + 1; }

struct XArgs {
  int nx, nxh;
  long rows;                 // ny*nz
  int rb;                    // rows per CTA (even)
  LinePlan pl;
  const double* den;         // prologue / epilogue inputs
  const double* dencg_in;
  const double* delj4_in;
  double2* specA;            // spectrum in / out
  const double2* specB;
  double* out1;              // dencg  (C2R2*) or pot4 (C2R_POT)
  double* out2;              // delj4  (C2R2*)
  const double* extra;       // C2R_POT: potx4 added after the correlation term (null: none)
  const double* extra2;      // C2R_POT: ualphas (alpha_s term) added next (null: none)
  double renor, cp4, cpp4, a0, a1;
  int lsolid;
  double C, beta, den_m;
};

HE_D double corr_source(double den, double dcg, double cp4, double cpp4) {
  return den * dcg * (cp4 + cpp4 * dcg);
}

// Hermitian-extended packed value Z[k] = A[k] + i B[k] of two half-spectrum rows.
HE_D double2 packed_c2r(const double2* ra, const double2* rb, int k, int n) {
  const int nh = n / 2;
  if (k <= nh) {
    double2 a = ra[k], b = rb[k];
    if (k == 0 || k == nh) { a.y = 0.0; b.y = 0.0; }
    return make_double2(a.x - b.y, a.y + b.x);
  }
  double2 a = ra[n - k], b = rb[n - k];
  return make_double2(a.x + b.y, -a.y + b.x);
}

// Split a transformed packed line into the half spectra of its real and imaginary rows.
template <int N>
HE_D double2 split_r2c(const double2* L, int k, int n, bool second) {
  const double2 z = L[sw<N>(k)];
  const double2 zc = cconj(L[sw<N>((n - k) % n)]);
  if (!second) return make_double2(0.5 * (z.x + zc.x), 0.5 * (z.y + zc.y));
  return make_double2(0.5 * (z.y - zc.y), -0.5 * (z.x - zc.x));
}

template <int MODE, int N, int TILE>
__global__ void __launch_bounds__(tile_threads(TILE)) k_xpass(const XArgs a) {
  extern __shared__ double2 smem[];
  const int n = (N > 0) ? N : a.nx;
  const int nxh = n / 2 + 1;
  const int ls = line_stride(n);
  const int RB = (N > 0) ? TILE : a.rb;
  const int tid = threadIdx.x, nthr = blockDim.x;
  const long r0 = (long)blockIdx.x * RB;
  double2* tw = smem;
  double2* P0 = smem + ((a.pl.stw_len + 1) & ~1);
  double2* P1 = P0 + RB * ls;
  load_twiddles(tw, a.pl);

  if constexpr (MODE == X_R2C_DEN || MODE == X_R2C_CORR) {
    const long g0 = r0 * n;
    for (int e = tid; e < RB * n; e += nthr) {
      const int row = e / n, x = e - row * n;
      double v = a.den[g0 + e];
      if constexpr (MODE == X_R2C_CORR) v = corr_source(v, a.dencg_in[g0 + e], a.cp4, a.cpp4);
      reinterpret_cast<double*>(&P0[(row >> 1) * ls + sw<N>(x)])[row & 1] = v;
    }
    __syncthreads();
    double2* R = fft_lines<N>(P0, P1, RB / 2, ls, a.pl, tw, false);
    for (int e = tid; e < RB * nxh; e += nthr) {
      const int row = e / nxh, k = e - row * nxh;
      a.specA[(r0 + row) * nxh + k] = split_r2c<N>(R + (row >> 1) * ls, k, n, row & 1);
    }
    return;
  }

  if constexpr (MODE == X_C2R2 || MODE == X_C2R2_CORR) {
    for (int e = tid; e < RB * n; e += nthr) {
      const int row = e / n, k = e - row * n;
      const double2* ra = a.specA + (r0 + row) * nxh;
      const double2* rbp = a.specB + (r0 + row) * nxh;
      P0[row * ls + sw<N>(k)] = packed_c2r(ra, rbp, k, n);
    }
    __syncthreads();
    double2* R = fft_lines<N>(P0, P1, RB, ls, a.pl, tw, true);
    double2* O = (R == P0) ? P1 : P0;
    for (int e = tid; e < RB * n; e += nthr) {
      const int row = e / n, x = e - row * n;
      const long g = (r0 + row) * n + x;
      const double2 z = R[row * ls + sw<N>(x)];
      const double dcg = z.x * a.renor;
      a.out1[g] = dcg;
      a.out2[g] = z.y * a.renor;
      if constexpr (MODE == X_C2R2_CORR)
        reinterpret_cast<double*>(&O[(row >> 1) * ls + sw<N>(x)])[row & 1] =
            corr_source(a.den[g], dcg, a.cp4, a.cpp4);
    }
    if constexpr (MODE == X_C2R2) return;
    __syncthreads();
    double2* S = (O == P0) ? P1 : P0;
    double2* R2 = fft_lines<N>(O, S, RB / 2, ls, a.pl, tw, false);
    for (int e = tid; e < RB * nxh; e += nthr) {
      const int row = e / nxh, k = e - row * nxh;
      a.specA[(r0 + row) * nxh + k] = split_r2c<N>(R2 + (row >> 1) * ls, k, n, row & 1);
    }
    return;
  }

  if constexpr (MODE == X_C2R_POT || MODE == X_C2R1) {
    // rows 2p and 2p+1 share complex line p
    for (int e = tid; e < (RB / 2) * n; e += nthr) {
      const int p = e / n, k = e - p * n;
      const double2* ra = a.specA + (r0 + 2 * p) * nxh;
      const double2* rbp = a.specA + (r0 + 2 * p + 1) * nxh;
      P0[p * ls + sw<N>(k)] = packed_c2r(ra, rbp, k, n);
    }
    __syncthreads();
    double2* R = fft_lines<N>(P0, P1, RB / 2, ls, a.pl, tw, true);
    for (int e = tid; e < RB * n; e += nthr) {
      const int row = e / n, x = e - row * n;
      const long g = (r0 + row) * n + x;
      const double2 z = R[(row >> 1) * ls + sw<N>(x)];
      const double sto1 = ((row & 1) ? z.y : z.x) * a.renor;
      if constexpr (MODE == X_C2R1) {
        a.out1[g] = sto1;
        continue;
      }
      const double dc = a.dencg_in[g];
      double pot = a.delj4_in[g] + dc * dc * (a.a0 + a.a1 * dc) + sto1;
      if (a.extra) pot = pot + a.extra[g];
      if (a.extra2) pot = pot + a.extra2[g];
      if (a.lsolid) {
        const double d = a.den[g];
        const double t = tanh(a.beta * (d - a.den_m));
        pot = pot + a.C * (1.0 + t + a.beta * d * (1.0 - t * t));
      }
      a.out1[g] = pot;
    }
  }
}

struct YZArgs {
  int nxh, ny, nz;
  int tkx;
  LinePlan pl;               // along y (k_ypass) or z (k_zconv)
  double2* arr[2];           // k_ypass: arrays transformed in place (blockIdx.z picks)
  bool inv;
  // k_zconv
  double2* io;               // input spectrum (after x,y); receives out1 in place
  double2* out2;             // second output (may be null)
  double2* fden_out;         // forward spectrum store (may be null)
  const double* k1;
  const double* k2;          // null: single kernel
};

template <int N, int TILE>
__global__ void __launch_bounds__(tile_threads(TILE)) k_ypass(const YZArgs a) {
  extern __shared__ double2 smem[];
  const int n = (N > 0) ? N : a.ny;
  const int ls = line_stride(n);
  const int TK = (N > 0) ? TILE : a.tkx;
  const int nxh = a.nxh;
  const int tid = threadIdx.x, nthr = blockDim.x;
  const int kx0 = blockIdx.x * TK;
  const int z = blockIdx.y;
  double2* arr = a.arr[blockIdx.z];
  double2* tw = smem;
  double2* P0 = smem + ((a.pl.stw_len + 1) & ~1);
  double2* P1 = P0 + TK * ls;
  load_twiddles(tw, a.pl);
  const long base = (long)nxh * n * z;
  for (int e = tid; e < TK * n; e += nthr) {
    const int j = e / TK, c = e - j * TK;
    const int kx = kx0 + c;
    P0[c * ls + sw<N>(j)] = (kx < nxh) ? arr[base + kx + (long)nxh * j] : make_double2(0.0, 0.0);
  }
  __syncthreads();
  double2* R = fft_lines<N>(P0, P1, TK, ls, a.pl, tw, a.inv);
  for (int e = tid; e < TK * n; e += nthr) {
    const int j = e / TK, c = e - j * TK;
    const int kx = kx0 + c;
    if (kx < nxh) arr[base + kx + (long)nxh * j] = R[c * ls + sw<N>(j)];
  }
}

template <int N, int TILE>
__global__ void __launch_bounds__(tile_threads(TILE)) k_zconv(const YZArgs a) {
  extern __shared__ double2 smem[];
  const int n = (N > 0) ? N : a.nz;
  const int ls = line_stride(n);
  const int TK = (N > 0) ? TILE : a.tkx;
  const int nxh = a.nxh;
  const int tid = threadIdx.x, nthr = blockDim.x;
  const int kx0 = blockIdx.x * TK;
  const int ky = blockIdx.y;
  double2* tw = smem;
  double2* P0 = smem + ((a.pl.stw_len + 1) & ~1);
  double2* P1 = P0 + TK * ls;
  double2* P2 = P1 + TK * ls;
  load_twiddles(tw, a.pl);
  const long plane = (long)nxh * a.ny;
  const long base = (long)nxh * ky;
  for (int e = tid; e < TK * n; e += nthr) {
    const int j = e / TK, c = e - j * TK;
    const int kx = kx0 + c;
    P0[c * ls + sw<N>(j)] = (kx < nxh) ? a.io[base + kx + plane * j] : make_double2(0.0, 0.0);
  }
  __syncthreads();
  double2* F = fft_lines<N>(P0, P1, TK, ls, a.pl, tw, false);
  double2* O = (F == P0) ? P1 : P0;
  for (int e = tid; e < TK * n; e += nthr) {
    const int j = e / TK, c = e - j * TK;
    const int kx = kx0 + c;
    const int s = c * ls + sw<N>(j);
    if (kx >= nxh) {
      F[s] = make_double2(0.0, 0.0);
      if (a.k2) P2[s] = make_double2(0.0, 0.0);
      continue;
    }
    const long g = base + kx + plane * j;
    const double2 f = F[s];
    if (a.fden_out) a.fden_out[g] = f;
    if (a.k2) {
      const double w2 = a.k2[g];
      P2[s] = make_double2(f.x * w2, f.y * w2);
    }
    const double w1 = a.k1[g];
    F[s] = make_double2(f.x * w1, f.y * w1);
  }
  __syncthreads();
  double2* R1 = fft_lines<N>(F, O, TK, ls, a.pl, tw, true);
  for (int e = tid; e < TK * n; e += nthr) {
    const int j = e / TK, c = e - j * TK;
    const int kx = kx0 + c;
    if (kx < nxh) a.io[base + kx + plane * j] = R1[c * ls + sw<N>(j)];
  }
  if (!a.k2) return;
  __syncthreads();
  double2* S = (R1 == F) ? O : F;
  double2* R2 = fft_lines<N>(P2, S, TK, ls, a.pl, tw, true);
  for (int e = tid; e < TK * n; e += nthr) {
    const int j = e / TK, c = e - j * TK;
    const int kx = kx0 + c;
    if (kx < nxh) a.out2[base + kx + plane * j] = R2[c * ls + sw<N>(j)];
  }
}

}  // namespace he
