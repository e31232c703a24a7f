// fft_kernels.cuh -- pencil passes of the mean-field convolutions (binary64, or binary32 in the
// mixed path).
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
  double renor1;             // C2R2 out1 and C2R_POT sto1: renor over the scale of the kernel
                             // that made specA (the mixed chain scales its wcgk copy)
  int lsolid;
  double C, beta, den_m;
  MemberMap mm;              // group members (blockIdx.y is the member)
};

HE_D double corr_source(double den, double dcg, double cp4, double cpp4) {
  return den * dcg * (cp4 + cpp4 * dcg);
}

// Hermitian-extended packed value Z[k] = A[k] + i B[k] of two half-spectrum rows.  hasb = false:
// the second row is zero (the last, unpaired row of an odd row count).  Only the real parts of
// the DC term and, for even n, of the Nyquist term enter a C2R.
template <typename C>
HE_D C packed_c2r(const C* ra, const C* rb, int k, int n, bool hasb = true) {
  using X = Cx<decltype(ra[0].x)>;
  const int nh = n / 2;
  if (k <= nh) {
    C a = ra[k], b = hasb ? rb[k] : X::make(0, 0);
    if (k == 0 || 2 * k == n) { a.y = 0; b.y = 0; }
    return X::make(a.x - b.y, a.y + b.x);
  }
  C a = ra[n - k], b = hasb ? rb[n - k] : X::make(0, 0);
  return X::make(a.x + b.y, -a.y + b.x);
}

// Split a transformed packed line into the half spectra of its real and imaginary rows.
template <int N, typename C>
HE_D C split_r2c(const C* L, int k, int n, bool second) {
  using Rt = decltype(L[0].x);
  using X = Cx<Rt>;
  const C z = L[sw<N>(k)];
  const C zc = cconj(L[sw<N>((n - k) % n)]);
  if (!second) return X::make(Rt(0.5) * (z.x + zc.x), Rt(0.5) * (z.y + zc.y));
  return X::make(Rt(0.5) * (z.y - zc.y), Rt(-0.5) * (z.x - zc.x));
}

// Dynamic shared memory viewed as the chain's complex type.
template <typename C>
HE_D C* smem_as() {
  extern __shared__ __align__(16) unsigned char he_smem_raw[];
  return reinterpret_cast<C*>(he_smem_raw);
}

// Inputs of one row tile that the x pass stages in shared memory: the spectrum rows of the C2R
// modes and the real rows of the R2C prologue / C2R epilogue (the quantum extras are read
// directly).
template <int MODE>
struct XStage {
  static constexpr int nspec = (MODE == X_C2R2 || MODE == X_C2R2_CORR) ? 2
                               : (MODE == X_C2R_POT || MODE == X_C2R1) ? 1 : 0;
  static constexpr int nreal = (MODE == X_R2C_DEN || MODE == X_C2R2_CORR) ? 1
                               : MODE == X_R2C_CORR ? 2 : MODE == X_C2R_POT ? 3 : 0;
};
// Bytes of one staged tile of RB rows (a multiple of 16).
template <int MODE, typename Rt>
HE_HD size_t xstage_bytes(int rb, int n) {
  return (size_t)XStage<MODE>::nspec * rb * (n / 2 + 1) * sizeof(typename Cx<Rt>::T) +
         (size_t)XStage<MODE>::nreal * rb * n * sizeof(Rt);
}
// Dynamic shared memory of an x-pass CTA: twiddles, two line buffers, two staged tiles.
template <int MODE, typename Rt>
HE_HD size_t xpass_smem(int stw_len, int rb, int n) {
  using C = typename Cx<Rt>::T;
  return sizeof(C) * (((size_t)stw_len + 1) / 2 * 2 + 2 * (size_t)rb * line_stride(n)) +
         2 * xstage_bytes<MODE, Rt>(rb, n);
}

// Rt = double: the binary64 chain; Rt = float: the mixed path, spectra, transforms and the
// real-space fields (den, dencg, delj4, pot4) in binary32, the pointwise prologue and epilogue
// arithmetic in binary64.
//
// Persistent and software-pipelined: CTA b transforms row tiles b, b + G, b + 2G, ... (G CTAs);
// while it transforms one tile, the inputs of its next tile are already in flight (cp.async of the
// tile's contiguous row ranges into the other stage buffer), so the load latency that bounds a
// load-transform-store CTA is hidden behind the transform.
constexpr int kXPipeThreads = 256;  // threads of a pipelined x-pass CTA, whatever its rows
template <int MODE, int N, int TILE, typename Rt, bool G>
__global__ void __launch_bounds__(kXPipeThreads) k_xpass(const XArgs a)
#ifdef HE_KERNEL_TU
{
  pdl_wait_and_trigger();
  const int mem = G ? (int)blockIdx.y : 0;  // G: blockIdx.y is the group member
  using C = typename Cx<Rt>::T;
  using Rs = Rt;  // real-space fields: binary64, binary32 in the mixed path
  using ST = XStage<MODE>;
  const Rs* extra = reinterpret_cast<const Rs*>(on_member<G>(a.mm, a.extra, mem));
  const Rs* extra2 = reinterpret_cast<const Rs*>(on_member<G>(a.mm, a.extra2, mem));
  Rs* out1 = reinterpret_cast<Rs*>(on_member<G>(a.mm, a.out1, mem));
  Rs* out2 = reinterpret_cast<Rs*>(on_member<G>(a.mm, a.out2, mem));
  C* smem = smem_as<C>();
  C* specA = reinterpret_cast<C*>(on_member<G>(a.mm, a.specA, mem));
  const C* specB = reinterpret_cast<const C*>(on_member<G>(a.mm, a.specB, mem));
  const int n = (N > 0) ? N : a.nx;
  const int nxh = n / 2 + 1;
  const int ls = line_stride(n);
  const int RB = (N > 0) ? TILE : a.rb;
  const int tid = threadIdx.x, nthr = kXPipeThreads;
  const long ntiles = a.rows / RB;
  C* tw = smem;
  C* P0 = smem + ((a.pl.stw_len + 1) & ~1);
  C* P1 = P0 + RB * ls;
  unsigned char* stage0 = reinterpret_cast<unsigned char*>(P1 + RB * ls);
  const size_t sbytes = xstage_bytes<MODE, Rt>(RB, n);
  const size_t spec_bytes = (size_t)RB * nxh * sizeof(C), real_bytes = (size_t)RB * n * sizeof(Rs);
  // real arrays staged per mode (prologue or epilogue inputs)
  const void* rsrc[3] = {nullptr, nullptr, nullptr};
  if constexpr (MODE == X_R2C_DEN || MODE == X_C2R2_CORR) rsrc[0] = on_member<G>(a.mm, a.den, mem);
  if constexpr (MODE == X_R2C_CORR) { rsrc[0] = on_member<G>(a.mm, a.den, mem); rsrc[1] = on_member<G>(a.mm, a.dencg_in, mem); }
  if constexpr (MODE == X_C2R_POT) { rsrc[0] = on_member<G>(a.mm, a.dencg_in, mem); rsrc[1] = on_member<G>(a.mm, a.delj4_in, mem); rsrc[2] = on_member<G>(a.mm, a.den, mem); }
  const int nreal = (MODE == X_C2R_POT && !a.lsolid) ? 2 : ST::nreal;  // den: penalty only
  auto issue = [&](int buf, long t) {
    unsigned char* st = stage0 + buf * sbytes;
    const long r0 = t * RB;
    if constexpr (ST::nspec >= 1) cp_async_range(st, specA + r0 * nxh, spec_bytes, tid, nthr);
    if constexpr (ST::nspec >= 2) cp_async_range(st + spec_bytes, specB + r0 * nxh, spec_bytes, tid, nthr);
#pragma unroll
    for (int k = 0; k < ST::nreal; ++k)
      if (k < nreal)
        cp_async_range(st + ST::nspec * spec_bytes + k * real_bytes,
                     static_cast<const Rs*>(rsrc[k]) + r0 * n, real_bytes, tid, nthr);
  };
  load_twiddles(tw, a.pl);

  long t = blockIdx.x;
  int buf = 0;
  if (t < ntiles) issue(0, t);
  cp_async_commit();
  for (; t < ntiles; t += gridDim.x, buf ^= 1) {
    if (t + gridDim.x < ntiles) issue(buf ^ 1, t + gridDim.x);
    cp_async_commit();
    cp_async_wait<1>();
    __syncthreads();
    const unsigned char* st = stage0 + buf * sbytes;
    const C* sA = reinterpret_cast<const C*>(st);
    const C* sB = reinterpret_cast<const C*>(st + spec_bytes);
    const Rs* sR0 = reinterpret_cast<const Rs*>(st + ST::nspec * spec_bytes);
    const Rs* sR1 = sR0 + RB * n;
    const Rs* sR2 = sR1 + RB * n;
    const long r0 = t * RB;

    if constexpr (MODE == X_R2C_DEN || MODE == X_R2C_CORR) {
      for (int e = tid; e < RB * n; e += nthr) {
        const int row = e / n, x = e - row * n;
        double v = sR0[e];
        if constexpr (MODE == X_R2C_CORR) v = corr_source(v, sR1[e], a.cp4, a.cpp4);
        reinterpret_cast<Rt*>(&P0[(row >> 1) * ls + sw<N>(x)])[row & 1] = Rt(v);
      }
      __syncthreads();
      C* R = fft_lines<N>(P0, P1, RB / 2, ls, a.pl, tw, false);
      for (int e = tid; e < RB * nxh; e += nthr) {
        const int row = e / nxh, k = e - row * nxh;
        specA[(r0 + row) * nxh + k] = split_r2c<N>(R + (row >> 1) * ls, k, n, row & 1);
      }
    }

    if constexpr (MODE == X_C2R2 || MODE == X_C2R2_CORR) {
      for (int e = tid; e < RB * n; e += nthr) {
        const int row = e / n, k = e - row * n;
        P0[row * ls + sw<N>(k)] = packed_c2r(sA + row * nxh, sB + row * nxh, k, n);
      }
      __syncthreads();
      C* R = fft_lines<N>(P0, P1, RB, ls, a.pl, tw, true);
      C* O = (R == P0) ? P1 : P0;
      for (int e = tid; e < RB * n; e += nthr) {
        const int row = e / n, x = e - row * n;
        const long g = (r0 + row) * n + x;
        const C z = R[row * ls + sw<N>(x)];
        const double dcg = double(z.x) * a.renor1;
        out1[g] = Rs(dcg);
        out2[g] = Rs(double(z.y) * a.renor);
        if constexpr (MODE == X_C2R2_CORR)
          reinterpret_cast<Rt*>(&O[(row >> 1) * ls + sw<N>(x)])[row & 1] =
              Rt(corr_source(sR0[e], dcg, a.cp4, a.cpp4));
      }
      if constexpr (MODE == X_C2R2_CORR) {
        __syncthreads();
        C* S = (O == P0) ? P1 : P0;
        C* R2 = fft_lines<N>(O, S, RB / 2, ls, a.pl, tw, false);
        for (int e = tid; e < RB * nxh; e += nthr) {
          const int row = e / nxh, k = e - row * nxh;
          specA[(r0 + row) * nxh + k] = split_r2c<N>(R2 + (row >> 1) * ls, k, n, row & 1);
        }
      }
    }

    if constexpr (MODE == X_C2R_POT || MODE == X_C2R1) {
      // rows 2p and 2p+1 share complex line p
      for (int e = tid; e < (RB / 2) * n; e += nthr) {
        const int p = e / n, k = e - p * n;
        P0[p * ls + sw<N>(k)] = packed_c2r(sA + (2 * p) * nxh, sA + (2 * p + 1) * nxh, k, n);
      }
      __syncthreads();
      C* R = fft_lines<N>(P0, P1, RB / 2, ls, a.pl, tw, true);
      for (int e = tid; e < RB * n; e += nthr) {
        const int row = e / n, x = e - row * n;
        const long g = (r0 + row) * n + x;
        const C z = R[(row >> 1) * ls + sw<N>(x)];
        if constexpr (MODE == X_C2R1) {
          out1[g] = Rs(double((row & 1) ? z.y : z.x) * a.renor);
        } else {
          const double sto1 = double((row & 1) ? z.y : z.x) * a.renor1;
          const double dc = sR0[e];
          double pot = double(sR1[e]) + dc * dc * (a.a0 + a.a1 * dc) + sto1;
          if (extra) pot = pot + extra[g];
          if (extra2) pot = pot + extra2[g];
          if (a.lsolid) {
            const double d = sR2[e];
            // tanh in the chain's precision (binary32 in the mixed path)
            const double th = tanh(Rt(a.beta) * (Rt(d) - Rt(a.den_m)));
            pot = pot + a.C * (1.0 + th + a.beta * d * (1.0 - th * th));
          }
          out1[g] = Rs(pot);
        }
      }
    }
    __syncthreads();  // stage buf and the line buffers are reused by the next tile
  }
  cp_async_wait<0>();
}
#else
;
#endif

// One-shot variant of k_xpass: one CTA per row tile, loading its inputs straight from global
// memory (no staging buffers, so less shared memory per CTA; the autotuner picks between the two).
template <int MODE, int N, int TILE, typename Rt, bool G>
__global__ void __launch_bounds__(tile_threads(TILE)) k_xpass_c(const XArgs a)
#ifdef HE_KERNEL_TU
{
  pdl_wait_and_trigger();
  const int mem = G ? (int)blockIdx.y : 0;  // G: blockIdx.y is the group member
  using C = typename Cx<Rt>::T;
  using Rs = Rt;  // real-space fields: binary64, binary32 in the mixed path
  const Rs* den = reinterpret_cast<const Rs*>(on_member<G>(a.mm, a.den, mem));
  const Rs* dencg_in = reinterpret_cast<const Rs*>(on_member<G>(a.mm, a.dencg_in, mem));
  const Rs* delj4_in = reinterpret_cast<const Rs*>(on_member<G>(a.mm, a.delj4_in, mem));
  const Rs* extra = reinterpret_cast<const Rs*>(on_member<G>(a.mm, a.extra, mem));
  const Rs* extra2 = reinterpret_cast<const Rs*>(on_member<G>(a.mm, a.extra2, mem));
  Rs* out1 = reinterpret_cast<Rs*>(on_member<G>(a.mm, a.out1, mem));
  Rs* out2 = reinterpret_cast<Rs*>(on_member<G>(a.mm, a.out2, mem));
  C* smem = smem_as<C>();
  C* specA = reinterpret_cast<C*>(on_member<G>(a.mm, a.specA, mem));
  const C* specB = reinterpret_cast<const C*>(on_member<G>(a.mm, a.specB, mem));
  const int n = (N > 0) ? N : a.nx;
  const int nxh = n / 2 + 1;
  const int ls = line_stride(n);
  const int RB = (N > 0) ? TILE : a.rb;
  const int tid = threadIdx.x;
  // compile-time thread count for the compile-time lengths: the element loops below unroll and
  // issue their global loads together
  const int nthr = (N > 0) ? tile_threads(TILE) : (int)blockDim.x;
  const long r0 = (long)blockIdx.x * RB;
  // rows past a.rows (the last tile of an odd row count, run-time lengths only) read as zero and
  // are not stored
  const long rows = a.rows;
  C* tw = smem;
  C* P0 = smem + ((a.pl.stw_len + 1) & ~1);
  C* P1 = P0 + RB * ls;
  load_twiddles(tw, a.pl);

  if constexpr (MODE == X_R2C_DEN || MODE == X_R2C_CORR) {
    const long g0 = r0 * n;
    for (int e = tid; e < RB * n; e += nthr) {
      const int row = e / n, x = e - row * n;
      double v = 0.0;
      if (r0 + row < rows) {
        v = den[g0 + e];
        if constexpr (MODE == X_R2C_CORR) v = corr_source(v, dencg_in[g0 + e], a.cp4, a.cpp4);
      }
      reinterpret_cast<Rt*>(&P0[(row >> 1) * ls + sw<N>(x)])[row & 1] = Rt(v);
    }
    __syncthreads();
    C* R = fft_lines<N>(P0, P1, RB / 2, ls, a.pl, tw, false);
    for (int e = tid; e < RB * nxh; e += nthr) {
      const int row = e / nxh, k = e - row * nxh;
      if (r0 + row < rows)
        specA[(r0 + row) * nxh + k] = split_r2c<N>(R + (row >> 1) * ls, k, n, row & 1);
    }
    return;
  }

  if constexpr (MODE == X_C2R2 || MODE == X_C2R2_CORR) {
    for (int e = tid; e < RB * n; e += nthr) {
      const int row = e / n, k = e - row * n;
      const bool in = r0 + row < rows;
      const C* ra = specA + (in ? r0 + row : 0) * nxh;
      const C* rbp = specB + (in ? r0 + row : 0) * nxh;
      P0[row * ls + sw<N>(k)] = in ? packed_c2r(ra, rbp, k, n) : Cx<Rt>::make(0, 0);
    }
    __syncthreads();
    C* R = fft_lines<N>(P0, P1, RB, ls, a.pl, tw, true);
    C* O = (R == P0) ? P1 : P0;
    for (int e = tid; e < RB * n; e += nthr) {
      const int row = e / n, x = e - row * n;
      const long g = (r0 + row) * n + x;
      const bool in = r0 + row < rows;
      const C z = R[row * ls + sw<N>(x)];
      const double dcg = double(z.x) * a.renor1;
      if (in) {
        out1[g] = Rs(dcg);
        out2[g] = Rs(double(z.y) * a.renor);
      }
      if constexpr (MODE == X_C2R2_CORR)
        reinterpret_cast<Rt*>(&O[(row >> 1) * ls + sw<N>(x)])[row & 1] =
            in ? Rt(corr_source(den[g], dcg, a.cp4, a.cpp4)) : Rt(0);
    }
    if constexpr (MODE == X_C2R2) return;
    __syncthreads();
    C* S = (O == P0) ? P1 : P0;
    C* R2 = fft_lines<N>(O, S, RB / 2, ls, a.pl, tw, false);
    for (int e = tid; e < RB * nxh; e += nthr) {
      const int row = e / nxh, k = e - row * nxh;
      if (r0 + row < rows)
        specA[(r0 + row) * nxh + k] = split_r2c<N>(R2 + (row >> 1) * ls, k, n, row & 1);
    }
    return;
  }

  if constexpr (MODE == X_C2R_POT || MODE == X_C2R1) {
    // rows 2p and 2p+1 share complex line p
    for (int e = tid; e < (RB / 2) * n; e += nthr) {
      const int p = e / n, k = e - p * n;
      const bool ina = r0 + 2 * p < rows, inb = r0 + 2 * p + 1 < rows;
      const C* ra = specA + (ina ? r0 + 2 * p : 0) * nxh;
      const C* rbp = specA + (inb ? r0 + 2 * p + 1 : 0) * nxh;
      P0[p * ls + sw<N>(k)] = ina ? packed_c2r(ra, rbp, k, n, inb) : Cx<Rt>::make(0, 0);
    }
    __syncthreads();
    C* R = fft_lines<N>(P0, P1, RB / 2, ls, a.pl, tw, true);
    for (int e = tid; e < RB * n; e += nthr) {
      const int row = e / n, x = e - row * n;
      if (r0 + row >= rows) continue;
      const long g = (r0 + row) * n + x;
      const C z = R[(row >> 1) * ls + sw<N>(x)];
      if constexpr (MODE == X_C2R1) {
        out1[g] = Rs(double((row & 1) ? z.y : z.x) * a.renor);
        continue;
      }
      const double sto1 = double((row & 1) ? z.y : z.x) * a.renor1;
      const double dc = dencg_in[g];
      double pot = delj4_in[g] + dc * dc * (a.a0 + a.a1 * dc) + sto1;
      if (extra) pot = pot + extra[g];
      if (extra2) pot = pot + extra2[g];
      if (a.lsolid) {
        const double d = den[g];
        const double t = tanh(Rt(a.beta) * (Rt(d) - Rt(a.den_m)));  // binary32 in the mixed path
        pot = pot + a.C * (1.0 + t + a.beta * d * (1.0 - t * t));
      }
      out1[g] = Rs(pot);
    }
  }
}
#else
;
#endif

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
  const float* k1f;          // binary32 copies of k1, k2 (the mixed chain)
  const float* k2f;
  int narr;                  // k_ypass: arrays per member (blockIdx.z = member x narr + array)
  MemberMap mm;              // group members (k_zconv: blockIdx.z is the member)
};

template <int N, int TILE, typename Rt, bool G>
__global__ void __launch_bounds__(tile_threads(TILE)) k_ypass(const YZArgs a)
#ifdef HE_KERNEL_TU
{
  pdl_wait_and_trigger();
  // G: blockIdx.z = member x narr + array; otherwise blockIdx.z is the array
  const int mem = G ? (int)blockIdx.z / a.narr : 0;
  const int ai = G ? (int)blockIdx.z % a.narr : (int)blockIdx.z;
  using C = typename Cx<Rt>::T;
  C* smem = smem_as<C>();
  const int n = (N > 0) ? N : a.ny;
  const int ls = line_stride(n);
  const int TK = (N > 0) ? TILE : a.tkx;
  const int nxh = a.nxh;
  const int tid = threadIdx.x;
  // compile-time thread count for the compile-time lengths: the element loops below unroll and
  // issue their global loads together
  const int nthr = (N > 0) ? tile_threads(TILE) : (int)blockDim.x;
  const int kx0 = blockIdx.x * TK;
  const int z = blockIdx.y;
  C* arr = reinterpret_cast<C*>(on_member<G>(a.mm, a.arr[ai], mem));
  C* tw = smem;
  C* P0 = smem + ((a.pl.stw_len + 1) & ~1);
  C* P1 = P0 + TK * ls;
  load_twiddles(tw, a.pl);
  const long base = (long)nxh * n * z;
  for (int e = tid; e < TK * n; e += nthr) {
    const int j = e / TK, c = e - j * TK;
    const int kx = kx0 + c;
    P0[c * ls + sw<N>(j)] = (kx < nxh) ? arr[base + kx + (long)nxh * j] : Cx<Rt>::make(0, 0);
  }
  __syncthreads();
  C* R = fft_lines<N>(P0, P1, TK, ls, a.pl, tw, a.inv);
  for (int e = tid; e < TK * n; e += nthr) {
    const int j = e / TK, c = e - j * TK;
    const int kx = kx0 + c;
    if (kx < nxh) arr[base + kx + (long)nxh * j] = R[c * ls + sw<N>(j)];
  }
}
#else
;
#endif

// TWO: the second kernel k2 (out2, and the forward spectrum stored in fden_out) -- a compile-time
// choice, so that the one-kernel convolution carries neither its registers nor its third line
// buffer (the host passes two line buffers of shared memory then).
template <int N, int TILE, typename Rt, bool G, bool TWO>
__global__ void __launch_bounds__(tile_threads(TILE)) k_zconv(const YZArgs a)
#ifdef HE_KERNEL_TU
{
  pdl_wait_and_trigger();
  const int mem = G ? (int)blockIdx.z : 0;  // G: blockIdx.z is the group member
  using C = typename Cx<Rt>::T;
  using X = Cx<Rt>;
  constexpr bool F32 = sizeof(Rt) == 4;
  C* smem = smem_as<C>();
  C* io = reinterpret_cast<C*>(on_member<G>(a.mm, a.io, mem));
  C* out2 = reinterpret_cast<C*>(on_member<G>(a.mm, a.out2, mem));
  C* fden_out = reinterpret_cast<C*>(on_member<G>(a.mm, a.fden_out, mem));
  const double* kern1 = on_member<G>(a.mm, a.k1, mem);
  const double* kern2 = on_member<G>(a.mm, a.k2, mem);
  const float* kern1f = on_member<G>(a.mm, a.k1f, mem);
  const float* kern2f = on_member<G>(a.mm, a.k2f, mem);
  constexpr bool two = TWO;
  const int n = (N > 0) ? N : a.nz;
  const int ls = line_stride(n);
  const int TK = (N > 0) ? TILE : a.tkx;
  const int nxh = a.nxh;
  const int tid = threadIdx.x;
  // compile-time thread count for the compile-time lengths: the element loops below unroll and
  // issue their global loads together
  const int nthr = (N > 0) ? tile_threads(TILE) : (int)blockDim.x;
  const int kx0 = blockIdx.x * TK;
  const int ky = blockIdx.y;
  C* tw = smem;
  C* P0 = smem + ((a.pl.stw_len + 1) & ~1);
  C* P1 = P0 + TK * ls;
  C* P2 = P1 + TK * ls;
  load_twiddles(tw, a.pl);
  const long plane = (long)nxh * a.ny;
  const long base = (long)nxh * ky;
  // compile-time lengths: element e = tid + j nthr, j < EPT, and the kernel values of the
  // multiply are loaded before the forward transform, so their latency hides behind it
  constexpr int EPT = (N > 0) ? N / 16 : 1;  // TK n / nthr with nthr = 16 TK
  Rt w1p[EPT], w2p[TWO ? EPT : 1];
  if constexpr (N > 0) {
#pragma unroll
    for (int j = 0; j < EPT; ++j) {
      const int e = tid + j * nthr;
      const int jj = e / TK, c = e - jj * TK;
      const bool ok = kx0 + c < nxh;
      const long g = base + (ok ? kx0 + c : 0) + plane * jj;
      w1p[j] = ok ? (F32 ? Rt(kern1f[g]) : Rt(kern1[g])) : Rt(0);
      if constexpr (TWO) w2p[j] = ok ? (F32 ? Rt(kern2f[g]) : Rt(kern2[g])) : Rt(0);
    }
  }
#pragma unroll
  for (int e = tid; e < TK * n; e += nthr) {
    const int j = e / TK, c = e - j * TK;
    const int kx = kx0 + c;
    P0[c * ls + sw<N>(j)] = (kx < nxh) ? io[base + kx + plane * j] : X::make(0, 0);
  }
  __syncthreads();
  C* F = fft_lines<N>(P0, P1, TK, ls, a.pl, tw, false);
  C* O = (F == P0) ? P1 : P0;
  auto multiply = [&](int e, Rt w1, Rt w2) {
    const int j = e / TK, c = e - j * TK;
    const int kx = kx0 + c;
    const int s = c * ls + sw<N>(j);
    if (kx >= nxh) {
      F[s] = X::make(0, 0);
      if (two) P2[s] = X::make(0, 0);
      return;
    }
    const long g = base + kx + plane * j;
    const C f = F[s];
    if (fden_out) fden_out[g] = f;
    if (two) P2[s] = X::make(f.x * w2, f.y * w2);
    F[s] = X::make(f.x * w1, f.y * w1);
  };
  if constexpr (N > 0) {
#pragma unroll
    for (int j = 0; j < EPT; ++j) multiply(tid + j * nthr, w1p[j], TWO ? w2p[TWO ? j : 0] : Rt(0));
  } else {
    for (int e = tid; e < TK * n; e += nthr) {
      const int j = e / TK, c = e - j * TK;
      const long g = base + min(kx0 + c, nxh - 1) + plane * j;
      const Rt w1 = F32 ? Rt(kern1f[g]) : Rt(kern1[g]);
      const Rt w2 = two ? (F32 ? Rt(kern2f[g]) : Rt(kern2[g])) : Rt(0);
      multiply(e, w1, w2);
    }
  }
  __syncthreads();
  C* R1 = fft_lines<N>(F, O, TK, ls, a.pl, tw, true);
  for (int e = tid; e < TK * n; e += nthr) {
    const int j = e / TK, c = e - j * TK;
    const int kx = kx0 + c;
    if (kx < nxh) io[base + kx + plane * j] = R1[c * ls + sw<N>(j)];
  }
  if (!two) return;
  __syncthreads();
  C* S = (R1 == F) ? O : F;
  C* R2 = fft_lines<N>(P2, S, TK, ls, a.pl, tw, true);
  for (int e = tid; e < TK * n; e += nthr) {
    const int j = e / TK, c = e - j * TK;
    const int kx = kx0 + c;
    if (kx < nxh) out2[base + kx + plane * j] = R2[c * ls + sw<N>(j)];
  }
}
#else
;
#endif

}  // namespace he
