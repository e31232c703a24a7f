// fft_yz.cuh -- the y and z passes of a convolution fused into one launch over a thread-block
// cluster's distributed shared memory (ny = nz = N, half spectrum (nxh, N, N) in the FFTW
// layout of fft.f90's work arrays).
//
// The classical field evaluation convolves the x-transformed density with the k-space kernels
// (Dynamics_TDDFT/poten.f90:138-154 and :166-171): forward y and z transforms, a pointwise
// product with wcgk / fvlj4, inverse z and y transforms.  Done as separate passes that is three
// launches and three round trips of the spectrum through L2 per convolution.  Here one cluster
// of CS CTAs owns a pair of kx columns, i.e. two whole (ky, kz) planes (2 N^2 values), spread
// over the cluster's shared memory:
//
//   load     CTA r holds P[k][z][y] for its CS-th of the z planes (z in Z_r), both kx;
//   y fwd    in place along y, every line of P;
//   for each kx of the pair:
//     gather   Q[ky][z] for its CS-th of the ky columns (ky in Y_r) and all z, read from the
//              owning CTAs' P through distributed shared memory;
//     z fwd    in place along z (optionally stored as fden, the forward spectrum),
//     product  with the kernel K[kx, ky, kz],
//     z inv    in place along z,
//     scatter  Q back into the owners' P;
//   y inv    in place along y, store.
//
// TWO = true (the dencg / delj4 convolution of poten.f90:138-154): after the first product's
// result is stored, the forward spectrum is read back per kx from fden, multiplied by the second
// kernel, z-inverse transformed, scattered, y-inverse transformed and stored as out2.
//
// The line transforms are the register DFTs of the y pass (fft_reg.cuh: N = N1 x N2, a radix-N1
// DFT and twiddle in registers, one exchange through a small shared buffer T, a radix-N2 DFT),
// run in place on shared-memory lines; a line's elements are XOR-swizzled within 128-byte groups
// by the line index, so column walks (the transposing gathers, the per-line register loads of
// consecutive lines) hit distinct banks.
//
// Where it pays: a 128^3 binary64 cluster needs 224 KB of shared memory per CTA, one CTA of 8
// warps per SM, and measured 2.6x slower than the separate passes (latency-bound on the
// distributed-shared-memory gathers); on 64^3 grids (80 KB per CTA) the autotuner compares it
// with the separate passes per context and keeps the faster.
#pragma once
#include <cooperative_groups.h>

#include "fft_reg.cuh"

namespace he {

namespace cgx = cooperative_groups;

constexpr int kYZThreads = 256;

// Shared memory of one CTA: P (2 kx x N/CS planes x N), Q (N/CS lines x N), T (exchange).
template <int N, int CS, typename Rt>
HE_HD constexpr size_t yz_smem() {
  using C = typename Cx<Rt>::T;
  constexpr int TB = kYZThreads / Split<N>::N2;
  return sizeof(C) * ((size_t)2 * (N / CS) * N + (size_t)(N / CS) * N + (size_t)TB * N);
}

// Position of element i of line l: XOR of i's low bits with the line index inside a 128-byte
// group of elements (8 binary64 or 16 binary32 complex values).
template <typename C>
HE_D int yz_swz(int l, int i) {
  constexpr int G = 128 / (int)sizeof(C);
  return i ^ (l & (G - 1));
}

// In-place DFT (forward exp(-i), or inverse exp(+i) unscaled) of nl lines of N elements at
// base (line l at base + l N, swizzled), TB lines at a time through the exchange buffer T.
template <int N, bool INV, typename C>
HE_D void yz_lines(C* base, int nl, C* T, const C* __restrict__ tw2) {
  constexpr int N1 = Split<N>::N1, N2 = Split<N>::N2;
  constexpr int TB = kYZThreads / N2;
  static_assert(TB % 8 == 0 && TB * N2 == kYZThreads, "a batch is TB lines x N2 threads");
  const int tid = threadIdx.x;
  for (int l0 = 0; l0 < nl; l0 += TB) {
    {
      const int lb = tid % TB, am = tid / TB;
      const int l = l0 + lb;
      if (l < nl) {
        const C* line = base + (size_t)l * N;
        C v[N1];
#pragma unroll
        for (int m = 0; m < N1; ++m) v[m] = line[yz_swz<C>(l, am + N2 * m)];
        RDft<N1, INV>::run(v);
#pragma unroll
        for (int k1 = 1; k1 < N1; ++k1) v[k1] = cmul_conj_if(v[k1], __ldg(&tw2[k1 * N2 + am]), INV);
#pragma unroll
        for (int k1 = 0; k1 < N1; ++k1) T[(k1 * N2 + am) * TB + lb] = v[k1];
      }
    }
    __syncthreads();
    if (tid < TB * N1) {
      const int lb = tid % TB, k1 = tid / TB;
      const int l = l0 + lb;
      if (l < nl) {
        C u[N2];
#pragma unroll
        for (int q = 0; q < N2; ++q) u[q] = T[(k1 * N2 + q) * TB + lb];
        RDft<N2, INV>::run(u);
        C* line = base + (size_t)l * N;
#pragma unroll
        for (int k2 = 0; k2 < N2; ++k2) line[yz_swz<C>(l, k1 + N1 * k2)] = u[k2];
      }
    }
    __syncthreads();
  }
}

struct YZConvArgs {
  int nxh;
  double2* io;             // in: x-transformed spectrum; out: first convolution (in place)
  double2* out2;           // TWO: second convolution
  double2* fden_out;       // forward spectrum (may be null; required when TWO)
  const double* k1;        // kernels (binary64 chain)
  const double* k2;
  const float* k1f;        // binary32 copies (binary32 chain)
  const float* k2f;
  const double2* tw2;      // register-DFT twiddles of the line length
  const float2* tw2f;
  MemberMap mm;            // group members (blockIdx.y is the member)
};

template <int N, int CS, bool TWO, typename Rt, bool G>
__global__ void __launch_bounds__(kYZThreads, 1) k_yzconv(const YZConvArgs a)
#ifdef HE_KERNEL_TU
{
  const int mem = G ? (int)blockIdx.y : 0;  // G: blockIdx.y is the group member
  using C = typename Cx<Rt>::T;
  using X = Cx<Rt>;
  constexpr bool F32 = sizeof(Rt) == 4;
  constexpr int NS = N / CS;        // z planes (y phase) and ky columns (z phase) per CTA
  static_assert(N % CS == 0 && (NS * N) % kYZThreads == 0, "whole elements per thread");
  cgx::cluster_group cluster = cgx::this_cluster();
  const int r = (int)cluster.block_rank();
  const int kx0 = 2 * (int)(blockIdx.x / CS);
  const int nkx = min(2, a.nxh - kx0);   // 1 for the last, odd column
  const int nxh = a.nxh;
  const long plane = (long)nxh * N;      // stride of z
  C* P = smem_as<C>();                   // [2][NS][N]  line (k, zl) = k NS + zl, along y
  C* Q = P + 2 * NS * N;                 // [NS][N]     line ky_l, along z
  C* T = Q + NS * N;                     // [TB][N]
  const C* tw2;
  if constexpr (F32) tw2 = reinterpret_cast<const C*>(a.tw2f);
  else tw2 = reinterpret_cast<const C*>(a.tw2);
  const int tid = threadIdx.x;
  C* io = reinterpret_cast<C*>(on_member<G>(a.mm, a.io, mem));
  C* out2 = reinterpret_cast<C*>(on_member<G>(a.mm, a.out2, mem));
  C* fden = reinterpret_cast<C*>(on_member<G>(a.mm, a.fden_out, mem));
  const double* kern1 = on_member<G>(a.mm, a.k1, mem);
  const double* kern2 = on_member<G>(a.mm, a.k2, mem);
  const float* kern1f = on_member<G>(a.mm, a.k1f, mem);
  const float* kern2f = on_member<G>(a.mm, a.k2f, mem);
  // Every data movement below is a loop of EPT elements per thread whose loads are all issued
  // before the first store (register batches of EB), so a thread has many loads in flight.
  constexpr int EPT = NS * N / kYZThreads;
  constexpr int EB = EPT < 8 ? EPT : 8;
  static_assert(EPT % EB == 0, "whole batches");

  // load: P[k][zl][y] = io[kx0 + k, y, r NS + zl]   (element e: y = e % N, zl = e / N)
  for (int j0 = 0; j0 < EPT; j0 += EB) {
    C v0[EB], v1[EB];
#pragma unroll
    for (int j = 0; j < EB; ++j) {
      const int e = tid + kYZThreads * (j0 + j);
      const long g = kx0 + (long)nxh * (e % N) + plane * (r * NS + e / N);
      v0[j] = io[g];
      v1[j] = (nkx > 1) ? io[g + 1] : X::make(0, 0);
    }
#pragma unroll
    for (int j = 0; j < EB; ++j) {
      const int e = tid + kYZThreads * (j0 + j);
      const int y = e % N, zl = e / N;
      P[(size_t)zl * N + yz_swz<C>(zl, y)] = v0[j];
      P[(size_t)(NS + zl) * N + yz_swz<C>(NS + zl, y)] = v1[j];
    }
  }
  __syncthreads();
  yz_lines<N, false>(P, nkx * NS, T, tw2);

  // one kx of the pair through the z phase; from_fden: Q from the stored forward spectrum
  // instead of the gathered planes; kernel 1 or 2.  Element e of Q: ky_l = e % NS, z = e / NS.
  auto z_phase = [&](int k, bool from_fden, bool second) {
    const int kx = kx0 + k;
    if (!from_fden) {
      cluster.sync();  // every CTA's P[k] holds its y-transformed planes
      for (int j0 = 0; j0 < EPT; j0 += EB) {
        C v[EB];
#pragma unroll
        for (int j = 0; j < EB; ++j) {
          const int e = tid + kYZThreads * (j0 + j);
          const int kyl = e % NS, z = e / NS;
          const int s = z / NS, zl = z - s * NS;
          const C* Ps = cluster.map_shared_rank(P, s);
          const int l = k * NS + zl;
          v[j] = Ps[(size_t)l * N + yz_swz<C>(l, r * NS + kyl)];
        }
#pragma unroll
        for (int j = 0; j < EB; ++j) {
          const int e = tid + kYZThreads * (j0 + j);
          const int kyl = e % NS, z = e / NS;
          Q[(size_t)kyl * N + yz_swz<C>(kyl, z)] = v[j];
        }
      }
      __syncthreads();
      yz_lines<N, false>(Q, NS, T, tw2);
    } else {
      for (int j0 = 0; j0 < EPT; j0 += EB) {
        C v[EB];
#pragma unroll
        for (int j = 0; j < EB; ++j) {
          const int e = tid + kYZThreads * (j0 + j);
          v[j] = fden[kx + (long)nxh * (r * NS + e % NS) + plane * (e / NS)];
        }
#pragma unroll
        for (int j = 0; j < EB; ++j) {
          const int e = tid + kYZThreads * (j0 + j);
          const int kyl = e % NS, z = e / NS;
          Q[(size_t)kyl * N + yz_swz<C>(kyl, z)] = v[j];
        }
      }
      __syncthreads();
    }
    // forward spectrum out (first pass), product with the kernel
    for (int j0 = 0; j0 < EPT; j0 += EB) {
      Rt w[EB];
#pragma unroll
      for (int j = 0; j < EB; ++j) {
        const int e = tid + kYZThreads * (j0 + j);
        const long g = kx + (long)nxh * (r * NS + e % NS) + plane * (e / NS);
        if constexpr (F32) w[j] = second ? kern2f[g] : kern1f[g];
        else w[j] = second ? kern2[g] : kern1[g];
      }
#pragma unroll
      for (int j = 0; j < EB; ++j) {
        const int e = tid + kYZThreads * (j0 + j);
        const int kyl = e % NS, z = e / NS;
        C& q = Q[(size_t)kyl * N + yz_swz<C>(kyl, z)];
        if (!from_fden && fden) fden[kx + (long)nxh * (r * NS + kyl) + plane * z] = q;
        q = X::make(q.x * w[j], q.y * w[j]);
      }
    }
    __syncthreads();
    yz_lines<N, true>(Q, NS, T, tw2);
    cluster.sync();  // every CTA is done reading P[k] (gather) and with its last y phase
    for (int j0 = 0; j0 < EPT; j0 += EB) {
      C v[EB];
#pragma unroll
      for (int j = 0; j < EB; ++j) {
        const int e = tid + kYZThreads * (j0 + j);
        v[j] = Q[(size_t)(e % NS) * N + yz_swz<C>(e % NS, e / NS)];
      }
#pragma unroll
      for (int j = 0; j < EB; ++j) {
        const int e = tid + kYZThreads * (j0 + j);
        const int kyl = e % NS, z = e / NS;
        const int s = z / NS, zl = z - s * NS;
        C* Ps = cluster.map_shared_rank(P, s);
        const int l = k * NS + zl;
        Ps[(size_t)l * N + yz_swz<C>(l, r * NS + kyl)] = v[j];
      }
    }
  };
  // y inverse and store of P into dst
  auto y_out = [&](C* dst) {
    cluster.sync();  // every scatter into this CTA's P has landed
    yz_lines<N, true>(P, nkx * NS, T, tw2);
    for (int e = tid; e < NS * N; e += kYZThreads) {
      const int y = e % N, zl = e / N;
      const long g = kx0 + (long)nxh * y + plane * (r * NS + zl);
      dst[g] = P[(size_t)zl * N + yz_swz<C>(zl, y)];
      if (nkx > 1) dst[g + 1] = P[(size_t)(NS + zl) * N + yz_swz<C>(NS + zl, y)];
    }
  };

  // (every CTA of a cluster has the same pair, so all take the same branches and barriers)
  for (int k = 0; k < nkx; ++k) z_phase(k, false, false);
  y_out(io);
  if constexpr (TWO) {
    cluster.sync();  // every owner is done with its P's first result before it is overwritten
    for (int k = 0; k < nkx; ++k) z_phase(k, true, true);
    y_out(out2);
  }
}
#else
;
#endif

}  // namespace he
