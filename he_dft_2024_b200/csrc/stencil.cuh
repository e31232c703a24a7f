// stencil.cuh -- 13-point finite differences along x, y and z, fused with their consumers.
//
// Restates Deriv3D_p / Deriv3D_pc (Dynamics_TDDFT/init_deriv_parallel.f90:373-648, :933-1209)
// with the boundary rows of Redef (redef.f:133-170): for icon=13 every boundary row is the centred
// row shifted with zero fill, i.e. a centred 13-point stencil over a zero-padded field; icon=8 and
// icon=18 wrap periodically / antiperiodically (init_deriv_parallel.f90:1094-1206); icon=24
// reflects evenly about the end points (redef.f:245-279).  An axis
// shorter than npd gives a zero derivative (init_deriv_parallel.f90:949-953).  The weights are
// the Bickley rows times Sto = 1/h**id.
//
// Kernel shape (2.5-D streaming, software pipelined): a CTA owns a TX x TY tile of the x-y plane
// and marches through a chunk of z.  Each thread keeps f(x,y,z-6..z+6) of its column in registers
// (the z derivative); the CTA stages the current plane with its 6-point x/y halo in shared memory
// (the x and y derivatives).  While plane z is being consumed, the next plane is already in
// flight: its halo and the consumer's pointwise operands by cp.async into the other half of
// double-buffered shared-memory stages (the halo zero-filled outside the grid for icon=13), and
// its z+7 column value by register prefetch.  One barrier per plane: the next plane's copies are
// issued right after it, into the buffers every thread finished reading before reaching it.
// Binary64 complex fields are further prefetched into L2 (stencil_l2_ahead planes beyond the
// copies: the operand rows, and the psi rows whose column values the register prefetch reads).
// Every field value is read from HBM once per chunk; halo re-reads hit L2.
// The consumer ('Op') receives the three derivatives, the centre value and its staged operands
// and does the fused pointwise work (H psi, predictor/corrector, reductions).
#pragma once
#include <type_traits>

#include "common.cuh"

namespace he {

struct StencilGeom {
  int nx, ny, nz;
  int zc;            // z-chunk per CTA
  int icon;          // 13, 8, 18 or 24
  int axis_on[3];    // 0 when n(axis) < npd
  int nzc;           // z-chunks per member: grid.z = nzc x members (0: grid.z, one member)
  int lcz;           // groups: consecutive z-chunks one CTA streams through (one partial each)
  MemberMap mm;      // group members' buffers (nmem = 1 outside a group)
  double w[3][13];   // scaled weights per axis
  float wf[3][13];   // the same in binary32 (stencils over binary32 fields)
};

// The weights of a field type: binary32 fields use wf.
template <typename T>
HE_D const auto& stencil_w(const StencilGeom& g) {
  if constexpr (sizeof(typename RealOf<T>::R) == 4) return g.wf;
  else return g.w;
}

// icon=24 (redef.f:245-279, then ICON=4 at :18-56): the boundary rows fold the centred row
// onto the grid as an even reflection about the first and last points, f(1-m) = f(1+m) and
// f(n+m) = f(n-m).
HE_HD int mirror_index(int i, int n) {
  if (i < 0) i = -i;
  else if (i >= n) i = 2 * (n - 1) - i;
  return min(max(i, 0), n - 1);
}

// Resolve (ix,iy,iz) under the boundary condition: returns false for a zero-padded point
// (icon=13), otherwise the in-range index and whether the value is negated (icon=18).
HE_D bool resolve_bc(const StencilGeom& g, int& ix, int& iy, int& iz, bool& neg) {
  neg = false;
  if (g.icon == 13)
    return !(ix < 0 || ix >= g.nx || iy < 0 || iy >= g.ny || iz < 0 || iz >= g.nz);
  if (g.icon == 24) {
    ix = mirror_index(ix, g.nx);
    iy = mirror_index(iy, g.ny);
    iz = mirror_index(iz, g.nz);
    return true;
  }
  const bool anti = (g.icon == 18);
  if (ix < 0) { ix += g.nx; neg ^= anti; } else if (ix >= g.nx) { ix -= g.nx; neg ^= anti; }
  if (iy < 0) { iy += g.ny; neg ^= anti; } else if (iy >= g.ny) { iy -= g.ny; neg ^= anti; }
  if (iz < 0) { iz += g.nz; neg ^= anti; } else if (iz >= g.nz) { iz -= g.nz; neg ^= anti; }
  // Axes shorter than 6 points (whose derivative is off) can still be out of range after one
  // wrap; keep the unused load inside the array.
  ix = min(max(ix, 0), g.nx - 1);
  iy = min(max(iy, 0), g.ny - 1);
  iz = min(max(iz, 0), g.nz - 1);
  return true;
}

template <typename T>
HE_D T load_bc(const T* __restrict__ f, const StencilGeom& g, int ix, int iy, int iz) {
  bool neg;
  if (!resolve_bc(g, ix, iy, iz, neg)) return zero_of(T());
  T v = f[(long)ix + (long)g.nx * ((long)iy + (long)g.ny * iz)];
  return neg_if(v, neg);
}

// Reductions: per-block partials, the last CTA to finish sums them in a fixed order.
struct ReduceTail {
  double* partials;
  unsigned* counter;
  double* out;
};
HE_D ReduceTail remap(const ReduceTail& r, const MemberMap& mm, int m) {
  return ReduceTail{mm(r.partials, m), mm(r.counter, m), mm(r.out, m)};
}

// Stencil ops that run over the members of a group carry remap(mm, m), which maps their device
// pointers to member m's buffers.
template <class O, class = void>
struct HasTimec : std::false_type {};
// Ops whose H psi carries the absorbing factor timec (ops.cuh Timec) take it as at_t(..., tr): the
// pass evaluates its x-y part once per column and loads each plane's z part one plane ahead.
template <class O>
struct HasTimec<O, std::void_t<decltype(std::declval<const O&>().tm.with_z(0.0, 0.0))>>
    : std::true_type {};
template <class O, class = void>
struct HasRemap : std::false_type {};
template <class O>
struct HasRemap<O, std::void_t<decltype(std::declval<O&>().remap(std::declval<const MemberMap&>(), 0))>>
    : std::true_type {};

template <int NV>
// nb partials, written by ncta CTAs (ncta < 0: one partial per CTA); the last CTA to finish sums
// them in a fixed order that depends on nb and the CTA's thread count only.
__device__ void reduce_tail(const ReduceTail& rt, long nb, long ncta = -1) {
  __shared__ bool s_last;
  const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  const int nthr = blockDim.x * blockDim.y * blockDim.z;
  if (tid == 0) {
    __threadfence();
    const unsigned t = atomicAdd(rt.counter, 1u);
    s_last = (t == (unsigned)((ncta < 0 ? nb : ncta) - 1));
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  double v[NV];
#pragma unroll
  for (int k = 0; k < NV; ++k) {
    double s = 0.0;
    for (long b = tid; b < nb; b += nthr) s += __ldcg(rt.partials + b * NV + k);
    v[k] = s;
  }
  block_reduce_store<NV>(v, rt.out);
  if (tid == 0) *rt.counter = 0u;
}

// Op interface:
//   using T;                      field element type (double, double2, float or float2)
//   static constexpr int NV;      number of FP64 block reductions (0 = none)
//   static constexpr int N8, N16; number of real / complex pointwise operand fields
//   const R* s8[N8]; const Z* s16[N16];  the operand fields (set by the host), R and Z the real
//                                        and complex types of T's precision (RealOf<T>)
//   HE_D void at(int ix,int iy,int iz,long idx,T dx,T dy,T dz,T c,const R* v8,
//                const Z* v16,int vs,double* acc) const;
//   where v8[k*vs] and v16[k*vs] are this point's operands of field k (staged in shared memory).
// Minimum resident CTAs per SM for a stencil instantiation (caps registers at 64K/(256*m)).
// (binary32 complex fields without reductions: 4, i.e. 64 registers; with binary64 reductions
// the consumers would spill at 64, and the corrector measured faster at 3 on 256^3 grids)
// An Op may set its own count with a static constexpr int kMinBlocks.
template <class O, class = void>
struct OpMinBlocks { static constexpr int v = 0; };
template <class O>
struct OpMinBlocks<O, std::void_t<decltype(O::kMinBlocks)>> { static constexpr int v = O::kMinBlocks; };
template <class Op>
constexpr int stencil_min_blocks() {
  using T = typename Op::T;
  if constexpr (OpMinBlocks<Op>::v > 0) return OpMinBlocks<Op>::v;
  return sizeof(T) == 16 ? 2 : (sizeof(T) == 8 ? (Op::NV > 0 ? 3 : 4) : 3);
}

// Planes of L2 prefetch ahead of the shared-memory copies (0 = none): binary64 complex fields
// only (128^3 FP64 step: corrector 106 -> 95 us, predictor 96 -> 85 us with 2; the binary32
// stencils measured no gain).
template <typename T>
constexpr int stencil_l2_ahead() { return sizeof(T) == 16 ? 2 : 0; }

// Dynamic shared memory of one stencil CTA: the double-buffered halo tile and the
// double-buffered operand stages.
template <class Op, int TX, int TY>
HE_HD constexpr size_t stencil_smem() {
  using RT = RealOf<typename Op::T>;
  return 2 * (size_t)(TY + 12) * (TX + 12) * sizeof(typename Op::T) +
         2 * (size_t)Op::N16 * TX * TY * sizeof(typename RT::Z) +
         2 * (size_t)Op::N8 * TX * TY * sizeof(typename RT::R);
}

// The stencil pass of one member; the CTA streams through z-chunks bz .. bz + nchunk - 1 of the
// member's nzc, with one reduction partial per chunk (so the sums do not depend on nchunk), and
// ncta CTAs per member report to the reduction tail (< 0: one per chunk).
template <class Op, int TX, int TY>
HE_D void stencil_run(const typename Op::T* __restrict__ f, const StencilGeom& g, const Op& op,
                      const ReduceTail& rt, int bz, int nzc, int nchunk = 1, long ncta = -1) {
  using T = typename Op::T;
  using R = typename RealOf<T>::R;
  using Z = typename RealOf<T>::Z;
  constexpr int NT = TX * TY;
  constexpr int NH = 12 * (TX + TY);       // halo elements per plane
  constexpr int HK = (NH + NT - 1) / NT;   // halo elements per thread
  constexpr int NV = Op::NV > 0 ? Op::NV : 1;
  constexpr int TILE = (TY + 12) * (TX + 12);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* tiles = reinterpret_cast<T*>(smem_raw);                                     // [2][TILE]
  Z* st16 = reinterpret_cast<Z*>(smem_raw + 2 * TILE * sizeof(T));  // [2][N16][NT]
  R* st8 = reinterpret_cast<R*>(st16 + 2 * Op::N16 * NT);           // [2][N8][NT]
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int tid = tx + TX * ty;
  const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
  const int ix = x0 + tx, iy = y0 + ty;
  const int z0 = bz * g.zc;
  const int z1 = min(z0 + nchunk * g.zc, g.nz);
  const bool inside = (ix < g.nx) && (iy < g.ny);
  const long plane = (long)g.nx * g.ny;
  const long idx0 = (long)min(ix, g.nx - 1) + (long)g.nx * min(iy, g.ny - 1);
  const bool anti = (g.icon == 18), wrap = (g.icon != 13);

  // This thread's halo elements: shared-memory slot, in-plane offset and x/y boundary status
  // (resolved once; only the z part changes per plane).
  int hslot[HK];
  long hoff[HK];
  bool hok[HK], hneg[HK];
#pragma unroll
  for (int k = 0; k < HK; ++k) {
    const int e = tid + k * NT;
    int sy = -1, sx = 0;
    if (e < 12 * TY) {  // x halo: 6 columns each side of the TY rows
      const int r = e / 12, c = e - r * 12;
      sy = r + 6;
      sx = (c < 6) ? c : TX + c;
    } else if (e < NH) {  // y halo: 6 rows each side of the TX columns
      const int e2 = e - 12 * TY;
      const int r = e2 / TX, c = e2 - r * TX;
      sy = (r < 6) ? r : TY + r;
      sx = c + 6;
    }
    hslot[k] = (sy < 0) ? -1 : sy * (TX + 12) + sx;
    int gx = x0 + sx - 6, gy = y0 + sy - 6, gz = 0;
    bool neg = false;
    hok[k] = (sy >= 0) && resolve_bc(g, gx, gy, gz, neg);
    hneg[k] = neg;
    hoff[k] = (long)gx + (long)g.nx * gy;
  }
  // Resolve plane index iz: false for a zero plane (icon=13), else the wrapped plane and sign.
  auto zplane = [&](int iz, int& zz, bool& zneg) -> bool {
    zneg = false;
    zz = iz;
    if (!wrap) return iz >= 0 && iz < g.nz;
    if (g.icon == 24) {
      zz = mirror_index(iz, g.nz);
      return true;
    }
    if (zz < 0) { zz += g.nz; zneg = anti; } else if (zz >= g.nz) { zz -= g.nz; zneg = anti; }
    zz = min(max(zz, 0), g.nz - 1);
    return true;
  };
  // Plane iz's halo and this thread's operands into stage buf (one cp.async group).
  auto issue_plane = [&](int buf, int iz) {
    int zz;
    bool zneg;
    const bool zok = zplane(iz, zz, zneg);
    T* tb = tiles + buf * TILE;
#pragma unroll
    for (int k = 0; k < HK; ++k) {
      if (hslot[k] < 0) continue;
      const bool ok = zok && hok[k];
      cp_async_elem(tb + hslot[k], ok ? f + hoff[k] + plane * zz : f, ok);
    }
    const long pi = idx0 + plane * iz;
#pragma unroll
    for (int k = 0; k < Op::N16; ++k)
      cp_async_elem(st16 + (buf * Op::N16 + k) * NT + tid, op.s16[k] + pi, true);
#pragma unroll
    for (int k = 0; k < Op::N8; ++k)
      cp_async_elem(st8 + (buf * Op::N8 + k) * NT + tid, op.s8[k] + pi, true);
    cp_async_commit();
  };
  auto fix_halo_sign = [&](int buf, int iz) {
    if (!anti) return;
    int zz;
    bool zneg;
    zplane(iz, zz, zneg);
    T* tb = tiles + buf * TILE;
#pragma unroll
    for (int k = 0; k < HK; ++k)
      if (hslot[k] >= 0 && (hneg[k] ^ zneg)) tb[hslot[k]] = neg_if(tb[hslot[k]], true);
  };
  auto column = [&](int iz) -> T {  // f at (ix, iy, iz) under the boundary condition
    int zz;
    bool zneg;
    if (!inside || !zplane(iz, zz, zneg)) return zero_of(T());
    return neg_if(f[idx0 + plane * zz], zneg);
  };

  double acc[NV];
#pragma unroll
  for (int k = 0; k < NV; ++k) acc[k] = 0.0;

  // L2 prefetch (prefetch.global.L2, one 128-byte line per instruction, addresses inside the
  // arrays only): the operand rows of plane iz, and the TY + 12 psi rows (x halo included) of
  // plane iz.
  constexpr int PF = stencil_l2_ahead<T>();
  auto l2_lines = [](const void* base, long bytes) {
    const char* end = static_cast<const char*>(base) + bytes;
    for (const char* p = (const char*)((uintptr_t)base & ~(uintptr_t)127); p < end; p += 128)
      asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
  };
  auto prefetch_ops = [&](int iz) {
    if (iz >= z1) return;
    const int nxr = min(TX, g.nx - x0);
    for (int r = tid; r < (Op::N16 + Op::N8) * TY; r += NT) {
      const int k = r / TY, yy = y0 + (r - k * TY);
      if (yy >= g.ny) continue;
      const long off = (long)x0 + (long)g.nx * (yy + (long)g.ny * iz);
      if (k < Op::N16) l2_lines(op.s16[k] + off, (long)nxr * sizeof(Z));
      else l2_lines(op.s8[k - Op::N16] + off, (long)nxr * sizeof(R));
    }
  };
  auto prefetch_psi = [&](int iz) {
    if (iz >= g.nz) return;
    const int xa = max(x0 - 6, 0), xb = min(x0 + TX + 6, g.nx);
    for (int r = tid; r < TY + 12; r += NT) {
      const int yy = y0 - 6 + r;
      if (yy < 0 || yy >= g.ny) continue;
      l2_lines(f + (long)xa + (long)g.nx * (yy + (long)g.ny * iz), (long)(xb - xa) * sizeof(T));
    }
  };

  // timec of this column: the x-y part, and the z part of the next plane (HasTimec)
  [[maybe_unused]] double txy = 0.0, azn = 0.0;
  if constexpr (HasTimec<Op>::value) {
    if (inside) txy = op.tm.xy(ix, iy);
    azn = op.tm.az[z0];
  }

  // Prologue: z-queue f(z0-6 .. z0+5), the next column value f(z0+6) and plane z0's stage.
  T q[13];
#pragma unroll
  for (int m = 0; m < 12; ++m) q[m + 1] = column(z0 - 6 + m);
  T qn = column(z0 + 6);
  issue_plane(0, z0);
  if (PF > 0) {
    for (int d = 1; d <= PF; ++d) {
      prefetch_ops(z0 + d);
      prefetch_psi(z0 + 6 + d);
    }
  }

  for (int iz = z0; iz < z1; ++iz) {
    const int b = (iz - z0) & 1;
    T* tb = tiles + b * TILE;
    [[maybe_unused]] const double azc = azn;
#pragma unroll
    for (int m = 0; m < 12; ++m) q[m] = q[m + 1];
    q[12] = qn;
    // Centre of plane iz: from the queue (threads past the grid edge stage the boundary value).
    // Buffer b was last read for plane iz-2, before the previous barrier.
    tb[(ty + 6) * (TX + 12) + tx + 6] = inside ? q[6] : load_bc(f, g, ix, iy, iz);
    cp_async_wait<0>();
    fix_halo_sign(b, iz);
    __syncthreads();
    // Plane iz+1 into buffer b^1, which every thread finished reading (plane iz-1) before the
    // barrier above.
    if (iz + 1 < z1) {
      issue_plane(b ^ 1, iz + 1);
      qn = column(iz + 7);
      if constexpr (HasTimec<Op>::value) azn = op.tm.az[iz + 1];
    }
    if (PF > 0) {
      prefetch_ops(iz + 1 + PF);
      prefetch_psi(iz + 7 + PF);
    }
    if (inside) {
      const auto& W = stencil_w<T>(g);
      T dx = zero_of(T()), dy = zero_of(T()), dz = zero_of(T());
      if (g.axis_on[0]) {
#pragma unroll
        for (int m = 0; m < 13; ++m) dx = axpy(W[0][m], tb[(ty + 6) * (TX + 12) + tx + m], dx);
      }
      if (g.axis_on[1]) {
#pragma unroll
        for (int m = 0; m < 13; ++m) dy = axpy(W[1][m], tb[(ty + m) * (TX + 12) + tx + 6], dy);
      }
      if (g.axis_on[2]) {
#pragma unroll
        for (int m = 0; m < 13; ++m) dz = axpy(W[2][m], q[m], dz);
      }
      if constexpr (HasTimec<Op>::value)
        op.at_t(ix, iy, iz, idx0 + plane * iz, dx, dy, dz, q[6], st8 + b * Op::N8 * NT + tid,
                st16 + b * Op::N16 * NT + tid, NT, acc, op.tm.with_z(txy, azc));
      else
        op.at(ix, iy, iz, idx0 + plane * iz, dx, dy, dz, q[6], st8 + b * Op::N8 * NT + tid,
              st16 + b * Op::N16 * NT + tid, NT, acc);
    }
    if constexpr (Op::NV > 0) {
      // the end of a chunk other than the last: its partial (the next flush is at least one
      // plane, and so one barrier, later)
      if (nchunk > 1 && iz + 1 < z1 && (iz + 1 - z0) % g.zc == 0) {
        const long c = bz + (iz - z0) / g.zc;
        const long blk = blockIdx.x + (long)gridDim.x * (blockIdx.y + (long)gridDim.y * c);
        block_reduce_store<NV>(acc, rt.partials + blk * NV);
#pragma unroll
        for (int k = 0; k < NV; ++k) acc[k] = 0.0;
      }
    }
  }
  if constexpr (Op::NV > 0) {
    const long nb = (long)gridDim.x * gridDim.y * nzc;
    const long c = bz + (z1 - 1 - z0) / g.zc;  // the last chunk
    const long blk = blockIdx.x + (long)gridDim.x * (blockIdx.y + (long)gridDim.y * c);
    block_reduce_store<NV>(acc, rt.partials + blk * NV);
    reduce_tail<NV>(rt, nb, ncta);
  }
}

// G = false: one context, blockIdx.z the z chunk, the arguments used as passed.  G = true: a
// group, blockIdx.z = member x nzc + chunk; the op (copied), the field and the reduction tail
// are mapped to the member's buffers.  Separate instantiations, so that a context outside a group
// runs no mapping code at all.
template <class Op, int TX, int TY, bool G>
__global__ void __launch_bounds__(TX* TY, stencil_min_blocks<Op>())
    k_stencil(const typename Op::T* __restrict__ f, const StencilGeom g, const Op op,
              const ReduceTail rt)
#ifdef HE_KERNEL_TU
{
  if constexpr (G) {
    // blockIdx.z = member x nphys + p; CTA p streams chunks p lcz .. p lcz + lcz - 1
    const int nzc = g.nzc, lcz = g.lcz > 0 ? g.lcz : 1;
    const int nphys = (nzc + lcz - 1) / lcz;
    const int mem = (int)blockIdx.z / nphys;
    const int bz = ((int)blockIdx.z - mem * nphys) * lcz;
    Op o = op;
    o.remap(g.mm, mem);
    stencil_run<Op, TX, TY>(g.mm(f, mem), g, o, remap(rt, g.mm, mem), bz, nzc, min(lcz, nzc - bz),
                            (long)gridDim.x * gridDim.y * nphys);
  } else {
    stencil_run<Op, TX, TY>(f, g, op, rt, (int)blockIdx.z, (int)gridDim.z);
  }
}
#else
;
#endif

}  // namespace he
