// stencil.cuh -- 13-point finite differences along x, y and z, fused with their consumers.
//
// Restates Deriv3D_p / Deriv3D_pc (Dynamics_TDDFT/init_deriv_parallel.f90:373-648, :933-1209)
// with the boundary rows of Redef (redef.f:133-170): for icon=13 every boundary row is the centred
// row shifted with zero fill, i.e. a centred 13-point stencil over a zero-padded field; icon=8 and
// icon=18 wrap periodically / antiperiodically (init_deriv_parallel.f90:1094-1206).  An axis
// shorter than npd gives a zero derivative (init_deriv_parallel.f90:949-953).  The weights are
// the Bickley rows times Sto = 1/h**id.
//
// Kernel shape (2.5-D streaming): a CTA owns a TX x TY tile of the x-y plane and marches through a
// chunk of z.  Each thread keeps the 13 values f(x,y,z-6..z+6) of its column in registers (the z
// derivative), and the CTA stages the current plane with a 6-point halo in shared memory (the x
// and y derivatives).  Every field value is read from HBM once per chunk; halo re-reads hit L2.
// The consumer ('Op') receives the three derivatives and the centre value and does the fused
// pointwise work (H psi, predictor/corrector, reductions) in the same pass.
#pragma once
#include "common.cuh"

namespace he {

struct StencilGeom {
  int nx, ny, nz;
  int zc;            // z-chunk per CTA
  int icon;          // 13, 8 or 18
  int axis_on[3];    // 0 when n(axis) < npd
  double w[3][13];   // scaled weights per axis
};

template <typename T>
HE_D T load_bc(const T* __restrict__ f, const StencilGeom& g, int ix, int iy, int iz) {
  bool neg = false;
  if (g.icon == 13) {
    if (ix < 0 || ix >= g.nx || iy < 0 || iy >= g.ny || iz < 0 || iz >= g.nz) return zero_of(T());
  } else {
    const bool anti = (g.icon == 18);
    if (ix < 0) { ix += g.nx; neg ^= anti; } else if (ix >= g.nx) { ix -= g.nx; neg ^= anti; }
    if (iy < 0) { iy += g.ny; neg ^= anti; } else if (iy >= g.ny) { iy -= g.ny; neg ^= anti; }
    if (iz < 0) { iz += g.nz; neg ^= anti; } else if (iz >= g.nz) { iz -= g.nz; neg ^= anti; }
    // Axes shorter than 6 points (whose derivative is off) can still be out of range after one
    // wrap; keep the unused load inside the array.
    ix = min(max(ix, 0), g.nx - 1);
    iy = min(max(iy, 0), g.ny - 1);
    iz = min(max(iz, 0), g.nz - 1);
  }
  T v = f[(long)ix + (long)g.nx * ((long)iy + (long)g.ny * iz)];
  return neg_if(v, neg);
}

// Op interface:
//   using T;                        field element type (double or double2)
//   static constexpr int NV;        number of FP64 block reductions (0 = none)
//   HE_D void at(int ix,int iy,int iz,long idx,T dx,T dy,T dz,T c,double* acc) const;
// k_stencil serves ops without reductions; ops.cuh adds k_stencil_red with the grid reduction.
template <class Op, int TX, int TY>
__global__ void __launch_bounds__(TX* TY)
    k_stencil(const typename Op::T* __restrict__ f, const StencilGeom g, const Op op) {
  using T = typename Op::T;
  __shared__ T tile[TY + 12][TX + 12];
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int tid = tx + TX * ty;
  const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
  const int ix = x0 + tx, iy = y0 + ty;
  const int z0 = blockIdx.z * g.zc;
  const int z1 = min(z0 + g.zc, g.nz);
  const bool inside = (ix < g.nx) && (iy < g.ny);
  double acc[1] = {0.0};

  T q[13];
#pragma unroll
  for (int m = 0; m < 12; ++m)
    q[m + 1] = inside ? load_bc(f, g, ix, iy, z0 - 6 + m) : zero_of(T());

  for (int iz = z0; iz < z1; ++iz) {
#pragma unroll
    for (int m = 0; m < 12; ++m) q[m] = q[m + 1];
    q[12] = inside ? load_bc(f, g, ix, iy, iz + 6) : zero_of(T());
    // Centre: threads past the grid edge (partial tiles) stage the boundary value instead
    // (zero for icon=13, the wrapped value for icon=8/18).
    tile[ty + 6][tx + 6] = inside ? q[6] : load_bc(f, g, ix, iy, iz);
    // x halo: 6 columns each side for the TY rows
    for (int e = tid; e < 12 * TY; e += TX * TY) {
      const int r = e / 12, c = e - r * 12;
      const int sx = (c < 6) ? c : TX + c;
      tile[r + 6][sx] = load_bc(f, g, x0 + sx - 6, y0 + r, iz);
    }
    // y halo: 6 rows each side for the TX columns
    for (int e = tid; e < 12 * TX; e += TX * TY) {
      const int r = e / TX, c = e - r * TX;
      const int sy = (r < 6) ? r : TY + r;
      tile[sy][c + 6] = load_bc(f, g, x0 + c, y0 + sy - 6, iz);
    }
    __syncthreads();
    if (inside) {
      T dx = zero_of(T()), dy = zero_of(T()), dz = zero_of(T());
      if (g.axis_on[0]) {
#pragma unroll
        for (int m = 0; m < 13; ++m) dx = axpy(g.w[0][m], tile[ty + 6][tx + m], dx);
      }
      if (g.axis_on[1]) {
#pragma unroll
        for (int m = 0; m < 13; ++m) dy = axpy(g.w[1][m], tile[ty + m][tx + 6], dy);
      }
      if (g.axis_on[2]) {
#pragma unroll
        for (int m = 0; m < 13; ++m) dz = axpy(g.w[2][m], q[m], dz);
      }
      const long idx = (long)ix + (long)g.nx * ((long)iy + (long)g.ny * iz);
      op.at(ix, iy, iz, idx, dx, dy, dz, q[6], acc);
    }
    __syncthreads();
  }
}

}  // namespace he
