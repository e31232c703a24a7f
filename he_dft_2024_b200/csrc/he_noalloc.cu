// he_noalloc.cu -- he_energy_noalloc: the energy() sums on device arrays the caller owns,
// without any device allocation.
//
// Who needs it: callers whose device memory is all owned by someone else and who therefore
// cannot let a library call cudaMalloc -- for example a Fortran driver whose arrays live in
// OpenACC or CUDA Fortran data regions sized once at start-up, or a job that reserves the GPU's
// memory up front in its own pool.  Such a caller holds psi, den, dencg, delj4 (and uimp) in its
// own arrays and only wants the energy diagnostics of them.  The context API (he_ctx_create)
// allocates its own copy of the whole state, so it does not fit them.
//
// The only device memory this entry point uses besides the caller's arrays is the file-scope
// array below: per-CTA partial sums of the reduction, the completion counter and the five final
// sums.  Its size is fixed: room for kNoAllocMaxBlocks = 8192 reduction blocks of the stencil
// grid (32 x 8 points x 16 planes each).  A 256^3 grid needs 4096 of them; grids needing more
// than 8192 are rejected with HE_ERR_ARG.  Every GPU that loads the library holds these 328,000
// bytes until the process exits.
//
// Only the OT and OP cores are accepted: for core4 = 'OTC' the reference adds the alpha_s energy
// (Dynamics_TDDFT/energy.f90:131-135) to etot4, which needs the alpha_s fields this entry point
// does not have, so it returns HE_ERR_ARG instead of a total without that term.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>

#include "../../include/he_dft.h"
#include "ops.cuh"

using namespace he;

namespace {

constexpr int kNoAllocMaxBlocks = 8192;
constexpr int kNoAllocNV = 5;  // OpEnergy sums
// [0, kNoAllocMaxBlocks*NV): partials; then one slot for the counter, then the NV sums.
constexpr int kCounterSlot = kNoAllocMaxBlocks * kNoAllocNV;
constexpr int kSumsSlot = kCounterSlot + 8;
constexpr int kScratchDoubles = kSumsSlot + 32;

static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

// Device address of g_noalloc_scratch on the current device.  In host code the array's name is
// only a host-side stand-in, so the address is looked up with the device current.  The lookup
// is repeated on every call (it is cheap): an address kept across calls would go stale when the
// caller resets the device (cudaDeviceReset) and the module is loaded again.  The first call on
// a device may load the library's device code, which is why it should come before any stream
// capture.
int scratch_for_current_device(double** out, char* err, size_t errlen) {
  double* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress((void**)&p, g_noalloc_scratch);
  if (e != cudaSuccess || !p) {
    if (err && errlen)
      snprintf(err, errlen, "cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
    return HE_ERR_CUDA;
  }
  *out = p;
  return HE_OK;
}

// core4 as the functional gives it: "OT " and "OP " (a trailing blank or NUL) are accepted.
bool core_ot_or_op(const char c[4]) {
  return c[0] == 'O' && (c[1] == 'T' || c[1] == 'P') && (c[2] == ' ' || c[2] == '\0');
}

void bickley13_rows(double w1[13]) {  // first-derivative row (newder.f:99-130, M=13, K=1)
  const double f6sq = 518400.0;
  const double fact[13] = {1, 1, 2, 6, 24, 120, 720, 5040, 40320, 362880, 3628800, 39916800,
                           479001600};
  for (int j = 0; j < 13; ++j) w1[j] = 0.0;
  for (int j = 1; j <= 6; ++j) {
    const double den1 = (double)j * fact[6 - j] * fact[6 + j];
    const double s = (j % 2 == 1) ? 1.0 : -1.0;
    w1[6 + j] = s * (f6sq / den1);
    w1[6 - j] = -w1[6 + j];
  }
}

template <typename T>
int launch_energy(const StencilGeom& g, dim3 grid, const OpEnergy<T>& op, const T* psi,
                  const ReduceTail& rt, cudaStream_t st, char* err, size_t errlen) {
  constexpr size_t smem = stencil_smem<OpEnergy<T>, 32, 8>();
  cudaError_t e = cudaFuncSetAttribute(k_stencil<OpEnergy<T>, 32, 8, false>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess) {
    k_stencil<OpEnergy<T>, 32, 8, false><<<grid, dim3(32, 8), smem, st>>>(psi, g, op, rt);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) {
    if (err && errlen) snprintf(err, errlen, "energy kernel launch failed: %s", cudaGetErrorString(e));
    return HE_ERR_CUDA;
  }
  return HE_OK;
}

}  // namespace

extern "C" int he_energy_noalloc(const he_grid_t* grid, const he_functional_t* fun, int mode,
                                 const void* psi, const double* den, const double* dencg,
                                 const double* delj4, const double* uimp, void* stream,
                                 he_energies_t* out, char* err, size_t errlen) {
  if (err && errlen) err[0] = '\0';
  auto bad = [&](const char* msg) {
    if (err && errlen) snprintf(err, errlen, "%s", msg);
    return HE_ERR_ARG;
  };
  if (!grid || !fun || !out) return bad("null grid, functional or output");
  if (mode != HE_MODE_DYNAMICS && mode != HE_MODE_STATICS) return bad("unknown mode");
  if (grid->npd != 13) return bad("npd must be 13");
  if (grid->icon != 13 && grid->icon != 8 && grid->icon != 18 &&
           grid->icon != 24) return bad("icon must be 13, 8, 18 or 24");
  if (grid->nx < 1 || grid->ny < 1 || grid->nz < 1) return bad("grid sizes must be positive");
  if (grid->xmax == 0.0 || grid->ymax == 0.0 || grid->zmax == 0.0)
    return bad("xmax, ymax, zmax must be non-zero");
  if (!core_ot_or_op(fun->core4))
    return bad("core4 must be 'OT ' or 'OP ': the 'OTC' total needs the alpha_s energy, which "
               "he_energy_noalloc does not compute (use he_energy)");
  StencilGeom g{};
  g.nx = grid->nx; g.ny = grid->ny; g.nz = grid->nz;
  g.icon = grid->icon;
  g.zc = (grid->nz >= 128) ? 16 : 8;
  const dim3 gd((grid->nx + 31) / 32, (grid->ny + 7) / 8, (grid->nz + g.zc - 1) / g.zc);
  const long nblocks = (long)gd.x * gd.y * gd.z;
  if (nblocks > kNoAllocMaxBlocks) {
    if (err && errlen)
      snprintf(err, errlen,
               "grid %dx%dx%d needs %ld reduction blocks; he_energy_noalloc holds at most %d "
               "(grids up to 256^3)", grid->nx, grid->ny, grid->nz, nblocks, kNoAllocMaxBlocks);
    return HE_ERR_ARG;
  }
  if (!psi || !den || !dencg || !delj4) return bad("null field pointer");

  double* scratch = nullptr;
  int st = scratch_for_current_device(&scratch, err, errlen);
  if (st != HE_OK) return st;
  cudaStream_t s = (cudaStream_t)stream;

  const double hx = 2.0 * std::fabs(grid->xmax) / grid->nx;
  const double hy = 2.0 * std::fabs(grid->ymax) / grid->ny;
  const double hz = 2.0 * std::fabs(grid->zmax) / grid->nz;
  double w1[13];
  bickley13_rows(w1);
  const double hs[3] = {hx, hy, hz};
  const int ns[3] = {grid->nx, grid->ny, grid->nz};
  for (int a = 0; a < 3; ++a) {
    g.axis_on[a] = ns[a] >= 13 ? 1 : 0;
    for (int m = 0; m < 13; ++m) g.w[a][m] = w1[m] * (1.0 / hs[a]);
  }

  // The completion counter must start at zero; the sums are overwritten by the last block.
  cudaError_t e = cudaMemsetAsync(scratch + kCounterSlot, 0, sizeof(double), s);
  if (e != cudaSuccess) {
    if (err && errlen) snprintf(err, errlen, "cudaMemsetAsync failed: %s", cudaGetErrorString(e));
    return HE_ERR_CUDA;
  }
  ReduceTail rt;
  rt.partials = scratch;
  rt.counter = reinterpret_cast<unsigned*>(scratch + kCounterSlot);
  rt.out = scratch + kSumsSlot;

  const double aux1 = 0.5 * fun->cp4, aux2 = (1.0 / 3.0) * fun->cpp4;
  if (mode == HE_MODE_DYNAMICS) {
    OpEnergy<double2> op{};
    op.s8[0] = den; op.s8[1] = dencg; op.s8[2] = delj4; op.s8[3] = uimp ? uimp : den;
    op.has_u = uimp ? 1 : 0;
    op.aux1 = aux1; op.aux2 = aux2;
    op.beta = fun->beta; op.den_m = fun->den_m; op.lsolid = fun->lsolid;
    st = launch_energy(g, gd, op, (const double2*)psi, rt, s, err, errlen);
  } else {
    OpEnergy<double> op{};
    op.s8[0] = den; op.s8[1] = dencg; op.s8[2] = delj4; op.s8[3] = uimp ? uimp : den;
    op.has_u = uimp ? 1 : 0;
    op.aux1 = aux1; op.aux2 = aux2;
    op.beta = fun->beta; op.den_m = fun->den_m; op.lsolid = fun->lsolid;
    st = launch_energy(g, gd, op, (const double*)psi, rt, s, err, errlen);
  }
  if (st != HE_OK) return st;
  double sums[kNoAllocNV];
  e = cudaMemcpyAsync(sums, scratch + kSumsSlot, sizeof(sums), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    if (err && errlen) snprintf(err, errlen, "reading the sums failed: %s", cudaGetErrorString(e));
    return HE_ERR_CUDA;
  }
  const double dxyz = hx * hy * hz;
  he_energies_t r{};
  r.esolid = fun->lsolid ? fun->C * sums[3] * dxyz : 0.0;
  r.ekin4 = fun->h2o2m4 * sums[0] * dxyz;
  r.elj4 = 0.5 * sums[1] * dxyz;
  r.ecor4 = sums[2] * dxyz;
  r.etot4 = r.ekin4 + r.elj4 + r.ecor4 + r.esolid;
  r.eHeX = uimp ? sums[4] * dxyz : 0.0;
  r.eimpu = r.eHeX;
  r.etot = r.etot4 + r.eimpu;
  *out = r;
  return HE_OK;
}
