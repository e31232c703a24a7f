// he_dft.cu -- context, host orchestration and C-ABI of the sm_100a mean-field / time-step path.
//
// The call surface mirrors the reference routines named in include/he_dft.h; this file only
// sequences device work.  All arithmetic on fields happens in the kernels of fft_kernels.cuh,
// ops.cuh and setup.cuh; there is no host or library fallback for any of it.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/he_dft.h"
#include "common.cuh"
#include "fft.cuh"
#include "fft_kernels.cuh"
#include "ops.cuh"
#include "setup.cuh"

using namespace he;

namespace {

constexpr double kMpU = 0.02061484;  // proton mass in K^-1 A^-2 (modules.f90:324)
constexpr int kTX = 32, kTY = 8;     // stencil tile
constexpr int kPwBlocks = 592;       // pointwise reduction grid (4 x 148 SMs)

// Reduction result slots in ctx->sums.
enum Slot {
  S_ERRHE = 0,
  S_EN = 1,      // 5 energy sums
  S_FORCE = 8,   // 3*kMaxImp force sums
  S_STAT_H = 40,
  S_STAT_N = 41,
  S_STAT_MU = 43,
  S_VARMU = 44,
  S_HMEAN0 = 45,
  S_STAT_PC = 46,   // k_stat_correct writes {sum |pc|, sum psi^2} to slots 46, 47
  S_COUNT = 64
};

}  // namespace

struct he_ctx {
  int mode = 0, prec = 0;
  int nx = 0, ny = 0, nz = 0, nxh = 0;
  long N = 0, Nk = 0;
  double xmax = 0, ymax = 0, zmax = 0, hx = 0, hy = 0, hz = 0, dxyz = 0, renor = 0;
  int icon = 13;
  he_functional_t fn{};
  int op_core = 0, otc = 0;
  double w1[13], w2[13];
  StencilGeom g1{}, g2{};
  cudaStream_t stream = nullptr, own = nullptr;
  std::string err;
  long long launches = 0;
  size_t bytes = 0;
  std::vector<void*> allocs;
  // FFT
  LinePlan plx{}, ply{}, plz{};
  int x_rb = 16, tkx = 16;
  int num_sms = 148;
  int tile_x = 16, tile_y = 16, tile_z = 16;  // autotuned tile variants (16 or 8 lines)
  size_t smem_x = 0, smem_y = 0, smem_z = 0;
  // k space
  double2 *fden = nullptr, *wA = nullptr, *wB = nullptr;
  double *fvlj4 = nullptr, *wcgk = nullptr, *kalfs = nullptr;
  bool kernels_ok = false;
  // real fields
  double *den = nullptr, *pot4 = nullptr, *dencg = nullptr, *delj4 = nullptr, *uimp = nullptr;
  double *dxden = nullptr, *dyden = nullptr, *dzden = nullptr;
  double *hpsi = nullptr, *t4 = nullptr, *timec = nullptr;
  // wave function ring (complex in dynamics, real in statics); psiold[s-1] is Fortran slot s
  void *psi = nullptr, *psiold[3] = {}, *hpsiold[2] = {}, *pc = nullptr, *q = nullptr,
       *scratch = nullptr;
  int ioldp[3] = {1, 2, 3}, ioldh[2] = {1, 2};
  // absorber
  double *tabx = nullptr, *taby = nullptr, *tabz = nullptr;
  double lambdah = 0.0;
  // impurities
  ImpDev* imp = nullptr;
  int n_imp = 0, npot = 0;
  double* pot_tab = nullptr;
  size_t pot_tab_cap = 0;
  double delinter = 0.0, rmaxinterpol = 0.0;
  bool force_fresh = false;
  // reductions
  double* partials = nullptr;
  size_t partials_cap = 0;
  unsigned* counter = nullptr;
  double* sums = nullptr;
  double* hsum = nullptr;  // pinned host mirror of sums
  // optional per-kernel CUDA-event timing (he_timing / he_timing_report)
  struct TRec {
    const char* name;
    cudaEvent_t a, b;
  };
  bool timing = false;
  std::vector<TRec> trec;
  std::vector<cudaEvent_t> evpool;
  size_t evnext = 0;
};

// ------------------------------------------------------------------------------------------------
// helpers
// ------------------------------------------------------------------------------------------------
static int fail(he_ctx_t* c, int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  if (c) c->err = buf;
  return code;
}

#define CK(call)                                                                         \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess)                                                               \
      return fail(ctx, HE_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_));     \
  } while (0)

#define LAUNCHED()                                                                       \
  do {                                                                                   \
    ++ctx->launches;                                                                     \
    tstop(ctx);                                                                          \
    cudaError_t e_ = cudaGetLastError();                                                 \
    if (e_ != cudaSuccess)                                                               \
      return fail(ctx, HE_ERR_CUDA, "kernel launch failed (%s:%d): %s", __FILE__,      \
                  __LINE__, cudaGetErrorString(e_));                                     \
  } while (0)

#define TRY(expr)            \
  do {                       \
    int s_ = (expr);         \
    if (s_ != HE_OK) return s_; \
  } while (0)

static cudaEvent_t tevent(he_ctx_t* ctx) {
  if (ctx->evnext == ctx->evpool.size()) {
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    ctx->evpool.push_back(e);
  }
  return ctx->evpool[ctx->evnext++];
}
// Marks the start of the next launch (named) when timing is on; LAUNCHED() marks its end.
static void tname(he_ctx_t* ctx, const char* name) {
  if (!ctx->timing) return;
  he_ctx::TRec r{name, tevent(ctx), nullptr};
  cudaEventRecord(r.a, ctx->stream);
  ctx->trec.push_back(r);
}
static void tstop(he_ctx_t* ctx) {
  if (!ctx->timing || ctx->trec.empty() || ctx->trec.back().b) return;
  ctx->trec.back().b = tevent(ctx);
  cudaEventRecord(ctx->trec.back().b, ctx->stream);
}

static int dalloc(he_ctx_t* ctx, void** p, size_t bytes) {
  cudaError_t e = cudaMalloc(p, bytes);
  if (e != cudaSuccess) {
    *p = nullptr;
    return fail(ctx, HE_ERR_NOMEM, "cudaMalloc(%zu) failed: %s", bytes, cudaGetErrorString(e));
  }
  ctx->allocs.push_back(*p);
  ctx->bytes += bytes;
  CK(cudaMemsetAsync(*p, 0, bytes, ctx->stream));
  return HE_OK;
}
template <typename T>
static int dalloc_t(he_ctx_t* ctx, T** p, size_t count) {
  return dalloc(ctx, reinterpret_cast<void**>(p), count * sizeof(T));
}

static bool factor_ok(int n) {
  if (n < 1) return false;
  while (n % 2 == 0) n /= 2;
  while (n % 3 == 0) n /= 3;
  while (n % 5 == 0) n /= 5;
  return n == 1;
}
static bool tstgrid_ok(int n) {  // tstgrid.f90:9-13
  static const int v[] = {1,   2,   3,   4,   5,   6,   8,   9,   10,  12,  15,  16,  18,  20,
                          24,  25,  27,  30,  32,  36,  40,  45,  48,  50,  54,  60,  64,  72,
                          75,  80,  81,  90,  96,  100, 108, 120, 125, 128, 135, 144, 150, 160,
                          162, 180, 192, 200, 216, 225, 240, 243, 250, 256, 320, 324, 384, 512};
  for (int x : v)
    if (x == n) return true;
  return false;
}

static int make_plan(he_ctx_t* ctx, int n, LinePlan* pl) {
  pl->n = n;
  pl->nst = num_stages(n);
  int m = n;
  for (int s = 0; s < pl->nst; ++s) {
    pl->rad[s] = radix_of(m);
    m /= pl->rad[s];
  }
  if (m != 1 || pl->nst > kMaxStages) return fail(ctx, HE_ERR_ARG, "FFT length %d is not 2^a 3^b 5^c", n);
  // Per-stage twiddles: stage s (radix R, ns = product of earlier radices) holds
  // exp(-2 pi i r k / (ns R)) at [(r-1)*ns + k], r = 1..R-1, k = 0..ns-1.
  std::vector<double2> stw;
  int ns = 1;
  for (int s = 0; s < pl->nst; ++s) {
    const int R = pl->rad[s];
    for (int r = 1; r < R; ++r)
      for (int k = 0; k < ns; ++k) {
        long double a = -2.0L * 3.14159265358979323846264338327950288L * r * k / ((long double)ns * R);
        stw.push_back(make_double2((double)cosl(a), (double)sinl(a)));
      }
    ns *= R;
  }
  if (stw.empty()) stw.push_back(make_double2(1.0, 0.0));
  double2* d = nullptr;
  TRY(dalloc_t(ctx, &d, stw.size()));
  CK(cudaMemcpyAsync(d, stw.data(), stw.size() * sizeof(double2), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  pl->tw = d;
  pl->stw = d;
  pl->stw_len = (int)stw.size();
  return HE_OK;
}

// 13-point Bickley rows (newder.f:99-130 table values for M=13, K=1,2 as exact rationals).
static void bickley13(double w1[13], double w2[13]) {
  const double f6sq = 518400.0;
  const double fact[13] = {1, 1, 2, 6, 24, 120, 720, 5040, 40320, 362880, 3628800, 39916800,
                           479001600};
  for (int j = 0; j < 13; ++j) w1[j] = w2[j] = 0.0;
  for (int j = 1; j <= 6; ++j) {
    const double den1 = (double)j * fact[6 - j] * fact[6 + j];
    const double den2 = (double)j * (double)j * fact[6 - j] * fact[6 + j];
    const double s = (j % 2 == 1) ? 1.0 : -1.0;
    w1[6 + j] = s * (f6sq / den1);
    w1[6 - j] = -w1[6 + j];
    w2[6 + j] = s * ((2.0 * f6sq) / den2);
    w2[6 - j] = w2[6 + j];
  }
  w2[6] = -5369.0 / 1800.0;
}

static void make_geom(he_ctx_t* ctx, int id, StencilGeom* g) {
  g->nx = ctx->nx; g->ny = ctx->ny; g->nz = ctx->nz;
  g->icon = ctx->icon;
  g->zc = (ctx->nz >= 128) ? 16 : 8;
  const double hs[3] = {ctx->hx, ctx->hy, ctx->hz};
  const int ns[3] = {ctx->nx, ctx->ny, ctx->nz};
  for (int a = 0; a < 3; ++a) {
    g->axis_on[a] = ns[a] >= 13 ? 1 : 0;
    const double sto = (id == 1) ? 1.0 / hs[a] : 1.0 / (hs[a] * hs[a]);
    for (int m = 0; m < 13; ++m) g->w[a][m] = ((id == 1) ? ctx->w1[m] : ctx->w2[m]) * sto;
  }
}

static dim3 stencil_grid(const he_ctx_t* ctx, const StencilGeom& g) {
  return dim3((ctx->nx + kTX - 1) / kTX, (ctx->ny + kTY - 1) / kTY, (ctx->nz + g.zc - 1) / g.zc);
}

static int ensure_partials(he_ctx_t* ctx, size_t count) {
  if (count <= ctx->partials_cap) return HE_OK;
  return fail(ctx, HE_ERR_STATE, "reduction buffer too small (%zu > %zu)", count,
              ctx->partials_cap);
}

static ReduceTail tail(he_ctx_t* ctx, int slot) {
  ReduceTail r;
  r.partials = ctx->partials;
  r.counter = ctx->counter;
  r.out = ctx->sums + slot;
  return r;
}

// z-chunk of a stencil launch.  A CTA marches one x-y tile through `zc` planes after a
// 12-plane prologue; the grid is (x tiles) x (y tiles) x ceil(nz/zc).  The chunk minimises
// waves x (zc + 6): waves = ceil(CTAs / (SMs x resident CTAs per SM)), and the prologue costs
// about half a step per plane.  The resident-CTA count is the kernel's occupancy, queried once
// per kernel and device.
static int choose_zc(const he_ctx_t* ctx, int occ) {
  const long tiles = (long)((ctx->nx + kTX - 1) / kTX) * ((ctx->ny + kTY - 1) / kTY);
  const long slots = (long)ctx->num_sms * (occ > 0 ? occ : 1);
  int best = ctx->nz, bestcost = 1 << 30;
  for (int zc = 4; zc <= ctx->nz; ++zc) {
    const long ctas = tiles * ((ctx->nz + zc - 1) / zc);
    const long waves = (ctas + slots - 1) / slots;
    const int cost = (int)(waves * (zc + 6));
    if (cost < bestcost) { bestcost = cost; best = zc; }
  }
  return std::max(1, std::min(best, ctx->nz));
}

template <class Op>
static int run_stencil(he_ctx_t* ctx, const StencilGeom& g0, const typename Op::T* f, const Op& op,
                       int slot = -1) {
  constexpr size_t smem = stencil_smem<Op, kTX, kTY>();
  static int occ = -1;  // resident CTAs per SM of this instantiation
  if (occ < 0) {
    CK(cudaFuncSetAttribute(k_stencil<Op, kTX, kTY>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            (int)smem));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_stencil<Op, kTX, kTY>, kTX * kTY, smem));
  }
  StencilGeom g = g0;
  g.zc = choose_zc(ctx, occ);
  dim3 grid = stencil_grid(ctx, g), block(kTX, kTY);
  ReduceTail rt{};
  if (Op::NV > 0) {
    TRY(ensure_partials(ctx, (size_t)grid.x * grid.y * grid.z * Op::NV));
    rt = tail(ctx, slot);
  }
  CK(cudaFuncSetAttribute(k_stencil<Op, kTX, kTY>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                          (int)smem));
  tname(ctx, Op::kname());
  k_stencil<Op, kTX, kTY><<<grid, block, smem, ctx->stream>>>(f, g, op, rt);
  LAUNCHED();
  return HE_OK;
}
template <class Op>
static int run_stencil_red(he_ctx_t* ctx, const StencilGeom& g, const typename Op::T* f,
                           const Op& op, int slot) {
  return run_stencil(ctx, g, f, op, slot);
}

static Timec timec_view(const he_ctx_t* ctx) {
  Timec t;
  t.ax = ctx->tabx; t.ay = ctx->taby; t.az = ctx->tabz;
  t.lambdah = ctx->lambdah;
  return t;
}

// ---- FFT pass launchers --------------------------------------------------------------------------
static XArgs xargs(he_ctx_t* ctx) {
  XArgs a{};
  a.nx = ctx->nx; a.nxh = ctx->nxh;
  a.rows = (long)ctx->ny * ctx->nz;
  a.rb = ctx->x_rb;
  a.pl = ctx->plx;
  a.renor = ctx->renor;
  a.cp4 = ctx->fn.cp4; a.cpp4 = ctx->fn.cpp4;
  a.a0 = ctx->fn.cp4 / 2.0; a.a1 = ctx->fn.cpp4 / 3.0;
  a.lsolid = ctx->fn.lsolid;
  a.C = ctx->fn.C; a.beta = ctx->fn.beta; a.den_m = ctx->fn.den_m;
  return a;
}
// Line lengths with a compile-time FFT instantiation; other admissible lengths run the same
// kernels with run-time sizes (N = 0).
#define HE_FFT_SIZES(X) X(32) X(64) X(96) X(128) X(160) X(192) X(256)

static size_t fft_smem(const LinePlan& pl, int lines, int nbuf) {
  return sizeof(double2) * (((size_t)pl.stw_len + 1) / 2 * 2 + (size_t)nbuf * lines * line_stride(pl.n));
}
static bool x_fast(const he_ctx_t* ctx, int tile) {
  switch (ctx->nx) {
#define HE_CASE(N) case N:
    HE_FFT_SIZES(HE_CASE)
#undef HE_CASE
    return ((long)ctx->ny * ctx->nz) % tile == 0;
    default: return false;
  }
}
static bool yz_fast(int n) {
  switch (n) {
#define HE_CASE(N) case N:
    HE_FFT_SIZES(HE_CASE)
#undef HE_CASE
    return true;
    default: return false;
  }
}

// Tile variants of the compile-time kernels: 16 lines per CTA (256 threads) or 8 (128 threads).
// he_ctx_create times both for each pass family on the context's grid and keeps the faster.
template <int MODE, int N, int TILE>
static int xpass_n(he_ctx_t* ctx, const XArgs& a) {
  const int rb = (N > 0) ? TILE : a.rb;
  const unsigned nb = (unsigned)((a.rows + rb - 1) / rb);
  const size_t smem = fft_smem(ctx->plx, rb, 2);
  const int nthr = (N > 0) ? tile_threads(TILE) : 256;
  static const char* names[5] = {"fft_x_r2c_den", "fft_x_r2c_corr", "fft_x_c2r_cg_lj",
                                 "fft_x_c2r_cg_lj_r2c_corr", "fft_x_c2r_pot4"};
  CK(cudaFuncSetAttribute(k_xpass<MODE, N, TILE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  tname(ctx, names[MODE]);
  k_xpass<MODE, N, TILE><<<nb, nthr, smem, ctx->stream>>>(a);
  LAUNCHED();
  return HE_OK;
}
template <int MODE>
static int xpass(he_ctx_t* ctx, const XArgs& a) {
  const int tile = ctx->tile_x;
  if (x_fast(ctx, tile)) {
    switch (ctx->nx) {
#define HE_CASE(N) \
  case N: return tile == 8 ? xpass_n<MODE, N, 8>(ctx, a) : xpass_n<MODE, N, 16>(ctx, a);
      HE_FFT_SIZES(HE_CASE)
#undef HE_CASE
    }
  }
  return xpass_n<MODE, 0, 16>(ctx, a);
}

template <int N, int TILE>
static int ypass_n(he_ctx_t* ctx, const YZArgs& a, int narr) {
  const int tk = (N > 0) ? TILE : ctx->tkx;
  const size_t smem = fft_smem(ctx->ply, tk, 2);
  const int nthr = (N > 0) ? tile_threads(TILE) : 256;
  dim3 grid((ctx->nxh + tk - 1) / tk, ctx->nz, narr);
  CK(cudaFuncSetAttribute(k_ypass<N, TILE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  tname(ctx, "fft_y");
  k_ypass<N, TILE><<<grid, nthr, smem, ctx->stream>>>(a);
  LAUNCHED();
  return HE_OK;
}
static int ypass(he_ctx_t* ctx, double2* a0, double2* a1, bool inv) {
  YZArgs a{};
  a.nxh = ctx->nxh; a.ny = ctx->ny; a.nz = ctx->nz; a.tkx = ctx->tkx;
  a.pl = ctx->ply;
  a.arr[0] = a0; a.arr[1] = a1 ? a1 : a0;
  a.inv = inv;
  const int narr = a1 ? 2 : 1;
  const int tile = ctx->tile_y;
  if (yz_fast(ctx->ny)) {
    switch (ctx->ny) {
#define HE_CASE(N) \
  case N: return tile == 8 ? ypass_n<N, 8>(ctx, a, narr) : ypass_n<N, 16>(ctx, a, narr);
      HE_FFT_SIZES(HE_CASE)
#undef HE_CASE
    }
  }
  return ypass_n<0, 16>(ctx, a, narr);
}

template <int N, int TILE>
static int zconv_n(he_ctx_t* ctx, const YZArgs& a) {
  const int tk = (N > 0) ? TILE : ctx->tkx;
  const size_t smem = fft_smem(ctx->plz, tk, 3);
  const int nthr = (N > 0) ? tile_threads(TILE) : 256;
  dim3 grid((ctx->nxh + tk - 1) / tk, ctx->ny, 1);
  CK(cudaFuncSetAttribute(k_zconv<N, TILE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  tname(ctx, a.k2 ? "fft_z_conv2" : "fft_z_conv1");
  k_zconv<N, TILE><<<grid, nthr, smem, ctx->stream>>>(a);
  LAUNCHED();
  return HE_OK;
}
static int zconv(he_ctx_t* ctx, double2* io, const double* k1, double2* out2, const double* k2,
                 double2* fden_out) {
  YZArgs a{};
  a.nxh = ctx->nxh; a.ny = ctx->ny; a.nz = ctx->nz; a.tkx = ctx->tkx;
  a.pl = ctx->plz;
  a.io = io; a.out2 = out2; a.fden_out = fden_out; a.k1 = k1; a.k2 = k2;
  const int tile = ctx->tile_z;
  if (yz_fast(ctx->nz)) {
    switch (ctx->nz) {
#define HE_CASE(N) \
  case N: return tile == 8 ? zconv_n<N, 8>(ctx, a) : zconv_n<N, 16>(ctx, a);
      HE_FFT_SIZES(HE_CASE)
#undef HE_CASE
    }
  }
  return zconv_n<0, 16>(ctx, a);
}

// fden = R2C(den); wA <- fden*wcgk and wB <- fden*fvlj4 back in (x-transformed) row space.
static int spectrum_cg_lj(he_ctx_t* ctx) {
  XArgs a = xargs(ctx);
  a.den = ctx->den;
  a.specA = ctx->wA;
  TRY(xpass<X_R2C_DEN>(ctx, a));
  TRY(ypass(ctx, ctx->wA, nullptr, false));
  TRY(zconv(ctx, ctx->wA, ctx->wcgk, ctx->wB, ctx->fvlj4, ctx->fden));
  TRY(ypass(ctx, ctx->wA, ctx->wB, true));
  return HE_OK;
}
// Correlation convolution of the spectrum in wA (already x-transformed) and pot4 assembly.
static int correlation_tail(he_ctx_t* ctx) {
  TRY(ypass(ctx, ctx->wA, nullptr, false));
  TRY(zconv(ctx, ctx->wA, ctx->wcgk, nullptr, nullptr, nullptr));
  TRY(ypass(ctx, ctx->wA, nullptr, true));
  XArgs a = xargs(ctx);
  a.specA = ctx->wA;
  a.den = ctx->den; a.dencg_in = ctx->dencg; a.delj4_in = ctx->delj4;
  a.out1 = ctx->pot4;
  return xpass<X_C2R_POT>(ctx, a);
}

// ---- module-array access -----------------------------------------------------------------------
static size_t wf_elem(const he_ctx_t* ctx) {
  return ctx->mode == HE_MODE_DYNAMICS ? sizeof(double2) : sizeof(double);
}

static int imp_pull(he_ctx_t* ctx, ImpDev* h) {
  CK(cudaMemcpyAsync(h, ctx->imp, sizeof(ImpDev), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return HE_OK;
}
static int imp_push(he_ctx_t* ctx, const ImpDev* h) {
  CK(cudaMemcpyAsync(ctx->imp, h, sizeof(ImpDev), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return HE_OK;
}

struct FieldRef {
  void* ptr;
  size_t bytes;
  bool kspace_real;
};

static int field_ref(he_ctx_t* ctx, int field, FieldRef* r) {
  const size_t N = ctx->N, Nk = ctx->Nk;
  const size_t wf = wf_elem(ctx) * N;
  r->kspace_real = false;
  switch (field) {
    case HE_F_PSI: *r = {ctx->psi, wf, false}; return HE_OK;
    case HE_F_DEN: *r = {ctx->den, 8 * N, false}; return HE_OK;
    case HE_F_POT4: *r = {ctx->pot4, 8 * N, false}; return HE_OK;
    case HE_F_DENCG: *r = {ctx->dencg, 8 * N, false}; return HE_OK;
    case HE_F_DELJ4: *r = {ctx->delj4, 8 * N, false}; return HE_OK;
    case HE_F_UIMP:
      if (!ctx->uimp) break;
      *r = {ctx->uimp, 8 * N, false};
      return HE_OK;
    case HE_F_FDEN: *r = {ctx->fden, 16 * Nk, false}; return HE_OK;
    case HE_F_PC: *r = {ctx->pc, wf, false}; return HE_OK;
    case HE_F_Q: *r = {ctx->q, wf, false}; return HE_OK;
    case HE_F_PSIOLD1: case HE_F_PSIOLD2: case HE_F_PSIOLD3:
      *r = {ctx->psiold[field - HE_F_PSIOLD1], wf, false};
      return HE_OK;
    case HE_F_HPSIOLD1: case HE_F_HPSIOLD2:
      *r = {ctx->hpsiold[field - HE_F_HPSIOLD1], wf, false};
      return HE_OK;
    case HE_F_DXDEN: case HE_F_DYDEN: case HE_F_DZDEN: {
      double* p = field == HE_F_DXDEN ? ctx->dxden : field == HE_F_DYDEN ? ctx->dyden : ctx->dzden;
      if (!p) return fail(ctx, HE_ERR_STATE, "density gradients not materialised (call he_derden)");
      *r = {p, 8 * N, false};
      return HE_OK;
    }
    case HE_F_HPSI:
      if (!ctx->hpsi) break;
      *r = {ctx->hpsi, 8 * N, false};
      return HE_OK;
    case HE_F_FVLJ4: *r = {ctx->fvlj4, 8 * Nk, true}; return HE_OK;
    case HE_F_WCGK: *r = {ctx->wcgk, 8 * Nk, true}; return HE_OK;
    default: break;
  }
  return fail(ctx, HE_ERR_ARG, "field %d is not available in this context", field);
}

static double* imp_member(ImpDev* h, int field, size_t* count) {
  const int n = h->n;
  switch (field) {
    case HE_F_RIMP: *count = 3 * n; return h->rimp;
    case HE_F_VIMP: *count = 3 * n; return h->vimp;
    case HE_F_AIMP: *count = 3 * n; return h->aimp;
    case HE_F_FIMP: *count = 3 * n; return h->F;
    case HE_F_RIMPOLD: *count = 9 * n; return h->rimpold;
    case HE_F_VIMPOLD: *count = 9 * n; return h->vimpold;
    case HE_F_AIMPOLD: *count = 6 * n; return h->aimpold;
    case HE_F_PCR: *count = 3 * n; return h->pcr;
    case HE_F_PCV: *count = 3 * n; return h->pcv;
    case HE_F_QR: *count = 3 * n; return h->qr;
    case HE_F_QV: *count = 3 * n; return h->qv;
    default: return nullptr;
  }
}

// ------------------------------------------------------------------------------------------------
// statics pointwise kernels (He_statics/steprkr.f90, steppcr.f90, evolo.f90, varmu.f90)
// ------------------------------------------------------------------------------------------------
namespace {

struct StatPW {
  long N;
  double dxyz, n4, dt, dtmin, sdmu, dmumax;
  const double* sums;
  double* psi;        // current psi (read)
  double* out;        // destination of the new psi
  double* po3;
  const double* po2;
  const double* h1;
  double* h2;
  double* pc;
  double* q;
  double* hsave;
  const double* hpsi;  // H psi (predictor / RK) or t4 (corrector)
  double* timec;
  double* den;
  double a, b, c;
  int jr;
};

__device__ __forceinline__ double local_dt(double hp, double ps, const StatPW& s) {
  return s.dt / (1.0 + exp((fabs(hp / ps) - s.dmumax) / s.sdmu)) + s.dtmin;
}

// steppcr predictor + modifier (steppcr.f90:40-61); acc = sum psi_new^2.
__global__ void __launch_bounds__(256) k_stat_predict(const StatPW s, const ReduceTail rt) {
  const double c112 = 112.0 / 121.0, c4o3 = 4.0 / 3.0;
  const double hmean = s.sums[S_STAT_H] * s.dxyz / s.n4;
  double acc[1] = {0.0};
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < s.N;
       i += (long)gridDim.x * blockDim.x) {
    const double ps = s.psi[i], hp = s.hpsi[i];
    const double tc = local_dt(hp, ps, s);
    s.timec[i] = tc;
    const double s4 = -(hp - hmean * ps);
    const double sto1 = s.po3[i] + c4o3 * tc * (2.0 * s4 - s.h1[i] + 2.0 * s.h2[i]);
    const double pn = sto1 - c112 * s.pc[i];
    s.po3[i] = pn;
    s.pc[i] = sto1;
    s.h2[i] = s4;
    acc[0] += pn * pn;
  }
  block_reduce_store<1>(acc, rt.partials + blockIdx.x);
  reduce_tail<1>(rt, gridDim.x);
}

// steppcr corrector + final value (steppcr.f90:78-90); acc = {sum |pc|, sum psi_new^2}.
__global__ void __launch_bounds__(256) k_stat_correct(const StatPW s, const ReduceTail rt) {
  const double c9 = 9.0 / 121.0;
  const double mu = s.sums[S_STAT_MU] * s.dxyz / s.n4;
  double acc[2] = {0.0, 0.0};
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < s.N;
       i += (long)gridDim.x * blockDim.x) {
    const double ps = s.psi[i];
    const double s4 = -(s.hpsi[i] - mu * ps);
    const double s5 =
        0.125 * (9.0 * s.po3[i] - s.po2[i] + 3.0 * s.timec[i] * (s4 + 2.0 * s.h1[i] - s.h2[i]));
    const double p = s.pc[i] - s5;
    s.pc[i] = p;
    const double o = s5 + c9 * p;
    s.out[i] = o;
    acc[0] += fabs(p);
    acc[1] += o * o;
  }
  block_reduce_store<2>(acc, rt.partials + 2 * blockIdx.x);
  reduce_tail<2>(rt, gridDim.x);
}

// steprkr stage update (steprkr.f90:160-179); acc = sum psi_new^2.
__global__ void __launch_bounds__(256) k_stat_rk(const StatPW s, const ReduceTail rt) {
  const double err = s.sums[S_STAT_H] * s.dxyz / s.n4;
  double acc[1] = {0.0};
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < s.N;
       i += (long)gridDim.x * blockDim.x) {
    const double ps = s.psi[i], hp = s.hpsi[i];
    if (s.jr == 0) s.timec[i] = local_dt(hp, ps, s);
    const double tc = s.timec[i];
    const double s4 = -(hp - err * ps);
    const double s1 = s.a * (s4 - s.b * s.q[i]);
    s.q[i] = s.q[i] + 3.0 * s1 - s.c * s4;
    if (s.hsave) s.hsave[i] = s4;
    const double o = ps + tc * s1;
    s.out[i] = o;
    acc[0] += o * o;
  }
  block_reduce_store<1>(acc, rt.partials + blockIdx.x);
  reduce_tail<1>(rt, gridDim.x);
}

// psi = |psi| * sqrt(n4/(sum psi^2 dxyz)); den = psi^2.
__global__ void __launch_bounds__(256) k_stat_normalize(double* psi, double* den, long N,
                                                        const double* sums, double n4,
                                                        double dxyz) {
  const double cnorm = sqrt(n4 / (sums[S_STAT_N] * dxyz));
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < N;
       i += (long)gridDim.x * blockDim.x) {
    const double v = fabs(psi[i]) * cnorm;
    psi[i] = v;
    den[i] = v * v;
  }
}

__global__ void __launch_bounds__(256) k_sumsq(const double* psi, long N, const ReduceTail rt) {
  double acc[1] = {0.0};
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < N;
       i += (long)gridDim.x * blockDim.x)
    acc[0] += psi[i] * psi[i];
  block_reduce_store<1>(acc, rt.partials + blockIdx.x);
  reduce_tail<1>(rt, gridDim.x);
}

// varmu: sum |hpsi - mu psi| * psi (varmu.f90:31).
__global__ void __launch_bounds__(256) k_varmu(const double* hpsi, const double* psi, long N,
                                               double mu, const ReduceTail rt) {
  double acc[1] = {0.0};
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < N;
       i += (long)gridDim.x * blockDim.x)
    acc[0] += fabs(hpsi[i] - mu * psi[i]) * psi[i];
  block_reduce_store<1>(acc, rt.partials + blockIdx.x);
  reduce_tail<1>(rt, gridDim.x);
}

__global__ void k_copy_slot(double* sums, int dst, int src) {
  if (threadIdx.x == 0 && blockIdx.x == 0) sums[dst] = sums[src];
}

}  // namespace

static int pw_blocks(const he_ctx_t* ctx) {
  long b = (ctx->N + 255) / 256;
  return (int)(b < kPwBlocks ? b : kPwBlocks);
}

template <int NI>
static int launch_impfield(he_ctx_t* ctx) {
  OpImpField<NI> op{};
  op.tab = ctx->pot_tab; op.imp = ctx->imp; op.uimp = ctx->uimp;
  op.n = ctx->n_imp; op.npot = ctx->npot;
  op.delinter = ctx->delinter; op.rmax = ctx->rmaxinterpol;
  op.xmax = ctx->xmax; op.ymax = ctx->ymax; op.zmax = ctx->zmax;
  op.hx = ctx->hx; op.hy = ctx->hy; op.hz = ctx->hz;
  return run_stencil_red(ctx, ctx->g1, ctx->den, op, S_FORCE);
}

static int field_eval(he_ctx_t* ctx) {  // potenimp; poten; forceimp
  TRY(he_potenimp(ctx));
  TRY(he_poten(ctx));
  return he_forceimp(ctx, nullptr);
}

static double host_pair_pot(const ImpDev& s, double r) {
  if (s.ii_kind == 0) return (r < s.ii_rcut) ? s.ii_umax : 0.0;
  if (r < s.ii_rcut) return s.ii_umax;
  const double e = 1.0 - std::exp(-s.ii_a * (r - s.ii_re));
  return s.ii_D * (e * e - 1.0);
}

static StatPW statpw(he_ctx_t* ctx, double dt, int n4) {
  StatPW s{};
  s.N = ctx->N;
  s.dxyz = ctx->dxyz;
  s.n4 = (double)n4;
  s.dt = dt;
  s.dtmin = 1.0e-10; s.sdmu = 1.0e-1; s.dmumax = 1.0e2;  // He_statics/modules.f90:299
  s.sums = ctx->sums;
  s.timec = ctx->timec;
  s.den = ctx->den;
  return s;
}

static int stat_hpsi(he_ctx_t* ctx, double* out, int slot) {
  OpHpsiR op{};
  op.s8[0] = ctx->pot4;
  op.out = out;
  op.h2o2m = ctx->fn.h2o2m4;
  return run_stencil_red(ctx, ctx->g2, (const double*)ctx->psi, op, slot);
}

static int stat_normalize(he_ctx_t* ctx, int n4) {
  tname(ctx, "statics_normalize");
  k_stat_normalize<<<pw_blocks(ctx), 256, 0, ctx->stream>>>((double*)ctx->psi, ctx->den, ctx->N,
                                                            ctx->sums, (double)n4, ctx->dxyz);
  LAUNCHED();
  return HE_OK;
}

static int read_sums(he_ctx_t* ctx) {
  CK(cudaMemcpyAsync(ctx->hsum, ctx->sums, S_COUNT * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return HE_OK;
}

// Tile autotuner: times the 16-line and 8-line variants of each FFT pass family on this
// context's grid (zero-filled work arrays, one warm-up and three timed launches each) and keeps
// the faster.  Runs once in he_ctx_create.
static int autotune_tiles(he_ctx_t* ctx) {
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  auto timed = [&](int (*fn)(he_ctx_t*), float* ms) -> int {
    TRY(fn(ctx));
    CK(cudaEventRecord(e0, ctx->stream));
    for (int r = 0; r < 3; ++r) TRY(fn(ctx));
    CK(cudaEventRecord(e1, ctx->stream));
    CK(cudaEventSynchronize(e1));
    CK(cudaEventElapsedTime(ms, e0, e1));
    return HE_OK;
  };
  auto pick = [&](int* knob, int (*fn)(he_ctx_t*)) -> int {
    float t16 = 0.0f, t8 = 0.0f;
    *knob = 16;
    TRY(timed(fn, &t16));
    *knob = 8;
    TRY(timed(fn, &t8));
    *knob = (t8 < t16) ? 8 : 16;
    return HE_OK;
  };
  int st = HE_OK;
  if (x_fast(ctx, 16) && x_fast(ctx, 8))
    st = pick(&ctx->tile_x, [](he_ctx_t* c) -> int {
      XArgs a = xargs(c);
      a.specA = c->wA; a.specB = c->wB; a.den = c->den;
      a.out1 = c->dencg; a.out2 = c->delj4;
      return xpass<X_C2R2_CORR>(c, a);
    });
  if (st == HE_OK && yz_fast(ctx->ny))
    st = pick(&ctx->tile_y, [](he_ctx_t* c) -> int { return ypass(c, c->wA, c->wB, true); });
  if (st == HE_OK && yz_fast(ctx->nz))
    st = pick(&ctx->tile_z, [](he_ctx_t* c) -> int {
      return zconv(c, c->wA, c->wcgk, c->wB, c->fvlj4, nullptr);
    });
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (st == HE_OK) CK(cudaMemsetAsync(ctx->wA, 0, 16 * ctx->Nk, ctx->stream));
  if (st == HE_OK) CK(cudaMemsetAsync(ctx->wB, 0, 16 * ctx->Nk, ctx->stream));
  return st;
}

// ------------------------------------------------------------------------------------------------
// C-ABI
// ------------------------------------------------------------------------------------------------
extern "C" {

int he_ctx_create(const he_grid_t* grid, const he_functional_t* fun, int mode, int precision,
                  he_ctx_t** out) {
  if (!out) return HE_ERR_ARG;
  *out = nullptr;
  if (!grid || !fun) return HE_ERR_ARG;
  he_ctx_t* ctx = new he_ctx_t();
  int st = HE_OK;
  auto bad = [&](int code, const char* msg) {
    ctx->err = msg;
    st = code;
  };
  if (mode != HE_MODE_DYNAMICS && mode != HE_MODE_STATICS) bad(HE_ERR_ARG, "unknown mode");
  else if (precision != HE_PREC_F64) bad(HE_ERR_ARG, "unknown precision");
  else if (grid->npd != 13) bad(HE_ERR_ARG, "npd must be 13");
  else if (grid->icon != 13 && grid->icon != 8 && grid->icon != 18)
    bad(HE_ERR_ARG, "icon must be 13, 8 or 18");
  else if (!tstgrid_ok(grid->nx) || !tstgrid_ok(grid->ny) || !tstgrid_ok(grid->nz))
    bad(HE_ERR_ARG, "grid size is not an admissible tstgrid value");
  else if (grid->nx % 2 || grid->ny < 2 || (grid->ny * (long)grid->nz) % 2)
    bad(HE_ERR_ARG, "nx must be even and ny*nz even");
  else if (!factor_ok(grid->nx) || !factor_ok(grid->ny) || !factor_ok(grid->nz))
    bad(HE_ERR_ARG, "grid size must be 2^a 3^b 5^c");
  else if (grid->xmax == 0.0 || grid->ymax == 0.0 || grid->zmax == 0.0)
    bad(HE_ERR_ARG, "xmax, ymax, zmax must be non-zero");
  if (st == HE_OK) {
    if (std::strncmp(fun->core4, "OTC", 3) == 0) bad(HE_ERR_ARG, "core4='OTC' (alpha_s term) is not built yet");
    else if (std::strncmp(fun->core4, "OP", 2) != 0 && std::strncmp(fun->core4, "OT", 2) != 0)
      bad(HE_ERR_ARG, "core4 must be 'OT ', 'OP ' or 'OTC'");
  }
  if (st != HE_OK) {
    *out = ctx;
    return st;
  }
  ctx->mode = mode;
  ctx->prec = precision;
  ctx->nx = grid->nx; ctx->ny = grid->ny; ctx->nz = grid->nz;
  ctx->nxh = grid->nx / 2 + 1;
  ctx->N = (long)grid->nx * grid->ny * grid->nz;
  ctx->Nk = (long)ctx->nxh * grid->ny * grid->nz;
  ctx->xmax = grid->xmax; ctx->ymax = grid->ymax; ctx->zmax = grid->zmax;
  ctx->hx = 2.0 * std::fabs(grid->xmax) / grid->nx;
  ctx->hy = 2.0 * std::fabs(grid->ymax) / grid->ny;
  ctx->hz = 2.0 * std::fabs(grid->zmax) / grid->nz;
  ctx->dxyz = ctx->hx * ctx->hy * ctx->hz;
  ctx->renor = 1.0 / (double)ctx->N;
  ctx->icon = grid->icon;
  ctx->fn = *fun;
  ctx->op_core = std::strncmp(fun->core4, "OP", 2) == 0;
  bickley13(ctx->w1, ctx->w2);
  make_geom(ctx, 1, &ctx->g1);
  make_geom(ctx, 2, &ctx->g2);
  *out = ctx;

  {
    int dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess)
      cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, dev);
  }
  cudaError_t e = cudaStreamCreateWithFlags(&ctx->own, cudaStreamNonBlocking);
  if (e != cudaSuccess)
    return fail(ctx, HE_ERR_CUDA, "cudaStreamCreate failed: %s", cudaGetErrorString(e));
  ctx->stream = ctx->own;

  // FFT plans and shared-memory budgets
  TRY(make_plan(ctx, ctx->nx, &ctx->plx));
  TRY(make_plan(ctx, ctx->ny, &ctx->ply));
  TRY(make_plan(ctx, ctx->nz, &ctx->plz));
  const int nmax = std::max(ctx->nx, std::max(ctx->ny, ctx->nz));
  ctx->tkx = tile_rows(nmax);
  ctx->x_rb = tile_rows(ctx->nx);
  while (ctx->x_rb > 2 && ((long)ctx->ny * ctx->nz) % ctx->x_rb) ctx->x_rb -= 2;
  ctx->smem_x = fft_smem(ctx->plx, tile_rows(ctx->nx), 2);
  ctx->smem_y = fft_smem(ctx->ply, ctx->tkx, 2);
  ctx->smem_z = fft_smem(ctx->plz, ctx->tkx, 3);
  int maxsm = 0, dev = 0;
  CK(cudaGetDevice(&dev));
  CK(cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  if ((int)ctx->smem_x > maxsm || (int)ctx->smem_y > maxsm || (int)ctx->smem_z > maxsm)
    return fail(ctx, HE_ERR_ARG, "grid too large for the shared-memory FFT passes");

  const size_t N = ctx->N, Nk = ctx->Nk;
  TRY(dalloc_t(ctx, &ctx->fden, Nk));
  TRY(dalloc_t(ctx, &ctx->wA, Nk));
  TRY(dalloc_t(ctx, &ctx->wB, Nk));
  TRY(dalloc_t(ctx, &ctx->fvlj4, Nk));
  TRY(dalloc_t(ctx, &ctx->wcgk, Nk));
  TRY(dalloc_t(ctx, &ctx->den, N));
  TRY(dalloc_t(ctx, &ctx->pot4, N));
  TRY(dalloc_t(ctx, &ctx->dencg, N));
  TRY(dalloc_t(ctx, &ctx->delj4, N));
  const size_t wf = wf_elem(ctx) * N;
  TRY(dalloc(ctx, &ctx->psi, wf));
  for (int s = 0; s < 3; ++s) TRY(dalloc(ctx, &ctx->psiold[s], wf));
  for (int s = 0; s < 2; ++s) TRY(dalloc(ctx, &ctx->hpsiold[s], wf));
  TRY(dalloc(ctx, &ctx->pc, wf));
  TRY(dalloc(ctx, &ctx->q, wf));
  TRY(dalloc(ctx, &ctx->scratch, wf));
  if (mode == HE_MODE_DYNAMICS) {
    TRY(dalloc_t(ctx, &ctx->uimp, N));
    TRY(dalloc_t(ctx, &ctx->tabx, ctx->nx));
    TRY(dalloc_t(ctx, &ctx->taby, ctx->ny));
    TRY(dalloc_t(ctx, &ctx->tabz, ctx->nz));
    TRY(dalloc_t(ctx, &ctx->imp, 1));
    he_absorber_t ab = {2.0, 1000.0, 2.0, 1000.0, 2.0, 1000.0, 2.0};  // DFT4He3d.f90:136-138
    TRY(he_set_absorber(ctx, &ab));
  } else {
    TRY(dalloc_t(ctx, &ctx->hpsi, N));
    TRY(dalloc_t(ctx, &ctx->t4, N));
    TRY(dalloc_t(ctx, &ctx->timec, N));
  }
  StencilGeom g4 = ctx->g2;
  g4.zc = 4;  // the smallest z-chunk choose_zc can pick
  dim3 sg = stencil_grid(ctx, g4);
  ctx->partials_cap = std::max((size_t)sg.x * sg.y * sg.z, (size_t)kPwBlocks) * (3 * kMaxImp);
  TRY(dalloc_t(ctx, &ctx->partials, ctx->partials_cap));
  TRY(dalloc_t(ctx, &ctx->counter, 1));
  TRY(dalloc_t(ctx, &ctx->sums, S_COUNT));
  CK(cudaMallocHost(&ctx->hsum, S_COUNT * sizeof(double)));
  TRY(autotune_tiles(ctx));
  CK(cudaStreamSynchronize(ctx->stream));
  return HE_OK;
}

void he_ctx_destroy(he_ctx_t* ctx) {
  if (!ctx) return;
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  for (void* p : ctx->allocs) cudaFree(p);
  if (ctx->hsum) cudaFreeHost(ctx->hsum);
  for (cudaEvent_t e : ctx->evpool) cudaEventDestroy(e);
  if (ctx->own) cudaStreamDestroy(ctx->own);
  delete ctx;
}

const char* he_last_error(const he_ctx_t* ctx) { return ctx ? ctx->err.c_str() : "null context"; }
long long he_launch_count(const he_ctx_t* ctx) { return ctx ? ctx->launches : 0; }
size_t he_device_bytes(const he_ctx_t* ctx) { return ctx ? ctx->bytes : 0; }

int he_set_stream(he_ctx_t* ctx, void* stream) {
  if (!ctx) return HE_ERR_ARG;
  CK(cudaStreamSynchronize(ctx->stream));
  ctx->stream = stream ? (cudaStream_t)stream : ctx->own;
  return HE_OK;
}

int he_synchronize(he_ctx_t* ctx) {
  if (!ctx) return HE_ERR_ARG;
  CK(cudaStreamSynchronize(ctx->stream));
  return HE_OK;
}

int he_set_kernels(he_ctx_t* ctx, const double* fvlj4, const double* wcgk, const double* kalfs) {
  if (!ctx || !fvlj4 || !wcgk) return fail(ctx, HE_ERR_ARG, "null kernel array");
  (void)kalfs;
  CK(cudaMemcpyAsync(ctx->fvlj4, fvlj4, 8 * ctx->Nk, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(ctx->wcgk, wcgk, 8 * ctx->Nk, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  ctx->kernels_ok = true;
  return HE_OK;
}

int he_compute_kernels(he_ctx_t* ctx) {
  if (!ctx) return HE_ERR_ARG;
  KernArgs a{};
  a.nx = ctx->nx; a.ny = ctx->ny; a.nz = ctx->nz; a.nxh = ctx->nxh;
  a.hx = ctx->hx; a.hy = ctx->hy; a.hz = ctx->hz;
  a.op_core = ctx->op_core; a.otc = 0;
  a.eps = ctx->fn.eps4; a.sigma = ctx->fn.sigma4; a.hc = ctx->fn.h4; a.l = ctx->fn.l;
  a.fvlj4 = ctx->fvlj4; a.wcgk = ctx->wcgk; a.kalfs = ctx->kalfs;
  tname(ctx, "kspace_kernels");
  k_kernels<<<kPwBlocks, 256, 0, ctx->stream>>>(a);
  LAUNCHED();
  CK(cudaStreamSynchronize(ctx->stream));
  ctx->kernels_ok = true;
  return HE_OK;
}

int he_set_absorber(he_ctx_t* ctx, const he_absorber_t* ab) {
  if (!ctx || !ab) return fail(ctx, HE_ERR_ARG, "null absorber");
  if (ctx->mode != HE_MODE_DYNAMICS) return fail(ctx, HE_ERR_STATE, "absorber is a dynamics setting");
  auto tab = [&](int n, double xm, double h, double mean, double surf, double* dst) -> int {
    std::vector<double> t(n);
    for (int i = 0; i < n; ++i) t[i] = std::tanh((std::fabs(-xm + h * i) - mean) / surf);
    CK(cudaMemcpyAsync(dst, t.data(), 8 * n, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return HE_OK;
  };
  TRY(tab(ctx->nx, ctx->xmax, ctx->hx, ab->txmean, ab->txsurf, ctx->tabx));
  TRY(tab(ctx->ny, ctx->ymax, ctx->hy, ab->tymean, ab->tysurf, ctx->taby));
  TRY(tab(ctx->nz, ctx->zmax, ctx->hz, ab->tzmean, ab->tzsurf, ctx->tabz));
  ctx->lambdah = ab->lambdah;
  return HE_OK;
}

int he_set_impurities(he_ctx_t* ctx, const he_impurities_t* im) {
  if (!ctx || !im) return fail(ctx, HE_ERR_ARG, "null impurity description");
  if (ctx->mode != HE_MODE_DYNAMICS) return fail(ctx, HE_ERR_STATE, "impurities are a dynamics setting");
  if (im->n_imp < 0 || im->n_imp > kMaxImp)
    return fail(ctx, HE_ERR_ARG, "n_imp must be in [0, %d]", kMaxImp);
  if (im->n_imp > 0 && (!im->potion || !im->m_imp_u || im->npot < 2 || im->delinter <= 0))
    return fail(ctx, HE_ERR_ARG, "incomplete impurity table");
  ImpDev h;
  std::memset(&h, 0, sizeof(h));
  h.n = im->n_imp;
  for (int k = 0; k < im->n_imp; ++k) h.m[k] = im->m_imp_u[k] * kMpU;
  for (int i = 0; i < 3; ++i) { h.ioldr[i] = i + 1; h.ioldv[i] = i + 1; }
  h.iolda[0] = 1; h.iolda[1] = 2;
  h.lgridnoout = 1;
  h.ii_kind = im->ii_kind; h.ii_D = im->ii_D; h.ii_re = im->ii_re; h.ii_a = im->ii_a;
  h.ii_rcut = im->ii_rcut; h.ii_umax = im->ii_umax;
  TRY(imp_push(ctx, &h));
  ctx->n_imp = im->n_imp;
  if (im->n_imp > 0) {
    const size_t need = (size_t)im->npot * im->n_imp;
    if (need > ctx->pot_tab_cap) {
      TRY(dalloc_t(ctx, &ctx->pot_tab, need));
      ctx->pot_tab_cap = need;
    }
    std::vector<double> t((size_t)im->npot * im->n_imp);
    for (int k = 0; k < im->n_imp; ++k)
      for (int i = 0; i < im->npot; ++i) t[(size_t)k * im->npot + i] = im->potion[k + (size_t)im->n_imp * i];
    CK(cudaMemcpyAsync(ctx->pot_tab, t.data(), 8 * t.size(), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
  }
  ctx->npot = im->npot;
  ctx->delinter = im->delinter;
  ctx->rmaxinterpol = im->rmaxinterpol;
  ctx->force_fresh = false;
  return HE_OK;
}

int he_upload(he_ctx_t* ctx, int field, const void* host, size_t bytes) {
  if (!ctx || !host) return fail(ctx, HE_ERR_ARG, "null argument");
  if (field >= HE_F_RIMP && field <= HE_F_QV) {
    if (ctx->mode != HE_MODE_DYNAMICS) return fail(ctx, HE_ERR_STATE, "no impurities in statics");
    ImpDev h;
    TRY(imp_pull(ctx, &h));
    size_t cnt = 0;
    double* m = imp_member(&h, field, &cnt);
    if (!m || bytes != cnt * 8) return fail(ctx, HE_ERR_ARG, "field %d: expected %zu bytes", field, cnt * 8);
    std::memcpy(m, host, bytes);
    TRY(imp_push(ctx, &h));
    ctx->force_fresh = false;
    return HE_OK;
  }
  if (field == HE_F_RING) return fail(ctx, HE_ERR_ARG, "ring indices are read-only");
  FieldRef r;
  TRY(field_ref(ctx, field, &r));
  if (bytes != r.bytes) return fail(ctx, HE_ERR_ARG, "field %d: expected %zu bytes, got %zu", field, r.bytes, bytes);
  CK(cudaMemcpyAsync(r.ptr, host, bytes, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  if (field == HE_F_FVLJ4 || field == HE_F_WCGK) ctx->kernels_ok = true;
  if (field == HE_F_DEN) ctx->force_fresh = false;
  return HE_OK;
}

int he_download(he_ctx_t* ctx, int field, void* host, size_t bytes) {
  if (!ctx || !host) return fail(ctx, HE_ERR_ARG, "null argument");
  if (field == HE_F_RING) {
    if (bytes != 13 * 8) return fail(ctx, HE_ERR_ARG, "ring: expected 104 bytes");
    double* o = (double*)host;
    for (int i = 0; i < 3; ++i) o[i] = ctx->ioldp[i];
    for (int i = 0; i < 2; ++i) o[3 + i] = ctx->ioldh[i];
    if (ctx->mode == HE_MODE_DYNAMICS) {
      ImpDev h;
      TRY(imp_pull(ctx, &h));
      for (int i = 0; i < 3; ++i) { o[5 + i] = h.ioldr[i]; o[8 + i] = h.ioldv[i]; }
      for (int i = 0; i < 2; ++i) o[11 + i] = h.iolda[i];
    } else {
      for (int i = 5; i < 13; ++i) o[i] = 0.0;
    }
    return HE_OK;
  }
  if (field >= HE_F_RIMP && field <= HE_F_QV) {
    if (ctx->mode != HE_MODE_DYNAMICS) return fail(ctx, HE_ERR_STATE, "no impurities in statics");
    ImpDev h;
    TRY(imp_pull(ctx, &h));
    size_t cnt = 0;
    double* m = imp_member(&h, field, &cnt);
    if (!m || bytes != cnt * 8) return fail(ctx, HE_ERR_ARG, "field %d: expected %zu bytes", field, cnt * 8);
    std::memcpy(host, m, bytes);
    return HE_OK;
  }
  FieldRef r;
  TRY(field_ref(ctx, field, &r));
  if (bytes != r.bytes) return fail(ctx, HE_ERR_ARG, "field %d: expected %zu bytes, got %zu", field, r.bytes, bytes);
  CK(cudaMemcpyAsync(host, r.ptr, bytes, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return HE_OK;
}

// ---- Dynamics_TDDFT ------------------------------------------------------------------------------
int he_poten(he_ctx_t* ctx) {
  if (!ctx) return HE_ERR_ARG;
  if (!ctx->kernels_ok) return fail(ctx, HE_ERR_STATE, "k-space kernels not set");
  if (ctx->mode == HE_MODE_STATICS) {
    // He_statics/poten.f90:27-115: delj4 from the last refreshed fden (cached by
    // he_refresh_density), correlation with the current den and the stale dencg.
    XArgs a = xargs(ctx);
    a.den = ctx->den; a.dencg_in = ctx->dencg;
    a.specA = ctx->wA;
    TRY(xpass<X_R2C_CORR>(ctx, a));
    return correlation_tail(ctx);
  }
  TRY(spectrum_cg_lj(ctx));
  XArgs a = xargs(ctx);
  a.specA = ctx->wA; a.specB = ctx->wB;
  a.den = ctx->den;
  a.out1 = ctx->dencg; a.out2 = ctx->delj4;
  TRY(xpass<X_C2R2_CORR>(ctx, a));
  return correlation_tail(ctx);
}


int he_potenimp(he_ctx_t* ctx) {
  if (!ctx) return HE_ERR_ARG;
  if (ctx->mode != HE_MODE_DYNAMICS) return fail(ctx, HE_ERR_STATE, "potenimp is a dynamics routine");
  if (ctx->n_imp == 0) {
    ctx->force_fresh = true;
    return HE_OK;
  }
  int st;
  if (ctx->n_imp <= 1) st = launch_impfield<1>(ctx);
  else if (ctx->n_imp <= 2) st = launch_impfield<2>(ctx);
  else if (ctx->n_imp <= 4) st = launch_impfield<4>(ctx);
  else st = launch_impfield<8>(ctx);
  if (st == HE_OK) ctx->force_fresh = true;
  return st;
}

int he_forceimp(he_ctx_t* ctx, double* F) {
  if (!ctx) return HE_ERR_ARG;
  if (ctx->mode != HE_MODE_DYNAMICS) return fail(ctx, HE_ERR_STATE, "forceimp is a dynamics routine");
  if (ctx->n_imp == 0) return HE_OK;
  // The fused field pass of he_potenimp accumulated sum(grad den * uimp_k) for the current den and
  // rimp; redo it if either changed since.
  if (!ctx->force_fresh) TRY(he_potenimp(ctx));
  tname(ctx, "impurity_force");
  k_imp_force<<<1, 128, 0, ctx->stream>>>(ctx->imp, ctx->sums + S_FORCE, ctx->dxyz);
  LAUNCHED();
  if (F) {
    ImpDev h;
    TRY(imp_pull(ctx, &h));
    std::memcpy(F, h.F, sizeof(double) * 3 * ctx->n_imp);
  }
  return HE_OK;
}

int he_set_accel(he_ctx_t* ctx) {
  if (!ctx) return HE_ERR_ARG;
  if (ctx->mode != HE_MODE_DYNAMICS) return fail(ctx, HE_ERR_STATE, "dynamics routine");
  if (ctx->n_imp == 0) return HE_OK;
  tname(ctx, "impurity_accel");
  k_imp_accel<<<1, 128, 0, ctx->stream>>>(ctx->imp);
  LAUNCHED();
  return HE_OK;
}


int he_steprk(he_ctx_t* ctx, double deltat) {
  if (!ctx) return HE_ERR_ARG;
  if (ctx->mode != HE_MODE_DYNAMICS) return fail(ctx, HE_ERR_STATE, "steprk is a dynamics routine");
  const double r2 = 1.0 / std::sqrt(2.0);
  const double arun[4] = {0.5, 1.0 - r2, 1.0 + r2, 1.0 / 6.0};
  const double brun[4] = {2.0, 1.0, 1.0, 2.0};
  const double crun[4] = {0.5, 1.0 - r2, 1.0 + r2, 0.5};
  for (int jr = 0; jr < 4; ++jr) {
    OpRK op{};
    op.s8[0] = ctx->pot4; op.s8[1] = ctx->uimp;
    op.s16[0] = (const double2*)ctx->q;
    op.q = (double2*)ctx->q;
    op.out = (double2*)(jr == 0 ? ctx->psiold[2] : ctx->scratch);
    op.hsave = jr == 0 ? (double2*)ctx->hpsiold[1] : nullptr;
    op.den = ctx->den;
    op.tm = timec_view(ctx);
    op.h2o2m = ctx->fn.h2o2m4;
    op.a = arun[jr]; op.b = brun[jr]; op.cc = crun[jr]; op.dt = deltat;
    TRY(run_stencil(ctx, ctx->g2, (const double2*)ctx->psi, op));
    if (jr == 0) {
      // psiold(3)=psiold(2), psiold(2)=psiold(1), psiold(1)=psi; hpsiold(2)=hpsiold(1),
      // hpsiold(1)=H psi -- done by relabelling buffers (steprk.f90:251-257).
      void* o3 = ctx->psiold[2];
      ctx->psiold[2] = ctx->psiold[1];
      ctx->psiold[1] = ctx->psiold[0];
      ctx->psiold[0] = ctx->psi;
      ctx->psi = o3;
      std::swap(ctx->hpsiold[0], ctx->hpsiold[1]);
    } else {
      std::swap(ctx->psi, ctx->scratch);
    }
    ctx->force_fresh = false;
    if (ctx->n_imp > 0) {
      tname(ctx, "impurity_rk");
      k_imp_rk<<<1, 128, 0, ctx->stream>>>(ctx->imp, jr, arun[jr], brun[jr], crun[jr], deltat);
      LAUNCHED();
    }
    if (jr <= 2) TRY(field_eval(ctx));
  }
  for (int i = 0; i < 3; ++i) ctx->ioldp[i] = i + 1;
  ctx->ioldh[0] = 1; ctx->ioldh[1] = 2;
  return HE_OK;
}

int he_steppc(he_ctx_t* ctx, double deltat, double* errHe, double* errimp, double* errvimp) {
  if (!ctx) return HE_ERR_ARG;
  if (ctx->mode != HE_MODE_DYNAMICS) return fail(ctx, HE_ERR_STATE, "steppc is a dynamics routine");
  const double c112 = 112.0 / 121.0, c9 = 9.0 / 121.0, c4o3 = 4.0 / 3.0;
  {
    OpPredict op{};
    op.s8[0] = ctx->pot4; op.s8[1] = ctx->uimp;
    op.po3 = (double2*)ctx->psiold[ctx->ioldp[2] - 1];
    op.h2 = (double2*)ctx->hpsiold[ctx->ioldh[1] - 1];
    op.pc = (double2*)ctx->pc;
    op.s16[0] = op.po3;
    op.s16[1] = (const double2*)ctx->hpsiold[ctx->ioldh[0] - 1];
    op.s16[2] = op.h2;
    op.s16[3] = op.pc;
    op.den = ctx->den;
    op.tm = timec_view(ctx);
    op.h2o2m = ctx->fn.h2o2m4;
    op.s43 = c4o3 * deltat;
    op.c112 = c112;
    TRY(run_stencil(ctx, ctx->g2, (const double2*)ctx->psi, op));
    std::swap(ctx->psi, ctx->psiold[ctx->ioldp[2] - 1]);
    std::swap(ctx->ioldh[0], ctx->ioldh[1]);
  }
  ctx->force_fresh = false;
  if (ctx->n_imp > 0) {
    tname(ctx, "impurity_predict");
    k_imp_predict<<<1, 128, 0, ctx->stream>>>(ctx->imp, deltat);
    LAUNCHED();
  }
  TRY(field_eval(ctx));
  {
    OpCorrect op{};
    op.s8[0] = ctx->pot4; op.s8[1] = ctx->uimp;
    op.s16[0] = (const double2*)ctx->psiold[ctx->ioldp[2] - 1];
    op.s16[1] = (const double2*)ctx->psiold[ctx->ioldp[1] - 1];
    op.s16[2] = (const double2*)ctx->hpsiold[ctx->ioldh[0] - 1];
    op.s16[3] = (const double2*)ctx->hpsiold[ctx->ioldh[1] - 1];
    op.s16[4] = (const double2*)ctx->pc;
    op.pc = (double2*)ctx->pc;
    op.out = (double2*)ctx->scratch;
    op.den = ctx->den;
    op.tm = timec_view(ctx);
    op.h2o2m = ctx->fn.h2o2m4;
    op.s3 = 3.0 * deltat;
    op.c9 = c9;
    TRY(run_stencil_red(ctx, ctx->g2, (const double2*)ctx->psi, op, S_ERRHE));
    std::swap(ctx->psi, ctx->scratch);
    const int a = ctx->ioldp[2];
    ctx->ioldp[2] = ctx->ioldp[1];
    ctx->ioldp[1] = ctx->ioldp[0];
    ctx->ioldp[0] = a;
  }
  ctx->force_fresh = false;
  if (ctx->n_imp > 0) {
    tname(ctx, "impurity_correct");
    k_imp_correct<<<1, 128, 0, ctx->stream>>>(ctx->imp, deltat);
    LAUNCHED();
  }
  if (errHe || errimp || errvimp) {
    CK(cudaMemcpyAsync(ctx->hsum, ctx->sums, S_COUNT * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    ImpDev h;
    if (ctx->n_imp > 0) TRY(imp_pull(ctx, &h));
    CK(cudaStreamSynchronize(ctx->stream));
    if (errHe) *errHe = c9 * ctx->hsum[S_ERRHE] / (double)ctx->N;
    if (errimp) *errimp = ctx->n_imp > 0 ? h.errimp : 0.0;
    if (errvimp) *errvimp = ctx->n_imp > 0 ? h.errvimp : 0.0;
  }
  return HE_OK;
}


int he_energy(he_ctx_t* ctx, he_energies_t* out) {
  if (!ctx || !out) return fail(ctx, HE_ERR_ARG, "null argument");
  if (ctx->mode == HE_MODE_DYNAMICS) {
    OpEnergy<double2> op{};
    op.s8[0] = ctx->den; op.s8[1] = ctx->dencg; op.s8[2] = ctx->delj4; op.s8[3] = ctx->uimp;
    op.has_u = 1;
    op.aux1 = 0.5 * ctx->fn.cp4; op.aux2 = (1.0 / 3.0) * ctx->fn.cpp4;
    op.beta = ctx->fn.beta; op.den_m = ctx->fn.den_m; op.lsolid = ctx->fn.lsolid;
    TRY(run_stencil_red(ctx, ctx->g1, (const double2*)ctx->psi, op, S_EN));
  } else {
    OpEnergy<double> op{};
    op.s8[0] = ctx->den; op.s8[1] = ctx->dencg; op.s8[2] = ctx->delj4; op.s8[3] = ctx->den;
    op.has_u = 0;
    op.aux1 = 0.5 * ctx->fn.cp4; op.aux2 = (1.0 / 3.0) * ctx->fn.cpp4;
    op.beta = ctx->fn.beta; op.den_m = ctx->fn.den_m; op.lsolid = ctx->fn.lsolid;
    TRY(run_stencil_red(ctx, ctx->g1, (const double*)ctx->psi, op, S_EN));
  }
  CK(cudaMemcpyAsync(ctx->hsum, ctx->sums, S_COUNT * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  const double* s = ctx->hsum + S_EN;
  const double dxyz = ctx->dxyz;
  he_energies_t e{};
  e.esolid = ctx->fn.lsolid ? ctx->fn.C * s[3] * dxyz : 0.0;
  e.ekin4 = ctx->fn.h2o2m4 * s[0] * dxyz;
  e.elj4 = 0.5 * s[1] * dxyz;
  e.ecor4 = s[2] * dxyz;
  e.etot4 = e.ekin4 + e.elj4 + e.ecor4 + e.esolid;
  e.ealphas = 0.0;
  if (ctx->mode == HE_MODE_DYNAMICS) {
    ImpDev h;
    TRY(imp_pull(ctx, &h));
    const int n = ctx->n_imp;
    for (int k = 0; k < n; ++k) {
      double v2 = 0.0;
      for (int c = 0; c < 3; ++c) v2 += h.vimp[k + n * c] * h.vimp[k + n * c];
      e.ekinx = e.ekinx + 0.5 * h.m[k] * v2;
    }
    e.eHeX = s[4] * dxyz;
    for (int k = 0; k < n; ++k)
      for (int m = k + 1; m < n; ++m) {
        double r2 = 0.0;
        for (int c = 0; c < 3; ++c) {
          const double d = h.rimp[k + n * c] - h.rimp[m + n * c];
          r2 += d * d;
        }
        e.eimpu_impu += host_pair_pot(h, std::sqrt(r2));
      }
    e.eimpu = e.ekinx + e.eHeX + e.eimpu_impu;
  }
  e.etot = e.etot4 + e.eimpu;
  *out = e;
  return HE_OK;
}

int he_derden(he_ctx_t* ctx) {
  if (!ctx) return HE_ERR_ARG;
  if (!ctx->dxden) {
    TRY(dalloc_t(ctx, &ctx->dxden, ctx->N));
    TRY(dalloc_t(ctx, &ctx->dyden, ctx->N));
    TRY(dalloc_t(ctx, &ctx->dzden, ctx->N));
  }
  OpDerden op{};
  op.gx = ctx->dxden; op.gy = ctx->dyden; op.gz = ctx->dzden;
  return run_stencil(ctx, ctx->g1, ctx->den, op);
}

int he_lstopimp(he_ctx_t* ctx, int* flag) {
  if (!ctx || !flag) return fail(ctx, HE_ERR_ARG, "null argument");
  *flag = 0;
  if (ctx->mode != HE_MODE_DYNAMICS || ctx->n_imp == 0) return HE_OK;
  ImpDev h;
  TRY(imp_pull(ctx, &h));
  *flag = h.lstopimp;
  return HE_OK;
}

// ---- He_statics ----------------------------------------------------------------------------------
int he_refresh_density(he_ctx_t* ctx) {
  if (!ctx) return HE_ERR_ARG;
  if (ctx->mode != HE_MODE_STATICS) return fail(ctx, HE_ERR_STATE, "statics routine");
  if (!ctx->kernels_ok) return fail(ctx, HE_ERR_STATE, "k-space kernels not set");
  TRY(he_derden(ctx));
  TRY(spectrum_cg_lj(ctx));
  XArgs a = xargs(ctx);
  a.specA = ctx->wA; a.specB = ctx->wB;
  a.out1 = ctx->dencg; a.out2 = ctx->delj4;
  return xpass<X_C2R2>(ctx, a);
}





int he_evolo0(he_ctx_t* ctx, double* mu4, double* mu4err, int n4) {
  if (!ctx || !mu4 || !mu4err) return fail(ctx, HE_ERR_ARG, "null argument");
  if (ctx->mode != HE_MODE_STATICS) return fail(ctx, HE_ERR_STATE, "statics routine");
  TRY(stat_hpsi(ctx, ctx->hpsi, S_STAT_H));
  tname(ctx, "statics_sumsq");
  k_sumsq<<<pw_blocks(ctx), 256, 0, ctx->stream>>>((const double*)ctx->psi, ctx->N, tail(ctx, S_STAT_N));
  LAUNCHED();
  TRY(stat_normalize(ctx, n4));
  TRY(read_sums(ctx));
  const double hmean = ctx->hsum[S_STAT_H] * ctx->dxyz / (double)n4;
  *mu4err = std::fabs(1.0 - *mu4 / hmean);
  *mu4 = hmean;
  return HE_OK;
}

int he_steprkr(he_ctx_t* ctx, double deltat, double* mu4, double* mu4err, int n4) {
  if (!ctx || !mu4 || !mu4err) return fail(ctx, HE_ERR_ARG, "null argument");
  if (ctx->mode != HE_MODE_STATICS) return fail(ctx, HE_ERR_STATE, "statics routine");
  const double r2 = 1.0 / std::sqrt(2.0);
  const double arun[4] = {0.5, 1.0 - r2, 1.0 + r2, 1.0 / 6.0};
  const double brun[4] = {2.0, 1.0, 1.0, 2.0};
  const double crun[4] = {0.5, 1.0 - r2, 1.0 + r2, 0.5};
  for (int jr = 0; jr < 4; ++jr) {
    TRY(stat_hpsi(ctx, ctx->hpsi, S_STAT_H));
    if (jr == 0) {
      tname(ctx, "copy_slot");
      tname(ctx, "copy_slot");
  k_copy_slot<<<1, 32, 0, ctx->stream>>>(ctx->sums, S_HMEAN0, S_STAT_H);
      LAUNCHED();
    }
    StatPW s = statpw(ctx, deltat, n4);
    s.psi = (double*)ctx->psi;
    s.hpsi = ctx->hpsi;
    s.q = (double*)ctx->q;
    s.out = (double*)(jr == 0 ? ctx->psiold[2] : ctx->scratch);
    s.hsave = jr == 0 ? (double*)ctx->hpsiold[1] : nullptr;
    s.a = arun[jr]; s.b = brun[jr]; s.c = crun[jr];
    s.jr = jr;
    tname(ctx, "statics_rk_update");
    k_stat_rk<<<pw_blocks(ctx), 256, 0, ctx->stream>>>(s, tail(ctx, S_STAT_N));
    LAUNCHED();
    if (jr == 0) {
      void* o3 = ctx->psiold[2];
      ctx->psiold[2] = ctx->psiold[1];
      ctx->psiold[1] = ctx->psiold[0];
      ctx->psiold[0] = ctx->psi;
      ctx->psi = o3;
      std::swap(ctx->hpsiold[0], ctx->hpsiold[1]);
    } else {
      std::swap(ctx->psi, ctx->scratch);
    }
    TRY(stat_normalize(ctx, n4));
    if (jr <= 2) TRY(he_poten(ctx));
  }
  for (int i = 0; i < 3; ++i) ctx->ioldp[i] = i + 1;
  ctx->ioldh[0] = 1; ctx->ioldh[1] = 2;
  TRY(read_sums(ctx));
  const double hmean = ctx->hsum[S_HMEAN0] * ctx->dxyz / (double)n4;
  *mu4err = std::fabs(1.0 - *mu4 / hmean);
  *mu4 = hmean;
  return HE_OK;
}

int he_steppcr(he_ctx_t* ctx, double deltat, double* mu4, double* mu4err, int n4, double* errpc) {
  if (!ctx || !mu4 || !mu4err) return fail(ctx, HE_ERR_ARG, "null argument");
  if (ctx->mode != HE_MODE_STATICS) return fail(ctx, HE_ERR_STATE, "statics routine");
  TRY(stat_hpsi(ctx, ctx->hpsi, S_STAT_H));
  {
    StatPW s = statpw(ctx, deltat, n4);
    s.psi = (double*)ctx->psi;
    s.hpsi = ctx->hpsi;
    s.po3 = (double*)ctx->psiold[ctx->ioldp[2] - 1];
    s.h1 = (const double*)ctx->hpsiold[ctx->ioldh[0] - 1];
    s.h2 = (double*)ctx->hpsiold[ctx->ioldh[1] - 1];
    s.pc = (double*)ctx->pc;
    tname(ctx, "statics_predict");
    k_stat_predict<<<pw_blocks(ctx), 256, 0, ctx->stream>>>(s, tail(ctx, S_STAT_N));
    LAUNCHED();
    std::swap(ctx->psi, ctx->psiold[ctx->ioldp[2] - 1]);
    std::swap(ctx->ioldh[0], ctx->ioldh[1]);
  }
  TRY(stat_normalize(ctx, n4));
  TRY(he_poten(ctx));
  TRY(stat_hpsi(ctx, ctx->t4, S_STAT_MU));
  {
    StatPW s = statpw(ctx, deltat, n4);
    s.psi = (double*)ctx->psi;
    s.hpsi = ctx->t4;
    s.po3 = (double*)ctx->psiold[ctx->ioldp[2] - 1];
    s.po2 = (const double*)ctx->psiold[ctx->ioldp[1] - 1];
    s.h1 = (const double*)ctx->hpsiold[ctx->ioldh[0] - 1];
    s.h2 = (double*)ctx->hpsiold[ctx->ioldh[1] - 1];
    s.pc = (double*)ctx->pc;
    s.out = (double*)ctx->scratch;
    ReduceTail rt = tail(ctx, S_STAT_PC);
    tname(ctx, "statics_correct");
    k_stat_correct<<<pw_blocks(ctx), 256, 0, ctx->stream>>>(s, rt);
    LAUNCHED();
    std::swap(ctx->psi, ctx->scratch);
  }
  // k_stat_correct leaves sum psi^2 in S_STAT_PC+1; the normalisation reads S_STAT_N.
  tname(ctx, "copy_slot");
  k_copy_slot<<<1, 32, 0, ctx->stream>>>(ctx->sums, S_STAT_N, S_STAT_PC + 1);
  LAUNCHED();
  TRY(stat_normalize(ctx, n4));
  const int a = ctx->ioldp[2];
  ctx->ioldp[2] = ctx->ioldp[1];
  ctx->ioldp[1] = ctx->ioldp[0];
  ctx->ioldp[0] = a;
  TRY(read_sums(ctx));
  const double hmean = ctx->hsum[S_STAT_H] * ctx->dxyz / (double)n4;
  if (errpc) *errpc = (9.0 / 121.0) * ctx->hsum[S_STAT_PC] / (double)ctx->N;
  *mu4err = std::fabs(1.0 - *mu4 / hmean);
  *mu4 = hmean;
  return HE_OK;
}

int he_varmu(he_ctx_t* ctx, int npart, double mu, double* errmu) {
  if (!ctx || !errmu) return fail(ctx, HE_ERR_ARG, "null argument");
  if (ctx->mode != HE_MODE_STATICS) return fail(ctx, HE_ERR_STATE, "statics routine");
  tname(ctx, "statics_varmu");
  k_varmu<<<pw_blocks(ctx), 256, 0, ctx->stream>>>(ctx->hpsi, (const double*)ctx->psi, ctx->N, mu,
                                                   tail(ctx, S_VARMU));
  LAUNCHED();
  TRY(read_sums(ctx));
  *errmu = ctx->hsum[S_VARMU] * ctx->dxyz / (double)npart;
  return HE_OK;
}

int he_timing(he_ctx_t* ctx, int enable) {
  if (!ctx) return HE_ERR_ARG;
  CK(cudaStreamSynchronize(ctx->stream));
  ctx->trec.clear();
  ctx->evnext = 0;
  ctx->timing = enable != 0;
  // Create the events up front so that recording never waits on event creation.
  while (enable && ctx->evpool.size() < 8192) {
    cudaEvent_t e = nullptr;
    CK(cudaEventCreate(&e));
    ctx->evpool.push_back(e);
  }
  return HE_OK;
}

int he_timing_report(he_ctx_t* ctx, he_kernel_time_t* out, int max, int* n) {
  if (!ctx || !n) return fail(ctx, HE_ERR_ARG, "null argument");
  CK(cudaStreamSynchronize(ctx->stream));
  std::vector<he_kernel_time_t> agg;
  for (const auto& r : ctx->trec) {
    if (!r.b) continue;
    float ms = 0.0f;
    CK(cudaEventElapsedTime(&ms, r.a, r.b));
    size_t k = 0;
    for (; k < agg.size(); ++k)
      if (std::strncmp(agg[k].name, r.name, sizeof(agg[k].name)) == 0) break;
    if (k == agg.size()) {
      he_kernel_time_t t{};
      std::strncpy(t.name, r.name, sizeof(t.name) - 1);
      agg.push_back(t);
    }
    agg[k].launches += 1;
    agg[k].ms += ms;
  }
  *n = (int)agg.size();
  for (int i = 0; i < (int)agg.size() && i < max; ++i) out[i] = agg[i];
  return HE_OK;
}

int he_tuned_tiles(const he_ctx_t* ctx, int* x, int* y, int* z) {
  if (!ctx || !x || !y || !z) return HE_ERR_ARG;
  *x = ctx->tile_x;
  *y = ctx->tile_y;
  *z = ctx->tile_z;
  return HE_OK;
}

}  // extern "C"
