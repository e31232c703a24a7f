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
#include <mutex>
#include <tuple>

#include "../../include/he_dft.h"
#include "kernels.cuh"

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
  S_STAT_PREV = 42,  // he_statics_iterations: S_STAT_H of the pass before the last
  S_STAT_MU = 43,
  S_VARMU = 44,
  S_HMEAN0 = 45,
  S_STAT_PC = 46,   // k_stat_correct writes {sum |pc|, sum psi^2} to slots 46, 47
  S_ERRX = 48,      // quantum: sum |pcx_i|, kMaxQImp slots
  S_QEK = 52,       // quantum: sum |grad psix_i|^2, kMaxQImp slots
  S_QHEX = 56,      // quantum: sum sto2*den (eHeX)
  S_QII = 57,       // quantum: impurity-pair sums (eimpu_impu), 6 slots
  S_QMOM = 64,      // quantum: moments, 4 per impurity
  S_ALF = 80,       // alpha_s energy sum
  S_OBS = 96,       // observables, 16 sums
  S_COUNT = 112
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
  // Side stream for the classical-impurity work (the impurity field pass over den and the
  // one-CTA integrator kernels), which overlaps the FFT chain and the He stencils.  Work on it
  // is joined into `stream` before any kernel that reads uimp or the impurity state, writes den,
  // or reduces through the shared partials, and before every host transfer or synchronisation.
  cudaStream_t aux = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  bool aux_pending = false, on_aux = false;
  // FFT passes with programmatic dependent launch: on for grids up to 160^3, whose passes last
  // 10-30 us so that hiding the launch gap pays (128^3 step: 0.714 -> 0.655 ms FP64, 0.430 ->
  // 0.396 ms mixed); off above (256^3 FP64 step measured 4 % slower with it)
  bool pdl = false;
  std::string err;
  long long launches = 0;
  size_t bytes = 0;
  std::vector<void*> allocs;
  std::vector<size_t> alloc_bytes;  // sizes of allocs, in the same order
  // group (he_ctx_group): this context as the leader of nmem members whose buffers the member
  // map pairs with this context's; every launch covers all members
  int nmem = 1;
  MemberMap mm{};
  std::vector<unsigned long long> mmhost;  // host copy of the map table
  // FFT
  LinePlan plx{}, ply{}, plz{};
  int x_rb = 16, tkx = 16;
  int num_sms = 148;
  int tile_x = 16, tile_y = 16, tile_z = 16;  // autotuned tile variants (16 or 8 lines)
  // x pass per mode (XMode): rows per tile and persistent pipelined (true) or one-shot
  int xtile[6] = {16, 16, 16, 16, 16, 16};
  bool zreg = false;  // z convolution with register line transforms (binary32 chain only)
  bool xyfuse = false;  // classical field evaluation with fused x-y plane passes (fft_xy.cuh)
  bool yzfuse = false;  // convolutions with the y and z passes fused over a cluster (fft_yz.cuh)
  int maxsm = 0;      // opt-in shared memory per block
  bool xpipe[6] = {false, false, false, false, false, false};
  std::string tune_log;                        // the autotuner's trials (he_autotune_report)
  size_t smem_x = 0, smem_y = 0, smem_z = 0;
  // k space
  double2 *fden = nullptr, *wA = nullptr, *wB = nullptr;
  double *fvlj4 = nullptr, *wcgk = nullptr, *kalfs = nullptr;
  // mixed precision (HE_PREC_MIXED): the FFT chain of the mean field in binary32, reading
  // binary32 copies of the kernels; spectra (fden, wA, wB) then hold float2
  bool mixed = false;
  float *fvlj4f = nullptr, *wcgkf = nullptr;
  // The C2R x pass packs dencg (~den) and delj4 (~den x |fvlj4(0)|, about 1e3 larger) into one
  // complex line; in binary32 the rounding noise of delj4 would swamp dencg.  The binary32 wcgk
  // copy is therefore scaled by the power of two nearest |fvlj4(0)/wcgk(0)| (exact), and every
  // C2R of a wcgk product divides it out again (XArgs::renor1).  1 in binary64.
  double cg_scale = 1.0;
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
  // alpha_s term (core4 = 'OTC'): alphasterm module arrays and work arrays
  double *denalf = nullptr, *falfs = nullptr, *intxalf = nullptr, *intyalf = nullptr,
         *intzalf = nullptr, *ualphas = nullptr, *ua_raw = nullptr;
  double *as1 = nullptr, *as2 = nullptr, *as3 = nullptr, *as4 = nullptr, *as5 = nullptr;
  // mixed path with OTC: the binary64 copy of den the alpha_s term runs on, and the binary32 copy
  // of ualphas the binary32 pot4 epilogue adds
  double* den64 = nullptr;
  float* ualphas_f = nullptr;
  // quantum impurities (HE_MODE_QUANTUM); psixold[i][s-1] is Fortran slot s of impurity i
  int nq = 0;
  double mu4 = 0.0, h2o2mx[kMaxQImp] = {};
  void *psix[kMaxQImp] = {}, *pcx[kMaxQImp] = {}, *qx[kMaxQImp] = {}, *xscratch = nullptr;
  void *psixold[kMaxQImp][3] = {}, *hpsixold[kMaxQImp][2] = {};
  double *denx[kMaxQImp] = {}, *upotx[kMaxQImp] = {}, *uimpk[kMaxQImp] = {};
  double* uimpkk[kMaxQImp * kMaxQImp] = {};  // (i,j) at i + kMaxQImp*j; null = no kernel
  float* uimpkf[kMaxQImp] = {};                // binary32 copies (mixed path)
  float* uimpkkf[kMaxQImp * kMaxQImp] = {};
  double* potx4 = nullptr;
  double2 *wC = nullptr, *wD = nullptr, *sx[kMaxQImp] = {};
  bool cglj_pending = false;  // wA/wB hold fden*wcgk, fden*fvlj4 of the current fden (x,y domain)
  // reductions
  double* partials = nullptr;
  size_t partials_cap = 0;
  unsigned* counter = nullptr;
  double* sums = nullptr;
  double* hsum = nullptr;  // pinned host mirror of sums
  ImpDev* himp = nullptr;  // pinned host mirror of the impurity struct
  // optional per-kernel CUDA-event timing (he_timing / he_timing_report)
  struct TRec {
    const char* name;
    cudaEvent_t a, b;
  };
  bool timing = false;
  std::vector<TRec> trec;
  std::vector<cudaEvent_t> evpool;
  size_t evnext = 0;
  // he_statics_iterations: one CUDA graph per statics pass, keyed by the state fingerprint before
  // it (with deltat and n4); each keeps the buffer relabelling that its pass leaves behind
  struct StatGraph {
    unsigned long long key;
    cudaGraphExec_t exec;
    void *psi, *scratch, *psiold[3], *hpsiold[2];
    int ioldp[3], ioldh[2];
    long long launches;
  };
  std::vector<StatGraph> stat_graphs;
  bool stat_warm = false;  // one pass ran eagerly (lazy allocations, shared-memory attributes)
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

// Drops the statics pass graphs (their arguments bake in the kernels, scales and FFT variants).
static void stat_graphs_clear(he_ctx_t* ctx) {
  for (auto& g : ctx->stat_graphs) cudaGraphExecDestroy(g.exec);
  ctx->stat_graphs.clear();
}

// Raises a kernel's dynamic shared-memory limit, once per kernel and device (the attribute
// persists; asking the driver on every launch costs host time in the gaps after each
// synchronising call).
static cudaError_t set_smem_attr(const void* fn, size_t smem) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  static std::mutex mu;
  static std::vector<std::tuple<const void*, int, size_t>> done;
  std::lock_guard<std::mutex> lock(mu);
  for (const auto& d : done)
    if (std::get<0>(d) == fn && std::get<1>(d) == dev && std::get<2>(d) >= smem) return cudaSuccess;
  e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess) done.emplace_back(fn, dev, smem);
  return e;
}

// Launch of an FFT pass (a kernel that starts with pdl_wait_and_trigger) on the context's current
// stream with programmatic stream serialisation.
template <typename... KArgs, typename... Args>
static cudaError_t launch_chain(he_ctx_t* ctx, void (*k)(KArgs...), dim3 grid, dim3 block,
                                size_t smem, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = ctx->stream;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = ctx->pdl ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, k, args...);
}

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
  ctx->alloc_bytes.push_back(bytes);
  ctx->bytes += bytes;
  CK(cudaMemsetAsync(*p, 0, bytes, ctx->stream));
  return HE_OK;
}
template <typename T>
static int dalloc_t(he_ctx_t* ctx, T** p, size_t count) {
  return dalloc(ctx, reinterpret_cast<void**>(p), count * sizeof(T));
}

// ---- side stream (see he_ctx::aux) ----------------------------------------------------------
static bool overlap_on(const he_ctx_t* ctx) {
  return ctx->aux && ctx->mode == HE_MODE_DYNAMICS && ctx->n_imp > 0 && !ctx->timing;
}
static int join_aux(he_ctx_t* ctx) {
  if (!ctx->aux_pending || ctx->on_aux) return HE_OK;
  CK(cudaEventRecord(ctx->ev_join, ctx->aux));
  CK(cudaStreamWaitEvent(ctx->stream, ctx->ev_join, 0));
  ctx->aux_pending = false;
  return HE_OK;
}
// Orders the side stream after everything issued so far on the main stream.
static int fork_aux(he_ctx_t* ctx) {
  CK(cudaEventRecord(ctx->ev_fork, ctx->stream));
  CK(cudaStreamWaitEvent(ctx->aux, ctx->ev_fork, 0));
  return HE_OK;
}
// Stream for an impurity-state kernel (the side stream when overlapping).  A side stream that
// has been joined is forked from the main stream first, so that its work always hangs off the
// main stream's order (and a step recorded into a CUDA graph records it).
static cudaStream_t imp_stream(he_ctx_t* ctx) {
  if (!overlap_on(ctx)) return ctx->stream;
  if (!ctx->aux_pending && !ctx->on_aux &&
      (cudaEventRecord(ctx->ev_fork, ctx->stream) != cudaSuccess ||
       cudaStreamWaitEvent(ctx->aux, ctx->ev_fork, 0) != cudaSuccess))
    return ctx->stream;  // fall back to the main stream (ordered, no overlap)
  ctx->aux_pending = true;
  return ctx->aux;
}
// Redirects the context's launches to the side stream for its lifetime.
struct OnAux {
  he_ctx_t* c;
  cudaStream_t saved;
  explicit OnAux(he_ctx_t* ctx) : c(ctx), saved(ctx->stream) {
    c->stream = c->aux;
    c->on_aux = true;
  }
  ~OnAux() {
    c->stream = saved;
    c->on_aux = false;
    c->aux_pending = true;
  }
};
static int sync_all(he_ctx_t* ctx) {
  TRY(join_aux(ctx));
  CK(cudaStreamSynchronize(ctx->stream));
  return HE_OK;
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
  {
    std::vector<float2> sf(stw.size());
    for (size_t i = 0; i < stw.size(); ++i) sf[i] = make_float2((float)stw[i].x, (float)stw[i].y);
    float2* df = nullptr;
    TRY(dalloc_t(ctx, &df, sf.size()));
    CK(cudaMemcpyAsync(df, sf.data(), sf.size() * sizeof(float2), cudaMemcpyHostToDevice, ctx->stream));
    TRY(sync_all(ctx));
    pl->stwf = df;
  }
  TRY(sync_all(ctx));
  pl->tw = d;
  pl->stw = d;
  pl->stw_len = (int)stw.size();
  pl->tw2 = nullptr;
  const int n1 = split_n1(n);
  if (n1 > 0) {  // register y pass: W_n^(a k1) at [k1 n2 + a]
    const int n2 = n / n1;
    std::vector<double2> t2((size_t)n);
    for (int k1 = 0; k1 < n1; ++k1)
      for (int a = 0; a < n2; ++a) {
        long double ang = -2.0L * 3.14159265358979323846264338327950288L * ((long)a * k1) / (long double)n;
        t2[(size_t)k1 * n2 + a] = make_double2((double)cosl(ang), (double)sinl(ang));
      }
    double2* d2 = nullptr;
    TRY(dalloc_t(ctx, &d2, t2.size()));
    CK(cudaMemcpyAsync(d2, t2.data(), t2.size() * sizeof(double2), cudaMemcpyHostToDevice, ctx->stream));
    pl->tw2 = d2;
    std::vector<float2> t2f(t2.size());
    for (size_t i = 0; i < t2.size(); ++i) t2f[i] = make_float2((float)t2[i].x, (float)t2[i].y);
    float2* d2f = nullptr;
    TRY(dalloc_t(ctx, &d2f, t2f.size()));
    CK(cudaMemcpyAsync(d2f, t2f.data(), t2f.size() * sizeof(float2), cudaMemcpyHostToDevice, ctx->stream));
    TRY(sync_all(ctx));
    pl->tw2f = d2f;
  }
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
    for (int m = 0; m < 13; ++m) {
      g->w[a][m] = ((id == 1) ? ctx->w1[m] : ctx->w2[m]) * sto;
      g->wf[a][m] = (float)g->w[a][m];
    }
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
  static int occ = -1;  // resident CTAs per SM of this instantiation (one context)
  if (occ < 0) {
    CK(set_smem_attr((const void*)k_stencil<Op, kTX, kTY, false>, smem));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_stencil<Op, kTX, kTY, false>, kTX * kTY, smem));
  }
  TRY(join_aux(ctx));  // stencils read uimp / write den / reduce through the shared partials
  // a group runs the instantiation that maps the op's pointers to each member's buffers; the z
  // chunking (and so every reduction's order) stays that of one context
  void (*k)(const typename Op::T*, StencilGeom, Op, ReduceTail) = k_stencil<Op, kTX, kTY, false>;
  if (ctx->nmem > 1) {
    if constexpr (HasRemap<Op>::value) k = k_stencil<Op, kTX, kTY, true>;
    else return fail(ctx, HE_ERR_STATE, "%s does not run over the members of a group", Op::kname());
  }
  StencilGeom g = g0;
  g.zc = choose_zc(ctx, occ);
  dim3 grid = stencil_grid(ctx, g), block(kTX, kTY);
  ReduceTail rt{};
  if (Op::NV > 0) {
    TRY(ensure_partials(ctx, (size_t)grid.x * grid.y * grid.z * Op::NV));
    rt = tail(ctx, slot);
  }
  g.nzc = (int)grid.z;  // z-chunks per member
  g.mm = ctx->mm;
  // a group's CTAs each stream through lcz consecutive chunks (at least 16 planes), so that the
  // 12-plane start of a chunk is paid once per CTA; the partials are still one per chunk
  g.lcz = ctx->nmem > 1 ? std::max(1, std::min(g.nzc, 16 / std::max(1, g.zc))) : 1;
  grid.z = (unsigned)(((g.nzc + g.lcz - 1) / g.lcz) * ctx->nmem);
  CK(set_smem_attr((const void*)k, smem));
  tname(ctx, Op::kname());
  k<<<grid, block, smem, ctx->stream>>>(f, g, op, rt);
  LAUNCHED();
  return HE_OK;
}
template <class Op>
static int run_stencil_red(he_ctx_t* ctx, const StencilGeom& g, const typename Op::T* f,
                           const Op& op, int slot) {
  return run_stencil(ctx, g, f, op, slot);
}

// Planes of a compensated pair buffer of the mixed path (psi, psiold, scratch): hi, then lo.
static float2* hi_plane(void* b) { return (float2*)b; }
static float2* lo_plane(const he_ctx_t* ctx, void* b) { return (float2*)b + ctx->N; }

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
  a.renor1 = ctx->renor / ctx->cg_scale;
  a.cp4 = ctx->fn.cp4; a.cpp4 = ctx->fn.cpp4;
  a.a0 = ctx->fn.cp4 / 2.0; a.a1 = ctx->fn.cpp4 / 3.0;
  a.lsolid = ctx->fn.lsolid;
  a.C = ctx->fn.C; a.beta = ctx->fn.beta; a.den_m = ctx->fn.den_m;
  a.mm = ctx->mm;
  return a;
}
// Line lengths with a compile-time FFT instantiation; other admissible lengths run the same
// kernels with run-time sizes (N = 0).
#define HE_FFT_SIZES(X) X(32) X(64) X(96) X(128) X(160) X(192) X(256)

static size_t fft_smem(const LinePlan& pl, int lines, int nbuf, size_t elem = sizeof(double2)) {
  return elem * (((size_t)pl.stw_len + 1) / 2 * 2 + (size_t)nbuf * lines * line_stride(pl.n));
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
// Rt: the chain's arithmetic (double, or float in the mixed-precision mode).
template <int MODE, int N, int TILE, typename Rt>
static int xpass_n(he_ctx_t* ctx, const XArgs& a) {
  const int rb = (N > 0) ? TILE : a.rb;
  // compile-time lengths: rb divides ny*nz (x_fast); run-time lengths: the last tile may be
  // partial (an odd row count), its missing rows read as zero and are not stored
  const long ntiles = (a.rows + rb - 1) / rb;
  const int nthr = (N > 0) ? tile_threads(TILE) : 256;
  static const char* names[6] = {"fft_x_r2c_den", "fft_x_r2c_corr", "fft_x_c2r_cg_lj",
                                 "fft_x_c2r_cg_lj_r2c_corr", "fft_x_c2r_pot4", "fft_x_c2r"};
  if (!ctx->xpipe[MODE] || N == 0) {
    const size_t csmem = fft_smem(ctx->plx, rb, 2, sizeof(typename Cx<Rt>::T));
    void (*kc)(XArgs) = ctx->nmem > 1 ? k_xpass_c<MODE, N, TILE, Rt, true> : k_xpass_c<MODE, N, TILE, Rt, false>;
    CK(set_smem_attr((const void*)kc, csmem));
    tname(ctx, names[MODE]);
    CK(launch_chain(ctx, kc, dim3((unsigned)ntiles, ctx->nmem), dim3(nthr), csmem, a));
    LAUNCHED();
    return HE_OK;
  }
  constexpr int pthr = kXPipeThreads;
  const size_t smem = xpass_smem<MODE, Rt>(ctx->plx.stw_len, rb, ctx->nx);
  // persistent grid: as many CTAs as fit on the device at once (the smem of the run-time-length
  // kernel depends on the grid, so its occupancy is queried per launch size)
  // (the tiles of a CTA, and so the grid, are those of one context in a group too)
  static size_t occ_smem = 0;
  static int occ = 0;
  if (occ_smem != smem) {
    CK(set_smem_attr((const void*)k_xpass<MODE, N, TILE, Rt, false>, smem));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_xpass<MODE, N, TILE, Rt, false>, pthr, smem));
    occ_smem = smem;
  }
  if (occ < 1) return fail(ctx, HE_ERR_STATE, "x pass: %zu bytes of shared memory do not fit an SM", smem);
  const unsigned nb = (unsigned)std::min<long>(ntiles, (long)occ * ctx->num_sms);
  void (*kp)(XArgs) = ctx->nmem > 1 ? k_xpass<MODE, N, TILE, Rt, true> : k_xpass<MODE, N, TILE, Rt, false>;
  CK(set_smem_attr((const void*)kp, smem));
  tname(ctx, names[MODE]);
  CK(launch_chain(ctx, kp, dim3(nb, ctx->nmem), dim3(pthr), smem, a));
  LAUNCHED();
  return HE_OK;
}
template <int MODE, typename Rt>
static int xpass_t(he_ctx_t* ctx, const XArgs& a) {
  const int tile = ctx->xtile[MODE];
  if (x_fast(ctx, tile)) {
    switch (ctx->nx) {
#define HE_CASE(N) \
  case N: return tile == 8 ? xpass_n<MODE, N, 8, Rt>(ctx, a) : xpass_n<MODE, N, 16, Rt>(ctx, a);
      HE_FFT_SIZES(HE_CASE)
#undef HE_CASE
    }
  }
  return xpass_n<MODE, 0, 16, Rt>(ctx, a);
}
template <int MODE>
static int xpass(he_ctx_t* ctx, const XArgs& a) {
  return ctx->mixed ? xpass_t<MODE, float>(ctx, a) : xpass_t<MODE, double>(ctx, a);
}

template <int N, int TILE, typename Rt>
static int ypass_n(he_ctx_t* ctx, const YZArgs& a, int narr) {
  using C = typename Cx<Rt>::T;
  const int tk = (N > 0) ? TILE : ctx->tkx;
  const size_t smem = fft_smem(ctx->ply, tk, 2, sizeof(C));
  const int nthr = (N > 0) ? tile_threads(TILE) : 256;
  dim3 grid((ctx->nxh + tk - 1) / tk, ctx->nz, narr * ctx->nmem);  // z: member x narr + array
  tname(ctx, "fft_y");
  if constexpr (N > 0) {
    // register line transform (fft_reg.cuh): TK columns x N2 threads, T[k1][a][c] in shared memory
    const size_t rsmem = sizeof(C) * (size_t)N * tk;
    const C* tw2;
    if constexpr (sizeof(Rt) == 4) tw2 = ctx->ply.tw2f;
    else tw2 = ctx->ply.tw2;
    void (*k)(YZArgs, const C*) = ctx->nmem > 1 ? k_ypass_reg<N, TILE, Rt, true> : k_ypass_reg<N, TILE, Rt, false>;
    CK(set_smem_attr((const void*)k, rsmem));
    CK(launch_chain(ctx, k, grid, dim3(yreg_threads(N, TILE)), rsmem, a, tw2));
  } else {
    void (*k)(YZArgs) = ctx->nmem > 1 ? k_ypass<N, TILE, Rt, true> : k_ypass<N, TILE, Rt, false>;
    CK(set_smem_attr((const void*)k, smem));
    CK(launch_chain(ctx, k, grid, dim3(nthr), smem, a));
  }
  LAUNCHED();
  return HE_OK;
}
template <typename Rt>
static int ypass_t(he_ctx_t* ctx, const YZArgs& a, int narr) {
  const int tile = ctx->tile_y;
  if (yz_fast(ctx->ny)) {
    switch (ctx->ny) {
#define HE_CASE(N) \
  case N: return tile == 8 ? ypass_n<N, 8, Rt>(ctx, a, narr) : ypass_n<N, 16, Rt>(ctx, a, narr);
      HE_FFT_SIZES(HE_CASE)
#undef HE_CASE
    }
  }
  return ypass_n<0, 16, Rt>(ctx, a, narr);
}
static int ypass(he_ctx_t* ctx, double2* a0, double2* a1, bool inv) {
  YZArgs a{};
  a.nxh = ctx->nxh; a.ny = ctx->ny; a.nz = ctx->nz; a.tkx = ctx->tkx;
  a.pl = ctx->ply;
  a.arr[0] = a0; a.arr[1] = a1 ? a1 : a0;
  a.inv = inv;
  const int narr = a1 ? 2 : 1;
  a.narr = narr;
  a.mm = ctx->mm;
  return ctx->mixed ? ypass_t<float>(ctx, a, narr) : ypass_t<double>(ctx, a, narr);
}

template <int N, int TILE, typename Rt>
static int zconv_n(he_ctx_t* ctx, const YZArgs& a) {
  const int tk = (N > 0) ? TILE : ctx->tkx;
  if constexpr (N > 0) {
    if (ctx->zreg) {  // register line transforms (fft_reg.cuh)
      using C = typename Cx<Rt>::T;
      const bool two = (sizeof(Rt) == 4) ? a.k2f != nullptr : a.k2 != nullptr;
      const size_t rsmem = sizeof(C) * (size_t)N * TILE * (two ? 2 : 1);
      const C* tw2;
      if constexpr (sizeof(Rt) == 4) tw2 = ctx->plz.tw2f;
      else tw2 = ctx->plz.tw2;
      void (*k)(YZArgs, const C*) = ctx->nmem > 1 ? k_zconv_reg<N, TILE, Rt, true> : k_zconv_reg<N, TILE, Rt, false>;
      CK(set_smem_attr((const void*)k, rsmem));
      dim3 grid((ctx->nxh + TILE - 1) / TILE, ctx->ny, ctx->nmem);
      tname(ctx, a.k2 ? "fft_z_conv2" : "fft_z_conv1");
      CK(launch_chain(ctx, k, grid, dim3(yreg_threads(N, TILE)), rsmem, a, tw2));
      LAUNCHED();
      return HE_OK;
    }
  }
  // one-kernel convolutions: two line buffers and no second kernel's registers
  const bool two = (sizeof(Rt) == 4) ? a.k2f != nullptr : a.k2 != nullptr;
  const size_t smem = fft_smem(ctx->plz, tk, two ? 3 : 2, sizeof(typename Cx<Rt>::T));
  const int nthr = (N > 0) ? tile_threads(TILE) : 256;
  dim3 grid((ctx->nxh + tk - 1) / tk, ctx->ny, ctx->nmem);
  void (*k)(YZArgs) = two ? (ctx->nmem > 1 ? k_zconv<N, TILE, Rt, true, true> : k_zconv<N, TILE, Rt, false, true>)
                          : (ctx->nmem > 1 ? k_zconv<N, TILE, Rt, true, false> : k_zconv<N, TILE, Rt, false, false>);
  CK(set_smem_attr((const void*)k, smem));
  tname(ctx, a.k2 ? "fft_z_conv2" : "fft_z_conv1");
  CK(launch_chain(ctx, k, grid, dim3(nthr), smem, a));
  LAUNCHED();
  return HE_OK;
}
template <typename Rt>
static int zconv_t(he_ctx_t* ctx, const YZArgs& a) {
  const int tile = ctx->tile_z;
  if (yz_fast(ctx->nz)) {
    switch (ctx->nz) {
#define HE_CASE(N) \
  case N: return tile == 8 ? zconv_n<N, 8, Rt>(ctx, a) : zconv_n<N, 16, Rt>(ctx, a);
      HE_FFT_SIZES(HE_CASE)
#undef HE_CASE
    }
  }
  return zconv_n<0, 16, Rt>(ctx, a);
}
// binary32 copy of a binary64 k-space kernel (the mixed chain reads these)
static const float* kernel_f32(const he_ctx_t* ctx, const double* k) {
  if (!k) return nullptr;
  if (k == ctx->wcgk) return ctx->wcgkf;
  if (k == ctx->fvlj4) return ctx->fvlj4f;
  for (int i = 0; i < kMaxQImp; ++i)
    if (k == ctx->uimpk[i]) return ctx->uimpkf[i];
  for (int i = 0; i < kMaxQImp * kMaxQImp; ++i)
    if (k == ctx->uimpkk[i]) return ctx->uimpkkf[i];
  return nullptr;
}
static int zconv(he_ctx_t* ctx, double2* io, const double* k1, double2* out2, const double* k2,
                 double2* fden_out) {
  YZArgs a{};
  a.nxh = ctx->nxh; a.ny = ctx->ny; a.nz = ctx->nz; a.tkx = ctx->tkx;
  a.pl = ctx->plz;
  a.io = io; a.out2 = out2; a.fden_out = fden_out; a.k1 = k1; a.k2 = k2;
  a.mm = ctx->mm;
  if (!ctx->mixed) return zconv_t<double>(ctx, a);
  a.k1f = kernel_f32(ctx, k1);
  a.k2f = kernel_f32(ctx, k2);
  if (!a.k1f || (k2 && !a.k2f)) return fail(ctx, HE_ERR_STATE, "no binary32 copy of a k-space kernel");
  return zconv_t<float>(ctx, a);
}

// ---- fused y-z convolutions (fft_yz.cuh): 64^3-sized y-z planes ----
static bool yz_fusable(const he_ctx_t* ctx) { return ctx->ny == 64 && ctx->nz == 64; }
template <int N, int CS, bool TWO, typename Rt>
static int yzconv_n(he_ctx_t* ctx, const YZConvArgs& a) {
  constexpr size_t smem = yz_smem<N, CS, Rt>();
  void (*k)(YZConvArgs) = ctx->nmem > 1 ? k_yzconv<N, CS, TWO, Rt, true> : k_yzconv<N, CS, TWO, Rt, false>;
  CK(set_smem_attr((const void*)k, smem));
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(((ctx->nxh + 1) / 2) * CS), ctx->nmem);
  cfg.blockDim = dim3(kYZThreads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = ctx->stream;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = CS;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  tname(ctx, TWO ? "fft_yz_conv2" : "fft_yz_conv1");
  CK(cudaLaunchKernelEx(&cfg, k, a));
  LAUNCHED();
  return HE_OK;
}
// io <- y^-1 z^-1 (K1 . z y io) [and out2 <- y^-1 z^-1 (K2 . z y io), fden_out <- z y io]
static int yzconv(he_ctx_t* ctx, double2* io, const double* k1, double2* out2, const double* k2,
                  double2* fden_out) {
  if (!yz_fusable(ctx)) return fail(ctx, HE_ERR_STATE, "no fused y-z convolution for this grid");
  YZConvArgs a{};
  a.nxh = ctx->nxh;
  a.io = io; a.out2 = out2; a.fden_out = fden_out; a.k1 = k1; a.k2 = k2;
  a.tw2 = ctx->ply.tw2; a.tw2f = ctx->ply.tw2f;
  a.mm = ctx->mm;
  const bool two = k2 != nullptr;
  if (two && (!out2 || !fden_out)) return fail(ctx, HE_ERR_STATE, "two-kernel convolution needs out2 and fden");
  if (ctx->mixed) {
    a.k1f = kernel_f32(ctx, k1);
    a.k2f = kernel_f32(ctx, k2);
    if (!a.k1f || (two && !a.k2f)) return fail(ctx, HE_ERR_STATE, "no binary32 copy of a k-space kernel");
    return two ? yzconv_n<64, 4, true, float>(ctx, a) : yzconv_n<64, 4, false, float>(ctx, a);
  }
  return two ? yzconv_n<64, 4, true, double>(ctx, a) : yzconv_n<64, 4, false, double>(ctx, a);
}

// fden = R2C(den); wA <- fden*wcgk and wB <- fden*fvlj4 back in (x-transformed) row space.
static int spectrum_cg_lj(he_ctx_t* ctx) {
  XArgs a = xargs(ctx);
  a.den = ctx->den;
  a.specA = ctx->wA;
  TRY(xpass<X_R2C_DEN>(ctx, a));
  if (ctx->yzfuse) return yzconv(ctx, ctx->wA, ctx->wcgk, ctx->wB, ctx->fvlj4, ctx->fden);
  TRY(ypass(ctx, ctx->wA, nullptr, false));
  TRY(zconv(ctx, ctx->wA, ctx->wcgk, ctx->wB, ctx->fvlj4, ctx->fden));
  TRY(ypass(ctx, ctx->wA, ctx->wB, true));
  return HE_OK;
}
// Correlation convolution of the spectrum in wA (already x-transformed) and pot4 assembly
// (extra: potx4 of the quantum impurities, or null).
static int correlation_tail(he_ctx_t* ctx, const double* extra = nullptr,
                            const double* extra2 = nullptr) {
  if (ctx->yzfuse) {
    TRY(yzconv(ctx, ctx->wA, ctx->wcgk, nullptr, nullptr, nullptr));
  } else {
    TRY(ypass(ctx, ctx->wA, nullptr, false));
    TRY(zconv(ctx, ctx->wA, ctx->wcgk, nullptr, nullptr, nullptr));
    TRY(ypass(ctx, ctx->wA, nullptr, true));
  }
  XArgs a = xargs(ctx);
  a.specA = ctx->wA;
  a.den = ctx->den; a.dencg_in = ctx->dencg; a.delj4_in = ctx->delj4;
  a.out1 = ctx->pot4;
  a.extra = extra;
  a.extra2 = extra2;
  return xpass<X_C2R_POT>(ctx, a);
}

// ---- fused x-y plane passes (fft_xy.cuh): binary32 chain, nx = ny in {64, 96, 128} ---------------
static bool xy_fusable(const he_ctx_t* ctx) {
  return ctx->mixed && ctx->nx == ctx->ny && (ctx->nx == 64 || ctx->nx == 96 || ctx->nx == 128) &&
         split_n1(ctx->nx) > 0 && ((long)ctx->nxh * ctx->ny) % 2 == 0;
}
static XYArgs xyargs(he_ctx_t* ctx) {
  XYArgs a{};
  a.twx = ctx->plx.tw2f; a.twy = ctx->ply.tw2f;
  a.renor = ctx->renor; a.renor1 = ctx->renor / ctx->cg_scale;
  a.cp4 = ctx->fn.cp4; a.cpp4 = ctx->fn.cpp4;
  a.a0 = ctx->fn.cp4 / 2.0; a.a1 = ctx->fn.cpp4 / 3.0;
  a.lsolid = ctx->fn.lsolid;
  a.C = ctx->fn.C; a.beta = ctx->fn.beta; a.den_m = ctx->fn.den_m;
  return a;
}
template <int N>
static int xy_launch(he_ctx_t* ctx, int kind, const XYArgs& a) {
  static const char* names[3] = {"fft_xy_r2c_den", "fft_xy_c2r_cg_lj_r2c_corr", "fft_xy_c2r_pot4"};
  void (*k)(XYArgs) = kind == 0 ? k_xy_r2c<N> : kind == 1 ? k_xy_c2r2_corr<N> : k_xy_c2r_pot<N>;
  const size_t smem = kind == 1 ? xy_smem_corr<N>() : xy_smem_r2c<N>();
  CK(set_smem_attr((const void*)k, smem));
  tname(ctx, names[kind]);
  CK(launch_chain(ctx, k, dim3(ctx->nz), dim3(kXYThreads), smem, a));
  LAUNCHED();
  return HE_OK;
}
static int xy_pass(he_ctx_t* ctx, int kind, const XYArgs& a) {
  switch (ctx->nx) {
    case 64: return xy_launch<64>(ctx, kind, a);
    case 96: return xy_launch<96>(ctx, kind, a);
    case 128: return xy_launch<128>(ctx, kind, a);
    default: return fail(ctx, HE_ERR_STATE, "fused x-y passes need nx = ny in {64, 96, 128}");
  }
}
// Dynamics_TDDFT/poten.f90:131-218 with fused plane passes: 5 launches instead of 9.
static int poten_fused(he_ctx_t* ctx, const double* extra, const double* extra2) {
  if (ctx->nmem > 1) return fail(ctx, HE_ERR_STATE, "the fused x-y field evaluation runs no groups");
  XYArgs a = xyargs(ctx);
  a.den = (const float*)ctx->den;
  a.specA = (float2*)ctx->wA;
  TRY(xy_pass(ctx, 0, a));
  TRY(zconv(ctx, ctx->wA, ctx->wcgk, ctx->wB, ctx->fvlj4, ctx->fden));
  a.specB = (const float2*)ctx->wB;
  a.out1 = (float*)ctx->dencg; a.out2 = (float*)ctx->delj4;
  TRY(xy_pass(ctx, 1, a));
  TRY(zconv(ctx, ctx->wA, ctx->wcgk, nullptr, nullptr, nullptr));
  XYArgs b = xyargs(ctx);
  b.specA = (float2*)ctx->wA;
  b.den = (const float*)ctx->den; b.dencg_in = (const float*)ctx->dencg;
  b.delj4_in = (const float*)ctx->delj4;
  b.extra = (const float*)extra; b.extra2 = (const float*)extra2;
  b.out1 = (float*)ctx->pot4;
  return xy_pass(ctx, 2, b);
}

// ---- module-array access -----------------------------------------------------------------------
static size_t wf_elem(const he_ctx_t* ctx) {
  return ctx->mode == HE_MODE_STATICS ? sizeof(double) : sizeof(double2);
}

static int imp_pull(he_ctx_t* ctx, ImpDev* h) {
  TRY(join_aux(ctx));
  // through the pinned mirror: an asynchronous copy that the one synchronisation covers
  ImpDev* m = ctx->himp ? ctx->himp : h;
  CK(cudaMemcpyAsync(m, ctx->imp, sizeof(ImpDev), cudaMemcpyDeviceToHost, ctx->stream));
  TRY(sync_all(ctx));
  if (m != h) std::memcpy(h, m, sizeof(ImpDev));
  return HE_OK;
}
static int imp_push(he_ctx_t* ctx, const ImpDev* h) {
  TRY(join_aux(ctx));
  CK(cudaMemcpyAsync(ctx->imp, h, sizeof(ImpDev), cudaMemcpyHostToDevice, ctx->stream));
  TRY(sync_all(ctx));
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
    case HE_F_DENALF: case HE_F_FALFS: case HE_F_INTXALF: case HE_F_INTYALF: case HE_F_INTZALF:
    case HE_F_UALPHAS: {
      if (!ctx->otc) break;
      double* const arr[6] = {ctx->denalf, ctx->falfs, ctx->intxalf, ctx->intyalf, ctx->intzalf,
                              ctx->ualphas};
      *r = {arr[field - HE_F_DENALF], 8 * N, false};
      return HE_OK;
    }
    case HE_F_KALFS:
      if (!ctx->otc) break;
      *r = {ctx->kalfs, 8 * Nk, true};
      return HE_OK;
    case HE_F_FVLJ4: *r = {ctx->fvlj4, 8 * Nk, true}; return HE_OK;
    case HE_F_WCGK: *r = {ctx->wcgk, 8 * Nk, true}; return HE_OK;
    default: break;
  }
  return fail(ctx, HE_ERR_ARG, "field %d is not available in this context", field);
}

// Device format of a module array.  binary64 everywhere except in the mixed path, where psi and
// psiold are compensated binary32 pairs (hi plane, then lo plane), pc, q, hpsiold and fden are
// float2, and den, pot4, dencg, delj4, uimp are float.  he_upload / he_download convert; the
// host side is always binary64.
enum FieldFmt { FMT_F64 = 0, FMT_R32 = 1, FMT_C32 = 2, FMT_HL = 3 };
static FieldFmt field_fmt(const he_ctx_t* ctx, int field) {
  if (!ctx->mixed) return FMT_F64;
  if (ctx->mode == HE_MODE_STATICS && field == HE_F_PC) return FMT_HL;  // holds sto1 (full size)
  if (field == HE_F_HPSI) return FMT_R32;
  switch (field) {
    case HE_F_PSI: case HE_F_PSIOLD1: case HE_F_PSIOLD2: case HE_F_PSIOLD3: return FMT_HL;
    case HE_F_PC: case HE_F_Q: case HE_F_HPSIOLD1: case HE_F_HPSIOLD2: case HE_F_FDEN: return FMT_C32;
    case HE_F_DEN: case HE_F_POT4: case HE_F_DENCG: case HE_F_DELJ4: case HE_F_UIMP: return FMT_R32;
    default: return FMT_F64;
  }
}
// binary64 host array of `bytes` bytes -> the device format's bytes in dev
static void to_device_fmt(FieldFmt f, const void* host, size_t bytes, std::vector<unsigned char>& dev) {
  const double* h = (const double*)host;
  const size_t nv = bytes / 8;
  if (f == FMT_R32 || f == FMT_C32) {
    dev.resize(nv * 4);
    float* d = (float*)dev.data();
    for (size_t i = 0; i < nv; ++i) d[i] = (float)h[i];
  } else {  // FMT_HL: (re, im) per point -> hi plane (re, im), lo plane (re, im)
    dev.resize(bytes);
    const size_t np = nv / 2;
    float* hi = (float*)dev.data();
    float* lo = hi + 2 * np;
    for (size_t i = 0; i < nv; ++i) {
      const HL v = hl_from(h[i]);
      hi[i] = v.hi;
      lo[i] = v.lo;
    }
  }
}
static void from_device_fmt(FieldFmt f, const std::vector<unsigned char>& dev, void* host, size_t bytes) {
  double* h = (double*)host;
  const size_t nv = bytes / 8;
  if (f == FMT_R32 || f == FMT_C32) {
    const float* d = (const float*)dev.data();
    for (size_t i = 0; i < nv; ++i) h[i] = (double)d[i];
  } else {
    const size_t np = nv / 2;
    const float* hi = (const float*)dev.data();
    const float* lo = hi + 2 * np;
    for (size_t i = 0; i < nv; ++i) h[i] = hl_value(HL{hi[i], lo[i]});
  }
}
static size_t device_fmt_bytes(FieldFmt f, size_t host_bytes) {
  return (f == FMT_R32 || f == FMT_C32) ? host_bytes / 2 : host_bytes;
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
  // reduction blocks: nlb logical blocks (one partial each, the element split of a grid of nlb
  // CTAs), lpb of them per CTA; groups give a CTA several so that it carries more work, with the
  // same partials, hence the same sums, as a context run alone (0: one per CTA, nlb = gridDim.x)
  int nlb, lpb;
  MemberMap mm;       // group members (blockIdx.y is the member)
  HE_D void remap(int m) {
    sums = mm(sums, m); psi = mm(psi, m); out = mm(out, m); po3 = mm(po3, m); po2 = mm(po2, m);
    h1 = mm(h1, m); h2 = mm(h2, m); pc = mm(pc, m); q = mm(q, m); hsave = mm(hsave, m);
    hpsi = mm(hpsi, m); timec = mm(timec, m); den = mm(den, m);
  }
};

__device__ __forceinline__ double local_dt(double hp, double ps, const StatPW& s) {
  return s.dt / (1.0 + exp((fabs(hp / ps) - s.dmumax) / s.sdmu)) + s.dtmin;
}

// steppcr predictor + modifier (steppcr.f90:40-61); acc = sum psi_new^2.
__global__ void __launch_bounds__(256) k_stat_predict(const StatPW s_in, const ReduceTail rt_in) {
  StatPW s = s_in;
  s.remap(blockIdx.y);
  const ReduceTail rt = remap(rt_in, s.mm, blockIdx.y);
  const double c112 = 112.0 / 121.0, c4o3 = 4.0 / 3.0;
  const double hmean = s.sums[S_STAT_H] * s.dxyz / s.n4;
  const int nlb = s.lpb > 0 ? s.nlb : (int)gridDim.x, lpb = s.lpb > 0 ? s.lpb : 1;
  for (int j = 0; j < lpb; ++j) {
  const int lb = blockIdx.x * lpb + j;
  double acc[1] = {0.0};
  for (long i = lb * (long)blockDim.x + threadIdx.x; i < s.N; i += (long)nlb * blockDim.x) {
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
  if (j > 0) __syncthreads();  // the block reduction's shared buffer is reused
  block_reduce_store<1>(acc, rt.partials + lb);
  }
  reduce_tail<1>(rt, nlb, gridDim.x);
}

// steppcr corrector + final value (steppcr.f90:78-90); acc = {sum |pc|, sum psi_new^2}.
__global__ void __launch_bounds__(256) k_stat_correct(const StatPW s_in, const ReduceTail rt_in) {
  StatPW s = s_in;
  s.remap(blockIdx.y);
  const ReduceTail rt = remap(rt_in, s.mm, blockIdx.y);
  const double c9 = 9.0 / 121.0;
  const double mu = s.sums[S_STAT_MU] * s.dxyz / s.n4;
  const int nlb = s.lpb > 0 ? s.nlb : (int)gridDim.x, lpb = s.lpb > 0 ? s.lpb : 1;
  for (int j = 0; j < lpb; ++j) {
  const int lb = blockIdx.x * lpb + j;
  double acc[2] = {0.0, 0.0};
  for (long i = lb * (long)blockDim.x + threadIdx.x; i < s.N; i += (long)nlb * blockDim.x) {
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
  if (j > 0) __syncthreads();  // the block reduction's shared buffer is reused
  block_reduce_store<2>(acc, rt.partials + 2 * lb);
  }
  reduce_tail<2>(rt, nlb, gridDim.x);
}

// steprkr stage update (steprkr.f90:160-179); acc = sum psi_new^2.
__global__ void __launch_bounds__(256) k_stat_rk(const StatPW s_in, const ReduceTail rt_in) {
  StatPW s = s_in;
  s.remap(blockIdx.y);
  const ReduceTail rt = remap(rt_in, s.mm, blockIdx.y);
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
                                                        const double* sums, int slot, double n4,
                                                        double dxyz, const MemberMap mm) {
  psi = mm(psi, blockIdx.y);
  den = mm(den, blockIdx.y);
  sums = mm(sums, blockIdx.y);
  const double cnorm = sqrt(n4 / (sums[slot] * dxyz));
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < N;
       i += (long)gridDim.x * blockDim.x) {
    const double v = fabs(psi[i]) * cnorm;
    psi[i] = v;
    den[i] = v * v;
  }
}

__global__ void __launch_bounds__(256) k_sumsq(const double* psi, long N, const ReduceTail rt_in,
                                               const MemberMap mm) {
  psi = mm(psi, blockIdx.y);
  const ReduceTail rt = remap(rt_in, mm, blockIdx.y);
  double acc[1] = {0.0};
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < N;
       i += (long)gridDim.x * blockDim.x)
    acc[0] += psi[i] * psi[i];
  block_reduce_store<1>(acc, rt.partials + blockIdx.x);
  reduce_tail<1>(rt, gridDim.x);
}

// varmu: sum |hpsi - mu psi| * psi (varmu.f90:31).
__global__ void __launch_bounds__(256) k_varmu(const double* hpsi, const double* psi, long N,
                                               double mu, const ReduceTail rt_in, const MemberMap mm) {
  hpsi = mm(hpsi, blockIdx.y);
  psi = mm(psi, blockIdx.y);
  const ReduceTail rt = remap(rt_in, mm, blockIdx.y);
  double acc[1] = {0.0};
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < N;
       i += (long)gridDim.x * blockDim.x)
    acc[0] += fabs(hpsi[i] - mu * psi[i]) * psi[i];
  block_reduce_store<1>(acc, rt.partials + blockIdx.x);
  reduce_tail<1>(rt, gridDim.x);
}

// ---- statics in the mixed path ------------------------------------------------------------------
// psi, psiold, the corrector's output and pc (which carries the full-size prediction sto1) are
// compensated binary32 pairs: hi plane [0, N), lo plane [N, 2N) of the 8N-byte buffer; H psi, q,
// hpsiold, timec, den are binary32.  The pointwise imaginary-time updates below do their few
// operations per point in binary64 on that storage; the norm, mu and error sums are binary64.
HE_D double ld_pair(const float* b, long i, long N) { return (double)b[i] + (double)b[N + i]; }
HE_D void st_pair(float* b, long i, long N, double v) {
  const float h = (float)v;
  b[i] = h;
  b[N + i] = (float)(v - (double)h);
}
struct StatPWM {
  long N;
  double dxyz, n4, dt, dtmin, sdmu, dmumax;
  const double* sums;
  const float* psi;  // pair
  float* out;        // pair
  float* po3;        // pair
  const float* po2;  // pair
  const float* h1;
  float* h2;
  float* pc;         // pair
  float* q;
  float* hsave;
  const float* hpsi;
  float* timec;
  double a, b, c;
  int jr;
};
HE_D double local_dt_m(double hp, double ps, const StatPWM& s) {
  return s.dt / (1.0 + exp((fabs(hp / ps) - s.dmumax) / s.sdmu)) + s.dtmin;
}
__global__ void __launch_bounds__(256) k_stat_predict_m(const StatPWM s, const ReduceTail rt) {
  const double c112 = 112.0 / 121.0, c4o3 = 4.0 / 3.0;
  const double hmean = s.sums[S_STAT_H] * s.dxyz / s.n4;
  double acc[1] = {0.0};
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < s.N; i += (long)gridDim.x * blockDim.x) {
    const double ps = ld_pair(s.psi, i, s.N), hp = s.hpsi[i];
    const double tc = local_dt_m(hp, ps, s);
    s.timec[i] = (float)tc;
    const double s4 = -(hp - hmean * ps);
    const double sto1 = ld_pair(s.po3, i, s.N) + c4o3 * tc * (2.0 * s4 - (double)s.h1[i] + 2.0 * (double)s.h2[i]);
    const double pn = sto1 - c112 * ld_pair(s.pc, i, s.N);
    st_pair(s.po3, i, s.N, pn);
    st_pair(s.pc, i, s.N, sto1);
    s.h2[i] = (float)s4;
    acc[0] += pn * pn;
  }
  block_reduce_store<1>(acc, rt.partials + blockIdx.x);
  reduce_tail<1>(rt, gridDim.x);
}
__global__ void __launch_bounds__(256) k_stat_correct_m(const StatPWM s, const ReduceTail rt) {
  const double c9 = 9.0 / 121.0;
  const double mu = s.sums[S_STAT_MU] * s.dxyz / s.n4;
  double acc[2] = {0.0, 0.0};
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < s.N; i += (long)gridDim.x * blockDim.x) {
    const double ps = ld_pair(s.psi, i, s.N);
    const double s4 = -((double)s.hpsi[i] - mu * ps);
    const double s5 = 0.125 * (9.0 * ld_pair(s.po3, i, s.N) - ld_pair(s.po2, i, s.N) +
                               3.0 * (double)s.timec[i] * (s4 + 2.0 * (double)s.h1[i] - (double)s.h2[i]));
    const double p = ld_pair(s.pc, i, s.N) - s5;
    st_pair(s.pc, i, s.N, p);
    const double o = s5 + c9 * p;
    st_pair(s.out, i, s.N, o);
    acc[0] += fabs(p);
    acc[1] += o * o;
  }
  block_reduce_store<2>(acc, rt.partials + 2 * blockIdx.x);
  reduce_tail<2>(rt, gridDim.x);
}
__global__ void __launch_bounds__(256) k_stat_rk_m(const StatPWM s, const ReduceTail rt) {
  const double err = s.sums[S_STAT_H] * s.dxyz / s.n4;
  double acc[1] = {0.0};
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < s.N; i += (long)gridDim.x * blockDim.x) {
    const double ps = ld_pair(s.psi, i, s.N), hp = s.hpsi[i];
    if (s.jr == 0) s.timec[i] = (float)local_dt_m(hp, ps, s);
    const double tc = s.timec[i];
    const double s4 = -(hp - err * ps);
    const double qq = s.q[i];
    const double s1 = s.a * (s4 - s.b * qq);
    s.q[i] = (float)(qq + 3.0 * s1 - s.c * s4);
    if (s.hsave) s.hsave[i] = (float)s4;
    const double o = ps + tc * s1;
    st_pair(s.out, i, s.N, o);
    acc[0] += o * o;
  }
  block_reduce_store<1>(acc, rt.partials + blockIdx.x);
  reduce_tail<1>(rt, gridDim.x);
}
__global__ void __launch_bounds__(256) k_stat_normalize_m(float* psi, float* den, long N,
                                                          const double* sums, int slot, double n4,
                                                          double dxyz) {
  const double cnorm = sqrt(n4 / (sums[slot] * dxyz));
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < N; i += (long)gridDim.x * blockDim.x) {
    const double v = fabs(ld_pair(psi, i, N)) * cnorm;
    st_pair(psi, i, N, v);
    den[i] = (float)(v * v);
  }
}
__global__ void __launch_bounds__(256) k_sumsq_m(const float* psi, long N, const ReduceTail rt) {
  double acc[1] = {0.0};
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < N; i += (long)gridDim.x * blockDim.x) {
    const double v = ld_pair(psi, i, N);
    acc[0] += v * v;
  }
  block_reduce_store<1>(acc, rt.partials + blockIdx.x);
  reduce_tail<1>(rt, gridDim.x);
}
__global__ void __launch_bounds__(256) k_varmu_m(const float* hpsi, const float* psi, long N, double mu,
                                                 const ReduceTail rt) {
  double acc[1] = {0.0};
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < N; i += (long)gridDim.x * blockDim.x) {
    const double v = ld_pair(psi, i, N);
    acc[0] += fabs((double)hpsi[i] - mu * v) * v;
  }
  block_reduce_store<1>(acc, rt.partials + blockIdx.x);
  reduce_tail<1>(rt, gridDim.x);
}

__global__ void k_copy_slot(double* sums, int dst, int src, const MemberMap mm) {
  sums = mm(sums, blockIdx.y);
  if (threadIdx.x == 0 && blockIdx.x == 0) sums[dst] = sums[src];
}

}  // namespace

static int pw_blocks(const he_ctx_t* ctx) {
  long b = (ctx->N + 255) / 256;
  return (int)(b < kPwBlocks ? b : kPwBlocks);
}
// Grid of a pointwise kernel: blockIdx.y is the member of a group.
static dim3 pw_grid(const he_ctx_t* ctx) { return dim3(pw_blocks(ctx), ctx->nmem); }
// Logical reduction blocks per CTA of the statics pointwise passes: 8 in a group (so that a CTA
// carries more than a couple of points per thread), 1 for a context alone.
static int pw_lpb(const he_ctx_t* ctx) { return (ctx->nmem > 1 && pw_blocks(ctx) % 8 == 0) ? 8 : 1; }
static dim3 pw_grid_lb(const he_ctx_t* ctx) { return dim3(pw_blocks(ctx) / pw_lpb(ctx), ctx->nmem); }

template <int NI, typename TT>
static int launch_impfield_t(he_ctx_t* ctx) {
  OpImpField<NI, TT> op{};
  op.tab = ctx->pot_tab; op.imp = ctx->imp; op.uimp = (TT*)ctx->uimp;
  op.n = ctx->n_imp; op.npot = ctx->npot;
  op.delinter = ctx->delinter; op.rmax = ctx->rmaxinterpol; op.inv_delinter = 1.0 / ctx->delinter;
  op.xmax = ctx->xmax; op.ymax = ctx->ymax; op.zmax = ctx->zmax;
  op.hx = ctx->hx; op.hy = ctx->hy; op.hz = ctx->hz;
  return run_stencil_red(ctx, ctx->g1, (const TT*)ctx->den, op, S_FORCE);
}
template <int NI>
static int launch_impfield(he_ctx_t* ctx) {
  return ctx->mixed ? launch_impfield_t<NI, float>(ctx) : launch_impfield_t<NI, double>(ctx);
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
  s.mm = ctx->mm;
  return s;
}

static StatPWM statpwm(he_ctx_t* ctx, double dt, int n4) {
  StatPWM s{};
  s.N = ctx->N;
  s.dxyz = ctx->dxyz;
  s.n4 = (double)n4;
  s.dt = dt;
  s.dtmin = 1.0e-10; s.sdmu = 1.0e-1; s.dmumax = 1.0e2;  // He_statics/modules.f90:299
  s.sums = ctx->sums;
  s.timec = (float*)ctx->timec;
  return s;
}
static int stat_hpsi(he_ctx_t* ctx, double* out, int slot) {
  if (ctx->mixed) {  // binary32 stencil on psi's hi plane
    OpHpsiRT<float> op{};
    op.s8[0] = (const float*)ctx->pot4;
    op.out = (float*)out;
    op.h2o2m = (float)ctx->fn.h2o2m4;
    return run_stencil_red(ctx, ctx->g2, (const float*)ctx->psi, op, slot);
  }
  OpHpsiR op{};
  op.s8[0] = ctx->pot4;
  op.out = out;
  op.h2o2m = ctx->fn.h2o2m4;
  return run_stencil_red(ctx, ctx->g2, (const double*)ctx->psi, op, slot);
}

// psi *= sqrt(n4 / (sum psi^2 dxyz)), den = psi^2, with the norm sum from `slot`
static int stat_normalize(he_ctx_t* ctx, int n4, int slot = S_STAT_N) {
  tname(ctx, "statics_normalize");
  if (ctx->mixed)
    k_stat_normalize_m<<<pw_blocks(ctx), 256, 0, ctx->stream>>>((float*)ctx->psi, (float*)ctx->den,
                                                                ctx->N, ctx->sums, slot, (double)n4,
                                                                ctx->dxyz);
  else
    k_stat_normalize<<<pw_grid_lb(ctx), 256, 0, ctx->stream>>>((double*)ctx->psi, ctx->den, ctx->N,
                                                            ctx->sums, slot, (double)n4, ctx->dxyz,
                                                            ctx->mm);
  LAUNCHED();
  return HE_OK;
}

static int read_sums(he_ctx_t* ctx) {
  TRY(join_aux(ctx));
  CK(cudaMemcpyAsync(ctx->hsum, ctx->sums, S_COUNT * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  TRY(sync_all(ctx));
  return HE_OK;
}

// Tile autotuner: times the 16-line and 8-line variants of each FFT pass family on this
// context's grid (zero-filled work arrays, one warm-up and three timed launches each) and keeps
// the faster.  Runs once in he_ctx_create.
// Shared memory of the pipelined x pass of `mode` with `rb` rows per tile in this context.
static size_t xpipe_smem(const he_ctx_t* ctx, int mode, int rb) {
  const int sl = ctx->plx.stw_len, n = ctx->nx;
  switch (mode) {
#define HE_XS(M) \
  case M: return ctx->mixed ? xpass_smem<M, float>(sl, rb, n) : xpass_smem<M, double>(sl, rb, n);
    HE_XS(X_R2C_DEN) HE_XS(X_R2C_CORR) HE_XS(X_C2R2) HE_XS(X_C2R2_CORR) HE_XS(X_C2R_POT) HE_XS(X_C2R1)
#undef HE_XS
    default: return 0;
  }
}

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
  auto pick = [&](int* knob, int (*fn)(he_ctx_t*), const char* what) -> int {
    float t16 = 0.0f, t8 = 0.0f;
    *knob = 16;
    TRY(timed(fn, &t16));
    *knob = 8;
    TRY(timed(fn, &t8));
    *knob = (t8 < t16) ? 8 : 16;
    char line[96];
    snprintf(line, sizeof line, "%s 16: %.2f us\n%s 8: %.2f us\n", what, 1e3f * t16 / 3.0f, what,
             1e3f * t8 / 3.0f);
    ctx->tune_log += line;
    return HE_OK;
  };
  int st = HE_OK;
  // x pass, per mode the step uses: {one-shot, pipelined} x {16, 8 rows}; a pipelined variant
  // whose shared memory does not fit an SM is skipped.  The trials run on the context's
  // (not yet initialised) work arrays; only their times matter.
  struct XTrial {
    int mode;
    const char* name;
    int (*fn)(he_ctx_t*);
  };
  const XTrial dyn_trials[3] = {
      {X_R2C_DEN, "x r2c den", [](he_ctx_t* c) -> int {
         XArgs a = xargs(c);
         a.den = c->den; a.specA = c->wA;
         return xpass<X_R2C_DEN>(c, a);
       }},
      {X_C2R2_CORR, "x c2r2 corr", [](he_ctx_t* c) -> int {
         XArgs a = xargs(c);
         a.specA = c->wA; a.specB = c->wB; a.den = c->den;
         a.out1 = c->dencg; a.out2 = c->delj4;
         return xpass<X_C2R2_CORR>(c, a);
       }},
      {X_C2R_POT, "x c2r pot", [](he_ctx_t* c) -> int {
         XArgs a = xargs(c);
         a.specA = c->wA; a.den = c->den; a.dencg_in = c->dencg; a.delj4_in = c->delj4;
         a.out1 = c->pot4;
         return xpass<X_C2R_POT>(c, a);
       }}};
  if (x_fast(ctx, 16) && x_fast(ctx, 8) && ctx->mode != HE_MODE_STATICS) {
    int maxsm = 0, dev = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    for (const XTrial& tr : dyn_trials) {
      float best = 1e30f;
      int best_tile = 16;
      bool best_pipe = false;
      for (int pipe = 0; pipe < 2 && st == HE_OK; ++pipe)
        for (int tile : {16, 8}) {
          if (pipe && (int)xpipe_smem(ctx, tr.mode, tile) > maxsm) continue;
          ctx->xpipe[tr.mode] = pipe != 0;
          ctx->xtile[tr.mode] = tile;
          float ms = 0.0f;
          st = timed(tr.fn, &ms);
          if (st != HE_OK) break;
          char line[96];
          snprintf(line, sizeof line, "%s %s %d: %.2f us\n", tr.name, pipe ? "pipelined" : "one-shot",
                   tile, 1e3f * ms / 3.0f);
          ctx->tune_log += line;
          if (ms < best) { best = ms; best_tile = tile; best_pipe = pipe != 0; }
        }
      ctx->xpipe[tr.mode] = best_pipe;
      ctx->xtile[tr.mode] = best_tile;
    }
    ctx->tile_x = ctx->xtile[X_C2R2_CORR];
  }
  if (st == HE_OK && yz_fast(ctx->ny))
    st = pick(&ctx->tile_y, [](he_ctx_t* c) -> int { return ypass(c, c->wA, c->wB, true); }, "y");
  if (st == HE_OK && yz_fast(ctx->nz)) {
    auto zfn = [](he_ctx_t* c) -> int { return zconv(c, c->wA, c->wcgk, c->wB, c->fvlj4, nullptr); };
    st = pick(&ctx->tile_z, zfn, "z");
    if (st == HE_OK) {
      // the register variant against the best shared-memory pass so far
      const int tile0 = ctx->tile_z;
      float t0 = 0.0f;
      st = timed(zfn, &t0);
      float best = t0;
      int best_tile = tile0;
      bool best_reg = false;
      ctx->zreg = true;
      for (int tile : {16, 8}) {
        if (st != HE_OK) break;
        ctx->tile_z = tile;
        float ms = 0.0f;
        st = timed(zfn, &ms);
        char line[96];
        snprintf(line, sizeof line, "z register %d: %.2f us\n", tile, 1e3f * ms / 3.0f);
        ctx->tune_log += line;
        if (ms < best) { best = ms; best_tile = tile; best_reg = true; }
      }
      ctx->zreg = best_reg;
      ctx->tile_z = best_tile;
    }
  }
  if (st == HE_OK && yz_fusable(ctx)) {
    // the two-kernel convolution (fden*wcgk, fden*fvlj4) with separate y / z passes against the
    // fused y-z kernel
    auto conv = [](he_ctx_t* c) -> int {
      if (c->yzfuse) return yzconv(c, c->wA, c->wcgk, c->wB, c->fvlj4, c->fden);
      TRY(ypass(c, c->wA, nullptr, false));
      TRY(zconv(c, c->wA, c->wcgk, c->wB, c->fvlj4, c->fden));
      return ypass(c, c->wA, c->wB, true);
    };
    float ts = 0.0f, tf = 0.0f;
    ctx->yzfuse = false;
    st = timed(conv, &ts);
    if (st == HE_OK) {
      ctx->yzfuse = true;
      st = timed(conv, &tf);
    }
    if (st == HE_OK) {
      char line[128];
      snprintf(line, sizeof line, "yz convolution separate passes: %.2f us\nyz convolution fused: %.2f us\n",
               1e3f * ts / 3.0f, 1e3f * tf / 3.0f);
      ctx->tune_log += line;
      ctx->yzfuse = tf < ts;
    } else {
      ctx->yzfuse = false;
    }
  }
  if (st == HE_OK && ctx->mode == HE_MODE_DYNAMICS && !ctx->otc && xy_fusable(ctx)) {
    // the whole classical field evaluation, plane-fused against the separate passes
    auto sep = [](he_ctx_t* c) -> int {
      TRY(spectrum_cg_lj(c));
      XArgs a = xargs(c);
      a.specA = c->wA; a.specB = c->wB; a.den = c->den;
      a.out1 = c->dencg; a.out2 = c->delj4;
      TRY(xpass<X_C2R2_CORR>(c, a));
      return correlation_tail(c, nullptr, nullptr);
    };
    auto fused = [](he_ctx_t* c) -> int { return poten_fused(c, nullptr, nullptr); };
    float ts = 0.0f, tf = 0.0f;
    st = timed(sep, &ts);
    if (st == HE_OK) st = timed(fused, &tf);
    if (st == HE_OK) {
      char line[128];
      snprintf(line, sizeof line, "field separate passes: %.2f us\nfield x-y fused: %.2f us\n",
               1e3f * ts / 3.0f, 1e3f * tf / 3.0f);
      ctx->tune_log += line;
      ctx->xyfuse = tf < ts;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (st == HE_OK) CK(cudaMemsetAsync(ctx->wA, 0, 16 * ctx->Nk, ctx->stream));
  if (st == HE_OK) CK(cudaMemsetAsync(ctx->wB, 0, 16 * ctx->Nk, ctx->stream));
  return st;
}

// ------------------------------------------------------------------------------------------------
// C-ABI
// ------------------------------------------------------------------------------------------------
// ------------------------------------------------------------------------------------------------
// alpha_s term (core4 = 'OTC'): term_alfa.f90:5-117
// ------------------------------------------------------------------------------------------------
template <int N, int TILE, typename Rt>
static int zmix_n(he_ctx_t* ctx, const ZMixArgs& a);
static int zmix(he_ctx_t* ctx, ZMixArgs a);
static int qkernels_to_f32(he_ctx_t* ctx);

// out[k] = C2R(R2C(in[k]) * ker) for n <= 3 real fields, through wB, wC, wD.
static int conv_fields(he_ctx_t* ctx, const double* const* in, double* const* out, int n,
                       const double* ker) {
  double2* buf[3] = {ctx->wB, ctx->wC, ctx->wD};
  XArgs a = xargs(ctx);
  for (int k = 0; k < n; ++k) {
    a.den = in[k];
    a.specA = buf[k];
    TRY(xpass<X_R2C_DEN>(ctx, a));
  }
  TRY(ypass(ctx, buf[0], n > 1 ? buf[1] : nullptr, false));
  if (n > 2) TRY(ypass(ctx, buf[2], nullptr, false));
  for (int k = 0; k < n; ++k) TRY(zconv(ctx, buf[k], ker, nullptr, nullptr, nullptr));
  TRY(ypass(ctx, buf[0], n > 1 ? buf[1] : nullptr, true));
  if (n > 2) TRY(ypass(ctx, buf[2], nullptr, true));
  XArgs c = xargs(ctx);
  int k = 0;
  if (n >= 2) {
    c.specA = buf[0]; c.specB = buf[1];
    c.out1 = out[0]; c.out2 = out[1];
    TRY(xpass<X_C2R2>(ctx, c));
    k = 2;
  }
  if (k < n) {
    XArgs d = xargs(ctx);
    d.specA = buf[k];
    d.out1 = out[k];
    TRY(xpass<X_C2R1>(ctx, d));
  }
  return HE_OK;
}

// denalf = C2R(fden * kalfs) (Dynamics_TDDFT/poten.f90:200-205; BCN4HeDFT.f90:1142-1148).
static int alfa_density(he_ctx_t* ctx) {
  ZMixArgs z{};
  z.nout = 1;
  z.out[0] = ctx->wC; z.nterm[0] = 1; z.src[0][0] = ctx->fden; z.ker[0][0] = ctx->kalfs;
  TRY(zmix(ctx, z));
  TRY(ypass(ctx, ctx->wC, nullptr, true));
  XArgs a = xargs(ctx);
  a.specA = ctx->wC;
  a.out1 = ctx->denalf;
  return xpass<X_C2R1>(ctx, a);
}

// term_alfa (needs denalf and materialised dxden/dyden/dzden); leaves ualphas, falfs, int*alf.
static int term_alfa(he_ctx_t* ctx) {
  const long N = ctx->N;
  const int nb = pw_blocks(ctx);
  tname(ctx, "alphas_pointwise");
  k_alf_src<<<nb, 256, 0, ctx->stream>>>(ctx->denalf, ctx->dxden, ctx->dyden, ctx->dzden,
                                         ctx->fn.den0s, N, ctx->falfs, ctx->as1, ctx->as2, ctx->as3);
  LAUNCHED();
  {
    const double* in[3] = {ctx->as1, ctx->as2, ctx->as3};
    double* out[3] = {ctx->intxalf, ctx->intyalf, ctx->intzalf};
    TRY(conv_fields(ctx, in, out, 3, ctx->kalfs));
  }
  tname(ctx, "alphas_pointwise");
  k_alf_dot<<<nb, 256, 0, ctx->stream>>>(ctx->dxden, ctx->dyden, ctx->dzden, ctx->intxalf,
                                         ctx->intyalf, ctx->intzalf, N, ctx->as1);
  LAUNCHED();
  {
    const double* in[1] = {ctx->as1};
    double* out[1] = {ctx->ua_raw};
    TRY(conv_fields(ctx, in, out, 1, ctx->kalfs));
  }
  tname(ctx, "alphas_pointwise");
  k_alf_fi<<<nb, 256, 0, ctx->stream>>>(ctx->falfs, ctx->intxalf, ctx->intyalf, ctx->intzalf, N,
                                        ctx->as1, ctx->as2, ctx->as3);
  LAUNCHED();
  OpAxisDeriv<0> dx{};
  dx.out = ctx->as4;
  TRY(run_stencil(ctx, ctx->g1, ctx->as1, dx));
  OpAxisDeriv<1> dy{};
  dy.out = ctx->as5;
  TRY(run_stencil(ctx, ctx->g1, ctx->as2, dy));
  OpAlfFinal fin{};
  fin.s8[0] = ctx->ua_raw; fin.s8[1] = ctx->as4; fin.s8[2] = ctx->as5;
  fin.out = ctx->ualphas;
  fin.den0s = ctx->fn.den0s; fin.h2o2m4 = ctx->fn.h2o2m4; fin.alphas = ctx->fn.alphas;
  return run_stencil(ctx, ctx->g1, ctx->as3, fin);
}

// The ealphas sum, queued into slot S_ALF (read with the other energy sums).
static int alfa_energy_sum(he_ctx_t* ctx) {
  tname(ctx, "alphas_energy");
  k_alf_energy<<<pw_blocks(ctx), 256, 0, ctx->stream>>>(ctx->falfs, ctx->dxden, ctx->dyden, ctx->dzden,
                                                        ctx->intxalf, ctx->intyalf, ctx->intzalf,
                                                        ctx->N, tail(ctx, S_ALF));
  LAUNCHED();
  return HE_OK;
}
static double alfa_energy(const he_ctx_t* ctx) {
  return -ctx->fn.h2o2m4 * 0.5 * ctx->fn.alphas * ctx->hsum[S_ALF] * ctx->dxyz;
}

__global__ void __launch_bounds__(256) k_to_f32(const double* __restrict__ a, float* __restrict__ b,
                                                long n, double scale);
__global__ void __launch_bounds__(256) k_to_f64(const float* __restrict__ a, double* __restrict__ b, long n);

// The binary64 passes inside a mixed-precision context: the pass dispatch reads ctx->mixed, the
// binary64 kernels are unscaled (cg_scale 1) and the x pass runs one-shot (the pipelined variant's
// tiles were tuned for the binary32 chain's shared memory).  Restored on scope exit.
struct Binary64Passes {
  he_ctx_t* c;
  bool mixed;
  double cg_scale;
  bool xpipe[6];
  explicit Binary64Passes(he_ctx_t* ctx) : c(ctx), mixed(ctx->mixed), cg_scale(ctx->cg_scale) {
    for (int m = 0; m < 6; ++m) { xpipe[m] = c->xpipe[m]; c->xpipe[m] = false; }
    c->mixed = false;
    c->cg_scale = 1.0;
  }
  ~Binary64Passes() {
    for (int m = 0; m < 6; ++m) c->xpipe[m] = xpipe[m];
    c->mixed = mixed;
    c->cg_scale = cg_scale;
  }
};

// grad den into dxden, dyden, dzden (binary64 den; derden.f90:26-28)
static int derden_of(he_ctx_t* ctx, const double* den) {
  if (!ctx->dxden) {
    TRY(dalloc_t(ctx, &ctx->dxden, ctx->N));
    TRY(dalloc_t(ctx, &ctx->dyden, ctx->N));
    TRY(dalloc_t(ctx, &ctx->dzden, ctx->N));
  }
  OpDerden op{};
  op.gx = ctx->dxden; op.gy = ctx->dyden; op.gz = ctx->dzden;
  return run_stencil(ctx, ctx->g1, den, op);
}

// core4 = 'OTC' in the dynamics modes: derden, the alpha_s density and term_alfa
// (Dynamics_TDDFT/poten.f90:144, :200-210; quantum poten.f90:48, :126-139).  The mixed path runs
// them in binary64 on a binary64 copy of den (denalf = C2R(R2C(den) kalfs), which equals the
// reference's C2R(fden kalfs) for the current den) and hands the binary32 epilogue a binary32
// copy of ualphas.  Returns the ualphas array the pot4 epilogue adds (binary32 or binary64).
static int otc_terms(he_ctx_t* ctx, const double** ualphas) {
  if (!ctx->mixed) {
    TRY(derden_of(ctx, ctx->den));
    TRY(alfa_density(ctx));
    TRY(term_alfa(ctx));
    *ualphas = ctx->ualphas;
    return HE_OK;
  }
  tname(ctx, "alphas_convert");
  k_to_f64<<<kPwBlocks, 256, 0, ctx->stream>>>((const float*)ctx->den, ctx->den64, ctx->N);
  LAUNCHED();
  {
    Binary64Passes f64(ctx);
    TRY(derden_of(ctx, ctx->den64));
    const double* in[1] = {ctx->den64};
    double* out[1] = {ctx->denalf};
    TRY(conv_fields(ctx, in, out, 1, ctx->kalfs));
    TRY(term_alfa(ctx));
  }
  tname(ctx, "alphas_convert");
  k_to_f32<<<kPwBlocks, 256, 0, ctx->stream>>>(ctx->ualphas, ctx->ualphas_f, ctx->N, 1.0);
  LAUNCHED();
  *ualphas = reinterpret_cast<const double*>(ctx->ualphas_f);
  return HE_OK;
}

// The statics refresh's part of the alpha_s term (BCN4HeDFT.f90:1142-1148): denalf from the
// refreshed fden (and, through he_derden, the gradients poten's term_alfa uses); in the mixed
// path both in binary64 from a binary64 copy of the refreshed den.
static int statics_alfa_density(he_ctx_t* ctx) {
  if (!ctx->mixed) return alfa_density(ctx);
  tname(ctx, "alphas_convert");
  k_to_f64<<<kPwBlocks, 256, 0, ctx->stream>>>((const float*)ctx->den, ctx->den64, ctx->N);
  LAUNCHED();
  Binary64Passes f64(ctx);
  TRY(derden_of(ctx, ctx->den64));
  const double* in[1] = {ctx->den64};
  double* out[1] = {ctx->denalf};
  return conv_fields(ctx, in, out, 1, ctx->kalfs);
}
// The statics poten's term_alfa (He_statics/poten.f90:86-91) on the refresh's denalf and
// gradients; the mixed path runs it in binary64 and returns ualphas' binary32 copy.
static int statics_term_alfa(he_ctx_t* ctx, const double** ualphas) {
  if (!ctx->mixed) {
    TRY(term_alfa(ctx));
    *ualphas = ctx->ualphas;
    return HE_OK;
  }
  {
    Binary64Passes f64(ctx);
    TRY(term_alfa(ctx));
  }
  tname(ctx, "alphas_convert");
  k_to_f32<<<kPwBlocks, 256, 0, ctx->stream>>>(ctx->ualphas, ctx->ualphas_f, ctx->N, 1.0);
  LAUNCHED();
  *ualphas = reinterpret_cast<const double*>(ctx->ualphas_f);
  return HE_OK;
}

// ------------------------------------------------------------------------------------------------
// quantum impurities (HE_MODE_QUANTUM, Dynamics_quantum_impurities)
// ------------------------------------------------------------------------------------------------
template <int N, int TILE, typename Rt>
static int zmix_n(he_ctx_t* ctx, const ZMixArgs& a) {
  const int tk = (N > 0) ? TILE : ctx->tkx;
  const size_t smem = fft_smem(ctx->plz, tk, 3, sizeof(typename Cx<Rt>::T));
  const int nthr = (N > 0) ? tile_threads(TILE) : 256;
  dim3 grid((ctx->nxh + tk - 1) / tk, ctx->ny, ctx->nmem);
  void (*k)(ZMixArgs) = ctx->nmem > 1 ? k_zmix<N, TILE, Rt, true> : k_zmix<N, TILE, Rt, false>;
  CK(set_smem_attr((const void*)k, smem));
  tname(ctx, a.nout == 0 ? "fft_z_fwd" : a.fwd_in ? "fft_z_mix_fwd" : "fft_z_mix");
  k<<<grid, nthr, smem, ctx->stream>>>(a);
  LAUNCHED();
  return HE_OK;
}
template <typename Rt>
static int zmix_t(he_ctx_t* ctx, const ZMixArgs& a) {
  const int tile = ctx->tile_z;
  if (yz_fast(ctx->nz)) {
    switch (ctx->nz) {
#define HE_CASE(N) \
  case N: return tile == 8 ? zmix_n<N, 8, Rt>(ctx, a) : zmix_n<N, 16, Rt>(ctx, a);
      HE_FFT_SIZES(HE_CASE)
#undef HE_CASE
    }
  }
  return zmix_n<0, 16, Rt>(ctx, a);
}
static int zmix(he_ctx_t* ctx, ZMixArgs a) {
  a.nxh = ctx->nxh; a.ny = ctx->ny; a.nz = ctx->nz; a.tkx = ctx->tkx;
  a.pl = ctx->plz;
  a.mm = ctx->mm;
  if (!ctx->mixed) return zmix_t<double>(ctx, a);
  // the binary32 chain reads the kernels' binary32 copies (passed through the same slots)
  for (int o = 0; o < a.nout; ++o)
    for (int t = 0; t < a.nterm[o]; ++t) {
      const float* kf = kernel_f32(ctx, a.ker[o][t]);
      if (!kf) return fail(ctx, HE_ERR_STATE, "no binary32 copy of a k-space kernel");
      a.ker[o][t] = reinterpret_cast<const double*>(kf);
    }
  return zmix_t<float>(ctx, a);
}

// One synthesis output: sum over terms of (spectrum x kernel), inverse-transformed into `out`.
struct QOut {
  double* out;
  int nterm;
  const double2* src[kMaxTerms];
  const double* ker[kMaxTerms];
};

// z synthesis of one or two outputs into wC (and wD), inverse y, and C2R in x.
static int q_synth(he_ctx_t* ctx, const QOut* o, int nout, const double2* fwd_in) {
  ZMixArgs z{};
  z.fwd_in = fwd_in;
  z.nout = nout;
  double2* buf[2] = {ctx->wC, ctx->wD};
  for (int k = 0; k < nout; ++k) {
    z.out[k] = buf[k];
    z.nterm[k] = o[k].nterm;
    for (int t = 0; t < o[k].nterm; ++t) { z.src[k][t] = o[k].src[t]; z.ker[k][t] = o[k].ker[t]; }
  }
  TRY(zmix(ctx, z));
  TRY(ypass(ctx, ctx->wC, nout > 1 ? ctx->wD : nullptr, true));
  XArgs a = xargs(ctx);
  a.renor1 = a.renor;  // no wcgk product here (its binary32 copy is the scaled one)
  a.specA = ctx->wC;
  a.out1 = o[0].out;
  if (nout > 1) {
    a.specB = ctx->wD;
    a.out2 = o[1].out;
    return xpass<X_C2R2>(ctx, a);
  }
  return xpass<X_C2R1>(ctx, a);
}

// Forward spectra (x, y, z) of the impurity densities |psix_i|^2 into sx[i].
static int q_denx_spectra(he_ctx_t* ctx) {
  XArgs a = xargs(ctx);
  for (int i = 0; i < ctx->nq; ++i) {
    a.den = ctx->denx[i];
    a.specA = ctx->sx[i];
    TRY(xpass<X_R2C_DEN>(ctx, a));
  }
  for (int i = 0; i < ctx->nq; i += 2) TRY(ypass(ctx, ctx->sx[i], i + 1 < ctx->nq ? ctx->sx[i + 1] : nullptr, false));
  for (int i = 0; i < ctx->nq; ++i) {
    ZMixArgs z{};
    z.fwd_in = ctx->sx[i];
    z.fwd_store = ctx->sx[i];
    TRY(zmix(ctx, z));
  }
  return HE_OK;
}

// potenimp (Dynamics_quantum_impurities/potenimp.f90:1-43): fden = R2C(den), potx4 and upotx_i.
// The forward pass of den also leaves fden*wcgk and fden*fvlj4 (x,y domain) in wA/wB for poten.
static int q_potenimp(he_ctx_t* ctx) {
  const int n = ctx->nq;
  XArgs a = xargs(ctx);
  a.den = ctx->den;
  a.specA = ctx->wA;
  TRY(xpass<X_R2C_DEN>(ctx, a));
  if (n == 1) {
    a.den = ctx->denx[0];
    a.specA = ctx->sx[0];
    TRY(xpass<X_R2C_DEN>(ctx, a));
    TRY(ypass(ctx, ctx->wA, ctx->sx[0], false));
  } else {
    TRY(ypass(ctx, ctx->wA, nullptr, false));
  }
  TRY(zconv(ctx, ctx->wA, ctx->wcgk, ctx->wB, ctx->fvlj4, ctx->fden));
  ctx->cglj_pending = true;
  if (n == 1) {
    // potx4 = C2R(R2C(|psix|^2) uimp_k), upotx = C2R(fden uimp_k), fused behind psix's z pass.
    QOut o[2] = {};
    o[0].out = ctx->potx4; o[0].nterm = 1; o[0].src[0] = nullptr; o[0].ker[0] = ctx->uimpk[0];
    o[1].out = ctx->upotx[0]; o[1].nterm = 1; o[1].src[0] = ctx->fden; o[1].ker[0] = ctx->uimpk[0];
    return q_synth(ctx, o, 2, ctx->sx[0]);
  }
  TRY(q_denx_spectra(ctx));
  // Outputs: potx4 = sum_i sx_i uimp_k_i; upotx_i = fden uimp_k_i + sum_{j != i} sx_j uimp_k_k(i,j).
  // (The reference sums the C2R of each term in real space; the sums here are taken in k space.)
  std::vector<QOut> outs(1 + n);
  outs[0] = QOut{};
  outs[0].out = ctx->potx4;
  for (int i = 0; i < n; ++i) {
    outs[0].src[outs[0].nterm] = ctx->sx[i];
    outs[0].ker[outs[0].nterm++] = ctx->uimpk[i];
  }
  for (int i = 0; i < n; ++i) {
    QOut& o = outs[1 + i];
    o = QOut{};
    o.out = ctx->upotx[i];
    o.src[o.nterm] = ctx->fden;
    o.ker[o.nterm++] = ctx->uimpk[i];
    for (int j = 0; j < n; ++j) {
      const double* kk = ctx->uimpkk[i + kMaxQImp * j];
      if (j == i || !kk) continue;
      o.src[o.nterm] = ctx->sx[j];
      o.ker[o.nterm++] = kk;
    }
  }
  for (size_t k = 0; k < outs.size(); k += 2) TRY(q_synth(ctx, &outs[k], k + 1 < outs.size() ? 2 : 1, nullptr));
  return HE_OK;
}

// poten (Dynamics_quantum_impurities/poten.f90:5-155): dencg, delj4 from fden, then the
// correlation term and pot4 = delj4 + dencg^2 (cp4/2 + cpp4/3 dencg) + sto1 + potx4 (+ penalty).
static int q_poten(he_ctx_t* ctx) {
  if (!ctx->cglj_pending) {
    ZMixArgs z{};
    z.nout = 2;
    z.out[0] = ctx->wA; z.nterm[0] = 1; z.src[0][0] = ctx->fden; z.ker[0][0] = ctx->wcgk;
    z.out[1] = ctx->wB; z.nterm[1] = 1; z.src[1][0] = ctx->fden; z.ker[1][0] = ctx->fvlj4;
    TRY(zmix(ctx, z));
  }
  ctx->cglj_pending = false;
  TRY(ypass(ctx, ctx->wA, ctx->wB, true));
  XArgs a = xargs(ctx);
  a.specA = ctx->wA; a.specB = ctx->wB;
  a.den = ctx->den;
  a.out1 = ctx->dencg; a.out2 = ctx->delj4;
  TRY(xpass<X_C2R2_CORR>(ctx, a));
  const double* ua = nullptr;
  if (ctx->otc) TRY(otc_terms(ctx, &ua));  // Dynamics_quantum_impurities/poten.f90:48, :126-139
  return correlation_tail(ctx, ctx->potx4, ua);
}

static int q_field(he_ctx_t* ctx) {
  TRY(q_potenimp(ctx));
  return q_poten(ctx);
}

static int q_cnorm2(he_ctx_t* ctx, int i) {
  tname(ctx, "impurity_density");
  if (ctx->mixed)
    k_cnorm2_pair<<<pw_grid(ctx), 256, 0, ctx->stream>>>(
        (const float2*)ctx->psix[i], (const float2*)ctx->psix[i] + ctx->N, (float*)ctx->denx[i], ctx->N,
        ctx->mm);
  else
    k_cnorm2<<<pw_grid(ctx), 256, 0, ctx->stream>>>((const double2*)ctx->psix[i], ctx->denx[i], ctx->N,
                                                    ctx->mm);
  LAUNCHED();
  return HE_OK;
}

// steprk (Dynamics_quantum_impurities/steprk.f90:1-124).  He and each impurity take the same
// RK-Gill stage; the field is re-evaluated after stages 1-3.
static int q_steprk(he_ctx_t* ctx, double deltat) {
  const double r2 = 1.0 / std::sqrt(2.0);
  const double arun[4] = {0.5, 1.0 - r2, 1.0 + r2, 1.0 / 6.0};
  const double brun[4] = {2.0, 1.0, 1.0, 2.0};
  const double crun[4] = {0.5, 1.0 - r2, 1.0 + r2, 0.5};
  for (int jr = 0; jr < 4; ++jr) {
    auto stage = [&](void*& f, void*& scratch, void* qq, void** po, void** ho, const double* pot,
                     double mu, double h2o2m, double* dens) -> int {
      if (ctx->mixed) {
        void* ob = jr == 0 ? po[2] : scratch;
        OpRKMQ op{};
        op.s8[0] = (const float*)pot;
        op.s16[0] = (const float2*)qq; op.s16[1] = lo_plane(ctx, f);
        op.q = (float2*)qq;
        op.out_hi = hi_plane(ob); op.out_lo = lo_plane(ctx, ob);
        op.hsave = jr == 0 ? (float2*)ho[1] : nullptr;
        op.den = (float*)dens;
        op.tm = timec_view(ctx);
        op.h2o2m = (float)h2o2m;
        op.mu = (float)mu;
        op.a = (float)arun[jr]; op.b = (float)brun[jr]; op.cc = (float)crun[jr]; op.dt = (float)deltat;
        TRY(run_stencil(ctx, ctx->g2, hi_plane(f), op));
      } else {
        OpRKQ op{};
        op.s8[0] = pot;
        op.s16[0] = (const double2*)qq;
        op.q = (double2*)qq;
        op.out = (double2*)(jr == 0 ? po[2] : scratch);
        op.hsave = jr == 0 ? (double2*)ho[1] : nullptr;
        op.den = dens;
        op.tm = timec_view(ctx);
        op.h2o2m = h2o2m;
        op.mu = mu;
        op.a = arun[jr]; op.b = brun[jr]; op.cc = crun[jr]; op.dt = deltat;
        TRY(run_stencil(ctx, ctx->g2, (const double2*)f, op));
      }
      if (jr == 0) {
        void* o3 = po[2];
        po[2] = po[1];
        po[1] = po[0];
        po[0] = f;
        f = o3;
        std::swap(ho[0], ho[1]);
      } else {
        std::swap(f, scratch);
      }
      return HE_OK;
    };
    TRY(stage(ctx->psi, ctx->scratch, ctx->q, ctx->psiold, ctx->hpsiold, ctx->pot4, ctx->mu4,
              ctx->fn.h2o2m4, ctx->den));
    for (int i = 0; i < ctx->nq; ++i)
      TRY(stage(ctx->psix[i], ctx->xscratch, ctx->qx[i], ctx->psixold[i], ctx->hpsixold[i],
                ctx->upotx[i], 0.0, ctx->h2o2mx[i], ctx->denx[i]));
    if (jr <= 2) TRY(q_field(ctx));
  }
  for (int i = 0; i < 3; ++i) ctx->ioldp[i] = i + 1;
  ctx->ioldh[0] = 1; ctx->ioldh[1] = 2;
  return HE_OK;
}

// steppc (Dynamics_quantum_impurities/steppc.f90:1-157): predictor + modifier for He and every
// impurity, potenimp + poten, corrector for all.  The impurities' ring indices ioldpx/ioldhx
// always equal ioldp/ioldh (both start at 1,2,3 / 1,2 and rotate together), so one set serves.
static int q_steppc(he_ctx_t* ctx, double deltat, double* errHe, double* errpsix) {
  const double c112 = 112.0 / 121.0, c9 = 9.0 / 121.0, c4o3 = 4.0 / 3.0;
  auto predict = [&](void*& f, void* pcc, void** po, void** ho, const double* pot, double mu,
                     double h2o2m, double* dens) -> int {
    if (ctx->mixed) {  // pc is left alone (see OpPredictMT)
      void* p3 = po[ctx->ioldp[2] - 1];
      OpPredictMQ op{};
      op.s8[0] = (const float*)pot;
      op.po3_hi = hi_plane(p3); op.po3_lo = lo_plane(ctx, p3);
      op.h2 = (float2*)ho[ctx->ioldh[1] - 1];
      op.s16[0] = op.po3_hi;
      op.s16[1] = op.po3_lo;
      op.s16[2] = (const float2*)ho[ctx->ioldh[0] - 1];
      op.s16[3] = op.h2;
      op.s16[4] = (const float2*)pcc;
      op.den = (float*)dens;
      op.tm = timec_view(ctx);
      op.h2o2m = (float)h2o2m;
      op.mu = (float)mu;
      op.s43 = (float)(c4o3 * deltat);
      op.c112 = (float)c112;
      TRY(run_stencil(ctx, ctx->g2, hi_plane(f), op));
      std::swap(f, po[ctx->ioldp[2] - 1]);
      return HE_OK;
    }
    OpPredictQ op{};
    op.s8[0] = pot;
    op.po3 = (double2*)po[ctx->ioldp[2] - 1];
    op.h2 = (double2*)ho[ctx->ioldh[1] - 1];
    op.pc = (double2*)pcc;
    op.s16[0] = op.po3;
    op.s16[1] = (const double2*)ho[ctx->ioldh[0] - 1];
    op.s16[2] = op.h2;
    op.s16[3] = op.pc;
    op.den = dens;
    op.tm = timec_view(ctx);
    op.h2o2m = h2o2m;
    op.mu = mu;
    op.s43 = c4o3 * deltat;
    op.c112 = c112;
    TRY(run_stencil(ctx, ctx->g2, (const double2*)f, op));
    std::swap(f, po[ctx->ioldp[2] - 1]);
    return HE_OK;
  };
  TRY(predict(ctx->psi, ctx->pc, ctx->psiold, ctx->hpsiold, ctx->pot4, ctx->mu4, ctx->fn.h2o2m4, ctx->den));
  for (int i = 0; i < ctx->nq; ++i)
    TRY(predict(ctx->psix[i], ctx->pcx[i], ctx->psixold[i], ctx->hpsixold[i], ctx->upotx[i], 0.0,
                ctx->h2o2mx[i], ctx->denx[i]));
  std::swap(ctx->ioldh[0], ctx->ioldh[1]);
  TRY(q_field(ctx));
  auto correct = [&](void*& f, void*& scratch, void* pcc, void** po, void** ho, const double* pot,
                     double mu, double h2o2m, double* dens, int slot) -> int {
    if (ctx->mixed) {
      void* a3 = po[ctx->ioldp[2] - 1];
      void* a2 = po[ctx->ioldp[1] - 1];
      OpCorrectMQ op{};
      op.s8[0] = (const float*)pot;
      op.s16[0] = lo_plane(ctx, f);
      op.s16[1] = hi_plane(a3); op.s16[2] = lo_plane(ctx, a3);
      op.s16[3] = hi_plane(a2); op.s16[4] = lo_plane(ctx, a2);
      op.s16[5] = (const float2*)ho[ctx->ioldh[0] - 1];
      op.s16[6] = (const float2*)ho[ctx->ioldh[1] - 1];
      op.s16[7] = (const float2*)pcc;
      op.pc = (float2*)pcc;
      op.out_hi = hi_plane(scratch); op.out_lo = lo_plane(ctx, scratch);
      op.den = (float*)dens;
      op.tm = timec_view(ctx);
      op.h2o2m = (float)h2o2m;
      op.mu = (float)mu;
      op.s3 = (float)(3.0 * deltat);
      op.c9 = (float)c9;
      op.c112 = (float)c112;
      TRY(run_stencil_red(ctx, ctx->g2, hi_plane(f), op, slot));
      std::swap(f, scratch);
      return HE_OK;
    }
    OpCorrectQ op{};
    op.s8[0] = pot;
    op.s16[0] = (const double2*)po[ctx->ioldp[2] - 1];
    op.s16[1] = (const double2*)po[ctx->ioldp[1] - 1];
    op.s16[2] = (const double2*)ho[ctx->ioldh[0] - 1];
    op.s16[3] = (const double2*)ho[ctx->ioldh[1] - 1];
    op.s16[4] = (const double2*)pcc;
    op.pc = (double2*)pcc;
    op.out = (double2*)scratch;
    op.den = dens;
    op.tm = timec_view(ctx);
    op.h2o2m = h2o2m;
    op.mu = mu;
    op.s3 = 3.0 * deltat;
    op.c9 = c9;
    TRY(run_stencil_red(ctx, ctx->g2, (const double2*)f, op, slot));
    std::swap(f, scratch);
    return HE_OK;
  };
  TRY(correct(ctx->psi, ctx->scratch, ctx->pc, ctx->psiold, ctx->hpsiold, ctx->pot4, ctx->mu4,
              ctx->fn.h2o2m4, ctx->den, S_ERRHE));
  for (int i = 0; i < ctx->nq; ++i)
    TRY(correct(ctx->psix[i], ctx->xscratch, ctx->pcx[i], ctx->psixold[i], ctx->hpsixold[i],
                ctx->upotx[i], 0.0, ctx->h2o2mx[i], ctx->denx[i], S_ERRX + i));
  const int a = ctx->ioldp[2];
  ctx->ioldp[2] = ctx->ioldp[1];
  ctx->ioldp[1] = ctx->ioldp[0];
  ctx->ioldp[0] = a;
  if (errHe || errpsix) {
    TRY(read_sums(ctx));
    if (errHe) *errHe = c9 * ctx->hsum[S_ERRHE] / (double)ctx->N;
    if (errpsix) {
      double e = 0.0;
      for (int i = 0; i < ctx->nq; ++i) e = e + c9 * ctx->hsum[S_ERRX + i];
      *errpsix = e / (double)ctx->N;
    }
  }
  return HE_OK;
}

static int q_dot(he_ctx_t* ctx, const double* x, const double* y, int slot) {
  tname(ctx, "dot_reduce");
  if (ctx->mixed)
    k_dot_f32<<<pw_grid(ctx), 256, 0, ctx->stream>>>((const float*)x, (const float*)y, ctx->N,
                                                      tail(ctx, slot), ctx->mm);
  else
    k_dot<<<pw_grid(ctx), 256, 0, ctx->stream>>>(x, y, ctx->N, tail(ctx, slot), ctx->mm);
  LAUNCHED();
  return HE_OK;
}

// energy (Dynamics_quantum_impurities/energy.f90:12-139).  sto2 of the reference lands in t4.
static int q_energy_launch(he_ctx_t* ctx) {
  const int n = ctx->nq;
  if (ctx->mixed) {
    OpEnergy<float2> op{};
    op.s8[0] = (const float*)ctx->den; op.s8[1] = (const float*)ctx->dencg;
    op.s8[2] = (const float*)ctx->delj4; op.s8[3] = (const float*)ctx->den;
    op.has_u = 0;
    op.aux1 = 0.5 * ctx->fn.cp4; op.aux2 = (1.0 / 3.0) * ctx->fn.cpp4;
    op.beta = ctx->fn.beta; op.den_m = ctx->fn.den_m; op.lsolid = ctx->fn.lsolid;
    TRY(run_stencil_red(ctx, ctx->g1, hi_plane(ctx->psi), op, S_EN));
    for (int k = 0; k < n; ++k) {
      OpGrad2T<float2> g{};
      TRY(run_stencil_red(ctx, ctx->g1, hi_plane(ctx->psix[k]), g, S_QEK + k));
    }
  } else {
    OpEnergy<double2> op{};
    op.s8[0] = ctx->den; op.s8[1] = ctx->dencg; op.s8[2] = ctx->delj4; op.s8[3] = ctx->den;
    op.has_u = 0;
    op.aux1 = 0.5 * ctx->fn.cp4; op.aux2 = (1.0 / 3.0) * ctx->fn.cpp4;
    op.beta = ctx->fn.beta; op.den_m = ctx->fn.den_m; op.lsolid = ctx->fn.lsolid;
    TRY(run_stencil_red(ctx, ctx->g1, (const double2*)ctx->psi, op, S_EN));
    for (int k = 0; k < n; ++k) {
      OpGrad2 g{};
      TRY(run_stencil_red(ctx, ctx->g1, (const double2*)ctx->psix[k], g, S_QEK + k));
    }
  }
  TRY(q_denx_spectra(ctx));
  QOut o{};
  o.out = ctx->t4;
  for (int k = 0; k < n; ++k) { o.src[o.nterm] = ctx->sx[k]; o.ker[o.nterm++] = ctx->uimpk[k]; }
  TRY(q_synth(ctx, &o, 1, nullptr));
  TRY(q_dot(ctx, ctx->t4, ctx->den, S_QHEX));
  int pair = 0;
  for (int k = 0; k < n; ++k)
    for (int m = k + 1; m < n; ++m, ++pair) {
      const double* kk = ctx->uimpkk[k + kMaxQImp * m];
      if (!kk) continue;
      QOut p{};
      p.out = ctx->t4;
      p.nterm = 1; p.src[0] = ctx->sx[k]; p.ker[0] = kk;
      TRY(q_synth(ctx, &p, 1, nullptr));
      TRY(q_dot(ctx, ctx->t4, ctx->denx[m], S_QII + pair));
    }
  if (ctx->otc) TRY(alfa_energy_sum(ctx));
  return HE_OK;
}
// The quantum energies from one member's reduction slots h (S_COUNT values).
static void q_energy_from(const he_ctx_t* ctx, const double* h, const double* ealphas,
                          he_energies_t* out) {
  const int n = ctx->nq;
  const double* s = h + S_EN;
  const double dxyz = ctx->dxyz;
  he_energies_t e{};
  e.esolid = ctx->fn.lsolid ? ctx->fn.C * s[3] * dxyz : 0.0;
  e.ekin4 = ctx->fn.h2o2m4 * s[0] * dxyz;
  e.elj4 = 0.5 * s[1] * dxyz;
  e.ecor4 = s[2] * dxyz;
  e.etot4 = e.ekin4 + e.elj4 + e.ecor4 + e.esolid;
  if (ealphas) {
    e.ealphas = *ealphas;
    e.etot4 = e.etot4 + e.ealphas;
  }
  for (int k = 0; k < n; ++k) e.ekinx = e.ekinx + ctx->h2o2mx[k] * h[S_QEK + k];
  e.ekinx = e.ekinx * dxyz;
  e.eHeX = h[S_QHEX] * dxyz;
  int pair = 0;
  for (int k = 0; k < n; ++k)
    for (int m = k + 1; m < n; ++m, ++pair)
      if (ctx->uimpkk[k + kMaxQImp * m]) e.eimpu_impu = e.eimpu_impu + h[S_QII + pair];
  e.eimpu_impu = e.eimpu_impu * dxyz;
  e.eimpu = e.ekinx + e.eHeX + e.eimpu_impu;
  e.etot = e.etot4 + e.eimpu;
  *out = e;
}
static int q_energy(he_ctx_t* ctx, he_energies_t* out) {
  TRY(q_energy_launch(ctx));
  TRY(read_sums(ctx));
  double ea = 0.0;
  if (ctx->otc) ea = alfa_energy(ctx);
  q_energy_from(ctx, ctx->hsum, ctx->otc ? &ea : nullptr, out);
  return HE_OK;
}

// ---- FT_V_spline (Dynamics_quantum_impurities/FT_V_spline.f90:14-276) --------------------------
// Host half: the cubic splines (mates.f:36-110, Maron's tridiagonal algorithm with prescribed end
// second derivatives; 1-based index helpers follow the reference's loops) and the small-q
// redefinition; the transform of the pieces, which is the O(N_p * N_FT_V_spline) part, is k_ftv.
namespace ftv {

constexpr double kRmax = 5000.0, kEps = 1.0e-8, kSmallQ = 1.0e-2, kDr = 0.05;

static double pair_value(const he_pairpot_t& v, double r) {
  if (r < v.rcut) return v.umax;
  if (v.kind == 0) return 0.0;
  const double e = 1.0 - std::exp(-v.a * (r - v.re));
  return v.D * (e * e - 1.0);
}

static void spline(const double* xv, const double* yv, double* av, double* bv, double* cv, double* dv,
                   double s1, double sn, int n) {
  auto X = [&](int i) { return xv[i - 1]; };
  auto Y = [&](int i) { return yv[i - 1]; };
  auto A = [&](int i) -> double& { return av[i - 1]; };
  auto B = [&](int i) -> double& { return bv[i - 1]; };
  auto C = [&](int i) -> double& { return cv[i - 1]; };
  auto D = [&](int i) -> double& { return dv[i - 1]; };
  const int n1 = n - 1, n2 = n - 2;
  for (int i = 1; i <= n1; ++i) {
    A(i) = X(i + 1) - X(i);
    D(i) = (Y(i + 1) - Y(i)) / A(i);
  }
  for (int i = 1; i <= n2; ++i) {
    B(i) = 2.0 * (A(i) + A(i + 1));
    const int k = n1 - i + 1;
    D(k) = 6.0 * (D(k) - D(k - 1));
  }
  D(2) = D(2) - A(1) * s1;
  D(n1) = D(n1) - A(n1) * sn;
  for (int i = 2; i <= n2; ++i) {
    const double r = A(i) / B(i - 1);
    B(i) = B(i) - r * A(i);
    D(i + 1) = D(i + 1) - r * D(i);
  }
  D(n1) = D(n1) / B(n2);
  for (int i = 2; i <= n2; ++i) {
    const int k = n1 - i + 1;
    D(k) = (D(k) - A(k) * D(k + 1)) / B(k - 1);
  }
  D(n) = sn;
  double si1 = s1;
  for (int i = 1; i <= n1; ++i) {
    const double si = si1;
    si1 = D(i + 1);
    const double h = A(i), hi = 1.0 / h;
    const double x0 = X(i), x1 = X(i + 1);
    A(i) = (hi / 6.0) * (si * (x1 * x1 * x1) - si1 * (x0 * x0 * x0)) + hi * (Y(i) * x1 - Y(i + 1) * x0) +
           (h / 6.0) * (si1 * x0 - si * x1);
    B(i) = (hi / 2.0) * (si1 * (x0 * x0) - si * (x1 * x1)) + hi * (Y(i + 1) - Y(i)) + (h / 6.0) * (si - si1);
    C(i) = (hi / 2.0) * (si * x1 - si1 * x0);
    D(i) = (hi / 6.0) * (si1 - si);
  }
}

// RAII device buffer for the set-up path.
struct DBuf {
  double* p = nullptr;
  ~DBuf() { if (p) cudaFree(p); }
  cudaError_t alloc(size_t n) { return cudaMalloc(&p, n * sizeof(double)); }
};

// Builds the momentum table P_p, Vpp and its spline (A..D, np entries) on `stream`.
static cudaError_t table(const he_pairpot_t& v, double pmax, double hp, int n, int parabolic,
                         cudaStream_t st, std::vector<double>& P, std::vector<double>& V,
                         std::vector<double>& A, std::vector<double>& B, std::vector<double>& C,
                         std::vector<double>& D, std::string* why) {
  if (n < 4) { *why = "n_spline must be at least 4"; return cudaErrorInvalidValue; }
  const double X1 = v.rcut + kEps, XN = kRmax;
  const double S1 = (pair_value(v, X1) - 2.0 * pair_value(v, X1 + kDr) + pair_value(v, X1 + kDr + kDr)) / (kDr * kDr);
  const double Sn = (pair_value(v, XN - kDr) - 2.0 * pair_value(v, XN) + pair_value(v, XN + kDr)) / (kDr * kDr);
  const double h = (XN - X1) / (n - 1);
  std::vector<double> x(n), y(n), a(n), b(n), c(n), d(n);
  for (int i = 1; i <= n; ++i) {
    x[i - 1] = (i - 1) * h + X1;
    y[i - 1] = pair_value(v, x[i - 1]);
  }
  spline(x.data(), y.data(), a.data(), b.data(), c.data(), d.data(), S1, Sn, n);
  const int np = (int)(pmax / hp + 1.5);
  if (np < 8) { *why = "momentum table too short"; return cudaErrorInvalidValue; }
  FtvArgs F{};
  F.n = n; F.hp = hp; F.r0 = v.rcut; F.f0 = v.umax; F.parabolic = parabolic;
  if (parabolic) {
    const double r0 = v.rcut, r1 = r0 + kDr, f0 = v.umax, f1 = pair_value(v, r1);
    F.aa = (f0 - f1) / (r0 * r0 - r1 * r1);
    F.cc = (r0 * r0 * f1 - r1 * r1 * f0) / (r0 * r0 - r1 * r1);
    if (F.aa > 0.0) { *why = "parabolic core fit is not inverted (FT_V_spline.f90:142-145)"; return cudaErrorInvalidValue; }
  }
  DBuf dx, da, db, dc, dd, dv;
  cudaError_t e;
  if ((e = dx.alloc(n)) || (e = da.alloc(n)) || (e = db.alloc(n)) || (e = dc.alloc(n)) ||
      (e = dd.alloc(n)) || (e = dv.alloc(np))) { *why = "device allocation"; return e; }
  const std::vector<double>* hs[5] = {&x, &a, &b, &c, &d};
  double* ds[5] = {dx.p, da.p, db.p, dc.p, dd.p};
  for (int k = 0; k < 5; ++k)
    if ((e = cudaMemcpyAsync(ds[k], hs[k]->data(), n * sizeof(double), cudaMemcpyHostToDevice, st))) {
      *why = "upload"; return e;
    }
  F.x = dx.p; F.a = da.p; F.b = db.p; F.c = dc.p; F.d = dd.p; F.vpp = dv.p;
  k_ftv<<<np, 256, 0, st>>>(F);
  if ((e = cudaGetLastError())) { *why = "k_ftv launch"; return e; }
  V.resize(np);
  if ((e = cudaMemcpyAsync(V.data(), dv.p, np * sizeof(double), cudaMemcpyDeviceToHost, st)) ||
      (e = cudaStreamSynchronize(st))) { *why = "k_ftv"; return e; }
  P.resize(np);
  for (int i = 0; i < np; ++i) P[i] = i * hp;
  // small-q redefinition (FT_V_spline.f90:229-258)
  double qx[4] = {0.0, 0, 0, 0}, qy[4] = {V[0], 0, 0, 0};
  int iaux = 1;
  for (int i = 2; i <= np; ++i) {
    if (P[i - 1] > kSmallQ) { ++iaux; qx[iaux - 1] = P[i - 1]; qy[iaux - 1] = V[i - 1]; }
    if (iaux == 4) break;
  }
  double qa[4], qb[4], qc[4], qd[4];
  spline(qx, qy, qa, qb, qc, qd, 0.0, 0.0, 4);
  for (int i = 2; i <= np; ++i) {
    const double p = P[i - 1];
    if (p <= kSmallQ) V[i - 1] = qa[0] + p * (qb[0] + p * (qc[0] + p * qd[0]));
    else break;
  }
  A.resize(np); B.resize(np); C.resize(np); D.resize(np);
  spline(P.data(), V.data(), A.data(), B.data(), C.data(), D.data(), 0.0, 0.0, np);
  return cudaSuccess;
}

}  // namespace ftv

// potenimpini (Dynamics_quantum_impurities/potenimpini.f90:116-163): uimp_k of one pair potential
// over this context's half spectrum; qmax = max(100, |pmax|), Hq = qmax/(max(10001,Nq)-1).
static int q_kernel(he_ctx_t* ctx, const he_pairpot_t& v, int nspline, int nq, int parabolic, double* dst) {
  const double pmx = 1.0 / (2.0 * ctx->hx), pmy = 1.0 / (2.0 * ctx->hy), pmz = 1.0 / (2.0 * ctx->hz);
  const double qmax = std::max(100.0, std::sqrt(pmx * pmx + pmy * pmy + pmz * pmz));
  const long Nq = std::max(10001L, (long)nq);
  const double hq = qmax / (double)(Nq - 1);
  std::vector<double> P, V, A, B, C, D;
  std::string why;
  cudaError_t e = ftv::table(v, qmax, hq, nspline, parabolic, ctx->stream, P, V, A, B, C, D, &why);
  if (e != cudaSuccess)
    return fail(ctx, e == cudaErrorInvalidValue ? HE_ERR_ARG : HE_ERR_CUDA, "FT_V_spline: %s (%s)",
                why.c_str(), cudaGetErrorString(e));
  const int np = (int)P.size();
  ftv::DBuf dP, dA, dB, dC, dD;
  CK(dP.alloc(np)); CK(dA.alloc(np)); CK(dB.alloc(np)); CK(dC.alloc(np)); CK(dD.alloc(np));
  CK(cudaMemcpyAsync(dP.p, P.data(), np * 8, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(dA.p, A.data(), np * 8, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(dB.p, B.data(), np * 8, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(dC.p, C.data(), np * 8, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(dD.p, D.data(), np * 8, cudaMemcpyHostToDevice, ctx->stream));
  UimpkArgs u{};
  u.P = dP.p; u.a = dA.p; u.b = dB.p; u.c = dC.p; u.d = dD.p; u.np = np;
  u.nx = ctx->nx; u.ny = ctx->ny; u.nz = ctx->nz; u.nxh = ctx->nxh;
  u.hx = ctx->hx; u.hy = ctx->hy; u.hz = ctx->hz;
  u.out = dst;
  tname(ctx, "uimp_k_spline");
  k_uimpk<<<kPwBlocks, 256, 0, ctx->stream>>>(u);
  LAUNCHED();
  TRY(sync_all(ctx));
  return HE_OK;
}

static bool qfield(int f) { return f >= HE_F_PSIX && f <= HE_F_UIMPKK; }

// Transfers of the per-impurity arrays (one device buffer per impurity and slot).
static int q_xfer(he_ctx_t* ctx, int field, void* host, size_t bytes, bool up) {
  if (ctx->mode != HE_MODE_QUANTUM || ctx->nq == 0)
    return fail(ctx, HE_ERR_STATE, "quantum-impurity fields need HE_MODE_QUANTUM and he_set_quantum_impurities");
  const int n = ctx->nq;
  const size_t N = ctx->N, Nk = ctx->Nk;
  std::vector<std::pair<void*, size_t>> parts;
  switch (field) {
    case HE_F_PSIX: for (int i = 0; i < n; ++i) parts.push_back({ctx->psix[i], 16 * N}); break;
    case HE_F_PCX: for (int i = 0; i < n; ++i) parts.push_back({ctx->pcx[i], 16 * N}); break;
    case HE_F_QX: for (int i = 0; i < n; ++i) parts.push_back({ctx->qx[i], 16 * N}); break;
    case HE_F_UPOTX: for (int i = 0; i < n; ++i) parts.push_back({ctx->upotx[i], 8 * N}); break;
    case HE_F_POTX4: parts.push_back({ctx->potx4, 8 * N}); break;
    case HE_F_PSIXOLD:
      for (int i = 0; i < n; ++i) for (int s = 0; s < 3; ++s) parts.push_back({ctx->psixold[i][s], 16 * N});
      break;
    case HE_F_HPSIXOLD:
      for (int i = 0; i < n; ++i) for (int s = 0; s < 2; ++s) parts.push_back({ctx->hpsixold[i][s], 16 * N});
      break;
    case HE_F_UIMPK: for (int i = 0; i < n; ++i) parts.push_back({ctx->uimpk[i], 8 * Nk}); break;
    case HE_F_UIMPKK:  // pairs without a kernel ('null', i == j) read as zero and are not stored
      for (int j = 0; j < n; ++j) for (int i = 0; i < n; ++i) parts.push_back({ctx->uimpkk[i + kMaxQImp * j], 8 * Nk});
      break;
    case HE_F_DENX: {
      if (up) return fail(ctx, HE_ERR_ARG, "denx is derived from psix (download only)");
      if (bytes != 8 * N) return fail(ctx, HE_ERR_ARG, "denx: expected %zu bytes", 8 * N);
      std::vector<double> acc(N, 0.0), t(N);
      std::vector<float> tf(ctx->mixed ? N : 0);
      for (int i = 0; i < n; ++i) {
        if (ctx->mixed) {
          CK(cudaMemcpyAsync(tf.data(), ctx->denx[i], 4 * N, cudaMemcpyDeviceToHost, ctx->stream));
          TRY(sync_all(ctx));
          for (size_t k = 0; k < N; ++k) t[k] = tf[k];
        } else {
          CK(cudaMemcpyAsync(t.data(), ctx->denx[i], 8 * N, cudaMemcpyDeviceToHost, ctx->stream));
          TRY(sync_all(ctx));
        }
        for (size_t k = 0; k < N; ++k) acc[k] = acc[k] + t[k];
      }
      std::memcpy(host, acc.data(), 8 * N);
      return HE_OK;
    }
    default: return fail(ctx, HE_ERR_ARG, "unknown field %d", field);
  }
  size_t total = 0;
  for (auto& p : parts) total += p.second;
  if (bytes != total) return fail(ctx, HE_ERR_ARG, "field %d: expected %zu bytes, got %zu", field, total, bytes);
  // device format of the field (binary64 unless the mixed path holds it narrower)
  FieldFmt fmt = FMT_F64;
  if (ctx->mixed) {
    if (field == HE_F_PSIX || field == HE_F_PSIXOLD) fmt = FMT_HL;
    else if (field == HE_F_PCX || field == HE_F_QX || field == HE_F_HPSIXOLD) fmt = FMT_C32;
    else if (field == HE_F_UPOTX || field == HE_F_POTX4) fmt = FMT_R32;
  }
  char* h = (char*)host;
  for (auto& p : parts) {
    if (fmt != FMT_F64 && p.first) {
      std::vector<unsigned char> dev;
      if (up) {
        to_device_fmt(fmt, h, p.second, dev);
        CK(cudaMemcpyAsync(p.first, dev.data(), dev.size(), cudaMemcpyHostToDevice, ctx->stream));
        TRY(sync_all(ctx));
      } else {
        dev.resize(device_fmt_bytes(fmt, p.second));
        CK(cudaMemcpyAsync(dev.data(), p.first, dev.size(), cudaMemcpyDeviceToHost, ctx->stream));
        TRY(sync_all(ctx));
        from_device_fmt(fmt, dev, h, p.second);
      }
    } else if (up) {
      if (p.first) CK(cudaMemcpyAsync(p.first, h, p.second, cudaMemcpyHostToDevice, ctx->stream));
    } else {
      if (p.first) CK(cudaMemcpyAsync(h, p.first, p.second, cudaMemcpyDeviceToHost, ctx->stream));
      else std::memset(h, 0, p.second);
    }
    h += p.second;
  }
  TRY(sync_all(ctx));
  if (up && (field == HE_F_UIMPK || field == HE_F_UIMPKK)) TRY(qkernels_to_f32(ctx));
  if (up && field == HE_F_PSIX)
    for (int i = 0; i < n; ++i) TRY(q_cnorm2(ctx, i));
  if (up && (field == HE_F_PSIX || field == HE_F_UIMPK || field == HE_F_UIMPKK)) ctx->cglj_pending = false;
  return HE_OK;
}

__global__ void __launch_bounds__(256) k_to_f32(const double* __restrict__ a, float* __restrict__ b,
                                                long n, double scale) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    b[i] = (float)(a[i] * scale);
}
__global__ void __launch_bounds__(256) k_to_f64(const float* __restrict__ a, double* __restrict__ b, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    b[i] = (double)a[i];
}
// Refreshes the binary32 kernel copies of the mixed chain after the binary64 kernels changed;
// wcgk's copy carries the power-of-two scale cg_scale (see he_ctx).
static int kernels_to_f32(he_ctx_t* ctx) {
  stat_graphs_clear(ctx);
  if (!ctx->mixed) return HE_OK;
  double k0[2];
  CK(cudaMemcpyAsync(&k0[0], ctx->fvlj4, 8, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaMemcpyAsync(&k0[1], ctx->wcgk, 8, cudaMemcpyDeviceToHost, ctx->stream));
  TRY(sync_all(ctx));
  ctx->cg_scale = 1.0;
  if (std::isfinite(k0[0]) && std::isfinite(k0[1]) && k0[0] != 0.0 && k0[1] != 0.0) {
    const int e = (int)std::lround(std::log2(std::fabs(k0[0] / k0[1])));
    ctx->cg_scale = std::ldexp(1.0, std::max(-30, std::min(30, e)));
  }
  tname(ctx, "kernels_to_f32");
  k_to_f32<<<kPwBlocks, 256, 0, ctx->stream>>>(ctx->fvlj4, ctx->fvlj4f, ctx->Nk, 1.0);
  LAUNCHED();
  tname(ctx, "kernels_to_f32");
  k_to_f32<<<kPwBlocks, 256, 0, ctx->stream>>>(ctx->wcgk, ctx->wcgkf, ctx->Nk, ctx->cg_scale);
  LAUNCHED();
  return HE_OK;
}

// Binary32 copies of the impurity kernels uimp_k_i and uimp_k_k(i,j) for the mixed path
// (allocated on first use; refreshed whenever the binary64 tables change).
static int qkernels_to_f32(he_ctx_t* ctx) {
  if (!ctx->mixed) return HE_OK;
  for (int i = 0; i < kMaxQImp; ++i) {
    if (!ctx->uimpk[i]) continue;
    if (!ctx->uimpkf[i]) TRY(dalloc_t(ctx, &ctx->uimpkf[i], ctx->Nk));
    tname(ctx, "kernels_to_f32");
    k_to_f32<<<kPwBlocks, 256, 0, ctx->stream>>>(ctx->uimpk[i], ctx->uimpkf[i], ctx->Nk, 1.0);
    LAUNCHED();
  }
  for (int j = 0; j < kMaxQImp * kMaxQImp; ++j) {
    if (!ctx->uimpkk[j]) continue;
    if (!ctx->uimpkkf[j]) TRY(dalloc_t(ctx, &ctx->uimpkkf[j], ctx->Nk));
    tname(ctx, "kernels_to_f32");
    k_to_f32<<<kPwBlocks, 256, 0, ctx->stream>>>(ctx->uimpkk[j], ctx->uimpkkf[j], ctx->Nk, 1.0);
    LAUNCHED();
  }
  return HE_OK;
}

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
  if (mode != HE_MODE_DYNAMICS && mode != HE_MODE_STATICS && mode != HE_MODE_QUANTUM)
    bad(HE_ERR_ARG, "unknown mode");
  else if (precision != HE_PREC_F64 && precision != HE_PREC_MIXED) bad(HE_ERR_ARG, "unknown precision");
  else if (grid->npd != 13) bad(HE_ERR_ARG, "npd must be 13");
  else if (grid->icon != 13 && grid->icon != 8 && grid->icon != 18 &&
           grid->icon != 24)
    bad(HE_ERR_ARG, "icon must be 13, 8, 18 or 24");
  else if (!tstgrid_ok(grid->nx) || !tstgrid_ok(grid->ny) || !tstgrid_ok(grid->nz))
    bad(HE_ERR_ARG, "grid size is not an admissible tstgrid value");
  else if (grid->ny < 2)
    bad(HE_ERR_ARG, "ny must be at least 2");
  else if (!factor_ok(grid->nx) || !factor_ok(grid->ny) || !factor_ok(grid->nz))
    bad(HE_ERR_ARG, "grid size must be 2^a 3^b 5^c");
  else if (grid->xmax == 0.0 || grid->ymax == 0.0 || grid->zmax == 0.0)
    bad(HE_ERR_ARG, "xmax, ymax, zmax must be non-zero");
  if (st == HE_OK) {
    if (std::strncmp(fun->core4, "OP", 2) != 0 && std::strncmp(fun->core4, "OT ", 3) != 0 &&
        std::strncmp(fun->core4, "OTC", 3) != 0)
      bad(HE_ERR_ARG, "core4 must be 'OT ', 'OP ' or 'OTC'");
    else if (std::strncmp(fun->core4, "OTC", 3) == 0 && !(fun->den0s != 0.0))
      bad(HE_ERR_ARG, "core4='OTC' needs den0s != 0");
  }
  if (st != HE_OK) {
    *out = ctx;
    return st;
  }
  ctx->mode = mode;
  ctx->prec = precision;
  ctx->mixed = precision == HE_PREC_MIXED;
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
  ctx->otc = std::strncmp(fun->core4, "OTC", 3) == 0;
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
  ctx->pdl = (long)ctx->nx * ctx->ny * ctx->nz <= 160L * 160 * 160;
  if (mode == HE_MODE_DYNAMICS) {
    e = cudaStreamCreateWithFlags(&ctx->aux, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ctx->ev_fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ctx->ev_join, cudaEventDisableTiming);
    if (e != cudaSuccess)
      return fail(ctx, HE_ERR_CUDA, "side stream creation failed: %s", cudaGetErrorString(e));
  }

  // FFT plans and shared-memory budgets
  TRY(make_plan(ctx, ctx->nx, &ctx->plx));
  TRY(make_plan(ctx, ctx->ny, &ctx->ply));
  TRY(make_plan(ctx, ctx->nz, &ctx->plz));
  const int nmax = std::max(ctx->nx, std::max(ctx->ny, ctx->nz));
  ctx->tkx = tile_rows(nmax);
  ctx->x_rb = tile_rows(ctx->nx);
  // an even tile that divides the row count, else (odd ny*nz) the default with a partial last tile
  if (((long)ctx->ny * ctx->nz) % 2 == 0)
    while (ctx->x_rb > 2 && ((long)ctx->ny * ctx->nz) % ctx->x_rb) ctx->x_rb -= 2;
  ctx->smem_x = fft_smem(ctx->plx, tile_rows(ctx->nx), 2);
  ctx->smem_y = fft_smem(ctx->ply, ctx->tkx, 2);
  ctx->smem_z = fft_smem(ctx->plz, ctx->tkx, 3);
  int maxsm = 0, dev = 0;
  CK(cudaGetDevice(&dev));
  CK(cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  ctx->maxsm = maxsm;
  if ((int)ctx->smem_x > maxsm || (int)ctx->smem_y > maxsm || (int)ctx->smem_z > maxsm)
    return fail(ctx, HE_ERR_ARG, "grid too large for the shared-memory FFT passes");

  const size_t N = ctx->N, Nk = ctx->Nk;
  TRY(dalloc_t(ctx, &ctx->fden, Nk));
  TRY(dalloc_t(ctx, &ctx->wA, Nk));
  TRY(dalloc_t(ctx, &ctx->wB, Nk));
  TRY(dalloc_t(ctx, &ctx->fvlj4, Nk));
  TRY(dalloc_t(ctx, &ctx->wcgk, Nk));
  if (ctx->mixed) {
    TRY(dalloc_t(ctx, &ctx->fvlj4f, Nk));
    TRY(dalloc_t(ctx, &ctx->wcgkf, Nk));
  }
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
  if (mode == HE_MODE_DYNAMICS) TRY(dalloc_t(ctx, &ctx->uimp, N));
  if (mode == HE_MODE_QUANTUM) {
    TRY(dalloc_t(ctx, &ctx->potx4, N));
    TRY(dalloc_t(ctx, &ctx->t4, N));
    TRY(dalloc(ctx, &ctx->xscratch, wf));
  }
  if (mode == HE_MODE_QUANTUM || ctx->otc) {
    TRY(dalloc_t(ctx, &ctx->wC, Nk));
    TRY(dalloc_t(ctx, &ctx->wD, Nk));
  }
  if (ctx->otc && ctx->mixed) {
    TRY(dalloc_t(ctx, &ctx->den64, N));
    TRY(dalloc_t(ctx, &ctx->ualphas_f, N));
  }
  if (ctx->otc) {
    TRY(dalloc_t(ctx, &ctx->kalfs, Nk));
    for (double** a : {&ctx->denalf, &ctx->falfs, &ctx->intxalf, &ctx->intyalf, &ctx->intzalf,
                       &ctx->ualphas, &ctx->ua_raw, &ctx->as1, &ctx->as2, &ctx->as3, &ctx->as4,
                       &ctx->as5, &ctx->dxden, &ctx->dyden, &ctx->dzden})
      TRY(dalloc_t(ctx, a, N));
  }
  if (mode != HE_MODE_STATICS) {
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
  if (mode == HE_MODE_DYNAMICS) CK(cudaMallocHost(&ctx->himp, sizeof(ImpDev)));
  TRY(autotune_tiles(ctx));
  TRY(sync_all(ctx));
  return HE_OK;
}

void he_ctx_destroy(he_ctx_t* ctx) {
  if (!ctx) return;
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  if (ctx->aux) cudaStreamSynchronize(ctx->aux);
  stat_graphs_clear(ctx);
  for (void* p : ctx->allocs) cudaFree(p);
  if (ctx->hsum) cudaFreeHost(ctx->hsum);
  if (ctx->himp) cudaFreeHost(ctx->himp);
  for (cudaEvent_t e : ctx->evpool) cudaEventDestroy(e);
  if (ctx->own) cudaStreamDestroy(ctx->own);
  if (ctx->aux) cudaStreamDestroy(ctx->aux);
  if (ctx->ev_fork) cudaEventDestroy(ctx->ev_fork);
  if (ctx->ev_join) cudaEventDestroy(ctx->ev_join);
  delete ctx;
}

const char* he_last_error(const he_ctx_t* ctx) { return ctx ? ctx->err.c_str() : "null context"; }
long long he_launch_count(const he_ctx_t* ctx) { return ctx ? ctx->launches : 0; }
size_t he_device_bytes(const he_ctx_t* ctx) { return ctx ? ctx->bytes : 0; }

int he_set_stream(he_ctx_t* ctx, void* stream) {
  if (!ctx) return HE_ERR_ARG;
  TRY(sync_all(ctx));
  ctx->stream = stream ? (cudaStream_t)stream : ctx->own;
  return HE_OK;
}

int he_synchronize(he_ctx_t* ctx) {
  if (!ctx) return HE_ERR_ARG;
  TRY(sync_all(ctx));
  return HE_OK;
}

int he_join(he_ctx_t* ctx) {
  if (!ctx) return HE_ERR_ARG;
  return join_aux(ctx);
}

int he_set_kernels(he_ctx_t* ctx, const double* fvlj4, const double* wcgk, const double* kalfs) {
  if (!ctx || !fvlj4 || !wcgk) return fail(ctx, HE_ERR_ARG, "null kernel array");
  if (ctx->otc && !kalfs) return fail(ctx, HE_ERR_ARG, "core4='OTC' needs kalfs");
  if (ctx->otc) CK(cudaMemcpyAsync(ctx->kalfs, kalfs, 8 * ctx->Nk, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(ctx->fvlj4, fvlj4, 8 * ctx->Nk, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(ctx->wcgk, wcgk, 8 * ctx->Nk, cudaMemcpyHostToDevice, ctx->stream));
  TRY(kernels_to_f32(ctx));
  TRY(sync_all(ctx));
  ctx->kernels_ok = true;
  return HE_OK;
}

int he_compute_kernels(he_ctx_t* ctx) {
  if (!ctx) return HE_ERR_ARG;
  KernArgs a{};
  a.nx = ctx->nx; a.ny = ctx->ny; a.nz = ctx->nz; a.nxh = ctx->nxh;
  a.hx = ctx->hx; a.hy = ctx->hy; a.hz = ctx->hz;
  a.op_core = ctx->op_core; a.otc = ctx->otc;
  a.eps = ctx->fn.eps4; a.sigma = ctx->fn.sigma4; a.hc = ctx->fn.h4; a.l = ctx->fn.l;
  a.fvlj4 = ctx->fvlj4; a.wcgk = ctx->wcgk; a.kalfs = ctx->kalfs;
  tname(ctx, "kspace_kernels");
  k_kernels<<<kPwBlocks, 256, 0, ctx->stream>>>(a);
  LAUNCHED();
  TRY(kernels_to_f32(ctx));
  TRY(sync_all(ctx));
  ctx->kernels_ok = true;
  return HE_OK;
}

int he_set_absorber(he_ctx_t* ctx, const he_absorber_t* ab) {
  if (!ctx || !ab) return fail(ctx, HE_ERR_ARG, "null absorber");
  if (ctx->mode == HE_MODE_STATICS) return fail(ctx, HE_ERR_STATE, "absorber is a dynamics setting");
  auto tab = [&](int n, double xm, double h, double mean, double surf, double* dst) -> int {
    std::vector<double> t(n);
    for (int i = 0; i < n; ++i) t[i] = std::tanh((std::fabs(-xm + h * i) - mean) / surf);
    CK(cudaMemcpyAsync(dst, t.data(), 8 * n, cudaMemcpyHostToDevice, ctx->stream));
    TRY(sync_all(ctx));
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
    TRY(sync_all(ctx));
  }
  ctx->npot = im->npot;
  ctx->delinter = im->delinter;
  ctx->rmaxinterpol = im->rmaxinterpol;
  ctx->force_fresh = false;
  return HE_OK;
}

int he_upload(he_ctx_t* ctx, int field, const void* host, size_t bytes) {
  if (!ctx || !host) return fail(ctx, HE_ERR_ARG, "null argument");
  TRY(join_aux(ctx));
  if (qfield(field)) return q_xfer(ctx, field, const_cast<void*>(host), bytes, true);
  if (field >= HE_F_RIMP && field <= HE_F_QV) {
    if (ctx->mode != HE_MODE_DYNAMICS) return fail(ctx, HE_ERR_STATE, "no impurities in statics");
    // only the member's bytes go to the device struct (no read-back, no wait): the driver uploads
    // aimp every iteration
    ImpDev h{};
    h.n = ctx->n_imp;
    size_t cnt = 0;
    double* m = imp_member(&h, field, &cnt);
    if (!m || bytes != cnt * 8) return fail(ctx, HE_ERR_ARG, "field %d: expected %zu bytes", field, cnt * 8);
    const size_t off = (size_t)((char*)m - (char*)&h);
    CK(cudaMemcpyAsync((char*)ctx->imp + off, host, bytes, cudaMemcpyHostToDevice, ctx->stream));
    ctx->force_fresh = false;
    return HE_OK;
  }
  if (field == HE_F_RING) return fail(ctx, HE_ERR_ARG, "ring indices are read-only");
  FieldRef r;
  TRY(field_ref(ctx, field, &r));
  if (bytes != r.bytes) return fail(ctx, HE_ERR_ARG, "field %d: expected %zu bytes, got %zu", field, r.bytes, bytes);
  const FieldFmt fmt = field_fmt(ctx, field);
  if (fmt == FMT_F64) {
    CK(cudaMemcpyAsync(r.ptr, host, bytes, cudaMemcpyHostToDevice, ctx->stream));
    TRY(sync_all(ctx));
  } else {
    std::vector<unsigned char> dev;
    to_device_fmt(fmt, host, bytes, dev);
    CK(cudaMemcpyAsync(r.ptr, dev.data(), dev.size(), cudaMemcpyHostToDevice, ctx->stream));
    TRY(sync_all(ctx));
  }
  if (field == HE_F_FVLJ4 || field == HE_F_WCGK) {
    ctx->kernels_ok = true;
    TRY(kernels_to_f32(ctx));
    TRY(sync_all(ctx));
  }

  if (field == HE_F_DEN) ctx->force_fresh = false;
  if (field == HE_F_DEN || field == HE_F_FDEN || field == HE_F_FVLJ4 || field == HE_F_WCGK)
    ctx->cglj_pending = false;
  return HE_OK;
}

// ---- groups ------------------------------------------------------------------------------------
// Member m's counterpart of one of the leader's device pointers (the host copy of the map).
static void* member_ptr(const he_ctx_t* L, const void* p, int m) {
  if (m == 0 || L->nmem <= 1 || !p) return const_cast<void*>(p);
  const int nb = (int)(L->mmhost.size() / (2 + L->nmem));
  const unsigned long long a = (unsigned long long)p;
  const unsigned long long* t = L->mmhost.data();
  int lo = 0, hi = nb - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) / 2;
    if (t[mid] <= a) lo = mid;
    else hi = mid - 1;
  }
  if (a < t[lo] || a >= t[lo] + t[nb + lo]) return const_cast<void*>(p);
  return (void*)(t[2 * nb + (size_t)m * nb + lo] + (a - t[lo]));
}

int he_ctx_group(he_ctx_t* const* ctxs, int n) {
  if (!ctxs || n < 1 || !ctxs[0]) return HE_ERR_ARG;
  he_ctx_t* L = ctxs[0];
  if (L->nmem != 1) return fail(L, HE_ERR_STATE, "the context already leads a group");
  if (n == 1) return HE_OK;
  if (L->otc || !((L->mode == HE_MODE_STATICS && !L->mixed) || L->mode == HE_MODE_QUANTUM))
    return fail(L, HE_ERR_ARG, "groups run the binary64 statics mode or the quantum-impurity mode "
                               "(either precision) with the OT or OP core");
  for (int m = 0; m < n; ++m) {
    he_ctx_t* c = ctxs[m];
    if (!c) return fail(L, HE_ERR_ARG, "null member %d", m);
    for (int j = 0; j < m; ++j)
      if (ctxs[j] == c) return fail(L, HE_ERR_ARG, "member %d repeats member %d", m, j);
    if (c->nmem != 1 || c->mode != L->mode || c->prec != L->prec || c->otc != L->otc ||
        c->nx != L->nx || c->ny != L->ny || c->nz != L->nz || c->xmax != L->xmax ||
        c->ymax != L->ymax || c->zmax != L->zmax || c->icon != L->icon || c->nq != L->nq ||
        c->cglj_pending != L->cglj_pending)
      return fail(L, HE_ERR_ARG, "member %d differs from the leader (mode, precision, grid or core)", m);
    if (!c->kernels_ok) return fail(L, HE_ERR_STATE, "member %d has no k-space kernels", m);
    if (c->xyfuse) return fail(L, HE_ERR_STATE, "member %d evaluates its field with the fused x-y passes, which run no groups", m);
    for (int i = 0; i < L->nq; ++i)
      if (c->h2o2mx[i] != L->h2o2mx[i]) return fail(L, HE_ERR_ARG, "member %d's impurity masses differ", m);
    // derden's gradients are allocated on first use; every member holds them before pairing
    if (L->mode == HE_MODE_STATICS && !c->dxden) {
      TRY(dalloc_t(c, &c->dxden, c->N));
      TRY(dalloc_t(c, &c->dyden, c->N));
      TRY(dalloc_t(c, &c->dzden, c->N));
    }
    TRY(join_aux(c));
    TRY(sync_all(c));
  }
  const size_t nb = L->allocs.size();
  for (int m = 1; m < n; ++m) {
    const he_ctx_t* c = ctxs[m];
    if (c->allocs.size() != nb || c->alloc_bytes != L->alloc_bytes)
      return fail(L, HE_ERR_STATE, "member %d does not hold the leader's set of buffers", m);
  }
  std::vector<size_t> order(nb);
  for (size_t i = 0; i < nb; ++i) order[i] = i;
  std::sort(order.begin(), order.end(), [&](size_t a, size_t b) {
    return (unsigned long long)L->allocs[a] < (unsigned long long)L->allocs[b];
  });
  std::vector<unsigned long long> t((2 + (size_t)n) * nb);
  for (size_t k = 0; k < nb; ++k) {
    const size_t i = order[k];
    t[k] = (unsigned long long)L->allocs[i];
    t[nb + k] = L->alloc_bytes[i];
    for (int m = 0; m < n; ++m) t[2 * nb + (size_t)m * nb + k] = (unsigned long long)ctxs[m]->allocs[i];
  }
  // the members' relabelled buffers (psi, psiold, hpsiold, scratch) must pair with the leader's
  auto index_of = [&](const he_ctx_t* c, const void* p) -> long {
    for (size_t i = 0; i < nb; ++i)
      if (c->allocs[i] == p) return (long)i;
    return -1;
  };
  auto ring = [](const he_ctx_t* c) {
    std::vector<const void*> v = {c->psi, c->scratch, c->psiold[0], c->psiold[1], c->psiold[2],
                                  c->hpsiold[0], c->hpsiold[1], c->xscratch};
    for (int i = 0; i < c->nq; ++i) {
      v.push_back(c->psix[i]);
      for (int k = 0; k < 3; ++k) v.push_back(c->psixold[i][k]);
      for (int k = 0; k < 2; ++k) v.push_back(c->hpsixold[i][k]);
    }
    return v;
  };
  const std::vector<const void*> lr = ring(L);
  for (int m = 1; m < n; ++m) {
    const he_ctx_t* c = ctxs[m];
    const std::vector<const void*> cr = ring(c);
    bool same = std::equal(c->ioldp, c->ioldp + 3, L->ioldp) && std::equal(c->ioldh, c->ioldh + 2, L->ioldh);
    for (size_t k = 0; k < lr.size() && same; ++k) same = index_of(L, lr[k]) == index_of(c, cr[k]);
    if (!same)
      return fail(L, HE_ERR_STATE, "member %d's ring buffers are relabelled differently from the leader's", m);
  }
  unsigned long long* dt = nullptr;
  TRY(dalloc_t(L, &dt, t.size()));
  {
    const cudaError_t e = cudaMemcpyAsync(dt, t.data(), t.size() * sizeof(unsigned long long),
                                          cudaMemcpyHostToDevice, L->stream);
    if (e != cudaSuccess) return fail(L, HE_ERR_CUDA, "map table upload failed: %s", cudaGetErrorString(e));
  }
  TRY(sync_all(L));
  L->mmhost = t;
  L->mm.tab = dt;
  L->mm.nbuf = (int)nb;
  L->mm.nmem = n;
  L->nmem = n;
  stat_graphs_clear(L);  // graphs recorded before launched the leader alone
  return HE_OK;
}

int he_group_size(const he_ctx_t* ctx) { return ctx ? ctx->nmem : 0; }

static int member_xfer(he_ctx_t* ctx, int member, int field, void* host, size_t bytes, bool up) {
  if (!ctx || !host) return fail(ctx, HE_ERR_ARG, "null argument");
  if (member < 0 || member >= ctx->nmem) return fail(ctx, HE_ERR_ARG, "member %d of %d", member, ctx->nmem);
  if (member == 0) return up ? he_upload(ctx, field, host, bytes) : he_download(ctx, field, host, bytes);
  if (field == HE_F_RING || qfield(field) || (field >= HE_F_RIMP && field <= HE_F_QV))
    return fail(ctx, HE_ERR_ARG, "field %d has no per-member copy in a statics group", field);
  TRY(join_aux(ctx));
  FieldRef r;
  TRY(field_ref(ctx, field, &r));
  if (bytes != r.bytes) return fail(ctx, HE_ERR_ARG, "field %d: expected %zu bytes, got %zu", field, r.bytes, bytes);
  void* d = member_ptr(ctx, r.ptr, member);
  if (d == r.ptr) return fail(ctx, HE_ERR_STATE, "field %d is not a per-member buffer", field);
  const FieldFmt fmt = field_fmt(ctx, field);  // binary32 storage of the mixed path converts
  if (fmt == FMT_F64) {
    if (up) CK(cudaMemcpyAsync(d, host, bytes, cudaMemcpyHostToDevice, ctx->stream));
    else CK(cudaMemcpyAsync(host, d, bytes, cudaMemcpyDeviceToHost, ctx->stream));
    return sync_all(ctx);
  }
  std::vector<unsigned char> dev;
  if (up) {
    to_device_fmt(fmt, host, bytes, dev);
    CK(cudaMemcpyAsync(d, dev.data(), dev.size(), cudaMemcpyHostToDevice, ctx->stream));
    return sync_all(ctx);
  }
  dev.resize(device_fmt_bytes(fmt, bytes));
  CK(cudaMemcpyAsync(dev.data(), d, dev.size(), cudaMemcpyDeviceToHost, ctx->stream));
  TRY(sync_all(ctx));
  from_device_fmt(fmt, dev, host, bytes);
  return HE_OK;
}
int he_upload_member(he_ctx_t* ctx, int member, int field, const void* host, size_t bytes) {
  return member_xfer(ctx, member, field, const_cast<void*>(host), bytes, true);
}
int he_download_member(he_ctx_t* ctx, int member, int field, void* host, size_t bytes) {
  return member_xfer(ctx, member, field, host, bytes, false);
}

// The reduction slots (sums) of every member, nmem x S_COUNT values from the last launches.
static int member_sums(he_ctx_t* ctx, std::vector<double>& out) {
  TRY(join_aux(ctx));
  out.assign((size_t)ctx->nmem * S_COUNT, 0.0);
  for (int m = 0; m < ctx->nmem; ++m)
    CK(cudaMemcpyAsync(out.data() + (size_t)m * S_COUNT, member_ptr(ctx, ctx->sums, m),
                       S_COUNT * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  return sync_all(ctx);
}

int he_member_mu(he_ctx_t* ctx, int n4, int after_rk, double* mu4) {
  if (!ctx || !mu4) return fail(ctx, HE_ERR_ARG, "null argument");
  if (ctx->mode != HE_MODE_STATICS) return fail(ctx, HE_ERR_STATE, "statics routine");
  std::vector<double> s;
  TRY(member_sums(ctx, s));
  const int slot = after_rk ? S_HMEAN0 : S_STAT_H;
  for (int m = 0; m < ctx->nmem; ++m) mu4[m] = s[(size_t)m * S_COUNT + slot] * ctx->dxyz / (double)n4;
  return HE_OK;
}

int he_energy_members(he_ctx_t* ctx, he_energies_t* out) {
  if (!ctx || !out) return fail(ctx, HE_ERR_ARG, "null argument");
  if (ctx->mode == HE_MODE_QUANTUM && !ctx->otc) {
    if (ctx->nq == 0) return fail(ctx, HE_ERR_STATE, "he_set_quantum_impurities first");
    TRY(q_energy_launch(ctx));
    std::vector<double> all;
    TRY(member_sums(ctx, all));
    for (int m = 0; m < ctx->nmem; ++m) q_energy_from(ctx, all.data() + (size_t)m * S_COUNT, nullptr, &out[m]);
    return HE_OK;
  }
  if (ctx->mode != HE_MODE_STATICS || ctx->mixed || ctx->otc)
    return fail(ctx, HE_ERR_STATE, "members' energies: binary64 statics or quantum groups (OT/OP cores)");
  TRY(he_energy(ctx, &out[0]));
  std::vector<double> all;
  TRY(member_sums(ctx, all));
  const double dxyz = ctx->dxyz;
  for (int m = 1; m < ctx->nmem; ++m) {
    const double* s = all.data() + (size_t)m * S_COUNT + S_EN;
    he_energies_t e{};
    e.esolid = ctx->fn.lsolid ? ctx->fn.C * s[3] * dxyz : 0.0;
    e.ekin4 = ctx->fn.h2o2m4 * s[0] * dxyz;
    e.elj4 = 0.5 * s[1] * dxyz;
    e.ecor4 = s[2] * dxyz;
    e.etot4 = e.ekin4 + e.elj4 + e.ecor4 + e.esolid;
    e.eimpu = 0.0;
    e.etot = e.etot4;
    out[m] = e;
  }
  return HE_OK;
}

int he_download(he_ctx_t* ctx, int field, void* host, size_t bytes) {
  if (!ctx || !host) return fail(ctx, HE_ERR_ARG, "null argument");
  TRY(join_aux(ctx));
  if (qfield(field)) return q_xfer(ctx, field, host, bytes, false);
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
  const FieldFmt fmt = field_fmt(ctx, field);
  if (fmt != FMT_F64) {
    std::vector<unsigned char> dev(device_fmt_bytes(fmt, bytes));
    CK(cudaMemcpyAsync(dev.data(), r.ptr, dev.size(), cudaMemcpyDeviceToHost, ctx->stream));
    TRY(sync_all(ctx));
    from_device_fmt(fmt, dev, host, bytes);
    return HE_OK;
  }
  CK(cudaMemcpyAsync(host, r.ptr, bytes, cudaMemcpyDeviceToHost, ctx->stream));
  TRY(sync_all(ctx));
  return HE_OK;
}

// ---- Dynamics_TDDFT ------------------------------------------------------------------------------
int he_poten(he_ctx_t* ctx) {
  if (!ctx) return HE_ERR_ARG;
  if (!ctx->kernels_ok) return fail(ctx, HE_ERR_STATE, "k-space kernels not set");
  if (ctx->mode == HE_MODE_QUANTUM) {
    if (ctx->nq == 0) return fail(ctx, HE_ERR_STATE, "he_set_quantum_impurities first");
    return q_poten(ctx);
  }
  if (ctx->mode == HE_MODE_STATICS) {
    // He_statics/poten.f90:27-115: delj4 from the last refreshed fden (cached by
    // he_refresh_density), correlation with the current den and the stale dencg.
    XArgs a = xargs(ctx);
    a.den = ctx->den; a.dencg_in = ctx->dencg;
    a.specA = ctx->wA;
    TRY(xpass<X_R2C_CORR>(ctx, a));
    const double* ua = nullptr;
    if (ctx->otc) TRY(statics_term_alfa(ctx, &ua));  // He_statics/poten.f90:86-91 (denalf from the refresh)
    return correlation_tail(ctx, nullptr, ua);
  }
  if (ctx->xyfuse && !ctx->otc) return poten_fused(ctx, nullptr, nullptr);
  TRY(spectrum_cg_lj(ctx));
  XArgs a = xargs(ctx);
  a.specA = ctx->wA; a.specB = ctx->wB;
  a.den = ctx->den;
  a.out1 = ctx->dencg; a.out2 = ctx->delj4;
  TRY(xpass<X_C2R2_CORR>(ctx, a));
  const double* ua = nullptr;
  if (ctx->otc) TRY(otc_terms(ctx, &ua));  // Dynamics_TDDFT/poten.f90:144, :200-210
  return correlation_tail(ctx, nullptr, ua);
}


int he_potenimp(he_ctx_t* ctx) {
  if (!ctx) return HE_ERR_ARG;
  if (ctx->mode == HE_MODE_QUANTUM) {
    if (ctx->nq == 0) return fail(ctx, HE_ERR_STATE, "he_set_quantum_impurities first");
    if (!ctx->kernels_ok) return fail(ctx, HE_ERR_STATE, "k-space kernels not set");
    return q_potenimp(ctx);
  }
  if (ctx->mode != HE_MODE_DYNAMICS) return fail(ctx, HE_ERR_STATE, "potenimp is a dynamics routine");
  if (ctx->n_imp == 0) {
    ctx->force_fresh = true;
    return HE_OK;
  }
  int st;
  auto launch = [&]() {
    if (ctx->n_imp <= 1) return launch_impfield<1>(ctx);
    if (ctx->n_imp <= 2) return launch_impfield<2>(ctx);
    if (ctx->n_imp <= 4) return launch_impfield<4>(ctx);
    return launch_impfield<8>(ctx);
  };
  if (overlap_on(ctx)) {
    // the field pass reads den (ready on the main stream) and the impurity state (side stream)
    TRY(fork_aux(ctx));
    OnAux on(ctx);
    st = launch();
  } else {
    st = launch();
  }
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
  k_imp_force<<<1, 128, 0, imp_stream(ctx)>>>(ctx->imp, ctx->sums + S_FORCE, ctx->dxyz);
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
  k_imp_accel<<<1, 128, 0, imp_stream(ctx)>>>(ctx->imp);
  LAUNCHED();
  return HE_OK;
}


int he_steprk(he_ctx_t* ctx, double deltat) {
  if (!ctx) return HE_ERR_ARG;
  if (ctx->mode == HE_MODE_QUANTUM) {
    if (ctx->nq == 0) return fail(ctx, HE_ERR_STATE, "he_set_quantum_impurities first");
    return q_steprk(ctx, deltat);
  }
  if (ctx->mode != HE_MODE_DYNAMICS) return fail(ctx, HE_ERR_STATE, "steprk is a dynamics routine");
  const double r2 = 1.0 / std::sqrt(2.0);
  const double arun[4] = {0.5, 1.0 - r2, 1.0 + r2, 1.0 / 6.0};
  const double brun[4] = {2.0, 1.0, 1.0, 2.0};
  const double crun[4] = {0.5, 1.0 - r2, 1.0 + r2, 0.5};
  for (int jr = 0; jr < 4; ++jr) {
    void* ob = jr == 0 ? ctx->psiold[2] : ctx->scratch;
    if (ctx->mixed) {
      OpRKM op{};
      op.s8[0] = (const float*)ctx->pot4; op.s8[1] = (const float*)ctx->uimp;
      op.s16[0] = (const float2*)ctx->q; op.s16[1] = lo_plane(ctx, ctx->psi);
      op.q = (float2*)ctx->q;
      op.out_hi = hi_plane(ob); op.out_lo = lo_plane(ctx, ob);
      op.hsave = jr == 0 ? (float2*)ctx->hpsiold[1] : nullptr;
      op.den = (float*)ctx->den;
      op.tm = timec_view(ctx);
      op.h2o2m = (float)ctx->fn.h2o2m4;
      op.a = (float)arun[jr]; op.b = (float)brun[jr]; op.cc = (float)crun[jr]; op.dt = (float)deltat;
      TRY(run_stencil(ctx, ctx->g2, hi_plane(ctx->psi), op));
    } else {
      OpRK op{};
      op.s8[0] = ctx->pot4; op.s8[1] = ctx->uimp;
      op.s16[0] = (const double2*)ctx->q;
      op.q = (double2*)ctx->q;
      op.out = (double2*)ob;
      op.hsave = jr == 0 ? (double2*)ctx->hpsiold[1] : nullptr;
      op.den = ctx->den;
      op.tm = timec_view(ctx);
      op.h2o2m = ctx->fn.h2o2m4;
      op.a = arun[jr]; op.b = brun[jr]; op.cc = crun[jr]; op.dt = deltat;
      TRY(run_stencil(ctx, ctx->g2, (const double2*)ctx->psi, op));
    }
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
      k_imp_rk<<<1, 128, 0, imp_stream(ctx)>>>(ctx->imp, jr, arun[jr], brun[jr], crun[jr], deltat);
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
  if (ctx->mode == HE_MODE_QUANTUM) {
    if (ctx->nq == 0) return fail(ctx, HE_ERR_STATE, "he_set_quantum_impurities first");
    if (errvimp) *errvimp = 0.0;
    return q_steppc(ctx, deltat, errHe, errimp);
  }
  if (ctx->mode != HE_MODE_DYNAMICS) return fail(ctx, HE_ERR_STATE, "steppc is a dynamics routine");
  const double c112 = 112.0 / 121.0, c9 = 9.0 / 121.0, c4o3 = 4.0 / 3.0;
  if (ctx->mixed) {
    void* p3 = ctx->psiold[ctx->ioldp[2] - 1];
    OpPredictM op{};
    op.s8[0] = (const float*)ctx->pot4; op.s8[1] = (const float*)ctx->uimp;
    op.po3_hi = hi_plane(p3); op.po3_lo = lo_plane(ctx, p3);
    op.h2 = (float2*)ctx->hpsiold[ctx->ioldh[1] - 1];
    op.s16[0] = op.po3_hi;
    op.s16[1] = op.po3_lo;
    op.s16[2] = (const float2*)ctx->hpsiold[ctx->ioldh[0] - 1];
    op.s16[3] = op.h2;
    op.s16[4] = (const float2*)ctx->pc;
    op.den = (float*)ctx->den;
    op.tm = timec_view(ctx);
    op.h2o2m = (float)ctx->fn.h2o2m4;
    op.s43 = (float)(c4o3 * deltat);
    op.c112 = (float)c112;
    TRY(run_stencil(ctx, ctx->g2, hi_plane(ctx->psi), op));
    std::swap(ctx->psi, ctx->psiold[ctx->ioldp[2] - 1]);
    std::swap(ctx->ioldh[0], ctx->ioldh[1]);
  } else {
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
    k_imp_predict<<<1, 128, 0, imp_stream(ctx)>>>(ctx->imp, deltat);
    LAUNCHED();
  }
  TRY(field_eval(ctx));
  if (ctx->mixed) {
    void* a3 = ctx->psiold[ctx->ioldp[2] - 1];
    void* a2 = ctx->psiold[ctx->ioldp[1] - 1];
    OpCorrectM op{};
    op.s8[0] = (const float*)ctx->pot4; op.s8[1] = (const float*)ctx->uimp;
    op.s16[0] = lo_plane(ctx, ctx->psi);
    op.s16[1] = hi_plane(a3); op.s16[2] = lo_plane(ctx, a3);
    op.s16[3] = hi_plane(a2); op.s16[4] = lo_plane(ctx, a2);
    op.s16[5] = (const float2*)ctx->hpsiold[ctx->ioldh[0] - 1];
    op.s16[6] = (const float2*)ctx->hpsiold[ctx->ioldh[1] - 1];
    op.s16[7] = (const float2*)ctx->pc;
    op.pc = (float2*)ctx->pc;
    op.out_hi = hi_plane(ctx->scratch); op.out_lo = lo_plane(ctx, ctx->scratch);
    op.den = (float*)ctx->den;
    op.tm = timec_view(ctx);
    op.h2o2m = (float)ctx->fn.h2o2m4;
    op.s3 = (float)(3.0 * deltat);
    op.c9 = (float)c9;
    op.c112 = (float)c112;
    TRY(run_stencil_red(ctx, ctx->g2, hi_plane(ctx->psi), op, S_ERRHE));
    std::swap(ctx->psi, ctx->scratch);
    const int a = ctx->ioldp[2];
    ctx->ioldp[2] = ctx->ioldp[1];
    ctx->ioldp[1] = ctx->ioldp[0];
    ctx->ioldp[0] = a;
  } else {
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
    k_imp_correct<<<1, 128, 0, imp_stream(ctx)>>>(ctx->imp, deltat);
    LAUNCHED();
  }
  if (errHe || errimp || errvimp) {
    TRY(join_aux(ctx));
    CK(cudaMemcpyAsync(ctx->hsum, ctx->sums, S_COUNT * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    ImpDev h;
    if (ctx->n_imp > 0) TRY(imp_pull(ctx, &h));
    TRY(sync_all(ctx));
    if (errHe) *errHe = c9 * ctx->hsum[S_ERRHE] / (double)ctx->N;
    if (errimp) *errimp = ctx->n_imp > 0 ? h.errimp : 0.0;
    if (errvimp) *errvimp = ctx->n_imp > 0 ? h.errvimp : 0.0;
  }
  return HE_OK;
}


int he_energy(he_ctx_t* ctx, he_energies_t* out) {
  if (!ctx || !out) return fail(ctx, HE_ERR_ARG, "null argument");
  if (ctx->mode == HE_MODE_QUANTUM) {
    if (ctx->nq == 0) return fail(ctx, HE_ERR_STATE, "he_set_quantum_impurities first");
    return q_energy(ctx, out);
  }
  if (ctx->mode == HE_MODE_DYNAMICS && ctx->mixed) {
    OpEnergy<float2> op{};
    op.s8[0] = (const float*)ctx->den; op.s8[1] = (const float*)ctx->dencg;
    op.s8[2] = (const float*)ctx->delj4; op.s8[3] = (const float*)ctx->uimp;
    op.has_u = 1;
    op.aux1 = 0.5 * ctx->fn.cp4; op.aux2 = (1.0 / 3.0) * ctx->fn.cpp4;
    op.beta = ctx->fn.beta; op.den_m = ctx->fn.den_m; op.lsolid = ctx->fn.lsolid;
    TRY(run_stencil_red(ctx, ctx->g1, hi_plane(ctx->psi), op, S_EN));
  } else if (ctx->mode == HE_MODE_DYNAMICS) {
    OpEnergy<double2> op{};
    op.s8[0] = ctx->den; op.s8[1] = ctx->dencg; op.s8[2] = ctx->delj4; op.s8[3] = ctx->uimp;
    op.has_u = 1;
    op.aux1 = 0.5 * ctx->fn.cp4; op.aux2 = (1.0 / 3.0) * ctx->fn.cpp4;
    op.beta = ctx->fn.beta; op.den_m = ctx->fn.den_m; op.lsolid = ctx->fn.lsolid;
    TRY(run_stencil_red(ctx, ctx->g1, (const double2*)ctx->psi, op, S_EN));
  } else if (ctx->mixed) {  // statics, binary32 fields and psi's hi plane
    OpEnergy<float> op{};
    op.s8[0] = (const float*)ctx->den; op.s8[1] = (const float*)ctx->dencg;
    op.s8[2] = (const float*)ctx->delj4; op.s8[3] = (const float*)ctx->den;
    op.has_u = 0;
    op.aux1 = 0.5 * ctx->fn.cp4; op.aux2 = (1.0 / 3.0) * ctx->fn.cpp4;
    op.beta = ctx->fn.beta; op.den_m = ctx->fn.den_m; op.lsolid = ctx->fn.lsolid;
    TRY(run_stencil_red(ctx, ctx->g1, (const float*)ctx->psi, op, S_EN));
  } else {
    OpEnergy<double> op{};
    op.s8[0] = ctx->den; op.s8[1] = ctx->dencg; op.s8[2] = ctx->delj4; op.s8[3] = ctx->den;
    op.has_u = 0;
    op.aux1 = 0.5 * ctx->fn.cp4; op.aux2 = (1.0 / 3.0) * ctx->fn.cpp4;
    op.beta = ctx->fn.beta; op.den_m = ctx->fn.den_m; op.lsolid = ctx->fn.lsolid;
    TRY(run_stencil_red(ctx, ctx->g1, (const double*)ctx->psi, op, S_EN));
  }
  if (ctx->otc) TRY(alfa_energy_sum(ctx));
  TRY(join_aux(ctx));
  CK(cudaMemcpyAsync(ctx->hsum, ctx->sums, S_COUNT * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  TRY(sync_all(ctx));
  const double* s = ctx->hsum + S_EN;
  const double dxyz = ctx->dxyz;
  he_energies_t e{};
  e.esolid = ctx->fn.lsolid ? ctx->fn.C * s[3] * dxyz : 0.0;
  e.ekin4 = ctx->fn.h2o2m4 * s[0] * dxyz;
  e.elj4 = 0.5 * s[1] * dxyz;
  e.ecor4 = s[2] * dxyz;
  e.etot4 = e.ekin4 + e.elj4 + e.ecor4 + e.esolid;
  e.ealphas = 0.0;
  if (ctx->otc) {
    e.ealphas = alfa_energy(ctx);
    e.etot4 = e.etot4 + e.ealphas;
  }
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
  if (ctx->mixed) return fail(ctx, HE_ERR_STATE, "derden is not part of the mixed-precision path");
  return derden_of(ctx, ctx->den);
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
  // the gradients feed only the alpha_s term: binary64 ones of a binary64 copy of den in the
  // mixed path with OTC, none in the mixed path otherwise
  if (!ctx->mixed) TRY(he_derden(ctx));
  TRY(spectrum_cg_lj(ctx));
  XArgs a = xargs(ctx);
  a.specA = ctx->wA; a.specB = ctx->wB;
  a.out1 = ctx->dencg; a.out2 = ctx->delj4;
  TRY(xpass<X_C2R2>(ctx, a));
  if (ctx->otc) TRY(statics_alfa_density(ctx));  // BCN4HeDFT.f90:1142-1148
  return HE_OK;
}





int he_evolo0(he_ctx_t* ctx, double* mu4, double* mu4err, int n4) {
  if (!ctx || !mu4 || !mu4err) return fail(ctx, HE_ERR_ARG, "null argument");
  if (ctx->mode != HE_MODE_STATICS) return fail(ctx, HE_ERR_STATE, "statics routine");
  TRY(stat_hpsi(ctx, ctx->hpsi, S_STAT_H));
  tname(ctx, "statics_sumsq");
  if (ctx->mixed)
    k_sumsq_m<<<pw_blocks(ctx), 256, 0, ctx->stream>>>((const float*)ctx->psi, ctx->N, tail(ctx, S_STAT_N));
  else
    k_sumsq<<<pw_grid(ctx), 256, 0, ctx->stream>>>((const double*)ctx->psi, ctx->N, tail(ctx, S_STAT_N),
                                                   ctx->mm);
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
      k_copy_slot<<<dim3(1, ctx->nmem), 32, 0, ctx->stream>>>(ctx->sums, S_HMEAN0, S_STAT_H, ctx->mm);
      LAUNCHED();
    }
    if (ctx->mixed) {
      StatPWM s = statpwm(ctx, deltat, n4);
      s.psi = (const float*)ctx->psi;
      s.hpsi = (const float*)ctx->hpsi;
      s.q = (float*)ctx->q;
      s.out = (float*)(jr == 0 ? ctx->psiold[2] : ctx->scratch);
      s.hsave = jr == 0 ? (float*)ctx->hpsiold[1] : nullptr;
      s.a = arun[jr]; s.b = brun[jr]; s.c = crun[jr];
      s.jr = jr;
      tname(ctx, "statics_rk_update_f32");
      k_stat_rk_m<<<pw_blocks(ctx), 256, 0, ctx->stream>>>(s, tail(ctx, S_STAT_N));
    } else {
      StatPW s = statpw(ctx, deltat, n4);
      s.psi = (double*)ctx->psi;
      s.hpsi = ctx->hpsi;
      s.q = (double*)ctx->q;
      s.out = (double*)(jr == 0 ? ctx->psiold[2] : ctx->scratch);
      s.hsave = jr == 0 ? (double*)ctx->hpsiold[1] : nullptr;
      s.a = arun[jr]; s.b = brun[jr]; s.c = crun[jr];
      s.jr = jr;
      tname(ctx, "statics_rk_update");
      k_stat_rk<<<pw_grid(ctx), 256, 0, ctx->stream>>>(s, tail(ctx, S_STAT_N));
    }
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

// steppcr's launches; the sums stay on the device (S_STAT_H, S_STAT_PC).
static int steppcr_launch(he_ctx_t* ctx, double deltat, int n4) {
  TRY(stat_hpsi(ctx, ctx->hpsi, S_STAT_H));
  if (ctx->mixed) {
    StatPWM s = statpwm(ctx, deltat, n4);
    s.psi = (const float*)ctx->psi;
    s.hpsi = (const float*)ctx->hpsi;
    s.po3 = (float*)ctx->psiold[ctx->ioldp[2] - 1];
    s.h1 = (const float*)ctx->hpsiold[ctx->ioldh[0] - 1];
    s.h2 = (float*)ctx->hpsiold[ctx->ioldh[1] - 1];
    s.pc = (float*)ctx->pc;
    tname(ctx, "statics_predict_f32");
    k_stat_predict_m<<<pw_blocks(ctx), 256, 0, ctx->stream>>>(s, tail(ctx, S_STAT_N));
    LAUNCHED();
    std::swap(ctx->psi, ctx->psiold[ctx->ioldp[2] - 1]);
    std::swap(ctx->ioldh[0], ctx->ioldh[1]);
  } else {
    StatPW s = statpw(ctx, deltat, n4);
    s.psi = (double*)ctx->psi;
    s.hpsi = ctx->hpsi;
    s.po3 = (double*)ctx->psiold[ctx->ioldp[2] - 1];
    s.h1 = (const double*)ctx->hpsiold[ctx->ioldh[0] - 1];
    s.h2 = (double*)ctx->hpsiold[ctx->ioldh[1] - 1];
    s.pc = (double*)ctx->pc;
    tname(ctx, "statics_predict");
    s.nlb = pw_blocks(ctx);
    s.lpb = pw_lpb(ctx);
    k_stat_predict<<<pw_grid_lb(ctx), 256, 0, ctx->stream>>>(s, tail(ctx, S_STAT_N));
    LAUNCHED();
    std::swap(ctx->psi, ctx->psiold[ctx->ioldp[2] - 1]);
    std::swap(ctx->ioldh[0], ctx->ioldh[1]);
  }
  TRY(stat_normalize(ctx, n4));
  TRY(he_poten(ctx));
  TRY(stat_hpsi(ctx, ctx->t4, S_STAT_MU));
  if (ctx->mixed) {
    StatPWM s = statpwm(ctx, deltat, n4);
    s.psi = (const float*)ctx->psi;
    s.hpsi = (const float*)ctx->t4;
    s.po3 = (float*)ctx->psiold[ctx->ioldp[2] - 1];
    s.po2 = (const float*)ctx->psiold[ctx->ioldp[1] - 1];
    s.h1 = (const float*)ctx->hpsiold[ctx->ioldh[0] - 1];
    s.h2 = (float*)ctx->hpsiold[ctx->ioldh[1] - 1];
    s.pc = (float*)ctx->pc;
    s.out = (float*)ctx->scratch;
    ReduceTail rt = tail(ctx, S_STAT_PC);
    tname(ctx, "statics_correct_f32");
    k_stat_correct_m<<<pw_blocks(ctx), 256, 0, ctx->stream>>>(s, rt);
    LAUNCHED();
    std::swap(ctx->psi, ctx->scratch);
  } else {
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
    s.nlb = pw_blocks(ctx);
    s.lpb = pw_lpb(ctx);
    k_stat_correct<<<pw_grid_lb(ctx), 256, 0, ctx->stream>>>(s, rt);
    LAUNCHED();
    std::swap(ctx->psi, ctx->scratch);
  }
  // k_stat_correct leaves sum psi^2 in S_STAT_PC+1, which the normalisation reads
  TRY(stat_normalize(ctx, n4, S_STAT_PC + 1));
  const int a = ctx->ioldp[2];
  ctx->ioldp[2] = ctx->ioldp[1];
  ctx->ioldp[1] = ctx->ioldp[0];
  ctx->ioldp[0] = a;
  return HE_OK;
}

int he_steppcr(he_ctx_t* ctx, double deltat, double* mu4, double* mu4err, int n4, double* errpc) {
  if (!ctx || !mu4 || !mu4err) return fail(ctx, HE_ERR_ARG, "null argument");
  if (ctx->mode != HE_MODE_STATICS) return fail(ctx, HE_ERR_STATE, "statics routine");
  TRY(steppcr_launch(ctx, deltat, n4));
  TRY(read_sums(ctx));
  const double hmean = ctx->hsum[S_STAT_H] * ctx->dxyz / (double)n4;
  if (errpc) *errpc = (9.0 / 121.0) * ctx->hsum[S_STAT_PC] / (double)ctx->N;
  *mu4err = std::fabs(1.0 - *mu4 / hmean);
  *mu4 = hmean;
  return HE_OK;
}

// One pass of the statics loop body with Lrkpc and ppot = 1 (BCN4HeDFT.f90:1120-1160): steppcr,
// derden, fden, dencg, poten; first S_STAT_H (the previous pass's hmean) is kept in S_STAT_PREV.
static int statics_pass(he_ctx_t* ctx, double deltat, int n4) {
  tname(ctx, "copy_slot");
  k_copy_slot<<<dim3(1, ctx->nmem), 32, 0, ctx->stream>>>(ctx->sums, S_STAT_PREV, S_STAT_H, ctx->mm);
  LAUNCHED();
  TRY(steppcr_launch(ctx, deltat, n4));
  TRY(he_refresh_density(ctx));
  return he_poten(ctx);
}

constexpr size_t kMaxStatGraphs = 64;  // the statics relabelling repeats after 30 passes

// A statics pass from the graph cache: replayed when this state was seen before, else captured
// (after one eager pass) and launched.  The host-side relabelling then follows the graph's.
static int statics_pass_graphed(he_ctx_t* ctx, double deltat, int n4) {
  if (ctx->timing || !ctx->stat_warm) {
    TRY(statics_pass(ctx, deltat, n4));
    ctx->stat_warm = true;
    return HE_OK;
  }
  unsigned long long key = 0;
  TRY(he_state_fingerprint(ctx, &key));
  const double kd[2] = {deltat, (double)n4};
  const unsigned char* b = reinterpret_cast<const unsigned char*>(kd);
  for (size_t i = 0; i < sizeof kd; ++i) { key ^= b[i]; key *= 1099511628211ull; }
  for (const auto& g : ctx->stat_graphs) {
    if (g.key != key) continue;
    CK(cudaGraphLaunch(g.exec, ctx->stream));
    ctx->psi = g.psi;
    ctx->scratch = g.scratch;
    for (int i = 0; i < 3; ++i) { ctx->psiold[i] = g.psiold[i]; ctx->ioldp[i] = g.ioldp[i]; }
    for (int i = 0; i < 2; ++i) { ctx->hpsiold[i] = g.hpsiold[i]; ctx->ioldh[i] = g.ioldh[i]; }
    ctx->launches += g.launches;
    return HE_OK;
  }
  if (ctx->stat_graphs.size() >= kMaxStatGraphs) return statics_pass(ctx, deltat, n4);
  // The capture records kernels without running them, while the pass relabels the ring on the
  // host as it goes.  Keep the relabelling from before the capture so that a capture or an
  // instantiation that fails leaves the context describing the buffers as they are.
  he_ctx::StatGraph before{};
  before.psi = ctx->psi;
  before.scratch = ctx->scratch;
  for (int i = 0; i < 3; ++i) { before.psiold[i] = ctx->psiold[i]; before.ioldp[i] = ctx->ioldp[i]; }
  for (int i = 0; i < 2; ++i) { before.hpsiold[i] = ctx->hpsiold[i]; before.ioldh[i] = ctx->ioldh[i]; }
  const long long l0 = ctx->launches;
  auto restore = [&]() {
    ctx->psi = before.psi;
    ctx->scratch = before.scratch;
    for (int i = 0; i < 3; ++i) { ctx->psiold[i] = before.psiold[i]; ctx->ioldp[i] = before.ioldp[i]; }
    for (int i = 0; i < 2; ++i) { ctx->hpsiold[i] = before.hpsiold[i]; ctx->ioldh[i] = before.ioldh[i]; }
    ctx->launches = l0;
  };
  CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeRelaxed));
  const int rc = statics_pass(ctx, deltat, n4);
  cudaGraph_t graph = nullptr;
  const cudaError_t ec = cudaStreamEndCapture(ctx->stream, &graph);
  if (rc != HE_OK || ec != cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    cudaGetLastError();
    restore();
    if (rc != HE_OK) return rc;
    return fail(ctx, HE_ERR_CUDA, "statics pass capture failed: %s", cudaGetErrorString(ec));
  }
  he_ctx::StatGraph g{};
  g.key = key;
  const cudaError_t ei = cudaGraphInstantiate(&g.exec, graph, 0);
  cudaGraphDestroy(graph);
  if (ei != cudaSuccess) {
    restore();
    return fail(ctx, HE_ERR_CUDA, "graph instantiation failed: %s", cudaGetErrorString(ei));
  }
  g.psi = ctx->psi;
  g.scratch = ctx->scratch;
  for (int i = 0; i < 3; ++i) { g.psiold[i] = ctx->psiold[i]; g.ioldp[i] = ctx->ioldp[i]; }
  for (int i = 0; i < 2; ++i) { g.hpsiold[i] = ctx->hpsiold[i]; g.ioldh[i] = ctx->ioldh[i]; }
  g.launches = ctx->launches - l0;
  ctx->stat_graphs.push_back(g);
  const cudaError_t el = cudaGraphLaunch(g.exec, ctx->stream);
  if (el != cudaSuccess) {
    restore();
    return fail(ctx, HE_ERR_CUDA, "graph launch failed: %s", cudaGetErrorString(el));
  }
  return HE_OK;
}

int he_statics_iterations(he_ctx_t* ctx, int niter, double deltat, double* mu4, double* mu4err, int n4,
                          double* errpc) {
  if (!ctx || !mu4 || !mu4err) return fail(ctx, HE_ERR_ARG, "null argument");
  if (niter < 1) return fail(ctx, HE_ERR_ARG, "niter must be positive");
  if (ctx->mode != HE_MODE_STATICS) return fail(ctx, HE_ERR_STATE, "statics routine");
  if (!ctx->kernels_ok) return fail(ctx, HE_ERR_STATE, "k-space kernels not set");
  TRY(join_aux(ctx));
  for (int k = 0; k < niter; ++k) TRY(statics_pass_graphed(ctx, deltat, n4));
  TRY(read_sums(ctx));
  const double hmean = ctx->hsum[S_STAT_H] * ctx->dxyz / (double)n4;
  const double prev = niter > 1 ? ctx->hsum[S_STAT_PREV] * ctx->dxyz / (double)n4 : *mu4;
  if (errpc) *errpc = (9.0 / 121.0) * ctx->hsum[S_STAT_PC] / (double)ctx->N;
  *mu4err = std::fabs(1.0 - prev / hmean);
  *mu4 = hmean;
  return HE_OK;
}

int he_statics_iterations_members(he_ctx_t* ctx, int niter, double deltat, int n4, double* mu4,
                                  double* mu4err, double* errpc) {
  if (!ctx || !mu4 || !mu4err) return fail(ctx, HE_ERR_ARG, "null argument");
  if (niter < 1) return fail(ctx, HE_ERR_ARG, "niter must be positive");
  if (ctx->mode != HE_MODE_STATICS) return fail(ctx, HE_ERR_STATE, "statics routine");
  if (!ctx->kernels_ok) return fail(ctx, HE_ERR_STATE, "k-space kernels not set");
  TRY(join_aux(ctx));
  for (int k = 0; k < niter; ++k) TRY(statics_pass_graphed(ctx, deltat, n4));
  std::vector<double> all;
  TRY(member_sums(ctx, all));
  for (int m = 0; m < ctx->nmem; ++m) {
    const double* h = all.data() + (size_t)m * S_COUNT;
    const double hmean = h[S_STAT_H] * ctx->dxyz / (double)n4;
    const double prev = niter > 1 ? h[S_STAT_PREV] * ctx->dxyz / (double)n4 : mu4[m];
    if (errpc) errpc[m] = (9.0 / 121.0) * h[S_STAT_PC] / (double)ctx->N;
    mu4err[m] = std::fabs(1.0 - prev / hmean);
    mu4[m] = hmean;
  }
  return HE_OK;
}

int he_varmu(he_ctx_t* ctx, int npart, double mu, double* errmu) {
  if (!ctx || !errmu) return fail(ctx, HE_ERR_ARG, "null argument");
  if (ctx->mode != HE_MODE_STATICS) return fail(ctx, HE_ERR_STATE, "statics routine");
  tname(ctx, "statics_varmu");
  if (ctx->mixed)
    k_varmu_m<<<pw_blocks(ctx), 256, 0, ctx->stream>>>((const float*)ctx->hpsi, (const float*)ctx->psi,
                                                       ctx->N, mu, tail(ctx, S_VARMU));
  else
    k_varmu<<<pw_grid(ctx), 256, 0, ctx->stream>>>(ctx->hpsi, (const double*)ctx->psi, ctx->N, mu,
                                                   tail(ctx, S_VARMU), ctx->mm);
  LAUNCHED();
  TRY(read_sums(ctx));
  *errmu = ctx->hsum[S_VARMU] * ctx->dxyz / (double)npart;
  return HE_OK;
}

int he_timing(he_ctx_t* ctx, int enable) {
  if (!ctx) return HE_ERR_ARG;
  TRY(sync_all(ctx));
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
  TRY(sync_all(ctx));
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

int he_set_fft_variant(he_ctx_t* ctx, int pass, int variant, int tile) {
  if (!ctx) return HE_ERR_ARG;
  stat_graphs_clear(ctx);
  if (tile != 8 && tile != 16) return fail(ctx, HE_ERR_ARG, "tile must be 8 or 16");
  if (variant != 0 && variant != 1) return fail(ctx, HE_ERR_ARG, "variant must be 0 or 1");
  switch (pass) {
    case 0:
      if (!x_fast(ctx, tile)) return fail(ctx, HE_ERR_ARG, "x pass: no compile-time variant for this grid");
      for (int m = 0; m < 6; ++m) {
        if (variant && (long)xpipe_smem(ctx, m, tile) > (long)ctx->maxsm)
          return fail(ctx, HE_ERR_ARG, "pipelined x pass with %d rows does not fit shared memory", tile);
      }
      for (int m = 0; m < 6; ++m) { ctx->xpipe[m] = variant != 0; ctx->xtile[m] = tile; }
      ctx->tile_x = tile;
      return HE_OK;
    case 1:
      if (variant != 1) return fail(ctx, HE_ERR_ARG, "the y pass has the register variant only");
      ctx->tile_y = tile;
      return HE_OK;
    case 2:
      ctx->zreg = variant != 0;
      ctx->tile_z = tile;
      return HE_OK;
    case 10:
      if (variant && !yz_fusable(ctx))
        return fail(ctx, HE_ERR_ARG, "fused y-z convolutions need ny = nz = 64");
      ctx->yzfuse = variant != 0;
      return HE_OK;
    case 9:
      if (variant && !xy_fusable(ctx))
        return fail(ctx, HE_ERR_ARG, "fused x-y passes need HE_PREC_MIXED and nx = ny in {64, 96, 128}");
      ctx->xyfuse = variant != 0;
      return HE_OK;
    default:
      if (pass >= 3 && pass < 9) {  // one x mode (XMode pass - 3)
        const int m = pass - 3;
        if (!x_fast(ctx, tile)) return fail(ctx, HE_ERR_ARG, "x pass: no compile-time variant for this grid");
        if (variant && (long)xpipe_smem(ctx, m, tile) > (long)ctx->maxsm)
          return fail(ctx, HE_ERR_ARG, "pipelined x pass with %d rows does not fit shared memory", tile);
        ctx->xpipe[m] = variant != 0;
        ctx->xtile[m] = tile;
        return HE_OK;
      }
      return fail(ctx, HE_ERR_ARG, "pass must be 0 (x), 1 (y), 2 (z), 3..8 (one x mode), 9 (x-y) or 10 (y-z)");
  }
}

int he_state_fingerprint(const he_ctx_t* ctx, unsigned long long* out) {
  if (!ctx || !out) return HE_ERR_ARG;
  // FNV-1a over everything a step's launches depend on besides the array contents: the buffer
  // relabelling (psi, psiold, hpsiold, scratch and the impurity wave functions' counterparts),
  // the ring indices and the lazy-evaluation flags
  unsigned long long h = 1469598103934665603ull;
  auto mix = [&](const void* p, size_t n) {
    const unsigned char* b = static_cast<const unsigned char*>(p);
    for (size_t i = 0; i < n; ++i) { h ^= b[i]; h *= 1099511628211ull; }
  };
  const void* bufs[] = {ctx->psi, ctx->scratch, ctx->psiold[0], ctx->psiold[1], ctx->psiold[2],
                        ctx->hpsiold[0], ctx->hpsiold[1], ctx->xscratch};
  mix(bufs, sizeof bufs);
  for (int i = 0; i < kMaxQImp; ++i) {
    mix(&ctx->psix[i], sizeof(void*));
    mix(ctx->psixold[i], sizeof ctx->psixold[i]);
    mix(ctx->hpsixold[i], sizeof ctx->hpsixold[i]);
  }
  mix(ctx->ioldp, sizeof ctx->ioldp);
  mix(ctx->ioldh, sizeof ctx->ioldh);
  const int flags[2] = {ctx->cglj_pending ? 1 : 0, ctx->force_fresh ? 1 : 0};
  mix(flags, sizeof flags);
  *out = h;
  return HE_OK;
}

int he_autotune_report(const he_ctx_t* ctx, char* buf, size_t len) {
  if (!ctx || !buf || len == 0) return HE_ERR_ARG;
  std::string t = ctx->tune_log;
  snprintf(buf, len, "%s", t.c_str());
  return HE_OK;
}

int he_tuned_tiles(const he_ctx_t* ctx, int* x, int* y, int* z) {
  if (!ctx || !x || !y || !z) return HE_ERR_ARG;
  *x = ctx->tile_x;
  *y = ctx->tile_y;
  *z = ctx->tile_z;
  return HE_OK;
}

int he_set_quantum_impurities(he_ctx_t* ctx, const he_qimpurities_t* q) {
  if (!ctx || !q) return fail(ctx, HE_ERR_ARG, "null argument");
  if (ctx->mode != HE_MODE_QUANTUM) return fail(ctx, HE_ERR_STATE, "quantum impurities need HE_MODE_QUANTUM");
  const int n = q->n_imp;
  if (n < 1 || n > kMaxQImp) return fail(ctx, HE_ERR_ARG, "n_imp must be in [1, %d]", kMaxQImp);
  if (!q->m_imp_u) return fail(ctx, HE_ERR_ARG, "null m_imp_u");
  if (ctx->nq != 0 && ctx->nq != n) return fail(ctx, HE_ERR_STATE, "n_imp cannot change once set");
  for (int i = 0; i < n; ++i)
    if (!(q->m_imp_u[i] > 0.0)) return fail(ctx, HE_ERR_ARG, "impurity masses must be positive");
  const int nspline = q->n_spline > 0 ? q->n_spline : 100001;
  const size_t N = ctx->N, Nk = ctx->Nk;
  if (ctx->nq == 0) {
    for (int i = 0; i < n; ++i) {
      TRY(dalloc(ctx, &ctx->psix[i], 16 * N));
      TRY(dalloc(ctx, &ctx->pcx[i], 16 * N));
      TRY(dalloc(ctx, &ctx->qx[i], 16 * N));
      for (int s = 0; s < 3; ++s) TRY(dalloc(ctx, &ctx->psixold[i][s], 16 * N));
      for (int s = 0; s < 2; ++s) TRY(dalloc(ctx, &ctx->hpsixold[i][s], 16 * N));
      TRY(dalloc_t(ctx, &ctx->denx[i], N));
      TRY(dalloc_t(ctx, &ctx->upotx[i], N));
      TRY(dalloc_t(ctx, &ctx->uimpk[i], Nk));
      TRY(dalloc_t(ctx, &ctx->sx[i], Nk));
    }
  }
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) {
      const bool want = i != j && (q->uimp_k_k || q->x_x[i + n * j].kind != 0);
      double*& kk = ctx->uimpkk[i + kMaxQImp * j];
      if (want && !kk) TRY(dalloc_t(ctx, &kk, Nk));
      if (!want) kk = nullptr;  // a buffer left from an earlier call stays allocated, unused
    }
  ctx->nq = n;
  ctx->mu4 = q->mu4;
  for (int i = 0; i < n; ++i) ctx->h2o2mx[i] = ctx->fn.h2o2m4 * 4.002603 / q->m_imp_u[i];
  // potenimpini: uimp_k_i and uimp_k_k(i,j), each distinct potential transformed once.
  for (int i = 0; i < n; ++i) {
    if (q->uimp_k) {
      CK(cudaMemcpyAsync(ctx->uimpk[i], q->uimp_k + Nk * i, 8 * Nk, cudaMemcpyHostToDevice, ctx->stream));
      continue;
    }
    const double* same = nullptr;
    for (int k = 0; k < i && !same; ++k)
      if (std::memcmp(&q->he_x[k], &q->he_x[i], sizeof(he_pairpot_t)) == 0) same = ctx->uimpk[k];
    if (same) CK(cudaMemcpyAsync(ctx->uimpk[i], same, 8 * Nk, cudaMemcpyDeviceToDevice, ctx->stream));
    else TRY(q_kernel(ctx, q->he_x[i], nspline, q->nq, q->parabolic, ctx->uimpk[i]));
  }
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < n; ++i) {
      double* kk = ctx->uimpkk[i + kMaxQImp * j];
      if (!kk) continue;
      if (q->uimp_k_k) {
        CK(cudaMemcpyAsync(kk, q->uimp_k_k + Nk * (i + (size_t)n * j), 8 * Nk, cudaMemcpyHostToDevice, ctx->stream));
        continue;
      }
      TRY(q_kernel(ctx, q->x_x[i + n * j], nspline, q->nq, q->parabolic, kk));
    }
  TRY(sync_all(ctx));
  TRY(qkernels_to_f32(ctx));
  for (int i = 0; i < n; ++i) TRY(q_cnorm2(ctx, i));
  for (int i = 0; i < 3; ++i) ctx->ioldp[i] = i + 1;
  ctx->ioldh[0] = 1; ctx->ioldh[1] = 2;
  ctx->cglj_pending = false;
  return HE_OK;
}

int he_qimp_moments(he_ctx_t* ctx, double* out) {
  if (!ctx || !out) return fail(ctx, HE_ERR_ARG, "null argument");
  if (ctx->mode != HE_MODE_QUANTUM || ctx->nq == 0)
    return fail(ctx, HE_ERR_STATE, "no quantum impurities");
  for (int i = 0; i < ctx->nq; ++i) {
    tname(ctx, "impurity_moments");
    if (ctx->mixed)
      k_moments<<<pw_grid(ctx), 256, 0, ctx->stream>>>(
          (const float2*)ctx->psix[i], ctx->nx, ctx->ny, ctx->N, -ctx->xmax, -ctx->ymax, -ctx->zmax,
          ctx->hx, ctx->hy, ctx->hz, tail(ctx, S_QMOM + 4 * i), ctx->mm);
    else
      k_moments<<<pw_grid(ctx), 256, 0, ctx->stream>>>(
          (const double2*)ctx->psix[i], ctx->nx, ctx->ny, ctx->N, -ctx->xmax, -ctx->ymax, -ctx->zmax,
          ctx->hx, ctx->hy, ctx->hz, tail(ctx, S_QMOM + 4 * i), ctx->mm);
    LAUNCHED();
  }
  TRY(read_sums(ctx));
  for (int i = 0; i < ctx->nq; ++i) {
    const double* m = ctx->hsum + S_QMOM + 4 * i;
    const double a = m[0] * ctx->dxyz;
    out[4 * i] = a;
    out[4 * i + 1] = m[1] * ctx->dxyz / a;
    out[4 * i + 2] = m[2] * ctx->dxyz / a;
    out[4 * i + 3] = m[3] * ctx->dxyz / a;
  }
  return HE_OK;
}

int he_qimp_moments_members(he_ctx_t* ctx, double* out) {
  if (!ctx || !out) return fail(ctx, HE_ERR_ARG, "null argument");
  std::vector<double> m0(4 * (size_t)std::max(ctx->nq, 1));
  TRY(he_qimp_moments(ctx, m0.data()));
  std::vector<double> all;
  TRY(member_sums(ctx, all));
  for (int mb = 0; mb < ctx->nmem; ++mb)
    for (int i = 0; i < ctx->nq; ++i) {
      const double* m = all.data() + (size_t)mb * S_COUNT + S_QMOM + 4 * i;
      double* o = out + 4 * ((size_t)mb * ctx->nq + i);
      const double a = m[0] * ctx->dxyz;
      o[0] = a;
      o[1] = m[1] * ctx->dxyz / a;
      o[2] = m[2] * ctx->dxyz / a;
      o[3] = m[3] * ctx->dxyz / a;
    }
  return HE_OK;
}

int he_ft_v_spline_table(const he_pairpot_t* pot, double pmax, double hp, int n_spline,
                         int parabolic, double* vpp, int n_p, char* err, size_t errlen) {
  if (err && errlen) err[0] = '\0';
  auto bad = [&](int code, const char* msg) {
    if (err && errlen) snprintf(err, errlen, "%s", msg);
    return code;
  };
  if (!pot || !vpp) return bad(HE_ERR_ARG, "null argument");
  if (!(hp > 0.0) || !(pmax > 0.0)) return bad(HE_ERR_ARG, "pmax and hp must be positive");
  if ((int)(pmax / hp + 1.5) != n_p) return bad(HE_ERR_ARG, "n_p must be int(pmax/hp + 1.5)");
  std::vector<double> P, V, A, B, C, D;
  std::string why;
  cudaStream_t st = nullptr;
  cudaError_t e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = ftv::table(*pot, pmax, hp, n_spline > 0 ? n_spline : 100001, parabolic, st, P, V, A, B, C, D, &why);
  if (st) cudaStreamDestroy(st);
  if (e != cudaSuccess) {
    if (err && errlen) snprintf(err, errlen, "FT_V_spline: %s (%s)", why.c_str(), cudaGetErrorString(e));
    return e == cudaErrorInvalidValue ? HE_ERR_ARG : HE_ERR_CUDA;
  }
  std::memcpy(vpp, V.data(), sizeof(double) * n_p);
  return HE_OK;
}

int he_observables(he_ctx_t* ctx, int npart, double* out) {
  if (!ctx || !out) return fail(ctx, HE_ERR_ARG, "null argument");
  if (ctx->mode == HE_MODE_STATICS) return fail(ctx, HE_ERR_STATE, "observables need a complex psi");
  if (npart <= 0) return fail(ctx, HE_ERR_ARG, "npart must be positive");
  if (ctx->mixed) {
    OpObservablesT<float2> op{};
    op.s8[0] = (const float*)ctx->den;
    op.x0 = -ctx->xmax; op.y0 = -ctx->ymax; op.z0 = -ctx->zmax;
    op.hx = ctx->hx; op.hy = ctx->hy; op.hz = ctx->hz;
    TRY(run_stencil_red(ctx, ctx->g1, hi_plane(ctx->psi), op, S_OBS));
  } else {
    OpObservables op{};
    op.s8[0] = ctx->den;
    op.x0 = -ctx->xmax; op.y0 = -ctx->ymax; op.z0 = -ctx->zmax;
    op.hx = ctx->hx; op.hy = ctx->hy; op.hz = ctx->hz;
    TRY(run_stencil_red(ctx, ctx->g1, (const double2*)ctx->psi, op, S_OBS));
  }
  TRY(read_sums(ctx));
  const double* s = ctx->hsum + S_OBS;
  const double dxyz = ctx->dxyz;
  const double mhe = 4.002572164 * kMpU;  // DFT4He3d.f90:103, :315
  const double auxn4 = s[9] * dxyz;
  const double xcm = s[10] * dxyz / npart, ycm = s[11] * dxyz / npart, zcm = s[12] * dxyz / npart;
  // <L> = Re sum i conj(psi) (r - r_cm) x grad psi dxyz, Re(i w) = -Im w
  const double lz = -(s[3] - s[4] - ycm * s[0] + xcm * s[1]) * dxyz;
  const double ly = -(s[5] - s[6] - xcm * s[2] + zcm * s[0]) * dxyz;
  const double lx = -(s[7] - s[8] - zcm * s[1] + ycm * s[2]) * dxyz;
  const double v[13] = {auxn4, xcm, ycm, zcm, lx, ly, lz,
                        s[0] * dxyz / (auxn4 * mhe), s[1] * dxyz / (auxn4 * mhe), s[2] * dxyz / (auxn4 * mhe),
                        s[13] * dxyz, s[14] * dxyz, s[15] * dxyz};
  std::memcpy(out, v, sizeof(v));
  return HE_OK;
}

}  // extern "C"
