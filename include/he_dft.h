/*
 * he_dft.h -- C-ABI of the B200 (sm_100a) mean-field and time-step path of BCN-4He-DFT.
 *
 * This is the drop-in boundary.  The reference Fortran drivers call argument-less subroutines
 * that work on module arrays (Dynamics_TDDFT/DFT4He3d.f90:566-576,677-697,709-715;
 * He_statics/BCN4HeDFT.f90:1113-1160,1217).  Here the same state lives in device memory owned by
 * an he_ctx_t; the caller uploads module arrays once (after readen/readenc), calls the
 * replacement routines, and downloads at I/O points (printout/printoutc, energy prints).
 *
 * Conventions
 *   - Every function returns 0 (HE_OK) on success; a non-zero status leaves a message in
 *     he_last_error().  Nothing aborts the process.
 *   - Host arrays use the reference's layout: Fortran column-major (nx,ny,nz), x fastest,
 *     complex interleaved (re,im) binary64, half spectrum (nx/2+1,ny,nz), impurity arrays
 *     (N_imp,3) column-major.  Host-side values are always binary64, whatever the device
 *     precision.
 *   - Work is queued on the context's CUDA stream; functions that return scalars through
 *     pointers synchronise that stream, functions given NULL scalar pointers do not.
 *   - A context is not thread-safe; use one context per host thread.
 */
#ifndef HE_DFT_H
#define HE_DFT_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HE_OK 0
#define HE_ERR_ARG 1      /* invalid argument or size */
#define HE_ERR_CUDA 2     /* CUDA runtime error (message has the CUDA error string) */
#define HE_ERR_STATE 3    /* call not valid in this context mode / before set-up */
#define HE_ERR_NOMEM 4    /* device allocation failed */

typedef struct he_ctx he_ctx_t;

/* HE_MODE_QUANTUM: real-time dynamics with quantum impurities (Dynamics_quantum_impurities):
 * complex psi plus impurity wave functions psix_i (he_set_quantum_impurities). */
enum he_mode { HE_MODE_DYNAMICS = 0, HE_MODE_STATICS = 1, HE_MODE_QUANTUM = 2 };
/* HE_PREC_F64: binary64 throughout.  HE_PREC_MIXED (every mode and core; with OTC the alpha_s
 * term runs in binary64 on a binary64 copy of den and adds a binary32 copy of ualphas to pot4;
 * in the quantum mode
 * psix and psixold are pairs too, upotx / potx4 / denx binary32; in the statics mode the real
 * psi, psiold and pc are pairs, H psi binary32, and the imaginary-time updates and the norm, mu
 * and error sums binary64): the FFT chain
 * of the mean field, the 13-point stencils and H psi run in binary32; den, pot4, dencg, delj4,
 * uimp, fden, pc, q and hpsiold are held in binary32; psi and psiold are held as compensated
 * binary32 pairs (about 48 significant bits) and updated with error-free transformations; the
 * reductions (energy, errHe, impurity forces) and the impurity's Newton integration stay binary64.
 * he_upload / he_download convert (host arrays are binary64 in every mode).  Between the
 * predictor and the corrector of he_steppc, pc keeps the corrector's value instead of the
 * unmodified prediction. */
enum he_precision { HE_PREC_F64 = 0, HE_PREC_MIXED = 1 };

/* Grid: Dynamics_TDDFT/modules.f90:88-105 (grid), deriva npd/icon :31-37.  h = 2*xmax/n and
 * x_i = -xmax + h*(i-1) (DFT4He3d.f90:265-329).  npd must be 13; icon 13 (zero padding), 8
 * (periodic), 18 (antiperiodic) or 24 (even reflection about the end points, redef.f:245-279).
 * n must be a tstgrid size (tstgrid.f90:9-13). */
typedef struct {
  int nx, ny, nz;
  double xmax, ymax, zmax;
  int npd, icon;
} he_grid_t;

/* Orsay-Trento functional: he4 and lenard4 modules (Dynamics_TDDFT/modules.f90:133-153,
 * :225-237).  core4 is the effective core after the driver's "If(Lsolid) core4='OT '" rule
 * (DFT4He3d.f90:456): "OT ", "OP " or "OTC".  h4 is the core radius the driver selects
 * (h4ot or h4op). */
typedef struct {
  char core4[4];
  double h4, eps4, sigma4;
  double cp4, cpp4, den4c, alphas, l, den0s, h2o2m4;
  int lsolid;
  double C, beta, den_m;
} he_functional_t;

/* Absorbing mask timec (DFT4He3d.f90:592-601): timec = (Lambdah*sum_axes(1+tanh((|x|-tmean)/
 * tsurf)), 1).  The device evaluates it from these parameters instead of storing the array. */
typedef struct {
  double lambdah, txmean, txsurf, tymean, tysurf, tzmean, tzsurf;
} he_absorber_t;

/* Classical impurities (classicimp/interpol modules, modules.f90:303-343,386-399).  potion is the
 * (N_imp, npot) table that potenimpini builds with Select_Pot (potenimpini.f90:31-59);
 * npot = 100*max(n)+1, delinter = rmax/(npot-1), rmaxinterpol = 4*max(xmax).  ii_* is the
 * impurity-impurity pair potential used by forceimp/energy: kind 0 = null, 1 = Morse
 * D[(1-exp(-a(r-re)))^2-1] (r < ii_rcut gives ii_umax). */
typedef struct {
  int n_imp;
  const double* m_imp_u; /* n_imp masses in u; m_imp = m_imp_u * mp_u (mp_u = 0.02061484) */
  const double* potion;
  int npot;
  double delinter, rmaxinterpol;
  int ii_kind;
  double ii_D, ii_re, ii_a, ii_rcut, ii_umax;
} he_impurities_t;

/* energies module (Dynamics_TDDFT/modules.f90:39-51). */
typedef struct {
  double etot4, ekin4, elj4, ecor4, esolid, ealphas;
  double ekinx, eHeX, eimpu_impu, eimpu, etot;
} he_energies_t;

/* Field identifiers for he_upload / he_download.  Sizes in binary64 words: N = nx*ny*nz,
 * Nk = (nx/2+1)*ny*nz.  Complex fields count 2 words per point. */
enum he_field {
  HE_F_PSI = 0,      /* dynamics: complex N; statics: real N */
  HE_F_DEN = 1,      /* real N */
  HE_F_POT4 = 2,     /* real N */
  HE_F_DENCG = 3,    /* real N */
  HE_F_DELJ4 = 4,    /* real N */
  HE_F_UIMP = 5,     /* real N (dynamics) */
  HE_F_FDEN = 6,     /* complex Nk */
  HE_F_PC = 7,       /* dynamics complex N; statics real N */
  HE_F_Q = 8,        /* dynamics complex N; statics real N */
  HE_F_PSIOLD1 = 9,  /* psiold(:,:,:,1..3), same type as psi */
  HE_F_PSIOLD2 = 10,
  HE_F_PSIOLD3 = 11,
  HE_F_HPSIOLD1 = 12, /* hpsiold(:,:,:,1..2) */
  HE_F_HPSIOLD2 = 13,
  HE_F_DXDEN = 14,   /* real N, materialised by he_derden */
  HE_F_DYDEN = 15,
  HE_F_DZDEN = 16,
  HE_F_HPSI = 17,    /* statics real N */
  HE_F_FVLJ4 = 18,   /* real Nk */
  HE_F_WCGK = 19,    /* real Nk */
  HE_F_RIMP = 20,    /* (N_imp,3) */
  HE_F_VIMP = 21,
  HE_F_AIMP = 22,
  HE_F_FIMP = 23,    /* F(N_imp,3) */
  HE_F_RIMPOLD = 24, /* (N_imp,3,3) */
  HE_F_VIMPOLD = 25, /* (N_imp,3,3) */
  HE_F_AIMPOLD = 26, /* (N_imp,3,2) */
  HE_F_PCR = 27,     /* (N_imp,3) */
  HE_F_PCV = 28,
  HE_F_QR = 29,
  HE_F_QV = 30,
  HE_F_RING = 31,    /* 13 ints as doubles: ioldp(3), ioldh(2), ioldr(3), ioldv(3), iolda(2);
                        HE_MODE_QUANTUM: ioldp(3), ioldh(2) (ioldpx/ioldhx hold the same values) */
  /* HE_MODE_QUANTUM (quantal_imp / rkpc modules, Dynamics_quantum_impurities/modules.f90:280-314) */
  HE_F_PSIX = 32,     /* psix(nx,ny,nz,N_imp) complex */
  HE_F_UPOTX = 33,    /* upotx(nx,ny,nz,N_imp) real */
  HE_F_POTX4 = 34,    /* potx4(nx,ny,nz) real */
  HE_F_DENX = 35,     /* denx = sum_i |psix_i|^2, real N (download only) */
  HE_F_PCX = 36,      /* pcx(nx,ny,nz,N_imp) complex */
  HE_F_QX = 37,       /* qx(nx,ny,nz,N_imp) complex */
  HE_F_PSIXOLD = 38,  /* psixold(nx,ny,nz,3,N_imp) complex */
  HE_F_HPSIXOLD = 39, /* hpsixold(nx,ny,nz,2,N_imp) complex */
  HE_F_UIMPK = 40,    /* uimp_k(nx/2+1,ny,nz,N_imp) real */
  HE_F_UIMPKK = 41,   /* uimp_k_k(nx/2+1,ny,nz,N_imp,N_imp) real (zero for 'null' pairs) */
  /* core4 = 'OTC' (alphasterm module, Dynamics_TDDFT/modules.f90; term_alfa.f90) */
  HE_F_DENALF = 42,   /* real N */
  HE_F_FALFS = 43,    /* real N */
  HE_F_INTXALF = 44,  /* real N */
  HE_F_INTYALF = 45,
  HE_F_INTZALF = 46,
  HE_F_UALPHAS = 47,  /* real N */
  HE_F_KALFS = 48     /* real Nk */
};

#define HE_MAX_QIMP 4

/* A radial pair potential behind Select_Pot(selec,r,r_cutoff,umax)'s contract
 * (V_impur.f90:90-2152; r < r_cutoff gives umax).  kind 0 = 'null' (zero beyond r_cutoff),
 * 1 = Morse D[(1-exp(-a(r-re)))^2-1] (no counterpart in the reference's table). */
typedef struct {
  int kind;
  double D, re, a, rcut, umax;
} he_pairpot_t;

/* Quantum impurities: the namelist /imp/ of Dynamics_quantum_impurities/DFT4He3d.f90:160-162 and
 * potenimpini's kernels (potenimpini.f90:116-163). */
typedef struct {
  int n_imp;                                   /* 1..HE_MAX_QIMP */
  const double* m_imp_u;                       /* masses in u (n_imp) */
  double mu4;                                  /* H psi uses pot4 - mu4 (0 unless Lbulk) */
  he_pairpot_t he_x[HE_MAX_QIMP];              /* Selec_gs_k / r_cutoff_gs_k / umax_gs_k */
  he_pairpot_t x_x[HE_MAX_QIMP * HE_MAX_QIMP]; /* Selec_gs_k_k(i,j) at i + n_imp*j */
  const double* uimp_k;   /* optional host uimp_k (nx/2+1,ny,nz,n_imp); NULL: FT_V_spline here */
  const double* uimp_k_k; /* optional host uimp_k_k (...,n_imp,n_imp); NULL: FT_V_spline here */
  int n_spline;           /* N_FT_V_spline (FT_V_spline.f90:2); 0 = 100001 */
  int nq;                 /* Nq (modules.f90:165); the transform uses max(10001, nq) momenta */
  int parabolic;          /* Lparabolic_fit_FT_V_spline */
} he_qimpurities_t;

/* Context life cycle.  Replaces the allocations of dimen.f90 and the plans of fftini
 * (Dynamics_TDDFT/fft.f90:5-91).  mode: HE_MODE_DYNAMICS (complex psi, Dynamics_TDDFT) or
 * HE_MODE_STATICS (real psi, He_statics).  All device memory is allocated here.  *out is set
 * whenever it is non-NULL, also on failure (so he_last_error can be read); destroy it. */
int he_ctx_create(const he_grid_t* grid, const he_functional_t* fun, int mode, int precision,
                  he_ctx_t** out);
void he_ctx_destroy(he_ctx_t* ctx);
const char* he_last_error(const he_ctx_t* ctx);
/* Number of kernel launches this context has issued (all of them hand-written CUDA). */
long long he_launch_count(const he_ctx_t* ctx);
/* Device bytes held by the context. */
size_t he_device_bytes(const he_ctx_t* ctx);
/* Use an external CUDA stream (cudaStream_t); NULL selects the context's own stream. */
int he_set_stream(he_ctx_t* ctx, void* stream);
int he_synchronize(he_ctx_t* ctx);
/* Orders the work this context has queued on its internal side stream (the impurity field and
 * integrator kernels of the dynamics mode) before whatever comes next on its stream, without
 * waiting on the host: the last call of a step recorded into a CUDA graph.  No counterpart in
 * the reference. */
int he_join(he_ctx_t* ctx);

/* k-space kernels.  he_set_kernels uploads host arrays computed by the reference's fforma/initcg
 * (fforma.f90:11-61, initcg.f90:32-49); kalfs may be NULL unless core4 = "OTC".
 * he_compute_kernels evaluates the same kernels on the device (fforma with its sine integral,
 * initcg, kalfs = exp(-(pi l p)^2) from DFT4He3d.f90:527-531). */
int he_set_kernels(he_ctx_t* ctx, const double* fvlj4, const double* wcgk, const double* kalfs);
int he_compute_kernels(he_ctx_t* ctx);

int he_set_absorber(he_ctx_t* ctx, const he_absorber_t* abs);
int he_set_impurities(he_ctx_t* ctx, const he_impurities_t* imp);

/* Module-array transfer.  bytes must equal the field's size (see enum he_field).  Both return
 * once the host buffer may be reused; the copy is ordered before every later call on the context
 * (field downloads and uploads wait for the device, impurity-array uploads do not). */
int he_upload(he_ctx_t* ctx, int field, const void* host, size_t bytes);
int he_download(he_ctx_t* ctx, int field, void* host, size_t bytes);

/* ---- Dynamics_TDDFT call surface ---- */
/* poten(): Dynamics_TDDFT/poten.f90:131-218 (pot4, dencg, delj4, fden from den). */
int he_poten(he_ctx_t* ctx);
/* potenimp() -> updatepoten(): potenimp.f90:1-19,83-123 (uimp from rimp).  Asynchronous; an
 * impurity outside the interpolation table raises the sticky lstopimp flag read by he_lstopimp. */
int he_potenimp(he_ctx_t* ctx);
/* lstopimp (interpol module, modules.f90:393): *flag = 1 once an impurity left the table
 * (potenimp.f90:104-109); the driver exits its loop on it (DFT4He3d.f90:895).  Synchronises. */
int he_lstopimp(he_ctx_t* ctx, int* flag);
/* forceimp(): potenimp.f90:23-67 (F from grad(den) and the impurity fields).  F may be NULL. */
int he_forceimp(he_ctx_t* ctx, double* F);
/* aimp = F/m_imp, as the driver does after forceimp (DFT4He3d.f90:571-573, :694-696). */
int he_set_accel(he_ctx_t* ctx);
/* steprk(deltat): steprk.f90:1-144.  steppc(deltat,errHe,errimp,errvimp): steppc.f90:1-180.
 * The error pointers may be NULL (no synchronisation). */
int he_steprk(he_ctx_t* ctx, double deltat);
int he_steppc(he_ctx_t* ctx, double deltat, double* errHe, double* errimp, double* errvimp);
/* energy(): Dynamics_TDDFT/energy.f90:107-178; statics He_statics/energy.f90:36-150. */
int he_energy(he_ctx_t* ctx, he_energies_t* out);
/* derden(): derden.f90:26-28, materialises dxden/dyden/dzden. */
int he_derden(he_ctx_t* ctx);

/* ---- Dynamics_quantum_impurities call surface (HE_MODE_QUANTUM) ----
 * he_potenimp: potenimp.f90:1-43 (fden, potx4, upotx from den and psix).  he_poten:
 * poten.f90:5-155 (pot4 with potx4; uses the fden of the last he_potenimp).  he_steprk:
 * steprk.f90:1-124; he_steppc(ctx, dt, errHe, errpsix, NULL): steppc.f90:1-157.  he_energy:
 * energy.f90:12-139 (ekinx, eHeX, eimpu_impu from the impurity wave functions). */
/* Sets the impurities and builds uimp_k / uimp_k_k: FT_V_spline's radial transform runs on the
 * device (one CTA per momentum) unless host tables are given. */
int he_set_quantum_impurities(he_ctx_t* ctx, const he_qimpurities_t* q);
/* Norm and centre of each impurity density, out[4i..4i+3] = {sum |psix_i|^2 dxyz, <x>, <y>, <z>}
 * (the per-step trajectory of Dynamics_quantum_impurities/DFT4He3d.f90:682-700).  Synchronises. */
int he_qimp_moments(he_ctx_t* ctx, double* out);
/* FT_V_spline's momentum table for one pair potential: vpp[i] = V(p = i*hp), i < n_p,
 * n_p = int(pmax/hp + 1.5), after the small-q redefinition (FT_V_spline.f90:229-258); n_spline
 * nodes for the radial spline (0 = 100001).  Context-free (allocates and frees its own device
 * memory on the current device); err[errlen] receives a message on failure. */
int he_ft_v_spline_table(const he_pairpot_t* pot, double pmax, double hp, int n_spline,
                         int parabolic, double* vpp, int n_p, char* err, size_t errlen);

/* Droplet observables the dynamics drivers print every pener steps
 * (Dynamics_TDDFT/DFT4He3d.f90:720-838 with r_cm.f90; Dynamics_quantum_impurities/DFT4He3d.f90
 * has the same): out[13] = {N = sum den dxyz, r_cm (x, y, z) = sum den r dxyz / npart,
 * <L> (x, y, z) = Re sum i conj(psi) (r - r_cm) x grad psi dxyz,
 * <Vcom> (x, y, z) = Re sum -i conj(psi) grad psi dxyz / (N mhe), mhe = 4.002572164 mp_u,
 * <r^2> (x, y, z) = sum den x^2 dxyz, ...}.  One fused pass over psi and den; synchronises.
 * Not in statics mode (real psi). */
int he_observables(he_ctx_t* ctx, int npart, double* out);

/* ---- He_statics call surface ---- */
/* The driver's per-iteration refresh (BCN4HeDFT.f90:1131-1155): derden, fftfw(den,fden),
 * dencg = fftbk(fden*wcgk), and delj4 = fftbk(fden*fvlj4) which the statics poten() recomputes
 * from that same fden until the next refresh (He_statics/poten.f90:27-31). */
int he_refresh_density(he_ctx_t* ctx);
/* evolo(0,mu4,mu4err,n4) as called once before the loop (BCN4HeDFT.f90:1050, evolo.f90:41-93). */
int he_evolo0(he_ctx_t* ctx, double* mu4, double* mu4err, int n4);
/* steprkr / steppcr (He_statics/steprkr.f90:1-96, steppcr.f90:1-108). errpc may be NULL. */
int he_steprkr(he_ctx_t* ctx, double deltat, double* mu4, double* mu4err, int n4);
int he_steppcr(he_ctx_t* ctx, double deltat, double* mu4, double* mu4err, int n4, double* errpc);
/* niter passes of the statics loop body with Lrkpc and ppot = 1 (BCN4HeDFT.f90:1120-1160):
 * steppcr, derden, fftfw(den,fden), dencg, poten -- what he_steppcr, he_refresh_density and
 * he_poten called niter times do, with the host reading the sums once at the end instead of
 * after every pass (the reference reads mu4 only where it prints, every pener iterations).
 * mu4, mu4err and errpc (may be NULL) are those of the last pass.  The passes run as CUDA
 * graphs, one per buffer relabelling (the ring repeats after 30 passes), captured on first use
 * after one eager pass and dropped when the k-space kernels or FFT variants change; with
 * he_timing on they run eagerly.  No counterpart call in the reference: it replaces the loop
 * body between two energy evaluations. */
int he_statics_iterations(he_ctx_t* ctx, int niter, double deltat, double* mu4, double* mu4err, int n4,
                          double* errpc);
/* varmu(npart,mu,errmu): He_statics/varmu.f90:31. */
int he_varmu(he_ctx_t* ctx, int npart, double mu, double* errmu);

/* ---- per-kernel timing (CUDA events on the context's stream) ---- */
/* The reference only times whole runs (Dynamics_TDDFT/DFT4He3d.f90:662-664,905-911; timer.f90);
 * these calls add per-kernel device times.  he_timing(ctx,1) clears and starts recording,
 * he_timing(ctx,0) stops; he_timing_report aggregates by kernel (synchronises). */
typedef struct {
  char name[40];
  long long launches;
  double ms;
} he_kernel_time_t;
int he_timing(he_ctx_t* ctx, int enable);
/* Tile sizes (lines per CTA, 16 or 8) the context's autotuner chose for the x, y and z FFT
 * passes at creation. */
int he_tuned_tiles(const he_ctx_t* ctx, int* x, int* y, int* z);
/* Text report of the FFT-pass autotuner's trials (one line per variant with its time per pass
 * and the x-pass variant chosen), NUL-terminated and truncated to len bytes.  No counterpart in
 * the reference (FFTW plans are fixed by fftini). */
int he_autotune_report(const he_ctx_t* ctx, char* buf, size_t len);
/* Overrides the autotuner's choice for one pass family (reproducible runs, tests): pass 0 = x
 * (variant 0 one-shot, 1 persistent pipelined; every mode), 1 = y (variant 1, the register
 * transform), 2 = z (variant 0 shared-memory Stockham, 1 register transform),
 * 3 + m = the x pass of one mode m only (0 R2C of den, 1 R2C of the statics correlation source,
 * 2 C2R of two spectra, 3 the same plus the correlation R2C, 4 C2R + pot4, 5 C2R of one
 * spectrum), 9 = the classical field evaluation with fused x-y plane passes (variant 1) or
 * separate passes (0; HE_PREC_MIXED, nx = ny in {64, 96, 128}, tile ignored but checked),
 * 10 = the convolutions with the y and z passes fused in one launch per convolution over a
 * thread-block cluster (variant 1) or as separate passes (0; ny = nz = 64, tile ignored but
 * checked);
 * tile = 8 or 16 lines.  HE_ERR_ARG for a variant this grid or precision does not have.  No
 * counterpart in the reference. */
int he_set_fft_variant(he_ctx_t* ctx, int pass, int variant, int tile);
/* A hash of the host-side state a step's launches depend on besides the arrays' contents: which
 * buffer currently plays psi, psiold, hpsiold, the scratch (and the impurity wave functions'
 * counterparts), the ring indices and the lazy-evaluation flags.  Steps issued from states with
 * equal fingerprints launch the same kernels on the same buffers, so a caller that records steps
 * into CUDA graphs can replay them once the fingerprint cycles back (the relabelling is
 * periodic).  No counterpart in the reference. */
int he_state_fingerprint(const he_ctx_t* ctx, unsigned long long* out);
int he_timing_report(he_ctx_t* ctx, he_kernel_time_t* out, int max, int* n);

/* ---- groups: several statics droplets or quantum-impurity trajectories, one launch per kernel ----
 * No counterpart in the reference (its drivers run one droplet per process).  he_ctx_group makes
 * ctxs[0] the leader of n contexts created alike (same mode, precision, grid, functional and
 * impurity masses; binary64 statics or quantum-impurity mode, OT or OP core), each set up on its own (uploads, he_set_kernels or
 * he_compute_kernels) and in the same ring state.  From then on every routine called on the
 * leader launches each kernel once with a grid dimension over the members, and every member's
 * CTAs work on that member's buffers (the quantum-impurity mode groups too, in either precision:
 * the members there are trajectories, e.g. with different impurity kicks); the members' contexts must stay alive and must not be
 * called directly until the leader is destroyed.  Scalars the leader's routines return are
 * member 0's; the *_members calls below return every member's, and he_upload_member /
 * he_download_member move member m's module arrays (m = 0 is the leader).  Routines outside the
 * statics loop of BCN4HeDFT.f90:1113-1160 (and energy, varmu) return HE_ERR_STATE in a group. */
int he_ctx_group(he_ctx_t* const* ctxs, int n);
/* Number of members the context leads (1 outside a group). */
int he_group_size(const he_ctx_t* ctx);
int he_upload_member(he_ctx_t* ctx, int member, int field, const void* host, size_t bytes);
int he_download_member(he_ctx_t* ctx, int member, int field, void* host, size_t bytes);
/* mu4[m] of each member as the last statics routine returns it for member 0: after he_steppcr or
 * he_evolo0 (after_rk = 0) sum(psi H psi) dxyz / n4 of the last H psi reduction, after
 * he_steprkr (after_rk = 1) that of its first stage. */
int he_member_mu(he_ctx_t* ctx, int n4, int after_rk, double* mu4);
/* he_statics_iterations for every member: mu4, mu4err (and errpc) are arrays of he_group_size
 * values; mu4 carries each member's previous value in (used when niter = 1). */
int he_statics_iterations_members(he_ctx_t* ctx, int niter, double deltat, int n4, double* mu4,
                                  double* mu4err, double* errpc);
/* energy() of every member into out[he_group_size(ctx)] (statics and quantum groups). */
int he_energy_members(he_ctx_t* ctx, he_energies_t* out);
/* he_qimp_moments of every member: out[4 (m nq + i) + 0..3] = norm, <x>, <y>, <z> of member m's
 * impurity i. */
int he_qimp_moments_members(he_ctx_t* ctx, double* out);

/* ---- energy sums without device allocation ----
 * No counterpart in the reference.  For callers that cannot let a library allocate device
 * memory because all of it belongs to them (a Fortran driver whose arrays live in OpenACC or
 * CUDA Fortran data regions sized at start-up, a job that reserves the GPU's memory in its own
 * pool): computes energy()'s He sums (ekin4, elj4, ecor4, esolid, etot4, and eHeX when uimp is
 * given) from the caller's device arrays psi (complex in HE_MODE_DYNAMICS, real in
 * HE_MODE_STATICS), den, dencg, delj4 and uimp (may be NULL), in the reference layout.  Calls no
 * cudaMalloc/cudaFree: the reduction scratch is a fixed 328,000-byte device array inside the
 * library (room for 8192 reduction blocks of 32x8x16 points: grids up to 256^3, which need 4096;
 * larger grids return HE_ERR_ARG), held on every GPU that loads the library until exit.  Each
 * call looks up that array's address on the current device; the first call on a device may load
 * the library's device code, so make it before any stream capture.  All calls share the array:
 * calls whose work overlaps on the GPU race.  core4 must be "OT " or "OP " (HE_ERR_ARG for "OTC",
 * whose etot4 includes the alpha_s energy, and for anything else).  Synchronises `stream` (cudaStream_t, NULL = default);
 * fills *out (impurity fields other than eHeX/eimpu are zero); on error writes a message to
 * err[errlen] when given. */
int he_energy_noalloc(const he_grid_t* grid, const he_functional_t* fun, int mode,
                      const void* psi, const double* den, const double* dencg,
                      const double* delj4, const double* uimp, void* stream,
                      he_energies_t* out, char* err, size_t errlen);

#ifdef __cplusplus
}
#endif
#endif /* HE_DFT_H */
