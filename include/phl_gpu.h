/*
 * phl_gpu.h -- C ABI of the B200 implementation of Phlegethon's explicit finite-volume step.
 *
 * The reference (source/source.F90, Fortran) has no plugin API: its seam is the pair of
 * module subroutines that time_loop calls on the whole local grid,
 *   hydro_step(mgrid, lgrid)             source/source.F90:6683  (defined 6847-13701)
 *   compute_hyperbolic_dt(mgrid, lgrid)  source/source.F90:6388, 6716 (defined 13707-13960)
 * plus the step-0 thermodynamics loop of time_loop (source/source.F90:6271-6383) and the table
 * reader load_helm_table (source/source.F90:23077-23156).  This header exports those entry points
 * with plain pointers and sizes so the Fortran driver can bind them with ISO_C_BINDING
 * (`bind(C)` interfaces).  Host arrays use the reference's own layout
 * (column-major, variable index fastest, ghost cells included, bounds of
 * initialize_simulation, source/source.F90:1219-1714); the library transposes them into its
 * device layout.
 *
 * Conventions: every function returns 0 (PHL_OK) or a negative PHL_E* code; no exception
 * crosses the ABI; device-side failures (Newton non-convergence, non-finite values) are
 * latched in a status word read by phl_get_status and never trap.  One context drives one GPU
 * on one stream and is not thread-safe, like the single-threaded caller it replaces.
 */
#ifndef PHL_GPU_H
#define PHL_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

#define PHL_ABI_VERSION 4

/* return codes */
#define PHL_OK 0
#define PHL_E_INVALID (-1)      /* bad argument or unsupported option combination */
#define PHL_E_CUDA (-2)         /* CUDA runtime error (allocation, launch, copy) */
#define PHL_E_NO_TABLE (-3)     /* Helmholtz EoS selected but no table loaded */
#define PHL_E_STATE (-4)        /* call out of order (e.g. step before upload) */
#define PHL_E_NO_DEVICE (-5)    /* no CUDA device / wrong architecture */
#define PHL_E_UNSUPPORTED (-6)  /* option recognised but not built */
#define PHL_E_TOO_LARGE (-7)    /* request beyond a fixed capacity */

/* Riemann solvers: compile-time options LHLLC_FLUX, HLLC_FLUX, HLLD_FLUX, LHLLD_FLUX */
#define PHL_LHLLC 0
#define PHL_HLLC 1
#define PHL_HLLD 2
#define PHL_LHLLD 3

/* boundary kinds: X?_PERIODIC, X?L_REFLECTIVE / X?U_REFLECTIVE */
#define PHL_BC_PERIODIC 0
#define PHL_BC_REFLECTIVE 1

/* option bits (the reference's compile-time -D flags) */
#define PHL_MHD (1 << 0)              /* USE_MHD */
#define PHL_WB (1 << 1)               /* USE_WB */
#define PHL_GRAVITY (1 << 2)          /* USE_GRAVITY (constant external field) */
#define PHL_EVOLVE_ETOT (1 << 3)      /* EVOLVE_ETOT */
#define PHL_HELMHOLTZ (1 << 4)        /* HELMHOLTZ_EOS */
#define PHL_FASTEOS (1 << 5)          /* USE_FASTEOS */
#define PHL_ADVECT_YE_IABAR (1 << 6)  /* ADVECT_YE_IABAR */
#define PHL_SHOCK_FLATTENING (1 << 7) /* USE_SHOCK_FLATTENING (ngc >= 3) */
#define PHL_FLUX_IS_ALL_MACH (1 << 8) /* FLUX_IS_ALL_MACH (LHLLC/LHLLD: upwind states outside the fan) */
#define PHL_CONSTANT_ACCELERATION (1 << 9) /* USE_CONSTANT_ACCELERATION with phl_config.acc */

/* arithmetic of the flux path */
#define PHL_FP64 0        /* FP64 throughout, bit-compatible with the reference order */
#define PHL_FP32_SPLIT 1  /* FP32 reconstruction/Riemann/EMF on WB deviations, FP64 state + EoS */

/* reconstruction (phl_config.reconstruction) */
#define PHL_REC_LIM2ND 0  /* LIM2ND_REC: van Leer PLM (source.F90:8141-8181) */
#define PHL_REC_PPH 1     /* PPH_REC: third order, scalars limited (source.F90:8183-8259) */
#define PHL_REC_LIM5TH 2  /* LIM5TH_REC: limited fifth order (source.F90:8261-8323) */

/* initial temperature guess for the (rho, e) -> T Newton inversion */
#define PHL_GUESS_WARM 0  /* previous-stage temperature, as the reference (source.F90:13649) */
#define PHL_GUESS_MLP 1   /* learned 4-64-64-1 guess, judged by <=3 Newton steps, else the
                                     warm guess (hydro step) or the bracket guess (EoS batch) */
#define PHL_GUESS_BRACKET 2 /* EoS batch only: cold guess from the table nodes bracketing e(rho, T)
                               at fixed rho*Ye (monotone search in T); T_inout is not read */
#define PHL_GUESS_MLP_RESCUE 3 /* hydro step only: the warm guess, and for every cell whose first
                                  warm Newton correction exceeds 2% of T the learned guess
                                  (judged as PHL_GUESS_MLP, the warm guess as its fallback) */

typedef struct phl_config {
  int abi_version;                 /* must be PHL_ABI_VERSION */
  int sdims;                       /* 2 or 3 (sdims_make) */
  int nx1, nx2, nx3;               /* global cells (nx?_make); nx3 = 1 in 2D */
  int ngc;                         /* ghost layers of the host arrays (ngc_make, 2 for PLM) */
  int nas;                         /* advected scalars (nas_make) */
  int nvars;                       /* 2 + sdims + nas */
  int flags;                       /* PHL_MHD | PHL_WB | ... */
  int riemann;                     /* PHL_LHLLC ... */
  int rk_stages;                   /* 2 (RK2_STEPPER) or 3 (RK3_STEPPER) */
  int bc[3][2];                    /* [dim][0 lower, 1 upper] PHL_BC_* */
  int precision;                   /* PHL_FP64 or PHL_FP32_SPLIT */
  int eos_guess;                   /* PHL_GUESS_WARM, or PHL_GUESS_MLP / PHL_GUESS_MLP_RESCUE for
                                      the learned guess in the step's Newton (FP32 split MHD form
                                      with the Helmholtz EoS; train or set the network before the
                                      first step) */
  int device;                      /* CUDA device ordinal */
  double x1l, x1u, x2l, x2u, x3l, x3u;
  double gamma_ad, mu;             /* initialize_simulation arguments */
  double cfl, mach_cutoff, mach_ct;/* cfl_make, Mach_cutoff_make, Mach_ct_make */
  int helm_nT, helm_nrho;          /* helm_nT_make, helm_nrho_make */
  double helm_ltlo, helm_lthi, helm_ldlo, helm_ldhi;
  int reconstruction;              /* PHL_REC_LIM2ND (LIM2ND_REC), PHL_REC_PPH, PHL_REC_LIM5TH
                                      (ngc >= 3) */
  double eps_sf;                   /* eps_sf_make (reference default 0.25): a cell whose summed
                                      central pressure jumps exceed eps_sf * p flags itself and
                                      its neighbours; read with PHL_SHOCK_FLATTENING */
  double acc[3];                   /* lgrid%acc (source.F90:965): body acceleration of
                                      USE_CONSTANT_ACCELERATION (cm/s^2; acc[2] unused in 2D) */
} phl_config;

/* Host arrays, laid out exactly as the locgrid members of the same name
 * (source/source.F90:839-1130).  Unused members may be NULL. */
typedef struct phl_fields {
  double *prim;            /* prim(1:nvars, lx1-ngc:ux1+ngc, lx2-ngc:ux2+ngc, lx3[-ngc]:ux3[+ngc]) */
  double *temp, *eint;     /* (lx1-ngc:ux1+ngc, ...) */
  double *gammaf;          /* gammaf(1:2, ...)            USE_FASTEOS */
  double *grav;            /* grav(1:sdims, ...)          USE_GRAVITY */
  double *phi_cc;          /* phi_cc(...)                 EVOLVE_ETOT */
  double *eq_prim_cc;      /* eq_prim_cc(1:3, ...)        USE_WB */
  double *eq_gammae_cc;    /* eq_gammae_cc(...)           USE_WB + USE_FASTEOS */
  double *b_cc;            /* b_cc(1:sdims, ...)          USE_MHD */
  double *phi_x[3];        /* phi_x1(lx1:ux1+1, lx2:ux2, lx3:ux3), ... */
  double *eq_prim_x[3];    /* eq_prim_x1(1:3, lx1:ux1+1, lx2:ux2, lx3:ux3), ... */
  double *eq_gammae_x[3];  /* eq_gammae_x1(lx1:ux1+1, ...), ... */
  double *b_x[3];          /* b_x1(lx1-1:ux1+2, lx2-1:ux2+1, lx3-1:ux3+1), ... (2D: lx3:ux3) */
} phl_fields;

typedef struct phl_status {
  long long newton_calls;         /* (rho,e)->T inversions since the last reset */
  long long newton_iterations;    /* total Newton iterations */
  long long newton_nonconverged;  /* inversions that used all 100 iterations */
  long long newton_clamped;       /* iterates that left [Tl_eos, Th_eos] and were reset */
  long long mlp_accepted;         /* MLP guesses that converged within 3 iterations */
  long long mlp_rejected;         /* MLP guesses that fell back to the warm/bracket guess */
  long long nonfinite;            /* non-finite or non-positive rho/p/T produced */
  long long guess_evaluations;    /* EoS evaluations spent building initial guesses (bracket
                                     search, cold energy of the learned guess's input) */
  long long tensor_core_stalls;   /* asynchronous operations (tensor-core products, bulk tensor
                                     copies) that did not complete within the poll limit */
  long long steps;                /* steps taken by this context */
  double time, dt, smax;
} phl_status;

typedef struct phl_ctx phl_ctx;

/* version and last-error text */
int phl_abi_version(void);
const char *phl_error_string(int code);

/* initialize_simulation equivalent for the device side: allocate the device-resident domain.
 * (source/source.F90:1150-1883) */
int phl_init(const phl_config *cfg, phl_ctx **ctx);
void phl_finalize(phl_ctx *ctx);

/* load_helm_table (source/source.F90:23077-23156): tables in helm_table_var(1:9,1:nrho,1:nT)
 * and dpdrho_table_var(1:4,1:nrho,1:nT) layout.  Node arrays are rebuilt from the
 * helm_* range parameters exactly as the reference does. */
int phl_load_helm_table(phl_ctx *ctx, const double *helm_table_var, const double *dpdrho_table_var);

/* Copy the reference-layout host arrays to the device (static background and dynamic state). */
int phl_upload_state(phl_ctx *ctx, const phl_fields *host);
/* Copy the dynamic state back (prim interior+ghost layout, temp, eint, gammaf, b_cc, b_x*).
 * Ghost cells of the host arrays are left untouched.  Called before write_output /
 * write_restart (source/source.F90:6583, 6638, 6752, 6822). */
int phl_download_state(phl_ctx *ctx, phl_fields *host);

/* Step-0 thermodynamics of time_loop (source/source.F90:6271-6383): eint, temp, gammaf from
 * (rho, p, temp guess); for MHD also b_cc from the face fields (source/source.F90:6012-6062). */
int phl_init_thermo(phl_ctx *ctx);

/* compute_hyperbolic_dt (source/source.F90:13707-13960).  Outputs may be NULL. */
int phl_compute_hyperbolic_dt(phl_ctx *ctx, double *dt, double *smax);

/* hydro_step (source/source.F90:6847-13701) with the context's current dt. */
int phl_hydro_step(phl_ctx *ctx);

/* dt and time held by the context (lgrid%dt, lgrid%time, lgrid%smax) */
int phl_set_time(phl_ctx *ctx, double time, double dt, double smax);
int phl_get_time(phl_ctx *ctx, double *time, double *dt, double *smax);

/* The body of time_loop's do-while without output (source/source.F90:6525-6748): for up to
 * nsteps steps while time < tmax: clamp dt to tmax (6662-6664), hydro_step, time += dt,
 * compute_hyperbolic_dt.  Runs asynchronously on the device as CUDA graphs; returns after the
 * last step has finished.  steps_done/time may be NULL. */
int phl_run_steps(phl_ctx *ctx, int nsteps, double tmax, int *steps_done, double *time);

/* Host-resident state, asynchronous: upload the dynamic state from `host` (prim, temp, eint,
 * gammaf, b_cc, b_x, laid out as for phl_upload_state; background members are not read),
 * advance exactly nsteps steps of time_loop (no tmax clamp), and download the dynamic state back
 * into the same arrays -- all queued on the context's streams; the call returns without waiting.
 * The whole arrays travel up (contiguous copies) and their interiors come down; the ghost
 * layers are neither read by the step nor written.
 * This is the per-step exchange of a driver that keeps its state in host memory (the reference's
 * own arrays) and wants the copies off the critical path: the upload of each chunk of host
 * planes waits only for the previous call's download of the same planes, so the two PCIe
 * directions overlap across consecutive calls.  Host arrays must be page-locked for the copies
 * to run asynchronously (pageable memory works but serialises them) and must not be touched
 * until phl_wait_host returns.  The context must have been set up by phl_upload_state (with the
 * background) and phl_compute_hyperbolic_dt first.  Every other entry point waits for pending
 * downloads before it starts.  No counterpart in the reference (its state never leaves the
 * host); the step it runs is hydro_step + compute_hyperbolic_dt as in phl_run_steps. */
int phl_run_steps_host_async(phl_ctx *ctx, phl_fields *host, int nsteps);
/* Block until every queued phl_run_steps_host_async call has written its results to host memory. */
int phl_wait_host(phl_ctx *ctx);

int phl_get_status(phl_ctx *ctx, phl_status *st);
int phl_reset_status(phl_ctx *ctx);

/* ---- Helmholtz (rho, e) -> T batch inversion (helm_rhoe_given, source/source.F90:24982-25019)
 * on n independent samples.  Pointers are device pointers.  T_inout holds the initial guess
 * for PHL_GUESS_WARM and receives the converged temperature.  p, cs, iters may be NULL. */
int phl_eos_invert_batch_device(phl_ctx *ctx, long long n, const double *rho, const double *e,
                                const double *abar, const double *zbar, double *T_inout,
                                double *p, double *cs, int *iters, int guess);
/* Same with host pointers (copies in and out included). */
int phl_eos_invert_batch(phl_ctx *ctx, long long n, const double *rho, const double *e,
                         const double *abar, const double *zbar, double *T_inout, double *p,
                         double *cs, int *iters, int guess);
/* Same as phl_eos_invert_batch, but allocates no device memory: the device copies of the
 * inputs and outputs live in one fixed array compiled into the library.  No counterpart in the
 * reference.  For callers that cannot call cudaMalloc during a run: a Fortran or C driver that
 * hands all free device memory to its own pool allocator at start-up (a cudaMalloc would then
 * fail), or one whose time loop must not allocate because cudaMalloc/cudaFree can synchronise
 * the whole device and stall the step pipeline.
 * At most PHL_NOALLOC_MAX_SAMPLES samples per call; larger n returns PHL_E_TOO_LARGE and does
 * nothing.  The first call on each device looks up the array's device address (a one-time,
 * thread-safe set-up): make that first call before any stream capture.  The array is shared by
 * every call and every context on a device and stays allocated until the process exits; it
 * keeps the last call's contents, and calls that overlap on the GPU race, so issue them one
 * after another.  Host pointers; copies in and out are included, and the call returns after
 * its results have reached the host. */
#define PHL_NOALLOC_MAX_SAMPLES 65536
int phl_eos_invert_batch_noalloc(phl_ctx *ctx, long long n, const double *rho, const double *e,
                                 const double *abar, const double *zbar, double *T_inout, double *p,
                                 double *cs, int *iters, int guess);
/* Forward EoS e(rho, T) on device pointers (helm_rhoT_given2 without dE/dT). */
int phl_eos_energy_device(phl_ctx *ctx, long long n, const double *rho, const double *T,
                          const double *abar, const double *zbar, double *e);

/* ---- learned temperature guess: MLP 4-64-64-1 (log10 rho, log10 e, Abar, Zbar -> log10 T),
 * BF16 weights with FP32 accumulation on the tensor cores.  No reference counterpart. */
#define PHL_MLP_NPARAMS (4 * 64 + 64 + 64 * 64 + 64 + 64 + 1)
/* Sample n (rho, T, Abar, Zbar) points from the sample range (phl_mlp_set_sample_range) with a
 * counter-based RNG (seed), evaluate e with the EoS, and train for `epochs` passes with Adam.
 * final_loss may be NULL.  Everything runs on the device with the project's own kernels. */
int phl_mlp_train(phl_ctx *ctx, long long n, unsigned long long seed, int epochs, int batch,
                  double lr, double *final_loss);
/* Range the training samples are drawn from, uniform in each coordinate: lo/hi[0] log10 rho,
 * [1] log10 T (inside the table), [2] Abar, [3] Zbar (1 <= lo <= hi); lo[k] == hi[k] fixes a
 * coordinate.  lo == NULL restores the default: log10 rho in [-2, 9], log10 T in [4, 10], Abar
 * in [1, 56], Zbar in [1, max(Abar/2, 1)].  A network trained on the range of the states a run
 * holds guesses them closer.  Takes effect at the next phl_mlp_train. */
int phl_mlp_set_sample_range(phl_ctx *ctx, const double *lo, const double *hi);
/* One gradient evaluation of the mean-squared loss on n training pairs (host pointers:
 * features n x 4 FP32, targets n FP32 in the network's output units), with the current
 * parameters; n must be a multiple of 64.  grad receives PHL_MLP_NPARAMS floats; loss may be NULL. */
int phl_mlp_gradient(phl_ctx *ctx, long long n, const float *features, const float *targets, float *grad,
                     double *loss);
/* FP32 master weights in the order W1(64x4), b1(64), W2(64x64), b2(64), W3(1x64), b3(1). */
int phl_mlp_get_params(phl_ctx *ctx, float *params);
int phl_mlp_set_params(phl_ctx *ctx, const float *params);
/* Inference log10 T = MLP(features) for n samples (device pointers, features n x 4 FP32). */
int phl_mlp_infer_device(phl_ctx *ctx, long long n, const float *features, float *out);

/* ---- raw device access for callers that keep their own device buffers (e.g. PyTorch).
 * Returns the device pointer of a named SoA field ("prim", "U", "temp", ...) or NULL. */
void *phl_device_field(phl_ctx *ctx, const char *name);
/* The CUDA stream (cudaStream_t) all work of the context runs on. */
void *phl_stream(phl_ctx *ctx);

#ifdef __cplusplus
}
#endif
#endif
