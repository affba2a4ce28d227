/*
 * phl_oracle.h -- CPU restatement of Phlegethon's explicit finite-volume step.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA path and the timed
 * CPU baseline in bench.py.  Nothing in the product (phlegethon_b200/) links or calls it.
 *
 * Parity status: UNPINNED against the reference's own execution.  The reference
 * (source/source.F90, Fortran 2003 + MPI + HDF5) cannot be compiled in this container or
 * on the GPU box (no gfortran/mpifort), and its tests are compile-only
 * (.github/workflows/build.yml:22-37) with no golden vectors.  The restatement is pinned
 * instead by known-answer tests (exact solutions, conservation, symmetries of the step,
 * thermodynamic identities, EoS round trips) and by an independent vectorised numpy
 * restatement, read from the Fortran separately (tests/numpy_restatement.py,
 * tests/numpy_restatement_eos.py), of every step option this library implements and of the
 * Helmholtz evaluation and inversions, which equals it bit for bit.
 *
 * Every routine follows the reference's operation order (including the parenthesisation of
 * long sums) so that an FMA-free double build reproduces it bit for bit.  Arrays use the
 * reference's own layout: Fortran column-major, variable index fastest, ghost cells included,
 * bounds as allocated in initialize_simulation (source/source.F90:1219-1714).
 */
#ifndef PHL_ORACLE_H
#define PHL_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Riemann solver selection (compile-time options LHLLC_FLUX/HLLC_FLUX/HLLD_FLUX/LHLLD_FLUX). */
enum { PHLO_LHLLC = 0, PHLO_HLLC = 1, PHLO_HLLD = 2, PHLO_LHLLD = 3 };
/* Boundary kinds per face (X?L_/X?U_ options, X?_PERIODIC). */
enum { PHLO_BC_PERIODIC = 0, PHLO_BC_REFLECTIVE = 1 };

/* Helmholtz table (load_helm_table, source/source.F90:23077-23156). */
typedef struct phlo_helm {
  int nT, nrho;
  double ltlo, lthi, ldlo, ldhi;
  double drho, dT;        /* log10 spacings (source.F90:23091-23092) */
  double *tab;            /* helm_table_var(1:9, 1:nrho, 1:nT), Fortran order */
  double *dpdr;           /* dpdrho_table_var(1:4, 1:nrho, 1:nT) */
  double *rho;            /* helm_rho(1:nrho) = 10**(ldlo+(i-1)*drho) */
  double *T;              /* helm_T(1:nT) */
  double Tl, Th;          /* Tl_eos = 10**ltlo, Th_eos = 10**lthi (source.F90:750-751) */
} phlo_helm;

/* Grid state mirroring the subset of `locgrid` (source/source.F90:839-1130) that the
 * explicit step touches, with the same array shapes.  All pointers are owned by the caller. */
typedef struct phlo_grid {
  /* compile-time options of the reference, as run-time fields */
  int sdims, nx1, nx2, nx3, ngc, nas, nvars;
  int mhd, wb, gravity, etot, helm, fasteos;
  int rec;                /* reconstruction: 0 LIM2ND_REC, 1 PPH_REC, 2 LIM5TH_REC (ngc >= 3) */
  int sf;                 /* USE_SHOCK_FLATTENING (ngc >= 3) */
  int all_mach;           /* FLUX_IS_ALL_MACH: upwind L/R states outside the wave fan (LHLLC, LHLLD) */
  int use_acc;            /* USE_CONSTANT_ACCELERATION with acc */
  double acc[3];
  int riemann, rk_stages;
  int bc[3][2];           /* [dim][lower/upper] */
  double gm, mu, cfl, mach_cutoff, mach_ct;
  double eps_sf;          /* eps_sf_make: pressure-jump threshold of the shock detector */
  double dx1, dx2, dx3, inv_dx1, inv_dx2, inv_dx3;
  double dt, smax, time;
  const phlo_helm *eos;
  int nthreads;           /* OpenMP threads for the sweeps (0 = runtime default) */

  /* cell arrays with ngc ghosts (2D: x3 has no ghosts) */
  double *prim;           /* (nvars, ...) */
  double *temp, *eint;
  double *gammaf;         /* (2, ...)  USE_FASTEOS */
  double *grav;           /* (sdims, ...) USE_GRAVITY */
  double *phi_cc;         /* EVOLVE_ETOT */
  double *eq_prim_cc;     /* (3, ...) USE_WB */
  double *eq_gammae_cc;   /* USE_WB+USE_FASTEOS */
  double *b_cc;           /* (sdims, ...) USE_MHD */
  /* face arrays without ghosts: x1 faces (nx1+1, nx2, nx3) etc. */
  double *phi_x[3];
  double *eq_prim_x[3];   /* (3, faces) */
  double *eq_gammae_x[3];
  /* face B with one ghost layer: b_x1(lx1-1:ux1+2, lx2-1:ux2+1, lx3-1:ux3+1) etc. */
  double *b_x[3];
  /* scratch owned by the caller, sized by phlo_scratch_doubles() */
  double *scratch;
} phlo_grid;

/* ---- Helmholtz EoS (source/source.F90:23686-25019) ---- */
void phlo_helm_setup_nodes(phlo_helm *h);   /* fills rho, T, drho, dT, Tl, Th */
void phlo_helm_rhoT_given_full(const phlo_helm *h, double rho, double T, double abar, double zbar,
                               double *P, double *E, double *sound, double *cv);
void phlo_helm_rhoT_given1(const phlo_helm *h, double rho, double T, double abar, double zbar,
                           double *P, double *dPdT, int return_dPdT);
void phlo_helm_rhoT_given2(const phlo_helm *h, double rho, double T, double abar, double zbar,
                           double *E, double *dEdT, int return_dEdT);
/* Newton inversions; return the iteration count used (<=100). */
/* per-face helm_rhoP_given calls and iterations since the last reset (test statistics) */
void phlo_face_newton_stats(long long *calls, long long *iters, int reset);
int phlo_helm_rhoP_given(const phlo_helm *h, double rho, double P0, double abar, double zbar,
                         double *T, double *E, double *sound, int return_sound);
int phlo_helm_rhoe_given(const phlo_helm *h, double rho, double E0, double abar, double zbar,
                         double *T, double *P, double *sound, int return_sound);

/* Cold initial guess for the (rho, e) -> T inversion of independent samples (no reference
 * counterpart; the reference always has a warm start): bisection over the table's T nodes for
 * E(rho, T_j) <= e, then linear interpolation of E between the bracketing nodes.  Returns the
 * EoS evaluations used. */
int phlo_eos_bracket_guess(const phlo_helm *h, double rho, double e, double abar, double zbar, double *T);
/* Batch inversion with helm_rhoe_given's Newton (guess 0: T holds the warm start; guess 2: the
 * bracket guess); T receives the result, iters (may be NULL) the Newton iterations.  OpenMP over
 * nthreads (0 = all). */
void phlo_eos_invert_batch(const phlo_helm *h, long n, const double *rho, const double *e, const double *abar,
                           const double *zbar, double *T, int *iters, int guess, int nthreads);

/* ---- Riemann solvers for one face, in the normal frame (source/source.F90:13969-16260) ----
 * q*: nvars primitive face states; g*: (gammae, gammac) face values for USE_FASTEOS, the face
 * temperature guess in g*[0] for the Helmholtz EoS without USE_FASTEOS (helm_rhoP_given per
 * side), NULL otherwise; b*: 3 components (normal first), MHD only.  flat: the face is
 * flattened (USE_SHOCK_FLATTENING): HLL flux instead of the selected solver. */
void phlo_riemann_hydro(const phlo_grid *g, const double *qL, const double *qR,
                        const double *gL, const double *gR, double *flux, int flat);
void phlo_riemann_mhd(const phlo_grid *g, const double *qL, const double *qR,
                      const double *bL, const double *bR, const double *gL, const double *gR,
                      double *flux, double *fluxb, int flat);

/* ---- step-level routines ---- */
long phlo_scratch_doubles(const phlo_grid *g);
/* step-0 thermodynamics of time_loop (source/source.F90:6271-6383): eint, temp, gammaf */
void phlo_init_thermo(phlo_grid *g);
/* compute_hyperbolic_dt (source/source.F90:13707-13960): sets g->smax and g->dt */
void phlo_compute_hyperbolic_dt(phlo_grid *g);
/* hydro_step (source/source.F90:6847-13701) for one dt */
void phlo_hydro_step(phlo_grid *g);

/* Sizes of the reference arrays for a grid (number of doubles). */
long phlo_cells_ghost(const phlo_grid *g);
long phlo_faces(const phlo_grid *g, int dir);
long phlo_bface(const phlo_grid *g, int dir);

#ifdef __cplusplus
}
#endif
#endif
