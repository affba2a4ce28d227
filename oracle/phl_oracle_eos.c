/*
 * phl_oracle_eos.c -- CPU restatement of the Helmholtz EoS routines of Phlegethon.
 * TEST INFRASTRUCTURE ONLY (checker and CPU baseline); parity unpinned, see phl_oracle.h.
 *
 * Follows source/source.F90:
 *   load_helm_table nodes        23089-23104
 *   helm_rhoT_given_full         23686-24232
 *   helm_rhoT_given1             24234-24569
 *   helm_rhoT_given2             24571-24941
 *   helm_rhoP_given (Newton)     24943-24980
 *   helm_rhoe_given (Newton)     24982-25019
 * Sums keep the reference's left-to-right order term by term.  Build without FMA
 * contraction (-ffp-contract=off) to reproduce the reference bit for bit.
 */
#include <math.h>
#include <omp.h>
#include "phl_oracle.h"

/* physical constants (source/source.F90:612-629) */
#define CONST_RGAS 8.31446261815324e7
#define CONST_RAD 7.565767381646406e-15
#define CONST_C 2.99792458e10
#define CONST_C2 8.987551787368177e20
#define HELM_TOL 1.0e-11
#define EM15 1.0e-15

void phlo_helm_setup_nodes(phlo_helm *h) {
  /* source.F90:23091-23104: helm_dT, helm_drho, helm_T(j)=10**(ltlo+(j-1)*dT) */
  h->dT = (h->lthi - h->ltlo) / (double)(h->nT - 1);
  h->drho = (h->ldhi - h->ldlo) / (double)(h->nrho - 1);
  for (int j = 0; j < h->nT; ++j) h->T[j] = pow(10.0, h->ltlo + (double)j * h->dT);
  for (int i = 0; i < h->nrho; ++i) h->rho[i] = pow(10.0, h->ldlo + (double)i * h->drho);
  h->Tl = pow(10.0, h->ltlo);
  h->Th = pow(10.0, h->lthi);
}

/* table access: helm_table_var(v, ih, jh) with 1-based v, ih, jh */
#define TAB(h, v, ih, jh) ((h)->tab[((v)-1) + 9 * (((ih)-1) + (long)(h)->nrho * ((jh)-1))])
#define DPD(h, v, ih, jh) ((h)->dpdr[((v)-1) + 4 * (((ih)-1) + (long)(h)->nrho * ((jh)-1))])

/* The 36 biquintic coefficients in the reference's loc_eos1..36 order: var v=1..9, corners
 * (ih,jh), (ih+1,jh), (ih,jh+1), (ih+1,jh+1). */
static void load36(const phlo_helm *h, int ih, int jh, double c[36]) {
  for (int v = 1; v <= 9; ++v) {
    c[4 * (v - 1) + 0] = TAB(h, v, ih, jh);
    c[4 * (v - 1) + 1] = TAB(h, v, ih + 1, jh);
    c[4 * (v - 1) + 2] = TAB(h, v, ih, jh + 1);
    c[4 * (v - 1) + 3] = TAB(h, v, ih + 1, jh + 1);
  }
}

/* rho-order and T-order of each table variable (id_f, id_dfdT, id_d2fdT2, id_dfdrho,
 * id_d2fdrho2, id_d2fdrhodT, id_d3fdrho2dT, id_d3fdrhodT2, id_d4fdrho2dT2; source.F90:520-528) */
static const int ORD_R[9] = {0, 0, 0, 1, 2, 1, 2, 1, 2};
static const int ORD_T[9] = {0, 1, 2, 0, 0, 1, 1, 2, 2};

/* sum_{n=1..36} c_n * R[n] * T[n], evaluated left to right as the reference writes it */
static double sum36(const double c[36], const double r[3][2], const double t[3][2]) {
  double s = 0.0;
  int first = 1;
  for (int v = 0; v < 9; ++v) {
    for (int q = 0; q < 4; ++q) {
      double term = (c[4 * v + q] * r[ORD_R[v]][q & 1]) * t[ORD_T[v]][q >> 1];
      if (first) { s = term; first = 0; } else { s = s + term; }
    }
  }
  return s;
}

typedef struct {
  int ih, jh;
  double Ye, rhos, x, y, omx, omy, drho, dT, drho2, dT2, idrho, idrho2, idT, idT2;
  double x2, x3, x4, x5, y2, y3, y4, y5, omx2, omx3, omx4, omx5, omy2, omy3, omy4, omy5;
} cellpos;

static void locate(const phlo_helm *h, double rho, double T, double abar, double zbar, cellpos *p) {
  double tmp;
  p->Ye = zbar / abar;
  p->rhos = rho * p->Ye;
  p->ih = (int)((log10(p->rhos) - log10(h->rho[0])) / h->drho) + 1;
  p->jh = (int)((log10(T) - log10(h->T[0])) / h->dT) + 1;
  tmp = h->rho[p->ih - 1];
  p->drho = h->rho[p->ih] - tmp;
  p->x = (p->rhos - tmp) / p->drho;
  p->omx = 1.0 - p->x;
  tmp = h->T[p->jh - 1];
  p->dT = h->T[p->jh] - tmp;
  p->y = (T - tmp) / p->dT;
  p->omy = 1.0 - p->y;
  p->drho2 = p->drho * p->drho;
  p->dT2 = p->dT * p->dT;
  p->idrho = 1.0 / p->drho;
  p->idrho2 = p->idrho * p->idrho;
  p->idT = 1.0 / p->dT;
  p->idT2 = p->idT * p->idT;
  p->x2 = p->x * p->x; p->x3 = p->x2 * p->x; p->x4 = p->x3 * p->x; p->x5 = p->x4 * p->x;
  p->omx2 = p->omx * p->omx; p->omx3 = p->omx2 * p->omx; p->omx4 = p->omx3 * p->omx;
  p->omx5 = p->omx4 * p->omx;
  p->y2 = p->y * p->y; p->y3 = p->y2 * p->y; p->y4 = p->y3 * p->y; p->y5 = p->y4 * p->y;
  p->omy2 = p->omy * p->omy; p->omy3 = p->omy2 * p->omy; p->omy4 = p->omy3 * p->omy;
  p->omy5 = p->omy4 * p->omy;
}

/* quintic Hermite basis in rho (source.F90:24708-24721) */
static void basis_r(const cellpos *p, double r[3][2]) {
  double x = p->x, x2 = p->x2, x3 = p->x3, x4 = p->x4, x5 = p->x5;
  double omx = p->omx, omx2 = p->omx2, omx3 = p->omx3, omx4 = p->omx4, omx5 = p->omx5;
  r[0][0] = -6.0 * x5 + 15.0 * x4 - 10.0 * x3 + 1.0;
  r[1][0] = (-3.0 * x5 + 8.0 * x4 - 6.0 * x3 + x) * p->drho;
  r[2][0] = (0.5 * (-x5 + 3.0 * x4 - 3.0 * x3 + x2)) * p->drho2;
  r[0][1] = -6.0 * omx5 + 15.0 * omx4 - 10.0 * omx3 + 1.0;
  r[1][1] = (3.0 * omx5 - 8.0 * omx4 + 6.0 * omx3 - omx) * p->drho;
  r[2][1] = (0.5 * (-omx5 + 3.0 * omx4 - 3.0 * omx3 + omx2)) * p->drho2;
}
static void basis_t(const cellpos *p, double t[3][2]) {
  double y = p->y, y2 = p->y2, y3 = p->y3, y4 = p->y4, y5 = p->y5;
  double omy = p->omy, omy2 = p->omy2, omy3 = p->omy3, omy4 = p->omy4, omy5 = p->omy5;
  t[0][0] = -6.0 * y5 + 15.0 * y4 - 10.0 * y3 + 1.0;
  t[1][0] = (-3.0 * y5 + 8.0 * y4 - 6.0 * y3 + y) * p->dT;
  t[2][0] = (0.5 * (-y5 + 3.0 * y4 - 3.0 * y3 + y2)) * p->dT2;
  t[0][1] = -6.0 * omy5 + 15.0 * omy4 - 10.0 * omy3 + 1.0;
  t[1][1] = (3.0 * omy5 - 8.0 * omy4 + 6.0 * omy3 - omy) * p->dT;
  t[2][1] = (0.5 * (-omy5 + 3.0 * omy4 - 3.0 * omy3 + omy2)) * p->dT2;
}
/* first derivatives (source.F90:23955-23960 for rho, 24786-24791 for T) */
static void dbasis_r(const cellpos *p, double r[3][2]) {
  double x = p->x, x2 = p->x2, x3 = p->x3, x4 = p->x4;
  double omx = p->omx, omx2 = p->omx2, omx3 = p->omx3, omx4 = p->omx4;
  r[0][0] = (-30.0 * x4 + 60.0 * x3 - 30.0 * x2) * p->idrho;
  r[1][0] = (-15.0 * x4 + 32.0 * x3 - 18.0 * x2 + 1.0);
  r[2][0] = (0.5 * (-5.0 * x4 + 12.0 * x3 - 9.0 * x2 + 2.0 * x)) * p->drho;
  r[0][1] = -(-30.0 * omx4 + 60.0 * omx3 - 30.0 * omx2) * p->idrho;
  r[1][1] = (-15.0 * omx4 + 32.0 * omx3 - 18.0 * omx2 + 1.0);
  r[2][1] = -(0.5 * (-5.0 * omx4 + 12.0 * omx3 - 9.0 * omx2 + 2.0 * omx)) * p->drho;
}
static void dbasis_t(const cellpos *p, double t[3][2]) {
  double y = p->y, y2 = p->y2, y3 = p->y3, y4 = p->y4;
  double omy = p->omy, omy2 = p->omy2, omy3 = p->omy3, omy4 = p->omy4;
  t[0][0] = (-30.0 * y4 + 60.0 * y3 - 30.0 * y2) * p->idT;
  t[1][0] = (-15.0 * y4 + 32.0 * y3 - 18.0 * y2 + 1.0);
  t[2][0] = (0.5 * (-5.0 * y4 + 12.0 * y3 - 9.0 * y2 + 2.0 * y)) * p->dT;
  t[0][1] = -(-30.0 * omy4 + 60.0 * omy3 - 30.0 * omy2) * p->idT;
  t[1][1] = (-15.0 * omy4 + 32.0 * omy3 - 18.0 * omy2 + 1.0);
  t[2][1] = -(0.5 * (-5.0 * omy4 + 12.0 * omy3 - 9.0 * omy2 + 2.0 * omy)) * p->dT;
}
/* second T derivatives (source.F90:24826-24831) */
static void ddbasis_t(const cellpos *p, double t[3][2]) {
  double y = p->y, y2 = p->y2, y3 = p->y3;
  double omy = p->omy, omy2 = p->omy2, omy3 = p->omy3;
  t[0][0] = (-120.0 * y3 + 180.0 * y2 - 60.0 * y) * p->idT2;
  t[1][0] = (-60.0 * y3 + 96.0 * y2 - 36.0 * y) * p->idT;
  t[2][0] = (0.5 * (-20.0 * y3 + 36.0 * y2 - 18.0 * y + 2.0));
  t[0][1] = (-120.0 * omy3 + 180.0 * omy2 - 60.0 * omy) * p->idT2;
  t[1][1] = -(-60.0 * omy3 + 96.0 * omy2 - 36.0 * omy) * p->idT;
  t[2][1] = (0.5 * (-20.0 * omy3 + 36.0 * omy2 - 18.0 * omy + 2.0));
}

void phlo_helm_rhoT_given2(const phlo_helm *h, double rho, double T, double abar, double zbar,
                           double *E, double *dEdT, int return_dEdT) {
  cellpos p;
  double c[36], r[3][2], t[3][2], dt[3][2];
  locate(h, rho, T, abar, zbar, &p);
  load36(h, p.ih, p.jh, c);
  basis_r(&p, r);
  basis_t(&p, t);
  double f = sum36(c, r, t);
  dbasis_t(&p, dt);
  double df_dT = sum36(c, r, dt);
  double df_dT2 = 0.0;
  if (return_dEdT) {
    double ddt[3][2];
    ddbasis_t(&p, ddt);
    df_dT2 = sum36(c, r, ddt);
  }
  double s = -p.Ye * df_dT;
  double ds_dT = -p.Ye * df_dT2;
  double e = p.Ye * f + T * s;
  double de = T * ds_dT;
  double T2 = T * T, T3 = T2 * T, T4 = T3 * T;
  double tmp = 1.0 / abar;
  e = e + 1.5 * CONST_RGAS * T * tmp + CONST_RAD * T4 / rho;
  de = de + 1.5 * CONST_RGAS * tmp + 4.0 * CONST_RAD * T3 / rho;
  *E = e;
  *dEdT = de;
}

void phlo_helm_rhoT_given1(const phlo_helm *h, double rho, double T, double abar, double zbar,
                           double *P, double *dPdT, int return_dPdT) {
  cellpos p;
  double c[36], r[3][2], t[3][2], dr[3][2];
  locate(h, rho, T, abar, zbar, &p);
  load36(h, p.ih, p.jh, c);
  basis_r(&p, r);
  basis_t(&p, t);
  dbasis_r(&p, dr);
  double df_drho = sum36(c, dr, t);
  double df_drhodT = 0.0;
  if (return_dPdT) {
    double dt[3][2];
    dbasis_t(&p, dt);
    df_drhodT = sum36(c, dr, dt);
  }
  double tmp = p.rhos * p.rhos;
  double pp = tmp * df_drho;
  double dp = tmp * df_drhodT;
  double T2 = T * T, T3 = T2 * T, T4 = T3 * T;
  tmp = 1.0 / abar;
  double pion = CONST_RGAS * rho * T * tmp;
  double dpiondt = CONST_RGAS * rho * tmp;
  pp = pp + pion + CONST_RAD * T4 * (1.0 / 3.0);
  dp = dp + dpiondt + (4.0 / 3.0) * CONST_RAD * T3;
  *P = pp;
  *dPdT = dp;
}

void phlo_helm_rhoT_given_full(const phlo_helm *h, double rho, double T, double abar, double zbar,
                               double *P, double *E, double *sound, double *cv) {
  cellpos p;
  double c[36], r[3][2], t[3][2], dr[3][2], dt[3][2], ddt[3][2];
  locate(h, rho, T, abar, zbar, &p);
  load36(h, p.ih, p.jh, c);
  basis_r(&p, r);
  basis_t(&p, t);
  double f = sum36(c, r, t);
  dbasis_r(&p, dr);
  double df_drho = sum36(c, dr, t);
  dbasis_t(&p, dt);
  double df_dT = sum36(c, r, dt);
  double df_drhodT = sum36(c, dr, dt);
  ddbasis_t(&p, ddt);
  double df_dT2 = sum36(c, r, ddt);

  /* bicubic Hermite of dP/drho (source.F90:24082-24118) */
  double x = p.x, x2 = p.x2, x3 = p.x3, omx = p.omx, omx2 = p.omx2, omx3 = p.omx3;
  double y = p.y, y2 = p.y2, y3 = p.y3, omy = p.omy, omy2 = p.omy2, omy3 = p.omy3;
  double p0r = 2.0 * x3 - 3.0 * x2 + 1.0;
  double p1r = (x3 - 2.0 * x2 + x) * p.drho;
  double p0mr = 2.0 * omx3 - 3.0 * omx2 + 1.0;
  double p1mr = -(omx3 - 2.0 * omx2 + omx) * p.drho;
  double p0t = 2.0 * y3 - 3.0 * y2 + 1.0;
  double p1t = (y3 - 2.0 * y2 + y) * p.dT;
  double p0mt = 2.0 * omy3 - 3.0 * omy2 + 1.0;
  double p1mt = -(omy3 - 2.0 * omy2 + omy) * p.dT;
  int ih = p.ih, jh = p.jh;
  double l[16];
  for (int v = 1; v <= 4; ++v) {
    l[4 * (v - 1) + 0] = DPD(h, v, ih, jh);
    l[4 * (v - 1) + 1] = DPD(h, v, ih + 1, jh);
    l[4 * (v - 1) + 2] = DPD(h, v, ih, jh + 1);
    l[4 * (v - 1) + 3] = DPD(h, v, ih + 1, jh + 1);
  }
  double dP_drho =
      l[0] * p0r * p0t + l[1] * p0mr * p0t + l[2] * p0r * p0mt + l[3] * p0mr * p0mt +
      l[4] * p0r * p1t + l[5] * p0mr * p1t + l[6] * p0r * p1mt + l[7] * p0mr * p1mt +
      l[8] * p1r * p0t + l[9] * p1mr * p0t + l[10] * p1r * p0mt + l[11] * p1mr * p0mt +
      l[12] * p1r * p1t + l[13] * p1mr * p1t + l[14] * p1r * p1mt + l[15] * p1mr * p1mt;
  dP_drho = p.Ye * dP_drho;

  double tmp = p.rhos * p.rhos;
  double pp = tmp * df_drho;
  double dP_dT = tmp * df_drhodT;
  double s = -p.Ye * df_dT;
  double ds_dT = -p.Ye * df_dT2;
  tmp = p.Ye * p.Ye;
  double ds_drho = -df_drhodT * tmp;
  double e = p.Ye * f + T * s;
  double dE_dT = T * ds_dT;
  double dE_drho = df_drho * tmp + T * ds_drho;
  tmp = 1.0 / abar;
  double T2 = T * T, T3 = T2 * T, T4 = T3 * T;
  double pion = CONST_RGAS * rho * T * tmp;
  double dpiondt = CONST_RGAS * rho * tmp;
  double dpiondd = CONST_RGAS * T * tmp;
  pp = pp + pion + CONST_RAD * T4 * (1.0 / 3.0);
  dP_dT = dP_dT + dpiondt + (4.0 / 3.0) * CONST_RAD * T3;
  dP_drho = dP_drho + dpiondd;
  e = e + 1.5 * CONST_RGAS * T * tmp + CONST_RAD * T4 / rho;
  dE_dT = dE_dT + 1.5 * CONST_RGAS * tmp + 4.0 * CONST_RAD * T3 / rho;
  dE_drho = dE_drho - CONST_RAD * T4 / (rho * rho);
  (void)dE_drho;
  double zz = pp / rho;
  double c_v = dE_dT;
  double chiT = T / pp * dP_dT;
  double chirho = dP_drho / zz;
  double xx = zz * chiT / (T * c_v);
  double gam1 = chiT * xx + chirho;
  double z = 1.0 + (e + CONST_C2) / zz;
  *P = pp;
  *E = e;
  *cv = c_v;
  *sound = CONST_C * sqrt(gam1 / z);
}

int phlo_helm_rhoP_given(const phlo_helm *h, double rho, double P0, double abar, double zbar,
                         double *T, double *E, double *sound, int return_sound) {
  double error = 1.0, P, dP_dT, res, Told = *T, cv = 0.0;
  int iter, used = 0;
  *sound = 0.0;
  for (iter = 1; iter <= 100; ++iter) {
    used = iter;
    phlo_helm_rhoT_given1(h, rho, *T, abar, zbar, &P, &dP_dT, 1);
    res = P - P0;
    *T = *T - res / dP_dT;
    error = fabs(res / P0);
    if ((*T < h->Tl) || (*T > h->Th)) {
      *T = Told;
      error = EM15;
    }
    if (error < HELM_TOL) break;
  }
  if (return_sound) {
    phlo_helm_rhoT_given_full(h, rho, *T, abar, zbar, &P, E, sound, &cv);
  } else {
    double dE;
    phlo_helm_rhoT_given2(h, rho, *T, abar, zbar, E, &dE, 0);
  }
  return used;
}

int phlo_helm_rhoe_given(const phlo_helm *h, double rho, double E0, double abar, double zbar,
                         double *T, double *P, double *sound, int return_sound) {
  double error = 1.0, E, dE_dT, res, Told = *T, cv = 0.0;
  int iter, used = 0;
  *sound = 0.0;
  for (iter = 1; iter <= 100; ++iter) {
    used = iter;
    phlo_helm_rhoT_given2(h, rho, *T, abar, zbar, &E, &dE_dT, 1);
    res = E - E0;
    *T = *T - res / dE_dT;
    error = fabs(res / E0);
    if ((*T < h->Tl) || (*T > h->Th)) {
      *T = Told;
      error = EM15;
    }
    if (error < HELM_TOL) break;
  }
  if (return_sound) {
    phlo_helm_rhoT_given_full(h, rho, *T, abar, zbar, P, &E, sound, &cv);
  } else {
    double dP;
    phlo_helm_rhoT_given1(h, rho, *T, abar, zbar, P, &dP, 0);
  }
  return used;
}

int phlo_eos_bracket_guess(const phlo_helm *h, double rho, double e, double abar, double zbar, double *T) {
  int lo = 0, hi = h->nT - 1, evals = 2;
  double elo, ehi, dd, em, w;
  phlo_helm_rhoT_given2(h, rho, h->T[lo], abar, zbar, &elo, &dd, 0);
  if (e <= elo) {
    *T = h->T[lo];
    return 1;
  }
  phlo_helm_rhoT_given2(h, rho, h->T[hi] * 0.999999, abar, zbar, &ehi, &dd, 0);
  if (e >= ehi) {
    *T = h->T[hi] * 0.999999;
    return 2;
  }
  while (hi - lo > 1) {
    int mid = (lo + hi) >> 1;
    phlo_helm_rhoT_given2(h, rho, h->T[mid], abar, zbar, &em, &dd, 0);
    ++evals;
    if (em <= e) {
      lo = mid;
      elo = em;
    } else {
      hi = mid;
      ehi = em;
    }
  }
  w = (e - elo) / (ehi - elo);
  *T = h->T[lo] + w * (h->T[hi] - h->T[lo]);
  return evals;
}

void phlo_eos_invert_batch(const phlo_helm *h, long n, const double *rho, const double *e, const double *abar,
                           const double *zbar, double *T, int *iters, int guess, int nthreads) {
  long i;
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 256)
  for (i = 0; i < n; ++i) {
    double t = T[i], P, snd;
    int it;
    if (guess == 2) phlo_eos_bracket_guess(h, rho[i], e[i], abar[i], zbar[i], &t);
    it = phlo_helm_rhoe_given(h, rho[i], e[i], abar[i], zbar[i], &t, &P, &snd, 0);
    T[i] = t;
    if (iters) iters[i] = it;
  }
}
