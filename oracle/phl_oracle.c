/*
 * phl_oracle.c -- CPU restatement of Phlegethon's explicit FV step (hydro_step, riemann,
 * compute_hyperbolic_dt, step-0 thermodynamics).
 * TEST INFRASTRUCTURE ONLY (checker and CPU baseline); parity unpinned, see phl_oracle.h.
 *
 * Reference map (source/source.F90):
 *   prim->cons, state0/state, b0 copies      7057-7147
 *   RK coefficients (RK2/RK3 Shu-Osher)      7018-7048
 *   WB deviation (rho', p', gammae')         7151-7168
 *   periodic self-copy of ghosts             2293-2306 / 2431-2444 (communicate_*)
 *   reflective physical BCs                  7532-7958 (bc_fac / bc_facb)
 *   shock detector (USE_SHOCK_FLATTENING)   8073-8136
 *   x1 sweep: LIM2ND PLM, B recon, WB add,   8138-9105
 *             FASTEOS gamma recon, flattening 8731-8878, riemann, EMF + sign_frho,
 *             WB flux fix, ETOT, res
 *   x2 sweep (rotation v,B / flux back)      9107-10301
 *   x3 sweep (cyclic rotation)               10303-11364
 *   EMF ghosts + reflective EMF BCs          11374-11964
 *   CT corner EMFs, face-B update, b_cc      11966-12487
 *   gravity source                           12606-12644
 *   constant acceleration                    12806-12836
 *   RK combine                               13518-13531
 *   cons->prim + EoS                         13533-13686
 *   hyperbolic dt                            13707-13960
 *   hydro Riemann LHLLC / HLLC               15611-16260
 *   MHD Riemann HLLD / LHLLD                 13969-15024
 * Loops over lines are OpenMP-parallel; every floating-point expression keeps the
 * reference's operand order.
 */
#include <math.h>

/* Iteration counts of the per-face helm_rhoP_given solves of the Riemann sides (Helmholtz without
 * USE_FASTEOS): how far the reference's face temperature guess 0.5 (T_L + T_R) is from the
 * answer, measured on the reference's own algorithm.  Test statistics only. */
static long long g_face_newton_calls = 0, g_face_newton_iters = 0;
static void face_newton_count(int iters) {
#pragma omp atomic
  g_face_newton_calls += 1;
#pragma omp atomic
  g_face_newton_iters += iters;
}
void phlo_face_newton_stats(long long *calls, long long *iters, int reset) {
  *calls = g_face_newton_calls;
  *iters = g_face_newton_iters;
  if (reset) g_face_newton_calls = g_face_newton_iters = 0;
}
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif
#include "phl_oracle.h"

#define CONST_RGAS 8.31446261815324e7

/* ---------------------------------------------------------------- array shapes */
typedef struct { int lo[3], hi[3], nv; long n[3]; } shp;

static shp mk(int nv, int l0, int h0, int l1, int h1, int l2, int h2) {
  shp s;
  s.nv = nv;
  s.lo[0] = l0; s.hi[0] = h0; s.lo[1] = l1; s.hi[1] = h1; s.lo[2] = l2; s.hi[2] = h2;
  for (int d = 0; d < 3; ++d) s.n[d] = s.hi[d] - s.lo[d] + 1;
  return s;
}
static inline long OFF(const shp *s, int iv, int i, int j, int k) {
  return iv + (long)s->nv * ((i - s->lo[0]) + s->n[0] * ((j - s->lo[1]) + s->n[1] * (long)(k - s->lo[2])));
}
static long ssize(const shp *s) { return (long)s->nv * s->n[0] * s->n[1] * s->n[2]; }

static int g3(const phlo_grid *g) { return g->sdims == 3 ? g->ngc : 0; }
static shp cellg(const phlo_grid *g, int nv) {
  int G = g->ngc, G3 = g3(g);
  return mk(nv, 1 - G, g->nx1 + G, 1 - G, g->nx2 + G, 1 - G3, g->nx3 + G3);
}
static shp interior(const phlo_grid *g, int nv) { return mk(nv, 1, g->nx1, 1, g->nx2, 1, g->nx3); }
static shp face(const phlo_grid *g, int nv, int d) {
  shp s = interior(g, nv);
  s.hi[d] += 1; s.n[d] += 1;
  return s;
}
/* b_x1(lx1-1:ux1+2, lx2-1:ux2+1, lx3-1:ux3+1) and its x2/x3 analogues (source.F90:1629-1645);
 * in 2D the x3 range is lx3:ux3.  emf_x*, sign_frho_x* share these bounds. */
static shp bface(const phlo_grid *g, int nv, int d) {
  int l3 = g->sdims == 3 ? 0 : 1, h3 = g->sdims == 3 ? g->nx3 + 1 : g->nx3;
  shp s = mk(nv, 0, g->nx1 + 1, 0, g->nx2 + 1, l3, h3);
  s.hi[d] += 1; s.n[d] += 1;
  return s;
}
/* corner EMF along axis a: (lx1:ux1+1, lx2:ux2+1, lx3:ux3) for a=3, etc. */
static shp corner(const phlo_grid *g, int a) {
  shp s = interior(g, 1);
  for (int d = 0; d < 3; ++d)
    if (d != a) { s.hi[d] += 1; s.n[d] += 1; }
  return s;
}

long phlo_cells_ghost(const phlo_grid *g) { shp s = cellg(g, 1); return ssize(&s); }
long phlo_faces(const phlo_grid *g, int d) { shp s = face(g, 1, d); return ssize(&s); }
long phlo_bface(const phlo_grid *g, int d) { shp s = bface(g, 1, d); return ssize(&s); }

/* ---------------------------------------------------------------- scratch */
typedef struct {
  double *state, *state0, *res;
  double *b0[3];
  double *emf[3], *sgn[3], *cor[3];
  double *flat;   /* is_flattened(cells), 0/1 (USE_SHOCK_FLATTENING) */
} scr_t;

long phlo_scratch_doubles(const phlo_grid *g) {
  shp in = interior(g, g->nvars);
  long n = 3 * ssize(&in);
  if (g->mhd) {
    for (int d = 0; d < g->sdims; ++d) {
      shp f = face(g, 1, d), b = bface(g, 3, d), b1 = bface(g, 1, d);
      n += ssize(&f) + ssize(&b) + ssize(&b1);
    }
    for (int a = 0; a < 3; ++a) {
      if (g->sdims == 2 && a != 2) continue;
      shp c = corner(g, a);
      n += ssize(&c);
    }
  }
  if (g->sf) {
    shp c = cellg(g, 1);
    n += ssize(&c);
  }
  return n;
}

static scr_t carve(phlo_grid *g) {
  scr_t s;
  memset(&s, 0, sizeof s);
  if (!g->scratch) g->scratch = (double *)calloc((size_t)phlo_scratch_doubles(g), sizeof(double));
  double *p = g->scratch;
  shp in = interior(g, g->nvars);
  s.state = p; p += ssize(&in);
  s.state0 = p; p += ssize(&in);
  s.res = p; p += ssize(&in);
  if (g->mhd) {
    for (int d = 0; d < g->sdims; ++d) {
      shp f = face(g, 1, d), b = bface(g, 3, d), b1 = bface(g, 1, d);
      s.b0[d] = p; p += ssize(&f);
      s.emf[d] = p; p += ssize(&b);
      s.sgn[d] = p; p += ssize(&b1);
    }
    for (int a = 0; a < 3; ++a) {
      if (g->sdims == 2 && a != 2) continue;
      shp c = corner(g, a);
      s.cor[a] = p; p += ssize(&c);
    }
  }
  if (g->sf) {
    shp c = cellg(g, 1);
    s.flat = p; p += ssize(&c);
  }
  return s;
}

/* ---------------------------------------------------------------- variable indices */
/* 0-based: rho, vx1..vx(sdims), p, scalars (source.F90:483-512) */
#define IRHO 0
#define IVX(d) (1 + (d))
static inline int IP(const phlo_grid *g) { return 1 + g->sdims; }
static inline int IAS1(const phlo_grid *g) { return 2 + g->sdims; }

static inline double sgnf(double x) { return copysign(1.0, x); }

/* ---------------------------------------------------------------- Riemann: hydro */
void phlo_riemann_hydro(const phlo_grid *g, const double *qL, const double *qR,
                        const double *gL, const double *gR, double *flux, int flat) {
  const int three = g->sdims == 3, ip = IP(g), ias = IAS1(g), nv = g->nvars;
  const double gm = g->gm, gmm1 = gm - 1.0, igmm1 = 1.0 / gmm1;
  double rhoL = qL[IRHO], inv_rhoL = 1.0 / rhoL, vx1L = qL[1], vx2L = qL[2], vx3L = three ? qL[3] : 0.0;
  double v2L = vx1L * vx1L + vx2L * vx2L + vx3L * vx3L;
  double pL = qL[ip], eint, cL, cR;
  if (g->fasteos) {
    eint = pL / (gL[0] - 1.0);
    cL = sqrt(gL[1] * pL * inv_rhoL);
  } else if (g->helm) {
    /* helm_rhoP_given from the face temperature guess (source.F90:15705-15720, 15777-15781) */
    double ye = qL[ias], abar = 1.0 / qL[ias + 1], zbar = ye * abar, T = gL[0];
    face_newton_count(phlo_helm_rhoP_given(g->eos, rhoL, pL, abar, zbar, &T, &eint, &cL, 1));
    eint = eint * rhoL;
  } else {
    eint = igmm1 * pL;
    cL = sqrt(gm * pL * inv_rhoL);
  }
  double rhoeL = eint + 0.5 * rhoL * v2L;
  double rhoR = qR[IRHO], inv_rhoR = 1.0 / rhoR, vx1R = qR[1], vx2R = qR[2], vx3R = three ? qR[3] : 0.0;
  double v2R = vx1R * vx1R + vx2R * vx2R + vx3R * vx3R;
  double pR = qR[ip];
  if (g->fasteos) {
    eint = pR / (gR[0] - 1.0);
    cR = sqrt(gR[1] * pR * inv_rhoR);
  } else if (g->helm) {
    double ye = qR[ias], abar = 1.0 / qR[ias + 1], zbar = ye * abar, T = gR[0];
    face_newton_count(phlo_helm_rhoP_given(g->eos, rhoR, pR, abar, zbar, &T, &eint, &cR, 1));
    eint = eint * rhoR;
  } else {
    eint = igmm1 * pR;
    cR = sqrt(gm * pR * inv_rhoR);
  }
  double rhoeR = eint + 0.5 * rhoR * v2R;
  double max_c = fmax(cL, cR);
  double sL = fmin(vx1L, vx1R) - max_c;
  double sR = fmax(vx1L, vx1R) + max_c;
  double dsuL = sL - vx1L, dsuR = sR - vx1R;
  double ustar = (pR - pL + rhoL * vx1L * dsuL - rhoR * vx1R * dsuR) / (rhoL * dsuL - rhoR * dsuR);
  double rhostarL = rhoL * (dsuL / (sL - ustar));
  double rhoestarL = rhostarL * (rhoeL * inv_rhoL + (ustar - vx1L) * (ustar + pL * inv_rhoL / dsuL));
  double rhostarR = rhoR * (dsuR / (sR - ustar));
  double rhoestarR = rhostarR * (rhoeR * inv_rhoR + (ustar - vx1R) * (ustar + pR * inv_rhoR / dsuR));

  if (flat) {
    /* HLL flux on a flattened face (source.F90:15929-16010) */
    double UL[16], UR[16], fL[16], fR[16];
    sL = fmin(0.0, sL);
    sR = fmax(0.0, sR);
    UL[IRHO] = rhoL; UL[1] = rhoL * vx1L; UL[2] = rhoL * vx2L; if (three) UL[3] = rhoL * vx3L; UL[ip] = rhoeL;
    for (int iv = ias; iv < nv; ++iv) UL[iv] = rhoL * qL[iv];
    UR[IRHO] = rhoR; UR[1] = rhoR * vx1R; UR[2] = rhoR * vx2R; if (three) UR[3] = rhoR * vx3R; UR[ip] = rhoeR;
    for (int iv = ias; iv < nv; ++iv) UR[iv] = rhoR * qR[iv];
    fL[IRHO] = rhoL * vx1L; fL[1] = rhoL * vx1L * vx1L + pL; fL[2] = rhoL * vx1L * vx2L;
    if (three) fL[3] = rhoL * vx1L * vx3L;
    fL[ip] = (rhoeL + pL) * vx1L;
    for (int iv = ias; iv < nv; ++iv) fL[iv] = UL[iv] * vx1L;
    fR[IRHO] = rhoR * vx1R; fR[1] = rhoR * vx1R * vx1R + pR; fR[2] = rhoR * vx1R * vx2R;
    if (three) fR[3] = rhoR * vx1R * vx3R;
    fR[ip] = (rhoeR + pR) * vx1R;
    for (int iv = ias; iv < nv; ++iv) fR[iv] = UR[iv] * vx1R;
    double dummy = 1.0 / (sR - sL), phi = sL * sR;
    for (int iv = 0; iv < nv; ++iv) flux[iv] = dummy * (sR * fL[iv] - sL * fR[iv] + phi * (UR[iv] - UL[iv]));
    return;
  }

  if (g->riemann == PHLO_LHLLC) {
    /* low-dissipation HLLC (source.F90:16012-16122, FLUX_IS_ALL_MACH off) */
    double machL = sqrt(v2L) / cL, machR = sqrt(v2R) / cR;
    double chi = fmin(1.0, fmax(machL, machR));
    chi = fmax(g->mach_cutoff, chi);
    double phi = chi * (2.0 - chi);
    double rhobar = 0.5 * (rhoL + rhoR), cbar = 0.5 * (cL + cR);
    double pstar = 0.5 * (pL + pR) - 0.5 * phi * rhobar * cbar * (vx1R - vx1L);
    if (g->all_mach && (sL > 0.0 || sR < 0.0)) {
      /* FLUX_IS_ALL_MACH: the upwind state's flux outside the wave fan (source.F90:16032-16077) */
      const int left = sL > 0.0;
      const double *q = left ? qL : qR;
      double rho = left ? rhoL : rhoR, vx1 = left ? vx1L : vx1R, vx2 = left ? vx2L : vx2R, vx3 = left ? vx3L : vx3R;
      double p = left ? pL : pR, rhoe = left ? rhoeL : rhoeR;
      flux[IRHO] = rho * vx1;
      flux[1] = rho * vx1 * vx1 + p;
      flux[2] = rho * vx1 * vx2;
      if (three) flux[3] = rho * vx1 * vx3;
      flux[ip] = (rhoe + p) * vx1;
      for (int iv = ias; iv < nv; ++iv) flux[iv] = rho * q[iv] * vx1;
      return;
    }
    double sgn = sgnf(ustar);
    double hp = 0.5 * (1.0 + sgn), hm = 0.5 * (1.0 - sgn);
    double rhostar = hp * rhostarL + hm * rhostarR;
    flux[IRHO] = rhostar * ustar;
    flux[1] = rhostar * ustar * ustar + pstar;
    flux[2] = rhostar * ustar * (hp * vx2L + hm * vx2R);
    if (three) flux[3] = rhostar * ustar * (hp * vx3L + hm * vx3R);
    flux[ip] = (hp * rhoestarL + hm * rhoestarR + pstar) * ustar;
    for (int iv = ias; iv < nv; ++iv) flux[iv] = rhostar * ustar * (hp * qL[iv] + hm * qR[iv]);
    return;
  }
  /* shock-capturing HLLC (source.F90:16124-16252) */
  double U[16], f[16], Us[16];
  const double *q;
  double rho, vx1, vx2, vx3, p, rhoe, rhostar, s;
  if (ustar > 0.0) {
    q = qL; rho = rhoL; vx1 = vx1L; vx2 = vx2L; vx3 = vx3L; p = pL; rhoe = rhoeL; rhostar = rhostarL;
    s = sL;
  } else {
    q = qR; rho = rhoR; vx1 = vx1R; vx2 = vx2R; vx3 = vx3R; p = pR; rhoe = rhoeR; rhostar = rhostarR;
    s = sR;
  }
  double rhoestar = ustar > 0.0 ? rhoestarL : rhoestarR;
  U[IRHO] = rho; U[1] = rho * vx1; U[2] = rho * vx2; if (three) U[3] = rho * vx3; U[ip] = rhoe;
  for (int iv = ias; iv < nv; ++iv) U[iv] = rho * q[iv];
  f[IRHO] = rho * vx1; f[1] = rho * vx1 * vx1 + p; f[2] = rho * vx1 * vx2;
  if (three) f[3] = rho * vx1 * vx3;
  f[ip] = (rhoe + p) * vx1;
  for (int iv = ias; iv < nv; ++iv) f[iv] = rho * vx1 * q[iv];
  int supersonic = ustar > 0.0 ? (sL >= 0.0) : (sR < 0.0);
  if (supersonic) {
    for (int iv = 0; iv < nv; ++iv) flux[iv] = f[iv];
  } else {
    Us[IRHO] = rhostar; Us[1] = rhostar * ustar; Us[2] = rhostar * vx2; if (three) Us[3] = rhostar * vx3;
    Us[ip] = rhoestar;
    for (int iv = ias; iv < nv; ++iv) Us[iv] = rhostar * q[iv];
    for (int iv = 0; iv < nv; ++iv) flux[iv] = f[iv] + s * (Us[iv] - U[iv]);
  }
}

/* ---------------------------------------------------------------- Riemann: MHD */
void phlo_riemann_mhd(const phlo_grid *g, const double *qL, const double *qR,
                      const double *bL, const double *bR, const double *gL, const double *gR,
                      double *flux, double *fluxb, int flat) {
  const int three = g->sdims == 3, ip = IP(g), ias = IAS1(g), nv = g->nvars;
  const double gm = g->gm, gmm1 = gm - 1.0, igmm1 = 1.0 / gmm1;
  double rhoL = qL[IRHO], inv_rhoL = 1.0 / rhoL, vx1L = qL[1], vx2L = qL[2], vx3L = three ? qL[3] : 0.0;
  double v2L = vx1L * vx1L + vx2L * vx2L + vx3L * vx3L;
  double pL = qL[ip], eint, c2L, c2R;
  if (g->fasteos) { eint = pL / (gL[0] - 1.0); c2L = gL[1] * pL * inv_rhoL; }
  else if (g->helm) {
    /* helm_rhoP_given from the face temperature guess (source.F90:14266-14275) */
    double ye = qL[ias], abar = 1.0 / qL[ias + 1], zbar = ye * abar, T = gL[0], sound;
    face_newton_count(phlo_helm_rhoP_given(g->eos, rhoL, pL, abar, zbar, &T, &eint, &sound, 1));
    eint = eint * rhoL;
    c2L = sound * sound;
  }
  else { eint = pL * igmm1; c2L = gm * pL * inv_rhoL; }
  double rhoeL = eint + 0.5 * rhoL * v2L;
  double bx1L = bL[0], bx2L = bL[1], bx3L = three ? bL[2] : 0.0;
  double rhoR = qR[IRHO], inv_rhoR = 1.0 / rhoR, vx1R = qR[1], vx2R = qR[2], vx3R = three ? qR[3] : 0.0;
  double v2R = vx1R * vx1R + vx2R * vx2R + vx3R * vx3R;
  double pR = qR[ip];
  if (g->fasteos) { eint = pR / (gR[0] - 1.0); c2R = gR[1] * pR * inv_rhoR; }
  else if (g->helm) {
    double ye = qR[ias], abar = 1.0 / qR[ias + 1], zbar = ye * abar, T = gR[0], sound;
    face_newton_count(phlo_helm_rhoP_given(g->eos, rhoR, pR, abar, zbar, &T, &eint, &sound, 1));
    eint = eint * rhoR;
    c2R = sound * sound;
  }
  else { eint = pR * igmm1; c2R = gm * pR * inv_rhoR; }
  double rhoeR = eint + 0.5 * rhoR * v2R;
  double bx1R = bR[0], bx2R = bR[1], bx3R = three ? bR[2] : 0.0;

  double bx1 = 0.5 * (bx1L + bx1R), bx1_2 = bx1 * bx1;
  double pbL = 0.5 * (bx1_2 + bx2L * bx2L + bx3L * bx3L);
  double pbR = 0.5 * (bx1_2 + bx2R * bx2R + bx3R * bx3R);
  rhoeL = rhoeL + pbL;
  rhoeR = rhoeR + pbR;
  double ptL = pL + pbL, ptR = pR + pbR;
  double a2L = 2.0 * pbL * inv_rhoL, a2R = 2.0 * pbR * inv_rhoR;
  double an2L = bx1_2 * inv_rhoL, an2R = bx1_2 * inv_rhoR;
  double dummy = c2L + a2L;
  double cL = sqrt(0.5 * (c2L + a2L + sqrt(dummy * dummy - 4.0 * c2L * an2L)));
  dummy = c2R + a2R;
  double cR = sqrt(0.5 * (c2R + a2R + sqrt(dummy * dummy - 4.0 * c2R * an2R)));
  double max_c = fmax(cL, cR);
  double sL = fmin(vx1L, vx1R) - max_c;
  double sR = fmax(vx1L, vx1R) + max_c;
  double dsuL = sL - vx1L, dsuR = sR - vx1R;
  double inv_temp1 = 1.0 / (dsuR * rhoR - dsuL * rhoL);
  double ustar = (dsuR * rhoR * vx1R - dsuL * rhoL * vx1L - ptR + ptL) * inv_temp1;
  double dsumL = sL - ustar, dsumR = sR - ustar;
  double phi = 1.0;
  if (g->riemann == PHLO_LHLLD) {
    /* source.F90:14364-14384 */
    dummy = v2L + a2L;
    double cu2L = 0.5 * (v2L + a2L + sqrt(dummy * dummy - 4.0 * v2L * an2L));
    dummy = v2R + a2R;
    double cu2R = 0.5 * (v2R + a2R + sqrt(dummy * dummy - 4.0 * v2R * an2R));
    double machL = sqrt(cu2L) / cL, machR = sqrt(cu2R) / cR;
    double mm = fmax(machL, machR);
    if (mm < 0.6) {
      double chi = fmin(1.0, fmax(machL, machR));
      chi = fmax(g->mach_cutoff, chi);
      phi = chi * (2.0 - chi);
    } else {
      phi = 1.0;
    }
  }
  if (flat) {
    /* HLL flux on a flattened face (source.F90:14386-14495) */
    double UL[16], UR[16], fL[16], fR[16], UbL[3], UbR[3], fbL[3], fbR[3];
    sL = fmin(0.0, sL);
    sR = fmax(0.0, sR);
    UL[IRHO] = rhoL; UL[1] = rhoL * vx1L; UL[2] = rhoL * vx2L; if (three) UL[3] = rhoL * vx3L; UL[ip] = rhoeL;
    for (int iv = ias; iv < nv; ++iv) UL[iv] = rhoL * qL[iv];
    UbL[0] = bx1; UbL[1] = bx2L; UbL[2] = bx3L;
    UR[IRHO] = rhoR; UR[1] = rhoR * vx1R; UR[2] = rhoR * vx2R; if (three) UR[3] = rhoR * vx3R; UR[ip] = rhoeR;
    for (int iv = ias; iv < nv; ++iv) UR[iv] = rhoR * qR[iv];
    UbR[0] = bx1; UbR[1] = bx2R; UbR[2] = bx3R;
    fL[IRHO] = rhoL * vx1L; fL[1] = rhoL * vx1L * vx1L + ptL - bx1_2; fL[2] = rhoL * vx1L * vx2L - bx1 * bx2L;
    if (three) fL[3] = rhoL * vx1L * vx3L - bx1 * bx3L;
    fL[ip] = (rhoeL + ptL) * vx1L - bx1 * (bx1 * vx1L + bx2L * vx2L + bx3L * vx3L);
    for (int iv = ias; iv < nv; ++iv) fL[iv] = UL[iv] * vx1L;
    fbL[0] = 0.0; fbL[1] = vx1L * bx2L - vx2L * bx1; fbL[2] = vx1L * bx3L - vx3L * bx1;
    fR[IRHO] = rhoR * vx1R; fR[1] = rhoR * vx1R * vx1R + ptR - bx1_2; fR[2] = rhoR * vx1R * vx2R - bx1 * bx2R;
    if (three) fR[3] = rhoR * vx1R * vx3R - bx1 * bx3R;
    fR[ip] = (rhoeR + ptR) * vx1R - bx1 * (bx1 * vx1R + bx2R * vx2R + bx3R * vx3R);
    for (int iv = ias; iv < nv; ++iv) fR[iv] = UR[iv] * vx1R;
    fbR[0] = 0.0; fbR[1] = vx1R * bx2R - vx2R * bx1; fbR[2] = vx1R * bx3R - vx3R * bx1;
    double dummy_h = 1.0 / (sR - sL), phi_h = sL * sR;
    for (int iv = 0; iv < nv; ++iv) flux[iv] = dummy_h * (sR * fL[iv] - sL * fR[iv] + phi_h * (UR[iv] - UL[iv]));
    for (int iv = 0; iv < (three ? 3 : 2); ++iv)
      fluxb[iv] = dummy_h * (sR * fbL[iv] - sL * fbR[iv] + phi_h * (UbR[iv] - UbL[iv]));
    return;
  }
  double pstar = (dsuR * rhoR * ptL - dsuL * rhoL * ptR - phi * rhoL * rhoR * dsuR * dsuL * (vx1L - vx1R)) * inv_temp1;
  double rhostarL = rhoL * dsuL / dsumL, rhostarR = rhoR * dsuR / dsumR;
  double a1_inv = 1.0 / (rhoL * dsuL * dsumL - bx1_2);
  double vx2starL = vx2L - bx1 * bx2L * (ustar - vx1L) * a1_inv;
  double bx2starL = bx2L * (rhoL * dsuL * dsuL - bx1_2) * a1_inv;
  double vx3starL = vx3L - bx1 * bx3L * (ustar - vx1L) * a1_inv;
  double bx3starL = bx3L * (rhoL * dsuL * dsuL - bx1_2) * a1_inv;
  double a2_inv = 1.0 / (rhoR * dsuR * dsumR - bx1_2);
  double vx2starR = vx2R - bx1 * bx2R * (ustar - vx1R) * a2_inv;
  double bx2starR = bx2R * (rhoR * dsuR * dsuR - bx1_2) * a2_inv;
  double vx3starR = vx3R - bx1 * bx3R * (ustar - vx1R) * a2_inv;
  double bx3starR = bx3R * (rhoR * dsuR * dsuR - bx1_2) * a2_inv;
  double vdotbL = vx1L * bx1 + vx2L * bx2L + vx3L * bx3L;
  double vdotbR = vx1R * bx1 + vx2R * bx2R + vx3R * bx3R;
  double vdotbstarL = ustar * bx1 + vx2starL * bx2starL + vx3starL * bx3starL;
  double vdotbstarR = ustar * bx1 + vx2starR * bx2starR + vx3starR * bx3starR;
  double rhoestarL = (dsuL * rhoeL - ptL * vx1L + pstar * ustar + bx1 * (vdotbL - vdotbstarL)) / dsumL;
  double rhoestarR = (dsuR * rhoeR - ptR * vx1R + pstar * ustar + bx1 * (vdotbR - vdotbstarR)) / dsumR;
  double sqrt_rhostarL = sqrt(rhostarL), sqrt_rhostarR = sqrt(rhostarR);
  double abs_bx1 = fabs(bx1);
  double sstarL = ustar - abs_bx1 / sqrt_rhostarL;
  double sstarR = ustar + abs_bx1 / sqrt_rhostarR;
  double inv_sqr_bar = 1.0 / (sqrt_rhostarL + sqrt_rhostarR);
  double sgn = sgnf(bx1);
  double vx22star = (sqrt_rhostarL * vx2starL + sqrt_rhostarR * vx2starR + (bx2starR - bx2starL) * sgn) * inv_sqr_bar;
  double bx22star = (sqrt_rhostarL * bx2starR + sqrt_rhostarR * bx2starL +
                     sqrt_rhostarL * sqrt_rhostarR * (vx2starR - vx2starL) * sgn) * inv_sqr_bar;
  double vx32star = (sqrt_rhostarL * vx3starL + sqrt_rhostarR * vx3starR + (bx3starR - bx3starL) * sgn) * inv_sqr_bar;
  double bx32star = (sqrt_rhostarL * bx3starR + sqrt_rhostarR * bx3starL +
                     sqrt_rhostarL * sqrt_rhostarR * (vx3starR - vx3starL) * sgn) * inv_sqr_bar;
  double vdotb2star = ustar * bx1 + vx22star * bx22star + vx32star * bx32star;
  double rhoe2starL = rhoestarL - sqrt_rhostarL * (vdotbstarL - vdotb2star) * sgn;
  double rhoe2starR = rhoestarR + sqrt_rhostarR * (vdotbstarR - vdotb2star) * sgn;

  fluxb[0] = 0.0;
  if (g->riemann == PHLO_LHLLD) {
    /* source.F90:14663-14732 */
    double rho, vx1, vx2, vx3, rhoe, bx2, bx3, pres = pstar;
    if (g->all_mach && sL > 0.0) {
      /* FLUX_IS_ALL_MACH: the outer states as well (source.F90:14576-14632) */
      rho = rhoL; vx1 = vx1L; vx2 = vx2L; vx3 = vx3L; rhoe = rhoeL; bx2 = bx2L; bx3 = bx3L; pres = ptL;
    } else if (sstarL > 0.0) {
      rho = rhostarL; vx1 = ustar; vx2 = vx2starL; vx3 = vx3starL; rhoe = rhoestarL; bx2 = bx2starL; bx3 = bx3starL;
    } else if (ustar > 0.0) {
      rho = rhostarL; vx1 = ustar; vx2 = vx22star; vx3 = vx32star; rhoe = rhoe2starL; bx2 = bx22star; bx3 = bx32star;
    } else if (sstarR > 0.0) {
      rho = rhostarR; vx1 = ustar; vx2 = vx22star; vx3 = vx32star; rhoe = rhoe2starR; bx2 = bx22star; bx3 = bx32star;
    } else if (!g->all_mach || sR > 0.0) {
      rho = rhostarR; vx1 = ustar; vx2 = vx2starR; vx3 = vx3starR; rhoe = rhoestarR; bx2 = bx2starR; bx3 = bx3starR;
    } else {
      rho = rhoR; vx1 = vx1R; vx2 = vx2R; vx3 = vx3R; rhoe = rhoeR; bx2 = bx2R; bx3 = bx3R; pres = ptR;
    }
    flux[IRHO] = rho * vx1;
    flux[1] = rho * vx1 * vx1 + pres - bx1_2;
    flux[2] = rho * vx1 * vx2 - bx1 * bx2;
    if (three) flux[3] = rho * vx1 * vx3 - bx1 * bx3;
    flux[ip] = (rhoe + pres) * vx1 - bx1 * (bx1 * vx1 + vx2 * bx2 + vx3 * bx3);
    double sg = sgnf(vx1), hp = 0.5 * (1.0 + sg), hm = 0.5 * (1.0 - sg);
    for (int iv = ias; iv < nv; ++iv) flux[iv] = rho * vx1 * (hp * qL[iv] + hm * qR[iv]);
    fluxb[1] = vx1 * bx2 - bx1 * vx2;
    if (three) fluxb[2] = vx1 * bx3 - bx1 * vx3;
    return;
  }
  /* HLLD (source.F90:14736-15016) */
  double U[16], f[16], Us[16], Uss[16], Ub[3], fb[3], Ubs[3], Ubss[3];
  const double *q;
  double rho, vx1, vx2, vx3, rhoe, pt, bx2, bx3, vdotb, rhostar, vx2s, vx3s, bx2s, bx3s, rhoes, rhoe2s;
  double s, sstar;
  int left = ustar > 0.0;
  if (left) {
    q = qL; rho = rhoL; vx1 = vx1L; vx2 = vx2L; vx3 = vx3L; rhoe = rhoeL; pt = ptL; bx2 = bx2L; bx3 = bx3L;
    vdotb = vdotbL; rhostar = rhostarL; vx2s = vx2starL; vx3s = vx3starL; bx2s = bx2starL; bx3s = bx3starL;
    rhoes = rhoestarL; rhoe2s = rhoe2starL; s = sL; sstar = sstarL;
  } else {
    q = qR; rho = rhoR; vx1 = vx1R; vx2 = vx2R; vx3 = vx3R; rhoe = rhoeR; pt = ptR; bx2 = bx2R; bx3 = bx3R;
    vdotb = vdotbR; rhostar = rhostarR; vx2s = vx2starR; vx3s = vx3starR; bx2s = bx2starR; bx3s = bx3starR;
    rhoes = rhoestarR; rhoe2s = rhoe2starR; s = sR; sstar = sstarR;
  }
  int nb = three ? 3 : 2;
  U[IRHO] = rho; U[1] = rho * vx1; U[2] = rho * vx2; if (three) U[3] = rho * vx3; U[ip] = rhoe;
  for (int iv = ias; iv < nv; ++iv) U[iv] = rho * q[iv];
  Ub[0] = bx1; Ub[1] = bx2; Ub[2] = bx3;
  f[IRHO] = rho * vx1; f[1] = rho * vx1 * vx1 + pt - bx1_2; f[2] = rho * vx1 * vx2 - bx1 * bx2;
  if (three) f[3] = rho * vx1 * vx3 - bx1 * bx3;
  f[ip] = (rhoe + pt) * vx1 - bx1 * vdotb;
  for (int iv = ias; iv < nv; ++iv) f[iv] = rho * vx1 * q[iv];
  fb[0] = 0.0; fb[1] = vx1 * bx2 - bx1 * vx2; fb[2] = vx1 * bx3 - bx1 * vx3;
  int outer = left ? (sL > 0.0) : (sR < 0.0);
  int single = left ? (sstarL > 0.0) : (sstarR < 0.0);
  (void)sstar;
  if (outer) {
    for (int iv = 0; iv < nv; ++iv) flux[iv] = f[iv];
    for (int iv = 0; iv < nb; ++iv) fluxb[iv] = fb[iv];
    return;
  }
  Us[IRHO] = rhostar; Us[1] = rhostar * ustar; Us[2] = rhostar * vx2s; if (three) Us[3] = rhostar * vx3s;
  Us[ip] = rhoes;
  for (int iv = ias; iv < nv; ++iv) Us[iv] = rhostar * q[iv];
  Ubs[0] = bx1; Ubs[1] = bx2s; Ubs[2] = bx3s;
  if (single) {
    for (int iv = 0; iv < nv; ++iv) flux[iv] = f[iv] + s * (Us[iv] - U[iv]);
    for (int iv = 0; iv < nb; ++iv) fluxb[iv] = fb[iv] + s * (Ubs[iv] - Ub[iv]);
    return;
  }
  double sst = left ? sstarL : sstarR;
  Uss[IRHO] = rhostar; Uss[1] = rhostar * ustar; Uss[2] = rhostar * vx22star; if (three) Uss[3] = rhostar * vx32star;
  Uss[ip] = rhoe2s;
  for (int iv = ias; iv < nv; ++iv) Uss[iv] = rhostar * q[iv];
  Ubss[0] = bx1; Ubss[1] = bx22star; Ubss[2] = bx32star;
  for (int iv = 0; iv < nv; ++iv) {
    double d0 = Us[iv];
    flux[iv] = f[iv] + s * (d0 - U[iv]) + sst * (Uss[iv] - d0);
  }
  for (int iv = 0; iv < nb; ++iv) {
    double d0 = Ubs[iv];
    fluxb[iv] = fb[iv] + s * (d0 - Ub[iv]) + sst * (Ubss[iv] - d0);
  }
}

/* ---------------------------------------------------------------- ghost fill */
/* Periodic wrap / reflective mirror of one index (1-based interior 1..n). */
static inline int map_idx(int i, int n, int bcl, int bcu, int *flip) {
  if (i < 1) {
    if (bcl == PHLO_BC_PERIODIC) return i + n;
    *flip = 1; return 1 - i;
  }
  if (i > n) {
    if (bcu == PHLO_BC_PERIODIC) return i - n;
    *flip = 1; return n - (i - n - 1);
  }
  return i;
}

/* Fill every ghost cell of a cell array with its periodic/reflective image.  Equivalent to
 * communicate_ndarray with corners on one brick followed by the reflective BC loops: each
 * ghost coordinate maps independently and vector component d flips under a mirror in d.
 * vec_kind: 0 none, 1 = velocity components at 1..sdims (prim), 2 = components 0..sdims-1 (B). */
static void fill_ghosts(const phlo_grid *g, double *a, int nv, int vec_kind) {
  shp s = cellg(g, nv);
  int n[3] = {g->nx1, g->nx2, g->nx3};
  for (int k = s.lo[2]; k <= s.hi[2]; ++k)
    for (int j = s.lo[1]; j <= s.hi[1]; ++j)
      for (int i = s.lo[0]; i <= s.hi[0]; ++i) {
        int c[3] = {i, j, k};
        int inside = 1;
        for (int d = 0; d < g->sdims; ++d) if (c[d] < 1 || c[d] > n[d]) inside = 0;
        if (inside) continue;
        int src[3] = {i, j, k}, flip[3] = {0, 0, 0};
        for (int d = 0; d < g->sdims; ++d) src[d] = map_idx(c[d], n[d], g->bc[d][0], g->bc[d][1], &flip[d]);
        for (int iv = 0; iv < nv; ++iv) {
          double v = a[OFF(&s, iv, src[0], src[1], src[2])];
          int d = -1;
          if (vec_kind == 1 && iv >= 1 && iv <= g->sdims) d = iv - 1;
          if (vec_kind == 2 && iv < g->sdims) d = iv;
          if (d >= 0 && flip[d]) v = -1.0 * v;
          a[OFF(&s, iv, i, j, k)] = v;
        }
      }
}

/* ---------------------------------------------------------------- helpers */
/* Face values (lo = left edge, hi = right edge) of the centre cell qc from its neighbours, by the
 * reference's reconstructions: LIM2ND_REC (source.F90:8141-8181), PPH_REC (8183-8259: third
 * order, limited only when `limited`), LIM5TH_REC (8261-8323: fifth order, always limited). */
static void rec_cell(int rec, int limited, double qmm, double qm, double qc, double qp, double qpp,
                     double *lo, double *hi) {
  if (rec == 0) {
    double slopef = qp - qc, slopeb = qc - qm, prod = slopef * slopeb, slope = 0.0;
    if (prod > 0.0) slope = prod / (slopef + slopeb);
    double tmp = 0.5 * slope;
    *lo = qc - tmp;
    *hi = qc + tmp;
    return;
  }
  double am, ap;
  if (rec == 1) {
    double tmp = (5.0 / 6.0) * qc;
    am = (1.0 / 3.0) * qm + tmp - (1.0 / 6.0) * qp;
    ap = -(1.0 / 6.0) * qm + tmp + (1.0 / 3.0) * qp;
    if (!limited) {
      *lo = am;
      *hi = ap;
      return;
    }
  } else {
    double tmp = 329.0 * qc;
    am = (-21.0 * qmm + 189.0 * qm + tmp - 91.0 * qp + 14.0 * qpp) * (1.0 / 420.0);
    ap = (14.0 * qmm - 91.0 * qm + tmp + 189.0 * qp - 21.0 * qpp) * (1.0 / 420.0);
  }
  double mn = fmin(qm, qc), mx = fmax(qm, qc);
  if (am < mn) am = mn;
  if (am > mx) am = mx;
  mn = fmin(qc, qp);
  mx = fmax(qc, qp);
  if (ap < mn) ap = mn;
  if (ap > mx) ap = mx;
  am = am - qc;
  ap = ap - qc;
  if (ap * am >= 0.0) {
    ap = 0.0;
    am = 0.0;
  } else {
    if (fabs(ap) >= 2.0 * fabs(am)) ap = -2.0 * am;
    if (fabs(am) >= 2.0 * fabs(ap)) am = -2.0 * ap;
  }
  *lo = am + qc;
  *hi = ap + qc;
}


static void rk_coeffs(int stages, double c[3][3]) {
  memset(c, 0, sizeof(double) * 9);
  if (stages == 2) {
    c[0][0] = 1.0; c[0][1] = 0.0; c[0][2] = -1.0;
    c[1][0] = 0.5; c[1][1] = 0.5; c[1][2] = -0.5;
  } else {
    c[0][0] = 1.0; c[0][1] = 0.0; c[0][2] = -1.0;
    c[1][0] = 0.75; c[1][1] = 0.25; c[1][2] = -0.25;
    c[2][0] = 1.0 / 3.0; c[2][1] = 2.0 / 3.0; c[2][2] = -(2.0 / 3.0);
  }
}

/* ---------------------------------------------------------------- shock detector */
/* USE_SHOCK_FLATTENING (source.F90:8073-8136): a cell whose summed central pressure jumps
 * |p(+1) - p(-1)| over all directions exceed eps_sf times its own pressure flags itself and its
 * 3x3(x3) neighbours.  Pressures are full values (deviation + equilibrium under WB), ghosts
 * included; cells lx-2..ux+2 are tested, so the test reads 3 ghost layers.  The flags of cells
 * lx-1..ux+1 are what the sweeps read; every flag is recomputed here, each stage. */
static void detect_shocks(phlo_grid *g, scr_t *S) {
  const int ip = IP(g), three = g->sdims == 3;
  shp sc = cellg(g, g->nvars), s1 = cellg(g, 1), s3c = cellg(g, 3);
  const int kl = three ? -1 : 1, ku = three ? g->nx3 + 2 : g->nx3;
  memset(S->flat, 0, sizeof(double) * (size_t)ssize(&s1));
#define PF(i, j, k) (g->wb ? g->prim[OFF(&sc, ip, i, j, k)] + g->eq_prim_cc[OFF(&s3c, 1, i, j, k)] \
                           : g->prim[OFF(&sc, ip, i, j, k)])
  for (int k = kl; k <= ku; ++k)
    for (int j = -1; j <= g->nx2 + 2; ++j)
      for (int i = -1; i <= g->nx1 + 2; ++i) {
        double tmp;
        if (three)
          tmp = (fabs(PF(i, j, k + 1) - PF(i, j, k - 1)) + fabs(PF(i, j + 1, k) - PF(i, j - 1, k)) +
                 fabs(PF(i + 1, j, k) - PF(i - 1, j, k))) / PF(i, j, k);
        else
          tmp = (fabs(PF(i, j + 1, k) - PF(i, j - 1, k)) + fabs(PF(i + 1, j, k) - PF(i - 1, j, k))) / PF(i, j, k);
        if (tmp > g->eps_sf) {
          for (int c = three ? -1 : 0; c <= (three ? 1 : 0); ++c)
            for (int b = -1; b <= 1; ++b)
              for (int a = -1; a <= 1; ++a) S->flat[OFF(&s1, 0, i + a, j + b, k + c)] = 1.0;
        }
      }
#undef PF
}

/* ---------------------------------------------------------------- one directional sweep */
static void sweep(phlo_grid *g, scr_t *S, int dir) {
  const int nv = g->nvars, ip = IP(g), sd = g->sdims, G = g->ngc;
  const int n[3] = {g->nx1, g->nx2, g->nx3};
  const double inv_dl = dir == 0 ? g->inv_dx1 : (dir == 1 ? g->inv_dx2 : g->inv_dx3);
  shp sc = cellg(g, nv), sb = cellg(g, sd), s1 = cellg(g, 1), s2 = cellg(g, 2), s3 = cellg(g, 3);
  shp sin_ = interior(g, nv), sf3 = face(g, 3, dir), sf1 = face(g, 1, dir);
  shp sbf = bface(g, 1, dir), se = bface(g, 3, dir);
  shp st1 = cellg(g, 1);
  const int helm_nf = g->helm && !g->fasteos; /* Helmholtz without USE_FASTEOS */
  (void)s3; (void)G;
  int ta = dir == 0 ? 1 : 0, tb = dir == 2 ? 1 : 2; /* transverse axes */
  int nl = n[dir];
  long nlines = (long)n[ta] * n[tb];

#pragma omp parallel num_threads(g->nthreads > 0 ? g->nthreads : omp_get_max_threads())
  {
    double *W = (double *)malloc(sizeof(double) * (size_t)nv * (nl + 6));
    double *Bc = (double *)malloc(sizeof(double) * 3 * (size_t)(nl + 6));
    double *Gf = (double *)malloc(sizeof(double) * 2 * (size_t)(nl + 6));
    double *qL = (double *)malloc(sizeof(double) * (size_t)nv * (nl + 2));
    double *qR = (double *)malloc(sizeof(double) * (size_t)nv * (nl + 2));
    double *fx = (double *)malloc(sizeof(double) * (size_t)nv * (nl + 2));
    double *bL = (double *)malloc(sizeof(double) * 3 * (size_t)(nl + 2));
    double *bR = (double *)malloc(sizeof(double) * 3 * (size_t)(nl + 2));
    double *fb = (double *)malloc(sizeof(double) * 3 * (size_t)(nl + 2));
    double *gL = (double *)malloc(sizeof(double) * 2 * (size_t)(nl + 2));
    double *gR = (double *)malloc(sizeof(double) * 2 * (size_t)(nl + 2));
    int *Fl = (int *)malloc(sizeof(int) * (size_t)(nl + 2));
#pragma omp for schedule(static)
    for (long line = 0; line < nlines; ++line) {
      int t0 = 1 + (int)(line % n[ta]), t1 = 1 + (int)(line / n[ta]);
      int c[3];
      c[ta] = t0; c[tb] = t1;
      if (sd == 2) c[2] = 1;
      /* gather the line: cells 1-ng .. n+ng (ng = 3 for LIM5TH, 2 otherwise) -> W[(m+2)*nv] */
      const int ngl = g->rec == 2 ? 3 : 2;
      for (int m = 1 - ngl; m <= nl + ngl; ++m) {
        c[dir] = m;
        for (int iv = 0; iv < nv; ++iv) W[(m + 2) * nv + iv] = g->prim[OFF(&sc, iv, c[0], c[1], c[2])];
        if (g->mhd) for (int iv = 0; iv < sd; ++iv) Bc[(m + 2) * 3 + iv] = g->b_cc[OFF(&sb, iv, c[0], c[1], c[2])];
        if (g->fasteos) for (int iv = 0; iv < 2; ++iv) Gf[(m + 2) * 2 + iv] = g->gammaf[OFF(&s2, iv, c[0], c[1], c[2])];
        if (helm_nf) Gf[(m + 2) * 2] = g->temp[OFF(&st1, 0, c[0], c[1], c[2])];
      }
#define WC(m) (W + ((m) + 2) * nv)
      /* is_flattened of cells 0..n+1 of the line (USE_SHOCK_FLATTENING) */
      for (int m = 0; m <= nl + 1; ++m) {
        c[dir] = m;
        Fl[m] = g->sf ? (int)S->flat[OFF(&st1, 0, c[0], c[1], c[2])] : 0;
      }
      /* reconstruction over cells 0..n+1: face f=m is the low face of cell m */
      for (int m = 0; m <= nl + 1; ++m) {
        for (int iv = 0; iv < nv; ++iv) {
          const int limited = g->rec == 2 || (g->rec == 1 && iv >= IAS1(g));
          double lo, hi;
          rec_cell(g->rec, limited, g->rec == 2 ? WC(m - 2)[iv] : 0.0, WC(m - 1)[iv], WC(m)[iv], WC(m + 1)[iv],
                   g->rec == 2 ? WC(m + 2)[iv] : 0.0, &lo, &hi);
          /* a flagged cell falls back to LIM2ND PLM (source.F90:8743-8789, 9635-9668) */
          if (Fl[m]) rec_cell(0, 1, 0.0, WC(m - 1)[iv], WC(m)[iv], WC(m + 1)[iv], 0.0, &lo, &hi);
          if (m >= 1) qR[m * nv + iv] = lo;
          if (m <= nl) qL[(m + 1) * nv + iv] = hi;
        }
      }
#define BC(m, iv) Bc[((m) + 2) * 3 + (iv)]
      if (g->mhd) {
        /* transverse B from b_cc (PPH unlimited), normal B = face value */
        for (int m = 0; m <= nl + 1; ++m) {
          for (int iv = 0; iv < sd; ++iv) {
            if (iv == dir) continue;
            double lo, hi;
            rec_cell(g->rec, g->rec == 2, g->rec == 2 ? BC(m - 2, iv) : 0.0, BC(m - 1, iv), BC(m, iv), BC(m + 1, iv),
                     g->rec == 2 ? BC(m + 2, iv) : 0.0, &lo, &hi);
            if (Fl[m]) rec_cell(0, 1, 0.0, BC(m - 1, iv), BC(m, iv), BC(m + 1, iv), 0.0, &lo, &hi);
            if (m >= 1) bR[m * 3 + iv] = lo;
            if (m <= nl) bL[(m + 1) * 3 + iv] = hi;
          }
        }
        for (int f = 1; f <= nl + 1; ++f) {
          c[dir] = f;
          double tmp = g->b_x[dir][OFF(&sbf, 0, c[0], c[1], c[2])];
          bL[f * 3 + dir] = tmp;
          bR[f * 3 + dir] = tmp;
        }
      }
      /* rotate into the normal frame */
      for (int f = 1; f <= nl + 1; ++f) {
        double *a[2] = {qL + f * nv, qR + f * nv};
        for (int s = 0; s < 2; ++s) {
          double *q = a[s];
          if (dir == 1) { double v1 = q[1], v2 = q[2]; q[1] = v2; q[2] = -v1; }
          if (dir == 2) { double v1 = q[1], v2 = q[2], v3 = q[3]; q[1] = v3; q[2] = v1; q[3] = v2; }
        }
        if (g->mhd) {
          double *b[2] = {bL + f * 3, bR + f * 3};
          for (int s = 0; s < 2; ++s) {
            double *q = b[s];
            if (dir == 1) { double v1 = q[0], v2 = q[1]; q[0] = v2; q[1] = -v1; }
            if (dir == 2) { double v1 = q[0], v2 = q[1], v3 = q[2]; q[0] = v3; q[1] = v1; q[2] = v2; }
          }
        }
      }
      /* WB add-back of the face equilibrium (source.F90:8473-8486) */
      if (g->wb) {
        for (int f = 1; f <= nl + 1; ++f) {
          c[dir] = f;
          double rho_eq = g->eq_prim_x[dir][OFF(&sf3, 0, c[0], c[1], c[2])];
          double p_eq = g->eq_prim_x[dir][OFF(&sf3, 1, c[0], c[1], c[2])];
          qL[f * nv + IRHO] = qL[f * nv + IRHO] + rho_eq;
          qR[f * nv + IRHO] = qR[f * nv + IRHO] + rho_eq;
          qL[f * nv + ip] = qL[f * nv + ip] + p_eq;
          qR[f * nv + ip] = qR[f * nv + ip] + p_eq;
        }
      }
      /* FASTEOS gamma_e, gamma_c reconstruction + WB add-back (source.F90:8497-8729) */
      if (g->fasteos) {
#define GF(m, iv) Gf[((m) + 2) * 2 + (iv)]
        /* the x1 sweep flattens its gammas after the WB add-back (below); x2 and x3 before it
         * (source.F90:9993-10031, 11135-11173) */
        const int sf_late = g->sf && g->wb && dir == 0;
        for (int iv = 0; iv < 2; ++iv) {
          for (int m = 0; m <= nl + 1; ++m) {
            double lo, hi;
            rec_cell(g->rec, g->rec == 2, g->rec == 2 ? GF(m - 2, iv) : 0.0, GF(m - 1, iv), GF(m, iv), GF(m + 1, iv),
                     g->rec == 2 ? GF(m + 2, iv) : 0.0, &lo, &hi);
            if (Fl[m] && !sf_late) rec_cell(0, 1, 0.0, GF(m - 1, iv), GF(m, iv), GF(m + 1, iv), 0.0, &lo, &hi);
            if (m >= 1) gR[m * 2 + iv] = lo;
            if (m <= nl) gL[(m + 1) * 2 + iv] = hi;
          }
        }
        if (g->wb) {
          for (int f = 1; f <= nl + 1; ++f) {
            c[dir] = f;
            double p_eq = g->eq_gammae_x[dir][OFF(&sf1, 0, c[0], c[1], c[2])];
            gL[f * 2] = gL[f * 2] + p_eq;
            gR[f * 2] = gR[f * 2] + p_eq;
          }
        }
        if (sf_late) {
          /* x1 sweep (source.F90:8829-8872): a flagged cell's PLM gammas replace its edge values
           * without the equilibrium gamma_e, and eq_gammae_x1 of that face is added once more to
           * the value on the OTHER side of the face; cells in ascending order */
          for (int m = 0; m <= nl + 1; ++m) {
            if (!Fl[m]) continue;
            double lo[2], hi[2];
            for (int iv = 0; iv < 2; ++iv) rec_cell(0, 1, 0.0, GF(m - 1, iv), GF(m, iv), GF(m + 1, iv), 0.0, &lo[iv], &hi[iv]);
            if (m >= 1) {
              for (int iv = 0; iv < 2; ++iv) gR[m * 2 + iv] = lo[iv];
              c[dir] = m;
              gL[m * 2] = gL[m * 2] + g->eq_gammae_x[dir][OFF(&sf1, 0, c[0], c[1], c[2])];
            }
            if (m <= nl) {
              for (int iv = 0; iv < 2; ++iv) gL[(m + 1) * 2 + iv] = hi[iv];
              c[dir] = m + 1;
              gR[(m + 1) * 2] = gR[(m + 1) * 2] + g->eq_gammae_x[dir][OFF(&sf1, 0, c[0], c[1], c[2])];
            }
          }
        }
      }
      /* without FASTEOS: the face temperature guess 1/2 (T(i-1) + T(i)) (source.F90:8488-8495) */
      if (helm_nf)
        for (int f = 1; f <= nl + 1; ++f) {
          double tf = 0.5 * (Gf[(f + 1) * 2] + Gf[(f + 2) * 2]);
          gL[f * 2] = tf;
          gR[f * 2] = tf;
        }
      /* Riemann solver per face */
      for (int f = 1; f <= nl + 1; ++f) {
        const int thermo = g->fasteos || helm_nf;
        const double *gl = thermo ? gL + f * 2 : NULL, *gr = thermo ? gR + f * 2 : NULL;
        const int flat = Fl[f - 1] || Fl[f]; /* source.F90:8732-8739 */
        if (g->mhd)
          phlo_riemann_mhd(g, qL + f * nv, qR + f * nv, bL + f * 3, bR + f * 3, gl, gr, fx + f * nv, fb + f * 3,
                           flat);
        else
          phlo_riemann_hydro(g, qL + f * nv, qR + f * nv, gl, gr, fx + f * nv, flat);
      }
      /* rotate fluxes back */
      for (int f = 1; f <= nl + 1; ++f) {
        double *q = fx + f * nv;
        if (dir == 1) { double v1 = q[1], v2 = q[2]; q[1] = -v2; q[2] = v1; }
        if (dir == 2) { double v1 = q[1], v2 = q[2], v3 = q[3]; q[1] = v2; q[2] = v3; q[3] = v1; }
        if (g->mhd) {
          double *b = fb + f * 3;
          if (dir == 1) { double v1 = b[0], v2 = b[1]; b[0] = -v2; b[1] = v1; }
          if (dir == 2) { double v1 = b[0], v2 = b[1], v3 = b[2]; b[0] = v2; b[1] = v3; b[2] = v1; }
        }
      }
      /* face EMFs and mass-flux signs (source.F90:8926-8951, 10113-10144, 11255-11286) */
      if (g->mhd) {
        for (int f = 1; f <= nl + 1; ++f) {
          c[dir] = f;
          double *e = S->emf[dir] + OFF(&se, 0, c[0], c[1], c[2]);
          double *b = fb + f * 3;
          if (dir == 0) { if (sd == 3) e[1] = b[2]; e[2] = -b[1]; }
          if (dir == 1) { if (sd == 3) e[0] = -b[2]; e[2] = b[0]; }
          if (dir == 2) { e[0] = b[1]; e[1] = -b[0]; }
          double tmp = 0.5 * (qL[f * nv + IRHO] + qR[f * nv + IRHO]) * g->smax;
          double mach = fx[f * nv + IRHO] / tmp, sgn = 0.0;
          if (mach > g->mach_ct) sgn = 1.0;
          if (mach < -g->mach_ct) sgn = -1.0;
          S->sgn[dir][OFF(&sbf, 0, c[0], c[1], c[2])] = sgn;
        }
      }
      /* WB momentum-flux fix and total-energy potential flux */
      for (int f = 1; f <= nl + 1; ++f) {
        c[dir] = f;
        if (g->wb) fx[f * nv + IVX(dir)] = fx[f * nv + IVX(dir)] - g->eq_prim_x[dir][OFF(&sf3, 1, c[0], c[1], c[2])];
      }
      if (g->etot) {
        for (int f = 1; f <= nl + 1; ++f) {
          c[dir] = f;
          fx[f * nv + ip] = fx[f * nv + ip] + fx[f * nv + IRHO] * g->phi_x[dir][OFF(&sf1, 0, c[0], c[1], c[2])];
        }
      }
      /* flux divergence */
      for (int m = 1; m <= nl; ++m) {
        c[dir] = m;
        double *r = S->res + OFF(&sin_, 0, c[0], c[1], c[2]);
        for (int iv = 0; iv < nv; ++iv) {
          double d = (fx[(m + 1) * nv + iv] - fx[m * nv + iv]) * inv_dl;
          r[iv] = dir == 0 ? d : r[iv] + d;
        }
      }
#undef WC
    }
    free(W); free(Bc); free(Gf); free(qL); free(qR); free(fx); free(bL); free(bR); free(fb); free(gL); free(gR); free(Fl);
  }
  (void)s1;
}

/* ---------------------------------------------------------------- EMF ghosts, CT */
static void emf_ghosts(phlo_grid *g, scr_t *S) {
  const int sd = g->sdims;
  const int n[3] = {g->nx1, g->nx2, g->nx3};
  /* periodic self-copy without corners: along every periodic dimension d2 != face dim,
   * ghost layer 0 <- n, n+1 <- 1, over the interior range of the other dims */
  for (int d = 0; d < sd; ++d) {
    shp se = bface(g, 3, d), sb = bface(g, 1, d);
    for (int d2 = 0; d2 < sd; ++d2) {
      if (g->bc[d2][0] != PHLO_BC_PERIODIC) continue;
      int hi[3] = {n[0], n[1], sd == 3 ? n[2] : 1};
      hi[d] += 1;
      int lo[3] = {1, 1, 1};
      /* copy along d2 (the face dimension d2==d uses the reference's range lx..ux+1) */
      int ext = hi[d2];
      for (int k = lo[2]; k <= hi[2]; ++k)
        for (int j = lo[1]; j <= hi[1]; ++j)
          for (int i = lo[0]; i <= hi[0]; ++i) {
            int c[3] = {i, j, k};
            if (c[d2] != ext && c[d2] != 1) continue;
            if (c[d2] == ext) {
              int t[3] = {i, j, k}; t[d2] = 0;
              for (int iv = 0; iv < 3; ++iv) S->emf[d][OFF(&se, iv, t[0], t[1], t[2])] = S->emf[d][OFF(&se, iv, i, j, k)];
              S->sgn[d][OFF(&sb, 0, t[0], t[1], t[2])] = S->sgn[d][OFF(&sb, 0, i, j, k)];
            }
            if (c[d2] == 1) {
              int t[3] = {i, j, k}; t[d2] = ext + 1;
              for (int iv = 0; iv < 3; ++iv) S->emf[d][OFF(&se, iv, t[0], t[1], t[2])] = S->emf[d][OFF(&se, iv, i, j, k)];
              S->sgn[d][OFF(&sb, 0, t[0], t[1], t[2])] = S->sgn[d][OFF(&sb, 0, i, j, k)];
            }
          }
    }
  }
  /* reflective EMF BCs (source.F90:11396-11964): for a wall normal to d2, the EMFs of the
   * transverse face arrays get factor +1 on component d2 and -1 on the others */
  for (int d2 = 0; d2 < sd; ++d2) {
    for (int side = 0; side < 2; ++side) {
      if (g->bc[d2][side] != PHLO_BC_REFLECTIVE) continue;
      double fac[3] = {-1.0, -1.0, -1.0};
      fac[d2] = 1.0;
      for (int d = 0; d < sd; ++d) {
        if (d == d2) continue;
        shp se = bface(g, 3, d), sb = bface(g, 1, d);
        int hi[3] = {n[0], n[1], sd == 3 ? n[2] : 1};
        hi[d] += 1;
        int gi = side == 0 ? 0 : n[d2] + 1, si = side == 0 ? 1 : n[d2];
        for (int k = 1; k <= hi[2]; ++k)
          for (int j = 1; j <= hi[1]; ++j)
            for (int i = 1; i <= hi[0]; ++i) {
              int c[3] = {i, j, k};
              if (c[d2] != 1) continue; /* iterate the wall plane once */
              int t[3] = {i, j, k}, s[3] = {i, j, k};
              t[d2] = gi; s[d2] = si;
              for (int iv = 0; iv < 3; ++iv)
                S->emf[d][OFF(&se, iv, t[0], t[1], t[2])] = fac[iv] * S->emf[d][OFF(&se, iv, s[0], s[1], s[2])];
              S->sgn[d][OFF(&sb, 0, t[0], t[1], t[2])] = S->sgn[d][OFF(&sb, 0, s[0], s[1], s[2])];
            }
      }
    }
  }
}

/* cell-centred -v x B component along axis a at cell (i,j,k) as the reference writes it */
static double emf_cc(const phlo_grid *g, int a, int i, int j, int k) {
  shp sc = cellg(g, g->nvars), sb = cellg(g, g->sdims);
  double *P = g->prim, *B = g->b_cc;
#define PV(d) P[OFF(&sc, IVX(d), i, j, k)]
#define BB(d) B[OFF(&sb, d, i, j, k)]
  if (a == 2) return -PV(0) * BB(1) + PV(1) * BB(0);
  if (a == 0) return PV(2) * BB(1) - PV(1) * BB(2);
  return PV(0) * BB(2) - PV(2) * BB(0);
#undef PV
#undef BB
}

static void ct_update(phlo_grid *g, scr_t *S, double a1, double a2, double a3) {
  const int sd = g->sdims;
  const int nx1 = g->nx1, nx2 = g->nx2, nx3 = g->nx3;
  /* corner EMFs (source.F90:11970-12027 for z; 12050-12107 x; 12128-12185 y).  For corner
   * axis a with in-plane axes (p, q): N/S are the p-face EMFs at q and q-1, E/W the q-face
   * EMFs at p and p-1. */
  for (int a = 0; a < 3; ++a) {
    if (sd == 2 && a != 2) continue;
    int pa, qa;
    if (a == 2) { pa = 0; qa = 1; } else if (a == 0) { pa = 1; qa = 2; } else { pa = 2; qa = 0; }
    shp sp = bface(g, 3, pa), sq = bface(g, 3, qa), spb = bface(g, 1, pa), sqb = bface(g, 1, qa);
    shp sc = corner(g, a);
#pragma omp parallel for collapse(2) num_threads(g->nthreads > 0 ? g->nthreads : omp_get_max_threads())
    for (int k = sc.lo[2]; k <= sc.hi[2]; ++k)
      for (int j = sc.lo[1]; j <= sc.hi[1]; ++j)
        for (int i = sc.lo[0]; i <= sc.hi[0]; ++i) {
          int c[3] = {i, j, k};
          int cqm[3] = {i, j, k}; cqm[qa] -= 1;  /* shift -1 along q */
          int cpm[3] = {i, j, k}; cpm[pa] -= 1;  /* shift -1 along p */
          int cpq[3] = {i, j, k}; cpq[pa] -= 1; cpq[qa] -= 1;
          double emf_N = S->emf[pa][OFF(&sp, a, c[0], c[1], c[2])];
          double emf_E = S->emf[qa][OFF(&sq, a, c[0], c[1], c[2])];
          double emf_S = S->emf[pa][OFF(&sp, a, cqm[0], cqm[1], cqm[2])];
          double emf_W = S->emf[qa][OFF(&sq, a, cpm[0], cpm[1], cpm[2])];
          double emf_SW = emf_cc(g, a, cpq[0], cpq[1], cpq[2]);
          double emf_NW = emf_cc(g, a, cpm[0], cpm[1], cpm[2]);
          double emf_NE = emf_cc(g, a, c[0], c[1], c[2]);
          double emf_SE = emf_cc(g, a, cqm[0], cqm[1], cqm[2]);
          double sgn = S->sgn[pa][OFF(&spb, 0, cqm[0], cqm[1], cqm[2])];
          double demf_S = 0.5 * (1.0 + sgn) * (emf_W - emf_SW) + 0.5 * (1.0 - sgn) * (emf_E - emf_SE);
          sgn = S->sgn[pa][OFF(&spb, 0, c[0], c[1], c[2])];
          double demf_N = 0.5 * (1.0 + sgn) * (emf_NW - emf_W) + 0.5 * (1.0 - sgn) * (emf_NE - emf_E);
          sgn = S->sgn[qa][OFF(&sqb, 0, cpm[0], cpm[1], cpm[2])];
          double demf_W = 0.5 * (1.0 + sgn) * (emf_S - emf_SW) + 0.5 * (1.0 - sgn) * (emf_N - emf_NW);
          sgn = S->sgn[qa][OFF(&sqb, 0, c[0], c[1], c[2])];
          double demf_E = 0.5 * (1.0 + sgn) * (emf_SE - emf_S) + 0.5 * (1.0 - sgn) * (emf_NE - emf_N);
          S->cor[a][OFF(&sc, 0, i, j, k)] =
              0.25 * (emf_S + emf_W + emf_N + emf_E + demf_S - demf_N + demf_W - demf_E);
        }
  }
  /* face-B update (source.F90:12208-12437) */
  shp c3 = corner(g, 2), c1 = corner(g, 0), c2 = corner(g, 1);
#define E3(i, j, k) S->cor[2][OFF(&c3, 0, i, j, k)]
#define E1(i, j, k) S->cor[0][OFF(&c1, 0, i, j, k)]
#define E2(i, j, k) S->cor[1][OFF(&c2, 0, i, j, k)]
  {
    shp sb = bface(g, 1, 0), sf = face(g, 1, 0);
    for (int k = 1; k <= nx3; ++k)
      for (int j = 1; j <= nx2; ++j)
        for (int i = 1; i <= nx1 + 1; ++i) {
          double tmp;
          if (sd == 2) tmp = (E3(i, j + 1, k) - E3(i, j, k)) * g->inv_dx2;
          else tmp = -(E2(i, j, k + 1) - E2(i, j, k)) * g->inv_dx3 + (E3(i, j + 1, k) - E3(i, j, k)) * g->inv_dx2;
          double *b = &g->b_x[0][OFF(&sb, 0, i, j, k)];
          *b = a1 * S->b0[0][OFF(&sf, 0, i, j, k)] + a2 * (*b) + a3 * tmp;
        }
  }
  {
    shp sb = bface(g, 1, 1), sf = face(g, 1, 1);
    for (int k = 1; k <= nx3; ++k)
      for (int j = 1; j <= nx2 + 1; ++j)
        for (int i = 1; i <= nx1; ++i) {
          double tmp;
          if (sd == 2) tmp = (E3(i, j, k) - E3(i + 1, j, k)) * g->inv_dx1;
          else tmp = (E1(i, j, k + 1) - E1(i, j, k)) * g->inv_dx3 + (E3(i, j, k) - E3(i + 1, j, k)) * g->inv_dx1;
          double *b = &g->b_x[1][OFF(&sb, 0, i, j, k)];
          *b = a1 * S->b0[1][OFF(&sf, 0, i, j, k)] + a2 * (*b) + a3 * tmp;
        }
  }
  if (sd == 3) {
    shp sb = bface(g, 1, 2), sf = face(g, 1, 2);
    for (int k = 1; k <= nx3 + 1; ++k)
      for (int j = 1; j <= nx2; ++j)
        for (int i = 1; i <= nx1; ++i) {
          double tmp = (E2(i + 1, j, k) - E2(i, j, k)) * g->inv_dx1 - (E1(i, j + 1, k) - E1(i, j, k)) * g->inv_dx2;
          double *b = &g->b_x[2][OFF(&sb, 0, i, j, k)];
          *b = a1 * S->b0[2][OFF(&sf, 0, i, j, k)] + a2 * (*b) + a3 * tmp;
        }
  }
#undef E1
#undef E2
#undef E3
  /* b_cc = face average (source.F90:12439-12487) */
  shp scb = cellg(g, sd);
  for (int d = 0; d < sd; ++d) {
    shp sb = bface(g, 1, d);
    for (int k = 1; k <= nx3; ++k)
      for (int j = 1; j <= nx2; ++j)
        for (int i = 1; i <= nx1; ++i) {
          int u[3] = {i, j, k}; u[d] += 1;
          g->b_cc[OFF(&scb, d, i, j, k)] =
              0.5 * (g->b_x[d][OFF(&sb, 0, u[0], u[1], u[2])] + g->b_x[d][OFF(&sb, 0, i, j, k)]);
        }
  }
}

/* ---------------------------------------------------------------- public step routines */
void phlo_init_thermo(phlo_grid *g) {
  shp sc = cellg(g, g->nvars), s1 = cellg(g, 1), s2 = cellg(g, 2);
  if (g->mhd) {
    /* time_loop computes b_cc from the face fields before step 0 (source.F90:6012-6062) */
    shp scb = cellg(g, g->sdims);
    for (int d = 0; d < g->sdims; ++d) {
      shp sb = bface(g, 1, d);
      for (int k = 1; k <= g->nx3; ++k)
        for (int j = 1; j <= g->nx2; ++j)
          for (int i = 1; i <= g->nx1; ++i) {
            int u[3] = {i, j, k}; u[d] += 1;
            g->b_cc[OFF(&scb, d, i, j, k)] =
                0.5 * (g->b_x[d][OFF(&sb, 0, u[0], u[1], u[2])] + g->b_x[d][OFF(&sb, 0, i, j, k)]);
          }
    }
  }
  const double gm = g->gm, gmm1 = gm - 1.0, igmm1 = 1.0 / gmm1, inv_mu = 1.0 / g->mu;
  const int ip = IP(g), ias = IAS1(g);
#pragma omp parallel for collapse(2) num_threads(g->nthreads > 0 ? g->nthreads : omp_get_max_threads())
  for (int k = 1; k <= g->nx3; ++k)
    for (int j = 1; j <= g->nx2; ++j)
      for (int i = 1; i <= g->nx1; ++i) {
        double rho = g->prim[OFF(&sc, IRHO, i, j, k)], p = g->prim[OFF(&sc, ip, i, j, k)];
        double eint, T;
        if (g->helm) {
          double abar = 1.0 / g->prim[OFF(&sc, ias + 1, i, j, k)];
          double ye = g->prim[OFF(&sc, ias, i, j, k)];
          double zbar = abar * ye, sound;
          T = g->temp[OFF(&s1, 0, i, j, k)];
          phlo_helm_rhoP_given(g->eos, rho, p, abar, zbar, &T, &eint, &sound, g->fasteos);
          eint = rho * eint;
          if (g->fasteos) {
            g->gammaf[OFF(&s2, 0, i, j, k)] = p / eint + 1.0;
            g->gammaf[OFF(&s2, 1, i, j, k)] = sound * sound * rho / p;
          }
        } else {
          T = p / (CONST_RGAS * rho * inv_mu);
          eint = p * igmm1;
        }
        g->eint[OFF(&s1, 0, i, j, k)] = eint;
        g->temp[OFF(&s1, 0, i, j, k)] = T;
      }
}

void phlo_compute_hyperbolic_dt(phlo_grid *g) {
  shp sc = cellg(g, g->nvars), s1 = cellg(g, 1), sb = cellg(g, g->sdims);
  const double gm = g->gm;
  const int ip = IP(g), ias = IAS1(g), three = g->sdims == 3;
  double smax = 0.0;
#pragma omp parallel for collapse(2) reduction(max : smax) num_threads(g->nthreads > 0 ? g->nthreads : omp_get_max_threads())
  for (int k = 1; k <= g->nx3; ++k)
    for (int j = 1; j <= g->nx2; ++j)
      for (int i = 1; i <= g->nx1; ++i) {
        double rho = g->prim[OFF(&sc, IRHO, i, j, k)];
        double vx1 = g->prim[OFF(&sc, 1, i, j, k)], vx2 = g->prim[OFF(&sc, 2, i, j, k)];
        double vx3 = three ? g->prim[OFF(&sc, 3, i, j, k)] : 0.0;
        double p = g->prim[OFF(&sc, ip, i, j, k)], c;
        if (g->helm) {
          double ye = g->prim[OFF(&sc, ias, i, j, k)];
          double abar = 1.0 / g->prim[OFF(&sc, ias + 1, i, j, k)];
          double zbar = ye * abar, T = g->temp[OFF(&s1, 0, i, j, k)], ei, cv;
          phlo_helm_rhoT_given_full(g->eos, rho, T, abar, zbar, &p, &ei, &c, &cv);
        } else {
          c = sqrt(gm * p / rho);
        }
        if (g->mhd) {
          double bx1 = g->b_cc[OFF(&sb, 0, i, j, k)], bx2 = g->b_cc[OFF(&sb, 1, i, j, k)];
          double bx3 = three ? g->b_cc[OFF(&sb, 2, i, j, k)] : 0.0;
          double ca2 = bx1 * bx1 + bx2 * bx2 + bx3 * bx3;
          c = sqrt(c * c + ca2 / rho);
        }
        double sx1 = (fabs(vx1) + c) * g->inv_dx1;
        double sx2 = (fabs(vx2) + c) * g->inv_dx2;
        double s;
        if (three) {
          double sx3 = (fabs(vx3) + c) * g->inv_dx3;
          s = sx3 + sx1 + sx2;
        } else {
          s = sx1 + sx2;
        }
        smax = fmax(smax, s);
      }
  g->smax = smax;
  g->dt = g->cfl / smax;
}

void phlo_hydro_step(phlo_grid *g) {
  const int nv = g->nvars, ip = IP(g), ias = IAS1(g), sd = g->sdims, three = sd == 3;
  const double gm = g->gm, gmm1 = gm - 1.0, inv_mu = 1.0 / g->mu;
  scr_t S = carve(g);
  shp sc = cellg(g, nv), s1 = cellg(g, 1), s2 = cellg(g, 2), sb = cellg(g, sd), sin_ = interior(g, nv);
  shp sg = cellg(g, sd), s3c = cellg(g, 3);
  double rkc[3][3];
  rk_coeffs(g->rk_stages, rkc);
  const int nthr = g->nthreads > 0 ? g->nthreads : omp_get_max_threads();

  /* prim -> cons (source.F90:7057-7117) */
#pragma omp parallel for collapse(2) num_threads(nthr)
  for (int k = 1; k <= g->nx3; ++k)
    for (int j = 1; j <= g->nx2; ++j)
      for (int i = 1; i <= g->nx1; ++i) {
        double *w = g->prim + OFF(&sc, 0, i, j, k);
        double *u = S.state0 + OFF(&sin_, 0, i, j, k);
        double rho = w[IRHO], vx1 = w[1], vx2 = w[2], vx3 = three ? w[3] : 0.0;
        u[IRHO] = rho;
        u[1] = rho * vx1;
        u[2] = rho * vx2;
        if (three) u[3] = rho * vx3;
        double eint = g->eint[OFF(&s1, 0, i, j, k)];
        double rhoe = eint + 0.5 * rho * (vx1 * vx1 + vx2 * vx2 + vx3 * vx3);
        if (g->mhd) {
          double bx1 = g->b_cc[OFF(&sb, 0, i, j, k)], bx2 = g->b_cc[OFF(&sb, 1, i, j, k)];
          double bx3 = three ? g->b_cc[OFF(&sb, 2, i, j, k)] : 0.0;
          rhoe = rhoe + 0.5 * (bx1 * bx1 + bx2 * bx2 + bx3 * bx3);
        }
        if (g->etot) rhoe = rhoe + rho * g->phi_cc[OFF(&s1, 0, i, j, k)];
        u[ip] = rhoe;
        for (int iv = ias; iv < nv; ++iv) u[iv] = rho * w[iv];
      }
  memcpy(S.state, S.state0, sizeof(double) * (size_t)ssize(&sin_));
  if (g->mhd) {
    for (int d = 0; d < sd; ++d) {
      shp sf = face(g, 1, d), sbf = bface(g, 1, d);
      for (int k = sf.lo[2]; k <= sf.hi[2]; ++k)
        for (int j = sf.lo[1]; j <= sf.hi[1]; ++j)
          for (int i = sf.lo[0]; i <= sf.hi[0]; ++i)
            S.b0[d][OFF(&sf, 0, i, j, k)] = g->b_x[d][OFF(&sbf, 0, i, j, k)];
    }
  }

  for (int irk = 0; irk < g->rk_stages; ++irk) {
    /* WB deviations (source.F90:7151-7168) */
    if (g->wb) {
#pragma omp parallel for collapse(2) num_threads(nthr)
      for (int k = 1; k <= g->nx3; ++k)
        for (int j = 1; j <= g->nx2; ++j)
          for (int i = 1; i <= g->nx1; ++i) {
            double *w = g->prim + OFF(&sc, 0, i, j, k);
            w[IRHO] = w[IRHO] - g->eq_prim_cc[OFF(&s3c, 0, i, j, k)];
            w[ip] = w[ip] - g->eq_prim_cc[OFF(&s3c, 1, i, j, k)];
            if (g->fasteos)
              g->gammaf[OFF(&s2, 0, i, j, k)] = g->gammaf[OFF(&s2, 0, i, j, k)] - g->eq_gammae_cc[OFF(&s1, 0, i, j, k)];
          }
    }
    /* ghosts: periodic images and reflective mirrors */
    fill_ghosts(g, g->prim, nv, 1);
    if (g->mhd) fill_ghosts(g, g->b_cc, sd, 2);
    if (g->fasteos) fill_ghosts(g, g->gammaf, 2, 0);
    if (g->helm && !g->fasteos) fill_ghosts(g, g->temp, 1, 0);

    if (g->sf) detect_shocks(g, &S);
    for (int dir = 0; dir < sd; ++dir) sweep(g, &S, dir);

    double a1 = rkc[irk][0], a2 = rkc[irk][1], a3 = rkc[irk][2] * g->dt;

    if (g->mhd) {
      emf_ghosts(g, &S);
      ct_update(g, &S, a1, a2, a3);
    }
    /* gravity source: rho is the deviation under WB (source.F90:12606-12644); without
     * EVOLVE_ETOT the energy gains the work of gravity on the current RK state's momentum
     * (source.F90:12631-12638, the x3 term first in 3D) */
    if (g->gravity) {
#pragma omp parallel for collapse(2) num_threads(nthr)
      for (int k = 1; k <= g->nx3; ++k)
        for (int j = 1; j <= g->nx2; ++j)
          for (int i = 1; i <= g->nx1; ++i) {
            double rho = g->prim[OFF(&sc, IRHO, i, j, k)];
            double *r = S.res + OFF(&sin_, 0, i, j, k);
            for (int d = 0; d < sd; ++d) r[IVX(d)] = r[IVX(d)] - rho * g->grav[OFF(&sg, d, i, j, k)];
            if (!g->etot) {
              const double *u = S.state + OFF(&sin_, 0, i, j, k);
              double e = r[ip];
              if (three) e = e - u[3] * g->grav[OFF(&sg, 2, i, j, k)];
              e = e - u[1] * g->grav[OFF(&sg, 0, i, j, k)];
              e = e - u[2] * g->grav[OFF(&sg, 1, i, j, k)];
              r[ip] = e;
            }
          }
    }
    /* USE_CONSTANT_ACCELERATION: rho a from the current state (source.F90:12806-12836) */
    if (g->use_acc) {
#pragma omp parallel for collapse(2) num_threads(nthr)
      for (int k = 1; k <= g->nx3; ++k)
        for (int j = 1; j <= g->nx2; ++j)
          for (int i = 1; i <= g->nx1; ++i) {
            const double *u = S.state + OFF(&sin_, 0, i, j, k);
            double *r = S.res + OFF(&sin_, 0, i, j, k);
            double rho = u[IRHO];
            for (int d = 0; d < sd; ++d) r[IVX(d)] = r[IVX(d)] - rho * g->acc[d];
            double e = r[ip];
            if (three) e = e - u[3] * g->acc[2];
            e = e - u[1] * g->acc[0];
            e = e - u[2] * g->acc[1];
            r[ip] = e;
          }
    }
    /* RK combine + cons -> prim (+EoS) (source.F90:13518-13686) */
#pragma omp parallel for collapse(2) num_threads(nthr)
    for (int k = 1; k <= g->nx3; ++k)
      for (int j = 1; j <= g->nx2; ++j)
        for (int i = 1; i <= g->nx1; ++i) {
          double *u = S.state + OFF(&sin_, 0, i, j, k);
          const double *u0 = S.state0 + OFF(&sin_, 0, i, j, k), *r = S.res + OFF(&sin_, 0, i, j, k);
          for (int iv = 0; iv < nv; ++iv) u[iv] = a1 * u0[iv] + a2 * u[iv] + a3 * r[iv];
          double rho = u[IRHO], rhovx1 = u[1], rhovx2 = u[2], rhovx3 = three ? u[3] : 0.0, rhoe = u[ip];
          double inv_rho = 1.0 / rho;
          double eint = rhoe - 0.5 * (rhovx1 * rhovx1 + rhovx2 * rhovx2 + rhovx3 * rhovx3) * inv_rho;
          if (g->mhd) {
            double bx1 = g->b_cc[OFF(&sb, 0, i, j, k)], bx2 = g->b_cc[OFF(&sb, 1, i, j, k)];
            double bx3 = three ? g->b_cc[OFF(&sb, 2, i, j, k)] : 0.0;
            eint = eint - 0.5 * (bx1 * bx1 + bx2 * bx2 + bx3 * bx3);
          }
          if (g->etot) eint = eint - rho * g->phi_cc[OFF(&s1, 0, i, j, k)];
          double *w = g->prim + OFF(&sc, 0, i, j, k);
          w[IRHO] = rho;
          w[1] = rhovx1 * inv_rho;
          w[2] = rhovx2 * inv_rho;
          if (three) w[3] = rhovx3 * inv_rho;
          double p;
          if (g->helm) {
            double ye = u[ias] * inv_rho;
            double abar = rho / u[ias + 1];
            double zbar = ye * abar, sound;
            double T = g->temp[OFF(&s1, 0, i, j, k)];
            phlo_helm_rhoe_given(g->eos, rho, eint * inv_rho, abar, zbar, &T, &p, &sound, 1);
            if (g->fasteos) {
              g->gammaf[OFF(&s2, 0, i, j, k)] = p / eint + 1.0;
              g->gammaf[OFF(&s2, 1, i, j, k)] = sound * sound * rho / p;
            }
            w[ip] = p;
            g->temp[OFF(&s1, 0, i, j, k)] = T;
          } else {
            p = gmm1 * eint;
            w[ip] = p;
            g->temp[OFF(&s1, 0, i, j, k)] = p / (rho * CONST_RGAS * inv_mu);
          }
          g->eint[OFF(&s1, 0, i, j, k)] = eint;
          for (int iv = ias; iv < nv; ++iv) w[iv] = u[iv] * inv_rho;
        }
  }
}
