// phl_eos_fast.cuh -- Helmholtz (rho, e) -> T inversion for the split-precision form.
//
// Same mathematics as helm_rhoe_given / helm_rhoT_given2 / helm_rhoT_given_full
// (source/source.F90:23686-25019): biquintic Hermite interpolation of the free energy, Newton on
// E(T) = e with the reference's tolerance, iteration cap and out-of-table reset.  The evaluation
// order differs: the density is fixed during a solve, so for the current table cell the 36
// coefficients are contracted once with the density basis into A[ot][jt] (value) and B[ot][jt]
// (d/drho), ot = T-derivative order of the table variable, jt = lower/upper T node, and the
// quintic Hermite combination in T is rewritten once as the monomial coefficients of a quintic
// in y = (T - T0) / dT.  An iteration then evaluates f, df/dy and d2f/dy2 by one Horner pass
// (15 fused multiply-adds); the contraction is redone only when T leaves the cell.  Results
// agree with the reference evaluation to rounding.
#pragma once
#include "phl_device.cuh"

namespace phl {

// table node index (1-based like the reference) of x in the log-spaced nodes: an estimate in
// single precision (within one node of the cell for any x in the table's range), then exact
// comparisons against the node values
__device__ __forceinline__ int helm_node_index(const double *nodes, int n, double log10_first, double dlog,
                                               double x) {
  const float lx = __log2f((float)x) * 0.30102999566398120f;
  int i = (int)(__fdividef(lx - (float)log10_first, (float)dlog)) + 1;
  i = max(1, min(i, n - 1));
  if (i < n - 1 && __ldg(nodes + i) <= x) ++i;
  if (i > 1 && __ldg(nodes + i - 1) > x) --i;
  return i;
}

// The quintic Hermite bases of the table interpolation (source.F90:24708-24738) and their first
// derivatives, in nested (Horner) form with fused multiply-adds: the same polynomials as hb0 ..
// hb1m of phl_device.cuh, which keep the reference's term order for the FP64 form; here they
// cost about half the operations and agree to rounding.  They weight the density direction of
// the contraction; the temperature direction is a quintic in monomial form (helm_hermite_poly).
__device__ __forceinline__ void fhb0(double x, double d, double d2, double b[3]) {
  const double x2 = x * x;
  b[0] = fma(x2 * x, fma(x, fma(-6.0, x, 15.0), -10.0), 1.0);
  b[1] = x * fma(x2, fma(x, fma(-3.0, x, 8.0), -6.0), 1.0) * d;
  b[2] = 0.5 * x2 * fma(x, fma(x, 3.0 - x, -3.0), 1.0) * d2;
}
__device__ __forceinline__ void fhb0m(double om, double d, double d2, double b[3]) {
  const double o2 = om * om;
  b[0] = fma(o2 * om, fma(om, fma(-6.0, om, 15.0), -10.0), 1.0);
  b[1] = -(om * fma(o2, fma(om, fma(-3.0, om, 8.0), -6.0), 1.0)) * d;
  b[2] = 0.5 * o2 * fma(om, fma(om, 3.0 - om, -3.0), 1.0) * d2;
}
__device__ __forceinline__ void fhb1(double x, double id, double d, double b[3]) {
  const double x2 = x * x;
  b[0] = x2 * fma(x, fma(-30.0, x, 60.0), -30.0) * id;
  b[1] = fma(x2, fma(x, fma(-15.0, x, 32.0), -18.0), 1.0);
  b[2] = 0.5 * x * fma(x, fma(x, fma(-5.0, x, 12.0), -9.0), 2.0) * d;
}
__device__ __forceinline__ void fhb1m(double om, double id, double d, double b[3]) {
  const double o2 = om * om;
  b[0] = -(o2 * fma(om, fma(-30.0, om, 60.0), -30.0)) * id;
  b[1] = fma(o2, fma(om, fma(-15.0, om, 32.0), -18.0), 1.0);
  b[2] = -(0.5 * om * fma(om, fma(om, fma(-5.0, om, 12.0), -9.0), 2.0)) * d;
}
struct HelmCell {
  int ih, jh;
  double Ye, rhos, x, drho;
  double c[6];                          // f of the current T cell: sum of c[m] y^m
  double T0, dT, idT;                   // lower T node, spacing and its inverse, current T cell
};

// Monomial coefficients in y of the quintic Hermite interpolant in T with nodal values, first
// and second T-derivatives A[0..2][0] (lower node) and A[0..2][1] (upper node) over a cell of
// width dT.  The bases psi0(y) = 1 - 10y^3 + 15y^4 - 6y^5, psi1(y) = y - 6y^3 + 8y^4 - 3y^5,
// psi2(y) = (y^2 - 3y^3 + 3y^4 - y^5) / 2 (the functions of source.F90:24708-24738) and their
// mirror images psi(1 - y) expanded in powers of y; the nodal difference b0 - a0 is formed first,
// so the large cubic-to-quintic terms carry it instead of the values themselves.
__device__ __forceinline__ void helm_hermite_poly(const double A[3][2], double dT, double c[6]) {
  const double a0 = A[0][0], a1 = A[1][0] * dT, a2 = A[2][0] * (dT * dT);
  const double b1 = A[1][1] * dT, b2 = A[2][1] * (dT * dT), d0 = A[0][1] - a0;
  c[0] = a0;
  c[1] = a1;
  c[2] = 0.5 * a2;
  c[3] = fma(10.0, d0, fma(-6.0, a1, fma(-4.0, b1, fma(-1.5, a2, 0.5 * b2))));
  c[4] = fma(-15.0, d0, fma(8.0, a1, fma(7.0, b1, fma(1.5, a2, -b2))));
  c[5] = fma(6.0, d0, fma(-3.0, a1, fma(-3.0, b1, fma(-0.5, a2, 0.5 * b2))));
}

// p(y), p'(y) and p''(y) / 2 of the quintic sum c[m] y^m in one Horner pass
__device__ __forceinline__ void poly5_eval(const double c[6], double y, double &p, double &d1, double &d2h) {
  p = c[5];
  d1 = 0.0;
  d2h = 0.0;
#pragma unroll
  for (int m = 4; m >= 0; --m) {
    d2h = fma(d2h, y, d1);
    d1 = fma(d1, y, p);
    p = fma(p, y, c[m]);
  }
}

// coefficients of T order ot (variables {0,3,4}, {1,5,6}, {2,7,8}: value, d/drho, d2/drho2 of
// f, f_T, f_TT) at the lower/upper T node jt, contracted with a density basis (r0, r1)
__device__ __forceinline__ void helm_cell_contract_with(const HelmTable &h, const HelmCell &c, int jh,
                                                        const double r0[3], const double r1[3], double out[3][2]) {
  const int var[3][3] = {{0, 3, 4}, {1, 5, 6}, {2, 7, 8}};
#pragma unroll
  for (int jt = 0; jt < 2; ++jt) {
    const double *lo = h.tab + 9 * ((long long)(c.ih - 1) + (long long)h.nrho * (jh - 1 + jt));
    const double *hi = lo + 9;
#pragma unroll
    for (int ot = 0; ot < 3; ++ot) {
      double a = 0.0;
#pragma unroll
      for (int orr = 0; orr < 3; ++orr)
        a = fma(__ldg(lo + var[ot][orr]), r0[orr], fma(__ldg(hi + var[ot][orr]), r1[orr], a));
      out[ot][jt] = a;
    }
  }
}

// density basis (value) of the cell, recomputed where needed instead of kept in registers
__device__ __forceinline__ void helm_cell_rbasis(const HelmCell &c, double r0[3], double r1[3]) {
  fhb0(c.x, c.drho, c.drho * c.drho, r0);
  fhb0m(1.0 - c.x, c.drho, c.drho * c.drho, r1);
}

__device__ __forceinline__ void helm_cell_contract(const HelmTable &h, HelmCell &c, int jh) {
  c.jh = jh;
  c.T0 = __ldg(h.T + jh - 1);
  c.dT = __ldg(h.T + jh) - c.T0;
  c.idT = __ldg(h.inv_dT + jh - 1);
  double r0[3], r1[3], A[3][2];
  helm_cell_rbasis(c, r0, r1);
  helm_cell_contract_with(h, c, jh, r0, r1, A);
  helm_hermite_poly(A, c.dT, c.c);
}

// density part of the cell: table row of rho * Ye and the position in it
__device__ __forceinline__ void helm_cell_init_rho(const HelmTable &h, HelmCell &c, double rho, double ye) {
  c.Ye = ye;
  c.rhos = rho * c.Ye;
  c.ih = helm_node_index(h.rho, h.nrho, h.log10_rho1, h.drho, c.rhos);
  double r_lo = __ldg(h.rho + c.ih - 1);
  c.drho = __ldg(h.rho + c.ih) - r_lo;
  c.x = (c.rhos - r_lo) * __ldg(h.inv_drho + c.ih - 1);
}

__device__ __forceinline__ void helm_cell_init(const HelmTable &h, HelmCell &c, double rho, double abar,
                                               double zbar, double T) {
  helm_cell_init_rho(h, c, rho, zbar / abar);
  helm_cell_contract(h, c, helm_node_index(h.T, h.nT, h.log10_T1, h.dT, T));
}

// specific energy at the table's lowest temperature T_lo (the cold energy the learned guess's
// features subtract) from the density part of the cell: at a temperature node the quintic T
// basis reduces to the node's value and first derivative, so only f and f_T of the row's first
// T node are contracted (given2's E at T_lo to rounding)
__device__ __forceinline__ double helm_cell_cold_energy(const HelmTable &h, const HelmCell &c, double irho,
                                                        double inv_abar) {
  double r0[3], r1[3];
  helm_cell_rbasis(c, r0, r1);
  const double *lo = h.tab + 9 * (long long)(c.ih - 1), *hi = lo + 9;
  const int var[2][3] = {{0, 3, 4}, {1, 5, 6}};
  double f = 0.0, fT = 0.0;
#pragma unroll
  for (int orr = 0; orr < 3; ++orr) {
    f = fma(__ldg(lo + var[0][orr]), r0[orr], fma(__ldg(hi + var[0][orr]), r1[orr], f));
    fT = fma(__ldg(lo + var[1][orr]), r0[orr], fma(__ldg(hi + var[1][orr]), r1[orr], fT));
  }
  const double T = __ldg(h.T), T3 = T * T * T;
  return c.Ye * (f - T * fT) + 1.5 * CONST_RGAS * T * inv_abar + CONST_RAD * T3 * T * irho;
}

// f, f_T, f_TT at T (T inside the current cell)
__device__ __forceinline__ void helm_cell_eval(const HelmCell &c, double T, double &f, double &fT, double &fTT) {
  const double idT = c.idT;
  double d1, d2h;
  poly5_eval(c.c, (T - c.T0) * idT, f, d1, d2h);
  fT = d1 * idT;
  fTT = 2.0 * d2h * (idT * idT);
}

// Newton on E(rho, T) = E0 from T (helm_rhoe_given's loop and exit rules); an iterate outside
// the table is reset to Told and ends the loop, as in the reference.  Returns iterations, sets
// converged / clamped.  On return `c` holds the cell of the final T.  A solve split into two
// calls (the second with the first call's starting T as Told) runs the same iterates as one.
__device__ __forceinline__ int helm_rhoe_fast_from(const HelmTable &h, HelmCell &c, double irho, double E0,
                                                   double inv_abar, double &T, double Told, int max_iter,
                                                   int &clamped, bool &converged) {
  const double inv_E0 = 1.0 / E0;
  converged = false;
  int used = 0;
  for (int iter = 1; iter <= max_iter; ++iter) {
    used = iter;
    if (T < c.T0 || T >= c.T0 + c.dT) helm_cell_contract(h, c, helm_node_index(h.T, h.nT, h.log10_T1, h.dT, T));
    double f, fT, fTT;
    helm_cell_eval(c, T, f, fT, fTT);
    // every operation spelled out (no contraction left to the compiler), so that the solve is
    // the same bit for bit wherever it is inlined and however its iterations are split
    const double T3 = __dmul_rn(__dmul_rn(T, T), T);
    const double ion = __dmul_rn(__dmul_rn(1.5 * CONST_RGAS, T), inv_abar);
    const double rad = __dmul_rn(__dmul_rn(CONST_RAD, __dmul_rn(T3, T)), irho);
    const double E = __fma_rn(c.Ye, __fma_rn(-T, fT, f), __dadd_rn(ion, rad));
    const double dE = __fma_rn(-__dmul_rn(c.Ye, T), fTT,
                               __dadd_rn(__dmul_rn(1.5 * CONST_RGAS, inv_abar), __dmul_rn(__dmul_rn(4.0 * CONST_RAD, T3), irho)));
    const double res = __dsub_rn(E, E0);
    T = __dsub_rn(T, __ddiv_rn(res, dE));
    double error = fabs(__dmul_rn(res, inv_E0));
    if ((T < h.Tl) || (T > h.Th)) {
      T = Told;
      error = EM15;
      ++clamped;
    }
    if (error < HELM_TOL) { converged = true; break; }
  }
  if (T < c.T0 || T >= c.T0 + c.dT) helm_cell_contract(h, c, helm_node_index(h.T, h.nT, h.log10_T1, h.dT, T));
  return used;
}

// the same from the warm start T (Told = T)
__device__ __forceinline__ int helm_rhoe_fast(const HelmTable &h, HelmCell &c, double irho, double E0,
                                              double inv_abar, double &T, int max_iter, int &clamped,
                                              bool &converged) {
  return helm_rhoe_fast_from(h, c, irho, E0, inv_abar, T, T, max_iter, clamped, converged);
}

// pressure and the square of the relativistic sound speed at (rho, T) from the prepared cell
// (given_full's output; irho = 1 / rho)
__device__ __forceinline__ void helm_cell_p_sound2(const HelmTable &h, const HelmCell &c, double rho, double irho,
                                                   double T, double inv_abar, double &P, double &sound2,
                                                   double *E_out = nullptr) {
  const double idT = c.idT;
  const double y = (T - c.T0) * idT, omy = 1.0 - y;
  double f, fT, fTT, fd, fdT;
  helm_cell_eval(c, T, f, fT, fTT);
  // d/drho contraction of the final cell, as a quintic in y
  {
    const double idrho = __ldg(h.inv_drho + c.ih - 1);
    double dr0[3], dr1[3], B[3][2], q[6], d2h;
    fhb1(c.x, idrho, c.drho, dr0);
    fhb1m(1.0 - c.x, idrho, c.drho, dr1);
    helm_cell_contract_with(h, c, c.jh, dr0, dr1, B);
    helm_hermite_poly(B, c.dT, q);
    poly5_eval(q, y, fd, fdT, d2h);
    fdT *= idT;
  }
  // bicubic dP/d(rho Ye) (source.F90:24082-24118)
  double x = c.x, omx = 1.0 - x;
  double p0r = (2.0 * x - 3.0) * x * x + 1.0, p1r = ((x - 2.0) * x + 1.0) * x * c.drho;
  double p0mr = (2.0 * omx - 3.0) * omx * omx + 1.0, p1mr = -((omx - 2.0) * omx + 1.0) * omx * c.drho;
  double p0t = (2.0 * y - 3.0) * y * y + 1.0, p1t = ((y - 2.0) * y + 1.0) * y * c.dT;
  double p0mt = (2.0 * omy - 3.0) * omy * omy + 1.0, p1mt = -((omy - 2.0) * omy + 1.0) * omy * c.dT;
  const double *q00 = h.dpdr + 4 * ((long long)(c.ih - 1) + (long long)h.nrho * (c.jh - 1));
  const double *q10 = q00 + 4, *q01 = q00 + 4 * (long long)h.nrho, *q11 = q01 + 4;
  double rb[2][2] = {{p0r, p0mr}, {p1r, p1mr}}, tb[2][2] = {{p0t, p0mt}, {p1t, p1mt}};
  const int ordr[4] = {0, 0, 1, 1}, ordt[4] = {0, 1, 0, 1};  // c, c_T, c_rho, c_rhoT
  double dpd = 0.0;
#pragma unroll
  for (int v = 0; v < 4; ++v) {
    dpd = fma(__ldg(q00 + v) * rb[ordr[v]][0], tb[ordt[v]][0], dpd);
    dpd = fma(__ldg(q10 + v) * rb[ordr[v]][1], tb[ordt[v]][0], dpd);
    dpd = fma(__ldg(q01 + v) * rb[ordr[v]][0], tb[ordt[v]][1], dpd);
    dpd = fma(__ldg(q11 + v) * rb[ordr[v]][1], tb[ordt[v]][1], dpd);
  }
  double dP_drho = c.Ye * dpd;
  double r2 = c.rhos * c.rhos;
  double T3 = T * T * T, T4 = T3 * T;
  P = r2 * fd + CONST_RGAS * rho * T * inv_abar + CONST_RAD * T4 * (1.0 / 3.0);
  double dP_dT = r2 * fdT + CONST_RGAS * rho * inv_abar + (4.0 / 3.0) * CONST_RAD * T3;
  dP_drho = dP_drho + CONST_RGAS * T * inv_abar;
  double E = c.Ye * (f - T * fT) + 1.5 * CONST_RGAS * T * inv_abar + CONST_RAD * T4 * irho;
  double cv = -c.Ye * T * fTT + 1.5 * CONST_RGAS * inv_abar + 4.0 * CONST_RAD * T3 * irho;
  // the reference's gam1 / z (chiT = T dP/dT / P, chirho = rho dP/drho / P, x = (P / rho) chiT /
  // (T cv), gam1 = chiT x + chirho, z = 1 + (E + c^2) rho / P) with the common factors 1 / P
  // and 1 / (rho cv) cancelled: one division instead of five
  const double rcv = rho * cv;
  const double num = T * dP_dT * dP_dT + rcv * (rho * dP_drho);
  const double den = P + (E + CONST_C2) * rho;
  sound2 = CONST_C2 * num / (rcv * den);
  if (E_out) *E_out = E;
}

// Newton on P(rho, T) = P0 from T (helm_rhoP_given's loop and exit rules, source.F90:24943-24980:
// helm_tol on |P - P0| / P0, at most 100 iterations, an iterate outside the table resets to the
// start and ends the loop).  The density is fixed, so the d/drho coefficients of the current T
// cell are contracted once (B, 36 table values); an iteration needs the T basis and 12
// products for f_rho and f_rhoT: P = (rho Ye)^2 f_rho + ions + radiation and dP/dT alike.  On
// return `c` holds the value contraction (A) of the final T's cell, for helm_cell_p_sound2.
__device__ __forceinline__ int helm_rhoP_fast(const HelmTable &h, HelmCell &c, double rho, double P0,
                                              double inv_abar, double &T, int &clamped) {
  const double Told = T, inv_P0 = 1.0 / P0, r2 = c.rhos * c.rhos;
  double B[3][2], dr0[3], dr1[3];
  {
    const double idrho = __ldg(h.inv_drho + c.ih - 1);
    fhb1(c.x, idrho, c.drho, dr0);
    fhb1m(1.0 - c.x, idrho, c.drho, dr1);
  }
  int jh = -1;
  double T0 = 0.0, dT = 0.0, idT = 0.0, q[6];
  int used = 0;
  for (int iter = 1; iter <= 100; ++iter) {
    used = iter;
    if (jh < 0 || T < T0 || T >= T0 + dT) {
      jh = helm_node_index(h.T, h.nT, h.log10_T1, h.dT, T);
      T0 = __ldg(h.T + jh - 1);
      dT = __ldg(h.T + jh) - T0;
      idT = __ldg(h.inv_dT + jh - 1);
      helm_cell_contract_with(h, c, jh, dr0, dr1, B);
      helm_hermite_poly(B, dT, q);
    }
    double fd, fdT, d2h;
    poly5_eval(q, (T - T0) * idT, fd, fdT, d2h);
    fdT *= idT;
    const double T3 = T * T * T;
    const double P = r2 * fd + CONST_RGAS * rho * T * inv_abar + CONST_RAD * T3 * T * (1.0 / 3.0);
    const double dP = r2 * fdT + CONST_RGAS * rho * inv_abar + (4.0 / 3.0) * CONST_RAD * T3;
    const double res = P - P0;
    T = T - res / dP;
    double error = fabs(res * inv_P0);
    if ((T < h.Tl) || (T > h.Th)) {
      T = Told;
      error = EM15;
      ++clamped;
    }
    if (error < HELM_TOL) break;
  }
  helm_cell_contract(h, c, helm_node_index(h.T, h.nT, h.log10_T1, h.dT, T));
  return used;
}

// helm_rhoP_given with return_sound for one Riemann side of the split form: rho * e and the
// sound speed at (rho, p), from the temperature guess T
__device__ __forceinline__ void helm_side_eos_fast_inl(const HelmTable &h, double rho, double p, double abar,
                                                       double zbar, double T, double &rhoe, double &sound) {
  HelmCell c;
  const double inv_abar = 1.0 / abar, irho = 1.0 / rho;
  helm_cell_init_rho(h, c, rho, zbar * inv_abar);
  int clamped = 0;
  helm_rhoP_fast(h, c, rho, p, inv_abar, T, clamped);
  double P, sound2, E;
  helm_cell_p_sound2(h, c, rho, irho, T, inv_abar, P, sound2, &E);
  rhoe = E * rho;
  sound = sqrt(sound2);
}

}  // namespace phl
