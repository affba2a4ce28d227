// phl_device.cuh -- device building blocks of the explicit FV step: ghost-index mapping,
// LIM2ND reconstruction, Riemann solvers (LHLLC/HLLC/HLLD/LHLLD) and the Helmholtz EoS.
//
// Every function mirrors the operation order of the corresponding reference routine in
// source/source.F90 (line ranges in each comment) so that the FP64 path, compiled without FMA
// contraction, reproduces the reference's rounding.  The same templates run in FP32 for the
// split-precision path (R = float), where the flux arithmetic is done on well-balanced
// deviations and only the state/EoS stay in FP64.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace phl {

constexpr double CONST_RGAS = 8.31446261815324e7;
constexpr double CONST_RAD = 7.565767381646406e-15;
constexpr double CONST_C = 2.99792458e10;
constexpr double CONST_C2 = 8.987551787368177e20;
constexpr double HELM_TOL = 1.0e-11;  // helm_tol (source.F90:754)
constexpr double EM15 = 1.0e-15;

enum { R_LHLLC = 0, R_HLLC = 1, R_HLLD = 2, R_LHLLD = 3 };
enum { BC_PERIODIC = 0, BC_REFLECTIVE = 1 };

// ------------------------------------------------------------------ grid description
struct Geo {
  int sdims, nx[3];
  long long N;        // interior cells
  int bc[3][2];
  double inv_dx[3];
  double gm, mu, cfl, mach_cutoff, mach_ct;
  int bg_profile;     // 1: background fields stored as profiles along x2
  int all_mach;       // FLUX_IS_ALL_MACH: LHLLC / LHLLD take the upwind state outside the wave fan
  int use_acc;        // USE_CONSTANT_ACCELERATION with the vector acc
  double acc[3];
};

// USE_CONSTANT_ACCELERATION (source.F90:12806-12836): body force rho a on the momenta and its
// work on the energy, from the current RK state u (before the stage's combine), subtracted from
// the residual in the reference's order
template <int DIM, int IP>
__device__ __forceinline__ void constant_acceleration(const Geo &g, const double *u, double *res) {
  const double rho = u[0];
#pragma unroll
  for (int d = 0; d < DIM; ++d) res[1 + d] = res[1 + d] - rho * g.acc[d];
  double r = res[IP];
  if (DIM == 3) r = r - u[3] * g.acc[2];
  r = r - u[1] * g.acc[0];
  r = r - u[2] * g.acc[1];
  res[IP] = r;
}

// Map a (possibly ghost) 0-based index along dimension d to its interior image.
// Periodic: wrap; reflective: mirror (ghost -1 <- 0, -2 <- 1), flip set.  The composition over
// dimensions equals communicate_ndarray (with corners) followed by the reflective BC loops
// (source.F90:2293-2306, 7532-7958).
__device__ __forceinline__ int map_index(int i, int n, int bcl, int bcu, bool &flip) {
  if (i < 0) {
    if (bcl == BC_PERIODIC) return i + n;
    flip = true;  // velocity / B component along this dimension changes sign
    return -1 - i;
  }
  if (i >= n) {
    if (bcu == BC_PERIODIC) return i - n;
    flip = true;
    return 2 * n - 1 - i;
  }
  return i;
}

// (i, j, k) of a linear index t = i + n0 * (j + n1 * k) with 32-bit unsigned division (index
// spaces stay below 2^32, checked at phl_init; 64-bit division is a long software sequence)
__device__ __forceinline__ void unflatten3(long long t, int n0, int n1, int &i, int &j, int &k) {
  const unsigned u = (unsigned)t, q = u / (unsigned)n0, r = q / (unsigned)n1;
  i = (int)(u - q * (unsigned)n0);
  j = (int)(q - r * (unsigned)n1);
  k = (int)r;
}

__device__ __forceinline__ long long lin(const Geo &g, int i, int j, int k) {
  return (long long)i + (long long)g.nx[0] * ((long long)j + (long long)g.nx[1] * k);
}

// ------------------------------------------------------------------ reconstructions
enum { REC_LIM2ND = 0, REC_PPH = 1, REC_LIM5TH = 2 };
// Edge values of the centre cell qc (lo = left edge, hi = right edge) from its neighbours:
// PPH_REC (source.F90:8183-8259; third order, limited only when `limited`, i.e. for the
// advected scalars) and LIM5TH_REC (source.F90:8261-8323; fifth order, always limited), with
// the reference's limiter and operation order.  LIM2ND_REC is plm below.
template <typename R, int REC>
__device__ __forceinline__ void rec_edges(bool limited, R qmm, R qm, R qc, R qp, R qpp, R &lo, R &hi) {
  R am, ap;
  if (REC == REC_PPH) {
    R tmp = R(5.0 / 6.0) * qc;
    am = R(1.0 / 3.0) * qm + tmp - R(1.0 / 6.0) * qp;
    ap = -R(1.0 / 6.0) * qm + tmp + R(1.0 / 3.0) * qp;
    if (!limited) {
      lo = am;
      hi = ap;
      return;
    }
  } else {
    R tmp = R(329) * qc;
    am = (-R(21) * qmm + R(189) * qm + tmp - R(91) * qp + R(14) * qpp) * R(1.0 / 420.0);
    ap = (R(14) * qmm - R(91) * qm + tmp + R(189) * qp - R(21) * qpp) * R(1.0 / 420.0);
  }
  R mn = fmin(qm, qc), mx = fmax(qm, qc);
  if (am < mn) am = mn;
  if (am > mx) am = mx;
  mn = fmin(qc, qp);
  mx = fmax(qc, qp);
  if (ap < mn) ap = mn;
  if (ap > mx) ap = mx;
  am = am - qc;
  ap = ap - qc;
  if (ap * am >= R(0)) {
    ap = R(0);
    am = R(0);
  } else {
    if (fabs(ap) >= R(2) * fabs(am)) ap = -R(2) * am;
    if (fabs(am) >= R(2) * fabs(ap)) am = -R(2) * ap;
  }
  lo = am + qc;
  hi = ap + qc;
}

// ------------------------------------------------------------------ LIM2ND reconstruction
// source.F90:8141-8181: slope = df*db/(df+db) if df*db > 0 else 0; faces at qc -/+ slope/2.
template <typename R>
__device__ __forceinline__ void plm(R qm, R qc, R qp, R &lo, R &hi) {
  R slopef = qp - qc, slopeb = qc - qm;
  R prod = slopef * slopeb;
  R slope = R(0);
  if (prod > R(0)) slope = prod / (slopef + slopeb);
  R tmp = R(0.5) * slope;
  lo = qc - tmp;
  hi = qc + tmp;
}

template <typename R>
__device__ __forceinline__ R sgn1(R x) { return copysign(R(1), x); }

// ------------------------------------------------------------------ hydro Riemann
// qL/qR: [rho, v1, v2, (v3), p, scalars...] in the normal frame.  Side thermodynamics by EOSM:
// EOS_IDEAL gamma-law; EOS_FAST gL/gR = (gammae, gammac) (USE_FASTEOS); EOS_GIVEN gL/gR =
// (rho*e, sound speed) already evaluated by helm_rhoP_given (Helmholtz without USE_FASTEOS,
// source.F90:15777-15781).  LHLLC source.F90:15681-16122 (Minoshima & Miyoshi low-dissipation
// pressure), HLLC source.F90:16124-16252.
enum { EOS_IDEAL = 0, EOS_FAST = 1, EOS_GIVEN = 2 };
template <typename R, int DIM, int NV, int EOSM, int RIEM>
__device__ __forceinline__ void riemann_hydro(const R *qL, const R *qR, const R *gL, const R *gR,
                                              R gm, R mach_cutoff, R *flux, bool flat = false,
                                              bool all_mach = false) {
  constexpr int IP = 1 + DIM, IAS = 2 + DIM;
  const R gmm1 = gm - R(1), igmm1 = R(1) / gmm1;
  R rhoL = qL[0], inv_rhoL = R(1) / rhoL, vx1L = qL[1], vx2L = qL[2], vx3L = DIM == 3 ? qL[3] : R(0);
  R v2L = vx1L * vx1L + vx2L * vx2L + vx3L * vx3L;
  R pL = qL[IP], eint, cL, cR;
  if (EOSM == EOS_FAST) { eint = pL / (gL[0] - R(1)); cL = sqrt(gL[1] * pL * inv_rhoL); }
  else if (EOSM == EOS_GIVEN) { eint = gL[0]; cL = gL[1]; }
  else { eint = igmm1 * pL; cL = sqrt(gm * pL * inv_rhoL); }
  R rhoeL = eint + R(0.5) * rhoL * v2L;
  R rhoR = qR[0], inv_rhoR = R(1) / rhoR, vx1R = qR[1], vx2R = qR[2], vx3R = DIM == 3 ? qR[3] : R(0);
  R v2R = vx1R * vx1R + vx2R * vx2R + vx3R * vx3R;
  R pR = qR[IP];
  if (EOSM == EOS_FAST) { eint = pR / (gR[0] - R(1)); cR = sqrt(gR[1] * pR * inv_rhoR); }
  else if (EOSM == EOS_GIVEN) { eint = gR[0]; cR = gR[1]; }
  else { eint = igmm1 * pR; cR = sqrt(gm * pR * inv_rhoR); }
  R rhoeR = eint + R(0.5) * rhoR * v2R;
  R max_c = fmax(cL, cR);
  R sL = fmin(vx1L, vx1R) - max_c;
  R sR = fmax(vx1L, vx1R) + max_c;
  R dsuL = sL - vx1L, dsuR = sR - vx1R;
  R ustar = (pR - pL + rhoL * vx1L * dsuL - rhoR * vx1R * dsuR) / (rhoL * dsuL - rhoR * dsuR);
  R rhostarL = rhoL * (dsuL / (sL - ustar));
  R rhoestarL = rhostarL * (rhoeL * inv_rhoL + (ustar - vx1L) * (ustar + pL * inv_rhoL / dsuL));
  R rhostarR = rhoR * (dsuR / (sR - ustar));
  R rhoestarR = rhostarR * (rhoeR * inv_rhoR + (ustar - vx1R) * (ustar + pR * inv_rhoR / dsuR));
  if (flat) {
    // two-wave HLL flux on a face next to a detected shock (USE_SHOCK_FLATTENING,
    // source.F90:15929-16010)
    sL = fmin(R(0), sL);
    sR = fmax(R(0), sR);
    R UL[NV], UR[NV], fL[NV], fR[NV];
    UL[0] = rhoL; UL[1] = rhoL * vx1L; UL[2] = rhoL * vx2L; if (DIM == 3) UL[3] = rhoL * vx3L; UL[IP] = rhoeL;
    UR[0] = rhoR; UR[1] = rhoR * vx1R; UR[2] = rhoR * vx2R; if (DIM == 3) UR[3] = rhoR * vx3R; UR[IP] = rhoeR;
    fL[0] = rhoL * vx1L; fL[1] = rhoL * vx1L * vx1L + pL; fL[2] = rhoL * vx1L * vx2L;
    if (DIM == 3) fL[3] = rhoL * vx1L * vx3L;
    fL[IP] = (rhoeL + pL) * vx1L;
    fR[0] = rhoR * vx1R; fR[1] = rhoR * vx1R * vx1R + pR; fR[2] = rhoR * vx1R * vx2R;
    if (DIM == 3) fR[3] = rhoR * vx1R * vx3R;
    fR[IP] = (rhoeR + pR) * vx1R;
#pragma unroll
    for (int iv = IAS; iv < NV; ++iv) {
      UL[iv] = rhoL * qL[iv];
      UR[iv] = rhoR * qR[iv];
      fL[iv] = UL[iv] * vx1L;
      fR[iv] = UR[iv] * vx1R;
    }
    const R dummy = R(1) / (sR - sL), phi = sL * sR;
#pragma unroll
    for (int iv = 0; iv < NV; ++iv) flux[iv] = dummy * (sR * fL[iv] - sL * fR[iv] + phi * (UR[iv] - UL[iv]));
    return;
  }
  if (RIEM == R_LHLLC) {
    R machL = sqrt(v2L) / cL, machR = sqrt(v2R) / cR;
    R chi = fmin(R(1), fmax(machL, machR));
    chi = fmax(mach_cutoff, chi);
    R phi = chi * (R(2) - chi);
    R rhobar = R(0.5) * (rhoL + rhoR), cbar = R(0.5) * (cL + cR);
    R pstar = R(0.5) * (pL + pR) - R(0.5) * phi * rhobar * cbar * (vx1R - vx1L);
    if (all_mach && (sL > R(0) || sR < R(0))) {
      // FLUX_IS_ALL_MACH: the upwind state's flux outside the wave fan (source.F90:16032-16077)
      const bool left = sL > R(0);
      const R *q = left ? qL : qR;
      R rho = left ? rhoL : rhoR, vx1 = left ? vx1L : vx1R, vx2 = left ? vx2L : vx2R, vx3 = left ? vx3L : vx3R;
      R p = left ? pL : pR, rhoe = left ? rhoeL : rhoeR;
      flux[0] = rho * vx1;
      flux[1] = rho * vx1 * vx1 + p;
      flux[2] = rho * vx1 * vx2;
      if (DIM == 3) flux[3] = rho * vx1 * vx3;
      flux[IP] = (rhoe + p) * vx1;
#pragma unroll
      for (int iv = IAS; iv < NV; ++iv) flux[iv] = rho * q[iv] * vx1;
      return;
    }
    R sgn = sgn1(ustar);
    R hp = R(0.5) * (R(1) + sgn), hm = R(0.5) * (R(1) - sgn);
    R rhostar = hp * rhostarL + hm * rhostarR;
    flux[0] = rhostar * ustar;
    flux[1] = rhostar * ustar * ustar + pstar;
    flux[2] = rhostar * ustar * (hp * vx2L + hm * vx2R);
    if (DIM == 3) flux[3] = rhostar * ustar * (hp * vx3L + hm * vx3R);
    flux[IP] = (hp * rhoestarL + hm * rhoestarR + pstar) * ustar;
#pragma unroll
    for (int iv = IAS; iv < NV; ++iv) flux[iv] = rhostar * ustar * (hp * qL[iv] + hm * qR[iv]);
  } else {
    const bool left = ustar > R(0);
    const R *q = left ? qL : qR;
    R rho = left ? rhoL : rhoR, vx1 = left ? vx1L : vx1R, vx2 = left ? vx2L : vx2R, vx3 = left ? vx3L : vx3R;
    R p = left ? pL : pR, rhoe = left ? rhoeL : rhoeR, rhostar = left ? rhostarL : rhostarR;
    R rhoestar = left ? rhoestarL : rhoestarR, s = left ? sL : sR;
    const bool sup = left ? (sL >= R(0)) : (sR < R(0));
    R U[NV], f[NV];
    U[0] = rho; U[1] = rho * vx1; U[2] = rho * vx2; if (DIM == 3) U[3] = rho * vx3; U[IP] = rhoe;
    f[0] = rho * vx1; f[1] = rho * vx1 * vx1 + p; f[2] = rho * vx1 * vx2;
    if (DIM == 3) f[3] = rho * vx1 * vx3;
    f[IP] = (rhoe + p) * vx1;
#pragma unroll
    for (int iv = IAS; iv < NV; ++iv) { U[iv] = rho * q[iv]; f[iv] = rho * vx1 * q[iv]; }
    if (sup) {
#pragma unroll
      for (int iv = 0; iv < NV; ++iv) flux[iv] = f[iv];
    } else {
      R Us[NV];
      Us[0] = rhostar; Us[1] = rhostar * ustar; Us[2] = rhostar * vx2; if (DIM == 3) Us[3] = rhostar * vx3;
      Us[IP] = rhoestar;
#pragma unroll
      for (int iv = IAS; iv < NV; ++iv) Us[iv] = rhostar * q[iv];
#pragma unroll
      for (int iv = 0; iv < NV; ++iv) flux[iv] = f[iv] + s * (Us[iv] - U[iv]);
    }
  }
}

// ------------------------------------------------------------------ MHD Riemann
// HLLD (Miyoshi & Kusano) source.F90:13969-15016, LHLLD source.F90:14364-14384, 14663-14732.
// b*: [Bn, Bt1, Bt2]; fluxb receives [0, Ft1, Ft2].
template <typename R, int DIM, int NV, int EOSM, int RIEM>
__device__ __forceinline__ void riemann_mhd(const R *qL, const R *qR, const R *bL, const R *bR,
                                            const R *gL, const R *gR, R gm, R mach_cutoff,
                                            R *flux, R *fluxb, bool flat = false, bool all_mach = false) {
  constexpr int IP = 1 + DIM, IAS = 2 + DIM;
  const R gmm1 = gm - R(1), igmm1 = R(1) / gmm1;
  R rhoL = qL[0], inv_rhoL = R(1) / rhoL, vx1L = qL[1], vx2L = qL[2], vx3L = DIM == 3 ? qL[3] : R(0);
  R v2L = vx1L * vx1L + vx2L * vx2L + vx3L * vx3L;
  R pL = qL[IP], eint, c2L, c2R;
  if (EOSM == EOS_FAST) { eint = pL / (gL[0] - R(1)); c2L = gL[1] * pL * inv_rhoL; }
  else if (EOSM == EOS_GIVEN) { eint = gL[0]; c2L = gL[1] * gL[1]; }
  else { eint = pL * igmm1; c2L = gm * pL * inv_rhoL; }
  R rhoeL = eint + R(0.5) * rhoL * v2L;
  R bx1L = bL[0], bx2L = bL[1], bx3L = DIM == 3 ? bL[2] : R(0);
  R rhoR = qR[0], inv_rhoR = R(1) / rhoR, vx1R = qR[1], vx2R = qR[2], vx3R = DIM == 3 ? qR[3] : R(0);
  R v2R = vx1R * vx1R + vx2R * vx2R + vx3R * vx3R;
  R pR = qR[IP];
  if (EOSM == EOS_FAST) { eint = pR / (gR[0] - R(1)); c2R = gR[1] * pR * inv_rhoR; }
  else if (EOSM == EOS_GIVEN) { eint = gR[0]; c2R = gR[1] * gR[1]; }
  else { eint = pR * igmm1; c2R = gm * pR * inv_rhoR; }
  R rhoeR = eint + R(0.5) * rhoR * v2R;
  R bx1R = bR[0], bx2R = bR[1], bx3R = DIM == 3 ? bR[2] : R(0);

  R bx1 = R(0.5) * (bx1L + bx1R), bx1_2 = bx1 * bx1;
  R pbL = R(0.5) * (bx1_2 + bx2L * bx2L + bx3L * bx3L);
  R pbR = R(0.5) * (bx1_2 + bx2R * bx2R + bx3R * bx3R);
  rhoeL = rhoeL + pbL;
  rhoeR = rhoeR + pbR;
  R ptL = pL + pbL, ptR = pR + pbR;
  R a2L = R(2) * pbL * inv_rhoL, a2R = R(2) * pbR * inv_rhoR;
  R an2L = bx1_2 * inv_rhoL, an2R = bx1_2 * inv_rhoR;
  R dummy = c2L + a2L;
  R cL = sqrt(R(0.5) * (c2L + a2L + sqrt(dummy * dummy - R(4) * c2L * an2L)));
  dummy = c2R + a2R;
  R cR = sqrt(R(0.5) * (c2R + a2R + sqrt(dummy * dummy - R(4) * c2R * an2R)));
  R max_c = fmax(cL, cR);
  R sL = fmin(vx1L, vx1R) - max_c;
  R sR = fmax(vx1L, vx1R) + max_c;
  R dsuL = sL - vx1L, dsuR = sR - vx1R;
  R inv_temp1 = R(1) / (dsuR * rhoR - dsuL * rhoL);
  R ustar = (dsuR * rhoR * vx1R - dsuL * rhoL * vx1L - ptR + ptL) * inv_temp1;
  R dsumL = sL - ustar, dsumR = sR - ustar;
  R phi = R(1);
  if (RIEM == R_LHLLD) {
    dummy = v2L + a2L;
    R cu2L = R(0.5) * (v2L + a2L + sqrt(dummy * dummy - R(4) * v2L * an2L));
    dummy = v2R + a2R;
    R cu2R = R(0.5) * (v2R + a2R + sqrt(dummy * dummy - R(4) * v2R * an2R));
    R machL = sqrt(cu2L) / cL, machR = sqrt(cu2R) / cR;
    R mm = fmax(machL, machR);
    if (mm < R(0.6)) {
      R chi = fmin(R(1), fmax(machL, machR));
      chi = fmax(mach_cutoff, chi);
      phi = chi * (R(2) - chi);
    } else {
      phi = R(1);
    }
  }
  if (flat) {
    // HLL flux on a flattened face (USE_SHOCK_FLATTENING, source.F90:14386-14495)
    sL = fmin(R(0), sL);
    sR = fmax(R(0), sR);
    R UL[NV], UR[NV], fL[NV], fR[NV];
    UL[0] = rhoL; UL[1] = rhoL * vx1L; UL[2] = rhoL * vx2L; if (DIM == 3) UL[3] = rhoL * vx3L; UL[IP] = rhoeL;
    UR[0] = rhoR; UR[1] = rhoR * vx1R; UR[2] = rhoR * vx2R; if (DIM == 3) UR[3] = rhoR * vx3R; UR[IP] = rhoeR;
    fL[0] = rhoL * vx1L; fL[1] = rhoL * vx1L * vx1L + ptL - bx1_2; fL[2] = rhoL * vx1L * vx2L - bx1 * bx2L;
    if (DIM == 3) fL[3] = rhoL * vx1L * vx3L - bx1 * bx3L;
    fL[IP] = (rhoeL + ptL) * vx1L - bx1 * (bx1 * vx1L + bx2L * vx2L + bx3L * vx3L);
    fR[0] = rhoR * vx1R; fR[1] = rhoR * vx1R * vx1R + ptR - bx1_2; fR[2] = rhoR * vx1R * vx2R - bx1 * bx2R;
    if (DIM == 3) fR[3] = rhoR * vx1R * vx3R - bx1 * bx3R;
    fR[IP] = (rhoeR + ptR) * vx1R - bx1 * (bx1 * vx1R + bx2R * vx2R + bx3R * vx3R);
#pragma unroll
    for (int iv = IAS; iv < NV; ++iv) {
      UL[iv] = rhoL * qL[iv];
      UR[iv] = rhoR * qR[iv];
      fL[iv] = UL[iv] * vx1L;
      fR[iv] = UR[iv] * vx1R;
    }
    const R UbL[3] = {bx1, bx2L, bx3L}, UbR[3] = {bx1, bx2R, bx3R};
    const R fbL[3] = {R(0), vx1L * bx2L - vx2L * bx1, vx1L * bx3L - vx3L * bx1};
    const R fbR[3] = {R(0), vx1R * bx2R - vx2R * bx1, vx1R * bx3R - vx3R * bx1};
    const R dh = R(1) / (sR - sL), ph = sL * sR;
#pragma unroll
    for (int iv = 0; iv < NV; ++iv) flux[iv] = dh * (sR * fL[iv] - sL * fR[iv] + ph * (UR[iv] - UL[iv]));
#pragma unroll
    for (int iv = 0; iv < DIM; ++iv) fluxb[iv] = dh * (sR * fbL[iv] - sL * fbR[iv] + ph * (UbR[iv] - UbL[iv]));
    return;
  }
  R pstar = (dsuR * rhoR * ptL - dsuL * rhoL * ptR - phi * rhoL * rhoR * dsuR * dsuL * (vx1L - vx1R)) * inv_temp1;
  R rhostarL = rhoL * dsuL / dsumL, rhostarR = rhoR * dsuR / dsumR;
  R a1_inv = R(1) / (rhoL * dsuL * dsumL - bx1_2);
  R vx2starL = vx2L - bx1 * bx2L * (ustar - vx1L) * a1_inv;
  R bx2starL = bx2L * (rhoL * dsuL * dsuL - bx1_2) * a1_inv;
  R vx3starL = vx3L - bx1 * bx3L * (ustar - vx1L) * a1_inv;
  R bx3starL = bx3L * (rhoL * dsuL * dsuL - bx1_2) * a1_inv;
  R a2_inv = R(1) / (rhoR * dsuR * dsumR - bx1_2);
  R vx2starR = vx2R - bx1 * bx2R * (ustar - vx1R) * a2_inv;
  R bx2starR = bx2R * (rhoR * dsuR * dsuR - bx1_2) * a2_inv;
  R vx3starR = vx3R - bx1 * bx3R * (ustar - vx1R) * a2_inv;
  R bx3starR = bx3R * (rhoR * dsuR * dsuR - bx1_2) * a2_inv;
  R vdotbL = vx1L * bx1 + vx2L * bx2L + vx3L * bx3L;
  R vdotbR = vx1R * bx1 + vx2R * bx2R + vx3R * bx3R;
  R vdotbstarL = ustar * bx1 + vx2starL * bx2starL + vx3starL * bx3starL;
  R vdotbstarR = ustar * bx1 + vx2starR * bx2starR + vx3starR * bx3starR;
  R rhoestarL = (dsuL * rhoeL - ptL * vx1L + pstar * ustar + bx1 * (vdotbL - vdotbstarL)) / dsumL;
  R rhoestarR = (dsuR * rhoeR - ptR * vx1R + pstar * ustar + bx1 * (vdotbR - vdotbstarR)) / dsumR;
  R sqrt_rhostarL = sqrt(rhostarL), sqrt_rhostarR = sqrt(rhostarR);
  R abs_bx1 = fabs(bx1);
  R sstarL = ustar - abs_bx1 / sqrt_rhostarL;
  R sstarR = ustar + abs_bx1 / sqrt_rhostarR;
  R inv_sqr_bar = R(1) / (sqrt_rhostarL + sqrt_rhostarR);
  R sgn = sgn1(bx1);
  R vx22star = (sqrt_rhostarL * vx2starL + sqrt_rhostarR * vx2starR + (bx2starR - bx2starL) * sgn) * inv_sqr_bar;
  R bx22star = (sqrt_rhostarL * bx2starR + sqrt_rhostarR * bx2starL +
                sqrt_rhostarL * sqrt_rhostarR * (vx2starR - vx2starL) * sgn) * inv_sqr_bar;
  R vx32star = (sqrt_rhostarL * vx3starL + sqrt_rhostarR * vx3starR + (bx3starR - bx3starL) * sgn) * inv_sqr_bar;
  R bx32star = (sqrt_rhostarL * bx3starR + sqrt_rhostarR * bx3starL +
                sqrt_rhostarL * sqrt_rhostarR * (vx3starR - vx3starL) * sgn) * inv_sqr_bar;
  R vdotb2star = ustar * bx1 + vx22star * bx22star + vx32star * bx32star;
  R rhoe2starL = rhoestarL - sqrt_rhostarL * (vdotbstarL - vdotb2star) * sgn;
  R rhoe2starR = rhoestarR + sqrt_rhostarR * (vdotbstarR - vdotb2star) * sgn;

  fluxb[0] = R(0);
  if (RIEM == R_LHLLD) {
    R rho, vx1, vx2, vx3, rhoe, bx2, bx3, pres = pstar;
    if (all_mach && sL > R(0)) {
      // FLUX_IS_ALL_MACH: the outer states as well (source.F90:14576-14632)
      rho = rhoL; vx1 = vx1L; vx2 = vx2L; vx3 = vx3L; rhoe = rhoeL; bx2 = bx2L; bx3 = bx3L; pres = ptL;
    } else if (sstarL > R(0)) {
      rho = rhostarL; vx1 = ustar; vx2 = vx2starL; vx3 = vx3starL; rhoe = rhoestarL; bx2 = bx2starL; bx3 = bx3starL;
    } else if (ustar > R(0)) {
      rho = rhostarL; vx1 = ustar; vx2 = vx22star; vx3 = vx32star; rhoe = rhoe2starL; bx2 = bx22star; bx3 = bx32star;
    } else if (sstarR > R(0)) {
      rho = rhostarR; vx1 = ustar; vx2 = vx22star; vx3 = vx32star; rhoe = rhoe2starR; bx2 = bx22star; bx3 = bx32star;
    } else if (!all_mach || sR > R(0)) {
      rho = rhostarR; vx1 = ustar; vx2 = vx2starR; vx3 = vx3starR; rhoe = rhoestarR; bx2 = bx2starR; bx3 = bx3starR;
    } else {
      rho = rhoR; vx1 = vx1R; vx2 = vx2R; vx3 = vx3R; rhoe = rhoeR; bx2 = bx2R; bx3 = bx3R; pres = ptR;
    }
    flux[0] = rho * vx1;
    flux[1] = rho * vx1 * vx1 + pres - bx1_2;
    flux[2] = rho * vx1 * vx2 - bx1 * bx2;
    if (DIM == 3) flux[3] = rho * vx1 * vx3 - bx1 * bx3;
    flux[IP] = (rhoe + pres) * vx1 - bx1 * (bx1 * vx1 + vx2 * bx2 + vx3 * bx3);
    R sg = sgn1(vx1), hp = R(0.5) * (R(1) + sg), hm = R(0.5) * (R(1) - sg);
#pragma unroll
    for (int iv = IAS; iv < NV; ++iv) flux[iv] = rho * vx1 * (hp * qL[iv] + hm * qR[iv]);
    fluxb[1] = vx1 * bx2 - bx1 * vx2;
    if (DIM == 3) fluxb[2] = vx1 * bx3 - bx1 * vx3;
    return;
  }
  const bool left = ustar > R(0);
  const R *q = left ? qL : qR;
  R rho = left ? rhoL : rhoR, vx1 = left ? vx1L : vx1R, vx2 = left ? vx2L : vx2R, vx3 = left ? vx3L : vx3R;
  R rhoe = left ? rhoeL : rhoeR, pt = left ? ptL : ptR, bx2 = left ? bx2L : bx2R, bx3 = left ? bx3L : bx3R;
  R vdotb = left ? vdotbL : vdotbR, rhostar = left ? rhostarL : rhostarR;
  R vx2s = left ? vx2starL : vx2starR, vx3s = left ? vx3starL : vx3starR;
  R bx2s = left ? bx2starL : bx2starR, bx3s = left ? bx3starL : bx3starR;
  R rhoes = left ? rhoestarL : rhoestarR, rhoe2s = left ? rhoe2starL : rhoe2starR;
  R s = left ? sL : sR, sst = left ? sstarL : sstarR;
  const bool outer = left ? (sL > R(0)) : (sR < R(0));
  const bool single = left ? (sstarL > R(0)) : (sstarR < R(0));
  constexpr int NB = DIM == 3 ? 3 : 2;
  R U[NV], f[NV], Ub[3], fb[3];
  U[0] = rho; U[1] = rho * vx1; U[2] = rho * vx2; if (DIM == 3) U[3] = rho * vx3; U[IP] = rhoe;
  f[0] = rho * vx1; f[1] = rho * vx1 * vx1 + pt - bx1_2; f[2] = rho * vx1 * vx2 - bx1 * bx2;
  if (DIM == 3) f[3] = rho * vx1 * vx3 - bx1 * bx3;
  f[IP] = (rhoe + pt) * vx1 - bx1 * vdotb;
#pragma unroll
  for (int iv = IAS; iv < NV; ++iv) { U[iv] = rho * q[iv]; f[iv] = rho * vx1 * q[iv]; }
  Ub[0] = bx1; Ub[1] = bx2; Ub[2] = bx3;
  fb[0] = R(0); fb[1] = vx1 * bx2 - bx1 * vx2; fb[2] = vx1 * bx3 - bx1 * vx3;
  if (outer) {
#pragma unroll
    for (int iv = 0; iv < NV; ++iv) flux[iv] = f[iv];
#pragma unroll
    for (int iv = 0; iv < NB; ++iv) fluxb[iv] = fb[iv];
    return;
  }
  R Us[NV], Ubs[3];
  Us[0] = rhostar; Us[1] = rhostar * ustar; Us[2] = rhostar * vx2s; if (DIM == 3) Us[3] = rhostar * vx3s;
  Us[IP] = rhoes;
#pragma unroll
  for (int iv = IAS; iv < NV; ++iv) Us[iv] = rhostar * q[iv];
  Ubs[0] = bx1; Ubs[1] = bx2s; Ubs[2] = bx3s;
  if (single) {
#pragma unroll
    for (int iv = 0; iv < NV; ++iv) flux[iv] = f[iv] + s * (Us[iv] - U[iv]);
#pragma unroll
    for (int iv = 0; iv < NB; ++iv) fluxb[iv] = fb[iv] + s * (Ubs[iv] - Ub[iv]);
    return;
  }
  R Uss[NV], Ubss[3];
  Uss[0] = rhostar; Uss[1] = rhostar * ustar; Uss[2] = rhostar * vx22star; if (DIM == 3) Uss[3] = rhostar * vx32star;
  Uss[IP] = rhoe2s;
#pragma unroll
  for (int iv = IAS; iv < NV; ++iv) Uss[iv] = rhostar * q[iv];
  Ubss[0] = bx1; Ubss[1] = bx22star; Ubss[2] = bx32star;
#pragma unroll
  for (int iv = 0; iv < NV; ++iv) {
    R d0 = Us[iv];
    flux[iv] = f[iv] + s * (d0 - U[iv]) + sst * (Uss[iv] - d0);
  }
#pragma unroll
  for (int iv = 0; iv < NB; ++iv) {
    R d0 = Ubs[iv];
    fluxb[iv] = fb[iv] + s * (d0 - Ub[iv]) + sst * (Ubss[iv] - d0);
  }
}

// ------------------------------------------------------------------ Helmholtz EoS
struct HelmTable {
  const double *tab;    // helm_table_var(1:9, 1:nrho, 1:nT)
  const double *dpdr;   // dpdrho_table_var(1:4, 1:nrho, 1:nT)
  const double *rho;    // helm_rho(1:nrho)
  const double *T;      // helm_T(1:nT)
  // reciprocal node spacings 1 / (helm_rho(i+1) - helm_rho(i)), 1 / (helm_T(j+1) - helm_T(j)),
  // index i-1 / j-1 (the same IEEE quotients a division at the point of use gives)
  const double *inv_drho, *inv_dT;
  int nrho, nT;
  double drho, dT, log10_rho1, log10_T1;  // log10(helm_rho(1)), log10(helm_T(1)) from the host
  double Tl, Th;
};

struct HelmPos {
  int ih, jh;  // 1-based like the reference
  double Ye, rhos, x, y, omx, omy, drho, dT, drho2, dT2, idrho, idT, idT2;
};

__device__ __forceinline__ void helm_locate(const HelmTable &h, double rho, double T, double abar,
                                            double zbar, HelmPos &p) {
  p.Ye = zbar / abar;
  p.rhos = rho * p.Ye;
  p.ih = (int)((log10(p.rhos) - h.log10_rho1) / h.drho) + 1;
  p.jh = (int)((log10(T) - h.log10_T1) / h.dT) + 1;
  // stay inside the table like the reference's arrays would (the reference does not check)
  p.ih = max(1, min(p.ih, h.nrho - 1));
  p.jh = max(1, min(p.jh, h.nT - 1));
  double tmp = __ldg(h.rho + p.ih - 1);
  p.drho = __ldg(h.rho + p.ih) - tmp;
  p.x = (p.rhos - tmp) / p.drho;
  p.omx = 1.0 - p.x;
  tmp = __ldg(h.T + p.jh - 1);
  p.dT = __ldg(h.T + p.jh) - tmp;
  p.y = (T - tmp) / p.dT;
  p.omy = 1.0 - p.y;
  p.drho2 = p.drho * p.drho;
  p.dT2 = p.dT * p.dT;
  p.idrho = 1.0 / p.drho;
  p.idT = 1.0 / p.dT;
  p.idT2 = p.idT * p.idT;
}

// quintic Hermite bases (source.F90:24708-24738) and their derivatives
__device__ __forceinline__ void hb0(double x, double d, double d2, double b[3]) {
  double x2 = x * x, x3 = x2 * x, x4 = x3 * x, x5 = x4 * x;
  b[0] = -6.0 * x5 + 15.0 * x4 - 10.0 * x3 + 1.0;
  b[1] = (-3.0 * x5 + 8.0 * x4 - 6.0 * x3 + x) * d;
  b[2] = (0.5 * (-x5 + 3.0 * x4 - 3.0 * x3 + x2)) * d2;
}
__device__ __forceinline__ void hb0m(double om, double d, double d2, double b[3]) {
  double o2 = om * om, o3 = o2 * om, o4 = o3 * om, o5 = o4 * om;
  b[0] = -6.0 * o5 + 15.0 * o4 - 10.0 * o3 + 1.0;
  b[1] = (3.0 * o5 - 8.0 * o4 + 6.0 * o3 - om) * d;
  b[2] = (0.5 * (-o5 + 3.0 * o4 - 3.0 * o3 + o2)) * d2;
}
__device__ __forceinline__ void hb1(double x, double id, double d, double b[3]) {
  double x2 = x * x, x3 = x2 * x, x4 = x3 * x;
  b[0] = (-30.0 * x4 + 60.0 * x3 - 30.0 * x2) * id;
  b[1] = (-15.0 * x4 + 32.0 * x3 - 18.0 * x2 + 1.0);
  b[2] = (0.5 * (-5.0 * x4 + 12.0 * x3 - 9.0 * x2 + 2.0 * x)) * d;
}
__device__ __forceinline__ void hb1m(double om, double id, double d, double b[3]) {
  double o2 = om * om, o3 = o2 * om, o4 = o3 * om;
  b[0] = -(-30.0 * o4 + 60.0 * o3 - 30.0 * o2) * id;
  b[1] = (-15.0 * o4 + 32.0 * o3 - 18.0 * o2 + 1.0);
  b[2] = -(0.5 * (-5.0 * o4 + 12.0 * o3 - 9.0 * o2 + 2.0 * om)) * d;
}
__device__ __forceinline__ void hb2(double y, double id2, double id, double b[3]) {
  double y2 = y * y, y3 = y2 * y;
  b[0] = (-120.0 * y3 + 180.0 * y2 - 60.0 * y) * id2;
  b[1] = (-60.0 * y3 + 96.0 * y2 - 36.0 * y) * id;
  b[2] = (0.5 * (-20.0 * y3 + 36.0 * y2 - 18.0 * y + 2.0));
}
__device__ __forceinline__ void hb2m(double om, double id2, double id, double b[3]) {
  double o2 = om * om, o3 = o2 * om;
  b[0] = (-120.0 * o3 + 180.0 * o2 - 60.0 * om) * id2;
  b[1] = -(-60.0 * o3 + 96.0 * o2 - 36.0 * om) * id;
  b[2] = (0.5 * (-20.0 * o3 + 36.0 * o2 - 18.0 * om + 2.0));
}

// Sum over the 36 coefficients in loc_eos1..36 order, left to right.  The rho-order and T-order
// of the 9 table variables (id_f .. id_d4fdrho2dT2, source.F90:520-528) are
// rho: 0,0,0,1,2,1,2,1,2 and T: 0,1,2,0,0,1,1,2,2.
__device__ __forceinline__ double helm_sum36(const double c[36], const double r0[3], const double r1[3],
                                             const double t0[3], const double t1[3]) {
  double s = 0.0;
#pragma unroll
  for (int v = 0; v < 9; ++v) {
    const int orr = v < 3 ? 0 : ((v & 1) ? 1 : 2);   // matches HELM_ORD_R
    const int ort = v == 0 ? 0 : (v == 1 ? 1 : (v == 2 ? 2 : (v <= 4 ? 0 : (v <= 6 ? 1 : 2))));
    double a = (c[4 * v + 0] * r0[orr]) * t0[ort];
    double b = (c[4 * v + 1] * r1[orr]) * t0[ort];
    double cc = (c[4 * v + 2] * r0[orr]) * t1[ort];
    double d = (c[4 * v + 3] * r1[orr]) * t1[ort];
    if (v == 0) s = a; else s = s + a;
    s = s + b;
    s = s + cc;
    s = s + d;
  }
  return s;
}

__device__ __forceinline__ void helm_load36(const HelmTable &h, int ih, int jh, double c[36]) {
  const double *p00 = h.tab + 9 * ((long long)(ih - 1) + (long long)h.nrho * (jh - 1));
  const double *p10 = p00 + 9;
  const double *p01 = p00 + 9 * (long long)h.nrho;
  const double *p11 = p01 + 9;
#pragma unroll
  for (int v = 0; v < 9; ++v) {
    c[4 * v + 0] = __ldg(p00 + v);
    c[4 * v + 1] = __ldg(p10 + v);
    c[4 * v + 2] = __ldg(p01 + v);
    c[4 * v + 3] = __ldg(p11 + v);
  }
}

// helm_rhoT_given2 (source.F90:24571-24941): E and dE/dT
__device__ __forceinline__ void helm_given2(const HelmTable &h, double rho, double T, double abar,
                                            double zbar, double &E, double &dEdT, bool want_deriv) {
  HelmPos p;
  helm_locate(h, rho, T, abar, zbar, p);
  double c[36];
  helm_load36(h, p.ih, p.jh, c);
  double r0[3], r1[3], t0[3], t1[3];
  hb0(p.x, p.drho, p.drho2, r0);
  hb0m(p.omx, p.drho, p.drho2, r1);
  hb0(p.y, p.dT, p.dT2, t0);
  hb0m(p.omy, p.dT, p.dT2, t1);
  double f = helm_sum36(c, r0, r1, t0, t1);
  double d0[3], d1[3];
  hb1(p.y, p.idT, p.dT, d0);
  hb1m(p.omy, p.idT, p.dT, d1);
  double df_dT = helm_sum36(c, r0, r1, d0, d1);
  double df_dT2 = 0.0;
  if (want_deriv) {
    double e0[3], e1[3];
    hb2(p.y, p.idT2, p.idT, e0);
    hb2m(p.omy, p.idT2, p.idT, e1);
    df_dT2 = helm_sum36(c, r0, r1, e0, e1);
  }
  double s = -p.Ye * df_dT;
  double ds_dT = -p.Ye * df_dT2;
  double e = p.Ye * f + T * s;
  double de = T * ds_dT;
  double T2 = T * T, T3 = T2 * T, T4 = T3 * T;
  double tmp = 1.0 / abar;
  e = e + 1.5 * CONST_RGAS * T * tmp + CONST_RAD * T4 / rho;
  de = de + 1.5 * CONST_RGAS * tmp + 4.0 * CONST_RAD * T3 / rho;
  E = e;
  dEdT = de;
}

// helm_rhoT_given1 (source.F90:24234-24569): P and dP/dT
__device__ __forceinline__ void helm_given1(const HelmTable &h, double rho, double T, double abar,
                                            double zbar, double &P, double &dPdT, bool want_deriv) {
  HelmPos p;
  helm_locate(h, rho, T, abar, zbar, p);
  double c[36];
  helm_load36(h, p.ih, p.jh, c);
  double r0[3], r1[3], t0[3], t1[3];
  hb1(p.x, p.idrho, p.drho, r0);
  hb1m(p.omx, p.idrho, p.drho, r1);
  hb0(p.y, p.dT, p.dT2, t0);
  hb0m(p.omy, p.dT, p.dT2, t1);
  double df_drho = helm_sum36(c, r0, r1, t0, t1);
  double df_drhodT = 0.0;
  if (want_deriv) {
    double d0[3], d1[3];
    hb1(p.y, p.idT, p.dT, d0);
    hb1m(p.omy, p.idT, p.dT, d1);
    df_drhodT = helm_sum36(c, r0, r1, d0, d1);
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
  P = pp;
  dPdT = dp;
}

// helm_rhoT_given_full (source.F90:23686-24232): P, E, relativistic sound speed, cv
__device__ __forceinline__ void helm_given_full(const HelmTable &h, double rho, double T, double abar,
                                                double zbar, double &P, double &E, double &sound,
                                                double &cv) {
  HelmPos p;
  helm_locate(h, rho, T, abar, zbar, p);
  double c[36];
  helm_load36(h, p.ih, p.jh, c);
  double r0[3], r1[3], t0[3], t1[3], dr0[3], dr1[3], dt0[3], dt1[3], et0[3], et1[3];
  hb0(p.x, p.drho, p.drho2, r0);
  hb0m(p.omx, p.drho, p.drho2, r1);
  hb0(p.y, p.dT, p.dT2, t0);
  hb0m(p.omy, p.dT, p.dT2, t1);
  double f = helm_sum36(c, r0, r1, t0, t1);
  hb1(p.x, p.idrho, p.drho, dr0);
  hb1m(p.omx, p.idrho, p.drho, dr1);
  double df_drho = helm_sum36(c, dr0, dr1, t0, t1);
  hb1(p.y, p.idT, p.dT, dt0);
  hb1m(p.omy, p.idT, p.dT, dt1);
  double df_dT = helm_sum36(c, r0, r1, dt0, dt1);
  double df_drhodT = helm_sum36(c, dr0, dr1, dt0, dt1);
  hb2(p.y, p.idT2, p.idT, et0);
  hb2m(p.omy, p.idT2, p.idT, et1);
  double df_dT2 = helm_sum36(c, r0, r1, et0, et1);
  // bicubic Hermite of dP/d(rho Ye) (source.F90:24082-24118)
  double x = p.x, x2 = x * x, x3 = x2 * x, omx = p.omx, omx2 = omx * omx, omx3 = omx2 * omx;
  double y = p.y, y2 = y * y, y3 = y2 * y, omy = p.omy, omy2 = omy * omy, omy3 = omy2 * omy;
  double p0r = 2.0 * x3 - 3.0 * x2 + 1.0;
  double p1r = (x3 - 2.0 * x2 + x) * p.drho;
  double p0mr = 2.0 * omx3 - 3.0 * omx2 + 1.0;
  double p1mr = -(omx3 - 2.0 * omx2 + omx) * p.drho;
  double p0t = 2.0 * y3 - 3.0 * y2 + 1.0;
  double p1t = (y3 - 2.0 * y2 + y) * p.dT;
  double p0mt = 2.0 * omy3 - 3.0 * omy2 + 1.0;
  double p1mt = -(omy3 - 2.0 * omy2 + omy) * p.dT;
  const double *q00 = h.dpdr + 4 * ((long long)(p.ih - 1) + (long long)h.nrho * (p.jh - 1));
  const double *q10 = q00 + 4, *q01 = q00 + 4 * (long long)h.nrho, *q11 = q01 + 4;
  double l[16];
#pragma unroll
  for (int v = 0; v < 4; ++v) {
    l[4 * v + 0] = __ldg(q00 + v);
    l[4 * v + 1] = __ldg(q10 + v);
    l[4 * v + 2] = __ldg(q01 + v);
    l[4 * v + 3] = __ldg(q11 + v);
  }
  double dP_drho = l[0] * p0r * p0t + l[1] * p0mr * p0t + l[2] * p0r * p0mt + l[3] * p0mr * p0mt +
                   l[4] * p0r * p1t + l[5] * p0mr * p1t + l[6] * p0r * p1mt + l[7] * p0mr * p1mt +
                   l[8] * p1r * p0t + l[9] * p1mr * p0t + l[10] * p1r * p0mt + l[11] * p1mr * p0mt +
                   l[12] * p1r * p1t + l[13] * p1mr * p1t + l[14] * p1r * p1mt + l[15] * p1mr * p1mt;
  dP_drho = p.Ye * dP_drho;
  double tmp = p.rhos * p.rhos;
  double pp = tmp * df_drho;
  double dP_dT = tmp * df_drhodT;
  double s = -p.Ye * df_dT;
  double ds_dT = -p.Ye * df_dT2;
  double e = p.Ye * f + T * s;
  double dE_dT = T * ds_dT;
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
  double zz = pp / rho;
  double c_v = dE_dT;
  double chiT = T / pp * dP_dT;
  double chirho = dP_drho / zz;
  double xx = zz * chiT / (T * c_v);
  double gam1 = chiT * xx + chirho;
  double z = 1.0 + (e + CONST_C2) / zz;
  P = pp;
  E = e;
  cv = c_v;
  sound = CONST_C * sqrt(gam1 / z);
}

// helm_rhoe_given Newton (source.F90:24982-25019).  Returns the iterations used; `clamped`
// counts resets to the starting guess after leaving [Tl_eos, Th_eos].
__device__ __forceinline__ int helm_rhoe_newton(const HelmTable &h, double rho, double E0, double abar,
                                                double zbar, double &T, int max_iter, int &clamped,
                                                bool *converged = nullptr) {
  double Told = T;
  int used = 0;
  bool conv = false;
  for (int iter = 1; iter <= max_iter; ++iter) {
    used = iter;
    double E, dE;
    helm_given2(h, rho, T, abar, zbar, E, dE, true);
    double res = E - E0;
    T = T - res / dE;
    double error = fabs(res / E0);
    if ((T < h.Tl) || (T > h.Th)) {
      T = Told;
      error = EM15;
      ++clamped;
    }
    if (error < HELM_TOL) { conv = true; break; }
  }
  if (converged) *converged = conv;
  return used;
}

// helm_rhoP_given Newton (source.F90:24943-24980)
__device__ __forceinline__ int helm_rhoP_newton(const HelmTable &h, double rho, double P0, double abar,
                                                double zbar, double &T, int &clamped) {
  double Told = T;
  int used = 0;
  for (int iter = 1; iter <= 100; ++iter) {
    used = iter;
    double P, dP;
    helm_given1(h, rho, T, abar, zbar, P, dP, true);
    double res = P - P0;
    T = T - res / dP;
    double error = fabs(res / P0);
    if ((T < h.Tl) || (T > h.Th)) {
      T = Told;
      error = EM15;
      ++clamped;
    }
    if (error < HELM_TOL) break;
  }
  return used;
}

// helm_rhoP_given with return_sound (source.F90:24943-24980) for one Riemann side: returns
// rho * e and the sound speed
__device__ __forceinline__ void helm_side_eos_inl(const HelmTable &h, double rho, double p, double abar,
                                                  double zbar, double T, double &rhoe, double &sound) {
  int clamped = 0;
  helm_rhoP_newton(h, rho, p, abar, zbar, T, clamped);
  double Pd, E, cv;
  helm_given_full(h, rho, T, abar, zbar, Pd, E, sound, cv);
  rhoe = E * rho;
}

}  // namespace phl
