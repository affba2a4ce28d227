// phl_split.cu -- FP32 split-precision form of the explicit FV step (hydro and MHD
// configurations).
//
// Storage per cell: conserved state U (FP64, carried across stages and steps), primitive
// deviations W' = (rho - rho_eq, v, p - p_eq, scalars) and (gammae - gammae_eq, gammac) in FP32,
// temperature and internal energy in FP64; MHD adds the face B (FP64), the scaled cell B and
// cell EMFs (FP32).  Reconstruction (LIM2ND, PPH, LIM5TH), the Riemann solvers, face and corner
// EMFs and the flux divergence run in FP32 on the well-balanced deviations: the pressure enters
// every flux as a deviation, so pR - pL, p* - p_eq,face and the momentum flux after the WB fix
// (source/source.F90:8953-8959) are formed without cancelling large numbers, and Mach 1e-3
// perturbations keep their FP32 precision.  The RK combine, the face-B update, cons->prim, the
// Helmholtz Newton inversion and the CFL maximum stay in FP64.  All FP32 quantities are in scaled
// units (rho / rho_ref, p / p_ref, v / v_ref with v_ref^2 = p_ref / rho_ref, phi / v_ref^2,
// B / sqrt(p_ref)), fixed per run, so products of deviations never leave FP32 range whatever the
// problem's cgs magnitudes.
//
// Hydro stage: one fused kernel (k_stage_split_tiled, TMA-staged planes; k_stage_split per
// cell).  MHD stage: k_face_split_mhd_walk (PLM) or k_face_split_mhd (PPH, LIM5TH) per
// direction, k_corner_split per axis, k_bface_split per direction, k_c2p_mhd_split; with the
// learned temperature guess k_c2p_mhd_split_features, k_mlp_guess, k_c2p_mhd_split_guessed.
#include <cuda_runtime.h>
#include <cudaTypedefs.h>
#include <cstdlib>
#include <algorithm>
#include <cstring>
#include "phl_eos_fast.cuh"
#include "phl_mlp.cuh"
#include "phl_umma.cuh"
// kernel namespace of this unit (FP32 flux arithmetic with contraction); see phl_kernels.cuh
#define PHL_KERNEL_UNIT split_unit
#include "phl_runner.h"

namespace phl {

// LIM2ND slope in FP32 without forming df*db (which can overflow or underflow): for df, db of
// the same sign, df*db/(df+db) = df * (db/(df+db)) with the second factor in (0, 1).
__device__ __forceinline__ void plm_f32(float qm, float qc, float qp, float &lo, float &hi) {
  float sf = qp - qc, sb = qc - qm;
  float slope = 0.0f;
  if ((sf > 0.0f && sb > 0.0f) || (sf < 0.0f && sb < 0.0f)) slope = sf * (sb / (sf + sb));
  float tmp = 0.5f * slope;
  lo = qc - tmp;
  hi = qc + tmp;
}

// --------------------------------------------------------------------- FP32 Riemann (hydro)
// qL/qR: [rho (full), v1, v2, (v3), p' (deviation), scalars...] in the normal frame, pe the face
// equilibrium pressure.  Returns the flux with the momentum flux already reduced by pe (the
// reference's WB fix).  Same solver as riemann_hydro (source.F90:15681-16252).
template <int DIM, int NV, int EOSM, int RIEM>
__device__ __forceinline__ void riemann_hydro_split(const float *qL, const float *qR, const float *gL,
                                                    const float *gR, float pe, float gm, float mach_cutoff,
                                                    float *flux, bool flat = false, bool all_mach = false) {
  constexpr int IP = 1 + DIM, IAS = 2 + DIM;
  const float igmm1 = 1.0f / (gm - 1.0f);
  float rhoL = qL[0], inv_rhoL = 1.0f / rhoL, vx1L = qL[1], vx2L = qL[2], vx3L = DIM == 3 ? qL[3] : 0.0f;
  float v2L = vx1L * vx1L + vx2L * vx2L + vx3L * vx3L;
  float pLd = qL[IP], pL = pe + pLd, eint, cL, cR;
  if (EOSM == EOS_FAST) { eint = pL / (gL[0] - 1.0f); cL = sqrtf(gL[1] * pL * inv_rhoL); }
  else if (EOSM == EOS_GIVEN) { eint = gL[0]; cL = gL[1]; }
  else { eint = igmm1 * pL; cL = sqrtf(gm * pL * inv_rhoL); }
  float rhoeL = eint + 0.5f * rhoL * v2L;
  float rhoR = qR[0], inv_rhoR = 1.0f / rhoR, vx1R = qR[1], vx2R = qR[2], vx3R = DIM == 3 ? qR[3] : 0.0f;
  float v2R = vx1R * vx1R + vx2R * vx2R + vx3R * vx3R;
  float pRd = qR[IP], pR = pe + pRd;
  if (EOSM == EOS_FAST) { eint = pR / (gR[0] - 1.0f); cR = sqrtf(gR[1] * pR * inv_rhoR); }
  else if (EOSM == EOS_GIVEN) { eint = gR[0]; cR = gR[1]; }
  else { eint = igmm1 * pR; cR = sqrtf(gm * pR * inv_rhoR); }
  float rhoeR = eint + 0.5f * rhoR * v2R;
  float max_c = fmaxf(cL, cR);
  float sL = fminf(vx1L, vx1R) - max_c;
  float sR = fmaxf(vx1L, vx1R) + max_c;
  float dsuL = sL - vx1L, dsuR = sR - vx1R;
  float ustar = ((pRd - pLd) + rhoL * vx1L * dsuL - rhoR * vx1R * dsuR) / (rhoL * dsuL - rhoR * dsuR);
  float rhostarL = rhoL * (dsuL / (sL - ustar));
  float rhoestarL = rhostarL * (rhoeL * inv_rhoL + (ustar - vx1L) * (ustar + pL * inv_rhoL / dsuL));
  float rhostarR = rhoR * (dsuR / (sR - ustar));
  float rhoestarR = rhostarR * (rhoeR * inv_rhoR + (ustar - vx1R) * (ustar + pR * inv_rhoR / dsuR));
  if (flat) {
    // HLL on a flattened face (USE_SHOCK_FLATTENING, source.F90:15929-16010); the momentum
    // flux takes the pressure deviations, sR pe - sL pe over sR - sL being exactly pe
    sL = fminf(0.0f, sL);
    sR = fmaxf(0.0f, sR);
    float UL[NV], UR[NV], fL[NV], fR[NV];
    UL[0] = rhoL; UL[1] = rhoL * vx1L; UL[2] = rhoL * vx2L; if (DIM == 3) UL[3] = rhoL * vx3L; UL[IP] = rhoeL;
    UR[0] = rhoR; UR[1] = rhoR * vx1R; UR[2] = rhoR * vx2R; if (DIM == 3) UR[3] = rhoR * vx3R; UR[IP] = rhoeR;
    fL[0] = rhoL * vx1L; fL[1] = rhoL * vx1L * vx1L + pLd; fL[2] = rhoL * vx1L * vx2L;
    if (DIM == 3) fL[3] = rhoL * vx1L * vx3L;
    fL[IP] = (rhoeL + pL) * vx1L;
    fR[0] = rhoR * vx1R; fR[1] = rhoR * vx1R * vx1R + pRd; fR[2] = rhoR * vx1R * vx2R;
    if (DIM == 3) fR[3] = rhoR * vx1R * vx3R;
    fR[IP] = (rhoeR + pR) * vx1R;
#pragma unroll
    for (int iv = IAS; iv < NV; ++iv) {
      UL[iv] = rhoL * qL[iv];
      UR[iv] = rhoR * qR[iv];
      fL[iv] = UL[iv] * vx1L;
      fR[iv] = UR[iv] * vx1R;
    }
    const float dh = 1.0f / (sR - sL), ph = sL * sR;
#pragma unroll
    for (int iv = 0; iv < NV; ++iv) flux[iv] = dh * (sR * fL[iv] - sL * fR[iv] + ph * (UR[iv] - UL[iv]));
    return;
  }
  if (RIEM == R_LHLLC) {
    float machL = sqrtf(v2L) / cL, machR = sqrtf(v2R) / cR;
    float chi = fminf(1.0f, fmaxf(machL, machR));
    chi = fmaxf(mach_cutoff, chi);
    float phi = chi * (2.0f - chi);
    float rhobar = 0.5f * (rhoL + rhoR), cbar = 0.5f * (cL + cR);
    float pstar_d = 0.5f * (pLd + pRd) - 0.5f * phi * rhobar * cbar * (vx1R - vx1L);
    if (all_mach && (sL > 0.0f || sR < 0.0f)) {
      // FLUX_IS_ALL_MACH: the upwind state outside the wave fan, pe removed from the momentum flux
      const bool left = sL > 0.0f;
      const float *q = left ? qL : qR;
      float rho = left ? rhoL : rhoR, vx1 = left ? vx1L : vx1R, vx2 = left ? vx2L : vx2R, vx3 = left ? vx3L : vx3R;
      float p = left ? pL : pR, pd = left ? pLd : pRd, rhoe = left ? rhoeL : rhoeR;
      flux[0] = rho * vx1;
      flux[1] = rho * vx1 * vx1 + pd;
      flux[2] = rho * vx1 * vx2;
      if (DIM == 3) flux[3] = rho * vx1 * vx3;
      flux[IP] = (rhoe + p) * vx1;
#pragma unroll
      for (int iv = IAS; iv < NV; ++iv) flux[iv] = rho * q[iv] * vx1;
      return;
    }
    float sgn = copysignf(1.0f, ustar);
    float hp = 0.5f * (1.0f + sgn), hm = 0.5f * (1.0f - sgn);
    float rhostar = hp * rhostarL + hm * rhostarR;
    float mflux = rhostar * ustar;
    flux[0] = mflux;
    flux[1] = mflux * ustar + pstar_d;
    flux[2] = mflux * (hp * vx2L + hm * vx2R);
    if (DIM == 3) flux[3] = mflux * (hp * vx3L + hm * vx3R);
    flux[IP] = (hp * rhoestarL + hm * rhoestarR + (pe + pstar_d)) * ustar;
#pragma unroll
    for (int iv = IAS; iv < NV; ++iv) flux[iv] = mflux * (hp * qL[iv] + hm * qR[iv]);
  } else {
    const bool left = ustar > 0.0f;
    const float *q = left ? qL : qR;
    float rho = left ? rhoL : rhoR, vx1 = left ? vx1L : vx1R, vx2 = left ? vx2L : vx2R, vx3 = left ? vx3L : vx3R;
    float p = left ? pL : pR, pd = left ? pLd : pRd, rhoe = left ? rhoeL : rhoeR;
    float rhostar = left ? rhostarL : rhostarR, rhoestar = left ? rhoestarL : rhoestarR, s = left ? sL : sR;
    const bool sup = left ? (sL >= 0.0f) : (sR < 0.0f);
    float U[NV], f[NV];
    U[0] = rho; U[1] = rho * vx1; U[2] = rho * vx2; if (DIM == 3) U[3] = rho * vx3; U[IP] = rhoe;
    f[0] = rho * vx1; f[1] = rho * vx1 * vx1 + pd; f[2] = rho * vx1 * vx2;
    if (DIM == 3) f[3] = rho * vx1 * vx3;
    f[IP] = (rhoe + p) * vx1;
#pragma unroll
    for (int iv = IAS; iv < NV; ++iv) { U[iv] = rho * q[iv]; f[iv] = rho * vx1 * q[iv]; }
    if (sup) {
#pragma unroll
      for (int iv = 0; iv < NV; ++iv) flux[iv] = f[iv];
    } else {
      float Us[NV];
      Us[0] = rhostar; Us[1] = rhostar * ustar; Us[2] = rhostar * vx2; if (DIM == 3) Us[3] = rhostar * vx3;
      Us[IP] = rhoestar;
#pragma unroll
      for (int iv = IAS; iv < NV; ++iv) Us[iv] = rhostar * q[iv];
#pragma unroll
      for (int iv = 0; iv < NV; ++iv) flux[iv] = f[iv] + s * (Us[iv] - U[iv]);
    }
  }
}

// --------------------------------------------------------------------- FP32 Riemann (MHD)
// HLLD / LHLLD (source.F90:13969-15024) on the split variables: qL/qR as for
// riemann_hydro_split, bL/bR the face B in the normal frame (units sqrt(p_ref)), pe the face
// equilibrium pressure.  Every difference of total pressures is formed from the deviations
// (pT' = p' + B^2/2), the star pressure as pe + pT*' with the weights of the reference, and the
// normal momentum flux is returned with pe removed (the reference's WB fix).  fluxb is the
// induction flux (0, v1 B2 - B1 v2, v1 B3 - B1 v3).
template <int DIM, int NV, int EOSM, int RIEM>
__device__ __forceinline__ void riemann_mhd_split(const float *qL, const float *qR, const float *bL,
                                                  const float *bR, const float *gL, const float *gR, float pe,
                                                  float gm, float mach_cutoff, float *flux, float *fluxb,
                                                  bool flat = false, bool all_mach = false) {
  constexpr int IP = 1 + DIM, IAS = 2 + DIM;
  const float igmm1 = 1.0f / (gm - 1.0f);
  float rhoL = qL[0], inv_rhoL = 1.0f / rhoL, vx1L = qL[1], vx2L = qL[2], vx3L = DIM == 3 ? qL[3] : 0.0f;
  float v2L = vx1L * vx1L + vx2L * vx2L + vx3L * vx3L;
  float pLd = qL[IP], pL = pe + pLd, eint, c2L, c2R;
  if (EOSM == EOS_FAST) { eint = pL / (gL[0] - 1.0f); c2L = gL[1] * pL * inv_rhoL; }
  else if (EOSM == EOS_GIVEN) { eint = gL[0]; c2L = gL[1] * gL[1]; }
  else { eint = pL * igmm1; c2L = gm * pL * inv_rhoL; }
  float rhoeL = eint + 0.5f * rhoL * v2L;
  float bx1L = bL[0], bx2L = bL[1], bx3L = DIM == 3 ? bL[2] : 0.0f;
  float rhoR = qR[0], inv_rhoR = 1.0f / rhoR, vx1R = qR[1], vx2R = qR[2], vx3R = DIM == 3 ? qR[3] : 0.0f;
  float v2R = vx1R * vx1R + vx2R * vx2R + vx3R * vx3R;
  float pRd = qR[IP], pR = pe + pRd;
  if (EOSM == EOS_FAST) { eint = pR / (gR[0] - 1.0f); c2R = gR[1] * pR * inv_rhoR; }
  else if (EOSM == EOS_GIVEN) { eint = gR[0]; c2R = gR[1] * gR[1]; }
  else { eint = pR * igmm1; c2R = gm * pR * inv_rhoR; }
  float rhoeR = eint + 0.5f * rhoR * v2R;
  float bx1R = bR[0], bx2R = bR[1], bx3R = DIM == 3 ? bR[2] : 0.0f;

  float bx1 = 0.5f * (bx1L + bx1R), bx1_2 = bx1 * bx1;
  float pbL = 0.5f * (bx1_2 + bx2L * bx2L + bx3L * bx3L);
  float pbR = 0.5f * (bx1_2 + bx2R * bx2R + bx3R * bx3R);
  rhoeL = rhoeL + pbL;
  rhoeR = rhoeR + pbR;
  float ptLd = pLd + pbL, ptRd = pRd + pbR;  // total pressure deviations
  float ptL = pe + ptLd, ptR = pe + ptRd;
  float a2L = 2.0f * pbL * inv_rhoL, a2R = 2.0f * pbR * inv_rhoR;
  float an2L = bx1_2 * inv_rhoL, an2R = bx1_2 * inv_rhoR;
  float dummy = c2L + a2L;
  const float cf2L = 0.5f * (c2L + a2L + sqrtf(fmaxf(dummy * dummy - 4.0f * c2L * an2L, 0.0f)));
  dummy = c2R + a2R;
  const float cf2R = 0.5f * (c2R + a2R + sqrtf(fmaxf(dummy * dummy - 4.0f * c2R * an2R, 0.0f)));
  float cL = sqrtf(cf2L), cR = sqrtf(cf2R);
  float max_c = fmaxf(cL, cR);
  float sL = fminf(vx1L, vx1R) - max_c;
  float sR = fmaxf(vx1L, vx1R) + max_c;
  float dsuL = sL - vx1L, dsuR = sR - vx1R;
  float inv_temp1 = 1.0f / (dsuR * rhoR - dsuL * rhoL);
  float ustar = (dsuR * rhoR * vx1R - dsuL * rhoL * vx1L - (ptRd - ptLd)) * inv_temp1;
  float dsumL = sL - ustar, dsumR = sR - ustar;
  float phi = 1.0f;
  if (RIEM == R_LHLLD) {
    dummy = v2L + a2L;
    float cu2L = 0.5f * (v2L + a2L + sqrtf(fmaxf(dummy * dummy - 4.0f * v2L * an2L, 0.0f)));
    dummy = v2R + a2R;
    float cu2R = 0.5f * (v2R + a2R + sqrtf(fmaxf(dummy * dummy - 4.0f * v2R * an2R, 0.0f)));
    // the fast Mach numbers compared as squares (cu^2 / cf^2): one square root, for the larger
    const float mm2 = fmaxf(cu2L / cf2L, cu2R / cf2R);
    if (mm2 < 0.36f) {
      float chi = fminf(1.0f, sqrtf(mm2));
      chi = fmaxf(mach_cutoff, chi);
      phi = chi * (2.0f - chi);
    }
  }
  if (flat) {
    // HLL on a flattened face (source.F90:14386-14495), total-pressure deviations in the
    // momentum flux as in the HLL of riemann_hydro_split
    sL = fminf(0.0f, sL);
    sR = fmaxf(0.0f, sR);
    float UL[NV], UR[NV], fL[NV], fR[NV];
    UL[0] = rhoL; UL[1] = rhoL * vx1L; UL[2] = rhoL * vx2L; if (DIM == 3) UL[3] = rhoL * vx3L; UL[IP] = rhoeL;
    UR[0] = rhoR; UR[1] = rhoR * vx1R; UR[2] = rhoR * vx2R; if (DIM == 3) UR[3] = rhoR * vx3R; UR[IP] = rhoeR;
    fL[0] = rhoL * vx1L; fL[1] = rhoL * vx1L * vx1L + ptLd - bx1_2; fL[2] = rhoL * vx1L * vx2L - bx1 * bx2L;
    if (DIM == 3) fL[3] = rhoL * vx1L * vx3L - bx1 * bx3L;
    fL[IP] = (rhoeL + ptL) * vx1L - bx1 * (bx1 * vx1L + bx2L * vx2L + bx3L * vx3L);
    fR[0] = rhoR * vx1R; fR[1] = rhoR * vx1R * vx1R + ptRd - bx1_2; fR[2] = rhoR * vx1R * vx2R - bx1 * bx2R;
    if (DIM == 3) fR[3] = rhoR * vx1R * vx3R - bx1 * bx3R;
    fR[IP] = (rhoeR + ptR) * vx1R - bx1 * (bx1 * vx1R + bx2R * vx2R + bx3R * vx3R);
#pragma unroll
    for (int iv = IAS; iv < NV; ++iv) {
      UL[iv] = rhoL * qL[iv];
      UR[iv] = rhoR * qR[iv];
      fL[iv] = UL[iv] * vx1L;
      fR[iv] = UR[iv] * vx1R;
    }
    const float UbL[3] = {bx1, bx2L, bx3L}, UbR[3] = {bx1, bx2R, bx3R};
    const float fbL[3] = {0.0f, vx1L * bx2L - vx2L * bx1, vx1L * bx3L - vx3L * bx1};
    const float fbR[3] = {0.0f, vx1R * bx2R - vx2R * bx1, vx1R * bx3R - vx3R * bx1};
    const float dh = 1.0f / (sR - sL), ph = sL * sR;
#pragma unroll
    for (int iv = 0; iv < NV; ++iv) flux[iv] = dh * (sR * fL[iv] - sL * fR[iv] + ph * (UR[iv] - UL[iv]));
#pragma unroll
    for (int iv = 0; iv < DIM; ++iv) fluxb[iv] = dh * (sR * fbL[iv] - sL * fbR[iv] + ph * (UbR[iv] - UbL[iv]));
    return;
  }
  // star total pressure: the weights sum to one, so pe factors out
  float pstar_d = (dsuR * rhoR * ptLd - dsuL * rhoL * ptRd - phi * rhoL * rhoR * dsuR * dsuL * (vx1L - vx1R)) *
                  inv_temp1;
  const float idsumL = 1.0f / dsumL, idsumR = 1.0f / dsumR;
  float rhostarL = rhoL * dsuL * idsumL, rhostarR = rhoR * dsuR * idsumR;
  float a1_inv = 1.0f / (rhoL * dsuL * dsumL - bx1_2);
  float vx2starL = vx2L - bx1 * bx2L * (ustar - vx1L) * a1_inv;
  float bx2starL = bx2L * (rhoL * dsuL * dsuL - bx1_2) * a1_inv;
  float vx3starL = vx3L - bx1 * bx3L * (ustar - vx1L) * a1_inv;
  float bx3starL = bx3L * (rhoL * dsuL * dsuL - bx1_2) * a1_inv;
  float a2_inv = 1.0f / (rhoR * dsuR * dsumR - bx1_2);
  float vx2starR = vx2R - bx1 * bx2R * (ustar - vx1R) * a2_inv;
  float bx2starR = bx2R * (rhoR * dsuR * dsuR - bx1_2) * a2_inv;
  float vx3starR = vx3R - bx1 * bx3R * (ustar - vx1R) * a2_inv;
  float bx3starR = bx3R * (rhoR * dsuR * dsuR - bx1_2) * a2_inv;
  float vdotbL = vx1L * bx1 + vx2L * bx2L + vx3L * bx3L;
  float vdotbR = vx1R * bx1 + vx2R * bx2R + vx3R * bx3R;
  float vdotbstarL = ustar * bx1 + vx2starL * bx2starL + vx3starL * bx3starL;
  float vdotbstarR = ustar * bx1 + vx2starR * bx2starR + vx3starR * bx3starR;
  // -pT u + pT* u* with pe factored: pe (u* - u) + (pT*' u* - pT' u)
  float rhoestarL = (dsuL * rhoeL + pe * (ustar - vx1L) + (pstar_d * ustar - ptLd * vx1L) +
                     bx1 * (vdotbL - vdotbstarL)) * idsumL;
  float rhoestarR = (dsuR * rhoeR + pe * (ustar - vx1R) + (pstar_d * ustar - ptRd * vx1R) +
                     bx1 * (vdotbR - vdotbstarR)) * idsumR;
  // sqrt(rho*) and 1 / sqrt(rho*) from one reciprocal square root per side
  const float rsqL = rsqrtf(rhostarL), rsqR = rsqrtf(rhostarR);
  float sqrt_rhostarL = rhostarL * rsqL, sqrt_rhostarR = rhostarR * rsqR;
  float abs_bx1 = fabsf(bx1);
  float sstarL = ustar - abs_bx1 * rsqL;
  float sstarR = ustar + abs_bx1 * rsqR;
  float inv_sqr_bar = 1.0f / (sqrt_rhostarL + sqrt_rhostarR);
  float sgn = copysignf(1.0f, bx1);
  float vx22star = (sqrt_rhostarL * vx2starL + sqrt_rhostarR * vx2starR + (bx2starR - bx2starL) * sgn) * inv_sqr_bar;
  float bx22star = (sqrt_rhostarL * bx2starR + sqrt_rhostarR * bx2starL +
                    sqrt_rhostarL * sqrt_rhostarR * (vx2starR - vx2starL) * sgn) * inv_sqr_bar;
  float vx32star = (sqrt_rhostarL * vx3starL + sqrt_rhostarR * vx3starR + (bx3starR - bx3starL) * sgn) * inv_sqr_bar;
  float bx32star = (sqrt_rhostarL * bx3starR + sqrt_rhostarR * bx3starL +
                    sqrt_rhostarL * sqrt_rhostarR * (vx3starR - vx3starL) * sgn) * inv_sqr_bar;
  float vdotb2star = ustar * bx1 + vx22star * bx22star + vx32star * bx32star;
  float rhoe2starL = rhoestarL - sqrt_rhostarL * (vdotbstarL - vdotb2star) * sgn;
  float rhoe2starR = rhoestarR + sqrt_rhostarR * (vdotbstarR - vdotb2star) * sgn;

  fluxb[0] = 0.0f;
  if (RIEM == R_LHLLD) {
    float rho, vx1, vx2, vx3, rhoe, bx2, bx3, pres_d = pstar_d;
    if (all_mach && sL > 0.0f) {
      // FLUX_IS_ALL_MACH: the outer states as well (source.F90:14576-14632)
      rho = rhoL; vx1 = vx1L; vx2 = vx2L; vx3 = vx3L; rhoe = rhoeL; bx2 = bx2L; bx3 = bx3L; pres_d = ptLd;
    } else if (sstarL > 0.0f) {
      rho = rhostarL; vx1 = ustar; vx2 = vx2starL; vx3 = vx3starL; rhoe = rhoestarL; bx2 = bx2starL; bx3 = bx3starL;
    } else if (ustar > 0.0f) {
      rho = rhostarL; vx1 = ustar; vx2 = vx22star; vx3 = vx32star; rhoe = rhoe2starL; bx2 = bx22star; bx3 = bx32star;
    } else if (sstarR > 0.0f) {
      rho = rhostarR; vx1 = ustar; vx2 = vx22star; vx3 = vx32star; rhoe = rhoe2starR; bx2 = bx22star; bx3 = bx32star;
    } else if (!all_mach || sR > 0.0f) {
      rho = rhostarR; vx1 = ustar; vx2 = vx2starR; vx3 = vx3starR; rhoe = rhoestarR; bx2 = bx2starR; bx3 = bx3starR;
    } else {
      rho = rhoR; vx1 = vx1R; vx2 = vx2R; vx3 = vx3R; rhoe = rhoeR; bx2 = bx2R; bx3 = bx3R; pres_d = ptRd;
    }
    flux[0] = rho * vx1;
    flux[1] = rho * vx1 * vx1 + pres_d - bx1_2;
    flux[2] = rho * vx1 * vx2 - bx1 * bx2;
    if (DIM == 3) flux[3] = rho * vx1 * vx3 - bx1 * bx3;
    flux[IP] = (rhoe + (pe + pres_d)) * vx1 - bx1 * (bx1 * vx1 + vx2 * bx2 + vx3 * bx3);
    float sg = copysignf(1.0f, vx1), hp = 0.5f * (1.0f + sg), hm = 0.5f * (1.0f - sg);
#pragma unroll
    for (int iv = IAS; iv < NV; ++iv) flux[iv] = rho * vx1 * (hp * qL[iv] + hm * qR[iv]);
    fluxb[1] = vx1 * bx2 - bx1 * vx2;
    if (DIM == 3) fluxb[2] = vx1 * bx3 - bx1 * vx3;
    return;
  }
  const bool left = ustar > 0.0f;
  const float *q = left ? qL : qR;
  float rho = left ? rhoL : rhoR, vx1 = left ? vx1L : vx1R, vx2 = left ? vx2L : vx2R, vx3 = left ? vx3L : vx3R;
  float rhoe = left ? rhoeL : rhoeR, pt = left ? ptL : ptR, ptd = left ? ptLd : ptRd;
  float bx2 = left ? bx2L : bx2R, bx3 = left ? bx3L : bx3R;
  float vdotb = left ? vdotbL : vdotbR, rhostar = left ? rhostarL : rhostarR;
  float vx2s = left ? vx2starL : vx2starR, vx3s = left ? vx3starL : vx3starR;
  float bx2s = left ? bx2starL : bx2starR, bx3s = left ? bx3starL : bx3starR;
  float rhoes = left ? rhoestarL : rhoestarR, rhoe2s = left ? rhoe2starL : rhoe2starR;
  float s = left ? sL : sR, sst = left ? sstarL : sstarR;
  const bool outer = left ? (sL > 0.0f) : (sR < 0.0f);
  const bool single = left ? (sstarL > 0.0f) : (sstarR < 0.0f);
  constexpr int NB = DIM == 3 ? 3 : 2;
  float U[NV], f[NV], Ub[3], fb[3];
  U[0] = rho; U[1] = rho * vx1; U[2] = rho * vx2; if (DIM == 3) U[3] = rho * vx3; U[IP] = rhoe;
  f[0] = rho * vx1; f[1] = rho * vx1 * vx1 + ptd - bx1_2; f[2] = rho * vx1 * vx2 - bx1 * bx2;
  if (DIM == 3) f[3] = rho * vx1 * vx3 - bx1 * bx3;
  f[IP] = (rhoe + pt) * vx1 - bx1 * vdotb;
#pragma unroll
  for (int iv = IAS; iv < NV; ++iv) { U[iv] = rho * q[iv]; f[iv] = rho * vx1 * q[iv]; }
  Ub[0] = bx1; Ub[1] = bx2; Ub[2] = bx3;
  fb[0] = 0.0f; fb[1] = vx1 * bx2 - bx1 * vx2; fb[2] = vx1 * bx3 - bx1 * vx3;
  if (outer) {
#pragma unroll
    for (int iv = 0; iv < NV; ++iv) flux[iv] = f[iv];
#pragma unroll
    for (int iv = 0; iv < NB; ++iv) fluxb[iv] = fb[iv];
    return;
  }
  float Us[NV], Ubs[3];
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
  float Uss[NV], Ubss[3];
  Uss[0] = rhostar; Uss[1] = rhostar * ustar; Uss[2] = rhostar * vx22star; if (DIM == 3) Uss[3] = rhostar * vx32star;
  Uss[IP] = rhoe2s;
#pragma unroll
  for (int iv = IAS; iv < NV; ++iv) Uss[iv] = rhostar * q[iv];
  Ubss[0] = bx1; Ubss[1] = bx22star; Ubss[2] = bx32star;
#pragma unroll
  for (int iv = 0; iv < NV; ++iv) {
    float d0 = Us[iv];
    flux[iv] = f[iv] + s * (d0 - U[iv]) + sst * (Uss[iv] - d0);
  }
#pragma unroll
  for (int iv = 0; iv < NB; ++iv) {
    float d0 = Ubs[iv];
    fluxb[iv] = fb[iv] + s * (d0 - Ub[iv]) + sst * (Ubss[iv] - d0);
  }
}

// --------------------------------------------------------------------- FP32 loads
template <class C>
__device__ __forceinline__ void load_wf(const Prm &P, int i, int j, int k, float w[C::NV], float g2[2]) {
  const Geo &g = P.g;
  bool f0 = false, f1 = false, f2 = false;
  int si = map_index(i, g.nx[0], g.bc[0][0], g.bc[0][1], f0);
  int sj = map_index(j, g.nx[1], g.bc[1][0], g.bc[1][1], f1);
  int sk = C::DIM == 3 ? map_index(k, g.nx[2], g.bc[2][0], g.bc[2][1], f2) : 0;
  long long c = lin(g, si, sj, sk);
#pragma unroll
  for (int iv = 0; iv < C::NV; ++iv) w[iv] = __ldg(P.Wf_in + (long long)iv * g.N + c);
  if (f0) w[1] = -w[1];
  if (f1) w[2] = -w[2];
  if (C::DIM == 3 && f2) w[3] = -w[3];
  if (C::HELM) {
    g2[0] = __ldg(P.gf_in + c);
    g2[1] = __ldg(P.gf_in + g.N + c);
  }
}

// the same for an interior cell given by its linear index (no mapping, no mirror)
template <class C>
__device__ __forceinline__ void load_wf_at(const Prm &P, long long c, float w[C::NV], float g2[2]) {
  const long long N = P.g.N;
#pragma unroll
  for (int iv = 0; iv < C::NV; ++iv) w[iv] = __ldg(P.Wf_in + iv * N + c);
  if (C::HELM) {
    g2[0] = __ldg(P.gf_in + c);
    g2[1] = __ldg(P.gf_in + N + c);
  }
}

// linear-index step between neighbours along d
__device__ __forceinline__ long long dir_stride(const Geo &g, int d) {
  return d == 0 ? 1 : (d == 1 ? (long long)g.nx[0] : (long long)g.nx[0] * g.nx[1]);
}

// States of the four cells m-2..m+1 around the low face of cell m: variable iv of cell s is
// w(s, iv), FASTEOS gamma q is g(s, q).
template <int NV>
struct RegCells {
  const float *w_[6], *g_[6];
  __device__ __forceinline__ float w(int s, int iv) const { return w_[s][iv]; }
  __device__ __forceinline__ float g(int s, int q) const { return g_[s][q]; }
};
// cells in a shared-memory array: variable iv of cell s at base[off[s] + iv * vs]
template <int NV>
struct SmemCells {
  const float *base;
  int off[4], vs;
  __device__ __forceinline__ float w(int s, int iv) const { return base[off[s] + iv * vs]; }
  __device__ __forceinline__ float g(int s, int q) const { return base[off[s] + (NV + q) * vs]; }
};

// the per-side helm_rhoP_given of the split form, out of line: the split stage kernels call it
// twice per face, and an inlined Helmholtz evaluation at each site costs them their registers.
// It runs the contracted-coefficient evaluation of phl_eos_fast.cuh (the FP64 form keeps the
// reference's evaluation order, helm_side_eos_inl); results agree to rounding.
static __device__ __noinline__ void helm_side_eos(const HelmTable &h, double rho, double p, double abar,
                                                  double zbar, double T, double &rhoe, double &sound) {
  helm_side_eos_fast_inl(h, rho, p, abar, zbar, T, rhoe, sound);
}

// Helmholtz without USE_FASTEOS, split form: helm_rhoP_given (FP64) for one side of a face from
// the scaled FP32 face state and temperature guess; returns rho*e and the sound speed, scaled
template <class C>
__device__ __forceinline__ void split_side_eos(const Prm &P, const float *q, float pe, float tguess, float &rhoe_s,
                                               float &c_s) {
  const double rho = (double)q[0] * P.rho_ref, p = ((double)pe + (double)q[C::IP]) * P.p_ref;
  const double ye = q[C::IAS], abar = 1.0 / (double)q[C::IAS + 1], zbar = ye * abar;
  double rhoe, snd;
  helm_side_eos(P.helm, rho, p, abar, zbar, (double)tguess, rhoe, snd);
  rhoe_s = (float)(rhoe * P.inv_p_ref);
  c_s = (float)(snd * P.inv_v_ref);
}

// FP32 face values of one variable from the values of cells m-3 .. m+2 (v[0] .. v[5]; LIM2ND and
// PPH read v[1] .. v[4])
template <class C>
__device__ __forceinline__ void rec_face_f32(const float v[6], bool limited, float &qL, float &qR) {
  float lo, hi;
  if (C::REC == REC_LIM2ND) {
    plm_f32(v[1], v[2], v[3], lo, hi);
    qL = hi;
    plm_f32(v[2], v[3], v[4], lo, hi);
    qR = lo;
  } else {
    rec_edges<float, C::REC>(limited, v[0], v[1], v[2], v[3], v[4], lo, hi);
    qL = hi;
    rec_edges<float, C::REC>(limited, v[1], v[2], v[3], v[4], v[5], lo, hi);
    qR = lo;
  }
}

// USE_SHOCK_FLATTENING on the FP32 edge values: v holds cells m-3..m+2 of the face; a flagged
// cell m-1 (fa) or m (fb) gives its edge by LIM2ND PLM (source.F90:8743-8827, 9635-9700)
__device__ __forceinline__ void flatten_face_f32(const float v[6], bool fa, bool fb, float &qL, float &qR) {
  float lo, hi;
  if (fa) {
    plm_f32(v[1], v[2], v[3], lo, hi);
    qL = hi;
  }
  if (fb) {
    plm_f32(v[2], v[3], v[4], lo, hi);
    qR = lo;
  }
}
// the x1 sweep's gamma handling on flagged faces with WB (source.F90:8829-8872), reproduced as
// written: PLM gammas without the equilibrium gamma_e replace the flagged side, and the face's
// eq_gammae_x1 is added once more to the other side; cell m-1 before cell m
__device__ __forceinline__ void flatten_gamma_x1(const float gv[2][6], bool fa, bool fb, float ge, float gL[2],
                                                 float gR[2]) {
  float lo, hi;
  if (fa) {
#pragma unroll
    for (int iv = 0; iv < 2; ++iv) {
      plm_f32(gv[iv][1], gv[iv][2], gv[iv][3], lo, hi);
      gL[iv] = hi;
    }
    gR[0] = gR[0] + ge;
  }
  if (fb) {
#pragma unroll
    for (int iv = 0; iv < 2; ++iv) {
      plm_f32(gv[iv][2], gv[iv][3], gv[iv][4], lo, hi);
      gR[iv] = lo;
    }
    gL[0] = gL[0] + ge;
  }
}

// flux through the low face of cell m along d from the FP32 deviation states of cells m-2..m+1
template <class C, class Cells>
__device__ __forceinline__ void face_flux_cells(const Prm &P, int d, int fi, int fj, int fk, const Cells &cl,
                                                float F[C::NV]) {
  constexpr int NV = C::NV, IP = C::IP, SW = C::SW;
  const Geo &g = P.g;
  // cl holds cells m-SW .. m+SW-1; v[] of rec_face_f32 holds cells m-3 .. m+2
  // USE_SHOCK_FLATTENING: is_flattened of cells m-1 (fa) and m (fb); a flagged cell's edges
  // fall back to LIM2ND PLM, and the face takes the HLL flux
  bool fa = false, fb = false;
  if (C::SF) {
    fa = P.sf_flag[sf_flag_index<C>(g, fi - (d == 0), fj - (d == 1), fk - (d == 2))] != 0;
    fb = P.sf_flag[sf_flag_index<C>(g, fi, fj, fk)] != 0;
  }
  float qL[NV], qR[NV];
#pragma unroll
  for (int iv = 0; iv < NV; ++iv) {
    float v[6];
#pragma unroll
    for (int q = 0; q < 6; ++q) v[q] = (q >= 3 - SW && q < 3 + SW) ? cl.w(q - (3 - SW), iv) : 0.0f;
    rec_face_f32<C>(v, C::REC == REC_LIM5TH || iv >= C::IAS, qL[iv], qR[iv]);
    if (C::SF && C::REC != REC_LIM2ND) flatten_face_f32(v, fa, fb, qL[iv], qR[iv]);
  }
  if (d == 1) {
    float a = qL[1], b = qL[2]; qL[1] = b; qL[2] = -a;
    a = qR[1]; b = qR[2]; qR[1] = b; qR[2] = -a;
  } else if (C::DIM == 3 && d == 2) {
    float a = qL[1], b = qL[2], c = qL[3]; qL[1] = c; qL[2] = a; qL[3] = b;
    a = qR[1]; b = qR[2]; c = qR[3]; qR[1] = c; qR[2] = a; qR[3] = b;
  }
  float pe = 0.0f, phi_f = 0.0f;
  long long fbg = 0;
  if (C::WB || C::ETOT) fbg = bg_face(g, d, fi, fj, fk);
  if (C::WB) {
    float rho_eq = __ldg(P.sf_rho_f[d] + fbg);
    qL[0] = rho_eq + qL[0];
    qR[0] = rho_eq + qR[0];
    pe = __ldg(P.sf_p_f[d] + fbg);
  }
  float gL[2] = {0.f, 0.f}, gR[2] = {0.f, 0.f};
  if (C::FAST) {
    const bool late = C::SF && C::WB && d == 0;
    float gv[2][6];
#pragma unroll
    for (int iv = 0; iv < 2; ++iv) {
#pragma unroll
      for (int q = 0; q < 6; ++q) gv[iv][q] = (q >= 3 - SW && q < 3 + SW) ? cl.g(q - (3 - SW), iv) : 0.0f;
      rec_face_f32<C>(gv[iv], C::REC == REC_LIM5TH, gL[iv], gR[iv]);
      if (C::SF && C::REC != REC_LIM2ND && !late) flatten_face_f32(gv[iv], fa, fb, gL[iv], gR[iv]);
    }
    if (C::WB) {
      float ge = __ldg(P.sf_ge_f[d] + fbg);
      gL[0] = gL[0] + ge;
      gR[0] = gR[0] + ge;
      if (late) flatten_gamma_x1(gv, fa, fb, ge, gL, gR);
    }
  } else if (C::HELM) {
    // without USE_FASTEOS the first gamma slot holds the stage input's temperature
    const float tface = 0.5f * (cl.g(SW - 1, 0) + cl.g(SW, 0));
    split_side_eos<C>(P, qL, pe, tface, gL[0], gL[1]);
    split_side_eos<C>(P, qR, pe, tface, gR[0], gR[1]);
  }
  riemann_hydro_split<C::DIM, NV, C::EOSM, C::RIEM>(qL, qR, gL, gR, pe, (float)g.gm, (float)g.mach_cutoff, F,
                                                    C::SF && (fa || fb), g.all_mach != 0);
  if (d == 1) {
    float a = F[1], b = F[2]; F[1] = -b; F[2] = a;
  } else if (C::DIM == 3 && d == 2) {
    float a = F[1], b = F[2], c = F[3]; F[1] = b; F[2] = c; F[3] = a;
  }
  if (C::ETOT) {
    phi_f = __ldg(P.sf_phi_f[d] + fbg);
    F[IP] = F[IP] + F[0] * phi_f;
  }
}

template <class C>
__device__ __forceinline__ void face_flux_split(const Prm &P, int d, int fi, int fj, int fk, const float *const *w,
                                                const float *const *gm, float F[C::NV]) {
  RegCells<C::NV> cl;
#pragma unroll
  for (int q = 0; q < 2 * C::SW; ++q) {
    cl.w_[q] = w[q];
    cl.g_[q] = gm[q];
  }
  face_flux_cells<C>(P, d, fi, fj, fk, cl, F);
}

// --------------------------------------------------------------------- split stage kernels
// Per-cell statistics of a stage, reduced once per block.
// per-thread counters (32-bit: a thread's cells times 100 iterations stay far below 2^32; the
// block sums go to the 64-bit counters of the context)
struct SplitStat {
  double smax = 0.0;
  unsigned calls = 0, iters = 0, nonconv = 0, clamp = 0, bad = 0;
  unsigned mlp_acc = 0, mlp_rej = 0, gevals = 0;  // learned guess in the step
};

// Everything of a stage after the flux divergence, for one cell: flux divergence to physical
// units, gravity, RK combine (FP64), cons -> prim with the Helmholtz Newton (FP64), FP32
// deviations out, and the cell's CFL speed in the last stage.  res: divergence in scaled units.
template <class C>
__device__ __forceinline__ void split_cell_update(const Prm &P, long long c, int i, int j, int k,
                                                  const float res[C::NV], float rho_dev, SplitStat &st) {
  constexpr int NV = C::NV, IP = C::IP, IAS = C::IAS, DIM = C::DIM;
  const Geo &g = P.g;
  const double dt = P.scal[1];
  // the Newton's warm start, loaded before the state stores so that its latency overlaps them
  const double Tw = C::HELM ? P.temp[c] : 0.0;
  // back to physical units: mass and scalar fluxes scale with rho_ref v_ref, momentum with
  // p_ref, energy with p_ref v_ref
  const double fm = P.rho_ref * P.v_ref, fe = P.p_ref * P.v_ref;
  double rd[NV];
  rd[0] = (double)res[0] * fm;
#pragma unroll
  for (int d = 0; d < DIM; ++d) rd[1 + d] = (double)res[1 + d] * P.p_ref;
  rd[IP] = (double)res[IP] * fe;
#pragma unroll
  for (int iv = IAS; iv < NV; ++iv) rd[iv] = (double)res[iv] * fm;
  const long long bc = bg_cc(g, i, j, k);
  if (C::GRAV) {
    const double rho_dev_phys = (double)rho_dev * P.rho_ref;
#pragma unroll
    for (int d = 0; d < DIM; ++d)
      rd[1 + d] -= rho_dev_phys * __ldg(P.grav + (long long)d * (g.bg_profile ? g.nx[1] : g.N) + bc);
  }
  double u0[NV], u[NV];
  if (P.first_stage) {
#pragma unroll
    for (int iv = 0; iv < NV; ++iv) {
      u0[iv] = P.U[(long long)iv * g.N + c];
      u[iv] = u0[iv];
      P.U0[(long long)iv * g.N + c] = u0[iv];
    }
  } else {
#pragma unroll
    for (int iv = 0; iv < NV; ++iv) {
      u0[iv] = P.U0[(long long)iv * g.N + c];
      u[iv] = P.U[(long long)iv * g.N + c];
    }
  }
  if (g.use_acc) constant_acceleration<DIM, IP>(g, u, rd);
  const double a1 = P.a1, a2 = P.a2, a3 = P.c3 * dt;
#pragma unroll
  for (int iv = 0; iv < NV; ++iv) {
    u[iv] = a1 * u0[iv] + a2 * u[iv] + a3 * rd[iv];
    P.U[(long long)iv * g.N + c] = u[iv];
  }
  // cons -> prim + EoS in FP64
  double rho = u[0], inv_rho = 1.0 / rho;
  double ke = u[1] * u[1] + u[2] * u[2] + (DIM == 3 ? u[3] * u[3] : 0.0);
  double eint = u[IP] - 0.5 * ke * inv_rho;
  if (C::ETOT) eint = eint - rho * __ldg(P.phi_cc + bc);
  double p, T, sound = 0.0;
  if (C::HELM) {
    double ye = u[IAS] * inv_rho, inv_abar = u[IAS + 1] * inv_rho;
    T = Tw;
    int clamped = 0;
    bool conv = false;
    HelmCell hc;
    helm_cell_init_rho(P.helm, hc, rho, ye);
    helm_cell_contract(P.helm, hc, helm_node_index(P.helm.T, P.helm.nT, P.helm.log10_T1, P.helm.dT, T));
    int it = helm_rhoe_fast(P.helm, hc, inv_rho, eint * inv_rho, inv_abar, T, 100, clamped, conv);
    st.calls += 1; st.iters += it; st.nonconv += !conv; st.clamp += clamped;
    double sound2;
    helm_cell_p_sound2(P.helm, hc, rho, inv_rho, T, inv_abar, p, sound2);
    if (P.last_stage) sound = sqrt(sound2);
    if (C::FAST) {
      // gamma_e to FP32 as a deviation from equilibrium (formed in FP64), gamma_c to FP32 as it is
      double ge = p / eint + 1.0;
      const float gc = (float)(sound2 * rho) / (float)p;
      if (C::WB) ge = ge - __ldg(P.eq_ge_cc + bc);
      P.gf_out[c] = (float)ge;
      P.gf_out[g.N + c] = gc;
    } else {
      P.gf_out[c] = (float)T;
    }
  } else {
    p = (g.gm - 1.0) * eint;
    T = p / (rho * CONST_RGAS * (1.0 / g.mu));
    sound = sqrt(g.gm * p / rho);
  }
  double rdev = rho, pdev = p;
  if (C::WB) {
    rdev = rho - __ldg(P.eq_rho_cc + bc);
    pdev = p - __ldg(P.eq_p_cc + bc);
  }
  P.Wf_out[c] = (float)(rdev * P.inv_rho_ref);
#pragma unroll
  for (int d = 0; d < DIM; ++d) P.Wf_out[(long long)(1 + d) * g.N + c] = (float)(u[1 + d] * inv_rho * P.inv_v_ref);
  P.Wf_out[(long long)IP * g.N + c] = (float)(pdev * P.inv_p_ref);
#pragma unroll
  for (int iv = IAS; iv < NV; ++iv) P.Wf_out[(long long)iv * g.N + c] = (float)(u[iv] * inv_rho);
  P.temp[c] = T;
  P.eint[c] = eint;
  if (!(rho > 0.0) || !(p > 0.0) || !(T > 0.0) || !isfinite(eint)) st.bad += 1;
  if (P.last_stage) {
    double sx1 = (fabs(u[1] * inv_rho) + sound) * g.inv_dx[0];
    double sx2 = (fabs(u[2] * inv_rho) + sound) * g.inv_dx[1];
    double sm = sx1 + sx2;
    if (DIM == 3) sm = (fabs(u[3] * inv_rho) + sound) * g.inv_dx[2] + sm;
    st.smax = fmax(st.smax, sm);
  }
}

template <class C>
__device__ __forceinline__ void split_stat_flush(const Prm &P, const SplitStat &st) {
  if (P.last_stage) block_max_atomic(st.smax, P.smax_bits);
  if (C::HELM) {
    block_sum_atomic(st.calls, P.stat + STAT_NEWTON_CALLS);
    block_sum_atomic(st.iters, P.stat + STAT_NEWTON_ITERS);
    block_sum_atomic(st.nonconv, P.stat + STAT_NEWTON_NONCONV);
    block_sum_atomic(st.clamp, P.stat + STAT_NEWTON_CLAMP);
    if (P.mlp_w) {
      block_sum_atomic(st.mlp_acc, P.stat + STAT_MLP_ACC);
      block_sum_atomic(st.mlp_rej, P.stat + STAT_MLP_REJ);
      block_sum_atomic(st.gevals, P.stat + STAT_GUESS_EVALS);
    }
  }
  block_sum_atomic(st.bad, P.stat + STAT_NONFINITE);
}

// One thread per cell; every face is solved by both of its cells.  Any grid size.
template <class C>
__global__ void __launch_bounds__(128) k_stage_split(Prm P) {
  if (!*P.active) return;
  constexpr int NV = C::NV, DIM = C::DIM;
  const Geo &g = P.g;
  long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  SplitStat st;
  if (c < g.N) {
    int i, j, k;
    unflatten3(c, g.nx[0], g.nx[1], i, j, k);
    float res[NV];
    float rho_dev = 0.0f;
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
      // cells c-SW .. c+SW along d: the low face reads the first 2 SW, the high face the last
      constexpr int NS = 2 * C::SW + 1;
      float w[NS][NV], gmv[NS][2];
#pragma unroll
      for (int s = 0; s < NS; ++s) {
        int ii = i + (d == 0 ? s - C::SW : 0), jj = j + (d == 1 ? s - C::SW : 0), kk = k + (d == 2 ? s - C::SW : 0);
        load_wf<C>(P, ii, jj, kk, w[s], gmv[s]);
      }
      if (d == 0) rho_dev = w[C::SW][0];
      const float *wp[NS], *gp[NS];
#pragma unroll
      for (int s = 0; s < NS; ++s) {
        wp[s] = w[s];
        gp[s] = gmv[s];
      }
      float Flo[NV], Fhi[NV];
      face_flux_split<C>(P, d, i, j, k, wp, gp, Flo);
      face_flux_split<C>(P, d, i + (d == 0), j + (d == 1), k + (d == 2), wp + 1, gp + 1, Fhi);
      const float inv_dl = (float)g.inv_dx[d];
#pragma unroll
      for (int iv = 0; iv < NV; ++iv) {
        float dd = (Fhi[iv] - Flo[iv]) * inv_dl;
        res[iv] = d == 0 ? dd : res[iv] + dd;
      }
    }
    split_cell_update<C>(P, c, i, j, k, res, rho_dev, st);
  }
  split_stat_flush<C>(P, st);
}

// 4-byte asynchronous global -> shared copy (cp.async, completes at the next wait)
__device__ __forceinline__ void cp_async4(float *smem_dst, const float *gmem_src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// Start the copy of the FP32 state of a (possibly ghost) cell into shared memory (variable q at
// dst[q * vs]); returns the velocity components to negate once the copy has landed (bit d for
// a mirrored dimension d, as load_wf does).
template <class C>
__device__ __forceinline__ void load_wf_async(const Prm &P, int i, int j, int k, float *dst, int vs) {
  const Geo &g = P.g;
  bool f0 = false, f1 = false, f2 = false;
  int si = map_index(i, g.nx[0], g.bc[0][0], g.bc[0][1], f0);
  int sj = map_index(j, g.nx[1], g.bc[1][0], g.bc[1][1], f1);
  int sk = map_index(k, g.nx[2], g.bc[2][0], g.bc[2][1], f2);
  long long c = lin(g, si, sj, sk);
#pragma unroll
  for (int iv = 0; iv < C::NV; ++iv) cp_async4(dst + iv * vs, P.Wf_in + (long long)iv * g.N + c);
  if (C::HELM) {
    cp_async4(dst + C::NV * vs, P.gf_in + c);
    cp_async4(dst + (C::NV + 1) * vs, P.gf_in + g.N + c);
  }
}
// after the copy of cell (i, j, k) has landed: negate the velocity components of its mirrored
// dimensions (what load_wf does on load)
__device__ __forceinline__ void fix_mirrored(const Geo &g, int i, int j, int k, float *dst, int vs) {
  bool f[3] = {false, false, false};
  map_index(i, g.nx[0], g.bc[0][0], g.bc[0][1], f[0]);
  map_index(j, g.nx[1], g.bc[1][0], g.bc[1][1], f[1]);
  map_index(k, g.nx[2], g.bc[2][0], g.bc[2][1], f[2]);
#pragma unroll
  for (int d = 0; d < 3; ++d)
    if (f[d]) dst[(1 + d) * vs] = -dst[(1 + d) * vs];
}

// 3D, face reuse: a block owns TX x TY columns of cells in (x1, x2) and marches KZ planes along
// x3.  Deviation states live in a shared-memory ring of five planes (k-1 .. k+3), each with a
// 2-cell halo in x1 and x2, filled by asynchronous copies one plane ahead of use.  Each x1 and
// x2 face of plane k is solved once into shared memory and each x3 face once per column (the
// upper face of plane k is the lower face of plane k+1, kept in registers): 3.16 solves per cell
// against 6 in k_stage_split.  The divergence sums the three directions in the same order as
// k_stage_split.  Requires nx1 % TX == nx2 % TY == nx3 % KZ == 0, blockDim.x == TX * TY and
// SplitTile<C, TX, TY>::bytes() of dynamic shared memory.
template <class C, int TX, int TY>
struct SplitTile {
  static constexpr int NQ = C::NV + (C::HELM ? 2 : 0);  // stored values per cell
  // plane rows are TX + 8 wide with the tile at x offset XO = 4: a tensor copy of the plane
  // starts at x = i0 - 4, a multiple of 4 floats (16 bytes) as bulk tensor copies require;
  // the faces read x offsets 2 .. TX + 5
  static constexpr int XO = 4, SX = TX + 8, SY = TY + 4, PL = SX * SY;
  static constexpr int NSLOT = 5;
  static constexpr int RING = NSLOT * NQ * PL;           // floats: [slot][q][y][x]
  static constexpr int FX = C::NV * TY * (TX + 1), FY = C::NV * (TY + 1) * TX;
  static constexpr int PLANE_BYTES = NQ * PL * 4;        // one staged plane, all fields
  static_assert(PLANE_BYTES % 128 == 0, "slots stay 128-byte aligned");
  static constexpr size_t MBAR_OFFSET = sizeof(float) * (size_t)(RING + FX + FY);  // 8-byte aligned
  static constexpr size_t bytes() { return MBAR_OFFSET + 8 * NSLOT; }
};

// Tensor maps of the stage's FP32 input for the bulk tensor copies: W' as a 4D tensor
// (x1, x2, x3, variable) and the two FASTEOS gammas likewise; box = one plane of the tile with
// its halo, all variables.
struct SplitMaps {
  CUtensorMap w, g;
};
constexpr int SPLIT_TMA_POLLS = 1 << 22;  // mbarrier polls before a stalled copy is reported

template <class C, int TX, int TY, int KZ>
__global__ void __launch_bounds__(TX * TY, 2) k_stage_split_tiled(Prm P, const __grid_constant__ SplitMaps maps,
                                                                  int use_tma) {
  if (!*P.active) return;
  using T = SplitTile<C, TX, TY>;
  constexpr int NV = C::NV, NQ = T::NQ, SX = T::SX, PL = T::PL, VS = PL, XO = T::XO;
  static_assert(C::DIM == 3, "tiled stage is 3D");
  constexpr int NHALO = 4 * TX + 4 * TY;  // halo cells the x1 and x2 faces read (no corners)
  static_assert(NHALO <= TX * TY, "one halo cell per thread");
  extern __shared__ __align__(128) float smem[];
  float *ring = smem;                      // [5][NQ][SY][SX]
  float *fx = smem + T::RING;              // [NV][TY][TX+1]
  float *fy = fx + T::FX;                  // [NV][TY+1][TX]
  uint64_t *mbar = reinterpret_cast<uint64_t *>(reinterpret_cast<unsigned char *>(smem) + T::MBAR_OFFSET);
  const Geo &g = P.g;
  const int tx = threadIdx.x % TX, ty = threadIdx.x / TX;
  const int i0 = blockIdx.x * TX, j0 = blockIdx.y * TY, k0 = blockIdx.z * KZ;
  const int i = i0 + tx, j = j0 + ty;
  const float idx = (float)g.inv_dx[0], idy = (float)g.inv_dx[1], idz = (float)g.inv_dx[2];
  const int own = (ty + 2) * SX + (tx + XO);  // own cell inside a plane
  auto slot = [&](int k) { return ((k - k0 + 2) % T::NSLOT) * NQ * PL; };
  SplitStat st;
  // Interior tiles (the plane with its halo lies inside the domain in x1 and x2, x3 periodic)
  // stage whole planes with bulk tensor copies; the others copy cell by cell with cp.async,
  // mapping ghost indices and mirroring velocities.
  const bool tma = use_tma && blockIdx.x >= 1 && blockIdx.x + 2 <= gridDim.x && blockIdx.y >= 1 &&
                   blockIdx.y + 2 <= gridDim.y;
  auto plane_copy = [&](int k) {
    // one thread: arm the slot's barrier and copy plane k (x3 wrapped) with all variables
    const int s = (k - k0 + 2) % T::NSLOT;
    int kz = k % g.nx[2];
    if (kz < 0) kz += g.nx[2];
    mbar_arrive_expect_tx(mbar + s, T::PLANE_BYTES);
    tma_load_4d(ring + s * NQ * PL, &maps.w, mbar + s, i0 - XO, j0 - 2, kz, 0);
    if (NQ > NV) tma_load_4d(ring + s * NQ * PL + NV * PL, &maps.g, mbar + s, i0 - XO, j0 - 2, kz, 0);
  };
  auto plane_wait = [&](int k) {
    // all threads: the n-th use of a slot completes phase n
    const int u = k - k0 + 2, s = u % T::NSLOT;
    if (!mbar_wait_bounded(mbar + s, (uint32_t)((u / T::NSLOT) & 1), SPLIT_TMA_POLLS) && threadIdx.x == 0)
      atomicAdd(P.stat + STAT_TC_STALLED, 1ull);
  };
  // this thread's halo cell (x1/x2 halo of every plane) for the cell-by-cell path, if any
  int hcell = -1, hx = 0, hy = 0;
  if ((int)threadIdx.x < NHALO) {
    const int h = threadIdx.x;
    if (h < 4 * TX) {
      const int r = h / TX;
      hx = XO + h % TX;
      hy = r < 2 ? r : TY + r;
    } else {
      const int h3 = h - 4 * TX, cc = h3 / TY;
      hy = 2 + h3 % TY;
      hx = cc < 2 ? XO - 2 + cc : XO + TX + cc - 2;
    }
    hcell = hy * SX + hx;
  }
  if (tma) {
    if (threadIdx.x < T::NSLOT) mbar_init(mbar + threadIdx.x, 1);
    __syncthreads();
    if (threadIdx.x == 0)
      for (int k = k0 - 2; k <= k0 + 2; ++k) plane_copy(k);
    for (int k = k0 - 2; k <= k0 + 2; ++k) plane_wait(k);
  } else {
    // prologue: planes k0-2 .. k0+2 of the own column, halo of plane k0
    for (int k = k0 - 2; k <= k0 + 2; ++k) load_wf_async<C>(P, i, j, k, ring + slot(k) + own, VS);
    if (hcell >= 0) load_wf_async<C>(P, i0 + hx - XO, j0 + hy - 2, k0, ring + slot(k0) + hcell, VS);
    cp_async_commit();
    cp_async_wait_all();
    for (int k = k0 - 2; k <= k0 + 2; ++k) fix_mirrored(g, i, j, k, ring + slot(k) + own, VS);
    if (hcell >= 0) fix_mirrored(g, i0 + hx - XO, j0 + hy - 2, k0, ring + slot(k0) + hcell, VS);
  }
  __syncthreads();
  float fz_lo[NV], fz_hi[NV];
  {
    SmemCells<NV> cl{ring, {slot(k0 - 2) + own, slot(k0 - 1) + own, slot(k0) + own, slot(k0 + 1) + own}, VS};
    face_flux_cells<C>(P, 2, i, j, k0, cl, fz_lo);
  }

#pragma unroll 1
  for (int kk = 0; kk < KZ; ++kk) {
    const int k = k0 + kk;
    const int sk = slot(k);
    // next copies: plane k+3 (tensor copy of the whole plane, or the own column) and the halo
    // of plane k+1 (cell-by-cell path); neither is read during this plane
    const bool next_own = kk + 3 <= KZ + 1, next_halo = !tma && kk + 1 < KZ && hcell >= 0;
    if (tma) {
      if (next_own && threadIdx.x == 0) plane_copy(k + 3);
    } else {
      if (next_own) load_wf_async<C>(P, i, j, k + 3, ring + slot(k + 3) + own, VS);
      if (next_halo) load_wf_async<C>(P, i0 + hx - XO, j0 + hy - 2, k + 1, ring + slot(k + 1) + hcell, VS);
      cp_async_commit();
    }
    {
      float F[NV];
      // low x1 face of the own cell
      SmemCells<NV> cx{ring, {sk + own - 2, sk + own - 1, sk + own, sk + own + 1}, VS};
      face_flux_cells<C>(P, 0, i, j, k, cx, F);
#pragma unroll
      for (int q = 0; q < NV; ++q) fx[(q * TY + ty) * (TX + 1) + tx] = F[q];
      // low x2 face of the own cell
      SmemCells<NV> cy{ring, {sk + own - 2 * SX, sk + own - SX, sk + own, sk + own + SX}, VS};
      face_flux_cells<C>(P, 1, i, j, k, cy, F);
#pragma unroll
      for (int q = 0; q < NV; ++q) fy[(q * (TY + 1) + ty) * TX + tx] = F[q];
      if (ty == 0) {
        // upper x2 face of the tile, column tx
        const int c = (TY + 2) * SX + tx + XO;
        SmemCells<NV> cu{ring, {sk + c - 2 * SX, sk + c - SX, sk + c, sk + c + SX}, VS};
        face_flux_cells<C>(P, 1, i, j0 + TY, k, cu, F);
#pragma unroll
        for (int q = 0; q < NV; ++q) fy[(q * (TY + 1) + TY) * TX + tx] = F[q];
      } else if (ty == 1 && tx < TY) {
        // upper x1 face of the tile, row tx
        const int c = (tx + 2) * SX + TX + XO;
        SmemCells<NV> cr{ring, {sk + c - 2, sk + c - 1, sk + c, sk + c + 1}, VS};
        face_flux_cells<C>(P, 0, i0 + TX, j0 + tx, k, cr, F);
#pragma unroll
        for (int q = 0; q < NV; ++q) fx[(q * TY + tx) * (TX + 1) + TX] = F[q];
      }
      // upper x3 face of the own cell
      SmemCells<NV> cz{ring, {slot(k - 1) + own, sk + own, slot(k + 1) + own, slot(k + 2) + own}, VS};
      face_flux_cells<C>(P, 2, i, j, k + 1, cz, fz_hi);
    }
    __syncthreads();
    float res[NV];
#pragma unroll
    for (int q = 0; q < NV; ++q) {
      float dd = (fx[(q * TY + ty) * (TX + 1) + tx + 1] - fx[(q * TY + ty) * (TX + 1) + tx]) * idx;
      dd = dd + (fy[(q * (TY + 1) + ty + 1) * TX + tx] - fy[(q * (TY + 1) + ty) * TX + tx]) * idy;
      res[q] = dd + (fz_hi[q] - fz_lo[q]) * idz;
      fz_lo[q] = fz_hi[q];
    }
    split_cell_update<C>(P, lin(g, i, j, k), i, j, k, res, ring[sk + own], st);
    if (tma) {
      if (next_own) plane_wait(k + 3);
    } else {
      cp_async_wait_all();
      if (next_own) fix_mirrored(g, i, j, k + 3, ring + slot(k + 3) + own, VS);
      if (next_halo) fix_mirrored(g, i0 + hx - XO, j0 + hy - 2, k + 1, ring + slot(k + 1) + hcell, VS);
    }
    __syncthreads();
  }
  split_stat_flush<C>(P, st);
}

// --------------------------------------------------------------------- shock detector (split)
// USE_SHOCK_FLATTENING on the split state (source.F90:8073-8136): the full pressure of a
// (possibly ghost) cell is its FP32 deviation in physical units plus the equilibrium stored
// for that ghost cell; marks go to P.sf_mark, and k_sf_flag forms is_flattened as in FP64
template <class C>
__device__ __forceinline__ double sf_pressure_split(const Prm &P, int i, int j, int k) {
  const Geo &g = P.g;
  bool f = false;
  int si = map_index(i, g.nx[0], g.bc[0][0], g.bc[0][1], f);
  int sj = map_index(j, g.nx[1], g.bc[1][0], g.bc[1][1], f);
  int sk = C::DIM == 3 ? map_index(k, g.nx[2], g.bc[2][0], g.bc[2][1], f) : 0;
  double p = (double)__ldg(P.Wf_in + (long long)C::IP * g.N + lin(g, si, sj, sk)) * P.p_ref;
  if (C::WB) {
    const int G = P.sf_G, G3 = C::DIM == 3 ? P.sf_G : 0;
    long long e = P.sf_eq_profile ? (long long)(j + G)
                                  : (long long)(i + G) + (long long)(g.nx[0] + 2 * G) *
                                        ((long long)(j + G) + (long long)(g.nx[1] + 2 * G) * (k + G3));
    p = p + __ldg(P.sf_eq_p + e);
  }
  return p;
}

template <class C>
__global__ void __launch_bounds__(256) k_sf_mark_split(Prm P) {
  if (!*P.active) return;
  const Geo &g = P.g;
  const long long n = sf_mark_cells<C>(g);
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int m0 = g.nx[0] + 4, m1 = g.nx[1] + 4;
  int i, j, k;
  unflatten3(t, m0, m1, i, j, k);
  i -= 2;
  j -= 2;
  k = C::DIM == 3 ? k - 2 : 0;
  double tmp;
  if (C::DIM == 3)
    tmp = (fabs(sf_pressure_split<C>(P, i, j, k + 1) - sf_pressure_split<C>(P, i, j, k - 1)) +
           fabs(sf_pressure_split<C>(P, i, j + 1, k) - sf_pressure_split<C>(P, i, j - 1, k)) +
           fabs(sf_pressure_split<C>(P, i + 1, j, k) - sf_pressure_split<C>(P, i - 1, j, k))) /
          sf_pressure_split<C>(P, i, j, k);
  else
    tmp = (fabs(sf_pressure_split<C>(P, i, j + 1, k) - sf_pressure_split<C>(P, i, j - 1, k)) +
           fabs(sf_pressure_split<C>(P, i + 1, j, k) - sf_pressure_split<C>(P, i - 1, j, k))) /
          sf_pressure_split<C>(P, i, j, k);
  P.sf_mark[t] = tmp > P.eps_sf ? 1 : 0;
}

// --------------------------------------------------------------------- split MHD
// Cell-centred B of a (possibly ghost) cell in units of b_ref, component d negated for each
// mirrored dimension d.
template <class C>
__device__ __forceinline__ void load_bccf(const Prm &P, int i, int j, int k, float b[3]) {
  const Geo &g = P.g;
  bool f0 = false, f1 = false, f2 = false;
  int si = map_index(i, g.nx[0], g.bc[0][0], g.bc[0][1], f0);
  int sj = map_index(j, g.nx[1], g.bc[1][0], g.bc[1][1], f1);
  int sk = C::DIM == 3 ? map_index(k, g.nx[2], g.bc[2][0], g.bc[2][1], f2) : 0;
  long long c = lin(g, si, sj, sk);
  b[0] = __ldg(P.bccf + c);
  b[1] = __ldg(P.bccf + g.N + c);
  b[2] = C::DIM == 3 ? __ldg(P.bccf + 2 * g.N + c) : 0.0f;
  if (f0) b[0] = -b[0];
  if (f1) b[1] = -b[1];
  if (C::DIM == 3 && f2) b[2] = -b[2];
}

template <class C>
__device__ __forceinline__ void load_bccf_at(const Prm &P, long long c, float b[3]) {
  b[0] = __ldg(P.bccf + c);
  b[1] = __ldg(P.bccf + P.g.N + c);
  b[2] = C::DIM == 3 ? __ldg(P.bccf + 2 * P.g.N + c) : 0.0f;
}

// Riemann part of an MHD face along d (face index fidx, background index fbg): the edge states
// in the cell frame (qL/qR in the order of the FP32 state, transverse B in bL/bR; FASTEOS gammas
// gL/gR with the equilibrium gamma_e already added, or the face temperature guess tface of the
// Helmholtz configurations without FASTEOS) are rotated to the normal frame, the WB background
// and the face-normal B are added, and the flux and the induction flux Fb come back in the cell
// frame with rho_L + rho_R for the CT upwinding sign (source.F90:8138-9105 with the MHD parts
// 8327-8469, 8926-8959)
template <class C>
__device__ __forceinline__ void face_solve_split_mhd(const Prm &P, int d, long long fidx, long long fbg, float qL[C::NV],
                                                     float qR[C::NV], float bL[3], float bR[3], const float gLin[2],
                                                     const float gRin[2], float tface, bool flat, float F[C::NV],
                                                     float Fb[3], float &rho_sum) {
  constexpr int NV = C::NV, IP = C::IP;
  const Geo &g = P.g;
  const float bn = (float)(P.bf[d][fidx] * P.inv_b_ref);
  bL[d] = bn;
  bR[d] = bn;
  if (d == 1) {
    float a = qL[1], c = qL[2]; qL[1] = c; qL[2] = -a;
    a = qR[1]; c = qR[2]; qR[1] = c; qR[2] = -a;
    a = bL[0]; c = bL[1]; bL[0] = c; bL[1] = -a;
    a = bR[0]; c = bR[1]; bR[0] = c; bR[1] = -a;
  } else if (C::DIM == 3 && d == 2) {
    float a = qL[1], c = qL[2], e = qL[3]; qL[1] = e; qL[2] = a; qL[3] = c;
    a = qR[1]; c = qR[2]; e = qR[3]; qR[1] = e; qR[2] = a; qR[3] = c;
    a = bL[0]; c = bL[1]; e = bL[2]; bL[0] = e; bL[1] = a; bL[2] = c;
    a = bR[0]; c = bR[1]; e = bR[2]; bR[0] = e; bR[1] = a; bR[2] = c;
  }
  float pe = 0.0f;
  if (C::WB) {
    float rho_eq = __ldg(P.sf_rho_f[d] + fbg);
    qL[0] = rho_eq + qL[0];
    qR[0] = rho_eq + qR[0];
    pe = __ldg(P.sf_p_f[d] + fbg);
  }
  float gL[2] = {gLin[0], gLin[1]}, gR[2] = {gRin[0], gRin[1]};
  if (!C::FAST && C::HELM) {
    split_side_eos<C>(P, qL, pe, tface, gL[0], gL[1]);
    split_side_eos<C>(P, qR, pe, tface, gR[0], gR[1]);
  }
  riemann_mhd_split<C::DIM, NV, C::EOSM, C::RIEM>(qL, qR, bL, bR, gL, gR, pe, (float)g.gm, (float)g.mach_cutoff, F,
                                                   Fb, flat, g.all_mach != 0);
  if (d == 1) {
    float a = F[1], c = F[2]; F[1] = -c; F[2] = a;
    a = Fb[0]; c = Fb[1]; Fb[0] = -c; Fb[1] = a;
  } else if (C::DIM == 3 && d == 2) {
    float a = F[1], c = F[2], e = F[3]; F[1] = c; F[2] = e; F[3] = a;
    a = Fb[0]; c = Fb[1]; e = Fb[2]; Fb[0] = c; Fb[1] = e; Fb[2] = a;
  }
  rho_sum = qL[0] + qR[0];
  if (C::ETOT) F[IP] = F[IP] + F[0] * __ldg(P.sf_phi_f[d] + fbg);
}

// MHD flux through the low face of cell m along d from cells m-SW..m+SW-1 (w, gm, b: cells
// m-3..m+2); reconstruction, then face_solve_split_mhd
template <class C>
__device__ __forceinline__ void face_flux_split_mhd(const Prm &P, int d, int fi, int fj, int fk, const float *const w[6],
                                                    const float *const gm[6], const float *const b[6], float F[C::NV],
                                                    float Fb[3], float &rho_sum) {
  constexpr int NV = C::NV;
  const Geo &g = P.g;
  bool fa = false, fb = false;  // USE_SHOCK_FLATTENING: is_flattened of cells m-1 and m
  if (C::SF) {
    fa = P.sf_flag[sf_flag_index<C>(g, fi - (d == 0), fj - (d == 1), fk - (d == 2))] != 0;
    fb = P.sf_flag[sf_flag_index<C>(g, fi, fj, fk)] != 0;
  }
  float qL[NV], qR[NV];
#pragma unroll
  for (int iv = 0; iv < NV; ++iv) {
    const float v[6] = {w[0][iv], w[1][iv], w[2][iv], w[3][iv], w[4][iv], w[5][iv]};
    rec_face_f32<C>(v, C::REC == REC_LIM5TH || iv >= C::IAS, qL[iv], qR[iv]);
    if (C::SF && C::REC != REC_LIM2ND) flatten_face_f32(v, fa, fb, qL[iv], qR[iv]);
  }
  float bL[3] = {0, 0, 0}, bR[3] = {0, 0, 0};
#pragma unroll
  for (int iv = 0; iv < C::DIM; ++iv) {
    if (iv == d) continue;
    const float v[6] = {b[0][iv], b[1][iv], b[2][iv], b[3][iv], b[4][iv], b[5][iv]};
    rec_face_f32<C>(v, C::REC == REC_LIM5TH, bL[iv], bR[iv]);
    if (C::SF && C::REC != REC_LIM2ND) flatten_face_f32(v, fa, fb, bL[iv], bR[iv]);
  }
  long long fbg = 0;
  if (C::WB || C::ETOT) fbg = bg_face(g, d, fi, fj, fk);
  float gL[2] = {0.f, 0.f}, gR[2] = {0.f, 0.f}, tface = 0.0f;
  if (C::FAST) {
    const bool late = C::SF && C::WB && d == 0;
    float gv[2][6];
#pragma unroll
    for (int iv = 0; iv < 2; ++iv) {
#pragma unroll
      for (int q = 0; q < 6; ++q) gv[iv][q] = gm[q][iv];
      rec_face_f32<C>(gv[iv], C::REC == REC_LIM5TH, gL[iv], gR[iv]);
      if (C::SF && C::REC != REC_LIM2ND && !late) flatten_face_f32(gv[iv], fa, fb, gL[iv], gR[iv]);
    }
    if (C::WB) {
      float ge = __ldg(P.sf_ge_f[d] + fbg);
      gL[0] = gL[0] + ge;
      gR[0] = gR[0] + ge;
      if (late) flatten_gamma_x1(gv, fa, fb, ge, gL, gR);
    }
  } else if (C::HELM) {
    tface = 0.5f * (gm[2][0] + gm[3][0]);
  }
  face_solve_split_mhd<C>(P, d, face_lin(g, d, fi, fj, fk), fbg, qL, qR, bL, bR, gL, gR, tface, C::SF && (fa || fb), F,
                          Fb, rho_sum);
}

// FP32 face EMF components (units v_ref b_ref) and the CT mass-flux sign (source.F90:8926-8951)
template <class C>
__device__ __forceinline__ void store_face_emf_split(const Prm &P, int d, long long fidx, int q, const float Fb[3],
                                                     float frho, float rho_sum, float smax_s) {
  const Geo &g = P.g;
  long long nf = nfaces(g, d);
  float *e = P.femf[d];
  if (d == 0) { if (C::DIM == 3) e[1 * nf + fidx] = Fb[2]; e[2 * nf + fidx] = -Fb[1]; }
  if (d == 1) { if (C::DIM == 3) e[0 * nf + fidx] = -Fb[2]; e[2 * nf + fidx] = Fb[0]; }
  if (d == 2) { e[0 * nf + fidx] = Fb[1]; e[1 * nf + fidx] = -Fb[0]; }
  // the reference's dead-band ratio f_rho / (rho_bar smax) in physical units: with f_rho and
  // rho in scaled units it carries one factor v_ref, folded into smax_s = smax / v_ref
  float mach = frho / (0.5f * rho_sum * smax_s), sgn = 0.0f;
  if (mach > (float)g.mach_ct) sgn = 1.0f;
  if (mach < -(float)g.mach_ct) sgn = -1.0f;
  // a reflective wall face has mirror-image states and no mass flux: the reference (no FMA) gets
  // exactly zero there, while FP32 with contracted products leaves a rounding residue whose sign
  // would select an upwind side; the wall's dead-band value is restored explicitly (q is the
  // face's index along d)
  if ((q == 0 && g.bc[d][0] != BC_PERIODIC) || (q == g.nx[d] && g.bc[d][1] != BC_PERIODIC)) sgn = 0.0f;
  P.fsgn[d][fidx] = sgn;
}

// MHD stage, part 1: one thread per face of direction d solves it once: the FP32 flux goes to
// P.fflux[d] ([NV][faces]), the face EMF and the CT sign to their arrays
// (one instantiation per direction D: index strides and rotations fold into constants)
template <class C, int D>
__device__ __forceinline__ void face_split_mhd_at(const Prm &P, long long f) {
  constexpr int d = D;
  constexpr int NV = C::NV;
  const Geo &g = P.g;
  const long long nf = nfaces(g, d);
  const int n0 = g.nx[0] + (d == 0), n1 = g.nx[1] + (d == 1);
  int fi, fj, fk;
  unflatten3(f, n0, n1, fi, fj, fk);
  // cells m-3 .. m+2 (the reconstruction reads m-SW .. m+SW-1); a stencil inside the domain
  // is read by linear index, one at a boundary maps each ghost index
  float w[6][NV], gm4[6][2], b4[6][3];
  const int fd = d == 0 ? fi : (d == 1 ? fj : fk);
  const bool inside = fd >= C::SW && fd + C::SW <= g.nx[d];
  const long long base = lin(g, fi, fj, fk), stride = dir_stride(g, d);
#pragma unroll
  for (int s = 0; s < 6; ++s) {
    gm4[s][0] = gm4[s][1] = 0.0f;
    b4[s][0] = b4[s][1] = b4[s][2] = 0.0f;
    if (s < 3 - C::SW || s >= 3 + C::SW) {
#pragma unroll
      for (int iv = 0; iv < NV; ++iv) w[s][iv] = 0.0f;
      continue;
    }
    if (inside) {
      const long long c = base + (s - 3) * stride;
      load_wf_at<C>(P, c, w[s], gm4[s]);
      load_bccf_at<C>(P, c, b4[s]);
    } else {
      const int ii = fi + (d == 0 ? s - 3 : 0), jj = fj + (d == 1 ? s - 3 : 0), kk = fk + (d == 2 ? s - 3 : 0);
      load_wf<C>(P, ii, jj, kk, w[s], gm4[s]);
      load_bccf<C>(P, ii, jj, kk, b4[s]);
    }
  }
  const float *const wv[6] = {w[0], w[1], w[2], w[3], w[4], w[5]};
  const float *const gv[6] = {gm4[0], gm4[1], gm4[2], gm4[3], gm4[4], gm4[5]};
  const float *const bv[6] = {b4[0], b4[1], b4[2], b4[3], b4[4], b4[5]};
  float F[NV], Fb[3], rs;
  face_flux_split_mhd<C>(P, d, fi, fj, fk, wv, gv, bv, F, Fb, rs);
#pragma unroll
  for (int iv = 0; iv < NV; ++iv) P.fflux[d][(long long)iv * nf + f] = F[iv];
  store_face_emf_split<C>(P, d, f, d == 0 ? fi : (d == 1 ? fj : fk), Fb, F[0], rs, (float)(P.scal[2] * P.inv_v_ref));
}

template <class C, int D>
__global__ void __launch_bounds__(128, C::MINB_FACE32) k_face_split_mhd(Prm P) {
  if (!*P.active) return;
  const long long f = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= nfaces(P.g, D)) return;
  face_split_mhd_at<C, D>(P, f);
}

// faces per thread of the walking face kernels: along x (threads of a warp step K0 cells apart,
// so their loads stay within a few cache lines) and along y, z (threads of a warp are
// neighbours in x and walk side by side)
constexpr int WALK_K0 = 4, WALK_K = 8;
// resident blocks of 128 threads per SM of the EoS half of the two-launch cons->prim
constexpr int C2P_EOS_MINB = 7;
// grid of the rescue-queue kernels: 4 blocks of 128 threads per SM of a B200 (148 SMs)
constexpr int RESCUE_BLOCKS = 4 * 148;
// resident blocks of 128 threads per SM the walking kernels are compiled for (72 registers; the
// 256^3 MHD stage took 4.46 ms at 7 against 4.53 at 6 and 4.50 at 8); without USE_FASTEOS, where
// each face runs two FP64 (rho, P) -> T solves, 4 (128 registers): a 256^3 MHD step took 36.9
// ms against 43.4 with the registers unbounded (253 registers, 2 blocks per SM), 37.5 at 3
constexpr int WALK_MINB = 7, WALK_MINB_GIVEN = 4;

// Raw values of one cell for the walking face kernel along D: the FP32 state (0 .. NV-1), the
// cell B components transverse to D (NBT of them from NV on; the component along D is not
// reconstructed, the face carries it) and the two FASTEOS gammas or the temperature (IG, IG+1).
template <class C, int D>
struct WalkCell {
  static constexpr int NBT = C::DIM - 1, IG = C::NV + NBT, NR = IG + 2;
  // cell B component held in transverse slot t
  static __device__ __forceinline__ constexpr int comp(int t) { return t < D ? t : t + 1; }
};

// q is the cell's index along D and c[] its other two coordinates; a cell inside the domain
// along D is read by linear index lc, a ghost maps its index.
template <class C, int D>
__device__ __forceinline__ void load_walk_cell(const Prm &P, const int c[3], int q, long long lc,
                                               float r[WalkCell<C, D>::NR]) {
  using L = WalkCell<C, D>;
  float *gm = r + L::IG;
  gm[0] = gm[1] = 0.0f;
  if (q >= 0 && q < P.g.nx[D]) {
    load_wf_at<C>(P, lc, r, gm);
#pragma unroll
    for (int t = 0; t < L::NBT; ++t) r[C::NV + t] = __ldg(P.bccf + L::comp(t) * P.g.N + lc);
  } else {
    const int i = D == 0 ? q : c[0], j = D == 1 ? q : c[1], k = D == 2 ? q : c[2];
    float b[3];
    load_wf<C>(P, i, j, k, r, gm);
    load_bccf<C>(P, i, j, k, b);
#pragma unroll
    for (int t = 0; t < L::NBT; ++t) r[C::NV + t] = b[L::comp(t)];
  }
}

// MHD stage, part 1 for LIM2ND reconstruction: one thread walks K consecutive faces along D.  A
// cell borders two faces of the walk, so its values are loaded and its PLM slope formed once
// (the per-face kernel does both twice) and its edge values are carried to the next face.  The
// faces, their arithmetic and the stored results are those of k_face_split_mhd.
template <class C, int D, int K>
__global__ void __launch_bounds__(128, C::EOSM == EOS_GIVEN ? WALK_MINB_GIVEN : WALK_MINB) k_face_split_mhd_walk(Prm P) {
  static_assert(C::REC == REC_LIM2ND, "the walk carries LIM2ND edge values");
  if (!*P.active) return;
  using L = WalkCell<C, D>;
  constexpr int NV = C::NV, NR = L::NR, IG = L::IG;
  const Geo &g = P.g;
  const int nd = g.nx[D] + 1, nch = (nd + K - 1) / K;
  const int e0 = D == 0 ? nch : g.nx[0], e1 = D == 1 ? nch : g.nx[1];
  const int e2 = D == 2 ? nch : (C::DIM == 3 ? g.nx[2] : 1);
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)e0 * e1 * e2) return;
  int c[3];
  unflatten3(t, e0, e1, c[0], c[1], c[2]);
  const int q0 = c[D] * K, qend = min(q0 + K, nd);
  c[D] = 0;
  const long long nf = nfaces(g, D), cstride = dir_stride(g, D);
  const long long fstride = D == 0 ? 1 : (D == 1 ? (long long)g.nx[0] : (long long)g.nx[0] * g.nx[1]);
  const long long crow = lin(g, c[0], c[1], c[2]), frow = face_lin(g, D, c[0], c[1], c[2]);
  const long long sfrow = C::SF ? sf_flag_index<C>(g, c[0], c[1], c[2]) : 0;
  const long long sfstride = D == 0 ? 1 : (D == 1 ? (long long)(g.nx[0] + 2) : (long long)(g.nx[0] + 2) * (g.nx[1] + 2));
  const float smax_s = (float)(P.scal[2] * P.inv_v_ref);
  // window: rm, rc = cells q-1, q; hip = edge values at the high side of cell q-1
  float rm[NR], rc[NR], rp[NR], lo[NR], hi[NR], hip[NR];
  load_walk_cell<C, D>(P, c, q0 - 2, crow + (long long)(q0 - 2) * cstride, rm);
  load_walk_cell<C, D>(P, c, q0 - 1, crow + (long long)(q0 - 1) * cstride, rc);
  load_walk_cell<C, D>(P, c, q0, crow + (long long)q0 * cstride, rp);
#pragma unroll
  for (int v = 0; v < NR; ++v) {
    plm_f32(rm[v], rc[v], rp[v], lo[v], hip[v]);
    rm[v] = rc[v];
    rc[v] = rp[v];
  }
  bool fprev = C::SF && P.sf_flag[sfrow + (long long)(q0 - 1) * sfstride] != 0;
#pragma unroll 1
  for (int q = q0; q < qend; ++q) {
    load_walk_cell<C, D>(P, c, q + 1, crow + (long long)(q + 1) * cstride, rp);
#pragma unroll
    for (int v = 0; v < NR; ++v) plm_f32(rm[v], rc[v], rp[v], lo[v], hi[v]);
    const bool fa = fprev, fb = C::SF && P.sf_flag[sfrow + (long long)q * sfstride] != 0;
    float qL[NV], qR[NV], bL[3] = {0.f, 0.f, 0.f}, bR[3] = {0.f, 0.f, 0.f}, gL[2] = {0.f, 0.f}, gR[2] = {0.f, 0.f};
#pragma unroll
    for (int iv = 0; iv < NV; ++iv) {
      qL[iv] = hip[iv];
      qR[iv] = lo[iv];
    }
#pragma unroll
    for (int t = 0; t < L::NBT; ++t) {
      bL[L::comp(t)] = hip[NV + t];
      bR[L::comp(t)] = lo[NV + t];
    }
    const long long fidx = frow + (long long)q * fstride;
    long long fbg = 0;
    if (C::WB || C::ETOT) fbg = g.bg_profile ? (long long)(D == 1 ? q : c[1]) : fidx;
    float tface = 0.0f;
    if (C::FAST) {
      gL[0] = hip[IG]; gL[1] = hip[IG + 1];
      gR[0] = lo[IG]; gR[1] = lo[IG + 1];
      if (C::WB) {
        const float ge = __ldg(P.sf_ge_f[D] + fbg);
        const float rL[2] = {gL[0], gL[1]}, rR[2] = {gR[0], gR[1]};
        gL[0] = gL[0] + ge;
        gR[0] = gR[0] + ge;
        // the x1 sweep's gamma handling on flagged faces (flatten_gamma_x1 with the LIM2ND
        // edges already at hand)
        if (C::SF && D == 0) {
          if (fa) { gL[0] = rL[0]; gL[1] = rL[1]; gR[0] = gR[0] + ge; }
          if (fb) { gR[0] = rR[0]; gR[1] = rR[1]; gL[0] = gL[0] + ge; }
        }
      }
    } else if (C::HELM) {
      tface = 0.5f * (rm[IG] + rc[IG]);
    }
    float F[NV], Fb[3], rs;
    face_solve_split_mhd<C>(P, D, fidx, fbg, qL, qR, bL, bR, gL, gR, tface, C::SF && (fa || fb), F, Fb, rs);
#pragma unroll
    for (int iv = 0; iv < NV; ++iv) P.fflux[D][(long long)iv * nf + fidx] = F[iv];
    store_face_emf_split<C>(P, D, fidx, q, Fb, F[0], rs, smax_s);
#pragma unroll
    for (int v = 0; v < NR; ++v) {
      hip[v] = hi[v];
      rm[v] = rc[v];
      rc[v] = rp[v];
    }
    fprev = fb;
  }
}

// MHD stage, part 1 for LIM2ND on grids that the direction's face tile divides: faces along D
// from tiles of cells staged in shared memory.  Tile (TX, TY, TZ) cells, one face per thread (the
// face below each cell along D).  Bulk tensor copies (TMA) stage the tile with two extra layers
// on either side along D (x1: four, so that the copy starts on a 16-byte boundary) of W', the
// cell B and the two gamma slots; layers outside the domain arrive zero-filled and the ghost
// layers the stencils need are then written by their threads with the ghost mapping and
// mirroring of load_wf.  Each thread forms the LIM2ND edges of its cell once into shared memory
// (the first TT threads also those of the layer below the tile), then solves its face and stores
// flux, face EMF and CT sign with coalesced stores.  A grid of one resident wave of blocks
// strides over the tiles, each block issuing its next tile's copies once the staged values are
// consumed; the faces at the upper domain boundary along D are solved after the tile loop.
// Faces, arithmetic and the solver are those of the walking kernels, which carry the same edges
// in registers and, along x1, would stride 4 cells per thread.
template <int D> struct FaceTile;
template <> struct FaceTile<0> { static constexpr int TX = 128, TY = 1, TZ = 1, MINB = 8; };
template <> struct FaceTile<1> { static constexpr int TX = 32, TY = 8, TZ = 1, MINB = 4; };
template <> struct FaceTile<2> { static constexpr int TX = 32, TY = 1, TZ = 8, MINB = 4; };

template <class C, int D>
struct FaceTileSmem {
  using T = FaceTile<D>;
  static constexpr int NT = T::TX * T::TY * T::TZ;                  // threads = faces per tile
  static constexpr int TD = D == 0 ? T::TX : (D == 1 ? T::TY : T::TZ);
  static constexpr int TT = NT / TD;                                // columns along D
  static constexpr int OX = D == 0 ? 4 : 0, OY = D == 1 ? 2 : 0, OZ = D == 2 ? 2 : 0;
  static constexpr int SX = T::TX + 2 * OX, SY = T::TY + 2 * OY, SZ = T::TZ + 2 * OZ;
  static constexpr int SC = SX * SY * SZ;                           // staged cells per variable
  static constexpr int SD = D == 0 ? 1 : (D == 1 ? SX : SX * SY);   // staged stride along D
  static constexpr int NE = C::NV + 5;                              // W', B (3), gamma slots (2)
  static constexpr int RW = ((C::NV * SC + 31) / 32) * 32;          // region sizes in floats,
  static constexpr int RB = ((3 * SC + 31) / 32) * 32;              // multiples of 128 bytes
  static constexpr int RG = ((2 * SC + 31) / 32) * 32;
  static constexpr int NEDGE = (TD + 1) * TT;                       // edge slots: layers -1 .. TD-1
  static constexpr bool STAGE_G = C::HELM;                          // gammas (FASTEOS) or T (without)
  static constexpr uint32_t BYTES = 4u * SC * (C::NV + 3 + (STAGE_G ? 2 : 0));
  float w[RW], b[RB], gm[RG];
  float lo[NE * NEDGE], hi[NE * NEDGE];
  uint64_t mbar;
};
struct FaceTileMaps {
  CUtensorMap w, b, g;
};

template <class C, int D>
__global__ void __launch_bounds__(FaceTileSmem<C, D>::NT, FaceTile<D>::MINB)
    k_face_split_mhd_tile(Prm P, const __grid_constant__ FaceTileMaps maps, int ntiles) {
  static_assert(C::REC == REC_LIM2ND && !C::SF, "tiled faces carry LIM2ND edges without flattening");
  if (!*P.active) return;
  using S_ = FaceTileSmem<C, D>;
  using T = FaceTile<D>;
  constexpr int NV = C::NV, NE = S_::NE, NED = S_::NEDGE, TT = S_::TT, SX = S_::SX, SY = S_::SY, SC = S_::SC;
  const Geo &g = P.g;
  const int t = threadIdx.x;
  __shared__ __align__(128) S_ S;
  const int nbx = g.nx[0] / T::TX, nby = g.nx[1] / T::TY;
  const int tx = t % T::TX, ty = (t / T::TX) % T::TY, tz = t / (T::TX * T::TY);
  const int td = D == 0 ? tx : (D == 1 ? ty : tz);
  const int col = D == 0 ? ty + T::TY * tz : (D == 1 ? tx + T::TX * tz : tx + T::TX * ty);  // < TT
  const int nD = g.nx[D];
  // origin of tile `tile`
  auto origin = [&](int tile, int &i0, int &j0, int &k0) {
    i0 = (tile % nbx) * T::TX;
    j0 = ((tile / nbx) % nby) * T::TY;
    k0 = (tile / (nbx * nby)) * T::TZ;
  };
  // one thread: the bulk tensor copies of a tile into the staging area, counted on the mbarrier
  // (the fence orders the generic-proxy reads and writes of the previous tile before the copy)
  auto issue = [&](int tile) {
    int i0, j0, k0;
    origin(tile, i0, j0, k0);
    fence_proxy_async_smem();
    mbar_arrive_expect_tx(&S.mbar, S_::BYTES);
    tma_load_4d(S.w, &maps.w, &S.mbar, i0 - S_::OX, j0 - S_::OY, k0 - S_::OZ, 0);
    tma_load_4d(S.b, &maps.b, &S.mbar, i0 - S_::OX, j0 - S_::OY, k0 - S_::OZ, 0);
    if (S_::STAGE_G) tma_load_4d(S.gm, &maps.g, &S.mbar, i0 - S_::OX, j0 - S_::OY, k0 - S_::OZ, 0);
  };
  // staged position of tile cell (x, y, z) relative to the tile origin
  auto spos = [&](int x, int y, int z) { return (x + S_::OX) + SX * ((y + S_::OY) + SY * (z + S_::OZ)); };
  // tile coordinates of column `cl` at layer `l` along D
  auto cell_of = [&](int cl, int l, int &x, int &y, int &z) {
    if (D == 0) { x = l; y = cl % T::TY; z = cl / T::TY; }
    else if (D == 1) { x = cl % T::TX; y = l; z = cl / T::TX; }
    else { x = cl % T::TX; y = cl / T::TX; z = l; }
  };
  if (t == 0) mbar_init(&S.mbar, 1);
  __syncthreads();
  int tile = blockIdx.x;
  if (t == 0 && tile < ntiles) issue(tile);
  // the block strides over the tiles; each copy is issued as soon as the previous tile's staged
  // values are consumed, so that it lands while that tile's faces are solved
  for (uint32_t it = 0; tile < ntiles; ++it, tile += gridDim.x) {
    int i0, j0, k0;
    origin(tile, i0, j0, k0);
    const int c0 = D == 0 ? i0 : (D == 1 ? j0 : k0);
    const bool landed = mbar_wait_bounded(&S.mbar, it & 1u, SPLIT_TMA_POLLS);
    // ghost layers -2, -1 (tile at the lower domain boundary) and nD, nD + 1 (upper) along D
    if (landed && t < 4 * TT) {
      const int side = t / (2 * TT), layer = (t / TT) % 2, cl = t % TT;
      const int l = side == 0 ? layer - 2 : S_::TD + layer;
      if ((side == 0 && c0 == 0) || (side == 1 && c0 + S_::TD == nD)) {
        int x, y, z;
        cell_of(cl, l, x, y, z);
        float wv[NV], gv[2] = {0.0f, 0.0f}, bv[3];
        load_wf<C>(P, i0 + x, j0 + y, k0 + z, wv, gv);
        load_bccf<C>(P, i0 + x, j0 + y, k0 + z, bv);
        const int pos = spos(x, y, z);
#pragma unroll
        for (int iv = 0; iv < NV; ++iv) S.w[iv * SC + pos] = wv[iv];
#pragma unroll
        for (int a = 0; a < 3; ++a) S.b[a * SC + pos] = bv[a];
        S.gm[pos] = gv[0];
        S.gm[SC + pos] = gv[1];
      }
    }
    if (__syncthreads_or(!landed)) {
      // a copy did not land in time (the whole block learns it at the barrier, so that every
      // thread leaves the loop together): report it, give it a second bounded chance to finish
      // before the block leaves, and leave the remaining tiles of this block (their faces are
      // then not trustworthy; the count says so)
      if (t == 0) atomicAdd(P.stat + STAT_TC_STALLED, 1ull);
      mbar_wait_bounded(&S.mbar, it & 1u, SPLIT_TMA_POLLS);
      break;
    }
    // LIM2ND edges of the cell at layer l of column cl into edge slot (l + 1) * TT + cl
    auto edges = [&](int cl, int l) {
      int x, y, z;
      cell_of(cl, l, x, y, z);
      const int pos = spos(x, y, z), slot = (l + 1) * TT + cl;
#pragma unroll
      for (int v = 0; v < NE; ++v) {
        const float *src = v < NV ? S.w + v * SC : (v < NV + 3 ? S.b + (v - NV) * SC : S.gm + (v - NV - 3) * SC);
        float lo, hi;
        plm_f32(src[pos - S_::SD], src[pos], src[pos + S_::SD], lo, hi);
        S.lo[v * NED + slot] = lo;
        S.hi[v * NED + slot] = hi;
      }
    };
    edges(col, td);
    if (t < TT) edges(t, -1);
    // without FASTEOS the face's temperature guess comes from the staged T, read before the
    // staging area is handed to the next copy
    float tface = 0.0f;
    if (!C::FAST && C::HELM) {
      const int pos = spos(tx, ty, tz);
      tface = 0.5f * (S.gm[pos - S_::SD] + S.gm[pos]);
    }
    __syncthreads();
    // the staged values are consumed: the next tile's copy overlaps this tile's solves
    if (t == 0 && tile + (int)gridDim.x < ntiles) issue(tile + gridDim.x);
    // the face below the own cell along D: edges of layers td - 1 (slot td * TT + col) and td
    const int sL = td * TT + col, sR = sL + TT;
    float qL[NV], qR[NV], bL[3] = {0.f, 0.f, 0.f}, bR[3] = {0.f, 0.f, 0.f}, gL[2] = {0.f, 0.f}, gR[2] = {0.f, 0.f};
#pragma unroll
    for (int iv = 0; iv < NV; ++iv) {
      qL[iv] = S.hi[iv * NED + sL];
      qR[iv] = S.lo[iv * NED + sR];
    }
#pragma unroll
    for (int a = 0; a < C::DIM; ++a) {
      if (a == D) continue;
      bL[a] = S.hi[(NV + a) * NED + sL];
      bR[a] = S.lo[(NV + a) * NED + sR];
    }
    const int fi = i0 + tx, fj = j0 + ty, fk = k0 + tz;
    const long long fidx = face_lin(g, D, fi, fj, fk);
    long long fbg = 0;
    if (C::WB || C::ETOT) fbg = g.bg_profile ? (long long)fj : fidx;
    if (C::FAST) {
      gL[0] = S.hi[(NV + 3) * NED + sL]; gL[1] = S.hi[(NV + 4) * NED + sL];
      gR[0] = S.lo[(NV + 3) * NED + sR]; gR[1] = S.lo[(NV + 4) * NED + sR];
      if (C::WB) {
        const float ge = __ldg(P.sf_ge_f[D] + fbg);
        gL[0] = gL[0] + ge;
        gR[0] = gR[0] + ge;
      }
    }
    float F[NV], Fb[3], rs;
    face_solve_split_mhd<C>(P, D, fidx, fbg, qL, qR, bL, bR, gL, gR, tface, false, F, Fb, rs);
    const long long nf = nfaces(g, D);
#pragma unroll
    for (int iv = 0; iv < NV; ++iv) P.fflux[D][(long long)iv * nf + fidx] = F[iv];
    store_face_emf_split<C>(P, D, fidx, c0 + td, Fb, F[0], rs, (float)(P.scal[2] * P.inv_v_ref));
  }
  // the faces at the upper domain boundary along D, one per thread, strided over the grid
  const int e0 = D == 0 ? g.nx[1] : g.nx[0], e1 = D == 2 ? g.nx[1] : (C::DIM == 3 ? g.nx[2] : 1);
  for (long long q = (long long)blockIdx.x * S_::NT + t; q < (long long)e0 * e1; q += (long long)gridDim.x * S_::NT) {
    const int a = (int)(q % e0), c = (int)(q / e0);
    const int fi = D == 0 ? g.nx[0] : a, fj = D == 0 ? a : (D == 1 ? g.nx[1] : c), fk = D == 2 ? g.nx[2] : c;
    face_split_mhd_at<C, D>(P, face_lin(g, D, fi, fj, fk));
  }
}

// FP32 face EMF / sign at a possibly-ghost transverse index (periodic wrap, or the reflective
// EMF BC: the wall-normal component keeps its sign, the others flip; source.F90:11374-11964)
template <class C>
__device__ __forceinline__ void face_emf_split_at(const Prm &P, int d, int comp, int i, int j, int k, float &e,
                                                  float &sgn) {
  const Geo &g = P.g;
  int c[3] = {i, j, k};
  float fac = 1.0f;
#pragma unroll
  for (int d2 = 0; d2 < C::DIM; ++d2) {
    if (d2 == d) continue;
    int n = g.nx[d2];
    if (c[d2] < 0) {
      if (g.bc[d2][0] == BC_PERIODIC) c[d2] += n;
      else { c[d2] = 0; if (comp != d2) fac = -fac; }
    } else if (c[d2] >= n) {
      if (g.bc[d2][1] == BC_PERIODIC) c[d2] -= n;
      else { c[d2] = n - 1; if (comp != d2) fac = -fac; }
    }
  }
  long long f = face_lin(g, d, c[0], c[1], c[2]);
  e = fac * P.femf[d][(long long)comp * nfaces(g, d) + f];
  sgn = P.fsgn[d][f];
}

// cell-centred -v x B (components 0..2) of FP32 velocity v and cell B b (scaled units)
__device__ __forceinline__ void cell_emf3(const float v[3], const float b[3], float e[3]) {
  e[2] = -v[0] * b[1] + v[1] * b[0];
  e[0] = v[2] * b[1] - v[1] * b[2];
  e[1] = v[0] * b[2] - v[2] * b[0];
}
// the stage input's cell EMFs, written by the kernel that produced its FP32 state
__device__ __forceinline__ void store_cell_emf(const Prm &P, long long c, const float v[3], const float b[3]) {
  float e[3];
  cell_emf3(v, b, e);
#pragma unroll
  for (int a = 0; a < 3; ++a) P.fecell[(long long)a * P.g.N + c] = e[a];
}

// cell-centred -v x B component a of a (possibly ghost) cell from the stored cell EMFs: a mirror
// in dimension d != a flips one factor of each product of component a
template <class C>
__device__ __forceinline__ float emf_cell_split(const Prm &P, int a, int i, int j, int k) {
  const Geo &g = P.g;
  bool f0 = false, f1 = false, f2 = false;
  int si = map_index(i, g.nx[0], g.bc[0][0], g.bc[0][1], f0);
  int sj = map_index(j, g.nx[1], g.bc[1][0], g.bc[1][1], f1);
  int sk = C::DIM == 3 ? map_index(k, g.nx[2], g.bc[2][0], g.bc[2][1], f2) : 0;
  float e = __ldg(P.fecell + (long long)a * g.N + lin(g, si, sj, sk));
  const bool flip = (a != 0 && f0) != ((a != 1 && f1) != (a != 2 && f2));
  return flip ? -e : e;
}

// corner EMF along axis A (source.F90:11966-12206), FP32, at corner (c[0], c[1], c[2]); INTERIOR:
// all four faces and cells lie inside the domain (linear indices, no wrap or mirror)
template <class C, int A, bool INTERIOR>
__device__ __forceinline__ float corner_emf_split(const Prm &P, const int c[3]) {
  constexpr int a = A, pa = A == 2 ? 0 : (A == 0 ? 1 : 2), qa = A == 2 ? 1 : (A == 0 ? 2 : 0);
  const Geo &g = P.g;
  float emf_N, emf_E, emf_S, emf_W, sgS, sgN, sgW, sgE, emf_SW, emf_NW, emf_NE, emf_SE;
  if (INTERIOR) {
    const long long fp = face_lin(g, pa, c[0], c[1], c[2]), fq = face_lin(g, qa, c[0], c[1], c[2]);
    const int p0 = g.nx[0] + (pa == 0), p1 = g.nx[1] + (pa == 1);  // face array of pa
    const int q0 = g.nx[0] + (qa == 0), q1 = g.nx[1] + (qa == 1);  // face array of qa
    const long long sp_q = qa == 0 ? 1 : (qa == 1 ? (long long)p0 : (long long)p0 * p1);  // step along qa
    const long long sq_p = pa == 0 ? 1 : (pa == 1 ? (long long)q0 : (long long)q0 * q1);  // step along pa
    const float *ep = P.femf[pa] + (long long)a * nfaces(g, pa), *eq = P.femf[qa] + (long long)a * nfaces(g, qa);
    emf_N = __ldg(ep + fp); sgN = __ldg(P.fsgn[pa] + fp);
    emf_S = __ldg(ep + fp - sp_q); sgS = __ldg(P.fsgn[pa] + fp - sp_q);
    emf_E = __ldg(eq + fq); sgE = __ldg(P.fsgn[qa] + fq);
    emf_W = __ldg(eq + fq - sq_p); sgW = __ldg(P.fsgn[qa] + fq - sq_p);
    const long long cc = lin(g, c[0], c[1], c[2]);
    const long long cp = pa == 0 ? 1 : (pa == 1 ? (long long)g.nx[0] : (long long)g.nx[0] * g.nx[1]);
    const long long cq = qa == 0 ? 1 : (qa == 1 ? (long long)g.nx[0] : (long long)g.nx[0] * g.nx[1]);
    const float *ec = P.fecell + (long long)a * g.N;
    emf_NE = __ldg(ec + cc);
    emf_NW = __ldg(ec + cc - cp);
    emf_SE = __ldg(ec + cc - cq);
    emf_SW = __ldg(ec + cc - cp - cq);
  } else {
    int cqm[3] = {c[0], c[1], c[2]}; cqm[qa] -= 1;
    int cpm[3] = {c[0], c[1], c[2]}; cpm[pa] -= 1;
    int cpq[3] = {c[0], c[1], c[2]}; cpq[pa] -= 1; cpq[qa] -= 1;
    face_emf_split_at<C>(P, pa, a, c[0], c[1], c[2], emf_N, sgN);
    face_emf_split_at<C>(P, qa, a, c[0], c[1], c[2], emf_E, sgE);
    face_emf_split_at<C>(P, pa, a, cqm[0], cqm[1], cqm[2], emf_S, sgS);
    face_emf_split_at<C>(P, qa, a, cpm[0], cpm[1], cpm[2], emf_W, sgW);
    emf_SW = emf_cell_split<C>(P, a, cpq[0], cpq[1], cpq[2]);
    emf_NW = emf_cell_split<C>(P, a, cpm[0], cpm[1], cpm[2]);
    emf_NE = emf_cell_split<C>(P, a, c[0], c[1], c[2]);
    emf_SE = emf_cell_split<C>(P, a, cqm[0], cqm[1], cqm[2]);
  }
  float sgn = sgS;
  float demf_S = 0.5f * (1.0f + sgn) * (emf_W - emf_SW) + 0.5f * (1.0f - sgn) * (emf_E - emf_SE);
  sgn = sgN;
  float demf_N = 0.5f * (1.0f + sgn) * (emf_NW - emf_W) + 0.5f * (1.0f - sgn) * (emf_NE - emf_E);
  sgn = sgW;
  float demf_W = 0.5f * (1.0f + sgn) * (emf_S - emf_SW) + 0.5f * (1.0f - sgn) * (emf_N - emf_NW);
  sgn = sgE;
  float demf_E = 0.5f * (1.0f + sgn) * (emf_SE - emf_S) + 0.5f * (1.0f - sgn) * (emf_NE - emf_N);
  return 0.25f * (emf_S + emf_W + emf_N + emf_E + demf_S - demf_N + demf_W - demf_E);
}

// Corner EMFs along axis A, one thread per corner (one instantiation per axis: the face and cell
// strides fold into constants).  The first nin_blocks blocks take the interior corners (1 <=
// c[pa] < nx[pa], 1 <= c[qa] < nx[qa]), which read their faces and cells by linear index with no
// branch; the blocks after them take the corners on the domain faces of pa and qa, which map
// their ghost indices.  Threads over all corners in array order had a quarter of their warps
// diverge into the mapping path, where the rows of corners (nx + 1 long) straddle the warps.
template <class C, int A>
__global__ void __launch_bounds__(256) k_corner_split(Prm P, unsigned nin_blocks) {
  constexpr int a = A, pa = A == 2 ? 0 : (A == 0 ? 1 : 2), qa = A == 2 ? 1 : (A == 0 ? 2 : 0);
  if (!*P.active) return;
  const Geo &g = P.g;
  int c[3];
  if (blockIdx.x < nin_blocks) {
    // interior extents per dimension (x1 fastest, as the arrays): nx - 1 from index 1 along pa
    // and qa, nx from index 0 along a
    const int e0 = a == 0 ? g.nx[0] : g.nx[0] - 1, e1 = a == 1 ? g.nx[1] : g.nx[1] - 1;
    const int e2 = C::DIM == 3 ? (a == 2 ? g.nx[2] : g.nx[2] - 1) : 1;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)e0 * e1 * e2) return;
    unflatten3(t, e0, e1, c[0], c[1], c[2]);
    c[0] += a != 0;
    c[1] += a != 1;
    if (C::DIM == 3) c[2] += a != 2;
    P.fcor[a][cor_lin(g, a, c[0], c[1], c[2])] = corner_emf_split<C, A, true>(P, c);
    return;
  }
  // the rim: per index along a, the border of the (nx[pa] + 1) x (nx[qa] + 1) rectangle of
  // corners, 2 (nx[pa] + nx[qa]) of them
  const int np_ = g.nx[pa], nq = g.nx[qa], na = C::DIM == 3 ? g.nx[a] : 1, rim = 2 * (np_ + nq);
  const long long t = (long long)(blockIdx.x - nin_blocks) * blockDim.x + threadIdx.x;
  if (t >= (long long)rim * na) return;
  const int m = (int)(t % rim);
  c[a] = (int)(t / rim);
  if (m < np_ + 1) { c[pa] = m; c[qa] = 0; }                             // qa = 0 row
  else if (m < 2 * (np_ + 1)) { c[pa] = m - (np_ + 1); c[qa] = nq; }       // qa = nx[qa] row
  else if (m < 2 * (np_ + 1) + (nq - 1)) { c[pa] = 0; c[qa] = m - 2 * (np_ + 1) + 1; }  // pa = 0 column
  else { c[pa] = np_; c[qa] = m - 2 * (np_ + 1) - (nq - 1) + 1; }         // pa = nx[pa] column
  P.fcor[a][cor_lin(g, a, c[0], c[1], c[2])] = corner_emf_split<C, A, false>(P, c);
}

// face-B update (source.F90:12208-12437) in FP64 from the FP32 corner EMFs; one thread per face
template <class C, int D>
__global__ void __launch_bounds__(256) k_bface_split(Prm P) {
  constexpr int d = D;
  if (!*P.active) return;
  const Geo &g = P.g;
  long long nf = nfaces(g, d);
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nf) return;
  int n0 = g.nx[0] + (d == 0), n1 = g.nx[1] + (d == 1);
  int i, j, k;
  unflatten3(t, n0, n1, i, j, k);
  const double dt = P.scal[1];
  const double a1 = P.a1, a2 = P.a2, a3 = P.c3 * dt * (P.v_ref * P.b_ref);
  const float *E1 = P.fcor[0], *E2 = P.fcor[1], *E3 = P.fcor[2];
  // differences of the FP32 corner EMFs are formed in FP64 (exact), so the discrete divergence
  // of the update cancels to FP64 rounding as in the FP64 form
  auto e = [](const float *E, long long q) { return (double)E[q]; };
  double tmp;
  if (d == 0) {
    if (C::DIM == 2) tmp = (e(E3, cor_lin(g, 2, i, j + 1, k)) - e(E3, cor_lin(g, 2, i, j, k))) * g.inv_dx[1];
    else tmp = -(e(E2, cor_lin(g, 1, i, j, k + 1)) - e(E2, cor_lin(g, 1, i, j, k))) * g.inv_dx[2] +
               (e(E3, cor_lin(g, 2, i, j + 1, k)) - e(E3, cor_lin(g, 2, i, j, k))) * g.inv_dx[1];
  } else if (d == 1) {
    if (C::DIM == 2) tmp = (e(E3, cor_lin(g, 2, i, j, k)) - e(E3, cor_lin(g, 2, i + 1, j, k))) * g.inv_dx[0];
    else tmp = (e(E1, cor_lin(g, 0, i, j, k + 1)) - e(E1, cor_lin(g, 0, i, j, k))) * g.inv_dx[2] +
               (e(E3, cor_lin(g, 2, i, j, k)) - e(E3, cor_lin(g, 2, i + 1, j, k))) * g.inv_dx[0];
  } else {
    tmp = (e(E2, cor_lin(g, 1, i + 1, j, k)) - e(E2, cor_lin(g, 1, i, j, k))) * g.inv_dx[0] -
          (e(E1, cor_lin(g, 0, i, j + 1, k)) - e(E1, cor_lin(g, 0, i, j, k))) * g.inv_dx[1];
  }
  double b = P.bf[d][t];
  double b0;
  if (P.first_stage) { b0 = b; P.b0f[d][t] = b; } else { b0 = P.b0f[d][t]; }
  P.bf[d][t] = a1 * b0 + a2 * b + a3 * tmp;
}

// New state of one cell that the EoS part of cons->prim needs (the rest is stored before it)
struct C2pState {
  double rho = 1.0, inv_rho = 1.0, eint = 0.0, ye = 0.0, inv_abar = 1.0;
  double Tw = 0.0;  // the stage input's temperature (the Newton's warm start), loaded up front
  long long bc = 0;
};

// MHD stage, part 3a: flux divergence from the face fluxes, gravity and the RK combine of U
// (FP64), b_cc from the updated faces (FP64); stores U (U0 in the first stage), scaled b_cc and
// what depends on the conserved state alone (FP32 velocities and scalars, cell EMFs), and
// returns what the EoS part needs
template <class C>
__device__ __forceinline__ void c2p_mhd_split_combine(const Prm &P, long long c, C2pState &cs) {
  constexpr int NV = C::NV, IP = C::IP, IAS = C::IAS, DIM = C::DIM;
  const Geo &g = P.g;
  double &rho = cs.rho, &inv_rho = cs.inv_rho, &eint = cs.eint, &ye = cs.ye, &inv_abar = cs.inv_abar;
  long long &bc = cs.bc;
  {
    int i, j, k;
    unflatten3(c, g.nx[0], g.nx[1], i, j, k);
    bc = bg_cc(g, i, j, k);
    double bcc[3] = {0, 0, 0}, u[NV];
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
      int ui = i + (d == 0), uj = j + (d == 1), uk = k + (d == 2);
      bcc[d] = 0.5 * (P.bf[d][face_lin(g, d, ui, uj, uk)] + P.bf[d][face_lin(g, d, i, j, k)]);
      P.bccf[(long long)d * g.N + c] = (float)(bcc[d] * P.inv_b_ref);
    }
    // flux divergence (directions in the order of the hydro stage), gravity, RK combine
    float res[NV];
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
      const long long nf = nfaces(g, d);
      const long long flo = face_lin(g, d, i, j, k), fhi = face_lin(g, d, i + (d == 0), j + (d == 1), k + (d == 2));
      const float inv_dl = (float)g.inv_dx[d];
#pragma unroll
      for (int iv = 0; iv < NV; ++iv) {
        float dd = (P.fflux[d][(long long)iv * nf + fhi] - P.fflux[d][(long long)iv * nf + flo]) * inv_dl;
        res[iv] = d == 0 ? dd : res[iv] + dd;
      }
    }
    const double fm = P.rho_ref * P.v_ref, fe = P.p_ref * P.v_ref;
    double rd[NV];
    rd[0] = (double)res[0] * fm;
#pragma unroll
    for (int d = 0; d < DIM; ++d) rd[1 + d] = (double)res[1 + d] * P.p_ref;
    rd[IP] = (double)res[IP] * fe;
#pragma unroll
    for (int iv = IAS; iv < NV; ++iv) rd[iv] = (double)res[iv] * fm;
    if (C::GRAV) {
      const double rho_dev_phys = (double)P.Wf_in[c] * P.rho_ref;
#pragma unroll
      for (int d = 0; d < DIM; ++d)
        rd[1 + d] -= rho_dev_phys * __ldg(P.grav + (long long)d * (g.bg_profile ? g.nx[1] : g.N) + bc);
    }
    {
      const double dt = P.scal[1], a1 = P.a1, a2 = P.a2, a3 = P.c3 * dt;
      double un[NV];
#pragma unroll
      for (int iv = 0; iv < NV; ++iv) un[iv] = P.U[(long long)iv * g.N + c];
      if (g.use_acc) constant_acceleration<DIM, IP>(g, un, rd);
#pragma unroll
      for (int iv = 0; iv < NV; ++iv) {
        double u0;
        if (P.first_stage) {
          u0 = un[iv];
          P.U0[(long long)iv * g.N + c] = un[iv];
        } else {
          u0 = P.U0[(long long)iv * g.N + c];
        }
        u[iv] = a1 * u0 + a2 * un[iv] + a3 * rd[iv];
        P.U[(long long)iv * g.N + c] = u[iv];
      }
    }
    rho = u[0];
    inv_rho = 1.0 / rho;
    double ke = u[1] * u[1] + u[2] * u[2] + (DIM == 3 ? u[3] * u[3] : 0.0);
    eint = u[IP] - 0.5 * ke * inv_rho;
    eint = eint - 0.5 * (bcc[0] * bcc[0] + bcc[1] * bcc[1] + bcc[2] * bcc[2]);
    if (C::ETOT) eint = eint - rho * __ldg(P.phi_cc + bc);
    float vf[3] = {0.f, 0.f, 0.f};
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
      vf[d] = (float)(u[1 + d] * inv_rho * P.inv_v_ref);
      P.Wf_out[(long long)(1 + d) * g.N + c] = vf[d];
    }
    {
      const float bf3[3] = {(float)(bcc[0] * P.inv_b_ref), (float)(bcc[1] * P.inv_b_ref),
                            DIM == 3 ? (float)(bcc[2] * P.inv_b_ref) : 0.0f};
      store_cell_emf(P, c, vf, bf3);
    }
#pragma unroll
    for (int iv = IAS; iv < NV; ++iv) P.Wf_out[(long long)iv * g.N + c] = (float)(u[iv] * inv_rho);
    if (C::HELM) {
      ye = u[IAS] * inv_rho;
      inv_abar = u[IAS + 1] * inv_rho;
    }
  }
}

// Temperature guess of the split MHD cons->prim Newton
enum { C2P_WARM = 0,    // the previous stage's temperature (the reference's warm start)
       C2P_LEARNED = 1, // the network's guess, judged by <= 3 Newton iterations
       C2P_RESCUE = 2   // the warm start; a cell whose first Newton correction exceeds
                        // RESCUE_STEP * T is queued for the learned guess instead
};
// first warm-start correction (relative) above which a cell is handed to the learned guess: the
// network's guesses are within ~0.2% (0.001 dex); from a start 2% off the warm Newton needs
// ~4 more iterations, from the learned guess ~3 in all
constexpr double RESCUE_STEP = 0.02;

// MHD stage, part 3b: cons -> prim of the new state with the Helmholtz Newton (FP64) from the
// warm guess (the previous stage's temperature), or (C2P_LEARNED) from the network's guess lT
// (log10 T; NaN for none): the guess is accepted when the reference Newton converges from it
// within 3 iterations without leaving the table, otherwise the Newton starts again from the
// warm guess.  FP32 density and pressure deviations, gammas, T and eint out; last stage the
// cell's CFL speed with the Alfven speed.  C2P_RESCUE: a cell whose warm start is poor stores
// eint, joins P.rescue_q and returns false with nothing else written (the rescue kernels finish
// it from the learned guess); the other cells run the warm-start Newton unchanged.
template <class C, int MODE>
__device__ __forceinline__ bool c2p_mhd_split_eos(const Prm &P, long long c, const C2pState &cs, float lT_mlp,
                                                  SplitStat &st) {
  constexpr bool LEARNED = MODE == C2P_LEARNED;
  constexpr int IP = C::IP, DIM = C::DIM;
  const Geo &g = P.g;
  const double rho = cs.rho, inv_rho = cs.inv_rho, eint = cs.eint, ye = cs.ye, inv_abar = cs.inv_abar;
  const long long bc = cs.bc;
  HelmCell hc;
  {
    double p, T, sound2;
    if (C::HELM) {
      int clamped = 0, it = 0;
      bool conv = false;
      if constexpr (LEARNED) {
        // judged guess: at most 3 reference Newton iterations from the learned guess (the
        // density part of the cell is already set)
        const bool have_guess = !isnan(lT_mlp);
        helm_cell_init_rho(P.helm, hc, rho, ye);
        if (have_guess) {
          T = fmin(fmax((double)exp10f(lT_mlp), P.helm.Tl * 1.000001), P.helm.Th * 0.999999);
          helm_cell_contract(P.helm, hc, helm_node_index(P.helm.T, P.helm.nT, P.helm.log10_T1, P.helm.dT, T));
          it = helm_rhoe_fast(P.helm, hc, inv_rho, eint * inv_rho, inv_abar, T, 3, clamped, conv);
        }
        if (have_guess && conv && clamped == 0) {
          st.mlp_acc += 1;
        } else {
          st.mlp_rej += 1;
          st.iters += it;
          clamped = 0;
          conv = false;
          T = cs.Tw;
          helm_cell_contract(P.helm, hc, helm_node_index(P.helm.T, P.helm.nT, P.helm.log10_T1, P.helm.dT, T));
          it = helm_rhoe_fast(P.helm, hc, inv_rho, eint * inv_rho, inv_abar, T, 100, clamped, conv);
        }
      } else if constexpr (MODE == C2P_RESCUE) {
        const double Tw = cs.Tw;
        T = Tw;
        helm_cell_init_rho(P.helm, hc, rho, ye);
        helm_cell_contract(P.helm, hc, helm_node_index(P.helm.T, P.helm.nT, P.helm.log10_T1, P.helm.dT, T));
        it = helm_rhoe_fast_from(P.helm, hc, inv_rho, eint * inv_rho, inv_abar, T, Tw, 1, clamped, conv);
        if (!conv && fabs(T - Tw) > RESCUE_STEP * Tw) {
          // poor warm start: the learned guess finishes this cell (its iteration is counted)
          st.iters += it;
          P.eint[c] = eint;
          const unsigned slot = atomicAdd(P.rescue_q, 1u);
          P.rescue_q[1 + slot] = (unsigned)c;
          return false;
        }
        if (!conv) it += helm_rhoe_fast_from(P.helm, hc, inv_rho, eint * inv_rho, inv_abar, T, Tw, 99, clamped, conv);
      } else {
        T = cs.Tw;
        helm_cell_init_rho(P.helm, hc, rho, ye);
        helm_cell_contract(P.helm, hc, helm_node_index(P.helm.T, P.helm.nT, P.helm.log10_T1, P.helm.dT, T));
        it = helm_rhoe_fast(P.helm, hc, inv_rho, eint * inv_rho, inv_abar, T, 100, clamped, conv);
      }
      st.calls += 1; st.iters += it; st.nonconv += !conv; st.clamp += clamped;
      helm_cell_p_sound2(P.helm, hc, rho, inv_rho, T, inv_abar, p, sound2);
      if (C::FAST) {
        // gamma_e goes to FP32 as a deviation from its equilibrium value, so it is formed in FP64;
        // gamma_c is stored as it is, to FP32 precision
        double ge = p / eint + 1.0;
        const float gc = (float)(sound2 * rho) / (float)p;
        if (C::WB) ge = ge - __ldg(P.eq_ge_cc + bc);
        P.gf_out[c] = (float)ge;
        P.gf_out[g.N + c] = gc;
      } else {
        P.gf_out[c] = (float)T;
      }
    } else {
      p = (g.gm - 1.0) * eint;
      T = p / (rho * CONST_RGAS * (1.0 / g.mu));
      sound2 = g.gm * p / rho;
    }
    double rdev = rho, pdev = p;
    if (C::WB) {
      rdev = rho - __ldg(P.eq_rho_cc + bc);
      pdev = p - __ldg(P.eq_p_cc + bc);
    }
    P.Wf_out[c] = (float)(rdev * P.inv_rho_ref);
    P.Wf_out[(long long)IP * g.N + c] = (float)(pdev * P.inv_p_ref);
    P.temp[c] = T;
    P.eint[c] = eint;
    if (!(rho > 0.0) || !(p > 0.0) || !(T > 0.0) || !isfinite(eint)) st.bad += 1;
    if (P.last_stage) {
      // |v| and b_cc^2 of the new state, read back (U and the face B are this cell's own)
      int i, j, k;
      unflatten3(c, g.nx[0], g.nx[1], i, j, k);
      double vabs[3] = {0.0, 0.0, 0.0}, ca2 = 0.0;
#pragma unroll
      for (int d = 0; d < DIM; ++d) {
        const double b = 0.5 * (P.bf[d][face_lin(g, d, i + (d == 0), j + (d == 1), k + (d == 2))] +
                                P.bf[d][face_lin(g, d, i, j, k)]);
        ca2 = d == 0 ? b * b : ca2 + b * b;
        vabs[d] = fabs(P.U[(long long)(1 + d) * g.N + c] * inv_rho);
      }
      double csnd = sqrt(sound2 + ca2 * inv_rho);
      double sx1 = (vabs[0] + csnd) * g.inv_dx[0];
      double sx2 = (vabs[1] + csnd) * g.inv_dx[1];
      double sm = sx1 + sx2;
      if (DIM == 3) sm = (vabs[2] + csnd) * g.inv_dx[2] + sm;
      st.smax = fmax(st.smax, sm);
    }
  }
  return true;
}

// cells per block of the cons->prim kernels
constexpr int C2P_BLOCK = 128;

template <class C, int MODE, int MINB = C::MINB_C2P32>
__global__ void __launch_bounds__(C2P_BLOCK, MINB) k_c2p_mhd_split(Prm P) {
  if (!*P.active) return;
  SplitStat st;
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c < P.g.N) {
    C2pState cs;
    // the warm start first: its load then overlaps the combine instead of following its stores
    if (C::HELM) cs.Tw = P.temp[c];
    c2p_mhd_split_combine<C>(P, c, cs);
    c2p_mhd_split_eos<C, MODE>(P, c, cs, 0.0f, st);
  }
  split_stat_flush<C>(P, st);
}

// cons->prim in two launches (PHL_C2P=two): the combine with the stores that depend on the
// conserved state alone (and eint), then the EoS part from U and eint read back; the second
// kernel holds only the Newton's registers and runs at a higher occupancy
template <class C>
__global__ void __launch_bounds__(128, C::MINB_C2P32) k_c2p_mhd_split_combine(Prm P) {
  if (!*P.active) return;
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= P.g.N) return;
  C2pState cs;
  c2p_mhd_split_combine<C>(P, c, cs);
  P.eint[c] = cs.eint;
}
template <class C>
__global__ void __launch_bounds__(128, C2P_EOS_MINB) k_c2p_mhd_split_eos(Prm P);

// the state of the combine for cell c, read back from U and eint
template <class C>
__device__ __forceinline__ void c2p_state_from_u(const Prm &P, long long c, C2pState &cs) {
  constexpr int IAS = C::IAS;
  const Geo &g = P.g;
  int i, j, k;
  unflatten3(c, g.nx[0], g.nx[1], i, j, k);
  cs.bc = bg_cc(g, i, j, k);
  cs.rho = P.U[c];
  cs.inv_rho = 1.0 / cs.rho;
  cs.eint = P.eint[c];
  if (C::HELM) cs.Tw = P.temp[c];
  cs.ye = P.U[(long long)IAS * g.N + c] * cs.inv_rho;
  cs.inv_abar = P.U[(long long)(IAS + 1) * g.N + c] * cs.inv_rho;
}

// the network's input features of a cell: log10 rho, log10 of the thermal energy (the cold
// energy E(rho, T_lo) from the density row of the table subtracted), Abar, Zbar, each scaled
template <class C>
__device__ __forceinline__ float4 c2p_features(const Prm &P, const C2pState &cs) {
  HelmCell hc;
  const double abar = 1.0 / cs.inv_abar, zbar = cs.ye * abar;
  helm_cell_init_rho(P.helm, hc, cs.rho, cs.ye);
  const double e_th = cs.eint * cs.inv_rho - helm_cell_cold_energy(P.helm, hc, cs.inv_rho, cs.inv_abar);
  float4 f;
  f.x = (log10f((float)cs.rho) - 3.5f) / 5.5f;
  f.y = (log10f((float)fmax(e_th, 1e-30)) - 19.5f) / 8.5f;
  f.z = (float)((abar - 28.5) / 27.5);
  f.w = (float)((zbar - 14.0) / 14.0);
  return f;
}

// Learned guess in the step, in three launches so that the cons->prim kernels keep their
// occupancy (a block-wide tensor-core product inside them would hold all their warps at its
// barriers): (1) the combine, storing eint and the network's features, (2) k_mlp_guess over
// all cells, (3) the EoS part from the stored state and guess.
template <class C>
__global__ void __launch_bounds__(128, C::MINB_C2P32) k_c2p_mhd_split_features(Prm P) {
  if (!*P.active) return;
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= P.g.N) return;
  C2pState cs;
  c2p_mhd_split_combine<C>(P, c, cs);
  P.eint[c] = cs.eint;
  reinterpret_cast<float4 *>(P.mlp_feat)[c] = c2p_features<C>(P, cs);
}

template <class C>
__global__ void __launch_bounds__(128, C::MINB_C2P32) k_c2p_mhd_split_guessed(Prm P) {
  if (!*P.active) return;
  SplitStat st;
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c < P.g.N) {
    // the state of the combine, read back: U and eint
    C2pState cs;
    c2p_state_from_u<C>(P, c, cs);
    st.gevals += 1;
    c2p_mhd_split_eos<C, C2P_LEARNED>(P, c, cs, P.mlp_out[c], st);
  }
  split_stat_flush<C>(P, st);
}

// network guesses for n samples (features [n][4] -> log10 T, NaN where the product stalled);
// the FP32 layers come in as a kernel argument (constant-bank operands)
static __global__ void __launch_bounds__(128) k_mlp_guess(const __grid_constant__ MlpSmall w,
                                                          const __nv_bfloat16 *w2bf, long long n, const float *feat,
                                                          float *out, const int *active, unsigned long long *stalled) {
  if (!*active) return;
  extern __shared__ __align__(128) unsigned char mlp_sm[];
  MlpUmmaSmem &S = *reinterpret_cast<MlpUmmaSmem *>(mlp_sm);
  mlp_cta_setup(w2bf, S);
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  float x[4] = {0.0f, 0.0f, 0.0f, 0.0f};
  if (t < n) {
    const float4 f = reinterpret_cast<const float4 *>(feat)[t];
    x[0] = f.x; x[1] = f.y; x[2] = f.z; x[3] = f.w;
  }
  bool ok = true, have = false;
  const float y = mlp_forward_tile(w, x, S, 0u, ok, have, stalled);
  mlp_cta_teardown(S);
  if (t < n) out[t] = have ? y : __int_as_float(0x7fc00000);
}

template <class C>
__global__ void __launch_bounds__(128, C2P_EOS_MINB) k_c2p_mhd_split_eos(Prm P) {
  if (!*P.active) return;
  SplitStat st;
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c < P.g.N) {
    C2pState cs;
    c2p_state_from_u<C>(P, c, cs);
    c2p_mhd_split_eos<C, C2P_WARM>(P, c, cs, 0.0f, st);
  }
  split_stat_flush<C>(P, st);
}

// ---- learned rescue of poor warm starts (eos_guess = PHL_GUESS_MLP_RESCUE): one kernel on a
// fixed grid over the queue that k_c2p_mhd_split<C, C2P_RESCUE> fills.  Tiles of 128 queue
// slots, strided over the blocks: each thread reads its cell's state back (U, eint) and forms
// the network's features, the block runs one tensor-core product for the tile, and each thread
// finishes its cell from the judged guess.  With an empty queue every block reads the count and
// returns; a block without a tile returns before it claims tensor memory.
template <class C>
__global__ void __launch_bounds__(128) k_c2p_rescue(Prm P, const __grid_constant__ MlpSmall w) {
  if (!*P.active) return;
  const long long n = P.rescue_q[0];
  if ((long long)blockIdx.x * blockDim.x >= n) return;
  extern __shared__ __align__(128) unsigned char mlp_sm[];
  MlpUmmaSmem &S = *reinterpret_cast<MlpUmmaSmem *>(mlp_sm);
  mlp_cta_setup(P.mlp_w2bf, S);
  SplitStat st;
  bool ok = true;
  uint32_t parity = 0;
  for (long long t0 = (long long)blockIdx.x * blockDim.x; t0 < n; t0 += (long long)gridDim.x * blockDim.x) {
    const long long q = t0 + threadIdx.x;
    C2pState cs;
    long long c = -1;
    float x[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    if (q < n) {
      c = P.rescue_q[1 + q];
      c2p_state_from_u<C>(P, c, cs);
      const float4 f = c2p_features<C>(P, cs);
      x[0] = f.x; x[1] = f.y; x[2] = f.z; x[3] = f.w;
    }
    bool have = false;
    const float y = mlp_forward_tile(w, x, S, parity, ok, have, P.stat + STAT_TC_STALLED);
    parity ^= 1u;
    if (c >= 0) {
      st.gevals += 1;
      c2p_mhd_split_eos<C, C2P_LEARNED>(P, c, cs, have ? y : __int_as_float(0x7fc00000), st);
    }
  }
  mlp_cta_teardown(S);
  split_stat_flush<C>(P, st);
}

// FP64 primitives (+eint, gammaf) -> U (FP64) and FP32 deviations (prim->cons of
// source.F90:7057-7117)
template <class C>
__global__ void k_split_from_prim(Prm P) {
  constexpr int NV = C::NV, IP = C::IP, IAS = C::IAS, DIM = C::DIM;
  const Geo &g = P.g;
  long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= g.N) return;
  int i, j, k;
  unflatten3(c, g.nx[0], g.nx[1], i, j, k);
  const long long bc = bg_cc(g, i, j, k);
  double w[NV];
#pragma unroll
  for (int iv = 0; iv < NV; ++iv) w[iv] = P.Win[(long long)iv * g.N + c];
  double rho = w[0], vx1 = w[1], vx2 = w[2], vx3 = DIM == 3 ? w[3] : 0.0;
  double u[NV];
  u[0] = rho; u[1] = rho * vx1; u[2] = rho * vx2; if (DIM == 3) u[3] = rho * vx3;
  double rhoe = P.eint[c] + 0.5 * rho * (vx1 * vx1 + vx2 * vx2 + vx3 * vx3);
  if (C::MHD) {
    double b0 = P.bcc_in[c], b1 = P.bcc_in[g.N + c], b2 = DIM == 3 ? P.bcc_in[2 * g.N + c] : 0.0;
    rhoe = rhoe + 0.5 * (b0 * b0 + b1 * b1 + b2 * b2);
    P.bccf[c] = (float)(b0 * P.inv_b_ref);
    P.bccf[g.N + c] = (float)(b1 * P.inv_b_ref);
    if (DIM == 3) P.bccf[2 * g.N + c] = (float)(b2 * P.inv_b_ref);
  }
  if (C::ETOT) rhoe = rhoe + rho * __ldg(P.phi_cc + bc);
  u[IP] = rhoe;
#pragma unroll
  for (int iv = IAS; iv < NV; ++iv) u[iv] = rho * w[iv];
#pragma unroll
  for (int iv = 0; iv < NV; ++iv) P.U[(long long)iv * g.N + c] = u[iv];
  double rdev = rho, pdev = w[IP];
  if (C::WB) {
    rdev = rho - __ldg(P.eq_rho_cc + bc);
    pdev = w[IP] - __ldg(P.eq_p_cc + bc);
  }
  P.Wf_out[c] = (float)(rdev / P.rho_ref);
#pragma unroll
  for (int d = 0; d < DIM; ++d) P.Wf_out[(long long)(1 + d) * g.N + c] = (float)(w[1 + d] / P.v_ref);
  if (C::MHD) {
    const float vf[3] = {(float)(w[1] / P.v_ref), (float)(w[2] / P.v_ref), DIM == 3 ? (float)(w[3] / P.v_ref) : 0.0f};
    const float bf3[3] = {P.bccf[c], P.bccf[g.N + c], DIM == 3 ? P.bccf[2 * g.N + c] : 0.0f};
    store_cell_emf(P, c, vf, bf3);
  }
  P.Wf_out[(long long)IP * g.N + c] = (float)(pdev / P.p_ref);
#pragma unroll
  for (int iv = IAS; iv < NV; ++iv) P.Wf_out[(long long)iv * g.N + c] = (float)w[iv];
  if (C::FAST) {
    double ge = P.gin[c];
    if (C::WB) ge = ge - __ldg(P.eq_ge_cc + bc);
    P.gf_out[c] = (float)ge;
    P.gf_out[g.N + c] = (float)P.gin[g.N + c];
  } else if (C::HELM) {
    P.gf_out[c] = (float)P.temp[c];
  }
}

// U (FP64) + temp -> FP64 primitives and gammaf (for download and the standalone dt)
template <class C>
__global__ void k_split_to_prim(Prm P) {
  constexpr int NV = C::NV, IP = C::IP, IAS = C::IAS, DIM = C::DIM;
  const Geo &g = P.g;
  long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= g.N) return;
  int i, j, k;
  unflatten3(c, g.nx[0], g.nx[1], i, j, k);
  const long long bc = bg_cc(g, i, j, k);
  double u[NV];
#pragma unroll
  for (int iv = 0; iv < NV; ++iv) u[iv] = P.U[(long long)iv * g.N + c];
  double rho = u[0], inv_rho = 1.0 / rho;
  double eint = P.eint[c];
  double p;
  if (C::HELM) {
    // pressure and sound speed at the state's temperature from the contracted table cell (the
    // evaluation of the split form's cons->prim, equal to given_full to rounding)
    const double inv_abar = u[IAS + 1] * inv_rho, ye = u[IAS] * inv_rho, T = P.temp[c];
    HelmCell hc;
    helm_cell_init_rho(P.helm, hc, rho, ye);
    helm_cell_contract(P.helm, hc, helm_node_index(P.helm.T, P.helm.nT, P.helm.log10_T1, P.helm.dT, T));
    double s2;
    helm_cell_p_sound2(P.helm, hc, rho, inv_rho, T, inv_abar, p, s2);
    if (C::FAST) {
      P.gout[c] = p / eint + 1.0;
      P.gout[g.N + c] = s2 * rho / p;
    } else {
      P.gout[c] = P.temp[c];
    }
  } else {
    p = (g.gm - 1.0) * eint;
  }
  if (C::MHD) {
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
      int ui = i + (d == 0), uj = j + (d == 1), uk = k + (d == 2);
      P.bcc_out[(long long)d * g.N + c] = 0.5 * (P.bf[d][face_lin(g, d, ui, uj, uk)] + P.bf[d][face_lin(g, d, i, j, k)]);
    }
  }
  P.Wout[c] = rho;
#pragma unroll
  for (int d = 0; d < DIM; ++d) P.Wout[(long long)(1 + d) * g.N + c] = u[1 + d] * inv_rho;
  P.Wout[(long long)IP * g.N + c] = p;
#pragma unroll
  for (int iv = IAS; iv < NV; ++iv) P.Wout[(long long)iv * g.N + c] = u[iv] * inv_rho;
  (void)bc;
}

namespace {
inline unsigned nblk(long long n, int t) { return (unsigned)((n + t - 1) / t); }

// cuTensorMapEncodeTiled from the driver, found through the runtime (no link to libcuda)
PFN_cuTensorMapEncodeTiled tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled>(p);
  }
  return fn;
}

// 4D map (x1, x2, x3, variable) over an FP32 SoA field block, box = (bx, by, bz, nvar)
bool encode_box_map(CUtensorMap *m, const float *base, int nvar, const Geo &g, int bx, int by, int bz) {
  PFN_cuTensorMapEncodeTiled enc = tensor_map_encoder();
  if (!enc || !base) return false;
  const cuuint64_t nx = (cuuint64_t)g.nx[0], ny = (cuuint64_t)g.nx[1], nz = (cuuint64_t)g.nx[2];
  const cuuint64_t dims[4] = {nx, ny, nz, (cuuint64_t)nvar};
  const cuuint64_t strides[3] = {nx * 4, nx * ny * 4, (cuuint64_t)g.N * 4};
  const cuuint32_t box[4] = {(cuuint32_t)bx, (cuuint32_t)by, (cuuint32_t)bz, (cuuint32_t)nvar};
  const cuuint32_t es[4] = {1, 1, 1, 1};
  return enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, const_cast<float *>(base), dims, strides, box, es,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}
bool encode_plane_map(CUtensorMap *m, const float *base, int nvar, const Geo &g, int bx, int by) {
  return encode_box_map(m, base, nvar, g, bx, by, 1);
}
}

template <class C>
struct SplitRunnerT : Runner {
  static constexpr int TX = 32, TY = 8, KZ = 16;
  bool attr_set = false;
  // tensor maps of the two FP32 state buffers (the stage input alternates between them)
  struct MapEntry {
    const float *w = nullptr;
    SplitMaps maps;
    bool ok = false;
  } map_cache[2];
  // maps of this stage's input, or false when interior tiles must also copy cell by cell
  bool stage_maps(const Prm &P, SplitMaps &out) {
    using T = SplitTile<C, TX, TY>;
    const Geo &g = P.g;
    // bulk copies need a periodic x3 (the plane index wraps) and interior tiles in x1 and x2
    if (g.bc[2][0] != BC_PERIODIC || g.nx[0] < 3 * TX || g.nx[1] < 3 * TY) return false;
    for (auto &e : map_cache)
      if (e.w == P.Wf_in) {
        out = e.maps;
        return e.ok;
      }
    MapEntry &e = map_cache[map_cache[0].w ? 1 : 0];
    e.w = P.Wf_in;
    e.ok = encode_plane_map(&e.maps.w, P.Wf_in, C::NV, g, T::SX, T::SY);
    if (e.ok && C::HELM) e.ok = encode_plane_map(&e.maps.g, P.gf_in, 2, g, T::SX, T::SY);
    out = e.maps;
    return e.ok;
  }
  // tensor maps of the tiled face kernels, per direction and stage input (W' and the gammas
  // alternate with the stage)
  struct TileMapEntry {
    const float *w = nullptr;
    FaceTileMaps maps;
    bool ok = false;
  } tile_cache[3][2];
  template <int D>
  bool tile_maps(const Prm &P, FaceTileMaps &out) {
    using S_ = FaceTileSmem<C, D>;
    for (auto &e : tile_cache[D])
      if (e.w == P.Wf_in) {
        out = e.maps;
        return e.ok;
      }
    TileMapEntry &e = tile_cache[D][tile_cache[D][0].w ? 1 : 0];
    e.w = P.Wf_in;
    e.ok = encode_box_map(&e.maps.w, P.Wf_in, C::NV, P.g, S_::SX, S_::SY, S_::SZ) &&
           encode_box_map(&e.maps.b, P.bccf, 3, P.g, S_::SX, S_::SY, S_::SZ);
    if (e.ok && C::HELM) e.ok = encode_box_map(&e.maps.g, P.gf_in, 2, P.g, S_::SX, S_::SY, S_::SZ);
    out = e.maps;
    return e.ok;
  }
  // blocks of the tiled face kernels resident on the GPU at once, per direction: the grid of
  // their tile loop (found at construction, outside any stream capture; 0 if unknown)
  long long tile_wave[3] = {0, 0, 0};
  template <class K>
  static long long wave_of(K kernel, int threads) {
    int dev = 0, sms = 0, nb = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kernel, threads, 0) != cudaSuccess)
      return 0;
    return (long long)sms * nb;
  }
  SplitRunnerT() {
    if constexpr (C::MHD && C::REC == REC_LIM2ND && !C::SF) {
      tile_wave[0] = wave_of(k_face_split_mhd_tile<C, 0>, FaceTileSmem<C, 0>::NT);
      tile_wave[1] = wave_of(k_face_split_mhd_tile<C, 1>, FaceTileSmem<C, 1>::NT);
      if constexpr (C::DIM == 3) tile_wave[2] = wave_of(k_face_split_mhd_tile<C, 2>, FaceTileSmem<C, 2>::NT);
    }
  }
  // resident blocks per SM the Helmholtz MHD cons->prim is compiled for: 8 (64 registers, ~100
  // B of spills), which ran a step at 256^3 in 13.56 ms against 13.89 at 7 (72 registers), 14.37
  // at 6 (80), 13.73 at 9 and 14.14 at 10: its time is latency, and more resident warps hide it
  // until the spills dominate; PHL_C2P_MINB=6 selects the 80-register build (comparison)
  const int c2p_minb = [] {
    const char *e = getenv("PHL_C2P_MINB");
    return e && atoi(e) == 6 ? 6 : 8;
  }();
  // PHL_C2P=two runs the warm-start cons->prim of the MHD stage as two launches
  const bool c2p_two = [] {
    const char *e = getenv("PHL_C2P");
    return e && strcmp(e, "two") == 0;
  }();
  // face kernel per direction: by default the shared-memory tiles along x1 (where the walking
  // kernel's threads stride K0 cells apart) and the walking kernels along x2 and x3 (threads of
  // a warp are neighbours in x1 there, and the walk, with no block barrier and the edges in
  // registers, ran 0.80 -> 0.67 ms per direction at 256^3); PHL_FACE_KERNEL=walk / =tile select
  // one kind for every direction (comparisons)
  const int face_kind = [] {
    const char *e = getenv("PHL_FACE_KERNEL");
    if (e && strcmp(e, "walk") == 0) return 0;
    if (e && strcmp(e, "tile") == 0) return 2;
    return 1;
  }();
  // faces along D from shared-memory tiles, when the grid is a multiple of the tile; false to
  // fall back to the walking kernel
  template <int D>
  bool launch_face_tiles(const Prm &P, cudaStream_t s) {
    if constexpr (C::SF || C::REC != REC_LIM2ND) {
      return false;
    } else {
      using T = FaceTile<D>;
      using S_ = FaceTileSmem<C, D>;
      const Geo &g = P.g;
      const int nz = C::DIM == 3 ? g.nx[2] : 1;
      // without USE_FASTEOS the walks serve every direction (36.9 ms per 256^3 MHD step against
      // 37.5 with the x1 tiles, whose 64 registers spill the two per-face EoS solves)
      if (face_kind == 0 || (face_kind == 1 && (D != 0 || C::EOSM == EOS_GIVEN))) return false;
      if (g.nx[0] % T::TX || g.nx[1] % T::TY || nz % T::TZ) return false;
      FaceTileMaps m;
      if (!tile_maps<D>(P, m)) return false;
      const long long ntiles = (long long)(g.nx[0] / T::TX) * (g.nx[1] / T::TY) * (nz / T::TZ);
      // one resident wave of blocks striding over the tiles (found at construction)
      const long long wave = tile_wave[D] > 0 ? tile_wave[D] : ntiles;
      k_face_split_mhd_tile<C, D><<<(unsigned)std::max(1ll, std::min(ntiles, wave)), S_::NT, 0, s>>>(P, m, (int)ntiles);
      return true;
    }
  }
  // PHL_STAGE_KERNEL=cell selects the per-cell kernel on any grid, =tiled_cpasync the tiled
  // kernel with cell-by-cell copies only (comparisons of the three)
  const bool allow_tiled = [] {
    const char *e = getenv("PHL_STAGE_KERNEL");
    return !(e && strcmp(e, "cell") == 0);
  }();
  const bool allow_tma = [] {
    const char *e = getenv("PHL_STAGE_KERNEL");
    return !(e && strcmp(e, "tiled_cpasync") == 0);
  }();
  bool tiled(const Geo &g) const {
    return allow_tiled && C::DIM == 3 && g.nx[0] % TX == 0 && g.nx[1] % TY == 0 && g.nx[2] % KZ == 0;
  }
  void stage(const Prm &P, cudaStream_t s) override {
    if constexpr (C::SF) {
      k_sf_mark_split<C><<<nblk(sf_mark_cells<C>(P.g), 256), 256, 0, s>>>(P);
      k_sf_flag<C><<<nblk(sf_flag_cells<C>(P.g), 256), 256, 0, s>>>(P);
    }
    if constexpr (C::MHD) {
      const Geo &g = P.g;
      auto nfc = [&](int d) {
        return (long long)(g.nx[0] + (d == 0)) * (g.nx[1] + (d == 1)) * (g.nx[2] + (d == 2));
      };
      if constexpr (C::REC == REC_LIM2ND) {
        // threads of the walking kernels: faces along D in chunks of K, times the other extents
        auto nwalk = [&](int d, int k) {
          long long n = (g.nx[d] + 1 + k - 1) / k;
          for (int a = 0; a < C::DIM; ++a)
            if (a != d) n *= g.nx[a];
          return n;
        };
        if (!launch_face_tiles<0>(P, s))
          k_face_split_mhd_walk<C, 0, WALK_K0><<<nblk(nwalk(0, WALK_K0), 128), 128, 0, s>>>(P);
        if (!launch_face_tiles<1>(P, s))
          k_face_split_mhd_walk<C, 1, WALK_K><<<nblk(nwalk(1, WALK_K), 128), 128, 0, s>>>(P);
        if constexpr (C::DIM == 3)
          if (!launch_face_tiles<2>(P, s))
            k_face_split_mhd_walk<C, 2, WALK_K><<<nblk(nwalk(2, WALK_K), 128), 128, 0, s>>>(P);
      } else {
        k_face_split_mhd<C, 0><<<nblk(nfc(0), 128), 128, 0, s>>>(P);
        k_face_split_mhd<C, 1><<<nblk(nfc(1), 128), 128, 0, s>>>(P);
        if constexpr (C::DIM == 3) k_face_split_mhd<C, 2><<<nblk(nfc(2), 128), 128, 0, s>>>(P);
      }
      if constexpr (C::DIM == 3) {
        corners<0>(P, s);
        corners<1>(P, s);
      }
      corners<2>(P, s);
      k_bface_split<C, 0><<<nblk(nfc(0), 256), 256, 0, s>>>(P);
      k_bface_split<C, 1><<<nblk(nfc(1), 256), 256, 0, s>>>(P);
      if constexpr (C::DIM == 3) k_bface_split<C, 2><<<nblk(nfc(2), 256), 256, 0, s>>>(P);
      if constexpr (C::HELM) {
        if (P.mlp_w && P.mlp_small && P.rescue_q) {
          // warm start everywhere; cells with a poor warm start through the learned guess
          cudaMemsetAsync(P.rescue_q, 0, sizeof(unsigned), s);
          if (C::HELM && c2p_minb == 8)
            k_c2p_mhd_split<C, C2P_RESCUE, 8><<<nblk(g.N, C2P_BLOCK), C2P_BLOCK, 0, s>>>(P);
          else
            k_c2p_mhd_split<C, C2P_RESCUE><<<nblk(g.N, C2P_BLOCK), C2P_BLOCK, 0, s>>>(P);
          k_c2p_rescue<C><<<RESCUE_BLOCKS, 128, sizeof(MlpUmmaSmem), s>>>(P, *P.mlp_small);
          return;
        }
        if (P.mlp_w && P.mlp_small && P.mlp_feat && P.mlp_out) {
          k_c2p_mhd_split_features<C><<<nblk(g.N, 128), 128, 0, s>>>(P);
          k_mlp_guess<<<nblk(g.N, 128), 128, sizeof(MlpUmmaSmem), s>>>(*P.mlp_small, P.mlp_w2bf, g.N, P.mlp_feat,
                                                                       P.mlp_out, P.active, P.stat + STAT_TC_STALLED);
          k_c2p_mhd_split_guessed<C><<<nblk(g.N, 128), 128, 0, s>>>(P);
          return;
        }
      }
      if (c2p_two) {
        k_c2p_mhd_split_combine<C><<<nblk(g.N, 128), 128, 0, s>>>(P);
        k_c2p_mhd_split_eos<C><<<nblk(g.N, 128), 128, 0, s>>>(P);
      } else if (C::HELM && c2p_minb == 8) {
        k_c2p_mhd_split<C, C2P_WARM, 8><<<nblk(g.N, C2P_BLOCK), C2P_BLOCK, 0, s>>>(P);
      } else {
        k_c2p_mhd_split<C, C2P_WARM><<<nblk(g.N, C2P_BLOCK), C2P_BLOCK, 0, s>>>(P);
      }
    } else {
      hydro_stage(P, s);
    }
  }
  // corner EMFs along axis A: the interior corners' blocks, then the rim's, in one launch
  template <int A>
  void corners(const Prm &P, cudaStream_t s) {
    constexpr int pa = A == 2 ? 0 : (A == 0 ? 1 : 2), qa = A == 2 ? 1 : (A == 0 ? 2 : 0);
    const Geo &g = P.g;
    const long long na = C::DIM == 3 ? g.nx[A] : 1;
    const long long nin = (long long)(g.nx[pa] - 1) * (g.nx[qa] - 1) * na;
    const long long nrim = 2ll * (g.nx[pa] + g.nx[qa]) * na;
    const unsigned bin = nblk(nin, 256);
    k_corner_split<C, A><<<bin + nblk(nrim, 256), 256, 0, s>>>(P, bin);
  }
  void hydro_stage(const Prm &P, cudaStream_t s) {
    if constexpr (C::DIM == 3 && C::SW == 2) {
      if (tiled(P.g)) {
        constexpr size_t sm = SplitTile<C, TX, TY>::bytes();
        if (!attr_set) {
          cudaFuncSetAttribute(k_stage_split_tiled<C, TX, TY, KZ>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)sm);
          attr_set = true;
        }
        dim3 grid(P.g.nx[0] / TX, P.g.nx[1] / TY, P.g.nx[2] / KZ);
        SplitMaps maps;
        memset(&maps, 0, sizeof(maps));
        const int use_tma = allow_tma && stage_maps(P, maps) ? 1 : 0;
        k_stage_split_tiled<C, TX, TY, KZ><<<grid, TX * TY, sm, s>>>(P, maps, use_tma);
        return;
      }
    }
    k_stage_split<C><<<nblk(P.g.N, 128), 128, 0, s>>>(P);
  }
  void split_from_prim(const Prm &P, cudaStream_t s) override {
    k_split_from_prim<C><<<nblk(P.g.N, 256), 256, 0, s>>>(P);
  }
  void split_to_prim(const Prm &P, cudaStream_t s) override {
    k_split_to_prim<C><<<nblk(P.g.N, 256), 256, 0, s>>>(P);
  }
};

#define PHL_SPLIT_LIST(X)                                   \
  X(2, 4, true, false, false, R_HLLD, false, REC_LIM2ND, false) \
  X(2, 4, true, false, false, R_LHLLD, false, REC_LIM2ND, false) \
  X(3, 5, true, false, false, R_HLLD, false, REC_LIM2ND, false) \
  X(3, 5, true, false, false, R_LHLLD, false, REC_LIM2ND, false) \
  X(3, 7, true, true, true, R_LHLLD, true, REC_LIM2ND, false) \
  X(3, 7, true, true, true, R_HLLD, true, REC_LIM2ND, false) \
  X(3, 7, true, true, true, R_LHLLD, false, REC_LIM2ND, false) \
  X(2, 4, false, false, false, R_LHLLC, false, REC_LIM2ND, false) \
  X(2, 4, false, false, false, R_HLLC, false, REC_LIM2ND, false) \
  X(2, 4, false, false, true, R_LHLLC, false, REC_LIM2ND, false) \
  X(2, 6, false, true, true, R_LHLLC, true, REC_LIM2ND, false) \
  X(3, 5, false, false, false, R_LHLLC, false, REC_LIM2ND, false) \
  X(3, 5, false, false, false, R_HLLC, false, REC_LIM2ND, false) \
  X(3, 7, false, true, true, R_LHLLC, true, REC_LIM2ND, false) \
  X(3, 7, false, true, true, R_HLLC, true, REC_LIM2ND, false) \
  X(3, 7, false, true, true, R_LHLLC, false, REC_LIM2ND, false) \
  X(3, 7, false, true, true, R_HLLC, false, REC_LIM2ND, false) \
  X(2, 4, true, false, false, R_HLLD, false, REC_LIM5TH, false) \
  X(3, 7, true, true, true, R_LHLLD, true, REC_PPH, false) \
  X(3, 7, true, true, true, R_LHLLD, true, REC_LIM5TH, false) \
  X(3, 7, false, true, true, R_LHLLC, true, REC_PPH, false) \
  X(3, 7, false, true, true, R_LHLLC, true, REC_LIM5TH, false) \
  X(2, 5, false, false, false, R_HLLC, false, REC_LIM2ND, true) \
  X(2, 4, true, false, false, R_HLLD, false, REC_LIM2ND, true) \
  X(3, 7, false, true, true, R_LHLLC, true, REC_LIM2ND, true) \
  X(3, 7, false, true, true, R_LHLLC, true, REC_PPH, true) \
  X(3, 7, true, true, true, R_LHLLD, true, REC_LIM2ND, true)

Runner *make_split_runner(int dim, int nv, bool mhd, bool helm, bool strat, int riem, bool fast, int rec, bool sf) {
#define X(D, N, M, H, S, R, F, REC, SF)                                                                      \
  if (dim == D && nv == N && mhd == M && helm == H && strat == S && riem == R && (!H || fast == F) &&         \
      rec == REC && sf == SF)                                                                                 \
    return new SplitRunnerT<Cfg<D, N, M, H, S, S, S, R, F, REC, SF>>();
  PHL_SPLIT_LIST(X)
#undef X
  return nullptr;
}

}  // namespace phl
