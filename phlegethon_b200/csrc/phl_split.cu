// phl_split.cu -- FP32 split-precision form of the explicit FV step (hydro configurations).
//
// Storage per cell: conserved state U (FP64, carried across stages and steps), primitive
// deviations W' = (rho - rho_eq, v, p - p_eq, scalars) and (gammae - gammae_eq, gammac) in FP32,
// temperature and internal energy in FP64.  Reconstruction (LIM2ND), the Riemann solver and
// the flux divergence run in FP32 on the well-balanced deviations: the pressure enters every
// flux as a deviation, so pR - pL, p* - p_eq,face and the momentum flux after the WB fix
// (source/source.F90:8953-8959) are formed without cancelling large numbers, and Mach 1e-3
// perturbations keep their FP32 precision.  The RK combine, cons->prim, the Helmholtz Newton
// inversion and the CFL maximum stay in FP64.  All FP32 quantities are in scaled units
// (rho / rho_ref, p / p_ref, v / v_ref with v_ref^2 = p_ref / rho_ref, phi / v_ref^2), fixed per run,
// so products of deviations never leave FP32 range whatever the problem's cgs magnitudes.
#include <cuda_runtime.h>
#include "phl_eos_fast.cuh"
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
template <int DIM, int NV, bool FAST, int RIEM>
__device__ __forceinline__ void riemann_hydro_split(const float *qL, const float *qR, const float *gL,
                                                    const float *gR, float pe, float gm, float mach_cutoff,
                                                    float *flux) {
  constexpr int IP = 1 + DIM, IAS = 2 + DIM;
  const float igmm1 = 1.0f / (gm - 1.0f);
  float rhoL = qL[0], inv_rhoL = 1.0f / rhoL, vx1L = qL[1], vx2L = qL[2], vx3L = DIM == 3 ? qL[3] : 0.0f;
  float v2L = vx1L * vx1L + vx2L * vx2L + vx3L * vx3L;
  float pLd = qL[IP], pL = pe + pLd, eint, cL, cR;
  if (FAST) { eint = pL / (gL[0] - 1.0f); cL = sqrtf(gL[1] * pL * inv_rhoL); }
  else { eint = igmm1 * pL; cL = sqrtf(gm * pL * inv_rhoL); }
  float rhoeL = eint + 0.5f * rhoL * v2L;
  float rhoR = qR[0], inv_rhoR = 1.0f / rhoR, vx1R = qR[1], vx2R = qR[2], vx3R = DIM == 3 ? qR[3] : 0.0f;
  float v2R = vx1R * vx1R + vx2R * vx2R + vx3R * vx3R;
  float pRd = qR[IP], pR = pe + pRd;
  if (FAST) { eint = pR / (gR[0] - 1.0f); cR = sqrtf(gR[1] * pR * inv_rhoR); }
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
  if (RIEM == R_LHLLC) {
    float machL = sqrtf(v2L) / cL, machR = sqrtf(v2R) / cR;
    float chi = fminf(1.0f, fmaxf(machL, machR));
    chi = fmaxf(mach_cutoff, chi);
    float phi = chi * (2.0f - chi);
    float rhobar = 0.5f * (rhoL + rhoR), cbar = 0.5f * (cL + cR);
    float pstar_d = 0.5f * (pLd + pRd) - 0.5f * phi * rhobar * cbar * (vx1R - vx1L);
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

// flux through the low face of cell m along d from the FP32 deviation states of cells m-2..m+1
template <class C>
__device__ __forceinline__ void face_flux_split(const Prm &P, int d, int fi, int fj, int fk, const float *wl2,
                                                const float *wl1, const float *wr1, const float *wr2,
                                                const float *gl2, const float *gl1, const float *gr1,
                                                const float *gr2, float F[C::NV]) {
  constexpr int NV = C::NV, IP = C::IP;
  const Geo &g = P.g;
  float qL[NV], qR[NV], lo, hi;
#pragma unroll
  for (int iv = 0; iv < NV; ++iv) {
    plm_f32(wl2[iv], wl1[iv], wr1[iv], lo, hi);
    qL[iv] = hi;
    plm_f32(wl1[iv], wr1[iv], wr2[iv], lo, hi);
    qR[iv] = lo;
  }
  if (d == 1) {
    float a = qL[1], b = qL[2]; qL[1] = b; qL[2] = -a;
    a = qR[1]; b = qR[2]; qR[1] = b; qR[2] = -a;
  } else if (C::DIM == 3 && d == 2) {
    float a = qL[1], b = qL[2], c = qL[3]; qL[1] = c; qL[2] = a; qL[3] = b;
    a = qR[1]; b = qR[2]; c = qR[3]; qR[1] = c; qR[2] = a; qR[3] = b;
  }
  float pe = 0.0f, phi_f = 0.0f;
  long long fb = 0;
  if (C::WB || C::ETOT) fb = bg_face(g, d, fi, fj, fk);
  if (C::WB) {
    float rho_eq = (float)(__ldg(P.eq_rho_f[d] + fb) / P.rho_ref);
    qL[0] = rho_eq + qL[0];
    qR[0] = rho_eq + qR[0];
    pe = (float)(__ldg(P.eq_p_f[d] + fb) / P.p_ref);
  }
  float gL[2] = {0.f, 0.f}, gR[2] = {0.f, 0.f};
  if (C::HELM) {
#pragma unroll
    for (int iv = 0; iv < 2; ++iv) {
      plm_f32(gl2[iv], gl1[iv], gr1[iv], lo, hi);
      gL[iv] = hi;
      plm_f32(gl1[iv], gr1[iv], gr2[iv], lo, hi);
      gR[iv] = lo;
    }
    if (C::WB) {
      float ge = (float)__ldg(P.eq_ge_f[d] + fb);
      gL[0] = gL[0] + ge;
      gR[0] = gR[0] + ge;
    }
  }
  riemann_hydro_split<C::DIM, NV, C::HELM, C::RIEM>(qL, qR, gL, gR, pe, (float)g.gm, (float)g.mach_cutoff, F);
  if (d == 1) {
    float a = F[1], b = F[2]; F[1] = -b; F[2] = a;
  } else if (C::DIM == 3 && d == 2) {
    float a = F[1], b = F[2], c = F[3]; F[1] = b; F[2] = c; F[3] = a;
  }
  if (C::ETOT) {
    phi_f = (float)(__ldg(P.phi_f[d] + fb) / (P.v_ref * P.v_ref));
    F[IP] = F[IP] + F[0] * phi_f;
  }
}

// --------------------------------------------------------------------- split stage kernel
template <class C>
__global__ void __launch_bounds__(128) k_stage_split(Prm P) {
  if (!*P.active) return;
  constexpr int NV = C::NV, IP = C::IP, IAS = C::IAS, DIM = C::DIM;
  const Geo &g = P.g;
  long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  double smax_loc = 0.0;
  unsigned long long n_calls = 0, n_iters = 0, n_nonconv = 0, n_clamp = 0, n_bad = 0;
  if (c < g.N) {
    const int i = (int)(c % g.nx[0]);
    const int j = (int)((c / g.nx[0]) % g.nx[1]);
    const int k = (int)(c / ((long long)g.nx[0] * g.nx[1]));
    const double dt = P.scal[1];
    float res[NV];
    float rho_dev = 0.0f;
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
      float w[5][NV], gm5[5][2];
#pragma unroll
      for (int s = 0; s < 5; ++s) {
        int ii = i + (d == 0 ? s - 2 : 0), jj = j + (d == 1 ? s - 2 : 0), kk = k + (d == 2 ? s - 2 : 0);
        load_wf<C>(P, ii, jj, kk, w[s], gm5[s]);
      }
      if (d == 0) rho_dev = w[2][0];
      float Flo[NV], Fhi[NV];
      face_flux_split<C>(P, d, i, j, k, w[0], w[1], w[2], w[3], gm5[0], gm5[1], gm5[2], gm5[3], Flo);
      face_flux_split<C>(P, d, i + (d == 0), j + (d == 1), k + (d == 2), w[1], w[2], w[3], w[4], gm5[1], gm5[2],
                         gm5[3], gm5[4], Fhi);
      const float inv_dl = (float)g.inv_dx[d];
#pragma unroll
      for (int iv = 0; iv < NV; ++iv) {
        float dd = (Fhi[iv] - Flo[iv]) * inv_dl;
        res[iv] = d == 0 ? dd : res[iv] + dd;
      }
    }
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
      double abar = 1.0 / inv_abar, zbar = ye * abar;
      T = P.temp[c];
      int clamped = 0;
      bool conv = false;
      HelmCell hc;
      helm_cell_init(P.helm, hc, rho, abar, zbar, T);
      int it = helm_rhoe_fast(P.helm, hc, rho, eint * inv_rho, inv_abar, T, 100, clamped, conv);
      n_calls += 1; n_iters += it; n_nonconv += !conv; n_clamp += clamped;
      helm_cell_p_sound(P.helm, hc, rho, T, inv_abar, p, sound);
      double ge = p / eint + 1.0, gc = sound * sound * rho / p;
      if (C::WB) ge = ge - __ldg(P.eq_ge_cc + bc);
      P.gf_out[c] = (float)ge;
      P.gf_out[g.N + c] = (float)gc;
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
    P.Wf_out[c] = (float)(rdev / P.rho_ref);
#pragma unroll
    for (int d = 0; d < DIM; ++d) P.Wf_out[(long long)(1 + d) * g.N + c] = (float)(u[1 + d] * inv_rho / P.v_ref);
    P.Wf_out[(long long)IP * g.N + c] = (float)(pdev / P.p_ref);
#pragma unroll
    for (int iv = IAS; iv < NV; ++iv) P.Wf_out[(long long)iv * g.N + c] = (float)(u[iv] * inv_rho);
    P.temp[c] = T;
    P.eint[c] = eint;
    if (!(rho > 0.0) || !(p > 0.0) || !(T > 0.0) || !isfinite(eint)) n_bad += 1;
    if (P.last_stage) {
      double sx1 = (fabs(u[1] * inv_rho) + sound) * g.inv_dx[0];
      double sx2 = (fabs(u[2] * inv_rho) + sound) * g.inv_dx[1];
      smax_loc = sx1 + sx2;
      if (DIM == 3) smax_loc = (fabs(u[3] * inv_rho) + sound) * g.inv_dx[2] + smax_loc;
    }
  }
  if (P.last_stage) block_max_atomic(smax_loc, P.smax_bits);
  if (C::HELM) {
    block_sum_atomic(n_calls, P.stat + STAT_NEWTON_CALLS);
    block_sum_atomic(n_iters, P.stat + STAT_NEWTON_ITERS);
    block_sum_atomic(n_nonconv, P.stat + STAT_NEWTON_NONCONV);
    block_sum_atomic(n_clamp, P.stat + STAT_NEWTON_CLAMP);
  }
  block_sum_atomic(n_bad, P.stat + STAT_NONFINITE);
}

// FP64 primitives (+eint, gammaf) -> U (FP64) and FP32 deviations (prim->cons of
// source.F90:7057-7117)
template <class C>
__global__ void k_split_from_prim(Prm P) {
  constexpr int NV = C::NV, IP = C::IP, IAS = C::IAS, DIM = C::DIM;
  const Geo &g = P.g;
  long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= g.N) return;
  const int i = (int)(c % g.nx[0]);
  const int j = (int)((c / g.nx[0]) % g.nx[1]);
  const int k = (int)(c / ((long long)g.nx[0] * g.nx[1]));
  const long long bc = bg_cc(g, i, j, k);
  double w[NV];
#pragma unroll
  for (int iv = 0; iv < NV; ++iv) w[iv] = P.Win[(long long)iv * g.N + c];
  double rho = w[0], vx1 = w[1], vx2 = w[2], vx3 = DIM == 3 ? w[3] : 0.0;
  double u[NV];
  u[0] = rho; u[1] = rho * vx1; u[2] = rho * vx2; if (DIM == 3) u[3] = rho * vx3;
  double rhoe = P.eint[c] + 0.5 * rho * (vx1 * vx1 + vx2 * vx2 + vx3 * vx3);
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
  P.Wf_out[(long long)IP * g.N + c] = (float)(pdev / P.p_ref);
#pragma unroll
  for (int iv = IAS; iv < NV; ++iv) P.Wf_out[(long long)iv * g.N + c] = (float)w[iv];
  if (C::HELM) {
    double ge = P.gin[c];
    if (C::WB) ge = ge - __ldg(P.eq_ge_cc + bc);
    P.gf_out[c] = (float)ge;
    P.gf_out[g.N + c] = (float)P.gin[g.N + c];
  }
}

// U (FP64) + temp -> FP64 primitives and gammaf (for download and the standalone dt)
template <class C>
__global__ void k_split_to_prim(Prm P) {
  constexpr int NV = C::NV, IP = C::IP, IAS = C::IAS, DIM = C::DIM;
  const Geo &g = P.g;
  long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= g.N) return;
  const int i = (int)(c % g.nx[0]);
  const int j = (int)((c / g.nx[0]) % g.nx[1]);
  const int k = (int)(c / ((long long)g.nx[0] * g.nx[1]));
  const long long bc = bg_cc(g, i, j, k);
  double u[NV];
#pragma unroll
  for (int iv = 0; iv < NV; ++iv) u[iv] = P.U[(long long)iv * g.N + c];
  double rho = u[0], inv_rho = 1.0 / rho;
  double eint = P.eint[c];
  double p;
  if (C::HELM) {
    double ye = u[IAS] * inv_rho, abar = rho / u[IAS + 1], zbar = ye * abar, E, s, cv;
    helm_given_full(P.helm, rho, P.temp[c], abar, zbar, p, E, s, cv);
    P.gout[c] = p / eint + 1.0;
    P.gout[g.N + c] = s * s * rho / p;
  } else {
    p = (g.gm - 1.0) * eint;
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
}

template <class C>
struct SplitRunnerT : Runner {
  void stage(const Prm &P, cudaStream_t s) override { k_stage_split<C><<<nblk(P.g.N, 128), 128, 0, s>>>(P); }
  void dt(const Prm &P, cudaStream_t s) override { k_dt<C><<<nblk(P.g.N, 256), 256, 0, s>>>(P); }
  void init_thermo(const Prm &P, cudaStream_t s) override {
    k_init_thermo<C><<<nblk(P.g.N, 128), 128, 0, s>>>(P);
  }
  void split_from_prim(const Prm &P, cudaStream_t s) override {
    k_split_from_prim<C><<<nblk(P.g.N, 256), 256, 0, s>>>(P);
  }
  void split_to_prim(const Prm &P, cudaStream_t s) override {
    k_split_to_prim<C><<<nblk(P.g.N, 256), 256, 0, s>>>(P);
  }
};

#define PHL_SPLIT_LIST(X)                 \
  X(2, 4, false, false, false, R_LHLLC)   \
  X(2, 4, false, false, false, R_HLLC)    \
  X(2, 4, false, false, true, R_LHLLC)    \
  X(2, 6, false, true, true, R_LHLLC)     \
  X(3, 5, false, false, false, R_LHLLC)   \
  X(3, 5, false, false, false, R_HLLC)    \
  X(3, 7, false, true, true, R_LHLLC)     \
  X(3, 7, false, true, true, R_HLLC)

Runner *make_split_runner(int dim, int nv, bool mhd, bool helm, bool strat, int riem) {
#define X(D, N, M, H, S, R)                                                              \
  if (dim == D && nv == N && mhd == M && helm == H && strat == S && riem == R)           \
    return new SplitRunnerT<Cfg<D, N, M, H, S, S, S, R>>();
  PHL_SPLIT_LIST(X)
#undef X
  return nullptr;
}

}  // namespace phl
