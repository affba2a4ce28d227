// phl_kernels.cuh -- stage kernels of the explicit FV step on the device-resident SoA domain.
//
// Device layout (no ghost cells are stored; ghost values are produced by index mapping):
//   W[iv][c]   primitive variables (full values), c = i + nx*(j + ny*k), ping-ponged per stage
//   U0, U      conserved state at the step start and the running RK state
//   eint, temp internal energy density and temperature (in place, own cell only)
//   gam[2][c]  (gammae, gammac) for USE_FASTEOS, ping-ponged with W
//   background fields (eq_prim, eq_gammae, phi, grav) either full arrays or profiles along x2
//   MHD: face fields bf[d] (interior faces only), b0f, face EMFs/signs, corner EMFs, bcc[3][c]
//
// The kernels take `Prm` by value.  Arithmetic follows source/source.F90 operation by operation
// so that the FP64 instantiation (compiled with --fmad=false) reproduces the reference.
#pragma once
#include <cuda_bf16.h>
#include "phl_device.cuh"

namespace phl {

// FAST_: USE_FASTEOS (gamma_e, gamma_c reconstructed to the faces); without it the Helmholtz
// configurations evaluate helm_rhoP_given per Riemann side from the face temperature guess
// SF_: USE_SHOCK_FLATTENING (shock detector, LIM2ND PLM in flagged cells, HLL on their faces)
template <int DIM_, int NV_, bool MHD_, bool HELM_, bool WB_, bool ETOT_, bool GRAV_, int RIEM_, bool FAST_ = HELM_,
          int REC_ = REC_LIM2ND, bool SF_ = false>
struct Cfg {
  static constexpr int DIM = DIM_, NV = NV_, RIEM = RIEM_, REC = REC_;
  static constexpr bool SF = SF_;
  // cells on each side of a face the reconstruction reads (3 for LIM5TH, 2 otherwise)
  static constexpr int SW = REC_ == REC_LIM5TH ? 3 : 2;
  static constexpr bool MHD = MHD_, HELM = HELM_, WB = WB_, ETOT = ETOT_, GRAV = GRAV_, FAST = HELM_ && FAST_;
  static constexpr int EOSM = !HELM_ ? EOS_IDEAL : (FAST_ ? EOS_FAST : EOS_GIVEN);
  static constexpr int IP = 1 + DIM, IAS = 2 + DIM;
  static_assert(!HELM || NV >= IAS + 2, "Helmholtz needs ADVECT_YE_IABAR scalars");
  // Resident blocks of 128 threads per SM that the register budgets of the face and cons->prim
  // kernels are sized for.  These kernels wait mostly on gathers and FP64 dependency chains and
  // run faster with more warps resident, even with a few registers spilled to L1 (measured on
  // B200 for the Helmholtz boxes); the variants whose inlined EoS or fifth-order stencil would
  // spill kilobytes keep the compiler's own budget (1).
  static constexpr int MINB_FACE64 = (EOSM == EOS_GIVEN || REC_ == REC_LIM5TH) ? 1 : 6;
  static constexpr int MINB_C2P64 = HELM_ ? 4 : 1;
  static constexpr int MINB_FACE32 = (EOSM == EOS_GIVEN || REC_ == REC_LIM5TH) ? 1 : 8;
  static constexpr int MINB_C2P32 = HELM_ ? 6 : 1;
};

struct MlpSmall;

struct Prm {
  Geo g;
  const double *__restrict__ Win;
  double *Wout;
  double *U, *U0, *eint, *temp;
  const double *__restrict__ gin;
  double *gout;
  // background (cell-centred: full N or profile ny; faces: full or profile)
  const double *eq_rho_cc, *eq_p_cc, *eq_ge_cc, *phi_cc, *grav;
  const double *eq_rho_f[3], *eq_p_f[3], *eq_ge_f[3], *phi_f[3];
  // MHD
  const double *bcc_in;
  double *bcc_out;
  double *bf[3], *b0f[3], *emf[3], *sgnf[3], *cor[3];
  // device scalars: [0] time, [1] dt, [2] smax, [3] tmax
  double *scal;
  unsigned long long *smax_bits;
  int *active;
  unsigned long long *stat;  // see STAT_* below
  HelmTable helm;
  double a1, a2, c3;
  int first_stage, last_stage;
  // FP32 split-precision path: primitive deviations and FASTEOS gammas, ping-ponged
  const float *__restrict__ Wf_in;
  float *Wf_out;
  const float *__restrict__ gf_in;
  float *gf_out;
  // reference scales of the FP32 split path: the FP32 deviations and fluxes are kept in units
  // of rho_ref, p_ref and v_ref = sqrt(p_ref / rho_ref) so that no product leaves FP32 range
  double rho_ref, p_ref, v_ref;
  double inv_rho_ref, inv_p_ref, inv_v_ref;
  // face background of the split path in those units, FP32 (x / ref rounded once at upload)
  const float *sf_rho_f[3], *sf_p_f[3], *sf_ge_f[3], *sf_phi_f[3];
  // MHD in the split path: B in units of b_ref = sqrt(p_ref) (magnetic pressure B^2/2 in p_ref),
  // EMFs in v_ref b_ref; cell-centred B, face EMFs, mass-flux signs and corner EMFs in FP32
  double b_ref, inv_b_ref;
  float *bccf;
  float *femf[3], *fsgn[3], *fcor[3];
  float *fflux[3];  // FP32 face fluxes [NV][faces] per direction
  float *fecell;    // FP32 cell-centred -v x B [3][cells] of the stage input (split MHD)
  double *dflux[3]; // FP64 MHD face fluxes [NV][faces] per direction
  // USE_SHOCK_FLATTENING: is_flattened of the cells -1..n per dimension (index + 1, bytes),
  // the detector's marks of cells -2..n+1 (index + 2), the pressure equilibrium with its ghost
  // layers (profile along x2 or full ghosted array, ghost offset sf_G), and eps_sf
  unsigned char *sf_flag, *sf_mark;
  // learned temperature guess inside the step (eos_guess = PHL_GUESS_MLP): the trained
  // network's FP32 parameters and BF16 copy of W2, nullptr for the warm start
  const float *mlp_w;
  const __nv_bfloat16 *mlp_w2bf;
  // host copy of the network's FP32 layer-1 and layer-3 parameters, read by the host when it
  // launches the learned cons->prim kernel (never dereferenced on the device)
  const MlpSmall *mlp_small;
  float *mlp_feat, *mlp_out;  // per-cell network inputs [cells][4] and log10 T guesses (NaN: none)
  // eos_guess = PHL_GUESS_MLP_RESCUE: cells whose warm start is poor, queued by cons->prim for
  // the learned guess ([0] count, then cell indices)
  unsigned int *rescue_q;
  const double *sf_eq_p;
  int sf_G, sf_eq_profile;
  double eps_sf;
};

enum { STAT_NEWTON_CALLS = 0, STAT_NEWTON_ITERS, STAT_NEWTON_NONCONV, STAT_NEWTON_CLAMP,
       STAT_MLP_ACC, STAT_MLP_REJ, STAT_NONFINITE, STAT_GUESS_EVALS, STAT_TC_STALLED, STAT_COUNT };

__device__ __forceinline__ long long bg_cc(const Geo &g, int i, int j, int k) {
  return g.bg_profile ? (long long)j : lin(g, i, j, k);
}
// face index along d: (i,j,k) with the d coordinate in 0..nx[d]
__device__ __forceinline__ long long face_lin(const Geo &g, int d, int i, int j, int k) {
  long long n0 = g.nx[0] + (d == 0), n1 = g.nx[1] + (d == 1);
  return (long long)i + n0 * ((long long)j + n1 * (long long)k);
}
__device__ __forceinline__ long long bg_face(const Geo &g, int d, int i, int j, int k) {
  return g.bg_profile ? (long long)j : face_lin(g, d, i, j, k);
}
__device__ __forceinline__ long long nfaces(const Geo &g, int d) {
  return (long long)(g.nx[0] + (d == 0)) * (g.nx[1] + (d == 1)) * (g.nx[2] + (d == 2));
}

// warp/block max of a non-negative double, then one atomic per block (bit patterns of
// non-negative doubles order like the values)
__device__ __forceinline__ void block_max_atomic(double v, unsigned long long *dst) {
  __shared__ double red[32];
  unsigned mask = 0xffffffffu;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(mask, v, o));
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int nw = (blockDim.x + 31) >> 5;
  if (lane == 0) red[wid] = v;
  __syncthreads();
  if (wid == 0) {
    v = lane < nw ? red[lane] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(mask, v, o));
    if (lane == 0) atomicMax(dst, (unsigned long long)__double_as_longlong(v));
  }
}

__device__ __forceinline__ void block_sum_atomic(unsigned long long v, unsigned long long *dst) {
  unsigned mask = 0xffffffffu;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(mask, v, o);
  if ((threadIdx.x & 31) == 0 && v) atomicAdd(dst, v);
}

// --------------------------------------------------------------------- cell loads
// Deviation primitive state of a (possibly ghost) cell: (W - eq) for rho and p under WB,
// velocity component d negated for each mirrored dimension d.
template <class C>
__device__ __forceinline__ void load_wdev(const Prm &P, int i, int j, int k, double w[C::NV]) {
  const Geo &g = P.g;
  bool f0 = false, f1 = false, f2 = false;
  int si = map_index(i, g.nx[0], g.bc[0][0], g.bc[0][1], f0);
  int sj = map_index(j, g.nx[1], g.bc[1][0], g.bc[1][1], f1);
  int sk = C::DIM == 3 ? map_index(k, g.nx[2], g.bc[2][0], g.bc[2][1], f2) : 0;
  long long c = lin(g, si, sj, sk);
#pragma unroll
  for (int iv = 0; iv < C::NV; ++iv) w[iv] = __ldg(P.Win + (long long)iv * g.N + c);
  if (C::WB) {
    long long b = bg_cc(g, si, sj, sk);
    w[0] = w[0] - __ldg(P.eq_rho_cc + b);
    w[C::IP] = w[C::IP] - __ldg(P.eq_p_cc + b);
  }
  if (f0) w[1] = -1.0 * w[1];
  if (f1) w[2] = -1.0 * w[2];
  if (C::DIM == 3 && f2) w[3] = -1.0 * w[3];
}

template <class C>
__device__ __forceinline__ void load_gdev(const Prm &P, int i, int j, int k, double gm_[2]) {
  const Geo &g = P.g;
  bool f = false;
  int si = map_index(i, g.nx[0], g.bc[0][0], g.bc[0][1], f);
  int sj = map_index(j, g.nx[1], g.bc[1][0], g.bc[1][1], f);
  int sk = C::DIM == 3 ? map_index(k, g.nx[2], g.bc[2][0], g.bc[2][1], f) : 0;
  long long c = lin(g, si, sj, sk);
  if (!C::FAST) {
    // without USE_FASTEOS the faces need the stage input's cell temperatures (the guess of
    // helm_rhoP_given); they ride in the first gamma slot, which is ping-ponged per stage
    gm_[0] = __ldg(P.gin + c);
    gm_[1] = 0.0;
    return;
  }
  gm_[0] = __ldg(P.gin + c);
  gm_[1] = __ldg(P.gin + g.N + c);
  if (C::WB) gm_[0] = gm_[0] - __ldg(P.eq_ge_cc + bg_cc(g, si, sj, sk));
}

template <class C>
__device__ __forceinline__ void load_bcc(const Prm &P, int i, int j, int k, double b[3]) {
  const Geo &g = P.g;
  bool f0 = false, f1 = false, f2 = false;
  int si = map_index(i, g.nx[0], g.bc[0][0], g.bc[0][1], f0);
  int sj = map_index(j, g.nx[1], g.bc[1][0], g.bc[1][1], f1);
  int sk = C::DIM == 3 ? map_index(k, g.nx[2], g.bc[2][0], g.bc[2][1], f2) : 0;
  long long c = lin(g, si, sj, sk);
  b[0] = __ldg(P.bcc_in + c);
  b[1] = __ldg(P.bcc_in + g.N + c);
  b[2] = C::DIM == 3 ? __ldg(P.bcc_in + 2 * g.N + c) : 0.0;
  if (f0) b[0] = -1.0 * b[0];
  if (f1) b[1] = -1.0 * b[1];
  if (C::DIM == 3 && f2) b[2] = -1.0 * b[2];
}

// The three loads above for an interior cell given by its linear index c and x2 index j (no
// mapping, no mirror)
template <class C>
__device__ __forceinline__ void load_cell_at(const Prm &P, long long c, int j, double w[C::NV], double gm_[2],
                                             double b[3]) {
  const Geo &g = P.g;
#pragma unroll
  for (int iv = 0; iv < C::NV; ++iv) w[iv] = __ldg(P.Win + (long long)iv * g.N + c);
  const long long bg = g.bg_profile ? (long long)j : c;
  if (C::WB) {
    w[0] = w[0] - __ldg(P.eq_rho_cc + bg);
    w[C::IP] = w[C::IP] - __ldg(P.eq_p_cc + bg);
  }
  if (C::HELM) {
    gm_[0] = __ldg(P.gin + c);
    gm_[1] = C::FAST ? __ldg(P.gin + g.N + c) : 0.0;
    if (C::FAST && C::WB) gm_[0] = gm_[0] - __ldg(P.eq_ge_cc + bg);
  }
  if (C::MHD) {
    b[0] = __ldg(P.bcc_in + c);
    b[1] = __ldg(P.bcc_in + g.N + c);
    b[2] = C::DIM == 3 ? __ldg(P.bcc_in + 2 * g.N + c) : 0.0;
  }
}

// --------------------------------------------------------------------- face flux
// Flux through the low face of cell `m` along d, given the deviation states of cells
// m-2..m+1 (wl2, wl1, wr1, wr2 = cells m-2, m-1, m, m+1).  Implements, for one face, the body
// of the x1/x2/x3 sweeps (source.F90:8138-9105, 9107-10301, 10303-11364).
// Left/right face values of variable iv: the right edge of cell m-1 and the left edge of cell m,
// from the cells m-3 .. m+2 (c[0] .. c[5]; the outer pair is read by LIM5TH only)
template <class C, typename R>
__device__ __forceinline__ void rec_face(const R *const c[6], int iv, bool limited, R &qL, R &qR) {
  R lo, hi;
  if (C::REC == REC_LIM2ND) {
    plm(c[1][iv], c[2][iv], c[3][iv], lo, hi);
    qL = hi;
    plm(c[2][iv], c[3][iv], c[4][iv], lo, hi);
    qR = lo;
  } else {
    const bool w5 = C::REC == REC_LIM5TH;
    rec_edges<R, C::REC>(limited, w5 ? c[0][iv] : R(0), c[1][iv], c[2][iv], c[3][iv], w5 ? c[4][iv] : R(0), lo, hi);
    qL = hi;
    rec_edges<R, C::REC>(limited, w5 ? c[1][iv] : R(0), c[2][iv], c[3][iv], c[4][iv], w5 ? c[5][iv] : R(0), lo, hi);
    qR = lo;
  }
}

// USE_SHOCK_FLATTENING: the left state of the face comes from the right edge of cell m-1
// (c[1..3]), the right state from the left edge of cell m (c[2..4]); a flagged cell gives both
// by LIM2ND PLM instead of the selected reconstruction (source.F90:8743-8827, 9635-9700,
// 10765-10830).  With LIM2ND selected nothing changes.
template <class C, typename R>
__device__ __forceinline__ void flatten_face(const R *const c[6], int iv, bool fa, bool fb, R &qL, R &qR) {
  if (C::REC == REC_LIM2ND) return;
  R lo, hi;
  if (fa) {
    plm(c[1][iv], c[2][iv], c[3][iv], lo, hi);
    qL = hi;
  }
  if (fb) {
    plm(c[2][iv], c[3][iv], c[4][iv], lo, hi);
    qR = lo;
  }
}

// fa, fb: is_flattened of cells m-1 and m (always false without USE_SHOCK_FLATTENING)
template <class C>
__device__ __forceinline__ void face_flux(const Prm &P, int d, int fi, int fj, int fk, const double *const w[6],
                                          const double *const gmv[6], const double *const bc[6], double F[C::NV],
                                          double Fb[3], double &rho_face_sum, bool fa = false, bool fb = false) {
  constexpr int NV = C::NV, IP = C::IP;
  const Geo &g = P.g;
  double qL[NV], qR[NV];
#pragma unroll
  for (int iv = 0; iv < NV; ++iv) {
    rec_face<C>(w, iv, C::REC == REC_LIM5TH || iv >= C::IAS, qL[iv], qR[iv]);
    if (C::SF) flatten_face<C>(w, iv, fa, fb, qL[iv], qR[iv]);
  }
  double bL[3] = {0, 0, 0}, bR[3] = {0, 0, 0};
  if (C::MHD) {
#pragma unroll
    for (int iv = 0; iv < C::DIM; ++iv) {
      if (iv == d) continue;
      rec_face<C>(bc, iv, C::REC == REC_LIM5TH, bL[iv], bR[iv]);
      if (C::SF) flatten_face<C>(bc, iv, fa, fb, bL[iv], bR[iv]);
    }
    double bn = P.bf[d][face_lin(g, d, fi, fj, fk)];
    bL[d] = bn;
    bR[d] = bn;
  }
  // rotation into the normal frame: x2 (v1,v2) <- (v2,-v1); x3 (v1,v2,v3) <- (v3,v1,v2)
  if (d == 1) {
    double a = qL[1], b = qL[2]; qL[1] = b; qL[2] = -a;
    a = qR[1]; b = qR[2]; qR[1] = b; qR[2] = -a;
    if (C::MHD) {
      a = bL[0]; b = bL[1]; bL[0] = b; bL[1] = -a;
      a = bR[0]; b = bR[1]; bR[0] = b; bR[1] = -a;
    }
  } else if (C::DIM == 3 && d == 2) {
    double a = qL[1], b = qL[2], c = qL[3]; qL[1] = c; qL[2] = a; qL[3] = b;
    a = qR[1]; b = qR[2]; c = qR[3]; qR[1] = c; qR[2] = a; qR[3] = b;
    if (C::MHD) {
      a = bL[0]; b = bL[1]; c = bL[2]; bL[0] = c; bL[1] = a; bL[2] = b;
      a = bR[0]; b = bR[1]; c = bR[2]; bR[0] = c; bR[1] = a; bR[2] = b;
    }
  }
  long long fbg = 0;
  if (C::WB || C::ETOT) fbg = bg_face(g, d, fi, fj, fk);
  if (C::WB) {
    double rho_eq = __ldg(P.eq_rho_f[d] + fbg), p_eq = __ldg(P.eq_p_f[d] + fbg);
    qL[0] = qL[0] + rho_eq;
    qR[0] = qR[0] + rho_eq;
    qL[IP] = qL[IP] + p_eq;
    qR[IP] = qR[IP] + p_eq;
  }
  double gL[2] = {0, 0}, gR[2] = {0, 0};
  if (C::FAST) {
    // the x1 sweep flattens the gammas after the WB add-back, x2 and x3 before it
    const bool late = C::SF && C::WB && d == 0;
#pragma unroll
    for (int iv = 0; iv < 2; ++iv) {
      rec_face<C>(gmv, iv, C::REC == REC_LIM5TH, gL[iv], gR[iv]);
      if (C::SF && !late) flatten_face<C>(gmv, iv, fa, fb, gL[iv], gR[iv]);
    }
    if (C::WB) {
      double ge = __ldg(P.eq_ge_f[d] + fbg);
      gL[0] = gL[0] + ge;
      gR[0] = gR[0] + ge;
      if (late) {
        // x1 sweep (source.F90:8829-8872), reproduced as written: a flagged cell's PLM gammas
        // replace its edge values without the equilibrium gamma_e, and eq_gammae_x1 of the
        // face is added once more to the value on the other side; cell m-1 before cell m
        double lo, hi;
        if (fa) {
#pragma unroll
          for (int iv = 0; iv < 2; ++iv) {
            plm(gmv[1][iv], gmv[2][iv], gmv[3][iv], lo, hi);
            gL[iv] = hi;
          }
          gR[0] = gR[0] + ge;
        }
        if (fb) {
#pragma unroll
          for (int iv = 0; iv < 2; ++iv) {
            plm(gmv[2][iv], gmv[3][iv], gmv[4][iv], lo, hi);
            gR[iv] = lo;
          }
          gL[0] = gL[0] + ge;
        }
      }
    }
  } else if (C::HELM) {
    // Helmholtz without USE_FASTEOS: helm_rhoP_given on each side of the face from the guess
    // 1/2 (T(m-1) + T(m)) (source.F90:8488-8495, 15705-15720, 15777-15781); passes rho*e and c
    const double tface = 0.5 * (gmv[2][0] + gmv[3][0]);
    double *gs[2] = {gL, gR};
    const double *qs[2] = {qL, qR};
#pragma unroll
    for (int side = 0; side < 2; ++side) {
      const double *q = qs[side];
      const double ye = q[C::IAS], abar = 1.0 / q[C::IAS + 1], zbar = ye * abar;
      helm_side_eos_inl(P.helm, q[0], q[IP], abar, zbar, tface, gs[side][0], gs[side][1]);
    }
  }
  const double gm = P.g.gm, mc = P.g.mach_cutoff;
  if (C::MHD) {
    riemann_mhd<double, C::DIM, NV, C::EOSM, C::RIEM>(qL, qR, bL, bR, gL, gR, gm, mc, F, Fb, C::SF && (fa || fb),
                                                      g.all_mach != 0);
  } else {
    riemann_hydro<double, C::DIM, NV, C::EOSM, C::RIEM>(qL, qR, gL, gR, gm, mc, F, C::SF && (fa || fb),
                                                        g.all_mach != 0);
  }
  // back to the lab frame
  if (d == 1) {
    double a = F[1], b = F[2]; F[1] = -b; F[2] = a;
    if (C::MHD) { a = Fb[0]; b = Fb[1]; Fb[0] = -b; Fb[1] = a; }
  } else if (C::DIM == 3 && d == 2) {
    double a = F[1], b = F[2], c = F[3]; F[1] = b; F[2] = c; F[3] = a;
    if (C::MHD) { a = Fb[0]; b = Fb[1]; c = Fb[2]; Fb[0] = b; Fb[1] = c; Fb[2] = a; }
  }
  rho_face_sum = qL[0] + qR[0];
  // MHD: the EMF/sign are taken before the WB momentum fix (source.F90:8926-8959)
  if (C::WB) F[1 + d] = F[1 + d] - __ldg(P.eq_p_f[d] + fbg);
  if (C::ETOT) F[IP] = F[IP] + F[0] * __ldg(P.phi_f[d] + fbg);
}

// EMF components of a face flux and the mass-flux sign (source.F90:8926-8951)
template <class C>
__device__ __forceinline__ void store_face_emf(const Prm &P, int d, long long fidx, const double Fb[3],
                                               double frho, double rho_face_sum, double smax) {
  const Geo &g = P.g;
  long long nf = nfaces(g, d);
  double *e = P.emf[d];
  if (d == 0) { if (C::DIM == 3) e[1 * nf + fidx] = Fb[2]; e[2 * nf + fidx] = -Fb[1]; }
  if (d == 1) { if (C::DIM == 3) e[0 * nf + fidx] = -Fb[2]; e[2 * nf + fidx] = Fb[0]; }
  if (d == 2) { e[0 * nf + fidx] = Fb[1]; e[1 * nf + fidx] = -Fb[0]; }
  double tmp = 0.5 * rho_face_sum * smax;
  double mach = frho / tmp, sgn = 0.0;
  if (mach > g.mach_ct) sgn = 1.0;
  if (mach < -g.mach_ct) sgn = -1.0;
  P.sgnf[d][fidx] = sgn;
}

// Every kernel below is a template that two translation units instantiate (the FP64 unit,
// compiled without FMA contraction, and the FP32 split unit, compiled with contraction and
// approximate division).  The host stub of a template kernel is a weak symbol: if both units
// instantiated the same kernel under the same name, the linker would keep one stub for two
// device images and the image that runs would depend on module load order.  Each unit therefore
// defines PHL_KERNEL_UNIT to its own name before including this header, which puts its
// instantiations into a namespace of its own (inline, so the code below names them as phl::).
#ifndef PHL_KERNEL_UNIT
#error "define PHL_KERNEL_UNIT (the including translation unit's kernel namespace) before including phl_kernels.cuh"
#endif
inline namespace PHL_KERNEL_UNIT {

// --------------------------------------------------------------------- shock detector
// USE_SHOCK_FLATTENING (source.F90:8073-8136).  is_flattened is kept for cells -1..n of every
// dimension (the cells whose edges the faces read), the detector's marks for cells -2..n+1.
template <class C>
__device__ __forceinline__ long long sf_flag_index(const Geo &g, int i, int j, int k) {
  return (long long)(i + 1) + (long long)(g.nx[0] + 2) * ((long long)(j + 1) + (long long)(g.nx[1] + 2) * (C::DIM == 3 ? k + 1 : 0));
}
template <class C>
__host__ __device__ __forceinline__ long long sf_flag_cells(const Geo &g) {
  return (long long)(g.nx[0] + 2) * (g.nx[1] + 2) * (C::DIM == 3 ? g.nx[2] + 2 : 1);
}
template <class C>
__host__ __device__ __forceinline__ long long sf_mark_cells(const Geo &g) {
  return (long long)(g.nx[0] + 4) * (g.nx[1] + 4) * (C::DIM == 3 ? g.nx[2] + 4 : 1);
}

// full pressure of a (possibly ghost) cell as the reference forms it: the communicated
// deviation plus the equilibrium stored for that ghost cell under WB
template <class C>
__device__ __forceinline__ double sf_pressure(const Prm &P, int i, int j, int k) {
  const Geo &g = P.g;
  bool f = false;
  int si = map_index(i, g.nx[0], g.bc[0][0], g.bc[0][1], f);
  int sj = map_index(j, g.nx[1], g.bc[1][0], g.bc[1][1], f);
  int sk = C::DIM == 3 ? map_index(k, g.nx[2], g.bc[2][0], g.bc[2][1], f) : 0;
  double p = __ldg(P.Win + (long long)C::IP * g.N + lin(g, si, sj, sk));
  if (C::WB) {
    p = p - __ldg(P.eq_p_cc + bg_cc(g, si, sj, sk));
    const int G = P.sf_G, G3 = C::DIM == 3 ? P.sf_G : 0;
    long long e = P.sf_eq_profile ? (long long)(j + G)
                                  : (long long)(i + G) + (long long)(g.nx[0] + 2 * G) *
                                        ((long long)(j + G) + (long long)(g.nx[1] + 2 * G) * (k + G3));
    p = p + __ldg(P.sf_eq_p + e);
  }
  return p;
}

// marks: summed central pressure jumps over all directions > eps_sf * p, cells -2..n+1
template <class C>
__global__ void __launch_bounds__(256) k_sf_mark(Prm P) {
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
    tmp = (fabs(sf_pressure<C>(P, i, j, k + 1) - sf_pressure<C>(P, i, j, k - 1)) +
           fabs(sf_pressure<C>(P, i, j + 1, k) - sf_pressure<C>(P, i, j - 1, k)) +
           fabs(sf_pressure<C>(P, i + 1, j, k) - sf_pressure<C>(P, i - 1, j, k))) /
          sf_pressure<C>(P, i, j, k);
  else
    tmp = (fabs(sf_pressure<C>(P, i, j + 1, k) - sf_pressure<C>(P, i, j - 1, k)) +
           fabs(sf_pressure<C>(P, i + 1, j, k) - sf_pressure<C>(P, i - 1, j, k))) /
          sf_pressure<C>(P, i, j, k);
  P.sf_mark[t] = tmp > P.eps_sf ? 1 : 0;
}

// is_flattened of cells -1..n: a mark anywhere in the 3x3(x3) neighbourhood
template <class C>
__global__ void __launch_bounds__(256) k_sf_flag(Prm P) {
  if (!*P.active) return;
  const Geo &g = P.g;
  const long long n = sf_flag_cells<C>(g);
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int f0 = g.nx[0] + 2, f1 = g.nx[1] + 2, m0 = g.nx[0] + 4, m1 = g.nx[1] + 4;
  int i, j, k;
  unflatten3(t, f0, f1, i, j, k);
  i -= 1;
  j -= 1;
  k = C::DIM == 3 ? k - 1 : 0;
  unsigned char any = 0;
#pragma unroll
  for (int c = (C::DIM == 3 ? -1 : 0); c <= (C::DIM == 3 ? 1 : 0); ++c)
#pragma unroll
    for (int b = -1; b <= 1; ++b)
#pragma unroll
      for (int a = -1; a <= 1; ++a)
        any |= P.sf_mark[(long long)(i + a + 2) + (long long)m0 * ((long long)(j + b + 2) +
                                                                   (long long)m1 * (C::DIM == 3 ? k + c + 2 : 0))];
  P.sf_flag[t] = any;
}

// --------------------------------------------------------------------- face fluxes
// One thread per face of direction d: the face flux of the x1/x2/x3 sweeps (source.F90:8138-9105,
// 9107-10301, 10303-11364), stored in P.dflux[d] for the divergence of k_c2p; for MHD also the
// face EMF and CT sign.  Each face is solved once; with --fmad=false the result equals what a
// per-cell loop over both faces of every cell computes.
template <class C, int D>
__global__ void __launch_bounds__(128, C::MINB_FACE64) k_face(Prm P) {
  constexpr int d = D;  // one instantiation per direction: strides and rotations fold
  if (!*P.active) return;
  constexpr int NV = C::NV;
  const Geo &g = P.g;
  const long long nf = nfaces(g, d);
  const long long f = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= nf) return;
  const int n0 = g.nx[0] + (d == 0), n1 = g.nx[1] + (d == 1);
  int fi, fj, fk;
  unflatten3(f, n0, n1, fi, fj, fk);
  // cells m-3 .. m+2 around the face (the reconstruction reads m-SW .. m+SW-1); a stencil inside
  // the domain is read by linear index, one at a boundary maps each ghost index
  double w[6][NV], gmv[6][2], bc[6][3];
  const int fd = d == 0 ? fi : (d == 1 ? fj : fk);
  const bool inside = fd >= C::SW && fd + C::SW <= g.nx[d];
  const long long base = lin(g, fi, fj, fk);
  const long long stride = d == 0 ? 1 : (d == 1 ? (long long)g.nx[0] : (long long)g.nx[0] * g.nx[1]);
#pragma unroll
  for (int s = 0; s < 6; ++s) {
    gmv[s][0] = gmv[s][1] = 0.0;
    bc[s][0] = bc[s][1] = bc[s][2] = 0.0;
    if (s < 3 - C::SW || s >= 3 + C::SW) {
#pragma unroll
      for (int iv = 0; iv < NV; ++iv) w[s][iv] = 0.0;
      continue;
    }
    if (inside) {
      load_cell_at<C>(P, base + (s - 3) * stride, fj + (d == 1 ? s - 3 : 0), w[s], gmv[s], bc[s]);
      continue;
    }
    const int ii = fi + (d == 0 ? s - 3 : 0), jj = fj + (d == 1 ? s - 3 : 0), kk = fk + (d == 2 ? s - 3 : 0);
    load_wdev<C>(P, ii, jj, kk, w[s]);
    if (C::HELM) load_gdev<C>(P, ii, jj, kk, gmv[s]);
    if (C::MHD) load_bcc<C>(P, ii, jj, kk, bc[s]);
  }
  const double *const wp[6] = {w[0], w[1], w[2], w[3], w[4], w[5]};
  const double *const gp[6] = {gmv[0], gmv[1], gmv[2], gmv[3], gmv[4], gmv[5]};
  const double *const bp[6] = {bc[0], bc[1], bc[2], bc[3], bc[4], bc[5]};
  bool fa = false, fb = false;
  if (C::SF) {
    fa = P.sf_flag[sf_flag_index<C>(g, fi - (d == 0), fj - (d == 1), fk - (d == 2))] != 0;
    fb = P.sf_flag[sf_flag_index<C>(g, fi, fj, fk)] != 0;
  }
  double F[NV], Fb[3], rs;
  face_flux<C>(P, d, fi, fj, fk, wp, gp, bp, F, Fb, rs, fa, fb);
#pragma unroll
  for (int iv = 0; iv < NV; ++iv) P.dflux[d][(long long)iv * nf + f] = F[iv];
  if (C::MHD) store_face_emf<C>(P, d, f, Fb, F[0], rs, P.scal[2]);
}

// --------------------------------------------------------------------- MHD: corner EMFs
// Face EMF / sign of a face array along `d` at a possibly-ghost transverse index
// (periodic wrap, or the reflective EMF BC: component == wall normal keeps its sign, the
// others flip; source.F90:11374-11964).
template <class C>
__device__ __forceinline__ void face_emf_at(const Prm &P, int d, int comp, int i, int j, int k, double &e,
                                            double &sgn) {
  const Geo &g = P.g;
  int c[3] = {i, j, k};
  double fac = 1.0;
#pragma unroll
  for (int d2 = 0; d2 < C::DIM; ++d2) {
    if (d2 == d) continue;
    int n = g.nx[d2];
    if (c[d2] < 0) {
      if (g.bc[d2][0] == BC_PERIODIC) c[d2] += n;
      else { c[d2] = 0; if (comp != d2) fac = -1.0 * fac; }
    } else if (c[d2] >= n) {
      if (g.bc[d2][1] == BC_PERIODIC) c[d2] -= n;
      else { c[d2] = n - 1; if (comp != d2) fac = -1.0 * fac; }
    }
  }
  long long f = face_lin(g, d, c[0], c[1], c[2]);
  e = fac * P.emf[d][(long long)comp * nfaces(g, d) + f];
  sgn = P.sgnf[d][f];
}

template <class C>
__device__ __forceinline__ double emf_cell(const Prm &P, int a, int i, int j, int k) {
  const Geo &g = P.g;
  bool f0 = false, f1 = false, f2 = false;
  int si = map_index(i, g.nx[0], g.bc[0][0], g.bc[0][1], f0);
  int sj = map_index(j, g.nx[1], g.bc[1][0], g.bc[1][1], f1);
  int sk = C::DIM == 3 ? map_index(k, g.nx[2], g.bc[2][0], g.bc[2][1], f2) : 0;
  long long c = lin(g, si, sj, sk);
  double v[3], b[3];
  v[0] = P.Win[g.N + c];
  v[1] = P.Win[2 * g.N + c];
  v[2] = C::DIM == 3 ? P.Win[3 * g.N + c] : 0.0;
  b[0] = P.bcc_in[c];
  b[1] = P.bcc_in[g.N + c];
  b[2] = C::DIM == 3 ? P.bcc_in[2 * g.N + c] : 0.0;
  if (f0) { v[0] = -1.0 * v[0]; b[0] = -1.0 * b[0]; }
  if (f1) { v[1] = -1.0 * v[1]; b[1] = -1.0 * b[1]; }
  if (f2) { v[2] = -1.0 * v[2]; b[2] = -1.0 * b[2]; }
  if (a == 2) return -v[0] * b[1] + v[1] * b[0];
  if (a == 0) return v[2] * b[1] - v[1] * b[2];
  return v[0] * b[2] - v[2] * b[0];
}

// corner EMF along axis a (source.F90:11966-12206); one thread per corner
template <class C, int A>
__global__ void __launch_bounds__(256) k_corner(Prm P) {
  constexpr int a = A;  // one instantiation per corner axis
  if (!*P.active) return;
  const Geo &g = P.g;
  int pa, qa;
  if (a == 2) { pa = 0; qa = 1; } else if (a == 0) { pa = 1; qa = 2; } else { pa = 2; qa = 0; }
  int n0 = g.nx[0] + (a != 0), n1 = g.nx[1] + (a != 1), n2 = C::DIM == 3 ? g.nx[2] + (a != 2) : 1;
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)n0 * n1 * n2) return;
  int c[3];
  unflatten3(t, n0, n1, c[0], c[1], c[2]);
  int cqm[3] = {c[0], c[1], c[2]}; cqm[qa] -= 1;
  int cpm[3] = {c[0], c[1], c[2]}; cpm[pa] -= 1;
  int cpq[3] = {c[0], c[1], c[2]}; cpq[pa] -= 1; cpq[qa] -= 1;
  double emf_N, emf_E, emf_S, emf_W, s_dummy;
  double sgS, sgN, sgW, sgE;
  face_emf_at<C>(P, pa, a, c[0], c[1], c[2], emf_N, sgN);
  face_emf_at<C>(P, qa, a, c[0], c[1], c[2], emf_E, sgE);
  face_emf_at<C>(P, pa, a, cqm[0], cqm[1], cqm[2], emf_S, sgS);
  face_emf_at<C>(P, qa, a, cpm[0], cpm[1], cpm[2], emf_W, sgW);
  (void)s_dummy;
  double emf_SW = emf_cell<C>(P, a, cpq[0], cpq[1], cpq[2]);
  double emf_NW = emf_cell<C>(P, a, cpm[0], cpm[1], cpm[2]);
  double emf_NE = emf_cell<C>(P, a, c[0], c[1], c[2]);
  double emf_SE = emf_cell<C>(P, a, cqm[0], cqm[1], cqm[2]);
  double sgn = sgS;
  double demf_S = 0.5 * (1.0 + sgn) * (emf_W - emf_SW) + 0.5 * (1.0 - sgn) * (emf_E - emf_SE);
  sgn = sgN;
  double demf_N = 0.5 * (1.0 + sgn) * (emf_NW - emf_W) + 0.5 * (1.0 - sgn) * (emf_NE - emf_E);
  sgn = sgW;
  double demf_W = 0.5 * (1.0 + sgn) * (emf_S - emf_SW) + 0.5 * (1.0 - sgn) * (emf_N - emf_NW);
  sgn = sgE;
  double demf_E = 0.5 * (1.0 + sgn) * (emf_SE - emf_S) + 0.5 * (1.0 - sgn) * (emf_NE - emf_N);
  P.cor[a][t] = 0.25 * (emf_S + emf_W + emf_N + emf_E + demf_S - demf_N + demf_W - demf_E);
}

__device__ __forceinline__ long long cor_lin(const Geo &g, int a, int i, int j, int k) {
  long long n0 = g.nx[0] + (a != 0), n1 = g.nx[1] + (a != 1);
  return (long long)i + n0 * ((long long)j + n1 * (long long)k);
}

// face-B update (source.F90:12208-12437); one thread per face of direction d
template <class C, int D>
__global__ void __launch_bounds__(256) k_bface(Prm P) {
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
  const double a1 = P.a1, a2 = P.a2, a3 = P.c3 * dt;
  const double *E1 = P.cor[0], *E2 = P.cor[1], *E3 = P.cor[2];
  double tmp;
  if (d == 0) {
    if (C::DIM == 2) tmp = (E3[cor_lin(g, 2, i, j + 1, k)] - E3[cor_lin(g, 2, i, j, k)]) * g.inv_dx[1];
    else tmp = -(E2[cor_lin(g, 1, i, j, k + 1)] - E2[cor_lin(g, 1, i, j, k)]) * g.inv_dx[2] +
               (E3[cor_lin(g, 2, i, j + 1, k)] - E3[cor_lin(g, 2, i, j, k)]) * g.inv_dx[1];
  } else if (d == 1) {
    if (C::DIM == 2) tmp = (E3[cor_lin(g, 2, i, j, k)] - E3[cor_lin(g, 2, i + 1, j, k)]) * g.inv_dx[0];
    else tmp = (E1[cor_lin(g, 0, i, j, k + 1)] - E1[cor_lin(g, 0, i, j, k)]) * g.inv_dx[2] +
               (E3[cor_lin(g, 2, i, j, k)] - E3[cor_lin(g, 2, i + 1, j, k)]) * g.inv_dx[0];
  } else {
    tmp = (E2[cor_lin(g, 1, i + 1, j, k)] - E2[cor_lin(g, 1, i, j, k)]) * g.inv_dx[0] -
          (E1[cor_lin(g, 0, i, j + 1, k)] - E1[cor_lin(g, 0, i, j, k)]) * g.inv_dx[1];
  }
  double b = P.bf[d][t];
  double b0;
  if (P.first_stage) { b0 = b; P.b0f[d][t] = b; } else { b0 = P.b0f[d][t]; }
  P.bf[d][t] = a1 * b0 + a2 * b + a3 * tmp;
}

// Stage end: flux divergence of the face fluxes, gravity and the RK combine of U
// (source.F90:9057-9102, 12606-12644, 13518-13531), b_cc from the updated faces, then
// cons->prim with the EoS (source.F90:12439-12487, 13533-13686), last stage also the CFL max
template <class C>
__global__ void __launch_bounds__(128, C::MINB_C2P64) k_c2p(Prm P) {
  if (!*P.active) return;
  constexpr int NV = C::NV, IP = C::IP, IAS = C::IAS, DIM = C::DIM;
  const Geo &g = P.g;
  long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  double smax_loc = 0.0;
  unsigned long long n_calls = 0, n_iters = 0, n_nonconv = 0, n_clamp = 0, n_bad = 0;
  if (c < g.N) {
    int i, j, k;
    unflatten3(c, g.nx[0], g.nx[1], i, j, k);
    double bcc[3] = {0, 0, 0};
    if (C::MHD) {
#pragma unroll
      for (int d = 0; d < DIM; ++d) {
        int ui = i + (d == 0), uj = j + (d == 1), uk = k + (d == 2);
        bcc[d] = 0.5 * (P.bf[d][face_lin(g, d, ui, uj, uk)] + P.bf[d][face_lin(g, d, i, j, k)]);
      }
    }
    // flux divergence of the face fluxes (directions in order), gravity and the RK combine
    double res[NV];
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
      const long long nf = nfaces(g, d);
      const long long flo = face_lin(g, d, i, j, k), fhi = face_lin(g, d, i + (d == 0), j + (d == 1), k + (d == 2));
      const double inv_dl = g.inv_dx[d];
#pragma unroll
      for (int iv = 0; iv < NV; ++iv) {
        double dd = (P.dflux[d][(long long)iv * nf + fhi] - P.dflux[d][(long long)iv * nf + flo]) * inv_dl;
        res[iv] = d == 0 ? dd : res[iv] + dd;
      }
    }
    double w[NV];
#pragma unroll
    for (int iv = 0; iv < NV; ++iv) w[iv] = P.Win[(long long)iv * g.N + c];
    if (C::GRAV) {
      const long long b = bg_cc(g, i, j, k);
      const double rho_dev = C::WB ? w[0] - __ldg(P.eq_rho_cc + b) : w[0];
#pragma unroll
      for (int d = 0; d < DIM; ++d)
        res[1 + d] = res[1 + d] - rho_dev * __ldg(P.grav + (long long)d * (g.bg_profile ? g.nx[1] : g.N) + b);
    }
    double u0[NV], u[NV];
    if (P.first_stage) {
      double rho0 = w[0], vx1 = w[1], vx2 = w[2], vx3 = DIM == 3 ? w[3] : 0.0;
      u0[0] = rho0;
      u0[1] = rho0 * vx1;
      u0[2] = rho0 * vx2;
      if (DIM == 3) u0[3] = rho0 * vx3;
      double rhoe0 = P.eint[c] + 0.5 * rho0 * (vx1 * vx1 + vx2 * vx2 + vx3 * vx3);
      if (C::MHD) {
        // magnetic energy of the stage input (b_cc before this stage's face update)
        double b0 = P.bcc_in[c], b1 = P.bcc_in[g.N + c], b2 = DIM == 3 ? P.bcc_in[2 * g.N + c] : 0.0;
        rhoe0 = rhoe0 + 0.5 * (b0 * b0 + b1 * b1 + b2 * b2);
      }
      if (C::ETOT) rhoe0 = rhoe0 + rho0 * __ldg(P.phi_cc + bg_cc(g, i, j, k));
      u0[IP] = rhoe0;
#pragma unroll
      for (int iv = IAS; iv < NV; ++iv) u0[iv] = rho0 * w[iv];
#pragma unroll
      for (int iv = 0; iv < NV; ++iv) { u[iv] = u0[iv]; P.U0[(long long)iv * g.N + c] = u0[iv]; }
    } else {
#pragma unroll
      for (int iv = 0; iv < NV; ++iv) {
        u0[iv] = P.U0[(long long)iv * g.N + c];
        u[iv] = P.U[(long long)iv * g.N + c];
      }
    }
    if (g.use_acc) constant_acceleration<DIM, IP>(g, u, res);
    {
      const double a1 = P.a1, a2 = P.a2, a3 = P.c3 * P.scal[1];
#pragma unroll
      for (int iv = 0; iv < NV; ++iv) {
        u[iv] = a1 * u0[iv] + a2 * u[iv] + a3 * res[iv];
        P.U[(long long)iv * g.N + c] = u[iv];
      }
    }
    // the stage input's b_cc has been read: store the new one
    if (C::MHD)
#pragma unroll
      for (int d = 0; d < DIM; ++d) P.bcc_out[(long long)d * g.N + c] = bcc[d];
    double rho = u[0], rhovx1 = u[1], rhovx2 = u[2], rhovx3 = DIM == 3 ? u[3] : 0.0, rhoe = u[IP];
    double inv_rho = 1.0 / rho;
    double eint = rhoe - 0.5 * (rhovx1 * rhovx1 + rhovx2 * rhovx2 + rhovx3 * rhovx3) * inv_rho;
    if (C::MHD) eint = eint - 0.5 * (bcc[0] * bcc[0] + bcc[1] * bcc[1] + bcc[2] * bcc[2]);
    if (C::ETOT) eint = eint - rho * __ldg(P.phi_cc + bg_cc(g, i, j, k));
    double wn[NV];
    wn[0] = rho;
    wn[1] = rhovx1 * inv_rho;
    wn[2] = rhovx2 * inv_rho;
    if (DIM == 3) wn[3] = rhovx3 * inv_rho;
    double p, T, sound = 0.0;
    if (C::HELM) {
      double ye = u[IAS] * inv_rho;
      double abar = rho / u[IAS + 1];
      double zbar = ye * abar;
      T = P.temp[c];
      int clamped = 0;
      int it = helm_rhoe_newton(P.helm, rho, eint * inv_rho, abar, zbar, T, 100, clamped);
      n_calls += 1; n_iters += it; n_nonconv += (it == 100); n_clamp += clamped;
      double E, cv;
      helm_given_full(P.helm, rho, T, abar, zbar, p, E, sound, cv);
      if (C::FAST) {
        P.gout[c] = p / eint + 1.0;
        P.gout[g.N + c] = sound * sound * rho / p;
      } else {
        P.gout[c] = T;
      }
    } else {
      p = (g.gm - 1.0) * eint;
      T = p / (rho * CONST_RGAS * (1.0 / g.mu));
    }
    wn[IP] = p;
#pragma unroll
    for (int iv = IAS; iv < NV; ++iv) wn[iv] = u[iv] * inv_rho;
#pragma unroll
    for (int iv = 0; iv < NV; ++iv) P.Wout[(long long)iv * g.N + c] = wn[iv];
    P.temp[c] = T;
    P.eint[c] = eint;
    if (!(rho > 0.0) || !(p > 0.0) || !(T > 0.0) || !isfinite(eint)) n_bad += 1;
    if (P.last_stage) {
      double cs;
      if (C::HELM) {
        double ye = wn[IAS], abar = 1.0 / wn[IAS + 1], zbar = ye * abar, pp, ei, cv;
        helm_given_full(P.helm, rho, T, abar, zbar, pp, ei, cs, cv);
      } else {
        cs = sqrt(g.gm * p / rho);
      }
      if (C::MHD) {
        double ca2 = bcc[0] * bcc[0] + bcc[1] * bcc[1] + bcc[2] * bcc[2];
        cs = sqrt(cs * cs + ca2 / rho);
      }
      double sx1 = (fabs(wn[1]) + cs) * g.inv_dx[0];
      double sx2 = (fabs(wn[2]) + cs) * g.inv_dx[1];
      if (DIM == 3) {
        double sx3 = (fabs(wn[3]) + cs) * g.inv_dx[2];
        smax_loc = sx3 + sx1 + sx2;
      } else {
        smax_loc = sx1 + sx2;
      }
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

// --------------------------------------------------------------------- dt (step 0)
template <class C>
__global__ void __launch_bounds__(256) k_dt(Prm P) {
  constexpr int IP = C::IP, IAS = C::IAS, DIM = C::DIM;
  const Geo &g = P.g;
  long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  double s = 0.0;
  if (c < g.N) {
    const double *W = P.Win;
    double rho = W[c], vx1 = W[g.N + c], vx2 = W[2 * g.N + c], vx3 = DIM == 3 ? W[3 * g.N + c] : 0.0;
    double p = W[(long long)IP * g.N + c], cs;
    if (C::HELM) {
      double ye = W[(long long)IAS * g.N + c], abar = 1.0 / W[(long long)(IAS + 1) * g.N + c];
      double zbar = ye * abar, T = P.temp[c], ei, cv;
      helm_given_full(P.helm, rho, T, abar, zbar, p, ei, cs, cv);
    } else {
      cs = sqrt(g.gm * p / rho);
    }
    if (C::MHD) {
      double b0 = P.bcc_in[c], b1 = P.bcc_in[g.N + c], b2 = DIM == 3 ? P.bcc_in[2 * g.N + c] : 0.0;
      double ca2 = b0 * b0 + b1 * b1 + b2 * b2;
      cs = sqrt(cs * cs + ca2 / rho);
    }
    double sx1 = (fabs(vx1) + cs) * g.inv_dx[0];
    double sx2 = (fabs(vx2) + cs) * g.inv_dx[1];
    if (DIM == 3) {
      double sx3 = (fabs(vx3) + cs) * g.inv_dx[2];
      s = sx3 + sx1 + sx2;
    } else {
      s = sx1 + sx2;
    }
  }
  block_max_atomic(s, P.smax_bits);
}

// step-0 thermodynamics (source.F90:6271-6383) and b_cc from faces (source.F90:6012-6062)
template <class C>
__global__ void __launch_bounds__(128) k_init_thermo(Prm P) {
  constexpr int IP = C::IP, IAS = C::IAS, DIM = C::DIM;
  const Geo &g = P.g;
  long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= g.N) return;
  int i, j, k;
  unflatten3(c, g.nx[0], g.nx[1], i, j, k);
  if (C::MHD) {
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
      int ui = i + (d == 0), uj = j + (d == 1), uk = k + (d == 2);
      P.bcc_out[(long long)d * g.N + c] =
          0.5 * (P.bf[d][face_lin(g, d, ui, uj, uk)] + P.bf[d][face_lin(g, d, i, j, k)]);
    }
  }
  const double *W = P.Win;
  double rho = W[c], p = W[(long long)IP * g.N + c], eint, T;
  if (C::HELM) {
    double abar = 1.0 / W[(long long)(IAS + 1) * g.N + c];
    double ye = W[(long long)IAS * g.N + c];
    double zbar = abar * ye, sound, cv, Pdummy;
    T = P.temp[c];
    int clamped = 0;
    helm_rhoP_newton(P.helm, rho, p, abar, zbar, T, clamped);
    helm_given_full(P.helm, rho, T, abar, zbar, Pdummy, eint, sound, cv);
    eint = rho * eint;
    if (C::FAST) {
      P.gout[c] = p / eint + 1.0;
      P.gout[g.N + c] = sound * sound * rho / p;
    } else {
      P.gout[c] = T;
    }
  } else {
    T = p / (CONST_RGAS * rho * (1.0 / g.mu));
    eint = p * (1.0 / (g.gm - 1.0));
  }
  P.eint[c] = eint;
  P.temp[c] = T;
}

}  // inline namespace PHL_KERNEL_UNIT
}  // namespace phl
