// phl_runtime.cu -- host runtime and C ABI (include/phl_gpu.h) of the B200 explicit FV step.
//
// One context = one device-resident domain on one stream.  The reference-layout host arrays
// (Fortran order, ghosts included) are staged to the device in one copy each and transposed
// by kernels into the SoA layout of phl_kernels.cuh.  Steps run as CUDA graphs with dt, time and
// the CFL maximum kept on the device (time_loop body, source/source.F90:6525-6748).
#include <cuda_runtime.h>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/phl_gpu.h"
// kernel namespace of this unit (FP64, no FMA contraction); see phl_kernels.cuh
#define PHL_KERNEL_UNIT fp64_unit
#include "phl_kernels.cuh"
#include "phl_runner.h"
#include "phl_eos_batch.cuh"

using namespace phl;

namespace {

thread_local std::string g_last_error;

#define CK(call)                                                                      \
  do {                                                                                \
    cudaError_t e_ = (call);                                                          \
    if (e_ != cudaSuccess) {                                                          \
      g_last_error = std::string(#call) + ": " + cudaGetErrorString(e_);              \
      return PHL_E_CUDA;                                                              \
    }                                                                                 \
  } while (0)

inline unsigned nblk(long long n, int t) { return (unsigned)((n + t - 1) / t); }

// ----------------------------------------------------------------------------- runners
template <class C>
struct RunnerT : Runner {
  void stage(const Prm &P, cudaStream_t s) override {
    const Geo &g = P.g;
    // each face once, then (MHD) corners and face B, then divergence + RK + cons->prim per cell
    if constexpr (C::SF) {
      k_sf_mark<C><<<nblk(sf_mark_cells<C>(g), 256), 256, 0, s>>>(P);
      k_sf_flag<C><<<nblk(sf_flag_cells<C>(g), 256), 256, 0, s>>>(P);
    }
    k_face<C, 0><<<nblk(nfaces_host(g, 0), 128), 128, 0, s>>>(P);
    k_face<C, 1><<<nblk(nfaces_host(g, 1), 128), 128, 0, s>>>(P);
    if constexpr (C::DIM == 3) k_face<C, 2><<<nblk(nfaces_host(g, 2), 128), 128, 0, s>>>(P);
    if constexpr (C::MHD) {
      auto ncor = [&](int a) {
        return (long long)(g.nx[0] + (a != 0)) * (g.nx[1] + (a != 1)) * (C::DIM == 3 ? g.nx[2] + (a != 2) : 1);
      };
      if constexpr (C::DIM == 3) {
        k_corner<C, 0><<<nblk(ncor(0), 256), 256, 0, s>>>(P);
        k_corner<C, 1><<<nblk(ncor(1), 256), 256, 0, s>>>(P);
      }
      k_corner<C, 2><<<nblk(ncor(2), 256), 256, 0, s>>>(P);
      k_bface<C, 0><<<nblk(nfaces_host(g, 0), 256), 256, 0, s>>>(P);
      k_bface<C, 1><<<nblk(nfaces_host(g, 1), 256), 256, 0, s>>>(P);
      if constexpr (C::DIM == 3) k_bface<C, 2><<<nblk(nfaces_host(g, 2), 256), 256, 0, s>>>(P);
    }
    k_c2p<C><<<nblk(g.N, 128), 128, 0, s>>>(P);
  }
  void dt(const Prm &P, cudaStream_t s) override { k_dt<C><<<nblk(P.g.N, 256), 256, 0, s>>>(P); }
  void init_thermo(const Prm &P, cudaStream_t s) override {
    k_init_thermo<C><<<nblk(P.g.N, 128), 128, 0, s>>>(P);
  }
  static long long nfaces_host(const Geo &g, int d) {
    return (long long)(g.nx[0] + (d == 0)) * (g.nx[1] + (d == 1)) * (g.nx[2] + (d == 2));
  }
};

// Instantiated option sets: (dims, nvars, MHD, Helmholtz, stratified = WB+ETOT+gravity, Riemann
// solver, USE_FASTEOS, reconstruction, USE_SHOCK_FLATTENING).  Other combinations return
// PHL_E_UNSUPPORTED.
#define PHL_RUNNER_LIST(X)                                         \
  X(2, 4, false, false, false, R_LHLLC, false, REC_LIM2ND, false)  \
  X(2, 4, false, false, false, R_HLLC, false, REC_LIM2ND, false)   \
  X(2, 4, false, false, true, R_LHLLC, false, REC_LIM2ND, false)   \
  X(2, 4, false, false, true, R_HLLC, false, REC_LIM2ND, false)    \
  X(2, 4, true, false, false, R_HLLD, false, REC_LIM2ND, false)    \
  X(2, 4, true, false, false, R_LHLLD, false, REC_LIM2ND, false)   \
  X(2, 6, false, true, true, R_LHLLC, true, REC_LIM2ND, false)     \
  X(2, 6, true, true, true, R_LHLLD, true, REC_LIM2ND, false)      \
  X(3, 5, false, false, false, R_LHLLC, false, REC_LIM2ND, false)  \
  X(3, 5, false, false, false, R_HLLC, false, REC_LIM2ND, false)   \
  X(3, 5, true, false, false, R_HLLD, false, REC_LIM2ND, false)    \
  X(3, 5, true, false, false, R_LHLLD, false, REC_LIM2ND, false)   \
  X(3, 7, false, true, true, R_LHLLC, true, REC_LIM2ND, false)     \
  X(3, 7, false, true, true, R_HLLC, true, REC_LIM2ND, false)      \
  X(3, 7, true, true, true, R_LHLLD, true, REC_LIM2ND, false)      \
  X(3, 7, true, true, true, R_HLLD, true, REC_LIM2ND, false)       \
  X(3, 7, false, true, true, R_LHLLC, false, REC_LIM2ND, false)    \
  X(3, 7, false, true, true, R_HLLC, false, REC_LIM2ND, false)     \
  X(3, 7, true, true, true, R_LHLLD, false, REC_LIM2ND, false)     \
  X(2, 4, true, false, false, R_HLLD, false, REC_PPH, false)       \
  X(2, 4, true, false, false, R_HLLD, false, REC_LIM5TH, false)    \
  X(3, 7, false, true, true, R_LHLLC, true, REC_PPH, false)        \
  X(3, 7, false, true, true, R_LHLLC, true, REC_LIM5TH, false)     \
  X(3, 7, true, true, true, R_LHLLD, true, REC_PPH, false)         \
  X(3, 7, true, true, true, R_LHLLD, true, REC_LIM5TH, false)      \
  X(2, 5, false, false, false, R_HLLC, false, REC_LIM2ND, true)    \
  X(2, 5, false, false, false, R_LHLLC, false, REC_LIM2ND, true)   \
  X(2, 5, false, false, false, R_HLLC, false, REC_PPH, true)       \
  X(2, 5, false, false, false, R_HLLC, false, REC_LIM5TH, true)    \
  X(2, 4, false, false, true, R_LHLLC, false, REC_LIM2ND, true)    \
  X(2, 4, true, false, false, R_HLLD, false, REC_LIM2ND, true)     \
  X(2, 4, true, false, false, R_HLLD, false, REC_LIM5TH, true)     \
  X(3, 7, false, true, true, R_LHLLC, true, REC_LIM2ND, true)      \
  X(3, 7, false, true, true, R_LHLLC, true, REC_PPH, true)         \
  X(3, 7, false, true, true, R_LHLLC, false, REC_LIM2ND, true)     \
  X(3, 7, true, true, true, R_LHLLD, true, REC_LIM2ND, true)

Runner *make_runner(int dim, int nv, bool mhd, bool helm, bool strat, int riem, bool fast, int rec, bool sf) {
#define X(D, N, M, H, S, R, F, REC, SF)                                                                      \
  if (dim == D && nv == N && mhd == M && helm == H && strat == S && riem == R && (!H || fast == F) &&         \
      rec == REC && sf == SF)                                                                                 \
    return new RunnerT<Cfg<D, N, M, H, S, S, S, R, F, REC, SF>>();
  PHL_RUNNER_LIST(X)
#undef X
  return nullptr;
}

// dst = (float)(src / ref): the split path's FP32 copy of a background array
__global__ void k_scale_f32(const double *src, float *dst, long long n, double ref) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = (float)(src[i] / ref);
}

// ----------------------------------------------------------------------------- transposes
// host reference layout (nv, n1g, n2g, n3g) with ghost offsets -> SoA interior [nv][N]
__global__ void k_unpack(const double *src, double *dst, int nv, int nx, int ny, int nz, int n1, int n2,
                         int o1, int o2, int o3, int ncomp, long long dst_stride) {
  long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  long long N = (long long)nx * ny * nz;
  if (c >= N) return;
  int i = (int)(c % nx), j = (int)((c / nx) % ny), k = (int)(c / ((long long)nx * ny));
  long long s = (long long)nv * ((long long)(i + o1) + (long long)n1 * ((long long)(j + o2) + (long long)n2 * (k + o3)));
  for (int iv = 0; iv < ncomp; ++iv) dst[(long long)iv * dst_stride + c] = src[s + iv];
}
__global__ void k_pack(const double *src, double *dst, int nv, int nx, int ny, int nz, int n1, int n2, int o1,
                       int o2, int o3, int ncomp, long long src_stride) {
  long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  long long N = (long long)nx * ny * nz;
  if (c >= N) return;
  int i = (int)(c % nx), j = (int)((c / nx) % ny), k = (int)(c / ((long long)nx * ny));
  long long s = (long long)nv * ((long long)(i + o1) + (long long)n1 * ((long long)(j + o2) + (long long)n2 * (k + o3)));
  for (int iv = 0; iv < ncomp; ++iv) dst[s + iv] = src[(long long)iv * src_stride + c];
}

// per-step scalar bookkeeping (time_loop, source.F90:6662-6664, 6710, 6716)
__global__ void k_pre_step(double *scal, int *active, unsigned long long *smax_bits, long long *step,
                           long long step_limit) {
  double time = scal[0], dt = scal[1], tmax = scal[3];
  int a = (time < tmax) && (*step < step_limit);
  *active = a;
  if (!a) return;
  if ((time + dt) > tmax) scal[1] = tmax - time;
  *smax_bits = 0ull;
}
__global__ void k_post_step(double *scal, const int *active, const unsigned long long *smax_bits,
                            long long *step, double cfl) {
  if (!*active) return;
  scal[0] = scal[0] + scal[1];
  double smax = __longlong_as_double((long long)*smax_bits);
  scal[2] = smax;
  scal[1] = cfl / smax;
  *step = *step + 1;
}
__global__ void k_set_active(int *active, unsigned long long *smax_bits) {
  *active = 1;
  *smax_bits = 0ull;
}
__global__ void k_finish_dt(double *scal, const unsigned long long *smax_bits, double cfl) {
  double smax = __longlong_as_double((long long)*smax_bits);
  scal[2] = smax;
  scal[1] = cfl / smax;
}

}  // namespace

// ----------------------------------------------------------------------------- context
struct phl_ctx {
  phl_config cfg;
  Geo geo;
  std::unique_ptr<Runner> runner;
  // FP64 runner of the same option set: dt and step-0 thermodynamics in both precision forms
  // (the split runner's own when that is the form; a second instance otherwise)
  std::unique_ptr<Runner> fp64_runner;
  Runner *thermo() { return fp64_runner ? fp64_runner.get() : runner.get(); }
  cudaStream_t stream = nullptr;
  int dim = 2, nv = 0;
  long long N = 0;
  // dynamic
  double *W[2] = {nullptr, nullptr}, *gam[2] = {nullptr, nullptr};
  float *Wf[2] = {nullptr, nullptr}, *gf[2] = {nullptr, nullptr};  // FP32 split path
  bool split = false;
  double rho_ref = 1.0, p_ref = 1.0, v_ref = 1.0;  // FP32 split-path scales
  bool refs_set = false;
  int cur = 0;
  double *U = nullptr, *U0 = nullptr, *eint = nullptr, *temp = nullptr;
  double *bcc = nullptr;
  double *bf[3] = {}, *b0f[3] = {}, *emf[3] = {}, *sgnf[3] = {}, *cor[3] = {};
  // background
  int bg_profile = 0;
  double *eq_rho_cc = nullptr, *eq_p_cc = nullptr, *eq_ge_cc = nullptr, *phi_cc = nullptr, *grav = nullptr;
  double *eq_rho_f[3] = {}, *eq_p_f[3] = {}, *eq_ge_f[3] = {}, *phi_f[3] = {};
  float *sf_rho_f[3] = {}, *sf_p_f[3] = {}, *sf_ge_f[3] = {}, *sf_phi_f[3] = {};  // split path
  float *bccf = nullptr, *femf[3] = {}, *fsgn[3] = {}, *fcor[3] = {};                // split MHD
  float *fflux[3] = {};
  float *fecell = nullptr;                                                             // split MHD
  float *mlp_feat = nullptr, *mlp_out = nullptr;  // learned guess in the split MHD step
  unsigned *rescue_q = nullptr;                    // PHL_GUESS_MLP_RESCUE queue (count + cells)
  double *dflux[3] = {};                                                               // FP64 MHD
  // USE_SHOCK_FLATTENING: flags, detector marks, ghosted pressure equilibrium (see Prm)
  unsigned char *sf_flag = nullptr, *sf_mark = nullptr;
  double *sf_eq_p = nullptr;
  int sf_eq_profile = 0;
  // scalars
  double *scal = nullptr;
  unsigned long long *smax_bits = nullptr;
  int *active = nullptr;
  long long *step = nullptr;
  unsigned long long *stat = nullptr;
  // table
  double *htab = nullptr, *hdpd = nullptr, *hrho = nullptr, *hT = nullptr, *hirho = nullptr, *hiT = nullptr;
  HelmTable helm{};
  bool table_loaded = false, uploaded = false, bg_uploaded = false;
  // host copy of the network's FP32 layers 1 and 3 (argument of the learned cons->prim kernel)
  MlpSmall mlp_small{};
  bool mlp_small_ok = false;
  // staging
  double *stage_buf = nullptr;
  size_t stage_bytes = 0;
  // graphs: one per parity of the W ping-pong
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  // asynchronous host-state pipeline (phl_run_steps_host_async): copy streams, staging images
  // of the dynamic host arrays, and the events that order one call's uploads after the previous
  // call's downloads chunk by chunk
  struct HostSlot {
    int ncomp = 0, h1 = 0, h2 = 0, h3 = 0;  // host extents (ghosts included; h3 = 1 in 2D)
    int fx = 0, fy = 0, fz = 0;             // interior extents (cells or faces)
    int o1 = 0, o2 = 0, o3 = 0;             // offset of the interior in the host array
    double *dev = nullptr;                  // SoA device field (cells: [ncomp][N])
    long long dev_stride = 0;
    double *in = nullptr, *out = nullptr;   // staging: ghosted host image, compact interior
    int chunk0 = 0, nchunk = 0, ppc = 1;    // chunks of ppc host planes along x3
    size_t plane() const { return (size_t)ncomp * h1 * h2; }
  };
  static constexpr int HOST_SLOTS = 8;  // prim, temp, eint, gammaf, b_cc, b_x1..3
  HostSlot hslot[HOST_SLOTS];
  bool hpipe_ready = false, hpipe_pending = false;
  cudaStream_t cin = nullptr, cout = nullptr;
  std::vector<cudaEvent_t> ev_chunk_out;  // per chunk: its download has landed
  cudaEvent_t ev_in[HOST_SLOTS] = {}, ev_pack[HOST_SLOTS] = {};
  // EoS batch scratch and MLP
  EosBatch eos;
  std::vector<void *> allocs;

  ~phl_ctx() {
    for (int p = 0; p < 2; ++p)
      if (graph[p]) cudaGraphExecDestroy(graph[p]);
    eos.release();
    for (cudaEvent_t e : ev_chunk_out) cudaEventDestroy(e);
    for (int q = 0; q < HOST_SLOTS; ++q) {
      if (ev_in[q]) cudaEventDestroy(ev_in[q]);
      if (ev_pack[q]) cudaEventDestroy(ev_pack[q]);
    }
    if (cin) cudaStreamDestroy(cin);
    if (cout) cudaStreamDestroy(cout);
    for (void *a : allocs) cudaFree(a);
    if (stream) cudaStreamDestroy(stream);
  }
  // wait for the downloads of earlier asynchronous host-state calls (every entry point that
  // reads or writes caller memory runs this first)
  int drain_host() {
    if (!hpipe_pending) return PHL_OK;
    CK(cudaStreamSynchronize(cout));
    CK(cudaStreamSynchronize(stream));
    hpipe_pending = false;
    return PHL_OK;
  }
  template <class T>
  int alloc(T **p, size_t count) {
    void *q = nullptr;
    if (count == 0) count = 1;
    cudaError_t e = cudaMalloc(&q, count * sizeof(T));
    if (e != cudaSuccess) {
      g_last_error = std::string("cudaMalloc: ") + cudaGetErrorString(e);
      return PHL_E_CUDA;
    }
    cudaMemsetAsync(q, 0, count * sizeof(T), stream);
    allocs.push_back(q);
    *p = (T *)q;
    return PHL_OK;
  }
  long long nfaces(int d) const {
    return (long long)(geo.nx[0] + (d == 0)) * (geo.nx[1] + (d == 1)) * (geo.nx[2] + (d == 2));
  }
  long long ncor(int a) const {
    return (long long)(geo.nx[0] + (a != 0)) * (geo.nx[1] + (a != 1)) * (dim == 3 ? geo.nx[2] + (a != 2) : 1);
  }
  int ensure_stage(size_t bytes) {
    if (bytes <= stage_bytes) return PHL_OK;
    if (stage_buf) cudaFree(stage_buf);
    stage_buf = nullptr;
    CK(cudaMalloc(&stage_buf, bytes));
    stage_bytes = bytes;
    return PHL_OK;
  }
  Prm prm(int stage_idx) const {
    Prm P;
    memset(&P, 0, sizeof(P));
    P.g = geo;
    int in = (cur + stage_idx) & 1;
    P.Win = W[in];
    P.Wout = W[in ^ 1];
    P.gin = gam[in];
    P.gout = gam[in ^ 1];
    P.Wf_in = Wf[in];
    P.Wf_out = Wf[in ^ 1];
    P.gf_in = gf[in];
    P.gf_out = gf[in ^ 1];
    P.rho_ref = rho_ref;
    P.p_ref = p_ref;
    P.v_ref = v_ref;
    P.inv_rho_ref = 1.0 / rho_ref;
    P.inv_p_ref = 1.0 / p_ref;
    P.inv_v_ref = 1.0 / v_ref;
    P.b_ref = sqrt(p_ref);
    P.inv_b_ref = 1.0 / P.b_ref;
    P.bccf = bccf;
    P.fecell = fecell;
    P.mlp_feat = mlp_feat;
    P.mlp_out = mlp_out;
    for (int d = 0; d < 3; ++d) {
      P.femf[d] = femf[d]; P.fsgn[d] = fsgn[d]; P.fcor[d] = fcor[d]; P.fflux[d] = fflux[d];
      P.dflux[d] = dflux[d];
    }
    P.U = U;
    P.U0 = U0;
    P.eint = eint;
    P.temp = temp;
    P.eq_rho_cc = eq_rho_cc; P.eq_p_cc = eq_p_cc; P.eq_ge_cc = eq_ge_cc; P.phi_cc = phi_cc; P.grav = grav;
    for (int d = 0; d < 3; ++d) {
      P.eq_rho_f[d] = eq_rho_f[d]; P.eq_p_f[d] = eq_p_f[d]; P.eq_ge_f[d] = eq_ge_f[d]; P.phi_f[d] = phi_f[d];
      P.sf_rho_f[d] = sf_rho_f[d]; P.sf_p_f[d] = sf_p_f[d]; P.sf_ge_f[d] = sf_ge_f[d]; P.sf_phi_f[d] = sf_phi_f[d];
      P.bf[d] = bf[d]; P.b0f[d] = b0f[d]; P.emf[d] = emf[d]; P.sgnf[d] = sgnf[d]; P.cor[d] = cor[d];
    }
    P.bcc_in = bcc;
    P.bcc_out = bcc;
    if ((cfg.eos_guess == PHL_GUESS_MLP || cfg.eos_guess == PHL_GUESS_MLP_RESCUE) && eos.mlp.ready) {
      MlpWeights mw = eos.mlp.weights();
      P.mlp_w = mw.w;
      P.mlp_w2bf = mw.w2bf;
      P.mlp_small = mlp_small_ok ? &mlp_small : nullptr;
      P.rescue_q = cfg.eos_guess == PHL_GUESS_MLP_RESCUE ? rescue_q : nullptr;
    }
    P.sf_flag = sf_flag;
    P.sf_mark = sf_mark;
    P.sf_eq_p = sf_eq_p;
    P.sf_G = cfg.ngc;
    P.sf_eq_profile = sf_eq_profile;
    P.eps_sf = cfg.eps_sf;
    P.scal = scal;
    P.smax_bits = smax_bits;
    P.active = active;
    P.stat = stat;
    P.helm = helm;
    double rk[3][3] = {{1.0, 0.0, -1.0}, {0.75, 0.25, -0.25}, {1.0 / 3.0, 2.0 / 3.0, -(2.0 / 3.0)}};
    if (cfg.rk_stages == 2) {
      rk[1][0] = 0.5; rk[1][1] = 0.5; rk[1][2] = -0.5;
    }
    P.a1 = rk[stage_idx][0];
    P.a2 = rk[stage_idx][1];
    P.c3 = rk[stage_idx][2];
    P.first_stage = stage_idx == 0;
    P.last_stage = stage_idx == cfg.rk_stages - 1;
    return P;
  }
  // split path: FP64 primitives of W[cur] -> U and the FP32 deviations of Wf[cur]
  // FP32 copies of the face background in the split path's units
  int scale_background(bool helm) {
    for (int d = 0; d < dim; ++d) {
      long long nf = geo.bg_profile ? (long long)(geo.nx[1] + (d == 1)) : nfaces(d);
      int rc;
      if (!sf_rho_f[d] && ((rc = alloc(&sf_rho_f[d], nf)) || (rc = alloc(&sf_p_f[d], nf)) ||
                           (rc = alloc(&sf_phi_f[d], nf)) || (rc = alloc(&sf_ge_f[d], nf))))
        return rc;
      k_scale_f32<<<nblk(nf, 256), 256, 0, stream>>>(eq_rho_f[d], sf_rho_f[d], nf, rho_ref);
      k_scale_f32<<<nblk(nf, 256), 256, 0, stream>>>(eq_p_f[d], sf_p_f[d], nf, p_ref);
      k_scale_f32<<<nblk(nf, 256), 256, 0, stream>>>(phi_f[d], sf_phi_f[d], nf, v_ref * v_ref);
      if (helm) k_scale_f32<<<nblk(nf, 256), 256, 0, stream>>>(eq_ge_f[d], sf_ge_f[d], nf, 1.0);
    }
    CK(cudaGetLastError());
    return PHL_OK;
  }
  void split_from_prim() {
    Prm P = prm(0);
    P.Win = W[cur];
    P.gin = gam[cur];
    P.Wf_out = Wf[cur];
    P.gf_out = gf[cur];
    runner->split_from_prim(P, stream);
  }
  // split path: U (+temp, eint) -> FP64 primitives and gammaf in W[cur], gam[cur]
  void split_to_prim() {
    Prm P = prm(0);
    P.Wout = W[cur];
    P.gout = gam[cur];
    runner->split_to_prim(P, stream);
  }
  void drop_graphs() {
    for (int p = 0; p < 2; ++p)
      if (graph[p]) { cudaGraphExecDestroy(graph[p]); graph[p] = nullptr; }
  }
  // hydro_step: all RK stages starting from W[cur]
  void launch_stages() {
    for (int s = 0; s < cfg.rk_stages; ++s) runner->stage(prm(s), stream);
  }
  // one time_loop iteration as a CUDA graph (captured on first use per W parity): tmax clamp,
  // the RK stages, time += dt, the next dt
  int launch_step_graph() {
    int p = cur;
    if (!graph[p]) {
      cudaGraph_t gph;
      CK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
      k_pre_step<<<1, 1, 0, stream>>>(scal, active, smax_bits, step, (long long)1 << 62);
      launch_stages();
      k_post_step<<<1, 1, 0, stream>>>(scal, active, smax_bits, step, cfg.cfl);
      CK(cudaStreamEndCapture(stream, &gph));
      cudaError_t e = cudaGraphInstantiate(&graph[p], gph, 0);
      cudaGraphDestroy(gph);
      if (e != cudaSuccess) {
        g_last_error = std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e);
        return PHL_E_CUDA;
      }
    }
    CK(cudaGraphLaunch(graph[p], stream));
    cur = (cur + cfg.rk_stages) & 1;
    return PHL_OK;
  }
};

namespace {

int check_cfg(const phl_config *c) {
  if (!c || c->abi_version != PHL_ABI_VERSION) return PHL_E_INVALID;
  if (c->sdims != 2 && c->sdims != 3) return PHL_E_INVALID;
  if (c->nx1 < 4 || c->nx2 < 4 || c->nx3 < 1) return PHL_E_INVALID;
  if (c->sdims == 2 && c->nx3 != 1) return PHL_E_INVALID;
  if (c->sdims == 3 && c->nx3 < 4) return PHL_E_INVALID;
  if (c->ngc < 2) return PHL_E_INVALID;
  // kernels decompose linear cell / face / corner indices with 32-bit arithmetic
  if ((double)(c->nx1 + 4) * (double)(c->nx2 + 4) * (double)(c->nx3 + 4) >= 4294967296.0) return PHL_E_TOO_LARGE;
  if (c->nvars != 2 + c->sdims + c->nas) return PHL_E_INVALID;
  if (c->rk_stages != 2 && c->rk_stages != 3) return PHL_E_INVALID;
  for (int d = 0; d < 3; ++d)
    for (int s = 0; s < 2; ++s)
      if (c->bc[d][s] != PHL_BC_PERIODIC && c->bc[d][s] != PHL_BC_REFLECTIVE) return PHL_E_INVALID;
  for (int d = 0; d < c->sdims; ++d)
    if ((c->bc[d][0] == PHL_BC_PERIODIC) != (c->bc[d][1] == PHL_BC_PERIODIC)) return PHL_E_INVALID;
  bool mhd = c->flags & PHL_MHD, helm = c->flags & PHL_HELMHOLTZ;
  if (mhd && (c->riemann != PHL_HLLD && c->riemann != PHL_LHLLD)) return PHL_E_INVALID;
  if (!mhd && (c->riemann != PHL_LHLLC && c->riemann != PHL_HLLC)) return PHL_E_INVALID;
  if (helm && !((c->flags & PHL_ADVECT_YE_IABAR) && c->nas >= 2)) return PHL_E_UNSUPPORTED;
  if (c->precision != PHL_FP64 && c->precision != PHL_FP32_SPLIT) return PHL_E_INVALID;
  if (c->reconstruction < PHL_REC_LIM2ND || c->reconstruction > PHL_REC_LIM5TH) return PHL_E_INVALID;
  if (c->reconstruction == PHL_REC_LIM5TH && c->ngc < 3) return PHL_E_INVALID;
  if (c->flags & PHL_SHOCK_FLATTENING) {
    // the detector tests cells lx-2..ux+2 with central differences: 3 ghost layers
    if (c->ngc < 3 || !(c->eps_sf == c->eps_sf)) return PHL_E_INVALID;
  }
  // the FP64 form keeps the reference's warm start (bit-exact); the learned guess inside the step
  // is built for the split MHD stage (Helmholtz), judged by the Newton with the warm start as
  // the fallback
  const bool learned = c->eos_guess == PHL_GUESS_MLP || c->eos_guess == PHL_GUESS_MLP_RESCUE;
  if (learned && !(c->precision == PHL_FP32_SPLIT && (c->flags & PHL_MHD) && (c->flags & PHL_HELMHOLTZ))) {
    g_last_error = "a learned eos_guess in the step is built for the FP32 split MHD form with the Helmholtz EoS";
    return PHL_E_UNSUPPORTED;
  }
  if (c->eos_guess != PHL_GUESS_WARM && !learned) return PHL_E_INVALID;
  return PHL_OK;
}

// Copy the interior box of a reference-layout host array (rows of `row` doubles, `pitch`
// doubles apart, `rows` of `rows_alloc` rows per slice, `slices` slices) from a compact device
// buffer, as one strided DMA: the host's ghost layers are left as they are.  Used device to
// host, where it runs at the link rate (host-to-device strided copies measured slower than
// sending the ghost layers along, so uploads copy whole arrays).
cudaError_t copy_box_d2h(const double *dev, double *host_start, size_t row, size_t pitch, size_t rows,
                         size_t rows_alloc, size_t slices, cudaStream_t s) {
  cudaMemcpy3DParms p;
  memset(&p, 0, sizeof(p));
  p.srcPtr = make_cudaPitchedPtr(const_cast<double *>(dev), row * sizeof(double), row, rows);
  p.dstPtr = make_cudaPitchedPtr(host_start, pitch * sizeof(double), pitch, rows_alloc);
  p.extent = make_cudaExtent(row * sizeof(double), rows, slices);
  p.kind = cudaMemcpyDeviceToHost;
  return cudaMemcpy3DAsync(&p, s);
}

// A background array (nv comps with a component index `comp`) is a profile along x2 when all
// its interior values agree along x1 and x3 for every x2 index.  On success fills prof[0..n2).
bool extract_profile(const double *a, int nv, int comp, int n1, int n2, int n3, int o1, int o2, int o3,
                     int ld1, int ld2, int nj, std::vector<double> &prof) {
  prof.assign(nj, 0.0);
  for (int j = 0; j < nj; ++j) {
    double ref = a[(size_t)nv * ((size_t)(0 + o1) + (size_t)ld1 * ((size_t)(j + o2) + (size_t)ld2 * (0 + o3))) + comp];
    for (int k = 0; k < n3; ++k)
      for (int i = 0; i < n1; ++i) {
        double v = a[(size_t)nv * ((size_t)(i + o1) + (size_t)ld1 * ((size_t)(j + o2) + (size_t)ld2 * (k + o3))) + comp];
        if (!(v == ref) && !(std::isnan(v) && std::isnan(ref))) return false;
      }
    prof[j] = ref;
  }
  (void)n2;
  return true;
}

}  // namespace

// =============================================================================== C ABI
extern "C" {

int phl_abi_version(void) { return PHL_ABI_VERSION; }

const char *phl_error_string(int code) {
  if (!g_last_error.empty() && code == PHL_E_CUDA) return g_last_error.c_str();
  switch (code) {
    case PHL_OK: return "ok";
    case PHL_E_INVALID: return "invalid argument or option combination";
    case PHL_E_CUDA: return "CUDA error";
    case PHL_E_NO_TABLE: return "Helmholtz table not loaded";
    case PHL_E_STATE: return "call out of order";
    case PHL_E_NO_DEVICE: return "no usable CUDA device";
    case PHL_E_UNSUPPORTED: return "option combination not built";
    case PHL_E_TOO_LARGE: return "size beyond capacity";
  }
  return "unknown error";
}

int phl_init(const phl_config *cfg, phl_ctx **out) {
  if (!out) return PHL_E_INVALID;
  *out = nullptr;
  int rc = check_cfg(cfg);
  if (rc) return rc;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= cfg->device) {
    g_last_error = "no CUDA device";
    return PHL_E_NO_DEVICE;
  }
  CK(cudaSetDevice(cfg->device));
  std::unique_ptr<phl_ctx> c(new phl_ctx());
  c->cfg = *cfg;
  c->dim = cfg->sdims;
  c->nv = cfg->nvars;
  bool mhd = cfg->flags & PHL_MHD, helm = cfg->flags & PHL_HELMHOLTZ;
  bool wb = cfg->flags & PHL_WB, etot = cfg->flags & PHL_EVOLVE_ETOT, grav = cfg->flags & PHL_GRAVITY;
  if (!(wb == etot && etot == grav)) return PHL_E_UNSUPPORTED;
  c->split = cfg->precision == PHL_FP32_SPLIT;
  const bool fast = cfg->flags & PHL_FASTEOS;
  const bool sf = (cfg->flags & PHL_SHOCK_FLATTENING) != 0;
  if (c->split) {
    c->runner.reset(make_split_runner(cfg->sdims, cfg->nvars, mhd, helm, wb, cfg->riemann, fast, cfg->reconstruction, sf));
    c->fp64_runner.reset(make_runner(cfg->sdims, cfg->nvars, mhd, helm, wb, cfg->riemann, fast, cfg->reconstruction, sf));
    if (!c->fp64_runner) return PHL_E_UNSUPPORTED;
  } else {
    c->runner.reset(make_runner(cfg->sdims, cfg->nvars, mhd, helm, wb, cfg->riemann, fast, cfg->reconstruction, sf));
  }
  if (!c->runner) return PHL_E_UNSUPPORTED;
  CK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
  Geo &g = c->geo;
  memset(&g, 0, sizeof(g));
  g.sdims = cfg->sdims;
  g.nx[0] = cfg->nx1; g.nx[1] = cfg->nx2; g.nx[2] = cfg->nx3;
  g.N = (long long)cfg->nx1 * cfg->nx2 * cfg->nx3;
  for (int d = 0; d < 3; ++d)
    for (int s = 0; s < 2; ++s) g.bc[d][s] = cfg->bc[d][s];
  // dx as initialize_simulation (source.F90:1717-1735)
  double dx1 = (cfg->x1u - cfg->x1l) / (double)cfg->nx1;
  double dx2 = (cfg->x2u - cfg->x2l) / (double)cfg->nx2;
  double dx3 = (cfg->x3u - cfg->x3l) / (double)cfg->nx3;
  g.inv_dx[0] = 1.0 / dx1; g.inv_dx[1] = 1.0 / dx2; g.inv_dx[2] = cfg->sdims == 3 ? 1.0 / dx3 : 0.0;
  g.gm = cfg->gamma_ad; g.mu = cfg->mu; g.cfl = cfg->cfl;
  g.mach_cutoff = cfg->mach_cutoff; g.mach_ct = cfg->mach_ct;
  g.all_mach = (cfg->flags & PHL_FLUX_IS_ALL_MACH) ? 1 : 0;
  g.use_acc = (cfg->flags & PHL_CONSTANT_ACCELERATION) ? 1 : 0;
  for (int d = 0; d < 3; ++d) g.acc[d] = g.use_acc ? cfg->acc[d] : 0.0;
  c->N = g.N;
  long long N = g.N;
  int nv = cfg->nvars;
  if ((rc = c->alloc(&c->W[0], (size_t)nv * N))) return rc;
  if ((rc = c->alloc(&c->W[1], (size_t)nv * N))) return rc;
  if ((rc = c->alloc(&c->U, (size_t)nv * N))) return rc;
  if ((rc = c->alloc(&c->U0, (size_t)nv * N))) return rc;
  if ((rc = c->alloc(&c->eint, (size_t)N))) return rc;
  if ((rc = c->alloc(&c->temp, (size_t)N))) return rc;
  if (helm) {
    if ((rc = c->alloc(&c->gam[0], (size_t)2 * N))) return rc;
    if ((rc = c->alloc(&c->gam[1], (size_t)2 * N))) return rc;
  }
  if (c->split) {
    for (int q = 0; q < 2; ++q) {
      if ((rc = c->alloc(&c->Wf[q], (size_t)nv * N))) return rc;
      if (helm && (rc = c->alloc(&c->gf[q], (size_t)2 * N))) return rc;
    }
  }
  if (cfg->flags & PHL_SHOCK_FLATTENING) {
    const long long nz2 = cfg->sdims == 3 ? 1 : 0;
    long long nflag = (long long)(cfg->nx1 + 2) * (cfg->nx2 + 2) * (cfg->nx3 + 2 * nz2);
    long long nmark = (long long)(cfg->nx1 + 4) * (cfg->nx2 + 4) * (cfg->nx3 + 4 * nz2);
    if ((rc = c->alloc(&c->sf_flag, (size_t)nflag))) return rc;
    if ((rc = c->alloc(&c->sf_mark, (size_t)nmark))) return rc;
  }
  if (mhd) {
    if ((rc = c->alloc(&c->bcc, (size_t)3 * N))) return rc;
    for (int d = 0; d < cfg->sdims; ++d) {
      long long nf = c->nfaces(d);
      if ((rc = c->alloc(&c->bf[d], (size_t)nf))) return rc;
      if ((rc = c->alloc(&c->b0f[d], (size_t)nf))) return rc;
      if ((rc = c->alloc(&c->emf[d], (size_t)3 * nf))) return rc;
      if ((rc = c->alloc(&c->sgnf[d], (size_t)nf))) return rc;
    }
    for (int a = 0; a < 3; ++a) {
      if (cfg->sdims == 2 && a != 2) continue;
      if ((rc = c->alloc(&c->cor[a], (size_t)c->ncor(a)))) return rc;
    }

    if (c->split) {
      if ((rc = c->alloc(&c->bccf, (size_t)3 * N))) return rc;
      if ((rc = c->alloc(&c->fecell, (size_t)3 * N))) return rc;
      if (cfg->eos_guess == PHL_GUESS_MLP) {
        if ((rc = c->alloc(&c->mlp_feat, (size_t)4 * N))) return rc;
        if ((rc = c->alloc(&c->mlp_out, (size_t)N))) return rc;
      }
      if (cfg->eos_guess == PHL_GUESS_MLP_RESCUE && (rc = c->alloc(&c->rescue_q, (size_t)N + 1))) return rc;
      for (int d = 0; d < cfg->sdims; ++d) {
        long long nf = c->nfaces(d);
        if ((rc = c->alloc(&c->femf[d], (size_t)3 * nf))) return rc;
        if ((rc = c->alloc(&c->fsgn[d], (size_t)nf))) return rc;
        if ((rc = c->alloc(&c->fflux[d], (size_t)nv * nf))) return rc;
      }
      for (int a = 0; a < 3; ++a) {
        if (cfg->sdims == 2 && a != 2) continue;
        if ((rc = c->alloc(&c->fcor[a], (size_t)c->ncor(a)))) return rc;
      }
    }
  }
  if (!c->split)
    for (int d = 0; d < cfg->sdims; ++d)
      if ((rc = c->alloc(&c->dflux[d], (size_t)nv * c->nfaces(d)))) return rc;
  if ((rc = c->alloc(&c->scal, 8))) return rc;
  if ((rc = c->alloc(&c->smax_bits, 1))) return rc;
  if ((rc = c->alloc(&c->active, 1))) return rc;
  if ((rc = c->alloc(&c->step, 1))) return rc;
  if ((rc = c->alloc(&c->stat, STAT_COUNT))) return rc;
  k_set_active<<<1, 1, 0, c->stream>>>(c->active, c->smax_bits);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(c->stream));
  *out = c.release();
  return PHL_OK;
}

void phl_finalize(phl_ctx *ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->cfg.device);
  ctx->drain_host();
  cudaStreamSynchronize(ctx->stream);
  delete ctx;
}

int phl_load_helm_table(phl_ctx *ctx, const double *tab, const double *dpdr) {
  if (!ctx || !tab || !dpdr) return PHL_E_INVALID;
  const phl_config &c = ctx->cfg;
  int nr = c.helm_nrho, nT = c.helm_nT;
  if (nr < 2 || nT < 2) return PHL_E_INVALID;
  CK(cudaSetDevice(c.device));
  int rc;
  if (!ctx->htab) {
    if ((rc = ctx->alloc(&ctx->htab, (size_t)9 * nr * nT))) return rc;
    if ((rc = ctx->alloc(&ctx->hdpd, (size_t)4 * nr * nT))) return rc;
    if ((rc = ctx->alloc(&ctx->hrho, (size_t)nr))) return rc;
    if ((rc = ctx->alloc(&ctx->hT, (size_t)nT))) return rc;
    if ((rc = ctx->alloc(&ctx->hirho, (size_t)nr))) return rc;
    if ((rc = ctx->alloc(&ctx->hiT, (size_t)nT))) return rc;
  }
  // nodes as load_helm_table builds them (source.F90:23091-23104)
  double dT = (c.helm_lthi - c.helm_ltlo) / (double)(nT - 1);
  double drho = (c.helm_ldhi - c.helm_ldlo) / (double)(nr - 1);
  std::vector<double> T(nT), rho(nr);
  for (int j = 0; j < nT; ++j) T[j] = std::pow(10.0, c.helm_ltlo + (double)j * dT);
  for (int i = 0; i < nr; ++i) rho[i] = std::pow(10.0, c.helm_ldlo + (double)i * drho);
  std::vector<double> irho(nr, 0.0), iT(nT, 0.0);
  for (int i = 0; i + 1 < nr; ++i) irho[i] = 1.0 / (rho[i + 1] - rho[i]);
  for (int j = 0; j + 1 < nT; ++j) iT[j] = 1.0 / (T[j + 1] - T[j]);
  CK(cudaMemcpyAsync(ctx->htab, tab, sizeof(double) * 9 * nr * nT, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(ctx->hdpd, dpdr, sizeof(double) * 4 * nr * nT, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(ctx->hrho, rho.data(), sizeof(double) * nr, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(ctx->hT, T.data(), sizeof(double) * nT, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(ctx->hirho, irho.data(), sizeof(double) * nr, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(ctx->hiT, iT.data(), sizeof(double) * nT, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  HelmTable &h = ctx->helm;
  h.tab = ctx->htab; h.dpdr = ctx->hdpd; h.rho = ctx->hrho; h.T = ctx->hT;
  h.inv_drho = ctx->hirho; h.inv_dT = ctx->hiT;
  h.nrho = nr; h.nT = nT; h.drho = drho; h.dT = dT;
  h.log10_rho1 = std::log10(rho[0]);
  h.log10_T1 = std::log10(T[0]);
  h.Tl = std::pow(10.0, c.helm_ltlo);
  h.Th = std::pow(10.0, c.helm_lthi);
  ctx->table_loaded = true;
  return PHL_OK;
}

int phl_upload_state(phl_ctx *ctx, const phl_fields *f) {
  if (!ctx || !f || !f->prim) return PHL_E_INVALID;
  const phl_config &c = ctx->cfg;
  CK(cudaSetDevice(c.device));
  if (int rc = ctx->drain_host()) return rc;
  cudaStream_t s = ctx->stream;
  const int G = c.ngc, G3 = c.sdims == 3 ? c.ngc : 0, sd = c.sdims, nv = c.nvars;
  const int nx = c.nx1, ny = c.nx2, nz = c.nx3;
  const int n1 = nx + 2 * G, n2 = ny + 2 * G, n3 = nz + 2 * G3;
  const long long Ng = (long long)n1 * n2 * n3, N = ctx->N;
  bool mhd = c.flags & PHL_MHD, helm = c.flags & PHL_HELMHOLTZ, strat = c.flags & PHL_WB;
  int rc;
  if ((rc = ctx->ensure_stage(sizeof(double) * (size_t)std::max<long long>(Ng * std::max(nv, 3), 1)))) return rc;
  auto unpack_cell = [&](const double *h, int ncomp_host, int ncomp, double *dst) -> int {
    CK(cudaMemcpyAsync(ctx->stage_buf, h, sizeof(double) * (size_t)ncomp_host * Ng, cudaMemcpyHostToDevice, s));
    k_unpack<<<nblk(N, 256), 256, 0, s>>>(ctx->stage_buf, dst, ncomp_host, nx, ny, nz, n1, n2, G, G, G3, ncomp, N);
    CK(cudaGetLastError());
    return PHL_OK;
  };
  ctx->cur = 0;
  if (ctx->split && !ctx->refs_set) {
    // scales of the FP32 split path: largest density and pressure of the first uploaded state
    double rmax = 0.0, pmax = 0.0;
    const int ip = 1 + sd;
    for (long long q = 0; q < Ng; ++q) {
      double r = std::fabs(f->prim[(size_t)nv * q]), pp = std::fabs(f->prim[(size_t)nv * q + ip]);
      if (std::isfinite(r) && r > rmax) rmax = r;
      if (std::isfinite(pp) && pp > pmax) pmax = pp;
    }
    ctx->rho_ref = rmax > 0.0 ? rmax : 1.0;
    ctx->p_ref = pmax > 0.0 ? pmax : 1.0;
    ctx->v_ref = std::sqrt(ctx->p_ref / ctx->rho_ref);
    ctx->refs_set = true;
  }
  if ((rc = unpack_cell(f->prim, nv, nv, ctx->W[0]))) return rc;
  if (f->temp && (rc = unpack_cell(f->temp, 1, 1, ctx->temp))) return rc;
  if (f->eint && (rc = unpack_cell(f->eint, 1, 1, ctx->eint))) return rc;
  const bool fast = c.flags & PHL_FASTEOS;
  if (helm && fast && f->gammaf && (rc = unpack_cell(f->gammaf, 2, 2, ctx->gam[0]))) return rc;
  // without USE_FASTEOS the first gamma slot carries the stage input's temperature
  if (helm && !fast && f->temp)
    CK(cudaMemcpyAsync(ctx->gam[0], ctx->temp, sizeof(double) * (size_t)N, cudaMemcpyDeviceToDevice, s));
  if (mhd && f->b_cc && (rc = unpack_cell(f->b_cc, sd, sd, ctx->bcc))) return rc;
  if (mhd) {
    // interior faces of b_x1(lx1-1:ux1+2, lx2-1:ux2+1, lx3-1:ux3+1), ...
    for (int d = 0; d < sd; ++d) {
      if (!f->b_x[d]) return PHL_E_INVALID;
      int b1 = nx + 2 + (d == 0), b2 = ny + 2 + (d == 1), b3 = sd == 3 ? nz + 2 + (d == 2) : 1;
      int o3 = sd == 3 ? 1 : 0;
      long long nb = (long long)b1 * b2 * b3;
      CK(cudaMemcpyAsync(ctx->stage_buf, f->b_x[d], sizeof(double) * nb, cudaMemcpyHostToDevice, s));
      k_unpack<<<nblk(ctx->nfaces(d), 256), 256, 0, s>>>(ctx->stage_buf, ctx->bf[d], 1, nx + (d == 0), ny + (d == 1),
                                                         nz + (d == 2), b1, b2, 1, 1, o3, 1, ctx->nfaces(d));
      CK(cudaGetLastError());
    }
  }
  if (strat && !f->eq_prim_cc && !ctx->bg_uploaded) return PHL_E_INVALID;
  if (strat && f->eq_prim_cc) {
    // background: profiles along x2 when uniform in x1/x3, otherwise full arrays.  A later
    // upload without background pointers refreshes only the dynamic state.
    if (!f->phi_cc || !f->grav) return PHL_E_INVALID;
    for (int d = 0; d < sd; ++d)
      if (!f->eq_prim_x[d] || !f->phi_x[d]) return PHL_E_INVALID;
    if (helm && (!f->eq_gammae_cc)) return PHL_E_INVALID;
    for (int d = 0; d < sd && helm; ++d)
      if (!f->eq_gammae_x[d]) return PHL_E_INVALID;
    std::vector<std::vector<double>> prof;
    bool ok = true;
    auto cellprof = [&](const double *a, int nvh, int comp) {
      std::vector<double> p;
      ok = ok && extract_profile(a, nvh, comp, nx, ny, nz, G, G, G3, n1, n2, ny, p);
      prof.push_back(p);
    };
    auto faceprof = [&](const double *a, int nvh, int comp, int d) {
      std::vector<double> p;
      int fx = nx + (d == 0), fy = ny + (d == 1), fz = nz + (d == 2);
      ok = ok && extract_profile(a, nvh, comp, fx, fy, fz, 0, 0, 0, fx, fy, fy, p);
      prof.push_back(p);
    };
    cellprof(f->eq_prim_cc, 3, 0);
    cellprof(f->eq_prim_cc, 3, 1);
    cellprof(f->phi_cc, 1, 0);
    for (int d = 0; d < sd; ++d) cellprof(f->grav, sd, d);
    if (helm) cellprof(f->eq_gammae_cc, 1, 0);
    for (int d = 0; d < sd; ++d) {
      faceprof(f->eq_prim_x[d], 3, 0, d);
      faceprof(f->eq_prim_x[d], 3, 1, d);
      faceprof(f->phi_x[d], 1, 0, d);
      if (helm) faceprof(f->eq_gammae_x[d], 1, 0, d);
    }
    ctx->bg_profile = ok ? 1 : 0;
    ctx->geo.bg_profile = ctx->bg_profile;
    auto need = [&](double **p, size_t n) -> int {
      if (!*p) return ctx->alloc(p, n);
      return PHL_OK;
    };
    size_t ncc = ok ? (size_t)ny : (size_t)N;
    if ((rc = need(&ctx->eq_rho_cc, ncc)) || (rc = need(&ctx->eq_p_cc, ncc)) || (rc = need(&ctx->phi_cc, ncc)) ||
        (rc = need(&ctx->grav, (size_t)sd * ncc)))
      return rc;
    if (helm && (rc = need(&ctx->eq_ge_cc, ncc))) return rc;
    for (int d = 0; d < sd; ++d) {
      size_t nf = ok ? (size_t)(ny + (d == 1)) : (size_t)ctx->nfaces(d);
      if ((rc = need(&ctx->eq_rho_f[d], nf)) || (rc = need(&ctx->eq_p_f[d], nf)) || (rc = need(&ctx->phi_f[d], nf)))
        return rc;
      if (helm && (rc = need(&ctx->eq_ge_f[d], nf))) return rc;
    }
    if (ok) {
      size_t q = 0;
      auto put = [&](double *dst) -> int {
        CK(cudaMemcpyAsync(dst, prof[q].data(), sizeof(double) * prof[q].size(), cudaMemcpyHostToDevice, s));
        ++q;
        return PHL_OK;
      };
      if ((rc = put(ctx->eq_rho_cc)) || (rc = put(ctx->eq_p_cc)) || (rc = put(ctx->phi_cc))) return rc;
      for (int d = 0; d < sd; ++d)
        if ((rc = put(ctx->grav + (size_t)d * ny))) return rc;
      if (helm && (rc = put(ctx->eq_ge_cc))) return rc;
      for (int d = 0; d < sd; ++d) {
        if ((rc = put(ctx->eq_rho_f[d])) || (rc = put(ctx->eq_p_f[d])) || (rc = put(ctx->phi_f[d]))) return rc;
        if (helm && (rc = put(ctx->eq_ge_f[d]))) return rc;
      }
      CK(cudaStreamSynchronize(s));  // host vectors go out of scope
    } else {
      if ((rc = unpack_cell(f->eq_prim_cc, 3, 1, ctx->eq_rho_cc))) return rc;
      // second component: unpack with a shifted base
      CK(cudaMemcpyAsync(ctx->stage_buf, f->eq_prim_cc, sizeof(double) * 3 * Ng, cudaMemcpyHostToDevice, s));
      k_unpack<<<nblk(N, 256), 256, 0, s>>>(ctx->stage_buf + 1, ctx->eq_p_cc, 3, nx, ny, nz, n1, n2, G, G, G3, 1, N);
      if ((rc = unpack_cell(f->phi_cc, 1, 1, ctx->phi_cc))) return rc;
      if ((rc = unpack_cell(f->grav, sd, sd, ctx->grav))) return rc;
      if (helm && (rc = unpack_cell(f->eq_gammae_cc, 1, 1, ctx->eq_ge_cc))) return rc;
      for (int d = 0; d < sd; ++d) {
        long long nf = ctx->nfaces(d);
        int fx = nx + (d == 0), fy = ny + (d == 1), fz = nz + (d == 2);
        CK(cudaMemcpyAsync(ctx->stage_buf, f->eq_prim_x[d], sizeof(double) * 3 * nf, cudaMemcpyHostToDevice, s));
        k_unpack<<<nblk(nf, 256), 256, 0, s>>>(ctx->stage_buf, ctx->eq_rho_f[d], 3, fx, fy, fz, fx, fy, 0, 0, 0, 1, nf);
        k_unpack<<<nblk(nf, 256), 256, 0, s>>>(ctx->stage_buf + 1, ctx->eq_p_f[d], 3, fx, fy, fz, fx, fy, 0, 0, 0, 1, nf);
        CK(cudaMemcpyAsync(ctx->phi_f[d], f->phi_x[d], sizeof(double) * nf, cudaMemcpyHostToDevice, s));
        if (helm) CK(cudaMemcpyAsync(ctx->eq_ge_f[d], f->eq_gammae_x[d], sizeof(double) * nf, cudaMemcpyHostToDevice, s));
        CK(cudaStreamSynchronize(s));
      }
    }
  }
  if ((c.flags & PHL_SHOCK_FLATTENING) && strat && f->eq_prim_cc) {
    // the shock detector reads the pressure equilibrium of 3 ghost layers as the caller set
    // them: kept as a profile along x2 when it is one over the ghosted array, else in full
    std::vector<double> prof;
    bool pr = extract_profile(f->eq_prim_cc, 3, 1, n1, n2, n3, 0, 0, 0, n1, n2, n2, prof);
    size_t ne = pr ? (size_t)n2 : (size_t)Ng;
    if (!ctx->sf_eq_p && (rc = ctx->alloc(&ctx->sf_eq_p, (size_t)Ng))) return rc;
    std::vector<double> full;
    if (!pr) {
      full.resize(ne);
      for (size_t q = 0; q < ne; ++q) full[q] = f->eq_prim_cc[3 * q + 1];
    }
    CK(cudaMemcpyAsync(ctx->sf_eq_p, pr ? prof.data() : full.data(), sizeof(double) * ne, cudaMemcpyHostToDevice, s));
    CK(cudaStreamSynchronize(s));  // host vectors go out of scope
    ctx->sf_eq_profile = pr ? 1 : 0;
  }
  if (ctx->split && strat && f->eq_prim_cc && (rc = ctx->scale_background(helm))) return rc;
  if (ctx->split && f->eint && (!strat || ctx->bg_uploaded || f->eq_prim_cc)) {
    ctx->split_from_prim();
    CK(cudaGetLastError());
  }
  CK(cudaStreamSynchronize(s));
  if (strat && f->eq_prim_cc) {
    ctx->bg_uploaded = true;
    // graphs bake the background layout into their kernel arguments
    for (int p = 0; p < 2; ++p)
      if (ctx->graph[p]) { cudaGraphExecDestroy(ctx->graph[p]); ctx->graph[p] = nullptr; }
  }
  ctx->uploaded = true;
  return PHL_OK;
}

int phl_download_state(phl_ctx *ctx, phl_fields *f) {
  if (!ctx || !f) return PHL_E_INVALID;
  const phl_config &c = ctx->cfg;
  CK(cudaSetDevice(c.device));
  if (int rc = ctx->drain_host()) return rc;
  cudaStream_t s = ctx->stream;
  const int G = c.ngc, G3 = c.sdims == 3 ? c.ngc : 0, sd = c.sdims, nv = c.nvars;
  const int nx = c.nx1, ny = c.nx2, nz = c.nx3;
  const int n1 = nx + 2 * G, n2 = ny + 2 * G, n3 = nz + 2 * G3;
  const long long Ng = (long long)n1 * n2 * n3, N = ctx->N;
  bool mhd = c.flags & PHL_MHD, helm = c.flags & PHL_HELMHOLTZ;
  int rc;
  if ((rc = ctx->ensure_stage(sizeof(double) * (size_t)Ng * std::max(nv, 3)))) return rc;
  if (ctx->split) {
    ctx->split_to_prim();
    CK(cudaGetLastError());
  }
  // transpose into a compact staging block, then one strided copy into the interior of the host
  // array (its ghost cells are left as they are); the stream orders the reuse of the block
  auto pack_cell = [&](double *h, int ncomp, const double *src) -> int {
    k_pack<<<nblk(N, 256), 256, 0, s>>>(src, ctx->stage_buf, ncomp, nx, ny, nz, nx, ny, 0, 0, 0, ncomp, N);
    CK(cudaGetLastError());
    double *start = h + (size_t)ncomp * ((size_t)G + (size_t)n1 * ((size_t)G + (size_t)n2 * G3));
    CK(copy_box_d2h(ctx->stage_buf, start, (size_t)ncomp * nx, (size_t)ncomp * n1, ny, n2, nz, s));
    return PHL_OK;
  };
  if (f->prim && (rc = pack_cell(f->prim, nv, ctx->W[ctx->cur]))) return rc;
  if (f->temp && (rc = pack_cell(f->temp, 1, ctx->temp))) return rc;
  if (f->eint && (rc = pack_cell(f->eint, 1, ctx->eint))) return rc;
  if (helm && (c.flags & PHL_FASTEOS) && f->gammaf && (rc = pack_cell(f->gammaf, 2, ctx->gam[ctx->cur]))) return rc;
  if (mhd && f->b_cc && (rc = pack_cell(f->b_cc, sd, ctx->bcc))) return rc;
  if (mhd) {
    for (int d = 0; d < sd; ++d) {
      if (!f->b_x[d]) continue;
      int b1 = nx + 2 + (d == 0), b2 = ny + 2 + (d == 1), b3 = sd == 3 ? nz + 2 + (d == 2) : 1;
      int o3 = sd == 3 ? 1 : 0;
      (void)b3;
      const int fx = nx + (d == 0), fy = ny + (d == 1), fz = nz + (d == 2);
      k_pack<<<nblk(ctx->nfaces(d), 256), 256, 0, s>>>(ctx->bf[d], ctx->stage_buf, 1, fx, fy, fz, fx, fy, 0, 0, 0, 1,
                                                       ctx->nfaces(d));
      CK(cudaGetLastError());
      double *start = f->b_x[d] + (1 + (size_t)b1 * (1 + (size_t)b2 * o3));
      CK(copy_box_d2h(ctx->stage_buf, start, fx, b1, fy, b2, fz, s));
    }
  }
  CK(cudaStreamSynchronize(s));
  return PHL_OK;
}

// step: the call advances the state (and so runs the cons->prim Newton with the selected guess)
static int ready(phl_ctx *ctx, bool step = false) {
  if (!ctx) return PHL_E_INVALID;
  if (int rc = ctx->drain_host()) return rc;
  if (!ctx->uploaded) return PHL_E_STATE;
  if ((ctx->cfg.flags & PHL_HELMHOLTZ) && !ctx->table_loaded) return PHL_E_NO_TABLE;
  if (step && (ctx->cfg.eos_guess == PHL_GUESS_MLP || ctx->cfg.eos_guess == PHL_GUESS_MLP_RESCUE) &&
      !ctx->eos.mlp.ready) {
    g_last_error = "eos_guess = PHL_GUESS_MLP: train the network (phl_mlp_train) or set its parameters first";
    return PHL_E_STATE;
  }
  return PHL_OK;
}

int phl_init_thermo(phl_ctx *ctx) {
  int rc = ready(ctx);
  if (rc) return rc;
  CK(cudaSetDevice(ctx->cfg.device));
  Prm P = ctx->prm(0);
  // write gammaf into the current buffer: gout must alias gin here
  P.Win = ctx->W[ctx->cur];
  P.gout = ctx->gam[ctx->cur];
  ctx->thermo()->init_thermo(P, ctx->stream);
  CK(cudaGetLastError());
  if (ctx->split) {
    ctx->split_from_prim();
    CK(cudaGetLastError());
  }
  CK(cudaStreamSynchronize(ctx->stream));
  return PHL_OK;
}

int phl_compute_hyperbolic_dt(phl_ctx *ctx, double *dt, double *smax) {
  int rc = ready(ctx);
  if (rc) return rc;
  CK(cudaSetDevice(ctx->cfg.device));
  if (ctx->split) ctx->split_to_prim();
  Prm P = ctx->prm(0);
  P.Win = ctx->W[ctx->cur];
  CK(cudaMemsetAsync(ctx->smax_bits, 0, sizeof(unsigned long long), ctx->stream));
  ctx->thermo()->dt(P, ctx->stream);
  k_finish_dt<<<1, 1, 0, ctx->stream>>>(ctx->scal, ctx->smax_bits, ctx->cfg.cfl);
  CK(cudaGetLastError());
  double sc[3];
  CK(cudaMemcpyAsync(sc, ctx->scal, sizeof(sc), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  if (dt) *dt = sc[1];
  if (smax) *smax = sc[2];
  return PHL_OK;
}

int phl_hydro_step(phl_ctx *ctx) {
  int rc = ready(ctx, true);
  if (rc) return rc;
  CK(cudaSetDevice(ctx->cfg.device));
  k_set_active<<<1, 1, 0, ctx->stream>>>(ctx->active, ctx->smax_bits);
  ctx->launch_stages();
  CK(cudaGetLastError());
  ctx->cur = (ctx->cur + ctx->cfg.rk_stages) & 1;
  CK(cudaStreamSynchronize(ctx->stream));
  return PHL_OK;
}

int phl_set_time(phl_ctx *ctx, double time, double dt, double smax) {
  if (!ctx) return PHL_E_INVALID;
  CK(cudaSetDevice(ctx->cfg.device));
  double sc[3] = {time, dt, smax};
  CK(cudaMemcpyAsync(ctx->scal, sc, sizeof(sc), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return PHL_OK;
}

int phl_get_time(phl_ctx *ctx, double *time, double *dt, double *smax) {
  if (!ctx) return PHL_E_INVALID;
  CK(cudaSetDevice(ctx->cfg.device));
  double sc[3];
  CK(cudaMemcpyAsync(sc, ctx->scal, sizeof(sc), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  if (time) *time = sc[0];
  if (dt) *dt = sc[1];
  if (smax) *smax = sc[2];
  return PHL_OK;
}

int phl_run_steps(phl_ctx *ctx, int nsteps, double tmax, int *steps_done, double *time) {
  int rc = ready(ctx, true);
  if (rc) return rc;
  if (nsteps < 0) return PHL_E_INVALID;
  CK(cudaSetDevice(ctx->cfg.device));
  cudaStream_t s = ctx->stream;
  long long step0 = 0;
  CK(cudaMemcpyAsync(&step0, ctx->step, sizeof(long long), cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(ctx->scal + 3, &tmax, sizeof(double), cudaMemcpyHostToDevice, s));
  CK(cudaStreamSynchronize(s));
  // graphs run with no device-side step limit: the host launches exactly nsteps of them and
  // the device stops by itself once time >= tmax.
  for (int n = 0; n < nsteps; ++n)
    if ((rc = ctx->launch_step_graph())) return rc;
  long long step1 = 0;
  double t = 0;
  CK(cudaMemcpyAsync(&step1, ctx->step, sizeof(long long), cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(&t, ctx->scal, sizeof(double), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  CK(cudaGetLastError());
  // steps skipped by the device (time >= tmax) did not swap the W buffers: recover parity
  long long skipped = (long long)nsteps - (step1 - step0);
  if (skipped > 0 && (ctx->cfg.rk_stages & 1)) ctx->cur = (int)((ctx->cur + skipped) & 1);
  if (steps_done) *steps_done = (int)(step1 - step0);
  if (time) *time = t;
  return PHL_OK;
}

}  // extern "C"

namespace {
// Lay out the pipeline's slots for this context (once): extents of each dynamic host array,
// its device field, staging images and chunking along x3.
int host_pipe_setup(phl_ctx *ctx) {
  if (ctx->hpipe_ready) return PHL_OK;
  const phl_config &c = ctx->cfg;
  const int G = c.ngc, G3 = c.sdims == 3 ? c.ngc : 0, sd = c.sdims, nv = c.nvars;
  const int nx = c.nx1, ny = c.nx2, nz = c.nx3;
  const bool mhd = c.flags & PHL_MHD, helm = c.flags & PHL_HELMHOLTZ, fast = c.flags & PHL_FASTEOS;
  auto cell = [&](int q, int ncomp, double *dev) {
    phl_ctx::HostSlot &h = ctx->hslot[q];
    h.ncomp = ncomp; h.h1 = nx + 2 * G; h.h2 = ny + 2 * G; h.h3 = nz + 2 * G3;
    h.fx = nx; h.fy = ny; h.fz = nz; h.o1 = G; h.o2 = G; h.o3 = G3;
    h.dev = dev; h.dev_stride = ctx->N;
  };
  cell(0, nv, nullptr);  // prim: W[cur], chosen per call
  cell(1, 1, ctx->temp);
  cell(2, 1, ctx->eint);
  if (helm && fast) cell(3, 2, nullptr);  // gammaf: gam[cur]
  if (mhd) cell(4, sd, ctx->bcc);
  for (int d = 0; d < sd && mhd; ++d) {
    phl_ctx::HostSlot &h = ctx->hslot[5 + d];
    h.ncomp = 1;
    h.h1 = nx + 2 + (d == 0); h.h2 = ny + 2 + (d == 1); h.h3 = sd == 3 ? nz + 2 + (d == 2) : 1;
    h.fx = nx + (d == 0); h.fy = ny + (d == 1); h.fz = sd == 3 ? nz + (d == 2) : 1;
    h.o1 = 1; h.o2 = 1; h.o3 = sd == 3 ? 1 : 0;
    h.dev = ctx->bf[d]; h.dev_stride = ctx->nfaces(d);
  }
  // chunks of about 64 MB: the upload of a chunk waits only for the previous call's download
  // of the same host planes, so the two directions overlap with a lag of one chunk
  const size_t chunk_bytes = (size_t)64 << 20;
  int nchunks = 0;
  for (int q = 0; q < phl_ctx::HOST_SLOTS; ++q) {
    phl_ctx::HostSlot &h = ctx->hslot[q];
    if (!h.ncomp) continue;
    size_t pb = h.plane() * sizeof(double);
    h.ppc = (int)std::max<size_t>(1, chunk_bytes / std::max<size_t>(pb, 1));
    h.nchunk = (h.h3 + h.ppc - 1) / h.ppc;
    h.chunk0 = nchunks;
    nchunks += h.nchunk;
    int rc;
    if ((rc = ctx->alloc(&h.in, h.plane() * h.h3)) ||
        (rc = ctx->alloc(&h.out, (size_t)h.ncomp * h.fx * h.fy * h.fz)))
      return rc;
    CK(cudaEventCreateWithFlags(&ctx->ev_in[q], cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&ctx->ev_pack[q], cudaEventDisableTiming));
  }
  ctx->ev_chunk_out.assign(nchunks, nullptr);
  for (int k = 0; k < nchunks; ++k) CK(cudaEventCreateWithFlags(&ctx->ev_chunk_out[k], cudaEventDisableTiming));
  CK(cudaStreamCreateWithFlags(&ctx->cin, cudaStreamNonBlocking));
  CK(cudaStreamCreateWithFlags(&ctx->cout, cudaStreamNonBlocking));
  CK(cudaStreamSynchronize(ctx->stream));  // the staging allocations are zeroed on it
  ctx->hpipe_ready = true;
  return PHL_OK;
}

__global__ void k_set_tmax_inf(double *scal) { scal[3] = __longlong_as_double(0x7ff0000000000000LL); }
}  // namespace

extern "C" {

int phl_run_steps_host_async(phl_ctx *ctx, phl_fields *f, int nsteps) {
  if (!ctx || !f || !f->prim || nsteps < 0) return PHL_E_INVALID;
  if ((ctx->cfg.flags & PHL_HELMHOLTZ) && !ctx->table_loaded) return PHL_E_NO_TABLE;
  if (!ctx->uploaded) return PHL_E_STATE;
  if ((ctx->cfg.eos_guess == PHL_GUESS_MLP || ctx->cfg.eos_guess == PHL_GUESS_MLP_RESCUE) && !ctx->eos.mlp.ready)
    return PHL_E_STATE;
  const phl_config &c = ctx->cfg;
  const bool mhd = c.flags & PHL_MHD, helm = c.flags & PHL_HELMHOLTZ, fast = c.flags & PHL_FASTEOS;
  for (int d = 0; d < c.sdims && mhd; ++d)
    if (!f->b_x[d]) return PHL_E_INVALID;
  CK(cudaSetDevice(c.device));
  int rc;
  if ((rc = host_pipe_setup(ctx))) return rc;
  cudaStream_t S = ctx->stream;
  double *host[phl_ctx::HOST_SLOTS] = {f->prim, f->temp, f->eint, (helm && fast) ? f->gammaf : nullptr,
                                       mhd ? f->b_cc : nullptr, mhd ? f->b_x[0] : nullptr,
                                       mhd ? f->b_x[1] : nullptr, mhd ? f->b_x[2] : nullptr};
  // ---- upload: whole host arrays chunk by chunk on the input stream, as contiguous copies (a
  // pitched host-to-device copy of the interior box alone doubled the time of a 256^3 MHD call
  // on B200); the kernels map every ghost index, so the host's ghost layers are never read
  ctx->cur = 0;
  ctx->hslot[0].dev = ctx->W[0];
  ctx->hslot[3].dev = ctx->gam[0];
  for (int q = 0; q < phl_ctx::HOST_SLOTS; ++q) {
    phl_ctx::HostSlot &h = ctx->hslot[q];
    if (!h.ncomp || !host[q]) continue;
    for (int k = 0; k < h.nchunk; ++k) {
      const int p0 = k * h.ppc, p1 = std::min(h.h3, p0 + h.ppc);
      const size_t off = h.plane() * p0;
      CK(cudaStreamWaitEvent(ctx->cin, ctx->ev_chunk_out[h.chunk0 + k], 0));
      CK(cudaMemcpyAsync(h.in + off, host[q] + off, sizeof(double) * h.plane() * (p1 - p0), cudaMemcpyHostToDevice,
                         ctx->cin));
    }
    CK(cudaEventRecord(ctx->ev_in[q], ctx->cin));
    CK(cudaStreamWaitEvent(S, ctx->ev_in[q], 0));
    const long long n = (long long)h.fx * h.fy * h.fz;
    k_unpack<<<nblk(n, 256), 256, 0, S>>>(h.in, h.dev, h.ncomp, h.fx, h.fy, h.fz, h.h1, h.h2, h.o1, h.o2, h.o3,
                                          h.ncomp, h.dev_stride);
    CK(cudaGetLastError());
  }
  // without USE_FASTEOS the first gamma slot carries the stage input's temperature
  if (helm && !fast && f->temp)
    CK(cudaMemcpyAsync(ctx->gam[0], ctx->temp, sizeof(double) * (size_t)ctx->N, cudaMemcpyDeviceToDevice, S));
  if (ctx->split) ctx->split_from_prim();
  // ---- exactly nsteps steps (no tmax clamp: a skipped step would leave W's parity unknown to
  // the host without a round trip)
  k_set_tmax_inf<<<1, 1, 0, S>>>(ctx->scal);
  for (int n = 0; n < nsteps; ++n)
    if ((rc = ctx->launch_step_graph())) return rc;
  CK(cudaGetLastError());
  // ---- download: interior of each array, chunk by chunk on the output stream
  if (ctx->split) ctx->split_to_prim();
  ctx->hslot[0].dev = ctx->W[ctx->cur];
  ctx->hslot[3].dev = ctx->gam[ctx->cur];
  for (int q = 0; q < phl_ctx::HOST_SLOTS; ++q) {
    phl_ctx::HostSlot &h = ctx->hslot[q];
    if (!h.ncomp || !host[q]) continue;
    const long long n = (long long)h.fx * h.fy * h.fz;
    k_pack<<<nblk(n, 256), 256, 0, S>>>(h.dev, h.out, h.ncomp, h.fx, h.fy, h.fz, h.fx, h.fy, 0, 0, 0, h.ncomp,
                                        h.dev_stride);
    CK(cudaGetLastError());
    CK(cudaEventRecord(ctx->ev_pack[q], S));
    CK(cudaStreamWaitEvent(ctx->cout, ctx->ev_pack[q], 0));
    for (int k = 0; k < h.nchunk; ++k) {
      // interior planes inside host planes [p0, p1)
      const int p0 = k * h.ppc, p1 = std::min(h.h3, p0 + h.ppc);
      const int q0 = std::max(p0 - h.o3, 0), q1 = std::min(p1 - h.o3, h.fz);
      if (q1 > q0) {
        const double *src = h.out + (size_t)h.ncomp * h.fx * h.fy * q0;
        double *dst = host[q] + (size_t)h.ncomp * ((size_t)h.o1 + (size_t)h.h1 * ((size_t)h.o2 + (size_t)h.h2 * (q0 + h.o3)));
        CK(copy_box_d2h(src, dst, (size_t)h.ncomp * h.fx, (size_t)h.ncomp * h.h1, h.fy, h.h2, q1 - q0, ctx->cout));
      }
      CK(cudaEventRecord(ctx->ev_chunk_out[h.chunk0 + k], ctx->cout));
    }
  }
  ctx->hpipe_pending = true;
  return PHL_OK;
}

int phl_wait_host(phl_ctx *ctx) {
  if (!ctx) return PHL_E_INVALID;
  CK(cudaSetDevice(ctx->cfg.device));
  int rc = ctx->drain_host();
  if (rc) return rc;
  CK(cudaGetLastError());
  return PHL_OK;
}

int phl_get_status(phl_ctx *ctx, phl_status *st) {
  if (!ctx || !st) return PHL_E_INVALID;
  CK(cudaSetDevice(ctx->cfg.device));
  unsigned long long h[STAT_COUNT];
  long long step = 0;
  double sc[3];
  CK(cudaMemcpyAsync(h, ctx->stat, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaMemcpyAsync(&step, ctx->step, sizeof(step), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaMemcpyAsync(sc, ctx->scal, sizeof(sc), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  memset(st, 0, sizeof(*st));
  st->newton_calls = (long long)h[STAT_NEWTON_CALLS];
  st->newton_iterations = (long long)h[STAT_NEWTON_ITERS];
  st->newton_nonconverged = (long long)h[STAT_NEWTON_NONCONV];
  st->newton_clamped = (long long)h[STAT_NEWTON_CLAMP];
  st->mlp_accepted = (long long)h[STAT_MLP_ACC];
  st->mlp_rejected = (long long)h[STAT_MLP_REJ];
  st->nonfinite = (long long)h[STAT_NONFINITE];
  st->guess_evaluations = (long long)h[STAT_GUESS_EVALS];
  st->tensor_core_stalls = (long long)h[STAT_TC_STALLED];
  st->steps = step;
  st->time = sc[0];
  st->dt = sc[1];
  st->smax = sc[2];
  return PHL_OK;
}

int phl_reset_status(phl_ctx *ctx) {
  if (!ctx) return PHL_E_INVALID;
  CK(cudaSetDevice(ctx->cfg.device));
  CK(cudaMemsetAsync(ctx->stat, 0, sizeof(unsigned long long) * STAT_COUNT, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return PHL_OK;
}

void *phl_device_field(phl_ctx *ctx, const char *name) {
  if (!ctx || !name) return nullptr;
  std::string n(name);
  if (n == "prim") return ctx->W[ctx->cur];
  if (n == "U") return ctx->U;
  if (n == "U0") return ctx->U0;
  if (n == "eint") return ctx->eint;
  if (n == "temp") return ctx->temp;
  if (n == "gammaf") return ctx->gam[ctx->cur];
  if (n == "b_cc") return ctx->bcc;
  if (n == "b_x1") return ctx->bf[0];
  if (n == "b_x2") return ctx->bf[1];
  if (n == "b_x3") return ctx->bf[2];
  if (n == "prim_dev32") return ctx->Wf[ctx->cur];
  if (n == "gammaf_dev32") return ctx->gf[ctx->cur];
  if (n == "b_cc32") return ctx->bccf;
  // CT scratch of the last stage: face EMFs [3][faces] and mass-flux signs per face direction,
  // corner EMFs per axis (FP64 form, and the FP32 arrays of the split form with suffix 32)
  static const char *dn[3] = {"1", "2", "3"};
  for (int d = 0; d < 3; ++d) {
    if (n == std::string("emf_x") + dn[d]) return ctx->emf[d];
    if (n == std::string("sign_x") + dn[d]) return ctx->sgnf[d];
    if (n == std::string("emf_corner") + dn[d]) return ctx->cor[d];
    if (n == std::string("emf_x") + dn[d] + "_32") return ctx->femf[d];
    if (n == std::string("sign_x") + dn[d] + "_32") return ctx->fsgn[d];
    if (n == std::string("emf_corner") + dn[d] + "_32") return ctx->fcor[d];
  }
  return nullptr;
}

void *phl_stream(phl_ctx *ctx) { return ctx ? (void *)ctx->stream : nullptr; }

// ---- the EoS batch and the MLP live in phl_eos_batch.cuh / phl_mlp.cu
int phl_eos_invert_batch_device(phl_ctx *ctx, long long n, const double *rho, const double *e,
                                const double *abar, const double *zbar, double *T_inout, double *p,
                                double *cs, int *iters, int guess) {
  if (!ctx || n < 0 || !rho || !e || !abar || !zbar || !T_inout) return PHL_E_INVALID;
  if (!ctx->table_loaded) return PHL_E_NO_TABLE;
  CK(cudaSetDevice(ctx->cfg.device));
  return ctx->eos.invert(ctx->helm, ctx->stream, n, rho, e, abar, zbar, T_inout, p, cs, iters, guess, ctx->stat);
}

int phl_eos_energy_device(phl_ctx *ctx, long long n, const double *rho, const double *T, const double *abar,
                          const double *zbar, double *e) {
  if (!ctx || n < 0 || !rho || !T || !abar || !zbar || !e) return PHL_E_INVALID;
  if (!ctx->table_loaded) return PHL_E_NO_TABLE;
  CK(cudaSetDevice(ctx->cfg.device));
  return ctx->eos.energy(ctx->helm, ctx->stream, n, rho, T, abar, zbar, e);
}

int phl_eos_invert_batch(phl_ctx *ctx, long long n, const double *rho, const double *e, const double *abar,
                         const double *zbar, double *T_inout, double *p, double *cs, int *iters, int guess) {
  if (!ctx || n < 0 || !rho || !e || !abar || !zbar || !T_inout) return PHL_E_INVALID;
  if (!ctx->table_loaded) return PHL_E_NO_TABLE;
  CK(cudaSetDevice(ctx->cfg.device));
  return ctx->eos.invert_host(ctx->helm, ctx->stream, n, rho, e, abar, zbar, T_inout, p, cs, iters, guess, ctx->stat);
}

}  // extern "C"

// ---- allocation-free EoS batch inversion.  Device copies of inputs and outputs live in one
// file-scope array per device image.  Host code must never hand `g_noalloc_scratch` to a kernel
// or a copy: in host code the name is only a stand-in for the symbol, and its device address is
// obtained once per device with cudaGetSymbolAddress.
namespace {
constexpr int NOALLOC_FIELDS = 7;  // rho, e, abar, zbar, T, p, cs
static __device__ __align__(256) double g_noalloc_scratch[NOALLOC_FIELDS * PHL_NOALLOC_MAX_SAMPLES];
static __device__ __align__(256) int g_noalloc_iters[PHL_NOALLOC_MAX_SAMPLES];
// queue of rejected learned guesses: count, then one entry per sample
static __device__ __align__(256) unsigned long long g_noalloc_queue[PHL_NOALLOC_MAX_SAMPLES + 1];
constexpr int NOALLOC_MAX_DEVICES = 64;
double *g_noalloc_dev[NOALLOC_MAX_DEVICES] = {};
int *g_noalloc_idev[NOALLOC_MAX_DEVICES] = {};
unsigned long long *g_noalloc_qdev[NOALLOC_MAX_DEVICES] = {};

int noalloc_symbol(void **dst, const void *symbol, const char *name) {
  cudaError_t e = cudaGetSymbolAddress(dst, symbol);
  if (e == cudaSuccess) return PHL_OK;
  g_last_error = std::string("cudaGetSymbolAddress(") + name + "): " + cudaGetErrorString(e);
  return PHL_E_CUDA;
}

std::mutex g_noalloc_mutex;

// once per device, with that device current; the mutex makes the first calls of several host
// threads on one device look the addresses up once
int noalloc_setup(int device, double **buf, int **ibuf, unsigned long long **queue) {
  if (device < 0 || device >= NOALLOC_MAX_DEVICES) return PHL_E_INVALID;
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!g_noalloc_dev[device]) {
    void *p = nullptr, *q = nullptr, *r = nullptr;
    int rc;
    if ((rc = noalloc_symbol(&p, g_noalloc_scratch, "g_noalloc_scratch"))) return rc;
    if ((rc = noalloc_symbol(&q, g_noalloc_iters, "g_noalloc_iters"))) return rc;
    if ((rc = noalloc_symbol(&r, g_noalloc_queue, "g_noalloc_queue"))) return rc;
    g_noalloc_idev[device] = static_cast<int *>(q);
    g_noalloc_qdev[device] = static_cast<unsigned long long *>(r);
    g_noalloc_dev[device] = static_cast<double *>(p);
  }
  *buf = g_noalloc_dev[device];
  *ibuf = g_noalloc_idev[device];
  *queue = g_noalloc_qdev[device];
  return PHL_OK;
}
}  // namespace

extern "C" int phl_eos_invert_batch_noalloc(phl_ctx *ctx, long long n, const double *rho, const double *e,
                                            const double *abar, const double *zbar, double *T_inout,
                                            double *p, double *cs, int *iters, int guess) {
  if (!ctx || n < 0 || !rho || !e || !abar || !zbar || !T_inout) return PHL_E_INVALID;
  if (n > PHL_NOALLOC_MAX_SAMPLES) {
    g_last_error = "phl_eos_invert_batch_noalloc: n exceeds PHL_NOALLOC_MAX_SAMPLES";
    return PHL_E_TOO_LARGE;
  }
  if (!ctx->table_loaded) return PHL_E_NO_TABLE;
  if (guess < 0 || guess > 2) return PHL_E_INVALID;
  if (guess == 1 && !ctx->eos.mlp.ready) return PHL_E_STATE;
  if (n == 0) return PHL_OK;
  CK(cudaSetDevice(ctx->cfg.device));
  double *buf = nullptr;
  int *ibuf = nullptr;
  unsigned long long *queue = nullptr;
  int rc = noalloc_setup(ctx->cfg.device, &buf, &ibuf, &queue);
  if (rc) return rc;
  cudaStream_t s = ctx->stream;
  const size_t M = PHL_NOALLOC_MAX_SAMPLES, b = sizeof(double) * (size_t)n;
  double *d_rho = buf, *d_e = buf + M, *d_a = buf + 2 * M, *d_z = buf + 3 * M, *d_T = buf + 4 * M;
  double *d_p = buf + 5 * M, *d_c = buf + 6 * M;
  // every element the kernel reads is copied in first; it writes every output it is asked for,
  // so nothing left in the array by an earlier call is ever read
  CK(cudaMemcpyAsync(d_rho, rho, b, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(d_e, e, b, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(d_a, abar, b, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(d_z, zbar, b, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(d_T, T_inout, b, cudaMemcpyHostToDevice, s));
  CK((cudaError_t)eos_launch(ctx->helm, s, n, d_rho, d_e, d_a, d_z, d_T, p ? d_p : nullptr, cs ? d_c : nullptr,
                             iters ? ibuf : nullptr, guess, ctx->eos.mlp.weights(), ctx->stat, queue,
                             ctx->eos.sm_count()));
  CK(cudaMemcpyAsync(T_inout, d_T, b, cudaMemcpyDeviceToHost, s));
  if (p) CK(cudaMemcpyAsync(p, d_p, b, cudaMemcpyDeviceToHost, s));
  if (cs) CK(cudaMemcpyAsync(cs, d_c, b, cudaMemcpyDeviceToHost, s));
  if (iters) CK(cudaMemcpyAsync(iters, ibuf, sizeof(int) * (size_t)n, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  return PHL_OK;
}

extern "C" {

int phl_mlp_train(phl_ctx *ctx, long long n, unsigned long long seed, int epochs, int batch, double lr,
                  double *final_loss) {
  if (!ctx || n <= 0 || epochs < 0 || batch <= 0) return PHL_E_INVALID;
  if (!ctx->table_loaded) return PHL_E_NO_TABLE;
  CK(cudaSetDevice(ctx->cfg.device));
  int rc = ctx->eos.mlp_train(ctx->helm, ctx->stream, n, seed, epochs, batch, lr, final_loss);
  ctx->drop_graphs();  // step graphs bake the network's parameters into their kernels
  ctx->mlp_small_ok = false;
  if (rc == 0) {
    std::vector<float> p(MLP_NPARAM);
    rc = ctx->eos.mlp_get(ctx->stream, p.data());
    if (rc == 0) {
      mlp_small_from_params(p.data(), ctx->mlp_small);
      ctx->mlp_small_ok = true;
    }
  }
  return rc;
}

int phl_mlp_set_sample_range(phl_ctx *ctx, const double *lo, const double *hi) {
  if (!ctx) return PHL_E_INVALID;
  MlpRange r;
  if (lo) {
    if (!hi) return PHL_E_INVALID;
    for (int k = 0; k < 4; ++k)
      if (!std::isfinite(lo[k]) || !std::isfinite(hi[k]) || lo[k] > hi[k]) return PHL_E_INVALID;
    if (lo[2] < 1.0 || lo[3] < 1.0) return PHL_E_INVALID;
    if (ctx->table_loaded && (lo[1] < std::log10(ctx->helm.Tl) || hi[1] > std::log10(ctx->helm.Th))) {
      g_last_error = "phl_mlp_set_sample_range: the log10 T range leaves the table";
      return PHL_E_INVALID;
    }
    r.lrho[0] = lo[0]; r.lrho[1] = hi[0];
    r.lT[0] = lo[1]; r.lT[1] = hi[1];
    r.abar[0] = lo[2]; r.abar[1] = hi[2];
    r.zbar[0] = lo[3]; r.zbar[1] = hi[3];
  }
  ctx->eos.mlp.range = r;
  return PHL_OK;
}

int phl_mlp_gradient(phl_ctx *ctx, long long n, const float *features, const float *targets, float *grad,
                     double *loss) {
  if (!ctx || n <= 0 || !features || !targets || !grad) return PHL_E_INVALID;
  CK(cudaSetDevice(ctx->cfg.device));
  return ctx->eos.mlp_gradient(ctx->stream, n, features, targets, grad, loss);
}

int phl_mlp_get_params(phl_ctx *ctx, float *params) {
  if (!ctx || !params) return PHL_E_INVALID;
  CK(cudaSetDevice(ctx->cfg.device));
  return ctx->eos.mlp_get(ctx->stream, params);
}

int phl_mlp_set_params(phl_ctx *ctx, const float *params) {
  if (!ctx || !params) return PHL_E_INVALID;
  CK(cudaSetDevice(ctx->cfg.device));
  int rc = ctx->eos.mlp_set(ctx->stream, params);
  ctx->drop_graphs();
  ctx->mlp_small_ok = rc == 0;
  if (rc == 0) mlp_small_from_params(params, ctx->mlp_small);
  return rc;
}

int phl_mlp_infer_device(phl_ctx *ctx, long long n, const float *features, float *out) {
  if (!ctx || n < 0 || !features || !out) return PHL_E_INVALID;
  CK(cudaSetDevice(ctx->cfg.device));
  return ctx->eos.mlp_infer(ctx->stream, n, features, out, ctx->stat + STAT_TC_STALLED);
}

}  // extern "C"
