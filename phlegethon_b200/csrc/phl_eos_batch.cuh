// phl_eos_batch.cuh -- batched Helmholtz (rho, e) -> T inversion (helm_rhoe_given,
// source/source.F90:24982-25019) on independent samples, with three initial guesses:
//   PHL_GUESS_WARM     caller-provided T (the reference's warm start, source.F90:13649)
//   PHL_GUESS_MLP      learned guess (phl_mlp.cuh), judged by <= 3 Newton iterations
//   PHL_GUESS_BRACKET  cold guess: bisection over the table's T nodes for E(rho,T_j) <= e,
//                      then linear interpolation of E between the bracketing nodes
// Newton always finishes to the reference tolerance (helm_tol = 1e-11), so only the iteration
// count depends on the guess.
#pragma once
#include <cuda_runtime.h>
#include <algorithm>
#include <cstdlib>
#include <string>
#include "phl_device.cuh"
#include "phl_mlp.cuh"

#define PHL_GUESS_BRACKET 2
#ifndef PHL_GUESS_MLP
#define PHL_GUESS_MLP 1
#endif

namespace phl {

constexpr int EOS_MINB_DEFAULT = 4;

// cold guess; returns the number of EoS evaluations the search used
__device__ __forceinline__ int bracket_guess(const HelmTable &h, double rho, double e, double abar, double zbar,
                                             double &Tg) {
  int lo = 0, hi = h.nT - 1;
  double elo, ehi, dd;
  helm_given2(h, rho, __ldg(h.T + lo), abar, zbar, elo, dd, false);
  if (e <= elo) { Tg = __ldg(h.T + lo); return 1; }
  helm_given2(h, rho, __ldg(h.T + hi) * 0.999999, abar, zbar, ehi, dd, false);
  if (e >= ehi) { Tg = __ldg(h.T + hi) * 0.999999; return 2; }
  int evals = 2;
  while (hi - lo > 1) {
    int mid = (lo + hi) >> 1;
    double em;
    helm_given2(h, rho, __ldg(h.T + mid), abar, zbar, em, dd, false);
    ++evals;
    if (em <= e) { lo = mid; elo = em; } else { hi = mid; ehi = em; }
  }
  double t0 = __ldg(h.T + lo), t1 = __ldg(h.T + hi);
  double w = (e - elo) / (ehi - elo);
  Tg = t0 + w * (t1 - t0);
  return evals;
}

__global__ void k_eos_energy(HelmTable h, long long n, const double *rho, const double *T, const double *abar,
                             const double *zbar, double *e) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  double E, dd;
  helm_given2(h, rho[t], T[t], abar[t], zbar[t], E, dd, false);
  e[t] = E;
}

// per-warp sums of the batch statistics into the context's counters
// (slots: calls, iterations, non-converged, clamped, mlp accepted, mlp rejected, guess evaluations)
struct EosStat {
  unsigned long long v[7] = {0, 0, 0, 0, 0, 0, 0};
  __device__ __forceinline__ void flush(unsigned long long *stat) const {
    const int slot[7] = {STAT_NEWTON_CALLS, STAT_NEWTON_ITERS, STAT_NEWTON_NONCONV, STAT_NEWTON_CLAMP,
                         STAT_MLP_ACC,      STAT_MLP_REJ,      STAT_GUESS_EVALS};
#pragma unroll
    for (int q = 0; q < 7; ++q) {
      unsigned long long x = v[q];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
      if ((threadIdx.x & 31) == 0 && x) atomicAdd(stat + slot[q], x);
    }
  }
};

// outputs of one finished inversion
__device__ __forceinline__ void eos_finish(const HelmTable &h, long long t, double r, double ab, double zb,
                                           double Tg, int used, double *T, double *p, double *cs, int *iters) {
  T[t] = Tg;
  if (p || cs) {
    double P, E, snd, cv;
    helm_given_full(h, r, Tg, ab, zb, P, E, snd, cv);
    if (p) p[t] = P;
    if (cs) cs[t] = snd;
  }
  if (iters) iters[t] = used;
}

// Phase 1.  guess 0 / 2: warm or bracket guess and the full Newton.  guess 1: the learned guess
// (computed per block of 128 samples on the tensor cores), judged by at most 3 reference
// Newton iterations; a sample whose guess did not converge within them without a reset is
// appended to `queue` (queue[0] = count, then index | judged iterations << 56) for phase 2, so
// that the fallback runs in converged warps instead of stalling the accepted lanes.
// LEARNED selects the learned-guess instantiation (guess 1); the other carries no tensor-core code.
template <bool LEARNED, int MINB>
__global__ void __launch_bounds__(128, MINB) k_eos_invert(HelmTable h, long long n, const double *rho, const double *e,
                                                    const double *abar, const double *zbar, double *T,
                                                    double *p, double *cs, int *iters, int guess, MlpWeights mw,
                                                    unsigned long long *stat, unsigned long long *queue) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  EosStat st;
  float lT_mlp = 0.0f;
  double ecold = 0.0;
  if constexpr (LEARNED) {
    extern __shared__ __align__(128) unsigned char sm[];
    MlpUmmaSmem &S = *reinterpret_cast<MlpUmmaSmem *>(sm);
    float feat[4] = {0, 0, 0, 0};
    if (t < n) {
      ecold = mlp_cold_energy(h, rho[t], abar[t], zbar[t]);
      st.v[6] = 1;
      mlp_features(rho[t], e[t] - ecold, abar[t], zbar[t], feat);
    }
    lT_mlp = mlp_forward_cta(mw, feat, S, stat + STAT_TC_STALLED);
  }
  bool reject = false;
  int judged = 0;
  if (t < n) {
    const double r = rho[t], ee = e[t], ab = abar[t], zb = zbar[t];
    double Tg;
    int used = 0, clamped = 0;
    bool conv = false;
    if constexpr (LEARNED) {
      Tg = fmin(fmax(exp10((double)lT_mlp), h.Tl * 1.000001), h.Th * 0.999999);
      used = helm_rhoe_newton(h, r, ee, ab, zb, Tg, 3, clamped, &conv);
      st.v[3] = clamped;
      if (conv && clamped == 0) {
        st.v[0] = 1;
        st.v[1] = used;
        st.v[4] = 1;
        eos_finish(h, t, r, ab, zb, Tg, used, T, p, cs, iters);
      } else {
        reject = true;
        judged = used;
        st.v[5] = 1;
      }
    } else {
      if (guess == PHL_GUESS_BRACKET) st.v[6] = bracket_guess(h, r, ee, ab, zb, Tg);
      else Tg = T[t];
      used = helm_rhoe_newton(h, r, ee, ab, zb, Tg, 100, clamped, &conv);
      st.v[0] = 1;
      st.v[1] = used;
      st.v[2] = !conv;
      st.v[3] = clamped;
      eos_finish(h, t, r, ab, zb, Tg, used, T, p, cs, iters);
    }
  }
  if constexpr (LEARNED) {
    // warp-aggregated append of the rejected samples
    const unsigned mask = __ballot_sync(0xffffffffu, reject);
    if (mask) {
      const int lane = threadIdx.x & 31, leader = __ffs(mask) - 1;
      unsigned long long base = 0;
      if (lane == leader) base = atomicAdd(queue, (unsigned long long)__popc(mask));
      base = __shfl_sync(0xffffffffu, base, leader);
      if (reject)
        queue[1 + base + __popc(mask & ((1u << lane) - 1u))] =
            (unsigned long long)t | ((unsigned long long)judged << 56);
    }
  }
  st.flush(stat);
}

// Phase 2 of the learned guess: the reference Newton from the bracket guess for the rejected
// samples (grid-stride over the queue written by phase 1)
template <int MINB>
__global__ void __launch_bounds__(128, MINB) k_eos_fallback(HelmTable h, const unsigned long long *queue,
                                                      const double *rho, const double *e, const double *abar,
                                                      const double *zbar, double *T, double *p, double *cs,
                                                      int *iters, unsigned long long *stat) {
  const long long count = (long long)queue[0];
  const long long stride = (long long)gridDim.x * blockDim.x;
  const long long first = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  // every lane runs the same number of trips so the warp-level flush stays converged
  const long long trips = (count + stride - 1) / stride;
  EosStat st;
  for (long long k = 0; k < trips; ++k) {
    const long long q = first + k * stride;
    if (q < count) {
      const unsigned long long ent = queue[1 + q];
      const long long t = (long long)(ent & ((1ull << 56) - 1));
      const int judged = (int)(ent >> 56);
      const double r = rho[t], ee = e[t], ab = abar[t], zb = zbar[t];
      double Tg;
      st.v[6] += bracket_guess(h, r, ee, ab, zb, Tg);
      int clamped = 0;
      bool conv = false;
      const int used = helm_rhoe_newton(h, r, ee, ab, zb, Tg, 100, clamped, &conv);
      st.v[0] += 1;
      st.v[1] += judged + used;
      st.v[2] += !conv;
      st.v[3] += clamped;
      eos_finish(h, t, r, ab, zb, Tg, judged + used, T, p, cs, iters);
    }
  }
  st.flush(stat);
}

// Launch the inversion on stream s (no synchronisation).  `queue` (n + 1 entries) is needed for
// the learned guess only.  Returns 0 or a cudaError_t.
// Resident blocks per SM the inversion kernels are compiled for: 4 caps them at 128 registers
// (2^24 samples on B200: learned guess 1.66e9 inversions/s, bracket 1.39e9, against 1.34e9 and
// 1.07e9 with 1, which lets the compiler keep the whole inlined evaluation in ~190 registers at
// two blocks per SM, and 1.17e9 / 1.04e9 with 6); PHL_EOS_MINB=1 or 3 selects the others.
inline int eos_minb() {
  static const int v = [] {
    const char *e = getenv("PHL_EOS_MINB");
    const int m = e ? atoi(e) : EOS_MINB_DEFAULT;
    return (m == 1 || m == 3 || m == 4) ? m : EOS_MINB_DEFAULT;
  }();
  return v;
}

template <int MINB>
inline int eos_launch_t(const HelmTable &h, cudaStream_t s, long long n, const double *rho, const double *e,
                        const double *abar, const double *zbar, double *T, double *p, double *cs, int *iters,
                        int guess, MlpWeights mw, unsigned long long *stat, unsigned long long *queue, int nsm) {
  const unsigned blocks = (unsigned)((n + 127) / 128);
  if (guess != PHL_GUESS_MLP) {
    k_eos_invert<false, MINB><<<blocks, 128, 0, s>>>(h, n, rho, e, abar, zbar, T, p, cs, iters, guess, mw, stat,
                                                      nullptr);
    return (int)cudaGetLastError();
  }
  const size_t sm = sizeof(MlpUmmaSmem);
  cudaError_t err = cudaFuncSetAttribute(k_eos_invert<true, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (err == cudaSuccess) err = cudaMemsetAsync(queue, 0, sizeof(unsigned long long), s);
  if (err != cudaSuccess) return (int)err;
  k_eos_invert<true, MINB><<<blocks, 128, sm, s>>>(h, n, rho, e, abar, zbar, T, p, cs, iters, guess, mw, stat, queue);
  // enough resident blocks to cover every SM several times; the loop covers any queue length
  const unsigned fb = (unsigned)std::min<long long>((long long)nsm * 8, (long long)blocks);
  k_eos_fallback<MINB><<<fb, 128, 0, s>>>(h, queue, rho, e, abar, zbar, T, p, cs, iters, stat);
  return (int)cudaGetLastError();
}

// Launch the inversion on stream s (no synchronisation).  `queue` (n + 1 entries) is needed for
// the learned guess only.  Returns 0 or a cudaError_t.
inline int eos_launch(const HelmTable &h, cudaStream_t s, long long n, const double *rho, const double *e,
                      const double *abar, const double *zbar, double *T, double *p, double *cs, int *iters,
                      int guess, MlpWeights mw, unsigned long long *stat, unsigned long long *queue, int nsm) {
  switch (eos_minb()) {
    case 3: return eos_launch_t<3>(h, s, n, rho, e, abar, zbar, T, p, cs, iters, guess, mw, stat, queue, nsm);
    case 4: return eos_launch_t<4>(h, s, n, rho, e, abar, zbar, T, p, cs, iters, guess, mw, stat, queue, nsm);
    default: return eos_launch_t<1>(h, s, n, rho, e, abar, zbar, T, p, cs, iters, guess, mw, stat, queue, nsm);
  }
}

struct EosBatch {
  Mlp mlp;
  double *hbuf = nullptr;  // staging for the host-pointer variant
  size_t hbytes = 0;
  int *ibuf = nullptr;
  size_t ibytes = 0;
  unsigned long long *queue = nullptr;  // rejected learned guesses (count + entries)
  long long qcap = 0;
  int nsm = 0;

  void release() {
    if (hbuf) cudaFree(hbuf);
    if (ibuf) cudaFree(ibuf);
    if (queue) cudaFree(queue);
    hbuf = nullptr;
    ibuf = nullptr;
    queue = nullptr;
    qcap = 0;
    mlp.release();
  }
  int sm_count() {
    if (!nsm) {
      int dev = 0;
      if (cudaGetDevice(&dev) != cudaSuccess ||
          cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        nsm = 148;
    }
    return nsm;
  }
  int energy(const HelmTable &h, cudaStream_t s, long long n, const double *rho, const double *T,
             const double *abar, const double *zbar, double *e) {
    if (n == 0) return 0;
    k_eos_energy<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(h, n, rho, T, abar, zbar, e);
    if (cudaGetLastError() != cudaSuccess) return -2;
    if (cudaStreamSynchronize(s) != cudaSuccess) return -2;
    return 0;
  }
  int invert(const HelmTable &h, cudaStream_t s, long long n, const double *rho, const double *e,
             const double *abar, const double *zbar, double *T, double *p, double *cs, int *iters, int guess,
             unsigned long long *stat) {
    if (guess < 0 || guess > 2) return -1;
    if (guess == PHL_GUESS_MLP && !mlp.ready) return -4;
    if (n == 0) return 0;
    if (guess == PHL_GUESS_MLP && qcap < n + 1) {
      if (queue) cudaFree(queue);
      queue = nullptr;
      qcap = 0;
      if (cudaMalloc(&queue, sizeof(unsigned long long) * (size_t)(n + 1)) != cudaSuccess) return -2;
      qcap = n + 1;
    }
    if (eos_launch(h, s, n, rho, e, abar, zbar, T, p, cs, iters, guess, mlp.weights(), stat, queue, sm_count()))
      return -2;
    if (cudaStreamSynchronize(s) != cudaSuccess) return -2;
    return 0;
  }
  int invert_host(const HelmTable &h, cudaStream_t s, long long n, const double *rho, const double *e,
                  const double *abar, const double *zbar, double *T, double *p, double *cs, int *iters, int guess,
                  unsigned long long *stat) {
    if (n == 0) return 0;
    size_t need = sizeof(double) * (size_t)n * 7;
    if (need > hbytes) {
      if (hbuf) cudaFree(hbuf);
      hbuf = nullptr;
      if (cudaMalloc(&hbuf, need) != cudaSuccess) { hbytes = 0; return -2; }
      hbytes = need;
    }
    if (iters && sizeof(int) * (size_t)n > ibytes) {
      if (ibuf) cudaFree(ibuf);
      ibuf = nullptr;
      if (cudaMalloc(&ibuf, sizeof(int) * (size_t)n) != cudaSuccess) { ibytes = 0; return -2; }
      ibytes = sizeof(int) * (size_t)n;
    }
    double *d_rho = hbuf, *d_e = hbuf + n, *d_a = hbuf + 2 * n, *d_z = hbuf + 3 * n, *d_T = hbuf + 4 * n;
    double *d_p = hbuf + 5 * n, *d_c = hbuf + 6 * n;
    size_t b = sizeof(double) * (size_t)n;
    if (cudaMemcpyAsync(d_rho, rho, b, cudaMemcpyHostToDevice, s) || cudaMemcpyAsync(d_e, e, b, cudaMemcpyHostToDevice, s) ||
        cudaMemcpyAsync(d_a, abar, b, cudaMemcpyHostToDevice, s) || cudaMemcpyAsync(d_z, zbar, b, cudaMemcpyHostToDevice, s) ||
        cudaMemcpyAsync(d_T, T, b, cudaMemcpyHostToDevice, s))
      return -2;
    int rc = invert(h, s, n, d_rho, d_e, d_a, d_z, d_T, p ? d_p : nullptr, cs ? d_c : nullptr,
                    iters ? ibuf : nullptr, guess, stat);
    if (rc) return rc;
    if (cudaMemcpyAsync(T, d_T, b, cudaMemcpyDeviceToHost, s)) return -2;
    if (p && cudaMemcpyAsync(p, d_p, b, cudaMemcpyDeviceToHost, s)) return -2;
    if (cs && cudaMemcpyAsync(cs, d_c, b, cudaMemcpyDeviceToHost, s)) return -2;
    if (iters && cudaMemcpyAsync(iters, ibuf, sizeof(int) * (size_t)n, cudaMemcpyDeviceToHost, s)) return -2;
    if (cudaStreamSynchronize(s) != cudaSuccess) return -2;
    return 0;
  }
  int mlp_train(const HelmTable &h, cudaStream_t s, long long n, unsigned long long seed, int epochs, int batch,
                double lr, double *final_loss) {
    return mlp.train(h, s, n, seed, epochs, batch, lr, final_loss);
  }
  int mlp_gradient(cudaStream_t s, long long n, const float *f, const float *t, float *g, double *loss) {
    return mlp.gradient_host(s, n, f, t, g, loss);
  }
  int mlp_get(cudaStream_t s, float *p) { return mlp.get(s, p); }
  int mlp_set(cudaStream_t s, const float *p) { return mlp.set(s, p); }
  int mlp_infer(cudaStream_t s, long long n, const float *f, float *o, unsigned long long *stalled) {
    return mlp.infer(s, n, f, o, stalled);
  }
};

}  // namespace phl
