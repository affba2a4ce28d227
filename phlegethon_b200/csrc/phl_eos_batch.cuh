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
#include <string>
#include "phl_device.cuh"
#include "phl_mlp.cuh"

#define PHL_GUESS_BRACKET 2

namespace phl {

__device__ __forceinline__ double bracket_guess(const HelmTable &h, double rho, double e, double abar, double zbar) {
  int lo = 0, hi = h.nT - 1;
  double elo, ehi, dd;
  helm_given2(h, rho, __ldg(h.T + lo), abar, zbar, elo, dd, false);
  if (e <= elo) return __ldg(h.T + lo);
  helm_given2(h, rho, __ldg(h.T + hi) * 0.999999, abar, zbar, ehi, dd, false);
  if (e >= ehi) return __ldg(h.T + hi) * 0.999999;
  while (hi - lo > 1) {
    int mid = (lo + hi) >> 1;
    double em;
    helm_given2(h, rho, __ldg(h.T + mid), abar, zbar, em, dd, false);
    if (em <= e) { lo = mid; elo = em; } else { hi = mid; ehi = em; }
  }
  double t0 = __ldg(h.T + lo), t1 = __ldg(h.T + hi);
  double w = (e - elo) / (ehi - elo);
  return t0 + w * (t1 - t0);
}

__global__ void k_eos_energy(HelmTable h, long long n, const double *rho, const double *T, const double *abar,
                             const double *zbar, double *e) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  double E, dd;
  helm_given2(h, rho[t], T[t], abar[t], zbar[t], E, dd, false);
  e[t] = E;
}

// stat: [0] calls [1] iterations [2] non-converged [3] clamped [4] mlp accepted [5] mlp rejected
__global__ void __launch_bounds__(128) k_eos_invert(HelmTable h, long long n, const double *rho, const double *e,
                                                    const double *abar, const double *zbar, double *T,
                                                    double *p, double *cs, int *iters, int guess, MlpWeights mw,
                                                    unsigned long long *stat) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long ncall = 0, nit = 0, nnc = 0, ncl = 0, nacc = 0, nrej = 0;
  if (t < n) {
    double r = rho[t], ee = e[t], ab = abar[t], zb = zbar[t];
    double Tg;
    int used = 0, clamped = 0;
    bool done = false;
    if (guess == 1) {
      // learned guess, judged by at most 3 reference Newton iterations
      float feat[4];
      mlp_features(r, ee, ab, zb, feat);
      double Ttry = exp10((double)mlp_forward_scalar(mw, feat));
      Ttry = fmin(fmax(Ttry, h.Tl * 1.000001), h.Th * 0.999999);
      int cl = 0;
      bool conv = false;
      int it = helm_rhoe_newton(h, r, ee, ab, zb, Ttry, 3, cl, &conv);
      used = it;
      if (conv && cl == 0) {
        Tg = Ttry;
        done = true;
        nacc = 1;
      } else {
        nrej = 1;
        Tg = bracket_guess(h, r, ee, ab, zb);
      }
    } else if (guess == PHL_GUESS_BRACKET) {
      Tg = bracket_guess(h, r, ee, ab, zb);
    } else {
      Tg = T[t];
    }
    if (!done) {
      bool conv = false;
      int it = helm_rhoe_newton(h, r, ee, ab, zb, Tg, 100, clamped, &conv);
      used += it;
      nnc = !conv;
    }
    ncall = 1;
    nit = used;
    ncl = clamped;
    T[t] = Tg;
    if (p || cs) {
      double P, E, s, cv;
      helm_given_full(h, r, Tg, ab, zb, P, E, s, cv);
      if (p) p[t] = P;
      if (cs) cs[t] = s;
    }
    if (iters) iters[t] = used;
  }
  unsigned mask = 0xffffffffu;
  unsigned long long v[6] = {ncall, nit, nnc, ncl, nacc, nrej};
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    unsigned long long x = v[q];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(mask, x, o);
    if ((threadIdx.x & 31) == 0 && x) atomicAdd(stat + q, x);
  }
}

struct EosBatch {
  Mlp mlp;
  double *hbuf = nullptr;  // staging for the host-pointer variant
  size_t hbytes = 0;
  int *ibuf = nullptr;
  size_t ibytes = 0;

  void release() {
    if (hbuf) cudaFree(hbuf);
    if (ibuf) cudaFree(ibuf);
    hbuf = nullptr;
    ibuf = nullptr;
    mlp.release();
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
    if (guess == 1 && !mlp.ready) return -4;
    if (n == 0) return 0;
    k_eos_invert<<<(unsigned)((n + 127) / 128), 128, 0, s>>>(h, n, rho, e, abar, zbar, T, p, cs, iters, guess,
                                                             mlp.weights(), stat);
    if (cudaGetLastError() != cudaSuccess) return -2;
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
  int mlp_get(cudaStream_t s, float *p) { return mlp.get(s, p); }
  int mlp_set(cudaStream_t s, const float *p) { return mlp.set(s, p); }
  int mlp_infer(cudaStream_t s, long long n, const float *f, float *o) { return mlp.infer(s, n, f, o); }
};

}  // namespace phl
