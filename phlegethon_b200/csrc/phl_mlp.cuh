// phl_mlp.cuh -- learned initial temperature guess for the (rho, e) -> T Newton inversion.
// No reference counterpart.  A 4-64-64-1 MLP maps (log10 rho, log10 e, Abar, Zbar), normalised,
// to log10 T.  Parameters live in FP32 (master copy for Adam) and BF16 (tensor-core operands).
#pragma once
#include <cuda_runtime.h>
#include <cuda_bf16.h>

namespace phl {

constexpr int MLP_IN = 4, MLP_H = 64;
constexpr int MLP_NPARAM = MLP_IN * MLP_H + MLP_H + MLP_H * MLP_H + MLP_H + MLP_H + 1;

// fixed input/output normalisation over config-4 style ranges
__device__ __forceinline__ void mlp_features(double rho, double e, double abar, double zbar, float f[4]) {
  f[0] = (float)((log10(rho) - 3.5) / 5.5);
  f[1] = (float)((log10(fabs(e) + 1e-300) - 16.0) / 6.0);
  f[2] = (float)((abar - 28.5) / 27.5);
  f[3] = (float)((zbar - 14.0) / 14.0);
}
__host__ __device__ __forceinline__ float mlp_out_scale() { return 3.0f; }
__host__ __device__ __forceinline__ float mlp_out_shift() { return 7.0f; }

struct MlpWeights {
  const float *w;  // FP32 params: W1[64][4], b1[64], W2[64][64], b2[64], W3[64], b3
};

// scalar FP32 forward pass of one sample (used where one thread owns one sample)
__device__ __forceinline__ float mlp_forward_scalar(const MlpWeights &m, const float x[4]) {
  const float *W1 = m.w, *b1 = W1 + MLP_H * MLP_IN, *W2 = b1 + MLP_H, *b2 = W2 + MLP_H * MLP_H;
  const float *W3 = b2 + MLP_H, *b3 = W3 + MLP_H;
  float h1[MLP_H];
#pragma unroll
  for (int o = 0; o < MLP_H; ++o) {
    float a = __ldg(b1 + o);
#pragma unroll
    for (int i = 0; i < MLP_IN; ++i) a += __ldg(W1 + o * MLP_IN + i) * x[i];
    h1[o] = a > 0.f ? a : 0.f;
  }
  float out = __ldg(b3);
  for (int o = 0; o < MLP_H; ++o) {
    float a = __ldg(b2 + o);
#pragma unroll
    for (int i = 0; i < MLP_H; ++i) a += __ldg(W2 + o * MLP_H + i) * h1[i];
    out += __ldg(W3 + o) * (a > 0.f ? a : 0.f);
  }
  return out * mlp_out_scale() + mlp_out_shift();
}

struct Mlp {
  bool ready = false;
  float *params = nullptr;
  void release() {
    if (params) cudaFree(params);
    params = nullptr;
    ready = false;
  }
  MlpWeights weights() const { return MlpWeights{params}; }
  int alloc() {
    if (params) return 0;
    if (cudaMalloc(&params, sizeof(float) * MLP_NPARAM) != cudaSuccess) return -2;
    return 0;
  }
  int set(cudaStream_t s, const float *h) {
    if (alloc()) return -2;
    if (cudaMemcpyAsync(params, h, sizeof(float) * MLP_NPARAM, cudaMemcpyHostToDevice, s) != cudaSuccess) return -2;
    if (cudaStreamSynchronize(s) != cudaSuccess) return -2;
    ready = true;
    return 0;
  }
  int get(cudaStream_t s, float *h) {
    if (!params) return -4;
    if (cudaMemcpyAsync(h, params, sizeof(float) * MLP_NPARAM, cudaMemcpyDeviceToHost, s) != cudaSuccess) return -2;
    if (cudaStreamSynchronize(s) != cudaSuccess) return -2;
    return 0;
  }
  int train(const HelmTable &, cudaStream_t, long long, unsigned long long, int, int, double, double *) { return -6; }
  int infer(cudaStream_t, long long, const float *, float *) { return -6; }
};

}  // namespace phl
