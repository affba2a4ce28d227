// phl_mlp.cuh -- learned initial temperature guess for the (rho, e) -> T Newton inversion.
// No reference counterpart.  A 4-64-64-1 MLP maps normalised (log10 rho, log10 e, Abar, Zbar)
// to log10 T.  Parameters: FP32 master copy (Adam) plus a BF16 copy of the 64x64 hidden layer,
// which runs on the tensor cores (BF16 operands, FP32 accumulate): tcgen05 MMAs with the
// accumulator in tensor memory for inference, warp-level MMAs for the 64-sample training tiles;
// the 4->64 input layer and the 64->1 output layer are FP32 on the CUDA cores.
//
// Training (all on the device): samples are drawn with a counter-based hash over the EoS
// benchmark ranges and labelled by the forward EoS (helm_rhoT_given2); each step a CTA takes 64
// samples through forward and backward passes (three 64x64x64 tensor-core products: layer-2
// forward, dH1 = dH2 W2, dW2 = dH2^T H1), writes its partial gradient, a second kernel sums the
// partials in a fixed order (deterministic), and a third applies Adam.
#pragma once
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <mma.h>
#include "phl_device.cuh"
#include "phl_umma.cuh"

namespace phl {

constexpr int MLP_IN = 4, MLP_H = 64;
// parameter layout: W1[64][4], b1[64], W2[64][64] (out, in), b2[64], W3[64], b3
constexpr int MLP_OFF_W1 = 0, MLP_OFF_B1 = 256, MLP_OFF_W2 = 320, MLP_OFF_B2 = 4416, MLP_OFF_W3 = 4480,
              MLP_OFF_B3 = 4544, MLP_NPARAM = 4545;
constexpr int MLP_TILE = 64;  // samples per CTA in training

// Inputs: log10 rho, log10 of the thermal part of the specific energy e_th = e - E(rho, T_lo)
// (T_lo the table's lowest temperature), Abar, Zbar, each mapped to about [-1, 1] over the EoS
// benchmark ranges.  Subtracting the cold energy removes the T-independent degenerate part, so
// log T stays a smooth function of the inputs where the electrons are degenerate.
__host__ __device__ __forceinline__ void mlp_features(double rho, double e_th, double abar, double zbar,
                                                      float f[4]) {
  f[0] = (float)((log10(rho) - 3.5) / 5.5);
  f[1] = (float)((log10(fmax(e_th, 1e-300)) - 19.5) / 8.5);
  f[2] = (float)((abar - 28.5) / 27.5);
  f[3] = (float)((zbar - 14.0) / 14.0);
}
// cold (lowest-table-temperature) specific energy of the mixture at rho
__device__ __forceinline__ double mlp_cold_energy(const HelmTable &h, double rho, double abar, double zbar) {
  double E, dE;
  helm_given2(h, rho, __ldg(h.T), abar, zbar, E, dE, false);
  return E;
}
// Fixed (non-trained) skip connection: log10 of the temperature at which ideal ions plus
// radiation alone would hold e_th, (T_ion^-4 + T_rad^-4)^(-1/4) with T_ion = e_th Abar / (3/2 R)
// and T_rad = (e_th rho / a)^(1/4); both parts are the analytic terms the reference adds outside
// the table.  It is computed from the features, so the network maps features -> log10 T as
//   log10 T = prior(features) + MLP_OUT_SCALE * y + MLP_OUT_SHIFT,
// and the trained part only learns what the electron table contributes.
__host__ __device__ __forceinline__ float mlp_prior(const float f[4]) {
  const float lrho = 5.5f * f[0] + 3.5f, le = 8.5f * f[1] + 19.5f, abar = 27.5f * f[2] + 28.5f;
  const float l_ion = le + log10f(abar) - 8.095925f;        // log10(3/2 R)
  const float l_rad = 0.25f * (le + lrho + 14.121147f);     // -log10(a)
  const float m = fminf(l_ion, l_rad);
  return m - 0.25f * log10f(1.0f + exp10f(-4.0f * fabsf(l_ion - l_rad)));
}
constexpr float MLP_OUT_SCALE = 0.5f, MLP_OUT_SHIFT = -0.75f;

struct MlpWeights {
  const float *w;               // FP32 master parameters
  const __nv_bfloat16 *w2bf;    // BF16 copy of W2 (row-major [out][in])
};

// Training-sample distribution: log10 rho ~ U[lrho], log10 T ~ U[lT], Abar ~ U[abar], and
// Zbar ~ U[zbar] when zbar[1] > 0, else Zbar ~ U[1, max(Abar/2, 1)].  The default is the EoS
// benchmark range; a run can narrow it to the states it holds (a network fitted over a smaller
// range guesses closer).
struct MlpRange {
  double lrho[2] = {-2.0, 9.0}, lT[2] = {4.0, 10.0}, abar[2] = {1.0, 56.0}, zbar[2] = {1.0, -1.0};
};

// counter-based hash for the samples
__device__ __forceinline__ unsigned long long mix64(unsigned long long x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}
__device__ __forceinline__ double u01(unsigned long long seed, long long i, int c) {
  unsigned long long h = mix64(mix64(seed ^ (unsigned long long)i * 0x100000001B3ull) + (unsigned long long)c);
  return (double)(h >> 11) * (1.0 / 9007199254740992.0);
}

static __global__ void k_mlp_make_samples(HelmTable h, long long n, unsigned long long seed, MlpRange r, float *feat,
                                          float *target) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double lrho = r.lrho[0] + (r.lrho[1] - r.lrho[0]) * u01(seed, i, 0);
  double lT = r.lT[0] + (r.lT[1] - r.lT[0]) * u01(seed, i, 1);
  double abar = r.abar[0] + (r.abar[1] - r.abar[0]) * u01(seed, i, 2);
  double zbar = r.zbar[1] > 0.0 ? r.zbar[0] + (r.zbar[1] - r.zbar[0]) * u01(seed, i, 3)
                                : 1.0 + fmax(abar * 0.5 - 1.0, 0.0) * u01(seed, i, 3);
  double rho = exp10(lrho), T = exp10(lT), E, dE;
  helm_given2(h, rho, T, abar, zbar, E, dE, false);
  float f[4];
  mlp_features(rho, E - mlp_cold_energy(h, rho, abar, zbar), abar, zbar, f);
  for (int k = 0; k < 4; ++k) feat[i * 4 + k] = f[k];
  target[i] = (float)((lT - (double)mlp_prior(f) - MLP_OUT_SHIFT) / MLP_OUT_SCALE);
}

// ------------------------------------------------------------------ training step (one CTA = 64 samples)
// shared layout (bytes): X 64x4 f32 | T 64 f32 | H1 64x64 f32 | H1b 64x64 bf16 | W2b 64x64 bf16 |
// Z 64x64 f32 (Z2, later dH1) | G 64x64 bf16 (dH2) | Gf 64x64 f32 (dH2) | y 64 f32
struct MlpTrainSmem {
  float X[MLP_TILE][4];
  float T[MLP_TILE];
  float y[MLP_TILE];
  float H1[MLP_TILE][MLP_H];
  float Z[MLP_TILE][MLP_H];
  float Gf[MLP_TILE][MLP_H];
  alignas(32) __nv_bfloat16 H1b[MLP_TILE][MLP_H];
  alignas(32) __nv_bfloat16 W2b[MLP_H][MLP_H];
  alignas(32) __nv_bfloat16 Gb[MLP_TILE][MLP_H];
  alignas(32) float dW2[MLP_H][MLP_H];
};

static __global__ void __launch_bounds__(128) k_mlp_train_step(const float *params, const __nv_bfloat16 *w2bf,
                                                        const float *feat, const float *target, long long n,
                                                        long long offset, int batch, float *partial,
                                                        float *loss_partial) {
  using namespace nvcuda;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  MlpTrainSmem &S = *reinterpret_cast<MlpTrainSmem *>(smem_raw);
  const int tid = threadIdx.x, warp = tid >> 5;
  const float *W1 = params + MLP_OFF_W1, *b1 = params + MLP_OFF_B1, *b2 = params + MLP_OFF_B2;
  const float *W3 = params + MLP_OFF_W3, b3 = params[MLP_OFF_B3];
  const long long base = offset + (long long)blockIdx.x * MLP_TILE;
  // samples (wrapping around the training set)
  for (int q = tid; q < MLP_TILE * 4; q += blockDim.x) {
    long long s = (base + q / 4) % n;
    S.X[q / 4][q % 4] = feat[s * 4 + q % 4];
  }
  for (int q = tid; q < MLP_TILE; q += blockDim.x) S.T[q] = target[(base + q) % n];
  for (int q = tid; q < MLP_H * MLP_H; q += blockDim.x) S.W2b[q / MLP_H][q % MLP_H] = w2bf[q];
  __syncthreads();
  // layer 1 (FP32)
  for (int q = tid; q < MLP_TILE * MLP_H; q += blockDim.x) {
    int s = q / MLP_H, o = q % MLP_H;
    float a = b1[o];
#pragma unroll
    for (int k = 0; k < 4; ++k) a = fmaf(W1[o * 4 + k], S.X[s][k], a);
    a = fmaxf(a, 0.0f);
    S.H1[s][o] = a;
    S.H1b[s][o] = __float2bfloat16(a);
  }
  __syncthreads();
  // layer 2 on the tensor cores: Z[s][o] = sum_i H1[s][i] W2[o][i]; warp w owns rows 16w..16w+15
  {
    wmma::fragment<wmma::matrix_a, 16, 16, 16, __nv_bfloat16, wmma::row_major> a;
    wmma::fragment<wmma::matrix_b, 16, 16, 16, __nv_bfloat16, wmma::col_major> b;
    wmma::fragment<wmma::accumulator, 16, 16, 16, float> acc;
#pragma unroll
    for (int nt = 0; nt < 4; ++nt) {
      wmma::fill_fragment(acc, 0.0f);
#pragma unroll
      for (int kt = 0; kt < 4; ++kt) {
        wmma::load_matrix_sync(a, &S.H1b[16 * warp][16 * kt], MLP_H);
        wmma::load_matrix_sync(b, &S.W2b[16 * nt][16 * kt], MLP_H);  // B(k=i, n=o) = W2[o][i]
        wmma::mma_sync(acc, a, b, acc);
      }
      wmma::store_matrix_sync(&S.Z[16 * warp][16 * nt], acc, MLP_H, wmma::mem_row_major);
    }
  }
  __syncthreads();
  // bias + ReLU -> H2 (kept in Z), output layer, loss gradient
  for (int q = tid; q < MLP_TILE * MLP_H; q += blockDim.x) {
    int s = q / MLP_H, o = q % MLP_H;
    S.Z[s][o] = fmaxf(S.Z[s][o] + b2[o], 0.0f);
  }
  __syncthreads();
  if (tid < MLP_TILE) {
    float a = b3;
    for (int o = 0; o < MLP_H; ++o) a = fmaf(W3[o], S.Z[tid][o], a);
    float d = a - S.T[tid];
    S.y[tid] = 2.0f * d / (float)batch;  // dL/dy for L = mean (y - t)^2
    loss_partial[blockIdx.x * MLP_TILE + tid] = d * d;
  }
  __syncthreads();
  // dH2 = dy W3 * relu'(H2)
  for (int q = tid; q < MLP_TILE * MLP_H; q += blockDim.x) {
    int s = q / MLP_H, o = q % MLP_H;
    float g = S.Z[s][o] > 0.0f ? S.y[s] * W3[o] : 0.0f;
    S.Gf[s][o] = g;
    S.Gb[s][o] = __float2bfloat16(g);
  }
  __syncthreads();
  float *P = partial + (long long)blockIdx.x * MLP_NPARAM;
  // dW3, b3, b2 from FP32 H2 / dH2
  for (int o = tid; o < MLP_H; o += blockDim.x) {
    float gw3 = 0.0f, gb2 = 0.0f;
    for (int s = 0; s < MLP_TILE; ++s) {
      gw3 = fmaf(S.y[s], S.Z[s][o], gw3);
      gb2 += S.Gf[s][o];
    }
    P[MLP_OFF_W3 + o] = gw3;
    P[MLP_OFF_B2 + o] = gb2;
  }
  if (tid == 0) {
    float g = 0.0f;
    for (int s = 0; s < MLP_TILE; ++s) g += S.y[s];
    P[MLP_OFF_B3] = g;
  }
  __syncthreads();
  // tensor cores: dH1pre[s][i] = sum_o dH2[s][o] W2[o][i] (into Z) and
  // dW2[o][i] = sum_s dH2[s][o] H1[s][i]
  {
    wmma::fragment<wmma::matrix_a, 16, 16, 16, __nv_bfloat16, wmma::row_major> a;
    wmma::fragment<wmma::matrix_b, 16, 16, 16, __nv_bfloat16, wmma::row_major> b;
    wmma::fragment<wmma::matrix_a, 16, 16, 16, __nv_bfloat16, wmma::col_major> at;
    wmma::fragment<wmma::accumulator, 16, 16, 16, float> acc;
#pragma unroll
    for (int nt = 0; nt < 4; ++nt) {
      wmma::fill_fragment(acc, 0.0f);
#pragma unroll
      for (int kt = 0; kt < 4; ++kt) {
        wmma::load_matrix_sync(a, &S.Gb[16 * warp][16 * kt], MLP_H);     // A(s, o) = dH2[s][o]
        wmma::load_matrix_sync(b, &S.W2b[16 * kt][16 * nt], MLP_H);      // B(k=o, n=i) = W2[o][i]
        wmma::mma_sync(acc, a, b, acc);
      }
      wmma::store_matrix_sync(&S.Z[16 * warp][16 * nt], acc, MLP_H, wmma::mem_row_major);
    }
#pragma unroll
    for (int nt = 0; nt < 4; ++nt) {
      wmma::fill_fragment(acc, 0.0f);
#pragma unroll
      for (int kt = 0; kt < 4; ++kt) {
        wmma::load_matrix_sync(at, &S.Gb[16 * kt][16 * warp], MLP_H);    // A(o, s) = dH2[s][o]
        wmma::load_matrix_sync(b, &S.H1b[16 * kt][16 * nt], MLP_H);      // B(k=s, n=i) = H1[s][i]
        wmma::mma_sync(acc, at, b, acc);
      }
      wmma::store_matrix_sync(&S.dW2[16 * warp][16 * nt], acc, MLP_H, wmma::mem_row_major);
    }
  }
  __syncthreads();
  for (int q = tid; q < MLP_H * MLP_H; q += blockDim.x) P[MLP_OFF_W2 + q] = S.dW2[q / MLP_H][q % MLP_H];
  // dH1 = dH1pre * relu'(H1); dW1, db1 (FP32)
  for (int q = tid; q < MLP_TILE * MLP_H; q += blockDim.x) {
    int s = q / MLP_H, i = q % MLP_H;
    S.Z[s][i] = S.H1[s][i] > 0.0f ? S.Z[s][i] : 0.0f;
  }
  __syncthreads();
  for (int o = tid; o < MLP_H; o += blockDim.x) {
    float g[4] = {0, 0, 0, 0}, gb = 0.0f;
    for (int s = 0; s < MLP_TILE; ++s) {
      float d = S.Z[s][o];
      gb += d;
#pragma unroll
      for (int k = 0; k < 4; ++k) g[k] = fmaf(d, S.X[s][k], g[k]);
    }
    for (int k = 0; k < 4; ++k) P[MLP_OFF_W1 + o * 4 + k] = g[k];
    P[MLP_OFF_B1 + o] = gb;
  }
}

// fixed-order sum of the per-CTA partial gradients
static __global__ void k_mlp_reduce(const float *partial, int nblocks, float *grad) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= MLP_NPARAM) return;
  float s = 0.0f;
  for (int b = 0; b < nblocks; ++b) s += partial[(long long)b * MLP_NPARAM + p];
  grad[p] = s;
}

static __global__ void k_mlp_adam(float *params, const float *grad, float *m, float *v, float lr, float b1, float b2,
                           float eps, int step, __nv_bfloat16 *w2bf) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= MLP_NPARAM) return;
  float g = grad[p];
  float mm = b1 * m[p] + (1.0f - b1) * g;
  float vv = b2 * v[p] + (1.0f - b2) * g * g;
  m[p] = mm;
  v[p] = vv;
  float mh = mm / (1.0f - powf(b1, (float)step)), vh = vv / (1.0f - powf(b2, (float)step));
  float w = params[p] - lr * mh / (sqrtf(vh) + eps);
  params[p] = w;
  if (p >= MLP_OFF_W2 && p < MLP_OFF_B2) w2bf[p - MLP_OFF_W2] = __float2bfloat16(w);
}

static __global__ void k_mlp_to_bf16(const float *params, __nv_bfloat16 *w2bf) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q < MLP_H * MLP_H) w2bf[q] = __float2bfloat16(params[MLP_OFF_W2 + q]);
}

static __global__ void k_mlp_init(float *params, unsigned long long seed) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= MLP_NPARAM) return;
  double u = u01(seed, p, 7) * 2.0 - 1.0;
  float w = 0.0f;
  if (p < MLP_OFF_B1) w = (float)(u * 0.5 * 1.7320508);                 // fan-in 4
  else if (p >= MLP_OFF_W2 && p < MLP_OFF_B2) w = (float)(u * 0.125 * 1.7320508 * 1.414);  // fan-in 64
  else if (p >= MLP_OFF_W3 && p < MLP_OFF_B3) w = (float)(u * 0.125 * 1.7320508);
  else if (p >= MLP_OFF_B1 && p < MLP_OFF_W2) w = 0.01f;
  else if (p >= MLP_OFF_B2 && p < MLP_OFF_W3) w = 0.01f;
  params[p] = w;
}

// ------------------------------------------------------------------ inference on tcgen05
// 128 samples per CTA of 128 threads (thread = sample): layer 1 per thread in FP32, written as
// BF16 row `tid` of A (128 x 64) in shared memory; one thread issues the layer-2 product
// D = A W2^T (M = 128, N = 64, K = 64 as four K = 16 MMAs) into 64 tensor-memory columns; each
// warp reads its 32 rows of D back (thread = row = sample) and finishes layer 3 in FP32.
struct MlpUmmaSmem {
  alignas(128) unsigned char A[128 * MLP_H * 2];  // hidden activations, core-matrix layout
  alignas(128) unsigned char B[MLP_H * MLP_H * 2];  // W2 [out][in], core-matrix layout
  uint64_t mbar;
  uint32_t tmem;
};
constexpr int MLP_UMMA_COLS = 64;         // FP32 accumulator columns (N)
constexpr int MLP_UMMA_POLLS = 1 << 22;   // mbarrier polls before a stalled MMA is reported

// All 128 threads of the block call this with uniform control flow.  A product that does not
// complete within the poll limit increments *stalled (once per warp) and leaves layer 2 at zero.
__device__ __forceinline__ float mlp_forward_cta(const MlpWeights &m, const float x[4], MlpUmmaSmem &S,
                                                 unsigned long long *stalled) {
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (warp == 0) {
    tmem_alloc(&S.tmem, MLP_UMMA_COLS);
    tmem_relinquish();
  }
  if (tid == 0) mbar_init(&S.mbar, 1);
  // W2 (row-major bf16 [out][in]) into the core-matrix layout, 16-byte pieces
  for (int q = tid; q < MLP_H * 8; q += blockDim.x) {
    const int n = q >> 3, c = q & 7;
    const uint4 v = __ldg(reinterpret_cast<const uint4 *>(m.w2bf + n * MLP_H) + c);
    *reinterpret_cast<uint4 *>(S.B + umma_kmajor_offset(n, 8 * c)) = v;
  }
  // layer 1 (FP32) -> BF16 row tid of A
  const float *W1 = m.w + MLP_OFF_W1, *b1 = m.w + MLP_OFF_B1;
#pragma unroll 2
  for (int c = 0; c < MLP_H / 8; ++c) {
    __align__(16) __nv_bfloat16 v[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int o = 8 * c + j;
      float a = __ldg(b1 + o);
#pragma unroll
      for (int k = 0; k < 4; ++k) a = fmaf(__ldg(W1 + o * 4 + k), x[k], a);
      v[j] = __float2bfloat16(fmaxf(a, 0.0f));
    }
    *reinterpret_cast<uint4 *>(S.A + umma_kmajor_offset(tid, 8 * c)) = *reinterpret_cast<const uint4 *>(v);
  }
  fence_proxy_async_smem();
  tc_fence_before_sync();
  __syncthreads();
  tc_fence_after_sync();
  const uint32_t tbase = S.tmem;
  if (tid == 0) {
    const uint32_t a0 = smem_u32(S.A), b0 = smem_u32(S.B);
    constexpr uint32_t idesc = umma_idesc_bf16(128, MLP_H);
#pragma unroll
    for (int kk = 0; kk < MLP_H / 16; ++kk)
      umma_bf16_f32(tbase, umma_desc(a0 + kk * UMMA_KSTEP_BYTES, UMMA_KCORE_BYTES, UMMA_ROW_GROUP_BYTES),
                    umma_desc(b0 + kk * UMMA_KSTEP_BYTES, UMMA_KCORE_BYTES, UMMA_ROW_GROUP_BYTES), idesc, kk > 0);
    umma_commit(&S.mbar);
  }
  // a phase seen complete by any lane is complete for the whole warp
  const bool done = __any_sync(0xffffffffu, mbar_wait_bounded(&S.mbar, 0, MLP_UMMA_POLLS));
  tc_fence_after_sync();
  float out = __ldg(m.w + MLP_OFF_B3);
  if (done) {
    const float *W3 = m.w + MLP_OFF_W3, *b2 = m.w + MLP_OFF_B2;
    const uint32_t row_addr = tbase + ((uint32_t)(warp * 32) << 16);
#pragma unroll
    for (int c = 0; c < MLP_H / 16; ++c) {
      float z[16];
      tmem_ld16(row_addr + 16 * c, z);
#pragma unroll
      for (int q = 0; q < 16; ++q) out = fmaf(__ldg(W3 + 16 * c + q), fmaxf(z[q] + __ldg(b2 + 16 * c + q), 0.0f), out);
    }
  } else {
    if (lane == 0 && stalled) atomicAdd(stalled, 1ull);
    // give the product a second bounded chance to land before its columns are released
    mbar_wait_bounded(&S.mbar, 0, MLP_UMMA_POLLS);
  }
  tc_fence_before_sync();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tbase, MLP_UMMA_COLS);
  return mlp_prior(x) + out * MLP_OUT_SCALE + MLP_OUT_SHIFT;
}

// The FP32 parameters of layers 1 and 3 by value: passed as a __grid_constant__ kernel argument
// they sit in the constant bank, and the fully unrolled layer arithmetic takes them as operands
// instead of loading them.
struct MlpSmall {
  float w1[MLP_H * MLP_IN], b1[MLP_H], b2[MLP_H], w3[MLP_H], b3;
};
inline void mlp_small_from_params(const float *p, MlpSmall &w) {
  for (int i = 0; i < MLP_H * MLP_IN; ++i) w.w1[i] = p[MLP_OFF_W1 + i];
  for (int i = 0; i < MLP_H; ++i) {
    w.b1[i] = p[MLP_OFF_B1 + i];
    w.b2[i] = p[MLP_OFF_B2 + i];
    w.w3[i] = p[MLP_OFF_W3 + i];
  }
  w.b3 = p[MLP_OFF_B3];
}

// mlp_forward_cta in three pieces, with the FP32 layers taken from an MlpSmall: the block sets up
// its tensor-memory columns, mbarrier and W2 in shared memory once (mlp_cta_setup), runs tiles of
// 128 samples (mlp_forward_tile: all 128 threads, uniform control flow; tile n of the block waits
// on the mbarrier phase of parity n & 1) and releases the columns (mlp_cta_teardown).  The step's
// guess kernel (k_mlp_guess) runs one tile per block.
__device__ __forceinline__ void mlp_cta_setup(const __nv_bfloat16 *w2bf, MlpUmmaSmem &S) {
  const int tid = threadIdx.x;
  if ((tid >> 5) == 0) {
    tmem_alloc(&S.tmem, MLP_UMMA_COLS);
    tmem_relinquish();
  }
  if (tid == 0) mbar_init(&S.mbar, 1);
  for (int q = tid; q < MLP_H * 8; q += blockDim.x) {
    const int n = q >> 3, c = q & 7;
    const uint4 v = __ldg(reinterpret_cast<const uint4 *>(w2bf + n * MLP_H) + c);
    *reinterpret_cast<uint4 *>(S.B + umma_kmajor_offset(n, 8 * c)) = v;
  }
}

// One tile: returns log10 T of this thread's sample.  ok (uniform over the block) says that the
// tensor-core path is usable: a product that does not complete within the poll limit counts in
// *stalled, gives no guess for its tile (have = false) and turns ok off for the block's later
// tiles, whose samples then get no guess either.
__device__ __forceinline__ float mlp_forward_tile(const MlpSmall &w, const float x[4], MlpUmmaSmem &S,
                                                  uint32_t parity, bool &ok, bool &have,
                                                  unsigned long long *stalled) {
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
#pragma unroll
  for (int c = 0; c < MLP_H / 8; ++c) {
    uint32_t pk[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      float h2[2];
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int o = 8 * c + 2 * j + e;
        float a = w.b1[o];
#pragma unroll
        for (int k = 0; k < 4; ++k) a = fmaf(w.w1[o * 4 + k], x[k], a);
        h2[e] = fmaxf(a, 0.0f);
      }
      __nv_bfloat162 b2v = __floats2bfloat162_rn(h2[0], h2[1]);
      pk[j] = *reinterpret_cast<uint32_t *>(&b2v);
    }
    *reinterpret_cast<uint4 *>(S.A + umma_kmajor_offset(tid, 8 * c)) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
  }
  fence_proxy_async_smem();
  tc_fence_before_sync();
  __syncthreads();
  tc_fence_after_sync();
  const uint32_t tbase = S.tmem;
  bool done = false;
  if (ok) {
    if (tid == 0) {
      const uint32_t a0 = smem_u32(S.A), b0 = smem_u32(S.B);
      constexpr uint32_t idesc = umma_idesc_bf16(128, MLP_H);
#pragma unroll
      for (int kk = 0; kk < MLP_H / 16; ++kk)
        umma_bf16_f32(tbase, umma_desc(a0 + kk * UMMA_KSTEP_BYTES, UMMA_KCORE_BYTES, UMMA_ROW_GROUP_BYTES),
                      umma_desc(b0 + kk * UMMA_KSTEP_BYTES, UMMA_KCORE_BYTES, UMMA_ROW_GROUP_BYTES), idesc, kk > 0);
      umma_commit(&S.mbar);
    }
    done = __any_sync(0xffffffffu, mbar_wait_bounded(&S.mbar, parity, MLP_UMMA_POLLS));
    tc_fence_after_sync();
  }
  float out = w.b3;
  if (done) {
    const uint32_t row_addr = tbase + ((uint32_t)(warp * 32) << 16);
#pragma unroll
    for (int c = 0; c < MLP_H / 16; ++c) {
      float z[16];
      tmem_ld16(row_addr + 16 * c, z);
#pragma unroll
      for (int q = 0; q < 16; ++q) out = fmaf(w.w3[16 * c + q], fmaxf(z[q] + w.b2[16 * c + q], 0.0f), out);
    }
  } else if (ok) {
    if (lane == 0 && stalled) atomicAdd(stalled, 1ull);
    // a second bounded chance for the product to land before A and the columns are reused
    mbar_wait_bounded(&S.mbar, parity, MLP_UMMA_POLLS);
  }
  tc_fence_before_sync();
  const bool all_done = __syncthreads_and(done);
  tc_fence_after_sync();
  have = done;
  ok = ok && all_done;
  return mlp_prior(x) + out * MLP_OUT_SCALE + MLP_OUT_SHIFT;
}

__device__ __forceinline__ void mlp_cta_teardown(MlpUmmaSmem &S) {
  tc_fence_before_sync();
  __syncthreads();
  tc_fence_after_sync();
  if ((threadIdx.x >> 5) == 0) tmem_dealloc(S.tmem, MLP_UMMA_COLS);
}

// per-sample inference kernel (features n x 4 -> log10 T), 128 threads per block
static __global__ void __launch_bounds__(128) k_mlp_infer(MlpWeights m, long long n, const float *feat, float *out,
                                                   unsigned long long *stalled) {
  __shared__ MlpUmmaSmem S;
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  float x[4] = {0, 0, 0, 0};
  if (t < n)
    for (int k = 0; k < 4; ++k) x[k] = feat[t * 4 + k];
  float y = mlp_forward_cta(m, x, S, stalled);
  if (t < n) out[t] = y;
}

struct Mlp {
  bool ready = false;
  MlpRange range;
  float *params = nullptr, *grad = nullptr, *m = nullptr, *v = nullptr, *partial = nullptr, *lossp = nullptr;
  float *feat = nullptr, *target = nullptr;
  __nv_bfloat16 *w2bf = nullptr;
  long long nsamp = 0;
  int npart = 0;

  void release() {
    for (void *p : {(void *)params, (void *)grad, (void *)m, (void *)v, (void *)partial, (void *)lossp,
                    (void *)feat, (void *)target, (void *)w2bf})
      if (p) cudaFree(p);
    params = grad = m = v = partial = lossp = feat = target = nullptr;
    w2bf = nullptr;
    ready = false;
  }
  MlpWeights weights() const { return MlpWeights{params, w2bf}; }
  int alloc() {
    if (params) return 0;
    if (cudaMalloc(&params, sizeof(float) * MLP_NPARAM) || cudaMalloc(&grad, sizeof(float) * MLP_NPARAM) ||
        cudaMalloc(&m, sizeof(float) * MLP_NPARAM) || cudaMalloc(&v, sizeof(float) * MLP_NPARAM) ||
        cudaMalloc(&w2bf, sizeof(__nv_bfloat16) * MLP_H * MLP_H))
      return -2;
    return 0;
  }
  int set(cudaStream_t s, const float *h) {
    if (alloc()) return -2;
    if (cudaMemcpyAsync(params, h, sizeof(float) * MLP_NPARAM, cudaMemcpyHostToDevice, s) != cudaSuccess) return -2;
    k_mlp_to_bf16<<<(MLP_H * MLP_H + 255) / 256, 256, 0, s>>>(params, w2bf);
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
  // one gradient evaluation on `batch` samples starting at `offset` (grad -> this->grad);
  // returns the mean squared loss through *loss when non-null
  int gradient(cudaStream_t s, long long offset, int batch, double *loss) {
    int nb = batch / MLP_TILE;
    size_t sm = sizeof(MlpTrainSmem);
    k_mlp_train_step<<<nb, 128, sm, s>>>(params, w2bf, feat, target, nsamp, offset, batch, partial, lossp);
    k_mlp_reduce<<<(MLP_NPARAM + 255) / 256, 256, 0, s>>>(partial, nb, grad);
    if (cudaGetLastError() != cudaSuccess) return -2;
    if (loss) {
      float *h = new float[batch];
      cudaMemcpyAsync(h, lossp, sizeof(float) * batch, cudaMemcpyDeviceToHost, s);
      if (cudaStreamSynchronize(s) != cudaSuccess) { delete[] h; return -2; }
      double acc = 0;
      for (int i = 0; i < batch; ++i) acc += h[i];
      *loss = acc / batch;
      delete[] h;
    }
    return 0;
  }
  int train(const HelmTable &h, cudaStream_t s, long long n, unsigned long long seed, int epochs, int batch,
            double lr, double *final_loss) {
    if (batch % MLP_TILE || batch <= 0 || n < batch) return -1;
    if (alloc()) return -2;
    if (n != nsamp) {
      if (feat) cudaFree(feat);
      if (target) cudaFree(target);
      feat = target = nullptr;
      if (cudaMalloc(&feat, sizeof(float) * 4 * n) || cudaMalloc(&target, sizeof(float) * n)) return -2;
      nsamp = n;
    }
    int nb = batch / MLP_TILE;
    if (nb > npart) {
      if (partial) cudaFree(partial);
      if (lossp) cudaFree(lossp);
      partial = lossp = nullptr;
      if (cudaMalloc(&partial, sizeof(float) * (size_t)nb * MLP_NPARAM) || cudaMalloc(&lossp, sizeof(float) * batch))
        return -2;
      npart = nb;
    }
    if (cudaFuncSetAttribute(k_mlp_train_step, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sizeof(MlpTrainSmem)) != cudaSuccess)
      return -2;
    k_mlp_make_samples<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(h, n, seed, range, feat, target);
    if (!ready) {
      k_mlp_init<<<(MLP_NPARAM + 255) / 256, 256, 0, s>>>(params, seed ^ 0xABCDEFull);
      k_mlp_to_bf16<<<(MLP_H * MLP_H + 255) / 256, 256, 0, s>>>(params, w2bf);
    }
    cudaMemsetAsync(m, 0, sizeof(float) * MLP_NPARAM, s);
    cudaMemsetAsync(v, 0, sizeof(float) * MLP_NPARAM, s);
    long long steps_per_epoch = n / batch;
    int step = 0;
    for (int ep = 0; ep < epochs; ++ep) {
      // cosine-free schedule: constant lr for the first half, then linear decay to lr/20
      for (long long k = 0; k < steps_per_epoch; ++k) {
        ++step;
        double frac = (double)(ep * steps_per_epoch + k) / (double)(epochs * steps_per_epoch);
        float lr_t = (float)(frac < 0.5 ? lr : lr * (1.0 - 1.9 * (frac - 0.5)));
        if (gradient(s, k * batch, batch, nullptr)) return -2;
        k_mlp_adam<<<(MLP_NPARAM + 255) / 256, 256, 0, s>>>(params, grad, m, v, lr_t, 0.9f, 0.999f, 1e-8f, step,
                                                           w2bf);
      }
    }
    if (cudaGetLastError() != cudaSuccess) return -2;
    if (final_loss) {
      if (gradient(s, 0, batch, final_loss)) return -2;
    }
    if (cudaStreamSynchronize(s) != cudaSuccess) return -2;
    ready = true;
    return 0;
  }
  // gradient on caller-provided pairs (host arrays), for checking against a CPU reference
  int gradient_host(cudaStream_t s, long long n, const float *hf, const float *ht, float *hg, double *loss) {
    if (!ready || n <= 0 || n % MLP_TILE) return -1;
    if (n != nsamp) {
      if (feat) cudaFree(feat);
      if (target) cudaFree(target);
      feat = target = nullptr;
      if (cudaMalloc(&feat, sizeof(float) * 4 * n) || cudaMalloc(&target, sizeof(float) * n)) return -2;
      nsamp = n;
    }
    int nb = (int)(n / MLP_TILE);
    if (nb > npart) {
      if (partial) cudaFree(partial);
      if (lossp) cudaFree(lossp);
      partial = lossp = nullptr;
      if (cudaMalloc(&partial, sizeof(float) * (size_t)nb * MLP_NPARAM) || cudaMalloc(&lossp, sizeof(float) * n))
        return -2;
      npart = nb;
    }
    if (cudaFuncSetAttribute(k_mlp_train_step, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sizeof(MlpTrainSmem)) != cudaSuccess)
      return -2;
    if (cudaMemcpyAsync(feat, hf, sizeof(float) * 4 * n, cudaMemcpyHostToDevice, s) ||
        cudaMemcpyAsync(target, ht, sizeof(float) * n, cudaMemcpyHostToDevice, s))
      return -2;
    if (gradient(s, 0, (int)n, loss)) return -2;
    if (cudaMemcpyAsync(hg, grad, sizeof(float) * MLP_NPARAM, cudaMemcpyDeviceToHost, s)) return -2;
    if (cudaStreamSynchronize(s) != cudaSuccess) return -2;
    return 0;
  }
  int infer(cudaStream_t s, long long n, const float *f, float *o, unsigned long long *stalled) {
    if (!ready) return -4;
    if (n == 0) return 0;
    k_mlp_infer<<<(unsigned)((n + 127) / 128), 128, 0, s>>>(weights(), n, f, o, stalled);
    if (cudaGetLastError() != cudaSuccess) return -2;
    if (cudaStreamSynchronize(s) != cudaSuccess) return -2;
    return 0;
  }
};

}  // namespace phl
