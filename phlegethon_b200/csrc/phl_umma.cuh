// phl_umma.cuh -- 5th-generation tensor-core (tcgen05) building blocks for the temperature-guess
// MLP: shared-memory matrix descriptors, the instruction descriptor of a BF16 x BF16 -> FP32
// product, tensor-memory allocation, MMA issue/commit, mbarrier waits with an iteration limit,
// and tensor-memory loads.  Written from the PTX ISA for sm_100a.
//
// Operand layout (no swizzle, K-major): a matrix of R rows x 64 bf16 columns is stored as
// 8 x 8 "core matrices" of 128 contiguous bytes (8 rows x 16 bytes); core matrix (r/8, k/8)
// starts at (r/8) * 1024 + (k/8) * 128 bytes, element (r, k) at + (r%8) * 16 + (k%8) * 2.  In the
// descriptor, the leading-dimension byte offset is the step between the two K-adjacent core
// matrices one MMA (K = 16) reads (128 B) and the stride byte offset the step between 8-row
// groups (1024 B); the k-th K = 16 slice starts 256 B further.
#pragma once
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cstdint>

namespace phl {

constexpr int UMMA_ROW_GROUP_BYTES = 1024;  // one 8-row group of a 64-column bf16 operand
constexpr int UMMA_KCORE_BYTES = 128;       // one 8 x 8 bf16 core matrix
constexpr int UMMA_KSTEP_BYTES = 256;       // K = 16 per MMA: two core matrices

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// byte offset of element (r, k) in the core-matrix layout above
__host__ __device__ __forceinline__ int umma_kmajor_offset(int r, int k) {
  return (r >> 3) * UMMA_ROW_GROUP_BYTES + (k >> 3) * UMMA_KCORE_BYTES + (r & 7) * 16 + (k & 7) * 2;
}

// shared-memory matrix descriptor: start address, leading / stride byte offsets (>> 4),
// descriptor version 1 (bits 46-47), no swizzle (bits 61-63 = 0)
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// instruction descriptor of kind::f16: FP32 accumulator (bits 4-5 = 1), A and B BF16 (bits 7-9,
// 10-12 = 1), both K-major, N / 8 in bits 17-22, M / 16 in bits 24-28
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// warp-wide: allocate `ncols` tensor-memory columns, address written to *dst (shared memory)
__device__ __forceinline__ void tmem_alloc(uint32_t *dst, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)), "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tc_fence_before_sync() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after_sync() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// generic-proxy shared-memory writes become visible to the tensor core (async proxy)
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// D[tmem] (+)= A[smem] * B[smem]^T, one thread issues
__device__ __forceinline__ void umma_bf16_f32(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                              uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}
// arrive on the mbarrier once every MMA issued so far by this thread has completed
__device__ __forceinline__ void umma_commit(uint64_t *mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(mbar))
               : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t *mbar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mbar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *mbar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(done)
      : "r"(smem_u32(mbar)), "r"(parity)
      : "memory");
  return done != 0;
}
// wait for phase `parity` to complete, at most `limit` polls; false when the limit ran out
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *mbar, uint32_t parity, int limit) {
  for (int it = 0; it < limit; ++it)
    if (mbar_try_wait(mbar, parity)) return true;
  return false;
}

// 32 lanes x 16 consecutive 32-bit columns: thread t of the warp receives lane (base lane + t)
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float v[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int q = 0; q < 16; ++q) v[q] = __uint_as_float(r[q]);
}

}  // namespace phl

// ------------------------------------------------------------------ TMA (bulk tensor copies)
#include <cuda.h>
namespace phl {
// arm an mbarrier for `bytes` of asynchronous copies (one arrival)
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *mbar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%1], %0;" ::"r"(bytes), "r"(smem_u32(mbar))
               : "memory");
}
// 4D tiled tensor copy global -> shared, completion counted on `mbar` (no multicast)
__device__ __forceinline__ void tma_load_4d(void *dst, const CUtensorMap *map, uint64_t *mbar, int c0, int c1, int c2,
                                            int c3) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5, %6}], "
      "[%2];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(mbar)), "r"(c0), "r"(c1), "r"(c2), "r"(c3)
      : "memory");
}
}  // namespace phl
