// Fifth-generation tensor-core helpers (sm_100a): tensor-memory allocation, the
// single-thread tcgen05.mma of kind::tf32 from shared-memory descriptors, completion
// through tcgen05.commit on an mbarrier (waited on with a time limit), tcgen05.ld of
// accumulator rows, and the fences that order tensor-core work against thread
// barriers.
//
// Shared-memory operands use the canonical K-major layout without swizzle: "core
// matrices" of 8 rows x 16 bytes (4 tf32 or 8 bf16 values per row); element (mn, k) of
// one K step (8 tf32 or 16 bf16 values, 32 bytes) at
//   (mn % 8) * 16 + (mn / 8) * SBO + (k / V) * LBO + (k % V) * (16 / V) bytes,
// V = 4 (tf32) or 8 (bf16). (MN-major tf32 operands exist only in a swizzled layout;
// these kernels use K-major operands throughout.)
#pragma once
#include <cstdint>

namespace n3ds {
namespace tc {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// ------------------------------------------------------------------ mbarrier

__device__ __forceinline__ void mbar_init(uint64_t* bar, int count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t phase) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(phase)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ uint64_t globaltimer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// Wait for the barrier's phase for at most limit_ns; false when the time ran out.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t phase, unsigned long long limit_ns) {
  if (mbar_try_wait(bar, phase)) return true;
  const uint64_t t0 = globaltimer_ns();
  while (!mbar_try_wait(bar, phase)) {
    if (globaltimer_ns() - t0 > limit_ns) return false;
  }
  return true;
}

// Generic-proxy writes to shared memory made visible to the tensor core's reads.
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// ------------------------------------------------------------ tensor memory

// Allocate ncols columns (a power of two >= 32) for the CTA; warp-wide. The base
// address is written to *slot in shared memory.
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)), "r"(ncols)
               : "memory");
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

// 16 consecutive 32-bit columns of this thread's lane (32x32b shape: lane = the
// warp's quarter of the 128 lanes + its lane id); taddr carries the lane in bits
// 31:16 and the column in bits 15:0.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

// ------------------------------------------------------------ descriptors + MMA

// Shared-memory matrix descriptor, no swizzle: start address, leading and stride
// byte offsets (all multiples of 16), version 1 (sm_100).
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr & 0x3FFFFu) >> 4) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::tf32 with float32 accumulation: M x N, A and B
// K-major (false) or MN-major (true).
__host__ __device__ constexpr uint32_t idesc_tf32(int M, int N, bool a_mn, bool b_mn) {
  return (1u << 4)                               // D format: f32
         | (2u << 7) | (2u << 10)                // A, B format: tf32
         | ((a_mn ? 1u : 0u) << 15) | ((b_mn ? 1u : 0u) << 16)  // major-ness
         | ((uint32_t)(N >> 3) << 17)            // N / 8
         | ((uint32_t)(M >> 4) << 24);           // M / 16
}

// Instruction descriptor of kind::f16 with bf16 A and B (both K-major) and float32
// accumulation: M x N, K = 16 per instruction.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
  return (1u << 4)                     // D format: f32
         | (1u << 7) | (1u << 10)      // A, B format: bf16
         | ((uint32_t)(N >> 3) << 17)  // N / 8
         | ((uint32_t)(M >> 4) << 24); // M / 16
}

// D[tmem] (+)= A * B^T over one K = 16 step of bf16 operands; issued by one thread.
__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         bool accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(
          d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate ? 1u : 0u)
      : "memory");
}

// D[tmem] (+)= A * B^T over one K = 8 step; issued by one thread.
__device__ __forceinline__ void mma_tf32(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         bool accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::"r"(
          d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate ? 1u : 0u)
      : "memory");
}
// Arrive once on the mbarrier when every MMA this thread issued before has completed.
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

// ------------------------------------------------------------ tf32 splitting

// x = hi + lo with hi the leading 11 significant bits (a tf32 value, low 13 bits
// zero) and lo the remainder rounded to tf32: hi*hi' + hi*lo' + lo*hi' then
// reproduces a float32 product to about 2^-21 (the three-term tf32 split).
__device__ __forceinline__ void split_tf32(float x, float& hi, float& lo) {
  hi = __uint_as_float(__float_as_uint(x) & 0xFFFFE000u);
  const float r = x - hi;
  uint32_t t;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(t) : "f"(r));
  lo = __uint_as_float(t);
}

}  // namespace tc
}  // namespace n3ds
