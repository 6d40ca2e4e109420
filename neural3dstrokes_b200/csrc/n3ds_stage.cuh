// Device helpers shared by the fused stroke-field kernels: bulk (TMA) copies into
// shared memory completed on an mbarrier with a bounded wait, the per-CTA stage of
// stroke records and culling data, scene-affinity work distribution.
#pragma once
#include "n3ds_eval.cuh"
#include "n3ds_field.cuh"

namespace n3ds {

// ----------------------------------------------------------- async-copy helpers

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, int count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
  // make the initialised barrier visible to the async (bulk-copy) proxy
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
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
// Wait for the mbarrier phase for at most limit_ns; false on timeout.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t phase, unsigned long long limit_ns) {
  if (mbar_try_wait(bar, phase)) return true;
  uint64_t t0 = globaltimer_ns();
  while (!mbar_try_wait(bar, phase)) {
    if (globaltimer_ns() - t0 > limit_ns) return false;
  }
  return true;
}
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ float seg_dist(V3 c, V3 A, V3 AB, float invL2) {
  V3 w = c - A;
  // clamp to the chord [0, 1] as the multiply's saturation (a NaN product comes from
  // non-finite coordinates, whose distance is not finite with either clamp)
  float tt = __saturatef(dot(w, AB) * invL2);
  V3 d = w - AB * tt;
  return sqrtf(dot(d, d));
}

__device__ __forceinline__ V3 shfl3(V3 v, int src) {
  return {__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src),
          __shfl_sync(0xffffffffu, v.z, src)};
}

// Home scene of this CTA: the last scene whose CTA range starts at or before it.
__device__ __forceinline__ int home_scene(const SegLaunch& L) {
  int h = 0;
  for (int i = 1; i < L.n_scenes; i++)
    if (L.sc[i].home_lo <= (int)blockIdx.x) h = i;
  return h;
}

// Scene with the most rays left to take, or -1 when every scene is taken (thread 0).
__device__ __forceinline__ int next_scene(const SegLaunch& L) {
  int best = -1, most = 0;
  for (int i = 0; i < L.n_scenes; i++) {
    const int left = L.sc[i].n_rays - *reinterpret_cast<volatile int*>(L.tile_counter + i);
    if (left > most) {
      most = left;
      best = i;
    }
  }
  return best;
}

__host__ __device__ constexpr size_t align16(size_t v) { return (v + 15) & ~size_t(15); }


struct Stage {
  float4* cull_a;
  float* cull_b;
  float* recs;
  float* gacc;
};

__device__ __forceinline__ Stage carve(unsigned char* smem, int cap, bool with_grads) {
  Stage s;
  s.cull_a = reinterpret_cast<float4*>(smem);
  s.cull_b = reinterpret_cast<float*>(smem + align16(cap * 16));
  s.recs = reinterpret_cast<float*>(smem + align16(cap * 16) + align16(cap * 4));
  s.gacc = with_grads ? s.recs + size_t(cap) * REC_FLOATS : nullptr;
  return s;
}

// Stage the scene's current chunk: records and culling spheres by bulk copy,
// culling margins by plain loads. Returns false on an mbarrier timeout. A timeout is
// terminal for the launch: the caller sets ST_WAIT_TIMEOUT in the status word and its
// CTA returns, so the host treats every output of the launch as invalid; the copies
// of a barrier that did not complete within the limit (one second by default) are
// not waited for. (test_stall arms the barrier without issuing the copies: every
// wait runs out and no copy is in flight when the CTA leaves.)
__device__ __forceinline__ bool stage_chunk(const SegLaunch& L, const SceneDesc& sc, const Stage& S, uint64_t* bar,
                            uint32_t& phase, int* s_fail) {
  const int n = sc.chunk_n;
  const long long g0 = (long long)sc.stroke_begin + sc.chunk_lo;
  if (n > 0) {
    if (threadIdx.x == 0) {
      fence_proxy_async();
      const uint32_t b_rec = uint32_t(n) * REC_FLOATS * 4;
      const uint32_t b_cull = uint32_t(n) * 16;
      mbar_expect_tx(bar, b_rec + b_cull);
      if (!L.test_stall) {
        bulk_g2s(S.recs, L.recs + g0 * REC_FLOATS, b_rec, bar);
        bulk_g2s(S.cull_a, L.cull_a + g0 * 4, b_cull, bar);
      }
    }
    for (int i = threadIdx.x; i < n; i += blockDim.x) S.cull_b[i] = L.cull_b[g0 + i];
    if (!mbar_wait_bounded(bar, phase, L.wait_limit_ns)) *s_fail = 1;
    phase ^= 1u;
  }
  __syncthreads();
  return *s_fail == 0;
}

// Sample i of ray `ray` (global sample index si = ray * n_samples + i): position and
// radius from the inputs, or cast from the ray as cast_rays does (render.py:20-25):
// t = (t0 + t1) / 2, x = d t + o, radius = r t.
__device__ __forceinline__ void load_sample(const SegLaunch& L, long long ray, int i, long long si, V3& x, float& r) {
  if (L.x) {
    x = v3(L.x[3 * si], L.x[3 * si + 1], L.x[3 * si + 2]);
    r = L.radius[si];
  } else {
    const float* td = L.tdist + ray * (L.n_samples + 1);
    const float t = (td[i] + td[i + 1]) * 0.5f;
    x = v3(__fadd_rn(__fmul_rn(L.dirs[3 * ray], t), L.origins[3 * ray]),
           __fadd_rn(__fmul_rn(L.dirs[3 * ray + 1], t), L.origins[3 * ray + 1]),
           __fadd_rn(__fmul_rn(L.dirs[3 * ray + 2], t), L.origins[3 * ray + 2]));
    r = L.radii[ray] * t;
  }
}

}  // namespace n3ds
