// The non-'over' composition modes of compose_strokes (the reference computes them
// with torch ops, source/strokelib/strokes.py:390-417): per sample, over the stroke
// axis,
//   max                      k_s = alpha_s,            pick s* = argmax k (first on ties)
//   max_density_weighted     k_s = alpha_s d_s,        pick s* = argmax k
//     density = alpha_s* d_s*, colour = colour_s*
//   softmax                  k_s = alpha_s / 0.05,     w = softmax(k)
//   softmax_density_weighted k_s = alpha_s d_s / 0.05, w = softmax(k)
//     density = sum_s w_s alpha_s d_s, colour = sum_s w_s colour_s
// One warp per sample, lanes striding the strokes; the backward recomputes the pick
// or the softmax weights and writes dL/dalpha and dL/dcolour per (sample, stroke),
// accumulating dL/d(density params) per CTA in shared memory before one global atomic
// per stroke.
#include <algorithm>

#include <cuda_runtime.h>

#include "../../include/n3ds.h"
#include "n3ds_math.cuh"

namespace n3ds {

namespace {

constexpr int CM_WARPS = 8;
constexpr float INV_TEMP = 1.0f / 0.05f;  // strokes.py:402,410
constexpr int CM_SMEM_STROKES = 8192;     // dL/d(density params) staged per CTA up to this many strokes

__device__ __forceinline__ bool is_weighted(int mode) {
  return mode == N3DS_COMPOSE_MAX_DENSITY_WEIGHTED || mode == N3DS_COMPOSE_SOFTMAX_DENSITY_WEIGHTED;
}
__device__ __forceinline__ bool is_max(int mode) {
  return mode == N3DS_COMPOSE_MAX || mode == N3DS_COMPOSE_MAX_DENSITY_WEIGHTED;
}

// Better (key, index) under torch.argmax ordering: larger key, NaN above everything,
// first index on ties.
__device__ __forceinline__ bool better(float k, int i, float kb, int ib) {
  const bool kn = k != k, bn = kb != kb;
  if (kn || bn) return kn && (!bn || i < ib);
  return k > kb || (k == kb && i < ib);
}

struct Pick {
  float key;
  int idx;
};

__device__ __forceinline__ Pick warp_argmax(float k, int i) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const float k2 = __shfl_xor_sync(0xffffffffu, k, o);
    const int i2 = __shfl_xor_sync(0xffffffffu, i, o);
    if (better(k2, i2, k, i)) {
      k = k2;
      i = i2;
    }
  }
  return {k, i};
}

__device__ __forceinline__ Pick sample_argmax(const float* a, const float* d, long long S, int mode, int lane) {
  float kb = -__int_as_float(0x7f800000);
  int ib = 0x7fffffff;
  for (long long s = lane; s < S; s += 32) {
    const float k = is_weighted(mode) ? a[s] * d[s] : a[s];
    if (better(k, (int)s, kb, ib)) {
      kb = k;
      ib = (int)s;
    }
  }
  return warp_argmax(kb, ib);
}

// max of the softmax keys and the partition sum
__device__ __forceinline__ void sample_softmax(const float* a, const float* d, long long S, int mode, int lane,
                                               float* mx, float* z) {
  float m = -__int_as_float(0x7f800000);
  for (long long s = lane; s < S; s += 32) {
    const float k = (is_weighted(mode) ? a[s] * d[s] : a[s]) * INV_TEMP;
    m = fmaxf(m, k);
  }
  m = warp_max(m);
  float zz = 0.f;
  for (long long s = lane; s < S; s += 32) {
    const float k = (is_weighted(mode) ? a[s] * d[s] : a[s]) * INV_TEMP;
    zz += expf(k - m);
  }
  *mx = m;
  *z = warp_sum(zz);
}

__global__ void compose_mode_fwd_kernel(int mode, float* density, float* color, const float* alphas,
                                        const float* colors, const float* dp, long long P, long long S, int C) {
  const int lane = threadIdx.x & 31;
  const long long p = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  if (p >= P) return;
  const float* a = alphas + p * S;
  const float* c = colors + p * S * C;
  if (is_max(mode)) {
    const Pick pk = sample_argmax(a, dp, S, mode, lane);
    if (S == 0) {
      if (lane == 0) density[p] = 0.f;
      if (lane < C) color[p * C + lane] = 0.f;
      return;
    }
    const long long s = pk.idx;
    if (lane == 0) density[p] = a[s] * dp[s];
    if (lane < C) color[p * C + lane] = c[s * C + lane];
    return;
  }
  float m, z;
  sample_softmax(a, dp, S, mode, lane, &m, &z);
  float dens = 0.f, c0 = 0.f, c1 = 0.f, c2 = 0.f;
  for (long long s = lane; s < S; s += 32) {
    const float k = (is_weighted(mode) ? a[s] * dp[s] : a[s]) * INV_TEMP;
    const float w = expf(k - m) / z;
    dens += w * (a[s] * dp[s]);
    c0 += w * c[s * C];
    if (C > 1) {
      c1 += w * c[s * C + 1];
      c2 += w * c[s * C + 2];
    }
  }
  dens = warp_sum(dens);
  c0 = warp_sum(c0);
  c1 = warp_sum(c1);
  c2 = warp_sum(c2);
  if (lane == 0) {
    density[p] = dens;
    color[p * C] = c0;
    if (C > 1) {
      color[p * C + 1] = c1;
      color[p * C + 2] = c2;
    }
  }
}

__global__ void compose_mode_bwd_kernel(int mode, float* g_alpha, float* g_colors, float* g_dp, const float* g_dens,
                                        const float* g_col, const float* alphas, const float* colors, const float* dp,
                                        long long P, long long S, int C) {
  extern __shared__ float s_gdp[];  // [min(S, CM_SMEM_STROKES)]
  const bool staged = S <= CM_SMEM_STROKES;
  if (staged)
    for (long long s = threadIdx.x; s < S; s += blockDim.x) s_gdp[s] = 0.f;
  __syncthreads();
  const int lane = threadIdx.x & 31;
  auto add_gdp = [&](long long s, float v) {
    if (v == 0.f) return;
    if (staged) atomicAdd(s_gdp + s, v);
    else atomicAdd(g_dp + s, v);
  };
  // grid-stride over samples: each CTA flushes its per-stroke sums once
  const long long warps_total = (long long)gridDim.x * (blockDim.x >> 5);
  for (long long p = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5; p < P; p += warps_total) {
    const float* a = alphas + p * S;
    const float* c = colors + p * S * C;
    float* ga = g_alpha + p * S;
    float* gc = g_colors + p * S * C;
    const float gd = g_dens ? g_dens[p] : 0.f;
    float gcol[3] = {0.f, 0.f, 0.f};
    if (g_col)
      for (int k = 0; k < C; k++) gcol[k] = g_col[p * C + k];
    if (is_max(mode)) {
      const Pick pk = sample_argmax(a, dp, S, mode, lane);
      for (long long s = lane; s < S; s += 32) {
        const bool hit = s == pk.idx;
        ga[s] = hit ? gd * dp[s] : 0.f;
        for (int k = 0; k < C; k++) gc[s * C + k] = hit ? gcol[k] : 0.f;
        if (hit) add_gdp(s, gd * a[s]);
      }
    } else {
      float m, z;
      sample_softmax(a, dp, S, mode, lane, &m, &z);
      // dL/dw_s = g_d alpha_s d_s + g_c . c_s ; T = sum_s w_s dL/dw_s
      float tsum = 0.f;
      for (long long s = lane; s < S; s += 32) {
        const float k = (is_weighted(mode) ? a[s] * dp[s] : a[s]) * INV_TEMP;
        const float w = expf(k - m) / z;
        float gw = gd * a[s] * dp[s];
        for (int q = 0; q < C; q++) gw += gcol[q] * c[s * C + q];
        tsum += w * gw;
      }
      tsum = warp_sum(tsum);
      for (long long s = lane; s < S; s += 32) {
        const float k = (is_weighted(mode) ? a[s] * dp[s] : a[s]) * INV_TEMP;
        const float w = expf(k - m) / z;
        float gw = gd * a[s] * dp[s];
        for (int q = 0; q < C; q++) gw += gcol[q] * c[s * C + q];
        const float gk = w * (gw - tsum) * INV_TEMP;  // dL/d(raw key: alpha, or alpha d)
        float gdp_s = gd * w * a[s];
        if (is_weighted(mode)) {
          ga[s] = gk * dp[s] + gd * w * dp[s];
          gdp_s += gk * a[s];
        } else {
          ga[s] = gk + gd * w * dp[s];
        }
        for (int q = 0; q < C; q++) gc[s * C + q] = gcol[q] * w;
        add_gdp(s, gdp_s);
      }
    }
  }
  if (staged) {
    __syncthreads();
    for (long long s = threadIdx.x; s < S; s += blockDim.x)
      if (s_gdp[s] != 0.f) atomicAdd(g_dp + s, s_gdp[s]);
  }
}

}  // namespace

cudaError_t launch_compose_mode_fwd(int mode, float* density, float* color, const float* alphas, const float* colors,
                                    const float* dp, long long P, long long S, int C, cudaStream_t st) {
  const long long threads = P * 32;
  const int bs = CM_WARPS * 32;
  compose_mode_fwd_kernel<<<(unsigned)((threads + bs - 1) / bs), bs, 0, st>>>(mode, density, color, alphas, colors,
                                                                              dp, P, S, C);
  return cudaGetLastError();
}

cudaError_t launch_compose_mode_bwd(int mode, float* g_alpha, float* g_colors, float* g_dp, const float* g_dens,
                                    const float* g_col, const float* alphas, const float* colors, const float* dp,
                                    long long P, long long S, int C, cudaStream_t st) {
  // a grid of a few CTAs per SM, each looping over samples, so that the per-stroke
  // shared accumulators are flushed a few thousand times at most
  const int bs = CM_WARPS * 32;
  const size_t smem = S <= CM_SMEM_STROKES ? size_t(std::max<long long>(S, 1)) * 4 : 0;
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(compose_mode_bwd_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
  }
  const long long blocks = std::min<long long>((P + CM_WARPS - 1) / CM_WARPS, 148LL * 4);
  compose_mode_bwd_kernel<<<(unsigned)std::max<long long>(blocks, 1), bs, smem, st>>>(
      mode, g_alpha, g_colors, g_dp, g_dens, g_col, alphas, colors, dp, P, S, C);
  return cudaGetLastError();
}

}  // namespace n3ds
