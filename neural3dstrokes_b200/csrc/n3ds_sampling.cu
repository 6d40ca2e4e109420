// Proposal resampling of ray intervals (the step that produces the stroke level's
// fence posts, models.py:147-185 with source/utils/stepfun.py), one warp per ray with
// the ray's step functions in shared memory:
//
//   max_dilate_weights (stepfun.py:136-147, max_dilate 120-133): pdf p = w / max(dt, eps);
//     fence posts t, t[:-1] - d and t[1:] + d merged in sorted order (three sorted
//     lists: each element's rank is its index plus binary-search counts in the other
//     two, ties ordered t < t0 < t1), clipped to the domain; the dilated pdf at post i
//     is the max of p_j over the intervals j with t0_j <= td_i < t1_j (a contiguous
//     range of j, found by two binary searches); weights = pdf * dt, renormalised.
//   sample_intervals (stepfun.py:280-317, sample 220-243, invert_cdf 211-218,
//     integrate_weights 150-171, sorted_interp 5-24): softmax of the logits, CDF
//     [0, min(cumsum, 1), 1], u = linspace + jitter (or the centred linspace), the
//     inverse CDF by binary search and linear interpolation, then the interval
//     midpoints with reflected, domain-clamped first and last fence posts.
//   resample (fused level, models.py:156-185): optional dilation and [1:-1] slice, the
//     logits where(s[1:] > s[:-1], log(w + padding), -inf), sampling, and
//     s_to_t(s) = s * far + (1 - s) * near (the identity ray-distance warp,
//     coord.py:56-99).
//
// The jitter values come from the caller (torch.rand drawn exactly as the reference
// draws them), so random sampling is reproducible against the reference.
#include <algorithm>
#include <cmath>
#include <string>

#include <cuda_runtime.h>

#include "../../include/n3ds.h"

namespace n3ds {
int report_error(int code, const std::string& msg);  // sets n3ds_last_error (n3ds_capi.cu)
}

namespace {

constexpr float EPS32 = 1.1920928955078125e-07f;  // torch.finfo(torch.float32).eps
constexpr int SAMPLE_WARPS = 8;
constexpr int MAX_BINS = 2048;

__device__ __forceinline__ float warp_sum_f(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ float warp_max_f(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// number of j in [0, n) with f(j) < x (strict) or <= x, for f non-decreasing in j
template <bool LE, typename F>
__device__ __forceinline__ int count_below(int n, float x, F f) {
  int lo = 0, hi = n;  // answer in [lo, hi]
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    const float v = f(mid);
    if (LE ? (v <= x) : (v < x)) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// Dilate the step function (t[0..M], w[0..M-1]) of one ray into td[0..3M] and
// wd[0..3M-1] (shared), all lanes of the warp taking part.
__device__ void dilate_ray(const float* t, const float* w, int M, float d, float lo, float hi, bool renorm,
                           float* p, float* td, float* wd, int lane) {
  for (int k = lane; k < M; k += 32) p[k] = w[k] / fmaxf(t[k + 1] - t[k], EPS32);
  auto T = [&](int j) { return t[j]; };
  auto T0 = [&](int j) { return t[j] - d; };
  auto T1 = [&](int j) { return t[j + 1] + d; };
  // stable merge of t (M+1), t0 (M), t1 (M)
  for (int k = lane; k <= M; k += 32) {
    const float a = t[k];
    const int r = k + count_below<false>(M, a, T0) + count_below<false>(M, a, T1);
    td[r] = fminf(fmaxf(a, lo), hi);
  }
  for (int k = lane; k < M; k += 32) {
    const float b = t[k] - d;
    const int r = k + count_below<true>(M + 1, b, T) + count_below<false>(M, b, T1);
    td[r] = fminf(fmaxf(b, lo), hi);
    const float c = t[k + 1] + d;
    const int rc = k + count_below<true>(M + 1, c, T) + count_below<true>(M, c, T0);
    td[rc] = fminf(fmaxf(c, lo), hi);
  }
  __syncwarp();
  // dilated pdf at post i (the last post's value is dropped): max p_j over
  // t0_j <= td_i < t1_j, i.e. j in [first j with t1_j > td_i, last j with t0_j <= td_i]
  const int L = 3 * M;
  float part = 0.f;
  for (int i = lane; i < L; i += 32) {
    const float x = td[i];
    const int j0 = count_below<true>(M, x, T1);       // first j with t1_j > x
    const int j1 = count_below<true>(M, x, T0) - 1;   // last j with t0_j <= x
    float pm = 0.f;
    for (int j = j0; j <= j1; j++) pm = fmaxf(pm, p[j]);
    const float wv = pm * (td[i + 1] - td[i]);
    wd[i] = wv;
    part += wv;
  }
  if (renorm) {
    const float s = fmaxf(warp_sum_f(part), EPS32);
    __syncwarp();
    for (int i = lane; i < L; i += 32) wd[i] = wd[i] / s;
  }
  __syncwarp();
}

// torch.linspace(a, b, n)[k] in float32 (the half-from-each-end evaluation)
__device__ __forceinline__ float linspace_at(float a, float b, int n, int k) {
  if (n == 1) return a;
  const float step = (b - a) / (float)(n - 1);
  return k < n / 2 ? a + step * (float)k : b - step * (float)(n - 1 - k);
}

// Sample N intervals of the step function (s[0..K], logits l[0..K-1]) of one ray;
// writes s_out[0..N] (global). cw (K+1) and cen (N) are shared scratch.
__device__ void sample_ray(const float* s, const float* l, int K, int N, const float* jit, bool single, float lin_a,
                           float lin_b, float max_jit, float lo, float hi, float* cw, float* cen, float* s_out,
                           float* t_out, float near, float far, int lane) {
  // softmax (exp(l - max) / sum)
  float mx = -INFINITY;
  for (int i = lane; i < K; i += 32) mx = fmaxf(mx, l[i]);
  mx = warp_max_f(mx);
  float z = 0.f;
  for (int i = lane; i < K; i += 32) z += expf(l[i] - mx);
  z = warp_sum_f(z);
  // CDF: cw[0] = 0, cw[i] = min(sum_{j<i} w_j, 1) for 0 < i < K, cw[K] = 1
  if (lane == 0) cw[0] = 0.f;
  float carry = 0.f;
  for (int i0 = 0; i0 < K - 1; i0 += 32) {
    const int i = i0 + lane;
    float v = i < K - 1 ? expf(l[i] - mx) / z : 0.f;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const float u = __shfl_up_sync(0xffffffffu, v, o);
      if (lane >= o) v += u;
    }
    v += carry;
    if (i < K - 1) cw[i + 1] = fminf(v, 1.f);
    carry = __shfl_sync(0xffffffffu, v, 31);
  }
  if (lane == 0) cw[K] = 1.f;
  __syncwarp();
  // u = linspace(lin_a, lin_b, N) (+ jitter * max_jit) and the inverse CDF
  for (int k = lane; k < N; k += 32) {
    float u = linspace_at(lin_a, lin_b, N, k);
    if (jit) u += jit[single ? 0 : k] * max_jit;
    // last j with cw_j <= u (cw_0 = 0 <= u), first index above it
    const int j = count_below<true>(K + 1, u, [&](int q) { return cw[q]; }) - 1;
    const int j0 = max(j, 0);
    const int j1 = min(j0 + 1, K);
    const float xp0 = cw[j0], xp1 = cw[j1];
    float off = (u - xp0) / (xp1 - xp0);
    if (off != off) off = 0.f;
    off = fminf(fmaxf(off, 0.f), 1.f);
    const float f0 = s[j0], f1 = s[j1];
    cen[k] = f0 + off * (f1 - f0);
  }
  __syncwarp();
  for (int k = lane; k <= N; k += 32) {
    float v;
    if (k == 0) {
      v = fmaxf(2.f * cen[0] - (cen[1] + cen[0]) / 2.f, lo);
    } else if (k == N) {
      v = fminf(2.f * cen[N - 1] - (cen[N - 1] + cen[N - 2]) / 2.f, hi);
    } else {
      v = (cen[k] + cen[k - 1]) / 2.f;
    }
    if (s_out) s_out[k] = v;
    if (t_out) t_out[k] = v * far + (1.f - v) * near;
  }
  __syncwarp();
}

struct ResampleArgs {
  float* s_out;
  float* t_out;
  const float* sdist;    // [R, M+1]
  const float* weights;  // [R, M] (weights mode) or logits [R, M] (logits mode)
  long long R;
  int M, N;
  float dilation;        // > 0: dilate first (then slice [1:-1])
  float padding;
  const float* jitter;   // [R] (single) or [R, N]; null: deterministic centres
  int single;
  float lo, hi;
  const float* near;     // [R] or null (then s_to_t is skipped)
  const float* far;
  float lin_a, lin_b, max_jit;  // linspace ends and jitter scale (stepfun.py:233-242, in double)
  int logits_mode;       // 1: `weights` holds logits, no dilation (sample_intervals)
  size_t warp_floats;
};

__global__ void resample_kernel(const ResampleArgs A) {
  extern __shared__ float sm[];
  const int lane = threadIdx.x & 31;
  const int wid = threadIdx.x >> 5;
  float* base = sm + (size_t)wid * A.warp_floats;
  const int M = A.M;
  float* t = base;              // M+1
  float* w = t + (M + 1);       // M
  float* p = w + M;             // M
  float* td = p + M;            // 3M+1
  float* wd = td + (3 * M + 1);  // 3M
  float* cw = wd + 3 * M;       // 3M+1
  float* cen = cw + (3 * M + 1);  // N
  for (long long r = (long long)blockIdx.x * (blockDim.x >> 5) + wid; r < A.R;
       r += (long long)gridDim.x * (blockDim.x >> 5)) {
    for (int k = lane; k <= M; k += 32) t[k] = A.sdist[r * (M + 1) + k];
    for (int k = lane; k < M; k += 32) w[k] = A.weights[r * M + k];
    __syncwarp();
    const float* s = t;
    const float* wsrc = w;
    int K = M;
    if (!A.logits_mode && A.dilation > 0.f) {
      dilate_ray(t, w, M, A.dilation, A.lo, A.hi, true, p, td, wd, lane);
      s = td + 1;       // td[1:-1]: 3M-1 posts
      wsrc = wd + 1;    // wd[1:-1]: 3M-2 bins
      K = 3 * M - 2;
    }
    if (!A.logits_mode) {
      // the logits overwrite their own weights in place (element i reads w_i only)
      float* lw = const_cast<float*>(wsrc);
      for (int i = lane; i < K; i += 32)
        lw[i] = s[i + 1] > s[i] ? logf(lw[i] + A.padding) : -INFINITY;
      __syncwarp();
    }
    const float* jit = A.jitter ? A.jitter + (A.single ? r : r * A.N) : nullptr;
    sample_ray(s, wsrc, K, A.N, jit, A.single != 0, A.lin_a, A.lin_b, A.max_jit, A.lo, A.hi, cw, cen,
               A.s_out ? A.s_out + r * (A.N + 1) : nullptr, A.t_out ? A.t_out + r * (A.N + 1) : nullptr,
               A.near ? A.near[r] : 0.f, A.far ? A.far[r] : 1.f, lane);
  }
}

struct DilateArgs {
  float* t_out;   // [R, 3M+1]
  float* w_out;   // [R, 3M]
  const float* t; // [R, M+1]
  const float* w; // [R, M]
  long long R;
  int M;
  float dilation, lo, hi;
  int renorm;
  size_t warp_floats;
};

__global__ void dilate_kernel(const DilateArgs A) {
  extern __shared__ float sm[];
  const int lane = threadIdx.x & 31;
  const int wid = threadIdx.x >> 5;
  float* base = sm + (size_t)wid * A.warp_floats;
  const int M = A.M;
  float* t = base;
  float* w = t + (M + 1);
  float* p = w + M;
  float* td = p + M;
  float* wd = td + (3 * M + 1);
  for (long long r = (long long)blockIdx.x * (blockDim.x >> 5) + wid; r < A.R;
       r += (long long)gridDim.x * (blockDim.x >> 5)) {
    for (int k = lane; k <= M; k += 32) t[k] = A.t[r * (M + 1) + k];
    for (int k = lane; k < M; k += 32) w[k] = A.w[r * M + k];
    __syncwarp();
    dilate_ray(t, w, M, A.dilation, A.lo, A.hi, A.renorm != 0, p, td, wd, lane);
    for (int k = lane; k <= 3 * M; k += 32) A.t_out[r * (3 * M + 1) + k] = td[k];
    for (int k = lane; k < 3 * M; k += 32) A.w_out[r * (3 * M) + k] = wd[k];
    __syncwarp();
  }
}

int launch_config(size_t warp_floats, int* warps, size_t* smem) {
  int dev = 0, optin = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  const size_t per = warp_floats * 4;
  int w = SAMPLE_WARPS;
  while (w > 1 && per * w > (size_t)optin) w--;
  if (per * w > (size_t)optin) return n3ds::report_error(N3DS_ERR_INVALID, "sampling: too many bins for shared memory");
  *warps = w;
  *smem = per * w;
  return N3DS_OK;
}

unsigned grid_rays(long long R, int warps) {
  const long long ctas = (R + warps - 1) / warps;
  return (unsigned)std::max<long long>(1, std::min<long long>(ctas, 148LL * 8));
}

template <typename K, typename Args>
int launch(K kernel, const Args& a, long long R, size_t warp_floats, cudaStream_t st, const char* what) {
  int warps;
  size_t smem;
  int rc = launch_config(warp_floats, &warps, &smem);
  if (rc) return rc;
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return n3ds::report_error(N3DS_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
  }
  kernel<<<grid_rays(R, warps), warps * 32, smem, st>>>(a);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return n3ds::report_error(N3DS_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
  return N3DS_OK;
}

}  // namespace

extern "C" int n3ds_max_dilate_weights(float* t_out, float* w_out, const float* t, const float* w, int64_t n_rays,
                                       int32_t n_bins, float dilation, float domain_lo, float domain_hi,
                                       int32_t renormalize, n3ds_stream_t stream) {
  if (n_rays < 0 || n_bins < 1 || n_bins > MAX_BINS)
    return n3ds::report_error(N3DS_ERR_INVALID, "max_dilate_weights: n_rays >= 0 and 1 <= n_bins <= " +
                                                    std::to_string(MAX_BINS) + " required");
  if (n_rays == 0) return N3DS_OK;
  if (!t_out || !w_out || !t || !w) return n3ds::report_error(N3DS_ERR_INVALID, "max_dilate_weights: null pointer");
  DilateArgs a{t_out, w_out, t, w, n_rays, n_bins, dilation, domain_lo, domain_hi, renormalize != 0, 0};
  a.warp_floats = size_t(n_bins + 1) + 2 * size_t(n_bins) + size_t(3 * n_bins + 1) + size_t(3 * n_bins);
  return launch(dilate_kernel, a, n_rays, a.warp_floats, reinterpret_cast<cudaStream_t>(stream),
                "max_dilate_weights");
}

static int resample_common(ResampleArgs& a, n3ds_stream_t stream, const char* what) {
  if (a.R < 0 || a.M < 1 || a.M > MAX_BINS || a.N < 2 || a.N > 16 * MAX_BINS)
    return n3ds::report_error(N3DS_ERR_INVALID, std::string(what) + ": n_rays >= 0, 1 <= n_bins <= " +
                                                    std::to_string(MAX_BINS) + " and n_samples >= 2 required");
  if (a.R == 0) return N3DS_OK;
  if (!a.sdist || !a.weights || (!a.s_out && !a.t_out))
    return n3ds::report_error(N3DS_ERR_INVALID, std::string(what) + ": inputs and an output required");
  if (a.t_out && (!a.near || !a.far))
    return n3ds::report_error(N3DS_ERR_INVALID, std::string(what) + ": tdist output needs near and far");
  const size_t M = a.M;
  a.warp_floats = (M + 1) + 2 * M + (3 * M + 1) + 3 * M + (3 * M + 1) + size_t(a.N);
  // the reference evaluates these in Python (double) before torch rounds them
  const double eps = 1.1920928955078125e-07, n = a.N;
  if (a.jitter) {
    const double u_max = eps + (1.0 - eps) / n;
    a.lin_a = 0.f;
    a.lin_b = (float)(1.0 - u_max);
    a.max_jit = (float)((1.0 - u_max) / (n - 1.0) - eps);
  } else {
    const double pad = 1.0 / (2.0 * n);
    a.lin_a = (float)pad;
    a.lin_b = (float)(1.0 - pad - eps);
    a.max_jit = 0.f;
  }
  return launch(resample_kernel, a, a.R, a.warp_floats, reinterpret_cast<cudaStream_t>(stream), what);
}

extern "C" int n3ds_sample_intervals(float* s_out, const float* t, const float* w_logits, int64_t n_rays,
                                     int32_t n_bins, int32_t n_samples, const float* jitter, int32_t single_jitter,
                                     float domain_lo, float domain_hi, n3ds_stream_t stream) {
  ResampleArgs a{};
  a.s_out = s_out;
  a.sdist = t;
  a.weights = w_logits;
  a.R = n_rays;
  a.M = n_bins;
  a.N = n_samples;
  a.jitter = jitter;
  a.single = single_jitter != 0;
  a.lo = domain_lo;
  a.hi = domain_hi;
  a.logits_mode = 1;
  return resample_common(a, stream, "sample_intervals");
}

extern "C" int n3ds_resample_intervals(float* s_out, float* t_out, const float* sdist, const float* weights,
                                       int64_t n_rays, int32_t n_bins, int32_t n_samples, float dilation,
                                       float resample_padding, const float* jitter, int32_t single_jitter,
                                       float domain_lo, float domain_hi, const float* near, const float* far,
                                       n3ds_stream_t stream) {
  ResampleArgs a{};
  a.s_out = s_out;
  a.t_out = t_out;
  a.sdist = sdist;
  a.weights = weights;
  a.R = n_rays;
  a.M = n_bins;
  a.N = n_samples;
  a.dilation = dilation;
  a.padding = resample_padding;
  a.jitter = jitter;
  a.single = single_jitter != 0;
  a.lo = domain_lo;
  a.hi = domain_hi;
  a.near = near;
  a.far = far;
  a.logits_mode = 0;
  return resample_common(a, stream, "resample_intervals");
}
