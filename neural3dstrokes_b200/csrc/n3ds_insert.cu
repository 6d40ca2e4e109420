// Stroke insertion and reset on the device: StrokeField.step_update
// (source/models.py:586-658) without a host round trip.
//
// The reference reads the stroke count and the reset count back to the host
// (.item(), nonzero, .cpu()) and samples each new stroke in a Python loop. Here the
// stroke count and the step of the last update live in device memory, and one
// single-CTA control kernel per training step
//   1. reads prev = stroke_step and takes next = min(max(next_target, prev), max),
//   2. lists the strokes below prev whose density is under reset_density (in index
//      order, as torch.nonzero),
//   3. decides the update as the reference does (models.py:604-605),
//   4. picks the top k errors (k = next - prev + resets) of the caller's error samples
//      by a 4-pass 8-bit radix select plus a bitonic sort of the selected keys in
//      shared memory (descending, ties by index), or the top shape-gradient rows,
//   5. writes the new strokes' and the reset strokes' parameters, drawn per shape type
//      as the reference samplers do (strokes.py:255-310; colours strokes.py:84-91)
//      from a counter-based hash (seed, training step, row, draw), and sets the reset
//      strokes' density to 1,
//   6. stores the new stroke count and update step.
// The gradient EMA (models.py:596-598) and the parameter clamp (models.py:576-584) are
// elementwise kernels. Random draws are not the reference's (its host torch RNG stream
// cannot be reproduced on the device); the distributions are.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>

#include <cuda_runtime.h>

#include "../../include/n3ds.h"

namespace n3ds {
int report_error(int code, const std::string& msg);  // sets n3ds_last_error (n3ds_capi.cu)
}

namespace {

constexpr int CTRL_THREADS = 1024;
constexpr float PI_F = 3.14159265358979f;

// ------------------------------------------------------------------ random draws

__device__ __forceinline__ uint64_t mix64(uint64_t z) {  // splitmix64 finaliser
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

struct Rng {
  uint64_t base;
  uint32_t n;
  __device__ Rng(uint64_t seed, long long step, long long row, uint32_t salt)
      : base(mix64(seed ^ mix64((uint64_t)step * 0xD1B54A32D192ED03ull ^ ((uint64_t)row << 20) ^ salt))), n(0) {}
  __device__ float uniform() {  // [0, 1), 24 bits
    return (float)(mix64(base + (uint64_t)(n++) * 0x9E3779B97F4A7C15ull) >> 40) * (1.0f / 16777216.0f);
  }
  __device__ float normal() {  // Box-Muller
    const float u1 = 1.0f - uniform(), u2 = uniform();
    return sqrtf(-2.0f * logf(u1)) * cosf(2.0f * PI_F * u2);
  }
};

// ------------------------------------------------------------------ samplers

// One stroke's shape parameters (strokes.py:255-306); centre_in: the error sample's
// coordinate or null. stroke_step sets the scale decay exp(-stroke_step / 200).
__device__ void sample_shape(const n3ds_stroke_sampler_t& s, long long stroke_step, const float* centre_in, Rng& rng,
                             float* out) {
  const float decay = expf(-(float)stroke_step / 200.f);
  float smin, smax, c[3];
  if (s.init_type == N3DS_INIT_RECON) {
    const float span = sqrtf(3.f);  // |[-0.5, 0.5]^3| diagonal
    smin = (0.02f + 0.12f * decay) * span;
    smax = (0.04f + 0.18f * decay) * span;
    for (int k = 0; k < 3; k++) c[k] = centre_in ? centre_in[k] : -0.5f + rng.uniform();
  } else if (s.init_type == N3DS_INIT_GEN_BOX) {
    const float span = sqrtf(3.f * 1.2f * 1.2f);
    for (int k = 0; k < 3; k++) c[k] = -0.6f + 1.2f * rng.uniform();
    const float dist = 1.f - 2.f * sqrtf(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]) / span;
    const float f = powf(4.f, -dist);
    smin = 0.05f * span * f;
    smax = 0.10f * span * f;
  } else {  // N3DS_INIT_GEN_SPHERE
    smin = 0.04f + 0.06f * decay;
    smax = 0.06f + 0.09f * decay;
    const float th = rng.uniform() * 2.f * PI_F, ph = rng.uniform() * 2.f * PI_F;
    const float rad = 1.f - decay;
    c[0] = rad * sinf(ph) * cosf(th);
    c[1] = rad * sinf(ph) * sinf(th);
    c[2] = rad * cosf(ph);
  }
  int o = 0;
  switch (s.base_sampler) {
    case N3DS_BASE_SAMPLER_ROUND: out[o++] = 0.8f * rng.uniform(); break;
    case N3DS_BASE_SAMPLER_TORUS: out[o++] = rng.uniform(); out[o++] = rng.uniform(); break;
    case N3DS_BASE_SAMPLER_CAPSULE: out[o++] = rng.uniform() + 0.25f; break;
    case N3DS_BASE_SAMPLER_LINE: out[o++] = rng.uniform() + 0.25f; out[o++] = rng.uniform() - 0.5f; break;
    case N3DS_BASE_SAMPLER_UNIFORM: out[o++] = rng.uniform(); break;
    case N3DS_BASE_SAMPLER_SPLINE: {  // strokes.py:28-37
      const float sc = rng.uniform() * (smax - smin) + smin;
      for (int p = 0; p < s.spline_points; p++)
        for (int k = 0; k < 3; k++) out[o++] = c[k] + (rng.uniform() - 0.5f) * sc;
      for (int r = 0; r < s.spline_radii; r++) out[o++] = (0.2f + 0.2f * rng.uniform()) * sc;
      break;
    }
    default: break;
  }
  if (s.s1) {
    out[o++] = rng.uniform() * (smax - smin) + smin;
  } else if (s.s3) {
    for (int k = 0; k < 3; k++) out[o++] = rng.uniform() * (smax - smin) + smin;
  }
  if (s.r)
    for (int k = 0; k < 3; k++) out[o++] = (rng.uniform() * 2.f - 1.f) * PI_F;
  if (s.t)
    for (int k = 0; k < 3; k++) out[o++] = c[k];
}

__device__ void sample_color(const n3ds_stroke_sampler_t& s, Rng& rng, float* out) {
  if (s.color_sampler == N3DS_COLOR_SAMPLER_UNIFORM) {
    for (int k = 0; k < s.n_color; k++) out[k] = rng.uniform();
  } else if (s.color_sampler == N3DS_COLOR_SAMPLER_GRADIENT) {
    for (int k = 0; k < 6; k++) out[k] = rng.uniform() - 0.5f;
    for (int k = 6; k < 12; k++) out[k] = rng.uniform();
  } else {
    for (int k = 0; k < s.n_color; k++) out[k] = rng.normal();
  }
}

// ------------------------------------------------------------------ block helpers

// Exclusive scan of v over the block (CTRL_THREADS threads); *total gets the sum.
__device__ int block_exclusive_scan(int v, int* warp_tot, int* total) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_tot[wid] = x;
  __syncthreads();
  if (wid == 0) {
    int t = lane < (CTRL_THREADS / 32) ? warp_tot[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, t, o);
      if (lane >= o) t += y;
    }
    warp_tot[lane] = t;  // inclusive warp-total prefix
  }
  __syncthreads();
  const int before = (wid > 0 ? warp_tot[wid - 1] : 0) + x - v;
  *total = warp_tot[CTRL_THREADS / 32 - 1];
  __syncthreads();
  return before;
}

__device__ __forceinline__ uint32_t order_key(float f) {  // larger float -> larger key; NaN on top
  const uint32_t u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

struct TopK {
  uint32_t* key;  // [cap] sort buffer (shared)
  int* idx;
  int cap;        // power of two
};

// Top k of keys(i), i in [0, n), into T (descending key, ascending index);
// returns the number kept (min(k, n)). keyfn(i) -> uint32 order key.
template <typename KeyFn>
__device__ int block_topk(int n, int k, KeyFn keyfn, TopK T, int* hist, int* warp_tot, int* sh) {
  k = min(k, n);
  if (k <= 0) return 0;
  // radix select of the k-th largest key
  uint32_t prefix = 0, mask = 0;
  int remaining = k;
  for (int shift = 24; shift >= 0; shift -= 8) {
    for (int d = threadIdx.x; d < 256; d += blockDim.x) hist[d] = 0;
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      const uint32_t key = keyfn(i);
      if ((key & mask) == prefix) atomicAdd(&hist[(key >> shift) & 255], 1);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      int cum = 0, d = 255;
      for (; d > 0; d--) {
        if (cum + hist[d] >= remaining) break;
        cum += hist[d];
      }
      sh[0] = d;
      sh[1] = remaining - cum;
    }
    __syncthreads();
    prefix |= (uint32_t)sh[0] << shift;
    mask |= 255u << shift;
    remaining = sh[1];
    __syncthreads();
  }
  const uint32_t thr = prefix;
  const int need_eq = remaining;  // keys equal to thr to keep (lowest indices first)
  // ordered compaction of key > thr and the first need_eq keys == thr
  int base_out = 0, base_eq = 0;
  for (int i0 = 0; i0 < n; i0 += blockDim.x) {
    const int i = i0 + threadIdx.x;
    const uint32_t key = i < n ? keyfn(i) : 0u;
    const int eq = (i < n && key == thr) ? 1 : 0;
    int eq_tot;
    const int eq_rank = base_eq + block_exclusive_scan(eq, warp_tot, &eq_tot);
    const int take = (i < n && (key > thr || (eq && eq_rank < need_eq))) ? 1 : 0;
    int take_tot;
    const int pos = base_out + block_exclusive_scan(take, warp_tot, &take_tot);
    if (take && pos < T.cap) {
      T.key[pos] = key;
      T.idx[pos] = i;
    }
    base_out += take_tot;
    base_eq += eq_tot;
  }
  const int kept = min(base_out, T.cap);
  for (int p = kept + threadIdx.x; p < T.cap; p += blockDim.x) {
    T.key[p] = 0u;
    T.idx[p] = 0x7fffffff;
  }
  __syncthreads();
  // bitonic sort: descending key, ascending index
  for (int size = 2; size <= T.cap; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int p = threadIdx.x; p < T.cap; p += blockDim.x) {
        const int q = p ^ stride;
        if (q > p) {
          const bool desc = (p & size) == 0;
          const uint32_t kp = T.key[p], kq = T.key[q];
          const int ip = T.idx[p], iq = T.idx[q];
          // "p before q" in the final order: larger key, or equal key and smaller index
          const bool p_first = kp > kq || (kp == kq && ip < iq);
          if (p_first != desc) {
            T.key[p] = kq; T.key[q] = kp;
            T.idx[p] = iq; T.idx[q] = ip;
          }
        }
      }
      __syncthreads();
    }
  }
  return min(k, kept);
}

struct StepArgs {
  n3ds_insert_config_t cfg;
  n3ds_stroke_sampler_t smp;
  float* shape;            // [max, n_shape]
  float* color;            // [max, n_color]
  float* density;          // [max]
  const float* grad_ema;   // [max, n_shape] or null
  int32_t* stroke_step;
  int32_t* last_update_step;
  long long cur_step;
  int next_target;
  float train_frac;
  const float* errors;     // [E] or null
  const float* coords;     // [E, 3]
  int n_errors;
  int* reset_idx;          // [max] scratch
  int* top_idx;            // [kcap] scratch
  float* top_params;       // [kcap, n_shape] scratch (shape-gradient mode)
  int sort_cap;
};

__global__ void __launch_bounds__(CTRL_THREADS, 1) insert_step_kernel(const StepArgs A) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ int hist[256];
  __shared__ int warp_tot[32];
  __shared__ int sh[4];
  TopK T;
  T.key = reinterpret_cast<uint32_t*>(smem);
  T.idx = reinterpret_cast<int*>(smem + (size_t)A.sort_cap * 4);
  T.cap = A.sort_cap;
  const n3ds_insert_config_t& C = A.cfg;
  const int prev = min(max(*A.stroke_step, 0), C.max_num_strokes);  // the state may hold anything
  const int last = *A.last_update_step;
  const int next = min(max(A.next_target, prev), C.max_num_strokes);
  // 2. strokes below prev to reset, in index order
  int n_reset = 0;
  for (int i0 = 0; i0 < prev; i0 += blockDim.x) {
    const int i = i0 + threadIdx.x;
    const int flag = (i < prev && A.density[i] < C.reset_density) ? 1 : 0;
    int tot;
    const int pos = n_reset + block_exclusive_scan(flag, warp_tot, &tot);
    if (flag) A.reset_idx[pos] = i;
    n_reset += tot;
  }
  __syncthreads();
  // 3. the reference's update condition
  const bool update = (next - prev >= C.min_update_interval) ||
                      (n_reset > 0 && A.cur_step - last >= C.min_reset_interval && A.train_frac < C.max_reset_frac);
  if (!update) return;
  const int k = next - prev + n_reset;
  // 4. top k error samples, or top shape-gradient rows
  int n_top = 0;
  const bool err_mode = prev > C.init_num_strokes && C.use_error_field && A.errors && A.n_errors > 0;
  const bool grad_mode = !err_mode && prev > C.init_num_strokes && C.use_shape_grads && A.grad_ema;
  if (err_mode) {
    const float* e = A.errors;
    n_top = block_topk(A.n_errors, k, [&](int i) { return order_key(e[i]); }, T, hist, warp_tot, sh);
  } else if (grad_mode) {
    // reset strokes score -inf (models.py:622); one row sum per stroke below prev
    const float* g = A.grad_ema;
    const int ns = A.smp.n_shape;
    const int* ri = A.reset_idx;
    auto score = [&](int i) {
      int lo = 0, hi = n_reset;  // reset_idx is sorted
      while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (ri[mid] < i) lo = mid + 1; else hi = mid;
      }
      if (lo < n_reset && ri[lo] == i) return order_key(-INFINITY);
      float s = 0.f;
      for (int j = 0; j < ns; j++) s += g[(size_t)i * ns + j];
      return order_key(s);
    };
    n_top = block_topk(prev, min(k, prev - n_reset), score, T, hist, warp_tot, sh);
  }
  for (int p = threadIdx.x; p < n_top; p += blockDim.x) A.top_idx[p] = T.idx[p];
  __syncthreads();
  if (grad_mode) {
    // copy the chosen rows before any row is rewritten: shape_top[p] + grad_ema[p] * rate
    // (the reference adds the EMA row at the position p, models.py:627-629)
    const int ns = A.smp.n_shape;
    for (int q = threadIdx.x; q < n_top * ns; q += blockDim.x) {
      const int p = q / ns, j = q % ns;
      A.top_params[q] = A.shape[(size_t)A.top_idx[p] * ns + j] + A.grad_ema[(size_t)p * ns + j] * C.shape_split_update_rate;
    }
  }
  __syncthreads();
  // 5. new strokes prev .. next-1, then the resets
  const int total = k;
  for (int q = threadIdx.x; q < total; q += blockDim.x) {
    const bool is_new = q < next - prev;
    const int row = is_new ? prev + q : A.reset_idx[q - (next - prev)];
    const long long sstep = is_new ? prev + q : next;
    float shape[32], col[32];
    Rng rng(C.seed, A.cur_step, row, 0x51u);
    if (grad_mode && q < n_top) {
      for (int j = 0; j < A.smp.n_shape; j++) shape[j] = A.top_params[(size_t)q * A.smp.n_shape + j];
    } else {
      float c3[3];
      const float* centre = nullptr;
      if (err_mode && q < n_top) {
        const int e = A.top_idx[q];
        c3[0] = A.coords[3 * (size_t)e];
        c3[1] = A.coords[3 * (size_t)e + 1];
        c3[2] = A.coords[3 * (size_t)e + 2];
        centre = c3;
      }
      sample_shape(A.smp, sstep, centre, rng, shape);
    }
    Rng crng(C.seed, A.cur_step, row, 0xC0u);
    sample_color(A.smp, crng, col);
    for (int j = 0; j < A.smp.n_shape; j++) A.shape[(size_t)row * A.smp.n_shape + j] = shape[j];
    for (int j = 0; j < A.smp.n_color; j++) A.color[(size_t)row * A.smp.n_color + j] = col[j];
    if (!is_new) A.density[row] = 1.0f;
  }
  __syncthreads();
  // 6. state
  if (threadIdx.x == 0) {
    *A.stroke_step = next;
    *A.last_update_step = (int32_t)A.cur_step;
  }
}

__global__ void ema_kernel(float* ema, const float* g, long long n, float decay) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    ema[i] = ema[i] * decay + g[i] * (1.0f - decay);
}

struct ClipCols {
  float lo[N3DS_CLIP_MAX_COLS], hi[N3DS_CLIP_MAX_COLS];  // NaN: no bound
};

__global__ void clip_kernel(float* x, long long rows, int cols, ClipCols c) {
  const long long n = rows * cols;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int j = (int)(i % cols);
    float v = x[i];
    if (c.lo[j] == c.lo[j]) v = fmaxf(v, c.lo[j]);
    if (c.hi[j] == c.hi[j]) v = fminf(v, c.hi[j]);
    x[i] = v;
  }
}

unsigned grid_for(long long n) {
  return (unsigned)std::max<long long>(1, std::min<long long>((n + 255) / 256, 148LL * 8));
}

int next_pow2(int v) {
  int p = 1;
  while (p < v) p <<= 1;
  return p;
}

}  // namespace

extern "C" size_t n3ds_insert_workspace_bytes(const n3ds_insert_config_t* cfg, const n3ds_stroke_sampler_t* smp) {
  if (!cfg || !smp || cfg->max_num_strokes < 1) return 0;
  const size_t m = (size_t)cfg->max_num_strokes;
  const size_t kcap = 2 * m;
  return m * 4 + kcap * 4 + kcap * (size_t)std::max(1, smp->n_shape) * 4 + 256;
}

extern "C" int n3ds_insert_step(const n3ds_insert_config_t* cfg, const n3ds_stroke_sampler_t* smp,
                                float* shape_params, float* color_params, float* density, const float* grad_ema,
                                int32_t* stroke_step, int32_t* last_update_step, int64_t cur_step,
                                int32_t next_target, float train_frac, const float* errors,
                                const float* error_coords, int64_t n_errors, void* workspace,
                                size_t workspace_bytes, n3ds_stream_t stream) {
  if (!cfg || !smp) return n3ds::report_error(N3DS_ERR_INVALID, "insert_step: config and sampler required");
  if (cfg->max_num_strokes < 1 || cfg->max_num_strokes > N3DS_INSERT_MAX_STROKES)
    return n3ds::report_error(N3DS_ERR_INVALID, "insert_step: max_num_strokes must be in [1, " +
                                                    std::to_string(N3DS_INSERT_MAX_STROKES) + "]");
  if (smp->n_shape < 0 || smp->n_shape > 32 || smp->n_color < 1 || smp->n_color > 32)
    return n3ds::report_error(N3DS_ERR_INVALID, "insert_step: n_shape must be in [0, 32], n_color in [1, 32]");
  {
    int expect = smp->s1 ? 1 : (smp->s3 ? 3 : 0);
    expect += (smp->r ? 3 : 0) + (smp->t ? 3 : 0);
    switch (smp->base_sampler) {
      case N3DS_BASE_SAMPLER_NONE: break;
      case N3DS_BASE_SAMPLER_TORUS: case N3DS_BASE_SAMPLER_LINE: expect += 2; break;
      case N3DS_BASE_SAMPLER_SPLINE:
        if (smp->spline_points < 1 || smp->spline_points > 4 || smp->spline_radii < 0 || smp->spline_radii > 2)
          return n3ds::report_error(N3DS_ERR_INVALID, "insert_step: spline sampler takes 1-4 points, 0-2 radii");
        expect += 3 * smp->spline_points + smp->spline_radii;
        break;
      case N3DS_BASE_SAMPLER_ROUND: case N3DS_BASE_SAMPLER_CAPSULE: case N3DS_BASE_SAMPLER_UNIFORM: expect += 1; break;
      default: return n3ds::report_error(N3DS_ERR_INVALID, "insert_step: unknown base sampler");
    }
    if (expect != smp->n_shape)
      return n3ds::report_error(N3DS_ERR_INVALID, "insert_step: n_shape " + std::to_string(smp->n_shape) +
                                                      " does not match the sampler's " + std::to_string(expect));
    if (smp->init_type < N3DS_INIT_RECON || smp->init_type > N3DS_INIT_GEN_SPHERE)
      return n3ds::report_error(N3DS_ERR_INVALID, "insert_step: unknown init type");
  }
  if (smp->color_sampler == N3DS_COLOR_SAMPLER_GRADIENT && smp->n_color != 12)
    return n3ds::report_error(N3DS_ERR_INVALID, "insert_step: the gradient colour sampler draws 12 values");
  if (!shape_params || !color_params || !density || !stroke_step || !last_update_step)
    return n3ds::report_error(N3DS_ERR_INVALID, "insert_step: parameter and state pointers required");
  if (n_errors < 0 || n_errors > 0x7fffffffLL || (n_errors > 0 && (!errors || !error_coords)))
    return n3ds::report_error(N3DS_ERR_INVALID, "insert_step: errors and error_coords [n_errors] required");
  const size_t need = n3ds_insert_workspace_bytes(cfg, smp);
  if (!workspace || workspace_bytes < need)
    return n3ds::report_error(N3DS_ERR_WORKSPACE, "insert_step: workspace needs " + std::to_string(need) + " bytes");
  const size_t m = (size_t)cfg->max_num_strokes, kcap = 2 * m;
  char* ws = static_cast<char*>(workspace);
  StepArgs a{};
  a.cfg = *cfg;
  a.smp = *smp;
  a.shape = shape_params;
  a.color = color_params;
  a.density = density;
  a.grad_ema = grad_ema;
  a.stroke_step = stroke_step;
  a.last_update_step = last_update_step;
  a.cur_step = cur_step;
  a.next_target = next_target;
  a.train_frac = train_frac;
  a.errors = n_errors > 0 ? errors : nullptr;
  a.coords = error_coords;
  a.n_errors = (int)n_errors;
  a.reset_idx = reinterpret_cast<int*>(ws);
  a.top_idx = reinterpret_cast<int*>(ws + m * 4);
  a.top_params = reinterpret_cast<float*>(ws + m * 4 + kcap * 4);
  a.sort_cap = next_pow2((int)std::max<size_t>(kcap, 2));
  const size_t smem = (size_t)a.sort_cap * 8;
  cudaError_t e = cudaFuncSetAttribute(insert_step_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return n3ds::report_error(N3DS_ERR_CUDA, std::string("insert_step: ") + cudaGetErrorString(e));
  insert_step_kernel<<<1, CTRL_THREADS, smem, reinterpret_cast<cudaStream_t>(stream)>>>(a);
  e = cudaGetLastError();
  if (e != cudaSuccess) return n3ds::report_error(N3DS_ERR_CUDA, std::string("insert_step: ") + cudaGetErrorString(e));
  return N3DS_OK;
}

extern "C" int n3ds_ema_update(float* ema, const float* grad, int64_t n, float decay, n3ds_stream_t stream) {
  if (n < 0 || (n > 0 && (!ema || !grad))) return n3ds::report_error(N3DS_ERR_INVALID, "ema_update: bad arguments");
  if (n == 0) return N3DS_OK;
  ema_kernel<<<grid_for(n), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(ema, grad, n, decay);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return n3ds::report_error(N3DS_ERR_CUDA, std::string("ema_update: ") + cudaGetErrorString(e));
  return N3DS_OK;
}

extern "C" int n3ds_clip_columns(float* x, int64_t rows, int32_t cols, const float* lo, const float* hi,
                                 n3ds_stream_t stream) {
  if (rows < 0 || cols < 1 || cols > N3DS_CLIP_MAX_COLS || (rows > 0 && !x) || !lo || !hi)
    return n3ds::report_error(N3DS_ERR_INVALID, "clip_columns: rows >= 0, 1 <= cols <= " +
                                                    std::to_string(N3DS_CLIP_MAX_COLS) + ", host lo / hi required");
  if (rows == 0) return N3DS_OK;
  ClipCols c;
  for (int j = 0; j < N3DS_CLIP_MAX_COLS; j++) c.lo[j] = c.hi[j] = NAN;
  std::memcpy(c.lo, lo, sizeof(float) * cols);
  std::memcpy(c.hi, hi, sizeof(float) * cols);
  clip_kernel<<<grid_for(rows * cols), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(x, rows, cols, c);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return n3ds::report_error(N3DS_ERR_CUDA, std::string("clip_columns: ") + cudaGetErrorString(e));
  return N3DS_OK;
}
