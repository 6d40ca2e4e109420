// Multi-resolution grid encoder (the reference's GridEncoder, source/gridencoder/
// src/gridencoder.cu and grid.py): per point and level, the multilinear (or
// smoothstep) interpolation of a C-channel table row at the 2^D corners of the
// point's cell, the table indexed densely or by the coherent prime hash.
//
// Layout (the reference's): inputs [B, D] float in [0, 1]; table [sO, C] of T;
// offsets [L + 1] int32 (level l owns rows offsets[l] .. offsets[l+1]); outputs
// [L, B, C]; dy_dx [B, L, D, C]; grad [L, B, C]. T is float, half or double.
//
// Schedule: one thread per (point, level) and levels outermost in the grid, so the
// CTAs of one level run together and that level's table (at most 2^21 rows x 16 B =
// 32 MB for the proposal network) stays in the 126 MB L2 while they do. A corner's
// C values are one vector load (16 B for C = 4 floats). The forward with dy_dx keeps
// the 2^D corner rows in registers and forms every directional difference from them;
// the reference gathers the 2^(D-1) x 2 x D rows again (24 for D = 3). The backward
// handles all C channels of a (point, level) in one thread and scatters each corner
// with one vector atomic (float2 / float4 atomicAdd, sm_90+) where the reference runs
// C/2 threads of two scalar atomics each.
//
// Traffic per (point, level), C = 4 floats: 12 B input, 8 x 16 B corner rows (L2
// hits once a level's table is resident), 16 B output; dy_dx adds D x 16 B.
#include <cstdint>
#include <string>
#include <type_traits>

#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "../../include/n3ds.h"
#include "n3ds_grid.cuh"

namespace n3ds {
int report_error(int code, const std::string& msg);  // sets n3ds_last_error (n3ds_capi.cu)
}

namespace {

constexpr int kThreads = 256;
using namespace n3ds::grid;

// gridencoder.cu:86-244. DYDX: also write dy/dx [B, L, D, C].
template <typename T, int D, int C, bool DYDX>
__global__ void __launch_bounds__(kThreads) grid_fwd_kernel(const float* __restrict__ inputs,
                                                             const T* __restrict__ table,
                                                             const int32_t* __restrict__ offsets,
                                                             T* __restrict__ outputs, T* __restrict__ dy_dx,
                                                             uint32_t B, uint32_t L, float S, uint32_t H, bool hash,
                                                             bool align, bool smooth, bool vec_in, bool vec_pair,
                                                             bool vec_out) {
  using A = typename Acc<T>::type;
  const uint32_t b = blockIdx.x * kThreads + threadIdx.x;
  if (b >= B) return;
  const uint32_t level = blockIdx.y;
  float x[D];
#pragma unroll
  for (int d = 0; d < D; d++) x[d] = __ldg(inputs + (size_t)b * D + d);
  T* out = outputs + ((size_t)level * B + b) * C;
  T* dd = DYDX ? dy_dx + ((size_t)b * L + level) * (size_t)(D * C) : nullptr;
  A res[C];
#pragma unroll
  for (int k = 0; k < C; k++) res[k] = A(0);
  if (!point_in_range(x, D)) {
    store_row<T, C>(out, vec_out, res);
    if (DYDX) {
#pragma unroll
      for (int d = 0; d < D; d++) store_row<T, C>(dd + d * C, vec_out, res);
    }
    return;
  }
  const Level lv = level_of(offsets, level, S, H);
  const T* tab = table + (size_t)lv.base * C;
  uint32_t cell[D];
  float frac[D], deriv[D];
  locate<D>(x, lv, align, smooth, cell, frac, deriv);

  // paired loads only where the level's rows miss L1 (2^21-row levels at 4 M points:
  // 0.127 -> 0.101 ms); on small levels, whose rows stay in L1, the pairing costs
  // more than it saves (levels of 5k-275k rows: 0.080 -> 0.098 ms)
  const bool pair_level = vec_pair && !(lv.base & 1u) && lv.hsize >= kPairMinRows;
  // corner rows kept in registers for the dy/dx differences when they fit
  constexpr bool kKeep = DYDX && (1 << D) * C <= 32;
  A rows[kKeep ? (1 << D) : 1][C];
  // corners 2j and 2j + 1 are x-neighbours: fetched together, summed in corner order
#pragma unroll
  for (int j = 0; j < (1 << (D - 1)); j++) {
    uint32_t c0[D], c1[D];
    const float w0 = corner_of<D>(2 * j, cell, frac, c0);
    const float w1 = corner_of<D>(2 * j + 1, cell, frac, c1);
    A v0[C], v1[C];
    const uint32_t r0 = cell_row<D>(c0, lv, hash, align), r1 = cell_row<D>(c1, lv, hash, align);
    load_rows2<T, C>(tab, r0, r1, vec_in, pair_level && (r0 | 1u) < lv.hsize, v0, v1);
#pragma unroll
    for (int k = 0; k < C; k++) res[k] += (A)w0 * v0[k];
#pragma unroll
    for (int k = 0; k < C; k++) res[k] += (A)w1 * v1[k];
    if constexpr (kKeep) {
#pragma unroll
      for (int k = 0; k < C; k++) { rows[2 * j][k] = v0[k]; rows[2 * j + 1][k] = v1[k]; }
    }
  }
  store_row<T, C>(out, vec_out, res);
  if constexpr (DYDX) {
    // d out / d x_gd = scale * deriv_gd * sum over the other axes' corners of
    // w_others * (row(upper along gd) - row(lower along gd))  (gridencoder.cu:203-242)
#pragma unroll
    for (int gd = 0; gd < D; gd++) {
      A g[C];
#pragma unroll
      for (int k = 0; k < C; k++) g[k] = A(0);
#pragma unroll
      for (int o = 0; o < (1 << (D - 1)); o++) {
        float w = lv.scale;
        int lo_corner = 0;
#pragma unroll
        for (int nd = 0; nd < D - 1; nd++) {
          const int d = nd >= gd ? nd + 1 : nd;
          const bool up = (o >> nd) & 1;
          w *= up ? frac[d] : 1.f - frac[d];
          lo_corner |= (up ? 1 : 0) << d;
        }
        const int hi_corner = lo_corner | (1 << gd);
        A lo[C], hi[C];
        if constexpr (kKeep) {
#pragma unroll
          for (int k = 0; k < C; k++) { lo[k] = rows[lo_corner][k]; hi[k] = rows[hi_corner][k]; }
        } else {
          uint32_t cc[D];
#pragma unroll
          for (int d = 0; d < D; d++) cc[d] = cell[d] + (uint32_t)((lo_corner >> d) & 1);
          load_row<T, C>(tab + (size_t)cell_row<D>(cc, lv, hash, align) * C, vec_in, lo);
          cc[gd] += 1u;
          load_row<T, C>(tab + (size_t)cell_row<D>(cc, lv, hash, align) * C, vec_in, hi);
        }
#pragma unroll
        for (int k = 0; k < C; k++) g[k] += (A)w * (hi[k] - lo[k]) * (A)deriv[gd];
      }
      store_row<T, C>(dd + gd * C, vec_out, g);
    }
  }
}

// gridencoder.cu:247-335: grad_table[corner rows] += w * grad[level, b, :].
// Samples along a ray sit next to each other in the batch, and at coarse levels runs
// of them share a cell, hence all 2^D corner rows: the reference's atomics then pile
// onto a few thousand rows (level 0 of the proposal grid has 4,920). Each warp finds
// its runs of equal cells (a ballot of run heads), sums a run's contributions per
// corner with a segmented shuffle scan of ceil(log2(longest run)) steps, and the
// run's last lane issues the atomic. A warp without runs takes the plain path.
template <typename T, int D, int C>
__global__ void __launch_bounds__(kThreads) grid_bwd_kernel(const T* __restrict__ grad, const float* __restrict__ inputs,
                                                             const int32_t* __restrict__ offsets, T* grad_table,
                                                             uint32_t B, float S, uint32_t H, bool hash, bool align,
                                                             bool smooth, bool vec_grad, bool vec_table) {
  using A = typename Acc<T>::type;
  constexpr unsigned kFull = 0xffffffffu;
  const uint32_t b = blockIdx.x * kThreads + threadIdx.x;
  if (__all_sync(kFull, b >= B)) return;  // whole warp past the end (warp-uniform)
  const uint32_t level = blockIdx.y;
  const int lane = threadIdx.x & 31;
  float x[D];
  bool valid = b < B;
#pragma unroll
  for (int d = 0; d < D; d++) x[d] = valid ? __ldg(inputs + (size_t)b * D + d) : 0.f;
  valid = valid && point_in_range(x, D);
  A g[C];
  if (valid) {
    load_row<T, C>(grad + ((size_t)level * B + b) * C, vec_grad, g);
  } else {
#pragma unroll
    for (int k = 0; k < C; k++) g[k] = A(0);
  }
  const Level lv = level_of(offsets, level, S, H);
  T* tab = grad_table + (size_t)lv.base * C;
  uint32_t cell[D];
  float frac[D], deriv[D];
  locate<D>(x, lv, align, smooth, cell, frac, deriv);

  // every lane executes every shuffle (full mask): no shuffle inside a short-circuit
  const int prev_valid = __shfl_up_sync(kFull, (int)valid, 1);
  bool head = !valid || lane == 0 || !prev_valid;
#pragma unroll
  for (int d = 0; d < D; d++) {
    const uint32_t prev = __shfl_up_sync(kFull, cell[d], 1);
    head = head || prev != cell[d];
  }
  const unsigned heads = __ballot_sync(kFull, head);
  if (heads == kFull) {  // no shared cells in this warp
    if (!valid) return;
#pragma unroll
    for (int corner = 0; corner < (1 << D); corner++) {
      uint32_t cc[D];
      const float w = corner_of<D>(corner, cell, frac, cc);
      A v[C];
#pragma unroll
      for (int k = 0; k < C; k++) v[k] = (A)w * g[k];
      scatter_row<T, C>(tab + (size_t)cell_row<D>(cc, lv, hash, align) * C, vec_table, v);
    }
    return;
  }
  const bool tail = lane == 31 || ((heads >> (lane + 1)) & 1u);
  const int head_lane = 31 - __clz(heads & (kFull >> (31 - lane)));
  const unsigned longest = __reduce_max_sync(kFull, tail ? (unsigned)(lane - head_lane + 1) : 0u);
#pragma unroll
  for (int corner = 0; corner < (1 << D); corner++) {
    uint32_t cc[D];
    const float w = valid ? corner_of<D>(corner, cell, frac, cc) : 0.f;
    A v[C];
#pragma unroll
    for (int k = 0; k < C; k++) v[k] = (A)w * g[k];
    for (unsigned off = 1; off < longest; off <<= 1) {
#pragma unroll
      for (int k = 0; k < C; k++) {
        const A t = __shfl_up_sync(kFull, v[k], off);
        if (lane - (int)off >= head_lane) v[k] += t;
      }
    }
    if (tail && valid) scatter_row<T, C>(tab + (size_t)cell_row<D>(cc, lv, hash, align) * C, vec_table, v);
  }
}

// gridencoder.cu:338-365: grad_inputs[b, d] = sum_l sum_c grad[l, b, c] dy_dx[b, l, d, c].
template <typename T, int D, int C>
__global__ void __launch_bounds__(kThreads) grid_input_bwd_kernel(const T* __restrict__ grad,
                                                                   const T* __restrict__ dy_dx, T* __restrict__ grad_inputs,
                                                                   uint32_t B, uint32_t L) {
  using A = typename Acc<T>::type;
  const size_t t = (size_t)blockIdx.x * kThreads + threadIdx.x;
  if (t >= (size_t)B * D) return;
  const size_t b = t / D;
  const int d = (int)(t - b * D);
  const T* dd = dy_dx + b * L * (size_t)(D * C) + d * C;
  A acc = A(0);
  for (uint32_t l = 0; l < L; l++) {
    const T* gr = grad + ((size_t)l * B + b) * C;
#pragma unroll
    for (int k = 0; k < C; k++) acc += to_acc<T>(gr[k]) * to_acc<T>(dd[(size_t)l * D * C + k]);
  }
  grad_inputs[t] = from_acc<T>(acc);
}

// gridencoder.cu:453-559: at the cell of each in-range point, grad += w sum_n(e - e_n)
// / sqrt(sum_n (e - e_n)^2 + 1e-9) per channel, n over the face neighbours within
// [0, resolution], w = weight / (2 D). Inputs have the table's type, as in the reference.
template <typename T, int D, int C>
__global__ void __launch_bounds__(kThreads) grid_tv_kernel(const T* __restrict__ inputs, const T* __restrict__ table,
                                                            T* grad, const int32_t* __restrict__ offsets, float weight,
                                                            uint32_t B, float S, uint32_t H, bool hash, bool align,
                                                            bool vec_table) {
  using A = typename Acc<T>::type;
  const uint32_t b = blockIdx.x * kThreads + threadIdx.x;
  if (b >= B) return;
  const uint32_t level = blockIdx.y;
  float x[D];
#pragma unroll
  for (int d = 0; d < D; d++) x[d] = (float)to_acc<T>(inputs[(size_t)b * D + d]);
  if (!point_in_range(x, D)) return;
  const Level lv = level_of(offsets, level, S, H);
  const T* tab = table + (size_t)lv.base * C;
  uint32_t cell[D];
  float frac[D], deriv[D];
  locate<D>(x, lv, align, false, cell, frac, deriv);
  const uint32_t row = cell_row<D>(cell, lv, hash, align);
  A e[C], s[C], sq[C];
  load_row<T, C>(tab + (size_t)row * C, vec_table, e);
#pragma unroll
  for (int k = 0; k < C; k++) s[k] = sq[k] = A(0);
#pragma unroll
  for (int d = 0; d < D; d++) {
    const uint32_t c0 = cell[d];
#pragma unroll
    for (int side = 0; side < 2; side++) {
      if (side == 0 ? !(c0 < lv.res) : !(c0 > 0u)) continue;
      cell[d] = side == 0 ? c0 + 1u : c0 - 1u;
      A n[C];
      load_row<T, C>(tab + (size_t)cell_row<D>(cell, lv, hash, align) * C, vec_table, n);
#pragma unroll
      for (int k = 0; k < C; k++) {
        const A diff = e[k] - n[k];
        s[k] += diff;
        sq[k] += diff * diff;
      }
    }
    cell[d] = c0;
  }
  const A w = (A)weight / (A)(2 * D);
  A v[C];
#pragma unroll
  for (int k = 0; k < C; k++) {
    if constexpr (std::is_same<A, double>::value) v[k] = w * s[k] / sqrt(sq[k] + 1e-9);
    else v[k] = w * s[k] * rsqrtf(sq[k] + 1e-9f);
  }
  scatter_row<T, C>(grad + ((size_t)lv.base + row) * C, vec_table, v);
}


bool aligned(const void* p, size_t bytes) { return ((uintptr_t)p % bytes) == 0; }

template <typename T, int C>
bool vec_ok(const void* p) {
  // vector loads / atomics move min(C * sizeof(T), 16) bytes at row starts
  const size_t w = C * sizeof(T) < 16 ? C * sizeof(T) : 16;
  return w > sizeof(T) && aligned(p, w);
}

struct Geo {
  uint32_t B, D, C, L;
  float S;
  uint32_t H;
  bool hash, align, smooth;
};

int launch_error(const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return n3ds::report_error(N3DS_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
  return N3DS_OK;
}

template <typename T, int D, int C>
int fwd_typed(const float* inputs, const void* table, const int32_t* offsets, void* outputs, void* dy_dx,
              const Geo& g, cudaStream_t st) {
  const dim3 grid((g.B + kThreads - 1) / kThreads, g.L);
  const bool vi = vec_ok<T, C>(table), vo = vec_ok<T, C>(outputs) && (!dy_dx || vec_ok<T, C>(dy_dx));
  const bool vp = pair_bytes<T, C>() > 0 && aligned(table, pair_bytes<T, C>() > 0 ? pair_bytes<T, C>() : 1);
  if (dy_dx)
    grid_fwd_kernel<T, D, C, true><<<grid, kThreads, 0, st>>>(inputs, (const T*)table, offsets, (T*)outputs, (T*)dy_dx,
                                                               g.B, g.L, g.S, g.H, g.hash, g.align, g.smooth, vi, vp,
                                                               vo);
  else
    grid_fwd_kernel<T, D, C, false><<<grid, kThreads, 0, st>>>(inputs, (const T*)table, offsets, (T*)outputs, nullptr,
                                                                g.B, g.L, g.S, g.H, g.hash, g.align, g.smooth, vi, vp,
                                                                vo);
  return launch_error("grid encode forward");
}

template <typename T, int D, int C>
int bwd_typed(const void* grad, const float* inputs, const int32_t* offsets, void* grad_table, const void* dy_dx,
              void* grad_inputs, const Geo& g, cudaStream_t st) {
  if (grad_table) {
    const dim3 grid((g.B + kThreads - 1) / kThreads, g.L);
    grid_bwd_kernel<T, D, C><<<grid, kThreads, 0, st>>>((const T*)grad, inputs, offsets, (T*)grad_table, g.B, g.S, g.H,
                                                         g.hash, g.align, g.smooth, vec_ok<T, C>(grad),
                                                         vec_ok<T, C>(grad_table));
    if (int rc = launch_error("grid encode backward")) return rc;
  }
  if (dy_dx && grad_inputs) {
    const size_t n = (size_t)g.B * D;
    grid_input_bwd_kernel<T, D, C><<<(unsigned)((n + kThreads - 1) / kThreads), kThreads, 0, st>>>(
        (const T*)grad, (const T*)dy_dx, (T*)grad_inputs, g.B, g.L);
    if (int rc = launch_error("grid encode input backward")) return rc;
  }
  return N3DS_OK;
}

template <typename T, int D, int C>
int tv_typed(const void* inputs, const void* table, void* grad, const int32_t* offsets, float weight, const Geo& g,
             cudaStream_t st) {
  const dim3 grid((g.B + kThreads - 1) / kThreads, g.L);
  grid_tv_kernel<T, D, C><<<grid, kThreads, 0, st>>>((const T*)inputs, (const T*)table, (T*)grad, offsets, weight, g.B,
                                                      g.S, g.H, g.hash, g.align,
                                                      vec_ok<T, C>(table) && vec_ok<T, C>(grad));
  return launch_error("grid total variation");
}

// Dispatch over dtype x D x C. F: a functor template called as F<T, D, C>::run(args...).
template <template <typename, int, int> class F, typename... Args>
int dispatch(int32_t dtype, uint32_t D, uint32_t C, Args... args) {
  auto by_c = [&](auto tag_t, auto tag_d) -> int {
    using T = typename decltype(tag_t)::type;
    constexpr int Dv = decltype(tag_d)::value;
    switch (C) {
      case 1: return F<T, Dv, 1>::run(args...);
      case 2: return F<T, Dv, 2>::run(args...);
      case 4: return F<T, Dv, 4>::run(args...);
      case 8: return F<T, Dv, 8>::run(args...);
    }
    return n3ds::report_error(N3DS_ERR_INVALID, "GridEncoding: C must be 1, 2, 4, or 8.");
  };
  auto by_d = [&](auto tag_t) -> int {
    switch (D) {
      case 2: return by_c(tag_t, std::integral_constant<int, 2>{});
      case 3: return by_c(tag_t, std::integral_constant<int, 3>{});
      case 4: return by_c(tag_t, std::integral_constant<int, 4>{});
      case 5: return by_c(tag_t, std::integral_constant<int, 5>{});
    }
    return n3ds::report_error(N3DS_ERR_INVALID, "GridEncoding: D must be 2, 3, 4, or 5.");
  };
  switch (dtype) {
    case N3DS_DTYPE_F32: return by_d(std::common_type<float>{});
    case N3DS_DTYPE_F16: return by_d(std::common_type<__half>{});
    case N3DS_DTYPE_F64: return by_d(std::common_type<double>{});
  }
  return n3ds::report_error(N3DS_ERR_INVALID, "grid encoder: dtype must be N3DS_DTYPE_F32, _F16 or _F64");
}

template <typename T, int D, int C> struct FwdOp {
  static int run(const float* i, const void* t, const int32_t* o, void* out, void* dd, Geo g, cudaStream_t s) {
    return fwd_typed<T, D, C>(i, t, o, out, dd, g, s);
  }
};
template <typename T, int D, int C> struct BwdOp {
  static int run(const void* gr, const float* i, const int32_t* o, void* gt, const void* dd, void* gi, Geo g,
                 cudaStream_t s) {
    return bwd_typed<T, D, C>(gr, i, o, gt, dd, gi, g, s);
  }
};
template <typename T, int D, int C> struct TvOp {
  static int run(const void* i, const void* t, void* gr, const int32_t* o, float w, Geo g, cudaStream_t s) {
    return tv_typed<T, D, C>(i, t, gr, o, w, g, s);
  }
};

int check_geo(const Geo& g, const void* inputs, const int32_t* offsets) {
  if (g.L < 1 || g.L > 65535) return n3ds::report_error(N3DS_ERR_INVALID, "grid encoder: levels must be in [1, 65535]");
  if (g.B > 0 && (!inputs || !offsets)) return n3ds::report_error(N3DS_ERR_INVALID, "grid encoder: inputs and offsets required");
  if (g.H < 1) return n3ds::report_error(N3DS_ERR_INVALID, "grid encoder: base resolution must be >= 1");
  return N3DS_OK;
}

}  // namespace

extern "C" int n3ds_grid_encode_forward(const float* inputs, const void* embeddings, const int32_t* offsets,
                                        void* outputs, uint32_t B, uint32_t D, uint32_t C, uint32_t L, float S,
                                        uint32_t H, void* dy_dx, uint32_t gridtype, int32_t align_corners,
                                        uint32_t interpolation, int32_t dtype, n3ds_stream_t stream) {
  const Geo g{B, D, C, L, S, H, gridtype == N3DS_GRID_HASH, align_corners != 0, interpolation == N3DS_INTERP_SMOOTHSTEP};
  if (int rc = check_geo(g, inputs, offsets)) return rc;
  if (B > 0 && (!embeddings || !outputs)) return n3ds::report_error(N3DS_ERR_INVALID, "grid encoder: embeddings and outputs required");
  if (B == 0) return N3DS_OK;
  return dispatch<FwdOp>(dtype, D, C, inputs, embeddings, offsets, outputs, dy_dx, g,
                         reinterpret_cast<cudaStream_t>(stream));
}

extern "C" int n3ds_grid_encode_backward(const void* grad, const float* inputs, const void* embeddings,
                                         const int32_t* offsets, void* grad_embeddings, uint32_t B, uint32_t D,
                                         uint32_t C, uint32_t L, float S, uint32_t H, const void* dy_dx,
                                         void* grad_inputs, uint32_t gridtype, int32_t align_corners,
                                         uint32_t interpolation, int32_t dtype, n3ds_stream_t stream) {
  (void)embeddings;  // the table gradient does not depend on the table
  const Geo g{B, D, C, L, S, H, gridtype == N3DS_GRID_HASH, align_corners != 0, interpolation == N3DS_INTERP_SMOOTHSTEP};
  if (int rc = check_geo(g, inputs, offsets)) return rc;
  if (B > 0 && !grad) return n3ds::report_error(N3DS_ERR_INVALID, "grid encoder: grad required");
  if (B == 0 || (!grad_embeddings && !(dy_dx && grad_inputs))) return N3DS_OK;
  return dispatch<BwdOp>(dtype, D, C, grad, inputs, offsets, grad_embeddings, dy_dx, grad_inputs, g,
                         reinterpret_cast<cudaStream_t>(stream));
}

extern "C" int n3ds_grid_total_variation(const void* inputs, const void* embeddings, void* grad,
                                         const int32_t* offsets, float weight, uint32_t B, uint32_t D, uint32_t C,
                                         uint32_t L, float S, uint32_t H, uint32_t gridtype, int32_t align_corners,
                                         int32_t dtype, n3ds_stream_t stream) {
  const Geo g{B, D, C, L, S, H, gridtype == N3DS_GRID_HASH, align_corners != 0, false};
  if (int rc = check_geo(g, inputs, offsets)) return rc;
  if (B > 0 && (!embeddings || !grad)) return n3ds::report_error(N3DS_ERR_INVALID, "grid encoder: embeddings and grad required");
  if (B == 0) return N3DS_OK;
  return dispatch<TvOp>(dtype, D, C, inputs, embeddings, grad, offsets, weight, g,
                        reinterpret_cast<cudaStream_t>(stream));
}
