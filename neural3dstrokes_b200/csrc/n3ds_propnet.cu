// Fused density network of the proposal and error fields (source/models.py:285-523:
// MLP.predict_density on the hash-grid encoder, density_layer = Linear(L*C, 64),
// ReLU, Linear(64, 1), then softplus(raw + density_bias); PropMLP and ErrorMLP with
// disable_rgb). The reference evaluates it as its grid kernels plus torch layers,
// which write and read the [points, 64] hidden activations several times; here one
// kernel per direction keeps them on chip.
//
// Schedule: persistent CTAs of 128 threads, one point per thread, tiles of 128
// points (the MMA's M).
// Forward, per tile: each thread warps its point, encodes it on the grid into
// registers and writes its feature row into the tile's A operand (hi and lo tf32
// halves); one thread issues the first layer as tcgen05.mma kind::tf32 (M 128, N 64,
// K = L*C padded to 8 or 16, three products per K step for the split) into tensor
// memory; every thread reads its accumulator row back with tcgen05.ld and finishes
// bias, ReLU, the 64-wide second layer and softplus on the CUDA cores.
// Backward, per tile: the forward's feature record is reloaded and the first layer
// recomputed on the tensor cores; each thread forms d raw = g e^z / (e^z + 1) (torch's
// softplus backward) and the ReLU mask of its 64 hidden units. Because the mask is
// exactly 0 or 1, the adjoint dh = d raw w2 mask factors into two bf16 products with
// float32 accuracy (kind::f16, K-major operands): dfeat = d raw (.) (mask . W1') with
// W1' = w2 (.) W1 in three bf16 terms (M 128 points, N 16, K 64), and
// dW1 = w2 (.) (mask^T . (d raw feat)) with d raw feat in three bf16 terms and d raw
// itself as one more column, which gives db1 (M 64 hidden, N 16, K 128 points),
// accumulated in tensor memory over all of the CTA's tiles. dW2 and db2 are warp
// reductions. dfeat goes straight into the grid's table scatter, runs of points in
// one cell summed in the warp before the atomic.
//
// Each wait for the tensor cores is bounded (one second unless set); when one runs
// out the kernel ORs bit 2 into the status word, waits once more (bounded) for
// anything still in flight, frees its tensor memory and returns.
#include <cstdint>
#include <string>

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "../../include/n3ds.h"
#include "n3ds_grid.cuh"
#include "n3ds_tc.cuh"

namespace n3ds {
int report_error(int code, const std::string& msg);  // sets n3ds_last_error (n3ds_capi.cu)
}

namespace {

using namespace n3ds::grid;
using namespace n3ds::tc;

constexpr int kTile = 128;                 // points per tile: MMA M and threads per CTA
constexpr int kHidden = N3DS_DENSITY_HIDDEN;
constexpr int kMaxFeat = 16;               // feature columns in shared memory (L * C <= 15, then d raw)
constexpr int kStatusWait = 2;             // the field's ST_WAIT_TIMEOUT bit

// Shared-memory layout (bytes), every tensor-core operand K-major without swizzle
// (n3ds_tc.cuh; tf32 takes 4 values, bf16 8 values per 16-byte core-matrix row).
// Forward and backward, tf32 hi and lo halves:
//   feature rows: element (p, f) at (f / 4) * 2048 + p * 16 + (f % 4) * 4 (A of the
//     first layer: M = points, K = features);
//   W1: element (j, f) at (f / 4) * 1024 + j * 16 + (f % 4) * 4 (B: N = hidden, K = f).
// Backward only, bf16:
//   W1' = w2 (.) W1 in three terms: element (f, j) at (j / 8) * 256 + f * 16 + (j % 8) * 2
//     (B of dfeat: N = f, K = hidden);
//   ReLU mask rows: element (p, j) at (j / 8) * 2048 + p * 16 + (j % 8) * 2 (A of dfeat:
//     M = points, K = hidden);
//   ReLU mask transposed: element (j, p) at (j / 8) * 2304 + (j % 8) * 16 + (p / 8) * 144
//     + (p % 8) * 2 (A of dW1: M = hidden, K = points);
//   dr (.) feat in three terms, dr itself in column L*C: element (f, p) at (f / 8) * 2304
//     + (f % 8) * 16 + (p / 8) * 144 + (p % 8) * 2 (B of dW1: N = f, K = points).
// The transposed tiles are written a column per thread; their 144-byte K chunks (128 +
// 16 of padding) put a warp's 32 columns on distinct banks.
constexpr uint32_t kW1pBytes = kMaxFeat * kHidden * 2;  // 2 KB per term
constexpr uint32_t kMaskBytes = kTile * kHidden * 2;    // 16 KB
constexpr uint32_t kPadChunk = 144, kPadGroup = 16 * kPadChunk;
constexpr uint32_t kMaskTBytes = (kHidden / 8) * kPadGroup;   // 18 KB
constexpr uint32_t kBpBytes = (kMaxFeat / 8) * kPadGroup;     // 4.5 KB per term
struct Misc {
  float b1[kHidden];
  float w2[kHidden];
  Level lv[kMaxFeat];
  uint64_t bar;
  uint32_t tmem;
  float b2;
};
// Offsets for kc 4-value feature chunks (2 when L * C <= 8, else 4): the feature and
// W1 tiles hold only the chunks the first layer reads.
struct Smem {
  uint32_t feat_hi, feat_lo, w1_hi, w1_lo, w1p, mask, maskt, bp, misc_fwd, misc_bwd, fwd_bytes, bwd_bytes;
};
__host__ __device__ constexpr Smem smem_layout(int kc) {
  Smem m{};
  m.feat_hi = 0;
  m.feat_lo = kc * 2048;
  m.w1_hi = 2 * kc * 2048;
  m.w1_lo = m.w1_hi + kc * 1024;
  m.w1p = m.w1_lo + kc * 1024;  // the forward's Misc, then the backward's tiles
  m.misc_fwd = m.w1p;
  m.mask = m.w1p + 3 * kW1pBytes;
  m.maskt = m.mask + kMaskBytes;
  m.bp = m.maskt + kMaskTBytes;
  m.misc_bwd = m.bp + 3 * kBpBytes;
  m.fwd_bytes = m.misc_fwd + (uint32_t)sizeof(Misc);
  m.bwd_bytes = m.misc_bwd + (uint32_t)sizeof(Misc);
  return m;
}
static_assert(smem_layout(4).misc_bwd % 16 == 0 && smem_layout(2).misc_bwd % 16 == 0, "16-byte operand alignment");

// Tensor-memory columns: first-layer accumulator [128 x 64], mask . W1' [128 x 16],
// mask^T . (dr feat) [64 x 16] (rows in lanes 0-15 of each 32-lane quarter, the
// M = 64 layout).
constexpr uint32_t COL_D1 = 0, COL_DF = 64, COL_DW = 96;
constexpr uint32_t kColsFwd = 64, kColsBwd = 128;

constexpr uint32_t IDESC_L1 = idesc_tf32(kTile, kHidden, false, false);  // feat x W1, tf32
constexpr uint32_t IDESC_DF = idesc_bf16(kTile, 16);                     // mask x W1', bf16
constexpr uint32_t IDESC_DW = idesc_bf16(kHidden, 16);                   // mask^T x (dr feat), bf16

struct NetLaunch {
  const float* coords;
  const float* table;
  const int32_t* offsets;
  const float *w1, *b1, *w2, *b2;
  const float* features_in;  // backward: the forward's record
  const float* grad_density;
  float* density;
  float* features_out;       // forward: the record, or null
  float* coords_warped;
  float *g_table, *g_w1, *g_b1, *g_w2, *g_b2;
  int32_t* status;
  long long n;
  uint32_t L, F, stride;     // levels, features (L * C), record floats per point
  float S;
  uint32_t H;
  float density_bias, warp_scale, grid_bound, inv_two_bound;
  int warp;
  bool raw_output;
  bool hash, align, vec_table, vec_pair;
  unsigned long long wait_ns;
  int test_stall;
};

// ------------------------------------------------------------ per-point steps

// The coordinate map of models.py:19-33 (and coord.contract, source/utils/coord.py:
// 5-11), then GridEncoder.forward's (x + bound) / (2 bound), rounded as torch's CUDA
// ops round them (a division by a Python scalar is a multiplication by its float32
// reciprocal; sqrt and division correctly rounded).
__device__ __forceinline__ void warp_point(const NetLaunch& P, float x0, float x1, float x2, float (&w)[3],
                                           float (&u)[3]) {
  w[0] = x0; w[1] = x1; w[2] = x2;
  if (P.warp == N3DS_WARP_SCALE) {
#pragma unroll
    for (int d = 0; d < 3; d++) w[d] = w[d] * P.warp_scale;
  } else if (P.warp == N3DS_WARP_CONTRACT) {
    const float eps = 1.1920928955078125e-7f;  // torch.finfo(float32).eps
    // torch.sum(x ** 2, dim=-1) as torch's CUDA reduction forms it for three values:
    // squares rounded, then (x0^2 + x2^2) + x1^2, no fused multiply-add
    const float m = fmaxf(__fadd_rn(__fadd_rn(__fmul_rn(x0, x0), __fmul_rn(x2, x2)), __fmul_rn(x1, x1)), eps);
    if (!(m <= 1.f)) {
      // correctly rounded square root and division, as torch's ops (the library is
      // built with approximate sqrt and division)
      const float k = __fdiv_rn(__fsub_rn(__fmul_rn(2.f, __fsqrt_rn(m)), 1.f), m);
#pragma unroll
      for (int d = 0; d < 3; d++) w[d] = k * w[d];
    }
#pragma unroll
    for (int d = 0; d < 3; d++) w[d] = w[d] * 0.5f;
  }
#pragma unroll
  for (int d = 0; d < 3; d++) u[d] = (w[d] + P.grid_bound) * P.inv_two_bound;
}

// L * C features of point u (grid_fwd_kernel's arithmetic, n3ds_grid.cu), zero when
// u leaves [0, 1]^3 as in the reference.
template <int C, int LMAX, bool EXACT>
__device__ __forceinline__ void encode_point(const NetLaunch& P, const Level* lvs, const float (&u)[3],
                                             float (&f)[kMaxFeat]) {
#pragma unroll
  for (int i = 0; i < kMaxFeat; i++) f[i] = 0.f;
  if (!point_in_range(u, 3)) return;
#pragma unroll
  for (int l = 0; l < LMAX; l++) {
    if (EXACT || l < (int)P.L) {  // EXACT: LMAX is the level count, no guard
      const Level lv = lvs[l];
      const float* tab = P.table + (size_t)lv.base * C;
      uint32_t cell[3];
      float frac[3], deriv[3];
      locate<3>(u, lv, P.align, false, cell, frac, deriv);
      const bool pair_level = P.vec_pair && !(lv.base & 1u) && lv.hsize >= kPairMinRows;
      float res[C];
#pragma unroll
      for (int c = 0; c < C; c++) res[c] = 0.f;
#pragma unroll
      for (int j = 0; j < 4; j++) {
        uint32_t c0[3], c1[3];
        const float w0 = corner_of<3>(2 * j, cell, frac, c0);
        const float w1 = corner_of<3>(2 * j + 1, cell, frac, c1);
        float v0[C], v1[C];
        const uint32_t r0 = cell_row<3>(c0, lv, P.hash, P.align), r1 = cell_row<3>(c1, lv, P.hash, P.align);
        load_rows2<float, C>(tab, r0, r1, P.vec_table, pair_level && (r0 | 1u) < lv.hsize, v0, v1);
#pragma unroll
        for (int c = 0; c < C; c++) res[c] += w0 * v0[c];
#pragma unroll
        for (int c = 0; c < C; c++) res[c] += w1 * v1[c];
      }
#pragma unroll
      for (int c = 0; c < C; c++) f[l * C + c] = res[c];
    }
  }
}

// The first n_chunks 4-value chunks of a 16-value row into the tile's hi and lo
// buffers.
template <int N>
__device__ __forceinline__ void store_split_row(uint8_t* hi_base, uint8_t* lo_base, uint32_t row_off,
                                                uint32_t chunk_stride, const float (&v)[N], int n_chunks) {
#pragma unroll
  for (int c = 0; c < N / 4; c++) {
    if (c >= n_chunks) break;
    float h[4], l[4];
#pragma unroll
    for (int k = 0; k < 4; k++) split_tf32(v[4 * c + k], h[k], l[k]);
    *reinterpret_cast<float4*>(hi_base + c * chunk_stride + row_off) = make_float4(h[0], h[1], h[2], h[3]);
    *reinterpret_cast<float4*>(lo_base + c * chunk_stride + row_off) = make_float4(l[0], l[1], l[2], l[3]);
  }
}

// torch.relu: NaN stays NaN.
__device__ __forceinline__ float relu_t(float x) { return (x > 0.f || x != x) ? x : 0.f; }

// torch's softplus (beta 1, threshold 20) and its backward, g * e^z / (e^z + 1)
// evaluated in that order.
__device__ __forceinline__ float softplus_t(float z) { return z > 20.f ? z : log1pf(expf(z)); }
__device__ __forceinline__ float softplus_backward_t(float g, float z) {
  if (z > 20.f) return g;
  const float e = expf(z);
  return __fdiv_rn(__fmul_rn(g, e), __fadd_rn(e, 1.f));
}

// Sum of v[0..15] over the warp's lanes by transposition: lane l returns the sum of
// slot l >> 1 (each slot ends in two lanes).
__device__ __forceinline__ float warp_slot_sum16(float (&v)[16], int lane) {
#pragma unroll
  for (int s = 0; s < 4; s++) {
    const int o = 16 >> s, n = 8 >> s;
    const bool up = (lane & o) != 0;
#pragma unroll
    for (int i = 0; i < 8; i++) {
      if (i < n) {
        const float send = up ? v[i] : v[i + n];
        const float keep = up ? v[i + n] : v[i];
        v[i] = keep + __shfl_xor_sync(0xffffffffu, send, o);
      }
    }
  }
  return v[0] + __shfl_xor_sync(0xffffffffu, v[0], 1);
}

// bf16 bits of x (round to nearest even) and x = h + m + l in three bf16 terms (each
// remainder exact in float32): 24 significant bits, a float32 value to about 2^-24.
__device__ __forceinline__ uint16_t bf16_bits(float x) { return __bfloat16_as_ushort(__float2bfloat16_rn(x)); }
__device__ __forceinline__ void split3_bf16(float x, uint16_t& h, uint16_t& m, uint16_t& l) {
  const __nv_bfloat16 bh = __float2bfloat16_rn(x);
  const float r1 = x - __bfloat162float(bh);
  const __nv_bfloat16 bm = __float2bfloat16_rn(r1);
  const float r2 = r1 - __bfloat162float(bm);
  h = __bfloat16_as_ushort(bh);
  m = __bfloat16_as_ushort(bm);
  l = bf16_bits(r2);
}

// CTA set-up shared by both kernels: W1 split into its tile buffers (and, for the
// backward, W1' = w2 (.) W1 in three bf16 terms), biases, the second layer, level
// geometry, the mbarrier and the tensor memory.
__device__ __forceinline__ void setup_cta(const NetLaunch& P, uint8_t* smem, const Smem& L, Misc* M, uint32_t cols,
                                          bool backward) {
  const int tid = threadIdx.x;
  const int kc = (int)(L.feat_lo / 2048);
  for (int i = tid; i < kHidden * kMaxFeat; i += kTile) {
    const int j = i / kMaxFeat, f = i % kMaxFeat;
    const float w = f < (int)P.F ? P.w1[j * P.F + f] : 0.f;
    if (f < 4 * kc) {
      float h, l;
      split_tf32(w, h, l);
      const uint32_t off = (f / 4) * 1024 + j * 16 + (f % 4) * 4;
      *reinterpret_cast<float*>(smem + L.w1_hi + off) = h;
      *reinterpret_cast<float*>(smem + L.w1_lo + off) = l;
    }
    if (backward) {
      uint16_t t[3];
      split3_bf16(w * P.w2[j], t[0], t[1], t[2]);
      const uint32_t o2 = (j / 8) * 256 + f * 16 + (j % 8) * 2;
#pragma unroll
      for (int k = 0; k < 3; k++) *reinterpret_cast<uint16_t*>(smem + L.w1p + k * kW1pBytes + o2) = t[k];
    }
  }
  if (tid < kHidden) {
    M->b1[tid] = P.b1[tid];
    M->w2[tid] = P.w2[tid];
  }
  if (tid < (int)P.L) M->lv[tid] = level_of(P.offsets, tid, P.S, P.H);
  if (tid == 0) {
    M->b2 = P.b2[0];
    mbar_init(&M->bar, 1);
  }
  if (tid < 32) tmem_alloc(&M->tmem, cols);
  fence_proxy_async();
  tc_fence_before_sync();
  __syncthreads();
  tc_fence_after_sync();
}

// Wait for the tensor cores' arrival on the barrier (bounded); CTA-uniform result.
// The phase advances only on success, so that a later wait still watches the phase
// that work in flight will complete.
__device__ __forceinline__ bool wait_mma(const NetLaunch& P, Misc* M, uint32_t& phase) {
  const bool ok = __syncthreads_and(mbar_wait_bounded(&M->bar, phase, P.wait_ns)) != 0;
  if (ok) {
    phase ^= 1u;
    tc_fence_after_sync();
  }
  return ok;
}

// Leave: after a timeout, one more bounded wait for work still in flight; then the
// tensor memory is freed by the warp that allocated it.
__device__ __forceinline__ void teardown(const NetLaunch& P, Misc* M, uint32_t phase, bool timed_out, uint32_t cols) {
  if (timed_out) {
    if (threadIdx.x == 0) {
      if (P.status) atomicOr(P.status, kStatusWait);
      if (!P.test_stall) mbar_wait_bounded(&M->bar, phase, P.wait_ns);
    }
  }
  tc_fence_before_sync();
  __syncthreads();
  tc_fence_after_sync();
  if (threadIdx.x < 32) tmem_dealloc(M->tmem, cols);
}

// ------------------------------------------------------------ forward

template <int C, int LMAX, bool EXACT>
__global__ void __launch_bounds__(kTile, 4) density_fwd_kernel(NetLaunch P) {
  extern __shared__ __align__(1024) uint8_t smem[];
  const Smem SL = smem_layout(P.F > 8 ? 4 : 2);
  Misc* M = reinterpret_cast<Misc*>(smem + SL.misc_fwd);
  setup_cta(P, smem, SL, M, kColsFwd, false);
  const int tid = threadIdx.x, warp = tid >> 5;
  const uint32_t tmem = M->tmem;
  const uint32_t lane_addr = tmem + ((uint32_t)(warp * 32) << 16);
  const int ks_count = (int)((P.F + 7) / 8);
  const long long n_tiles = (P.n + kTile - 1) / kTile;
  uint32_t phase = 0;
  bool timed_out = false;
  for (long long tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
    const long long b = tile * kTile + tid;
    const bool valid = b < P.n;
    float f[kMaxFeat];
    {
      float x[3] = {0.f, 0.f, 0.f}, w[3], u[3];
      if (valid) {
        x[0] = P.coords[3 * b];
        x[1] = P.coords[3 * b + 1];
        x[2] = P.coords[3 * b + 2];
      }
      warp_point(P, x[0], x[1], x[2], w, u);
      if (valid) {
        encode_point<C, LMAX, EXACT>(P, M->lv, u, f);
        if (P.coords_warped) {
          P.coords_warped[3 * b] = w[0];
          P.coords_warped[3 * b + 1] = w[1];
          P.coords_warped[3 * b + 2] = w[2];
        }
        if (P.features_out) {
          float4* rec = reinterpret_cast<float4*>(P.features_out + b * P.stride);
#pragma unroll
          for (int c = 0; c < kMaxFeat / 4; c++) {
            if (c < (int)(P.stride / 4)) rec[c] = make_float4(f[4 * c], f[4 * c + 1], f[4 * c + 2], f[4 * c + 3]);
          }
        }
      } else {
#pragma unroll
        for (int i = 0; i < kMaxFeat; i++) f[i] = 0.f;
      }
    }
    store_split_row(smem + SL.feat_hi, smem + SL.feat_lo, tid * 16, 2048, f, 2 * ks_count);
    fence_proxy_async();
    tc_fence_before_sync();
    __syncthreads();
    tc_fence_after_sync();
    if (tid == 0 && !P.test_stall) {
      const uint32_t fh = smem_u32(smem + SL.feat_hi), fl = smem_u32(smem + SL.feat_lo);
      const uint32_t wh = smem_u32(smem + SL.w1_hi), wl = smem_u32(smem + SL.w1_lo);
      for (int ks = 0; ks < ks_count; ks++) {
        const uint64_t a_hi = smem_desc(fh + ks * 4096, 2048, 128), a_lo = smem_desc(fl + ks * 4096, 2048, 128);
        const uint64_t b_hi = smem_desc(wh + ks * 2048, 1024, 128), b_lo = smem_desc(wl + ks * 2048, 1024, 128);
        mma_tf32(tmem + COL_D1, a_lo, b_hi, IDESC_L1, ks > 0);
        mma_tf32(tmem + COL_D1, a_hi, b_lo, IDESC_L1, true);
        mma_tf32(tmem + COL_D1, a_hi, b_hi, IDESC_L1, true);
      }
      mma_commit(&M->bar);
    }
    if (!wait_mma(P, M, phase)) {
      timed_out = true;
      break;
    }
    float raw = M->b2;
#pragma unroll
    for (int c = 0; c < kHidden / 16; c++) {
      float v[16];
      tmem_ld16(lane_addr + COL_D1 + c * 16, v);
#pragma unroll
      for (int k = 0; k < 16; k++) raw = fmaf(relu_t(v[k] + M->b1[c * 16 + k]), M->w2[c * 16 + k], raw);
    }
    if (valid) P.density[b] = P.raw_output ? raw : softplus_t(raw + P.density_bias);
  }
  teardown(P, M, phase, timed_out, kColsFwd);
}

// ------------------------------------------------------------ backward

// grad_table[corner rows of point u at level lv] += w * g, with runs of lanes in one
// cell summed first (grid_bwd_kernel's scheme, n3ds_grid.cu). Every lane calls it.
template <int C>
__device__ __forceinline__ void scatter_level(const NetLaunch& P, const Level& lv, const float (&u)[3], bool valid,
                                              const float (&g)[C], int lane) {
  constexpr unsigned kFull = 0xffffffffu;
  float* tab = P.g_table + (size_t)lv.base * C;
  uint32_t cell[3];
  float frac[3], deriv[3];
  locate<3>(u, lv, P.align, false, cell, frac, deriv);
  const int prev_valid = __shfl_up_sync(kFull, (int)valid, 1);
  bool head = !valid || lane == 0 || !prev_valid;
#pragma unroll
  for (int d = 0; d < 3; d++) {
    const uint32_t prev = __shfl_up_sync(kFull, cell[d], 1);
    head = head || prev != cell[d];
  }
  const unsigned heads = __ballot_sync(kFull, head);
  if (heads == kFull) {
    if (!valid) return;
#pragma unroll
    for (int corner = 0; corner < 8; corner++) {
      uint32_t cc[3];
      const float w = corner_of<3>(corner, cell, frac, cc);
      float v[C];
#pragma unroll
      for (int c = 0; c < C; c++) v[c] = w * g[c];
      scatter_row<float, C>(tab + (size_t)cell_row<3>(cc, lv, P.hash, P.align) * C, P.vec_table, v);
    }
    return;
  }
  const bool tail = lane == 31 || ((heads >> (lane + 1)) & 1u);
  const int head_lane = 31 - __clz(heads & (kFull >> (31 - lane)));
  const unsigned longest = __reduce_max_sync(kFull, tail ? (unsigned)(lane - head_lane + 1) : 0u);
#pragma unroll
  for (int corner = 0; corner < 8; corner++) {
    uint32_t cc[3];
    const float w = valid ? corner_of<3>(corner, cell, frac, cc) : 0.f;
    float v[C];
#pragma unroll
    for (int c = 0; c < C; c++) v[c] = w * g[c];
    for (unsigned off = 1; off < longest; off <<= 1) {
#pragma unroll
      for (int c = 0; c < C; c++) {
        const float t = __shfl_up_sync(kFull, v[c], off);
        if (lane - (int)off >= head_lane) v[c] += t;
      }
    }
    if (tail && valid) scatter_row<float, C>(tab + (size_t)cell_row<3>(cc, lv, P.hash, P.align) * C, P.vec_table, v);
  }
}

// Backward. With mask[p, j] = [pre > 0] (exactly 0 or 1 in bf16) the ReLU adjoint
// dh = dr w2 mask factors as
//   dfeat[p, f] = dr[p] sum_j mask[p, j] W1'[j, f],      W1' = w2 (.) W1,
//   dW1[j, f]   = w2[j] sum_p mask[p, j] (dr feat)[p, f],  db1 the same with feat = 1,
// two bf16 products whose operand terms are exact (the mask) or float32 split in three
// bf16 terms, accumulated in float32: float32 accuracy from kind::f16 MMAs with
// K-major operands only.
// The inputs of a tile (coordinates, feature record, upstream gradient) of this
// thread's point; FP floats of features (8 when L * C <= 8, else 16).
template <int FP>
struct BwdIn {
  float x[3];
  float f[FP];
  float g;
  bool valid;
};
template <int FP>
__device__ __forceinline__ void load_bwd_in(const NetLaunch& P, long long b, BwdIn<FP>& in) {
  in.valid = b < P.n;
  in.g = 0.f;
#pragma unroll
  for (int i = 0; i < 3; i++) in.x[i] = 0.f;
#pragma unroll
  for (int i = 0; i < FP; i++) in.f[i] = 0.f;
  if (!in.valid) return;
#pragma unroll
  for (int i = 0; i < 3; i++) in.x[i] = P.coords[3 * b + i];
  const float4* rec = reinterpret_cast<const float4*>(P.features_in + b * P.stride);
#pragma unroll
  for (int c = 0; c < FP / 4; c++) {
    if (c < (int)(P.stride / 4)) {
      const float4 r = rec[c];
      in.f[4 * c] = r.x; in.f[4 * c + 1] = r.y; in.f[4 * c + 2] = r.z; in.f[4 * c + 3] = r.w;
    }
  }
  in.g = P.grad_density[b];
}

template <int C, int LMAX, bool EXACT>
__global__ void __launch_bounds__(kTile, 3) density_bwd_kernel(NetLaunch P) {
  constexpr int FP = C * LMAX <= 8 ? 8 : 16;
  extern __shared__ __align__(1024) uint8_t smem[];
  const Smem SL = smem_layout(P.F > 8 ? 4 : 2);
  Misc* M = reinterpret_cast<Misc*>(smem + SL.misc_bwd);
  // the d raw (.) feat tile's columns beyond L * C (d raw itself) stay zero: cleared
  // once here, the tiles write columns 0 .. L * C only
  for (uint32_t i = threadIdx.x; i < 3 * kBpBytes / 4; i += kTile) reinterpret_cast<float*>(smem + SL.bp)[i] = 0.f;
  setup_cta(P, smem, SL, M, kColsBwd, true);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t tmem = M->tmem;
  const uint32_t lane_addr = tmem + ((uint32_t)(warp * 32) << 16);
  const int ks_count = (int)((P.F + 7) / 8);
  const long long n_tiles = (P.n + kTile - 1) / kTile;
  uint32_t phase = 0;
  bool timed_out = false, any = false;
  float acc_w2[kHidden / 16] = {0.f, 0.f, 0.f, 0.f};
  float acc_b2 = 0.f;
  const uint32_t fh = smem_u32(smem + SL.feat_hi), fl = smem_u32(smem + SL.feat_lo);
  const uint32_t wh = smem_u32(smem + SL.w1_hi), wl = smem_u32(smem + SL.w1_lo);
  const uint32_t w1p = smem_u32(smem + SL.w1p), mask = smem_u32(smem + SL.mask);
  const uint32_t maskt = smem_u32(smem + SL.maskt), bp = smem_u32(smem + SL.bp);
  // this thread's column offset in the transposed tiles
  const uint32_t col_off = (uint32_t)(tid / 8) * kPadChunk + (uint32_t)(tid % 8) * 2;
  BwdIn<FP> in;
  load_bwd_in<FP>(P, (long long)blockIdx.x * kTile + tid, in);
  for (long long tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
    const bool valid = in.valid;
    const float g = in.g;
    float u[3] = {0.f, 0.f, 0.f};
    float f[FP];
#pragma unroll
    for (int i = 0; i < FP; i++) f[i] = i < (int)P.F ? in.f[i] : 0.f;
    if (valid) {
      float w[3];
      warp_point(P, in.x[0], in.x[1], in.x[2], w, u);
    }
    store_split_row<FP>(smem + SL.feat_hi, smem + SL.feat_lo, tid * 16, 2048, f, 2 * ks_count);
    fence_proxy_async();
    tc_fence_before_sync();
    __syncthreads();
    tc_fence_after_sync();
    if (tid == 0 && !P.test_stall) {
      for (int ks = 0; ks < ks_count; ks++) {
        const uint64_t a_hi = smem_desc(fh + ks * 4096, 2048, 128), a_lo = smem_desc(fl + ks * 4096, 2048, 128);
        const uint64_t b_hi = smem_desc(wh + ks * 2048, 1024, 128), b_lo = smem_desc(wl + ks * 2048, 1024, 128);
        mma_tf32(tmem + COL_D1, a_lo, b_hi, IDESC_L1, ks > 0);
        mma_tf32(tmem + COL_D1, a_hi, b_lo, IDESC_L1, true);
        mma_tf32(tmem + COL_D1, a_hi, b_hi, IDESC_L1, true);
      }
      mma_commit(&M->bar);
    }
    if (!wait_mma(P, M, phase)) {
      timed_out = true;
      break;
    }
    // raw, then d raw through softplus
    float raw = M->b2;
#pragma unroll
    for (int c = 0; c < kHidden / 16; c++) {
      float v[16];
      tmem_ld16(lane_addr + COL_D1 + c * 16, v);
#pragma unroll
      for (int k = 0; k < 16; k++) raw = fmaf(relu_t(v[k] + M->b1[c * 16 + k]), M->w2[c * 16 + k], raw);
    }
    const float dr = P.raw_output ? g : softplus_backward_t(g, raw + P.density_bias);
    {
      float s = dr;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
      acc_b2 += s;
    }
    // the ReLU mask (rows and transposed) and dW2 (warp sums of dr relu(pre))
#pragma unroll
    for (int c = 0; c < kHidden / 16; c++) {
      float v[16];
      tmem_ld16(lane_addr + COL_D1 + c * 16, v);
      uint32_t words[8];
#pragma unroll
      for (int k = 0; k < 16; k++) {
        const float pre = v[k] + M->b1[c * 16 + k];
        // torch.relu's backward passes the gradient unless the output is <= 0 (NaN passes)
        const uint32_t one = pre <= 0.f ? 0u : 0x3F80u;
        if (k % 2 == 0) words[k / 2] = one;
        else words[k / 2] |= one << 16;
        const int j = c * 16 + k;
        *reinterpret_cast<uint16_t*>(smem + SL.maskt + (j / 8) * kPadGroup + (j % 8) * 16 + col_off) =
            (uint16_t)one;
        v[k] = dr * relu_t(pre);
      }
      *reinterpret_cast<uint4*>(smem + SL.mask + (2 * c) * 2048 + tid * 16) =
          make_uint4(words[0], words[1], words[2], words[3]);
      *reinterpret_cast<uint4*>(smem + SL.mask + (2 * c + 1) * 2048 + tid * 16) =
          make_uint4(words[4], words[5], words[6], words[7]);
      acc_w2[c] += warp_slot_sum16(v, lane);
    }
    // dr (.) feat and dr (column L * C), three bf16 terms, transposed
    auto put_bp = [&](int i, float x) {
      uint16_t t[3];
      split3_bf16(x, t[0], t[1], t[2]);
      const uint32_t o = (i / 8) * kPadGroup + (i % 8) * 16 + col_off;
#pragma unroll
      for (int k = 0; k < 3; k++) *reinterpret_cast<uint16_t*>(smem + SL.bp + k * kBpBytes + o) = t[k];
    };
#pragma unroll
    for (int i = 0; i < FP; i++) {
      if (i < (int)P.F) put_bp(i, dr * f[i]);
    }
    put_bp((int)P.F, dr);
    fence_proxy_async();
    tc_fence_before_sync();
    __syncthreads();
    tc_fence_after_sync();
    if (tid == 0 && !P.test_stall) {
      // mask . W1' (M 128 points, N 16, K 64 hidden)
      for (int ks = 0; ks < kHidden / 16; ks++) {
        const uint64_t a = smem_desc(mask + ks * 4096, 2048, 128);
#pragma unroll
        for (int t = 0; t < 3; t++)
          mma_bf16(tmem + COL_DF, a, smem_desc(w1p + t * kW1pBytes + ks * 512, 256, 128), IDESC_DF, ks > 0 || t > 0);
      }
      // mask^T . (dr feat) (M 64 hidden, N 16, K 128 points), accumulated over tiles
      for (int ks = 0; ks < kTile / 16; ks++) {
        const uint64_t a = smem_desc(maskt + ks * 2 * kPadChunk, kPadChunk, kPadGroup);
#pragma unroll
        for (int t = 0; t < 3; t++)
          mma_bf16(tmem + COL_DW, a, smem_desc(bp + t * kBpBytes + ks * 2 * kPadChunk, kPadChunk, kPadGroup),
                   IDESC_DW, any || ks > 0 || t > 0);
      }
      mma_commit(&M->bar);
    }
    any = true;
    // the next tile's inputs, fetched while the tensor cores work and the scatter runs
    load_bwd_in<FP>(P, (tile + gridDim.x) * kTile + tid, in);
    if (!wait_mma(P, M, phase)) {
      timed_out = true;
      break;
    }
    float df[16];
    tmem_ld16(lane_addr + COL_DF, df);
    const bool in_grid = valid && point_in_range(u, 3);
#pragma unroll
    for (int l = 0; l < LMAX; l++) {
      if (EXACT || l < (int)P.L) {
        float gl[C];
#pragma unroll
        for (int c = 0; c < C; c++) gl[c] = in_grid ? dr * df[l * C + c] : 0.f;
        scatter_level<C>(P, M->lv[l], u, in_grid, gl, lane);
      }
    }
  }
  if (any && !timed_out) {
    float v[16];
    tmem_ld16(lane_addr + COL_DW, v);
    if (lane < 16) {  // M = 64 rows: lanes 0-15 of each quarter
      const int j = warp * 16 + lane;
      const float w2j = M->w2[j];
#pragma unroll
      for (int i = 0; i < kMaxFeat; i++) {
        if (i < (int)P.F) atomicAdd(P.g_w1 + j * P.F + i, w2j * v[i]);
        else if (i == (int)P.F) atomicAdd(P.g_b1 + j, w2j * v[i]);
      }
    }
    if ((lane & 1) == 0) {
#pragma unroll
      for (int c = 0; c < kHidden / 16; c++) atomicAdd(P.g_w2 + c * 16 + (lane >> 1), acc_w2[c]);
    }
    if (lane == 0) atomicAdd(P.g_b2, acc_b2);
  }
  teardown(P, M, phase, timed_out, kColsBwd);
}

// ------------------------------------------------------------ hash-decay statistics

constexpr int kRedThreads = 256;
constexpr int kRedUnroll = 4;  // float4 loads in flight per thread

// Level l's rows are one contiguous run of rows(l) * C floats, read as float4 when the
// table is 16-byte aligned and the run starts and ends on a 4-float boundary (always
// for GridEncoder's levels, rounded to multiples of 8 rows): element e of the run
// holds channel e % C, and with C in 1, 2, 4 that is its float4 position % C.
__device__ __forceinline__ void level_run(const int32_t* offsets, uint32_t l, uint32_t C, uint32_t& r0,
                                          uint32_t& rows) {
  r0 = (uint32_t)offsets[l];
  rows = (uint32_t)offsets[l + 1] - r0;
}

// Per (level, channel) means of squares; blocks of one level stride over its run.
__global__ void __launch_bounds__(kRedThreads) level_sumsq_kernel(const float* __restrict__ table,
                                                                  const int32_t* __restrict__ offsets, uint32_t C,
                                                                  uint32_t n_ch, bool vec, float* __restrict__ out) {
  const uint32_t l = blockIdx.y;
  uint32_t r0, rows;
  level_run(offsets, l, C, r0, rows);
  const float inv_rows = 1.f / (float)rows;
  const float* run = table + (size_t)r0 * C;
  const size_t n = (size_t)rows * C;
  float acc[4] = {0.f, 0.f, 0.f, 0.f};  // by position in a float4: channel = position % C
  const size_t stride = (size_t)gridDim.x * kRedThreads;
  if (vec && ((size_t)r0 * C) % 4 == 0 && n % 4 == 0) {
    const float4* v = reinterpret_cast<const float4*>(run);
    const size_t n4 = n / 4;
    for (size_t i = (size_t)blockIdx.x * kRedThreads + threadIdx.x; i < n4; i += kRedUnroll * stride) {
      float4 q[kRedUnroll];
#pragma unroll
      for (int k = 0; k < kRedUnroll; k++) q[k] = i + k * stride < n4 ? __ldg(v + i + k * stride) : make_float4(0, 0, 0, 0);
#pragma unroll
      for (int k = 0; k < kRedUnroll; k++) {
        acc[0] = fmaf(q[k].x, q[k].x, acc[0]);
        acc[1] = fmaf(q[k].y, q[k].y, acc[1]);
        acc[2] = fmaf(q[k].z, q[k].z, acc[2]);
        acc[3] = fmaf(q[k].w, q[k].w, acc[3]);
      }
    }
  } else {
    for (size_t i = (size_t)blockIdx.x * kRedThreads + threadIdx.x; i < n; i += stride) {
      const float t = run[i];
      acc[i % 4] = fmaf(t, t, acc[i % 4]);
    }
  }
  // fold positions into channels (position p holds channel p % C)
  float ch[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
  for (int q = 0; q < 4; q++) ch[q % C] += acc[q];
  __shared__ float red[kRedThreads / 32][4];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int c = 0; c < 4; c++) {
    float t = ch[c];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if (lane == 0) red[w][c] = t;
  }
  __syncthreads();
  if (threadIdx.x < n_ch) {
    float t = 0.f;
    for (int i = 0; i < kRedThreads / 32; i++) t += red[i][threadIdx.x];
    atomicAdd(out + l * C + threadIdx.x, t * inv_rows);
  }
}

// grad_table[row, c] += grad_out[l, c] * 2 * table[row, c] / rows(l) for the reduced
// channels c < n_ch.
__global__ void __launch_bounds__(kRedThreads) level_sumsq_bwd_kernel(const float* __restrict__ table,
                                                                      const int32_t* __restrict__ offsets,
                                                                      uint32_t C, uint32_t n_ch, bool vec,
                                                                      const float* __restrict__ grad_out,
                                                                      float* __restrict__ grad_table) {
  const uint32_t l = blockIdx.y;
  uint32_t r0, rows;
  level_run(offsets, l, C, r0, rows);
  const float s = 2.f / (float)rows;
  float k4[4];
#pragma unroll
  for (int q = 0; q < 4; q++) k4[q] = (uint32_t)(q % C) < n_ch ? grad_out[l * C + q % C] * s : 0.f;
  const size_t n = (size_t)rows * C;
  const size_t stride = (size_t)gridDim.x * kRedThreads;
  const float* run = table + (size_t)r0 * C;
  float* grun = grad_table + (size_t)r0 * C;
  if (vec && ((size_t)r0 * C) % 4 == 0 && n % 4 == 0) {
    const float4* v = reinterpret_cast<const float4*>(run);
    float4* gv = reinterpret_cast<float4*>(grun);
    const size_t n4 = n / 4;
    for (size_t i = (size_t)blockIdx.x * kRedThreads + threadIdx.x; i < n4; i += kRedUnroll * stride) {
      float4 q[kRedUnroll], g[kRedUnroll];
#pragma unroll
      for (int k = 0; k < kRedUnroll; k++) {
        if (i + k * stride < n4) {
          q[k] = __ldg(v + i + k * stride);
          g[k] = gv[i + k * stride];
        }
      }
#pragma unroll
      for (int k = 0; k < kRedUnroll; k++) {
        if (i + k * stride < n4) {
          g[k].x = fmaf(k4[0], q[k].x, g[k].x);
          g[k].y = fmaf(k4[1], q[k].y, g[k].y);
          g[k].z = fmaf(k4[2], q[k].z, g[k].z);
          g[k].w = fmaf(k4[3], q[k].w, g[k].w);
          gv[i + k * stride] = g[k];
        }
      }
    }
  } else {
    for (size_t i = (size_t)blockIdx.x * kRedThreads + threadIdx.x; i < n; i += stride)
      grun[i] = fmaf(k4[i % 4], run[i], grun[i]);
  }
}

// Blocks per level: enough for about eight resident CTAs per SM over all levels.
dim3 level_grid(uint32_t L) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  uint32_t per = (uint32_t)(sms * 8) / L;
  return dim3(per < 16 ? 16 : per, L);
}

// ------------------------------------------------------------ host side

int launch_error(const char* what) {
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return n3ds::report_error(N3DS_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
  return N3DS_OK;
}

bool aligned(const void* p, size_t bytes) { return ((uintptr_t)p % bytes) == 0; }

int check_net(const n3ds_density_net_t* net, int64_t n) {
  if (!net) return n3ds::report_error(N3DS_ERR_INVALID, "density net: null descriptor");
  if (n < 0) return n3ds::report_error(N3DS_ERR_INVALID, "density net: negative point count");
  const uint32_t C = net->level_dim, L = net->n_levels;
  if (C != 1 && C != 2 && C != 4)
    return n3ds::report_error(N3DS_ERR_UNSUPPORTED, "density net: level_dim must be 1, 2 or 4");
  // the product tiles have 16 columns: L * C features and the column of d raw
  if (L < 1 || L * C > (uint32_t)kMaxFeat - 1)
    return n3ds::report_error(N3DS_ERR_UNSUPPORTED, "density net: n_levels * level_dim must be in [1, 15]");
  if (net->base_resolution < 1) return n3ds::report_error(N3DS_ERR_INVALID, "density net: base resolution must be >= 1");
  if (net->warp != N3DS_WARP_SCALE && net->warp != N3DS_WARP_CONTRACT && net->warp != N3DS_WARP_NONE)
    return n3ds::report_error(N3DS_ERR_INVALID, "density net: unknown warp");
  if (!(net->grid_bound > 0.f)) return n3ds::report_error(N3DS_ERR_INVALID, "density net: grid_bound must be > 0");
  if (n > 0 && (!net->table || !net->offsets || !net->w1 || !net->b1 || !net->w2 || !net->b2))
    return n3ds::report_error(N3DS_ERR_INVALID, "density net: table, offsets and the four layer tensors are required");
  return N3DS_OK;
}

NetLaunch make_launch(const n3ds_density_net_t* net, const float* coords, int64_t n) {
  NetLaunch P{};
  P.coords = coords;
  P.table = net->table;
  P.offsets = net->offsets;
  P.w1 = net->w1;
  P.b1 = net->b1;
  P.w2 = net->w2;
  P.b2 = net->b2;
  P.status = net->status;
  P.n = n;
  P.L = net->n_levels;
  P.F = net->n_levels * net->level_dim;
  P.stride = (P.F + 3) / 4 * 4;
  P.S = net->log2_per_level_scale;
  P.H = net->base_resolution;
  P.density_bias = net->density_bias;
  P.warp = net->warp;
  P.raw_output = net->raw_output != 0;
  P.warp_scale = net->warp_scale;
  P.grid_bound = net->grid_bound;
  P.inv_two_bound = 1.f / (2.f * net->grid_bound);
  P.hash = net->gridtype == N3DS_GRID_HASH;
  P.align = net->align_corners != 0;
  const uint32_t C = net->level_dim;
  const size_t vw = C * 4 < 16 ? C * 4 : 16;
  P.vec_table = vw > 4 && aligned(net->table, vw);
  // a pair of rows is one load of 2 C floats (8, 16 or 32 bytes), aligned to its size
  P.vec_pair = aligned(net->table, 2 * C * 4);
  P.wait_ns = (unsigned long long)(net->wait_limit_us > 0 ? net->wait_limit_us : 1000000) * 1000ull;
  P.test_stall = net->test_stall;
  return P;
}

// CTAs the kernel can keep resident on the device (cached per kernel and device): the
// limits of its registers, shared memory (carveout set to the maximum) and threads,
// and at most 512 / cols per SM so that every resident CTA's tensor-memory
// allocation succeeds at once. (The runtime's occupancy calculator answers one CTA
// per SM for these tensor-memory kernels, below what the hardware runs.)
template <typename K>
int resident(K kernel, uint32_t smem_max, uint32_t smem, uint32_t cols, int* cache) {
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 16) dev = 0;
  if (cache[dev] == 0) {
    // the larger layout's size, so that either layout launches whichever came first
    cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_max);
    cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    cudaFuncAttributes fa{};
    int regs_sm = 0, smem_sm = 0, reserved = 0, threads_sm = 0, sms = 0;
    cudaFuncGetAttributes(&fa, kernel);
    cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev);
    cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
    cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev);
    cudaDeviceGetAttribute(&threads_sm, cudaDevAttrMaxThreadsPerMultiProcessor, dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int regs_warp = ((fa.numRegs > 0 ? fa.numRegs : 255) * 32 + 255) / 256 * 256;  // 256-register units
    const int by_regs = regs_sm / (regs_warp * (kTile / 32));
    const int by_smem = smem_sm / ((int)smem + (int)fa.sharedSizeBytes + reserved);
    const int by_threads = threads_sm / kTile;
    int blocks = by_regs < by_smem ? by_regs : by_smem;
    if (by_threads < blocks) blocks = by_threads;
    if (blocks > (int)(512 / cols)) blocks = (int)(512 / cols);
    cache[dev] = (blocks > 0 ? blocks : 1) * (sms > 0 ? sms : 1);
  }
  return cache[dev];
}

int g_resident[2];  // CTAs of the last forward and backward launch

template <int C, int LMAX, bool EXACT>
int fwd_c(const NetLaunch& P, cudaStream_t st) {
  static int cache[2][16] = {{0}};
  const int kc = P.F > 8 ? 4 : 2;
  const uint32_t smem = smem_layout(kc).fwd_bytes;
  const int slots = resident(density_fwd_kernel<C, LMAX, EXACT>, smem_layout(4).fwd_bytes, smem, kColsFwd, cache[kc / 4]);
  g_resident[0] = slots;
  const long long tiles = (P.n + kTile - 1) / kTile;
  const int grid = (int)(tiles < slots ? tiles : slots);
  density_fwd_kernel<C, LMAX, EXACT><<<grid, kTile, smem, st>>>(P);
  return launch_error("density net forward");
}

template <int C, int LMAX, bool EXACT>
int bwd_c(const NetLaunch& P, cudaStream_t st) {
  static int cache[2][16] = {{0}};
  const int kc = P.F > 8 ? 4 : 2;
  const uint32_t smem = smem_layout(kc).bwd_bytes;
  const int slots = resident(density_bwd_kernel<C, LMAX, EXACT>, smem_layout(4).bwd_bytes, smem, kColsBwd, cache[kc / 4]);
  g_resident[1] = slots;
  const long long tiles = (P.n + kTile - 1) / kTile;
  const int grid = (int)(tiles < slots ? tiles : slots);
  density_bwd_kernel<C, LMAX, EXACT><<<grid, kTile, smem, st>>>(P);
  return launch_error("density net backward");
}

// Instantiations by level_dim and the level count: exact counts for the stroke model's
// networks (PropMLP 6 and 8 levels x 1 channel, ErrorMLP 5 x 2; unguarded level loops,
// so every level's gathers can be in flight together), else a bound (8 or 15 levels
// for C = 1, 7 for C = 2, 3 for C = 4) with a guard per level.
template <bool BWD, int C, int LMAX, bool EXACT>
int launch_net(const NetLaunch& P, cudaStream_t st) {
  return BWD ? bwd_c<C, LMAX, EXACT>(P, st) : fwd_c<C, LMAX, EXACT>(P, st);
}
template <bool BWD>
int dispatch_net(const NetLaunch& P, uint32_t C, cudaStream_t st) {
  if (C == 1) {
    if (P.L == 6) return launch_net<BWD, 1, 6, true>(P, st);
    if (P.L == 8) return launch_net<BWD, 1, 8, true>(P, st);
    if (P.L < 8) return launch_net<BWD, 1, 8, false>(P, st);
    return launch_net<BWD, 1, 15, false>(P, st);
  }
  if (C == 2) {
    if (P.L == 5) return launch_net<BWD, 2, 5, true>(P, st);
    return launch_net<BWD, 2, 7, false>(P, st);
  }
  return launch_net<BWD, 4, 3, false>(P, st);
}

int check_levels(const float* table, const int32_t* offsets, uint32_t L, uint32_t C, const void* out) {
  if (L < 1 || L > 65535) return n3ds::report_error(N3DS_ERR_INVALID, "level statistics: levels must be in [1, 65535]");
  if (C != 1 && C != 2 && C != 4)
    return n3ds::report_error(N3DS_ERR_UNSUPPORTED, "level statistics: level_dim must be 1, 2 or 4");
  if (!table || !offsets || !out) return n3ds::report_error(N3DS_ERR_INVALID, "level statistics: null pointer");
  return N3DS_OK;
}

}  // namespace

extern "C" int n3ds_density_net_resident_ctas(int32_t backward) {
  return g_resident[backward ? 1 : 0];
}

extern "C" int n3ds_density_net_feature_stride(uint32_t n_levels, uint32_t level_dim) {
  return (int)((n_levels * level_dim + 3) / 4 * 4);
}

extern "C" int n3ds_density_net_forward(const n3ds_density_net_t* net, const float* coords, int64_t n_points,
                                        float* density, float* features, float* coords_warped,
                                        n3ds_stream_t stream) {
  if (int rc = check_net(net, n_points)) return rc;
  if (n_points == 0) return N3DS_OK;
  if (!coords || !density) return n3ds::report_error(N3DS_ERR_INVALID, "density net: coords and density are required");
  if (features && !aligned(features, 16))
    return n3ds::report_error(N3DS_ERR_INVALID, "density net: the feature record must be 16-byte aligned");
  NetLaunch P = make_launch(net, coords, n_points);
  P.density = density;
  P.features_out = features;
  P.coords_warped = coords_warped;
  const cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  return dispatch_net<false>(P, net->level_dim, st);
}

extern "C" int n3ds_density_net_backward(const n3ds_density_net_t* net, const float* coords, const float* features,
                                         const float* grad_density, int64_t n_points, float* grad_table,
                                         float* grad_w1, float* grad_b1, float* grad_w2, float* grad_b2,
                                         n3ds_stream_t stream) {
  if (int rc = check_net(net, n_points)) return rc;
  if (n_points == 0) return N3DS_OK;
  if (!coords || !features || !grad_density || !grad_table || !grad_w1 || !grad_b1 || !grad_w2 || !grad_b2)
    return n3ds::report_error(N3DS_ERR_INVALID, "density net backward: every input and gradient pointer is required");
  if (!aligned(features, 16))
    return n3ds::report_error(N3DS_ERR_INVALID, "density net: the feature record must be 16-byte aligned");
  NetLaunch P = make_launch(net, coords, n_points);
  P.features_in = features;
  P.grad_density = grad_density;
  P.g_table = grad_table;
  P.g_w1 = grad_w1;
  P.g_b1 = grad_b1;
  P.g_w2 = grad_w2;
  P.g_b2 = grad_b2;
  const size_t vw = net->level_dim * 4 < 16 ? net->level_dim * 4 : 16;
  P.vec_table = vw > 4 && aligned(grad_table, vw);
  const cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  return dispatch_net<true>(P, net->level_dim, st);
}

extern "C" int n3ds_grid_level_mean_sq(const float* table, const int32_t* offsets, uint32_t n_levels,
                                       uint32_t level_dim, int32_t all_channels, float* out, n3ds_stream_t stream) {
  if (int rc = check_levels(table, offsets, n_levels, level_dim, out)) return rc;
  const cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  if (cudaMemsetAsync(out, 0, sizeof(float) * n_levels * level_dim, st) != cudaSuccess)
    return launch_error("level statistics: clear");
  const bool vec = level_dim <= 4 && 4 % level_dim == 0 && aligned(table, 16);
  level_sumsq_kernel<<<level_grid(n_levels), kRedThreads, 0, st>>>(table, offsets, level_dim,
                                                                  all_channels ? level_dim : 1u, vec, out);
  return launch_error("level statistics");
}

extern "C" int n3ds_grid_level_mean_sq_backward(const float* table, const int32_t* offsets, uint32_t n_levels,
                                                uint32_t level_dim, int32_t all_channels, const float* grad_out,
                                                float* grad_table, n3ds_stream_t stream) {
  if (int rc = check_levels(table, offsets, n_levels, level_dim, grad_table)) return rc;
  if (!grad_out) return n3ds::report_error(N3DS_ERR_INVALID, "level statistics backward: null gradient");
  const bool vec = level_dim <= 4 && 4 % level_dim == 0 && aligned(table, 16) && aligned(grad_table, 16);
  level_sumsq_bwd_kernel<<<level_grid(n_levels), kRedThreads, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      table, offsets, level_dim, all_channels ? level_dim : 1u, vec, grad_out, grad_table);
  return launch_error("level statistics backward");
}
