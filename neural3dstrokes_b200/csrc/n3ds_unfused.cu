// The reference `_strokelib` operators over dense [P, S] tensors, B200 style.
//
// The reference runs one thread per (sample, stroke) with 32-bit indices and up to
// 14 global atomics per pair (strokes_backward.cu), and one thread per sample with
// row-strided reads (compositing.cu). Here:
// - stroke forward: a warp evaluates 32 samples x 32 strokes with the stroke record
//   broadcast from shared memory, and writes alpha / colour rows coalesced through a
//   transposed shared-memory tile;
// - stroke backward: lane = stroke; each lane accumulates its stroke's reduced
//   gradient slots in registers across all samples the warp visits (no per-pair
//   atomics), grad_x is a warp sum per sample;
// - compose forward / exact backward: a warp per sample row, lane = stroke within a
//   32-stroke chunk, transmittance by shuffle product-scans and the composites under
//   each stroke by a shuffle scan of affine maps (no division by 1 - alpha); rows are
//   streamed coalesced, nothing is staged in shared memory. The compat backward (the
//   reference's own formulas, which divide by 1 - alpha) keeps lane = sample with the
//   reference's serial loop over 32-row tiles transposed in shared memory.
// All indices are 64-bit.
#include <algorithm>

#include "n3ds_eval.cuh"
#include "n3ds_unfused.cuh"

namespace n3ds {

constexpr int UF_WARPS = 4;

// Forward: a block stages one 32-stroke block's records (and culling spheres) once and
// its warps sweep 32-point tiles of it (persistent grid). Each warp evaluates the
// tile with lane = point, the stroke warp-uniform, into a transposed shared tile, then
// writes the [32 points x 32 strokes] block of alpha (and sdf) rows: as float4 rows
// (8 lanes per row, 4 rows per store) when the rows are 16-byte aligned, else lane =
// stroke. The constant-rgb colour block is the same for every point, so each lane
// keeps the (at most) three float4 / scalars it stores per tile in registers.
// With culling (alpha alone requested: no sdf, no texcoords), a stroke whose culling
// sphere provably keeps alpha at exactly 0 in float32 at all 32 points of the tile (the
// reference's own value there; see n3ds_stroke_forward) is not evaluated and stores 0.
// Curve class of a launch (a drop-in call has one sdf_id): the kernel carries only that
// class's evaluation code, so the primitive kernels hold far fewer registers.
enum UfClass : int { UF_PRIM = 0, UF_QUAD = 1, UF_CUBIC = 2 };

template <int CLS>
__device__ __forceinline__ float uf_alpha(const float* rec, V3 x, float rinv, float* sdf_out) {
  const float4 h = rec4(rec)[0];
  const int kind = __float_as_int(h.x);
  const int mode = (kind >> 8) & 3;
  float sdf, f = 1.f;
  if (CLS == UF_PRIM) {
    const V3 p = prim_local(rec, x);
    sdf = prim_sdf(kind & 15, p, rec);
    if (kind & K_S3FAC) f = s3_factor(kind & 15, p, xyz(rec4(rec)[R_S / 4]), rec);
  } else if (CLS == UF_QUAD) {
    QuadFwd q;
    sdf = quad_eval(rec, x, q);
  } else {
    CubicFwd c;
    sdf = cubic_eval(rec, x, c, (kind & 15) == B_CATMULL_ROM);
  }
  *sdf_out = sdf;
  if (mode == STEP_HARD) return sdf <= 0.f ? 1.f : 0.f;
  return soft_alpha(mode, -sdf * (h.y * f * rinv));
}

template <int CLS>
__global__ void __launch_bounds__(UF_WARPS * 32, 6) uf_stroke_fwd_kernel(const UfStroke L) {
  __shared__ __align__(16) float recs[32 * REC_FLOATS];
  __shared__ float4 cull_c[32];
  __shared__ float cull_r[32];
  __shared__ float ta[UF_WARPS][32][33];
  // the SDF tile (dynamic shared memory) only when the sdf output is requested
  extern __shared__ float tsd_dyn[];
  float(*tsd)[32][33] = reinterpret_cast<float(*)[32][33]>(tsd_dyn);
  const int s0 = blockIdx.y * 32;
  const int ns = min(32, L.n_strokes - s0);
  for (int i = threadIdx.x; i < ns * REC_FLOATS; i += blockDim.x) recs[i] = L.recs[(long long)s0 * REC_FLOATS + i];
  const bool cull = L.cull_a != nullptr;
  if (cull && threadIdx.x < ns) {
    cull_c[threadIdx.x] = reinterpret_cast<const float4*>(L.cull_a)[s0 + threadIdx.x];
    cull_r[threadIdx.x] = fabsf(L.cull_b[s0 + threadIdx.x]);
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long long S = L.n_strokes;
  const bool vec = ns == 32 && (S & 3) == 0 && (reinterpret_cast<uintptr_t>(L.alpha) & 15) == 0 &&
                   (reinterpret_cast<uintptr_t>(L.color) & 15) == 0 &&
                   (reinterpret_cast<uintptr_t>(L.sdf) & 15) == 0;
  // constant colour of stroke j, channel ch, at element 3 j + ch of a tile row
  auto col_elem = [&](int e) { return recs[(e / 3) * REC_FLOATS + R_COLOR + e % 3]; };
  // vector stores: float4 (lane + 8 k) % 24 of the 96-float row, k = t % 3;
  // lane-per-element stores: elements lane, lane + 32, lane + 64
  auto pat = [&](int k) {
    const int q = (lane + 8 * k) % 24;
    return vec ? make_float4(col_elem(4 * q), col_elem(4 * q + 1), col_elem(4 * q + 2), col_elem(4 * q + 3))
               : make_float4(0.f, 0.f, 0.f, 0.f);
  };
  auto elem = [&](int k) { return lane + 32 * k < 3 * ns ? col_elem(lane + 32 * k) : 0.f; };
  const float4 cp0 = pat(0), cp1 = pat(1), cp2 = pat(2);
  const float cv0 = elem(0), cv1 = elem(1), cv2 = elem(2);
  for (long long p0 = ((long long)blockIdx.x * UF_WARPS + warp) * 32; p0 < L.n_points;
       p0 += (long long)gridDim.x * UF_WARPS * 32) {
    const long long p = p0 + lane;
    const long long pp = p < L.n_points ? p : p0;
    const V3 x = v3(L.x[3 * pp], L.x[3 * pp + 1], L.x[3 * pp + 2]);
    const float r = L.radius[pp];
    const float rinv = 1.f / r;
    for (int j = 0; j < ns; j++) {
      bool need = true;
      if (cull) {
        const float4 c = cull_c[j];
        const float dx = x.x - c.x, dy = x.y - c.y, dz = x.z - c.z;
        const float lim = c.w + cull_r[j] * r;
        const bool out = lim >= 0.f && dx * dx + dy * dy + dz * dz > lim * lim;
        need = __any_sync(0xffffffffu, !out);
      }
      float a = 0.f, sd = 0.f;
      if (need) a = uf_alpha<CLS>(recs + j * REC_FLOATS, x, rinv, &sd);
      ta[warp][lane][j] = a;
      if (L.sdf) tsd[warp][lane][j] = sd;
    }
    __syncwarp();
    const int rows = (int)min(32LL, L.n_points - p0);
    if (vec && rows == 32) {
      const int c4 = (lane & 7) * 4;
#pragma unroll
      for (int t = 0; t < 8; t++) {
        const int rr = t * 4 + (lane >> 3);
        const long long row = (p0 + rr) * S + s0 + c4;
        *reinterpret_cast<float4*>(L.alpha + row) =
            make_float4(ta[warp][rr][c4], ta[warp][rr][c4 + 1], ta[warp][rr][c4 + 2], ta[warp][rr][c4 + 3]);
        if (L.sdf)
          *reinterpret_cast<float4*>(L.sdf + row) =
              make_float4(tsd[warp][rr][c4], tsd[warp][rr][c4 + 1], tsd[warp][rr][c4 + 2], tsd[warp][rr][c4 + 3]);
      }
      if (L.color_const) {
        // 32 rows x 24 float4: store q = lane + 32 t is float4 (q % 24) of row q / 24
#pragma unroll
        for (int t = 0; t < 24; t++) {
          const int q = lane + 32 * t;
          const int rr = q / 24;
          *reinterpret_cast<float4*>(L.color + ((p0 + rr) * S + s0) * 3 + (q - rr * 24) * 4) =
              t % 3 == 0 ? cp0 : (t % 3 == 1 ? cp1 : cp2);
        }
      }
    } else {
      for (int rr = 0; rr < rows; rr++) {
        const long long row = (p0 + rr) * S + s0;
        if (lane < ns) {
          L.alpha[row + lane] = ta[warp][rr][lane];
          if (L.sdf) L.sdf[row + lane] = tsd[warp][rr][lane];
        }
        if (L.color_const) {
          if (lane < 3 * ns) L.color[row * 3 + lane] = cv0;
          if (lane + 32 < 3 * ns) L.color[row * 3 + lane + 32] = cv1;
          if (lane + 64 < 3 * ns) L.color[row * 3 + lane + 64] = cv2;
        }
      }
    }
    __syncwarp();
  }
}

// CLS: the call's curve class (one sdf_id per call), so that the kernel carries only
// that class's evaluation and adjoint; COMPAT: L.compat as a constant.
template <int CLS, int COMPAT>
__global__ void __launch_bounds__(UF_WARPS * 32) uf_stroke_bwd_kernel(const UfStroke L) {
  constexpr int NV = CLS == UF_CUBIC ? 32 : 16;
  constexpr int compat = COMPAT;
  // padded stride (17 float4): rows stay 16-byte aligned and lane-indexed 128-bit
  // record loads of a quarter warp hit distinct banks
  constexpr int RS = REC_FLOATS + 4;
  __shared__ __align__(16) float recs[32 * RS];
  const int s0 = blockIdx.y * 32;
  const int ns = min(32, L.n_strokes - s0);
  for (int i = threadIdx.x; i < ns * REC_FLOATS; i += blockDim.x)
    recs[(i / REC_FLOATS) * RS + (i % REC_FLOATS)] = L.recs[(long long)s0 * REC_FLOATS + i];
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const bool active = lane < ns;
  const float* rec = recs + (active ? lane : 0) * RS;
  const int kind = __float_as_int(rec[R_KIND]);
  const int base = kind & 15;
  const int mode = (kind >> 8) & 3;
  const long long S = L.n_strokes;
  float v[NV];
#pragma unroll
  for (int j = 0; j < NV; j++) v[j] = 0.f;
  // The next sample's inputs are fetched (read-only path) before this sample's
  // recompute and adjoint, so their latency overlaps the work: without it each
  // iteration's loads wait behind the previous iteration's grad_x atomics.
  struct In {
    float x0, x1, x2, r, ga, a, gs, gc0, gc1, gc2;
  };
  auto fetch = [&](long long q, In& in) {
    in = In{0.f, 0.f, 0.f, 1.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    if (q >= L.n_points) return;
    in.x0 = __ldg(L.x + 3 * q);
    in.x1 = __ldg(L.x + 3 * q + 1);
    in.x2 = __ldg(L.x + 3 * q + 2);
    in.r = __ldg(L.radius + q);
    if (!active) return;
    const long long qi = q * S + s0 + lane;
    in.ga = __ldg(L.g_alpha + qi);
    in.a = __ldg(L.alpha_in + qi);
    if (L.g_sdf) in.gs = __ldg(L.g_sdf + qi);
    if (L.color_const) {
      in.gc0 = __ldg(L.g_color + 3 * qi);
      in.gc1 = __ldg(L.g_color + 3 * qi + 1);
      in.gc2 = __ldg(L.g_color + 3 * qi + 2);
    }
  };
  const long long pstep = (long long)gridDim.x * UF_WARPS;
  long long p = (long long)blockIdx.x * UF_WARPS + warp;
  In cur;
  fetch(p, cur);
  for (; p < L.n_points; p += pstep) {
    In nxt;
    fetch(p + pstep, nxt);
    const V3 x = v3(cur.x0, cur.x1, cur.x2);
    const float rinv = 1.f / cur.r;
    const float ga = cur.ga, a = cur.a, gs = cur.gs;
    if (active && L.color_const) {
      v[G_COLOR] += cur.gc0;
      v[G_COLOR + 1] += cur.gc1;
      v[G_COLOR + 2] += cur.gc2;
    }

    float sdf, f = 1.f;
    V3 pl;
    QuadFwd qf;
    CubicFwd cf;
    if (CLS == UF_PRIM) {
      pl = prim_local(rec, x);
      sdf = prim_sdf(base, pl, rec);
      if (kind & K_S3FAC) f = s3_factor(base, pl, xyz(rec4(rec)[R_S / 4]), rec);
    } else if (CLS == UF_QUAD) {
      sdf = quad_eval(rec, x, qf);
    } else {
      sdf = cubic_eval(rec, x, cf, base == B_CATMULL_ROM);
    }
    const float kk = rec[R_KFIX] * f * rinv;
    const float m = -sdf * kk;
    float dsdf, K;
    if (mode == STEP_HARD) {
      dsdf = gs;
      K = 0.f;
    } else if (compat) {
      // strokes_backward.cu:85-94: dAlpha/dSDF from the saved alpha
      const float dad = mode == STEP_LAPLACE ? (a < 0.5f ? a : 1.0f - a) * -kk
                                             : ((a > 0.f && a < 0.9999f) ? -kk : 0.f);
      dsdf = ga * dad + gs;
      K = 0.f;
    } else {
      const float dm = soft_dm(mode, m, a, ga);
      dsdf = -kk * dm + gs;
      K = m * dm;
    }
    v[G_K] += K;
    V3 gx;
    if (CLS == UF_PRIM) {
      gx = prim_backprop(rec, kind, pl, dsdf, K, v, compat);
    } else if (CLS == UF_QUAD) {
      gx = quad_adjoint(rec, qf, dsdf, v + G_CTRL);
    } else {
      gx = cubic_adjoint(rec, x, cf, dsdf, v + G_CTRL, compat, base == B_CATMULL_ROM);
      if (compat) gx = gx * dsdf;  // the reference multiplies by dL/dSDF again
    }
    if (L.grad_x) {
      const float sx = warp_sum(gx.x), sy = warp_sum(gx.y), sz = warp_sum(gx.z);
      if (lane == 0) {
        atomicAdd(L.grad_x + 3 * p, sx);
        atomicAdd(L.grad_x + 3 * p + 1, sy);
        atomicAdd(L.grad_x + 3 * p + 2, sz);
      }
    }
    cur = nxt;
  }
  if (active) {
    float* dst = L.gslots + (long long)(s0 + lane) * GRAD_SLOTS;
#pragma unroll
    for (int j = 0; j < NV; j++)
      if (v[j] != 0.f) atomicAdd(dst + j, v[j]);
  }
}

// ------------------------------------------------------------------ compose

constexpr int UCB_WARPS = 2;    // compat compose backward (twice the tiles per warp)

template <int C, int W>
struct ComposeTiles {
  float a[W][32][33];
  float c[W][32][32 * C + 1];
};
template <int C, int W>
struct ComposeBwdTiles {
  ComposeTiles<C, W> t;
  float x[W][32][33];          // per-pair alpha grad / T_s tile
  float g[W][32][32 * C + 1];  // per-pair colour grad tile
};

// Load a tile of 32 sample rows x nb strokes starting at stroke s_first, stroke
// order descending (dir = -1) or ascending (dir = +1), into the warp's tiles.
template <int C, int W>
__device__ __forceinline__ void load_tile(ComposeTiles<C, W>& t, int warp, int lane, const UfCompose& L, long long p0,
                                          int rows, int s_first, int nb, int dir, const float* extra,
                                          float (*te)[33]) {
  const long long S = L.n_strokes;
  for (int rr = 0; rr < rows; rr++) {
    const long long row = (p0 + rr) * S;
    if (lane < nb) {
      const long long s = s_first + dir * lane;
      t.a[warp][rr][lane] = L.alphas[row + s];
      if (extra) te[rr][lane] = extra[row + s];
    }
    for (int e = lane; e < nb * C; e += 32) {
      const int j = e / C, ch = e - j * C;
      t.c[warp][rr][j * C + ch] = L.colors[(row + s_first + dir * j) * C + ch];
    }
  }
}

// One warp per sample row [S] (compositing.cu:10-59 restated): lanes take 32
// strokes at a time, top chunk first, lane 0 the topmost stroke of its chunk. The
// transmittance above each stroke is the chunk's incoming T times an exclusive
// shuffle product-scan of (1 - a) over the lanes above; every lane keeps partial
// density / colour sums, reduced over the warp at the end of the row. Loads are
// coalesced row segments, nothing is staged: the kernel streams alphas and colours
// once (16 B per pair for C = 3).
constexpr int UCR_WARPS = 8;  // row kernels: warps per block

__device__ __forceinline__ float excl_prod_up(float v, int lane) {
  // exclusive product over lanes below (lower index); lane 0 gets 1
  for (int o = 1; o < 32; o <<= 1) {
    const float y = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v *= y;
  }
  const float e = __shfl_up_sync(0xffffffffu, v, 1);
  return lane == 0 ? 1.0f : e;
}

template <int C>
__global__ void __launch_bounds__(UCR_WARPS * 32) uf_compose_fwd_rows(const UfCompose L) {
  const int lane = threadIdx.x & 31;
  const long long S = L.n_strokes;
  const int nch = (int)((S + 31) / 32);
  for (long long p = (long long)blockIdx.x * UCR_WARPS + (threadIdx.x >> 5); p < L.n_points;
       p += (long long)gridDim.x * UCR_WARPS) {
    const float* __restrict__ arow = L.alphas + p * S;
    const float* __restrict__ crow = L.colors + p * S * C;
    float T = 1.0f, dens = 0.0f, col[C];
#pragma unroll
    for (int ch = 0; ch < C; ch++) col[ch] = 0.0f;
    for (int k = nch - 1; k >= 0; k--) {
      const long long s = (long long)k * 32 + 31 - lane;  // descending within the chunk
      const bool in = s < S;
      const float a = in ? __ldg(arow + s) : 0.0f;
      const float om = 1.0f - a;
      const float Ts = T * excl_prod_up(om, lane);
      if (in && a != 0.0f) {  // compositing.cu:37
        const float w = a * Ts;
        dens += __ldg(L.density + s) * w;
#pragma unroll
        for (int ch = 0; ch < C; ch++) col[ch] += __ldg(crow + s * C + ch) * w;
      }
      // T below the chunk: the product of every lane's factor
      float all = om;
      for (int o = 16; o > 0; o >>= 1) all *= __shfl_xor_sync(0xffffffffu, all, o);
      T *= all;
    }
    dens = warp_sum(dens);
#pragma unroll
    for (int ch = 0; ch < C; ch++) col[ch] = warp_sum(col[ch]);
    if (lane == 0) {
      const float scale = 1.0f / (1.0f + 1e-6f - T);
      L.density_out[p] = dens;
#pragma unroll
      for (int ch = 0; ch < C; ch++) L.color_out[p * C + ch] = clampf(col[ch] * scale, 0.0f, 1.0f);
    }
  }
}

// compose_forward for 16-byte aligned rows with S % 4 == 0: compositing is an
// associative combination of per-range summaries (T = product of 1 - a, D and C the
// density and colour composited within the range; a range on top combines with the
// one below as T_t T_b, D_t + T_t D_b, C_t + T_t C_b). Lane l takes the contiguous
// strokes [4 g l, 4 g (l + 1)) of a 128 g-stroke round (g float4 groups: all of a row
// up to 1024 strokes in one round), loads them as float4 (alpha, colour, density),
// composites them serially from its top stroke down (alpha 0 skipped, compositing.cu:37),
// then one ordered warp reduction (lane 31 on top) gives the round's summary; rounds
// combine in the same way from the top of the row down.
template <int C, int G>
__global__ void __launch_bounds__(UCR_WARPS * 32) uf_compose_fwd_vec(const UfCompose L) {
  const int lane = threadIdx.x & 31;
  const long long S = L.n_strokes;
  constexpr int RS = 128 * G;  // strokes per round
  const int nr = (int)((S + RS - 1) / RS);
  for (long long p = (long long)blockIdx.x * UCR_WARPS + (threadIdx.x >> 5); p < L.n_points;
       p += (long long)gridDim.x * UCR_WARPS) {
    const float4* __restrict__ arow = reinterpret_cast<const float4*>(L.alphas + p * S);
    const float4* __restrict__ crow = reinterpret_cast<const float4*>(L.colors + p * S * C);
    const float4* __restrict__ drow = reinterpret_cast<const float4*>(L.density);
    float T = 1.0f, dens = 0.0f, col[C];
#pragma unroll
    for (int ch = 0; ch < C; ch++) col[ch] = 0.0f;
    for (int k = nr - 1; k >= 0; k--) {
      // this lane's float4 groups of the round, bottom first: gq .. gq + G - 1
      const long long gq = ((long long)k * 32 + lane) * G;
      float a[4 * G], d[4 * G], c[4 * G * C];
#pragma unroll
      for (int i = 0; i < G; i++) {
        const bool in = (gq + i) * 4 < S;
        const float4 av = in ? __ldg(arow + gq + i) : make_float4(0.f, 0.f, 0.f, 0.f);
        const float4 dv = in ? __ldg(drow + gq + i) : make_float4(0.f, 0.f, 0.f, 0.f);
        a[4 * i] = av.x; a[4 * i + 1] = av.y; a[4 * i + 2] = av.z; a[4 * i + 3] = av.w;
        d[4 * i] = dv.x; d[4 * i + 1] = dv.y; d[4 * i + 2] = dv.z; d[4 * i + 3] = dv.w;
#pragma unroll
        for (int h = 0; h < C; h++) {
          const float4 cv = in ? __ldg(crow + (gq + i) * C + h) : make_float4(0.f, 0.f, 0.f, 0.f);
          c[4 * C * i + 4 * h] = cv.x; c[4 * C * i + 4 * h + 1] = cv.y;
          c[4 * C * i + 4 * h + 2] = cv.z; c[4 * C * i + 4 * h + 3] = cv.w;
        }
      }
      // this lane's range, top stroke first
      float t = 1.0f, dd = 0.0f, cc[C];
#pragma unroll
      for (int ch = 0; ch < C; ch++) cc[ch] = 0.0f;
#pragma unroll
      for (int j = 4 * G - 1; j >= 0; j--) {
        if (a[j] != 0.0f) {  // compositing.cu:37
          const float w = a[j] * t;
          dd += d[j] * w;
#pragma unroll
          for (int ch = 0; ch < C; ch++) cc[ch] += c[j * C + ch] * w;
          t *= 1.0f - a[j];
        }
      }
      // ordered reduction: lane l + o is on top of lane l
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const float tt = __shfl_down_sync(0xffffffffu, t, o);
        const float td = __shfl_down_sync(0xffffffffu, dd, o);
        float tc[C];
#pragma unroll
        for (int ch = 0; ch < C; ch++) tc[ch] = __shfl_down_sync(0xffffffffu, cc[ch], o);
        if (lane + o < 32 && (lane & (2 * o - 1)) == 0) {
          dd = td + tt * dd;
#pragma unroll
          for (int ch = 0; ch < C; ch++) cc[ch] = tc[ch] + tt * cc[ch];
          t = tt * t;
        }
      }
      // the rounds above this one are on top
      dens += T * dd;
#pragma unroll
      for (int ch = 0; ch < C; ch++) col[ch] += T * cc[ch];
      T *= t;
    }
    if (lane == 0) {
      const float scale = 1.0f / (1.0f + 1e-6f - T);
      L.density_out[p] = dens;
#pragma unroll
      for (int ch = 0; ch < C; ch++) L.color_out[p * C + ch] = clampf(col[ch] * scale, 0.0f, 1.0f);
    }
  }
}

// Exact adjoint, one warp per row. Pass 1 (top-down, as the forward) gives the
// totals and stores each chunk's incoming transmittance (one float per 32 strokes).
// Pass 2 (bottom-up) needs, per stroke s, T_s (the chunk's T times a suffix product
// over the lanes above) and U, V, B: density, colour and transmittance composited
// over the strokes below s, i.e. the affine recurrences x <- (1 - a) x + b (b = d a,
// c a, 0) run from the bottom. They come from an inclusive shuffle scan of the lanes'
// affine maps (m = 1 - a, b), shifted by one lane and applied to the carry from the
// chunks below. Then dL/da_s = T_s [g_d (d_s - U) + g_C.(c_s - V) - g_T B] and
// dL/dc_s = g_C a_s T_s, accumulated into the caller's buffers; the density-parameter
// gradient sum_p g_d a_s T_s goes through a per-block shared array (one global atomic
// per stroke and block).
constexpr int UCR_ACC_MAX = 12288;  // strokes with a shared accumulator (48 KB)

template <int C>
__global__ void __launch_bounds__(UCR_WARPS * 32) uf_compose_bwd_rows(const UfCompose L) {
  extern __shared__ float gdp_acc[];
  const int lane = threadIdx.x & 31;
  const long long S = L.n_strokes;
  const int nch = (int)((S + 31) / 32);
  const int nacc = L.g_density_params ? (int)(S < UCR_ACC_MAX ? S : UCR_ACC_MAX) : 0;
  for (int i = threadIdx.x; i < nacc; i += blockDim.x) gdp_acc[i] = 0.0f;
  __syncthreads();
  for (long long p = (long long)blockIdx.x * UCR_WARPS + (threadIdx.x >> 5); p < L.n_points;
       p += (long long)gridDim.x * UCR_WARPS) {
    const float* __restrict__ arow = L.alphas + p * S;
    const float* __restrict__ crow = L.colors + p * S * C;
    float* tin = L.t_scratch + p * nch;
    // pass 1: totals, chunk transmittances
    float T = 1.0f, dens = 0.0f, col[C];
#pragma unroll
    for (int ch = 0; ch < C; ch++) col[ch] = 0.0f;
    for (int k = nch - 1; k >= 0; k--) {
      if (lane == 0) tin[k] = T;
      const long long s = (long long)k * 32 + 31 - lane;
      const bool in = s < S;
      const float a = in ? __ldg(arow + s) : 0.0f;
      const float om = 1.0f - a;
      const float Ts = T * excl_prod_up(om, lane);
      if (in && a != 0.0f) {
        const float w = a * Ts;
        dens += __ldg(L.density + s) * w;
#pragma unroll
        for (int ch = 0; ch < C; ch++) col[ch] += __ldg(crow + s * C + ch) * w;
      }
      float all = om;
      for (int o = 16; o > 0; o >>= 1) all *= __shfl_xor_sync(0xffffffffu, all, o);
      T *= all;
    }
    for (int o = 16; o > 0; o >>= 1) {  // butterfly: every lane gets the totals
      dens += __shfl_xor_sync(0xffffffffu, dens, o);
#pragma unroll
      for (int ch = 0; ch < C; ch++) col[ch] += __shfl_xor_sync(0xffffffffu, col[ch], o);
    }
    __syncwarp();  // pass 1's chunk transmittances are visible to the whole warp
    const float gd = L.g_density ? L.g_density[p] : 0.0f;
    const float scale = 1.0f / (1.0f + 1e-6f - T);
    float gC[C], gT = 0.0f;
#pragma unroll
    for (int ch = 0; ch < C; ch++) {
      const float sc = col[ch] * scale;
      const float gc = (L.g_color && sc >= 0.0f && sc <= 1.0f) ? L.g_color[p * C + ch] : 0.0f;
      gC[ch] = gc * scale;
      gT += gc * col[ch] * scale * scale;
    }
    // pass 2: bottom-up
    float cU = 0.0f, cV[C], cB = 1.0f;
#pragma unroll
    for (int ch = 0; ch < C; ch++) cV[ch] = 0.0f;
    for (int k = 0; k < nch; k++) {
      const long long s = (long long)k * 32 + lane;  // ascending within the chunk
      const bool in = s < S;
      const float a = in ? __ldg(arow + s) : 0.0f;
      const float d = in ? __ldg(L.density + s) : 0.0f;
      float c[C];
#pragma unroll
      for (int ch = 0; ch < C; ch++) c[ch] = in ? __ldg(crow + s * C + ch) : 0.0f;
      const float om = 1.0f - a;
      // T_s: chunk T times the product over the lanes above (higher index)
      float suf = om;
      for (int o = 1; o < 32; o <<= 1) {
        const float y = __shfl_down_sync(0xffffffffu, suf, o);
        if (lane + o < 32) suf *= y;
      }
      float sx = __shfl_down_sync(0xffffffffu, suf, 1);
      if (lane == 31) sx = 1.0f;
      const float Ts = tin[k] * sx;
      // inclusive scan of the affine maps x -> m x + b over the lanes below and this one
      float m = om, bU = d * a, bV[C];
#pragma unroll
      for (int ch = 0; ch < C; ch++) bV[ch] = c[ch] * a;
      for (int o = 1; o < 32; o <<= 1) {
        const float ym = __shfl_up_sync(0xffffffffu, m, o);
        const float yU = __shfl_up_sync(0xffffffffu, bU, o);
        float yV[C];
#pragma unroll
        for (int ch = 0; ch < C; ch++) yV[ch] = __shfl_up_sync(0xffffffffu, bV[ch], o);
        if (lane >= o) {
          bU = fmaf(m, yU, bU);
#pragma unroll
          for (int ch = 0; ch < C; ch++) bV[ch] = fmaf(m, yV[ch], bV[ch]);
          m *= ym;
        }
      }
      // exclusive (the strokes below s) = the previous lane's inclusive map
      float em = __shfl_up_sync(0xffffffffu, m, 1), eU = __shfl_up_sync(0xffffffffu, bU, 1), eV[C];
#pragma unroll
      for (int ch = 0; ch < C; ch++) eV[ch] = __shfl_up_sync(0xffffffffu, bV[ch], 1);
      if (lane == 0) {
        em = 1.0f;
        eU = 0.0f;
#pragma unroll
        for (int ch = 0; ch < C; ch++) eV[ch] = 0.0f;
      }
      const float U = fmaf(em, cU, eU), Bs = em * cB;
      float inner = gd * (d - U) - gT * Bs;
#pragma unroll
      for (int ch = 0; ch < C; ch++) inner += gC[ch] * (c[ch] - fmaf(em, cV[ch], eV[ch]));
      if (in) {
        const float w = a * Ts;
        L.g_alphas[p * S + s] += Ts * inner;
#pragma unroll
        for (int ch = 0; ch < C; ch++) L.g_colors[(p * S + s) * C + ch] += gC[ch] * w;
        if (L.g_density_params) {
          const float g = gd * w;
          if (g != 0.0f) {
            if (s < nacc) atomicAdd(gdp_acc + s, g);
            else atomicAdd(L.g_density_params + s, g);
          }
        }
      }
      // carry: the whole chunk's map (lane 31's inclusive)
      const float am = __shfl_sync(0xffffffffu, m, 31), aU = __shfl_sync(0xffffffffu, bU, 31);
      cU = fmaf(am, cU, aU);
#pragma unroll
      for (int ch = 0; ch < C; ch++) cV[ch] = fmaf(am, cV[ch], __shfl_sync(0xffffffffu, bV[ch], 31));
      cB *= am;
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < nacc; i += blockDim.x)
    if (gdp_acc[i] != 0.0f) atomicAdd(L.g_density_params + i, gdp_acc[i]);
}

// Exact adjoint for 16-byte aligned rows with S % 4 == 0 (the float4 layout of
// uf_compose_fwd_vec: lane l holds the contiguous strokes [4 g l, 4 g (l + 1)) of a
// 128 g-stroke round). Pass 1 (top-down) gives the totals and each round's incoming
// transmittance. Pass 2 (bottom-up), per round: T_s of every stroke from an exclusive
// product scan over the lanes above and the lane's own strokes above s; U, V, B (the
// density, colour and transmittance composited below s) from an exclusive scan of the
// lanes' affine range maps x -> m x + b from the bottom, applied to the carry of the
// rounds below, then stepped through the lane's strokes bottom-up. dL/da_s and
// dL/dc_s accumulate into the caller's rows as float4 read-modify-writes. When a row
// is one round, a lane's strokes are the same in every row it visits, so the
// density-parameter gradient sums in registers until the warp is done.
template <int C, int G>
__global__ void __launch_bounds__(UCR_WARPS * 32) uf_compose_bwd_vec(const UfCompose L) {
  extern __shared__ float gdp_acc[];
  const int lane = threadIdx.x & 31;
  const long long S = L.n_strokes;
  constexpr int RS = 128 * G;
  constexpr int NJ = 4 * G;
  const int nr = (int)((S + RS - 1) / RS);
  const int nacc = L.g_density_params ? (int)(S < UCR_ACC_MAX ? S : UCR_ACC_MAX) : 0;
  for (int i = threadIdx.x; i < nacc; i += blockDim.x) gdp_acc[i] = 0.0f;
  __syncthreads();
  float gdp_reg[NJ];
#pragma unroll
  for (int j = 0; j < NJ; j++) gdp_reg[j] = 0.0f;
  const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
  for (long long p = (long long)blockIdx.x * UCR_WARPS + (threadIdx.x >> 5); p < L.n_points;
       p += (long long)gridDim.x * UCR_WARPS) {
    const float4* __restrict__ arow = reinterpret_cast<const float4*>(L.alphas + p * S);
    const float4* __restrict__ crow = reinterpret_cast<const float4*>(L.colors + p * S * C);
    const float4* __restrict__ drow = reinterpret_cast<const float4*>(L.density);
    float* tin = L.t_scratch + p * nr;
    float a[NJ], d[NJ], c[NJ * C];
    auto load = [&](int k) {
      const long long gq = ((long long)k * 32 + lane) * G;
#pragma unroll
      for (int i = 0; i < G; i++) {
        const bool in = (gq + i) * 4 < S;
        const float4 av = in ? __ldg(arow + gq + i) : z4;
        const float4 dv = in ? __ldg(drow + gq + i) : z4;
        a[4 * i] = av.x; a[4 * i + 1] = av.y; a[4 * i + 2] = av.z; a[4 * i + 3] = av.w;
        d[4 * i] = dv.x; d[4 * i + 1] = dv.y; d[4 * i + 2] = dv.z; d[4 * i + 3] = dv.w;
#pragma unroll
        for (int h = 0; h < C; h++) {
          const float4 cv = in ? __ldg(crow + (gq + i) * C + h) : z4;
          c[4 * C * i + 4 * h] = cv.x; c[4 * C * i + 4 * h + 1] = cv.y;
          c[4 * C * i + 4 * h + 2] = cv.z; c[4 * C * i + 4 * h + 3] = cv.w;
        }
      }
    };
    // pass 1: totals (every lane), each round's incoming transmittance
    float T = 1.0f, dens = 0.0f, col[C];
#pragma unroll
    for (int ch = 0; ch < C; ch++) col[ch] = 0.0f;
    for (int k = nr - 1; k >= 0; k--) {
      if (nr > 1 && lane == 0) tin[k] = T;
      load(k);
      float t = 1.0f, dd = 0.0f, cc[C];
#pragma unroll
      for (int ch = 0; ch < C; ch++) cc[ch] = 0.0f;
#pragma unroll
      for (int j = NJ - 1; j >= 0; j--) {
        if (a[j] != 0.0f) {
          const float w = a[j] * t;
          dd += d[j] * w;
#pragma unroll
          for (int ch = 0; ch < C; ch++) cc[ch] += c[j * C + ch] * w;
          t *= 1.0f - a[j];
        }
      }
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const float tt = __shfl_down_sync(0xffffffffu, t, o);
        const float td = __shfl_down_sync(0xffffffffu, dd, o);
        float tc[C];
#pragma unroll
        for (int ch = 0; ch < C; ch++) tc[ch] = __shfl_down_sync(0xffffffffu, cc[ch], o);
        if (lane + o < 32 && (lane & (2 * o - 1)) == 0) {
          dd = td + tt * dd;
#pragma unroll
          for (int ch = 0; ch < C; ch++) cc[ch] = tc[ch] + tt * cc[ch];
          t = tt * t;
        }
      }
      t = __shfl_sync(0xffffffffu, t, 0);
      dd = __shfl_sync(0xffffffffu, dd, 0);
      dens += T * dd;
#pragma unroll
      for (int ch = 0; ch < C; ch++) col[ch] += T * __shfl_sync(0xffffffffu, cc[ch], 0);
      T *= t;
    }
    if (nr > 1) __syncwarp();  // pass 1's round transmittances are visible to the whole warp
    const float gd = L.g_density ? L.g_density[p] : 0.0f;
    const float scale = 1.0f / (1.0f + 1e-6f - T);
    float gC[C], gT = 0.0f;
#pragma unroll
    for (int ch = 0; ch < C; ch++) {
      const float sc = col[ch] * scale;
      const float gc = (L.g_color && sc >= 0.0f && sc <= 1.0f) ? L.g_color[p * C + ch] : 0.0f;
      gC[ch] = gc * scale;
      gT += gc * col[ch] * scale * scale;
    }
    // pass 2: bottom-up
    float cU = 0.0f, cV[C], cB = 1.0f;
#pragma unroll
    for (int ch = 0; ch < C; ch++) cV[ch] = 0.0f;
    for (int k = 0; k < nr; k++) {
      if (nr > 1) load(k);
      const float Ttop = nr > 1 ? tin[k] : 1.0f;
      // transmittance above this lane's strokes: exclusive product over the lanes above
      float tl = 1.0f;
#pragma unroll
      for (int j = 0; j < NJ; j++) tl *= 1.0f - a[j];
      float suf = tl;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const float y = __shfl_down_sync(0xffffffffu, suf, o);
        if (lane + o < 32) suf *= y;
      }
      float Tx = __shfl_down_sync(0xffffffffu, suf, 1);
      if (lane == 31) Tx = 1.0f;
      float Ts[NJ];
      {
        float tcur = Ttop * Tx;
#pragma unroll
        for (int j = NJ - 1; j >= 0; j--) {
          Ts[j] = tcur;
          tcur *= 1.0f - a[j];
        }
      }
      // this lane's affine range map, bottom-up: x -> m x + b
      float m = 1.0f, bU = 0.0f, bV[C];
#pragma unroll
      for (int ch = 0; ch < C; ch++) bV[ch] = 0.0f;
#pragma unroll
      for (int j = 0; j < NJ; j++) {
        const float om = 1.0f - a[j];
        bU = fmaf(om, bU, d[j] * a[j]);
#pragma unroll
        for (int ch = 0; ch < C; ch++) bV[ch] = fmaf(om, bV[ch], c[j * C + ch] * a[j]);
        m *= om;
      }
      // inclusive scan of the range maps from lane 0 up (a lower lane is below)
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const float ym = __shfl_up_sync(0xffffffffu, m, o);
        const float yU = __shfl_up_sync(0xffffffffu, bU, o);
        float yV[C];
#pragma unroll
        for (int ch = 0; ch < C; ch++) yV[ch] = __shfl_up_sync(0xffffffffu, bV[ch], o);
        if (lane >= o) {
          bU = fmaf(m, yU, bU);
#pragma unroll
          for (int ch = 0; ch < C; ch++) bV[ch] = fmaf(m, yV[ch], bV[ch]);
          m *= ym;
        }
      }
      float em = __shfl_up_sync(0xffffffffu, m, 1), eU = __shfl_up_sync(0xffffffffu, bU, 1), eV[C];
#pragma unroll
      for (int ch = 0; ch < C; ch++) eV[ch] = __shfl_up_sync(0xffffffffu, bV[ch], 1);
      if (lane == 0) {
        em = 1.0f;
        eU = 0.0f;
#pragma unroll
        for (int ch = 0; ch < C; ch++) eV[ch] = 0.0f;
      }
      // composites below this lane's bottom stroke, then through its strokes
      float U = fmaf(em, cU, eU), B = em * cB, V[C];
#pragma unroll
      for (int ch = 0; ch < C; ch++) V[ch] = fmaf(em, cV[ch], eV[ch]);
      float ga[NJ], gcc[NJ * C], gw[NJ];
#pragma unroll
      for (int j = 0; j < NJ; j++) {
        float inner = gd * (d[j] - U) - gT * B;
#pragma unroll
        for (int ch = 0; ch < C; ch++) inner += gC[ch] * (c[j * C + ch] - V[ch]);
        const float w = a[j] * Ts[j];
        ga[j] = Ts[j] * inner;
#pragma unroll
        for (int ch = 0; ch < C; ch++) gcc[j * C + ch] = gC[ch] * w;
        gw[j] = gd * w;
        const float om = 1.0f - a[j];
        U = fmaf(om, U, d[j] * a[j]);
#pragma unroll
        for (int ch = 0; ch < C; ch++) V[ch] = fmaf(om, V[ch], c[j * C + ch] * a[j]);
        B *= om;
      }
      // accumulate into the caller's rows
      const long long gq = ((long long)k * 32 + lane) * G;
      float4* garow = reinterpret_cast<float4*>(L.g_alphas + p * S);
      float4* gcrow = reinterpret_cast<float4*>(L.g_colors + p * S * C);
#pragma unroll
      for (int i = 0; i < G; i++) {
        if ((gq + i) * 4 < S) {
          float4 v = garow[gq + i];
          v.x += ga[4 * i]; v.y += ga[4 * i + 1]; v.z += ga[4 * i + 2]; v.w += ga[4 * i + 3];
          garow[gq + i] = v;
#pragma unroll
          for (int h = 0; h < C; h++) {
            float4 u = gcrow[(gq + i) * C + h];
            u.x += gcc[4 * C * i + 4 * h]; u.y += gcc[4 * C * i + 4 * h + 1];
            u.z += gcc[4 * C * i + 4 * h + 2]; u.w += gcc[4 * C * i + 4 * h + 3];
            gcrow[(gq + i) * C + h] = u;
          }
        }
      }
      if (L.g_density_params) {
        if (nr == 1) {
#pragma unroll
          for (int j = 0; j < NJ; j++) gdp_reg[j] += gw[j];
        } else {
#pragma unroll
          for (int j = 0; j < NJ; j++) {
            const long long s = gq * 4 + j;
            if (s < S && gw[j] != 0.0f) {
              if (s < UCR_ACC_MAX) atomicAdd(gdp_acc + s, gw[j]);
              else atomicAdd(L.g_density_params + s, gw[j]);
            }
          }
        }
      }
      // carry: the whole round's map (lane 31's inclusive scan) applied to the rounds below
      const float m31 = __shfl_sync(0xffffffffu, m, 31);
      cU = fmaf(m31, cU, __shfl_sync(0xffffffffu, bU, 31));
#pragma unroll
      for (int ch = 0; ch < C; ch++) cV[ch] = fmaf(m31, cV[ch], __shfl_sync(0xffffffffu, bV[ch], 31));
      cB *= m31;
    }
  }
  if (L.g_density_params) {
    if (nr == 1) {
#pragma unroll
      for (int j = 0; j < NJ; j++) {
        const long long s = (long long)lane * NJ + j;
        if (s < S && gdp_reg[j] != 0.0f) atomicAdd(gdp_acc + s, gdp_reg[j]);
      }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < nacc; i += blockDim.x)
      if (gdp_acc[i] != 0.0f) atomicAdd(L.g_density_params + i, gdp_acc[i]);
  }
}


template <int C>
__global__ void __launch_bounds__(UCB_WARPS * 32) uf_compose_bwd_kernel(const UfCompose L) {
  extern __shared__ __align__(16) unsigned char dsm[];
  ComposeBwdTiles<C, UCB_WARPS>& bt = *reinterpret_cast<ComposeBwdTiles<C, UCB_WARPS>*>(dsm);
  ComposeTiles<C, UCB_WARPS>& t = bt.t;
  auto& tx = bt.x;
  auto& tg = bt.g;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int S = L.n_strokes;
  const long long SS = S;
  for (long long p0 = ((long long)blockIdx.x * UCB_WARPS + warp) * 32; p0 < L.n_points;
       p0 += (long long)gridDim.x * UCB_WARPS * 32) {
    const int rows = (int)min(32LL, L.n_points - p0);
    const long long p = p0 + lane;
    const bool on = lane < rows;
    // sweep 1 (top-down): totals; exact mode also stores T before each stroke
    float T = 1.0f, dens = 0.0f, col[C];
#pragma unroll
    for (int ch = 0; ch < C; ch++) col[ch] = 0.0f;
    for (int hi = S - 1; hi >= 0; hi -= 32) {
      const int nb = min(32, hi + 1);
      load_tile<C, UCB_WARPS>(t, warp, lane, L, p0, rows, hi, nb, -1, nullptr, nullptr);
      __syncwarp();
      if (on) {
        for (int j = 0; j < nb; j++) {
          const float a = t.a[warp][lane][j];
          tx[warp][lane][j] = T;
          if (a == 0.0f) continue;
          const float w = a * T;
          T *= (1.0f - a);
          dens += L.density[hi - j] * w;
#pragma unroll
          for (int ch = 0; ch < C; ch++) col[ch] += t.c[warp][lane][j * C + ch] * w;
        }
      }
      __syncwarp();
      if (!L.compat) {
        for (int rr = 0; rr < rows; rr++)
          if (lane < nb) L.t_scratch[(p0 + rr) * SS + hi - lane] = tx[warp][rr][lane];
        __syncwarp();
      }
    }
    const float gd = (on && L.g_density) ? L.g_density[p] : 0.0f;
    const float O = 1.0f + 1e-6f - T;
    const float scale = 1.0f / O;
    float gc[C];
#pragma unroll
    for (int ch = 0; ch < C; ch++) {
      const float sc = col[ch] * scale;
      gc[ch] = (on && L.g_color && sc >= 0.0f && sc <= 1.0f) ? L.g_color[p * C + ch] : 0.0f;
    }
    if (L.compat) {
      // compositing.cu:116-156, top-down
      float T2 = 1.0f, d2 = 0.0f, c2[C];
#pragma unroll
      for (int ch = 0; ch < C; ch++) c2[ch] = 0.0f;
      for (int hi = S - 1; hi >= 0; hi -= 32) {
        const int nb = min(32, hi + 1);
        load_tile<C, UCB_WARPS>(t, warp, lane, L, p0, rows, hi, nb, -1, nullptr, nullptr);
        __syncwarp();
        for (int j = 0; j < nb; j++) {
          const float a = t.a[warp][lane][j];
          const float ds = L.density[hi - j];
          float w = 0.0f;
          if (a > 0.0f) {
            w = a * T2;
            T2 *= (1.0f - a);
            d2 += ds * w;
#pragma unroll
            for (int ch = 0; ch < C; ch++) c2[ch] += t.c[warp][lane][j * C + ch] * w;
          }
          float sd = 1.0f / fmaxf(1.0f - a, 1e-6f);
          float ga = gd * (T2 * ds - (dens - d2)) * sd;
          sd *= scale * scale;
#pragma unroll
          for (int ch = 0; ch < C; ch++) {
            ga += gc[ch] * (T2 * t.c[warp][lane][j * C + ch] * (O - a) - (col[ch] - c2[ch])) * sd;
            tg[warp][lane][j * C + ch] = on ? gc[ch] * scale * w : 0.0f;
          }
          tx[warp][lane][j] = on ? ga : 0.0f;
          t.a[warp][lane][j] = on ? gd * w : 0.0f;  // reuse: density-param contribution
        }
        __syncwarp();
        for (int rr = 0; rr < rows; rr++) {
          const long long row = (p0 + rr) * SS;
          if (lane < nb) L.g_alphas[row + hi - lane] += tx[warp][rr][lane];
          for (int e = lane; e < nb * C; e += 32) {
            const int j = e / C, ch = e - j * C;
            L.g_colors[(row + hi - j) * C + ch] += tg[warp][rr][j * C + ch];
          }
        }
        if (lane < nb) {
          float sum = 0.0f;
          for (int rr = 0; rr < rows; rr++) sum += t.a[warp][rr][lane];
          if (sum != 0.0f) atomicAdd(L.g_density_params + hi - lane, sum);
        }
        __syncwarp();
      }
    } else {
      // exact: dL/da_s = T_s [g_d (d_s - U) + g_C.(c_s - V) - g_T B], U/V/B composited
      // bottom-up over the strokes below s
      float gC[C], gT = 0.0f;
#pragma unroll
      for (int ch = 0; ch < C; ch++) {
        gC[ch] = gc[ch] * scale;
        gT += gc[ch] * col[ch] * scale * scale;
      }
      float U = 0.0f, V[C], B = 1.0f;
#pragma unroll
      for (int ch = 0; ch < C; ch++) V[ch] = 0.0f;
      for (int lo = 0; lo < S; lo += 32) {
        const int nb = min(32, S - lo);
        load_tile<C, UCB_WARPS>(t, warp, lane, L, p0, rows, lo, nb, +1, L.t_scratch, tx[warp]);
        __syncwarp();
        for (int j = 0; j < nb; j++) {
          const float a = t.a[warp][lane][j];
          const float Ts = tx[warp][lane][j];
          const float ds = L.density[lo + j];
          const float w = a * Ts;
          float inner = gd * (ds - U) - gT * B;
#pragma unroll
          for (int ch = 0; ch < C; ch++) {
            const float cs = t.c[warp][lane][j * C + ch];
            inner += gC[ch] * (cs - V[ch]);
            tg[warp][lane][j * C + ch] = on ? gC[ch] * w : 0.0f;
            V[ch] = cs * a + (1.0f - a) * V[ch];
          }
          U = ds * a + (1.0f - a) * U;
          B *= (1.0f - a);
          tx[warp][lane][j] = on ? Ts * inner : 0.0f;
          t.a[warp][lane][j] = on ? gd * w : 0.0f;
        }
        __syncwarp();
        for (int rr = 0; rr < rows; rr++) {
          const long long row = (p0 + rr) * SS;
          if (lane < nb) L.g_alphas[row + lo + lane] += tx[warp][rr][lane];
          for (int e = lane; e < nb * C; e += 32) {
            const int j = e / C, ch = e - j * C;
            L.g_colors[(row + lo + j) * C + ch] += tg[warp][rr][j * C + ch];
          }
        }
        if (lane < nb) {
          float sum = 0.0f;
          for (int rr = 0; rr < rows; rr++) sum += t.a[warp][rr][lane];
          if (sum != 0.0f) atomicAdd(L.g_density_params + lo + lane, sum);
        }
        __syncwarp();
      }
    }
  }
}

static int grid_for(long long items, int per_block) {
  long long g = (items + per_block - 1) / per_block;
  if (g > 148LL * 16) g = 148LL * 16;
  if (g < 1) g = 1;
  return (int)g;
}

cudaError_t launch_uf_stroke_fwd(const UfStroke& L, int base, cudaStream_t st) {
  // persistent: about six resident blocks per SM in total (25 KB of shared memory
  // each, 42 KB with the sdf tile), spread over the stroke blocks; each warp then sweeps
  // several point tiles
  const int sblocks = (L.n_strokes + 31) / 32;
  long long gx = (148LL * 6 + sblocks - 1) / sblocks;
  const long long tiles = (L.n_points + UF_WARPS * 32 - 1) / (UF_WARPS * 32);
  if (gx > tiles) gx = tiles;
  if (gx < 1) gx = 1;
  dim3 grid((unsigned)gx, sblocks);
  const size_t dyn = L.sdf ? sizeof(float) * UF_WARPS * 32 * 33 : 0;
  if (base <= B_TETRAHEDRON)
    uf_stroke_fwd_kernel<UF_PRIM><<<grid, UF_WARPS * 32, dyn, st>>>(L);
  else if (base == B_QUAD_BEZIER)
    uf_stroke_fwd_kernel<UF_QUAD><<<grid, UF_WARPS * 32, dyn, st>>>(L);
  else
    uf_stroke_fwd_kernel<UF_CUBIC><<<grid, UF_WARPS * 32, dyn, st>>>(L);
  return cudaGetLastError();
}

cudaError_t launch_uf_stroke_bwd(const UfStroke& L, int base, cudaStream_t st) {
  const int cls = base_is_cubic_curve(base) ? UF_CUBIC : (base == B_QUAD_BEZIER ? UF_QUAD : UF_PRIM);
  auto* k = cls == UF_PRIM ? (L.compat ? uf_stroke_bwd_kernel<UF_PRIM, 1> : uf_stroke_bwd_kernel<UF_PRIM, 0>)
            : cls == UF_QUAD ? (L.compat ? uf_stroke_bwd_kernel<UF_QUAD, 1> : uf_stroke_bwd_kernel<UF_QUAD, 0>)
                             : (L.compat ? uf_stroke_bwd_kernel<UF_CUBIC, 1> : uf_stroke_bwd_kernel<UF_CUBIC, 0>);
  // one wave of sample-parallel blocks (registers decide how many fit)
  const int sblocks = (L.n_strokes + 31) / 32;
  long long want = 1;
  cudaError_t e = one_wave_blocks(k, UF_WARPS * 32, sblocks, (L.n_points + UF_WARPS - 1) / UF_WARPS, &want);
  if (e != cudaSuccess) return e;
  dim3 grid((unsigned)want, sblocks);
  k<<<grid, UF_WARPS * 32, 0, st>>>(L);
  return cudaGetLastError();
}

template <typename K>
static cudaError_t launch_dyn(K kernel, int grid, int threads, size_t smem, const UfCompose& L, cudaStream_t st) {
  cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  kernel<<<grid, threads, smem, st>>>(L);
  return cudaGetLastError();
}

cudaError_t launch_uf_compose_fwd(const UfCompose& L, cudaStream_t st) {
  const int grid = grid_for(L.n_points, UCR_WARPS);  // one row per warp
  const bool vec = (L.n_strokes & 3) == 0 && (reinterpret_cast<uintptr_t>(L.alphas) & 15) == 0 &&
                   (reinterpret_cast<uintptr_t>(L.colors) & 15) == 0 &&
                   (reinterpret_cast<uintptr_t>(L.density) & 15) == 0;
  if (vec) {
    // float4 groups per lane: enough for a whole row in one round up to 512 strokes
    const int g = L.n_strokes <= 128 ? 1 : (L.n_strokes <= 256 ? 2 : 4);
    if (L.color_dim == 1) {
      if (g == 1) uf_compose_fwd_vec<1, 1><<<grid, UCR_WARPS * 32, 0, st>>>(L);
      else if (g == 2) uf_compose_fwd_vec<1, 2><<<grid, UCR_WARPS * 32, 0, st>>>(L);
      else uf_compose_fwd_vec<1, 4><<<grid, UCR_WARPS * 32, 0, st>>>(L);
    } else {
      if (g == 1) uf_compose_fwd_vec<3, 1><<<grid, UCR_WARPS * 32, 0, st>>>(L);
      else if (g == 2) uf_compose_fwd_vec<3, 2><<<grid, UCR_WARPS * 32, 0, st>>>(L);
      else uf_compose_fwd_vec<3, 4><<<grid, UCR_WARPS * 32, 0, st>>>(L);
    }
    return cudaGetLastError();
  }
  if (L.color_dim == 1)
    uf_compose_fwd_rows<1><<<grid, UCR_WARPS * 32, 0, st>>>(L);
  else
    uf_compose_fwd_rows<3><<<grid, UCR_WARPS * 32, 0, st>>>(L);
  return cudaGetLastError();
}

cudaError_t launch_uf_compose_bwd(const UfCompose& L, cudaStream_t st) {
  const bool vec = !L.compat && (L.n_strokes & 3) == 0 && L.n_strokes <= UCR_ACC_MAX &&
                   (reinterpret_cast<uintptr_t>(L.alphas) & 15) == 0 &&
                   (reinterpret_cast<uintptr_t>(L.colors) & 15) == 0 &&
                   (reinterpret_cast<uintptr_t>(L.density) & 15) == 0 &&
                   (reinterpret_cast<uintptr_t>(L.g_alphas) & 15) == 0 &&
                   (reinterpret_cast<uintptr_t>(L.g_colors) & 15) == 0;
  if (vec) {
    // a few blocks per SM: every warp visits many rows (fewer density-parameter flushes)
    int grid = grid_for(L.n_points, UCR_WARPS);
    if (grid > 148 * 4) grid = 148 * 4;
    const size_t smem = L.g_density_params ? size_t(L.n_strokes) * 4 : 0;
    // one or two float4 groups per lane (rows beyond 256 strokes take several rounds:
    // wider lanes would hold ~190 floats of row state and spill)
    const bool g1 = L.n_strokes <= 128;
#define N3DS_CBV(CC, GG) launch_dyn(uf_compose_bwd_vec<CC, GG>, grid, UCR_WARPS * 32, smem, L, st)
    if (L.color_dim == 1) return g1 ? N3DS_CBV(1, 1) : N3DS_CBV(1, 2);
    return g1 ? N3DS_CBV(3, 1) : N3DS_CBV(3, 2);
#undef N3DS_CBV
  }
  if (!L.compat) {  // exact adjoint: one row per warp
    const int grid = grid_for(L.n_points, UCR_WARPS);
    const size_t smem = L.g_density_params ? size_t(std::min<long long>(L.n_strokes, UCR_ACC_MAX)) * 4 : 0;
    if (L.color_dim == 1)
      uf_compose_bwd_rows<1><<<grid, UCR_WARPS * 32, smem, st>>>(L);
    else
      uf_compose_bwd_rows<3><<<grid, UCR_WARPS * 32, smem, st>>>(L);
    return cudaGetLastError();
  }
  // the reference's formulas (compat): 32-row tiles in shared memory
  const int grid = grid_for(L.n_points, UCB_WARPS * 32);
  if (L.color_dim == 1)
    return launch_dyn(uf_compose_bwd_kernel<1>, grid, UCB_WARPS * 32, sizeof(ComposeBwdTiles<1, UCB_WARPS>), L, st);
  return launch_dyn(uf_compose_bwd_kernel<3>, grid, UCB_WARPS * 32, sizeof(ComposeBwdTiles<3, UCB_WARPS>), L, st);
}

}  // namespace n3ds
