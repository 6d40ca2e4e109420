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

__global__ void __launch_bounds__(UF_WARPS * 32) uf_stroke_fwd_kernel(const UfStroke L) {
  __shared__ __align__(16) float recs[32 * REC_FLOATS];
  __shared__ float ta[UF_WARPS][32][33];
  __shared__ float tsd[UF_WARPS][32][33];
  const int s0 = blockIdx.y * 32;
  const int ns = min(32, L.n_strokes - s0);
  for (int i = threadIdx.x; i < ns * REC_FLOATS; i += blockDim.x) recs[i] = L.recs[(long long)s0 * REC_FLOATS + i];
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long long S = L.n_strokes;
  for (long long p0 = ((long long)blockIdx.x * UF_WARPS + warp) * 32; p0 < L.n_points;
       p0 += (long long)gridDim.x * UF_WARPS * 32) {
    const long long p = p0 + lane;
    const long long pp = p < L.n_points ? p : p0;
    const V3 x = v3(L.x[3 * pp], L.x[3 * pp + 1], L.x[3 * pp + 2]);
    const float rinv = 1.f / L.radius[pp];
    for (int j = 0; j < ns; j++) {
      float sdf;
      ta[warp][lane][j] = pair_alpha(recs + j * REC_FLOATS, x, rinv, &sdf);
      tsd[warp][lane][j] = sdf;
    }
    __syncwarp();
    const int rows = (int)min(32LL, L.n_points - p0);
    for (int rr = 0; rr < rows; rr++) {
      const long long row = (p0 + rr) * S + s0;
      if (lane < ns) {
        L.alpha[row + lane] = ta[warp][rr][lane];
        if (L.sdf) L.sdf[row + lane] = tsd[warp][rr][lane];
      }
      if (L.color_const)
        for (int e = lane; e < 3 * ns; e += 32) L.color[row * 3 + e] = recs[(e / 3) * REC_FLOATS + R_COLOR + e % 3];
    }
    __syncwarp();
  }
}

template <int NV>
__global__ void __launch_bounds__(UF_WARPS * 32) uf_stroke_bwd_kernel(const UfStroke L) {
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
    if (base <= B_TETRAHEDRON) {
      pl = prim_local(rec, x);
      sdf = prim_sdf(base, pl, rec);
      if (kind & K_S3FAC) f = s3_factor(base, pl, xyz(rec4(rec)[R_S / 4]), rec);
    } else if (base == B_QUAD_BEZIER) {
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
    } else if (L.compat) {
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
    if (base <= B_TETRAHEDRON) {
      gx = prim_backprop(rec, kind, pl, dsdf, K, v, L.compat);
    } else if (base == B_QUAD_BEZIER) {
      gx = quad_adjoint(rec, qf, dsdf, v + G_CTRL);
    } else {
      gx = cubic_adjoint(rec, x, cf, dsdf, v + G_CTRL, L.compat, base == B_CATMULL_ROM);
      if (L.compat) gx = gx * dsdf;  // the reference multiplies by dL/dSDF again
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
  (void)base;
  dim3 grid(grid_for(L.n_points, UF_WARPS * 32), (L.n_strokes + 31) / 32);
  uf_stroke_fwd_kernel<<<grid, UF_WARPS * 32, 0, st>>>(L);
  return cudaGetLastError();
}

cudaError_t launch_uf_stroke_bwd(const UfStroke& L, int base, cudaStream_t st) {
  // enough sample-parallel blocks per stroke block to fill the machine
  const int sblocks = (L.n_strokes + 31) / 32;
  long long want = (148LL * 8 + sblocks - 1) / sblocks;
  long long cap = (L.n_points + UF_WARPS - 1) / UF_WARPS;
  if (want > cap) want = cap;
  if (want < 1) want = 1;
  dim3 grid((unsigned)want, sblocks);
  if (base_is_cubic_curve(base))
    uf_stroke_bwd_kernel<32><<<grid, UF_WARPS * 32, 0, st>>>(L);
  else
    uf_stroke_bwd_kernel<16><<<grid, UF_WARPS * 32, 0, st>>>(L);
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
  if (L.color_dim == 1)
    uf_compose_fwd_rows<1><<<grid, UCR_WARPS * 32, 0, st>>>(L);
  else
    uf_compose_fwd_rows<3><<<grid, UCR_WARPS * 32, 0, st>>>(L);
  return cudaGetLastError();
}

cudaError_t launch_uf_compose_bwd(const UfCompose& L, cudaStream_t st) {
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
