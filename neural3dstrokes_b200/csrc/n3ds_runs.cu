// Sample-run kernels of the fused stroke field: the same forward and exact adjoint as
// the segment kernels (n3ds_field.cu), with the (sample, stroke) pairs packed densely
// into warps.
//
// A warp owns one work unit: up to 64 consecutive samples of one ray (two per lane).
// For each 32-stroke block of the staged chunk, lane j takes stroke (top - j) and
// intersects its culling sphere (radius R_b + c_m r_max, grown by the samples' largest
// distance rho from the unit's chord) with the chord: the samples within reach form
// one contiguous RUN of sample indices, found by binary search of the samples' chord
// parameters (monotone along a ray; a unit whose samples are not monotone takes every
// sample). Only samples inside the run can have alpha above the cut, so only those
// pairs are evaluated: about a third of what 32-sample segments evaluate.
//
// Runs are collected in compositing order (descending stroke index) into a per-warp
// list of up to 32 runs / 256 pairs. The list is then processed in phases:
//   table    pairs are laid out grouped by primitive type (so a batch of 32 pairs
//            mostly runs one SDF branch), one table entry (run, sample) per pair;
//   evaluate lane = pair: transform, SDF, soft step -> alpha, in batches of 32;
//   compose  lane = sample: runs in stroke order, over-compositing from the alphas.
// The backward recomputes alpha the same way, runs the composite adjoint per sample in
// stroke order (storing dL/dm per pair and reducing colour / density gradients per
// run), then per pair evaluates the SDF and transform adjoint and reduces the
// per-stroke gradient slots across the lanes of each run with a segmented shuffle
// scan (runs are contiguous lanes), one shared atomic per slot and run.
#include "n3ds_stage.cuh"

namespace n3ds {

constexpr int RUN_UNIT = 64;   // samples per work unit (two per lane)
constexpr int RUN_CAP = 32;    // runs per list (one per lane when laying out pairs)
constexpr int PAIR_CAP = 256;  // pairs per list

// Per-warp scratch in shared memory.
struct RunBuf {
  float u[RUN_UNIT];     // chord parameter of each sample of the unit
  int run_sk[RUN_CAP];   // stroke slot | base type << 16
  int run_in[RUN_CAP];   // first sample | sample count << 8
  int table[PAIR_CAP];   // run << 8 | sample, pairs grouped by base type
  float val[PAIR_CAP];   // alpha per pair; dL/dm after the backward's compose phase
};

struct RunStage {
  Stage s;
  unsigned char* base;   // [cap] base SDF type of each staged stroke
  RunBuf* bufs;          // [warps]
  float* gxb;            // [warps][3 * RUN_UNIT] backward: dL/dx of the unit's samples
};

__host__ __device__ constexpr size_t run_smem_bytes(int cap, int warps, bool backward) {
  return align16(size_t(cap) * 16) + align16(size_t(cap) * 4) + size_t(cap) * REC_FLOATS * 4 +
         (backward ? size_t(cap) * GRAD_SLOTS * 4 : 0) + align16(size_t(cap)) + size_t(warps) * sizeof(RunBuf) +
         (backward ? size_t(warps) * 3 * RUN_UNIT * 4 : 0);
}

size_t run_fwd_smem(int cap, int warps) { return run_smem_bytes(cap, warps, false); }
size_t run_bwd_smem(int cap, int warps) { return run_smem_bytes(cap, warps, true); }

__device__ __forceinline__ RunStage run_carve(unsigned char* smem, int cap, int warps, bool backward) {
  RunStage r;
  r.s = carve(smem, cap, backward);
  unsigned char* p = smem + align16(size_t(cap) * 16) + align16(size_t(cap) * 4) + size_t(cap) * REC_FLOATS * 4 +
                     (backward ? size_t(cap) * GRAD_SLOTS * 4 : 0);
  r.base = p;
  p += align16(size_t(cap));
  r.bufs = reinterpret_cast<RunBuf*>(p);
  p += size_t(warps) * sizeof(RunBuf);
  r.gxb = backward ? reinterpret_cast<float*>(p) : nullptr;
  return r;
}

// Base type of every staged record, for grouping pairs by SDF branch.
__device__ __forceinline__ void stage_bases(const RunStage& R, int n) {
  for (int i = threadIdx.x; i < n; i += blockDim.x)
    R.base[i] = (unsigned char)(__float_as_int(R.s.recs[size_t(i) * REC_FLOATS + R_KIND]) & 15);
  __syncthreads();
}

// Geometry of one work unit; lane holds samples lane and lane + 32.
struct Unit {
  long long si0;  // first sample (global)
  int cnt;        // samples in the unit
  V3 x[2];
  float r[2];
  V3 A, AB;       // chord from the first to the last sample
  float invL2;
  float rho;      // largest distance of a sample from the chord line
  float rmax;     // largest |radius|
  bool mono;      // chord parameters non-decreasing along the unit
};

__device__ __forceinline__ void unit_setup(const SegLaunch& L, long long si0, int cnt, int lane, RunBuf& B,
                                           Unit& U) {
  U.si0 = si0;
  U.cnt = cnt;
#pragma unroll
  for (int b = 0; b < 2; b++) {
    const int j = lane + 32 * b;
    const long long si = si0 + (j < cnt ? j : 0);
    const long long ray = si / L.n_samples;
    load_sample(L, ray, (int)(si - ray * L.n_samples), si, U.x[b], U.r[b]);
  }
  U.A = shfl3(U.x[0], 0);
  const V3 last = cnt <= 32 ? shfl3(U.x[0], cnt - 1) : shfl3(U.x[1], cnt - 33);
  U.AB = last - U.A;
  const float l2 = dot(U.AB, U.AB);
  U.invL2 = l2 > 0.f ? 1.f / l2 : 0.f;
  float u[2], dev = 0.f, rm = 0.f;
#pragma unroll
  for (int b = 0; b < 2; b++) {
    const int j = lane + 32 * b;
    const V3 w = U.x[b] - U.A;
    u[b] = dot(w, U.AB) * U.invL2;
    const V3 q = w - U.AB * u[b];
    if (j < cnt) {
      dev = fmaxf(dev, sqrtf(dot(q, q)));
      rm = fmaxf(rm, fabsf(U.r[b]));
      B.u[j] = u[b];
    }
  }
  U.rho = warp_max(dev);
  U.rmax = warp_max(rm);
  // monotone: u_j <= u_{j+1} for every consecutive pair (NaN fails)
  const float n0 = __shfl_down_sync(0xffffffffu, u[0], 1);
  const float n1 = __shfl_down_sync(0xffffffffu, u[1], 1);
  const float h1 = __shfl_sync(0xffffffffu, u[1], 0);
  const float next0 = lane < 31 ? n0 : h1;
  const bool ok0 = !(lane + 1 < cnt) || (u[0] <= next0);
  const bool ok1 = !(lane + 33 < cnt) || (u[1] <= n1);
  U.mono = __all_sync(0xffffffffu, ok0 && ok1);
  __syncwarp();
}

// First index j in [0, n) with u[j] >= v (n if none).
__device__ __forceinline__ int lower_bound_u(const float* u, int n, float v) {
  int lo = 0, len = n;
  while (len > 0) {
    const int half = len >> 1;
    if (u[lo + half] < v) {
      lo += half + 1;
      len -= half + 1;
    } else {
      len = half;
    }
  }
  return lo;
}
// First index j in [0, n) with u[j] > v (n if none).
__device__ __forceinline__ int upper_bound_u(const float* u, int n, float v) {
  int lo = 0, len = n;
  while (len > 0) {
    const int half = len >> 1;
    if (!(v < u[lo + half])) {
      lo += half + 1;
      len -= half + 1;
    } else {
      len = half;
    }
  }
  return lo;
}

// Run of stroke sl (staged slot) for this unit: first sample and count (0: culled).
__device__ __forceinline__ int stroke_run(const RunStage& R, const Unit& U, const RunBuf& B, int sl, int* i0) {
  const float4 ca = R.s.cull_a[sl];
  const float Rr = ca.w + fabsf(R.s.cull_b[sl]) * U.rmax + U.rho;
  const V3 w = v3(ca.x, ca.y, ca.z) - U.A;
  const float uc = dot(w, U.AB) * U.invL2;
  const V3 q = w - U.AB * uc;
  const float perp2 = dot(q, q);
  if (perp2 > Rr * Rr) return 0;  // NaN compares false: such strokes stay candidates
  int lo = 0, hi = U.cnt - 1;
  if (U.mono) {
    // chord parameters within reach; the small widening absorbs rounding
    const float h = sqrtf(fmaxf(Rr * Rr - perp2, 0.f) * U.invL2) + 1e-5f;
    const float u0 = uc - h, u1 = uc + h;
    if (isfinite(u0) && isfinite(u1)) {
      lo = lower_bound_u(B.u, U.cnt, u0);
      hi = upper_bound_u(B.u, U.cnt, u1) - 1;
    }
  }
  *i0 = lo;
  return hi >= lo ? hi - lo + 1 : 0;
}

// Lay out the list's pairs grouped by base type: returns this lane's run (lane < nruns)
// first pair index; writes the pair table. kcount (lane k) counts pairs of base k.
__device__ __forceinline__ int layout_pairs(RunBuf& B, int nruns, int lane, int* sk_out, int* in_out,
                                            unsigned long long* kcount) {
  const bool own = lane < nruns;
  const int sk = own ? B.run_sk[lane] : 0;
  const int in = own ? B.run_in[lane] : 0;
  const int kind = sk >> 16;
  const int n = in >> 8;
  unsigned present = __reduce_or_sync(0xffffffffu, own ? 1u << kind : 0u);
  int base = 0, start = 0;
  while (present) {
    const int k = __ffs(present) - 1;
    present &= present - 1;
    const int v = (own && kind == k) ? n : 0;
    int incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    if (own && kind == k) base = start + incl - v;
    const int tot = __shfl_sync(0xffffffffu, incl, 31);
    if (kcount && lane == k) *kcount += (unsigned long long)tot;
    start += tot;
  }
  for (int r = 0; r < nruns; r++) {
    const int rin = __shfl_sync(0xffffffffu, in, r);
    const int rb = __shfl_sync(0xffffffffu, base, r);
    const int i0 = rin & 255, cnt = rin >> 8;
    for (int j = lane; j < cnt; j += 32) B.table[rb + j] = (r << 8) | (i0 + j);
  }
  __syncwarp();
  *sk_out = sk;
  *in_out = in;
  return base;
}

// Alpha of every pair of the list into B.val.
__device__ __forceinline__ void eval_pairs(const SegLaunch& L, const RunStage& R, RunBuf& B, const Unit& U,
                                           int npairs, int lane) {
  for (int p0 = 0; p0 < npairs; p0 += 32) {
    const int p = p0 + lane;
    if (p < npairs) {
      const int e = B.table[p];
      const int slot = B.run_sk[e >> 8] & 0xffff;
      const long long si = U.si0 + (e & 255);
      const long long ray = si / L.n_samples;
      V3 x;
      float rr;
      load_sample(L, ray, (int)(si - ray * L.n_samples), si, x, rr);
      B.val[p] = pair_alpha(R.s.recs + size_t(slot) * REC_FLOATS, x, 1.f / rr);
    }
  }
  __syncwarp();
}

// Collect the runs of one 32-stroke block into the list, processing the list with
// `flush` whenever it would overflow.
template <typename Flush>
__device__ __forceinline__ void add_block_runs(const RunStage& R, const Unit& U, RunBuf& B, int hi, int lane,
                                               int& nruns, int& npairs, Flush&& flush) {
  const int sl = hi - lane;
  int i0 = 0, n = 0;
  if (sl >= 0) n = stroke_run(R, U, B, sl, &i0);
  unsigned mask = __ballot_sync(0xffffffffu, n > 0);
  const unsigned lt = (1u << lane) - 1u;
  while (mask) {
    const bool mine = (mask >> lane) & 1u;
    int incl = mine ? n : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    const int rank = __popc(mask & lt);
    const bool fits = mine && (nruns + rank < RUN_CAP) && (npairs + incl <= PAIR_CAP);
    const unsigned take = __ballot_sync(0xffffffffu, fits);
    if (take) {
      if (fits) {
        B.run_sk[nruns + rank] = sl | (int(R.base[sl]) << 16);
        B.run_in[nruns + rank] = i0 | (n << 8);
      }
      const int last = 31 - __clz(take);
      nruns += __popc(take);
      npairs += __shfl_sync(0xffffffffu, incl, last);
      mask &= ~take;
      __syncwarp();
    }
    if (mask) {
      flush();
      nruns = 0;
      npairs = 0;
    }
  }
}

// ================================================================== forward

template <int WARPS>
__global__ void __launch_bounds__(WARPS * 32, 1) run_fwd_kernel(const __grid_constant__ SegLaunch L) {
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ uint64_t bar;
  __shared__ int s_scene, s_fail;
  const RunStage R = run_carve(smem, L.chunk_cap, WARPS, false);
  const int lane = threadIdx.x & 31;
  RunBuf& B = R.bufs[threadIdx.x >> 5];
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    s_fail = 0;
  }
  unsigned long long kcount = 0;  // lane k: evaluated pairs of base k
  uint32_t phase = 0;
  const int upr = (L.n_samples + RUN_UNIT - 1) / RUN_UNIT;
  int sci = home_scene(L);
  while (sci >= 0) {
    if (!stage_chunk(L, L.sc[sci], R.s, &bar, phase, &s_fail)) {
      if (threadIdx.x == 0) atomicOr(L.status, ST_WAIT_TIMEOUT);
      return;
    }
    stage_bases(R, L.sc[sci].chunk_n);
    const SceneDesc& sc = L.sc[sci];
    int* counter = L.tile_counter + sci;
    const int n_units = sc.n_rays * upr;
    int item = 0;
    if (lane == 0) item = atomicAdd(counter, 1);
    item = __shfl_sync(0xffffffffu, item, 0);
    while (item < n_units) {
      const int ray_local = item / upr;
      const int j0 = (item - ray_local * upr) * RUN_UNIT;
      const int cnt = min(RUN_UNIT, L.n_samples - j0);
      Unit U;
      unit_setup(L, (sc.ray_begin + ray_local) * L.n_samples + j0, cnt, lane, B, U);
      float T[2], sig[2], cr[2], cg[2], cb[2];
#pragma unroll
      for (int b = 0; b < 2; b++) {
        const int j = lane + 32 * b;
        if (sc.first_pass || j >= cnt) {
          T[b] = 1.f; sig[b] = cr[b] = cg[b] = cb[b] = 0.f;
        } else {
          const float* st = L.state + 5 * (U.si0 + j);
          T[b] = st[0]; sig[b] = st[1]; cr[b] = st[2]; cg[b] = st[3]; cb[b] = st[4];
        }
      }
      int nruns = 0, npairs = 0;
      auto flush = [&]() {
        int sk, in;
        const int base = layout_pairs(B, nruns, lane, &sk, &in, &kcount);
        eval_pairs(L, R, B, U, npairs, lane);
        for (int r = 0; r < nruns; r++) {
          const int rin = __shfl_sync(0xffffffffu, in, r);
          const int rb = __shfl_sync(0xffffffffu, base, r);
          const int slot = __shfl_sync(0xffffffffu, sk, r) & 0xffff;
          const int i0 = rin & 255, n = rin >> 8;
          const float* rec = R.s.recs + size_t(slot) * REC_FLOATS;
          const float d = rec[R_DENSITY];
          const float4 col = rec4(rec)[R_COLOR / 4];
#pragma unroll
          for (int b = 0; b < 2; b++) {
            const unsigned o = unsigned(lane + 32 * b - i0);
            if (o < unsigned(n)) {
              const float a = B.val[rb + o];
              const float w = a * T[b];
              T[b] *= (1.0f - a);
              sig[b] += d * w;
              cr[b] += col.x * w;
              cg[b] += col.y * w;
              cb[b] += col.z * w;
            }
          }
        }
        __syncwarp();
      };
      for (int hi = sc.chunk_n - 1; hi >= 0; hi -= 32) add_block_runs(R, U, B, hi, lane, nruns, npairs, flush);
      if (nruns) flush();
#pragma unroll
      for (int b = 0; b < 2; b++) {
        const int j = lane + 32 * b;
        if (j < cnt) {
          float* st = L.state + 5 * (U.si0 + j);
          st[0] = T[b]; st[1] = sig[b]; st[2] = cr[b]; st[3] = cg[b]; st[4] = cb[b];
        }
      }
      if (lane == 0) item = atomicAdd(counter, 1);
      item = __shfl_sync(0xffffffffu, item, 0);
    }
    __syncthreads();  // every warp is done with the staged chunk
    if (threadIdx.x == 0) s_scene = next_scene(L);
    __syncthreads();
    sci = s_scene;
  }
  if (L.stats && lane < 16 && kcount) {
    atomicAdd(L.stats, kcount);
    atomicAdd(L.stats + 1 + lane, kcount);
  }
}

// ================================================================= backward

// Running composite adjoint of one sample (see compose_step in n3ds_field.cu).
struct SampleAdj {
  float T, Ps, Pr, Pg, Pb;      // running, through the previous stroke
  float gs, gcr, gcg, gcb, gT;  // seeds
  float sig, Cr, Cg, Cb, Tf;    // forward totals
};

// One compose step in terms of alpha; returns dL/dm, adds the colour / density
// gradient contributions (g_c w, g_sigma w) into cacc.
__device__ __forceinline__ float compose_adj(float d, float4 col, float a, int mode, SampleAdj& s, float (&cacc)[4],
                                             int compat) {
  const float w = a * s.T;
  const float T1 = s.T * (1.0f - a);
  s.Ps += d * w;
  s.Pr += col.x * w;
  s.Pg += col.y * w;
  s.Pb += col.z * w;
  cacc[0] += s.gcr * w;
  cacc[1] += s.gcg * w;
  cacc[2] += s.gcb * w;
  cacc[3] += s.gs * w;
  float dm = 0.f;
  if (!compat) {
    const float G = s.gs * (T1 * d - (s.sig - s.Ps)) + s.gcr * (T1 * col.x - (s.Cr - s.Pr)) +
                    s.gcg * (T1 * col.y - (s.Cg - s.Pg)) + s.gcb * (T1 * col.z - (s.Cb - s.Pb)) - s.gT * s.Tf;
    // soft_dm_from_G with m <= 0 <=> alpha <= 1/2 (laplace), band 0 < alpha < 0.9999 (linear)
    if (mode == STEP_LAPLACE) dm = a <= 0.5f ? G * a / (1.f - a) : G;
    else if (mode == STEP_LINEAR) dm = (a > 0.f && a < 0.9999f) ? G / (1.f - a) : 0.f;
  } else {
    const float O = 1.0f + 1e-6f - s.Tf;
    const float sc = 1.f / fmaxf(1.0f - a, 1e-6f);
    float ga = s.gs * (T1 * d - (s.sig - s.Ps)) * sc;
    ga += (s.gcr * (T1 * col.x * (O - a) - (s.Cr - s.Pr)) + s.gcg * (T1 * col.y * (O - a) - (s.Cg - s.Pg)) +
           s.gcb * (T1 * col.z * (O - a) - (s.Cb - s.Pb))) *
          (sc / O);
    if (mode == STEP_LAPLACE) dm = ga * (a <= 0.5f ? a : 1.f - a);
    else if (mode == STEP_LINEAR) dm = (a > 0.f && a < 0.9999f) ? ga : 0.f;
  }
  s.T = T1;
  return dm;
}

constexpr int RED_LO = G_K;   // slots reduced per pair: G_K .. G_K + 15
constexpr int RED_N = 16;

template <int WARPS>
__global__ void __launch_bounds__(WARPS * 32, 1) run_bwd_kernel(const __grid_constant__ SegLaunch L) {
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ uint64_t bar;
  __shared__ int s_scene, s_fail;
  const RunStage R = run_carve(smem, L.chunk_cap, WARPS, true);
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int nthr = blockDim.x;
  RunBuf& B = R.bufs[warp];
  float* gxb = R.gxb + warp * (3 * RUN_UNIT);
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    s_fail = 0;
  }
  for (int i = threadIdx.x; i < L.chunk_cap * GRAD_SLOTS; i += nthr) R.s.gacc[i] = 0.f;
  __syncthreads();
  uint32_t phase = 0;
  const int compat = L.compat;
  const int upr = (L.n_samples + RUN_UNIT - 1) / RUN_UNIT;

  auto flush_slots = [&](int sci) {
    const SceneDesc& o = L.sc[sci];
    float* dst = L.gslots + ((long long)o.stroke_begin + o.chunk_lo) * GRAD_SLOTS;
    for (int i = threadIdx.x; i < o.chunk_n * GRAD_SLOTS; i += nthr) {
      float v = R.s.gacc[i];
      if (v != 0.f) {
        atomicAdd(dst + i, v);
        R.s.gacc[i] = 0.f;
      }
    }
  };

  int sci = home_scene(L);
  while (sci >= 0) {
    if (!stage_chunk(L, L.sc[sci], R.s, &bar, phase, &s_fail)) {
      if (threadIdx.x == 0) atomicOr(L.status, ST_WAIT_TIMEOUT);
      return;
    }
    stage_bases(R, L.sc[sci].chunk_n);
    const SceneDesc& sc = L.sc[sci];
    int* counter = L.tile_counter + sci;
    const int n_units = sc.n_rays * upr;
    int item = 0;
    if (lane == 0) item = atomicAdd(counter, 1);
    item = __shfl_sync(0xffffffffu, item, 0);
    while (item < n_units) {
      const int ray_local = item / upr;
      const int j0 = (item - ray_local * upr) * RUN_UNIT;
      const int cnt = min(RUN_UNIT, L.n_samples - j0);
      Unit U;
      unit_setup(L, (sc.ray_begin + ray_local) * L.n_samples + j0, cnt, lane, B, U);
      SampleAdj s[2];
#pragma unroll
      for (int b = 0; b < 2; b++) {
        const int j = lane + 32 * b;
        const bool act = j < cnt;
        const long long si = U.si0 + (act ? j : 0);
        const float* st = L.state + 5 * si;
        s[b].Tf = st[0]; s[b].sig = st[1]; s[b].Cr = st[2]; s[b].Cg = st[3]; s[b].Cb = st[4];
        const float* sd = L.seeds + 5 * si;
        s[b].gs = sd[0]; s[b].gcr = sd[1]; s[b].gcg = sd[2]; s[b].gcb = sd[3]; s[b].gT = sd[4];
        if (!act) s[b].gs = s[b].gcr = s[b].gcg = s[b].gcb = s[b].gT = 0.f;
        V3 g0 = v3(0.f, 0.f, 0.f);
        if (sc.first_pass) {
          s[b].T = 1.f; s[b].Ps = s[b].Pr = s[b].Pg = s[b].Pb = 0.f;
        } else {
          const float* bs = L.bstate + 8 * si;
          s[b].T = bs[0]; s[b].Ps = bs[1]; s[b].Pr = bs[2]; s[b].Pg = bs[3]; s[b].Pb = bs[4];
          g0 = v3(bs[5], bs[6], bs[7]);
        }
        gxb[3 * j] = g0.x;
        gxb[3 * j + 1] = g0.y;
        gxb[3 * j + 2] = g0.z;
      }
      __syncwarp();
      int nruns = 0, npairs = 0;
      auto flush = [&]() {
        int sk, in;
        const int base = layout_pairs(B, nruns, lane, &sk, &in, nullptr);
        eval_pairs(L, R, B, U, npairs, lane);
        // composite adjoint per sample, runs in stroke order: dL/dm per pair into B.val,
        // colour / density gradients reduced per run
        for (int r = 0; r < nruns; r++) {
          const int rin = __shfl_sync(0xffffffffu, in, r);
          const int rb = __shfl_sync(0xffffffffu, base, r);
          const int slot = __shfl_sync(0xffffffffu, sk, r) & 0xffff;
          const int i0 = rin & 255, n = rin >> 8;
          const float* rec = R.s.recs + size_t(slot) * REC_FLOATS;
          const float d = rec[R_DENSITY];
          const float4 col = rec4(rec)[R_COLOR / 4];
          const int mode = (__float_as_int(rec[R_KIND]) >> 8) & 3;
          float cacc[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
          for (int b = 0; b < 2; b++) {
            const unsigned o = unsigned(lane + 32 * b - i0);
            if (o < unsigned(n)) B.val[rb + o] = compose_adj(d, col, B.val[rb + o], mode, s[b], cacc, compat);
          }
          // 4-value transpose reduction: lane l ends with the total of value l & 3
          {
            const bool up1 = lane & 1;
            float a0 = (up1 ? cacc[2] : cacc[0]) + __shfl_xor_sync(0xffffffffu, up1 ? cacc[0] : cacc[2], 1);
            float a1 = (up1 ? cacc[3] : cacc[1]) + __shfl_xor_sync(0xffffffffu, up1 ? cacc[1] : cacc[3], 1);
            const bool up2 = lane & 2;
            float t = (up2 ? a1 : a0) + __shfl_xor_sync(0xffffffffu, up2 ? a0 : a1, 2);
#pragma unroll
            for (int o = 4; o < 32; o <<= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
            // lane bits (1, 2) select value 2 * bit0 + bit1
            if (lane < 4 && t != 0.f)
              atomicAdd(R.s.gacc + size_t(slot) * GRAD_SLOTS + G_COLOR + ((lane & 1) << 1 | (lane >> 1)), t);
          }
        }
        __syncwarp();
        // SDF / transform adjoint per pair; segmented reduction over each run's lanes
        for (int p0 = 0; p0 < npairs; p0 += 32) {
          const int p = p0 + lane;
          float v[RED_LO + RED_N];
#pragma unroll
          for (int i = 0; i < RED_LO + RED_N; i++) v[i] = 0.f;
          int run = -1, slot = 0;
          if (p < npairs) {
            const int e = B.table[p];
            run = e >> 8;
            const int j = e & 255;
            slot = B.run_sk[run] & 0xffff;
            const long long si = U.si0 + j;
            const long long ray = si / L.n_samples;
            V3 x;
            float rr;
            load_sample(L, ray, (int)(si - ray * L.n_samples), si, x, rr);
            const float rinv = 1.f / rr;
            const float dm = B.val[p];
            const float* rec = R.s.recs + size_t(slot) * REC_FLOATS;
            const float4 h = rec4(rec)[0];
            const int kind = __float_as_int(h.x);
            const int bse = kind & 15;
            V3 g;
            if (bse <= B_TETRAHEDRON) {
              const V3 pl = prim_local(rec, x);
              const float sdf = prim_sdf(bse, pl, rec);
              const float f = (kind & K_S3FAC) ? s3_factor(bse, pl, xyz(rec4(rec)[R_S / 4]), rec) : 1.f;
              const float kk = h.y * f * rinv;
              const float m = -sdf * kk;
              const float K = m * dm;
              v[G_K] = K;
              g = prim_backprop(rec, kind, pl, -kk * dm, K, v, compat);
            } else if (bse == B_QUAD_BEZIER) {
              QuadFwd qf;
              const float sdf = quad_eval(rec, x, qf);
              const float kk = h.y * rinv;
              v[G_K] = -sdf * kk * dm;
              g = quad_adjoint(rec, qf, -kk * dm, v + G_CTRL);
            } else {
              CubicFwd cf;
              const float sdf = cubic_eval(rec, x, cf, bse == B_CATMULL_ROM);
              const float kk = h.y * rinv;
              const float dsdf = -kk * dm;
              v[G_K] = -sdf * kk * dm;
              g = cubic_adjoint(rec, x, cf, dsdf, v + G_CTRL, compat, bse == B_CATMULL_ROM);
              if (compat) g = g * dsdf;  // the reference multiplies by dL/dSDF again
            }
            atomicAdd(gxb + 3 * j, g.x);
            atomicAdd(gxb + 3 * j + 1, g.y);
            atomicAdd(gxb + 3 * j + 2, g.z);
          }
          // runs occupy contiguous lanes: reverse segmented scan, run heads hold totals
#pragma unroll
          for (int o = 1; o < 32; o <<= 1) {
            const int rr = __shfl_down_sync(0xffffffffu, run, o);
            const bool same = (lane + o < 32) && rr == run;
#pragma unroll
            for (int i = RED_LO; i < RED_LO + RED_N; i++) {
              const float t = __shfl_down_sync(0xffffffffu, v[i], o);
              if (same) v[i] += t;
            }
          }
          const int prev = __shfl_up_sync(0xffffffffu, run, 1);
          if (run >= 0 && (lane == 0 || prev != run)) {
            float* row = R.s.gacc + size_t(slot) * GRAD_SLOTS;
#pragma unroll
            for (int i = RED_LO; i < RED_LO + RED_N; i++)
              if (v[i] != 0.f) atomicAdd(row + i, v[i]);
          }
        }
        __syncwarp();
      };
      for (int hi = sc.chunk_n - 1; hi >= 0; hi -= 32) add_block_runs(R, U, B, hi, lane, nruns, npairs, flush);
      if (nruns) flush();
#pragma unroll
      for (int b = 0; b < 2; b++) {
        const int j = lane + 32 * b;
        if (j < cnt) {
          const long long si = U.si0 + j;
          const V3 g = v3(gxb[3 * j], gxb[3 * j + 1], gxb[3 * j + 2]);
          if (sc.last_pass) {
            if (L.grad_x) {
              L.grad_x[3 * si] = g.x;
              L.grad_x[3 * si + 1] = g.y;
              L.grad_x[3 * si + 2] = g.z;
            }
          } else {
            float* bs = L.bstate + 8 * si;
            bs[0] = s[b].T; bs[1] = s[b].Ps; bs[2] = s[b].Pr; bs[3] = s[b].Pg; bs[4] = s[b].Pb;
            bs[5] = g.x; bs[6] = g.y; bs[7] = g.z;
          }
        }
      }
      __syncwarp();
      if (lane == 0) item = atomicAdd(counter, 1);
      item = __shfl_sync(0xffffffffu, item, 0);
    }
    __syncthreads();  // every warp is done with the staged chunk
    flush_slots(sci);
    if (threadIdx.x == 0) s_scene = next_scene(L);
    __syncthreads();
    sci = s_scene;
  }
}

// ================================================================ launchers

template <int W, bool BWD>
static cudaError_t launch_run_w(const SegLaunch& L, int grid, size_t smem, cudaStream_t st) {
  auto* k = BWD ? run_bwd_kernel<W> : run_fwd_kernel<W>;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  k<<<grid, W * 32, smem, st>>>(L);
  return cudaGetLastError();
}

cudaError_t launch_run_fwd(const SegLaunch& L, int grid, int warps, size_t smem, cudaStream_t st) {
  switch (warps) {
    case 4: return launch_run_w<4, false>(L, grid, smem, st);
    case 8: return launch_run_w<8, false>(L, grid, smem, st);
    case 16: return launch_run_w<16, false>(L, grid, smem, st);
    default: return cudaErrorInvalidValue;
  }
}
cudaError_t launch_run_bwd(const SegLaunch& L, int grid, int warps, size_t smem, cudaStream_t st) {
  switch (warps) {
    case 4: return launch_run_w<4, true>(L, grid, smem, st);
    case 8: return launch_run_w<8, true>(L, grid, smem, st);
    case 16: return launch_run_w<16, true>(L, grid, smem, st);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace n3ds
