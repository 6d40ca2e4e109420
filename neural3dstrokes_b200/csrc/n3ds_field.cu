// Fused stroke-field kernels for sm_100a.
//
// Work decomposition. A ray's N samples are split into segments of up to 32
// consecutive samples; one warp owns one segment at a time (lane = sample). Stroke
// records of the current scene are staged into shared memory by one bulk
// (cp.async.bulk / TMA) copy per chunk of strokes, completed on an mbarrier. For each
// segment the forward warp first culls the chunk: lane j tests stroke (top - j) of a
// 32-stroke block against the segment's bounding capsule, and a ballot gives the
// surviving strokes in descending index order, i.e. the reference compositing order
// (compositing.cu:34, last stroke on top); the survivors that carry an exact reach
// test (tetrahedra, octahedra, curves) are then tested 32 at a time, one per lane.
// Every lane then evaluates the surviving strokes for its own sample; the stroke (and
// so the SDF type) is warp-uniform, so mixed-type scenes run without divergence. The
// forward records, per segment and 32-stroke block, which survivors reach the alpha
// threshold at some sample; the backward reads those words instead of culling.
//
// Persistent CTAs (one per SM) with scene affinity: the host gives every scene of a
// launch a share of the CTAs proportional to its work (rays x strokes in the chunk),
// and each CTA stages its home scene once. Its warps take whole rays (all their
// segments) from that scene's counter; when the scene runs dry the CTA synchronises
// once and moves to the scene with the most rays left, restaging its records. So a
// CTA waits for its slowest warp only at a scene change, a few times per launch.
// Scenes with more strokes than one stage holds run in several passes (one launch
// each), carrying the per-sample composite state through HBM.
//
// The backward recomputes each sample's stroke alphas from the forward checkpoint
// (final T, density and colour sum per sample), evaluates the exact adjoint of the
// overlay composite in the division-safe form
//   (1 - a_s) dL/da_s = g_sigma (T_{s+1} d_s - suffix_sigma)
//                     + g_C . (T_{s+1} c_s - suffix_C) - g_T T_final,
// and reduces per-stroke gradients across the warp with a transpose reduction
// before one shared-memory atomic per value; CTAs flush to global memory once per
// staged chunk. Template switches compile out what a call does not need: the mask
// recording (a forward no backward follows), the pair counters (statistics) and the
// sample-position gradient.
#include "n3ds_stage.cuh"

namespace n3ds {

__host__ __device__ inline size_t stage_bytes(int cap) { return align16(cap * 16) + align16(cap * 4) + size_t(cap) * REC_FLOATS * 4; }
// forward: the stage plus, per warp, 32 words of polytope-test rejections
size_t seg_fwd_smem(int cap, int warps) { return stage_bytes(cap) + size_t(warps) * 32 * 4; }
size_t seg_bwd_smem(int cap) { return stage_bytes(cap) + size_t(cap) * GRAD_SLOTS * 4; }

// Segment geometry shared by both directions.
struct SegCtx {
  long long si;   // this lane's sample index
  bool active;
  V3 x;
  float r, rinv;
  V3 A, AB;
  float invL2, rho, rmax;
};

// Culling geometry of a segment whose lanes 0 .. cnt - 1 hold its samples: the chord
// A..B, the samples' spread rho about it and the largest sample radius.
__device__ __forceinline__ void seg_geometry(SegCtx& c, int cnt) {
  c.A = shfl3(c.x, 0);
  V3 B = shfl3(c.x, cnt - 1);
  c.AB = B - c.A;
  float l2 = dot(c.AB, c.AB);
  c.invL2 = l2 > 0.f ? 1.f / l2 : 0.f;
  c.rho = warp_max(c.active ? seg_dist(c.x, c.A, c.AB, c.invL2) : 0.f);
  c.rmax = warp_max(c.active ? fabsf(c.r) : 0.f);
}

// GEOM: with the culling geometry (a backward that reads the forward's block masks
// needs none).
template <bool GEOM = true>
__device__ __forceinline__ SegCtx seg_setup(const SegLaunch& L, const SceneDesc& sc, int seg, int lane) {
  SegCtx c;
  const int spr = L.segs_per_ray;
  const int ray_local = seg / spr;
  const int g = seg - ray_local * spr;
  const long long ray = sc.ray_begin + ray_local;
  const int i0 = g * 32;
  const int cnt = min(32, L.n_samples - i0);
  c.active = lane < cnt;
  c.si = ray * L.n_samples + i0 + (c.active ? lane : 0);
  load_sample(L, ray, i0 + (c.active ? lane : 0), c.si, c.x, c.r);
  c.rinv = 1.f / c.r;
  if (GEOM) seg_geometry(c, cnt);
  return c;
}

// Tetrahedron / octahedron reach test (cull_block, flagged strokes). Their SDFs are
// (g(p) - 1) / sqrt(3) with g the largest of the diagonal forms +-x +-y +-z (four of
// them for the tetrahedron, strokes_sdf.h:584-588, 607-613), so the samples where
// alpha reaches the cut lie in the polytope g(p) <= 1 + sqrt(3) tau_local, tau_local
// = R_PLANE / sqrt(3) * r. Every sample of the segment is within rho of the chord A..B,
// so the chord, in the stroke's local frame, is clipped against the planes offset by
// that distance (|n| = sqrt(3)); an empty interval means no sample can reach the cut.
__device__ __forceinline__ bool polytope_reachable(const float* rec, const SegCtx& c) {
  const float4 m0 = rec4(rec)[R_M / 4], m1 = rec4(rec)[R_M / 4 + 1], m2 = rec4(rec)[R_M / 4 + 2];
  const V3 dA = v3(c.A.x - m0.w, c.A.y - m1.w, c.A.z - m2.w);
  const V3 dB = dA + c.AB;
  const V3 a = v3(fmaf(m0.x, dA.x, fmaf(m0.y, dA.y, m0.z * dA.z)), fmaf(m1.x, dA.x, fmaf(m1.y, dA.y, m1.z * dA.z)),
                  fmaf(m2.x, dA.x, fmaf(m2.y, dA.y, m2.z * dA.z)));
  const V3 b = v3(fmaf(m0.x, dB.x, fmaf(m0.y, dB.y, m0.z * dB.z)), fmaf(m1.x, dB.x, fmaf(m1.y, dB.y, m1.z * dB.z)),
                  fmaf(m2.x, dB.x, fmaf(m2.y, dB.y, m2.z * dB.z)));
  const float cc = (1.f + rec[R_PLANE] * c.rmax + 1.7320508f * c.rho * rec[R_SINV]) * 1.0001f + 1e-5f;
  float lo = 0.f, hi = 1.f;
  bool out = false;
  auto plane = [&](float fa, float fb) {
    fa -= cc;
    fb -= cc;
    if (fa > 0.f && fb > 0.f) out = true;
    else if (fa > 0.f) lo = fmaxf(lo, fa / (fa - fb));
    else if (fb > 0.f) hi = fminf(hi, fa / (fa - fb));
  };
  const float ua = a.x + a.y, va = a.x - a.y, ub = b.x + b.y, vb = b.x - b.y;
  // the tetrahedron's faces: |x + y| - z and |x - y| + z
  plane(ua - a.z, ub - b.z);
  plane(-ua - a.z, -ub - b.z);
  plane(va + a.z, vb + b.z);
  plane(-va + a.z, -vb + b.z);
  if ((__float_as_int(rec[R_KIND]) & 15) == B_OCTAHEDRON) {  // the other four
    plane(ua + a.z, ub + b.z);
    plane(-ua + a.z, -ub + b.z);
    plane(va - a.z, vb - b.z);
    plane(-va - a.z, -vb - b.z);
  }
  return !out && lo <= hi + 1e-6f;
}

// Ellipsoid reach test (flagged per-axis-scaled spheres): the chord, in the stroke's
// local frame, must pass within 1 + R_PLANE r_max of the origin; the samples' distance
// rho to the chord grows by at most 1 / s_min in that frame.
__device__ __forceinline__ bool ellipsoid_reachable(const float* rec, const SegCtx& c) {
  const float4 m0 = rec4(rec)[R_M / 4], m1 = rec4(rec)[R_M / 4 + 1], m2 = rec4(rec)[R_M / 4 + 2];
  const V3 dA = v3(c.A.x - m0.w, c.A.y - m1.w, c.A.z - m2.w);
  const V3 dB = dA + c.AB;
  const V3 a = v3(fmaf(m0.x, dA.x, fmaf(m0.y, dA.y, m0.z * dA.z)), fmaf(m1.x, dA.x, fmaf(m1.y, dA.y, m1.z * dA.z)),
                  fmaf(m2.x, dA.x, fmaf(m2.y, dA.y, m2.z * dA.z)));
  const V3 b = v3(fmaf(m0.x, dB.x, fmaf(m0.y, dB.y, m0.z * dB.z)), fmaf(m1.x, dB.x, fmaf(m1.y, dB.y, m1.z * dB.z)),
                  fmaf(m2.x, dB.x, fmaf(m2.y, dB.y, m2.z * dB.z)));
  const float sinv = fmaxf(rec[R_SINV], fmaxf(rec[R_SINV + 1], rec[R_SINV + 2]));
  const float reach = (1.f + rec[R_PLANE] * c.rmax + c.rho * sinv) * 1.0001f + 1e-5f;
  const V3 ab = b - a;
  const float l2 = dot(ab, ab);
  const float u = l2 > 0.f ? clampf(-dot(a, ab) / l2, 0.f, 1.f) : 0.f;
  const V3 q = a + ab * u;
  return dot(q, q) <= reach * reach;
}

// Capsule reach test (flagged capsules with h > 0): the SDF is the distance to the
// axis segment y in [-h, h] minus 1 (strokes_sdf.h:434-440), so alpha reaches the cut
// only within 1 + tau_local of that segment (R_PLANE = tau_local per unit radius).
// The local chord's distance to the axis segment (closest points of two segments,
// clamped to both) must not exceed it, widened by the samples' spread about the chord.
__device__ __forceinline__ bool capsule_reachable(const float* rec, const SegCtx& c) {
  const float4 m0 = rec4(rec)[R_M / 4], m1 = rec4(rec)[R_M / 4 + 1], m2 = rec4(rec)[R_M / 4 + 2];
  const V3 dA = v3(c.A.x - m0.w, c.A.y - m1.w, c.A.z - m2.w);
  const V3 dB = dA + c.AB;
  const V3 a = v3(fmaf(m0.x, dA.x, fmaf(m0.y, dA.y, m0.z * dA.z)), fmaf(m1.x, dA.x, fmaf(m1.y, dA.y, m1.z * dA.z)),
                  fmaf(m2.x, dA.x, fmaf(m2.y, dA.y, m2.z * dA.z)));
  const V3 b = v3(fmaf(m0.x, dB.x, fmaf(m0.y, dB.y, m0.z * dB.z)), fmaf(m1.x, dB.x, fmaf(m1.y, dB.y, m1.z * dB.z)),
                  fmaf(m2.x, dB.x, fmaf(m2.y, dB.y, m2.z * dB.z)));
  const float h = rec[R_BP];
  const float reach = (1.f + rec[R_PLANE] * c.rmax + c.rho * rec[R_SINV]) * 1.0001f + 1e-5f;
  // chord a + u d, u in [0, 1]; axis (0, v, 0), v in [-h, h]
  const V3 d = b - a;
  const float dd = dot(d, d);
  // u minimising the distance to the axis line, then v on the clamped axis, then u again
  float u = 0.f;
  const float den = dd - d.y * d.y;  // |d|^2 - d_y^2: the chord's part across the axis
  if (den > 1e-12f * fmaxf(dd, 1e-30f)) u = clampf(-(a.x * d.x + a.z * d.z) / den, 0.f, 1.f);
  float v = clampf(a.y + u * d.y, -h, h);
  if (dd > 0.f) u = clampf((d.x * -a.x + d.y * (v - a.y) + d.z * -a.z) / dd, 0.f, 1.f);
  v = clampf(a.y + u * d.y, -h, h);
  const V3 q = v3(a.x + u * d.x, a.y + u * d.y - v, a.z + u * d.z);
  return dot(q, q) <= reach * reach;
}

// Curve reach test (the forward's batched pass, flagged curves). Every sample where
// alpha reaches the cut is within r_max + tau of the curve (the SDF uses the distance
// to one curve point, no less than the true distance), the curve within eps of its
// polyline (R_CTEST = r_max + eps), each polyline piece within its half-length of its
// midpoint, and the segment's samples within rho of the chord: the chord has to pass
// within half-length + R_CTEST + margin r_max + rho of some piece's midpoint. The
// pieces are visited from a lane-dependent start, so that lanes reading different
// strokes' records fall into different shared-memory banks.
__device__ __forceinline__ bool curve_reachable(const float* rec, const SegCtx& c, float margin, int lane) {
  const float reach = rec[R_CTEST] + margin * c.rmax + c.rho;
  if ((__float_as_int(rec[R_KIND]) & 15) == B_QUAD_BEZIER) {
    const float4 qA = rec4(rec)[R_QA / 4], qa = rec4(rec)[R_Qa / 4], qb = rec4(rec)[R_Qb / 4];
    const V3 A = xyz(qA), a2 = xyz(qa) * 2.f, b = xyz(qb);
    auto at = [&](float t) { return A + (a2 + b * t) * t; };  // B(t) = A + 2 a t + b t^2
    int p = lane & 7;
    V3 v0 = at(p * 0.125f);
    for (int k = 0; k < 8; k++) {
      const V3 v1 = at((p + 1) * 0.125f);
      const V3 m = (v0 + v1) * 0.5f, h = (v1 - v0) * 0.5f;
      if (seg_dist(m, c.A, c.AB, c.invL2) <= sqrtf(dot(h, h)) + reach) return true;
      p = (p + 1) & 7;
      v0 = p == 0 ? A : v1;
    }
    return false;
  }
  int p = lane % CUBIC_SEGMENTS;
  V3 v0 = v3(rec[R_CV + 3 * p], rec[R_CV + 3 * p + 1], rec[R_CV + 3 * p + 2]);
  for (int k = 0; k < CUBIC_SEGMENTS; k++) {
    const V3 v1 = v3(rec[R_CV + 3 * p + 3], rec[R_CV + 3 * p + 4], rec[R_CV + 3 * p + 5]);
    const V3 m = (v0 + v1) * 0.5f, h = (v1 - v0) * 0.5f;
    if (seg_dist(m, c.A, c.AB, c.invL2) <= sqrtf(dot(h, h)) + reach) return true;
    p = p + 1 == CUBIC_SEGMENTS ? 0 : p + 1;
    v0 = p == 0 ? v3(rec[R_CV], rec[R_CV + 1], rec[R_CV + 2]) : v1;
  }
  return false;
}

// Sphere test of one 32-stroke block (lane j: stroke hi - j) against the segment's
// capsule; the ballot of the survivors. The survivors flagged for an exact reach test
// are these and the block's flag word (flagged_words); the forward batches those tests.
__device__ __forceinline__ unsigned cull_block_sphere(const Stage& S, const SegCtx& c, int hi, int lane) {
  const int sl = hi - lane;
  bool cand = false;
  if (sl >= 0) {
    float4 ca = S.cull_a[sl];
    float d = seg_dist(v3(ca.x, ca.y, ca.z), c.A, c.AB, c.invL2);
    cand = !(d - c.rho > ca.w + fabsf(S.cull_b[sl]) * c.rmax);
  }
  return __ballot_sync(0xffffffffu, cand);
}

// The strokes of the staged chunk flagged for an exact reach test (the margin's sign
// bit, set by the prep kernel), one word per 32-stroke block: lane k returns block k's.
__device__ __forceinline__ unsigned flagged_words(const Stage& S, int chunk_n, int lane) {
  unsigned mine = 0u;
  for (int k = 0; 32 * k < chunk_n; k++) {
    const int sl = chunk_n - 1 - 32 * k - lane;
    const unsigned f = __ballot_sync(0xffffffffu, sl >= 0 && __float_as_int(S.cull_b[sl]) < 0);
    if (lane == k) mine = f;
  }
  return mine;
}

// ================================================================== forward

// RECORD: write the stroke-block masks (L.block_masks non-null) for the backward.
// STATS: count evaluated pairs per base type into L.stats (non-null).
// COMMON: every stroke of the launch is a common primitive (the caller's hint, checked
// by the prep kernel): the kernel carries only those six bases' evaluation code.
template <int WARPS, bool RECORD, bool STATS, bool COMMON>
__global__ void __launch_bounds__(WARPS * 32, 1) seg_fwd_kernel(const __grid_constant__ SegLaunch L) {
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ uint64_t bar;
  __shared__ int s_scene, s_fail;
  const Stage S = carve(smem, L.chunk_cap, false);
  const int lane = threadIdx.x & 31;
  // this warp's 32 words of polytope-test rejections (one per block of the chunk)
  unsigned* const kill = reinterpret_cast<unsigned*>(smem + stage_bytes(L.chunk_cap)) + (threadIdx.x >> 5) * 32;
  kill[lane] = 0u;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    s_fail = 0;
  }
  unsigned long long kcount = 0;  // lane k: evaluated (sample, stroke) pairs of base k
  uint32_t phase = 0;
  int sci = home_scene(L);
  while (sci >= 0) {
    if (!stage_chunk(L, L.sc[sci], S, &bar, phase, &s_fail)) {
      if (threadIdx.x == 0) atomicOr(L.status, ST_WAIT_TIMEOUT);
      return;
    }
    const SceneDesc& sc = L.sc[sci];
    const unsigned my_flag = flagged_words(S, sc.chunk_n, lane);
    int* counter = L.tile_counter + sci;
    int item = 0;
    if (lane == 0) item = atomicAdd(counter, L.rays_per_item);
    item = __shfl_sync(0xffffffffu, item, 0);
    while (item < sc.n_rays) {
      const int item_end = min(item + L.rays_per_item, sc.n_rays);
      for (int ray_local = item; ray_local < item_end; ray_local++) {
        for (int g = 0; g < L.segs_per_ray; g++) {
          SegCtx c = seg_setup(L, sc, ray_local * L.segs_per_ray + g, lane);
          float T, sig, cr, cg, cb;
          if (sc.first_pass) {
            T = 1.f; sig = cr = cg = cb = 0.f;
          } else {
            const float* st = L.state + 5 * c.si;
            T = st[0]; sig = st[1]; cr = st[2]; cg = st[3]; cb = st[4];
          }
          const unsigned nact = __popc(__ballot_sync(0xffffffffu, c.active));
          unsigned* bm = RECORD ? L.block_masks + sc.mask_begin +
                                      (long long)(ray_local * L.segs_per_ray + g) * sc.mask_words
                                : nullptr;
          // Culling in three steps. 1: the sphere test of every block of the chunk (at most
          // 32 blocks); lane k keeps block k's survivors and its polytope-flagged subset.
          const int nblk = (sc.chunk_n + 31) >> 5;
          unsigned my_mask = 0u;
          for (int k = 0; k < nblk; k++) {
            const unsigned m = cull_block_sphere(S, c, sc.chunk_n - 1 - 32 * k, lane);
            if (lane == k) my_mask = m;
          }
          const unsigned my_poly = my_mask & my_flag;
          // 2: the flagged candidates of all blocks, 32 per pass, one per lane: the owner
          // block is the last with prefix count <= the candidate's index (5-step binary
          // search over the lanes), the stroke its n-th flagged bit; rejections are
          // collected in this warp's kill words.
          if (__any_sync(0xffffffffu, my_poly != 0u)) {
            const int cnt = __popc(my_poly);
            int incl = cnt;
  #pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
              const int y = __shfl_up_sync(0xffffffffu, incl, o);
              if (lane >= o) incl += y;
            }
            const int off = incl - cnt;
            const int total = __shfl_sync(0xffffffffu, incl, 31);
            for (int g0 = 0; g0 < total; g0 += 32) {
              const int g = g0 + lane;
              int kk = 0;
  #pragma unroll
              for (int step = 16; step > 0; step >>= 1) {
                const int o = __shfl_sync(0xffffffffu, off, (kk + step) & 31);
                if (o <= g) kk += step;
              }
              const unsigned pm = __shfl_sync(0xffffffffu, my_poly, kk);
              const int okk = __shfl_sync(0xffffffffu, off, kk);
              if (g < total) {
                unsigned x = pm;
                for (int n = g - okk; n > 0; n--) x &= x - 1u;
                const int bit = __ffs(x) - 1;
                const int slot = sc.chunk_n - 1 - 32 * kk - bit;
                const float* rec = S.recs + size_t(slot) * REC_FLOATS;
                const int rb = __float_as_int(rec[R_KIND]) & 15;
                const bool reach = rb == B_SPHERE        ? ellipsoid_reachable(rec, c)
                                   : rb == B_CAPSULE     ? capsule_reachable(rec, c)
                                   : rb <= B_TETRAHEDRON ? polytope_reachable(rec, c)
                                   : COMMON              ? true
                                                         : curve_reachable(rec, c, fabsf(S.cull_b[slot]), lane);
                if (!reach) atomicOr(kill + kk, 1u << bit);
              }
            }
            __syncwarp();
            my_mask &= ~kill[lane];
            kill[lane] = 0u;
            __syncwarp();
          }
          // 3: evaluate the survivors block by block in compositing order, visiting only
          // the blocks with survivors (lane k's word is block k's, lanes >= nblk hold 0)
          unsigned todo = __ballot_sync(0xffffffffu, my_mask != 0u);
          while (todo) {
            const int k = __ffs(todo) - 1;
            todo &= todo - 1u;
            const int hi = sc.chunk_n - 1 - 32 * k;
            unsigned mask = __shfl_sync(0xffffffffu, my_mask, k);
            unsigned kept = 0;  // this lane's strokes of the block whose adjoint the backward needs
            while (mask) {
              const int b = __ffs(mask) - 1;
              mask &= mask - 1;
              const float* rec = S.recs + size_t(hi - b) * REC_FLOATS;
              const float a = COMMON ? pair_alpha_common(rec, c.x, c.rinv) : pair_alpha(rec, c.x, c.rinv);
              if (RECORD && a >= L.skip_alpha) kept |= 1u << b;
              if (STATS && lane == (__float_as_int(rec[R_KIND]) & 15)) kcount += nact;
              const float w = a * T;
              const float4 col = rec4(rec)[R_COLOR / 4];
              T *= (1.0f - a);
              sig += rec[R_DENSITY] * w;
              cr += col.x * w;
              cg += col.y * w;
              cb += col.z * w;
            }
            // the words start at zero (cleared before the launch): store the non-empty ones
            if (RECORD) {
              kept = __reduce_or_sync(0xffffffffu, c.active ? kept : 0u);
              if (lane == 0 && kept) bm[(sc.n_strokes - 1 - (sc.chunk_lo + hi)) >> 5] = kept;
            }
          }
          if (c.active) {
            float* st = L.state + 5 * c.si;
            st[0] = T; st[1] = sig; st[2] = cr; st[3] = cg; st[4] = cb;
          }
        }
      }
      if (lane == 0) item = atomicAdd(counter, L.rays_per_item);
      item = __shfl_sync(0xffffffffu, item, 0);
    }
    __syncthreads();  // every warp is done with the staged chunk
    if (threadIdx.x == 0) s_scene = next_scene(L);
    __syncthreads();
    sci = s_scene;
  }
  if (STATS && lane < 16 && kcount) {
    atomicAdd(L.stats, kcount);
    atomicAdd(L.stats + 1 + lane, kcount);
  }
}

// ================================================================= backward

__device__ __forceinline__ void gacc_add(float* row, int idx, float v) {
  if (v != 0.f) atomicAdd(row + idx, v);
}

template <int NV>
__device__ __forceinline__ void reduce_into(float (&v)[NV], float* row, int lane) {
  int idx;
  float tot = warp_transpose_reduce<NV>(v, lane, &idx);
  if (NV == 32 || lane < 16) gacc_add(row, idx, tot);
}

struct CompAdj {
  float T, Ps, Pr, Pg, Pb;          // running (through the previous stroke)
  float gs, gcr, gcg, gcb, gT;      // seeds
  float sig, Cr, Cg, Cb, Tf;        // forward totals
};

// Compose step + exact adjoint for one stroke; returns dL/dm. Writes colour /
// density slots. compat: the reference compose adjoint (compositing.cu:104-155).
__device__ __forceinline__ float compose_step(const float* rec, float a, float m, int mode, CompAdj& s,
                                              float* v, int compat) {
  const float d = rec[R_DENSITY];
  const float4 col = rec4(rec)[R_COLOR / 4];
  const float c0 = col.x, c1 = col.y, c2 = col.z;
  const float w = a * s.T;
  const float T1 = s.T * (1.0f - a);
  s.Ps += d * w;
  s.Pr += c0 * w;
  s.Pg += c1 * w;
  s.Pb += c2 * w;
  v[G_COLOR + 0] += s.gcr * w;
  v[G_COLOR + 1] += s.gcg * w;
  v[G_COLOR + 2] += s.gcb * w;
  v[G_DENSITY] += s.gs * w;
  float dm;
  if (!compat) {
    const float G = s.gs * (T1 * d - (s.sig - s.Ps)) + s.gcr * (T1 * c0 - (s.Cr - s.Pr)) +
                    s.gcg * (T1 * c1 - (s.Cg - s.Pg)) + s.gcb * (T1 * c2 - (s.Cb - s.Pb)) - s.gT * s.Tf;
    dm = soft_dm_from_G(mode, m, a, G);
  } else {
    // reference: dL/da = [g_d (T' d - suf_d) + sum g_c O (T' c (O - a) - suf_c) / O^2] / max(1 - a, 1e-6)
    const float O = 1.0f + 1e-6f - s.Tf;
    const float sc = 1.f / fmaxf(1.0f - a, 1e-6f);
    float ga = s.gs * (T1 * d - (s.sig - s.Ps)) * sc;
    ga += (s.gcr * (T1 * c0 * (O - a) - (s.Cr - s.Pr)) + s.gcg * (T1 * c1 * (O - a) - (s.Cg - s.Pg)) +
           s.gcb * (T1 * c2 * (O - a) - (s.Cb - s.Pb))) * (sc / O);
    dm = soft_dm(mode, m, a, ga);
  }
  s.T = T1;
  return dm;
}

// Composite prefix update only, for a stroke whose alpha is below the skip threshold
// at every sample of the segment: its gradient contributions (all proportional to
// alpha) are dropped like those of a culled stroke, later strokes still see its
// (tiny) occlusion.
__device__ __forceinline__ void compose_skip(const float* rec, float a, CompAdj& s) {
  const float d = rec[R_DENSITY];
  const float4 col = rec4(rec)[R_COLOR / 4];
  const float w = a * s.T;
  s.Ps += d * w;
  s.Pr += col.x * w;
  s.Pg += col.y * w;
  s.Pb += col.z * w;
  s.T *= (1.0f - a);
}

// GX: the sample-position gradient is wanted (L.grad_x non-null); without it the
// kernel carries no position gradient at all. COMPAT: L.compat as a constant (the
// reference's gradient formulas, 1, or the exact adjoint, 0), so that the adjoint's
// formula choices are made at compile time. MASKS: the forward recorded stroke-block
// masks (L.block_masks non-null); the kernel then carries no culling code. If the
// masks were recorded at another threshold (their tag), it visits every block: the
// per-candidate test of the skip threshold makes the decisions culling would make.
// STATS: count the evaluated pairs into L.stats (non-null).
template <int WARPS, bool GX, int COMPAT, bool MASKS, bool STATS>
__global__ void __launch_bounds__(WARPS * 32, 1) seg_bwd_kernel(const __grid_constant__ SegLaunch L) {
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ uint64_t bar;
  __shared__ int s_scene, s_fail;
  const Stage S = carve(smem, L.chunk_cap, true);
  const int lane = threadIdx.x & 31;
  const int nthr = blockDim.x;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    s_fail = 0;
  }
  for (int i = threadIdx.x; i < L.chunk_cap * GRAD_SLOTS; i += nthr) S.gacc[i] = 0.f;
  __syncthreads();
  uint32_t phase = 0;
  constexpr int compat = COMPAT;
  const bool tag_ok = MASKS && *L.mask_tag == __float_as_int(L.skip_alpha);
  constexpr bool kGeom = !MASKS;  // the culling geometry only where the kernel culls
  unsigned long long bcount = 0;  // lane 0: evaluated (sample, stroke) pairs

  auto flush = [&](int sci) {
    const SceneDesc& o = L.sc[sci];
    float* dst = L.gslots + ((long long)o.stroke_begin + o.chunk_lo) * GRAD_SLOTS;
    for (int i = threadIdx.x; i < o.chunk_n * GRAD_SLOTS; i += nthr) {
      float v = S.gacc[i];
      if (v != 0.f) {
        atomicAdd(dst + i, v);
        S.gacc[i] = 0.f;
      }
    }
  };

  int sci = home_scene(L);
  while (sci >= 0) {
    if (!stage_chunk(L, L.sc[sci], S, &bar, phase, &s_fail)) {
      if (threadIdx.x == 0) atomicOr(L.status, ST_WAIT_TIMEOUT);
      return;
    }
    const SceneDesc& sc = L.sc[sci];
    int* counter = L.tile_counter + sci;
    int item = 0;
    if (lane == 0) item = atomicAdd(counter, L.rays_per_item);
    item = __shfl_sync(0xffffffffu, item, 0);
    while (item < sc.n_rays) {
      const int item_end = min(item + L.rays_per_item, sc.n_rays);
      for (int ray_local = item; ray_local < item_end; ray_local++) {
        for (int g = 0; g < L.segs_per_ray; g++) {
          SegCtx c = seg_setup<kGeom>(L, sc, ray_local * L.segs_per_ray + g, lane);
          CompAdj s;
          {
            const float* st = L.state + 5 * c.si;
            s.Tf = st[0]; s.sig = st[1]; s.Cr = st[2]; s.Cg = st[3]; s.Cb = st[4];
            const float* sd = L.seeds + 5 * c.si;
            s.gs = sd[0]; s.gcr = sd[1]; s.gcg = sd[2]; s.gcb = sd[3]; s.gT = sd[4];
            if (!c.active) {
              s.gs = s.gcr = s.gcg = s.gcb = s.gT = 0.f;
            }
          }
          V3 gx;
          if (sc.first_pass) {
            s.T = 1.f; s.Ps = s.Pr = s.Pg = s.Pb = 0.f;
            gx = v3(0.f, 0.f, 0.f);
          } else {
            const float* b = L.bstate + 8 * c.si;
            s.T = b[0]; s.Ps = b[1]; s.Pr = b[2]; s.Pg = b[3]; s.Pb = b[4];
            gx = GX ? v3(b[5], b[6], b[7]) : v3(0.f, 0.f, 0.f);
          }
          const unsigned nact = __popc(__ballot_sync(0xffffffffu, c.active));
          // The chunk's blocks (at most 32: stages hold at most 1024 strokes, in multiples
          // of 32) are mask words w0 .. w0 + nblk - 1 of the segment; lane k holds block
          // k's word, and only the blocks with a kept stroke are visited. Without masks
          // every block is visited and culled.
          const int nblk = (sc.chunk_n + 31) >> 5;
          unsigned held = 0u, todo;
          if (MASKS) {
            if (tag_ok) {
              const unsigned* bm = L.block_masks + sc.mask_begin +
                                   (long long)(ray_local * L.segs_per_ray + g) * sc.mask_words;
              const int w0 = (sc.n_strokes - sc.chunk_lo - sc.chunk_n) >> 5;
              held = lane < nblk ? bm[w0 + lane] : 0u;
            } else {
              held = lane < nblk ? 0xffffffffu : 0u;
            }
            todo = __ballot_sync(0xffffffffu, held != 0u);
          } else {
            todo = nblk >= 32 ? 0xffffffffu : (1u << nblk) - 1u;
          }
          while (todo) {
            const int k = __ffs(todo) - 1;
            todo &= todo - 1u;
            const int hi = sc.chunk_n - 1 - 32 * k;
            unsigned mask;
            if (MASKS) {
              mask = __shfl_sync(0xffffffffu, held, k);
              if (hi < 31) mask &= (2u << hi) - 1u;  // only strokes hi .. 0 exist in the last block
            } else {
              mask = cull_block_sphere(S, c, hi, lane);  // conservative: no exact reach tests here
            }
            while (mask) {
              const int b = __ffs(mask) - 1;
              mask &= mask - 1;
              const int sl = hi - b;
              const float* rec = S.recs + size_t(sl) * REC_FLOATS;
              float* row = S.gacc + size_t(sl) * GRAD_SLOTS;
              if (STATS) bcount += nact;
              const float4 h = rec4(rec)[0];
              const int kind = __float_as_int(h.x);
              const int base = kind & 15;
              const int mode = (kind >> 8) & 3;
              // gradient slots start at -0.0: -0 + x == x exactly, so each slot's first
              // `+=` compiles to a plain move (0 + x does not fold: it turns -0 into +0)
              if (base <= B_TETRAHEDRON) {
                float v[16];
    #pragma unroll
                for (int j = 0; j < 16; j++) v[j] = -0.f;
                const V3 p = prim_local(rec, c.x);
                const float sdf = prim_sdf(base, p, rec);
                const float f = (kind & K_S3FAC) ? s3_factor(base, p, xyz(rec4(rec)[R_S / 4]), rec) : 1.f;
                const float kk = h.y * f * c.rinv;
                const float m = -sdf * kk;
                const float a = mode == STEP_HARD ? (sdf <= 0.f ? 1.f : 0.f) : soft_alpha(mode, m);
                const bool below = __all_sync(0xffffffffu, !c.active || a < L.skip_alpha);
                if (below || (kind & K_FROZEN)) {  // the kind word is warp-uniform
                  compose_skip(rec, a, s);
                  continue;
                }
                const float dm = compose_step(rec, a, m, mode, s, v, compat);
                const float K = m * dm;
                v[G_K] += K;
                const V3 gp = prim_backprop(rec, kind, p, -kk * dm, K, v, compat);
                if (GX) gx += gp;
                reduce_into<16>(v, row, lane);
              } else if (base == B_QUAD_BEZIER) {
                float v[16];
    #pragma unroll
                for (int j = 0; j < 16; j++) v[j] = -0.f;
                QuadFwd qf;
                const float sdf = quad_eval(rec, c.x, qf);
                const float kk = h.y * c.rinv;
                const float m = -sdf * kk;
                const float a = mode == STEP_HARD ? (sdf <= 0.f ? 1.f : 0.f) : soft_alpha(mode, m);
                const bool below = __all_sync(0xffffffffu, !c.active || a < L.skip_alpha);
                if (below || (kind & K_FROZEN)) {  // the kind word is warp-uniform
                  compose_skip(rec, a, s);
                  continue;
                }
                const float dm = compose_step(rec, a, m, mode, s, v, compat);
                v[G_K] += m * dm;
                const V3 gq = quad_adjoint(rec, qf, -kk * dm, v + G_CTRL);
                if (GX) gx += gq;
                reduce_into<16>(v, row, lane);
              } else {
                float v[32];
    #pragma unroll
                for (int j = 0; j < 32; j++) v[j] = -0.f;
                CubicFwd cf;
                const float sdf = cubic_eval(rec, c.x, cf, base == B_CATMULL_ROM);
                const float kk = h.y * c.rinv;
                const float m = -sdf * kk;
                const float a = mode == STEP_HARD ? (sdf <= 0.f ? 1.f : 0.f) : soft_alpha(mode, m);
                const bool below = __all_sync(0xffffffffu, !c.active || a < L.skip_alpha);
                if (below || (kind & K_FROZEN)) {  // the kind word is warp-uniform
                  compose_skip(rec, a, s);
                  continue;
                }
                const float dm = compose_step(rec, a, m, mode, s, v, compat);
                const float dsdf = -kk * dm;
                v[G_K] += m * dm;
                V3 g = cubic_adjoint(rec, c.x, cf, dsdf, v + G_CTRL, compat, base == B_CATMULL_ROM);
                if (compat) g = g * dsdf;  // the reference multiplies by dL/dSDF again
                if (GX) gx += g;
                reduce_into<32>(v, row, lane);
              }
            }
          }
          if (c.active) {
            if (sc.last_pass) {
              if (GX) {
                L.grad_x[3 * c.si] = gx.x;
                L.grad_x[3 * c.si + 1] = gx.y;
                L.grad_x[3 * c.si + 2] = gx.z;
              }
            } else {
              float* b = L.bstate + 8 * c.si;
              b[0] = s.T; b[1] = s.Ps; b[2] = s.Pr; b[3] = s.Pg; b[4] = s.Pb;
              if (GX) {
                b[5] = gx.x; b[6] = gx.y; b[7] = gx.z;
              }
            }
          }
        }
      }
      if (lane == 0) item = atomicAdd(counter, L.rays_per_item);
      item = __shfl_sync(0xffffffffu, item, 0);
    }
    __syncthreads();  // every warp is done with the staged chunk
    flush(sci);
    if (threadIdx.x == 0) s_scene = next_scene(L);
    __syncthreads();
    sci = s_scene;
  }
  if (STATS && lane == 0 && bcount) atomicAdd(L.stats, bcount);
}

// ============================================================== ray kernels

// One warp per ray: volume rendering of the composited samples
// (render.py:29-48 compute_alpha_weights, 51-88 volumetric_rendering).
__global__ void ray_fwd_kernel(const RayLaunch L) {
  const long long ray = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (ray >= L.n_rays) return;
  const int N = L.n_samples;
  const float* td = L.tdist + ray * (N + 1);
  const float dn = sqrtf(L.dirs[3 * ray] * L.dirs[3 * ray] + L.dirs[3 * ray + 1] * L.dirs[3 * ray + 1] +
                         L.dirs[3 * ray + 2] * L.dirs[3 * ray + 2]);
  float carry = 0.f, acc = 0.f, r = 0.f, g = 0.f, b = 0.f, D = 0.f;
  for (int i0 = 0; i0 < N; i0 += 32) {
    const int i = i0 + lane;
    const bool on = i < N;
    float tau = 0.f, cr = 0.f, cg = 0.f, cb = 0.f, tm = 0.f;
    if (on) {
      const float* st = L.state + 5 * (ray * N + i);
      const float T = st[0], sig = st[1];
      const float inv = 1.0f / (1.0f + 1e-6f - T);
      cr = clampf(st[2] * inv, 0.f, 1.f);
      cg = clampf(st[3] * inv, 0.f, 1.f);
      cb = clampf(st[4] * inv, 0.f, 1.f);
      const float t0 = td[i], t1 = td[i + 1];
      tm = 0.5f * (t0 + t1);
      tau = sig * ((t1 - t0) * dn);
      if (L.opaque && i == N - 1) tau = __int_as_float(0x7f800000);
    }
    const float incl = warp_inclusive_scan(on && isfinite(tau) ? tau : 0.f, lane);
    const float excl = incl - (on && isfinite(tau) ? tau : 0.f);
    const float tr = expf(-(carry + excl));
    const float a = isinf(tau) ? 1.f : -expm1f(-tau);
    const float w = on ? a * tr : 0.f;
    acc += w;
    r += w * cr; g += w * cg; b += w * cb;
    D += w * tm;
    carry += __shfl_sync(0xffffffffu, incl, 31);
  }
  acc = warp_sum(acc);
  r = warp_sum(r); g = warp_sum(g); b = warp_sum(b);
  D = warp_sum(D);
  if (lane == 0) {
    const float bgw = fmaxf(1.f - acc, 0.f);
    float br = L.bg_value, bgg = L.bg_value, bb = L.bg_value;
    if (L.bg) { br = L.bg[3 * ray]; bgg = L.bg[3 * ray + 1]; bb = L.bg[3 * ray + 2]; }
    L.rgb[3 * ray] = r + bgw * br;
    L.rgb[3 * ray + 1] = g + bgw * bgg;
    L.rgb[3 * ray + 2] = b + bgw * bb;
    L.acc[ray] = acc;
    const float eps = 1.1920929e-07f;  // float32 machine epsilon (render.py:76)
    float val = D / fmaxf(acc, eps);
    if (isnan(val)) val = __int_as_float(0x7f800000);
    L.depth[ray] = clampf(val, td[0], td[N]);
  }
}

// One warp per ray: adjoint of the volume rendering, producing per-sample seeds
// g_sigma = dL/dsigma, g_C = dL/d(colour sum), g_T = dL/dT_final.
__global__ void ray_bwd_kernel(const RayLaunch L) {
  const long long ray = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (ray >= L.n_rays) return;
  const int N = L.n_samples;
  const float* td = L.tdist + ray * (N + 1);
  const float dn = sqrtf(L.dirs[3 * ray] * L.dirs[3 * ray] + L.dirs[3 * ray + 1] * L.dirs[3 * ray + 1] +
                         L.dirs[3 * ray + 2] * L.dirs[3 * ray + 2]);
  float grr = 0.f, grg = 0.f, grb = 0.f, gacc = 0.f, gdep = 0.f;
  if (L.g_rgb) { grr = L.g_rgb[3 * ray]; grg = L.g_rgb[3 * ray + 1]; grb = L.g_rgb[3 * ray + 2]; }
  if (L.g_acc) gacc = L.g_acc[ray];
  if (L.g_depth) gdep = L.g_depth[ray];
  float br = L.bg_value, bgg = L.bg_value, bb = L.bg_value;
  if (L.bg) { br = L.bg[3 * ray]; bgg = L.bg[3 * ray + 1]; bb = L.bg[3 * ray + 2]; }

  // Per-sample forward quantities (recomputed in each sweep).
  struct Smp { float w, tr_next, delta, cr, cg, cb, inv, tm, Cr, Cg, Cb; bool on, opq; };
  auto sample = [&](int i, float carry_in, float* incl_out) {
    Smp s;
    s.on = i < N;
    float tau = 0.f;
    s.cr = s.cg = s.cb = s.tm = s.delta = s.inv = s.Cr = s.Cg = s.Cb = 0.f;
    s.opq = false;
    if (s.on) {
      const float* st = L.state + 5 * (ray * N + i);
      const float T = st[0], sig = st[1];
      s.inv = 1.0f / (1.0f + 1e-6f - T);
      s.Cr = st[2]; s.Cg = st[3]; s.Cb = st[4];
      s.cr = clampf(s.Cr * s.inv, 0.f, 1.f);
      s.cg = clampf(s.Cg * s.inv, 0.f, 1.f);
      s.cb = clampf(s.Cb * s.inv, 0.f, 1.f);
      const float t0 = td[i], t1 = td[i + 1];
      s.tm = 0.5f * (t0 + t1);
      s.delta = (t1 - t0) * dn;
      tau = sig * s.delta;
      s.opq = L.opaque && i == N - 1;
    }
    const float ft = (s.on && !s.opq) ? tau : 0.f;
    const float incl = warp_inclusive_scan(ft, lane);
    const float excl = incl - ft;
    const float tr = expf(-(carry_in + excl));
    const float a = s.opq ? 1.f : -expm1f(-tau);
    s.w = s.on ? a * tr : 0.f;
    s.tr_next = s.opq ? 0.f : expf(-(carry_in + incl));
    *incl_out = __shfl_sync(0xffffffffu, incl, 31);
    return s;
  };

  // sweep 1: totals
  float carry = 0.f, acc = 0.f, D = 0.f;
  for (int i0 = 0; i0 < N; i0 += 32) {
    float tot;
    Smp s = sample(i0 + lane, carry, &tot);
    acc += s.w;
    D += s.w * s.tm;
    carry += tot;
  }
  acc = warp_sum(acc);
  D = warp_sum(D);
  const float eps = 1.1920929e-07f;
  float dacc = gacc;
  if (1.f - acc >= 0.f) dacc -= grr * br + grg * bgg + grb * bb;
  float gD = 0.f;
  {
    const float val = D / fmaxf(acc, eps);
    if (isfinite(val) && val >= td[0] && val <= td[N]) {
      gD = gdep / fmaxf(acc, eps);
      if (acc >= eps) dacc += -gdep * D / (acc * acc);
    }
  }
  // sweep 2: Z = sum_j dL/dw_j w_j
  carry = 0.f;
  float Z = 0.f;
  for (int i0 = 0; i0 < N; i0 += 32) {
    float tot;
    Smp s = sample(i0 + lane, carry, &tot);
    const float gw = dacc + grr * s.cr + grg * s.cg + grb * s.cb + gD * s.tm;
    Z += gw * s.w;
    carry += tot;
  }
  Z = warp_sum(Z);
  // sweep 3: seeds
  carry = 0.f;
  float zcarry = 0.f;
  for (int i0 = 0; i0 < N; i0 += 32) {
    const int i = i0 + lane;
    float tot;
    Smp s = sample(i, carry, &tot);
    const float gw = dacc + grr * s.cr + grg * s.cg + grb * s.cb + gD * s.tm;
    const float zi = warp_inclusive_scan(gw * s.w, lane);
    const float suffix = Z - (zcarry + zi);
    zcarry += __shfl_sync(0xffffffffu, zi, 31);
    carry += tot;
    if (s.on) {
      const float gtau = gw * s.tr_next - suffix;
      const float gsig = s.opq ? 0.f : gtau * s.delta;
      // colour normalisation c = clamp(C / O, 0, 1), O = 1 + 1e-6 - T
      const float mr = (s.Cr * s.inv >= 0.f && s.Cr * s.inv <= 1.f) ? 1.f : 0.f;
      const float mg = (s.Cg * s.inv >= 0.f && s.Cg * s.inv <= 1.f) ? 1.f : 0.f;
      const float mb = (s.Cb * s.inv >= 0.f && s.Cb * s.inv <= 1.f) ? 1.f : 0.f;
      const float dcr = mr * s.w * grr, dcg = mg * s.w * grg, dcb = mb * s.w * grb;
      float* sd = L.seeds + 5 * (ray * N + i);
      sd[0] = gsig;
      sd[1] = dcr * s.inv;
      sd[2] = dcg * s.inv;
      sd[3] = dcb * s.inv;
      sd[4] = (dcr * s.Cr + dcg * s.Cg + dcb * s.Cb) * s.inv * s.inv;
    }
  }
}

// ============================================================ prep/finalize

__global__ void prep_kernel(const PrepLaunch P) {
  const long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (s < P.n_counters) P.counters[s] = 0;
  if (P.mask_tag && s == 0) *P.mask_tag = P.mask_tag_value;
  if (P.stats && s < 18) P.stats[s] = 0ull;
  if (s >= P.n_strokes) return;
  if (P.gslots) {
    float* g = P.gslots + s * GRAD_SLOTS;
#pragma unroll
    for (int j = 0; j < GRAD_SLOTS; j++) g[j] = 0.f;
  }
  float* rec = P.recs + s * REC_FLOATS;
  const int wstate = window_state(P.window, P.n_win_scenes, P.win_begin, s);
  if (wstate == 2) {
    // Absent stroke (beyond its scene's active count): a culling sphere of radius
    // -inf keeps it out of every candidate set, and should a sample with NaN
    // coordinates reach it anyway, the record is a hard-step round cube whose SDF is
    // +1 everywhere (p = 0, radius -2) with a zero slope: alpha and every gradient
    // contribution are exactly 0. Its parameters are never read.
    for (int j = 0; j < REC_FLOATS; j++) rec[j] = 0.f;
    rec[R_KIND] = __int_as_float(B_ROUND_CUBE | (STEP_HARD << 8));
    rec[R_BP] = -2.f;
    P.cull_a[4 * s] = 0.f; P.cull_a[4 * s + 1] = 0.f; P.cull_a[4 * s + 2] = 0.f;
    P.cull_a[4 * s + 3] = __int_as_float(0xff800000);
    P.cull_b[s] = 0.f;
    return;
  }
  const int sid = P.sdf_ids ? P.sdf_ids[s] : P.uniform_sdf_id;
  const int base = (sid >> 4) & 15;
  const int flags = sid & 15;
  const float* prm = P.shape_params + s * (long long)P.param_stride;
  const int np = sdf_id_param_count(sid);
  const bool s1 = flags & F_S1;
  const bool s3 = !s1 && (flags & F_S3);
  if (!base_supported(base) || np > P.param_stride || sid < 0 || sid > 255 ||
      ((base > B_TETRAHEDRON) && flags != 0) || (P.base_mask && !((P.base_mask >> base) & 1u))) {
    // Unsupported stroke: flag it, never read its parameters, and make every
    // sample that meets it NaN (the culling sphere is infinite) so that the error
    // cannot pass silently.
    atomicOr(P.status, ST_BAD_KIND);
    for (int j = 0; j < REC_FLOATS; j++) rec[j] = 0.f;
    rec[R_KIND] = __int_as_float(B_CAPPED_TORUS | (STEP_LAPLACE << 8));
    rec[R_KFIX] = __int_as_float(0x7fc00000);
    P.cull_a[4 * s] = 0.f; P.cull_a[4 * s + 1] = 0.f; P.cull_a[4 * s + 2] = 0.f;
    P.cull_a[4 * s + 3] = __int_as_float(0x7f800000);
    P.cull_b[s] = 0.f;
    return;
  }
  const float delta = P.sdf_delta ? P.sdf_delta[s] : P.uniform_delta;
  const int mode = delta > 0.f ? (P.use_laplace ? STEP_LAPLACE : STEP_LINEAR) : STEP_HARD;
  const float kappa = P.use_laplace ? 2.f : 0.5f;
  int off = np;
  V3 t = v3(0.f, 0.f, 0.f), sc = v3(1.f, 1.f, 1.f);
  M3 R;
  R.r0 = v3(1.f, 0.f, 0.f); R.r1 = v3(0.f, 1.f, 0.f); R.r2 = v3(0.f, 0.f, 1.f);
  if (flags & F_T) { off -= 3; t = v3(prm[off], prm[off + 1], prm[off + 2]); }
  if (flags & F_R) { off -= 3; R = euler_matrix(v3(prm[off], prm[off + 1], prm[off + 2])); }
  if (s1) { off -= 1; sc = v3(prm[off], prm[off], prm[off]); }
  else if (s3) { off -= 3; sc = v3(prm[off], prm[off + 1], prm[off + 2]); }
  int kind = base | (flags << 4) | (mode << 8);
  const bool s1k = s1 && P.inv_scale_radius;
  const bool s3f = s3 && P.inv_scale_radius;
  if (s1k) kind |= K_S1K;
  if (s3f) kind |= K_S3FAC;
  if (wstate == 1) kind |= K_FROZEN;
  for (int j = 0; j < REC_FLOATS; j++) rec[j] = 0.f;
  rec[R_KIND] = __int_as_float(kind);
  const float* col = P.color_params + s * (long long)P.color_stride;
  rec[R_COLOR] = col[0];
  rec[R_COLOR + 1] = col[1];
  rec[R_COLOR + 2] = col[2];
  rec[R_DENSITY] = P.density ? P.density[s] : 0.f;
  rec[R_KFIX] = kappa / delta * (s1k ? sc.x : 1.f);
  rec[R_DELTA] = delta;

  // culling: sdf_local >= Lg (|p| - rho0) with p the local point; world centre cw
  float rho0 = 1.f, Lg = 1.f, smax = fmaxf(sc.x, fmaxf(sc.y, sc.z)), smin = fminf(sc.x, fminf(sc.y, sc.z));
  V3 cw = t;
  float Rb;
  bool bound_ok = true;  // false: no finite culling bound (the stroke is never culled)
  if (base <= B_TETRAHEDRON) {
    // M = S^-1 R^T: row i is column i of R divided by s_i; the row's w holds t_i
    const V3 mr[3] = {v3(R.r0.x, R.r1.x, R.r2.x) * (1.f / sc.x), v3(R.r0.y, R.r1.y, R.r2.y) * (1.f / sc.y),
                      v3(R.r0.z, R.r1.z, R.r2.z) * (1.f / sc.z)};
    for (int i = 0; i < 3; i++) {
      rec[R_M + 4 * i] = mr[i].x;
      rec[R_M + 4 * i + 1] = mr[i].y;
      rec[R_M + 4 * i + 2] = mr[i].z;
    }
    rec[R_M + 3] = t.x; rec[R_M + 7] = t.y; rec[R_M + 11] = t.z;
    rec[R_S] = sc.x; rec[R_S + 1] = sc.y; rec[R_S + 2] = sc.z;
    rec[R_SINV] = 1.f / sc.x; rec[R_SINV + 1] = 1.f / sc.y; rec[R_SINV + 2] = 1.f / sc.z;
    const float bp = base_param_count(base) > 0 ? prm[0] : 0.f;
    const float bp2 = base_param_count(base) > 1 ? prm[1] : 0.f;
    rec[R_BP] = bp;
    rec[R_BP2] = bp2;
    if (base == B_CAPPED_TORUS) {
      rec[R_TSIN] = sinf(bp);
      rec[R_TCOS] = cosf(bp);
    }
    // bounds sdf_local >= Lg (|p| - rho0): exact distances (Lg = 1) minus the largest
    // radius; for the polytopes, the facet-distance maximum over the gauge of the body
    // (inradius / circumradius)
    switch (base) {
      case B_SPHERE: rho0 = 1.f; Lg = 1.f; break;
      case B_CUBE: rho0 = 1.7320509f; Lg = 1.f; break;
      case B_ROUND_CUBE: rho0 = fmaxf(1.7320509f + bp, 0.f); Lg = 1.f; break;
      case B_CAPPED_TORUS: rho0 = 1.f + fmaxf(bp2, 0.f); Lg = 1.f; break;
      case B_CAPSULE: rho0 = 1.f + fabsf(bp); Lg = 1.f; break;
      case B_LINE: rho0 = fabsf(bp) + 1.f + fabsf(bp2); Lg = 1.f; break;
      case B_TRIPRISM: {
        const float rc = sqrtf(1.f + bp * bp);  // vertices (x, z) = (0, 1), (+-0.866, -0.5), |y| = h
        rho0 = rc;
        Lg = fminf(bp, 0.5f) / rc * 0.9999f;
        bound_ok = bp > 0.f;
        break;
      }
      case B_OCTAHEDRON: rho0 = 1.f; Lg = 0.5773502f; break;
      case B_TETRAHEDRON: rho0 = 1.7320511f; Lg = 0.3333333f; break;
      default: break;
    }
    Rb = smax * rho0;
  } else if (base == B_QUAD_BEZIER) {
    V3 A = v3(prm[0], prm[1], prm[2]), B = v3(prm[3], prm[4], prm[5]), C = v3(prm[6], prm[7], prm[8]);
    V3 a = B - A;
    V3 b = (A - B * 2.0f) + C;
    V3 c = a * 2.0f;
    for (int j = 0; j < 3; j++) {
      rec[R_QA + j] = (&A.x)[j];
      rec[R_Qa + j] = (&a.x)[j]; rec[R_Qb + j] = (&b.x)[j]; rec[R_Qc + j] = (&c.x)[j];
    }
    rec[R_QR1] = prm[9];
    rec[R_QR2] = prm[10];
    const float kk = 1.0f / dot(b, b);
    rec[R_QKK] = kk;
    rec[R_QKX] = kk * dot(a, b);
    rec[R_QAA2] = 2.0f * dot(a, a);
    rec[R_QAB] = dot(a, b);
    cw = (A + B + C) * (1.f / 3.f);
    float rc = fmaxf(sqrtf(dot(A - cw, A - cw)), fmaxf(sqrtf(dot(B - cw, B - cw)), sqrtf(dot(C - cw, C - cw))));
    Rb = rc + fmaxf(prm[9], prm[10]);
    smax = smin = 1.f;
    // 8 chords at t = k/8: curve-to-chord distance <= max|B''| dt^2 / 8 = |b| / 256
    rec[R_CTEST] = (fmaxf(prm[9], prm[10]) + sqrtf(dot(b, b)) * (1.f / 256.f)) * 1.0001f;
  } else {
    // cubic Bezier: the control points; Catmull-Rom: its power-basis coefficients
    // (A, B, C, D of t^3, t^2, t, 1, strokes_sdf.h:1340-1349). hull[] holds Bezier
    // control points of the same curve for the culling bound (convex-hull property).
    const bool power = base == B_CATMULL_ROM;
    V3 P4[4], hull[4];
    for (int k = 0; k < 4; k++) P4[k] = v3(prm[3 * k], prm[3 * k + 1], prm[3 * k + 2]);
    if (power) {
      const V3 p0 = P4[0], p1 = P4[1], p2 = P4[2], p3 = P4[3];
      const float t01 = sqrtf(sqrtf(dot(p0 - p1, p0 - p1)) + 1e-8f);
      const float t12 = sqrtf(sqrtf(dot(p1 - p2, p1 - p2)) + 1e-8f);
      const float t23 = sqrtf(sqrtf(dot(p2 - p3, p2 - p3)) + 1e-8f);
      const V3 m1 = (p2 - p1) + ((p1 - p0) / t01 - (p2 - p0) / (t01 + t12)) * t12;
      const V3 m2 = (p2 - p1) + ((p3 - p2) / t23 - (p3 - p1) / (t12 + t23)) * t12;
      P4[0] = (p1 - p2) * 2.0f + m1 + m2;
      P4[1] = (p2 - p1) * 3.0f - m1 * 2.0f - m2;
      P4[2] = m1;
      P4[3] = p1;
      hull[0] = p1;
      hull[1] = p1 + m1 * (1.f / 3.f);
      hull[2] = p2 - m2 * (1.f / 3.f);
      hull[3] = p2;
    } else {
      for (int k = 0; k < 4; k++) hull[k] = P4[k];
    }
    for (int k = 0; k < 4; k++) {
      rec[R_CA + 4 * k] = P4[k].x; rec[R_CA + 4 * k + 1] = P4[k].y; rec[R_CA + 4 * k + 2] = P4[k].z;
    }
    rec[R_CR1] = prm[12];
    rec[R_CR2] = prm[13];
    constexpr float step = 1.0f / CUBIC_SEGMENTS;
    for (int i = 0; i <= CUBIC_SEGMENTS; i++) {
      const float ti = i * step;
      float w[4];
      curve_weights(ti, w, power);
      V3 v = P4[0] * w[0] + P4[1] * w[1] + P4[2] * w[2] + P4[3] * w[3];
      rec[R_CV + 3 * i] = v.x; rec[R_CV + 3 * i + 1] = v.y; rec[R_CV + 3 * i + 2] = v.z;
    }
    // curve-to-polyline distance <= max|B''| dt^2 / 8, |B''| <= 6 max second difference
    // of the Bezier control points (the hull points of either curve)
    {
      const V3 d0 = (hull[0] - hull[1] * 2.f) + hull[2], d1 = (hull[1] - hull[2] * 2.f) + hull[3];
      const float dd = fmaxf(sqrtf(dot(d0, d0)), sqrtf(dot(d1, d1)));
      rec[R_CTEST] = (fmaxf(prm[12], prm[13]) + dd * (6.f * step * step / 8.f)) * 1.0001f;
    }
    cw = (hull[0] + hull[1] + hull[2] + hull[3]) * 0.25f;
    float rc = 0.f;
    for (int k = 0; k < 4; k++) rc = fmaxf(rc, sqrtf(dot(hull[k] - cw, hull[k] - cw)));
    // the polyline vertices are on the curve, inside the hull; the margin covers rounding
    Rb = rc * 1.0001f + fmaxf(prm[12], prm[13]);
    smax = smin = 1.f;
  }
  // margin per unit sample radius: the soft-step argument m = sdf * k exceeds the
  // cut m_cut (alpha = exp(-m_cut)/2) beyond Rb + cm * r.
  float cm = 0.f;
  bool cull = true;
  if (mode != STEP_HARD) {
    const float mcut = mode == STEP_LINEAR ? 0.5f : P.cull_m;
    if (mode == STEP_LAPLACE && P.cull_m < 0.f) cull = false;
    if (base > B_TETRAHEDRON) {
      cm = mcut * delta / kappa;
    } else if (s1) {
      cm = mcut * delta * (P.inv_scale_radius ? 1.f : sc.x) / (kappa * Lg);
    } else if (s3) {
      if (P.inv_scale_radius)
        cm = base == B_SPHERE ? mcut * delta / kappa : mcut * delta * smax / (kappa * Lg * smin);
      else
        cm = mcut * delta * smax / (kappa * Lg);
    } else {
      cm = mcut * delta / (kappa * Lg);
    }
  }
  if (!cull || !bound_ok) Rb = __int_as_float(0x7f800000);
  P.cull_a[4 * s] = cw.x; P.cull_a[4 * s + 1] = cw.y; P.cull_a[4 * s + 2] = cw.z;
  P.cull_a[4 * s + 3] = Rb * 1.0001f + 1e-6f;
  // Tetrahedra and octahedra without per-axis scale also get the exact polytope test
  // of cull_block (flagged by the margin's sign bit): their alpha reaches the cut only
  // where the local SDF is below tau_local = cm r Lg / s, i.e. inside the polytope
  // {gauge(p) <= 1 + sqrt(3) tau_local}, which fills 12 % (tetrahedron) / 32 %
  // (octahedron) of the bounding sphere.
  // (without culling the margin is meaningless, and may be negative: store 0 so that
  // the sign bit flags the polytope test alone)
  // Per-axis-scaled spheres (ellipsoids): alpha reaches the cut only where the local
  // radius |p| <= 1 + tau_local, tau_local = m_cut delta r / (kappa f) with the radius
  // factor f >= s_min under inv_scale_radius (f = 1 without it).
  // Capsules (h > 0) with one scale: the SDF is the exact distance to the axis segment
  // minus 1 (Lg = 1), so tau_local = cm / s per unit radius; the capsule fills 1/(h+1)^2
  // of its bounding sphere's cross-section. (A slab test for boxes culls 12 % of their
  // candidates and costs more than it saves: the batched pass reads 32 strokes'
  // records per lane, a bank conflict per record load.)
  const bool ell = base == B_SPHERE && s3 && cull && bound_ok;
  const bool cap = base == B_CAPSULE && rec[R_BP] > 0.f && !s3 && cull && bound_ok;
  const bool plane = ((base == B_OCTAHEDRON || base == B_TETRAHEDRON) && !s3 && cull && bound_ok) ||
                     (base >= B_QUAD_BEZIER && cull && bound_ok) || ell || cap;  // curves: the piece test
  if (plane && (base == B_OCTAHEDRON || base == B_TETRAHEDRON)) rec[R_PLANE] = 1.7320508f * cm * Lg / sc.x;
  if (cap) rec[R_PLANE] = cm * Lg / sc.x;
  if (ell) {
    const float mc = mode == STEP_HARD ? 0.f : (mode == STEP_LINEAR ? 0.5f : P.cull_m);
    rec[R_PLANE] = fmaxf(mc, 0.f) * delta / kappa / (P.inv_scale_radius ? smin : 1.f);
  }
  const float margin = (cull && bound_ok) ? fmaxf(cm, 0.f) * 1.0001f : 0.f;
  P.cull_b[s] = plane ? -margin : margin;
}

__device__ void prim_param_grads(const FinalizeLaunch& F, long long s, int base, int flags, const float* g,
                                 const float* rec, float* out);
__device__ void catmull_param_grads(const float* prm, const float* gc, int compat, float* out);

// Convert reduced slots into gradients of the raw reference-layout parameters.
__global__ void finalize_kernel(const FinalizeLaunch F) {
  const long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (s >= F.n_strokes) return;
  const float* g = F.gslots + s * GRAD_SLOTS;
  const float* rec = F.recs + s * REC_FLOATS;
  const int sid = F.sdf_ids ? F.sdf_ids[s] : F.uniform_sdf_id;
  const int base = (sid >> 4) & 15;
  const int flags = sid & 15;
  const bool acc = F.accumulate != 0;
  auto put = [&](float* dst, float v) { *dst = acc ? *dst + v : v; };
  if (window_state(F.window, F.n_win_scenes, F.win_begin, s) != 0) {
    // frozen or absent: no gradient
    float* gc = F.grad_color + s * (long long)F.color_stride;
    put(gc, 0.f); put(gc + 1, 0.f); put(gc + 2, 0.f);
    if (F.grad_density) put(F.grad_density + s, 0.f);
    if (F.grad_delta) put(F.grad_delta + s, 0.f);
    float* out = F.grad_shape + s * (long long)F.param_stride;
    for (int j = 0; j < F.param_stride; j++) put(out + j, 0.f);
    return;
  }
  float* gc = F.grad_color + s * (long long)F.color_stride;
  put(gc, g[G_COLOR]);
  put(gc + 1, g[G_COLOR + 1]);
  put(gc + 2, g[G_COLOR + 2]);
  if (F.grad_density) put(F.grad_density + s, g[G_DENSITY]);
  const float delta = F.sdf_delta ? F.sdf_delta[s] : F.uniform_delta;
  if (F.grad_delta) put(F.grad_delta + s, (delta > 0.f && !F.compat) ? -g[G_K] / delta : 0.f);
  float* out = F.grad_shape + s * (long long)F.param_stride;
  float o[64];
  for (int j = 0; j < F.param_stride && j < 64; j++) o[j] = 0.f;
  if (base == B_QUAD_BEZIER) {
    for (int j = 0; j < 11; j++) o[j] = g[G_CTRL + j];
  } else if (base == B_CUBIC_BEZIER) {
    for (int j = 0; j < 14; j++) o[j] = g[G_CTRL + j];
  } else if (base == B_CATMULL_ROM) {
    catmull_param_grads(F.shape_params + s * (long long)F.param_stride, g + G_CTRL, F.compat, o);
  } else if (base <= B_TETRAHEDRON) {
    prim_param_grads(F, s, base, flags, g, rec, o);
  }
  for (int j = 0; j < F.param_stride && j < 64; j++) put(out + j, o[j]);
}

// Primitive slots -> [base, scale (1|3), euler (3), translation (3)] gradients.
__device__ void prim_param_grads(const FinalizeLaunch& F, long long s, int base, int flags, const float* g,
                                 const float* rec, float* out) {
  const bool s1 = flags & F_S1;
  const bool s3 = !s1 && (flags & F_S3);
  int off = 0;
  const int nb = base_param_count(base);
  if (nb > 0) out[0] = g[G_BP];
  if (nb > 1) out[1] = g[G_BP2];
  off = nb;
  if (s1) { out[off] = g[G_SCALE]; off += 1; }
  else if (s3) { out[off] = g[G_SCALE]; out[off + 1] = g[G_SCALE + 1]; out[off + 2] = g[G_SCALE + 2]; off += 3; }
  if (flags & F_R) {
    const float* e = F.shape_params + s * (long long)F.param_stride + off;
    const float sx = sinf(e[0]), cx = cosf(e[0]), sy = sinf(e[1]), cy = cosf(e[1]);
    const float tx = g[G_TORQUE], ty = g[G_TORQUE + 1], tz = g[G_TORQUE + 2];
    // dL/de = w_k . torque with w_x = e_x, w_y = Rx^T e_y, w_z = R^T e_z
    out[off] = tx;
    out[off + 1] = cx * ty - sx * tz;
    out[off + 2] = -sy * tx + sx * cy * ty + cx * cy * tz;
    off += 3;
  }
  if (flags & F_T) {
    // dL/dt = -M^T sum g_p
    const float gx = g[G_GP], gy = g[G_GP + 1], gz = g[G_GP + 2];
    for (int j = 0; j < 3; j++)
      out[off + j] = -(rec[R_M + j] * gx + rec[R_M + 4 + j] * gy + rec[R_M + 8 + j] * gz);
  }
}

// Catmull-Rom: gradients of the power-basis coefficients (gc[0..11] = dL/dA, B, C, D;
// gc[12], gc[13] = dL/dr1, r2) -> gradients of the raw control points p0..p3 and radii.
// Exact: reverse mode through A = 2(p1 - p2) + m1 + m2, B = 3(p2 - p1) - 2 m1 - m2,
// C = m1, D = p1 and the centripetal tangents m1, m2 with knot gaps
// t_ij = sqrt(|p_i - p_j| + 1e-8). compat: the reference's formulas
// (strokes_sdf.h:1404-1437), which chain the knot gaps element-wise.
__device__ void catmull_param_grads(const float* prm, const float* gc, int compat, float* out) {
  const V3 p0 = ld3(prm), p1 = ld3(prm + 3), p2 = ld3(prm + 6), p3 = ld3(prm + 9);
  const V3 gA = ld3(gc), gB = ld3(gc + 3), gC = ld3(gc + 6), gD = ld3(gc + 9);
  const V3 d01 = p0 - p1, d12 = p1 - p2, d23 = p2 - p3;
  const float l01 = sqrtf(dot(d01, d01)), l12 = sqrtf(dot(d12, d12)), l23 = sqrtf(dot(d23, d23));
  const float t01 = sqrtf(l01 + 1e-8f), t12 = sqrtf(l12 + 1e-8f), t23 = sqrtf(l23 + 1e-8f);
  V3 g0, g1 = gA * 2.f - gB * 3.f + gD, g2 = gB * 3.f - gA * 2.f, g3;
  const V3 gm1 = gA - gB * 2.f + gC, gm2 = gA - gB;
  if (compat) {
    const float dm1_dp0 = t12 / (t01 + t12) - t12 / t01, dm1_dp1 = -1.f + t12 / t01,
                dm1_dp2 = 1.f - t12 / (t01 + t12), dm2_dp1 = -1.f + t12 / (t12 + t23),
                dm2_dp2 = 1.f - t12 / t23, dm2_dp3 = t12 / t23 - t12 / (t12 + t23);
    const V3 dm1_dt01 = ((p2 - p0) / ((t01 + t12) * (t01 + t12)) - (p1 - p0) / (t01 * t01)) * t12;
    const V3 dm1_dt12 = (p1 - p0) / t01 + (p2 - p0) * (t12 / ((t01 + t12) * (t01 + t12))) - (p2 - p0) / (t01 + t12);
    const V3 dm2_dt12 = (p2 - p1) / t23 + (p3 - p1) * (t12 / ((t12 + t23) * (t12 + t23))) - (p3 - p1) / (t12 + t23);
    const V3 dm2_dt23 = ((p2 - p3) / (t23 * t23) + (p3 - p1) / ((t12 + t23) * (t12 + t23))) * t12;
    const V3 dt01 = d01 / (2.f * powf(dot(d01, d01) + 1e-8f, 0.75f));
    const V3 dt12 = d12 / (2.f * powf(dot(d12, d12) + 1e-8f, 0.75f));
    const V3 dt23 = d23 / (2.f * powf(dot(d23, d23) + 1e-8f, 0.75f));
    g0 = gm1 * (dm1_dt01 * dt01 + dm1_dp0);
    g1 += gm1 * (dm1_dt12 * dt12 - dm1_dt01 * dt01 + dm1_dp1) + gm2 * (dm2_dt12 * dt12 + dm2_dp1);
    g2 += gm1 * (dm1_dp2 - dm1_dt12 * dt12) + gm2 * (dm2_dt23 * dt23 - dm2_dt12 * dt12 + dm2_dp2);
    g3 = gm2 * (dm2_dp3 - dm2_dt23 * dt23);
  } else {
    g0 = v3(0.f, 0.f, 0.f);
    g3 = v3(0.f, 0.f, 0.f);
    float gt01 = 0.f, gt12 = 0.f, gt23 = 0.f;
    // m1 = p2 - p1 + t12 (u - v), u = (p1 - p0) / t01, v = (p2 - p0) / (t01 + t12)
    {
      const V3 u = (p1 - p0) / t01, v = (p2 - p0) / (t01 + t12);
      g2 += gm1;
      g1 -= gm1;
      gt12 += dot(gm1, u - v);
      const V3 gu = gm1 * t12;
      g1 += gu / t01;
      g0 -= gu / t01;
      gt01 -= dot(gu, p1 - p0) / (t01 * t01);
      const float S = t01 + t12;
      g2 -= gu / S;
      g0 += gu / S;
      const float gS = dot(gu, p2 - p0) / (S * S);
      gt01 += gS;
      gt12 += gS;
    }
    // m2 = p2 - p1 + t12 (u2 - v2), u2 = (p3 - p2) / t23, v2 = (p3 - p1) / (t12 + t23)
    {
      const V3 u = (p3 - p2) / t23, v = (p3 - p1) / (t12 + t23);
      g2 += gm2;
      g1 -= gm2;
      gt12 += dot(gm2, u - v);
      const V3 gu = gm2 * t12;
      g3 += gu / t23;
      g2 -= gu / t23;
      gt23 -= dot(gu, p3 - p2) / (t23 * t23);
      const float S = t12 + t23;
      g3 -= gu / S;
      g1 += gu / S;
      const float gS = dot(gu, p3 - p1) / (S * S);
      gt12 += gS;
      gt23 += gS;
    }
    // t_ij = sqrt(|d_ij| + 1e-8), d_ij = p_i - p_j
    if (l01 > 0.f) { const V3 q = d01 * (gt01 / (2.f * t01 * l01)); g0 += q; g1 -= q; }
    if (l12 > 0.f) { const V3 q = d12 * (gt12 / (2.f * t12 * l12)); g1 += q; g2 -= q; }
    if (l23 > 0.f) { const V3 q = d23 * (gt23 / (2.f * t23 * l23)); g2 += q; g3 -= q; }
  }
  const V3 gs[4] = {g0, g1, g2, g3};
  for (int k = 0; k < 4; k++) {
    out[3 * k] = gs[k].x;
    out[3 * k + 1] = gs[k].y;
    out[3 * k + 2] = gs[k].z;
  }
  out[12] = gc[12];
  out[13] = gc[13];
}

// ================================================================ launchers

void launch_prep(const PrepLaunch& p, cudaStream_t st) {
  long long n = p.n_strokes > p.n_counters ? p.n_strokes : p.n_counters;
  if (n < 1) n = 1;
  const int threads = 128;
  prep_kernel<<<(unsigned)((n + threads - 1) / threads), threads, 0, st>>>(p);
}

template <int W, bool COMMON>
static cudaError_t launch_fwd_wc(const SegLaunch& L, int grid, size_t smem, cudaStream_t st) {
  auto* k = L.block_masks ? (L.stats ? seg_fwd_kernel<W, true, true, COMMON> : seg_fwd_kernel<W, true, false, COMMON>)
                          : (L.stats ? seg_fwd_kernel<W, false, true, COMMON> : seg_fwd_kernel<W, false, false, COMMON>);
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  k<<<grid, W * 32, smem, st>>>(L);
  return cudaGetLastError();
}
template <int W>
static cudaError_t launch_fwd_w(const SegLaunch& L, int grid, size_t smem, cudaStream_t st) {
  return L.common_only ? launch_fwd_wc<W, true>(L, grid, smem, st) : launch_fwd_wc<W, false>(L, grid, smem, st);
}
template <int W, bool STATS>
static cudaError_t launch_bwd_ws(const SegLaunch& L, int grid, size_t smem, cudaStream_t st) {
  auto* k = L.block_masks ? (L.compat ? (L.grad_x ? seg_bwd_kernel<W, true, 1, true, STATS>
                                                  : seg_bwd_kernel<W, false, 1, true, STATS>)
                                      : (L.grad_x ? seg_bwd_kernel<W, true, 0, true, STATS>
                                                  : seg_bwd_kernel<W, false, 0, true, STATS>))
                          : (L.compat ? (L.grad_x ? seg_bwd_kernel<W, true, 1, false, STATS>
                                                  : seg_bwd_kernel<W, false, 1, false, STATS>)
                                      : (L.grad_x ? seg_bwd_kernel<W, true, 0, false, STATS>
                                                  : seg_bwd_kernel<W, false, 0, false, STATS>));
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  k<<<grid, W * 32, smem, st>>>(L);
  return cudaGetLastError();
}
template <int W>
static cudaError_t launch_bwd_w(const SegLaunch& L, int grid, size_t smem, cudaStream_t st) {
  return L.stats ? launch_bwd_ws<W, true>(L, grid, smem, st) : launch_bwd_ws<W, false>(L, grid, smem, st);
}

cudaError_t launch_seg_fwd(const SegLaunch& L, int grid, int warps, size_t smem, cudaStream_t st) {
  switch (warps) {
    case 4: return launch_fwd_w<4>(L, grid, smem, st);
    case 8: return launch_fwd_w<8>(L, grid, smem, st);
    case 16: return launch_fwd_w<16>(L, grid, smem, st);
    case 24: return launch_fwd_w<24>(L, grid, smem, st);
    case 32: return launch_fwd_w<32>(L, grid, smem, st);
    default: return cudaErrorInvalidValue;
  }
}
cudaError_t launch_seg_bwd(const SegLaunch& L, int grid, int warps, size_t smem, cudaStream_t st) {
  switch (warps) {
    case 4: return launch_bwd_w<4>(L, grid, smem, st);
    case 8: return launch_bwd_w<8>(L, grid, smem, st);
    case 16: return launch_bwd_w<16>(L, grid, smem, st);
    case 20: return launch_bwd_w<20>(L, grid, smem, st);
    case 24: return launch_bwd_w<24>(L, grid, smem, st);
    case 32: return launch_bwd_w<32>(L, grid, smem, st);  // 64 registers, a small spill
    default: return cudaErrorInvalidValue;
  }
}

void launch_ray_fwd(const RayLaunch& L, cudaStream_t st) {
  const long long threads = L.n_rays * 32;
  const int bs = 256;
  ray_fwd_kernel<<<(unsigned)((threads + bs - 1) / bs), bs, 0, st>>>(L);
}
void launch_ray_bwd(const RayLaunch& L, cudaStream_t st) {
  const long long threads = L.n_rays * 32;
  const int bs = 256;
  ray_bwd_kernel<<<(unsigned)((threads + bs - 1) / bs), bs, 0, st>>>(L);
}
void launch_finalize(const FinalizeLaunch& L, cudaStream_t st) {
  const int bs = 128;
  finalize_kernel<<<(unsigned)((L.n_strokes + bs - 1) / bs), bs, 0, st>>>(L);
}

}  // namespace n3ds
