// C ABI of the stroke-field library: argument validation, workspace layout, pass
// planning and kernel dispatch. Allocates nothing; every launch goes to the caller's
// stream; no host synchronisation except in n3ds_field_read_status.
#include <algorithm>
#include <initializer_list>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/n3ds.h"
#include "n3ds_field.cuh"
#include "n3ds_record.cuh"
#include "n3ds_unfused.cuh"
#include "n3ds_adam.cuh"

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

#define N3DS_CUDA_TRY(expr)                                                              \
  do {                                                                                   \
    cudaError_t e_ = (expr);                                                             \
    if (e_ != cudaSuccess)                                                               \
      return fail(N3DS_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e_));   \
  } while (0)

struct DevInfo {
  int sms = 0;
  int smem_optin = 0;
};

DevInfo dev_info() {
  static DevInfo cache[64];
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) dev = 0;
  DevInfo& d = cache[dev];
  if (d.sms == 0) {
    cudaDeviceGetAttribute(&d.sms, cudaDevAttrMultiProcessorCount, dev);
    cudaDeviceGetAttribute(&d.smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (d.sms <= 0) d.sms = 148;
    if (d.smem_optin <= 0) d.smem_optin = 227 * 1024;
  }
  return d;
}

constexpr size_t align256(size_t v) { return (v + 255) & ~size_t(255); }

struct WsLayout {
  size_t recs, cull_a, cull_b, state, seeds, bstate, gslots, counters, masks, status, stats, mask_tag, total;
};
// Ray counters: one block of MAX_SCENES_PER_LAUNCH per segment-kernel launch, the
// first half for forward launches, the second for backward launches.
constexpr int N_LAUNCH_SLOTS = 64;
constexpr int N_COUNTERS = N_LAUNCH_SLOTS * n3ds::MAX_SCENES_PER_LAUNCH;

// Stroke-block mask words of a batch: per scene, segments x ceil(strokes / 32).
long long mask_words(const n3ds_batch_t* b) {
  const long long spr = (b->n_samples + 31) / 32;
  long long total = 0;
  for (int i = 0; i < b->n_scenes; i++) total += b->n_rays[i] * spr * ((b->n_strokes[i] + 31) / 32);
  return total;
}

WsLayout ws_layout(long long total_rays, int N, long long S, long long n_mask_words) {
  WsLayout w{};
  size_t off = 0;
  auto take = [&](size_t bytes) {
    size_t o = off;
    off = align256(off + bytes);
    return o;
  };
  const size_t P = size_t(total_rays) * size_t(N);
  // header: int32 status at +0, uint64 evaluated pairs at +8, uint64 per-base counts at
  // +16, uint64 backward-evaluated pairs at +144, int32 stroke-block mask tag at +248
  w.status = take(256);
  w.stats = w.status + 8;
  w.mask_tag = w.status + 248;
  w.recs = take(size_t(S) * n3ds::REC_FLOATS * 4);
  w.cull_a = take(size_t(S) * 16);
  w.cull_b = take(size_t(S + 4) * 4);
  w.state = take(P * 5 * 4);
  w.seeds = take(P * 5 * 4);
  w.bstate = take(P * 8 * 4);
  w.gslots = take(size_t(S) * n3ds::GRAD_SLOTS * 4);
  w.counters = take(N_COUNTERS * 4);
  w.masks = take(size_t(n_mask_words) * 4);
  w.total = off;
  return w;
}

struct Resolved {
  float cull_m, cull_alpha;
  int chunk_fwd, chunk_bwd, warps, schedule, grad_mode;
  int warps_fwd, warps_bwd;  // per direction (the forward segment kernel runs 24 warps by default)
  void* const* events;
  int forward_only;
  int count_pairs;
  unsigned long long wait_limit_ns;
  int test_stall;
  int rays_per_item;
};

void record_event(const Resolved& rv, int i, cudaStream_t st) {
  if (rv.events && rv.events[i]) cudaEventRecord(static_cast<cudaEvent_t>(rv.events[i]), st);
}

Resolved resolve(const n3ds_options_t* o) {
  n3ds_options_t d;
  n3ds_default_options(&d);
  if (!o) o = &d;
  Resolved r;
  // alpha = exp(-m)/2 beyond the cut: m_cut = -ln(2 alpha_cut)
  r.cull_m = o->cull_alpha > 0.f ? -logf(2.f * o->cull_alpha) : -1.f;
  if (o->cull_alpha > 0.f && r.cull_m < 0.f) r.cull_m = 0.f;
  const DevInfo di = dev_info();
  r.cull_alpha = o->cull_alpha > 0.f ? o->cull_alpha : 0.f;
  r.warps = o->warps > 0 ? o->warps : 16;
  r.schedule = o->schedule == N3DS_SCHEDULE_RUNS ? N3DS_SCHEDULE_RUNS : N3DS_SCHEDULE_SEGMENTS;
  const bool runs = r.schedule == N3DS_SCHEDULE_RUNS;
  // 24 warps only for the forward segment kernel (76 registers); the others hold
  // 100+ registers per thread and run at most 16
  // instantiated CTA sizes: segment forward 4-32 warps (64 registers), segment backward
  // 4-24 (94 registers at 20 warps, 80 with a small spill at 24), run kernels 4-16
  // largest instantiated CTA size not above the request
  auto pick = [](int w, std::initializer_list<int> sizes) {
    int best = 4;
    for (int s : sizes)
      if (s <= w && s > best) best = s;
    return best;
  };
  // defaults: the fastest measured on the benchmark workloads (32 / 24 for segments)
  const int wf = o->warps > 0 ? o->warps : (runs ? 16 : 32);
  const int wb = o->warps_bwd > 0 ? o->warps_bwd : (runs ? 16 : 24);
  r.warps_fwd = runs ? pick(wf, {4, 8, 16}) : pick(wf, {4, 8, 16, 24, 32});
  r.warps_bwd = runs ? pick(wb, {4, 8, 16}) : pick(wb, {4, 8, 16, 20, 24, 32});
  r.warps = r.warps_bwd;
  const size_t budget = size_t(di.smem_optin) - 256;  // room for static shared memory
  // default stages: the largest multiple of 32 strokes that fits the shared memory
  // (multiples of 32, so that the 32-stroke blocks of every pass line up with the
  // stroke-block mask words in both directions)
  // (at most 1024 = 32 blocks of 32: the forward keeps one block's mask per lane)
  int cf = o->chunk_fwd > 0 ? std::min(1024, std::max(32, o->chunk_fwd / 32 * 32)) : 1024;
  int cb = o->chunk_bwd > 0 ? std::min(1024, std::max(32, o->chunk_bwd / 32 * 32)) : 1024;
  auto fwd_smem = [&](int c) { return runs ? n3ds::run_fwd_smem(c, r.warps_fwd) : n3ds::seg_fwd_smem(c, r.warps_fwd); };
  auto bwd_smem = [&](int c) { return runs ? n3ds::run_bwd_smem(c, r.warps_bwd) : n3ds::seg_bwd_smem(c); };
  while (cf > 32 && fwd_smem(cf) > budget) cf -= 32;
  while (cb > 32 && bwd_smem(cb) > budget) cb -= 32;
  r.chunk_fwd = cf;
  r.chunk_bwd = cb;
  r.grad_mode = o->grad_mode;
  r.forward_only = o->forward_only != 0;
  r.count_pairs = o->count_pairs != 0;
  r.events = o->timing_events;
  r.wait_limit_ns = o->wait_limit_us > 0 ? (unsigned long long)o->wait_limit_us * 1000ull : 1000000000ull;
  r.test_stall = o->test_stall_staging != 0;
  r.rays_per_item = o->rays_per_item >= 4 ? 4 : (o->rays_per_item >= 2 ? 2 : 1);
  return r;
}

int check_batch(const n3ds_batch_t* b, long long* total_rays, long long* total_strokes) {
  if (!b || b->n_scenes < 1 || !b->n_rays || !b->n_strokes)
    return fail(N3DS_ERR_INVALID, "batch: n_scenes >= 1 and host n_rays / n_strokes arrays required");
  if (b->n_samples < 1) return fail(N3DS_ERR_INVALID, "batch: n_samples must be >= 1");
  long long R = 0, S = 0;
  for (int i = 0; i < b->n_scenes; i++) {
    if (b->n_rays[i] < 0 || b->n_strokes[i] < 0)
      return fail(N3DS_ERR_INVALID, "batch: negative ray or stroke count");
    if (b->n_rays[i] * ((b->n_samples + 31) / 32) > 0x7fffffffLL)
      return fail(N3DS_ERR_INVALID, "batch: too many segments in one scene");
    R += b->n_rays[i];
    S += b->n_strokes[i];
  }
  if (S > 0x7fffffffLL) return fail(N3DS_ERR_INVALID, "batch: too many strokes");
  *total_rays = R;
  *total_strokes = S;
  return N3DS_OK;
}

// Plan and launch the segment passes of one direction.
int run_seg_passes(bool backward, const n3ds_batch_t* b, const Resolved& rv, n3ds::SegLaunch base,
                   int counter_base, cudaStream_t st, int* launch_count = nullptr) {
  const int cap = backward ? rv.chunk_bwd : rv.chunk_fwd;
  const int spr = (b->n_samples + 31) / 32;
  const bool runs = rv.schedule == N3DS_SCHEDULE_RUNS;
  // work items per ray: the whole ray (segments) or 64-sample units (runs)
  const int ipr = runs ? (b->n_samples + n3ds::RUN_UNIT_SAMPLES - 1) / n3ds::RUN_UNIT_SAMPLES : 1;
  std::vector<long long> ray_begin(b->n_scenes), stroke_begin(b->n_scenes), mask_begin(b->n_scenes);
  std::vector<int> nch(b->n_scenes);
  long long r0 = 0, s0 = 0, m0 = 0;
  int passes = 1;
  for (int i = 0; i < b->n_scenes; i++) {
    ray_begin[i] = r0;
    stroke_begin[i] = s0;
    mask_begin[i] = m0;
    m0 += b->n_rays[i] * spr * ((b->n_strokes[i] + 31) / 32);
    r0 += b->n_rays[i];
    s0 += b->n_strokes[i];
    nch[i] = std::max(1, (b->n_strokes[i] + cap - 1) / cap);
    passes = std::max(passes, nch[i]);
  }
  const DevInfo di = dev_info();
  const int warps = backward ? rv.warps_bwd : rv.warps_fwd;
  const size_t smem = runs ? (backward ? n3ds::run_bwd_smem(cap, warps) : n3ds::run_fwd_smem(cap, warps))
                           : (backward ? n3ds::seg_bwd_smem(cap) : n3ds::seg_fwd_smem(cap, warps));
  int counter = 0;
  for (int pass = 0; pass < passes; pass++) {
    std::vector<int> scenes;
    for (int i = 0; i < b->n_scenes; i++)
      if (nch[i] > pass && b->n_rays[i] > 0) scenes.push_back(i);
    for (size_t g = 0; g < scenes.size(); g += n3ds::MAX_SCENES_PER_LAUNCH) {
      n3ds::SegLaunch L = base;
      L.chunk_cap = cap;
      L.segs_per_ray = spr;
      L.schedule = rv.schedule;
      L.n_scenes = 0;
      long long tiles = 0;
      double work_total = 0.0;
      std::vector<double> work;
      for (size_t k = g; k < scenes.size() && k < g + n3ds::MAX_SCENES_PER_LAUNCH; k++) {
        const int i = scenes[k];
        n3ds::SceneDesc& d = L.sc[L.n_scenes++];
        d.ray_begin = ray_begin[i];
        d.n_rays = (int)b->n_rays[i];
        d.stroke_begin = (int)stroke_begin[i];
        d.n_strokes = b->n_strokes[i];
        const int hi = b->n_strokes[i] - pass * cap;
        const int lo = std::max(0, hi - cap);
        d.chunk_lo = lo;
        d.chunk_n = std::max(0, hi - lo);
        d.first_pass = pass == 0;
        d.last_pass = pass == nch[i] - 1;
        d.mask_words = (b->n_strokes[i] + 31) / 32;
        d.mask_begin = mask_begin[i];
        if ((long long)d.n_rays * ipr > 0x7fffffffLL)
          return fail(N3DS_ERR_INVALID, "too many rays in one scene for 32-bit work counters");
        tiles += (long long)d.n_rays * ipr;
        // cost model: per ray, a fixed part (loads, segment setup) worth ~16 strokes
        // plus the culling and evaluation of the chunk
        work.push_back(double(d.n_rays) * double(d.chunk_n + 16));
        work_total += work.back();
      }
      if (tiles == 0) continue;
      if (counter >= N_LAUNCH_SLOTS / 2)
        return fail(N3DS_ERR_INVALID, "batch needs too many launches (raise chunk size or split the batch)");
      if (launch_count) {  // planning only
        ++*launch_count;
        continue;
      }
      L.tiles_total = (int)std::min<long long>(tiles, 0x7fffffffLL);
      L.tile_counter = base.tile_counter + (counter_base + counter++) * n3ds::MAX_SCENES_PER_LAUNCH;
      const int grid = (int)std::min<long long>(tiles, di.sms);
      // scene affinity: scene k's home CTAs start at its work prefix x grid
      double prefix = 0.0;
      for (int k = 0; k < L.n_scenes; k++) {
        L.sc[k].home_lo = (int)std::lround(prefix / work_total * grid);
        prefix += work[k];
      }
      cudaError_t e = runs ? (backward ? n3ds::launch_run_bwd(L, grid, warps, smem, st)
                                       : n3ds::launch_run_fwd(L, grid, warps, smem, st))
                           : (backward ? n3ds::launch_seg_bwd(L, grid, warps, smem, st)
                                       : n3ds::launch_seg_fwd(L, grid, warps, smem, st));
      if (e != cudaSuccess) return fail(N3DS_ERR_CUDA, std::string("segment kernel launch: ") + cudaGetErrorString(e));
    }
  }
  return N3DS_OK;
}

}  // namespace

namespace n3ds {
// Error reporting for entry points defined in other translation units.
int report_error(int code, const std::string& msg) { return fail(code, msg); }
}  // namespace n3ds

extern "C" {

const char* n3ds_last_error(void) { return g_last_error.c_str(); }
int n3ds_version(void) { return 100; }

void n3ds_default_options(n3ds_options_t* opt) {
  if (!opt) return;
  opt->cull_alpha = 1e-9f;
  opt->chunk_fwd = 0;
  opt->chunk_bwd = 0;
  opt->warps = 0;
  opt->schedule = 0;
  opt->grad_mode = N3DS_GRAD_EXACT;
  opt->timing_events = nullptr;
  opt->warps_bwd = 0;
  opt->forward_only = 0;
  opt->count_pairs = 0;
  opt->wait_limit_us = 0;
  opt->test_stall_staging = 0;
  opt->rays_per_item = 0;
}

size_t n3ds_field_workspace_bytes(const n3ds_batch_t* batch, const n3ds_options_t* opt) {
  (void)opt;
  long long R = 0, S = 0;
  if (check_batch(batch, &R, &S) != N3DS_OK) return 0;
  return ws_layout(R, batch->n_samples, S, mask_words(batch)).total;
}

static int field_common(const n3ds_batch_t* batch, const n3ds_rays_t* rays, const n3ds_strokes_t* strokes,
                        void* ws, size_t ws_bytes, long long* R, long long* S, WsLayout* lay) {
  int rc = check_batch(batch, R, S);
  if (rc) return rc;
  if (!rays || (*R > 0 && (!rays->tdist || !rays->dirs)))
    return fail(N3DS_ERR_INVALID, "rays: tdist and dirs are required");
  if (*R > 0 && !(rays->x ? rays->radius != nullptr : (rays->origins && rays->radii)))
    return fail(N3DS_ERR_INVALID, "rays: x and radius, or origins and radii (samples cast in-kernel), are required");
  if (!strokes || (*S > 0 && (!strokes->sdf_ids || !strokes->shape_params || !strokes->color_params ||
                              !strokes->density || !strokes->sdf_delta)))
    return fail(N3DS_ERR_INVALID, "strokes: sdf_ids, shape_params, color_params, density, sdf_delta required");
  if (*S > 0 && (strokes->param_stride < 1 || strokes->param_stride > 64))
    return fail(N3DS_ERR_INVALID, "strokes: param_stride must be in [1, 64]");
  if (strokes && strokes->stroke_window && batch->n_scenes > n3ds::MAX_SCENES_PER_LAUNCH)
    return fail(N3DS_ERR_UNSUPPORTED, "strokes: a stroke window covers at most " +
                                          std::to_string(n3ds::MAX_SCENES_PER_LAUNCH) + " scenes");
  *lay = ws_layout(*R, batch->n_samples, *S, mask_words(batch));
  if (!ws || ws_bytes < lay->total)
    return fail(N3DS_ERR_WORKSPACE, "workspace too small: need " + std::to_string(lay->total) + " bytes");
  if (reinterpret_cast<uintptr_t>(ws) % 256)
    return fail(N3DS_ERR_INVALID, "workspace must be 256-byte aligned");
  return N3DS_OK;
}

// Stroke window of a batch (at most MAX_SCENES_PER_LAUNCH scenes): the device pairs
// and the scenes' stroke offsets.
static void fill_window(const n3ds_batch_t* b, const n3ds_strokes_t* s, const int** window, int* n_scenes,
                        int* begin) {
  *window = s->stroke_window;
  *n_scenes = 0;
  if (!s->stroke_window) return;
  *n_scenes = b->n_scenes;
  int off = 0;
  for (int i = 0; i < b->n_scenes; i++) {
    begin[i] = off;
    off += b->n_strokes[i];
  }
  begin[b->n_scenes] = off;
}

static n3ds::PrepLaunch make_prep(const n3ds_strokes_t* s, long long S, const Resolved& rv, char* ws,
                                  const WsLayout& lay, bool zero_slots) {
  n3ds::PrepLaunch p{};
  p.sdf_ids = s->sdf_ids;
  p.uniform_sdf_id = -1;
  p.shape_params = s->shape_params;
  p.param_stride = s->param_stride;
  p.color_params = s->color_params;
  p.color_stride = 3;
  p.density = s->density;
  p.sdf_delta = s->sdf_delta;
  p.use_laplace = s->use_laplace_transform;
  p.inv_scale_radius = s->inv_scale_radius;
  p.cull_m = rv.cull_m;
  p.n_strokes = S;
  p.recs = reinterpret_cast<float*>(ws + lay.recs);
  p.cull_a = reinterpret_cast<float*>(ws + lay.cull_a);
  p.cull_b = reinterpret_cast<float*>(ws + lay.cull_b);
  p.status = reinterpret_cast<int*>(ws + lay.status);
  p.counters = reinterpret_cast<int*>(ws + lay.counters);
  p.n_counters = N_COUNTERS;
  p.gslots = zero_slots ? reinterpret_cast<float*>(ws + lay.gslots) : nullptr;
  p.stats = zero_slots ? nullptr : reinterpret_cast<unsigned long long*>(ws + lay.stats);
  if (!zero_slots) {
    // forward: tag the stroke-block masks the segment kernels are about to write with
    // the skip threshold they use (the run schedule writes none)
    p.mask_tag = reinterpret_cast<int*>(ws + lay.mask_tag);
    float tag = rv.cull_alpha;
    int bits;
    std::memcpy(&bits, &tag, sizeof(bits));
    p.mask_tag_value = (rv.schedule == N3DS_SCHEDULE_SEGMENTS && !rv.forward_only) ? bits : -1;
  }
  return p;
}

static n3ds::SegLaunch make_seg(const n3ds_batch_t* b, const n3ds_rays_t* rays, char* ws, const WsLayout& lay,
                                int compat) {
  n3ds::SegLaunch L{};
  L.x = rays->x;
  L.radius = rays->radius;
  L.origins = rays->origins;
  L.dirs = rays->dirs;
  L.tdist = rays->tdist;
  L.radii = rays->radii;
  L.n_samples = b->n_samples;
  L.recs = reinterpret_cast<const float*>(ws + lay.recs);
  L.cull_a = reinterpret_cast<const float*>(ws + lay.cull_a);
  L.cull_b = reinterpret_cast<const float*>(ws + lay.cull_b);
  L.state = reinterpret_cast<float*>(ws + lay.state);
  L.seeds = reinterpret_cast<const float*>(ws + lay.seeds);
  L.bstate = reinterpret_cast<float*>(ws + lay.bstate);
  L.gslots = reinterpret_cast<float*>(ws + lay.gslots);
  L.compat = compat;
  L.tile_counter = reinterpret_cast<int*>(ws + lay.counters);
  L.status = reinterpret_cast<int*>(ws + lay.status);
  L.stats = reinterpret_cast<unsigned long long*>(ws + lay.stats);
  L.block_masks = reinterpret_cast<unsigned*>(ws + lay.masks);
  L.mask_tag = reinterpret_cast<const int*>(ws + lay.mask_tag);
  L.wait_limit_ns = 1000000000ull;  // one second unless the options say otherwise
  L.test_stall = 0;
  L.rays_per_item = 1;
  return L;
}

static n3ds::RayLaunch make_ray(const n3ds_batch_t* b, const n3ds_rays_t* rays, char* ws, const WsLayout& lay,
                                long long R) {
  n3ds::RayLaunch L{};
  L.state = reinterpret_cast<const float*>(ws + lay.state);
  L.tdist = rays->tdist;
  L.dirs = rays->dirs;
  L.bg = rays->bg;
  L.bg_value = rays->bg_value;
  L.opaque = rays->opaque_background;
  L.n_rays = R;
  L.n_samples = b->n_samples;
  L.seeds = reinterpret_cast<float*>(ws + lay.seeds);
  return L;
}

int n3ds_field_forward(const n3ds_batch_t* batch, const n3ds_rays_t* rays, const n3ds_strokes_t* strokes,
                       const n3ds_options_t* opt, float* rgb, float* acc, float* depth, void* workspace,
                       size_t workspace_bytes, n3ds_stream_t stream) {
  long long R, S;
  WsLayout lay;
  int rc = field_common(batch, rays, strokes, workspace, workspace_bytes, &R, &S, &lay);
  if (rc) return rc;
  if (R > 0 && (!rgb || !acc || !depth)) return fail(N3DS_ERR_INVALID, "rgb, acc and depth outputs are required");
  const Resolved rv = resolve(opt);
  if (strokes->stroke_window && rv.schedule != N3DS_SCHEDULE_SEGMENTS)
    return fail(N3DS_ERR_UNSUPPORTED, "a stroke window needs the segment schedule");
  char* ws = static_cast<char*>(workspace);
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  // the status word covers one forward and the backward after it (the prep kernel
  // sets bits of it, so it is cleared before that kernel rather than by it)
  N3DS_CUDA_TRY(cudaMemsetAsync(ws + lay.status, 0, sizeof(int32_t), st));
  n3ds::PrepLaunch prep = make_prep(strokes, S, rv, ws, lay, false);
  fill_window(batch, strokes, &prep.window, &prep.n_win_scenes, prep.win_begin);
  prep.base_mask = strokes->base_mask;
  n3ds::launch_prep(prep, st);
  N3DS_CUDA_TRY(cudaGetLastError());
  record_event(rv, 0, st);
  n3ds::SegLaunch FL = make_seg(batch, rays, ws, lay, 0);
  FL.wait_limit_ns = rv.wait_limit_ns;
  FL.test_stall = rv.test_stall;
  FL.rays_per_item = rv.rays_per_item;
  FL.common_only = strokes->base_mask != 0 && (strokes->base_mask & ~n3ds::COMMON_BASES) == 0;
  FL.skip_alpha = rv.cull_alpha;
  if (!rv.count_pairs) FL.stats = nullptr;
  if (rv.forward_only || rv.schedule != N3DS_SCHEDULE_SEGMENTS) {
    FL.block_masks = nullptr;
  } else if (lay.masks < lay.total) {
    // the segment kernels store only non-empty mask words
    N3DS_CUDA_TRY(cudaMemsetAsync(ws + lay.masks, 0, lay.total - lay.masks, st));
  }
  rc = run_seg_passes(false, batch, rv, FL, 0, st);
  if (rc) return rc;
  record_event(rv, 1, st);
  if (R > 0) {
    n3ds::RayLaunch L = make_ray(batch, rays, ws, lay, R);
    L.rgb = rgb;
    L.acc = acc;
    L.depth = depth;
    n3ds::launch_ray_fwd(L, st);
    N3DS_CUDA_TRY(cudaGetLastError());
  }
  return N3DS_OK;
}

int n3ds_field_backward(const n3ds_batch_t* batch, const n3ds_rays_t* rays, const n3ds_strokes_t* strokes,
                        const n3ds_options_t* opt, const float* grad_rgb, const float* grad_acc,
                        const float* grad_depth, float* grad_x, float* grad_shape, float* grad_color,
                        float* grad_density, float* grad_sdf_delta, void* workspace, size_t workspace_bytes,
                        n3ds_stream_t stream) {
  long long R, S;
  WsLayout lay;
  int rc = field_common(batch, rays, strokes, workspace, workspace_bytes, &R, &S, &lay);
  if (rc) return rc;
  if (S > 0 && (!grad_shape || !grad_color || !grad_density))
    return fail(N3DS_ERR_INVALID, "grad_shape, grad_color and grad_density outputs are required");
  const Resolved rv = resolve(opt);
  if (strokes->stroke_window && rv.schedule != N3DS_SCHEDULE_SEGMENTS)
    return fail(N3DS_ERR_UNSUPPORTED, "a stroke window needs the segment schedule");
  const int compat = rv.grad_mode == N3DS_GRAD_COMPAT;
  char* ws = static_cast<char*>(workspace);
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  n3ds::PrepLaunch prep = make_prep(strokes, S, rv, ws, lay, true);
  fill_window(batch, strokes, &prep.window, &prep.n_win_scenes, prep.win_begin);
  prep.base_mask = strokes->base_mask;
  n3ds::launch_prep(prep, st);
  N3DS_CUDA_TRY(cudaGetLastError());
  if (R > 0) {
    n3ds::RayLaunch L = make_ray(batch, rays, ws, lay, R);
    L.g_rgb = grad_rgb;
    L.g_acc = grad_acc;
    L.g_depth = grad_depth;
    n3ds::launch_ray_bwd(L, st);
    N3DS_CUDA_TRY(cudaGetLastError());
  }
  n3ds::SegLaunch SL = make_seg(batch, rays, ws, lay, compat);
  SL.wait_limit_ns = rv.wait_limit_ns;
  SL.test_stall = rv.test_stall;
  SL.rays_per_item = rv.rays_per_item;
  SL.grad_x = grad_x;
  SL.stats = rv.count_pairs ? reinterpret_cast<unsigned long long*>(ws + lay.stats) + 17 : nullptr;  // pairs
  SL.skip_alpha = rv.cull_alpha;
  record_event(rv, 2, st);
  rc = run_seg_passes(true, batch, rv, SL, N_LAUNCH_SLOTS / 2, st);
  if (rc) return rc;
  record_event(rv, 3, st);
  if (S > 0) {
    n3ds::FinalizeLaunch F{};
    F.sdf_ids = strokes->sdf_ids;
    F.shape_params = strokes->shape_params;
    F.param_stride = strokes->param_stride;
    F.sdf_delta = strokes->sdf_delta;
    F.recs = reinterpret_cast<const float*>(ws + lay.recs);
    F.gslots = reinterpret_cast<const float*>(ws + lay.gslots);
    F.n_strokes = S;
    F.compat = compat;
    F.grad_shape = grad_shape;
    F.grad_color = grad_color;
    F.grad_density = grad_density;
    F.grad_delta = grad_sdf_delta;
    F.accumulate = 0;
    F.color_stride = 3;
    fill_window(batch, strokes, &F.window, &F.n_win_scenes, F.win_begin);
    n3ds::launch_finalize(F, st);
    N3DS_CUDA_TRY(cudaGetLastError());
  }
  return N3DS_OK;
}

int n3ds_compose_mode_forward(int mode, float* density_out, float* color_out, const float* alphas,
                              const float* colors, const float* density_params, int64_t n_points,
                              int64_t n_strokes, int64_t color_dim, n3ds_stream_t stream) {
  if (mode < N3DS_COMPOSE_MAX || mode > N3DS_COMPOSE_SOFTMAX_DENSITY_WEIGHTED)
    return fail(N3DS_ERR_INVALID, "unknown composition mode " + std::to_string(mode));
  if (color_dim != 1 && color_dim != 3) return fail(N3DS_ERR_INVALID, "Unsupported color dimension");
  if (n_points < 0 || n_strokes < 0) return fail(N3DS_ERR_INVALID, "negative size");
  if (n_points == 0) return N3DS_OK;
  if (!density_out || !color_out || (n_strokes > 0 && (!alphas || !colors || !density_params)))
    return fail(N3DS_ERR_INVALID, "null tensor pointer");
  N3DS_CUDA_TRY(n3ds::launch_compose_mode_fwd(mode, density_out, color_out, alphas, colors, density_params, n_points,
                                              n_strokes, (int)color_dim, reinterpret_cast<cudaStream_t>(stream)));
  return N3DS_OK;
}

int n3ds_compose_mode_backward(int mode, float* grad_alphas, float* grad_colors, float* grad_density_params,
                               const float* grad_density_out, const float* grad_color_out, const float* alphas,
                               const float* colors, const float* density_params, int64_t n_points,
                               int64_t n_strokes, int64_t color_dim, n3ds_stream_t stream) {
  if (mode < N3DS_COMPOSE_MAX || mode > N3DS_COMPOSE_SOFTMAX_DENSITY_WEIGHTED)
    return fail(N3DS_ERR_INVALID, "unknown composition mode " + std::to_string(mode));
  if (color_dim != 1 && color_dim != 3) return fail(N3DS_ERR_INVALID, "Unsupported color dimension");
  if (n_points < 0 || n_strokes < 0) return fail(N3DS_ERR_INVALID, "negative size");
  if (n_points == 0 || n_strokes == 0) return N3DS_OK;
  if (!grad_alphas || !grad_colors || !grad_density_params || !alphas || !colors || !density_params)
    return fail(N3DS_ERR_INVALID, "null tensor pointer");
  N3DS_CUDA_TRY(n3ds::launch_compose_mode_bwd(mode, grad_alphas, grad_colors, grad_density_params, grad_density_out,
                                              grad_color_out, alphas, colors, density_params, n_points, n_strokes,
                                              (int)color_dim, reinterpret_cast<cudaStream_t>(stream)));
  return N3DS_OK;
}

int n3ds_field_resolve_options(const n3ds_options_t* opt, n3ds_options_t* out) {
  if (!out) return fail(N3DS_ERR_INVALID, "out is required");
  n3ds_options_t d;
  n3ds_default_options(&d);
  const n3ds_options_t* o = opt ? opt : &d;
  const Resolved rv = resolve(o);
  *out = *o;
  out->chunk_fwd = rv.chunk_fwd;
  out->chunk_bwd = rv.chunk_bwd;
  out->warps = rv.warps_fwd;
  out->warps_bwd = rv.warps_bwd;
  out->schedule = rv.schedule;
  out->grad_mode = rv.grad_mode;
  out->rays_per_item = rv.rays_per_item;
  return N3DS_OK;
}

int n3ds_field_launch_count(const n3ds_batch_t* batch, const n3ds_options_t* opt, int32_t* forward,
                            int32_t* backward) {
  long long R = 0, S = 0;
  int rc = check_batch(batch, &R, &S);
  if (rc) return rc;
  const Resolved rv = resolve(opt);
  int f = 0, b = 0;
  n3ds::SegLaunch dummy{};
  run_seg_passes(false, batch, rv, dummy, 0, nullptr, &f);
  run_seg_passes(true, batch, rv, dummy, 0, nullptr, &b);
  // forward: prep + segment passes + ray render; backward: prep + ray adjoint +
  // segment passes + finalize
  if (forward) *forward = 1 + f + (R > 0 ? 1 : 0);
  if (backward) *backward = 1 + (R > 0 ? 1 : 0) + b + (S > 0 ? 1 : 0);
  return N3DS_OK;
}

int n3ds_field_read_pair_counts(void* workspace, uint64_t* per_base, n3ds_stream_t stream) {
  if (!workspace || !per_base) return fail(N3DS_ERR_INVALID, "workspace and per_base required");
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  N3DS_CUDA_TRY(cudaMemcpyAsync(per_base, static_cast<char*>(workspace) + 16, 16 * sizeof(uint64_t),
                                cudaMemcpyDeviceToHost, st));
  N3DS_CUDA_TRY(cudaStreamSynchronize(st));
  return N3DS_OK;
}

int n3ds_field_read_backward_pairs(void* workspace, uint64_t* pairs, n3ds_stream_t stream) {
  if (!workspace || !pairs) return fail(N3DS_ERR_INVALID, "workspace and pairs required");
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  N3DS_CUDA_TRY(cudaMemcpyAsync(pairs, static_cast<char*>(workspace) + 8 + 17 * sizeof(uint64_t), sizeof(uint64_t),
                                cudaMemcpyDeviceToHost, st));
  N3DS_CUDA_TRY(cudaStreamSynchronize(st));
  return N3DS_OK;
}

int n3ds_field_read_status(void* workspace, int32_t* status, uint64_t* evaluated_pairs, n3ds_stream_t stream) {
  if (!workspace) return fail(N3DS_ERR_INVALID, "workspace required");
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  unsigned long long hdr[2] = {0ull, 0ull};
  N3DS_CUDA_TRY(cudaMemcpyAsync(hdr, workspace, sizeof(hdr), cudaMemcpyDeviceToHost, st));
  N3DS_CUDA_TRY(cudaStreamSynchronize(st));
  N3DS_CUDA_TRY(cudaMemsetAsync(workspace, 0, sizeof(int32_t), st));
  int32_t sv;
  std::memcpy(&sv, &hdr[0], sizeof(sv));
  if (status) *status = sv;
  if (evaluated_pairs) *evaluated_pairs = hdr[1];
  return N3DS_OK;
}


// ------------------------------------------------------------- layer 1 operators

size_t n3ds_stroke_workspace_bytes(int64_t n_strokes) {
  if (n_strokes < 0) return 0;
  return n3ds::stroke_workspace_bytes(size_t(n_strokes));
}

namespace {
struct StrokeWs {
  float *recs, *cull_a, *cull_b, *gslots;
  int* status;
};
StrokeWs stroke_ws(void* ws, int64_t S) {
  char* b = static_cast<char*>(ws);
  StrokeWs w;
  size_t off = 0;
  w.status = reinterpret_cast<int*>(b + off);
  off += 256;
  w.recs = reinterpret_cast<float*>(b + off);
  off += align256(size_t(S) * n3ds::REC_FLOATS * 4);
  w.cull_a = reinterpret_cast<float*>(b + off);
  off += align256(size_t(S) * 16);
  w.cull_b = reinterpret_cast<float*>(b + off);
  off += align256(size_t(S + 4) * 4);
  w.gslots = reinterpret_cast<float*>(b + off);
  return w;
}

int check_stroke_args(uint32_t sdf_id, uint32_t color_id, int64_t n_points, int64_t n_viewdirs, int64_t n_strokes,
                      int64_t n_shape_params, int64_t n_color_params, int64_t n_texcoord, void* ws, size_t ws_bytes) {
  // fn_id bound as strokes_forward.cu:202-204, then this build's implemented subset
  if (sdf_id * 4u + color_id >= 12u * 16u * 4u) return fail(N3DS_ERR_INVALID, "fn_id must be in [0, num_fn_ids]");
  if (color_id > 3) return fail(N3DS_ERR_INVALID, "color_id must be 0-3");
  const int base = (int)(sdf_id >> 4);
  if (!n3ds::base_supported(base))
    return fail(N3DS_ERR_INVALID, "sdf base " + std::to_string(base) + " does not exist (bases 0-11)");
  if (base > n3ds::B_TETRAHEDRON && (sdf_id & 15u))
    return fail(N3DS_ERR_UNSUPPORTED, "Bezier strokes take no transform flags");
  if (n_texcoord != 0 && n_texcoord < 2 * n_points * n_strokes)
    return fail(N3DS_ERR_INVALID, "texcoord_output must hold [P, S, 2] floats");
  if (n_points < 0 || n_strokes < 0) return fail(N3DS_ERR_INVALID, "negative sizes");
  if (n_viewdirs <= 0 && n_points > 0) return fail(N3DS_ERR_INVALID, "viewdir must have at least one row");
  if (n_strokes > 0 && n_shape_params < n3ds::sdf_id_param_count((int)sdf_id))
    return fail(N3DS_ERR_INVALID, "shape_params has " + std::to_string(n_shape_params) + " columns, sdf_id needs " +
                                      std::to_string(n3ds::sdf_id_param_count((int)sdf_id)));
  const int64_t need_c = color_id == 0 ? 3 : (color_id == 3 ? 27 : 12);
  if (n_strokes > 0 && n_color_params < need_c)
    return fail(N3DS_ERR_INVALID, "color_params needs " + std::to_string(need_c) + " columns for color_id " +
                                      std::to_string(color_id));
  if (color_id >= 2 && n_viewdirs > 0 && n_points % n_viewdirs != 0)
    return fail(N3DS_ERR_INVALID, "the points must be a whole number of samples per view direction");
  if (n_strokes > 65535LL * 32) return fail(N3DS_ERR_INVALID, "too many strokes");
  if (!ws || ws_bytes < n3ds_stroke_workspace_bytes(n_strokes))
    return fail(N3DS_ERR_WORKSPACE, "workspace too small: need " + std::to_string(n3ds_stroke_workspace_bytes(n_strokes)));
  if (reinterpret_cast<uintptr_t>(ws) % 256) return fail(N3DS_ERR_INVALID, "workspace must be 256-byte aligned");
  return N3DS_OK;
}

n3ds::PrepLaunch uniform_prep(const StrokeWs& w, const float* shape_params, int64_t n_shape_params,
                              const float* color_params, int64_t n_color_params, int64_t S, uint32_t sdf_id,
                              float sdf_delta, int laplace, int inv_scale, bool zero_slots) {
  n3ds::PrepLaunch p{};
  p.sdf_ids = nullptr;
  p.uniform_sdf_id = (int)sdf_id;
  p.shape_params = shape_params;
  p.param_stride = (int)n_shape_params;
  p.color_params = color_params;
  p.color_stride = (int)n_color_params;
  p.density = nullptr;
  p.sdf_delta = nullptr;
  p.uniform_delta = sdf_delta;
  p.use_laplace = laplace;
  p.inv_scale_radius = inv_scale;
  p.cull_m = -1.f;
  p.n_strokes = S;
  p.recs = w.recs;
  p.cull_a = w.cull_a;
  p.cull_b = w.cull_b;
  p.status = w.status;
  p.counters = nullptr;
  p.n_counters = 0;
  p.gslots = zero_slots ? w.gslots : nullptr;
  p.stats = nullptr;
  return p;
}
n3ds::UfColor color_launch(const float* x, const float* viewdir, const float* recs, const float* color_params,
                           int64_t n_color_params, uint32_t color_id, int64_t P, int64_t n_viewdirs, int64_t S) {
  n3ds::UfColor C{};
  C.x = x;
  C.viewdir = viewdir;
  C.recs = recs;
  C.color_params = color_params;
  C.color_stride = (int)n_color_params;
  C.color_id = (int)color_id;
  C.n_points = P;
  C.spr = n_viewdirs > 0 ? std::max<int64_t>(1, P / n_viewdirs) : 1;
  C.n_strokes = (int)S;
  return C;
}

}  // namespace

int n3ds_stroke_forward(float* alpha_out, float* color_out, float* sdf_out, float* texcoord_out, int64_t n_texcoord,
                        const float* x,
                        const float* radius, const float* viewdir, const float* shape_params,
                        const float* color_params, int64_t n_points, int64_t n_viewdirs, int64_t n_strokes,
                        int64_t n_shape_params, int64_t n_color_params, uint32_t sdf_id, uint32_t color_id,
                        float sdf_delta, int use_laplace_transform, int inv_scale_radius, void* workspace,
                        size_t workspace_bytes, n3ds_stream_t stream) {
  int rc = check_stroke_args(sdf_id, color_id, n_points, n_viewdirs, n_strokes, n_shape_params, n_color_params,
                             n_texcoord, workspace, workspace_bytes);
  if (rc) return rc;
  if (n_points == 0 || n_strokes == 0) return N3DS_OK;
  if (!alpha_out || !color_out || !x || !radius || !shape_params || !color_params)
    return fail(N3DS_ERR_INVALID, "null tensor pointer");
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  StrokeWs w = stroke_ws(workspace, n_strokes);
  // With alpha the only per-pair output, pairs whose alpha is exactly 0 in float32 are
  // not evaluated: the culling bound keeps the soft-step argument beyond m = 104 for the
  // laplace step (alpha = exp(-m) / 2 < 2^-150 rounds to 0, the reference's own float32
  // value, even with denormals), beyond the linear step's zero (m >= 0.5) and outside
  // the hard step's surface. (A looser cut would not be exact for a caller: compose's
  // colour normalisation 1 / (1 + 1e-6 - T) magnifies alphas near 1e-9 at empty samples.)
  const bool cull = sdf_out == nullptr && n_texcoord == 0;
  n3ds::PrepLaunch prep = uniform_prep(w, shape_params, n_shape_params, color_params, n_color_params, n_strokes,
                                       sdf_id, sdf_delta, use_laplace_transform, inv_scale_radius, false);
  if (cull) prep.cull_m = 104.f;
  n3ds::launch_prep(prep, st);
  N3DS_CUDA_TRY(cudaGetLastError());
  n3ds::UfStroke L{};
  L.cull_a = cull ? w.cull_a : nullptr;
  L.cull_b = cull ? w.cull_b : nullptr;
  L.x = x;
  L.radius = radius;
  L.recs = w.recs;
  L.n_points = n_points;
  L.n_strokes = (int)n_strokes;
  L.alpha = alpha_out;
  L.color = color_out;
  L.sdf = sdf_out;
  L.color_const = color_id == 0;
  N3DS_CUDA_TRY(n3ds::launch_uf_stroke_fwd(L, (int)(sdf_id >> 4), st));
  if (color_id != 0) {
    if (color_id >= 2 && !viewdir) return fail(N3DS_ERR_INVALID, "viewdir is required by the SH colour fields");
    n3ds::UfColor C = color_launch(x, viewdir, w.recs, color_params, n_color_params, color_id, n_points, n_viewdirs,
                                   n_strokes);
    C.color = color_out;
    N3DS_CUDA_TRY(n3ds::launch_uf_color_fwd(C, st));
  }
  if (n_texcoord != 0) {
    if (!texcoord_out) return fail(N3DS_ERR_INVALID, "texcoord_out is null");
    n3ds::UfColor C = color_launch(x, viewdir, w.recs, color_params, n_color_params, color_id, n_points, n_viewdirs,
                                   n_strokes);
    N3DS_CUDA_TRY(n3ds::launch_uf_texcoord(C, texcoord_out, st));
  }
  return N3DS_OK;
}

int n3ds_stroke_backward(float* grad_shape_params, float* grad_color_params, float* grad_x, const float* grad_alpha,
                         const float* grad_color, const float* grad_sdf, const float* x, const float* radius,
                         const float* viewdir, const float* alpha, const float* shape_params,
                         const float* color_params, int64_t n_points, int64_t n_viewdirs, int64_t n_strokes,
                         int64_t n_shape_params, int64_t n_color_params, uint32_t sdf_id, uint32_t color_id,
                         float sdf_delta, int use_laplace_transform, int inv_scale_radius, int grad_mode,
                         void* workspace, size_t workspace_bytes, n3ds_stream_t stream) {
  int rc = check_stroke_args(sdf_id, color_id, n_points, n_viewdirs, n_strokes, n_shape_params, n_color_params, 0,
                             workspace, workspace_bytes);
  if (rc) return rc;
  if (n_strokes == 0) return N3DS_OK;
  if (!grad_shape_params || !grad_color_params || !grad_alpha || !grad_color || !x || !radius || !alpha ||
      !shape_params || !color_params)
    return fail(N3DS_ERR_INVALID, "null tensor pointer");
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  StrokeWs w = stroke_ws(workspace, n_strokes);
  n3ds::launch_prep(uniform_prep(w, shape_params, n_shape_params, color_params, n_color_params, n_strokes, sdf_id,
                                 sdf_delta, use_laplace_transform, inv_scale_radius, true),
                    st);
  N3DS_CUDA_TRY(cudaGetLastError());
  const int compat = grad_mode == N3DS_GRAD_COMPAT;
  if (n_points > 0) {
    n3ds::UfStroke L{};
    L.x = x;
    L.radius = radius;
    L.recs = w.recs;
    L.n_points = n_points;
    L.n_strokes = (int)n_strokes;
    L.g_alpha = grad_alpha;
    L.g_color = grad_color;
    L.g_sdf = grad_sdf;
    L.alpha_in = alpha;
    L.grad_x = grad_x;
    L.gslots = w.gslots;
    L.compat = compat;
    L.color_const = color_id == 0;
    N3DS_CUDA_TRY(n3ds::launch_uf_stroke_bwd(L, (int)(sdf_id >> 4), st));
    if (color_id != 0) {
      if (color_id >= 2 && !viewdir) return fail(N3DS_ERR_INVALID, "viewdir is required by the SH colour fields");
      n3ds::UfColor C = color_launch(x, viewdir, w.recs, color_params, n_color_params, color_id, n_points,
                                     n_viewdirs, n_strokes);
      C.g_color = grad_color;
      C.grad_color_params = grad_color_params;
      C.gslots = w.gslots;
      C.grad_x = grad_x;
      C.compat = compat;
      N3DS_CUDA_TRY(n3ds::launch_uf_color_bwd(C, st));
    }
  }
  n3ds::FinalizeLaunch F{};
  F.sdf_ids = nullptr;
  F.uniform_sdf_id = (int)sdf_id;
  F.shape_params = shape_params;
  F.param_stride = (int)n_shape_params;
  F.sdf_delta = nullptr;
  F.uniform_delta = sdf_delta;
  F.recs = w.recs;
  F.gslots = w.gslots;
  F.n_strokes = n_strokes;
  F.compat = compat;
  F.grad_shape = grad_shape_params;
  F.grad_color = grad_color_params;
  F.color_stride = (int)n_color_params;
  F.grad_density = nullptr;
  F.grad_delta = nullptr;
  F.accumulate = 1;
  n3ds::launch_finalize(F, st);
  N3DS_CUDA_TRY(cudaGetLastError());
  return N3DS_OK;
}

int n3ds_compose_forward(float* density_out, float* color_out, const float* alphas, const float* colors,
                         const float* density_params, int64_t n_points, int64_t n_strokes, int64_t color_dim,
                         n3ds_stream_t stream) {
  if (color_dim != 1 && color_dim != 3)
    return fail(N3DS_ERR_UNSUPPORTED, "Unsupported color dimension: " + std::to_string(color_dim));
  if (n_points < 0 || n_strokes < 0) return fail(N3DS_ERR_INVALID, "negative sizes");
  if (n_points == 0) return N3DS_OK;
  if (!density_out || !color_out || (n_strokes > 0 && (!alphas || !colors || !density_params)))
    return fail(N3DS_ERR_INVALID, "null tensor pointer");
  if (n_strokes > 0x7fffffffLL) return fail(N3DS_ERR_INVALID, "too many strokes");
  n3ds::UfCompose L{};
  L.alphas = alphas;
  L.colors = colors;
  L.density = density_params;
  L.n_points = n_points;
  L.n_strokes = (int)n_strokes;
  L.color_dim = (int)color_dim;
  L.density_out = density_out;
  L.color_out = color_out;
  N3DS_CUDA_TRY(n3ds::launch_uf_compose_fwd(L, reinterpret_cast<cudaStream_t>(stream)));
  return N3DS_OK;
}

size_t n3ds_compose_workspace_bytes(int64_t n_points, int64_t n_strokes, int grad_mode) {
  if (grad_mode == N3DS_GRAD_COMPAT || n_points <= 0 || n_strokes <= 0) return 0;
  return size_t(n_points) * size_t((n_strokes + 31) / 32) * 4;  // one transmittance per row and 32 strokes
}

int n3ds_compose_backward(float* grad_alphas, float* grad_colors, float* grad_density_params,
                          const float* grad_density_out, const float* grad_color_out, const float* alphas,
                          const float* colors, const float* density_params, int64_t n_points, int64_t n_strokes,
                          int64_t color_dim, int grad_mode, void* workspace, size_t workspace_bytes,
                          n3ds_stream_t stream) {
  if (color_dim != 1 && color_dim != 3)
    return fail(N3DS_ERR_UNSUPPORTED, "Unsupported color dimension: " + std::to_string(color_dim));
  if (n_points < 0 || n_strokes < 0) return fail(N3DS_ERR_INVALID, "negative sizes");
  if (n_points == 0 || n_strokes == 0) return N3DS_OK;
  if (!grad_alphas || !grad_colors || !grad_density_params || !alphas || !colors || !density_params)
    return fail(N3DS_ERR_INVALID, "null tensor pointer");
  const int compat = grad_mode == N3DS_GRAD_COMPAT;
  if (!compat && (!workspace || workspace_bytes < n3ds_compose_workspace_bytes(n_points, n_strokes, grad_mode)))
    return fail(N3DS_ERR_WORKSPACE, "exact compose backward needs P*ceil(S/32)*4 bytes of workspace");
  n3ds::UfCompose L{};
  L.alphas = alphas;
  L.colors = colors;
  L.density = density_params;
  L.n_points = n_points;
  L.n_strokes = (int)n_strokes;
  L.color_dim = (int)color_dim;
  L.g_density = grad_density_out;
  L.g_color = grad_color_out;
  L.g_alphas = grad_alphas;
  L.g_colors = grad_colors;
  L.g_density_params = grad_density_params;
  L.t_scratch = static_cast<float*>(workspace);
  L.compat = compat;
  N3DS_CUDA_TRY(n3ds::launch_uf_compose_bwd(L, reinterpret_cast<cudaStream_t>(stream)));
  return N3DS_OK;
}

// ---------------------------------------------------------------------- Adam

int n3ds_adam_step(float* param, const float* grad, float* exp_avg, float* exp_avg_sq, const float* lo,
                   const float* hi, int64_t n, float lr, float beta1, float beta2, float eps, const int32_t* step,
                   n3ds_stream_t stream) {
  if (n < 0) return fail(N3DS_ERR_INVALID, "negative size");
  if (n == 0) return N3DS_OK;
  if (!param || !grad || !exp_avg || !exp_avg_sq || !step) return fail(N3DS_ERR_INVALID, "null pointer");
  N3DS_CUDA_TRY(n3ds::launch_adam(param, grad, exp_avg, exp_avg_sq, lo, hi, n, lr, beta1, beta2, eps, step,
                                  reinterpret_cast<cudaStream_t>(stream)));
  return N3DS_OK;
}

}  // extern "C"
