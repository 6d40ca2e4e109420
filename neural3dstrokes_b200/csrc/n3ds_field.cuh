// Launch descriptors and kernel declarations of the fused stroke field.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace n3ds {

constexpr int MAX_SCENES_PER_LAUNCH = 40;

// One scene of a (possibly batched) launch. Rays, samples and strokes of all
// scenes are concatenated; these give the scene's slice.
struct SceneDesc {
  long long ray_begin;   // first ray (global)
  int n_rays;
  int stroke_begin;      // first stroke (global)
  int n_strokes;
  int home_lo;           // first CTA whose home is this scene (CTAs home_lo .. next scene's home_lo - 1)
  int chunk_lo;          // stroke range of the current pass, scene-local
  int chunk_n;
  int first_pass;        // 1: composite state starts fresh
  int last_pass;         // 1: the pass that finishes the scene
  int mask_words;        // ceil(n_strokes / 32): stroke-block words per segment
  long long mask_begin;  // first word of the scene's stroke-block masks (segment-major)
};

struct SegLaunch {
  const float* x;          // [P*3], or null: samples cast from the rays below
  const float* radius;     // [P]
  const float* origins;    // [R*3] (cast mode)
  const float* dirs;       // [R*3] (cast mode)
  const float* tdist;      // [R*(N+1)] (cast mode)
  const float* radii;      // [R] (cast mode)
  int n_samples;           // samples per ray
  int segs_per_ray;        // ceil(n_samples / 32)
  int rays_per_item;       // rays a warp claims per atomic on the scene's work counter (>= 1)
  const float* recs;       // [S*64] prepared stroke records
  const float* cull_a;     // [S*4]  culling sphere (cx, cy, cz, R)
  const float* cull_b;     // [S(+pad)] culling margin per unit radius
  float* state;            // [P*5] composite state / forward checkpoint (T, sigma, C)
  const float* seeds;      // [P*5] backward seeds (g_sigma, g_C, g_T)
  float* bstate;           // [P*8] backward running state between passes
  float* grad_x;           // [P*3] or null
  float* gslots;           // [S*32] reduced per-stroke gradient slots
  int compat;              // reference gradient formulas
  float skip_alpha;        // forward: mask threshold; backward: skip the adjoint of a stroke whose alpha is below this at
                           // every sample of a segment (the culling threshold; 0 never skips)
  int n_scenes;
  int tiles_total;         // work items (rays) in the launch
  int schedule;            // N3DS_SCHEDULE_SEGMENTS or N3DS_SCHEDULE_RUNS
  int chunk_cap;           // strokes per shared-memory stage
  int* tile_counter;       // [n_scenes] next ray of each scene (zeroed before the launch)
  int* status;
  unsigned long long* stats;  // [0] evaluated (sample, stroke) pairs
  // Stroke-block masks, one 32-bit word per (segment, block of 32 strokes counted
  // from the scene's top stroke): bit b = stroke (top - b) survived culling and has
  // alpha >= skip_alpha at some sample of the segment. The forward stores the non-zero
  // words when non-null (the host clears the array first); the backward reads them
  // instead of culling when mask_tag holds the bits of its skip_alpha (written by the
  // forward's prep kernel).
  unsigned* block_masks;
  const int* mask_tag;
  int common_only;                   // forward: every stroke is a common primitive (pair_alpha_common)
  unsigned long long wait_limit_ns;  // bounded waits give up after this long
  int test_stall;                    // arm the staging barrier without the copies (test of the wait limit)
  SceneDesc sc[MAX_SCENES_PER_LAUNCH];
};

struct RayLaunch {
  const float* state;      // [P*5]
  const float* tdist;      // [R*(N+1)]
  const float* dirs;       // [R*3]
  const float* bg;         // [R*3] or null
  float bg_value;
  int opaque;
  long long n_rays;
  int n_samples;
  float* rgb;              // [R*3]
  float* acc;              // [R]
  float* depth;            // [R]
  // backward
  const float* g_rgb;      // [R*3] or null
  const float* g_acc;      // [R] or null
  const float* g_depth;    // [R] or null
  float* seeds;            // [P*5]
};

struct PrepLaunch {
  const int* sdf_ids;      // [S], or null with uniform_sdf_id
  int uniform_sdf_id;
  const float* shape_params;
  int param_stride;
  const float* color_params;
  int color_stride;
  const float* density;    // [S] or null (zero density)
  const float* sdf_delta;  // [S] or null with uniform_delta
  float uniform_delta;
  int use_laplace;
  int inv_scale_radius;
  float cull_m;            // soft-step argument beyond which a stroke is dropped; <0 disables
  long long n_strokes;
  float* recs;
  float* cull_a;
  float* cull_b;
  int* status;
  // zeroed by the prep kernel (graph-capture friendly resets)
  int* counters;
  int n_counters;
  float* gslots;           // zeroed when non-null
  unsigned long long* stats;
  int* mask_tag;           // set to mask_tag_value when non-null
  int mask_tag_value;
  // optional per-scene stroke windows (n3ds_strokes_t::stroke_window): device
  // (frozen, active) pairs; win_begin[b] .. win_begin[b+1] are scene b's strokes
  const int* window;
  int n_win_scenes;
  int win_begin[MAX_SCENES_PER_LAUNCH + 1];
  // the caller's hint of the bases present (bit b = base b; 0 = any): a stroke of
  // another base is treated as an unsupported kind
  unsigned base_mask;
};

struct FinalizeLaunch {
  const int* sdf_ids;      // [S], or null with uniform_sdf_id
  int uniform_sdf_id;
  const float* shape_params;
  int param_stride;
  const float* sdf_delta;  // [S] or null with uniform_delta
  float uniform_delta;
  const float* recs;
  const float* gslots;
  long long n_strokes;
  int compat;
  float* grad_shape;       // [S*param_stride]
  float* grad_color;       // [S*3]
  float* grad_density;     // [S]
  float* grad_delta;       // [S] or null
  int accumulate;          // 1: add into the outputs instead of overwriting
  int color_stride;        // floats per stroke row of grad_color (3 for the fused path)
  // optional stroke windows, as in PrepLaunch: strokes outside [frozen, active) get
  // zero gradients
  const int* window;
  int n_win_scenes;
  int win_begin[MAX_SCENES_PER_LAUNCH + 1];
};

// Window state of stroke s: 0 active, 1 frozen (no gradient), 2 absent.
__device__ __forceinline__ int window_state(const int* window, int n_win_scenes, const int* win_begin, long long s) {
  if (!window) return 0;
  int b = 0;
  while (b + 1 < n_win_scenes && s >= win_begin[b + 1]) b++;
  const long long i = s - win_begin[b];
  if (i >= window[2 * b + 1]) return 2;
  return i < window[2 * b] ? 1 : 0;
}

// status word bits
constexpr int ST_BAD_KIND = 1;
constexpr int ST_WAIT_TIMEOUT = 2;

void launch_prep(const PrepLaunch& p, cudaStream_t st);
cudaError_t launch_seg_fwd(const SegLaunch& L, int grid, int warps, size_t smem, cudaStream_t st);
cudaError_t launch_seg_bwd(const SegLaunch& L, int grid, int warps, size_t smem, cudaStream_t st);
void launch_ray_fwd(const RayLaunch& L, cudaStream_t st);
void launch_ray_bwd(const RayLaunch& L, cudaStream_t st);
void launch_finalize(const FinalizeLaunch& L, cudaStream_t st);

size_t seg_fwd_smem(int chunk_cap, int warps);
size_t seg_bwd_smem(int chunk_cap);

// sample-run kernels (n3ds_runs.cu): same launch descriptor, work items are units of
// up to 64 samples of a ray
constexpr int RUN_UNIT_SAMPLES = 64;
cudaError_t launch_run_fwd(const SegLaunch& L, int grid, int warps, size_t smem, cudaStream_t st);
cudaError_t launch_run_bwd(const SegLaunch& L, int grid, int warps, size_t smem, cudaStream_t st);
size_t run_fwd_smem(int chunk_cap, int warps);
size_t run_bwd_smem(int chunk_cap, int warps);

}  // namespace n3ds
