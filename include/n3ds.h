/*
 * n3ds: B200-native (sm_100a) stroke field of Neural 3D Strokes, C ABI.
 *
 * Every entry point takes device pointers, int64 sizes and a CUDA stream, launches
 * asynchronously on that stream, allocates nothing, and returns 0 or an N3DS_ERR_*
 * code; n3ds_last_error() gives the message of the last failure on the calling
 * thread. Float buffers are float32, C-contiguous.
 *
 * Two layers:
 *  1. The four operators of the reference's native module `_strokelib`
 *     (source/strokelib/src/bindings.cpp:6-11), same argument meaning and order,
 *     with tensors replaced by pointers + sizes. Gradient outputs accumulate into
 *     caller-zeroed buffers, as in the reference (strokes.py:212-216, 365-367).
 *  2. The fused stroke field: stroke evaluation, soft step, overlay compositing and
 *     volume rendering in one forward, its exact adjoint in one backward, for one
 *     scene or a batch of uneven scenes, graph-capturable (no host syncs, no
 *     allocation; scratch lives in a caller-provided workspace).
 */
#ifndef N3DS_H_
#define N3DS_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* n3ds_stream_t; /* = cudaStream_t */

#define N3DS_OK 0
#define N3DS_ERR_INVALID 1     /* bad argument (shape, null pointer, size) */
#define N3DS_ERR_UNSUPPORTED 2 /* colour type or output outside the implemented set */
#define N3DS_ERR_CUDA 3        /* a CUDA call failed */
#define N3DS_ERR_WORKSPACE 4   /* workspace too small */
#define N3DS_ERR_DEVICE 5      /* a kernel reported a device-side error status */

/* Work decomposition of the fused field kernels: a warp per 32-sample segment with
 * every lane evaluating each surviving stroke, or a warp per 64-sample unit with the
 * (sample, stroke) pairs inside each stroke's reach packed densely into lanes. */
#define N3DS_SCHEDULE_SEGMENTS 1
#define N3DS_SCHEDULE_RUNS 2

#define N3DS_GRAD_EXACT 0  /* exact adjoint of the forward (checked against float64 finite differences) */
#define N3DS_GRAD_COMPAT 1 /* the reference's hand-written backward formulas */

/* Message of the last failure on this thread (empty string if none). */
const char* n3ds_last_error(void);
/* Library version, major * 10000 + minor * 100 + patch. */
int n3ds_version(void);

/* ------------------------------------------------------------------------------
 * Layer 1: reference `_strokelib` operators
 * ------------------------------------------------------------------------------ */

/* Workspace bytes needed by n3ds_stroke_forward / n3ds_stroke_backward for
 * n_strokes strokes (prepared per-stroke records). */
size_t n3ds_stroke_workspace_bytes(int64_t n_strokes);

/* Replaces stroke_forward (strokes_forward.cu:170-225; declared strokes.h:14-27).
 * alpha_out [P,S], color_out [P,S,3], sdf_out [P,S] or NULL, texcoord_out [P,S,2] with
 * n_texcoord its float count (0 and NULL: not produced). x [P,3], radius [P], viewdir
 * [R,3] (the SH colour fields read viewdir[p / (P / R)]), shape_params [S,Ps],
 * color_params [S,Pc]. sdf_id / color_id as produced by the reference get_stroke
 * (strokes.py:95-106): every base SDF; colour 0 constant rgb, 1 gradient rgb (12
 * params), 2 SH2 (12), 3 SH3 (27). */
int n3ds_stroke_forward(float* alpha_out, float* color_out, float* sdf_out, float* texcoord_out, int64_t n_texcoord,
                        const float* x, const float* radius, const float* viewdir,
                        const float* shape_params, const float* color_params, int64_t n_points,
                        int64_t n_viewdirs, int64_t n_strokes, int64_t n_shape_params,
                        int64_t n_color_params, uint32_t sdf_id, uint32_t color_id, float sdf_delta,
                        int use_laplace_transform, int inv_scale_radius, void* workspace,
                        size_t workspace_bytes, n3ds_stream_t stream);

/* Replaces stroke_backward (strokes_backward.cu:224-287; declared strokes.h:38-54).
 * Accumulates into grad_shape_params [S,Ps], grad_color_params [S,Pc] and grad_x [P,3]
 * (NULL to skip). grad_sdf may be NULL. alpha is the forward's alpha_out.
 * grad_mode: N3DS_GRAD_EXACT or N3DS_GRAD_COMPAT. */
int n3ds_stroke_backward(float* grad_shape_params, float* grad_color_params, float* grad_x,
                         const float* grad_alpha, const float* grad_color, const float* grad_sdf,
                         const float* x, const float* radius, const float* viewdir,
                         const float* alpha, const float* shape_params, const float* color_params,
                         int64_t n_points, int64_t n_viewdirs, int64_t n_strokes,
                         int64_t n_shape_params, int64_t n_color_params, uint32_t sdf_id,
                         uint32_t color_id, float sdf_delta, int use_laplace_transform,
                         int inv_scale_radius, int grad_mode, void* workspace,
                         size_t workspace_bytes, n3ds_stream_t stream);

/* Replaces compose_forward (compositing.cu:159-204; declared compositing.h:11-15).
 * density_out [P], color_out [P,C], alphas [P,S], colors [P,S,C], density_params [S];
 * C in {1, 3}. */
int n3ds_compose_forward(float* density_out, float* color_out, const float* alphas,
                         const float* colors, const float* density_params, int64_t n_points,
                         int64_t n_strokes, int64_t color_dim, n3ds_stream_t stream);

/* Workspace bytes of n3ds_compose_backward: P*ceil(S/32) floats in exact mode (the
 * transmittance in front of every 32-stroke chunk of a row), 0 in compat mode. */
size_t n3ds_compose_workspace_bytes(int64_t n_points, int64_t n_strokes, int grad_mode);

/* Replaces compose_backward (compositing.cu:206-263; declared compositing.h:25-32).
 * Accumulates into grad_alphas [P,S], grad_colors [P,S,C], grad_density_params [S].
 * grad_density_out [P] and grad_color_out [P,C] may be NULL (treated as zero).
 * Exact mode is division-free (a top-down and a bottom-up sweep) and needs
 * n3ds_compose_workspace_bytes of scratch. */
int n3ds_compose_backward(float* grad_alphas, float* grad_colors, float* grad_density_params,
                          const float* grad_density_out, const float* grad_color_out,
                          const float* alphas, const float* colors, const float* density_params,
                          int64_t n_points, int64_t n_strokes, int64_t color_dim, int grad_mode,
                          void* workspace, size_t workspace_bytes, n3ds_stream_t stream);

/* Composition modes of compose_strokes other than 'over' (strokes.py:390-417). */
#define N3DS_COMPOSE_MAX 1
#define N3DS_COMPOSE_MAX_DENSITY_WEIGHTED 2
#define N3DS_COMPOSE_SOFTMAX 3
#define N3DS_COMPOSE_SOFTMAX_DENSITY_WEIGHTED 4

/* Replaces the torch code of compose_strokes for the modes above (strokes.py:390-417;
 * the reference has no native kernel for them). density_out [P], color_out [P,C]
 * (written), alphas [P,S], colors [P,S,C], density_params [S]; C in {1, 3}. max modes
 * pick the first maximum (NaN counts as the largest), as torch.argmax. */
int n3ds_compose_mode_forward(int mode, float* density_out, float* color_out, const float* alphas,
                              const float* colors, const float* density_params, int64_t n_points,
                              int64_t n_strokes, int64_t color_dim, n3ds_stream_t stream);

/* Backward of n3ds_compose_mode_forward: writes (overwrites) grad_alphas [P,S] and
 * grad_colors [P,S,C]; accumulates into grad_density_params [S] (caller-zeroed).
 * grad_density_out [P] and grad_color_out [P,C] may be NULL (zero). */
int n3ds_compose_mode_backward(int mode, float* grad_alphas, float* grad_colors, float* grad_density_params,
                               const float* grad_density_out, const float* grad_color_out,
                               const float* alphas, const float* colors, const float* density_params,
                               int64_t n_points, int64_t n_strokes, int64_t color_dim,
                               n3ds_stream_t stream);

/* Maximum n_strokes of n3ds_stroke_forward_static. */
#define N3DS_STATIC_MAX_STROKES 4096

/* n3ds_stroke_forward without a workspace argument (no counterpart in the reference):
 * for callers that hold no device allocator of their own (a C or FFI host that only
 * passes through tensors it was given) or must not allocate once running (cudaMalloc
 * synchronises the device and can fail under a fixed memory budget). Its scratch, the
 * prepared records of up to N3DS_STATIC_MAX_STROKES strokes (1.7 MB), is one
 * file-scope device array per device; more strokes return N3DS_ERR_INVALID. Nothing
 * in the scratch has to start at zero. Two calls in flight on the same device at once
 * race on that scratch; calls on one stream are ordered. The first call on a device
 * (with that device current) looks the array's address up with cudaGetSymbolAddress;
 * a caller that records the call into a stream capture makes one call on that device
 * before capturing. The address is kept for the process's life: do not call this entry
 * point after a cudaDeviceReset of that device. Same arguments, outputs and errors as
 * n3ds_stroke_forward. */
int n3ds_stroke_forward_static(float* alpha_out, float* color_out, float* sdf_out, float* texcoord_out,
                               int64_t n_texcoord,
                               const float* x, const float* radius, const float* viewdir,
                               const float* shape_params, const float* color_params, int64_t n_points,
                               int64_t n_viewdirs, int64_t n_strokes, int64_t n_shape_params,
                               int64_t n_color_params, uint32_t sdf_id, uint32_t color_id,
                               float sdf_delta, int use_laplace_transform, int inv_scale_radius,
                               n3ds_stream_t stream);

/* ------------------------------------------------------------------------------
 * Layer 2: fused stroke field
 * (StrokeField.predict_density models.py:660-711 + compute_alpha_weights /
 *  volumetric_rendering render.py:29-88, as driven by Model.forward models.py:191-235)
 * ------------------------------------------------------------------------------ */

/* Scene batch: scene i owns n_rays[i] consecutive rays and n_strokes[i] consecutive
 * strokes of the concatenated arrays. Host arrays. */
typedef struct n3ds_batch {
  int32_t n_scenes;
  const int64_t* n_rays;    /* host [n_scenes] */
  const int32_t* n_strokes; /* host [n_scenes] */
  int32_t n_samples;        /* samples per ray, all scenes */
} n3ds_batch_t;

typedef struct n3ds_rays {
  const float* x;      /* [R*N*3] sample positions, or NULL to cast them from the rays */
  const float* radius; /* [R*N] sample radii (unused when x is NULL) */
  const float* tdist;  /* [R*(N+1)] fence-post distances */
  const float* dirs;   /* [R*3] ray directions (their norm scales the intervals) */
  const float* bg;     /* [R*3] background colour, or NULL to use bg_value */
  float bg_value;
  int32_t opaque_background;
  /* with x == NULL the kernels cast the samples themselves (cast_rays, render.py:5-26):
   * x_i = dirs * t_i + origins, radius_i = radii * t_i, t_i = (tdist_i + tdist_i+1) / 2 */
  const float* origins; /* [R*3] */
  const float* radii;   /* [R] base radii */
} n3ds_rays_t;

typedef struct n3ds_strokes {
  const int32_t* sdf_ids;     /* [S] reference sdf_id per stroke (device) */
  const float* shape_params;  /* [S*param_stride], reference layout, zero-padded */
  int32_t param_stride;
  const float* color_params;  /* [S*3] constant rgb */
  const float* density;       /* [S] density (already times density_scale) */
  const float* sdf_delta;     /* [S] softness per stroke */
  int32_t use_laplace_transform;
  int32_t inv_scale_radius;
  /* Optional stroke window per scene, device int32 [n_scenes*2] = (frozen, active)
   * pairs, or NULL (every stroke active). Read on the device by the kernels, so the
   * window can follow a device-side stroke count with no host round trip (the
   * truncation of StrokeField.predict_density, models.py:665-673, 686-702). Scene
   * strokes at local index >= active are absent: no alpha, no gradient. Strokes below
   * frozen are composited as usual but receive no gradient and contribute none to
   * grad_x (the reference evaluates them under torch.no_grad and concatenates them
   * before the optimised ones, which keeps the stroke order). Needs the segment
   * schedule and at most 40 scenes. */
  const int32_t* stroke_window;
  /* Optional hint: bit b set when strokes of base b (sdf_id >> 4) may occur, 0 = any.
   * When the hint names only the common primitives (sphere / ellipsoid, cube / box,
   * round cube / box, capsule, octahedron, tetrahedron), the forward runs a build
   * that carries only their code. A stroke outside the hint is an unsupported kind
   * (status bit 1, NaN outputs). */
  uint32_t base_mask;
} n3ds_strokes_t;

typedef struct n3ds_options {
  float cull_alpha;   /* drop a stroke where its alpha provably stays below this; <= 0: no culling */
  int32_t chunk_fwd;  /* strokes per shared-memory stage, forward (0 = auto; else rounded
                         down to a multiple of 32, within [32, 1024]) */
  int32_t chunk_bwd;  /* strokes per shared-memory stage, backward (same rules) */
  int32_t warps;      /* warps per CTA, forward: 4, 8, 16, 24, 32 (0 = auto) */
  int32_t schedule;   /* N3DS_SCHEDULE_* (0 = auto: segments) */
  int32_t grad_mode;  /* N3DS_GRAD_EXACT or N3DS_GRAD_COMPAT */
  /* optional: 4 cudaEvent_t recorded on the stream around the segment kernels
   * (forward begin/end, backward begin/end), or NULL */
  void* const* timing_events;
  int32_t warps_bwd;  /* warps per CTA, backward: 4, 8, 16, 20, 24, 32 (0 = auto) */
  /* 1: no backward follows this forward, so the segment kernels skip recording which
   * strokes the backward needs (a backward after such a forward culls by itself) */
  int32_t forward_only;
  /* 1: count the evaluated (sample, stroke) pairs, per base SDF type in the forward and
   * in total in the backward (n3ds_field_read_status, _read_pair_counts,
   * _read_backward_pairs); 0 (default): those counters stay 0 and the kernels skip the
   * per-candidate bookkeeping */
  int32_t count_pairs;
  /* limit of every bounded device-side wait (the stroke staging barrier), in
   * microseconds; 0 = the default, one second. A wait that runs out sets status bit 2
   * (N3DS_ERR_DEVICE through n3ds_field_read_status) and its CTA stops; the launch's
   * outputs are then invalid */
  int32_t wait_limit_us;
  /* test of the bounded wait: 1 arms the staging barrier for the stage's bytes
   * without issuing the copies, so every wait runs out and reports (no copy is left
   * in flight). 0 in any real use */
  int32_t test_stall_staging;
  /* rays a warp claims per work item in the segment schedule: 1, 2 or 4 (0 = 1), i.e.
   * 64, 128 or 256 samples per claim at 64 samples per ray; larger claims take fewer
   * atomics on the scene's work counter, smaller ones balance the tail better */
  int32_t rays_per_item;
} n3ds_options_t;

/* Fill *opt with the defaults. */
void n3ds_default_options(n3ds_options_t* opt);

/* The launch configuration the library uses for *opt on the current device: auto
 * (0) stage sizes, warps and schedule replaced by their resolved values. */
int n3ds_field_resolve_options(const n3ds_options_t* opt, n3ds_options_t* out);

/* Workspace bytes for a batch (forward checkpoint, backward seeds and state,
 * prepared records, reduction slots, counters). total_strokes = sum of n_strokes. */
size_t n3ds_field_workspace_bytes(const n3ds_batch_t* batch, const n3ds_options_t* opt);

/* Forward: rgb [R*3], acc [R], depth [R]. Leaves the checkpoint in the workspace. */
int n3ds_field_forward(const n3ds_batch_t* batch, const n3ds_rays_t* rays,
                       const n3ds_strokes_t* strokes, const n3ds_options_t* opt, float* rgb,
                       float* acc, float* depth, void* workspace, size_t workspace_bytes,
                       n3ds_stream_t stream);

/* Backward of the preceding n3ds_field_forward with the same inputs and workspace.
 * Upstream grads may be NULL (zero). Writes (overwrites) grad_x [R*N*3] (NULL to
 * skip), grad_shape [S*param_stride], grad_color [S*3], grad_density [S],
 * grad_sdf_delta [S] (NULL to skip). */
int n3ds_field_backward(const n3ds_batch_t* batch, const n3ds_rays_t* rays,
                        const n3ds_strokes_t* strokes, const n3ds_options_t* opt,
                        const float* grad_rgb, const float* grad_acc, const float* grad_depth,
                        float* grad_x, float* grad_shape, float* grad_color, float* grad_density,
                        float* grad_sdf_delta, void* workspace, size_t workspace_bytes,
                        n3ds_stream_t stream);

/* Synchronously read (and clear) the device status word and the count of evaluated
 * (sample, stroke) pairs of the last forward (with options.count_pairs; else 0).
 * n3ds_field_forward clears the status
 * word first, so it reports the last forward and the backwards after it: 0 = fine,
 * bit 1 = an unsupported sdf id, bit 2 = a bounded wait gave up. */
int n3ds_field_read_status(void* workspace, int32_t* status, uint64_t* evaluated_pairs,
                           n3ds_stream_t stream);

/* Number of kernel launches one n3ds_field_forward / n3ds_field_backward makes for
 * this batch and these options (host-only planning, no device work). */
int n3ds_field_launch_count(const n3ds_batch_t* batch, const n3ds_options_t* opt, int32_t* forward,
                            int32_t* backward);

/* Synchronously read the evaluated (sample, stroke) pairs of the last forward per base
 * SDF type (16 counters, indexed by sdf_id >> 4). */
int n3ds_field_read_pair_counts(void* workspace, uint64_t* per_base, n3ds_stream_t stream);

/* Image texture of stroke colours and alphas (ImageTexture, source/textures.py:36-83,
 * applied between stroke_fn and compose_strokes at models.py:704-706), over n
 * (sample, stroke) pairs: tint = bilinear sample of image [channels, height, width]
 * at texcoords [n,2] as F.grid_sample(image, texcoords * 2 - 1, align_corners=True)
 * with zero padding; color_out [n,3] = (colors * tint_ratio + 1 - tint_ratio) * tint
 * (a 1-channel tint broadcasts); alpha_out [n] = alphas * mean(tint) when
 * modulate_alpha, else alphas (alpha_out may be NULL). channels must be 1 or 3. */
int n3ds_texture_forward(float* color_out, float* alpha_out, const float* texcoords, const float* colors,
                         const float* alphas, int64_t n, const float* image, int32_t channels, int32_t height,
                         int32_t width, float tint_ratio, int32_t modulate_alpha, n3ds_stream_t stream);

/* Backward of n3ds_texture_forward: writes (overwrites) grad_colors [n,3] =
 * grad_color_out * tint * tint_ratio and grad_alphas [n] = grad_alpha_out * mean(tint)
 * (modulate_alpha) or grad_alpha_out; NULL upstream grads count as zero, NULL outputs
 * are skipped. No gradient for texcoords or the image (none in the reference). */
int n3ds_texture_backward(float* grad_colors, float* grad_alphas, const float* grad_color_out,
                          const float* grad_alpha_out, const float* texcoords, int64_t n, const float* image,
                          int32_t channels, int32_t height, int32_t width, float tint_ratio,
                          int32_t modulate_alpha, n3ds_stream_t stream);
/* The same with the texture packed once by n3ds_texture_pack into [height, width]
 * float4 texels (r, g, b, 0; a grayscale texture replicated), one 16-byte load per
 * bilinear corner instead of one per corner and channel; packed must be 16-byte
 * aligned and hold height * width * 4 floats. channels is the original count. Results
 * equal the planar functions'. */
int n3ds_texture_pack(float* packed, const float* image, int32_t channels, int32_t height, int32_t width,
                      n3ds_stream_t stream);
int n3ds_texture_forward_packed(float* color_out, float* alpha_out, const float* texcoords, const float* colors,
                                const float* alphas, int64_t n, const float* packed, int32_t channels,
                                int32_t height, int32_t width, float tint_ratio, int32_t modulate_alpha,
                                n3ds_stream_t stream);
int n3ds_texture_backward_packed(float* grad_colors, float* grad_alphas, const float* grad_color_out,
                                 const float* grad_alpha_out, const float* texcoords, int64_t n,
                                 const float* packed, int32_t channels, int32_t height, int32_t width,
                                 float tint_ratio, int32_t modulate_alpha, n3ds_stream_t stream);

/* Proposal resampling of ray intervals (source/utils/stepfun.py; the step that makes
 * the stroke level's fence posts, models.py:147-185). One warp per ray; n_bins <= 2048.
 *
 * n3ds_max_dilate_weights: stepfun.max_dilate_weights (stepfun.py:136-147) of the step
 * functions t [R, n_bins+1], w [R, n_bins] into t_out [R, 3 n_bins + 1] and
 * w_out [R, 3 n_bins]. */
int n3ds_max_dilate_weights(float* t_out, float* w_out, const float* t, const float* w, int64_t n_rays,
                            int32_t n_bins, float dilation, float domain_lo, float domain_hi, int32_t renormalize,
                            n3ds_stream_t stream);

/* stepfun.sample_intervals (stepfun.py:280-317): n_samples intervals [R, n_samples+1]
 * from t [R, n_bins+1] and w_logits [R, n_bins]. jitter: NULL for the deterministic
 * centred samples (rand=False), else the uniform [0,1) draws of the reference's
 * torch.rand, [R] when single_jitter or [R, n_samples]. n_samples >= 2. */
int n3ds_sample_intervals(float* s_out, const float* t, const float* w_logits, int64_t n_rays, int32_t n_bins,
                          int32_t n_samples, const float* jitter, int32_t single_jitter, float domain_lo,
                          float domain_hi, n3ds_stream_t stream);

/* One proposal level fused (models.py:156-185): if dilation > 0, max_dilate_weights
 * with renormalisation and the [1:-1] slice; logits where(s[1:] > s[:-1],
 * log(w + resample_padding), -inf); sample_intervals; and tdist = s * far + (1 - s) *
 * near (the identity ray-distance warp). Outputs s_out and/or t_out [R, n_samples+1]
 * (t_out needs near, far [R]). */
int n3ds_resample_intervals(float* s_out, float* t_out, const float* sdist, const float* weights, int64_t n_rays,
                            int32_t n_bins, int32_t n_samples, float dilation, float resample_padding,
                            const float* jitter, int32_t single_jitter, float domain_lo, float domain_hi,
                            const float* near, const float* far, n3ds_stream_t stream);

/* Stroke insertion and reset on the device: StrokeField.step_update
 * (source/models.py:586-658) with the stroke count in device memory, so a training
 * step needs no host round trip. */
#define N3DS_INSERT_MAX_STROKES 8192
#define N3DS_INIT_RECON 0      /* strokes.py:258-270 */
#define N3DS_INIT_GEN_BOX 1    /* strokes.py:271-278 */
#define N3DS_INIT_GEN_SPHERE 2 /* strokes.py:279-289 */
#define N3DS_BASE_SAMPLER_NONE 0
#define N3DS_BASE_SAMPLER_ROUND 1    /* 0.8 u (round cube / box) */
#define N3DS_BASE_SAMPLER_TORUS 2    /* u, u (capped torus) */
#define N3DS_BASE_SAMPLER_CAPSULE 3  /* u + 0.25 */
#define N3DS_BASE_SAMPLER_LINE 4     /* u + 0.25, u - 0.5 */
#define N3DS_BASE_SAMPLER_UNIFORM 5  /* u (triangular prism) */
#define N3DS_BASE_SAMPLER_SPLINE 6   /* control points around the centre + radii (strokes.py:28-37) */
#define N3DS_COLOR_SAMPLER_UNIFORM 0  /* constant_rgb: u x n_color */
#define N3DS_COLOR_SAMPLER_GRADIENT 1 /* gradient_rgb: u - 0.5 x 6, u x 6 */
#define N3DS_COLOR_SAMPLER_NORMAL 2   /* constant_sh2 / sh3: N(0, 1) x n_color */

typedef struct {
  int32_t n_shape;        /* shape parameters per stroke (must match the flags below) */
  int32_t n_color;        /* colour parameters per stroke */
  int32_t base_sampler;   /* N3DS_BASE_SAMPLER_* */
  int32_t spline_points;  /* spline sampler: control points (1-4) */
  int32_t spline_radii;   /* spline sampler: radii (0-2) */
  int32_t t, r, s1, s3;   /* translation, rotation, single / per-axis scale parameters */
  int32_t init_type;      /* N3DS_INIT_* */
  int32_t color_sampler;  /* N3DS_COLOR_SAMPLER_* */
} n3ds_stroke_sampler_t;

typedef struct {
  int32_t max_num_strokes;     /* <= N3DS_INSERT_MAX_STROKES */
  int32_t init_num_strokes;
  float reset_density;         /* -INFINITY when the densities are not trained */
  int32_t use_error_field;
  int32_t use_shape_grads;
  float shape_split_update_rate;
  int32_t min_update_interval;
  int32_t min_reset_interval;
  float max_reset_frac;
  uint64_t seed;               /* random draws: hash of (seed, training step, row, draw) */
} n3ds_insert_config_t;

/* Scratch bytes of n3ds_insert_step. */
size_t n3ds_insert_workspace_bytes(const n3ds_insert_config_t* cfg, const n3ds_stroke_sampler_t* smp);

/* One step_update: stroke_step / last_update_step are device int32 scalars (the
 * stroke count and the training step of the last update). next_target is the host's
 * min(int(max_num * clamp(train_frac, 0, 1)^step_power) + init_num, max_num) for
 * cur_step (models.py:589-594); the kernel takes next = max(next_target, stroke_step).
 * errors [n_errors] / error_coords [n_errors, 3] are the caller's error-field samples
 * (may be NULL / 0); grad_ema [max, n_shape] the shape-gradient EMA (may be NULL).
 * Parameters: shape_params [max, n_shape], color_params [max, n_color], density [max]
 * rows are rewritten in place. No host synchronisation: the host passes the step's
 * scalars (cur_step, next_target, train_frac) as arguments, everything that depends on
 * device data (stroke count, resets, the update decision) stays on the device. */
int n3ds_insert_step(const n3ds_insert_config_t* cfg, const n3ds_stroke_sampler_t* smp, float* shape_params,
                     float* color_params, float* density, const float* grad_ema, int32_t* stroke_step,
                     int32_t* last_update_step, int64_t cur_step, int32_t next_target, float train_frac,
                     const float* errors, const float* error_coords, int64_t n_errors, void* workspace,
                     size_t workspace_bytes, n3ds_stream_t stream);

/* ema = ema * decay + grad * (1 - decay) over n floats (models.py:596-598). */
int n3ds_ema_update(float* ema, const float* grad, int64_t n, float decay, n3ds_stream_t stream);

/* Clamp each column j of x [rows, cols] to [lo[j], hi[j]] (host arrays; NaN = no bound),
 * as StrokeField.clip_params (models.py:576-584). cols <= N3DS_CLIP_MAX_COLS. */
#define N3DS_CLIP_MAX_COLS 32
int n3ds_clip_columns(float* x, int64_t rows, int32_t cols, const float* lo, const float* hi, n3ds_stream_t stream);

/* Synchronously read the (sample, stroke) pairs that the backwards since the last
 * forward evaluated (segment schedule; the forward resets the count). With the
 * stroke-block masks of its forward the backward evaluates only the strokes that
 * reach the skip threshold somewhere in a segment, far fewer than the forward. */
int n3ds_field_read_backward_pairs(void* workspace, uint64_t* pairs, n3ds_stream_t stream);

/* Adam step fused with the reference's parameter clamp (utils/training.py:119-136,
 * models.py:576-584) over n floats: m = b1 m + (1-b1) g; v = b2 v + (1-b2) g^2;
 * p -= lr * mhat / (sqrt(vhat) + eps); then p = clamp(p, lo, hi) where lo/hi may be
 * NULL. step is read from device memory (incremented by the caller's graph). */
int n3ds_adam_step(float* param, const float* grad, float* exp_avg, float* exp_avg_sq,
                   const float* lo, const float* hi, int64_t n, float lr, float beta1, float beta2,
                   float eps, const int32_t* step, n3ds_stream_t stream);

/* Multi-resolution grid encoder (source/gridencoder/src/gridencoder.h:7-14, the
 * `_gridencoder` module's grid_encode_forward / grid_encode_backward /
 * grad_total_variation). All pointers are device pointers; embeddings, outputs,
 * dy_dx, grad, grad_embeddings and grad_inputs have the element type `dtype`,
 * inputs are float (the total variation's inputs have `dtype` too, as in the
 * reference). Shapes: inputs [B, D] in [0, 1] (points outside give zeros and no
 * gradient); embeddings [offsets[L], C]; offsets [L + 1] int32; outputs [L, B, C];
 * dy_dx [B, L * D * C] or NULL; grad [L, B, C]. S = log2(per-level scale), H = base
 * resolution. D in {2, 3, 4, 5}, C in {1, 2, 4, 8}. grad_embeddings (and the total
 * variation's grad) are accumulated into (zero them first); grad_inputs is written
 * when both it and dy_dx are given. */
#define N3DS_DTYPE_F32 0
#define N3DS_DTYPE_F16 1
#define N3DS_DTYPE_F64 2
#define N3DS_GRID_HASH 0
#define N3DS_GRID_TILED 1
#define N3DS_INTERP_LINEAR 0
#define N3DS_INTERP_SMOOTHSTEP 1
int n3ds_grid_encode_forward(const float* inputs, const void* embeddings, const int32_t* offsets, void* outputs,
                             uint32_t B, uint32_t D, uint32_t C, uint32_t L, float S, uint32_t H, void* dy_dx,
                             uint32_t gridtype, int32_t align_corners, uint32_t interpolation, int32_t dtype,
                             n3ds_stream_t stream);
int n3ds_grid_encode_backward(const void* grad, const float* inputs, const void* embeddings, const int32_t* offsets,
                              void* grad_embeddings, uint32_t B, uint32_t D, uint32_t C, uint32_t L, float S,
                              uint32_t H, const void* dy_dx, void* grad_inputs, uint32_t gridtype,
                              int32_t align_corners, uint32_t interpolation, int32_t dtype, n3ds_stream_t stream);
/* grad += the total-variation gradient at the cells of B points (random points when
 * the caller draws them), source/gridencoder/src/gridencoder.cu:453-559. */
int n3ds_grid_total_variation(const void* inputs, const void* embeddings, void* grad, const int32_t* offsets,
                              float weight, uint32_t B, uint32_t D, uint32_t C, uint32_t L, float S, uint32_t H,
                              uint32_t gridtype, int32_t align_corners, int32_t dtype, n3ds_stream_t stream);

/* Fused density network of the proposal and error fields: MLP.predict_density plus
 * the density activation with disable_rgb (source/models.py:362-372, 430-431; PropMLP
 * :501-504, ErrorMLP.sample_error :513-523). Per point: warp the coordinates
 * (`warp`), map them to [0, 1] by the encoder's bound, encode them on the hash grid
 * (n_levels x level_dim features, as n3ds_grid_encode_forward), then
 * raw = w2 . relu(w1 f + b1) + b2 and density = softplus(raw + density_bias)
 * (torch's softplus: the identity above 20). The first layer runs on the tensor
 * cores (tcgen05, tf32 with a three-term split: float32 accuracy). The reference
 * runs it as torch layers; this network has no counterpart in its native code.
 * Constraints: level_dim in {1, 2, 4}, n_levels * level_dim <= 16, 64 hidden units,
 * float32 everywhere, linear interpolation. */
#define N3DS_WARP_SCALE 0    /* coords * warp_scale (the reference's warp_fn None: / (bbox_size / 2)) */
#define N3DS_WARP_CONTRACT 1 /* coord.contract(coords) / 2 (warp_fn 'contract') */
#define N3DS_WARP_NONE 2     /* coords as given (no_warp=True) */
#define N3DS_DENSITY_HIDDEN 64
typedef struct n3ds_density_net {
  const float* table;          /* [offsets[L], level_dim] GridEncoder.embeddings */
  const int32_t* offsets;      /* [n_levels + 1] GridEncoder.offsets */
  uint32_t n_levels;           /* L */
  uint32_t level_dim;          /* C */
  float log2_per_level_scale;  /* S = log2(per_level_scale) */
  uint32_t base_resolution;    /* H */
  uint32_t gridtype;           /* N3DS_GRID_HASH or N3DS_GRID_TILED */
  int32_t align_corners;
  const float* w1;             /* [64, L * C] density_layer[0].weight */
  const float* b1;             /* [64] density_layer[0].bias */
  const float* w2;             /* [64] density_layer[2].weight ([1, 64]) */
  const float* b2;             /* [1] density_layer[2].bias */
  float density_bias;          /* MLP.density_bias */
  int32_t warp;                /* N3DS_WARP_* */
  float warp_scale;            /* float32(1 / (bbox_size / 2)) for N3DS_WARP_SCALE */
  float grid_bound;            /* GridEncoder.forward's bound (1.0 in predict_density) */
  int32_t raw_output;          /* nonzero: `density` receives raw (predict_density's
                                  raw_density, no bias or softplus) and the backward
                                  takes its gradient */
  int32_t* status;             /* device int32 or NULL; bit 2 (value 2) is ORed in when
                                  a bounded wait for the tensor cores ran out (the
                                  call's outputs are then invalid) */
  int32_t wait_limit_us;       /* limit of each such wait; 0: one second */
  int32_t test_stall;          /* test hook: withhold the tensor-core work so that the
                                  first wait runs out (0 in normal use) */
} n3ds_density_net_t;
/* Persistent CTAs the last forward (backward = 0) or backward launch of this process
 * used (resident CTAs per SM x SMs), 0 before the first; a diagnostic. */
int n3ds_density_net_resident_ctas(int32_t backward);
/* Floats per point of the feature record written by the forward for the backward:
 * L * C rounded up to a multiple of 4. */
int n3ds_density_net_feature_stride(uint32_t n_levels, uint32_t level_dim);
/* density [n] (and, when not NULL, features [n, stride] for the backward and the
 * warped coordinates [n, 3], the module's `coord` output); coords [n, 3]. */
int n3ds_density_net_forward(const n3ds_density_net_t* net, const float* coords, int64_t n_points, float* density,
                             float* features, float* coords_warped, n3ds_stream_t stream);
/* The adjoint of the forward with respect to the table and the four layer tensors,
 * accumulated into grad_table [offsets[L], C], grad_w1 [64, L * C], grad_b1 [64],
 * grad_w2 [64] and grad_b2 [1] (zero them first); features are the forward's
 * record, grad_density [n]. No gradient with respect to the coordinates. */
int n3ds_density_net_backward(const n3ds_density_net_t* net, const float* coords, const float* features,
                              const float* grad_density, int64_t n_points, float* grad_table, float* grad_w1,
                              float* grad_b1, float* grad_w2, float* grad_b2, n3ds_stream_t stream);
/* Hash-decay statistics of a float32 table (source/models.py:472-488):
 * out[l, c] = mean over level l's rows of table[row, c]^2, for every channel when
 * all_channels is nonzero (torch_scatter's segment_coo), else for channel 0 with
 * the other channels 0 (the scatter_reduce_ fallback the reference takes without
 * torch_scatter). level_dim 1, 2 or 4. out [L, C] is overwritten. The backward adds
 * grad_out[l, c] * 2 * table[row, c] / rows(l) to grad_table. */
int n3ds_grid_level_mean_sq(const float* table, const int32_t* offsets, uint32_t n_levels, uint32_t level_dim,
                            int32_t all_channels, float* out, n3ds_stream_t stream);
int n3ds_grid_level_mean_sq_backward(const float* table, const int32_t* offsets, uint32_t n_levels,
                                     uint32_t level_dim, int32_t all_channels, const float* grad_out,
                                     float* grad_table, n3ds_stream_t stream);

/* FP32 FMA throughput probe (no counterpart in the reference; a measurement aid for
 * the roofline of these FP32-bound kernels): one launch of `blocks` x 256 threads,
 * each doing iters x 16 fused multiply-adds, i.e. blocks*256*iters*32 flops.
 * out needs blocks*256 floats (written only to keep the work alive). */
int n3ds_fp32_probe(float* out, int32_t blocks, int32_t iters, n3ds_stream_t stream);

#ifdef __cplusplus
}
#endif

#endif /* N3DS_H_ */
