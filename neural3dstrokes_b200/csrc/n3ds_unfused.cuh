// The reference `_strokelib` operators over dense [P, S] tensors (drop-in layer).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace n3ds {

struct UfStroke {
  const float* x;          // [P*3]
  const float* radius;     // [P]
  const float* recs;       // [S*64] prepared records (uniform sdf_id)
  long long n_points;
  int n_strokes;
  // forward outputs
  float* alpha;            // [P*S]
  float* color;            // [P*S*3]
  float* sdf;              // [P*S] or null
  // backward
  const float* g_alpha;    // [P*S]
  const float* g_color;    // [P*S*3]
  const float* g_sdf;      // [P*S] or null
  const float* alpha_in;   // [P*S] saved alpha
  float* grad_x;           // [P*3] or null (accumulated)
  float* gslots;           // [S*32] reduced slots
  int compat;
  int color_const;         // 1: constant rgb colour (written / reduced here); else a colour field kernel runs
  // forward culling (only alpha requested): [S] culling spheres (centre, radius) and
  // margins per unit sample radius from the prep kernel, or null (every pair evaluated)
  const float* cull_a;
  const float* cull_b;
};

// Colour fields (n3ds_colors.cu): gradient rgb (color_id 1), SH2 (2), SH3 (3).
struct UfColor {
  const float* x;              // [P*3]
  const float* viewdir;        // [R*3]
  const float* recs;           // [S*64] prepared records
  const float* color_params;   // [S*color_stride]
  int color_stride;
  int color_id;
  long long n_points;
  long long spr;               // points per view direction
  int n_strokes;
  float* color;                // forward: [P*S*3]
  const float* g_color;        // backward: [P*S*3]
  float* grad_color_params;    // backward: [S*color_stride], accumulated
  float* gslots;               // backward, exact mode: position term into the transform slots
  float* grad_x;               // backward, exact mode: [P*3] or null, accumulated
  int compat;
};
cudaError_t launch_uf_color_fwd(const UfColor& L, cudaStream_t st);
cudaError_t launch_uf_color_bwd(const UfColor& L, cudaStream_t st);
// texture coordinates [P*S*2] of the local samples (uses x, recs, n_points, n_strokes)
cudaError_t launch_uf_texcoord(const UfColor& L, float* texcoord, cudaStream_t st);

struct UfCompose {
  const float* alphas;     // [P*S]
  const float* colors;     // [P*S*C]
  const float* density;    // [S]
  long long n_points;
  int n_strokes;
  int color_dim;
  float* density_out;      // [P]
  float* color_out;        // [P*C]
  const float* g_density;  // [P] or null
  const float* g_color;    // [P*C] or null
  float* g_alphas;         // [P*S] accumulated
  float* g_colors;         // [P*S*C] accumulated
  float* g_density_params; // [S] accumulated
  float* t_scratch;        // [P*S] exact mode only
  int compat;
};

// Blocks per 32-stroke block for a kernel whose warps stride over the samples: one wave
// of the blocks of `kernel` that fit on the device together (threads per block given,
// no dynamic shared memory), spread over `sblocks` stroke blocks, at most `cap`. A
// grid sized for more blocks than fit leaves a second, partial wave that idles most
// of the machine.
template <typename K>
inline cudaError_t one_wave_blocks(K kernel, int threads, int sblocks, long long cap, long long* out) {
  int dev = 0, sms = 148, per_sm = 1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, 0);
  if (e != cudaSuccess) return e;
  long long want = ((long long)sms * (per_sm > 0 ? per_sm : 1) + sblocks - 1) / sblocks;
  if (want > cap) want = cap;
  *out = want < 1 ? 1 : want;
  return cudaSuccess;
}

cudaError_t launch_uf_stroke_fwd(const UfStroke& L, int base, cudaStream_t st);
cudaError_t launch_uf_stroke_bwd(const UfStroke& L, int base, cudaStream_t st);
cudaError_t launch_uf_compose_fwd(const UfCompose& L, cudaStream_t st);
cudaError_t launch_uf_compose_bwd(const UfCompose& L, cudaStream_t st);

// non-'over' composition modes (n3ds_compose_modes.cu)
cudaError_t launch_compose_mode_fwd(int mode, float* density, float* color, const float* alphas, const float* colors,
                                    const float* dp, long long P, long long S, int C, cudaStream_t st);
cudaError_t launch_compose_mode_bwd(int mode, float* g_alpha, float* g_colors, float* g_dp, const float* g_dens,
                                    const float* g_col, const float* alphas, const float* colors, const float* dp,
                                    long long P, long long S, int C, cudaStream_t st);

}  // namespace n3ds
