// Colour fields of the drop-in stroke operators (strokes_color.h:50-171): colour per
// (sample, stroke) for
//   gradient rgb  lerp(c0, c1, sigmoid(5 t - 2.5)), t the projection of the unit-frame
//                 (local) sample on the segment pos0 -> pos1 (12 parameters);
//   SH2 / SH3     sigmoid(sum_i coef_i Y_i(viewdir)) per channel, real spherical
//                 harmonics of the world view direction (12 / 27 parameters).
// Lane = stroke (32 strokes per warp tile) and a loop over samples, so the colour rows
// are written and read coalesced and each lane keeps its stroke's parameters and
// parameter gradients in registers. The backward accumulates the colour-parameter
// gradients (the reference's formulas, exact in the parameters) and, in exact mode,
// the gradient rgb's dependence on the sample position, which it sends through the
// stroke transform into the reduced slots and grad_x (the reference drops that term).
#include "n3ds_eval.cuh"
#include "n3ds_unfused.cuh"

namespace n3ds {

namespace {

constexpr int COL_WARPS = 4;
constexpr int COL_RS = REC_FLOATS + 4;  // padded record stride (lane-indexed 128-bit loads)

__device__ __forceinline__ float sigmoidf_(float v) { return 1.f / (1.f + expf(-v)); }

// Real spherical-harmonic basis up to degree 2 (4 terms) or 3 (9 terms), the polynomial
// forms with the standard normalisations (Y00 = 1/(2 sqrt(pi)), Y1m = sqrt(3)/(2 sqrt(pi))
// {-y, z, -x}, Y2m from sqrt(15)/(2 sqrt(pi)), sqrt(5)/(4 sqrt(pi)), sqrt(15)/(4 sqrt(pi))).
template <int N>
__device__ __forceinline__ void sh_basis(V3 d, float (&w)[N]) {
  const float c0 = 0.28209479177387814f, c1 = 0.48860251190291992f;
  w[0] = c0;
  w[1] = -c1 * d.y;
  w[2] = c1 * d.z;
  w[3] = -c1 * d.x;
  if constexpr (N == 9) {
    const float c2 = 1.0925484305920792f, c20 = 0.31539156525252005f, c22 = 0.54627421529603959f;
    w[4] = c2 * d.x * d.y;
    w[5] = -c2 * d.y * d.z;
    w[6] = c20 * (3.f * d.z * d.z - 1.f);
    w[7] = -c2 * d.x * d.z;
    w[8] = c22 * (d.x * d.x - d.y * d.y);
  }
}

template <int CT>
struct ColorDims {
  static constexpr int NP = CT == 3 ? 27 : 12;  // colour parameters
  static constexpr int NB = CT == 3 ? 9 : 4;    // SH terms
};

// Local (unit-frame) sample of the stroke: the primitives' inverse transform; the
// curves have none.
__device__ __forceinline__ V3 unit_pos(const float* rec, int base, V3 x) {
  return base <= B_TETRAHEDRON ? prim_local(rec, x) : x;
}

// Gradient rgb at local p; t its sigmoid blend weight, d0 / d1 the projection terms.
__device__ __forceinline__ V3 gradient_rgb(const float (&cp)[12], V3 p, float* t, float* d0, float* d1, V3* v0,
                                           V3* v1) {
  const V3 pos0 = v3(cp[0], cp[1], cp[2]), pos1 = v3(cp[3], cp[4], cp[5]);
  *v0 = p - pos0;
  *v1 = pos1 - pos0;
  *d0 = dot(*v0, *v1);
  *d1 = dot(*v1, *v1);
  *t = sigmoidf_(*d0 / *d1 * 5.0f - 2.5f);
  return v3(cp[6], cp[7], cp[8]) * (1.0f - *t) + v3(cp[9], cp[10], cp[11]) * *t;
}

// dL/d(local p) through the transform: scale / rotation / translation slots (the
// transform part of prim_backprop) and dL/dx = M^T g.
__device__ __forceinline__ V3 transform_backprop(const float* rec, int kind, V3 p, V3 gp, float (&v)[9]) {
  const int flags = (kind >> 4) & 15;
  const V3 s = xyz(rec4(rec)[R_S / 4]), si = xyz(rec4(rec)[R_SINV / 4]);
  if (flags & F_S1) {
    v[6] += -dot(gp, p) * si.x;
  } else if (flags & F_S3) {
    v[6] += -gp.x * p.x * si.x;
    v[7] += -gp.y * p.y * si.y;
    v[8] += -gp.z * p.z * si.z;
  }
  if (flags & F_R) {
    const V3 tq = cross(gp * si, s * p);
    v[3] += tq.x;
    v[4] += tq.y;
    v[5] += tq.z;
  }
  v[0] += gp.x;
  v[1] += gp.y;
  v[2] += gp.z;
  return xyz(rec4(rec)[R_M / 4]) * gp.x + xyz(rec4(rec)[R_M / 4 + 1]) * gp.y + xyz(rec4(rec)[R_M / 4 + 2]) * gp.z;
}

template <int CT>
__global__ void __launch_bounds__(COL_WARPS * 32) uf_color_fwd_kernel(const UfColor L) {
  constexpr int NP = ColorDims<CT>::NP;
  __shared__ __align__(16) float recs[32 * COL_RS];
  const int s0 = blockIdx.y * 32;
  const int ns = min(32, L.n_strokes - s0);
  if (CT == 1)
    for (int i = threadIdx.x; i < ns * REC_FLOATS; i += blockDim.x)
      recs[(i / REC_FLOATS) * COL_RS + (i % REC_FLOATS)] = L.recs[(long long)s0 * REC_FLOATS + i];
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const bool active = lane < ns;
  const long long s = s0 + (active ? lane : 0);
  const float* rec = recs + (active ? lane : 0) * COL_RS;
  const int kind = CT == 1 ? __float_as_int(rec[R_KIND]) : 0;
  float cp[NP];
#pragma unroll
  for (int k = 0; k < NP; k++) cp[k] = L.color_params[s * L.color_stride + k];
  const long long S = L.n_strokes;
  for (long long p = (long long)blockIdx.x * COL_WARPS + warp; p < L.n_points; p += (long long)gridDim.x * COL_WARPS) {
    V3 c;
    if constexpr (CT == 1) {
      const V3 x = v3(L.x[3 * p], L.x[3 * p + 1], L.x[3 * p + 2]);
      float t, d0, d1;
      V3 v0, v1;
      c = gradient_rgb(cp, unit_pos(rec, kind & 15, x), &t, &d0, &d1, &v0, &v1);
    } else {
      const long long r = p / L.spr;
      float w[ColorDims<CT>::NB];
      sh_basis(v3(L.viewdir[3 * r], L.viewdir[3 * r + 1], L.viewdir[3 * r + 2]), w);
      float acc[3] = {0.f, 0.f, 0.f};
#pragma unroll
      for (int i = 0; i < ColorDims<CT>::NB; i++)
#pragma unroll
        for (int q = 0; q < 3; q++) acc[q] += cp[3 * i + q] * w[i];
      c = v3(sigmoidf_(acc[0]), sigmoidf_(acc[1]), sigmoidf_(acc[2]));
    }
    if (active) {
      float* o = L.color + (p * S + s) * 3;
      o[0] = c.x;
      o[1] = c.y;
      o[2] = c.z;
    }
  }
}

template <int CT>
__global__ void __launch_bounds__(COL_WARPS * 32) uf_color_bwd_kernel(const UfColor L) {
  constexpr int NP = ColorDims<CT>::NP;
  __shared__ __align__(16) float recs[32 * COL_RS];
  const int s0 = blockIdx.y * 32;
  const int ns = min(32, L.n_strokes - s0);
  if (CT == 1)
    for (int i = threadIdx.x; i < ns * REC_FLOATS; i += blockDim.x)
      recs[(i / REC_FLOATS) * COL_RS + (i % REC_FLOATS)] = L.recs[(long long)s0 * REC_FLOATS + i];
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const bool active = lane < ns;
  const long long s = s0 + (active ? lane : 0);
  const float* rec = recs + (active ? lane : 0) * COL_RS;
  const int kind = CT == 1 ? __float_as_int(rec[R_KIND]) : 0;
  const int base = kind & 15;
  float cp[NP], gcp[NP];
#pragma unroll
  for (int k = 0; k < NP; k++) {
    cp[k] = L.color_params[s * L.color_stride + k];
    gcp[k] = 0.f;
  }
  float v[9] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};  // GP, torque, scale slots
  const bool with_pos = CT == 1 && !L.compat;
  const long long S = L.n_strokes;
  for (long long p = (long long)blockIdx.x * COL_WARPS + warp; p < L.n_points; p += (long long)gridDim.x * COL_WARPS) {
    const float* gcol = L.g_color + (p * S + s) * 3;
    const V3 g = active ? v3(gcol[0], gcol[1], gcol[2]) : v3(0.f, 0.f, 0.f);
    if constexpr (CT == 1) {
      const V3 x = v3(L.x[3 * p], L.x[3 * p + 1], L.x[3 * p + 2]);
      const V3 pl = unit_pos(rec, base, x);
      float t, d0, d1;
      V3 v0, v1;
      gradient_rgb(cp, pl, &t, &d0, &d1, &v0, &v1);
      // strokes_color.h:82-96
      const float gt = dot(g, v3(cp[9] - cp[6], cp[10] - cp[7], cp[11] - cp[8]));
      const float gtr = 5.0f * t * (1.0f - t) * gt;
      const float gd0 = gtr / d1, gd1 = -gtr * d0 / (d1 * d1);
      const V3 gv1 = v0 * gd0 + v1 * (gd1 * 2.0f);
      const V3 gv0 = v1 * gd0;
      const V3 gp0 = -gv0 - gv1;
      gcp[0] += gp0.x; gcp[1] += gp0.y; gcp[2] += gp0.z;
      gcp[3] += gv1.x; gcp[4] += gv1.y; gcp[5] += gv1.z;
      gcp[6] += g.x * (1.0f - t); gcp[7] += g.y * (1.0f - t); gcp[8] += g.z * (1.0f - t);
      gcp[9] += g.x * t; gcp[10] += g.y * t; gcp[11] += g.z * t;
      if (with_pos) {
        // dL/d(local p) = dL/dv0 = gd0 v1
        const V3 gx = base <= B_TETRAHEDRON ? transform_backprop(rec, kind, pl, gv0, v) : gv0;
        if (L.grad_x) {
          const float sx = warp_sum(gx.x), sy = warp_sum(gx.y), sz = warp_sum(gx.z);
          if (lane == 0) {
            atomicAdd(L.grad_x + 3 * p, sx);
            atomicAdd(L.grad_x + 3 * p + 1, sy);
            atomicAdd(L.grad_x + 3 * p + 2, sz);
          }
        }
      }
    } else {
      const long long r = p / L.spr;
      constexpr int NB = ColorDims<CT>::NB;
      float w[NB];
      sh_basis(v3(L.viewdir[3 * r], L.viewdir[3 * r + 1], L.viewdir[3 * r + 2]), w);
      float acc[3] = {0.f, 0.f, 0.f};
#pragma unroll
      for (int i = 0; i < NB; i++)
#pragma unroll
        for (int q = 0; q < 3; q++) acc[q] += cp[3 * i + q] * w[i];
      float gr[3];
      const float gq[3] = {g.x, g.y, g.z};
#pragma unroll
      for (int q = 0; q < 3; q++) {
        const float c = sigmoidf_(acc[q]);
        gr[q] = gq[q] * c * (1.0f - c);
      }
#pragma unroll
      for (int i = 0; i < NB; i++)
#pragma unroll
        for (int q = 0; q < 3; q++) gcp[3 * i + q] += gr[q] * w[i];
    }
  }
  if (active) {
#pragma unroll
    for (int k = 0; k < NP; k++)
      if (gcp[k] != 0.f) atomicAdd(L.grad_color_params + s * L.color_stride + k, gcp[k]);
    if (with_pos && base <= B_TETRAHEDRON) {
      float* row = L.gslots + s * GRAD_SLOTS;
#pragma unroll
      for (int k = 0; k < 3; k++) {
        if (v[k] != 0.f) atomicAdd(row + G_GP + k, v[k]);
        if (v[3 + k] != 0.f) atomicAdd(row + G_TORQUE + k, v[3 + k]);
        if (v[6 + k] != 0.f) atomicAdd(row + G_SCALE + k, v[6 + k]);
      }
    }
  }
}

// Orders the axes of d by the values sc (permute_multiscale_axis, strokes_sdf.h:212-222).
__device__ __forceinline__ V3 permute_by(V3 d, V3 sc) {
  if (sc.x > sc.y) {
    if (sc.y > sc.z) return d;
    return sc.x > sc.z ? V3{d.x, d.z, d.y} : V3{d.z, d.x, d.y};
  }
  if (sc.z > sc.y) return V3{d.z, d.y, d.x};
  return sc.x > sc.z ? V3{d.y, d.x, d.z} : V3{d.y, d.z, d.x};
}

// Texture coordinates of the local sample (BaseSDF::texcoord: sphere strokes_sdf.h:259-267,
// cube and round cube 302-310 / 359-367, capsule 455-467, line 510-522; (0, 0) for the
// other bases). The per-axis permutation reads three values at the offset each base
// uses there: the scales, or for the round cube its radius and two scales.
__device__ __forceinline__ float2 prim_texcoord(const float* rec, int kind, V3 p) {
  constexpr float PI_F = 3.14159265358979323846f;
  const int base = kind & 15;
  const bool s3 = ((kind >> 4) & F_S3) && !((kind >> 4) & F_S1);
  const V3 s = xyz(rec4(rec)[R_S / 4]);
  switch (base) {
    case B_SPHERE: {
      V3 d = p * rsqrtf(dot(p, p));
      if (s3) d = permute_by(d, s);
      return make_float2(asinf(clampf(d.x, -1.f, 1.f)) / PI_F + 0.5f, atan2f(d.z, d.y) / (2.0f * PI_F) + 0.5f);
    }
    case B_CUBE:
    case B_ROUND_CUBE: {
      V3 uvt = p * 0.5f + 0.5f;
      if (s3) uvt = permute_by(uvt, base == B_CUBE ? s : V3{rec[R_BP], s.x, s.y});
      return make_float2(clampf(uvt.x, 0.f, 1.f), clampf(uvt.y, 0.f, 1.f));
    }
    case B_CAPSULE:
    case B_LINE: {
      const float h = rec[R_BP];
      const float u = base == B_CAPSULE ? clampf((p.y / (h + 1.0f)) * 0.5f + 0.5f, 0.f, 1.f)
                                        : clampf((p.y + h + 1.0f - rec[R_BP2]) / (2.0f * h + 2.0f), 0.f, 1.f);
      // the capsule reads its scales after the half-length; the line (single-scale in
      // every reference shape) would read its radius change first
      const V3 sc = base == B_CAPSULE ? s : V3{rec[R_BP2], s.x, s.y};
      if (s3 && sc.z > sc.x) p = V3{p.z, p.y, p.x};
      return make_float2(u, atan2f(p.z, p.x) / (2.0f * PI_F) + 0.5f);
    }
    default:
      return make_float2(0.f, 0.f);
  }
}

__global__ void __launch_bounds__(COL_WARPS * 32) uf_texcoord_kernel(const UfColor L, float* texcoord) {
  __shared__ __align__(16) float recs[32 * COL_RS];
  const int s0 = blockIdx.y * 32;
  const int ns = min(32, L.n_strokes - s0);
  for (int i = threadIdx.x; i < ns * REC_FLOATS; i += blockDim.x)
    recs[(i / REC_FLOATS) * COL_RS + (i % REC_FLOATS)] = L.recs[(long long)s0 * REC_FLOATS + i];
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const bool active = lane < ns;
  const long long s = s0 + (active ? lane : 0);
  const float* rec = recs + (active ? lane : 0) * COL_RS;
  const int kind = __float_as_int(rec[R_KIND]);
  const long long S = L.n_strokes;
  for (long long p = (long long)blockIdx.x * COL_WARPS + warp; p < L.n_points; p += (long long)gridDim.x * COL_WARPS) {
    const V3 x = v3(L.x[3 * p], L.x[3 * p + 1], L.x[3 * p + 2]);
    const float2 uv = prim_texcoord(rec, kind, unit_pos(rec, kind & 15, x));
    if (active) {
      texcoord[(p * S + s) * 2] = uv.x;
      texcoord[(p * S + s) * 2 + 1] = uv.y;
    }
  }
}

// one wave of the kernel's resident blocks over the stroke blocks
template <typename K>
cudaError_t color_grid(const UfColor& L, K kernel, dim3* grid) {
  const int sblocks = (L.n_strokes + 31) / 32;
  long long want = 1;
  cudaError_t e = one_wave_blocks(kernel, COL_WARPS * 32, sblocks, (L.n_points + COL_WARPS - 1) / COL_WARPS, &want);
  *grid = dim3((unsigned)want, sblocks);
  return e;
}

}  // namespace

cudaError_t launch_uf_color_fwd(const UfColor& L, cudaStream_t st) {
  if (L.color_id < 1 || L.color_id > 3) return cudaErrorInvalidValue;
  auto* k = L.color_id == 1 ? uf_color_fwd_kernel<1> : L.color_id == 2 ? uf_color_fwd_kernel<2> : uf_color_fwd_kernel<3>;
  dim3 grid;
  cudaError_t e = color_grid(L, k, &grid);
  if (e != cudaSuccess) return e;
  k<<<grid, COL_WARPS * 32, 0, st>>>(L);
  return cudaGetLastError();
}

cudaError_t launch_uf_texcoord(const UfColor& L, float* texcoord, cudaStream_t st) {
  dim3 grid;
  cudaError_t e = color_grid(L, uf_texcoord_kernel, &grid);
  if (e != cudaSuccess) return e;
  uf_texcoord_kernel<<<grid, COL_WARPS * 32, 0, st>>>(L, texcoord);
  return cudaGetLastError();
}

cudaError_t launch_uf_color_bwd(const UfColor& L, cudaStream_t st) {
  if (L.color_id < 1 || L.color_id > 3) return cudaErrorInvalidValue;
  auto* k = L.color_id == 1 ? uf_color_bwd_kernel<1> : L.color_id == 2 ? uf_color_bwd_kernel<2> : uf_color_bwd_kernel<3>;
  dim3 grid;
  cudaError_t e = color_grid(L, k, &grid);
  if (e != cudaSuccess) return e;
  k<<<grid, COL_WARPS * 32, 0, st>>>(L);
  return cudaGetLastError();
}

}  // namespace n3ds
