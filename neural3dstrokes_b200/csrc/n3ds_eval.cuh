// Per-(sample, stroke) evaluation shared by the fused and the unfused kernels:
// inverse transform, SDF, radius rescale, soft step (strokes_forward.cu:57-90).
#pragma once
#include "n3ds_sdf.cuh"

namespace n3ds {

// extra kind-word bits set by the prep kernel
constexpr int K_S3FAC = 1 << 10;  // multi-scale radius factor applies (S3 and inv_scale_radius)
constexpr int K_S1K = 1 << 11;    // single-scale s is folded into the soft-step slope
constexpr int K_FROZEN = 1 << 12; // composited, but no gradient of its own and none into grad_x

__device__ __forceinline__ float soft_alpha(int mode, float m) {
  if (mode == STEP_LAPLACE) return laplace_alpha(m);
  if (mode == STEP_LINEAR) return clampf(m + 0.5f, 0.f, 0.9999f);
  return 0.f;  // STEP_HARD handled by the caller from the sign of the SDF
}

// Local-frame sample p = M (x - t) (three 128-bit loads). The translation is
// subtracted first: folding it into an offset c = -M t cancels catastrophically for
// small strokes far from the origin.
__device__ __forceinline__ V3 prim_local(const float* rec, V3 x) {
  const float4 m0 = rec4(rec)[R_M / 4], m1 = rec4(rec)[R_M / 4 + 1], m2 = rec4(rec)[R_M / 4 + 2];
  const V3 d = {x.x - m0.w, x.y - m1.w, x.z - m2.w};
  return {fmaf(m0.x, d.x, fmaf(m0.y, d.y, m0.z * d.z)), fmaf(m1.x, d.x, fmaf(m1.y, d.y, m1.z * d.z)),
          fmaf(m2.x, d.x, fmaf(m2.y, d.y, m2.z * d.z))};
}

// Forward alpha of one stroke record at world sample x; rinv = 1 / sample radius.
// Optionally returns the SDF value.
__device__ __forceinline__ float pair_alpha(const float* rec, V3 x, float rinv, float* sdf_out = nullptr) {
  const float4 h = rec4(rec)[0];
  const int kind = __float_as_int(h.x);
  const int base = kind & 15;
  const int mode = (kind >> 8) & 3;
  float sdf, f = 1.f;
  if (base <= B_TETRAHEDRON) {
    V3 p = prim_local(rec, x);
    sdf = prim_sdf(base, p, rec);
    if (kind & K_S3FAC) f = s3_factor(base, p, xyz(rec4(rec)[R_S / 4]), rec);
  } else if (base == B_QUAD_BEZIER) {
    QuadFwd q;
    sdf = quad_eval(rec, x, q);
  } else {
    CubicFwd c;
    sdf = cubic_eval(rec, x, c, base == B_CATMULL_ROM);
  }
  if (sdf_out) *sdf_out = sdf;
  if (mode == STEP_HARD) return sdf <= 0.f ? 1.f : 0.f;
  float k = h.y * f * rinv;
  return soft_alpha(mode, -sdf * k);
}

template <int BASE>
__device__ __forceinline__ float common_sdf(V3 p, int kind, const float* rec, float* f) {
  const float sdf = prim_sdf(BASE, p, rec);
  if (kind & K_S3FAC) *f = s3_factor(BASE, p, xyz(rec4(rec)[R_S / 4]), rec);
  return sdf;
}

// pair_alpha for a launch whose strokes are all common primitives: the dispatch (and
// so the kernel's code) covers those six bases only; any other base gives NaN (the
// prep kernel flags such a stroke as an unsupported kind before this runs).
__device__ __forceinline__ float pair_alpha_common(const float* rec, V3 x, float rinv) {
  const float4 h = rec4(rec)[0];
  const int kind = __float_as_int(h.x);
  const int mode = (kind >> 8) & 3;
  const V3 p = prim_local(rec, x);
  float sdf, f = 1.f;
  switch (kind & 15) {
    case B_SPHERE: sdf = common_sdf<B_SPHERE>(p, kind, rec, &f); break;
    case B_CUBE: sdf = common_sdf<B_CUBE>(p, kind, rec, &f); break;
    case B_ROUND_CUBE: sdf = common_sdf<B_ROUND_CUBE>(p, kind, rec, &f); break;
    case B_CAPSULE: sdf = common_sdf<B_CAPSULE>(p, kind, rec, &f); break;
    case B_OCTAHEDRON: sdf = common_sdf<B_OCTAHEDRON>(p, kind, rec, &f); break;
    case B_TETRAHEDRON: sdf = common_sdf<B_TETRAHEDRON>(p, kind, rec, &f); break;
    default: sdf = __int_as_float(0x7fc00000); break;
  }
  if (mode == STEP_HARD) return sdf <= 0.f ? 1.f : 0.f;
  return soft_alpha(mode, -sdf * (h.y * f * rinv));
}

// dL/dm of the soft step given G = (1 - alpha) dL/dalpha (division-safe form).
__device__ __forceinline__ float soft_dm_from_G(int mode, float m, float alpha, float G) {
  if (mode == STEP_LAPLACE) return m <= 0.f ? G * alpha / (1.f - alpha) : G;
  if (mode == STEP_LINEAR) {
    float a = m + 0.5f;
    return (a > 0.f && a < 0.9999f) ? G / (1.f - alpha) : 0.f;
  }
  return 0.f;
}

// dL/dm of the soft step given dL/dalpha.
__device__ __forceinline__ float soft_dm(int mode, float m, float alpha, float galpha) {
  if (mode == STEP_LAPLACE) return galpha * (m <= 0.f ? alpha : 1.f - alpha);
  if (mode == STEP_LINEAR) {
    float a = m + 0.5f;
    return (a > 0.f && a < 0.9999f) ? galpha : 0.f;
  }
  return 0.f;
}

// Adjoint of the primitive part for upstream dsdf = dL/dSDF and K = dL/dk * k.
// Accumulates into the primitive reduction slots v[] (G_GP, G_TORQUE, G_SCALE,
// G_BP layout) and returns dL/dx (world).
// compat != 0: the reference formulas (no scale/position dependence through the
// soft-step width, cube exterior 2*max(q,0)).
__device__ __forceinline__ V3 prim_backprop(const float* rec, int kind, V3 p, float dsdf, float K,
                                            float* v, int compat) {
  int base = kind & 15;
  int flags = (kind >> 4) & 15;
  float gbp[2];
  V3 gp = prim_grad(base, p, rec, gbp, compat) * dsdf;
  v[G_BP] += gbp[0] * dsdf;
  v[G_BP2] += gbp[1] * dsdf;
  V3 s = xyz(rec4(rec)[R_S / 4]), si = xyz(rec4(rec)[R_SINV / 4]);
  V3 q = s * p;
  float kfac = compat ? 0.f : K;
  if ((kind & K_S3FAC) && !compat) {
    if (base == B_SPHERE) {
      // f = |q|/|p|: dL/dp += K (s^2 p/|q|^2 - p/|p|^2); dL/ds_i += K p_i^2 s_i/|q|^2
      float pp = dot(p, p), qq = dot(q, q);
      gp += (s * q) * (K / qq) + p * (-K / pp);
      V3 hs = (p * q) * (K / qq);
      v[G_SCALE + 0] += hs.x;
      v[G_SCALE + 1] += hs.y;
      v[G_SCALE + 2] += hs.z;
    } else {
      // f = |s g| / |g| with g the reference gradient (s3_factor): d ln f / ds_i =
      // s_i g_i^2 / |s g|^2, d ln f / dg = s^2 g / |s g|^2 - g / |g|^2
      float unused[2];
      const V3 g = prim_grad(base, p, rec, unused, 1);
      const V3 s2g = s * s * g;
      const float ff = dot(s2g, g), gg = dot(g, g);
      if (ff > 0.f && gg > 0.f) {
        const V3 hs = (s * g * g) * (K / ff);
        v[G_SCALE + 0] += hs.x;
        v[G_SCALE + 1] += hs.y;
        v[G_SCALE + 2] += hs.z;
        float gb0;
        gp += s3_dir_adjoint(base, p, rec, s2g * (1.f / ff) - g * (1.f / gg), &gb0) * K;
        v[G_BP] += gb0 * K;
      }
    }
  }
  if (flags & F_S1) {
    v[G_SCALE] += (-dot(gp, p) + ((kind & K_S1K) ? kfac : 0.f)) * si.x;
  } else if (flags & F_S3) {
    v[G_SCALE + 0] += -gp.x * p.x * si.x;
    v[G_SCALE + 1] += -gp.y * p.y * si.y;
    v[G_SCALE + 2] += -gp.z * p.z * si.z;
  }
  if (flags & F_R) {
    V3 tq = cross(gp * si, q);
    v[G_TORQUE + 0] += tq.x;
    v[G_TORQUE + 1] += tq.y;
    v[G_TORQUE + 2] += tq.z;
  }
  v[G_GP + 0] += gp.x;
  v[G_GP + 1] += gp.y;
  v[G_GP + 2] += gp.z;
  // dL/dx = M^T gp
  return xyz(rec4(rec)[R_M / 4]) * gp.x + xyz(rec4(rec)[R_M / 4 + 1]) * gp.y + xyz(rec4(rec)[R_M / 4 + 2]) * gp.z;
}

// Warp transpose-reduction of NV per-lane values: after it, lane l holds the warp
// total of value index bitrev(l) (NV = 32), or of bitrev4(l & 15) (NV = 16, lanes l
// and l ^ 16 hold the same total). Each halving step exchanges half the values.
template <int N, int O, int NV>
struct TransposeStep {
  __device__ __forceinline__ static void run(float (&v)[NV], int lane) {
    const bool up = (lane & O) != 0;
#pragma unroll
    for (int j = 0; j < N / 2; j++) {
      float lo = v[j], hi = v[j + N / 2];
      float send = up ? lo : hi;
      float keep = up ? hi : lo;
      v[j] = keep + __shfl_xor_sync(0xffffffffu, send, O);
    }
    TransposeStep<N / 2, O * 2, NV>::run(v, lane);
  }
};
template <int O, int NV>
struct TransposeStep<1, O, NV> {
  __device__ __forceinline__ static void run(float (&)[NV], int) {}
};

template <int NV>
__device__ __forceinline__ float warp_transpose_reduce(float (&v)[NV], int lane, int* idx) {
  TransposeStep<NV, 1, NV>::run(v, lane);
  if (NV == 16) {
    v[0] += __shfl_xor_sync(0xffffffffu, v[0], 16);
    *idx = (int)(__brev((unsigned)(lane & 15)) >> 28);
  } else {
    *idx = (int)(__brev((unsigned)lane) >> 27);
  }
  return v[0];
}

}  // namespace n3ds
