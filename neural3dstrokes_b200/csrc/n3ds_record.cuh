// Per-stroke record: the form in which a stroke is staged into shared memory.
//
// A prep kernel turns each stroke's raw reference-layout parameters (base params,
// then scale, Euler angles, translation, read backwards from the row end as in
// strokes_sdf.h:164-191) into one fixed 64-float (256 B) record holding everything
// the per-sample inner loops need, with all per-stroke invariants hoisted: the
// combined inverse transform M = S^-1 R^T, the soft-step slope, the culling sphere,
// the quadratic-Bezier closed-form constants, the cubic-Bezier polyline vertices.
#pragma once
#include "n3ds_math.cuh"

namespace n3ds {

constexpr int REC_FLOATS = 64;  // 256 bytes, 16-byte aligned for bulk copies

// kind word = base | flags << 4 | step_mode << 8
enum Base : int {
  B_SPHERE = 0, B_CUBE = 1, B_ROUND_CUBE = 2, B_CAPPED_TORUS = 3, B_CAPSULE = 4, B_LINE = 5,
  B_TRIPRISM = 6, B_OCTAHEDRON = 7, B_TETRAHEDRON = 8, B_QUAD_BEZIER = 9, B_CUBIC_BEZIER = 10,
  B_CATMULL_ROM = 11
};
constexpr int F_T = 1, F_R = 2, F_S1 = 4, F_S3 = 8;
enum StepMode : int { STEP_HARD = 0, STEP_LAPLACE = 1, STEP_LINEAR = 2 };

__host__ __device__ __forceinline__ int kind_base(int k) { return k & 15; }
__host__ __device__ __forceinline__ int kind_flags(int k) { return (k >> 4) & 15; }
__host__ __device__ __forceinline__ int kind_step(int k) { return (k >> 8) & 3; }

// Number of leading base parameters per base (the reference strokes.py:40-82 tables).
__host__ __device__ __forceinline__ int base_param_count(int base) {
  switch (base) {
    case B_ROUND_CUBE: return 1;
    case B_CAPPED_TORUS: return 2;
    case B_CAPSULE: return 1;
    case B_LINE: return 2;
    case B_TRIPRISM: return 1;
    case B_QUAD_BEZIER: return 11;
    case B_CUBIC_BEZIER: return 14;
    case B_CATMULL_ROM: return 14;
    default: return 0;
  }
}
__host__ __device__ __forceinline__ bool base_supported(int base) {
  return base == B_SPHERE || base == B_CUBE || base == B_ROUND_CUBE || base == B_CAPSULE ||
         base == B_OCTAHEDRON || base == B_TETRAHEDRON || base == B_QUAD_BEZIER ||
         base == B_CUBIC_BEZIER;
}
// Shape-parameter count of a reference sdf_id (strokes.py:227-252).
__host__ __device__ __forceinline__ int sdf_id_param_count(int sdf_id) {
  int base = sdf_id >> 4;
  int n = base_param_count(base);
  if (sdf_id & F_S1) n += 1;
  else if (sdf_id & F_S3) n += 3;
  if (sdf_id & F_R) n += 3;
  if (sdf_id & F_T) n += 3;
  return n;
}

// ---- record field offsets
constexpr int R_KIND = 0;      // int bits
constexpr int R_COLOR = 1;     // 3
constexpr int R_DENSITY = 4;
constexpr int R_KFIX = 5;      // kappa/delta (times s for single-scale with inv_scale_radius)
constexpr int R_DELTA = 6;
constexpr int R_CULL_R = 7;    // culling sphere radius (world)
constexpr int R_CULL_C = 8;    // 3, culling sphere centre (world)
constexpr int R_CULL_M = 11;   // culling margin per unit sample radius
// primitives
constexpr int R_M = 12;        // 9, rows of M = S^-1 R^T
constexpr int R_T = 21;        // 3, translation
constexpr int R_S = 24;        // 3, scale per axis
constexpr int R_SINV = 27;     // 3, 1/scale per axis
constexpr int R_BP = 30;       // base parameter (round-cube radius / capsule half-length)
// quadratic Bezier
constexpr int R_QA = 12, R_QB = 15, R_QC = 18;     // control points
constexpr int R_Qa = 21, R_Qb = 24, R_Qc = 27;     // a = B-A, b = A-2B+C, c = 2a
constexpr int R_QR1 = 30, R_QR2 = 31;
constexpr int R_QKK = 32, R_QKX = 33, R_QAA2 = 34; // 1/|b|^2, kk*(a.b), 2|a|^2
constexpr int R_QAB = 35;                          // a.b
// cubic Bezier
constexpr int R_CA = 12, R_CB = 15, R_CC = 18, R_CD = 21;
constexpr int R_CR1 = 24, R_CR2 = 25;
constexpr int R_CV = 26;       // 11 polyline vertices, 33 floats (26..58)
constexpr int CUBIC_SEGMENTS = 10;

// ---- per-stroke reduced-gradient slots (GRAD_SLOTS floats per stroke)
constexpr int GRAD_SLOTS = 32;
constexpr int G_COLOR = 0;     // 3: sum g_C * w
constexpr int G_DENSITY = 3;   // sum g_sigma * w
constexpr int G_K = 4;         // sum dL/dk * k  (softness and scale-through-width)
// primitives
constexpr int G_GP = 5;        // 3: sum of dL/dp (local frame)
constexpr int G_TORQUE = 8;    // 3: sum (S^-1 g_p) x (S p)
constexpr int G_SCALE = 11;    // 3: per-axis scale gradient (S1 uses the first)
constexpr int G_BP = 14;       // base parameter
constexpr int G_PRIM_USED = 15;
// Beziers: raw control-point and radius gradients
constexpr int G_CTRL = 5;      // quad: 9 + r1, r2 (5..15); cubic: 12 + r1, r2 (5..18)

__device__ __forceinline__ V3 ld3(const float* p) { return v3(p[0], p[1], p[2]); }

}  // namespace n3ds
