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
// The common primitives: sphere / ellipsoid, cube / box, round cube / box, capsule,
// octahedron, tetrahedron (every stroke of the reference's primitive configurations).
constexpr unsigned COMMON_BASES = (1u << B_SPHERE) | (1u << B_CUBE) | (1u << B_ROUND_CUBE) | (1u << B_CAPSULE) |
                                  (1u << B_OCTAHEDRON) | (1u << B_TETRAHEDRON);
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
__host__ __device__ __forceinline__ bool base_supported(int base) { return base >= 0 && base <= B_CATMULL_ROM; }
// Curves evaluated through the polyline machinery (power-basis coefficients for
// Catmull-Rom, Bernstein control points for the cubic Bezier).
__host__ __device__ __forceinline__ bool base_is_cubic_curve(int base) {
  return base == B_CUBIC_BEZIER || base == B_CATMULL_ROM;
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

// ---- record field offsets (floats). Hot fields sit in 16-byte groups so the inner
// loops read them with 128-bit shared-memory loads (rec4(rec)[k]).
// q0: kind word, soft-step slope, density, softness
constexpr int R_KIND = 0;      // int bits
constexpr int R_KFIX = 1;      // kappa/delta (times s for single-scale with inv_scale_radius)
constexpr int R_DENSITY = 2;
constexpr int R_DELTA = 3;
// q1: colour, base parameter (round-cube radius / capsule half-length)
constexpr int R_COLOR = 4;     // 3
constexpr int R_BP = 7;        // first base parameter (round-cube radius, capsule / line half-length,
                               // torus cap angle, prism half-height)
// primitives
constexpr int R_M = 8;         // q2..q4: rows (m_i0, m_i1, m_i2, t_i), p = M (x - t),
                               // M = S^-1 R^T (t is subtracted first: M x - M t cancels)
constexpr int R_S = 20;        // q5: scale per axis
constexpr int R_SINV = 24;     // q6: 1/scale per axis
// second base parameter and derived constants (primitives; q7)
constexpr int R_BP2 = 28;      // torus tube radius, line radius change
constexpr int R_TSIN = 29, R_TCOS = 30;  // sin, cos of the torus cap angle
constexpr int R_PLANE = 31;    // reach test per unit sample radius: tetrahedron / octahedron sqrt(3) tau_local,
                               // per-axis-scaled sphere and capsule tau_local
// quadratic Bezier
constexpr int R_QA = 8, R_QKK = 11;    // q2: A, 1/|b|^2
constexpr int R_Qa = 12, R_QKX = 15;   // q3: a = B - A, kk (a.b)
constexpr int R_Qb = 16, R_QAA2 = 19;  // q4: b = A - 2B + C, 2 |a|^2
constexpr int R_Qc = 20, R_QAB = 23;   // q5: c = 2a, a.b
constexpr int R_QR1 = 24, R_QR2 = 25;  // q6: radii
// cubic Bezier (Bernstein control points A..D) / Catmull-Rom (power-basis
// coefficients of t^3, t^2, t, 1, strokes_sdf.h:1333-1349)
constexpr int R_CA = 8, R_CR1 = 11;    // q2: A, r1
constexpr int R_CB = 12, R_CR2 = 15;   // q3: B, r2
constexpr int R_CC = 16, R_CD = 20;    // q4, q5: C, D
constexpr int R_CV = 24;       // 11 polyline vertices, 33 floats (24..56), read as 9 float4
// every curve: culling radius of its polyline pieces beyond their half-length (the
// largest tube radius plus the curve's distance bound to its polyline)
constexpr int R_CTEST = 60;
constexpr int CUBIC_SEGMENTS = 10;

__device__ __forceinline__ const float4* rec4(const float* rec) { return reinterpret_cast<const float4*>(rec); }
__device__ __forceinline__ V3 xyz(float4 v) { return {v.x, v.y, v.z}; }

// ---- per-stroke reduced-gradient slots (GRAD_SLOTS floats per stroke)
constexpr int GRAD_SLOTS = 32;
constexpr int G_COLOR = 0;     // 3: sum g_C * w
constexpr int G_DENSITY = 3;   // sum g_sigma * w
constexpr int G_K = 4;         // sum dL/dk * k  (softness and scale-through-width)
// primitives
constexpr int G_GP = 5;        // 3: sum of dL/dp (local frame)
constexpr int G_TORQUE = 8;    // 3: sum (S^-1 g_p) x (S p)
constexpr int G_SCALE = 11;    // 3: per-axis scale gradient (S1 uses the first)
constexpr int G_BP = 14;       // first base parameter
constexpr int G_BP2 = 15;      // second base parameter
// Beziers: raw control-point and radius gradients
constexpr int G_CTRL = 5;      // quad: 9 + r1, r2 (5..15); cubic / Catmull-Rom: 12 + r1, r2 (5..18)

__device__ __forceinline__ V3 ld3(const float* p) { return v3(p[0], p[1], p[2]); }

// Scratch bytes of the drop-in stroke operators for n strokes: a 256-byte header
// (status word), the prepared records, culling spheres (float4) and margins (n + 4
// floats; written by the shared prep kernel), GRAD_SLOTS reduction slots per stroke,
// and 256 bytes of tail padding, each block 256-byte aligned. The one formula behind
// n3ds_stroke_workspace_bytes and the static scratch of n3ds_stroke_forward_static.
__host__ __device__ constexpr size_t stroke_workspace_bytes(size_t n) {
  return 256 + ((n * REC_FLOATS * 4 + 255) & ~size_t(255)) + ((n * 16 + 255) & ~size_t(255)) +
         (((n + 4) * 4 + 255) & ~size_t(255)) + ((n * GRAD_SLOTS * 4 + 255) & ~size_t(255)) + 256;
}

}  // namespace n3ds
