// Small device-side vector helpers and the soft-step math shared by every kernel.
//
// Float semantics follow the reference strokelib device code where they change
// results: clamp is fmaxf(lo, fminf(x, hi)) (a NaN input maps to hi), and sign tests
// use `v < 0 ? -1 : 1` (never 0).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace n3ds {

struct V3 {
  float x, y, z;
};

__host__ __device__ __forceinline__ V3 v3(float x, float y, float z) { return V3{x, y, z}; }
__host__ __device__ __forceinline__ V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__host__ __device__ __forceinline__ V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__host__ __device__ __forceinline__ V3 operator-(V3 a) { return {-a.x, -a.y, -a.z}; }
__host__ __device__ __forceinline__ V3 operator*(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
__host__ __device__ __forceinline__ V3 operator*(float s, V3 a) { return {a.x * s, a.y * s, a.z * s}; }
__host__ __device__ __forceinline__ V3 operator*(V3 a, V3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
__host__ __device__ __forceinline__ V3 operator/(V3 a, V3 b) { return {a.x / b.x, a.y / b.y, a.z / b.z}; }
__host__ __device__ __forceinline__ V3 operator/(V3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
__host__ __device__ __forceinline__ V3 operator+(V3 a, float s) { return {a.x + s, a.y + s, a.z + s}; }
__host__ __device__ __forceinline__ V3 operator-(V3 a, float s) { return {a.x - s, a.y - s, a.z - s}; }
__host__ __device__ __forceinline__ V3 operator-(float s, V3 a) { return {s - a.x, s - a.y, s - a.z}; }
__host__ __device__ __forceinline__ V3& operator+=(V3& a, V3 b) { a.x += b.x; a.y += b.y; a.z += b.z; return a; }
__host__ __device__ __forceinline__ V3& operator-=(V3& a, V3 b) { a.x -= b.x; a.y -= b.y; a.z -= b.z; return a; }
__host__ __device__ __forceinline__ float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__host__ __device__ __forceinline__ V3 cross(V3 a, V3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__host__ __device__ __forceinline__ V3 vabs(V3 a) { return {fabsf(a.x), fabsf(a.y), fabsf(a.z)}; }
__host__ __device__ __forceinline__ V3 vmax0(V3 a) { return {fmaxf(a.x, 0.f), fmaxf(a.y, 0.f), fmaxf(a.z, 0.f)}; }
__host__ __device__ __forceinline__ float sgn(float v) { return v < 0.f ? -1.f : 1.f; }
__host__ __device__ __forceinline__ V3 vsgn(V3 a) { return {sgn(a.x), sgn(a.y), sgn(a.z)}; }
__host__ __device__ __forceinline__ float clampf(float v, float lo, float hi) { return fmaxf(lo, fminf(v, hi)); }
__host__ __device__ __forceinline__ float max3(V3 a) { return fmaxf(a.x, fmaxf(a.y, a.z)); }

// 3x3 matrix, row-major, stored as three rows.
struct M3 {
  V3 r0, r1, r2;
};
__host__ __device__ __forceinline__ V3 mul(const M3& m, V3 v) { return {dot(m.r0, v), dot(m.r1, v), dot(m.r2, v)}; }
__host__ __device__ __forceinline__ V3 mul_t(const M3& m, V3 v) {  // m^T v
  return m.r0 * v.x + m.r1 * v.y + m.r2 * v.z;
}

// Euler rotation R = Rz(e.z) Ry(e.y) Rx(e.x); the same matrix entries as the
// reference rotate_point (strokes_sdf.h:28-39).
__host__ __device__ inline M3 euler_matrix(V3 e) {
  float sx = sinf(e.x), sy = sinf(e.y), sz = sinf(e.z);
  float cx = cosf(e.x), cy = cosf(e.y), cz = cosf(e.z);
  M3 r;
  r.r0 = {cy * cz, sx * sy * cz - cx * sz, sx * sz + cx * sy * cz};
  r.r1 = {cy * sz, cx * cz + sx * sy * sz, cx * sy * sz - sx * cz};
  r.r2 = {-sy, sx * cy, cx * cy};
  return r;
}

// Laplace-CDF soft step on the argument m = -sdf * k (common.h:48-51):
// alpha = m <= 0 ? exp(m)/2 : 1 - exp(-m)/2, written with one exp of -|m|.
__device__ __forceinline__ float laplace_alpha(float m) {
  float e = 0.5f * __expf(-fabsf(m));
  return m <= 0.f ? e : 1.f - e;
}

__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
// Inclusive prefix sum across the warp (lane order).
__device__ __forceinline__ float warp_inclusive_scan(float v, int lane) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    float n = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += n;
  }
  return v;
}

}  // namespace n3ds
