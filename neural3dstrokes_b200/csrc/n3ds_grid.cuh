// Device helpers of the multi-resolution grid encoder, shared by the encoder's own
// kernels (n3ds_grid.cu) and the fused density network (n3ds_propnet.cu): level
// geometry, the row index of a cell (dense or coherent prime hash), row loads and
// scatters, and the cell / corner arithmetic, each following the reference's
// source/gridencoder/src/gridencoder.cu at the lines cited.
#pragma once
#include <cstdint>
#include <type_traits>

#include <cuda_fp16.h>
#include <cuda_runtime.h>

namespace n3ds {
namespace grid {

constexpr uint32_t kPairMinRows = 1u << 19;  // smallest level that uses paired row loads

// Coherent hash primes of the reference (gridencoder.cu:51), the first seven of
// Instant-NGP's table; prime 1 keeps x coherent.
static __device__ __constant__ uint32_t kPrimes[7] = {1u, 2654435761u, 805459861u, 3674653429u,
                                                      2097192037u, 1434869437u, 2165219737u};

// Accumulator type: float for float and half tables, double for double.
template <typename T> struct Acc { using type = float; };
template <> struct Acc<double> { using type = double; };

template <typename T> __device__ __forceinline__ typename Acc<T>::type to_acc(T v) { return (typename Acc<T>::type)v; }
template <> __device__ __forceinline__ float to_acc<__half>(__half v) { return __half2float(v); }
template <typename T> __device__ __forceinline__ T from_acc(typename Acc<T>::type v) { return (T)v; }
template <> __device__ __forceinline__ __half from_acc<__half>(float v) { return __float2half_rn(v); }

struct Level {
  uint32_t base;   // first row of the level
  uint32_t hsize;  // rows of the level
  uint32_t res;    // resolution (cells per axis + 1, the reference's ceil(scale) + 1)
  float scale;     // 2^(level S) H - 1
  bool pow2;       // hsize is a power of two: modulo by mask
};

// gridencoder.cu:126-128.
__device__ __forceinline__ Level level_of(const int32_t* offsets, uint32_t level, float S, uint32_t H) {
  Level lv;
  const uint32_t o0 = (uint32_t)__ldg(offsets + level), o1 = (uint32_t)__ldg(offsets + level + 1);
  lv.base = o0;
  lv.hsize = o1 - o0;
  lv.scale = fmaf(exp2f((float)level * S), (float)H, -1.f);
  lv.res = (uint32_t)ceilf(lv.scale) + 1u;
  lv.pow2 = (lv.hsize & (lv.hsize - 1u)) == 0u;
  return lv;
}

// Row within the level of integer cell c (get_grid_index, gridencoder.cu:65-82):
// row-major over the (res or res + 1)^D lattice while it fits, else (hash grids)
// the XOR of cell x prime; both taken modulo the level's row count. uint32 math.
template <int D>
__device__ __forceinline__ uint32_t cell_row(const uint32_t (&c)[D], const Level& lv, bool hash, bool align) {
  const uint32_t mult = align ? lv.res : lv.res + 1u;
  uint32_t stride = 1u, index = 0u;
#pragma unroll
  for (int d = 0; d < D; d++) {
    if (stride > lv.hsize) break;
    index += c[d] * stride;
    stride *= mult;
  }
  if (hash && stride > lv.hsize) {
    index = 0u;
#pragma unroll
    for (int d = 0; d < D; d++) index ^= c[d] * kPrimes[d];
  }
  return lv.pow2 ? (index & (lv.hsize - 1u)) : (index % lv.hsize);
}

// C values of one row, as one vector load where the table allows it.
template <typename T, int C>
__device__ __forceinline__ void load_row(const T* __restrict__ row, bool vec, typename Acc<T>::type (&v)[C]) {
  if constexpr (std::is_same<T, float>::value && (C == 2 || C == 4 || C == 8)) {
    if (vec) {
      if constexpr (C == 2) {
        const float2 a = __ldg(reinterpret_cast<const float2*>(row));
        v[0] = a.x; v[1] = a.y;
      } else {
#pragma unroll
        for (int k = 0; k < C; k += 4) {
          const float4 a = __ldg(reinterpret_cast<const float4*>(row + k));
          v[k] = a.x; v[k + 1] = a.y; v[k + 2] = a.z; v[k + 3] = a.w;
        }
      }
      return;
    }
  }
  if constexpr (std::is_same<T, __half>::value && (C == 4 || C == 8)) {
    if (vec) {
      if constexpr (C == 4) {
        const uint2 a = __ldg(reinterpret_cast<const uint2*>(row));
        const float2 lo = __half22float2(*reinterpret_cast<const __half2*>(&a.x));
        const float2 hi = __half22float2(*reinterpret_cast<const __half2*>(&a.y));
        v[0] = lo.x; v[1] = lo.y; v[2] = hi.x; v[3] = hi.y;
      } else {
        const uint4 a = __ldg(reinterpret_cast<const uint4*>(row));
        const uint32_t w[4] = {a.x, a.y, a.z, a.w};
#pragma unroll
        for (int k = 0; k < 4; k++) {
          const float2 f = __half22float2(*reinterpret_cast<const __half2*>(&w[k]));
          v[2 * k] = f.x; v[2 * k + 1] = f.y;
        }
      }
      return;
    }
  }
#pragma unroll
  for (int k = 0; k < C; k++) v[k] = to_acc<T>(row[k]);
}

// Bytes of an aligned pair of rows (2k, 2k + 1) when one vector load can fetch it
// (float C = 1, 2, 4: 8, 16, 32 B; half C = 2, 4: 8, 16 B), else 0.
template <typename T, int C>
__host__ __device__ constexpr int pair_bytes() {
  return (std::is_same<T, float>::value && C <= 4) || (std::is_same<T, __half>::value && (C == 2 || C == 4))
             ? 2 * C * (int)sizeof(T)
             : 0;
}

// Rows r0 and r1 of a level. When both lie in one aligned pair (r0 >> 1 == r1 >> 1:
// the x-neighbours of a cell with even x under the coherent hash, or of an even
// row in a dense level) one load of the pair serves both, one L1 lookup instead of
// two; the 32-byte case uses the sm_100 256-bit load.
template <typename T, int C>
__device__ __forceinline__ void load_rows2(const T* __restrict__ tab, uint32_t r0, uint32_t r1, bool vec, bool vec_pair,
                                           typename Acc<T>::type (&v0)[C], typename Acc<T>::type (&v1)[C]) {
  constexpr int P = pair_bytes<T, C>();
  if constexpr (P > 0) {
    // vec_pair: the table is aligned to the pair, the level starts on an even row and
    // row r0 | 1 exists (offsets from the C ABI may be odd)
    if (vec_pair && (r0 >> 1) == (r1 >> 1)) {
      const T* base = tab + (size_t)(r0 & ~1u) * C;
      float lo[C], hi[C];
      if constexpr (P == 32) {
        float a[8];
        asm("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
            : "=f"(a[0]), "=f"(a[1]), "=f"(a[2]), "=f"(a[3]), "=f"(a[4]), "=f"(a[5]), "=f"(a[6]), "=f"(a[7])
            : "l"(base));
#pragma unroll
        for (int k = 0; k < 4; k++) { lo[k] = a[k]; hi[k] = a[4 + k]; }
      } else if constexpr (std::is_same<T, float>::value) {
        if constexpr (P == 16) {
          const float4 a = __ldg(reinterpret_cast<const float4*>(base));
          lo[0] = a.x; lo[1] = a.y; hi[0] = a.z; hi[1] = a.w;
        } else {
          const float2 a = __ldg(reinterpret_cast<const float2*>(base));
          lo[0] = a.x; hi[0] = a.y;
        }
      } else {  // half, 8 or 16 bytes
        uint32_t w[4];
        if constexpr (P == 16) {
          const uint4 a = __ldg(reinterpret_cast<const uint4*>(base));
          w[0] = a.x; w[1] = a.y; w[2] = a.z; w[3] = a.w;
        } else {
          const uint2 a = __ldg(reinterpret_cast<const uint2*>(base));
          w[0] = a.x; w[1] = a.y;
        }
        float f[2 * C];
#pragma unroll
        for (int k = 0; k < C; k++) {
          const float2 h = __half22float2(*reinterpret_cast<const __half2*>(&w[k]));
          f[2 * k] = h.x; f[2 * k + 1] = h.y;
        }
#pragma unroll
        for (int k = 0; k < C; k++) { lo[k] = f[k]; hi[k] = f[C + k]; }
      }
#pragma unroll
      for (int k = 0; k < C; k++) {
        v0[k] = (r0 & 1u) ? hi[k] : lo[k];
        v1[k] = (r1 & 1u) ? hi[k] : lo[k];
      }
      return;
    }
  }
  load_row<T, C>(tab + (size_t)r0 * C, vec, v0);
  load_row<T, C>(tab + (size_t)r1 * C, vec, v1);
}

template <typename T, int C>
__device__ __forceinline__ void store_row(T* __restrict__ row, bool vec, const typename Acc<T>::type (&v)[C]) {
  if constexpr (std::is_same<T, float>::value && (C == 2 || C == 4 || C == 8)) {
    if (vec) {
      if constexpr (C == 2) {
        *reinterpret_cast<float2*>(row) = make_float2(v[0], v[1]);
      } else {
#pragma unroll
        for (int k = 0; k < C; k += 4)
          *reinterpret_cast<float4*>(row + k) = make_float4(v[k], v[k + 1], v[k + 2], v[k + 3]);
      }
      return;
    }
  }
#pragma unroll
  for (int k = 0; k < C; k++) row[k] = from_acc<T>(v[k]);
}

// row[k] += v[k] for k < C, atomically: vector float atomics where aligned, __half2
// pairs for half tables, scalar otherwise.
template <typename T, int C>
__device__ __forceinline__ void scatter_row(T* row, bool vec, const typename Acc<T>::type (&v)[C]) {
  if constexpr (std::is_same<T, float>::value && (C == 2 || C == 4 || C == 8)) {
    if (vec) {
      if constexpr (C == 2) {
        atomicAdd(reinterpret_cast<float2*>(row), make_float2(v[0], v[1]));
      } else {
#pragma unroll
        for (int k = 0; k < C; k += 4)
          atomicAdd(reinterpret_cast<float4*>(row + k), make_float4(v[k], v[k + 1], v[k + 2], v[k + 3]));
      }
      return;
    }
  }
  if constexpr (std::is_same<T, __half>::value && C >= 2) {
    if (vec) {
#pragma unroll
      for (int k = 0; k < C; k += 2) atomicAdd(reinterpret_cast<__half2*>(row + k), __floats2half2_rn(v[k], v[k + 1]));
      return;
    }
  }
#pragma unroll
  for (int k = 0; k < C; k++) atomicAdd(row + k, from_acc<T>(v[k]));
}

template <typename P>
__device__ __forceinline__ bool point_in_range(const P* x, int D) {
  bool ok = true;
  for (int d = 0; d < D; d++) {
    const float v = (float)x[d];
    ok &= !(v < 0.f || v > 1.f);  // NaN counts as in range, as in the reference's test
  }
  return ok;
}

// Cell and interpolation fractions of a point at one level (gridencoder.cu:134-150).
template <int D>
__device__ __forceinline__ void locate(const float* x, const Level& lv, bool align, bool smooth, uint32_t (&cell)[D],
                                       float (&frac)[D], float (&deriv)[D]) {
#pragma unroll
  for (int d = 0; d < D; d++) {
    const float p = fmaf(x[d], lv.scale, align ? 0.f : 0.5f);
    const float f = floorf(p);
    cell[d] = (uint32_t)f;
    const float t = p - f;
    if (smooth) {
      deriv[d] = 6.f * t * (1.f - t);
      frac[d] = t * t * (3.f - 2.f * t);
    } else {
      deriv[d] = 1.f;
      frac[d] = t;
    }
  }
}

// Weight and cell of corner `corner` (bit d set: the upper neighbour along d),
// the product taken in axis order as the reference does.
template <int D>
__device__ __forceinline__ float corner_of(int corner, const uint32_t (&cell)[D], const float (&frac)[D],
                                           uint32_t (&cc)[D]) {
  float w = 1.f;
#pragma unroll
  for (int d = 0; d < D; d++) {
    const bool up = (corner >> d) & 1;
    w *= up ? frac[d] : 1.f - frac[d];
    cc[d] = cell[d] + (up ? 1u : 0u);
  }
  return w;
}

}  // namespace grid
}  // namespace n3ds
