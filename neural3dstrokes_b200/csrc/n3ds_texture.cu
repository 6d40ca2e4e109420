// Image texture modulation of stroke colours and alphas (the reference's ImageTexture,
// source/textures.py:36-83), one thread per (sample, stroke) pair:
//   tint    = bilinear sample of the texture [C, H, W] at texcoord (u, v), as
//             F.grid_sample(image, (u, v) * 2 - 1, align_corners=True) with zero
//             padding outside the image (textures.py:58-60);
//   colour' = (colour * tint_ratio + (1 - tint_ratio)) * tint   (C = 1 broadcasts)
//   alpha'  = alpha * mean(tint) when modulate_alpha, else alpha  (textures.py:77-81).
// The backward gives dL/dcolour = dL/dcolour' * tint * tint_ratio and dL/dalpha =
// dL/dalpha' * mean(tint) (or the identity); the texture is a buffer and texcoords
// carry no gradient in the reference, so neither gets one here.
//
// Traffic: texcoord 8 B, colour 12 B, alpha 4 B in, colour 12 B and alpha 4 B out per
// pair (40 B); the texture itself (256 x 256 x 3 floats = 768 KB by default) stays in
// L2 / L1 after the first touches. The texel gathers are L1-lookup bound, so the
// packed entry points read float4 texels: 4 lookups per pair instead of 12.
#include <algorithm>
#include <cstdint>
#include <string>

#include <cuda_runtime.h>

#include "../../include/n3ds.h"

namespace n3ds {
int report_error(int code, const std::string& msg);  // sets n3ds_last_error (n3ds_capi.cu)
}

namespace {

struct Tex {
  const float* image;  // [C, H, W]
  int C, H, W;
};

// Bilinear tap of channel c at unnormalised pixel coordinates (ix, iy), corners
// outside the image read as zero.
__device__ __forceinline__ float tex_value(const Tex& t, int c, int x, int y) {
  if (x < 0 || y < 0 || x >= t.W || y >= t.H) return 0.f;
  return __ldg(t.image + ((size_t)c * t.H + y) * t.W + x);
}

// tint[0..C-1] at texcoord (u, v), with grid_sample's unnormalisation for
// align_corners=True: ix = ((g + 1) / 2) (W - 1), g = u * 2 - 1.
__device__ __forceinline__ void sample_tint(const Tex& t, float u, float v, float* tint) {
  const float gx = u * 2.f - 1.f, gy = v * 2.f - 1.f;
  // beyond one pixel outside the image every corner reads zero, so clamping there
  // changes nothing and keeps the integer conversion in range
  const float ix = fminf(fmaxf(((gx + 1.f) / 2.f) * (float)(t.W - 1), -2.f), (float)t.W + 1.f);
  const float iy = fminf(fmaxf(((gy + 1.f) / 2.f) * (float)(t.H - 1), -2.f), (float)t.H + 1.f);
  const float fx = floorf(ix), fy = floorf(iy);
  const int x0 = (int)fx, y0 = (int)fy;
  const float wx1 = ix - fx, wx0 = (fx + 1.f) - ix;
  const float wy1 = iy - fy, wy0 = (fy + 1.f) - iy;
  for (int c = 0; c < t.C; c++) {
    tint[c] = tex_value(t, c, x0, y0) * (wx0 * wy0) + tex_value(t, c, x0 + 1, y0) * (wx1 * wy0) +
              tex_value(t, c, x0, y0 + 1) * (wx0 * wy1) + tex_value(t, c, x0 + 1, y0 + 1) * (wx1 * wy1);
  }
}

// The same tap on the texture packed as [H, W] float4 texels (r, g, b, 0; a grayscale
// texture replicated into r, g, b): one 16-byte load per corner instead of one per
// corner and channel. The sums keep the planar order, so the tints are equal.
__device__ __forceinline__ float4 texel(const float4* img, int W, int H, int x, int y) {
  if (x < 0 || y < 0 || x >= W || y >= H) return make_float4(0.f, 0.f, 0.f, 0.f);
  return __ldg(img + (size_t)y * W + x);
}

__device__ __forceinline__ void sample_tint_packed(const float4* img, int H, int W, float u, float v, float* tint) {
  const float gx = u * 2.f - 1.f, gy = v * 2.f - 1.f;
  const float ix = fminf(fmaxf(((gx + 1.f) / 2.f) * (float)(W - 1), -2.f), (float)W + 1.f);
  const float iy = fminf(fmaxf(((gy + 1.f) / 2.f) * (float)(H - 1), -2.f), (float)H + 1.f);
  const float fx = floorf(ix), fy = floorf(iy);
  const int x0 = (int)fx, y0 = (int)fy;
  const float wx1 = ix - fx, wx0 = (fx + 1.f) - ix;
  const float wy1 = iy - fy, wy0 = (fy + 1.f) - iy;
  const float4 t00 = texel(img, W, H, x0, y0), t10 = texel(img, W, H, x0 + 1, y0);
  const float4 t01 = texel(img, W, H, x0, y0 + 1), t11 = texel(img, W, H, x0 + 1, y0 + 1);
  const float w00 = wx0 * wy0, w10 = wx1 * wy0, w01 = wx0 * wy1, w11 = wx1 * wy1;
  tint[0] = t00.x * w00 + t10.x * w10 + t01.x * w01 + t11.x * w11;
  tint[1] = t00.y * w00 + t10.y * w10 + t01.y * w01 + t11.y * w11;
  tint[2] = t00.z * w00 + t10.z * w10 + t01.z * w01 + t11.z * w11;
}

// Non-finite coordinates give a zero tint (no pixel is read).
__device__ __forceinline__ bool coords_ok(float u, float v) { return isfinite(u) && isfinite(v); }

template <bool PACKED>
__device__ __forceinline__ void tint_at(const Tex& t, float u, float v, float* tint) {
  tint[0] = tint[1] = tint[2] = 0.f;
  if (!coords_ok(u, v)) return;
  if (PACKED) {
    sample_tint_packed(reinterpret_cast<const float4*>(t.image), t.H, t.W, u, v, tint);
  } else {
    sample_tint(t, u, v, tint);
    if (t.C == 1) tint[1] = tint[2] = tint[0];
  }
}

template <bool PACKED>
__global__ void texture_fwd_kernel(float* color_out, float* alpha_out, const float* texcoords, const float* colors,
                                   const float* alphas, long long n, Tex t, float tint_ratio, int modulate) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    float tint[3];
    tint_at<PACKED>(t, texcoords[2 * i], texcoords[2 * i + 1], tint);
    const float base = 1.f - tint_ratio;
    color_out[3 * i] = (colors[3 * i] * tint_ratio + base) * tint[0];
    color_out[3 * i + 1] = (colors[3 * i + 1] * tint_ratio + base) * tint[1];
    color_out[3 * i + 2] = (colors[3 * i + 2] * tint_ratio + base) * tint[2];
    if (alpha_out) {
      const float a = alphas[i];
      alpha_out[i] = modulate ? a * (t.C == 1 ? tint[0] : (tint[0] + tint[1] + tint[2]) / 3.f) : a;
    }
  }
}

template <bool PACKED>
__global__ void texture_bwd_kernel(float* grad_colors, float* grad_alphas, const float* g_color,
                                   const float* g_alpha, const float* texcoords, long long n, Tex t,
                                   float tint_ratio, int modulate) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    float tint[3];
    tint_at<PACKED>(t, texcoords[2 * i], texcoords[2 * i + 1], tint);
    if (grad_colors) {
      for (int k = 0; k < 3; k++) grad_colors[3 * i + k] = g_color ? g_color[3 * i + k] * tint[k] * tint_ratio : 0.f;
    }
    if (grad_alphas) {
      const float g = g_alpha ? g_alpha[i] : 0.f;
      grad_alphas[i] = modulate ? g * (t.C == 1 ? tint[0] : (tint[0] + tint[1] + tint[2]) / 3.f) : g;
    }
  }
}

// Packed texture, four pairs per thread: texcoords as two float4, colours and the
// outputs as three float4 (12 floats = four RGB triples), alphas as one. For
// 16-byte-aligned arrays; pairs past 4 * n4 go to the scalar kernels.
__device__ __forceinline__ void tints4(const Tex& t, const float4& ta, const float4& tb, float (&tn)[12]) {
  const float u[4] = {ta.x, ta.z, tb.x, tb.z}, v[4] = {ta.y, ta.w, tb.y, tb.w};
#pragma unroll
  for (int k = 0; k < 4; k++) {
    float tk[3];
    tint_at<true>(t, u[k], v[k], tk);
    tn[3 * k] = tk[0];
    tn[3 * k + 1] = tk[1];
    tn[3 * k + 2] = tk[2];
  }
}

__device__ __forceinline__ float mean_tint(const Tex& t, const float (&tn)[12], int k) {
  return t.C == 1 ? tn[3 * k] : (tn[3 * k] + tn[3 * k + 1] + tn[3 * k + 2]) / 3.f;
}

__global__ void texture_fwd_vec_kernel(float4* color_out, float4* alpha_out, const float4* texcoords,
                                       const float4* colors, const float4* alphas, long long n4, Tex t,
                                       float tint_ratio, int modulate) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n4; q += (long long)gridDim.x * blockDim.x) {
    float tn[12];
    tints4(t, texcoords[2 * q], texcoords[2 * q + 1], tn);
    const float base = 1.f - tint_ratio;
#pragma unroll
    for (int j = 0; j < 3; j++) {
      const float4 c = colors[3 * q + j];
      color_out[3 * q + j] = make_float4((c.x * tint_ratio + base) * tn[4 * j], (c.y * tint_ratio + base) * tn[4 * j + 1],
                                         (c.z * tint_ratio + base) * tn[4 * j + 2],
                                         (c.w * tint_ratio + base) * tn[4 * j + 3]);
    }
    if (alpha_out) {
      float4 a = alphas[q];
      if (modulate) {
        a.x *= mean_tint(t, tn, 0);
        a.y *= mean_tint(t, tn, 1);
        a.z *= mean_tint(t, tn, 2);
        a.w *= mean_tint(t, tn, 3);
      }
      alpha_out[q] = a;
    }
  }
}

__global__ void texture_bwd_vec_kernel(float4* grad_colors, float4* grad_alphas, const float4* g_color,
                                       const float4* g_alpha, const float4* texcoords, long long n4, Tex t,
                                       float tint_ratio, int modulate) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n4; q += (long long)gridDim.x * blockDim.x) {
    float tn[12];
    tints4(t, texcoords[2 * q], texcoords[2 * q + 1], tn);
    if (grad_colors) {
#pragma unroll
      for (int j = 0; j < 3; j++) {
        const float4 g = g_color ? g_color[3 * q + j] : make_float4(0.f, 0.f, 0.f, 0.f);
        grad_colors[3 * q + j] = make_float4(g.x * tn[4 * j] * tint_ratio, g.y * tn[4 * j + 1] * tint_ratio,
                                             g.z * tn[4 * j + 2] * tint_ratio, g.w * tn[4 * j + 3] * tint_ratio);
      }
    }
    if (grad_alphas) {
      float4 g = g_alpha ? g_alpha[q] : make_float4(0.f, 0.f, 0.f, 0.f);
      if (modulate) {
        g.x *= mean_tint(t, tn, 0);
        g.y *= mean_tint(t, tn, 1);
        g.z *= mean_tint(t, tn, 2);
        g.w *= mean_tint(t, tn, 3);
      }
      grad_alphas[q] = g;
    }
  }
}

bool al16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

// [C, H, W] -> [H, W] float4 texels (r, g, b, 0), grayscale replicated.
__global__ void texture_pack_kernel(float4* packed, const float* image, int C, int H, int W) {
  const long long hw = (long long)H * W;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < hw; i += (long long)gridDim.x * blockDim.x) {
    const float r = image[i];
    packed[i] = C == 1 ? make_float4(r, r, r, 0.f) : make_float4(r, image[hw + i], image[2 * hw + i], 0.f);
  }
}

int check_texture(int64_t n, const float* texcoords, const float* image, int32_t channels, int32_t height,
                  int32_t width) {
  if (n < 0) return n3ds::report_error(N3DS_ERR_INVALID, "texture: n must be >= 0");
  if (channels != 1 && channels != 3)
    return n3ds::report_error(N3DS_ERR_INVALID, "texture: the image must have 1 (grayscale) or 3 (RGB) channels, got " +
                                                    std::to_string(channels));
  if (height < 1 || width < 1) return n3ds::report_error(N3DS_ERR_INVALID, "texture: image height and width must be >= 1");
  if (n > 0 && (!texcoords || !image)) return n3ds::report_error(N3DS_ERR_INVALID, "texture: texcoords and image required");
  return N3DS_OK;
}

// Blocks of 256 threads for n items of a grid-stride kernel: at most one wave of the
// blocks of `kernel` that fit on the device together (a capped grid larger than that
// leaves a partial last wave).
template <typename K>
unsigned grid_for(K kernel, long long n) {
  const long long blocks = (n + 255) / 256;
  int dev = 0, sms = 148, per_sm = 8;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) !=
                                                 cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, 256, 0) != cudaSuccess || per_sm < 1) {
    sms = 148;
    per_sm = 8;
  }
  return (unsigned)std::max<long long>(1, std::min<long long>(blocks, (long long)sms * per_sm));
}

}  // namespace

extern "C" int n3ds_texture_forward(float* color_out, float* alpha_out, const float* texcoords, const float* colors,
                                    const float* alphas, int64_t n, const float* image, int32_t channels,
                                    int32_t height, int32_t width, float tint_ratio, int32_t modulate_alpha,
                                    n3ds_stream_t stream) {
  int rc = check_texture(n, texcoords, image, channels, height, width);
  if (rc) return rc;
  if (n > 0 && (!color_out || !colors)) return n3ds::report_error(N3DS_ERR_INVALID, "texture: colors and color_out required");
  if (n > 0 && alpha_out && !alphas) return n3ds::report_error(N3DS_ERR_INVALID, "texture: alpha_out needs alphas");
  if (n == 0) return N3DS_OK;
  Tex t{image, channels, height, width};
  const unsigned grid = grid_for(texture_fwd_kernel<false>, n);
  texture_fwd_kernel<false><<<grid, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      color_out, alpha_out, texcoords, colors, alphas, n, t, tint_ratio, modulate_alpha != 0);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return n3ds::report_error(N3DS_ERR_CUDA, std::string("texture forward: ") + cudaGetErrorString(e));
  return N3DS_OK;
}

extern "C" int n3ds_texture_backward(float* grad_colors, float* grad_alphas, const float* grad_color_out,
                                     const float* grad_alpha_out, const float* texcoords, int64_t n,
                                     const float* image, int32_t channels, int32_t height, int32_t width,
                                     float tint_ratio, int32_t modulate_alpha, n3ds_stream_t stream) {
  int rc = check_texture(n, texcoords, image, channels, height, width);
  if (rc) return rc;
  if (n == 0 || (!grad_colors && !grad_alphas)) return N3DS_OK;
  Tex t{image, channels, height, width};
  const unsigned grid = grid_for(texture_bwd_kernel<false>, n);
  texture_bwd_kernel<false><<<grid, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      grad_colors, grad_alphas, grad_color_out, grad_alpha_out, texcoords, n, t, tint_ratio, modulate_alpha != 0);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return n3ds::report_error(N3DS_ERR_CUDA, std::string("texture backward: ") + cudaGetErrorString(e));
  return N3DS_OK;
}

extern "C" int n3ds_texture_pack(float* packed, const float* image, int32_t channels, int32_t height, int32_t width,
                                 n3ds_stream_t stream) {
  int rc = check_texture(0, nullptr, image, channels, height, width);
  if (rc) return rc;
  if (!packed || !image) return n3ds::report_error(N3DS_ERR_INVALID, "texture pack: image and packed required");
  if (reinterpret_cast<uintptr_t>(packed) % 16)
    return n3ds::report_error(N3DS_ERR_INVALID, "texture pack: packed must be 16-byte aligned");
  const unsigned grid = grid_for(texture_pack_kernel, (long long)height * width);
  texture_pack_kernel<<<grid, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      reinterpret_cast<float4*>(packed), image, channels, height, width);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return n3ds::report_error(N3DS_ERR_CUDA, std::string("texture pack: ") + cudaGetErrorString(e));
  return N3DS_OK;
}

extern "C" int n3ds_texture_forward_packed(float* color_out, float* alpha_out, const float* texcoords,
                                           const float* colors, const float* alphas, int64_t n, const float* packed,
                                           int32_t channels, int32_t height, int32_t width, float tint_ratio,
                                           int32_t modulate_alpha, n3ds_stream_t stream) {
  int rc = check_texture(n, texcoords, packed, channels, height, width);
  if (rc) return rc;
  if (n > 0 && (!color_out || !colors)) return n3ds::report_error(N3DS_ERR_INVALID, "texture: colors and color_out required");
  if (n > 0 && alpha_out && !alphas) return n3ds::report_error(N3DS_ERR_INVALID, "texture: alpha_out needs alphas");
  if (packed && reinterpret_cast<uintptr_t>(packed) % 16)
    return n3ds::report_error(N3DS_ERR_INVALID, "texture: packed must be 16-byte aligned");
  if (n == 0) return N3DS_OK;
  Tex t{packed, channels, height, width};
  const cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  long long done = 0;
  if (al16(color_out) && al16(texcoords) && al16(colors) && (!alpha_out || (al16(alpha_out) && al16(alphas)))) {
    const long long n4 = n / 4;
    if (n4 > 0)
      texture_fwd_vec_kernel<<<grid_for(texture_fwd_vec_kernel, n4), 256, 0, st>>>(
          reinterpret_cast<float4*>(color_out), reinterpret_cast<float4*>(alpha_out),
          reinterpret_cast<const float4*>(texcoords), reinterpret_cast<const float4*>(colors),
          reinterpret_cast<const float4*>(alphas), n4, t, tint_ratio, modulate_alpha != 0);
    done = 4 * n4;
  }
  if (done < n)
    texture_fwd_kernel<true><<<grid_for(texture_fwd_kernel<true>, n - done), 256, 0, st>>>(
        color_out + 3 * done, alpha_out ? alpha_out + done : nullptr, texcoords + 2 * done, colors + 3 * done,
        alphas ? alphas + done : nullptr, n - done, t, tint_ratio, modulate_alpha != 0);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return n3ds::report_error(N3DS_ERR_CUDA, std::string("texture forward: ") + cudaGetErrorString(e));
  return N3DS_OK;
}

extern "C" int n3ds_texture_backward_packed(float* grad_colors, float* grad_alphas, const float* grad_color_out,
                                            const float* grad_alpha_out, const float* texcoords, int64_t n,
                                            const float* packed, int32_t channels, int32_t height, int32_t width,
                                            float tint_ratio, int32_t modulate_alpha, n3ds_stream_t stream) {
  int rc = check_texture(n, texcoords, packed, channels, height, width);
  if (rc) return rc;
  if (packed && reinterpret_cast<uintptr_t>(packed) % 16)
    return n3ds::report_error(N3DS_ERR_INVALID, "texture: packed must be 16-byte aligned");
  if (n == 0 || (!grad_colors && !grad_alphas)) return N3DS_OK;
  Tex t{packed, channels, height, width};
  const cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  long long done = 0;
  if (al16(texcoords) && (!grad_colors || al16(grad_colors)) && (!grad_color_out || al16(grad_color_out)) &&
      (!grad_alphas || al16(grad_alphas)) && (!grad_alpha_out || al16(grad_alpha_out))) {
    const long long n4 = n / 4;
    if (n4 > 0)
      texture_bwd_vec_kernel<<<grid_for(texture_bwd_vec_kernel, n4), 256, 0, st>>>(
          reinterpret_cast<float4*>(grad_colors), reinterpret_cast<float4*>(grad_alphas),
          reinterpret_cast<const float4*>(grad_color_out), reinterpret_cast<const float4*>(grad_alpha_out),
          reinterpret_cast<const float4*>(texcoords), n4, t, tint_ratio, modulate_alpha != 0);
    done = 4 * n4;
  }
  if (done < n)
    texture_bwd_kernel<true><<<grid_for(texture_bwd_kernel<true>, n - done), 256, 0, st>>>(
        grad_colors ? grad_colors + 3 * done : nullptr, grad_alphas ? grad_alphas + done : nullptr,
        grad_color_out ? grad_color_out + 3 * done : nullptr, grad_alpha_out ? grad_alpha_out + done : nullptr,
        texcoords + 2 * done, n - done, t, tint_ratio, modulate_alpha != 0);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return n3ds::report_error(N3DS_ERR_CUDA, std::string("texture backward: ") + cudaGetErrorString(e));
  return N3DS_OK;
}
