// FP32 FMA-pipe throughput probe: the denominator of the roofline of the FP32-bound
// stroke kernels (the driver's peak file measures HBM copy and bf16 GEMM only).
// Each thread runs 16 independent FMA chains for `iters` iterations, so the SM's FMA
// pipes stay busy without dependence stalls; one launch performs
// blocks * threads * iters * 16 FMAs (2 flops each).
#include "../../include/n3ds.h"
#include <cuda_runtime.h>

namespace {
__global__ void __launch_bounds__(256) fma_probe_kernel(float* out, int iters, float a, float b) {
  float x[16];
#pragma unroll
  for (int k = 0; k < 16; k++) x[k] = threadIdx.x * 1e-3f + k;
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int k = 0; k < 16; k++) x[k] = fmaf(x[k], a, b);
  }
  float s = 0.f;
#pragma unroll
  for (int k = 0; k < 16; k++) s += x[k];
  if (s == 1234.5f) out[blockIdx.x * blockDim.x + threadIdx.x] = s;  // keeps the chains live
}
}  // namespace

extern "C" int n3ds_fp32_probe(float* out, int32_t blocks, int32_t iters, n3ds_stream_t stream) {
  if (blocks < 1 || iters < 1 || !out) return N3DS_ERR_INVALID;
  fma_probe_kernel<<<blocks, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(out, iters, 0.9999f, 1e-4f);
  return cudaGetLastError() == cudaSuccess ? N3DS_OK : N3DS_ERR_CUDA;
}
