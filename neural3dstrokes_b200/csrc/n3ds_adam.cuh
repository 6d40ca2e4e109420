// Adam step fused with the parameter clamp (graph-captured training loop).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace n3ds {
cudaError_t launch_adam(float* param, const float* grad, float* m, float* v, const float* lo, const float* hi,
                        long long n, float lr, float b1, float b2, float eps, const int* step, cudaStream_t st);
}
