// Adam with bias correction (torch.optim.Adam semantics; the reference builds it with
// betas (0.9, 0.99), eps 1e-15: utils/training.py:119-136), preceded by the
// reference's gradient nan_to_num (utils/training.py:67-78) and followed by its
// parameter clamp (models.py:576-584). The step count is read from device memory so a
// captured CUDA graph can replay it.
#include <cfloat>
#include "n3ds_adam.cuh"

namespace n3ds {

__global__ void adam_kernel(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, const float* __restrict__ lo, const float* __restrict__ hi,
                            long long n, float lr, float b1, float b2, float eps, const int* __restrict__ step) {
  const int t = *step;
  const float bc1 = 1.f - powf(b1, (float)t);
  const float bc2 = 1.f - powf(b2, (float)t);
  const float step_size = lr / bc1;
  const float bc2_sqrt = sqrtf(bc2);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    float gi = g[i];
    if (isnan(gi)) gi = 0.f;
    else if (isinf(gi)) gi = gi > 0.f ? FLT_MAX : -FLT_MAX;
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    float pi = p[i] - step_size * mi / (sqrtf(vi) / bc2_sqrt + eps);
    if (lo) pi = fmaxf(pi, lo[i]);
    if (hi) pi = fminf(pi, hi[i]);
    p[i] = pi;
  }
}

cudaError_t launch_adam(float* param, const float* grad, float* m, float* v, const float* lo, const float* hi,
                        long long n, float lr, float b1, float b2, float eps, const int* step, cudaStream_t st) {
  long long blocks = (n + 255) / 256;
  if (blocks > 148LL * 8) blocks = 148LL * 8;
  adam_kernel<<<(unsigned)blocks, 256, 0, st>>>(param, grad, m, v, lo, hi, n, lr, b1, b2, eps, step);
  return cudaGetLastError();
}

}  // namespace n3ds
