// MSE loss / gradient (src/layers/mse_loss_layer.cu:22-67) and a multi-tensor
// Adam update (src/optimizers/adam.cu:12-73) that updates every parameter
// group in a single launch instead of one launch per group.
#include "ds_common.cuh"
#include "ds_internal.h"

namespace ds {

namespace {

constexpr int kThreads = 256;

// L = sum_px sum_c (r - t)^2 / P.  Grid-stride, one atomic per CTA.
__global__ void __launch_bounds__(kThreads)
    mse_forward_kernel(const float* __restrict__ px, const float* __restrict__ tgt, int64_t npix,
                       float* __restrict__ loss) {
  __shared__ float red[kThreads / 32];
  const float scale = 1.f / (float)npix;
  float s = 0.f;
  for (int64_t i = blockIdx.x * (int64_t)kThreads + threadIdx.x; i < npix;
       i += (int64_t)gridDim.x * kThreads) {
    float dR = px[i * 3 + 0] - tgt[i * 3 + 0];
    float dG = px[i * 3 + 1] - tgt[i * 3 + 1];
    float dB = px[i * 3 + 2] - tgt[i * 3 + 2];
    s += (dR * dR + dG * dG + dB * dB) * scale;
  }
  s = warp_sum(s);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    float t = 0.f;
    for (int k = 0; k < kThreads / 32; ++k) t += red[k];
    atomicAdd(loss, t);
  }
}

__global__ void __launch_bounds__(kThreads)
    mse_backward_kernel(const float* __restrict__ px, const float* __restrict__ tgt, int64_t npix,
                        float* __restrict__ grad) {
  int64_t i = blockIdx.x * (int64_t)kThreads + threadIdx.x;
  if (i >= npix) return;
  const float scale = 2.f / (float)npix;
  grad[i * 3 + 0] = scale * (px[i * 3 + 0] - tgt[i * 3 + 0]);
  grad[i * 3 + 1] = scale * (px[i * 3 + 1] - tgt[i * 3 + 1]);
  grad[i * 3 + 2] = scale * (px[i * 3 + 2] - tgt[i * 3 + 2]);
}

constexpr int kMaxGroups = 32;
constexpr int kAdamItems = 4;  // elements per thread
constexpr int kAdamSpan = kThreads * kAdamItems;

struct AdamBatch {
  ds_adam_group g[kMaxGroups];
  int first_block[kMaxGroups + 1];
  int n;
  float b1, b2, eps, bc1, bc2;
};

__global__ void __launch_bounds__(kThreads) adam_multi_kernel(const AdamBatch B) {
  const int blk = blockIdx.x;
  int gi = 0;
  while (gi + 1 < B.n && B.first_block[gi + 1] <= blk) ++gi;
  const ds_adam_group G = B.g[gi];
  const int64_t base = (int64_t)(blk - B.first_block[gi]) * kAdamSpan;
#pragma unroll
  for (int k = 0; k < kAdamItems; ++k) {
    const int64_t idx = base + k * kThreads + threadIdx.x;
    if (idx < G.n) {
      float g = G.grad[idx];
      float m = G.m[idx] = B.b1 * G.m[idx] + (1.f - B.b1) * g;
      float v = G.v[idx] = B.b2 * G.v[idx] + (1.f - B.b2) * g * g;
      float m_hat = m * B.bc1;
      float v_hat = v * B.bc2;
      G.param[idx] -= G.lr * m_hat / (sqrtf(v_hat) + B.eps);
    }
  }
}

}  // namespace

int launch_mse_forward(const float* px, const float* tgt, int64_t npix, float* loss, float*,
                       uint32_t*, cudaStream_t s) {
  DS_CUDA(cudaMemsetAsync(loss, 0, sizeof(float), s));
  if (npix <= 0) return DS_OK;
  int64_t want = (npix + kThreads - 1) / kThreads;
  int blocks = (int)(want < 148 * 8 ? want : 148 * 8);
  mse_forward_kernel<<<blocks, kThreads, 0, s>>>(px, tgt, npix, loss);
  return cuda_status(cudaGetLastError());
}

int launch_mse_backward(const float* px, const float* tgt, int64_t npix, float* grad,
                        cudaStream_t s) {
  if (npix <= 0) return DS_OK;
  mse_backward_kernel<<<(unsigned)((npix + kThreads - 1) / kThreads), kThreads, 0, s>>>(
      px, tgt, npix, grad);
  return cuda_status(cudaGetLastError());
}

int launch_adam_multi(const ds_adam_group* groups, int n_groups, float beta1, float beta2,
                      float eps, float bc1, float bc2, cudaStream_t s) {
  int k = 0;
  while (k < n_groups) {
    AdamBatch B;
    B.n = 0;
    B.b1 = beta1;
    B.b2 = beta2;
    B.eps = eps;
    B.bc1 = bc1;
    B.bc2 = bc2;
    int blocks = 0;
    for (; k < n_groups && B.n < kMaxGroups; ++k) {
      if (groups[k].n <= 0) continue;
      B.g[B.n] = groups[k];
      B.first_block[B.n] = blocks;
      blocks += (int)((groups[k].n + kAdamSpan - 1) / kAdamSpan);
      ++B.n;
    }
    B.first_block[B.n] = blocks;
    if (blocks > 0) {
      adam_multi_kernel<<<blocks, kThreads, 0, s>>>(B);
      DS_CUDA(cudaGetLastError());
    }
  }
  return DS_OK;
}

}  // namespace ds
