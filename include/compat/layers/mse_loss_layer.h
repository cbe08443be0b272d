// MSELossLayer (src/layers/mse_loss_layer.h:11-44) on libdiffsplat_b200:
// L = sum_px sum_c (r - t)^2 / pixels, dL/dr = 2 (r - t) / pixels.
#pragma once
#include "../cuda/cuda_buffer.h"
#include "ds_compat_views.h"
#include "layer.h"

class MSELossLayer : public Layer {
 public:
  void allocate(int width, int height) {
    num_pixels = (size_t)width * height;
    d_grad_pixels.allocate(num_pixels * 3);
    d_loss.allocate(1);
  }
  void forward() override {
    DS_COMPAT_CHECK(ds_mse_forward(d_in_pixels, d_target_pixels, (int64_t)num_pixels,
                                   d_loss.ptr, nullptr));
  }
  void backward() override {
    DS_COMPAT_CHECK(ds_mse_backward(d_in_pixels, d_target_pixels, (int64_t)num_pixels,
                                    d_grad_pixels.ptr, nullptr));
  }
  void zeroGrad() override { d_grad_pixels.zero(); }
  void setInput(const float* pixels) { d_in_pixels = pixels; }
  void setTarget(const float* target) { d_target_pixels = target; }
  CudaBuffer<float>& getGradInput() { return d_grad_pixels; }
  float getLoss() const {
    float v = 0.f;
    CUDA_CHECK(cudaMemcpy(&v, d_loss.ptr, sizeof(float), cudaMemcpyDeviceToHost));
    return v;
  }

 private:
  const float* d_in_pixels = nullptr;
  const float* d_target_pixels = nullptr;
  CudaBuffer<float> d_loss;
  CudaBuffer<float> d_grad_pixels;
  size_t num_pixels = 0;
};
