// NDC-space splats after projection and their gradients (src/types/splat2d.h:13-45).
#pragma once
#include "gpu_soa.h"

struct Splat2DParams : GpuSoA {
  CudaBuffer<float> pos_x, pos_y, pos_z;
  CudaBuffer<float> cov_xx, cov_xy, cov_yy;
  CudaBuffer<float> color_r, color_g, color_b;
  CudaBuffer<float> opacity;
  std::vector<CudaBuffer<float>*> fields() override {
    return {&pos_x, &pos_y, &pos_z, &cov_xx, &cov_xy, &cov_yy, &color_r, &color_g, &color_b,
            &opacity};
  }
};

struct Splat2DGrads : GpuSoA {
  CudaBuffer<float> grad_pos_x, grad_pos_y, grad_pos_z;
  CudaBuffer<float> grad_cov_xx, grad_cov_xy, grad_cov_yy;
  CudaBuffer<float> grad_color_r, grad_color_g, grad_color_b;
  CudaBuffer<float> grad_opacity;
  std::vector<CudaBuffer<float>*> fields() override {
    return {&grad_pos_x,   &grad_pos_y,   &grad_pos_z,   &grad_cov_xx, &grad_cov_xy,
            &grad_cov_yy,  &grad_color_r, &grad_color_g, &grad_color_b, &grad_opacity};
  }
};
