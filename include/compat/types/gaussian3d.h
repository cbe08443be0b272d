// Gaussian parameters on the host (AoS) and on the GPU (SoA), with the field
// order of src/types/gaussian3d.h:13-120.  sh_rest buffers are band-major:
// sh_rest_r[band * count + i]; the host struct stores them channel-first.
#pragma once
#include <vector>

#include "../cuda/cuda_buffer.h"
#include "../utils/sh_consts.h"
#include "gpu_soa.h"

struct Gaussian3D {
  float pos_x, pos_y, pos_z;
  float scale_x, scale_y, scale_z;       // log-scale
  float rot_w, rot_x, rot_y, rot_z;      // quaternion
  float sh_dc_r, sh_dc_g, sh_dc_b;
  float sh_rest[45] = {};                // R bands, then G, then B
  float logit_opacity;
};

struct Gaussian3DParams : GpuSoA {
  CudaBuffer<float> pos_x, pos_y, pos_z;
  CudaBuffer<float> scale_x, scale_y, scale_z;
  CudaBuffer<float> rot_w, rot_x, rot_y, rot_z;
  CudaBuffer<float> sh_dc_r, sh_dc_g, sh_dc_b;
  CudaBuffer<float> sh_rest_r, sh_rest_g, sh_rest_b;
  CudaBuffer<float> logit_opacity;
  int sh_num_bands = 0;

  std::vector<CudaBuffer<float>*> fields() override {
    return {&pos_x,   &pos_y,   &pos_z,   &scale_x,   &scale_y,   &scale_z,
            &rot_w,   &rot_x,   &rot_y,   &rot_z,     &sh_dc_r,   &sh_dc_g,
            &sh_dc_b, &sh_rest_r, &sh_rest_g, &sh_rest_b, &logit_opacity};
  }
  void allocate(int n) override { allocate(n, 0); }
  void allocate(int n, int sh_degree) {
    for (auto* f : {&pos_x, &pos_y, &pos_z, &scale_x, &scale_y, &scale_z, &rot_w, &rot_x, &rot_y,
                    &rot_z, &sh_dc_r, &sh_dc_g, &sh_dc_b, &logit_opacity})
      f->allocate(n);
    sh_num_bands = sh_degree_to_bands(sh_degree);
    if (sh_num_bands > 0)
      for (auto* f : {&sh_rest_r, &sh_rest_g, &sh_rest_b}) f->allocate((size_t)n * sh_num_bands);
    count = n;
  }
};

struct Gaussian3DGrads : GpuSoA {
  CudaBuffer<float> grad_pos_x, grad_pos_y, grad_pos_z;
  CudaBuffer<float> grad_scale_x, grad_scale_y, grad_scale_z;
  CudaBuffer<float> grad_rot_w, grad_rot_x, grad_rot_y, grad_rot_z;
  CudaBuffer<float> grad_sh_dc_r, grad_sh_dc_g, grad_sh_dc_b;
  CudaBuffer<float> grad_sh_rest_r, grad_sh_rest_g, grad_sh_rest_b;
  CudaBuffer<float> grad_logit_opacity;
  int sh_num_bands = 0;

  std::vector<CudaBuffer<float>*> fields() override {
    return {&grad_pos_x,     &grad_pos_y,     &grad_pos_z,     &grad_scale_x,  &grad_scale_y,
            &grad_scale_z,   &grad_rot_w,     &grad_rot_x,     &grad_rot_y,    &grad_rot_z,
            &grad_sh_dc_r,   &grad_sh_dc_g,   &grad_sh_dc_b,   &grad_sh_rest_r, &grad_sh_rest_g,
            &grad_sh_rest_b, &grad_logit_opacity};
  }
  void allocate(int n) override { allocate(n, 0); }
  void allocate(int n, int sh_degree) {
    for (auto* f : {&grad_pos_x, &grad_pos_y, &grad_pos_z, &grad_scale_x, &grad_scale_y,
                    &grad_scale_z, &grad_rot_w, &grad_rot_x, &grad_rot_y, &grad_rot_z,
                    &grad_sh_dc_r, &grad_sh_dc_g, &grad_sh_dc_b, &grad_logit_opacity})
      f->allocate(n);
    sh_num_bands = sh_degree_to_bands(sh_degree);
    if (sh_num_bands > 0)
      for (auto* f : {&grad_sh_rest_r, &grad_sh_rest_g, &grad_sh_rest_b})
        f->allocate((size_t)n * sh_num_bands);
    count = n;
  }
};
