// PerspProjectLayer (src/layers/persp_project_layer.h:24-38) on
// libdiffsplat_b200.  The PV matrix is kept per layer and passed with each
// call (the reference keeps one process-wide __constant__ copy).
#pragma once
#include "ds_compat_views.h"
#include "layer.h"

class PerspProjectLayer
    : public TypedLayer<Splat3DParams, Splat2DParams, Splat3DGrads, Splat2DGrads> {
 public:
  void forward() override {
    output.count = input->count;
    ds_splat3d in = ds_compat::view(*input, input->count);
    ds_splat2d out = ds_compat::view(output, input->count);
    DS_COMPAT_CHECK(ds_project_forward(&in, h_pv, &out, nullptr));
  }
  void backward() override {
    ds_splat3d in = ds_compat::view(*input, input->count);
    ds_splat2d gout = ds_compat::view(*grad_output, input->count);
    ds_splat3d gin = ds_compat::view(grad_input, input->count);
    DS_COMPAT_CHECK(ds_project_backward_ex(&in, h_pv, &gout, &gin, grad_mode, nullptr));
  }
  // PV = proj * view, column-major.
  void setCamera(const ds_compat::Mat4Arg& view, const ds_compat::Mat4Arg& proj) {
    ds_compat::mat4_mul(proj.m, view.m, h_pv);
  }
  // DS_GRAD_REFERENCE or DS_GRAD_EXACT (default: ds_default_grad_mode()).
  void setGradMode(int mode) { grad_mode = mode; }

 private:
  float h_pv[16] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1};
  int grad_mode = ds_default_grad_mode();
};
