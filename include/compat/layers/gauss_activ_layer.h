// GaussActivLayer (src/layers/gauss_activ_layer.h:26-47) on libdiffsplat_b200:
// Cov3D from log-scale + quaternion, SH colour (degree 0-3) + 0.5 clamped to
// [0, 1], sigmoid opacity; backward writes grad_input.
#pragma once
#include "ds_compat_views.h"
#include "layer.h"

class GaussActivLayer
    : public TypedLayer<Gaussian3DParams, Splat3DParams, Gaussian3DGrads, Splat3DGrads> {
 public:
  void forward() override {
    output.count = input->count;
    ds_gaussian3d in = ds_compat::view(*input);
    ds_splat3d out = ds_compat::view(output, input->count);
    float cam[3] = {cam_pos.x, cam_pos.y, cam_pos.z};
    DS_COMPAT_CHECK(ds_activ_forward(&in, sh_degree, cam, &out, nullptr));
  }
  void backward() override {
    ds_gaussian3d in = ds_compat::view(*input);
    ds_splat3d out = ds_compat::view(output, input->count);
    ds_splat3d gout = ds_compat::view(*grad_output, input->count);
    ds_gaussian3d gin = ds_compat::view(grad_input);
    float cam[3] = {cam_pos.x, cam_pos.y, cam_pos.z};
    DS_COMPAT_CHECK(ds_activ_backward(&in, &out, &gout, sh_degree, cam, &gin, nullptr));
  }
  void setSHDegree(int degree) { sh_degree = degree; }
  void setCameraPosition(const ds_compat::Vec3Arg& pos) { cam_pos = pos; }
  void allocateGrad(int n) override { grad_input.allocate(n, sh_degree); }

 private:
  int sh_degree = 0;
  ds_compat::Vec3Arg cam_pos;
};
