// Host <-> device transfer of Gaussians (src/utils/gaussian3d_io.h): the host
// struct stores SH rest channel-first, the device buffers band-major.
#pragma once
#include <vector>

#include "../cuda/cuda_check.h"
#include "../types/gaussian3d.h"

inline void uploadGaussians(Gaussian3DParams& params, const std::vector<Gaussian3D>& host,
                            int sh_degree = 0) {
  const int n = (int)host.size();
  params.allocate(n, sh_degree);
  const int K = params.sh_num_bands;
  std::vector<float> tmp((size_t)n * (K > 0 ? K : 1));
  auto put = [&](CudaBuffer<float>& dst, float Gaussian3D::*field) {
    for (int i = 0; i < n; ++i) tmp[i] = host[i].*field;
    CUDA_CHECK(cudaMemcpy(dst.ptr, tmp.data(), n * sizeof(float), cudaMemcpyHostToDevice));
  };
  put(params.pos_x, &Gaussian3D::pos_x);
  put(params.pos_y, &Gaussian3D::pos_y);
  put(params.pos_z, &Gaussian3D::pos_z);
  put(params.scale_x, &Gaussian3D::scale_x);
  put(params.scale_y, &Gaussian3D::scale_y);
  put(params.scale_z, &Gaussian3D::scale_z);
  put(params.rot_w, &Gaussian3D::rot_w);
  put(params.rot_x, &Gaussian3D::rot_x);
  put(params.rot_y, &Gaussian3D::rot_y);
  put(params.rot_z, &Gaussian3D::rot_z);
  put(params.sh_dc_r, &Gaussian3D::sh_dc_r);
  put(params.sh_dc_g, &Gaussian3D::sh_dc_g);
  put(params.sh_dc_b, &Gaussian3D::sh_dc_b);
  put(params.logit_opacity, &Gaussian3D::logit_opacity);
  CudaBuffer<float>* rest[3] = {&params.sh_rest_r, &params.sh_rest_g, &params.sh_rest_b};
  for (int c = 0; c < 3 && K > 0; ++c) {
    for (int b = 0; b < K; ++b)
      for (int i = 0; i < n; ++i) tmp[(size_t)b * n + i] = host[i].sh_rest[c * K + b];
    CUDA_CHECK(cudaMemcpy(rest[c]->ptr, tmp.data(), (size_t)K * n * sizeof(float),
                          cudaMemcpyHostToDevice));
  }
}

inline std::vector<Gaussian3D> downloadGaussians(const Gaussian3DParams& params) {
  const int n = params.count, K = params.sh_num_bands;
  std::vector<Gaussian3D> host(n);
  std::vector<float> tmp((size_t)n * (K > 0 ? K : 1));
  auto get = [&](const CudaBuffer<float>& src, float Gaussian3D::*field) {
    CUDA_CHECK(cudaMemcpy(tmp.data(), src.ptr, n * sizeof(float), cudaMemcpyDeviceToHost));
    for (int i = 0; i < n; ++i) host[i].*field = tmp[i];
  };
  get(params.pos_x, &Gaussian3D::pos_x);
  get(params.pos_y, &Gaussian3D::pos_y);
  get(params.pos_z, &Gaussian3D::pos_z);
  get(params.scale_x, &Gaussian3D::scale_x);
  get(params.scale_y, &Gaussian3D::scale_y);
  get(params.scale_z, &Gaussian3D::scale_z);
  get(params.rot_w, &Gaussian3D::rot_w);
  get(params.rot_x, &Gaussian3D::rot_x);
  get(params.rot_y, &Gaussian3D::rot_y);
  get(params.rot_z, &Gaussian3D::rot_z);
  get(params.sh_dc_r, &Gaussian3D::sh_dc_r);
  get(params.sh_dc_g, &Gaussian3D::sh_dc_g);
  get(params.sh_dc_b, &Gaussian3D::sh_dc_b);
  get(params.logit_opacity, &Gaussian3D::logit_opacity);
  const CudaBuffer<float>* rest[3] = {&params.sh_rest_r, &params.sh_rest_g, &params.sh_rest_b};
  for (int c = 0; c < 3 && K > 0; ++c) {
    CUDA_CHECK(cudaMemcpy(tmp.data(), rest[c]->ptr, (size_t)K * n * sizeof(float),
                          cudaMemcpyDeviceToHost));
    for (int b = 0; b < K; ++b)
      for (int i = 0; i < n; ++i) host[i].sh_rest[c * K + b] = tmp[(size_t)b * n + i];
  }
  return host;
}
