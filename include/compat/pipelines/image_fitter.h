// ImageFitter (src/pipelines/image_fitter.h:23-66) on the fused,
// graph-captured step of libdiffsplat_b200 (ds_fitter_*).  The same sequence:
// init(w, h) sets the reference's orthographic camera in pixel units,
// randomInitGaussians(count, seed) its random init, initLayers() builds the
// step, step() runs zeroGrad + forward + backward + Adam.  The target comes
// from setTargetPixels (host RGB float [h*w*3] in [0, 1]).
#pragma once
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../diffsplat_b200.h"
#include "../cuda/cuda_check.h"
#include "../optimizers/gaussian3d_adam.h"
#include "../types/gaussian3d.h"

class ImageFitter {
 public:
  ~ImageFitter() {
    if (fitter) ds_fitter_destroy(fitter);
  }

  void init(int w, int h) {
    width = w;
    height = h;
    // glm::ortho(-w/2, w/2, -h/2, h/2, -z, z) with z = min(w, h)/8, identity view
    const float hw = width * 0.5f, hh = height * 0.5f;
    const float zr = std::min(hw, hh) * 0.25f;
    const float l = -hw, r = hw, b = -hh, t = hh, n = -zr, f = zr;
    std::fill(pv, pv + 16, 0.f);
    pv[0] = 2.f / (r - l);
    pv[5] = 2.f / (t - b);
    pv[10] = -2.f / (f - n);
    pv[12] = -(r + l) / (r - l);
    pv[13] = -(t + b) / (t - b);
    pv[14] = -(f + n) / (f - n);
    pv[15] = 1.f;
  }

  // Host target image, RGB float [h*w*3] in [0, 1], rows top to bottom.
  void setTargetPixels(const float* rgb) {
    target.assign(rgb, rgb + (size_t)width * height * 3);
  }

  // Random init in pixel-unit world space (src/utils/splat_utils.h:10-51):
  // position uniform in the image rectangle (depth +-min(w,h)/8), isotropic
  // log-scale ln 2 + U(-0.5, 0.5), identity rotation, random colour, opacity
  // U(0.6, 1.0).
  void randomInitGaussians(int count, int seed = -1) {
    if (seed < 0) seed = (int)std::chrono::system_clock::now().time_since_epoch().count();
    std::mt19937 rng(seed);
    std::uniform_real_distribution<float> sym(-1.f, 1.f), unit(0.f, 1.f);
    const float hw = width * 0.5f, hh = height * 0.5f, ls = logf(2.f);
    host.assign(count, Gaussian3D{});
    for (auto& g : host) {
      g.pos_x = sym(rng) * hw;
      g.pos_y = sym(rng) * hh;
      g.pos_z = sym(rng) * std::min(hw, hh) * 0.25f;
      const float s = sym(rng) * 0.5;
      g.scale_x = g.scale_y = g.scale_z = ls + s;
      g.rot_w = 1.f;
      g.rot_x = g.rot_y = g.rot_z = 0.f;
      g.sh_dc_r = (unit(rng) - 0.5f) / SH_C0;
      g.sh_dc_g = (unit(rng) - 0.5f) / SH_C0;
      g.sh_dc_b = (unit(rng) - 0.5f) / SH_C0;
      const float o = 0.6f + 0.4f * unit(rng);
      g.logit_opacity = logf(o / (1.f - o));
    }
  }

  void initLayers(const Gaussian3DAdamConfig& adam = {}) {
    if (host.empty()) throw std::runtime_error("[ImageFitter] no Gaussians");
    if (target.empty()) throw std::runtime_error("[ImageFitter] no target image");
    ds_fitter_config cfg;
    ds_fitter_default_config(&cfg);
    cfg.width = width;
    cfg.height = height;
    cfg.count = (int)host.size();
    cfg.lr_pos = adam.lr_pos;
    cfg.lr_scale = adam.lr_scale;
    cfg.lr_rot = adam.lr_rot;
    cfg.lr_sh_dc = adam.lr_sh_dc;
    cfg.lr_sh_rest = adam.lr_sh_rest;
    cfg.lr_opacity = adam.lr_opacity;
    cfg.beta1 = adam.adam.beta1;
    cfg.beta2 = adam.adam.beta2;
    cfg.epsilon = adam.adam.epsilon;
    int st = ds_fitter_create(&cfg, &fitter);
    if (st != DS_OK) throw std::runtime_error(std::string("[ImageFitter] ") + ds_status_string(st));
    ds_gaussian3d p;
    ds_fitter_params(fitter, &p);
    const int n = cfg.count;
    std::vector<float> col(n);
    auto put = [&](float* dst, float Gaussian3D::*field) {
      for (int i = 0; i < n; ++i) col[i] = host[i].*field;
      CUDA_CHECK(cudaMemcpy(dst, col.data(), n * sizeof(float), cudaMemcpyHostToDevice));
    };
    put(p.pos_x, &Gaussian3D::pos_x);
    put(p.pos_y, &Gaussian3D::pos_y);
    put(p.pos_z, &Gaussian3D::pos_z);
    put(p.scale_x, &Gaussian3D::scale_x);
    put(p.scale_y, &Gaussian3D::scale_y);
    put(p.scale_z, &Gaussian3D::scale_z);
    put(p.rot_w, &Gaussian3D::rot_w);
    put(p.rot_x, &Gaussian3D::rot_x);
    put(p.rot_y, &Gaussian3D::rot_y);
    put(p.rot_z, &Gaussian3D::rot_z);
    put(p.sh_dc_r, &Gaussian3D::sh_dc_r);
    put(p.sh_dc_g, &Gaussian3D::sh_dc_g);
    put(p.sh_dc_b, &Gaussian3D::sh_dc_b);
    put(p.logit_opacity, &Gaussian3D::logit_opacity);
    float* d_target = nullptr;
    CUDA_CHECK(cudaMalloc(&d_target, target.size() * sizeof(float)));
    CUDA_CHECK(cudaMemcpy(d_target, target.data(), target.size() * sizeof(float),
                          cudaMemcpyHostToDevice));
    DS_COMPAT_CHECK(ds_fitter_set_target(fitter, d_target, nullptr));
    CUDA_CHECK(cudaDeviceSynchronize());
    CUDA_CHECK(cudaFree(d_target));
    const float cam[3] = {0.f, 0.f, 0.f};
    DS_COMPAT_CHECK(ds_fitter_set_camera(fitter, pv, cam, nullptr));
  }

  void step() {
    if (!is_running) return;
    DS_COMPAT_CHECK(ds_fitter_step(fitter, 1, nullptr));
  }

  float* getOutput() {
    float* img = nullptr;
    ds_fitter_output(fitter, &img);
    return img;
  }
  int getIterCount() const {
    int c = 0;
    if (fitter) ds_fitter_step_count(fitter, &c);
    return c;
  }
  float getLoss() const {
    float l = 0.f;
    if (fitter) DS_COMPAT_CHECK(ds_fitter_loss(fitter, &l, nullptr));
    return l;
  }
  bool isRunning() const { return is_running; }
  void setRunning(bool v) { is_running = v; }

 private:
  int width = 0, height = 0;
  bool is_running = true;
  float pv[16] = {};
  std::vector<Gaussian3D> host;
  std::vector<float> target;
  ds_fitter* fitter = nullptr;
};
