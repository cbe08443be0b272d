// Adam over parameter groups (src/optimizers/adam.h:5-70) on libdiffsplat_b200:
// step() updates every group with one kernel launch (ds_adam_step); bias
// corrections 1 / (1 - powf(beta, t)) are computed on the host as the reference does.
#pragma once
#include <vector>

#include "../../diffsplat_b200.h"
#include "../cuda/cuda_buffer.h"

struct AdamParams {
  float beta1 = 0.9f;
  float beta2 = 0.999f;
  float epsilon = 1e-8f;
};

struct AdamGroup {
  float* param;
  const float* grad;
  int n;
  float lr;
  CudaBuffer<float> m, v;
  AdamGroup(float* p, const float* g, int n_, float lr_) : param(p), grad(g), n(n_), lr(lr_) {
    m.allocate(n_);
    m.zero();
    v.allocate(n_);
    v.zero();
  }
  AdamGroup(AdamGroup&&) = default;
  AdamGroup& operator=(AdamGroup&&) = default;
  AdamGroup(const AdamGroup&) = delete;
  AdamGroup& operator=(const AdamGroup&) = delete;
};

class Adam {
 public:
  void init(const AdamParams& p = {}) { hp = p; }
  void addGroup(CudaBuffer<float>& param, const CudaBuffer<float>& grad, int n, float lr) {
    groups.emplace_back(param.ptr, grad.ptr, n, lr);
  }
  void setLr(int idx, float lr) { groups[idx].lr = lr; }
  void step() {
    ++step_count;
    std::vector<ds_adam_group> g;
    g.reserve(groups.size());
    for (auto& x : groups) g.push_back({x.param, x.grad, x.m.ptr, x.v.ptr, x.n, x.lr});
    DS_COMPAT_CHECK(ds_adam_step(g.data(), (int)g.size(), hp.beta1, hp.beta2, hp.epsilon,
                                 step_count, nullptr));
  }
  int getStepCount() const { return step_count; }
  const AdamParams& getParams() const { return hp; }

 private:
  AdamParams hp;
  std::vector<AdamGroup> groups;
  int step_count = 0;
};
