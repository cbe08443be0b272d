// Per-field learning rates and registration of every Gaussian3D buffer with
// Adam (src/optimizers/gaussian3d_adam.h:11-55).
#pragma once
#include "../types/gaussian3d.h"
#include "adam.h"

struct Gaussian3DAdamConfig {
  float lr_pos = 1.6e-2f;
  float lr_scale = 1.0e-3f;
  float lr_rot = 6.0e-4f;
  float lr_sh_dc = 6.0e-3f;
  float lr_sh_rest = 6.0e-3f;
  float lr_opacity = 6.0e-3f;
  AdamParams adam = {};
};

inline void registerGaussian3DGroups(Adam& adam, Gaussian3DParams& p, Gaussian3DGrads& g,
                                     const Gaussian3DAdamConfig& cfg = {}) {
  const int n = p.count;
  adam.addGroup(p.pos_x, g.grad_pos_x, n, cfg.lr_pos);
  adam.addGroup(p.pos_y, g.grad_pos_y, n, cfg.lr_pos);
  adam.addGroup(p.pos_z, g.grad_pos_z, n, cfg.lr_pos);
  adam.addGroup(p.scale_x, g.grad_scale_x, n, cfg.lr_scale);
  adam.addGroup(p.scale_y, g.grad_scale_y, n, cfg.lr_scale);
  adam.addGroup(p.scale_z, g.grad_scale_z, n, cfg.lr_scale);
  adam.addGroup(p.rot_w, g.grad_rot_w, n, cfg.lr_rot);
  adam.addGroup(p.rot_x, g.grad_rot_x, n, cfg.lr_rot);
  adam.addGroup(p.rot_y, g.grad_rot_y, n, cfg.lr_rot);
  adam.addGroup(p.rot_z, g.grad_rot_z, n, cfg.lr_rot);
  adam.addGroup(p.sh_dc_r, g.grad_sh_dc_r, n, cfg.lr_sh_dc);
  adam.addGroup(p.sh_dc_g, g.grad_sh_dc_g, n, cfg.lr_sh_dc);
  adam.addGroup(p.sh_dc_b, g.grad_sh_dc_b, n, cfg.lr_sh_dc);
  adam.addGroup(p.logit_opacity, g.grad_logit_opacity, n, cfg.lr_opacity);
  if (p.sh_num_bands > 0) {
    const int m = n * p.sh_num_bands;
    adam.addGroup(p.sh_rest_r, g.grad_sh_rest_r, m, cfg.lr_sh_rest);
    adam.addGroup(p.sh_rest_g, g.grad_sh_rest_g, m, cfg.lr_sh_rest);
    adam.addGroup(p.sh_rest_b, g.grad_sh_rest_b, m, cfg.lr_sh_rest);
  }
}
