// SplatUtils (src/utils/splat_utils.h): randomInit draws, per splat and in
// this order, x, y, z ~ U(-1, 1) scaled to the image rectangle (depth to
// min(w, h) / 8), one U(-1, 1) log-scale offset around ln 2 shared by the three
// axes (times 0.5), three U(0, 1) colours mapped to SH DC, and an opacity
// U(0.6, 1.0) stored as a logit, from std::mt19937(seed); normalizeScene calls
// ds_normalize_scene.
#pragma once
#include <algorithm>
#include <cmath>
#include <random>
#include <vector>

#include "../../diffsplat_b200.h"
#include "../types/gaussian3d.h"
#include "sh_consts.h"

namespace SplatUtils {

inline std::vector<Gaussian3D> randomInit(int count, int width, int height, int seed) {
  std::mt19937 rng(seed);
  std::uniform_real_distribution<float> sym(-1.f, 1.f), unit(0.f, 1.f);
  const float hw = width * 0.5f, hh = height * 0.5f, ls = logf(2.f);
  const float depth = std::min(hw, hh) * 0.25f;
  std::vector<Gaussian3D> out((size_t)count);
  for (auto& g : out) {
    g.pos_x = sym(rng) * hw;
    g.pos_y = sym(rng) * hh;
    g.pos_z = sym(rng) * depth;
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
  return out;
}

inline void normalizeScene(std::vector<Gaussian3D>& splats, float scene_scale = 1.f) {
  ds_normalize_scene(reinterpret_cast<float*>(splats.data()), (int64_t)splats.size(),
                     scene_scale);
}

}  // namespace SplatUtils
