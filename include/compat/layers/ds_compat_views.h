// Conversions from the drop-in SoA types to the C ABI structs of
// libdiffsplat_b200, and camera argument types that accept glm values (or any
// type with the same members) without depending on glm.
#pragma once
#include "../../diffsplat_b200.h"
#include "../types/gaussian3d.h"
#include "../types/splat2d.h"
#include "../types/splat3d.h"

namespace ds_compat {

inline float* P(const CudaBuffer<float>& b) { return b.ptr; }

inline ds_gaussian3d view(const Gaussian3DParams& p) {
  return {P(p.pos_x),   P(p.pos_y),   P(p.pos_z),   P(p.scale_x),   P(p.scale_y),
          P(p.scale_z), P(p.rot_w),   P(p.rot_x),   P(p.rot_y),     P(p.rot_z),
          P(p.sh_dc_r), P(p.sh_dc_g), P(p.sh_dc_b), P(p.sh_rest_r), P(p.sh_rest_g),
          P(p.sh_rest_b), P(p.logit_opacity), p.count, p.sh_num_bands};
}
inline ds_gaussian3d view(const Gaussian3DGrads& g) {
  return {P(g.grad_pos_x),   P(g.grad_pos_y),   P(g.grad_pos_z),     P(g.grad_scale_x),
          P(g.grad_scale_y), P(g.grad_scale_z), P(g.grad_rot_w),     P(g.grad_rot_x),
          P(g.grad_rot_y),   P(g.grad_rot_z),   P(g.grad_sh_dc_r),   P(g.grad_sh_dc_g),
          P(g.grad_sh_dc_b), P(g.grad_sh_rest_r), P(g.grad_sh_rest_g), P(g.grad_sh_rest_b),
          P(g.grad_logit_opacity), g.count, g.sh_num_bands};
}
inline ds_splat3d view(const Splat3DParams& s, int count) {
  return {P(s.pos_x),  P(s.pos_y),  P(s.pos_z),   P(s.cov_xx),  P(s.cov_xy),  P(s.cov_xz),
          P(s.cov_yy), P(s.cov_yz), P(s.cov_zz),  P(s.color_r), P(s.color_g), P(s.color_b),
          P(s.opacity), count};
}
inline ds_splat3d view(const Splat3DGrads& g, int count) {
  return {P(g.grad_pos_x),   P(g.grad_pos_y),   P(g.grad_pos_z),   P(g.grad_cov_xx),
          P(g.grad_cov_xy),  P(g.grad_cov_xz),  P(g.grad_cov_yy),  P(g.grad_cov_yz),
          P(g.grad_cov_zz),  P(g.grad_color_r), P(g.grad_color_g), P(g.grad_color_b),
          P(g.grad_opacity), count};
}
inline ds_splat2d view(const Splat2DParams& s, int count) {
  return {P(s.pos_x),   P(s.pos_y),   P(s.pos_z),   P(s.cov_xx),  P(s.cov_xy),
          P(s.cov_yy),  P(s.color_r), P(s.color_g), P(s.color_b), P(s.opacity), count};
}
inline ds_splat2d view(const Splat2DGrads& g, int count) {
  return {P(g.grad_pos_x),   P(g.grad_pos_y),   P(g.grad_pos_z),   P(g.grad_cov_xx),
          P(g.grad_cov_xy),  P(g.grad_cov_yy),  P(g.grad_color_r), P(g.grad_color_g),
          P(g.grad_color_b), P(g.grad_opacity), count};
}

// 3-vector argument: brace-initialisable, or converted from any type with
// x, y, z members (glm::vec3).
struct Vec3Arg {
  float x = 0.f, y = 0.f, z = 0.f;
  Vec3Arg() = default;
  Vec3Arg(float a, float b, float c) : x(a), y(b), z(c) {}
  template <class V>
  Vec3Arg(const V& v) : x(v.x), y(v.y), z(v.z) {}
};

// 4x4 matrix argument, column-major m[col * 4 + row], converted from any type
// indexed as M[col][row] (glm::mat4).
struct Mat4Arg {
  float m[16];
  template <class M>
  Mat4Arg(const M& mat) {
    for (int c = 0; c < 4; ++c)
      for (int r = 0; r < 4; ++r) m[c * 4 + r] = mat[c][r];
  }
};

// A * B of column-major matrices, summing k = 0..3 in order (the reference's
// glm product of proj * view).
inline void mat4_mul(const float* A, const float* B, float* out) {
  for (int c = 0; c < 4; ++c)
    for (int r = 0; r < 4; ++r)
      out[c * 4 + r] = A[0 * 4 + r] * B[c * 4 + 0] + A[1 * 4 + r] * B[c * 4 + 1] +
                       A[2 * 4 + r] * B[c * 4 + 2] + A[3 * 4 + r] * B[c * 4 + 3];
}

}  // namespace ds_compat
