// Real spherical-harmonic constants, 3DGS band ordering (src/utils/sh_consts.h).
#pragma once

static constexpr float SH_C0 = 0.28209479177387814f;
static constexpr float SH_C1 = 0.4886025119029199f;
static constexpr float SH_C2_0 = 1.0925484305920792f;
static constexpr float SH_C2_1 = -1.0925484305920792f;
static constexpr float SH_C2_2 = 0.3153915652525200f;
static constexpr float SH_C2_3 = -1.0925484305920792f;
static constexpr float SH_C2_4 = 0.5462742152960396f;
static constexpr float SH_C3_0 = -0.5900435899266435f;
static constexpr float SH_C3_1 = 2.8906114426405540f;
static constexpr float SH_C3_2 = -0.4570457994644658f;
static constexpr float SH_C3_3 = 0.3731763325901154f;
static constexpr float SH_C3_4 = -0.4570457994644658f;
static constexpr float SH_C3_5 = 1.4453057213202770f;
static constexpr float SH_C3_6 = -0.5900435899266435f;

// Higher-order bands (excluding DC) of an SH degree: 0, 3, 8, 15.
inline int sh_degree_to_bands(int degree) {
  int n = 0;
  for (int l = 1; l <= degree; ++l) n += 2 * l + 1;
  return n;
}
