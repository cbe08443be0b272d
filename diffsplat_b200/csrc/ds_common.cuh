// Device-side helpers shared by every diffsplat_b200 kernel.
//
// The arithmetic in the helpers marked "parity" follows the reference's own
// expression trees term for term (src/cuda/math_ops.cuh:34-37, :72-79, :94-101)
// because the tile keys and tile counts downstream of them must be bit-identical
// to the reference CUDA build, and this file is compiled with the same
// --use_fast_math flag the reference uses (CMakeLists.txt:121-127).
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace ds {

// ---------------------------------------------------------------------------
// Constants of the compositing model (src/layers/tile_rasterize_layer.cu:18-26)
// ---------------------------------------------------------------------------
constexpr int   kTile       = 16;            // pixels per tile edge
constexpr int   kTilePixels = kTile * kTile; // 256 threads per tile CTA
constexpr float kMaxAlpha   = 0.99f;
constexpr float kAlphaThres = 1.0f / 255.0f;
constexpr float kTThres     = 0.0001f;

// Real spherical-harmonic basis constants, 3DGS band ordering (src/utils/sh_consts.h:7-27).
constexpr float kC0   = 0.28209479177387814f;
constexpr float kC1   = 0.4886025119029199f;
constexpr float kC2_0 = 1.0925484305920792f;
constexpr float kC2_1 = -1.0925484305920792f;
constexpr float kC2_2 = 0.3153915652525200f;
constexpr float kC2_3 = -1.0925484305920792f;
constexpr float kC2_4 = 0.5462742152960396f;
constexpr float kC3_0 = -0.5900435899266435f;
constexpr float kC3_1 = 2.8906114426405540f;
constexpr float kC3_2 = -0.4570457994644658f;
constexpr float kC3_3 = 0.3731763325901154f;
constexpr float kC3_4 = -0.4570457994644658f;
constexpr float kC3_5 = 1.4453057213202770f;
constexpr float kC3_6 = -0.5900435899266435f;

__host__ __device__ inline int sh_bands(int degree) {
  int n = 0;
  for (int l = 1; l <= degree; ++l) n += 2 * l + 1;
  return n;
}

// Waits until the kernel this one was launched after with programmatic
// dependent launch (launch_pdl) has completed and its writes are visible; a
// no-op for an ordinary launch.  Kernels of the step chain call it first.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// ---------------------------------------------------------------------------
// Quaternion / rotation (parity)
// ---------------------------------------------------------------------------
struct UnitQuat {
  float w, x, y, z;
  float inv_norm;
};

// Rounding of the sums on the tile-key path is pinned with explicit
// fma/mul/add intrinsics: nvcc's choice of which product to fuse depends on the
// surrounding code, and the forms below are the ones that reproduce the
// reference build's FP32 results bit for bit (measured against it on the GPU
// over 10^5 random splats with a general camera).
__device__ __forceinline__ UnitQuat unit_quat(float w, float x, float y, float z) {
  float n2 = __fmaf_rn(z, z, __fmaf_rn(y, y, __fmaf_rn(w, w, __fmul_rn(x, x))));
  float inv = rsqrtf(fmaxf(n2, 1e-12f));
  return {w * inv, x * inv, y * inv, z * inv, inv};
}

struct Rot3 {
  float r00, r01, r02, r10, r11, r12, r20, r21, r22;
};

// R = I + 2 [ -(y^2+z^2)  xy-wz  xz+wy ; xy+wz  -(x^2+z^2)  yz-wx ; xz-wy  yz+wx  -(x^2+y^2) ]
__device__ __forceinline__ Rot3 rot_from_quat(float qw, float qx, float qy, float qz) {
  Rot3 R;
  R.r00 = 1.f - 2.f * __fadd_rn(__fmul_rn(qy, qy), __fmul_rn(qz, qz));
  R.r01 = 2.f * __fmaf_rn(qx, qy, -__fmul_rn(qw, qz));
  R.r02 = 2.f * __fmaf_rn(qx, qz, __fmul_rn(qw, qy));
  R.r10 = 2.f * __fmaf_rn(qx, qy, __fmul_rn(qw, qz));
  R.r11 = 1.f - 2.f * __fmaf_rn(qx, qx, __fmul_rn(qz, qz));
  R.r12 = 2.f * __fmaf_rn(qy, qz, -__fmul_rn(qw, qx));
  R.r20 = 2.f * __fmaf_rn(qx, qz, -__fmul_rn(qw, qy));
  R.r21 = 2.f * __fmaf_rn(qy, qz, __fmul_rn(qw, qx));
  R.r22 = 1.f - 2.f * __fmaf_rn(qx, qx, __fmul_rn(qy, qy));
  return R;
}

// a0 b0 + a1 b1 + a2 b2 with the first product fused (A) or the second (B).
__device__ __forceinline__ float dot3_a(float a0, float b0, float a1, float b1, float a2,
                                        float b2) {
  return __fmaf_rn(a2, b2, __fmaf_rn(a1, b1, __fmul_rn(a0, b0)));
}
__device__ __forceinline__ float dot3_b(float a0, float b0, float a1, float b1, float a2,
                                        float b2) {
  return __fmaf_rn(a2, b2, __fmaf_rn(a0, b0, __fmul_rn(a1, b1)));
}

__device__ __forceinline__ float3 dir_to_camera(float cx, float cy, float cz, float px, float py,
                                                float pz) {
  float dx = cx - px, dy = cy - py, dz = cz - pz;
  float inv = rsqrtf(fmaxf(dx * dx + dy * dy + dz * dz, 1e-12f));
  return make_float3(dx * inv, dy * inv, dz * inv);
}

// Upper-triangle covariance (R S)(R S)^T from a raw quaternion and log-scales (parity).
struct Cov3 {
  float xx, xy, xz, yy, yz, zz;
};

__device__ __forceinline__ Cov3 cov3_from(const Rot3& R, float sx, float sy, float sz) {
  float m00 = R.r00 * sx, m01 = R.r01 * sy, m02 = R.r02 * sz;
  float m10 = R.r10 * sx, m11 = R.r11 * sy, m12 = R.r12 * sz;
  float m20 = R.r20 * sx, m21 = R.r21 * sy, m22 = R.r22 * sz;
  Cov3 c;
  c.xx = dot3_a(m00, m00, m01, m01, m02, m02);
  c.xy = dot3_b(m00, m10, m01, m11, m02, m12);
  c.xz = dot3_a(m00, m20, m01, m21, m02, m22);
  c.yy = dot3_b(m10, m10, m11, m11, m12, m12);
  c.yz = dot3_b(m10, m20, m11, m21, m12, m22);
  c.zz = dot3_b(m20, m20, m21, m21, m22, m22);
  return c;
}

// ---------------------------------------------------------------------------
// Spherical harmonics: colour = sum_lm c_lm Y_lm(dir) + 0.5.  The expression
// order follows src/layers/gauss_activ_layer.cu:106-162 so FP32 results agree
// with the reference to the last bit.  `rest` points at band 0 of one channel,
// `stride` is the splat count (band-major layout [band * count + i]).
// ---------------------------------------------------------------------------
struct ShBasis {
  float y[15];
};

// Loads of a stored attribute as FP32 (FP32 or BF16 storage).
__device__ __forceinline__ float ldv(float x) { return x; }
__device__ __forceinline__ float ldv(__nv_bfloat16 x) { return __bfloat162float(x); }

template <typename T>
__device__ __forceinline__ float sh_channel(float dc, const T* __restrict__ rest, int stride,
                                            int degree, float3 v) {
  float c = dc * kC0;
  if (degree >= 1) {
    c += kC1 * (-v.y * ldv(rest[0 * stride]) + v.z * ldv(rest[1 * stride]) -
                v.x * ldv(rest[2 * stride]));
  }
  if (degree >= 2) {
    float xx = v.x * v.x, yy = v.y * v.y, zz = v.z * v.z;
    float xy = v.x * v.y, yz = v.y * v.z, xz = v.x * v.z;
    c += kC2_0 * xy * ldv(rest[3 * stride]) + kC2_1 * yz * ldv(rest[4 * stride]) +
         kC2_2 * (2 * zz - xx - yy) * ldv(rest[5 * stride]) + kC2_3 * xz * ldv(rest[6 * stride]) +
         kC2_4 * (xx - yy) * ldv(rest[7 * stride]);
  }
  if (degree >= 3) {
    float xx = v.x * v.x, yy = v.y * v.y, zz = v.z * v.z;
    float xy = v.x * v.y;
    c += kC3_0 * v.y * (3 * xx - yy) * ldv(rest[8 * stride]) +
         kC3_1 * xy * v.z * ldv(rest[9 * stride]) +
         kC3_2 * v.y * (4 * zz - xx - yy) * ldv(rest[10 * stride]) +
         kC3_3 * v.z * (2 * zz - 3 * xx - 3 * yy) * ldv(rest[11 * stride]) +
         kC3_4 * v.x * (4 * zz - xx - yy) * ldv(rest[12 * stride]) +
         kC3_5 * v.z * (xx - yy) * ldv(rest[13 * stride]) +
         kC3_6 * v.x * (xx - 3 * yy) * ldv(rest[14 * stride]);
  }
  return c;
}

// Basis values Y_lm(dir) for the SH backward (gauss_activ_layer.cu:342-401).
__device__ __forceinline__ void sh_basis(int degree, float3 v, float* y) {
  if (degree >= 1) {
    y[0] = kC1 * (-v.y);
    y[1] = kC1 * (v.z);
    y[2] = kC1 * (-v.x);
  }
  if (degree >= 2) {
    float xx = v.x * v.x, yy = v.y * v.y, zz = v.z * v.z;
    float xy = v.x * v.y, yz = v.y * v.z, xz = v.x * v.z;
    y[3] = kC2_0 * xy;
    y[4] = kC2_1 * yz;
    y[5] = kC2_2 * (2 * zz - xx - yy);
    y[6] = kC2_3 * xz;
    y[7] = kC2_4 * (xx - yy);
    if (degree >= 3) {
      y[8] = kC3_0 * v.y * (3 * xx - yy);
      y[9] = kC3_1 * xy * v.z;
      y[10] = kC3_2 * v.y * (4 * zz - xx - yy);
      y[11] = kC3_3 * v.z * (2 * zz - 3 * xx - 3 * yy);
      y[12] = kC3_4 * v.x * (4 * zz - xx - yy);
      y[13] = kC3_5 * v.z * (xx - yy);
      y[14] = kC3_6 * v.x * (xx - 3 * yy);
    }
  }
}

__device__ __forceinline__ float clamp01(float c) { return fminf(fmaxf(c, 0.f), 1.f); }

// ---------------------------------------------------------------------------
// Perspective projection (parity): pv is column-major, pv[col*4 + row].
// ---------------------------------------------------------------------------
struct Mat4 {
  float m[16];
};

struct Proj2 {
  float ndc_x, ndc_y, ndc_z;
  float cxx, cxy, cyy;
  float j00, j01, j02, j10, j11, j12;
  bool culled;
};

__device__ __forceinline__ void project_jacobian(const Mat4& P, float x, float y, float z,
                                                 float& clip_x, float& clip_y, float& clip_z,
                                                 float& clip_w) {
  clip_x = __fadd_rn(dot3_a(P.m[4], y, P.m[0], x, P.m[8], z), P.m[12]);
  clip_y = __fadd_rn(dot3_a(P.m[5], y, P.m[1], x, P.m[9], z), P.m[13]);
  clip_z = __fadd_rn(dot3_a(P.m[6], y, P.m[2], x, P.m[10], z), P.m[14]);
  clip_w = __fadd_rn(dot3_a(P.m[7], y, P.m[3], x, P.m[11], z), P.m[15]);
}

struct Jac2 {
  float j00, j01, j02, j10, j11, j12;
};

__device__ __forceinline__ Jac2 jacobian(const Mat4& P, float clip_x, float clip_y, float clip_w,
                                         float inv_w2) {
  Jac2 J;
  J.j00 = __fmaf_rn(P.m[0], clip_w, -__fmul_rn(clip_x, P.m[3])) * inv_w2;
  J.j01 = __fmaf_rn(P.m[4], clip_w, -__fmul_rn(clip_x, P.m[7])) * inv_w2;
  J.j02 = __fmaf_rn(P.m[8], clip_w, -__fmul_rn(clip_x, P.m[11])) * inv_w2;
  J.j10 = __fmaf_rn(P.m[1], clip_w, -__fmul_rn(clip_y, P.m[3])) * inv_w2;
  J.j11 = __fmaf_rn(P.m[5], clip_w, -__fmul_rn(clip_y, P.m[7])) * inv_w2;
  J.j12 = __fmaf_rn(P.m[9], clip_w, -__fmul_rn(clip_y, P.m[11])) * inv_w2;
  return J;
}

struct Cov2 {
  float xx, xy, yy;
};

// Cov2D = J Cov3D J^T, upper triangle (persp_project_layer.cu:131-142).
__device__ __forceinline__ Cov2 cov2_from(const Jac2& J, float cxx, float cxy, float cxz, float cyy,
                                          float cyz, float czz) {
  float js00 = dot3_b(J.j00, cxx, J.j01, cxy, J.j02, cxz);
  float js01 = dot3_b(J.j00, cxy, J.j01, cyy, J.j02, cyz);
  float js02 = dot3_b(J.j00, cxz, J.j01, cyz, J.j02, czz);
  float js10 = dot3_b(J.j10, cxx, J.j11, cxy, J.j12, cxz);
  float js11 = dot3_b(J.j10, cxy, J.j11, cyy, J.j12, cyz);
  float js12 = dot3_b(J.j10, cxz, J.j11, cyz, J.j12, czz);
  Cov2 c;
  c.xx = dot3_b(J.j00, js00, J.j01, js01, J.j02, js02);
  c.xy = dot3_b(J.j00, js10, J.j01, js11, J.j02, js12);
  c.yy = dot3_b(J.j10, js10, J.j11, js11, J.j12, js12);
  return c;
}

// ---------------------------------------------------------------------------
// Tile rectangle of the 3-sigma AABB (parity; tile_rasterize_layer.cu:84-118).
// Returns false when the splat is culled.
// ---------------------------------------------------------------------------
struct TileRect {
  int x0, x1, y0, y1;
};

// det of Cov2D and the conic's quadratic form dx^2 a + 2 dx dy b + dy^2 c, in
// the reference's rounding (tile_rasterize_layer.cu:150, :321, :341).
__device__ __forceinline__ float conic_det(float cxx, float cxy, float cyy) {
  return __fmaf_rn(cxx, cyy, -__fmul_rn(cxy, cxy));
}
__device__ __forceinline__ float conic_dist2(float dx, float dy, float a, float b, float c) {
  const float t2 = __fmul_rn(__fmul_rn(2.f, dx), dy);
  return __fmaf_rn(__fmul_rn(dy, dy), c, __fmaf_rn(__fmul_rn(dx, dx), a, __fmul_rn(t2, b)));
}

template <int TS = kTile>
__device__ __forceinline__ bool tile_rect(float x, float y, float z, float cxx, float cxy, float cyy,
                                          int width, int height, int ntx, int nty, TileRect& r) {
  if (!(fabsf(x) <= 1.0f && fabsf(y) <= 1.0f && fabsf(z) <= 1.0f)) return false;
  float det = conic_det(cxx, cxy, cyy);
  if (!(det > 0.f)) return false;
  float extent_x = 3.f * sqrtf(cxx);
  float extent_y = 3.f * sqrtf(cyy);
  float pixel_ndc = fmaxf(2.f / width, 2.f / height);
  if (!(fmaxf(extent_x, extent_y) * 2.f >= pixel_ndc)) return false;
  float min_x = x - extent_x, max_x = x + extent_x;
  float min_y = y - extent_y, max_y = y + extent_y;
  const float fx = (float)width / TS;
  const float fy = (float)height / TS;
  r.x0 = max((int)floorf((min_x + 1.f) * 0.5f * fx), 0);
  r.x1 = min((int)floorf((max_x + 1.f) * 0.5f * fx), ntx - 1);
  r.y0 = max((int)floorf((1.f - max_y) * 0.5f * fy), 0);
  r.y1 = min((int)floorf((1.f - min_y) * 0.5f * fy), nty - 1);
  return r.x0 <= r.x1 && r.y0 <= r.y1;
}

// Order-preserving map of an IEEE float to uint32 (tile_rasterize_layer.cu:30-38).
__device__ __forceinline__ uint32_t depth_bits(float depth) {
  uint32_t u = __float_as_uint(depth);
  return (u >> 31) ? ~u : (u ^ 0x80000000u);
}

// ---------------------------------------------------------------------------
// Per-splat compositing record.  Three float4 per splat, written once by the
// preprocess and gathered per (tile, splat) pair by the composite kernels:
//   A = {ndc x, ndc y, cull half-width x, cull half-width y}
//   B = {conic xx, conic xy, conic yy, opacity}
//   C = {r, g, b, sigma cut}
// plus idet (1/det of Cov2D) used only by the backward.
// The conic is computed with the reference's formula (tile_rasterize_layer.cu:
// 260-272) so the per-pixel Gaussian value is bit-identical.  The culling box
// and sigma cut are conservative bounds of the region where the reference's
// own tests (sigma >= 0, alpha >= 1/255) can accept the splat, so skipping
// pairs outside them never changes a result.
// ---------------------------------------------------------------------------
struct Record {
  float4 a, b, c;
  float idet;
};

__device__ __forceinline__ Record make_record(float x, float y, float cxx, float cxy, float cyy,
                                              float r, float g, float b, float opac) {
  Record rec;
  float det = conic_det(cxx, cxy, cyy);
  float idet = 1.f / det;
  float icxx = cyy * idet;
  float icxy = -cxy * idet;
  float icyy = cxx * idet;
  rec.idet = idet;
  // alpha = min(0.99, o*exp(-sigma)) >= 1/255 needs sigma <= ln(255 o); 0.01 of slack
  // in sigma covers the approximate exp and every rounding step.
  float cut = logf(255.f * opac) + 0.01f;
  float hx, hy;
  if (cut != cut) {  // NaN opacity: the reference still composites the splat
    cut = __int_as_float(0x7f800000);
    hx = hy = __int_as_float(0x7f800000);
  } else if (cut < 0.f) {
    hx = hy = -__int_as_float(0x7f800000);  // never visible anywhere
  } else {
    // Lower bound of the computed quadratic form: shrink the diagonal by a
    // relative 1e-5 of the magnitudes so FP32 cancellation cannot escape the box.
    const float k = 1e-5f;
    float a = icxx - k * (fabsf(icxx) + fabsf(icxy));
    float c = icyy - k * (fabsf(icyy) + fabsf(icxy));
    float dA = a * c - icxy * icxy;
    float R = 2.f * cut;
    if (a > 0.f && c > 0.f && dA > 0.f) {
      hx = sqrtf(R * c / dA) * 1.0001f + 1e-7f;
      hy = sqrtf(R * a / dA) * 1.0001f + 1e-7f;
      if (!(hx <= 3.0e38f)) hx = __int_as_float(0x7f800000);
      if (!(hy <= 3.0e38f)) hy = __int_as_float(0x7f800000);
    } else {
      hx = hy = __int_as_float(0x7f800000);
    }
  }
  rec.a = make_float4(x, y, hx, hy);
  rec.b = make_float4(icxx, icxy, icyy, opac);
  rec.c = make_float4(r, g, b, cut);
  return rec;
}

// ---------------------------------------------------------------------------
// Warp helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ uint32_t warp_sum_u32(uint32_t v) {
  return __reduce_add_sync(0xffffffffu, v);
}

__device__ __forceinline__ int warp_max(int v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Reduces eight per-lane values across the warp with 9 shuffles (a transposing
// butterfly): on return, lane l holds the warp-wide sum of value (l >> 2).
__device__ __forceinline__ float warp_sum8_transposed(const float (&v)[8], int lane) {
  const bool b4 = lane & 16, b3 = lane & 8, b2 = lane & 4;
  float u[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    float keep = b4 ? v[k + 4] : v[k];
    float send = b4 ? v[k] : v[k + 4];
    u[k] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
  }
  float w[2];
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    float keep = b3 ? u[k + 2] : u[k];
    float send = b3 ? u[k] : u[k + 2];
    w[k] = keep + __shfl_xor_sync(0xffffffffu, send, 8);
  }
  float keep = b2 ? w[1] : w[0];
  float send = b2 ? w[0] : w[1];
  float z = keep + __shfl_xor_sync(0xffffffffu, send, 4);
  z += __shfl_xor_sync(0xffffffffu, z, 2);
  z += __shfl_xor_sync(0xffffffffu, z, 1);
  return z;
}

// Two hits' 8 values each, reduced over the warp at once: after the first
// exchange (xor 16) lanes 0-15 carry hit 0 and lanes 16-31 hit 1, then the
// 8-value transposed tree runs within each half.  Even lane l ends up with
// the warp sum of value (l >> 1) & 7 of hit l >> 4.
__device__ __forceinline__ float warp_sum16_transposed(const float (&v0)[8], const float (&v1)[8],
                                                       int lane) {
  const bool b4 = lane & 16, b3 = lane & 8, b2 = lane & 4, b1 = lane & 2;
  float u[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const float keep = b4 ? v1[k] : v0[k];
    const float send = b4 ? v0[k] : v1[k];
    u[k] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
  }
  float w[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const float keep = b3 ? u[k + 4] : u[k];
    const float send = b3 ? u[k] : u[k + 4];
    w[k] = keep + __shfl_xor_sync(0xffffffffu, send, 8);
  }
  float x[2];
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    const float keep = b2 ? w[k + 2] : w[k];
    const float send = b2 ? w[k] : w[k + 2];
    x[k] = keep + __shfl_xor_sync(0xffffffffu, send, 4);
  }
  const float keep = b1 ? x[1] : x[0];
  const float send = b1 ? x[0] : x[1];
  float z = keep + __shfl_xor_sync(0xffffffffu, send, 2);
  z += __shfl_xor_sync(0xffffffffu, z, 1);
  return z;
}

// Two values' warp sums at once: lanes 0-15 end with the sum of a0, lanes
// 16-31 with the sum of a1.
__device__ __forceinline__ float warp_sum2_transposed(float a0, float a1, int lane) {
  const bool b4 = lane & 16;
  float z = (b4 ? a1 : a0) + __shfl_xor_sync(0xffffffffu, b4 ? a0 : a1, 16);
#pragma unroll
  for (int o = 8; o > 0; o >>= 1) z += __shfl_xor_sync(0xffffffffu, z, o);
  return z;
}

// Position gradient through the position dependence of J (Cov2D = J S J^T),
// which the reference's projection backward leaves out.  H is dL/dCov2D in the
// full-matrix convention (off-diagonal = stored gradient / 2), S the 3D
// covariance.  dL/dJ = 2 H J S and
//   dJ[r][k]/dp_m = (P[r][k] P[3][m] - P[r][m] P[3][k]) / w^2 - 2 J[r][k] P[3][m] / w
// with P[r][k] = pv[k*4 + r].
__device__ __forceinline__ float3 jacobian_position_grad(const Mat4& P, const Jac2& J,
                                                         float clip_w, float hxx, float hxy,
                                                         float hyy, float sxx, float sxy,
                                                         float sxz, float syy, float syz,
                                                         float szz) {
  const float Jm[2][3] = {{J.j00, J.j01, J.j02}, {J.j10, J.j11, J.j12}};
  const float Hm[2][2] = {{hxx, hxy}, {hxy, hyy}};
  const float Sm[3][3] = {{sxx, sxy, sxz}, {sxy, syy, syz}, {sxz, syz, szz}};
  float dJ[2][3];
#pragma unroll
  for (int r = 0; r < 2; ++r)
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      float acc = 0.f;
#pragma unroll
      for (int c = 0; c < 2; ++c)
#pragma unroll
        for (int l = 0; l < 3; ++l) acc += Hm[r][c] * Jm[c][l] * Sm[l][k];
      dJ[r][k] = 2.f * acc;
    }
  const float iw = 1.f / clip_w;
  const float iw2 = iw * iw;
  float g[3];
#pragma unroll
  for (int m = 0; m < 3; ++m) {
    float acc = 0.f;
#pragma unroll
    for (int r = 0; r < 2; ++r)
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const float d = (P.m[k * 4 + r] * P.m[m * 4 + 3] - P.m[m * 4 + r] * P.m[k * 4 + 3]) * iw2 -
                        2.f * Jm[r][k] * P.m[m * 4 + 3] * iw;
        acc += dJ[r][k] * d;
      }
    g[m] = acc;
  }
  return make_float3(g[0], g[1], g[2]);
}

}  // namespace ds
