// Activation (Gaussian3D -> Splat3D) and perspective projection (Splat3D ->
// Splat2D) kernels behind the per-layer C ABI entries, plus their backward.
//
// Semantics follow src/layers/gauss_activ_layer.cu:37-407 and
// src/layers/persp_project_layer.cu:40-267: quaternion normalised with a 1e-12
// floor, colour = SH + 0.5 clamped to [0,1] with a strict-interior gradient
// gate, sigmoid opacity, clip_w <= 0 culled by writing only ndc_z = FLT_MAX,
// no low-pass dilation, off-diagonal covariance gradients in the full-matrix
// convention, view direction treated as a constant in the backward.
#include <float.h>

#include "ds_common.cuh"
#include "ds_internal.h"

namespace ds {

__global__ void __launch_bounds__(256) activ_fwd_kernel(ds_gaussian3d in, int degree, float cam_x,
                                                        float cam_y, float cam_z, ds_splat3d out) {
  const int n = in.count;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float px = in.pos_x[i], py = in.pos_y[i], pz = in.pos_z[i];
  out.pos_x[i] = px;
  out.pos_y[i] = py;
  out.pos_z[i] = pz;
  UnitQuat q = unit_quat(in.rot_w[i], in.rot_x[i], in.rot_y[i], in.rot_z[i]);
  Rot3 R = rot_from_quat(q.w, q.x, q.y, q.z);
  float sx = expf(in.scale_x[i]), sy = expf(in.scale_y[i]), sz = expf(in.scale_z[i]);
  Cov3 c = cov3_from(R, sx, sy, sz);
  out.cov_xx[i] = c.xx;
  out.cov_xy[i] = c.xy;
  out.cov_xz[i] = c.xz;
  out.cov_yy[i] = c.yy;
  out.cov_yz[i] = c.yz;
  out.cov_zz[i] = c.zz;
  float3 v = dir_to_camera(cam_x, cam_y, cam_z, px, py, pz);
  float cr = sh_channel(in.sh_dc_r[i], degree > 0 ? in.sh_rest_r + i : nullptr, n, degree, v);
  float cg = sh_channel(in.sh_dc_g[i], degree > 0 ? in.sh_rest_g + i : nullptr, n, degree, v);
  float cb = sh_channel(in.sh_dc_b[i], degree > 0 ? in.sh_rest_b + i : nullptr, n, degree, v);
  out.color_r[i] = clamp01(cr + 0.5f);
  out.color_g[i] = clamp01(cg + 0.5f);
  out.color_b[i] = clamp01(cb + 0.5f);
  out.opacity[i] = 1.f / (1.f + expf(-in.logit_opacity[i]));
}

// dL/d(log-scale), dL/d(raw quaternion) from G = dL/dCov3D (full-matrix
// convention) through Cov = M M^T, M = R S (gauss_activ_layer.cu:259-329).
struct CovGrad {
  float ds_x, ds_y, ds_z, dq_w, dq_x, dq_y, dq_z;
};

__device__ __forceinline__ CovGrad cov3_backward(float rw, float rx, float ry, float rz, float lsx,
                                                 float lsy, float lsz, float g_xx, float g_xy,
                                                 float g_xz, float g_yy, float g_yz, float g_zz) {
  UnitQuat nq = unit_quat(rw, rx, ry, rz);
  Rot3 R = rot_from_quat(nq.w, nq.x, nq.y, nq.z);
  float sx = expf(lsx), sy = expf(lsy), sz = expf(lsz);
  float m00 = R.r00 * sx, m01 = R.r01 * sy, m02 = R.r02 * sz;
  float m10 = R.r10 * sx, m11 = R.r11 * sy, m12 = R.r12 * sz;
  float m20 = R.r20 * sx, m21 = R.r21 * sy, m22 = R.r22 * sz;
  float dm00 = 2.f * (g_xx * m00 + g_xy * m10 + g_xz * m20);
  float dm01 = 2.f * (g_xx * m01 + g_xy * m11 + g_xz * m21);
  float dm02 = 2.f * (g_xx * m02 + g_xy * m12 + g_xz * m22);
  float dm10 = 2.f * (g_xy * m00 + g_yy * m10 + g_yz * m20);
  float dm11 = 2.f * (g_xy * m01 + g_yy * m11 + g_yz * m21);
  float dm12 = 2.f * (g_xy * m02 + g_yy * m12 + g_yz * m22);
  float dm20 = 2.f * (g_xz * m00 + g_yz * m10 + g_zz * m20);
  float dm21 = 2.f * (g_xz * m01 + g_yz * m11 + g_zz * m21);
  float dm22 = 2.f * (g_xz * m02 + g_yz * m12 + g_zz * m22);
  CovGrad o;
  o.ds_x = (dm00 * R.r00 + dm10 * R.r10 + dm20 * R.r20) * sx;
  o.ds_y = (dm01 * R.r01 + dm11 * R.r11 + dm21 * R.r21) * sy;
  o.ds_z = (dm02 * R.r02 + dm12 * R.r12 + dm22 * R.r22) * sz;
  float dr00 = dm00 * sx, dr10 = dm10 * sx, dr20 = dm20 * sx;
  float dr01 = dm01 * sy, dr11 = dm11 * sy, dr21 = dm21 * sy;
  float dr02 = dm02 * sz, dr12 = dm12 * sz, dr22 = dm22 * sz;
  float dqw = 2.f * (dr10 * nq.z - dr20 * nq.y + dr01 * (-nq.z) + dr21 * nq.x + dr02 * nq.y +
                     dr12 * (-nq.x));
  float dqx = 2.f * (dr10 * nq.y + dr20 * nq.z + dr01 * nq.y + dr11 * (-2.f * nq.x) + dr21 * nq.w +
                     dr02 * nq.z + dr12 * (-nq.w) + dr22 * (-2.f * nq.x));
  float dqy = 2.f * (dr00 * (-2.f * nq.y) + dr10 * nq.x + dr20 * (-nq.w) + dr01 * nq.x +
                     dr12 * nq.z + dr21 * nq.z + dr22 * (-2.f * nq.y) + dr02 * nq.w);
  float dqz = 2.f * (dr00 * (-2.f * nq.z) + dr10 * nq.w + dr20 * nq.x + dr01 * (-nq.w) +
                     dr11 * (-2.f * nq.z) + dr12 * nq.y + dr21 * nq.y + dr02 * nq.x);
  float dot = dqw * nq.w + dqx * nq.x + dqy * nq.y + dqz * nq.z;
  o.dq_w = nq.inv_norm * (dqw - dot * nq.w);
  o.dq_x = nq.inv_norm * (dqx - dot * nq.x);
  o.dq_y = nq.inv_norm * (dqy - dot * nq.y);
  o.dq_z = nq.inv_norm * (dqz - dot * nq.z);
  return o;
}

__global__ void __launch_bounds__(256)
    activ_bwd_kernel(ds_gaussian3d in, ds_splat3d saved, ds_splat3d gout, int degree, float cam_x,
                     float cam_y, float cam_z, ds_gaussian3d gin) {
  const int n = in.count;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  gin.pos_x[i] = gout.pos_x[i];
  gin.pos_y[i] = gout.pos_y[i];
  gin.pos_z[i] = gout.pos_z[i];
  CovGrad cg = cov3_backward(in.rot_w[i], in.rot_x[i], in.rot_y[i], in.rot_z[i], in.scale_x[i],
                             in.scale_y[i], in.scale_z[i], gout.cov_xx[i], gout.cov_xy[i],
                             gout.cov_xz[i], gout.cov_yy[i], gout.cov_yz[i], gout.cov_zz[i]);
  gin.scale_x[i] = cg.ds_x;
  gin.scale_y[i] = cg.ds_y;
  gin.scale_z[i] = cg.ds_z;
  gin.rot_w[i] = cg.dq_w;
  gin.rot_x[i] = cg.dq_x;
  gin.rot_y[i] = cg.dq_y;
  gin.rot_z[i] = cg.dq_z;
  float cr = saved.color_r[i], cgc = saved.color_g[i], cb = saved.color_b[i];
  float dR = (cr > 0.f && cr < 1.f) ? gout.color_r[i] : 0.f;
  float dG = (cgc > 0.f && cgc < 1.f) ? gout.color_g[i] : 0.f;
  float dB = (cb > 0.f && cb < 1.f) ? gout.color_b[i] : 0.f;
  gin.sh_dc_r[i] = dR * kC0;
  gin.sh_dc_g[i] = dG * kC0;
  gin.sh_dc_b[i] = dB * kC0;
  if (degree >= 1) {
    float3 v = dir_to_camera(cam_x, cam_y, cam_z, in.pos_x[i], in.pos_y[i], in.pos_z[i]);
    float y[15];
    sh_basis(degree, v, y);
    const int nb = sh_bands(degree);
    for (int b = 0; b < nb; ++b) {
      gin.sh_rest_r[b * n + i] = dR * y[b];
      gin.sh_rest_g[b * n + i] = dG * y[b];
      gin.sh_rest_b[b * n + i] = dB * y[b];
    }
  }
  float s = saved.opacity[i];
  gin.logit_opacity[i] = gout.opacity[i] * s * (1.f - s);
}

__global__ void __launch_bounds__(256) project_fwd_kernel(ds_splat3d in, Mat4 P, ds_splat2d out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= in.count) return;
  float x = in.pos_x[i], y = in.pos_y[i], z = in.pos_z[i];
  float clip_x, clip_y, clip_z, clip_w;
  project_jacobian(P, x, y, z, clip_x, clip_y, clip_z, clip_w);
  if (clip_w <= 0.f) {
    out.pos_z[i] = FLT_MAX;  // other outputs keep their previous contents
    return;
  }
  float inv_w = 1.f / clip_w;
  float inv_w2 = inv_w * inv_w;
  out.pos_x[i] = clip_x * inv_w;
  out.pos_y[i] = clip_y * inv_w;
  out.pos_z[i] = clip_z * inv_w;
  Jac2 J = jacobian(P, clip_x, clip_y, clip_w, inv_w2);
  Cov2 c = cov2_from(J, in.cov_xx[i], in.cov_xy[i], in.cov_xz[i], in.cov_yy[i], in.cov_yz[i],
                     in.cov_zz[i]);
  out.cov_xx[i] = c.xx;
  out.cov_xy[i] = c.xy;
  out.cov_yy[i] = c.yy;
  out.color_r[i] = in.color_r[i];
  out.color_g[i] = in.color_g[i];
  out.color_b[i] = in.color_b[i];
  out.opacity[i] = in.opacity[i];
}

// dL/dCov3D = J^T H J with H = [[gxx, gxy/2], [gxy/2, gyy]] and dL/dpos = J^T dndc_xy
// (persp_project_layer.cu:244-260).
struct ProjGrad {
  float px, py, pz, cxx, cxy, cxz, cyy, cyz, czz;
};

__device__ __forceinline__ ProjGrad project_backward(const Jac2& J, float gx, float gy, float dcxx,
                                                     float dcxy, float dcyy) {
  ProjGrad o;
  const float j00 = J.j00, j01 = J.j01, j02 = J.j02, j10 = J.j10, j11 = J.j11, j12 = J.j12;
  float hdxy = 0.5f * dcxy;
  o.cxx = j00 * j00 * dcxx + j00 * j10 * dcxy + j10 * j10 * dcyy;
  o.cxy = j00 * j01 * dcxx + hdxy * (j00 * j11 + j10 * j01) + j10 * j11 * dcyy;
  o.cxz = j00 * j02 * dcxx + hdxy * (j00 * j12 + j10 * j02) + j10 * j12 * dcyy;
  o.cyy = j01 * j01 * dcxx + j01 * j11 * dcxy + j11 * j11 * dcyy;
  o.cyz = j01 * j02 * dcxx + hdxy * (j01 * j12 + j11 * j02) + j11 * j12 * dcyy;
  o.czz = j02 * j02 * dcxx + j02 * j12 * dcxy + j12 * j12 * dcyy;
  o.px = gx * j00 + gy * j10;
  o.py = gx * j01 + gy * j11;
  o.pz = gx * j02 + gy * j12;
  return o;
}

__global__ void __launch_bounds__(256)
    project_bwd_kernel(ds_splat3d in, Mat4 P, ds_splat2d gout, ds_splat3d gin, int exact) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= in.count) return;
  float x = in.pos_x[i], y = in.pos_y[i], z = in.pos_z[i];
  float clip_x, clip_y, clip_z, clip_w;
  project_jacobian(P, x, y, z, clip_x, clip_y, clip_z, clip_w);
  if (clip_w <= 0.f) {
    gin.pos_x[i] = 0.f;
    gin.pos_y[i] = 0.f;
    gin.pos_z[i] = 0.f;
    gin.cov_xx[i] = 0.f;
    gin.cov_xy[i] = 0.f;
    gin.cov_xz[i] = 0.f;
    gin.cov_yy[i] = 0.f;
    gin.cov_yz[i] = 0.f;
    gin.cov_zz[i] = 0.f;
    gin.color_r[i] = 0.f;
    gin.color_g[i] = 0.f;
    gin.color_b[i] = 0.f;
    gin.opacity[i] = 0.f;
    return;
  }
  float inv_w = 1.f / clip_w;
  float inv_w2 = inv_w * inv_w;
  Jac2 J = jacobian(P, clip_x, clip_y, clip_w, inv_w2);
  ProjGrad g = project_backward(J, gout.pos_x[i], gout.pos_y[i], gout.cov_xx[i], gout.cov_xy[i],
                                gout.cov_yy[i]);
  gin.cov_xx[i] = g.cxx;
  gin.cov_xy[i] = g.cxy;
  gin.cov_xz[i] = g.cxz;
  gin.cov_yy[i] = g.cyy;
  gin.cov_yz[i] = g.cyz;
  gin.cov_zz[i] = g.czz;
  gin.pos_x[i] = g.px;
  gin.pos_y[i] = g.py;
  gin.pos_z[i] = g.pz;
  if (exact) {
    float3 e = jacobian_position_grad(P, J, clip_w, gout.cov_xx[i], 0.5f * gout.cov_xy[i],
                                      gout.cov_yy[i], in.cov_xx[i], in.cov_xy[i], in.cov_xz[i],
                                      in.cov_yy[i], in.cov_yz[i], in.cov_zz[i]);
    gin.pos_x[i] = g.px + e.x;
    gin.pos_y[i] = g.py + e.y;
    gin.pos_z[i] = g.pz + e.z;
  }
  gin.color_r[i] = gout.color_r[i];
  gin.color_g[i] = gout.color_g[i];
  gin.color_b[i] = gout.color_b[i];
  gin.opacity[i] = gout.opacity[i];
}

// ---------------------------------------------------------------------------
// Host launchers
// ---------------------------------------------------------------------------
static inline int blocks_for(int64_t n, int threads) { return (int)((n + threads - 1) / threads); }

int launch_activ_forward(const ds_gaussian3d& in, int degree, const float cam[3],
                         const ds_splat3d& out, cudaStream_t s) {
  if (in.count <= 0) return DS_OK;
  activ_fwd_kernel<<<blocks_for(in.count, 256), 256, 0, s>>>(in, degree, cam[0], cam[1], cam[2],
                                                             out);
  return cuda_status(cudaGetLastError());
}

int launch_activ_backward(const ds_gaussian3d& in, const ds_splat3d& saved,
                          const ds_splat3d& gout, int degree, const float cam[3],
                          const ds_gaussian3d& gin, cudaStream_t s) {
  if (in.count <= 0) return DS_OK;
  activ_bwd_kernel<<<blocks_for(in.count, 256), 256, 0, s>>>(in, saved, gout, degree, cam[0],
                                                             cam[1], cam[2], gin);
  return cuda_status(cudaGetLastError());
}

int launch_project_forward(const ds_splat3d& in, const float pv[16], const ds_splat2d& out,
                           cudaStream_t s) {
  if (in.count <= 0) return DS_OK;
  Mat4 P;
  for (int k = 0; k < 16; ++k) P.m[k] = pv[k];
  project_fwd_kernel<<<blocks_for(in.count, 256), 256, 0, s>>>(in, P, out);
  return cuda_status(cudaGetLastError());
}

int launch_project_backward(const ds_splat3d& in, const float pv[16], const ds_splat2d& gout,
                            const ds_splat3d& gin, int mode, cudaStream_t s) {
  if (in.count <= 0) return DS_OK;
  Mat4 P;
  for (int k = 0; k < 16; ++k) P.m[k] = pv[k];
  project_bwd_kernel<<<blocks_for(in.count, 256), 256, 0, s>>>(in, P, gout, gin,
                                                               mode == DS_GRAD_EXACT ? 1 : 0);
  return cuda_status(cudaGetLastError());
}

}  // namespace ds
