// Fused training step of ImageFitter::step (src/pipelines/image_fitter.cpp:103-112).
//
// The reference runs ~40 launches per step, one blocking host read of
// n_isects and one launch per Adam group.  Here the step is a fixed sequence
// of kernels with no host synchronisation, captured once into a CUDA graph:
//
//   step_begin         step counter, Adam bias corrections (host-computed
//                      table, identical to the reference's powf), resets
//   preprocess         activation + projection + tile rectangle + record,
//                      one thread per splat; Splat3D/Splat2D never hit HBM
//   build_lists        depth sort, emission scan, emission, tile sort, ranges
//   composite fwd      image, alphas, last ids and the MSE loss
//   composite bwd      dL/dpixel from the image and target (MSE backward
//                      fused), one gradient record per (tile, splat)
//   backward_adam      per splat: sum of its records -> projection backward
//                      -> activation backward -> Adam on all 14 + 3K fields
//
// Gradients of one step equal the layer pipeline's up to float summation
// order; zeroGrad is unnecessary because every gradient is written, not
// accumulated.
#include <float.h>
#include <math.h>

#include <algorithm>
#include <new>
#include <vector>

#include "ds_common.cuh"
#include "ds_internal.h"
#include "ds_preprocess.cuh"

namespace ds {

namespace {

constexpr int kThreads = 256;
constexpr int kBcTableMax = 1 << 20;

struct Lrs {
  float pos, scale, rot, sh_dc, sh_rest, opacity;
};

__global__ void step_begin_kernel(DevScalars* sc, const float2* __restrict__ bc_table,
                                  int table_len, float2* __restrict__ bc_out) {
  uint32_t t = sc->step + 1u;
  sc->step = t;
  sc->visible = 0u;
  sc->ticket = 0u;
  sc->n_splats = sc->n_splats;  // set once at creation
  float2 bc = make_float2(1.f, 1.f);
  if ((int)t <= table_len) bc = bc_table[t - 1];
  *bc_out = bc;
}

__device__ __forceinline__ void adam1(float& p, float& m, float& v, float g, float lr, float b1,
                                      float b2, float eps, float bc1, float bc2) {
  m = b1 * m + (1.f - b1) * g;
  v = b2 * v + (1.f - b2) * g * g;
  float m_hat = m * bc1;
  float v_hat = v * bc2;
  p -= lr * m_hat / (sqrtf(v_hat) + eps);
}

// Integer hash "lowbias32" (C. Wellons, 2018): the random bits of the
// stochastic rounding of BF16 Adam moments, from (element, field, step).
__device__ __forceinline__ uint32_t mix32(uint32_t x) {
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  x ^= x >> 16;
  return x;
}

// FP32 -> BF16 with stochastic rounding: adds 16 random bits below the kept
// mantissa and truncates, so E[result] = x.  An Adam moment updated by
// (1 - beta2) = 1e-3 of itself per step would otherwise round back to its old
// value forever under round-to-nearest (BF16 keeps 8 significant bits).
__device__ __forceinline__ __nv_bfloat16 bf16_stochastic(float x, uint32_t r) {
  uint32_t u = __float_as_uint(x);
  if ((u & 0x7f800000u) == 0x7f800000u) return __float2bfloat16_rn(x);
  u += r & 0xffffu;
  return __ushort_as_bfloat16((unsigned short)(u >> 16));
}

__device__ __forceinline__ void store_moment(float* p, float x, uint32_t) { *p = x; }
__device__ __forceinline__ void store_moment(__nv_bfloat16* p, float x, uint32_t r) {
  *p = bf16_stochastic(x, r);
}

// Adam on one element of the FP32 master p with moments of type T; `key`
// identifies (element, field, step) for the stochastic rounding of BF16 moments.
template <typename T>
__device__ __forceinline__ void adam_at(float* __restrict__ p, T* __restrict__ m,
                                        T* __restrict__ v, int64_t i, float g, float lr, float b1,
                                        float b2, float eps, float bc1, float bc2, uint32_t key) {
  float pp = p[i], mm = ldv(m[i]), vv = ldv(v[i]);
  adam1(pp, mm, vv, g, lr, b1, b2, eps, bc1, bc2);
  p[i] = pp;
  const uint32_t h = mix32(key ^ mix32((uint32_t)i));
  store_moment(m + i, mm, h);
  store_moment(v + i, vv, mix32(h + 0x9e3779b9u));
}

struct AdamHyper {
  float b1, b2, eps;
};

// dL/dCov3D -> dL/d(log-scale, raw quaternion); identical to the layer
// backward in ds_activ_project.cu (gauss_activ_layer.cu:259-329).
__device__ __forceinline__ void cov_backward(float rw, float rx, float ry, float rz, float lsx,
                                             float lsy, float lsz, float g_xx, float g_xy,
                                             float g_xz, float g_yy, float g_yz, float g_zz,
                                             float* d) {
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
  d[0] = (dm00 * R.r00 + dm10 * R.r10 + dm20 * R.r20) * sx;
  d[1] = (dm01 * R.r01 + dm11 * R.r11 + dm21 * R.r21) * sy;
  d[2] = (dm02 * R.r02 + dm12 * R.r12 + dm22 * R.r22) * sz;
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
  d[3] = nq.inv_norm * (dqw - dot * nq.w);
  d[4] = nq.inv_norm * (dqx - dot * nq.x);
  d[5] = nq.inv_norm * (dqy - dot * nq.y);
  d[6] = nq.inv_norm * (dqz - dot * nq.z);
}

// Backward of one step and Adam.  P holds the FP32 masters (updated in
// place), R the attributes the forward rendered (P itself in FP32 storage; in
// BF16 storage the render copy, rewritten from the updated masters), M and V
// the moments in the storage type.
template <typename T>
__global__ void __launch_bounds__(kThreads)
    fit_backward_adam_kernel(ds_gaussian3d P, Soa<T> R, Soa<T> M, Soa<T> V, ds_gaussian3d G,
                             int keep_grads, int exact, int degree, const Camera* __restrict__ camp,
                             const float* __restrict__ g2sum, const float2* __restrict__ bcp,
                             const DevScalars* __restrict__ sc, Lrs lr, AdamHyper h) {
  constexpr bool kBf16 = sizeof(T) == 2;
  __shared__ Mat4 sP;
  __shared__ float sCam[3];
  if (threadIdx.x < 16) sP.m[threadIdx.x] = camp->pv[threadIdx.x];
  if (threadIdx.x < 3) sCam[threadIdx.x] = camp->cam[threadIdx.x];
  __syncthreads();
  const int n = P.count;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float2 bc = *bcp;
  const uint32_t step = kBf16 ? sc->step : 0u;

  // 1) Splat2D gradient = sum of this splat's per-tile records (segment_reduce_kernel).
  float g2[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) g2[k] = g2sum[(size_t)k * n + i];
  // g2 = {color r, g, b, ndc x, ndc y, cov2 xx, xy, yy, opacity}

  // 2) projection backward (persp_project_layer.cu:245-305)
  const float px = P.pos_x[i], py = P.pos_y[i], pz = P.pos_z[i];
  const float rw = ldv(R.rot_w[i]), rx = ldv(R.rot_x[i]), ry = ldv(R.rot_y[i]),
              rz = ldv(R.rot_z[i]);
  const float lsx = ldv(R.scale_x[i]), lsy = ldv(R.scale_y[i]), lsz = ldv(R.scale_z[i]);
  float clip_x, clip_y, clip_z, clip_w;
  project_jacobian(sP, px, py, pz, clip_x, clip_y, clip_z, clip_w);
  float gpos[3] = {0.f, 0.f, 0.f};
  float gcov[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  float gcol[3] = {0.f, 0.f, 0.f};
  float gop = 0.f;
  if (clip_w > 0.f) {
    const float inv_w = 1.f / clip_w;
    const float inv_w2 = inv_w * inv_w;
    Jac2 J = jacobian(sP, clip_x, clip_y, clip_w, inv_w2);
    const float j00 = J.j00, j01 = J.j01, j02 = J.j02, j10 = J.j10, j11 = J.j11, j12 = J.j12;
    const float dcxx = g2[5], dcxy = g2[6], dcyy = g2[7];
    const float hdxy = 0.5f * dcxy;
    gcov[0] = j00 * j00 * dcxx + j00 * j10 * dcxy + j10 * j10 * dcyy;
    gcov[1] = j00 * j01 * dcxx + hdxy * (j00 * j11 + j10 * j01) + j10 * j11 * dcyy;
    gcov[2] = j00 * j02 * dcxx + hdxy * (j00 * j12 + j10 * j02) + j10 * j12 * dcyy;
    gcov[3] = j01 * j01 * dcxx + j01 * j11 * dcxy + j11 * j11 * dcyy;
    gcov[4] = j01 * j02 * dcxx + hdxy * (j01 * j12 + j11 * j02) + j11 * j12 * dcyy;
    gcov[5] = j02 * j02 * dcxx + j02 * j12 * dcxy + j12 * j12 * dcyy;
    gpos[0] = g2[3] * j00 + g2[4] * j10;
    gpos[1] = g2[3] * j01 + g2[4] * j11;
    gpos[2] = g2[3] * j02 + g2[4] * j12;
    gcol[0] = g2[0];
    gcol[1] = g2[1];
    gcol[2] = g2[2];
    gop = g2[8];
    if (exact) {
      UnitQuat q = unit_quat(rw, rx, ry, rz);
      Rot3 Rm = rot_from_quat(q.w, q.x, q.y, q.z);
      Cov3 c3 = cov3_from(Rm, expf(lsx), expf(lsy), expf(lsz));
      float3 e = jacobian_position_grad(sP, J, clip_w, dcxx, hdxy, dcyy, c3.xx, c3.xy, c3.xz,
                                        c3.yy, c3.yz, c3.zz);
      gpos[0] += e.x;
      gpos[1] += e.y;
      gpos[2] += e.z;
    }
  }

  // 3) activation backward (gauss_activ_layer.cu:254-406)
  float d[7];
  cov_backward(rw, rx, ry, rz, lsx, lsy, lsz, gcov[0], gcov[1], gcov[2], gcov[3], gcov[4],
               gcov[5], d);
  const float3 v = dir_to_camera(sCam[0], sCam[1], sCam[2], px, py, pz);
  float y[15];
  sh_basis(degree, v, y);
  const T* no = nullptr;
  const float dc_r = ldv(R.sh_dc_r[i]), dc_g = ldv(R.sh_dc_g[i]), dc_b = ldv(R.sh_dc_b[i]);
  const float col_r =
      clamp01(sh_channel(dc_r, degree > 0 ? R.sh_rest_r + i : no, n, degree, v) + 0.5f);
  const float col_g =
      clamp01(sh_channel(dc_g, degree > 0 ? R.sh_rest_g + i : no, n, degree, v) + 0.5f);
  const float col_b =
      clamp01(sh_channel(dc_b, degree > 0 ? R.sh_rest_b + i : no, n, degree, v) + 0.5f);
  const float dR = (col_r > 0.f && col_r < 1.f) ? gcol[0] : 0.f;
  const float dG = (col_g > 0.f && col_g < 1.f) ? gcol[1] : 0.f;
  const float dB = (col_b > 0.f && col_b < 1.f) ? gcol[2] : 0.f;
  const float logit = ldv(R.logit_opacity[i]);
  const float s = 1.f / (1.f + expf(-logit));
  const float glogit = gop * s * (1.f - s);

  if (keep_grads) {
    G.pos_x[i] = gpos[0];
    G.pos_y[i] = gpos[1];
    G.pos_z[i] = gpos[2];
    G.scale_x[i] = d[0];
    G.scale_y[i] = d[1];
    G.scale_z[i] = d[2];
    G.rot_w[i] = d[3];
    G.rot_x[i] = d[4];
    G.rot_y[i] = d[5];
    G.rot_z[i] = d[6];
    G.sh_dc_r[i] = dR * kC0;
    G.sh_dc_g[i] = dG * kC0;
    G.sh_dc_b[i] = dB * kC0;
    G.logit_opacity[i] = glogit;
    const int nb = sh_bands(degree);
    for (int b = 0; b < nb; ++b) {
      G.sh_rest_r[(int64_t)b * n + i] = dR * y[b];
      G.sh_rest_g[(int64_t)b * n + i] = dG * y[b];
      G.sh_rest_b[(int64_t)b * n + i] = dB * y[b];
    }
  }

  // 4) Adam on every field (adam.cu:12-37), group learning rates of
  //    registerGaussian3DGroups (gaussian3d_adam.h:27-55).  In BF16 storage
  //    the render copy of every non-position field follows its master.
  const float b1 = h.b1, b2 = h.b2, eps = h.eps, bc1 = bc.x, bc2 = bc.y;
  uint32_t field = 0;
  auto upd = [&](float* p, T* m, T* vv, T* r, int64_t k, float g, float l) {
    adam_at(p, m, vv, k, g, l, b1, b2, eps, bc1, bc2, mix32(step * 32u + field++));
    if (kBf16 && r) r[k] = __float2bfloat16_rn(p[k]);
  };
  upd(P.pos_x, M.pos_x, V.pos_x, nullptr, i, gpos[0], lr.pos);
  upd(P.pos_y, M.pos_y, V.pos_y, nullptr, i, gpos[1], lr.pos);
  upd(P.pos_z, M.pos_z, V.pos_z, nullptr, i, gpos[2], lr.pos);
  upd(P.scale_x, M.scale_x, V.scale_x, R.scale_x, i, d[0], lr.scale);
  upd(P.scale_y, M.scale_y, V.scale_y, R.scale_y, i, d[1], lr.scale);
  upd(P.scale_z, M.scale_z, V.scale_z, R.scale_z, i, d[2], lr.scale);
  upd(P.rot_w, M.rot_w, V.rot_w, R.rot_w, i, d[3], lr.rot);
  upd(P.rot_x, M.rot_x, V.rot_x, R.rot_x, i, d[4], lr.rot);
  upd(P.rot_y, M.rot_y, V.rot_y, R.rot_y, i, d[5], lr.rot);
  upd(P.rot_z, M.rot_z, V.rot_z, R.rot_z, i, d[6], lr.rot);
  upd(P.sh_dc_r, M.sh_dc_r, V.sh_dc_r, R.sh_dc_r, i, dR * kC0, lr.sh_dc);
  upd(P.sh_dc_g, M.sh_dc_g, V.sh_dc_g, R.sh_dc_g, i, dG * kC0, lr.sh_dc);
  upd(P.sh_dc_b, M.sh_dc_b, V.sh_dc_b, R.sh_dc_b, i, dB * kC0, lr.sh_dc);
  upd(P.logit_opacity, M.logit_opacity, V.logit_opacity, R.logit_opacity, i, glogit,
      lr.opacity);
  const int nb = P.sh_num_bands;
  const int nb_used = sh_bands(degree);
  for (int b = 0; b < nb; ++b) {
    const int64_t k = (int64_t)b * n + i;
    const float yb = b < nb_used ? y[b] : 0.f;
    field = 16u + 3u * (uint32_t)b;
    upd(P.sh_rest_r, M.sh_rest_r, V.sh_rest_r, R.sh_rest_r, k, dR * yb, lr.sh_rest);
    upd(P.sh_rest_g, M.sh_rest_g, V.sh_rest_g, R.sh_rest_g, k, dG * yb, lr.sh_rest);
    upd(P.sh_rest_b, M.sh_rest_b, V.sh_rest_b, R.sh_rest_b, k, dB * yb, lr.sh_rest);
  }
}

}  // namespace

}  // namespace ds

struct ds_fitter {
  ds_fitter_config cfg{};
  int bands = 0;
  size_t floats = 0;  // per SoA
  float* params_mem = nullptr;
  float* m_mem = nullptr;
  float* v_mem = nullptr;
  float* g_mem = nullptr;
  ds_gaussian3d P{}, M{}, V{}, G{};
  // BF16 storage: render copy of the masters and the Adam moments
  __nv_bfloat16* render_mem = nullptr;
  ds::Soa<__nv_bfloat16> R16{}, M16{}, V16{};
  bool render_dirty = true;
  float* target = nullptr;
  float* image = nullptr;
  ds::RasterBuffers rb;
  ds::Camera* cam_dev = nullptr;
  float2* bc_table = nullptr;
  float2* bc_cur = nullptr;
  int bc_len = 0;
  bool have_target = false, have_camera = false;
  cudaStream_t capture_stream = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int host_steps = 0;
};

namespace ds {

// Enqueues one training step.  When ev != nullptr (8 events) the stage
// boundaries are recorded: ev[0] start, [1] preprocess, [2] depth sort,
// [3] scan + emission, [4] tile sort + ranges, [5] composite forward,
// [6] composite backward, [7] backward + Adam.
static int fitter_enqueue(ds_fitter* f, cudaStream_t s, cudaEvent_t* ev = nullptr) {
  RasterBuffers& rb = f->rb;
  const int n = f->cfg.count;
  if (ev) DS_CUDA(cudaEventRecord(ev[0], s));
  step_begin_kernel<<<1, 1, 0, s>>>(rb.scalars, f->bc_table, f->bc_len, f->bc_cur);
  DS_CUDA(cudaGetLastError());
  const int blocks = (n + kThreads - 1) / kThreads;
  const bool bf16 = f->cfg.storage == DS_STORAGE_BF16;
  if (bf16)
    fit_preprocess_kernel<<<blocks, kThreads, 0, s>>>(
        f->P, f->R16, f->cfg.sh_degree, f->cam_dev, rb.width, rb.height, rb.ntx, rb.nty,
        rb.rec_a, rb.rec_b, rb.rec_c, rb.rec_idet, rb.rect, rb.counts, rb.depth_keys, rb.scalars);
  else
    fit_preprocess_kernel<<<blocks, kThreads, 0, s>>>(
        f->P, soa_of(f->P), f->cfg.sh_degree, f->cam_dev, rb.width, rb.height, rb.ntx, rb.nty,
        rb.rec_a, rb.rec_b, rb.rec_c, rb.rec_idet, rb.rect, rb.counts, rb.depth_keys, rb.scalars);
  DS_CUDA(cudaGetLastError());
  if (ev) DS_CUDA(cudaEventRecord(ev[1], s));
  DS_TRY(raster_build_lists(rb, n, s, ev ? ev + 2 : nullptr));
  DS_TRY(raster_composite_forward(rb, f->image, f->target, s));
  if (ev) DS_CUDA(cudaEventRecord(ev[5], s));
  DS_TRY(raster_composite_backward(rb, f->image, nullptr, f->target, s));
  if (ev) DS_CUDA(cudaEventRecord(ev[6], s));
  DS_TRY(raster_reduce_grads_soa(rb, n, s));
  Lrs lr{f->cfg.lr_pos, f->cfg.lr_scale, f->cfg.lr_rot, f->cfg.lr_sh_dc, f->cfg.lr_sh_rest,
         f->cfg.lr_opacity};
  AdamHyper h{f->cfg.beta1, f->cfg.beta2, f->cfg.epsilon};
  const int keep = f->g_mem ? 1 : 0, exact = f->cfg.grad_mode == DS_GRAD_EXACT ? 1 : 0;
  if (bf16)
    fit_backward_adam_kernel<<<blocks, kThreads, 0, s>>>(f->P, f->R16, f->M16, f->V16, f->G, keep,
                                                         exact, f->cfg.sh_degree, f->cam_dev,
                                                         rb.g2, f->bc_cur, rb.scalars, lr, h);
  else
    fit_backward_adam_kernel<<<blocks, kThreads, 0, s>>>(
        f->P, soa_of(f->P), soa_of(f->M), soa_of(f->V), f->G, keep, exact, f->cfg.sh_degree,
        f->cam_dev, rb.g2, f->bc_cur, rb.scalars, lr, h);
  DS_CUDA(cudaGetLastError());
  if (ev) DS_CUDA(cudaEventRecord(ev[7], s));
  return DS_OK;
}

// BF16 storage: rewrites the render copy from the masters after the caller
// changed them (outside the captured graph, on the step's stream).
static int refresh_render_copy(ds_fitter* f, cudaStream_t s) {
  if (f->cfg.storage != DS_STORAGE_BF16 || !f->render_dirty) return DS_OK;
  const size_t blocks = std::min<size_t>((f->floats + kThreads - 1) / kThreads, 148 * 16);
  to_bf16_kernel<<<(unsigned)blocks, kThreads, 0, s>>>(f->params_mem, f->render_mem, f->floats);
  DS_CUDA(cudaGetLastError());
  f->render_dirty = false;
  return DS_OK;
}

}  // namespace ds

extern "C" {

int ds_fitter_default_config(ds_fitter_config* cfg) {
  if (!cfg) return DS_ERR_ARG;
  *cfg = ds_fitter_config{};
  cfg->width = 0;
  cfg->height = 0;
  cfg->count = 0;
  cfg->sh_degree = 0;
  cfg->max_isects = 0;
  cfg->lr_pos = 1.6e-2f;
  cfg->lr_scale = 1.0e-3f;
  cfg->lr_rot = 6.0e-4f;
  cfg->lr_sh_dc = 6.0e-3f;
  cfg->lr_sh_rest = 6.0e-3f;
  cfg->lr_opacity = 6.0e-3f;
  cfg->beta1 = 0.9f;
  cfg->beta2 = 0.999f;
  cfg->epsilon = 1e-8f;
  cfg->storage = DS_STORAGE_FP32;
  cfg->use_graph = 1;
  cfg->grad_mode = ds_default_grad_mode();
  cfg->schedule = ds::composite_longest_first() ? DS_SCHEDULE_LONGEST_FIRST : DS_SCHEDULE_RASTER;
  return DS_OK;
}

int ds_fitter_destroy(ds_fitter* f) {
  if (!f) return DS_ERR_ARG;
  if (f->exec) cudaGraphExecDestroy(f->exec);
  if (f->graph) cudaGraphDestroy(f->graph);
  if (f->capture_stream) cudaStreamDestroy(f->capture_stream);
  ds::raster_free(f->rb);
  cudaFree(f->params_mem);
  cudaFree(f->m_mem);
  cudaFree(f->v_mem);
  cudaFree(f->g_mem);
  cudaFree(f->render_mem);
  cudaFree(f->target);
  cudaFree(f->image);
  cudaFree(f->cam_dev);
  cudaFree(f->bc_table);
  cudaFree(f->bc_cur);
  delete f;
  return DS_OK;
}

static int ds_fitter_create_impl(const ds_fitter_config* cfg, int keep_grads, ds_fitter** out) {
  if (!cfg || !out) return DS_ERR_ARG;
  *out = nullptr;
  if (cfg->width <= 0 || cfg->height <= 0 || cfg->count <= 0 || cfg->sh_degree < 0 ||
      cfg->sh_degree > 3)
    return DS_ERR_ARG;
  if (cfg->storage != DS_STORAGE_FP32 && cfg->storage != DS_STORAGE_BF16) return DS_ERR_ARG;
  if (cfg->grad_mode != DS_GRAD_REFERENCE && cfg->grad_mode != DS_GRAD_EXACT) return DS_ERR_ARG;
  if (cfg->schedule != DS_SCHEDULE_LONGEST_FIRST && cfg->schedule != DS_SCHEDULE_RASTER)
    return DS_ERR_ARG;
  ds_fitter* f = new (std::nothrow) ds_fitter();
  if (!f) return DS_ERR_OOM;
  f->cfg = *cfg;
  f->bands = ds::sh_bands(cfg->sh_degree);
  const int n = cfg->count;
  f->floats = (size_t)n * (14 + 3 * f->bands);
  int st = DS_OK;
  auto fail = [&](int code) {
    ds_fitter_destroy(f);
    return code;
  };
  const bool bf16 = cfg->storage == DS_STORAGE_BF16;
  const size_t mom_bytes = f->floats * (bf16 ? 2 : 4);
  if ((st = ds::cuda_status(cudaMalloc(&f->params_mem, f->floats * 4)))) return fail(st);
  if ((st = ds::cuda_status(cudaMalloc(&f->m_mem, mom_bytes)))) return fail(st);
  if ((st = ds::cuda_status(cudaMalloc(&f->v_mem, mom_bytes)))) return fail(st);
  cudaMemset(f->params_mem, 0, f->floats * 4);
  cudaMemset(f->m_mem, 0, mom_bytes);
  cudaMemset(f->v_mem, 0, mom_bytes);
  ds::carve(f->params_mem, n, f->bands, f->P);
  if (bf16) {
    if ((st = ds::cuda_status(cudaMalloc(&f->render_mem, f->floats * 2)))) return fail(st);
    cudaMemset(f->render_mem, 0, f->floats * 2);
    ds::carve_soa(f->render_mem, n, f->bands, f->R16);
    ds::carve_soa((__nv_bfloat16*)f->m_mem, n, f->bands, f->M16);
    ds::carve_soa((__nv_bfloat16*)f->v_mem, n, f->bands, f->V16);
    f->M = f->V = ds_gaussian3d{};  // FP32 views do not exist in this mode
  } else {
    ds::carve(f->m_mem, n, f->bands, f->M);
    ds::carve(f->v_mem, n, f->bands, f->V);
  }
  if (keep_grads) {
    if ((st = ds::cuda_status(cudaMalloc(&f->g_mem, f->floats * 4)))) return fail(st);
    cudaMemset(f->g_mem, 0, f->floats * 4);
    ds::carve(f->g_mem, n, f->bands, f->G);
  } else {
    f->G = f->P;  // never written (keep_grads == 0)
  }
  const size_t px = (size_t)cfg->width * cfg->height;
  if ((st = ds::cuda_status(cudaMalloc(&f->target, px * 3 * 4)))) return fail(st);
  if ((st = ds::cuda_status(cudaMalloc(&f->image, px * 3 * 4)))) return fail(st);
  cudaMemset(f->image, 0, px * 3 * 4);
  if ((st = ds::raster_alloc(f->rb, cfg->width, cfg->height, n, cfg->max_isects))) return fail(st);
  f->rb.grad_mode = cfg->grad_mode;
  f->rb.schedule = cfg->schedule;
  if ((st = ds::cuda_status(cudaMalloc(&f->cam_dev, sizeof(ds::Camera))))) return fail(st);
  cudaMemset(f->cam_dev, 0, sizeof(ds::Camera));
  // Bias-correction table: bc_k(t) = 1 / (1 - powf(beta_k, t)) on the host, like
  // the reference (adam.cu:61-62).  Past the table both corrections are 1.0f.
  std::vector<float2> tab;
  for (int t = 1; t <= ds::kBcTableMax; ++t) {
    float p1 = powf(cfg->beta1, (float)t), p2 = powf(cfg->beta2, (float)t);
    float bc1 = 1.f / (1.f - p1), bc2 = 1.f / (1.f - p2);
    tab.push_back(make_float2(bc1, bc2));
    if (bc1 == 1.f && bc2 == 1.f) break;
  }
  f->bc_len = (int)tab.size();
  if ((st = ds::cuda_status(cudaMalloc(&f->bc_table, tab.size() * sizeof(float2))))) return fail(st);
  if ((st = ds::cuda_status(cudaMalloc(&f->bc_cur, sizeof(float2))))) return fail(st);
  cudaMemcpy(f->bc_table, tab.data(), tab.size() * sizeof(float2), cudaMemcpyHostToDevice);
  // The depth sort reads its element count from device memory.
  uint32_t nn = (uint32_t)n;
  cudaMemcpy(&f->rb.scalars->n_splats, &nn, sizeof(uint32_t), cudaMemcpyHostToDevice);
  if ((st = ds::cuda_status(cudaStreamCreateWithFlags(&f->capture_stream, cudaStreamNonBlocking))))
    return fail(st);
  if ((st = ds::cuda_status(cudaDeviceSynchronize()))) return fail(st);
  *out = f;
  return DS_OK;
}

int ds_fitter_create(const ds_fitter_config* cfg, ds_fitter** out) {
  return ds_fitter_create_impl(cfg, 0, out);
}

int ds_fitter_params(ds_fitter* f, ds_gaussian3d* out) {
  if (!f || !out) return DS_ERR_ARG;
  *out = f->P;
  f->render_dirty = true;
  return DS_OK;
}

int ds_fitter_params_updated(ds_fitter* f) {
  if (!f) return DS_ERR_ARG;
  f->render_dirty = true;
  return DS_OK;
}

int ds_fitter_set_target(ds_fitter* f, const float* target, ds_stream stream) {
  if (!f || !target) return DS_ERR_ARG;
  const size_t bytes = (size_t)f->cfg.width * f->cfg.height * 3 * sizeof(float);
  DS_CUDA(cudaMemcpyAsync(f->target, target, bytes, cudaMemcpyDefault, (cudaStream_t)stream));
  f->have_target = true;
  return DS_OK;
}

int ds_fitter_set_camera(ds_fitter* f, const float pv[16], const float cam_pos[3],
                         ds_stream stream) {
  if (!f || !pv || !cam_pos) return DS_ERR_ARG;
  ds::Camera c;
  for (int k = 0; k < 16; ++k) c.pv[k] = pv[k];
  for (int k = 0; k < 3; ++k) c.cam[k] = cam_pos[k];
  c.pad = 0.f;
  DS_CUDA(cudaMemcpyAsync(f->cam_dev, &c, sizeof(c), cudaMemcpyHostToDevice, (cudaStream_t)stream));
  // cudaMemcpyAsync from pageable memory returns after staging the source, so
  // the local may go out of scope.
  f->have_camera = true;
  return DS_OK;
}

int ds_fitter_step(ds_fitter* f, int n_steps, ds_stream stream) {
  if (!f || n_steps < 0) return DS_ERR_ARG;
  if (!f->have_target || !f->have_camera) return DS_ERR_STATE;
  cudaStream_t s = (cudaStream_t)stream;
  if (f->cfg.use_graph && !f->exec) {
    DS_CUDA(cudaStreamBeginCapture(f->capture_stream, cudaStreamCaptureModeThreadLocal));
    int st = ds::fitter_enqueue(f, f->capture_stream);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(f->capture_stream, &g);
    if (st != DS_OK) {
      if (g) cudaGraphDestroy(g);
      return st;
    }
    DS_CUDA(e);
    f->graph = g;
    DS_CUDA(cudaGraphInstantiate(&f->exec, f->graph, 0));
  }
  if (n_steps > 0) DS_TRY(ds::refresh_render_copy(f, s));
  for (int k = 0; k < n_steps; ++k) {
    if (f->exec) {
      DS_CUDA(cudaGraphLaunch(f->exec, s));
    } else {
      DS_TRY(ds::fitter_enqueue(f, s));
    }
    ++f->host_steps;
  }
  return DS_OK;
}

int ds_fitter_loss(ds_fitter* f, float* loss, ds_stream stream) {
  if (!f || !loss) return DS_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  DS_CUDA(cudaMemcpyAsync(loss, &f->rb.scalars->loss, sizeof(float), cudaMemcpyDeviceToHost, s));
  DS_CUDA(cudaStreamSynchronize(s));
  return DS_OK;
}

int ds_fitter_output(ds_fitter* f, float** image) {
  if (!f || !image) return DS_ERR_ARG;
  *image = f->image;
  return DS_OK;
}

int ds_fitter_step_count(ds_fitter* f, int* out) {
  if (!f || !out) return DS_ERR_ARG;
  *out = f->host_steps;
  return DS_OK;
}

int ds_fitter_status(ds_fitter* f, uint32_t* flags) {
  if (!f || !flags) return DS_ERR_ARG;
  DS_CUDA(cudaDeviceSynchronize());
  uint32_t st = 0, zero = 0;
  DS_CUDA(cudaMemcpy(&st, &f->rb.scalars->status, sizeof(uint32_t), cudaMemcpyDeviceToHost));
  DS_CUDA(cudaMemcpy(&f->rb.scalars->status, &zero, sizeof(uint32_t), cudaMemcpyHostToDevice));
  *flags = st;
  return (st & ds::kStatusIsectOverflow) ? DS_ERR_ISECT_OVERFLOW : DS_OK;
}

int ds_fitter_profile_step(ds_fitter* f, float* stage_ms, int n_stages, ds_stream stream) {
  if (!f || !stage_ms || n_stages < 7) return DS_ERR_ARG;
  if (!f->have_target || !f->have_camera) return DS_ERR_STATE;
  cudaStream_t s = (cudaStream_t)stream;
  cudaEvent_t ev[8];
  DS_TRY(ds::refresh_render_copy(f, s));
  for (int k = 0; k < 8; ++k) DS_CUDA(cudaEventCreate(&ev[k]));
  int st = ds::fitter_enqueue(f, s, ev);
  if (st == DS_OK) st = ds::cuda_status(cudaEventSynchronize(ev[7]));
  if (st == DS_OK) {
    for (int k = 0; k < 7; ++k) {
      float ms = 0.f;
      cudaEventElapsedTime(&ms, ev[k], ev[k + 1]);
      stage_ms[k] = ms;
    }
    ++f->host_steps;
  }
  for (int k = 0; k < 8; ++k) cudaEventDestroy(ev[k]);
  return st;
}

int ds_fitter_counters(ds_fitter* f, uint64_t* out, int n) {
  if (!f || !out || n < 3) return DS_ERR_ARG;
  DS_CUDA(cudaDeviceSynchronize());
  ds::DevScalars sc;
  DS_CUDA(cudaMemcpy(&sc, f->rb.scalars, sizeof(sc), cudaMemcpyDeviceToHost));
  out[0] = sc.n_isects_raw;
  out[1] = sc.visible;
  out[2] = sc.step;
  return DS_OK;
}

int ds_fitter_pair_stats(ds_fitter* f, uint64_t* out, int n, ds_stream stream) {
  if (!f || !out || n < 2) return DS_ERR_ARG;
  if (f->host_steps == 0) return DS_ERR_STATE;
  cudaStream_t s = (cudaStream_t)stream;
  DS_TRY(ds::raster_composite_count(f->rb, f->image, s));
  DS_CUDA(cudaStreamSynchronize(s));
  unsigned long long p[2];
  DS_CUDA(cudaMemcpy(p, f->rb.scalars->pairs, sizeof(p), cudaMemcpyDeviceToHost));
  out[0] = p[0];
  out[1] = p[1];
  return DS_OK;
}

// Test hook: a fitter that also writes the Gaussian3D gradients of each step.
int ds_fitter_create_with_grads(const ds_fitter_config* cfg, ds_fitter** out) {
  return ds_fitter_create_impl(cfg, 1, out);
}

int ds_fitter_grads(ds_fitter* f, ds_gaussian3d* out) {
  if (!f || !out) return DS_ERR_ARG;
  if (!f->g_mem) return DS_ERR_STATE;
  *out = f->G;
  return DS_OK;
}

int ds_fitter_moments(ds_fitter* f, ds_gaussian3d* m, ds_gaussian3d* v) {
  if (!f || !m || !v) return DS_ERR_ARG;
  if (f->cfg.storage != DS_STORAGE_FP32) return DS_ERR_STATE;
  *m = f->M;
  *v = f->V;
  return DS_OK;
}

}  // extern "C"
