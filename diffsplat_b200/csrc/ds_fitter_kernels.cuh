// Kernels of the fused training step shared by the single fitter
// (ds_fitter.cu) and the batched fitter (ds_batch.cu): step begin (Adam bias
// corrections), and per-splat projection backward -> activation backward ->
// Adam on every field.
#pragma once
#include <float.h>
#include <math.h>

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
  pdl_wait();
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
template <typename T, bool kBatch = false>
__global__ void __launch_bounds__(kThreads)
    fit_backward_adam_kernel(ds_gaussian3d P, Soa<T> R, Soa<T> M, Soa<T> V, ds_gaussian3d G,
                             int keep_grads, int exact, int degree, const Camera* __restrict__ camp,
                             const float* __restrict__ g2sum, GradSegments seg,
                             const float2* __restrict__ bcp,
                             const DevScalars* __restrict__ sc, Lrs lr, AdamHyper h,
                             const uint16_t* __restrict__ inst_of_splat = nullptr,
                             const uint32_t* __restrict__ visible = nullptr,
                             float* __restrict__ grad_accum = nullptr,
                             uint32_t* __restrict__ grad_count = nullptr) {
  pdl_wait();
  constexpr bool kBf16 = sizeof(T) == 2;
  __shared__ Mat4 sP;
  __shared__ float sCam[3];
  if (!kBatch) {
    if (threadIdx.x < 16) sP.m[threadIdx.x] = camp->pv[threadIdx.x];
    if (threadIdx.x < 3) sCam[threadIdx.x] = camp->cam[threadIdx.x];
  }
  __syncthreads();
  const int n = P.count;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const Camera* cam_i = kBatch ? camp + inst_of_splat[i] : camp;
  const Mat4& PV = kBatch ? *reinterpret_cast<const Mat4*>(cam_i->pv) : sP;
  const float* eye = kBatch ? cam_i->cam : sCam;
  const float2 bc = *bcp;
  const uint32_t step = kBf16 ? sc->step : 0u;

  // 1) Splat2D gradient = sum of this splat's per-tile records: summed here in
  // record order when it has at most kSerialRecords tiles, else read from the
  // long-segment reduction (segment_reduce_long_kernel).
  float g2[9];
  {
    const uint32_t c = seg.counts[i];
    unsigned long long s0 = 0, e0 = 0;
    if (c) {
      s0 = seg.start[i];
      e0 = s0 + c;
      if (e0 > seg.cap) e0 = seg.cap;
    }
    if (c > kSerialRecords) {
#pragma unroll
      for (int k = 0; k < 9; ++k) g2[k] = g2sum[(size_t)k * n + i];
    } else {
#pragma unroll
      for (int k = 0; k < 9; ++k) g2[k] = 0.f;
      if (e0 > s0) {
        // records of the tiles whose list ends (for compositing) before this
        // splat were not written: skip them
        const ushort4 rc = seg.rect[i];
        const uint32_t w = (uint32_t)(rc.y - rc.x + 1);
        uint32_t row0, pitch;
        seg_origin(seg, (uint32_t)i, rc, row0, pitch);
        const unsigned long long key = seg_key(seg, (uint32_t)i);
        uint32_t tx = 0, trow = row0;
        for (unsigned long long q = s0; q < e0; ++q) {
          if (key < seg.tile_bound[trow + tx]) {
            const float* r = seg.rec + q * 9;
#pragma unroll
            for (int k = 0; k < 9; ++k) g2[k] += r[k];
          }
          if (++tx == w) {
            tx = 0;
            trow += pitch;
          }
        }
      }
    }
  }
  // g2 = {color r, g, b, ndc x, ndc y, cov2 xx, xy, yy, opacity}
  if (grad_accum && visible[i] > 0u) {
    // densification statistics: norm of the NDC position gradient, steps visible
    grad_accum[i] += sqrtf(g2[3] * g2[3] + g2[4] * g2[4]);
    grad_count[i] += 1u;
  }

  // 2) projection backward (persp_project_layer.cu:173-267)
  const float px = P.pos_x[i], py = P.pos_y[i], pz = P.pos_z[i];
  const float rw = ldv(R.rot_w[i]), rx = ldv(R.rot_x[i]), ry = ldv(R.rot_y[i]),
              rz = ldv(R.rot_z[i]);
  const float lsx = ldv(R.scale_x[i]), lsy = ldv(R.scale_y[i]), lsz = ldv(R.scale_z[i]);
  float clip_x, clip_y, clip_z, clip_w;
  project_jacobian(PV, px, py, pz, clip_x, clip_y, clip_z, clip_w);
  float gpos[3] = {0.f, 0.f, 0.f};
  float gcov[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  float gcol[3] = {0.f, 0.f, 0.f};
  float gop = 0.f;
  if (clip_w > 0.f) {
    const float inv_w = 1.f / clip_w;
    const float inv_w2 = inv_w * inv_w;
    Jac2 J = jacobian(PV, clip_x, clip_y, clip_w, inv_w2);
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
      float3 e = jacobian_position_grad(PV, J, clip_w, dcxx, hdxy, dcyy, c3.xx, c3.xy, c3.xz,
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
  const float3 v = dir_to_camera(eye[0], eye[1], eye[2], px, py, pz);
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
  //    the render copy of every non-position field follows its master.  All
  //    loads of a group of fields are issued before its first store (the
  //    arrays could alias as far as the compiler knows), so they overlap.
  const float b1 = h.b1, b2 = h.b2, eps = h.eps, bc1 = bc.x, bc2 = bc.y;
  const uint32_t salt = step * 0x85ebca6bu;
  auto finish = [&](float* p, T* m, T* vv, T* r, int64_t k, uint32_t field, float pk, float mk,
                    float vk, float g, float l) {
    adam1(pk, mk, vk, g, l, b1, b2, eps, bc1, bc2);
    p[k] = pk;
    // one hash per element: its low 16 bits round m, its high 16 bits round v
    const uint32_t hs = mix32((uint32_t)k * 0x9e3779b1u ^ salt ^ field * 0xc2b2ae35u);
    store_moment(m + k, mk, hs);
    store_moment(vv + k, vk, hs >> 16);
    if (kBf16 && r) r[k] = __float2bfloat16_rn(pk);
  };
  {
    float* pf[14] = {P.pos_x,   P.pos_y,   P.pos_z,   P.scale_x, P.scale_y,
                     P.scale_z, P.rot_w,   P.rot_x,   P.rot_y,   P.rot_z,
                     P.sh_dc_r, P.sh_dc_g, P.sh_dc_b, P.logit_opacity};
    T* mf[14] = {M.pos_x,   M.pos_y,   M.pos_z,   M.scale_x, M.scale_y,
                 M.scale_z, M.rot_w,   M.rot_x,   M.rot_y,   M.rot_z,
                 M.sh_dc_r, M.sh_dc_g, M.sh_dc_b, M.logit_opacity};
    T* vf[14] = {V.pos_x,   V.pos_y,   V.pos_z,   V.scale_x, V.scale_y,
                 V.scale_z, V.rot_w,   V.rot_x,   V.rot_y,   V.rot_z,
                 V.sh_dc_r, V.sh_dc_g, V.sh_dc_b, V.logit_opacity};
    T* rf[14] = {nullptr,   nullptr,   nullptr,   R.scale_x, R.scale_y,
                 R.scale_z, R.rot_w,   R.rot_x,   R.rot_y,   R.rot_z,
                 R.sh_dc_r, R.sh_dc_g, R.sh_dc_b, R.logit_opacity};
    const float g[14] = {gpos[0], gpos[1], gpos[2], d[0],     d[1],     d[2],     d[3],
                         d[4],    d[5],    d[6],    dR * kC0, dG * kC0, dB * kC0, glogit};
    const float lf[14] = {lr.pos, lr.pos, lr.pos, lr.scale, lr.scale, lr.scale,  lr.rot,
                          lr.rot, lr.rot, lr.rot, lr.sh_dc, lr.sh_dc, lr.sh_dc, lr.opacity};
    float pp[14], mm[14], vv[14];
#pragma unroll
    for (int k = 0; k < 14; ++k) {
      pp[k] = pf[k][i];
      mm[k] = ldv(mf[k][i]);
      vv[k] = ldv(vf[k][i]);
    }
#pragma unroll
    for (int k = 0; k < 14; ++k)
      finish(pf[k], mf[k], vf[k], rf[k], i, (uint32_t)k, pp[k], mm[k], vv[k], g[k], lf[k]);
  }
  const int nb = P.sh_num_bands;
  const int nb_used = sh_bands(degree);
  if (nb > 0) {
    float* pr[3] = {P.sh_rest_r, P.sh_rest_g, P.sh_rest_b};
    T* mr[3] = {M.sh_rest_r, M.sh_rest_g, M.sh_rest_b};
    T* vr[3] = {V.sh_rest_r, V.sh_rest_g, V.sh_rest_b};
    T* rr[3] = {R.sh_rest_r, R.sh_rest_g, R.sh_rest_b};
    const float dc[3] = {dR, dG, dB};
    float cp[3], cm[3], cv[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      cp[c] = pr[c][i];
      cm[c] = ldv(mr[c][i]);
      cv[c] = ldv(vr[c][i]);
    }
    for (int b = 0; b < nb; ++b) {
      // band b + 1 is loaded before band b is stored
      float np[3] = {0.f, 0.f, 0.f}, nm[3] = {0.f, 0.f, 0.f}, nv[3] = {0.f, 0.f, 0.f};
      if (b + 1 < nb) {
        const int64_t k1 = (int64_t)(b + 1) * n + i;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          np[c] = pr[c][k1];
          nm[c] = ldv(mr[c][k1]);
          nv[c] = ldv(vr[c][k1]);
        }
      }
      const int64_t k = (int64_t)b * n + i;
      const float yb = b < nb_used ? y[b] : 0.f;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        finish(pr[c], mr[c], vr[c], rr[c], k, 16u + 3u * (uint32_t)b + (uint32_t)c, cp[c], cm[c],
               cv[c], dc[c] * yb, lr.sh_rest);
        cp[c] = np[c];
        cm[c] = nm[c];
        cv[c] = nv[c];
      }
    }
  }
}

// Bias-correction table on the device: bc_k(t) = 1 / (1 - powf(beta_k, t)),
// computed on the host like the reference (adam.cu:61-62), up to the step at
// which both corrections reach 1.0f (step_begin_kernel uses 1.0f past it).
inline int make_bc_table(float beta1, float beta2, float2** table, int* len) {
  std::vector<float2> tab;
  for (int t = 1; t <= kBcTableMax; ++t) {
    const float p1 = powf(beta1, (float)t), p2 = powf(beta2, (float)t);
    const float bc1 = 1.f / (1.f - p1), bc2 = 1.f / (1.f - p2);
    tab.push_back(make_float2(bc1, bc2));
    if (bc1 == 1.f && bc2 == 1.f) break;
  }
  *len = (int)tab.size();
  DS_CUDA(cudaMalloc(table, tab.size() * sizeof(float2)));
  DS_CUDA(cudaMemcpy(*table, tab.data(), tab.size() * sizeof(float2), cudaMemcpyHostToDevice));
  return DS_OK;
}

}  // namespace

}  // namespace ds
