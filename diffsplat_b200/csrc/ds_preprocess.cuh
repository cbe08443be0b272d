// Per-splat preprocess shared by the fused fitter and the forward-only
// renderer: activation (src/layers/gauss_activ_layer.cu:37-170) and
// projection (src/layers/persp_project_layer.cu:40-149) fused with the tile
// rectangle (src/layers/tile_rasterize_layer.cu:52-144) and the compositing
// record, one thread per splat; Splat3D / Splat2D never reach HBM.  Also the
// SoA views of the FP32 / BF16 storage modes.
#pragma once
#include <float.h>
#include <math.h>

#include "ds_common.cuh"
#include "ds_internal.h"

namespace ds {

namespace {

constexpr int kPreThreads = 256;

struct Camera {
  float pv[16];
  float cam[3];
  float pad;
};

// Parameter SoA in a storage type T: FP32 (the masters themselves) or BF16
// (the render copy and Adam moments of the BF16 storage mode).  Field order
// and layout are those of ds_gaussian3d.
template <typename T>
struct Soa {
  T *pos_x, *pos_y, *pos_z;
  T *scale_x, *scale_y, *scale_z;
  T *rot_w, *rot_x, *rot_y, *rot_z;
  T *sh_dc_r, *sh_dc_g, *sh_dc_b;
  T *sh_rest_r, *sh_rest_g, *sh_rest_b;
  T *logit_opacity;
  int count, sh_num_bands;
};

Soa<float> soa_of(const ds_gaussian3d& g) {
  Soa<float> s;
  s.pos_x = g.pos_x, s.pos_y = g.pos_y, s.pos_z = g.pos_z;
  s.scale_x = g.scale_x, s.scale_y = g.scale_y, s.scale_z = g.scale_z;
  s.rot_w = g.rot_w, s.rot_x = g.rot_x, s.rot_y = g.rot_y, s.rot_z = g.rot_z;
  s.sh_dc_r = g.sh_dc_r, s.sh_dc_g = g.sh_dc_g, s.sh_dc_b = g.sh_dc_b;
  s.sh_rest_r = g.sh_rest_r, s.sh_rest_g = g.sh_rest_g, s.sh_rest_b = g.sh_rest_b;
  s.logit_opacity = g.logit_opacity;
  s.count = g.count, s.sh_num_bands = g.sh_num_bands;
  return s;
}

// Preprocess of one step: positions from the FP32 masters P, every other
// attribute from R (P itself in FP32 storage, the BF16 render copy otherwise).
//
// Batch mode (kBatch): splat i belongs to instance inst_of_splat[i], whose
// camera is camp[inst] and whose image and tile grid (TS-pixel tiles) are
// geom[inst]; W, H, ntx, nty are then ignored.
template <typename T, int TS = kTile, bool kBatch = false>
__global__ void __launch_bounds__(kPreThreads)
    fit_preprocess_kernel(ds_gaussian3d P, Soa<T> R, int degree, const Camera* __restrict__ camp,
                          int W, int H, int ntx, int nty, float4* __restrict__ ra,
                          float4* __restrict__ rb, float4* __restrict__ rc,
                          float* __restrict__ ridet, ushort4* __restrict__ rect,
                          uint32_t* __restrict__ counts, uint32_t* __restrict__ depth_keys,
                          DevScalars* __restrict__ sc,
                          const uint16_t* __restrict__ inst_of_splat = nullptr,
                          const InstGeom* __restrict__ geom = nullptr) {
  pdl_wait();
  __shared__ Mat4 sP;
  __shared__ float sCam[3];
  if (!kBatch) {
    if (threadIdx.x < 16) sP.m[threadIdx.x] = camp->pv[threadIdx.x];
    if (threadIdx.x < 3) sCam[threadIdx.x] = camp->cam[threadIdx.x];
  }
  __syncthreads();
  const int n = P.count;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  bool vis = false;
  if (i < n) {
    const Camera* cam_i = camp;
    if (kBatch) {
      const int inst = inst_of_splat[i];
      const InstGeom g = geom[inst];
      cam_i = camp + inst;
      W = g.width, H = g.height, ntx = g.ntx, nty = g.nty;
    }
    const Mat4& PV = kBatch ? *reinterpret_cast<const Mat4*>(cam_i->pv) : sP;
    const float* eye = kBatch ? cam_i->cam : sCam;
    const float px = P.pos_x[i], py = P.pos_y[i], pz = P.pos_z[i];
    float clip_x, clip_y, clip_z, clip_w;
    project_jacobian(PV, px, py, pz, clip_x, clip_y, clip_z, clip_w);
    TileRect r;
    float ndc_x = 0.f, ndc_y = 0.f;
    Cov2 c2 = {0.f, 0.f, 0.f};
    if (clip_w > 0.f) {
      UnitQuat q = unit_quat(ldv(R.rot_w[i]), ldv(R.rot_x[i]), ldv(R.rot_y[i]), ldv(R.rot_z[i]));
      Rot3 Rm = rot_from_quat(q.w, q.x, q.y, q.z);
      Cov3 c3 = cov3_from(Rm, expf(ldv(R.scale_x[i])), expf(ldv(R.scale_y[i])),
                          expf(ldv(R.scale_z[i])));
      const float inv_w = 1.f / clip_w;
      const float inv_w2 = inv_w * inv_w;
      ndc_x = clip_x * inv_w;
      ndc_y = clip_y * inv_w;
      const float ndc_z = clip_z * inv_w;
      Jac2 J = jacobian(PV, clip_x, clip_y, clip_w, inv_w2);
      c2 = cov2_from(J, c3.xx, c3.xy, c3.xz, c3.yy, c3.yz, c3.zz);
      vis = tile_rect<TS>(ndc_x, ndc_y, ndc_z, c2.xx, c2.xy, c2.yy, W, H, ntx, nty, r);
      if (vis) {
        float3 v = dir_to_camera(eye[0], eye[1], eye[2], px, py, pz);
        const T* no = nullptr;
        const float cr = clamp01(
            sh_channel(ldv(R.sh_dc_r[i]), degree > 0 ? R.sh_rest_r + i : no, n, degree, v) + 0.5f);
        const float cg = clamp01(
            sh_channel(ldv(R.sh_dc_g[i]), degree > 0 ? R.sh_rest_g + i : no, n, degree, v) + 0.5f);
        const float cb = clamp01(
            sh_channel(ldv(R.sh_dc_b[i]), degree > 0 ? R.sh_rest_b + i : no, n, degree, v) + 0.5f);
        const float op = 1.f / (1.f + expf(-ldv(R.logit_opacity[i])));
        Record rec = make_record(ndc_x, ndc_y, c2.xx, c2.xy, c2.yy, cr, cg, cb, op);
        ra[i] = rec.a;
        rb[i] = rec.b;
        rc[i] = rec.c;
        ridet[i] = rec.idet;
        rect[i] = make_ushort4(r.x0, r.x1, r.y0, r.y1);
        counts[i] = (uint32_t)((r.x1 - r.x0 + 1) * (r.y1 - r.y0 + 1));
        depth_keys[i] = depth_bits(ndc_z);
      }
    }
    if (!vis) {
      counts[i] = 0u;
      depth_keys[i] = 0xffffffffu;
    }
  }
  unsigned m = __ballot_sync(0xffffffffu, vis);
  if ((threadIdx.x & 31) == 0 && m) atomicAdd(&sc->visible, (uint32_t)__popc(m));
}

// Render copy of the BF16 storage mode from the FP32 masters (whole SoA,
// round to nearest).
__global__ void __launch_bounds__(kPreThreads)
    to_bf16_kernel(const float* __restrict__ src, __nv_bfloat16* __restrict__ dst, size_t n) {
  for (size_t k = blockIdx.x * (size_t)kPreThreads + threadIdx.x; k < n;
       k += (size_t)gridDim.x * kPreThreads)
    dst[k] = __float2bfloat16_rn(src[k]);
}

// Lays out one SoA over a single allocation (ds_gaussian3d field order).
template <typename T>
void carve_soa(T* base, int n, int bands, Soa<T>& g) {
  T** f[14] = {&g.pos_x,   &g.pos_y,   &g.pos_z,   &g.scale_x, &g.scale_y,
               &g.scale_z, &g.rot_w,   &g.rot_x,   &g.rot_y,   &g.rot_z,
               &g.sh_dc_r, &g.sh_dc_g, &g.sh_dc_b, &g.logit_opacity};
  size_t off = 0;
  for (int k = 0; k < 14; ++k) {
    *f[k] = base + off;
    off += (size_t)n;
  }
  if (bands > 0) {
    g.sh_rest_r = base + off;
    off += (size_t)n * bands;
    g.sh_rest_g = base + off;
    off += (size_t)n * bands;
    g.sh_rest_b = base + off;
  } else {
    g.sh_rest_r = g.sh_rest_g = g.sh_rest_b = nullptr;
  }
  g.count = n;
  g.sh_num_bands = bands;
}

// Lays out one ds_gaussian3d view over a single allocation.
void carve(float* base, int n, int bands, ds_gaussian3d& g) {
  Soa<float> t;
  carve_soa(base, n, bands, t);
  g.pos_x = t.pos_x, g.pos_y = t.pos_y, g.pos_z = t.pos_z;
  g.scale_x = t.scale_x, g.scale_y = t.scale_y, g.scale_z = t.scale_z;
  g.rot_w = t.rot_w, g.rot_x = t.rot_x, g.rot_y = t.rot_y, g.rot_z = t.rot_z;
  g.sh_dc_r = t.sh_dc_r, g.sh_dc_g = t.sh_dc_g, g.sh_dc_b = t.sh_dc_b;
  g.sh_rest_r = t.sh_rest_r, g.sh_rest_g = t.sh_rest_g, g.sh_rest_b = t.sh_rest_b;
  g.logit_opacity = t.logit_opacity;
  g.count = n;
  g.sh_num_bands = bands;
}

}  // namespace

}  // namespace ds
