// Reference harness: wires the REFERENCE's own layers (compiled from its
// sources, see oracle/Makefile) exactly like tests/grad_check.cu:72-132 and
// ImageFitter::initLayers (src/pipelines/image_fitter.cpp:63-101), and exposes
// them through a small C ABI for the parity tests and bench.py's reference arm.
// TEST INFRASTRUCTURE: nothing here is part of the product.
//
// The rasterizer's sorted keys / ids / ranges are private members of
// TileRasterizeLayer; the harness reads them by making the members visible in
// this translation unit only (the class layout is unchanged).
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <vector>

#include "cuda/cuda_check.h"
#include "layers/gauss_activ_layer.h"
#include "layers/mse_loss_layer.h"
#include "layers/persp_project_layer.h"
#define private public
#include "layers/tile_rasterize_layer.h"
#undef private
#include "optimizers/gaussian3d_adam.h"
#include "pipelines/pipeline.h"
#include "types/gaussian3d.h"
#include "utils/gaussian3d_io.h"

namespace {

struct RefScene {
  int W = 0, H = 0, n = 0, degree = 0, bands = 0;
  Gaussian3DParams params;
  CudaBuffer<float> target;
  GaussActivLayer atv;
  PerspProjectLayer psp;
  TileRasterizeLayer ras;
  MSELossLayer mse;
  Pipeline pipeline;
  Adam adam;
};

// host params: field-major float [14 + 3K][n] in the order pos xyz, log-scale
// xyz, quat wxyz, sh_dc rgb, logit, sh_rest r (K rows), g (K rows), b (K rows).
void upload(RefScene& s, const float* hp) {
  const int n = s.n, K = s.bands;
  std::vector<Gaussian3D> g(n);
  for (int i = 0; i < n; ++i) {
    auto p = [&](int f) { return hp[(size_t)f * n + i]; };
    Gaussian3D& q = g[i];
    q.pos_x = p(0);
    q.pos_y = p(1);
    q.pos_z = p(2);
    q.scale_x = p(3);
    q.scale_y = p(4);
    q.scale_z = p(5);
    q.rot_w = p(6);
    q.rot_x = p(7);
    q.rot_y = p(8);
    q.rot_z = p(9);
    q.sh_dc_r = p(10);
    q.sh_dc_g = p(11);
    q.sh_dc_b = p(12);
    q.logit_opacity = p(13);
    for (int c = 0; c < 3; ++c)
      for (int b = 0; b < K; ++b) q.sh_rest[c * K + b] = p(14 + c * K + b);
  }
  uploadGaussians(s.params, g, s.degree);
}

}  // namespace

extern "C" {

// lrs: pos, scale, rot, sh_dc, sh_rest, opacity (Gaussian3DAdamConfig order).
void* ref_create(int W, int H, int n, int degree, const float* host_params,
                 const float* host_target, const float pv[16], const float cam[3],
                 const float lrs[6]) {
  RefScene* s = new RefScene();
  s->W = W;
  s->H = H;
  s->n = n;
  s->degree = degree;
  s->bands = sh_degree_to_bands(degree);
  upload(*s, host_params);
  s->target.allocate((size_t)W * H * 3);
  CUDA_CHECK(cudaMemcpy(s->target.ptr, host_target, (size_t)W * H * 3 * sizeof(float),
                        cudaMemcpyHostToDevice));
  s->atv.setSHDegree(degree);
  s->atv.allocate(n);
  s->psp.allocate(n);
  s->ras.allocate(W, H, n);
  s->mse.allocate(W, H);
  s->atv.allocateGrad(n);
  s->psp.allocateGrad(n);
  s->ras.allocateGrad(n);
  glm::mat4 view(1.f), proj;
  std::memcpy(glm::value_ptr(proj), pv, 16 * sizeof(float));
  s->psp.setCamera(view, proj);
  s->atv.setCameraPosition({cam[0], cam[1], cam[2]});
  s->atv.setInput(&s->params);
  s->psp.setInput(&s->atv.getOutput());
  s->ras.setInput(&s->psp.getOutput());
  s->mse.setInput(s->ras.getOutput());
  s->mse.setTarget(s->target.ptr);
  s->ras.setGradOutput(&s->mse.getGradInput());
  s->psp.setGradOutput(&s->ras.getGradInput());
  s->atv.setGradOutput(&s->psp.getGradInput());
  s->pipeline.add(&s->atv);
  s->pipeline.add(&s->psp);
  s->pipeline.add(&s->ras);
  s->pipeline.add(&s->mse);
  Gaussian3DAdamConfig cfg;
  cfg.lr_pos = lrs[0];
  cfg.lr_scale = lrs[1];
  cfg.lr_rot = lrs[2];
  cfg.lr_sh_dc = lrs[3];
  cfg.lr_sh_rest = lrs[4];
  cfg.lr_opacity = lrs[5];
  s->adam.init();
  registerGaussian3DGroups(s->adam, s->params, s->atv.getGradInput(), cfg);
  CUDA_CHECK(cudaDeviceSynchronize());
  return s;
}

void ref_destroy(void* h) { delete (RefScene*)h; }

// Overwrites the parameters in place (Adam state untouched).
void ref_set_params(void* h, const float* host_params) {
  RefScene* s = (RefScene*)h;
  const int n = s->n, K = s->bands;
  float* dst[14] = {s->params.pos_x,   s->params.pos_y,   s->params.pos_z,   s->params.scale_x,
                    s->params.scale_y, s->params.scale_z, s->params.rot_w,   s->params.rot_x,
                    s->params.rot_y,   s->params.rot_z,   s->params.sh_dc_r, s->params.sh_dc_g,
                    s->params.sh_dc_b, s->params.logit_opacity};
  for (int f = 0; f < 14; ++f)
    cudaMemcpy(dst[f], host_params + (size_t)f * n, n * sizeof(float), cudaMemcpyHostToDevice);
  if (K > 0) {
    float* rest[3] = {s->params.sh_rest_r, s->params.sh_rest_g, s->params.sh_rest_b};
    for (int c = 0; c < 3; ++c)
      cudaMemcpy(rest[c], host_params + (size_t)(14 + c * K) * n, (size_t)K * n * sizeof(float),
                 cudaMemcpyHostToDevice);
  }
  cudaDeviceSynchronize();
}

void ref_zero_grad(void* h) { ((RefScene*)h)->pipeline.zeroGrad(); }
void ref_forward(void* h) { ((RefScene*)h)->pipeline.forward(); }
void ref_backward(void* h) { ((RefScene*)h)->pipeline.backward(); }
void ref_adam_step(void* h) { ((RefScene*)h)->adam.step(); }

// One ImageFitter::step (src/pipelines/image_fitter.cpp:103-112).
void ref_step(void* h) {
  RefScene* s = (RefScene*)h;
  s->pipeline.zeroGrad();
  s->pipeline.forward();
  s->pipeline.backward();
  s->adam.step();
}

float ref_loss(void* h) { return ((RefScene*)h)->mse.getLoss(); }
int ref_sync(void) { return (int)cudaDeviceSynchronize(); }

uint32_t ref_n_isects(void* h) {
  RefScene* s = (RefScene*)h;
  uint32_t n = 0;
  cudaMemcpy(&n, s->ras.d_n_isects.ptr, 4, cudaMemcpyDeviceToHost);
  return n;
}

uint32_t ref_visible(void* h) { return ((RefScene*)h)->ras.getVisibleCount(); }

// what: 0 keys u64[n_isects], 1 ids u32[n_isects], 2 ranges int2[tiles],
//       3 image f32[H*W*3], 4 alphas f32[H*W], 5 last_ids i32[H*W],
//       6 Gaussian3D grads f32[14+3K][n], 7 params f32[14+3K][n],
//       8 Splat2D (projection output) f32[10][n], 9 Splat2D grads f32[10][n],
//       10 Splat3D (activation output) f32[13][n], 11 Splat3D grads f32[13][n]
int ref_download(void* h, int what, void* host) {
  RefScene* s = (RefScene*)h;
  cudaDeviceSynchronize();
  const size_t n = s->n, px = (size_t)s->W * s->H;
  const int K = s->bands;
  auto soa = [&](std::vector<CudaBuffer<float>*> f, size_t rows_each) {
    float* out = (float*)host;
    size_t off = 0;
    for (auto* b : f) {
      cudaMemcpy(out + off, b->ptr, rows_each * n * sizeof(float), cudaMemcpyDeviceToHost);
      off += rows_each * n;
    }
  };
  switch (what) {
    case 0: {
      uint32_t m = ref_n_isects(h);
      cudaMemcpy(host, s->ras.d_isect_ids_sorted.ptr, (size_t)m * 8, cudaMemcpyDeviceToHost);
      return 0;
    }
    case 1: {
      uint32_t m = ref_n_isects(h);
      cudaMemcpy(host, s->ras.d_flatten_ids.ptr, (size_t)m * 4, cudaMemcpyDeviceToHost);
      return 0;
    }
    case 2:
      cudaMemcpy(host, s->ras.d_tile_offsets.ptr,
                 (size_t)s->ras.num_tiles_x * s->ras.num_tiles_y * 8, cudaMemcpyDeviceToHost);
      return 0;
    case 3:
      cudaMemcpy(host, s->ras.getOutput().ptr, px * 3 * 4, cudaMemcpyDeviceToHost);
      return 0;
    case 4:
      cudaMemcpy(host, s->ras.d_render_alphas.ptr, px * 4, cudaMemcpyDeviceToHost);
      return 0;
    case 5:
      cudaMemcpy(host, s->ras.d_last_ids.ptr, px * 4, cudaMemcpyDeviceToHost);
      return 0;
    case 6:
    case 7: {
      if (what == 6) {
        auto& g = s->atv.getGradInput();
        soa({&g.grad_pos_x, &g.grad_pos_y, &g.grad_pos_z, &g.grad_scale_x, &g.grad_scale_y,
             &g.grad_scale_z, &g.grad_rot_w, &g.grad_rot_x, &g.grad_rot_y, &g.grad_rot_z,
             &g.grad_sh_dc_r, &g.grad_sh_dc_g, &g.grad_sh_dc_b, &g.grad_logit_opacity},
            1);
        if (K > 0) {
          float* out = (float*)host + 14 * n;
          cudaMemcpy(out, g.grad_sh_rest_r.ptr, K * n * 4, cudaMemcpyDeviceToHost);
          cudaMemcpy(out + K * n, g.grad_sh_rest_g.ptr, K * n * 4, cudaMemcpyDeviceToHost);
          cudaMemcpy(out + 2 * K * n, g.grad_sh_rest_b.ptr, K * n * 4, cudaMemcpyDeviceToHost);
        }
      } else {
        auto& g = s->params;
        soa({&g.pos_x, &g.pos_y, &g.pos_z, &g.scale_x, &g.scale_y, &g.scale_z, &g.rot_w,
             &g.rot_x, &g.rot_y, &g.rot_z, &g.sh_dc_r, &g.sh_dc_g, &g.sh_dc_b, &g.logit_opacity},
            1);
        if (K > 0) {
          float* out = (float*)host + 14 * n;
          cudaMemcpy(out, g.sh_rest_r.ptr, K * n * 4, cudaMemcpyDeviceToHost);
          cudaMemcpy(out + K * n, g.sh_rest_g.ptr, K * n * 4, cudaMemcpyDeviceToHost);
          cudaMemcpy(out + 2 * K * n, g.sh_rest_b.ptr, K * n * 4, cudaMemcpyDeviceToHost);
        }
      }
      return 0;
    }
    case 8:
      soa(s->psp.getOutput().fields(), 1);
      return 0;
    case 9:
      soa(s->ras.getGradInput().fields(), 1);
      return 0;
    case 10:
      soa(s->atv.getOutput().fields(), 1);
      return 0;
    case 11:
      soa(s->psp.getGradInput().fields(), 1);
      return 0;
    default:
      return -1;
  }
}

}  // extern "C"
