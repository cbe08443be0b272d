// Batched fitting of many independent instances of uneven image size and
// splat count in one training step: one launch per stage over all instances,
// captured once into a CUDA graph.  No reference counterpart (the reference
// steps one ImageFitter at a time, src/pipelines/image_fitter.cpp:103-112).
//
// Layout: the instances' splats are concatenated into one parameter SoA
// (instance k owns splats [first_k, first_k + n_k) of every row), their tile
// grids into one batch-wide tile index (instance k's tiles start at
// tile_off_k) and their images into one pixel array.  inst_of_splat and
// tile_inst map splats and tiles back to instances; InstGeom holds each
// instance's image, grid and offsets; every instance has its own camera.
// Sorting by batch-wide tile id groups each tile's pairs exactly as in a
// single fitter, so the stages are those of ds_fitter.cu with per-splat and
// per-tile geometry lookups; the composite CTA schedule (longest list first)
// balances the load across instances.  Per-instance losses are the ordered
// sums of their tiles' partials (deterministic).
#include <float.h>
#include <math.h>

#include <algorithm>
#include <new>
#include <vector>

#include "ds_common.cuh"
#include "ds_fitter_kernels.cuh"
#include "ds_internal.h"
#include "ds_preprocess.cuh"

namespace ds {
namespace {

// One warp per instance: sum of its tiles' loss partials in tile order.
__global__ void batch_loss_kernel(const float* __restrict__ partials,
                                  const InstGeom* __restrict__ geom, int instances,
                                  float* __restrict__ losses) {
  const int k = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (k >= instances) return;
  const InstGeom g = geom[k];
  const int tiles = g.ntx * g.nty;
  float s = 0.f;
  for (int t = lane; t < tiles; t += 32) s += partials[g.tile_off + t];
  s = warp_sum(s);
  if (lane == 0) losses[k] = s;
}

}  // namespace
}  // namespace ds

struct ds_batch {
  ds_batch_config cfg{};
  int instances = 0;
  int bands = 0;
  int total_splats = 0;
  int64_t total_pixels = 0;
  int total_tiles = 0;
  size_t floats = 0;  // per SoA (all instances)
  std::vector<ds::InstGeom> geom;
  float* params_mem = nullptr;
  void* m_mem = nullptr;
  void* v_mem = nullptr;
  __nv_bfloat16* render_mem = nullptr;
  ds_gaussian3d P{}, M{}, V{};
  ds::Soa<__nv_bfloat16> R16{}, M16{}, V16{};
  bool render_dirty = true;
  float* targets = nullptr;
  float* images = nullptr;
  float* losses = nullptr;
  uint16_t* inst_of_splat = nullptr;
  uint16_t* tile_inst = nullptr;
  ds::InstGeom* geom_dev = nullptr;
  ds::Camera* cams = nullptr;
  ds::HostStage cam_stage;
  ds::RasterBuffers rb;
  float2* bc_table = nullptr;
  float2* bc_cur = nullptr;
  int bc_len = 0;
  cudaStream_t capture_stream = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int host_steps = 0;
};

namespace ds {

template <typename T, int TS>
static void launch_batch_preprocess(ds_batch* b, const Soa<T>& R, cudaStream_t s) {
  RasterBuffers& rb = b->rb;
  const unsigned blocks = (unsigned)((b->total_splats + kPreThreads - 1) / kPreThreads);
  fit_preprocess_kernel<T, TS, true><<<blocks, kPreThreads, 0, s>>>(
      b->P, R, b->cfg.sh_degree, b->cams, 0, 0, 0, 0, rb.rec_a, rb.rec_b, rb.rec_c, rb.rec_idet,
      rb.rect, rb.counts, rb.depth_keys, rb.scalars, b->inst_of_splat, b->geom_dev);
}

template <typename T>
static void batch_preprocess(ds_batch* b, const Soa<T>& R, cudaStream_t s) {
  switch (b->cfg.tile_size) {
    case 8: launch_batch_preprocess<T, 8>(b, R, s); break;
    case 32: launch_batch_preprocess<T, 32>(b, R, s); break;
    default: launch_batch_preprocess<T, 16>(b, R, s); break;
  }
}

static int batch_enqueue(ds_batch* b, cudaStream_t s) {
  RasterBuffers& rb = b->rb;
  const int n = b->total_splats;
  step_begin_kernel<<<1, 1, 0, s>>>(rb.scalars, b->bc_table, b->bc_len, b->bc_cur);
  DS_CUDA(cudaGetLastError());
  const bool bf16 = b->cfg.storage == DS_STORAGE_BF16;
  if (bf16) batch_preprocess(b, b->R16, s);
  else batch_preprocess(b, soa_of(b->P), s);
  DS_CUDA(cudaGetLastError());
  DS_TRY(raster_build_lists(rb, n, s, nullptr, true));
  DS_TRY(raster_composite_forward(rb, b->images, b->targets, s));
  batch_loss_kernel<<<(b->instances * 32 + 255) / 256, 256, 0, s>>>(
      rb.loss_partials, b->geom_dev, b->instances, b->losses);
  DS_CUDA(cudaGetLastError());
  DS_TRY(raster_composite_backward(rb, b->images, nullptr, b->targets, s));
  DS_TRY(raster_reduce_long_grads(rb, n, s));
  Lrs lr{b->cfg.lr_pos, b->cfg.lr_scale, b->cfg.lr_rot, b->cfg.lr_sh_dc, b->cfg.lr_sh_rest,
         b->cfg.lr_opacity};
  AdamHyper h{b->cfg.beta1, b->cfg.beta2, b->cfg.epsilon};
  const int blocks = (n + kThreads - 1) / kThreads;
  const int exact = b->cfg.grad_mode == DS_GRAD_EXACT ? 1 : 0;
  ds_gaussian3d G = b->P;  // unused: keep_grads == 0
  if (bf16)
    fit_backward_adam_kernel<__nv_bfloat16, true><<<blocks, kThreads, 0, s>>>(
        b->P, b->R16, b->M16, b->V16, G, 0, exact, b->cfg.sh_degree, b->cams, rb.g2,
        grad_segments(rb), b->bc_cur, rb.scalars, lr, h, b->inst_of_splat);
  else
    fit_backward_adam_kernel<float, true><<<blocks, kThreads, 0, s>>>(
        b->P, soa_of(b->P), soa_of(b->M), soa_of(b->V), G, 0, exact, b->cfg.sh_degree, b->cams,
        rb.g2, grad_segments(rb), b->bc_cur, rb.scalars, lr, h, b->inst_of_splat);
  return cuda_status(cudaGetLastError());
}

static int batch_refresh(ds_batch* b, cudaStream_t s) {
  if (b->cfg.storage != DS_STORAGE_BF16 || !b->render_dirty) return DS_OK;
  const size_t blocks = std::min<size_t>((b->floats + kThreads - 1) / kThreads, 148 * 16);
  to_bf16_kernel<<<(unsigned)blocks, kThreads, 0, s>>>(b->params_mem, b->render_mem, b->floats);
  DS_CUDA(cudaGetLastError());
  b->render_dirty = false;
  return DS_OK;
}

}  // namespace ds

extern "C" {

int ds_batch_default_config(ds_batch_config* cfg) {
  if (!cfg) return DS_ERR_ARG;
  ds_fitter_config f;
  ds_fitter_default_config(&f);
  *cfg = ds_batch_config{};
  cfg->lr_pos = f.lr_pos;
  cfg->lr_scale = f.lr_scale;
  cfg->lr_rot = f.lr_rot;
  cfg->lr_sh_dc = f.lr_sh_dc;
  cfg->lr_sh_rest = f.lr_sh_rest;
  cfg->lr_opacity = f.lr_opacity;
  cfg->beta1 = f.beta1;
  cfg->beta2 = f.beta2;
  cfg->epsilon = f.epsilon;
  cfg->storage = DS_STORAGE_BF16;
  cfg->use_graph = 1;
  cfg->grad_mode = f.grad_mode;
  cfg->schedule = DS_SCHEDULE_LONGEST_FIRST;
  cfg->tile_size = 16;
  cfg->pixels_per_thread = 1;
  return DS_OK;
}

int ds_batch_destroy(ds_batch* b) {
  if (!b) return DS_ERR_ARG;
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  if (b->capture_stream) cudaStreamDestroy(b->capture_stream);
  ds::raster_free(b->rb);
  for (void* p : {(void*)b->params_mem, b->m_mem, b->v_mem, (void*)b->render_mem,
                  (void*)b->targets, (void*)b->images, (void*)b->losses, (void*)b->inst_of_splat,
                  (void*)b->tile_inst, (void*)b->geom_dev, (void*)b->cams, (void*)b->bc_table,
                  (void*)b->bc_cur})
    cudaFree(p);
  delete b;
  return DS_OK;
}

int ds_batch_create(const ds_batch_config* cfg, const ds_batch_instance* inst, ds_batch** out) {
  if (!cfg || !inst || !out) return DS_ERR_ARG;
  *out = nullptr;
  const int I = cfg->instances;
  if (I <= 0 || I > 65535 || cfg->sh_degree < 0 || cfg->sh_degree > 3) return DS_ERR_ARG;
  if (cfg->storage != DS_STORAGE_FP32 && cfg->storage != DS_STORAGE_BF16) return DS_ERR_ARG;
  if (cfg->grad_mode != DS_GRAD_REFERENCE && cfg->grad_mode != DS_GRAD_EXACT) return DS_ERR_ARG;
  if (cfg->schedule != DS_SCHEDULE_LONGEST_FIRST && cfg->schedule != DS_SCHEDULE_RASTER)
    return DS_ERR_ARG;
  const int TS = cfg->tile_size;
  if (TS != 8 && TS != 16 && TS != 32) return DS_ERR_ARG;
  if (cfg->pixels_per_thread != 1 && cfg->pixels_per_thread != 2) return DS_ERR_ARG;
  ds_batch* b = new (std::nothrow) ds_batch();
  if (!b) return DS_ERR_OOM;
  auto fail = [&](int code) {
    ds_batch_destroy(b);
    return code;
  };
  b->cfg = *cfg;
  b->instances = I;
  b->bands = ds::sh_bands(cfg->sh_degree);
  int64_t splats = 0, pixels = 0, tiles = 0;
  b->geom.resize(I);
  for (int k = 0; k < I; ++k) {
    const ds_batch_instance& d = inst[k];
    if (d.width <= 0 || d.height <= 0 || d.count <= 0) return fail(DS_ERR_ARG);
    ds::InstGeom& g = b->geom[k];
    g.width = d.width;
    g.height = d.height;
    g.ntx = (d.width + TS - 1) / TS;
    g.nty = (d.height + TS - 1) / TS;
    if (g.ntx > 65535 || g.nty > 65535) return fail(DS_ERR_ARG);
    g.tile_off = (int)tiles;
    g.pix_off = (int)pixels;
    g.splat_off = (int)splats;
    g.count = d.count;
    splats += d.count;
    pixels += (int64_t)d.width * d.height;
    tiles += (int64_t)g.ntx * g.nty;
  }
  if (splats > INT32_MAX / 2 || pixels > INT32_MAX / 4 || tiles > INT32_MAX / 2)
    return fail(DS_ERR_ARG);
  b->total_splats = (int)splats;
  b->total_pixels = pixels;
  b->total_tiles = (int)tiles;
  const int n = b->total_splats;
  b->floats = (size_t)n * (14 + 3 * b->bands);
  const bool bf16 = cfg->storage == DS_STORAGE_BF16;
  const size_t mom = b->floats * (bf16 ? 2 : 4);
  int st;
  if ((st = ds::cuda_status(ds::device_alloc(&b->params_mem, b->floats * 4)))) return fail(st);
  if ((st = ds::cuda_status(ds::device_alloc(&b->m_mem, mom)))) return fail(st);
  if ((st = ds::cuda_status(ds::device_alloc(&b->v_mem, mom)))) return fail(st);
  cudaMemset(b->params_mem, 0, b->floats * 4);
  cudaMemset(b->m_mem, 0, mom);
  cudaMemset(b->v_mem, 0, mom);
  ds::carve(b->params_mem, n, b->bands, b->P);
  if (bf16) {
    if ((st = ds::cuda_status(ds::device_alloc(&b->render_mem, b->floats * 2)))) return fail(st);
    cudaMemset(b->render_mem, 0, b->floats * 2);
    ds::carve_soa(b->render_mem, n, b->bands, b->R16);
    ds::carve_soa((__nv_bfloat16*)b->m_mem, n, b->bands, b->M16);
    ds::carve_soa((__nv_bfloat16*)b->v_mem, n, b->bands, b->V16);
  } else {
    ds::carve((float*)b->m_mem, n, b->bands, b->M);
    ds::carve((float*)b->v_mem, n, b->bands, b->V);
  }
  if ((st = ds::cuda_status(ds::device_alloc(&b->targets, (size_t)pixels * 12)))) return fail(st);
  if ((st = ds::cuda_status(ds::device_alloc(&b->images, (size_t)pixels * 12)))) return fail(st);
  if ((st = ds::cuda_status(ds::device_alloc(&b->losses, (size_t)I * 4)))) return fail(st);
  cudaMemset(b->targets, 0, (size_t)pixels * 12);
  cudaMemset(b->images, 0, (size_t)pixels * 12);
  cudaMemset(b->losses, 0, (size_t)I * 4);
  // splat -> instance, tile -> instance, geometry, cameras
  std::vector<uint16_t> sinst((size_t)n), tinst((size_t)tiles);
  for (int k = 0; k < I; ++k) {
    const ds::InstGeom& g = b->geom[k];
    std::fill(sinst.begin() + g.splat_off, sinst.begin() + g.splat_off + g.count, (uint16_t)k);
    std::fill(tinst.begin() + g.tile_off, tinst.begin() + g.tile_off + g.ntx * g.nty,
              (uint16_t)k);
  }
  if ((st = ds::cuda_status(ds::device_alloc(&b->inst_of_splat, sinst.size() * 2)))) return fail(st);
  if ((st = ds::cuda_status(ds::device_alloc(&b->tile_inst, tinst.size() * 2)))) return fail(st);
  if ((st = ds::cuda_status(ds::device_alloc(&b->geom_dev, (size_t)I * sizeof(ds::InstGeom)))))
    return fail(st);
  if ((st = ds::cuda_status(ds::device_alloc(&b->cams, (size_t)I * sizeof(ds::Camera))))) return fail(st);
  cudaMemcpy(b->inst_of_splat, sinst.data(), sinst.size() * 2, cudaMemcpyHostToDevice);
  cudaMemcpy(b->tile_inst, tinst.data(), tinst.size() * 2, cudaMemcpyHostToDevice);
  cudaMemcpy(b->geom_dev, b->geom.data(), (size_t)I * sizeof(ds::InstGeom),
             cudaMemcpyHostToDevice);
  cudaMemset(b->cams, 0, (size_t)I * sizeof(ds::Camera));
  if ((st = ds::raster_alloc_batch(b->rb, pixels, (int)tiles, TS, n, cfg->max_isects)))
    return fail(st);
  b->rb.grad_mode = cfg->grad_mode;
  b->rb.schedule = cfg->schedule;
  b->rb.ppt = cfg->pixels_per_thread;
  b->rb.ppt_bwd = cfg->pixels_per_thread;
  b->rb.inst_of_splat = b->inst_of_splat;
  b->rb.tile_inst = b->tile_inst;
  b->rb.geom = b->geom_dev;
  b->rb.instances = I;
  if ((st = ds::make_bc_table(cfg->beta1, cfg->beta2, &b->bc_table, &b->bc_len))) return fail(st);
  if ((st = ds::cuda_status(ds::device_alloc(&b->bc_cur, sizeof(float2))))) return fail(st);
  uint32_t nn = (uint32_t)n;
  cudaMemcpy(&b->rb.scalars->n_splats, &nn, sizeof(uint32_t), cudaMemcpyHostToDevice);
  if ((st = ds::cuda_status(cudaStreamCreateWithFlags(&b->capture_stream, cudaStreamNonBlocking))))
    return fail(st);
  if ((st = ds::cuda_status(cudaDeviceSynchronize()))) return fail(st);
  *out = b;
  return DS_OK;
}

int ds_batch_params(ds_batch* b, ds_gaussian3d* out) {
  if (!b || !out) return DS_ERR_ARG;
  *out = b->P;
  b->render_dirty = true;
  return DS_OK;
}

int ds_batch_instance_range(ds_batch* b, int k, int32_t* first_splat, int32_t* count) {
  if (!b || !first_splat || !count || k < 0 || k >= b->instances) return DS_ERR_ARG;
  *first_splat = b->geom[k].splat_off;
  *count = b->geom[k].count;
  return DS_OK;
}

int ds_batch_params_updated(ds_batch* b) {
  if (!b) return DS_ERR_ARG;
  b->render_dirty = true;
  return DS_OK;
}

int ds_batch_set_target(ds_batch* b, int k, const float* target, ds_stream stream) {
  if (!b || !target || k < 0 || k >= b->instances) return DS_ERR_ARG;
  const ds::InstGeom& g = b->geom[k];
  DS_CUDA(cudaMemcpyAsync(b->targets + (size_t)g.pix_off * 3, target,
                          (size_t)g.width * g.height * 12, cudaMemcpyDefault,
                          (cudaStream_t)stream));
  return DS_OK;
}

int ds_batch_set_camera(ds_batch* b, int k, const float pv[16], const float cam_pos[3],
                        ds_stream stream) {
  if (!b || !pv || !cam_pos || k < 0 || k >= b->instances) return DS_ERR_ARG;
  ds::Camera c;
  for (int q = 0; q < 16; ++q) c.pv[q] = pv[q];
  for (int q = 0; q < 3; ++q) c.cam[q] = cam_pos[q];
  c.pad = 0.f;
  DS_TRY(b->cam_stage.upload(b->cams + k, &c, sizeof(c), (cudaStream_t)stream));
  return DS_OK;
}

int ds_batch_step(ds_batch* b, int n_steps, ds_stream stream) {
  if (!b || n_steps < 0) return DS_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  if (b->cfg.use_graph && !b->exec) {
    DS_CUDA(cudaStreamBeginCapture(b->capture_stream, cudaStreamCaptureModeThreadLocal));
    int st = ds::batch_enqueue(b, b->capture_stream);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(b->capture_stream, &g);
    if (st != DS_OK) {
      if (g) cudaGraphDestroy(g);
      return st;
    }
    DS_CUDA(e);
    b->graph = g;
    DS_CUDA(cudaGraphInstantiate(&b->exec, b->graph, 0));
  }
  if (n_steps > 0) DS_TRY(ds::batch_refresh(b, s));
  for (int k = 0; k < n_steps; ++k) {
    if (b->exec) DS_CUDA(cudaGraphLaunch(b->exec, s));
    else DS_TRY(ds::batch_enqueue(b, s));
    ++b->host_steps;
  }
  return DS_OK;
}

int ds_batch_losses(ds_batch* b, float* losses, ds_stream stream) {
  if (!b || !losses) return DS_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  DS_CUDA(cudaMemcpyAsync(losses, b->losses, (size_t)b->instances * 4, cudaMemcpyDeviceToHost, s));
  DS_CUDA(cudaStreamSynchronize(s));
  return DS_OK;
}

int ds_batch_output(ds_batch* b, int k, float** image) {
  if (!b || !image || k < 0 || k >= b->instances) return DS_ERR_ARG;
  *image = b->images + (size_t)b->geom[k].pix_off * 3;
  return DS_OK;
}

int ds_batch_counters(ds_batch* b, uint64_t* out, int n) {
  if (!b || !out || n < 3) return DS_ERR_ARG;
  DS_CUDA(cudaDeviceSynchronize());
  ds::DevScalars sc;
  DS_CUDA(cudaMemcpy(&sc, b->rb.scalars, sizeof(sc), cudaMemcpyDeviceToHost));
  out[0] = sc.n_isects_raw;
  out[1] = sc.visible;
  out[2] = sc.step;
  return DS_OK;
}

int ds_batch_status(ds_batch* b, uint32_t* flags) {
  if (!b || !flags) return DS_ERR_ARG;
  DS_CUDA(cudaDeviceSynchronize());
  uint32_t st = 0, zero = 0;
  DS_CUDA(cudaMemcpy(&st, &b->rb.scalars->status, sizeof(uint32_t), cudaMemcpyDeviceToHost));
  DS_CUDA(cudaMemcpy(&b->rb.scalars->status, &zero, sizeof(uint32_t), cudaMemcpyHostToDevice));
  *flags = st;
  return ds::status_code(st);
}

}  // extern "C"
