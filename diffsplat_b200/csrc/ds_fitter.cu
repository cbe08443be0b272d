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
#include "ds_fitter_kernels.cuh"
#include "ds_preprocess.cuh"

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
  int capacity = 0;               // splats the raster buffers hold (densification room)
  float* grad_accum = nullptr;    // densification statistics [capacity]
  uint32_t* grad_count = nullptr;
  float* target = nullptr;
  float* image = nullptr;
  ds::RasterBuffers rb;
  ds::Camera* cam_dev = nullptr;
  ds::HostStage cam_stage;
  float2* bc_table = nullptr;
  float2* bc_cur = nullptr;
  int bc_len = 0;
  bool have_target = false, have_camera = false;
  cudaStream_t capture_stream = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int host_steps = 0;
  float* loss_host = nullptr;  // pinned slot of the loss read-back
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
  DS_CUDA(launch_pdl(step_begin_kernel, dim3(1), dim3(1), 0, s, rb.scalars, f->bc_table, f->bc_len,
                     f->bc_cur));
  const int blocks = (n + kThreads - 1) / kThreads;
  const bool bf16 = f->cfg.storage == DS_STORAGE_BF16;
  if (bf16)
    DS_CUDA(launch_pdl(fit_preprocess_kernel<__nv_bfloat16>, dim3(blocks), dim3(kThreads), 0, s,
                       f->P, f->R16, f->cfg.sh_degree, f->cam_dev, rb.width, rb.height, rb.ntx,
                       rb.nty, rb.rec_a, rb.rec_b, rb.rec_c, rb.rec_idet, rb.rect, rb.counts,
                       rb.depth_keys, rb.scalars, nullptr, nullptr));
  else
    DS_CUDA(launch_pdl(fit_preprocess_kernel<float>, dim3(blocks), dim3(kThreads), 0, s, f->P,
                       soa_of(f->P), f->cfg.sh_degree, f->cam_dev, rb.width, rb.height, rb.ntx,
                       rb.nty, rb.rec_a, rb.rec_b, rb.rec_c, rb.rec_idet, rb.rect, rb.counts,
                       rb.depth_keys, rb.scalars, nullptr, nullptr));
  if (ev) DS_CUDA(cudaEventRecord(ev[1], s));
  DS_TRY(raster_build_lists(rb, n, s, ev ? ev + 2 : nullptr, true));
  DS_TRY(raster_composite_forward(rb, f->image, f->target, s));
  if (ev) DS_CUDA(cudaEventRecord(ev[5], s));
  DS_TRY(raster_composite_backward(rb, f->image, nullptr, f->target, s));
  if (ev) DS_CUDA(cudaEventRecord(ev[6], s));
  DS_TRY(raster_reduce_long_grads(rb, n, s));
  Lrs lr{f->cfg.lr_pos, f->cfg.lr_scale, f->cfg.lr_rot, f->cfg.lr_sh_dc, f->cfg.lr_sh_rest,
         f->cfg.lr_opacity};
  AdamHyper h{f->cfg.beta1, f->cfg.beta2, f->cfg.epsilon};
  const int keep = f->g_mem ? 1 : 0, exact = f->cfg.grad_mode == DS_GRAD_EXACT ? 1 : 0;
  if (bf16)
    DS_CUDA(launch_pdl(fit_backward_adam_kernel<__nv_bfloat16>, dim3(blocks), dim3(kThreads), 0,
                       s, f->P, f->R16, f->M16, f->V16, f->G, keep, exact, f->cfg.sh_degree,
                       f->cam_dev, rb.g2, grad_segments(rb), f->bc_cur, rb.scalars, lr, h,
                       nullptr, rb.counts, f->grad_accum, f->grad_count));
  else
    DS_CUDA(launch_pdl(fit_backward_adam_kernel<float>, dim3(blocks), dim3(kThreads), 0, s, f->P,
                       soa_of(f->P), soa_of(f->M), soa_of(f->V), f->G, keep, exact,
                       f->cfg.sh_degree, f->cam_dev, rb.g2, grad_segments(rb), f->bc_cur,
                       rb.scalars, lr, h, nullptr, rb.counts, f->grad_accum, f->grad_count));
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
  cudaFree(f->grad_accum);
  cudaFree(f->grad_count);
  cudaFree(f->target);
  cudaFree(f->image);
  cudaFree(f->cam_dev);
  cudaFree(f->bc_table);
  cudaFree(f->bc_cur);
  if (f->loss_host) cudaFreeHost(f->loss_host);
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
  if ((st = ds::cuda_status(ds::device_alloc(&f->params_mem, f->floats * 4)))) return fail(st);
  if ((st = ds::cuda_status(ds::device_alloc(&f->m_mem, mom_bytes)))) return fail(st);
  if ((st = ds::cuda_status(ds::device_alloc(&f->v_mem, mom_bytes)))) return fail(st);
  cudaMemset(f->params_mem, 0, f->floats * 4);
  cudaMemset(f->m_mem, 0, mom_bytes);
  cudaMemset(f->v_mem, 0, mom_bytes);
  ds::carve(f->params_mem, n, f->bands, f->P);
  if (bf16) {
    if ((st = ds::cuda_status(ds::device_alloc(&f->render_mem, f->floats * 2)))) return fail(st);
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
    if ((st = ds::cuda_status(ds::device_alloc(&f->g_mem, f->floats * 4)))) return fail(st);
    cudaMemset(f->g_mem, 0, f->floats * 4);
    ds::carve(f->g_mem, n, f->bands, f->G);
  } else {
    f->G = f->P;  // never written (keep_grads == 0)
  }
  const size_t px = (size_t)cfg->width * cfg->height;
  if ((st = ds::cuda_status(ds::device_alloc(&f->target, px * 3 * 4)))) return fail(st);
  if ((st = ds::cuda_status(ds::device_alloc(&f->image, px * 3 * 4)))) return fail(st);
  cudaMemset(f->image, 0, px * 3 * 4);
  f->capacity = std::max(n, cfg->capacity);
  if ((st = ds::raster_alloc(f->rb, cfg->width, cfg->height, f->capacity, cfg->max_isects)))
    return fail(st);
  if (f->capacity > n) {
    if ((st = ds::cuda_status(ds::device_alloc(&f->grad_accum, (size_t)f->capacity * 4)))) return fail(st);
    if ((st = ds::cuda_status(ds::device_alloc(&f->grad_count, (size_t)f->capacity * 4)))) return fail(st);
    cudaMemset(f->grad_accum, 0, (size_t)f->capacity * 4);
    cudaMemset(f->grad_count, 0, (size_t)f->capacity * 4);
  }
  f->rb.grad_mode = cfg->grad_mode;
  f->rb.schedule = cfg->schedule;
  if ((st = ds::cuda_status(ds::device_alloc(&f->cam_dev, sizeof(ds::Camera))))) return fail(st);
  cudaMemset(f->cam_dev, 0, sizeof(ds::Camera));
  if ((st = ds::make_bc_table(cfg->beta1, cfg->beta2, &f->bc_table, &f->bc_len))) return fail(st);
  if ((st = ds::cuda_status(ds::device_alloc(&f->bc_cur, sizeof(float2))))) return fail(st);
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
  DS_TRY(f->cam_stage.upload(f->cam_dev, &c, sizeof(c), (cudaStream_t)stream));
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
  if (!f->loss_host) DS_CUDA(cudaHostAlloc((void**)&f->loss_host, sizeof(float), cudaHostAllocDefault));
  DS_CUDA(cudaMemcpyAsync(f->loss_host, &f->rb.scalars->loss, sizeof(float),
                          cudaMemcpyDeviceToHost, s));
  DS_CUDA(cudaStreamSynchronize(s));
  *loss = *f->loss_host;
  return DS_OK;
}

int ds_fitter_loss_device(ds_fitter* f, float** loss) {
  if (!f || !loss) return DS_ERR_ARG;
  *loss = &f->rb.scalars->loss;
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
  return ds::status_code(st);
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

int ds_fitter_download(ds_fitter* f, int what, void* host, int64_t bytes) {
  if (!f || !host || bytes < 0) return DS_ERR_ARG;
  if (f->host_steps == 0) return DS_ERR_STATE;
  return ds::raster_download(f->rb, f->cfg.count, what, host, bytes);
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

// ---- adaptive density control ------------------------------------------------
namespace ds {
namespace {

// Per splat: 0 pruned, 1 kept, 2 kept + clone, 3 split into two children.
__global__ void densify_decide_kernel(ds_gaussian3d P, const float* __restrict__ gsum,
                                      const uint32_t* __restrict__ gcnt, ds_densify_params dp,
                                      uint8_t* __restrict__ mode, uint32_t* __restrict__ emit) {
  const int n = P.count;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float op = 1.f / (1.f + expf(-P.logit_opacity[i]));
  uint8_t m = 1;
  if (op < dp.min_opacity) {
    m = 0;
  } else if (gcnt[i] > 0u && gsum[i] / (float)gcnt[i] >= dp.grad_threshold) {
    const float smax = expf(fmaxf(P.scale_x[i], fmaxf(P.scale_y[i], P.scale_z[i])));
    m = smax <= dp.scale_threshold ? 2 : 3;
  }
  mode[i] = m;
  emit[i] = m == 0 ? 0u : (m == 1 ? 1u : 2u);
}

// Standard normal deviate from two hash draws (Box-Muller).
__device__ __forceinline__ float gauss(uint32_t key) {
  const float u1 = ((mix32(key) >> 8) + 1u) * (1.f / 16777217.f);
  const float u2 = (mix32(key ^ 0x9e3779b9u) >> 8) * (1.f / 16777216.f);
  return sqrtf(-2.f * logf(u1)) * cosf(6.28318530718f * u2);
}

__global__ void densify_scatter_kernel(ds_gaussian3d P, ds_gaussian3d M, ds_gaussian3d V,
                                       const uint8_t* __restrict__ mode,
                                       const unsigned long long* __restrict__ offs,
                                       ds_gaussian3d Q, ds_gaussian3d MQ, ds_gaussian3d VQ,
                                       uint32_t seed) {
  const int n = P.count, nq = Q.count, nb = P.sh_num_bands;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || mode[i] == 0) return;
  const int dst = (int)offs[i];
  auto field = [](const ds_gaussian3d& g, int k) -> float* {
    switch (k) {
      case 0: return g.pos_x;
      case 1: return g.pos_y;
      case 2: return g.pos_z;
      case 3: return g.scale_x;
      case 4: return g.scale_y;
      case 5: return g.scale_z;
      case 6: return g.rot_w;
      case 7: return g.rot_x;
      case 8: return g.rot_y;
      case 9: return g.rot_z;
      case 10: return g.sh_dc_r;
      case 11: return g.sh_dc_g;
      case 12: return g.sh_dc_b;
      default: return g.logit_opacity;
    }
  };
  const uint8_t m = mode[i];
  const int copies = m == 1 ? 1 : 2;
  for (int c = 0; c < copies; ++c) {
    const int j = dst + c;
    const bool fresh = m == 3 || c == 1;  // new splats start from zero moments
    for (int k = 0; k < 14; ++k) {
      field(Q, k)[j] = field(P, k)[i];
      field(MQ, k)[j] = fresh ? 0.f : field(M, k)[i];
      field(VQ, k)[j] = fresh ? 0.f : field(V, k)[i];
    }
    for (int b = 0; b < nb; ++b) {
      const float* ps[3] = {P.sh_rest_r, P.sh_rest_g, P.sh_rest_b};
      float* qs[3] = {Q.sh_rest_r, Q.sh_rest_g, Q.sh_rest_b};
      const float* ms[3] = {M.sh_rest_r, M.sh_rest_g, M.sh_rest_b};
      float* mq[3] = {MQ.sh_rest_r, MQ.sh_rest_g, MQ.sh_rest_b};
      const float* vs[3] = {V.sh_rest_r, V.sh_rest_g, V.sh_rest_b};
      float* vq[3] = {VQ.sh_rest_r, VQ.sh_rest_g, VQ.sh_rest_b};
      for (int ch = 0; ch < 3; ++ch) {
        qs[ch][(int64_t)b * nq + j] = ps[ch][(int64_t)b * n + i];
        mq[ch][(int64_t)b * nq + j] = fresh ? 0.f : ms[ch][(int64_t)b * n + i];
        vq[ch][(int64_t)b * nq + j] = fresh ? 0.f : vs[ch][(int64_t)b * n + i];
      }
    }
    if (m == 3) {
      // child of a split: position drawn from the parent's Gaussian, scales / 1.6
      UnitQuat q = unit_quat(P.rot_w[i], P.rot_x[i], P.rot_y[i], P.rot_z[i]);
      Rot3 R = rot_from_quat(q.w, q.x, q.y, q.z);
      const uint32_t key = mix32(seed) ^ mix32((uint32_t)i * 2u + (uint32_t)c);
      const float sx = expf(P.scale_x[i]) * gauss(key * 3u + 0u);
      const float sy = expf(P.scale_y[i]) * gauss(key * 3u + 1u);
      const float sz = expf(P.scale_z[i]) * gauss(key * 3u + 2u);
      Q.pos_x[j] = P.pos_x[i] + R.r00 * sx + R.r01 * sy + R.r02 * sz;
      Q.pos_y[j] = P.pos_y[i] + R.r10 * sx + R.r11 * sy + R.r12 * sz;
      Q.pos_z[j] = P.pos_z[i] + R.r20 * sx + R.r21 * sy + R.r22 * sz;
      const float shrink = logf(1.6f);
      Q.scale_x[j] = P.scale_x[i] - shrink;
      Q.scale_y[j] = P.scale_y[i] - shrink;
      Q.scale_z[j] = P.scale_z[i] - shrink;
    }
  }
}

}  // namespace
}  // namespace ds

extern "C" {

int ds_fitter_densify(ds_fitter* f, const ds_densify_params* p, int32_t* new_count,
                      ds_stream stream) {
  if (!f || !p || !new_count) return DS_ERR_ARG;
  if (!f->grad_accum || f->cfg.storage != DS_STORAGE_FP32 || f->g_mem) return DS_ERR_STATE;
  cudaStream_t s = (cudaStream_t)stream;
  const int n = f->cfg.count;
  uint8_t* mode = nullptr;
  uint32_t *emit = nullptr, *iota = nullptr, *total32 = nullptr, *status = nullptr;
  unsigned long long *offs = nullptr, *total = nullptr;
  float *np = nullptr, *nm = nullptr, *nv = nullptr;
  int st = DS_OK;
  auto cleanup = [&]() {
    for (void* q : {(void*)mode, (void*)emit, (void*)iota, (void*)total32, (void*)status,
                    (void*)offs, (void*)total, (void*)np, (void*)nm, (void*)nv})
      cudaFree(q);
  };
  auto fail = [&](int code) {
    cleanup();
    return code;
  };
  if ((st = ds::cuda_status(ds::device_alloc(&mode, n))) ||
      (st = ds::cuda_status(ds::device_alloc(&emit, (size_t)n * 4))) ||
      (st = ds::cuda_status(ds::device_alloc(&iota, (size_t)n * 4))) ||
      (st = ds::cuda_status(ds::device_alloc(&offs, (size_t)n * 8))) ||
      (st = ds::cuda_status(ds::device_alloc(&total, 8))) ||
      (st = ds::cuda_status(ds::device_alloc(&total32, 4))) ||
      (st = ds::cuda_status(ds::device_alloc(&status, 4))))
    return fail(st);
  std::vector<uint32_t> h_iota(n);
  for (int k = 0; k < n; ++k) h_iota[k] = (uint32_t)k;
  if ((st = ds::cuda_status(cudaMemcpyAsync(iota, h_iota.data(), (size_t)n * 4,
                                            cudaMemcpyHostToDevice, s))))
    return fail(st);
  const int blocks = (n + ds::kThreads - 1) / ds::kThreads;
  ds::densify_decide_kernel<<<blocks, ds::kThreads, 0, s>>>(f->P, f->grad_accum, f->grad_count,
                                                            *p, mode, emit);
  if ((st = ds::scan_counts_permuted(emit, iota, (uint32_t)n, offs, total32, total, 0xffffffffu,
                                     status, f->rb.scan, s)))
    return fail(st);
  unsigned long long h_total = 0;
  if ((st = ds::cuda_status(cudaMemcpyAsync(&h_total, total, 8, cudaMemcpyDeviceToHost, s))) ||
      (st = ds::cuda_status(cudaStreamSynchronize(s))))
    return fail(st);
  if (h_total == 0 || h_total > (unsigned long long)f->capacity) return fail(DS_ERR_OOM);
  const int n2 = (int)h_total;
  const size_t floats = (size_t)n2 * (14 + 3 * f->bands);
  if ((st = ds::cuda_status(ds::device_alloc(&np, floats * 4))) ||
      (st = ds::cuda_status(ds::device_alloc(&nm, floats * 4))) ||
      (st = ds::cuda_status(ds::device_alloc(&nv, floats * 4))))
    return fail(st);
  ds_gaussian3d Q, MQ, VQ;
  ds::carve(np, n2, f->bands, Q);
  ds::carve(nm, n2, f->bands, MQ);
  ds::carve(nv, n2, f->bands, VQ);
  ds::densify_scatter_kernel<<<blocks, ds::kThreads, 0, s>>>(f->P, f->M, f->V, mode, offs, Q, MQ,
                                                             VQ, p->seed);
  uint32_t nn = (uint32_t)n2;
  if ((st = ds::cuda_status(cudaGetLastError())) ||
      (st = ds::cuda_status(cudaMemcpyAsync(&f->rb.scalars->n_splats, &nn, 4,
                                            cudaMemcpyHostToDevice, s))) ||
      (st = ds::cuda_status(cudaMemsetAsync(f->grad_accum, 0, (size_t)f->capacity * 4, s))) ||
      (st = ds::cuda_status(cudaMemsetAsync(f->grad_count, 0, (size_t)f->capacity * 4, s))) ||
      (st = ds::cuda_status(cudaStreamSynchronize(s))))
    return fail(st);
  // swap in the new parameter set; the next step recaptures the graph
  cudaFree(f->params_mem);
  cudaFree(f->m_mem);
  cudaFree(f->v_mem);
  f->params_mem = np;
  f->m_mem = nm;
  f->v_mem = nv;
  np = nm = nv = nullptr;
  f->P = Q;
  f->M = MQ;
  f->V = VQ;
  f->G = Q;
  f->floats = floats;
  f->cfg.count = n2;
  if (f->exec) cudaGraphExecDestroy(f->exec);
  if (f->graph) cudaGraphDestroy(f->graph);
  f->exec = nullptr;
  f->graph = nullptr;
  cleanup();
  *new_count = n2;
  return DS_OK;
}

int ds_fitter_density_stats(ds_fitter* f, float** grad_accum, uint32_t** visible_steps) {
  if (!f || !grad_accum || !visible_steps) return DS_ERR_ARG;
  if (!f->grad_accum) return DS_ERR_STATE;
  *grad_accum = f->grad_accum;
  *visible_steps = f->grad_count;
  return DS_OK;
}

}  // extern "C"
