// C ABI entry points of the per-layer path (include/diffsplat_b200.h).
#include <math.h>
#include <string.h>

#include <atomic>
#include <new>
#include <vector>

#include "ds_common.cuh"
#include "ds_internal.h"

struct ds_raster {
  ds::RasterBuffers rb;
  int last_count = 0;
};

namespace {

bool g3_ok(const ds_gaussian3d* g, int degree) {
  if (!g || g->count < 0) return false;
  if (g->count == 0) return true;
  if (!g->pos_x || !g->pos_y || !g->pos_z || !g->scale_x || !g->scale_y || !g->scale_z ||
      !g->rot_w || !g->rot_x || !g->rot_y || !g->rot_z || !g->sh_dc_r || !g->sh_dc_g ||
      !g->sh_dc_b || !g->logit_opacity)
    return false;
  if (degree > 0) {
    if (g->sh_num_bands < ds::sh_bands(degree)) return false;
    if (!g->sh_rest_r || !g->sh_rest_g || !g->sh_rest_b) return false;
  }
  return true;
}

bool s3_ok(const ds_splat3d* s) {
  if (!s || s->count < 0) return false;
  if (s->count == 0) return true;
  return s->pos_x && s->pos_y && s->pos_z && s->cov_xx && s->cov_xy && s->cov_xz && s->cov_yy &&
         s->cov_yz && s->cov_zz && s->color_r && s->color_g && s->color_b && s->opacity;
}

bool s2_ok(const ds_splat2d* s) {
  if (!s || s->count < 0) return false;
  if (s->count == 0) return true;
  return s->pos_x && s->pos_y && s->pos_z && s->cov_xx && s->cov_xy && s->cov_yy && s->color_r &&
         s->color_g && s->color_b && s->opacity;
}

}  // namespace

namespace {
int g_default_grad_mode = -1;  // -1: not yet read from the environment
// Successful device allocations left before they fail; -1: no limit.
std::atomic<int64_t> g_alloc_budget{-1};
}

namespace ds {
cudaError_t device_alloc_bytes(void** p, size_t bytes) {
  int64_t left = g_alloc_budget.load();
  while (left >= 0) {
    if (left == 0) {
      *p = nullptr;
      return cudaErrorMemoryAllocation;
    }
    if (g_alloc_budget.compare_exchange_weak(left, left - 1)) break;
  }
  return cudaMalloc(p, bytes);
}
}  // namespace ds

extern "C" {

int ds_debug_fail_allocations_after(int64_t n) {
  g_alloc_budget.store(n < 0 ? -1 : n);
  return DS_OK;
}

int ds_default_grad_mode(void) {
  if (g_default_grad_mode < 0) {
    const char* e = getenv("DS_GRAD_MODE");
    g_default_grad_mode =
        (e && strcmp(e, "exact") == 0) ? DS_GRAD_EXACT : DS_GRAD_REFERENCE;
  }
  return g_default_grad_mode;
}

int ds_set_default_grad_mode(int mode) {
  if (mode != DS_GRAD_REFERENCE && mode != DS_GRAD_EXACT) return DS_ERR_ARG;
  g_default_grad_mode = mode;
  return DS_OK;
}

int ds_abi_version(void) { return DS_ABI_VERSION; }

const char* ds_status_string(int status) {
  switch (status) {
    case DS_OK: return "ok";
    case DS_ERR_ARG: return "invalid argument";
    case DS_ERR_OOM: return "device allocation failed";
    case DS_ERR_CUDA: return "CUDA error";
    case DS_ERR_ISECT_OVERFLOW: return "intersection buffer overflow";
    case DS_ERR_STATE: return "invalid state";
    case DS_ERR_NO_DEVICE: return "no sm_100 CUDA device";
    case DS_ERR_INTERNAL: return "device-side consistency check failed";
    default: return "unknown status";
  }
}

int ds_device_check(void) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return DS_ERR_NO_DEVICE;
  cudaDeviceProp p;
  if (cudaGetDeviceProperties(&p, dev) != cudaSuccess) return DS_ERR_NO_DEVICE;
  return p.major == 10 ? DS_OK : DS_ERR_NO_DEVICE;
}

int ds_activ_forward(const ds_gaussian3d* in, int sh_degree, const float cam_pos[3],
                     const ds_splat3d* out, ds_stream stream) {
  if (sh_degree < 0 || sh_degree > 3 || !cam_pos || !g3_ok(in, sh_degree) || !s3_ok(out) ||
      out->count < in->count)
    return DS_ERR_ARG;
  return ds::launch_activ_forward(*in, sh_degree, cam_pos, *out, (cudaStream_t)stream);
}

int ds_activ_backward(const ds_gaussian3d* in, const ds_splat3d* out, const ds_splat3d* grad_out,
                      int sh_degree, const float cam_pos[3], const ds_gaussian3d* grad_in,
                      ds_stream stream) {
  if (sh_degree < 0 || sh_degree > 3 || !cam_pos || !g3_ok(in, sh_degree) || !s3_ok(out) ||
      !s3_ok(grad_out) || !g3_ok(grad_in, sh_degree))
    return DS_ERR_ARG;
  return ds::launch_activ_backward(*in, *out, *grad_out, sh_degree, cam_pos, *grad_in,
                                   (cudaStream_t)stream);
}

int ds_project_forward(const ds_splat3d* in, const float pv[16], const ds_splat2d* out,
                       ds_stream stream) {
  if (!pv || !s3_ok(in) || !s2_ok(out)) return DS_ERR_ARG;
  return ds::launch_project_forward(*in, pv, *out, (cudaStream_t)stream);
}

int ds_project_backward(const ds_splat3d* in, const float pv[16], const ds_splat2d* grad_out,
                        const ds_splat3d* grad_in, ds_stream stream) {
  if (!pv || !s3_ok(in) || !s2_ok(grad_out) || !s3_ok(grad_in)) return DS_ERR_ARG;
  return ds::launch_project_backward(*in, pv, *grad_out, *grad_in, ds_default_grad_mode(),
                                     (cudaStream_t)stream);
}

int ds_project_backward_ex(const ds_splat3d* in, const float pv[16], const ds_splat2d* grad_out,
                           const ds_splat3d* grad_in, int grad_mode, ds_stream stream) {
  if (!pv || !s3_ok(in) || !s2_ok(grad_out) || !s3_ok(grad_in)) return DS_ERR_ARG;
  if (grad_mode != DS_GRAD_REFERENCE && grad_mode != DS_GRAD_EXACT) return DS_ERR_ARG;
  return ds::launch_project_backward(*in, pv, *grad_out, *grad_in, grad_mode,
                                     (cudaStream_t)stream);
}

int ds_raster_create(int width, int height, int max_splats, int64_t max_isects, ds_raster** out) {
  if (!out) return DS_ERR_ARG;
  *out = nullptr;
  ds_raster* r = new (std::nothrow) ds_raster();
  if (!r) return DS_ERR_OOM;
  int st = ds::raster_alloc(r->rb, width, height, max_splats, max_isects);
  r->rb.grad_mode = ds_default_grad_mode();
  if (st != DS_OK) {
    ds::raster_free(r->rb);
    delete r;
    return st;
  }
  *out = r;
  return DS_OK;
}

int ds_raster_resize(ds_raster* r, int width, int height) {
  if (!r) return DS_ERR_ARG;
  return ds::raster_resize(r->rb, width, height);
}

int ds_raster_set_grad_mode(ds_raster* r, int mode) {
  if (!r || (mode != DS_GRAD_REFERENCE && mode != DS_GRAD_EXACT)) return DS_ERR_ARG;
  r->rb.grad_mode = mode;
  return DS_OK;
}

int ds_raster_forward(ds_raster* r, const ds_splat2d* in, float* out_rgb, ds_stream stream) {
  if (!r || !s2_ok(in) || !out_rgb || in->count > r->rb.max_splats) return DS_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  DS_TRY(ds::raster_prepare_from_splat2d(r->rb, *in, s));
  DS_TRY(ds::raster_build_lists(r->rb, in->count, s, nullptr, true));
  DS_TRY(ds::raster_composite_forward(r->rb, out_rgb, nullptr, s));
  r->last_count = in->count;
  return DS_OK;
}

int ds_raster_backward(ds_raster* r, const ds_splat2d* in, const float* grad_rgb,
                       const ds_splat2d* grad_in, ds_stream stream) {
  if (!r || !s2_ok(in) || !grad_rgb || !s2_ok(grad_in) || in->count != r->last_count)
    return DS_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  DS_TRY(ds::raster_composite_backward(r->rb, nullptr, grad_rgb, nullptr, s));
  DS_TRY(ds::raster_reduce_grads(r->rb, *grad_in, in->count, s));
  return DS_OK;
}

int ds_raster_visible_count(ds_raster* r, uint32_t* out) {
  if (!r || !out) return DS_ERR_ARG;
  DS_CUDA(cudaDeviceSynchronize());
  DS_CUDA(cudaMemcpy(out, &r->rb.scalars->visible, sizeof(uint32_t), cudaMemcpyDeviceToHost));
  return DS_OK;
}

int ds_raster_isect_count(ds_raster* r, uint32_t* out) {
  if (!r || !out) return DS_ERR_ARG;
  DS_CUDA(cudaDeviceSynchronize());
  unsigned long long raw = 0;
  DS_CUDA(cudaMemcpy(&raw, &r->rb.scalars->n_isects_raw, sizeof(raw), cudaMemcpyDeviceToHost));
  *out = raw > 0xffffffffull ? 0xffffffffu : (uint32_t)raw;
  return DS_OK;
}

int ds_raster_status(ds_raster* r, uint32_t* flags) {
  if (!r || !flags) return DS_ERR_ARG;
  DS_CUDA(cudaDeviceSynchronize());
  uint32_t st = 0, zero = 0;
  DS_CUDA(cudaMemcpy(&st, &r->rb.scalars->status, sizeof(uint32_t), cudaMemcpyDeviceToHost));
  DS_CUDA(cudaMemcpy(&r->rb.scalars->status, &zero, sizeof(uint32_t), cudaMemcpyHostToDevice));
  *flags = st;
  return ds::status_code(st);
}

int ds_raster_download(ds_raster* r, int what, void* host, int64_t bytes) {
  if (!r || !host || bytes < 0) return DS_ERR_ARG;
  return ds::raster_download(r->rb, r->last_count, what, host, bytes);
}

int ds_raster_destroy(ds_raster* r) {
  if (!r) return DS_ERR_ARG;
  ds::raster_free(r->rb);
  delete r;
  return DS_OK;
}

int ds_mse_forward(const float* pixels, const float* target, int64_t num_pixels, float* loss,
                   ds_stream stream) {
  if (!pixels || !target || !loss || num_pixels < 0) return DS_ERR_ARG;
  return ds::launch_mse_forward(pixels, target, num_pixels, loss, nullptr, nullptr,
                                (cudaStream_t)stream);
}

int ds_mse_backward(const float* pixels, const float* target, int64_t num_pixels, float* grad,
                    ds_stream stream) {
  if (!pixels || !target || !grad || num_pixels < 0) return DS_ERR_ARG;
  return ds::launch_mse_backward(pixels, target, num_pixels, grad, (cudaStream_t)stream);
}

int ds_adam_step(const ds_adam_group* groups, int n_groups, float beta1, float beta2,
                 float epsilon, int step, ds_stream stream) {
  if (n_groups < 0 || (n_groups > 0 && !groups) || step < 1) return DS_ERR_ARG;
  for (int k = 0; k < n_groups; ++k)
    if (groups[k].n > 0 && (!groups[k].param || !groups[k].grad || !groups[k].m || !groups[k].v))
      return DS_ERR_ARG;
  const float bc1 = 1.f / (1.f - powf(beta1, (float)step));
  const float bc2 = 1.f / (1.f - powf(beta2, (float)step));
  return ds::launch_adam_multi(groups, n_groups, beta1, beta2, epsilon, bc1, bc2,
                               (cudaStream_t)stream);
}

}  // extern "C"
