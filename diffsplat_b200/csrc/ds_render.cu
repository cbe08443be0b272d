// Forward-only renderer: SplatRenderer::render (src/pipelines/splat_renderer.cpp:84-91),
// i.e. GaussActiv -> PerspProject -> TileRasterize forward, as one preprocess
// kernel (activation + projection + tile rectangle + record), the list build
// (depth sort, emission, tile sort, ranges, tile schedule) and the composite
// forward.  No gradient buffers are allocated beyond what the list build needs.
#include <algorithm>
#include <new>

#include "ds_common.cuh"
#include "ds_internal.h"
#include "ds_preprocess.cuh"

struct ds_renderer {
  int storage = DS_STORAGE_FP32;
  int sh_degree = 0;         // degree the SH buffers hold
  int active_degree = 0;     // degree evaluated (setActiveSHDegree)
  int max_splats = 0;
  int count = 0;
  int bands = 0;
  ds_gaussian3d P{};         // FP32 views (positions always read from here)
  __nv_bfloat16* copy_mem = nullptr;  // BF16 storage: converted attributes
  size_t copy_elems = 0;
  ds::Soa<__nv_bfloat16> R16{};
  ds::RasterBuffers rb;
  ds::Camera* cam_dev = nullptr;
  ds::HostStage cam_stage;
  float* image = nullptr;
  bool have_params = false;
};

namespace {

size_t image_floats(int w, int h) { return (size_t)w * h * 3; }

}  // namespace

extern "C" {

int ds_renderer_create(int width, int height, int max_splats, int sh_degree, int64_t max_isects,
                       int storage, ds_renderer** out) {
  if (!out) return DS_ERR_ARG;
  *out = nullptr;
  if (width <= 0 || height <= 0 || max_splats <= 0 || sh_degree < 0 || sh_degree > 3)
    return DS_ERR_ARG;
  if (storage != DS_STORAGE_FP32 && storage != DS_STORAGE_BF16) return DS_ERR_ARG;
  ds_renderer* r = new (std::nothrow) ds_renderer();
  if (!r) return DS_ERR_OOM;
  auto fail = [&](int code) {
    ds_renderer_destroy(r);
    return code;
  };
  r->storage = storage;
  r->sh_degree = sh_degree;
  r->active_degree = sh_degree;
  r->max_splats = max_splats;
  r->bands = ds::sh_bands(sh_degree);
  int st;
  if ((st = ds::raster_alloc(r->rb, width, height, max_splats, max_isects))) return fail(st);
  if ((st = ds::cuda_status(ds::device_alloc(&r->cam_dev, sizeof(ds::Camera))))) return fail(st);
  cudaMemset(r->cam_dev, 0, sizeof(ds::Camera));
  if ((st = ds::cuda_status(ds::device_alloc(&r->image, image_floats(width, height) * 4))))
    return fail(st);
  cudaMemset(r->image, 0, image_floats(width, height) * 4);
  if (storage == DS_STORAGE_BF16) {
    r->copy_elems = (size_t)max_splats * (14 + 3 * r->bands);
    if ((st = ds::cuda_status(ds::device_alloc(&r->copy_mem, r->copy_elems * 2)))) return fail(st);
  }
  if ((st = ds::cuda_status(cudaDeviceSynchronize()))) return fail(st);
  *out = r;
  return DS_OK;
}

int ds_renderer_set_params(ds_renderer* r, const ds_gaussian3d* params, ds_stream stream) {
  if (!r || !params) return DS_ERR_ARG;
  const int n = params->count;
  if (n < 0 || n > r->max_splats) return DS_ERR_ARG;
  if (params->sh_num_bands != r->bands) return DS_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  r->P = *params;
  r->count = n;
  if (r->storage == DS_STORAGE_BF16 && n > 0) {
    ds::carve_soa(r->copy_mem, n, r->bands, r->R16);
    float* src[17] = {params->pos_x,   params->pos_y,   params->pos_z,   params->scale_x,
                      params->scale_y, params->scale_z, params->rot_w,   params->rot_x,
                      params->rot_y,   params->rot_z,   params->sh_dc_r, params->sh_dc_g,
                      params->sh_dc_b, params->logit_opacity, params->sh_rest_r,
                      params->sh_rest_g, params->sh_rest_b};
    __nv_bfloat16* dst[17] = {r->R16.pos_x,   r->R16.pos_y,   r->R16.pos_z,   r->R16.scale_x,
                              r->R16.scale_y, r->R16.scale_z, r->R16.rot_w,   r->R16.rot_x,
                              r->R16.rot_y,   r->R16.rot_z,   r->R16.sh_dc_r, r->R16.sh_dc_g,
                              r->R16.sh_dc_b, r->R16.logit_opacity, r->R16.sh_rest_r,
                              r->R16.sh_rest_g, r->R16.sh_rest_b};
    for (int k = 0; k < 17; ++k) {
      const size_t len = (size_t)n * (k < 14 ? 1 : r->bands);
      if (len == 0 || !src[k]) continue;
      const unsigned blocks = (unsigned)std::min<size_t>((len + 255) / 256, 148 * 8);
      ds::to_bf16_kernel<<<blocks, ds::kPreThreads, 0, s>>>(src[k], dst[k], len);
    }
    DS_CUDA(cudaGetLastError());
  }
  uint32_t nn = (uint32_t)n;
  DS_CUDA(cudaMemcpyAsync(&r->rb.scalars->n_splats, &nn, sizeof(uint32_t),
                          cudaMemcpyHostToDevice, s));
  DS_CUDA(cudaStreamSynchronize(s));
  r->have_params = true;
  return DS_OK;
}

int ds_renderer_set_sh_degree(ds_renderer* r, int degree) {
  if (!r || degree < 0 || degree > r->sh_degree) return DS_ERR_ARG;
  r->active_degree = degree;
  return DS_OK;
}

int ds_renderer_render(ds_renderer* r, const float pv[16], const float cam_pos[3],
                       ds_stream stream) {
  if (!r || !pv || !cam_pos) return DS_ERR_ARG;
  if (!r->have_params) return DS_ERR_STATE;
  cudaStream_t s = (cudaStream_t)stream;
  ds::Camera c;
  for (int k = 0; k < 16; ++k) c.pv[k] = pv[k];
  for (int k = 0; k < 3; ++k) c.cam[k] = cam_pos[k];
  c.pad = 0.f;
  DS_TRY(r->cam_stage.upload(r->cam_dev, &c, sizeof(c), s));
  ds::RasterBuffers& rb = r->rb;
  DS_CUDA(cudaMemsetAsync(&rb.scalars->visible, 0, sizeof(uint32_t), s));
  const int n = r->count;
  if (n > 0) {
    const unsigned blocks = (unsigned)((n + ds::kPreThreads - 1) / ds::kPreThreads);
    if (r->storage == DS_STORAGE_BF16)
      ds::fit_preprocess_kernel<<<blocks, ds::kPreThreads, 0, s>>>(
          r->P, r->R16, r->active_degree, r->cam_dev, rb.width, rb.height, rb.ntx, rb.nty,
          rb.rec_a, rb.rec_b, rb.rec_c, rb.rec_idet, rb.rect, rb.counts, rb.depth_keys,
          rb.scalars);
    else
      ds::fit_preprocess_kernel<<<blocks, ds::kPreThreads, 0, s>>>(
          r->P, ds::soa_of(r->P), r->active_degree, r->cam_dev, rb.width, rb.height, rb.ntx,
          rb.nty, rb.rec_a, rb.rec_b, rb.rec_c, rb.rec_idet, rb.rect, rb.counts, rb.depth_keys,
          rb.scalars);
    DS_CUDA(cudaGetLastError());
  }
  DS_TRY(ds::raster_build_lists(rb, n, s));
  return ds::raster_composite_forward(rb, r->image, nullptr, s);
}

int ds_renderer_output(ds_renderer* r, float** rgb) {
  if (!r || !rgb) return DS_ERR_ARG;
  *rgb = r->image;
  return DS_OK;
}

int ds_renderer_resize(ds_renderer* r, int width, int height) {
  if (!r || width <= 0 || height <= 0) return DS_ERR_ARG;
  DS_CUDA(cudaDeviceSynchronize());
  DS_TRY(ds::raster_resize(r->rb, width, height));
  cudaFree(r->image);
  r->image = nullptr;
  DS_CUDA(ds::device_alloc(&r->image, image_floats(width, height) * 4));
  DS_CUDA(cudaMemset(r->image, 0, image_floats(width, height) * 4));
  return DS_OK;
}

int ds_renderer_counts(ds_renderer* r, uint64_t* out, int n) {
  if (!r || !out || n < 2) return DS_ERR_ARG;
  DS_CUDA(cudaDeviceSynchronize());
  ds::DevScalars sc;
  DS_CUDA(cudaMemcpy(&sc, r->rb.scalars, sizeof(sc), cudaMemcpyDeviceToHost));
  out[0] = sc.visible;
  out[1] = sc.n_isects_raw;
  return DS_OK;
}

int ds_renderer_status(ds_renderer* r, uint32_t* flags) {
  if (!r || !flags) return DS_ERR_ARG;
  DS_CUDA(cudaDeviceSynchronize());
  uint32_t st = 0, zero = 0;
  DS_CUDA(cudaMemcpy(&st, &r->rb.scalars->status, sizeof(uint32_t), cudaMemcpyDeviceToHost));
  DS_CUDA(cudaMemcpy(&r->rb.scalars->status, &zero, sizeof(uint32_t), cudaMemcpyHostToDevice));
  *flags = st;
  return ds::status_code(st);
}

int ds_renderer_destroy(ds_renderer* r) {
  if (!r) return DS_ERR_ARG;
  ds::raster_free(r->rb);
  cudaFree(r->cam_dev);
  cudaFree(r->image);
  cudaFree(r->copy_mem);
  delete r;
  return DS_OK;
}

}  // extern "C"
