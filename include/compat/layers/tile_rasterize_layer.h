// TileRasterizeLayer (src/layers/tile_rasterize_layer.h:23-60) on a ds_raster
// handle of libdiffsplat_b200: tile keys, sort, ranges, front-to-back
// compositing into output [H*W*3]; backward accumulates into grad_input.
#pragma once
#include <cstdint>

#include "ds_compat_views.h"
#include "layer.h"

class TileRasterizeLayer
    : public TypedLayer<Splat2DParams, CudaBuffer<float>, Splat2DGrads, CudaBuffer<float>> {
 public:
  ~TileRasterizeLayer() {
    if (handle) ds_raster_destroy(handle);
  }
  using TypedLayer::allocate;
  void allocate(int width, int height, int count) {
    if (handle) ds_raster_destroy(handle);
    handle = nullptr;
    DS_COMPAT_CHECK(ds_raster_create(width, height, count, 0, &handle));
    if (handle) ds_raster_set_grad_mode(handle, grad_mode);
    w = width;
    h = height;
    output.allocate((size_t)width * height * 3);
  }
  void resize(int new_width, int new_height) {
    if (new_width == w && new_height == h) return;
    DS_COMPAT_CHECK(ds_raster_resize(handle, new_width, new_height));
    w = new_width;
    h = new_height;
    output.allocate((size_t)w * h * 3);
  }
  void forward() override {
    ds_splat2d in = ds_compat::view(*input, input->count);
    DS_COMPAT_CHECK(ds_raster_forward(handle, &in, output.ptr, nullptr));
  }
  void backward() override {
    ds_splat2d in = ds_compat::view(*input, input->count);
    ds_splat2d gin = ds_compat::view(grad_input, input->count);
    DS_COMPAT_CHECK(ds_raster_backward(handle, &in, grad_output->ptr, &gin, nullptr));
  }
  uint32_t getVisibleCount() {
    uint32_t c = 0;
    DS_COMPAT_CHECK(ds_raster_visible_count(handle, &c));
    return c;
  }
  void setGradMode(int mode) {
    grad_mode = mode;
    if (handle) ds_raster_set_grad_mode(handle, mode);
  }

 private:
  ds_raster* handle = nullptr;
  int w = 0, h = 0;
  int grad_mode = ds_default_grad_mode();
};
