// ImageLoader / ImageSaver (src/io/image_io.h:17-47) over ds_image_* of
// libdiffsplat_b200: host decode (PNG, PPM / PGM), aspect fit + pad on the
// GPU, PNG writing.  A failed load returns an empty LoadedImage, like the
// reference.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../diffsplat_b200.h"

struct LoadedImage {
  std::vector<float> pixels;  // RGB [0, 1]
  int canvas_w = 0;
  int canvas_h = 0;
  int src_w = 0;
  int src_h = 0;
};

class ImageLoader {
 public:
  static LoadedImage load(const std::string& path, int target_w, int target_h, int padding = 0) {
    int w = 0, h = 0;
    if (ds_image_probe(path.c_str(), &w, &h) != DS_OK) return {};
    std::vector<uint8_t> rgb((size_t)w * h * 3);
    if (ds_image_read_rgb8(path.c_str(), rgb.data(), (int64_t)rgb.size(), &w, &h) != DS_OK)
      return {};
    uint8_t* d_src = nullptr;
    float* d_dst = nullptr;
    LoadedImage out;
    const size_t canvas = (size_t)target_w * target_h * 3;
    if (cudaMalloc(&d_src, rgb.size()) == cudaSuccess &&
        cudaMalloc(&d_dst, canvas * sizeof(float)) == cudaSuccess &&
        cudaMemcpy(d_src, rgb.data(), rgb.size(), cudaMemcpyHostToDevice) == cudaSuccess &&
        ds_image_fit(d_src, w, h, target_w, target_h, padding, d_dst, nullptr, nullptr,
                     nullptr) == DS_OK) {
      out.pixels.resize(canvas);
      if (cudaMemcpy(out.pixels.data(), d_dst, canvas * sizeof(float), cudaMemcpyDeviceToHost) ==
          cudaSuccess)
        out = LoadedImage{out.pixels, target_w, target_h, w, h};
      else
        out = LoadedImage{};
    }
    cudaFree(d_src);
    cudaFree(d_dst);
    return out;
  }
};

class ImageSaver {
 public:
  static void saveAsPNG(const float* d_pixels, int width, int height, const std::string& path) {
    std::vector<float> h((size_t)width * height * 3);
    cudaMemcpy(h.data(), d_pixels, h.size() * sizeof(float), cudaMemcpyDeviceToHost);
    ds_image_write_png(path.c_str(), h.data(), width, height);
  }
};
