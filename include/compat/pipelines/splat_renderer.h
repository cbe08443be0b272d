// SplatRenderer (src/pipelines/splat_renderer.h:17-60): forward-only viewing
// of a PLY scene on ds_renderer_* of libdiffsplat_b200.  reloadPLY loads,
// normalises (SplatUtils::normalizeScene) and uploads the scene; render(view,
// proj, cam_pos) runs activation + projection + rasterisation forward with
// PV = proj * view; getOutput() is the device RGB image [h*w*3].
#pragma once
#include <stdexcept>
#include <string>

#include "../../diffsplat_b200.h"
#include "../io/ply_io.h"
#include "../layers/ds_compat_views.h"
#include "../utils/gaussian3d_io.h"
#include "../utils/splat_utils.h"

class SplatRenderer {
 public:
  ~SplatRenderer() {
    if (renderer) ds_renderer_destroy(renderer);
  }

  void init(int w, int h) {
    width = w;
    height = h;
  }

  void reloadPLY(const std::string& path, float sceneScale = 1.f) {
    loaded = false;
    if (renderer) {
      ds_renderer_destroy(renderer);
      renderer = nullptr;
    }
    PLYLoadResult r = PLYLoader::load(path);
    if (r.splats.empty()) throw std::runtime_error("[SplatRenderer] PLY loaded 0 splats: " + path);
    SplatUtils::normalizeScene(r.splats, sceneScale);
    sh_degree = r.sh_degree;
    uploadGaussians(gaussian_params, r.splats, sh_degree);
    check(ds_renderer_create(width, height, gaussian_params.count, sh_degree, 0, DS_STORAGE_FP32,
                             &renderer));
    ds_gaussian3d v = ds_compat::view(gaussian_params);
    check(ds_renderer_set_params(renderer, &v, nullptr));
    loaded = true;
  }

  bool isLoaded() const { return loaded; }

  void render(ds_compat::Mat4Arg view, ds_compat::Mat4Arg proj, ds_compat::Vec3Arg cam_pos) {
    if (!renderer) return;
    float pv[16];
    ds_compat::mat4_mul(proj.m, view.m, pv);
    const float cam[3] = {cam_pos.x, cam_pos.y, cam_pos.z};
    check(ds_renderer_render(renderer, pv, cam, nullptr));
  }

  void resize(int newWidth, int newHeight) {
    width = newWidth;
    height = newHeight;
    if (renderer) check(ds_renderer_resize(renderer, width, height));
  }

  float* getOutput() {
    float* p = nullptr;
    if (renderer) ds_renderer_output(renderer, &p);
    return p;
  }

  uint32_t getVisibleCount() {
    uint64_t c[2] = {0, 0};
    if (renderer) ds_renderer_counts(renderer, c, 2);
    return (uint32_t)c[0];
  }

  int getMaxSHDegree() const { return sh_degree; }
  void setActiveSHDegree(int d) {
    if (renderer) check(ds_renderer_set_sh_degree(renderer, d));
  }

 private:
  static void check(int st) {
    if (st != DS_OK) throw std::runtime_error(std::string("[SplatRenderer] ") + ds_status_string(st));
  }

  int width = 0, height = 0, sh_degree = 0;
  bool loaded = false;
  Gaussian3DParams gaussian_params;
  ds_renderer* renderer = nullptr;
};
