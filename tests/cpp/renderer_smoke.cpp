// C++ smoke test of the drop-in viewer API: PLYSaver writes a random scene,
// SplatRenderer::reloadPLY loads, normalises and uploads it, render() draws it
// from a camera on the +z axis.  Exit code 0 when splats are visible and the
// image holds colour.
#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

#include "io/ply_io.h"
#include "pipelines/splat_renderer.h"
#include "utils/splat_utils.h"

int main(int argc, char** argv) {
  const std::string path = argc > 1 ? argv[1] : "renderer_smoke.ply";
  const int W = 320, H = 240;
  std::vector<Gaussian3D> scene = SplatUtils::randomInit(5000, 200, 200, 3);
  PLYSaver::save(path, scene, 0);
  SplatRenderer r;
  r.init(W, H);
  r.reloadPLY(path, 1.f);
  if (!r.isLoaded() || r.getMaxSHDegree() != 0) return 2;
  // view: camera at z = 3 looking down -z; proj: GL perspective, fovy 60 deg
  float view[4][4] = {{1, 0, 0, 0}, {0, 1, 0, 0}, {0, 0, 1, 0}, {0, 0, -3, 1}};
  const float f = 1.f / std::tan(0.5f * 1.0471976f), n = 0.1f, fa = 100.f;
  float proj[4][4] = {{f * H / W, 0, 0, 0},
                      {0, f, 0, 0},
                      {0, 0, -(fa + n) / (fa - n), -1},
                      {0, 0, -2 * fa * n / (fa - n), 0}};
  r.render(view, proj, ds_compat::Vec3Arg(0.f, 0.f, 3.f));
  std::vector<float> img((size_t)W * H * 3);
  cudaMemcpy(img.data(), r.getOutput(), img.size() * sizeof(float), cudaMemcpyDeviceToHost);
  double sum = 0.0;
  for (float v : img) sum += v;
  const unsigned vis = r.getVisibleCount();
  std::printf("visible %u of %zu, mean %.4f\n", vis, scene.size(), sum / img.size());
  return (vis > 1000 && sum > 0.0 && std::isfinite(sum)) ? 0 : 1;
}
