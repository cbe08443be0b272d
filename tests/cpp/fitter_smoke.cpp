// C++ smoke test of the drop-in API: the reference's ImageFitter sequence
// (init, random init, initLayers, step, getLoss) on libdiffsplat_b200.
// Exit code 0 when the loss drops by half within 200 steps.
#include <cmath>
#include <cstdio>
#include <vector>

#include "pipelines/image_fitter.h"

int main() {
  const int W = 128, H = 96;
  std::vector<float> target((size_t)W * H * 3);
  for (int i = 0; i < H; ++i)
    for (int j = 0; j < W; ++j) {
      float* p = &target[((size_t)i * W + j) * 3];
      p[0] = 0.2f + 0.6f * j / W;
      p[1] = 0.2f + 0.6f * i / H;
      p[2] = ((i / 8 + j / 8) % 2) ? 0.8f : 0.3f;
    }
  ImageFitter fitter;
  fitter.init(W, H);
  fitter.setTargetPixels(target.data());
  fitter.randomInitGaussians(2000, 7);
  fitter.initLayers();
  fitter.step();
  const float l0 = fitter.getLoss();
  for (int k = 0; k < 199; ++k) fitter.step();
  const float l1 = fitter.getLoss();
  std::printf("loss %.6f -> %.6f after %d steps\n", l0, l1, fitter.getIterCount());
  return (std::isfinite(l1) && l1 < 0.5f * l0) ? 0 : 1;
}
