// C entry points around the reference's own host PLY reader and writer
// (src/io/ply_io.cpp: PLYLoader::load, PLYSaver::save), built from the
// reference sources by `make -C oracle ref REF=<reference tree>` into
// oracle/_ref/libdsref_ply.so.
//
// TEST INFRASTRUCTURE ONLY: the CPU PLY tests and tests/golden/make_golden_ply.py
// use it to check ds_ply_read / ds_ply_write against the reference's code.
// Splats cross the boundary as the reference's host record Gaussian3D
// (src/types/gaussian3d.h:13-21), 59 floats each.
#include <stdint.h>
#include <string.h>

#include <exception>
#include <vector>

#include "io/ply_io.h"

static_assert(sizeof(Gaussian3D) == 59 * sizeof(float), "Gaussian3D is 59 packed floats");

extern "C" int ref_ply_save(const char* path, const float* splats, int64_t count, int sh_num_bands) {
  try {
    std::vector<Gaussian3D> v((size_t)count);
    if (count) memcpy(v.data(), splats, (size_t)count * sizeof(Gaussian3D));
    PLYSaver::save(path, v, sh_num_bands);
  } catch (const std::exception&) {
    return 1;
  }
  return 0;
}

extern "C" int ref_ply_load(const char* path, float* splats, int64_t capacity, int64_t* count,
                            int* sh_degree) {
  try {
    PLYLoadResult r = PLYLoader::load(path);
    *count = (int64_t)r.splats.size();
    *sh_degree = r.sh_degree;
    if (*count > capacity) return 2;
    if (*count) memcpy(splats, r.splats.data(), (size_t)*count * sizeof(Gaussian3D));
  } catch (const std::exception&) {
    return 1;
  }
  return 0;
}
