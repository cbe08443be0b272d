// PLYLoader / PLYSaver (src/io/ply_io.h:28-57) over ds_ply_* of
// libdiffsplat_b200: binary little-endian 3DGS PLY, OpenCV frame on disk,
// OpenGL frame in memory, SH degree from the f_rest_* count.  Errors throw
// std::runtime_error (the reference's log_fatal throws).
#pragma once
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../diffsplat_b200.h"
#include "../types/gaussian3d.h"

static_assert(sizeof(Gaussian3D) == 59 * sizeof(float), "Gaussian3D must be 59 packed floats");

struct PLYLoadResult {
  std::vector<Gaussian3D> splats;
  int sh_degree = 0;
};

class PLYLoader {
 public:
  static PLYLoadResult load(const std::string& path) {
    int64_t n = 0;
    int deg = 0;
    if (ds_ply_probe(path.c_str(), &n, &deg) != DS_OK)
      throw std::runtime_error("[PLYLoader] cannot read " + path);
    PLYLoadResult r;
    r.splats.resize((size_t)n);
    if (ds_ply_read(path.c_str(), reinterpret_cast<float*>(r.splats.data()), n, &n, &deg) != DS_OK)
      throw std::runtime_error("[PLYLoader] malformed PLY " + path);
    r.sh_degree = deg;
    return r;
  }
};

class PLYSaver {
 public:
  static void save(const std::string& path, const std::vector<Gaussian3D>& splats,
                   int sh_num_bands = 0) {
    if (ds_ply_write(path.c_str(), reinterpret_cast<const float*>(splats.data()),
                     (int64_t)splats.size(), sh_num_bands) != DS_OK)
      throw std::runtime_error("[PLYSaver] cannot write " + path);
  }
};
