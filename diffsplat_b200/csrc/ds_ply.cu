// Host I/O of splat scenes: binary little-endian 3DGS PLY files
// (src/io/ply_io.cpp:15-227) and scene normalisation (src/utils/splat_utils.h,
// normalizeScene).  Splats cross this boundary as arrays of the reference's
// host record Gaussian3D (src/types/gaussian3d.h:13-21): 59 floats per splat,
// pos xyz, log-scale xyz, quaternion wxyz, SH DC rgb, 45 SH-rest floats stored
// channel-first (R bands, then G, then B), logit opacity.
//
// Conventions kept from the reference: files are in the OpenCV frame (y down,
// z forward) and splats in the OpenGL frame, so y, z and the quaternion's y, z
// are negated on read and on write; the SH degree of a file follows from its
// f_rest_* count (>= 45 -> 3, >= 24 -> 2, >= 9 -> 1).
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <new>
#include <cmath>
#include <fstream>
#include <sstream>
#include <string>
#include <unordered_map>
#include <vector>

#include "diffsplat_b200.h"

namespace {

constexpr int kRec = 59;  // floats per Gaussian3D record
constexpr int kPos = 0, kScale = 3, kRot = 6, kDc = 10, kRest = 13, kLogit = 58;

struct Header {
  int64_t count = 0;
  std::vector<std::string> props;  // float properties in file order
  std::streampos data = 0;
  bool ok = false;
  bool float_only = true;
};

bool ends_with_ply(const char* path) {
  std::string p(path);
  const size_t dot = p.find_last_of('.');
  if (dot == std::string::npos) return false;
  std::string ext = p.substr(dot + 1);
  for (char& c : ext) c = (char)tolower((unsigned char)c);
  return ext == "ply";
}

Header read_header(std::ifstream& f) {
  Header h;
  std::string line;
  bool binary_le = false;
  while (std::getline(f, line)) {
    if (!line.empty() && line.back() == '\r') line.pop_back();
    std::istringstream ss(line);
    std::string a, b, c;
    ss >> a >> b >> c;
    if (a == "format") {
      binary_le = b == "binary_little_endian";
    } else if (a == "element" && b == "vertex") {
      h.count = std::stoll(c);
    } else if (a == "property") {
      if (b != "float") h.float_only = false;
      h.props.push_back(c);
    } else if (a == "end_header") {
      h.data = f.tellg();
      h.ok = binary_le;
      return h;
    }
  }
  return h;
}

int degree_of(const std::vector<std::string>& props, int* bands) {
  int rest = 0;
  for (const auto& p : props)
    if (p.rfind("f_rest_", 0) == 0) ++rest;
  const int k = rest / 3;
  int deg = 0, nb = 0;
  if (k >= 15) deg = 3, nb = 15;
  else if (k >= 8) deg = 2, nb = 8;
  else if (k >= 3) deg = 1, nb = 3;
  if (bands) *bands = nb;
  return deg;
}

}  // namespace

extern "C" {

static int ds_ply_probe_impl(const char* path, int64_t* count, int* sh_degree) {
  if (!path || !count || !sh_degree || !ends_with_ply(path)) return DS_ERR_ARG;
  std::ifstream f(path, std::ios::binary);
  if (!f.is_open()) return DS_ERR_ARG;
  Header h = read_header(f);
  if (!h.ok || !h.float_only || h.count <= 0) return DS_ERR_ARG;
  *count = h.count;
  *sh_degree = degree_of(h.props, nullptr);
  return DS_OK;
}

static int ds_ply_read_impl(const char* path, float* splats, int64_t capacity, int64_t* count,
                int* sh_degree) {
  if (!path || !splats || !count || !sh_degree || !ends_with_ply(path)) return DS_ERR_ARG;
  std::ifstream f(path, std::ios::binary);
  if (!f.is_open()) return DS_ERR_ARG;
  Header h = read_header(f);
  if (!h.ok || !h.float_only || h.count <= 0) return DS_ERR_ARG;
  if (h.count > capacity) return DS_ERR_ARG;
  std::unordered_map<std::string, int> at;
  for (int k = 0; k < (int)h.props.size(); ++k) at[h.props[k]] = k;
  const char* need[14] = {"x",       "y",       "z",       "scale_0", "scale_1",
                          "scale_2", "rot_0",   "rot_1",   "rot_2",   "rot_3",
                          "f_dc_0",  "f_dc_1",  "f_dc_2",  "opacity"};
  const int slot[14] = {kPos,     kPos + 1, kPos + 2, kScale, kScale + 1, kScale + 2, kRot,
                        kRot + 1, kRot + 2, kRot + 3, kDc,    kDc + 1,    kDc + 2,    kLogit};
  int src[14];
  for (int k = 0; k < 14; ++k) {
    auto it = at.find(need[k]);
    if (it == at.end()) return DS_ERR_ARG;
    src[k] = it->second;
  }
  int nb = 0;
  const int deg = degree_of(h.props, &nb);
  std::vector<int> rest(3 * nb, -1);
  for (int b = 0; b < 3 * nb; ++b) {
    auto it = at.find("f_rest_" + std::to_string(b));
    if (it != at.end()) rest[b] = it->second;
  }
  const size_t stride = h.props.size();
  std::vector<float> row(stride);
  for (int64_t i = 0; i < h.count; ++i) {
    if (!f.read(reinterpret_cast<char*>(row.data()), (std::streamsize)(stride * sizeof(float))))
      return DS_ERR_ARG;
    float* g = splats + i * kRec;
    std::fill(g, g + kRec, 0.f);
    for (int k = 0; k < 14; ++k) g[slot[k]] = row[src[k]];
    for (int b = 0; b < 3 * nb; ++b)
      if (rest[b] >= 0) g[kRest + b] = row[rest[b]];
    // OpenCV -> OpenGL: flip y and z, and the quaternion's y and z
    g[kPos + 1] = -g[kPos + 1];
    g[kPos + 2] = -g[kPos + 2];
    g[kRot + 2] = -g[kRot + 2];
    g[kRot + 3] = -g[kRot + 3];
  }
  *count = h.count;
  *sh_degree = deg;
  return DS_OK;
}

static int ds_ply_write_impl(const char* path, const float* splats, int64_t count, int sh_num_bands) {
  if (!path || (!splats && count > 0) || count < 0) return DS_ERR_ARG;
  if (sh_num_bands != 0 && sh_num_bands != 3 && sh_num_bands != 8 && sh_num_bands != 15)
    return DS_ERR_ARG;
  std::ofstream f(path, std::ios::binary);
  if (!f.is_open()) return DS_ERR_ARG;
  const int nr = 3 * sh_num_bands;
  f << "ply\nformat binary_little_endian 1.0\nelement vertex " << count << "\n";
  auto prop = [&](const std::string& name) { f << "property float " << name << "\n"; };
  for (const char* p : {"x", "y", "z", "f_dc_0", "f_dc_1", "f_dc_2"}) prop(p);
  for (int k = 0; k < nr; ++k) prop("f_rest_" + std::to_string(k));
  for (const char* p : {"opacity", "scale_0", "scale_1", "scale_2", "rot_0", "rot_1", "rot_2",
                        "rot_3"})
    prop(p);
  f << "end_header\n";
  std::vector<float> row(14 + nr);
  for (int64_t i = 0; i < count; ++i) {
    const float* g = splats + i * kRec;
    int k = 0;
    row[k++] = g[kPos];
    row[k++] = -g[kPos + 1];
    row[k++] = -g[kPos + 2];
    for (int c = 0; c < 3; ++c) row[k++] = g[kDc + c];
    for (int b = 0; b < nr; ++b) row[k++] = g[kRest + b];
    row[k++] = g[kLogit];
    for (int c = 0; c < 3; ++c) row[k++] = g[kScale + c];
    row[k++] = g[kRot];
    row[k++] = g[kRot + 1];
    row[k++] = -g[kRot + 2];
    row[k++] = -g[kRot + 3];
    f.write(reinterpret_cast<const char*>(row.data()), (std::streamsize)(row.size() * 4));
  }
  return f.good() ? DS_OK : DS_ERR_ARG;
}

int ds_normalize_scene(float* splats, int64_t count, float scene_scale) {
  if ((!splats && count > 0) || count < 0) return DS_ERR_ARG;
  if (count == 0) return DS_OK;
  // centroid with sequential FP32 sums, then the largest |coordinate|
  float c[3] = {0.f, 0.f, 0.f};
  for (int64_t i = 0; i < count; ++i)
    for (int a = 0; a < 3; ++a) c[a] += splats[i * kRec + kPos + a];
  const float inv = 1.f / (float)count;
  for (int a = 0; a < 3; ++a) c[a] *= inv;
  float ext = 0.f;
  for (int64_t i = 0; i < count; ++i)
    for (int a = 0; a < 3; ++a) {
      float& p = splats[i * kRec + kPos + a];
      p -= c[a];
      ext = std::max(ext, std::fabs(p));
    }
  if (ext > 0.f) {
    const float s = scene_scale / ext;
    const float ls = logf(s);
    for (int64_t i = 0; i < count; ++i) {
      for (int a = 0; a < 3; ++a) splats[i * kRec + kPos + a] *= s;
      for (int a = 0; a < 3; ++a) splats[i * kRec + kScale + a] += ls;
    }
  }
  return DS_OK;
}

// C++ exceptions (allocation, malformed numbers) become status codes at the ABI.
int ds_ply_probe(const char* path, int64_t* count, int* sh_degree) {
  try {
    return ds_ply_probe_impl(path, count, sh_degree);
  } catch (const std::bad_alloc&) {
    return DS_ERR_OOM;
  } catch (...) {
    return DS_ERR_ARG;
  }
}

int ds_ply_read(const char* path, float* splats, int64_t capacity, int64_t* count, int* sh_degree) {
  try {
    return ds_ply_read_impl(path, splats, capacity, count, sh_degree);
  } catch (const std::bad_alloc&) {
    return DS_ERR_OOM;
  } catch (...) {
    return DS_ERR_ARG;
  }
}

int ds_ply_write(const char* path, const float* splats, int64_t count, int sh_num_bands) {
  try {
    return ds_ply_write_impl(path, splats, count, sh_num_bands);
  } catch (const std::bad_alloc&) {
    return DS_ERR_OOM;
  } catch (...) {
    return DS_ERR_ARG;
  }
}

}  // extern "C"
