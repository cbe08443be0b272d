// Minimal project-written subset of the glm API (vec3, mat4 with column-major
// storage m[col][row], matrix product, value_ptr, ortho, perspective, lookAt)
// sufficient to compile the reference's sources and tests, whose glm
// submodule is absent.  Conventions: OpenGL right-handed, clip depth -1..1.
// TEST INFRASTRUCTURE: used only to build the reference and its grad_check.
#pragma once
#include <cmath>

namespace glm {

struct vec3 {
  float x = 0.f, y = 0.f, z = 0.f;
  vec3() = default;
  vec3(float a, float b, float c) : x(a), y(b), z(c) {}
  explicit vec3(float s) : x(s), y(s), z(s) {}
  float& operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
  float operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};

inline vec3 operator-(const vec3& a, const vec3& b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline vec3 operator+(const vec3& a, const vec3& b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline vec3 operator*(const vec3& a, float s) { return {a.x * s, a.y * s, a.z * s}; }
inline float dot(const vec3& a, const vec3& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline vec3 cross(const vec3& a, const vec3& b) {
  return {a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y};
}
inline vec3 normalize(const vec3& a) { return a * (1.f / std::sqrt(dot(a, a))); }

struct vec4 {
  float v[4] = {0.f, 0.f, 0.f, 0.f};
  float& operator[](int i) { return v[i]; }
  float operator[](int i) const { return v[i]; }
};

struct mat4 {
  vec4 c[4];  // columns
  mat4() = default;
  explicit mat4(float d) {
    for (int k = 0; k < 4; ++k) c[k][k] = d;
  }
  vec4& operator[](int i) { return c[i]; }
  const vec4& operator[](int i) const { return c[i]; }
};

// (A * B)[col][row] = sum_k A[k][row] * B[col][k]
inline mat4 operator*(const mat4& A, const mat4& B) {
  mat4 R;
  for (int col = 0; col < 4; ++col)
    for (int row = 0; row < 4; ++row)
      R[col][row] = A[0][row] * B[col][0] + A[1][row] * B[col][1] + A[2][row] * B[col][2] +
                    A[3][row] * B[col][3];
  return R;
}

inline mat4 ortho(float l, float r, float b, float t, float n, float f) {
  mat4 M(1.f);
  M[0][0] = 2.f / (r - l);
  M[1][1] = 2.f / (t - b);
  M[2][2] = -2.f / (f - n);
  M[3][0] = -(r + l) / (r - l);
  M[3][1] = -(t + b) / (t - b);
  M[3][2] = -(f + n) / (f - n);
  return M;
}

inline mat4 perspective(float fovy, float aspect, float n, float f) {
  const float th = std::tan(fovy / 2.f);
  mat4 M(0.f);
  M[0][0] = 1.f / (aspect * th);
  M[1][1] = 1.f / th;
  M[2][2] = -(f + n) / (f - n);
  M[2][3] = -1.f;
  M[3][2] = -(2.f * f * n) / (f - n);
  return M;
}

inline mat4 lookAt(const vec3& eye, const vec3& center, const vec3& up) {
  const vec3 fw = normalize(center - eye);
  const vec3 s = normalize(cross(fw, up));
  const vec3 u = cross(s, fw);
  mat4 M(1.f);
  M[0][0] = s.x;
  M[1][0] = s.y;
  M[2][0] = s.z;
  M[0][1] = u.x;
  M[1][1] = u.y;
  M[2][1] = u.z;
  M[0][2] = -fw.x;
  M[1][2] = -fw.y;
  M[2][2] = -fw.z;
  M[3][0] = -dot(s, eye);
  M[3][1] = -dot(u, eye);
  M[3][2] = dot(fw, eye);
  return M;
}

inline const float* value_ptr(const mat4& m) { return &m.c[0].v[0]; }
inline float* value_ptr(mat4& m) { return &m.c[0].v[0]; }

}  // namespace glm
