// FP64 CPU oracle of the diffsplat training path.  TEST INFRASTRUCTURE ONLY:
// used by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg as
// the checker, never by the product path.
//
// A scalar double-precision restatement of the reference's algorithm (the
// reference ships no CPU path):
//   activation   src/layers/gauss_activ_layer.cu:37-170 (fwd), :198-407 (bwd)
//   projection   src/layers/persp_project_layer.cu:40-149 (fwd), :173-267 (bwd)
//   tile assign  src/layers/tile_rasterize_layer.cu:30-38 (keys), :52-144
//   ranges       src/layers/tile_rasterize_layer.cu:148-162
//   composite    src/layers/tile_rasterize_layer.cu:192-309 (fwd), :356-578 (bwd)
//   MSE          src/layers/mse_loss_layer.cu:22-67
//   Adam         src/optimizers/adam.cu:12-73
// with the thresholds of tile_rasterize_layer.cu:18-26 and the SH constants of
// src/utils/sh_consts.h.  Where FP64 and the reference's FP32 arithmetic can
// take different branches (a tile bound within rounding of an integer, an
// alpha within rounding of 1/255, ...), the oracle reports the affected splat or
// pixel as "ambiguous" so tests can exclude exactly those.
//
// Array conventions (all double unless noted, field-major [field][n]):
//   params  : 14 + 3K rows: pos xyz, log-scale xyz, quat wxyz, sh_dc rgb,
//             logit, then sh_rest r (K rows), g (K rows), b (K rows)
//   splat3d : 13 rows: pos xyz, cov xx xy xz yy yz zz, rgb, opacity
//   splat2d : 10 rows: ndc xyz, cov xx xy yy, rgb, opacity
//   image   : [H*W*3] interleaved RGB
#include <algorithm>
#include <array>
#include <atomic>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

namespace {

constexpr int kTile = 16;
constexpr double kMaxAlpha = 0.99f;      // the reference's float constants, widened
constexpr double kAlphaThres = 1.0f / 255.0f;
constexpr double kTThres = 0.0001f;

constexpr double C0 = 0.28209479177387814;
constexpr double C1 = 0.4886025119029199;
constexpr double C2[5] = {1.0925484305920792, -1.0925484305920792, 0.3153915652525200,
                          -1.0925484305920792, 0.5462742152960396};
constexpr double C3[7] = {-0.5900435899266435, 2.8906114426405540, -0.4570457994644658,
                          0.3731763325901154,  -0.4570457994644658, 1.4453057213202770,
                          -0.5900435899266435};

int bands_of(int degree) {
  int n = 0;
  for (int l = 1; l <= degree; ++l) n += 2 * l + 1;
  return n;
}

void sh_basis(int degree, double x, double y, double z, double* Y) {
  if (degree >= 1) {
    Y[0] = C1 * (-y);
    Y[1] = C1 * z;
    Y[2] = C1 * (-x);
  }
  if (degree >= 2) {
    double xx = x * x, yy = y * y, zz = z * z, xy = x * y, yz = y * z, xz = x * z;
    Y[3] = C2[0] * xy;
    Y[4] = C2[1] * yz;
    Y[5] = C2[2] * (2 * zz - xx - yy);
    Y[6] = C2[3] * xz;
    Y[7] = C2[4] * (xx - yy);
    if (degree >= 3) {
      Y[8] = C3[0] * y * (3 * xx - yy);
      Y[9] = C3[1] * xy * z;
      Y[10] = C3[2] * y * (4 * zz - xx - yy);
      Y[11] = C3[3] * z * (2 * zz - 3 * xx - 3 * yy);
      Y[12] = C3[4] * x * (4 * zz - xx - yy);
      Y[13] = C3[5] * z * (xx - yy);
      Y[14] = C3[6] * x * (xx - 3 * yy);
    }
  }
}

struct Quat {
  double w, x, y, z, inv;
};

Quat normalize(double w, double x, double y, double z) {
  double inv = 1.0 / std::sqrt(std::max(w * w + x * x + y * y + z * z, 1e-12));
  return {w * inv, x * inv, y * inv, z * inv, inv};
}

void rot(const Quat& q, double R[3][3]) {
  R[0][0] = 1 - 2 * (q.y * q.y + q.z * q.z);
  R[0][1] = 2 * (q.x * q.y - q.w * q.z);
  R[0][2] = 2 * (q.x * q.z + q.w * q.y);
  R[1][0] = 2 * (q.x * q.y + q.w * q.z);
  R[1][1] = 1 - 2 * (q.x * q.x + q.z * q.z);
  R[1][2] = 2 * (q.y * q.z - q.w * q.x);
  R[2][0] = 2 * (q.x * q.z - q.w * q.y);
  R[2][1] = 2 * (q.y * q.z + q.w * q.x);
  R[2][2] = 1 - 2 * (q.x * q.x + q.y * q.y);
}

void view_dir(const double cam[3], double px, double py, double pz, double v[3]) {
  double dx = cam[0] - px, dy = cam[1] - py, dz = cam[2] - pz;
  double inv = 1.0 / std::sqrt(std::max(dx * dx + dy * dy + dz * dz, 1e-12));
  v[0] = dx * inv;
  v[1] = dy * inv;
  v[2] = dz * inv;
}

double pixel_ndc_x(int j, int W) { return 2.0 * (j + 0.5) / W - 1.0; }
double pixel_ndc_y(int i, int H) { return 1.0 - 2.0 * (i + 0.5) / H; }

// Distance of v to the nearest integer.
double frac_dist(double v) { return std::fabs(v - std::nearbyint(v)); }

template <typename F>
void parallel_for(int n, int threads, F&& fn) {
  if (threads <= 1 || n < 2) {
    for (int i = 0; i < n; ++i) fn(i);
    return;
  }
  std::atomic<int> next{0};
  std::vector<std::thread> pool;
  for (int t = 0; t < threads; ++t)
    pool.emplace_back([&] {
      for (int i; (i = next.fetch_add(1)) < n;) fn(i);
    });
  for (auto& th : pool) th.join();
}

}  // namespace

extern "C" {

int orc_sh_bands(int degree) { return bands_of(degree); }

// ---- activation -----------------------------------------------------------
void orc_activ_forward(int n, int degree, const double* P, const double cam[3], double* S3) {
  const int K = bands_of(degree);
  const int Kp = K;  // rows per channel in P
  for (int i = 0; i < n; ++i) {
    auto p = [&](int f) { return P[(size_t)f * n + i]; };
    for (int k = 0; k < 3; ++k) S3[(size_t)k * n + i] = p(k);
    Quat q = normalize(p(6), p(7), p(8), p(9));
    double R[3][3];
    rot(q, R);
    double s[3] = {std::exp(p(3)), std::exp(p(4)), std::exp(p(5))};
    double M[3][3];
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) M[r][c] = R[r][c] * s[c];
    double C[3][3];
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) C[r][c] = M[r][0] * M[c][0] + M[r][1] * M[c][1] + M[r][2] * M[c][2];
    S3[3 * (size_t)n + i] = C[0][0];
    S3[4 * (size_t)n + i] = C[0][1];
    S3[5 * (size_t)n + i] = C[0][2];
    S3[6 * (size_t)n + i] = C[1][1];
    S3[7 * (size_t)n + i] = C[1][2];
    S3[8 * (size_t)n + i] = C[2][2];
    double v[3];
    view_dir(cam, p(0), p(1), p(2), v);
    double Y[15];
    sh_basis(degree, v[0], v[1], v[2], Y);
    for (int ch = 0; ch < 3; ++ch) {
      double c = p(10 + ch) * C0;
      for (int b = 0; b < K; ++b) c += Y[b] * p(14 + ch * Kp + b);
      S3[(size_t)(9 + ch) * n + i] = std::min(std::max(c + 0.5, 0.0), 1.0);
    }
    S3[12 * (size_t)n + i] = 1.0 / (1.0 + std::exp(-p(13)));
  }
}

// Writes dL/dparams for all 14 + 3K rows (rows beyond the active degree are 0).
void orc_activ_backward(int n, int degree, int K_alloc, const double* P, const double cam[3],
                        const double* S3, const double* G3, double* GP) {
  const int K = bands_of(degree);
  const int rows = 14 + 3 * K_alloc;
  std::memset(GP, 0, sizeof(double) * (size_t)rows * n);
  for (int i = 0; i < n; ++i) {
    auto p = [&](int f) { return P[(size_t)f * n + i]; };
    auto g3 = [&](int f) { return G3[(size_t)f * n + i]; };
    auto gp = [&](int f) -> double& { return GP[(size_t)f * n + i]; };
    for (int k = 0; k < 3; ++k) gp(k) = g3(k);
    Quat q = normalize(p(6), p(7), p(8), p(9));
    double R[3][3];
    rot(q, R);
    double s[3] = {std::exp(p(3)), std::exp(p(4)), std::exp(p(5))};
    double M[3][3];
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) M[r][c] = R[r][c] * s[c];
    // G full-matrix: off-diagonals as stored (already halved upstream).
    double G[3][3] = {{g3(3), g3(4), g3(5)}, {g3(4), g3(6), g3(7)}, {g3(5), g3(7), g3(8)}};
    double dM[3][3];
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) dM[r][c] = 2 * (G[r][0] * M[0][c] + G[r][1] * M[1][c] + G[r][2] * M[2][c]);
    for (int c = 0; c < 3; ++c) gp(3 + c) = (dM[0][c] * R[0][c] + dM[1][c] * R[1][c] + dM[2][c] * R[2][c]) * s[c];
    double dR[3][3];
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) dR[r][c] = dM[r][c] * s[c];
    // dR/dq of the Rodrigues form (unit q).
    const double w = q.w, x = q.x, y = q.y, z = q.z;
    double dqw = 2 * (-z * dR[0][1] + y * dR[0][2] + z * dR[1][0] - x * dR[1][2] - y * dR[2][0] + x * dR[2][1]);
    double dqx = 2 * (y * dR[0][1] + z * dR[0][2] + y * dR[1][0] - 2 * x * dR[1][1] - w * dR[1][2] +
                      z * dR[2][0] + w * dR[2][1] - 2 * x * dR[2][2]);
    double dqy = 2 * (-2 * y * dR[0][0] + x * dR[0][1] + w * dR[0][2] + x * dR[1][0] + z * dR[1][2] -
                      w * dR[2][0] + z * dR[2][1] - 2 * y * dR[2][2]);
    double dqz = 2 * (-2 * z * dR[0][0] - w * dR[0][1] + x * dR[0][2] + w * dR[1][0] - 2 * z * dR[1][1] +
                      y * dR[1][2] + x * dR[2][0] + y * dR[2][1]);
    double dot = dqw * w + dqx * x + dqy * y + dqz * z;
    gp(6) = q.inv * (dqw - dot * w);
    gp(7) = q.inv * (dqx - dot * x);
    gp(8) = q.inv * (dqy - dot * y);
    gp(9) = q.inv * (dqz - dot * z);
    double v[3];
    view_dir(cam, p(0), p(1), p(2), v);
    double Y[15];
    sh_basis(degree, v[0], v[1], v[2], Y);
    for (int ch = 0; ch < 3; ++ch) {
      double col = S3[(size_t)(9 + ch) * n + i];
      double d = (col > 0.0 && col < 1.0) ? g3(9 + ch) : 0.0;
      gp(10 + ch) = d * C0;
      for (int b = 0; b < K; ++b) gp(14 + ch * K_alloc + b) = d * Y[b];
    }
    double sg = S3[12 * (size_t)n + i];
    gp(13) = g3(12) * sg * (1 - sg);
  }
}

// ---- projection -----------------------------------------------------------
// pv column-major pv[col*4+row].  culled[i] = 1 when clip_w <= 0 (then only
// ndc_z = FLT_MAX is meaningful, the rest is written as 0).
void orc_project_forward(int n, const double* S3, const double pv[16], double* S2, int* culled) {
  for (int i = 0; i < n; ++i) {
    auto s = [&](int f) { return S3[(size_t)f * n + i]; };
    double x = s(0), y = s(1), z = s(2);
    double cx = pv[0] * x + pv[4] * y + pv[8] * z + pv[12];
    double cy = pv[1] * x + pv[5] * y + pv[9] * z + pv[13];
    double cz = pv[2] * x + pv[6] * y + pv[10] * z + pv[14];
    double cw = pv[3] * x + pv[7] * y + pv[11] * z + pv[15];
    for (int k = 0; k < 10; ++k) S2[(size_t)k * n + i] = 0.0;
    if (cw <= 0.0) {
      S2[2 * (size_t)n + i] = (double)FLT_MAX;
      culled[i] = 1;
      continue;
    }
    culled[i] = 0;
    S2[0 * (size_t)n + i] = cx / cw;
    S2[1 * (size_t)n + i] = cy / cw;
    S2[2 * (size_t)n + i] = cz / cw;
    double J[2][3];
    for (int k = 0; k < 3; ++k) {
      J[0][k] = (pv[k * 4 + 0] * cw - cx * pv[k * 4 + 3]) / (cw * cw);
      J[1][k] = (pv[k * 4 + 1] * cw - cy * pv[k * 4 + 3]) / (cw * cw);
    }
    double C[3][3] = {{s(3), s(4), s(5)}, {s(4), s(6), s(7)}, {s(5), s(7), s(8)}};
    double JC[2][3];
    for (int r = 0; r < 2; ++r)
      for (int c = 0; c < 3; ++c) JC[r][c] = J[r][0] * C[0][c] + J[r][1] * C[1][c] + J[r][2] * C[2][c];
    auto dot3 = [&](int a, int b) { return JC[a][0] * J[b][0] + JC[a][1] * J[b][1] + JC[a][2] * J[b][2]; };
    S2[3 * (size_t)n + i] = dot3(0, 0);
    S2[4 * (size_t)n + i] = dot3(1, 0);
    S2[5 * (size_t)n + i] = dot3(1, 1);
    for (int k = 0; k < 4; ++k) S2[(size_t)(6 + k) * n + i] = s(9 + k);
  }
}

// exact == 1 adds the dependence of J (hence Cov2D) on the position, which the
// reference's backward leaves out (persp_project_layer.cu:245-260 uses only
// J^T dndc for the position).
void orc_project_backward(int n, const double* S3, const double pv[16], const double* G2,
                          int exact, double* G3) {
  for (int i = 0; i < n; ++i) {
    auto s = [&](int f) { return S3[(size_t)f * n + i]; };
    auto g2 = [&](int f) { return G2[(size_t)f * n + i]; };
    double x = s(0), y = s(1), z = s(2);
    double cx = pv[0] * x + pv[4] * y + pv[8] * z + pv[12];
    double cy = pv[1] * x + pv[5] * y + pv[9] * z + pv[13];
    double cw = pv[3] * x + pv[7] * y + pv[11] * z + pv[15];
    for (int k = 0; k < 13; ++k) G3[(size_t)k * n + i] = 0.0;
    if (cw <= 0.0) continue;
    double J[2][3];
    for (int k = 0; k < 3; ++k) {
      J[0][k] = (pv[k * 4 + 0] * cw - cx * pv[k * 4 + 3]) / (cw * cw);
      J[1][k] = (pv[k * 4 + 1] * cw - cy * pv[k * 4 + 3]) / (cw * cw);
    }
    double H[2][2] = {{g2(3), 0.5 * g2(4)}, {0.5 * g2(4), g2(5)}};
    double D[3][3];
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) {
        double acc = 0;
        for (int r = 0; r < 2; ++r)
          for (int c = 0; c < 2; ++c) acc += J[r][a] * H[r][c] * J[c][b];
        D[a][b] = acc;
      }
    G3[3 * (size_t)n + i] = D[0][0];
    G3[4 * (size_t)n + i] = D[0][1];
    G3[5 * (size_t)n + i] = D[0][2];
    G3[6 * (size_t)n + i] = D[1][1];
    G3[7 * (size_t)n + i] = D[1][2];
    G3[8 * (size_t)n + i] = D[2][2];
    for (int k = 0; k < 3; ++k) G3[(size_t)k * n + i] = g2(0) * J[0][k] + g2(1) * J[1][k];
    for (int k = 0; k < 4; ++k) G3[(size_t)(9 + k) * n + i] = g2(6 + k);
    if (exact) {
      // dL/dJ = 2 H J Sigma;  dJ[r][k]/dp_m = (P[r][k] P[3][m] - P[r][m] P[3][k]) / w^2
      //                                      - 2 J[r][k] P[3][m] / w,  P[r][k] = pv[k*4+r].
      double Sg[3][3] = {{s(3), s(4), s(5)}, {s(4), s(6), s(7)}, {s(5), s(7), s(8)}};
      double dJ[2][3];
      for (int r = 0; r < 2; ++r)
        for (int k = 0; k < 3; ++k) {
          double acc = 0;
          for (int c = 0; c < 2; ++c)
            for (int l = 0; l < 3; ++l) acc += H[r][c] * J[c][l] * Sg[l][k];
          dJ[r][k] = 2 * acc;
        }
      for (int m = 0; m < 3; ++m) {
        double acc = 0;
        for (int r = 0; r < 2; ++r)
          for (int k = 0; k < 3; ++k) {
            double d = (pv[k * 4 + r] * pv[m * 4 + 3] - pv[m * 4 + r] * pv[k * 4 + 3]) / (cw * cw) -
                       2 * J[r][k] * pv[m * 4 + 3] / cw;
            acc += dJ[r][k] * d;
          }
        G3[(size_t)m * n + i] += acc;
      }
    }
  }
}

// ---- tile assignment --------------------------------------------------------
// rect[4*i..] = {x0, x1, y0, y1}; counts[i] = covered tiles (0 when culled).
// ambiguous[i] = 1 when a branch or a floor() is within `tol` of flipping.
void orc_tile_assign(int n, const double* S2, int W, int H, double tol, int32_t* rect,
                     uint32_t* counts, int32_t* ambiguous) {
  const int ntx = (W + kTile - 1) / kTile, nty = (H + kTile - 1) / kTile;
  const double fx = (double)W / kTile, fy = (double)H / kTile;
  const double pixel_ndc = std::max(2.0 / W, 2.0 / H);
  for (int i = 0; i < n; ++i) {
    auto s = [&](int f) { return S2[(size_t)f * n + i]; };
    double x = s(0), y = s(1), z = s(2), cxx = s(3), cxy = s(4), cyy = s(5);
    counts[i] = 0;
    ambiguous[i] = 0;
    rect[4 * i + 0] = 0;
    rect[4 * i + 1] = -1;
    rect[4 * i + 2] = 0;
    rect[4 * i + 3] = -1;
    auto near = [&](double a, double b) { return std::fabs(a - b) <= tol * std::max(1.0, std::fabs(b)); };
    if (near(std::fabs(x), 1.0) || near(std::fabs(y), 1.0) || near(std::fabs(z), 1.0)) ambiguous[i] = 1;
    if (!(std::fabs(x) <= 1.0 && std::fabs(y) <= 1.0 && std::fabs(z) <= 1.0)) continue;
    double det = cxx * cyy - cxy * cxy;
    if (std::fabs(det) <= tol * std::max(cxx * cyy, cxy * cxy)) ambiguous[i] = 1;
    if (!(det > 0.0)) continue;
    double ex = 3.0 * std::sqrt(cxx), ey = 3.0 * std::sqrt(cyy);
    if (near(std::max(ex, ey) * 2.0, pixel_ndc)) ambiguous[i] = 1;
    if (!(std::max(ex, ey) * 2.0 >= pixel_ndc)) continue;
    double v[4] = {(x - ex + 1.0) * 0.5 * fx, (x + ex + 1.0) * 0.5 * fx, (1.0 - (y + ey)) * 0.5 * fy,
                   (1.0 - (y - ey)) * 0.5 * fy};
    for (double t : v)
      if (frac_dist(t) <= tol * std::max(1.0, std::fabs(t))) ambiguous[i] = 1;
    int x0 = std::max((int)std::floor(v[0]), 0), x1 = std::min((int)std::floor(v[1]), ntx - 1);
    int y0 = std::max((int)std::floor(v[2]), 0), y1 = std::min((int)std::floor(v[3]), nty - 1);
    if (x0 <= x1 && y0 <= y1) {
      rect[4 * i + 0] = x0;
      rect[4 * i + 1] = x1;
      rect[4 * i + 2] = y0;
      rect[4 * i + 3] = y1;
      counts[i] = (uint32_t)((x1 - x0 + 1) * (y1 - y0 + 1));
    }
  }
}

// Order-preserving uint32 of the float32 value of z (tile_rasterize_layer.cu:30-38).
uint32_t orc_depth_bits(double z) {
  float f = (float)z;
  uint32_t u;
  std::memcpy(&u, &f, 4);
  return (u >> 31) ? ~u : (u ^ 0x80000000u);
}

// Emits and sorts all (tile, splat) pairs: order by (tile, depth, id).  Writes
// keys (tile << 32 | depth bits of float32 z), ids, and per-tile ranges
// [2*tiles] ({0,0} for empty tiles).  Returns the number of pairs (or -1 when
// more than `cap`).
int64_t orc_build_lists(int n, const double* S2, int W, int H, const int32_t* rect,
                        const uint32_t* counts, int64_t cap, uint64_t* keys, uint32_t* ids,
                        int32_t* ranges) {
  const int ntx = (W + kTile - 1) / kTile, nty = (H + kTile - 1) / kTile;
  struct Pair {
    uint32_t tile;
    double z;
    uint32_t id;
  };
  std::vector<Pair> pairs;
  for (int i = 0; i < n; ++i) {
    if (!counts[i]) continue;
    for (int ty = rect[4 * i + 2]; ty <= rect[4 * i + 3]; ++ty)
      for (int tx = rect[4 * i + 0]; tx <= rect[4 * i + 1]; ++tx)
        pairs.push_back({(uint32_t)(ty * ntx + tx), S2[2 * (size_t)n + i], (uint32_t)i});
  }
  if ((int64_t)pairs.size() > cap) return -1;
  std::stable_sort(pairs.begin(), pairs.end(), [](const Pair& a, const Pair& b) {
    if (a.tile != b.tile) return a.tile < b.tile;
    return a.z < b.z;  // ids ascending within ties: stable over id order
  });
  const int tiles = ntx * nty;
  for (int t = 0; t < 2 * tiles; ++t) ranges[t] = 0;
  for (size_t q = 0; q < pairs.size(); ++q) {
    keys[q] = ((uint64_t)pairs[q].tile << 32) | orc_depth_bits(pairs[q].z);
    ids[q] = pairs[q].id;
    const uint32_t t = pairs[q].tile;
    if (q == 0 || pairs[q - 1].tile != t) ranges[2 * t] = (int32_t)q;
    if (q + 1 == pairs.size() || pairs[q + 1].tile != t) ranges[2 * t + 1] = (int32_t)(q + 1);
  }
  return (int64_t)pairs.size();
}

// ---- composite ----------------------------------------------------------------
// Front-to-back blend.  px_amb[p] = 1 when a threshold test at that pixel is
// within `tol` (relative) of flipping.  last_ids as in the reference: sorted
// list index of the last contributor (0 when none).
void orc_composite_forward(int n, const double* S2, int W, int H, const uint32_t* ids,
                           const int32_t* ranges, double tol, int threads, double* rgb,
                           double* alpha_out, int32_t* last_ids, int32_t* px_amb) {
  const int ntx = (W + kTile - 1) / kTile, nty = (H + kTile - 1) / kTile;
  parallel_for(ntx * nty, threads, [&](int tile) {
    const int trow = tile / ntx, tcol = tile % ntx;
    const int start = ranges[2 * tile], end = ranges[2 * tile + 1];
    for (int ly = 0; ly < kTile; ++ly)
      for (int lx = 0; lx < kTile; ++lx) {
        const int i = trow * kTile + ly, j = tcol * kTile + lx;
        if (i >= H || j >= W) continue;
        const int pix = i * W + j;
        const double px = pixel_ndc_x(j, W), py = pixel_ndc_y(i, H);
        double T = 1.0, C[3] = {0, 0, 0};
        int32_t cur = 0;
        int amb = 0;
        for (int q = start; q < end; ++q) {
          const uint32_t g = ids[q];
          auto s = [&](int f) { return S2[(size_t)f * n + g]; };
          const double cxx = s(3), cxy = s(4), cyy = s(5);
          const double det = cxx * cyy - cxy * cxy;
          const double a = cyy / det, b = -cxy / det, c = cxx / det;
          const double dx = s(0) - px, dy = s(1) - py;
          const double dist2 = dx * dx * a + 2 * dx * dy * b + dy * dy * c;
          const double sigma = 0.5 * dist2;
          if (std::fabs(sigma) <= tol) amb = 1;
          if (sigma < 0.0) continue;
          const double raw = s(9) * std::exp(-sigma);
          if (std::fabs(raw - kMaxAlpha) <= tol * kMaxAlpha) amb = 1;
          const double al = std::min(kMaxAlpha, raw);
          if (std::fabs(al - kAlphaThres) <= tol * kAlphaThres) amb = 1;
          if (al < kAlphaThres) continue;
          const double vis = al * T;
          for (int k = 0; k < 3; ++k) C[k] += s(6 + k) * vis;
          cur = q;
          T = T * (1.0 - al);
          if (std::fabs(T - kTThres) <= tol * kTThres) amb = 1;
          if (T <= kTThres) break;
        }
        for (int k = 0; k < 3; ++k) rgb[(size_t)pix * 3 + k] = C[k];
        alpha_out[pix] = 1.0 - T;
        last_ids[pix] = cur;
        px_amb[pix] = amb;
      }
  });
}

// Backward of orc_composite_forward (tile_rasterize_layer.cu:356-578): reverse
// walk with T_before = T / max(1 - alpha, 1e-6).  Accumulates into G2
// (10 rows; pos_z row untouched).
void orc_composite_backward(int n, const double* S2, int W, int H, const uint32_t* ids,
                            const int32_t* ranges, const double* alpha_fwd,
                            const int32_t* last_ids, const double* grad_rgb, int threads,
                            int exact, double* G2) {
  const int ntx = (W + kTile - 1) / kTile, nty = (H + kTile - 1) / kTile;
  const int tiles = ntx * nty;
  // Per-tile partials then a deterministic merge keeps this thread-safe.
  std::vector<std::vector<std::pair<uint32_t, std::array<double, 9>>>> part(tiles);
  parallel_for(tiles, threads, [&](int tile) {
    const int trow = tile / ntx, tcol = tile % ntx;
    const int start = ranges[2 * tile], end = ranges[2 * tile + 1];
    if (end <= start) return;
    std::vector<std::array<double, 9>> acc(end - start, std::array<double, 9>{});
    for (int ly = 0; ly < kTile; ++ly)
      for (int lx = 0; lx < kTile; ++lx) {
        const int i = trow * kTile + ly, j = tcol * kTile + lx;
        if (i >= H || j >= W) continue;
        const int pix = i * W + j;
        const double px = pixel_ndc_x(j, W), py = pixel_ndc_y(i, H);
        double T = 1.0 - alpha_fwd[pix];
        const int last = last_ids[pix];
        const double gr = grad_rgb[(size_t)pix * 3], gg = grad_rgb[(size_t)pix * 3 + 1],
                     gb = grad_rgb[(size_t)pix * 3 + 2];
        double accum[3] = {0, 0, 0};
        for (int q = std::min(end - 1, last); q >= start; --q) {
          const uint32_t g = ids[q];
          auto s = [&](int f) { return S2[(size_t)f * n + g]; };
          const double cxx = s(3), cxy = s(4), cyy = s(5);
          const double det = cxx * cyy - cxy * cxy;
          const double idet = 1.0 / det;
          const double a = cyy * idet, b = -cxy * idet, c = cxx * idet;
          const double dx = s(0) - px, dy = s(1) - py;
          const double dist2 = dx * dx * a + 2 * dx * dy * b + dy * dy * c;
          const double sigma = 0.5 * dist2;
          if (sigma < 0.0) continue;
          const double op = s(9);
          const double ge = std::exp(-sigma);
          const double al = std::min(kMaxAlpha, op * ge);
          if (al < kAlphaThres) continue;
          const double Tb = T / std::max(1.0 - al, 1e-6);
          const double fac = al * Tb;
          auto& A = acc[q - start];
          A[0] += fac * gr;
          A[1] += fac * gg;
          A[2] += fac * gb;
          const double col[3] = {s(6), s(7), s(8)};
          // The reference accumulates absolute weights c_j alpha_j T_j of the splats
          // behind and multiplies by T_before; the true derivative divides that
          // sum by T_after = T_before (1 - alpha) instead (exact == 1).
          const double sc = exact ? 1.0 / (Tb * std::max(1.0 - al, 1e-6)) : 1.0;
          const double v_alpha = Tb * ((col[0] - accum[0] * sc) * gr + (col[1] - accum[1] * sc) * gg +
                                       (col[2] - accum[2] * sc) * gb);
          if (op * ge <= kMaxAlpha) {
            A[8] += ge * v_alpha;
            const double v_dist2 = 0.5 * (-op * ge * v_alpha);
            const double ddx = 2 * (dx * a + dy * b), ddy = 2 * (dx * b + dy * c);
            A[3] += v_dist2 * ddx;
            A[4] += v_dist2 * ddy;
            A[5] += v_dist2 * (-0.25 * ddx * ddx);
            A[7] += v_dist2 * (-0.25 * ddy * ddy);
            A[6] += v_dist2 * (-2 * b * dist2 - 2 * dx * dy * idet);
          }
          for (int k = 0; k < 3; ++k) accum[k] += col[k] * fac;
          T = Tb;
        }
      }
    for (int q = start; q < end; ++q) part[tile].push_back({ids[q], acc[q - start]});
  });
  // rows of G2: 0 x, 1 y, 2 z, 3 cxx, 4 cxy, 5 cyy, 6 r, 7 g, 8 b, 9 opacity
  const int map[9] = {6, 7, 8, 0, 1, 3, 4, 5, 9};
  for (int t = 0; t < tiles; ++t)
    for (auto& pr : part[t])
      for (int k = 0; k < 9; ++k) G2[(size_t)map[k] * n + pr.first] += pr.second[k];
}

// ---- loss / Adam ------------------------------------------------------------------
double orc_mse_forward(int64_t npix, const double* px, const double* tgt) {
  double s = 0;
  for (int64_t i = 0; i < npix * 3; ++i) s += (px[i] - tgt[i]) * (px[i] - tgt[i]);
  return s / (double)npix;
}

void orc_mse_backward(int64_t npix, const double* px, const double* tgt, double* grad) {
  for (int64_t i = 0; i < npix * 3; ++i) grad[i] = 2.0 / (double)npix * (px[i] - tgt[i]);
}

void orc_adam(int64_t n, double* p, const double* g, double* m, double* v, double lr, double b1,
              double b2, double eps, int step) {
  const double bc1 = 1.0 / (1.0 - std::pow(b1, step)), bc2 = 1.0 / (1.0 - std::pow(b2, step));
  for (int64_t i = 0; i < n; ++i) {
    m[i] = b1 * m[i] + (1 - b1) * g[i];
    v[i] = b2 * v[i] + (1 - b2) * g[i] * g[i];
    p[i] -= lr * (m[i] * bc1) / (std::sqrt(v[i] * bc2) + eps);
  }
}

}  // extern "C"
