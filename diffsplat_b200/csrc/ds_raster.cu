// Tile rasterizer: per-splat records and tile rectangles, depth-ordered
// deterministic emission of (tile, splat) pairs, tile sort, tile ranges,
// front-to-back compositing and its backward.
//
// Reference behaviour (src/layers/tile_rasterize_layer.cu):
//   tile assignment :52-144, keys :30-38, ranges :148-162,
//   composite forward :192-309, composite backward :356-578.
// Design differences (same results):
//   * Pairs are emitted in (depth, splat id) order at offsets from an exclusive
//     scan instead of atomicAdd slots, then stably sorted by tile id only.  The
//     sorted list therefore equals the reference's 64-bit (tile | depth) order
//     with equal keys in ascending splat id -- deterministic run to run.
//   * The conic is computed once per splat instead of once per (tile, splat).
//   * Each warp covers an 8x4 pixel block and skips splats whose conservative
//     acceptance box misses the block (make_record in ds_common.cuh).
//   * The backward writes one 9-float gradient record per (tile, splat) pair
//     (warp transpose-reduction, then shared-memory accumulation across the
//     CTA) and a per-splat kernel sums each splat's records: no global atomics.
#include <float.h>

#include "ds_common.cuh"
#include "ds_internal.h"

namespace ds {

namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ void count_visible(bool vis, uint32_t* visible) {
  unsigned m = __ballot_sync(0xffffffffu, vis);
  if ((threadIdx.x & 31) == 0 && m) atomicAdd(visible, (uint32_t)__popc(m));
}

// Splat2D SoA -> records / rectangles / counts / depth keys (layer-API path).
__global__ void __launch_bounds__(kThreads)
    prep_splat2d_kernel(ds_splat2d in, int n, int W, int H, int ntx, int nty, float4* ra,
                        float4* rb, float4* rc, float* ridet, ushort4* rect, uint32_t* counts,
                        uint32_t* depth_keys, DevScalars* sc) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) sc->n_splats = (uint32_t)n;
  bool vis = false;
  if (i < n) {
    float x = in.pos_x[i], y = in.pos_y[i], z = in.pos_z[i];
    float cxx = in.cov_xx[i], cxy = in.cov_xy[i], cyy = in.cov_yy[i];
    TileRect r;
    vis = tile_rect(x, y, z, cxx, cxy, cyy, W, H, ntx, nty, r);
    if (vis) {
      Record rec = make_record(x, y, cxx, cxy, cyy, in.color_r[i], in.color_g[i], in.color_b[i],
                               in.opacity[i]);
      ra[i] = rec.a;
      rb[i] = rec.b;
      rc[i] = rec.c;
      ridet[i] = rec.idet;
      rect[i] = make_ushort4(r.x0, r.x1, r.y0, r.y1);
      counts[i] = (uint32_t)((r.x1 - r.x0 + 1) * (r.y1 - r.y0 + 1));
      depth_keys[i] = depth_bits(z);
    } else {
      counts[i] = 0u;
      depth_keys[i] = 0xffffffffu;
    }
  }
  count_visible(vis, &sc->visible);
}

__global__ void __launch_bounds__(kThreads)
    emit_kernel(const uint32_t* __restrict__ perm, const uint32_t* __restrict__ counts,
                const unsigned long long* __restrict__ offsets, const ushort4* __restrict__ rect,
                int n, int ntx, uint32_t cap, uint32_t* __restrict__ tile_keys,
                uint32_t* __restrict__ emit_splat, uint32_t* __restrict__ seg_start) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  uint32_t i = perm[p];
  uint32_t c = counts[i];
  if (c == 0) return;
  unsigned long long off = offsets[p];
  seg_start[i] = (uint32_t)(off < cap ? off : cap);
  if (off >= cap) return;
  ushort4 r = rect[i];
  unsigned long long e = off;
  for (int ty = r.z; ty <= r.w; ++ty) {
    for (int tx = r.x; tx <= r.y; ++tx) {
      if (e >= cap) return;
      tile_keys[e] = (uint32_t)(ty * ntx + tx);
      emit_splat[e] = i;
      ++e;
    }
  }
}

__global__ void __launch_bounds__(kThreads)
    ranges_kernel(const uint32_t* __restrict__ sorted_tile, const uint32_t* __restrict__ n_dev,
                  int tiles, int2* __restrict__ ranges) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= tiles) return;
  const uint32_t n = *n_dev;
  auto lower = [&](uint32_t key) {
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
      uint32_t mid = (lo + hi) >> 1;
      if (sorted_tile[mid] < key) lo = mid + 1;
      else hi = mid;
    }
    return lo;
  };
  uint32_t a = lower((uint32_t)t), b = lower((uint32_t)t + 1u);
  ranges[t] = a < b ? make_int2((int)a, (int)b) : make_int2(0, 0);
}

// Pixel of this thread inside its tile: warp w covers an 8x4 block.
struct PixelMap {
  int i, j;  // row, column
  bool inside;
  float px, py;                    // NDC pixel centre (reference formula)
  float wx_lo, wx_hi, wy_lo, wy_hi;  // extremes of the warp's pixel centres
};

__device__ __forceinline__ PixelMap pixel_map(int tile, int ntx, int W, int H) {
  PixelMap m;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int trow = tile / ntx, tcol = tile - trow * ntx;
  m.i = trow * kTile + (w >> 1) * 4 + (lane >> 3);
  m.j = tcol * kTile + (w & 1) * 8 + (lane & 7);
  m.inside = m.i < H && m.j < W;
  m.px = 2.f * (m.j + 0.5f) / W - 1.f;
  m.py = 1.f - 2.f * (m.i + 0.5f) / H;
  float xl = m.px, xh = m.px, yl = m.py, yh = m.py;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    xl = fminf(xl, __shfl_xor_sync(0xffffffffu, xl, o));
    xh = fmaxf(xh, __shfl_xor_sync(0xffffffffu, xh, o));
    yl = fminf(yl, __shfl_xor_sync(0xffffffffu, yl, o));
    yh = fmaxf(yh, __shfl_xor_sync(0xffffffffu, yh, o));
  }
  m.wx_lo = xl;
  m.wx_hi = xh;
  m.wy_lo = yl;
  m.wy_hi = yh;
  return m;
}

__device__ __forceinline__ bool misses_warp(const float4& a, const PixelMap& m) {
  return a.x + a.z < m.wx_lo || a.x - a.z > m.wx_hi || a.y + a.w < m.wy_lo ||
         a.y - a.w > m.wy_hi;
}

template <bool kLoss>
__global__ void __launch_bounds__(kThreads)
    composite_fwd_kernel(const float4* __restrict__ ra, const float4* __restrict__ rb,
                         const float4* __restrict__ rc, const uint32_t* __restrict__ sorted_splat,
                         const int2* __restrict__ ranges, float* __restrict__ out_rgb,
                         float* __restrict__ out_alpha, int32_t* __restrict__ last_ids, int W,
                         int H, int ntx, const float* __restrict__ target,
                         float* __restrict__ loss_partials, DevScalars* __restrict__ sc) {
  __shared__ float4 sA[kThreads], sB[kThreads], sC[kThreads];
  __shared__ float red[kThreads / 32];
  const int tile = blockIdx.x;
  const PixelMap m = pixel_map(tile, ntx, W, H);
  const int2 range = ranges[tile];
  const int start = range.x, end = range.y;
  float T = 1.f, Cr = 0.f, Cg = 0.f, Cb = 0.f;
  uint32_t cur = 0;
  bool done = !m.inside;
  for (int b0 = start; b0 < end; b0 += kThreads) {
    if (__syncthreads_count(done) >= kThreads) break;
    const int idx = b0 + threadIdx.x;
    if (idx < end) {
      uint32_t g = sorted_splat[idx];
      sA[threadIdx.x] = ra[g];
      sB[threadIdx.x] = rb[g];
      sC[threadIdx.x] = rc[g];
    }
    __syncthreads();
    const int bs = min(kThreads, end - b0);
    if (__any_sync(0xffffffffu, !done)) {
      for (int t = 0; t < bs; ++t) {
        const float4 a = sA[t];
        if (misses_warp(a, m)) continue;
        if (!done) {
          const float4 b = sB[t];
          const float dx = a.x - m.px;
          const float dy = a.y - m.py;
          const float dist2 = dx * dx * b.x + 2.f * dx * dy * b.y + dy * dy * b.z;
          const float sigma = 0.5f * dist2;
          const float4 c = sC[t];
          if (!(sigma < 0.f) && !(sigma > c.w)) {
            const float alpha = fminf(kMaxAlpha, b.w * __expf(-sigma));
            if (!(alpha < kAlphaThres)) {
              const float vis = alpha * T;
              Cr += c.x * vis;
              Cg += c.y * vis;
              Cb += c.z * vis;
              cur = (uint32_t)(b0 + t);
              T = T * (1.f - alpha);
              if (T <= kTThres) done = true;
            }
          }
        }
        if (!__any_sync(0xffffffffu, !done)) break;
      }
    }
  }
  const int pix = m.i * W + m.j;
  float l = 0.f;
  if (m.inside) {
    out_rgb[pix * 3 + 0] = Cr;
    out_rgb[pix * 3 + 1] = Cg;
    out_rgb[pix * 3 + 2] = Cb;
    out_alpha[pix] = 1.f - T;
    last_ids[pix] = (int32_t)cur;
    if (kLoss) {
      const float scale = 1.f / (float)(W * H);
      float dR = Cr - target[pix * 3 + 0];
      float dG = Cg - target[pix * 3 + 1];
      float dB = Cb - target[pix * 3 + 2];
      l = (dR * dR + dG * dG + dB * dB) * scale;
    }
  }
  if (kLoss) {
    l = warp_sum(l);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = l;
    __syncthreads();
    __shared__ bool last;
    if (threadIdx.x == 0) {
      float s = 0.f;
      for (int k = 0; k < kThreads / 32; ++k) s += red[k];
      loss_partials[tile] = s;
      __threadfence();
      last = atomicAdd(&sc->ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (last) {
      // Deterministic final reduction in tile order by the last CTA to finish.
      __threadfence();
      float s = 0.f;
      for (int k = threadIdx.x; k < (int)gridDim.x; k += kThreads) s += ((volatile float*)loss_partials)[k];
      s = warp_sum(s);
      if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
      __syncthreads();
      if (threadIdx.x == 0) {
        float tot = 0.f;
        for (int k = 0; k < kThreads / 32; ++k) tot += red[k];
        sc->loss = tot;
        sc->ticket = 0u;
      }
    }
  }
}

template <bool kFusedLoss, bool kExact>
__global__ void __launch_bounds__(kThreads)
    composite_bwd_kernel(const float4* __restrict__ ra, const float4* __restrict__ rb,
                         const float4* __restrict__ rc, const float* __restrict__ ridet,
                         const uint32_t* __restrict__ sorted_splat,
                         const uint32_t* __restrict__ sorted_emit, const int2* __restrict__ ranges,
                         const float* __restrict__ alphas, const int32_t* __restrict__ last_ids,
                         const float* __restrict__ grad_or_image, const float* __restrict__ target,
                         float* __restrict__ isect_grad, int W, int H, int ntx) {
  __shared__ float4 sA[kThreads], sB[kThreads], sC[kThreads];
  __shared__ float sI[kThreads];
  __shared__ float acc[kThreads * 9];
  const int tile = blockIdx.x;
  const int2 range = ranges[tile];
  const int start = range.x, end = range.y;
  if (end <= start) return;
  const PixelMap m = pixel_map(tile, ntx, W, H);
  const int lane = threadIdx.x & 31;
  const int pix = min(m.i * W + m.j, W * H - 1);
  float T = 1.f - alphas[pix];
  const int32_t bin_final = m.inside ? last_ids[pix] : -1;
  const int32_t warp_final = warp_max(bin_final);
  float gr = 0.f, gg = 0.f, gb = 0.f;
  if (m.inside) {
    if (kFusedLoss) {
      const float scale = 2.f / (float)(W * H);
      gr = scale * (grad_or_image[pix * 3 + 0] - target[pix * 3 + 0]);
      gg = scale * (grad_or_image[pix * 3 + 1] - target[pix * 3 + 1]);
      gb = scale * (grad_or_image[pix * 3 + 2] - target[pix * 3 + 2]);
    } else {
      gr = grad_or_image[pix * 3 + 0];
      gg = grad_or_image[pix * 3 + 1];
      gb = grad_or_image[pix * 3 + 2];
    }
  }
  float accr = 0.f, accg = 0.f, accb = 0.f;
  const int nb = (end - start + kThreads - 1) / kThreads;
  for (int bi = 0; bi < nb; ++bi) {
    const int batch_end = end - 1 - kThreads * bi;
    const int bs = min(kThreads, batch_end + 1 - start);
    __syncthreads();
    const int li = batch_end - (int)threadIdx.x;
    if (li >= start) {
      uint32_t g = sorted_splat[li];
      sA[threadIdx.x] = ra[g];
      sB[threadIdx.x] = rb[g];
      sC[threadIdx.x] = rc[g];
      sI[threadIdx.x] = ridet[g];
    }
#pragma unroll
    for (int k = 0; k < 9; ++k) acc[threadIdx.x * 9 + k] = 0.f;
    __syncthreads();
    const int t_start = max(0, batch_end - warp_final);
    for (int t = t_start; t < bs; ++t) {
      const float4 a = sA[t];
      if (misses_warp(a, m)) continue;
      bool valid = m.inside && (batch_end - t) <= bin_final;
      const float4 b = sB[t];
      float alpha = 0.f, opac = 0.f, g_exp = 0.f, dx = 0.f, dy = 0.f, dist2 = 0.f;
      if (valid) {
        dx = a.x - m.px;
        dy = a.y - m.py;
        dist2 = dx * dx * b.x + 2.f * dx * dy * b.y + dy * dy * b.z;
        const float sigma = 0.5f * dist2;
        if (sigma < 0.f || sigma > sC[t].w) {
          valid = false;
        } else {
          opac = b.w;
          g_exp = __expf(-sigma);
          alpha = fminf(kMaxAlpha, opac * g_exp);
          if (alpha < kAlphaThres) valid = false;
        }
      }
      if (!__any_sync(0xffffffffu, valid)) continue;
      float v[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
      float v_a = 0.f;
      if (valid) {
        const float4 c = sC[t];
        const float T_before = T / fmaxf(1.f - alpha, 1e-6f);
        const float fac = alpha * T_before;
        v[0] = fac * gr;
        v[1] = fac * gg;
        v[2] = fac * gb;
        // Reference recurrence (tile_rasterize_layer.cu:518-521): the colour
        // behind is the sum of absolute weights c_j alpha_j T_j, scaled by
        // T_before.  The exact derivative divides that sum by T_after instead.
        const float ia = kExact ? 1.f / T : 1.f;
        const float v_alpha = T_before * ((c.x - accr * ia) * gr + (c.y - accg * ia) * gg +
                                          (c.z - accb * ia) * gb);
        if (opac * g_exp <= kMaxAlpha) {
          v_a = g_exp * v_alpha;
          const float v_sigma = -opac * g_exp * v_alpha;
          const float v_dist2 = 0.5f * v_sigma;
          const float ddx = 2.f * (dx * b.x + dy * b.y);
          const float ddy = 2.f * (dx * b.y + dy * b.z);
          v[3] = v_dist2 * ddx;
          v[4] = v_dist2 * ddy;
          v[5] = v_dist2 * (-0.25f * ddx * ddx);
          v[7] = v_dist2 * (-0.25f * ddy * ddy);
          v[6] = v_dist2 * (-2.f * b.y * dist2 - 2.f * dx * dy * sI[t]);
        }
        accr += c.x * fac;
        accg += c.y * fac;
        accb += c.z * fac;
        T = T_before;
      }
      // v = {dr, dg, db, dx, dy, dcxx, dcxy, dcyy}; lane 4k ends up with the warp sum of v[k].
      const float s8 = warp_sum8_transposed(v, lane);
      const float sa = warp_sum(v_a);
      if ((lane & 3) == 0) atomicAdd(&acc[t * 9 + (lane >> 2)], s8);
      if (lane == 0) atomicAdd(&acc[t * 9 + 8], sa);
    }
    __syncthreads();
    if (li >= start) {
      const uint32_t e = sorted_emit[li];
      float* dst = isect_grad + (size_t)e * 9;
#pragma unroll
      for (int k = 0; k < 9; ++k) dst[k] = acc[threadIdx.x * 9 + k];
    }
  }
}

// Sums each splat's per-tile gradient records into the Splat2D gradient SoA (accumulating).
__global__ void __launch_bounds__(kThreads)
    reduce_grads_kernel(const float* __restrict__ isect_grad, const uint32_t* __restrict__ seg_start,
                        const uint32_t* __restrict__ counts, uint32_t cap, int n, ds_splat2d gin) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t c = counts[i];
  if (c == 0) return;
  unsigned long long s = seg_start[i];
  unsigned long long e = s + c;
  if (e > cap) e = cap;
  float g[9] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  for (unsigned long long q = s; q < e; ++q) {
    const float* r = isect_grad + q * 9;
#pragma unroll
    for (int k = 0; k < 9; ++k) g[k] += r[k];
  }
  gin.color_r[i] += g[0];
  gin.color_g[i] += g[1];
  gin.color_b[i] += g[2];
  gin.pos_x[i] += g[3];
  gin.pos_y[i] += g[4];
  gin.cov_xx[i] += g[5];
  gin.cov_xy[i] += g[6];
  gin.cov_yy[i] += g[7];
  gin.opacity[i] += g[8];
}

template <typename T>
int alloc(T** p, size_t n) {
  *p = nullptr;
  if (n == 0) n = 1;
  return cuda_status(cudaMalloc((void**)p, n * sizeof(T)));
}

template <typename T>
void release(T*& p) {
  if (p) cudaFree(p);
  p = nullptr;
}

int ceil_log2(int x) {
  int b = 0;
  while ((1 << b) < x) ++b;
  return b;
}

}  // namespace

int raster_alloc(RasterBuffers& rb, int width, int height, int max_splats, int64_t cap) {
  if (width <= 0 || height <= 0 || max_splats < 0) return DS_ERR_ARG;
  if (cap <= 0) cap = (int64_t)1 << 25;
  if (cap > ((int64_t)1 << 31)) return DS_ERR_ARG;
  rb.max_splats = max_splats;
  rb.cap = cap;
  const size_t n = (size_t)max_splats;
  DS_TRY(alloc(&rb.rec_a, n));
  DS_TRY(alloc(&rb.rec_b, n));
  DS_TRY(alloc(&rb.rec_c, n));
  DS_TRY(alloc(&rb.rec_idet, n));
  DS_TRY(alloc(&rb.rect, n));
  DS_TRY(alloc(&rb.counts, n));
  DS_TRY(alloc(&rb.seg_start, n));
  DS_TRY(alloc(&rb.depth_keys, n));
  DS_TRY(alloc(&rb.depth_k0, n));
  DS_TRY(alloc(&rb.depth_k1, n));
  DS_TRY(alloc(&rb.depth_v0, n));
  DS_TRY(alloc(&rb.depth_v1, n));
  DS_TRY(alloc(&rb.emit_offsets, n));
  const size_t c = (size_t)cap;
  DS_TRY(alloc(&rb.tile_k0, c));
  DS_TRY(alloc(&rb.tile_k1, c));
  DS_TRY(alloc(&rb.tile_v0, c));
  DS_TRY(alloc(&rb.tile_v1, c));
  DS_TRY(alloc(&rb.emit_splat, c));
  DS_TRY(alloc(&rb.sorted_splat, c));
  DS_TRY(alloc(&rb.isect_grad, c * 9));
  DS_TRY(alloc(&rb.sort.hist, (size_t)256 * kSortBlocks));
  DS_TRY(alloc(&rb.scan.partials, (size_t)kSortBlocks + 1));
  DS_TRY(alloc(&rb.scalars, 1));
  DS_CUDA(cudaMemset(rb.scalars, 0, sizeof(DevScalars)));
  // Splats that are never visible keep count 0 until the first forward writes them.
  DS_CUDA(cudaMemset(rb.counts, 0, n * sizeof(uint32_t) + (n == 0 ? 4 : 0)));
  return raster_resize(rb, width, height);
}

int raster_resize(RasterBuffers& rb, int width, int height) {
  if (width <= 0 || height <= 0) return DS_ERR_ARG;
  if (width == rb.width && height == rb.height) return DS_OK;
  release(rb.ranges);
  release(rb.alphas);
  release(rb.last_ids);
  release(rb.loss_partials);
  rb.width = width;
  rb.height = height;
  rb.ntx = (width + kTile - 1) / kTile;
  rb.nty = (height + kTile - 1) / kTile;
  rb.tiles = rb.ntx * rb.nty;
  if (rb.ntx > 65535 || rb.nty > 65535) return DS_ERR_ARG;
  const size_t px = (size_t)width * height;
  DS_TRY(alloc(&rb.ranges, (size_t)rb.tiles));
  DS_TRY(alloc(&rb.alphas, px));
  DS_TRY(alloc(&rb.last_ids, px));
  DS_TRY(alloc(&rb.loss_partials, (size_t)rb.tiles));
  DS_CUDA(cudaMemset(rb.ranges, 0, rb.tiles * sizeof(int2)));
  return DS_OK;
}

void raster_free(RasterBuffers& rb) {
  release(rb.rec_a);
  release(rb.rec_b);
  release(rb.rec_c);
  release(rb.rec_idet);
  release(rb.rect);
  release(rb.counts);
  release(rb.seg_start);
  release(rb.depth_keys);
  release(rb.depth_k0);
  release(rb.depth_k1);
  release(rb.depth_v0);
  release(rb.depth_v1);
  release(rb.emit_offsets);
  release(rb.tile_k0);
  release(rb.tile_k1);
  release(rb.tile_v0);
  release(rb.tile_v1);
  release(rb.emit_splat);
  release(rb.sorted_splat);
  release(rb.isect_grad);
  release(rb.sort.hist);
  release(rb.scan.partials);
  release(rb.scalars);
  release(rb.ranges);
  release(rb.alphas);
  release(rb.last_ids);
  release(rb.loss_partials);
  rb.width = rb.height = 0;
}

int raster_prepare_from_splat2d(RasterBuffers& rb, const ds_splat2d& in, cudaStream_t s) {
  const int n = in.count;
  if (n > rb.max_splats) return DS_ERR_ARG;
  DS_CUDA(cudaMemsetAsync(&rb.scalars->visible, 0, sizeof(uint32_t), s));
  const int blocks = n > 0 ? (n + kThreads - 1) / kThreads : 1;
  prep_splat2d_kernel<<<blocks, kThreads, 0, s>>>(in, n, rb.width, rb.height, rb.ntx, rb.nty,
                                                  rb.rec_a, rb.rec_b, rb.rec_c, rb.rec_idet,
                                                  rb.rect, rb.counts, rb.depth_keys, rb.scalars);
  return cuda_status(cudaGetLastError());
}

int raster_build_lists(RasterBuffers& rb, int n, cudaStream_t s, cudaEvent_t* ev) {
  DevScalars* sc = rb.scalars;
  if (n > 0) {
    // 1) depth order of the splats: stable sort of (depth bits, id)
    DS_TRY(radix_sort_pairs(rb.depth_keys, nullptr, rb.depth_k0, rb.depth_v0, rb.depth_k1,
                            rb.depth_v1, &rb.depth_sorted_keys, &rb.depth_perm, &sc->n_splats,
                            (uint32_t)rb.max_splats, 32, nullptr, nullptr, rb.sort, s));
    if (ev) DS_CUDA(cudaEventRecord(ev[0], s));
    // 2) emission offsets in depth order
    DS_TRY(scan_counts_permuted(rb.counts, rb.depth_perm, (uint32_t)n, rb.emit_offsets,
                                &sc->n_isects, &sc->n_isects_raw, (uint32_t)rb.cap, &sc->status,
                                rb.scan, s));
    // 3) emit (tile, emission index) pairs grouped by splat in depth order
    emit_kernel<<<(n + kThreads - 1) / kThreads, kThreads, 0, s>>>(
        rb.depth_perm, rb.counts, rb.emit_offsets, rb.rect, n, rb.ntx, (uint32_t)rb.cap,
        rb.tile_k0, rb.emit_splat, rb.seg_start);
    DS_CUDA(cudaGetLastError());
    if (ev) DS_CUDA(cudaEventRecord(ev[1], s));
    // 4) stable sort by tile id; last pass gathers the splat id of each pair
    DS_TRY(radix_sort_pairs(rb.tile_k0, nullptr, rb.tile_k1, rb.tile_v1, rb.tile_k0, rb.tile_v0,
                            &rb.sorted_tile, &rb.sorted_emit, &sc->n_isects, (uint32_t)rb.cap,
                            ceil_log2(rb.tiles), rb.emit_splat, rb.sorted_splat, rb.sort, s));
  } else {
    DS_CUDA(cudaMemsetAsync(&sc->n_isects, 0, sizeof(uint32_t), s));
    DS_CUDA(cudaMemsetAsync(&sc->n_isects_raw, 0, sizeof(unsigned long long), s));
    rb.sorted_tile = rb.tile_k0;
    rb.sorted_emit = rb.tile_v0;
    if (ev) {
      DS_CUDA(cudaEventRecord(ev[0], s));
      DS_CUDA(cudaEventRecord(ev[1], s));
    }
  }
  // 5) per-tile ranges
  ranges_kernel<<<(rb.tiles + kThreads - 1) / kThreads, kThreads, 0, s>>>(
      rb.sorted_tile, &sc->n_isects, rb.tiles, rb.ranges);
  DS_CUDA(cudaGetLastError());
  if (ev) DS_CUDA(cudaEventRecord(ev[2], s));
  return DS_OK;
}

int raster_composite_forward(RasterBuffers& rb, float* out_rgb, const float* target,
                             cudaStream_t s) {
  if (target) {
    composite_fwd_kernel<true><<<rb.tiles, kThreads, 0, s>>>(
        rb.rec_a, rb.rec_b, rb.rec_c, rb.sorted_splat, rb.ranges, out_rgb, rb.alphas,
        rb.last_ids, rb.width, rb.height, rb.ntx, target, rb.loss_partials, rb.scalars);
  } else {
    composite_fwd_kernel<false><<<rb.tiles, kThreads, 0, s>>>(
        rb.rec_a, rb.rec_b, rb.rec_c, rb.sorted_splat, rb.ranges, out_rgb, rb.alphas,
        rb.last_ids, rb.width, rb.height, rb.ntx, nullptr, nullptr, rb.scalars);
  }
  return cuda_status(cudaGetLastError());
}

int raster_composite_backward(RasterBuffers& rb, const float* image, const float* grad_rgb,
                              const float* target, cudaStream_t s) {
#define DS_BWD_ARGS                                                                              \
  rb.rec_a, rb.rec_b, rb.rec_c, rb.rec_idet, rb.sorted_splat, rb.sorted_emit, rb.ranges,       \
      rb.alphas, rb.last_ids, grad_rgb ? grad_rgb : image, grad_rgb ? nullptr : target,          \
      rb.isect_grad, rb.width, rb.height, rb.ntx
  const bool exact = rb.grad_mode == DS_GRAD_EXACT;
  if (grad_rgb) {
    if (exact)
      composite_bwd_kernel<false, true><<<rb.tiles, kThreads, 0, s>>>(DS_BWD_ARGS);
    else
      composite_bwd_kernel<false, false><<<rb.tiles, kThreads, 0, s>>>(DS_BWD_ARGS);
  } else {
    if (exact)
      composite_bwd_kernel<true, true><<<rb.tiles, kThreads, 0, s>>>(DS_BWD_ARGS);
    else
      composite_bwd_kernel<true, false><<<rb.tiles, kThreads, 0, s>>>(DS_BWD_ARGS);
  }
#undef DS_BWD_ARGS
  return cuda_status(cudaGetLastError());
}

int raster_reduce_grads(RasterBuffers& rb, const ds_splat2d& gin, int n, cudaStream_t s) {
  if (n <= 0) return DS_OK;
  reduce_grads_kernel<<<(n + kThreads - 1) / kThreads, kThreads, 0, s>>>(
      rb.isect_grad, rb.seg_start, rb.counts, (uint32_t)rb.cap, n, gin);
  return cuda_status(cudaGetLastError());
}

}  // namespace ds
