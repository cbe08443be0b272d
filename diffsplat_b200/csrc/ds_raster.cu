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
//   * The composite kernels (ds_composite.cu) write one 9-float gradient
//     record per (tile, splat) pair and a warp per splat sums each splat's
//     records here: no global atomics, deterministic gradients.
#include <float.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <vector>

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

// TK: the tile id's type, 16 bits on the counting path (at most
// kCountSortMaxTiles tiles), 32 for the radix passes.
template <typename TK>
__global__ void __launch_bounds__(kThreads)
    emit_kernel(const uint32_t* __restrict__ perm, const uint32_t* __restrict__ counts,
                const unsigned long long* __restrict__ offsets, const ushort4* __restrict__ rect,
                int n, int ntx, uint32_t cap, TK* __restrict__ tile_keys,
                uint32_t* __restrict__ emit_splat, uint32_t* __restrict__ seg_start,
                const uint16_t* __restrict__ inst_of_splat, const InstGeom* __restrict__ geom,
                int2* __restrict__ ranges, int tiles) {
  pdl_wait();
  // The tile ranges of this forward start empty: after the radix tile sort
  // ranges_kernel fills only the non-empty ones (the counting sort's scan
  // writes every tile's).
  for (int64_t q = (int64_t)blockIdx.x * kThreads + threadIdx.x; q < tiles;
       q += (int64_t)gridDim.x * kThreads)
    ranges[q] = make_int2(0, 0);
  // Four lanes (a quad) per splat in depth order: they load its count, offset
  // and tile rectangle and write its tiles (row-major over the rectangle) to
  // consecutive emission slots, four at a time.  Splats with more than
  // kQuadTiles tiles are written by the whole warp instead, one after another,
  // their values broadcast from the quad.  In a batch the tile id is
  // batch-wide: the instance's first tile plus its row-major tile index.
  constexpr uint32_t kQuadTiles = 64;
  const int64_t t = (int64_t)blockIdx.x * kThreads + threadIdx.x;
  const int lane = threadIdx.x & 31, q = lane & 3;
  if ((t - lane) / 4 >= n) return;  // uniform per warp
  const int p = (int)(t / 4);
  uint32_t i = 0, m = 0, x0 = 0, w = 1, y0 = 0, base = 0, pitch = (uint32_t)ntx;
  unsigned long long off = 0;
  if (p < n) {
    i = perm[p];
    const uint32_t c = counts[i];
    if (c) {
      off = offsets[p];
      if (q == 0) seg_start[i] = (uint32_t)(off < cap ? off : cap);
      if (off < cap) {
        unsigned long long end = off + c;
        if (end > cap) end = cap;
        m = (uint32_t)(end - off);
        const ushort4 r = rect[i];
        x0 = r.x;
        w = (uint32_t)(r.y - r.x + 1);
        y0 = r.z;
        if (geom) {
          const InstGeom g = geom[inst_of_splat[i]];
          base = (uint32_t)g.tile_off;
          pitch = (uint32_t)g.ntx;
        }
      }
    }
  }
  // Row of entry k of a rectangle wd tiles wide: a float estimate from the
  // reciprocal (off by at most a few for k < 2^24), stepped to the exact
  // floor(k / wd).
  auto row_of = [](uint32_t k, uint32_t wd, float inv) {
    uint32_t r = (uint32_t)((float)k * inv);
    while (r > 0u && r * wd > k) --r;
    while ((r + 1u) * wd <= k) ++r;
    return r;
  };
  if (m > 0 && m <= kQuadTiles) {
    const float inv = 1.f / (float)w;
    const uint32_t row0 = base + y0 * pitch + x0;
    for (uint32_t k = q; k < m; k += 4) {
      const uint32_t ty = row_of(k, w, inv);
      tile_keys[off + k] = (TK)(row0 + ty * pitch + (k - ty * w));
      emit_splat[off + k] = i;
    }
  }
  uint32_t todo = __ballot_sync(0xffffffffu, q == 0 && m > kQuadTiles);
  const bool batch = geom != nullptr;  // uniform
  while (todo) {
    const int src = __ffs(todo) - 1;
    todo &= todo - 1u;
    const uint32_t sm = __shfl_sync(0xffffffffu, m, src);
    const uint32_t soff = __shfl_sync(0xffffffffu, (uint32_t)off, src);  // off < cap < 2^32
    const uint32_t si = __shfl_sync(0xffffffffu, i, src);
    const uint32_t sx = __shfl_sync(0xffffffffu, x0, src);
    const uint32_t sw = __shfl_sync(0xffffffffu, w, src);
    const uint32_t sy = __shfl_sync(0xffffffffu, y0, src);
    uint32_t sb = 0, sp = pitch;
    if (batch) {
      sb = __shfl_sync(0xffffffffu, base, src);
      sp = __shfl_sync(0xffffffffu, pitch, src);
    }
    const float sinv = 1.f / (float)sw;
    const uint32_t row0 = sb + sy * sp + sx;
    for (uint32_t k = lane; k < sm; k += 32) {
      const uint32_t ty = row_of(k, sw, sinv);
      tile_keys[soff + k] = (TK)(row0 + ty * sp + (k - ty * sw));
      emit_splat[soff + k] = si;
    }
  }
}

// Sums each splat's per-tile gradient records, which are contiguous in
// emission order.  One thread per splat with at most kSerialRecords tiles sums
// them in record order; a fixed grid of warps takes the splats on the
// emission scan's long list one per warp (grid-stride).  Each splat is summed
// by exactly one thread or warp in a fixed order.  kAccumulate adds the sums into a Splat2D gradient SoA (layer
// API); otherwise they are written to g2[k * n + i], k = {r, g, b, ndc x,
// ndc y, cov xx, cov xy, cov yy, opacity}.
constexpr int kLongWarps = 148 * 256;  // enough for one long segment per warp in typical scenes

template <bool kAccumulate>
__device__ __forceinline__ void store_g2(int k, uint32_t i, int n, float v, float* g2,
                                         const ds_splat2d& gin) {
  if (kAccumulate) {
    float* dst = k == 0 ? gin.color_r : k == 1 ? gin.color_g : k == 2 ? gin.color_b
               : k == 3 ? gin.pos_x : k == 4 ? gin.pos_y : k == 5 ? gin.cov_xx
               : k == 6 ? gin.cov_xy : k == 7 ? gin.cov_yy : gin.opacity;
    dst[i] += v;
  } else {
    g2[(size_t)k * n + i] = v;
  }
}

__device__ __forceinline__ void segment_of(const uint32_t* __restrict__ perm,
                                           const unsigned long long* __restrict__ offsets,
                                           const uint32_t* __restrict__ counts, uint32_t cap,
                                           int p, uint32_t& i, uint32_t& c,
                                           unsigned long long& s, unsigned long long& e) {
  i = perm[p];
  c = counts[i];
  s = e = 0;
  if (c) {
    s = offsets[p];
    e = s + c;
    if (e > cap) e = cap;
    if (s > e) s = e;
  }
}

template <bool kAccumulate>
__global__ void __launch_bounds__(kThreads)
    segment_reduce_short_kernel(const float* __restrict__ isect_grad,
                                const uint32_t* __restrict__ perm,
                                const unsigned long long* __restrict__ offsets,
                                const uint32_t* __restrict__ counts, uint32_t cap, int n,
                                float* __restrict__ g2, ds_splat2d gin, GradSegments seg) {
  const int p = (int)(blockIdx.x * (int64_t)kThreads + threadIdx.x);
  if (p >= n) return;
  uint32_t i, c;
  unsigned long long s, e;
  segment_of(perm, offsets, counts, cap, p, i, c, s, e);
  if (c > kSerialRecords || (kAccumulate && c == 0)) return;
  float v[9] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  if (e > s) {
    const ushort4 rc = seg.rect[i];
    const uint32_t w = (uint32_t)(rc.y - rc.x + 1);
    uint32_t row0, pitch;
    seg_origin(seg, i, rc, row0, pitch);
    const unsigned long long key = seg_key(seg, i);
    uint32_t tx = 0, trow = row0;
    for (unsigned long long q = s; q < e; ++q) {
      if (key < seg.tile_bound[trow + tx]) {
        const float* r = isect_grad + q * 9;
#pragma unroll
        for (int k = 0; k < 9; ++k) v[k] += r[k];
      }
      if (++tx == w) {
        tx = 0;
        trow += pitch;
      }
    }
  }
#pragma unroll
  for (int k = 0; k < 9; ++k) store_g2<kAccumulate>(k, i, n, v[k], g2, gin);
}

template <bool kAccumulate>
__global__ void __launch_bounds__(kThreads)
    segment_reduce_long_kernel(const float* __restrict__ isect_grad, int n,
                               float* __restrict__ g2, ds_splat2d gin,
                               const uint4* __restrict__ long_list,
                               DevScalars* __restrict__ sc, GradSegments sg) {
  pdl_wait();
  const int lane = threadIdx.x & 31;
  const uint32_t total = sc->n_long;
  for (uint32_t w = (uint32_t)((blockIdx.x * (int64_t)kThreads + threadIdx.x) >> 5); w < total;
       w += (uint32_t)(gridDim.x * (kThreads / 32))) {
    const uint4 seg = long_list[w];
    const uint32_t i = seg.x;
    const unsigned long long s = seg.y, e = seg.z;
    float v[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    float a = 0.f;
    const ushort4 rc = sg.rect[i];
    const uint32_t wd = (uint32_t)(rc.y - rc.x + 1);
    uint32_t row0, pitch;
    seg_origin(sg, i, rc, row0, pitch);
    const unsigned long long key = seg_key(sg, i);
    // record q is tile k = q - first of the row-major rectangle; lanes step by
    // 32 = 32 / wd rows and 32 % wd columns
    const uint32_t first = sg.start[i];
    uint32_t ty = 0, tx = 0;
    if (s + lane < e) {
      const uint32_t k = (uint32_t)(s + lane - first);
      ty = k / wd;
      tx = k - ty * wd;
    }
    const uint32_t dy = 32u / wd, dx = 32u - dy * wd;
    for (unsigned long long q = s + lane; q < e; q += 32) {
      if (key < sg.tile_bound[row0 + ty * pitch + tx]) {
        const float* r = isect_grad + q * 9;
#pragma unroll
        for (int k = 0; k < 8; ++k) v[k] += r[k];
        a += r[8];
      }
      ty += dy;
      tx += dx;
      if (tx >= wd) {
        tx -= wd;
        ++ty;
      }
    }
    const float s8 = warp_sum8_transposed(v, lane);
    const float sa = warp_sum(a);
    if ((lane & 3) == 0) store_g2<kAccumulate>(lane >> 2, i, n, s8, g2, gin);
    if (lane == 0) store_g2<kAccumulate>(8, i, n, sa, g2, gin);
  }
  (void)n;
}

template <bool kAccumulate>
int launch_long_reduce(RasterBuffers& rb, int n, const ds_splat2d& gin, cudaStream_t s) {
  const int64_t warps = std::min<int64_t>(n, kLongWarps);
  const unsigned blocks = (unsigned)((warps * 32 + kThreads - 1) / kThreads);
  DS_CUDA(launch_pdl(segment_reduce_long_kernel<kAccumulate>, dim3(blocks), dim3(kThreads), 0, s,
                     rb.isect_grad, n, rb.g2, gin, rb.long_list, rb.scalars, grad_segments(rb)));
  return cuda_status(cudaGetLastError());
}

__global__ void __launch_bounds__(kThreads)
    ranges_kernel(const uint32_t* __restrict__ sorted_tile, const uint32_t* __restrict__ n_dev,
                  int* __restrict__ ranges, uint32_t tiles, uint32_t* __restrict__ status) {
  pdl_wait();
  // ranges[t] = [first, last + 1) of tile t in the sorted pairs, from the
  // boundaries between neighbouring ids (grid-stride; the ranges of tiles with
  // no pair stay (0, 0) from the memset before).
  const uint32_t n = *n_dev;
  for (uint32_t q = blockIdx.x * kThreads + threadIdx.x; q < n; q += gridDim.x * kThreads) {
    const uint32_t t = sorted_tile[q];
    if (t >= tiles) {  // self-check: never for a correct sort; no write outside ranges
      atomicOr(status, kStatusBadTile);
      continue;
    }
    if (q == 0 || sorted_tile[q - 1] != t) ranges[2 * (size_t)t] = (int)q;
    if (q + 1 == n || sorted_tile[q + 1] != t) ranges[2 * (size_t)t + 1] = (int)(q + 1);
  }
}

// ---- stable counting sort of the pairs by tile --------------------------------
// The emission lays the pairs out grouped by splat in (depth, id) order; a
// stable partition by tile id gives each tile's list in that order, which is
// the reference's 64-bit (tile | depth) key order with equal keys by id.
// The n pairs are split into count_chunks contiguous chunks (one CTA each,
// split again into contiguous warp runs):
//   tile_count_kernel   per chunk, pairs per tile -> hist[chunk][tile]
//   tile_offsets_kernel per tile, exclusive prefix of hist over the chunks
//                       (in place) and the total; the last CTA to finish
//                       scans the totals into the tile ranges and orders
//                       the tiles for the composite (longest first)
//   tile_scatter_kernel per chunk, each warp ranks its run in order (match
//                       over the lanes' tile ids) and writes every pair's
//                       splat id to range start + chunk prefix + warp
//                       prefix + rank.  (The composite backward finds a
//                       pair's emission index from the splat's first one and
//                       the tile's place in its rectangle, so none is stored.)
// One pass over the pairs instead of ceil(log2 T / 8) radix passes, and the
// ranges come out of the scan.
constexpr int kOffsetThreads = 1024;  // 32 tiles x 32 slices of the chunk column

__device__ __forceinline__ void chunk_of(uint32_t n, uint32_t chunks, uint32_t c, uint32_t& lo,
                                         uint32_t& hi) {
  const uint32_t per = (n + chunks - 1) / chunks;
  lo = min(n, c * per);
  hi = min(n, lo + per);
}

__global__ void __launch_bounds__(kThreads)
    tile_count_kernel(const uint16_t* __restrict__ tile_keys, const uint32_t* __restrict__ n_dev,
                      int tiles, uint32_t* __restrict__ hist, uint32_t* __restrict__ status) {
  pdl_wait();
  extern __shared__ uint32_t cnt[];  // [tiles]
  for (int t = threadIdx.x; t < tiles; t += kThreads) cnt[t] = 0u;
  __syncthreads();
  uint32_t lo, hi;
  chunk_of(*n_dev, gridDim.x, blockIdx.x, lo, hi);
  // loads in flight per thread (4 of them: tile sort 0.0806 vs 0.0788 ms at
  // step 25 of the 1280x720 / 60000-splat fit, B200)
  constexpr int kAhead = 8;
  for (uint32_t e0 = lo + threadIdx.x; e0 < hi; e0 += kThreads * kAhead) {
    uint32_t tk[kAhead];
#pragma unroll
    for (int u = 0; u < kAhead; ++u) {
      const uint32_t e = e0 + u * kThreads;
      tk[u] = e < hi ? (uint32_t)tile_keys[e] : 0xfffffffeu;
    }
#pragma unroll
    for (int u = 0; u < kAhead; ++u) {
      if (tk[u] < (uint32_t)tiles) atomicAdd(&cnt[tk[u]], 1u);
      else if (tk[u] != 0xfffffffeu) atomicOr(status, kStatusBadTile);  // never when correct
    }
  }
  __syncthreads();
  uint32_t* row = hist + (size_t)blockIdx.x * tiles;
  for (int t = threadIdx.x; t < tiles; t += kThreads) row[t] = cnt[t];
}

__device__ void order_tiles(const int2* __restrict__ ranges, int tiles, int32_t* __restrict__ order);

__global__ void __launch_bounds__(kOffsetThreads)
    tile_offsets_kernel(uint32_t* __restrict__ hist, int chunks, int tiles,
                        uint32_t* __restrict__ totals, int2* __restrict__ ranges,
                        DevScalars* __restrict__ sc, int32_t* __restrict__ order) {
  pdl_wait();
  constexpr int kSlices = kOffsetThreads / 32;
  __shared__ uint32_t part[kSlices][33];
  __shared__ uint32_t wsum[kSlices];
  __shared__ bool last;
  const int lane = threadIdx.x & 31, s = threadIdx.x >> 5;
  const int t = blockIdx.x * 32 + lane;
  const int r0 = s * chunks / kSlices, r1 = (s + 1) * chunks / kSlices;
  uint32_t sum = 0;
  if (t < tiles) {
#pragma unroll 4
    for (int r = r0; r < r1; ++r) sum += hist[(size_t)r * tiles + t];
  }
  part[s][lane] = sum;
  __syncthreads();
  uint32_t run = 0;
  for (int k = 0; k < s; ++k) run += part[k][lane];
  if (t < tiles) {
    for (int r = r0; r < r1; ++r) {
      const size_t q = (size_t)r * tiles + t;
      const uint32_t v = hist[q];
      hist[q] = run;
      run += v;
    }
    if (s == kSlices - 1) totals[t] = run;
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(&sc->sort_ticket, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  // Last CTA: exclusive scan of the totals into the ranges; each thread takes
  // a contiguous run of tiles.
  const int per = (tiles + kOffsetThreads - 1) / kOffsetThreads;
  const int a = min(tiles, threadIdx.x * per), b = min(tiles, a + per);
  uint32_t mine = 0;
  for (int k = a; k < b; ++k) mine += ((volatile uint32_t*)totals)[k];
  uint32_t incl = mine;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += v;
  }
  if (lane == 31) wsum[s] = incl;
  __syncthreads();
  if (s == 0) {
    const uint32_t w = wsum[lane];
    uint32_t wi = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t v = __shfl_up_sync(0xffffffffu, wi, o);
      if (lane >= o) wi += v;
    }
    wsum[lane] = wi - w;  // exclusive over the warps
  }
  __syncthreads();
  uint32_t base = incl - mine + wsum[s];
  for (int k = a; k < b; ++k) {
    const uint32_t c = ((volatile uint32_t*)totals)[k];
    ranges[k] = c ? make_int2((int)base, (int)(base + c)) : make_int2(0, 0);
    base += c;
  }
  if (threadIdx.x == 0) sc->sort_ticket = 0u;
  if (order) {
    // the longest-first composite schedule from the ranges just written
    __syncthreads();
    order_tiles(ranges, tiles, order);
  }
}

// kScatterWarps warps per CTA; dynamic shared memory 4 tiles + 2 kScatterWarps
// tp B (tp = tiles rounded up to even): the tiles' bases and each warp's
// 16-bit offsets inside the chunk, a warp's row padded to whole 32-bit words
// so that its counts can be taken by 32-bit shared atomics on pairs of them
// (a run has at most 8192 pairs, so a count never carries into its
// neighbour).  Counting with atomics instead of ranking equal tiles with
// __match_any_sync: tile sort 0.081 -> 0.058 ms at step 25 of the 1280x720 /
// 60000-splat fit (B200); the scatter itself needs the in-order ranks.  A
// chunk of more than 65535 pairs (only when the live pair count exceeds
// kSortBlocks * 65535) does not fit 16-bit offsets: warp 0 then walks the
// whole chunk alone with 32-bit counters in the same shared memory.
constexpr int kScatterWarps = 8;
constexpr uint32_t kScatterChunk16 = 65535;

__global__ void __launch_bounds__(32 * kScatterWarps)
    tile_scatter_kernel(const uint16_t* __restrict__ tile_keys,
                        const uint32_t* __restrict__ emit_splat, const uint32_t* __restrict__ n_dev,
                        int tiles, const uint32_t* __restrict__ hist,
                        const int2* __restrict__ ranges, uint32_t* __restrict__ sorted_splat) {
  pdl_wait();
  extern __shared__ uint32_t smem[];
  constexpr int NT = 32 * kScatterWarps;
  uint32_t* base = smem;                                         // [tiles]
  const int tp = (tiles + 1) & ~1;  // warp rows padded to whole 32-bit words
  uint16_t* woff = reinterpret_cast<uint16_t*>(smem + tiles);   // [warps][tp]
  uint32_t* wide = smem + tiles;                                 // [tiles] (large chunks)
  uint32_t lo, hi;
  chunk_of(*n_dev, gridDim.x, blockIdx.x, lo, hi);
  if (lo >= hi) return;  // uniform
  const bool big = hi - lo > kScatterChunk16;  // uniform
  const int warps = big ? 1 : kScatterWarps;
  const uint32_t* prefix = hist + (size_t)blockIdx.x * tiles;
  for (int t = threadIdx.x; t < tiles; t += NT) base[t] = (uint32_t)ranges[t].x + prefix[t];
  if (big) {
    for (int t = threadIdx.x; t < tiles; t += NT) wide[t] = 0u;
  } else {
    for (int q = threadIdx.x; q < kScatterWarps * tp / 2; q += NT) wide[q] = 0u;
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const uint32_t lt = (1u << lane) - 1u;
  const uint32_t per = (hi - lo + warps - 1) / warps;
  const uint32_t wlo = w < warps ? min(hi, lo + w * per) : hi, whi = min(hi, wlo + per);
  uint16_t* mine = woff + (size_t)w * tp;
  // The run is walked kAhead warp-steps at a time with all their loads issued
  // first: the steps depend on one another only through the shared counters.
  constexpr int kAhead = 8;
  if (!big) {
    // 1) pairs per tile in this warp's run
    for (uint32_t e0 = wlo; e0 < whi; e0 += 32 * kAhead) {
      uint32_t tk[kAhead];
#pragma unroll
      for (int u = 0; u < kAhead; ++u) {
        const uint32_t e = e0 + 32 * u + lane;
        tk[u] = e < whi ? (uint32_t)tile_keys[e] : 0xffffffffu;
      }
      uint32_t* mine32 = reinterpret_cast<uint32_t*>(mine);
#pragma unroll
      for (int u = 0; u < kAhead; ++u) {
        const uint32_t t = tk[u];
        if (t < (uint32_t)tiles) atomicAdd(&mine32[t >> 1], 1u << ((t & 1u) * 16u));
      }
    }
    __syncthreads();
    // 2) exclusive prefix over the warps, per tile (at most the chunk size)
    for (int t = threadIdx.x; t < tiles; t += NT) {
      uint32_t run = 0;
#pragma unroll
      for (int k = 0; k < kScatterWarps; ++k) {
        const uint32_t c = woff[(size_t)k * tp + t];
        woff[(size_t)k * tp + t] = (uint16_t)run;
        run += c;
      }
    }
    __syncthreads();
  }
  // 3) each pair to its slot, in order
  for (uint32_t e0 = wlo; e0 < whi; e0 += 32 * kAhead) {
    uint32_t tk[kAhead], sp[kAhead];
#pragma unroll
    for (int u = 0; u < kAhead; ++u) {
      const uint32_t e = e0 + 32 * u + lane;
      tk[u] = e < whi ? (uint32_t)tile_keys[e] : 0xffffffffu;
      sp[u] = e < whi ? emit_splat[e] : 0u;
    }
#pragma unroll
    for (int u = 0; u < kAhead; ++u) {
      const uint32_t t = tk[u];
      const bool valid = t < (uint32_t)tiles;  // false past the run's end
      if (__all_sync(0xffffffffu, sp[u] == __shfl_sync(0xffffffffu, sp[u], 0))) {
        // all 32 pairs of the step come from one splat, whose tiles are
        // distinct: each pair is the first of its tile here, no ranking is
        // needed (most steps, the pairs being grouped by splat; tile sort
        // 0.058 -> 0.054 ms at step 25 of the 1280x720 / 60000-splat fit)
        if (valid) {
          uint32_t p;
          if (big) {
            p = base[t] + wide[t];
            wide[t] += 1u;
          } else {
            p = base[t] + mine[t];
            mine[t] = (uint16_t)(mine[t] + 1u);
          }
          sorted_splat[p] = sp[u];
        }
      } else {
        const uint32_t peers = __match_any_sync(0xffffffffu, t);
        const int leader = __ffs(peers) - 1;
        uint32_t p0 = 0;
        if (valid && lane == leader) {
          const uint32_t n_peers = (uint32_t)__popc(peers);
          if (big) {
            p0 = base[t] + wide[t];
            wide[t] += n_peers;
          } else {
            p0 = base[t] + mine[t];
            mine[t] = (uint16_t)(mine[t] + n_peers);
          }
        }
        p0 = __shfl_sync(0xffffffffu, p0, leader);
        if (valid) sorted_splat[p0 + __popc(peers & lt)] = sp[u];
      }
      __syncwarp();
    }
  }
}

// Longest-first schedule of the composite CTAs: tiles bucketed by their list
// length (quarter-octave buckets), buckets in descending order.  The heaviest
// tiles start in the first wave, so they no longer set the kernel's tail.  The
// order inside a bucket is arbitrary (plain shared atomics hand out the
// slots); every tile's result is independent of it.
constexpr int kOrderBuckets = 128;

__device__ __forceinline__ int work_bucket(int2 r) {
  const uint32_t len = (uint32_t)max(r.y - r.x, 0);
  if (len == 0) return 0;
  const int l = 31 - __clz(len);
  const uint32_t sub = l >= 2 ? (len >> (l - 2)) & 3u : (len << (2 - l)) & 3u;
  return min(kOrderBuckets - 1, 1 + 4 * l + (int)sub);
}

// The schedule of tiles [0, tiles) from their ranges, by one 1024-thread CTA.
__device__ void order_tiles(const int2* __restrict__ ranges, int tiles, int32_t* __restrict__ order) {
  __shared__ uint32_t cnt[kOrderBuckets];
  __shared__ uint32_t off[kOrderBuckets];
  for (int b = threadIdx.x; b < kOrderBuckets; b += blockDim.x) cnt[b] = 0u;
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int rounds = (tiles + (int)blockDim.x - 1) / (int)blockDim.x;
  for (int r = 0; r < rounds; ++r) {
    const int t = r * blockDim.x + threadIdx.x;
    if (t < tiles) atomicAdd(&cnt[work_bucket(ranges[t])], 1u);
  }
  __syncthreads();
  if (threadIdx.x < 32) {
    // lane l owns buckets 127-4l .. 124-4l (descending); exclusive scan over lanes
    uint32_t v[4], s = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      v[k] = cnt[kOrderBuckets - 1 - 4 * lane - k];
      s += v[k];
    }
    uint32_t incl = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    uint32_t run = incl - s;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      off[kOrderBuckets - 1 - 4 * lane - k] = run;
      run += v[k];
    }
  }
  __syncthreads();
  for (int r = 0; r < rounds; ++r) {
    const int t = r * blockDim.x + threadIdx.x;
    if (t < tiles) order[atomicAdd(&off[work_bucket(ranges[t])], 1u)] = t;
  }
}

__global__ void __launch_bounds__(1024)
    tile_order_kernel(const int2* __restrict__ ranges, int tiles, int32_t* __restrict__ order) {
  pdl_wait();
  order_tiles(ranges, tiles, order);
}

template <typename T>
int alloc(T** p, size_t n) {
  *p = nullptr;
  if (n == 0) n = 1;
  return cuda_status(ds::device_alloc((void**)p, n * sizeof(T)));
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

static int raster_alloc_splats(RasterBuffers& rb, int max_splats, int64_t cap) {
  if (cap <= 0) cap = (int64_t)1 << 25;
  if (cap > ((int64_t)1 << 31)) return DS_ERR_ARG;
  rb.max_splats = max_splats;
  rb.cap = cap;
  rb.ppt = composite_default_ppt();
  rb.ppt_bwd = composite_default_ppt_bwd();
  rb.schedule = composite_longest_first() ? DS_SCHEDULE_LONGEST_FIRST : DS_SCHEDULE_RASTER;
  const size_t n = (size_t)max_splats;
  DS_TRY(alloc(&rb.rec_a, n));
  DS_TRY(alloc(&rb.rec_b, n));
  DS_TRY(alloc(&rb.rec_c, n));
  DS_TRY(alloc(&rb.rec_idet, n));
  DS_TRY(alloc(&rb.rect, n));
  DS_TRY(alloc(&rb.counts, n));
  DS_TRY(alloc(&rb.seg_start, n));
  DS_TRY(alloc(&rb.long_list, n));
  DS_TRY(alloc(&rb.depth_keys, n));
  DS_TRY(alloc(&rb.depth_k0, n));
  DS_TRY(alloc(&rb.depth_k1, n));
  DS_TRY(alloc(&rb.depth_v0, n));
  DS_TRY(alloc(&rb.depth_v1, n));
  DS_TRY(alloc(&rb.emit_offsets, n));
  DS_TRY(alloc(&rb.g2, n * 9));
  const size_t c = (size_t)cap;
  DS_TRY(alloc(&rb.tile_k0, c));
  DS_TRY(alloc(&rb.tile_k1, c));
  DS_TRY(alloc(&rb.tile_v0, c));
  DS_TRY(alloc(&rb.tile_v1, c));
  DS_TRY(alloc(&rb.emit_splat, c));
  DS_TRY(alloc(&rb.sorted_splat, c));
  DS_TRY(alloc(&rb.isect_grad, c * 9));
  DS_TRY(alloc(&rb.sort.hist, (size_t)256 * (kSortBlocks + 1)));
  DS_TRY(alloc(&rb.scan.partials, (size_t)kSortBlocks + 1));
  DS_TRY(alloc(&rb.scan.long_partials, (size_t)kSortBlocks));
  DS_TRY(alloc(&rb.scalars, 1));
  DS_CUDA(cudaMemset(rb.scalars, 0, sizeof(DevScalars)));
  // Splats that are never visible keep count 0 until the first forward writes them.
  DS_CUDA(cudaMemset(rb.counts, 0, n * sizeof(uint32_t) + (n == 0 ? 4 : 0)));
  return DS_OK;
}

// Scratch of the counting sort for a grid of rb.tiles tiles (none beyond
// kCountSortMaxTiles, or with DS_TILE_SORT=radix: the radix path then runs).
static int alloc_count_sort(RasterBuffers& rb) {
  release(rb.tile_hist);
  release(rb.tile_totals);
  rb.count_chunks = 0;
  static const bool radix_only = [] {
    const char* e = getenv("DS_TILE_SORT");
    return e && strcmp(e, "radix") == 0;
  }();
  if (radix_only || rb.tiles <= 0 || rb.tiles > kCountSortMaxTiles) return DS_OK;
  // one chunk per 2 x 148 SMs, at least 512 pairs each
  rb.count_chunks = (int)std::max<int64_t>(1, std::min<int64_t>(kSortBlocks, (rb.cap + 511) / 512));
  DS_TRY(alloc(&rb.tile_hist, (size_t)rb.count_chunks * rb.tiles));
  DS_TRY(alloc(&rb.tile_totals, (size_t)rb.tiles));
  // the scatter's shared memory (up to 160 KB) is opted into once per device
  static uint64_t smem_set = 0;
  int dev = 0;
  DS_CUDA(cudaGetDevice(&dev));
  if (dev >= 64 || !(smem_set >> dev & 1u)) {
    const int most = kCountSortMaxTiles * (4 + 2 * kScatterWarps) + 64;
    DS_CUDA(cudaFuncSetAttribute(tile_scatter_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 most));
    if (dev < 64) smem_set |= 1ull << dev;
  }
  return DS_OK;
}

int raster_alloc(RasterBuffers& rb, int width, int height, int max_splats, int64_t cap) {
  if (width <= 0 || height <= 0 || max_splats < 0) return DS_ERR_ARG;
  DS_TRY(raster_alloc_splats(rb, max_splats, cap));
  return raster_resize(rb, width, height);
}

int raster_alloc_batch(RasterBuffers& rb, int64_t pixels, int tiles, int tile_size,
                       int max_splats, int64_t cap) {
  if (pixels <= 0 || tiles <= 0 || max_splats < 0) return DS_ERR_ARG;
  if (tile_size != 8 && tile_size != 16 && tile_size != 32) return DS_ERR_ARG;
  DS_TRY(raster_alloc_splats(rb, max_splats, cap));
  rb.tile_size = tile_size;
  rb.width = (int)pixels;  // batch: flat pixel count; per-instance sizes live in geom
  rb.height = 1;
  rb.ntx = tiles;
  rb.nty = 1;
  rb.tiles = tiles;
  DS_TRY(alloc(&rb.ranges, (size_t)tiles));
  DS_TRY(alloc(&rb.tile_bound, (size_t)tiles));
  DS_TRY(alloc(&rb.tile_order, (size_t)tiles));
  DS_TRY(alloc(&rb.alphas, (size_t)pixels));
  DS_TRY(alloc(&rb.last_ids, (size_t)pixels));
  DS_TRY(alloc(&rb.loss_partials, (size_t)tiles));
  DS_CUDA(cudaMemset(rb.ranges, 0, tiles * sizeof(int2)));
  return alloc_count_sort(rb);
}

int raster_resize(RasterBuffers& rb, int width, int height) {
  if (width <= 0 || height <= 0) return DS_ERR_ARG;
  if (width == rb.width && height == rb.height) return DS_OK;
  release(rb.ranges);
  release(rb.tile_bound);
  release(rb.tile_order);
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
  DS_TRY(alloc(&rb.tile_bound, (size_t)rb.tiles));
  DS_TRY(alloc(&rb.tile_order, (size_t)rb.tiles));
  DS_TRY(alloc(&rb.alphas, px));
  DS_TRY(alloc(&rb.last_ids, px));
  DS_TRY(alloc(&rb.loss_partials, (size_t)rb.tiles));
  DS_CUDA(cudaMemset(rb.ranges, 0, rb.tiles * sizeof(int2)));
  return alloc_count_sort(rb);
}

void raster_free(RasterBuffers& rb) {
  release(rb.rec_a);
  release(rb.rec_b);
  release(rb.rec_c);
  release(rb.rec_idet);
  release(rb.rect);
  release(rb.counts);
  release(rb.seg_start);
  release(rb.long_list);
  release(rb.depth_keys);
  release(rb.depth_k0);
  release(rb.depth_k1);
  release(rb.depth_v0);
  release(rb.depth_v1);
  release(rb.emit_offsets);
  release(rb.g2);
  release(rb.tile_k0);
  release(rb.tile_k1);
  release(rb.tile_v0);
  release(rb.tile_v1);
  release(rb.emit_splat);
  release(rb.sorted_splat);
  release(rb.isect_grad);
  release(rb.sort.hist);
  release(rb.scan.partials);
  release(rb.scan.long_partials);
  release(rb.scalars);
  release(rb.ranges);
  release(rb.tile_bound);
  release(rb.tile_order);
  release(rb.alphas);
  release(rb.last_ids);
  release(rb.loss_partials);
  release(rb.tile_hist);
  release(rb.tile_totals);
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

int raster_build_lists(RasterBuffers& rb, int n, cudaStream_t s, cudaEvent_t* ev,
                       bool with_long_list) {
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
                                rb.scan, s, with_long_list ? rb.long_list : nullptr, &sc->n_long));
    // 3) emit (tile, emission index) pairs grouped by splat in depth order
    const dim3 emit_grid((unsigned)(((int64_t)n * 4 + kThreads - 1) / kThreads));
    static_assert(kCountSortMaxTiles <= 65536, "counting-path tile ids are 16-bit");
    uint16_t* tile16 = reinterpret_cast<uint16_t*>(rb.tile_k0);  // counting path
    if (rb.tile_hist) {
      DS_CUDA(launch_pdl(emit_kernel<uint16_t>, emit_grid, dim3(kThreads), 0, s, rb.depth_perm,
                         rb.counts, rb.emit_offsets, rb.rect, n, rb.ntx, (uint32_t)rb.cap, tile16,
                         rb.emit_splat, rb.seg_start, rb.inst_of_splat, rb.geom, rb.ranges,
                         rb.tiles));
    } else {
      DS_CUDA(launch_pdl(emit_kernel<uint32_t>, emit_grid, dim3(kThreads), 0, s, rb.depth_perm,
                         rb.counts, rb.emit_offsets, rb.rect, n, rb.ntx, (uint32_t)rb.cap,
                         rb.tile_k0, rb.emit_splat, rb.seg_start, rb.inst_of_splat, rb.geom,
                         rb.ranges, rb.tiles));
    }
    if (ev) DS_CUDA(cudaEventRecord(ev[1], s));
    if (rb.tile_hist) {
      // 4) stable counting sort by tile id; the ranges come out of its scan
      const int T = rb.tiles, G = rb.count_chunks;
      const size_t cnt_smem = (size_t)T * 4;
      const size_t sct_smem = (size_t)T * 4 + (size_t)((T + 1) & ~1) * 2 * kScatterWarps;
      DS_CUDA(launch_pdl(tile_count_kernel, dim3(G), dim3(kThreads), cnt_smem, s, tile16,
                         &sc->n_isects, T, rb.tile_hist, &sc->status));
      int32_t* order = (rb.tile_order && rb.schedule == DS_SCHEDULE_LONGEST_FIRST)
                           ? rb.tile_order : nullptr;
      DS_CUDA(launch_pdl(tile_offsets_kernel, dim3((T + 31) / 32), dim3(kOffsetThreads), 0, s,
                         rb.tile_hist, G, T, rb.tile_totals, rb.ranges, sc, order));
      DS_CUDA(launch_pdl(tile_scatter_kernel, dim3(G), dim3(32 * kScatterWarps), sct_smem, s,
                         tile16,
                         rb.emit_splat, &sc->n_isects, T, rb.tile_hist, rb.ranges,
                         rb.sorted_splat));
      rb.sorted_tile = nullptr;
      if (ev) DS_CUDA(cudaEventRecord(ev[2], s));
      return cuda_status(cudaGetLastError());
    }
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
  // 5) per-tile ranges (cleared by the emission, or here when nothing was emitted)
  if (n <= 0) DS_CUDA(cudaMemsetAsync(rb.ranges, 0, (size_t)rb.tiles * sizeof(int2), s));
  {
    const int64_t want = (rb.cap + kThreads - 1) / kThreads;
    const unsigned blocks = (unsigned)std::max<int64_t>(1, std::min<int64_t>(want, 148 * 8));
    DS_CUDA(launch_pdl(ranges_kernel, dim3(blocks), dim3(kThreads), 0, s, rb.sorted_tile,
                       &sc->n_isects, reinterpret_cast<int*>(rb.ranges), (uint32_t)rb.tiles,
                       &sc->status));
  }
  DS_CUDA(cudaGetLastError());
  if (rb.tile_order && rb.schedule == DS_SCHEDULE_LONGEST_FIRST) {
    DS_CUDA(launch_pdl(tile_order_kernel, dim3(1), dim3(1024), 0, s, rb.ranges, rb.tiles,
                       rb.tile_order));
  }
  if (ev) DS_CUDA(cudaEventRecord(ev[2], s));
  return DS_OK;
}

int raster_download(const RasterBuffers& rb, int n_splats, int what, void* host, int64_t bytes) {
  if (!host || bytes < 0 || n_splats < 0) return DS_ERR_ARG;
  DS_CUDA(cudaDeviceSynchronize());
  uint32_t n = 0;
  DS_CUDA(cudaMemcpy(&n, &rb.scalars->n_isects, sizeof(uint32_t), cudaMemcpyDeviceToHost));
  const size_t px = (size_t)rb.width * rb.height;
  switch (what) {
    case DS_RASTER_KEYS: {
      // (tile id << 32) | depth bits of the pair's splat, in sorted order
      if ((size_t)bytes < (size_t)n * 8) return DS_ERR_ARG;
      if (n == 0) return DS_OK;
      // the tile of each sorted pair, from the tile ranges
      std::vector<uint32_t> tiles(n, 0xffffffffu), ids(n), depth(n_splats > 0 ? n_splats : 1);
      std::vector<int2> rg(rb.tiles > 0 ? rb.tiles : 1);
      DS_CUDA(cudaMemcpy(rg.data(), rb.ranges, (size_t)rb.tiles * 8, cudaMemcpyDeviceToHost));
      for (int t = 0; t < rb.tiles; ++t)
        for (int q = std::max(rg[t].x, 0); q < rg[t].y && q < (int64_t)n; ++q) tiles[q] = (uint32_t)t;
      DS_CUDA(cudaMemcpy(ids.data(), rb.sorted_splat, (size_t)n * 4, cudaMemcpyDeviceToHost));
      DS_CUDA(cudaMemcpy(depth.data(), rb.depth_keys, (size_t)n_splats * 4,
                         cudaMemcpyDeviceToHost));
      uint64_t* k = (uint64_t*)host;
      for (uint32_t q = 0; q < n; ++q) {
        if (ids[q] >= (uint32_t)n_splats || tiles[q] == 0xffffffffu) return DS_ERR_INTERNAL;
        k[q] = ((uint64_t)tiles[q] << 32) | depth[ids[q]];
      }
      return DS_OK;
    }
    case DS_RASTER_IDS:
      if ((size_t)bytes < (size_t)n * 4) return DS_ERR_ARG;
      if (n) DS_CUDA(cudaMemcpy(host, rb.sorted_splat, (size_t)n * 4, cudaMemcpyDeviceToHost));
      return DS_OK;
    case DS_RASTER_RANGES:
      if ((size_t)bytes < (size_t)rb.tiles * 8) return DS_ERR_ARG;
      DS_CUDA(cudaMemcpy(host, rb.ranges, (size_t)rb.tiles * 8, cudaMemcpyDeviceToHost));
      return DS_OK;
    case DS_RASTER_LAST_IDS:
      if ((size_t)bytes < px * 4) return DS_ERR_ARG;
      DS_CUDA(cudaMemcpy(host, rb.last_ids, px * 4, cudaMemcpyDeviceToHost));
      return DS_OK;
    case DS_RASTER_ALPHAS:
      if ((size_t)bytes < px * 4) return DS_ERR_ARG;
      DS_CUDA(cudaMemcpy(host, rb.alphas, px * 4, cudaMemcpyDeviceToHost));
      return DS_OK;
    case DS_RASTER_COUNTS:
      if ((size_t)bytes < (size_t)n_splats * 4) return DS_ERR_ARG;
      if (n_splats)
        DS_CUDA(cudaMemcpy(host, rb.counts, (size_t)n_splats * 4, cudaMemcpyDeviceToHost));
      return DS_OK;
    case DS_RASTER_CONICS:
      if ((size_t)bytes < (size_t)n_splats * 16) return DS_ERR_ARG;
      if (n_splats)
        DS_CUDA(cudaMemcpy(host, rb.rec_b, (size_t)n_splats * 16, cudaMemcpyDeviceToHost));
      return DS_OK;
    default:
      return DS_ERR_ARG;
  }
}

int raster_reduce_grads(RasterBuffers& rb, const ds_splat2d& gin, int n, cudaStream_t s) {
  if (n <= 0) return DS_OK;
  segment_reduce_short_kernel<true><<<(unsigned)(((int64_t)n + kThreads - 1) / kThreads), kThreads,
                                      0, s>>>(rb.isect_grad, rb.depth_perm, rb.emit_offsets,
                                              rb.counts, (uint32_t)rb.cap, n, rb.g2, gin,
                                              grad_segments(rb));
  DS_CUDA(cudaGetLastError());
  return launch_long_reduce<true>(rb, n, gin, s);
}

int raster_reduce_long_grads(RasterBuffers& rb, int n, cudaStream_t s) {
  if (n <= 0) return DS_OK;
  return launch_long_reduce<false>(rb, n, ds_splat2d{}, s);
}

}  // namespace ds
