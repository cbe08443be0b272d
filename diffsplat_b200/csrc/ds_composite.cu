// Front-to-back compositing of one tile per CTA and its backward.
//
// Semantics: src/layers/tile_rasterize_layer.cu:192-309 (forward) and
// :356-578 (backward): NDC pixel centres, conic from Cov2D, sigma < 0 skip,
// alpha = min(0.99, o exp(-sigma)), alpha < 1/255 skip, termination after
// including the splat that brings T to <= 1e-4, last_ids = sorted-list index of
// the last contributor, backward by reverse traversal with
// T_before = T / max(1 - alpha, 1e-6).
//
// Layout: tiles are TS x TS pixels (16, the reference's TILE_SIZE; batches may
// use 8 or 32); each thread owns PPT pixels of one column (PPT = 1, 2 or 4); a
// warp covers a BW x BH block (8x4, 8x8 or 16x8 pixels).  When a batch of
// splats is staged in shared memory, each splat's acceptance box is tested
// once against every warp's block; each warp then walks only its own hits
// (ballot words of the per-splat warp masks), so shared-memory reads and
// (backward) the warp reduction are shared by 32 * PPT pixels and misses cost
// nothing in the inner loop.  The backward keeps one gradient partial per warp
// and splat in shared memory and sums the warps in a fixed order: gradients
// are deterministic run to run.
//
// Batch mode (kBatch): tile indices are batch-wide; tile_inst / geom give each
// tile's instance, image size, tile grid and first pixel.
#include <stdlib.h>
#include <string.h>

#include "ds_common.cuh"
#include "ds_internal.h"

namespace ds {

namespace {

constexpr int kFwdBatch = 256;  // splats staged in shared memory per forward batch
#ifndef DS_FWD_GROUP
#define DS_FWD_GROUP 4
#endif
constexpr int kFwdGroupPpt1 = DS_FWD_GROUP;  // forward hits evaluated together at 1 px/thread
#ifndef DS_BWD_GROUP
#define DS_BWD_GROUP 2
#endif
constexpr int kBwdGroupPpt1 = DS_BWD_GROUP;  // backward hits evaluated together at 1 px/thread
#ifndef DS_FWD_MIN_BLOCKS
#define DS_FWD_MIN_BLOCKS 4
#endif
#ifndef DS_BWD_MIN_BLOCKS
#define DS_BWD_MIN_BLOCKS 3
#endif

// Backward layout chosen per forward when ppt_bwd is 0: two pixels per thread
// (8x8-pixel warp blocks, one warp reduction per 64 pixels) when the
// forward's hits had at least 24.7 contributing pixels of the 32 of an 8x4
// block on average, one otherwise.  Measured on the 1280x720 / 60000-splat fit
// at steps 25-4000: the two-pixel backward is faster down to about 24.7 (0.49
// vs 0.63 ms at 26.6, early in the fit), equal there and slower below (0.64
// vs 0.48 ms at 21.9, late).  Chosen for a whole frame: a per-tile choice
// (two launches splitting the tiles) measured slower than either layout alone.
constexpr uint32_t kDenseLanesX10 = 247;

template <int PPT, int TS>
struct Lay {
  static constexpr int kThreads = TS * TS / PPT;
  static constexpr int kWarps = kThreads / 32;
  static constexpr int BW = PPT == 4 ? 16 : 8;  // warp block width
  static constexpr int BH = 32 * PPT / BW;      // warp block height
  static constexpr int kLaneRows = 32 / BW;     // rows between a thread's pixels
  static constexpr int kWarpsX = TS / BW;
  // backward batch: the per-warp partials (kWarps x kBwdBatch x 36 B) stay within 36 KB
  static constexpr int kBwdBatch = 1024 / kWarps < 128 ? 1024 / kWarps : 128;
  // resident CTAs per SM the register allocation must allow (256-thread CTAs)
  static constexpr int kMinBlocksFwd = kThreads == 256 ? DS_FWD_MIN_BLOCKS : 1;
  // 128-thread backward (two pixels per thread): 7 CTAs per SM caps it at 70
  // registers with no spills (93 unbounded, 5 CTAs; bwd 0.488 -> 0.471 ms on
  // the 1280x720 fit at step 25, B200); 8 CTAs (64 registers) measured slower.
  // 256-thread backward (one pixel per thread): 3 CTAs per SM (up to 85
  // registers); at 4 (64 registers) it spills, 0.479 -> 0.503 ms at step 1010
  static constexpr int kMinBlocksBwd = kThreads == 256 ? DS_BWD_MIN_BLOCKS
                                                        : (kThreads == 128 ? 7 : 1);
  // hits evaluated together: only at 1 pixel per thread; with more pixels the
  // per-pixel state already fills the registers (batch64, B200: grouping
  // at 2 pixels per thread cost 0.6% there and 5% before the backward
  // was limited to one hit per group)
  static constexpr int kFwdGroup = PPT == 1 ? kFwdGroupPpt1 : 1;
  static constexpr int kBwdGroup = PPT == 1 ? kBwdGroupPpt1 : 1;
  static_assert(kThreads % 32 == 0 && BW <= TS && kWarps <= 32, "unsupported tile layout");
};

// Where a tile lies: its image size, its tile grid, its index in that grid and
// the first pixel of its image in the pixel arrays.
struct TileGeo {
  int W, H, ntx, local, pix_off;
};

template <bool kBatch>
__device__ __forceinline__ TileGeo tile_geo(int tile, int W, int H, int ntx,
                                            const uint16_t* __restrict__ tile_inst,
                                            const InstGeom* __restrict__ geom) {
  if (!kBatch) return TileGeo{W, H, ntx, tile, 0};
  const InstGeom g = geom[tile_inst[tile]];
  return TileGeo{g.width, g.height, g.ntx, tile - g.tile_off, g.pix_off};
}

template <int PPT>
struct Pixels {
  int j;       // column
  int i[PPT];  // rows
  bool inside[PPT];
  float px;
  float py[PPT];
  float wx_lo, wx_hi, wy_lo, wy_hi;  // extremes of the warp's pixel centres (NDC)
};

template <int PPT, int TS>
__device__ __forceinline__ Pixels<PPT> pixels(int tile, int ntx, int W, int H) {
  using Lc = Lay<PPT, TS>;
  Pixels<PPT> m;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int trow = tile / ntx, tcol = tile - trow * ntx;
  const int lx = lane % Lc::BW, ly = lane / Lc::BW;
  const int wx = w % Lc::kWarpsX, wy = w / Lc::kWarpsX;
  m.j = tcol * TS + wx * Lc::BW + lx;
  m.px = 2.f * (m.j + 0.5f) / W - 1.f;
  float yl = 3.0e38f, yh = -3.0e38f;
#pragma unroll
  for (int k = 0; k < PPT; ++k) {
    m.i[k] = trow * TS + wy * Lc::BH + ly + k * Lc::kLaneRows;
    m.inside[k] = m.i[k] < H && m.j < W;
    m.py[k] = 1.f - 2.f * (m.i[k] + 0.5f) / H;
    yl = fminf(yl, m.py[k]);
    yh = fmaxf(yh, m.py[k]);
  }
  float xl = m.px, xh = m.px;
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

// Acceptance-box test of a splat record against one warp's pixel box
// {x_lo, x_hi, y_lo, y_hi}.
__device__ __forceinline__ bool misses(const float4& a, const float4& box) {
  return a.x + a.z < box.x || a.x - a.z > box.y || a.y + a.w < box.z || a.y - a.w > box.w;
}

// Whether any point of a warp's pixel box can reach the splat's sigma cut:
// the minimum over the box of a lower bound of the conic's quadratic form
// (diagonal shrunk by 1e-5 relative, as for the acceptance box) is at the
// centre when the box holds it, else at the clamped stationary point of one
// of the four edges.  The 0.01 of slack in the cut covers the rounding, so a
// pixel that can pass the per-pixel tests is never skipped.
__device__ __forceinline__ bool ellipse_hits(const float4& a, const float4& b, float cut,
                                             const float4& box) {
  if (misses(a, box)) return false;
  if (!(a.z <= 3.0e38f && a.w <= 3.0e38f)) return true;  // unbounded region
  const float x0 = box.x - a.x, x1 = box.y - a.x, y0 = box.z - a.y, y1 = box.w - a.y;
  if (x0 <= 0.f && x1 >= 0.f && y0 <= 0.f && y1 >= 0.f) return true;
  const float k = 1e-5f;
  const float qa = b.x - k * (fabsf(b.x) + fabsf(b.y));
  const float qc = b.z - k * (fabsf(b.z) + fabsf(b.y));
  const float qb = b.y;
  if (!(qa > 0.f && qc > 0.f)) return true;
  const float ia = 1.f / qa, ic = 1.f / qc;
  float m = 3.0e38f;
#pragma unroll
  for (int e = 0; e < 2; ++e) {
    const float X = e ? x1 : x0;
    const float y = fminf(fmaxf(-qb * X * ic, y0), y1);
    m = fminf(m, qa * X * X + 2.f * qb * X * y + qc * y * y);
    const float Y = e ? y1 : y0;
    const float x = fminf(fmaxf(-qb * Y * ia, x0), x1);
    m = fminf(m, qa * x * x + 2.f * qb * x * Y + qc * Y * Y);
  }
  return 0.5f * m <= cut;
}

// Forward alpha of a splat at a pixel (0 when the splat is skipped there):
// sigma < 0, or alpha below 1/255.  Beyond the cut (ln(255 o) + 0.01, used by
// the warp-block tests) alpha is below 0.99 / 255 and fails the threshold test
// by itself, so the pixel loop does not test sigma against the cut.
__device__ __forceinline__ float splat_alpha(float dx, float dy, const float4& b, float cut) {
  (void)cut;
  const float sigma = 0.5f * conic_dist2(dx, dy, b.x, b.y, b.z);
  if (sigma < 0.f) return 0.f;
  const float alpha = fminf(kMaxAlpha, b.w * __expf(-sigma));
  return alpha < kAlphaThres ? 0.f : alpha;
}

// One splat of a batch, loaded into registers a batch ahead of its use so the
// gathers overlap the current batch's compositing.
struct Staged {
  float4 a, b, c;
  float idet;
  bool ok;
};

// Bit w set: the splat can reach warp w's pixel block.
template <int NW>
__device__ __forceinline__ uint32_t warp_hits(const float4& a, const float4& b, float cut,
                                              const float4* box) {
  uint32_t mk = 0;
#pragma unroll
  for (int w = 0; w < NW; ++w) mk |= ellipse_hits(a, b, cut, box[w]) ? (1u << w) : 0u;
  return mk;
}

template <int PPT, int TS, bool kLoss, bool kCount, bool kBatch>
__global__ void __launch_bounds__(Lay<PPT, TS>::kThreads, Lay<PPT, TS>::kMinBlocksFwd)
    composite_fwd_kernel(const float4* __restrict__ ra, const float4* __restrict__ rb,
                         const float4* __restrict__ rc, const uint32_t* __restrict__ sorted_splat,
                         const int2* __restrict__ ranges, const int32_t* __restrict__ order,
                         float* __restrict__ out_rgb, float* __restrict__ out_alpha,
                         int32_t* __restrict__ last_ids, int W_, int H_, int ntx_,
                         const uint16_t* __restrict__ tile_inst, const InstGeom* __restrict__ geom,
                         const float* __restrict__ target, float* __restrict__ loss_partials,
                         DevScalars* __restrict__ sc, DevScalars* __restrict__ mode_sc) {
  pdl_wait();
  using Lc = Lay<PPT, TS>;
  constexpr int NT = Lc::kThreads;
  constexpr int NW = Lc::kWarps;
  __shared__ float4 sA[kFwdBatch], sB[kFwdBatch], sC[kFwdBatch];
  __shared__ uint32_t sHits[NW], sLanes[NW];
  __shared__ uint32_t sMask[kFwdBatch];
  __shared__ float4 sBox[NW];
  __shared__ float red[NW];
  __shared__ bool last;
  const int tile = order ? order[blockIdx.x] : (int)blockIdx.x;
  const TileGeo tg = tile_geo<kBatch>(tile, W_, H_, ntx_, tile_inst, geom);
  const int W = tg.W, H = tg.H;
  const Pixels<PPT> m = pixels<PPT, TS>(tg.local, tg.ntx, W, H);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) sBox[w] = make_float4(m.wx_lo, m.wx_hi, m.wy_lo, m.wy_hi);
  const int2 range = ranges[tile];
  const int start = range.x, end = range.y;
  float T[PPT], Cr[PPT], Cg[PPT], Cb[PPT];
  uint32_t cur[PPT];
  bool done[PPT];
  bool all_done = true;
  uint32_t n_contrib = 0, n_tested = 0;
  uint32_t n_hits = 0, n_lanes = 0;  // this warp's hits and their contributing lanes
#pragma unroll
  for (int k = 0; k < PPT; ++k) {
    T[k] = 1.f;
    Cr[k] = Cg[k] = Cb[k] = 0.f;
    cur[k] = 0;
    done[k] = !m.inside[k];
    all_done = all_done && done[k];
  }
  constexpr int R = (kFwdBatch + NT - 1) / NT;  // splats each thread stages
  Staged pf[R];
  auto prefetch = [&](int b0) {
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int l = threadIdx.x + r * NT, idx = b0 + l;
      pf[r].ok = l < kFwdBatch && idx < end;
      if (pf[r].ok) {
        const uint32_t g = sorted_splat[idx];
        pf[r].a = ra[g];
        pf[r].b = rb[g];
        pf[r].c = rc[g];
      }
    }
  };
  prefetch(start);
  for (int b0 = start; b0 < end; b0 += kFwdBatch) {
    if (__syncthreads_count(all_done) >= NT) break;
    // Stage the batch; each splat's warp-overlap mask is computed once here
    // so that every warp walks only the splats that can touch its pixels.
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int l = threadIdx.x + r * NT;
      if (l < kFwdBatch) {
        uint32_t mk = 0u;
        if (pf[r].ok) {
          sA[l] = pf[r].a;
          sB[l] = pf[r].b;
          sC[l] = pf[r].c;
          mk = warp_hits<NW>(pf[r].a, pf[r].b, pf[r].c.w, sBox);
        }
        sMask[l] = mk;
      }
    }
    if (b0 + kFwdBatch < end) prefetch(b0 + kFwdBatch);
    __syncthreads();
    const int bs = min(kFwdBatch, end - b0);
    bool stop = !__any_sync(0xffffffffu, !all_done);
    for (int kw = 0; kw * 32 < bs && !stop; ++kw) {
      const int l = kw * 32 + lane;
      uint32_t word = __ballot_sync(0xffffffffu, l < bs && ((sMask[l] >> w) & 1u));
      // Hits are taken Lc::kFwdGroup at a time: all their alphas are computed
      // before any is composited (front to back), so the conic / exp chains of
      // the group overlap.
      while (word) {
        int tg[Lc::kFwdGroup];
        int ng = 0;
#pragma unroll
        for (int g = 0; g < Lc::kFwdGroup; ++g) {
          tg[g] = word ? kw * 32 + __ffs(word) - 1 : tg[0];  // word is warp-uniform
          ng += word ? 1 : 0;
          word &= word - 1u;
        }
        n_hits += (uint32_t)ng;
        float4 ag[Lc::kFwdGroup], bg[Lc::kFwdGroup], cg[Lc::kFwdGroup];
#pragma unroll
        for (int g = 0; g < Lc::kFwdGroup; ++g) {
          ag[g] = sA[tg[g]];
          bg[g] = sB[tg[g]];
          cg[g] = sC[tg[g]];
        }
#pragma unroll
        for (int k = 0; k < PPT; ++k) {
          if (done[k]) continue;
          float al[Lc::kFwdGroup];
#pragma unroll
          for (int g = 0; g < Lc::kFwdGroup; ++g)
            al[g] = splat_alpha(ag[g].x - m.px, ag[g].y - m.py[k], bg[g], cg[g].w);
#pragma unroll
          for (int g = 0; g < Lc::kFwdGroup; ++g) {
            if (g >= ng || done[k]) break;
            if (kCount) ++n_tested;
            if (al[g] > 0.f) {
              if (kCount) ++n_contrib;
              ++n_lanes;
              const float vis = al[g] * T[k];
              Cr[k] = __fmaf_rn(cg[g].x, vis, Cr[k]);
              Cg[k] = __fmaf_rn(cg[g].y, vis, Cg[k]);
              Cb[k] = __fmaf_rn(cg[g].z, vis, Cb[k]);
              cur[k] = (uint32_t)(b0 + tg[g]);
              T[k] = T[k] * (1.f - al[g]);
              if (T[k] <= kTThres) done[k] = true;
            }
          }
        }
        all_done = true;
#pragma unroll
        for (int k = 0; k < PPT; ++k) all_done = all_done && done[k];
        if (!__any_sync(0xffffffffu, !all_done)) {
          stop = true;
          break;
        }
      }
    }
  }
  if (kCount) {
    uint32_t a = n_contrib, t = n_tested;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      a += __shfl_xor_sync(0xffffffffu, a, o);
      t += __shfl_xor_sync(0xffffffffu, t, o);
    }
    if ((threadIdx.x & 31) == 0) {
      atomicAdd(&sc->pairs[0], (unsigned long long)a);
      atomicAdd(&sc->pairs[1], (unsigned long long)t);
    }
  }
  if (mode_sc) {
    const uint32_t lanes = warp_sum_u32(n_lanes);
    if (lane == 0) {
      sHits[w] = n_hits;
      sLanes[w] = lanes;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      unsigned long long h = 0, c = 0;
#pragma unroll
      for (int k = 0; k < NW; ++k) {
        h += sHits[k];
        c += sLanes[k];
      }
      atomicAdd(&mode_sc->mode_hits, h);
      atomicAdd(&mode_sc->mode_lanes, c);
      __threadfence();
      if (atomicAdd(&mode_sc->mode_ticket, 1u) == gridDim.x - 1) {
        // the last CTA decides for the frame and clears the sums
        __threadfence();
        const unsigned long long th = atomicAdd(&mode_sc->mode_hits, 0ull);
        const unsigned long long tc = atomicAdd(&mode_sc->mode_lanes, 0ull);
        mode_sc->bwd_ppt = (th > 0ull && 10ull * tc >= kDenseLanesX10 * th) ? 2u : 1u;
        mode_sc->mode_hits = 0ull;
        mode_sc->mode_lanes = 0ull;
        mode_sc->mode_ticket = 0u;
      }
    }
  }
  float l = 0.f;
#pragma unroll
  for (int k = 0; k < PPT; ++k) {
    if (!m.inside[k]) continue;
    const int pix = tg.pix_off + m.i[k] * W + m.j;
    out_rgb[pix * 3 + 0] = Cr[k];
    out_rgb[pix * 3 + 1] = Cg[k];
    out_rgb[pix * 3 + 2] = Cb[k];
    out_alpha[pix] = 1.f - T[k];
    last_ids[pix] = (int32_t)cur[k];
    if (kLoss) {
      const float scale = 1.f / (float)(W * H);
      const float dR = Cr[k] - target[pix * 3 + 0];
      const float dG = Cg[k] - target[pix * 3 + 1];
      const float dB = Cb[k] - target[pix * 3 + 2];
      l += (dR * dR + dG * dG + dB * dB) * scale;
    }
  }
  if (kLoss) {
    l = warp_sum(l);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = l;
    __syncthreads();
    if (threadIdx.x == 0) {
      float s = 0.f;
      for (int k = 0; k < Lc::kWarps; ++k) s += red[k];
      loss_partials[tile] = s;
      if (!kBatch) {
        __threadfence();
        last = atomicAdd(&sc->ticket, 1u) == gridDim.x - 1;
      }
    }
    __syncthreads();
    // Batches sum their per-instance losses in batch_loss_kernel instead.
    if (!kBatch && last) {
      // The last CTA to finish sums the per-tile partials in tile order.
      __threadfence();
      float s = 0.f;
      for (int k = threadIdx.x; k < (int)gridDim.x; k += NT)
        s += ((volatile float*)loss_partials)[k];
      s = warp_sum(s);
      if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
      __syncthreads();
      if (threadIdx.x == 0) {
        float tot = 0.f;
        for (int k = 0; k < Lc::kWarps; ++k) tot += red[k];
        sc->loss = tot;
        sc->ticket = 0u;
      }
    }
  }
}

template <int PPT, int TS, bool kFusedLoss, bool kExact, bool kBatch>
__global__ void __launch_bounds__(Lay<PPT, TS>::kThreads, Lay<PPT, TS>::kMinBlocksBwd)
    composite_bwd_kernel(const float4* __restrict__ ra, const float4* __restrict__ rb,
                         const float4* __restrict__ rc, const float* __restrict__ ridet,
                         const uint32_t* __restrict__ sorted_splat,
                         const uint32_t* __restrict__ seg_start,
                         const ushort4* __restrict__ rect, const int2* __restrict__ ranges,
                         const int32_t* __restrict__ order, const float* __restrict__ alphas,
                         const int32_t* __restrict__ last_ids,
                         const float* __restrict__ grad_or_image, const float* __restrict__ target,
                         float* __restrict__ isect_grad, int W_, int H_, int ntx_,
                         const uint16_t* __restrict__ tile_inst,
                         const InstGeom* __restrict__ geom,
                         const uint32_t* __restrict__ depth_keys,
                         unsigned long long* __restrict__ tile_bound,
                         const DevScalars* __restrict__ mode_sc) {
  pdl_wait();
  using Lc = Lay<PPT, TS>;
  constexpr int NT = Lc::kThreads;
  constexpr int NW = Lc::kWarps;
  constexpr int B = Lc::kBwdBatch;
  __shared__ float4 sA[B], sB[B], sC[B];
  __shared__ float sI[B];
  __shared__ uint32_t sG[2][B];  // splat ids of the staged batch and the next
  __shared__ int sRC[2];
  __shared__ uint32_t sMask[B];
  __shared__ float4 sBox[NW];
  __shared__ __align__(16) float part[NW][B * 9];  // per-warp partial of each batch splat
  __shared__ int32_t sFinal[NW];
  const int tile = order ? order[blockIdx.x] : (int)blockIdx.x;
  // ppt_bwd == 0: the forward chose the layout for this frame; the other
  // layout's launch returns at once
  if (mode_sc && (PPT == 2) != (mode_sc->bwd_ppt == 2u)) return;
  const int2 range = ranges[tile];
  const int start = range.x;
  if (range.y <= start) {
    if (threadIdx.x == 0) tile_bound[tile] = 0ull;
    return;
  }
  const TileGeo tg = tile_geo<kBatch>(tile, W_, H_, ntx_, tile_inst, geom);
  const int W = tg.W, H = tg.H;
  const Pixels<PPT> m = pixels<PPT, TS>(tg.local, tg.ntx, W, H);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (threadIdx.x == 0) {  // the tile's row and column in its grid, for the record indices
    sRC[0] = tg.local / tg.ntx;
    sRC[1] = tg.local - sRC[0] * tg.ntx;
  }
  if (lane == 0) sBox[w] = make_float4(m.wx_lo, m.wx_hi, m.wy_lo, m.wy_hi);
  // acc[k]: over the splats behind (already visited), weight x (colour . dL/dpixel)
  float T[PPT], gr[PPT], gg[PPT], gb[PPT], acc[PPT];
  int32_t fin[PPT];
  int32_t my_final = -1;
#pragma unroll
  for (int k = 0; k < PPT; ++k) {
    const int pix = tg.pix_off + min(m.i[k] * W + m.j, W * H - 1);
    T[k] = 1.f - alphas[pix];
    fin[k] = m.inside[k] ? last_ids[pix] : -1;
    my_final = max(my_final, fin[k]);
    gr[k] = gg[k] = gb[k] = 0.f;
    if (m.inside[k]) {
      if (kFusedLoss) {
        const float scale = 2.f / (float)(W * H);
        gr[k] = scale * (grad_or_image[pix * 3 + 0] - target[pix * 3 + 0]);
        gg[k] = scale * (grad_or_image[pix * 3 + 1] - target[pix * 3 + 1]);
        gb[k] = scale * (grad_or_image[pix * 3 + 2] - target[pix * 3 + 2]);
      } else {
        gr[k] = grad_or_image[pix * 3 + 0];
        gg[k] = grad_or_image[pix * 3 + 1];
        gb[k] = grad_or_image[pix * 3 + 2];
      }
    }
    acc[k] = 0.f;
  }
  const int32_t warp_final = warp_max(my_final);
  // Pairs after the tile's last contributing splat reach no pixel: the list
  // ends there for the backward, and no record is written for them (their
  // consumers skip them by tile_bound).
  if (lane == 0) sFinal[w] = warp_final;
  __syncthreads();
  int32_t tile_final = sFinal[0];
#pragma unroll
  for (int k = 1; k < NW; ++k) tile_final = max(tile_final, sFinal[k]);
  const int end = min(range.y, tile_final + 1);
  if (threadIdx.x == 0) {
    unsigned long long bound = 0ull;
    if (end > start) {
      const uint32_t last = sorted_splat[end - 1];
      bound = (((unsigned long long)depth_keys[last] << 32) | last) + 1ull;
    }
    tile_bound[tile] = bound;
  }
  if (end <= start) return;
  const int nb = (end - start + B - 1) / B;
  // Threads per staged splat: with twice as many threads as batch slots, two
  // threads share a splat's warp-block tests and its cross-warp sum.
  constexpr int kSplit = NT >= 2 * B ? 2 : 1;
  constexpr int R = (B * kSplit + NT - 1) / NT;  // splats each thread stages
  Staged pf[R];
  // batch bi holds sorted indices end - 1 - B bi down to end - B (bi + 1)
  auto prefetch = [&](int bi) {
    const int batch_end = end - 1 - B * bi;
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int l = (threadIdx.x + r * NT) / kSplit, li = batch_end - l;
      pf[r].ok = l < B && li >= start;
      if (pf[r].ok) {
        const uint32_t g = sorted_splat[li];
        pf[r].a = ra[g];
        pf[r].b = rb[g];
        pf[r].c = rc[g];
        pf[r].idet = ridet[g];
        if ((threadIdx.x + r * NT) % kSplit == 0) sG[bi & 1][l] = g;
      }
    }
  };
  prefetch(0);
  for (int bi = 0; bi < nb; ++bi) {
    const int batch_end = end - 1 - B * bi;  // farthest splat of the batch
    const int bs = min(B, batch_end + 1 - start);
    __syncthreads();
    // stage the batch back to front: slot l holds sorted index batch_end - l
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int slot = threadIdx.x + r * NT, l = slot / kSplit, h = slot % kSplit;
      uint32_t mk = 0u;
      if (l < B && pf[r].ok) {
        if (kSplit == 1) {
          mk = warp_hits<NW>(pf[r].a, pf[r].b, pf[r].c.w, sBox);
        } else {
          // this thread tests half of the warp blocks
#pragma unroll
          for (int k = 0; k < NW / 2; ++k) {
            const int wb = h * (NW / 2) + k;
            mk |= ellipse_hits(pf[r].a, pf[r].b, pf[r].c.w, sBox[wb]) ? (1u << wb) : 0u;
          }
        }
        if (h == 0) {
          sA[l] = pf[r].a;
          sB[l] = pf[r].b;
          sC[l] = pf[r].c;
          sI[l] = pf[r].idet;
        }
      }
      if (kSplit == 2) mk |= __shfl_xor_sync(0xffffffffu, mk, 1);  // pairs are adjacent lanes
      if (l < B && h == 0) sMask[l] = mk;
    }
    if (bi + 1 < nb) prefetch(bi + 1);
    {
      float4* p4 = reinterpret_cast<float4*>(&part[0][0]);
      for (int q = threadIdx.x; q < NW * B * 9 / 4; q += NT) p4[q] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    __syncthreads();
    const int t_start = max(0, batch_end - warp_final);
    for (int kw = 0; kw * 32 < bs; ++kw) {
      const int l = kw * 32 + lane;
      uint32_t word =
          __ballot_sync(0xffffffffu, l >= t_start && l < bs && ((sMask[l] >> w) & 1u));
      // Hits are taken Lc::kBwdGroup at a time: the conic / exp / alpha of all of
      // them first (independent of T), then the recurrence back to front, then
      // the warp reductions, which overlap.
      while (word) {
        int tg[Lc::kBwdGroup];
        int ng = 0;
#pragma unroll
        for (int g = 0; g < Lc::kBwdGroup; ++g) {
          tg[g] = word ? kw * 32 + __ffs(word) - 1 : tg[0];  // word is warp-uniform
          ng += word ? 1 : 0;
          word &= word - 1u;
        }
        float4 ag[Lc::kBwdGroup], bg[Lc::kBwdGroup], cg[Lc::kBwdGroup];
        float ig[Lc::kBwdGroup];
#pragma unroll
        for (int g = 0; g < Lc::kBwdGroup; ++g) {
          ag[g] = sA[tg[g]];
          bg[g] = sB[tg[g]];
          cg[g] = sC[tg[g]];
          ig[g] = sI[tg[g]];
        }
        float v[Lc::kBwdGroup][8], va[Lc::kBwdGroup];
        bool any[Lc::kBwdGroup];
#pragma unroll
        for (int g = 0; g < Lc::kBwdGroup; ++g) {
#pragma unroll
          for (int q = 0; q < 8; ++q) v[g][q] = 0.f;
          va[g] = 0.f;
          any[g] = false;
        }
#pragma unroll
        for (int k = 0; k < PPT; ++k) {
          if (!m.inside[k]) continue;
          float dxg[Lc::kBwdGroup], dyg[Lc::kBwdGroup], d2g[Lc::kBwdGroup], eg[Lc::kBwdGroup], alg[Lc::kBwdGroup];
          bool pg[Lc::kBwdGroup];
#pragma unroll
          for (int g = 0; g < Lc::kBwdGroup; ++g) {
            dxg[g] = ag[g].x - m.px;
            dyg[g] = ag[g].y - m.py[k];
            d2g[g] = conic_dist2(dxg[g], dyg[g], bg[g].x, bg[g].y, bg[g].z);
            const float sigma = 0.5f * d2g[g];
            eg[g] = __expf(-sigma);
            alg[g] = fminf(kMaxAlpha, bg[g].w * eg[g]);
            pg[g] = g < ng && batch_end - tg[g] <= fin[k] && !(sigma < 0.f) &&
                    !(alg[g] < kAlphaThres);
          }
#pragma unroll
          for (int g = 0; g < Lc::kBwdGroup; ++g) {
            if (!pg[g]) continue;
            const float4 b = bg[g], c = cg[g];
            const float dx = dxg[g], dy = dyg[g], dist2 = d2g[g], g_exp = eg[g], alpha = alg[g];
            const float opac = b.w;
            any[g] = true;
            const float T_before = T[k] / fmaxf(1.f - alpha, 1e-6f);
            const float fac = alpha * T_before;
            v[g][0] += fac * gr[k];
            v[g][1] += fac * gg[k];
            v[g][2] += fac * gb[k];
            // Reference recurrence (tile_rasterize_layer.cu:518-521) weighs the
            // colour behind (absolute weights c_j alpha_j T_j) by T_before; the
            // exact derivative divides it by T_after instead.  The three
            // colour channels enter only through their dot product with
            // dL/dpixel.
            const float cg_k = c.x * gr[k] + c.y * gg[k] + c.z * gb[k];
            const float ia = kExact ? 1.f / T[k] : 1.f;
            const float v_alpha = T_before * (cg_k - acc[k] * ia);
            if (opac * g_exp <= kMaxAlpha) {
              va[g] += g_exp * v_alpha;
              // s = -2 dL/d(dist2).  With u = dx bx + dy by and w = dx by + dy
              // bz, d dist2 / d(ndc x, ndc y) = (2u, 2w) and d dist2 / d(conic)
              // gives the Cov2D terms -u^2, -w^2 and -2 (by dist2 + dx dy idet).
              const float s = opac * g_exp * v_alpha;
              const float u = dx * b.x + dy * b.y;
              const float wv = dx * b.y + dy * b.z;
              v[g][3] -= s * u;
              v[g][4] -= s * wv;
              const float hs = 0.5f * s;
              v[g][5] += hs * u * u;
              v[g][7] += hs * wv * wv;
              v[g][6] += s * (b.y * dist2 + dx * dy * ig[g]);
            }
            acc[k] += cg_k * fac;
            T[k] = T_before;
          }
        }
        bool hit_any[Lc::kBwdGroup];
#pragma unroll
        for (int g = 0; g < Lc::kBwdGroup; ++g) hit_any[g] = __any_sync(0xffffffffu, any[g]);
        if (Lc::kBwdGroup == 2 && hit_any[0] && hit_any[Lc::kBwdGroup - 1]) {
          // both hits contributed: one butterfly for their 2 x 9 sums
          const float s16 = warp_sum16_transposed(v[0], v[Lc::kBwdGroup - 1], lane);
          const float s2 = warp_sum2_transposed(va[0], va[Lc::kBwdGroup - 1], lane);
          const int gh = lane >> 4;
          if ((lane & 1) == 0) part[w][tg[gh] * 9 + ((lane >> 1) & 7)] = s16;
          if ((lane & 15) == 0) part[w][tg[gh] * 9 + 8] = s2;
        } else {
#pragma unroll
          for (int g = 0; g < Lc::kBwdGroup; ++g) {
            if (!hit_any[g]) continue;
            // lane 4q ends up with the warp sum of v[q]
            const float s8 = warp_sum8_transposed(v[g], lane);
            const float sa = warp_sum(va[g]);
            if ((lane & 3) == 0) part[w][tg[g] * 9 + (lane >> 2)] = s8;
            if (lane == 0) part[w][tg[g] * 9 + 8] = sa;
          }
        }
      }
    }
    __syncthreads();
    const int trow = sRC[0], tcol = sRC[1];
    for (int slot = threadIdx.x; slot < bs * kSplit; slot += NT) {
      const int l = slot / kSplit, h = slot % kSplit;
      // the pair's emission index: the splat's first one plus the tile's
      // row-major index in the splat's tile rectangle
      const uint32_t g = sG[bi & 1][l];
      const ushort4 r = rect[g];
      const uint32_t e = seg_start[g] + (uint32_t)(trow - r.z) * (uint32_t)(r.y - r.x + 1) +
                         (uint32_t)(tcol - r.x);
      float* dst = isect_grad + (size_t)e * 9;
#pragma unroll
      for (int q = h; q < 9; q += kSplit) {
        float s = 0.f;
#pragma unroll
        for (int ww = 0; ww < NW; ++ww) s += part[ww][l * 9 + q];
        dst[q] = s;
      }
    }
  }
}

const int32_t* schedule(const RasterBuffers& rb) {
  return rb.schedule == DS_SCHEDULE_LONGEST_FIRST ? rb.tile_order : nullptr;
}

// Whether the forward chooses the backward's layout (see kDenseLanesX10).
bool adaptive_bwd(const RasterBuffers& rb) {
  return rb.ppt_bwd == 0 && rb.ppt == 1 && !rb.geom;
}

template <int PPT, int TS, bool kBatch>
void launch_fwd(RasterBuffers& rb, float* out_rgb, const float* target, bool count,
                cudaStream_t s) {
  constexpr int NT = Lay<PPT, TS>::kThreads;
  const int32_t* order = schedule(rb);
  DevScalars* mode = (!count && PPT == 1 && adaptive_bwd(rb)) ? rb.scalars : nullptr;
#define DS_FWD(L, C)                                                                         \
  launch_pdl(composite_fwd_kernel<PPT, TS, L, C, kBatch>, dim3(rb.tiles), dim3(NT), 0, s,     \
             rb.rec_a, rb.rec_b, rb.rec_c, rb.sorted_splat, rb.ranges, order, out_rgb,        \
             rb.alphas, rb.last_ids, rb.width, rb.height, rb.ntx, rb.tile_inst, rb.geom,      \
             L ? target : nullptr, L ? rb.loss_partials : nullptr, rb.scalars, mode)
  if (count) DS_FWD(false, true);
  else if (target) DS_FWD(true, false);
  else DS_FWD(false, false);
#undef DS_FWD
}

template <int PPT, int TS, bool kBatch>
void launch_bwd(RasterBuffers& rb, const float* image, const float* grad_rgb, const float* target,
                cudaStream_t s, const DevScalars* mode = nullptr) {
  constexpr int NT = Lay<PPT, TS>::kThreads;
  const float* g = grad_rgb ? grad_rgb : image;
  const float* t = grad_rgb ? nullptr : target;
  const bool exact = rb.grad_mode == DS_GRAD_EXACT;
  const int32_t* order = schedule(rb);
#define DS_BWD(F, E)                                                                         \
  launch_pdl(composite_bwd_kernel<PPT, TS, F, E, kBatch>, dim3(rb.tiles), dim3(NT), 0, s,     \
             rb.rec_a, rb.rec_b, rb.rec_c, rb.rec_idet, rb.sorted_splat, rb.seg_start, rb.rect,\
             rb.ranges, order, rb.alphas, rb.last_ids, g, t, rb.isect_grad, rb.width,         \
             rb.height, rb.ntx, rb.tile_inst, rb.geom, rb.depth_keys, rb.tile_bound, mode)
  if (grad_rgb) {
    if (exact) DS_BWD(false, true);
    else DS_BWD(false, false);
  } else {
    if (exact) DS_BWD(true, true);
    else DS_BWD(true, false);
  }
#undef DS_BWD
}

struct FwdOp {
  RasterBuffers& rb;
  float* out_rgb;
  const float* target;
  bool count;
  cudaStream_t s;
  template <int P, int T, bool B>
  void run() const {
    launch_fwd<P, T, B>(rb, out_rgb, target, count, s);
  }
};

struct BwdOp {
  RasterBuffers& rb;
  const float* image;
  const float* grad_rgb;
  const float* target;
  cudaStream_t s;
  template <int P, int T, bool B>
  void run() const {
    launch_bwd<P, T, B>(rb, image, grad_rgb, target, s);
  }
};

// Single instance: 16x16 tiles, PPT 1, 2 or 4.  Batch: tiles of 8, 16 or 32
// pixels with PPT 1 or 2.
template <class F>
int dispatch(const RasterBuffers& rb, const F& f, bool backward = false) {
  const int ppt = (backward && rb.ppt_bwd != 0) ? rb.ppt_bwd : rb.ppt;
  if (!rb.geom) {
    switch (ppt) {
      case 4: f.template run<4, 16, false>(); return DS_OK;
      case 2: f.template run<2, 16, false>(); return DS_OK;
      default: f.template run<1, 16, false>(); return DS_OK;
    }
  }
  const bool two = ppt == 2;
  switch (rb.tile_size) {
    case 8:
      if (two) f.template run<2, 8, true>();
      else f.template run<1, 8, true>();
      return DS_OK;
    case 32:
      if (two) f.template run<2, 32, true>();
      else f.template run<1, 32, true>();
      return DS_OK;
    default:
      if (two) f.template run<2, 16, true>();
      else f.template run<1, 16, true>();
      return DS_OK;
  }
}

}  // namespace

int composite_default_ppt() {
  const char* e = getenv("DS_COMPOSITE_PPT");
  if (e) {
    int v = atoi(e);
    if (v == 1 || v == 2 || v == 4) return v;
  }
  // Fastest on the 1280x720 / 60000-splat fitter with the longest-first tile
  // schedule (B200, 1000 steps: 1 -> 688, 2 -> 631, 4 -> 454 steps/s).
  return 1;
}

int composite_default_ppt_bwd() {
  const char* e = getenv("DS_COMPOSITE_PPT_BWD");
  if (e) {
    int v = atoi(e);
    if (v == 1 || v == 2 || v == 4) return v;
  }
  // chosen per forward (kDenseLanesX10) behind a one-pixel-per-thread forward
  return composite_default_ppt() == 1 ? 0 : composite_default_ppt();
}

bool composite_longest_first() {
  static const bool on = [] {
    const char* e = getenv("DS_TILE_SCHEDULE");
    return !(e && strcmp(e, "raster") == 0);
  }();
  return on;
}

int raster_composite_forward(RasterBuffers& rb, float* out_rgb, const float* target,
                             cudaStream_t s) {
  dispatch(rb, FwdOp{rb, out_rgb, target, false, s});
  return cuda_status(cudaGetLastError());
}

int raster_composite_count(RasterBuffers& rb, float* out_rgb, cudaStream_t s) {
  DS_CUDA(cudaMemsetAsync(rb.scalars->pairs, 0, sizeof(rb.scalars->pairs), s));
  dispatch(rb, FwdOp{rb, out_rgb, nullptr, true, s});
  return cuda_status(cudaGetLastError());
}

int raster_composite_backward(RasterBuffers& rb, const float* image, const float* grad_rgb,
                              const float* target, cudaStream_t s) {
  if (adaptive_bwd(rb)) {
    // the launch of the layout the forward chose does the work
    launch_bwd<2, 16, false>(rb, image, grad_rgb, target, s, rb.scalars);
    launch_bwd<1, 16, false>(rb, image, grad_rgb, target, s, rb.scalars);
  } else {
    dispatch(rb, BwdOp{rb, image, grad_rgb, target, s}, true);
  }
  return cuda_status(cudaGetLastError());
}

}  // namespace ds
