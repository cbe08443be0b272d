// Stable LSD radix sort of (uint32 key, uint32 value) pairs and the exclusive
// scan that turns per-splat tile counts into emission offsets.
//
// This replaces the reference's cub::DeviceRadixSort::SortPairs over all 64
// key bits (src/layers/tile_rasterize_layer.cu:664-684).  The rasterizer sorts
// in two stages instead (depth keys of the splats, then tile ids of the
// emitted pairs, see ds_raster.cu), and each stage only sorts the bits it
// needs.  Element counts are read from device memory and every launch has a
// fixed grid, so the sort runs inside a captured CUDA graph without the
// reference's host read of n_isects (:660-661).
//
// Per pass (8-bit digit), three kernels:
//   hist    : per-CTA digit histogram of its contiguous chunk -> hist[digit][cta]
//   scan    : 32 CTAs, one warp per digit row, scan the digit-major
//             histogram into per-CTA exclusive offsets and row totals (the
//             scatter adds the prefix of the 256 digit totals itself)
//   scatter : each CTA re-reads its chunk 2048 items at a time, ranks items
//             stably inside each warp with __match_any_sync, combines warp
//             counts in shared memory and writes every item to its slot.
#include "ds_common.cuh"
#include "ds_internal.h"

namespace ds {

namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kItems = kSortTileItems / kThreads;  // 8 per lane

// Items per CTA: n split over G CTAs, rounded up to whole 2048-item tiles.
__device__ __forceinline__ uint32_t sort_chunk(uint32_t n, uint32_t G) {
  uint32_t per = (n + G - 1) / G;
  return (per + kSortTileItems - 1) / kSortTileItems * kSortTileItems;
}

__global__ void __launch_bounds__(kThreads)
    radix_hist_kernel(const uint32_t* __restrict__ keys, const uint32_t* __restrict__ n_dev,
                      uint32_t cap, int shift, uint32_t* __restrict__ hist) {
  pdl_wait();
  __shared__ uint32_t h[256];
  const uint32_t G = gridDim.x;
  const uint32_t n = min(*n_dev, cap);
  const uint32_t chunk = sort_chunk(n, G);
  const uint32_t begin = min(blockIdx.x * chunk, n);
  const uint32_t end = min(begin + chunk, n);
  h[threadIdx.x] = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31;
  // kItems loads in flight per thread, then warp-aggregated shared-memory
  // counting: one atomic per distinct digit per warp and item slot.
  for (uint32_t t0 = begin; t0 < end; t0 += kSortTileItems) {
    uint32_t d[kItems];
#pragma unroll
    for (int it = 0; it < kItems; ++it) {
      const uint32_t i = t0 + it * kThreads + threadIdx.x;
      d[it] = i < end ? ((keys[i] >> shift) & 255u) : 0x100u;
    }
#pragma unroll
    for (int it = 0; it < kItems; ++it) {
      // one atomic for a warp whose 32 keys share the digit (the high digits
      // of depth keys nearly always do), else one per key
      if (__all_sync(0xffffffffu, d[it] == __shfl_sync(0xffffffffu, d[it], 0))) {
        if (d[it] < 256u && lane == 0) atomicAdd(&h[d[it]], 32u);
      } else if (d[it] < 256u) {
        atomicAdd(&h[d[it]], 1u);
      }
    }
  }
  __syncthreads();
  hist[threadIdx.x * G + blockIdx.x] = h[threadIdx.x];
}

// Row scan of the digit-major histogram hist[digit * G + cta]: one warp per
// digit (256 / kWarps CTAs) loads its G counts at once, writes their exclusive
// scan in place and the row total to hist[256 * kSortBlocks + digit].  The
// scatter CTAs add the exclusive scan of the 256 totals themselves, so no
// single CTA walks the whole histogram.
constexpr int kRowChunks = (kSortBlocks + 31) / 32;

__global__ void __launch_bounds__(kThreads) scan_hist_kernel(uint32_t* __restrict__ hist, int G) {
  pdl_wait();
  const int lane = threadIdx.x & 31;
  const int d = blockIdx.x * kWarps + (threadIdx.x >> 5);
  uint32_t* row = hist + (size_t)d * G;
  uint32_t v[kRowChunks];
#pragma unroll
  for (int j = 0; j < kRowChunks; ++j) {
    const int b = j * 32 + lane;
    v[j] = b < G ? row[b] : 0u;
  }
  uint32_t carry = 0;
#pragma unroll
  for (int j = 0; j < kRowChunks; ++j) {
    const int b = j * 32 + lane;
    uint32_t incl = v[j];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    if (b < G) row[b] = carry + incl - v[j];
    carry += __shfl_sync(0xffffffffu, incl, 31);
  }
  if (lane == 0) hist[(size_t)256 * kSortBlocks + d] = carry;
}

// Each CTA takes its chunk 2048 items at a time: ranks them stably inside each
// warp with __match_any_sync, turns the per-warp digit counts into tile-local
// offsets, stages the tile in digit order in shared memory and writes it out
// in that order, so items of one digit leave as contiguous runs.
__global__ void __launch_bounds__(kThreads)
    radix_scatter_kernel(const uint32_t* __restrict__ kin, const uint32_t* __restrict__ vin,
                         int iota, uint32_t* __restrict__ kout, uint32_t* __restrict__ vout,
                         const uint32_t* __restrict__ n_dev, uint32_t cap, int shift,
                         const uint32_t* __restrict__ offs, const uint32_t* __restrict__ gsrc,
                         uint32_t* __restrict__ gdst) {
  pdl_wait();
  __shared__ uint32_t cnt[kWarps][256];  // per-warp digit counts, then per-warp offsets
  __shared__ uint32_t gbase[256];        // output position of the tile's first item of a digit
  __shared__ uint32_t lstart[256];       // tile-local start of each digit
  __shared__ uint32_t skey[kSortTileItems];
  __shared__ uint32_t sval[kSortTileItems];
  __shared__ uint32_t wt[kWarps];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const uint32_t n = min(*n_dev, cap);
  const uint32_t chunk = sort_chunk(n, gridDim.x);
  const uint32_t begin = min(blockIdx.x * chunk, n);
  const uint32_t end = min(begin + chunk, n);
  if (begin >= end) return;
  // thread t owns digit t: block exclusive scan of a per-digit value
  auto block_excl = [&](uint32_t v) {
    uint32_t incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    if (lane == 31) wt[w] = incl;
    __syncthreads();
    uint32_t wb = 0;
#pragma unroll
    for (int k = 0; k < kWarps; ++k) wb += k < w ? wt[k] : 0u;
    __syncthreads();
    return wb + incl - v;
  };
  // digit base = exclusive scan of the digit totals + this CTA's row offset
  gbase[threadIdx.x] = offs[threadIdx.x * gridDim.x + blockIdx.x] +
                       block_excl(offs[(size_t)256 * kSortBlocks + threadIdx.x]);
  const uint32_t lt = (1u << lane) - 1u;
  for (uint32_t t0 = begin; t0 < end; t0 += kSortTileItems) {
    for (int d = lane; d < 256; d += 32) cnt[w][d] = 0;
    __syncwarp();
    uint32_t key[kItems], val[kItems], rank[kItems];
#pragma unroll
    for (int it = 0; it < kItems; ++it) {
      const uint32_t idx = t0 + w * 256 + it * 32 + lane;
      const bool ok = idx < end;
      key[it] = ok ? kin[idx] : 0u;
      val[it] = ok ? (iota ? idx : vin[idx]) : 0u;
    }
#pragma unroll
    for (int it = 0; it < kItems; ++it) {
      const uint32_t idx = t0 + w * 256 + it * 32 + lane;
      const bool ok = idx < end;
      const uint32_t d = ok ? ((key[it] >> shift) & 255u) : 0x100u;
      // a warp whose 32 keys share the digit ranks them by lane, no match
      const uint32_t peers = __all_sync(0xffffffffu, d == __shfl_sync(0xffffffffu, d, 0))
                                 ? 0xffffffffu : __match_any_sync(0xffffffffu, d);
      const uint32_t pre = ok ? cnt[w][d] : 0u;
      __syncwarp();
      if (ok && lane == __ffs(peers) - 1) cnt[w][d] = pre + __popc(peers);
      __syncwarp();
      rank[it] = pre + __popc(peers & lt);
    }
    __syncthreads();
    uint32_t total;
    {
      uint32_t run = 0;
#pragma unroll
      for (int ww = 0; ww < kWarps; ++ww) {
        const uint32_t c = cnt[ww][threadIdx.x];
        cnt[ww][threadIdx.x] = run;
        run += c;
      }
      total = run;
      lstart[threadIdx.x] = block_excl(run);
    }
    __syncthreads();
#pragma unroll
    for (int it = 0; it < kItems; ++it) {
      const uint32_t idx = t0 + w * 256 + it * 32 + lane;
      if (idx < end) {
        const uint32_t d = (key[it] >> shift) & 255u;
        const uint32_t lp = lstart[d] + cnt[w][d] + rank[it];
        skey[lp] = key[it];
        sval[lp] = val[it];
      }
    }
    __syncthreads();
    const uint32_t items = min(end - t0, (uint32_t)kSortTileItems);
    for (uint32_t j = threadIdx.x; j < items; j += kThreads) {
      const uint32_t k = skey[j], v = sval[j];
      const uint32_t d = (k >> shift) & 255u;
      const uint32_t dst = gbase[d] + j - lstart[d];
      kout[dst] = k;
      vout[dst] = v;
      if (gdst) gdst[dst] = gsrc[v];
    }
    __syncthreads();
    gbase[threadIdx.x] += total;
    __syncthreads();
  }
}

// ---- permuted exclusive scan of counts -----------------------------------
constexpr int kScanItems = 4;

__device__ __forceinline__ uint32_t scan_chunk(uint32_t n) {
  uint32_t per = (n + kSortBlocks - 1) / kSortBlocks;
  const uint32_t step = kThreads * kScanItems;
  return (per + step - 1) / step * step;
}

// With long_partials / long_list set, the same passes also count the splats
// whose tile count exceeds kSerialRecords and write their depth-order
// positions, in depth order, to long_list (their number to *n_long): the list
// the long-segment gradient reduction walks.
__global__ void __launch_bounds__(kThreads)
    scan_partial_kernel(const uint32_t* __restrict__ counts, const uint32_t* __restrict__ perm,
                        uint32_t n, unsigned long long* __restrict__ partials,
                        uint32_t* __restrict__ long_partials) {
  pdl_wait();
  __shared__ unsigned long long wsum[kWarps];
  __shared__ uint32_t wlong[kWarps];
  const uint32_t chunk = scan_chunk(n);
  const uint32_t begin = min(blockIdx.x * chunk, n);
  const uint32_t end = min(begin + chunk, n);
  unsigned long long s = 0;
  uint32_t l = 0;
  for (uint32_t p = begin + threadIdx.x; p < end; p += kThreads) {
    const uint32_t c = counts[perm[p]];
    s += c;
    l += c > kSerialRecords ? 1u : 0u;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    s += __shfl_xor_sync(0xffffffffu, s, o);
    l += __shfl_xor_sync(0xffffffffu, l, o);
  }
  if ((threadIdx.x & 31) == 0) {
    wsum[threadIdx.x >> 5] = s;
    wlong[threadIdx.x >> 5] = l;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long t = 0;
    uint32_t tl = 0;
    for (int k = 0; k < kWarps; ++k) {
      t += wsum[k];
      tl += wlong[k];
    }
    partials[blockIdx.x] = t;
    if (long_partials) long_partials[blockIdx.x] = tl;
  }
}

__global__ void __launch_bounds__(kThreads)
    scan_final_kernel(const uint32_t* __restrict__ counts, const uint32_t* __restrict__ perm,
                      uint32_t n, const unsigned long long* __restrict__ partials,
                      unsigned long long* __restrict__ offsets,
                      const uint32_t* __restrict__ long_partials,
                      uint4* __restrict__ long_list, uint32_t cap,
                      uint32_t* __restrict__ n_clamped, unsigned long long* __restrict__ raw,
                      uint32_t* __restrict__ n_long, uint32_t* __restrict__ status) {
  pdl_wait();
  __shared__ unsigned long long wsum[kWarps], wall[kWarps];
  __shared__ uint32_t wlong[kWarps], wlall[kWarps];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  // carry = sum of the chunks before this CTA's; CTA 0 also writes the totals
  unsigned long long carry = 0, all = 0;
  uint32_t lcarry = 0, lall = 0;
  for (int i = threadIdx.x; i < (int)gridDim.x; i += kThreads) {
    const unsigned long long v = partials[i];
    const uint32_t lv = long_list ? long_partials[i] : 0u;
    if (i < (int)blockIdx.x) {
      carry += v;
      lcarry += lv;
    }
    all += v;
    lall += lv;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    carry += __shfl_xor_sync(0xffffffffu, carry, o);
    lcarry += __shfl_xor_sync(0xffffffffu, lcarry, o);
    all += __shfl_xor_sync(0xffffffffu, all, o);
    lall += __shfl_xor_sync(0xffffffffu, lall, o);
  }
  if (lane == 0) {
    wsum[w] = carry;
    wlong[w] = lcarry;
    wall[w] = all;
    wlall[w] = lall;
  }
  __syncthreads();
  carry = all = 0;
  lcarry = lall = 0;
#pragma unroll
  for (int k = 0; k < kWarps; ++k) {
    carry += wsum[k];
    lcarry += wlong[k];
    all += wall[k];
    lall += wlall[k];
  }
  __syncthreads();
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    *raw = all;
    *n_clamped = (uint32_t)(all < (unsigned long long)cap ? all : cap);
    if (all > (unsigned long long)cap) atomicOr(status, kStatusIsectOverflow);
    if (n_long) *n_long = lall;
  }
  const uint32_t chunk = scan_chunk(n);
  const uint32_t begin = min(blockIdx.x * chunk, n);
  const uint32_t end = min(begin + chunk, n);
  if (begin >= end) return;
  for (uint32_t t0 = begin; t0 < end; t0 += kThreads * kScanItems) {
    uint32_t c[kScanItems], pi[kScanItems];
    unsigned long long s = 0;
    uint32_t lmask = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
      uint32_t p = t0 + threadIdx.x * kScanItems + k;
      pi[k] = p < end ? perm[p] : 0u;
      c[k] = p < end ? counts[pi[k]] : 0u;
      s += c[k];
      lmask |= (c[k] > kSerialRecords ? 1u : 0u) << k;
    }
    const uint32_t ls = __popc(lmask);
    unsigned long long incl = s;
    uint32_t lincl = ls;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      unsigned long long t = __shfl_up_sync(0xffffffffu, incl, o);
      uint32_t tl = __shfl_up_sync(0xffffffffu, lincl, o);
      if (lane >= o) {
        incl += t;
        lincl += tl;
      }
    }
    if (lane == 31) {
      wsum[w] = incl;
      wlong[w] = lincl;
    }
    __syncthreads();
    unsigned long long wbase = 0, tot = 0;
    uint32_t lbase = 0, ltot = 0;
#pragma unroll
    for (int k = 0; k < kWarps; ++k) {
      const unsigned long long v = wsum[k];
      const uint32_t lv = wlong[k];
      if (k < w) {
        wbase += v;
        lbase += lv;
      }
      tot += v;
      ltot += lv;
    }
    unsigned long long excl = carry + wbase + incl - s;
    uint32_t lexcl = lcarry + lbase + lincl - ls;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
      uint32_t p = t0 + threadIdx.x * kScanItems + k;
      const unsigned long long s0 = excl;
      if (p < end) offsets[p] = s0;
      excl += c[k];
      if (long_list && (lmask >> k & 1u)) {
        // {splat, first record, end of its records}, clamped to the capacity
        const unsigned long long cp = cap;
        long_list[lexcl++] = make_uint4(pi[k], (uint32_t)(s0 < cp ? s0 : cp),
                                        (uint32_t)(excl < cp ? excl : cp), 0u);
      }
    }
    carry += tot;
    lcarry += ltot;
    __syncthreads();
  }
}

}  // namespace

int radix_sort_pairs(const uint32_t* kin, const uint32_t* vin, uint32_t* ka, uint32_t* va,
                     uint32_t* kb, uint32_t* vb, uint32_t** out_k, uint32_t** out_v,
                     const uint32_t* n_dev, uint32_t cap, int bits, const uint32_t* gather_src,
                     uint32_t* gather_dst, SortScratch& scratch, cudaStream_t s) {
  const int passes = bits <= 0 ? 1 : (bits + 7) / 8;
  // One CTA per 2048-item tile of the capacity, at most kSortBlocks.
  const uint64_t tiles = ((uint64_t)cap + kSortTileItems - 1) / kSortTileItems;
  const int G = (int)(tiles < 1 ? 1 : (tiles > (uint64_t)kSortBlocks ? kSortBlocks : tiles));
  const uint32_t* src_k = kin;
  const uint32_t* src_v = vin;
  uint32_t* dst_k = ka;
  uint32_t* dst_v = va;
  for (int p = 0; p < passes; ++p) {
    const int shift = 8 * p;
    const bool last = p == passes - 1;
    DS_CUDA(launch_pdl(radix_hist_kernel, dim3(G), dim3(kThreads), 0, s, src_k, n_dev, cap, shift,
                       scratch.hist));
    DS_CUDA(launch_pdl(scan_hist_kernel, dim3(256 / kWarps), dim3(kThreads), 0, s, scratch.hist,
                       G));
    DS_CUDA(launch_pdl(radix_scatter_kernel, dim3(G), dim3(kThreads), 0, s, src_k, src_v,
                       src_v == nullptr ? 1 : 0, dst_k, dst_v, n_dev, cap, shift,
                       (const uint32_t*)scratch.hist, last ? gather_src : nullptr,
                       last ? gather_dst : nullptr));
    *out_k = dst_k;
    *out_v = dst_v;
    src_k = dst_k;
    src_v = dst_v;
    dst_k = (dst_k == ka) ? kb : ka;
    dst_v = (dst_v == va) ? vb : va;
  }
  return cuda_status(cudaGetLastError());
}

int scan_counts_permuted(const uint32_t* counts, const uint32_t* perm, uint32_t n,
                         unsigned long long* offsets, uint32_t* n_clamped,
                         unsigned long long* raw_total, uint32_t cap, uint32_t* status,
                         ScanScratch& scratch, cudaStream_t s, uint4* long_list,
                         uint32_t* n_long) {
  if (long_list && (!scratch.long_partials || !n_long)) return DS_ERR_ARG;
  uint32_t* lp = long_list ? scratch.long_partials : nullptr;
  DS_CUDA(launch_pdl(scan_partial_kernel, dim3(kSortBlocks), dim3(kThreads), 0, s, counts, perm,
                     n, scratch.partials, lp));
  DS_CUDA(launch_pdl(scan_final_kernel, dim3(kSortBlocks), dim3(kThreads), 0, s, counts, perm, n,
                     (const unsigned long long*)scratch.partials, offsets, (const uint32_t*)lp,
                     long_list, cap, n_clamped, raw_total, long_list ? n_long : nullptr, status));
  return cuda_status(cudaGetLastError());
}

}  // namespace ds
