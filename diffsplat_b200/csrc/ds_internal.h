// Internal host-side declarations shared by the .cu files of libdiffsplat_b200.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <utility>

#include "../../include/diffsplat_b200.h"

namespace ds {

inline int cuda_status(cudaError_t e) {
  if (e == cudaSuccess) return DS_OK;
  if (e == cudaErrorMemoryAllocation) return DS_ERR_OOM;
  return DS_ERR_CUDA;
}

#define DS_TRY(expr)                 \
  do {                               \
    int _st = (expr);                \
    if (_st != DS_OK) return _st;    \
  } while (0)

#define DS_CUDA(expr) DS_TRY(::ds::cuda_status(expr))

// Every device allocation of the library goes through device_alloc, so that a
// test can make the allocations after a given count fail as out of memory
// (ds_debug_fail_allocations_after) and exercise each clean-up path.
cudaError_t device_alloc_bytes(void** p, size_t bytes);
template <typename T>
inline cudaError_t device_alloc(T** p, size_t bytes) {
  return device_alloc_bytes(reinterpret_cast<void**>(p), bytes);
}

// Launches `kernel` with programmatic dependent launch: its CTAs may be
// scheduled while the previous kernel in the stream finishes, and it waits
// for that kernel (pdl_wait) before its first memory access.
template <typename... P, typename... A>
inline cudaError_t launch_pdl(void (*kernel)(P...), dim3 grid, dim3 block, size_t smem,
                              cudaStream_t s, A&&... args) {
  cudaLaunchAttribute attr;
  attr.id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr.val.programmaticStreamSerializationAllowed = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cfg.attrs = &attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, std::forward<A>(args)...);
}

// Small host -> device uploads (cameras) through a ring of pinned slots
// (ds_stage.cu): an upload waits only for the copy that used its slot kSlots
// uploads earlier, never for the stream, and no pending copy sees its source
// change.  A copy from pageable memory would instead return only once the
// stream had reached it.
struct HostStage {
  static constexpr int kSlots = 8;
  static constexpr size_t kSlotBytes = 128;
  unsigned char* host = nullptr;
  cudaEvent_t ev[kSlots] = {};
  int next = 0;
  HostStage() = default;
  HostStage(const HostStage&) = delete;
  HostStage& operator=(const HostStage&) = delete;
  ~HostStage();
  int upload(void* dst, const void* src, size_t bytes, cudaStream_t s);
  void release();
};

// Sticky error bits written by kernels into a device status word.
enum StatusBits : uint32_t {
  kStatusIsectOverflow = 1u << 0,  // more (tile, splat) pairs than the buffer holds
  kStatusBadTile = 1u << 1,        // a sorted pair's tile id lies outside the grid
};

// Status code for sticky StatusBits read back by a status call.
inline int status_code(uint32_t bits) {
  if (bits & kStatusIsectOverflow) return DS_ERR_ISECT_OVERFLOW;
  if (bits & kStatusBadTile) return DS_ERR_INTERNAL;
  return DS_OK;
}

// Layer kernels (ds_activ_project.cu)
int launch_activ_forward(const ds_gaussian3d& in, int degree, const float cam[3],
                         const ds_splat3d& out, cudaStream_t s);
int launch_activ_backward(const ds_gaussian3d& in, const ds_splat3d& saved,
                          const ds_splat3d& gout, int degree, const float cam[3],
                          const ds_gaussian3d& gin, cudaStream_t s);
int launch_project_forward(const ds_splat3d& in, const float pv[16], const ds_splat2d& out,
                           cudaStream_t s);
int launch_project_backward(const ds_splat3d& in, const float pv[16], const ds_splat2d& gout,
                            const ds_splat3d& gin, int mode, cudaStream_t s);

// ---------------------------------------------------------------------------
// Stable LSD radix sort of (uint32 key, uint32 value) pairs (ds_sort.cu).
// The element count is read from device memory so the whole pipeline can be
// captured into a CUDA graph.  Fixed grid of kSortBlocks CTAs.
// ---------------------------------------------------------------------------
constexpr int kSortBlocks = 296;    // 2 x 148 SMs
// Tile grids up to this size sort their pairs by a single stable counting
// pass (ds_raster.cu); larger ones by radix passes over the tile id.
constexpr int kCountSortMaxTiles = 8192;
constexpr int kSortTileItems = 2048;  // items per CTA iteration (8 warps x 32 lanes x 8)

struct SortScratch {
  uint32_t* hist = nullptr;  // [256 * kSortBlocks] counts, then [256] digit totals
};

// Sorts n = min(*n_dev, cap) pairs by key bits [0, bits).  Pass 0 reads
// (kin, vin) and writes (ka, va); later passes alternate (ka, va) <-> (kb, vb).
// kb may alias kin (the input is consumed by pass 0); ka may not.  *out_k /
// *out_v receive the buffers holding the result.  vin == nullptr means the
// input values are 0..n-1.  When gather_src != nullptr, the last pass also
// writes gather_dst[q] = gather_src[value[q]].
int radix_sort_pairs(const uint32_t* kin, const uint32_t* vin, uint32_t* ka, uint32_t* va,
                     uint32_t* kb, uint32_t* vb, uint32_t** out_k, uint32_t** out_v,
                     const uint32_t* n_dev, uint32_t cap, int bits, const uint32_t* gather_src,
                     uint32_t* gather_dst, SortScratch& scratch, cudaStream_t s);

// Exclusive scan of counts gathered through a permutation:
//   offsets[p] = sum_{q < p} counts[perm[q]]   (64-bit),
//   *raw_total = the full sum, *n_clamped = min(raw_total, cap), and the
//   overflow bit is or-ed into *status when raw_total > cap.
// Gradient records of a splat's tiles are contiguous in emission order.  A
// splat with at most kSerialRecords tiles has its records summed by one thread
// in record order; one with more by a warp (lane-strided partial sums, then a
// tree), taken from the list of those splats that the emission scan writes.
constexpr uint32_t kSerialRecords = 8;

struct ScanScratch {
  unsigned long long* partials = nullptr;  // [kSortBlocks + 1]
  uint32_t* long_partials = nullptr;       // [kSortBlocks]; only for the long list
};
// offsets[p] = exclusive sum of counts[perm[q]], q < p.  With long_list set,
// also long_list[0 .. *n_long) = {perm[p], offsets[p], offsets[p] +
// counts[perm[p]]} (offsets clamped to cap) for the positions p with
// counts[perm[p]] > kSerialRecords, ascending in p.
int scan_counts_permuted(const uint32_t* counts, const uint32_t* perm, uint32_t n,
                         unsigned long long* offsets, uint32_t* n_clamped,
                         unsigned long long* raw_total, uint32_t cap, uint32_t* status,
                         ScanScratch& scratch, cudaStream_t s, uint4* long_list = nullptr,
                         uint32_t* n_long = nullptr);

// Device-resident scalars of one rasterizer / fitter.
struct DevScalars {
  uint32_t n_isects;  // (tile, splat) pairs of the last forward, clamped to capacity
  uint32_t visible;   // splats with a non-empty tile rectangle
  uint32_t status;    // sticky StatusBits
  uint32_t ticket;    // CTA-completion counter of the fused loss reduction
  uint32_t n_splats;  // element count of the depth sort
  uint32_t step;      // Adam step count (fitter)
  uint32_t n_long;    // splats with more than kSerialRecords tiles (last emission scan)
  uint32_t sort_ticket;  // CTA-completion counter of the tile-offset scan
  unsigned long long n_isects_raw;  // unclamped pair count
  float loss;
  float pad2;
  unsigned long long pairs[2];  // counting forward: contributing, tested (pixel, splat) pairs
  // Backward layout of the last forward (ppt_bwd == 0): its hits and their
  // contributing lanes summed over the CTAs, the last CTA's decision
  unsigned long long mode_hits, mode_lanes;
  uint32_t mode_ticket;
  uint32_t bwd_ppt;  // 2: two pixels per thread; otherwise one
};

// ---------------------------------------------------------------------------
// Rasterizer state (ds_raster.cu), shared by the layer API and the fitter.
// ---------------------------------------------------------------------------
// One fitting instance of a batch: its image, its tile grid and where its
// tiles and pixels start in the batch-wide tile and pixel arrays.
struct InstGeom {
  int width, height, ntx, nty;
  int tile_off, pix_off, splat_off, count;
};

struct RasterBuffers {
  int width = 0, height = 0, ntx = 0, nty = 0, tiles = 0;
  int max_splats = 0;
  int64_t cap = 0;  // intersection capacity
  int grad_mode = DS_GRAD_REFERENCE;
  int ppt = 2;      // pixels per thread of the composite forward (1, 2 or 4)
  // pixels per thread of the composite backward (1, 2 or 4), or 0: chosen
  // per forward, 2 when its hits covered the warps' pixel blocks densely and 1
  // otherwise (single-instance 16-pixel tiles; DevScalars::bwd_ppt)
  int ppt_bwd = 2;
  int schedule = DS_SCHEDULE_LONGEST_FIRST;  // composite tile order
  int tile_size = 16;  // pixels per tile edge: 16 (reference); batches may use 8 or 32

  // Batch mode (several independent instances in one set of buffers): set
  // together, null for a single instance.  Tiles and pixels are the
  // concatenation of the instances' grids and images.
  const uint16_t* inst_of_splat = nullptr;  // [max_splats]
  const uint16_t* tile_inst = nullptr;      // [tiles]
  const InstGeom* geom = nullptr;           // [instances]
  int instances = 0;

  // per splat
  float4* rec_a = nullptr;
  float4* rec_b = nullptr;
  float4* rec_c = nullptr;
  float* rec_idet = nullptr;
  ushort4* rect = nullptr;     // tile rectangle {x0, x1, y0, y1}
  uint32_t* counts = nullptr;  // tiles per splat (0 = invisible)
  uint32_t* seg_start = nullptr;  // first emission index of each splat
  uint4* long_list = nullptr;  // {splat, first record, record end} of splats with long segments
  uint32_t* depth_keys = nullptr;  // depth key of each splat (0xffffffff when invisible)
  uint32_t* depth_k0 = nullptr;    // ping-pong buffers of the depth sort
  uint32_t* depth_k1 = nullptr;
  uint32_t* depth_v0 = nullptr;
  uint32_t* depth_v1 = nullptr;
  unsigned long long* emit_offsets = nullptr;  // exclusive scan of counts in depth order
  float* g2 = nullptr;  // [9][max_splats] per-splat Splat2D gradient sums (fitter path)

  // per intersection
  uint32_t* tile_k0 = nullptr;
  uint32_t* tile_k1 = nullptr;
  uint32_t* tile_v0 = nullptr;
  uint32_t* tile_v1 = nullptr;
  uint32_t* emit_splat = nullptr;  // splat id of each emission slot
  uint32_t* sorted_splat = nullptr;
  float* isect_grad = nullptr;  // [cap * 9] per-(tile, splat) gradient partials

  // results of the last sort (point into the ping-pong buffers)
  uint32_t* sorted_tile = nullptr;
  uint32_t* sorted_emit = nullptr;  // radix path: emission index of each sorted pair
  uint32_t* depth_perm = nullptr;         // depth-sorted splat ids
  uint32_t* depth_sorted_keys = nullptr;  // their depth keys

  // Counting sort of the pairs by tile (grids of at most kCountSortMaxTiles
  // tiles; null: the radix path): per-chunk tile counts, then their column
  // prefix [count_chunks][tiles], and the per-tile totals.
  uint32_t* tile_hist = nullptr;
  uint32_t* tile_totals = nullptr;
  int count_chunks = 0;

  // per tile / pixel
  unsigned long long* tile_bound = nullptr;  // see GradSegments
  int2* ranges = nullptr;
  int32_t* tile_order = nullptr;  // composite schedule: tiles by descending list length
  float* alphas = nullptr;
  int32_t* last_ids = nullptr;
  float* loss_partials = nullptr;  // [tiles]

  DevScalars* scalars = nullptr;

  SortScratch sort;
  ScanScratch scan;
};

// Where a consumer finds splat i's gradient records: [start[i], start[i] +
// counts[i]) clamped to cap, 9 floats each, record k for the k-th tile of the
// splat's rectangle in row-major order.  The composite backward writes no
// record for a pair that lies in its tile's list after the tile's last
// contributing splat (nothing reaches a pixel from there); tile_bound[t] is 1 +
// the (depth key << 32 | splat id) of that last splat, 0 when none: record k
// counts only when the splat's key is below the bound of its tile.
struct GradSegments {
  const float* rec;
  const uint32_t* counts;
  const uint32_t* start;
  uint32_t cap;
  const unsigned long long* tile_bound;
  const uint32_t* depth_keys;
  const ushort4* rect;
  int ntx;
  const uint16_t* inst_of_splat;  // batches: tile ids are batch-wide
  const InstGeom* geom;
};
inline GradSegments grad_segments(const RasterBuffers& rb) {
  return GradSegments{rb.isect_grad, rb.counts, rb.seg_start, (uint32_t)rb.cap, rb.tile_bound,
                      rb.depth_keys, rb.rect, rb.ntx, rb.inst_of_splat, rb.geom};
}

#ifdef __CUDACC__
__device__ __forceinline__ unsigned long long seg_key(const GradSegments& g, uint32_t i) {
  return ((unsigned long long)g.depth_keys[i] << 32) | i;
}
// First tile id of the splat's rectangle and its row pitch.
__device__ __forceinline__ void seg_origin(const GradSegments& g, uint32_t i, const ushort4& r,
                                           uint32_t& row0, uint32_t& pitch) {
  uint32_t base = 0;
  pitch = (uint32_t)g.ntx;
  if (g.geom) {
    const InstGeom gg = g.geom[g.inst_of_splat[i]];
    base = (uint32_t)gg.tile_off;
    pitch = (uint32_t)gg.ntx;
  }
  row0 = base + (uint32_t)r.z * pitch + r.x;
}
#endif

int raster_alloc(RasterBuffers& rb, int width, int height, int max_splats, int64_t cap);
// Pixels per thread of the composite kernels; DS_COMPOSITE_PPT=1|2|4 overrides
// the default (a tuning knob: results are identical for every value).
int composite_default_ppt();
int composite_default_ppt_bwd();
// Composite CTA schedule: longest tile lists first (default) or raster order
// (DS_TILE_SCHEDULE=raster).
bool composite_longest_first();
int raster_resize(RasterBuffers& rb, int width, int height);
// Batch-mode allocation: `tiles` tiles of tile_size^2 pixels over `pixels`
// pixels in all (the concatenated instance grids); the geometry arrays are set
// by the caller.
int raster_alloc_batch(RasterBuffers& rb, int64_t pixels, int tiles, int tile_size,
                       int max_splats, int64_t cap);
void raster_free(RasterBuffers& rb);

// Everything after the per-splat records exist: depth sort, emission, tile
// sort, ranges.  Records, rect, counts and depth_keys must be filled for n splats.
// with_long_list: also write rb.long_list / scalars->n_long (callers that
// reduce gradients afterwards).
int raster_build_lists(RasterBuffers& rb, int n, cudaStream_t s, cudaEvent_t* ev = nullptr,
                       bool with_long_list = false);

// Copies the state of the last forward to host memory (synchronises the
// device); `what` is one of DS_RASTER_KEYS .. DS_RASTER_COUNTS and n_splats the
// splat count of that forward.
int raster_download(const RasterBuffers& rb, int n_splats, int what, void* host, int64_t bytes);

// Composite forward.  When target != nullptr the per-tile squared error is
// also accumulated and reduced into rb.scalars->loss (L = sum / pixels).
// Forward that also counts (pixel, splat) pairs into scalars->pairs (which it
// zeroes first): [0] pairs that contribute (alpha >= 1/255 before the pixel
// terminates), [1] pairs the kernel evaluates (pixel alive, splat inside the
// warp's acceptance box).  Outputs are those of raster_composite_forward.
int raster_composite_count(RasterBuffers& rb, float* out_rgb, cudaStream_t s);
int raster_composite_forward(RasterBuffers& rb, float* out_rgb, const float* target,
                             cudaStream_t s);
// Composite backward into rb.isect_grad.  dL/dpixel is read from grad_rgb, or,
// when grad_rgb == nullptr, computed as 2/P (image - target).
int raster_composite_backward(RasterBuffers& rb, const float* image, const float* grad_rgb,
                              const float* target, cudaStream_t s);

// Layer-API preprocess from Splat2D SoA, and reduction of isect_grad into Splat2D grads.
int raster_prepare_from_splat2d(RasterBuffers& rb, const ds_splat2d& in, cudaStream_t s);
int raster_reduce_grads(RasterBuffers& rb, const ds_splat2d& gin, int n, cudaStream_t s);
// The sums of the long segments only (the splats on rb.long_list), written to
// rb.g2[k * n + i]; the fitters' backward kernel sums the short segments
// itself from grad_segments(rb).
int raster_reduce_long_grads(RasterBuffers& rb, int n, cudaStream_t s);

// Losses and Adam (ds_loss_adam.cu)
int launch_mse_forward(const float* px, const float* tgt, int64_t npix, float* loss,
                       float* partials, uint32_t* ticket, cudaStream_t s);
int launch_mse_backward(const float* px, const float* tgt, int64_t npix, float* grad,
                        cudaStream_t s);
int launch_adam_multi(const ds_adam_group* groups, int n_groups, float beta1, float beta2,
                      float eps, float bc1, float bc2, cudaStream_t s);

}  // namespace ds
