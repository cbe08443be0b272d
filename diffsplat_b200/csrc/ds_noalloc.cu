// Rasterizer forward that allocates no device memory.
//
// Some callers cannot let a library call cudaMalloc: an application that hands
// all device memory to its own pool allocator (a library-side cudaMalloc
// fails or fragments its budget), or a per-frame render loop in which
// cudaMalloc / cudaFree would implicitly synchronise the device and stall the
// frame.  ds_raster_forward_noalloc renders with the same kernels as
// ds_raster_forward, but every intermediate buffer (records, sort keys, tile
// lists, ranges, per-pixel state) lives in one file-scope __device__ array
// that the driver sets aside when the library is loaded and that every GPU
// holds until the process exits.
//
// The array bounds the problem size: at most kMaxSplats splats, an image of at
// most kMaxPixels pixels and kMaxTiles 16x16 tiles, and kMaxIsects
// (tile, splat) pairs; pairs beyond that are dropped (the deepest ones, as
// ds_raster_forward drops them beyond its capacity) and a sticky overflow bit
// is set in the array, which ds_raster_noalloc_status reads and clears.  All
// calls on one device share the array, so calls that overlap on the GPU
// (different streams or host threads) race: issue them on one stream.  The
// first call on each device (and the first after a device reset) looks the
// array's device address up (cudaGetSymbolAddress) with that device current;
// make that first call before any stream capture.
#include <stddef.h>

#include <mutex>

#include "ds_common.cuh"
#include "ds_internal.h"

namespace ds {

namespace {

constexpr int kMaxSplats = 8192;
constexpr int kMaxIsects = 1 << 17;
constexpr int kMaxPixels = 256 * 256;
constexpr int kMaxTiles = 1024;
constexpr int kMaxDevices = 64;

constexpr size_t up256(size_t b) { return (b + 255) / 256 * 256; }

// Sub-buffers, in carving order: 13 per-splat arrays (16 B per splat each,
// enough for the widest), 6 per-pair arrays, 2 per-pixel arrays, tile ranges,
// sort histogram, scan partials and the device scalars: about 5.7 MB.
constexpr size_t kIsectBytes = 4 * (size_t)kMaxIsects;  // each of 6 pair arrays
constexpr size_t kTotalBytes =
    13 * up256(16 * (size_t)kMaxSplats) +
    6 * up256(kIsectBytes) + 2 * up256(4 * (size_t)kMaxPixels) + up256(8 * (size_t)kMaxTiles) +
    up256(4 * 256 * ((size_t)kSortBlocks + 1)) + up256(8 * ((size_t)kSortBlocks + 1)) +
    up256(sizeof(DevScalars));

static __device__ __align__(256) unsigned char g_noalloc_scratch[kTotalBytes];

// The array's device address per device, with the id of the context it was
// looked up in: after a device reset (cudaDeviceReset, or another runtime in
// the process resetting the primary context) the module is loaded again and
// the array may move, so a changed context id triggers a new lookup.
struct ScratchSlot {
  void* ptr = nullptr;
  unsigned long long ctx = 0;
};
std::mutex g_mutex;
ScratchSlot g_slot[kMaxDevices];

using CtxGetCurrentFn = int (*)(void** ctx);
using CtxGetIdFn = int (*)(void* ctx, unsigned long long* id);
CtxGetCurrentFn g_ctx_current = nullptr;
CtxGetIdFn g_ctx_id = nullptr;
bool g_ctx_fns_looked_up = false;

// Id of the calling thread's current context (driver entry points reached
// through the runtime, so the library needs no libcuda link); false when
// there is none or the driver does not offer the calls.  Called under g_mutex.
bool current_ctx_id(unsigned long long* id) {
  if (!g_ctx_fns_looked_up) {
    g_ctx_fns_looked_up = true;
    void* a = nullptr;
    void* b = nullptr;
    cudaDriverEntryPointQueryResult qa, qb;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &a, cudaEnableDefault, &qa) == cudaSuccess &&
        qa == cudaDriverEntryPointSuccess &&
        cudaGetDriverEntryPoint("cuCtxGetId", &b, cudaEnableDefault, &qb) == cudaSuccess &&
        qb == cudaDriverEntryPointSuccess) {
      g_ctx_current = reinterpret_cast<CtxGetCurrentFn>(a);
      g_ctx_id = reinterpret_cast<CtxGetIdFn>(b);
    }
  }
  if (!g_ctx_current || !g_ctx_id) return false;
  void* ctx = nullptr;
  if (g_ctx_current(&ctx) != 0 || !ctx) return false;
  return g_ctx_id(ctx, id) == 0;
}

int scratch_base(void** out) {
  int dev = 0;
  DS_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return DS_ERR_NO_DEVICE;
  std::lock_guard<std::mutex> lock(g_mutex);
  ScratchSlot& slot = g_slot[dev];
  unsigned long long ctx = 0;
  const bool known = current_ctx_id(&ctx);
  if (!slot.ptr || !known || slot.ctx != ctx) {
    void* p = nullptr;
    DS_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    slot.ptr = p;
    // the lookup makes the primary context current if none was
    slot.ctx = current_ctx_id(&ctx) ? ctx : 0;
  }
  *out = slot.ptr;
  return DS_OK;
}

struct Carver {
  unsigned char* p;
  template <typename T>
  T* take(size_t bytes) {
    T* r = reinterpret_cast<T*>(p);
    p += up256(bytes);
    return r;
  }
};

}  // namespace

// Offset of the DevScalars block in the array (the carving order of
// ds_raster_forward_noalloc).
constexpr size_t kScalarsOffset = kTotalBytes - up256(sizeof(DevScalars));

}  // namespace ds

extern "C" int ds_raster_forward_noalloc(const ds_splat2d* in, int width, int height,
                                         float* out_rgb, ds_stream stream) {
  using namespace ds;
  if (!in || !out_rgb || width <= 0 || height <= 0 || in->count < 0) return DS_ERR_ARG;
  if (in->count > kMaxSplats) return DS_ERR_ARG;
  if ((int64_t)width * height > kMaxPixels) return DS_ERR_ARG;
  const int ntx = (width + kTile - 1) / kTile, nty = (height + kTile - 1) / kTile;
  if ((int64_t)ntx * nty > kMaxTiles) return DS_ERR_ARG;
  if (in->count > 0 && !(in->pos_x && in->pos_y && in->pos_z && in->cov_xx && in->cov_xy &&
                         in->cov_yy && in->color_r && in->color_g && in->color_b && in->opacity))
    return DS_ERR_ARG;
  void* base = nullptr;
  DS_TRY(scratch_base(&base));
  Carver c{static_cast<unsigned char*>(base)};
  RasterBuffers rb;
  rb.width = width;
  rb.height = height;
  rb.ntx = ntx;
  rb.nty = nty;
  rb.tiles = ntx * nty;
  rb.max_splats = kMaxSplats;
  rb.cap = kMaxIsects;
  rb.ppt = composite_default_ppt();
  rb.ppt_bwd = rb.ppt;  // forward only: no backward layout to choose
  const size_t n = kMaxSplats;
  rb.rec_a = c.take<float4>(16 * n);
  rb.rec_b = c.take<float4>(16 * n);
  rb.rec_c = c.take<float4>(16 * n);
  rb.rec_idet = c.take<float>(16 * n);
  rb.rect = c.take<ushort4>(16 * n);
  rb.counts = c.take<uint32_t>(16 * n);
  rb.seg_start = c.take<uint32_t>(16 * n);
  rb.depth_keys = c.take<uint32_t>(16 * n);
  rb.depth_k0 = c.take<uint32_t>(16 * n);
  rb.depth_k1 = c.take<uint32_t>(16 * n);
  rb.depth_v0 = c.take<uint32_t>(16 * n);
  rb.depth_v1 = c.take<uint32_t>(16 * n);
  rb.emit_offsets = c.take<unsigned long long>(16 * n);
  rb.tile_k0 = c.take<uint32_t>(kIsectBytes);
  rb.tile_k1 = c.take<uint32_t>(kIsectBytes);
  rb.tile_v0 = c.take<uint32_t>(kIsectBytes);
  rb.tile_v1 = c.take<uint32_t>(kIsectBytes);
  rb.emit_splat = c.take<uint32_t>(kIsectBytes);
  rb.sorted_splat = c.take<uint32_t>(kIsectBytes);
  rb.alphas = c.take<float>(4 * (size_t)kMaxPixels);
  rb.last_ids = c.take<int32_t>(4 * (size_t)kMaxPixels);
  rb.ranges = c.take<int2>(8 * (size_t)kMaxTiles);
  rb.sort.hist = c.take<uint32_t>(4 * 256 * ((size_t)kSortBlocks + 1));
  rb.scan.partials = c.take<unsigned long long>(8 * ((size_t)kSortBlocks + 1));
  rb.scalars = c.take<DevScalars>(sizeof(DevScalars));
  if (reinterpret_cast<unsigned char*>(rb.scalars) !=
      static_cast<unsigned char*>(base) + kScalarsOffset)
    return DS_ERR_INTERNAL;
  // The forward does not produce gradients; these stay unset.
  rb.isect_grad = nullptr;
  rb.g2 = nullptr;
  rb.loss_partials = nullptr;
  cudaStream_t s = (cudaStream_t)stream;
  // The array keeps the previous call's contents: reset the pair and visible
  // counts (the scalars before `status`); the sticky status bits stay until
  // ds_raster_noalloc_status reads them.
  static_assert(offsetof(DevScalars, status) == 2 * sizeof(uint32_t), "DevScalars layout");
  DS_CUDA(cudaMemsetAsync(rb.scalars, 0, offsetof(DevScalars, status), s));
  DS_TRY(raster_prepare_from_splat2d(rb, *in, s));
  DS_TRY(raster_build_lists(rb, in->count, s));
  DS_TRY(raster_composite_forward(rb, out_rgb, nullptr, s));
  return DS_OK;
}

extern "C" int ds_raster_noalloc_status(uint32_t* flags, ds_stream stream) {
  using namespace ds;
  if (!flags) return DS_ERR_ARG;
  void* base = nullptr;
  DS_TRY(scratch_base(&base));
  DevScalars* sc = reinterpret_cast<DevScalars*>(static_cast<unsigned char*>(base) + kScalarsOffset);
  cudaStream_t s = (cudaStream_t)stream;
  uint32_t st = 0;
  DS_CUDA(cudaMemcpyAsync(&st, &sc->status, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  DS_CUDA(cudaMemsetAsync(&sc->status, 0, sizeof(uint32_t), s));
  DS_CUDA(cudaStreamSynchronize(s));
  *flags = st;
  return status_code(st);
}
