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
// (tile, splat) pairs; pairs beyond that are dropped, as the reference drops
// pairs beyond its buffer.  All calls on one device share the array, so calls
// that overlap on the GPU (different streams or host threads) race: issue them
// on one stream.  The first call on each device looks the array's device
// address up (cudaGetSymbolAddress) with that device current; make that first
// call before any stream capture.
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

std::mutex g_mutex;
void* g_scratch_ptr[kMaxDevices] = {};

int scratch_base(void** out) {
  int dev = 0;
  DS_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return DS_ERR_NO_DEVICE;
  std::lock_guard<std::mutex> lock(g_mutex);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    DS_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    g_scratch_ptr[dev] = p;
  }
  *out = g_scratch_ptr[dev];
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
  rb.ppt_bwd = composite_default_ppt_bwd();
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
  // The forward does not produce gradients; these stay unset.
  rb.isect_grad = nullptr;
  rb.g2 = nullptr;
  rb.loss_partials = nullptr;
  cudaStream_t s = (cudaStream_t)stream;
  // The array keeps the previous call's contents: reset the counters.
  DS_CUDA(cudaMemsetAsync(rb.scalars, 0, sizeof(DevScalars), s));
  DS_TRY(raster_prepare_from_splat2d(rb, *in, s));
  DS_TRY(raster_build_lists(rb, in->count, s));
  DS_TRY(raster_composite_forward(rb, out_rgb, nullptr, s));
  return DS_OK;
}
