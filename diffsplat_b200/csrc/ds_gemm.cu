// BF16 tensor-core GEMM for sm_100a (tcgen05 + TMA + TMEM) and the
// convolution helpers of the learned initializer.  No reference counterpart.
//
//   D[M, N] = A[M, K] . B[N, K]^T      A, B BF16, K-major (row-major, K inner)
//
// One CTA per 128 x BN output tile (BN = 32, 64, 128 or 256), 4 warps:
//   warp 0 lane 0  TMA producer: 128 x 64 A and BN x 64 B tiles, 128-byte
//                  swizzle, into a 4-stage shared-memory ring (full/empty
//                  mbarriers with transaction counts)
//   warp 1 lane 0  MMA issuer: tcgen05.mma kind::f16 (BF16 in, FP32 accumulate
//                  in TMEM), four K=16 steps per stage; tcgen05.commit frees
//                  the stage and finally signals the epilogue
//   warps 0-3      epilogue: tcgen05.ld 32 lanes x 32 columns per warp and
//                  step, fused bias / GELU, stores to global memory
// Every mbarrier wait is bounded; on timeout the CTA records an error code,
// drains what it issued (bounded again), frees its TMEM and returns.  The
// pipeline waits poll up to a runtime limit (ds_gemm_set_spin_limit); the
// drain always polls up to kSpinLimit, so the copies and MMAs a CTA issued
// have landed before it frees its TMEM and shared memory even when the
// pipeline limit was set low.
// Split-K (blockIdx.z) writes FP32 partials that gemm_reduce_splits sums in
// a fixed order.
#include <cuda.h>
#include <cuda_bf16.h>
#include <stdint.h>

#include <algorithm>
#include <mutex>

#include "ds_common.cuh"
#include "ds_internal.h"

namespace ds {
namespace {

constexpr int kBM = 128, kBK = 64, kStages = 4, kGemmThreads = 128;
constexpr uint32_t kSpinLimit = 1u << 24;  // default pipeline limit and the drain's limit
uint32_t g_spin_limit = kSpinLimit;

enum Epilogue : int { kEpiF32 = 0, kEpiBiasGeluBf16 = 1, kEpiBiasF32 = 2 };

struct GemmArgs {
  int M, N, K;
  int kb_per_split;   // K blocks of 64 per split
  float* D;           // kEpiF32 / kEpiBiasF32: [splits][M][ldd]
  int ldd;
  __nv_bfloat16* Y;   // kEpiBiasGeluBf16: gelu(acc + bias)   [M][ldy]
  __nv_bfloat16* Z;   // kEpiBiasGeluBf16: acc + bias         [M][ldy]
  int ldy;
  const float* bias;  // [N] or null
  uint32_t* err;      // set non-zero when a wait times out
  uint32_t spin;      // polls per pipeline wait
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

// Bounded wait for the phase with the given parity; false on timeout.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity,
                                          uint32_t limit = kSpinLimit) {
  const uint32_t a = smem_u32(bar);
  for (uint32_t it = 0; it < limit; ++it) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(a), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, uint64_t* bar,
                                            int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, "
      "{%3, %4}], [%2];" ::"r"(smem_u32(dst)),
      "l"((uint64_t)map), "r"(smem_u32(bar)), "r"(x), "r"(y)
      : "memory");
}

// K-major operand tile in shared memory, 128-byte swizzle: rows of 64 BF16
// (128 B), 8-row groups 1024 B apart.
__device__ __forceinline__ uint64_t smem_desc_sw128(uint32_t addr) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFFu);        // start address
  d |= (uint64_t)1u << 16;                        // leading byte offset (16 B, unused)
  d |= (uint64_t)(1024u >> 4) << 32;              // stride byte offset
  d |= (uint64_t)1u << 46;                        // descriptor version (sm_100)
  d |= (uint64_t)2u << 61;                        // 128-byte swizzle
  return d;
}

// kind::f16 instruction descriptor: BF16 A and B, FP32 D, both K-major.
__host__ __device__ constexpr uint32_t instr_desc_bf16(int m, int n) {
  return (1u << 4)                     // D format F32
         | (1u << 7)                   // A format BF16
         | (1u << 10)                  // B format BF16
         | ((uint32_t)(n >> 3) << 17)  // N
         | ((uint32_t)(m >> 4) << 24); // M
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc,
                                          uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
      "%12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, "
      "%30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
        "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]),
        "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// GELU with the tanh form: 0.5 x (1 + tanh(sqrt(2/pi) (x + 0.044715 x^3))).
__device__ __forceinline__ float gelu(float x) {
  const float u = 0.7978845608f * (x + 0.044715f * x * x * x);
  return 0.5f * x * (1.f + tanhf(u));
}

__device__ __forceinline__ float gelu_grad(float x) {
  const float u = 0.7978845608f * (x + 0.044715f * x * x * x);
  const float t = tanhf(u);
  const float du = 0.7978845608f * (1.f + 3.f * 0.044715f * x * x);
  return 0.5f * (1.f + t) + 0.5f * x * (1.f - t * t) * du;
}

template <int BN, int EPI>
__global__ void __launch_bounds__(kGemmThreads, 1)
    gemm_bf16_tn_kernel(const __grid_constant__ CUtensorMap mapA,
                        const __grid_constant__ CUtensorMap mapB, GemmArgs g) {
  constexpr uint32_t kBytesA = kBM * kBK * 2, kBytesB = BN * kBK * 2;
  constexpr uint32_t kTmemCols = BN < 32 ? 32 : BN;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint8_t* tileA = smem;
  uint8_t* tileB = smem + kStages * kBytesA;
  uint64_t* full = (uint64_t*)(tileB + kStages * kBytesB);
  uint64_t* empty = full + kStages;
  uint64_t* done = empty + kStages;
  uint32_t* tmem_slot = (uint32_t*)(done + 1);
  __shared__ int failed;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.x * kBM, n0 = blockIdx.y * BN;
  const int kb_total = (g.K + kBK - 1) / kBK;
  const int kb0 = blockIdx.z * g.kb_per_split;
  const int kb1 = min(kb_total, kb0 + g.kb_per_split);
  const int nkb = max(kb1 - kb0, 0);

  if (threadIdx.x == 0) {
    failed = 0;
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(done, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tmem_slot)),
                 "r"(kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  int issued = 0;
  if (warp == 0 && lane == 0) {
    // producer
    for (int i = 0; i < nkb; ++i) {
      const int s = i % kStages;
      const uint32_t ph = (uint32_t)(i / kStages) & 1u;
      if (!mbar_wait(&empty[s], ph ^ 1u, g.spin)) {
        atomicExch(&failed, 1);
        break;
      }
      mbar_expect_tx(&full[s], kBytesA + kBytesB);
      const int k = (kb0 + i) * kBK;
      tma_load_2d(tileA + s * kBytesA, &mapA, &full[s], k, m0);
      tma_load_2d(tileB + s * kBytesB, &mapB, &full[s], k, n0);
      ++issued;
    }
  } else if (warp == 1 && lane == 0) {
    // MMA issuer
    constexpr uint32_t idesc = instr_desc_bf16(kBM, BN);
    for (int i = 0; i < nkb; ++i) {
      const int s = i % kStages;
      const uint32_t ph = (uint32_t)(i / kStages) & 1u;
      if (!mbar_wait(&full[s], ph, g.spin)) {
        atomicExch(&failed, 1);
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t a = smem_u32(tileA + s * kBytesA), b = smem_u32(tileB + s * kBytesB);
#pragma unroll
      for (int kk = 0; kk < kBK / 16; ++kk)
        umma_bf16(tmem, smem_desc_sw128(a + kk * 32), smem_desc_sw128(b + kk * 32), idesc,
                  (i > 0 || kk > 0) ? 1u : 0u);
      umma_commit(&empty[s]);
    }
    umma_commit(done);
  }
  __syncwarp();

  // epilogue: every warp reads its 32 TMEM lanes (= rows m0 + 32 warp + lane)
  const bool ok = __all_sync(0xffffffffu, mbar_wait(done, 0, g.spin));
  if (!ok) atomicExch(&failed, 1);
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const int row = m0 + warp * 32 + lane;
  if (ok && nkb > 0) {
#pragma unroll 1
    for (int c0 = 0; c0 < BN; c0 += 32) {
      uint32_t r[32];
      tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, r);
      if (row < g.M) {
        if (EPI == kEpiBiasGeluBf16) {
          __nv_bfloat16* yrow = g.Y + (size_t)row * g.ldy;
          __nv_bfloat16* zrow = g.Z + (size_t)row * g.ldy;
#pragma unroll
          for (int j = 0; j < 32; j += 2) {
            const int col = n0 + c0 + j;
            if (col + 1 < g.N) {
              const float z0 = __uint_as_float(r[j]) + (g.bias ? g.bias[col] : 0.f);
              const float z1 = __uint_as_float(r[j + 1]) + (g.bias ? g.bias[col + 1] : 0.f);
              *reinterpret_cast<__nv_bfloat162*>(zrow + col) = __floats2bfloat162_rn(z0, z1);
              *reinterpret_cast<__nv_bfloat162*>(yrow + col) =
                  __floats2bfloat162_rn(gelu(z0), gelu(z1));
            } else if (col < g.N) {
              const float z0 = __uint_as_float(r[j]) + (g.bias ? g.bias[col] : 0.f);
              zrow[col] = __float2bfloat16_rn(z0);
              yrow[col] = __float2bfloat16_rn(gelu(z0));
            }
          }
        } else {
          float* drow = g.D + ((size_t)blockIdx.z * g.M + row) * g.ldd;
#pragma unroll
          for (int j = 0; j < 32; ++j) {
            const int col = n0 + c0 + j;
            if (col < g.N) {
              float v = __uint_as_float(r[j]);
              if (EPI == kEpiBiasF32 && g.bias) v += g.bias[col];
              drow[col] = v;
            }
          }
        }
      }
    }
  } else if (nkb == 0 && row < g.M && EPI != kEpiBiasGeluBf16) {
    // empty K range of a split: its partial is zero
    float* drow = g.D + ((size_t)blockIdx.z * g.M + row) * g.ldd;
    for (int col = n0; col < min(g.N, n0 + BN); ++col) drow[col] = 0.f;
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (failed) {
    // Drain before freeing TMEM and shared memory: the copies still in flight
    // (at most the last kStages issued: an earlier stage was reused only
    // after its copy had landed and been consumed) and the MMAs the issuer
    // committed to `done`.
    if (warp == 0 && lane == 0) {
      for (int i = max(0, issued - kStages); i < issued; ++i)
        mbar_wait(&full[i % kStages], (uint32_t)(i / kStages) & 1u, kSpinLimit);
      mbar_wait(done, 0, kSpinLimit);
      atomicOr(g.err, 1u);
    }
    __syncthreads();
  }
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(kTmemCols));
  }
}

// Sum of the split-K partials in split order: D[M][ldd] = sum_s P[s][M][ldd].
__global__ void gemm_reduce_splits(const float* __restrict__ P, float* __restrict__ D, int M,
                                   int N, int ldd, int splits) {
  const int64_t total = (int64_t)M * N;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = i / N, c = i - r * N;
    float s = 0.f;
    for (int k = 0; k < splits; ++k) s += P[((int64_t)k * M + r) * ldd + c];
    D[r * ldd + c] = s;
  }
}

using EncodeFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                              const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                              const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                              CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeFn encode_fn() {
  static EncodeFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (EncodeFn)p;
  });
  return fn;
}

// 2-D BF16 tensor map of a row-major [rows][cols] matrix with leading dimension
// ld elements, box {64, box_rows}, 128-byte swizzle, zero fill out of bounds.
int make_map(CUtensorMap* map, const void* base, int rows, int cols, int ld, int box_rows) {
  EncodeFn fn = encode_fn();
  if (!fn) return DS_ERR_CUDA;
  if (((uintptr_t)base & 15) || (ld * 2) % 16) return DS_ERR_ARG;
  cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
  cuuint32_t box[2] = {(cuuint32_t)kBK, (cuuint32_t)box_rows};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides,
                  box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? DS_OK : DS_ERR_ARG;
}

template <int BN, int EPI>
int launch_gemm(const CUtensorMap& ma, const CUtensorMap& mb, const GemmArgs& g, int splits,
                cudaStream_t s) {
  constexpr size_t smem = 1024 + kStages * (kBM * kBK * 2 + BN * kBK * 2) + 256;
  static std::once_flag once;
  static cudaError_t attr = cudaSuccess;
  std::call_once(once, [] {
    attr = cudaFuncSetAttribute(gemm_bf16_tn_kernel<BN, EPI>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  });
  DS_CUDA(attr);
  dim3 grid((g.M + kBM - 1) / kBM, (g.N + BN - 1) / BN, splits);
  gemm_bf16_tn_kernel<BN, EPI><<<grid, kGemmThreads, smem, s>>>(ma, mb, g);
  return cuda_status(cudaGetLastError());
}

template <int EPI>
int gemm_dispatch(const CUtensorMap& ma, const CUtensorMap& mb, const GemmArgs& g, int bn,
                  int splits, cudaStream_t s) {
  switch (bn) {
    case 32: return launch_gemm<32, EPI>(ma, mb, g, splits, s);
    case 64: return launch_gemm<64, EPI>(ma, mb, g, splits, s);
    case 128: return launch_gemm<128, EPI>(ma, mb, g, splits, s);
    default: return launch_gemm<256, EPI>(ma, mb, g, splits, s);
  }
}

}  // namespace
}  // namespace ds


// ---- convolution helpers (NHWC BF16 activations, 3x3 kernels, padding 1) ----
namespace ds {
namespace {

// col[m][k], m = (b, oy, ox), k = tap * C + c (tap = ky * 3 + kx), zero for
// k >= 9C and for taps outside the image.
__global__ void im2col_kernel(const __nv_bfloat16* __restrict__ x, int B, int H, int W, int C,
                              int stride, int Ho, int Wo, int Kp, __nv_bfloat16* __restrict__ col) {
  const int64_t total = (int64_t)B * Ho * Wo * Kp;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int k = (int)(i % Kp);
    const int64_t m = i / Kp;
    const int ox = (int)(m % Wo), oy = (int)((m / Wo) % Ho), b = (int)(m / ((int64_t)Wo * Ho));
    __nv_bfloat16 v = __float2bfloat16_rn(0.f);
    if (k < 9 * C) {
      const int tap = k / C, c = k - tap * C;
      const int iy = oy * stride - 1 + tap / 3, ix = ox * stride - 1 + tap % 3;
      if (iy >= 0 && iy < H && ix >= 0 && ix < W) v = x[(((int64_t)b * H + iy) * W + ix) * C + c];
    }
    col[i] = v;
  }
}

// dx[b][iy][ix][c] = sum over the taps that read (iy, ix) of dcol[m][tap * C + c],
// times gelu'(z[b][iy][ix][c]) when z is given (the producing layer's GELU).
__global__ void col2im_kernel(const float* __restrict__ dcol, int B, int H, int W, int C,
                              int stride, int Ho, int Wo, int Kp,
                              const __nv_bfloat16* __restrict__ z, __nv_bfloat16* __restrict__ dx) {
  const int64_t total = (int64_t)B * H * W * C;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int c = (int)(i % C);
    const int64_t p = i / C;
    const int ix = (int)(p % W), iy = (int)((p / W) % H), b = (int)(p / ((int64_t)W * H));
    float s = 0.f;
    for (int ky = 0; ky < 3; ++ky) {
      const int ty = iy + 1 - ky;
      if (ty < 0 || ty % stride) continue;
      const int oy = ty / stride;
      if (oy >= Ho) continue;
      for (int kx = 0; kx < 3; ++kx) {
        const int tx = ix + 1 - kx;
        if (tx < 0 || tx % stride) continue;
        const int ox = tx / stride;
        if (ox >= Wo) continue;
        const int64_t m = ((int64_t)b * Ho + oy) * Wo + ox;
        s += dcol[m * Kp + (ky * 3 + kx) * C + c];
      }
    }
    if (z) s *= gelu_grad(__bfloat162float(z[i]));
    dx[i] = __float2bfloat16_rn(s);
  }
}

// out[c][r] = in[r][c] through 32 x 32 shared-memory tiles (blockIdx.x over
// row tiles, which may exceed the 65535 limit of gridDim.y).
__global__ void transpose_bf16_kernel(const __nv_bfloat16* __restrict__ in, int rows, int cols,
                                      __nv_bfloat16* __restrict__ out) {
  __shared__ __nv_bfloat16 t[32][33];
  const int r0 = blockIdx.x * 32, c0 = blockIdx.y * 32;
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int r = r0 + k, c = c0 + threadIdx.x;
    if (r < rows && c < cols) t[k][threadIdx.x] = in[(int64_t)r * cols + c];
  }
  __syncthreads();
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int c = c0 + k, r = r0 + threadIdx.x;
    if (r < rows && c < cols) out[(int64_t)c * rows + r] = t[threadIdx.x][k];
  }
}

// Column sums of a [M][C] BF16 matrix in two fixed-order passes.
__global__ void colsum_partial_kernel(const __nv_bfloat16* __restrict__ a, int64_t M, int C,
                                      int chunk, float* __restrict__ part) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= C) return;
  const int64_t r0 = (int64_t)blockIdx.y * chunk, r1 = min(M, r0 + chunk);
  float s = 0.f;
  for (int64_t r = r0; r < r1; ++r) s += __bfloat162float(a[r * C + c]);
  part[(int64_t)blockIdx.y * C + c] = s;
}

__global__ void colsum_final_kernel(const float* __restrict__ part, int parts, int C,
                                    float* __restrict__ out) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= C) return;
  float s = 0.f;
  for (int k = 0; k < parts; ++k) s += part[(int64_t)k * C + c];
  out[c] = s;
}

// AdamW (decoupled weight decay) on FP32 master weights; writes the BF16
// copy the GEMMs read.
__global__ void adamw_kernel(float* __restrict__ p, const float* __restrict__ g,
                             float* __restrict__ m, float* __restrict__ v, int64_t n, float lr,
                             float b1, float b2, float eps, float wd, float bc1, float bc2,
                             __nv_bfloat16* __restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    float w = p[i] * (1.f - lr * wd);
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w -= lr * (mi * bc1) / (sqrtf(vi * bc2) + eps);
    p[i] = w;
    if (out) out[i] = __float2bfloat16_rn(w);
  }
}

__global__ void cast_bf16_kernel(const float* __restrict__ in, int64_t n,
                                 __nv_bfloat16* __restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    out[i] = __float2bfloat16_rn(in[i]);
}

// Head of the learned initializer: per cell (i, j) of a G x G grid, 4 splats of
// 14 channels {dx, dy, dz, log-scale xyz, quaternion wxyz, SH DC rgb, logit}.
// Splat s = (i * G + j) * 4 + q of image b gets
//   pos = base[s] + (dx, dy, dz) * step_xyz,  log-scale = base_ls + ls,
//   quaternion = (1, 0, 0, 0) + q, DC and logit as predicted,
// written to the field-major [14][B * S] parameter rows (S = 4 G^2).
__global__ void head_decode_kernel(const float* __restrict__ out, int B, int G,
                                   const float* __restrict__ base, float3 step, float base_ls,
                                   float* __restrict__ params) {
  const int S = 4 * G * G;
  const int64_t total = (int64_t)B * S;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int s = (int)(t % S);
    const int cell = s >> 2, q = s & 3;
    const int64_t b = t / S;
    const float* o = out + ((int64_t)b * G * G + cell) * 56 + q * 14;
    const int64_t n = total;
    params[0 * n + t] = base[3 * s + 0] + o[0] * step.x;
    params[1 * n + t] = base[3 * s + 1] + o[1] * step.y;
    params[2 * n + t] = base[3 * s + 2] + o[2] * step.z;
    for (int k = 3; k < 6; ++k) params[k * n + t] = base_ls + o[k];
    params[6 * n + t] = 1.f + o[6];
    for (int k = 7; k < 14; ++k) params[k * n + t] = o[k];
  }
}

// Gradient of the head output from parameter gradients (transpose of the
// decode), combined with an L1 term: dparams = w_render * g_render +
// w_l1 * sign(params - target), as BF16 [B * G * G][56].
__global__ void head_encode_grad_kernel(const float* __restrict__ g_render,
                                        const float* __restrict__ params,
                                        const float* __restrict__ target, float w_render,
                                        float w_l1, int B, int G, float3 step,
                                        __nv_bfloat16* __restrict__ dout) {
  const int S = 4 * G * G;
  const int64_t total = (int64_t)B * S;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int s = (int)(t % S);
    const int cell = s >> 2, q = s & 3;
    const int64_t b = t / S;
    __nv_bfloat16* o = dout + ((int64_t)b * G * G + cell) * 56 + q * 14;
    for (int k = 0; k < 14; ++k) {
      const int64_t i = (int64_t)k * total + t;
      float g = g_render ? w_render * g_render[i] : 0.f;
      if (target) {
        const float d = params[i] - target[i];
        g += w_l1 * (d > 0.f ? 1.f : (d < 0.f ? -1.f : 0.f));
      }
      if (k == 0) g *= step.x;
      if (k == 1) g *= step.y;
      if (k == 2) g *= step.z;
      o[k] = __float2bfloat16_rn(g);
    }
  }
}

unsigned grid_for(int64_t n) {
  const int64_t b = (n + 255) / 256;
  return (unsigned)(b < 148 * 32 ? (b > 0 ? b : 1) : 148 * 32);
}

}  // namespace
}  // namespace ds

extern "C" {

int ds_gemm_bf16_tn(const void* A, int lda, const void* B, int ldb, int M, int N, int K,
                    int epilogue, float* D, int ldd, void* Y, void* Z, int ldy, const float* bias,
                    int splits, float* workspace, uint32_t* err, ds_stream stream) {
  if (!A || !B || M <= 0 || N <= 0 || K <= 0 || !err) return DS_ERR_ARG;
  if (epilogue < 0 || epilogue > 2) return DS_ERR_ARG;
  if (epilogue == ds::kEpiBiasGeluBf16 && (!Y || !Z || ldy < N)) return DS_ERR_ARG;
  if (epilogue != ds::kEpiBiasGeluBf16 && (!D || ldd < N)) return DS_ERR_ARG;
  if (splits < 1) splits = 1;
  if (splits > 1 && (epilogue != ds::kEpiF32 || !workspace)) return DS_ERR_ARG;
  // Widest tile that covers N, narrowed while the grid leaves SMs idle.
  int bn = N <= 32 ? 32 : N <= 64 ? 64 : N <= 128 ? 128 : 256;
  const int64_t mt = (M + ds::kBM - 1) / ds::kBM;
  int sms = 148;
  {
    int dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess)
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  }
  while (bn > 64 && mt * ((N + bn - 1) / bn) * splits < sms) bn /= 2;
  CUtensorMap ma, mb;
  DS_TRY(ds::make_map(&ma, A, M, K, lda, ds::kBM));
  DS_TRY(ds::make_map(&mb, B, N, K, ldb, bn));
  const int kb_total = (K + ds::kBK - 1) / ds::kBK;
  if (splits > kb_total) splits = kb_total;
  ds::GemmArgs g{};
  g.M = M;
  g.N = N;
  g.K = K;
  g.kb_per_split = (kb_total + splits - 1) / splits;
  splits = (kb_total + g.kb_per_split - 1) / g.kb_per_split;
  g.D = splits > 1 ? workspace : D;
  g.ldd = ldd;
  g.Y = (__nv_bfloat16*)Y;
  g.Z = (__nv_bfloat16*)Z;
  g.ldy = ldy;
  g.bias = bias;
  g.err = err;
  g.spin = ds::g_spin_limit;
  cudaStream_t s = (cudaStream_t)stream;
  int st;
  switch (epilogue) {
    case ds::kEpiBiasGeluBf16: st = ds::gemm_dispatch<ds::kEpiBiasGeluBf16>(ma, mb, g, bn, 1, s); break;
    case ds::kEpiBiasF32: st = ds::gemm_dispatch<ds::kEpiBiasF32>(ma, mb, g, bn, 1, s); break;
    default: st = ds::gemm_dispatch<ds::kEpiF32>(ma, mb, g, bn, splits, s); break;
  }
  DS_TRY(st);
  if (splits > 1) {
    ds::gemm_reduce_splits<<<ds::grid_for((int64_t)M * N), 256, 0, s>>>(workspace, D, M, N, ldd,
                                                                        splits);
    DS_CUDA(cudaGetLastError());
  }
  return DS_OK;
}

int ds_gemm_set_spin_limit(uint32_t polls) {
  ds::g_spin_limit = polls == 0 ? ds::kSpinLimit : polls;
  return DS_OK;
}

int ds_im2col_bf16(const void* x, int B, int H, int W, int C, int stride, int Kp, void* col,
                   ds_stream stream) {
  if (!x || !col || B <= 0 || H <= 0 || W <= 0 || C <= 0 || (stride != 1 && stride != 2) ||
      Kp < 9 * C)
    return DS_ERR_ARG;
  const int Ho = (H - 1) / stride + 1, Wo = (W - 1) / stride + 1;
  const int64_t n = (int64_t)B * Ho * Wo * Kp;
  ds::im2col_kernel<<<ds::grid_for(n), 256, 0, (cudaStream_t)stream>>>(
      (const __nv_bfloat16*)x, B, H, W, C, stride, Ho, Wo, Kp, (__nv_bfloat16*)col);
  return ds::cuda_status(cudaGetLastError());
}

int ds_col2im_bf16(const float* dcol, int B, int H, int W, int C, int stride, int Kp,
                   const void* z, void* dx, ds_stream stream) {
  if (!dcol || !dx || B <= 0 || H <= 0 || W <= 0 || C <= 0 || (stride != 1 && stride != 2) ||
      Kp < 9 * C)
    return DS_ERR_ARG;
  const int Ho = (H - 1) / stride + 1, Wo = (W - 1) / stride + 1;
  const int64_t n = (int64_t)B * H * W * C;
  ds::col2im_kernel<<<ds::grid_for(n), 256, 0, (cudaStream_t)stream>>>(
      dcol, B, H, W, C, stride, Ho, Wo, Kp, (const __nv_bfloat16*)z, (__nv_bfloat16*)dx);
  return ds::cuda_status(cudaGetLastError());
}

int ds_transpose_bf16(const void* in, int rows, int cols, void* out, ds_stream stream) {
  if (!in || !out || rows <= 0 || cols <= 0) return DS_ERR_ARG;
  if ((cols + 31) / 32 > 65535) return DS_ERR_ARG;
  dim3 grid((rows + 31) / 32, (cols + 31) / 32);
  ds::transpose_bf16_kernel<<<grid, dim3(32, 8), 0, (cudaStream_t)stream>>>(
      (const __nv_bfloat16*)in, rows, cols, (__nv_bfloat16*)out);
  return ds::cuda_status(cudaGetLastError());
}

int ds_colsum_bf16(const void* a, int64_t M, int C, float* workspace, int max_parts, float* out,
                   ds_stream stream) {
  if (!a || !out || !workspace || M <= 0 || C <= 0 || max_parts < 1) return DS_ERR_ARG;
  const int chunk = (int)std::max<int64_t>(256, (M + max_parts - 1) / max_parts);
  const int parts = (int)((M + chunk - 1) / chunk);
  cudaStream_t s = (cudaStream_t)stream;
  ds::colsum_partial_kernel<<<dim3((C + 63) / 64, parts), 64, 0, s>>>(
      (const __nv_bfloat16*)a, M, C, chunk, workspace);
  ds::colsum_final_kernel<<<(C + 63) / 64, 64, 0, s>>>(workspace, parts, C, out);
  return ds::cuda_status(cudaGetLastError());
}

int ds_adamw(float* p, const float* g, float* m, float* v, int64_t n, float lr, float beta1,
             float beta2, float eps, float weight_decay, int step, void* bf16_out,
             ds_stream stream) {
  if (!p || !g || !m || !v || n <= 0 || step < 1) return DS_ERR_ARG;
  const float bc1 = 1.f / (1.f - powf(beta1, (float)step));
  const float bc2 = 1.f / (1.f - powf(beta2, (float)step));
  ds::adamw_kernel<<<ds::grid_for(n), 256, 0, (cudaStream_t)stream>>>(
      p, g, m, v, n, lr, beta1, beta2, eps, weight_decay, bc1, bc2, (__nv_bfloat16*)bf16_out);
  return ds::cuda_status(cudaGetLastError());
}

int ds_head_decode(const float* out, int B, int G, const float* base, const float step[3],
                   float base_log_scale, float* params, ds_stream stream) {
  if (!out || !base || !step || !params || B <= 0 || G <= 0) return DS_ERR_ARG;
  const int64_t n = (int64_t)B * 4 * G * G;
  ds::head_decode_kernel<<<ds::grid_for(n), 256, 0, (cudaStream_t)stream>>>(
      out, B, G, base, make_float3(step[0], step[1], step[2]), base_log_scale, params);
  return ds::cuda_status(cudaGetLastError());
}

int ds_head_encode_grad(const float* g_render, const float* params, const float* target,
                        float w_render, float w_l1, int B, int G, const float step[3], void* dout,
                        ds_stream stream) {
  if (!params || !step || !dout || B <= 0 || G <= 0) return DS_ERR_ARG;
  const int64_t n = (int64_t)B * 4 * G * G;
  ds::head_encode_grad_kernel<<<ds::grid_for(n), 256, 0, (cudaStream_t)stream>>>(
      g_render, params, target, w_render, w_l1, B, G, make_float3(step[0], step[1], step[2]),
      (__nv_bfloat16*)dout);
  return ds::cuda_status(cudaGetLastError());
}

int ds_cast_bf16(const float* in, int64_t n, void* out, ds_stream stream) {
  if (!in || !out || n <= 0) return DS_ERR_ARG;
  ds::cast_bf16_kernel<<<ds::grid_for(n), 256, 0, (cudaStream_t)stream>>>(in, n,
                                                                         (__nv_bfloat16*)out);
  return ds::cuda_status(cudaGetLastError());
}

}  // extern "C"
