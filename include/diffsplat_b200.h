/*
 * diffsplat_b200 -- C ABI of the B200 (sm_100a) differentiable Gaussian-splatting
 * training path.
 *
 * Every entry point takes plain device pointers, sizes and a CUDA stream (as
 * void*), and returns an int status (DS_OK == 0).  Calls that launch work are
 * stream-ordered and asynchronous unless their comment says they synchronise.
 * Buffers passed in are owned by the caller; opaque handles (ds_raster,
 * ds_fitter) own the scratch they allocate and free it in *_destroy.
 *
 * Struct field order and array layouts are those of the reference's SoA types,
 * so a caller holding reference buffers can pass them unchanged:
 *   ds_gaussian3d  <->  Gaussian3DParams / Gaussian3DGrads (src/types/gaussian3d.h:34-120)
 *   ds_splat3d     <->  Splat3DParams / Splat3DGrads       (src/types/splat3d.h:14-51)
 *   ds_splat2d     <->  Splat2DParams / Splat2DGrads       (src/types/splat2d.h:13-45)
 * Higher-order SH buffers are band-major: sh_rest_r[band * count + i].
 * Images are interleaved RGB float [H*W*3], row-major, top row first.
 */
#ifndef DIFFSPLAT_B200_H
#define DIFFSPLAT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DS_ABI_VERSION 1

/* Status codes. */
#define DS_OK 0
#define DS_ERR_ARG 1            /* invalid argument (null pointer, bad size, bad degree) */
#define DS_ERR_OOM 2            /* device allocation failed */
#define DS_ERR_CUDA 3           /* a CUDA runtime call or kernel launch failed */
#define DS_ERR_ISECT_OVERFLOW 4 /* more (tile, splat) pairs than the intersection buffer holds */
#define DS_ERR_STATE 5          /* call made in the wrong state (e.g. step before set_target) */
#define DS_ERR_NO_DEVICE 6      /* no CUDA device, or not an sm_100 device */
#define DS_ERR_INTERNAL 7       /* a device-side consistency check failed (results of the step invalid) */

/* Storage modes for ds_fitter. */
#define DS_STORAGE_FP32 0 /* all attributes, SH and Adam moments in FP32 */
/* DS_STORAGE_BF16: scale, rotation, SH and opacity are rendered from a BF16
 * copy of the FP32 master weights (rewritten after every Adam update, round to
 * nearest); positions stay FP32; Adam m and v are BF16 with stochastic rounding.
 * Transmittance, blending and gradient sums stay FP32. */
#define DS_STORAGE_BF16 1

/* Gradient of the compositing backward with respect to alpha.
 * DS_GRAD_REFERENCE reproduces the reference's recurrence
 * (src/layers/tile_rasterize_layer.cu:518-521), which weighs the colour of the
 * splats behind by T_before instead of dividing it by T_after; it is the true
 * derivative only when no later splat contributes.  DS_GRAD_EXACT is the true
 * derivative (matches finite differences). */
#define DS_GRAD_REFERENCE 0
#define DS_GRAD_EXACT 1

/* Order in which the composite kernels visit tiles (results do not depend on
 * it): the longest tile lists first (default), or raster order. */
#define DS_SCHEDULE_LONGEST_FIRST 0
#define DS_SCHEDULE_RASTER 1

typedef void *ds_stream; /* cudaStream_t; NULL selects the legacy default stream */

typedef struct ds_gaussian3d {
  float *pos_x, *pos_y, *pos_z;
  float *scale_x, *scale_y, *scale_z;       /* log-scale */
  float *rot_w, *rot_x, *rot_y, *rot_z;     /* raw quaternion, normalised in kernel */
  float *sh_dc_r, *sh_dc_g, *sh_dc_b;
  float *sh_rest_r, *sh_rest_g, *sh_rest_b; /* [band*count + i]; NULL when sh_num_bands == 0 */
  float *logit_opacity;
  int32_t count;
  int32_t sh_num_bands; /* 0, 3, 8 or 15 */
} ds_gaussian3d;

typedef struct ds_splat3d {
  float *pos_x, *pos_y, *pos_z;
  float *cov_xx, *cov_xy, *cov_xz;
  float *cov_yy, *cov_yz, *cov_zz;
  float *color_r, *color_g, *color_b;
  float *opacity;
  int32_t count;
} ds_splat3d;

typedef struct ds_splat2d {
  float *pos_x, *pos_y, *pos_z;    /* NDC */
  float *cov_xx, *cov_xy, *cov_yy; /* NDC units */
  float *color_r, *color_g, *color_b;
  float *opacity;
  int32_t count;
} ds_splat2d;

/* Process-wide default gradient mode, used by new raster handles, by
 * ds_fitter_default_config, by ds_project_backward and by the drop-in C++
 * layers.  Initialised from the environment variable DS_GRAD_MODE
 * ("reference" or "exact"; DS_GRAD_REFERENCE when unset). */
int ds_set_default_grad_mode(int mode);
int ds_default_grad_mode(void);

/* Test hook for failure detection (no reference counterpart): after n more
 * successful device allocations, the library's next ones fail as if the
 * device were out of memory, so every create / densify call can be driven
 * through its clean-up path; n < 0 turns this off.  Process-wide. */
int ds_debug_fail_allocations_after(int64_t n);

/* Library information. */
int ds_abi_version(void);
const char *ds_status_string(int status);
/* Returns DS_OK when a device of compute capability 10.x is present. */
int ds_device_check(void);

/* ---- Activation: replaces GaussActivLayer::forward / ::backward
 *      (src/layers/gauss_activ_layer.cu:411-440, :442-476; kernels :37-170, :198-407).
 *      cam_pos is the host array setCameraPosition() stores
 *      (src/layers/gauss_activ_layer.h:33). */
int ds_activ_forward(const ds_gaussian3d *in, int sh_degree, const float cam_pos[3],
                     const ds_splat3d *out, ds_stream stream);
/* Writes (does not accumulate) grad_in; reads the saved forward output `out`
 * for the clamp and sigmoid gates, like the reference. */
int ds_activ_backward(const ds_gaussian3d *in, const ds_splat3d *out, const ds_splat3d *grad_out,
                      int sh_degree, const float cam_pos[3], const ds_gaussian3d *grad_in,
                      ds_stream stream);

/* ---- Projection: replaces PerspProjectLayer::forward / ::backward / ::setCamera
 *      (src/layers/persp_project_layer.cu:278-296, :298-317, :269-274).
 *      pv is the column-major 16-float PV = proj * view that setCamera uploads;
 *      here it is passed per call, so two layers may use different cameras. */
int ds_project_forward(const ds_splat3d *in, const float pv[16], const ds_splat2d *out,
                       ds_stream stream);
int ds_project_backward(const ds_splat3d *in, const float pv[16], const ds_splat2d *grad_out,
                        const ds_splat3d *grad_in, ds_stream stream);
/* Same with a gradient mode: DS_GRAD_EXACT also carries the position
 * dependence of the Jacobian (hence of Cov2D) into dL/dpos, which the
 * reference's backward (persp_project_layer.cu:245-260) leaves out. */
int ds_project_backward_ex(const ds_splat3d *in, const float pv[16], const ds_splat2d *grad_out,
                           const ds_splat3d *grad_in, int grad_mode, ds_stream stream);

/* ---- Tile rasterizer: replaces TileRasterizeLayer (src/layers/tile_rasterize_layer.h:23-60,
 *      .cu:591-617 allocate, :619-633 resize, :637-708 forward, :710-728 backward,
 *      :582-587 getVisibleCount).  The handle owns the intersection buffers. */
typedef struct ds_raster ds_raster;

/* max_isects <= 0 selects the reference's 2^25 pairs. */
int ds_raster_create(int width, int height, int max_splats, int64_t max_isects, ds_raster **out);
int ds_raster_resize(ds_raster *r, int width, int height);
/* DS_GRAD_REFERENCE (default) or DS_GRAD_EXACT for the following backward calls. */
int ds_raster_set_grad_mode(ds_raster *r, int mode);
/* Forward: tile keys, sort, ranges and front-to-back compositing into out_rgb
 * [H*W*3] (overwritten, background black).  Asynchronous: no host sync. */
int ds_raster_forward(ds_raster *r, const ds_splat2d *in, float *out_rgb, ds_stream stream);
/* Backward of the last forward.  ACCUMULATES into grad_in (like the reference's
 * atomicAdd into zeroed buffers), deterministically. */
int ds_raster_backward(ds_raster *r, const ds_splat2d *in, const float *grad_rgb,
                       const ds_splat2d *grad_in, ds_stream stream);
/* Number of splats with a non-empty tile rectangle in the last forward (synchronises). */
int ds_raster_visible_count(ds_raster *r, uint32_t *out);
/* Number of (tile, splat) pairs of the last forward, before clamping to capacity (synchronises). */
int ds_raster_isect_count(ds_raster *r, uint32_t *out);
/* Reads and clears the sticky status bits (synchronises).  Returns
 * DS_ERR_ISECT_OVERFLOW when a forward since the last call overflowed. */
int ds_raster_status(ds_raster *r, uint32_t *flags);
/* Copies internal state of the last forward to host memory (synchronises):
 *   DS_RASTER_KEYS      uint64 [n_isects]  sorted (tile_id << 32 | depth bits) keys
 *   DS_RASTER_IDS       uint32 [n_isects]  sorted splat ids (ascending id within equal keys)
 *   DS_RASTER_RANGES    int32  [2*tiles]   per-tile {start, end}; {0,0} for empty tiles
 *   DS_RASTER_LAST_IDS  int32  [H*W]       sorted-list index of each pixel's last contributor
 *   DS_RASTER_ALPHAS    float  [H*W]       1 - final transmittance
 *   DS_RASTER_COUNTS    uint32 [count]     tiles covered per splat
 *   DS_RASTER_CONICS    float  [count*4]   per splat {a, b, c, opacity}: the inverse of
 *                                          its Splat2D covariance [[a, b], [b, c]] as the
 *                                          compositing evaluates it (reference: computed at
 *                                          batch load, tile_rasterize_layer.cu:260-272);
 *                                          meaningful for splats with a non-zero count */
#define DS_RASTER_KEYS 0
#define DS_RASTER_IDS 1
#define DS_RASTER_RANGES 2
#define DS_RASTER_LAST_IDS 3
#define DS_RASTER_ALPHAS 4
#define DS_RASTER_COUNTS 5
#define DS_RASTER_CONICS 6
int ds_raster_download(ds_raster *r, int what, void *host, int64_t bytes);
int ds_raster_destroy(ds_raster *r);

/* Forward rasterization that allocates no device memory (no counterpart in the
 * reference).  For callers that cannot let a library call cudaMalloc: an
 * application whose own pool allocator owns all device memory, or a per-frame
 * loop in which cudaMalloc / cudaFree would synchronise the device.  Same
 * kernels and same image as ds_raster_create + ds_raster_forward, with every
 * intermediate buffer in one ~5.7 MB __device__ array of the library that each
 * GPU holds until the process exits.  Limits: count <= 8192 splats,
 * width * height <= 65536 pixels, at most 1024 16x16 tiles (DS_ERR_ARG
 * beyond); (tile, splat) pairs beyond 131072 are dropped, the deepest first,
 * exactly as ds_raster_forward drops pairs beyond a 131072-pair capacity, and
 * a sticky overflow bit is set that ds_raster_noalloc_status reports.  All
 * calls on a device share the array, so calls that overlap on the GPU race:
 * issue them on one stream.  The first call on each device, and the first
 * after a device reset, looks up the array's device address; make it before
 * any stream capture.  Asynchronous. */
int ds_raster_forward_noalloc(const ds_splat2d *in, int width, int height, float *out_rgb,
                              ds_stream stream);
/* Reads and clears the sticky status bits of ds_raster_forward_noalloc on the
 * current device (synchronises `stream`; allocates nothing).  Returns
 * DS_ERR_ISECT_OVERFLOW when a call since the last read dropped pairs. */
int ds_raster_noalloc_status(uint32_t *flags, ds_stream stream);

/* ---- Loss: replaces MSELossLayer::forward / ::backward / ::getLoss
 *      (src/layers/mse_loss_layer.cu:85-92, :94-99, :101-105).
 *      L = sum_px sum_c (r - t)^2 / num_pixels  (normalised by pixels, not pixels*3).
 *      ds_mse_forward overwrites *loss (device scalar). */
int ds_mse_forward(const float *pixels, const float *target, int64_t num_pixels, float *loss,
                   ds_stream stream);
int ds_mse_backward(const float *pixels, const float *target, int64_t num_pixels, float *grad,
                    ds_stream stream);

/* ---- Adam: replaces Adam::step (src/optimizers/adam.cu:59-73, kernel :12-37).
 *      All groups are updated by ONE launch.  `step` is the 1-based step count
 *      after increment; bias corrections are computed on the host exactly as
 *      the reference does (1 / (1 - powf(beta, step))). */
typedef struct ds_adam_group {
  float *param;
  const float *grad;
  float *m;
  float *v;
  int64_t n;
  float lr;
} ds_adam_group;
int ds_adam_step(const ds_adam_group *groups, int n_groups, float beta1, float beta2,
                 float epsilon, int step, ds_stream stream);

/* ---- Fused fitter: one training step of ImageFitter::step
 *      (src/pipelines/image_fitter.cpp:103-112: zeroGrad, forward, backward, Adam)
 *      with the layers of src/pipelines/image_fitter.cpp:63-101 fused into a
 *      fixed sequence of kernels that is captured once into a CUDA graph.
 *      Learning rates default to Gaussian3DAdamConfig (src/optimizers/gaussian3d_adam.h:11-19). */
typedef struct ds_fitter ds_fitter;

typedef struct ds_fitter_config {
  int32_t width, height;
  int32_t count;      /* splats */
  int32_t sh_degree;  /* 0..3 */
  int64_t max_isects; /* <= 0: 2^25 */
  float lr_pos, lr_scale, lr_rot, lr_sh_dc, lr_sh_rest, lr_opacity;
  float beta1, beta2, epsilon;
  int32_t storage;   /* DS_STORAGE_FP32 / DS_STORAGE_BF16 */
  int32_t use_graph; /* 1: capture the step into a CUDA graph on first use */
  int32_t grad_mode; /* DS_GRAD_REFERENCE (default) / DS_GRAD_EXACT */
  int32_t schedule;  /* DS_SCHEDULE_LONGEST_FIRST (default) / DS_SCHEDULE_RASTER */
  int32_t capacity;  /* > count: room for densification (ds_fitter_densify); 0 = count */
} ds_fitter_config;

int ds_fitter_default_config(ds_fitter_config *cfg);
int ds_fitter_create(const ds_fitter_config *cfg, ds_fitter **out);
/* Device views of the fitter's FP32 master parameters (write them before the first step). */
int ds_fitter_params(ds_fitter *f, ds_gaussian3d *out);
/* Tells the fitter the masters were written through the ds_fitter_params view
 * (BF16 storage rebuilds its render copy before the next step; FP32: no-op). */
int ds_fitter_params_updated(ds_fitter *f);
/* Copies the target image [H*W*3] from a device pointer. */
int ds_fitter_set_target(ds_fitter *f, const float *target, ds_stream stream);
/* Camera for the following steps (column-major PV and world camera position, host arrays). */
int ds_fitter_set_camera(ds_fitter *f, const float pv[16], const float cam_pos[3],
                         ds_stream stream);
/* Runs n_steps training steps (asynchronous). */
int ds_fitter_step(ds_fitter *f, int n_steps, ds_stream stream);
/* Loss of the most recent step's forward (synchronises the stream). */
int ds_fitter_loss(ds_fitter *f, float *loss, ds_stream stream);
/* Device address of the loss scalar each step writes (float): lets a caller
 * copy it asynchronously, e.g. read step k's loss while step k + 1 runs. */
int ds_fitter_loss_device(ds_fitter *f, float **loss);
/* Device pointer of the rendered image [H*W*3] of the most recent forward. */
int ds_fitter_output(ds_fitter *f, float **image);
int ds_fitter_step_count(ds_fitter *f, int *out);
/* Reads and clears sticky status bits (synchronises). */
int ds_fitter_status(ds_fitter *f, uint32_t *flags);
int ds_fitter_destroy(ds_fitter *f);

/* Inspection hooks of the fused fitter (no reference counterpart: the
 * reference exposes its gradients through GaussActivLayer::getGradInput,
 * src/layers/layer.h:59).  A fitter made by ds_fitter_create_with_grads also
 * writes each step's Gaussian3D gradients, readable through ds_fitter_grads;
 * ds_fitter_moments returns device views of the Adam first/second moments. */
int ds_fitter_create_with_grads(const ds_fitter_config *cfg, ds_fitter **out);
/* One step run eagerly with CUDA events between its stages (synchronises);
 * stage_ms[0..6] = preprocess, depth sort, scan + emission, tile sort + ranges,
 * composite forward, composite backward, backward + Adam.  It advances the
 * optimizer like ds_fitter_step. */
int ds_fitter_profile_step(ds_fitter *f, float *stage_ms, int n_stages, ds_stream stream);
/* out[0] = (tile, splat) pairs, out[1] = visible splats, out[2] = device step
 * count, all of the most recent step (synchronises). */
int ds_fitter_counters(ds_fitter *f, uint64_t *out, int n);
/* Re-runs the composite forward of the most recent step with pair counters
 * (no reference counterpart; measurement only): out[0] = (pixel, splat) pairs
 * that contribute (alpha >= 1/255 before the pixel terminates), out[1] = pairs
 * the kernel evaluates.  Rewrites the same image; synchronises. */
int ds_fitter_pair_stats(ds_fitter *f, uint64_t *out, int n, ds_stream stream);
/* Copies the tile lists and per-pixel state of the most recent step's forward
 * to host memory (synchronises the device), with the codes and layouts of
 * ds_raster_download (DS_RASTER_KEYS .. DS_RASTER_COUNTS).  That forward ran on
 * the parameters as they were before the step's Adam update.  No reference
 * counterpart: the reference keeps these lists inside TileRasterizeLayer
 * (src/layers/tile_rasterize_layer.h:23-60); this hook lets a test compare the
 * fused step's lists with the layer path's. */
int ds_fitter_download(ds_fitter *f, int what, void *host, int64_t bytes);
int ds_fitter_grads(ds_fitter *f, ds_gaussian3d *out);
int ds_fitter_moments(ds_fitter *f, ds_gaussian3d *m, ds_gaussian3d *v);

/* Adaptive density control (no reference counterpart: a TODO of the reference,
 * README.md:10).  A fitter created with capacity > count accumulates, per
 * splat, the norm of its NDC position gradient over the steps in which it was
 * visible.  ds_fitter_densify then rebuilds the splat set in one pass:
 * splats with opacity < min_opacity are pruned; splats whose mean gradient
 * norm is >= grad_threshold are cloned (largest scale <= scale_threshold,
 * world units) or split into two children sampled from their Gaussian with
 * scales / 1.6 (larger ones); survivors keep their Adam moments, new splats
 * start from zero moments; the statistics restart.  The count may not exceed
 * the capacity (DS_ERR_OOM, nothing changed).  FP32 storage, without
 * gradient inspection.  The next step recaptures the graph. */
typedef struct ds_densify_params {
  float grad_threshold;
  float scale_threshold;
  float min_opacity;
  uint32_t seed;
} ds_densify_params;
int ds_fitter_densify(ds_fitter *f, const ds_densify_params *p, int32_t *new_count,
                      ds_stream stream);
/* Device views of the statistics [count]: gradient-norm sums and visible steps. */
int ds_fitter_density_stats(ds_fitter *f, float **grad_accum, uint32_t **visible_steps);

/* ---- Batched fitting (no reference counterpart) ----
 * Many independent ImageFitter-style instances of uneven image size and splat
 * count stepped together: every stage is one launch over all instances, the
 * step is captured once into a CUDA graph.  Splats of all instances share one
 * parameter SoA (ds_batch_params, count = all splats; instance k owns columns
 * [first, first + count) of ds_batch_instance_range); each instance has its
 * own target, camera, image and loss.  tile_size 8, 16 or 32 and
 * pixels_per_thread 1 or 2 select the composite kernels (16 is the
 * reference's tile; other sizes change which splats a tile lists, not the
 * compositing rule).  Default storage is BF16 (FP32 masters). */
typedef struct ds_batch ds_batch;
typedef struct ds_batch_instance {
  int32_t width, height, count, reserved;
} ds_batch_instance;
typedef struct ds_batch_config {
  int32_t instances;
  int32_t sh_degree;
  int64_t max_isects; /* all instances together; <= 0: 2^25 */
  float lr_pos, lr_scale, lr_rot, lr_sh_dc, lr_sh_rest, lr_opacity;
  float beta1, beta2, epsilon;
  int32_t storage;
  int32_t use_graph;
  int32_t grad_mode;
  int32_t schedule;
  int32_t tile_size;         /* 8, 16 or 32 */
  int32_t pixels_per_thread; /* 1 or 2 */
} ds_batch_config;
int ds_batch_default_config(ds_batch_config *cfg);
int ds_batch_create(const ds_batch_config *cfg, const ds_batch_instance *instances,
                    ds_batch **out);
int ds_batch_params(ds_batch *b, ds_gaussian3d *out);
int ds_batch_instance_range(ds_batch *b, int instance, int32_t *first_splat, int32_t *count);
int ds_batch_params_updated(ds_batch *b);
int ds_batch_set_target(ds_batch *b, int instance, const float *target, ds_stream stream);
int ds_batch_set_camera(ds_batch *b, int instance, const float pv[16], const float cam_pos[3],
                        ds_stream stream);
int ds_batch_step(ds_batch *b, int n_steps, ds_stream stream);
/* Per-instance losses of the most recent step (host array [instances]; synchronises). */
int ds_batch_losses(ds_batch *b, float *losses, ds_stream stream);
int ds_batch_output(ds_batch *b, int instance, float **image);
/* out[0] = (tile, splat) pairs, out[1] = visible splats, out[2] = step count (synchronises). */
int ds_batch_counters(ds_batch *b, uint64_t *out, int n);
int ds_batch_status(ds_batch *b, uint32_t *flags);
int ds_batch_destroy(ds_batch *b);

/* ---- BF16 tensor-core kernels of the learned initializer (no reference counterpart) ----
 * ds_gemm_bf16_tn: D[M,N] = A[M,K] . B[N,K]^T with A, B BF16 row-major (K
 * inner, leading dimensions lda / ldb elements, 16-byte aligned rows) on
 * tcgen05 tensor cores with FP32 accumulation.  epilogue 0: FP32 D (ldd);
 * 1: Z = BF16(acc + bias), Y = BF16(gelu(acc + bias)) (ldy); 2: FP32 D = acc +
 * bias.  splits > 1 (epilogue 0 only) splits K over CTAs into `workspace`
 * [splits*M*ldd floats] and sums the splits in order.  *err becomes non-zero
 * if a CTA's pipeline wait timed out (the result is then invalid). */
int ds_gemm_bf16_tn(const void *A, int lda, const void *B, int ldb, int M, int N, int K,
                    int epilogue, float *D, int ldd, void *Y, void *Z, int ldy, const float *bias,
                    int splits, float *workspace, uint32_t *err, ds_stream stream);
/* Polls each pipeline wait of ds_gemm_bf16_tn makes before it gives up and
 * reports through *err (process-wide; 0 restores the default of 2^24, which
 * no healthy pipeline reaches).  A low limit exercises that failure path: the
 * CTAs still let what they issued land before they free their TMEM and
 * shared memory, and the device stays usable.  No reference counterpart. */
int ds_gemm_set_spin_limit(uint32_t polls);
/* 3x3 convolution with padding 1 and stride 1 or 2 on NHWC BF16 tensors:
 * im2col writes col[B*Ho*Wo][Kp] (k = (ky*3 + kx)*C + c, zero for k >= 9C);
 * col2im sums dcol back onto dx[B][H][W][C] and multiplies by gelu'(z) when z
 * is given. */
int ds_im2col_bf16(const void *x, int B, int H, int W, int C, int stride, int Kp, void *col,
                   ds_stream stream);
int ds_col2im_bf16(const float *dcol, int B, int H, int W, int C, int stride, int Kp,
                   const void *z, void *dx, ds_stream stream);
int ds_transpose_bf16(const void *in, int rows, int cols, void *out, ds_stream stream);
/* out[c] = sum_m a[m][c]; workspace holds max_parts * C floats. */
int ds_colsum_bf16(const void *a, int64_t M, int C, float *workspace, int max_parts, float *out,
                   ds_stream stream);
/* AdamW on FP32 master weights (decoupled decay), optional BF16 copy out. */
int ds_adamw(float *p, const float *g, float *m, float *v, int64_t n, float lr, float beta1,
             float beta2, float eps, float weight_decay, int step, void *bf16_out,
             ds_stream stream);
int ds_cast_bf16(const float *in, int64_t n, void *out, ds_stream stream);
/* Initializer head on a G x G grid, 4 splats per cell, 14 channels per splat
 * {dx, dy, dz, log-scale xyz, quaternion wxyz, SH DC rgb, logit}: decode the
 * FP32 head output [B*G*G][56] into field-major parameter rows [14][B*4*G*G]
 * (pos = base + d * step, log-scale = base_log_scale + ls, quaternion =
 * (1,0,0,0) + q), and map parameter gradients back (w_render * g_render +
 * w_l1 * sign(params - target); either term optional) as BF16 [B*G*G][56]. */
int ds_head_decode(const float *out, int B, int G, const float *base, const float step[3],
                   float base_log_scale, float *params, ds_stream stream);
int ds_head_encode_grad(const float *g_render, const float *params, const float *target,
                        float w_render, float w_l1, int B, int G, const float step[3], void *dout,
                        ds_stream stream);

/* ---- Image targets: ImageLoader / ImageSaver (src/io/image_io.h:17-47) ----
 * Decoding on the host: PNG (8-bit, non-interlaced; grey, grey+alpha, RGB,
 * RGBA, palette) and binary PPM / PGM, to 8-bit RGB (JPEG is not supported).
 * ds_image_fit: aspect-preserving fit of a device RGB8 image into a device
 * float canvas [H*W*3] with `padding` pixels of margin, centred, black
 * outside, values / 255 (area filter when shrinking, bilinear when
 * enlarging).  ds_image_write_png: host RGB float in [0, 1] -> 8-bit PNG. */
int ds_image_probe(const char *path, int *width, int *height);
int ds_image_read_rgb8(const char *path, uint8_t *rgb, int64_t capacity, int *width,
                       int *height);
int ds_image_fit(const uint8_t *src_rgb, int src_w, int src_h, int canvas_w, int canvas_h,
                 int padding, float *dst_rgb, int *fit_w, int *fit_h, ds_stream stream);
int ds_image_write_png(const char *path, const float *rgb, int width, int height);

/* ---- Forward-only renderer: SplatRenderer (src/pipelines/splat_renderer.h:17-60) ----
 * render() = GaussActiv -> PerspProject -> TileRasterize forward
 * (src/pipelines/splat_renderer.cpp:84-91) into an owned [H*W*3] image.
 * FP32 storage reads the caller's parameter buffers on every render (keep them
 * alive); BF16 storage converts scale, rotation, SH and opacity into its own
 * BF16 copy at ds_renderer_set_params (positions stay FP32). */
typedef struct ds_renderer ds_renderer;
int ds_renderer_create(int width, int height, int max_splats, int sh_degree, int64_t max_isects,
                       int storage, ds_renderer **out);
int ds_renderer_set_params(ds_renderer *r, const ds_gaussian3d *params, ds_stream stream);
/* setActiveSHDegree: evaluate SH up to `degree` (<= the buffers' degree). */
int ds_renderer_set_sh_degree(ds_renderer *r, int degree);
int ds_renderer_render(ds_renderer *r, const float pv[16], const float cam_pos[3],
                       ds_stream stream);
int ds_renderer_output(ds_renderer *r, float **rgb);
int ds_renderer_resize(ds_renderer *r, int width, int height);
/* out[0] = visible splats, out[1] = (tile, splat) pairs of the last render (synchronises). */
int ds_renderer_counts(ds_renderer *r, uint64_t *out, int n);
int ds_renderer_status(ds_renderer *r, uint32_t *flags);
int ds_renderer_destroy(ds_renderer *r);

/* ---- Scene I/O on the host: PLYLoader / PLYSaver (src/io/ply_io.h:28-57) and
 * SplatUtils::normalizeScene (src/utils/splat_utils.h) ----
 * Splats are arrays of the reference's host record Gaussian3D
 * (src/types/gaussian3d.h:13-21): 59 floats each (pos xyz, log-scale xyz,
 * quaternion wxyz, SH DC rgb, 45 SH-rest floats channel-first, logit opacity).
 * Files are binary little-endian 3DGS PLY in the OpenCV frame; y, z and the
 * quaternion's y, z are negated on read and write (OpenGL frame in memory).
 * Errors (missing file or property, wrong extension, short file) return DS_ERR_ARG. */
int ds_ply_probe(const char *path, int64_t *count, int *sh_degree);
int ds_ply_read(const char *path, float *splats, int64_t capacity, int64_t *count,
                int *sh_degree);
/* Writes x y z f_dc_0..2 f_rest_0..(3K-1) opacity scale_0..2 rot_0..3, K = sh_num_bands. */
int ds_ply_write(const char *path, const float *splats, int64_t count, int sh_num_bands);
/* Centres the positions on their centroid and scales the largest |coordinate|
 * to scene_scale, adding log(scale) to the log-scales. */
int ds_normalize_scene(float *splats, int64_t count, float scene_scale);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* DIFFSPLAT_B200_H */
