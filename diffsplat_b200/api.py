"""Python front end of the C ABI, operating on CUDA torch tensors.

SoA tensors are field-major 2-D float32 tensors on the GPU:
  Gaussian3D  [14 + 3K, n]  pos xyz, log-scale xyz, quat wxyz, sh_dc rgb, logit,
                            sh_rest r (K rows), g (K rows), b (K rows)
  Splat3D     [13, n]       pos xyz, cov xx xy xz yy yz zz, rgb, opacity
  Splat2D     [10, n]       ndc xyz, cov xx xy yy, rgb, opacity
(the row orders of the reference's SoA types, src/types/*.h, with the SH rest
moved after the logit so the 14 scalar fields are contiguous).  Images are
[H, W, 3] float32.  Torch provides device memory and the stream; every
computation runs in libdiffsplat_b200.so.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib as L
from .scenes import sh_bands

# row index of each Gaussian3D struct field in the [14 + 3K, n] layout
_G3_ROWS = {"pos_x": 0, "pos_y": 1, "pos_z": 2, "scale_x": 3, "scale_y": 4, "scale_z": 5,
            "rot_w": 6, "rot_x": 7, "rot_y": 8, "rot_z": 9, "sh_dc_r": 10, "sh_dc_g": 11,
            "sh_dc_b": 12, "logit_opacity": 13}


def _stream(stream=None) -> int:
    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream


def _check2d(t: torch.Tensor, rows: int | None = None) -> None:
    if not (t.is_cuda and t.dtype == torch.float32 and t.dim() == 2 and t.is_contiguous()):
        raise ValueError("expected a contiguous float32 CUDA tensor [rows, n]")
    if rows is not None and t.shape[0] != rows:
        raise ValueError(f"expected {rows} rows, got {t.shape[0]}")


def g3_view(t: torch.Tensor, bands: int) -> L.Gaussian3D:
    _check2d(t, 14 + 3 * bands)
    n = t.shape[1]
    base = t.data_ptr()
    g = L.Gaussian3D()
    for name, row in _G3_ROWS.items():
        setattr(g, name, base + 4 * row * n)
    if bands > 0:
        g.sh_rest_r = base + 4 * 14 * n
        g.sh_rest_g = base + 4 * (14 + bands) * n
        g.sh_rest_b = base + 4 * (14 + 2 * bands) * n
    g.count = n
    g.sh_num_bands = bands
    return g


def g3_tensor_from_view(g: L.Gaussian3D) -> torch.Tensor:
    """Wraps a contiguous Gaussian3D allocation (as laid out by ds_fitter) as a
    [14 + 3K, n] tensor view without copying."""
    n, K = g.count, g.sh_num_bands
    rows = 14 + 3 * K
    # ds_fitter carves pos..logit (14 rows) then rest r, g, b: same as _G3_ROWS except
    # the logit row, which precedes the rest in both layouts.
    ptr = g.pos_x
    if g.logit_opacity != ptr + 4 * 13 * n:
        raise ValueError("Gaussian3D view is not in the contiguous fitter layout")
    return _wrap_device(ptr, (rows, n))


def _wrap_device(ptr: int, shape) -> torch.Tensor:
    numel = int(np.prod(shape))

    class _Holder:
        __cuda_array_interface__ = {
            "shape": tuple(shape), "typestr": "<f4", "data": (ptr, False), "version": 3,
            "strides": None}

    return torch.as_tensor(_Holder(), device="cuda").view(*shape) if numel else torch.empty(
        shape, device="cuda")


def s3_view(t: torch.Tensor) -> L.Splat3D:
    _check2d(t, 13)
    n = t.shape[1]
    s = L.Splat3D()
    for k, name in enumerate(L.SPLAT3D_FIELDS):
        setattr(s, name, t.data_ptr() + 4 * k * n)
    s.count = n
    return s


def s2_view(t: torch.Tensor) -> L.Splat2D:
    _check2d(t, 10)
    n = t.shape[1]
    s = L.Splat2D()
    for k, name in enumerate(L.SPLAT2D_FIELDS):
        setattr(s, name, t.data_ptr() + 4 * k * n)
    s.count = n
    return s


# ---- GaussActivLayer ---------------------------------------------------------------
def activ_forward(params: torch.Tensor, degree: int, cam_pos, out: torch.Tensor | None = None,
                  stream=None) -> torch.Tensor:
    bands = params.shape[0] - 14
    if bands % 3:
        raise ValueError("params rows must be 14 + 3K")
    n = params.shape[1]
    if out is None:
        out = torch.zeros((13, n), device=params.device, dtype=torch.float32)
    L.call("ds_activ_forward", C.byref(g3_view(params, bands // 3)), degree,
           L.fptr(cam_pos), C.byref(s3_view(out)), _stream(stream))
    return out


def activ_backward(params, saved_out, grad_out, degree: int, cam_pos, grad_in=None, stream=None):
    bands = (params.shape[0] - 14) // 3
    if grad_in is None:
        grad_in = torch.zeros_like(params)
    L.call("ds_activ_backward", C.byref(g3_view(params, bands)), C.byref(s3_view(saved_out)),
           C.byref(s3_view(grad_out)), degree, L.fptr(cam_pos), C.byref(g3_view(grad_in, bands)),
           _stream(stream))
    return grad_in


# ---- PerspProjectLayer ---------------------------------------------------------------
def project_forward(s3: torch.Tensor, pv, out: torch.Tensor | None = None, stream=None):
    if out is None:
        out = torch.zeros((10, s3.shape[1]), device=s3.device, dtype=torch.float32)
    L.call("ds_project_forward", C.byref(s3_view(s3)), L.fptr(pv), C.byref(s2_view(out)),
           _stream(stream))
    return out


def project_backward(s3: torch.Tensor, pv, grad_out: torch.Tensor, grad_in=None, stream=None,
                     grad_mode: int = L.DS_GRAD_REFERENCE):
    if grad_in is None:
        grad_in = torch.zeros((13, s3.shape[1]), device=s3.device, dtype=torch.float32)
    L.call("ds_project_backward_ex", C.byref(s3_view(s3)), L.fptr(pv),
           C.byref(s2_view(grad_out)), C.byref(s3_view(grad_in)), grad_mode, _stream(stream))
    return grad_in


# ---- TileRasterizeLayer ----------------------------------------------------------------
class Rasterizer:
    """Owns a ds_raster handle (the reference's TileRasterizeLayer state)."""

    def __init__(self, width: int, height: int, max_splats: int, max_isects: int = 0):
        h = C.c_void_p()
        L.call("ds_raster_create", width, height, max_splats, max_isects, C.byref(h))
        self.h = h
        self.width, self.height = width, height
        self.tiles = ((width + 15) // 16) * ((height + 15) // 16)

    def set_grad_mode(self, mode: int) -> None:
        L.call("ds_raster_set_grad_mode", self.h, mode)

    def close(self):
        if self.h:
            L.lib().ds_raster_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def forward(self, s2: torch.Tensor, out: torch.Tensor | None = None, stream=None):
        if out is None:
            out = torch.empty((self.height, self.width, 3), device=s2.device, dtype=torch.float32)
        L.call("ds_raster_forward", self.h, C.byref(s2_view(s2)), out.data_ptr(), _stream(stream))
        return out

    def backward(self, s2: torch.Tensor, grad_rgb: torch.Tensor, grad_in=None, stream=None):
        if grad_in is None:
            grad_in = torch.zeros_like(s2)
        L.call("ds_raster_backward", self.h, C.byref(s2_view(s2)), grad_rgb.data_ptr(),
               C.byref(s2_view(grad_in)), _stream(stream))
        return grad_in

    def visible_count(self) -> int:
        v = C.c_uint32()
        L.call("ds_raster_visible_count", self.h, C.byref(v))
        return v.value

    def isect_count(self) -> int:
        v = C.c_uint32()
        L.call("ds_raster_isect_count", self.h, C.byref(v))
        return v.value

    def status(self) -> tuple[int, int]:
        v = C.c_uint32()
        code = L.lib().ds_raster_status(self.h, C.byref(v))
        return code, v.value

    def download(self, what: int, n_splats: int = 0) -> np.ndarray:
        n = min(self.isect_count(), 1 << 31)
        px = self.width * self.height
        spec = {L.DS_RASTER_KEYS: (np.uint64, n), L.DS_RASTER_IDS: (np.uint32, n),
                L.DS_RASTER_RANGES: (np.int32, 2 * self.tiles),
                L.DS_RASTER_LAST_IDS: (np.int32, px), L.DS_RASTER_ALPHAS: (np.float32, px),
                L.DS_RASTER_COUNTS: (np.uint32, n_splats),
                L.DS_RASTER_CONICS: (np.float32, 4 * n_splats)}[what]
        arr = np.zeros(max(spec[1], 1), spec[0])
        L.call("ds_raster_download", self.h, what, arr.ctypes.data, arr.nbytes)
        return arr[:spec[1]]


# ---- MSELossLayer --------------------------------------------------------------------
def mse_forward(pixels: torch.Tensor, target: torch.Tensor, stream=None) -> torch.Tensor:
    loss = torch.empty(1, device=pixels.device, dtype=torch.float32)
    L.call("ds_mse_forward", pixels.data_ptr(), target.data_ptr(), pixels.numel() // 3,
           loss.data_ptr(), _stream(stream))
    return loss


def mse_backward(pixels: torch.Tensor, target: torch.Tensor, stream=None) -> torch.Tensor:
    grad = torch.empty_like(pixels)
    L.call("ds_mse_backward", pixels.data_ptr(), target.data_ptr(), pixels.numel() // 3,
           grad.data_ptr(), _stream(stream))
    return grad


# ---- Adam --------------------------------------------------------------------------------
def adam_step(groups, step: int, beta1=0.9, beta2=0.999, eps=1e-8, stream=None) -> None:
    """groups: iterable of (param, grad, m, v, lr) float32 CUDA tensors."""
    gs = list(groups)
    arr = (L.AdamGroup * max(len(gs), 1))()
    for k, (p, g, m, v, lr) in enumerate(gs):
        arr[k] = L.AdamGroup(p.data_ptr(), g.data_ptr(), m.data_ptr(), v.data_ptr(), p.numel(),
                             float(lr))
    L.call("ds_adam_step", arr, len(gs), beta1, beta2, eps, step, _stream(stream))


# ---- fused fitter ----------------------------------------------------------------------
class _CountView:
    """uint32 device vector view (cuda array interface)."""

    def __init__(self, ptr: int, n: int):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<u4", "data": (ptr, False),
                                          "version": 3, "strides": None}


class Fitter:
    """Owns a ds_fitter (the graph-captured ImageFitter::step)."""

    def __init__(self, width: int, height: int, count: int, sh_degree: int = 0, lrs=None,
                 max_isects: int = 0, use_graph: bool = True, keep_grads: bool = False,
                 storage: int = L.DS_STORAGE_FP32, betas=(0.9, 0.999), eps: float = 1e-8,
                 grad_mode: int = L.DS_GRAD_REFERENCE, schedule: int | None = None,
                 capacity: int = 0):
        cfg = L.FitterConfig()
        L.call("ds_fitter_default_config", C.byref(cfg))
        cfg.width, cfg.height, cfg.count, cfg.sh_degree = width, height, count, sh_degree
        cfg.max_isects = max_isects
        if lrs is not None:
            (cfg.lr_pos, cfg.lr_scale, cfg.lr_rot, cfg.lr_sh_dc, cfg.lr_sh_rest,
             cfg.lr_opacity) = lrs
        cfg.beta1, cfg.beta2 = betas
        cfg.epsilon = eps
        cfg.storage = storage
        cfg.use_graph = 1 if use_graph else 0
        cfg.grad_mode = grad_mode
        if schedule is not None:
            cfg.schedule = schedule
        cfg.capacity = capacity
        h = C.c_void_p()
        L.call("ds_fitter_create_with_grads" if keep_grads else "ds_fitter_create", C.byref(cfg),
               C.byref(h))
        self.h = h
        self.width, self.height, self.count, self.sh_degree = width, height, count, sh_degree
        self.bands = sh_bands(sh_degree)
        g = L.Gaussian3D()
        L.call("ds_fitter_params", self.h, C.byref(g))
        self.params = g3_tensor_from_view(g)
        self.keep_grads = keep_grads

    def close(self):
        if self.h:
            L.lib().ds_fitter_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_params(self, params) -> None:
        self.params.copy_(torch.as_tensor(params, device="cuda"))
        L.call("ds_fitter_params_updated", self.h)

    def densify(self, grad_threshold: float, scale_threshold: float, min_opacity: float = 0.005,
                seed: int = 0, stream=None) -> int:
        """Prune / clone / split from the accumulated gradient statistics (needs
        capacity > count at creation); returns the new splat count."""
        p = L.DensifyParams(grad_threshold, scale_threshold, min_opacity, seed)
        n = C.c_int32()
        L.call("ds_fitter_densify", self.h, C.byref(p), C.byref(n), _stream(stream))
        g = L.Gaussian3D()
        L.call("ds_fitter_params", self.h, C.byref(g))
        self.params = g3_tensor_from_view(g)
        self.count = n.value
        return n.value

    def density_stats(self):
        """(gradient-norm sums, visible steps) per splat as CUDA tensors."""
        a, c = C.c_void_p(), C.c_void_p()
        L.call("ds_fitter_density_stats", self.h, C.byref(a), C.byref(c))
        g = _wrap_device(a.value, (self.count,))
        cnt = torch.as_tensor(_CountView(c.value, self.count), device="cuda")
        return g, cnt

    def set_target(self, target: torch.Tensor, stream=None) -> None:
        target = target.contiguous()
        L.call("ds_fitter_set_target", self.h, target.data_ptr(), _stream(stream))
        self._target = target

    def set_camera(self, pv, cam_pos, stream=None) -> None:
        L.call("ds_fitter_set_camera", self.h, L.fptr(pv), L.fptr(cam_pos), _stream(stream))

    def step(self, n: int = 1, stream=None) -> None:
        L.call("ds_fitter_step", self.h, n, _stream(stream))

    def loss(self, stream=None) -> float:
        v = C.c_float()
        L.call("ds_fitter_loss", self.h, C.byref(v), _stream(stream))
        return v.value

    def image(self) -> torch.Tensor:
        p = C.c_void_p()
        L.call("ds_fitter_output", self.h, C.byref(p))
        return _wrap_device(p.value, (self.height, self.width, 3))

    def loss_device(self) -> torch.Tensor:
        """The device scalar each step writes its loss to (float32 [1] view)."""
        p = C.c_void_p()
        L.call("ds_fitter_loss_device", self.h, C.byref(p))
        return _wrap_device(p.value, (1,))

    def grads(self) -> torch.Tensor:
        g = L.Gaussian3D()
        L.call("ds_fitter_grads", self.h, C.byref(g))
        return g3_tensor_from_view(g)

    def moments(self):
        m, v = L.Gaussian3D(), L.Gaussian3D()
        L.call("ds_fitter_moments", self.h, C.byref(m), C.byref(v))
        return g3_tensor_from_view(m), g3_tensor_from_view(v)

    def status(self) -> tuple[int, int]:
        v = C.c_uint32()
        code = L.lib().ds_fitter_status(self.h, C.byref(v))
        return code, v.value

    STAGES = ("preprocess", "depth_sort", "scan_emit", "tile_sort_ranges", "composite_fwd",
              "composite_bwd", "backward_adam")

    def profile_step(self, stream=None) -> dict:
        """One eager step with CUDA events between stages; returns ms per stage."""
        ms = (C.c_float * 7)()
        L.call("ds_fitter_profile_step", self.h, ms, 7, _stream(stream))
        return dict(zip(self.STAGES, list(ms)))

    def counters(self) -> dict:
        out = (C.c_uint64 * 3)()
        L.call("ds_fitter_counters", self.h, out, 3)
        return {"n_isects": int(out[0]), "visible": int(out[1]), "step": int(out[2])}

    def download(self, what: int) -> np.ndarray:
        """Tile lists / per-pixel state of the most recent step's forward (the
        DS_RASTER_* codes of Rasterizer.download)."""
        n = min(self.counters()["n_isects"], 1 << 31)
        px = self.width * self.height
        tiles = ((self.width + 15) // 16) * ((self.height + 15) // 16)
        spec = {L.DS_RASTER_KEYS: (np.uint64, n), L.DS_RASTER_IDS: (np.uint32, n),
                L.DS_RASTER_RANGES: (np.int32, 2 * tiles),
                L.DS_RASTER_LAST_IDS: (np.int32, px), L.DS_RASTER_ALPHAS: (np.float32, px),
                L.DS_RASTER_COUNTS: (np.uint32, self.count),
                L.DS_RASTER_CONICS: (np.float32, 4 * self.count)}[what]
        arr = np.zeros(max(spec[1], 1), spec[0])
        L.call("ds_fitter_download", self.h, what, arr.ctypes.data, arr.nbytes)
        return arr[:spec[1]]

    def pair_stats(self) -> dict:
        """(pixel, splat) pairs of the most recent step's composite: those that
        contribute and those the kernel evaluates."""
        out = (C.c_uint64 * 2)()
        L.call("ds_fitter_pair_stats", self.h, out, 2, _stream())
        return {"contributing": int(out[0]), "evaluated": int(out[1])}


class Renderer:
    """Owns a ds_renderer: the forward-only SplatRenderer path."""

    def __init__(self, width: int, height: int, max_splats: int, sh_degree: int = 0,
                 max_isects: int = 0, storage: int = L.DS_STORAGE_FP32):
        h = C.c_void_p()
        L.call("ds_renderer_create", width, height, max_splats, sh_degree, max_isects, storage,
               C.byref(h))
        self.h = h
        self.width, self.height, self.sh_degree = width, height, sh_degree
        self.bands = sh_bands(sh_degree)
        self._params = None

    def close(self):
        if self.h:
            L.call("ds_renderer_destroy", self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_params(self, params: torch.Tensor, stream=None) -> None:
        """params: contiguous float32 CUDA tensor [14 + 3K, n] (kept referenced)."""
        g = g3_view(params, self.bands)
        L.call("ds_renderer_set_params", self.h, C.byref(g), _stream(stream))
        self._params = params

    def set_sh_degree(self, degree: int) -> None:
        L.call("ds_renderer_set_sh_degree", self.h, degree)

    def render(self, pv, cam_pos, stream=None) -> torch.Tensor:
        L.call("ds_renderer_render", self.h, L.fptr(pv), L.fptr(cam_pos), _stream(stream))
        return self.image()

    def image(self) -> torch.Tensor:
        p = C.c_void_p()
        L.call("ds_renderer_output", self.h, C.byref(p))
        return _wrap_device(p.value, (self.height, self.width, 3))

    def resize(self, width: int, height: int) -> None:
        L.call("ds_renderer_resize", self.h, width, height)
        self.width, self.height = width, height

    def counts(self) -> dict:
        out = (C.c_uint64 * 2)()
        L.call("ds_renderer_counts", self.h, out, 2)
        return {"visible": int(out[0]), "n_isects": int(out[1])}

    def status(self) -> tuple[int, int]:
        flags = C.c_uint32()
        code = L.lib().ds_renderer_status(self.h, C.byref(flags))
        return code, int(flags.value)


# ---- scene I/O (host) --------------------------------------------------------

G3_RECORD = 59  # floats of the reference's host Gaussian3D record


def records_to_params(rec: np.ndarray, sh_degree: int) -> np.ndarray:
    """[n, 59] Gaussian3D records -> [14 + 3K, n] parameter rows (SH rest band-major)."""
    K = sh_bands(sh_degree)
    n = rec.shape[0]
    P = np.zeros((14 + 3 * K, n), np.float32)
    P[0:13] = rec[:, 0:13].T
    P[13] = rec[:, 58]
    P[14:14 + 3 * K] = rec[:, 13:13 + 3 * K].T
    return P


def params_to_records(P: np.ndarray) -> np.ndarray:
    K = (P.shape[0] - 14) // 3
    rec = np.zeros((P.shape[1], G3_RECORD), np.float32)
    rec[:, 0:13] = P[0:13].T
    rec[:, 58] = P[13]
    rec[:, 13:13 + 3 * K] = P[14:14 + 3 * K].T
    return rec


def read_ply(path) -> tuple[np.ndarray, int]:
    """PLYLoader::load: returns ([n, 59] Gaussian3D records, SH degree)."""
    p = str(path).encode()
    n, deg = C.c_int64(), C.c_int()
    L.call("ds_ply_probe", p, C.byref(n), C.byref(deg))
    rec = np.zeros((n.value, G3_RECORD), np.float32)
    L.call("ds_ply_read", p, rec.ctypes.data_as(C.POINTER(C.c_float)), n.value, C.byref(n),
           C.byref(deg))
    return rec, deg.value


def write_ply(path, rec: np.ndarray, sh_num_bands: int = 0) -> None:
    """PLYSaver::save of [n, 59] Gaussian3D records."""
    rec = np.ascontiguousarray(rec, np.float32)
    L.call("ds_ply_write", str(path).encode(), rec.ctypes.data_as(C.POINTER(C.c_float)),
           rec.shape[0], sh_num_bands)


def normalize_scene(rec: np.ndarray, scene_scale: float = 1.0) -> np.ndarray:
    """SplatUtils::normalizeScene on a copy of [n, 59] records."""
    out = np.ascontiguousarray(rec, np.float32).copy()
    L.call("ds_normalize_scene", out.ctypes.data_as(C.POINTER(C.c_float)), out.shape[0],
           scene_scale)
    return out


class Batch:
    """Owns a ds_batch: many independent fitting instances stepped together.

    sizes: [(width, height, splat count)] per instance."""

    def __init__(self, sizes, sh_degree: int = 0, lrs=None, max_isects: int = 0,
                 storage: int = L.DS_STORAGE_BF16, tile_size: int = 16, ppt: int = 1,
                 schedule: int = L.DS_SCHEDULE_LONGEST_FIRST, use_graph: bool = True,
                 grad_mode: int = L.DS_GRAD_REFERENCE, betas=(0.9, 0.999), eps: float = 1e-8):
        cfg = L.BatchConfig()
        L.call("ds_batch_default_config", C.byref(cfg))
        cfg.instances, cfg.sh_degree, cfg.max_isects = len(sizes), sh_degree, max_isects
        if lrs is not None:
            (cfg.lr_pos, cfg.lr_scale, cfg.lr_rot, cfg.lr_sh_dc, cfg.lr_sh_rest,
             cfg.lr_opacity) = lrs
        cfg.beta1, cfg.beta2 = betas
        cfg.epsilon = eps
        cfg.storage, cfg.use_graph, cfg.grad_mode = storage, 1 if use_graph else 0, grad_mode
        cfg.schedule, cfg.tile_size, cfg.pixels_per_thread = schedule, tile_size, ppt
        inst = (L.BatchInstance * len(sizes))()
        for k, (w, h, n) in enumerate(sizes):
            inst[k].width, inst[k].height, inst[k].count = w, h, n
        h = C.c_void_p()
        L.call("ds_batch_create", C.byref(cfg), inst, C.byref(h))
        self.h = h
        self.sizes = [tuple(s) for s in sizes]
        self.sh_degree = sh_degree
        self.bands = sh_bands(sh_degree)
        g = L.Gaussian3D()
        L.call("ds_batch_params", self.h, C.byref(g))
        self.params = _wrap_device(g.pos_x, (14 + 3 * self.bands, g.count))
        self.ranges = []
        for k in range(len(sizes)):
            a, n = C.c_int32(), C.c_int32()
            L.call("ds_batch_instance_range", self.h, k, C.byref(a), C.byref(n))
            self.ranges.append((a.value, n.value))

    def close(self):
        if self.h:
            L.call("ds_batch_destroy", self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def instance_params(self, k: int) -> torch.Tensor:
        a, n = self.ranges[k]
        return self.params[:, a:a + n]

    def set_params(self, k: int, params) -> None:
        a, n = self.ranges[k]
        self.params[:, a:a + n].copy_(torch.as_tensor(params, device="cuda"))
        L.call("ds_batch_params_updated", self.h)

    def set_target(self, k: int, target: torch.Tensor, stream=None) -> None:
        target = target.contiguous()
        L.call("ds_batch_set_target", self.h, k, target.data_ptr(), _stream(stream))
        torch.cuda.current_stream().synchronize()

    def set_camera(self, k: int, pv, cam_pos, stream=None) -> None:
        L.call("ds_batch_set_camera", self.h, k, L.fptr(pv), L.fptr(cam_pos), _stream(stream))

    def step(self, n: int = 1, stream=None) -> None:
        L.call("ds_batch_step", self.h, n, _stream(stream))

    def losses(self, stream=None) -> np.ndarray:
        out = np.zeros(len(self.sizes), np.float32)
        L.call("ds_batch_losses", self.h, out.ctypes.data_as(C.POINTER(C.c_float)),
               _stream(stream))
        return out

    def image(self, k: int) -> torch.Tensor:
        p = C.c_void_p()
        L.call("ds_batch_output", self.h, k, C.byref(p))
        w, h, _ = self.sizes[k]
        return _wrap_device(p.value, (h, w, 3))

    def counters(self) -> dict:
        out = (C.c_uint64 * 3)()
        L.call("ds_batch_counters", self.h, out, 3)
        return {"n_isects": int(out[0]), "visible": int(out[1]), "step": int(out[2])}

    def status(self) -> tuple[int, int]:
        flags = C.c_uint32()
        code = L.lib().ds_batch_status(self.h, C.byref(flags))
        return code, int(flags.value)


# ---- image targets -------------------------------------------------------------

def read_image(path) -> np.ndarray:
    """PNG / PPM / PGM -> [H, W, 3] uint8 (ImageLoader's decode step)."""
    p = str(path).encode()
    w, h = C.c_int(), C.c_int()
    L.call("ds_image_probe", p, C.byref(w), C.byref(h))
    out = np.zeros((h.value, w.value, 3), np.uint8)
    L.call("ds_image_read_rgb8", p, out.ctypes.data, out.size, C.byref(w), C.byref(h))
    return out


def fit_image(rgb8: np.ndarray, width: int, height: int, padding: int = 0, stream=None):
    """Aspect fit + pad of an RGB8 image onto a [height, width, 3] float canvas on
    the GPU (ImageLoader::load's resize and placement).  Returns (canvas, (fit_w, fit_h))."""
    src = torch.as_tensor(np.ascontiguousarray(rgb8, np.uint8), device="cuda")
    out = torch.empty(height, width, 3, dtype=torch.float32, device="cuda")
    fw, fh = C.c_int(), C.c_int()
    L.call("ds_image_fit", src.data_ptr(), rgb8.shape[1], rgb8.shape[0], width, height, padding,
           out.data_ptr(), C.byref(fw), C.byref(fh), _stream(stream))
    torch.cuda.current_stream().synchronize()
    return out, (fw.value, fh.value)


def load_image(path, width: int, height: int, padding: int = 0):
    return fit_image(read_image(path), width, height, padding)


def write_png(path, rgb) -> None:
    """ImageSaver::saveAsPNG of an RGB float image in [0, 1] ([H, W, 3])."""
    a = np.ascontiguousarray(rgb.detach().cpu().numpy() if torch.is_tensor(rgb) else rgb,
                             np.float32)
    L.call("ds_image_write_png", str(path).encode(), a.ctypes.data, a.shape[1], a.shape[0])
