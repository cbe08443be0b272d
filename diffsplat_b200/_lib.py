"""ctypes binding of libdiffsplat_b200.so (the C ABI in include/diffsplat_b200.h).

The library is loaded from diffsplat_b200/lib/.  There is no fallback: when the
shared library is missing or no sm_100 device is present, the call raises.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "lib" / "libdiffsplat_b200.so"

DS_OK = 0
DS_ERR_ARG = 1
DS_ERR_OOM = 2
DS_ERR_CUDA = 3
DS_ERR_ISECT_OVERFLOW = 4
DS_ERR_STATE = 5
DS_ERR_NO_DEVICE = 6
DS_ERR_INTERNAL = 7

DS_GRAD_REFERENCE = 0
DS_GRAD_EXACT = 1

DS_STORAGE_FP32 = 0
DS_STORAGE_BF16 = 1
DS_SCHEDULE_LONGEST_FIRST = 0
DS_SCHEDULE_RASTER = 1

DS_RASTER_KEYS = 0
DS_RASTER_IDS = 1
DS_RASTER_RANGES = 2
DS_RASTER_LAST_IDS = 3
DS_RASTER_ALPHAS = 4
DS_RASTER_COUNTS = 5
DS_RASTER_CONICS = 6

_fp = C.POINTER(C.c_float)
_vp = C.c_void_p


class Gaussian3D(C.Structure):
    _fields_ = [(n, _vp) for n in (
        "pos_x", "pos_y", "pos_z", "scale_x", "scale_y", "scale_z",
        "rot_w", "rot_x", "rot_y", "rot_z", "sh_dc_r", "sh_dc_g", "sh_dc_b",
        "sh_rest_r", "sh_rest_g", "sh_rest_b", "logit_opacity")] + [
        ("count", C.c_int32), ("sh_num_bands", C.c_int32)]


class Splat3D(C.Structure):
    _fields_ = [(n, _vp) for n in (
        "pos_x", "pos_y", "pos_z", "cov_xx", "cov_xy", "cov_xz", "cov_yy", "cov_yz", "cov_zz",
        "color_r", "color_g", "color_b", "opacity")] + [("count", C.c_int32)]


class Splat2D(C.Structure):
    _fields_ = [(n, _vp) for n in (
        "pos_x", "pos_y", "pos_z", "cov_xx", "cov_xy", "cov_yy",
        "color_r", "color_g", "color_b", "opacity")] + [("count", C.c_int32)]


class AdamGroup(C.Structure):
    _fields_ = [("param", _vp), ("grad", _vp), ("m", _vp), ("v", _vp),
                ("n", C.c_int64), ("lr", C.c_float)]


class FitterConfig(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("count", C.c_int32),
                ("sh_degree", C.c_int32), ("max_isects", C.c_int64),
                ("lr_pos", C.c_float), ("lr_scale", C.c_float), ("lr_rot", C.c_float),
                ("lr_sh_dc", C.c_float), ("lr_sh_rest", C.c_float), ("lr_opacity", C.c_float),
                ("beta1", C.c_float), ("beta2", C.c_float), ("epsilon", C.c_float),
                ("storage", C.c_int32), ("use_graph", C.c_int32), ("grad_mode", C.c_int32),
                ("schedule", C.c_int32), ("capacity", C.c_int32)]


GAUSSIAN3D_FIELDS = ("pos_x", "pos_y", "pos_z", "scale_x", "scale_y", "scale_z",
                     "rot_w", "rot_x", "rot_y", "rot_z", "sh_dc_r", "sh_dc_g", "sh_dc_b",
                     "logit_opacity")
SPLAT3D_FIELDS = tuple(n for n, _ in Splat3D._fields_[:-1])
SPLAT2D_FIELDS = tuple(n for n, _ in Splat2D._fields_[:-1])

class DensifyParams(C.Structure):
    _fields_ = [("grad_threshold", C.c_float), ("scale_threshold", C.c_float),
                ("min_opacity", C.c_float), ("seed", C.c_uint32)]


class BatchInstance(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("count", C.c_int32),
                ("reserved", C.c_int32)]


class BatchConfig(C.Structure):
    _fields_ = [("instances", C.c_int32), ("sh_degree", C.c_int32), ("max_isects", C.c_int64)] + [
        (n, C.c_float) for n in ("lr_pos", "lr_scale", "lr_rot", "lr_sh_dc", "lr_sh_rest",
                                 "lr_opacity", "beta1", "beta2", "epsilon")] + [
        (n, C.c_int32) for n in ("storage", "use_graph", "grad_mode", "schedule", "tile_size",
                                 "pixels_per_thread")]


_SIGS = {
    "ds_abi_version": (C.c_int, []),
    "ds_status_string": (C.c_char_p, [C.c_int]),
    "ds_device_check": (C.c_int, []),
    "ds_debug_fail_allocations_after": (C.c_int, [C.c_int64]),
    "ds_activ_forward": (C.c_int, [C.POINTER(Gaussian3D), C.c_int, _fp, C.POINTER(Splat3D), _vp]),
    "ds_activ_backward": (C.c_int, [C.POINTER(Gaussian3D), C.POINTER(Splat3D), C.POINTER(Splat3D),
                                    C.c_int, _fp, C.POINTER(Gaussian3D), _vp]),
    "ds_project_forward": (C.c_int, [C.POINTER(Splat3D), _fp, C.POINTER(Splat2D), _vp]),
    "ds_project_backward": (C.c_int, [C.POINTER(Splat3D), _fp, C.POINTER(Splat2D),
                                      C.POINTER(Splat3D), _vp]),
    "ds_project_backward_ex": (C.c_int, [C.POINTER(Splat3D), _fp, C.POINTER(Splat2D),
                                         C.POINTER(Splat3D), C.c_int, _vp]),
    "ds_raster_create": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int64, C.POINTER(_vp)]),
    "ds_raster_resize": (C.c_int, [_vp, C.c_int, C.c_int]),
    "ds_raster_set_grad_mode": (C.c_int, [_vp, C.c_int]),
    "ds_raster_forward": (C.c_int, [_vp, C.POINTER(Splat2D), _vp, _vp]),
    "ds_raster_backward": (C.c_int, [_vp, C.POINTER(Splat2D), _vp, C.POINTER(Splat2D), _vp]),
    "ds_raster_visible_count": (C.c_int, [_vp, C.POINTER(C.c_uint32)]),
    "ds_raster_isect_count": (C.c_int, [_vp, C.POINTER(C.c_uint32)]),
    "ds_raster_status": (C.c_int, [_vp, C.POINTER(C.c_uint32)]),
    "ds_raster_download": (C.c_int, [_vp, C.c_int, _vp, C.c_int64]),
    "ds_raster_destroy": (C.c_int, [_vp]),
    "ds_raster_forward_noalloc": (C.c_int, [C.POINTER(Splat2D), C.c_int, C.c_int, _vp, _vp]),
    "ds_raster_noalloc_status": (C.c_int, [C.POINTER(C.c_uint32), _vp]),
    "ds_mse_forward": (C.c_int, [_vp, _vp, C.c_int64, _vp, _vp]),
    "ds_mse_backward": (C.c_int, [_vp, _vp, C.c_int64, _vp, _vp]),
    "ds_adam_step": (C.c_int, [C.POINTER(AdamGroup), C.c_int, C.c_float, C.c_float, C.c_float,
                               C.c_int, _vp]),
    "ds_fitter_default_config": (C.c_int, [C.POINTER(FitterConfig)]),
    "ds_fitter_create": (C.c_int, [C.POINTER(FitterConfig), C.POINTER(_vp)]),
    "ds_fitter_create_with_grads": (C.c_int, [C.POINTER(FitterConfig), C.POINTER(_vp)]),
    "ds_fitter_params": (C.c_int, [_vp, C.POINTER(Gaussian3D)]),
    "ds_fitter_grads": (C.c_int, [_vp, C.POINTER(Gaussian3D)]),
    "ds_fitter_moments": (C.c_int, [_vp, C.POINTER(Gaussian3D), C.POINTER(Gaussian3D)]),
    "ds_fitter_set_target": (C.c_int, [_vp, _vp, _vp]),
    "ds_fitter_set_camera": (C.c_int, [_vp, _fp, _fp, _vp]),
    "ds_fitter_step": (C.c_int, [_vp, C.c_int, _vp]),
    "ds_fitter_loss": (C.c_int, [_vp, C.POINTER(C.c_float), _vp]),
    "ds_fitter_output": (C.c_int, [_vp, C.POINTER(_vp)]),
    "ds_fitter_loss_device": (C.c_int, [_vp, C.POINTER(_vp)]),
    "ds_fitter_step_count": (C.c_int, [_vp, C.POINTER(C.c_int)]),
    "ds_fitter_status": (C.c_int, [_vp, C.POINTER(C.c_uint32)]),
    "ds_fitter_destroy": (C.c_int, [_vp]),
    "ds_fitter_profile_step": (C.c_int, [_vp, _fp, C.c_int, _vp]),
    "ds_fitter_counters": (C.c_int, [_vp, C.POINTER(C.c_uint64), C.c_int]),
    "ds_fitter_pair_stats": (C.c_int, [_vp, C.POINTER(C.c_uint64), C.c_int, _vp]),
    "ds_fitter_params_updated": (C.c_int, [_vp]),
    "ds_fitter_download": (C.c_int, [_vp, C.c_int, _vp, C.c_int64]),
    "ds_fitter_densify": (C.c_int, [_vp, C.POINTER(DensifyParams), C.POINTER(C.c_int32), _vp]),
    "ds_fitter_density_stats": (C.c_int, [_vp, C.POINTER(_vp), C.POINTER(_vp)]),
    "ds_batch_default_config": (C.c_int, [C.POINTER(BatchConfig)]),
    "ds_batch_create": (C.c_int, [C.POINTER(BatchConfig), C.POINTER(BatchInstance),
                                  C.POINTER(_vp)]),
    "ds_batch_params": (C.c_int, [_vp, C.POINTER(Gaussian3D)]),
    "ds_batch_instance_range": (C.c_int, [_vp, C.c_int, C.POINTER(C.c_int32),
                                          C.POINTER(C.c_int32)]),
    "ds_batch_params_updated": (C.c_int, [_vp]),
    "ds_batch_set_target": (C.c_int, [_vp, C.c_int, _vp, _vp]),
    "ds_batch_set_camera": (C.c_int, [_vp, C.c_int, _fp, _fp, _vp]),
    "ds_batch_step": (C.c_int, [_vp, C.c_int, _vp]),
    "ds_batch_losses": (C.c_int, [_vp, _fp, _vp]),
    "ds_batch_output": (C.c_int, [_vp, C.c_int, C.POINTER(_vp)]),
    "ds_batch_counters": (C.c_int, [_vp, C.POINTER(C.c_uint64), C.c_int]),
    "ds_batch_status": (C.c_int, [_vp, C.POINTER(C.c_uint32)]),
    "ds_batch_destroy": (C.c_int, [_vp]),
    "ds_gemm_bf16_tn": (C.c_int, [_vp, C.c_int, _vp, C.c_int, C.c_int, C.c_int, C.c_int,
                                  C.c_int, _vp, C.c_int, _vp, _vp, C.c_int, _vp, C.c_int, _vp,
                                  _vp, _vp]),
    "ds_gemm_set_spin_limit": (C.c_int, [C.c_uint32]),
    "ds_im2col_bf16": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _vp,
                                 _vp]),
    "ds_col2im_bf16": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _vp,
                                 _vp, _vp]),
    "ds_transpose_bf16": (C.c_int, [_vp, C.c_int, C.c_int, _vp, _vp]),
    "ds_colsum_bf16": (C.c_int, [_vp, C.c_int64, C.c_int, _vp, C.c_int, _vp, _vp]),
    "ds_adamw": (C.c_int, [_vp, _vp, _vp, _vp, C.c_int64, C.c_float, C.c_float, C.c_float,
                           C.c_float, C.c_float, C.c_int, _vp, _vp]),
    "ds_cast_bf16": (C.c_int, [_vp, C.c_int64, _vp, _vp]),
    "ds_head_decode": (C.c_int, [_vp, C.c_int, C.c_int, _vp, _fp, C.c_float, _vp, _vp]),
    "ds_head_encode_grad": (C.c_int, [_vp, _vp, _vp, C.c_float, C.c_float, C.c_int, C.c_int, _fp,
                                      _vp, _vp]),
    "ds_image_probe": (C.c_int, [C.c_char_p, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "ds_image_read_rgb8": (C.c_int, [C.c_char_p, _vp, C.c_int64, C.POINTER(C.c_int),
                                     C.POINTER(C.c_int)]),
    "ds_image_fit": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _vp,
                               C.POINTER(C.c_int), C.POINTER(C.c_int), _vp]),
    "ds_image_write_png": (C.c_int, [C.c_char_p, _vp, C.c_int, C.c_int]),
    "ds_renderer_create": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int64, C.c_int,
                                     C.POINTER(_vp)]),
    "ds_renderer_set_params": (C.c_int, [_vp, C.POINTER(Gaussian3D), _vp]),
    "ds_renderer_set_sh_degree": (C.c_int, [_vp, C.c_int]),
    "ds_renderer_render": (C.c_int, [_vp, _fp, _fp, _vp]),
    "ds_renderer_output": (C.c_int, [_vp, C.POINTER(_vp)]),
    "ds_renderer_resize": (C.c_int, [_vp, C.c_int, C.c_int]),
    "ds_renderer_counts": (C.c_int, [_vp, C.POINTER(C.c_uint64), C.c_int]),
    "ds_renderer_status": (C.c_int, [_vp, C.POINTER(C.c_uint32)]),
    "ds_renderer_destroy": (C.c_int, [_vp]),
    "ds_ply_probe": (C.c_int, [C.c_char_p, C.POINTER(C.c_int64), C.POINTER(C.c_int)]),
    "ds_ply_read": (C.c_int, [C.c_char_p, _fp, C.c_int64, C.POINTER(C.c_int64),
                              C.POINTER(C.c_int)]),
    "ds_ply_write": (C.c_int, [C.c_char_p, _fp, C.c_int64, C.c_int]),
    "ds_normalize_scene": (C.c_int, [_fp, C.c_int64, C.c_float]),
}

_lib = None


class DSError(RuntimeError):
    def __init__(self, fn: str, code: int):
        msg = lib().ds_status_string(code).decode() if _lib is not None else str(code)
        super().__init__(f"{fn} failed: {msg} ({code})")
        self.code = code


def lib() -> C.CDLL:
    """Loads the shared library (raises when it is absent)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(
                f"{LIB_PATH} is missing; build it with `python -m diffsplat_b200.build`")
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(fn: str, code: int) -> None:
    if code != DS_OK:
        raise DSError(fn, code)


def call(fn: str, *args) -> None:
    check(fn, getattr(lib(), fn)(*args))


def fptr(values):
    """float * of `values` for one call: a C-contiguous float32 NumPy array is
    passed in place (the pointer keeps it alive), anything else is copied."""
    if type(values).__module__ == "numpy" and values.dtype.char == "f" \
            and values.flags.c_contiguous:
        return values.ctypes.data_as(_fp)
    return (C.c_float * len(values))(*[float(v) for v in values])
