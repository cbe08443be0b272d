"""numpy front end of the FP64 CPU oracle (oracle/oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's cpu_baseline leg as the checker.  Array layouts are those of
oracle.cpp (field-major float64).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "liboracle.so"

_d = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_i32 = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_u32 = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
_u64 = np.ctypeslib.ndpointer(dtype=np.uint64, flags="C_CONTIGUOUS")

_lib = None


def build() -> Path:
    src = HERE / "oracle.cpp"
    if not LIB.exists() or LIB.stat().st_mtime < src.stat().st_mtime:
        subprocess.run(["make", "-C", str(HERE), "all"], check=True, capture_output=True)
    return LIB


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(str(LIB))
        sig = {
            "orc_sh_bands": (C.c_int, [C.c_int]),
            "orc_activ_forward": (None, [C.c_int, C.c_int, _d, _d, _d]),
            "orc_activ_backward": (None, [C.c_int, C.c_int, C.c_int, _d, _d, _d, _d, _d]),
            "orc_project_forward": (None, [C.c_int, _d, _d, _d, _i32]),
            "orc_project_backward": (None, [C.c_int, _d, _d, _d, C.c_int, _d]),
            "orc_tile_assign": (None, [C.c_int, _d, C.c_int, C.c_int, C.c_double, _i32, _u32, _i32]),
            "orc_depth_bits": (C.c_uint32, [C.c_double]),
            "orc_build_lists": (C.c_int64, [C.c_int, _d, C.c_int, C.c_int, _i32, _u32, C.c_int64,
                                            _u64, _u32, _i32]),
            "orc_composite_forward": (None, [C.c_int, _d, C.c_int, C.c_int, _u32, _i32, C.c_double,
                                             C.c_int, _d, _d, _i32, _i32]),
            "orc_composite_backward": (None, [C.c_int, _d, C.c_int, C.c_int, _u32, _i32, _d, _i32,
                                              _d, C.c_int, C.c_int, _d]),
            "orc_mse_forward": (C.c_double, [C.c_int64, _d, _d]),
            "orc_mse_backward": (None, [C.c_int64, _d, _d, _d]),
            "orc_adam": (None, [C.c_int64, _d, _d, _d, _d, C.c_double, C.c_double, C.c_double,
                                C.c_double, C.c_int]),
        }
        for k, (res, args) in sig.items():
            f = getattr(L, k)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def sh_bands(degree: int) -> int:
    return int(lib().orc_sh_bands(degree))


def activ_forward(P, degree, cam):
    P = _f64(P)
    n = P.shape[1]
    S3 = np.zeros((13, n))
    lib().orc_activ_forward(n, degree, P, _f64(cam), S3)
    return S3


def activ_backward(P, degree, cam, S3, G3):
    P = _f64(P)
    n = P.shape[1]
    K = (P.shape[0] - 14) // 3
    GP = np.zeros_like(P)
    lib().orc_activ_backward(n, degree, K, P, _f64(cam), _f64(S3), _f64(G3), GP)
    return GP


def project_forward(S3, pv):
    S3 = _f64(S3)
    n = S3.shape[1]
    S2 = np.zeros((10, n))
    culled = np.zeros(n, np.int32)
    lib().orc_project_forward(n, S3, _f64(pv), S2, culled)
    return S2, culled


def project_backward(S3, pv, G2, exact=False):
    S3 = _f64(S3)
    n = S3.shape[1]
    G3 = np.zeros((13, n))
    lib().orc_project_backward(n, S3, _f64(pv), _f64(G2), 1 if exact else 0, G3)
    return G3


def tile_assign(S2, W, H, tol=1e-5):
    S2 = _f64(S2)
    n = S2.shape[1]
    rect = np.zeros(4 * n, np.int32)
    counts = np.zeros(n, np.uint32)
    amb = np.zeros(n, np.int32)
    lib().orc_tile_assign(n, S2, W, H, tol, rect, counts, amb)
    return rect.reshape(n, 4), counts, amb


def build_lists(S2, W, H, rect, counts, cap=1 << 26):
    S2 = _f64(S2)
    n = S2.shape[1]
    total = int(np.sum(counts, dtype=np.int64))
    keys = np.zeros(max(total, 1), np.uint64)
    ids = np.zeros(max(total, 1), np.uint32)
    tiles = ((W + 15) // 16) * ((H + 15) // 16)
    ranges = np.zeros(2 * tiles, np.int32)
    m = lib().orc_build_lists(n, S2, W, H, np.ascontiguousarray(rect.reshape(-1), np.int32),
                              np.ascontiguousarray(counts, np.uint32), cap, keys, ids, ranges)
    if m < 0:
        raise ValueError("intersection capacity exceeded")
    return keys[:m], ids[:m], ranges


def composite_forward(S2, W, H, ids, ranges, tol=1e-5, threads=None):
    S2 = _f64(S2)
    n = S2.shape[1]
    rgb = np.zeros(H * W * 3)
    alpha = np.zeros(H * W)
    last = np.zeros(H * W, np.int32)
    amb = np.zeros(H * W, np.int32)
    lib().orc_composite_forward(n, S2, W, H, np.ascontiguousarray(ids, np.uint32),
                                np.ascontiguousarray(ranges, np.int32), tol,
                                threads or os.cpu_count() or 1, rgb, alpha, last, amb)
    return rgb.reshape(H, W, 3), alpha.reshape(H, W), last.reshape(H, W), amb.reshape(H, W)


def composite_backward(S2, W, H, ids, ranges, alpha, last_ids, grad_rgb, threads=None, exact=False):
    S2 = _f64(S2)
    n = S2.shape[1]
    G2 = np.zeros((10, n))
    lib().orc_composite_backward(n, S2, W, H, np.ascontiguousarray(ids, np.uint32),
                                 np.ascontiguousarray(ranges, np.int32),
                                 _f64(alpha).reshape(-1),
                                 np.ascontiguousarray(last_ids, np.int32).reshape(-1),
                                 _f64(grad_rgb).reshape(-1), threads or os.cpu_count() or 1,
                                 1 if exact else 0, G2)
    return G2


def mse_forward(px, tgt):
    px, tgt = _f64(px).reshape(-1), _f64(tgt).reshape(-1)
    return float(lib().orc_mse_forward(px.size // 3, px, tgt))


def mse_backward(px, tgt):
    px, tgt = _f64(px).reshape(-1), _f64(tgt).reshape(-1)
    g = np.zeros_like(px)
    lib().orc_mse_backward(px.size // 3, px, tgt, g)
    return g


def adam(p, g, m, v, lr, step, b1=0.9, b2=0.999, eps=1e-8):
    p, m, v = _f64(p).copy(), _f64(m).copy(), _f64(v).copy()
    g = _f64(g)
    lib().orc_adam(p.size, p.reshape(-1), g.reshape(-1), m.reshape(-1), v.reshape(-1), lr, b1, b2,
                   eps, step)
    return p, m, v


def adam_gaussian3d(p, g, m, v, lrs, step, b1=0.9, b2=0.999, eps=1e-8):
    """Adam over a field-major Gaussian3D parameter array [14 + 3K, n] with the
    per-group learning rates lrs = (pos, scale, rot, sh_dc, sh_rest, opacity)
    of registerGaussian3DGroups (src/optimizers/gaussian3d_adam.h:27-55)."""
    p, m, v = _f64(p).copy(), _f64(m).copy(), _f64(v).copy()
    g = _f64(g)
    rows = p.shape[0]
    groups = [(0, 3, lrs[0]), (3, 6, lrs[1]), (6, 10, lrs[2]), (10, 13, lrs[3]),
              (13, 14, lrs[5])] + ([(14, rows, lrs[4])] if rows > 14 else [])
    for a, b, lr in groups:
        pa, ma, va = p[a:b].copy(), m[a:b].copy(), v[a:b].copy()
        ga = np.ascontiguousarray(g[a:b])
        lib().orc_adam(pa.size, pa.reshape(-1), ga.reshape(-1), ma.reshape(-1), va.reshape(-1),
                       float(lr), b1, b2, eps, step)
        p[a:b], m[a:b], v[a:b] = pa, ma, va
    return p, m, v


@dataclass
class Forward:
    S3: np.ndarray
    S2: np.ndarray
    culled: np.ndarray
    rect: np.ndarray
    counts: np.ndarray
    tile_amb: np.ndarray
    keys: np.ndarray
    ids: np.ndarray
    ranges: np.ndarray
    image: np.ndarray
    alpha: np.ndarray
    last_ids: np.ndarray
    px_amb: np.ndarray
    loss: float | None


def forward(P, degree, cam, pv, W, H, target=None, tol=1e-5, threads=None) -> Forward:
    """Full FP64 forward: activation -> projection -> tiles -> sort -> composite -> MSE."""
    S3 = activ_forward(P, degree, cam)
    S2, culled = project_forward(S3, pv)
    rect, counts, tamb = tile_assign(S2, W, H, tol)
    keys, ids, ranges = build_lists(S2, W, H, rect, counts)
    img, alpha, last, pamb = composite_forward(S2, W, H, ids, ranges, tol, threads)
    loss = mse_forward(img, target) if target is not None else None
    return Forward(S3, S2, culled, rect, counts, tamb, keys, ids, ranges, img, alpha, last, pamb,
                   loss)


def backward(P, degree, cam, pv, W, H, fw: Forward, grad_rgb, threads=None, exact=False):
    """Full FP64 backward; returns (dL/dparams, dL/dSplat2D, dL/dSplat3D).
    exact=False follows the reference's recurrence, exact=True the true derivative."""
    G2 = composite_backward(fw.S2, W, H, fw.ids, fw.ranges, fw.alpha, fw.last_ids, grad_rgb,
                            threads, exact)
    G3 = project_backward(fw.S3, pv, G2, exact)
    GP = activ_backward(P, degree, cam, fw.S3, G3)
    return GP, G2, G3


def loss_and_grads(P, degree, cam, pv, W, H, target, threads=None, exact=False):
    fw = forward(P, degree, cam, pv, W, H, target, threads=threads)
    g = mse_backward(fw.image, target).reshape(H, W, 3)
    GP, G2, G3 = backward(P, degree, cam, pv, W, H, fw, g, threads, exact)
    return fw, GP
