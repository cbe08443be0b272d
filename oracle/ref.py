"""ctypes front end of the reference harness (oracle/_ref/libdsref.so: the
reference's own CUDA layers built for sm_100a by oracle/Makefile).

TEST INFRASTRUCTURE ONLY: used by the GPU parity tests, the golden-fixture
script and bench.py's reference arm.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_ref" / "libdsref.so"
_lib = None


def available() -> bool:
    return LIB.exists()


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB.exists():
            raise RuntimeError(f"{LIB} is missing (built by `make -C oracle ref` where the "
                               "reference sources are present)")
        L = C.CDLL(str(LIB))
        fp = C.POINTER(C.c_float)
        L.ref_create.restype = C.c_void_p
        L.ref_create.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, fp, fp, fp, fp, fp]
        for name in ("ref_destroy", "ref_zero_grad", "ref_forward", "ref_backward",
                     "ref_adam_step", "ref_step"):
            getattr(L, name).restype = None
            getattr(L, name).argtypes = [C.c_void_p]
        L.ref_set_params.restype = None
        L.ref_set_params.argtypes = [C.c_void_p, fp]
        L.ref_loss.restype = C.c_float
        L.ref_loss.argtypes = [C.c_void_p]
        L.ref_sync.restype = C.c_int
        L.ref_sync.argtypes = []
        L.ref_n_isects.restype = C.c_uint32
        L.ref_n_isects.argtypes = [C.c_void_p]
        L.ref_visible.restype = C.c_uint32
        L.ref_visible.argtypes = [C.c_void_p]
        L.ref_download.restype = C.c_int
        L.ref_download.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
        _lib = L
    return _lib


def _fp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_float))


class RefScene:
    """The reference's layers wired like ImageFitter (activ -> proj -> raster -> mse, Adam)."""

    def __init__(self, W, H, params, degree, target, pv, cam, lrs):
        self.W, self.H, self.degree = W, H, degree
        self.params = np.ascontiguousarray(params, np.float32)
        self.n = self.params.shape[1]
        self.bands = (self.params.shape[0] - 14) // 3
        self._keep = [np.ascontiguousarray(target, np.float32).reshape(-1),
                      np.ascontiguousarray(pv, np.float32), np.ascontiguousarray(cam, np.float32),
                      np.ascontiguousarray(lrs, np.float32)]
        self.h = lib().ref_create(W, H, self.n, degree, _fp(self.params), *[_fp(a) for a in self._keep])
        self.tiles = ((W + 15) // 16) * ((H + 15) // 16)

    def close(self):
        if self.h:
            lib().ref_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_params(self, params):
        p = np.ascontiguousarray(params, np.float32)
        lib().ref_set_params(self.h, _fp(p))

    def zero_grad(self):
        lib().ref_zero_grad(self.h)

    def forward(self):
        lib().ref_forward(self.h)

    def backward(self):
        lib().ref_backward(self.h)

    def adam_step(self):
        lib().ref_adam_step(self.h)

    def step(self):
        lib().ref_step(self.h)

    def loss(self) -> float:
        return float(lib().ref_loss(self.h))

    def n_isects(self) -> int:
        return int(lib().ref_n_isects(self.h))

    def visible(self) -> int:
        return int(lib().ref_visible(self.h))

    def download(self, what: int) -> np.ndarray:
        m = self.n_isects()
        px = self.W * self.H
        rows = 14 + 3 * self.bands
        spec = {0: (np.uint64, m), 1: (np.uint32, m), 2: (np.int32, 2 * self.tiles),
                3: (np.float32, px * 3), 4: (np.float32, px), 5: (np.int32, px),
                6: (np.float32, rows * self.n), 7: (np.float32, rows * self.n),
                8: (np.float32, 10 * self.n), 9: (np.float32, 10 * self.n),
                10: (np.float32, 13 * self.n), 11: (np.float32, 13 * self.n)}[what]
        arr = np.zeros(max(spec[1], 1), spec[0])
        if lib().ref_download(self.h, what, arr.ctypes.data) != 0:
            raise RuntimeError("ref_download failed")
        arr = arr[:spec[1]]
        if what in (6, 7):
            return arr.reshape(rows, self.n)
        if what in (8, 9):
            return arr.reshape(10, self.n)
        if what in (10, 11):
            return arr.reshape(13, self.n)
        if what == 3:
            return arr.reshape(self.H, self.W, 3)
        if what in (4, 5):
            return arr.reshape(self.H, self.W)
        return arr


def canonical_order(keys: np.ndarray, ids: np.ndarray):
    """Sorts ids ascending within runs of equal keys (the reference's slot order
    inside equal keys depends on atomicAdd timing)."""
    order = np.lexsort((ids, keys))
    return keys[order], ids[order]
