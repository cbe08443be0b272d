"""ctypes front end of the reference's own host PLY reader and writer
(oracle/_ref/libdsref_ply.so, built from src/io/ply_io.cpp by oracle/Makefile).

TEST INFRASTRUCTURE ONLY: the CPU PLY tests and tests/golden/make_golden_ply.py.
Splats are [n, 59] float32 rows of the reference's host record Gaussian3D.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB = Path(__file__).resolve().parent / "_ref" / "libdsref_ply.so"
_lib = None


def available() -> bool:
    return LIB.exists()


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        L = C.CDLL(str(LIB))
        L.ref_ply_save.restype = C.c_int
        L.ref_ply_save.argtypes = [C.c_char_p, C.c_void_p, C.c_int64, C.c_int]
        L.ref_ply_load.restype = C.c_int
        L.ref_ply_load.argtypes = [C.c_char_p, C.c_void_p, C.c_int64, C.POINTER(C.c_int64),
                                   C.POINTER(C.c_int)]
        _lib = L
    return _lib


def save(path, splats: np.ndarray, sh_num_bands: int) -> None:
    rec = np.ascontiguousarray(splats, np.float32)
    assert rec.ndim == 2 and rec.shape[1] == 59
    if lib().ref_ply_save(str(path).encode(), rec.ctypes.data, rec.shape[0], sh_num_bands):
        raise RuntimeError(f"PLYSaver::save failed for {path}")


def load(path, capacity: int = 1 << 20):
    out = np.zeros((capacity, 59), np.float32)
    n, deg = C.c_int64(), C.c_int()
    if lib().ref_ply_load(str(path).encode(), out.ctypes.data, capacity, C.byref(n),
                          C.byref(deg)):
        raise RuntimeError(f"PLYLoader::load failed for {path}")
    return out[:n.value].copy(), deg.value
