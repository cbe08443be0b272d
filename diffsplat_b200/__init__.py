"""diffsplat_b200: B200 (sm_100a) differentiable Gaussian-splatting training path.

The compute lives in libdiffsplat_b200.so (C ABI: include/diffsplat_b200.h).
`diffsplat_b200.api` wraps it for CUDA torch tensors; the C++ drop-in headers
for the reference's Layer / Pipeline / Adam API are in include/compat/.
"""
from . import _lib  # noqa: F401

__all__ = ["_lib"]
