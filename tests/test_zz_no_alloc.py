"""ds_raster_forward_noalloc: the rasterizer forward for callers that cannot
let the library allocate device memory (their own allocator owns the GPU, or
cudaMalloc's implicit synchronisation would stall a frame loop).  It must
render exactly what ds_raster_forward renders, on consecutive calls that reuse
its built-in scratch array, drop pairs beyond its fixed pair limit exactly as a
rasterizer of that capacity drops them and report the overflow through
ds_raster_noalloc_status, and reject sizes beyond that array's limits.

This file is collected last so that a run stopping at the first failure has
already run every other test."""
import ctypes as C

import numpy as np
import pytest

from diffsplat_b200.scenes import small_problem
from tests.helpers import rel_err

pytestmark = pytest.mark.gpu

IMG_TOL = 1e-5  # the image tolerance of the parity tests


def _splat2d(prob):
    import torch
    from diffsplat_b200 import api
    P = torch.tensor(prob.params, device="cuda")
    S3 = api.activ_forward(P, prob.sh_degree, prob.cam)
    return api.project_forward(S3, prob.pv)


def test_noalloc_forward_matches_raster_forward_twice(cuda_lib):
    import torch
    from diffsplat_b200 import _lib as L
    from diffsplat_b200 import api
    # Two calls in a row with different scenes and image sizes: the second call
    # must not see anything the first one left in the shared array.
    for W, H, n, seed in ((160, 120, 3000, 3), (200, 96, 1200, 4)):
        prob = small_problem(W, H, n, seed=seed, log_scale_mean=-2.8)
        s2 = _splat2d(prob)
        R = api.Rasterizer(W, H, n, 1 << 20)
        ref_img = R.forward(s2)
        img = torch.full((H, W, 3), -1.0, device="cuda")
        L.call("ds_raster_forward_noalloc", C.byref(api.s2_view(s2)), W, H, img.data_ptr(),
               torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        a, b = img.cpu().numpy(), ref_img.cpu().numpy()
        assert R.isect_count() < (1 << 17)
        assert rel_err(a, b) <= IMG_TOL
        assert np.array_equal(a, b)  # same kernels, deterministic
        R.close()


def test_noalloc_overflow_matches_capped_rasterizer_and_is_reported(cuda_lib):
    import torch
    from diffsplat_b200 import _lib as L
    from diffsplat_b200 import api
    W = H = 256
    n = 8000
    cap = 1 << 17  # the no-allocation entry's pair limit
    st = torch.cuda.current_stream().cuda_stream
    flags = C.c_uint32()
    L.lib().ds_raster_noalloc_status(C.byref(flags), st)  # clear what earlier calls left
    prob = small_problem(W, H, n, seed=5, log_scale_mean=-1.8)
    s2 = _splat2d(prob)
    R = api.Rasterizer(W, H, n, cap)
    ref_img = R.forward(s2)
    assert R.isect_count() > cap  # the case really overflows
    code, bits = R.status()
    assert code == L.DS_ERR_ISECT_OVERFLOW and bits & 1
    for _ in range(2):
        img = torch.full((H, W, 3), -1.0, device="cuda")
        L.call("ds_raster_forward_noalloc", C.byref(api.s2_view(s2)), W, H, img.data_ptr(), st)
        code = L.lib().ds_raster_noalloc_status(C.byref(flags), st)
        assert code == L.DS_ERR_ISECT_OVERFLOW and flags.value & 1
        assert np.array_equal(img.cpu().numpy(), ref_img.cpu().numpy())
    R.close()
    # a call within the limit afterwards reports a clean status
    prob = small_problem(96, 64, 300, seed=6)
    s2 = _splat2d(prob)
    img = torch.empty((64, 96, 3), device="cuda")
    L.call("ds_raster_forward_noalloc", C.byref(api.s2_view(s2)), 96, 64, img.data_ptr(), st)
    assert L.lib().ds_raster_noalloc_status(C.byref(flags), st) == L.DS_OK and flags.value == 0


def test_noalloc_rejects_sizes_beyond_its_limits(cuda_lib):
    import torch
    from diffsplat_b200 import _lib as L
    from diffsplat_b200 import api
    s2 = torch.zeros((10, 8193), device="cuda")
    img = torch.empty((16, 16, 3), device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    assert L.lib().ds_raster_forward_noalloc(C.byref(api.s2_view(s2)), 16, 16, img.data_ptr(),
                                             st) == L.DS_ERR_ARG
    s2 = torch.zeros((10, 16), device="cuda")
    big = torch.empty((257, 256, 3), device="cuda")
    assert L.lib().ds_raster_forward_noalloc(C.byref(api.s2_view(s2)), 256, 257, big.data_ptr(),
                                             st) == L.DS_ERR_ARG
