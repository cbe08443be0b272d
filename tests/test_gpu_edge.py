"""Edge cases of the CUDA path: empty and fully culled inputs, ragged image
sizes, screen-filling splats, argument errors."""
import numpy as np
import pytest

from diffsplat_b200.scenes import small_problem
from tests.helpers import ds_layers, ref_layers, rel_err

pytestmark = pytest.mark.gpu


def test_zero_splats(cuda_lib):
    import torch
    from diffsplat_b200 import api
    R = api.Rasterizer(48, 33, 16, 1 << 12)
    s2 = torch.zeros((10, 0), device="cuda")
    img = R.forward(s2)
    torch.cuda.synchronize()
    assert img.abs().max().item() == 0.0
    assert R.isect_count() == 0 and R.visible_count() == 0
    g = R.backward(s2, torch.ones_like(img))
    assert g.shape == (10, 0)
    R.close()


def test_all_splats_behind_camera(cuda_lib):
    prob = small_problem(64, 48, 200, seed=3)
    prob.params[2] = -np.abs(prob.params[2])  # z < 0: clip_w <= 0 for every splat
    me = ds_layers(prob)
    assert me["n_isects"] == 0 and me["visible"] == 0
    assert np.abs(me["image"]).max() == 0.0
    assert np.abs(me["GP"]).max() == 0.0
    assert (me["S2"][2] == np.float32(3.4028234663852886e38)).all()


def test_screen_filling_splats_match_reference(cuda_lib):
    from oracle import ref
    if not ref.available():
        pytest.skip("reference build absent")
    prob = small_problem(80, 56, 60, seed=6, log_scale_mean=0.5)
    me, rf = ds_layers(prob), ref_layers(prob)
    assert me["n_isects"] == rf["n_isects"]
    assert np.array_equal(me["keys"], rf["keys"]) and np.array_equal(me["ids"], rf["ids"])
    assert rel_err(me["image"], rf["image"]) <= 1e-5


def test_bad_arguments_are_rejected(cuda_lib):
    import ctypes as C
    from diffsplat_b200 import _lib as L
    h = C.c_void_p()
    assert L.lib().ds_raster_create(0, 10, 10, 0, C.byref(h)) == L.DS_ERR_ARG
    assert L.lib().ds_raster_create(10, 10, -1, 0, C.byref(h)) == L.DS_ERR_ARG
    g = L.Gaussian3D()
    s = L.Splat3D()
    g.count = 4
    s.count = 4
    cam = L.fptr([0, 0, 0])
    assert L.lib().ds_activ_forward(C.byref(g), 0, cam, C.byref(s), None) == L.DS_ERR_ARG
    assert L.lib().ds_activ_forward(C.byref(g), 5, cam, C.byref(s), None) == L.DS_ERR_ARG
    cfg = L.FitterConfig()
    L.lib().ds_fitter_default_config(C.byref(cfg))
    assert L.lib().ds_fitter_create(C.byref(cfg), C.byref(h)) == L.DS_ERR_ARG  # zero sizes


# ---- failure injection on the host ------------------------------------------------
def _sweep_allocations(create, use):
    """Runs create() with the device allocations failing after k successes,
    k = 0, 1, ...: every attempt must fail with DS_ERR_OOM and no handle
    until one succeeds; then the hook is off and a fresh object works."""
    import ctypes as C
    from diffsplat_b200 import _lib as L
    k = 0
    try:
        while True:
            assert k < 400
            L.lib().ds_debug_fail_allocations_after(k)
            h = C.c_void_p(1)
            st = create(h)
            if st == L.DS_OK:
                break
            assert st == L.DS_ERR_OOM and h.value is None, (k, st)
            k += 1
    finally:
        L.lib().ds_debug_fail_allocations_after(-1)
    assert k > 3  # the call allocates several buffers; each failure point was taken
    return h, k


def test_fitter_create_fails_cleanly_at_every_allocation(cuda_lib):
    import ctypes as C
    import torch
    from diffsplat_b200 import _lib as L
    from diffsplat_b200 import api
    prob = small_problem(64, 48, 300, seed=2)
    cfg = L.FitterConfig()
    L.lib().ds_fitter_default_config(C.byref(cfg))
    cfg.width, cfg.height, cfg.count = prob.width, prob.height, 300
    cfg.max_isects = 1 << 16
    h, k = _sweep_allocations(lambda h: L.lib().ds_fitter_create(C.byref(cfg), C.byref(h)), None)
    assert L.lib().ds_fitter_destroy(h) == L.DS_OK
    f = api.Fitter(prob.width, prob.height, 300, 0, lrs=prob.lrs, max_isects=1 << 16)
    f.set_params(prob.params)
    f.set_target(torch.tensor(prob.target, device="cuda"))
    f.set_camera(prob.pv, prob.cam)
    f.step(3)
    assert np.isfinite(f.loss())
    assert f.status() == (0, 0)
    f.close()


def test_raster_renderer_batch_create_fail_cleanly_at_every_allocation(cuda_lib):
    import ctypes as C
    from diffsplat_b200 import _lib as L
    h, _ = _sweep_allocations(lambda h: L.lib().ds_raster_create(96, 64, 500, 1 << 15,
                                                                 C.byref(h)), None)
    assert L.lib().ds_raster_destroy(h) == L.DS_OK
    h, _ = _sweep_allocations(lambda h: L.lib().ds_renderer_create(
        96, 64, 500, 1, 1 << 15, L.DS_STORAGE_BF16, C.byref(h)), None)
    assert L.lib().ds_renderer_destroy(h) == L.DS_OK
    cfg = L.BatchConfig()
    L.lib().ds_batch_default_config(C.byref(cfg))
    cfg.instances = 2
    cfg.max_isects = 1 << 15
    inst = (L.BatchInstance * 2)(L.BatchInstance(32, 32, 50, 0), L.BatchInstance(48, 16, 70, 0))
    h, _ = _sweep_allocations(lambda h: L.lib().ds_batch_create(C.byref(cfg), inst, C.byref(h)),
                              None)
    assert L.lib().ds_batch_destroy(h) == L.DS_OK


def test_nan_parameters_behave_like_the_reference(cuda_lib):
    """NaN in a splat's position, log-scale, opacity logit or colour: culled
    or composited exactly as the reference does (a NaN position or scale fails
    its on-screen / determinant tests; a NaN opacity still composites at the
    0.99 alpha clamp, src/layers/tile_rasterize_layer.cu:277-297).  Same
    lists, same image with the same NaN pixels, and the step reports no
    error."""
    from oracle import ref
    if not ref.available():
        pytest.skip("reference build absent")
    prob = small_problem(96, 64, 300, seed=12)
    nan = np.float32("nan")
    prob.params[0, 3] = nan    # position x
    prob.params[4, 5] = nan    # log-scale y
    prob.params[13, 9] = nan   # opacity logit
    prob.params[11, 11] = nan  # SH DC green
    me, rf = ds_layers(prob), ref_layers(prob)
    assert me["n_isects"] == rf["n_isects"] > 0
    assert me["visible"] == rf["visible"]
    assert np.array_equal(me["keys"], rf["keys"]) and np.array_equal(me["ids"], rf["ids"])
    assert np.array_equal(me["ranges"], rf["ranges"])
    a, b = me["image"], rf["image"]
    assert np.array_equal(np.isnan(a), np.isnan(b))
    fin = np.isfinite(b)
    assert rel_err(a[fin], b[fin]) <= 1e-5
