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
