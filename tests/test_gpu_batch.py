"""GPU tests of batched fitting (ds_batch_*): with FP32 storage and 16-pixel
tiles every instance of a batch follows exactly the trajectory of its own
single-instance fitter (bit-identical parameters); BF16 batches are
deterministic (graph = eager) and fit as well as the FP32 sequential fitters;
8- and 32-pixel tiles train."""
import numpy as np
import pytest

from diffsplat_b200.scenes import psnr_from_ref_loss, small_problem

pytestmark = pytest.mark.gpu

SIZES = [(96, 64, 400), (128, 128, 900), (64, 48, 200), (160, 96, 1200)]


def _problems(sh_degree=0):
    return [small_problem(w, h, n, seed=70 + k, sh_degree=sh_degree)
            for k, (w, h, n) in enumerate(SIZES)]


def _batch(probs, **kw):
    import torch
    from diffsplat_b200 import api
    b = api.Batch([(p.width, p.height, p.params.shape[1]) for p in probs],
                  sh_degree=probs[0].sh_degree, lrs=probs[0].lrs, max_isects=1 << 22, **kw)
    for k, p in enumerate(probs):
        b.set_params(k, p.params)
        b.set_target(k, torch.tensor(p.target, device="cuda"))
        b.set_camera(k, p.pv, p.cam)
    return b


def _single(p, steps, **kw):
    import torch
    from diffsplat_b200 import api
    f = api.Fitter(p.width, p.height, p.params.shape[1], p.sh_degree, lrs=p.lrs,
                   max_isects=1 << 22, **kw)
    f.set_params(p.params)
    f.set_target(torch.tensor(p.target, device="cuda"))
    f.set_camera(p.pv, p.cam)
    f.step(steps)
    out = f.params.cpu().numpy().copy(), f.loss()
    f.close()
    return out


@pytest.mark.parametrize("deg", [0, 2])
def test_fp32_batch_equals_single_fitters(cuda_lib, deg):
    from diffsplat_b200 import _lib as L
    probs = _problems(deg)
    b = _batch(probs, storage=L.DS_STORAGE_FP32, tile_size=16, ppt=1)
    b.step(3)
    losses = b.losses()
    for k, p in enumerate(probs):
        mine = b.instance_params(k).cpu().numpy()
        ref, ref_loss = _single(p, 3, schedule=L.DS_SCHEDULE_LONGEST_FIRST)
        assert np.array_equal(mine.view(np.uint32), ref.view(np.uint32)), f"instance {k}"
        assert abs(losses[k] - ref_loss) <= 1e-6 * ref_loss
    b.close()


def test_bf16_batch_graph_equals_eager(cuda_lib):
    probs = _problems(1)
    a = _batch(probs, use_graph=True)
    e = _batch(probs, use_graph=False)
    a.step(4)
    e.step(4)
    assert np.array_equal(a.params.cpu().numpy().view(np.uint32),
                          e.params.cpu().numpy().view(np.uint32))
    assert np.array_equal(a.losses(), e.losses())
    a.close()
    e.close()


@pytest.mark.parametrize("tile,ppt", [(8, 1), (8, 2), (16, 2), (32, 1), (32, 2)])
def test_tile_sizes_train(cuda_lib, tile, ppt):
    probs = _problems(0)
    b = _batch(probs, tile_size=tile, ppt=ppt)
    b.step(1)
    l0 = b.losses()
    b.step(150)
    l1 = b.losses()
    code, flags = b.status()
    assert code == 0 and flags == 0
    assert np.isfinite(l1).all() and (l1 < 0.6 * l0).all(), (l0, l1)
    b.close()


def test_bf16_batch_psnr_tracks_fp32_sequential(cuda_lib):
    """Per-instance PSNR after 300 steps: BF16 batch vs each instance fitted
    alone by the FP32 fitter."""
    probs = _problems(0)
    b = _batch(probs)
    b.step(300)
    got = [psnr_from_ref_loss(x) for x in b.losses()]
    b.close()
    ref = [psnr_from_ref_loss(_single(p, 300)[1]) for p in probs]
    print("PSNR bf16 batch", np.round(got, 2), "fp32 sequential", np.round(ref, 2))
    assert min(g - r for g, r in zip(got, ref)) > -0.5
