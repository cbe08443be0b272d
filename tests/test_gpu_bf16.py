"""BF16 storage mode of the fused fitter (DS_STORAGE_BF16): scale, rotation, SH
and opacity rendered from a BF16 copy of FP32 masters, BF16 Adam moments with
stochastic rounding.  Each result's error against the FP64 oracle is measured
and bounded here."""
import numpy as np
import pytest

from diffsplat_b200.scenes import small_problem
from tests.helpers import rel_err, render_params

pytestmark = pytest.mark.gpu


def _fitter(prob, storage, **kw):
    import torch
    from diffsplat_b200 import api
    f = api.Fitter(prob.width, prob.height, prob.params.shape[1], prob.sh_degree, lrs=prob.lrs,
                   max_isects=1 << 20, storage=storage, **kw)
    f.set_params(prob.params)
    f.set_target(torch.tensor(prob.target, device="cuda"))
    f.set_camera(prob.pv, prob.cam)
    return f


@pytest.mark.parametrize("deg", [0, 3])
def test_bf16_step_is_exact_on_what_it_renders(cuda_lib, deg):
    """Loss and gradients equal the FP64 oracle's evaluated at the BF16-rounded
    attributes, to FP32 accuracy: BF16 storage changes the inputs, not the math."""
    from diffsplat_b200 import _lib as L
    from oracle import oracle as O
    prob = small_problem(96, 64, 300, seed=31 + deg, sh_degree=deg)
    f = _fitter(prob, L.DS_STORAGE_BF16, keep_grads=True)
    f.step(1)
    loss = f.loss()
    G = f.grads().cpu().numpy()
    f.close()
    R = render_params(prob.params).astype(np.float64)
    fw, GP = O.loss_and_grads(R, deg, prob.cam, prob.pv, prob.width, prob.height, prob.target)
    assert abs(loss - fw.loss) <= 1e-5 * fw.loss
    for row in range(G.shape[0]):
        assert rel_err(G[row], GP[row], floor=1e-9) <= 1e-4, f"row {row}"


def test_bf16_error_against_fp64_oracle_on_masters(cuda_lib):
    """Per-result error of one BF16 step against the FP64 oracle at the FP32
    masters (the quantisation error of the mode), with the FP32 mode beside it."""
    from diffsplat_b200 import _lib as L
    from oracle import oracle as O
    prob = small_problem(128, 96, 600, seed=35, sh_degree=1)
    P64 = prob.params.astype(np.float64)
    fw, GP = O.loss_and_grads(P64, 1, prob.cam, prob.pv, prob.width, prob.height, prob.target)
    out = {}
    for name, storage in (("fp32", L.DS_STORAGE_FP32), ("bf16", L.DS_STORAGE_BF16)):
        f = _fitter(prob, storage, keep_grads=True)
        f.step(1)
        out[name] = dict(loss=abs(f.loss() - fw.loss) / fw.loss,
                         image=float(np.abs(f.image().cpu().numpy() - fw.image).max()),
                         grad=rel_err(f.grads().cpu().numpy(), GP))
        f.close()
    print("error vs FP64 oracle at the masters:", out)
    assert out["fp32"]["loss"] < 1e-5 and out["fp32"]["grad"] < 1e-4
    assert out["bf16"]["loss"] < 2e-2
    assert out["bf16"]["image"] < 0.1
    assert out["bf16"]["grad"] < 0.5


def test_bf16_graph_and_eager_bit_identical(cuda_lib):
    """Stochastic rounding draws from (element, field, step): deterministic."""
    from diffsplat_b200 import _lib as L
    prob = small_problem(112, 80, 400, seed=5, sh_degree=2)
    a = _fitter(prob, L.DS_STORAGE_BF16, use_graph=True)
    b = _fitter(prob, L.DS_STORAGE_BF16, use_graph=False)
    a.step(5)
    b.step(5)
    assert np.array_equal(a.params.cpu().numpy().view(np.uint32),
                          b.params.cpu().numpy().view(np.uint32))
    a.close()
    b.close()


def test_bf16_training_tracks_fp32(cuda_lib):
    from diffsplat_b200 import _lib as L
    from diffsplat_b200.scenes import psnr_from_ref_loss
    prob = small_problem(128, 128, 2000, seed=8, sh_degree=0)
    psnr = {}
    for name, storage in (("fp32", L.DS_STORAGE_FP32), ("bf16", L.DS_STORAGE_BF16)):
        f = _fitter(prob, storage)
        f.step(400)
        psnr[name] = psnr_from_ref_loss(f.loss())
        code, flags = f.status()
        assert code == 0
        f.close()
    print("PSNR after 400 steps:", psnr)
    assert psnr["bf16"] > psnr["fp32"] - 0.5
