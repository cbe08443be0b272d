"""GPU tests of adaptive density control (ds_fitter_densify): the statistics,
the prune / clone / split rule and the rebuilt parameter and moment arrays
against a NumPy restatement, capacity handling, and training after it."""
import numpy as np
import pytest

from diffsplat_b200.scenes import small_problem

pytestmark = pytest.mark.gpu


def _fitter(prob, capacity, **kw):
    import torch
    from diffsplat_b200 import api
    f = api.Fitter(prob.width, prob.height, prob.params.shape[1], prob.sh_degree, lrs=prob.lrs,
                   max_isects=1 << 21, capacity=capacity, **kw)
    f.set_params(prob.params)
    f.set_target(torch.tensor(prob.target, device="cuda"))
    f.set_camera(prob.pv, prob.cam)
    return f


@pytest.mark.parametrize("deg", [0, 1])
def test_densify_matches_rule(cuda_lib, deg):
    prob = small_problem(128, 96, 800, seed=90 + deg, sh_degree=deg)
    f = _fitter(prob, capacity=4000)
    f.step(20)
    g, c = f.density_stats()
    g, c = g.cpu().numpy().copy(), c.cpu().numpy().astype(np.int64)
    assert (c <= 20).all() and (c > 0).any() and (g >= 0).all()
    P = f.params.cpu().numpy().copy()
    m, v = f.moments()
    M, V = m.cpu().numpy().copy(), v.cpu().numpy().copy()
    mean = np.where(c > 0, g / np.maximum(c, 1), 0)
    thr = float(np.quantile(mean[c > 0], 0.7))
    smax = np.exp(P[3:6].max(axis=0))
    sthr = float(np.median(smax))
    op = 1 / (1 + np.exp(-P[13].astype(np.float64)))
    minop = float(np.quantile(op, 0.1))
    mode = np.where(op < minop, 0, np.where((c > 0) & (mean >= thr), np.where(smax <= sthr, 2, 3), 1))
    emit = np.where(mode == 0, 0, np.where(mode == 1, 1, 2))
    n2 = f.densify(thr, sthr, minop, seed=7)
    assert n2 == emit.sum() and n2 == f.count
    Q = f.params.cpu().numpy()
    mq, vq = f.moments()
    MQ, VQ = mq.cpu().numpy(), vq.cpu().numpy()
    offs = np.concatenate([[0], np.cumsum(emit)[:-1]])
    for i in np.nonzero(mode)[0][:400]:
        j = offs[i]
        if mode[i] in (1, 2):
            assert np.array_equal(Q[:, j], P[:, i]) and np.array_equal(MQ[:, j], M[:, i])
            assert np.array_equal(VQ[:, j], V[:, i])
        if mode[i] == 2:
            assert np.array_equal(Q[:, j + 1], P[:, i]) and (MQ[:, j + 1] == 0).all()
        if mode[i] == 3:
            for k in (j, j + 1):
                assert np.allclose(Q[3:6, k], P[3:6, i] - np.log(1.6), atol=1e-5)
                assert np.array_equal(Q[6:, k], P[6:, i])
                d = np.abs(Q[0:3, k] - P[0:3, i]).max()
                assert d < 6 * np.exp(P[3:6, i].max())
                assert (MQ[:, k] == 0).all() and (VQ[:, k] == 0).all()
    g2, c2 = f.density_stats()
    assert (c2.cpu().numpy() == 0).all()
    l0 = None
    f.step(1)
    l0 = f.loss()
    f.step(100)
    assert f.loss() < l0
    code, flags = f.status()
    assert code == 0
    f.close()


def test_densify_over_capacity_changes_nothing(cuda_lib):
    from diffsplat_b200 import _lib as L
    prob = small_problem(96, 64, 500, seed=97)
    f = _fitter(prob, capacity=520)
    f.step(10)
    before = f.params.cpu().numpy().copy()
    with pytest.raises(L.DSError):
        f.densify(0.0, 1e9, 0.0)   # clones every visible splat: > capacity
    assert f.count == 500 and np.array_equal(f.params.cpu().numpy(), before)
    f.step(2)
    f.close()
