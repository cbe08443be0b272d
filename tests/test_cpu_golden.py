"""Pins the FP64 oracle against golden vectors made by the reference's own CUDA
layers (tests/golden/*.npz, written by tests/golden/make_golden.py from a build
of src/layers/*.cu and src/optimizers/adam.cu).

The oracle follows the reference's gradient recurrences here (exact=False), so
every stage must agree with the reference to FP32 rounding: tile ids, splat ids
and tile ranges exactly, the depth half of each key to a few units in the last
place (the oracle's depth is FP64 rounded once), and the float stages to the
tolerances written in each assert."""
from pathlib import Path

import numpy as np
import pytest

from helpers import not_culled, rel_err
from oracle import oracle as O

GOLDEN = Path(__file__).resolve().parent / "golden"
CASES = ["grad_check_8", "persp_sh0_48x32", "persp_sh1_64x40", "persp_sh3_80x48"]


def _load(name):
    d = np.load(GOLDEN / f"{name}.npz")
    W, H, deg = (int(x) for x in d["meta"])
    return d, W, H, deg


def _row_lrs(lrs, rows):
    """Per-row learning rate in the [14 + 3K, n] layout: pos, scale, rot, sh_dc,
    opacity, then the SH rest (Gaussian3DAdamConfig's six groups)."""
    lr = np.empty(rows)
    lr[0:3], lr[3:6], lr[6:10], lr[10:13], lr[13], lr[14:] = (
        lrs[0], lrs[1], lrs[2], lrs[3], lrs[5], lrs[4])
    return lr


@pytest.fixture(scope="module", params=CASES)
def case(request):
    d, W, H, deg = _load(request.param)
    P = d["params"].astype(np.float64)
    fw, GP = O.loss_and_grads(P, deg, d["cam"], d["pv"], W, H, d["target"], exact=False)
    return request.param, d, W, H, deg, P, fw, GP


def test_no_ambiguous_tiles_or_pixels(case):
    _, d, *_, fw, _ = case
    assert fw.tile_amb.sum() == 0 and fw.px_amb.sum() == 0
    assert np.array_equal(fw.culled == 0, not_culled(d["S2"]))


def test_splat3d_and_splat2d(case):
    _, d, *_, fw, _ = case
    vis = not_culled(d["S2"])
    assert rel_err(fw.S3, d["S3"]) < 1e-6
    assert rel_err(fw.S2[:, vis], d["S2"][:, vis]) < 1e-6


def test_sorted_pairs_and_ranges(case):
    _, d, *_, fw, _ = case
    assert len(fw.keys) == len(d["keys"])
    assert np.array_equal(fw.keys >> np.uint64(32), d["keys"] >> np.uint64(32))
    assert np.array_equal(fw.ids, d["ids"])
    assert np.array_equal(fw.ranges, d["ranges"])
    lo = np.uint64(0xFFFFFFFF)
    dz = np.abs((fw.keys & lo).astype(np.int64) - (d["keys"] & lo).astype(np.int64))
    assert dz.max() <= 4


def test_image_alpha_last_ids_loss(case):
    _, d, *_, fw, _ = case
    assert np.abs(fw.image - d["image"]).max() < 1e-5
    assert np.abs(fw.alpha - d["alphas"]).max() < 1e-5
    assert np.array_equal(fw.last_ids, d["last_ids"])
    assert abs(fw.loss - float(d["loss"])) <= 1e-6 * abs(float(d["loss"]))


def test_parameter_gradients(case):
    _, d, *_, GP = case
    assert rel_err(GP, d["GP"]) < 1e-5
    assert np.abs(GP - d["GP"]).max() < 1e-6 * np.abs(d["GP"]).max() + 1e-9


def test_first_adam_step(case):
    """The first Adam step moves each parameter by about lr * sign(g), so the
    check is relative to each row's learning rate."""
    _, d, *_, P, _, GP = case
    lr = _row_lrs(d["lrs"], P.shape[0])
    after = np.empty_like(P)
    for r in range(P.shape[0]):
        z = np.zeros_like(P[r])
        after[r], _, _ = O.adam(P[r], GP[r], z, z, lr[r], 1)
    assert (np.abs(after - d["params_after_adam"]) / lr[:, None]).max() < 1e-3


def test_first_adam_step_grouped(case):
    """The grouped oracle Adam (the CPU baseline's optimizer) applies the
    registerGaussian3DGroups learning rates row by row, like the reference's
    Adam::step on the golden fixture."""
    _, d, *_, P, _, GP = case
    lr = _row_lrs(d["lrs"], P.shape[0])
    z = np.zeros_like(P)
    after, _, _ = O.adam_gaussian3d(P, GP, z, z, tuple(float(x) for x in d["lrs"]), 1)
    assert (np.abs(after - d["params_after_adam"]) / lr[:, None]).max() < 1e-3
