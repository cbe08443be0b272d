"""The two tile-sort paths of the rasterizer give the same lists.

Grids of at most 8192 tiles sort the (tile, splat) pairs by one stable
counting pass whose scan also yields the tile ranges; larger grids (and the
allocation-free forward) use radix passes over the tile id followed by a
boundary search for the ranges.  Both must equal the reference's sorted
(tile << 32 | depth) order with equal keys by splat id
(src/layers/tile_rasterize_layer.cu:52-162)."""
import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

from diffsplat_b200.scenes import small_problem
from tests.helpers import ds_layers, ref_layers

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]

CASES = [(160, 90, 600, 4), (1920, 1080, 6000, 5), (2048, 1024, 6000, 6)]


def _lists(W, H, n, seed, log_scale_mean=-2.5, cap=1 << 23):
    prob = small_problem(W, H, n, seed=seed, log_scale_mean=log_scale_mean)
    out = ds_layers(prob, max_isects=cap)
    return prob, out


def _radix_lists(tmp_path, W, H, n, seed, log_scale_mean=-2.5, cap=1 << 23):
    """The same layer run in a process that forces the radix path."""
    dst = tmp_path / f"radix_{W}x{H}.npz"
    code = (
        "import sys; sys.path.insert(0, %r)\n"
        "import numpy as np\n"
        "from tests.test_gpu_tile_sort import _lists\n"
        "_, o = _lists(%d, %d, %d, %d, %r, %d)\n"
        "np.savez(%r, keys=o['keys'], ids=o['ids'], ranges=o['ranges'], image=o['image'],"
        " G2=o['G2'])\n" % (str(ROOT), W, H, n, seed, log_scale_mean, cap, str(dst)))
    env = dict(os.environ, DS_TILE_SORT="radix")
    r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    return np.load(dst)


@pytest.mark.parametrize("W,H,n,seed", CASES)
def test_counting_and_radix_tile_sorts_agree(cuda_lib, tmp_path, W, H, n, seed):
    _, me = _lists(W, H, n, seed)
    rx = _radix_lists(tmp_path, W, H, n, seed)
    assert 0 < me["n_isects"] < (1 << 23)
    for k in ("keys", "ids", "ranges"):
        assert np.array_equal(me[k], rx[k]), k
    assert np.array_equal(me["image"].view(np.uint32), rx["image"].view(np.uint32))
    assert np.array_equal(me["G2"].view(np.uint32), rx["G2"].view(np.uint32))


def test_counting_sort_chunks_beyond_16_bit_offsets(cuda_lib, tmp_path):
    """About 22M pairs: each of the 296 chunks holds more than 65535 pairs,
    beyond the scatter's 16-bit per-warp offsets, so every chunk is walked by
    one warp with 32-bit counters.  Same lists as the radix path."""
    args = (1024, 1024, 20000, 8, -1.2, 1 << 25)
    _, me = _lists(*args)
    assert 296 * 65535 < me["n_isects"] < (1 << 25)
    rx = _radix_lists(tmp_path, *args)
    for k in ("keys", "ids", "ranges"):
        assert np.array_equal(me[k], rx[k]), k
    assert np.array_equal(me["image"].view(np.uint32), rx["image"].view(np.uint32))


@pytest.mark.parametrize("W,H", [(2048, 1024), (2064, 1024)])
def test_largest_counting_grid_and_first_radix_grid_vs_reference(cuda_lib, W, H):
    """8192 tiles (the largest grid of the counting pass) and 8256 tiles (the
    first that takes the radix passes): bit-exact lists against the
    reference build."""
    from oracle import ref
    if not ref.available():
        pytest.skip("reference build absent")
    prob = small_problem(W, H, 5000, seed=9, log_scale_mean=-2.5)
    me = ds_layers(prob, max_isects=1 << 23)
    rf = ref_layers(prob)
    assert me["n_isects"] == rf["n_isects"] > 0
    assert me["n_isects"] < (1 << 23)
    assert np.array_equal(me["keys"], rf["keys"])
    assert np.array_equal(me["ids"], rf["ids"])
    assert np.array_equal(me["ranges"], rf["ranges"])
