"""Host scene I/O through the C ABI (no GPU): PLY read/write in the layout of
src/io/ply_io.cpp and SplatUtils::normalizeScene (src/utils/splat_utils.h)."""
import numpy as np
import pytest

from diffsplat_b200 import _lib as L
from diffsplat_b200 import api

PROPS_3DGS = ["x", "y", "z", "nx", "ny", "nz", "f_dc_0", "f_dc_1", "f_dc_2"]


def _records(n, bands, seed=0):
    rng = np.random.default_rng(seed)
    rec = rng.normal(size=(n, 59)).astype(np.float32)
    rec[:, 13 + 3 * bands:58] = 0.0
    return rec


@pytest.mark.parametrize("bands,deg", [(0, 0), (3, 1), (8, 2), (15, 3)])
def test_round_trip(tmp_path, bands, deg):
    rec = _records(257, bands, seed=bands)
    path = tmp_path / "scene.ply"
    api.write_ply(path, rec, bands)
    back, d = api.read_ply(path)
    assert d == deg
    assert np.array_equal(back.view(np.uint32), rec.view(np.uint32))


def test_reads_training_layout_with_frame_flip(tmp_path):
    """A file in the property order written by 3DGS training (normals, f_dc,
    f_rest, opacity, scale, rot) is read by name; y, z and the quaternion's
    y, z change sign (OpenCV -> OpenGL)."""
    n, K = 10, 3
    rng = np.random.default_rng(3)
    names = PROPS_3DGS + [f"f_rest_{k}" for k in range(3 * K)] + [
        "opacity", "scale_0", "scale_1", "scale_2", "rot_0", "rot_1", "rot_2", "rot_3"]
    data = rng.normal(size=(n, len(names))).astype(np.float32)
    header = ("ply\nformat binary_little_endian 1.0\n"
              f"element vertex {n}\n" + "".join(f"property float {p}\n" for p in names) +
              "end_header\n")
    path = tmp_path / "train.ply"
    path.write_bytes(header.encode() + data.tobytes())
    rec, deg = api.read_ply(path)
    col = {p: data[:, k] for k, p in enumerate(names)}
    assert deg == 1
    assert np.array_equal(rec[:, 0], col["x"])
    assert np.array_equal(rec[:, 1], -col["y"])
    assert np.array_equal(rec[:, 2], -col["z"])
    assert np.array_equal(rec[:, 3:6], np.stack([col[f"scale_{k}"] for k in range(3)], 1))
    assert np.array_equal(rec[:, 6], col["rot_0"])
    assert np.array_equal(rec[:, 7], col["rot_1"])
    assert np.array_equal(rec[:, 8], -col["rot_2"])
    assert np.array_equal(rec[:, 9], -col["rot_3"])
    assert np.array_equal(rec[:, 10:13], np.stack([col[f"f_dc_{k}"] for k in range(3)], 1))
    assert np.array_equal(rec[:, 13:13 + 3 * K],
                          np.stack([col[f"f_rest_{k}"] for k in range(3 * K)], 1))
    assert np.array_equal(rec[:, 58], col["opacity"])
    assert (rec[:, 13 + 3 * K:58] == 0).all()


def test_params_conversion_round_trip():
    rec = _records(40, 8, seed=5)
    P = api.records_to_params(rec, 2)
    assert P.shape == (14 + 24, 40)
    assert np.array_equal(P[13], rec[:, 58])
    assert np.array_equal(P[14 + 8 * 1 + 2], rec[:, 13 + 8 + 2])  # G channel, band 2
    assert np.array_equal(api.params_to_records(P), rec)


def test_errors(tmp_path):
    rec = _records(4, 0)
    good = tmp_path / "a.ply"
    api.write_ply(good, rec, 0)
    with pytest.raises(L.DSError):
        api.read_ply(tmp_path / "missing.ply")
    txt = tmp_path / "a.txt"
    txt.write_bytes(good.read_bytes())
    with pytest.raises(L.DSError):
        api.read_ply(txt)
    short = tmp_path / "short.ply"
    short.write_bytes(good.read_bytes()[:-8])
    with pytest.raises(L.DSError):
        api.read_ply(short)
    no_rot = tmp_path / "norot.ply"
    no_rot.write_bytes(good.read_bytes().replace(b"property float rot_3\n", b""))
    with pytest.raises(L.DSError):
        api.read_ply(no_rot)
    with pytest.raises(L.DSError):
        api.write_ply(tmp_path / "b.ply", rec, 5)


def test_normalize_scene_matches_restatement():
    """Centroid by sequential FP32 sums, shift, scale the largest |coordinate| to
    scene_scale, add log(scale) to the log-scales."""
    rng = np.random.default_rng(9)
    rec = _records(1000, 0)
    rec[:, 0:3] = rng.normal(3.0, 5.0, size=(1000, 3)).astype(np.float32)
    out = api.normalize_scene(rec, 2.0)
    pos = rec[:, 0:3].copy()
    c = np.add.accumulate(pos, axis=0, dtype=np.float32)[-1] * (np.float32(1) / np.float32(1000))
    pos = pos - c
    ext = np.abs(pos).max()
    s = np.float32(2.0) / ext
    assert np.array_equal(out[:, 0:3], pos * s)
    assert np.allclose(out[:, 3:6], rec[:, 3:6] + np.log(np.float64(s)), rtol=0, atol=1e-6)
    assert np.abs(out[:, 0:3]).max() == np.float32(2.0)
    assert np.array_equal(out[:, 6:], rec[:, 6:])


# ---- against the reference's own PLY code (src/io/ply_io.cpp) -------------------
from pathlib import Path  # noqa: E402

GOLDEN = Path(__file__).resolve().parent / "golden"


@pytest.mark.parametrize("name,bands,deg", [("sh0", 0, 0), ("sh3", 15, 3)])
def test_reads_files_written_by_reference_saver(name, bands, deg):
    """tests/golden/ref_*.ply were written by the reference's PLYSaver::save
    (tests/golden/make_golden_ply.py): ds_ply_read gives back the records they
    were written from, and what the reference's PLYLoader::load read from the
    same file, bit for bit."""
    d = np.load(GOLDEN / "ply_records.npz")
    rec, got_deg = api.read_ply(GOLDEN / f"ref_{name}.ply")
    assert got_deg == deg == int(d[f"{name}_degree"])
    assert np.array_equal(rec.view(np.uint32), d[f"{name}_records"].view(np.uint32))
    assert np.array_equal(rec.view(np.uint32), d[f"{name}_loaded"].view(np.uint32))


@pytest.mark.parametrize("bands,deg", [(0, 0), (3, 1), (8, 2), (15, 3)])
def test_writer_matches_reference_saver_byte_for_byte(tmp_path, bands, deg):
    """ds_ply_write produces the same bytes as PLYSaver::save for the same
    records, and PLYLoader::load reads our file back to those records."""
    from oracle import ref_ply
    if not ref_ply.available():
        pytest.skip("oracle/_ref/libdsref_ply.so not built (needs the reference sources)")
    rec = _records(97, bands, seed=40 + bands)
    ours, theirs = tmp_path / "ours.ply", tmp_path / "theirs.ply"
    api.write_ply(ours, rec, bands)
    ref_ply.save(theirs, rec, bands)
    assert ours.read_bytes() == theirs.read_bytes()
    back, d = ref_ply.load(ours)
    assert d == deg
    assert np.array_equal(back.view(np.uint32), rec.view(np.uint32))


def test_golden_files_are_the_reference_savers_output():
    """The committed fixtures equal what the reference's saver writes now."""
    from oracle import ref_ply
    if not ref_ply.available():
        pytest.skip("oracle/_ref/libdsref_ply.so not built (needs the reference sources)")
    import tempfile
    d = np.load(GOLDEN / "ply_records.npz")
    with tempfile.TemporaryDirectory() as t:
        for name, bands in (("sh0", 0), ("sh3", 15)):
            p = Path(t) / f"{name}.ply"
            ref_ply.save(p, d[f"{name}_records"], bands)
            assert p.read_bytes() == (GOLDEN / f"ref_{name}.ply").read_bytes()
