"""Host image I/O through the C ABI (no GPU): the PNG / PPM decoder against
PIL's encoder and decoder (test-only), the PNG writer's bytes, and errors."""
import numpy as np
import pytest

from diffsplat_b200 import _lib as L
from diffsplat_b200 import api

PIL = pytest.importorskip("PIL.Image")


def _img(h, w, seed):
    rng = np.random.default_rng(seed)
    base = rng.integers(0, 256, (h, w, 3), dtype=np.uint8)
    # smooth regions make the filters and back-references non-trivial
    base[: h // 2, : w // 2] = np.linspace(0, 255, w // 2, dtype=np.uint8)[None, :, None]
    return base


@pytest.mark.parametrize("mode", ["RGB", "RGBA", "L", "LA", "P"])
@pytest.mark.parametrize("optimize", [False, True])
def test_png_decode_matches_pil(tmp_path, mode, optimize):
    a = _img(37, 53, 1)
    im = PIL.fromarray(a, "RGB")
    if mode == "P":
        im = im.quantize(64)
    else:
        im = im.convert(mode)
    path = tmp_path / "x.png"
    im.save(path, optimize=optimize, compress_level=9)
    ref = np.asarray(PIL.open(path).convert("RGB"))
    got = api.read_image(path)
    assert got.shape == ref.shape and np.array_equal(got, ref)


def test_png_decode_large_with_all_filters(tmp_path):
    a = _img(300, 411, 2)
    path = tmp_path / "big.png"
    PIL.fromarray(a).save(path, optimize=True)
    assert np.array_equal(api.read_image(path), a)


def test_ppm_pgm(tmp_path):
    a = _img(20, 30, 3)
    PIL.fromarray(a).save(tmp_path / "x.ppm")
    assert np.array_equal(api.read_image(tmp_path / "x.ppm"), a)
    PIL.fromarray(a[..., 0]).save(tmp_path / "x.pgm")
    assert np.array_equal(api.read_image(tmp_path / "x.pgm"), np.repeat(a[..., :1], 3, axis=2))


def test_write_png_quantises_like_reference(tmp_path):
    rng = np.random.default_rng(4)
    f = rng.uniform(-0.2, 1.2, (23, 31, 3)).astype(np.float32)
    path = tmp_path / "out.png"
    api.write_png(path, f)
    got = np.asarray(PIL.open(path).convert("RGB"))
    want = np.clip(f * np.float32(255), 0, 255).astype(np.uint8)  # truncation, as the reference
    assert np.array_equal(got, want)
    assert np.array_equal(api.read_image(path), want)


def test_errors(tmp_path):
    a = _img(16, 16, 5)
    good = tmp_path / "a.png"
    PIL.fromarray(a).save(good)
    bad = tmp_path / "bad.png"
    bad.write_bytes(good.read_bytes()[:60])
    with pytest.raises(L.DSError):
        api.read_image(bad)
    with pytest.raises(L.DSError):
        api.read_image(tmp_path / "missing.png")
    jpg = tmp_path / "a.jpg"
    PIL.fromarray(a).save(jpg)
    with pytest.raises(L.DSError):
        api.read_image(jpg)


def _png_chunk(kind: bytes, data: bytes) -> bytes:
    import struct
    import zlib
    return struct.pack(">I", len(data)) + kind + data + struct.pack(
        ">I", zlib.crc32(kind + data) & 0xFFFFFFFF)


def test_png_stream_expanding_past_the_image_is_rejected(tmp_path):
    """A tiny IDAT that inflates far beyond the (stride + 1) * H bytes its
    header announces fails the decode instead of expanding in memory."""
    import struct
    import zlib
    W = H = 4
    ihdr = struct.pack(">IIBBBBB", W, H, 8, 2, 0, 0, 0)
    bomb = zlib.compress(b"\0" * (64 << 20), 9)  # 64 MiB of zeros in about 64 KB
    assert len(bomb) < (1 << 17)
    png = b"\x89PNG\r\n\x1a\n" + _png_chunk(b"IHDR", ihdr) + _png_chunk(b"IDAT", bomb) + \
        _png_chunk(b"IEND", b"")
    path = tmp_path / "bomb.png"
    path.write_bytes(png)
    with pytest.raises(L.DSError):
        api.read_image(path)
    # the same header with exactly its rows decodes
    rows = b"".join(b"\0" + bytes(range(3 * W)) for _ in range(H))
    ok = b"\x89PNG\r\n\x1a\n" + _png_chunk(b"IHDR", ihdr) + _png_chunk(
        b"IDAT", zlib.compress(rows)) + _png_chunk(b"IEND", b"")
    path.write_bytes(ok)
    img = api.read_image(path)
    assert img.shape == (H, W, 3) and np.array_equal(img[0].reshape(-1), np.arange(3 * W))
