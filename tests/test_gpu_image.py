"""GPU test of the aspect fit + pad of image targets (ds_image_fit) against a
NumPy FP64 restatement of the same geometry and filters (tolerance 1e-5)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _fit_ref(src, W, H, pad):
    sh, sw = src.shape[:2]
    scale = np.float32(min(np.float32(W - 2 * pad) / np.float32(sw),
                           np.float32(H - 2 * pad) / np.float32(sh)))
    fw, fh = max(1, int(np.float32(sw) * scale)), max(1, int(np.float32(sh) * scale))
    ox, oy = (W - fw) // 2, (H - fh) // 2
    out = np.zeros((H, W, 3))
    sx, sy = sw / fw, sh / fh
    s = src.astype(np.float64)
    for y in range(fh):
        for x in range(fw):
            if sx > 1 or sy > 1:
                x0, x1, y0, y1 = x * sx, (x + 1) * sx, y * sy, (y + 1) * sy
                acc, wsum = np.zeros(3), 0.0
                for v in range(int(np.floor(y0)), min(int(np.ceil(y1)), sh)):
                    wy = min(y1, v + 1) - max(y0, v)
                    for u in range(int(np.floor(x0)), min(int(np.ceil(x1)), sw)):
                        wx = min(x1, u + 1) - max(x0, u)
                        acc += wx * wy * s[v, u]
                        wsum += wx * wy
                val = acc / wsum
            else:
                u = min(max((x + 0.5) * sx - 0.5, 0), sw - 1)
                v = min(max((y + 0.5) * sy - 0.5, 0), sh - 1)
                u0, v0 = int(u), int(v)
                u1, v1 = min(u0 + 1, sw - 1), min(v0 + 1, sh - 1)
                tu, tv = u - u0, v - v0
                top = s[v0, u0] + (s[v0, u1] - s[v0, u0]) * tu
                bot = s[v1, u0] + (s[v1, u1] - s[v1, u0]) * tu
                val = top + (bot - top) * tv
            out[oy + y, ox + x] = val / 255.0
    return out, (fw, fh)


@pytest.mark.parametrize("sw,sh,W,H,pad", [(97, 61, 64, 64, 0), (40, 30, 128, 96, 4),
                                           (50, 120, 80, 60, 2), (64, 64, 64, 64, 0)])
def test_fit_matches_restatement(cuda_lib, sw, sh, W, H, pad):
    from diffsplat_b200 import api
    rng = np.random.default_rng(sw * 31 + sh)
    src = rng.integers(0, 256, (sh, sw, 3), dtype=np.uint8)
    got, fit = api.fit_image(src, W, H, pad)
    ref, fit_ref = _fit_ref(src, W, H, pad)
    assert fit == fit_ref
    assert np.abs(got.cpu().numpy() - ref).max() < 1e-5
