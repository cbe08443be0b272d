"""Shared runners for the parity tests: the library's layer path, the fused
fitter, the reference build (oracle/_ref) and the FP64 oracle on one problem."""
from __future__ import annotations

import numpy as np

FLT_MAX = np.float32(3.4028234663852886e38)


def rel_err(a, b, floor: float = 1e-12) -> float:
    """Norm-wise relative error ||a - b|| / max(||b||, floor)."""
    a = np.asarray(a, np.float64).reshape(-1)
    b = np.asarray(b, np.float64).reshape(-1)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), floor))


def ds_layers(prob, grad_mode=0, max_isects=1 << 22):
    """Runs the library's per-layer C ABI path (GaussActiv -> PerspProject ->
    TileRasterize -> MSE, then the backward of each)."""
    import torch
    from diffsplat_b200 import _lib as L
    from diffsplat_b200 import api

    n = prob.params.shape[1]
    P = torch.tensor(prob.params, device="cuda")
    S3 = api.activ_forward(P, prob.sh_degree, prob.cam)
    S2 = api.project_forward(S3, prob.pv)
    R = api.Rasterizer(prob.width, prob.height, n, max_isects)
    R.set_grad_mode(grad_mode)
    img = R.forward(S2)
    tgt = torch.tensor(prob.target, device="cuda")
    loss = api.mse_forward(img, tgt)
    gimg = api.mse_backward(img, tgt)
    G2 = R.backward(S2, gimg)
    G3 = api.project_backward(S3, prob.pv, G2, grad_mode=grad_mode)
    GP = api.activ_backward(P, S3, G3, prob.sh_degree, prob.cam)
    torch.cuda.synchronize()
    out = dict(
        S3=S3.cpu().numpy(), S2=S2.cpu().numpy(), image=img.cpu().numpy(),
        loss=float(loss.item()), G2=G2.cpu().numpy(), G3=G3.cpu().numpy(), GP=GP.cpu().numpy(),
        n_isects=R.isect_count(), visible=R.visible_count(),
        keys=R.download(L.DS_RASTER_KEYS), ids=R.download(L.DS_RASTER_IDS),
        ranges=R.download(L.DS_RASTER_RANGES),
        last_ids=R.download(L.DS_RASTER_LAST_IDS).reshape(prob.height, prob.width),
        alphas=R.download(L.DS_RASTER_ALPHAS).reshape(prob.height, prob.width),
        counts=R.download(L.DS_RASTER_COUNTS, n))
    R.close()
    return out


def ref_layers(prob):
    """Runs the reference's own layers (oracle/_ref/libdsref.so) on the same problem."""
    from oracle import ref

    R = ref.RefScene(prob.width, prob.height, prob.params, prob.sh_degree, prob.target, prob.pv,
                     prob.cam, prob.lrs)
    R.zero_grad()
    R.forward()
    loss = R.loss()
    R.backward()
    keys, ids = ref.canonical_order(R.download(0), R.download(1))
    out = dict(S3=R.download(10), S2=R.download(8), image=R.download(3), loss=loss,
               G2=R.download(9), G3=R.download(11), GP=R.download(6), n_isects=R.n_isects(),
               visible=R.visible(), keys=keys, ids=ids, ranges=R.download(2),
               alphas=R.download(4), last_ids=R.download(5))
    R.close()
    return out


def not_culled(S2: np.ndarray) -> np.ndarray:
    return S2[2] != FLT_MAX


def bf16_round(x):
    """FP32 -> BF16 -> FP32, round to nearest even (the BF16 render copy's rounding)."""
    u = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def render_params(P):
    """The attributes a BF16-storage forward reads: positions FP32, the rest BF16."""
    R = bf16_round(P)
    R[0:3] = P[0:3]
    return R
