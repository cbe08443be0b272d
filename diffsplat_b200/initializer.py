"""Learned initializer: a 5-level 3x3-conv encoder (channels 32-64-128-256-256,
GELU, BF16 weights and activations, FP32 accumulation on tcgen05 tensor
cores) with a head that predicts 4 splats per cell of a 64 x 64 grid from a
512 x 512 RGB target.  Trained with an L1 loss on the parameters of splats
fitted by the plain fitter plus the rendered-image L2 loss through this
library's activation / projection / rasterizer forward and backward; AdamW.

Splats are in the pinhole frame of the plain small fitter: camera at the
origin looking +z, fx = fy = image width, centred principal point; cell
(i, j) holds splats at the centres of its 2 x 2 sub-cells at depth 4.  With a
zero head the network outputs that grid (identity rotations, 3-pixel sigma,
grey colour, opacity 0.5), which is also the init the training pairs are
fitted from, so predicted and fitted splat k correspond by index.
"""
from __future__ import annotations

import math

import numpy as np
import torch

from . import _lib as L
from . import api, nn
from .scenes import pinhole_pv

CHANNELS = (32, 64, 128, 256, 256)
STRIDES = (1, 2, 2, 2, 1)
Z0 = 4.0


class Initializer:
    def __init__(self, size: int = 512, seed: int = 0):
        assert size % 8 == 0
        self.size = size
        self.grid = size // 8
        gen = torch.Generator().manual_seed(seed)
        cin, self.layers = 3, []
        for c, s in zip(CHANNELS, STRIDES):
            self.layers.append(nn.Conv3x3(cin, c, s, gelu=True, gen=gen))
            cin = c
        self.head = nn.Conv3x3(cin, 56, 1, gelu=False, gen=gen)
        self.head.w.zero_()
        self.head.w16.zero_()
        self.gemm = nn.Gemm()
        f = float(size)
        self.fx = f
        self.pv = pinhole_pv(size, size, f, f, size / 2, size / 2)
        self.cam = np.zeros(3, np.float32)
        G = self.grid
        base = np.zeros((G * G * 4, 3), np.float32)
        for i in range(G):
            for j in range(G):
                for q in range(4):
                    u = 8 * j + 2 + 4 * (q % 2) + 0.5
                    v = 8 * i + 2 + 4 * (q // 2) + 0.5
                    s = (i * G + j) * 4 + q
                    base[s] = [(u - size / 2) * Z0 / f, (v - size / 2) * Z0 / f, Z0]
        self.base = torch.tensor(base.reshape(-1), device="cuda")
        self.step = (8.0 * Z0 / f, 8.0 * Z0 / f, 1.0)
        self.base_ls = math.log(3.0 * Z0 / f)

    @property
    def splats(self) -> int:
        return 4 * self.grid * self.grid

    def modules(self):
        return self.layers + [self.head]

    def parameters(self):
        return [p for m in self.modules() for p in m.params()]

    def forward(self, images: torch.Tensor) -> torch.Tensor:
        """images [B, S, S, 3] FP32 CUDA -> head output [B * G * G, 56] FP32."""
        x = nn.cast_bf16(images)
        self.zs = []
        for layer in self.layers:
            z, x = layer.forward(self.gemm, x)
            self.zs.append(z)
        out, _ = self.head.forward(self.gemm, x)
        self.batch = images.shape[0]
        return out.reshape(-1, 56)

    def decode(self, out: torch.Tensor) -> torch.Tensor:
        """Head output -> field-major splat parameters [14, B * splats]."""
        B = out.shape[0] // (self.grid * self.grid)
        params = torch.empty(14, B * self.splats, dtype=torch.float32, device="cuda")
        L.call("ds_head_decode", out.data_ptr(), B, self.grid, self.base.data_ptr(),
               L.fptr(self.step), self.base_ls, params.data_ptr(), nn._s())
        return params

    def backward(self, params, g_render=None, target=None, w_render=1.0, w_l1=1.0):
        """Gradients of w_render * rendered loss + w_l1 * L1(params - target)
        (g_render = dL/dparams of the rendered loss, target = fitted params;
        the L1 term's weight is per parameter) into every layer's gw / gb."""
        B = self.batch
        dout = torch.empty(B * self.grid * self.grid, 56, dtype=torch.bfloat16, device="cuda")
        L.call("ds_head_encode_grad", nn._p(g_render), params.data_ptr(), nn._p(target),
               float(w_render), float(w_l1), B, self.grid, L.fptr(self.step), dout.data_ptr(),
               nn._s())
        G = self.grid
        dz = self.head.backward(self.gemm, dout.view(B, G, G, 56), z_prev=self.zs[-1])
        for k in range(len(self.layers) - 1, -1, -1):
            zp = self.zs[k - 1] if k > 0 else None
            dz = self.layers[k].backward(self.gemm, dz, z_prev=zp, need_dx=k > 0)

    def predict(self, image: torch.Tensor) -> np.ndarray:
        """One target [S, S, 3] -> initial parameters [14, splats] (numpy)."""
        out = self.forward(image[None].contiguous())
        return self.decode(out).cpu().numpy()

    def zero_params(self, batch: int = 1) -> np.ndarray:
        """The grid init (zero head output) for `batch` images: [14, batch * splats]."""
        out = torch.zeros(batch * self.grid * self.grid, 56, device="cuda")
        return self.decode(out).cpu().numpy()


def render_loss_grads(init: Initializer, params: torch.Tensor, targets: torch.Tensor):
    """Reference MSE of each image's splats against its target and
    dL/dparams through the layer pipeline (activation, projection,
    rasterizer, MSE and their backward).  params [14, B * splats]."""
    B, S = targets.shape[0], init.splats
    grads = torch.empty_like(params)
    losses = []
    size = init.size
    r = getattr(init, "_raster", None)
    if r is None:
        r = init._raster = api.Rasterizer(size, size, S, 1 << 22)
    for b in range(B):
        P = params[:, b * S:(b + 1) * S].contiguous()
        s3 = api.activ_forward(P, 0, init.cam)
        s2 = api.project_forward(s3, init.pv)
        img = r.forward(s2)
        t = targets[b]
        losses.append(api.mse_forward(img, t).clone())
        gimg = api.mse_backward(img, t)
        g2 = r.backward(s2, gimg)
        g3 = api.project_backward(s3, init.pv, g2)
        grads[:, b * S:(b + 1) * S] = api.activ_backward(P, s3, g3, 0, init.cam)
    return torch.cat(losses), grads


# ---- training pairs, training, evaluation -----------------------------------

def make_targets_gpu(count: int, size: int = 512, seed: int = 0) -> torch.Tensor:
    """The same target recipe evaluated in FP32 on the GPU (synthetic training
    data for large datasets): [count, size, size, 3] CUDA float32, quantised
    to 1/255 steps."""
    g = torch.Generator().manual_seed(seed)
    u = torch.arange(size, device="cuda", dtype=torch.float32)[None, :] + 0.5
    v = torch.arange(size, device="cuda", dtype=torch.float32)[:, None] + 0.5
    base = torch.stack([0.15 + 0.5 * u / size + 0 * v, 0.15 + 0.5 * v / size + 0 * u,
                        0.65 - 0.25 * (u / size + v / size)], -1)
    checker = ((torch.floor(u / 8.0) + torch.floor(v / 8.0)) % 2.0)
    base = base + (0.1 * checker - 0.05)[..., None]
    out = torch.empty(count, size, size, 3, device="cuda")
    for k in range(count):
        nb = int(torch.randint(500, 3001, (1,), generator=g))
        cx = torch.rand(nb, generator=g).cuda() * size
        cy = torch.rand(nb, generator=g).cuda() * size
        sg = (2.0 + 38.0 * torch.rand(nb, generator=g)).cuda()
        col = torch.rand(nb, 3, generator=g).cuda()
        img = base.clone()
        for a in range(0, nb, 256):
            d2 = ((u[None] - cx[a:a + 256, None, None]) ** 2 +
                  (v[None] - cy[a:a + 256, None, None]) ** 2)
            w = torch.exp(-d2 / (2.0 * sg[a:a + 256, None, None] ** 2))
            img += 0.5 * torch.einsum("bhw,bc->hwc", w, col[a:a + 256] - 0.5)
        out[k] = torch.round(img.clamp(0.0, 1.0) * 255.0) / 255.0
    return out


def make_targets(count: int, size: int = 512, seed: int = 0) -> np.ndarray:
    """Procedural targets of the plain small fitter's recipe at `size`^2 with
    500-3000 blobs each: [count, size, size, 3] float32."""
    from .scenes import make_target
    rng = np.random.Generator(np.random.PCG64(seed))
    blobs = rng.integers(500, 3001, count)
    return np.stack([make_target(size, size, int(blobs[k]), seed * 1_000_003 + k)
                     for k in range(count)])


def fit_pairs(init: Initializer, targets, steps: int, batch: int = 64,
              storage: int = L.DS_STORAGE_BF16) -> np.ndarray:
    """Splats fitted to each target by the batched fitter from the grid init:
    [count, 14, splats] float32."""
    from .scenes import PLAIN_SMALL_LRS
    S, n = init.size, init.splats
    P0 = init.zero_params(1)
    out = np.zeros((len(targets), 14, n), np.float32)
    for a in range(0, len(targets), batch):
        idx = range(a, min(a + batch, len(targets)))
        b = api.Batch([(S, S, n)] * len(idx), lrs=PLAIN_SMALL_LRS, storage=storage,
                      max_isects=len(idx) * n * 16)
        for k, t in enumerate(idx):
            b.set_params(k, P0)
            b.set_target(k, torch.as_tensor(targets[t], device="cuda"))
            b.set_camera(k, init.pv, init.cam)
        b.step(steps)
        for k, t in enumerate(idx):
            out[t] = b.instance_params(k).cpu().numpy()
        b.close()
    return out


def train(init: Initializer, targets: np.ndarray, fitted: np.ndarray, steps: int,
          batch: int = 32, lr: float = 3e-4, weight_decay: float = 1e-2, w_render: float = 10.0,
          seed: int = 0, log_every: int = 0):
    """AdamW on L1(params - fitted) (mean over entries) + w_render * rendered
    MSE (mean over images).  Returns [(step, l1, render_mse)]."""
    rng = np.random.Generator(np.random.PCG64(seed))
    opt = nn.AdamW(init.parameters(), lr=lr, weight_decay=weight_decay)
    hist = []
    n = len(targets)
    for it in range(steps):
        idx = rng.choice(n, size=min(batch, n), replace=False)
        imgs = (targets[torch.as_tensor(idx, device="cuda")] if torch.is_tensor(targets)
                else torch.tensor(targets[idx], device="cuda"))
        fit = torch.tensor(np.concatenate(list(fitted[idx]), axis=1), device="cuda")
        out = init.forward(imgs)
        params = init.decode(out)
        losses, g = render_loss_grads(init, params, imgs)
        B = len(idx)
        init.backward(params, g_render=g, target=fit, w_render=w_render / B,
                      w_l1=1.0 / params.numel())
        opt.step()
        if log_every and (it % log_every == 0 or it == steps - 1):
            l1 = float((params - fit).abs().mean())
            hist.append((it, l1, float(losses.mean())))
    init.gemm.check()
    return hist


def psnr(loss: float) -> float:
    from .scenes import psnr_from_ref_loss
    return psnr_from_ref_loss(loss)


def steps_to_psnr(params0: np.ndarray, target: np.ndarray, init: Initializer, goal: float,
                  max_steps: int, check_every: int = 10) -> dict:
    """Plain FP32 fitter from params0 until the PSNR reaches `goal` (checked
    every `check_every` steps): steps, device seconds, final PSNR."""
    from .scenes import PLAIN_SMALL_LRS
    S = init.size
    f = api.Fitter(S, S, params0.shape[1], 0, lrs=PLAIN_SMALL_LRS, max_isects=1 << 22)
    f.set_params(params0)
    f.set_target(torch.as_tensor(target, device="cuda"))
    f.set_camera(init.pv, init.cam)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    steps, p0, p = 0, None, 0.0
    a.record()
    while steps < max_steps:
        f.step(check_every)
        steps += check_every
        p = psnr(f.loss())
        if p0 is None:
            p0 = p
        if p >= goal:
            break
    b.record()
    torch.cuda.synchronize()
    f.close()
    return {"steps": steps, "seconds": a.elapsed_time(b) / 1e3, "psnr": p, "psnr_first": p0,
            "reached": p >= goal}


def random_init(init: Initializer, seed: int) -> np.ndarray:
    """The plain small fitter's random init for the initializer's camera and
    splat count (means in the frustum at depth 2-6, log-scales N(-3, 0.5))."""
    from .scenes import random_splats
    S = init.size
    return random_splats(init.splats, S, S, init.fx, init.fx, S / 2, S / 2, seed)


def evaluate(init: Initializer, targets, goal: float = 28.0, max_steps: int = 2000,
             seed: int = 0) -> dict:
    """Steps and seconds to `goal` dB per held-out target for three inits:
    random (the plain small fitter's), grid (the zero-head output, i.e. the
    method without the trained network) and learned; the learned init falls
    back to random when its first-check PSNR is below the random init's.
    Learned seconds include the network forward."""
    rows = []
    grid = init.zero_params(1)
    for k, t in enumerate(targets):
        img = torch.as_tensor(t, device="cuda")
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        P_learn = init.predict(img)
        b.record()
        torch.cuda.synchronize()
        net_s = a.elapsed_time(b) / 1e3
        rnd = steps_to_psnr(random_init(init, seed * 7919 + k), t, init, goal, max_steps)
        grd = steps_to_psnr(grid, t, init, goal, max_steps)
        lrn = steps_to_psnr(P_learn, t, init, goal, max_steps)
        # a NaN first PSNR (a prediction that does not render) falls back too
        fallback = not (lrn["psnr_first"] >= rnd["psnr_first"])
        if fallback:
            lrn = dict(rnd)
        lrn["seconds"] += net_s
        rows.append({"random": rnd, "grid": grd, "learned": lrn, "fallback": fallback,
                     "net_s": net_s})
    out = {"goal_db": goal, "max_steps": max_steps, "targets": len(rows),
           "fallbacks": sum(r["fallback"] for r in rows)}
    for arm in ("random", "grid", "learned"):
        out[f"{arm}_steps"] = float(np.mean([r[arm]["steps"] for r in rows]))
        out[f"{arm}_seconds"] = float(np.mean([r[arm]["seconds"] for r in rows]))
        out[f"{arm}_reached"] = int(sum(r[arm]["reached"] for r in rows))
        out[f"{arm}_psnr_first"] = float(np.mean([r[arm]["psnr_first"] for r in rows]))
        out[f"{arm}_psnr_final"] = float(np.mean([r[arm]["psnr"] for r in rows]))
    return out
