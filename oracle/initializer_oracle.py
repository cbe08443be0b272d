"""FP64 CPU restatement of the learned initializer's network (test
infrastructure only): the same 3x3 convolutions (padding 1), tanh-form GELU,
head and head decode as diffsplat_b200/initializer.py, evaluated with torch in
float64 on the CPU from the network's BF16 weights, with autograd for the
gradients.  Parity unpinned: there is no reference counterpart."""
from __future__ import annotations

import torch
import torch.nn.functional as F


def weights_fp64(conv):
    """[Cout, Kp] (k = (ky*3 + kx)*Cin + c) BF16 weights -> OIHW float64."""
    w = conv.w16.detach().cpu().double()[:, :9 * conv.cin]
    return w.view(conv.cout, 3, 3, conv.cin).permute(0, 3, 1, 2).contiguous()


def forward(init, images, weights=None):
    """images [B, S, S, 3] -> head output [B * G * G, 56] (float64), with the
    per-layer weights and biases as leaf tensors (returned for autograd)."""
    x = images.detach().cpu().double().to(torch.bfloat16).double().permute(0, 3, 1, 2)
    if weights is None:
        weights = [(weights_fp64(m).requires_grad_(True),
                    m.b.detach().cpu().double().requires_grad_(True)) for m in init.modules()]
    for (w, b), m in zip(weights[:-1], init.layers):
        x = F.gelu(F.conv2d(x, w, b, stride=m.stride, padding=1), approximate="tanh")
    w, b = weights[-1]
    out = F.conv2d(x, w, b, stride=1, padding=1)
    return out.permute(0, 2, 3, 1).reshape(-1, 56), weights


def decode(init, out):
    """Head output -> [14, B * splats] parameters (float64)."""
    G = init.grid
    B = out.shape[0] // (G * G)
    o = out.view(B, G * G, 4, 14).reshape(B * G * G * 4, 14)
    base = init.base.detach().cpu().double().view(-1, 3).repeat(B, 1)
    step = torch.tensor(init.step, dtype=torch.float64)
    p = torch.empty_like(o)
    p[:, 0:3] = base + o[:, 0:3] * step
    p[:, 3:6] = init.base_ls + o[:, 3:6]
    p[:, 6] = 1.0 + o[:, 6]
    p[:, 7:14] = o[:, 7:14]
    return p.T
