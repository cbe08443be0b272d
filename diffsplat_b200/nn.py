"""Tensor-core building blocks of the learned initializer on the C ABI:
BF16 GEMM (tcgen05), 3x3 convolutions as im2col + GEMM with fused bias/GELU,
their backward (col2im with the producing layer's GELU derivative, weight
gradients by split-K GEMM over pixels) and AdamW.  Activations are NHWC BF16;
torch tensors are only the memory.
"""
from __future__ import annotations

import ctypes as C
import math

import torch

from . import _lib as L

EPI_F32, EPI_BIAS_GELU, EPI_BIAS_F32 = 0, 1, 2


def _s():
    return torch.cuda.current_stream().cuda_stream


def _p(t):
    return None if t is None else t.data_ptr()


class Gemm:
    """D[M, N] = A[M, K] . B[N, K]^T (BF16 in, FP32 accumulate)."""

    def __init__(self):
        self.err = torch.zeros(1, dtype=torch.int32, device="cuda")
        self.ws = torch.empty(0, dtype=torch.float32, device="cuda")

    def __call__(self, A, B, epilogue=EPI_F32, bias=None, D=None, Y=None, Z=None, splits=1):
        assert A.dtype == torch.bfloat16 and B.dtype == torch.bfloat16
        M, K = A.shape
        N, K2 = B.shape
        assert K == K2 and A.stride(1) == 1 and B.stride(1) == 1
        if epilogue == EPI_BIAS_GELU:
            Y = Y if Y is not None else torch.empty(M, N, dtype=torch.bfloat16, device="cuda")
            Z = Z if Z is not None else torch.empty(M, N, dtype=torch.bfloat16, device="cuda")
            ldd, ldy = N, Y.stride(0)
        else:
            D = D if D is not None else torch.empty(M, N, dtype=torch.float32, device="cuda")
            ldd, ldy = D.stride(0), N
        ws = None
        if splits > 1:
            need = splits * M * ldd
            if self.ws.numel() < need:
                self.ws = torch.empty(need, dtype=torch.float32, device="cuda")
            ws = self.ws
        L.call("ds_gemm_bf16_tn", A.data_ptr(), A.stride(0), B.data_ptr(), B.stride(0), M, N, K,
               epilogue, _p(D), ldd, _p(Y), _p(Z), ldy, _p(bias), splits, _p(ws),
               self.err.data_ptr(), _s())
        return (Z, Y) if epilogue == EPI_BIAS_GELU else D

    def check(self):
        if int(self.err.item()) != 0:
            raise RuntimeError("tensor-core GEMM pipeline wait timed out")

    def clear(self):
        self.err.zero_()


def set_spin_limit(polls: int = 0) -> None:
    """Polls per pipeline wait of the GEMM before it reports a timeout
    (0: the default).  Lowered only to test the timeout path."""
    L.call("ds_gemm_set_spin_limit", polls)


def kpad(c_in: int) -> int:
    """im2col width: 9 * c_in rounded up to 64 (one 128-byte K block)."""
    return (9 * c_in + 63) // 64 * 64


def im2col(x, stride, kp=None):
    B, H, W, Cin = x.shape
    kp = kp or kpad(Cin)
    Ho, Wo = (H - 1) // stride + 1, (W - 1) // stride + 1
    col = torch.empty(B * Ho * Wo, kp, dtype=torch.bfloat16, device="cuda")
    L.call("ds_im2col_bf16", x.data_ptr(), B, H, W, Cin, stride, kp, col.data_ptr(), _s())
    return col, (B, Ho, Wo)


def col2im(dcol, shape, stride, z=None):
    B, H, W, Cin = shape
    dx = torch.empty(B, H, W, Cin, dtype=torch.bfloat16, device="cuda")
    L.call("ds_col2im_bf16", dcol.data_ptr(), B, H, W, Cin, stride, dcol.shape[1], _p(z),
           dx.data_ptr(), _s())
    return dx


def transpose(a):
    r, c = a.shape
    out = torch.empty(c, r, dtype=torch.bfloat16, device="cuda")
    L.call("ds_transpose_bf16", a.data_ptr(), r, c, out.data_ptr(), _s())
    return out


def colsum(a):
    M, Cn = a.shape
    parts = 148 * 4
    ws = torch.empty(parts * Cn, dtype=torch.float32, device="cuda")
    out = torch.empty(Cn, dtype=torch.float32, device="cuda")
    L.call("ds_colsum_bf16", a.data_ptr(), M, Cn, ws.data_ptr(), parts, out.data_ptr(), _s())
    return out


def cast_bf16(x):
    out = torch.empty(x.shape, dtype=torch.bfloat16, device="cuda")
    L.call("ds_cast_bf16", x.contiguous().data_ptr(), x.numel(), out.data_ptr(), _s())
    return out


class AdamW:
    def __init__(self, params, lr=3e-4, betas=(0.9, 0.999), eps=1e-8, weight_decay=1e-2):
        self.params = params  # [(fp32 master, fp32 grad, bf16 copy or None)]
        self.m = [torch.zeros_like(p) for p, _, _ in params]
        self.v = [torch.zeros_like(p) for p, _, _ in params]
        self.lr, self.betas, self.eps, self.wd = lr, betas, eps, weight_decay
        self.t = 0

    def step(self):
        self.t += 1
        for (p, g, copy), m, v in zip(self.params, self.m, self.v):
            L.call("ds_adamw", p.data_ptr(), g.data_ptr(), m.data_ptr(), v.data_ptr(), p.numel(),
                   C.c_float(self.lr), C.c_float(self.betas[0]), C.c_float(self.betas[1]),
                   C.c_float(self.eps), C.c_float(self.wd), self.t, _p(copy), _s())


class Conv3x3:
    """3x3 convolution, padding 1, stride 1 or 2, NHWC BF16, weights [Cout,
    Kp] with k = (ky * 3 + kx) * Cin + c (FP32 master + BF16 copy)."""

    def __init__(self, cin, cout, stride=1, gelu=True, gen=None):
        self.cin, self.cout, self.stride, self.gelu = cin, cout, stride, gelu
        self.kp = kpad(cin)
        std = math.sqrt(2.0 / (9 * cin))
        w = torch.zeros(cout, self.kp, dtype=torch.float32)
        w[:, :9 * cin] = torch.randn(cout, 9 * cin, generator=gen) * std
        self.w = w.cuda()
        self.b = torch.zeros(cout, dtype=torch.float32, device="cuda")
        self.w16 = self.w.to(torch.bfloat16)
        self.gw = torch.zeros_like(self.w)
        self.gb = torch.zeros_like(self.b)

    def params(self):
        return [(self.w, self.gw, self.w16), (self.b, self.gb, None)]

    def forward(self, gemm, x):
        """x [B, H, W, Cin] BF16 -> (z, y) [B, Ho, Wo, Cout] (y = gelu(z) BF16, or
        z only as FP32 when the layer has no GELU)."""
        col, (B, Ho, Wo) = im2col(x, self.stride, self.kp)
        self.col, self.in_shape = col, tuple(x.shape)
        if self.gelu:
            z, y = gemm(col, self.w16, EPI_BIAS_GELU, bias=self.b)
            return z.view(B, Ho, Wo, self.cout), y.view(B, Ho, Wo, self.cout)
        d = gemm(col, self.w16, EPI_BIAS_F32, bias=self.b)
        return d.view(B, Ho, Wo, self.cout), None

    def backward(self, gemm, dz, z_prev=None, need_dx=True):
        """dz [B, Ho, Wo, Cout] BF16 (gradient of this layer's pre-activation) ->
        weight/bias gradients (stored) and the gradient of the previous layer's
        pre-activation (times gelu'(z_prev)) or of the input."""
        M = dz.numel() // self.cout
        dz2 = dz.reshape(M, self.cout)
        self.gb.copy_(colsum(dz2))
        dzt = transpose(dz2)              # [Cout, M]
        colt = transpose(self.col)        # [Kp, M]
        splits = max(1, min(64, M // 4096))
        gemm(dzt, colt, EPI_F32, D=self.gw, splits=splits)
        if not need_dx:
            return None
        wt = transpose(self.w16)          # [Kp, Cout]
        dcol = gemm(dz2, wt, EPI_F32)     # [M, Kp]
        return col2im(dcol, self.in_shape, self.stride, z_prev)
