"""GPU tests of the tcgen05 BF16 GEMM and the convolution kernels of the
learned initializer against plain PyTorch FP32 references of the same ops
(BF16 inputs widened to FP32; tolerance 2e-3 relative for GEMMs, which sum
BF16 products in FP32, and 2e-2 where a result is stored as BF16)."""
import pytest

pytestmark = pytest.mark.gpu


def _rel(a, b):
    a, b = a.detach().float(), b.detach().float()
    return float((a - b).norm() / b.norm().clamp_min(1e-12))


@pytest.mark.parametrize("M,N,K,splits", [(256, 64, 128, 1), (300, 40, 104, 1), (128, 256, 1024, 1),
                                          (640, 130, 320, 1), (512, 32, 64, 1),
                                          (256, 96, 4096, 4), (1000, 200, 576, 3)])
def test_gemm_matches_fp32(cuda_lib, M, N, K, splits):
    import torch
    from diffsplat_b200 import nn
    g = torch.Generator().manual_seed(M * 7 + N)
    A = torch.randn(M, K, generator=g).to(torch.bfloat16).cuda()
    B = torch.randn(N, K, generator=g).to(torch.bfloat16).cuda()
    gemm = nn.Gemm()
    D = gemm(A, B, splits=splits)
    torch.cuda.synchronize()
    gemm.check()
    ref = A.float() @ B.float().T
    assert _rel(D, ref) < 2e-3


def test_gemm_bias_gelu_epilogue(cuda_lib):
    import torch
    from diffsplat_b200 import nn
    g = torch.Generator().manual_seed(3)
    A = torch.randn(384, 192, generator=g).to(torch.bfloat16).cuda()
    B = (0.1 * torch.randn(64, 192, generator=g)).to(torch.bfloat16).cuda()
    bias = torch.randn(64, generator=g).cuda()
    gemm = nn.Gemm()
    z, y = gemm(A, B, nn.EPI_BIAS_GELU, bias=bias)
    zf = gemm(A, B, nn.EPI_BIAS_F32, bias=bias)
    torch.cuda.synchronize()
    gemm.check()
    zr = A.float() @ B.float().T + bias
    assert _rel(zf, zr) < 2e-3
    assert _rel(z, zr) < 1e-2
    assert _rel(y, torch.nn.functional.gelu(zr, approximate="tanh")) < 1e-2


@pytest.mark.parametrize("cin,cout,stride,H", [(3, 32, 1, 40), (32, 64, 2, 34), (64, 128, 2, 16),
                                               (128, 256, 1, 8)])
def test_conv_forward_backward_matches_fp32(cuda_lib, cin, cout, stride, H):
    import torch
    import torch.nn.functional as F
    from diffsplat_b200 import nn
    gen = torch.Generator().manual_seed(cin + cout)
    B, W = 2, H + 6
    conv = nn.Conv3x3(cin, cout, stride, gelu=True, gen=gen)
    x = torch.randn(B, H, W, cin, generator=gen).to(torch.bfloat16).cuda()
    zprev = torch.randn(B, H, W, cin, generator=gen).to(torch.bfloat16).cuda()
    gemm = nn.Gemm()
    z, y = conv.forward(gemm, x)
    # FP32 reference with the same BF16 inputs and weights
    w4 = conv.w16.float()[:, :9 * cin].view(cout, 3, 3, cin).permute(0, 3, 1, 2).contiguous()
    xr = x.float().permute(0, 3, 1, 2).requires_grad_(True)
    wr = w4.clone().requires_grad_(True)
    br = conv.b.clone().requires_grad_(True)
    zr = F.conv2d(xr, wr, br, stride=stride, padding=1)
    assert _rel(z.permute(0, 3, 1, 2), zr) < 1e-2
    assert _rel(y.permute(0, 3, 1, 2), F.gelu(zr, approximate="tanh")) < 1e-2
    dz = torch.randn(z.shape, generator=gen).to(torch.bfloat16).cuda()
    dx = conv.backward(gemm, dz, z_prev=zprev)
    torch.cuda.synchronize()
    gemm.check()
    zr.backward(dz.float().permute(0, 3, 1, 2))
    gw = conv.gw[:, :9 * cin].view(cout, 3, 3, cin).permute(0, 3, 1, 2)
    assert _rel(gw, wr.grad) < 2e-3
    assert _rel(conv.gb, br.grad) < 2e-3
    zp = zprev.float().permute(0, 3, 1, 2).requires_grad_(True)
    gref = torch.autograd.grad(F.gelu(zp, approximate="tanh"), zp, xr.grad)[0]
    assert _rel(dx.permute(0, 3, 1, 2), gref) < 1e-2
    assert (conv.gw[:, 9 * cin:] == 0).all()


def test_pipeline_wait_timeout_is_reported_and_device_stays_usable(cuda_lib):
    """Failure detection without a GPU fault: with the pipeline waits limited
    to one poll, the TMA copies cannot land in time, so the CTAs give up,
    let what they issued land, free their TMEM and set the error word that
    Gemm.check() turns into an exception.  The next GEMM with the default
    limit on the same context is correct."""
    import torch
    from diffsplat_b200 import nn
    g = torch.Generator().manual_seed(11)
    A = torch.randn(2048, 1152, generator=g).to(torch.bfloat16).cuda()
    B = torch.randn(256, 1152, generator=g).to(torch.bfloat16).cuda()
    gemm = nn.Gemm()
    nn.set_spin_limit(1)
    try:
        gemm(A, B)
        torch.cuda.synchronize()
    finally:
        nn.set_spin_limit(0)
    with pytest.raises(RuntimeError, match="timed out"):
        gemm.check()
    gemm.clear()
    D = gemm(A, B)
    torch.cuda.synchronize()
    gemm.check()
    assert _rel(D, A.float() @ B.float().T) < 2e-3
