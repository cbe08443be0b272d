"""GPU tests of the learned initializer: its head output and every weight and
bias gradient against the FP64 CPU oracle of the same network
(oracle/initializer_oracle.py, BF16 weights, FP64 arithmetic; tolerances 3e-2
relative for the BF16-activation forward, 5e-2 for gradients), the head
decode, and that training lowers both loss terms."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rel(a, b):
    a = np.asarray(a, np.float64).reshape(-1)
    b = np.asarray(b, np.float64).reshape(-1)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def _net(size=64, seed=0):
    import torch
    from diffsplat_b200.initializer import Initializer
    init = Initializer(size=size, seed=seed)
    g = torch.Generator().manual_seed(seed + 1)
    w = torch.randn(init.head.w.shape, generator=g) * 0.02
    w[:, 9 * init.head.cin:] = 0
    init.head.w.copy_(w)
    init.head.w16.copy_(w.to(torch.bfloat16))
    for m in init.modules():
        m.b.copy_(torch.randn(m.b.shape, generator=g) * 0.05)
    return init


def test_head_decode_matches_oracle(cuda_lib):
    import torch
    from oracle import initializer_oracle as IO
    init = _net()
    out = torch.randn(2 * init.grid * init.grid, 56, device="cuda")
    mine = init.decode(out).cpu().numpy()
    ref = IO.decode(init, out.cpu().double()).numpy()
    assert np.abs(mine - ref).max() < 1e-5


def test_gradients_match_cpu_oracle(cuda_lib):
    import torch
    from oracle import initializer_oracle as IO
    init = _net()
    g = torch.Generator().manual_seed(5)
    imgs = torch.rand(2, 64, 64, 3, generator=g).cuda()
    out = init.forward(imgs)
    params = init.decode(out)
    sgn = torch.where(torch.rand(params.shape, generator=g) < 0.5, -1.0, 1.0).cuda()
    target = params - 0.5 * sgn
    init.backward(params, target=target, w_l1=1.0)
    torch.cuda.synchronize()
    init.gemm.check()
    out64, weights = IO.forward(init, imgs)
    assert _rel(out.cpu().numpy(), out64.detach().numpy()) < 3e-2
    p64 = IO.decode(init, out64)
    (p64 - target.cpu().double()).abs().sum().backward()
    for k, (m, (w, b)) in enumerate(zip(init.modules(), weights)):
        gw = m.gw[:, :9 * m.cin].view(m.cout, 3, 3, m.cin).permute(0, 3, 1, 2)
        assert _rel(gw.cpu().numpy(), w.grad.numpy()) < 5e-2, f"layer {k} weights"
        assert _rel(m.gb.cpu().numpy(), b.grad.numpy()) < 5e-2, f"layer {k} bias"


def test_training_lowers_both_losses(cuda_lib):
    from diffsplat_b200 import initializer as I
    init = I.Initializer(size=64, seed=3)
    targets = I.make_targets(16, size=64, seed=3)
    fitted = I.fit_pairs(init, targets, steps=60, batch=16)
    hist = I.train(init, targets, fitted, steps=60, batch=8, lr=1e-3, log_every=59)
    (_, l1a, ra), (_, l1b, rb) = hist[0], hist[-1]
    assert l1b < l1a and rb < ra, hist
