"""GPU tests of the learned initializer: its head output and every weight and
bias gradient against the FP64 CPU oracle of the same network
(oracle/initializer_oracle.py, BF16 weights, FP64 arithmetic; tolerances 3e-2
relative for the BF16-activation forward, 5e-2 for gradients), the head
decode, that training lowers both loss terms, what the trained network gains
over the fitter without it, and the fallback to random init."""
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


@pytest.fixture(scope="module")
def trained_128(cuda_lib):
    """A 128 x 128 initializer (16 x 16 grid, 1024 splats) trained on 96
    targets whose splats the batched fitter fitted for 300 steps; 4 further
    targets held out."""
    from diffsplat_b200 import initializer as I
    init = I.Initializer(size=128, seed=0)
    targets = I.make_targets(100, size=128, seed=21)
    fitted = I.fit_pairs(init, targets[:96], steps=300, batch=32)
    I.train(init, targets[:96], fitted, steps=300, batch=16, lr=1e-3)
    return init, targets[96:]


def test_learned_init_reaches_the_goal_sooner_than_random_and_grid(trained_128):
    """What the trained network gains over the method without it: on held-out
    targets the learned init reaches 24 dB in fewer fitter steps and fewer
    device seconds (network forward included) than the plain fitter's random
    init and than the grid init (the zero-head output: the same fitter and
    splat layout without the network), and needs no fallback."""
    from diffsplat_b200 import initializer as I
    init, held = trained_128
    ev = I.evaluate(init, held, goal=24.0, max_steps=600)
    assert ev["fallbacks"] == 0
    assert ev["learned_reached"] == len(held)
    assert ev["learned_steps"] < ev["grid_steps"] < ev["random_steps"], ev
    assert ev["learned_seconds"] < ev["grid_seconds"], ev
    assert ev["learned_seconds"] < ev["random_seconds"], ev


def test_fallback_to_random_when_the_prediction_is_worse(cuda_lib):
    """A prediction that renders worse than random init is not used:
    evaluate() falls back to the random init, which then is the learned row.
    The prediction here puts every splat behind the camera, so its image
    stays black, on bright targets (black is 0.7 and 1.4 dB from them)."""
    import numpy as np
    from diffsplat_b200 import initializer as I
    init = I.Initializer(size=64, seed=4)
    bad = init.zero_params(1)
    bad[2] = -4.0  # z < 0: every splat culled
    init.predict = lambda image: bad
    targets = np.stack([I.make_targets(2, size=64, seed=5)[0],
                        I.make_targets(2, size=64, seed=6)[0]])
    ev = I.evaluate(init, targets, goal=22.0, max_steps=100)
    assert ev["fallbacks"] == 2, ev
    assert ev["learned_steps"] == ev["random_steps"]
    assert ev["learned_psnr_first"] == ev["random_psnr_first"]
