"""Generates tests/golden/*.npz from the reference's own CUDA layers
(oracle/_ref/libdsref.so, built from the reference sources by oracle/Makefile).
Needs a GPU; run from the repository root:

    python tests/golden/make_golden.py

Each fixture holds the inputs (params, target, camera) and the reference's
outputs of one ImageFitter-style pass: Splat3D, Splat2D, sorted keys / ids
(equal keys canonicalised by id), tile ranges, image, loss, the Splat2D /
Splat3D / Gaussian3D gradients, and the parameters after one Adam step.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from diffsplat_b200.scenes import FitProblem, small_problem  # noqa: E402
from oracle import ref  # noqa: E402

OUT = Path(__file__).resolve().parent


def grad_check_problem() -> FitProblem:
    """tests/grad_check.cu:72-132: 8 splats, 32x32, orthographic camera."""
    n, W, H = 8, 32, 32
    P = np.zeros((14, n), np.float32)
    for i in range(n):
        P[0, i] = (i % 4) * 4.0 - 6.0
        P[1, i] = (i // 4) * 6.0 - 3.0
        P[2, i] = i * 0.1
        P[3:6, i] = [1.2, 0.8, 0.5]
        P[6:10, i] = [0.991, 0.0, 0.0, 0.131]
        P[13, i] = 2.0
    hw, hh = np.float32(W * 0.5), np.float32(H * 0.5)
    zr = np.float32(min(hw, hh) * np.float32(0.25))
    M = np.zeros((4, 4), np.float32)
    M[0, 0] = np.float32(2) / (hw - (-hw))
    M[1, 1] = np.float32(2) / (hh - (-hh))
    M[2, 2] = np.float32(-2) / (zr - (-zr))
    M[0, 3] = -(hw + (-hw)) / (hw - (-hw))
    M[1, 3] = -(hh + (-hh)) / (hh - (-hh))
    M[2, 3] = -(zr + (-zr)) / (zr - (-zr))
    M[3, 3] = 1
    tgt = np.full((H, W, 3), 0.7, np.float32)
    return FitProblem(W, H, P, tgt, M.T.reshape(-1).copy(), np.array([0, 0, 5], np.float32), 0,
                      (1.6e-2, 1e-3, 6e-4, 6e-3, 6e-3, 6e-3))


PROBLEMS = {
    "grad_check_8": grad_check_problem,
    "persp_sh0_48x32": lambda: small_problem(48, 32, 24, seed=40, sh_degree=0, log_scale_mean=-2.3),
    "persp_sh1_64x40": lambda: small_problem(64, 40, 60, seed=41, sh_degree=1, log_scale_mean=-2.5),
    "persp_sh3_80x48": lambda: small_problem(80, 48, 90, seed=42, sh_degree=3, log_scale_mean=-2.6),
}


def main() -> None:
    for name, make in PROBLEMS.items():
        prob = make()
        R = ref.RefScene(prob.width, prob.height, prob.params, prob.sh_degree, prob.target,
                         prob.pv, prob.cam, prob.lrs)
        R.zero_grad()
        R.forward()
        loss = R.loss()
        R.backward()
        keys, ids = ref.canonical_order(R.download(0), R.download(1))
        out = dict(params=prob.params, target=prob.target, pv=prob.pv, cam=prob.cam,
                   lrs=np.asarray(prob.lrs, np.float32),
                   meta=np.array([prob.width, prob.height, prob.sh_degree], np.int32),
                   S3=R.download(10), S2=R.download(8), keys=keys, ids=ids,
                   ranges=R.download(2), image=R.download(3), alphas=R.download(4),
                   last_ids=R.download(5), loss=np.float32(loss), G2=R.download(9),
                   G3=R.download(11), GP=R.download(6))
        R.adam_step()
        out["params_after_adam"] = R.download(7)
        R.close()
        np.savez_compressed(OUT / f"{name}.npz", **out)
        print(name, "pairs", len(keys), "loss", loss)


if __name__ == "__main__":
    main()
