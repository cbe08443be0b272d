"""Seeded procedural workloads (no dataset is involved).

Targets: a linear colour gradient, plus random 2D Gaussian blobs (centres
uniform, sigma uniform in [2, 40] px, colours uniform), plus an 8-px
checkerboard of amplitude 0.1, clamped, quantised to uint8 and divided by 255
(the reference's image convention, src/io/image_io.cpp:64-66).

Splat init (pinhole camera at the origin looking +z): depth z ~ U[2, 6], pixel
(u, v) ~ U[0, W) x U[0, H), x = (u - cx) z / fx, y = (v - cy) z / fy;
log-scales ~ N(-3, 0.5); quaternion = normalise(N(0,1)^4); opacity logit 0;
SH-DC = (U[0,1] - 0.5) / SH_C0 (the reference's random colour init,
src/utils/splat_utils.h:39-42).

Draw order per seed (numpy PCG64): target blobs (centres, sigmas, colours),
then splats (z, u, v, log-scales, quaternions, colours).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

SH_C0 = 0.28209479177387814


def sh_bands(degree: int) -> int:
    return sum(2 * l + 1 for l in range(1, degree + 1))


def make_target(width: int, height: int, blobs: int, seed: int) -> np.ndarray:
    """Returns float32 [H, W, 3] in [0, 1], quantised to 1/255 steps."""
    rng = np.random.Generator(np.random.PCG64(seed))
    cx = rng.uniform(0, width, blobs)
    cy = rng.uniform(0, height, blobs)
    sg = rng.uniform(2.0, 40.0, blobs)
    col = rng.uniform(0.0, 1.0, (blobs, 3))
    u = np.arange(width, dtype=np.float64)[None, :] + 0.5
    v = np.arange(height, dtype=np.float64)[:, None] + 0.5
    img = np.empty((height, width, 3), np.float64)
    img[..., 0] = 0.15 + 0.5 * u / width
    img[..., 1] = 0.15 + 0.5 * v / height
    img[..., 2] = 0.65 - 0.25 * (u / width + v / height)
    acc = np.zeros((height, width, 3), np.float64)
    for k in range(blobs):
        r = 3.0 * sg[k]
        x0, x1 = max(int(cx[k] - r), 0), min(int(cx[k] + r) + 1, width)
        y0, y1 = max(int(cy[k] - r), 0), min(int(cy[k] + r) + 1, height)
        if x0 >= x1 or y0 >= y1:
            continue
        du = u[:, x0:x1] - cx[k]
        dv = v[y0:y1, :] - cy[k]
        g = np.exp(-(du * du + dv * dv) / (2.0 * sg[k] * sg[k]))
        acc[y0:y1, x0:x1, :] += 0.5 * g[..., None] * (col[k] - 0.5)[None, None, :]
    img += acc
    checker = ((np.floor(u / 8.0) + np.floor(v / 8.0)) % 2.0)
    img += (0.1 * checker - 0.05)[..., None]
    img = np.clip(img, 0.0, 1.0)
    q = np.round(img * 255.0).astype(np.uint8)
    return (q.astype(np.float32) / np.float32(255.0))


def pinhole_pv(width: int, height: int, fx: float, fy: float, cx: float, cy: float,
               near: float = 0.01, far: float = 100.0) -> np.ndarray:
    """Column-major 16-float PV of a pinhole camera at the origin looking +z,
    y down in pixels / up in NDC (clip_w = z)."""
    M = np.array([
        [2 * fx / width, 0, 2 * cx / width - 1, 0],
        [0, -2 * fy / height, 1 - 2 * cy / height, 0],
        [0, 0, (far + near) / (far - near), -2 * far * near / (far - near)],
        [0, 0, 1, 0]], dtype=np.float64)
    return M.T.reshape(-1).astype(np.float32)  # column-major


def look_at_perspective_pv(eye, center, up, fovy: float, aspect: float, near: float,
                           far: float) -> np.ndarray:
    """Column-major PV = perspective * lookAt (OpenGL conventions, float32)."""
    eye = np.asarray(eye, np.float32)
    center = np.asarray(center, np.float32)
    up = np.asarray(up, np.float32)
    f = center - eye
    f = f / np.float32(np.sqrt(np.dot(f, f)))
    s = np.cross(f, up)
    s = s / np.float32(np.sqrt(np.dot(s, s)))
    u = np.cross(s, f)
    V = np.eye(4, dtype=np.float32)
    V[0, :3] = s
    V[1, :3] = u
    V[2, :3] = -f
    V[0, 3] = -np.dot(s, eye)
    V[1, 3] = -np.dot(u, eye)
    V[2, 3] = np.dot(f, eye)
    th = np.float32(math.tan(fovy / 2.0))
    P = np.zeros((4, 4), np.float32)
    P[0, 0] = 1.0 / (aspect * th)
    P[1, 1] = 1.0 / th
    P[2, 2] = -(far + near) / (far - near)
    P[3, 2] = -1.0
    P[2, 3] = -(2.0 * far * near) / (far - near)
    return (P @ V).T.reshape(-1).astype(np.float32)


def random_splats(n: int, width: int, height: int, fx: float, fy: float, cx: float, cy: float,
                  seed: int, sh_degree: int = 0, log_scale_mean: float = -3.0,
                  log_scale_std: float = 0.5, zmin: float = 2.0, zmax: float = 6.0,
                  rng: np.random.Generator | None = None) -> np.ndarray:
    """Field-major float32 [14 + 3K, n]: pos xyz, log-scale xyz, quat wxyz,
    sh_dc rgb, logit, sh_rest r (K rows), g, b."""
    if rng is None:
        rng = np.random.Generator(np.random.PCG64(seed))
    K = sh_bands(sh_degree)
    P = np.zeros((14 + 3 * K, n), np.float32)
    z = rng.uniform(zmin, zmax, n)
    u = rng.uniform(0, width, n)
    v = rng.uniform(0, height, n)
    P[0] = (u - cx) * z / fx
    P[1] = (v - cy) * z / fy
    P[2] = z
    P[3:6] = rng.normal(log_scale_mean, log_scale_std, (3, n))
    q = rng.normal(0.0, 1.0, (4, n))
    q /= np.linalg.norm(q, axis=0, keepdims=True)
    P[6:10] = q
    P[10:13] = (rng.uniform(0.0, 1.0, (3, n)) - 0.5) / SH_C0
    P[13] = 0.0
    return P


@dataclass
class FitProblem:
    width: int
    height: int
    params: np.ndarray  # [14 + 3K, n] float32
    target: np.ndarray  # [H, W, 3] float32
    pv: np.ndarray      # [16] float32 column-major
    cam: np.ndarray     # [3] float32
    sh_degree: int
    lrs: tuple          # pos, scale, rot, sh_dc, sh_rest, opacity


# Learning rates: Gaussian3DAdamConfig defaults (src/optimizers/gaussian3d_adam.h:11-19).
REFERENCE_LRS = (1.6e-2, 1.0e-3, 6.0e-4, 6.0e-3, 6.0e-3, 6.0e-3)
PLAIN_SMALL_LRS = (1e-3, 1e-3, 6.0e-4, 5e-2, 5e-2, 5e-2)


def plain_small(seed: int = 0) -> FitProblem:
    """256x256, 200 blobs, 4096 splats, fx = fy = 256, c = 128, SH 0."""
    W = H = 256
    tgt = make_target(W, H, 200, seed)
    P = random_splats(4096, W, H, 256.0, 256.0, 128.0, 128.0, seed + 1)
    return FitProblem(W, H, P, tgt, pinhole_pv(W, H, 256.0, 256.0, 128.0, 128.0),
                      np.zeros(3, np.float32), 0, PLAIN_SMALL_LRS)


def reference_default(seed: int = 0) -> FitProblem:
    """1280x720, 2000 blobs, 60000 splats, fx = fy = 1000, c = (640, 360), SH 0."""
    W, H = 1280, 720
    tgt = make_target(W, H, 2000, seed)
    P = random_splats(60000, W, H, 1000.0, 1000.0, 640.0, 360.0, seed + 1)
    return FitProblem(W, H, P, tgt, pinhole_pv(W, H, 1000.0, 1000.0, 640.0, 360.0),
                      np.zeros(3, np.float32), 0, REFERENCE_LRS)


def small_problem(width: int, height: int, n: int, seed: int, sh_degree: int = 0,
                  blobs: int = 20, log_scale_mean: float = -3.0) -> FitProblem:
    """Scaled-down variant of the plain fitter for parity tests."""
    f = float(max(width, height))
    tgt = make_target(width, height, blobs, seed)
    rng = np.random.Generator(np.random.PCG64(seed + 7))
    P = random_splats(n, width, height, f, f, width / 2, height / 2, seed, sh_degree,
                      log_scale_mean=log_scale_mean, rng=rng)
    K = sh_bands(sh_degree)
    if K:
        P[14:] = rng.normal(0.0, 0.3, (3 * K, n)).astype(np.float32)
    P[13] = rng.normal(0.0, 1.0, n).astype(np.float32)
    cam = np.array([0.05, -0.03, -0.2], np.float32)
    return FitProblem(width, height, P, tgt, pinhole_pv(width, height, f, f, width / 2, height / 2),
                      cam, sh_degree, PLAIN_SMALL_LRS)


def psnr_from_ref_loss(loss: float) -> float:
    """PSNR of the per-element MSE; the reference loss divides by pixels, not
    pixels x 3 (src/layers/mse_loss_layer.cu:31)."""
    mse = max(loss / 3.0, 1e-20)
    return 10.0 * math.log10(1.0 / mse)


def viewer_scene(n: int = 1_000_000, seed: int = 0, surfaces: int = 20,
                 sh_degree: int = 3) -> np.ndarray:
    """Viewer-style scene: means on `surfaces` random planes and spheres inside a
    radius-10 ball with sigma = 0.02 jitter, log-scales ~N(-4.5, 0.7), opacity
    logits ~N(0, 1.5), SH DC ~N(0, 0.5), higher bands ~N(0, 0.05), random
    rotations.  Field-major float32 [14 + 3K, n]."""
    rng = np.random.Generator(np.random.PCG64(seed))
    K = sh_bands(sh_degree)
    P = np.zeros((14 + 3 * K, n), np.float32)
    which = rng.integers(0, surfaces, n)
    pos = np.zeros((n, 3))
    for s in range(surfaces):
        idx = np.nonzero(which == s)[0]
        m = idx.size
        c = rng.normal(size=3)
        c = c / np.linalg.norm(c) * rng.uniform(0.0, 6.0)
        if s % 2 == 0:  # plane patch through c
            nrm = rng.normal(size=3)
            nrm /= np.linalg.norm(nrm)
            a = np.cross(nrm, [1.0, 0.0, 0.0] if abs(nrm[0]) < 0.9 else [0.0, 1.0, 0.0])
            a /= np.linalg.norm(a)
            b = np.cross(nrm, a)
            half = rng.uniform(1.0, 4.0)
            uv = rng.uniform(-half, half, (m, 2))
            pts = c + uv[:, :1] * a + uv[:, 1:] * b
        else:  # sphere around c
            r = rng.uniform(0.5, 3.0)
            d = rng.normal(size=(m, 3))
            d /= np.linalg.norm(d, axis=1, keepdims=True)
            pts = c + r * d
        pts = pts + rng.normal(0.0, 0.02, (m, 3))
        nrmp = np.linalg.norm(pts, axis=1, keepdims=True)
        pts = np.where(nrmp > 10.0, pts / nrmp * 10.0, pts)
        pos[idx] = pts
    P[0:3] = pos.T
    P[3:6] = rng.normal(-4.5, 0.7, (3, n))
    q = rng.normal(0.0, 1.0, (4, n))
    P[6:10] = q / np.linalg.norm(q, axis=0, keepdims=True)
    P[10:13] = rng.normal(0.0, 0.5, (3, n))
    P[13] = rng.normal(0.0, 1.5, n)
    if K:
        P[14:] = rng.normal(0.0, 0.05, (3 * K, n))
    return P


def orbit_cameras(count: int = 16, radius: float = 15.0, width: int = 1920, height: int = 1080,
                  fx: float = 1200.0, near: float = 0.1, far: float = 100.0):
    """`count` cameras on a horizontal circle of `radius` looking at the origin
    (GL lookAt + perspective, fovy = 2 atan(height / 2 / fx)): [(pv, eye)]."""
    fovy = 2.0 * math.atan(height / 2.0 / fx)
    cams = []
    for k in range(count):
        a = 2.0 * math.pi * k / count
        eye = np.array([radius * math.cos(a), 2.0, radius * math.sin(a)], np.float32)
        pv = look_at_perspective_pv(eye, [0.0, 0.0, 0.0], [0.0, 1.0, 0.0], fovy, width / height,
                                    near, far)
        cams.append((pv, eye))
    return cams


BATCH_SIZES = [(128, 128), (256, 256), (512, 512), (640, 480), (1024, 768)]


def batch_problems(count: int = 64, seed: int = 0, nmin: int = 2000,
                   nmax: int = 200_000) -> list:
    """Uneven fitting instances built like the small plain fitter, each from its
    own seed: image size drawn from BATCH_SIZES, splat count log-uniform in
    [nmin, nmax], pinhole camera with fx = fy = width and a centred principal
    point, procedural target with 200 blobs per 256x256 of area (at least 100)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    probs = []
    for k in range(count):
        W, H = BATCH_SIZES[int(rng.integers(0, len(BATCH_SIZES)))]
        n = int(round(math.exp(rng.uniform(math.log(nmin), math.log(nmax)))))
        s = seed * 100_003 + k
        blobs = max(100, int(200 * W * H / (256 * 256)))
        f = float(W)
        probs.append(FitProblem(W, H, random_splats(n, W, H, f, f, W / 2, H / 2, s + 1),
                                make_target(W, H, blobs, s), pinhole_pv(W, H, f, f, W / 2, H / 2),
                                np.zeros(3, np.float32), 0, PLAIN_SMALL_LRS))
    return probs
