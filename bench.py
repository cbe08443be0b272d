"""Benchmark: fwd+bwd+Adam training steps/s of the reference-default fitter
(1280x720 procedural target, 60000 splats, SH degree 0, 16x16 tiles, L2 loss,
Adam) on one B200, through the fused graph-captured step of libdiffsplat_b200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One process per GPU (torchrun for N > 1); every rank fits its own independent
instance (replicas: the path has no data exchange), so scaling is weak and the
job value is the sum over ranks of steps / max-over-ranks time.
L2 hygiene: a 256 MiB buffer is overwritten between timed steps, outside the
timed events, so every step starts with a cold 126 MB L2.
End to end (`e2e`): a second fitter on the same trajectory, stepped through the
public API with, every step, the camera uploaded from pinned host memory and
the loss copied to a pinned host slot and read by the host (step k's loss is
read once step k + 1 is enqueued).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "fwd+bwd+Adam steps/s (reference-default fitter, 1280x720, 60000 splats)"
FLUSH_BYTES = 256 << 20


class ClockSampler:
    """Samples SM clocks and throttle reasons with nvidia-smi while running."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.rows: list[list[str]] = []
        self._stop = threading.Event()
        self._t = threading.Thread(target=self._run, daemon=True)

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(
                    ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                     "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                if out.returncode == 0 and out.stdout.strip():
                    self.rows.append([x.strip() for x in out.stdout.strip().split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self) -> dict:
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows for k in range(4)
                          if len(r) > 3 + k and r[3 + k].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.rows)}


def dist_setup(gpus: int):
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(0)
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(world, value: float, device: str = "cuda") -> float:
    """The largest `value` over the ranks (the process group's backend must
    reduce tensors on `device`: NCCL on "cuda", gloo on "cpu")."""
    if world == 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def measured_peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return {"hbm_gbs": d.get("hbm_gbs", 6650.0), "sm_max_mhz": d.get("sm_max_mhz", 1965.0),
                "src": "measured"}
    return {"hbm_gbs": 6650.0, "sm_max_mhz": 1965.0, "src": "fallback"}


def fp32_peak_tflops(sm_mhz: float) -> float:
    """Non-tensor FP32 peak: SMs x 128 lanes x 2 (FMA) x SM clock."""
    import torch
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    return sms * 128 * 2 * sm_mhz * 1e6 / 1e12


# FP32 operations per contributing (pixel, splat) pair, counted from the kernels'
# per-pixel code (an FMA is 2): forward 24 (+1 exp), backward 70 (+1 exp, 1 rcp).
FLOPS_PER_PAIR = {"composite_fwd": 24, "composite_bwd": 70}

# DRAM bytes (read + write) per (tile, splat) pair of one composite launch, from
# one ncu capture of the same 1280x720 / 60000-splat workload (profile run,
# step 21, 3,085,820 pairs: forward 22.40 MB, backward 59.55 MB), scaled by
# the bench's own pair count.
NCU_DRAM_BYTES_PER_ISECT = {"composite_fwd": 22.396416e6 / 3085820,
                            "composite_bwd": (47.626240e6 + 11.928064e6) / 3085820}


def kernels_per_step(tiles: int) -> int:
    # step_begin, preprocess, 4 depth-sort passes x 3, count scan x 2, emission,
    # tile sort (grids of up to 8192 tiles: count, offsets + ranges, scatter;
    # larger: 3 kernels per radix pass over the tile id, then ranges and the
    # tile schedule), composite forward, composite backward (two launches, one per
    # pixel layout, each taking its own tiles), long-segment reduce,
    # backward + Adam (which sums the short segments itself)
    if tiles <= 8192:
        tile_sort = 3  # the offsets kernel also writes the tile schedule
    else:
        tile_sort = 3 * max(1, (max(1, (tiles - 1).bit_length()) + 7) // 8) + 1 + 1
    return 2 + 12 + 2 + 1 + tile_sort + 1 + 2 + 2


def stage_bytes(n: int, isects: int, pixels: int, bands: int = 0) -> dict:
    """Algorithmic HBM bytes per step of each stage group, by the per-unit
    figures of the path's measurement plan (FP32 storage):
      activation + projection  (14 + 3K) * 4 B read + 40 B written per splat
      tile assign              24 B read per splat + 12 B written per pair
      sort                     24 B per pair (the single-pass lower bound)
      ranges                   8 B per pair
      composite forward        40 B per pair + 20 B per pixel
      composite backward       44 B per pair + 20 B per pixel
      Adam                     28 B per parameter element (p, g, m, v)."""
    elems = 14 + 3 * bands
    return {
        "preprocess": n * (elems * 4 + 40),
        "lists": n * 24 + isects * (12 + 24 + 8),
        "composite_fwd": isects * 40 + pixels * 20,
        "composite_bwd": isects * 44 + pixels * 20,
        "backward_adam": n * elems * 28,
    }


# Stage groups of the fitter's profile step timed against each algorithmic figure.
STAGE_GROUPS = {"preprocess": ("preprocess",),
                "lists": ("depth_sort", "scan_emit", "tile_sort_ranges"),
                "composite_fwd": ("composite_fwd",), "composite_bwd": ("composite_bwd",),
                "backward_adam": ("backward_adam",)}


def cpu_baseline_oracle(prob, budget_s: float = 10.0) -> dict:
    """FP64 oracle: fwd+bwd+Adam steps of the same workload from its initial state
    on all host cores, as many as fit in about budget_s seconds."""
    from oracle import oracle as O
    threads = os.cpu_count() or 1
    P = prob.params.astype(np.float64)
    m, v = np.zeros_like(P), np.zeros_like(P)
    t0 = time.perf_counter()
    steps = 0
    while steps == 0 or time.perf_counter() - t0 < budget_s:
        fw, gp = O.loss_and_grads(P, prob.sh_degree, prob.cam, prob.pv, prob.width, prob.height,
                                  prob.target, threads=threads)
        P, m, v = O.adam_gaussian3d(P, gp, m, v, prob.lrs, steps + 1)
        steps += 1
    dt = time.perf_counter() - t0
    return {"value": steps / dt, "unit": "steps/s", "cores": threads, "kind": "port",
            "sample": f"{steps} fwd+bwd+Adam steps of the same 1280x720 / 60000-splat workload "
                      f"from its initial state ({dt:.1f} s)"}


def run_ours(args, world, rank, local):
    import torch
    from diffsplat_b200 import api
    from diffsplat_b200.scenes import reference_default, psnr_from_ref_loss

    prob = reference_default(seed=rank)
    n = prob.params.shape[1]
    tgt = torch.tensor(prob.target, device="cuda")

    def make():
        f = api.Fitter(prob.width, prob.height, n, prob.sh_degree, lrs=prob.lrs)
        f.set_params(prob.params)
        f.set_target(tgt)
        f.set_camera(prob.pv, prob.cam)
        return f

    # Device-timed arm and end-to-end arm run the same trajectory (same initial
    # state, same warm-up), so both time the same per-step work.
    f, g = make(), make()
    flush = torch.empty(FLUSH_BYTES // 4, device="cuda")
    for _ in range(args.warmup):
        f.step(1)
        g.step(1)
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    barrier(world)
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        for k in range(args.steps):
            flush.fill_(float(k))
            ev[k][0].record()
            f.step(1)
            ev[k][1].record()
        torch.cuda.synchronize()
    barrier(world)
    t_ms = sum(a.elapsed_time(b) for a, b in ev)
    t_max = max_over_ranks(world, t_ms)
    loss = f.loss()
    # end to end through the public API: every step uploads the camera from
    # pinned host memory (H2D) and copies its loss into a pinned host slot
    # (D2H); the host reads step k's loss once step k + 1 is enqueued (two
    # slots), as a training loop that logs every loss without stalling would
    cam_pv = torch.tensor(prob.pv).pin_memory()
    cam_pos = torch.tensor(prob.cam).pin_memory()
    loss_dev = g.loss_device()
    slots = torch.empty(2, dtype=torch.float32).pin_memory()
    copied = [torch.cuda.Event() for _ in range(args.steps)]
    e2e_ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(args.steps)]
    e2e_losses = []
    for k in range(args.steps):
        flush.fill_(float(k))
        e2e_ev[k][0].record()
        g.set_camera(cam_pv.numpy(), cam_pos.numpy())
        g.step(1)
        slots[k % 2:k % 2 + 1].copy_(loss_dev, non_blocking=True)
        copied[k].record()
        e2e_ev[k][1].record()
        if k > 0:
            copied[k - 1].synchronize()
            e2e_losses.append(float(slots[(k - 1) % 2]))
    copied[-1].synchronize()
    e2e_losses.append(float(slots[(args.steps - 1) % 2]))
    assert len(e2e_losses) == args.steps and all(math.isfinite(x) for x in e2e_losses)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(world, sum(a.elapsed_time(b) for a, b in e2e_ev))
    g.close()
    # per-stage device times (eager step with events between stages)
    stages = {s: 0.0 for s in api.Fitter.STAGES}
    reps = 5
    for _ in range(reps):
        flush.fill_(0.0)
        for s, v in f.profile_step().items():
            stages[s] += v / reps
    cnt = f.counters()
    pairs = f.pair_stats()
    code, flags = f.status()
    f.close()
    out = dict(t_ms=t_max, e2e_ms=e2e_ms, loss=loss, psnr=psnr_from_ref_loss(loss),
               stages=stages, counters=cnt, pairs=pairs, clocks=clk.summary(), status=code,
               prob=prob)
    return out


def run_reference(args, world, rank, local):
    import torch
    from oracle import ref
    from diffsplat_b200.scenes import reference_default

    if not ref.available():
        return None, "reference build oracle/_ref/libdsref.so is absent"
    prob = reference_default(seed=rank)
    R = ref.RefScene(prob.width, prob.height, prob.params, prob.sh_degree, prob.target, prob.pv,
                     prob.cam, prob.lrs)
    flush = torch.empty(FLUSH_BYTES // 4, device="cuda")
    for _ in range(args.warmup):
        R.step()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    with ClockSampler(local) as clk:
        for k in range(args.steps):
            flush.fill_(float(k))
            ev[k][0].record()
            R.step()  # the reference runs on the legacy default stream
            ev[k][1].record()
        torch.cuda.synchronize()
    t_ms = sum(a.elapsed_time(b) for a, b in ev)
    loss = R.loss()
    R.close()
    return dict(t_ms=t_ms, loss=loss, clocks=clk.summary()), None


def profile_run(args):
    """Eager (non-graph) steps of the bench workload for profilers: every kernel
    is a separate launch, device memory stays under 1 GB.  With --workload
    viewer-sh3: eager fitter steps of the 1M-splat SH-3 scene at 1920x1080
    from its first orbit camera (about 2 GB)."""
    import torch
    from diffsplat_b200 import api
    from diffsplat_b200.scenes import reference_default
    torch.cuda.set_device(0)
    if args.workload == "viewer-sh3":
        from diffsplat_b200.scenes import make_target, orbit_cameras, viewer_scene
        W, H, n = 1920, 1080, 1_000_000
        f = api.Fitter(W, H, n, 3, max_isects=1 << 23, use_graph=False)
        f.set_params(torch.tensor(viewer_scene(n, seed=0), device="cuda"))
        f.set_target(torch.tensor(make_target(W, H, 2000, 7), device="cuda"))
        f.set_camera(*orbit_cameras(16, width=W, height=H, fx=1200.0)[0])
        f.step(args.warmup + args.steps)
        torch.cuda.synchronize()
        code, _ = f.status()
        print(f"profile run (viewer-sh3): {args.warmup + args.steps} steps, status {code}")
        f.close()
        if code != 0:
            sys.exit(1)
        return
    prob = reference_default(seed=0)
    f = api.Fitter(prob.width, prob.height, prob.params.shape[1], prob.sh_degree, lrs=prob.lrs,
                   max_isects=1 << 22, use_graph=False)
    f.set_params(prob.params)
    f.set_target(torch.tensor(prob.target, device="cuda"))
    f.set_camera(prob.pv, prob.cam)
    f.step(args.warmup + args.steps)
    torch.cuda.synchronize()
    code, flags = f.status()
    cnt = f.counters()
    print(f"profile run: {args.warmup + args.steps} steps, loss {f.loss():.6f}, status {code}, "
          f"pairs of the last step {cnt['n_isects']}")
    f.close()
    if code != 0:
        sys.exit(1)


def run_isects(args) -> dict:
    """(tile, splat) pairs I per splat N of every config, from this build's
    forward (whose pair counts equal the reference's: the parity tests compare
    them bit for bit): c0 and c1 at the fit's initial state and, for c1, after
    25 and 1010 steps; c2 for each of the 16 orbit cameras; c3 per instance at
    its initial state; c4 for random splats on 512^2 targets."""
    import torch
    from diffsplat_b200 import api
    from diffsplat_b200.scenes import (batch_problems, orbit_cameras, plain_small,
                                       reference_default, small_problem, viewer_scene)
    torch.cuda.set_device(0)

    def render_pairs(prob, max_isects=0):
        r = api.Renderer(prob.width, prob.height, prob.params.shape[1], prob.sh_degree,
                         max_isects=max_isects)
        r.set_params(torch.tensor(prob.params, device="cuda").contiguous())
        r.render(prob.pv, prob.cam)
        torch.cuda.synchronize()
        c = r.counts()
        r.close()
        return c

    out = {}
    for name, prob in [("c0 256x256, 4096 splats", plain_small(0)),
                       ("c1 1280x720, 60000 splats", reference_default(0)),
                       ("c4 512x512, 16384 random splats", small_problem(512, 512, 16384, 0))]:
        c = render_pairs(prob)
        n = prob.params.shape[1]
        out[name] = {"N": n, "I": c["n_isects"], "I_per_N": c["n_isects"] / n,
                     "visible": c["visible"]}
    prob = reference_default(0)
    n = prob.params.shape[1]
    f = api.Fitter(prob.width, prob.height, n, prob.sh_degree, lrs=prob.lrs)
    f.set_params(prob.params)
    f.set_target(torch.tensor(prob.target, device="cuda"))
    f.set_camera(prob.pv, prob.cam)
    fit, done = {}, 0
    for k in (25, 1010):
        f.step(k - done)
        done = k
        c = f.counters()
        fit[f"step {k}"] = {"I": c["n_isects"], "I_per_N": c["n_isects"] / n}
    f.close()
    out["c1 1280x720, 60000 splats"]["fit"] = fit
    P = viewer_scene()
    n = P.shape[1]
    r = api.Renderer(1920, 1080, n, 3)
    r.set_params(torch.tensor(P, device="cuda").contiguous())
    per_cam = []
    for pv, eye in orbit_cameras():
        r.render(pv, eye)
        torch.cuda.synchronize()
        per_cam.append(r.counts()["n_isects"])
    r.close()
    out["c2 1920x1080, 1M splats, SH 3"] = {"N": n, "I_per_camera": per_cam,
                                            "I_per_N_mean": float(np.mean(per_cam)) / n}
    inst = []
    for prob in batch_problems():
        c = render_pairs(prob)
        inst.append((prob.width, prob.height, prob.params.shape[1], c["n_isects"]))
    out["c3 64 instances"] = {
        "I_total": sum(x[3] for x in inst), "N_total": sum(x[2] for x in inst),
        "I_per_N_min": min(x[3] / x[2] for x in inst),
        "I_per_N_max": max(x[3] / x[2] for x in inst),
        "instances": [{"W": w, "H": h, "N": m, "I": i} for w, h, m, i in inst]}
    return out


def run_viewer(args) -> dict:
    """Viewer-style SH-3 scene: 1M splats, 1920x1080, 16 orbit cameras (fx 1200).
    Forward-only renders (the SplatRenderer path) and fwd+bwd+Adam fitter steps,
    FP32 and BF16 storage.  The scene (236 MB of FP32 parameters) exceeds L2."""
    import torch
    from diffsplat_b200 import _lib as L
    from diffsplat_b200 import api
    from diffsplat_b200.scenes import make_target, orbit_cameras, viewer_scene
    torch.cuda.set_device(0)
    W, H, n = 1920, 1080, 1_000_000
    P = torch.tensor(viewer_scene(n, seed=0), device="cuda")
    cams = orbit_cameras(16, width=W, height=H, fx=1200.0)
    tgt = torch.tensor(make_target(W, H, 2000, 7), device="cuda")
    reps = max(1, args.steps // 100)
    out = {}
    for name, storage in (("fp32", L.DS_STORAGE_FP32), ("bf16", L.DS_STORAGE_BF16)):
        r = api.Renderer(W, H, n, 3, storage=storage)
        r.set_params(P)
        for pv, eye in cams[:3]:
            r.render(pv, eye)
        torch.cuda.synchronize()
        evs, isects = [], []
        with ClockSampler(0) as clk:
            for _ in range(reps):
                for pv, eye in cams:
                    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    a.record()
                    r.render(pv, eye)
                    b.record()
                    evs.append((a, b))
            torch.cuda.synchronize()
        for pv, eye in cams:
            r.render(pv, eye)
            isects.append(r.counts()["n_isects"])
        code, _ = r.status()
        r.close()
        fwd_ms = sum(a.elapsed_time(b) for a, b in evs) / len(evs)
        f = api.Fitter(W, H, n, 3, storage=storage)
        f.set_params(P)
        f.set_target(tgt)
        f.set_camera(*cams[0])
        f.step(args.warmup)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        f.step(reps * 10)
        b.record()
        torch.cuda.synchronize()
        step_ms = a.elapsed_time(b) / (reps * 10)
        stages = f.profile_step()
        code2, _ = f.status()
        f.close()
        out[name] = {"forward_frames_per_s": 1e3 / fwd_ms, "forward_ms": fwd_ms,
                     "forward_mpix_per_s": W * H / fwd_ms / 1e3,
                     "fwd_bwd_adam_steps_per_s": 1e3 / step_ms, "fwd_bwd_adam_ms": step_ms,
                     "stage_ms": stages, "n_isects_per_camera": isects,
                     "status": max(code, code2), "clocks": clk.summary()}
    return out


def run_batch(args) -> dict:
    """64 uneven fitting instances (sizes from {128^2, 256^2, 512^2, 640x480,
    1024x768}, 2k-200k splats log-uniform) in one graph-captured step with
    BF16 storage and autotuned tile size / pixels per thread / CTA schedule,
    against the same instances fitted one after another by the FP32 fitter."""
    import torch
    from diffsplat_b200 import _lib as L
    from diffsplat_b200 import api, autotune
    from diffsplat_b200.scenes import batch_problems, psnr_from_ref_loss
    torch.cuda.set_device(0)
    probs = batch_problems(64, seed=0)
    sizes = [(p.width, p.height, p.params.shape[1]) for p in probs]
    targets = [torch.tensor(p.target, device="cuda") for p in probs]
    lrs = probs[0].lrs

    def setup(b):
        for k, p in enumerate(probs):
            b.set_params(k, p.params)
            b.set_target(k, targets[k])
            b.set_camera(k, p.pv, p.cam)

    cap = 1 << 27  # pairs of all 64 instances (about 27M at 32-pixel tiles)
    best, table = autotune.tune_batch(sizes, setup, lrs=lrs, max_isects=cap)
    b = api.Batch(sizes, lrs=lrs, max_isects=cap, **best)
    setup(b)
    b.step(args.warmup)
    torch.cuda.synchronize()
    steps = args.steps
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(0) as clk:
        t0.record()
        b.step(steps)
        t1.record()
        torch.cuda.synchronize()
    batch_ms = t0.elapsed_time(t1)
    batch_psnr = [psnr_from_ref_loss(x) for x in b.losses()]
    code, _ = b.status()
    isects = b.counters()["n_isects"]
    b.close()
    # sequential FP32 fitters, same number of steps each
    seq_ms, seq_psnr = 0.0, []
    for k, p in enumerate(probs):
        f = api.Fitter(p.width, p.height, p.params.shape[1], 0, lrs=lrs)
        f.set_params(p.params)
        f.set_target(targets[k])
        f.set_camera(p.pv, p.cam)
        f.step(args.warmup)
        torch.cuda.synchronize()
        a, c = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        f.step(steps)
        c.record()
        torch.cuda.synchronize()
        seq_ms += a.elapsed_time(c)
        seq_psnr.append(psnr_from_ref_loss(f.loss()))
        f.close()
    pixels = sum(w * h for w, h, _ in sizes)
    dpsnr = [x - y for x, y in zip(batch_psnr, seq_psnr)]
    return {"instances": len(sizes), "splats": sum(n for _, _, n in sizes), "pixels": pixels,
            "tuned": best, "tuning_ms_per_step": [[c, ms] for c, ms in table],
            "batch_steps_per_s": steps / (batch_ms / 1e3),
            "batch_instance_steps_per_s": len(sizes) * steps / (batch_ms / 1e3),
            "batch_mpix_per_s": pixels * steps / (batch_ms / 1e3) / 1e6,
            "sequential_fp32_instance_steps_per_s": len(sizes) * steps / (seq_ms / 1e3),
            "speedup_vs_sequential": seq_ms / batch_ms,
            "psnr_batch_bf16": batch_psnr, "psnr_sequential_fp32": seq_psnr,
            "psnr_delta_min": min(dpsnr), "psnr_delta_mean": sum(dpsnr) / len(dpsnr),
            "n_isects": isects, "status": code, "clocks": clk.summary()}


def gemm_tflops(M: int, N: int, K: int, reps: int = 10) -> float:
    """Device TFLOP/s of the tcgen05 GEMM D = A . B^T (BF16 in, FP32 out)."""
    import torch
    from diffsplat_b200 import nn
    A = torch.randn(M, K, device="cuda").to(torch.bfloat16)
    B = torch.randn(N, K, device="cuda").to(torch.bfloat16)
    D = torch.empty(M, N, device="cuda")
    g = nn.Gemm()
    for _ in range(3):
        g(A, B, D=D)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(reps):
        g(A, B, D=D)
    b.record()
    torch.cuda.synchronize()
    g.check()
    return 2.0 * M * N * K * reps / (a.elapsed_time(b) * 1e-3) / 1e12


def run_init(args) -> dict:
    """Learned initializer at 512^2: training pairs fitted by the batched BF16
    fitter from the grid init, network training (AdamW, batch 32), and steps /
    seconds to 28 dB on held-out targets for random, grid and learned inits,
    plus learned init + batched BF16 fitting of all held-out targets at once."""
    import torch
    from diffsplat_b200 import api, initializer as I
    from diffsplat_b200.scenes import PLAIN_SMALL_LRS
    torch.cuda.set_device(0)
    n_train, n_eval, fit_steps = 256, 16, 500
    init = I.Initializer(512, seed=0)
    t0 = time.perf_counter()
    targets = I.make_targets_gpu(n_train + n_eval, 512, seed=11)
    torch.cuda.synchronize()
    t_targets = time.perf_counter() - t0
    t0 = time.perf_counter()
    fitted = I.fit_pairs(init, targets[:n_train], steps=fit_steps, batch=64)
    t_pairs = time.perf_counter() - t0
    # network forward at batch 32: algorithmic FLOPs 2 * Ho * Wo * Cout * 9 * Cin per layer
    flops, h, cin = 0, 512, 3
    for c, s in zip(I.CHANNELS, I.STRIDES):
        h = (h - 1) // s + 1
        flops += 2 * h * h * c * 9 * cin
        cin = c
    flops += 2 * h * h * 56 * 9 * cin
    imgs = targets[:32].contiguous()
    for _ in range(2):
        init.forward(imgs)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(5):
        init.forward(imgs)
    b.record()
    torch.cuda.synchronize()
    fwd_ms = a.elapsed_time(b) / 5
    t0 = time.perf_counter()
    hist = I.train(init, targets[:n_train], fitted, steps=args.steps, batch=32, log_every=50)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0
    held = targets[n_train:]
    ev = I.evaluate(init, held, goal=28.0, max_steps=2000)
    # final PSNR at an equal step budget, the three inits side by side
    equal = {"steps": 2000, "random": [], "grid": [], "learned": []}
    grid0 = init.zero_params(1)
    for k in range(len(held)):
        t = held[k]
        for arm, p0 in (("random", I.random_init(init, k)), ("grid", grid0),
                        ("learned", init.predict(t))):
            r = I.steps_to_psnr(p0, t, init, goal=1e9, max_steps=equal["steps"], check_every=500)
            equal[arm].append(r["psnr"])
    for arm in ("random", "grid", "learned"):
        equal[f"{arm}_mean"] = float(np.mean(equal[arm]))
    d = np.array(equal["learned"]) - np.array(equal["random"])
    equal["learned_minus_random_mean"] = float(d.mean())
    equal["learned_minus_random_min"] = float(d.min())
    # learned init + batched BF16 fitting of all held-out targets together
    a.record()
    out = init.forward(held.contiguous())
    P = init.decode(out).cpu().numpy()
    S = init.splats
    bt = api.Batch([(512, 512, S)] * n_eval, lrs=PLAIN_SMALL_LRS, max_isects=n_eval * S * 16)
    for k in range(n_eval):
        bt.set_params(k, P[:, k * S:(k + 1) * S])
        bt.set_target(k, held[k])
        bt.set_camera(k, init.pv, init.cam)
    steps = 0
    while steps < 2000:
        bt.step(10)
        steps += 10
        if min(I.psnr(x) for x in bt.losses()) >= 28.0:
            break
    b.record()
    torch.cuda.synchronize()
    batch_s = a.elapsed_time(b) / 1e3
    final = [I.psnr(x) for x in bt.losses()]
    bt.close()
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (
        ROOT / "MEASURED_PEAKS.json").exists() else {"bf16_tflops": 1590.0}
    big = gemm_tflops(8192, 8192, 8192)
    l5 = gemm_tflops(32 * 64 * 64, 256, 2304)
    return {"train_pairs": n_train, "fit_steps": fit_steps, "eval_targets": n_eval,
            "seconds": {"targets": t_targets, "pairs": t_pairs, "train": t_train},
            "train_steps": args.steps, "train_history": hist,
            "net_forward_ms_batch32": fwd_ms,
            "net_forward_tflops": flops * 32 / (fwd_ms * 1e-3) / 1e12,
            "gemm_tflops_8192cubed": big, "gemm_tflops_level5": l5,
            "bf16_peak_tflops": peaks.get("bf16_tflops"),
            "gemm_frac_8192cubed": big / peaks.get("bf16_tflops", 1590.0),
            "eval": {k: v for k, v in ev.items() if k != "rows"},
            "equal_steps_final_psnr": equal,
            "learned_batched_bf16_seconds_all": batch_s, "learned_batched_steps": steps,
            "learned_batched_psnr_min": min(final),
            "random_fp32_sequential_seconds_all": ev["random_seconds"] * n_eval,
            "random_fp32_reached": ev["random_reached"]}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile-run", action="store_true",
                    help="untimed: warmup + steps eager steps of the same workload with a "
                         "2^22-pair buffer (for ncu captures); prints no JSON line")
    ap.add_argument("--gemm", default=None, metavar="M,N,K",
                    help="time one BF16 tensor-core GEMM shape and print its TFLOP/s")
    ap.add_argument("--workload", choices=["fitter", "viewer-sh3", "batch64", "init", "isects"],
                    default="fitter",
                    help="fitter: the headline 1280x720 / 60000-splat training step; "
                         "viewer-sh3: 1M-splat SH-3 scene at 1920x1080, forward and fwd+bwd; "
                         "batch64: 64 uneven instances in one batched step vs sequential; "
                         "init: learned initializer training and seconds to 28 dB; "
                         "isects: (tile, splat) pairs per splat of every config (untimed)")
    args = ap.parse_args()
    if args.profile_run:
        profile_run(args)
        return
    if args.gemm:
        import torch
        torch.cuda.set_device(0)
        M, N, K = (int(x) for x in args.gemm.split(","))
        tf = gemm_tflops(M, N, K, reps=max(1, args.steps))
        print(json.dumps({"metric": "tcgen05 BF16 GEMM TFLOP/s", "M": M, "N": N, "K": K,
                          "value": tf, "unit": "TFLOP/s"}))
        return
    if args.workload == "isects":
        print(json.dumps({"metric": "(tile, splat) pairs per splat, per config",
                          "data": "synthetic", **run_isects(args)}))
        return
    if args.workload == "init":
        res = run_init(args)
        print(json.dumps({
            "metric": "wall-time to 28 dB PSNR, learned vs random init (512^2, 16384 splats)",
            "unit": "s", "n_gpus": 1, "higher_is_better": False, "data": "synthetic",
            "config": {"workload": "5-level conv initializer 32-64-128-256-256, 64x64x4 splats, "
                                   "512^2 procedural targets (500-3000 blobs)"},
            "value": res["eval"]["learned_seconds"], **res}))
        return
    if args.workload == "batch64":
        res = run_batch(args)
        print(json.dumps({
            "metric": "batch64: aggregate instance-steps/s (fwd+bwd+Adam), BF16 batched",
            "unit": "instance-steps/s", "n_gpus": 1, "higher_is_better": True,
            "data": "synthetic", "steps": args.steps, "warmup": args.warmup,
            "config": {"workload": "64 instances, sizes {128^2, 256^2, 512^2, 640x480, "
                                   "1024x768}, 2k-200k splats log-uniform, SH 0"},
            "value": res["batch_instance_steps_per_s"], **res}))
        return
    if args.workload == "viewer-sh3":
        res = run_viewer(args)
        print(json.dumps({
            "metric": "viewer-sh3: forward frames/s and fwd+bwd+Adam steps/s",
            "unit": "frames/s", "n_gpus": 1, "higher_is_better": True, "data": "synthetic",
            "config": {"workload": "1M splats on 20 planes/spheres in a radius-10 ball, SH 3, "
                                   "1920x1080, 16 orbit cameras (radius 15, fx 1200)",
                       "splats": 1_000_000, "width": 1920, "height": 1080, "sh_degree": 3},
            "value": res["fp32"]["forward_frames_per_s"], "fp32": res["fp32"],
            "bf16": res["bf16"]}))
        return
    args.warmup = max(args.warmup, 3)
    world, rank, local = dist_setup(args.gpus)
    config = {"workload": "reference-default fitter: 1280x720 procedural target (2000 blobs), "
                          "60000 splats, SH 0, 16x16 tiles, MSE, Adam (Gaussian3DAdamConfig lrs)",
              "width": 1280, "height": 720, "splats": 60000, "sh_degree": 0,
              "l2": "256 MiB flush between timed steps", "parallelism": f"replicas x{world}",
              "steps_before_timed": args.warmup,
              "fit_state": f"timed steps {args.warmup + 1}-{args.warmup + args.steps} of the fit "
                           "from its initial state (the composite's cost falls as the fit "
                           "proceeds)"}
    line = {"metric": METRIC, "unit": "steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded procedural)",
            "config": config}
    if args.impl == "reference":
        if rank != 0:
            return
        res, why = run_reference(args, 1, 0, local)
        if res is None:
            print(json.dumps({"impl": "reference", "unavailable": why}))
            return
        v = args.steps / (res["t_ms"] / 1e3)
        line.update({"impl": "reference", "n_gpus": 1, "value": v,
                     "ms_per_step": res["t_ms"] / args.steps, "clocks": res["clocks"],
                     "final_loss": res["loss"],
                     "e2e": {"value": v, "unit": "steps/s", "h2d_bytes_per_step": 0,
                             "d2h_bytes_per_step": 0},
                     "cpu_baseline": {"value": v, "unit": "steps/s", "cores": 1,
                                      "kind": "reference",
                                      "sample": "the reference's own CUDA layers (it has no CPU "
                                                "path) built for sm_100a, driven by 1 host "
                                                "thread; ImageFitter::step per step"}})
        print(json.dumps(line))
        return
    r = run_ours(args, world, rank, local)
    if rank != 0:
        return
    prob = r["prob"]
    steps_total = world * args.steps
    value = steps_total / (r["t_ms"] / 1e3)
    pixels = prob.width * prob.height
    tiles = ((prob.width + 15) // 16) * ((prob.height + 15) // 16)
    isects = r["counters"]["n_isects"]
    n = prob.params.shape[1]
    sb = stage_bytes(n, isects, pixels, [0, 3, 8, 15][prob.sh_degree])
    stages = r["stages"]
    dom = max(stages, key=stages.get)
    peaks = measured_peaks()
    pairs = r["pairs"]["contributing"]
    fp32_peak = fp32_peak_tflops(r["clocks"].get("sm_max_mhz") or peaks["sm_max_mhz"])
    tflops = {k: pairs * FLOPS_PER_PAIR[k] / (stages[k] * 1e-3) / 1e12 for k in FLOPS_PER_PAIR}
    dom_bytes = sb.get(dom, 0)
    gbs = dom_bytes / (stages[dom] * 1e-3) / 1e9
    traffic = NCU_DRAM_BYTES_PER_ISECT.get(dom)
    stage_hbm = {}
    for g, parts in STAGE_GROUPS.items():
        ms = sum(stages[p] for p in parts)
        a = sb[g] / (ms * 1e-3) / 1e9
        stage_hbm[g] = {"algorithmic_bytes": sb[g], "ms": ms, "achieved_gbs": a,
                        "frac": a / peaks["hbm_gbs"]}
    line.update({
        "value": value, "ms_per_step": r["t_ms"] / args.steps,
        "mpix_per_s": value * pixels / 1e6,
        "e2e": {"value": steps_total / (r["e2e_ms"] / 1e3), "unit": "steps/s",
                "h2d_bytes_per_step": 80, "d2h_bytes_per_step": 4},
        "gpu_launches": kernels_per_step(tiles) * args.steps,
        "clocks": r["clocks"],
        "roofline": {"bound": "fp32", "kernel": dom, "achieved": tflops.get(dom),
                     "peak": fp32_peak, "unit": "TFLOP/s",
                     "frac": tflops[dom] / fp32_peak if dom in tflops else None,
                     "traffic": traffic * isects if traffic else None,
                     "peak_src": "nominal: SMs x 128 FP32 lanes x 2 x max SM clock",
                     "algorithmic_flops": pairs * FLOPS_PER_PAIR.get(dom, 0),
                     "contributing_pairs": pairs,
                     "evaluated_pairs": r["pairs"]["evaluated"],
                     "composite_fwd_tflops": tflops["composite_fwd"],
                     "hbm": {"achieved": gbs, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                             "frac": gbs / peaks["hbm_gbs"], "peak_src": peaks["src"],
                             "algorithmic_bytes": dom_bytes}},
        "stage_hbm": {"peak_gbs": peaks["hbm_gbs"], "peak_src": peaks["src"], **stage_hbm},
        "stage_ms": stages, "n_isects": isects, "visible": r["counters"]["visible"],
        "final_loss": r["loss"], "status": r["status"],
    })
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_oracle(prob)
    print(json.dumps(line))


if __name__ == "__main__":
    main()
