"""Autotuner of the batched fitter: picks the composite tile size (8, 16 or 32
pixels), pixels per thread (1 or 2) and CTA schedule (longest tile list first
or raster order) for a given batch by timing a few steps of each candidate on
the batch's own inputs with CUDA events.

    best, table = tune_batch(sizes, setup, sh_degree=0)
    batch = api.Batch(sizes, **best)

`setup(batch)` loads a candidate batch's parameters, targets and cameras; the
trial batches are discarded, so the tuned batch starts from the same state.
"""
from __future__ import annotations

import itertools

from . import _lib as L
from . import api

TILE_SIZES = (8, 16, 32)
PPTS = (1, 2)
SCHEDULES = (L.DS_SCHEDULE_LONGEST_FIRST, L.DS_SCHEDULE_RASTER)


def tune_batch(sizes, setup, sh_degree: int = 0, steps: int = 6, warmup: int = 2,
               candidates=None, **batch_kw):
    """Returns ({"tile_size", "ppt", "schedule"} of the fastest candidate,
    [(candidate, ms per step)] for all)."""
    import torch
    if candidates is None:
        candidates = [dict(tile_size=t, ppt=p, schedule=s)
                      for t, p, s in itertools.product(TILE_SIZES, PPTS, SCHEDULES)]
    table = []
    for cand in candidates:
        b = api.Batch(sizes, sh_degree=sh_degree, **cand, **batch_kw)
        try:
            setup(b)
            b.step(warmup)
            torch.cuda.synchronize()
            t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            t0.record()
            b.step(steps)
            t1.record()
            torch.cuda.synchronize()
            code, _ = b.status()
            ms = t0.elapsed_time(t1) / steps if code == L.DS_OK else float("inf")
        finally:
            b.close()
        table.append((cand, ms))
    best = min(table, key=lambda x: x[1])[0]
    return dict(best), table
