"""bench.py's host-side arithmetic: launches per step, the algorithmic bytes of
each stage group (the per-unit figures of the measurement plan), and the
clock record's summary, on the CPU."""
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))

import bench  # noqa: E402


def test_launches_per_step():
    # counting tile sort (grids of up to 8192 tiles): 25 launches
    assert bench.kernels_per_step(3600) == 25
    assert bench.kernels_per_step(8192) == 25
    # radix tile sort beyond: 3 kernels per 8-bit pass over the tile id, then
    # the ranges and the schedule
    assert bench.kernels_per_step(8256) == 22 + 3 * 2 + 2
    assert bench.kernels_per_step(1 << 17) == 22 + 3 * 3 + 2


def test_stage_bytes_follow_the_per_unit_figures():
    n, pairs, pixels = 60000, 3085820, 1280 * 720
    b = bench.stage_bytes(n, pairs, pixels)
    assert b["preprocess"] == n * (14 * 4 + 40)  # 96 B per splat at SH 0
    assert b["lists"] == n * 24 + pairs * (12 + 24 + 8)
    assert b["composite_fwd"] == pairs * 40 + pixels * 20
    assert b["composite_bwd"] == pairs * 44 + pixels * 20
    assert b["backward_adam"] == n * 14 * 28
    # SH 3: 15 bands per channel
    b3 = bench.stage_bytes(1_000_000, 0, 0, bands=15)
    assert b3["preprocess"] == 1_000_000 * ((14 + 45) * 4 + 40)
    assert b3["backward_adam"] == 1_000_000 * (14 + 45) * 28
    assert set(bench.STAGE_GROUPS) == set(b)


def test_clock_summary():
    c = bench.ClockSampler(0)
    assert c.summary()["reasons"] == ["unsampled"]
    c.rows = [["1965", "1965", "700.1", "Not Active", "Not Active", "Not Active", "Not Active"],
              ["1950", "1965", "990.0", "Not Active", "Not Active", "Not Active", "Active"],
              ["1965", "1965", "995.0", "Not Active", "Not Active", "Not Active", "Active"]]
    s = c.summary()
    assert s["sm_mhz"] == 1965.0
    assert s["sm_max_mhz"] == 1965.0
    assert s["reasons"] == ["sw_power_cap"]
    assert s["samples"] == 3
    c.rows.append(["1200", "1965", "400.0", "Active", "Not Active", "Not Active", "Not Active"])
    assert bench.ClockSampler.summary(c)["reasons"] == ["hw_slowdown", "sw_power_cap"]
