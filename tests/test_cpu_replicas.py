"""bench.py's multi-GPU plumbing (replicas: a barrier around the timed steps
and the time taken as the maximum over the ranks) on world-size-2 gloo process
groups on the CPU."""
import multiprocessing as mp
import os
import socket
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, port: int, values, q) -> None:
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE="2")
    sys.path.insert(0, str(ROOT))
    import datetime

    import torch.distributed as dist

    import bench
    dist.init_process_group("gloo", rank=rank, world_size=2,
                            timeout=datetime.timedelta(seconds=60))
    try:
        bench.barrier(2)
        got = bench.max_over_ranks(2, values[rank], device="cpu")
        bench.barrier(2)
        q.put((rank, got))
    finally:
        dist.destroy_process_group()


def _run(values):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, port, values, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    return dict(q.get(timeout=5) for _ in procs)


def test_max_over_ranks_is_the_slowest_rank():
    got = _run([12.5, 7.25])
    assert got == {0: 12.5, 1: 12.5}
    got = _run([3.0, 4.0])
    assert got == {0: 4.0, 1: 4.0}


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, str(ROOT))
    import bench
    assert bench.max_over_ranks(1, 2.5) == 2.5
    bench.barrier(1)
