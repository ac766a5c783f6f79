"""The bench's multi-rank plumbing on two gloo ranks (CPU): every rank takes the same collective steps, the
time is the maximum over ranks and the work the sum (one independent population per rank, weak scaling)."""
import os
import socket
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, str(ROOT))
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    import bench

    # per-rank timing and work as the bench reports them
    ms = bench.max_over_ranks(10.0 * (rank + 1), world)
    steps = bench.sum_over_ranks(1000.0 * (rank + 1), world)
    bench.barrier(world)
    out[rank] = (ms, steps, steps / (ms * 1e-3))
    dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_bench_reductions_over_two_gloo_ranks():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(90)
        assert p.exitcode == 0
    for r in range(world):
        ms, steps, value = out[r]
        assert ms == 20.0  # the slowest rank
        assert steps == 3000.0  # both populations' game steps
        assert value == pytest.approx(150_000.0)  # whole-job throughput: all work / slowest time


def test_single_rank_is_the_identity():
    sys.path.insert(0, str(ROOT))
    import bench

    assert bench.max_over_ranks(7.5, 1) == 7.5 and bench.sum_over_ranks(3.0, 1) == 3.0
