"""bench.py's multi-rank logic on CPU: two gloo ranks, each timing its own
replica; the reported step time is the max over ranks and the value is the
whole-job aggregate (replicas only: the filtering path has no exchange)."""

import os
import sys

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank_main(rank, world, port, q):
    sys.path.insert(0, ROOT)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        local_ms = [3.0, 5.0][rank]
        ms = bench.reduce_step_time(local_ms, world, torch.device("cpu"), dist, torch)
        q.put((rank, ms, bench.aggregate_value(1000, world, ms)))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_aggregate():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    for rank, ms, value in got:
        assert ms == pytest.approx(5.0)
        assert value == pytest.approx(1000 * 2 / 5e-3 / 1e9)
