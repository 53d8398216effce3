"""Multi-GPU runs of bench.py are replicas (the factorisation does not shard):
every rank fits and predicts its own copy, the step time is the maximum over
ranks, and the whole-job value counts one job per rank.  The collective part
is checked here with world_size 2 on the CPU (gloo)."""
import os
import sys

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _worker(rank, world, port, values, out):
    sys.path.insert(0, ROOT)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        got = bench.max_over_ranks(values[rank], dist, torch.device("cpu"))
        out.put((rank, got, bench.aggregate_seconds(got, world)))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo_world2():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    values = [12.5, 31.25]
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_worker, args=(r, 2, port, values, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res = sorted(out.get(timeout=10) for _ in range(2))
    for rank, got, agg in res:
        assert got == max(values)
        assert agg == pytest.approx(max(values) / 1e3 / 2)


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks(7.0, None, torch.device("cpu")) == 7.0
    assert bench.aggregate_seconds(250.0, 1) == pytest.approx(0.25)
