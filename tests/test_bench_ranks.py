"""The multi-rank arithmetic of bench.py on CPU: two gloo ranks (the N > 1
path runs one independent replica per rank, with no collective on the data
path; only the timings are reduced, max over ranks)."""
import os
import sys

import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _rank(rank, world, port, out):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # rank r timed 10 + r ms for the steps and 50 - r ms end to end
        ms, e2e = bench.max_over_ranks([10.0 + rank, 50.0 - rank], dist)
        out[rank] = (ms, e2e, bench.job_value(world, 1000, 4, ms))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_job_value_with_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    port = 29500 + os.getpid() % 2000
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    for r in range(2):
        ms, e2e, value = out[r]
        assert ms == 11.0 and e2e == 50.0
        assert value == pytest.approx(2 * 1000 * 4 / 0.011)


def test_single_rank_needs_no_collective():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks([3.0, 4.0]) == [3.0, 4.0]
    assert bench.job_value(1, 100, 2, 1.0) == pytest.approx(2e5)
