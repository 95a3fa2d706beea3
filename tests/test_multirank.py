"""The multi-rank path of bench.py on CPU: two gloo ranks (world size 2).

Each rank solves its own instances, so the only cross-rank steps are the
max-over-ranks reduction of the timed region and the whole-job value; these
run here without a GPU.
"""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        ms = 10.0 + 5.0 * rank  # rank 1 is the slower one
        slowest = bench.max_over_ranks(ms, dist, "cpu")
        out[rank] = (slowest, bench.job_value(world, 16, slowest), tuple(bench.instance_seeds(rank, 16)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_ranks_reduce_to_the_slowest_time():
    ctx = mp.get_context("spawn")
    world, port = 2, _free_port()
    with ctx.Manager() as mgr:
        out = mgr.dict()
        procs = [ctx.Process(target=_rank_main, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=120)
            assert p.exitcode == 0
        res = dict(out)
    assert res[0][0] == res[1][0] == pytest.approx(15.0)
    # whole-job value: both ranks' 16 instances over the slowest rank's time
    assert res[0][1] == pytest.approx(2 * 16 / 0.015)
    # disjoint instance sets
    assert not set(res[0][2]) & set(res[1][2])


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(12.5, None, "cpu") == 12.5
    assert bench.job_value(1, 16, 20.0) == pytest.approx(800.0)
