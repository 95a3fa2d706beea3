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


def _rank_solve_main(rank, world, port, out):
    """Each rank builds its own instances (the bench's per-rank seeds on a
    small torso) and solves the first with the oracle; the ranks exchange only
    digests of their warp fields."""
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import hashlib
    import torch
    import torch.distributed as dist
    import bench
    import oracle
    from multiviewdynrecon_b200 import abi, synth
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        base = synth.torso_multi_view(seed=13, num_nodes=256, num_views=2, width=96, height=72,
                                      features_per_view=30, cross_per_pair=30)
        scenes = [synth.perturb_warp_field(base, seed=sd) for sd in bench.instance_seeds(rank, 3)]
        o = oracle.Oracle(scenes[0], abi.make_config(scenes[0]))
        o.solve(2, 5)
        solved = o.get(abi.ARRAY_NODE_SE3)
        digest = hashlib.sha256(solved.tobytes()).hexdigest()
        inputs = [hashlib.sha256(s.node_se3.tobytes()).hexdigest() for s in scenes]
        # the only collective: gather the digests for the check
        got = [None] * world
        dist.all_gather_object(got, (digest, inputs))
        out[rank] = (got, digest)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_rank_local_instances_are_built_and_solved_independently(oracle_mod):
    from multiviewdynrecon_b200 import abi, synth
    import bench
    ctx = mp.get_context("spawn")
    world, port = 2, _free_port()
    with ctx.Manager() as mgr:
        out = mgr.dict()
        procs = [ctx.Process(target=_rank_solve_main, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=300)
            assert p.exitcode == 0
        res = dict(out)
    gathered = res[0][0]
    assert gathered == res[1][0]
    # disjoint inputs across ranks
    assert not set(gathered[0][1]) & set(gathered[1][1])
    # each rank's result is the single-process solve of the same instance
    import hashlib
    base = synth.torso_multi_view(seed=13, num_nodes=256, num_views=2, width=96, height=72,
                                  features_per_view=30, cross_per_pair=30)
    for rank in range(world):
        scene = synth.perturb_warp_field(base, seed=bench.instance_seeds(rank, 3)[0])
        o = oracle_mod.Oracle(scene, abi.make_config(scene))
        o.solve(2, 5)
        assert hashlib.sha256(o.get(abi.ARRAY_NODE_SE3).tobytes()).hexdigest() == gathered[rank][0]
