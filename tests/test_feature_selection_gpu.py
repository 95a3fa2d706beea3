"""Sparse feature selection on the GPU (part of the index build) against the
oracle: the same kept pairs in the same order (bit-exact index and term
records), then the solve against the FP64 oracle."""
import ctypes as C

import numpy as np
import pytest
import torch

from conftest import rel_norm_error, small_scene
from multiviewdynrecon_b200 import abi, lib, synth
from multiviewdynrecon_b200.solver import DeviceScene, NonRigidSolver

pytestmark = pytest.mark.gpu

INDEX_ARRAYS = [abi.ARRAY_NODE2TERM_OFFSET, abi.ARRAY_NODE2TERM_INDEX, abi.ARRAY_HALF_NODEPAIR_KEY,
                abi.ARRAY_NODEPAIR_TERM_INDEX, abi.ARRAY_NODEPAIR_KEY, abi.ARRAY_NODEPAIR_TERM_RANGE,
                abi.ARRAY_BLKROW_OFFSET]


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    lib()


def bits(a):
    return np.ascontiguousarray(a).view(np.uint8)


@pytest.mark.parametrize("kind", ["torso", "body", "sphere_rigid"])
def test_selected_index_bit_exact(oracle_mod, kind):
    scene = synth.with_feature_pairs(small_scene(kind), per_view=300, seed=4)
    cfg = abi.make_config(scene)
    g = NonRigidSolver(cfg)
    g.set_solver_input(scene)
    g.build_index()
    o = oracle_mod.Oracle(scene, cfg)
    o.build_index()
    gc, oc = g.counts(), o.counts()
    assert gc.error_flags == 0
    assert gc.feature_terms == oc.feature_terms > 100
    for f in ("dense_terms", "smooth_terms", "foreground_terms", "cross_terms", "node2term_entries",
              "nodepair_entries", "half_pairs"):
        assert getattr(gc, f) == getattr(oc, f), f
    for which in INDEX_ARRAYS:
        assert np.array_equal(bits(g.get_array(which)), bits(o.get(which))), which
    # the selected terms' positions, to the bit
    assert np.array_equal(bits(g.get_array(abi.ARRAY_FEATURE_TERMS)), bits(o.get(abi.ARRAY_FEATURE_TERMS)))
    # the warped feature records: the GPU keeps the capacity as the stride
    g.gn_iteration(1)
    torch.cuda.synchronize()
    o.eval_terms()
    gw = g.get_array(abi.ARRAY_WARPED_CORRESPONDENCE).reshape(-1, 8)[:oc.feature_terms]
    ow = o.get(abi.ARRAY_WARPED_CORRESPONDENCE).reshape(-1, 8)[:oc.feature_terms]
    np.testing.assert_allclose(gw, ow, atol=1e-5)
    g.close()


@pytest.mark.parametrize("kind", ["torso", "body"])
def test_selected_solve_vs_fp64_oracle(oracle_mod, kind):
    scene = synth.with_feature_pairs(small_scene(kind), per_view=300, seed=6)
    cfg = abi.make_config(scene, precision=abi.PRECISION_MIXED)
    g = NonRigidSolver(cfg)
    g.set_solver_input(scene)
    g.build_index()
    o64 = oracle_mod.Oracle(scene, cfg, fp64=True)
    o64.build_index()
    for it in range(scene.gn_iterations):
        o64.set_node_se3(g.get_array(abi.ARRAY_NODE_SE3))
        g.gn_iteration(scene.pcg_iterations)
        torch.cuda.synchronize()
        o64.freeze(g.get_array(abi.ARRAY_TERM_JACOBIAN), g.get_array(abi.ARRAY_SMOOTH_TERMS))
        o64.eval_terms()
        o64.assemble()
        o64.pcg(scene.pcg_iterations)
        assert rel_norm_error(g.get_array(abi.ARRAY_INCREMENT), o64.get(abi.ARRAY_INCREMENT, as_double=True)) < 1e-4
    g.close()


def test_graph_replay_reselects():
    """The selection runs inside every (graph-replayed) solve: two solves of
    the same inputs give the same warp field."""
    scene = synth.with_feature_pairs(small_scene("torso"), per_view=300, seed=1)
    cfg = abi.make_config(scene)
    from multiviewdynrecon_b200.solver import BatchSolver
    b = BatchSolver(cfg, 2)
    ds = DeviceScene(scene)
    b.set_input(0, ds)
    b.set_input(1, ds)
    b.solve(3, 10, use_graph=True)
    a0, a1 = b.node_se3(0), b.node_se3(1)
    assert torch.equal(a0, a1)
    b.set_input(0, ds)
    b.set_input(1, ds)
    b.solve(3, 10, use_graph=True)
    assert torch.equal(b.node_se3(0), a0)
    b.close()


def test_feature_pair_argument_checks():
    scene = synth.with_feature_pairs(small_scene("torso"), per_view=50, seed=3)
    ds = DeviceScene(scene)

    def status(cfg, mutate):
        s = NonRigidSolver(cfg)
        inp = abi.Inputs.from_buffer_copy(ds.inputs)
        mutate(inp)
        st = lib().mvdr_set_inputs(s.h, C.byref(inp), None)
        s.close()
        return st

    cfg = abi.make_config(scene)
    assert status(cfg, lambda i: None) == abi.MVDR_OK
    off = abi.make_config(scene, use_feature=False)
    assert status(off, lambda i: None) == abi.MVDR_EINVAL

    def both(i):
        i.feature.count = 1
        i.feature.target_vertex = i.feature.reference_vertex = i.feature.knn = i.feature.knn_weight = \
            i.feature_pairs.live_vertex_map[0]
    assert status(cfg, both) == abi.MVDR_EINVAL
    small = abi.make_config(scene, max_feature_terms=10)
    assert status(small, lambda i: None) == abi.MVDR_ECAPACITY

    def unbound_view(i):
        i.feature_pairs.count[scene.num_views] = 5
    assert status(cfg, unbound_view) == abi.MVDR_EINVAL

    def no_live(i):
        i.feature_pairs.live_vertex_map[0] = None
    assert status(cfg, no_live) == abi.MVDR_EINVAL
