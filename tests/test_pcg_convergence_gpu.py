"""The convergence-checked PCG on the GPU: the device decides the stop (no
host synchronisation), per instance; the residual history matches the FP64
oracle's; a stopped solve equals the fixed-count solve of as many
iterations, bit for bit."""
import ctypes as C

import numpy as np
import pytest
import torch

from conftest import rel_norm_error, small_scene
from multiviewdynrecon_b200 import abi, lib
from multiviewdynrecon_b200.solver import BatchSolver, DeviceScene, NonRigidSolver

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    lib()


def one_iteration(scene, cfg, pcg):
    s = NonRigidSolver(cfg)
    s.set_solver_input(scene)
    s.build_index()
    s.gn_iteration(pcg)
    torch.cuda.synchronize()
    return s


@pytest.mark.parametrize("kind", ["sphere", "torso"])
def test_history_matches_oracle(oracle_mod, kind):
    scene = small_scene(kind)
    cfg = abi.make_config(scene, precision=abi.PRECISION_MIXED)
    s = one_iteration(scene, cfg, 20)
    hist = s.get_array(abi.ARRAY_PCG_RESIDUALS)
    assert hist.shape == (1, abi.MVDR_PCG_HISTORY)
    h = hist[0]
    assert np.all(np.isfinite(h[:20])) and np.all(np.isnan(h[20:]))
    o = oracle_mod.Oracle(scene, cfg, fp64=True)
    o.build_index()
    o.freeze(s.get_array(abi.ARRAY_TERM_JACOBIAN), s.get_array(abi.ARRAY_SMOOTH_TERMS))
    o.eval_terms()
    o.assemble()
    o.pcg(20)
    want = o.pcg_history()
    # delta decays by orders of magnitude; each entry to 1e-4 of itself
    np.testing.assert_allclose(h[:20], want, rtol=1e-4, atol=0)
    s.close()


@pytest.mark.parametrize("kind", ["sphere", "torso"])
@pytest.mark.parametrize("precision", [abi.PRECISION_MIXED, abi.PRECISION_FP32])
def test_stop_equals_fixed_count(oracle_mod, kind, precision):
    scene = small_scene(kind)
    tol = 1e-2
    chk = one_iteration(scene, abi.make_config(scene, precision=precision, pcg_tolerance=tol), 60)
    h = chk.get_array(abi.ARRAY_PCG_RESIDUALS)[0]
    ran = int(np.sum(np.isfinite(h))) - 1  # iterations completed before the stop
    assert 1 <= ran < 59
    assert abs(h[ran]) < tol * tol * abs(h[0]) <= abs(h[ran - 1]) or ran == 1
    fixed = one_iteration(scene, abi.make_config(scene, precision=precision), ran)
    assert np.array_equal(chk.get_array(abi.ARRAY_INCREMENT), fixed.get_array(abi.ARRAY_INCREMENT))
    # the FP64 oracle stops at the same iteration or one off
    o = oracle_mod.Oracle(scene, abi.make_config(scene, pcg_tolerance=tol), fp64=True)
    o.build_index()
    o.freeze(chk.get_array(abi.ARRAY_TERM_JACOBIAN), chk.get_array(abi.ARRAY_SMOOTH_TERMS))
    o.eval_terms()
    o.assemble()
    o.pcg(60)
    assert abs((len(o.pcg_history()) - 1) - ran) <= 1
    chk.close()
    fixed.close()


def test_instances_stop_independently():
    """Two instances of a batch (both 160x120, as one batch needs) reach the
    tolerance at their own iterations; each equals its single-instance
    solve, inside a replayed graph too."""
    a, b = small_scene("torso"), small_scene("sphere")
    caps = dict(max_nodes=max(a.num_nodes, b.num_nodes), max_views=3, width=a.width, height=a.height,
                use_foreground=False, use_feature=True, use_cross_view=True,
                max_surfels=max(a.num_surfels, b.num_surfels),
                max_feature_terms=max(a.feature.count, b.feature.count),
                max_cross_terms=max(a.cross_view.count, b.cross_view.count), pcg_tolerance=3e-2)
    cfg = abi.make_config(None, **caps)
    batch = BatchSolver(cfg, 2)
    da, db = DeviceScene(a), DeviceScene(b)
    batch.set_input(0, da)
    batch.set_input(1, db)
    batch.solve(2, 40, use_graph=True)
    got = [batch.node_se3(0).cpu().numpy(), batch.node_se3(1).cpu().numpy()]
    hs = [batch.instance(i).get_array(abi.ARRAY_PCG_RESIDUALS) for i in range(2)]
    for i, (scene, ds) in enumerate(((a, da), (b, db))):
        single = BatchSolver(cfg, 1)
        single.set_input(0, ds)
        single.solve(2, 40, use_graph=False)
        assert np.array_equal(single.node_se3(0).cpu().numpy(), got[i])
        single.close()
    ran = [[int(np.sum(np.isfinite(h[g]))) - 1 for g in range(2)] for h in hs]
    assert all(1 <= r < 39 for rr in ran for r in rr)
    batch.close()
