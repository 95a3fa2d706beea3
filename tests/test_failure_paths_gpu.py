"""Failure detection and degenerate inputs on the GPU, made without a GPU fault.

* NaN in a host input (an observation map, a node's warp) reaches a residual,
  the PCG step or the warp field, and the next checked read reports
  MVDR_ENONFINITE (the reference would carry the NaN on silently).
* The persistent PCG's bounded barrier: with every barrier waiting for one
  arrival that never comes and a 2 ms limit, the kernel's CTAs give up and
  return, and the checked read reports MVDR_ETIMEOUT. No wait is unbounded.
* A node that no term touches gets the damped identity block, a zero
  increment and an unchanged warp, and leaves every other node's solve
  bit-identical.
Each test then runs a clean solve to show that the context is still usable.
"""
import copy

import numpy as np
import pytest
import torch

from conftest import small_scene
from multiviewdynrecon_b200 import MvdrError, abi
from multiviewdynrecon_b200.solver import BatchSolver, NonRigidSolver

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import multiviewdynrecon_b200 as m
    m.lib()


def _clean_solve(scene):
    s = NonRigidSolver(abi.make_config(scene))
    s.set_solver_input(scene)
    s.solve_non_rigid_alignment(2, 5)
    out = s.solved_node_se3()
    assert torch.isfinite(out).all()
    s.close()


def _with_nan(scene, where):
    s = copy.copy(scene)
    if where == "observation":
        views = []
        from dataclasses import replace
        for k, v in enumerate(scene.views):
            m = v.vertex_confidence_map.copy()
            if k == 0:
                m[:, :, :3] = np.nan
            views.append(replace(v, vertex_confidence_map=m))
        s.views = views
    elif where == "warp_field":
        dq = scene.node_se3.copy()
        dq[7, :] = np.nan
        s.node_se3 = dq
    else:
        raise KeyError(where)
    return s


@pytest.mark.parametrize("where", ["observation", "warp_field"])
@pytest.mark.parametrize("precision", [abi.PRECISION_MIXED, abi.PRECISION_FP32])
def test_nonfinite_input_is_reported(where, precision):
    scene = small_scene("torso")
    bad = _with_nan(scene, where)
    s = NonRigidSolver(abi.make_config(bad, precision=precision))
    s.set_solver_input(bad)
    s.solve_non_rigid_alignment(2, 5)
    with pytest.raises(MvdrError) as e:
        s.solved_node_se3()
    assert e.value.status == abi.MVDR_ENONFINITE
    s.close()
    _clean_solve(scene)


def test_persistent_barrier_timeout_is_reported():
    scene = small_scene("torso")
    b = BatchSolver(abi.make_config(scene), 2)
    b.set_pcg_persistent(True)
    b.set_wait_limit(2_000_000, extra_arrivals=1)  # 2 ms, one arrival that never comes
    for i in range(2):
        b.set_input(i, scene)
    b.solve(1, 5, use_graph=False)
    torch.cuda.synchronize()
    for i in range(2):
        assert b.instance(i).counts().error_flags != 0
        with pytest.raises(MvdrError) as e:
            b.node_se3(i)
        assert e.value.status == abi.MVDR_ETIMEOUT
    # back to the default limit: the same batch solves cleanly again
    b.set_wait_limit(500_000_000, extra_arrivals=0)
    for i in range(2):
        b.set_input(i, scene)
    b.solve(2, 5, use_graph=False)
    for i in range(2):
        assert torch.isfinite(b.node_se3(i)).all()
    b.close()


def test_wait_limit_arguments_are_checked():
    scene = small_scene("torso")
    b = BatchSolver(abi.make_config(scene), 1)
    with pytest.raises(MvdrError) as e:
        b.set_wait_limit(0)
    assert e.value.status == abi.MVDR_EINVAL
    with pytest.raises(MvdrError):
        b.set_wait_limit(11_000_000_000)
    b.close()


@pytest.mark.parametrize("precision", [abi.PRECISION_MIXED, abi.PRECISION_FP32])
def test_node_without_terms(precision):
    """An extra node far from the surface, referenced by no skinning entry,
    graph edge or correspondence."""
    scene = small_scene("torso")
    iso = copy.copy(scene)
    iso.canonical_nodes = np.concatenate([scene.canonical_nodes, np.array([[5.0, 5.0, 5.0, 1.0]], np.float32)])
    ident = np.array([[0, 0, 0, 1, 0, 0, 0, 0]], np.float32)
    iso.node_se3 = np.concatenate([scene.node_se3, ident])
    n = scene.num_nodes
    cfg = abi.make_config(iso, precision=precision)  # the same capacities for both solves
    a, b = NonRigidSolver(cfg), NonRigidSolver(cfg)
    a.set_solver_input(scene)
    b.set_solver_input(iso)
    for s in (a, b):
        s.solve_non_rigid_alignment(scene.gn_iterations, scene.pcg_iterations)
    xa = a.get_array(abi.ARRAY_INCREMENT)
    xb = b.get_array(abi.ARRAY_INCREMENT)
    assert np.array_equal(xb[n], np.zeros(6, np.float32))
    assert np.array_equal(xb[:n], xa)
    fa, fb = a.solved_node_se3().cpu().numpy(), b.solved_node_se3().cpu().numpy()
    assert np.array_equal(fb[:n], fa)
    assert np.array_equal(fb[n], ident[0])
    d = b.get_array(abi.ARRAY_DIAG_BLOCKS).reshape(-1, 6, 6)[n]
    assert np.allclose(d, 1e-2 * np.eye(6), rtol=0, atol=1e-9)
    assert b.counts().error_flags == 0
