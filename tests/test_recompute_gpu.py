"""Matrix-free PCG with the pixel terms re-derived in every iteration
(recompute_jacobians, as ApplyJtJMatrixFreeIndexed.cu:222-348 does) against
the stored-record form and the FP64 oracle."""
import numpy as np
import pytest
import torch

from conftest import rel_norm_error, small_scene
from multiviewdynrecon_b200 import abi, lib
from multiviewdynrecon_b200.solver import NonRigidSolver

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    lib()


@pytest.mark.parametrize("kind", ["sphere", "torso", "body"])
@pytest.mark.parametrize("precision", [abi.PRECISION_MIXED, abi.PRECISION_FP32])
def test_recompute_equals_stored_records(oracle_mod, kind, precision):
    scene = small_scene(kind)
    out = {}
    for rec in (False, True):
        cfg = abi.make_config(scene, precision=precision, mode=abi.MODE_MATRIX_FREE, recompute_jacobians=rec)
        s = NonRigidSolver(cfg)
        s.set_solver_input(scene)
        s.build_index()
        incs = []
        for _ in range(scene.gn_iterations):
            s.gn_iteration(scene.pcg_iterations)
            torch.cuda.synchronize()
            incs.append(s.get_array(abi.ARRAY_INCREMENT))
        out[rec] = (incs, s.get_array(abi.ARRAY_NODE_SE3), s)
    # the same device function gives both forms' records; the compiler may
    # contract its arithmetic differently in the two kernels, so the bar is a
    # relative 1e-6 (mixed) / 1e-4 (FP32) rather than bit equality
    tol = 1e-6 if precision == abi.PRECISION_MIXED else 1e-4
    for a, b in zip(out[False][0], out[True][0]):
        assert rel_norm_error(b, a) < tol
    assert rel_norm_error(out[True][1], out[False][1]) < tol
    if precision == abi.PRECISION_MIXED:
        # and the first increment against the FP64 oracle
        s = out[True][2]
        cfg = abi.make_config(scene, precision=precision, mode=abi.MODE_MATRIX_FREE, recompute_jacobians=True)
        g = NonRigidSolver(cfg)
        g.set_solver_input(scene)
        g.build_index()
        g.gn_iteration(scene.pcg_iterations)
        torch.cuda.synchronize()
        o = oracle_mod.Oracle(scene, abi.make_config(scene), fp64=True)
        o.build_index()
        o.freeze(g.get_array(abi.ARRAY_TERM_JACOBIAN), g.get_array(abi.ARRAY_SMOOTH_TERMS))
        o.eval_terms()
        o.assemble()
        o.pcg(scene.pcg_iterations)
        assert rel_norm_error(g.get_array(abi.ARRAY_INCREMENT), o.get(abi.ARRAY_INCREMENT, as_double=True)) < 1e-4
        g.close()
    for rec in (False, True):
        out[rec][2].close()
