"""The convergence-checked PCG (BlockPCG::SolveConvergeChecked,
core/NonRigidSolver/BlockPCG.cuh:339-377) in the oracle: the solve stops
after the first iteration k >= 1 whose delta_k = r.M^-1 r is below
tol^2 delta_0, and equals the fixed-count solve of k iterations (CPU)."""
import ctypes as C

import numpy as np
import pytest

from conftest import small_scene
from multiviewdynrecon_b200 import abi


@pytest.mark.parametrize("kind", ["sphere", "torso"])
@pytest.mark.parametrize("tol", [1e-1, 1e-2])
def test_oracle_stops_at_the_first_small_delta(oracle_mod, kind, tol):
    scene = small_scene(kind)
    full = oracle_mod.Oracle(scene, abi.make_config(scene), fp64=True)
    full.build_index()
    full.eval_terms()
    full.assemble()
    full.pcg(60)
    hist = full.pcg_history()
    assert len(hist) == 60 and np.all(np.diff(np.log(hist[:10])) < 0.5)
    below = np.nonzero(np.abs(hist[1:]) < tol * tol * abs(hist[0]))[0]
    assert len(below), "the tolerance is reached within 60 iterations"
    k = int(below[0]) + 1
    chk = oracle_mod.Oracle(scene, abi.make_config(scene, pcg_tolerance=tol), fp64=True)
    chk.build_index()
    chk.eval_terms()
    chk.assemble()
    chk.pcg(60)
    assert len(chk.pcg_history()) == k + 1
    np.testing.assert_array_equal(chk.pcg_history(), hist[:k + 1])
    fixed = oracle_mod.Oracle(scene, abi.make_config(scene), fp64=True)
    fixed.build_index()
    fixed.eval_terms()
    fixed.assemble()
    fixed.pcg(k)
    np.testing.assert_array_equal(chk.get(abi.ARRAY_INCREMENT, as_double=True),
                                  fixed.get(abi.ARRAY_INCREMENT, as_double=True))


def test_tolerance_validation():
    """A tolerance outside [0, 1) is refused at create, before any CUDA call."""
    from multiviewdynrecon_b200 import lib
    scene = small_scene("sphere")
    for bad in (1.5, -0.1, float("nan")):
        cfg = abi.make_config(scene, pcg_tolerance=bad)
        h = C.c_void_p()
        assert lib().mvdr_create(C.byref(cfg), C.byref(h)) == abi.MVDR_EINVAL
        assert b"pcg_tolerance" in lib().mvdr_last_error_string()


def test_recompute_needs_the_matrix_free_mode():
    """recompute_jacobians with the materialised operator is refused at create."""
    from multiviewdynrecon_b200 import lib
    scene = small_scene("sphere")
    cfg = abi.make_config(scene, mode=abi.MODE_MATERIALIZED, recompute_jacobians=True)
    h = C.c_void_p()
    assert lib().mvdr_create(C.byref(cfg), C.byref(h)) == abi.MVDR_EINVAL
    assert b"matrix-free" in lib().mvdr_last_error_string()
