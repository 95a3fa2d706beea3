"""Parity at the benchmark configurations' full sizes (through the C ABI).

* Plain method, 1 view: 640x480 sphere section, 2048 nodes, dense depth and
  smooth terms, 3 Gauss-Newton x 10 PCG iterations, in plain FP32 (the
  configuration's own arithmetic) and in mixed precision.
* Multi-view: 3 views at 640x480 around the torso, 4096 nodes, every term
  (dense depth, foreground, 1000 features per view, 2000 cross-view pairs per
  adjacent view pair), 5 Gauss-Newton x 15 PCG iterations, mixed precision -
  the configuration the benchmark times.

For each: the index (every array) bit-exact against the oracle; every
Gauss-Newton increment against the FP64 oracle linearised at the GPU's warp
field of that iteration, with the GPU's projected pixels and validity
decisions (relative 2-norm below 1e-4 in mixed precision; 2e-3 in FP32, whose
15-iteration float PCG loses that much); the energy of every iteration within
1e-4 of the FP64 oracle's; and the final energy of the whole solve, each side
on its own trajectory, within 1e-3.

A third test runs the elastic penalty schedule's local phase
(PenaltyConstants.cpp:39-51: foreground and feature weights 0 after the global
iterations) and checks its increments the same way.
"""
import numpy as np
import pytest
import torch

from conftest import rel_norm_error
from multiviewdynrecon_b200 import abi, synth
from multiviewdynrecon_b200.solver import NonRigidSolver

pytestmark = pytest.mark.gpu

INDEX_ARRAYS = [abi.ARRAY_DENSE_PIXELS, abi.ARRAY_DENSE_KNN, abi.ARRAY_DENSE_KNN_WEIGHT,
                abi.ARRAY_FOREGROUND_PIXELS, abi.ARRAY_NODE2TERM_OFFSET, abi.ARRAY_NODE2TERM_INDEX,
                abi.ARRAY_HALF_NODEPAIR_KEY, abi.ARRAY_NODEPAIR_TERM_INDEX, abi.ARRAY_NODEPAIR_KEY,
                abi.ARRAY_NODEPAIR_TERM_RANGE, abi.ARRAY_BLKROW_OFFSET, abi.ARRAY_BINBLOCK_ROWPTR,
                abi.ARRAY_BINBLOCK_COLPTR]

_SCENES = {}


def scene_of(kind):
    if kind not in _SCENES:
        if kind == "sphere":
            _SCENES[kind] = synth.sphere_single_view(seed=1, num_nodes=2048, width=640, height=480)
        elif kind == "torso":
            _SCENES[kind] = synth.torso_multi_view(seed=2, num_nodes=4096, num_views=3, width=640, height=480)
        else:
            raise KeyError(kind)
    return _SCENES[kind]


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import multiviewdynrecon_b200 as m
    m.lib()


def check_solve(oracle_mod, scene, cfg, gn, pcg, tol):
    g = NonRigidSolver(cfg)
    g.set_solver_input(scene)
    g.build_index()
    o = oracle_mod.Oracle(scene, cfg)
    o.build_index()
    gc, oc = g.counts(), o.counts()
    assert gc.error_flags == 0
    for f in ("dense_terms", "smooth_terms", "foreground_terms", "feature_terms", "cross_terms",
              "node2term_entries", "nodepair_entries", "half_pairs", "num_bins", "binblock_nnz"):
        assert getattr(gc, f) == getattr(oc, f), f
    for which in INDEX_ARRAYS:
        a, b = g.get_array(which), o.get(which)
        assert a.shape == b.shape, which
        assert np.array_equal(np.ascontiguousarray(a).view(np.uint8), np.ascontiguousarray(b).view(np.uint8)), which
    del o
    o64 = oracle_mod.Oracle(scene, cfg, fp64=True)
    o64.build_index()
    errs, energies = [], []
    for it in range(gn):
        o64.set_node_se3(g.get_array(abi.ARRAY_NODE_SE3))
        g.gn_iteration(pcg)
        torch.cuda.synchronize()
        o64.freeze(g.get_array(abi.ARRAY_TERM_JACOBIAN), g.get_array(abi.ARRAY_SMOOTH_TERMS))
        o64.eval_terms()
        o64.assemble()
        energies.append((g.energy(), o64.energy()))
        o64.pcg(pcg)
        o64.update()  # keeps the oracle's iteration counter (penalty schedule) in step
        errs.append(rel_norm_error(g.get_array(abi.ARRAY_INCREMENT), o64.get(abi.ARRAY_INCREMENT, as_double=True)))
    assert g.counts().error_flags == 0
    assert max(errs) < tol, errs
    for eg, eo in energies:
        assert abs(eg - eo) <= 1e-4 * abs(eo), (eg, eo)
    assert energies[-1][0] < energies[0][0]
    return g, errs


@pytest.mark.parametrize("kind,precision,tol", [("sphere", abi.PRECISION_FP32, 2e-3),
                                                ("sphere", abi.PRECISION_MIXED, 1e-4),
                                                ("torso", abi.PRECISION_MIXED, 1e-4)])
def test_full_size_increments_vs_fp64(oracle_mod, kind, precision, tol):
    scene = scene_of(kind)
    cfg = abi.make_config(scene, precision=precision)
    check_solve(oracle_mod, scene, cfg, scene.gn_iterations, scene.pcg_iterations, tol)


@pytest.mark.parametrize("kind", ["sphere", "torso"])
def test_full_size_final_energy(oracle_mod, kind):
    """Whole solves, each side on its own trajectory."""
    scene = scene_of(kind)
    cfg = abi.make_config(scene, precision=abi.PRECISION_MIXED)
    g = NonRigidSolver(cfg)
    g.set_solver_input(scene)
    g.solve_non_rigid_alignment(scene.gn_iterations, scene.pcg_iterations)
    g.gn_iteration(1)  # evaluates the energy at the solved warp field
    eg = g.energy()
    o64 = oracle_mod.Oracle(scene, cfg, fp64=True)
    o64.solve(scene.gn_iterations, scene.pcg_iterations)
    o64.eval_terms()
    o64.assemble()
    eo = o64.energy()
    assert abs(eg - eo) <= 1e-3 * eo, (eg, eo)


def test_local_phase_of_the_penalty_schedule(oracle_mod):
    """Two global iterations, then three local ones in which the foreground
    and feature weights drop to 0 and only dense, smooth and cross-view terms
    remain (PenaltyConstants.cpp:25-51)."""
    scene = scene_of("torso")
    cfg = abi.make_config(scene, precision=abi.PRECISION_MIXED, num_global_iterations=2)
    _, errs = check_solve(oracle_mod, scene, cfg, 5, scene.pcg_iterations, 1e-4)
    assert len(errs) == 5
