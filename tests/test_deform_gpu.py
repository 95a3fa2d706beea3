"""The post-solve deformation path on the GPU against the oracle.

forward/inverse warp, node errors and error maps: every float equal to the
oracle's (deform.cu runs uncontracted IEEE operations in the oracle's order;
the node sums are exact fixed point). The correction: the same guide
choices, values within 1e-5 (its quaternion power uses atan2f, sinf and
cosf, whose last bits differ between the GPU and the host library).
"""
import numpy as np
import pytest
import torch

from conftest import small_scene
from multiviewdynrecon_b200 import abi, synth
from multiviewdynrecon_b200.deform import SurfelNodeDeformer
from multiviewdynrecon_b200.solver import NonRigidSolver

pytestmark = pytest.mark.gpu

IDENT = np.array([0, 0, 0, 1, 0, 0, 0, 0], np.float32)


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import multiviewdynrecon_b200 as m
    m.lib()


def dev(a, dtype=None):
    a = np.ascontiguousarray(a)
    if a.dtype == np.uint16:
        a = a.view(np.int16)
    return torch.from_numpy(a.copy()).cuda()


def host(t):
    return t.cpu().numpy()


def same(a, b):
    """Equal as floats (+0 == -0), NaN where the other has NaN."""
    a, b = np.asarray(a), np.asarray(b)
    return np.array_equal(a, b, equal_nan=True)


def surfels(scene):
    g = synth.solver_map_geometry(scene, warped=False)
    return g["reference_vertex_confid"], g["reference_normal_radius"]


@pytest.mark.parametrize("kind", ["sphere", "torso", "body"])
def test_forward_and_inverse_warp_bit_exact(oracle_mod, kind):
    scene = small_scene(kind)
    v, n = surfels(scene)
    nk, nw = synth.node_skinning(scene)
    nodes = synth.node_views(scene)
    knn = scene.surfel_knn.copy()
    knn[7, 1] = scene.num_nodes + 3  # a bad index: NaN outputs, no out-of-range read
    lv, ln, live = SurfelNodeDeformer.forward_warp_surfels_and_nodes(
        dev(scene.node_se3), dev(knn), dev(scene.surfel_knn_weight), dev(v), dev(n), dev(nk), dev(nw), dev(nodes))
    torch.cuda.synchronize()
    ov, on, olive = oracle_mod.forward_warp(scene.node_se3, knn, scene.surfel_knn_weight, v, n, nk, nw, nodes)
    assert same(host(lv), ov) and same(host(ln), on) and same(host(live), olive)
    assert np.isnan(host(lv)[7, 0])
    rng = np.random.default_rng(1)
    S = len(v)
    Rc = synth.rodrigues_batch(rng.normal(0, 0.05, (S, 3)))
    correct = np.concatenate([np.transpose(Rc, (0, 2, 1)).reshape(S, 9), rng.normal(0, 0.01, (S, 3))],
                             1).astype(np.float32)
    for cs in (None, correct):
        rv, rn = SurfelNodeDeformer.inverse_warp_surfels(dev(scene.node_se3), dev(knn), dev(scene.surfel_knn_weight),
                                                         lv, ln, None if cs is None else dev(cs))
        torch.cuda.synchronize()
        orv, orn = oracle_mod.inverse_warp(scene.node_se3, knn, scene.surfel_knn_weight, ov, on, cs)
        assert same(host(rv), orv) and same(host(rn), orn)


def make_solver(scene):
    """A solver bound to the scene: its current warp field is the scene's."""
    s = NonRigidSolver(abi.make_config(scene))
    ds = s.set_solver_input(scene)
    return s, ds


@pytest.mark.parametrize("kind", ["sphere", "torso", "body"])
def test_node_error_bit_exact(oracle_mod, kind):
    scene = small_scene(kind)
    s, _ = make_solver(scene)
    got = s.compute_alignment_error_on_nodes(maps=True)
    torch.cuda.synchronize()
    want = oracle_mod.node_error(scene, scene.node_se3, maps=True)
    for k in ("accumulated_error", "accumulated_weight", "united_error"):
        assert same(host(got[k]), want[k]), k
    assert np.array_equal(host(got["large_error_mark"]).astype(np.uint32), want["large_error_mark"])
    for v in range(scene.num_views):
        assert same(host(got["alignment_error_map"][v]), want["alignment_error_map"][v]), v
        assert same(host(got["node_error_map"][v]), want["node_error_map"][v]), v
    # repeatable: the fixed-point sums do not depend on the atomics' order
    again = s.compute_alignment_error_on_nodes()
    assert torch.equal(again["united_error"], got["united_error"])
    s.close()


def test_node_error_after_a_solve_is_smaller(oracle_mod):
    scene = small_scene("torso")
    s, _ = make_solver(scene)
    before = s.compute_alignment_error_on_nodes()["united_error"].clone()
    s.solve_non_rigid_alignment(scene.gn_iterations, scene.pcg_iterations)
    after = s.compute_alignment_error_on_nodes()["united_error"]
    torch.cuda.synchronize()
    assert after.mean().item() < before.mean().item()
    want = oracle_mod.node_error(scene, s.get_array(abi.ARRAY_NODE_SE3))
    assert same(host(after), want["united_error"])
    s.close()


def correction_case(oracle_mod, scene, seed):
    nk, nw = synth.node_skinning(scene)
    v, n = surfels(scene)
    lv, ln, live = oracle_mod.forward_warp(scene.node_se3, scene.surfel_knn, scene.surfel_knn_weight, v, n, nk, nw,
                                           synth.node_views(scene))
    united = np.random.default_rng(seed).uniform(0, 1, scene.num_nodes).astype(np.float32)
    return dict(guides=synth.correction_guides(scene, seed=seed), united_error=united, node_se3=scene.node_se3,
                live_nodes=live, node_knn=nk, node_weight=nw, live_vertex=lv, live_normal=ln,
                surfel_knn=scene.surfel_knn, surfel_weight=scene.surfel_knn_weight)


@pytest.mark.parametrize("kind", ["sphere", "torso", "body"])
def test_correction_matches_oracle(oracle_mod, kind):
    scene = small_scene(kind)
    case = correction_case(oracle_mod, scene, 5)
    want = oracle_mod.correct_large_error_nodes(scene, **case)
    s, _ = make_solver(scene)
    t = {k: dev(v) for k, v in case.items() if k != "guides"}
    guides = [tuple(dev(a) for a in g) for g in case["guides"]]
    corr = s.correct_large_error_node(guides, t["united_error"], t["live_nodes"], t["node_knn"], t["node_weight"],
                                      t["live_vertex"], t["live_normal"], t["surfel_knn"], t["surfel_weight"],
                                      node_se3=t["node_se3"])
    torch.cuda.synchronize()
    gc = host(corr)
    # the same nodes chose a guide: identity corrections coincide exactly
    ident = np.all(want["correction"] == IDENT, axis=1)
    assert np.array_equal(np.all(gc == IDENT, axis=1), ident)
    assert (~ident).sum() > 5
    np.testing.assert_allclose(gc, want["correction"], atol=1e-5)
    np.testing.assert_allclose(host(t["node_se3"]), want["node_se3"], atol=1e-5)
    np.testing.assert_allclose(host(t["live_nodes"]), want["live_nodes"], atol=1e-5)
    np.testing.assert_allclose(host(t["live_vertex"]), want["live_vertex"], atol=1e-5)
    np.testing.assert_allclose(host(t["live_normal"]), want["live_normal"], atol=1e-5)
    # the corrected field is the solver's current warp field
    assert np.array_equal(s.get_array(abi.ARRAY_NODE_SE3), host(t["node_se3"]))
    s.close()


def test_correction_in_the_solver_field():
    """node_se3 = None corrects the solver's own warp field in place."""
    import oracle
    scene = small_scene("torso")
    case = correction_case(oracle, scene, 9)
    s, _ = make_solver(scene)
    t = {k: dev(v) for k, v in case.items() if k != "guides"}
    guides = [tuple(dev(a) for a in g) for g in case["guides"]]
    s.correct_large_error_node(guides, t["united_error"], t["live_nodes"], t["node_knn"], t["node_weight"],
                               t["live_vertex"], t["live_normal"], t["surfel_knn"], t["surfel_weight"])
    torch.cuda.synchronize()
    want = oracle.correct_large_error_nodes(scene, **case)
    np.testing.assert_allclose(s.get_array(abi.ARRAY_NODE_SE3), want["node_se3"], atol=1e-5)
    s.close()
