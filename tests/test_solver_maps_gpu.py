"""The solver-map renderer on the GPU against the oracle (bit-exact).

mvdr_render_solver_maps resolves the depth test with a 64-bit atomicMin of
(camera z bits, surfel id) per pixel; the oracle draws the surfels in order
with a strictly-less depth test. Both compute every float in the same order
without contraction, so the maps must be identical bit for bit, including
the clear values, for sized and one-pixel points and both cull modes. The
last test feeds the rendered maps to the solver and checks the solve against
the FP64 oracle run on the oracle's maps.
"""
import ctypes as C
import dataclasses

import numpy as np
import pytest
import torch

from conftest import rel_norm_error, small_scene
from multiviewdynrecon_b200 import abi, synth
from multiviewdynrecon_b200.solver import DeviceScene, NonRigidSolver
from multiviewdynrecon_b200.solver_maps import SolverMapRenderer, geometry_to_device

pytestmark = pytest.mark.gpu

MAPS = ("reference_vertex_map", "reference_normal_map", "live_vertex_map", "live_normal_map", "index_map",
        "normalized_rgb_map")


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import multiviewdynrecon_b200 as m
    m.lib()


def bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def render_gpu(scene, g, recent=True, sized_view0=False):
    r = SolverMapRenderer(scene.width, scene.height, scene.num_views, sized_view0=sized_view0)
    dg = geometry_to_device(g)
    if recent:
        r.draw_solver_maps_with_recent_observation(dg, 10.0, scene.views)
    else:
        r.draw_solver_maps_confident_observation(dg, 10.0, scene.views)
    torch.cuda.synchronize()
    return r


@pytest.mark.parametrize("kind", ["sphere", "torso", "body"])
@pytest.mark.parametrize("recent", [True, False])
@pytest.mark.parametrize("sized_view0", [False, True])
def test_render_bit_exact(oracle_mod, kind, recent, sized_view0):
    scene = small_scene(kind)
    g = synth.solver_map_geometry(scene)
    r = render_gpu(scene, g, recent, sized_view0)
    prm = abi.solver_map_params(scene.width, scene.height, time_threshold=3.0 if recent else -1.0)
    want = oracle_mod.render_solver_maps(g, prm, scene.views,
                                         sized=[sized_view0 and v == 0 for v in range(scene.num_views)])
    for v in range(scene.num_views):
        got = {k: t.cpu().numpy() for k, t in r.maps(v).items()}
        for k in MAPS:
            assert np.array_equal(bits(got[k]), bits(want[v][k])), (v, k)
        assert (want[v]["index_map"] != 0xFFFFFFFF).sum() > 100


def test_render_pitched_and_partial_outputs(oracle_mod):
    """A row pitch wider than the image and only the index map requested:
    the index map is the same and nothing is written past each row."""
    scene = small_scene("torso")
    g = synth.solver_map_geometry(scene)
    W, H, pitch = scene.width, scene.height, scene.width + 24
    dg = geometry_to_device(g)
    idx = torch.full((scene.num_views, H, pitch), 7, dtype=torch.int32, device="cuda")
    zb = torch.empty((scene.num_views, H, pitch), dtype=torch.int64, device="cuda")
    vs = (abi.SolverMapView * scene.num_views)()
    for v, view in enumerate(scene.views):
        vs[v] = abi.solver_map_view(view, {"index_map": idx[v].data_ptr(), "depth_index": zb[v].data_ptr()},
                                    pitch=pitch)
    geo = abi.surfel_geometry(scene.num_surfels, {k: t.data_ptr() for k, t in dg.items()})
    prm = abi.solver_map_params(W, H)
    import multiviewdynrecon_b200 as m
    m.check(m.lib().mvdr_render_solver_maps(C.byref(geo), C.byref(prm), vs, scene.num_views, None))
    torch.cuda.synchronize()
    want = oracle_mod.render_solver_maps(g, prm, scene.views)
    got = idx.cpu().numpy().view(np.uint32)
    for v in range(scene.num_views):
        assert np.array_equal(got[v, :, :W], want[v]["index_map"]), v
        assert np.all(got[v, :, W:] == 7)


def test_render_without_surfels():
    scene = small_scene("sphere")
    g = {k: a[:0] for k, a in synth.solver_map_geometry(scene).items()}
    r = SolverMapRenderer(scene.width, scene.height, 1)
    for t in (r.reference_vertex, r.live_normal, r.normalized_rgb):
        t.fill_(3.0)
    r.draw_solver_maps_with_recent_observation(geometry_to_device(g), 10.0, scene.views)
    torch.cuda.synchronize()
    assert torch.all(r.index == -1)
    for t in (r.reference_vertex, r.reference_normal, r.live_vertex, r.live_normal, r.normalized_rgb):
        assert torch.all(t == 0)


def test_render_is_deterministic():
    scene = small_scene("body")
    g = geometry_to_device(synth.solver_map_geometry(scene))
    r = SolverMapRenderer(scene.width, scene.height, scene.num_views, sized_view0=True)
    outs = []
    for _ in range(3):
        r.draw_solver_maps_with_recent_observation(g, 10.0, scene.views)
        torch.cuda.synchronize()
        outs.append([t.clone() for t in (r.index, r.reference_vertex, r.normalized_rgb)])
    for o in outs[1:]:
        for a, b in zip(outs[0], o):
            assert torch.equal(a, b)


@pytest.mark.parametrize("kind", ["torso", "body"])
def test_rendered_maps_drive_the_solve(oracle_mod, kind):
    """Renderer -> solver on the device: the solver reads the rendered maps
    in place; each Gauss-Newton increment matches the FP64 oracle run on the
    oracle's own maps (identical, by the bit-exact test) within the solver's
    tolerance."""
    scene = small_scene(kind)
    g = synth.solver_map_geometry(scene, warped=False)
    r = render_gpu(scene, g)
    prm = abi.solver_map_params(scene.width, scene.height)
    omaps = oracle_mod.render_solver_maps(g, prm, scene.views)
    views = [dataclasses.replace(view, reference_vertex_map=m["reference_vertex_map"],
                                 reference_normal_map=m["reference_normal_map"], index_map=m["index_map"],
                                 normalized_rgb_map=m["normalized_rgb_map"])
             for view, m in zip(scene.views, omaps)]
    oscene = dataclasses.replace(scene, views=views)
    cfg = abi.make_config(scene, precision=abi.PRECISION_MIXED)
    ds = r.bind(DeviceScene(scene))
    s = NonRigidSolver(cfg)
    s.set_solver_input(ds)
    s.build_index()
    o64 = oracle_mod.Oracle(oscene, cfg, fp64=True)
    o64.build_index()
    assert s.counts().dense_terms == o64.counts().dense_terms > 0
    for it in range(2):
        o64.set_node_se3(s.get_array(abi.ARRAY_NODE_SE3))
        s.gn_iteration(scene.pcg_iterations)
        torch.cuda.synchronize()
        o64.freeze(s.get_array(abi.ARRAY_TERM_JACOBIAN), s.get_array(abi.ARRAY_SMOOTH_TERMS))
        o64.eval_terms()
        o64.assemble()
        o64.pcg(scene.pcg_iterations)
        assert rel_norm_error(s.get_array(abi.ARRAY_INCREMENT), o64.get(abi.ARRAY_INCREMENT, as_double=True)) < 1e-4
    s.close()
