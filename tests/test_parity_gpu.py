"""Parity of the CUDA solver (through the C ABI) with the CPU oracle.

Bars:
* index and bin-block CSR structure: bit-exact;
* per-term Jacobians / residuals: maxRelativeError (sanity_check.cpp:50-73)
  below 1e-4 with a small cutoff; projected-pixel choices that differ because
  of FMA rounding at a threshold are counted and must stay below 0.1 %;
* JtJ diagonal / off-diagonal blocks and Jt r built from the same term data:
  below 1e-4;
* PCG increment: relative 2-norm error against the FP64 oracle below 1e-4 in
  mixed precision (2e-3 in plain FP32);
* warp-field update from the same increment: below 1e-4.
"""
import numpy as np
import pytest
import torch

from conftest import max_relative_error, rel_norm_error, small_scene
from multiviewdynrecon_b200 import abi
from multiviewdynrecon_b200.solver import BatchSolver, DeviceScene, NonRigidSolver, StreamedBatch

pytestmark = pytest.mark.gpu

KINDS = ["sphere", "sphere_rigid", "torso", "torso_rigid", "body"]
INDEX_ARRAYS = [abi.ARRAY_DENSE_PIXELS, abi.ARRAY_DENSE_KNN, abi.ARRAY_DENSE_KNN_WEIGHT,
                abi.ARRAY_FOREGROUND_PIXELS, abi.ARRAY_NODE2TERM_OFFSET, abi.ARRAY_NODE2TERM_INDEX,
                abi.ARRAY_HALF_NODEPAIR_KEY, abi.ARRAY_NODEPAIR_TERM_INDEX, abi.ARRAY_NODEPAIR_KEY,
                abi.ARRAY_NODEPAIR_TERM_RANGE, abi.ARRAY_BLKROW_OFFSET, abi.ARRAY_BINBLOCK_ROWPTR,
                abi.ARRAY_BINBLOCK_COLPTR]


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import multiviewdynrecon_b200 as m
    m.lib()


def make_gpu(scene, precision=abi.PRECISION_MIXED, mode=abi.MODE_MATERIALIZED, **kw):
    cfg = abi.make_config(scene, precision=precision, mode=mode, **kw)
    s = NonRigidSolver(cfg)
    s.set_solver_input(scene)
    return s, cfg


def bits(a):
    a = np.ascontiguousarray(a)
    return a.view(np.uint8)


@pytest.mark.parametrize("kind", KINDS)
def test_index_bit_exact(oracle_mod, kind):
    scene = small_scene(kind)
    g, cfg = make_gpu(scene)
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
        assert np.array_equal(bits(a), bits(b)), which


def _stage_compare(oracle_mod, scene, precision):
    g, cfg = make_gpu(scene, precision=precision)
    g.build_index()
    g.gn_iteration(scene.pcg_iterations)
    torch.cuda.synchronize()
    o = oracle_mod.Oracle(scene, cfg)
    o.build_index()
    o.eval_terms()
    return g, o, cfg


@pytest.mark.parametrize("kind", KINDS)
def test_term_evaluation(oracle_mod, kind):
    scene = small_scene(kind)
    g, o, _ = _stage_compare(oracle_mod, scene, abi.PRECISION_MIXED)
    gj, oj = g.get_array(abi.ARRAY_TERM_JACOBIAN), o.get(abi.ARRAY_TERM_JACOBIAN)
    assert gj.shape == oj.shape
    same = gj[:, 7].view(np.uint32) == oj[:, 7].view(np.uint32)
    assert (~same).sum() <= max(2, int(1e-3 * len(same)))
    scale = np.abs(oj[same, :7]).max() if same.any() else 1.0
    assert max_relative_error(gj[same, :7], oj[same, :7], 1e-6 * scale) < 1e-4
    gs, os_ = g.get_array(abi.ARRAY_SMOOTH_TERMS), o.get(abi.ARRAY_SMOOTH_TERMS)
    assert np.array_equal(gs[:, 6], os_[:, 6])
    assert max_relative_error(gs[:, :6], os_[:, :6], 1e-6) < 1e-4
    gw, ow = g.get_array(abi.ARRAY_WARPED_CORRESPONDENCE), o.get(abi.ARRAY_WARPED_CORRESPONDENCE)
    assert max_relative_error(gw, ow, 1e-6) < 1e-4


@pytest.mark.parametrize("flags", [abi.COMPAT_REF_FOREGROUND_FRAME,
                                   abi.COMPAT_REF_FOREGROUND_FRAME | abi.COMPAT_REF_VIEW_LOOKUP])
@pytest.mark.parametrize("precision", [abi.PRECISION_MIXED, abi.PRECISION_FP32])
def test_term_evaluation_reference_compat_forms(oracle_mod, flags, precision):
    """The reference's own forms of the foreground term (vertex warped in its
    camera's frame) and of the pixel-to-view lookup: the kernel's terms equal
    the oracle's, and its foreground terms equal an independent restatement of
    density_map_jacobian.cuh:12-79 (with the pixel's own view)."""
    from image_terms import foreground_terms
    scene = small_scene("torso")
    g, cfg = make_gpu(scene, precision=precision, compat_flags=flags)
    g.build_index()
    g.gn_iteration(scene.pcg_iterations)
    torch.cuda.synchronize()
    o = oracle_mod.Oracle(scene, cfg)
    o.build_index()
    o.eval_terms()
    gj, oj = g.get_array(abi.ARRAY_TERM_JACOBIAN), o.get(abi.ARRAY_TERM_JACOBIAN)
    assert gj.shape == oj.shape
    same = gj[:, 7].view(np.uint32) == oj[:, 7].view(np.uint32)
    assert (~same).sum() <= max(2, int(1e-3 * len(same)))
    scale = np.abs(oj[same, :7]).max()
    assert max_relative_error(gj[same, :7], oj[same, :7], 1e-6 * scale) < 1e-4
    if not flags & abi.COMPAT_REF_VIEW_LOOKUP:
        Td = g.counts().dense_terms
        want = foreground_terms(scene, g.get_array(abi.ARRAY_FOREGROUND_PIXELS), frame0=False)
        got = gj[Td:].astype(np.float64)
        gp = np.ascontiguousarray(gj[Td:, 7]).view(np.uint32).astype(np.int64)
        gp = np.where(gp == abi.MVDR_INVALID_INDEX, -1, gp)
        ok = gp == want[:, 7].astype(np.int64)
        assert ok.mean() > 0.999
        assert max_relative_error(got[ok, :7], want[ok, :7], 1e-6 * np.abs(want[:, :7]).max()) < 1e-4


@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("precision", [abi.PRECISION_MIXED, abi.PRECISION_FP32])
def test_assembly_and_pcg(oracle_mod, kind, precision):
    scene = small_scene(kind)
    g, o, cfg = _stage_compare(oracle_mod, scene, precision)
    # the oracle assembles from the GPU's own term data
    o.set_term_data(g.get_array(abi.ARRAY_TERM_JACOBIAN), g.get_array(abi.ARRAY_SMOOTH_TERMS),
                    g.get_array(abi.ARRAY_WARPED_CORRESPONDENCE))
    o.assemble()
    for which in (abi.ARRAY_DIAG_BLOCKS, abi.ARRAY_JTR, abi.ARRAY_OFFDIAG_BLOCKS):
        a, b = g.get_array(which), o.get(which, as_double=True)
        assert a.shape == b.shape, which
        assert max_relative_error(a, b, 1e-6 * np.abs(b).max()) < 1e-4, which
    bb_g, bb_o = g.get_array(abi.ARRAY_BINBLOCK_DATA), o.get(abi.ARRAY_BINBLOCK_DATA, as_double=True)
    assert max_relative_error(bb_g, bb_o, 1e-6 * np.abs(bb_o).max()) < 1e-4
    # preconditioner: M D = I per block, to the accuracy the block's condition
    # number allows in the arithmetic used (float Gauss-Jordan or double
    # Cholesky rounded to float for the export)
    D = g.get_array(abi.ARRAY_DIAG_BLOCKS).reshape(-1, 6, 6).astype(np.float64)
    M = g.get_array(abi.ARRAY_PRECONDITIONER).reshape(-1, 6, 6).astype(np.float64)
    eye_err = np.abs(M @ D - np.eye(6)).max(axis=(1, 2))
    cond = np.linalg.cond(D)
    bound = (200.0 if precision == abi.PRECISION_FP32 else 20.0) * cond * 2.0 ** -24 + 1e-6
    assert (eye_err <= bound).all(), (eye_err / bound).max()
    # PCG increment vs the FP64 oracle on the same system
    o64 = oracle_mod.Oracle(scene, cfg, fp64=True)
    o64.build_index()
    o64.eval_terms()
    o64.set_term_data(g.get_array(abi.ARRAY_TERM_JACOBIAN), g.get_array(abi.ARRAY_SMOOTH_TERMS),
                      g.get_array(abi.ARRAY_WARPED_CORRESPONDENCE))
    o64.assemble()
    o64.pcg(scene.pcg_iterations)
    x64 = o64.get(abi.ARRAY_INCREMENT, as_double=True)
    xg = g.get_array(abi.ARRAY_INCREMENT)
    tol = 1e-4 if precision == abi.PRECISION_MIXED else 2e-3
    assert rel_norm_error(xg, x64) < tol
    # update from the GPU's increment
    o.set_increment(xg.reshape(-1))
    o.update()
    assert max_relative_error(g.get_array(abi.ARRAY_NODE_SE3), o.get(abi.ARRAY_NODE_SE3), 1e-6) < 1e-4


@pytest.mark.parametrize("kind", ["sphere", "torso", "body"])
def test_solve_vs_fp64_oracle(oracle_mod, kind):
    """Every Gauss-Newton increment of the mixed-precision solve against the
    FP64 oracle run from the same warp field, with the discrete projection and
    validity choices taken from the GPU run."""
    scene = small_scene(kind)
    g, cfg = make_gpu(scene, precision=abi.PRECISION_MIXED)
    g.build_index()
    o64 = oracle_mod.Oracle(scene, cfg, fp64=True)
    o64.build_index()
    energies = []
    for it in range(scene.gn_iterations):
        # the oracle restarts every iteration from the GPU's warp field, so
        # each increment is compared on the same linearisation
        o64.set_node_se3(g.get_array(abi.ARRAY_NODE_SE3))
        g.gn_iteration(scene.pcg_iterations)
        torch.cuda.synchronize()
        jr, sm = g.get_array(abi.ARRAY_TERM_JACOBIAN), g.get_array(abi.ARRAY_SMOOTH_TERMS)
        o64.freeze(jr, sm)
        o64.eval_terms()
        o64.assemble()
        energies.append((g.energy(), o64.energy()))
        o64.pcg(scene.pcg_iterations)
        x64 = o64.get(abi.ARRAY_INCREMENT, as_double=True)
        xg = g.get_array(abi.ARRAY_INCREMENT)
        assert rel_norm_error(xg, x64) < 1e-4, it
    for eg, eo in energies:
        assert abs(eg - eo) <= 1e-4 * abs(eo)
    assert energies[-1][0] < energies[0][0]


@pytest.mark.parametrize("kind", ["sphere", "torso"])
def test_trajectory_vs_fp64_oracle(oracle_mod, kind):
    """Whole solves, each side on its own trajectory: the final energies of the
    mixed-precision GPU solve and the FP64 oracle agree to 1e-3."""
    scene = small_scene(kind)
    g, cfg = make_gpu(scene, precision=abi.PRECISION_MIXED)
    g.solve_non_rigid_alignment(scene.gn_iterations, scene.pcg_iterations)
    g.gn_iteration(1)  # evaluates the energy at the solved warp field
    eg = g.energy()
    o64 = oracle_mod.Oracle(scene, cfg, fp64=True)
    o64.solve(scene.gn_iterations, scene.pcg_iterations)
    o64.eval_terms()
    o64.assemble()
    eo = o64.energy()
    assert abs(eg - eo) <= 1e-3 * eo, (eg, eo)


@pytest.mark.parametrize("kind", ["sphere", "torso"])
def test_matrix_free_equals_materialized(oracle_mod, kind):
    scene = small_scene(kind)
    a, _ = make_gpu(scene, mode=abi.MODE_MATERIALIZED)
    b, _ = make_gpu(scene, mode=abi.MODE_MATRIX_FREE)
    for s in (a, b):
        s.build_index()
        s.gn_iteration(scene.pcg_iterations)
    torch.cuda.synchronize()
    x = torch.randn(6 * scene.num_nodes, device="cuda")
    ya, yb = a.apply_jtj(x), b.apply_jtj(x)
    assert rel_norm_error(yb.cpu().numpy(), ya.cpu().numpy()) < 1e-5
    assert rel_norm_error(b.get_array(abi.ARRAY_INCREMENT), a.get_array(abi.ARRAY_INCREMENT)) < 1e-4
    # and both equal the oracle's assembled operator
    o = oracle_mod.Oracle(scene, abi.make_config(scene), fp64=True)
    o.build_index()
    o.eval_terms()
    o.set_term_data(a.get_array(abi.ARRAY_TERM_JACOBIAN), a.get_array(abi.ARRAY_SMOOTH_TERMS),
                    a.get_array(abi.ARRAY_WARPED_CORRESPONDENCE))
    o.assemble()
    yo = o.apply_jtj(x.cpu().numpy().astype(np.float64))
    assert rel_norm_error(ya.cpu().numpy(), yo) < 1e-5


def test_batch_graph_and_determinism():
    """Uneven instances in one batch give bit-identical results to solving them
    one by one; the graph replay equals direct launches; reruns are identical."""
    scenes = [small_scene("torso"), small_scene("sphere"), small_scene("body")]
    n = max(s.num_nodes for s in scenes)
    caps = dict(max_nodes=n, max_views=3, width=192, height=120, use_foreground=True, use_feature=True,
                use_cross_view=True, max_surfels=max(s.num_surfels for s in scenes),
                max_feature_terms=max(s.feature.count for s in scenes),
                max_cross_terms=max(s.cross_view.count for s in scenes))

    def pad(scene):
        # bring every scene to the batch image size (zero / invalid padding)
        from copy import copy
        s2 = copy(scene)
        views = []
        for v in scene.views:
            def p(a, fill):
                out = np.full((120, 192) + a.shape[2:], fill, a.dtype)
                out[:a.shape[0], :a.shape[1]] = a
                return out
            from dataclasses import replace
            views.append(replace(v, reference_vertex_map=p(v.reference_vertex_map, 0),
                                 reference_normal_map=p(v.reference_normal_map, 0),
                                 index_map=p(v.index_map, 0xFFFFFFFF),
                                 vertex_confidence_map=p(v.vertex_confidence_map, 0),
                                 normal_radius_map=p(v.normal_radius_map, 0),
                                 filtered_foreground_mask=p(v.filtered_foreground_mask, 0),
                                 foreground_mask_gradient=p(v.foreground_mask_gradient, 0)))
        s2.views = views
        s2.width, s2.height = 192, 120
        return s2

    padded = [pad(s) for s in scenes]
    cfg = abi.make_config(None, **caps)
    batch = BatchSolver(cfg, len(padded))
    dev = [DeviceScene(s) for s in padded]

    def run(use_graph):
        # binding the inputs resets every warp field to its initial value
        for i, ds in enumerate(dev):
            batch.set_input(i, ds)
        batch.solve(3, 10, use_graph=use_graph)
        return [batch.node_se3(i).cpu().numpy() for i in range(len(padded))]

    direct = run(False)
    graph = run(True)
    again = run(True)
    for i, s in enumerate(padded):
        single = NonRigidSolver(cfg)
        single.set_solver_input(s)
        single.solve_non_rigid_alignment(3, 10)
        ref = single.solved_node_se3().cpu().numpy()
        assert np.array_equal(bits(direct[i]), bits(ref)), i
        assert np.array_equal(bits(graph[i]), bits(ref)), i
        assert np.array_equal(bits(again[i]), bits(ref)), i


def test_host_inputs_match_device_inputs():
    scene = small_scene("torso")
    a, cfg = make_gpu(scene)
    a.solve_non_rigid_alignment(2, 10)
    b = NonRigidSolver(cfg)
    b.set_solver_input_host(DeviceScene(scene, pin=True))
    b.solve_non_rigid_alignment(2, 10)
    assert np.array_equal(bits(a.solved_node_se3().cpu().numpy()), bits(b.solved_node_se3().cpu().numpy()))


def test_capacity_overflow_is_reported():
    from multiviewdynrecon_b200 import MvdrError
    scene = small_scene("sphere")
    cfg = abi.make_config(scene)
    cfg.max_terms_per_node = 16  # far below the real per-node term count
    s = NonRigidSolver(cfg)
    s.set_solver_input(scene)
    s.solve_non_rigid_alignment(1, 2)
    with pytest.raises(MvdrError) as e:
        s.solved_node_se3()
    assert e.value.status == abi.MVDR_ECAPACITY
    # the context stays usable
    ok, _ = make_gpu(scene)
    ok.solve_non_rigid_alignment(1, 2)
    ok.solved_node_se3()


def test_async_warp_field_copy_matches_checked_copy():
    """mvdr_copy_node_se3_async enqueues the same warp field that the checked
    mvdr_get_node_se3 returns, into pinned host memory on a side stream."""
    scene = small_scene("torso")
    g, _ = make_gpu(scene)
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        g.solve_non_rigid_alignment(scene.gn_iterations, scene.pcg_iterations, stream=stream)
        out = torch.empty((scene.num_nodes, 8), dtype=torch.float32, pin_memory=True)
        g.solved_node_se3_async(out, stream=stream)
    stream.synchronize()
    assert g.counts(stream=stream).error_flags == 0
    ref = g.solved_node_se3(stream=stream).cpu()
    assert torch.equal(out, ref)


@pytest.mark.parametrize("mode", [abi.MODE_MATERIALIZED, abi.MODE_MATRIX_FREE])
def test_adjoint_products_vs_finite_differences(oracle_mod, mode):
    """Jt r and JtJ p of the mixed-precision solver (materialised BSR and the
    matrix-free adjoint pair) against central finite differences (step 2e-4
    per twist coordinate, FP64 oracle residuals with the GPU's pixel and
    validity decisions) on 64 random nodes. The warp field is uniform, where
    the skinning Jacobian model is exact."""
    from fd_adjoint import DAMPING, fd_adjoint_reference, fd_config, random_coords, uniform_field
    scene = uniform_field(small_scene("torso"))
    cfg = fd_config(scene, precision=abi.PRECISION_MIXED, mode=mode)
    g = NonRigidSolver(cfg)
    g.set_solver_input(scene)
    g.build_index()
    g.gn_iteration(1)
    torch.cuda.synchronize()
    rng = np.random.default_rng(22)
    coords = random_coords(rng, scene.num_nodes)
    p = rng.normal(size=len(coords)).astype(np.float32)
    b_fd, jtjp_fd, _ = fd_adjoint_reference(oracle_mod, scene, cfg, coords, p.astype(np.float64),
                                            g.get_array(abi.ARRAY_TERM_JACOBIAN),
                                            g.get_array(abi.ARRAY_SMOOTH_TERMS))
    b = g.get_array(abi.ARRAY_JTR).reshape(-1, 6).astype(np.float64)
    assert rel_norm_error(np.array([b[n, c] for n, c in coords]), b_fd) < 1e-4
    x = np.zeros(6 * scene.num_nodes, np.float32)
    for (n, c), v in zip(coords, p):
        x[6 * n + c] += v
    y = g.apply_jtj(torch.from_numpy(x).cuda()).cpu().numpy().astype(np.float64)
    y_g = np.array([y[6 * n + c] - DAMPING * x[6 * n + c] for n, c in coords])
    assert rel_norm_error(y_g, jtjp_fd) < 1e-4


# FP32: 5 GN x 15 PCG iterations in float amplify a reordered sum to about
# 1e-2 of the increment (measured between two tile shapes)
@pytest.mark.parametrize("precision,tol", [(abi.PRECISION_MIXED, 1e-5), (abi.PRECISION_FP32, 3e-2)])
def test_every_spmv_shape_solves_the_same_system(precision, tol):
    """Every SpMV tile shape gives the first shape's increments up to the
    order of its sums, and reruns of one shape are bit-identical."""
    scene = small_scene("torso")
    cfg = abi.make_config(scene, precision=precision)
    b = BatchSolver(cfg, 2)
    results = []
    for k in list(range(abi.NUM_SPMV_SHAPES)) + [abi.NUM_SPMV_SHAPES - 1]:
        b.set_spmv_shape(k)
        for i in range(2):
            b.set_input(i, scene)
        b.solve(scene.gn_iterations, scene.pcg_iterations)
        torch.cuda.synchronize()
        results.append([b.instance(i).get_array(abi.ARRAY_INCREMENT) for i in range(2)])
    for k, res in enumerate(results[:-1]):
        for i in range(2):
            assert rel_norm_error(res[i], results[0][i]) < tol, (abi.SPMV_SHAPES[k], i)
    for i in range(2):
        assert np.array_equal(results[-1][i], results[-2][i])


@pytest.mark.parametrize("precision,tol", [(abi.PRECISION_MIXED, 1e-5), (abi.PRECISION_FP32, 3e-2)])
def test_persistent_pcg_solves_the_same_system(precision, tol):
    """The persistent PCG (one cooperative launch per PCG solve, instances of
    uneven size on their own CTAs and barriers) gives the launched PCG's
    increments up to the grouping of its dot sums; reruns are bit-identical."""
    scenes = [small_scene("torso"), small_scene("sphere")]  # both 160 x 120
    caps = dict(max_nodes=max(s.num_nodes for s in scenes), max_views=3, width=160, height=120,
                use_foreground=True, use_feature=True, use_cross_view=True,
                max_surfels=max(s.num_surfels for s in scenes),
                max_feature_terms=max(s.feature.count for s in scenes),
                max_cross_terms=max(s.cross_view.count for s in scenes))
    cfg = abi.make_config(None, precision=precision, **caps)
    ref, per = BatchSolver(cfg, 2), BatchSolver(cfg, 2)
    per.set_pcg_persistent(True)
    out = {}
    for name, b in (("ref", ref), ("per", per), ("per2", per)):
        for i, s in enumerate(scenes):
            b.set_input(i, s)
        b.solve(3, 10)
        torch.cuda.synchronize()
        out[name] = [b.instance(i).get_array(abi.ARRAY_INCREMENT) for i in range(2)]
        assert all(b.instance(i).counts().error_flags == 0 for i in range(2))
    for i in range(2):
        assert rel_norm_error(out["per"][i], out["ref"][i]) < tol
        assert np.array_equal(out["per"][i], out["per2"][i])


def test_streamed_batch_equals_one_batch():
    """A batch split into lanes of concurrent graphs on their own streams
    (two lanes of 2 and 1 instances here) gives every instance's warp field
    bit for bit as one batch of all instances does; results read on the
    caller's stream after solve() see the lanes' work, also on replays."""
    scenes = [small_scene("torso"), small_scene("sphere"), small_scene("torso")]  # all 160 x 120
    caps = dict(max_nodes=max(s.num_nodes for s in scenes), max_views=3, width=160, height=120,
                use_foreground=True, use_feature=True, use_cross_view=True,
                max_surfels=max(s.num_surfels for s in scenes),
                max_feature_terms=max(s.feature.count for s in scenes),
                max_cross_terms=max(s.cross_view.count for s in scenes))
    cfg = abi.make_config(None, **caps)
    dev = [DeviceScene(s) for s in scenes]
    one, lanes = BatchSolver(cfg, 3), StreamedBatch(cfg, 3, lanes=2)
    assert lanes.sizes == [2, 1] and lanes.lane_of(2) == (1, 0)
    caller = torch.cuda.Stream()
    out = {}
    for name, b, graph in (("one", one, True), ("direct", lanes, False), ("graph", lanes, True),
                           ("again", lanes, True)):
        with torch.cuda.stream(caller):
            for i, ds in enumerate(dev):
                b.set_input(i, ds, stream=caller)
            b.solve(3, 10, use_graph=graph, stream=caller)
            out[name] = [b.node_se3(i, stream=caller) for i in range(3)]
        caller.synchronize()
        out[name] = [t.cpu().numpy() for t in out[name]]
    for name in ("direct", "graph", "again"):
        for i in range(3):
            assert np.array_equal(bits(out[name][i]), bits(out["one"][i])), (name, i)
    assert all(lanes.instance(i).counts().error_flags == 0 for i in range(3))
    lanes.close()
    one.close()


def test_autotuned_spmv_shape_solves_the_same_system():
    """mvdr_batch_autotune picks one of the SpMV tile shapes; solves with the
    chosen shape agree with the default shape's (only the order of the row
    sums differs)."""
    scene = small_scene("torso")
    cfg = abi.make_config(scene, precision=abi.PRECISION_MIXED)
    ref = BatchSolver(cfg, 2)
    tuned = BatchSolver(cfg, 2)
    for b in (ref, tuned):
        for i in range(2):
            b.set_input(i, scene)
    shape, times = tuned.autotune()
    assert shape in abi.SPMV_SHAPES and len(times) == abi.NUM_SPMV_SHAPES and min(times) > 0
    for i in range(2):
        tuned.set_input(i, scene)  # the autotuner ran one iteration
    for b in (ref, tuned):
        b.solve(scene.gn_iterations, scene.pcg_iterations)
    torch.cuda.synchronize()
    for i in range(2):
        xa = ref.instance(i).get_array(abi.ARRAY_INCREMENT)
        xb = tuned.instance(i).get_array(abi.ARRAY_INCREMENT)
        assert rel_norm_error(xb, xa) < 1e-5


def test_matrix_free_stage_only_in_matrix_free_mode():
    """mvdr_batch_enqueue_stage(MVDR_STAGE_MATRIX_FREE) runs one matrix-free
    PCG product on the state of the last solve; its J.d scratch exists only in
    the matrix-free mode, so the materialised mode rejects it with
    MVDR_EINVAL and launches nothing."""
    import ctypes as C
    from multiviewdynrecon_b200 import lib
    scene = small_scene("torso")
    for mode, want in ((abi.MODE_MATRIX_FREE, abi.MVDR_OK), (abi.MODE_MATERIALIZED, abi.MVDR_EINVAL)):
        b = BatchSolver(abi.make_config(scene, mode=mode), 1)
        b.set_input(0, scene)
        b.solve(1, 5)
        torch.cuda.synchronize()
        k0 = lib().mvdr_kernel_launch_count()
        st = lib().mvdr_batch_enqueue_stage(b.h, abi.STAGE_MATRIX_FREE,
                                            C.c_void_p(torch.cuda.current_stream().cuda_stream))
        torch.cuda.synchronize()
        assert st == want
        assert lib().mvdr_kernel_launch_count() - k0 == (2 if want == abi.MVDR_OK else 0)
        assert b.instance(0).counts().error_flags == 0
        b.close()


@pytest.mark.parametrize("flags", [0, abi.COMPAT_REF_FOREGROUND_FRAME])
@pytest.mark.parametrize("precision", [abi.PRECISION_MIXED, abi.PRECISION_FP32])
def test_density_term_parity(oracle_mod, flags, precision):
    """The density (colour) term of every dense pixel: the kernel's records
    equal the oracle's and an independent restatement of
    computeDensityMapJacobian (DensityForegroundJacobianResidual.cu:41-91)."""
    from image_terms import density_terms
    scene = small_scene("torso")
    g, cfg = make_gpu(scene, precision=precision, compat_flags=flags, use_density=True, num_global_iterations=0)
    g.build_index()
    g.gn_iteration(scene.pcg_iterations)
    torch.cuda.synchronize()
    o = oracle_mod.Oracle(scene, cfg)
    o.build_index()
    o.eval_terms()
    gd, od = g.get_array(abi.ARRAY_DENSITY_JACOBIAN), o.get(abi.ARRAY_DENSITY_JACOBIAN)
    assert gd.shape == od.shape and len(gd) == g.counts().dense_terms
    same = gd[:, 7].view(np.uint32) == od[:, 7].view(np.uint32)
    assert (~same).sum() <= max(2, int(1e-3 * len(same)))
    scale = np.abs(od[same, :7]).max()
    assert max_relative_error(gd[same, :7], od[same, :7], 1e-6 * scale) < 1e-4
    want = density_terms(scene, g.get_array(abi.ARRAY_DENSE_PIXELS), frame0=not flags)
    gp = np.ascontiguousarray(gd[:, 7]).view(np.uint32).astype(np.int64)
    gp = np.where(gp == abi.MVDR_INVALID_INDEX, -1, gp)
    ok = gp == want[:, 7].astype(np.int64)
    assert ok.mean() > 0.999
    assert max_relative_error(gd[ok, :7].astype(np.float64), want[ok, :7],
                              1e-6 * np.abs(want[:, :7]).max()) < 1e-4


@pytest.mark.parametrize("mode", [abi.MODE_MATERIALIZED, abi.MODE_MATRIX_FREE])
def test_density_solve_vs_fp64_oracle(oracle_mod, mode):
    """Gauss-Newton increments with the density term active (lambda 1e-2 from
    the first iteration) against the FP64 oracle from the same warp field, with
    the GPU's pixel decisions for both image terms."""
    scene = small_scene("torso")
    g, cfg = make_gpu(scene, mode=mode, use_density=True, num_global_iterations=0)
    g.build_index()
    o64 = oracle_mod.Oracle(scene, cfg, fp64=True)
    o64.build_index()
    for it in range(3):
        o64.set_node_se3(g.get_array(abi.ARRAY_NODE_SE3))
        g.gn_iteration(scene.pcg_iterations)
        torch.cuda.synchronize()
        o64.freeze(g.get_array(abi.ARRAY_TERM_JACOBIAN), g.get_array(abi.ARRAY_SMOOTH_TERMS),
                   g.get_array(abi.ARRAY_DENSITY_JACOBIAN))
        o64.eval_terms()
        o64.assemble()
        assert abs(g.energy() - o64.energy()) <= 1e-4 * abs(o64.energy()), it
        o64.pcg(scene.pcg_iterations)
        o64.update()
        assert rel_norm_error(g.get_array(abi.ARRAY_INCREMENT), o64.get(abi.ARRAY_INCREMENT, as_double=True)) < 1e-4, it
    assert g.counts().error_flags == 0
