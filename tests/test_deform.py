"""The post-solve deformation path on the CPU: the oracle's restatement of
SurfelNodeDeformer (core/Geometry/SurfelNodeDeformer.cu), the node alignment
error (core/NonRigidSolver/DenseDepthAlignmentError.cu:16-238) and the
large-error correction (core/NonRigidSolver/NonRigidSolver.cu:93-227),
checked against known answers and an independent numpy restatement; and the
C ABI's argument checks of the four entry points (no GPU)."""
import ctypes as C

import numpy as np
import pytest

from conftest import small_scene
from multiviewdynrecon_b200 import abi, synth

IDENT = np.array([0, 0, 0, 1, 0, 0, 0, 0], np.float32)


def surfels(scene):
    g = synth.solver_map_geometry(scene, warped=False)
    return g["reference_vertex_confid"], g["reference_normal_radius"]


def test_translation_field_moves_by_the_translation(oracle_mod):
    scene = small_scene("sphere")
    t = np.array([0.01, -0.02, 0.03], np.float32)
    field = np.tile(IDENT, (scene.num_nodes, 1))
    field[:, 4:7] = t / 2  # dual part: (t / 2, 0) * q0 with q0 the identity
    v, n = surfels(scene)
    lv, ln, _ = oracle_mod.forward_warp(field, scene.surfel_knn, scene.surfel_knn_weight, v, n)
    # the blend of equal unit quaternions normalises back to them only up to
    # rounding of the weight sum; rotation and translation stay exact to 1 ulp
    np.testing.assert_allclose(lv[:, :3], v[:, :3] + t, atol=2e-7, rtol=0)
    np.testing.assert_allclose(ln[:, :3], n[:, :3], atol=2e-7, rtol=0)
    assert np.array_equal(lv[:, 3], v[:, 3]) and np.array_equal(ln[:, 3], n[:, 3])


def test_forward_matches_numpy_and_inverse_undoes_it(oracle_mod):
    scene = small_scene("torso")
    v, n = surfels(scene)
    nk, nw = synth.node_skinning(scene)
    nodes = synth.node_views(scene)
    lv, ln, live = oracle_mod.forward_warp(scene.node_se3, scene.surfel_knn, scene.surfel_knn_weight, v, n, nk, nw,
                                           nodes)
    R, t = synth.blend_warp(scene.node_se3, scene.surfel_knn, scene.surfel_knn_weight)
    np.testing.assert_allclose(lv[:, :3], np.einsum("sij,sj->si", R, v[:, :3]) + t, atol=2e-6)
    np.testing.assert_allclose(ln[:, :3], np.einsum("sij,sj->si", R, n[:, :3]), atol=2e-6)
    Rn, tn = synth.blend_warp(scene.node_se3, nk, nw)
    np.testing.assert_allclose(live[:, :3], np.einsum("sij,sj->si", Rn, nodes[:, :3]) + tn, atol=2e-6)
    assert np.array_equal(live[:, 3], nodes[:, 3])
    rv, rn = oracle_mod.inverse_warp(scene.node_se3, scene.surfel_knn, scene.surfel_knn_weight, lv, ln)
    np.testing.assert_allclose(rv, v, atol=1e-6)
    np.testing.assert_allclose(rn, n, atol=1e-6)


def test_inverse_with_correction_transform(oracle_mod):
    scene = small_scene("sphere")
    v, n = surfels(scene)
    rng = np.random.default_rng(3)
    S = len(v)
    Rc = synth.rodrigues_batch(rng.normal(0, 0.05, (S, 3)))
    tc = rng.normal(0, 0.01, (S, 3))
    correct = np.concatenate([np.transpose(Rc, (0, 2, 1)).reshape(S, 9), tc], 1).astype(np.float32)
    # live = warp(correct * canonical): the inverse with `correct` recovers canonical
    cv = np.einsum("sij,sj->si", Rc, v[:, :3]) + tc
    cn = np.einsum("sij,sj->si", Rc, n[:, :3])
    lv, ln, _ = oracle_mod.forward_warp(scene.node_se3, scene.surfel_knn, scene.surfel_knn_weight,
                                        np.concatenate([cv, v[:, 3:]], 1), np.concatenate([cn, n[:, 3:]], 1))
    rv, rn = oracle_mod.inverse_warp(scene.node_se3, scene.surfel_knn, scene.surfel_knn_weight, lv, ln, correct)
    np.testing.assert_allclose(rv, v, atol=2e-6)
    np.testing.assert_allclose(rn, n, atol=2e-6)


def test_bad_knn_gives_nan(oracle_mod):
    scene = small_scene("sphere")
    v, n = surfels(scene)
    knn = scene.surfel_knn.copy()
    knn[5, 2] = scene.num_nodes
    lv, ln, _ = oracle_mod.forward_warp(scene.node_se3, knn, scene.surfel_knn_weight, v, n)
    assert np.all(np.isnan(lv[5, :3])) and np.all(np.isnan(ln[5, :3])) and lv[5, 3] == v[5, 3]
    assert np.all(np.isfinite(np.delete(lv, 5, 0)))


# --------------------------------------------------------------------------
# node alignment error: an independent float64 numpy restatement
# --------------------------------------------------------------------------

def _rows(m):
    m = np.asarray(m, np.float64)
    return m[:9].reshape(3, 3).T, m[9:12]


def numpy_node_error(scene, field, threshold=0.2):
    N, W, H = scene.num_nodes, scene.width, scene.height
    acc_e, acc_w = np.zeros(N), np.zeros(N)
    maps = []
    for view in scene.views:
        Rw, tw = _rows(view.world2camera)
        Ri, ti = _rows(view.initial_camera_se3)
        idx = view.index_map.reshape(-1)
        pix = np.nonzero(idx != 0xFFFFFFFF)[0]
        s = idx[pix]
        knn, w = scene.surfel_knn[s], scene.surfel_knn_weight[s].astype(np.float64)
        R, t = synth.blend_warp(field, knn, w)
        rv = view.reference_vertex_map.reshape(-1, 4)[pix, :3].astype(np.float64)
        rn = view.reference_normal_map.reshape(-1, 4)[pix, :3].astype(np.float64)
        cv, cn = rv @ Ri.T + ti, rn @ Ri.T
        wv, wn = np.einsum("sij,sj->si", R, cv) + t, np.einsum("sij,sj->si", R, cn)
        c1 = ((wv @ Rw.T + tw) - ti) @ Ri
        n1 = (wn @ Rw.T) @ Ri
        cx, cy, fx, fy = view.intrinsic.astype(np.float64)
        ix = np.rint(c1[:, 0] / c1[:, 2] * fx + cx).astype(np.int64)
        iy = np.rint(c1[:, 1] / c1[:, 2] * fy + cy).astype(np.int64)
        obs_v = view.vertex_confidence_map.astype(np.float64)
        obs_n = view.normal_radius_map.astype(np.float64)
        err = np.full(len(pix), 0.1)
        found = np.zeros(len(pix), bool)
        for dy in (-1, 0, 1):
            for dx in (-1, 0, 1):
                x, y = ix + dx, iy + dy
                inside = (x >= 0) & (y >= 0) & (x < W) & (y < H)
                xc, yc = np.clip(x, 0, W - 1), np.clip(y, 0, H - 1)
                dv = np.where(inside[:, None], obs_v[yc, xc, :3], 0.0)
                dn = np.where(inside[:, None], obs_n[yc, xc, :3], 0.0)
                nz = ~np.all(np.abs(dv) < 1e-3, axis=1)
                found |= nz & ((n1 * dn).sum(1) > 0.7)
                err = np.minimum(err, np.abs(c1 - dv).sum(1))
        inside = (ix >= 0) & (iy >= 0) & (ix < W) & (iy < H)
        fg = np.where(inside, view.filtered_foreground_mask[np.clip(iy, 0, H - 1), np.clip(ix, 0, W - 1)], 0.0)
        err = np.where(found, err, np.where(fg < 0.9, 0.03 * fg, 0.1))
        m = np.zeros(H * W)
        m[pix] = err
        maps.append(m.reshape(H, W))
        big = err > 1e-6
        for k in range(4):
            np.add.at(acc_e, knn[big, k], w[big, k] * err[big])
            np.add.at(acc_w, knn[big, k], w[big, k])
    united = (acc_e / (acc_w + 1e-4)) / 0.1
    mark = united > threshold
    none = acc_e < 1e-10
    united[none], mark[none] = 1.0, True
    return dict(accumulated_error=acc_e, accumulated_weight=acc_w, united_error=united, large_error_mark=mark,
                alignment_error_map=maps)


@pytest.mark.parametrize("kind", ["sphere", "torso", "body"])
@pytest.mark.parametrize("field", ["identity", "perturbed"])
def test_node_error_matches_numpy(oracle_mod, kind, field):
    scene = small_scene(kind)
    f = np.tile(IDENT, (scene.num_nodes, 1)) if field == "identity" else scene.node_se3
    got = oracle_mod.node_error(scene, f, maps=True)
    want = numpy_node_error(scene, f)
    for v in range(scene.num_views):
        a, b = got["alignment_error_map"][v], want["alignment_error_map"][v]
        close = np.abs(a - b) <= 1e-5
        # a projection on a rounding boundary may pick the neighbouring window
        assert close.mean() > 0.999, (v, close.mean())
    np.testing.assert_allclose(got["accumulated_weight"], want["accumulated_weight"], rtol=1e-3, atol=1e-3)
    np.testing.assert_allclose(got["united_error"], want["united_error"], rtol=2e-2, atol=2e-3)
    assert np.mean(got["large_error_mark"].astype(bool) == want["large_error_mark"]) > 0.99


def test_node_error_is_larger_for_the_perturbed_field(oracle_mod):
    scene = small_scene("torso")
    e0 = oracle_mod.node_error(scene, np.tile(IDENT, (scene.num_nodes, 1)))["united_error"]
    e1 = oracle_mod.node_error(scene, scene.node_se3)["united_error"]
    assert e1.mean() > 2 * e0.mean()


def test_node_error_map_interpolates_node_errors(oracle_mod):
    scene = small_scene("sphere")
    got = oracle_mod.node_error(scene, scene.node_se3, maps=True)
    view = scene.views[0]
    ys, xs = np.nonzero(view.index_map != 0xFFFFFFFF)
    s = view.index_map[ys, xs]
    unit = got["accumulated_error"] / got["accumulated_weight"]
    w = scene.surfel_knn_weight[s].astype(np.float64)
    want = (unit[scene.surfel_knn[s]] * w).sum(1) / (w.sum(1) + 1e-4)
    np.testing.assert_allclose(got["node_error_map"][0][ys, xs], want, rtol=1e-5, atol=1e-7)
    assert np.all(got["node_error_map"][0][view.index_map == 0xFFFFFFFF] == 0)


# --------------------------------------------------------------------------
# correction of large-error nodes
# --------------------------------------------------------------------------

def correction_inputs(scene, united, guides):
    nk, nw = synth.node_skinning(scene)
    v, n = surfels(scene)
    lv, ln, live = synth_forward(scene, v, n, nk, nw)
    return dict(scene=scene, guides=guides, united_error=united, node_se3=scene.node_se3, live_nodes=live,
                node_knn=nk, node_weight=nw, live_vertex=lv, live_normal=ln, surfel_knn=scene.surfel_knn,
                surfel_weight=scene.surfel_knn_weight)


def synth_forward(scene, v, n, nk, nw):
    import oracle
    return oracle.forward_warp(scene.node_se3, scene.surfel_knn, scene.surfel_knn_weight, v, n, nk, nw,
                               synth.node_views(scene))


def constant_guides(scene, R, t):
    out = []
    for se3, valid, prev in synth.correction_guides(scene):
        se3 = np.zeros_like(se3)
        se3[..., :9] = np.asarray(R, np.float32).T.reshape(9)
        se3[..., 9:] = t
        out.append((se3, valid, prev))
    return out


def test_small_errors_get_identity_and_nothing_moves(oracle_mod):
    scene = small_scene("torso")
    united = np.full(scene.num_nodes, 0.1, np.float32)
    inp = correction_inputs(scene, united, synth.correction_guides(scene))
    res = oracle_mod.correct_large_error_nodes(**inp)
    assert np.array_equal(res["correction"], np.tile(IDENT, (scene.num_nodes, 1)))
    np.testing.assert_allclose(res["live_vertex"], inp["live_vertex"], atol=1e-6)
    np.testing.assert_allclose(res["node_se3"], inp["node_se3"], atol=1e-6)


def test_constant_translation_guide_moves_large_error_nodes(oracle_mod):
    """Every guide translates by d in the camera: a node with error e and a
    guide within reach gets the screw motion e * (R_init d) in frame 0; a node
    whose four neighbours all got it moves by that amount."""
    scene = small_scene("sphere")
    d = np.array([0.004, -0.002, 0.003], np.float32)
    united = np.full(scene.num_nodes, 0.5, np.float32)
    inp = correction_inputs(scene, united, constant_guides(scene, np.eye(3), d))
    res = oracle_mod.correct_large_error_nodes(**inp)
    Ri, _ = _rows(scene.views[0].initial_camera_se3)
    Rw, _ = _rows(scene.views[0].world2camera)
    want_t = 0.5 * (Rw.T @ Ri @ d)
    corr = res["correction"]
    moved = np.abs(corr[:, 4:7]).sum(1) > 0
    assert moved.mean() > 0.3
    # a pure translation: q0 stays the identity, q1 = (t / 2, 0)
    np.testing.assert_allclose(corr[moved, :4], np.tile([0, 0, 0, 1], (moved.sum(), 1)), atol=1e-5)
    np.testing.assert_allclose(2 * corr[moved, 4:7], np.tile(want_t, (moved.sum(), 1)), atol=2e-6)
    nk = inp["node_knn"]
    full = moved[nk].all(1)
    assert full.sum() > 10
    step = res["live_nodes"][full, :3] - inp["live_nodes"][full, :3]
    np.testing.assert_allclose(step, np.tile(want_t, (full.sum(), 1)), atol=2e-6)


# --------------------------------------------------------------------------
# C ABI argument checks (before any CUDA call)
# --------------------------------------------------------------------------

def test_deform_argument_validation():
    import multiviewdynrecon_b200 as m
    L = m.lib()
    s = abi.DeformSurfels()
    s.num_surfels = 4
    buf = np.zeros(64, np.float32)
    assert L.mvdr_forward_warp(None, 1, C.byref(s), None, None) == abi.MVDR_EINVAL
    assert L.mvdr_forward_warp(C.c_void_p(buf.ctypes.data), 1, None, None, None) == abi.MVDR_EINVAL
    assert L.mvdr_forward_warp(C.c_void_p(buf.ctypes.data), 1, C.byref(s), None, None) == abi.MVDR_EINVAL  # arrays
    addr = (buf.ctypes.data + 15) & ~15
    for f in ("knn", "knn_weight", "in_vertex", "in_normal", "out_vertex", "out_normal"):
        setattr(s, f, addr)
    assert L.mvdr_forward_warp(C.c_void_p(addr), 0, C.byref(s), None, None) == abi.MVDR_EINVAL  # no field
    s.in_vertex = addr + 4
    assert L.mvdr_forward_warp(C.c_void_p(addr), 1, C.byref(s), None, None) == abi.MVDR_EINVAL  # misaligned
    assert b"aligned" in L.mvdr_last_error_string()
    s.in_vertex = addr
    assert L.mvdr_inverse_warp(C.c_void_p(addr), 1, C.c_void_p(addr + 8), C.byref(s), None) == abi.MVDR_EINVAL
    assert L.mvdr_compute_node_error(None, C.byref(abi.NodeError()), None) == abi.MVDR_EINVAL
    assert L.mvdr_correct_large_error_nodes(None, C.byref(abi.Correction()), None) == abi.MVDR_EINVAL
