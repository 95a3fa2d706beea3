"""Sparse feature selection from raw pixel pairs (CPU): the oracle's
restatement of SparseCorrespondenceHandler's choose and compact kernels
(core/NonRigidSolver/SparseCorrespondenceHandler.cu:18-199, nearest-distance
form) against an independent numpy restatement and hand-built cases."""
import dataclasses

import numpy as np
import pytest

from conftest import small_scene
from multiviewdynrecon_b200 import abi, synth

INVALID = 0xFFFFFFFF


def _rows(m):
    m = np.asarray(m, np.float64)
    return m[:9].reshape(3, 3).T, m[9:12]


def numpy_select(scene):
    """Per candidate: the observed pixel (last window row's first non-zero
    vertex, centre preferred), the rendered pixel (nearest live vertex among
    the window's surfel pixels; outside the image the index reads 0 and the
    live vertex zero), the 5 cm test on the reference vertex."""
    H, W = scene.height, scene.width
    T, R, K, Wt = [], [], [], []
    for v, (pairs, live, edge) in enumerate(scene.feature_pairs):
        view = scene.views[v]
        obs = view.vertex_confidence_map
        idx = view.index_map
        Ri, ti = _rows(view.initial_camera_se3)
        Rw, tw = _rows(view.world2camera)

        def o4(x, y):
            return obs[y, x] if 0 <= x < W and 0 <= y < H else np.zeros(4, np.float32)

        def zero(a):
            return bool(np.all(np.abs(a[:3].astype(np.float64)) < 1e-3))

        for x0, y0, z0, w0 in pairs.astype(np.int64):
            dp = None
            for y in range(w0 - 1, w0 + 2):
                for x in range(z0 - 1, z0 + 2):
                    if not zero(o4(x, y)):
                        dp = (x, y)
                        break
            if not zero(o4(z0, w0)):
                dp = (z0, w0)
            if dp is None or not (0 <= dp[0] < W and 0 <= dp[1] < H):
                continue
            if edge is not None and edge[dp[1], dp[0]] == 1:
                continue
            ov = obs[dp[1], dp[0]].astype(np.float32)
            gp, best = None, np.float32(100.0)
            for y in range(y0 - 1, y0 + 2):
                for x in range(x0 - 1, x0 + 2):
                    inside = 0 <= x < W and 0 <= y < H
                    s = idx[y, x] if inside else 0
                    if s != INVALID:
                        lv = live[y, x] if inside else np.zeros(4, np.float32)
                        d = np.float32(((ov[:3] - lv[:3]) ** 2).sum(dtype=np.float32))
                        if d < best:
                            gp, best = (x, y), d
            if gp is None or not (0 <= gp[0] < W and 0 <= gp[1] < H):
                continue
            s = idx[gp[1], gp[0]]
            rv = view.reference_vertex_map[gp[1], gp[0]]
            if s >= scene.num_surfels or ((rv[:3] - ov[:3]) ** 2).sum() >= 2.5e-3:
                continue
            r0 = Ri @ rv[:3] + ti
            d0 = Ri @ ov[:3] + ti
            t0 = Rw.T @ (d0 - tw)
            T.append([*t0, 1.0])
            R.append([*r0, rv[3]])
            K.append(scene.surfel_knn[s])
            Wt.append(scene.surfel_knn_weight[s])
    return np.array(T), np.array(R), np.array(K, np.uint16).reshape(-1, 4), np.array(Wt).reshape(-1, 4)


@pytest.mark.parametrize("kind", ["torso", "body", "sphere_rigid"])
def test_selection_matches_numpy(oracle_mod, kind):
    scene = synth.with_feature_pairs(small_scene(kind), per_view=300, seed=4)
    o = oracle_mod.Oracle(scene, abi.make_config(scene))
    t, r, k, w = o.feature_terms()
    T, R, K, Wt = numpy_select(scene)
    assert len(t) == len(T) > 100
    np.testing.assert_allclose(t, T, atol=2e-6)
    np.testing.assert_allclose(r, R, atol=2e-6)
    assert np.array_equal(k, K) and np.array_equal(w, Wt.astype(np.float32))
    # most in-surface pairs are kept; far outliers and edge pixels are not
    assert len(t) < sum(len(p[0]) for p in scene.feature_pairs)


def test_feature_pairs_drive_the_feature_term(oracle_mod):
    """A scene's own correspondences and pairs built from them select
    features whose targets sit on the observed surface."""
    scene = synth.with_feature_pairs(small_scene("torso"), per_view=200, seed=2, outlier_fraction=0.0)
    o = oracle_mod.Oracle(scene, abi.make_config(scene))
    o.build_index()
    c = o.counts()
    t, r, _, _ = o.feature_terms()
    assert c.feature_terms == len(t) > 300
    # target and reference are the same surface point up to the warp's
    # perturbation and the depth noise: a few millimetres
    assert np.median(np.linalg.norm(t[:, :3] - r[:, :3], axis=1)) < 0.01


def small_case():
    """A 12 x 10 single view: a plane at depth 1 covering x in [2, 9],
    y in [2, 7]; surfel ids row-major; one edge pixel."""
    scene = small_scene("sphere")
    W, H = 12, 10
    idx = np.full((H, W), INVALID, np.uint32)
    ref = np.zeros((H, W, 4), np.float32)
    obs = np.zeros((H, W, 4), np.float32)
    sid = 0
    for y in range(2, 8):
        for x in range(2, 10):
            idx[y, x] = sid
            sid += 1
            ref[y, x] = [0.01 * x, 0.01 * y, 1.0, 1.0]
            obs[y, x] = [0.01 * x + 0.001, 0.01 * y, 1.0, 1.0]
    edge = np.zeros((H, W), np.uint8)
    edge[5, 9] = 1
    view = dataclasses.replace(scene.views[0], reference_vertex_map=ref, reference_normal_map=ref.copy(),
                               index_map=idx, vertex_confidence_map=obs, normal_radius_map=obs.copy(),
                               filtered_foreground_mask=np.zeros((H, W), np.float32),
                               foreground_mask_gradient=np.zeros((H, W, 2), np.float32),
                               world2camera=np.array([1, 0, 0, 0, 1, 0, 0, 0, 1, 0, 0, 0], np.float32),
                               initial_camera_se3=np.array([1, 0, 0, 0, 1, 0, 0, 0, 1, 0, 0, 0], np.float32))
    knn = np.tile(np.arange(4, dtype=np.uint16), (sid, 1))
    wts = np.full((sid, 4), 0.25, np.float32)
    pairs = np.array([[4, 4, 4, 4],     # 0: kept as is
                      [0, 0, 4, 4],     # 1: no surfel in the rendered window: dropped
                      [3, 3, 0, 0],     # 2: no observation in the depth window: dropped
                      [9, 5, 9, 5],     # 3: observed pixel on an edge: dropped
                      [1, 4, 6, 1],     # 4: both windows reach the plane only at their edge
                      [5, 5, 5, 5]],    # 5: kept
                     np.uint16)
    live = ref.copy()
    s2 = dataclasses.replace(scene, width=W, height=H, views=[view], surfel_knn=knn, surfel_knn_weight=wts,
                             feature=synth.Correspondences.empty(), cross_view=synth.Correspondences.empty(),
                             feature_pairs=[(pairs, live, edge)], terms={"feature": True})
    return s2


def test_hand_built_pairs(oracle_mod):
    scene = small_case()
    o = oracle_mod.Oracle(scene, abi.make_config(scene))
    t, r, k, w = o.feature_terms()
    # kept: pairs 0, 4 and 5 in candidate order
    assert len(t) == 3
    np.testing.assert_allclose(r[0, :3], [0.04, 0.04, 1.0], atol=1e-7)
    np.testing.assert_allclose(t[0, :3], [0.041, 0.04, 1.0], atol=1e-7)
    # pair 4: the depth window around (6, 1) has observations in its last row
    # only, and the scan keeps that row's first one: (5, 2), vertex
    # (0.051, 0.02, 1). The rendered window x in [0, 2], y in [3, 5] has
    # surfels at x = 2 only; the nearest live vertex is at (2, 3).
    np.testing.assert_allclose(r[1, :3], [0.02, 0.03, 1.0], atol=1e-7)
    np.testing.assert_allclose(t[1, :3], [0.051, 0.02, 1.0], atol=1e-7)
    np.testing.assert_allclose(r[2, :3], [0.05, 0.05, 1.0], atol=1e-7)
    T, R, K, Wt = numpy_select(scene)
    np.testing.assert_allclose(t, T, atol=1e-7)
    np.testing.assert_allclose(r, R, atol=1e-7)
