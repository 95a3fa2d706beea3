"""The solver-map renderer: oracle known answers and host checks (no GPU).

The reference renders its solver maps with OpenGL (render/shaders/
SolverMap.vert, SolverMapSized.vert, SolverMapIndexMap.vert, SolverMap.frag,
drawn by render/RendererDraw.cpp:384-480): every surfel is a point, culled
when it lies behind the camera, beyond max depth + 0.05, or is unstable and
not recently observed; projected with the pinhole model; drawn over the
pixels whose centres lie inside the point's square (one pixel, or the sized
shader's disc extent); kept where it is strictly nearer than what is there
(GL_LESS on a cleared depth buffer). The oracle restates that pipeline in
surfel order. These tests pin it with hand-computed answers and with an
independent float32 numpy restatement, and check the C ABI's argument
validation.
"""
import ctypes as C
import dataclasses

import numpy as np
import pytest

from conftest import small_scene
from multiviewdynrecon_b200 import abi, synth

INVALID = 0xFFFFFFFF
IDENT = np.array([1, 0, 0, 0, 1, 0, 0, 0, 1, 0, 0, 0], np.float32)


@dataclasses.dataclass
class Cam:
    world2camera: np.ndarray
    initial_camera_se3: np.ndarray
    intrinsic: np.ndarray


def tiny_camera(init=IDENT):
    return Cam(IDENT.copy(), np.asarray(init, np.float32), np.array([4.0, 3.0, 4.0, 4.0], np.float32))


def geometry(points, normals=None, confid=None, radius=None, rgb=None, times=None):
    n = len(points)
    p = np.asarray(points, np.float32)
    nr = np.asarray(normals if normals is not None else [[0, 0, -1]] * n, np.float32)
    cf = np.asarray(confid if confid is not None else [15.0] * n, np.float32)
    rd = np.asarray(radius if radius is not None else [1.0] * n, np.float32)
    ct = np.zeros((n, 4), np.float32)
    ct[:, 0] = synth.pack_rgb(np.asarray(rgb if rgb is not None else [[0.2, 0.4, 0.6]] * n))
    t = np.asarray(times if times is not None else [(3.0, 10.0)] * n, np.float32)
    ct[:, 1], ct[:, 2] = t[:, 0], t[:, 1]
    ref_v = np.concatenate([p, cf[:, None]], 1)
    ref_n = np.concatenate([nr, rd[:, None]], 1)
    return dict(reference_vertex_confid=ref_v, reference_normal_radius=ref_n,
                live_vertex_confid=ref_v.copy(), live_normal_radius=ref_n.copy(), color_time=ct)


def params(W=8, H=6, **kw):
    return abi.solver_map_params(W, H, **kw)


def drawn(maps):
    idx = maps["index_map"]
    return {(int(u), int(w)): int(idx[w, u]) for w, u in zip(*np.nonzero(idx != INVALID))}


def test_nearest_surfel_wins_and_ties_keep_the_first(oracle_mod):
    # fx = fy = 4, cx = 4, cy = 3: (0.1, -0.05, 1) projects to (4.4, 2.8),
    # inside pixel (4, 2) whose centre is (4.5, 2.5)
    pts = [[0.2, -0.1, 2.0],        # 0: same pixel, farther
           [0.1, -0.05, 1.0],       # 1: nearest
           [0.1, -0.05, 1.0],       # 2: same depth as 1, drawn later
           [-0.9, -0.6375, 1.5]]    # 3: projects to (1.6, 1.3): pixel (1, 1)
    m = oracle_mod.render_solver_maps(geometry(pts), params(), [tiny_camera()])[0]
    assert drawn(m) == {(4, 2): 1, (1, 1): 3}
    # the winner's attributes (identity camera: frame 0 = camera frame)
    p1 = np.array([0.1, -0.05, 1.0, 1.0], np.float32)
    np.testing.assert_array_equal(m["reference_vertex_map"][2, 4], p1)
    np.testing.assert_array_equal(m["reference_normal_map"][2, 4], np.float32([0, 0, -1, 0]))
    np.testing.assert_array_equal(m["live_vertex_map"][2, 4], p1)
    rgb = np.float32(np.array([51, 102, 153], np.float32) / np.float32(255))
    np.testing.assert_array_equal(m["normalized_rgb_map"][2, 4], [*rgb, 3.0])  # w: color_time.y
    # clear values elsewhere
    assert np.all(m["reference_vertex_map"][0, 0] == 0) and m["index_map"][0, 0] == INVALID


def test_culling_and_clipping(oracle_mod):
    pts = [[0.1, -0.05, 1.0],       # 0: unstable (confidence 5 < 10) and observed 4 frames ago: culled
           [-0.9, -0.6375, 1.5],    # 1: unstable but observed 2 frames ago: drawn
           [0.1, -0.05, -1.0],      # 2: behind the camera
           [0.1, -0.05, 3.1],       # 3: beyond max depth 3 + 0.05
           [-1.2, 0.0, 1.0],        # 4: projects to x = -0.8, outside the image
           [0.0, 0.0, 3.04]]        # 5: inside max depth + 0.05, projects to the corner (4, 3):
    #                                  the pixel with centre (3.5, 2.5) in [3.5, 4.5) x [2.5, 3.5)
    g = geometry(pts, confid=[5, 5, 15, 15, 15, 15], times=[(0, 6), (0, 8), (0, 10), (0, 10), (0, 10), (0, 10)])
    m = oracle_mod.render_solver_maps(g, params(current_time=10.0, time_threshold=3.0), [tiny_camera()])[0]
    assert drawn(m) == {(1, 1): 1, (3, 2): 5}
    # time threshold -1 (confident observation only): no unstable surfel
    m = oracle_mod.render_solver_maps(g, params(current_time=10.0, time_threshold=-1.0), [tiny_camera()])[0]
    assert drawn(m) == {(3, 2): 5}


def test_sized_points_cover_the_disc_extent(oracle_mod):
    # a disc facing the camera at depth 1: its corners project fx * s away
    # from the centre, s = radius * sqrt(2) * 1e-3; radius 300 mm gives a
    # point of 2 * 4 * 0.4243 = 3.39 pixels centred at (2.5, 3.5): pixels
    # u, w with centres within 1.70 of it, 3 x 3
    g = geometry([[-0.375, 0.125, 1.0], [0.1, -0.05, 1.0]], radius=[300.0, 1.0])
    m = oracle_mod.render_solver_maps(g, params(), [tiny_camera()], sized=[True])[0]
    want = {(u, w): 0 for u in (1, 2, 3) for w in (2, 3, 4)}
    want[(4, 2)] = 1    # a tiny disc is clamped to one pixel
    assert drawn(m) == want
    assert m["normalized_rgb_map"][3, 2, 3] == 1.0   # the sized shader's alpha


def test_initial_camera_frame(oracle_mod):
    """The point is moved by initialCameraSE3^-1 before world2camera, and the
    maps hold the attributes in that camera's frame."""
    R = synth.rodrigues(np.array([0.0, 0.3, 0.0]))
    t = np.array([0.2, 0.0, 0.1])
    init = synth.mat34_pack(R, t).astype(np.float32)
    p_cam = np.array([0.1, -0.05, 1.0])
    p_world = R @ p_cam + t
    n_world = R @ np.array([0.0, 0.0, -1.0])
    g = geometry([p_world], normals=[n_world])
    m = oracle_mod.render_solver_maps(g, params(), [tiny_camera(init)])[0]
    assert drawn(m) == {(4, 2): 0}
    np.testing.assert_allclose(m["reference_vertex_map"][2, 4, :3], p_cam, atol=1e-6)
    np.testing.assert_allclose(m["reference_normal_map"][2, 4, :3], [0, 0, -1], atol=1e-6)


# --------------------------------------------------------------------------
# an independent float32 restatement (numpy, vectorised)
# --------------------------------------------------------------------------

def _rows(m):
    m = np.asarray(m, np.float32)
    return m[:9].reshape(3, 3).T.copy(), m[9:12].copy()


def _pt(R, t, p):
    return np.stack([R[r, 0] * p[:, 0] + R[r, 1] * p[:, 1] + R[r, 2] * p[:, 2] + t[r] for r in range(3)], 1)


def _dir(R, p):
    return np.stack([R[r, 0] * p[:, 0] + R[r, 1] * p[:, 1] + R[r, 2] * p[:, 2] for r in range(3)], 1)


def _normalise(v):
    inv = np.float32(1.0) / np.sqrt(v[:, 0] * v[:, 0] + v[:, 1] * v[:, 1] + v[:, 2] * v[:, 2])
    return v * inv[:, None]


def numpy_render(g, prm, cam, sized):
    W, H = prm.width, prm.height
    Rw, tw = _rows(cam.world2camera)
    Ri, ti = _rows(cam.initial_camera_se3)
    Rv = Ri.T.copy()
    tv = -(Rv[:, 0] * ti[0] + Rv[:, 1] * ti[1] + Rv[:, 2] * ti[2])
    cx, cy, fx, fy = [np.float32(x) for x in cam.intrinsic]
    lv = g["live_vertex_confid"][:, :3]
    pc = _pt(Rw, tw, _pt(Rv, tv, lv))
    z = pc[:, 2]
    ct = g["color_time"]
    keep = ~((z > np.float32(prm.max_depth) + np.float32(0.05)) | ~(z > 0) |
             ((g["reference_vertex_confid"][:, 3] < np.float32(prm.confidence_threshold)) &
              (np.abs(ct[:, 2] - np.float32(prm.current_time)) >= np.float32(prm.time_threshold))))

    def proj(q):
        return (fx * q[:, 0]) / q[:, 2] + cx, (fy * q[:, 1]) / q[:, 2] + cy

    with np.errstate(all="ignore"):
        xw, yw = proj(pc)
        keep &= (xw >= 0) & (xw <= np.float32(W)) & (yw >= 0) & (yw <= np.float32(H))
        size = np.ones(len(lv), np.float32)
        if sized:
            n = _normalise(_dir(Rw, _dir(Rv, g["live_normal_radius"][:, :3])))
            s = g["reference_normal_radius"][:, 3] * np.float32(1.41421356) * np.float32(0.001)
            x0 = _normalise(np.stack([n[:, 1] - n[:, 2], -n[:, 0], n[:, 0]], 1))
            x1 = x0 * s[:, None]
            y1 = np.stack([n[:, 1] * x1[:, 2] - n[:, 2] * x1[:, 1], n[:, 2] * x1[:, 0] - n[:, 0] * x1[:, 2],
                           n[:, 0] * x1[:, 1] - n[:, 1] * x1[:, 0]], 1)
            P = [proj(pc + x1), proj(pc + y1), proj(pc - y1), proj(pc - x1)]
            px, py = np.stack([p[0] for p in P]), np.stack([p[1] for p in P])
            xd, yd = px.max(0) - px.min(0), py.max(0) - py.min(0)
            size = np.minimum(np.maximum(np.maximum(np.float32(0), np.minimum(np.abs(xd), np.abs(yd))),
                                         np.float32(1)), np.float32(2047))
        h = np.float32(0.5) * size
        u0 = np.maximum(0, np.ceil(xw - h - np.float32(0.5)))
        u1 = np.minimum(W, np.ceil(xw + h - np.float32(0.5)))
        w0 = np.maximum(0, np.ceil(yw - h - np.float32(0.5)))
        w1 = np.minimum(H, np.ceil(yw + h - np.float32(0.5)))
    sid = np.nonzero(keep)[0]
    u0, u1, w0, w1 = [a[sid].astype(np.int64) for a in (u0, u1, w0, w1)]
    span = int(max(1, (u1 - u0).max(initial=1), (w1 - w0).max(initial=1)))
    pix, zs, ids = [], [], []
    for dw in range(span):
        for du in range(span):
            ok = (u0 + du < u1) & (w0 + dw < w1)
            pix.append(((w0 + dw) * W + u0 + du)[ok])
            zs.append(z[sid][ok])
            ids.append(sid[ok])
    pix, zs, ids = np.concatenate(pix), np.concatenate(zs), np.concatenate(ids)
    order = np.lexsort((ids, zs, pix))
    pix, ids = pix[order], ids[order]
    first = np.ones(len(pix), bool)
    first[1:] = pix[1:] != pix[:-1]
    index = np.full(H * W, INVALID, np.uint32)
    index[pix[first]] = ids[first]
    return index.reshape(H, W)


@pytest.mark.parametrize("kind,sized", [("torso", (True, False, False)), ("body", (False, False, False)),
                                        ("body", (True, True, True))])
@pytest.mark.parametrize("recent", [True, False])
def test_oracle_matches_numpy_restatement(oracle_mod, kind, sized, recent):
    scene = small_scene(kind)
    g = synth.solver_map_geometry(scene)
    prm = abi.solver_map_params(scene.width, scene.height, time_threshold=3.0 if recent else -1.0)
    maps = oracle_mod.render_solver_maps(g, prm, scene.views, sized=sized)
    for v, view in enumerate(scene.views):
        want = numpy_render(g, prm, view, sized[v])
        assert np.array_equal(maps[v]["index_map"], want), v
        assert (want != INVALID).mean() > 0.05


def test_rendered_maps_are_the_scene_surface(oracle_mod):
    """Rendered from unwarped surfels, a drawn pixel mostly holds a surfel
    that the scene's own ray cast put within a pixel of it, at nearly the ray
    cast's point. (The ray cast puts a pixel's surfel at the pixel's corner
    in GL's convention, so some pixels get none of their own and show another
    view's surfel, at silhouettes one of a farther surface.)"""
    scene = small_scene("torso")
    g = synth.solver_map_geometry(scene, warped=False)
    prm = abi.solver_map_params(scene.width, scene.height, time_threshold=100.0)
    maps = oracle_mod.render_solver_maps(g, prm, scene.views)
    for v, view in enumerate(scene.views):
        idx = maps[v]["index_map"]
        H, W = idx.shape
        home = np.full((scene.num_surfels, 2), -1)
        ys, xs = np.nonzero(view.index_map != INVALID)
        home[view.index_map[ys, xs]] = np.stack([xs, ys], 1)
        ys, xs = np.nonzero(idx != INVALID)
        s = idx[ys, xs]
        own = home[s, 0] >= 0
        assert own.mean() > 0.5
        d = np.abs(home[s[own]] - np.stack([xs[own], ys[own]], 1)).max(1)
        assert np.mean(d <= 1) > 0.97
        hit = view.index_map[ys, xs] != INVALID
        gap = np.linalg.norm(maps[v]["reference_vertex_map"][ys, xs, :3] - view.reference_vertex_map[ys, xs, :3], axis=1)
        footprint = view.reference_vertex_map[ys, xs, 2] / view.intrinsic[2]
        assert np.median(gap[hit] / footprint[hit]) < 2.0
        # the reference vertex map holds the surfel in the camera's frame
        ref = maps[v]["reference_vertex_map"][ys[own], xs[own], :3]
        hx, hy = home[s[own], 0], home[s[own], 1]
        np.testing.assert_allclose(ref, view.reference_vertex_map[hy, hx, :3], atol=2e-5)


# --------------------------------------------------------------------------
# the C ABI's argument checks (they return before any CUDA call)
# --------------------------------------------------------------------------

def test_render_argument_validation():
    import multiviewdynrecon_b200 as m
    L = m.lib()
    scene = small_scene("sphere")
    g = synth.solver_map_geometry(scene)
    arrs = {k: np.ascontiguousarray(v) for k, v in g.items()}
    geo = abi.surfel_geometry(scene.num_surfels, {k: a.ctypes.data for k, a in arrs.items()})
    idx = np.zeros((scene.height, scene.width), np.uint32)
    zb = np.zeros((scene.height, scene.width), np.uint64)
    good = {"index_map": idx.ctypes.data, "depth_index": zb.ctypes.data}
    prm = abi.solver_map_params(scene.width, scene.height)

    def call(geo=geo, prm=prm, views=None, n=1):
        vs = (abi.SolverMapView * max(n, 1))()
        for k in range(max(n, 1)):
            vs[k] = (views or [abi.solver_map_view(scene.views[0], good)])[min(k, len(views or [0]) - 1)]
        return L.mvdr_render_solver_maps(C.byref(geo) if geo is not None else None,
                                         C.byref(prm) if prm is not None else None, vs, n, None)

    assert call(geo=None) == abi.MVDR_EINVAL
    assert call(prm=None) == abi.MVDR_EINVAL
    assert call(n=0) == abi.MVDR_EINVAL
    assert call(n=abi.MVDR_MAX_VIEWS + 1) == abi.MVDR_EINVAL
    assert call(prm=abi.solver_map_params(0, scene.height)) == abi.MVDR_EINVAL
    assert call(prm=abi.solver_map_params(scene.width, 70000)) == abi.MVDR_EINVAL
    missing = abi.surfel_geometry(scene.num_surfels, {**{k: a.ctypes.data for k, a in arrs.items()},
                                                      "color_time": None})
    assert call(geo=missing) == abi.MVDR_EINVAL
    assert call(views=[abi.solver_map_view(scene.views[0], {"depth_index": zb.ctypes.data})]) == abi.MVDR_EINVAL
    assert call(views=[abi.solver_map_view(scene.views[0], {"index_map": idx.ctypes.data})]) == abi.MVDR_EINVAL
    short = abi.solver_map_view(scene.views[0], good, pitch=scene.width - 1)
    assert call(views=[short]) == abi.MVDR_EINVAL
    # a bad second view is refused before the first is touched
    assert call(views=[abi.solver_map_view(scene.views[0], good), short], n=2) == abi.MVDR_EINVAL
    assert b"pitch" in L.mvdr_last_error_string()
