"""Seeded synthetic scenes for the non-rigid Gauss-Newton solver.

The reference solver consumes, per camera view, the solver maps rendered from
the canonical surfel model (render/Renderer.h:381-388), the camera observation
(base/CameraObservation.h:16-63), the warp field (WarpField.h:157-161), the
surfel skinning (SurfelGeometry.h:179-182) and the compacted sparse / cross-view
correspondences (SparseCorrespondenceHandler.cu:152-199). Its own data set is
not available, so these generators produce the same arrays from analytic
shapes:

* a shape is ray-cast per pixel (pinhole, the projection of
  render/shaders/SolverMap.vert:23-29 run backwards), nearest hit wins;
* one surfel per valid pixel footprint; the reference vertex/normal maps hold
  the canonical surfel in that camera's frame and the index map its id;
* the observation is the same surface with N(0, 2 mm) depth noise;
* nodes are Poisson-disk samples of the surfels (dart throwing), 8-NN node
  graph as WarpField.cu:15-57 (self excluded), 4-NN skinning weights
  exp(-d^2 / 2r^2) normalised as CanonicalNodesSkinner.cu:395-420;
* the initial warp field is a per-node random SE(3) perturbation (rotation
  about the node, sigma 2 deg; translation sigma 5 mm) of the identity, which
  is the true warp, so the solve pulls the nodes back towards identity.

Frame 0 is camera 0's frame. ``initial_camera_se3`` maps camera v to frame 0;
``world2camera`` is the rigid correction of frame 0 (identity unless asked).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
from scipy import ndimage
from scipy.spatial import cKDTree

INVALID_INDEX = np.uint32(0xFFFFFFFF)


# --------------------------------------------------------------------------
# small rigid-transform helpers (float64); mat34 = (3x3 rotation, 3 translation)
# --------------------------------------------------------------------------

def rodrigues(w):
    w = np.asarray(w, dtype=np.float64)
    th = np.linalg.norm(w)
    if th < 1e-12:
        return np.eye(3)
    k = w / th
    K = np.array([[0, -k[2], k[1]], [k[2], 0, -k[0]], [-k[1], k[0], 0]])
    return np.eye(3) + math.sin(th) * K + (1 - math.cos(th)) * (K @ K)


def rodrigues_batch(w):
    """(n,3) axis-angle -> (n,3,3) rotation matrices."""
    w = np.asarray(w, dtype=np.float64)
    th = np.linalg.norm(w, axis=1)
    k = w / np.maximum(th, 1e-30)[:, None]
    K = np.zeros((len(w), 3, 3))
    K[:, 0, 1], K[:, 0, 2] = -k[:, 2], k[:, 1]
    K[:, 1, 0], K[:, 1, 2] = k[:, 2], -k[:, 0]
    K[:, 2, 0], K[:, 2, 1] = -k[:, 1], k[:, 0]
    s = np.sin(th)[:, None, None]
    c = (1 - np.cos(th))[:, None, None]
    R = np.eye(3)[None] + s * K + c * (K @ K)
    R[th < 1e-12] = np.eye(3)
    return R


def look_at(eye, target, up=(0.0, -1.0, 0.0)):
    """Camera-to-frame-0 pose of a camera at `eye` looking at `target`
    (camera z forward, y down)."""
    eye = np.asarray(eye, np.float64)
    z = np.asarray(target, np.float64) - eye
    z /= np.linalg.norm(z)
    x = np.cross(up, z)
    x /= np.linalg.norm(x)
    y = np.cross(z, x)
    R = np.stack([x, y, z], axis=1)  # columns = camera axes in frame 0
    return R, eye


def mat34_pack(R, t):
    """Reference mat34 layout: rotation columns then translation (12 floats)."""
    return np.concatenate([np.asarray(R, np.float64).T.reshape(-1), np.asarray(t, np.float64)]).astype(np.float32)


def mat_to_quat(R):
    """Quaternion(mat33) of math/DualQuaternion/Quaternion.h:46-77, vectorised,
    returned as (x, y, z, w). Evaluated in float32 like the reference."""
    R = np.asarray(R, dtype=np.float32)
    m00, m01, m02 = R[:, 0, 0], R[:, 0, 1], R[:, 0, 2]
    m10, m11, m12 = R[:, 1, 0], R[:, 1, 1], R[:, 1, 2]
    m20, m21, m22 = R[:, 2, 0], R[:, 2, 1], R[:, 2, 2]
    n = len(R)
    q = np.zeros((n, 4), np.float32)
    tr = m00 + m11 + m22
    c0 = tr > 0
    c1 = (~c0) & (m00 > m11) & (m00 > m22)
    c2 = (~c0) & (~c1) & (m11 > m22)
    c3 = ~(c0 | c1 | c2)
    with np.errstate(divide="ignore", invalid="ignore"):
        s = np.sqrt(tr + np.float32(1)) * np.float32(2)
        q[c0] = np.stack([(m21 - m12) / s, (m02 - m20) / s, (m10 - m01) / s, s * np.float32(0.25)], 1)[c0]
        s = np.sqrt(np.float32(1) + m00 - m11 - m22) * np.float32(2)
        q[c1] = np.stack([np.float32(0.25) * s, (m01 + m10) / s, (m02 + m20) / s, (m21 - m12) / s], 1)[c1]
        s = np.sqrt(np.float32(1) + m11 - m00 - m22) * np.float32(2)
        q[c2] = np.stack([(m01 + m10) / s, np.float32(0.25) * s, (m12 + m21) / s, (m02 - m20) / s], 1)[c2]
        s = np.sqrt(np.float32(1) + m22 - m00 - m11) * np.float32(2)
        q[c3] = np.stack([(m02 + m20) / s, (m12 + m21) / s, np.float32(0.25) * s, (m10 - m01) / s], 1)[c3]
    return q


def quat_mul(a, b):
    """Hamilton product of (x, y, z, w) quaternions (Quaternion.h:303-312)."""
    ax, ay, az, aw = a[:, 0], a[:, 1], a[:, 2], a[:, 3]
    bx, by, bz, bw = b[:, 0], b[:, 1], b[:, 2], b[:, 3]
    w = aw * bw - ax * bx - ay * by - az * bz
    x = aw * bx + ax * bw + ay * bz - az * by
    y = aw * by - ax * bz + ay * bw + az * bx
    z = aw * bz + ax * by - ay * bx + az * bw
    return np.stack([x, y, z, w], 1)


def se3_to_dq(R, t):
    """DualQuaternion(mat34) of DualQuaternion.h:123-130: q0 = quat(R),
    q1 = (0, t/2) * q0. Returns (n, 8) float32: q0 xyzw, q1 xyzw."""
    q0 = mat_to_quat(R)
    t = np.asarray(t, np.float32)
    tq = np.concatenate([np.float32(0.5) * t, np.zeros((len(t), 1), np.float32)], 1)
    q1 = quat_mul(tq, q0).astype(np.float32)
    return np.concatenate([q0, q1], 1).astype(np.float32)


# --------------------------------------------------------------------------
# analytic shapes (ray casting)
# --------------------------------------------------------------------------

class Ellipsoid:
    def __init__(self, center, axes, R=None):
        self.c = np.asarray(center, np.float64)
        self.a = np.asarray(axes, np.float64)
        self.R = np.eye(3) if R is None else np.asarray(R, np.float64)

    def intersect(self, o, d):
        # local frame: p = R^T (x - c) / a
        ol = ((o - self.c) @ self.R) / self.a
        dl = (d @ self.R) / self.a
        A = np.sum(dl * dl, 1)
        B = 2 * np.sum(ol * dl, 1)
        C = np.sum(ol * ol, 1) - 1
        disc = B * B - 4 * A * C
        t = np.full(len(d), np.inf)
        ok = disc > 0
        sq = np.sqrt(np.where(ok, disc, 0))
        t0 = (-B - sq) / (2 * A)
        t1 = (-B + sq) / (2 * A)
        tt = np.where(t0 > 1e-6, t0, t1)
        ok &= tt > 1e-6
        t[ok] = tt[ok]
        p = o + d * np.where(ok, t, 0.0)[:, None]
        pl = ((p - self.c) @ self.R) / (self.a * self.a)
        n = pl @ self.R.T
        n /= np.maximum(np.linalg.norm(n, axis=1, keepdims=True), 1e-30)
        return t, n


class Capsule:
    def __init__(self, p0, p1, radius):
        self.p0 = np.asarray(p0, np.float64)
        self.p1 = np.asarray(p1, np.float64)
        self.r = float(radius)

    def intersect(self, o, d):
        ba = self.p1 - self.p0
        oa = o - self.p0
        baba = ba @ ba
        bard = d @ ba
        baoa = oa @ ba
        rdoa = np.sum(d * oa, 1)
        oaoa = np.sum(oa * oa, 1)
        a = baba - bard * bard
        b = baba * rdoa - baoa * bard
        c = baba * oaoa - baoa * baoa - self.r * self.r * baba
        h = b * b - a * c
        t = np.full(len(d), np.inf)
        ok = h >= 0
        sh = np.sqrt(np.where(ok, h, 0))
        with np.errstate(divide="ignore", invalid="ignore"):
            tc = (-b - sh) / a
        y = baoa + tc * bard
        body = ok & (y > 0) & (y < baba) & (tc > 1e-6)
        t[body] = tc[body]
        # caps
        rest = ok & ~body
        oc = np.where((y <= 0)[:, None], oa, o - self.p1)
        bcap = np.sum(d * oc, 1)
        ccap = np.sum(oc * oc, 1) - self.r * self.r
        hcap = bcap * bcap - ccap
        tcap = -bcap - np.sqrt(np.maximum(hcap, 0))
        capok = rest & (hcap > 0) & (tcap > 1e-6)
        t[capok] = tcap[capok]
        p = o + d * np.where(np.isfinite(t), t, 0.0)[:, None]
        # normal: direction from the closest axis point
        s = np.clip(((p - self.p0) @ ba) / baba, 0, 1)
        q = self.p0 + s[:, None] * ba
        n = p - q
        n /= np.maximum(np.linalg.norm(n, axis=1, keepdims=True), 1e-30)
        return t, n


def surface_colour(p):
    """Normalised rgb of a frame-0 surface point: smooth stripes of a few
    centimetres, different per channel."""
    p = np.asarray(p, np.float64)
    r = 0.5 + 0.3 * np.sin(40.0 * p[:, 0] + 3.0 * p[:, 2])
    g = 0.5 + 0.3 * np.cos(35.0 * p[:, 1] - 2.0 * p[:, 0])
    b = 0.5 + 0.2 * np.sin(25.0 * (p[:, 0] + p[:, 1] + p[:, 2]))
    return np.stack([r, g, b], 1).astype(np.float32)


def cast(shapes, o, d):
    t = np.full(len(d), np.inf)
    n = np.zeros((len(d), 3))
    for s in shapes:
        ts, ns = s.intersect(o, d)
        better = ts < t
        t[better] = ts[better]
        n[better] = ns[better]
    return t, n


# --------------------------------------------------------------------------
# the scene container
# --------------------------------------------------------------------------

@dataclass
class View:
    reference_vertex_map: np.ndarray      # (H, W, 4) float32
    reference_normal_map: np.ndarray      # (H, W, 4) float32
    index_map: np.ndarray                 # (H, W) uint32
    vertex_confidence_map: np.ndarray     # (H, W, 4) float32
    normal_radius_map: np.ndarray         # (H, W, 4) float32
    filtered_foreground_mask: np.ndarray  # (H, W) float32
    foreground_mask_gradient: np.ndarray  # (H, W, 2) float32
    intrinsic: np.ndarray                 # (4,) principal_x, principal_y, focal_x, focal_y
    world2camera: np.ndarray              # (12,) mat34
    initial_camera_se3: np.ndarray        # (12,) mat34
    # density (colour) term: rendered normalised rgb of the reference surface,
    # and the observed grey level with its image gradient
    normalized_rgb_map: np.ndarray = None     # (H, W, 4) float32
    density_map: np.ndarray = None            # (H, W) float32
    density_gradient_map: np.ndarray = None   # (H, W, 2) float32


@dataclass
class Correspondences:
    target_vertex: np.ndarray      # (T, 4) float32
    reference_vertex: np.ndarray   # (T, 4) float32
    knn: np.ndarray                # (T, 4) uint16
    knn_weight: np.ndarray         # (T, 4) float32

    @property
    def count(self):
        return int(len(self.knn))

    @staticmethod
    def empty():
        return Correspondences(np.zeros((0, 4), np.float32), np.zeros((0, 4), np.float32),
                               np.zeros((0, 4), np.uint16), np.zeros((0, 4), np.float32))


@dataclass
class Scene:
    name: str
    width: int
    height: int
    views: list
    surfel_knn: np.ndarray          # (S, 4) uint16
    surfel_knn_weight: np.ndarray   # (S, 4) float32
    node_se3: np.ndarray            # (N, 8) float32
    canonical_nodes: np.ndarray     # (N, 4) float32
    node_graph: np.ndarray          # (8N, 2) uint16
    feature: Correspondences
    cross_view: Correspondences
    node_radius: float = 0.025
    terms: dict = field(default_factory=dict)   # which terms the config asks for
    # the surfels behind the index maps, in frame 0 (surfel id = row)
    surfel_position: np.ndarray = None   # (S, 3) float64
    surfel_normal: np.ndarray = None     # (S, 3) float64
    # raw sparse-feature pixel pairs per view, selected by the solver: a list
    # of (pairs (n, 4) uint16, live vertex map (H, W, 4), edge mask (H, W)
    # uint8); `feature` is then empty
    feature_pairs: list = None
    gn_iterations: int = 3
    pcg_iterations: int = 10

    @property
    def num_nodes(self):
        return int(len(self.node_se3))

    @property
    def num_views(self):
        return len(self.views)

    @property
    def num_surfels(self):
        return int(len(self.surfel_knn))

    def dense_term_count(self):
        return int(sum(int((v.index_map != INVALID_INDEX).sum()) for v in self.views))


# --------------------------------------------------------------------------
# generator
# --------------------------------------------------------------------------

def _pixel_rays(W, H, fx, fy, cx, cy):
    u, v = np.meshgrid(np.arange(W, dtype=np.float64), np.arange(H, dtype=np.float64))
    d = np.stack([(u - cx) / fx, (v - cy) / fy, np.ones_like(u)], -1).reshape(-1, 3)
    return d  # un-normalised, z = 1


def _poisson_disk(points, n, rng, r_hint):
    """Dart throwing over a random permutation of `points` with the largest
    radius that still accepts at least `n` samples; returns n indices."""
    pts = np.asarray(points, np.float64)
    order = rng.permutation(len(pts))

    ordered = pts[order]
    tree = cKDTree(ordered)

    def throw(r):
        # greedy pass in `order`: a candidate is accepted when no accepted
        # point lies within r (strictly); the neighbour lists come from one
        # vectorised KD-tree query
        nbrs = tree.query_ball_point(ordered, r * (1.0 - 1e-12))
        blocked = np.zeros(len(order), bool)
        acc = []
        for k in range(len(order)):
            if blocked[k]:
                continue
            acc.append(order[k])
            if len(acc) >= n:
                break
            blocked[nbrs[k]] = True
        return acc

    # thin the candidate set first so the sequential pass stays short
    r = r_hint
    for _ in range(40):
        acc = throw(r)
        if len(acc) >= n:
            return np.asarray(acc[:n], np.int64)
        r *= 0.9
    raise RuntimeError("poisson disk sampling failed")


def _candidate_thin(points, target, rng):
    """Voxel subsample to about `target` candidates (one random point per voxel)."""
    pts = np.asarray(points, np.float64)
    lo = pts.min(0)
    ext = max(float((pts.max(0) - lo).max()), 1e-3)
    s = ext / 50.0
    for _ in range(60):
        keys = np.floor((pts - lo) / s).astype(np.int64)
        _, first = np.unique(keys[:, 0] * 1_000_003 * 1_000_003 + keys[:, 1] * 1_000_003 + keys[:, 2],
                             return_index=True)
        if len(first) > 4 * target:
            s *= 1.25
        elif len(first) < 2 * target:
            s *= 0.8
        else:
            break
    return first


def _knn_weights(d2, r):
    w = np.exp(-d2 / (2.0 * r * r))
    w /= np.maximum(w.sum(1, keepdims=True), 1e-30)
    return w.astype(np.float32)


def _build(name, shapes, cams, W, H, fx, fy, cx, cy, num_nodes, seed, *, auto_radius=False, node_radius=0.025,
           depth_noise=0.002, rot_sigma_deg=2.0, trans_sigma=0.005, features_per_view=0,
           cross_per_pair=0, rigid_offset=False, terms=None, gn=3, pcg=10, outlier_fraction=0.05):
    rng = np.random.default_rng(seed)
    dirs = _pixel_rays(W, H, fx, fy, cx, cy)
    dirn = dirs / np.linalg.norm(dirs, axis=1, keepdims=True)

    if rigid_offset:
        Rw = rodrigues(rng.normal(0, math.radians(1.0), 3))
        tw = rng.normal(0, 0.01, 3)
    else:
        Rw, tw = np.eye(3), np.zeros(3)

    surfel_pos, surfel_nrm = [], []
    per_view = []
    for (Rc, oc) in cams:
        o = np.repeat(oc[None], len(dirs), 0)
        dw = dirn @ Rc.T
        t, nw = cast(shapes, o, dw)
        valid = np.isfinite(t)
        pw = o + dw * np.where(valid, t, 0.0)[:, None]
        # surfels of this view, canonical = frame 0 (the true warp is identity)
        vid = np.nonzero(valid)[0]
        base = sum(len(p) for p in surfel_pos)
        surfel_pos.append(pw[vid])
        surfel_nrm.append(nw[vid])
        per_view.append((Rc, oc, valid, vid, base, pw, nw, t))

    surfels = np.concatenate(surfel_pos, 0)
    surfel_normals = np.concatenate(surfel_nrm, 0)

    # nodes
    cand = _candidate_thin(surfels, 3 * num_nodes, rng)
    r_hint = 0.08
    if auto_radius:
        # start the dart throwing near its final radius: the surface area from
        # the candidates' spacing, then sqrt(area / n) with a margin (a few
        # passes instead of tens for large node counts)
        d_nn = cKDTree(surfels[cand]).query(surfels[cand], k=2)[0][:, 1]
        area = len(cand) * float(np.mean(d_nn)) ** 2
        r_hint = 1.3 * math.sqrt(area / num_nodes)
    nodes_idx = _poisson_disk(surfels[cand], num_nodes, rng, r_hint=r_hint)
    node_pos = surfels[cand][nodes_idx]
    tree = cKDTree(node_pos)
    dgraph, igraph = tree.query(node_pos, k=9)
    graph = np.zeros((num_nodes * 8, 2), np.uint16)
    graph[:, 0] = np.repeat(np.arange(num_nodes), 8)
    graph[:, 1] = igraph[:, 1:9].reshape(-1)

    d_s, i_s = tree.query(surfels, k=4)
    surfel_knn = i_s.astype(np.uint16)
    surfel_w = _knn_weights(d_s * d_s, node_radius)

    # warp field: perturbation about each node
    Rn = rodrigues_batch(rng.normal(0, math.radians(rot_sigma_deg), (num_nodes, 3)))
    tn = rng.normal(0, trans_sigma, (num_nodes, 3))
    trans = node_pos - np.einsum("nij,nj->ni", Rn, node_pos) + tn
    node_se3 = se3_to_dq(Rn, trans)
    canonical_nodes = np.concatenate([node_pos, np.ones((num_nodes, 1))], 1).astype(np.float32)

    views = []
    for vi, (Rc, oc, valid, vid, base, pw, nw, t) in enumerate(per_view):
        # camera v -> frame 0
        Rinit, tinit = Rc, oc
        ref_v = np.zeros((H * W, 4), np.float32)
        ref_n = np.zeros((H * W, 4), np.float32)
        pc = (pw[vid] - tinit) @ Rinit          # frame 0 -> camera v
        nc = nw[vid] @ Rinit
        ref_v[vid, :3] = pc
        ref_v[vid, 3] = 1.0
        ref_n[vid, :3] = nc
        ref_n[vid, 3] = node_radius * 0.1
        idx = np.full(H * W, INVALID_INDEX, np.uint32)
        idx[vid] = (base + np.arange(len(vid))).astype(np.uint32)
        # observation: the live surface (identity warp) seen through the rigid
        # offset, with depth noise along the ray
        obs_v = np.zeros((H * W, 4), np.float32)
        obs_n = np.zeros((H * W, 4), np.float32)
        # live point in frame 0 after the rigid correction: x' = Rw x + tw;
        # camera-v coordinates: Rinit^T (x' - tinit)
        pl = pw[vid] @ Rw.T + tw
        pcl = (pl - tinit) @ Rinit
        z = pcl[:, 2]
        zn = z + rng.normal(0, depth_noise, len(z))
        pcl = pcl * (zn / z)[:, None]
        ncl = (nw[vid] @ Rw.T) @ Rinit
        obs_v[vid, :3] = pcl
        obs_v[vid, 3] = 1.0
        obs_n[vid, :3] = ncl
        obs_n[vid, 3] = 0.002
        # foreground: filtered inverse silhouette (0 deep inside the object)
        mask = valid.reshape(H, W).astype(np.float32)
        filt = ndimage.gaussian_filter(1.0 - mask, sigma=2.0).astype(np.float32)
        gy, gx = np.gradient(filt)
        grad = np.stack([gx, gy], -1).astype(np.float32)
        # colour: a smooth texture fixed to the surface; the reference render
        # shows it at each surfel, the observation shows the live surface's
        # grey level (rgb2density) with noise, blurred by 1 px
        rgb = np.zeros((H * W, 4), np.float32)
        rgb[vid, :3] = surface_colour(pw[vid])
        rgb[vid, 3] = 1.0
        grey = np.zeros(H * W, np.float32)
        # (a generator of its own, so that the other arrays of a seed stay
        # as they were before the colour maps existed)
        crng = np.random.default_rng([seed, 7919, vi])
        grey[vid] = (0.299 * rgb[vid, 0] + 0.587 * rgb[vid, 1] + 0.114 * rgb[vid, 2]
                     + crng.normal(0, 0.005, len(vid)))
        grey = ndimage.gaussian_filter(grey.reshape(H, W), sigma=1.0).astype(np.float32)
        dgy, dgx = np.gradient(grey)
        dgrad = np.stack([dgx, dgy], -1).astype(np.float32)
        views.append(View(
            reference_vertex_map=ref_v.reshape(H, W, 4),
            reference_normal_map=ref_n.reshape(H, W, 4),
            index_map=idx.reshape(H, W),
            vertex_confidence_map=obs_v.reshape(H, W, 4),
            normal_radius_map=obs_n.reshape(H, W, 4),
            filtered_foreground_mask=filt,
            foreground_mask_gradient=grad,
            intrinsic=np.array([cx, cy, fx, fy], np.float32),
            world2camera=mat34_pack(Rw, tw),
            initial_camera_se3=mat34_pack(Rinit, tinit),
            normalized_rgb_map=rgb.reshape(H, W, 4),
            density_map=grey,
            density_gradient_map=dgrad,
        ))

    def correspondences(src_surfels, tgt_points):
        k = len(src_surfels)
        ref = np.concatenate([surfels[src_surfels], np.ones((k, 1))], 1).astype(np.float32)
        tgt = np.concatenate([tgt_points, np.ones((k, 1))], 1).astype(np.float32)
        return Correspondences(tgt, ref, surfel_knn[src_surfels].copy(), surfel_w[src_surfels].copy())

    # sparse features: pixel pairs within each view, 5% outliers
    feats = []
    if features_per_view > 0:
        for vi, (Rc, oc, valid, vid, base, pw, nw, t) in enumerate(per_view):
            pick = rng.choice(len(vid), size=min(features_per_view, len(vid)), replace=False)
            src = base + pick
            obs = views[vi].vertex_confidence_map.reshape(-1, 4)[vid[pick], :3].astype(np.float64)
            tgt = obs @ Rc.T + oc                               # camera v -> frame 0
            tgt = (tgt - tw) @ Rw                               # undo the rigid correction
            out = rng.random(len(pick)) < outlier_fraction
            tgt[out] += rng.normal(0, 0.1, (int(out.sum()), 3))
            feats.append(correspondences(src, tgt))
    # cross-view correspondences between adjacent views
    cross = []
    if cross_per_pair > 0 and len(cams) > 1:
        pairs = [(a, (a + 1) % len(cams)) for a in range(len(cams))] if len(cams) > 2 else [(0, 1)]
        for (a, b) in pairs:
            Rc_a, oc_a, valid_a, vid_a, base_a = per_view[a][:5]
            Rb, ob = cams[b]
            pts = surfels[base_a:base_a + len(vid_a)]
            pcb = (pts - ob) @ Rb
            with np.errstate(divide="ignore", invalid="ignore"):
                u = np.rint(pcb[:, 0] / pcb[:, 2] * fx + cx).astype(np.int64)
                v = np.rint(pcb[:, 1] / pcb[:, 2] * fy + cy).astype(np.int64)
            inside = (pcb[:, 2] > 0.05) & (u >= 0) & (u < W) & (v >= 0) & (v < H)
            cand_idx = np.nonzero(inside)[0]
            if len(cand_idx) == 0:
                continue
            obs_b = views[b].vertex_confidence_map.reshape(-1, 4)[v[cand_idx] * W + u[cand_idx], :3].astype(np.float64)
            tgt = obs_b @ Rb.T + ob
            tgt = (tgt - tw) @ Rw
            close = (np.linalg.norm(tgt - pts[cand_idx], axis=1) < 0.01) & (np.abs(obs_b[:, 2]) > 0)
            cand_idx, tgt = cand_idx[close], tgt[close]
            if len(cand_idx) == 0:
                continue
            pick = rng.choice(len(cand_idx), size=min(cross_per_pair, len(cand_idx)), replace=False)
            cross.append(correspondences(base_a + cand_idx[pick], tgt[pick]))

    def cat(lst):
        if not lst:
            return Correspondences.empty()
        return Correspondences(*[np.concatenate([getattr(c, f) for c in lst], 0)
                                 for f in ("target_vertex", "reference_vertex", "knn", "knn_weight")])

    return Scene(name=name, width=W, height=H, views=views, surfel_knn=surfel_knn,
                 surfel_knn_weight=surfel_w, node_se3=node_se3, canonical_nodes=canonical_nodes,
                 node_graph=graph, feature=cat(feats), cross_view=cat(cross), node_radius=node_radius,
                 terms=terms or {}, gn_iterations=gn, pcg_iterations=pcg, surfel_position=surfels,
                 surfel_normal=surfel_normals)


# --------------------------------------------------------------------------
# surfel geometry for the solver-map renderer
# --------------------------------------------------------------------------

def blend_warp(node_se3, knn, w):
    """Surfel-wise rigid motions of the blended warp field (DQ blend,
    normalise, se3 matrix) in float64: returns R (S, 3, 3), t (S, 3)."""
    q = np.einsum("sk,skc->sc", np.asarray(w, np.float64), np.asarray(node_se3, np.float64)[knn.astype(np.int64)])
    q0, q1 = q[:, :4], q[:, 4:]
    inv = 1.0 / np.linalg.norm(q0, axis=1)
    q0, q1 = q0 * inv[:, None], q1 * inv[:, None]
    q1 = q1 - np.einsum("sc,sc->s", q0, q1)[:, None] * q0
    x, y, z, ww = q0.T
    R = np.stack([np.stack([1 - 2 * y * y - 2 * z * z, 2 * x * y - 2 * z * ww, 2 * x * z + 2 * y * ww], -1),
                  np.stack([2 * x * y + 2 * z * ww, 1 - 2 * x * x - 2 * z * z, 2 * y * z - 2 * x * ww], -1),
                  np.stack([2 * x * z - 2 * y * ww, 2 * y * z + 2 * x * ww, 1 - 2 * x * x - 2 * y * y], -1)], 1)
    a = 2 * q1
    t = np.stack([a[:, 3] * -x + a[:, 0] * ww + a[:, 1] * -z - a[:, 2] * -y,
                  a[:, 3] * -y - a[:, 0] * -z + a[:, 1] * ww + a[:, 2] * -x,
                  a[:, 3] * -z + a[:, 0] * -y - a[:, 1] * -x + a[:, 2] * ww], -1)
    return R, t


def pack_rgb(rgb):
    """Colour packed as the renderer reads it: 8-bit r, g, b in bits 16-23,
    8-15 and 0-7 of color_time.x's float bits (the top byte is 0)."""
    c = np.clip(np.rint(np.asarray(rgb, np.float64) * 255.0), 0, 255).astype(np.uint32)
    return ((c[:, 0] << 16) | (c[:, 1] << 8) | c[:, 2]).view(np.float32)


def solver_map_geometry(scene, seed=0, current_time=10.0, warped=True):
    """The scene's surfels as the renderer's five float4 arrays: reference
    vertex + confidence, reference normal + radius (mm), live vertex and
    normal (the reference surfels moved by the scene's warp field, or copies
    when `warped` is False) and (packed colour, initial time, last observed
    time, 0). Confidence in [0, 20) and observation times in
    [current_time - 6, current_time] so that the stable/recent cull of the
    renderer has both outcomes."""
    rng = np.random.default_rng([seed, 104729])
    S = scene.num_surfels
    p = np.asarray(scene.surfel_position, np.float64)
    n = np.asarray(scene.surfel_normal, np.float64)
    # a disc about as wide as the pixel footprint in view 0 (mm): 1.4 to 4.2
    # pixels across there
    m = np.asarray(scene.views[0].initial_camera_se3, np.float64)
    depth = np.abs((p - m[9:12]) @ m[:9].reshape(3, 3).T[:, 2])
    fx = float(scene.views[0].intrinsic[2])
    radius = depth / fx * 1000.0 * rng.uniform(0.5, 1.5, S)
    ref_v = np.concatenate([p, rng.uniform(0.0, 20.0, (S, 1))], 1).astype(np.float32)
    ref_n = np.concatenate([n, radius[:, None]], 1).astype(np.float32)
    if warped:
        R, t = blend_warp(scene.node_se3, scene.surfel_knn, scene.surfel_knn_weight)
        lp = np.einsum("sij,sj->si", R, p) + t
        ln = np.einsum("sij,sj->si", R, n)
    else:
        lp, ln = p, n
    live_v = np.concatenate([lp, ref_v[:, 3:4]], 1).astype(np.float32)
    live_n = np.concatenate([ln, radius[:, None]], 1).astype(np.float32)
    ct = np.zeros((S, 4), np.float32)
    ct[:, 0] = pack_rgb(surface_colour(p))
    ct[:, 1] = rng.integers(0, int(current_time) + 1, S).astype(np.float32)
    ct[:, 2] = (current_time - rng.integers(0, 7, S)).astype(np.float32)
    return dict(reference_vertex_confid=ref_v, reference_normal_radius=ref_n, live_vertex_confid=live_v,
                live_normal_radius=live_n, color_time=ct)


# --------------------------------------------------------------------------
# raw sparse-feature pixel pairs
# --------------------------------------------------------------------------

def with_feature_pairs(scene, per_view=400, seed=0, outlier_fraction=0.1):
    """A copy of `scene` whose feature term comes from raw pixel pairs: per
    view, pairs (x, y, z, w) of a rendered pixel with a surfel and a nearby
    observed pixel (jitter of one pixel, `outlier_fraction` of them up to
    six pixels away), the rendered live vertex map (the reference surface
    moved by the scene's warp field, camera frame) and the observation's
    silhouette edges."""
    import dataclasses
    rng = np.random.default_rng([seed, 7349])
    H, W = scene.height, scene.width
    out = []
    for view in scene.views:
        idx = view.index_map
        ys, xs = np.nonzero(idx != INVALID_INDEX)
        pick = rng.choice(len(xs), size=min(per_view, len(xs)), replace=False)
        x, y = xs[pick], ys[pick]
        far = rng.random(len(x)) < outlier_fraction
        jx = np.where(far, rng.integers(-6, 7, len(x)), rng.integers(-1, 2, len(x)))
        jy = np.where(far, rng.integers(-6, 7, len(x)), rng.integers(-1, 2, len(x)))
        z, w = np.clip(x + jx, 0, W - 1), np.clip(y + jy, 0, H - 1)
        pairs = np.stack([x, y, z, w], 1).astype(np.uint16)
        # live vertex map: warp(init * reference) brought back to the camera
        m = np.asarray(view.initial_camera_se3, np.float64)
        Ri, ti = m[:9].reshape(3, 3).T, m[9:12]
        live = np.zeros((H, W, 4), np.float32)
        s = idx[ys, xs]
        R, t = blend_warp(scene.node_se3, scene.surfel_knn[s], scene.surfel_knn_weight[s])
        ref0 = view.reference_vertex_map[ys, xs, :3].astype(np.float64) @ Ri.T + ti
        lv = np.einsum("sij,sj->si", R, ref0) + t
        live[ys, xs, :3] = (lv - ti) @ Ri
        live[ys, xs, 3] = 1.0
        observed = np.abs(view.vertex_confidence_map[..., 2]) > 0
        pad = np.pad(observed, 1, constant_values=False)
        inner = pad[:-2, 1:-1] & pad[2:, 1:-1] & pad[1:-1, :-2] & pad[1:-1, 2:]
        edge = (observed & ~inner).astype(np.uint8)
        out.append((pairs, live, edge))
    return dataclasses.replace(scene, feature=Correspondences.empty(), feature_pairs=out,
                               terms={**scene.terms, "feature": True})


# --------------------------------------------------------------------------
# inputs of the post-solve deformation and correction
# --------------------------------------------------------------------------

def node_skinning(scene):
    """Each node's 4 nearest nodes (itself first) and their weights, as the
    warp field's nodesKNN / nodesKNNWeight."""
    p = np.asarray(scene.canonical_nodes, np.float64)[:, :3]
    d, i = cKDTree(p).query(p, k=4)
    return i.astype(np.uint16), _knn_weights(d * d, scene.node_radius)


def node_views(scene):
    """Canonical nodes with w encoding the view that sees each one best
    (i + 1 for view i, decoded as i < w <= i + 1): the view in whose camera
    the node is nearest."""
    nodes = np.asarray(scene.canonical_nodes, np.float32).copy()
    best = np.full(len(nodes), np.inf)
    for v, view in enumerate(scene.views):
        m = np.asarray(view.initial_camera_se3, np.float64)
        z = ((nodes[:, :3] - m[9:12]) @ m[:9].reshape(3, 3).T)[:, 2]
        z = np.where(z > 0, z, np.inf)
        better = z < best
        nodes[better, 3] = v + 1
        best[better] = z[better]
    return nodes


def correction_guides(scene, seed=0, valid_fraction=0.5, step_mm=4.0):
    """Per view: a correspondence SE3 map (previous -> current frame, camera
    frame; a small rotation and a translation of a few millimetres, varying
    per pixel), its validity (valid_fraction of the observed pixels) and the
    previous frame's vertex map (the observation)."""
    rng = np.random.default_rng([seed, 3571])
    H, W = scene.height, scene.width
    out = []
    for view in scene.views:
        prev = np.ascontiguousarray(view.vertex_confidence_map, np.float32)
        observed = np.abs(prev[..., 2]) > 0
        valid = (observed & (rng.random((H, W)) < valid_fraction)).astype(np.uint8)
        se3 = np.zeros((H, W, 12), np.float32)
        w = rng.normal(0, np.radians(0.5), (H * W, 3))
        R = rodrigues_batch(w).reshape(H, W, 3, 3)
        se3[..., :9] = np.transpose(R, (0, 1, 3, 2)).reshape(H, W, 9)  # rotation columns
        se3[..., 9:] = rng.normal(0, step_mm * 1e-3, (H, W, 3))
        out.append((se3, valid, prev))
    return out


# --------------------------------------------------------------------------
# the workloads
# --------------------------------------------------------------------------

def sphere_single_view(seed=1, num_nodes=2048, width=640, height=480, rigid_offset=False):
    """Plain method, 1 view: unit-radius sphere section at 1.5 m, fx=fy=570,
    cx=320, cy=240 (scaled with the image size), 2048 nodes, dense depth and
    smooth terms, 3 GN x 10 PCG."""
    sx = width / 640.0
    sy = height / 480.0
    cams = [(np.eye(3), np.zeros(3))]
    shapes = [Ellipsoid((0, 0, 2.5), (1.0, 1.0, 1.0))]
    return _build("sphere_1view", shapes, cams, width, height, 570.0 * sx, 570.0 * sy, 320.0 * sx, 240.0 * sy,
                  num_nodes, seed, rigid_offset=rigid_offset,
                  terms=dict(foreground=False, feature=False, cross_view=False), gn=3, pcg=10)


def torso_multi_view(seed=2, num_nodes=4096, num_views=3, width=640, height=480, features_per_view=1000,
                     cross_per_pair=2000, rigid_offset=False, distance=1.3, auto_radius=False):
    """Multi-view: `num_views` cameras spaced evenly (120 deg for 3) around a
    torso-like ellipsoid (semi-axes 0.25/0.15/0.6 m), all terms, 5 GN x 15 PCG."""
    sx = width / 640.0
    sy = height / 480.0
    center = np.array([0.0, 0.0, distance])
    shapes = [Ellipsoid(center, (0.25, 0.6, 0.15))]
    cams = []
    for k in range(num_views):
        ang = 2 * math.pi * k / num_views
        eye = center + distance * np.array([math.sin(ang), 0.0, -math.cos(ang)])
        R, o = look_at(eye, center)
        if k == 0:
            # frame 0 is camera 0's frame
            R, o = np.eye(3), np.zeros(3)
        cams.append((R, o))
    return _build(f"torso_{num_views}view", shapes, cams, width, height, 570.0 * sx, 570.0 * sy, 320.0 * sx,
                  240.0 * sy, num_nodes, seed, auto_radius=auto_radius, features_per_view=features_per_view,
                  cross_per_pair=cross_per_pair, rigid_offset=rigid_offset,
                  terms=dict(foreground=True, feature=True, cross_view=True), gn=5, pcg=15)


def articulated_body(seed=5, num_nodes=32768, num_views=5, width=1280, height=720, cross_total=20000,
                     distance=2.2, auto_radius=False, focal_scale=1.0):
    """Large single solve: ellipsoid torso + 4 capsule limbs with random joint
    bends <= 30 deg, `num_views` views, 8 GN x 20 PCG. `focal_scale`
    multiplies the focal length (570 px at 640 wide): 5 frames the body so
    that it fills about 87 % of each 1280x720 view, about 4M dense terms."""
    rng = np.random.default_rng(seed + 1000)
    center = np.array([0.0, 0.0, distance])
    shapes = [Ellipsoid(center, (0.25, 0.45, 0.15))]
    limbs = [((-0.3, -0.3), (-1, 0.2)), ((0.3, -0.3), (1, 0.2)), ((-0.12, 0.45), (-0.15, 1)),
             ((0.12, 0.45), (0.15, 1))]
    for (anchor, dirn) in limbs:
        bend = math.radians(rng.uniform(-30, 30))
        d = np.array([dirn[0], dirn[1], 0.0])
        d /= np.linalg.norm(d)
        Rb = rodrigues(np.array([0, 0, 1.0]) * bend)
        d = Rb @ d
        p0 = center + np.array([anchor[0], anchor[1], 0.0])
        p1 = p0 + 0.55 * d
        shapes.append(Capsule(p0, p1, 0.06))
    cams = []
    for k in range(num_views):
        ang = 2 * math.pi * k / num_views
        eye = center + distance * np.array([math.sin(ang), 0.0, -math.cos(ang)])
        R, o = look_at(eye, center)
        if k == 0:
            R, o = np.eye(3), np.zeros(3)
        cams.append((R, o))
    fx = 570.0 * width / 640.0 * focal_scale
    per_pair = cross_total // max(1, num_views)
    return _build("articulated_5view", shapes, cams, width, height, fx, fx, width / 2.0, height / 2.0, num_nodes,
                  seed, auto_radius=auto_radius, features_per_view=0, cross_per_pair=per_pair,
                  terms=dict(foreground=False, feature=False, cross_view=True), gn=8, pcg=20)


def batch_instances(seed=4, count=16, min_nodes=1024, max_nodes=16384, width=640, height=480):
    """Batched uneven solves: node counts log-uniform in [1024, 16384], 1-4
    views each, term mix as the multi-view workload."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        n = int(round(math.exp(rng.uniform(math.log(min_nodes), math.log(max_nodes)))))
        v = int(rng.integers(1, 5))
        out.append(torso_multi_view(seed=seed * 100 + k, num_nodes=n, num_views=v, width=width, height=height,
                                    auto_radius=True))
    return out


def perturb_warp_field(scene, seed, rot_sigma_deg=2.0, trans_sigma=0.005):
    """A new scene sharing every array of `scene` except a fresh initial warp
    field (another draw of the per-node perturbation)."""
    rng = np.random.default_rng(seed)
    n = scene.num_nodes
    pos = scene.canonical_nodes[:, :3].astype(np.float64)
    Rn = rodrigues_batch(rng.normal(0, math.radians(rot_sigma_deg), (n, 3)))
    tn = rng.normal(0, trans_sigma, (n, 3))
    trans = pos - np.einsum("nij,nj->ni", Rn, pos) + tn
    import copy
    s = copy.copy(scene)
    s.node_se3 = se3_to_dq(Rn, trans)
    return s


WORKLOADS = {
    "sphere_1view": sphere_single_view,
    "torso_3view": torso_multi_view,
    "articulated_5view": articulated_body,
}
