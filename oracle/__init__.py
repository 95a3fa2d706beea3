"""Python binding of the CPU oracle - TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may import
this package. It restates the reference NonRigidSolver algorithm on the CPU
(oracle/oracle.cpp) and is used as the checker, never as the product.

The reference cannot be built whole and ships no golden vectors. Its
header-only solver math (dual quaternions, the ICP and smooth-term Jacobians,
the 6x6 Gauss-Jordan inverse, the node-pair encoding, the term offsets, the
image-term Jacobian) is compiled from the reference tree into
oracle/_ref/libref_pin.so (oracle/Makefile, target `ref`) and the oracle is
checked against it (tests/test_ref_pin.py, tests/golden/ref_vectors.npz);
the rest is pinned by known-answer tests (tests/test_oracle.py).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from multiviewdynrecon_b200 import abi

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None


REFERENCE_TREE = "/root/reference"
_REF_PATH = os.path.join(_HERE, "_ref", "libref_pin.so")
_ref_lib = None


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    # the reference-pinning harness needs the reference tree; elsewhere the
    # library built here (oracle/_ref) is used as it is
    if os.path.isdir(REFERENCE_TREE):
        subprocess.run(["make", "-s", "-C", _HERE, "ref", f"REF={REFERENCE_TREE}"], check=True)


def ref_lib():
    """The reference's own header math compiled by oracle/Makefile (target
    `ref`), or None when it has not been built."""
    global _ref_lib
    if _ref_lib is None and os.path.exists(_REF_PATH):
        L = C.CDLL(_REF_PATH)
        vp, u16, u32, i32, f32 = C.c_void_p, C.c_uint16, C.c_uint32, C.c_int, C.c_float
        for name, argt in (("ref_blend_se3", [vp, vp, vp, vp]), ("ref_dq_to_mat34", [vp, vp]),
                           ("ref_mat34_to_dq", [vp, vp]), ("ref_gauss_jordan6", [vp, vp]),
                           ("ref_p2p_jacobian", [vp, vp, vp]), ("ref_p2p_jt_residual", [vp, vp, vp]),
                           ("ref_smooth_jacobian", [vp, vp, i32, vp]), ("ref_smooth_jt_residual", [vp, vp, i32, vp]),
                           ("ref_term_offsets", [vp, vp, vp, vp])):
            getattr(L, name).argtypes = argt
            getattr(L, name).restype = None
        L.ref_huber.argtypes, L.ref_huber.restype = [f32], f32
        L.ref_encode_nodepair.argtypes, L.ref_encode_nodepair.restype = [u16, u16], u32
        L.ref_image_terms.argtypes = [u32, u32, u32, vp, vp, vp, vp, vp, u32, vp, vp, vp, vp, vp, u32, vp, vp]
        L.ref_image_terms.restype = i32
        _ref_lib = L
    return _ref_lib


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(
                os.path.join(_HERE, "oracle.cpp")):
            build()
        L = C.CDLL(_LIB_PATH)
        L.orc_create.restype = C.c_void_p
        L.orc_create.argtypes = [C.POINTER(abi.Config), C.POINTER(abi.Inputs), C.c_int]
        for name in ("orc_destroy", "orc_build_index", "orc_eval_terms", "orc_assemble", "orc_update",
                     "orc_unfreeze"):
            getattr(L, name).argtypes = [C.c_void_p]
            getattr(L, name).restype = None
        L.orc_pcg.argtypes = [C.c_void_p, C.c_uint32]
        L.orc_gn_iteration.argtypes = [C.c_void_p, C.c_uint32]
        L.orc_solve.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32]
        L.orc_set_term_data.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_freeze_decisions.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_freeze_density.argtypes = [C.c_void_p, C.c_void_p]
        L.orc_set_increment.argtypes = [C.c_void_p, C.c_void_p]
        L.orc_set_node_se3.argtypes = [C.c_void_p, C.c_void_p]
        L.orc_energy.restype = C.c_double
        L.orc_energy.argtypes = [C.c_void_p]
        L.orc_energy_now.restype = C.c_double
        L.orc_energy_now.argtypes = [C.c_void_p]
        L.orc_counts.argtypes = [C.c_void_p, C.POINTER(abi.Counts)]
        L.orc_get.restype = C.c_longlong
        L.orc_get.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_size_t, C.c_int]
        L.orc_apply_jtj.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_dq_to_mat34.argtypes = [C.c_void_p, C.c_void_p]
        L.orc_mat34_to_dq.argtypes = [C.c_void_p, C.c_void_p]
        L.orc_apply_twist.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_set_node_se3_f64.argtypes = [C.c_void_p, C.c_void_p]
        L.orc_gauss_jordan_inverse.argtypes = [C.c_void_p, C.c_void_p]
        L.orc_blend_se3.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_huber.argtypes, L.orc_huber.restype = [C.c_float], C.c_float
        L.orc_smooth_rows.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
        L.orc_p2p_rows.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_cholesky_inverse.argtypes = [C.c_void_p, C.c_void_p]
        L.orc_render_solver_maps.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32]
        L.orc_pcg_history.restype = C.c_uint32
        L.orc_pcg_history.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32]
        L.orc_feature_terms.restype = C.c_uint32
        L.orc_feature_terms.argtypes = [C.c_void_p] * 5
        L.orc_forward_warp.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32] + [C.c_void_p] * 6 + \
            [C.c_uint32] + [C.c_void_p] * 4
        L.orc_inverse_warp.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32] + [C.c_void_p] * 6
        L.orc_node_error.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p, C.c_float] + [C.c_void_p] * 6
        L.orc_correct_large_error_nodes.argtypes = [C.c_void_p, C.c_float, C.c_void_p]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


# element type and per-item width of each array id
_ARRAY_SPEC = {
    abi.ARRAY_DENSE_PIXELS: (np.uint16, 4), abi.ARRAY_DENSE_KNN: (np.uint16, 4),
    abi.ARRAY_DENSE_KNN_WEIGHT: (np.float32, 4), abi.ARRAY_FOREGROUND_PIXELS: (np.uint16, 4),
    abi.ARRAY_NODE2TERM_OFFSET: (np.uint32, 1), abi.ARRAY_NODE2TERM_INDEX: (np.uint32, 1),
    abi.ARRAY_HALF_NODEPAIR_KEY: (np.uint32, 1), abi.ARRAY_NODEPAIR_TERM_INDEX: (np.uint32, 1),
    abi.ARRAY_NODEPAIR_KEY: (np.uint32, 1), abi.ARRAY_NODEPAIR_TERM_RANGE: (np.uint32, 2),
    abi.ARRAY_BLKROW_OFFSET: (np.uint32, 1), abi.ARRAY_BINBLOCK_ROWPTR: (np.int32, 1),
    abi.ARRAY_BINBLOCK_COLPTR: (np.int32, 1), abi.ARRAY_TERM_JACOBIAN: (np.float32, 8),
    abi.ARRAY_SMOOTH_TERMS: (np.float32, 12), abi.ARRAY_WARPED_CORRESPONDENCE: (np.float32, 8),
    abi.ARRAY_DIAG_BLOCKS: (np.float32, 36), abi.ARRAY_JTR: (np.float32, 6),
    abi.ARRAY_PRECONDITIONER: (np.float32, 36), abi.ARRAY_OFFDIAG_BLOCKS: (np.float32, 36),
    abi.ARRAY_BINBLOCK_DATA: (np.float32, 1), abi.ARRAY_INCREMENT: (np.float32, 6),
    abi.ARRAY_NODE_SE3: (np.float32, 8), abi.ARRAY_DENSITY_JACOBIAN: (np.float32, 8),
    abi.ARRAY_FEATURE_TERMS: (np.float32, 8), abi.ARRAY_PCG_RESIDUALS: (np.float64, abi.MVDR_PCG_HISTORY),
}
REAL_ARRAYS = {abi.ARRAY_DIAG_BLOCKS, abi.ARRAY_JTR, abi.ARRAY_PRECONDITIONER, abi.ARRAY_OFFDIAG_BLOCKS,
               abi.ARRAY_BINBLOCK_DATA, abi.ARRAY_INCREMENT, abi.ARRAY_NODE_SE3}


class Oracle:
    """CPU restatement of one solve. `fp64` selects double arithmetic."""

    def __init__(self, scene, config, fp64=False):
        self.scene = scene
        self.config = config
        self._keep = []

        def ptr(name, arr):
            a = np.ascontiguousarray(arr)
            self._keep.append(a)
            return a.ctypes.data

        self.inputs = abi.fill_inputs(scene, ptr, bool(config.use_density))
        self.h = lib().orc_create(C.byref(config), C.byref(self.inputs), int(fp64))
        if not self.h:
            raise ValueError("oracle rejected the inputs")
        self.fp64 = fp64

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            lib().orc_destroy(h)
            self.h = None

    # stages
    def pcg_history(self):
        """delta at the start of each PCG iteration of the last PCG solve."""
        n = lib().orc_pcg_history(self.h, None, 0)
        out = np.zeros(n, np.float64)
        lib().orc_pcg_history(self.h, _p(out), n)
        return out

    def feature_terms(self):
        """The feature terms (bound, or selected from raw pixel pairs):
        target (T, 4), reference (T, 4), knn (T, 4) uint16, weights (T, 4)."""
        n = lib().orc_feature_terms(self.h, None, None, None, None)
        t, r, w = (np.zeros((n, 4), np.float32) for _ in range(3))
        k = np.zeros((n, 4), np.uint16)
        lib().orc_feature_terms(self.h, _p(t), _p(r), _p(k), _p(w))
        return t, r, k, w

    def build_index(self):
        lib().orc_build_index(self.h)

    def eval_terms(self):
        lib().orc_eval_terms(self.h)

    def assemble(self):
        lib().orc_assemble(self.h)

    def pcg(self, iters):
        lib().orc_pcg(self.h, iters)

    def update(self):
        lib().orc_update(self.h)

    def gn_iteration(self, pcg):
        lib().orc_gn_iteration(self.h, pcg)

    def solve(self, gn, pcg):
        lib().orc_solve(self.h, gn, pcg)

    def set_term_data(self, term_jr=None, smooth=None, warped=None):
        keep = [None if a is None else np.ascontiguousarray(a, np.float32) for a in (term_jr, smooth, warped)]
        lib().orc_set_term_data(self.h, *[None if a is None else _p(a) for a in keep])

    def freeze(self, term_jr, smooth, density_jr=None):
        """Freeze projected pixels / validity from another run's term data
        (and the density term's pixels when its records are given)."""
        jr = np.ascontiguousarray(term_jr, np.float32).reshape(-1, 8)
        pix = np.ascontiguousarray(jr[:, 7].view(np.uint32))
        sv = np.ascontiguousarray((np.asarray(smooth, np.float32).reshape(-1, 12)[:, 6] != 0).astype(np.uint8))
        lib().orc_freeze_decisions(self.h, _p(pix), _p(sv))
        if density_jr is not None:
            dj = np.ascontiguousarray(density_jr, np.float32).reshape(-1, 8)
            dp = np.ascontiguousarray(dj[:, 7].view(np.uint32))
            lib().orc_freeze_density(self.h, _p(dp))

    def unfreeze(self):
        lib().orc_unfreeze(self.h)

    def set_increment(self, x):
        x = np.ascontiguousarray(x, np.float32)
        lib().orc_set_increment(self.h, _p(x))

    def set_node_se3(self, dq):
        """Continue from another run's warp field (N x 8; float32 is taken as
        is, float64 keeps its full precision)."""
        if np.asarray(dq).dtype == np.float64:
            dq = np.ascontiguousarray(dq, np.float64)
            lib().orc_set_node_se3_f64(self.h, _p(dq))
            return
        dq = np.ascontiguousarray(dq, np.float32)
        lib().orc_set_node_se3(self.h, _p(dq))

    def energy(self):
        return lib().orc_energy(self.h)

    def counts(self):
        c = abi.Counts()
        lib().orc_counts(self.h, C.byref(c))
        return c

    def get(self, which, as_double=False):
        dt, width = _ARRAY_SPEC[which]
        if as_double and which in REAL_ARRAYS:
            dt = np.float64
        cap = 1 << 20
        while True:
            buf = np.empty(cap // np.dtype(dt).itemsize, dt)
            n = lib().orc_get(self.h, which, _p(buf), buf.nbytes, int(as_double))
            if n >= 0:
                out = buf[: n // np.dtype(dt).itemsize]
                return out.reshape(-1, width) if width > 1 else out
            cap *= 4

    def apply_jtj(self, x):
        x = np.ascontiguousarray(x, np.float64)
        y = np.empty_like(x)
        lib().orc_apply_jtj(self.h, _p(x), _p(y))
        return y


# known-answer helpers over the restated math
def dq_to_mat34(dq):
    dq = np.ascontiguousarray(dq, np.float32)
    out = np.empty(12, np.float32)
    lib().orc_dq_to_mat34(_p(dq), _p(out))
    return out


def mat34_to_dq(m):
    m = np.ascontiguousarray(m, np.float32)
    out = np.empty(8, np.float32)
    lib().orc_mat34_to_dq(_p(m), _p(out))
    return out


def apply_twist(dq, tw):
    dq = np.ascontiguousarray(dq, np.float64)
    tw = np.ascontiguousarray(tw, np.float64)
    out = np.empty(8, np.float64)
    lib().orc_apply_twist(_p(dq), _p(tw), _p(out))
    return out


def gauss_jordan_inverse(A):
    A = np.ascontiguousarray(A, np.float64).reshape(36)
    out = np.empty(36, np.float64)
    lib().orc_gauss_jordan_inverse(_p(A), _p(out))
    return out.reshape(6, 6)


def cholesky_inverse(A):
    A = np.ascontiguousarray(A, np.float64).reshape(36)
    out = np.empty(36, np.float64)
    lib().orc_cholesky_inverse(_p(A), _p(out))
    return out.reshape(6, 6)


def render_solver_maps(geometry, params, views, sized=None):
    """The oracle's restatement of the solver-map pass. `geometry`: dict of
    the five (S, 4) float32 surfel arrays; `params`: abi.SolverMapParams;
    `views`: scene views (cameras). Returns per view a dict of host maps
    (the names of abi.SOLVER_MAP_OUTPUTS minus depth_index)."""
    arrs = {k: np.ascontiguousarray(geometry[k], np.float32) for k in abi.SURFEL_ARRAYS}
    n = len(arrs["live_vertex_confid"])
    g = abi.surfel_geometry(n, {k: a.ctypes.data for k, a in arrs.items()})
    H, W = params.height, params.width
    out, mv = [], (abi.SolverMapView * len(views))()
    for v, view in enumerate(views):
        maps = {k: np.zeros((H, W, 4), np.float32) for k in ("reference_vertex_map", "reference_normal_map",
                                                            "live_vertex_map", "live_normal_map",
                                                            "normalized_rgb_map")}
        maps["index_map"] = np.zeros((H, W), np.uint32)
        out.append(maps)
        mv[v] = abi.solver_map_view(view, {k: a.ctypes.data for k, a in maps.items()},
                                     sized_points=bool(sized[v]) if sized is not None else False)
    lib().orc_render_solver_maps(C.byref(g), C.byref(params), mv, len(views))
    return out


def _f32(a, shape=None):
    a = np.ascontiguousarray(a, np.float32)
    return a if shape is None else a.reshape(shape)


def forward_warp(field, knn, weight, vertex, normal, node_knn=None, node_weight=None, nodes=None):
    """SurfelNodeDeformer::ForwardWarpSurfelsAndNodes on host arrays: returns
    live vertices, live normals and (with nodes) live nodes."""
    field = _f32(field, (-1, 8))
    knn = np.ascontiguousarray(knn, np.uint16)
    w, v, n = _f32(weight), _f32(vertex), _f32(normal)
    S = len(knn)
    ov, on = np.zeros((S, 4), np.float32), np.zeros((S, 4), np.float32)
    N = 0 if nodes is None else len(nodes)
    nk = np.ascontiguousarray(node_knn if N else np.zeros((0, 4)), np.uint16)
    nw, nd = _f32(node_weight if N else np.zeros((0, 4))), _f32(nodes if N else np.zeros((0, 4)))
    live = np.zeros((N, 4), np.float32)
    lib().orc_forward_warp(_p(field), len(field), S, _p(knn), _p(w), _p(v), _p(n), _p(ov), _p(on), N, _p(nk),
                           _p(nw), _p(nd), _p(live))
    return ov, on, live


def inverse_warp(field, knn, weight, vertex, normal, correct=None):
    """SurfelNodeDeformer::InverseWarpSurfels on host arrays; `correct` is
    (S, 12) mat34 (rotation columns, translation) or None."""
    field = _f32(field, (-1, 8))
    knn = np.ascontiguousarray(knn, np.uint16)
    w, v, n = _f32(weight), _f32(vertex), _f32(normal)
    S = len(knn)
    ov, on = np.zeros((S, 4), np.float32), np.zeros((S, 4), np.float32)
    cs = None if correct is None else _f32(correct, (-1, 12))
    lib().orc_inverse_warp(_p(field), len(field), None if cs is None else _p(cs), S, _p(knn), _p(w), _p(v), _p(n),
                           _p(ov), _p(on))
    return ov, on


def node_error(scene, field, threshold=0.2, maps=False):
    """DenseDepthHandler::ComputeNodewiseError (+ the two error maps) on the
    scene's maps with the warp field `field` (N, 8)."""
    keep = []

    def ptr(name, arr):
        a = np.ascontiguousarray(arr)
        keep.append(a)
        return a.ctypes.data

    inp = abi.fill_inputs(scene, ptr)
    field = _f32(field, (-1, 8))
    N, V, W, H = scene.num_nodes, scene.num_views, scene.width, scene.height
    out = {k: np.zeros(N, np.float32) for k in ("accumulated_error", "accumulated_weight", "united_error")}
    out["large_error_mark"] = np.zeros(N, np.uint32)
    am = [np.zeros((H, W), np.float32) for _ in range(V)] if maps else []
    nm = [np.zeros((H, W), np.float32) for _ in range(V)] if maps else []
    amp = (C.c_void_p * V)(*[a.ctypes.data for a in am]) if maps else None
    nmp = (C.c_void_p * V)(*[a.ctypes.data for a in nm]) if maps else None
    lib().orc_node_error(C.byref(inp), W, H, _p(field), threshold, _p(out["accumulated_error"]),
                         _p(out["accumulated_weight"]), _p(out["united_error"]), _p(out["large_error_mark"]),
                         C.cast(amp, C.c_void_p) if maps else None, C.cast(nmp, C.c_void_p) if maps else None)
    if maps:
        out["alignment_error_map"], out["node_error_map"] = am, nm
    return out


def correct_large_error_nodes(scene, guides, united_error, node_se3, live_nodes, node_knn, node_weight, live_vertex,
                              live_normal, surfel_knn, surfel_weight, threshold=0.2, node_radius=None):
    """NonRigidSolver::CorrectLargeErrorNode (correspondence form) on host
    arrays; `guides` per view (se3 map (H, W, 12), valid (H, W) uint8,
    previous vertex map (H, W, 4)). Returns the corrected arrays and the
    per-node corrections."""
    keep = []

    def ptr(name, arr):
        a = np.ascontiguousarray(arr)
        keep.append(a)
        return a.ctypes.data

    inp = abi.fill_inputs(scene, ptr)
    res = {"node_se3": _f32(node_se3, (-1, 8)).copy(), "live_nodes": _f32(live_nodes).copy(),
           "live_vertex": _f32(live_vertex).copy(), "live_normal": _f32(live_normal).copy(),
           "correction": np.zeros((scene.num_nodes, 8), np.float32)}
    c = abi.Correction()
    c.width, c.height = scene.width, scene.height
    for v, (se3, valid, prev) in enumerate(guides):
        arrs = (_f32(se3), np.ascontiguousarray(valid, np.uint8), _f32(prev))
        keep.extend(arrs)
        c.views[v].se3_map, c.views[v].valid_map, c.views[v].previous_vertex_map = [a.ctypes.data for a in arrs]
        c.views[v].pitch = 0
    ue = _f32(united_error)
    nk, nw = np.ascontiguousarray(node_knn, np.uint16), _f32(node_weight)
    sk, sw = np.ascontiguousarray(surfel_knn, np.uint16), _f32(surfel_weight)
    keep.extend([ue, nk, nw, sk, sw])
    c.united_error, c.error_threshold = ue.ctypes.data, threshold
    c.node_se3, c.live_nodes = res["node_se3"].ctypes.data, res["live_nodes"].ctypes.data
    c.node_knn, c.node_knn_weight = nk.ctypes.data, nw.ctypes.data
    c.num_surfels = len(sk)
    c.live_vertex, c.live_normal = res["live_vertex"].ctypes.data, res["live_normal"].ctypes.data
    c.surfel_knn, c.surfel_knn_weight = sk.ctypes.data, sw.ctypes.data
    c.correction = res["correction"].ctypes.data
    lib().orc_correct_large_error_nodes(C.byref(inp), scene.node_radius if node_radius is None else node_radius,
                                        C.byref(c))
    return res
