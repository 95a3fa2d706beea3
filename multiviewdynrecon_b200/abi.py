"""ctypes mirror of include/mvdr.h.

The structures here must match the C declarations field for field; the
layout test in tests/test_abi.py checks sizes and offsets against the compiled
library's own `mvdr_abi_layout` report.
"""
from __future__ import annotations

import ctypes as C

MVDR_ABI_VERSION = 3
MVDR_MAX_VIEWS = 8
MVDR_INVALID_INDEX = 0xFFFFFFFF

MVDR_OK, MVDR_EINVAL, MVDR_ECAPACITY, MVDR_ECUDA, MVDR_ETIMEOUT, MVDR_ENONFINITE, MVDR_ESTATE = range(7)
STATUS_NAMES = {0: "MVDR_OK", 1: "MVDR_EINVAL", 2: "MVDR_ECAPACITY", 3: "MVDR_ECUDA", 4: "MVDR_ETIMEOUT",
                5: "MVDR_ENONFINITE", 6: "MVDR_ESTATE"}

PRECISION_FP32, PRECISION_MIXED = 0, 1
MODE_MATERIALIZED, MODE_MATRIX_FREE = 0, 1
COMPAT_REF_VIEW_LOOKUP = 1
COMPAT_REF_FOREGROUND_FRAME = 2
(STAGE_INDEX, STAGE_TERMS, STAGE_DIAG, STAGE_OFFDIAG, STAGE_SPMV, STAGE_PCG_UPDATE, STAGE_UPDATE,
 STAGE_DIRECTION, STAGE_MATRIX_FREE, STAGE_SCALE) = range(10)
# SpMV tile shapes (block rows per CTA, threads per scalar row / 6, form) in
# the autotuner's order. Form 0 reads a lower block's row and exchanges the
# column sums through shared memory; form 1 reads its column.
SPMV_SHAPES = [(16, 2, 0), (8, 2, 0), (16, 1, 0), (32, 1, 0), (16, 3, 0), (8, 4, 0), (32, 2, 0),
               (16, 1, 1), (32, 1, 1), (8, 2, 1), (16, 2, 1), (4, 4, 1)]
NUM_SPMV_SHAPES = len(SPMV_SHAPES)

(ARRAY_DENSE_PIXELS, ARRAY_DENSE_KNN, ARRAY_DENSE_KNN_WEIGHT, ARRAY_FOREGROUND_PIXELS, ARRAY_NODE2TERM_OFFSET,
 ARRAY_NODE2TERM_INDEX, ARRAY_HALF_NODEPAIR_KEY, ARRAY_NODEPAIR_TERM_INDEX, ARRAY_NODEPAIR_KEY,
 ARRAY_NODEPAIR_TERM_RANGE, ARRAY_BLKROW_OFFSET, ARRAY_BINBLOCK_ROWPTR, ARRAY_BINBLOCK_COLPTR,
 ARRAY_TERM_JACOBIAN, ARRAY_SMOOTH_TERMS, ARRAY_WARPED_CORRESPONDENCE, ARRAY_DIAG_BLOCKS, ARRAY_JTR,
 ARRAY_PRECONDITIONER, ARRAY_OFFDIAG_BLOCKS, ARRAY_BINBLOCK_DATA, ARRAY_INCREMENT, ARRAY_NODE_SE3,
 ARRAY_DENSITY_JACOBIAN, ARRAY_FEATURE_TERMS, ARRAY_PCG_RESIDUALS) = range(26)
MVDR_PCG_HISTORY = 257


class Float4(C.Structure):
    _fields_ = [("x", C.c_float), ("y", C.c_float), ("z", C.c_float), ("w", C.c_float)]


class DualQuaternion(C.Structure):
    _fields_ = [("q0", C.c_float * 4), ("q1", C.c_float * 4)]


class Mat34(C.Structure):
    _fields_ = [("rot", C.c_float * 9), ("trans", C.c_float * 3)]


class Intrinsic(C.Structure):
    _fields_ = [("principal_x", C.c_float), ("principal_y", C.c_float), ("focal_x", C.c_float),
                ("focal_y", C.c_float)]


class Penalty(C.Structure):
    _fields_ = [("smooth", C.c_float), ("density", C.c_float), ("foreground", C.c_float), ("feature", C.c_float),
                ("cross_view", C.c_float)]


class Config(C.Structure):
    _fields_ = [
        ("abi_version", C.c_uint32),
        ("max_nodes", C.c_uint32), ("max_views", C.c_uint32), ("image_width", C.c_uint32),
        ("image_height", C.c_uint32), ("max_surfels", C.c_uint32), ("max_feature_terms", C.c_uint32),
        ("max_cross_terms", C.c_uint32), ("max_dense_terms", C.c_uint32), ("max_foreground_terms", C.c_uint32),
        ("max_node_pairs", C.c_uint32), ("max_terms_per_node", C.c_uint32),
        ("node_radius", C.c_float), ("precision", C.c_int32), ("mode", C.c_int32),
        ("use_foreground", C.c_int32), ("use_feature", C.c_int32), ("use_cross_view", C.c_int32),
        ("use_elastic_penalty", C.c_int32), ("num_global_iterations", C.c_int32), ("compat_flags", C.c_uint32),
        ("penalty", Penalty), ("use_density", C.c_int32), ("pcg_tolerance", C.c_float),
        ("recompute_jacobians", C.c_int32),
    ]


class ViewInputs(C.Structure):
    _fields_ = [
        ("reference_vertex_map", C.c_void_p), ("reference_normal_map", C.c_void_p), ("index_map", C.c_void_p),
        ("vertex_confidence_map", C.c_void_p), ("normal_radius_map", C.c_void_p),
        ("filtered_foreground_mask", C.c_void_p), ("foreground_mask_gradient", C.c_void_p),
        ("pitch", C.c_uint32), ("intrinsic", Intrinsic), ("world2camera", Mat34),
        ("initial_camera_se3", Mat34),
        ("normalized_rgb_map", C.c_void_p), ("density_map", C.c_void_p), ("density_gradient_map", C.c_void_p),
    ]


class ViewTextures(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in (
        "reference_vertex_map", "reference_normal_map", "index_map", "normalized_rgb_map", "vertex_confidence_map",
        "normal_radius_map", "filtered_foreground_mask", "foreground_mask_gradient", "density_map",
        "density_gradient_map")]


class Correspondences(C.Structure):
    _fields_ = [("count", C.c_uint32), ("target_vertex", C.c_void_p), ("reference_vertex", C.c_void_p),
                ("knn", C.c_void_p), ("knn_weight", C.c_void_p)]


class FeaturePairs(C.Structure):
    _fields_ = [("count", C.c_uint32 * MVDR_MAX_VIEWS), ("pixel_pairs", C.c_void_p * MVDR_MAX_VIEWS),
                ("live_vertex_map", C.c_void_p * MVDR_MAX_VIEWS), ("edge_mask", C.c_void_p * MVDR_MAX_VIEWS)]


class Inputs(C.Structure):
    _fields_ = [
        ("num_views", C.c_uint32), ("num_nodes", C.c_uint32), ("num_surfels", C.c_uint32),
        ("num_graph_edges", C.c_uint32), ("views", ViewInputs * MVDR_MAX_VIEWS),
        ("surfel_knn", C.c_void_p), ("surfel_knn_weight", C.c_void_p), ("node_se3", C.c_void_p),
        ("canonical_node_coords", C.c_void_p), ("node_graph", C.c_void_p),
        ("feature", Correspondences), ("cross_view", Correspondences), ("feature_pairs", FeaturePairs),
    ]


class Counts(C.Structure):
    _fields_ = [(n, C.c_uint32) for n in (
        "dense_terms", "smooth_terms", "foreground_terms", "feature_terms", "cross_terms", "node2term_entries",
        "nodepair_entries", "half_pairs", "num_bins", "binblock_nnz", "error_flags", "reserved")]


class SurfelGeometry(C.Structure):
    _fields_ = [("num_surfels", C.c_uint32), ("reference_vertex_confid", C.c_void_p),
                ("reference_normal_radius", C.c_void_p), ("live_vertex_confid", C.c_void_p),
                ("live_normal_radius", C.c_void_p), ("color_time", C.c_void_p)]


class SolverMapParams(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("max_depth", C.c_float),
                ("current_time", C.c_float), ("confidence_threshold", C.c_float), ("time_threshold", C.c_float)]


class SolverMapView(C.Structure):
    _fields_ = [("world2camera", Mat34), ("initial_camera_se3", Mat34), ("intrinsic", Intrinsic),
                ("sized_points", C.c_int32), ("pitch", C.c_uint32), ("reference_vertex_map", C.c_void_p),
                ("reference_normal_map", C.c_void_p), ("live_vertex_map", C.c_void_p),
                ("live_normal_map", C.c_void_p), ("index_map", C.c_void_p), ("normalized_rgb_map", C.c_void_p),
                ("depth_index", C.c_void_p)]


class DeformSurfels(C.Structure):
    _fields_ = [("num_surfels", C.c_uint32), ("knn", C.c_void_p), ("knn_weight", C.c_void_p),
                ("in_vertex", C.c_void_p), ("in_normal", C.c_void_p), ("out_vertex", C.c_void_p),
                ("out_normal", C.c_void_p)]


class DeformNodes(C.Structure):
    _fields_ = [("num_nodes", C.c_uint32), ("knn", C.c_void_p), ("knn_weight", C.c_void_p),
                ("canonical_nodes", C.c_void_p), ("live_nodes", C.c_void_p)]


class NodeError(C.Structure):
    _fields_ = [("accumulated_error", C.c_void_p), ("accumulated_weight", C.c_void_p),
                ("united_error", C.c_void_p), ("large_error_mark", C.c_void_p), ("threshold", C.c_float),
                ("alignment_error_map", C.c_void_p * MVDR_MAX_VIEWS), ("node_error_map", C.c_void_p * MVDR_MAX_VIEWS)]


class CorrectionView(C.Structure):
    _fields_ = [("se3_map", C.c_void_p), ("valid_map", C.c_void_p), ("previous_vertex_map", C.c_void_p),
                ("pitch", C.c_uint32)]


class Correction(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("views", CorrectionView * MVDR_MAX_VIEWS),
                ("united_error", C.c_void_p), ("error_threshold", C.c_float), ("node_se3", C.c_void_p),
                ("live_nodes", C.c_void_p), ("node_knn", C.c_void_p), ("node_knn_weight", C.c_void_p),
                ("num_surfels", C.c_uint32), ("live_vertex", C.c_void_p), ("live_normal", C.c_void_p),
                ("surfel_knn", C.c_void_p), ("surfel_knn_weight", C.c_void_p), ("correction", C.c_void_p)]


STRUCTS = {"mvdr_float4": Float4, "mvdr_dual_quaternion": DualQuaternion, "mvdr_mat34": Mat34,
           "mvdr_intrinsic": Intrinsic, "mvdr_penalty": Penalty, "mvdr_config": Config,
           "mvdr_view_inputs": ViewInputs, "mvdr_correspondences": Correspondences, "mvdr_inputs": Inputs,
           "mvdr_counts": Counts, "mvdr_view_textures": ViewTextures, "mvdr_feature_pairs": FeaturePairs,
           "mvdr_surfel_geometry": SurfelGeometry,
           "mvdr_solver_map_params": SolverMapParams, "mvdr_solver_map_view": SolverMapView,
           "mvdr_deform_surfels": DeformSurfels, "mvdr_deform_nodes": DeformNodes, "mvdr_node_error": NodeError,
           "mvdr_correction_view": CorrectionView, "mvdr_correction": Correction}


def make_config(scene=None, *, max_nodes=4096, max_views=3, width=640, height=480, precision=PRECISION_MIXED,
                mode=MODE_MATERIALIZED, use_foreground=None, use_feature=None, use_cross_view=None,
                max_surfels=None, max_feature_terms=None, max_cross_terms=None, elastic=True,
                num_global_iterations=1 << 20, compat_flags=0, node_radius=0.025, use_density=None,
                pcg_tolerance=0.0, recompute_jacobians=False):
    """Configuration for a scene (or explicit capacities). With the elastic
    schedule on and num_global_iterations large, every iteration uses the
    global lambdas (all terms active)."""
    cfg = Config()
    cfg.abi_version = MVDR_ABI_VERSION
    if scene is not None:
        max_nodes = max(max_nodes if max_nodes != 4096 else 0, scene.num_nodes)
        max_views = scene.num_views
        width, height = scene.width, scene.height
        terms = scene.terms or {}
        if use_foreground is None:
            use_foreground = terms.get("foreground", False)
        if use_feature is None:
            use_feature = terms.get("feature", False)
        if use_cross_view is None:
            use_cross_view = terms.get("cross_view", False)
        if use_density is None:
            use_density = terms.get("density", False)
        max_surfels = max_surfels or scene.num_surfels
        pairs = sum(len(p[0]) for p in (getattr(scene, "feature_pairs", None) or []))
        max_feature_terms = max_feature_terms if max_feature_terms is not None else max(scene.feature.count, pairs)
        max_cross_terms = max_cross_terms if max_cross_terms is not None else scene.cross_view.count
        node_radius = scene.node_radius
    cfg.max_nodes = max_nodes
    cfg.max_views = max_views
    cfg.image_width = width
    cfg.image_height = height
    cfg.max_surfels = max_surfels or max_views * width * height
    cfg.max_feature_terms = max_feature_terms or 0
    cfg.max_cross_terms = max_cross_terms or 0
    cfg.max_dense_terms = 0
    cfg.max_foreground_terms = 0
    cfg.max_node_pairs = 0
    cfg.max_terms_per_node = 0
    cfg.node_radius = node_radius
    cfg.precision = precision
    cfg.mode = mode
    cfg.use_foreground = int(bool(use_foreground))
    cfg.use_feature = int(bool(use_feature))
    cfg.use_cross_view = int(bool(use_cross_view))
    cfg.use_elastic_penalty = int(bool(elastic))
    cfg.num_global_iterations = num_global_iterations
    cfg.compat_flags = compat_flags
    cfg.penalty = Penalty(2.5, 0.0, 0.0, 0.7, 0.1)  # PenaltyConstants::setDefaultValue
    cfg.use_density = int(bool(use_density))
    cfg.pcg_tolerance = pcg_tolerance
    cfg.recompute_jacobians = int(bool(recompute_jacobians))
    return cfg


def _mat34(a):
    m = Mat34()
    for i in range(9):
        m.rot[i] = float(a[i])
    for i in range(3):
        m.trans[i] = float(a[9 + i])
    return m


def fill_inputs(scene, ptr, density=False):
    """Build an Inputs struct for `scene`; `ptr(name, array)` returns the
    address to store for each array (a host numpy pointer or a device
    pointer). Names are stable keys so callers can cache uploads. The density
    maps are included only with `density` (a configuration with the density
    term on)."""
    inp = Inputs()
    inp.num_views = scene.num_views
    inp.num_nodes = scene.num_nodes
    inp.num_surfels = scene.num_surfels
    inp.num_graph_edges = len(scene.node_graph)
    for v, view in enumerate(scene.views):
        vi = inp.views[v]
        vi.reference_vertex_map = ptr(f"v{v}.ref_v", view.reference_vertex_map)
        vi.reference_normal_map = ptr(f"v{v}.ref_n", view.reference_normal_map)
        vi.index_map = ptr(f"v{v}.index", view.index_map)
        vi.vertex_confidence_map = ptr(f"v{v}.obs_v", view.vertex_confidence_map)
        vi.normal_radius_map = ptr(f"v{v}.obs_n", view.normal_radius_map)
        vi.filtered_foreground_mask = ptr(f"v{v}.fg", view.filtered_foreground_mask)
        vi.foreground_mask_gradient = ptr(f"v{v}.fg_grad", view.foreground_mask_gradient)
        if density and getattr(view, "density_map", None) is not None:
            vi.normalized_rgb_map = ptr(f"v{v}.rgb", view.normalized_rgb_map)
            vi.density_map = ptr(f"v{v}.dens", view.density_map)
            vi.density_gradient_map = ptr(f"v{v}.dens_grad", view.density_gradient_map)
        vi.pitch = 0
        vi.intrinsic = Intrinsic(*[float(x) for x in view.intrinsic])
        vi.world2camera = _mat34(view.world2camera)
        vi.initial_camera_se3 = _mat34(view.initial_camera_se3)
    inp.surfel_knn = ptr("surfel_knn", scene.surfel_knn)
    inp.surfel_knn_weight = ptr("surfel_w", scene.surfel_knn_weight)
    inp.node_se3 = ptr("node_se3", scene.node_se3)
    inp.canonical_node_coords = ptr("nodes", scene.canonical_nodes)
    inp.node_graph = ptr("graph", scene.node_graph)
    for name, corr, dst in (("feat", scene.feature, inp.feature), ("cross", scene.cross_view, inp.cross_view)):
        dst.count = corr.count
        dst.target_vertex = ptr(f"{name}.target", corr.target_vertex)
        dst.reference_vertex = ptr(f"{name}.ref", corr.reference_vertex)
        dst.knn = ptr(f"{name}.knn", corr.knn)
        dst.knn_weight = ptr(f"{name}.w", corr.knn_weight)
    for v, (pairs, live, edge) in enumerate(getattr(scene, "feature_pairs", None) or []):
        inp.feature_pairs.count[v] = len(pairs)
        inp.feature_pairs.pixel_pairs[v] = ptr(f"v{v}.fp_pairs", pairs)
        inp.feature_pairs.live_vertex_map[v] = ptr(f"v{v}.fp_live", live)
        inp.feature_pairs.edge_mask[v] = None if edge is None else ptr(f"v{v}.fp_edge", edge)
    return inp


SOLVER_MAP_OUTPUTS = ("reference_vertex_map", "reference_normal_map", "live_vertex_map", "live_normal_map",
                      "index_map", "normalized_rgb_map", "depth_index")
SURFEL_ARRAYS = ("reference_vertex_confid", "reference_normal_radius", "live_vertex_confid", "live_normal_radius",
                 "color_time")


def surfel_geometry(num_surfels, ptrs):
    """mvdr_surfel_geometry over the five arrays `ptrs[name]` (addresses)."""
    g = SurfelGeometry()
    g.num_surfels = num_surfels
    for name in SURFEL_ARRAYS:
        setattr(g, name, ptrs[name])
    return g


def solver_map_params(width, height, max_depth=3.0, current_time=10.0, confidence_threshold=10.0,
                      time_threshold=3.0):
    return SolverMapParams(width, height, max_depth, current_time, confidence_threshold, time_threshold)


def solver_map_view(view, ptrs, sized_points=False, pitch=0):
    """mvdr_solver_map_view for a scene view's camera (world2camera,
    initial_camera_se3, intrinsic); `ptrs` maps SOLVER_MAP_OUTPUTS names to
    addresses (absent or None: that map is not written)."""
    mv = SolverMapView()
    mv.world2camera = _mat34(view.world2camera)
    mv.initial_camera_se3 = _mat34(view.initial_camera_se3)
    mv.intrinsic = Intrinsic(*[float(x) for x in view.intrinsic])
    mv.sized_points = int(bool(sized_points))
    mv.pitch = pitch
    for name in SOLVER_MAP_OUTPUTS:
        setattr(mv, name, ptrs.get(name))
    return mv

