/*
 * mvdr.h - C ABI of the B200-native non-rigid Gauss-Newton solver.
 *
 * This library replaces the NonRigidSolver stage of MultiViewDynRecon
 * (core/NonRigidSolver/NonRigidSolver.h:78-541). The reference drives that
 * stage through three calls:
 *
 *   SetSolverInput(...)        core/NonRigidSolver/NonRigidSolver.h:133-140
 *   SolveNonRigidAlignment()   core/NonRigidSolver/NonRigidSolver.h:254
 *   SolvedNodeSE3()            core/NonRigidSolver/NonRigidSolver.h:214
 *
 * and they map to mvdr_set_inputs / mvdr_solve / mvdr_get_node_se3 below.
 * The remaining entry points expose the intermediate products of the solve
 * (term index, Jacobians, JtJ blocks, preconditioner, PCG increment) so that a
 * caller can check them against the reference's host sanity-check routines.
 *
 * Conventions
 *  - All structs are plain C, no CUDA or torch types. Streams are passed as
 *    void* and interpreted as cudaStream_t (NULL = legacy default stream).
 *  - Array pointers in mvdr_inputs are DEVICE pointers owned by the caller
 *    (non-owning views, like the reference's DeviceArrayView). They must stay
 *    valid until the next mvdr_set_inputs on the same solver.
 *  - Every workspace buffer is allocated by mvdr_create / mvdr_batch_create.
 *    Nothing is allocated by mvdr_set_inputs, build_index, gn_iteration or
 *    solve. (mvdr_set_inputs_host allocates its input copies once; the
 *    diagnostic mvdr_get_array exports use a temporary buffer.)
 *  - Every call returns an mvdr_status. No call aborts the process; a CUDA
 *    error is returned as MVDR_ECUDA and its text is kept for
 *    mvdr_last_error_string.
 *  - A solver is used by one host thread at a time; all work is enqueued on
 *    the stream given to each call.
 */
#ifndef MVDR_H_
#define MVDR_H_

#include <stddef.h>
#include <stdint.h>

#if defined(_WIN32)
#define MVDR_API __declspec(dllexport)
#else
#define MVDR_API __attribute__((visibility("default")))
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define MVDR_ABI_VERSION 3u
#define MVDR_MAX_VIEWS 8u
#define MVDR_INVALID_INDEX 0xFFFFFFFFu

/* Status codes. The reference aborts on these conditions instead
 * (CHECKCUDA exit, base/DeviceAPI/safe_call.hpp:58-72; ResizeArrayOrException,
 * base/DeviceReadWrite/DeviceBufferArray.h:134-141). */
typedef enum mvdr_status {
    MVDR_OK = 0,
    MVDR_EINVAL = 1,      /* bad argument or inconsistent sizes            */
    MVDR_ECAPACITY = 2,   /* a size exceeds the capacity given at create    */
    MVDR_ECUDA = 3,       /* a CUDA runtime call failed                     */
    MVDR_ETIMEOUT = 4,    /* a bounded device-side wait gave up             */
    MVDR_ENONFINITE = 5,  /* NaN/Inf found in inputs or in the solution     */
    MVDR_ESTATE = 6       /* call out of order (e.g. solve before inputs)   */
} mvdr_status;

/* Arithmetic of the linear solve.
 * FP32:  everything in float; Gauss-Jordan 6x6 inverse; float dot products
 *        (the reference's arithmetic, BlockPCG.cuh:187-458,
 *        BlockDiagonalPreconditionerInverse.cu:7-41).
 * MIXED: Jacobians, stored residuals and PCG vectors in float. Double is used
 *        where float rounding would move the increment by more than 1e-4:
 *        the warped-point / residual chain of each term (positions of about
 *        1 m give residuals of about 1 mm), the accumulation and storage of the
 *        JtJ blocks, the accumulation of Jt r, the SpMV row sums, the PCG dot
 *        products and norms, and the 6x6 block Cholesky of the
 *        preconditioner. */
typedef enum mvdr_precision {
    MVDR_PRECISION_FP32 = 0,
    MVDR_PRECISION_MIXED = 1
} mvdr_precision;

/* How PCG applies JtJ.
 * MATERIALIZED: off-diagonal 6x6 blocks are assembled into BSR storage once
 *   per Gauss-Newton iteration (JtJMaterializer.cu:270-528).
 * MATRIX_FREE: JtJ.p is evaluated per PCG iteration from the term Jacobians
 *   through the adjoint pair J.p / Jt.y (ApplyJacobianDot.cu:127-198,
 *   ApplyJacobianTransposeDot.cu:29-155). Unlike the reference's matrix-free
 *   operator it includes the cross-view term and the 1e-2 diagonal damping,
 *   so both modes solve the same system. */
typedef enum mvdr_mode {
    MVDR_MODE_MATERIALIZED = 0,
    MVDR_MODE_MATRIX_FREE = 1
} mvdr_mode;

/* Compatibility switches reproducing reference behaviour that this library
 * corrects by default. */
enum {
    /* Sample each compacted pixel's maps by the cumulative per-view lookup of
     * CalculateDensityMapCameraViewDpt (DenseDepthJacobianResidual.cu:14-22)
     * instead of the pixel's own view tag. Only differs when num_views > 1. */
    MVDR_COMPAT_REF_VIEW_LOOKUP = 1u << 0,
    /* Warp the foreground (and density) term's reference vertex as it is
     * stored in its camera's frame, as computeImageDensityJacobainAndResidual
     * does (density_map_jacobian.cuh:32-36), instead of first moving it to
     * frame 0 with InitialCameraSE3 like the dense-depth term
     * (DenseDepthJacobianResidual.cu:43-50) and the foreground pixel
     * selection (DensityForegroundMapHandler.cu:60-72). Only differs for
     * views whose InitialCameraSE3 is not the identity. */
    MVDR_COMPAT_REF_FOREGROUND_FRAME = 1u << 1
};

typedef struct mvdr_float4 { float x, y, z, w; } mvdr_float4;

/* Same memory layout as the reference DualQuaternion
 * (math/DualQuaternion/DualQuaternion.h:99-102): two quaternions stored as
 * float4 (x, y, z, w), real part q0 first. 32 bytes. */
typedef struct mvdr_dual_quaternion { float q0[4]; float q1[4]; } mvdr_dual_quaternion;

/* Same layout as the reference mat34 (math/MatUtils.h:19-20, 401-403): the
 * rotation as three float3 COLUMNS, then the translation. 48 bytes. */
typedef struct mvdr_mat34 { float rot[9]; float trans[3]; } mvdr_mat34;

/* Same field order as the reference Intrinsic (base/CommonTypes.h:79-105). */
typedef struct mvdr_intrinsic { float principal_x, principal_y, focal_x, focal_y; } mvdr_intrinsic;

/* Term weights lambda (PenaltyConstants.h:9-46). The dense-depth weight is
 * fixed at 1 as in the reference. */
typedef struct mvdr_penalty {
    float smooth;
    float density;
    float foreground;
    float feature;
    float cross_view;
} mvdr_penalty;

typedef struct mvdr_config {
    uint32_t abi_version;        /* must be MVDR_ABI_VERSION                  */
    /* capacities (the reference's compile-time maxima, made runtime) */
    uint32_t max_nodes;          /* <= 65535                                   */
    uint32_t max_views;          /* <= MVDR_MAX_VIEWS                          */
    uint32_t image_width;
    uint32_t image_height;
    uint32_t max_surfels;
    uint32_t max_feature_terms;
    uint32_t max_cross_terms;
    uint32_t max_dense_terms;    /* 0: max_views * width * height              */
    uint32_t max_foreground_terms; /* 0: max_dense_terms                       */
    uint32_t max_node_pairs;     /* unique unordered pairs; 0: 16 * max_nodes  */
    uint32_t max_terms_per_node; /* terms touching one node; 0: 4096           */
    /* numerics */
    float node_radius;           /* NODE_RADIUS (base/GlobalConfigs.h:85)      */
    int32_t precision;           /* mvdr_precision                            */
    int32_t mode;                /* mvdr_mode                                 */
    int32_t use_foreground;      /* foreground-mask term                      */
    int32_t use_feature;         /* sparse feature term                       */
    int32_t use_cross_view;      /* cross-view correspondence term            */
    int32_t use_elastic_penalty; /* global/local lambda schedule              */
    int32_t num_global_iterations; /* GN iterations that use global lambdas   */
    uint32_t compat_flags;       /* MVDR_COMPAT_*                             */
    /* penalties used when use_elastic_penalty == 0; with the schedule on, the
     * values of PenaltyConstants.cpp:25-51 are used instead. */
    mvdr_penalty penalty;
    /* density (colour) term: a second scalar residual on every dense-depth
     * pixel, observed grey level minus the rendered one, as the reference
     * adds it under USE_DENSE_IMAGE_DENSITY_TERM (PreconditionerBlocked.cu:
     * 216-219, JtDotResidualIndexed.cu:162-165, JtJMaterializer.cu:312-315,
     * ResidualEvaluator.cu:94-99). Its weight is 1e-2 in the local phase of
     * the schedule and 0 in the global phase (PenaltyConstants.cpp:25-45),
     * penalty.density without the schedule. Needs the three density maps of
     * every view. */
    int32_t use_density;
    /* Convergence check of every PCG solve (BlockPCG::SolveConvergeChecked,
     * BlockPCG.cuh:339-377): the solve stops after the first iteration whose
     * delta = r.M^-1 r is below pcg_tolerance^2 times the initial delta, the
     * test made on the device (the later iterations' kernels of that instance
     * return at once), so solves stay capturable in a CUDA graph. 0 (the
     * default) runs the fixed iteration count (BlockPCG::Solve). The launched
     * PCG form only: with a tolerance the persistent form is not used. */
    float pcg_tolerance;
    /* Matrix-free mode only: the J.d / Jt.y products of every PCG iteration
     * evaluate each dense and foreground pixel term again from the maps and
     * the warp field (as ApplyJtJMatrixFreeIndexed.cu:222-348 does) instead
     * of reading the 32-byte record the term evaluation stored. The records
     * are still kept, for the preconditioner's diagonal blocks, so this saves
     * no memory; it trades their reads for the evaluation's arithmetic. */
    int32_t recompute_jacobians;
} mvdr_config;

/* Per-view inputs: the rendered solver maps (Renderer::SolverMaps,
 * render/Renderer.h:381-388), the camera observation maps
 * (CameraObservation, base/CameraObservation.h:16-63) and the view's camera
 * parameters. Maps are dense row-major image_height x image_width arrays with
 * a row pitch of `pitch` elements (0 = image_width). */
typedef struct mvdr_view_inputs {
    const mvdr_float4* reference_vertex_map;   /* canonical vertex, this camera's frame */
    const mvdr_float4* reference_normal_map;   /* canonical normal, this camera's frame */
    const uint32_t* index_map;                 /* surfel index or MVDR_INVALID_INDEX   */
    const mvdr_float4* vertex_confidence_map;  /* observed depth vertex                */
    const mvdr_float4* normal_radius_map;      /* observed depth normal                */
    const float* filtered_foreground_mask;     /* may be NULL if foreground is off     */
    const float* foreground_mask_gradient;     /* float2 per pixel; may be NULL        */
    uint32_t pitch;
    mvdr_intrinsic intrinsic;                  /* ClipColorIntrinsic[v]                */
    mvdr_mat34 world2camera;                   /* world2Camera[v] (canonical2Live)     */
    mvdr_mat34 initial_camera_se3;             /* InitialCameraSE3[v]: camera v -> 0   */
    /* density term only (may be NULL otherwise): */
    const mvdr_float4* normalized_rgb_map;     /* SolverMaps::normalized_rgb_map       */
    const float* density_map;                  /* CameraObservation::grayScaleMap      */
    const float* density_gradient_map;         /* grayScaleGradientMap, float2 per pixel */
} mvdr_view_inputs;

/* Correspondence terms after selection and compaction, as held by
 * Point2PointICPTerm2Jacobian (core/NonRigidSolver/solver_types.h:150-160):
 * target (observed, live frame 0), reference (canonical, frame 0), 4-NN. */
typedef struct mvdr_correspondences {
    uint32_t count;
    const mvdr_float4* target_vertex;
    const mvdr_float4* reference_vertex;
    const uint16_t* knn;           /* ushort4 per term */
    const mvdr_float4* knn_weight;
} mvdr_correspondences;

/* Raw sparse-feature pixel pairs per view, as CameraObservation carries them
 * (CameraObservation.h:53-56), for the solver to select and compact on the
 * device (SparseCorrespondenceHandler.cu:100-199, the nearest-distance form
 * that solver_constants.h:9 enables). A pair (x, y, z, w) names a pixel of
 * the rendered solver maps and a pixel of the observation. Per pair the
 * observed pixel is the first non-zero depth vertex of the 3x3 window at
 * (z, w) in row order, the centre preferred, dropped on an edge pixel; the
 * rendered pixel is the 3x3 window pixel at (x, y) with a surfel whose live
 * vertex is nearest the observed vertex; the pair is kept when the reference
 * vertex there is within 5 cm (squared distance 2.5e-3) of the observed
 * vertex. Kept pairs become the feature terms in candidate order: target =
 * camera2world (the inverse of world2camera) of the observed vertex moved to
 * frame 0, reference = the reference vertex moved to frame 0, skinning of
 * the rendered pixel's surfel. The count of kept pairs stays on the device.
 * When any view has pairs, `feature` must be empty. */
typedef struct mvdr_feature_pairs {
    uint32_t count[MVDR_MAX_VIEWS];                     /* candidate pairs per view */
    const uint16_t* pixel_pairs[MVDR_MAX_VIEWS];        /* ushort4 per pair          */
    const mvdr_float4* live_vertex_map[MVDR_MAX_VIEWS]; /* SolverMaps::warp_vertex_map, the view's pitch */
    const uint8_t* edge_mask[MVDR_MAX_VIEWS];           /* 1 = edge; NULL: no edges  */
} mvdr_feature_pairs;

typedef struct mvdr_inputs {
    uint32_t num_views;
    uint32_t num_nodes;
    uint32_t num_surfels;
    uint32_t num_graph_edges;      /* entries of node_graph (8 * num_nodes)  */
    mvdr_view_inputs views[MVDR_MAX_VIEWS];
    /* SurfelGeometry::NonRigidSolverInput (SurfelGeometry.h:179-182) */
    const uint16_t* surfel_knn;            /* ushort4 per surfel */
    const mvdr_float4* surfel_knn_weight;
    /* WarpField::NonRigidSolverInput (WarpField.h:157-161) */
    const mvdr_dual_quaternion* node_se3;
    const mvdr_float4* canonical_node_coords;
    const uint16_t* node_graph;            /* ushort2 (i, j) per edge */
    mvdr_correspondences feature;          /* SparseCorrespondenceHandler output */
    mvdr_correspondences cross_view;       /* CrossViewCorrespondenceHandler output */
    mvdr_feature_pairs feature_pairs;      /* raw pairs, selected on the device (optional) */
} mvdr_inputs;

/* Sizes produced by the index build (host-readable after a stream sync). */
typedef struct mvdr_counts {
    uint32_t dense_terms;       /* T_d: valid index-map pixels, all views   */
    uint32_t smooth_terms;      /* T_s                                      */
    uint32_t foreground_terms;  /* T_f                                      */
    uint32_t feature_terms;     /* T_p                                      */
    uint32_t cross_terms;       /* T_c                                      */
    uint32_t node2term_entries; /* K1                                       */
    uint32_t nodepair_entries;  /* K2 (valid entries)                       */
    uint32_t half_pairs;        /* P                                        */
    uint32_t num_bins;          /* bins of 32 scalar rows                   */
    uint32_t binblock_nnz;      /* scalar slots of the bin-block CSR         */
    uint32_t error_flags;       /* device-side capacity/timeout flags        */
    uint32_t reserved;
} mvdr_counts;

typedef struct mvdr_solver mvdr_solver;
typedef struct mvdr_batch mvdr_batch;

/* ---- life cycle ------------------------------------------------------- */

/* Fills *cfg with defaults for the given capacities. */
MVDR_API void mvdr_config_default(mvdr_config* cfg, uint32_t max_nodes, uint32_t max_views,
                         uint32_t image_width, uint32_t image_height);

/* NonRigidSolver::NonRigidSolver + AllocateBuffer (NonRigidSolver.h:103,117). */
MVDR_API int mvdr_create(const mvdr_config* cfg, mvdr_solver** out);
/* ReleaseBuffer + destructor (NonRigidSolver.h:108,123). */
MVDR_API int mvdr_destroy(mvdr_solver* solver);

/* SetSolverInput (NonRigidSolver.cpp:77-97): binds the caller's device arrays
 * and resets the iteration state to inputs->node_se3
 * (SolverIterationData::SetWarpFieldInitialValue, SolverIterationData.cpp:37-50). */
MVDR_API int mvdr_set_inputs(mvdr_solver* solver, const mvdr_inputs* inputs, void* stream);

/* As mvdr_set_inputs, but every array pointer is a HOST pointer; the data is
 * copied into solver-owned device buffers on `stream` (pinned host memory
 * makes the copies asynchronous). The first call on an instance, or a call
 * with larger inputs than before, allocates those device buffers. */
MVDR_API int mvdr_set_inputs_host(mvdr_solver* solver, const mvdr_inputs* inputs, void* stream);

/* The per-view maps as the reference hands them over: texture objects
 * (cudaTextureObject_t, passed as uint64_t) of Renderer::SolverMaps
 * (render/Renderer.h:381-388) and CameraObservation
 * (base/CameraObservation.h:16-63), which the reference samples with
 * tex2D at integer pixel coordinates (DenseDepthJacobianResidual.cu:40-41,
 * 68-69). 0 marks a map that is not used (the foreground maps when the
 * foreground term is off, the density maps when the density term is off). */
typedef struct mvdr_view_textures {
    uint64_t reference_vertex_map;      /* SolverMaps::reference_vertex_map, float4  */
    uint64_t reference_normal_map;      /* SolverMaps::reference_normal_map, float4  */
    uint64_t index_map;                 /* SolverMaps::index_map, unsigned int       */
    uint64_t normalized_rgb_map;        /* SolverMaps::normalized_rgb_map, float4    */
    uint64_t vertex_confidence_map;     /* CameraObservation::vertexConfidenceMap    */
    uint64_t normal_radius_map;         /* CameraObservation::normalRadiusMap        */
    uint64_t filtered_foreground_mask;  /* filteredForegroundMask, float             */
    uint64_t foreground_mask_gradient;  /* foregroundMaskGradientMap, float2         */
    uint64_t density_map;               /* grayScaleMap, float                       */
    uint64_t density_gradient_map;      /* grayScaleGradientMap, float2              */
} mvdr_view_textures;

/* SetSolverInput with the maps as texture objects (NonRigidSolver.h:133-140
 * takes Renderer::SolverMaps and CameraObservation, whose maps are texture
 * objects). textures[v] gives view v's maps; the map pointers and pitch of
 * inputs->views[v] are ignored, every other field of *inputs is used as by
 * mvdr_set_inputs (device pointers). Each map's resource (a cudaArray, as
 * the reference's GL interop and texture helpers create, or pitched / linear
 * device memory) is copied on `stream` into solver-owned buffers of
 * image_width x image_height elements; a map of another size or channel
 * format is rejected with MVDR_EINVAL, a mipmapped array too. The first call
 * allocates those buffers. The solve then reads the copies, so the textures'
 * memory may change after the copy has run on the stream. */
MVDR_API int mvdr_set_inputs_textures(mvdr_solver* solver, const mvdr_inputs* inputs,
                                      const mvdr_view_textures* textures, void* stream);

/* The solver's warp field in device memory (num_nodes dual quaternions): the
 * counterpart of the reference's SolvedNodeSE3() device view
 * (NonRigidSolver.h:214). The pointer stays valid until the solver (or its
 * batch) is destroyed; its contents are those of the last solve enqueued, so
 * read it on that stream (or after synchronising it). Device-side errors are
 * not checked here: read error_flags with mvdr_get_counts. */
MVDR_API int mvdr_node_se3_device(mvdr_solver* solver, const mvdr_dual_quaternion** device_ptr);

/* ---- solver maps (the renderer's solver-map pass, on CUDA) ---------------
 * The reference renders its solver maps with OpenGL: every surfel is a point
 * (render/shaders/SolverMap.vert, SolverMapSized.vert, SolverMapIndexMap.vert,
 * SolverMap.frag; drawn by RendererDraw.cpp:384-480), depth-tested with
 * GL_LESS against a float depth buffer cleared to 1, into float4 vertex,
 * normal and rgb maps and an unsigned index map. mvdr_render_solver_maps
 * produces the same maps with CUDA kernels on the caller's buffers. */
typedef struct mvdr_surfel_geometry {
    uint32_t num_surfels;
    const mvdr_float4* reference_vertex_confid;  /* canonical vertex (frame 0), confidence */
    const mvdr_float4* reference_normal_radius;  /* canonical normal, radius (mm)          */
    const mvdr_float4* live_vertex_confid;       /* warped (live) vertex                   */
    const mvdr_float4* live_normal_radius;       /* warped normal                          */
    const mvdr_float4* color_time;               /* x: packed 0xRRGGBB as float bits,
                                                    y: written to the rgb map's w,
                                                    z: time last observed               */
} mvdr_surfel_geometry;

typedef struct mvdr_solver_map_params {
    uint32_t width, height;        /* map size in pixels                                   */
    float max_depth;               /* widthHeightMaxMinDepth.z: points beyond max_depth + 0.05 m are dropped */
    float current_time;            /* the frame's time                                     */
    float confidence_threshold;    /* kStableSurfelConfidenceThreshold                      */
    float time_threshold;          /* kRenderingRecentTimeThreshold; a negative value drops
                                      every surfel below the confidence threshold
                                      (DrawSolverMapsConfidentObservation)                 */
} mvdr_solver_map_params;

typedef struct mvdr_solver_map_view {
    mvdr_mat34 world2camera;       /* the view's world2camera                              */
    mvdr_mat34 initial_camera_se3; /* camera v -> frame 0 (identity for view 0); the maps
                                      hold its inverse applied to the surfel attributes   */
    mvdr_intrinsic intrinsic;      /* the renderer's intrinsic of this view                */
    int32_t sized_points;          /* 1: each point covers the projected surfel disc
                                      (SolverMapSized.vert, view 0 with USE_DENSE_SOLVER_MAPS);
                                      0: one-pixel points (SolverMapIndexMap.vert)         */
    uint32_t pitch;                /* row pitch of the outputs in elements (0 = width)     */
    /* outputs, device memory, height x pitch elements each (any may be NULL
       except index_map and depth_index) */
    mvdr_float4* reference_vertex_map;
    mvdr_float4* reference_normal_map;
    mvdr_float4* live_vertex_map;
    mvdr_float4* live_normal_map;
    uint32_t* index_map;           /* surfel id, MVDR_INVALID_INDEX where nothing lands    */
    mvdr_float4* normalized_rgb_map;
    uint64_t* depth_index;         /* caller-owned scratch: the depth test's (depth, id)
                                      words, height x pitch                               */
} mvdr_solver_map_view;

/* Render the solver maps of num_views views (<= MVDR_MAX_VIEWS) on `stream`.
 * No allocation and no host synchronisation. Equal depths resolve to the
 * smaller surfel id, as the first point drawn wins GL_LESS. Points whose
 * centre falls outside the image are dropped, as GL clips points by their
 * centre. The rasteriser's sub-pixel snapping is not reproduced: a point
 * covers the pixels whose centres lie in the square of its size around its
 * projection. */
MVDR_API int mvdr_render_solver_maps(const mvdr_surfel_geometry* surfels, const mvdr_solver_map_params* params,
                                     const mvdr_solver_map_view* views, uint32_t num_views, void* stream);

/* ---- after the solve: moving the surfels and nodes, node errors, and the
 * correction of badly aligned nodes ----------------------------------------
 * The reference's SurfelNodeDeformer (core/Geometry/SurfelNodeDeformer.cu)
 * moves the canonical surfels and nodes with the solved warp field and back;
 * DenseDepthHandler (core/NonRigidSolver/DenseDepthAlignmentError.cu:97-370)
 * measures how well each node's surface matches the depth observation; and
 * NonRigidSolver::CorrectLargeErrorNode (NonRigidSolver.cu:93-227,377-425)
 * pulls nodes with a large error towards guiding correspondences. */

/* Surfels to move: forward (canonical -> live) or inverse (live -> canonical).
 * A surfel whose KNN names a node at or past the node count gets NaN outputs
 * (no out-of-range read). */
typedef struct mvdr_deform_surfels {
    uint32_t num_surfels;
    const uint16_t* knn;            /* ushort4 per surfel */
    const mvdr_float4* knn_weight;
    const mvdr_float4* in_vertex;   /* xyz + confidence (w kept) */
    const mvdr_float4* in_normal;   /* xyz + radius (w kept) */
    mvdr_float4* out_vertex;
    mvdr_float4* out_normal;
} mvdr_deform_surfels;

/* Nodes moved by the forward warp: live = blend(nodes' own KNN) applied to
 * the canonical coordinate, its w (which encodes the node's view) kept. */
typedef struct mvdr_deform_nodes {
    uint32_t num_nodes;
    const uint16_t* knn;            /* ushort4 per node: nodesKNN */
    const mvdr_float4* knn_weight;
    const mvdr_float4* canonical_nodes;
    mvdr_float4* live_nodes;
} mvdr_deform_nodes;

/* SurfelNodeDeformer::ForwardWarpSurfelsAndNodes (SurfelNodeDeformer.cu:9-206):
 * out = se3(blend) * in for every surfel and (when `nodes` is not NULL) every
 * node. node_se3 holds num_node_se3 dual quaternions (device). */
MVDR_API int mvdr_forward_warp(const mvdr_dual_quaternion* node_se3, uint32_t num_node_se3,
                               const mvdr_deform_surfels* surfels, const mvdr_deform_nodes* nodes, void* stream);
/* SurfelNodeDeformer::InverseWarpSurfels (SurfelNodeDeformer.cu:63-119,
 * 229-318): out = se3(blend)^-1 * in, then, when correct_se3 (one mat34 per
 * surfel, device) is not NULL, out = correct_se3^-1 * out. */
MVDR_API int mvdr_inverse_warp(const mvdr_dual_quaternion* node_se3, uint32_t num_node_se3,
                               const mvdr_mat34* correct_se3, const mvdr_deform_surfels* surfels, void* stream);

/* Node alignment errors of the solver's bound inputs under its current warp
 * field (NonRigidSolver::ComputeAlignmentErrorOnNodes ->
 * DenseDepthHandler::ComputeNodewiseError). Per rendered pixel of every view
 * the error is the smallest L1 distance between the warped reference vertex
 * (camera frame) and the observed vertices of the 3x3 window at its
 * projection, at most 0.1 m; without a compatible observed vertex (normal dot
 * > 0.7) it is 0.03 x the filtered foreground mask when that is below 0.9,
 * else 0.1. Errors above 1e-6 are added with the pixel's skinning weights to
 * its four nodes. The sums are kept in 2^-32 fixed point, so they do not
 * depend on the order of the additions. Outputs (device, N = bound nodes):
 * the sums, united_error = (sum_err / (sum_w + 1e-4)) / 0.1 (1 for a node
 * with no error), and large_error_mark = united_error > threshold (or no
 * error); optional per-view maps: the per-pixel error
 * (ComputeAlignmentErrorMapDirect) and the node errors interpolated back to
 * the pixels (ComputeAlignmentErrorMapFromNode). Maps are width x height
 * floats, rows `width` apart. */
typedef struct mvdr_node_error {
    float* accumulated_error;   /* [N] */
    float* accumulated_weight;  /* [N] */
    float* united_error;        /* [N] */
    uint32_t* large_error_mark; /* [N] 1 = large */
    float threshold;            /* the reference passes 0.2 */
    float* alignment_error_map[MVDR_MAX_VIEWS];  /* optional */
    float* node_error_map[MVDR_MAX_VIEWS];       /* optional */
} mvdr_node_error;
MVDR_API int mvdr_compute_node_error(mvdr_solver* solver, const mvdr_node_error* out, void* stream);

/* Guides of one view for the correction: the correspondence SE3 map
 * (previous frame -> current frame, camera frame), its validity (1 = valid)
 * and the previous frame's vertex map, each width x height with rows `pitch`
 * elements apart (0 = width). */
typedef struct mvdr_correction_view {
    const mvdr_mat34* se3_map;
    const uint8_t* valid_map;
    const mvdr_float4* previous_vertex_map;
    uint32_t pitch;
} mvdr_correction_view;

/* NonRigidSolver::CorrectLargeErrorNode, correspondence form
 * (NonRigidSolver.cu:93-139,154-227,377-425). For every node whose united
 * error is above error_threshold, the node's live coordinate is projected into
 * the view its w names (i < w <= i + 1); within the 5x5 window there, the
 * valid guide whose previous vertex is nearest (squared distance below 1e-4)
 * and that moves the node by less than 2 node radii gives the node's
 * correction, brought to frame 0 and scaled by the error
 * (DualQuaternion::operator*(float)). Other nodes get the identity. The
 * corrections are then blended at every surfel and node: live surfels and
 * live nodes are moved, and each node's SE3 becomes blend * SE3. The
 * corrected warp field is written to node_se3 and becomes the solver's
 * current warp field. Cameras come from the solver's bound inputs. */
typedef struct mvdr_correction {
    uint32_t width, height;                         /* of the guide maps */
    mvdr_correction_view views[MVDR_MAX_VIEWS];     /* the bound views' guides */
    const float* united_error;                      /* [N], from mvdr_compute_node_error */
    float error_threshold;                          /* the reference uses 0.2 */
    mvdr_dual_quaternion* node_se3;                 /* [N] in/out; NULL: the solver's current field */
    mvdr_float4* live_nodes;                        /* [N] in/out */
    const uint16_t* node_knn;                       /* ushort4 [N] */
    const mvdr_float4* node_knn_weight;             /* [N] */
    uint32_t num_surfels;
    mvdr_float4* live_vertex;                       /* [S] in/out */
    mvdr_float4* live_normal;                       /* [S] in/out */
    const uint16_t* surfel_knn;                     /* ushort4 [S] */
    const mvdr_float4* surfel_knn_weight;           /* [S] */
    mvdr_dual_quaternion* correction;               /* [N] out: each node's correction */
} mvdr_correction;
MVDR_API int mvdr_correct_large_error_nodes(mvdr_solver* solver, const mvdr_correction* c, void* stream);

/* ---- input bundles (replay of one solve's inputs) -----------------------
 * mvdr_save_input_bundle writes the configuration and every input array
 * bound to the solver (device or owned copies) to a file; it synchronises
 * `stream`. mvdr_load_input_bundle reads such a file into host memory: the
 * bundle's config and inputs (HOST pointers into the bundle) can be given to
 * mvdr_create and mvdr_set_inputs_host to replay the solve, e.g. to reproduce
 * a parity failure on real inputs. The reference has no counterpart. */
typedef struct mvdr_input_bundle mvdr_input_bundle;
MVDR_API int mvdr_save_input_bundle(mvdr_solver* solver, const char* path, void* stream);
MVDR_API int mvdr_load_input_bundle(const char* path, mvdr_input_bundle** out);
MVDR_API const mvdr_config* mvdr_input_bundle_config(const mvdr_input_bundle* bundle);
MVDR_API const mvdr_inputs* mvdr_input_bundle_inputs(const mvdr_input_bundle* bundle);
MVDR_API void mvdr_free_input_bundle(mvdr_input_bundle* bundle);

/* buildSolverIndexStreamed (NonRigidSolver.h:257, body not in the reference):
 * pixel selection and compaction (ImageTermKNNFetcher.cu:19-137,
 * DensityForegroundMapHandler.cu:34-146), node->term index
 * (Node2TermsIndex.cu:8-187), node-pair->term index and bin-block CSR
 * structure (NodePair2TermsIndex.cu:11-296, NodePairRowColumnIndex.cu:19-308).
 * No host synchronisation. */
MVDR_API int mvdr_build_index(mvdr_solver* solver, void* stream);

/* One Gauss-Newton iteration (solverIteration{Global,Local}IterationStreamed,
 * NonRigidSolver.h:258-259): term evaluation, preconditioner and RHS, JtJ
 * materialisation (MATERIALIZED mode), block PCG with `pcg_iterations`
 * iterations, warp-field update (SolverIterationData.cu:9-94). */
MVDR_API int mvdr_gn_iteration(mvdr_solver* solver, uint32_t pcg_iterations, void* stream);

/* SolveNonRigidAlignment (NonRigidSolver.h:254): build_index followed by
 * `gn_iterations` Gauss-Newton iterations. */
MVDR_API int mvdr_solve(mvdr_solver* solver, uint32_t gn_iterations, uint32_t pcg_iterations, void* stream);

/* SolvedNodeSE3 (NonRigidSolver.h:214): copies the current node SE(3) array
 * (num_nodes dual quaternions) to `dst`, which may be host or device memory. */
MVDR_API int mvdr_get_node_se3(mvdr_solver* solver, mvdr_dual_quaternion* dst, void* stream);
/* Enqueue a copy of the current warp field (num_nodes dual quaternions) into
 * dst (device or pinned host memory) on `stream` and return at once: the
 * counterpart of the reference's SolvedNodeSE3() device view, for callers
 * that overlap solves. Unlike mvdr_get_node_se3 it does not read the device
 * error record; read error_flags with mvdr_get_counts once the stream is
 * done. */
MVDR_API int mvdr_copy_node_se3_async(mvdr_solver* solver, mvdr_dual_quaternion* dst, void* stream);

/* Synchronises `stream` and returns the sizes of the current index. */
MVDR_API int mvdr_get_counts(mvdr_solver* solver, mvdr_counts* out, void* stream);

/* Energy sum (lambda * r)^2 of the terms evaluated by the last Gauss-Newton
 * iteration, accumulated in double (ResidualEvaluator.cu:71-226). */
MVDR_API int mvdr_get_energy(mvdr_solver* solver, double* energy, void* stream);

/* ---- intermediate products (for checks) --------------------------------
 * `which` selects an array, `dst` receives it (host or device memory),
 * `capacity_bytes` is the size of dst; *written_bytes returns the byte count.
 * The call synchronises `stream`. */
enum {
    MVDR_ARRAY_DENSE_PIXELS = 0,        /* ushort4 (x, y, view, 0) per dense term          */
    MVDR_ARRAY_DENSE_KNN = 1,           /* ushort4 per dense term                          */
    MVDR_ARRAY_DENSE_KNN_WEIGHT = 2,    /* float4 per dense term                           */
    MVDR_ARRAY_FOREGROUND_PIXELS = 3,   /* ushort4 per foreground term                     */
    MVDR_ARRAY_NODE2TERM_OFFSET = 4,    /* uint32 [N+1]                                    */
    MVDR_ARRAY_NODE2TERM_INDEX = 5,     /* uint32 [K1]                                     */
    MVDR_ARRAY_HALF_NODEPAIR_KEY = 6,   /* uint32 [P]: i*4096+j for i<j (4096 -> 2^ceil(log2 N) past 4096) */
    MVDR_ARRAY_NODEPAIR_TERM_INDEX = 7, /* uint32 [K2]                                     */
    MVDR_ARRAY_NODEPAIR_KEY = 8,        /* uint32 [2P]: symmetric keys, sorted             */
    MVDR_ARRAY_NODEPAIR_TERM_RANGE = 9, /* uint2  [2P]                                     */
    MVDR_ARRAY_BLKROW_OFFSET = 10,      /* uint32 [N+1]                                    */
    MVDR_ARRAY_BINBLOCK_ROWPTR = 11,    /* int32  [32*(nbins+1)]                           */
    MVDR_ARRAY_BINBLOCK_COLPTR = 12,    /* int32  [binblock_nnz/6]                         */
    MVDR_ARRAY_TERM_JACOBIAN = 13,      /* float [T_d+T_f][8]: twist gradient (6), residual, pad */
    MVDR_ARRAY_SMOOTH_TERMS = 14,       /* float [T_s][12]: Ti_xj (3), Tj_xj (3), validity, pad,
                                           residual Ti_xj - Tj_xj (3), pad                     */
    MVDR_ARRAY_WARPED_CORRESPONDENCE = 15, /* float [T_p+T_c][8]: warped reference vertex (3),
                                              1, residual warped - target (3), pad            */
    MVDR_ARRAY_DIAG_BLOCKS = 16,        /* float [N][36] JtJ diagonal blocks incl. damping  */
    MVDR_ARRAY_JTR = 17,                /* float [N][6]  b = -Jt r                          */
    MVDR_ARRAY_PRECONDITIONER = 18,     /* float [N][36] inverse of the diagonal blocks      */
    MVDR_ARRAY_OFFDIAG_BLOCKS = 19,     /* float [2P][36] in symmetric-key order, blk[6k+r] = A(r,k) */
    MVDR_ARRAY_BINBLOCK_DATA = 20,      /* float [binblock_nnz] bin-block CSR values        */
    MVDR_ARRAY_INCREMENT = 21,          /* float [6N] PCG solution of the last iteration     */
    MVDR_ARRAY_NODE_SE3 = 22,           /* dual quaternion [N] current warp field            */
    MVDR_ARRAY_DENSITY_JACOBIAN = 23,   /* float [T_d][8]: density twist gradient (6), residual,
                                           projected pixel (use_density only)                */
    MVDR_ARRAY_FEATURE_TERMS = 24,      /* float [T_p][8]: target vertex (4), reference vertex
                                           (4) of the feature terms (bound or selected)      */
    MVDR_ARRAY_PCG_RESIDUALS = 25       /* double [G][MVDR_PCG_HISTORY]: per Gauss-Newton
                                           iteration g < 64 of the last solve, delta_k of
                                           each PCG iteration k (delta_0 first); NaN after
                                           the last iteration run                            */
};
#define MVDR_PCG_HISTORY 257u /* delta_0 and up to 256 PCG iterations per Gauss-Newton iteration */
MVDR_API int mvdr_get_array(mvdr_solver* solver, int which, void* dst, size_t capacity_bytes,
                   size_t* written_bytes, void* stream);

/* y = JtJ x with the operator of the last Gauss-Newton iteration, in the
 * current mode (bin-block/BSR SpMV or matrix-free adjoint pair). x and y are
 * device arrays of 6*num_nodes floats. */
MVDR_API int mvdr_apply_jtj(mvdr_solver* solver, const float* x, float* y, void* stream);

/* ---- block SpMV without device allocation -------------------------------
 * No counterpart in the reference. Every other entry point works on a solver
 * handle whose workspaces mvdr_create allocates with cudaMalloc. This one is
 * for callers that cannot allocate device memory: a host application whose
 * GPU memory is owned by another allocator, or a real-time loop that forbids
 * cudaMalloc after start-up because it may synchronise the device.
 *
 * y = A x and *x_dot_y = x.y (summed in double) for a 6x6 block-sparse matrix
 * in block-CSR form: block row i holds stored blocks rowptr[i] ..
 * rowptr[i+1]-1, block s sits in block column colidx[s] with
 * blocks[36 s + 6 r + k] = A(r, k). x and y hold 6*num_block_rows floats;
 * every pointer is device memory on the current device. This is the operator
 * step of the PCG (the SpMV with its fused dot product) on a matrix the caller
 * owns; mvdr_apply_jtj computes the same product on a solver's own matrix.
 *
 * It calls no cudaMalloc, cudaFree or allocating library routine. Its scratch
 * (per-CTA partial sums, a completion ticket and an error flag, 64 KiB) is a
 * static device array that each GPU loading the library holds until the
 * process exits. The first call on a device looks up that array's address
 * (cudaGetSymbolAddress), so make the first call on each device before any
 * stream capture. Every later call on a stream that is not capturing looks the
 * address up again, so a cudaDeviceReset between calls leaves no stale
 * address behind. All calls share the array: calls whose work overlaps on the
 * GPU (on different streams, or from several host threads) race and give wrong
 * results; serialise them. num_block_rows above MVDR_NOALLOC_MAX_BLOCK_ROWS is
 * rejected with MVDR_ECAPACITY. A column index outside [0, num_block_rows)
 * skips its block and sets *x_dot_y to NaN. */
#define MVDR_NOALLOC_MAX_BLOCK_ROWS 262144u
MVDR_API int mvdr_bsr6_spmv_dot_noalloc(uint32_t num_block_rows, uint32_t num_blocks, const int32_t* rowptr,
                                        const int32_t* colidx, const float* blocks, const float* x, float* y,
                                        double* x_dot_y, void* stream);

/* ---- batched solves (many independent instances per launch) ------------- */

/* All instances share the capacities of *cfg; their actual sizes may differ. */
MVDR_API int mvdr_batch_create(const mvdr_config* cfg, uint32_t num_instances, mvdr_batch** out);
MVDR_API int mvdr_batch_destroy(mvdr_batch* batch);
MVDR_API int mvdr_batch_set_inputs(mvdr_batch* batch, uint32_t instance, const mvdr_inputs* inputs, void* stream);
MVDR_API int mvdr_batch_set_inputs_host(mvdr_batch* batch, uint32_t instance, const mvdr_inputs* inputs, void* stream);
/* Index build and `gn_iterations` Gauss-Newton iterations for every instance;
 * each stage is one launch over all instances. When use_graph is non-zero the
 * Gauss-Newton iterations are captured once as a CUDA graph and replayed. */
MVDR_API int mvdr_batch_solve(mvdr_batch* batch, uint32_t gn_iterations, uint32_t pcg_iterations,
                     int use_graph, void* stream);
/* Choose the PCG SpMV tile shape (block rows per CTA, threads per scalar row
 * / 6, and the form: 0 reads a lower block's rows and exchanges the column
 * sums through shared memory, 1 reads its columns) for this batch's
 * matrices. It builds the index and runs one
 * Gauss-Newton iteration on the bound inputs, which moves the warp fields
 * (bind the inputs again before solving), then times every candidate shape
 * on the assembled operator, keeps the fastest for later solves and drops the
 * captured graphs. Writes the chosen shape to *rows / *split / *form (each
 * may be NULL) and, when
 * times_ms is not NULL, the mean time of each candidate (up to `capacity`
 * entries, in candidate order). Synchronises `stream`. A matrix-free batch
 * keeps its shape. */
MVDR_API int mvdr_batch_autotune(mvdr_batch* batch, void* stream, double* times_ms, uint32_t capacity,
                                 uint32_t* rows, uint32_t* split, uint32_t* form);
/* Use SpMV tile shape `shape` (0 .. MVDR_NUM_SPMV_SHAPES - 1, the
 * autotuner's candidate order) for later solves of this batch, in place of
 * the autotuner's choice; drops the captured graphs. */
#define MVDR_NUM_SPMV_SHAPES 12u
MVDR_API int mvdr_batch_set_spmv_shape(mvdr_batch* batch, uint32_t shape);
/* on != 0: run each PCG solve of a materialised batch as one persistent
 * cooperative launch (the CTAs split among the instances, each instance's
 * CTAs stepping through its iterations with their own barriers) instead of
 * two or three launches per iteration; on == 0 restores the launches. Drops the
 * captured graphs. MVDR_EINVAL for a matrix-free batch or a batch with more
 * instances than the device holds co-resident CTAs of the kernel. */
MVDR_API int mvdr_batch_set_pcg_persistent(mvdr_batch* batch, int on);
/* Bounded waits of the persistent PCG. Each instance barrier gives up after
 * `limit_ns` nanoseconds (default 0.5 s, at most 10 s): the kernel's CTAs
 * return, the instance is flagged and the next checked read reports
 * MVDR_ETIMEOUT; the context stays usable. `extra_arrivals` > 0 makes every
 * barrier wait for that many arrivals beyond the instance's own CTAs, which
 * never come: it exists to exercise the timeout path and is 0 otherwise.
 * The reference has no bounded waits (its PCG is launched kernel by kernel,
 * BlockPCG.cuh:383-458). Drops the captured graphs. */
MVDR_API int mvdr_batch_set_wait_limit(mvdr_batch* batch, uint64_t limit_ns, uint32_t extra_arrivals);
MVDR_API int mvdr_batch_get_node_se3(mvdr_batch* batch, uint32_t instance, mvdr_dual_quaternion* dst, void* stream);
MVDR_API int mvdr_batch_copy_node_se3_async(mvdr_batch* batch, uint32_t instance, mvdr_dual_quaternion* dst,
                                            void* stream);
/* The single-instance view of one batch member (not owned; do not destroy). */
MVDR_API int mvdr_batch_instance(mvdr_batch* batch, uint32_t instance, mvdr_solver** out);

/* ---- diagnostics -------------------------------------------------------- */

/* Stages of one Gauss-Newton iteration, for timing one stage in isolation. */
enum {
    MVDR_STAGE_INDEX = 0,      /* the whole index build                          */
    MVDR_STAGE_TERMS = 1,      /* term evaluation                                */
    MVDR_STAGE_DIAG = 2,       /* diagonal blocks, Jt r and the preconditioner   */
    MVDR_STAGE_OFFDIAG = 3,    /* off-diagonal JtJ blocks (materialised mode)    */
    MVDR_STAGE_SPMV = 4,       /* one PCG SpMV (q = A d, d.q) on the current d   */
    MVDR_STAGE_PCG_UPDATE = 5, /* one PCG vector update (x, r, s, r.s)           */
    MVDR_STAGE_UPDATE = 6,     /* warp-field update                              */
    MVDR_STAGE_DIRECTION = 7,  /* one PCG direction update d = s + beta d_prev   */
    MVDR_STAGE_MATRIX_FREE = 8, /* one matrix-free product q = (JtJ + 1e-2 I) d
                                  and d.q, as J.d per term then Jt per node
                                  (matrix-free mode only; EINVAL otherwise)      */
    MVDR_STAGE_SCALE = 9       /* the block-Jacobi scaling of the off-diagonal
                                  blocks into float (mixed precision,
                                  materialised mode only; EINVAL otherwise)      */
};
/* Enqueue the kernels of one stage for every instance of the batch, with the
 * lambdas of Gauss-Newton iteration 0. The stage reads the state left by the
 * previous solve and overwrites that stage's outputs, so a later solve must
 * start again from mvdr_batch_set_inputs. No host synchronisation. */
MVDR_API int mvdr_batch_enqueue_stage(mvdr_batch* batch, int stage, void* stream);

/* Text of the last error recorded on this host thread. */
MVDR_API const char* mvdr_last_error_string(void);
/* Number of kernel launches this library has enqueued since load (a graph
 * launch counts once). */
MVDR_API uint64_t mvdr_kernel_launch_count(void);
/* sizeof() of the public struct `name` ("mvdr_config", "mvdr_inputs", ...) as
 * compiled into this library, so a binding can check its own layout. */
MVDR_API int mvdr_abi_layout(const char* name, size_t* size);

#ifdef __cplusplus
}
#endif
#endif /* MVDR_H_ */
