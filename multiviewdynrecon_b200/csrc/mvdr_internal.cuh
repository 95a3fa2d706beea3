// Internal declarations of the B200 non-rigid solver: device math, the
// per-instance descriptor that every kernel reads, and the kernel launchers.
//
// Batching: every kernel takes the descriptor array of all instances and uses
// blockIdx.y as the instance index. Grid sizes come from the capacities fixed
// at create time, and data-dependent sizes (dense-term count, node pairs, ...)
// are read from device memory, so a whole solve runs without a host
// synchronisation and can be captured once as a CUDA graph.
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/mvdr.h"

namespace mvdr {

constexpr int kWarp = 32;
constexpr uint32_t kInvalid = 0xFFFFFFFFu;
constexpr uint32_t kTransposedBlock = 0x80000000u;
// entry-count buckets of the half pairs (bucket 0 = longest; counts of
// kLenBuckets - 1 or more share bucket 0)
constexpr uint32_t kLenBuckets = 256;
__host__ __device__ constexpr uint32_t len_bucket_of(uint32_t len) {
    return kLenBuckets - 1 - (len < kLenBuckets - 1 ? len : kLenBuckets - 1);
}

// Element (r, k) of a stored 6x6 JtJ block. The layout keeps row r as three
// pairs (k = 0-1, 2-3, 4-5) at pair slots r, 6 + r, 12 + r, so six threads that
// each read one row with three pair loads cover the block in three
// contiguous, non-overlapping sweeps (a row read never shares a sector with
// another instruction's read).
__host__ __device__ constexpr uint32_t blk_idx(uint32_t r, uint32_t k) { return 12 * (k >> 1) + 2 * r + (k & 1); }

// The scaled operator's float blocks and the float copy of the PCG direction
// keep each row of six values in 32 bytes (two padding floats), so that a
// thread reads a block row or a node's direction in one 256-bit load.
constexpr uint32_t kScaledRow = 8;                  // floats per stored row
constexpr uint32_t kScaledBlock = 6 * kScaledRow;   // floats per stored block

constexpr uint32_t kChunkPixels = 2048;  // pixels per compaction CTA (256 threads x 8)

// error flag bits (DeviceCounts::error_flags)
enum : uint32_t {
    kErrDenseCapacity = 1u << 0,
    kErrForegroundCapacity = 1u << 1,
    kErrNode2TermCapacity = 1u << 2,
    kErrNodePairEntryCapacity = 1u << 3,
    kErrHalfPairCapacity = 1u << 4,
    kErrSegmentTooLong = 1u << 5,
    kErrRowTooLong = 1u << 6,
    kErrBinBlockCapacity = 1u << 7,
    kErrNonFinite = 1u << 8,
    kErrBadNodeIndex = 1u << 9,
    kErrWaitTimeout = 1u << 10,  // a bounded device-side wait gave up
};

// ------------------------------------------------------------- math ----

struct M34 {  // row-major rotation + translation
    float r[9];
    float t[3];
};

__host__ __device__ inline float3 mk3(float x, float y, float z) { return make_float3(x, y, z); }
__host__ __device__ inline float3 add3(float3 a, float3 b) { return mk3(a.x + b.x, a.y + b.y, a.z + b.z); }
__host__ __device__ inline float3 sub3(float3 a, float3 b) { return mk3(a.x - b.x, a.y - b.y, a.z - b.z); }
__host__ __device__ inline float3 mul3(float s, float3 a) { return mk3(s * a.x, s * a.y, s * a.z); }
__host__ __device__ inline float dot3(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__host__ __device__ inline float3 cross3(float3 a, float3 b) {
    return mk3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__host__ __device__ inline float3 rot3(const M34& m, float3 v) {
    return mk3(m.r[0] * v.x + m.r[1] * v.y + m.r[2] * v.z, m.r[3] * v.x + m.r[4] * v.y + m.r[5] * v.z,
               m.r[6] * v.x + m.r[7] * v.y + m.r[8] * v.z);
}
__host__ __device__ inline float3 rotT3(const M34& m, float3 v) {
    return mk3(m.r[0] * v.x + m.r[3] * v.y + m.r[6] * v.z, m.r[1] * v.x + m.r[4] * v.y + m.r[7] * v.z,
               m.r[2] * v.x + m.r[5] * v.y + m.r[8] * v.z);
}
__host__ __device__ inline float3 apply3(const M34& m, float3 v) {
    float3 a = rot3(m, v);
    return mk3(a.x + m.t[0], a.y + m.t[1], a.z + m.t[2]);
}

// dual quaternion: q0 = (x, y, z, w) real part, q1 dual part
struct DQ {
    float4 q0, q1;
};

// one 256-bit load: `field` is the solver's own 32-byte aligned warp field
__device__ inline DQ load_dq(const DQ* field, uint32_t i) {
    DQ d;
    asm volatile("ld.global.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                 : "=f"(d.q0.x), "=f"(d.q0.y), "=f"(d.q0.z), "=f"(d.q0.w), "=f"(d.q1.x), "=f"(d.q1.y), "=f"(d.q1.z),
                   "=f"(d.q1.w)
                 : "l"(field + i));
    return d;
}

// averageDualQuaternion (DualQuaternion.h:381-393): linear blend of 4 nodes
__device__ inline DQ blend_dq(const DQ* field, ushort4 knn, float4 w) {
    const DQ a = load_dq(field, knn.x), b = load_dq(field, knn.y), c = load_dq(field, knn.z),
             d = load_dq(field, knn.w);
    DQ o;
    o.q0.x = w.x * a.q0.x; o.q0.y = w.x * a.q0.y; o.q0.z = w.x * a.q0.z; o.q0.w = w.x * a.q0.w;
    o.q1.x = w.x * a.q1.x; o.q1.y = w.x * a.q1.y; o.q1.z = w.x * a.q1.z; o.q1.w = w.x * a.q1.w;
    o.q0.x += w.y * b.q0.x; o.q0.y += w.y * b.q0.y; o.q0.z += w.y * b.q0.z; o.q0.w += w.y * b.q0.w;
    o.q1.x += w.y * b.q1.x; o.q1.y += w.y * b.q1.y; o.q1.z += w.y * b.q1.z; o.q1.w += w.y * b.q1.w;
    o.q0.x += w.z * c.q0.x; o.q0.y += w.z * c.q0.y; o.q0.z += w.z * c.q0.z; o.q0.w += w.z * c.q0.w;
    o.q1.x += w.z * c.q1.x; o.q1.y += w.z * c.q1.y; o.q1.z += w.z * c.q1.z; o.q1.w += w.z * c.q1.w;
    o.q0.x += w.w * d.q0.x; o.q0.y += w.w * d.q0.y; o.q0.z += w.w * d.q0.z; o.q0.w += w.w * d.q0.w;
    o.q1.x += w.w * d.q1.x; o.q1.y += w.w * d.q1.y; o.q1.z += w.w * d.q1.z; o.q1.w += w.w * d.q1.w;
    return o;
}

__device__ inline float qdot(float4 a, float4 b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }

// q1 * conj(q0) * 2, vector part (translation of a unit dual quaternion)
__device__ inline float3 dq_translation(float4 q0, float4 q1) {
    const float4 a = make_float4(2.f * q1.x, 2.f * q1.y, 2.f * q1.z, 2.f * q1.w);
    const float4 b = make_float4(-q0.x, -q0.y, -q0.z, q0.w);
    // Hamilton product a*b, vector part
    return mk3(a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y, a.w * b.y - a.x * b.z + a.y * b.w + a.z * b.x,
               a.w * b.z + a.x * b.y - a.y * b.x + a.z * b.w);
}

__device__ inline void quat_rotation(float4 q, float* r) {
    r[0] = 1.f - 2.f * q.y * q.y - 2.f * q.z * q.z;
    r[1] = 2.f * q.x * q.y - 2.f * q.z * q.w;
    r[2] = 2.f * q.x * q.z + 2.f * q.y * q.w;
    r[3] = 2.f * q.x * q.y + 2.f * q.z * q.w;
    r[4] = 1.f - 2.f * q.x * q.x - 2.f * q.z * q.z;
    r[5] = 2.f * q.y * q.z - 2.f * q.x * q.w;
    r[6] = 2.f * q.x * q.z - 2.f * q.y * q.w;
    r[7] = 2.f * q.y * q.z + 2.f * q.x * q.w;
    r[8] = 1.f - 2.f * q.x * q.x - 2.f * q.y * q.y;
}

// DualQuaternion::normalize (DualQuaternion.h:281-287)
__device__ inline DQ dq_normalize(DQ d) {
    const float inv = rsqrtf(qdot(d.q0, d.q0));
    d.q0 = make_float4(inv * d.q0.x, inv * d.q0.y, inv * d.q0.z, inv * d.q0.w);
    d.q1 = make_float4(inv * d.q1.x, inv * d.q1.y, inv * d.q1.z, inv * d.q1.w);
    const float dd = qdot(d.q0, d.q1);
    d.q1 = make_float4(d.q1.x - dd * d.q0.x, d.q1.y - dd * d.q0.y, d.q1.z - dd * d.q0.z, d.q1.w - dd * d.q0.w);
    return d;
}

// DualQuaternion::se3_matrix (DualQuaternion.h:326-332)
__device__ inline M34 dq_se3(DQ d) {
    d = dq_normalize(d);
    M34 m;
    quat_rotation(d.q0, m.r);
    const float3 t = dq_translation(d.q0, d.q1);
    m.t[0] = t.x; m.t[1] = t.y; m.t[2] = t.z;
    return m;
}

// DualQuaternion::operator mat34 (DualQuaternion.h:309-319): normalised, then
// Quaternion::matrix() which normalises the rotation quaternion once more
__device__ inline M34 dq_to_mat34(DQ d) {
    d = dq_normalize(d);
    float4 q = d.q0;
    const float inv2 = rsqrtf(qdot(q, q));
    q = make_float4(inv2 * q.x, inv2 * q.y, inv2 * q.z, inv2 * q.w);
    M34 m;
    quat_rotation(q, m.r);
    const float3 t = dq_translation(d.q0, d.q1);
    m.t[0] = t.x; m.t[1] = t.y; m.t[2] = t.z;
    return m;
}

// ------------------------------------------------------- descriptor ----

struct ViewDesc {
    const float4* ref_v;
    const float4* ref_n;
    const uint32_t* index;
    const float4* obs_v;
    const float4* obs_n;
    const float* fg;
    const float2* fg_grad;
    const float4* rgb;        // density term: rendered normalised rgb (solver map)
    const float* dens;        // density term: observed grey level
    const float2* dens_grad;  // density term: its image gradient
    uint32_t pitch;
    float cx, cy, fx, fy;
    M34 w2c, init, init_inv;
    M34 c2w;  // the inverse of w2c (camera2World of the sparse feature selection)
    // the same transforms in double, for the mixed-precision residual chain
    double w2c_d[12], init_d[12], init_inv_d[12];  // row-major rotation, then translation
};

// device-resident sizes of one instance (written by the index build)
struct DeviceCounts {
    uint32_t dense_terms;
    uint32_t smooth_terms;
    uint32_t foreground_terms;
    uint32_t feature_terms;
    uint32_t cross_terms;
    uint32_t node2term_entries;
    uint32_t nodepair_entries;
    uint32_t half_pairs;
    uint32_t num_bins;
    uint32_t binblock_nnz;
    uint32_t error_flags;
    uint32_t reserved;
    uint32_t term_offset[5];  // prefix ends of Dense, Smooth, Foreground, Feature, Cross
    uint32_t dense_view_count[MVDR_MAX_VIEWS];
    uint32_t fg_view_count[MVDR_MAX_VIEWS];
    uint32_t pcg_stop;          // PCG iteration at which the convergence check stopped (0: running)
    uint32_t reserved2[3];
    double pcg_delta0;          // delta_0 of the current PCG solve
};

struct InstDesc {
    // host-known sizes (set_inputs)
    uint32_t num_views, N, S, E, Tp, Tc;
    uint32_t width, height;
    uint32_t enc;         // node-pair key multiplier (4096, or 2^k >= N)
    uint32_t compat;
    uint32_t use_fg;
    uint32_t use_density;
    float node_radius;
    ViewDesc views[MVDR_MAX_VIEWS];
    const ushort4* surfel_knn;
    const float4* surfel_w;
    const float4* nodes;
    const ushort2* graph;
    const float4* feat_target;
    const float4* feat_ref;
    const ushort4* feat_knn;
    const float4* feat_w;
    const float4* cross_target;
    const float4* cross_ref;
    const ushort4* cross_knn;
    const float4* cross_w;
    // device-side selection of the feature terms from raw pixel pairs
    // (mvdr_feature_pairs); feat_* then point at the fp_* outputs and Tp is
    // the capacity (the layout stride), the count being counts->feature_terms
    uint32_t feat_select;
    uint32_t fp_offset[MVDR_MAX_VIEWS + 1];  // candidate pairs before each view
    const ushort4* fp_pairs[MVDR_MAX_VIEWS];
    const float4* fp_live[MVDR_MAX_VIEWS];
    const uint8_t* fp_edge[MVDR_MAX_VIEWS];
    uint32_t* fp_keep;       // [max_tp] 1 = kept, then its exclusive prefix
    ushort4* fp_chosen;      // [max_tp] (rendered x, y, observed x, y)
    float4* fp_target;       // [max_tp]
    float4* fp_ref;
    ushort4* fp_knn;
    float4* fp_w;

    // ---- workspace (solver-owned) ----
    DeviceCounts* counts;
    DQ* se3;                // current warp field
    // compaction: per dense/foreground term
    uint32_t* chunk_count;  // [num chunk slots]
    uint32_t* pix_mask;     // predicate bit per pixel of the current compaction [views * chunks * 64]
    ushort4* dense_pix;     // (x, y, view, 0)
    ushort4* dense_knn;
    float4* dense_w;
    float4* dense_cv;       // canonical vertex in frame 0
    float4* dense_cv_lo;    // mixed precision: double transform minus dense_cv (x, y, z)
    float4* dense_cn;       // canonical normal in frame 0; w: rendered grey level (density term)
    ushort4* fg_pix;
    ushort4* fg_knn;
    float4* fg_w;
    float4* fg_cv;
    // node -> term
    uint32_t* n2t_count;    // [N+1]
    uint32_t* n2t_offset;   // [N+1]
    uint32_t* n2t_cursor;   // [N]
    uint32_t* n2t_index;    // [K1 cap]
    float* n2t_w;           // [K1 cap] skinning weight of the entry's node in its term (0 for smooth)
    // node pair -> term
    uint32_t* row_count;    // [N+1] entries (j, t) with j > i per row
    uint32_t* row_offset;   // [N+1]
    uint32_t* np_index;     // [K2 cap]
    float2* np_w;           // [K2 cap] skinning weights of the pair's (i, j) nodes in the entry's term
    uint32_t* upper_count;  // [N+1]
    uint32_t* half_offset;  // [N+1]
    uint32_t* tmp_key;      // [K2 cap] per-row unique pairs before compaction
    uint32_t* tmp_start;    // [K2 cap]
    uint32_t* half_key;     // [P cap]
    uint2* half_range;      // [P cap]
    uint32_t* pair_order;   // [P cap] half pairs grouped by entry count, longest first
    uint32_t* len_bucket;   // [2 * kLenBuckets] pairs per entry-count bucket, then scatter cursors
    uint32_t* lower_count;  // [N+1]
    uint32_t* lower_cursor; // [N]
    uint32_t* blkrow_offset;// [N+1]
    uint32_t* sym_key;      // [2P cap]
    uint2* sym_range;       // [2P cap]
    uint32_t* sym_half;     // [2P cap] half pair of each symmetric entry
    // bin-block CSR structure (reference layout, for checks and the bin-block SpMV)
    uint32_t* bin_scan;     // [nbins+1]
    int32_t* bb_rowptr;     // [32 (nbins+1)]
    int32_t* bb_colptr;     // [bb cap / 6]
    float* bb_data;         // [bb cap]
    // per-iteration term data
    float4* term_jr;        // 2 float4 per dense+fg term: J(6), r, pixel bits
    float4* density_jr;     // 2 float4 per dense term (density term): J(6), r, pixel bits
    float4* smooth;         // 3 float4 per smooth term: Ti_xj(3), Tj_xj(3), valid, 0, r(3), 0
    float4* warped;         // 2 float4 per feature+cross term: warped(3), 1, raw residual(3), 0
    // assembly
    float* diag;            // [36N] JtJ diagonal blocks incl. damping
    float* minv;            // [36N] preconditioner (inverse diagonal), float
    double* chol;           // [21N] Cholesky factors (mixed precision)
    float* jtr;                // [6N]
    double* jtr_d;          // mixed precision: Jt r in double
    // JtJ in half storage: per block row i its diagonal block at
    // half_offset[i] + i, then the upper blocks of its half pairs h at h + i + 1
    // (element order blk_idx). A lower block (i, j), j < i, is the transpose
    // of the stored block of pair (j, i).
    float* bsr;             // FP32: [(N + P cap) * 36]
    double* bsr_d;          // mixed precision: the same blocks in double
    // mixed precision, materialised: the operator of the PCG scaled by the
    // diagonal blocks' Cholesky factors, A^ = L^-1 A L^-T (identity diagonal
    // blocks, not stored): its upper blocks A^_ij = L_i^-1 A_ij L_j^-T in
    // float, row-major with rows of kScaledRow floats (element (r, k) at
    // 8 r + k), kScaledBlock floats per block at the half-storage block
    // positions of bsr_d
    float* bsr_s;
    float* df;              // [8N] the PCG direction of the scaled system in float, 8 floats per node
    // per entry of the full (symmetric) block-row layout, row i: the diagonal,
    // then its symmetric keys in order [N + 2P cap]
    // (half-storage block | kTransposedBlock when read transposed, block column)
    uint2* bsr_ent;
    // pcg vectors [6N each]
    // PCG vectors [6N] (d double-buffered by iteration parity): float for
    // FP32, double for mixed precision (PcgVec selects)
    float* x;
    float* r;
    float* s;
    float* q;
    float* d0;
    float* d1;
    double* x_d;
    double* r_d;
    double* s_d;
    double* q_d;
    double* d0_d;
    double* d1_d;
    float* jp;              // matrix-free scratch: J.p per scalar term
    double* partials;       // per-CTA partial sums: 4 regions of part_stride
    uint32_t part_stride;   // >= the CTAs per instance of any launch
    uint32_t* pcg_bar;      // persistent PCG: this instance's barrier counter (batch-owned)
    double* energy;         // [max GN iterations + 1]
    unsigned long long* node_err_acc;  // [2N] node alignment error and weight sums, 2^-32 fixed point
    double* pcg_hist;       // [kPcgHistRows][MVDR_PCG_HISTORY] delta_k per GN iteration
    float pcg_tol;          // convergence tolerance (0: fixed iteration count)
    uint32_t recompute_jr;  // matrix-free products re-derive the pixel terms' records

    // capacities
    uint32_t cap_dense, cap_fg, cap_k1, cap_k2, cap_pairs, cap_seg, cap_bb;
    uint32_t chunks_per_view;
};

struct LaunchCfg {
    uint32_t B;            // instances
    uint32_t max_nodes, max_views, width, height;
    uint32_t cap_dense, cap_fg, cap_terms, cap_k1, cap_k2, cap_pairs, cap_seg, cap_bb;
    uint32_t max_edges, max_tp, max_tc;
    uint32_t chunks_per_view;
    int precision, mode;
    int use_density;
    int sm_count;
    int spmv_shape;  // index into the SpMV tile shapes (chosen by the autotuner)
    // persistent PCG: one cooperative launch per PCG solve (materialised mode)
    int pcg_persistent;
    uint32_t pcg_grid;   // co-resident CTAs of pcg_persistent_kernel
    uint32_t* pcg_bars;  // B barrier counters, 32 words apart
    // bounded waits of the persistent PCG's instance barriers: the limit of
    // each wait, and arrivals each barrier waits for beyond the instance's
    // CTAs (non-zero only to exercise the timeout path)
    uint64_t wait_limit_ns;
    uint32_t wait_extra_arrivals;
    float pcg_tol;  // PCG convergence tolerance (0: fixed iteration count)
    int recompute_jr;  // matrix-free products re-derive the pixel terms' records
};

constexpr uint32_t kPcgHistRows = 64;  // GN iterations whose PCG residuals are kept

constexpr uint64_t kDefaultWaitLimitNs = 500ull * 1000 * 1000;  // a barrier step takes microseconds
constexpr uint64_t kMaxWaitLimitNs = 10ull * 1000 * 1000 * 1000;

// ----------------------------------------------------------- launchers --
// Each launcher enqueues kernels on `st` for all instances. They return
// cudaGetLastError() of the last launch.
void count_launch();

// co-resident CTAs of the persistent PCG kernel on this device (0 on error)
uint32_t persistent_pcg_grid(int mixed, int sm_count);

// raise the dynamic shared-memory limit of the segment-sort kernels
cudaError_t set_index_smem_limits(size_t seg_bytes);

// SpMV tile shapes the autotuner chooses from: block rows per CTA and threads
// per scalar row (each taking every `split`-th block of the row)
struct SpmvShape {
    uint32_t rows, split, form;
};
constexpr int kNumSpmvShapes = 12;
extern const SpmvShape kSpmvShapes[kNumSpmvShapes];
// one PCG SpMV (q = A d, d.q) with the shape lc.spmv_shape
cudaError_t launch_spmv(const LaunchCfg& lc, InstDesc* d, int parity, cudaStream_t st);

cudaError_t launch_build_index(const LaunchCfg& lc, InstDesc* d_inst, cudaStream_t st);
// term evaluation; also stores the energy partials that launch_energy sums
cudaError_t launch_eval_terms(const LaunchCfg& lc, InstDesc* d_inst, const mvdr_penalty& lam, cudaStream_t st);
cudaError_t launch_assemble(const LaunchCfg& lc, InstDesc* d_inst, const mvdr_penalty& lam, bool materialize,
                            cudaStream_t st);
// The materialised assembly with the off-diagonal blocks on `side` while the
// diagonal blocks run on `st` (forked after the work queued on `st`, joined
// back before the scaling, which needs both); inside a stream capture the
// two become parallel branches of the graph.
cudaError_t launch_assemble_forked(const LaunchCfg& lc, InstDesc* d_inst, const mvdr_penalty& lam, cudaStream_t st,
                                   cudaStream_t side, cudaEvent_t fork, cudaEvent_t join);
cudaError_t launch_energy(const LaunchCfg& lc, InstDesc* d_inst, uint32_t slot, cudaStream_t st);
cudaError_t launch_pcg(const LaunchCfg& lc, InstDesc* d_inst, const mvdr_penalty& lam, uint32_t iters, uint32_t gn,
                       cudaStream_t st);
cudaError_t launch_update(const LaunchCfg& lc, InstDesc* d_inst, cudaStream_t st);
cudaError_t launch_stage(const LaunchCfg& lc, InstDesc* d_inst, const mvdr_penalty& lam, int stage, cudaStream_t st);
cudaError_t launch_apply_jtj(const LaunchCfg& lc, InstDesc* d_inst, const mvdr_penalty& lam, const float* x,
                             float* y, cudaStream_t st);
cudaError_t launch_export_offdiag(const LaunchCfg& lc, InstDesc* d_inst, uint32_t inst, float* out,
                                  cudaStream_t st);
cudaError_t launch_export_preconditioner(const LaunchCfg& lc, InstDesc* d_inst, uint32_t inst, float* out,
                                         cudaStream_t st);

}  // namespace mvdr
