// Host side of the solver: the NonRigidSolver-shaped batch object, its
// workspace arena, the Gauss-Newton orchestration (buildSolverIndexStreamed /
// solverIteration*Streamed, whose bodies are missing from the reference), the
// CUDA-graph capture of whole solves, and the extern "C" layer of mvdr.h.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "batch.cuh"
#include "kernels_common.cuh"

namespace mvdr {

static std::atomic<uint64_t> g_launches{0};
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

static thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

// the same error record for entry points defined in other files
int record_failure(int code, const std::string& msg) { return fail(code, msg); }

#define CU(call)                                                                                  \
    do {                                                                                          \
        cudaError_t e__ = (call);                                                                 \
        if (e__ != cudaSuccess)                                                                   \
            return fail(MVDR_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e__));        \
    } while (0)

// bin-block CSR values for the diagnostic export (diagnostic path only)
__global__ void export_binblock_fill_kernel(const InstDesc* insts, uint32_t inst, float* out) {
    // assembleBinBlockCSRKernel (JtJMaterializerBinBlockCSR.cu:8-37)
    const InstDesc& I = insts[inst];
    const uint32_t rows = 6 * I.N;
    for (uint32_t row = blockIdx.x * blockDim.x + threadIdx.x; row < rows; row += gridDim.x * blockDim.x) {
        uint32_t off = (uint32_t)I.bb_rowptr[row];
        const uint32_t br = row / 6, in = row % 6;
        for (int k = 0; k < 6; ++k, off += 32) out[off] = I.diag[36 * (size_t)br + in + 6 * k];
        for (uint32_t s = I.blkrow_offset[br]; s < I.blkrow_offset[br + 1]; ++s)
            for (int k = 0; k < 6; ++k, off += 32) out[off] = stored_block_element(I, s + br + 1, in, k);
    }
}

struct Arena {
    char* base = nullptr;
    size_t off = 0, size = 0;
    template <class T> T* take(size_t n) {
        const size_t bytes = ((n * sizeof(T)) + 255) & ~(size_t)255;
        T* p = reinterpret_cast<T*>(base ? base + off : nullptr);
        off += bytes;
        return p;
    }
};

Batch::~Batch() {
    for (auto& kv : graphs) cudaGraphExecDestroy(kv.second);
    for (auto& o : owned)
        if (o.mem) cudaFree(o.mem);
    for (auto& o : staged)
        if (o.mem) cudaFree(o.mem);
    if (d_inst) cudaFree(d_inst);
    if (d_bars) cudaFree(d_bars);
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (ev_join) cudaEventDestroy(ev_join);
    if (side) cudaStreamDestroy(side);
    if (arena) cudaFree(arena);
    for (auto* v : views) delete v;
}

static mvdr_penalty penalty_for(const mvdr_config& c, uint32_t iter) {
    mvdr_penalty p{};
    if (!c.use_elastic_penalty) {
        p = c.penalty;
        if (!c.use_density) p.density = 0.0f;
        return p;
    }
    if ((int64_t)iter < (int64_t)c.num_global_iterations) {  // PenaltyConstants.cpp:25-37
        p.smooth = 5.0f;
        p.density = 0.0f;
        p.foreground = c.use_foreground ? 2e-3f : 0.0f;
        p.feature = 1.0f;
        p.cross_view = c.use_cross_view ? 1.0f : 0.0f;
    } else {  // PenaltyConstants.cpp:39-51
        p.smooth = 5.0f;
        p.density = c.use_density ? 1e-2f : 0.0f;
        p.foreground = 0.0f;
        p.feature = 0.0f;
        p.cross_view = c.use_cross_view ? 1.0f : 0.0f;
    }
    return p;
}

static size_t layout_instance(Arena& a, InstDesc& I, const LaunchCfg& lc, uint32_t cap_edges, uint32_t max_tp,
                              uint32_t max_tc, uint32_t partial_slots) {
    const size_t N = lc.max_nodes;
    I.counts = a.take<DeviceCounts>(1);
    I.se3 = a.take<DQ>(N);
    I.chunk_count = a.take<uint32_t>((size_t)lc.chunks_per_view * lc.max_views + 1);
    I.pix_mask = a.take<uint32_t>((size_t)lc.chunks_per_view * lc.max_views * (kChunkPixels / 32));
    I.dense_pix = a.take<ushort4>(lc.cap_dense);
    I.dense_knn = a.take<ushort4>(lc.cap_dense);
    I.dense_w = a.take<float4>(lc.cap_dense);
    I.dense_cv = a.take<float4>(lc.cap_dense);
    I.dense_cv_lo = a.take<float4>(lc.cap_dense);
    I.dense_cn = a.take<float4>(lc.cap_dense);
    I.fg_pix = a.take<ushort4>(lc.cap_fg);
    I.fg_knn = a.take<ushort4>(lc.cap_fg);
    I.fg_w = a.take<float4>(lc.cap_fg);
    I.fg_cv = a.take<float4>(lc.cap_fg);
    I.n2t_count = a.take<uint32_t>(N + 1);
    I.n2t_offset = a.take<uint32_t>(N + 1);
    I.n2t_cursor = a.take<uint32_t>(N + 1);
    I.n2t_index = a.take<uint32_t>(lc.cap_k1);
    I.n2t_w = a.take<float>(lc.cap_k1);
    I.row_count = a.take<uint32_t>(N + 1);
    I.row_offset = a.take<uint32_t>(N + 1);
    I.np_index = a.take<uint32_t>(lc.cap_k2);
    I.np_w = a.take<float2>(lc.cap_k2);
    I.upper_count = a.take<uint32_t>(N + 1);
    I.half_offset = a.take<uint32_t>(N + 1);
    I.tmp_key = a.take<uint32_t>(lc.cap_k2);
    I.tmp_start = a.take<uint32_t>(lc.cap_k2);
    I.half_key = a.take<uint32_t>(lc.cap_pairs);
    I.half_range = a.take<uint2>(lc.cap_pairs);
    I.pair_order = a.take<uint32_t>(lc.cap_pairs);
    I.len_bucket = a.take<uint32_t>(2 * kLenBuckets);
    I.lower_count = a.take<uint32_t>(N + 1);
    I.lower_cursor = a.take<uint32_t>(N + 1);
    I.blkrow_offset = a.take<uint32_t>(N + 1);
    I.sym_key = a.take<uint32_t>(2 * (size_t)lc.cap_pairs);
    I.sym_range = a.take<uint2>(2 * (size_t)lc.cap_pairs);
    I.sym_half = a.take<uint32_t>(2 * (size_t)lc.cap_pairs);
    const size_t nbins = (6 * N + 31) / 32;
    I.bin_scan = a.take<uint32_t>(nbins + 2);
    I.bb_rowptr = a.take<int32_t>(32 * (nbins + 1));
    I.bb_colptr = a.take<int32_t>(lc.cap_bb / 6 + 1);
    I.bb_data = nullptr;
    I.term_jr = a.take<float4>(2 * ((size_t)lc.cap_dense + lc.cap_fg));
    I.density_jr = lc.use_density ? a.take<float4>(2 * (size_t)lc.cap_dense) : nullptr;
    I.smooth = a.take<float4>(3 * (size_t)cap_edges);
    I.warped = a.take<float4>(2 * ((size_t)max_tp + max_tc + 1));
    I.diag = a.take<float>(36 * N);
    I.minv = a.take<float>(36 * N);
    I.chol = a.take<double>(21 * N);
    I.jtr = a.take<float>(6 * N);  // also the float export in mixed precision
    I.jtr_d = lc.precision == MVDR_PRECISION_MIXED ? a.take<double>(6 * N) : nullptr;
    const bool mixed = lc.precision == MVDR_PRECISION_MIXED;
    I.bsr = mixed ? nullptr : a.take<float>(36 * (N + (size_t)lc.cap_pairs));
    I.bsr_d = mixed ? a.take<double>(36 * (N + (size_t)lc.cap_pairs)) : nullptr;
    I.bsr_ent = a.take<uint2>(N + 2 * (size_t)lc.cap_pairs);
    const bool scaled = mixed && lc.mode == MVDR_MODE_MATERIALIZED;
    I.bsr_s = scaled ? a.take<float>(kScaledBlock * (N + (size_t)lc.cap_pairs)) : nullptr;
    I.df = scaled ? a.take<float>(kScaledRow * N) : nullptr;
    if (mixed) {
        I.x_d = a.take<double>(6 * N);
        I.r_d = a.take<double>(6 * N);
        I.s_d = a.take<double>(6 * N);
        I.q_d = a.take<double>(6 * N);
        I.d0_d = a.take<double>(6 * N);
        I.d1_d = a.take<double>(6 * N);
    } else {
        I.x = a.take<float>(6 * N);
        I.r = a.take<float>(6 * N);
        I.s = a.take<float>(6 * N);
        I.q = a.take<float>(6 * N);
        I.d0 = a.take<float>(6 * N);
        I.d1 = a.take<float>(6 * N);
    }
    // J.p per scalar term of the matrix-free operator (double in mixed precision)
    I.jp = lc.mode == MVDR_MODE_MATRIX_FREE ? a.take<float>(6 * (size_t)lc.cap_terms) : nullptr;
    // region 0: energy; 1, 2: PCG delta by iteration parity; 3: d.q; 4: the
    // density term's energy
    I.partials = a.take<double>(7 * (size_t)partial_slots);
    I.part_stride = partial_slots;
    I.energy = a.take<double>(64);
    I.node_err_acc = a.take<unsigned long long>(2 * N);
    I.pcg_hist = a.take<double>((size_t)kPcgHistRows * MVDR_PCG_HISTORY);
    I.pcg_tol = lc.pcg_tol;
    I.recompute_jr = (uint32_t)lc.recompute_jr;
    if (max_tp) {  // device-side feature selection
        I.fp_keep = a.take<uint32_t>(max_tp);
        I.fp_chosen = a.take<ushort4>(max_tp);
        I.fp_target = a.take<float4>(max_tp);
        I.fp_ref = a.take<float4>(max_tp);
        I.fp_knn = a.take<ushort4>(max_tp);
        I.fp_w = a.take<float4>(max_tp);
    }
    I.cap_dense = lc.cap_dense;
    I.cap_fg = lc.cap_fg;
    I.cap_k1 = lc.cap_k1;
    I.cap_k2 = lc.cap_k2;
    I.cap_pairs = lc.cap_pairs;
    I.cap_seg = lc.cap_seg;
    I.cap_bb = lc.cap_bb;
    I.chunks_per_view = lc.chunks_per_view;
    return a.off;
}

static int create_batch(const mvdr_config* cfg, uint32_t B, Batch** out) {
    if (!cfg || !out || B == 0) return fail(MVDR_EINVAL, "null argument or zero instances");
    if (cfg->abi_version != MVDR_ABI_VERSION) return fail(MVDR_EINVAL, "abi_version mismatch");
    if (cfg->max_nodes == 0 || cfg->max_nodes > 65535) return fail(MVDR_EINVAL, "max_nodes must be in [1, 65535]");
    if (cfg->max_views == 0 || cfg->max_views > MVDR_MAX_VIEWS) return fail(MVDR_EINVAL, "max_views out of range");
    if (cfg->image_width == 0 || cfg->image_height == 0 || cfg->image_width > 65535 || cfg->image_height > 65535)
        return fail(MVDR_EINVAL, "image size out of range");
    if (cfg->precision != MVDR_PRECISION_FP32 && cfg->precision != MVDR_PRECISION_MIXED)
        return fail(MVDR_EINVAL, "unknown precision");
    if (cfg->mode != MVDR_MODE_MATERIALIZED && cfg->mode != MVDR_MODE_MATRIX_FREE)
        return fail(MVDR_EINVAL, "unknown mode");
    if (!(cfg->pcg_tolerance >= 0.0f && cfg->pcg_tolerance < 1.0f))
        return fail(MVDR_EINVAL, "pcg_tolerance must be in [0, 1)");
    if (cfg->recompute_jacobians && cfg->mode != MVDR_MODE_MATRIX_FREE)
        return fail(MVDR_EINVAL, "recompute_jacobians needs the matrix-free mode");
    int dev = 0;
    CU(cudaGetDevice(&dev));
    cudaDeviceProp prop;
    CU(cudaGetDeviceProperties(&prop, dev));

    Batch* b = new Batch();
    b->cfg = *cfg;
    b->B = B;
    LaunchCfg& lc = b->lc;
    lc.B = B;
    lc.max_nodes = cfg->max_nodes;
    lc.max_views = cfg->max_views;
    lc.width = cfg->image_width;
    lc.height = cfg->image_height;
    const uint64_t pix = (uint64_t)cfg->max_views * cfg->image_width * cfg->image_height;
    lc.cap_dense = cfg->max_dense_terms ? cfg->max_dense_terms : (uint32_t)std::min<uint64_t>(pix, 0x7fffffffu);
    lc.cap_fg = cfg->use_foreground ? (cfg->max_foreground_terms ? cfg->max_foreground_terms : lc.cap_dense) : 0;
    lc.max_tp = cfg->use_feature ? cfg->max_feature_terms : 0;
    lc.max_tc = cfg->use_cross_view ? cfg->max_cross_terms : 0;
    b->cap_edges = 8 * cfg->max_nodes;
    lc.max_edges = b->cap_edges;
    const uint64_t four = (uint64_t)lc.cap_dense + lc.cap_fg + lc.max_tp + lc.max_tc;
    const uint64_t k1 = 4 * four + 2 * (uint64_t)b->cap_edges;
    const uint64_t k2 = 6 * four + (uint64_t)b->cap_edges;
    if (k2 > 0x7fffffffull) {
        delete b;
        return fail(MVDR_ECAPACITY, "term capacities exceed 2^31 index entries");
    }
    lc.cap_terms = (uint32_t)(four + b->cap_edges);
    lc.cap_k1 = (uint32_t)k1;
    lc.cap_k2 = (uint32_t)k2;
    lc.cap_pairs = cfg->max_node_pairs ? cfg->max_node_pairs : 16 * cfg->max_nodes;
    // shared-memory sort capacities are powers of two: the bitonic sort pads
    // a segment up to the next power of two
    auto pow2 = [](uint32_t v) { uint32_t p = 1; while (p < v) p <<= 1; return p; };
    lc.cap_seg = std::min<uint32_t>(pow2(cfg->max_terms_per_node ? cfg->max_terms_per_node : 4096), 16384);
    lc.cap_bb = 36 * (cfg->max_nodes + 2 * lc.cap_pairs);
    lc.chunks_per_view = (cfg->image_width * cfg->image_height + kChunkPixels - 1) / kChunkPixels;
    lc.precision = cfg->precision;
    lc.mode = cfg->mode;
    lc.use_density = cfg->use_density ? 1 : 0;
    lc.pcg_tol = cfg->pcg_tolerance;
    lc.recompute_jr = cfg->recompute_jacobians ? 1 : 0;
    lc.sm_count = prop.multiProcessorCount;

    const size_t smem_seg = (size_t)lc.cap_seg * 4;
    if (smem_seg > (size_t)prop.sharedMemPerBlockOptin) {
        delete b;
        return fail(MVDR_EINVAL, "max_terms_per_node too large for shared memory");
    }
    if (set_index_smem_limits(smem_seg) != cudaSuccess) {
        delete b;
        return fail(MVDR_ECUDA, "cudaFuncSetAttribute failed");
    }

    const uint32_t gmax = std::max<uint32_t>({(lc.max_nodes + 255) / 256, (lc.max_nodes + 31) / 32,
                                              (lc.max_nodes + 7) / 8, (uint32_t)lc.sm_count * 8}) + 8;
    // size one instance, then allocate all
    Arena sizing;
    InstDesc tmp{};
    const size_t per = layout_instance(sizing, tmp, lc, b->cap_edges, lc.max_tp, lc.max_tc, gmax);
    b->per_inst_bytes = per;
    b->arena_bytes = per * B;
    cudaError_t e = cudaMalloc(&b->arena, b->arena_bytes);
    if (e != cudaSuccess) {
        delete b;
        return fail(MVDR_ECUDA, std::string("workspace allocation failed: ") + cudaGetErrorString(e));
    }
    e = cudaMemset(b->arena, 0, b->arena_bytes);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_inst, sizeof(InstDesc) * B);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_bars, sizeof(uint32_t) * 32 * B);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->side, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->ev_join, cudaEventDisableTiming);
    if (e != cudaSuccess) {
        delete b;
        return fail(MVDR_ECUDA, std::string("workspace setup failed: ") + cudaGetErrorString(e));
    }
    b->host.resize(B);
    for (uint32_t i = 0; i < B; ++i) {
        Arena a;
        a.base = static_cast<char*>(b->arena) + per * i;
        InstDesc& I = b->host[i];
        std::memset(&I, 0, sizeof(I));
        layout_instance(a, I, lc, b->cap_edges, lc.max_tp, lc.max_tc, gmax);
        I.pcg_bar = b->d_bars + 32 * i;
    }
    b->lc.pcg_bars = b->d_bars;
    b->lc.pcg_persistent = 0;
    b->lc.wait_limit_ns = kDefaultWaitLimitNs;
    b->lc.wait_extra_arrivals = 0;
    b->lc.pcg_grid = persistent_pcg_grid(lc.precision == MVDR_PRECISION_MIXED, lc.sm_count);
    b->owned.resize(B);
    b->staged.resize(B);
    b->bound.resize(B);
    b->has_inputs.assign(B, 0);
    b->uploaded.resize(B);
    b->uploaded_valid.assign(B, 0);
    e = cudaMemcpy(b->d_inst, b->host.data(), sizeof(InstDesc) * B, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        delete b;
        return fail(MVDR_ECUDA, std::string("descriptor upload failed: ") + cudaGetErrorString(e));
    }
    b->views.resize(B);
    for (uint32_t i = 0; i < B; ++i) {
        b->views[i] = new SolverView();
        b->views[i]->s = mvdr_solver{b, i, false};
    }
    *out = b;
    return MVDR_OK;
}

static M34 load34(const mvdr_mat34& a) {
    M34 m;
    for (int c = 0; c < 3; ++c)
        for (int r = 0; r < 3; ++r) m.r[3 * r + c] = a.rot[3 * c + r];
    for (int r = 0; r < 3; ++r) m.t[r] = a.trans[r];
    return m;
}

// mat34::inverse (math/MatUtils.h:585-590) in float
static M34 inverse34(const M34& a) {
    M34 o;
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) o.r[3 * r + c] = a.r[3 * c + r];
    for (int r = 0; r < 3; ++r) o.t[r] = -(o.r[3 * r] * a.t[0] + o.r[3 * r + 1] * a.t[1] + o.r[3 * r + 2] * a.t[2]);
    return o;
}

int check_inputs(const Batch& b, const mvdr_inputs* in) {
    const mvdr_config& c = b.cfg;
    if (!in) return fail(MVDR_EINVAL, "inputs is null");
    if (in->num_views == 0 || in->num_views > c.max_views) return fail(MVDR_ECAPACITY, "num_views exceeds max_views");
    if (in->num_nodes == 0 || in->num_nodes > c.max_nodes) return fail(MVDR_ECAPACITY, "num_nodes exceeds max_nodes");
    if (in->num_surfels > c.max_surfels && c.max_surfels) return fail(MVDR_ECAPACITY, "num_surfels exceeds max_surfels");
    if (in->num_graph_edges > b.cap_edges) return fail(MVDR_ECAPACITY, "node graph larger than 8 * max_nodes");
    if (c.use_feature && in->feature.count > c.max_feature_terms)
        return fail(MVDR_ECAPACITY, "feature terms exceed max_feature_terms");
    if (c.use_cross_view && in->cross_view.count > c.max_cross_terms)
        return fail(MVDR_ECAPACITY, "cross-view terms exceed max_cross_terms");
    if (!in->node_se3 || !in->canonical_node_coords || (in->num_graph_edges && !in->node_graph) ||
        (in->num_surfels && (!in->surfel_knn || !in->surfel_knn_weight)))
        return fail(MVDR_EINVAL, "missing node or surfel arrays");
    for (uint32_t v = 0; v < in->num_views; ++v) {
        const mvdr_view_inputs& V = in->views[v];
        if (!V.reference_vertex_map || !V.reference_normal_map || !V.index_map || !V.vertex_confidence_map ||
            !V.normal_radius_map)
            return fail(MVDR_EINVAL, "missing view maps");
        if (V.pitch && V.pitch < c.image_width) return fail(MVDR_EINVAL, "pitch smaller than image width");
        if (c.use_foreground && (!V.filtered_foreground_mask || !V.foreground_mask_gradient))
            return fail(MVDR_EINVAL, "foreground term on but mask maps missing");
        if (c.use_density && (!V.normalized_rgb_map || !V.density_map || !V.density_gradient_map))
            return fail(MVDR_EINVAL, "density term on but density maps missing");
    }
    if (c.use_feature && in->feature.count &&
        (!in->feature.target_vertex || !in->feature.reference_vertex || !in->feature.knn || !in->feature.knn_weight))
        return fail(MVDR_EINVAL, "missing feature arrays");
    uint64_t pairs = 0;
    for (uint32_t v = 0; v < MVDR_MAX_VIEWS; ++v) {
        const uint32_t n = in->feature_pairs.count[v];
        if (!n) continue;
        if (v >= in->num_views) return fail(MVDR_EINVAL, "feature pixel pairs given for a view that is not bound");
        if (!in->feature_pairs.pixel_pairs[v] || !in->feature_pairs.live_vertex_map[v])
            return fail(MVDR_EINVAL, "feature pixel pairs need their pairs and the live vertex map");
        pairs += n;
    }
    if (pairs) {
        if (!c.use_feature) return fail(MVDR_EINVAL, "feature pixel pairs given with the feature term off");
        if (in->feature.count) return fail(MVDR_EINVAL, "give either feature pixel pairs or feature correspondences");
        if (pairs > c.max_feature_terms) return fail(MVDR_ECAPACITY, "feature pixel pairs exceed max_feature_terms");
    }
    if (c.use_cross_view && in->cross_view.count &&
        (!in->cross_view.target_vertex || !in->cross_view.reference_vertex || !in->cross_view.knn ||
         !in->cross_view.knn_weight))
        return fail(MVDR_EINVAL, "missing cross-view arrays");
    return MVDR_OK;
}

int bind_inputs(Batch& b, uint32_t inst, const mvdr_inputs* in, cudaStream_t st) {
    int rc = check_inputs(b, in);
    if (rc != MVDR_OK) return rc;
    const mvdr_config& c = b.cfg;
    InstDesc& I = b.host[inst];
    I.num_views = in->num_views;
    I.N = in->num_nodes;
    I.S = in->num_surfels;
    I.E = in->num_graph_edges;
    I.Tp = c.use_feature ? in->feature.count : 0;
    I.Tc = c.use_cross_view ? in->cross_view.count : 0;
    I.width = c.image_width;
    I.height = c.image_height;
    uint32_t enc = 4096;  // EncodeUtils.h:187-204, widened past 4096 nodes
    while (enc < I.N) enc <<= 1;
    I.enc = enc;
    I.compat = c.compat_flags;
    I.use_fg = c.use_foreground ? 1u : 0u;
    I.use_density = c.use_density ? 1u : 0u;
    I.node_radius = c.node_radius;
    for (uint32_t v = 0; v < MVDR_MAX_VIEWS; ++v) {
        ViewDesc& V = I.views[v];
        std::memset(&V, 0, sizeof(V));
        if (v >= in->num_views) continue;
        const mvdr_view_inputs& S = in->views[v];
        V.ref_v = reinterpret_cast<const float4*>(S.reference_vertex_map);
        V.ref_n = reinterpret_cast<const float4*>(S.reference_normal_map);
        V.index = S.index_map;
        V.obs_v = reinterpret_cast<const float4*>(S.vertex_confidence_map);
        V.obs_n = reinterpret_cast<const float4*>(S.normal_radius_map);
        // the mask is bound whenever given: the post-solve node error reads it
        V.fg = S.filtered_foreground_mask;
        V.fg_grad = c.use_foreground ? reinterpret_cast<const float2*>(S.foreground_mask_gradient) : nullptr;
        V.rgb = c.use_density ? reinterpret_cast<const float4*>(S.normalized_rgb_map) : nullptr;
        V.dens = c.use_density ? S.density_map : nullptr;
        V.dens_grad = c.use_density ? reinterpret_cast<const float2*>(S.density_gradient_map) : nullptr;
        V.pitch = S.pitch ? S.pitch : c.image_width;
        V.cx = S.intrinsic.principal_x;
        V.cy = S.intrinsic.principal_y;
        V.fx = S.intrinsic.focal_x;
        V.fy = S.intrinsic.focal_y;
        V.w2c = load34(S.world2camera);
        V.init = load34(S.initial_camera_se3);
        V.init_inv = inverse34(V.init);
        V.c2w = inverse34(V.w2c);
        // double copies for the mixed-precision residual chain
        const M34* src[3] = {&V.w2c, &V.init, &V.init_inv};
        double* dst[3] = {V.w2c_d, V.init_d, V.init_inv_d};
        for (int m = 0; m < 3; ++m) {
            for (int q = 0; q < 9; ++q) dst[m][q] = (double)src[m]->r[q];
            for (int q = 0; q < 3; ++q) dst[m][9 + q] = (double)src[m]->t[q];
        }
    }
    I.surfel_knn = reinterpret_cast<const ushort4*>(in->surfel_knn);
    I.surfel_w = reinterpret_cast<const float4*>(in->surfel_knn_weight);
    I.nodes = reinterpret_cast<const float4*>(in->canonical_node_coords);
    I.graph = reinterpret_cast<const ushort2*>(in->node_graph);
    I.feat_target = reinterpret_cast<const float4*>(in->feature.target_vertex);
    I.feat_ref = reinterpret_cast<const float4*>(in->feature.reference_vertex);
    I.feat_knn = reinterpret_cast<const ushort4*>(in->feature.knn);
    I.feat_w = reinterpret_cast<const float4*>(in->feature.knn_weight);
    I.cross_target = reinterpret_cast<const float4*>(in->cross_view.target_vertex);
    I.cross_ref = reinterpret_cast<const float4*>(in->cross_view.reference_vertex);
    I.cross_knn = reinterpret_cast<const ushort4*>(in->cross_view.knn);
    I.cross_w = reinterpret_cast<const float4*>(in->cross_view.knn_weight);
    uint32_t pairs = 0;
    for (uint32_t v = 0; v < MVDR_MAX_VIEWS; ++v) {
        I.fp_offset[v] = pairs;
        const bool on = v < in->num_views && c.use_feature;
        const uint32_t n = on ? in->feature_pairs.count[v] : 0;
        I.fp_pairs[v] = n ? reinterpret_cast<const ushort4*>(in->feature_pairs.pixel_pairs[v]) : nullptr;
        I.fp_live[v] = n ? reinterpret_cast<const float4*>(in->feature_pairs.live_vertex_map[v]) : nullptr;
        I.fp_edge[v] = n ? in->feature_pairs.edge_mask[v] : nullptr;
        pairs += n;
    }
    I.fp_offset[MVDR_MAX_VIEWS] = pairs;
    I.feat_select = pairs ? 1u : 0u;
    if (pairs) {
        // the selected terms live in the solver's arrays; Tp is the capacity
        I.Tp = c.max_feature_terms;
        I.feat_target = I.fp_target;
        I.feat_ref = I.fp_ref;
        I.feat_knn = I.fp_knn;
        I.feat_w = I.fp_w;
    }
    // SolverIterationData::SetWarpFieldInitialValue (SolverIterationData.cpp:37-50)
    CU(cudaMemcpyAsync(I.se3, in->node_se3, sizeof(DQ) * I.N, cudaMemcpyDefault, st));
    CU(cudaMemsetAsync(I.counts, 0, sizeof(DeviceCounts), st));
    if (!b.uploaded_valid[inst] || std::memcmp(&b.uploaded[inst], &I, sizeof(InstDesc)) != 0) {
        CU(cudaMemcpyAsync(b.d_inst + inst, &I, sizeof(InstDesc), cudaMemcpyHostToDevice, st));
        b.uploaded[inst] = I;
        b.uploaded_valid[inst] = 1;
    }
    b.has_inputs[inst] = 1;
    b.bound[inst] = *in;
    b.gn_iter = 0;
    return MVDR_OK;
}

// copy host arrays into owned device buffers, then bind them
static int bind_inputs_host(Batch& b, uint32_t inst, const mvdr_inputs* in, cudaStream_t st) {
    int rc = check_inputs(b, in);
    if (rc != MVDR_OK) return rc;
    const mvdr_config& c = b.cfg;
    const size_t W = c.image_width, H = c.image_height;
    struct Item { const void* src; size_t bytes; };
    std::vector<Item> items;
    mvdr_inputs dev = *in;
    auto add = [&](const void* src, size_t bytes) { items.push_back({src, bytes}); };
    for (uint32_t v = 0; v < in->num_views; ++v) {
        const mvdr_view_inputs& V = in->views[v];
        const size_t pitch = V.pitch ? V.pitch : W;
        const size_t np = pitch * H;
        add(V.reference_vertex_map, 16 * np);
        add(V.reference_normal_map, 16 * np);
        add(V.index_map, 4 * np);
        add(V.vertex_confidence_map, 16 * np);
        add(V.normal_radius_map, 16 * np);
        add(V.filtered_foreground_mask, V.filtered_foreground_mask ? 4 * np : 0);
        add(c.use_foreground ? V.foreground_mask_gradient : nullptr, c.use_foreground ? 8 * np : 0);
        add(c.use_density ? V.normalized_rgb_map : nullptr, c.use_density ? 16 * np : 0);
        add(c.use_density ? V.density_map : nullptr, c.use_density ? 4 * np : 0);
        add(c.use_density ? V.density_gradient_map : nullptr, c.use_density ? 8 * np : 0);
    }
    add(in->surfel_knn, 8 * (size_t)in->num_surfels);
    add(in->surfel_knn_weight, 16 * (size_t)in->num_surfels);
    add(in->node_se3, 32 * (size_t)in->num_nodes);
    add(in->canonical_node_coords, 16 * (size_t)in->num_nodes);
    add(in->node_graph, 4 * (size_t)in->num_graph_edges);
    const uint32_t tp = c.use_feature ? in->feature.count : 0, tc = c.use_cross_view ? in->cross_view.count : 0;
    add(in->feature.target_vertex, 16 * (size_t)tp);
    add(in->feature.reference_vertex, 16 * (size_t)tp);
    add(in->feature.knn, 8 * (size_t)tp);
    add(in->feature.knn_weight, 16 * (size_t)tp);
    add(in->cross_view.target_vertex, 16 * (size_t)tc);
    add(in->cross_view.reference_vertex, 16 * (size_t)tc);
    add(in->cross_view.knn, 8 * (size_t)tc);
    add(in->cross_view.knn_weight, 16 * (size_t)tc);
    for (uint32_t v = 0; v < in->num_views; ++v) {
        const uint32_t n = c.use_feature ? in->feature_pairs.count[v] : 0;
        const size_t np = (size_t)(in->views[v].pitch ? in->views[v].pitch : W) * H;
        add(n ? in->feature_pairs.pixel_pairs[v] : nullptr, 8 * (size_t)n);
        add(n ? in->feature_pairs.live_vertex_map[v] : nullptr, n ? 16 * np : 0);
        add(n ? in->feature_pairs.edge_mask[v] : nullptr, n && in->feature_pairs.edge_mask[v] ? np : 0);
    }
    size_t total = 0;
    for (auto& it : items) total += (it.bytes + 255) & ~(size_t)255;
    OwnedInputs& o = b.owned[inst];
    if (o.bytes < total) {
        // first call (or larger inputs): allocate the device copies once
        if (o.mem) CU(cudaFree(o.mem));
        o.mem = nullptr;
        o.bytes = 0;
        CU(cudaMalloc(&o.mem, total));
        o.bytes = total;
    }
    std::vector<void*> dst(items.size(), nullptr);
    // Arrays that follow each other on the host at the same offsets as their
    // device copies (gaps below 256 bytes, as a packing allocator leaves) are
    // sent as one copy: a few large transfers instead of one per array keep
    // the stream's queue short, so the caller's thread does not stall when it
    // overlaps uploads with solves.
    const char* run_src = nullptr;
    char* run_dst = nullptr;
    size_t run_len = 0;
    auto flush = [&]() -> cudaError_t {
        cudaError_t e = cudaSuccess;
        if (run_len) e = cudaMemcpyAsync(run_dst, run_src, run_len, cudaMemcpyHostToDevice, st);
        run_len = 0;
        return e;
    };
    size_t off = 0;
    for (size_t i = 0; i < items.size(); ++i) {
        if (items[i].bytes && items[i].src) {
            char* d = static_cast<char*>(o.mem) + off;
            const char* src = static_cast<const char*>(items[i].src);
            dst[i] = d;
            const bool joins = run_len && src >= run_src + run_len && (size_t)(src - (run_src + run_len)) < 256 &&
                               (size_t)(src - run_src) == (size_t)(d - run_dst);
            if (joins) {
                run_len = (size_t)(src - run_src) + items[i].bytes;
            } else {
                CU(flush());
                run_src = src;
                run_dst = d;
                run_len = items[i].bytes;
            }
        }
        off += (items[i].bytes + 255) & ~(size_t)255;
    }
    CU(flush());
    size_t k = 0;
    for (uint32_t v = 0; v < in->num_views; ++v) {
        mvdr_view_inputs& V = dev.views[v];
        V.reference_vertex_map = (const mvdr_float4*)dst[k++];
        V.reference_normal_map = (const mvdr_float4*)dst[k++];
        V.index_map = (const uint32_t*)dst[k++];
        V.vertex_confidence_map = (const mvdr_float4*)dst[k++];
        V.normal_radius_map = (const mvdr_float4*)dst[k++];
        V.filtered_foreground_mask = (const float*)dst[k++];
        V.foreground_mask_gradient = (const float*)dst[k++];
        V.normalized_rgb_map = (const mvdr_float4*)dst[k++];
        V.density_map = (const float*)dst[k++];
        V.density_gradient_map = (const float*)dst[k++];
    }
    dev.surfel_knn = (const uint16_t*)dst[k++];
    dev.surfel_knn_weight = (const mvdr_float4*)dst[k++];
    dev.node_se3 = (const mvdr_dual_quaternion*)dst[k++];
    dev.canonical_node_coords = (const mvdr_float4*)dst[k++];
    dev.node_graph = (const uint16_t*)dst[k++];
    dev.feature.target_vertex = (const mvdr_float4*)dst[k++];
    dev.feature.reference_vertex = (const mvdr_float4*)dst[k++];
    dev.feature.knn = (const uint16_t*)dst[k++];
    dev.feature.knn_weight = (const mvdr_float4*)dst[k++];
    dev.cross_view.target_vertex = (const mvdr_float4*)dst[k++];
    dev.cross_view.reference_vertex = (const mvdr_float4*)dst[k++];
    dev.cross_view.knn = (const uint16_t*)dst[k++];
    dev.cross_view.knn_weight = (const mvdr_float4*)dst[k++];
    for (uint32_t v = 0; v < in->num_views; ++v) {
        dev.feature_pairs.pixel_pairs[v] = (const uint16_t*)dst[k++];
        dev.feature_pairs.live_vertex_map[v] = (const mvdr_float4*)dst[k++];
        dev.feature_pairs.edge_mask[v] = (const uint8_t*)dst[k++];
    }
    return bind_inputs(b, inst, &dev, st);
}

static int all_bound(const Batch& b) {
    for (uint32_t i = 0; i < b.B; ++i)
        if (!b.has_inputs[i]) return fail(MVDR_ESTATE, "inputs not set for every instance");
    return MVDR_OK;
}

// NVTX ranges around the enqueued stages, for profilers (`ncu --nvtx
// --nvtx-include "mvdr/pcg/"` takes one stage's kernels); without a tool
// attached the calls return at once
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
};

static int enqueue_index(Batch& b, cudaStream_t st) {
    NvtxRange range("mvdr/index");
    // zero the per-build counters of every instance
    for (uint32_t i = 0; i < b.B; ++i) {
        const InstDesc& I = b.host[i];
        CU(cudaMemsetAsync(I.counts, 0, sizeof(DeviceCounts), st));
        CU(cudaMemsetAsync(I.n2t_count, 0, sizeof(uint32_t) * (b.lc.max_nodes + 1), st));
    }
    CU(launch_build_index(b.lc, b.d_inst, st));
    return MVDR_OK;
}

static int enqueue_iteration(Batch& b, uint32_t iter, uint32_t pcg, cudaStream_t st) {
    NvtxRange range("mvdr/gn_iteration");
    const mvdr_penalty lam = penalty_for(b.cfg, iter);
    {
        NvtxRange r("mvdr/terms");
        CU(launch_eval_terms(b.lc, b.d_inst, lam, st));
        CU(launch_energy(b.lc, b.d_inst, std::min<uint32_t>(iter, 63), st));
    }
    {
        NvtxRange r("mvdr/assemble");
        if (b.cfg.mode == MVDR_MODE_MATERIALIZED)
            CU(launch_assemble_forked(b.lc, b.d_inst, lam, st, b.side, b.ev_fork, b.ev_join));
        else
            CU(launch_assemble(b.lc, b.d_inst, lam, false, st));
    }
    {
        NvtxRange r("mvdr/pcg");
        CU(launch_pcg(b.lc, b.d_inst, lam, pcg, iter, st));
    }
    {
        NvtxRange r("mvdr/update");
        CU(launch_update(b.lc, b.d_inst, st));
    }
    return MVDR_OK;
}

static int solve_batch(Batch& b, uint32_t gn, uint32_t pcg, bool graph, cudaStream_t st) {
    NvtxRange range("mvdr/solve");
    int rc = all_bound(b);
    if (rc != MVDR_OK) return rc;
    if (gn > 63) return fail(MVDR_EINVAL, "at most 63 Gauss-Newton iterations per solve");
    if (!graph) {
        rc = enqueue_index(b, st);
        if (rc != MVDR_OK) return rc;
        for (uint32_t k = 0; k < gn; ++k) {
            rc = enqueue_iteration(b, k, pcg, st);
            if (rc != MVDR_OK) return rc;
        }
        b.gn_iter = gn;
        return MVDR_OK;
    }
    auto key = std::make_pair(gn, pcg);
    auto it = b.graphs.find(key);
    if (it == b.graphs.end()) {
        // capture the whole solve once; the descriptors are read from device
        // memory, so the graph stays valid across set_inputs calls
        cudaStream_t cap;
        CU(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) {
            cudaStreamDestroy(cap);
            return fail(MVDR_ECUDA, std::string("begin capture: ") + cudaGetErrorString(e));
        }
        rc = enqueue_index(b, cap);
        for (uint32_t k = 0; rc == MVDR_OK && k < gn; ++k) rc = enqueue_iteration(b, k, pcg, cap);
        e = cudaStreamEndCapture(cap, &g);
        cudaStreamDestroy(cap);
        if (rc != MVDR_OK) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        if (e != cudaSuccess) return fail(MVDR_ECUDA, std::string("end capture: ") + cudaGetErrorString(e));
        cudaGraphExec_t ex = nullptr;
        e = cudaGraphInstantiate(&ex, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return fail(MVDR_ECUDA, std::string("instantiate: ") + cudaGetErrorString(e));
        it = b.graphs.emplace(key, ex).first;
    }
    CU(cudaGraphLaunch(it->second, st));
    count_launch();
    b.gn_iter = gn;
    return MVDR_OK;
}

static int read_counts(Batch& b, uint32_t inst, DeviceCounts& c, cudaStream_t st) {
    CU(cudaStreamSynchronize(st));
    CU(cudaMemcpy(&c, b.host[inst].counts, sizeof(DeviceCounts), cudaMemcpyDeviceToHost));
    return MVDR_OK;
}

static int check_flags(const DeviceCounts& c) {
    if (c.error_flags & (kErrDenseCapacity | kErrForegroundCapacity | kErrNode2TermCapacity |
                         kErrNodePairEntryCapacity | kErrHalfPairCapacity | kErrSegmentTooLong | kErrRowTooLong |
                         kErrBinBlockCapacity)) {
        char buf[96];
        std::snprintf(buf, sizeof(buf), "device capacity exceeded (flags 0x%x)", c.error_flags);
        return fail(MVDR_ECAPACITY, buf);
    }
    if (c.error_flags & kErrBadNodeIndex) return fail(MVDR_EINVAL, "node or surfel index out of range in inputs");
    if (c.error_flags & kErrWaitTimeout) return fail(MVDR_ETIMEOUT, "a bounded device-side wait gave up");
    if (c.error_flags & kErrNonFinite)
        return fail(MVDR_ENONFINITE, "NaN or Inf in a residual, the PCG step or the warp field");
    return MVDR_OK;
}

// a double vector exported as float (the export format of JTR / INCREMENT)
static int copy_out_as_float(void* dst, const double* src, size_t count, size_t cap, size_t* written) {
    if (written) *written = 4 * count;
    if (4 * count > cap) return fail(MVDR_ECAPACITY, "destination buffer too small");
    std::vector<double> h(count);
    if (count) CU(cudaMemcpy(h.data(), src, 8 * count, cudaMemcpyDeviceToHost));
    std::vector<float> f(h.begin(), h.end());
    if (count) CU(cudaMemcpy(dst, f.data(), 4 * count, cudaMemcpyDefault));
    return MVDR_OK;
}

static int copy_out(void* dst, const void* src, size_t bytes, size_t cap, size_t* written) {
    if (written) *written = bytes;
    if (bytes > cap) return fail(MVDR_ECAPACITY, "destination buffer too small");
    if (bytes) CU(cudaMemcpy(dst, src, bytes, cudaMemcpyDefault));
    return MVDR_OK;
}

static int get_array(Batch& b, uint32_t inst, int which, void* dst, size_t cap, size_t* written, cudaStream_t st) {
    DeviceCounts c;
    int rc = read_counts(b, inst, c, st);
    if (rc != MVDR_OK) return rc;
    const InstDesc& I = b.host[inst];
    const size_t N = I.N, P = c.half_pairs;
    switch (which) {
        case MVDR_ARRAY_DENSE_PIXELS: return copy_out(dst, I.dense_pix, 8 * (size_t)c.dense_terms, cap, written);
        case MVDR_ARRAY_DENSE_KNN: return copy_out(dst, I.dense_knn, 8 * (size_t)c.dense_terms, cap, written);
        case MVDR_ARRAY_DENSE_KNN_WEIGHT: return copy_out(dst, I.dense_w, 16 * (size_t)c.dense_terms, cap, written);
        case MVDR_ARRAY_FOREGROUND_PIXELS: return copy_out(dst, I.fg_pix, 8 * (size_t)c.foreground_terms, cap, written);
        case MVDR_ARRAY_NODE2TERM_OFFSET: return copy_out(dst, I.n2t_offset, 4 * (N + 1), cap, written);
        case MVDR_ARRAY_NODE2TERM_INDEX: return copy_out(dst, I.n2t_index, 4 * (size_t)c.node2term_entries, cap, written);
        case MVDR_ARRAY_HALF_NODEPAIR_KEY: return copy_out(dst, I.half_key, 4 * P, cap, written);
        case MVDR_ARRAY_NODEPAIR_TERM_INDEX: return copy_out(dst, I.np_index, 4 * (size_t)c.nodepair_entries, cap, written);
        case MVDR_ARRAY_NODEPAIR_KEY: return copy_out(dst, I.sym_key, 8 * P, cap, written);
        case MVDR_ARRAY_NODEPAIR_TERM_RANGE: return copy_out(dst, I.sym_range, 16 * P, cap, written);
        case MVDR_ARRAY_BLKROW_OFFSET: return copy_out(dst, I.blkrow_offset, 4 * (N + 1), cap, written);
        case MVDR_ARRAY_BINBLOCK_ROWPTR:
            return copy_out(dst, I.bb_rowptr, 4 * 32 * ((size_t)c.num_bins + 1), cap, written);
        case MVDR_ARRAY_BINBLOCK_COLPTR: return copy_out(dst, I.bb_colptr, 4 * ((size_t)c.binblock_nnz / 6), cap, written);
        case MVDR_ARRAY_TERM_JACOBIAN:
            return copy_out(dst, I.term_jr, 32 * ((size_t)c.dense_terms + c.foreground_terms), cap, written);
        case MVDR_ARRAY_SMOOTH_TERMS: return copy_out(dst, I.smooth, 48 * (size_t)I.E, cap, written);
        case MVDR_ARRAY_WARPED_CORRESPONDENCE:
            return copy_out(dst, I.warped, 32 * ((size_t)I.Tp + I.Tc), cap, written);
        case MVDR_ARRAY_DIAG_BLOCKS: return copy_out(dst, I.diag, 4 * 36 * N, cap, written);
        case MVDR_ARRAY_JTR:
            return I.jtr_d ? copy_out_as_float(dst, I.jtr_d, 6 * N, cap, written)
                           : copy_out(dst, I.jtr, 4 * 6 * N, cap, written);
        case MVDR_ARRAY_INCREMENT:
            return I.x_d ? copy_out_as_float(dst, I.x_d, 6 * N, cap, written)
                         : copy_out(dst, I.x, 4 * 6 * N, cap, written);
        case MVDR_ARRAY_NODE_SE3: return copy_out(dst, I.se3, 32 * N, cap, written);
        case MVDR_ARRAY_DENSITY_JACOBIAN:
            if (!I.density_jr) return fail(MVDR_EINVAL, "the density term is off");
            return copy_out(dst, I.density_jr, 32 * (size_t)c.dense_terms, cap, written);
        case MVDR_ARRAY_PCG_RESIDUALS: {
            const size_t rows = std::min<size_t>(b.gn_iter, kPcgHistRows);
            return copy_out(dst, I.pcg_hist, sizeof(double) * MVDR_PCG_HISTORY * rows, cap, written);
        }
        case MVDR_ARRAY_FEATURE_TERMS: {
            // (target, reference) per term, interleaved on the host
            const size_t n = c.feature_terms;
            *written = 32 * n;
            if (cap < 32 * n) return fail(MVDR_ECAPACITY, "destination too small");
            if (n == 0) return MVDR_OK;
            std::vector<float4> t(n), r(n);
            CU(cudaMemcpy(t.data(), I.feat_target, 16 * n, cudaMemcpyDeviceToHost));
            CU(cudaMemcpy(r.data(), I.feat_ref, 16 * n, cudaMemcpyDeviceToHost));
            float4* out = static_cast<float4*>(dst);
            for (size_t k = 0; k < n; ++k) {
                out[2 * k] = t[k];
                out[2 * k + 1] = r[k];
            }
            return MVDR_OK;
        }
        case MVDR_ARRAY_PRECONDITIONER:
        case MVDR_ARRAY_OFFDIAG_BLOCKS:
        case MVDR_ARRAY_BINBLOCK_DATA: {
            size_t bytes = which == MVDR_ARRAY_PRECONDITIONER ? 4 * 36 * N
                           : which == MVDR_ARRAY_OFFDIAG_BLOCKS ? 4 * 36 * 2 * P
                                                                 : 4 * (size_t)c.binblock_nnz;
            if (written) *written = bytes;
            if (bytes > cap) return fail(MVDR_ECAPACITY, "destination buffer too small");
            if (bytes == 0) return MVDR_OK;
            // diagnostic path: a temporary device buffer for the reformatted array
            float* tmp = nullptr;
            CU(cudaMalloc(&tmp, bytes));
            cudaError_t e;
            if (which == MVDR_ARRAY_PRECONDITIONER) e = launch_export_preconditioner(b.lc, b.d_inst, inst, tmp, st);
            else if (which == MVDR_ARRAY_OFFDIAG_BLOCKS) e = launch_export_offdiag(b.lc, b.d_inst, inst, tmp, st);
            else {
                e = cudaMemsetAsync(tmp, 0, bytes, st);
                if (e == cudaSuccess) {
                    export_binblock_fill_kernel<<<b.lc.sm_count * 4, 256, 0, st>>>(b.d_inst, inst, tmp);
                    count_launch();
                    e = cudaGetLastError();
                }
            }
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
            if (e == cudaSuccess) e = cudaMemcpy(dst, tmp, bytes, cudaMemcpyDefault);
            cudaFree(tmp);
            if (e != cudaSuccess) return fail(MVDR_ECUDA, std::string("export: ") + cudaGetErrorString(e));
            return MVDR_OK;
        }
        default: return fail(MVDR_EINVAL, "unknown array id");
    }
}

}  // namespace mvdr

using namespace mvdr;

// ------------------------------------------------------------- C ABI -----
extern "C" {

void mvdr_config_default(mvdr_config* cfg, uint32_t max_nodes, uint32_t max_views, uint32_t image_width,
                         uint32_t image_height) {
    if (!cfg) return;
    std::memset(cfg, 0, sizeof(*cfg));
    cfg->abi_version = MVDR_ABI_VERSION;
    cfg->max_nodes = max_nodes;
    cfg->max_views = max_views;
    cfg->image_width = image_width;
    cfg->image_height = image_height;
    cfg->max_surfels = max_views * image_width * image_height;
    cfg->node_radius = 0.025f;
    cfg->precision = MVDR_PRECISION_MIXED;
    cfg->mode = MVDR_MODE_MATERIALIZED;
    cfg->use_elastic_penalty = 1;
    cfg->num_global_iterations = 3;
    cfg->penalty = mvdr_penalty{2.5f, 0.0f, 0.0f, 0.7f, 0.1f};  // PenaltyConstants::setDefaultValue
}

int mvdr_create(const mvdr_config* cfg, mvdr_solver** out) {
    if (!out) return fail(MVDR_EINVAL, "out is null");
    Batch* b = nullptr;
    int rc = create_batch(cfg, 1, &b);
    if (rc != MVDR_OK) return rc;
    *out = new mvdr_solver{b, 0, true};
    return MVDR_OK;
}

int mvdr_destroy(mvdr_solver* s) {
    if (!s) return MVDR_OK;
    if (!s->owns) return fail(MVDR_EINVAL, "solver belongs to a batch; destroy the batch");
    delete s->batch;
    delete s;
    return MVDR_OK;
}

int mvdr_set_inputs(mvdr_solver* s, const mvdr_inputs* in, void* stream) {
    if (!s) return fail(MVDR_EINVAL, "solver is null");
    return bind_inputs(*s->batch, s->inst, in, (cudaStream_t)stream);
}

int mvdr_set_inputs_host(mvdr_solver* s, const mvdr_inputs* in, void* stream) {
    if (!s) return fail(MVDR_EINVAL, "solver is null");
    return bind_inputs_host(*s->batch, s->inst, in, (cudaStream_t)stream);
}

int mvdr_build_index(mvdr_solver* s, void* stream) {
    if (!s) return fail(MVDR_EINVAL, "solver is null");
    if (!s->owns) return fail(MVDR_EINVAL, "use mvdr_batch_solve for batch members");
    int rc = all_bound(*s->batch);
    if (rc != MVDR_OK) return rc;
    rc = enqueue_index(*s->batch, (cudaStream_t)stream);
    if (rc == MVDR_OK) s->batch->gn_iter = 0;
    return rc;
}

int mvdr_gn_iteration(mvdr_solver* s, uint32_t pcg_iterations, void* stream) {
    if (!s) return fail(MVDR_EINVAL, "solver is null");
    if (!s->owns) return fail(MVDR_EINVAL, "use mvdr_batch_solve for batch members");
    Batch& b = *s->batch;
    int rc = all_bound(b);
    if (rc != MVDR_OK) return rc;
    if (b.gn_iter >= 63) return fail(MVDR_EINVAL, "too many Gauss-Newton iterations");
    rc = enqueue_iteration(b, b.gn_iter, pcg_iterations, (cudaStream_t)stream);
    if (rc == MVDR_OK) b.gn_iter++;
    return rc;
}

int mvdr_solve(mvdr_solver* s, uint32_t gn, uint32_t pcg, void* stream) {
    if (!s) return fail(MVDR_EINVAL, "solver is null");
    if (!s->owns) return fail(MVDR_EINVAL, "use mvdr_batch_solve for batch members");
    return solve_batch(*s->batch, gn, pcg, false, (cudaStream_t)stream);
}

int mvdr_get_node_se3(mvdr_solver* s, mvdr_dual_quaternion* dst, void* stream) {
    if (!s || !dst) return fail(MVDR_EINVAL, "null argument");
    Batch& b = *s->batch;
    DeviceCounts c;
    int rc = read_counts(b, s->inst, c, (cudaStream_t)stream);
    if (rc != MVDR_OK) return rc;
    rc = check_flags(c);
    if (rc != MVDR_OK) return rc;
    CU(cudaMemcpy(dst, b.host[s->inst].se3, sizeof(DQ) * b.host[s->inst].N, cudaMemcpyDefault));
    return MVDR_OK;
}

int mvdr_copy_node_se3_async(mvdr_solver* s, mvdr_dual_quaternion* dst, void* stream) {
    if (!s || !dst) return fail(MVDR_EINVAL, "null argument");
    Batch& b = *s->batch;
    CU(cudaMemcpyAsync(dst, b.host[s->inst].se3, sizeof(DQ) * b.host[s->inst].N, cudaMemcpyDefault,
                       (cudaStream_t)stream));
    return MVDR_OK;
}

int mvdr_get_counts(mvdr_solver* s, mvdr_counts* out, void* stream) {
    if (!s || !out) return fail(MVDR_EINVAL, "null argument");
    DeviceCounts c;
    int rc = read_counts(*s->batch, s->inst, c, (cudaStream_t)stream);
    if (rc != MVDR_OK) return rc;
    std::memcpy(out, &c, sizeof(mvdr_counts));
    return MVDR_OK;
}

int mvdr_get_energy(mvdr_solver* s, double* energy, void* stream) {
    if (!s || !energy) return fail(MVDR_EINVAL, "null argument");
    Batch& b = *s->batch;
    if (b.gn_iter == 0) return fail(MVDR_ESTATE, "no Gauss-Newton iteration has run");
    CU(cudaStreamSynchronize((cudaStream_t)stream));
    const uint32_t slot = std::min<uint32_t>(b.gn_iter - 1, 63);
    CU(cudaMemcpy(energy, b.host[s->inst].energy + slot, sizeof(double), cudaMemcpyDeviceToHost));
    return MVDR_OK;
}

int mvdr_get_array(mvdr_solver* s, int which, void* dst, size_t cap, size_t* written, void* stream) {
    if (!s || !dst) return fail(MVDR_EINVAL, "null argument");
    return get_array(*s->batch, s->inst, which, dst, cap, written, (cudaStream_t)stream);
}

int mvdr_apply_jtj(mvdr_solver* s, const float* x, float* y, void* stream) {
    if (!s || !x || !y) return fail(MVDR_EINVAL, "null argument");
    Batch& b = *s->batch;
    if (b.gn_iter == 0) return fail(MVDR_ESTATE, "no Gauss-Newton iteration has run");
    LaunchCfg lc = b.lc;
    lc.B = 1;
    const mvdr_penalty lam = penalty_for(b.cfg, b.gn_iter - 1);
    CU(launch_apply_jtj(lc, b.d_inst + s->inst, lam, x, y, (cudaStream_t)stream));
    return MVDR_OK;
}

int mvdr_batch_create(const mvdr_config* cfg, uint32_t n, mvdr_batch** out) {
    if (!out) return fail(MVDR_EINVAL, "out is null");
    Batch* b = nullptr;
    int rc = create_batch(cfg, n, &b);
    if (rc != MVDR_OK) return rc;
    *out = new mvdr_batch{b};
    return MVDR_OK;
}

int mvdr_batch_destroy(mvdr_batch* b) {
    if (!b) return MVDR_OK;
    delete b->batch;
    delete b;
    return MVDR_OK;
}

int mvdr_batch_set_inputs(mvdr_batch* b, uint32_t i, const mvdr_inputs* in, void* stream) {
    if (!b || i >= b->batch->B) return fail(MVDR_EINVAL, "bad batch or instance");
    return bind_inputs(*b->batch, i, in, (cudaStream_t)stream);
}

int mvdr_batch_set_inputs_host(mvdr_batch* b, uint32_t i, const mvdr_inputs* in, void* stream) {
    if (!b || i >= b->batch->B) return fail(MVDR_EINVAL, "bad batch or instance");
    return bind_inputs_host(*b->batch, i, in, (cudaStream_t)stream);
}

int mvdr_batch_solve(mvdr_batch* b, uint32_t gn, uint32_t pcg, int use_graph, void* stream) {
    if (!b) return fail(MVDR_EINVAL, "batch is null");
    return solve_batch(*b->batch, gn, pcg, use_graph != 0, (cudaStream_t)stream);
}

int mvdr_batch_get_node_se3(mvdr_batch* b, uint32_t i, mvdr_dual_quaternion* dst, void* stream) {
    if (!b || i >= b->batch->B) return fail(MVDR_EINVAL, "bad batch or instance");
    return mvdr_get_node_se3(&b->batch->views[i]->s, dst, stream);
}

int mvdr_batch_copy_node_se3_async(mvdr_batch* b, uint32_t i, mvdr_dual_quaternion* dst, void* stream) {
    if (!b || i >= b->batch->B) return fail(MVDR_EINVAL, "bad batch or instance");
    return mvdr_copy_node_se3_async(&b->batch->views[i]->s, dst, stream);
}

int mvdr_batch_autotune(mvdr_batch* bh, void* stream, double* times_ms, uint32_t capacity, uint32_t* rows,
                        uint32_t* split, uint32_t* form) {
    if (!bh) return fail(MVDR_EINVAL, "batch is null");
    Batch& b = *bh->batch;
    const cudaStream_t st = (cudaStream_t)stream;
    if (b.cfg.mode == MVDR_MODE_MATERIALIZED) {
        int rc = all_bound(b);
        if (rc != MVDR_OK) return rc;
        rc = enqueue_index(b, st);
        if (rc == MVDR_OK) rc = enqueue_iteration(b, 0, 1, st);
        if (rc != MVDR_OK) return rc;
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        CU(cudaEventCreate(&e0));
        CU(cudaEventCreate(&e1));
        constexpr int kReps = 20;
        int best = 0;
        float best_ms = 0.f;
        cudaError_t e = cudaSuccess;
        for (int i = 0; i < kNumSpmvShapes && e == cudaSuccess; ++i) {
            LaunchCfg lc = b.lc;
            lc.spmv_shape = i;
            for (int w = 0; w < 2 && e == cudaSuccess; ++w) e = launch_spmv(lc, b.d_inst, 0, st);
            if (e == cudaSuccess) e = cudaEventRecord(e0, st);
            for (int r = 0; r < kReps && e == cudaSuccess; ++r) e = launch_spmv(lc, b.d_inst, 0, st);
            if (e == cudaSuccess) e = cudaEventRecord(e1, st);
            if (e == cudaSuccess) e = cudaEventSynchronize(e1);
            float ms = 0.f;
            if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
            ms /= kReps;
            if (times_ms && (uint32_t)i < capacity) times_ms[i] = ms;
            if (i == 0 || ms < best_ms) {
                best = i;
                best_ms = ms;
            }
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (e != cudaSuccess) return fail(MVDR_ECUDA, std::string("autotune: ") + cudaGetErrorString(e));
        b.lc.spmv_shape = best;
        for (auto& kv : b.graphs) cudaGraphExecDestroy(kv.second);
        b.graphs.clear();
        b.gn_iter = 0;
    }
    if (rows) *rows = kSpmvShapes[b.lc.spmv_shape].rows;
    if (split) *split = kSpmvShapes[b.lc.spmv_shape].split;
    if (form) *form = kSpmvShapes[b.lc.spmv_shape].form;
    return MVDR_OK;
}

static_assert(kNumSpmvShapes == (int)MVDR_NUM_SPMV_SHAPES, "public shape count");

int mvdr_batch_set_spmv_shape(mvdr_batch* bh, uint32_t shape) {
    if (!bh || shape >= (uint32_t)kNumSpmvShapes) return fail(MVDR_EINVAL, "bad batch or SpMV shape");
    Batch& b = *bh->batch;
    b.lc.spmv_shape = (int)shape;
    for (auto& kv : b.graphs) cudaGraphExecDestroy(kv.second);
    b.graphs.clear();
    return MVDR_OK;
}

int mvdr_batch_set_pcg_persistent(mvdr_batch* bh, int on) {
    if (!bh) return fail(MVDR_EINVAL, "batch is null");
    Batch& b = *bh->batch;
    if (on && b.cfg.mode != MVDR_MODE_MATERIALIZED) return fail(MVDR_EINVAL, "persistent PCG needs the materialised mode");
    if (on && b.lc.pcg_grid < b.B) return fail(MVDR_EINVAL, "more instances than co-resident persistent CTAs");
    b.lc.pcg_persistent = on ? 1 : 0;
    for (auto& kv : b.graphs) cudaGraphExecDestroy(kv.second);
    b.graphs.clear();
    return MVDR_OK;
}

int mvdr_batch_set_wait_limit(mvdr_batch* bh, uint64_t limit_ns, uint32_t extra_arrivals) {
    if (!bh) return fail(MVDR_EINVAL, "batch is null");
    if (limit_ns == 0 || limit_ns > kMaxWaitLimitNs) return fail(MVDR_EINVAL, "wait limit must be in (0, 10 s]");
    Batch& b = *bh->batch;
    b.lc.wait_limit_ns = limit_ns;
    b.lc.wait_extra_arrivals = extra_arrivals;
    for (auto& kv : b.graphs) cudaGraphExecDestroy(kv.second);
    b.graphs.clear();
    return MVDR_OK;
}

int mvdr_batch_instance(mvdr_batch* b, uint32_t i, mvdr_solver** out) {
    if (!b || !out || i >= b->batch->B) return fail(MVDR_EINVAL, "bad batch or instance");
    *out = &b->batch->views[i]->s;
    return MVDR_OK;
}

int mvdr_batch_enqueue_stage(mvdr_batch* b, int stage, void* stream) {
    if (!b) return fail(MVDR_EINVAL, "batch is null");
    Batch& bb = *b->batch;
    int rc = all_bound(bb);
    if (rc != MVDR_OK) return rc;
    if (stage == MVDR_STAGE_INDEX) return enqueue_index(bb, (cudaStream_t)stream);
    if (stage < MVDR_STAGE_INDEX || stage > MVDR_STAGE_SCALE) return fail(MVDR_EINVAL, "unknown stage");
    // the J.d scratch exists only in the matrix-free mode
    if (stage == MVDR_STAGE_MATRIX_FREE && bb.cfg.mode != MVDR_MODE_MATRIX_FREE)
        return fail(MVDR_EINVAL, "the matrix-free stage needs the matrix-free mode");
    if (stage == MVDR_STAGE_SCALE && (bb.cfg.mode != MVDR_MODE_MATERIALIZED || bb.cfg.precision != MVDR_PRECISION_MIXED))
        return fail(MVDR_EINVAL, "the scaling stage needs mixed precision in the materialised mode");
    // a stage runs in full even when the last solve's convergence check
    // stopped its PCG (the flag is read only with a tolerance)
    if (bb.cfg.pcg_tolerance > 0.0f)
        for (uint32_t i = 0; i < bb.B; ++i)
            CU(cudaMemsetAsync(&bb.host[i].counts->pcg_stop, 0, sizeof(uint32_t), (cudaStream_t)stream));
    CU(launch_stage(bb.lc, bb.d_inst, penalty_for(bb.cfg, 0), stage, (cudaStream_t)stream));
    return MVDR_OK;
}

const char* mvdr_last_error_string(void) { return g_last_error.c_str(); }

uint64_t mvdr_kernel_launch_count(void) { return g_launches.load(); }

/* Layout report for the binding's self-check: sizes of the public structs. */
int mvdr_abi_layout(const char* name, size_t* size) {
    if (!name || !size) return MVDR_EINVAL;
    const struct { const char* n; size_t s; } table[] = {
        {"mvdr_float4", sizeof(mvdr_float4)}, {"mvdr_dual_quaternion", sizeof(mvdr_dual_quaternion)},
        {"mvdr_mat34", sizeof(mvdr_mat34)}, {"mvdr_intrinsic", sizeof(mvdr_intrinsic)},
        {"mvdr_penalty", sizeof(mvdr_penalty)}, {"mvdr_config", sizeof(mvdr_config)},
        {"mvdr_view_inputs", sizeof(mvdr_view_inputs)}, {"mvdr_correspondences", sizeof(mvdr_correspondences)},
        {"mvdr_inputs", sizeof(mvdr_inputs)}, {"mvdr_counts", sizeof(mvdr_counts)},
        {"mvdr_view_textures", sizeof(mvdr_view_textures)}, {"mvdr_feature_pairs", sizeof(mvdr_feature_pairs)},
        {"mvdr_surfel_geometry", sizeof(mvdr_surfel_geometry)},
        {"mvdr_solver_map_params", sizeof(mvdr_solver_map_params)},
        {"mvdr_solver_map_view", sizeof(mvdr_solver_map_view)}, {"mvdr_deform_surfels", sizeof(mvdr_deform_surfels)},
        {"mvdr_deform_nodes", sizeof(mvdr_deform_nodes)}, {"mvdr_node_error", sizeof(mvdr_node_error)},
        {"mvdr_correction_view", sizeof(mvdr_correction_view)}, {"mvdr_correction", sizeof(mvdr_correction)}};
    for (const auto& t : table)
        if (std::strcmp(t.n, name) == 0) { *size = t.s; return MVDR_OK; }
    return MVDR_EINVAL;
}

}  // extern "C"
