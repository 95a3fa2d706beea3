// Index build: pixel selection and compaction, node -> term index, node-pair
// -> term index, symmetric block-row structure and the bin-block CSR layout.
//
// Reference: ImageTermKNNFetcher.cu:19-137, DensityForegroundMapHandler.cu:17-146,
// Node2TermsIndex.cu:8-187, NodePair2TermsIndex.cu:11-296,
// NodePairRowColumnIndex.cu:19-308.
//
// The reference sorts (node, term) and (pair, term) key/value arrays with
// global CUB radix sorts and stable ordering. Both orders are the same as
// sorting unique composite keys (node, term) and (pair, term), so here the
// entries are counted and scattered into per-node segments with integer
// atomics and each short segment is then sorted in shared memory. The result
// is independent of the scatter order, hence bit-exact with the reference
// order and reproducible run to run. No host synchronisation is needed: every
// size lives in DeviceCounts.
#include "kernels_common.cuh"

namespace mvdr {

constexpr uint32_t kChunk = kChunkPixels;

// ----------------------------------------------------- input checks -----
// Node ids of the skinning, the node graph and the correspondences must be
// below num_nodes and surfel ids below num_surfels; otherwise the instance is
// flagged and every kernel that would index with them skips its work.
__global__ void __launch_bounds__(256) input_check_kernel(const InstDesc* insts, uint32_t width, uint32_t height) {
    const InstDesc& I = insts[blockIdx.y];
    const uint32_t stride = gridDim.x * blockDim.x;
    const uint32_t t0 = blockIdx.x * blockDim.x + threadIdx.x;
    bool bad = false;
    for (uint32_t i = t0; i < I.S; i += stride) {
        const ushort4 k = I.surfel_knn[i];
        bad |= k.x >= I.N || k.y >= I.N || k.z >= I.N || k.w >= I.N;
    }
    for (uint32_t i = t0; i < I.E; i += stride) {
        const ushort2 e = I.graph[i];
        bad |= e.x >= I.N || e.y >= I.N;
    }
    // selected feature terms take their skinning from the (checked) surfels
    const uint32_t tp = I.feat_select ? 0u : I.Tp;
    for (uint32_t i = t0; i < tp; i += stride) {
        const ushort4 k = I.feat_knn[i];
        bad |= k.x >= I.N || k.y >= I.N || k.z >= I.N || k.w >= I.N;
    }
    for (uint32_t i = t0; i < I.Tc; i += stride) {
        const ushort4 k = I.cross_knn[i];
        bad |= k.x >= I.N || k.y >= I.N || k.z >= I.N || k.w >= I.N;
    }
    const uint32_t npix = width * height;
    for (uint32_t v = 0; v < I.num_views; ++v) {
        const ViewDesc& V = I.views[v];
        for (uint32_t p = t0; p < npix; p += stride) {
            const uint32_t s = V.index[(size_t)(p / width) * V.pitch + p % width];
            bad |= s != kInvalid && s >= I.S;
        }
    }
    if (bad) set_error(I, kErrBadNodeIndex);
}

// ------------------------------------------------------- compaction -----

// a surfel id past the surfel array marks the pixel invalid (and is reported
// by input_check_kernel)
struct DensePred {
    __device__ static inline bool eval(const InstDesc& I, uint32_t v, uint32_t x, uint32_t y) {
        const ViewDesc& V = I.views[v];
        return V.index[(size_t)y * V.pitch + x] < I.S;
    }
};

// markValidColorForegroundMapsPixelKernel (DensityForegroundMapHandler.cu:34-105):
// project the initially warped surfel; keep it when it lands inside the image,
// faces the camera (cos > 0.5) and the filtered mask there is non-zero.
struct ForegroundPred {
    __device__ static inline bool eval(const InstDesc& I, uint32_t v, uint32_t x, uint32_t y) {
        const ViewDesc& V = I.views[v];
        const size_t p = (size_t)y * V.pitch + x;
        const uint32_t s = V.index[p];
        if (!I.use_fg || s >= I.S || V.fg == nullptr || bad_inputs(I)) return false;
        const float4 cv = V.ref_v[p], cn = V.ref_n[p];
        const float3 cv0 = apply3(V.init, mk3(cv.x, cv.y, cv.z));
        const float3 cn0 = rot3(V.init, mk3(cn.x, cn.y, cn.z));
        const M34 se3 = dq_se3(blend_dq(I.se3, I.surfel_knn[s], I.surfel_w[s]));
        const float3 wv = apply3(se3, cv0), wn = rot3(se3, cn0);
        const float3 vc = apply3(V.init_inv, apply3(V.w2c, wv));
        const float3 nc = rot3(V.init_inv, rot3(V.w2c, wn));
        const float inv = rsqrtf(dot3(vc, vc));
        const float cosang = -dot3(mul3(inv, vc), nc);
        const int u = project_coord(vc.x, vc.z, V.fx, V.cx);
        const int w = project_coord(vc.y, vc.z, V.fy, V.cy);
        if (u < 0 || u >= (int)I.width || w < 0 || w >= (int)I.height || !(cosang > 0.5f)) return false;
        return V.fg[(size_t)w * V.pitch + u] > 1e-5f;  // isValidForegroundMaskPixel
    }
};

template <class Pred>
__global__ void __launch_bounds__(256, 6) compact_count_kernel(const InstDesc* insts, uint32_t width, uint32_t height,
                                                            uint32_t cpv) {
    const InstDesc& I = insts[blockIdx.y];
    const uint32_t view = blockIdx.x / cpv, c = blockIdx.x % cpv;
    uint32_t cnt = 0;
    if (view < I.num_views) {
        const uint32_t npix = width * height;
        for (uint32_t k = 0; k < kChunk / 256; ++k) {
            const uint32_t p = c * kChunk + k * 256 + threadIdx.x;
            const bool ok = p < npix && Pred::eval(I, view, p % width, p / width);
            // the write pass reads the predicate back from these bits
            const uint32_t bal = __ballot_sync(0xffffffffu, ok);
            if (lane_id() == 0) I.pix_mask[(size_t)view * cpv * (kChunk / 32) + p / 32] = bal;
            cnt += ok ? 1u : 0u;
        }
    }
    cnt = warp_sum(cnt);
    __shared__ uint32_t ws[8];
    if (lane_id() == 0) ws[threadIdx.x >> 5] = cnt;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int i = 0; i < 8; ++i) t += ws[i];
        I.chunk_count[blockIdx.x] = t;
    }
}

// exclusive scan of the chunk counts; per-view totals; capacity check
__global__ void __launch_bounds__(1024) compact_scan_kernel(const InstDesc* insts, uint32_t cpv, uint32_t max_views,
                                                            int foreground) {
    const InstDesc& I = insts[blockIdx.y];
    DeviceCounts* C = I.counts;
    // per-view totals before the scan
    if (threadIdx.x < MVDR_MAX_VIEWS) {
        uint32_t t = 0;
        if (threadIdx.x < max_views)
            for (uint32_t c = 0; c < cpv; ++c) t += I.chunk_count[threadIdx.x * cpv + c];
        if (foreground) C->fg_view_count[threadIdx.x] = t;
        else C->dense_view_count[threadIdx.x] = t;
    }
    __syncthreads();
    uint32_t total = 0;
    __shared__ uint32_t tot;
    block_exclusive_scan_inplace(I.chunk_count, cpv * max_views, &tot);
    __syncthreads();
    if (threadIdx.x == 0) {
        total = tot;
        const uint32_t cap = foreground ? I.cap_fg : I.cap_dense;
        if (total > cap) {
            atomicOr(&C->error_flags, foreground ? kErrForegroundCapacity : kErrDenseCapacity);
            total = cap;
        }
        if (foreground) C->foreground_terms = total;
        else C->dense_terms = total;
    }
}

template <class Pred>
__global__ void __launch_bounds__(256) compact_write_kernel(const InstDesc* insts, uint32_t width, uint32_t height,
                                                            uint32_t cpv, int foreground) {
    const InstDesc& I = insts[blockIdx.y];
    const uint32_t view = blockIdx.x / cpv, c = blockIdx.x % cpv;
    if (view >= I.num_views) return;
    const uint32_t cap = foreground ? I.cap_fg : I.cap_dense;
    __shared__ uint32_t wtot[8];
    uint32_t carry = I.chunk_count[blockIdx.x];
    for (uint32_t k = 0; k < kChunk / 256; ++k) {
        const uint32_t p = c * kChunk + k * 256 + threadIdx.x;
        const uint32_t x = p % width, y = p / width;
        const uint32_t bal = I.pix_mask[(size_t)view * cpv * (kChunk / 32) + p / 32];
        const bool ok = (bal >> lane_id()) & 1u;
        const uint32_t lane_prefix = __popc(bal & ((1u << lane_id()) - 1u));
        if (lane_id() == 0) wtot[threadIdx.x >> 5] = __popc(bal);
        __syncthreads();
        uint32_t wbase = 0, slice = 0;
        for (uint32_t w = 0; w < 8; ++w) {
            if (w < (threadIdx.x >> 5)) wbase += wtot[w];
            slice += wtot[w];
        }
        if (ok) {
            const uint32_t out = carry + wbase + lane_prefix;
            if (out < cap) {
                const ViewDesc& V = I.views[view];
                const uint32_t s = V.index[(size_t)y * V.pitch + x];
                if (s < I.S) {
                    const ushort4 pix = make_ushort4((unsigned short)x, (unsigned short)y, (unsigned short)view, 0);
                    if (foreground) {
                        I.fg_pix[out] = pix;
                        I.fg_knn[out] = I.surfel_knn[s];
                        I.fg_w[out] = I.surfel_w[s];
                    } else {
                        I.dense_pix[out] = pix;
                        I.dense_knn[out] = I.surfel_knn[s];
                        I.dense_w[out] = I.surfel_w[s];
                    }
                } else {
                    set_error(I, kErrBadNodeIndex);
                }
            }
        }
        carry += slice;
        __syncthreads();
    }
}

// view whose maps a compacted pixel samples: its own tag, or in compat mode
// the reference's lookup that reads per-view counts as offsets
// (DenseDepthJacobianResidual.cu:14-22)
__device__ inline uint32_t sample_view(const InstDesc& I, ushort4 pix, uint32_t idx, const uint32_t* view_count) {
    if (!(I.compat & MVDR_COMPAT_REF_VIEW_LOOKUP)) return pix.z;
    for (uint32_t i = 0; i < I.num_views; ++i) {
        if (i == I.num_views - 1) return i;
        if (view_count[i] <= idx && idx < view_count[i + 1]) return i;
    }
    return I.num_views - 1;
}

// canonical vertex / normal of each compacted pixel in frame 0; constant over
// the Gauss-Newton iterations, so computed once per index build
__global__ void __launch_bounds__(256) prepare_pixels_kernel(const InstDesc* insts, bool mixed) {
    const InstDesc& I = insts[blockIdx.y];
    const DeviceCounts* C = I.counts;
    const uint32_t Td = C->dense_terms, Tf = C->foreground_terms;
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < Td + Tf; t += gridDim.x * blockDim.x) {
        const bool fg = t >= Td;
        const uint32_t k = fg ? t - Td : t;
        const ushort4 pix = fg ? I.fg_pix[k] : I.dense_pix[k];
        const uint32_t v = sample_view(I, pix, k, fg ? C->fg_view_count : C->dense_view_count);
        const ViewDesc& V = I.views[v];
        const size_t p = (size_t)pix.y * V.pitch + pix.x;
        const float4 cv = V.ref_v[p];
        // the foreground term's vertex stays in its camera's frame in the
        // reference's form (density_map_jacobian.cuh:32-36)
        const bool raw_frame = fg && (I.compat & MVDR_COMPAT_REF_FOREGROUND_FRAME);
        float3 a = raw_frame ? mk3(cv.x, cv.y, cv.z) : apply3(V.init, mk3(cv.x, cv.y, cv.z));
        if (!fg && mixed) {
            // The point-to-plane residual subtracts two ~1 m positions, and
            // near convergence Jt r cancels by orders of magnitude more, so
            // the FP32 rounding of this transform (~1e-7 m) would dominate
            // the increment. Keep the transform in double as hi + lo floats.
            const double* m = V.init_d;
            double ad[3];
#pragma unroll
            for (int r = 0; r < 3; ++r)
                ad[r] = m[3 * r] * (double)cv.x + m[3 * r + 1] * (double)cv.y + m[3 * r + 2] * (double)cv.z + m[9 + r];
            a = mk3((float)ad[0], (float)ad[1], (float)ad[2]);
            I.dense_cv_lo[k] = make_float4((float)(ad[0] - (double)a.x), (float)(ad[1] - (double)a.y),
                                           (float)(ad[2] - (double)a.z), 0.f);
        }
        if (fg) {
            I.fg_cv[k] = make_float4(a.x, a.y, a.z, __uint_as_float(v));
        } else {
            const float4 cn = V.ref_n[p];
            const float3 b = rot3(V.init, mk3(cn.x, cn.y, cn.z));
            // the rendered grey level of the density term: rgb2density of the
            // normalised rgb solver map (ColorTypeTransfer.h:51-56,
            // DensityForegroundJacobianResidual.cu:51-52)
            float geo = 0.f;
            if (I.use_density) {
                const float4 c = V.rgb[p];
                geo = 0.299f * c.x + 0.587f * c.y + 0.114f * c.z;
            }
            I.dense_cv[k] = make_float4(a.x, a.y, a.z, __uint_as_float(v));
            I.dense_cn[k] = make_float4(b.x, b.y, b.z, geo);
        }
    }
}

// ------------------------------------------- sparse feature selection -----
// SparseCorrespondenceHandler (SparseCorrespondenceHandler.cu:18-199), the
// nearest-distance form (USE_NEAREST_DISTANCE_PAIRS, solver_constants.h:9).
// Maps are read with the reference's border addressing: outside the image a
// float4 map reads zero and the index map reads 0, which counts as a surfel
// (it is not 0xFFFFFFFF); such a pixel's coordinate then wraps to 0xFFFF as
// an unsigned short and fails the image-size test, as in the reference.

__device__ inline float4 border4(const float4* m, int x, int y, uint32_t W, uint32_t H, uint32_t pitch) {
    if (x < 0 || y < 0 || x >= (int)W || y >= (int)H) return make_float4(0.f, 0.f, 0.f, 0.f);
    return m[(size_t)y * pitch + x];
}

// is_zero_vertex (VectorUtils.h:214-216): the 1e-3 bound is a double
__device__ inline bool zero_vertex4(float4 v) {
    return (double)fabsf(v.x) < 1e-3 && (double)fabsf(v.y) < 1e-3 && (double)fabsf(v.z) < 1e-3;
}

// The selection's float arithmetic is written with round-to-nearest
// intrinsics, which the compiler does not contract into FMAs: the kept pairs
// and the term positions are then the CPU restatement's to the bit (a one-ulp
// shift of a target moves the small late-iteration residuals measurably).
__device__ inline float sq_dist3(float4 a, float4 b) {
    const float dx = __fsub_rn(a.x, b.x), dy = __fsub_rn(a.y, b.y), dz = __fsub_rn(a.z, b.z);
    return __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
}

// m * p + t, uncontracted (mat34 applied as the reference writes it)
__device__ inline float3 apply3_rn(const M34& m, float3 p) {
    float o[3];
#pragma unroll
    for (int r = 0; r < 3; ++r)
        o[r] = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(m.r[3 * r], p.x), __fmul_rn(m.r[3 * r + 1], p.y)),
                                   __fmul_rn(m.r[3 * r + 2], p.z)),
                         m.t[r]);
    return mk3(o[0], o[1], o[2]);
}

// chooseValidPixelKernel: one thread per candidate pair
__global__ void __launch_bounds__(256) feat_choose_kernel(const InstDesc* insts) {
    const InstDesc& I = insts[blockIdx.y];
    if (!I.feat_select) return;
    const uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= I.fp_offset[MVDR_MAX_VIEWS]) return;
    uint32_t v = 0;
    while (v + 1 < I.num_views && idx >= I.fp_offset[v + 1]) ++v;
    const ViewDesc& V = I.views[v];
    const uint32_t W = I.width, H = I.height, P = V.pitch;
    const ushort4 pair = I.fp_pairs[v][idx - I.fp_offset[v]];
    // validDepthPixelInWindow: the last row's first non-zero vertex, the
    // centre preferred
    ushort2 dp = make_ushort2(0xFFFF, 0xFFFF);
    for (int y = (int)pair.w - 1; y <= (int)pair.w + 1; ++y)
        for (int x = (int)pair.z - 1; x <= (int)pair.z + 1; ++x)
            if (!zero_vertex4(border4(V.obs_v, x, y, W, H, P))) {
                dp = make_ushort2((unsigned short)x, (unsigned short)y);
                break;
            }
    if (!zero_vertex4(border4(V.obs_v, pair.z, pair.w, W, H, P))) dp = make_ushort2(pair.z, pair.w);
    uint32_t keep = 0;
    ushort4 chosen = make_ushort4(0, 0, 0, 0);
    const uint8_t* edge = I.fp_edge[v];
    const bool on_edge = edge && dp.x < W && dp.y < H && edge[(size_t)dp.y * P + dp.x] == 1;
    if (dp.x < W && dp.y < H && !on_edge) {
        const float4 ov = V.obs_v[(size_t)dp.y * P + dp.x];
        // validGeometryPixelInWindow (nearest form): the window pixel with a
        // surfel whose live vertex is nearest the observed vertex
        ushort2 gp = make_ushort2(0xFFFF, 0xFFFF);
        float best = 100.0f;
        for (int y = (int)pair.y - 1; y <= (int)pair.y + 1; ++y)
            for (int x = (int)pair.x - 1; x <= (int)pair.x + 1; ++x) {
                const bool in = x >= 0 && y >= 0 && x < (int)W && y < (int)H;
                const uint32_t s = in ? V.index[(size_t)y * P + x] : 0u;
                if (s != kInvalid) {
                    const float d = sq_dist3(ov, border4(I.fp_live[v], x, y, W, H, P));
                    if (d < best) {
                        gp = make_ushort2((unsigned short)x, (unsigned short)y);
                        best = d;
                    }
                }
            }
        if (gp.x < W && gp.y < H) {
            const size_t o = (size_t)gp.y * P + gp.x;
            const uint32_t s = V.index[o];
            // a pixel without a valid surfel id cannot give a skinning
            if (s < I.S && sq_dist3(V.ref_v[o], ov) < 2.5e-3f) {
                keep = 1;
                chosen = make_ushort4(gp.x, gp.y, dp.x, dp.y);
            }
        }
    }
    I.fp_keep[idx] = keep;
    I.fp_chosen[idx] = chosen;
}

// compactQueryValidPairsKernel: kept pairs in candidate order (one CTA of
// 1024 threads per instance: an exclusive scan of the keep flags, then each
// kept pair written at its prefix)
__global__ void __launch_bounds__(1024) feat_compact_kernel(const InstDesc* insts) {
    const InstDesc& I = insts[blockIdx.y];
    if (!I.feat_select) return;
    const uint32_t n = I.fp_offset[MVDR_MAX_VIEWS];
    __shared__ uint32_t total;
    block_exclusive_scan_inplace(I.fp_keep, n, &total);
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
        const uint32_t o = I.fp_keep[i];
        const uint32_t next = i + 1 < n ? I.fp_keep[i + 1] : total;
        if (next == o) continue;
        uint32_t v = 0;
        while (v + 1 < I.num_views && i >= I.fp_offset[v + 1]) ++v;
        const ViewDesc& V = I.views[v];
        const ushort4 c = I.fp_chosen[i];
        const size_t og = (size_t)c.y * V.pitch + c.x, oo = (size_t)c.w * V.pitch + c.z;
        const float4 rv = V.ref_v[og];
        const float3 r0 = apply3_rn(V.init, mk3(rv.x, rv.y, rv.z));
        const float4 dv = V.obs_v[oo];
        const float3 t0 = apply3_rn(V.c2w, apply3_rn(V.init, mk3(dv.x, dv.y, dv.z)));
        const uint32_t s = V.index[og];
        I.fp_target[o] = make_float4(t0.x, t0.y, t0.z, 1.0f);
        I.fp_ref[o] = make_float4(r0.x, r0.y, r0.z, rv.w);
        I.fp_knn[o] = I.surfel_knn[s];
        I.fp_w[o] = I.surfel_w[s];
    }
    if (threadIdx.x == 0) I.counts->feature_terms = total;
}

// size2offset (term_offset_types.h:44-64) on the device
__global__ void term_offsets_kernel(const InstDesc* insts) {
    const InstDesc& I = insts[blockIdx.y];
    if (threadIdx.x != 0) return;
    DeviceCounts* C = I.counts;
    C->smooth_terms = I.E;
    // selected feature terms: their count was written by feat_compact_kernel
    const uint32_t tp = I.feat_select ? C->feature_terms : I.Tp;
    C->feature_terms = tp;
    C->cross_terms = I.Tc;
    uint32_t o = C->dense_terms;
    C->term_offset[0] = o;
    o += I.E;
    C->term_offset[1] = o;
    o += C->foreground_terms;
    C->term_offset[2] = o;
    o += tp;
    C->term_offset[3] = o;
    o += I.Tc;
    C->term_offset[4] = o;
}

// ------------------------------------------------------ node -> term -----

// Neighbouring pixels share their KNN nodes, so the lanes of a warp that
// hold the same node are merged (match_any) and one lane adds the group's
// count: one atomic per distinct node and slot in the warp.
__global__ void __launch_bounds__(256) n2t_count_kernel(const InstDesc* insts) {
    const InstDesc& I = insts[blockIdx.y];
    if (bad_inputs(I)) return;
    TermOffsets off;
    off.load(I.counts);
    const uint32_t T = off.o[4], lane = lane_id();
    const uint32_t stride = gridDim.x * blockDim.x;
    // the warp's 32 terms per step, so that every lane takes part in the match
    for (uint32_t tw = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); tw < T; tw += stride) {
        const uint32_t t = tw + lane;
        uint32_t a[4] = {0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu};
        if (t < T) {
            uint32_t k;
            const TermType ty = off.typed(t, k);
            const ushort4 n = term_nodes(I, ty, k);
            const uint32_t m = ty == kSmooth ? 2 : 4;
            const unsigned short v[4] = {n.x, n.y, n.z, n.w};
            for (uint32_t j = 0; j < m; ++j) {
                if (v[j] < I.N) a[j] = v[j];
                else set_error(I, kErrBadNodeIndex);
            }
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const uint32_t grp = __match_any_sync(0xffffffffu, a[j]);
            if (a[j] != 0xFFFFFFFFu && lane == (uint32_t)(__ffs(grp) - 1))
                atomicAdd(&I.n2t_count[a[j]], (uint32_t)__popc(grp));
        }
    }
}
// single-CTA exclusive scans over per-node arrays
enum ScanWhat : int { kScanN2T = 0, kScanRows = 1, kScanUpper = 2, kScanBlkRows = 3, kScanBins = 4 };

__global__ void __launch_bounds__(1024) node_scan_kernel(const InstDesc* insts, int what) {
    const InstDesc& I = insts[blockIdx.y];
    DeviceCounts* C = I.counts;
    __shared__ uint32_t total;
    const uint32_t N = I.N;
    switch (what) {
        case kScanN2T: {
            for (uint32_t i = threadIdx.x; i <= N; i += blockDim.x) {
                I.n2t_offset[i] = i < N ? I.n2t_count[i] : 0u;
                if (i < N) I.n2t_cursor[i] = 0;
            }
            __syncthreads();
            block_exclusive_scan_inplace(I.n2t_offset, N + 1, &total);
            __syncthreads();
            if (threadIdx.x == 0) {
                C->node2term_entries = total;
                if (total > I.cap_k1) atomicOr(&C->error_flags, kErrNode2TermCapacity);
            }
            break;
        }
        case kScanRows: {
            for (uint32_t i = threadIdx.x; i <= N; i += blockDim.x) I.row_offset[i] = i < N ? I.row_count[i] : 0u;
            __syncthreads();
            block_exclusive_scan_inplace(I.row_offset, N + 1, &total);
            __syncthreads();
            if (threadIdx.x == 0) {
                C->nodepair_entries = total;
                if (total > I.cap_k2) atomicOr(&C->error_flags, kErrNodePairEntryCapacity);
            }
            break;
        }
        case kScanUpper: {
            for (uint32_t i = threadIdx.x; i <= N; i += blockDim.x) {
                I.half_offset[i] = i < N ? I.upper_count[i] : 0u;
                if (i < N) { I.lower_count[i] = 0; I.lower_cursor[i] = 0; }
            }
            for (uint32_t i = threadIdx.x; i < kLenBuckets; i += blockDim.x) I.len_bucket[i] = 0;
            __syncthreads();
            block_exclusive_scan_inplace(I.half_offset, N + 1, &total);
            __syncthreads();
            if (threadIdx.x == 0) {
                C->half_pairs = total;
                if (total > I.cap_pairs) atomicOr(&C->error_flags, kErrHalfPairCapacity);
            }
            break;
        }
        case kScanBlkRows: {
            for (uint32_t i = threadIdx.x; i <= N; i += blockDim.x)
                I.blkrow_offset[i] = i < N ? I.lower_count[i] + I.upper_count[i] : 0u;
            __syncthreads();
            block_exclusive_scan_inplace(I.blkrow_offset, N + 1, &total);
            // start of every entry-count bucket in pair_order (a cursor per bucket)
            if (threadIdx.x == 0) {
                uint32_t acc = 0;
                for (uint32_t b = 0; b < kLenBuckets; ++b) {
                    I.len_bucket[kLenBuckets + b] = acc;
                    acc += I.len_bucket[b];
                }
            }
            break;
        }
        case kScanBins: {
            const uint32_t nb = C->num_bins;
            __syncthreads();
            block_exclusive_scan_inplace(I.bin_scan, nb + 1, &total);
            __syncthreads();
            if (threadIdx.x == 0) {
                C->binblock_nnz = I.bin_scan[nb];
                if (I.bin_scan[nb] > I.cap_bb) atomicOr(&C->error_flags, kErrBinBlockCapacity);
            }
            break;
        }
        default: break;
    }
}

// The same grouping: the group's first lane reserves the group's slots and
// every lane takes its rank in the group (the sort that follows orders them).
__global__ void __launch_bounds__(256) n2t_scatter_kernel(const InstDesc* insts) {
    const InstDesc& I = insts[blockIdx.y];
    TermOffsets off;
    off.load(I.counts);
    const uint32_t T = off.o[4], lane = lane_id();
    const uint32_t K1 = I.counts->node2term_entries;
    if (K1 > I.cap_k1) return;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t tw = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); tw < T; tw += stride) {
        const uint32_t t = tw + lane;
        uint32_t a[4] = {0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu};
        if (t < T) {
            uint32_t k;
            const TermType ty = off.typed(t, k);
            const ushort4 n = term_nodes(I, ty, k);
            const uint32_t m = ty == kSmooth ? 2 : 4;
            const unsigned short v[4] = {n.x, n.y, n.z, n.w};
            for (uint32_t j = 0; j < m; ++j)
                if (v[j] < I.N) a[j] = v[j];
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const uint32_t grp = __match_any_sync(0xffffffffu, a[j]);
            const uint32_t leader = __ffs(grp) - 1;
            uint32_t base = 0;
            if (a[j] != 0xFFFFFFFFu && lane == leader) base = atomicAdd(&I.n2t_cursor[a[j]], (uint32_t)__popc(grp));
            base = __shfl_sync(0xffffffffu, base, leader);
            if (a[j] != 0xFFFFFFFFu)
                I.n2t_index[I.n2t_offset[a[j]] + base + __popc(grp & ((1u << lane) - 1u))] = t;
        }
    }
}

// Sort each node's term segment ascending, one warp per node, in registers:
// element i = 32 s + lane sits in slot s of a lane; a bitonic network over
// kSlots * 32 keys exchanges across lanes with shuffles (partner distance
// < 32) and inside a lane between slots otherwise. A launch takes the
// segments of (min_len, 32 kSlots] terms; three launches (8, 16, 32 slots)
// cover up to kWarpSortMax, and n2t_sort_kernel the longer ones.
constexpr uint32_t kWarpSortMax = 1024;

template <int kSlots>
__global__ void __launch_bounds__(256) n2t_warp_sort_kernel(const InstDesc* insts, uint32_t min_len) {
    constexpr int kWarpSortSlots = kSlots;
    constexpr uint32_t kMax = 32u * kSlots;
    const InstDesc& I = insts[blockIdx.y];
    if (I.counts->node2term_entries > I.cap_k1) return;
    const uint32_t lane = lane_id();
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    for (uint32_t node = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); node < I.N; node += warps) {
        const uint32_t b = I.n2t_offset[node], e = I.n2t_offset[node + 1];
        const uint32_t len = e - b;
        if (len <= min_len || len <= 1 || len > kMax) continue;
        if (len > I.cap_seg) {  // the segment exceeds max_terms_per_node
            if (lane == 0) set_error(I, kErrSegmentTooLong);
            continue;
        }
        uint32_t v[kWarpSortSlots];
#pragma unroll
        for (int sl = 0; sl < kWarpSortSlots; ++sl) {
            const uint32_t i = 32u * sl + lane;
            v[sl] = i < len ? I.n2t_index[b + i] : 0xFFFFFFFFu;
        }
#pragma unroll
        for (uint32_t k = 2; k <= kMax; k <<= 1) {
#pragma unroll
            for (uint32_t j = k >> 1; j > 0; j >>= 1) {
                if (j >= 32) {
                    const int sj = (int)(j >> 5);
#pragma unroll
                    for (int sl = 0; sl < kWarpSortSlots; ++sl) {
                        if (sl & sj) continue;
                        const uint32_t i = 32u * sl + lane;
                        const bool up = (i & k) == 0;
                        const uint32_t a = v[sl], c = v[sl | sj];
                        v[sl] = up ? min(a, c) : max(a, c);
                        v[sl | sj] = up ? max(a, c) : min(a, c);
                    }
                } else {
#pragma unroll
                    for (int sl = 0; sl < kWarpSortSlots; ++sl) {
                        const uint32_t i = 32u * sl + lane;
                        const uint32_t o = __shfl_xor_sync(0xffffffffu, v[sl], j);
                        const bool up = (i & k) == 0, lower = (i & j) == 0;
                        v[sl] = (up == lower) ? min(v[sl], o) : max(v[sl], o);
                    }
                }
            }
        }
#pragma unroll
        for (int sl = 0; sl < kWarpSortSlots; ++sl) {
            const uint32_t i = 32u * sl + lane;
            if (i < len) I.n2t_index[b + i] = v[sl];
        }
    }
}

// sort each node's term segment ascending (one CTA per node) for the
// segments longer than kWarpSortMax
__global__ void __launch_bounds__(256) n2t_sort_kernel(const InstDesc* insts) {
    extern __shared__ uint32_t s32[];
    const InstDesc& I = insts[blockIdx.y];
    if (I.counts->node2term_entries > I.cap_k1) return;
    for (uint32_t node = blockIdx.x; node < I.N; node += gridDim.x) {
        const uint32_t b = I.n2t_offset[node], e = I.n2t_offset[node + 1];
        const uint32_t len = e - b;
        if (len <= kWarpSortMax) continue;
        if (len > I.cap_seg) {
            if (threadIdx.x == 0) set_error(I, kErrSegmentTooLong);
            continue;
        }
        const uint32_t n2 = next_pow2(len);
        for (uint32_t i = threadIdx.x; i < n2; i += blockDim.x) s32[i] = i < len ? I.n2t_index[b + i] : 0xFFFFFFFFu;
        __syncthreads();
        block_bitonic_sort(s32, n2);
        for (uint32_t i = threadIdx.x; i < len; i += blockDim.x) I.n2t_index[b + i] = s32[i];
        __syncthreads();
    }
}

// ------------------------------------------------ node pair -> term -----
// Row i of the upper triangle holds the entries (j, t) for every term t of
// node i and every other node j > i of t: the reference's half-pair keys
// (computeKVNodePairKNN, NodePair2TermsIndex.cu:11-28; smooth pairs :71-81)
// grouped by their smaller node.

__device__ inline uint32_t upper_entries_of(const InstDesc& I, const TermOffsets& off, uint32_t node, uint32_t t,
                                            uint32_t js[4]) {
    uint32_t k;
    const TermType ty = off.typed(t, k);
    const ushort4 n = term_nodes(I, ty, k);
    uint32_t c = 0;
    if (ty == kSmooth) {
        // the smooth term contributes one pair (min, max) to the row of min
        const uint32_t a = n.x, b = n.y;
        if (a == node && b > node && b < I.N) js[c++] = b;
        else if (b == node && a > node && a < I.N) js[c++] = a;
        // a node listed twice in the same smooth term (a == b) gives no pair
        return c;
    }
    const unsigned short a[4] = {n.x, n.y, n.z, n.w};
    for (int q = 0; q < 4; ++q)
        if (a[q] > node && a[q] < I.N) js[c++] = a[q];
    return c;
}

// warp per node: number of upper entries of the row
__global__ void __launch_bounds__(256) np_row_count_kernel(const InstDesc* insts) {
    const InstDesc& I = insts[blockIdx.y];
    if (I.counts->node2term_entries > I.cap_k1) return;
    TermOffsets off;
    off.load(I.counts);
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    for (uint32_t node = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); node < I.N; node += warps) {
        const uint32_t b = I.n2t_offset[node], e = I.n2t_offset[node + 1];
        uint32_t c = 0;
        for (uint32_t p = b + lane_id(); p < e; p += 32) {
            uint32_t js[4];
            c += upper_entries_of(I, off, node, I.n2t_index[p], js);
        }
        c = warp_sum(c);
        if (lane_id() == 0) I.row_count[node] = c;
    }
}

// Warp per node: the row's (j, t) entries, j > node, in ascending (j, t) order
// without sorting. The node's term list is already ascending in t, so for
// each distinct partner j (ascending, found by a warp minimum) one sweep of
// the list emits the terms that contain j, in t order, and finds the next
// partner. The first kRowCache * 32 terms stay in registers (the term id and
// its partners, packed 16-bit), the next kRowSpill * 32 in shared memory;
// longer lists re-derive the rest each sweep. A
// term that lists a partner twice contributes two adjacent entries, like the
// duplicate keys of a sort. Writes np_index, the per-pair (key, start) of the
// row and upper_count.
constexpr int kRowCache = 8;

__device__ inline void unpack_partners(uint2 pk, uint32_t j[4]) {
    j[0] = pk.x & 0xFFFFu; j[1] = pk.x >> 16; j[2] = pk.y & 0xFFFFu; j[3] = pk.y >> 16;
}

// the term's partners above `node` packed as four 16-bit ids (0xFFFF = none)
__device__ inline uint2 packed_partners(const InstDesc& I, const TermOffsets& off, uint32_t node, uint32_t t) {
    uint32_t js[4];
    const uint32_t c = upper_entries_of(I, off, node, t, js);
    uint32_t v[4] = {0xFFFFu, 0xFFFFu, 0xFFFFu, 0xFFFFu};
    for (uint32_t q = 0; q < c; ++q) v[q] = js[q];
    return make_uint2(v[0] | (v[1] << 16), v[2] | (v[3] << 16));
}

// terms kRowCache * 32 .. kRowCache * 32 + kRowSpill * 32 of a node's list
// wait in shared memory (the same (term, partners) pairs), so that the sweeps
// re-read them without re-deriving their partners
constexpr int kRowSpill = 8;

__global__ void __launch_bounds__(256, 4) np_row_build_kernel(const InstDesc* insts) {
    __shared__ uint32_t s_t[8][kRowSpill * 32];
    __shared__ uint2 s_pk[8][kRowSpill * 32];
    const InstDesc& I = insts[blockIdx.y];
    const DeviceCounts* C = I.counts;
    if (C->node2term_entries > I.cap_k1 || C->nodepair_entries > I.cap_k2) return;
    TermOffsets off;
    off.load(I.counts);
    const uint32_t lane = lane_id(), w = threadIdx.x >> 5;
    const uint32_t lt_mask = (1u << lane) - 1u;
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    for (uint32_t node = blockIdx.x * (blockDim.x >> 5) + w; node < I.N; node += warps) {
        const uint32_t b0 = I.n2t_offset[node], b1 = I.n2t_offset[node + 1];
        const uint32_t out = I.row_offset[node], len = I.row_count[node];
        uint32_t ct[kRowCache];
        uint2 cj[kRowCache];
#pragma unroll
        for (int m = 0; m < kRowCache; ++m) {
            const uint32_t p = b0 + lane + 32u * m;
            ct[m] = p < b1 ? I.n2t_index[p] : kInvalid;
            cj[m] = p < b1 ? packed_partners(I, off, node, ct[m]) : make_uint2(0xFFFFFFFFu, 0xFFFFFFFFu);
        }
        // the spill slices in shared memory (entries past b1 hold no partners)
        const uint32_t spill0 = b0 + 32u * kRowCache;
        const uint32_t spill1 = min(b1, spill0 + 32u * kRowSpill);
        __syncwarp();
        const uint32_t nspill = spill1 > spill0 ? (spill1 - spill0 + 31u) / 32u : 0u;  // whole slices
        for (uint32_t q = lane; q < 32u * nspill; q += 32) {
            const uint32_t p = spill0 + q;
            const uint32_t t = p < b1 ? I.n2t_index[p] : kInvalid;
            s_t[w][q] = t;
            s_pk[w][q] = p < b1 ? packed_partners(I, off, node, t) : make_uint2(0xFFFFFFFFu, 0xFFFFFFFFu);
        }
        __syncwarp();
        // emit the slice's entries for partner j at out + pos; returns the
        // smallest partner above j seen in the slice
        auto slice = [&](uint32_t t, uint2 pk, uint32_t j, uint32_t& pos) -> uint32_t {
            uint32_t js[4];
            unpack_partners(pk, js);
            uint32_t mult = 0, nxt = 0xFFFFFFFFu;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                mult += js[q] == j ? 1u : 0u;
                if (js[q] != 0xFFFFu && js[q] > j) nxt = min(nxt, js[q]);
            }
            uint32_t pre, total;
            if (__any_sync(0xffffffffu, mult > 1)) {
                pre = mult;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const uint32_t v = __shfl_up_sync(0xffffffffu, pre, o);
                    if (lane >= (uint32_t)o) pre += v;
                }
                total = __shfl_sync(0xffffffffu, pre, 31);
                pre -= mult;
            } else {
                const uint32_t bal = __ballot_sync(0xffffffffu, mult != 0);
                pre = __popc(bal & lt_mask);
                total = __popc(bal);
            }
            for (uint32_t c = 0; c < mult; ++c)
                if (pos + pre + c < len) I.np_index[out + pos + pre + c] = t;
            pos += total;
            return nxt;
        };
        // first partner: the smallest id above node
        uint32_t j;
        {
            uint32_t mn = 0xFFFFFFFFu;
#pragma unroll
            for (int m = 0; m < kRowCache; ++m) {
                uint32_t js[4];
                unpack_partners(cj[m], js);
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    if (js[q] != 0xFFFFu) mn = min(mn, js[q]);
            }
            for (uint32_t p = b0 + 32u * kRowCache + lane; p < b1; p += 32) {
                uint32_t js[4];
                unpack_partners(p < spill1 ? s_pk[w][p - spill0] : packed_partners(I, off, node, I.n2t_index[p]), js);
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    if (js[q] != 0xFFFFu) mn = min(mn, js[q]);
            }
            j = warp_min_u32(mn);
        }
        uint32_t pos = 0, runs = 0;
        while (j != 0xFFFFFFFFu) {
            if (lane == 0 && pos < len) {
                I.tmp_key[out + runs] = node * I.enc + j;
                I.tmp_start[out + runs] = out + pos;
            }
            uint32_t nxt = 0xFFFFFFFFu;
#pragma unroll
            for (int m = 0; m < kRowCache; ++m) {
                if (b0 + 32u * m >= b1) break;  // warp-uniform
                nxt = min(nxt, slice(ct[m], cj[m], j, pos));
            }
            for (uint32_t base = b0 + 32u * kRowCache; base < b1; base += 32) {
                const uint32_t p = base + lane;
                uint32_t t;
                uint2 pk;
                if (base < spill1) {  // warp-uniform: a spilled slice
                    t = s_t[w][p - spill0];
                    pk = s_pk[w][p - spill0];
                } else {
                    t = p < b1 ? I.n2t_index[p] : kInvalid;
                    pk = p < b1 ? packed_partners(I, off, node, t) : make_uint2(0xFFFFFFFFu, 0xFFFFFFFFu);
                }
                nxt = min(nxt, slice(t, pk, j, pos));
            }
            ++runs;
            j = warp_min_u32(nxt);
        }
        if (lane == 0) I.upper_count[node] = runs;
    }
}

// warp per node: copy the row's unique pairs to the compact half-pair arrays
// and count the lower-triangle entries of each column
__global__ void __launch_bounds__(256) np_half_compact_kernel(const InstDesc* insts) {
    const InstDesc& I = insts[blockIdx.y];
    const DeviceCounts* C = I.counts;
    if (C->half_pairs > I.cap_pairs || C->nodepair_entries > I.cap_k2 || C->node2term_entries > I.cap_k1) return;
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    for (uint32_t node = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); node < I.N; node += warps) {
        const uint32_t nu = I.upper_count[node];
        const uint32_t ro = I.row_offset[node], re = I.row_offset[node + 1];
        const uint32_t h0 = I.half_offset[node];
        for (uint32_t u = lane_id(); u < nu; u += 32) {
            const uint32_t key = I.tmp_key[ro + u];
            const uint32_t start = I.tmp_start[ro + u];
            const uint32_t end = (u + 1 < nu) ? I.tmp_start[ro + u + 1] : re;
            I.half_key[h0 + u] = key;
            I.half_range[h0 + u] = make_uint2(start, end);
            atomicAdd(&I.lower_count[key % I.enc], 1u);
            atomicAdd(&I.len_bucket[len_bucket_of(end - start)], 1u);
        }
    }
}

// warp per node: place the row's upper entries and scatter its pairs into the
// lower part of each partner row (unordered there; sorted next)
__global__ void __launch_bounds__(256) np_sym_scatter_kernel(const InstDesc* insts) {
    const InstDesc& I = insts[blockIdx.y];
    const DeviceCounts* C = I.counts;
    if (C->half_pairs > I.cap_pairs || C->nodepair_entries > I.cap_k2 || C->node2term_entries > I.cap_k1) return;
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    for (uint32_t node = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); node < I.N; node += warps) {
        const uint32_t nu = I.upper_count[node];
        const uint32_t h0 = I.half_offset[node];
        const uint32_t up0 = I.blkrow_offset[node] + I.lower_count[node];
        for (uint32_t u = lane_id(); u < nu; u += 32) {
            const uint32_t h = h0 + u;
            const uint32_t key = I.half_key[h];
            const uint2 rg = I.half_range[h];
            const uint32_t s = up0 + u;
            I.sym_key[s] = key;
            I.sym_range[s] = rg;
            I.sym_half[s] = h;
            // the order in which the off-diagonal kernel takes the pairs; each
            // pair is summed by one thread, so the order leaves results unchanged
            I.pair_order[atomicAdd(&I.len_bucket[kLenBuckets + len_bucket_of(rg.y - rg.x)], 1u)] = h;
            const uint32_t j = key % I.enc;
            const uint32_t pos = I.blkrow_offset[j] + atomicAdd(&I.lower_cursor[j], 1u);
            I.sym_key[pos] = j * I.enc + node;
            I.sym_range[pos] = rg;
            I.sym_half[pos] = h;
        }
    }
}

// warp per row: sort the lower part by key (keys are unique) by ranking
__global__ void __launch_bounds__(128) np_lower_sort_kernel(const InstDesc* insts) {
    constexpr uint32_t kMaxLower = 256;
    __shared__ uint32_t sk[4][kMaxLower];
    __shared__ uint2 sr[4][kMaxLower];
    __shared__ uint32_t sh[4][kMaxLower];
    const InstDesc& I = insts[blockIdx.y];
    const DeviceCounts* C = I.counts;
    if (C->half_pairs > I.cap_pairs || C->nodepair_entries > I.cap_k2 || C->node2term_entries > I.cap_k1) return;
    const uint32_t w = threadIdx.x >> 5;
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    for (uint32_t node = blockIdx.x * (blockDim.x >> 5) + w; node < I.N; node += warps) {
        const uint32_t nl = I.lower_count[node];
        const uint32_t b = I.blkrow_offset[node];
        if (nl > kMaxLower) {
            if (lane_id() == 0) set_error(I, kErrRowTooLong);
            continue;
        }
        for (uint32_t i = lane_id(); i < nl; i += 32) {
            sk[w][i] = I.sym_key[b + i];
            sr[w][i] = I.sym_range[b + i];
            sh[w][i] = I.sym_half[b + i];
        }
        __syncwarp();
        for (uint32_t i = lane_id(); i < nl; i += 32) {
            const uint32_t key = sk[w][i];
            uint32_t rank = 0;
            for (uint32_t m = 0; m < nl; ++m) rank += sk[w][m] < key ? 1u : 0u;
            I.sym_key[b + rank] = key;
            I.sym_range[b + rank] = sr[w][i];
            I.sym_half[b + rank] = sh[w][i];
        }
        __syncwarp();
        // column and half-storage position of every entry of this block row:
        // the diagonal first, then the row's symmetric keys (lower part sorted
        // above, upper part written by np_sym_scatter_kernel); pair h sits in
        // row min(i, j) at h + min(i, j) + 1
        const uint32_t ne = I.blkrow_offset[node + 1] - b, mask = I.enc - 1;
        for (uint32_t i = lane_id(); i <= ne; i += 32) {
            uint32_t col = node, pos = I.half_offset[node] + node;
            if (i > 0) {
                col = I.sym_key[b + i - 1] & mask;
                pos = I.sym_half[b + i - 1] + min(node, col) + 1;
                if (col < node) pos |= kTransposedBlock;
            }
            I.bsr_ent[b + node + i] = make_uint2(pos, col);
        }
        __syncwarp();
    }
}

// --------------------------------------------------- bin-block CSR -------
// computeBinLengthKernel (NodePairRowColumnIndex.cu:64-119), multi-CTA: the
// bin width is 6 x the longest block row (diagonal included) among the block
// rows that the bin's 32 scalar rows touch
__global__ void __launch_bounds__(256) bin_length_kernel(const InstDesc* insts) {
    const InstDesc& I = insts[blockIdx.y];
    const uint32_t nb = (6 * I.N + 31) / 32;
    if (blockIdx.x == 0 && threadIdx.x == 0) I.counts->num_bins = nb;
    for (uint32_t b = blockIdx.x * blockDim.x + threadIdx.x; b <= nb; b += gridDim.x * blockDim.x) {
        if (b == nb) { I.bin_scan[b] = 0; continue; }
        const uint32_t r0 = 32 * b / 6;
        uint32_t r1 = (32 * b + 31) / 6;
        r1 = min(r1, I.N - 1);
        uint32_t mx = 0;
        for (uint32_t r = r0; r <= r1; ++r) mx = max(mx, 1 + I.blkrow_offset[r + 1] - I.blkrow_offset[r]);
        I.bin_scan[b] = 32 * 6 * mx;
    }
}

// computeBinBlockedCSRRowPtrKernel (NodePairRowColumnIndex.cu:122-132) and the
// 0xFF fill of the column array (:273-281)
__global__ void __launch_bounds__(256) bin_rowptr_kernel(const InstDesc* insts) {
    const InstDesc& I = insts[blockIdx.y];
    const DeviceCounts* C = I.counts;
    const uint32_t nb = C->num_bins;
    if (C->binblock_nnz > I.cap_bb) return;
    const uint32_t ncol = C->binblock_nnz / 6;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < 32 * (nb + 1); i += stride)
        I.bb_rowptr[i] = (int32_t)(i % 32 + I.bin_scan[i / 32]);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < ncol; i += stride) I.bb_colptr[i] = -1;
}

// computeBinBlockedCSRColPtrKernel (NodePairRowColumnIndex.cu:136-179)
__global__ void __launch_bounds__(256) bin_colptr_kernel(const InstDesc* insts) {
    const InstDesc& I = insts[blockIdx.y];
    const DeviceCounts* C = I.counts;
    if (C->binblock_nnz > I.cap_bb || C->half_pairs > I.cap_pairs) return;
    const uint32_t rows = 6 * I.N;
    for (uint32_t row = blockIdx.x * blockDim.x + threadIdx.x; row < rows; row += gridDim.x * blockDim.x) {
        const uint32_t br = row / 6, lane = row % 32;
        const uint32_t data = (uint32_t)(row % 32) + I.bin_scan[row / 32];
        uint32_t col = (data - lane) / 6 + lane;
        I.bb_colptr[col] = (int32_t)(6 * br);
        col += 32;
        for (uint32_t s = I.blkrow_offset[br]; s < I.blkrow_offset[br + 1]; ++s, col += 32)
            I.bb_colptr[col] = (int32_t)(6 * (I.sym_key[s] % I.enc));
    }
}

// ------------------------------------------------- per-entry weights -----
// The skinning weight of each index entry's node(s) in its term, recorded once
// per solve (the weights are inputs), so that the assembly kernels read one
// coalesced value per entry instead of the term's node and weight records.
// The values are those of weight_of (PreconditionerBlocked.cu:23-29).

// warp per node: n2t_w[p] for the node's terms
__global__ void __launch_bounds__(256) n2t_weight_kernel(const InstDesc* insts) {
    const InstDesc& I = insts[blockIdx.y];
    if (I.counts->node2term_entries > I.cap_k1) return;
    TermOffsets off;
    off.load(I.counts);
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    for (uint32_t node = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); node < I.N; node += warps) {
        const uint32_t b0 = I.n2t_offset[node], b1 = I.n2t_offset[node + 1];
        for (uint32_t p = b0 + lane_id(); p < b1; p += 32) {
            uint32_t k;
            const TermType ty = off.typed(I.n2t_index[p], k);
            I.n2t_w[p] = ty == kSmooth || ty == kInvalidTerm
                             ? 0.f
                             : weight_of(term_nodes(I, ty, k), term_weights(I, ty, k), node);
        }
    }
}

// warp per node i: np_w[p] = (w_i, w_j) for the terms of each pair (i, j),
// pair by pair, the lanes over the pair's entries
__global__ void __launch_bounds__(256) np_weight_kernel(const InstDesc* insts) {
    const InstDesc& I = insts[blockIdx.y];
    const DeviceCounts* C = I.counts;
    if (C->half_pairs > I.cap_pairs || C->nodepair_entries > I.cap_k2 || C->node2term_entries > I.cap_k1) return;
    TermOffsets off;
    off.load(C);
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    for (uint32_t ni = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); ni < I.N; ni += warps) {
        const uint32_t h0 = I.half_offset[ni], nu = I.upper_count[ni];
        for (uint32_t h = h0; h < h0 + nu; ++h) {
            const uint32_t nj = I.half_key[h] % I.enc;
            const uint2 rg = I.half_range[h];
            for (uint32_t p = rg.x + lane_id(); p < rg.y; p += 32) {
                uint32_t k;
                const TermType ty = off.typed(I.np_index[p], k);
                float2 w = make_float2(0.f, 0.f);
                if (ty != kSmooth && ty != kInvalidTerm) {
                    const ushort4 kn = term_nodes(I, ty, k);
                    const float4 w4 = term_weights(I, ty, k);
                    w = make_float2(weight_of(kn, w4, ni), weight_of(kn, w4, nj));
                }
                I.np_w[p] = w;
            }
        }
    }
}

// ------------------------------------------------------------ launch -----

static inline dim3 grid2(uint32_t x, uint32_t B) { return dim3(x ? x : 1, B); }

cudaError_t set_index_smem_limits(size_t seg_bytes) {
    return cudaFuncSetAttribute(n2t_sort_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)seg_bytes);
}

cudaError_t launch_build_index(const LaunchCfg& lc, InstDesc* d, cudaStream_t st) {
    const uint32_t B = lc.B;
    const uint32_t cpv = lc.chunks_per_view;
    const uint32_t spread = (uint32_t)lc.sm_count * 4;  // grid-stride kernels
    MVDR_LAUNCH(input_check_kernel, grid2(spread, B), 256, 0, st, d, lc.width, lc.height);
    // dense pixels
    MVDR_LAUNCH(compact_count_kernel<DensePred>, grid2(cpv * lc.max_views, B), 256, 0, st, d, lc.width, lc.height, cpv);
    MVDR_LAUNCH(compact_scan_kernel, grid2(1, B), 1024, 0, st, d, cpv, lc.max_views, 0);
    MVDR_LAUNCH(compact_write_kernel<DensePred>, grid2(cpv * lc.max_views, B), 256, 0, st, d, lc.width, lc.height, cpv, 0);
    // foreground pixels (the predicate is false when the term is off)
    MVDR_LAUNCH(compact_count_kernel<ForegroundPred>, grid2(cpv * lc.max_views, B), 256, 0, st, d, lc.width, lc.height, cpv);
    MVDR_LAUNCH(compact_scan_kernel, grid2(1, B), 1024, 0, st, d, cpv, lc.max_views, 1);
    MVDR_LAUNCH(compact_write_kernel<ForegroundPred>, grid2(cpv * lc.max_views, B), 256, 0, st, d, lc.width, lc.height, cpv, 1);
    MVDR_LAUNCH(prepare_pixels_kernel, grid2(spread, B), 256, 0, st, d, lc.precision == MVDR_PRECISION_MIXED);
    if (lc.max_tp) {
        MVDR_LAUNCH(feat_choose_kernel, grid2((lc.max_tp + 255) / 256, B), 256, 0, st, d);
        MVDR_LAUNCH(feat_compact_kernel, grid2(1, B), 1024, 0, st, d);
    }
    MVDR_LAUNCH(term_offsets_kernel, grid2(1, B), 32, 0, st, d);
    // node -> term
    MVDR_LAUNCH(n2t_count_kernel, grid2(spread, B), 256, 0, st, d);
    MVDR_LAUNCH(node_scan_kernel, grid2(1, B), 1024, 0, st, d, (int)kScanN2T);
    MVDR_LAUNCH(n2t_scatter_kernel, grid2(spread, B), 256, 0, st, d);
    MVDR_LAUNCH(n2t_warp_sort_kernel<8>, grid2((lc.max_nodes + 7) / 8, B), 256, 0, st, d, 0u);
    MVDR_LAUNCH(n2t_warp_sort_kernel<16>, grid2((lc.max_nodes + 7) / 8, B), 256, 0, st, d, 256u);
    MVDR_LAUNCH(n2t_warp_sort_kernel<32>, grid2((lc.max_nodes + 7) / 8, B), 256, 0, st, d, 512u);
    MVDR_LAUNCH(n2t_sort_kernel, grid2(min(lc.max_nodes, (uint32_t)lc.sm_count), B), 256, (size_t)lc.cap_seg * 4, st,
                d);
    // node pair -> term
    MVDR_LAUNCH(np_row_count_kernel, grid2((lc.max_nodes + 7) / 8, B), 256, 0, st, d);
    MVDR_LAUNCH(node_scan_kernel, grid2(1, B), 1024, 0, st, d, (int)kScanRows);
    MVDR_LAUNCH(np_row_build_kernel, grid2((lc.max_nodes + 7) / 8, B), 256, 0, st, d);
    MVDR_LAUNCH(node_scan_kernel, grid2(1, B), 1024, 0, st, d, (int)kScanUpper);
    MVDR_LAUNCH(np_half_compact_kernel, grid2((lc.max_nodes + 7) / 8, B), 256, 0, st, d);
    MVDR_LAUNCH(node_scan_kernel, grid2(1, B), 1024, 0, st, d, (int)kScanBlkRows);
    MVDR_LAUNCH(np_sym_scatter_kernel, grid2((lc.max_nodes + 7) / 8, B), 256, 0, st, d);
    MVDR_LAUNCH(np_lower_sort_kernel, grid2((lc.max_nodes + 3) / 4, B), 128, 0, st, d);
    MVDR_LAUNCH(n2t_weight_kernel, grid2((lc.max_nodes + 7) / 8, B), 256, 0, st, d);
    MVDR_LAUNCH(np_weight_kernel, grid2((lc.max_nodes + 7) / 8, B), 256, 0, st, d);
    // bin-block CSR structure
    MVDR_LAUNCH(bin_length_kernel, grid2((6 * lc.max_nodes / 32 + 256) / 256, B), 256, 0, st, d);
    MVDR_LAUNCH(node_scan_kernel, grid2(1, B), 1024, 0, st, d, (int)kScanBins);
    MVDR_LAUNCH(bin_rowptr_kernel, grid2(spread, B), 256, 0, st, d);
    MVDR_LAUNCH(bin_colptr_kernel, grid2((6 * lc.max_nodes + 255) / 256, B), 256, 0, st, d);
    return cudaGetLastError();
}

}  // namespace mvdr
