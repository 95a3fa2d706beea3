// Device helpers shared by the solver kernels: warp/block reductions and
// scans, shared-memory bitonic sort, term-type decoding and launch counting.
#pragma once

#include "mvdr_internal.cuh"

namespace mvdr {

#define MVDR_LAUNCH(kernel, grid, block, smem, stream, ...)      \
    do {                                                          \
        kernel<<<(grid), (block), (smem), (stream)>>>(__VA_ARGS__); \
        count_launch();                                           \
    } while (0)

__device__ inline uint32_t lane_id() { return threadIdx.x & 31u; }

template <class T> __device__ inline T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ inline uint32_t warp_max_u32(uint32_t v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

__device__ inline uint32_t warp_min_u32(uint32_t v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = min(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// inclusive warp scan
__device__ inline uint32_t warp_inclusive_scan(uint32_t v) {
    const uint32_t lane = lane_id();
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t n = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= (uint32_t)o) v += n;
    }
    return v;
}

// Reduce NV per-lane values across the warp with a shfl_down tree per value;
// after the call lane 0 holds the complete sums in v[0..NV). The order of the
// additions is fixed, so the result is reproducible run to run.
template <int NV, class T> __device__ inline void warp_reduce_to_lane0(T (&v)[NV]) {
#pragma unroll
    for (int i = 0; i < NV; ++i) {
        T x = v[i];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        v[i] = x;
    }
}

// Block-wide exclusive scan of a[0..n) in global memory, in place, by one CTA.
// Writes the total to *total (if not null). blockDim.x must be 1024.
__device__ inline void block_exclusive_scan_inplace(uint32_t* a, uint32_t n, uint32_t* total,
                                                    const uint32_t* add = nullptr) {
    __shared__ uint32_t warp_tot[32];
    __shared__ uint32_t carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const uint32_t tid = threadIdx.x;
    for (uint32_t base = 0; base < n; base += 1024u * 8u) {
        // each thread scans 8 consecutive items of this tile
        uint32_t v[8];
        uint32_t sum = 0;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const uint32_t i = base + tid * 8u + k;
            uint32_t x = 0;
            if (i < n) x = a[i] + (add ? add[i] : 0u);
            v[k] = sum;
            sum += x;
        }
        const uint32_t incl = warp_inclusive_scan(sum);
        if (lane_id() == 31) warp_tot[tid >> 5] = incl;
        __syncthreads();
        if (tid < 32) {
            const uint32_t w = warp_tot[tid];
            const uint32_t wi = warp_inclusive_scan(w);
            warp_tot[tid] = wi - w;
        }
        __syncthreads();
        const uint32_t off = carry + warp_tot[tid >> 5] + incl - sum;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const uint32_t i = base + tid * 8u + k;
            if (i < n) a[i] = off + v[k];
        }
        __syncthreads();
        if (tid == 1023) carry = off + sum;
        __syncthreads();
    }
    if (total && threadIdx.x == 0) *total = carry;
}

// In-place ascending bitonic sort of s[0..n2) in shared memory, n2 a power
// of two; the caller pads with the maximum key.
template <class K> __device__ inline void block_bitonic_sort(K* s, uint32_t n2) {
    for (uint32_t k = 2; k <= n2; k <<= 1) {
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            for (uint32_t i = threadIdx.x; i < n2; i += blockDim.x) {
                const uint32_t ixj = i ^ j;
                if (ixj > i) {
                    const K a = s[i], b = s[ixj];
                    const bool up = (i & k) == 0;
                    if ((a > b) == up) {
                        s[i] = b;
                        s[ixj] = a;
                    }
                }
            }
            __syncthreads();
        }
    }
}

__device__ inline uint32_t next_pow2(uint32_t v) {
    uint32_t p = 1;
    while (p < v) p <<= 1;
    return p;
}

// term types in the reference's prefix order (base/term_offset_types.h:11-18)
enum TermType : uint32_t { kDense = 0, kSmooth = 1, kForeground = 2, kFeature = 3, kCross = 4, kInvalidTerm = 5 };

struct TermOffsets {
    uint32_t o[5];
    __device__ inline void load(const DeviceCounts* c) {
#pragma unroll
        for (int i = 0; i < 5; ++i) o[i] = c->term_offset[i];
    }
    // query_typed_index (term_offset_types.h:66-99)
    __device__ inline TermType typed(uint32_t t, uint32_t& k) const {
        if (t < o[0]) { k = t; return kDense; }
        if (t < o[1]) { k = t - o[0]; return kSmooth; }
        if (t < o[2]) { k = t - o[1]; return kForeground; }
        if (t < o[3]) { k = t - o[2]; return kFeature; }
        if (t < o[4]) { k = t - o[3]; return kCross; }
        k = kInvalid;
        return kInvalidTerm;
    }
};

// The (up to) four nodes of a term; smooth terms have two (z = w = 0xFFFF).
__device__ inline ushort4 term_nodes(const InstDesc& I, TermType ty, uint32_t k) {
    switch (ty) {
        case kDense: return I.dense_knn[k];
        case kForeground: return I.fg_knn[k];
        case kFeature: return I.feat_knn[k];
        case kCross: return I.cross_knn[k];
        case kSmooth: {
            const ushort2 e = I.graph[k];
            return make_ushort4(e.x, e.y, 0xFFFF, 0xFFFF);
        }
        default: return make_ushort4(0xFFFF, 0xFFFF, 0xFFFF, 0xFFFF);
    }
}

__device__ inline float4 term_weights(const InstDesc& I, TermType ty, uint32_t k) {
    switch (ty) {
        case kDense: return I.dense_w[k];
        case kForeground: return I.fg_w[k];
        case kFeature: return I.feat_w[k];
        case kCross: return I.cross_w[k];
        default: return make_float4(1.f, 1.f, 0.f, 0.f);
    }
}

// weight of `node` among the term's four neighbours (the offset trick of
// PreconditionerBlocked.cu:23-29)
__device__ inline float weight_of(ushort4 knn, float4 w, uint32_t node) {
    const int o = 0 * (node == knn.x) + 1 * (node == knn.y) + 2 * (node == knn.z) + 3 * (node == knn.w);
    return o == 0 ? w.x : (o == 1 ? w.y : (o == 2 ? w.z : w.w));
}

__device__ inline void set_error(const InstDesc& I, uint32_t bit) { atomicOr(&I.counts->error_flags, bit); }

// Jt r and the PCG vectors in the arithmetic of the linear solve: float for
// FP32, double for mixed precision (where float rounding of the right-hand
// side or the vectors alone moves the increment of a 15k-node system by
// ~2e-4)
template <bool MIXED> struct PcgVec;
template <> struct PcgVec<true> {
    using T = double;
    __device__ static T* jtr(const InstDesc& I) { return I.jtr_d; }
    __device__ static T* x(const InstDesc& I) { return I.x_d; }
    __device__ static T* r(const InstDesc& I) { return I.r_d; }
    __device__ static T* s(const InstDesc& I) { return I.s_d; }
    __device__ static T* q(const InstDesc& I) { return I.q_d; }
    __device__ static T* d(const InstDesc& I, int odd) { return odd ? I.d1_d : I.d0_d; }
};
template <> struct PcgVec<false> {
    using T = float;
    __device__ static T* jtr(const InstDesc& I) { return I.jtr; }
    __device__ static T* x(const InstDesc& I) { return I.x; }
    __device__ static T* r(const InstDesc& I) { return I.r; }
    __device__ static T* s(const InstDesc& I) { return I.s; }
    __device__ static T* q(const InstDesc& I) { return I.q; }
    __device__ static T* d(const InstDesc& I, int odd) { return odd ? I.d1 : I.d0; }
};

// A(r, k) of entry e of the full block-row layout, read from the half storage
__device__ inline float stored_block_element(const InstDesc& I, uint32_t e, uint32_t r, uint32_t k) {
    const uint32_t pos = I.bsr_ent[e].x;
    const size_t blk = 36 * (size_t)(pos & ~kTransposedBlock);
    const uint32_t idx = (pos & kTransposedBlock) ? blk_idx(k, r) : blk_idx(r, k);
    return I.bsr_d ? (float)I.bsr_d[blk + idx] : I.bsr[blk + idx];
}

// true when this instance's index is complete: every count within its
// capacity and no segment or row skipped. Kernels that walk the block-row
// structure skip an instance whose index is not (its host call then reports
// the capacity error).
__device__ inline bool index_complete(const InstDesc& I) {
    const DeviceCounts* C = I.counts;
    constexpr uint32_t kIndexErrors = kErrNode2TermCapacity | kErrNodePairEntryCapacity | kErrHalfPairCapacity |
                                      kErrSegmentTooLong | kErrRowTooLong;
    return C->node2term_entries <= I.cap_k1 && C->nodepair_entries <= I.cap_k2 && C->half_pairs <= I.cap_pairs &&
           (*(volatile const uint32_t*)&C->error_flags & kIndexErrors) == 0;
}

// The 32-byte record (two float4) at p in one 256-bit load (p 32-byte aligned)
__device__ inline void load_record32(const float4* p, float4& a, float4& b) {
    asm volatile("ld.global.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                 : "=f"(a.x), "=f"(a.y), "=f"(a.z), "=f"(a.w), "=f"(b.x), "=f"(b.y), "=f"(b.z), "=f"(b.w)
                 : "l"(p));
}

// Eight floats at a 32-byte-aligned address in one 256-bit load
__device__ inline void load8f(const float* p, float (&v)[8]) {
    asm volatile("ld.global.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                 : "=f"(v[0]), "=f"(v[1]), "=f"(v[2]), "=f"(v[3]), "=f"(v[4]), "=f"(v[5]), "=f"(v[6]), "=f"(v[7])
                 : "l"(p));
}

// the float direction's position of vector element e (node e / 6, row e % 6)
__device__ inline size_t df_pos(size_t e) { return e + 2 * (e / 6); }

// true when the input check found an out-of-range node or surfel id
__device__ inline bool bad_inputs(const InstDesc& I) {
    return (*(volatile const uint32_t*)&I.counts->error_flags & kErrBadNodeIndex) != 0;
}

// __float2int_rn of the reference projection; the divide is double because
// the reference writes `z + 1e-10` with a double literal
__device__ inline int project_coord(float a, float z, float f, float c) {
    const double v = ((double)a / ((double)z + 1e-10)) * (double)f + (double)c;
    return __float2int_rn((float)v);
}

// compute_feature_huber_weight (huber_weight.h:11-27)
__device__ inline float huber_weight(float r) {
    const float a = fabsf(r);
    return a < 7.5e-2f ? 1.0f : 7.5e-2f / a;
}

}  // namespace mvdr
