// After the solve: moving surfels and nodes with the warp field, per-node
// alignment errors, and the correction of nodes with a large error.
//
//   forward_warp_kernel   SurfelNodeDeformer::ForwardWarpSurfelsAndNodes
//                         (core/Geometry/SurfelNodeDeformer.cu:9-57,131-206)
//   inverse_warp_kernel   SurfelNodeDeformer::InverseWarpSurfels
//                         (SurfelNodeDeformer.cu:63-119,229-318)
//   node_error_kernel     computeAlignmentErrorWindowSearch +
//                         computeAlignmentErrorMapKernel +
//                         computeNodeAlignmentErrorFromMapKernel
//                         (core/NonRigidSolver/DenseDepthAlignmentError.cu:16-179)
//   node_united_kernel    computeLargeErrorNodeNum (DenseDepthAlignmentError.cu:181-196)
//   node_error_map_kernel collectAlignmentErrorMapFromNodeKernel (:198-238)
//   guided_node_kernel    computeSuitableCorrespondenceGuidedSe3 +
//                         computeCorrespondenceGuidedNodesSE3
//                         (core/NonRigidSolver/NonRigidSolver.cu:93-166)
//   correct_kernel        CorrectWarpVertexAndNodeKernel (NonRigidSolver.cu:168-227)
//
// The node error sums are accumulated with 64-bit integer atomics in 2^-32
// fixed point: exact, so the sums do not depend on the order in which pixels
// add to a node (the reference's float atomics do). This file is compiled
// with -fmad=false and normalises with an IEEE 1/sqrt, so every float result
// equals the CPU restatement's, except those of the correction's quaternion
// power (atan2f, sinf, cosf).
#include <cstring>
#include <string>

#include "batch.cuh"
#include "kernels_common.cuh"

namespace mvdr {
namespace {

constexpr float kMaxAlignmentError = 0.1f;  // d_maximum_alignment_error (solver_constants.h:45)
constexpr int kAlignHalfWindow = 1;         // window_halfsize (DenseDepthAlignmentError.cu:11)
constexpr int kCorrHalfWindow = 2;          // CorrSearchWindowHalfSize (NonRigidSolver.h:41)
constexpr float kFixedOne = 4294967296.0f;  // 2^32: the node sums' fixed-point unit
constexpr double kFixedInv = 1.0 / 4294967296.0;

// ------------------------------------------------------------ quaternions ----
// float4 (x, y, z, w); products and sums in the reference's operation order
// (math/DualQuaternion/Quaternion.h:260-312)
__device__ inline float4 qmul(float4 a, float4 b) {
    float4 q;
    q.w = a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z;
    q.x = a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y;
    q.y = a.w * b.y - a.x * b.z + a.y * b.w + a.z * b.x;
    q.z = a.w * b.z + a.x * b.y - a.y * b.x + a.z * b.w;
    return q;
}
__device__ inline float4 qscale(float s, float4 q) { return make_float4(s * q.x, s * q.y, s * q.z, s * q.w); }
__device__ inline float4 qadd(float4 a, float4 b) { return make_float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }
__device__ inline float4 qconj(float4 q) { return make_float4(-q.x, -q.y, -q.z, q.w); }

__device__ inline DQ load_dq_any(const DQ* f, uint32_t i) {
    const float4* p = reinterpret_cast<const float4*>(f + i);
    DQ d;
    d.q0 = p[0];
    d.q1 = p[1];
    return d;
}

// averageDualQuaternion (DualQuaternion.h:381-393)
__device__ inline DQ blend(const DQ* f, ushort4 k, float4 w) {
    const DQ a = load_dq_any(f, k.x), b = load_dq_any(f, k.y), c = load_dq_any(f, k.z), d = load_dq_any(f, k.w);
    DQ o;
    o.q0 = qscale(w.x, a.q0);
    o.q1 = qscale(w.x, a.q1);
    o.q0 = qadd(o.q0, qscale(w.y, b.q0));
    o.q1 = qadd(o.q1, qscale(w.y, b.q1));
    o.q0 = qadd(o.q0, qscale(w.z, c.q0));
    o.q1 = qadd(o.q1, qscale(w.z, c.q1));
    o.q0 = qadd(o.q0, qscale(w.w, d.q0));
    o.q1 = qadd(o.q1, qscale(w.w, d.q1));
    return o;
}

// DualQuaternion::normalize (DualQuaternion.h:281-287) with an IEEE 1/sqrt
__device__ inline DQ normalized(DQ d) {
    const float inv = 1.0f / sqrtf(qdot(d.q0, d.q0));
    d.q0 = qscale(inv, d.q0);
    d.q1 = qscale(inv, d.q1);
    const float dd = qdot(d.q0, d.q1);
    d.q1 = make_float4(d.q1.x - dd * d.q0.x, d.q1.y - dd * d.q0.y, d.q1.z - dd * d.q0.z, d.q1.w - dd * d.q0.w);
    return d;
}

// DualQuaternion::se3_matrix (DualQuaternion.h:326-332) of an already
// normalised dual quaternion
__device__ inline M34 se3_of_normalized(const DQ& d) {
    M34 m;
    quat_rotation(d.q0, m.r);
    const float4 t = qmul(qscale(2.0f, d.q1), qconj(d.q0));
    m.t[0] = t.x;
    m.t[1] = t.y;
    m.t[2] = t.z;
    return m;
}

// mat34::operator* (MatUtils.h:449-455)
__device__ inline M34 mul34(const M34& a, const M34& b) {
    M34 o;
    for (int r = 0; r < 3; ++r) {
        for (int c = 0; c < 3; ++c)
            o.r[3 * r + c] = a.r[3 * r] * b.r[c] + a.r[3 * r + 1] * b.r[3 + c] + a.r[3 * r + 2] * b.r[6 + c];
        o.t[r] = (a.r[3 * r] * b.t[0] + a.r[3 * r + 1] * b.t[1] + a.r[3 * r + 2] * b.t[2]) + a.t[r];
    }
    return o;
}
// mat34::inverse (MatUtils.h:585-590)
__device__ inline M34 inverse34(const M34& a) {
    M34 o;
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) o.r[3 * r + c] = a.r[3 * c + r];
    for (int r = 0; r < 3; ++r) o.t[r] = -(o.r[3 * r] * a.t[0] + o.r[3 * r + 1] * a.t[1] + o.r[3 * r + 2] * a.t[2]);
    return o;
}

// DualQuaternion(const mat34&) (DualQuaternion.h:123-130) through
// Quaternion(const mat33&) (Quaternion.h:46-77)
__device__ inline DQ dq_from_mat34(const M34& a) {
    const float* m = a.r;
    float4 q;
    const float tr = m[0] + m[4] + m[8];
    if (tr > 0) {
        const float s = sqrtf(tr + 1.0f) * 2;
        q.w = s * 0.25f; q.x = (m[7] - m[5]) / s; q.y = (m[2] - m[6]) / s; q.z = (m[3] - m[1]) / s;
    } else if ((m[0] > m[4]) && (m[0] > m[8])) {
        const float s = sqrtf(1.0f + m[0] - m[4] - m[8]) * 2;
        q.w = (m[7] - m[5]) / s; q.x = 0.25f * s; q.y = (m[1] + m[3]) / s; q.z = (m[2] + m[6]) / s;
    } else if (m[4] > m[8]) {
        const float s = sqrtf(1.0f + m[4] - m[0] - m[8]) * 2;
        q.w = (m[2] - m[6]) / s; q.x = (m[1] + m[3]) / s; q.y = 0.25f * s; q.z = (m[5] + m[7]) / s;
    } else {
        const float s = sqrtf(1.0f + m[8] - m[0] - m[4]) * 2;
        q.w = (m[3] - m[1]) / s; q.x = (m[2] + m[6]) / s; q.y = (m[5] + m[7]) / s; q.z = 0.25f * s;
    }
    DQ d;
    d.q0 = q;
    d.q1 = qmul(make_float4(0.5f * a.t[0], 0.5f * a.t[1], 0.5f * a.t[2], 0.0f), q);
    return d;
}

// DualQuaternion::operator*(float) (DualQuaternion.h:165-177): the
// screw motion scaled by t in [1e-10, 1], via Quaternion::pow
// (Quaternion.h:235-249)
__device__ inline DQ dq_pow_scale(const DQ& d, float ratio) {
    float t = ratio;
    if (t > 1.0f) t = 1.0f;
    else if (t < 1e-10f) t = 1e-10f;
    const float4 q0 = d.q0;
    const float norm = sqrtf(q0.x * q0.x + q0.y * q0.y + q0.z * q0.z);
    const float theta = atan2f(norm, q0.w);
    const float nt = theta * t;
    const float sn = sinf(nt);
    float4 p;
    if (fabsf(norm) < 1e-6f) {
        p = make_float4(0.0f, 0.0f, 0.0f, cosf(nt));
    } else {
        const float scale = sn / norm;
        p = make_float4(q0.x * scale, q0.y * scale, q0.z * scale, cosf(nt));
    }
    DQ o;
    o.q0 = p;
    o.q1 = qmul(qscale(t, qmul(d.q1, qconj(q0))), p);
    return o;
}

// mvdr_mat34 (the reference's mat34: rotation columns, then translation) to
// the row-major M34
__device__ inline M34 load_mat34(const mvdr_mat34* p) {
    const float4* q = reinterpret_cast<const float4*>(p);
    const float4 a = q[0], b = q[1], c = q[2];
    const float f[12] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w, c.x, c.y, c.z, c.w};
    M34 m;
    for (int r = 0; r < 3; ++r)
        for (int col = 0; col < 3; ++col) m.r[3 * r + col] = f[3 * col + r];
    m.t[0] = f[9];
    m.t[1] = f[10];
    m.t[2] = f[11];
    return m;
}

__device__ inline DQ identity_dq() {
    DQ d;
    d.q0 = make_float4(0.f, 0.f, 0.f, 1.f);
    d.q1 = make_float4(0.f, 0.f, 0.f, 0.f);
    return d;
}

__device__ inline float3 xyz(float4 v) { return make_float3(v.x, v.y, v.z); }
__device__ inline bool knn_ok(ushort4 k, uint32_t n) { return k.x < n && k.y < n && k.z < n && k.w < n; }
constexpr float kNaN = __builtin_nanf("");

// ----------------------------------------------------------- warp kernels ----

struct WarpArgs {
    const DQ* field;
    uint32_t num_field;
    // surfels
    uint32_t S;
    const ushort4* knn;
    const float4* w;
    const float4* in_v;
    const float4* in_n;
    float4* out_v;
    float4* out_n;
    // nodes (forward only)
    uint32_t N;
    const ushort4* node_knn;
    const float4* node_w;
    const float4* nodes;
    float4* live_nodes;
    // inverse only
    const mvdr_mat34* correct;
};

__global__ void __launch_bounds__(256) forward_warp_kernel(const __grid_constant__ WarpArgs a) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.S + a.N) return;
    const bool surfel = i < a.S;
    const uint32_t k = surfel ? i : i - a.S;
    const ushort4 knn = surfel ? a.knn[k] : a.node_knn[k];
    const float4 w = surfel ? a.w[k] : a.node_w[k];
    const float4 v = surfel ? a.in_v[k] : a.nodes[k];
    const float4 n = surfel ? a.in_n[k] : make_float4(0.f, 0.f, 0.f, 0.f);
    float4 ov, on;
    if (knn_ok(knn, a.num_field)) {
        const M34 se3 = se3_of_normalized(normalized(blend(a.field, knn, w)));
        const float3 p = apply3(se3, xyz(v)), q = rot3(se3, xyz(n));
        ov = make_float4(p.x, p.y, p.z, v.w);
        on = make_float4(q.x, q.y, q.z, n.w);
    } else {
        ov = make_float4(kNaN, kNaN, kNaN, v.w);
        on = make_float4(kNaN, kNaN, kNaN, n.w);
    }
    if (surfel) {
        a.out_v[k] = ov;
        a.out_n[k] = on;
    } else {
        a.live_nodes[k] = ov;
    }
}

__global__ void __launch_bounds__(256) inverse_warp_kernel(const __grid_constant__ WarpArgs a) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.S) return;
    const ushort4 knn = a.knn[i];
    const float4 v = a.in_v[i], n = a.in_n[i];
    float3 p = make_float3(kNaN, kNaN, kNaN), q = p;
    if (knn_ok(knn, a.num_field)) {
        const M34 se3 = se3_of_normalized(normalized(blend(a.field, knn, a.w[i])));
        // apply_inversed_se3: R^T (v - t)
        p = rotT3(se3, make_float3(v.x - se3.t[0], v.y - se3.t[1], v.z - se3.t[2]));
        q = rotT3(se3, xyz(n));
        if (a.correct) {
            const M34 ci = inverse34(load_mat34(a.correct + i));
            p = apply3(ci, p);
            q = rot3(ci, q);
        }
    }
    a.out_v[i] = make_float4(p.x, p.y, p.z, v.w);
    a.out_n[i] = make_float4(q.x, q.y, q.z, n.w);
}

// ------------------------------------------------------------ node error ----

struct NodeErrArgs {
    unsigned long long* acc;  // [2N]: error sums, then weight sums (fixed point)
    float* align_map[MVDR_MAX_VIEWS];
    float* node_map[MVDR_MAX_VIEWS];
    float* acc_error;
    float* acc_weight;
    float* united;
    uint32_t* mark;
    float threshold;
};

// border addressing: outside the image a map reads as zero (the reference's
// textures use cudaAddressModeBorder)
__device__ inline float4 tex4(const float4* m, int x, int y, uint32_t W, uint32_t H, uint32_t pitch) {
    if (x < 0 || y < 0 || x >= (int)W || y >= (int)H) return make_float4(0.f, 0.f, 0.f, 0.f);
    return m[(size_t)y * pitch + x];
}

// is_zero_vertex (VectorUtils.h:214-216): the 1e-3 bound is a double
__device__ inline bool zero_vertex(float4 v) {
    return (double)fabsf(v.x) < 1e-3 && (double)fabsf(v.y) < 1e-3 && (double)fabsf(v.z) < 1e-3;
}

// computeAlignmentErrorWindowSearch: the pixel's alignment error, 0 when no
// surfel is rendered there; knn/weight receive the pixel's skinning
__device__ float pixel_alignment_error(const InstDesc& I, const ViewDesc& V, uint32_t x, uint32_t y, ushort4& knn,
                                       float4& weight) {
    const size_t o = (size_t)y * V.pitch + x;
    const uint32_t s = V.index[o];
    if (s == kInvalid || s >= I.S) return 0.0f;
    knn = I.surfel_knn[s];
    weight = I.surfel_w[s];
    if (!knn_ok(knn, I.N)) return 0.0f;
    const float4 rv = V.ref_v[o], rn = V.ref_n[o];
    const float3 cv = apply3(V.init, xyz(rv)), cn = rot3(V.init, xyz(rn));
    const M34 se3 = se3_of_normalized(normalized(blend(I.se3, knn, weight)));
    const float3 wv = apply3(se3, cv), wn = rot3(se3, cn);
    const float3 c1 = apply3(V.init_inv, apply3(V.w2c, wv));
    const float3 n1 = rot3(V.init_inv, rot3(V.w2c, wn));
    const int W = (int)I.width, H = (int)I.height;
    // __float2int_rn saturates (NaN -> 0); a projection further than one
    // window outside the image reads only border zeros either way, so it is
    // clamped there to keep the window loop bounded
    int ix = project_coord(c1.x, c1.z, V.fx, V.cx), iy = project_coord(c1.y, c1.z, V.fy, V.cy);
    ix = min(max(ix, -2), W + 1);
    iy = min(max(iy, -2), H + 1);
    float err = kMaxAlignmentError;
    bool found = false;
    for (int dy = iy - kAlignHalfWindow; dy <= iy + kAlignHalfWindow; ++dy) {
        for (int dx = ix - kAlignHalfWindow; dx <= ix + kAlignHalfWindow; ++dx) {
            const float4 dv = tex4(V.obs_v, dx, dy, W, H, V.pitch);
            const float4 dn = tex4(V.obs_n, dx, dy, W, H, V.pitch);
            if (!zero_vertex(dv) && (n1.x * dn.x + n1.y * dn.y + n1.z * dn.z) > 0.7f) found = true;
            const float e = fabsf(c1.x - dv.x) + fabsf(c1.y - dv.y) + fabsf(c1.z - dv.z);
            if (e < err) err = e;
        }
    }
    if (!found) {
        float fg = 0.0f;
        if (V.fg && ix >= 0 && iy >= 0 && ix < W && iy < H) fg = V.fg[(size_t)iy * V.pitch + ix];
        err = fg < 0.9f ? 0.03f * fg : kMaxAlignmentError;
    }
    return err;
}

// v in 2^-32 units, rounded to nearest even; NaN counts as 0 and the range
// is clamped to +-2^62 so that the conversion is defined
__device__ inline unsigned long long to_fixed(float v) {
    float s = v * kFixedOne;
    if (!(s == s)) s = 0.0f;
    s = fminf(fmaxf(s, -4.611686e18f), 4.611686e18f);
    return (unsigned long long)__float2ll_rn(s);
}

__global__ void __launch_bounds__(256) node_error_kernel(const InstDesc* __restrict__ insts, uint32_t inst,
                                                         const __grid_constant__ NodeErrArgs a) {
    const InstDesc& I = insts[inst];
    const uint32_t v = blockIdx.y;
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= I.width * I.height) return;
    const uint32_t x = p % I.width, y = p / I.width;
    ushort4 knn = make_ushort4(0, 0, 0, 0);
    float4 w = make_float4(0.f, 0.f, 0.f, 0.f);
    const float err = pixel_alignment_error(I, I.views[v], x, y, knn, w);
    if (a.align_map[v]) a.align_map[v][p] = err;
    if (err > 1e-6f) {
        const uint32_t N = I.N;
        const uint16_t nk[4] = {knn.x, knn.y, knn.z, knn.w};
        const float wk[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            atomicAdd(a.acc + nk[k], to_fixed(wk[k] * err));
            atomicAdd(a.acc + N + nk[k], to_fixed(wk[k]));
        }
    }
}

__global__ void __launch_bounds__(256) node_united_kernel(const InstDesc* __restrict__ insts, uint32_t inst,
                                                          const __grid_constant__ NodeErrArgs a) {
    const InstDesc& I = insts[inst];
    const uint32_t n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= I.N) return;
    const float e = (float)((double)(long long)a.acc[n] * kFixedInv);
    const float w = (float)((double)(long long)a.acc[I.N + n] * kFixedInv);
    float u = (e / (w + 1e-4f)) / kMaxAlignmentError;
    uint32_t mark = u > a.threshold ? 1u : 0u;
    if (e < 1e-10f) {  // no rendered pixel with an error: treated as large
        mark = 1u;
        u = 1.0f;
    }
    a.acc_error[n] = e;
    a.acc_weight[n] = w;
    a.united[n] = u;
    a.mark[n] = mark;
}

__global__ void __launch_bounds__(256) node_error_map_kernel(const InstDesc* __restrict__ insts, uint32_t inst,
                                                             const __grid_constant__ NodeErrArgs a) {
    const InstDesc& I = insts[inst];
    const uint32_t v = blockIdx.y;
    float* out = a.node_map[v];
    if (!out) return;
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= I.width * I.height) return;
    const ViewDesc& V = I.views[v];
    const uint32_t x = p % I.width, y = p / I.width;
    const uint32_t s = V.index[(size_t)y * V.pitch + x];
    float f = 0.0f;
    if (s != kInvalid && s < I.S) {
        const ushort4 knn = I.surfel_knn[s];
        const float4 w = I.surfel_w[s];
        if (knn_ok(knn, I.N)) {
            const uint16_t nk[4] = {knn.x, knn.y, knn.z, knn.w};
            const float wk[4] = {w.x, w.y, w.z, w.w};
            float ae = 0.0f, aw = 0.0f;
            for (int k = 0; k < 4; ++k) {
                const float unit = a.acc_error[nk[k]] / a.acc_weight[nk[k]];
                ae += unit * wk[k];
                aw += wk[k];
            }
            f = ae / (aw + 1e-4f);
        }
    }
    out[p] = f;
}

// ------------------------------------------------------------- correction ----

struct CorrArgs {
    const mvdr_mat34* se3_map[MVDR_MAX_VIEWS];
    const uint8_t* valid[MVDR_MAX_VIEWS];
    const float4* prev[MVDR_MAX_VIEWS];
    uint32_t pitch[MVDR_MAX_VIEWS];
    uint32_t cols, rows;
    const float* united;
    float threshold;
    float four_radius_sq;  // 4 NODE_RADIUS^2
    DQ* field;             // corrected in place
    float4* live_nodes;
    const ushort4* node_knn;
    const float4* node_w;
    uint32_t S;
    float4* live_v;
    float4* live_n;
    const ushort4* surfel_knn;
    const float4* surfel_w;
    DQ* correction;
};

// decodeNodesCameraView (base/CommonUtils.h:111-118): the view i with
// i < w <= i + 1, or none
__device__ inline int node_view(float w, uint32_t views) {
    for (uint32_t i = 0; i < views; ++i)
        if ((float)i < w && w <= (float)(i + 1)) return (int)i;
    return -1;
}

__device__ inline float sqdist(float3 a, float3 b) {
    return (a.x - b.x) * (a.x - b.x) + (a.y - b.y) * (a.y - b.y) + (a.z - b.z) * (a.z - b.z);
}

// computeSuitableCorrespondenceGuidedSe3 (NonRigidSolver.cu:93-139)
__device__ M34 guided_se3(const InstDesc& I, const CorrArgs& a, int view, float4 node) {
    const ViewDesc& V = I.views[view];
    const float3 c = apply3(V.init_inv, apply3(V.w2c, xyz(node)));
    // __float2uint_rn of the same double expression as the pixel projection
    const double vx = ((double)c.x / ((double)c.z + 1e-10)) * (double)V.fx + (double)V.cx;
    const double vy = ((double)c.y / ((double)c.z + 1e-10)) * (double)V.fy + (double)V.cy;
    const uint32_t ux = __float2uint_rn((float)vx), uy = __float2uint_rn((float)vy);
    M34 s;
    for (int k = 0; k < 9; ++k) s.r[k] = (k % 4 == 0) ? 1.0f : 0.0f;
    s.t[0] = s.t[1] = s.t[2] = 0.0f;
    const uint32_t h = kCorrHalfWindow;
    if (ux >= a.cols - h || ux < h || uy >= a.rows - h || uy < h) return s;
    float best = 1e6f;
    const uint32_t pitch = a.pitch[view];
    for (uint32_t i = ux - h; i <= ux + h; ++i) {
        for (uint32_t j = uy - h; j <= uy + h; ++j) {
            const size_t o = (size_t)j * pitch + i;
            const float4 pv = a.prev[view][o];
            if (a.valid[view][o] == 1 && !zero_vertex(pv)) {
                const M34 g = load_mat34(a.se3_map[view] + o);
                const float d = sqdist(c, xyz(pv));
                const float3 moved = apply3(g, c);
                if (best > d && d < 1e-4f && sqdist(moved, c) < a.four_radius_sq) {
                    best = d;
                    s = g;
                }
            }
        }
    }
    // back to frame 0: world2camera^-1 * initialSE3 * s * initialSE3^-1 * world2camera
    return mul34(mul34(mul34(mul34(inverse34(V.w2c), V.init), s), V.init_inv), V.w2c);
}

__global__ void __launch_bounds__(128) guided_node_kernel(const InstDesc* __restrict__ insts, uint32_t inst,
                                                          const __grid_constant__ CorrArgs a) {
    const InstDesc& I = insts[inst];
    const uint32_t n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= I.N) return;
    const float err = a.united[n];
    DQ d = identity_dq();
    if (err > a.threshold) {
        const float4 node = a.live_nodes[n];
        const int view = node_view(node.w, I.num_views);
        if (view >= 0) d = dq_pow_scale(dq_from_mat34(guided_se3(I, a, view, node)), err);
    }
    float4* out = reinterpret_cast<float4*>(a.correction + n);
    out[0] = d.q0;
    out[1] = d.q1;
}

__global__ void __launch_bounds__(128) correct_kernel(const InstDesc* __restrict__ insts, uint32_t inst,
                                                      const __grid_constant__ CorrArgs a) {
    const InstDesc& I = insts[inst];
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.S + I.N) return;
    const bool surfel = i < a.S;
    const uint32_t k = surfel ? i : i - a.S;
    const ushort4 knn = surfel ? a.surfel_knn[k] : a.node_knn[k];
    const float4 w = surfel ? a.surfel_w[k] : a.node_w[k];
    const float4 v = surfel ? a.live_v[k] : a.live_nodes[k];
    const float4 nrm = surfel ? a.live_n[k] : make_float4(0.f, 0.f, 0.f, 0.f);
    float4 ov = make_float4(kNaN, kNaN, kNaN, v.w), on = make_float4(kNaN, kNaN, kNaN, nrm.w);
    DQ avg;
    const bool ok = knn_ok(knn, I.N);
    if (ok) {
        // se3_matrix normalises the blend in place; the node update uses it
        avg = normalized(blend(a.correction, knn, w));
        const M34 se3 = se3_of_normalized(avg);
        const float3 p = apply3(se3, xyz(v)), q = rot3(se3, xyz(nrm));
        ov = make_float4(p.x, p.y, p.z, v.w);
        on = make_float4(q.x, q.y, q.z, nrm.w);
    }
    if (surfel) {
        a.live_v[k] = ov;
        a.live_n[k] = on;
        return;
    }
    a.live_nodes[k] = ov;
    float4* f = reinterpret_cast<float4*>(a.field + k);
    if (!ok) {
        f[0] = make_float4(kNaN, kNaN, kNaN, kNaN);
        f[1] = f[0];
        return;
    }
    // DualQuaternion::operator* (DualQuaternion.h:152-157): avg * field
    const float4 f0 = f[0], f1 = f[1];
    f[0] = qmul(avg.q0, f0);
    f[1] = qadd(qmul(avg.q1, f0), qmul(avg.q0, f1));
}

bool aligned16(const void* p) { return ((uintptr_t)p & 15u) == 0; }

int check_surfels(const mvdr_deform_surfels* s, const char* fn) {
    if (!s) return fail(MVDR_EINVAL, std::string(fn) + ": null surfels");
    if (s->num_surfels == 0) return MVDR_OK;
    if (!s->knn || !s->knn_weight || !s->in_vertex || !s->in_normal || !s->out_vertex || !s->out_normal)
        return fail(MVDR_EINVAL, std::string(fn) + ": missing surfel array");
    if (!aligned16(s->knn_weight) || !aligned16(s->in_vertex) || !aligned16(s->in_normal) ||
        !aligned16(s->out_vertex) || !aligned16(s->out_normal) || ((uintptr_t)s->knn & 7u))
        return fail(MVDR_EINVAL, std::string(fn) + ": surfel arrays must be 16-byte aligned (knn 8-byte)");
    return MVDR_OK;
}

int launch_error(const char* fn) {
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(MVDR_ECUDA, std::string(fn) + ": " + cudaGetErrorString(e));
    return MVDR_OK;
}

int solver_state(mvdr_solver* s, const char* fn, Batch** b, InstDesc** I) {
    if (!s || !s->batch) return fail(MVDR_EINVAL, std::string(fn) + ": null solver");
    if (!s->batch->has_inputs[s->inst]) return fail(MVDR_ESTATE, std::string(fn) + ": inputs not set");
    *b = s->batch;
    *I = &s->batch->host[s->inst];
    return MVDR_OK;
}

}  // namespace
}  // namespace mvdr

using namespace mvdr;

extern "C" int mvdr_forward_warp(const mvdr_dual_quaternion* node_se3, uint32_t num_node_se3,
                                 const mvdr_deform_surfels* surfels, const mvdr_deform_nodes* nodes, void* stream) {
    const char* fn = "mvdr_forward_warp";
    if (int st = check_surfels(surfels, fn)) return st;
    if (!node_se3 || num_node_se3 == 0 || !aligned16(node_se3))
        return fail(MVDR_EINVAL, "mvdr_forward_warp: node_se3 must be a non-empty 16-byte aligned array");
    WarpArgs a;
    std::memset(&a, 0, sizeof(a));
    a.field = reinterpret_cast<const DQ*>(node_se3);
    a.num_field = num_node_se3;
    a.S = surfels->num_surfels;
    a.knn = reinterpret_cast<const ushort4*>(surfels->knn);
    a.w = reinterpret_cast<const float4*>(surfels->knn_weight);
    a.in_v = reinterpret_cast<const float4*>(surfels->in_vertex);
    a.in_n = reinterpret_cast<const float4*>(surfels->in_normal);
    a.out_v = reinterpret_cast<float4*>(surfels->out_vertex);
    a.out_n = reinterpret_cast<float4*>(surfels->out_normal);
    if (nodes && nodes->num_nodes) {
        if (!nodes->knn || !nodes->knn_weight || !nodes->canonical_nodes || !nodes->live_nodes)
            return fail(MVDR_EINVAL, "mvdr_forward_warp: missing node array");
        if (!aligned16(nodes->knn_weight) || !aligned16(nodes->canonical_nodes) || !aligned16(nodes->live_nodes) ||
            ((uintptr_t)nodes->knn & 7u))
            return fail(MVDR_EINVAL, "mvdr_forward_warp: node arrays must be 16-byte aligned (knn 8-byte)");
        a.N = nodes->num_nodes;
        a.node_knn = reinterpret_cast<const ushort4*>(nodes->knn);
        a.node_w = reinterpret_cast<const float4*>(nodes->knn_weight);
        a.nodes = reinterpret_cast<const float4*>(nodes->canonical_nodes);
        a.live_nodes = reinterpret_cast<float4*>(nodes->live_nodes);
    }
    const uint64_t total = (uint64_t)a.S + a.N;
    if (total == 0) return MVDR_OK;
    if (total > 0xFFFFFFFFull - 256) return fail(MVDR_ECAPACITY, "mvdr_forward_warp: too many points");
    MVDR_LAUNCH(forward_warp_kernel, dim3((uint32_t)((total + 255) / 256)), 256, 0, (cudaStream_t)stream, a);
    return launch_error(fn);
}

extern "C" int mvdr_inverse_warp(const mvdr_dual_quaternion* node_se3, uint32_t num_node_se3,
                                 const mvdr_mat34* correct_se3, const mvdr_deform_surfels* surfels, void* stream) {
    const char* fn = "mvdr_inverse_warp";
    if (int st = check_surfels(surfels, fn)) return st;
    if (!node_se3 || num_node_se3 == 0 || !aligned16(node_se3))
        return fail(MVDR_EINVAL, "mvdr_inverse_warp: node_se3 must be a non-empty 16-byte aligned array");
    if (correct_se3 && !aligned16(correct_se3))
        return fail(MVDR_EINVAL, "mvdr_inverse_warp: correct_se3 must be 16-byte aligned");
    if (surfels->num_surfels == 0) return MVDR_OK;
    WarpArgs a;
    std::memset(&a, 0, sizeof(a));
    a.field = reinterpret_cast<const DQ*>(node_se3);
    a.num_field = num_node_se3;
    a.S = surfels->num_surfels;
    a.knn = reinterpret_cast<const ushort4*>(surfels->knn);
    a.w = reinterpret_cast<const float4*>(surfels->knn_weight);
    a.in_v = reinterpret_cast<const float4*>(surfels->in_vertex);
    a.in_n = reinterpret_cast<const float4*>(surfels->in_normal);
    a.out_v = reinterpret_cast<float4*>(surfels->out_vertex);
    a.out_n = reinterpret_cast<float4*>(surfels->out_normal);
    a.correct = correct_se3;
    MVDR_LAUNCH(inverse_warp_kernel, dim3((a.S + 255) / 256), 256, 0, (cudaStream_t)stream, a);
    return launch_error(fn);
}

extern "C" int mvdr_compute_node_error(mvdr_solver* solver, const mvdr_node_error* out, void* stream) {
    const char* fn = "mvdr_compute_node_error";
    Batch* b = nullptr;
    InstDesc* I = nullptr;
    if (int st = solver_state(solver, fn, &b, &I)) return st;
    if (!out || !out->accumulated_error || !out->accumulated_weight || !out->united_error || !out->large_error_mark)
        return fail(MVDR_EINVAL, "mvdr_compute_node_error: missing output array");
    for (uint32_t v = I->num_views; v < MVDR_MAX_VIEWS; ++v)
        if (out->alignment_error_map[v] || out->node_error_map[v])
            return fail(MVDR_EINVAL, "mvdr_compute_node_error: a map is given for a view that is not bound");
    for (uint32_t v = 0; v < I->num_views; ++v)
        if (!I->views[v].fg)
            return fail(MVDR_EINVAL, "mvdr_compute_node_error: every view needs its filtered foreground mask");
    const cudaStream_t st = (cudaStream_t)stream;
    NodeErrArgs a;
    std::memset(&a, 0, sizeof(a));
    a.acc = I->node_err_acc;
    for (uint32_t v = 0; v < I->num_views; ++v) {
        a.align_map[v] = out->alignment_error_map[v];
        a.node_map[v] = out->node_error_map[v];
    }
    a.acc_error = out->accumulated_error;
    a.acc_weight = out->accumulated_weight;
    a.united = out->united_error;
    a.mark = out->large_error_mark;
    a.threshold = out->threshold;
    cudaError_t e = cudaMemsetAsync(a.acc, 0, 2 * sizeof(unsigned long long) * I->N, st);
    if (e != cudaSuccess) return fail(MVDR_ECUDA, std::string(fn) + ": " + cudaGetErrorString(e));
    const InstDesc* d_inst = b->d_inst;
    const uint32_t inst = solver->inst;
    const uint32_t npix = I->width * I->height;
    MVDR_LAUNCH(node_error_kernel, dim3((npix + 255) / 256, I->num_views), 256, 0, st, d_inst, inst, a);
    MVDR_LAUNCH(node_united_kernel, dim3((I->N + 255) / 256), 256, 0, st, d_inst, inst, a);
    bool maps = false;
    for (uint32_t v = 0; v < I->num_views; ++v) maps |= a.node_map[v] != nullptr;
    if (maps) MVDR_LAUNCH(node_error_map_kernel, dim3((npix + 255) / 256, I->num_views), 256, 0, st, d_inst, inst, a);
    return launch_error(fn);
}

extern "C" int mvdr_correct_large_error_nodes(mvdr_solver* solver, const mvdr_correction* c, void* stream) {
    const char* fn = "mvdr_correct_large_error_nodes";
    Batch* b = nullptr;
    InstDesc* I = nullptr;
    if (int st = solver_state(solver, fn, &b, &I)) return st;
    if (!c || !c->united_error || !c->live_nodes || !c->node_knn || !c->node_knn_weight || !c->correction)
        return fail(MVDR_EINVAL, "mvdr_correct_large_error_nodes: missing node array");
    if (c->num_surfels && (!c->live_vertex || !c->live_normal || !c->surfel_knn || !c->surfel_knn_weight))
        return fail(MVDR_EINVAL, "mvdr_correct_large_error_nodes: missing surfel array");
    if (c->width < 5 || c->height < 5 || c->width > 65535 || c->height > 65535)
        return fail(MVDR_EINVAL, "mvdr_correct_large_error_nodes: guide map size out of range");
    const void* a16[] = {c->live_nodes, c->node_knn_weight, c->correction, c->node_se3, c->live_vertex,
                         c->live_normal, c->surfel_knn_weight};
    for (const void* p : a16)
        if (p && !aligned16(p)) return fail(MVDR_EINVAL, "mvdr_correct_large_error_nodes: arrays must be 16-byte aligned");
    CorrArgs a;
    std::memset(&a, 0, sizeof(a));
    for (uint32_t v = 0; v < I->num_views; ++v) {
        const mvdr_correction_view& g = c->views[v];
        if (!g.se3_map || !g.valid_map || !g.previous_vertex_map)
            return fail(MVDR_EINVAL, "mvdr_correct_large_error_nodes: missing guide map of a bound view");
        if (!aligned16(g.se3_map) || !aligned16(g.previous_vertex_map))
            return fail(MVDR_EINVAL, "mvdr_correct_large_error_nodes: guide maps must be 16-byte aligned");
        a.pitch[v] = g.pitch ? g.pitch : c->width;
        if (a.pitch[v] < c->width) return fail(MVDR_EINVAL, "mvdr_correct_large_error_nodes: pitch below width");
        a.se3_map[v] = g.se3_map;
        a.valid[v] = g.valid_map;
        a.prev[v] = reinterpret_cast<const float4*>(g.previous_vertex_map);
    }
    a.cols = c->width;
    a.rows = c->height;
    a.united = c->united_error;
    a.threshold = c->error_threshold;
    a.four_radius_sq = 4.0f * I->node_radius * I->node_radius;
    a.field = c->node_se3 ? reinterpret_cast<DQ*>(c->node_se3) : I->se3;
    a.live_nodes = reinterpret_cast<float4*>(c->live_nodes);
    a.node_knn = reinterpret_cast<const ushort4*>(c->node_knn);
    a.node_w = reinterpret_cast<const float4*>(c->node_knn_weight);
    a.S = c->num_surfels;
    a.live_v = reinterpret_cast<float4*>(c->live_vertex);
    a.live_n = reinterpret_cast<float4*>(c->live_normal);
    a.surfel_knn = reinterpret_cast<const ushort4*>(c->surfel_knn);
    a.surfel_w = reinterpret_cast<const float4*>(c->surfel_knn_weight);
    a.correction = reinterpret_cast<DQ*>(c->correction);
    const cudaStream_t st = (cudaStream_t)stream;
    const InstDesc* d_inst = b->d_inst;
    const uint32_t inst = solver->inst;
    MVDR_LAUNCH(guided_node_kernel, dim3((I->N + 127) / 128), 128, 0, st, d_inst, inst, a);
    const uint64_t total = (uint64_t)a.S + I->N;
    MVDR_LAUNCH(correct_kernel, dim3((uint32_t)((total + 127) / 128)), 128, 0, st, d_inst, inst, a);
    if (a.field != I->se3) {
        // the corrected field becomes the solver's current warp field
        const cudaError_t e = cudaMemcpyAsync(I->se3, a.field, sizeof(DQ) * I->N, cudaMemcpyDeviceToDevice, st);
        if (e != cudaSuccess) return fail(MVDR_ECUDA, std::string(fn) + ": " + cudaGetErrorString(e));
    }
    return launch_error(fn);
}
