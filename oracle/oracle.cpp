/*
 * CPU oracle for the non-rigid Gauss-Newton solver - TEST INFRASTRUCTURE.
 *
 * This file restates, on the CPU and in plain C++, the algorithm of the
 * reference NonRigidSolver stage (MultiViewDynRecon core/NonRigidSolver). It
 * exists only so that tests/, the smoke check and bench.py's CPU-baseline leg
 * can check and time the CUDA library against it. Nothing in the library
 * links or calls this file.
 *
 * Parity is unpinned against reference outputs: the reference cannot be
 * compiled here (it needs Eigen, PCL, TensorRT and Windows headers, and the
 * solve orchestrator and base/Constants.cpp are absent) and it ships no golden
 * vectors (pcg_test.dat / pcg_result.dat are missing,
 * block6x6_pcg_weber.cpp:14-58). The restatement is instead pinned by the
 * mathematical known-answer tests in tests/test_oracle.py.
 *
 * Two arithmetic modes:
 *   fp64 == 0: per-term residuals and Jacobians in float with the reference's
 *              operation order (the projection divide in double as the
 *              reference's `z + 1e-10` literal promotes it); sums accumulated
 *              in double; PCG vectors in float.
 *   fp64 == 1: everything in double.
 * In either mode discrete choices (projected pixel, validity) may be frozen
 * from another run with orc_freeze_decisions.
 */
#include "../include/mvdr.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <numeric>
#include <string>
#include <thread>
#include <vector>

namespace {

using u16 = uint16_t;
using u32 = uint32_t;

// ------------------------------------------------------------------ math ---

template <class R> struct V3 { R x, y, z; };
template <class R> inline V3<R> v3(R x, R y, R z) { return {x, y, z}; }
template <class R> inline V3<R> operator+(V3<R> a, V3<R> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class R> inline V3<R> operator-(V3<R> a, V3<R> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class R> inline V3<R> operator*(R s, V3<R> a) { return {s * a.x, s * a.y, s * a.z}; }
template <class R> inline R dot(V3<R> a, V3<R> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class R> inline V3<R> vcross(V3<R> a, V3<R> b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

// 3x4 rigid transform; m[r][c] row-major here (the ABI stores columns).
template <class R> struct M34 {
    R m[3][3];
    R t[3];
    V3<R> rot(V3<R> v) const {
        return {m[0][0] * v.x + m[0][1] * v.y + m[0][2] * v.z, m[1][0] * v.x + m[1][1] * v.y + m[1][2] * v.z,
                m[2][0] * v.x + m[2][1] * v.y + m[2][2] * v.z};
    }
    V3<R> rotT(V3<R> v) const {  // mat33::transpose_dot
        return {m[0][0] * v.x + m[1][0] * v.y + m[2][0] * v.z, m[0][1] * v.x + m[1][1] * v.y + m[2][1] * v.z,
                m[0][2] * v.x + m[1][2] * v.y + m[2][2] * v.z};
    }
    V3<R> apply(V3<R> v) const { V3<R> r = rot(v); return {r.x + t[0], r.y + t[1], r.z + t[2]}; }
};

template <class R> M34<R> load_mat34(const mvdr_mat34& a) {
    M34<R> o;
    for (int c = 0; c < 3; ++c)
        for (int r = 0; r < 3; ++r) o.m[r][c] = (R)a.rot[3 * c + r];
    for (int r = 0; r < 3; ++r) o.t[r] = (R)a.trans[r];
    return o;
}

// mat34::inverse (math/MatUtils.h:585-590), evaluated in float like the reference
template <class R> M34<R> inverse34(const M34<R>& a) {
    M34<R> o;
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) o.m[r][c] = a.m[c][r];
    for (int r = 0; r < 3; ++r) o.t[r] = -(o.m[r][0] * a.t[0] + o.m[r][1] * a.t[1] + o.m[r][2] * a.t[2]);
    return o;
}

// quaternion (x, y, z, w), Quaternion.h
template <class R> struct Q { R x, y, z, w; };
template <class R> inline Q<R> qmul(Q<R> a, Q<R> b) {  // Quaternion.h:303-312
    Q<R> q;
    q.w = a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z;
    q.x = a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y;
    q.y = a.w * b.y - a.x * b.z + a.y * b.w + a.z * b.x;
    q.z = a.w * b.z + a.x * b.y - a.y * b.x + a.z * b.w;
    return q;
}
template <class R> inline Q<R> qconj(Q<R> a) { return {-a.x, -a.y, -a.z, a.w}; }
template <class R> inline Q<R> qscale(R s, Q<R> a) { return {s * a.x, s * a.y, s * a.z, s * a.w}; }
template <class R> inline R qdot(Q<R> a, Q<R> b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }

template <class R> struct DQ { Q<R> q0, q1; };

template <class R> inline DQ<R> load_dq(const mvdr_dual_quaternion& d) {
    return {{(R)d.q0[0], (R)d.q0[1], (R)d.q0[2], (R)d.q0[3]}, {(R)d.q1[0], (R)d.q1[1], (R)d.q1[2], (R)d.q1[3]}};
}

// averageDualQuaternion (DualQuaternion.h:381-393)
template <class R>
inline DQ<R> blend(const std::vector<DQ<R>>& field, const u16 knn[4], const float w[4]) {
    DQ<R> a{{0, 0, 0, 0}, {0, 0, 0, 0}};
    for (int k = 0; k < 4; ++k) {
        const DQ<R>& d = field[knn[k]];
        const R s = (R)w[k];
        a.q0 = {a.q0.x + s * d.q0.x, a.q0.y + s * d.q0.y, a.q0.z + s * d.q0.z, a.q0.w + s * d.q0.w};
        a.q1 = {a.q1.x + s * d.q1.x, a.q1.y + s * d.q1.y, a.q1.z + s * d.q1.z, a.q1.w + s * d.q1.w};
    }
    return a;
}

template <class R> inline R inv_sqrt(R v) { return (R)1 / std::sqrt(v); }

// DualQuaternion::se3_matrix (DualQuaternion.h:281-287, 326-332)
template <class R> inline M34<R> se3_matrix(DQ<R> d) {
    const R inv = inv_sqrt(qdot(d.q0, d.q0));
    d.q0 = qscale(inv, d.q0);
    d.q1 = qscale(inv, d.q1);
    const R dd = qdot(d.q0, d.q1);
    d.q1 = {d.q1.x - dd * d.q0.x, d.q1.y - dd * d.q0.y, d.q1.z - dd * d.q0.z, d.q1.w - dd * d.q0.w};
    const Q<R> q = d.q0;
    M34<R> m;  // Quaternion::rotation_matrix(false), Quaternion.h:207-220
    m.m[0][0] = 1 - 2 * q.y * q.y - 2 * q.z * q.z;
    m.m[0][1] = 2 * q.x * q.y - 2 * q.z * q.w;
    m.m[0][2] = 2 * q.x * q.z + 2 * q.y * q.w;
    m.m[1][0] = 2 * q.x * q.y + 2 * q.z * q.w;
    m.m[1][1] = 1 - 2 * q.x * q.x - 2 * q.z * q.z;
    m.m[1][2] = 2 * q.y * q.z - 2 * q.x * q.w;
    m.m[2][0] = 2 * q.x * q.z - 2 * q.y * q.w;
    m.m[2][1] = 2 * q.y * q.z + 2 * q.x * q.w;
    m.m[2][2] = 1 - 2 * q.x * q.x - 2 * q.y * q.y;
    const Q<R> tp = qmul(qscale((R)2, d.q1), qconj(d.q0));
    m.t[0] = tp.x;
    m.t[1] = tp.y;
    m.t[2] = tp.z;
    return m;
}

// DualQuaternion::operator mat34 (DualQuaternion.h:309-319): normalized(), then
// Quaternion::matrix() (normalises q0 again, Quaternion.h:183-200)
template <class R> inline M34<R> dq_to_mat34(DQ<R> d) {
    const R inv = inv_sqrt(qdot(d.q0, d.q0));
    d.q0 = qscale(inv, d.q0);
    d.q1 = qscale(inv, d.q1);
    const R dd = qdot(d.q0, d.q1);
    d.q1 = {d.q1.x - dd * d.q0.x, d.q1.y - dd * d.q0.y, d.q1.z - dd * d.q0.z, d.q1.w - dd * d.q0.w};
    Q<R> q = d.q0;
    const R inv2 = inv_sqrt(qdot(q, q));
    q = qscale(inv2, q);
    M34<R> m;
    m.m[0][0] = 1 - 2 * q.y * q.y - 2 * q.z * q.z;
    m.m[0][1] = 2 * q.x * q.y - 2 * q.z * q.w;
    m.m[0][2] = 2 * q.x * q.z + 2 * q.y * q.w;
    m.m[1][0] = 2 * q.x * q.y + 2 * q.z * q.w;
    m.m[1][1] = 1 - 2 * q.x * q.x - 2 * q.z * q.z;
    m.m[1][2] = 2 * q.y * q.z - 2 * q.x * q.w;
    m.m[2][0] = 2 * q.x * q.z - 2 * q.y * q.w;
    m.m[2][1] = 2 * q.y * q.z + 2 * q.x * q.w;
    m.m[2][2] = 1 - 2 * q.x * q.x - 2 * q.y * q.y;
    const Q<R> tp = qmul(qscale((R)2, d.q1), qconj(d.q0));
    m.t[0] = tp.x;
    m.t[1] = tp.y;
    m.t[2] = tp.z;
    return m;
}

// Quaternion(mat33) (Quaternion.h:46-77)
template <class R> inline Q<R> mat_to_quat(const M34<R>& a) {
    const auto& m = a.m;
    Q<R> q;
    const R tr = m[0][0] + m[1][1] + m[2][2];
    if (tr > 0) {
        const R s = std::sqrt(tr + (R)1) * 2;
        q.w = s * (R)0.25;
        q.x = (m[2][1] - m[1][2]) / s;
        q.y = (m[0][2] - m[2][0]) / s;
        q.z = (m[1][0] - m[0][1]) / s;
    } else if ((m[0][0] > m[1][1]) && (m[0][0] > m[2][2])) {
        const R s = std::sqrt((R)1 + m[0][0] - m[1][1] - m[2][2]) * 2;
        q.w = (m[2][1] - m[1][2]) / s;
        q.x = (R)0.25 * s;
        q.y = (m[0][1] + m[1][0]) / s;
        q.z = (m[0][2] + m[2][0]) / s;
    } else if (m[1][1] > m[2][2]) {
        const R s = std::sqrt((R)1 + m[1][1] - m[0][0] - m[2][2]) * 2;
        q.w = (m[0][2] - m[2][0]) / s;
        q.x = (m[0][1] + m[1][0]) / s;
        q.y = (R)0.25 * s;
        q.z = (m[1][2] + m[2][1]) / s;
    } else {
        const R s = std::sqrt((R)1 + m[2][2] - m[0][0] - m[1][1]) * 2;
        q.w = (m[1][0] - m[0][1]) / s;
        q.x = (m[0][2] + m[2][0]) / s;
        q.y = (m[1][2] + m[2][1]) / s;
        q.z = (R)0.25 * s;
    }
    return q;
}

// DualQuaternion(mat34) (DualQuaternion.h:123-130)
template <class R> inline DQ<R> mat34_to_dq(const M34<R>& a) {
    DQ<R> d;
    d.q0 = mat_to_quat(a);
    const Q<R> tq{(R)0.5 * a.t[0], (R)0.5 * a.t[1], (R)0.5 * a.t[2], (R)0};
    d.q1 = qmul(tq, d.q0);  // vec_part * rot_part: q1 = tq*q0 + 1*0
    return d;
}

// applyWarpFieldUpdateKernel (SolverIterationData.cu:9-57)
template <class R> inline DQ<R> apply_twist(DQ<R> prev, const R tw[6]) {
    M34<R> se3;
    const V3<R> w{tw[0], tw[1], tw[2]};
    if (std::fabs(w.x) + std::fabs(w.y) + std::fabs(w.z) < (R)1e-4) {
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) se3.m[r][c] = (r == c) ? (R)1 : (R)0;
    } else {
        const R angle = std::sqrt(dot(w, w));
        const V3<R> axis = ((R)1 / angle) * w;
        const R c = std::cos(angle), s = std::sin(angle), t = (R)1 - c;
        se3.m[0][0] = t * axis.x * axis.x + c;
        se3.m[0][1] = t * axis.x * axis.y - axis.z * s;
        se3.m[0][2] = t * axis.x * axis.z + axis.y * s;
        se3.m[1][0] = t * axis.x * axis.y + axis.z * s;
        se3.m[1][1] = t * axis.y * axis.y + c;
        se3.m[1][2] = t * axis.y * axis.z - axis.x * s;
        se3.m[2][0] = t * axis.x * axis.z - axis.y * s;
        se3.m[2][1] = t * axis.y * axis.z + axis.x * s;
        se3.m[2][2] = t * axis.z * axis.z + c;
    }
    se3.t[0] = tw[3];
    se3.t[1] = tw[4];
    se3.t[2] = tw[5];
    const M34<R> p = dq_to_mat34(prev);
    M34<R> n;  // mat34::operator* (MatUtils.h:449-455)
    for (int r = 0; r < 3; ++r) {
        for (int c = 0; c < 3; ++c)
            n.m[r][c] = se3.m[r][0] * p.m[0][c] + se3.m[r][1] * p.m[1][c] + se3.m[r][2] * p.m[2][c];
        n.t[r] = se3.m[r][0] * p.t[0] + se3.m[r][1] * p.t[1] + se3.m[r][2] * p.t[2] + se3.t[r];
    }
    return mat34_to_dq(n);
}

// compute_feature_huber_weight (huber_weight.h:11-27)
template <class R> inline R huber(R r) {
    const R a = std::fabs(r);
    const R c = (R)7.5e-2f;
    return a < c ? (R)1 : c / a;
}

// __float2int_rn: round to nearest, ties to even
inline int rint_even(float v) { return (int)std::nearbyint(v); }

// --------------------------------------------------------------- oracle ---

enum TermType { kDense = 0, kSmooth = 1, kForeground = 2, kFeature = 3, kCross = 4, kInvalid = 5 };

struct ViewData {
    std::vector<mvdr_float4> ref_v, ref_n, obs_v, obs_n;
    std::vector<u32> index;
    std::vector<float> fg_mask, fg_grad;
    std::vector<mvdr_float4> rgb;          // density term: rendered normalised rgb
    std::vector<float> dens, dens_grad;    // density term: observed grey level, gradient
    mvdr_intrinsic intr;
    mvdr_mat34 w2c, init;
};

struct Corr {
    std::vector<mvdr_float4> target, ref, w;
    std::vector<u16> knn;
};

struct Oracle {
    mvdr_config cfg;
    int fp64 = 0;
    u32 W = 0, H = 0, V = 0, N = 0, S = 0, E = 0;
    std::vector<ViewData> views;
    std::vector<u16> surfel_knn;
    std::vector<mvdr_float4> surfel_w;
    std::vector<mvdr_dual_quaternion> node_se3_init;
    std::vector<mvdr_float4> nodes;
    std::vector<u16> graph;
    Corr feat, cross;

    // current warp field, kept in double; rounded to float at each update
    std::vector<DQ<double>> se3d;
    std::vector<double> pcg_history;  // delta at the start of each PCG iteration of the last solve
    int gn_iter = 0;

    // compaction
    std::vector<u16> dense_pix, dense_knn, fg_pix, fg_knn;  // 4 per term
    std::vector<mvdr_float4> dense_w, fg_w;
    u32 Td = 0, Ts = 0, Tf = 0, Tp = 0, Tc = 0;
    u32 off[5] = {0, 0, 0, 0, 0};

    // index
    std::vector<u32> n2t_offset, n2t_index;
    u32 enc = 4096;
    std::vector<u32> half_keys, np_index, sym_keys, ranges, blkrow_offset;
    std::vector<int32_t> rowptr, colptr;
    u32 nbins = 0, binnnz = 0;

    // term data (float layout of the ABI)
    std::vector<float> term_jr;   // 8 per dense+fg term
    std::vector<float> density_jr;  // 8 per dense term: density J (6), residual, pixel (use_density)
    std::vector<u32> frozen_density;  // frozen projected pixels of the density term
    std::vector<float> smooth;    // 8 per smooth term
    std::vector<float> warped;    // 4 per feature+cross term
    // frozen decisions: per dense+fg term the projected pixel (v*W+u) or invalid
    std::vector<u32> frozen_pixel;
    std::vector<uint8_t> frozen_smooth;
    bool frozen = false;

    // assembly
    std::vector<double> D, b, Minv, offdiag, bbdata, x;
    double energy = 0;
    mvdr_penalty lambda{};

    u32 enc_mult() const {
        u32 m = 4096;
        while (m < N) m <<= 1;
        return m;
    }

    void penalty_for(int iter) {
        if (!cfg.use_elastic_penalty) {
            lambda = cfg.penalty;
            if (!cfg.use_density) lambda.density = 0.0f;
            return;
        }
        if (iter < cfg.num_global_iterations) {  // PenaltyConstants.cpp:25-37
            lambda.smooth = 5.0f;
            lambda.density = 0.0f;
            lambda.foreground = cfg.use_foreground ? 2e-3f : 0.0f;
            lambda.feature = 1.0f;
            lambda.cross_view = cfg.use_cross_view ? 1.0f : 0.0f;
        } else {  // PenaltyConstants.cpp:39-51
            lambda.smooth = 5.0f;
            lambda.density = cfg.use_density ? 1e-2f : 0.0f;
            lambda.foreground = 0.0f;
            lambda.feature = 0.0f;
            lambda.cross_view = cfg.use_cross_view ? 1.0f : 0.0f;
        }
    }

    // ---------------------------------------------------------- inputs ---
    int set_inputs(const mvdr_config* c, const mvdr_inputs* in) {
        cfg = *c;
        W = c->image_width;
        H = c->image_height;
        V = in->num_views;
        N = in->num_nodes;
        S = in->num_surfels;
        E = in->num_graph_edges;
        if (V > MVDR_MAX_VIEWS || N == 0) return MVDR_EINVAL;
        views.assign(V, ViewData());
        const size_t P = (size_t)W * H;
        for (u32 v = 0; v < V; ++v) {
            const mvdr_view_inputs& vi = in->views[v];
            const u32 pitch = vi.pitch ? vi.pitch : W;
            ViewData& d = views[v];
            d.ref_v.resize(P); d.ref_n.resize(P); d.obs_v.resize(P); d.obs_n.resize(P); d.index.resize(P);
            for (u32 y = 0; y < H; ++y)
                for (u32 x = 0; x < W; ++x) {
                    const size_t s = (size_t)y * pitch + x, t = (size_t)y * W + x;
                    d.ref_v[t] = vi.reference_vertex_map[s];
                    d.ref_n[t] = vi.reference_normal_map[s];
                    d.obs_v[t] = vi.vertex_confidence_map[s];
                    d.obs_n[t] = vi.normal_radius_map[s];
                    d.index[t] = vi.index_map[s];
                }
            if (vi.filtered_foreground_mask && vi.foreground_mask_gradient) {
                d.fg_mask.resize(P);
                d.fg_grad.resize(2 * P);
                for (u32 y = 0; y < H; ++y)
                    for (u32 x = 0; x < W; ++x) {
                        const size_t s = (size_t)y * pitch + x, t = (size_t)y * W + x;
                        d.fg_mask[t] = vi.filtered_foreground_mask[s];
                        d.fg_grad[2 * t] = vi.foreground_mask_gradient[2 * s];
                        d.fg_grad[2 * t + 1] = vi.foreground_mask_gradient[2 * s + 1];
                    }
            }
            if (c->use_density && vi.normalized_rgb_map && vi.density_map && vi.density_gradient_map) {
                d.rgb.resize(P);
                d.dens.resize(P);
                d.dens_grad.resize(2 * P);
                for (u32 y = 0; y < H; ++y)
                    for (u32 x = 0; x < W; ++x) {
                        const size_t s = (size_t)y * pitch + x, t = (size_t)y * W + x;
                        d.rgb[t] = vi.normalized_rgb_map[s];
                        d.dens[t] = vi.density_map[s];
                        d.dens_grad[2 * t] = vi.density_gradient_map[2 * s];
                        d.dens_grad[2 * t + 1] = vi.density_gradient_map[2 * s + 1];
                    }
            }
            d.intr = vi.intrinsic;
            d.w2c = vi.world2camera;
            d.init = vi.initial_camera_se3;
        }
        surfel_knn.assign(in->surfel_knn, in->surfel_knn + 4 * (size_t)S);
        surfel_w.assign(in->surfel_knn_weight, in->surfel_knn_weight + S);
        node_se3_init.assign(in->node_se3, in->node_se3 + N);
        nodes.assign(in->canonical_node_coords, in->canonical_node_coords + N);
        graph.assign(in->node_graph, in->node_graph + 2 * (size_t)E);
        auto copy_corr = [](Corr& o, const mvdr_correspondences& c, bool on) {
            const u32 n = on ? c.count : 0;
            o.target.assign(c.target_vertex, c.target_vertex + n);
            o.ref.assign(c.reference_vertex, c.reference_vertex + n);
            o.w.assign(c.knn_weight, c.knn_weight + n);
            o.knn.assign(c.knn, c.knn + 4 * (size_t)n);
        };
        copy_corr(feat, in->feature, cfg.use_feature != 0);
        copy_corr(cross, in->cross_view, cfg.use_cross_view != 0);
        if (cfg.use_feature) select_features(in);
        se3d.resize(N);
        for (u32 i = 0; i < N; ++i) se3d[i] = load_dq<double>(node_se3_init[i]);
        gn_iter = 0;
        frozen = false;
        return MVDR_OK;
    }

    // SparseCorrespondenceHandler (SparseCorrespondenceHandler.cu:18-199), the
    // nearest-distance form: raw pixel pairs -> feature terms, in candidate
    // order. Border addressing: outside the image a float4 map reads zero and
    // the index map reads 0 (a "surfel"); such a pixel's coordinate wraps to
    // 0xFFFF and fails the image-size test.
    void select_features(const mvdr_inputs* in) {
        const mvdr_feature_pairs& fp = in->feature_pairs;
        bool any = false;
        for (u32 v = 0; v < V; ++v) any |= fp.count[v] != 0;
        if (!any) return;
        feat = Corr();
        auto zero = [](const mvdr_float4& a) {
            return (double)std::fabs(a.x) < 1e-3 && (double)std::fabs(a.y) < 1e-3 && (double)std::fabs(a.z) < 1e-3;
        };
        auto sq = [](const mvdr_float4& a, const mvdr_float4& b) {
            return (a.x - b.x) * (a.x - b.x) + (a.y - b.y) * (a.y - b.y) + (a.z - b.z) * (a.z - b.z);
        };
        for (u32 v = 0; v < V; ++v) {
            const ViewData& d = views[v];
            const mvdr_view_inputs& vi = in->views[v];
            const u32 pitch = vi.pitch ? vi.pitch : W;
            auto at4 = [&](const std::vector<mvdr_float4>& m, int x, int y) {
                if (x < 0 || y < 0 || x >= (int)W || y >= (int)H) return mvdr_float4{0, 0, 0, 0};
                return m[(size_t)y * W + x];
            };
            auto live = [&](int x, int y) {
                if (x < 0 || y < 0 || x >= (int)W || y >= (int)H) return mvdr_float4{0, 0, 0, 0};
                return fp.live_vertex_map[v][(size_t)y * pitch + x];
            };
            const M34<float> init = load_mat34<float>(d.init);
            const M34<float> c2w = inverse34(load_mat34<float>(d.w2c));
            for (u32 k = 0; k < fp.count[v]; ++k) {
                const u16* pr = fp.pixel_pairs[v] + 4 * (size_t)k;
                u16 dx = 0xFFFF, dy = 0xFFFF;
                for (int y = (int)pr[3] - 1; y <= (int)pr[3] + 1; ++y)
                    for (int x = (int)pr[2] - 1; x <= (int)pr[2] + 1; ++x)
                        if (!zero(at4(d.obs_v, x, y))) {
                            dx = (u16)x;
                            dy = (u16)y;
                            break;
                        }
                if (!zero(at4(d.obs_v, pr[2], pr[3]))) {
                    dx = pr[2];
                    dy = pr[3];
                }
                if (!(dx < W && dy < H)) continue;
                if (fp.edge_mask[v] && fp.edge_mask[v][(size_t)dy * pitch + dx] == 1) continue;
                const mvdr_float4 ov = d.obs_v[(size_t)dy * W + dx];
                u16 gx = 0xFFFF, gy = 0xFFFF;
                float best = 100.0f;
                for (int y = (int)pr[1] - 1; y <= (int)pr[1] + 1; ++y)
                    for (int x = (int)pr[0] - 1; x <= (int)pr[0] + 1; ++x) {
                        const bool inside = x >= 0 && y >= 0 && x < (int)W && y < (int)H;
                        const u32 s = inside ? d.index[(size_t)y * W + x] : 0u;
                        if (s != MVDR_INVALID_INDEX) {
                            const float dd = sq(ov, live(x, y));
                            if (dd < best) {
                                gx = (u16)x;
                                gy = (u16)y;
                                best = dd;
                            }
                        }
                    }
                if (!(gx < W && gy < H)) continue;
                const size_t og = (size_t)gy * W + gx;
                const u32 s = d.index[og];
                if (!(s < S && sq(d.ref_v[og], ov) < 2.5e-3f)) continue;
                const mvdr_float4 rv = d.ref_v[og];
                const V3<float> r0 = init.apply({rv.x, rv.y, rv.z});
                const mvdr_float4 dv = ov;  // the observed vertex at the chosen depth pixel
                const V3<float> t0 = c2w.apply(init.apply({dv.x, dv.y, dv.z}));
                feat.target.push_back({t0.x, t0.y, t0.z, 1.0f});
                feat.ref.push_back({r0.x, r0.y, r0.z, rv.w});
                feat.w.push_back(surfel_w[s]);
                for (int j = 0; j < 4; ++j) feat.knn.push_back(surfel_knn[4 * (size_t)s + j]);
            }
        }
    }

    template <class R> std::vector<DQ<R>> field() const {
        std::vector<DQ<R>> f(N);
        for (u32 i = 0; i < N; ++i) {
            const DQ<double>& d = se3d[i];
            f[i] = {{(R)d.q0.x, (R)d.q0.y, (R)d.q0.z, (R)d.q0.w}, {(R)d.q1.x, (R)d.q1.y, (R)d.q1.z, (R)d.q1.w}};
        }
        return f;
    }

    // view of compacted pixel `idx` (DenseDepthJacobianResidual.cu:14-22 in compat mode)
    u32 view_of(u32 idx, const u16* pix, const std::vector<u32>& per_view_count) const {
        if (!(cfg.compat_flags & MVDR_COMPAT_REF_VIEW_LOOKUP)) return pix[4 * idx + 2];
        for (u32 i = 0; i < V; ++i) {
            if (i == V - 1) return i;
            if (per_view_count[i] <= idx && idx < per_view_count[i + 1]) return i;
        }
        return V - 1;
    }
    std::vector<u32> dense_view_count, fg_view_count;

    // ----------------------------------------------------- compaction ---
    // ImageTermKNNFetcher.cu:19-68 + NonRigidSolver.cu:14-34 (pixel knn)
    void compact_dense() {
        dense_pix.clear(); dense_knn.clear(); dense_w.clear();
        dense_view_count.assign(V, 0);
        for (u32 v = 0; v < V; ++v)
            for (u32 y = 0; y < H; ++y)
                for (u32 x = 0; x < W; ++x) {
                    const u32 s = views[v].index[(size_t)y * W + x];
                    if (s == MVDR_INVALID_INDEX) continue;
                    dense_pix.insert(dense_pix.end(), {(u16)x, (u16)y, (u16)v, 0});
                    dense_knn.insert(dense_knn.end(), surfel_knn.begin() + 4 * (size_t)s,
                                     surfel_knn.begin() + 4 * (size_t)s + 4);
                    dense_w.push_back(surfel_w[s]);
                    dense_view_count[v]++;
                }
        Td = (u32)dense_w.size();
    }

    // DensityForegroundMapHandler.cu:17-146 with the initial warp field
    void compact_foreground() {
        fg_pix.clear(); fg_knn.clear(); fg_w.clear();
        fg_view_count.assign(V, 0);
        if (!cfg.use_foreground) { Tf = 0; return; }
        const auto f = field<float>();
        for (u32 v = 0; v < V; ++v) {
            const ViewData& d = views[v];
            if (d.fg_mask.empty()) continue;
            const M34<float> init = load_mat34<float>(d.init), w2c = load_mat34<float>(d.w2c);
            const M34<float> inv = inverse34(init);
            for (u32 y = 0; y < H; ++y)
                for (u32 x = 0; x < W; ++x) {
                    const u32 s = d.index[(size_t)y * W + x];
                    if (s == MVDR_INVALID_INDEX) continue;
                    const mvdr_float4 cv = d.ref_v[(size_t)y * W + x], cn = d.ref_n[(size_t)y * W + x];
                    const V3<float> cv0 = init.apply(v3(cv.x, cv.y, cv.z));
                    const V3<float> cn0 = init.rot(v3(cn.x, cn.y, cn.z));
                    const M34<float> se3 = se3_matrix(blend(f, &surfel_knn[4 * (size_t)s], &surfel_w[s].x));
                    const V3<float> wv = se3.apply(cv0), wn = se3.rot(cn0);
                    V3<float> vc = inv.apply(w2c.apply(wv));
                    V3<float> nc = inv.rot(w2c.rot(wn));
                    const float ninv = 1.0f / std::sqrt(dot(vc, vc));
                    const V3<float> dir = ninv * vc;
                    const float cosang = -dot(dir, nc);
                    const int u = rint_even((float)(((double)vc.x / ((double)vc.z + 1e-10)) * (double)d.intr.focal_x +
                                                    (double)d.intr.principal_x));
                    const int vv = rint_even((float)(((double)vc.y / ((double)vc.z + 1e-10)) * (double)d.intr.focal_y +
                                                     (double)d.intr.principal_y));
                    bool ok = false;
                    if (u >= 0 && u < (int)W && vv >= 0 && vv < (int)H && cosang > 0.5f) {
                        if (d.fg_mask[(size_t)vv * W + u] > 1e-5f) ok = true;
                    }
                    if (!ok) continue;
                    fg_pix.insert(fg_pix.end(), {(u16)x, (u16)y, (u16)v, 0});
                    fg_knn.insert(fg_knn.end(), surfel_knn.begin() + 4 * (size_t)s, surfel_knn.begin() + 4 * (size_t)s + 4);
                    fg_w.push_back(surfel_w[s]);
                    fg_view_count[v]++;
                }
        }
        Tf = (u32)fg_w.size();
    }

    // ---------------------------------------------------------- index ---
    const u16* knn_of(TermType t, u32 k) const {
        switch (t) {
            case kDense: return &dense_knn[4 * (size_t)k];
            case kForeground: return &fg_knn[4 * (size_t)k];
            case kFeature: return &feat.knn[4 * (size_t)k];
            case kCross: return &cross.knn[4 * (size_t)k];
            default: return nullptr;
        }
    }
    const float* w_of(TermType t, u32 k) const {
        switch (t) {
            case kDense: return &dense_w[k].x;
            case kForeground: return &fg_w[k].x;
            case kFeature: return &feat.w[k].x;
            case kCross: return &cross.w[k].x;
            default: return nullptr;
        }
    }
    // query_typed_index (base/term_offset_types.h:66-99)
    void typed(u32 term, TermType& t, u32& k) const {
        if (term < off[0]) { t = kDense; k = term; return; }
        if (term < off[1]) { t = kSmooth; k = term - off[0]; return; }
        if (term < off[2]) { t = kForeground; k = term - off[1]; return; }
        if (term < off[3]) { t = kFeature; k = term - off[2]; return; }
        if (term < off[4]) { t = kCross; k = term - off[3]; return; }
        t = kInvalid; k = 0xFFFFFFFFu;
    }

    void build_index() {
        compact_dense();
        compact_foreground();
        Ts = E;
        Tp = (u32)feat.w.size();
        Tc = (u32)cross.w.size();
        // size2offset (term_offset_types.h:44-64)
        off[0] = Td; off[1] = off[0] + Ts; off[2] = off[1] + Tf; off[3] = off[2] + Tp; off[4] = off[3] + Tc;
        const u32 T = off[4];

        // node -> term: buildTermKeyValueKernel (Node2TermsIndex.cu:8-110), stable sort
        std::vector<u16> keys;
        std::vector<u32> vals;
        keys.reserve(4 * (size_t)T);
        vals.reserve(4 * (size_t)T);
        for (u32 term = 0; term < T; ++term) {
            TermType t; u32 k;
            typed(term, t, k);
            if (t == kSmooth) {
                keys.push_back(graph[2 * (size_t)k]); vals.push_back(term);
                keys.push_back(graph[2 * (size_t)k + 1]); vals.push_back(term);
            } else {
                const u16* kn = knn_of(t, k);
                for (int j = 0; j < 4; ++j) { keys.push_back(kn[j]); vals.push_back(term); }
            }
        }
        std::vector<u32> order(keys.size());
        std::iota(order.begin(), order.end(), 0u);
        std::stable_sort(order.begin(), order.end(), [&](u32 a, u32 b2) { return keys[a] < keys[b2]; });
        n2t_index.resize(order.size());
        std::vector<u16> sorted_keys(order.size());
        for (size_t i = 0; i < order.size(); ++i) { n2t_index[i] = vals[order[i]]; sorted_keys[i] = keys[order[i]]; }
        // computeTermOffsetKernel (Node2TermsIndex.cu:112-134) as a CSR offset;
        // nodes without terms (left unwritten by the reference) get the lower bound
        n2t_offset.assign(N + 1, 0);
        {
            size_t p = 0;
            for (u32 n = 0; n <= N; ++n) {
                while (p < sorted_keys.size() && sorted_keys[p] < n) ++p;
                n2t_offset[n] = (u32)p;
            }
        }

        // node pair -> term: buildKeyValuePairKernel (NodePair2TermsIndex.cu:30-102)
        enc = enc_mult();
        auto encode = [&](u32 i, u32 j) { return i * enc + j; };
        std::vector<u32> pk, pv;
        for (u32 term = 0; term < T; ++term) {
            TermType t; u32 k;
            typed(term, t, k);
            u32 key[6];
            int save = 6;
            for (int i = 0; i < 6; ++i) key[i] = 0xFFFFFFFFu;
            if (t == kSmooth) {
                const u16 a = graph[2 * (size_t)k], b2 = graph[2 * (size_t)k + 1];
                if (a < b2) key[0] = encode(a, b2);
                else if (b2 < a) key[0] = encode(b2, a);
                save = 1;
            } else {
                const u16* kn = knn_of(t, k);
                int o = 0;  // computeKVNodePairKNN (NodePair2TermsIndex.cu:11-28)
                for (int i = 0; i < 4; ++i)
                    for (int j = 0; j < 4; ++j)
                        if (kn[i] < kn[j]) key[o++] = encode(kn[i], kn[j]);
            }
            for (int i = 0; i < save; ++i) { pk.push_back(key[i]); pv.push_back(term); }
        }
        order.resize(pk.size());
        std::iota(order.begin(), order.end(), 0u);
        std::stable_sort(order.begin(), order.end(), [&](u32 a, u32 b2) { return pk[a] < pk[b2]; });
        std::vector<u32> skeys(order.size());
        np_index.resize(order.size());
        for (size_t i = 0; i < order.size(); ++i) { skeys[i] = pk[order[i]]; np_index[i] = pv[order[i]]; }
        // segment + compaction (NodePair2TermsIndex.cu:105-163); keys at or
        // past the encoding range are invalid
        half_keys.clear();
        std::vector<u32> half_off;
        for (size_t i = 0; i < skeys.size(); ++i) {
            const u32 key = skeys[i];
            const bool valid = key != 0xFFFFFFFFu && key / enc < N && key % enc < N;
            if (!valid) continue;
            if (i == 0 || skeys[i - 1] != key) { half_keys.push_back(key); half_off.push_back((u32)i); }
        }
        // the reference sets the last end to the full array size
        // (NodePair2TermsIndex.cu:152-161); with valid inputs that is the
        // number of valid entries
        u32 valid_entries = 0;
        for (u32 key : skeys)
            if (key != 0xFFFFFFFFu && key / enc < N && key % enc < N) ++valid_entries;
        half_off.push_back(valid_entries);
        np_index.resize(valid_entries);
        // symmetric keys, sorted (computeSymmetricNodePairKernel + sort, :165-185, :253-271)
        const size_t P = half_keys.size();
        std::vector<std::pair<u32, std::pair<u32, u32>>> sym(2 * P);
        for (size_t h = 0; h < P; ++h) {
            const u32 i = half_keys[h] / enc, j = half_keys[h] % enc;
            sym[2 * h] = {half_keys[h], {half_off[h], half_off[h + 1]}};
            sym[2 * h + 1] = {encode(j, i), {half_off[h], half_off[h + 1]}};
        }
        std::stable_sort(sym.begin(), sym.end(), [](const auto& a, const auto& b2) { return a.first < b2.first; });
        sym_keys.resize(2 * P);
        ranges.resize(4 * P);
        for (size_t s = 0; s < 2 * P; ++s) {
            sym_keys[s] = sym[s].first;
            ranges[2 * s] = sym[s].second.first;
            ranges[2 * s + 1] = sym[s].second.second;
        }
        // computeRowOffsetKernel (NodePairRowColumnIndex.cu:19-48) as a CSR offset
        blkrow_offset.assign(N + 1, 0);
        {
            size_t p = 0;
            for (u32 n = 0; n <= N; ++n) {
                while (p < sym_keys.size() && sym_keys[p] / enc < n) ++p;
                blkrow_offset[n] = (u32)p;
            }
        }
        // bin lengths, rowptr, colptr (NodePairRowColumnIndex.cu:52-179)
        const u32 msize = 6 * N;
        nbins = (msize + 31) / 32;
        std::vector<u32> binlen(nbins), binscan(nbins + 1, 0);
        for (u32 bI = 0; bI < nbins; ++bI) {
            const u32 begin = 32 * bI / 6;
            u32 end = (32 * bI + 31) / 6;
            end = std::min(end, N - 1);
            u32 mx = 0;
            for (u32 r = begin; r <= end; ++r) mx = std::max(mx, 1 + blkrow_offset[r + 1] - blkrow_offset[r]);
            binlen[bI] = 6 * mx;
            binscan[bI + 1] = binscan[bI] + 32 * binlen[bI];
        }
        binnnz = binscan[nbins];
        rowptr.resize(32 * (size_t)(nbins + 1));
        for (size_t idx = 0; idx < rowptr.size(); ++idx) rowptr[idx] = (int32_t)(idx % 32 + binscan[idx / 32]);
        colptr.assign(binnnz / 6, -1);
        for (u32 row = 0; row < msize; ++row) {
            const u32 blkrow = row / 6, lane = row % 32;
            const int data_off = rowptr[row];
            u32 col = (u32)(data_off - (int)lane) / 6 + lane;
            colptr[col] = (int32_t)(6 * blkrow);
            col += 32;
            for (u32 s = blkrow_offset[blkrow]; s < blkrow_offset[blkrow + 1]; ++s, col += 32)
                colptr[col] = (int32_t)(6 * (sym_keys[s] % enc));
        }
    }

    // -------------------------------------------------------- terms ------
    template <class R> void eval_terms_t() {
        const auto f = field<R>();
        term_jr.assign(8 * (size_t)(Td + Tf), 0.0f);
        smooth.assign(12 * (size_t)Ts, 0.0f);
        warped.assign(8 * (size_t)(Tp + Tc), 0.0f);
        std::vector<M34<R>> init(V), inv(V), w2c(V);
        for (u32 v = 0; v < V; ++v) {
            const M34<float> i32 = load_mat34<float>(views[v].init);
            const M34<float> iv32 = inverse34(i32);  // InitialCameraSE3Inverse in float
            for (int r = 0; r < 3; ++r) {
                for (int c = 0; c < 3; ++c) { init[v].m[r][c] = i32.m[r][c]; inv[v].m[r][c] = iv32.m[r][c]; }
                init[v].t[r] = i32.t[r];
                inv[v].t[r] = iv32.t[r];
            }
            w2c[v] = load_mat34<R>(views[v].w2c);
        }
        // dense depth: computeDenseDepthJacobianKernel (DenseDepthJacobianResidual.cu:24-104)
        for (u32 idx = 0; idx < Td; ++idx) {
            const u16* px = &dense_pix[4 * (size_t)idx];
            const u32 v = view_of(idx, dense_pix.data(), dense_view_count);
            const ViewData& d = views[v];
            const size_t p = (size_t)px[1] * W + px[0];
            const V3<R> cv{(R)d.ref_v[p].x, (R)d.ref_v[p].y, (R)d.ref_v[p].z};
            const V3<R> cn{(R)d.ref_n[p].x, (R)d.ref_n[p].y, (R)d.ref_n[p].z};
            const V3<R> cv0 = init[v].apply(cv), cn0 = init[v].rot(cn);
            const M34<R> se3 = se3_matrix(blend(f, &dense_knn[4 * (size_t)idx], &dense_w[idx].x));
            const V3<R> wv = se3.apply(cv0), wn = se3.rot(cn0);
            V3<R> vc = w2c[v].apply(wv), nc = w2c[v].rot(wn);
            vc = inv[v].apply(vc);
            nc = inv[v].rot(nc);
            float* out = &term_jr[8 * (size_t)idx];
            u32 pix_choice = MVDR_INVALID_INDEX;
            bool valid = false;
            V3<R> dv{0, 0, 0}, dn{0, 0, 0};
            if (frozen) {
                pix_choice = frozen_pixel[idx];
                valid = pix_choice != MVDR_INVALID_INDEX;
                if (valid) {
                    const mvdr_float4 a = d.obs_v[pix_choice], bb = d.obs_n[pix_choice];
                    dv = {(R)a.x, (R)a.y, (R)a.z};
                    dn = {(R)bb.x, (R)bb.y, (R)bb.z};
                }
            } else {
                const int u = rint_even((float)(((double)vc.x / ((double)vc.z + 1e-10)) * (double)d.intr.focal_x +
                                                (double)d.intr.principal_x));
                const int vv = rint_even((float)(((double)vc.y / ((double)vc.z + 1e-10)) * (double)d.intr.focal_y +
                                                 (double)d.intr.principal_y));
                if (u >= 0 && u < (int)W && vv >= 0 && vv < (int)H) {
                    const size_t q = (size_t)vv * W + u;
                    const mvdr_float4 a = d.obs_v[q], bb = d.obs_n[q];
                    dv = {(R)a.x, (R)a.y, (R)a.z};
                    dn = {(R)bb.x, (R)bb.y, (R)bb.z};
                    valid = true;
                    if (std::fabs(a.x) < 1e-3 && std::fabs(a.y) < 1e-3 && std::fabs(a.z) < 1e-3) valid = false;
                    if (dot(dn, nc) < (R)0.7f) valid = false;
                    const V3<R> df = dv - vc;
                    if (dot(df, df) > (R)(0.075f * 0.075f)) valid = false;
                    if (valid) pix_choice = (u32)q;
                }
            }
            if (valid) {
                const R r = dot(dn, vc - dv);
                V3<R> tr = init[v].rot(dn);  // InitialCameraSE3.rot.dot(normal)
                tr = w2c[v].rotT(tr);
                const V3<R> rot = vcross(wv, tr);
                out[0] = (float)rot.x; out[1] = (float)rot.y; out[2] = (float)rot.z;
                out[3] = (float)tr.x; out[4] = (float)tr.y; out[5] = (float)tr.z;
                out[6] = (float)r;
            }
            std::memcpy(&out[7], &pix_choice, 4);
        }
        // smooth: forwardWarpSmootherNodeKernel (NodeGraphSmoothHandler.cu:10-43)
        const R clip = (R)(64.0f * (cfg.node_radius * cfg.node_radius));
        for (u32 k = 0; k < Ts; ++k) {
            const u16 i = graph[2 * (size_t)k], j = graph[2 * (size_t)k + 1];
            const V3<R> xi{(R)nodes[i].x, (R)nodes[i].y, (R)nodes[i].z};
            const V3<R> xj{(R)nodes[j].x, (R)nodes[j].y, (R)nodes[j].z};
            const M34<R> Ti = se3_matrix(f[i]), Tj = se3_matrix(f[j]);
            const V3<R> a = Ti.apply(xj), bq = Tj.apply(xj);
            const V3<R> dd = xi - xj;
            float valid = dot(dd, dd) > clip ? 0.0f : 1.0f;
            if (frozen) valid = frozen_smooth[k] ? 1.0f : 0.0f;
            // record: Ti xj, Tj xj, validity, 0, residual Ti xj - Tj xj (in R), 0
            float* o = &smooth[12 * (size_t)k];
            o[0] = (float)a.x; o[1] = (float)a.y; o[2] = (float)a.z;
            o[3] = (float)bq.x; o[4] = (float)bq.y; o[5] = (float)bq.z;
            o[6] = valid;
            o[7] = 0;
            o[8] = (float)(a.x - bq.x); o[9] = (float)(a.y - bq.y); o[10] = (float)(a.z - bq.z);
            o[11] = 0;
        }
        // foreground: computeForegroundMaskJacobian + computeImageDensityJacobainAndResidual
        // (DensityForegroundJacobianResidual.cu:93-142, density_map_jacobian.cuh:12-79).
        // The reference vertex is taken to frame 0 first, as the dense term
        // does; MVDR_COMPAT_REF_FOREGROUND_FRAME warps it in its own camera's
        // frame, as density_map_jacobian.cuh:32-36 does.
        const bool raw_frame = (cfg.compat_flags & MVDR_COMPAT_REF_FOREGROUND_FRAME) != 0;
        for (u32 idx = 0; idx < Tf; ++idx) {
            const u16* px = &fg_pix[4 * (size_t)idx];
            const u32 v = view_of(idx, fg_pix.data(), fg_view_count);
            const ViewData& d = views[v];
            const size_t p = (size_t)px[1] * W + px[0];
            const V3<R> cv = {(R)d.ref_v[p].x, (R)d.ref_v[p].y, (R)d.ref_v[p].z};
            const V3<R> cv0 = raw_frame ? cv : init[v].apply(cv);
            const M34<R> se3 = se3_matrix(blend(f, &fg_knn[4 * (size_t)idx], &fg_w[idx].x));
            const V3<R> wv = se3.apply(cv0);
            V3<R> vc = w2c[v].apply(wv);
            vc = inv[v].apply(vc);
            float* out = &term_jr[8 * (size_t)(Td + idx)];
            u32 pix_choice = MVDR_INVALID_INDEX;
            if (frozen) {
                pix_choice = frozen_pixel[Td + idx];
            } else {
                const int u = rint_even((float)(((double)vc.x / ((double)vc.z + 1e-10)) * (double)d.intr.focal_x +
                                                (double)d.intr.principal_x));
                const int vv = rint_even((float)(((double)vc.y / ((double)vc.z + 1e-10)) * (double)d.intr.focal_y +
                                                 (double)d.intr.principal_y));
                if (u >= 0 && u < (int)W && vv >= 0 && vv < (int)H) pix_choice = (u32)((size_t)vv * W + u);
            }
            if (pix_choice != MVDR_INVALID_INDEX && !d.fg_mask.empty()) {
                const R img = (R)d.fg_mask[pix_choice];
                const R gx = (R)d.fg_grad[2 * (size_t)pix_choice], gy = (R)d.fg_grad[2 * (size_t)pix_choice + 1];
                const R fx = (R)d.intr.focal_x, fy = (R)d.intr.focal_y;
                V3<R> g;
                g.x = gx * fx / vc.z;
                g.y = gy * fy / vc.z;
                g.z = (R)(-1.0f) / (vc.z * vc.z) * (fx * vc.x * gx + fy * vc.y * gy);
                g = init[v].rot(g);
                g = w2c[v].rotT(g);
                out[0] = (float)(-g.y * wv.z + g.z * wv.y);
                out[1] = (float)(g.x * wv.z - g.z * wv.x);
                out[2] = (float)(-g.x * wv.y + g.y * wv.x);
                out[3] = (float)g.x; out[4] = (float)g.y; out[5] = (float)g.z;
                out[6] = (float)(img - (R)0);
            }
            std::memcpy(&out[7], &pix_choice, 4);
        }
        // density: computeDensityMapJacobian (DensityForegroundJacobianResidual.cu:41-91)
        // with computeImageDensityJacobainAndResidual (density_map_jacobian.cuh:12-79):
        // per dense pixel, observed minus rendered grey level (rgb2density,
        // ColorTypeTransfer.h:51-56); the vertex warped as the dense term warps
        // it, or in its camera's frame under MVDR_COMPAT_REF_FOREGROUND_FRAME
        density_jr.assign(cfg.use_density ? 8 * (size_t)Td : 0, 0.0f);
        for (u32 idx = 0; cfg.use_density && idx < Td; ++idx) {
            const u16* px = &dense_pix[4 * (size_t)idx];
            const u32 v = view_of(idx, dense_pix.data(), dense_view_count);
            const ViewData& d = views[v];
            if (d.dens.empty()) continue;
            const size_t p = (size_t)px[1] * W + px[0];
            const V3<R> cv{(R)d.ref_v[p].x, (R)d.ref_v[p].y, (R)d.ref_v[p].z};
            const V3<R> p0 = raw_frame ? cv : init[v].apply(cv);
            const M34<R> se3 = se3_matrix(blend(f, &dense_knn[4 * (size_t)idx], &dense_w[idx].x));
            const V3<R> wv = se3.apply(p0);
            const V3<R> vc = inv[v].apply(w2c[v].apply(wv));
            u32 pix_choice = MVDR_INVALID_INDEX;
            if (!frozen_density.empty()) {
                pix_choice = frozen_density[idx];
            } else {
                const int u = rint_even((float)(((double)vc.x / ((double)vc.z + 1e-10)) * (double)d.intr.focal_x +
                                                (double)d.intr.principal_x));
                const int vv = rint_even((float)(((double)vc.y / ((double)vc.z + 1e-10)) * (double)d.intr.focal_y +
                                                 (double)d.intr.principal_y));
                if (u >= 0 && u < (int)W && vv >= 0 && vv < (int)H) pix_choice = (u32)((size_t)vv * W + u);
            }
            float* out = &density_jr[8 * (size_t)idx];
            if (pix_choice != MVDR_INVALID_INDEX) {
                const mvdr_float4 c = d.rgb[p];
                const float geo = 0.299f * c.x + 0.587f * c.y + 0.114f * c.z;
                const R img = (R)d.dens[pix_choice];
                const R gx = (R)d.dens_grad[2 * (size_t)pix_choice], gy = (R)d.dens_grad[2 * (size_t)pix_choice + 1];
                const R fx = (R)d.intr.focal_x, fy = (R)d.intr.focal_y;
                V3<R> g;
                g.x = gx * fx / vc.z;
                g.y = gy * fy / vc.z;
                g.z = (R)(-1.0f) / (vc.z * vc.z) * (fx * vc.x * gx + fy * vc.y * gy);
                g = w2c[v].rotT(init[v].rot(g));
                out[0] = (float)(-g.y * wv.z + g.z * wv.y);
                out[1] = (float)(g.x * wv.z - g.z * wv.x);
                out[2] = (float)(-g.x * wv.y + g.y * wv.x);
                out[3] = (float)g.x; out[4] = (float)g.y; out[5] = (float)g.z;
                out[6] = (float)(img - (R)geo);
            }
            std::memcpy(&out[7], &pix_choice, 4);
        }
        // sparse feature / cross view: forwardWarpFeatureVertexKernel
        // (SparseCorrespondenceHandler.cu:202-220)
        // record: warped vertex, 1, raw residual warped - target (in R), 0
        auto warp_corr = [&](const Corr& c, u32 count, u32 base) {
            for (u32 k = 0; k < count; ++k) {
                const M34<R> se3 = se3_matrix(blend(f, &c.knn[4 * (size_t)k], &c.w[k].x));
                const V3<R> w = se3.apply(V3<R>{(R)c.ref[k].x, (R)c.ref[k].y, (R)c.ref[k].z});
                float* o = &warped[8 * (size_t)(base + k)];
                o[0] = (float)w.x; o[1] = (float)w.y; o[2] = (float)w.z; o[3] = 1.0f;
                o[4] = (float)(w.x - (R)c.target[k].x);
                o[5] = (float)(w.y - (R)c.target[k].y);
                o[6] = (float)(w.z - (R)c.target[k].z);
                o[7] = 0.0f;
            }
        };
        warp_corr(feat, Tp, 0);
        warp_corr(cross, Tc, Tp);
    }

    // computeSmoothTermJacobian (geometry_icp_jacobian.cuh:359-382) for the
    // record s (Ti xj, Tj xj, validity, 0, residual Ti xj - Tj xj, 0): the
    // rows of node i (is_i) or node j; 0 channels for an invalid edge
    static int smooth_rows(const float* s, bool is_i, double J[3][6], double r[3]) {
        if (s[6] == 0.0f) return 0;
        const double a[3] = {s[0], s[1], s[2]}, bq[3] = {s[3], s[4], s[5]};
        const double sg = is_i ? 1.0 : -1.0;
        const double* p = is_i ? a : bq;
        const double rot[3][3] = {{0, p[2], -p[1]}, {-p[2], 0, p[0]}, {p[1], -p[0], 0}};
        for (int c = 0; c < 3; ++c) {
            for (int i = 0; i < 3; ++i) J[c][i] = sg * rot[c][i];
            for (int i = 0; i < 3; ++i) J[c][3 + i] = (c == i) ? sg : 0.0;
            r[c] = s[8 + c];
        }
        return 3;
    }

    // computePointToPointICPTermJacobian / residual (geometry_icp_jacobian.cuh:50-120)
    // for the record wv (warped vertex, 1, raw residual warped - target, 0):
    // Huber-weighted rows and residuals
    static int p2p_rows(const float* wv, double J[3][6], double r[3]) {
        const float raw[3] = {wv[4], wv[5], wv[6]};
        const double rot[3][3] = {{0, wv[2], -wv[1]}, {-wv[2], 0, wv[0]}, {wv[1], -wv[0], 0}};
        for (int ch = 0; ch < 3; ++ch) {
            const double hw = huber<float>(raw[ch]);
            for (int i = 0; i < 3; ++i) J[ch][i] = hw * rot[ch][i];
            for (int i = 0; i < 3; ++i) J[ch][3 + i] = (ch == i) ? hw : 0.0;
            r[ch] = hw * raw[ch];
        }
        return 3;
    }

    // per-term weighted Jacobian rows of term `term` for node `node`:
    // returns channel count (0 invalid) and fills J[ch][6], r[ch], lambda^2
    int term_rows(u32 term, u32 node, double J[3][6], double r[3], double& lam2, double& wnode) const {
        TermType t; u32 k;
        typed(term, t, k);
        auto weight_of = [&](const u16* kn, const float* w) {
            const int o = 0 * (node == kn[0]) + 1 * (node == kn[1]) + 2 * (node == kn[2]) + 3 * (node == kn[3]);
            return (double)w[o];
        };
        switch (t) {
            case kDense:
            case kForeground: {
                const float* jr = &term_jr[8 * (size_t)(t == kDense ? k : Td + k)];
                for (int i = 0; i < 6; ++i) J[0][i] = jr[i];
                r[0] = jr[6];
                lam2 = t == kDense ? 1.0 : (double)lambda.foreground * lambda.foreground;
                wnode = weight_of(knn_of(t, k), w_of(t, k));
                if (t == kDense && !density_jr.empty() && lambda.density != 0.0f) {
                    // the density residual of the same pixel (the reference adds
                    // it in the DenseImage slot, PreconditionerBlocked.cu:216-219),
                    // as a second channel scaled by lambda_density (lam2 = 1 here)
                    const float* dj = &density_jr[8 * (size_t)k];
                    const double ld = (double)lambda.density;
                    for (int i = 0; i < 6; ++i) J[1][i] = ld * dj[i];
                    r[1] = ld * dj[6];
                    return 2;
                }
                return 1;
            }
            case kSmooth: {
                lam2 = (double)lambda.smooth * lambda.smooth;
                wnode = 1.0;
                return smooth_rows(&smooth[12 * (size_t)k], node == graph[2 * (size_t)k], J, r);
            }
            case kFeature:
            case kCross: {
                lam2 = t == kFeature ? (double)lambda.feature * lambda.feature
                                     : (double)lambda.cross_view * lambda.cross_view;
                wnode = weight_of(knn_of(t, k), w_of(t, k));
                return p2p_rows(&warped[8 * (size_t)(t == kFeature ? k : Tp + k)], J, r);
            }
            default: return 0;
        }
    }

    // diagonal blocks + damping, Jt r, preconditioner (PreconditionerBlocked.cu:172-284,
    // JtDotResidualIndexed.cu:116-224, BlockDiagonalPreconditionerInverse.cu:7-41)
    void assemble_diag() {
        D.assign(36 * (size_t)N, 0.0);
        b.assign(6 * (size_t)N, 0.0);
        for (u32 n = 0; n < N; ++n) {
            double* Dn = &D[36 * (size_t)n];
            double* bn = &b[6 * (size_t)n];
            for (u32 e = n2t_offset[n]; e < n2t_offset[n + 1]; ++e) {
                double J[3][6], r[3], lam2, w;
                const int ch = term_rows(n2t_index[e], n, J, r, lam2, w);
                for (int c = 0; c < ch; ++c) {
                    for (int i = 0; i < 6; ++i) {
                        for (int j = 0; j < 6; ++j) Dn[6 * i + j] += lam2 * (w * J[c][i]) * (w * J[c][j]);
                        bn[i] -= lam2 * w * J[c][i] * r[c];
                    }
                }
            }
            for (int i = 0; i < 6; ++i) Dn[7 * i] += (double)1e-2f;
        }
        Minv.assign(36 * (size_t)N, 0.0);
        for (u32 n = 0; n < N; ++n) {
            if (fp64) inverse_cholesky(&D[36 * (size_t)n], &Minv[36 * (size_t)n]);
            else inverse_gauss_jordan(&D[36 * (size_t)n], &Minv[36 * (size_t)n]);
        }
    }

    // DenseGaussian<6>::Inverse with pivoting (DenseGaussian.h:55-125), float
    static void inverse_gauss_jordan(const double* Din, double* out) {
        float m[36];
        for (int i = 0; i < 36; ++i) m[i] = (float)Din[i];  // column-major flatten, symmetric input
        auto fl = [](int r, int c) { return r + c * 6; };
        int perm[6] = {0, 1, 2, 3, 4, 5}, reloc[6];
        for (int i = 0; i < 6; ++i) {
            int piv = i;
            float pv = std::fabs(m[fl(i, i)]);
            for (int j = i + 1; j < 6; ++j)
                if (pv < std::fabs(m[fl(j, i)])) { pv = std::fabs(m[fl(j, i)]); piv = j; }
            for (int k = 0; k < 6; ++k) std::swap(m[fl(i, k)], m[fl(piv, k)]);
            std::swap(perm[i], perm[piv]);
            reloc[i] = perm[i];
            const float inv = 1.0f / m[fl(i, i)];
            for (int k = 0; k < 6; ++k) m[fl(i, k)] *= inv;
            m[fl(i, i)] = inv;
            for (int r = 0; r < 6; ++r) {
                if (r == i) continue;
                const float a = m[fl(r, i)];
                for (int k = 0; k < 6; ++k) m[fl(r, k)] -= a * m[fl(i, k)];
                m[fl(r, i)] = -a * m[fl(i, i)];
            }
        }
        for (int j = 0; j < 6; ++j)
            for (int i = 0; i < 6; ++i) out[6 * reloc[j] + i] = m[fl(i, j)];
    }

    static void inverse_cholesky(const double* A, double* out) {
        double L[6][6] = {};
        for (int j = 0; j < 6; ++j) {
            double s = A[6 * j + j];
            for (int k = 0; k < j; ++k) s -= L[j][k] * L[j][k];
            L[j][j] = std::sqrt(s);
            for (int i = j + 1; i < 6; ++i) {
                double t = A[6 * i + j];
                for (int k = 0; k < j; ++k) t -= L[i][k] * L[j][k];
                L[i][j] = t / L[j][j];
            }
        }
        for (int c = 0; c < 6; ++c) {
            double y[6], z[6];
            for (int i = 0; i < 6; ++i) {
                double t = (i == c) ? 1.0 : 0.0;
                for (int k = 0; k < i; ++k) t -= L[i][k] * y[k];
                y[i] = t / L[i][i];
            }
            for (int i = 5; i >= 0; --i) {
                double t = y[i];
                for (int k = i + 1; k < 6; ++k) t -= L[k][i] * z[k];
                z[i] = t / L[i][i];
            }
            for (int i = 0; i < 6; ++i) out[6 * i + c] = z[i];
        }
    }

    // off-diagonal blocks per symmetric key (JtJMaterializer.cu:270-365)
    // stored as blk[6k + r] = A(r, k), r indexing the row node's twist
    void assemble_offdiag() {
        const size_t P2 = sym_keys.size();
        offdiag.assign(36 * P2, 0.0);
        for (size_t s = 0; s < P2; ++s) {
            const u32 ni = sym_keys[s] / enc, nj = sym_keys[s] % enc;
            double* blk = &offdiag[36 * s];
            for (u32 e = ranges[2 * s]; e < ranges[2 * s + 1]; ++e) {
                const u32 term = np_index[e];
                double Ji[3][6], Jj[3][6], ri[3], rj[3], lam2, wi, wj;
                const int ch = term_rows(term, ni, Ji, ri, lam2, wi);
                term_rows(term, nj, Jj, rj, lam2, wj);
                for (int c = 0; c < ch; ++c)
                    for (int k = 0; k < 6; ++k)
                        for (int r = 0; r < 6; ++r) blk[6 * k + r] += lam2 * (wi * Ji[c][r]) * (wj * Jj[c][k]);
            }
        }
    }

    // assembleBinBlockCSRKernel (JtJMaterializerBinBlockCSR.cu:8-37)
    void assemble_binblock() {
        bbdata.assign(binnnz, 0.0);
        for (u32 row = 0; row < 6 * N; ++row) {
            int off0 = rowptr[row];
            const u32 br = row / 6, in = row % 6;
            for (int k = 0; k < 6; ++k, off0 += 32) bbdata[off0] = D[36 * (size_t)br + in + 6 * k];
            for (u32 s = blkrow_offset[br]; s < blkrow_offset[br + 1]; ++s)
                for (int k = 0; k < 6; ++k, off0 += 32) bbdata[off0] = offdiag[36 * (size_t)s + in + 6 * k];
        }
    }

    // BinBlockCSR<6>::SparseMV (BinBlockCSR.cuh:6-34), in R
    template <class R> void spmv(const std::vector<R>& xin, std::vector<R>& y) const {
        y.assign(6 * (size_t)N, (R)0);
        for (u32 row = 0; row < 6 * N; ++row) {
            int begin = rowptr[row];
            const int end = rowptr[row + 32];
            const int inbin = begin & 31;
            int col_off = (begin - inbin) / 6 + inbin;
            double acc = 0;
            while (begin < end) {
                const int col = colptr[col_off];
                for (int i = 0; i < 6; ++i) {
                    const double a = bbdata[begin];
                    const double xv = col >= 0 ? (double)xin[col + i] : 0.0;
                    acc += a * xv;
                    begin += 32;
                }
                col_off += 32;
            }
            y[row] = (R)acc;
        }
    }

    // BlockPCG<6>::SolveNoConvergeCheck (BlockPCG.cuh:65-181, 317-335)
    template <class R> void pcg_t(u32 iters) {
        const size_t n = 6 * (size_t)N;
        std::vector<R> r(n), d(n), q(n), s(n), t(n), xx(n, (R)0), Mi(36 * (size_t)N), bb(n);
        for (size_t i = 0; i < Mi.size(); ++i) Mi[i] = (R)Minv[i];
        for (size_t i = 0; i < n; ++i) bb[i] = (R)b[i];
        auto precond = [&](const std::vector<R>& in, std::vector<R>& out) {
            for (u32 nd = 0; nd < N; ++nd)
                for (int j = 0; j < 6; ++j) {
                    double acc = 0;
                    for (int i = 0; i < 6; ++i) acc += (double)Mi[36 * (size_t)nd + 6 * j + i] * (double)in[6 * nd + i];
                    out[6 * nd + j] = (R)acc;
                }
        };
        auto vdot = [&](const std::vector<R>& a, const std::vector<R>& c) {
            double acc = 0;
            for (size_t i = 0; i < n; ++i) acc += (double)a[i] * (double)c[i];
            return (R)acc;
        };
        r = bb;
        precond(r, d);
        R delta = vdot(r, d);
        const R delta0 = delta;
        const double tol2 = (double)cfg.pcg_tolerance * (double)cfg.pcg_tolerance;
        pcg_history.clear();
        for (u32 it = 0; it < iters; ++it) {
            // SolveConvergeChecked (BlockPCG.cuh:339-377): delta at the start of
            // each iteration against tol^2 delta_0
            pcg_history.push_back((double)delta);
            if (it > 0 && cfg.pcg_tolerance > 0.0f && std::fabs((double)delta) < tol2 * std::fabs((double)delta0))
                break;
            spmv<R>(d, q);
            const R dq = vdot(d, q);
            // a zero d.q (a right-hand side that is exactly zero) gives a zero
            // step where the reference would divide 0 by 0
            const R alpha = dq != (R)0 ? delta / dq : (R)0;
            for (size_t i = 0; i < n; ++i) { xx[i] += alpha * d[i]; t[i] = r[i] - alpha * q[i]; }
            precond(t, s);
            const R delta_old = delta;
            delta = vdot(t, s);
            const R beta = delta_old != (R)0 ? delta / delta_old : (R)0;
            for (size_t i = 0; i < n; ++i) d[i] = s[i] + beta * d[i];
            std::swap(r, t);
        }
        x.assign(n, 0.0);
        for (size_t i = 0; i < n; ++i) x[i] = (double)xx[i];
    }

    void update() {
        for (u32 i = 0; i < N; ++i) {
            if (fp64) {
                const double tw[6] = {x[6 * i], x[6 * i + 1], x[6 * i + 2], x[6 * i + 3], x[6 * i + 4], x[6 * i + 5]};
                se3d[i] = apply_twist<double>(se3d[i], tw);
            } else {
                const float tw[6] = {(float)x[6 * i], (float)x[6 * i + 1], (float)x[6 * i + 2],
                                     (float)x[6 * i + 3], (float)x[6 * i + 4], (float)x[6 * i + 5]};
                const DQ<double>& o = se3d[i];
                const DQ<float> p{{(float)o.q0.x, (float)o.q0.y, (float)o.q0.z, (float)o.q0.w},
                                  {(float)o.q1.x, (float)o.q1.y, (float)o.q1.z, (float)o.q1.w}};
                const DQ<float> n2 = apply_twist<float>(p, tw);
                se3d[i] = {{n2.q0.x, n2.q0.y, n2.q0.z, n2.q0.w}, {n2.q1.x, n2.q1.y, n2.q1.z, n2.q1.w}};
            }
        }
        gn_iter++;
    }

    // computeTermResidualKernel (ResidualEvaluator.cu:71-142), squared, summed in double
    double compute_energy() const {
        double e = 0;
        for (u32 k = 0; k < Td; ++k) { const double r = term_jr[8 * (size_t)k + 6]; e += r * r; }
        for (size_t k = 0; k < density_jr.size() / 8; ++k) {  // ResidualEvaluator.cu:94-99
            const double r = (double)(lambda.density * density_jr[8 * k + 6]);
            e += r * r;
        }
        for (u32 k = 0; k < Ts; ++k) {
            const float* s = &smooth[12 * (size_t)k];
            if (s[6] == 0.0f) continue;
            for (int c = 0; c < 3; ++c) { const double r = (double)lambda.smooth * s[8 + c]; e += r * r; }
        }
        for (u32 k = 0; k < Tf; ++k) {
            const double r = (double)lambda.foreground * term_jr[8 * (size_t)(Td + k) + 6];
            e += r * r;
        }
        auto p2p = [&](const Corr& c, u32 count, u32 base, float lam) {
            for (u32 k = 0; k < count; ++k) {
                const float* wv = &warped[8 * (size_t)(base + k)];
                (void)c;
                const float raw[3] = {wv[4], wv[5], wv[6]};
                for (int ch = 0; ch < 3; ++ch) {
                    const double r = (double)lam * (huber<float>(raw[ch]) * raw[ch]);
                    e += r * r;
                }
            }
        };
        p2p(feat, Tp, 0, lambda.feature);
        p2p(cross, Tc, Tp, lambda.cross_view);
        return e;
    }

    void gn_prepare() {
        penalty_for(gn_iter);
        if (fp64) eval_terms_t<double>(); else eval_terms_t<float>();
    }
    void gn_assemble() {
        assemble_diag();
        assemble_offdiag();
        assemble_binblock();
        energy = compute_energy();
    }
    void gn_solve(u32 pcg) {
        if (fp64) pcg_t<double>(pcg); else pcg_t<float>(pcg);
    }
};

}  // namespace

// ------------------------------------------------------------- C entry ---
extern "C" {

void* orc_create(const mvdr_config* cfg, const mvdr_inputs* host_inputs, int fp64) {
    Oracle* o = new Oracle();
    o->fp64 = fp64;
    if (o->set_inputs(cfg, host_inputs) != MVDR_OK) { delete o; return nullptr; }
    return o;
}
void orc_destroy(void* h) { delete (Oracle*)h; }

void orc_build_index(void* h) { ((Oracle*)h)->build_index(); }

/* delta at the start of each PCG iteration of the last PCG solve (delta_0
 * first); returns how many, copying at most `cap`. */
uint32_t orc_pcg_history(void* h, double* out, uint32_t cap) {
    const Oracle* o = (const Oracle*)h;
    const uint32_t n = (uint32_t)o->pcg_history.size();
    for (uint32_t k = 0; k < n && k < cap; ++k) out[k] = o->pcg_history[k];
    return n;
}

/* The feature terms as bound or selected from raw pixel pairs: returns their
 * count and, when the pointers are not NULL, copies target, reference,
 * ushort4 knn and weights. */
uint32_t orc_feature_terms(void* h, mvdr_float4* target, mvdr_float4* ref, uint16_t* knn, mvdr_float4* w) {
    const Oracle* o = (const Oracle*)h;
    const size_t n = o->feat.w.size();
    if (target) std::memcpy(target, o->feat.target.data(), 16 * n);
    if (ref) std::memcpy(ref, o->feat.ref.data(), 16 * n);
    if (knn) std::memcpy(knn, o->feat.knn.data(), 8 * n);
    if (w) std::memcpy(w, o->feat.w.data(), 16 * n);
    return (uint32_t)n;
}

/* Evaluate the terms of the current Gauss-Newton iteration (penalty schedule
 * of that iteration included). */
void orc_eval_terms(void* h) { ((Oracle*)h)->gn_prepare(); }

/* Replace the evaluated term data by another run's (ABI float layouts). */
void orc_set_term_data(void* h, const float* term_jr, const float* smooth, const float* warped) {
    Oracle* o = (Oracle*)h;
    if (term_jr) std::memcpy(o->term_jr.data(), term_jr, o->term_jr.size() * 4);
    if (smooth) std::memcpy(o->smooth.data(), smooth, o->smooth.size() * 4);
    if (warped) std::memcpy(o->warped.data(), warped, o->warped.size() * 4);
}

/* Freeze the discrete choices of the term evaluation: per dense+foreground
 * term the projected pixel (or 0xFFFFFFFF), per smooth term the validity. */
void orc_freeze_decisions(void* h, const uint32_t* pixels, const uint8_t* smooth_valid) {
    Oracle* o = (Oracle*)h;
    o->frozen_pixel.assign(pixels, pixels + (o->Td + o->Tf));
    o->frozen_smooth.assign(smooth_valid, smooth_valid + o->Ts);
    o->frozen = true;
}
void orc_unfreeze(void* h) {
    ((Oracle*)h)->frozen = false;
    ((Oracle*)h)->frozen_density.clear();
}

/* Freeze the density term's projected pixels (one per dense term). */
void orc_freeze_density(void* h, const uint32_t* pixels) {
    Oracle* o = (Oracle*)h;
    o->frozen_density.assign(pixels, pixels + o->Td);
}

void orc_assemble(void* h) { ((Oracle*)h)->gn_assemble(); }
void orc_pcg(void* h, uint32_t iters) { ((Oracle*)h)->gn_solve(iters); }
void orc_set_increment(void* h, const float* x) {
    Oracle* o = (Oracle*)h;
    o->x.assign(x, x + 6 * (size_t)o->N);
}
void orc_update(void* h) { ((Oracle*)h)->update(); }

/* Replace the current warp field (num_nodes dual quaternions, float). */
void orc_set_node_se3(void* h, const float* dq) {
    Oracle* o = (Oracle*)h;
    for (uint32_t i = 0; i < o->N; ++i) {
        const float* d = dq + 8 * (size_t)i;
        o->se3d[i] = {{d[0], d[1], d[2], d[3]}, {d[4], d[5], d[6], d[7]}};
    }
}

/* Replace the current warp field with double-precision dual quaternions
 * (finite-difference checks perturb the field below float resolution). */
void orc_set_node_se3_f64(void* h, const double* dq) {
    Oracle* o = (Oracle*)h;
    for (uint32_t i = 0; i < o->N; ++i) {
        const double* d = dq + 8 * (size_t)i;
        o->se3d[i] = {{d[0], d[1], d[2], d[3]}, {d[4], d[5], d[6], d[7]}};
    }
}

/* One full Gauss-Newton iteration. */
void orc_gn_iteration(void* h, uint32_t pcg) {
    Oracle* o = (Oracle*)h;
    o->gn_prepare();
    o->gn_assemble();
    o->gn_solve(pcg);
    o->update();
}
void orc_solve(void* h, uint32_t gn, uint32_t pcg) {
    Oracle* o = (Oracle*)h;
    o->build_index();
    for (uint32_t k = 0; k < gn; ++k) orc_gn_iteration(h, pcg);
}

double orc_energy(void* h) { return ((Oracle*)h)->energy; }
double orc_energy_now(void* h) { return ((Oracle*)h)->compute_energy(); }

void orc_counts(void* h, mvdr_counts* c) {
    Oracle* o = (Oracle*)h;
    std::memset(c, 0, sizeof(*c));
    c->dense_terms = o->Td; c->smooth_terms = o->Ts; c->foreground_terms = o->Tf;
    c->feature_terms = o->Tp; c->cross_terms = o->Tc;
    c->node2term_entries = (uint32_t)o->n2t_index.size();
    c->nodepair_entries = (uint32_t)o->np_index.size();
    c->half_pairs = (uint32_t)o->half_keys.size();
    c->num_bins = o->nbins;
    c->binblock_nnz = o->binnnz;
}

/* Copy array `which` (mvdr_get_array ids). Real-valued arrays are written as
 * float unless `as_double` is set. Returns bytes written or -1. */
long long orc_get(void* h, int which, void* dst, size_t cap, int as_double) {
    Oracle* o = (Oracle*)h;
    auto put = [&](const void* src, size_t bytes) -> long long {
        if (bytes > cap) return -1;
        if (bytes) std::memcpy(dst, src, bytes);
        return (long long)bytes;
    };
    auto put_real = [&](const std::vector<double>& v) -> long long {
        if (as_double) return put(v.data(), v.size() * 8);
        if (v.size() * 4 > cap) return -1;
        float* f = (float*)dst;
        for (size_t i = 0; i < v.size(); ++i) f[i] = (float)v[i];
        return (long long)(v.size() * 4);
    };
    switch (which) {
        case MVDR_ARRAY_DENSE_PIXELS: return put(o->dense_pix.data(), o->dense_pix.size() * 2);
        case MVDR_ARRAY_DENSE_KNN: return put(o->dense_knn.data(), o->dense_knn.size() * 2);
        case MVDR_ARRAY_DENSE_KNN_WEIGHT: return put(o->dense_w.data(), o->dense_w.size() * 16);
        case MVDR_ARRAY_FOREGROUND_PIXELS: return put(o->fg_pix.data(), o->fg_pix.size() * 2);
        case MVDR_ARRAY_NODE2TERM_OFFSET: return put(o->n2t_offset.data(), o->n2t_offset.size() * 4);
        case MVDR_ARRAY_NODE2TERM_INDEX: return put(o->n2t_index.data(), o->n2t_index.size() * 4);
        case MVDR_ARRAY_HALF_NODEPAIR_KEY: return put(o->half_keys.data(), o->half_keys.size() * 4);
        case MVDR_ARRAY_NODEPAIR_TERM_INDEX: return put(o->np_index.data(), o->np_index.size() * 4);
        case MVDR_ARRAY_NODEPAIR_KEY: return put(o->sym_keys.data(), o->sym_keys.size() * 4);
        case MVDR_ARRAY_NODEPAIR_TERM_RANGE: return put(o->ranges.data(), o->ranges.size() * 4);
        case MVDR_ARRAY_BLKROW_OFFSET: return put(o->blkrow_offset.data(), o->blkrow_offset.size() * 4);
        case MVDR_ARRAY_BINBLOCK_ROWPTR: return put(o->rowptr.data(), o->rowptr.size() * 4);
        case MVDR_ARRAY_BINBLOCK_COLPTR: return put(o->colptr.data(), o->colptr.size() * 4);
        case MVDR_ARRAY_TERM_JACOBIAN: return put(o->term_jr.data(), o->term_jr.size() * 4);
        case MVDR_ARRAY_DENSITY_JACOBIAN: return put(o->density_jr.data(), o->density_jr.size() * 4);
        case MVDR_ARRAY_FEATURE_TERMS: {
            std::vector<mvdr_float4> tr;
            for (size_t k = 0; k < o->feat.w.size(); ++k) {
                tr.push_back(o->feat.target[k]);
                tr.push_back(o->feat.ref[k]);
            }
            return put(tr.data(), tr.size() * 16);
        }
        case MVDR_ARRAY_SMOOTH_TERMS: return put(o->smooth.data(), o->smooth.size() * 4);
        case MVDR_ARRAY_WARPED_CORRESPONDENCE: return put(o->warped.data(), o->warped.size() * 4);
        case MVDR_ARRAY_DIAG_BLOCKS: return put_real(o->D);
        case MVDR_ARRAY_JTR: return put_real(o->b);
        case MVDR_ARRAY_PRECONDITIONER: return put_real(o->Minv);
        case MVDR_ARRAY_OFFDIAG_BLOCKS: return put_real(o->offdiag);
        case MVDR_ARRAY_BINBLOCK_DATA: return put_real(o->bbdata);
        case MVDR_ARRAY_INCREMENT: return put_real(o->x);
        case MVDR_ARRAY_NODE_SE3: {
            std::vector<double> v(8 * (size_t)o->N);
            for (uint32_t i = 0; i < o->N; ++i) {
                const auto& d = o->se3d[i];
                const double a[8] = {d.q0.x, d.q0.y, d.q0.z, d.q0.w, d.q1.x, d.q1.y, d.q1.z, d.q1.w};
                for (int k = 0; k < 8; ++k) v[8 * (size_t)i + k] = a[k];
            }
            return put_real(v);
        }
        default: return -1;
    }
}

/* y = A x with the assembled bin-block operator (double). */
void orc_apply_jtj(void* h, const double* xin, double* y) {
    Oracle* o = (Oracle*)h;
    std::vector<double> xv(xin, xin + 6 * (size_t)o->N), yv;
    o->spmv<double>(xv, yv);
    std::memcpy(y, yv.data(), yv.size() * 8);
}

/* Known-answer helpers over the restated math. */
/* DualQuaternion::operator mat34 (DualQuaternion.h:309-319) in float. */
void orc_dq_to_mat34(const float* dq8, float* m12) {
    const DQ<float> d{{dq8[0], dq8[1], dq8[2], dq8[3]}, {dq8[4], dq8[5], dq8[6], dq8[7]}};
    const M34<float> m = dq_to_mat34(d);
    for (int c = 0; c < 3; ++c)
        for (int r = 0; r < 3; ++r) m12[3 * c + r] = m.m[r][c];
    for (int r = 0; r < 3; ++r) m12[9 + r] = m.t[r];
}
void orc_mat34_to_dq(const float* m12, float* dq8) {
    M34<float> m;
    for (int c = 0; c < 3; ++c)
        for (int r = 0; r < 3; ++r) m.m[r][c] = m12[3 * c + r];
    for (int r = 0; r < 3; ++r) m.t[r] = m12[9 + r];
    const DQ<float> d = mat34_to_dq(m);
    const float a[8] = {d.q0.x, d.q0.y, d.q0.z, d.q0.w, d.q1.x, d.q1.y, d.q1.z, d.q1.w};
    std::memcpy(dq8, a, 32);
}
void orc_apply_twist(const double* dq8, const double* tw6, double* out8) {
    const DQ<double> d{{dq8[0], dq8[1], dq8[2], dq8[3]}, {dq8[4], dq8[5], dq8[6], dq8[7]}};
    const DQ<double> n = apply_twist<double>(d, tw6);
    const double a[8] = {n.q0.x, n.q0.y, n.q0.z, n.q0.w, n.q1.x, n.q1.y, n.q1.z, n.q1.w};
    std::memcpy(out8, a, 64);
}
void orc_gauss_jordan_inverse(const double* A36, double* out36) { Oracle::inverse_gauss_jordan(A36, out36); }

/* ---- after the solve (the oracle's restatement of csrc/deform.cu) ------- */

// __float2int_rn / __float2uint_rn: round to nearest even, NaN -> 0,
// saturating at the type's range
static int f2i_rn_sat(float v) {
    if (v != v) return 0;
    if (v >= 2147483648.0f) return 2147483647;
    if (v < -2147483648.0f) return (-2147483647 - 1);
    return (int)std::nearbyint(v);
}
static uint32_t f2u_rn_sat(float v) {
    if (v != v) return 0;
    if (v >= 4294967296.0f) return 0xFFFFFFFFu;
    const float r = std::nearbyint(v);
    return r <= 0.0f ? 0u : (uint32_t)r;
}

static M34<float> normalized_se3(DQ<float> d, DQ<float>* normalized_out = nullptr) {
    const float inv = 1.0f / std::sqrt(qdot(d.q0, d.q0));
    d.q0 = qscale(inv, d.q0);
    d.q1 = qscale(inv, d.q1);
    const float dd = qdot(d.q0, d.q1);
    d.q1 = {d.q1.x - dd * d.q0.x, d.q1.y - dd * d.q0.y, d.q1.z - dd * d.q0.z, d.q1.w - dd * d.q0.w};
    if (normalized_out) *normalized_out = d;
    const Q<float> q = d.q0;
    M34<float> m;  // Quaternion::rotation_matrix(false), Quaternion.h:207-220
    m.m[0][0] = 1 - 2 * q.y * q.y - 2 * q.z * q.z;
    m.m[0][1] = 2 * q.x * q.y - 2 * q.z * q.w;
    m.m[0][2] = 2 * q.x * q.z + 2 * q.y * q.w;
    m.m[1][0] = 2 * q.x * q.y + 2 * q.z * q.w;
    m.m[1][1] = 1 - 2 * q.x * q.x - 2 * q.z * q.z;
    m.m[1][2] = 2 * q.y * q.z - 2 * q.x * q.w;
    m.m[2][0] = 2 * q.x * q.z - 2 * q.y * q.w;
    m.m[2][1] = 2 * q.y * q.z + 2 * q.x * q.w;
    m.m[2][2] = 1 - 2 * q.x * q.x - 2 * q.y * q.y;
    const Q<float> tp = qmul(qscale(2.0f, d.q1), qconj(d.q0));
    m.t[0] = tp.x;
    m.t[1] = tp.y;
    m.t[2] = tp.z;
    return m;
}

static DQ<float> blend_f(const mvdr_dual_quaternion* field, const uint16_t* knn, const mvdr_float4& w) {
    const float ws[4] = {w.x, w.y, w.z, w.w};
    DQ<float> a;
    for (int k = 0; k < 4; ++k) {
        const DQ<float> d = load_dq<float>(field[knn[k]]);
        const float s = ws[k];
        if (k == 0) {
            a.q0 = qscale(s, d.q0);
            a.q1 = qscale(s, d.q1);
        } else {
            a.q0 = {a.q0.x + s * d.q0.x, a.q0.y + s * d.q0.y, a.q0.z + s * d.q0.z, a.q0.w + s * d.q0.w};
            a.q1 = {a.q1.x + s * d.q1.x, a.q1.y + s * d.q1.y, a.q1.z + s * d.q1.z, a.q1.w + s * d.q1.w};
        }
    }
    return a;
}

static bool knn_in(const uint16_t* k, uint32_t n) { return k[0] < n && k[1] < n && k[2] < n && k[3] < n; }

static M34<float> mul34f(const M34<float>& a, const M34<float>& b) {  // mat34::operator*
    M34<float> o;
    for (int r = 0; r < 3; ++r) {
        for (int c = 0; c < 3; ++c) o.m[r][c] = a.m[r][0] * b.m[0][c] + a.m[r][1] * b.m[1][c] + a.m[r][2] * b.m[2][c];
        o.t[r] = (a.m[r][0] * b.t[0] + a.m[r][1] * b.t[1] + a.m[r][2] * b.t[2]) + a.t[r];
    }
    return o;
}

/* SurfelNodeDeformer::ForwardWarpSurfelsAndNodes (SurfelNodeDeformer.cu:9-57):
 * HOST arrays. */
void orc_forward_warp(const mvdr_dual_quaternion* field, uint32_t num_field, uint32_t S, const uint16_t* knn,
                      const mvdr_float4* w, const mvdr_float4* in_v, const mvdr_float4* in_n, mvdr_float4* out_v,
                      mvdr_float4* out_n, uint32_t N, const uint16_t* node_knn, const mvdr_float4* node_w,
                      const mvdr_float4* nodes, mvdr_float4* live_nodes) {
    const float nan = std::numeric_limits<float>::quiet_NaN();
    for (uint32_t i = 0; i < S + N; ++i) {
        const bool surfel = i < S;
        const uint32_t k = surfel ? i : i - S;
        const uint16_t* kk = surfel ? knn + 4 * (size_t)k : node_knn + 4 * (size_t)k;
        const mvdr_float4 ww = surfel ? w[k] : node_w[k];
        const mvdr_float4 v = surfel ? in_v[k] : nodes[k];
        const mvdr_float4 n = surfel ? in_n[k] : mvdr_float4{0, 0, 0, 0};
        mvdr_float4 ov{nan, nan, nan, v.w}, on{nan, nan, nan, n.w};
        if (knn_in(kk, num_field)) {
            const M34<float> se3 = normalized_se3(blend_f(field, kk, ww));
            const V3<float> p = se3.apply({v.x, v.y, v.z}), q = se3.rot({n.x, n.y, n.z});
            ov = {p.x, p.y, p.z, v.w};
            on = {q.x, q.y, q.z, n.w};
        }
        if (surfel) {
            out_v[k] = ov;
            out_n[k] = on;
        } else {
            live_nodes[k] = ov;
        }
    }
}

/* SurfelNodeDeformer::InverseWarpSurfels (SurfelNodeDeformer.cu:63-119):
 * HOST arrays; correct may be NULL. */
void orc_inverse_warp(const mvdr_dual_quaternion* field, uint32_t num_field, const mvdr_mat34* correct, uint32_t S,
                      const uint16_t* knn, const mvdr_float4* w, const mvdr_float4* in_v, const mvdr_float4* in_n,
                      mvdr_float4* out_v, mvdr_float4* out_n) {
    const float nan = std::numeric_limits<float>::quiet_NaN();
    for (uint32_t i = 0; i < S; ++i) {
        const mvdr_float4 v = in_v[i], n = in_n[i];
        V3<float> p{nan, nan, nan}, q = p;
        if (knn_in(knn + 4 * (size_t)i, num_field)) {
            const M34<float> se3 = normalized_se3(blend_f(field, knn + 4 * (size_t)i, w[i]));
            p = se3.rotT({v.x - se3.t[0], v.y - se3.t[1], v.z - se3.t[2]});
            q = se3.rotT({n.x, n.y, n.z});
            if (correct) {
                const M34<float> ci = inverse34(load_mat34<float>(correct[i]));
                p = ci.apply(p);
                q = ci.rot(q);
            }
        }
        out_v[i] = {p.x, p.y, p.z, v.w};
        out_n[i] = {q.x, q.y, q.z, n.w};
    }
}

static bool zero_vertex_f(const mvdr_float4& v) {
    return (double)std::fabs(v.x) < 1e-3 && (double)std::fabs(v.y) < 1e-3 && (double)std::fabs(v.z) < 1e-3;
}

static uint64_t to_fixed_f(float v) {
    float s = v * 4294967296.0f;
    if (s != s) s = 0.0f;
    s = std::fmin(std::fmax(s, -4.611686e18f), 4.611686e18f);
    return (uint64_t)(int64_t)std::llrint(s);
}

/* DenseDepthHandler::ComputeNodewiseError, ComputeAlignmentErrorMapDirect and
 * ComputeAlignmentErrorMapFromNode (DenseDepthAlignmentError.cu:16-238) on
 * HOST inputs: `in` with host map pointers (rows `pitch` or W apart), the
 * warp field `field` (in->num_nodes dual quaternions). Node sums in 2^-32
 * fixed point. Maps (optional, W x H) per view. */
void orc_node_error(const mvdr_inputs* in, uint32_t W, uint32_t H, const mvdr_dual_quaternion* field, float threshold,
                    float* acc_error, float* acc_weight, float* united, uint32_t* mark, float* const* align_maps,
                    float* const* node_maps) {
    const uint32_t N = in->num_nodes, S = in->num_surfels;
    std::vector<uint64_t> acc(2 * (size_t)N, 0);
    const uint16_t* sk = in->surfel_knn;
    for (uint32_t v = 0; v < in->num_views; ++v) {
        const mvdr_view_inputs& vi = in->views[v];
        const uint32_t pitch = vi.pitch ? vi.pitch : W;
        const M34<float> w2c = load_mat34<float>(vi.world2camera), init = load_mat34<float>(vi.initial_camera_se3);
        const M34<float> iinv = inverse34(init);
        for (uint32_t y = 0; y < H; ++y)
            for (uint32_t x = 0; x < W; ++x) {
                const size_t o = (size_t)y * pitch + x;
                float err = 0.0f;
                const uint32_t s = vi.index_map[o];
                const uint16_t* kk = nullptr;
                mvdr_float4 ww{0, 0, 0, 0};
                if (s != MVDR_INVALID_INDEX && s < S && knn_in(sk + 4 * (size_t)s, N)) {
                    kk = sk + 4 * (size_t)s;
                    ww = in->surfel_knn_weight[s];
                    const mvdr_float4 rv = vi.reference_vertex_map[o], rn = vi.reference_normal_map[o];
                    const V3<float> cv = init.apply({rv.x, rv.y, rv.z}), cn = init.rot({rn.x, rn.y, rn.z});
                    const M34<float> se3 = normalized_se3(blend_f(field, kk, ww));
                    const V3<float> wv = se3.apply(cv), wn = se3.rot(cn);
                    const V3<float> c1 = iinv.apply(w2c.apply(wv)), n1 = iinv.rot(w2c.rot(wn));
                    const mvdr_intrinsic& K = vi.intrinsic;
                    int ix = f2i_rn_sat((float)(((double)c1.x / ((double)c1.z + 1e-10)) * (double)K.focal_x +
                                                (double)K.principal_x));
                    int iy = f2i_rn_sat((float)(((double)c1.y / ((double)c1.z + 1e-10)) * (double)K.focal_y +
                                                (double)K.principal_y));
                    ix = std::min(std::max(ix, -2), (int)W + 1);
                    iy = std::min(std::max(iy, -2), (int)H + 1);
                    err = 0.1f;
                    bool found = false;
                    for (int dy = iy - 1; dy <= iy + 1; ++dy)
                        for (int dx = ix - 1; dx <= ix + 1; ++dx) {
                            mvdr_float4 dv{0, 0, 0, 0}, dn{0, 0, 0, 0};
                            if (dx >= 0 && dy >= 0 && dx < (int)W && dy < (int)H) {
                                dv = vi.vertex_confidence_map[(size_t)dy * pitch + dx];
                                dn = vi.normal_radius_map[(size_t)dy * pitch + dx];
                            }
                            if (!zero_vertex_f(dv) && (n1.x * dn.x + n1.y * dn.y + n1.z * dn.z) > 0.7f) found = true;
                            const float e = std::fabs(c1.x - dv.x) + std::fabs(c1.y - dv.y) + std::fabs(c1.z - dv.z);
                            if (e < err) err = e;
                        }
                    if (!found) {
                        float fg = 0.0f;
                        if (ix >= 0 && iy >= 0 && ix < (int)W && iy < (int)H)
                            fg = vi.filtered_foreground_mask[(size_t)iy * pitch + ix];
                        err = fg < 0.9f ? 0.03f * fg : 0.1f;
                    }
                }
                if (align_maps && align_maps[v]) align_maps[v][(size_t)y * W + x] = err;
                if (err > 1e-6f) {
                    const float wk[4] = {ww.x, ww.y, ww.z, ww.w};
                    for (int k = 0; k < 4; ++k) {
                        acc[kk[k]] += to_fixed_f(wk[k] * err);
                        acc[N + kk[k]] += to_fixed_f(wk[k]);
                    }
                }
            }
    }
    for (uint32_t n = 0; n < N; ++n) {
        const float e = (float)((double)(int64_t)acc[n] * (1.0 / 4294967296.0));
        const float w = (float)((double)(int64_t)acc[N + n] * (1.0 / 4294967296.0));
        float u = (e / (w + 1e-4f)) / 0.1f;
        uint32_t m = u > threshold ? 1u : 0u;
        if (e < 1e-10f) {
            m = 1u;
            u = 1.0f;
        }
        acc_error[n] = e;
        acc_weight[n] = w;
        united[n] = u;
        mark[n] = m;
    }
    if (!node_maps) return;
    for (uint32_t v = 0; v < in->num_views; ++v) {
        if (!node_maps[v]) continue;
        const mvdr_view_inputs& vi = in->views[v];
        const uint32_t pitch = vi.pitch ? vi.pitch : W;
        for (uint32_t y = 0; y < H; ++y)
            for (uint32_t x = 0; x < W; ++x) {
                const uint32_t s = vi.index_map[(size_t)y * pitch + x];
                float f = 0.0f;
                if (s != MVDR_INVALID_INDEX && s < S && knn_in(sk + 4 * (size_t)s, N)) {
                    const uint16_t* kk = sk + 4 * (size_t)s;
                    const mvdr_float4 ww = in->surfel_knn_weight[s];
                    const float wk[4] = {ww.x, ww.y, ww.z, ww.w};
                    float ae = 0.0f, aw = 0.0f;
                    for (int k = 0; k < 4; ++k) {
                        const float unit = acc_error[kk[k]] / acc_weight[kk[k]];
                        ae += unit * wk[k];
                        aw += wk[k];
                    }
                    f = ae / (aw + 1e-4f);
                }
                node_maps[v][(size_t)y * W + x] = f;
            }
    }
}

/* NonRigidSolver::CorrectLargeErrorNode, correspondence form
 * (NonRigidSolver.cu:93-227): cameras from `in` (host), every array of `c`
 * HOST memory; c->node_se3 must be given (corrected in place). */
void orc_correct_large_error_nodes(const mvdr_inputs* in, float node_radius, const mvdr_correction* c) {
    const uint32_t N = in->num_nodes, V = in->num_views;
    const float nan = std::numeric_limits<float>::quiet_NaN();
    const float four_r2 = 4.0f * node_radius * node_radius;
    std::vector<DQ<float>> corr(N);
    for (uint32_t n = 0; n < N; ++n) {
        DQ<float> d{{0, 0, 0, 1}, {0, 0, 0, 0}};
        const float err = c->united_error[n];
        if (err > c->error_threshold) {
            const mvdr_float4 node = c->live_nodes[n];
            int view = -1;
            for (uint32_t i = 0; i < V; ++i)
                if ((float)i < node.w && node.w <= (float)(i + 1)) { view = (int)i; break; }
            if (view >= 0) {
                const mvdr_view_inputs& vi = in->views[view];
                const mvdr_correction_view& g = c->views[view];
                const uint32_t pitch = g.pitch ? g.pitch : c->width;
                const M34<float> w2c = load_mat34<float>(vi.world2camera), init = load_mat34<float>(vi.initial_camera_se3);
                const M34<float> iinv = inverse34(init);
                const V3<float> cc = iinv.apply(w2c.apply({node.x, node.y, node.z}));
                const mvdr_intrinsic& K = vi.intrinsic;
                const uint32_t ux = f2u_rn_sat((float)(((double)cc.x / ((double)cc.z + 1e-10)) * (double)K.focal_x +
                                                       (double)K.principal_x));
                const uint32_t uy = f2u_rn_sat((float)(((double)cc.y / ((double)cc.z + 1e-10)) * (double)K.focal_y +
                                                       (double)K.principal_y));
                M34<float> sel;
                for (int r = 0; r < 3; ++r) {
                    for (int k = 0; k < 3; ++k) sel.m[r][k] = r == k ? 1.0f : 0.0f;
                    sel.t[r] = 0.0f;
                }
                const uint32_t h = 2;
                if (!(ux >= c->width - h || ux < h || uy >= c->height - h || uy < h)) {
                    float best = 1e6f;
                    for (uint32_t i = ux - h; i <= ux + h; ++i)
                        for (uint32_t j = uy - h; j <= uy + h; ++j) {
                            const size_t o = (size_t)j * pitch + i;
                            const mvdr_float4 pv = g.previous_vertex_map[o];
                            if (g.valid_map[o] == 1 && !zero_vertex_f(pv)) {
                                const M34<float> gm = load_mat34<float>(g.se3_map[o]);
                                const float dx = cc.x - pv.x, dy = cc.y - pv.y, dz = cc.z - pv.z;
                                const float dist = dx * dx + dy * dy + dz * dz;
                                const V3<float> mv = gm.apply(cc);
                                const float ex = mv.x - cc.x, ey = mv.y - cc.y, ez = mv.z - cc.z;
                                if (best > dist && dist < 1e-4f && (ex * ex + ey * ey + ez * ez) < four_r2) {
                                    best = dist;
                                    sel = gm;
                                }
                            }
                        }
                    sel = mul34f(mul34f(mul34f(mul34f(inverse34(w2c), init), sel), iinv), w2c);
                }
                // DualQuaternion(mat34), then operator*(float) via Quaternion::pow
                const DQ<float> m = mat34_to_dq(sel);
                float t = err;
                if (t > 1.0f) t = 1.0f;
                else if (t < 1e-10f) t = 1e-10f;
                const Q<float> q0 = m.q0;
                const float norm = std::sqrt(q0.x * q0.x + q0.y * q0.y + q0.z * q0.z);
                const float nt = std::atan2(norm, q0.w) * t;
                const float sn = std::sin(nt);
                Q<float> p;
                if (std::fabs(norm) < 1e-6f) {
                    p = {0.0f, 0.0f, 0.0f, std::cos(nt)};
                } else {
                    const float scale = sn / norm;
                    p = {q0.x * scale, q0.y * scale, q0.z * scale, std::cos(nt)};
                }
                d.q0 = p;
                d.q1 = qmul(qscale(t, qmul(m.q1, qconj(q0))), p);
            }
        }
        corr[n] = d;
        c->correction[n] = {{d.q0.x, d.q0.y, d.q0.z, d.q0.w}, {d.q1.x, d.q1.y, d.q1.z, d.q1.w}};
    }
    const uint32_t S = c->num_surfels;
    for (uint32_t i = 0; i < S + N; ++i) {
        const bool surfel = i < S;
        const uint32_t k = surfel ? i : i - S;
        const uint16_t* kk = surfel ? c->surfel_knn + 4 * (size_t)k : c->node_knn + 4 * (size_t)k;
        const mvdr_float4 ww = surfel ? c->surfel_knn_weight[k] : c->node_knn_weight[k];
        const mvdr_float4 v = surfel ? c->live_vertex[k] : c->live_nodes[k];
        const mvdr_float4 nr = surfel ? c->live_normal[k] : mvdr_float4{0, 0, 0, 0};
        mvdr_float4 ov{nan, nan, nan, v.w}, on{nan, nan, nan, nr.w};
        const bool ok = knn_in(kk, N);
        DQ<float> avg{};
        if (ok) {
            const M34<float> se3 = normalized_se3(blend_f(c->correction, kk, ww), &avg);
            const V3<float> p = se3.apply({v.x, v.y, v.z}), q = se3.rot({nr.x, nr.y, nr.z});
            ov = {p.x, p.y, p.z, v.w};
            on = {q.x, q.y, q.z, nr.w};
        }
        if (surfel) {
            c->live_vertex[k] = ov;
            c->live_normal[k] = on;
            continue;
        }
        c->live_nodes[k] = ov;
        mvdr_dual_quaternion& f = c->node_se3[k];
        if (!ok) {
            for (int j = 0; j < 4; ++j) f.q0[j] = f.q1[j] = nan;
            continue;
        }
        const DQ<float> cur = load_dq<float>(f);
        const Q<float> a0 = qmul(avg.q0, cur.q0);
        const Q<float> b1 = qmul(avg.q1, cur.q0), b2 = qmul(avg.q0, cur.q1);
        const Q<float> a1{b1.x + b2.x, b1.y + b2.y, b1.z + b2.z, b1.w + b2.w};
        f = {{a0.x, a0.y, a0.z, a0.w}, {a1.x, a1.y, a1.z, a1.w}};
    }
}

/* The renderer's solver-map pass (render/shaders/SolverMap.vert,
 * SolverMapSized.vert, SolverMapIndexMap.vert, SolverMap.frag; drawn by
 * RendererDraw.cpp:384-480) restated as the GL pipeline runs it: points drawn
 * in surfel order, each covering the pixels whose centres lie in the square of
 * its size around its projection, kept where their depth is strictly below
 * the depth buffer's (GL_LESS, buffer cleared to 1 = nothing drawn). Every
 * pointer is HOST memory; depth_index is not used. Float arithmetic without
 * contraction, in the kernel's operation order. */
void orc_render_solver_maps(const mvdr_surfel_geometry* g, const mvdr_solver_map_params* prm,
                            const mvdr_solver_map_view* views, uint32_t num_views) {
    const uint32_t W = prm->width, H = prm->height;
    auto rows = [](const mvdr_mat34& m, float* o) {
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) o[3 * r + c] = m.rot[3 * c + r];
        for (int r = 0; r < 3; ++r) o[9 + r] = m.trans[r];
    };
    auto pt = [](const float* m, const float* p, float* o) {
        for (int r = 0; r < 3; ++r) o[r] = m[3 * r] * p[0] + m[3 * r + 1] * p[1] + m[3 * r + 2] * p[2] + m[9 + r];
    };
    auto dir = [](const float* m, const float* p, float* o) {
        for (int r = 0; r < 3; ++r) o[r] = m[3 * r] * p[0] + m[3 * r + 1] * p[1] + m[3 * r + 2] * p[2];
    };
    auto nrm = [](float* v) {
        const float inv = 1.0f / std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        for (int k = 0; k < 3; ++k) v[k] *= inv;
    };
    for (uint32_t v = 0; v < num_views; ++v) {
        const mvdr_solver_map_view& V = views[v];
        const uint32_t pitch = V.pitch ? V.pitch : W;
        float w2c[12], init[12], inv[12];
        rows(V.world2camera, w2c);
        rows(V.initial_camera_se3, init);
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) inv[3 * r + c] = init[3 * c + r];
        for (int r = 0; r < 3; ++r) inv[9 + r] = -(inv[3 * r] * init[9] + inv[3 * r + 1] * init[10] + inv[3 * r + 2] * init[11]);
        const float fx = V.intrinsic.focal_x, fy = V.intrinsic.focal_y, cx = V.intrinsic.principal_x,
                    cy = V.intrinsic.principal_y;
        std::vector<float> depth((size_t)W * H, INFINITY);
        std::vector<uint32_t> who((size_t)W * H, MVDR_INVALID_INDEX);
        for (uint32_t s = 0; s < g->num_surfels; ++s) {
            const mvdr_float4 lv = g->live_vertex_confid[s];
            const float l3[3] = {lv.x, lv.y, lv.z};
            float p1[3], pc[3];
            pt(inv, l3, p1);
            pt(w2c, p1, pc);
            const mvdr_float4 ct = g->color_time[s];
            if (pc[2] > prm->max_depth + 0.05f || !(pc[2] > 0.0f) ||
                (g->reference_vertex_confid[s].w < prm->confidence_threshold &&
                 std::fabs(ct.z - prm->current_time) >= prm->time_threshold))
                continue;
            const float xw = (fx * pc[0]) / pc[2] + cx, yw = (fy * pc[1]) / pc[2] + cy;
            if (!(xw >= 0.0f && xw <= (float)W && yw >= 0.0f && yw <= (float)H)) continue;
            float size = 1.0f;
            if (V.sized_points) {
                const mvdr_float4 ln = g->live_normal_radius[s];
                const float l4[3] = {ln.x, ln.y, ln.z};
                float t[3], n[3];
                dir(inv, l4, t);
                dir(w2c, t, n);
                nrm(n);
                const float scale = g->reference_normal_radius[s].w * 1.41421356f * 0.001f;
                float x0[3] = {n[1] - n[2], -n[0], n[0]};
                nrm(x0);
                const float x1[3] = {x0[0] * scale, x0[1] * scale, x0[2] * scale};
                const float y1[3] = {n[1] * x1[2] - n[2] * x1[1], n[2] * x1[0] - n[0] * x1[2], n[0] * x1[1] - n[1] * x1[0]};
                float px[4], py[4];
                const float* ds[4] = {x1, y1, y1, x1};
                const float sg[4] = {1.f, 1.f, -1.f, -1.f};
                for (int k = 0; k < 4; ++k) {
                    const float q[3] = {sg[k] > 0 ? pc[0] + ds[k][0] : pc[0] - ds[k][0],
                                        sg[k] > 0 ? pc[1] + ds[k][1] : pc[1] - ds[k][1],
                                        sg[k] > 0 ? pc[2] + ds[k][2] : pc[2] - ds[k][2]};
                    px[k] = (fx * q[0]) / q[2] + cx;
                    py[k] = (fy * q[1]) / q[2] + cy;
                }
                const float xd = std::max(px[0], std::max(px[1], std::max(px[2], px[3]))) -
                                 std::min(px[0], std::min(px[1], std::min(px[2], px[3])));
                const float yd = std::max(py[0], std::max(py[1], std::max(py[2], py[3]))) -
                                 std::min(py[0], std::min(py[1], std::min(py[2], py[3])));
                size = std::min(std::max(std::max(0.0f, std::min(std::fabs(xd), std::fabs(yd))), 1.0f), 2047.0f);
            }
            const float h = 0.5f * size;
            const int u0 = std::max(0, (int)std::ceil(xw - h - 0.5f)), u1 = std::min((int)W, (int)std::ceil(xw + h - 0.5f));
            const int w0 = std::max(0, (int)std::ceil(yw - h - 0.5f)), w1 = std::min((int)H, (int)std::ceil(yw + h - 0.5f));
            for (int w = w0; w < w1; ++w)
                for (int u = u0; u < u1; ++u) {
                    const size_t q = (size_t)w * W + u;
                    if (pc[2] < depth[q]) {  // GL_LESS: an equal depth keeps the point drawn first
                        depth[q] = pc[2];
                        who[q] = s;
                    }
                }
        }
        for (uint32_t w = 0; w < H; ++w)
            for (uint32_t u = 0; u < W; ++u) {
                const uint32_t id = who[(size_t)w * W + u];
                const size_t o = (size_t)w * pitch + u;
                mvdr_float4 rv{0, 0, 0, 0}, rn{0, 0, 0, 0}, lv{0, 0, 0, 0}, ln{0, 0, 0, 0}, rgb{0, 0, 0, 0};
                if (id != MVDR_INVALID_INDEX) {
                    const mvdr_float4 a0 = g->reference_vertex_confid[id], a1 = g->reference_normal_radius[id],
                                      a2 = g->live_vertex_confid[id], a3 = g->live_normal_radius[id];
                    const float i0[3] = {a0.x, a0.y, a0.z}, i1[3] = {a1.x, a1.y, a1.z}, i2[3] = {a2.x, a2.y, a2.z},
                                i3[3] = {a3.x, a3.y, a3.z};
                    float q0[3], q1[3], q2[3], q3[3];
                    pt(inv, i0, q0);
                    dir(inv, i1, q1);
                    pt(inv, i2, q2);
                    dir(inv, i3, q3);
                    rv = {q0[0], q0[1], q0[2], 1.0f};
                    rn = {q1[0], q1[1], q1[2], 0.0f};
                    lv = {q2[0], q2[1], q2[2], 1.0f};
                    ln = {q3[0], q3[1], q3[2], 0.0f};
                    uint32_t bits;
                    std::memcpy(&bits, &g->color_time[id].x, 4);
                    rgb = {(float)((bits & 0x00FF0000u) >> 16) / 255.f, (float)((bits & 0x0000FF00u) >> 8) / 255.f,
                           (float)(bits & 0x000000FFu) / 255.f, V.sized_points ? 1.0f : g->color_time[id].y};
                }
                if (V.reference_vertex_map) V.reference_vertex_map[o] = rv;
                if (V.reference_normal_map) V.reference_normal_map[o] = rn;
                if (V.live_vertex_map) V.live_vertex_map[o] = lv;
                if (V.live_normal_map) V.live_normal_map[o] = ln;
                if (V.normalized_rgb_map) V.normalized_rgb_map[o] = rgb;
                V.index_map[o] = id;
            }
    }
}

/* The oracle's float DQ blend of four nodes and its se3 matrix, in the
 * mvdr_mat34 layout (rotation columns, translation). */
void orc_blend_se3(const float* field, const uint16_t* knn, const float* w, float* mat12) {
    std::vector<DQ<float>> f(4);
    for (int k = 0; k < 4; ++k) {
        const float* d = field + 8 * (size_t)knn[k];
        f[k] = {{d[0], d[1], d[2], d[3]}, {d[4], d[5], d[6], d[7]}};
    }
    const u16 local[4] = {0, 1, 2, 3};
    const M34<float> m = se3_matrix(blend(f, local, w));
    for (int c = 0; c < 3; ++c)
        for (int r = 0; r < 3; ++r) mat12[3 * c + r] = m.m[r][c];
    for (int r = 0; r < 3; ++r) mat12[9 + r] = m.t[r];
}

float orc_huber(float r) { return huber<float>(r); }

/* The oracle's Jacobian rows (3 x 6) and residuals of a smooth-term record
 * (12 floats) for node i (is_i) or j, and of a point-to-point record (8
 * floats). Returns the channel count. */
int orc_smooth_rows(const float* s12, int is_i, double* J18, double* r3) {
    double J[3][6], r[3];
    const int ch = Oracle::smooth_rows(s12, is_i != 0, J, r);
    for (int c = 0; c < 3; ++c) {
        for (int i = 0; i < 6; ++i) J18[6 * c + i] = ch ? J[c][i] : 0.0;
        r3[c] = ch ? r[c] : 0.0;
    }
    return ch;
}
int orc_p2p_rows(const float* wv8, double* J18, double* r3) {
    double J[3][6], r[3];
    const int ch = Oracle::p2p_rows(wv8, J, r);
    for (int c = 0; c < 3; ++c) {
        for (int i = 0; i < 6; ++i) J18[6 * c + i] = J[c][i];
        r3[c] = r[c];
    }
    return ch;
}
void orc_cholesky_inverse(const double* A36, double* out36) { Oracle::inverse_cholesky(A36, out36); }

}  // extern "C"
