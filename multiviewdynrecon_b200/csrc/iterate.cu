// Per Gauss-Newton iteration kernels: term evaluation, JtJ diagonal blocks /
// Jt r / block preconditioner, off-diagonal JtJ blocks into BSR storage,
// block-Jacobi PCG (materialised or matrix-free), warp-field update, energy.
//
// Reference: DenseDepthJacobianResidual.cu:24-104, NodeGraphSmoothHandler.cu:10-43,
// DensityForegroundJacobianResidual.cu:93-142 with density_map_jacobian.cuh:12-79,
// SparseCorrespondenceHandler.cu:202-220, PreconditionerBlocked.cu:172-284,
// JtDotResidualIndexed.cu:116-224, BlockDiagonalPreconditionerInverse.cu:7-41,
// JtJMaterializer.cu:270-365, BlockPCG.cuh:65-181,317-335,
// ApplyJacobianDot.cu:127-198, ApplyJacobianTransposeDot.cu:29-155,
// SolverIterationData.cu:9-57, ResidualEvaluator.cu:71-142.
//
// Accumulation: every per-node and per-pair sum is a warp-shuffle reduction
// of lane partials; global reductions use per-CTA partials summed in a fixed
// order by the kernel that consumes them (PCG dots, energy). No floating-point
// atomics, so every result is reproducible run to run.
#include <type_traits>

#include "kernels_common.cuh"

namespace mvdr {

// reduction region of the density term's energy partials (regions 0-3: the
// term energy, the PCG delta by parity, d.q)
constexpr uint32_t kRegDensityEnergy = 4;

// ------------------------------------------------------- term evaluation --
// The position chain of every term (blend, normalise, warp, camera
// transforms, projection, residual) runs in T: float reproduces the reference
// arithmetic (FP32 mode); double keeps the millimetre residuals of metre-scale
// positions accurate (mixed mode). Jacobians are stored in float either way.

template <class T> struct V3T { T x, y, z; };
template <class T> __device__ inline V3T<T> v3t(T x, T y, T z) { return {x, y, z}; }
template <class T> __device__ inline V3T<T> sub(V3T<T> a, V3T<T> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class T> __device__ inline T dotv(V3T<T> a, V3T<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class T> struct R34T { T r[9]; T t[3]; };
template <class T> __device__ inline V3T<T> rotv(const R34T<T>& m, V3T<T> v) {
    return {m.r[0] * v.x + m.r[1] * v.y + m.r[2] * v.z, m.r[3] * v.x + m.r[4] * v.y + m.r[5] * v.z,
            m.r[6] * v.x + m.r[7] * v.y + m.r[8] * v.z};
}
template <class T> __device__ inline V3T<T> appv(const R34T<T>& m, V3T<T> v) {
    const V3T<T> a = rotv(m, v);
    return {a.x + m.t[0], a.y + m.t[1], a.z + m.t[2]};
}

template <class T> __device__ inline T cvt(float x);
template <> __device__ inline float cvt<float>(float x) { return x; }
template <> __device__ inline double cvt<double>(float x) { return (double)x; }
template <class T> __device__ inline T rsqrt_t(T x);
template <> __device__ inline float rsqrt_t<float>(float x) { return rsqrtf(x); }
template <> __device__ inline double rsqrt_t<double>(double x) { return rsqrt(x); }

template <class T> __device__ inline R34T<T> view_mat(const ViewDesc& V, int which);
template <> __device__ inline R34T<float> view_mat<float>(const ViewDesc& V, int which) {
    const M34& m = which == 0 ? V.w2c : (which == 1 ? V.init : V.init_inv);
    R34T<float> o;
#pragma unroll
    for (int q = 0; q < 9; ++q) o.r[q] = m.r[q];
#pragma unroll
    for (int q = 0; q < 3; ++q) o.t[q] = m.t[q];
    return o;
}
template <> __device__ inline R34T<double> view_mat<double>(const ViewDesc& V, int which) {
    const double* m = which == 0 ? V.w2c_d : (which == 1 ? V.init_d : V.init_inv_d);
    R34T<double> o;
#pragma unroll
    for (int q = 0; q < 9; ++q) o.r[q] = m[q];
#pragma unroll
    for (int q = 0; q < 3; ++q) o.t[q] = m[9 + q];
    return o;
}

// averageDualQuaternion + DualQuaternion::se3_matrix (DualQuaternion.h:281-393)
// in T; `n` nodes (1 for a single node's own transform)
template <class T>
__device__ inline R34T<T> blended_se3(const DQ* field, const unsigned short* nodes, const float* w, int n) {
    T q0[4] = {0, 0, 0, 0}, q1[4] = {0, 0, 0, 0};
    for (int k = 0; k < n; ++k) {
        const DQ d = load_dq(field, nodes[k]);
        const T s = cvt<T>(w[k]);
        q0[0] += s * cvt<T>(d.q0.x); q0[1] += s * cvt<T>(d.q0.y); q0[2] += s * cvt<T>(d.q0.z); q0[3] += s * cvt<T>(d.q0.w);
        q1[0] += s * cvt<T>(d.q1.x); q1[1] += s * cvt<T>(d.q1.y); q1[2] += s * cvt<T>(d.q1.z); q1[3] += s * cvt<T>(d.q1.w);
    }
    const T inv = rsqrt_t<T>(q0[0] * q0[0] + q0[1] * q0[1] + q0[2] * q0[2] + q0[3] * q0[3]);
#pragma unroll
    for (int i = 0; i < 4; ++i) { q0[i] *= inv; q1[i] *= inv; }
    const T dd = q0[0] * q1[0] + q0[1] * q1[1] + q0[2] * q1[2] + q0[3] * q1[3];
#pragma unroll
    for (int i = 0; i < 4; ++i) q1[i] -= dd * q0[i];
    const T x = q0[0], y = q0[1], z = q0[2], ww = q0[3];
    R34T<T> m;
    m.r[0] = 1 - 2 * y * y - 2 * z * z; m.r[1] = 2 * x * y - 2 * z * ww; m.r[2] = 2 * x * z + 2 * y * ww;
    m.r[3] = 2 * x * y + 2 * z * ww; m.r[4] = 1 - 2 * x * x - 2 * z * z; m.r[5] = 2 * y * z - 2 * x * ww;
    m.r[6] = 2 * x * z - 2 * y * ww; m.r[7] = 2 * y * z + 2 * x * ww; m.r[8] = 1 - 2 * x * x - 2 * y * y;
    // 2 q1 conj(q0), vector part
    const T a0 = 2 * q1[0], a1 = 2 * q1[1], a2 = 2 * q1[2], a3 = 2 * q1[3];
    const T b0 = -x, b1 = -y, b2 = -z, b3 = ww;
    m.t[0] = a3 * b0 + a0 * b3 + a1 * b2 - a2 * b1;
    m.t[1] = a3 * b1 - a0 * b2 + a1 * b3 + a2 * b0;
    m.t[2] = a3 * b2 + a0 * b1 - a1 * b0 + a2 * b3;
    return m;
}

// computeImageDensityJacobainAndResidual (density_map_jacobian.cuh:54-69): the
// image gradient `gr` at the projected pixel, chained through the pinhole
// projection of the camera point vc and the two rotations to a twist
// gradient at the warped vertex wv: o0 = (rotation part, g.x), g_yz = (g.y, g.z)
__device__ inline void image_twist_gradient(const ViewDesc& V, float3 vc, float3 wv, float2 gr, float4& o0,
                                            float2& g_yz) {
    float3 g;
    g.x = gr.x * V.fx / vc.z;
    g.y = gr.y * V.fy / vc.z;
    g.z = -1.0f / (vc.z * vc.z) * (V.fx * vc.x * gr.x + V.fy * vc.y * gr.y);
    g = rotT3(V.w2c, rot3(V.init, g));
    o0 = make_float4(-g.y * wv.z + g.z * wv.y, g.x * wv.z - g.z * wv.x, -g.x * wv.y + g.y * wv.x, g.x);
    g_yz = make_float2(g.y, g.z);
}

// 4 CTAs per SM (64 registers, a few spilled) hide the gathers of the warp
// field and the maps better than 2 (-32 % measured)
// The dense-depth term of compacted pixel k under the current warp field
// (computeDenseDepthJacobianKernel, DenseDepthJacobianResidual.cu:24-104): the
// 32-byte record (twist gradient, residual, projected pixel; J = 0 and the
// pixel 0xFFFFFFFF when the correspondence is invalid). The term evaluation
// stores it; the matrix-free products recompute it when asked to.
template <class T>
__device__ inline void dense_record(const InstDesc& I, uint32_t k, float4& o0, float4& o1, bool& nonfinite) {
    const float4 cv = I.dense_cv[k], cn = I.dense_cn[k];
    const uint32_t v = __float_as_uint(cv.w);
    const ViewDesc& V = I.views[v];
    const ushort4 kn = I.dense_knn[k];
    const float4 w4 = I.dense_w[k];
    const unsigned short nodes[4] = {kn.x, kn.y, kn.z, kn.w};
    const float wts[4] = {w4.x, w4.y, w4.z, w4.w};
    const R34T<T> se3 = blended_se3<T>(I.se3, nodes, wts, 4);
    const R34T<T> w2c = view_mat<T>(V, 0), iinv = view_mat<T>(V, 2);
    V3T<T> cvt3 = v3t(cvt<T>(cv.x), cvt<T>(cv.y), cvt<T>(cv.z));
    if constexpr (sizeof(T) == 8) {
        const float4 lo = I.dense_cv_lo[k];
        cvt3 = v3t(cvt3.x + cvt<T>(lo.x), cvt3.y + cvt<T>(lo.y), cvt3.z + cvt<T>(lo.z));
    }
    const V3T<T> wv = appv(se3, cvt3);
    const V3T<T> wn = rotv(se3, v3t(cvt<T>(cn.x), cvt<T>(cn.y), cvt<T>(cn.z)));
    const V3T<T> vc = appv(iinv, appv(w2c, wv));
    const V3T<T> nc = rotv(iinv, rotv(w2c, wn));
    const int u = project_coord((float)vc.x, (float)vc.z, V.fx, V.cx);
    const int w = project_coord((float)vc.y, (float)vc.z, V.fy, V.cy);
    nonfinite |= !isfinite((float)vc.x) || !isfinite((float)vc.y) || !isfinite((float)vc.z);
    o0 = make_float4(0.f, 0.f, 0.f, 0.f);
    o1 = make_float4(0.f, 0.f, 0.f, __uint_as_float(kInvalid));
    if (u >= 0 && u < (int)I.width && w >= 0 && w < (int)I.height) {
        const size_t p = (size_t)w * V.pitch + u;
        const float4 dv4 = V.obs_v[p], dn4 = V.obs_n[p];
        const V3T<T> dv = v3t(cvt<T>(dv4.x), cvt<T>(dv4.y), cvt<T>(dv4.z));
        const V3T<T> dn = v3t(cvt<T>(dn4.x), cvt<T>(dn4.y), cvt<T>(dn4.z));
        bool valid = true;
        if (fabsf(dv4.x) < 1e-3f && fabsf(dv4.y) < 1e-3f && fabsf(dv4.z) < 1e-3f) valid = false;
        if (dotv(dn, nc) < (T)0.7f) valid = false;
        const V3T<T> df = sub(dv, vc);
        if (dotv(df, df) > (T)(0.075f * 0.075f)) valid = false;
        if (valid) {
            const float r = (float)dotv(dn, sub(vc, dv));
            nonfinite |= !isfinite(r);
            const float3 dnf = mk3(dn4.x, dn4.y, dn4.z);
            const float3 tr = rotT3(V.w2c, rot3(V.init, dnf));
            const float3 ro = cross3(mk3((float)wv.x, (float)wv.y, (float)wv.z), tr);
            o0 = make_float4(ro.x, ro.y, ro.z, tr.x);
            o1 = make_float4(tr.y, tr.z, r, __uint_as_float((uint32_t)w * I.width + (uint32_t)u));
        }
    }
}

// The foreground-mask term of compacted pixel k
// (computeForegroundMaskJacobian + computeImageDensityJacobainAndResidual,
// DensityForegroundJacobianResidual.cu:93-142); fg_cv holds the canonical
// vertex in frame 0, as the dense term uses it, or with
// MVDR_COMPAT_REF_FOREGROUND_FRAME in its own camera's frame, as
// density_map_jacobian.cuh:32-36 warps it.
template <class T>
__device__ inline void fg_record(const InstDesc& I, uint32_t k, float4& o0, float4& o1, bool& nonfinite) {
    const float4 cv = I.fg_cv[k];
    const uint32_t v = __float_as_uint(cv.w);
    const ViewDesc& V = I.views[v];
    const ushort4 kn = I.fg_knn[k];
    const float4 w4 = I.fg_w[k];
    const unsigned short nodes[4] = {kn.x, kn.y, kn.z, kn.w};
    const float wts[4] = {w4.x, w4.y, w4.z, w4.w};
    const R34T<T> se3 = blended_se3<T>(I.se3, nodes, wts, 4);
    const R34T<T> w2c = view_mat<T>(V, 0), iinv = view_mat<T>(V, 2);
    const V3T<T> wvt = appv(se3, v3t(cvt<T>(cv.x), cvt<T>(cv.y), cvt<T>(cv.z)));
    const V3T<T> vct = appv(iinv, appv(w2c, wvt));
    const float3 wv = mk3((float)wvt.x, (float)wvt.y, (float)wvt.z);
    const float3 vc = mk3((float)vct.x, (float)vct.y, (float)vct.z);
    const int u = project_coord(vc.x, vc.z, V.fx, V.cx);
    const int w = project_coord(vc.y, vc.z, V.fy, V.cy);
    nonfinite |= !isfinite(vc.x) || !isfinite(vc.y) || !isfinite(vc.z);
    o0 = make_float4(0.f, 0.f, 0.f, 0.f);
    o1 = make_float4(0.f, 0.f, 0.f, __uint_as_float(kInvalid));
    if (u >= 0 && u < (int)I.width && w >= 0 && w < (int)I.height && V.fg != nullptr) {
        const size_t p = (size_t)w * V.pitch + u;
        const float img = V.fg[p];
        float2 gyz;
        image_twist_gradient(V, vc, wv, V.fg_grad[p], o0, gyz);
        // geometry density 0 (DensityForegroundJacobianResidual.cu:103)
        o1 = make_float4(gyz.x, gyz.y, img - 0.0f, __uint_as_float((uint32_t)w * I.width + (uint32_t)u));
        nonfinite |= !isfinite(o1.z) || !isfinite(o0.w) || !isfinite(gyz.x) || !isfinite(gyz.y);
    }
}

template <class T>
__global__ void __launch_bounds__(256, 4) eval_terms_kernel(const InstDesc* insts, mvdr_penalty lam) {
    const InstDesc& I = insts[blockIdx.y];
    TermOffsets off;
    off.load(I.counts);
    const uint32_t Td = off.o[0];
    const uint32_t T_all = bad_inputs(I) ? 0u : off.o[4];
    // the lambda-weighted squared residuals of this CTA's terms
    // (ResidualEvaluator.cu:71-226): the energy of the linearisation point
    double energy = 0;
    // a NaN or Inf in a warped point or a residual (from the inputs or the
    // warp field) flags the instance, MVDR_ENONFINITE on the host
    bool nonfinite = false;
    const float clip = 64.f * I.node_radius * I.node_radius;
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < T_all; t += gridDim.x * blockDim.x) {
        uint32_t k;
        const TermType ty = off.typed(t, k);
        if (ty == kDense) {
            float4 o0, o1;
            dense_record<T>(I, k, o0, o1, nonfinite);
            I.term_jr[2 * (size_t)k] = o0;
            I.term_jr[2 * (size_t)k + 1] = o1;
            energy += (double)o1.z * o1.z;
        } else if (ty == kSmooth) {
            // forwardWarpSmootherNodeKernel (NodeGraphSmoothHandler.cu:10-43)
            const ushort2 e = I.graph[k];
            const float4 xi = I.nodes[e.x], xj = I.nodes[e.y];
            const float one = 1.f;
            const R34T<T> Ti = blended_se3<T>(I.se3, &e.x, &one, 1), Tj = blended_se3<T>(I.se3, &e.y, &one, 1);
            const V3T<T> xjt = v3t(cvt<T>(xj.x), cvt<T>(xj.y), cvt<T>(xj.z));
            const V3T<T> a = appv(Ti, xjt), b = appv(Tj, xjt);
            const float3 dd = mk3(xi.x - xj.x, xi.y - xj.y, xi.z - xj.z);
            const float valid = dot3(dd, dd) > clip ? 0.f : 1.f;
            I.smooth[3 * (size_t)k] = make_float4((float)a.x, (float)a.y, (float)a.z, (float)b.x);
            I.smooth[3 * (size_t)k + 1] = make_float4((float)b.y, (float)b.z, valid, 0.f);
            const float4 rr = make_float4((float)(a.x - b.x), (float)(a.y - b.y), (float)(a.z - b.z), 0.f);
            nonfinite |= !isfinite(rr.x) || !isfinite(rr.y) || !isfinite(rr.z);
            I.smooth[3 * (size_t)k + 2] = rr;
            if (valid != 0.f) {
                const float r0 = lam.smooth * rr.x, r1 = lam.smooth * rr.y, r2 = lam.smooth * rr.z;
                energy += (double)r0 * r0 + (double)r1 * r1 + (double)r2 * r2;
            }
        } else if (ty == kForeground) {
            float4 o0, o1;
            fg_record<T>(I, k, o0, o1, nonfinite);
            I.term_jr[2 * (size_t)(Td + k)] = o0;
            I.term_jr[2 * (size_t)(Td + k) + 1] = o1;
            {
                const float v = lam.foreground * o1.z;
                energy += (double)v * v;
            }
        } else if (ty == kFeature || ty == kCross) {
            // forwardWarpFeatureVertexKernel (SparseCorrespondenceHandler.cu:202-220)
            const bool f = ty == kFeature;
            const float4 ref = f ? I.feat_ref[k] : I.cross_ref[k];
            const float4 tg = f ? I.feat_target[k] : I.cross_target[k];
            const ushort4 kn = f ? I.feat_knn[k] : I.cross_knn[k];
            const float4 w4 = f ? I.feat_w[k] : I.cross_w[k];
            const unsigned short nodes[4] = {kn.x, kn.y, kn.z, kn.w};
            const float wts[4] = {w4.x, w4.y, w4.z, w4.w};
            const R34T<T> se3 = blended_se3<T>(I.se3, nodes, wts, 4);
            const V3T<T> wv = appv(se3, v3t(cvt<T>(ref.x), cvt<T>(ref.y), cvt<T>(ref.z)));
            const V3T<T> raw = sub(wv, v3t(cvt<T>(tg.x), cvt<T>(tg.y), cvt<T>(tg.z)));
            nonfinite |= !isfinite((float)raw.x) || !isfinite((float)raw.y) || !isfinite((float)raw.z);
            const size_t o = 2 * (size_t)(f ? k : I.Tp + k);
            I.warped[o] = make_float4((float)wv.x, (float)wv.y, (float)wv.z, 1.0f);
            I.warped[o + 1] = make_float4((float)raw.x, (float)raw.y, (float)raw.z, 0.0f);
            const float l = f ? lam.feature : lam.cross_view;
            const float rv[3] = {(float)raw.x, (float)raw.y, (float)raw.z};
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const float v = l * (huber_weight(rv[c]) * rv[c]);
                energy += (double)v * v;
            }
        }
    }
    if (__any_sync(0xffffffffu, nonfinite) && lane_id() == 0) set_error(I, kErrNonFinite);
    // one partial per CTA (reduction region 0), summed by energy_sum_kernel
    __shared__ double ws[8];
    energy = warp_sum(energy);
    if (lane_id() == 0) ws[threadIdx.x >> 5] = energy;
    __syncthreads();
    if (threadIdx.x == 0) {
        double e = 0;
        for (uint32_t w = 0; w < (blockDim.x >> 5); ++w) e += ws[w];
        I.partials[blockIdx.x] = e;
    }
}

// computeDensityMapJacobian (DensityForegroundJacobianResidual.cu:41-91): the
// second residual of every dense pixel, the observed grey level at the
// projected pixel minus the rendered one, with the image-gradient Jacobian of
// computeImageDensityJacobainAndResidual. The vertex is warped as the dense
// term warps it (frame 0), or in its camera's frame under
// MVDR_COMPAT_REF_FOREGROUND_FRAME. A kernel of its own, launched only when
// the term is on, so that it adds no registers to the term evaluation. Its
// weighted squared residuals go to reduction region kRegDensityEnergy.
template <class T>
__global__ void __launch_bounds__(256, 2) eval_density_kernel(const InstDesc* insts, mvdr_penalty lam) {
    const InstDesc& I = insts[blockIdx.y];
    const uint32_t Td = bad_inputs(I) ? 0u : I.counts->term_offset[0];
    double energy = 0;
    bool nonfinite = false;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < Td; k += gridDim.x * blockDim.x) {
        const float4 cv = I.dense_cv[k], cn = I.dense_cn[k];
        const ViewDesc& V = I.views[__float_as_uint(cv.w)];
        const ushort4 kn = I.dense_knn[k];
        const float4 w4 = I.dense_w[k];
        const unsigned short nodes[4] = {kn.x, kn.y, kn.z, kn.w};
        const float wts[4] = {w4.x, w4.y, w4.z, w4.w};
        const R34T<T> se3 = blended_se3<T>(I.se3, nodes, wts, 4);
        const R34T<T> w2c = view_mat<T>(V, 0), iinv = view_mat<T>(V, 2);
        V3T<T> p0;
        if (I.compat & MVDR_COMPAT_REF_FOREGROUND_FRAME) {
            const ushort4 px = I.dense_pix[k];
            const float4 rv = V.ref_v[(size_t)px.y * V.pitch + px.x];
            p0 = v3t(cvt<T>(rv.x), cvt<T>(rv.y), cvt<T>(rv.z));
        } else {
            p0 = v3t(cvt<T>(cv.x), cvt<T>(cv.y), cvt<T>(cv.z));
            if constexpr (sizeof(T) == 8) {
                const float4 lo = I.dense_cv_lo[k];
                p0 = v3t(p0.x + cvt<T>(lo.x), p0.y + cvt<T>(lo.y), p0.z + cvt<T>(lo.z));
            }
        }
        const V3T<T> wr = appv(se3, p0);
        const V3T<T> vr = appv(iinv, appv(w2c, wr));
        const float3 wvf = mk3((float)wr.x, (float)wr.y, (float)wr.z);
        const float3 vcf = mk3((float)vr.x, (float)vr.y, (float)vr.z);
        const int u = project_coord((float)vr.x, (float)vr.z, V.fx, V.cx);
        const int w = project_coord((float)vr.y, (float)vr.z, V.fy, V.cy);
        nonfinite |= !isfinite(vcf.x) || !isfinite(vcf.y) || !isfinite(vcf.z);
        float4 d0 = make_float4(0.f, 0.f, 0.f, 0.f), d1 = make_float4(0.f, 0.f, 0.f, __uint_as_float(kInvalid));
        if (u >= 0 && u < (int)I.width && w >= 0 && w < (int)I.height) {
            const size_t p = (size_t)w * V.pitch + u;
            float2 gyz;
            image_twist_gradient(V, vcf, wvf, V.dens_grad[p], d0, gyz);
            d1 = make_float4(gyz.x, gyz.y, V.dens[p] - cn.w, __uint_as_float((uint32_t)w * I.width + (uint32_t)u));
            nonfinite |= !isfinite(d1.z) || !isfinite(d0.w) || !isfinite(gyz.x) || !isfinite(gyz.y);
        }
        I.density_jr[2 * (size_t)k] = d0;
        I.density_jr[2 * (size_t)k + 1] = d1;
        const float dv = lam.density * d1.z;
        energy += (double)dv * dv;
    }
    if (__any_sync(0xffffffffu, nonfinite) && lane_id() == 0) set_error(I, kErrNonFinite);
    __shared__ double ws[8];
    energy = warp_sum(energy);
    if (lane_id() == 0) ws[threadIdx.x >> 5] = energy;
    __syncthreads();
    if (threadIdx.x == 0) {
        double e = 0;
        for (uint32_t q = 0; q < (blockDim.x >> 5); ++q) e += ws[q];
        I.partials[(size_t)kRegDensityEnergy * I.part_stride + blockIdx.x] = e;
    }
}

// --------------------------------------------- per-term Jacobian rows -----
// The weighted Jacobian rows that term t contributes to node `node`:
// J[c][0..5] (rotation, translation), residual r[c]; returns the channel count
// (0 when the term is invalid) and sets lam2 and the node's skinning weight.
struct TermRows {
    float J[3][6];
    float r[3];
    float lam2;
    float w;
};

__device__ inline void skew_rows(float3 p, float sg, float hw[3], TermRows& o) {
    // rows of [p]x^T (geometry_icp_jacobian.cuh:323-343, 91-120)
    o.J[0][0] = 0.f;           o.J[0][1] = sg * hw[0] * p.z;  o.J[0][2] = -sg * hw[0] * p.y;
    o.J[1][0] = -sg * hw[1] * p.z; o.J[1][1] = 0.f;           o.J[1][2] = sg * hw[1] * p.x;
    o.J[2][0] = sg * hw[2] * p.y;  o.J[2][1] = -sg * hw[2] * p.x; o.J[2][2] = 0.f;
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int i = 0; i < 3; ++i) o.J[c][3 + i] = (c == i) ? sg * hw[c] : 0.f;
}

__device__ inline int term_rows(const InstDesc& I, const TermOffsets& off, const mvdr_penalty& lam, uint32_t t,
                                uint32_t node, TermRows& o) {
    uint32_t k;
    const TermType ty = off.typed(t, k);
    switch (ty) {
        case kDense:
        case kForeground: {
            const uint32_t idx = ty == kDense ? k : off.o[0] + k;
            const float4 a = I.term_jr[2 * (size_t)idx], b = I.term_jr[2 * (size_t)idx + 1];
            o.J[0][0] = a.x; o.J[0][1] = a.y; o.J[0][2] = a.z; o.J[0][3] = a.w; o.J[0][4] = b.x; o.J[0][5] = b.y;
            o.r[0] = b.z;
            o.lam2 = ty == kDense ? 1.0f : lam.foreground * lam.foreground;
            o.w = weight_of(term_nodes(I, ty, k), term_weights(I, ty, k), node);
            return 1;
        }
        case kSmooth: {
            const float4 a = I.smooth[3 * (size_t)k], b = I.smooth[3 * (size_t)k + 1];
            if (b.z == 0.f) return 0;
            const float4 rr = I.smooth[3 * (size_t)k + 2];
            const bool is_i = node == I.graph[k].x;
            const float3 ti = mk3(a.x, a.y, a.z), tj = mk3(a.w, b.x, b.y);
            float one[3] = {1.f, 1.f, 1.f};
            skew_rows(is_i ? ti : tj, is_i ? 1.f : -1.f, one, o);
            o.r[0] = rr.x; o.r[1] = rr.y; o.r[2] = rr.z;
            o.lam2 = lam.smooth * lam.smooth;
            o.w = 1.f;
            return 3;
        }
        case kFeature:
        case kCross: {
            const bool f = ty == kFeature;
            const float4 wv = I.warped[2 * (size_t)(f ? k : I.Tp + k)];
            const float4 rw = I.warped[2 * (size_t)(f ? k : I.Tp + k) + 1];
            const float raw[3] = {rw.x, rw.y, rw.z};
            float hw[3] = {huber_weight(raw[0]), huber_weight(raw[1]), huber_weight(raw[2])};
            skew_rows(mk3(wv.x, wv.y, wv.z), 1.f, hw, o);
            o.r[0] = hw[0] * raw[0]; o.r[1] = hw[1] * raw[1]; o.r[2] = hw[2] * raw[2];
            o.lam2 = f ? lam.feature * lam.feature : lam.cross_view * lam.cross_view;
            o.w = weight_of(term_nodes(I, ty, k), term_weights(I, ty, k), node);
            return 3;
        }
        default: return 0;
    }
}

// ------------------------------------------ diagonal blocks, Jt r, M^-1 ----

__device__ constexpr int upper_index(int i, int j) { return i * 6 - (i * (i - 1)) / 2 + (j - i); }

// DenseGaussian<6>::Inverse with partial pivoting (DenseGaussian.h:55-125)
__device__ inline void gauss_jordan6(const float* Din, float* out) {
    float m[36];
#pragma unroll
    for (int i = 0; i < 36; ++i) m[i] = Din[i];  // column-major, symmetric input
    int perm[6] = {0, 1, 2, 3, 4, 5}, reloc[6];
    for (int i = 0; i < 6; ++i) {
        int piv = i;
        float pv = fabsf(m[i + 6 * i]);
        for (int j = i + 1; j < 6; ++j)
            if (pv < fabsf(m[j + 6 * i])) { pv = fabsf(m[j + 6 * i]); piv = j; }
        for (int k = 0; k < 6; ++k) { const float tmp = m[i + 6 * k]; m[i + 6 * k] = m[piv + 6 * k]; m[piv + 6 * k] = tmp; }
        { const int tp = perm[i]; perm[i] = perm[piv]; perm[piv] = tp; }
        reloc[i] = perm[i];
        const float inv = 1.0f / m[i + 6 * i];
        for (int k = 0; k < 6; ++k) m[i + 6 * k] *= inv;
        m[i + 6 * i] = inv;
        for (int r = 0; r < 6; ++r) {
            if (r == i) continue;
            const float a = m[r + 6 * i];
            for (int k = 0; k < 6; ++k) m[r + 6 * k] -= a * m[i + 6 * k];
            m[r + 6 * i] = -a * m[i + 6 * i];
        }
    }
    for (int j = 0; j < 6; ++j)
        for (int i = 0; i < 6; ++i) out[6 * reloc[j] + i] = m[i + 6 * j];
}

// 6x6 Cholesky in double; packed lower triangle L[i(i+1)/2 + j], j <= i, with
// the RECIPROCALS of the diagonal stored on the diagonal so that the solves
// applied every PCG iteration only multiply
template <class T> __device__ inline void cholesky6(const T* A, double* L) {
#pragma unroll
    for (int j = 0; j < 6; ++j) {
        double s = A[6 * j + j];
#pragma unroll
        for (int k = 0; k < j; ++k) s -= L[j * (j + 1) / 2 + k] * L[j * (j + 1) / 2 + k];
        const double inv = 1.0 / sqrt(s);
        L[j * (j + 1) / 2 + j] = inv;
#pragma unroll
        for (int i = j + 1; i < 6; ++i) {
            double t = A[6 * i + j];
#pragma unroll
            for (int k = 0; k < j; ++k) t -= L[i * (i + 1) / 2 + k] * L[j * (j + 1) / 2 + k];
            L[i * (i + 1) / 2 + j] = t * inv;
        }
    }
}

__device__ inline void cholesky6_solve(const double* L, const double* b, double* x) {
    double y[6];
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        double t = b[i];
#pragma unroll
        for (int k = 0; k < i; ++k) t -= L[i * (i + 1) / 2 + k] * y[k];
        y[i] = t * L[i * (i + 1) / 2 + i];
    }
#pragma unroll
    for (int i = 5; i >= 0; --i) {
        double t = y[i];
#pragma unroll
        for (int k = i + 1; k < 6; ++k) t -= L[k * (k + 1) / 2 + i] * x[k];
        x[i] = t * L[i * (i + 1) / 2 + i];
    }
}

// Mixed precision keeps the assembled JtJ blocks in double: rounding them to
// float moves the PCG increment by 1.3e-4 to 5e-4 on these blocks, whose
// condition numbers reach 1e5, and rounding only the off-diagonal blocks still
// moves it by up to 1.5e-4. The PCG itself runs on the float blocks of the
// scaled operator (scale_offdiag_kernel), whose entries are of order one.
template <bool MIXED> struct BlockStore;
template <> struct BlockStore<true> {
    using V = double;
    __device__ static V* ptr(const InstDesc& I) { return I.bsr_d; }
};
template <> struct BlockStore<false> {
    using V = float;
    __device__ static V* ptr(const InstDesc& I) { return I.bsr; }
};

// ------------------------------------------------- JtJ block helpers -----
// Twist Jacobian row of a point-to-point or smooth residual at point p
// (geometry_icp_jacobian.cuh:91-120, 323-343): f_c(p) = [row c of [p]x^T ; e_c].
template <class T> __device__ inline void twist_rows(T px, T py, T pz, T f[3][6]) {
    f[0][0] = 0;   f[0][1] = pz;  f[0][2] = -py; f[0][3] = 1; f[0][4] = 0; f[0][5] = 0;
    f[1][0] = -pz; f[1][1] = 0;   f[1][2] = px;  f[1][3] = 0; f[1][4] = 1; f[1][5] = 0;
    f[2][0] = py;  f[2][1] = -px; f[2][2] = 0;   f[2][3] = 0; f[2][4] = 0; f[2][5] = 1;
}

// (sum_c f_c(p) f_c(q)^T)(r, k) for the twist rows above; with r and k known
// at compile time this folds to at most three products
template <class T> __device__ inline T twist_rows_product(const T p[3], const T q[3], int r, int k) {
    // f_c(p)[r] for r < 3: the rows of [p]x^T
    auto sk = [](const T v[3], int c, int rr) -> T {
        if (c == 0) return rr == 0 ? (T)0 : (rr == 1 ? v[2] : -v[1]);
        if (c == 1) return rr == 0 ? -v[2] : (rr == 1 ? (T)0 : v[0]);
        return rr == 0 ? v[1] : (rr == 1 ? -v[0] : (T)0);
    };
    if (r < 3 && k < 3) return sk(p, 0, r) * sk(q, 0, k) + sk(p, 1, r) * sk(q, 1, k) + sk(p, 2, r) * sk(q, 2, k);
    if (r < 3) return sk(p, k - 3, r);
    if (k < 3) return sk(q, r - 3, k);
    return r == k ? (T)1 : (T)0;
}

// upper-triangle index of a symmetric 6x6 block (r <= k)
__device__ constexpr int sym_idx(int r, int k) { return r * 6 - (r * (r - 1)) / 2 + (k - r); }

// S += sg g^T on the upper triangle (sg is a multiple of g, so the product is
// symmetric)
// S += (c g) g^T on the upper triangle, (c g_r) formed once per row r
template <class Acc>
__device__ inline void add_scaled_outer(Acc S[21], Acc c, const Acc g[6]) {
#pragma unroll
    for (int r = 0; r < 6; ++r) {
        const Acc sr = c * g[r];
#pragma unroll
        for (int k = r; k < 6; ++k) S[sym_idx(r, k)] += sr * g[k];
    }
}

template <class Acc>
__device__ inline void add_sym_outer(Acc S[21], const Acc sg[6], const Acc g[6]) {
#pragma unroll
    for (int r = 0; r < 6; ++r)
#pragma unroll
        for (int k = r; k < 6; ++k) S[sym_idx(r, k)] += sg[r] * g[k];
}

// ---------------------------------------------------- diagonal blocks ----
// One warp per node. The lanes take the node's terms round-robin and keep
// D_i = sum_t lambda_t^2 w_ti^2 sum_c g_c g_c^T (21 upper-triangle sums) and
// b_i = -sum_t lambda_t^2 w_ti sum_c g_c r_c (6 sums) in registers; a fixed
// reduce-scatter (five halving exchanges) then leaves each of 27 lanes with
// one warp total, so the result does not depend on scheduling. computeBlockDiagonalPreconditionerKernel and
// computeJtResidualWithIndexKernel (PreconditionerBlocked.cu:18-399,
// JtDotResidualIndexed.cu:18-382) compute the same sums. A CTA takes
// kDiagNodes nodes; their damped blocks wait in shared memory and one warp
// then factors them, a node per lane (Cholesky in double for mixed precision,
// the Gauss-Jordan inverse of BlockDiagonalPreconditionerInverse.cu:7-60 in
// float).
constexpr uint32_t kDiagNodes = 32;

// 4 CTAs per SM (128 registers, no spills): with the term loads software-
// pipelined, fewer but spill-free warps win (measured against 5 CTAs)
template <bool MIXED>
__global__ void __launch_bounds__(128, 4) diag_rhs_kernel(const InstDesc* insts, mvdr_penalty lam) {
    using Acc = typename std::conditional<MIXED, double, float>::type;
    __shared__ Acc s_blocks[kDiagNodes][21];
    const InstDesc& I = insts[blockIdx.y];
    const DeviceCounts* C = I.counts;
    if (C->node2term_entries > I.cap_k1 || C->half_pairs > I.cap_pairs) return;
    TermOffsets off;
    off.load(C);
    const uint32_t lane = lane_id(), warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const Acc l2_fg = (Acc)(lam.foreground * lam.foreground), l2_smooth = (Acc)(lam.smooth * lam.smooth);
    const Acc l2_feat = (Acc)(lam.feature * lam.feature), l2_cross = (Acc)(lam.cross_view * lam.cross_view);
    // the density channel of the dense pixels (0 when the term is off or its
    // weight is 0 in this iteration's phase)
    const bool dens_on = I.use_density && lam.density != 0.f;
    const Acc l2_dens = (Acc)(lam.density * lam.density);
    // the upper-triangle entry (orr, okk) of D whose total this lane receives
    uint32_t orr = 0, okk = 0;
    for (uint32_t r = 0, q = 0; r < 6; ++r)
        for (uint32_t k = r; k < 6; ++k, ++q)
            if (q == lane) { orr = r; okk = k; }
    for (uint32_t base = blockIdx.x * kDiagNodes; base < I.N; base += gridDim.x * kDiagNodes) {
        for (uint32_t j = warp; j < kDiagNodes && base + j < I.N; j += nwarps) {
            const uint32_t node = base + j;
            const uint32_t b0 = I.n2t_offset[node], b1 = I.n2t_offset[node + 1];
            Acc S[21], R[6];
#pragma unroll
            for (int q = 0; q < 21; ++q) S[q] = 0;
#pragma unroll
            for (int q = 0; q < 6; ++q) R[q] = 0;
            // software pipeline over the lane's terms: the term id two steps
            // ahead and the pixel-term record and weight one step ahead are in
            // flight while the current term is summed
            uint32_t t1 = b0 + lane < b1 ? I.n2t_index[b0 + lane] : kInvalid;
            uint32_t t2 = b0 + lane + 32 < b1 ? I.n2t_index[b0 + lane + 32] : kInvalid;
            float4 pa = make_float4(0.f, 0.f, 0.f, 0.f), pb = pa;
            float pw = 0.f;
            auto fetch_pixel_term = [&](uint32_t t, uint32_t pp) {
                uint32_t k;
                const TermType ty = off.typed(t, k);
                if (ty == kDense || ty == kForeground) {
                    const uint32_t idx = ty == kDense ? k : off.o[0] + k;
                    pa = I.term_jr[2 * (size_t)idx];
                    pb = I.term_jr[2 * (size_t)idx + 1];
                    pw = I.n2t_w[pp];
                }
            };
            if (b0 + lane < b1) fetch_pixel_term(t1, b0 + lane);
            for (uint32_t p = b0 + lane; p < b1; p += 32) {
                const uint32_t t = t1;
                const float4 a = pa, b = pb;
                const float wf = pw;
                t1 = t2;
                if (p + 64 < b1) t2 = I.n2t_index[p + 64];
                if (p + 32 < b1) fetch_pixel_term(t1, p + 32);
                uint32_t k;
                const TermType ty = off.typed(t, k);
                if (ty == kDense || ty == kForeground) {
                    const Acc w = (Acc)wf;
                    if (__float_as_uint(b.w) != kInvalid) {  // an invalid term has J = 0, r = 0
                        const Acc l2 = ty == kDense ? (Acc)1 : l2_fg;
                        const Acc g[6] = {(Acc)a.x, (Acc)a.y, (Acc)a.z, (Acc)a.w, (Acc)b.x, (Acc)b.y};
                        const Acc sw = l2 * w * w, rw = -l2 * w * (Acc)b.z;
#pragma unroll
                        for (int q = 0; q < 6; ++q) R[q] += rw * g[q];
                        add_scaled_outer(S, sw, g);
                    }
                    if (ty == kDense && dens_on) {
                        float4 da, db;
                        load_record32(I.density_jr + 2 * (size_t)k, da, db);
                        if (__float_as_uint(db.w) != kInvalid) {
                            const Acc g[6] = {(Acc)da.x, (Acc)da.y, (Acc)da.z, (Acc)da.w, (Acc)db.x, (Acc)db.y};
                            const Acc sw = l2_dens * w * w, rw = -l2_dens * w * (Acc)db.z;
#pragma unroll
                            for (int q = 0; q < 6; ++q) R[q] += rw * g[q];
                            add_scaled_outer(S, sw, g);
                        }
                    }
                } else if (ty == kSmooth) {
                    // computeSmoothTermJacobian (geometry_icp_jacobian.cuh:323-343):
                    // J_i,c = f_c(T_i x_j), J_j,c = -f_c(T_j x_j)
                    const float4 a = I.smooth[3 * (size_t)k], b = I.smooth[3 * (size_t)k + 1];
                    if (b.z == 0.f) continue;
                    const float4 rr = I.smooth[3 * (size_t)k + 2];
                    const bool is_i = node == I.graph[k].x;
                    const float4 pt = is_i ? a : make_float4(a.w, b.x, b.y, 0.f);
                    Acc fr[3][6];
                    twist_rows<Acc>((Acc)pt.x, (Acc)pt.y, (Acc)pt.z, fr);
                    const Acc rc[3] = {(Acc)rr.x, (Acc)rr.y, (Acc)rr.z};
                    const Acc sgn = is_i ? (Acc)1 : (Acc)-1;
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        const Acc rw = -l2_smooth * sgn * rc[c];
#pragma unroll
                        for (int q = 0; q < 6; ++q) R[q] += rw * fr[c][q];
                        add_scaled_outer(S, l2_smooth, fr[c]);
                    }
                } else if (ty == kFeature || ty == kCross) {
                    const bool f = ty == kFeature;
                    const float4 wv = I.warped[2 * (size_t)(f ? k : I.Tp + k)];
                    const float4 raw = I.warped[2 * (size_t)(f ? k : I.Tp + k) + 1];
                    const Acc l2 = f ? l2_feat : l2_cross;
                    const Acc w = (Acc)I.n2t_w[p];
                    Acc fr[3][6];
                    twist_rows<Acc>((Acc)wv.x, (Acc)wv.y, (Acc)wv.z, fr);
                    const float rv[3] = {raw.x, raw.y, raw.z};
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        const Acc hw = (Acc)huber_weight(rv[c]);
                        const Acc rw = -l2 * hw * (Acc)rv[c];
                        Acc g[6];
#pragma unroll
                        for (int q = 0; q < 6; ++q) {
                            g[q] = w * hw * fr[c][q];
                            R[q] += rw * g[q];
                        }
                        add_scaled_outer(S, l2, g);
                    }
                }
            }
            // fixed-order reduce-scatter: five halving steps leave lane q with
            // the warp total of value q (q < 21: D entry q, 21 + k: b_k)
            Acc v[32];
#pragma unroll
            for (int q = 0; q < 21; ++q) v[q] = S[q];
#pragma unroll
            for (int q = 0; q < 6; ++q) v[21 + q] = R[q];
#pragma unroll
            for (int q = 27; q < 32; ++q) v[q] = 0;
#pragma unroll
            for (int dist = 16; dist > 0; dist >>= 1) {
                const bool upper = (lane & (uint32_t)dist) != 0;
#pragma unroll
                for (int i = 0; i < dist; ++i) {
                    const Acc keep = upper ? v[i + dist] : v[i];
                    const Acc send = upper ? v[i] : v[i + dist];
                    v[i] = keep + __shfl_xor_sync(0xffffffffu, send, dist);
                }
            }
            const Acc tot = v[0];
            const size_t blk = 36 * (size_t)(I.half_offset[node] + node);
            typename BlockStore<MIXED>::V* store = BlockStore<MIXED>::ptr(I);
            if (lane < 21) {
                const Acc d = tot + (orr == okk ? (Acc)1e-2f : (Acc)0);  // damping
                I.diag[36 * (size_t)node + 6 * orr + okk] = (float)d;
                I.diag[36 * (size_t)node + 6 * okk + orr] = (float)d;
                store[blk + blk_idx(orr, okk)] = d;
                store[blk + blk_idx(okk, orr)] = d;
                s_blocks[j][lane] = d;
            } else if (lane < 27) {
                PcgVec<MIXED>::jtr(I)[6 * (size_t)node + lane - 21] = tot;
            }
        }
        __syncthreads();
        if (warp == 0 && base + lane < I.N) {
            const uint32_t node = base + lane;
            Acc D[36];
#pragma unroll
            for (int r = 0; r < 6; ++r)
#pragma unroll
                for (int k2 = 0; k2 < 6; ++k2) D[6 * r + k2] = s_blocks[lane][r <= k2 ? sym_idx(r, k2) : sym_idx(k2, r)];
            if constexpr (MIXED) {
                double L[21];
                cholesky6(D, L);
#pragma unroll
                for (int i = 0; i < 21; ++i) I.chol[21 * (size_t)node + i] = L[i];
            } else {
                float Df[36], Mi[36];
#pragma unroll
                for (int i = 0; i < 36; ++i) Df[i] = (float)D[i];
                gauss_jordan6(Df, Mi);
#pragma unroll
                for (int i = 0; i < 36; ++i) I.minv[36 * (size_t)node + i] = Mi[i];
            }
        }
        __syncthreads();
    }
}

// --------------------------------------------------- off-diagonal blocks --
// One thread per unordered pair (i < j), accumulating in registers. Every
// term type but smooth contributes w_i w_j lambda^2 sum_c g_c g_c^T (dense and
// foreground: one channel g = J; feature and cross: three Huber-weighted twist
// rows), a symmetric product, so the thread keeps the 21 upper-triangle sums
// only. A pair has at most two smooth terms (its graph edges i->j and j->i);
// their asymmetric contribution -lambda_s^2 sum_c f_c(p_i) f_c(p_j)^T is added
// when the block is written. computeJtJNonDiagonalBlockKernel and
// computeSmoothJtJBlock (JtJMaterializer.cu:20-528, jtj_block_jacobian.cuh:8-65)
// compute the same sums; only the upper block (i, j) is stored, (j, i) is read
// as its transpose.
template <bool MIXED>
__global__ void __launch_bounds__(128, 4) offdiag_kernel(const InstDesc* insts, mvdr_penalty lam) {
    using Acc = typename std::conditional<MIXED, double, float>::type;
    const InstDesc& I = insts[blockIdx.y];
    const DeviceCounts* C = I.counts;
    if (C->node2term_entries > I.cap_k1 || C->half_pairs > I.cap_pairs || C->nodepair_entries > I.cap_k2) return;
    TermOffsets off;
    off.load(C);
    const uint32_t P = C->half_pairs;
    const Acc l2_fg = (Acc)(lam.foreground * lam.foreground);
    const Acc l2_feat = (Acc)(lam.feature * lam.feature), l2_cross = (Acc)(lam.cross_view * lam.cross_view);
    const bool dens_on = I.use_density && lam.density != 0.f;
    const Acc l2_dens = (Acc)(lam.density * lam.density);
    // pairs grouped by entry count, so the lanes of a warp loop equally long
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < P; i += gridDim.x * blockDim.x) {
        const uint32_t h = I.pair_order[i];
        const uint32_t ni = I.half_key[h] / I.enc;
        const uint2 rg = I.half_range[h];
        Acc S[21];
#pragma unroll
        for (int q = 0; q < 21; ++q) S[q] = 0;
        uint32_t smooth_k[2] = {kInvalid, kInvalid};
        // software pipeline over the pair's entries: the term id two entries
        // ahead and the pixel-term record one entry ahead are in flight while
        // the current entry is summed
        uint32_t t_next = rg.x < rg.y ? I.np_index[rg.x] : 0u;
        uint32_t t_next2 = rg.x + 1 < rg.y ? I.np_index[rg.x + 1] : 0u;
        float4 pa = make_float4(0.f, 0.f, 0.f, 0.f), pb = pa;
        float2 pw = make_float2(0.f, 0.f);
        auto fetch_pixel_term = [&](uint32_t t, uint32_t p) {
            uint32_t k;
            const TermType ty = off.typed(t, k);
            if (ty == kDense || ty == kForeground) {
                const uint32_t idx = ty == kDense ? k : off.o[0] + k;
                load_record32(I.term_jr + 2 * (size_t)idx, pa, pb);
                pw = I.np_w[p];
            }
        };
        if (rg.x < rg.y) fetch_pixel_term(t_next, rg.x);
        for (uint32_t p = rg.x; p < rg.y; ++p) {
            const uint32_t t = t_next;
            const float4 a = pa, b = pb;
            const float2 wij = pw;
            t_next = t_next2;
            if (p + 2 < rg.y) t_next2 = I.np_index[p + 2];
            if (p + 1 < rg.y) fetch_pixel_term(t_next, p + 1);
            uint32_t k;
            const TermType ty = off.typed(t, k);
            if (ty == kDense || ty == kForeground) {
                const Acc wij2 = (Acc)wij.x * (Acc)wij.y;
                if (__float_as_uint(b.w) != kInvalid) {  // an invalid term has J = 0
                    const Acc s = ty == kForeground ? wij2 * l2_fg : wij2;
                    const Acc g[6] = {(Acc)a.x, (Acc)a.y, (Acc)a.z, (Acc)a.w, (Acc)b.x, (Acc)b.y};
                    add_scaled_outer(S, s, g);
                }
                if (ty == kDense && dens_on) {
                    float4 da, db;
                    load_record32(I.density_jr + 2 * (size_t)k, da, db);
                    if (__float_as_uint(db.w) != kInvalid) {
                        const Acc g[6] = {(Acc)da.x, (Acc)da.y, (Acc)da.z, (Acc)da.w, (Acc)db.x, (Acc)db.y};
                        add_scaled_outer(S, wij2 * l2_dens, g);
                    }
                }
            } else if (ty == kSmooth) {
                if (smooth_k[0] == kInvalid) smooth_k[0] = k;
                else smooth_k[1] = k;
            } else if (ty == kFeature || ty == kCross) {
                const bool f = ty == kFeature;
                const float4 wv = I.warped[2 * (size_t)(f ? k : I.Tp + k)];
                const float4 rw = I.warped[2 * (size_t)(f ? k : I.Tp + k) + 1];
                const float2 wp = I.np_w[p];
                const Acc s = (Acc)wp.x * (Acc)wp.y * (f ? l2_feat : l2_cross);
                const float hw[3] = {huber_weight(rw.x), huber_weight(rw.y), huber_weight(rw.z)};
                Acc fr[3][6];
                twist_rows<Acc>((Acc)wv.x, (Acc)wv.y, (Acc)wv.z, fr);
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    Acc g[6];
#pragma unroll
                    for (int q = 0; q < 6; ++q) g[q] = (Acc)hw[c] * fr[c][q];
                    add_scaled_outer(S, s, g);
                }
            }
        }
        // smooth terms: J_i,c = +-f_c(p_i), J_j,c = -+f_c(p_j), so their
        // product carries a minus (geometry_icp_jacobian.cuh:323-343); the
        // elements of sum_c f_c(p_i) f_c(p_j)^T come from the two points
        Acc pi[2][3], pj[2][3];
        bool has[2] = {false, false};
#pragma unroll
        for (int m = 0; m < 2; ++m) {
            if (smooth_k[m] == kInvalid) continue;
            const uint32_t k = smooth_k[m];
            const float4 a = I.smooth[3 * (size_t)k], b = I.smooth[3 * (size_t)k + 1];
            if (b.z == 0.f) continue;
            const bool is_i = ni == I.graph[k].x;
            const float4 qi = is_i ? a : make_float4(a.w, b.x, b.y, 0.f);
            const float4 qj = is_i ? make_float4(a.w, b.x, b.y, 0.f) : a;
            pi[m][0] = (Acc)qi.x; pi[m][1] = (Acc)qi.y; pi[m][2] = (Acc)qi.z;
            pj[m][0] = (Acc)qj.x; pj[m][1] = (Acc)qj.y; pj[m][2] = (Acc)qj.z;
            has[m] = true;
        }
        const Acc l2_smooth = -(Acc)(lam.smooth * lam.smooth);
        typename BlockStore<MIXED>::V* out = BlockStore<MIXED>::ptr(I) + 36 * (size_t)(h + ni + 1);
#pragma unroll
        for (int r = 0; r < 6; ++r)
#pragma unroll
            for (int k = 0; k < 6; ++k) {
                Acc v = S[r <= k ? sym_idx(r, k) : sym_idx(k, r)];
#pragma unroll
                for (int m = 0; m < 2; ++m)
                    if (has[m]) v += l2_smooth * twist_rows_product<Acc>(pi[m], pj[m], r, k);
                out[blk_idx(r, k)] = v;
            }
    }
}

// ------------------------------------------------ scaled operator -------
// Mixed precision, materialised: the PCG runs on A^ = L^-1 A L^-T, where
// D_i = L_i L_i^T are the damped diagonal blocks (block-Jacobi scaling). Its
// diagonal blocks are the identity and its off-diagonal blocks
// A^_ij = L_i^-1 A_ij L_j^-T have entries of order one, so float storage and a
// float SpMV perturb the increment by about 1e-6 of its size, where float
// storage of A itself (condition numbers of the blocks up to 1e5) moves it by
// 1e-4 to 5e-4. In exact arithmetic the iterates are those of block-Jacobi PCG
// on A (BlockPCG.cuh:65-181): x = L^-T x^, r^ = L^-1 r, and r^.r^ = r.M^-1 r.
// This kernel forms A^_ij from the double block A_ij (i < j) that
// offdiag_kernel stored: 8 lanes per pair, lane k of the first six solves
// column k of L_i Y = A_ij, the pair's lanes exchange Y through shared memory,
// and lane k then solves L_j z = Y(k, :)^T, which is row k of A^_ij.
constexpr uint32_t kScalePairsPerCta = 16;

__device__ inline void chol_forward(const double* L, const double* b, double* y) {
#pragma unroll
    for (int r = 0; r < 6; ++r) {
        double t = b[r];
#pragma unroll
        for (int m = 0; m < r; ++m) t -= L[r * (r + 1) / 2 + m] * y[m];
        y[r] = t * L[r * (r + 1) / 2 + r];  // the diagonal holds reciprocals
    }
}

__device__ inline void chol_backward(const double* L, const double* y, double* x) {
#pragma unroll
    for (int r = 5; r >= 0; --r) {
        double t = y[r];
#pragma unroll
        for (int m = r + 1; m < 6; ++m) t -= L[m * (m + 1) / 2 + r] * x[m];
        x[r] = t * L[r * (r + 1) / 2 + r];
    }
}

__global__ void __launch_bounds__(128) scale_offdiag_kernel(const InstDesc* insts) {
    const InstDesc& I = insts[blockIdx.y];
    if (!index_complete(I)) return;
    const uint32_t P = I.counts->half_pairs;
    __shared__ double s_y[kScalePairsPerCta][6][7];
    const uint32_t lp = threadIdx.x >> 3, k = threadIdx.x & 7;
    for (uint32_t base = blockIdx.x * kScalePairsPerCta; base < P; base += gridDim.x * kScalePairsPerCta) {
        const uint32_t h = base + lp;
        const bool has = h < P && k < 6;
        size_t blk = 0;
        uint32_t j = 0;
        if (has) {
            const uint32_t key = I.half_key[h];
            const uint32_t i = key / I.enc;
            j = key % I.enc;
            blk = 36 * (size_t)(h + i + 1);
            double L[21], a[6], y[6];
#pragma unroll
            for (int q = 0; q < 21; ++q) L[q] = I.chol[21 * (size_t)i + q];
#pragma unroll
            for (int r = 0; r < 6; ++r) a[r] = I.bsr_d[blk + blk_idx(r, k)];
            chol_forward(L, a, y);
#pragma unroll
            for (int r = 0; r < 6; ++r) s_y[lp][r][k] = y[r];
        }
        __syncwarp();  // the 8 lanes of a pair are in one warp
        if (has) {
            double L[21], yr[6], z[6];
#pragma unroll
            for (int q = 0; q < 21; ++q) L[q] = I.chol[21 * (size_t)j + q];
#pragma unroll
            for (int c = 0; c < 6; ++c) yr[c] = s_y[lp][k][c];
            chol_forward(L, yr, z);
            float4* out = reinterpret_cast<float4*>(I.bsr_s + (blk / 36) * kScaledBlock + kScaledRow * k);
            out[0] = make_float4((float)z[0], (float)z[1], (float)z[2], (float)z[3]);
            out[1] = make_float4((float)z[4], (float)z[5], 0.f, 0.f);
        }
        __syncwarp();
    }
}

// x = L^-T x^ per node: the increment of the unscaled system, in place
__global__ void __launch_bounds__(128) pcg_unscale_kernel(const InstDesc* insts) {
    const InstDesc& I = insts[blockIdx.y];
    for (uint32_t node = blockIdx.x * blockDim.x + threadIdx.x; node < I.N; node += gridDim.x * blockDim.x) {
        double L[21], xh[6], x[6];
#pragma unroll
        for (int q = 0; q < 21; ++q) L[q] = I.chol[21 * (size_t)node + q];
#pragma unroll
        for (int q = 0; q < 6; ++q) xh[q] = I.x_d[6 * (size_t)node + q];
        chol_backward(L, xh, x);
#pragma unroll
        for (int q = 0; q < 6; ++q) I.x_d[6 * (size_t)node + q] = x[q];
    }
}

// ----------------------------------------------------------- reductions ---
// Split reduction for the PCG dots. Every CTA of the producing launch stores
// its block sum in a region of the partials; a kernel launched after it on
// the same stream sums the stored partials with one warp in a fixed order.
// Each consuming CTA computes the same value, and no producing CTA waits for
// the others (no ticket, fence or atomic on the SpMV's critical path).
// Regions: kRegDelta + parity holds delta = r.s of the iteration with that
// parity (pcg_init writes iteration 0's, pcg_update the next one's), kRegDq
// holds d.q of the current iteration; the scaled SpMV also stores r.q and q.q
// (kRegRq, kRegQq), from which the fused update forms the next delta.
constexpr uint32_t kRegDelta = 1, kRegDq = 3, kRegRq = 5, kRegQq = 6;

template <class T>
__device__ inline void store_block_partial(const InstDesc& I, uint32_t region, T v, uint32_t slot = 0xFFFFFFFFu) {
    __shared__ T ws[32];
    v = warp_sum(v);
    if (lane_id() == 0) ws[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        T s = 0;
        for (uint32_t w = 0; w < (blockDim.x >> 5); ++w) s += ws[w];
        I.partials[(size_t)region * I.part_stride + (slot == 0xFFFFFFFFu ? blockIdx.x : slot)] = (double)s;
    }
}

// three block sums at once (one barrier), to three regions
template <class T>
__device__ inline void store_block_partials3(const InstDesc& I, uint32_t r0, T v0, uint32_t r1, T v1, uint32_t r2,
                                             T v2) {
    __shared__ T ws3[3][32];
    v0 = warp_sum(v0);
    v1 = warp_sum(v1);
    v2 = warp_sum(v2);
    if (lane_id() == 0) {
        ws3[0][threadIdx.x >> 5] = v0;
        ws3[1][threadIdx.x >> 5] = v1;
        ws3[2][threadIdx.x >> 5] = v2;
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        T s = 0;
        for (uint32_t w = 0; w < (blockDim.x >> 5); ++w) s += ws3[threadIdx.x][w];
        const uint32_t r = threadIdx.x == 0 ? r0 : (threadIdx.x == 1 ? r1 : r2);
        I.partials[(size_t)r * I.part_stride + blockIdx.x] = (double)s;
    }
}

// The sums of the partials of four regions (warp w sums regions w, w + warps,
// ...; each in a fixed order), in every thread. blockDim.x >= 64.
template <class T>
__device__ inline void sum_four_block_partials(const InstDesc& I, const uint32_t (&reg)[4], const uint32_t (&cnt)[4],
                                               T (&out)[4]) {
    __shared__ T total[4];
    const uint32_t warps = blockDim.x >> 5;
    for (uint32_t q = threadIdx.x >> 5; q < 4; q += warps) {
        const double* p = I.partials + (size_t)reg[q] * I.part_stride;
        T s = 0;
        for (uint32_t c = lane_id(); c < cnt[q]; c += 32) s += (T)__ldcg(p + c);
        s = warp_sum(s);
        if (lane_id() == 0) total[q] = s;
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < 4; ++q) out[q] = total[q];
}

// The sums of the partials of two regions (warp 0 sums region a, warp 1
// region b, each in a fixed order), in every thread. blockDim.x >= 64.
template <class T>
__device__ inline void sum_two_block_partials(const InstDesc& I, uint32_t ra, uint32_t na, uint32_t rb, uint32_t nb,
                                              T* a, T* b) {
    __shared__ T total[2];
    const uint32_t w = threadIdx.x >> 5;
    if (w < 2) {
        const double* p = I.partials + (size_t)(w == 0 ? ra : rb) * I.part_stride;
        const uint32_t n = w == 0 ? na : nb;
        T s = 0;
        for (uint32_t c = lane_id(); c < n; c += 32) s += (T)__ldcg(p + c);
        s = warp_sum(s);
        if (lane_id() == 0) total[w] = s;
    }
    __syncthreads();
    *a = total[0];
    *b = total[1];
}

// beta = delta_k / delta_(k-1) of iteration k (0 for the first), from the
// `nd` partials of the init / update launches; *delta receives delta_k
template <class T>
__device__ inline T pcg_beta(const InstDesc& I, int parity, int first, uint32_t nd, T* delta = nullptr) {
    T dk, dkm1;
    sum_two_block_partials<T>(I, kRegDelta + parity, nd, kRegDelta + (parity ^ 1), nd, &dk, &dkm1);
    if (delta) *delta = dk;
    // a zero delta_(k-1) (the residual vanished) restarts with d = s
    return first || dkm1 == (T)0 ? (T)0 : dk / dkm1;
}

// The convergence check (BlockPCG::SolveConvergeChecked, BlockPCG.cuh:
// 339-377) stopped this instance's PCG solve: its later iterations' kernels
// return at once. Only with a tolerance; the flag is cleared by pcg_init.
__device__ inline bool pcg_stopped(const InstDesc& I) {
    return I.pcg_tol > 0.f && *(volatile const uint32_t*)&I.counts->pcg_stop != 0u;
}

// alpha = delta / d.q; a zero d.q (an exactly zero right-hand side) gives a
// zero step where the reference (BlockPCG.cuh:120-161) divides 0 by 0. A
// non-finite alpha (NaN or Inf reached the system) flags the instance, from
// the instance's `leader` CTA only.
template <class T> __device__ inline T pcg_alpha(const InstDesc& I, T delta, T dq, bool leader) {
    const T alpha = dq != (T)0 ? delta / dq : (T)0;
    if (leader && threadIdx.x == 0 && !isfinite(alpha)) set_error(I, kErrNonFinite);
    return alpha;
}

// ---------------------------------------------------------------- PCG -----

// blockPCGZeroInitKernel (BlockPCG.cuh:65-111): r = b, s = M^-1 b, x = 0,
// delta = r.s; the first direction is d = s (beta = 0). SCALED (the scaled
// operator A^ of the materialised mixed mode): r^ = L^-1 b, s = r^,
// delta = r^.r^, the same delta.
template <bool MIXED, bool SCALED>
__global__ void __launch_bounds__(256) pcg_init_kernel(const InstDesc* insts) {
    static_assert(MIXED || !SCALED, "the scaled operator is mixed precision");
    const InstDesc& I = insts[blockIdx.y];
    using T = typename std::conditional<MIXED, double, float>::type;
    using PV = PcgVec<MIXED>;
    T part = 0;
    if (blockIdx.x == 0 && threadIdx.x == 0) I.counts->pcg_stop = 0u;
    for (uint32_t node = blockIdx.x * blockDim.x + threadIdx.x; node < I.N; node += gridDim.x * blockDim.x) {
        T bv[6], sv[6];
#pragma unroll
        for (int i = 0; i < 6; ++i) bv[i] = PV::jtr(I)[6 * (size_t)node + i];
        if constexpr (SCALED) {
            double L[21];
#pragma unroll
            for (int q = 0; q < 21; ++q) L[q] = I.chol[21 * (size_t)node + q];
            chol_forward(L, bv, sv);
#pragma unroll
            for (int i = 0; i < 6; ++i) bv[i] = sv[i];
        } else if constexpr (MIXED) {
            cholesky6_solve(I.chol + 21 * (size_t)node, bv, sv);
        } else {
#pragma unroll
            for (int j = 0; j < 6; ++j) {
                float a = 0.f;
#pragma unroll
                for (int i = 0; i < 6; ++i) a += I.minv[36 * (size_t)node + 6 * j + i] * bv[i];
                sv[j] = a;
            }
        }
#pragma unroll
        for (int i = 0; i < 6; ++i) {
            const size_t e = 6 * (size_t)node + i;
            PV::r(I)[e] = bv[i];
            PV::s(I)[e] = sv[i];
            PV::d(I, 1)[e] = 0;
            PV::x(I)[e] = 0;
            part += bv[i] * sv[i];
        }
    }
    store_block_partial<T>(I, kRegDelta, part);
}

// One scalar row r of y = A x for block row br, walking the full block-row
// layout over the half storage; accumulates in the storage precision.
template <bool MIXED>
__device__ inline float bsr_row(const InstDesc& I, uint32_t br, uint32_t r, const float* x) {
    using V = typename BlockStore<MIXED>::V;
    const V* store = BlockStore<MIXED>::ptr(I);
    const uint32_t e0 = I.blkrow_offset[br] + br, e1 = I.blkrow_offset[br + 1] + br + 1;
    V acc = 0;
    for (uint32_t e = e0; e < e1; ++e) {
        const uint2 ent = I.bsr_ent[e];
        const uint32_t pos = ent.x;
        const V* blk = store + 36 * (size_t)(pos & ~kTransposedBlock);
        const bool tr = (pos & kTransposedBlock) != 0;
        const float* xc = x + 6 * (size_t)ent.y;
#pragma unroll
        for (int k = 0; k < 6; ++k) acc += blk[tr ? blk_idx(k, r) : blk_idx(r, k)] * (V)xc[k];
    }
    return (float)acc;
}

// ----------------------------------------------------- PCG direction ----
// d = s + beta d_prev (BlockPCG.cuh:167-181), formed once per iteration for
// the whole vector, so that the SpMV reads its operand directly. SCALED: s is
// r^ itself, and the float copy of d that the float SpMV reads is written too.
// Every CTA sums the same partials in the same order, so all reach the same
// delta_k and the same convergence decision; CTA 0 records delta_k in the
// residual history of GN iteration `gn` and, on convergence, the stop.
template <bool MIXED, bool SCALED>
__global__ void __launch_bounds__(256) pcg_direction_kernel(const InstDesc* insts, int parity, int first,
                                                            uint32_t nd, uint32_t gn, uint32_t it) {
    const InstDesc& I = insts[blockIdx.y];
    using PV = PcgVec<MIXED>;
    using T = typename PV::T;
    if (pcg_stopped(I)) return;
    // one element per thread (the grid covers 6N), loaded before beta's sums
    const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    const bool has = e < 6 * I.N;
    const T* sp = SCALED ? PV::r(I) : PV::s(I);
    const T sv = has ? sp[e] : (T)0, dp = has ? PV::d(I, !parity)[e] : (T)0;
    T dk;
    const T beta = pcg_beta<T>(I, parity, first, nd, &dk);
    DeviceCounts* C = I.counts;
    double* hist = gn < kPcgHistRows ? I.pcg_hist + (size_t)gn * MVDR_PCG_HISTORY : nullptr;
    if (blockIdx.x == 0) {
        if (first) {
            if (threadIdx.x == 0) C->pcg_delta0 = (double)dk;
            if (hist)
                for (uint32_t k = 1 + threadIdx.x; k < MVDR_PCG_HISTORY; k += blockDim.x) hist[k] = __longlong_as_double(0x7ff8000000000000ll);
        }
        if (hist && threadIdx.x == 0 && it < MVDR_PCG_HISTORY) hist[it] = (double)dk;
    }
    if (!first && I.pcg_tol > 0.f) {
        const double d0 = first ? (double)dk : C->pcg_delta0;
        const double tol2 = (double)I.pcg_tol * (double)I.pcg_tol;
        if (fabs((double)dk) < tol2 * fabs(d0)) {
            if (blockIdx.x == 0 && threadIdx.x == 0) C->pcg_stop = it;
            return;
        }
    }
    if (has) {
        const T d = sv + beta * dp;
        PV::d(I, parity)[e] = d;
        if constexpr (SCALED) I.df[df_pos(e)] = (float)d;
    }
}

// ------------------------------------------------------- tiled SpMV -----
// A CTA owns ROWS consecutive block rows; SPLIT threads per scalar row take
// every SPLIT-th block of the row (the autotuner picks ROWS and SPLIT). Thread r of a row reads row r of each
// stored block (three pair loads; the six threads together sweep the block
// contiguously, see blk_idx) and the column's direction from the L2-resident
// d. For an upper or diagonal block that row gives y_r directly; for a lower
// block, stored as its transpose, it is column r of the needed block and adds
// x_r times it to all six rows, which the row's threads sum through shared
// memory at the end. Block and direction addresses depend only on the
// sequential (position, column) entries, so many loads stay in flight. The
// stored transpose of a lower block belongs to a row of this or an earlier
// tile, so it is usually still in L2.
const SpmvShape kSpmvShapes[kNumSpmvShapes] = {{16, 2, 0}, {8, 2, 0},  {16, 1, 0}, {32, 1, 0}, {16, 3, 0}, {8, 4, 0},
                                                {32, 2, 0}, {16, 1, 1}, {32, 1, 1}, {8, 2, 1},  {16, 2, 1}, {4, 4, 1}};

template <class V> struct Pair;
template <> struct Pair<double> { using type = double2; };
template <> struct Pair<float> { using type = float2; };

// the SpMV operand: this iteration's direction
template <bool MIXED> __device__ inline const typename BlockStore<MIXED>::V* direction(const InstDesc& I, int parity) {
    return PcgVec<MIXED>::d(I, parity);
}

// q = A d, d.q partial; alpha = delta / d.q
template <bool MIXED, uint32_t kTileRows, uint32_t kTileSplit>
__global__ void __launch_bounds__(6 * kTileSplit * kTileRows) pcg_spmv_kernel(const InstDesc* insts, int parity) {
    using V = typename BlockStore<MIXED>::V;
    using V2 = typename Pair<V>::type;
    __shared__ V s_cols[kTileRows][kTileSplit * 6][7];
    const InstDesc& I = insts[blockIdx.y];
    using T = typename std::conditional<MIXED, double, float>::type;
    const V* store = BlockStore<MIXED>::ptr(I);
    const V* xvec = direction<MIXED>(I, parity);
    const uint32_t t = threadIdx.x;
    T part = 0;
    const uint32_t r0 = blockIdx.x * kTileRows;
    if (pcg_stopped(I)) return;
    if (r0 < I.N && index_complete(I)) {
        const uint32_t r1 = min(r0 + kTileRows, I.N);
        const uint32_t lr = t / (6 * kTileSplit), half = (t / 6) % kTileSplit, rr = t % 6, row = r0 + lr;
        const bool computes = row < r1;
        V acc = 0;
        V col_acc[6] = {0, 0, 0, 0, 0, 0};
        if (computes) {
            const uint32_t rb = I.blkrow_offset[row] + row, re = I.blkrow_offset[row + 1] + row + 1;
#pragma unroll 2
            for (uint32_t b = rb + half; b < re; b += kTileSplit) {
                const uint2 ent = I.bsr_ent[b];
                const uint32_t pos = ent.x, col = ent.y;
                const V2* blk = reinterpret_cast<const V2*>(store + 36 * (size_t)(pos & ~kTransposedBlock));
                const V2 a01 = blk[rr], a23 = blk[6 + rr], a45 = blk[12 + rr];
                const V av[6] = {a01.x, a01.y, a23.x, a23.y, a45.x, a45.y};
                const V* xc = xvec + 6 * (size_t)col;
                if (pos & kTransposedBlock) {
                    const V xr = xc[rr];
#pragma unroll
                    for (int k = 0; k < 6; ++k) col_acc[k] += av[k] * xr;
                } else {
                    const V2* x2 = reinterpret_cast<const V2*>(xc);
                    const V2 x01 = x2[0], x23 = x2[1], x45 = x2[2];
                    const V xv[6] = {x01.x, x01.y, x23.x, x23.y, x45.x, x45.y};
#pragma unroll
                    for (int k = 0; k < 6; ++k) acc += av[k] * xv[k];
                }
            }
            // slot 6 of a thread's row-sum entry holds its direct (row) sum
#pragma unroll
            for (int k = 0; k < 6; ++k) s_cols[lr][6 * half + rr][k] = col_acc[k];
            s_cols[lr][6 * half + rr][6] = acc;
        }
        __syncthreads();
        if (computes && half == 0) {
            acc = 0;
#pragma unroll
            for (uint32_t h = 0; h < kTileSplit; ++h) {
                acc += s_cols[lr][6 * h + rr][6];
#pragma unroll
                for (int c = 0; c < 6; ++c) acc += s_cols[lr][6 * h + c][rr];
            }
            const size_t e = 6 * (size_t)row + rr;
            PcgVec<MIXED>::q(I)[e] = acc;
            part += (T)xvec[e] * (T)acc;
        }
    }
    store_block_partial<T>(I, kRegDq, part);
}

// Column form: thread r of a row reads, for a lower entry, column r of the
// stored block (six scalar loads from the three 96-byte pair columns), so
// every entry adds to the thread's own q_r and no shared-memory exchange is
// needed; SPLIT > 1 sums the split threads' q_r in shared memory.
template <bool MIXED, uint32_t kTileRows, uint32_t kTileSplit>
__global__ void __launch_bounds__(6 * kTileSplit * kTileRows) pcg_spmv_col_kernel(const InstDesc* insts, int parity) {
    using V = typename BlockStore<MIXED>::V;
    using V2 = typename Pair<V>::type;
    using T = typename std::conditional<MIXED, double, float>::type;
    static_assert((6 * kTileSplit * kTileRows) % 32 == 0, "whole warps");
    __shared__ V s_part[kTileSplit > 1 ? kTileRows * 6 * kTileSplit : 1];
    const InstDesc& I = insts[blockIdx.y];
    const V* store = BlockStore<MIXED>::ptr(I);
    const V* xvec = direction<MIXED>(I, parity);
    const uint32_t t = threadIdx.x;
    T part = 0;
    const uint32_t r0 = blockIdx.x * kTileRows;
    if (pcg_stopped(I)) return;
    if (r0 < I.N && index_complete(I)) {
        const uint32_t r1 = min(r0 + kTileRows, I.N);
        const uint32_t lr = t / (6 * kTileSplit), half = (t / 6) % kTileSplit, rr = t % 6, row = r0 + lr;
        const bool computes = row < r1;
        V acc = 0;
        if (computes) {
            const uint32_t rb = I.blkrow_offset[row] + row, re = I.blkrow_offset[row + 1] + row + 1;
            const uint32_t cfirst = blk_idx(0, rr);  // column rr: cfirst + 2k, k = 0..5
#pragma unroll 2
            for (uint32_t b = rb + half; b < re; b += kTileSplit) {
                const uint2 ent = I.bsr_ent[b];
                const V* blk = store + 36 * (size_t)(ent.x & ~kTransposedBlock);
                const V2* x2 = reinterpret_cast<const V2*>(xvec + 6 * (size_t)ent.y);
                const V2 x01 = x2[0], x23 = x2[1], x45 = x2[2];
                const V xv[6] = {x01.x, x01.y, x23.x, x23.y, x45.x, x45.y};
                V av[6];
                if (ent.x & kTransposedBlock) {
#pragma unroll
                    for (int k = 0; k < 6; ++k) av[k] = blk[cfirst + 2 * k];
                } else {
                    const V2* b2 = reinterpret_cast<const V2*>(blk);
                    const V2 a01 = b2[rr], a23 = b2[6 + rr], a45 = b2[12 + rr];
                    av[0] = a01.x; av[1] = a01.y; av[2] = a23.x; av[3] = a23.y; av[4] = a45.x; av[5] = a45.y;
                }
#pragma unroll
                for (int k = 0; k < 6; ++k) acc += av[k] * xv[k];
            }
        }
        if constexpr (kTileSplit > 1) {
            if (computes) s_part[(lr * kTileSplit + half) * 6 + rr] = acc;
            __syncthreads();
            if (computes && half == 0) {
                acc = 0;
#pragma unroll
                for (uint32_t h = 0; h < kTileSplit; ++h) acc += s_part[(lr * kTileSplit + h) * 6 + rr];
            }
        }
        if (computes && half == 0) {
            const size_t e = 6 * (size_t)row + rr;
            PcgVec<MIXED>::q(I)[e] = acc;
            part += (T)xvec[e] * (T)acc;
        }
    }
    store_block_partial<T>(I, kRegDq, part);
}

// SpMV of the scaled operator (mixed precision, materialised):
// q^_i = d^_i + sum_{j != i} A^_ij d^_j. The identity diagonal is not read;
// the off-diagonal blocks are float, row-major, and the product runs in
// float on the float copy of d^ (about 1e-7 relative per row, far below the
// 1e-4 budget of the increment); q^ and the d^.q^ partial are double. An
// upper entry (j > i) reads row r of its stored block; a lower entry reads
// the stored A^_ji, whose column r is row r of A^_ij: FORM 1 reads that
// column (six 4-byte loads), FORM 0 reads row r of A^_ji and adds d^_j(r)
// times it to all six rows, which the row's threads sum through shared
// memory at the end. The float blocks are row-major with each row padded to
// 32 bytes (kScaledRow), so a thread reads its block row, and the column's
// float direction, in one 256-bit load each, and the six threads of a row
// read one stored block as 192 contiguous bytes.
template <uint32_t kTileRows, uint32_t kTileSplit, uint32_t kForm>
__global__ void __launch_bounds__(6 * kTileSplit * kTileRows) pcg_spmv_scaled_kernel(const InstDesc* insts,
                                                                                  int parity) {
    static_assert((6 * kTileSplit * kTileRows) % 32 == 0, "whole warps");
    constexpr uint32_t kSlots = kForm == 0 ? 7 : 1;  // per thread: column sums (form 0) and its row sum
    __shared__ float s_x[(kForm == 0 || kTileSplit > 1) ? kTileRows * kTileSplit * 6 * kSlots : 1];
    const InstDesc& I = insts[blockIdx.y];
    const float* store = I.bsr_s;
    const float* xf = I.df;
    const double* xd = PcgVec<true>::d(I, parity);
    const uint32_t t = threadIdx.x;
    double part = 0, prq = 0, pqq = 0;  // d.q, r.q, q.q
    const uint32_t r0 = blockIdx.x * kTileRows;
    if (pcg_stopped(I)) return;
    if (r0 < I.N && index_complete(I)) {
        const uint32_t r1 = min(r0 + kTileRows, I.N);
        const uint32_t lr = t / (6 * kTileSplit), half = (t / 6) % kTileSplit, rr = t % 6, row = r0 + lr;
        const bool computes = row < r1;
        float acc = 0.f;
        float col_acc[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        if (computes) {
            // the row's first entry is its diagonal block: the identity, added below
            const uint32_t rb = I.blkrow_offset[row] + row + 1, re = I.blkrow_offset[row + 1] + row + 1;
#pragma unroll 2
            for (uint32_t b = rb + half; b < re; b += kTileSplit) {
                const uint2 ent = I.bsr_ent[b];
                const float* blk = store + kScaledBlock * (size_t)(ent.x & ~kTransposedBlock);
                const float* xc = xf + kScaledRow * (size_t)ent.y;
                const bool lower = (ent.x & kTransposedBlock) != 0;
                if (kForm == 0 && lower) {
                    float av[8];
                    load8f(blk + kScaledRow * rr, av);
                    const float xr = xc[rr];
#pragma unroll
                    for (int k = 0; k < 6; ++k) col_acc[k] += av[k] * xr;
                } else {
                    float av[8], xv[8];
                    if (lower) {
#pragma unroll
                        for (int k = 0; k < 6; ++k) av[k] = blk[kScaledRow * k + rr];
                    } else {
                        load8f(blk + kScaledRow * rr, av);
                    }
                    load8f(xc, xv);
                    acc += av[0] * xv[0] + av[1] * xv[1] + av[2] * xv[2] + av[3] * xv[3] + av[4] * xv[4] +
                           av[5] * xv[5];
                }
            }
        }
        if constexpr (kForm == 0 || kTileSplit > 1) {
            // slot 6 (form 0) / slot 0 holds a thread's row sum, slots 0-5 its column sums
            float* mine = s_x + ((lr * kTileSplit + half) * 6 + rr) * kSlots;
            if (computes) {
                if constexpr (kForm == 0) {
#pragma unroll
                    for (int k = 0; k < 6; ++k) mine[k] = col_acc[k];
                    mine[6] = acc;
                } else {
                    mine[0] = acc;
                }
            }
            __syncthreads();
            if (computes && half == 0) {
                acc = 0.f;
#pragma unroll
                for (uint32_t hh = 0; hh < kTileSplit; ++hh) {
                    const float* base = s_x + (lr * kTileSplit + hh) * 6 * kSlots;
                    if constexpr (kForm == 0) {
                        acc += base[rr * kSlots + 6];
#pragma unroll
                        for (int c = 0; c < 6; ++c) acc += base[c * kSlots + rr];
                    } else {
                        acc += base[rr];
                    }
                }
            }
        }
        if (computes && half == 0) {
            const size_t e = 6 * (size_t)row + rr;
            const double dv = xd[e];
            const double q = dv + (double)acc;
            PcgVec<true>::q(I)[e] = q;
            part += dv * q;
            prq += PcgVec<true>::r(I)[e] * q;
            pqq += q * q;
        }
    }
    store_block_partials3<double>(I, kRegDq, part, kRegRq, prq, kRegQq, pqq);
}

// blockPCGSecondUpdateKernel (BlockPCG.cuh:120-161): alpha = delta / d.q,
// x += alpha d, r -= alpha q, s = M^-1 r, delta_new = r.s (beta follows in
// the next direction). A thread per node; the grid covers every node. The
// node's vectors and preconditioner are loaded before the partial sums, so
// their latency overlaps the sums. `nd` and `nq`: CTAs of the launches that
// stored the delta and d.q partials. SCALED: the preconditioner is the
// identity (s = r^, not stored), delta_new = r^.r^.
// FUSE (the scaled form): the kernel also forms the next direction
// d_(k+1) = r^_(k+1) + beta d_k, so that no direction kernel runs between
// iterations. beta = delta_(k+1) / delta_k needs delta_(k+1) before any CTA
// has finished, so it is taken from the identity
// r_(k+1).r_(k+1) = delta_k - 2 alpha r_k.q_k + alpha^2 q_k.q_k, with the
// r.q and q.q sums that the SpMV stored; the directly summed delta_(k+1)
// (this kernel's partials) still gives the next alpha and the residual
// history, recorded here for iteration `it` of GN iteration `gn`. With a
// tolerance the convergence test of iteration `it` (the direction kernel's)
// is made here: on a stop no CTA applies the step, so the solve equals the
// fixed-count solve of `it` iterations.
template <bool MIXED, bool SCALED, bool FUSE>
__global__ void __launch_bounds__(256) pcg_update_kernel(const InstDesc* insts, int parity, uint32_t nd,
                                                         uint32_t nq, uint32_t gn, uint32_t it) {
    static_assert(!FUSE || SCALED, "the fused direction is the scaled form's");
    const InstDesc& I = insts[blockIdx.y];
    if (pcg_stopped(I)) return;
    using PV = PcgVec<MIXED>;
    using T = typename PV::T;
    using T2 = typename Pair<T>::type;
    constexpr int kPre = SCALED ? 1 : (MIXED ? 21 : 36);  // Cholesky factor / inverse entries
    const uint32_t node = blockIdx.x * blockDim.x + threadIdx.x;
    const bool has = node < I.N;
    T xv[6], dv[6], rv[6], qv[6];
    T pre[kPre];
    if (has) {
        auto load6 = [&](const T* v, T out[6]) {
            const T2* p = reinterpret_cast<const T2*>(v + 6 * (size_t)node);
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                const T2 w = p[i];
                out[2 * i] = w.x;
                out[2 * i + 1] = w.y;
            }
        };
        load6(PV::x(I), xv);
        load6(PV::d(I, parity), dv);
        load6(PV::r(I), rv);
        load6(PV::q(I), qv);
#pragma unroll
        for (int i = 0; i < kPre; ++i) {
            if constexpr (SCALED) pre[i] = 0;
            else if constexpr (MIXED) pre[i] = I.chol[21 * (size_t)node + i];
            else pre[i] = I.minv[36 * (size_t)node + i];
        }
    }
    T delta, dq, rq = 0, qq = 0;
    if constexpr (FUSE) {
        T sums[4];
        sum_four_block_partials<T>(I, {kRegDelta + (uint32_t)parity, kRegDq, kRegRq, kRegQq}, {nd, nq, nq, nq}, sums);
        delta = sums[0];
        dq = sums[1];
        rq = sums[2];
        qq = sums[3];
        double* hist = gn < kPcgHistRows ? I.pcg_hist + (size_t)gn * MVDR_PCG_HISTORY : nullptr;
        if (blockIdx.x == 0 && threadIdx.x == 0 && hist && it < MVDR_PCG_HISTORY) hist[it] = (double)delta;
        if (it > 0 && I.pcg_tol > 0.f) {
            const double tol2 = (double)I.pcg_tol * (double)I.pcg_tol;
            if (fabs((double)delta) < tol2 * fabs(I.counts->pcg_delta0)) {
                if (blockIdx.x == 0 && threadIdx.x == 0) I.counts->pcg_stop = it;
                return;  // the same decision in every thread of every CTA
            }
        }
    } else {
        sum_two_block_partials<T>(I, kRegDelta + parity, nd, kRegDq, nq, &delta, &dq);
    }
    const T alpha = pcg_alpha<T>(I, delta, dq, blockIdx.x == 0);
    T part = 0;
    if (has) {
        T sv[6];
#pragma unroll
        for (int i = 0; i < 6; ++i) {
            xv[i] += alpha * dv[i];
            rv[i] -= alpha * qv[i];
        }
        if constexpr (SCALED) {
#pragma unroll
            for (int i = 0; i < 6; ++i) sv[i] = rv[i];
        } else if constexpr (MIXED) {
            cholesky6_solve(pre, rv, sv);
        } else {
#pragma unroll
            for (int j = 0; j < 6; ++j) {
                float a = 0.f;
#pragma unroll
                for (int i = 0; i < 6; ++i) a += pre[6 * j + i] * rv[i];
                sv[j] = a;
            }
        }
        auto store6 = [&](T* v, const T in[6]) {
            T2* p = reinterpret_cast<T2*>(v + 6 * (size_t)node);
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                T2 w;
                w.x = in[2 * i];
                w.y = in[2 * i + 1];
                p[i] = w;
            }
        };
        store6(PV::x(I), xv);
        store6(PV::r(I), rv);
        if constexpr (!SCALED) store6(PV::s(I), sv);
#pragma unroll
        for (int i = 0; i < 6; ++i) part += rv[i] * sv[i];
        if constexpr (FUSE) {
            const T dnext = delta - (T)2 * alpha * rq + alpha * alpha * qq;
            const T beta = delta != (T)0 ? dnext / delta : (T)0;  // a vanished residual restarts with d = r^
            T dn[6];
#pragma unroll
            for (int i = 0; i < 6; ++i) dn[i] = rv[i] + beta * dv[i];
            store6(PV::d(I, parity ^ 1), dn);
            float4* f = reinterpret_cast<float4*>(I.df + kScaledRow * (size_t)node);
            f[0] = make_float4((float)dn[0], (float)dn[1], (float)dn[2], (float)dn[3]);
            f[1] = make_float4((float)dn[4], (float)dn[5], 0.f, 0.f);
        }
    }
    store_block_partial<T>(I, kRegDelta + (parity ^ 1), part);
}

// ------------------------------------------------------ persistent PCG ---
// One cooperative launch runs every PCG iteration of every instance. The
// CTAs are split among the instances (one each, the rest in proportion to
// their node counts: the per-instance work queues); an instance's CTAs run
// init, then per iteration the direction, the SpMV (column form, kPersistRows
// block rows per tile) and the update, and meet at an instance barrier
// between steps. Instances never wait for one another, so one instance's
// barrier and reduction latency overlaps the others' loads. The dots are the
// same split reductions as in the launched form, with one partial per CTA of
// the instance.
constexpr uint32_t kPersistThreads = 256, kPersistRows = 40;

__device__ inline uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ inline uint32_t ld_acquire_u32(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// All CTAs of the instance arrive; returns false (and flags the instance)
// when the wait exceeds limit_ns.
__device__ inline bool instance_barrier(const InstDesc& I, uint32_t* ctr, uint32_t target, uint64_t limit_ns) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        atomicAdd(ctr, 1u);
        int ok = 1;
        if (ld_acquire_u32(ctr) < target) {
            const uint64_t t0 = global_ns();
            while (ld_acquire_u32(ctr) < target) {
                if (global_ns() - t0 > limit_ns) {
                    ok = 0;
                    set_error(I, kErrWaitTimeout);
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

template <bool MIXED>
__global__ void __launch_bounds__(kPersistThreads, 3) pcg_persistent_kernel(const InstDesc* insts, uint32_t B,
                                                                              uint32_t iters, uint64_t limit_ns,
                                                                              uint32_t extra) {
    using PV = PcgVec<MIXED>;
    using T = typename PV::T;
    using V = typename BlockStore<MIXED>::V;
    using V2 = typename Pair<V>::type;
    // this CTA's instance: instance i owns CTAs [i + (G - B) P_i / P, ...),
    // P_i the nodes of the instances before it
    const uint32_t G = gridDim.x;
    uint64_t total = 0;
    for (uint32_t i = 0; i < B; ++i) total += insts[i].N;
    uint32_t inst = 0, c0 = 0, c1 = 0;
    uint64_t pre = 0;
    for (uint32_t i = 0; i < B; ++i) {
        const uint64_t nxt = pre + insts[i].N;
        const uint32_t b0 = i + (uint32_t)((G - B) * pre / (total ? total : 1));
        const uint32_t b1 = i + 1 + (uint32_t)((G - B) * nxt / (total ? total : 1));
        if (blockIdx.x >= b0 && blockIdx.x < b1) { inst = i; c0 = b0; c1 = b1; }
        pre = nxt;
    }
    const InstDesc& I = insts[inst];
    const uint32_t c = blockIdx.x - c0, nc = c1 - c0;
    uint32_t* bar = I.pcg_bar;
    uint32_t passed = 0;
    const uint32_t tid = threadIdx.x, nt = blockDim.x;
    const bool index_ok = index_complete(I);
    // init: r = b, s = M^-1 b, x = 0, d_prev = 0, delta_0. Mixed precision
    // runs on the scaled operator (scale_offdiag_kernel): r^ = L^-1 b, s = r^.
    {
        T part = 0;
        for (uint32_t node = c * nt + tid; node < I.N; node += nc * nt) {
            T bv[6], sv[6];
#pragma unroll
            for (int i = 0; i < 6; ++i) bv[i] = PV::jtr(I)[6 * (size_t)node + i];
            if constexpr (MIXED) {
                double L[21];
#pragma unroll
                for (int q = 0; q < 21; ++q) L[q] = I.chol[21 * (size_t)node + q];
                chol_forward(L, bv, sv);
#pragma unroll
                for (int i = 0; i < 6; ++i) bv[i] = sv[i];
            } else {
#pragma unroll
                for (int j = 0; j < 6; ++j) {
                    float a = 0.f;
#pragma unroll
                    for (int i = 0; i < 6; ++i) a += I.minv[36 * (size_t)node + 6 * j + i] * bv[i];
                    sv[j] = a;
                }
            }
#pragma unroll
            for (int i = 0; i < 6; ++i) {
                const size_t e = 6 * (size_t)node + i;
                PV::r(I)[e] = bv[i];
                PV::s(I)[e] = sv[i];
                PV::d(I, 1)[e] = 0;
                PV::x(I)[e] = 0;
                part += bv[i] * sv[i];
            }
        }
        store_block_partial<T>(I, kRegDelta, part, c);
    }
    if (!instance_barrier(I, bar, ++passed * nc + extra, limit_ns)) return;
    for (uint32_t it = 0; it < iters; ++it) {
        const int parity = (int)(it & 1u);
        // direction
        {
            const T beta = pcg_beta<T>(I, parity, it == 0, nc);
            const T* dprev = PV::d(I, !parity);
            T* dcur = PV::d(I, parity);
            const T* sv = MIXED ? PV::r(I) : PV::s(I);
            for (uint32_t e = c * nt + tid; e < 6 * I.N; e += nc * nt) {
                const T dv = sv[e] + beta * dprev[e];
                dcur[e] = dv;
                if constexpr (MIXED) I.df[df_pos(e)] = (float)dv;
            }
        }
        if (!instance_barrier(I, bar, ++passed * nc + extra, limit_ns)) return;
        // SpMV over tiles of kPersistRows block rows, column form (mixed
        // precision: the scaled operator in float, as pcg_spmv_scaled_kernel)
        if constexpr (MIXED) {
            const double* xd = PV::d(I, parity);
            double part = 0;
            const uint32_t lr = tid / 6, rr = tid % 6;
            for (uint32_t r0 = c * kPersistRows; index_ok && r0 < I.N; r0 += nc * kPersistRows) {
                const uint32_t row = r0 + lr;
                if (lr >= kPersistRows || row >= I.N) continue;
                const uint32_t rb = I.blkrow_offset[row] + row + 1, re = I.blkrow_offset[row + 1] + row + 1;
                float acc = 0.f;
#pragma unroll 2
                for (uint32_t b = rb; b < re; ++b) {
                    const uint2 ent = I.bsr_ent[b];
                    const float* blk = I.bsr_s + kScaledBlock * (size_t)(ent.x & ~kTransposedBlock);
                    float av[8], xv[8];
                    if (ent.x & kTransposedBlock) {
#pragma unroll
                        for (int k = 0; k < 6; ++k) av[k] = blk[kScaledRow * k + rr];
                    } else {
                        load8f(blk + kScaledRow * rr, av);
                    }
                    load8f(I.df + kScaledRow * (size_t)ent.y, xv);
                    acc += av[0] * xv[0] + av[1] * xv[1] + av[2] * xv[2] + av[3] * xv[3] + av[4] * xv[4] +
                           av[5] * xv[5];
                }
                const size_t e = 6 * (size_t)row + rr;
                const double q = xd[e] + (double)acc;
                PV::q(I)[e] = q;
                part += xd[e] * q;
            }
            store_block_partial<double>(I, kRegDq, part, c);
        } else {
            const V* store = BlockStore<MIXED>::ptr(I);
            const V* xvec = PV::d(I, parity);
            T part = 0;
            const uint32_t lr = tid / 6, rr = tid % 6;
            for (uint32_t r0 = c * kPersistRows; index_ok && r0 < I.N; r0 += nc * kPersistRows) {
                const uint32_t row = r0 + lr;
                if (lr >= kPersistRows || row >= I.N) continue;
                const uint32_t rb = I.blkrow_offset[row] + row, re = I.blkrow_offset[row + 1] + row + 1;
                const uint32_t cfirst = blk_idx(0, rr);
                V acc = 0;
#pragma unroll 2
                for (uint32_t b = rb; b < re; ++b) {
                    const uint2 ent = I.bsr_ent[b];
                    const V* blk = store + 36 * (size_t)(ent.x & ~kTransposedBlock);
                    const V2* x2 = reinterpret_cast<const V2*>(xvec + 6 * (size_t)ent.y);
                    const V2 x01 = x2[0], x23 = x2[1], x45 = x2[2];
                    const V xv[6] = {x01.x, x01.y, x23.x, x23.y, x45.x, x45.y};
                    V av[6];
                    if (ent.x & kTransposedBlock) {
#pragma unroll
                        for (int k = 0; k < 6; ++k) av[k] = blk[cfirst + 2 * k];
                    } else {
                        const V2* b2 = reinterpret_cast<const V2*>(blk);
                        const V2 a01 = b2[rr], a23 = b2[6 + rr], a45 = b2[12 + rr];
                        av[0] = a01.x; av[1] = a01.y; av[2] = a23.x; av[3] = a23.y; av[4] = a45.x; av[5] = a45.y;
                    }
#pragma unroll
                    for (int k = 0; k < 6; ++k) acc += av[k] * xv[k];
                }
                const size_t e = 6 * (size_t)row + rr;
                PV::q(I)[e] = acc;
                part += (T)xvec[e] * (T)acc;
            }
            store_block_partial<T>(I, kRegDq, part, c);
        }
        if (!instance_barrier(I, bar, ++passed * nc + extra, limit_ns)) return;
        // update: alpha = delta / d.q, x, r, s, delta_new
        {
            T delta, dq;
            sum_two_block_partials<T>(I, kRegDelta + parity, nc, kRegDq, nc, &delta, &dq);
            const T alpha = pcg_alpha<T>(I, delta, dq, c == 0);
            const T* d = PV::d(I, parity);
            T part = 0;
            for (uint32_t node = c * nt + tid; node < I.N; node += nc * nt) {
                T rv[6], sv[6];
#pragma unroll
                for (int i = 0; i < 6; ++i) {
                    const size_t e = 6 * (size_t)node + i;
                    PV::x(I)[e] += alpha * d[e];
                    rv[i] = PV::r(I)[e] - alpha * PV::q(I)[e];
                    PV::r(I)[e] = rv[i];
                }
                if constexpr (MIXED) {
#pragma unroll
                    for (int i = 0; i < 6; ++i) sv[i] = rv[i];  // the scaled operator: s = r^
                } else {
#pragma unroll
                    for (int j = 0; j < 6; ++j) {
                        float a = 0.f;
#pragma unroll
                        for (int i = 0; i < 6; ++i) a += I.minv[36 * (size_t)node + 6 * j + i] * rv[i];
                        sv[j] = a;
                    }
                }
#pragma unroll
                for (int i = 0; i < 6; ++i) {
                    if constexpr (!MIXED) PV::s(I)[6 * (size_t)node + i] = sv[i];
                    part += rv[i] * sv[i];
                }
            }
            store_block_partial<T>(I, kRegDelta + (parity ^ 1), part, c);
        }
        if (!instance_barrier(I, bar, ++passed * nc + extra, limit_ns)) return;
    }
    // mixed precision: x = L^-T x^ for this CTA's nodes (the nodes it updated)
    if constexpr (MIXED) {
        for (uint32_t node = c * nt + tid; node < I.N; node += nc * nt) {
            double L[21], xh[6], x[6];
#pragma unroll
            for (int q = 0; q < 21; ++q) L[q] = I.chol[21 * (size_t)node + q];
#pragma unroll
            for (int q = 0; q < 6; ++q) xh[q] = I.x_d[6 * (size_t)node + q];
            chol_backward(L, xh, x);
#pragma unroll
            for (int q = 0; q < 6; ++q) I.x_d[6 * (size_t)node + q] = x[q];
        }
    }
}

// ------------------------------------------------------ matrix-free JtJ ---
// A pixel term's record for the matrix-free products: the one the term
// evaluation stored, or (recompute_jacobians) evaluated again from the maps
// and the current warp field, as ApplyJtJMatrixFreeIndexed.cu:222-348
// re-derives every term in every PCG iteration. The same function computes
// both, so the two forms use the same values. The kernels are instantiated
// for stored records only (RECOMP false: no registers for the
// re-derivation) and for the per-instance choice (RECOMP true), which the
// solver launches when the configuration asks for re-derived terms.
template <class T, bool RECOMP>
__device__ inline void pixel_record(const InstDesc& I, TermType ty, uint32_t k, uint32_t idx, float4& a, float4& b) {
    if (RECOMP && I.recompute_jr) {
        bool nonfinite = false;  // flagged by the term evaluation of this iteration
        if (ty == kDense) dense_record<T>(I, k, a, b, nonfinite);
        else fg_record<T>(I, k, a, b, nonfinite);
    } else {
        load_record32(I.term_jr + 2 * (size_t)idx, a, b);
    }
}

// a node's six direction components: the PCG direction d (fused) in pair
// loads (the solver's own 16-byte-aligned vector), or the float operand xin
template <class Acc>
__device__ inline void load_node6(int fused, const Acc* dv, const float* xin, uint32_t node, Acc (&x)[6]) {
    if (fused) {
        using P = typename std::conditional<sizeof(Acc) == 8, double2, float2>::type;
        const P* p2 = reinterpret_cast<const P*>(dv + 6 * (size_t)node);
        const P a = p2[0], b = p2[1], c = p2[2];
        x[0] = a.x; x[1] = a.y; x[2] = b.x; x[3] = b.y; x[4] = c.x; x[5] = c.y;
    } else {  // a caller's vector: no alignment beyond 4 bytes assumed
#pragma unroll
        for (int i = 0; i < 6; ++i) x[i] = (Acc)xin[6 * (size_t)node + i];
    }
}

// The stored-record kernels run 4 CTAs per SM (64 registers, a few spilled):
// measured faster than 3 (0.42 against 0.36 ms per PCG iteration on the
// 16-instance torso batch) and than 6 (0.37 ms); the re-deriving kernels run
// 2 CTAs per SM (up to 128 registers: the term evaluation's chain inline).
// J.p per term (ApplyJacobianDot.cu:127-198), stored channel-major:
// jp[c * T + t], T the solve's term count. A pixel term's rows for its nodes
// are one Jacobian row scaled by each node's skinning weight, so its J.p is
// that row times the weight-blended p (one record load per term). With
// `fused` set p is the PCG direction d of this iteration, else xin.
template <bool MIXED, bool RECOMP>
__global__ void __launch_bounds__(256, RECOMP ? 2 : 4) apply_j_kernel(const InstDesc* insts, const float* xin, int parity, int fused,
                                                      mvdr_penalty lam) {
    using Acc = typename std::conditional<MIXED, double, float>::type;
    const InstDesc& I = insts[blockIdx.y];
    if (bad_inputs(I) || (fused && pcg_stopped(I))) return;
    TermOffsets off;
    off.load(I.counts);
    const uint32_t T = off.o[4];
    const typename PcgVec<MIXED>::T* dv = PcgVec<MIXED>::d(I, parity);
    // mixed precision keeps J.p in double (jp holds 3 doubles per term)
    Acc* jp = reinterpret_cast<Acc*>(I.jp);
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < T; t += gridDim.x * blockDim.x) {
        uint32_t k;
        const TermType ty = off.typed(t, k);
        const ushort4 nn = term_nodes(I, ty, k);
        const unsigned short nodes[4] = {nn.x, nn.y, nn.z, nn.w};
        if (ty == kDense || ty == kForeground) {
            const uint32_t idx = ty == kDense ? k : off.o[0] + k;
            float4 ra, rb;
            pixel_record<Acc, RECOMP>(I, ty, k, idx, ra, rb);
            const float4 w4 = term_weights(I, ty, k);
            Acc pb[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const uint32_t node = nodes[q];
                if (node >= I.N) continue;
                const Acc w = (Acc)weight_of(nn, w4, node);
                Acc x6[6];
                load_node6<Acc>(fused, dv, xin, node, x6);
#pragma unroll
                for (int i = 0; i < 6; ++i) pb[i] += w * x6[i];
            }
            const Acc g[6] = {(Acc)ra.x, (Acc)ra.y, (Acc)ra.z, (Acc)ra.w, (Acc)rb.x, (Acc)rb.y};
            Acc o = 0;
#pragma unroll
            for (int i = 0; i < 6; ++i) o += g[i] * pb[i];
            jp[t] = o;
            if (ty == kDense && I.use_density && lam.density != 0.f) {
                // the density channel of the pixel (channel 1)
                float4 da, db;
                load_record32(I.density_jr + 2 * (size_t)k, da, db);
                const Acc gd[6] = {(Acc)da.x, (Acc)da.y, (Acc)da.z, (Acc)da.w, (Acc)db.x, (Acc)db.y};
                Acc od = 0;
#pragma unroll
                for (int i = 0; i < 6; ++i) od += gd[i] * pb[i];
                jp[(size_t)T + t] = od;  // a zero record (invalid term) gives 0
            }
            continue;
        }
        const int m = ty == kSmooth ? 2 : 4;
        Acc out[3] = {0, 0, 0};
        for (int q = 0; q < m; ++q) {
            const uint32_t node = nodes[q];
            if (node >= I.N) continue;
            TermRows tr;
            const int ch = term_rows(I, off, lam, t, node, tr);
            Acc p[6];
            load_node6<Acc>(fused, dv, xin, node, p);
            for (int c = 0; c < ch; ++c) {
                Acc a = 0;
#pragma unroll
                for (int i = 0; i < 6; ++i) a += (Acc)tr.J[c][i] * p[i];
                out[c] += (Acc)tr.w * a;
            }
        }
        jp[t] = out[0];
        jp[(size_t)T + t] = out[1];
        jp[2 * (size_t)T + t] = out[2];
    }
}

// Jt.y per node (ApplyJacobianTransposeDot.cu:29-155) plus the 1e-2 damping;
// warp per node, the lanes over its terms. A pixel term's row is its record
// scaled by the entry's recorded skinning weight. With `pcg` set the operand
// is this iteration's direction d; the kernel stores q and the d.q partial,
// like pcg_spmv_kernel.
template <bool MIXED, bool RECOMP>
__global__ void __launch_bounds__(256, RECOMP ? 2 : 4) apply_jt_kernel(const InstDesc* insts, const float* xin, float* yout, int pcg,
                                                       int parity, mvdr_penalty lam) {
    const InstDesc& I = insts[blockIdx.y];
    if (pcg && pcg_stopped(I)) return;
    using T = typename std::conditional<MIXED, double, float>::type;
    TermOffsets off;
    off.load(I.counts);
    const uint32_t Tn = off.o[4];
    using PV = PcgVec<MIXED>;
    const T* dcur = PV::d(I, parity);
    const T* jp = reinterpret_cast<const T*>(I.jp);
    const T l2_fg = (T)(lam.foreground * lam.foreground);
    const bool dens_on = I.use_density && lam.density != 0.f;
    const T l2_dens = (T)(lam.density * lam.density);
    T part = 0;
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    for (uint32_t node = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); node < I.N; node += warps) {
        T acc[6] = {0, 0, 0, 0, 0, 0};
        const uint32_t b = I.n2t_offset[node], e = I.n2t_offset[node + 1];
        for (uint32_t p = b + lane_id(); p < e; p += 32) {
            const uint32_t t = I.n2t_index[p];
            uint32_t k;
            const TermType ty = off.typed(t, k);
            if (ty == kDense || ty == kForeground) {
                const uint32_t idx = ty == kDense ? k : off.o[0] + k;
                float4 ra, rb;
                pixel_record<T, RECOMP>(I, ty, k, idx, ra, rb);
                const T wn = (T)I.n2t_w[p];
                const T sc = (ty == kDense ? (T)1 : l2_fg) * wn;
                const T y = jp[t];
                const float g[6] = {ra.x, ra.y, ra.z, ra.w, rb.x, rb.y};
#pragma unroll
                for (int i = 0; i < 6; ++i) acc[i] += sc * (T)g[i] * y;
                if (ty == kDense && dens_on) {
                    float4 da, db;
                    load_record32(I.density_jr + 2 * (size_t)k, da, db);
                    const T sd = l2_dens * wn, yd = jp[(size_t)Tn + t];
                    const float gd[6] = {da.x, da.y, da.z, da.w, db.x, db.y};
#pragma unroll
                    for (int i = 0; i < 6; ++i) acc[i] += sd * (T)gd[i] * yd;
                }
                continue;
            }
            TermRows tr;
            const int ch = term_rows(I, off, lam, t, node, tr);
            const T sc = (T)tr.lam2 * (T)tr.w;
            for (int c = 0; c < ch; ++c) {
                const T y = jp[(size_t)c * Tn + t];
#pragma unroll
                for (int i = 0; i < 6; ++i) acc[i] += sc * (T)tr.J[c][i] * y;
            }
        }
        // fixed-order reduce-scatter of the 6 sums (padded to 8): three
        // halving exchanges leave value q with lanes 4q .. 4q + 3, two
        // butterfly steps finish it
        const uint32_t lane = lane_id();
        T v[8] = {acc[0], acc[1], acc[2], acc[3], acc[4], acc[5], (T)0, (T)0};
#pragma unroll
        for (int dist = 16, n = 4; dist >= 4; dist >>= 1, n >>= 1) {
            const bool upper = (lane & (uint32_t)dist) != 0;
#pragma unroll
            for (int i = 0; i < n; ++i) {
                const T keep = upper ? v[i + n] : v[i];
                const T send = upper ? v[i] : v[i + n];
                v[i] = keep + __shfl_xor_sync(0xffffffffu, send, dist);
            }
        }
        v[0] += __shfl_xor_sync(0xffffffffu, v[0], 2);
        v[0] += __shfl_xor_sync(0xffffffffu, v[0], 1);
        const uint32_t qi = lane >> 2;
        if ((lane & 3u) == 0 && qi < 6) {
            const size_t el = 6 * (size_t)node + qi;
            const T dv = pcg ? dcur[el] : (T)xin[el];
            const T qv = v[0] + (T)1e-2f * dv;
            if (pcg) {
                PV::q(I)[el] = qv;
                part += dv * qv;
            } else {
                yout[el] = (float)qv;
            }
        }
    }
    if (pcg) store_block_partial<T>(I, kRegDq, part);
}

// y = A x with the materialised operator (no PCG side effects)
template <bool MIXED>
__global__ void __launch_bounds__(192) bsr_apply_kernel(const InstDesc* insts, const float* xin, float* yout) {
    const InstDesc& I = insts[blockIdx.y];
    const uint32_t rows_per_cta = blockDim.x / 6;
    for (uint32_t base = blockIdx.x * rows_per_cta; base < I.N; base += gridDim.x * rows_per_cta) {
        const uint32_t br = base + threadIdx.x / 6;
        const uint32_t r = threadIdx.x % 6;
        if (threadIdx.x >= rows_per_cta * 6 || br >= I.N) continue;
        yout[6 * (size_t)br + r] = index_complete(I) ? bsr_row<MIXED>(I, br, r, xin) : 0.f;
    }
}

// ----------------------------------------------------------- update -------
// applyWarpFieldUpdateKernel (SolverIterationData.cu:9-57)
template <bool MIXED>
__global__ void __launch_bounds__(128) update_kernel(const InstDesc* insts) {
    const InstDesc& I = insts[blockIdx.y];
    for (uint32_t node = blockIdx.x * blockDim.x + threadIdx.x; node < I.N; node += gridDim.x * blockDim.x) {
        float tw[6];
#pragma unroll
        for (int i = 0; i < 6; ++i) tw[i] = (float)PcgVec<MIXED>::x(I)[6 * (size_t)node + i];
        M34 se3;
        const float3 w = mk3(tw[0], tw[1], tw[2]);
        if (fabsf(w.x) + fabsf(w.y) + fabsf(w.z) < 1e-4f) {
#pragma unroll
            for (int i = 0; i < 9; ++i) se3.r[i] = (i % 4 == 0) ? 1.f : 0.f;
        } else {
            const float angle = sqrtf(dot3(w, w));
            const float3 ax = mul3(1.0f / angle, w);
            const float c = cosf(angle), s = sinf(angle), t = 1.0f - c;
            se3.r[0] = t * ax.x * ax.x + c;
            se3.r[1] = t * ax.x * ax.y - ax.z * s;
            se3.r[2] = t * ax.x * ax.z + ax.y * s;
            se3.r[3] = t * ax.x * ax.y + ax.z * s;
            se3.r[4] = t * ax.y * ax.y + c;
            se3.r[5] = t * ax.y * ax.z - ax.x * s;
            se3.r[6] = t * ax.x * ax.z - ax.y * s;
            se3.r[7] = t * ax.y * ax.z + ax.x * s;
            se3.r[8] = t * ax.z * ax.z + c;
        }
        se3.t[0] = tw[3]; se3.t[1] = tw[4]; se3.t[2] = tw[5];
        // two 128-bit read-only loads: this kernel's loads of the field are
        // coalesced (node per thread), the 256-bit form only helps gathers
        DQ cur;
        cur.q0 = __ldg(reinterpret_cast<const float4*>(I.se3 + node));
        cur.q1 = __ldg(reinterpret_cast<const float4*>(I.se3 + node) + 1);
        const M34 p = dq_to_mat34(cur);
        M34 n;
#pragma unroll
        for (int r = 0; r < 3; ++r) {
#pragma unroll
            for (int c = 0; c < 3; ++c)
                n.r[3 * r + c] = se3.r[3 * r] * p.r[c] + se3.r[3 * r + 1] * p.r[3 + c] + se3.r[3 * r + 2] * p.r[6 + c];
            n.t[r] = se3.r[3 * r] * p.t[0] + se3.r[3 * r + 1] * p.t[1] + se3.r[3 * r + 2] * p.t[2] + se3.t[r];
        }
        // DualQuaternion(mat34) (DualQuaternion.h:123-130) via Quaternion(mat33) (Quaternion.h:46-77)
        const float* m = n.r;
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
        const float4 tq = make_float4(0.5f * n.t[0], 0.5f * n.t[1], 0.5f * n.t[2], 0.f);
        float4 q1;  // tq * q
        q1.w = tq.w * q.w - tq.x * q.x - tq.y * q.y - tq.z * q.z;
        q1.x = tq.w * q.x + tq.x * q.w + tq.y * q.z - tq.z * q.y;
        q1.y = tq.w * q.y - tq.x * q.z + tq.y * q.w + tq.z * q.x;
        q1.z = tq.w * q.z + tq.x * q.y - tq.y * q.x + tq.z * q.w;
        if (!isfinite(q.x) || !isfinite(q.y) || !isfinite(q.z) || !isfinite(q.w) || !isfinite(q1.x) ||
            !isfinite(q1.y) || !isfinite(q1.z) || !isfinite(q1.w))
            set_error(I, kErrNonFinite);
        float4* out = reinterpret_cast<float4*>(I.se3 + node);
        out[0] = q;
        out[1] = q1;
    }
}

// ------------------------------------------------------------- energy -----
// computeTermResidualKernel (ResidualEvaluator.cu:71-142): sum (lambda r)^2
// The energy of the linearisation point: the term evaluation's `count`
// per-CTA partials summed in a fixed order (one CTA per instance)
__global__ void __launch_bounds__(256) energy_sum_kernel(const InstDesc* insts, uint32_t count, uint32_t slot,
                                                         uint32_t density_count) {
    const InstDesc& I = insts[blockIdx.y];
    __shared__ double ws[8];
    double e = 0;
    for (uint32_t c = threadIdx.x; c < count; c += blockDim.x) e += I.partials[c];
    for (uint32_t c = threadIdx.x; c < density_count; c += blockDim.x)
        e += I.partials[(size_t)kRegDensityEnergy * I.part_stride + c];
    e = warp_sum(e);
    if (lane_id() == 0) ws[threadIdx.x >> 5] = e;
    __syncthreads();
    if (threadIdx.x == 0) {
        double tot = 0;
        for (uint32_t w = 0; w < (blockDim.x >> 5); ++w) tot += ws[w];
        I.energy[slot] = tot;
    }
}

// --------------------------------------------------------- exports -------
// symmetric-key order, reference layout blk[6k + r] = A(r, k)
__global__ void export_offdiag_kernel(const InstDesc* insts, uint32_t inst, float* out) {
    const InstDesc& I = insts[inst];
    const uint32_t P2 = 2 * I.counts->half_pairs;
    const uint32_t mask = I.enc - 1;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < 36 * P2; i += gridDim.x * blockDim.x) {
        const uint32_t s = i / 36, e = i % 36;
        const uint32_t row = I.sym_key[s] / I.enc;
        (void)mask;
        out[i] = stored_block_element(I, s + row + 1, e % 6, e / 6);
    }
}

__global__ void export_preconditioner_kernel(const InstDesc* insts, uint32_t inst, float* out, int mixed) {
    const InstDesc& I = insts[inst];
    for (uint32_t node = blockIdx.x * blockDim.x + threadIdx.x; node < I.N; node += gridDim.x * blockDim.x) {
        if (!mixed) {
            for (int i = 0; i < 36; ++i) out[36 * (size_t)node + i] = I.minv[36 * (size_t)node + i];
            continue;
        }
        for (int c = 0; c < 6; ++c) {
            double e[6] = {0, 0, 0, 0, 0, 0}, x[6];
            e[c] = 1.0;
            cholesky6_solve(I.chol + 21 * (size_t)node, e, x);
            for (int r = 0; r < 6; ++r) out[36 * (size_t)node + 6 * r + c] = (float)x[r];
        }
    }
}

// ------------------------------------------------------------- launch -----

static inline dim3 grid2(uint32_t x, uint32_t B) { return dim3(x ? x : 1, B); }

static uint32_t eval_terms_grid(const LaunchCfg& lc) {
    return min((lc.cap_terms + 255) / 256, (uint32_t)lc.sm_count * 8);
}

// CTAs per instance of the density kernel
static uint32_t eval_density_grid(const LaunchCfg& lc) {
    return min((lc.cap_dense + 255) / 256, (uint32_t)lc.sm_count * 8);
}

cudaError_t launch_eval_terms(const LaunchCfg& lc, InstDesc* d, const mvdr_penalty& lam, cudaStream_t st) {
    const uint32_t g = eval_terms_grid(lc);
    if (lc.precision == MVDR_PRECISION_MIXED) MVDR_LAUNCH(eval_terms_kernel<double>, grid2(g, lc.B), 256, 0, st, d, lam);
    else MVDR_LAUNCH(eval_terms_kernel<float>, grid2(g, lc.B), 256, 0, st, d, lam);
    if (lc.use_density) {
        const uint32_t gd = eval_density_grid(lc);
        if (lc.precision == MVDR_PRECISION_MIXED) MVDR_LAUNCH(eval_density_kernel<double>, grid2(gd, lc.B), 256, 0, st, d, lam);
        else MVDR_LAUNCH(eval_density_kernel<float>, grid2(gd, lc.B), 256, 0, st, d, lam);
    }
    return cudaGetLastError();
}

// CTAs per instance of the operator scaling (16 pairs per CTA)
static uint32_t scale_grid(const LaunchCfg& lc) {
    return min((lc.cap_pairs + kScalePairsPerCta - 1) / kScalePairsPerCta, (uint32_t)lc.sm_count * 16);
}

// J.d then Jt.(J.d) (+ damping): `fused` takes the PCG direction of `parity`
// as the operand and stores q with its d.q partials, else x -> y
static void launch_apply_pair(const LaunchCfg& lc, InstDesc* d, const float* x, float* y, int parity, int fused,
                              uint32_t gterm, uint32_t gwarp, uint32_t B, const mvdr_penalty& lam, cudaStream_t st) {
    const bool mixed = lc.precision == MVDR_PRECISION_MIXED;
    if (mixed && lc.recompute_jr) {
        MVDR_LAUNCH((apply_j_kernel<true, true>), grid2(gterm, B), 256, 0, st, d, x, parity, fused, lam);
        MVDR_LAUNCH((apply_jt_kernel<true, true>), grid2(gwarp, B), 256, 0, st, d, x, y, fused, parity, lam);
    } else if (mixed) {
        MVDR_LAUNCH((apply_j_kernel<true, false>), grid2(gterm, B), 256, 0, st, d, x, parity, fused, lam);
        MVDR_LAUNCH((apply_jt_kernel<true, false>), grid2(gwarp, B), 256, 0, st, d, x, y, fused, parity, lam);
    } else if (lc.recompute_jr) {
        MVDR_LAUNCH((apply_j_kernel<false, true>), grid2(gterm, B), 256, 0, st, d, x, parity, fused, lam);
        MVDR_LAUNCH((apply_jt_kernel<false, true>), grid2(gwarp, B), 256, 0, st, d, x, y, fused, parity, lam);
    } else {
        MVDR_LAUNCH((apply_j_kernel<false, false>), grid2(gterm, B), 256, 0, st, d, x, parity, fused, lam);
        MVDR_LAUNCH((apply_jt_kernel<false, false>), grid2(gwarp, B), 256, 0, st, d, x, y, fused, parity, lam);
    }
}

cudaError_t launch_assemble(const LaunchCfg& lc, InstDesc* d, const mvdr_penalty& lam, bool materialize,
                            cudaStream_t st) {
    const uint32_t gn = (lc.max_nodes + kDiagNodes - 1) / kDiagNodes;
    if (lc.precision == MVDR_PRECISION_MIXED) MVDR_LAUNCH(diag_rhs_kernel<true>, grid2(gn, lc.B), 128, 0, st, d, lam);
    else MVDR_LAUNCH(diag_rhs_kernel<false>, grid2(gn, lc.B), 128, 0, st, d, lam);
    if (materialize) {
        const uint32_t gp = min((lc.cap_pairs + 127) / 128, (uint32_t)lc.sm_count * 8);
        if (lc.precision == MVDR_PRECISION_MIXED) {
            MVDR_LAUNCH(offdiag_kernel<true>, grid2(gp, lc.B), 128, 0, st, d, lam);
            MVDR_LAUNCH(scale_offdiag_kernel, grid2(scale_grid(lc), lc.B), 128, 0, st, d);
        } else {
            MVDR_LAUNCH(offdiag_kernel<false>, grid2(gp, lc.B), 128, 0, st, d, lam);
        }
    }
    return cudaGetLastError();
}

// diag_rhs_kernel and offdiag_kernel read the same term records and write
// disjoint outputs (the diagonal blocks, factors and Jt r; the upper blocks),
// so they run side by side; the scaling reads both.
cudaError_t launch_assemble_forked(const LaunchCfg& lc, InstDesc* d, const mvdr_penalty& lam, cudaStream_t st,
                                   cudaStream_t side, cudaEvent_t fork, cudaEvent_t join) {
    const bool mixed = lc.precision == MVDR_PRECISION_MIXED;
    cudaError_t e = cudaEventRecord(fork, st);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(side, fork, 0);
    if (e != cudaSuccess) return e;
    const uint32_t gp = min((lc.cap_pairs + 127) / 128, (uint32_t)lc.sm_count * 8);
    if (mixed) MVDR_LAUNCH(offdiag_kernel<true>, grid2(gp, lc.B), 128, 0, side, d, lam);
    else MVDR_LAUNCH(offdiag_kernel<false>, grid2(gp, lc.B), 128, 0, side, d, lam);
    e = cudaEventRecord(join, side);
    const uint32_t gn = (lc.max_nodes + kDiagNodes - 1) / kDiagNodes;
    if (mixed) MVDR_LAUNCH(diag_rhs_kernel<true>, grid2(gn, lc.B), 128, 0, st, d, lam);
    else MVDR_LAUNCH(diag_rhs_kernel<false>, grid2(gn, lc.B), 128, 0, st, d, lam);
    // the join is made even after a failed record, so that a capture ends
    const cudaError_t w = cudaStreamWaitEvent(st, join, 0);
    if (e == cudaSuccess) e = w;
    if (e != cudaSuccess) return e;
    if (mixed) MVDR_LAUNCH(scale_offdiag_kernel, grid2(scale_grid(lc), lc.B), 128, 0, st, d);
    return cudaGetLastError();
}

cudaError_t launch_energy(const LaunchCfg& lc, InstDesc* d, uint32_t slot, cudaStream_t st) {
    MVDR_LAUNCH(energy_sum_kernel, grid2(1, lc.B), 256, 0, st, d, eval_terms_grid(lc), slot,
                lc.use_density ? eval_density_grid(lc) : 0u);
    return cudaGetLastError();
}

// PCG init and update: a thread per node in CTAs of 64, so that the small
// grid spreads over every SM
constexpr uint32_t kPcgNodeThreads = 64;

// CTAs per instance of the SpMV launch with the current shape
static uint32_t spmv_grid(const LaunchCfg& lc) {
    const uint32_t R = kSpmvShapes[lc.spmv_shape].rows;
    return (lc.max_nodes + R - 1) / R;
}

uint32_t persistent_pcg_grid(int mixed, int sm_count) {
    int nb = 0;
    const cudaError_t e =
        mixed ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, pcg_persistent_kernel<true>, kPersistThreads, 0)
              : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, pcg_persistent_kernel<false>, kPersistThreads, 0);
    return e == cudaSuccess && nb > 0 ? (uint32_t)nb * (uint32_t)sm_count : 0u;
}

// one cooperative launch: every CTA is resident, so the instance barriers
// cannot wait on a CTA that has not started
static cudaError_t launch_pcg_persistent(const LaunchCfg& lc, InstDesc* d, uint32_t iters, cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(lc.pcg_bars, 0, sizeof(uint32_t) * 32 * lc.B, st);
    if (e != cudaSuccess) return e;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(lc.pcg_grid);
    cfg.blockDim = dim3(kPersistThreads);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    const uint32_t B = lc.B;
    e = lc.precision == MVDR_PRECISION_MIXED
            ? cudaLaunchKernelEx(&cfg, pcg_persistent_kernel<true>, (const InstDesc*)d, B, iters, lc.wait_limit_ns,
                                 lc.wait_extra_arrivals)
            : cudaLaunchKernelEx(&cfg, pcg_persistent_kernel<false>, (const InstDesc*)d, B, iters, lc.wait_limit_ns,
                                 lc.wait_extra_arrivals);
    count_launch();
    return e;
}

cudaError_t launch_pcg(const LaunchCfg& lc, InstDesc* d, const mvdr_penalty& lam, uint32_t iters, uint32_t gn,
                       cudaStream_t st) {
    // the convergence check runs in the launched form only
    if (lc.pcg_persistent && lc.mode == MVDR_MODE_MATERIALIZED && lc.pcg_tol == 0.f)
        return launch_pcg_persistent(lc, d, iters, st);
    const bool mixed = lc.precision == MVDR_PRECISION_MIXED;
    // the update's and direction's grids cover every node / element
    const uint32_t gnode = (lc.max_nodes + kPcgNodeThreads - 1) / kPcgNodeThreads;
    const uint32_t gvec = (6 * lc.max_nodes + 255) / 256;
    const uint32_t gwarp = (lc.max_nodes + 7) / 8;
    const uint32_t gterm = min((lc.cap_terms + 255) / 256, (uint32_t)lc.sm_count * 8);
    // mixed precision, materialised: PCG on the scaled operator (scale_offdiag_kernel)
    const bool scaled = mixed && lc.mode == MVDR_MODE_MATERIALIZED;
    if (scaled) MVDR_LAUNCH((pcg_init_kernel<true, true>), grid2(gnode, lc.B), kPcgNodeThreads, 0, st, d);
    else if (mixed) MVDR_LAUNCH((pcg_init_kernel<true, false>), grid2(gnode, lc.B), kPcgNodeThreads, 0, st, d);
    else MVDR_LAUNCH((pcg_init_kernel<false, false>), grid2(gnode, lc.B), kPcgNodeThreads, 0, st, d);
    for (uint32_t it = 0; it < iters; ++it) {
        const int parity = (int)(it & 1u), first = it == 0;
        uint32_t nq;  // CTAs that store the d.q partials
        // d = s + beta d_prev, then q = A d with its d.q partials. The scaled
        // form's update forms each next direction (pcg_update_kernel FUSE),
        // so its direction kernel runs for the first iteration only.
        if (scaled) {
            if (first)
                MVDR_LAUNCH((pcg_direction_kernel<true, true>), grid2(gvec, lc.B), 256, 0, st, d, parity, first, gnode, gn, it);
        } else if (mixed) {
            MVDR_LAUNCH((pcg_direction_kernel<true, false>), grid2(gvec, lc.B), 256, 0, st, d, parity, first, gnode, gn, it);
        } else {
            MVDR_LAUNCH((pcg_direction_kernel<false, false>), grid2(gvec, lc.B), 256, 0, st, d, parity, first, gnode, gn, it);
        }
        if (lc.mode == MVDR_MODE_MATRIX_FREE) {
            // J.d per term, then Jt per node (+ damping, q, d.q)
            launch_apply_pair(lc, d, nullptr, nullptr, parity, 1, gterm, gwarp, lc.B, lam, st);
            nq = gwarp;
        } else {
            const cudaError_t e = launch_spmv(lc, d, parity, st);
            if (e != cudaSuccess) return e;
            nq = spmv_grid(lc);
        }
        if (scaled) MVDR_LAUNCH((pcg_update_kernel<true, true, true>), grid2(gnode, lc.B), kPcgNodeThreads, 0, st, d, parity, gnode, nq, gn, it);
        else if (mixed) MVDR_LAUNCH((pcg_update_kernel<true, false, false>), grid2(gnode, lc.B), kPcgNodeThreads, 0, st, d, parity, gnode, nq, gn, it);
        else MVDR_LAUNCH((pcg_update_kernel<false, false, false>), grid2(gnode, lc.B), kPcgNodeThreads, 0, st, d, parity, gnode, nq, gn, it);
    }
    if (scaled) MVDR_LAUNCH(pcg_unscale_kernel, grid2((lc.max_nodes + 127) / 128, lc.B), 128, 0, st, d);
    return cudaGetLastError();
}

template <bool MIXED, uint32_t R, uint32_t S>
static void spmv_shape_launch(const LaunchCfg& lc, InstDesc* d, int parity, cudaStream_t st) {
    auto* kernel = &pcg_spmv_kernel<MIXED, R, S>;
    MVDR_LAUNCH(kernel, grid2((lc.max_nodes + R - 1) / R, lc.B), 6 * S * R, 0, st, d, parity);
}

template <bool MIXED, uint32_t R, uint32_t S>
static void spmv_col_launch(const LaunchCfg& lc, InstDesc* d, int parity, cudaStream_t st) {
    auto* kernel = &pcg_spmv_col_kernel<MIXED, R, S>;
    MVDR_LAUNCH(kernel, grid2((lc.max_nodes + R - 1) / R, lc.B), 6 * S * R, 0, st, d, parity);
}

template <bool MIXED>
static void spmv_dispatch(const LaunchCfg& lc, InstDesc* d, int parity, cudaStream_t st) {
    switch (lc.spmv_shape) {
        case 1: spmv_shape_launch<MIXED, 8, 2>(lc, d, parity, st); break;
        case 2: spmv_shape_launch<MIXED, 16, 1>(lc, d, parity, st); break;
        case 3: spmv_shape_launch<MIXED, 32, 1>(lc, d, parity, st); break;
        case 4: spmv_shape_launch<MIXED, 16, 3>(lc, d, parity, st); break;
        case 5: spmv_shape_launch<MIXED, 8, 4>(lc, d, parity, st); break;
        case 6: spmv_shape_launch<MIXED, 32, 2>(lc, d, parity, st); break;
        case 7: spmv_col_launch<MIXED, 16, 1>(lc, d, parity, st); break;
        case 8: spmv_col_launch<MIXED, 32, 1>(lc, d, parity, st); break;
        case 9: spmv_col_launch<MIXED, 8, 2>(lc, d, parity, st); break;
        case 10: spmv_col_launch<MIXED, 16, 2>(lc, d, parity, st); break;
        case 11: spmv_col_launch<MIXED, 4, 4>(lc, d, parity, st); break;
        default: spmv_shape_launch<MIXED, 16, 2>(lc, d, parity, st); break;
    }
}

template <uint32_t R, uint32_t S, uint32_t F>
static void spmv_scaled_launch(const LaunchCfg& lc, InstDesc* d, int parity, cudaStream_t st) {
    auto* kernel = &pcg_spmv_scaled_kernel<R, S, F>;
    MVDR_LAUNCH(kernel, grid2((lc.max_nodes + R - 1) / R, lc.B), 6 * S * R, 0, st, d, parity);
}

// the shapes of kSpmvShapes for the scaled operator
static void spmv_scaled_dispatch(const LaunchCfg& lc, InstDesc* d, int parity, cudaStream_t st) {
    switch (lc.spmv_shape) {
        case 1: spmv_scaled_launch<8, 2, 0>(lc, d, parity, st); break;
        case 2: spmv_scaled_launch<16, 1, 0>(lc, d, parity, st); break;
        case 3: spmv_scaled_launch<32, 1, 0>(lc, d, parity, st); break;
        case 4: spmv_scaled_launch<16, 3, 0>(lc, d, parity, st); break;
        case 5: spmv_scaled_launch<8, 4, 0>(lc, d, parity, st); break;
        case 6: spmv_scaled_launch<32, 2, 0>(lc, d, parity, st); break;
        case 7: spmv_scaled_launch<16, 1, 1>(lc, d, parity, st); break;
        case 8: spmv_scaled_launch<32, 1, 1>(lc, d, parity, st); break;
        case 9: spmv_scaled_launch<8, 2, 1>(lc, d, parity, st); break;
        case 10: spmv_scaled_launch<16, 2, 1>(lc, d, parity, st); break;
        case 11: spmv_scaled_launch<4, 4, 1>(lc, d, parity, st); break;
        default: spmv_scaled_launch<16, 2, 0>(lc, d, parity, st); break;
    }
}

cudaError_t launch_spmv(const LaunchCfg& lc, InstDesc* d, int parity, cudaStream_t st) {
    if (lc.precision == MVDR_PRECISION_MIXED) spmv_scaled_dispatch(lc, d, parity, st);
    else spmv_dispatch<false>(lc, d, parity, st);
    return cudaGetLastError();
}

cudaError_t launch_stage(const LaunchCfg& lc, InstDesc* d, const mvdr_penalty& lam, int stage, cudaStream_t st) {
    const bool mixed = lc.precision == MVDR_PRECISION_MIXED;
    const bool scaled = mixed && lc.mode == MVDR_MODE_MATERIALIZED;
    const uint32_t gnode = (lc.max_nodes + kPcgNodeThreads - 1) / kPcgNodeThreads;
    const uint32_t gvec = (6 * lc.max_nodes + 255) / 256;
    const uint32_t gn = (lc.max_nodes + kDiagNodes - 1) / kDiagNodes;
    switch (stage) {
        case MVDR_STAGE_TERMS: return launch_eval_terms(lc, d, lam, st);
        case MVDR_STAGE_DIAG:
            if (mixed) MVDR_LAUNCH(diag_rhs_kernel<true>, grid2(gn, lc.B), 128, 0, st, d, lam);
            else MVDR_LAUNCH(diag_rhs_kernel<false>, grid2(gn, lc.B), 128, 0, st, d, lam);
            break;
        case MVDR_STAGE_OFFDIAG: {
            const uint32_t gp = min((lc.cap_pairs + 127) / 128, (uint32_t)lc.sm_count * 8);
            if (mixed) MVDR_LAUNCH(offdiag_kernel<true>, grid2(gp, lc.B), 128, 0, st, d, lam);
            else MVDR_LAUNCH(offdiag_kernel<false>, grid2(gp, lc.B), 128, 0, st, d, lam);
            break;
        }
        case MVDR_STAGE_SPMV:
            return launch_spmv(lc, d, 0, st);
        case MVDR_STAGE_DIRECTION:
            // (no residual history, no convergence test: an iteration past the first)
            if (scaled) MVDR_LAUNCH((pcg_direction_kernel<true, true>), grid2(gvec, lc.B), 256, 0, st, d, 0, 0, gnode, ~0u, 1u);
            else if (mixed) MVDR_LAUNCH((pcg_direction_kernel<true, false>), grid2(gvec, lc.B), 256, 0, st, d, 0, 0, gnode, ~0u, 1u);
            else MVDR_LAUNCH((pcg_direction_kernel<false, false>), grid2(gvec, lc.B), 256, 0, st, d, 0, 0, gnode, ~0u, 1u);
            break;
        case MVDR_STAGE_PCG_UPDATE:
            // (the form the solve runs; no residual history)
            if (scaled) MVDR_LAUNCH((pcg_update_kernel<true, true, true>), grid2(gnode, lc.B), kPcgNodeThreads, 0, st, d, 0, gnode, spmv_grid(lc), ~0u, 1u);
            else if (mixed) MVDR_LAUNCH((pcg_update_kernel<true, false, false>), grid2(gnode, lc.B), kPcgNodeThreads, 0, st, d, 0, gnode, spmv_grid(lc), ~0u, 1u);
            else MVDR_LAUNCH((pcg_update_kernel<false, false, false>), grid2(gnode, lc.B), kPcgNodeThreads, 0, st, d, 0, gnode, spmv_grid(lc), ~0u, 1u);
            break;
        case MVDR_STAGE_SCALE:
            if (!scaled) return cudaErrorInvalidValue;
            MVDR_LAUNCH(scale_offdiag_kernel, grid2(scale_grid(lc), lc.B), 128, 0, st, d);
            break;
        case MVDR_STAGE_UPDATE: return launch_update(lc, d, st);
        case MVDR_STAGE_MATRIX_FREE: {
            // the launches of one matrix-free PCG iteration after its direction
            const uint32_t gwarp = (lc.max_nodes + 7) / 8;
            const uint32_t gterm = min((lc.cap_terms + 255) / 256, (uint32_t)lc.sm_count * 8);
            launch_apply_pair(lc, d, nullptr, nullptr, 0, 1, gterm, gwarp, lc.B, lam, st);
            break;
        }
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_update(const LaunchCfg& lc, InstDesc* d, cudaStream_t st) {
    const uint32_t g = (lc.max_nodes + 127) / 128;
    if (lc.precision == MVDR_PRECISION_MIXED) MVDR_LAUNCH(update_kernel<true>, grid2(g, lc.B), 128, 0, st, d);
    else MVDR_LAUNCH(update_kernel<false>, grid2(g, lc.B), 128, 0, st, d);
    return cudaGetLastError();
}

cudaError_t launch_apply_jtj(const LaunchCfg& lc, InstDesc* d, const mvdr_penalty& lam, const float* x, float* y,
                             cudaStream_t st) {
    // single instance view: d points at the instance's descriptor, B = 1
    if (lc.mode == MVDR_MODE_MATRIX_FREE) {
        const uint32_t gterm = min((lc.cap_terms + 255) / 256, (uint32_t)lc.sm_count * 8);
        launch_apply_pair(lc, d, x, y, 0, 0, gterm, (lc.max_nodes + 7) / 8, 1, lam, st);
    } else {
        if (lc.precision == MVDR_PRECISION_MIXED)
            MVDR_LAUNCH(bsr_apply_kernel<true>, grid2((lc.max_nodes + 31) / 32, 1), 192, 0, st, d, x, y);
        else
            MVDR_LAUNCH(bsr_apply_kernel<false>, grid2((lc.max_nodes + 31) / 32, 1), 192, 0, st, d, x, y);
    }
    return cudaGetLastError();
}

cudaError_t launch_export_offdiag(const LaunchCfg& lc, InstDesc* d, uint32_t inst, float* out, cudaStream_t st) {
    MVDR_LAUNCH(export_offdiag_kernel, dim3(lc.sm_count * 4), 256, 0, st, d, inst, out);
    return cudaGetLastError();
}

cudaError_t launch_export_preconditioner(const LaunchCfg& lc, InstDesc* d, uint32_t inst, float* out,
                                         cudaStream_t st) {
    MVDR_LAUNCH(export_preconditioner_kernel, dim3((lc.max_nodes + 127) / 128), 128, 0, st, d, inst, out,
                lc.precision == MVDR_PRECISION_MIXED ? 1 : 0);
    return cudaGetLastError();
}

}  // namespace mvdr
