// Reference-pinning harness - TEST INFRASTRUCTURE.
//
// Compiles the reference's own header-only solver math (from the reference
// tree, with the stand-in headers of oracle/ref_shim for its Eigen, PCL and
// TensorRT includes) into oracle/_ref/libref_pin.so, so that the tests can
// check the oracle's restatement against the reference's code on the same
// inputs. The recipe is oracle/Makefile (target `ref`); nothing here is
// copied from the reference: every function below only calls it.
//
//   ref_blend_se3           averageDualQuaternion + DualQuaternion::se3_matrix
//                           (math/DualQuaternion/DualQuaternion.h:326-332,381-393)
//   ref_dq_to_mat34         DualQuaternion::operator mat34 (DualQuaternion.h:309-319)
//   ref_mat34_to_dq         DualQuaternion(const mat34&) (DualQuaternion.h:123-130)
//   ref_gauss_jordan6       DenseGaussian<6>::Inverse (core/NonRigidSolver/DenseGaussian.h:55-125)
//   ref_huber               compute_feature_huber_weight (huber_weight.h:25-27)
//   ref_p2p_jacobian        computePointToPointICPTermJacobian (geometry_icp_jacobian.cuh:91-120)
//   ref_p2p_jt_residual     computePoint2PointJtResidual (geometry_icp_jacobian.cuh:148-178)
//   ref_smooth_jacobian     computeSmoothTermJacobian, one node (geometry_icp_jacobian.cuh:359-382)
//   ref_smooth_jt_residual  computeSmoothTermJtResidual (geometry_icp_jacobian.cuh:399-437)
//   ref_encode_nodepair     encode_nodepair (base/EncodeUtils.h:187-192)
//   ref_term_offsets        size2offset + query_typed_index (base/term_offset_types.h:44-99)
//   ref_image_terms         computeImageDensityJacobainAndResidual
//                           (density_map_jacobian.cuh:12-79), run in a kernel
//                           on texture objects (needs a GPU)
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <vector>

#include <base/EncodeUtils.h>
#include <base/term_offset_types.h>
#include <core/NonRigidSolver/DenseGaussian.h>
#include <core/NonRigidSolver/density_map_jacobian.cuh>
#include <core/NonRigidSolver/geometry_icp_jacobian.cuh>
#include <core/NonRigidSolver/huber_weight.h>
#include <math/DualQuaternion/DualQuaternion.h>

using namespace SparseSurfelFusion;

namespace {

static_assert(sizeof(DualQuaternion) == 32, "DualQuaternion is two float4");
static_assert(sizeof(mat34) == 48, "mat34 is three float3 columns and a float3");

DualQuaternion load_dq(const float* p) {
    DualQuaternion d;
    std::memcpy(&d, p, 32);
    return d;
}
void store_mat34(const mat34& m, float* out) { std::memcpy(out, &m, 48); }
void store_gradient(const TwistGradientOfScalarCost& g, float* out) {
    out[0] = g.rotation.x; out[1] = g.rotation.y; out[2] = g.rotation.z;
    out[3] = g.translation.x; out[4] = g.translation.y; out[5] = g.translation.z;
}

// one image term per thread: the reference's function on this thread's inputs
__global__ void image_terms_kernel(uint32_t count, const float4* ref_vertex, const uint16_t* camera,
                                   const ushort4* knn, const float4* weight, const float* geometry,
                                   const DualQuaternion* field, const cudaTextureObject_t* image,
                                   const cudaTextureObject_t* gradient, const Intrinsic* intrinsic,
                                   const mat34* world2camera, const mat34* initial, unsigned width, unsigned height,
                                   float* out) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
    const unsigned short v = camera[k];
    TwistGradientOfScalarCost g;
    float r = 0.f;
    device::computeImageDensityJacobainAndResidual(initial[v], v, image[v], gradient[v], width, height,
                                                   ref_vertex[k], geometry[k], knn[k], weight[k], field,
                                                   intrinsic[v], world2camera[v], g, r);
    float* o = out + 7 * (size_t)k;
    o[0] = g.rotation.x; o[1] = g.rotation.y; o[2] = g.rotation.z;
    o[3] = g.translation.x; o[4] = g.translation.y; o[5] = g.translation.z;
    o[6] = r;
}

template <class T> T* to_device(const T* host, size_t n, std::vector<void*>& keep) {
    void* p = nullptr;
    if (cudaMalloc(&p, n * sizeof(T) + 16) != cudaSuccess) return nullptr;
    cudaMemcpy(p, host, n * sizeof(T), cudaMemcpyHostToDevice);
    keep.push_back(p);
    return static_cast<T*>(p);
}

}  // namespace

extern "C" {

void ref_blend_se3(const float* field, const uint16_t* knn, const float* w, float* mat12) {
    std::vector<DualQuaternion> f(4);
    for (int k = 0; k < 4; ++k) f[k] = load_dq(field + 8 * (size_t)knn[k]);
    // averageDualQuaternion indexes the field; give it the four nodes at 0..3
    DualQuaternion d = averageDualQuaternion(f.data(), make_ushort4(0, 1, 2, 3), make_float4(w[0], w[1], w[2], w[3]));
    store_mat34(d.se3_matrix(), mat12);
}

void ref_dq_to_mat34(const float* dq8, float* mat12) {
    const DualQuaternion d = load_dq(dq8);
    store_mat34((mat34)d, mat12);
}

void ref_mat34_to_dq(const float* mat12, float* dq8) {
    mat34 m;
    std::memcpy(&m, mat12, 48);
    const DualQuaternion d(m);
    std::memcpy(dq8, &d, 32);
}

void ref_gauss_jordan6(const float* in36, float* out36) {
    float m[36];
    std::memcpy(m, in36, sizeof(m));  // column major, as DenseGaussian assumes
    DenseGaussian<6>::Inverse(m, out36);
}

float ref_huber(float r) { return compute_feature_huber_weight(r); }

void ref_p2p_jacobian(const float* target4, const float* warped4, float* out18) {
    TwistGradientOfScalarCost g[3];
    device::computePointToPointICPTermJacobian(make_float4(target4[0], target4[1], target4[2], target4[3]),
                                               make_float4(warped4[0], warped4[1], warped4[2], warped4[3]), g);
    for (int c = 0; c < 3; ++c) store_gradient(g[c], out18 + 6 * c);
}

void ref_p2p_jt_residual(const float* target4, const float* warped4, float* out6) {
    device::computePoint2PointJtResidual(make_float4(target4[0], target4[1], target4[2], target4[3]),
                                         make_float4(warped4[0], warped4[1], warped4[2], warped4[3]), out6);
}

void ref_smooth_jacobian(const float* ti_xj, const float* tj_xj, int is_node_i, float* out18) {
    TwistGradientOfScalarCost g[3];
    device::computeSmoothTermJacobian(make_float3(ti_xj[0], ti_xj[1], ti_xj[2]), make_float3(tj_xj[0], tj_xj[1], tj_xj[2]),
                                      is_node_i != 0, g);
    for (int c = 0; c < 3; ++c) store_gradient(g[c], out18 + 6 * c);
}

void ref_smooth_jt_residual(const float* ti_xj, const float* tj_xj, int is_node_i, float* out6) {
    device::computeSmoothTermJtResidual(make_float3(ti_xj[0], ti_xj[1], ti_xj[2]),
                                        make_float3(tj_xj[0], tj_xj[1], tj_xj[2]), is_node_i != 0, out6);
}

uint32_t ref_encode_nodepair(uint16_t i, uint16_t j) { return encode_nodepair(i, j); }

// sizes (dense, smooth, foreground, feature, cross) -> prefix offsets; then
// the (type, typed index) of every term id in [0, total)
void ref_term_offsets(const uint32_t* sizes5, uint32_t* offsets5, uint32_t* types, uint32_t* typed) {
    std::vector<ushort4> d(sizes5[0]), f(sizes5[2]), p(sizes5[3]), c(sizes5[4]);
    std::vector<ushort2> s(sizes5[1]);
    TermTypeOffset off;
    size2offset(off, DeviceArrayView<ushort4>(d.data(), d.size()), DeviceArrayView<ushort2>(s.data(), s.size()),
                DeviceArrayView<ushort4>(f.data(), f.size()), DeviceArrayView<ushort4>(p.data(), p.size()),
                DeviceArrayView<ushort4>(c.data(), c.size()));
    for (int k = 0; k < 5; ++k) offsets5[k] = off.offset_value[k];
    for (uint32_t t = 0; t < off.TermSize(); ++t) {
        TermType ty;
        unsigned k;
        query_typed_index(t, off, ty, k);
        types[t] = (uint32_t)ty;
        typed[t] = k;
    }
}

// The reference's image-term function on the GPU. Maps: per view an image
// (float) and its gradient (float2), height x width, packed rows; terms:
// reference vertex, camera, 4-NN and weights, geometry density; field: the
// warp field (8 floats per node); out: 7 floats per term (gradient, residual).
// Returns 0 on success, a CUDA error code otherwise.
int ref_image_terms(uint32_t views, uint32_t width, uint32_t height, const float* const* images,
                    const float* const* gradients, const float* intrinsics4, const float* world2camera12,
                    const float* initial12, uint32_t count, const float* ref_vertex4, const uint16_t* camera,
                    const uint16_t* knn4, const float* weight4, const float* geometry, uint32_t nodes,
                    const float* field8, float* out7) {
    std::vector<void*> keep;
    std::vector<cudaArray_t> arrays;
    std::vector<cudaTextureObject_t> img(views), grad(views);
    cudaError_t e = cudaSuccess;
    auto make = [&](const void* host, cudaChannelFormatDesc fmt, size_t elem) -> cudaTextureObject_t {
        cudaArray_t a = nullptr;
        if ((e = cudaMallocArray(&a, &fmt, width, height)) != cudaSuccess) return 0;
        arrays.push_back(a);
        if ((e = cudaMemcpy2DToArray(a, 0, 0, host, width * elem, width * elem, height, cudaMemcpyHostToDevice)) !=
            cudaSuccess)
            return 0;
        cudaResourceDesc rd;
        std::memset(&rd, 0, sizeof(rd));
        rd.resType = cudaResourceTypeArray;
        rd.res.array.array = a;
        cudaTextureDesc td;
        std::memset(&td, 0, sizeof(td));
        td.addressMode[0] = td.addressMode[1] = cudaAddressModeClamp;
        td.filterMode = cudaFilterModePoint;
        td.readMode = cudaReadModeElementType;
        cudaTextureObject_t t = 0;
        e = cudaCreateTextureObject(&t, &rd, &td, nullptr);
        return t;
    };
    for (uint32_t v = 0; v < views && e == cudaSuccess; ++v) {
        img[v] = make(images[v], cudaCreateChannelDesc<float>(), 4);
        if (e == cudaSuccess) grad[v] = make(gradients[v], cudaCreateChannelDesc<float2>(), 8);
    }
    std::vector<Intrinsic> intr(views);
    std::vector<mat34> w2c(views), init(views);
    for (uint32_t v = 0; v < views; ++v) {
        intr[v].principal_x = intrinsics4[4 * v];
        intr[v].principal_y = intrinsics4[4 * v + 1];
        intr[v].focal_x = intrinsics4[4 * v + 2];
        intr[v].focal_y = intrinsics4[4 * v + 3];
        std::memcpy(&w2c[v], world2camera12 + 12 * v, 48);
        std::memcpy(&init[v], initial12 + 12 * v, 48);
    }
    float* d_out = nullptr;
    if (e == cudaSuccess && count) {
        auto* d_img = to_device(img.data(), views, keep);
        auto* d_grad = to_device(grad.data(), views, keep);
        auto* d_intr = to_device(intr.data(), views, keep);
        auto* d_w2c = to_device(w2c.data(), views, keep);
        auto* d_init = to_device(init.data(), views, keep);
        auto* d_ref = to_device(reinterpret_cast<const float4*>(ref_vertex4), count, keep);
        auto* d_cam = to_device(camera, count, keep);
        auto* d_knn = to_device(reinterpret_cast<const ushort4*>(knn4), count, keep);
        auto* d_w = to_device(reinterpret_cast<const float4*>(weight4), count, keep);
        auto* d_geo = to_device(geometry, count, keep);
        auto* d_field = to_device(reinterpret_cast<const DualQuaternion*>(field8), nodes, keep);
        e = cudaMalloc(&d_out, 7 * sizeof(float) * count);
        if (e == cudaSuccess && d_img && d_grad && d_intr && d_w2c && d_init && d_ref && d_cam && d_knn && d_w &&
            d_geo && d_field) {
            image_terms_kernel<<<(count + 127) / 128, 128>>>(count, d_ref, d_cam, d_knn, d_w, d_geo, d_field, d_img,
                                                           d_grad, d_intr, d_w2c, d_init, width, height, d_out);
            e = cudaGetLastError();
            if (e == cudaSuccess) e = cudaMemcpy(out7, d_out, 7 * sizeof(float) * count, cudaMemcpyDeviceToHost);
        } else if (e == cudaSuccess) {
            e = cudaErrorMemoryAllocation;
        }
    }
    if (d_out) cudaFree(d_out);
    for (void* p : keep) cudaFree(p);
    for (uint32_t v = 0; v < views; ++v) {
        if (img[v]) cudaDestroyTextureObject(img[v]);
        if (grad[v]) cudaDestroyTextureObject(grad[v]);
    }
    for (cudaArray_t a : arrays) cudaFreeArray(a);
    return (int)e;
}

}  // extern "C"
