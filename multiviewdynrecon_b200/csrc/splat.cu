// The renderer's solver-map pass on CUDA (mvdr_render_solver_maps).
//
// The reference draws every surfel as an OpenGL point into six render targets
// (render/shaders/SolverMap.vert, SolverMapSized.vert, SolverMapIndexMap.vert,
// SolverMap.frag, drawn by RendererDraw.cpp:384-480) with a GL_LESS depth test
// against a float depth buffer cleared to 1 (GLRenderMaps.cpp:207-218). Here
// that is two kernels:
//   splat   - a thread per surfel, for every view: cull, project, size the
//             point, and for every pixel the point covers an atomicMin of
//             (camera z bits << 32 | id) into a 64-bit depth-index word.
//             Positive floats order as their bit patterns, so the minimum is
//             the nearest surfel and, among equal depths, the smallest id:
//             the point drawn first, which is the one GL_LESS keeps. The
//             result does not depend on the order in which threads run.
//   resolve - a thread per pixel of each view: write the winning surfel's
//             attributes (a point's fragments all carry its vertex outputs)
//             or the clear values.
// This file is compiled with -fmad=false: every float operation is a single
// IEEE operation, as in the CPU restatement the tests compare it with.
#include <algorithm>
#include <cstring>
#include <string>

#include "batch.cuh"
#include "kernels_common.cuh"

namespace mvdr {
namespace {

constexpr float kMaxPointSize = 2047.0f;  // the implementation's point-size range is [1, 2047]

struct SplatView {
    float w2c[12];  // row-major rotation, translation
    float inv[12];  // inverse of initial_camera_se3, row-major rotation, translation
    float cx, cy, fx, fy;
    int sized;
    uint32_t pitch;
    float4* ref_v;
    float4* ref_n;
    float4* live_v;
    float4* live_n;
    uint32_t* index;
    float4* rgb;
    unsigned long long* zbuf;
};

struct SplatArgs {
    SplatView v[MVDR_MAX_VIEWS];
    uint32_t num_views, any_sized;
    uint32_t num_surfels, width, height;
    float max_depth, now, conf_thr, time_thr;
    const float4* ref_vc;
    const float4* ref_nr;
    const float4* live_v;
    const float4* live_n;
    const float4* color_time;
};

__device__ inline float3 mat_point(const float* m, float3 p) {
    return make_float3(m[0] * p.x + m[1] * p.y + m[2] * p.z + m[9], m[3] * p.x + m[4] * p.y + m[5] * p.z + m[10],
                       m[6] * p.x + m[7] * p.y + m[8] * p.z + m[11]);
}
__device__ inline float3 mat_dir(const float* m, float3 p) {
    return make_float3(m[0] * p.x + m[1] * p.y + m[2] * p.z, m[3] * p.x + m[4] * p.y + m[5] * p.z,
                       m[6] * p.x + m[7] * p.y + m[8] * p.z);
}
__device__ inline float3 normalized3(float3 v) {
    const float inv = 1.0f / sqrtf(v.x * v.x + v.y * v.y + v.z * v.z);
    return make_float3(v.x * inv, v.y * inv, v.z * inv);
}
// project_point_image of SolverMapSized.vert: ((fx x) / z + cx, (fy y) / z + cy)
__device__ inline float2 image_point(const SplatView& V, float3 p) {
    return make_float2((V.fx * p.x) / p.z + V.cx, (V.fy * p.y) / p.z + V.cy);
}

// One thread per surfel, every view: the surfel's attributes are read once
// and splatted into each view's depth-index buffer.
__global__ void __launch_bounds__(256) splat_kernel(const __grid_constant__ SplatArgs a) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= a.num_surfels) return;
    const float4 lv = a.live_v[s];
    const float4 ct = a.color_time[s];
    const float conf = a.ref_vc[s].w;
    // the culling test that does not depend on the view: unstable and not
    // recently observed
    if (conf < a.conf_thr && fabsf(ct.z - a.now) >= a.time_thr) return;
    float4 ln = make_float4(0.f, 0.f, 0.f, 0.f);
    float radius = 0.0f;
    if (a.any_sized) {
        ln = a.live_n[s];
        radius = a.ref_nr[s].w;
    }
    for (uint32_t v = 0; v < a.num_views; ++v) {
        const SplatView& V = a.v[v];
        // the point in the view's camera: world2camera * initialCameraSE3^-1 * live
        const float3 pc = mat_point(V.w2c, mat_point(V.inv, make_float3(lv.x, lv.y, lv.z)));
        if (pc.z > a.max_depth + 0.05f || !(pc.z > 0.0f)) continue;  // culled (moved out of the clip volume)
        const float2 c = image_point(V, pc);
        // GL clips a point by its centre: the window position must be in the image
        if (!(c.x >= 0.0f && c.x <= (float)a.width && c.y >= 0.0f && c.y <= (float)a.height)) continue;
        float size = 1.0f;
        if (V.sized) {
            // SolverMapSized.vert: the extent of the surfel's disc in the image
            const float3 n = normalized3(mat_dir(V.w2c, mat_dir(V.inv, make_float3(ln.x, ln.y, ln.z))));
            const float scale = radius * 1.41421356f * 0.001f;
            const float3 x0 = normalized3(make_float3(n.y - n.z, -n.x, n.x));
            const float3 x1 = make_float3(x0.x * scale, x0.y * scale, x0.z * scale);
            const float3 y1 =
                make_float3(n.y * x1.z - n.z * x1.y, n.z * x1.x - n.x * x1.z, n.x * x1.y - n.y * x1.x);
            const float2 p1 = image_point(V, make_float3(pc.x + x1.x, pc.y + x1.y, pc.z + x1.z));
            const float2 p2 = image_point(V, make_float3(pc.x + y1.x, pc.y + y1.y, pc.z + y1.z));
            const float2 p3 = image_point(V, make_float3(pc.x - y1.x, pc.y - y1.y, pc.z - y1.z));
            const float2 p4 = image_point(V, make_float3(pc.x - x1.x, pc.y - x1.y, pc.z - x1.z));
            const float xd =
                fmaxf(p1.x, fmaxf(p2.x, fmaxf(p3.x, p4.x))) - fminf(p1.x, fminf(p2.x, fminf(p3.x, p4.x)));
            const float yd =
                fmaxf(p1.y, fmaxf(p2.y, fmaxf(p3.y, p4.y))) - fminf(p1.y, fminf(p2.y, fminf(p3.y, p4.y)));
            size = fminf(fmaxf(fmaxf(0.0f, fminf(fabsf(xd), fabsf(yd))), 1.0f), kMaxPointSize);
        }
        // the pixels whose centres lie in [c - size/2, c + size/2)
        const float h = 0.5f * size;
        const int u0 = max(0, (int)ceilf(c.x - h - 0.5f)), u1 = min((int)a.width, (int)ceilf(c.x + h - 0.5f));
        const int w0 = max(0, (int)ceilf(c.y - h - 0.5f)), w1 = min((int)a.height, (int)ceilf(c.y + h - 0.5f));
        const unsigned long long key = ((unsigned long long)__float_as_uint(pc.z) << 32) | s;
        for (int w = w0; w < w1; ++w)
            for (int u = u0; u < u1; ++u) atomicMin(V.zbuf + (size_t)w * V.pitch + u, key);
    }
}

__global__ void __launch_bounds__(256) resolve_kernel(const __grid_constant__ SplatArgs a) {
    const SplatView& V = a.v[blockIdx.y];
    const size_t npix = (size_t)a.width * a.height;
    for (size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x; p < npix; p += (size_t)gridDim.x * blockDim.x) {
        const uint32_t u = (uint32_t)(p % a.width), w = (uint32_t)(p / a.width);
        const size_t o = (size_t)w * V.pitch + u;
        const unsigned long long key = V.zbuf[o];
        float4 rv = make_float4(0.f, 0.f, 0.f, 0.f), rn = rv, lv = rv, ln = rv, rgb = rv;
        uint32_t id = kInvalid;
        if (key != ~0ull) {
            id = (uint32_t)(key & 0xffffffffull);
            const float4 a_rv = a.ref_vc[id], a_rn = a.ref_nr[id], a_lv = a.live_v[id], a_ln = a.live_n[id];
            const float4 ct = a.color_time[id];
            // SolverMapIndexMap.vert: the attributes in camera v's frame
            const float3 q0 = mat_point(V.inv, make_float3(a_rv.x, a_rv.y, a_rv.z));
            const float3 q1 = mat_dir(V.inv, make_float3(a_rn.x, a_rn.y, a_rn.z));
            const float3 q2 = mat_point(V.inv, make_float3(a_lv.x, a_lv.y, a_lv.z));
            const float3 q3 = mat_dir(V.inv, make_float3(a_ln.x, a_ln.y, a_ln.z));
            rv = make_float4(q0.x, q0.y, q0.z, 1.0f);
            rn = make_float4(q1.x, q1.y, q1.z, 0.0f);
            lv = make_float4(q2.x, q2.y, q2.z, 1.0f);
            ln = make_float4(q3.x, q3.y, q3.z, 0.0f);
            const uint32_t bits = __float_as_uint(ct.x);  // floatBitsToInt(color_time.x)
            rgb = make_float4((float)((bits & 0x00FF0000u) >> 16) / 255.f, (float)((bits & 0x0000FF00u) >> 8) / 255.f,
                              (float)(bits & 0x000000FFu) / 255.f, V.sized ? 1.0f : ct.y);
        }
        if (V.ref_v) V.ref_v[o] = rv;
        if (V.ref_n) V.ref_n[o] = rn;
        if (V.live_v) V.live_v[o] = lv;
        if (V.live_n) V.live_n[o] = ln;
        if (V.rgb) V.rgb[o] = rgb;
        V.index[o] = id;
    }
}

void load_rows(const mvdr_mat34& m, float* out) {
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) out[3 * r + c] = m.rot[3 * c + r];
    for (int r = 0; r < 3; ++r) out[9 + r] = m.trans[r];
}

}  // namespace
}  // namespace mvdr

using namespace mvdr;

extern "C" int mvdr_render_solver_maps(const mvdr_surfel_geometry* g, const mvdr_solver_map_params* prm,
                                       const mvdr_solver_map_view* views, uint32_t num_views, void* stream) {
    if (!g || !prm || !views) return fail(MVDR_EINVAL, "mvdr_render_solver_maps: null argument");
    if (num_views == 0 || num_views > MVDR_MAX_VIEWS)
        return fail(MVDR_EINVAL, "mvdr_render_solver_maps: num_views must be in [1, MVDR_MAX_VIEWS]");
    if (prm->width == 0 || prm->height == 0 || prm->width > 65535 || prm->height > 65535)
        return fail(MVDR_EINVAL, "mvdr_render_solver_maps: image size out of range");
    if (g->num_surfels && (!g->reference_vertex_confid || !g->reference_normal_radius || !g->live_vertex_confid ||
                           !g->live_normal_radius || !g->color_time))
        return fail(MVDR_EINVAL, "mvdr_render_solver_maps: missing surfel arrays");
    if (g->num_surfels == 0xFFFFFFFFu) return fail(MVDR_ECAPACITY, "mvdr_render_solver_maps: too many surfels");
    SplatArgs a;
    std::memset(&a, 0, sizeof(a));
    a.num_views = num_views;
    a.num_surfels = g->num_surfels;
    a.width = prm->width;
    a.height = prm->height;
    a.max_depth = prm->max_depth;
    a.now = prm->current_time;
    a.conf_thr = prm->confidence_threshold;
    a.time_thr = prm->time_threshold;
    a.ref_vc = reinterpret_cast<const float4*>(g->reference_vertex_confid);
    a.ref_nr = reinterpret_cast<const float4*>(g->reference_normal_radius);
    a.live_v = reinterpret_cast<const float4*>(g->live_vertex_confid);
    a.live_n = reinterpret_cast<const float4*>(g->live_normal_radius);
    a.color_time = reinterpret_cast<const float4*>(g->color_time);
    const cudaStream_t st = (cudaStream_t)stream;
    for (uint32_t v = 0; v < num_views; ++v) {
        const mvdr_solver_map_view& in = views[v];
        SplatView& V = a.v[v];
        if (!in.index_map || !in.depth_index)
            return fail(MVDR_EINVAL, "mvdr_render_solver_maps: index_map and depth_index are required");
        V.pitch = in.pitch ? in.pitch : prm->width;
        if (V.pitch < prm->width) return fail(MVDR_EINVAL, "mvdr_render_solver_maps: pitch smaller than width");
        load_rows(in.world2camera, V.w2c);
        // mat34::inverse (math/MatUtils.h:585-590) in float
        float init[12];
        load_rows(in.initial_camera_se3, init);
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) V.inv[3 * r + c] = init[3 * c + r];
        for (int r = 0; r < 3; ++r)
            V.inv[9 + r] = -(V.inv[3 * r] * init[9] + V.inv[3 * r + 1] * init[10] + V.inv[3 * r + 2] * init[11]);
        V.cx = in.intrinsic.principal_x;
        V.cy = in.intrinsic.principal_y;
        V.fx = in.intrinsic.focal_x;
        V.fy = in.intrinsic.focal_y;
        V.sized = in.sized_points ? 1 : 0;
        a.any_sized |= (uint32_t)V.sized;
        V.ref_v = reinterpret_cast<float4*>(in.reference_vertex_map);
        V.ref_n = reinterpret_cast<float4*>(in.reference_normal_map);
        V.live_v = reinterpret_cast<float4*>(in.live_vertex_map);
        V.live_n = reinterpret_cast<float4*>(in.live_normal_map);
        V.index = in.index_map;
        V.rgb = reinterpret_cast<float4*>(in.normalized_rgb_map);
        V.zbuf = reinterpret_cast<unsigned long long*>(in.depth_index);
    }
    // every argument is checked before the first call into CUDA
    for (uint32_t v = 0; v < num_views; ++v) {
        // the depth test starts from "nothing drawn"
        const cudaError_t e =
            cudaMemsetAsync(a.v[v].zbuf, 0xFF, sizeof(unsigned long long) * a.v[v].pitch * prm->height, st);
        if (e != cudaSuccess) return fail(MVDR_ECUDA, std::string("mvdr_render_solver_maps: ") + cudaGetErrorString(e));
    }
    if (g->num_surfels)
        MVDR_LAUNCH(splat_kernel, dim3((g->num_surfels + 255) / 256), 256, 0, st, a);
    int sms = 148;
    int dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const size_t npix = (size_t)prm->width * prm->height;
    const uint32_t blocks = (uint32_t)std::min<size_t>((npix + 255) / 256, 8u * (size_t)sms);
    MVDR_LAUNCH(resolve_kernel, dim3(blocks, num_views), 256, 0, st, a);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(MVDR_ECUDA, std::string("mvdr_render_solver_maps: ") + cudaGetErrorString(e));
    return MVDR_OK;
}
