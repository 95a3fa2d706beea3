// Native test of the texture-object boundary, compiled against include/mvdr.h
// and linked to libmvdr.so (no Python in the path).
//
// The reference hands the solver its maps as cudaTextureObject_t
// (Renderer::SolverMaps, CameraObservation). This program loads an input
// bundle, solves it once with the maps as plain device arrays
// (mvdr_set_inputs_host) and once with the maps behind texture objects
// (mvdr_set_inputs_textures): cudaArrays for even views, pitched device
// memory for odd views. The two warp fields must be bit-identical, and the
// device view mvdr_node_se3_device must hold the same field. A map whose
// channel format differs from the expected one must be rejected.
//
// usage: texture_boundary <bundle> <gauss-newton iterations> <pcg iterations>
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "mvdr.h"

#define CHECK_CUDA(x)                                                                            \
    do {                                                                                         \
        cudaError_t e = (x);                                                                     \
        if (e != cudaSuccess) {                                                                  \
            std::fprintf(stderr, "%s:%d %s: %s\n", __FILE__, __LINE__, #x, cudaGetErrorString(e)); \
            std::exit(2);                                                                        \
        }                                                                                        \
    } while (0)
#define CHECK_MVDR(x)                                                                                \
    do {                                                                                             \
        int s = (x);                                                                                 \
        if (s != MVDR_OK) {                                                                          \
            std::fprintf(stderr, "%s:%d %s: status %d: %s\n", __FILE__, __LINE__, #x, s, mvdr_last_error_string()); \
            std::exit(3);                                                                            \
        }                                                                                            \
    } while (0)

namespace {

struct Map {
    const void* host;         // the bundle's copy
    uint64_t* tex;            // where its texture handle goes
    cudaChannelFormatDesc fmt;
    size_t elem;
};

std::vector<void*> g_device_buffers;
std::vector<cudaArray_t> g_arrays;
std::vector<cudaTextureObject_t> g_textures;

// a texture over a copy of `host` (width x height elements, packed rows):
// a cudaArray or pitched device memory
cudaTextureObject_t make_texture(const void* host, const cudaChannelFormatDesc& fmt, size_t elem, uint32_t w,
                                 uint32_t h, bool as_array) {
    cudaResourceDesc rd;
    std::memset(&rd, 0, sizeof(rd));
    if (as_array) {
        cudaArray_t a = nullptr;
        CHECK_CUDA(cudaMallocArray(&a, &fmt, w, h));
        CHECK_CUDA(cudaMemcpy2DToArray(a, 0, 0, host, w * elem, w * elem, h, cudaMemcpyHostToDevice));
        g_arrays.push_back(a);
        rd.resType = cudaResourceTypeArray;
        rd.res.array.array = a;
    } else {
        void* p = nullptr;
        size_t pitch = 0;
        CHECK_CUDA(cudaMallocPitch(&p, &pitch, w * elem, h));
        CHECK_CUDA(cudaMemcpy2D(p, pitch, host, w * elem, w * elem, h, cudaMemcpyHostToDevice));
        g_device_buffers.push_back(p);
        rd.resType = cudaResourceTypePitch2D;
        rd.res.pitch2D.devPtr = p;
        rd.res.pitch2D.desc = fmt;
        rd.res.pitch2D.width = w;
        rd.res.pitch2D.height = h;
        rd.res.pitch2D.pitchInBytes = pitch;
    }
    cudaTextureDesc td;
    std::memset(&td, 0, sizeof(td));
    td.addressMode[0] = td.addressMode[1] = cudaAddressModeClamp;
    td.filterMode = cudaFilterModePoint;
    td.readMode = cudaReadModeElementType;
    td.normalizedCoords = 0;
    cudaTextureObject_t t = 0;
    CHECK_CUDA(cudaCreateTextureObject(&t, &rd, &td, nullptr));
    g_textures.push_back(t);
    return t;
}

const void* to_device(const void* host, size_t bytes) {
    if (!host || !bytes) return nullptr;
    void* p = nullptr;
    CHECK_CUDA(cudaMalloc(&p, bytes));
    CHECK_CUDA(cudaMemcpy(p, host, bytes, cudaMemcpyHostToDevice));
    g_device_buffers.push_back(p);
    return p;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc != 4) {
        std::fprintf(stderr, "usage: %s <bundle> <gn> <pcg>\n", argv[0]);
        return 64;
    }
    const uint32_t gn = (uint32_t)std::atoi(argv[2]), pcg = (uint32_t)std::atoi(argv[3]);
    mvdr_input_bundle* bundle = nullptr;
    CHECK_MVDR(mvdr_load_input_bundle(argv[1], &bundle));
    const mvdr_config cfg = *mvdr_input_bundle_config(bundle);
    const mvdr_inputs host_in = *mvdr_input_bundle_inputs(bundle);
    const uint32_t W = cfg.image_width, H = cfg.image_height, N = host_in.num_nodes;
    cudaStream_t st;
    CHECK_CUDA(cudaStreamCreate(&st));

    // A: the maps as device arrays
    mvdr_solver* a = nullptr;
    CHECK_MVDR(mvdr_create(&cfg, &a));
    CHECK_MVDR(mvdr_set_inputs_host(a, &host_in, st));
    CHECK_MVDR(mvdr_solve(a, gn, pcg, st));
    std::vector<mvdr_dual_quaternion> fa(N), fb(N), fc(N);
    CHECK_MVDR(mvdr_get_node_se3(a, fa.data(), st));

    // B: the maps behind texture objects, the other arrays on the device
    std::vector<mvdr_view_textures> tex(host_in.num_views);
    std::memset(tex.data(), 0, tex.size() * sizeof(mvdr_view_textures));
    const cudaChannelFormatDesc f4 = cudaCreateChannelDesc<float4>(), f1 = cudaCreateChannelDesc<float>(),
                                f2 = cudaCreateChannelDesc<float2>(), u1 = cudaCreateChannelDesc<unsigned int>();
    for (uint32_t v = 0; v < host_in.num_views; ++v) {
        const mvdr_view_inputs& V = host_in.views[v];
        mvdr_view_textures& T = tex[v];
        const Map maps[] = {
            {V.reference_vertex_map, &T.reference_vertex_map, f4, 16},
            {V.reference_normal_map, &T.reference_normal_map, f4, 16},
            {V.index_map, &T.index_map, u1, 4},
            {V.normalized_rgb_map, &T.normalized_rgb_map, f4, 16},
            {V.vertex_confidence_map, &T.vertex_confidence_map, f4, 16},
            {V.normal_radius_map, &T.normal_radius_map, f4, 16},
            {V.filtered_foreground_mask, &T.filtered_foreground_mask, f1, 4},
            {V.foreground_mask_gradient, &T.foreground_mask_gradient, f2, 8},
            {V.density_map, &T.density_map, f1, 4},
            {V.density_gradient_map, &T.density_gradient_map, f2, 8},
        };
        for (const Map& m : maps)
            if (m.host) *m.tex = make_texture(m.host, m.fmt, m.elem, W, H, v % 2 == 0);
    }
    mvdr_inputs dev_in = host_in;
    dev_in.surfel_knn = (const uint16_t*)to_device(host_in.surfel_knn, 8 * (size_t)host_in.num_surfels);
    dev_in.surfel_knn_weight = (const mvdr_float4*)to_device(host_in.surfel_knn_weight, 16 * (size_t)host_in.num_surfels);
    dev_in.node_se3 = (const mvdr_dual_quaternion*)to_device(host_in.node_se3, 32 * (size_t)N);
    dev_in.canonical_node_coords = (const mvdr_float4*)to_device(host_in.canonical_node_coords, 16 * (size_t)N);
    dev_in.node_graph = (const uint16_t*)to_device(host_in.node_graph, 4 * (size_t)host_in.num_graph_edges);
    for (mvdr_correspondences* c : {&dev_in.feature, &dev_in.cross_view}) {
        const size_t n = c->count;
        c->target_vertex = (const mvdr_float4*)to_device(c->target_vertex, 16 * n);
        c->reference_vertex = (const mvdr_float4*)to_device(c->reference_vertex, 16 * n);
        c->knn = (const uint16_t*)to_device(c->knn, 8 * n);
        c->knn_weight = (const mvdr_float4*)to_device(c->knn_weight, 16 * n);
    }
    mvdr_solver* b = nullptr;
    CHECK_MVDR(mvdr_create(&cfg, &b));
    CHECK_MVDR(mvdr_set_inputs_textures(b, &dev_in, tex.data(), st));
    CHECK_MVDR(mvdr_solve(b, gn, pcg, st));
    CHECK_MVDR(mvdr_get_node_se3(b, fb.data(), st));
    const mvdr_dual_quaternion* view = nullptr;
    CHECK_MVDR(mvdr_node_se3_device(b, &view));
    CHECK_CUDA(cudaMemcpyAsync(fc.data(), view, sizeof(mvdr_dual_quaternion) * N, cudaMemcpyDeviceToHost, st));
    CHECK_CUDA(cudaStreamSynchronize(st));

    int bad = 0;
    if (std::memcmp(fa.data(), fb.data(), sizeof(mvdr_dual_quaternion) * N) != 0) {
        std::fprintf(stderr, "texture-fed solve differs from the pointer-fed solve\n");
        bad = 1;
    }
    if (std::memcmp(fb.data(), fc.data(), sizeof(mvdr_dual_quaternion) * N) != 0) {
        std::fprintf(stderr, "mvdr_node_se3_device differs from mvdr_get_node_se3\n");
        bad = 1;
    }
    // a float map where the reference vertex map (float4) belongs is refused
    mvdr_view_textures wrong = tex[0];
    wrong.reference_vertex_map = tex[0].filtered_foreground_mask ? tex[0].filtered_foreground_mask : tex[0].index_map;
    std::vector<mvdr_view_textures> wrong_all = tex;
    wrong_all[0] = wrong;
    const int s = mvdr_set_inputs_textures(b, &dev_in, wrong_all.data(), st);
    if (s != MVDR_EINVAL) {
        std::fprintf(stderr, "a map of the wrong format gave status %d, not MVDR_EINVAL\n", s);
        bad = 1;
    }

    for (cudaTextureObject_t t : g_textures) cudaDestroyTextureObject(t);
    for (cudaArray_t arr : g_arrays) cudaFreeArray(arr);
    for (void* p : g_device_buffers) cudaFree(p);
    mvdr_destroy(a);
    mvdr_destroy(b);
    mvdr_free_input_bundle(bundle);
    cudaStreamDestroy(st);
    if (!bad) std::printf("texture boundary ok: %u nodes, %u views, bit-identical\n", N, host_in.num_views);
    return bad;
}
