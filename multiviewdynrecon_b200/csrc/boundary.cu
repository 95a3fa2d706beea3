// The reference-facing edges of the C ABI beyond device pointers: maps handed
// over as texture objects (the form in which the reference's NonRigidSolver
// receives Renderer::SolverMaps and CameraObservation), the warp field as a
// device view (SolvedNodeSE3), and input bundles that replay one solve's
// inputs.
#include <cstddef>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "batch.cuh"

namespace mvdr {
namespace {

#define CU(call)                                                                           \
    do {                                                                                   \
        cudaError_t e__ = (call);                                                          \
        if (e__ != cudaSuccess)                                                            \
            return fail(MVDR_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e__)); \
    } while (0)

// Pointer fields of the public structs are read and written through their
// addresses with memcpy, so that one routine serves fields of different
// pointer types without aliasing them.
inline const void* get_ptr(const void* field) {
    const void* p;
    std::memcpy(&p, field, sizeof(p));
    return p;
}
inline void set_ptr(void* field, const void* p) { std::memcpy(field, &p, sizeof(p)); }

// One map of a view: the offsets of its texture handle in mvdr_view_textures
// and of its pointer in mvdr_view_inputs, its element size and channels.
struct MapSpec {
    size_t tex;
    size_t ptr;
    uint32_t elem_bytes;
    uint32_t channels;  // 32-bit channels of the element
    bool integer;       // unsigned int element (the index map)
};

#define MVDR_MAP(name, bytes, ch, integer) \
    {offsetof(mvdr_view_textures, name), offsetof(mvdr_view_inputs, name), bytes, ch, integer}
const MapSpec kMaps[] = {
    MVDR_MAP(reference_vertex_map, 16, 4, false),    MVDR_MAP(reference_normal_map, 16, 4, false),
    MVDR_MAP(index_map, 4, 1, true),                 MVDR_MAP(normalized_rgb_map, 16, 4, false),
    MVDR_MAP(vertex_confidence_map, 16, 4, false),   MVDR_MAP(normal_radius_map, 16, 4, false),
    MVDR_MAP(filtered_foreground_mask, 4, 1, false), MVDR_MAP(foreground_mask_gradient, 8, 2, false),
    MVDR_MAP(density_map, 4, 1, false),              MVDR_MAP(density_gradient_map, 8, 2, false),
};
#undef MVDR_MAP

inline uint64_t tex_of(const mvdr_view_textures& t, const MapSpec& m) {
    uint64_t h;
    std::memcpy(&h, reinterpret_cast<const char*>(&t) + m.tex, sizeof(h));
    return h;
}
inline void* map_field(mvdr_view_inputs& V, const MapSpec& m) { return reinterpret_cast<char*>(&V) + m.ptr; }
constexpr int kNumMaps = sizeof(kMaps) / sizeof(kMaps[0]);

// does a channel descriptor describe the map's element (32-bit channels of
// the right kind)?
bool channels_match(const cudaChannelFormatDesc& d, const MapSpec& m) {
    const int bits[4] = {d.x, d.y, d.z, d.w};
    for (uint32_t c = 0; c < 4; ++c)
        if (bits[c] != (c < m.channels ? 32 : 0)) return false;
    return m.integer ? d.f == cudaChannelFormatKindUnsigned : d.f == cudaChannelFormatKindFloat;
}

// Copy the resource behind texture `tex` (width x height elements of
// m.elem_bytes) into `dst` (rows packed, pitch = width) on `st`.
int stage_map(uint64_t tex, const MapSpec& m, uint32_t width, uint32_t height, void* dst, cudaStream_t st,
              const char* name) {
    cudaResourceDesc rd;
    std::memset(&rd, 0, sizeof(rd));
    CU(cudaGetTextureObjectResourceDesc(&rd, (cudaTextureObject_t)tex));
    const size_t row = (size_t)width * m.elem_bytes;
    switch (rd.resType) {
        case cudaResourceTypeArray: {
            cudaChannelFormatDesc d;
            cudaExtent ext;
            unsigned int flags = 0;
            CU(cudaArrayGetInfo(&d, &ext, &flags, rd.res.array.array));
            if (!channels_match(d, m)) return fail(MVDR_EINVAL, std::string(name) + ": array channel format differs");
            if (ext.width != width || ext.height != height || ext.depth > 1)
                return fail(MVDR_EINVAL, std::string(name) + ": array extent differs from the image size");
            CU(cudaMemcpy2DFromArrayAsync(dst, row, rd.res.array.array, 0, 0, row, height, cudaMemcpyDeviceToDevice,
                                          st));
            return MVDR_OK;
        }
        case cudaResourceTypePitch2D: {
            if (!channels_match(rd.res.pitch2D.desc, m))
                return fail(MVDR_EINVAL, std::string(name) + ": pitched channel format differs");
            if (rd.res.pitch2D.width != width || rd.res.pitch2D.height != height)
                return fail(MVDR_EINVAL, std::string(name) + ": pitched extent differs from the image size");
            CU(cudaMemcpy2DAsync(dst, row, rd.res.pitch2D.devPtr, rd.res.pitch2D.pitchInBytes, row, height,
                                 cudaMemcpyDeviceToDevice, st));
            return MVDR_OK;
        }
        case cudaResourceTypeLinear: {
            if (!channels_match(rd.res.linear.desc, m))
                return fail(MVDR_EINVAL, std::string(name) + ": linear channel format differs");
            if (rd.res.linear.sizeInBytes < row * height)
                return fail(MVDR_EINVAL, std::string(name) + ": linear buffer smaller than the image");
            CU(cudaMemcpyAsync(dst, rd.res.linear.devPtr, row * height, cudaMemcpyDeviceToDevice, st));
            return MVDR_OK;
        }
        default:
            return fail(MVDR_EINVAL, std::string(name) + ": unsupported texture resource (mipmapped array)");
    }
}

const char* const kMapNames[kNumMaps] = {"reference_vertex_map", "reference_normal_map", "index_map",
                                         "normalized_rgb_map", "vertex_confidence_map", "normal_radius_map",
                                         "filtered_foreground_mask", "foreground_mask_gradient", "density_map",
                                         "density_gradient_map"};

// Maps a configuration needs; the filtered foreground mask is also carried
// when it is given with the foreground term off (the post-solve node error
// reads it).
bool map_used(const mvdr_config& c, int k, bool given) {
    if (k == 3 || k == 8 || k == 9) return c.use_density != 0;
    if (k == 6) return c.use_foreground != 0 || given;
    if (k == 7) return c.use_foreground != 0;
    return true;
}

// ---------------------------------------------------------------- bundles --
// File: magic, config, inputs (pointer fields meaningless), then every input
// array as (uint64 byte count, bytes) in the order of input_arrays().

constexpr char kBundleMagic[8] = {'M', 'V', 'D', 'R', 'I', 'B', 0, 2};

struct InputArray {
    void* field;  // address of the pointer field in the mvdr_inputs
    size_t bytes;
};

std::vector<InputArray> input_arrays(const mvdr_config& c, mvdr_inputs& in) {
    std::vector<InputArray> v;
    const size_t H = c.image_height;
    auto add = [&](void* f, size_t bytes) { v.push_back({f, bytes}); };
    for (uint32_t k = 0; k < in.num_views && k < MVDR_MAX_VIEWS; ++k) {
        mvdr_view_inputs& V = in.views[k];
        const size_t np = (size_t)(V.pitch ? V.pitch : c.image_width) * H;
        for (int m = 0; m < kNumMaps; ++m)
            add(map_field(V, kMaps[m]),
                map_used(c, m, get_ptr(map_field(V, kMaps[m])) != nullptr) ? (size_t)kMaps[m].elem_bytes * np : 0);
    }
    const uint32_t tp = c.use_feature ? in.feature.count : 0, tc = c.use_cross_view ? in.cross_view.count : 0;
    add(&in.surfel_knn, 8 * (size_t)in.num_surfels);
    add(&in.surfel_knn_weight, 16 * (size_t)in.num_surfels);
    add(&in.node_se3, 32 * (size_t)in.num_nodes);
    add(&in.canonical_node_coords, 16 * (size_t)in.num_nodes);
    add(&in.node_graph, 4 * (size_t)in.num_graph_edges);
    for (mvdr_correspondences* cc : {&in.feature, &in.cross_view}) {
        const size_t n = cc == &in.feature ? tp : tc;
        add(&cc->target_vertex, 16 * n);
        add(&cc->reference_vertex, 16 * n);
        add(&cc->knn, 8 * n);
        add(&cc->knn_weight, 16 * n);
    }
    for (uint32_t k = 0; k < in.num_views && k < MVDR_MAX_VIEWS; ++k) {
        mvdr_feature_pairs& fp = in.feature_pairs;
        const size_t n = c.use_feature ? fp.count[k] : 0;
        const size_t np = (size_t)(in.views[k].pitch ? in.views[k].pitch : c.image_width) * H;
        add(&fp.pixel_pairs[k], 8 * n);
        add(&fp.live_vertex_map[k], n ? 16 * np : 0);
        add(&fp.edge_mask[k], n && fp.edge_mask[k] ? np : 0);
    }
    return v;
}

}  // namespace
}  // namespace mvdr

struct mvdr_input_bundle {
    mvdr_config config;
    mvdr_inputs inputs;
    std::vector<std::vector<unsigned char>> arrays;
};

using namespace mvdr;

extern "C" {

int mvdr_set_inputs_textures(mvdr_solver* s, const mvdr_inputs* in, const mvdr_view_textures* tex, void* stream) {
    if (!s || !in || !tex) return fail(MVDR_EINVAL, "null argument");
    Batch& b = *s->batch;
    const mvdr_config& c = b.cfg;
    if (in->num_views == 0 || in->num_views > c.max_views) return fail(MVDR_ECAPACITY, "num_views exceeds max_views");
    const cudaStream_t st = (cudaStream_t)stream;
    // staging layout: every used map of every view, packed rows, 256-byte aligned
    const size_t np = (size_t)c.image_width * c.image_height;
    size_t total = 0;
    for (uint32_t v = 0; v < in->num_views; ++v)
        for (int m = 0; m < kNumMaps; ++m)
            if (map_used(c, m, tex_of(tex[v], kMaps[m]) != 0))
                total += ((size_t)kMaps[m].elem_bytes * np + 255) & ~(size_t)255;
    OwnedInputs& o = b.staged[s->inst];
    if (o.bytes < total) {
        if (o.mem) CU(cudaFree(o.mem));
        o.mem = nullptr;
        o.bytes = 0;
        CU(cudaMalloc(&o.mem, total));
        o.bytes = total;
    }
    mvdr_inputs dev = *in;
    size_t off = 0;
    for (uint32_t v = 0; v < in->num_views; ++v) {
        mvdr_view_inputs& V = dev.views[v];
        V.pitch = 0;
        for (int m = 0; m < kNumMaps; ++m) {
            set_ptr(map_field(V, kMaps[m]), nullptr);
            const uint64_t h = tex_of(tex[v], kMaps[m]);
            if (!map_used(c, m, h != 0)) continue;
            if (!h) return fail(MVDR_EINVAL, std::string(kMapNames[m]) + " texture missing for view " + std::to_string(v));
            void* dst = static_cast<char*>(o.mem) + off;
            const int rc = stage_map(h, kMaps[m], c.image_width, c.image_height, dst, st, kMapNames[m]);
            if (rc != MVDR_OK) return rc;
            set_ptr(map_field(V, kMaps[m]), dst);
            off += ((size_t)kMaps[m].elem_bytes * np + 255) & ~(size_t)255;
        }
    }
    return bind_inputs(b, s->inst, &dev, st);
}

int mvdr_node_se3_device(mvdr_solver* s, const mvdr_dual_quaternion** out) {
    if (!s || !out) return fail(MVDR_EINVAL, "null argument");
    *out = reinterpret_cast<const mvdr_dual_quaternion*>(s->batch->host[s->inst].se3);
    return MVDR_OK;
}

int mvdr_save_input_bundle(mvdr_solver* s, const char* path, void* stream) {
    if (!s || !path) return fail(MVDR_EINVAL, "null argument");
    Batch& b = *s->batch;
    if (!b.has_inputs[s->inst]) return fail(MVDR_ESTATE, "no inputs bound");
    CU(cudaStreamSynchronize((cudaStream_t)stream));
    mvdr_inputs in = b.bound[s->inst];
    std::vector<InputArray> arrays = input_arrays(b.cfg, in);
    std::unique_ptr<FILE, int (*)(FILE*)> f(std::fopen(path, "wb"), &std::fclose);
    if (!f) return fail(MVDR_EINVAL, std::string("cannot open ") + path);
    bool ok = std::fwrite(kBundleMagic, 1, 8, f.get()) == 8 &&
              std::fwrite(&b.cfg, sizeof(mvdr_config), 1, f.get()) == 1 &&
              std::fwrite(&in, sizeof(mvdr_inputs), 1, f.get()) == 1;
    std::vector<unsigned char> host;
    for (const InputArray& a : arrays) {
        const void* src = get_ptr(a.field);
        const uint64_t n = src ? a.bytes : 0;
        ok = ok && std::fwrite(&n, 8, 1, f.get()) == 1;
        if (!ok || n == 0) continue;
        host.resize(n);
        CU(cudaMemcpy(host.data(), src, n, cudaMemcpyDefault));
        ok = std::fwrite(host.data(), 1, n, f.get()) == n;
    }
    if (!ok) return fail(MVDR_ECUDA, std::string("write failed: ") + path);
    return MVDR_OK;
}

int mvdr_load_input_bundle(const char* path, mvdr_input_bundle** out) {
    if (!path || !out) return fail(MVDR_EINVAL, "null argument");
    std::unique_ptr<FILE, int (*)(FILE*)> f(std::fopen(path, "rb"), &std::fclose);
    if (!f) return fail(MVDR_EINVAL, std::string("cannot open ") + path);
    char magic[8];
    std::unique_ptr<mvdr_input_bundle> bd(new mvdr_input_bundle());
    if (std::fread(magic, 1, 8, f.get()) != 8 || std::memcmp(magic, kBundleMagic, 8) != 0)
        return fail(MVDR_EINVAL, std::string("not an input bundle: ") + path);
    if (std::fread(&bd->config, sizeof(mvdr_config), 1, f.get()) != 1 ||
        std::fread(&bd->inputs, sizeof(mvdr_inputs), 1, f.get()) != 1)
        return fail(MVDR_EINVAL, "truncated bundle header");
    if (bd->config.abi_version != MVDR_ABI_VERSION) return fail(MVDR_EINVAL, "bundle written by another ABI version");
    if (bd->inputs.num_views > MVDR_MAX_VIEWS) return fail(MVDR_EINVAL, "corrupt bundle: view count");
    std::vector<InputArray> arrays = input_arrays(bd->config, bd->inputs);
    bd->arrays.resize(arrays.size());
    for (size_t k = 0; k < arrays.size(); ++k) {
        uint64_t n = 0;
        if (std::fread(&n, 8, 1, f.get()) != 1) return fail(MVDR_EINVAL, "truncated bundle");
        set_ptr(arrays[k].field, nullptr);
        if (n == 0) continue;
        if (n != arrays[k].bytes) return fail(MVDR_EINVAL, "corrupt bundle: array size");
        bd->arrays[k].resize(n);
        if (std::fread(bd->arrays[k].data(), 1, n, f.get()) != n) return fail(MVDR_EINVAL, "truncated bundle");
        set_ptr(arrays[k].field, bd->arrays[k].data());
    }
    *out = bd.release();
    return MVDR_OK;
}

const mvdr_config* mvdr_input_bundle_config(const mvdr_input_bundle* b) { return b ? &b->config : nullptr; }
const mvdr_inputs* mvdr_input_bundle_inputs(const mvdr_input_bundle* b) { return b ? &b->inputs : nullptr; }
void mvdr_free_input_bundle(mvdr_input_bundle* b) { delete b; }

}  // extern "C"
