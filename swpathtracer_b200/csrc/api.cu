// api.cu -- context, acceleration structure and scene entry points of the C-ABI (include/spt.h).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <thread>
#include <fstream>
#include <memory>
#include <new>

#include <cstdlib>

#include "spt_internal.h"
#include "wide_build.h"

namespace spt {

spt_status fail(spt_context* ctx, spt_status s, const std::string& msg) {
    if (ctx) ctx->err = msg;
    return s;
}

spt_status cuda_fail(spt_context* ctx, cudaError_t e, const char* what) {
    std::string m = std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
    return fail(ctx, e == cudaErrorMemoryAllocation ? SPT_ERR_OUT_OF_MEMORY : SPT_ERR_CUDA, m);
}

spt_status scratch(spt_context* ctx, int i, size_t bytes, void** out) {
    if (ctx->scratch_bytes[i] < bytes) {
        if (ctx->scratch[i]) SPT_CUDA(ctx, cudaFree(ctx->scratch[i]));
        ctx->scratch[i] = nullptr;
        ctx->scratch_bytes[i] = 0;
        size_t grow = bytes + bytes / 4;
        SPT_CUDA(ctx, cudaMalloc(&ctx->scratch[i], grow));
        ctx->scratch_bytes[i] = grow;
    }
    *out = ctx->scratch[i];
    return SPT_OK;
}

spt_status stream_scratch(spt_context* ctx, cudaStream_t s, size_t bytes, void** out) {
    *out = nullptr;
    int k = -1;
    for (int i = 0; i < spt_context::kStreamScratch && k < 0; ++i)
        if (ctx->sscratch[i] && ctx->sscratch_stream[i] == s) k = i;
    for (int i = 0; i < spt_context::kStreamScratch && k < 0; ++i)
        if (!ctx->sscratch[i]) k = i;
    if (k < 0) return SPT_OK;
    if (ctx->sscratch_bytes[k] < bytes) {
        // cudaFree waits for the device, so no work still reads the old buffer
        if (ctx->sscratch[k]) SPT_CUDA(ctx, cudaFree(ctx->sscratch[k]));
        ctx->sscratch[k] = nullptr;
        ctx->sscratch_bytes[k] = 0;
        SPT_CUDA(ctx, cudaMalloc(&ctx->sscratch[k], bytes));
        ctx->sscratch_bytes[k] = bytes;
    }
    ctx->sscratch_stream[k] = s;
    *out = ctx->sscratch[k];
    return SPT_OK;
}

spt_status pinned(spt_context* ctx, size_t bytes, void** out) {
    if (ctx->pinned_bytes < bytes) {
        if (ctx->pinned) SPT_CUDA(ctx, cudaFreeHost(ctx->pinned));
        ctx->pinned = nullptr;
        ctx->pinned_bytes = 0;
        SPT_CUDA(ctx, cudaMallocHost(&ctx->pinned, bytes));
        ctx->pinned_bytes = bytes;
    }
    *out = ctx->pinned;
    return SPT_OK;
}

spt_status ring_slot(spt_context* ctx, unsigned long long** out) {
    if (!ctx->d_fetch) SPT_CUDA(ctx, cudaMalloc(&ctx->d_fetch, kFetchRing * sizeof(unsigned long long)));
    *out = ctx->d_fetch + (ctx->fetch_slot++ % kFetchRing);
    return SPT_OK;
}

spt_status fetch_counter(spt_context* ctx, cudaStream_t s, unsigned long long** out) {
    unsigned long long* c = nullptr;
    spt_status st = ring_slot(ctx, &c);
    if (st != SPT_OK) return st;
    SPT_CUDA(ctx, cudaMemsetAsync(c, 0, sizeof(unsigned long long), s));
    *out = c;
    return SPT_OK;
}

int persistent_grid(spt_context* ctx, const void* kernel, int block) {
    int sms = 148, per_sm = 1;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, block, 0) != cudaSuccess || per_sm < 1) per_sm = 1;
    return sms * per_sm;
}

spt_status check_status(spt_context* ctx) {
    uint32_t st = 0;
    SPT_CUDA(ctx, cudaMemcpyAsync(&st, ctx->d_status, sizeof(st), cudaMemcpyDeviceToHost, ctx->stream));
    SPT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (!st) return SPT_OK;
    SPT_CUDA(ctx, cudaMemsetAsync(ctx->d_status, 0, sizeof(uint32_t), ctx->stream));
    if (st & 4u) return fail(ctx, SPT_ERR_TIMEOUT, "a bounded device loop ran out of iterations");
    if (st & 2u) return fail(ctx, SPT_ERR_OVERFLOW, "a device work queue overflowed");
    return fail(ctx, SPT_ERR_OVERFLOW, "a traversal stack overflowed");
}

spt_status make_camera(spt_context* ctx, const spt_camera* c, DevCamera& k) {
    if (!c) return fail(ctx, SPT_ERR_INVALID_ARGUMENT, "camera is NULL");
    if (c->width == 0 || c->height == 0) return fail(ctx, SPT_ERR_INVALID_ARGUMENT, "image width/height must be > 0");
    if (c->type != SPT_CAMERA_PINHOLE && c->type != SPT_CAMERA_ORTHOGRAPHIC)
        return fail(ctx, SPT_ERR_INVALID_ARGUMENT, "unknown camera type");
    if (static_cast<uint64_t>(c->vp_left) + c->vp_width > c->width ||
        static_cast<uint64_t>(c->vp_top) + c->vp_height > c->height)
        return fail(ctx, SPT_ERR_INVALID_ARGUMENT, "viewport exceeds the image");
    std::memset(&k, 0, sizeof(k));
    k.type = c->type;
    V3 pos = v3(c->position[0], c->position[1], c->position[2]);
    V3 look = v3(c->look_at[0], c->look_at[1], c->look_at[2]);
    V3 up = v3(c->up[0], c->up[1], c->up[2]);
    V3 dir = normalize(look - pos);          // camera.cpp:9
    V3 u = normalize(cross(up, -dir));       // camera.cpp:10
    V3 w = -dir;
    V3 v = cross(w, u);                      // onb.cpp:18-27
    const float l2w[9] = {u.x, u.y, u.z, v.x, v.y, v.z, w.x, w.y, w.z};
    std::memcpy(k.l2w, l2w, sizeof(l2w));
    k.pos[0] = pos.x; k.pos[1] = pos.y; k.pos[2] = pos.z;
    if (c->type == SPT_CAMERA_PINHOLE) {     // pinhole_camera.cpp:3-12
        float a = c->width * 0.5f;
        double b = c->height * 0.5;
        float ang = c->fov_deg * 0.5f * kPi / 180.0f;  // DEG_TO_RAD expands without parentheses
        float vpd = static_cast<float>(b / std::tan(static_cast<double>(ang)));
        k.luc[0] = -a; k.luc[1] = static_cast<float>(b); k.luc[2] = -vpd;
    } else {                                 // orthographic_camera.cpp:5-19
        float ww = c->max_x - c->min_x, wh = c->max_y - c->min_y;
        k.luc[0] = c->min_x; k.luc[1] = c->max_y; k.luc[2] = 0.0f;
        k.pdx = ww / c->width;
        k.pdy = wh / c->height;
        V3 od = mat_mul(k.l2w, v3(0.0f, 0.0f, -1.0f));
        k.odir[0] = od.x; k.odir[1] = od.y; k.odir[2] = od.z;
    }
    k.width = c->width;
    k.height = c->height;
    k.vp_top = c->vp_top;
    k.vp_left = c->vp_left;
    k.vp_width = c->vp_width;
    k.vp_height = c->vp_height;
    return SPT_OK;
}

namespace {

// f(begin, end) over [0, n) in chunks on the host's threads; for loops whose iterations write
// disjoint, preallocated outputs (the results do not depend on the split).
template <typename F>
void parallel_for(size_t n, F f) {
    const size_t max_t = std::max(1u, std::thread::hardware_concurrency());
    const size_t t = std::min(max_t, (n + 65535) / 65536);
    if (t <= 1) {
        f(size_t{0}, n);
        return;
    }
    std::vector<std::thread> pool;
    const size_t chunk = (n + t - 1) / t;
    for (size_t k = 0; k < t; ++k) {
        const size_t a = k * chunk, b = std::min(n, a + chunk);
        if (a < b) pool.emplace_back(f, a, b);
    }
    for (auto& th : pool) th.join();
}

inline float bits_f(uint32_t u) {
    float f;
    std::memcpy(&f, &u, sizeof(f));
    return f;
}

spt_status validate_desc(spt_context* ctx, const spt_scene_desc* d) {
    if (!d) return fail(ctx, SPT_ERR_INVALID_ARGUMENT, "scene description is NULL");
    if (d->n_prims && (!d->prim_type || !d->prim_data || !d->prim_material))
        return fail(ctx, SPT_ERR_INVALID_ARGUMENT, "primitive arrays are NULL");
    if (d->n_bsdfs && !d->bsdfs) return fail(ctx, SPT_ERR_INVALID_ARGUMENT, "bsdf array is NULL");
    if (d->n_layered && (!d->layered_offsets || !d->layered_bsdf_ids))
        return fail(ctx, SPT_ERR_INVALID_ARGUMENT, "layered bsdf arrays are NULL");
    if (d->n_materials && !d->materials) return fail(ctx, SPT_ERR_INVALID_ARGUMENT, "material array is NULL");
    for (uint32_t i = 0; i < d->n_bsdfs; ++i) {
        const spt_bsdf& b = d->bsdfs[i];
        if (b.type < SPT_BSDF_LAMBERTIAN || b.type > SPT_BSDF_COOK_TORRANCE)
            return fail(ctx, SPT_ERR_INVALID_ARGUMENT, "bsdf " + std::to_string(i) + " has an unknown type");
        if (b.sampler != SPT_SAMPLER_UNIFORM && b.sampler != SPT_SAMPLER_IMPORTANCE)
            return fail(ctx, SPT_ERR_INVALID_ARGUMENT, "bsdf " + std::to_string(i) + " has an unknown sampler");
    }
    for (uint32_t i = 0; i < d->n_layered; ++i) {
        if (d->layered_offsets[i] > d->layered_offsets[i + 1])
            return fail(ctx, SPT_ERR_INVALID_ARGUMENT, "layered_offsets must be non-decreasing");
        if (d->layered_offsets[i + 1] == d->layered_offsets[i])
            return fail(ctx, SPT_ERR_INVALID_ARGUMENT, "layered bsdf " + std::to_string(i) + " has no layer");
        for (uint32_t k = d->layered_offsets[i]; k < d->layered_offsets[i + 1]; ++k)
            if (d->layered_bsdf_ids[k] >= d->n_bsdfs)
                return fail(ctx, SPT_ERR_INVALID_ARGUMENT, "layered bsdf refers to a missing bsdf");
    }
    for (uint32_t i = 0; i < d->n_materials; ++i)
        if (d->materials[i].layered_bsdf >= d->n_layered)
            return fail(ctx, SPT_ERR_INVALID_ARGUMENT, "material refers to a missing layered bsdf");
    for (uint32_t i = 0; i < d->n_prims; ++i) {
        if (d->prim_type[i] > SPT_PRIM_SPHERE)
            return fail(ctx, SPT_ERR_INVALID_ARGUMENT, "primitive " + std::to_string(i) + " has an unknown type");
        if (d->prim_type[i] == SPT_PRIM_SMOOTH_TRIANGLE && !d->prim_normals)
            return fail(ctx, SPT_ERR_INVALID_ARGUMENT, "smooth triangles need prim_normals");
        if (d->prim_material[i] >= d->n_materials)
            return fail(ctx, SPT_ERR_INVALID_ARGUMENT, "primitive " + std::to_string(i) + " refers to a missing material");
    }
    if (d->accel < SPT_ACCEL_NONE || d->accel > SPT_ACCEL_SBVH_SAH)
        return fail(ctx, SPT_ERR_INVALID_ARGUMENT, "unknown acceleration structure type");
    return SPT_OK;
}

// Scene arrays placed in one device allocation at 256-byte aligned offsets, then copied in.
struct Upload {
    struct Entry {
        const void* src;
        size_t bytes, offset;
        const void** dst;
    };
    std::vector<Entry> entries;
    size_t total = 0;
    template <typename T>
    void add(const std::vector<T>& host, const T** dst) {
        *dst = nullptr;
        if (host.empty()) return;
        const size_t off = (total + 255) & ~static_cast<size_t>(255);
        entries.push_back(Entry{host.data(), host.size() * sizeof(T), off, reinterpret_cast<const void**>(dst)});
        total = off + host.size() * sizeof(T);
    }
    spt_status commit(spt_scene* sc) {
        if (total == 0) return SPT_OK;
        void* base = nullptr;
        SPT_CUDA(sc->ctx, cudaMalloc(&base, total));
        sc->allocations.push_back(base);
        sc->bytes += total;
        for (const Entry& e : entries) {
            char* p = static_cast<char*>(base) + e.offset;
            SPT_CUDA(sc->ctx, cudaMemcpy(p, e.src, e.bytes, cudaMemcpyHostToDevice));
            *e.dst = p;
        }
        return SPT_OK;
    }
};


}  // namespace
}  // namespace spt

using namespace spt;

extern "C" {

uint32_t spt_abi_version(void) { return SPT_ABI_VERSION; }

spt_status spt_create(int device, spt_context** out) {
    if (!out) return SPT_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    auto ctx = std::unique_ptr<spt_context>(new (std::nothrow) spt_context());
    if (!ctx) return SPT_ERR_OUT_OF_MEMORY;
    ctx->device = device;
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || device < 0 || device >= n) return SPT_ERR_CUDA;
    if (cudaSetDevice(device) != cudaSuccess) return SPT_ERR_CUDA;
    if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) return SPT_ERR_CUDA;
    for (int i = 0; i < spt_context::kPipe; ++i) {
        if (cudaStreamCreateWithFlags(&ctx->pipe[i], cudaStreamNonBlocking) != cudaSuccess) return SPT_ERR_CUDA;
        if (cudaEventCreateWithFlags(&ctx->ev_pipe[i], cudaEventDisableTiming) != cudaSuccess) return SPT_ERR_CUDA;
    }
    if (cudaEventCreate(&ctx->ev0) != cudaSuccess || cudaEventCreate(&ctx->ev1) != cudaSuccess) return SPT_ERR_CUDA;
    if (cudaMalloc(&ctx->d_status, sizeof(uint32_t)) != cudaSuccess) return SPT_ERR_OUT_OF_MEMORY;
    if (cudaMemset(ctx->d_status, 0, sizeof(uint32_t)) != cudaSuccess) return SPT_ERR_CUDA;
    *out = ctx.release();
    return SPT_OK;
}

spt_status spt_destroy(spt_context* ctx) {
    if (!ctx) return SPT_ERR_INVALID_ARGUMENT;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    for (int i = 0; i < spt_context::kScratchSlots; ++i)
        if (ctx->scratch[i]) cudaFree(ctx->scratch[i]);
    for (int i = 0; i < spt_context::kStreamScratch; ++i)
        if (ctx->sscratch[i]) cudaFree(ctx->sscratch[i]);
    if (ctx->pinned) cudaFreeHost(ctx->pinned);
    if (ctx->d_status) cudaFree(ctx->d_status);
    if (ctx->d_fetch) cudaFree(ctx->d_fetch);
    if (ctx->ev0) cudaEventDestroy(ctx->ev0);
    if (ctx->ev1) cudaEventDestroy(ctx->ev1);
    for (int i = 0; i < spt_context::kPipe; ++i) {
        if (ctx->pipe[i]) {
            cudaStreamSynchronize(ctx->pipe[i]);
            cudaStreamDestroy(ctx->pipe[i]);
        }
        if (ctx->ev_pipe[i]) cudaEventDestroy(ctx->ev_pipe[i]);
    }
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return SPT_OK;
}

const char* spt_last_error(const spt_context* ctx) { return ctx ? ctx->err.c_str() : "context is NULL"; }

spt_status spt_bvh_build(const spt_scene_desc* desc, int n_threads, spt_bvh** out) {
    if (!out) return SPT_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    spt_status s = validate_desc(nullptr, desc);
    if (s != SPT_OK) return s;
    auto b = std::unique_ptr<spt_bvh>(new (std::nothrow) spt_bvh());
    if (!b) return SPT_ERR_OUT_OF_MEMORY;
    const char* err = nullptr;
    try {
        if (!build_sah_tree(*desc, n_threads, b->tree, &err)) return SPT_ERR_UNSUPPORTED;
    } catch (const std::bad_alloc&) {
        return SPT_ERR_OUT_OF_MEMORY;
    }
    *out = b.release();
    return SPT_OK;
}

spt_status spt_bvh_build_device(spt_context* ctx, const spt_scene_desc* desc, spt_bvh** out) {
    if (!ctx || !out) return fail(ctx, SPT_ERR_INVALID_ARGUMENT, "NULL argument");
    *out = nullptr;
    spt_status s = validate_desc(ctx, desc);
    if (s != SPT_OK) return s;
    SPT_CUDA(ctx, cudaSetDevice(ctx->device));
    auto b = std::unique_ptr<spt_bvh>(new (std::nothrow) spt_bvh());
    if (!b) return fail(ctx, SPT_ERR_OUT_OF_MEMORY, "host memory");
    try {
        s = build_ploc_tree(ctx, *desc, b->tree);
    } catch (const std::bad_alloc&) {
        return fail(ctx, SPT_ERR_OUT_OF_MEMORY, "host memory for the device BVH build");
    }
    if (s != SPT_OK) return s;
    *out = b.release();
    return SPT_OK;
}

spt_status spt_bvh_stats_get(const spt_bvh* bvh, spt_bvh_stats* out) {
    if (!bvh || !out) return SPT_ERR_INVALID_ARGUMENT;
    *out = bvh->tree.stats;
    return SPT_OK;
}

spt_status spt_bvh_export(const spt_bvh* bvh, spt_bvh2_node* nodes, uint64_t* n_nodes, uint32_t* ref_prim,
                          uint64_t* n_refs) {
    if (!bvh || !n_nodes || !n_refs) return SPT_ERR_INVALID_ARGUMENT;
    *n_nodes = bvh->tree.nodes.size();
    *n_refs = bvh->tree.refs.size();
    if (nodes) std::memcpy(nodes, bvh->tree.nodes.data(), bvh->tree.nodes.size() * sizeof(spt_bvh2_node));
    if (ref_prim) std::memcpy(ref_prim, bvh->tree.refs.data(), bvh->tree.refs.size() * sizeof(uint32_t));
    return SPT_OK;
}

spt_status spt_bvh_free(spt_bvh* bvh) {
    delete bvh;
    return SPT_OK;
}

spt_status spt_scene_create(spt_context* ctx, const spt_scene_desc* d, const spt_bvh* bvh, spt_scene** out) {
    if (!ctx || !out) return SPT_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    spt_status s = validate_desc(ctx, d);
    if (s != SPT_OK) return s;
    SPT_CUDA(ctx, cudaSetDevice(ctx->device));
    try {
        const uint32_t n = d->n_prims;
        HostBvh local;
        const HostBvh* tree = nullptr;
        const bool no_accel = d->accel == SPT_ACCEL_NONE;
        if (!no_accel && n) {
            if (bvh) {
                tree = &bvh->tree;
                if (tree->refs.size() != n) return fail(ctx, SPT_ERR_INVALID_ARGUMENT, "tree was built for another scene");
            } else {
                const char* err = "";
                if (!build_sah_tree(*d, 0, local, &err)) return fail(ctx, SPT_ERR_UNSUPPORTED, err);
                tree = &local;
            }
            if (tree->stats.tree_height + 2 > static_cast<uint64_t>(kStack))
                return fail(ctx, SPT_ERR_UNSUPPORTED,
                            "tree height " + std::to_string(tree->stats.tree_height) + " exceeds the traversal stack");
        }
        auto sc = std::unique_ptr<spt_scene>(new spt_scene());
        sc->ctx = ctx;
        DevScene& S = sc->dev;
        S.n_prims = n;
        S.empty = n == 0;
        S.no_accel = no_accel;
        for (int k = 0; k < 3; ++k) S.bg[k] = d->background[k];
        // slot order: leaf order of the tree, or input order without one
        std::vector<uint32_t> slot_prim(n);
        for (uint32_t i = 0; i < n; ++i) slot_prim[i] = tree ? tree->refs[i] : i;
        std::vector<float4> tri(3ull * n);
        std::vector<float4> face(n);
        std::vector<float4> smooth;
        bool any_smooth = false, any_sphere = false;
        for (uint32_t i = 0; i < n; ++i) {
            any_smooth |= d->prim_type[i] == SPT_PRIM_SMOOTH_TRIANGLE;
            any_sphere |= d->prim_type[i] == SPT_PRIM_SPHERE;
        }
        if (any_smooth) smooth.resize(3ull * n);
        parallel_for(n, [&](size_t a, size_t b) {
            for (size_t i = a; i < b; ++i) {
                const float* p = d->prim_data + 9ull * i;
                if (d->prim_type[i] == SPT_PRIM_SPHERE) {
                    face[i] = make_float4(p[0], p[1], p[2], p[3]);
                } else {
                    V3 v0 = v3(p[0], p[1], p[2]), v1 = v3(p[3], p[4], p[5]), v2 = v3(p[6], p[7], p[8]);
                    V3 nn = normalize(cross(v1 - v0, v2 - v0));  // triangle.cpp:6
                    face[i] = make_float4(nn.x, nn.y, nn.z, 0.0f);
                    if (d->prim_type[i] == SPT_PRIM_SMOOTH_TRIANGLE) {
                        const float* q = d->prim_normals + 9ull * i;
                        for (int k = 0; k < 3; ++k)
                            smooth[3ull * i + k] = make_float4(q[3 * k], q[3 * k + 1], q[3 * k + 2], 0.0f);
                    }
                }
            }
        });
        // leaf ordinals for the slots (filled below)
        std::vector<uint32_t> slot_leaf(n, 0);
        std::vector<float4> pair;
        std::vector<int2> leaf;
        std::vector<float> leaf_box;
        std::vector<spt_bvh2_node> node2;
        if (tree) {
            const auto& nodes = tree->nodes;
            const size_t nn = nodes.size();
            std::vector<int> ord(nn);
            uint32_t n_inner = 0, n_leaf = 0;
            for (size_t i = 0; i < nn; ++i) ord[i] = nodes[i].count ? ~static_cast<int>(n_leaf++) : static_cast<int>(n_inner++);
            pair.resize(4ull * n_inner);
            leaf.resize(n_leaf);
            leaf_box.resize(6ull * n_leaf);
            parallel_for(nn, [&](size_t a, size_t b) {   // leaves cover disjoint slot ranges
                for (size_t i = a; i < b; ++i) {
                    const spt_bvh2_node& nd = nodes[i];
                    if (nd.count) {
                        int l = ~ord[i];
                        leaf[l] = make_int2(static_cast<int>(nd.right), static_cast<int>(nd.count));
                        for (int k = 0; k < 3; ++k) {
                            leaf_box[6ull * l + k] = nd.min[k];
                            leaf_box[6ull * l + 3 + k] = nd.max[k];
                        }
                        for (uint32_t k = 0; k < nd.count; ++k) slot_leaf[nd.right + k] = static_cast<uint32_t>(l);
                    } else {
                        const spt_bvh2_node& L = nodes[i + 1];
                        const spt_bvh2_node& R = nodes[nd.right];
                        float4* p = &pair[4ull * ord[i]];
                        p[0] = make_float4(L.min[0], L.min[1], L.min[2], L.max[0]);
                        p[1] = make_float4(L.max[1], L.max[2], R.min[0], R.min[1]);
                        p[2] = make_float4(R.min[2], R.max[0], R.max[1], R.max[2]);
                        int4 refs = make_int4(ord[i + 1], ord[nd.right], 0, 0);
                        std::memcpy(&p[3], &refs, sizeof(refs));
                    }
                }
            });
            node2 = nodes;
            S.n_inner = n_inner;
            S.n_leaves = n_leaf;
            S.n_nodes2 = static_cast<uint32_t>(nn);
            S.root_is_leaf = nodes[0].count ? 1 : 0;
            for (int k = 0; k < 3; ++k) {
                S.root_min[k] = nodes[0].min[k];
                S.root_max[k] = nodes[0].max[k];
            }
            sc->tree_height = static_cast<uint32_t>(tree->stats.tree_height);
        } else {
            S.root_is_leaf = 1;
            leaf.push_back(make_int2(0, static_cast<int>(n)));
            leaf_box.assign(6, 0.0f);
            S.n_leaves = 1;
        }
        parallel_for(n, [&](size_t a, size_t b) {
            for (size_t s2 = a; s2 < b; ++s2) {
                const uint32_t i = slot_prim[s2];
                const float* p = d->prim_data + 9ull * i;
                float4* r = &tri[3ull * s2];
                if (d->prim_type[i] == SPT_PRIM_SPHERE) {
                    r[0] = make_float4(p[0], p[1], p[2], bits_f(i));
                    r[1] = make_float4(p[3], 0.0f, 0.0f, bits_f(slot_leaf[s2]));
                    r[2] = make_float4(0.0f, 0.0f, 0.0f, bits_f(SPT_PRIM_SPHERE));
                } else {
                    r[0] = make_float4(p[0], p[1], p[2], bits_f(i));
                    r[1] = make_float4(p[3] - p[0], p[4] - p[1], p[5] - p[2], bits_f(slot_leaf[s2]));
                    r[2] = make_float4(p[6] - p[0], p[7] - p[1], p[8] - p[2], bits_f(d->prim_type[i]));
                }
            }
        });
        // 8-wide quantized tree over the same leaves (traverse_wide.cuh)
        std::vector<WideNode> wnodes;
        std::vector<float4> wtri;
        if (tree) {
            WideBvh wb;
            build_wide(tree->nodes, wb);
            wnodes.swap(wb.nodes);
            // levels of the wide tree (breadth-first order: a node's inner children follow it), and
            // from them the most traversal stack entries a ray can need, 2 (levels - 1)
            std::vector<uint8_t> level(wnodes.size(), 1);
            uint32_t levels = wnodes.empty() ? 0 : 1;
            for (size_t k = 0; k < wnodes.size(); ++k) {
                const uint32_t nc = static_cast<uint32_t>(__builtin_popcount(wnodes[k].imask));
                for (uint32_t c = 0; c < nc; ++c) {
                    const size_t ch = static_cast<size_t>(wnodes[k].child_base) + c;
                    if (ch <= k || ch >= wnodes.size())
                        return fail(ctx, SPT_ERR_INTERNAL, "8-wide tree is not in breadth-first order");
                    level[ch] = static_cast<uint8_t>(std::min(255, level[k] + 1));
                    levels = std::max<uint32_t>(levels, level[ch]);
                }
            }
            sc->wide_stack_bound = levels > 1 ? 2 * (levels - 1) : 0;
            wtri.resize(3ull * wb.tri_rank.size());
            parallel_for(wb.tri_rank.size(), [&](size_t a, size_t b) {
                for (size_t k = a; k < b; ++k) {
                    const uint32_t rk = wb.tri_rank[k];
                    const float4* r = &tri[3ull * rk];
                    const uint32_t type = d->prim_type[slot_prim[rk]];
                    if (type == SPT_PRIM_SPHERE) {
                        wtri[3 * k] = make_float4(r[0].x, r[0].y, r[0].z, bits_f(rk));
                        wtri[3 * k + 1] = make_float4(0.0f, 0.0f, 0.0f, bits_f(type));
                        wtri[3 * k + 2] = make_float4(r[1].x, 0.0f, 0.0f, r[1].w);
                    } else {
                        wtri[3 * k] = make_float4(r[0].x, r[0].y, r[0].z, bits_f(rk));
                        wtri[3 * k + 1] = make_float4(r[1].x, r[1].y, r[1].z, bits_f(type));
                        wtri[3 * k + 2] = make_float4(r[2].x, r[2].y, r[2].z, r[1].w);  // leaf id
                    }
                }
            });
            const char* env = std::getenv("SPT_TRAVERSAL");
            S.traversal = 2;  // wide nodes, persistent dynamic fetch where a kernel supports it
            if (env && std::string(env) == "binary") S.traversal = 0;
            if (env && std::string(env) == "wide") S.traversal = 1;
        }
        // materials
        std::vector<DevBsdf> bs(d->n_bsdfs);
        for (uint32_t i = 0; i < d->n_bsdfs; ++i) {
            const spt_bsdf& b = d->bsdfs[i];
            DevBsdf& o = bs[i];
            std::memset(&o, 0, sizeof(o));
            o.type = b.type;
            o.sampler = b.sampler;
            o.r = b.rgb[0]; o.g = b.rgb[1]; o.b = b.rgb[2];
            o.scalar = b.scalar;
            o.br = b.rgb[0] / kPi; o.bg = b.rgb[1] / kPi; o.bb = b.rgb[2] / kPi;  // lambertian.cpp:6
        }
        std::vector<DevMaterial> ms(d->n_materials);
        std::vector<int> layers;
        bool any_em = false;
        for (uint32_t i = 0; i < d->n_materials; ++i) {
            const spt_material& m = d->materials[i];
            DevMaterial& o = ms[i];
            std::memset(&o, 0, sizeof(o));
            o.layer_begin = static_cast<int>(layers.size());
            for (uint32_t k = d->layered_offsets[m.layered_bsdf]; k < d->layered_offsets[m.layered_bsdf + 1]; ++k)
                layers.push_back(static_cast<int>(d->layered_bsdf_ids[k]));
            o.layer_count = static_cast<int>(layers.size()) - o.layer_begin;
            o.er = m.emission[0]; o.eg = m.emission[1]; o.eb = m.emission[2];
            sc->any_layered |= o.layer_count > 1;
            any_em |= (m.emission[0] != 0.0f || m.emission[1] != 0.0f || m.emission[2] != 0.0f);
        }
        std::vector<uint32_t> pm(d->prim_material, d->prim_material + n);
        std::vector<uint8_t> pt(d->prim_type, d->prim_type + n);
        S.has_spheres = any_sphere;
        sc->n_materials = d->n_materials;
        sc->any_emission = any_em;
        std::vector<uint4> raw(wnodes.size() * 5);
        if (!wnodes.empty()) std::memcpy(raw.data(), wnodes.data(), wnodes.size() * sizeof(WideNode));
        const uint4* wn = nullptr;
        // every array in one device allocation (one cudaMalloc per scene instead of fourteen)
        Upload up;
        up.add(tri, &S.tri);
        up.add(pair, &S.pair);
        up.add(leaf, &S.leaf);
        up.add(leaf_box, &S.leaf_box);
        up.add(node2, &S.node2);
        up.add(face, &S.face_normal);
        up.add(smooth, &S.smooth_normal);
        up.add(pm, &S.prim_mat);
        up.add(pt, &S.prim_type);
        up.add(bs, &S.bsdf);
        up.add(ms, &S.mat);
        up.add(layers, &S.layer_ids);
        up.add(raw, &wn);
        up.add(wtri, &S.wtri);
        if ((s = up.commit(sc.get())) != SPT_OK) return s;
        S.wnode = wn;
        S.n_wnodes = static_cast<uint32_t>(wnodes.size());
        *out = sc.release();
        return SPT_OK;
    } catch (const std::bad_alloc&) {
        return fail(ctx, SPT_ERR_OUT_OF_MEMORY, "host allocation failed while preparing the scene");
    }
}

spt_status spt_scene_destroy(spt_scene* sc) {
    if (!sc) return SPT_ERR_INVALID_ARGUMENT;
    cudaSetDevice(sc->ctx->device);
    cudaStreamSynchronize(sc->ctx->stream);
    for (void* p : sc->allocations) cudaFree(p);
    delete sc;
    return SPT_OK;
}

uint64_t spt_scene_device_bytes(const spt_scene* sc) { return sc ? sc->bytes : 0; }

// ImageBuffer::convertTosRGB + saveToFile (core/image_buffer.cpp:22-47); rgb is row-major [y][x].
spt_status spt_write_ppm(const char* path, const float* rgb, uint32_t width, uint32_t height, int32_t to_srgb) {
    if (!path || !rgb) return SPT_ERR_INVALID_ARGUMENT;
    std::ofstream f(path);
    if (!f) return SPT_ERR_INVALID_ARGUMENT;
    auto clampf = [](float x) { return std::min(std::max(x, 0.0f), 1.0f); };
    f << "P3" << std::endl << width << " " << height << std::endl << 255 << std::endl;
    for (uint32_t y = 0; y < height; ++y)
        for (uint32_t x = 0; x < width; ++x)
            for (int k = 0; k < 3; ++k) {
                float c = rgb[(static_cast<uint64_t>(y) * width + x) * 3 + k];
                // the reference's unqualified pow resolves to the double version
                if (to_srgb) c = static_cast<float>(std::pow(static_cast<double>(clampf(c)), static_cast<double>(1.0f / 2.2f)));
                f << static_cast<int>(clampf(c) * 255.0f + 0.5f) << " ";
            }
    return f ? SPT_OK : SPT_ERR_INTERNAL;
}

}  // extern "C"
