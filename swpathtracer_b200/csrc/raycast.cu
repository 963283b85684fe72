// raycast.cu -- batched ray queries and the three ray-cast integrators.
//
//   k_intersect   closest hit per ray (AccelStructure::intersect, accel_structure.h:29-30)
//   k_count       the reference's exhaustive traversal: tests / passes per ray
//   k_raycast     camera ray generation fused with the query and the pixel value of one
//                 ray-caster mode (integrators/raycaster.h:62-99 + normal_raycaster.cpp:19-31,
//                 depth_raycaster.cpp:36-48, int_test_count_raycaster.cpp:75-85)
#include <cstring>
#include <limits>

#include "spt_internal.h"
#include "traverse_wide.cuh"

namespace spt {
namespace {

constexpr int kBlock = 128;

// Ray i of a batch in either host layout: STRIDE 8 = {origin, pad, direction, pad} as two float4;
// STRIDE 6 = the reference's Ray (core/ray.h: two glm::vec3, 24 bytes) as three float2.  STREAM
// reads with the evict-first hint (rays are read once).
template <int STRIDE, bool STREAM>
__device__ __forceinline__ void load_ray(const float* __restrict__ rays, uint64_t i, V3& o, V3& d) {
    if (STRIDE == 8) {
        const float4* r = reinterpret_cast<const float4*>(rays) + 2 * i;
        const float4 a = STREAM ? __ldcs(r) : __ldg(r), b = STREAM ? __ldcs(r + 1) : __ldg(r + 1);
        o = f3v(a);
        d = f3v(b);
    } else {
        const float2* r = reinterpret_cast<const float2*>(rays) + 3 * i;
        const float2 a = STREAM ? __ldcs(r) : __ldg(r), b = STREAM ? __ldcs(r + 1) : __ldg(r + 1),
                     c = STREAM ? __ldcs(r + 2) : __ldg(r + 2);
        o = v3(a.x, a.y, b.x);
        d = v3(b.y, c.x, c.y);
    }
}

// Persistent variant: wide traversal, lanes refilled from a global ray counter (traverse_wide.cuh).
// 10 blocks of 128 per SM (at most 48 registers): 40 resident warps to hide the node-fetch latency.
// Rays are read and hits written once, with the evict-first (streaming) cache hint, so the ray and
// hit streams (48 B per ray, 768 MB per 2^24 rays) push less of the scene out of L2: +1 %.
template <int STRIDE>
__global__ void __launch_bounds__(kBlock, 10) k_intersect_df(DevScene S, const float* __restrict__ rays, uint64_t n,
                                                         spt_hit* __restrict__ hits, uint32_t* status,
                                                         unsigned long long* next) {
    persistent_trace(
        S, n, next, status, [&](uint64_t i, V3& o, V3& d) { load_ray<STRIDE, true>(rays, i, o, d); },
        [&](uint64_t i, const Hit1& h) {
            __stcs(reinterpret_cast<float4*>(hits + i),
                   make_float4(h.t, __uint_as_float(h.found ? slot_prim(S, h.slot) : SPT_MISS), h.u, h.v));
        });
}

// The same kernel over a batch in coherence order (ray_order.cu): the k-th ray it takes is order[k],
// for k below *count (the rays that meet the root box), and its hit goes to place k of hits_ordered,
// so that neighbouring lanes write neighbouring hits (scattered 16-byte stores cost partial-sector
// writes in DRAM).
template <int STRIDE>
__global__ void __launch_bounds__(kBlock, 10) k_intersect_df_ordered(DevScene S, const float* __restrict__ rays,
                                                                 const uint32_t* __restrict__ order,
                                                                 const uint32_t* __restrict__ count,
                                                                 spt_hit* __restrict__ hits_ordered, uint32_t* status,
                                                                 unsigned long long* next) {
    const uint64_t traced = __ldg(count);
    persistent_trace(
        S, traced, next, status, [&](uint64_t k, V3& o, V3& d) { load_ray<STRIDE, true>(rays, __ldg(order + k), o, d); },
        [&](uint64_t k, const Hit1& h) {
            __stcs(reinterpret_cast<float4*>(hits_ordered + k),
                   make_float4(h.t, __uint_as_float(h.found ? slot_prim(S, h.slot) : SPT_MISS), h.u, h.v));
        });
}

// The same kernel with its own work counted (node visits, primitive tests): the work behind the
// throughput of k_intersect_df, for comparison with the reference traversal's test counts.
__global__ void __launch_bounds__(kBlock, 10) k_intersect_df_counted(DevScene S, const float* __restrict__ rays,
                                                                 uint64_t n, spt_hit* __restrict__ hits,
                                                                 uint32_t* status, unsigned long long* next,
                                                                 unsigned long long* counts) {
    persistent_trace<true>(
        S, n, next, status, [&](uint64_t i, V3& o, V3& d) { load_ray<8, true>(rays, i, o, d); },
        [&](uint64_t i, const Hit1& h) {
            __stcs(reinterpret_cast<float4*>(hits + i),
                   make_float4(h.t, __uint_as_float(h.found ? slot_prim(S, h.slot) : SPT_MISS), h.u, h.v));
        },
        counts);
}

template <int TRAV, int STRIDE>
__global__ void __launch_bounds__(kBlock) k_intersect(DevScene S, const float* __restrict__ rays, uint64_t n,
                                                      spt_hit* __restrict__ hits, uint32_t* status) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    V3 ro, rd;
    load_ray<STRIDE, false>(rays, i, ro, rd);
    Hit1 h = trace_closest<TRAV>(S, ro, rd, status);
    spt_hit o;
    o.t = h.t;
    o.prim_id = h.found ? slot_prim(S, h.slot) : SPT_MISS;
    o.u = h.u;
    o.v = h.v;
    hits[i] = o;
}

template <int STRIDE>
__global__ void __launch_bounds__(kBlock) k_count(DevScene S, const float* __restrict__ rays, uint64_t n,
                                                  spt_hit* __restrict__ ref_hits, uint32_t* __restrict__ tests,
                                                  uint32_t* __restrict__ nhits, uint32_t* __restrict__ prim_tests,
                                                  uint32_t* status) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    V3 ro, rd;
    load_ray<STRIDE, false>(rays, i, ro, rd);
    CountOut c;
    Hit1 h = count_traverse<kStack>(S, ro, rd, c, status);
    if (ref_hits) {
        spt_hit o;
        o.t = h.t;
        o.prim_id = h.found ? slot_prim(S, h.slot) : SPT_MISS;
        o.u = h.u;
        o.v = h.v;
        ref_hits[i] = o;
    }
    if (tests) tests[i] = c.tests;
    if (nhits) nhits[i] = c.hits;
    if (prim_tests) prim_tests[i] = c.prim_tests;
}

// Per-image statistics of integrator.h:47-54, reduced per warp then once per warp to global.
struct StatAcc {
    unsigned long long sum_tests, sum_hits, min_tests, max_tests, min_hits, max_hits;
};

__device__ __forceinline__ void reduce_stats(StatAcc* g, bool valid, uint32_t tests, uint32_t hits) {
    unsigned long long st = valid ? tests : 0ull, sh = valid ? hits : 0ull;
    unsigned mnt = valid ? tests : 0xFFFFFFFFu, mxt = valid ? tests : 0u;
    unsigned mnh = valid ? hits : 0xFFFFFFFFu, mxh = valid ? hits : 0u;
    for (int o = 16; o > 0; o >>= 1) {
        st += __shfl_xor_sync(0xFFFFFFFFu, st, o);
        sh += __shfl_xor_sync(0xFFFFFFFFu, sh, o);
    }
    mnt = __reduce_min_sync(0xFFFFFFFFu, mnt);
    mxt = __reduce_max_sync(0xFFFFFFFFu, mxt);
    mnh = __reduce_min_sync(0xFFFFFFFFu, mnh);
    mxh = __reduce_max_sync(0xFFFFFFFFu, mxh);
    if ((threadIdx.x & 31) == 0 && mnt != 0xFFFFFFFFu) {
        atomicAdd(&g->sum_tests, st);
        atomicAdd(&g->sum_hits, sh);
        atomicMin(&g->min_tests, static_cast<unsigned long long>(mnt));
        atomicMax(&g->max_tests, static_cast<unsigned long long>(mxt));
        atomicMin(&g->min_hits, static_cast<unsigned long long>(mnh));
        atomicMax(&g->max_hits, static_cast<unsigned long long>(mxh));
    }
}

// 256 threads cover a 16x16 pixel tile; each warp an 8x4 sub-tile, so neighbouring lanes trace
// neighbouring pixels (coherent primary rays).
__device__ __forceinline__ void tile_pixel(uint32_t& x, uint32_t& y) {
    const uint32_t lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    x = blockIdx.x * 16 + (w & 1) * 8 + (lane & 7);
    y = blockIdx.y * 16 + (w >> 1) * 4 + (lane >> 3);
}

template <int MODE, int TRAV>
__global__ void __launch_bounds__(256) k_raycast(DevScene S, DevCamera cam, void* __restrict__ out,
                                                 StatAcc* stats, uint32_t* status) {
    uint32_t x, y;
    tile_pixel(x, y);
    const bool valid = x < cam.width && y < cam.height;
    uint32_t tests = 0, hits = 0;
    if (valid) {
        V3 o, d;
        camera_ray(cam, static_cast<float>(x) + 0.5f, static_cast<float>(y) + 0.5f, o, d);
        const uint64_t idx = static_cast<uint64_t>(y) * cam.width + x;
        if (MODE == SPT_RAYCAST_COUNT || stats) {
            CountOut c;
            Hit1 h = count_traverse<kStack>(S, o, d, c, status);
            tests = c.tests;
            hits = c.hits;
            if (MODE == SPT_RAYCAST_COUNT) {
                static_cast<long long*>(out)[idx] = static_cast<long long>(c.tests);
            } else if (MODE == SPT_RAYCAST_DEPTH) {
                static_cast<float*>(out)[idx] = h.found ? h.t : -1.0f;
            } else {
                V3 nrm = v3(0.0f, 0.0f, 0.0f);
                if (h.found) {
                    const uint32_t prim = slot_prim(S, h.slot);
                    nrm = hit_normal(S, prim, h.u, h.v, hit_pos(S.prim_type[prim] == SPT_PRIM_SPHERE, o, d, h.t));
                }
                float* q = static_cast<float*>(out) + 3 * idx;
                q[0] = nrm.x; q[1] = nrm.y; q[2] = nrm.z;
            }
        } else {
            Hit1 h = trace_closest<TRAV>(S, o, d, status);
            if (MODE == SPT_RAYCAST_DEPTH) {
                static_cast<float*>(out)[idx] = h.found ? h.t : -1.0f;
            } else {
                V3 nrm = v3(0.0f, 0.0f, 0.0f);
                if (h.found) {
                    const uint32_t prim = slot_prim(S, h.slot);
                    nrm = hit_normal(S, prim, h.u, h.v, hit_pos(S.prim_type[prim] == SPT_PRIM_SPHERE, o, d, h.t));
                }
                float* q = static_cast<float*>(out) + 3 * idx;
                q[0] = nrm.x; q[1] = nrm.y; q[2] = nrm.z;
            }
        }
    }
    if (stats) reduce_stats(stats, valid, tests, hits);
}

inline unsigned blocks_for(uint64_t n, int block) { return static_cast<unsigned>((n + block - 1) / block); }

}  // namespace

namespace {

// the persistent kernel's grid on the context's device (one computation per context and ray layout)
template <int STRIDE>
int df_grid(spt_context* ctx) {
    int& grid = ctx->df_grid[STRIDE == 6 ? 1 : 0];
    if (!grid) grid = persistent_grid(ctx, reinterpret_cast<const void*>(k_intersect_df<STRIDE>), kBlock);
    return grid;
}

// A caller's traced count held to the batch: *out = min(order[2n], n), so that an order made for
// another batch cannot take the traversal past this one's order entries and hit slots; and the
// persistent kernel's ray counter zeroed, in the same one-thread launch.
__global__ void k_order_count_clamp(const uint32_t* __restrict__ order, uint64_t n, uint32_t* __restrict__ out,
                                    unsigned long long* __restrict__ next) {
    const uint32_t c = order[2 * n];
    *out = c < n ? c : static_cast<uint32_t>(n);
    *next = 0ull;
}

// The persistent closest-hit launch (in the order `order` when it is not NULL, over the count at
// `count`, the hits then in that order; the ordered kernel has the plain one's registers and block,
// so the same grid).
template <int STRIDE>
spt_status launch_df(spt_context* ctx, const spt_scene* sc, const float* d_rays, uint64_t n, spt_hit* d_hits,
                     unsigned long long* next, cudaStream_t s, const uint32_t* order = nullptr,
                     const uint32_t* count = nullptr) {
    if (order)
        k_intersect_df_ordered<STRIDE>
            <<<df_grid<STRIDE>(ctx), kBlock, 0, s>>>(sc->dev, d_rays, order, count, d_hits, ctx->d_status, next);
    else
        k_intersect_df<STRIDE><<<df_grid<STRIDE>(ctx), kBlock, 0, s>>>(sc->dev, d_rays, n, d_hits, ctx->d_status, next);
    SPT_CUDA(ctx, cudaGetLastError());
    return SPT_OK;
}

template <int STRIDE>
spt_status launch_intersect_t(spt_context* ctx, const spt_scene* sc, const float* d_rays, uint64_t n, spt_hit* d_hits,
                              cudaStream_t s, bool order) {
    if (sc->dev.traversal == 2) {
        unsigned long long* next = nullptr;
        spt_status st = fetch_counter(ctx, s, &next);
        if (st != SPT_OK) return st;
        if (order && n >= order_min_rays() && n <= 0xFFFFFFFFull) {
            // this stream's buffers: the hits in the order first (16-byte aligned for the kernel's
            // float4 stores whatever n is), then the keys (n words), the order, its inverse and the
            // traced count (2n + 1), and the sort's counts
            const size_t work = order_scratch_bytes(ctx);
            void* mem = nullptr;
            if ((st = stream_scratch(ctx, s, (7 * n + 1) * sizeof(uint32_t) + work, &mem)) != SPT_OK) return st;
            if (mem) {
                spt_hit* ordered = static_cast<spt_hit*>(mem);
                uint32_t* keys = reinterpret_cast<uint32_t*>(ordered + n);
                uint32_t* ord = keys + n;
                uint32_t* w = keys + 3 * n + 1;
                if ((st = order_rays(ctx, sc, d_rays, n, STRIDE, s, keys, w, ord)) != SPT_OK) return st;
                if ((st = launch_df<STRIDE>(ctx, sc, d_rays, n, ordered, next, s, ord, ord + 2 * n)) != SPT_OK) return st;
                return unorder_hits(ctx, ordered, ord, n, d_hits, s);
            }
            // every per-stream buffer belongs to another stream: the batch's own order
        }
        return launch_df<STRIDE>(ctx, sc, d_rays, n, d_hits, next, s);
    } else if (sc->dev.traversal == 1) {
        k_intersect<1, STRIDE><<<blocks_for(n, kBlock), kBlock, 0, s>>>(sc->dev, d_rays, n, d_hits, ctx->d_status);
    } else {
        k_intersect<0, STRIDE><<<blocks_for(n, kBlock), kBlock, 0, s>>>(sc->dev, d_rays, n, d_hits, ctx->d_status);
    }
    SPT_CUDA(ctx, cudaGetLastError());
    return SPT_OK;
}

}  // namespace

spt_status launch_intersect(spt_context* ctx, const spt_scene* sc, const float* d_rays, uint64_t n, spt_hit* d_hits,
                            cudaStream_t s, int stride, bool order) {
    if (n == 0) return SPT_OK;
    if (n > (1ull << 36)) return fail(ctx, SPT_ERR_INVALID_ARGUMENT, "too many rays in one call");
    if (stride == 6) return launch_intersect_t<6>(ctx, sc, d_rays, n, d_hits, s, order);
    return launch_intersect_t<8>(ctx, sc, d_rays, n, d_hits, s, order);
}

// launch_intersect with the persistent kernel's ray counter supplied by the caller (zeroed on stream s
// before this launch) instead of taken from the context's ring, which is allocated on first use.
spt_status launch_intersect_fixed(spt_context* ctx, const spt_scene* sc, const float* d_rays, uint64_t n,
                                  spt_hit* d_hits, unsigned long long* next, cudaStream_t s) {
    if (n == 0) return SPT_OK;
    if (sc->dev.traversal != 2) return launch_intersect(ctx, sc, d_rays, n, d_hits, s);  // no counter needed
    return launch_df<8>(ctx, sc, d_rays, n, d_hits, next, s);
}

// k_intersect_df_counted over n rays (8 floats each); counts (device): node visits, primitive tests.
spt_status launch_intersect_counted(spt_context* ctx, const spt_scene* sc, const float* d_rays, uint64_t n,
                                   spt_hit* d_hits, unsigned long long* counts, cudaStream_t s) {
    if (n == 0) return SPT_OK;
    if (sc->dev.traversal != 2) return fail(ctx, SPT_ERR_UNSUPPORTED, "the scene has no 8-wide tree");
    unsigned long long* next = nullptr;
    spt_status st = fetch_counter(ctx, s, &next);
    if (st != SPT_OK) return st;
    static_assert(sizeof(unsigned long long) == 8, "");
    k_intersect_df_counted<<<df_grid<8>(ctx), kBlock, 0, s>>>(sc->dev, d_rays, n, d_hits, ctx->d_status, next, counts);
    SPT_CUDA(ctx, cudaGetLastError());
    return SPT_OK;
}

spt_status launch_count(spt_context* ctx, const spt_scene* sc, const float* d_rays, uint64_t n, spt_hit* d_ref_hits,
                        uint32_t* d_tests, uint32_t* d_hits, uint32_t* d_prim_tests, cudaStream_t s, int stride) {
    if (n == 0) return SPT_OK;
    if (n > (1ull << 36)) return fail(ctx, SPT_ERR_INVALID_ARGUMENT, "too many rays in one call");
    if (stride == 6)
        k_count<6><<<blocks_for(n, kBlock), kBlock, 0, s>>>(sc->dev, d_rays, n, d_ref_hits, d_tests, d_hits,
                                                            d_prim_tests, ctx->d_status);
    else
        k_count<8><<<blocks_for(n, kBlock), kBlock, 0, s>>>(sc->dev, d_rays, n, d_ref_hits, d_tests, d_hits,
                                                            d_prim_tests, ctx->d_status);
    SPT_CUDA(ctx, cudaGetLastError());
    return SPT_OK;
}

static spt_status launch_raycast(spt_context* ctx, const spt_scene* sc, const DevCamera& cam, int32_t mode, void* d_out,
                                 StatAcc* d_stats, cudaStream_t s) {
    dim3 grid((cam.width + 15) / 16, (cam.height + 15) / 16);
    const bool w = sc->dev.traversal >= 1;
    if (mode == SPT_RAYCAST_NORMAL) {
        if (w) k_raycast<SPT_RAYCAST_NORMAL, 1><<<grid, 256, 0, s>>>(sc->dev, cam, d_out, d_stats, ctx->d_status);
        else k_raycast<SPT_RAYCAST_NORMAL, 0><<<grid, 256, 0, s>>>(sc->dev, cam, d_out, d_stats, ctx->d_status);
    } else if (mode == SPT_RAYCAST_DEPTH) {
        if (w) k_raycast<SPT_RAYCAST_DEPTH, 1><<<grid, 256, 0, s>>>(sc->dev, cam, d_out, d_stats, ctx->d_status);
        else k_raycast<SPT_RAYCAST_DEPTH, 0><<<grid, 256, 0, s>>>(sc->dev, cam, d_out, d_stats, ctx->d_status);
    } else {
        k_raycast<SPT_RAYCAST_COUNT, 0><<<grid, 256, 0, s>>>(sc->dev, cam, d_out, d_stats, ctx->d_status);
    }
    SPT_CUDA(ctx, cudaGetLastError());
    return SPT_OK;
}

}  // namespace spt

namespace spt {
namespace {

constexpr uint64_t kPipeChunk = 1ull << 20;  // rays per pipeline chunk (32 MB in, 16 MB out)

bool is_pinned(const void* p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

// Host buffers in page-locked memory: the batch goes through in chunks over the context's pipeline
// streams, chunk c on stream c % kPipe, so the copy in of one chunk, the query of another and the
// copy out of a third run at the same time (PCIe is full duplex).  Each stream owns one set of
// device buffers; its chunks are in stream order, so a set is reused only after its last chunk's
// copy out.
spt_status intersect_pipelined(spt_context* ctx, const spt_scene* sc, const float* rays, uint64_t n, spt_hit* hits,
                               uint32_t* tests, uint32_t* nhits, int stride) {
    const int P = spt_context::kPipe;
    const uint64_t ray_bytes = 4ull * stride;
    const size_t set_bytes = kPipeChunk * (ray_bytes + sizeof(spt_hit) + 4 + 4);
    void* mem;
    spt_status st = scratch(ctx, 9, set_bytes * P, &mem);
    if (st != SPT_OK) return st;
    // the pipeline streams start after whatever the context's stream has queued
    SPT_CUDA(ctx, cudaEventRecord(ctx->ev_pipe[0], ctx->stream));
    for (int i = 0; i < P; ++i) SPT_CUDA(ctx, cudaStreamWaitEvent(ctx->pipe[i], ctx->ev_pipe[0], 0));
    const uint64_t chunks = (n + kPipeChunk - 1) / kPipeChunk;
    for (uint64_t c = 0; c < chunks; ++c) {
        const int i = static_cast<int>(c % P);
        cudaStream_t s = ctx->pipe[i];
        char* base = static_cast<char*>(mem) + set_bytes * i;
        float* d_rays = reinterpret_cast<float*>(base);
        spt_hit* d_hits = reinterpret_cast<spt_hit*>(base + kPipeChunk * ray_bytes);
        uint32_t* d_tests = reinterpret_cast<uint32_t*>(base + kPipeChunk * (ray_bytes + sizeof(spt_hit)));
        uint32_t* d_nh = d_tests + kPipeChunk;
        const uint64_t first = c * kPipeChunk, m = std::min(kPipeChunk, n - first);
        SPT_CUDA(ctx, cudaMemcpyAsync(d_rays, rays + static_cast<uint64_t>(stride) * first, m * ray_bytes,
                                      cudaMemcpyHostToDevice, s));
        if ((st = launch_intersect(ctx, sc, d_rays, m, d_hits, s, stride, true)) != SPT_OK) return st;
        if (tests || nhits)
            if ((st = launch_count(ctx, sc, d_rays, m, nullptr, tests ? d_tests : nullptr, nhits ? d_nh : nullptr,
                                   nullptr, s, stride)) != SPT_OK)
                return st;
        SPT_CUDA(ctx, cudaMemcpyAsync(hits + first, d_hits, m * sizeof(spt_hit), cudaMemcpyDeviceToHost, s));
        if (tests) SPT_CUDA(ctx, cudaMemcpyAsync(tests + first, d_tests, m * 4, cudaMemcpyDeviceToHost, s));
        if (nhits) SPT_CUDA(ctx, cudaMemcpyAsync(nhits + first, d_nh, m * 4, cudaMemcpyDeviceToHost, s));
    }
    // the context's stream continues after every chunk
    for (int i = 0; i < P; ++i) {
        SPT_CUDA(ctx, cudaEventRecord(ctx->ev_pipe[i], ctx->pipe[i]));
        SPT_CUDA(ctx, cudaStreamWaitEvent(ctx->stream, ctx->ev_pipe[i], 0));
    }
    return check_status(ctx);
}

// spt_intersect / spt_intersect_packed: stride floats per host ray.
spt_status intersect_host(spt_context* ctx, const spt_scene* sc, const float* rays, uint64_t n, spt_hit* hits,
                          uint32_t* tests, uint32_t* nhits, int stride) {
    if (!ctx || !sc || (n && (!rays || !hits))) return fail(ctx, SPT_ERR_INVALID_ARGUMENT, "NULL argument");
    if (n == 0) return SPT_OK;
    SPT_CUDA(ctx, cudaSetDevice(ctx->device));
    if (n > kPipeChunk && is_pinned(rays) && is_pinned(hits) && (!tests || is_pinned(tests)) &&
        (!nhits || is_pinned(nhits)))
        return intersect_pipelined(ctx, sc, rays, n, hits, tests, nhits, stride);
    spt_status st;
    void *d_rays, *d_hits, *d_tests = nullptr, *d_nh = nullptr;
    const uint64_t ray_bytes = 4ull * stride;
    if ((st = scratch(ctx, 0, n * ray_bytes, &d_rays)) != SPT_OK) return st;
    if ((st = scratch(ctx, 1, n * sizeof(spt_hit), &d_hits)) != SPT_OK) return st;
    if (tests && (st = scratch(ctx, 2, n * 4, &d_tests)) != SPT_OK) return st;
    if (nhits && (st = scratch(ctx, 3, n * 4, &d_nh)) != SPT_OK) return st;
    SPT_CUDA(ctx, cudaMemcpyAsync(d_rays, rays, n * ray_bytes, cudaMemcpyHostToDevice, ctx->stream));
    if ((st = launch_intersect(ctx, sc, static_cast<float*>(d_rays), n, static_cast<spt_hit*>(d_hits), ctx->stream,
                               stride, true)) != SPT_OK)
        return st;
    if (tests || nhits)
        if ((st = launch_count(ctx, sc, static_cast<float*>(d_rays), n, nullptr, static_cast<uint32_t*>(d_tests),
                               static_cast<uint32_t*>(d_nh), nullptr, ctx->stream, stride)) != SPT_OK)
            return st;
    SPT_CUDA(ctx, cudaMemcpyAsync(hits, d_hits, n * sizeof(spt_hit), cudaMemcpyDeviceToHost, ctx->stream));
    if (tests) SPT_CUDA(ctx, cudaMemcpyAsync(tests, d_tests, n * 4, cudaMemcpyDeviceToHost, ctx->stream));
    if (nhits) SPT_CUDA(ctx, cudaMemcpyAsync(nhits, d_nh, n * 4, cudaMemcpyDeviceToHost, ctx->stream));
    return check_status(ctx);
}

}  // namespace
}  // namespace spt

using namespace spt;

extern "C" {

spt_status spt_intersect(spt_context* ctx, const spt_scene* sc, const float* rays, uint64_t n, spt_hit* hits,
                         uint32_t* tests, uint32_t* nhits) {
    return intersect_host(ctx, sc, rays, n, hits, tests, nhits, 8);
}

spt_status spt_intersect_packed(spt_context* ctx, const spt_scene* sc, const float* rays, uint64_t n, spt_hit* hits,
                                uint32_t* tests, uint32_t* nhits) {
    return intersect_host(ctx, sc, rays, n, hits, tests, nhits, 6);
}

spt_status spt_intersect_device(spt_context* ctx, const spt_scene* sc, const float* d_rays, uint64_t n,
                                spt_hit* d_hits, void* stream) {
    if (!ctx || !sc || (n && (!d_rays || !d_hits))) return fail(ctx, SPT_ERR_INVALID_ARGUMENT, "NULL argument");
    return launch_intersect(ctx, sc, d_rays, n, d_hits, static_cast<cudaStream_t>(stream), 8, true);
}

spt_status spt_ray_order_device(spt_context* ctx, const spt_scene* sc, const float* d_rays, uint64_t n,
                                uint32_t* d_order, void* stream) {
    if (!ctx || !sc || (n && (!d_rays || !d_order))) return fail(ctx, SPT_ERR_INVALID_ARGUMENT, "NULL argument");
    if (n == 0) return SPT_OK;
    if (n > 0xFFFFFFFFull) return fail(ctx, SPT_ERR_INVALID_ARGUMENT, "a ray order holds fewer than 2^32 rays");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    void* mem = nullptr;
    spt_status st = stream_scratch(ctx, s, n * sizeof(uint32_t) + order_scratch_bytes(ctx), &mem);
    if (st != SPT_OK) return st;
    if (!mem) return fail(ctx, SPT_ERR_UNSUPPORTED, "ray order buffers are held by eight other streams");
    uint32_t* keys = static_cast<uint32_t*>(mem);
    return order_rays(ctx, sc, d_rays, n, 8, s, keys, keys + n, d_order);
}

spt_status spt_intersect_ordered_device(spt_context* ctx, const spt_scene* sc, const float* d_rays,
                                        const uint32_t* d_order, uint64_t n, spt_hit* d_hits_ordered, void* stream) {
    if (!ctx || !sc || (n && (!d_rays || !d_order || !d_hits_ordered)))
        return fail(ctx, SPT_ERR_INVALID_ARGUMENT, "NULL argument");
    if (n == 0) return SPT_OK;
    if (n > 0xFFFFFFFFull) return fail(ctx, SPT_ERR_INVALID_ARGUMENT, "a ray order holds fewer than 2^32 rays");
    if (sc->dev.traversal != 2) return fail(ctx, SPT_ERR_UNSUPPORTED, "ordered queries run on the 8-wide persistent traversal");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // two slots of the counter ring: the ray counter and the clamped count, both set by one kernel
    unsigned long long *next = nullptr, *count_slot = nullptr;
    spt_status st = ring_slot(ctx, &next);
    if (st != SPT_OK) return st;
    if ((st = ring_slot(ctx, &count_slot)) != SPT_OK) return st;
    uint32_t* count = reinterpret_cast<uint32_t*>(count_slot);
    k_order_count_clamp<<<1, 1, 0, s>>>(d_order, n, count, next);
    SPT_CUDA(ctx, cudaGetLastError());
    return launch_df<8>(ctx, sc, d_rays, n, d_hits_ordered, next, s, d_order, count);
}

spt_status spt_hits_unorder_device(spt_context* ctx, const uint32_t* d_order, uint64_t n, const spt_hit* d_hits_ordered,
                                   spt_hit* d_hits, void* stream) {
    if (!ctx || (n && (!d_order || !d_hits_ordered || !d_hits))) return fail(ctx, SPT_ERR_INVALID_ARGUMENT, "NULL argument");
    if (n == 0) return SPT_OK;
    if (n > 0xFFFFFFFFull) return fail(ctx, SPT_ERR_INVALID_ARGUMENT, "a ray order holds fewer than 2^32 rays");
    return unorder_hits(ctx, d_hits_ordered, d_order, n, d_hits, static_cast<cudaStream_t>(stream));
}

spt_status spt_traversal_work_device(spt_context* ctx, const spt_scene* sc, const float* d_rays, uint64_t n,
                                     spt_hit* d_hits, uint64_t* work) {
    if (!ctx || !sc || !work || (n && (!d_rays || !d_hits)))
        return fail(ctx, SPT_ERR_INVALID_ARGUMENT, "NULL argument");
    SPT_CUDA(ctx, cudaSetDevice(ctx->device));
    void* d_counts;
    spt_status st = scratch(ctx, 10, 2 * sizeof(unsigned long long), &d_counts);
    if (st != SPT_OK) return st;
    auto* c = static_cast<unsigned long long*>(d_counts);
    SPT_CUDA(ctx, cudaMemsetAsync(c, 0, 2 * sizeof(unsigned long long), ctx->stream));
    if ((st = launch_intersect_counted(ctx, sc, d_rays, n, d_hits, c, ctx->stream)) != SPT_OK) return st;
    unsigned long long h[2] = {0, 0};
    SPT_CUDA(ctx, cudaMemcpyAsync(h, c, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
    if ((st = check_status(ctx)) != SPT_OK) return st;   // synchronises the stream
    work[0] = h[0];
    work[1] = h[1];
    return SPT_OK;
}

spt_status spt_count_device(spt_context* ctx, const spt_scene* sc, const float* d_rays, uint64_t n,
                            spt_hit* d_ref_hits, uint32_t* d_tests, uint32_t* d_hits, uint32_t* d_prim_tests,
                            void* stream) {
    if (!ctx || !sc || (n && !d_rays)) return fail(ctx, SPT_ERR_INVALID_ARGUMENT, "NULL argument");
    return launch_count(ctx, sc, d_rays, n, d_ref_hits, d_tests, d_hits, d_prim_tests, static_cast<cudaStream_t>(stream));
}

spt_status spt_raycast_image(spt_context* ctx, const spt_scene* sc, const spt_camera* cam, int32_t mode,
                             void* out_host, spt_render_stats* stats) {
    if (!ctx || !sc || !out_host) return fail(ctx, SPT_ERR_INVALID_ARGUMENT, "NULL argument");
    if (mode < SPT_RAYCAST_NORMAL || mode > SPT_RAYCAST_COUNT) return fail(ctx, SPT_ERR_INVALID_ARGUMENT, "unknown mode");
    SPT_CUDA(ctx, cudaSetDevice(ctx->device));
    DevCamera dc;
    spt_status st = make_camera(ctx, cam, dc);
    if (st != SPT_OK) return st;
    const uint64_t npx = static_cast<uint64_t>(dc.width) * dc.height;
    const size_t elem = mode == SPT_RAYCAST_NORMAL ? 12 : (mode == SPT_RAYCAST_DEPTH ? 4 : 8);
    void *d_out, *d_stats = nullptr;
    if ((st = scratch(ctx, 0, npx * elem, &d_out)) != SPT_OK) return st;
    if (stats) {
        if ((st = scratch(ctx, 4, sizeof(StatAcc), &d_stats)) != SPT_OK) return st;
        StatAcc init{0, 0, std::numeric_limits<unsigned long long>::max(), 0,
                     std::numeric_limits<unsigned long long>::max(), 0};
        SPT_CUDA(ctx, cudaMemcpyAsync(d_stats, &init, sizeof(init), cudaMemcpyHostToDevice, ctx->stream));
    }
    SPT_CUDA(ctx, cudaEventRecord(ctx->ev0, ctx->stream));
    if ((st = launch_raycast(ctx, sc, dc, mode, d_out, static_cast<StatAcc*>(d_stats), ctx->stream)) != SPT_OK) return st;
    SPT_CUDA(ctx, cudaEventRecord(ctx->ev1, ctx->stream));
    SPT_CUDA(ctx, cudaMemcpyAsync(out_host, d_out, npx * elem, cudaMemcpyDeviceToHost, ctx->stream));
    StatAcc acc{};
    if (stats) SPT_CUDA(ctx, cudaMemcpyAsync(&acc, d_stats, sizeof(acc), cudaMemcpyDeviceToHost, ctx->stream));
    st = check_status(ctx);
    if (st != SPT_OK) return st;
    if (stats) {
        std::memset(stats, 0, sizeof(*stats));
        stats->int_tests = acc.sum_tests;
        stats->int_hits = acc.sum_hits;
        stats->min_tests_pp = acc.min_tests;
        stats->max_tests_pp = acc.max_tests;
        stats->min_hits_pp = acc.min_hits;
        stats->max_hits_pp = acc.max_hits;
        stats->paths = npx;
        stats->segments = npx;
        float ms = 0.0f;
        SPT_CUDA(ctx, cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
        stats->gpu_ms = ms;
    }
    return SPT_OK;
}

spt_status spt_raycast_image_device(spt_context* ctx, const spt_scene* sc, const spt_camera* cam, int32_t mode,
                                    void* d_out, void* stream) {
    if (!ctx || !sc || !d_out) return fail(ctx, SPT_ERR_INVALID_ARGUMENT, "NULL argument");
    if (mode < SPT_RAYCAST_NORMAL || mode > SPT_RAYCAST_COUNT) return fail(ctx, SPT_ERR_INVALID_ARGUMENT, "unknown mode");
    DevCamera dc;
    spt_status st = make_camera(ctx, cam, dc);
    if (st != SPT_OK) return st;
    return launch_raycast(ctx, sc, dc, mode, d_out, nullptr, static_cast<cudaStream_t>(stream));
}

}  // extern "C"
