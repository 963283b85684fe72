// pathtrace.cu -- the path tracer (integrators/pathtracer.cpp:12-147) as a wavefront.
//
// A fixed pool of path slots (SoA, ping-pong) is refilled with new camera paths as old ones end:
//
//   k_generate  camera rays for free slots (pixel sampler + camera, pathtracer.cpp:104-113)
//   k_extend    closest hit for every live slot (traverse.cuh; the same kernel code as the ray casters)
//   k_shade     emission, layered BSDF walk, russian roulette and the next ray
//               (pathtracer.cpp:21-54); surviving paths are appended, warp-aggregated, to the other
//               buffer; finished paths add their radiance to the image
//   k_advance   one thread: moves the counters to the next iteration
//
// Random numbers: Philox-4x32-10 keyed by the seed, counter (path index, stream, block), stream 0
// for the pixel sample and stream depth+1 for the BSDF walk and roulette at that depth.  The path
// index is (spp_offset + sample) * viewport_pixels + viewport_pixel, so an image does not depend
// on slot assignment or scheduling (up to the order of the float atomic adds into the image).
#include <algorithm>
#include <cstring>

#include "shade.cuh"
#include "spt_internal.h"
#include "traverse.cuh"

namespace spt {
namespace {

struct PtConst {
    DevScene S;
    DevCamera cam;
    uint64_t seed;
    uint64_t total;        // camera paths to trace
    uint32_t spp, nsub;    // samples per pixel (after the square rounding), strata per axis
    float sw;              // stratum width
    int sampler, rr, path_length, cap;
    uint32_t npix;         // viewport pixels
    uint32_t spp_offset;
    uint32_t capacity;     // path slots
    float* image;          // W*H*3 radiance sums
};

struct PathBuf {
    float4* o;   // origin, pixel (viewport index) bits
    float4* d;   // direction, sample index bits
    float4* b;   // throughput, depth bits
    float4* l;   // radiance so far
};

struct Counters {
    unsigned long long next_path;   // camera paths generated so far
    unsigned long long segments;    // rays traced so far
    uint32_t n_alive;               // live slots at the start of the iteration (in the current buffer)
    uint32_t n_next;                // slots appended to the other buffer by k_shade
    uint32_t iterations;
    uint32_t pad;
};

__device__ __forceinline__ uint32_t n_new_paths(const PtConst& C, const Counters& c) {
    const unsigned long long rem = C.total - c.next_path;
    const uint32_t room = C.capacity - c.n_alive;
    return rem < room ? static_cast<uint32_t>(rem) : room;
}

__global__ void __launch_bounds__(256) k_generate(PtConst C, const Counters* __restrict__ ctr, PathBuf cur) {
    const Counters c = *ctr;
    const uint32_t n_new = n_new_paths(C, c);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n_new; i += gridDim.x * blockDim.x) {
        const unsigned long long g = c.next_path + i;
        const uint32_t si = static_cast<uint32_t>(g / C.npix);
        const uint32_t pix = static_cast<uint32_t>(g - static_cast<unsigned long long>(si) * C.npix);
        const uint32_t xx = pix % C.cam.vp_width, yy = pix / C.cam.vp_width;
        const uint32_t x = C.cam.vp_left + xx, y = C.cam.vp_top + yy;
        const uint32_t sg = C.spp_offset + si;
        const unsigned long long path = static_cast<unsigned long long>(sg) * C.npix + pix;
        float sx, sy;
        if (C.sampler == SPT_PIXEL_UNIFORM) {  // uniform_pixel_sampler.cpp:7-10
            Stream cs(C.seed, path, 0);
            sx = cs.next();
            sy = cs.next();
        } else {
            const uint32_t a = si / C.nsub, b = si % C.nsub;
            if (C.sampler == SPT_PIXEL_REGULAR) {  // regular_pixel_sampler.cpp:10-13
                float off = C.sw * 0.5f;
                sx = C.sw * a + off;
                sy = C.sw * b + off;
            } else {  // jittered_pixel_sampler.cpp:11-20
                Stream cs(C.seed, path, 0);
                float u0 = cs.next(), u1 = cs.next();
                sx = C.sw * a + C.sw * u0;
                sy = C.sw * b + C.sw * u1;
            }
        }
        V3 o, d;
        camera_ray(C.cam, static_cast<float>(x) + sx, static_cast<float>(y) + sy, o, d);
        const uint32_t slot = c.n_alive + i;
        cur.o[slot] = make_float4(o.x, o.y, o.z, __uint_as_float(pix));
        cur.d[slot] = make_float4(d.x, d.y, d.z, __uint_as_float(sg));
        cur.b[slot] = make_float4(1.0f, 1.0f, 1.0f, __int_as_float(0));
        cur.l[slot] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    }
}

__global__ void __launch_bounds__(128) k_extend(PtConst C, const Counters* __restrict__ ctr, PathBuf cur,
                                                float4* __restrict__ hits, uint32_t* status) {
    const Counters c = *ctr;
    const uint32_t n = c.n_alive + n_new_paths(C, c);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 o = cur.o[i], d = cur.d[i];
        Hit1 h = closest_hit<kStack>(C.S, f3v(o), f3v(d), status);
        hits[i] = make_float4(h.t, __uint_as_float(h.found ? slot_prim(C.S, h.slot) : SPT_MISS), h.u, h.v);
    }
}

__device__ __forceinline__ void splat(const PtConst& C, uint32_t pix, V3 L) {
    const uint32_t x = C.cam.vp_left + pix % C.cam.vp_width, y = C.cam.vp_top + pix / C.cam.vp_width;
    float* p = C.image + 3ull * (static_cast<uint64_t>(y) * C.cam.width + x);
    if (L.x != 0.0f) atomicAdd(p, L.x);
    if (L.y != 0.0f) atomicAdd(p + 1, L.y);
    if (L.z != 0.0f) atomicAdd(p + 2, L.z);
}

__global__ void __launch_bounds__(128) k_shade(PtConst C, Counters* __restrict__ ctr, PathBuf cur, PathBuf nxt,
                                               const float4* __restrict__ hits) {
    const Counters c = *ctr;
    const uint32_t n = c.n_alive + n_new_paths(C, c);
    const uint32_t lane = threadIdx.x & 31;
    // all lanes of a warp iterate together so the append below can be warp-aggregated
    for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
        const uint32_t i = base + threadIdx.x;
        bool keep = false;
        float4 wo_o, wo_d, wo_b, wo_l;
        if (i < n) {
            const float4 o4 = cur.o[i], d4 = cur.d[i], b4 = cur.b[i], l4 = cur.l[i], h4 = hits[i];
            const uint32_t pix = __float_as_uint(o4.w), sg = __float_as_uint(d4.w);
            const int depth = __float_as_int(b4.w);
            const uint64_t path = static_cast<uint64_t>(sg) * C.npix + pix;
            const V3 o = f3v(o4), d = f3v(d4);
            V3 beta = f3v(b4), L = f3v(l4);
            const uint32_t prim = __float_as_uint(h4.y);
            bool done = false;
            if (prim == SPT_MISS) {  // pathtracer.cpp:21-26
                if (depth == 0) L = L + beta * v3(C.S.bg[0], C.S.bg[1], C.S.bg[2]);
                done = true;
            } else {
                const float t = h4.x;
                const bool sphere = C.S.prim_type[prim] == SPT_PRIM_SPHERE;
                const V3 pos = hit_pos(sphere, o, d, t);
                const V3 nrm = hit_normal(C.S, prim, h4.z, h4.w, pos);
                const DevMaterial m = C.S.mat[C.S.prim_mat[prim]];
                float frame[9];
                onb_from_normal(nrm, frame);                       // pathtracer.cpp:28-30
                const V3 wo = normalize(mat_tmul(frame, -d));
                Stream bs(C.seed, path, static_cast<uint32_t>(depth) + 1u);
                LayerEval e = eval_layered(C.S, m, wo, bs);
                const V3 wwi = mat_mul(frame, e.wi);               // pathtracer.cpp:37-38
                const V3 no = pos + wwi * 1e-3f;
                L = L + beta * v3(m.er, m.eg, m.eb);
                const float k = fmaxf(fmaxf(e.refl.x, e.refl.y), e.refl.z);
                if (C.rr && depth >= C.path_length) {              // pathtracer.cpp:43-49
                    if ((bs.next() < k) && (depth < C.cap)) e.f = e.f / k;
                    else done = true;
                } else if (C.rr && depth >= C.cap) {
                    done = true;
                }
                if (!done) {
                    beta = ((beta * e.f) * e.wi.y) / e.pdf;        // pathtracer.cpp:52-54
                    if ((beta.x == 0.0f && beta.y == 0.0f && beta.z == 0.0f) ||
                        (!C.rr && depth + 1 >= C.path_length)) {   // the next trace would return 0
                        done = true;
                    } else {
                        keep = true;
                        wo_o = make_float4(no.x, no.y, no.z, o4.w);
                        wo_d = make_float4(wwi.x, wwi.y, wwi.z, d4.w);
                        wo_b = make_float4(beta.x, beta.y, beta.z, __int_as_float(depth + 1));
                        wo_l = make_float4(L.x, L.y, L.z, 0.0f);
                    }
                }
            }
            if (done) splat(C, pix, L);
        }
        const unsigned mask = __ballot_sync(0xFFFFFFFFu, keep);
        if (mask) {
            uint32_t first = 0;
            if (lane == 0) first = atomicAdd(&ctr->n_next, static_cast<uint32_t>(__popc(mask)));
            first = __shfl_sync(0xFFFFFFFFu, first, 0);
            if (keep) {
                const uint32_t slot = first + __popc(mask & ((1u << lane) - 1u));
                nxt.o[slot] = wo_o;
                nxt.d[slot] = wo_d;
                nxt.b[slot] = wo_b;
                nxt.l[slot] = wo_l;
            }
        }
    }
}

__global__ void k_advance(PtConst C, Counters* ctr) {
    Counters c = *ctr;
    const uint32_t n_new = n_new_paths(C, c);
    c.segments += c.n_alive + n_new;
    c.next_path += n_new;
    c.n_alive = c.n_next;
    c.n_next = 0;
    c.iterations += 1;
    *ctr = c;
}

__global__ void k_finalize(float* image, uint64_t n, float inv_spp) {
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x)
        image[i] = image[i] * inv_spp;
}

}  // namespace

}  // namespace spt

using namespace spt;

namespace {

spt_status pathtrace_impl(spt_context* ctx, const spt_scene* sc, const spt_camera* cam, const spt_pt_params* p,
                          float* d_image, spt_render_stats* stats) {
    if (!ctx || !sc || !p || !d_image) return fail(ctx, SPT_ERR_INVALID_ARGUMENT, "NULL argument");
    if (p->pixel_sampler < SPT_PIXEL_UNIFORM || p->pixel_sampler > SPT_PIXEL_JITTERED)
        return fail(ctx, SPT_ERR_INVALID_ARGUMENT, "unknown pixel sampler");
    if (p->termination != SPT_TERMINATE_MAX_DEPTH && p->termination != SPT_TERMINATE_RUSSIAN_ROULETTE)
        return fail(ctx, SPT_ERR_INVALID_ARGUMENT, "unknown path termination criterion");
    if (p->spp == 0) return fail(ctx, SPT_ERR_INVALID_ARGUMENT, "spp must be > 0");
    if (p->path_length < 0 || p->max_depth < 0) return fail(ctx, SPT_ERR_INVALID_ARGUMENT, "negative path length");
    SPT_CUDA(ctx, cudaSetDevice(ctx->device));
    PtConst C;
    std::memset(&C, 0, sizeof(C));
    spt_status st = make_camera(ctx, cam, C.cam);
    if (st != SPT_OK) return st;
    C.S = sc->dev;
    C.seed = p->seed;
    C.sampler = p->pixel_sampler;
    C.spp = p->spp;
    C.nsub = 1;
    C.sw = 1.0f;
    if (p->pixel_sampler != SPT_PIXEL_UNIFORM) {  // regular/jittered round spp up to a square
        C.nsub = static_cast<uint32_t>(std::ceil(std::sqrt(static_cast<double>(p->spp))));
        C.spp = C.nsub * C.nsub;
        C.sw = 1.0f / C.nsub;
    }
    C.rr = p->termination == SPT_TERMINATE_RUSSIAN_ROULETTE;
    C.path_length = p->path_length;
    C.cap = p->max_depth > 0 ? p->max_depth - 1 : 1000;
    C.npix = C.cam.vp_width * C.cam.vp_height;
    C.spp_offset = p->spp_offset;
    C.total = static_cast<uint64_t>(C.npix) * C.spp;
    C.image = d_image;
    const uint64_t img_elems = 3ull * C.cam.width * C.cam.height;
    SPT_CUDA(ctx, cudaMemsetAsync(d_image, 0, img_elems * sizeof(float), ctx->stream));
    if (C.total == 0 || (!C.rr && C.path_length <= 0)) {
        if (stats) std::memset(stats, 0, sizeof(*stats));
        return check_status(ctx);
    }
    uint64_t cap = std::min<uint64_t>(C.total, 1ull << 21);
    C.capacity = static_cast<uint32_t>(cap);
    // scratch: 2 path buffers (4 float4 each) + hits + counters
    void* mem;
    const size_t buf_bytes = cap * sizeof(float4);
    if ((st = scratch(ctx, 5, buf_bytes * 9 + sizeof(Counters) + 256, &mem)) != SPT_OK) return st;
    char* base = static_cast<char*>(mem);
    PathBuf A{reinterpret_cast<float4*>(base), reinterpret_cast<float4*>(base + buf_bytes),
              reinterpret_cast<float4*>(base + 2 * buf_bytes), reinterpret_cast<float4*>(base + 3 * buf_bytes)};
    PathBuf B{reinterpret_cast<float4*>(base + 4 * buf_bytes), reinterpret_cast<float4*>(base + 5 * buf_bytes),
              reinterpret_cast<float4*>(base + 6 * buf_bytes), reinterpret_cast<float4*>(base + 7 * buf_bytes)};
    float4* hits = reinterpret_cast<float4*>(base + 8 * buf_bytes);
    Counters* d_ctr = reinterpret_cast<Counters*>(base + 9 * buf_bytes);
    SPT_CUDA(ctx, cudaMemsetAsync(d_ctr, 0, sizeof(Counters), ctx->stream));
    Counters* h_ctr;
    if ((st = pinned(ctx, sizeof(Counters), reinterpret_cast<void**>(&h_ctr))) != SPT_OK) return st;
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
    const unsigned g_gen = static_cast<unsigned>(std::min<uint64_t>((cap + 255) / 256, 8ull * sms));
    const unsigned g_ext = static_cast<unsigned>(std::min<uint64_t>((cap + 127) / 128, 16ull * sms));
    SPT_CUDA(ctx, cudaEventRecord(ctx->ev0, ctx->stream));
    // Bounded loop: a path can live at most 1001 bounces (the roulette cap), plus one iteration
    // per pool refill; the check below ends it as soon as all paths are done.
    const uint64_t max_iter = (C.total / cap + 2) * 1100ull;
    uint64_t it = 0;
    bool done = false;
    while (!done) {
        for (int k = 0; k < 8; ++k, ++it) {
            PathBuf& cur = (it & 1) ? B : A;
            PathBuf& nxt = (it & 1) ? A : B;
            k_generate<<<g_gen, 256, 0, ctx->stream>>>(C, d_ctr, cur);
            k_extend<<<g_ext, 128, 0, ctx->stream>>>(C, d_ctr, cur, hits, ctx->d_status);
            k_shade<<<g_ext, 128, 0, ctx->stream>>>(C, d_ctr, cur, nxt, hits);
            k_advance<<<1, 1, 0, ctx->stream>>>(C, d_ctr);
        }
        SPT_CUDA(ctx, cudaGetLastError());
        SPT_CUDA(ctx, cudaMemcpyAsync(h_ctr, d_ctr, sizeof(Counters), cudaMemcpyDeviceToHost, ctx->stream));
        SPT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        done = h_ctr->next_path >= C.total && h_ctr->n_alive == 0;
        if (!done && it > max_iter) return fail(ctx, SPT_ERR_TIMEOUT, "path tracer did not finish its bounded loop");
    }
    k_finalize<<<static_cast<unsigned>(std::min<uint64_t>((img_elems + 255) / 256, 4096)), 256, 0, ctx->stream>>>(
        d_image, img_elems, 1.0f / static_cast<float>(C.spp));
    SPT_CUDA(ctx, cudaGetLastError());
    SPT_CUDA(ctx, cudaEventRecord(ctx->ev1, ctx->stream));
    st = check_status(ctx);
    if (st != SPT_OK) return st;
    if (stats) {
        std::memset(stats, 0, sizeof(*stats));
        stats->paths = C.total;
        stats->segments = h_ctr->segments;
        float ms = 0.0f;
        SPT_CUDA(ctx, cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
        stats->gpu_ms = ms;
    }
    return SPT_OK;
}

}  // namespace

extern "C" {

spt_status spt_pathtrace(spt_context* ctx, const spt_scene* sc, const spt_camera* cam, const spt_pt_params* p,
                         float* out_rgb_host, spt_render_stats* stats) {
    if (!ctx || !sc || !cam || !p || !out_rgb_host) return fail(ctx, SPT_ERR_INVALID_ARGUMENT, "NULL argument");
    if (cam->width == 0 || cam->height == 0) return fail(ctx, SPT_ERR_INVALID_ARGUMENT, "empty image");
    const size_t bytes = 3ull * cam->width * cam->height * sizeof(float);
    void* d_img;
    spt_status st = scratch(ctx, 6, bytes, &d_img);
    if (st != SPT_OK) return st;
    st = pathtrace_impl(ctx, sc, cam, p, static_cast<float*>(d_img), stats);
    if (st != SPT_OK) return st;
    SPT_CUDA(ctx, cudaMemcpyAsync(out_rgb_host, d_img, bytes, cudaMemcpyDeviceToHost, ctx->stream));
    SPT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return SPT_OK;
}

spt_status spt_pathtrace_device(spt_context* ctx, const spt_scene* sc, const spt_camera* cam, const spt_pt_params* p,
                                float* d_out_rgb, spt_render_stats* stats) {
    return pathtrace_impl(ctx, sc, cam, p, d_out_rgb, stats);
}

}  // extern "C"
