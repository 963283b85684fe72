// pathtrace.cu -- the path tracer (integrators/pathtracer.cpp:12-147) as a wavefront over a batch
// of scenes.
//
// A pool of path slots (SoA, ping-pong) is refilled with new camera paths as old ones end.  Each
// iteration runs four kernels:
//
//   k_generate  camera rays for free slots (pixel sampler + camera, pathtracer.cpp:104-113)
//   k_extend    closest hit for every live slot (traverse*.cuh, the ray casters' traversal)
//   k_shade     emission, layered BSDF walk, russian roulette and the next ray
//               (pathtracer.cpp:21-54); surviving paths are appended, warp-aggregated, to the other
//               buffer; finished paths add their radiance to their scene's image
//   k_advance   one thread: moves the counters to the next iteration
//
// A batch is a table of jobs (scene + camera + settings); the camera paths of all jobs form one index
// space, so scenes of very different sizes share the pool, and the iterations are replayed from one
// CUDA graph.  A single-scene render is a batch of one.
//
// Random numbers: Philox-4x32-10 keyed by the job's seed, counter (path index, stream, block), stream 0
// for the pixel sample and stream depth+1 for the BSDF walk and roulette at that depth.  The path
// index is (spp_offset + sample) * viewport_pixels + viewport_pixel, so an image does not depend on
// slot assignment, batch composition or tuning (up to the order of the float atomic adds).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "guided_shade.cuh"
#include "guiding_host.h"
#include "shade.cuh"
#include "spt_internal.h"
#include "traverse_wide.cuh"
#include "wavefront.h"

namespace spt {
namespace {

struct Wave {
    const PtJob* jobs;
    uint32_t n_jobs;
    uint64_t total;        // camera paths of all jobs
    uint32_t capacity;     // path slots
    uint32_t stack_limit;  // traversal stack entries a lane may use in the persistent extend kernel
};

struct PathBuf {
    float4* o;   // origin, pixel (viewport index) bits
    float4* d;   // direction, sample index bits
    float4* b;   // throughput, depth | job << 16
    float4* l;   // radiance so far
    uint4* r;    // guided renders: the path's last four training records (generation << 24 | index)
};

struct Counters {
    unsigned long long next_path;   // camera paths generated so far
    unsigned long long segments;    // rays traced so far
    unsigned long long fetch;       // ray counter of the persistent extend kernel
    uint32_t n_alive;               // live slots at the start of the iteration (in the current buffer)
    uint32_t n_next;                // slots appended to the other buffer by k_shade
    uint32_t iterations;
    uint32_t spare;
    uint32_t rec_count;             // training records written into the current generation
    uint32_t rec_gen;               // generation of the record buffer (bumped when it is consumed)
    uint32_t train_on;              // record training data
    uint32_t pad;
};

// Guided renders (guided_shade.cuh): the guide's inputs and outputs for this iteration's hits and the
// training-record buffers.
struct GuideIO {
    float mix;
    uint32_t rec_cap;
    uint32_t depth;        // vertices at path depth < depth are guided
    const float* cache;    // the guide's mixture per (position cell, normal axis): guide::kCacheEntry floats each
    uint8_t* touched;      // per cache entry: set when a guided vertex reads it (the next refresh includes it)
    uint32_t cache_res;    // cells per axis over the guide's box
    float lo[3], inv_ext[3];
    float4* rec;           // 4 float4 per record (spt_guide_record layout)
    float4* recx;          // 2 float4 per record: throughput at the record, radiance gathered after it
};

constexpr uint32_t kNoRec = 0xFFFFFFFFu;
constexpr uint32_t kRecBatches = 4;   // training records held per render: this many optimiser batches
constexpr uint32_t kTrainEpochs = 4;  // optimiser passes over each filled record buffer

__device__ __forceinline__ uint32_t n_new_paths(const Wave& W, const Counters& c) {
    const unsigned long long rem = W.total - c.next_path;
    const uint32_t room = W.capacity - c.n_alive;
    return rem < room ? static_cast<uint32_t>(rem) : room;
}

__device__ __forceinline__ uint32_t job_of(const Wave& W, unsigned long long g) {
    uint32_t lo = 0, hi = W.n_jobs;  // last job with first <= g
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (W.jobs[mid].first <= g) lo = mid;
        else hi = mid;
    }
    return lo;
}

__global__ void __launch_bounds__(256) k_generate(Wave W, const Counters* __restrict__ ctr, PathBuf cur) {
    const Counters c = *ctr;
    const uint32_t n_new = n_new_paths(W, c);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n_new; i += gridDim.x * blockDim.x) {
        const unsigned long long g = c.next_path + i;
        const uint32_t j = job_of(W, g);
        const PtJob& J = W.jobs[j];
        const unsigned long long lg = g - J.first;
        const uint32_t sr = static_cast<uint32_t>(lg / J.npix);
        const uint32_t pix = static_cast<uint32_t>(lg - static_cast<unsigned long long>(sr) * J.npix);
        const uint32_t si = J.s_begin + sr;   // sample index within the pixel's spp
        const uint32_t xx = pix % J.cam.vp_width, yy = pix / J.cam.vp_width;
        const uint32_t x = J.cam.vp_left + xx, y = J.cam.vp_top + yy;
        const uint32_t sg = J.spp_offset + si;
        const unsigned long long path = static_cast<unsigned long long>(sg) * J.npix + pix;
        float sx, sy;
        if (J.sampler == SPT_PIXEL_UNIFORM) {  // uniform_pixel_sampler.cpp:7-10
            Stream cs(J.seed, path, 0);
            sx = cs.next();
            sy = cs.next();
        } else {
            const uint32_t a = si / J.nsub, b = si % J.nsub;
            if (J.sampler == SPT_PIXEL_REGULAR) {  // regular_pixel_sampler.cpp:10-13
                float off = J.sw * 0.5f;
                sx = J.sw * a + off;
                sy = J.sw * b + off;
            } else {  // jittered_pixel_sampler.cpp:11-20
                Stream cs(J.seed, path, 0);
                float u0 = cs.next(), u1 = cs.next();
                sx = J.sw * a + J.sw * u0;
                sy = J.sw * b + J.sw * u1;
            }
        }
        V3 o, d;
        camera_ray(J.cam, static_cast<float>(x) + sx, static_cast<float>(y) + sy, o, d);
        const uint32_t slot = c.n_alive + i;
        cur.o[slot] = make_float4(o.x, o.y, o.z, __uint_as_float(pix));
        cur.d[slot] = make_float4(d.x, d.y, d.z, __uint_as_float(sg));
        cur.b[slot] = make_float4(1.0f, 1.0f, 1.0f, __uint_as_float(j << 16));
        cur.l[slot] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        if (cur.r) cur.r[slot] = make_uint4(kNoRec, kNoRec, kNoRec, kNoRec);
    }
}

// The guide's cache entry of a surface point: its cell in a cache_res^3 grid over the guide's box and
// the axis (with sign) its normal is closest to.
__device__ __forceinline__ uint32_t cache_cell(const GuideIO& G, V3 pos, V3 nrm) {
    const float hi = 0.99999994f;
    const float qx = fminf(fmaxf((pos.x - G.lo[0]) * G.inv_ext[0], 0.0f), hi);
    const float qy = fminf(fmaxf((pos.y - G.lo[1]) * G.inv_ext[1], 0.0f), hi);
    const float qz = fminf(fmaxf((pos.z - G.lo[2]) * G.inv_ext[2], 0.0f), hi);
    const uint32_t r = G.cache_res;
    const uint32_t ix = static_cast<uint32_t>(qx * r), iy = static_cast<uint32_t>(qy * r), iz = static_cast<uint32_t>(qz * r);
    const float ax = fabsf(nrm.x), ay = fabsf(nrm.y), az = fabsf(nrm.z);
    const uint32_t bin = (ax >= ay && ax >= az) ? (nrm.x < 0.0f ? 1u : 0u)
                         : (ay >= az)           ? (nrm.y < 0.0f ? 3u : 2u)
                                                : (nrm.z < 0.0f ? 5u : 4u);
    return ((iz * r + iy) * r + ix) * 6u + bin;
}

__device__ __forceinline__ float4 hit_record(const DevScene& S, const Hit1& h) {
    return make_float4(h.t, __uint_as_float(h.found ? slot_prim(S, h.slot) : SPT_MISS), h.u, h.v);
}

template <int TRAV>
__global__ void __launch_bounds__(256) k_extend(Wave W, const Counters* __restrict__ ctr, PathBuf cur,
                                                float4* __restrict__ hits, uint32_t* status) {
    const Counters c = *ctr;
    const uint32_t n = c.n_alive + n_new_paths(W, c);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 o = cur.o[i], d = cur.d[i];
        const DevScene& S = W.jobs[__float_as_uint(cur.b[i].w) >> 16].S;
        Hit1 h = trace_closest<TRAV>(S, f3v(o), f3v(d), status);
        hits[i] = hit_record(S, h);
    }
}

// Persistent extend: lanes take live slots from the iteration's counter as their rays finish.
// DEPTH: the lane's traversal stack depth (tune.stack); W.stack_limit may hold it lower.
template <int DEPTH>
__global__ void __launch_bounds__(128) k_extend_df(Wave W, Counters* __restrict__ ctr, PathBuf cur,
                                                   float4* __restrict__ hits, uint32_t* status) {
    const Counters c = *ctr;
    const uint32_t n = c.n_alive + n_new_paths(W, c);
    const uint32_t lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    const int limit = static_cast<int>(W.stack_limit);
    WideTraversalT<true, DEPTH> tr;
    // the lane's scene, held by value: the fields the traversal reads stay in registers instead of
    // being reloaded from the job table at every node
    DevScene S{};
    bool active = false, exhausted = false;
    unsigned long long mine = 0, pool = 0, pool_end = 0;
    for (;;) {
        const unsigned need = __ballot_sync(0xFFFFFFFFu, !active && !exhausted);
        if (need) {
            const uint32_t cnt = __popc(need), rank = __popc(need & lt);
            const unsigned long long have = pool_end - pool;
            unsigned long long fresh = 0;
            if (have < cnt) {
                if (lane == 0) fresh = atomicAdd(&ctr->fetch, static_cast<unsigned long long>(kChunk));
                fresh = __shfl_sync(0xFFFFFFFFu, fresh, 0);
            }
            if (!active && !exhausted) {
                mine = rank < have ? pool + rank : fresh + (rank - have);
                if (mine >= n) {
                    exhausted = true;
                } else {
                    S = W.jobs[__float_as_uint(cur.b[mine].w) >> 16].S;
                    active = tr.start(S, f3v(cur.o[mine]), f3v(cur.d[mine]));
                    if (!active) hits[mine] = hit_record(S, tr.h);
                }
            }
            if (have < cnt) {
                pool = fresh + (cnt - have);
                pool_end = fresh + kChunk;
            } else {
                pool += cnt;
            }
        }
        if (__all_sync(0xFFFFFFFFu, !active && exhausted)) break;
        if (active && !tr.step(S, status, limit)) {
            if (tr.finish(S)) {
                hits[mine] = hit_record(S, tr.h);
                active = false;
            }
        }
    }
}

__device__ __forceinline__ void splat(const PtJob& J, uint32_t pix, V3 L) {
    const uint32_t x = J.cam.vp_left + pix % J.cam.vp_width, y = J.cam.vp_top + pix / J.cam.vp_width;
    float* p = J.image + 3ull * (static_cast<uint64_t>(y) * J.cam.width + x);
    if (L.x != 0.0f) atomicAdd(p, L.x);
    if (L.y != 0.0f) atomicAdd(p + 1, L.y);
    if (L.z != 0.0f) atomicAdd(p + 2, L.z);
}

__device__ __forceinline__ bool rec_live(uint32_t r, uint32_t gen) { return r != kNoRec && (r >> 24) == (gen & 0xFFu); }

// ---- shading grouped by material class (tune.sort_shading) ------------------------------------
// A class is what decides the shade kernel's control flow: a miss, a layered stack, or the type of a
// single-layer BSDF.  The slots of an iteration are counted per class, the counts turned into
// offsets, and the slot indices scattered into `order`, so the warps of k_shade take the paths of one
// class together.  The order is only a permutation of slots: every path computes the same values.
constexpr int kShadeClasses = 8;   // miss, layered, 4 single-layer BSDF types (+ 2 spare)

__device__ __forceinline__ int shade_class(const Wave& W, const PathBuf& cur, const float4* hits, uint32_t i) {
    const uint32_t prim = __float_as_uint(hits[i].y);
    if (prim == SPT_MISS) return 0;
    const PtJob& J = W.jobs[__float_as_uint(cur.b[i].w) >> 16];
    const DevMaterial m = J.S.mat[J.S.prim_mat[prim]];
    if (m.layer_count != 1) return 1;
    return 2 + (J.S.bsdf[J.S.layer_ids[m.layer_begin]].type & 3);
}

// counts[k] += slots of class k (block-local histogram, one atomic per class per block)
__global__ void __launch_bounds__(256) k_class_count(Wave W, const Counters* __restrict__ ctr, PathBuf cur,
                                                     const float4* __restrict__ hits, uint32_t* counts) {
    __shared__ uint32_t h[kShadeClasses];
    if (threadIdx.x < kShadeClasses) h[threadIdx.x] = 0;
    __syncthreads();
    const Counters c = *ctr;
    const uint32_t n = c.n_alive + n_new_paths(W, c);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        atomicAdd(&h[shade_class(W, cur, hits, i)], 1u);
    __syncthreads();
    if (threadIdx.x < kShadeClasses && h[threadIdx.x]) atomicAdd(&counts[threadIdx.x], h[threadIdx.x]);
}

// cursors[k] = counts[0] + ... + counts[k-1]; counts cleared for the next iteration
__global__ void k_class_offsets(uint32_t* counts, uint32_t* cursors) {
    uint32_t sum = 0;
    for (int k = 0; k < kShadeClasses; ++k) {
        cursors[k] = sum;
        sum += counts[k];
        counts[k] = 0;
    }
}

__global__ void __launch_bounds__(256) k_class_scatter(Wave W, const Counters* __restrict__ ctr, PathBuf cur,
                                                       const float4* __restrict__ hits, uint32_t* cursors,
                                                       uint32_t* __restrict__ order) {
    const Counters c = *ctr;
    const uint32_t n = c.n_alive + n_new_paths(W, c);
    const uint32_t lane = threadIdx.x & 31;
    for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
        const uint32_t i = base + threadIdx.x;
        const int k = i < n ? shade_class(W, cur, hits, i) : -1;
        for (int q = 0; q < kShadeClasses; ++q) {   // warp-aggregated append per class
            const unsigned mask = __ballot_sync(0xFFFFFFFFu, k == q);
            if (!mask) continue;
            uint32_t first = 0;
            if (lane == __ffs(mask) - 1) first = atomicAdd(&cursors[q], static_cast<uint32_t>(__popc(mask)));
            first = __shfl_sync(0xFFFFFFFFu, first, __ffs(mask) - 1);
            if (k == q) order[first + __popc(mask & ((1u << lane) - 1u))] = i;
        }
    }
}

// Shading is latency-bound, so occupancy pays: at most 80 registers (three blocks of 256 threads per
// SM) runs plain shading 1-3 % faster than the 114 registers it takes unbounded, despite a few
// spilled bytes, and guided shading as fast as its unbounded 122 (148 with a one-block bound: 7 %
// slower).
// RECORDS: the guided render still trains, so paths carry the ids of their open training records and
// add the emission they find to them.  Once the guide is frozen (the last pass of a guided render,
// nearly all of its samples) that state is neither read nor written.
template <bool GUIDED, bool RECORDS>
__global__ void __launch_bounds__(256, 3) k_shade(Wave W, Counters* __restrict__ ctr, PathBuf cur, PathBuf nxt,
                                               const float4* __restrict__ hits, GuideIO G,
                                               const uint32_t* __restrict__ order) {
    const Counters c = *ctr;
    const uint32_t n = c.n_alive + n_new_paths(W, c);
    const uint32_t lane = threadIdx.x & 31;
    // all lanes of a warp iterate together so the append below can be warp-aggregated
    for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
        const uint32_t j = base + threadIdx.x;
        bool keep = false;
        float4 wo_o, wo_d, wo_b, wo_l;
        uint4 rr = make_uint4(kNoRec, kNoRec, kNoRec, kNoRec);
        if (j < n) {
            const uint32_t i = order ? order[j] : j;   // the slot this lane shades
            // the slot's last use in this iteration (the buffer is rewritten as the next one's output):
            // evict-first loads leave L2 to the scene
            const float4 o4 = __ldcs(cur.o + i), d4 = __ldcs(cur.d + i), b4 = __ldcs(cur.b + i), l4 = __ldcs(cur.l + i),
                         h4 = __ldcs(hits + i);
            if (GUIDED && RECORDS) rr = cur.r[i];
            const uint32_t pix = __float_as_uint(o4.w), sg = __float_as_uint(d4.w);
            const uint32_t jd = __float_as_uint(b4.w);
            const int depth = static_cast<int>(jd & 0xFFFFu);
            const PtJob& J = W.jobs[jd >> 16];
            const uint64_t path = static_cast<uint64_t>(sg) * J.npix + pix;
            const V3 o = f3v(o4), d = f3v(d4);
            V3 beta = f3v(b4), L = f3v(l4);
            const uint32_t prim = __float_as_uint(h4.y);
            bool done = false;
            if (prim == SPT_MISS) {  // pathtracer.cpp:21-26
                if (depth == 0) L = L + beta * v3(J.S.bg[0], J.S.bg[1], J.S.bg[2]);
                done = true;
            } else {
                const float t = h4.x;
                const bool sphere = J.S.prim_type[prim] == SPT_PRIM_SPHERE;
                const V3 pos = hit_pos(sphere, o, d, t);
                const V3 nrm = hit_normal(J.S, prim, h4.z, h4.w, pos);
                const DevMaterial m = J.S.mat[J.S.prim_mat[prim]];
                float frame[9];
                onb_from_normal(nrm, frame);                       // pathtracer.cpp:28-30
                const V3 wo = normalize(mat_tmul(frame, -d));
                Stream bs(J.seed, path, static_cast<uint32_t>(depth) + 1u);
                V3 f, refl, wi, wwi;
                float pdf;
                // guided: single-layer materials (guided_sample), and the coated stack from outside
                // (its walk below is the second technique)
                const bool coat = GUIDED && coated(J.S, m);
                const uint32_t gi = (GUIDED && static_cast<uint32_t>(depth) < G.depth && guidable(J.S, m) &&
                                     (!coat || wo.y > 0.0f))
                                        ? cache_cell(G, pos, nrm)
                                        : kNoRec;
                const float* entry = G.cache + static_cast<uint64_t>(guide::kCacheEntry) * (gi != kNoRec ? gi : 0u);
                if (GUIDED && gi != kNoRec) G.touched[gi] = 1;
                bool sampled = false;
                if (GUIDED && gi != kNoRec && (!coat || bs.next() < G.mix)) {
                    const GuidedSample gs = coat ? coated_guide_sample(J.S, m, frame, wo, entry, G.mix, bs)
                                                 : guided_sample(J.S, m, frame, wo, entry, G.mix, bs);
                    f = gs.f;
                    refl = gs.refl;
                    wi = gs.wi_local;
                    wwi = gs.wi_world;
                    pdf = gs.p;
                    sampled = true;
                }
                if (!sampled) {
                    const LayerEval e = eval_layered(J.S, m, wo, bs);
                    f = e.f;
                    refl = e.refl;
                    wi = e.wi;
                    pdf = e.pdf;
                    wwi = mat_mul(frame, e.wi);                    // pathtracer.cpp:37-38
                    if (GUIDED && gi != kNoRec) coated_walk_weight(J.S, m, wo, wwi, e, entry, G.mix, f, pdf);
                }
                if (GUIDED && gi != kNoRec && !(pdf > 0.0f)) {
                    f = v3(0.0f, 0.0f, 0.0f);
                    pdf = 1.0f;
                }
                const V3 no = pos + wwi * 1e-3f;
                const V3 le = v3(m.er, m.eg, m.eb);
                if (GUIDED && RECORDS && (le.x != 0.0f || le.y != 0.0f || le.z != 0.0f)) {
                    // radiance reaching the path's open training records
                    const V3 add = beta * le;
                    const uint32_t ids[4] = {rr.x, rr.y, rr.z, rr.w};
                    for (int k = 0; k < 4; ++k)
                        if (rec_live(ids[k], c.rec_gen)) {
                            float4* sx = G.recx + 2ull * (ids[k] & 0xFFFFFFu) + 1;
                            const float4 v = *sx;
                            *sx = make_float4(v.x + add.x, v.y + add.y, v.z + add.z, 0.0f);
                        }
                }
                L = L + beta * le;
                const float k = fmaxf(fmaxf(refl.x, refl.y), refl.z);
                if (J.rr && depth >= J.path_length) {              // pathtracer.cpp:43-49
                    if ((bs.next() < k) && (depth < J.cap)) f = f / k;
                    else done = true;
                } else if (J.rr && depth >= J.cap) {
                    done = true;
                }
                if (!done) {
                    const V3 beta0 = beta;
                    beta = ((beta * f) * wi.y) / pdf;              // pathtracer.cpp:52-54
                    if ((beta.x == 0.0f && beta.y == 0.0f && beta.z == 0.0f) ||
                        (!J.rr && depth + 1 >= J.path_length) ||  // the next trace would return 0
                        (GUIDED && !(isfinite(beta.x) && isfinite(beta.y) && isfinite(beta.z)))) {
                        done = true;
                    } else {
                        if (GUIDED && RECORDS && gi != kNoRec && c.train_on) {
                            const uint32_t r = atomicAdd(&ctr->rec_count, 1u);
                            if (r < G.rec_cap) {
                                G.rec[4ull * r] = make_float4(pos.x, pos.y, pos.z, 0.0f);
                                G.rec[4ull * r + 1] = make_float4(nrm.x, nrm.y, nrm.z, 0.0f);
                                G.rec[4ull * r + 2] = make_float4(-d.x, -d.y, -d.z, 0.0f);
                                G.rec[4ull * r + 3] = make_float4(wwi.x, wwi.y, wwi.z, 0.0f);
                                G.recx[2ull * r] = make_float4(beta0.x, beta0.y, beta0.z, 0.0f);
                                G.recx[2ull * r + 1] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                                rr = make_uint4(((c.rec_gen & 0xFFu) << 24) | r, rr.x, rr.y, rr.z);
                            }
                        }
                        keep = true;
                        wo_o = make_float4(no.x, no.y, no.z, o4.w);
                        wo_d = make_float4(wwi.x, wwi.y, wwi.z, d4.w);
                        wo_b = make_float4(beta.x, beta.y, beta.z, __uint_as_float(jd + 1u));
                        wo_l = make_float4(L.x, L.y, L.z, 0.0f);
                    }
                }
            }
            if (done) splat(J, pix, L);
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
                if (GUIDED && RECORDS) nxt.r[slot] = rr;
            }
        }
    }
}

__global__ void k_advance(Wave W, Counters* ctr) {
    Counters c = *ctr;
    const uint32_t n_new = n_new_paths(W, c);
    c.segments += c.n_alive + n_new;
    c.next_path += n_new;
    c.n_alive = c.n_next;
    c.n_next = 0;
    c.fetch = 0;
    c.iterations += 1;
    *ctr = c;
}

// End of one pass of the render's device-side loop (a conditional WHILE node of the CUDA graph): loop
// again unless every path has ended, or stop with the timeout status bit once the iteration budget
// is spent.  The budget bounds the loop whatever the kernels before it did.
__global__ void k_continue(Wave W, const Counters* __restrict__ ctr, uint32_t max_iter, uint32_t* status,
                           cudaGraphConditionalHandle loop) {
    const Counters c = *ctr;
    const bool done = c.next_path >= W.total && c.n_alive == 0;
    const bool spent = !done && c.iterations >= max_iter;
    if (spent) atomicOr(status, 4u);
    cudaGraphSetConditional(loop, (done || spent) ? 0u : 1u);
}

// Training weight of every record: luminance of (radiance gathered after the record / throughput at it),
// i.e. the path's estimate of f cos Li / p at the record, clamped to [0, 1e3] (NaN -> 0).  A record
// with a non-finite position, normal or direction (none is expected; one would turn every parameter
// of the guide into NaN through its gradient) becomes a zero-weight record at the origin.
__global__ void k_record_weights(float4* __restrict__ rec, const float4* __restrict__ recx, uint32_t n) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 b = recx[2 * i], sx = recx[2 * i + 1];
        const float r = b.x > 0.0f ? sx.x / b.x : 0.0f, g = b.y > 0.0f ? sx.y / b.y : 0.0f,
                    bl = b.z > 0.0f ? sx.z / b.z : 0.0f;
        const float w = 0.2126f * r + 0.7152f * g + 0.0722f * bl;
        bool finite = true;
        for (int k = 0; k < 4; ++k) {
            const float4 f = rec[4 * i + k];
            finite = finite && isfinite(f.x) && isfinite(f.y) && isfinite(f.z);
        }
        if (finite) {
            rec[4 * i].w = fminf(fmaxf(w, 0.0f), 1e3f);
        } else {
            rec[4 * i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            rec[4 * i + 1] = make_float4(0.0f, 1.0f, 0.0f, 0.0f);
            rec[4 * i + 2] = make_float4(0.0f, 1.0f, 0.0f, 0.0f);
            rec[4 * i + 3] = make_float4(0.0f, 1.0f, 0.0f, 0.0f);
        }
    }
}

__global__ void k_next_generation(Counters* ctr, uint32_t train_on) {
    ctr->rec_count = 0;
    ctr->rec_gen += 1;
    ctr->train_on = train_on;
}

__global__ void k_finalize(float* image, uint64_t n, float inv_spp) {
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x)
        image[i] = image[i] * inv_spp;
}

}  // namespace

spt_status make_job(spt_context* ctx, const spt_scene* sc, const spt_camera* cam, const spt_pt_params* p, float* d_image,
                    PtJob& J) {
    if (!sc || !cam || !p || !d_image) return fail(ctx, SPT_ERR_INVALID_ARGUMENT, "NULL argument");
    if (p->pixel_sampler < SPT_PIXEL_UNIFORM || p->pixel_sampler > SPT_PIXEL_JITTERED)
        return fail(ctx, SPT_ERR_INVALID_ARGUMENT, "unknown pixel sampler");
    if (p->termination != SPT_TERMINATE_MAX_DEPTH && p->termination != SPT_TERMINATE_RUSSIAN_ROULETTE)
        return fail(ctx, SPT_ERR_INVALID_ARGUMENT, "unknown path termination criterion");
    if (p->spp == 0) return fail(ctx, SPT_ERR_INVALID_ARGUMENT, "spp must be > 0");
    if (p->path_length < 0 || p->max_depth < 0) return fail(ctx, SPT_ERR_INVALID_ARGUMENT, "negative path length");
    std::memset(&J, 0, sizeof(J));
    spt_status st = make_camera(ctx, cam, J.cam);
    if (st != SPT_OK) return st;
    J.S = sc->dev;
    J.seed = p->seed;
    J.sampler = p->pixel_sampler;
    J.spp = p->spp;
    J.nsub = 1;
    J.sw = 1.0f;
    if (p->pixel_sampler != SPT_PIXEL_UNIFORM) {  // regular/jittered round spp up to a square
        J.nsub = static_cast<uint32_t>(std::ceil(std::sqrt(static_cast<double>(p->spp))));
        J.spp = J.nsub * J.nsub;
        J.sw = 1.0f / J.nsub;
    }
    J.rr = p->termination == SPT_TERMINATE_RUSSIAN_ROULETTE;
    J.path_length = p->path_length;
    J.cap = p->max_depth > 0 ? p->max_depth - 1 : 1000;
    if (J.cap > 0xFFFE) J.cap = 0xFFFE;  // depth is kept in 16 bits
    J.npix = J.cam.vp_width * J.cam.vp_height;
    J.spp_offset = p->spp_offset;
    J.image = d_image;
    J.layered = sc->any_layered ? 1u : 0u;
    J.stack_bound = sc->wide_stack_bound;
    set_sample_range(J, 0, J.spp);
    return SPT_OK;
}

void set_sample_range(PtJob& J, uint32_t s_begin, uint32_t s_end) {
    J.s_end = std::min(s_end, J.spp);
    J.s_begin = std::min(s_begin, J.s_end);
    const bool empty = !J.rr && J.path_length <= 0;   // the reference traces nothing at all then
    J.total = empty ? 0 : static_cast<uint64_t>(J.npix) * (J.s_end - J.s_begin);
}

spt_tune default_tune() {
    spt_tune t;
    std::memset(&t, 0, sizeof(t));
    t.capacity = 1u << 21;
    t.extend_block = 128;
    t.shade_block = 128;
    t.traversal = -1;
    t.check_every = 8;
    t.stack = 0;
    t.stack_limit = 0;
    t.max_iterations = 0;
    return t;
}

spt_status render_jobs(spt_context* ctx, std::vector<PtJob>& jobs, const spt_tune& tune, uint64_t* segments,
                       float* gpu_ms, guide::Guide* guide, uint32_t train_budget, uint32_t* train_steps) {
    SPT_CUDA(ctx, cudaSetDevice(ctx->device));
    if (jobs.empty() || jobs.size() >= (1u << 16))
        return fail(ctx, SPT_ERR_INVALID_ARGUMENT, "a batch holds 1 to 65535 jobs");
    auto block_ok = [](uint32_t b) { return b == 0 || (b % 32 == 0 && b <= 256); };
    if (!block_ok(tune.extend_block) || !block_ok(tune.shade_block))
        return fail(ctx, SPT_ERR_INVALID_ARGUMENT, "tune block sizes must be multiples of 32 up to 256");
    if (tune.traversal < -1 || tune.traversal > 2) return fail(ctx, SPT_ERR_INVALID_ARGUMENT, "unknown traversal");
    if (tune.stack != 0 && tune.stack != 16 && tune.stack != 24 && tune.stack != 32)
        return fail(ctx, SPT_ERR_INVALID_ARGUMENT, "tune.stack must be 0, 16, 24 or 32");
    if (train_steps) *train_steps = 0;
    uint64_t total = 0;
    int trav = 2;
    for (PtJob& J : jobs) {
        J.first = total;
        total += J.total;
        if (J.total) trav = std::min(trav, J.S.traversal);  // a scene without a wide tree forces binary
        const uint64_t img_elems = 3ull * J.cam.width * J.cam.height;
        if (J.s_begin == 0) SPT_CUDA(ctx, cudaMemsetAsync(J.image, 0, img_elems * sizeof(float), ctx->stream));
    }
    // Default: the scene's best (8-wide, persistent with dynamic fetch and postponed triangles):
    // measured 427 vs 405 Mpaths/s on the box workload and 254 vs 233 on the layered one against
    // the 8-wide tree with one thread per path.
    if (tune.traversal >= 0 && tune.traversal <= trav) trav = tune.traversal;
    *segments = 0;
    *gpu_ms = 0.0f;
    if (total == 0) return check_status(ctx);
    const uint64_t cap = std::min<uint64_t>(total, std::max<uint32_t>(tune.capacity, 1024u));
    // Buffer stride: the pool size, or for guided renders (a series of growing passes) the full
    // tuned capacity, so later passes reuse the first pass's scratch instead of growing it.
    const uint64_t stride = guide ? std::max<uint64_t>(cap, std::max<uint32_t>(tune.capacity, 1024u)) : cap;
    spt_status st;
    void* mem;
    const size_t buf_bytes = stride * sizeof(float4);
    const size_t job_bytes = jobs.size() * sizeof(PtJob);
    const size_t order_bytes = (stride * sizeof(uint32_t) + 255) & ~static_cast<size_t>(255);
    if ((st = scratch(ctx, 5, buf_bytes * 9 + sizeof(Counters) + job_bytes + 512 + order_bytes + 256, &mem)) != SPT_OK)
        return st;
    char* base = static_cast<char*>(mem);
    PathBuf A{reinterpret_cast<float4*>(base), reinterpret_cast<float4*>(base + buf_bytes),
              reinterpret_cast<float4*>(base + 2 * buf_bytes), reinterpret_cast<float4*>(base + 3 * buf_bytes), nullptr};
    PathBuf B{reinterpret_cast<float4*>(base + 4 * buf_bytes), reinterpret_cast<float4*>(base + 5 * buf_bytes),
              reinterpret_cast<float4*>(base + 6 * buf_bytes), reinterpret_cast<float4*>(base + 7 * buf_bytes),
              nullptr};
    float4* hits = reinterpret_cast<float4*>(base + 8 * buf_bytes);
    Counters* d_ctr = reinterpret_cast<Counters*>(base + 9 * buf_bytes);
    PtJob* d_jobs = reinterpret_cast<PtJob*>(base + 9 * buf_bytes + 256);
    char* tail = base + 9 * buf_bytes + 256 + ((job_bytes + 255) & ~static_cast<size_t>(255));
    uint32_t* d_order = reinterpret_cast<uint32_t*>(tail);
    uint32_t* d_class = reinterpret_cast<uint32_t*>(tail + order_bytes);   // counts[8], cursors[8]
    bool any_layered = false;
    for (const PtJob& J : jobs) any_layered |= J.layered != 0;
    // measured: +8 % on the layered 1.3M-tri workload, -6 % on the box of Lambertian walls
    const bool sort_shading = tune.sort_shading == 1 || (tune.sort_shading == 0 && any_layered);
    SPT_CUDA(ctx, cudaMemsetAsync(d_ctr, 0, sizeof(Counters), ctx->stream));
    if (sort_shading) SPT_CUDA(ctx, cudaMemsetAsync(d_class, 0, 2 * kShadeClasses * sizeof(uint32_t), ctx->stream));
    SPT_CUDA(ctx, cudaMemcpyAsync(d_jobs, jobs.data(), job_bytes, cudaMemcpyHostToDevice, ctx->stream));
    GuideIO G{};
    uint32_t batch = 0, rec_cap = 0;
    if (guide) {
        // guided state: record ids per path, the guide's per-hit inputs/outputs, training records
        batch = guide->cfg.batch;
        if (batch > (1u << 24) / kRecBatches)
            return fail(ctx, SPT_ERR_INVALID_ARGUMENT, "guide batch must be at most 2^22 records");
        rec_cap = kRecBatches * batch;
        void* gm;
        const size_t gbytes = 2 * stride * sizeof(uint4) + static_cast<size_t>(rec_cap) * 6 * sizeof(float4) + 1024;
        if ((st = scratch(ctx, 2, gbytes, &gm)) != SPT_OK) return st;
        char* g = static_cast<char*>(gm);
        A.r = reinterpret_cast<uint4*>(g);
        B.r = A.r + stride;
        G.rec = reinterpret_cast<float4*>(B.r + stride);
        G.recx = G.rec + 4ull * rec_cap;
        G.mix = guide->cfg.mix;
        G.rec_cap = rec_cap;
        G.depth = guide->cfg.guided_depth ? guide->cfg.guided_depth : 0xFFFFFFFFu;
        if ((st = guide->refresh_cache()) != SPT_OK) return st;
        guide->touched_any = true;
        G.cache = guide->cache;
        G.touched = guide->touched;
        G.cache_res = guide->cache_res;
        for (int k = 0; k < 3; ++k) {
            G.lo[k] = guide->model.lo[k];
            G.inv_ext[k] = guide->model.inv_ext[k];
        }
        const uint32_t on = train_budget > 0 ? 1u : 0u;
        SPT_CUDA(ctx, cudaMemcpyAsync(&d_ctr->train_on, &on, sizeof(on), cudaMemcpyHostToDevice, ctx->stream));
        SPT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    }
    Counters* h_ctr;
    if ((st = pinned(ctx, sizeof(Counters), reinterpret_cast<void**>(&h_ctr))) != SPT_OK) return st;
    // traversal stack of the persistent extend kernel: the compiled depth (tune.stack, or the smallest
    // of 16 / 24 / 32 that holds the deepest wide tree of the batch) and the entries a lane may use
    uint32_t depth = tune.stack;
    if (depth == 0) {
        uint32_t need = 0;
        for (const PtJob& J : jobs) need = std::max(need, J.stack_bound);
        depth = need <= 16 ? 16 : need <= 24 ? 24 : 32;
    }
    const uint32_t limit = tune.stack_limit ? std::min(tune.stack_limit, depth) : depth;
    Wave W{d_jobs, static_cast<uint32_t>(jobs.size()), total, static_cast<uint32_t>(cap), limit};
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
    const unsigned eb = tune.extend_block ? tune.extend_block : 128, sb = tune.shade_block ? tune.shade_block : 128;
    const unsigned g_gen = static_cast<unsigned>(std::min<uint64_t>((cap + 255) / 256, 8ull * sms));
    const unsigned g_ext = static_cast<unsigned>(std::min<uint64_t>((cap + eb - 1) / eb, 16ull * sms * 128 / eb));
    const unsigned g_shd = static_cast<unsigned>(std::min<uint64_t>((cap + sb - 1) / sb, 16ull * sms * 128 / sb));
    auto ext_df = depth == 16 ? k_extend_df<16> : depth == 24 ? k_extend_df<24> : k_extend_df<32>;
    int per_sm = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ext_df, 128, 0);
    const unsigned g_df = static_cast<unsigned>(sms * std::max(1, per_sm));
    // Bound of the loop: a path lives at most ~1001 bounces (the roulette cap), plus one iteration per
    // pool refill; tune.max_iterations may set a lower budget.
    uint64_t max_iter = std::min<uint64_t>((total / cap + 2) * 1100ull, 0xFFFFFFF0ull);
    if (tune.max_iterations) max_iter = std::min<uint64_t>(max_iter, tune.max_iterations);
    // Only a guide that trains during the render needs the host between iterations (it runs the
    // optimiser steps on the records the paths wrote), or a caller that asks for the host-driven loop
    // (tune.host_loop).  Every other render is one launch of a graph whose WHILE node repeats two
    // iterations until k_continue sees the pool drained.
    const bool host_loop = (guide && train_budget > 0) || tune.host_loop != 0;
    auto record_iterations = [&](cudaGraphConditionalHandle* loop) {
        for (int it = 0; it < 2; ++it) {
            PathBuf& cur = it ? B : A;
            PathBuf& nxt = it ? A : B;
            k_generate<<<g_gen, 256, 0, ctx->stream>>>(W, d_ctr, cur);
            if (trav == 2) ext_df<<<g_df, 128, 0, ctx->stream>>>(W, d_ctr, cur, hits, ctx->d_status);
            else if (trav == 1) k_extend<1><<<g_ext, eb, 0, ctx->stream>>>(W, d_ctr, cur, hits, ctx->d_status);
            else k_extend<0><<<g_ext, eb, 0, ctx->stream>>>(W, d_ctr, cur, hits, ctx->d_status);
            const uint32_t* order = nullptr;
            if (sort_shading) {
                k_class_count<<<g_shd, 256, 0, ctx->stream>>>(W, d_ctr, cur, hits, d_class);
                k_class_offsets<<<1, 1, 0, ctx->stream>>>(d_class, d_class + kShadeClasses);
                k_class_scatter<<<g_shd, 256, 0, ctx->stream>>>(W, d_ctr, cur, hits, d_class + kShadeClasses, d_order);
                order = d_order;
            }
            if (guide) {
                if (train_budget > 0) k_shade<true, true><<<g_shd, sb, 0, ctx->stream>>>(W, d_ctr, cur, nxt, hits, G, order);
                else k_shade<true, false><<<g_shd, sb, 0, ctx->stream>>>(W, d_ctr, cur, nxt, hits, G, order);
            } else {
                k_shade<false, false><<<g_shd, sb, 0, ctx->stream>>>(W, d_ctr, cur, nxt, hits, G, order);
            }
            k_advance<<<1, 1, 0, ctx->stream>>>(W, d_ctr);
        }
        if (loop)
            k_continue<<<1, 1, 0, ctx->stream>>>(W, d_ctr, static_cast<uint32_t>(max_iter), ctx->d_status, *loop);
    };
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaError_t ce = cudaSuccess;
    if (host_loop) {
        // one graph = two iterations (A -> B, B -> A), replayed by the host loop below
        SPT_CUDA(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
        record_iterations(nullptr);
        ce = cudaStreamEndCapture(ctx->stream, &graph);
        if (ce != cudaSuccess) return cuda_fail(ctx, ce, "cudaStreamEndCapture");
    } else {
        SPT_CUDA(ctx, cudaGraphCreate(&graph, 0));
        cudaGraphConditionalHandle loop;
        // zero-initialised in place: the C++ view of this struct has no default constructor
        alignas(cudaGraphNodeParams) unsigned char cp_bytes[sizeof(cudaGraphNodeParams)] = {};
        cudaGraphNodeParams& cp = *reinterpret_cast<cudaGraphNodeParams*>(cp_bytes);
        ce = cudaGraphConditionalHandleCreate(&loop, graph, 1u, cudaGraphCondAssignDefault);
        if (ce == cudaSuccess) {
            cp.type = cudaGraphNodeTypeConditional;
            cp.conditional.handle = loop;
            cp.conditional.type = cudaGraphCondTypeWhile;
            cp.conditional.size = 1;
            cudaGraphNode_t node;
            ce = cudaGraphAddNode(&node, graph, nullptr, 0, &cp);
        }
        if (ce == cudaSuccess)
            ce = cudaStreamBeginCaptureToGraph(ctx->stream, cp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                               cudaStreamCaptureModeThreadLocal);
        if (ce != cudaSuccess) {
            cudaGraphDestroy(graph);
            return cuda_fail(ctx, ce, "building the render loop graph");
        }
        record_iterations(&loop);
        cudaGraph_t body = nullptr;
        ce = cudaStreamEndCapture(ctx->stream, &body);
        if (ce != cudaSuccess) {
            cudaGraphDestroy(graph);
            return cuda_fail(ctx, ce, "cudaStreamEndCapture (render loop body)");
        }
    }
    ce = cudaGraphInstantiate(&exec, graph, 0);
    if (ce != cudaSuccess) {
        cudaGraphDestroy(graph);
        return cuda_fail(ctx, ce, "cudaGraphInstantiate");
    }
    SPT_CUDA(ctx, cudaEventRecord(ctx->ev0, ctx->stream));
    const unsigned check = std::max(1u, tune.check_every / 2);
    uint64_t it = 0;
    bool done = false;
    bool training = guide && train_budget > 0, pending = false;
    uint32_t steps = 0;
    // kTrainEpochs passes of optimiser steps over the n records in the buffer, batch records per step
    // (a short tail joins no step of its own), then a fresh generation of records.
    auto train = [&](uint32_t n) -> spt_status {
        k_record_weights<<<256, 256, 0, ctx->stream>>>(G.rec, G.recx, n);
        for (uint32_t e = 0; e < kTrainEpochs; ++e)
            for (uint32_t off = 0; off < n && steps < train_budget; off += batch) {
                const uint32_t m = std::min(batch, n - off);
                if (m < batch / 4 && off > 0) break;
                spt_status s2 = guide->step(G.rec + 4ull * off, m, nullptr);
                if (s2 != SPT_OK) return s2;
                ++steps;
            }
        training = steps < train_budget;
        spt_status s3 = guide->refresh_cache();   // the next iterations sample the updated guide
        if (s3 != SPT_OK) return s3;
        k_next_generation<<<1, 1, 0, ctx->stream>>>(d_ctr, training ? 1u : 0u);
        return SPT_OK;
    };
    st = SPT_OK;
    if (!host_loop) {
        // the whole render: one launch, one wait
        ce = cudaGraphLaunch(exec, ctx->stream);
        if (ce == cudaSuccess) ce = cudaMemcpyAsync(h_ctr, d_ctr, sizeof(Counters), cudaMemcpyDeviceToHost, ctx->stream);
        if (ce == cudaSuccess) ce = cudaStreamSynchronize(ctx->stream);
        if (ce != cudaSuccess) st = cuda_fail(ctx, ce, "path tracer render loop");
        if (st == SPT_OK) st = check_status(ctx);   // timeout (budget spent) or stack overflow
        done = true;
    }
    while (!done) {
        for (unsigned k = 0; k < check; ++k, it += 2) {
            ce = cudaGraphLaunch(exec, ctx->stream);
            if (ce != cudaSuccess) break;
        }
        if (ce != cudaSuccess) {
            st = cuda_fail(ctx, ce, "cudaGraphLaunch");
            break;
        }
        ce = cudaMemcpyAsync(h_ctr, d_ctr, sizeof(Counters), cudaMemcpyDeviceToHost, ctx->stream);
        if (ce == cudaSuccess) ce = cudaStreamSynchronize(ctx->stream);
        if (ce != cudaSuccess) {
            st = cuda_fail(ctx, ce, "path tracer iteration");
            break;
        }
        done = h_ctr->next_path >= total && h_ctr->n_alive == 0;
        const uint32_t n_rec = std::min(h_ctr->rec_count, rec_cap);
        if (training && done) {
            // every path has ended: all records carry their final radiance
            if (n_rec >= std::min(batch, 1024u) && (st = train(n_rec)) != SPT_OK) break;
        } else if (training && n_rec >= rec_cap) {
            // A full record buffer takes no more records; its paths keep adding the radiance they
            // find.  The steps wait one check interval (check_every bounces) so most of it is in.
            if (!pending) {
                pending = true;
            } else {
                pending = false;
                if ((st = train(n_rec)) != SPT_OK) break;
            }
        }
        if (!done && it >= max_iter) {
            st = fail(ctx, SPT_ERR_TIMEOUT, "path tracer did not finish its bounded loop");
            break;
        }
    }
    cudaGraphExecDestroy(exec);
    cudaGraphDestroy(graph);
    if (train_steps) *train_steps = steps;
    if (st != SPT_OK) return st;
    for (const PtJob& J : jobs) {
        if (J.s_end != J.spp) continue;
        const uint64_t img_elems = 3ull * J.cam.width * J.cam.height;
        k_finalize<<<static_cast<unsigned>(std::min<uint64_t>((img_elems + 255) / 256, 4096)), 256, 0, ctx->stream>>>(
            J.image, img_elems, 1.0f / static_cast<float>(J.spp));
    }
    SPT_CUDA(ctx, cudaGetLastError());
    SPT_CUDA(ctx, cudaEventRecord(ctx->ev1, ctx->stream));
    st = check_status(ctx);
    if (st != SPT_OK) return st;
    *segments = h_ctr->segments;
    SPT_CUDA(ctx, cudaEventElapsedTime(gpu_ms, ctx->ev0, ctx->ev1));
    return SPT_OK;
}

}  // namespace spt

using namespace spt;

namespace {

spt_status pathtrace_impl(spt_context* ctx, const spt_scene* sc, const spt_camera* cam, const spt_pt_params* p,
                          float* d_image, spt_render_stats* stats) {
    if (!ctx) return SPT_ERR_INVALID_ARGUMENT;
    std::vector<PtJob> jobs(1);
    spt_status st = make_job(ctx, sc, cam, p, d_image, jobs[0]);
    if (st != SPT_OK) return st;
    uint64_t segs = 0;
    float ms = 0.0f;
    st = render_jobs(ctx, jobs, default_tune(), &segs, &ms);
    if (st != SPT_OK) return st;
    if (stats) {
        std::memset(stats, 0, sizeof(*stats));
        stats->paths = jobs[0].total;
        stats->segments = segs;
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
