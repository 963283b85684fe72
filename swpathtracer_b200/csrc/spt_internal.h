// spt_internal.h -- host-side objects behind the C-ABI handles.
#pragma once

#include <cuda_runtime.h>

#include <cstdio>
#include <string>
#include <vector>

#include "../../include/spt.h"
#include "bvh_build.h"
#include "spt_device.cuh"

struct spt_bvh {
    spt::HostBvh tree;
};

struct spt_context {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // streams of the chunked host-buffer pipeline (spt_intersect): copies in, queries and copies out
    // of successive chunks overlap; ev_pipe[i] orders a chunk after the previous user of its buffers
    static constexpr int kPipe = 4;
    cudaStream_t pipe[kPipe] = {};
    cudaEvent_t ev_pipe[kPipe] = {};
    uint32_t* d_status = nullptr;  // device error word: bit 0 stack overflow, bit 1 queue overflow, bit 2 timeout
    std::string err;
    // scratch buffers reused across calls (grown on demand)
    static constexpr int kScratchSlots = 12;
    void* scratch[kScratchSlots] = {};
    size_t scratch_bytes[kScratchSlots] = {};
    void* pinned = nullptr;
    size_t pinned_bytes = 0;
    // ray counters of the persistent (dynamic-fetch) kernels: a ring, one slot per launch
    unsigned long long* d_fetch = nullptr;
    uint32_t fetch_slot = 0;
    // grid of the persistent closest-hit kernel on this context's device, per ray layout (0: 8
    // floats per ray, 1: 6), computed on first use
    int df_grid[2] = {0, 0};
    // device address of the static buffer of spt_intersect_noalloc (noalloc.cu), looked up on first use
    void* noalloc_scratch = nullptr;
    // buffers of the ray ordering pass (ray_order.cu), one per stream that ran a large query, so
    // that queries on different streams never share one
    static constexpr int kStreamScratch = 8;
    cudaStream_t sscratch_stream[kStreamScratch] = {};
    void* sscratch[kStreamScratch] = {};
    size_t sscratch_bytes[kStreamScratch] = {};
};

struct spt_scene {
    spt_context* ctx = nullptr;
    spt::DevScene dev{};
    std::vector<void*> allocations;
    uint64_t bytes = 0;
    uint32_t tree_height = 0;
    uint32_t wide_stack_bound = 0;  // 2 (levels - 1) of the 8-wide tree: the most stack entries a traversal needs
    uint32_t n_materials = 0;
    bool any_emission = false;
    bool any_layered = false;      // a material with more than one BSDF layer
};

namespace spt {

// Status helpers: every entry point records a message and returns a status, never throws.
spt_status fail(spt_context* ctx, spt_status s, const std::string& msg);
// The device builder behind spt_bvh_build_device (bvh_gpu.cu).
spt_status build_ploc_tree(spt_context* ctx, const spt_scene_desc& d, HostBvh& out);
spt_status cuda_fail(spt_context* ctx, cudaError_t e, const char* what);
#define SPT_CUDA(ctx, call)                                          \
    do {                                                             \
        cudaError_t e_ = (call);                                     \
        if (e_ != cudaSuccess) return spt::cuda_fail((ctx), e_, #call); \
    } while (0)

// Grows scratch slot `i` of the context to at least `bytes`.
spt_status scratch(spt_context* ctx, int i, size_t bytes, void** out);
// A buffer of at least `bytes` that only work on stream s uses; *out = NULL when every per-stream
// buffer already belongs to another stream.
spt_status stream_scratch(spt_context* ctx, cudaStream_t s, size_t bytes, void** out);
spt_status pinned(spt_context* ctx, size_t bytes, void** out);

// Reads the device status word and maps it to a status (resets it).
spt_status check_status(spt_context* ctx);

// Host computation of the camera constants (cameras/camera.cpp:3-11, pinhole_camera.cpp:3-12,
// orthographic_camera.cpp:5-19).
spt_status make_camera(spt_context* ctx, const spt_camera* cam, DevCamera& out);

// Kernel launchers (raycast.cu)
// stride: floats per ray, 8 ({origin, pad, direction, pad}) or 6 (the reference's Ray, core/ray.h).
// order: a batch of at least order_min_rays() rays on the persistent traversal is first put in
// coherence order (order_rays); the hits are the same either way.
spt_status launch_intersect(spt_context* ctx, const spt_scene* sc, const float* d_rays, uint64_t n, spt_hit* d_hits,
                            cudaStream_t s, int stride = 8, bool order = false);
// ray_order.cu: the coherence order of n < 2^32 device rays on stream s.  keys: n entries, work:
// order_scratch_bytes(ctx) bytes, order: 2n + 1 entries (order[k] = the k-th ray to trace for k below
// order[2n], the rays that meet the root box; order[n + i] = ray i's place, 0xFFFFFFFF for a ray that
// misses).  unorder_hits: hits[i] = ordered[order[n + i]], or the miss record.
uint64_t order_min_rays();
size_t order_scratch_bytes(spt_context* ctx);
spt_status order_rays(spt_context* ctx, const spt_scene* sc, const float* d_rays, uint64_t n, int stride,
                      cudaStream_t s, uint32_t* keys, uint32_t* work, uint32_t* order);
spt_status unorder_hits(spt_context* ctx, const spt_hit* ordered, const uint32_t* order, uint64_t n, spt_hit* hits,
                        cudaStream_t s);
spt_status launch_count(spt_context* ctx, const spt_scene* sc, const float* d_rays, uint64_t n, spt_hit* d_ref_hits,
                        uint32_t* d_tests, uint32_t* d_hits, uint32_t* d_prim_tests, cudaStream_t s, int stride = 8);

constexpr int kStack = 64;
constexpr uint32_t kFetchRing = 1024;

// Zeroes the next counter of the ring on stream s and returns it (persistent kernels).
spt_status fetch_counter(spt_context* ctx, cudaStream_t s, unsigned long long** out);
// The next slot of the ring as it is (the caller's kernel initialises it).
spt_status ring_slot(spt_context* ctx, unsigned long long** out);
// Blocks of `block` threads that fill every SM once for `kernel` (persistent launches).
int persistent_grid(spt_context* ctx, const void* kernel, int block);

}  // namespace spt
