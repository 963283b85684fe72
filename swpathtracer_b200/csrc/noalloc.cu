// noalloc.cu -- spt_intersect_noalloc: the closest-hit query of spt_intersect (host buffers in and
// out) with all of its device-side scratch in one static buffer, so that a call allocates nothing.
//
// Why it exists: spt_intersect stages rays, hits and counts in per-context scratch buffers that grow
// by cudaFree + cudaMalloc, and the persistent kernel's ray counter ring is allocated on first use.
// Two kinds of caller cannot have that happen inside the call.  A caller that shares the device with
// other busy streams cannot pay for cudaFree, which waits for all work on the device.  A caller that
// has already reserved the device's memory for itself (a renderer embedded in an application that
// owns a fixed memory budget) cannot count on cudaMalloc succeeding in the middle of a frame.  This
// entry point touches no allocator: its scratch lives in g_scratch below, which the CUDA runtime
// places when it loads this file's module, and its host side uses the caller's own buffers.
//
// Limits and rules of use:
//   * at most kNoAllocRays rays per call; larger batches are rejected (split them);
//   * g_scratch is one buffer per device shared by every context in the process: calls that overlap
//     in time on the same device (two threads, or two streams of different contexts) race on it and
//     must be serialised by the caller;
//   * the fetch counter must be zero when the kernel starts; every call clears it on its own stream
//     before the launch.  Nothing else needs clearing: the ray area is overwritten by the upload and
//     the hit and count areas by the kernels, for every index below n;
//   * the first call with a context resolves the buffer's address with cudaGetSymbolAddress (with the
//     context's device current), which may load the module; make that first call before any stream
//     capture begins on the device.  The address is kept in the context, so a context must not be
//     used after a cudaDeviceReset of its device (no context of this library may).
#include "spt_internal.h"

namespace spt {

// raycast.cu: the closest-hit launch with a caller-provided ray counter (zeroed by the caller).
spt_status launch_intersect_fixed(spt_context* ctx, const spt_scene* sc, const float* d_rays, uint64_t n,
                                  spt_hit* d_hits, unsigned long long* next, cudaStream_t s);

namespace {

constexpr uint64_t kNoAllocRays = 1ull << 16;
// layout: fetch counter (256 B), rays (32 B each), hits (16 B each), tests (4 B each), passes (4 B each)
constexpr size_t kRaysOff = 256;
constexpr size_t kHitsOff = kRaysOff + kNoAllocRays * 32;
constexpr size_t kTestsOff = kHitsOff + kNoAllocRays * sizeof(spt_hit);
constexpr size_t kPassesOff = kTestsOff + kNoAllocRays * sizeof(uint32_t);
constexpr size_t kScratchBytes = kPassesOff + kNoAllocRays * sizeof(uint32_t);  // 3.5 MiB + 256 B
static_assert(kHitsOff % 256 == 0 && kTestsOff % 256 == 0 && kPassesOff % 256 == 0, "aligned areas");

__device__ __align__(256) unsigned char g_scratch[kScratchBytes];

// Device address of g_scratch on the context's device, looked up once per context (with the context's
// device current) and kept in the context: a context lives on one device, and its lifetime ends before
// that device's primary context could be reset under it.
spt_status scratch_address(spt_context* ctx, unsigned char** out) {
    if (!ctx->noalloc_scratch) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);  // the caller made ctx->device current
        if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaGetSymbolAddress(static scratch)");
        ctx->noalloc_scratch = p;
    }
    *out = static_cast<unsigned char*>(ctx->noalloc_scratch);
    return SPT_OK;
}

}  // namespace
}  // namespace spt

using namespace spt;

extern "C" {

spt_status spt_intersect_noalloc(spt_context* ctx, const spt_scene* sc, const float* rays, uint64_t n, spt_hit* hits,
                                 uint32_t* tests, uint32_t* nhits) {
    if (!ctx || !sc || (n && (!rays || !hits))) return fail(ctx, SPT_ERR_INVALID_ARGUMENT, "NULL argument");
    if (n > kNoAllocRays)
        return fail(ctx, SPT_ERR_INVALID_ARGUMENT,
                    "spt_intersect_noalloc takes at most 65536 rays per call (its static buffer's size)");
    if (n == 0) return SPT_OK;
    SPT_CUDA(ctx, cudaSetDevice(ctx->device));
    unsigned char* base;
    spt_status st = scratch_address(ctx, &base);
    if (st != SPT_OK) return st;
    unsigned long long* next = reinterpret_cast<unsigned long long*>(base);
    float* d_rays = reinterpret_cast<float*>(base + kRaysOff);
    spt_hit* d_hits = reinterpret_cast<spt_hit*>(base + kHitsOff);
    uint32_t* d_tests = tests ? reinterpret_cast<uint32_t*>(base + kTestsOff) : nullptr;
    uint32_t* d_passes = nhits ? reinterpret_cast<uint32_t*>(base + kPassesOff) : nullptr;
    SPT_CUDA(ctx, cudaMemsetAsync(next, 0, sizeof(unsigned long long), ctx->stream));
    SPT_CUDA(ctx, cudaMemcpyAsync(d_rays, rays, n * 32, cudaMemcpyHostToDevice, ctx->stream));
    if ((st = launch_intersect_fixed(ctx, sc, d_rays, n, d_hits, next, ctx->stream)) != SPT_OK) return st;
    if (tests || nhits)
        if ((st = launch_count(ctx, sc, d_rays, n, nullptr, d_tests, d_passes, nullptr, ctx->stream)) != SPT_OK)
            return st;
    SPT_CUDA(ctx, cudaMemcpyAsync(hits, d_hits, n * sizeof(spt_hit), cudaMemcpyDeviceToHost, ctx->stream));
    if (tests) SPT_CUDA(ctx, cudaMemcpyAsync(tests, d_tests, n * 4, cudaMemcpyDeviceToHost, ctx->stream));
    if (nhits) SPT_CUDA(ctx, cudaMemcpyAsync(nhits, d_passes, n * 4, cudaMemcpyDeviceToHost, ctx->stream));
    return check_status(ctx);
}

}  // extern "C"
