// ray_order.cu -- coherence order of a large batch of ray queries.
//
// Incoherent rays (random origins, random directions) leave the 8-wide traversal's warps diverged:
// the lanes of a warp walk unrelated parts of the tree.  Before the persistent closest-hit kernel runs
// a large batch, the batch is put in an order in which neighbouring rays start where their neighbours
// start and point where they point; the kernel takes its rays in that order and writes each hit at
// the ray's place in the order, and a gather puts the hits back at each ray's own index (nothing a
// caller sees changes).
//
// The key of a ray is where it enters the scene's root box (a Morton code of the entry point, 4 bits
// per axis, or of the origin when the ray starts inside) above the octant of its direction.  A ray
// that the traversal's own root test rejects takes no place in the order: the gather writes its miss
// record, and the traversal runs only over the rays that meet the box (their count is the order's
// last entry).  The order is a counting sort over the keys without global atomics: every block
// counts its contiguous share of the rays in a shared-memory histogram (k_order_count), one thread per
// key turns the per-block counts into each block's first place per key and the key's total
// (k_order_offsets), and every block scans the totals for the keys' bases and places its rays again
// from its own counters (k_order_scatter), writing the order and its inverse.  The order of rays
// within one block's share of a key follows shared-memory atomics and is not fixed; no result
// depends on it.
#include <algorithm>

#include "spt_internal.h"

namespace spt {
namespace {

constexpr int kEntryBits = 4;                                      // per axis of the entry point
constexpr uint32_t kBins = 1u << (3 * kEntryBits + 3);             // entry cell x direction octant
constexpr uint32_t kMiss = 0xFFFFFFFFu;                            // key of a ray that misses the root box
constexpr int kOrderThreads = 1024;
constexpr size_t kOrderSmem = kBins * sizeof(uint32_t);            // 128 KB
constexpr int kUnroll = 4;                                         // independent loads per thread and pass

__device__ __forceinline__ uint32_t spread3(uint32_t x) {   // bits of x at every third position
    uint32_t r = 0;
#pragma unroll
    for (int b = 0; b < kEntryBits; ++b) r |= ((x >> b) & 1u) << (3 * b);
    return r;
}

__device__ __forceinline__ uint32_t quantise(float v, float lo, float inv, uint32_t cells) {
    const float q = (v - lo) * inv * static_cast<float>(cells);
    // NaN and out-of-range values clamp to the grid (fmaxf returns 0 for NaN)
    return static_cast<uint32_t>(fminf(fmaxf(q, 0.0f), static_cast<float>(cells - 1)));
}

template <int STRIDE>
__device__ __forceinline__ void order_ray(const float* __restrict__ rays, uint64_t i, V3& o, V3& d) {
    if (STRIDE == 8) {
        const float4* r = reinterpret_cast<const float4*>(rays) + 2 * i;
        o = f3v(__ldg(r));
        d = f3v(__ldg(r + 1));
    } else {
        const float2* r = reinterpret_cast<const float2*>(rays) + 3 * i;
        const float2 a = __ldg(r), b = __ldg(r + 1), c = __ldg(r + 2);
        o = v3(a.x, a.y, b.x);
        d = v3(b.y, c.x, c.y);
    }
}

// The key of a ray, or kMiss when the traversal's own root test (the same slab test on the same
// values, so the same verdict bit for bit) rejects it: such a ray's hit is the miss record.
__device__ __forceinline__ uint32_t ray_key(const DevScene& S, V3 o, V3 d) {
    if (S.empty) return kMiss;
    const RayInv ri = ray_inv(o, d);
    float t0, t1;
    if (!slab(ri, S.root_min[0], S.root_min[1], S.root_min[2], S.root_max[0], S.root_max[1], S.root_max[2], t0, t1))
        return kMiss;
    const float te = fmaxf(t0, 0.0f);   // the entry point, or the origin inside the box
    const float od[3] = {o.x, o.y, o.z}, dd[3] = {d.x, d.y, d.z};
    uint32_t m = 0;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float ext = S.root_max[k] - S.root_min[k];
        const float inv = ext > 0.0f ? 1.0f / ext : 0.0f;
        m |= spread3(quantise(od[k] + dd[k] * te, S.root_min[k], inv, 1u << kEntryBits)) << k;
    }
    const uint32_t oct = (d.x < 0.0f ? 1u : 0u) | (d.y < 0.0f ? 2u : 0u) | (d.z < 0.0f ? 4u : 0u);
    return (m << 3) | oct;
}

// Block g's share of the rays: [g * per, min(n, (g + 1) * per)).
__device__ __forceinline__ void share(uint32_t n, uint32_t& lo, uint32_t& hi) {
    const uint32_t per = (n + gridDim.x - 1) / gridDim.x;
    lo = min(n, blockIdx.x * per);
    hi = min(n, lo + per);
}

// The key of every ray, and every block's count per key: counts[g * kBins + key].
template <int STRIDE>
__global__ void __launch_bounds__(kOrderThreads) k_order_count(DevScene S, const float* __restrict__ rays, uint32_t n,
                                                              uint32_t* __restrict__ keys,
                                                              uint32_t* __restrict__ counts) {
    extern __shared__ uint32_t hist[];
    for (uint32_t b = threadIdx.x; b < kBins; b += blockDim.x) hist[b] = 0;
    __syncthreads();
    uint32_t lo, hi;
    share(n, lo, hi);
    // kUnroll rays per thread and pass, their loads first, so more loads are in flight
    for (uint64_t base = lo + threadIdx.x; base < hi; base += kUnroll * blockDim.x) {
        V3 o[kUnroll], d[kUnroll];
#pragma unroll
        for (int j = 0; j < kUnroll; ++j) {
            const uint64_t i = base + static_cast<uint64_t>(j) * blockDim.x;
            if (i < hi) order_ray<STRIDE>(rays, i, o[j], d[j]);
        }
#pragma unroll
        for (int j = 0; j < kUnroll; ++j) {
            const uint64_t i = base + static_cast<uint64_t>(j) * blockDim.x;
            if (i < hi) {
                const uint32_t key = ray_key(S, o[j], d[j]);
                keys[i] = key;
                if (key != kMiss) atomicAdd(hist + key, 1u);
            }
        }
    }
    __syncthreads();
    uint32_t* out = counts + static_cast<uint64_t>(blockIdx.x) * kBins;
    for (uint32_t b = threadIdx.x; b < kBins; b += blockDim.x) out[b] = hist[b];
}

// Per key: every block's count becomes the number of rays of that key in the blocks before it, and
// the key's total goes to totals[key].  A block takes 32 keys (one per lane) and its 32 warps a run of
// blocks each; the warps' sums meet in shared memory.
constexpr int kMaxRowsPerWarp = 8;   // blocks of the count pass per warp: up to 256 SMs
__global__ void __launch_bounds__(1024) k_order_offsets(uint32_t* __restrict__ counts, uint32_t blocks,
                                                        uint32_t* __restrict__ totals) {
    __shared__ uint32_t part[32][33];
    const uint32_t lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
    const uint32_t b = blockIdx.x * 32 + lane;
    const uint32_t per = (blocks + 31) / 32;
    const uint32_t g0 = w * per;
    uint32_t v[kMaxRowsPerWarp], sum = 0;
#pragma unroll
    for (int j = 0; j < kMaxRowsPerWarp; ++j) {
        const uint32_t g = g0 + j;
        v[j] = (j < static_cast<int>(per) && g < blocks && b < kBins) ? counts[static_cast<uint64_t>(g) * kBins + b] : 0u;
        sum += v[j];
    }
    part[w][lane] = sum;
    __syncthreads();
    uint32_t run = 0;
    for (uint32_t k = 0; k < w; ++k) run += part[k][lane];
#pragma unroll
    for (int j = 0; j < kMaxRowsPerWarp; ++j) {
        const uint32_t g = g0 + j;
        if (j < static_cast<int>(per) && g < blocks && b < kBins) counts[static_cast<uint64_t>(g) * kBins + b] = run;
        run += v[j];
    }
    if (w == 31 && b < kBins) totals[b] = run;
}

// Exclusive scan of kBins counts in shared memory, in place, by a block of kOrderThreads threads: in
// chunks of kOrderThreads consecutive keys, one key per thread (conflict-free shared-memory access),
// each chunk's total carried into the next; returns the sum to every thread.
__device__ __forceinline__ uint32_t scan_bins(uint32_t* tot) {
    __shared__ uint32_t warp_sums[32];
    static_assert(kBins % kOrderThreads == 0 && kOrderThreads == 1024, "whole chunks of 32 warps");
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    uint32_t carry = 0;
    for (uint32_t c = 0; c < kBins / kOrderThreads; ++c) {
        const uint32_t idx = c * kOrderThreads + threadIdx.x;
        const uint32_t v = tot[idx];
        uint32_t x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
            if (lane >= static_cast<uint32_t>(o)) x += y;
        }
        if (lane == 31) warp_sums[warp] = x;
        __syncthreads();
        if (warp == 0) {
            uint32_t w = warp_sums[lane];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, w, o);
                if (lane >= static_cast<uint32_t>(o)) w += y;
            }
            warp_sums[lane] = w;
        }
        __syncthreads();
        tot[idx] = carry + (warp ? warp_sums[warp - 1] : 0u) + x - v;
        carry += warp_sums[31];
        __syncthreads();   // warp_sums is rewritten by the next chunk
    }
    return carry;
}

// Every block places its rays: order[p] = i and order[n + i] = p, p from the block's counters (the
// key's base plus the rays of that key in earlier blocks); a ray that misses gets no place
// (order[n + i] = kMiss).
__global__ void __launch_bounds__(kOrderThreads) k_order_scatter(const uint32_t* __restrict__ keys, uint32_t n,
                                                                const uint32_t* __restrict__ counts,
                                                                const uint32_t* __restrict__ totals,
                                                                uint32_t* __restrict__ order) {
    extern __shared__ uint32_t next[];
    // every block scans the key totals itself (128 KB from L2) for the keys' bases
    for (uint32_t b = threadIdx.x; b < kBins; b += blockDim.x) next[b] = totals[b];
    __syncthreads();
    const uint32_t traced = scan_bins(next);
    if (blockIdx.x == 0 && threadIdx.x == 0) order[2ull * n] = traced;   // every ray that meets the root box
    const uint32_t* mine = counts + static_cast<uint64_t>(blockIdx.x) * kBins;
    for (uint32_t b = threadIdx.x; b < kBins; b += blockDim.x) next[b] += mine[b];
    __syncthreads();
    uint32_t lo, hi;
    share(n, lo, hi);
    for (uint64_t base = lo + threadIdx.x; base < hi; base += kUnroll * blockDim.x) {
        uint32_t k[kUnroll];
#pragma unroll
        for (int j = 0; j < kUnroll; ++j) {
            const uint64_t i = base + static_cast<uint64_t>(j) * blockDim.x;
            k[j] = i < hi ? keys[i] : 0u;
        }
#pragma unroll
        for (int j = 0; j < kUnroll; ++j) {
            const uint64_t i = base + static_cast<uint64_t>(j) * blockDim.x;
            if (i < hi) {
                uint32_t p = kMiss;
                if (k[j] != kMiss) {
                    p = atomicAdd(next + k[j], 1u);
                    order[p] = static_cast<uint32_t>(i);
                }
                order[static_cast<uint64_t>(n) + i] = p;
            }
        }
    }
}

// hits[i] = ordered[inverse[i]]: the hits back at the rays' own places; a ray with no place (kMiss,
// or any place outside the batch) gets the record the traversal writes for a ray its root test
// rejects (t = +inf, SPT_MISS, u = v = 0).
__global__ void __launch_bounds__(256) k_order_gather(const spt_hit* __restrict__ ordered,
                                                      const uint32_t* __restrict__ inverse, uint32_t n,
                                                      spt_hit* __restrict__ hits) {
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t base = blockIdx.x * blockDim.x + threadIdx.x; base < n; base += kUnroll * stride) {
        float4 h[kUnroll];
#pragma unroll
        for (int j = 0; j < kUnroll; ++j) {
            const uint64_t i = base + static_cast<uint64_t>(j) * stride;
            if (i < n) {
                const uint32_t p = __ldg(inverse + i);
                h[j] = p < n ? __ldg(reinterpret_cast<const float4*>(ordered) + p)
                                  : make_float4(__int_as_float(0x7f800000), __uint_as_float(SPT_MISS), 0.0f, 0.0f);
            }
        }
#pragma unroll
        for (int j = 0; j < kUnroll; ++j) {
            const uint64_t i = base + static_cast<uint64_t>(j) * stride;
            if (i < n) __stcs(reinterpret_cast<float4*>(hits) + i, h[j]);
        }
    }
}

int order_blocks(spt_context* ctx) {
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
    return sms;   // one 1024-thread block with a 128 KB histogram per SM
}

}  // namespace

uint64_t order_min_rays() { return 1ull << 21; }

size_t order_scratch_bytes(spt_context* ctx) {
    return (static_cast<size_t>(order_blocks(ctx)) * kBins + kBins) * sizeof(uint32_t);
}

spt_status order_rays(spt_context* ctx, const spt_scene* sc, const float* d_rays, uint64_t n, int stride,
                      cudaStream_t s, uint32_t* keys, uint32_t* work, uint32_t* order) {
    // the histograms' shared memory (above the default 48 KB), set on the context's device each call
    SPT_CUDA(ctx, cudaFuncSetAttribute(stride == 6 ? k_order_count<6> : k_order_count<8>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(kOrderSmem)));
    SPT_CUDA(ctx, cudaFuncSetAttribute(k_order_scatter, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(kOrderSmem)));
    const uint32_t n32 = static_cast<uint32_t>(n);
    const int blocks = order_blocks(ctx);
    if (blocks > 32 * kMaxRowsPerWarp) return fail(ctx, SPT_ERR_UNSUPPORTED, "more SMs than the ray order supports");
    uint32_t* counts = work;
    uint32_t* totals = work + static_cast<size_t>(blocks) * kBins;
    if (stride == 6)
        k_order_count<6><<<blocks, kOrderThreads, kOrderSmem, s>>>(sc->dev, d_rays, n32, keys, counts);
    else
        k_order_count<8><<<blocks, kOrderThreads, kOrderSmem, s>>>(sc->dev, d_rays, n32, keys, counts);
    k_order_offsets<<<(kBins + 31) / 32, 1024, 0, s>>>(counts, static_cast<uint32_t>(blocks), totals);
    k_order_scatter<<<blocks, kOrderThreads, kOrderSmem, s>>>(keys, n32, counts, totals, order);
    SPT_CUDA(ctx, cudaGetLastError());
    return SPT_OK;
}

spt_status unorder_hits(spt_context* ctx, const spt_hit* ordered, const uint32_t* order, uint64_t n, spt_hit* hits,
                        cudaStream_t s) {
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
    const unsigned g = static_cast<unsigned>(std::min<uint64_t>((n + 255) / 256, 16ull * sms));
    k_order_gather<<<g, 256, 0, s>>>(ordered, order + n, static_cast<uint32_t>(n), hits);
    SPT_CUDA(ctx, cudaGetLastError());
    return SPT_OK;
}

}  // namespace spt
