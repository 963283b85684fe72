// bvh_gpu.cu -- binary BVH built on the device, for scenes that do not need the reference's own tree.
//
// The reference builds its tree with a full SAH sweep on one host thread (acceleration/sbvh.cpp:12-37,
// 58-421).  build_sah_tree reproduces that tree exactly, which the bit-exact hit counts and equal-t tie
// breaks need, but it takes about a second at 1.3M triangles.  This builder makes a tree of similar
// quality in milliseconds:
//
//  1. primitive boxes and centroids as the reference computes them (bvh_build.cpp: prim_bounds);
//  2. 63-bit Morton codes of the centroids (21 bits per axis over the centroid bounds), radix-sorted;
//  3. Parallel Locally-Ordered Clustering (D. Meister and J. Bittner, "Parallel Locally-Ordered
//     Clustering for Bounding Volume Hierarchy Construction", IEEE TVCG 2018): every cluster finds
//     the cluster within kRadius positions of it in Morton order whose union box has the smallest
//     surface area; mutual nearest neighbours merge; the array is compacted; repeat until one is left;
//  4. a bottom-up SAH pass with the reference's constants (a node costs 2 x 1.2 plus its
//     children's costs weighted by area ratio; a leaf costs 1 per primitive) turns each subtree that
//     is cheaper as one leaf into a leaf of at most kMaxLeaf primitives;
//  5. the depth-first, left-first layout and box rule of the reference's tree: the root box is the
//     union of the primitive boxes, every other box is its primitives' union inflated by 1e-3
//     (sbvh.cpp:409-412).  The traversals' exactness argument needs only that rule.
//
// Closest hits over this tree equal those over the reference's tree except where two primitives are
// hit at the same t: the tie goes to the earlier primitive in this tree's depth-first leaf order.  Hit
// counts (the reference's exhaustive traversal) are this tree's counts, not the reference's.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <vector>

#include "bvh_build.h"
#include "spt_internal.h"

namespace spt {
namespace {

constexpr int kRadius = 16;        // PLOC search radius (positions on each side)
constexpr int kTile = 256;         // clusters per block of the neighbour search
// Primitives per collapsed leaf.  The 8-wide collapse packs up to three per child slot anyway, and
// on the 1.31M-triangle mesh small leaves traverse fastest: 2,584 Mrays/s at 1, 2,528 at 2, 2,463 at
// 3, 2,259 at 8 (the reference's own tree: 2,689).  At 1 the tree has twice the nodes, and the host
// side of scene creation (the 8-wide collapse) takes 1.06 s instead of 0.58 s.
constexpr uint32_t kMaxLeaf = 2;

// glm::min / glm::max as the reference uses them (aabb.h)
__device__ __forceinline__ float gmin_d(float x, float y) { return (y < x) ? y : x; }
__device__ __forceinline__ float gmax_d(float x, float y) { return (x < y) ? y : x; }

// AABB::getArea (aabb.cpp:11-16)
__device__ __forceinline__ float area_d(float4 mn, float4 mx) {
    const float l = mx.x - mn.x, m = mx.y - mn.y, n = mx.z - mn.z;
    return 2.0f * (l * (m + n) + m * n);
}

// float <-> unsigned with the same order (for atomicMin / atomicMax on float bounds)
__device__ __forceinline__ uint32_t ordered(float f) {
    const uint32_t b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float unordered(uint32_t u) {
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7FFFFFFFu) : ~u);
}

// Primitive boxes and centroids (bvh_build.cpp: prim_bounds, the reference's Triangle/Sphere
// getAABB and getCentroid), and the centroid bounds as ordered integers: cb[0..2] min, cb[3..5] max.
__global__ void k_prim_boxes(const float* __restrict__ prim, const uint8_t* __restrict__ type, uint32_t n,
                             float4* __restrict__ bmin, float4* __restrict__ bmax, float4* __restrict__ cen,
                             uint32_t* __restrict__ cb) {
    uint32_t lo[3] = {0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu}, hi[3] = {0u, 0u, 0u};
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float* p = prim + 9ull * i;
        float mn[3], mx[3], c[3];
        if (type[i] == SPT_PRIM_SPHERE) {
            for (int k = 0; k < 3; ++k) {
                mn[k] = p[k] - p[3];
                mx[k] = p[k] + p[3];
                c[k] = p[k];
            }
        } else {
            for (int k = 0; k < 3; ++k) {
                mn[k] = gmin_d(gmin_d(p[k], p[3 + k]), p[6 + k]);
                mx[k] = gmax_d(gmax_d(p[k], p[3 + k]), p[6 + k]);
                c[k] = ((p[k] + p[3 + k]) + p[6 + k]) * (1.0f / 3.0f);
            }
        }
        bmin[i] = make_float4(mn[0], mn[1], mn[2], 0.0f);
        bmax[i] = make_float4(mx[0], mx[1], mx[2], 0.0f);
        cen[i] = make_float4(c[0], c[1], c[2], 0.0f);
        for (int k = 0; k < 3; ++k) {
            lo[k] = min(lo[k], ordered(c[k]));
            hi[k] = max(hi[k], ordered(c[k]));
        }
    }
    for (int k = 0; k < 3; ++k) {
        for (int off = 16; off; off >>= 1) {
            lo[k] = min(lo[k], __shfl_xor_sync(0xFFFFFFFFu, lo[k], off));
            hi[k] = max(hi[k], __shfl_xor_sync(0xFFFFFFFFu, hi[k], off));
        }
    }
    if ((threadIdx.x & 31) == 0) {
        for (int k = 0; k < 3; ++k) {
            atomicMin(cb + k, lo[k]);
            atomicMax(cb + 3 + k, hi[k]);
        }
    }
}

// 21 bits of x spread to every third bit
__device__ __forceinline__ uint64_t spread21(uint32_t x) {
    uint64_t v = x & 0x1FFFFFu;
    v = (v | (v << 32)) & 0x1F00000000FFFFull;
    v = (v | (v << 16)) & 0x1F0000FF0000FFull;
    v = (v | (v << 8)) & 0x100F00F00F00F00Full;
    v = (v | (v << 4)) & 0x10C30C30C30C30C3ull;
    v = (v | (v << 2)) & 0x1249249249249249ull;
    return v;
}

__global__ void k_morton(const float4* __restrict__ cen, uint32_t n, const uint32_t* __restrict__ cb,
                         uint64_t* __restrict__ keys, uint32_t* __restrict__ vals) {
    float lo[3], scale[3];
    for (int k = 0; k < 3; ++k) {
        lo[k] = unordered(cb[k]);
        const float ext = unordered(cb[3 + k]) - lo[k];
        scale[k] = ext > 0.0f ? 2097151.0f / ext : 0.0f;
    }
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 c = cen[i];
        const float q[3] = {c.x, c.y, c.z};
        uint64_t key = 0;
        for (int k = 0; k < 3; ++k) {
            const float f = fminf(fmaxf((q[k] - lo[k]) * scale[k], 0.0f), 2097151.0f);
            key |= spread21(static_cast<uint32_t>(f)) << (2 - k);
        }
        keys[i] = key;
        vals[i] = i;
    }
}

// Node store: boxes as two float4, children as int2 (leaf: x = -1, y = primitive id).
struct Nodes {
    float4* mn;
    float4* mx;
    int2* child;
};

// Per-node state of the collapse (bottom-up) and of the depth-first layout (top-down).
struct Tree {
    uint32_t* cnt;       // primitives below
    float* cost;         // SAH cost of the subtree as emitted
    uint8_t* col;        // emitted as one leaf
    uint32_t* outsize;   // output nodes the subtree emits
    uint32_t* idx;       // output index (emitted nodes)
    uint32_t* rb;        // offset of the subtree's first primitive in the reference list
    uint8_t* state;      // 1: emitted inner node, 2: emitted leaf, 0: inside an emitted leaf
};

__global__ void k_leaves(const uint32_t* __restrict__ order, uint32_t n, const float4* __restrict__ bmin,
                         const float4* __restrict__ bmax, Nodes N, Tree T, uint32_t* __restrict__ cur) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t p = order[i];
        N.mn[i] = bmin[p];
        N.mx[i] = bmax[p];
        N.child[i] = make_int2(-1, static_cast<int>(p));
        T.cnt[i] = 1u;
        T.cost[i] = 1.0f;
        T.col[i] = 1u;
        T.outsize[i] = 1u;
        cur[i] = i;
    }
}

// nn[i]: the cluster within kRadius positions of i whose union box with i has the smallest area, from
// a shared-memory copy of the tile and its halo.  Candidates are ranked by the key (area, |i - j|,
// min(i, j) & 1, min(i, j)), which is symmetric in i and j and a strict order on pairs, so the
// globally smallest pair is always mutual and every pass merges.  On equal areas (coincident
// primitives) it pairs neighbours (2k, 2k + 1), which halves the array instead of merging one pair
// per pass.
__global__ void __launch_bounds__(kTile) k_nearest(const uint32_t* __restrict__ cur, uint32_t m, Nodes N,
                                                    uint32_t* __restrict__ nn) {
    __shared__ float4 smn[kTile + 2 * kRadius], smx[kTile + 2 * kRadius];
    const int64_t base = static_cast<int64_t>(blockIdx.x) * kTile - kRadius;
    for (int t = threadIdx.x; t < kTile + 2 * kRadius; t += blockDim.x) {
        const int64_t g = base + t;
        if (g >= 0 && g < static_cast<int64_t>(m)) {
            const uint32_t c = cur[g];
            smn[t] = N.mn[c];
            smx[t] = N.mx[c];
        }
    }
    __syncthreads();
    const int64_t i = static_cast<int64_t>(blockIdx.x) * kTile + threadIdx.x;
    if (i >= static_cast<int64_t>(m)) return;
    const int li = threadIdx.x + kRadius;
    const float4 amn = smn[li], amx = smx[li];
    float best = __int_as_float(0x7F800000);
    int bd = 0, bp = 0;
    int64_t bj = i;
    for (int off = -kRadius; off <= kRadius; ++off) {
        const int64_t j = i + off;
        if (off == 0 || j < 0 || j >= static_cast<int64_t>(m)) continue;
        const float4 bmn = smn[li + off], bmx = smx[li + off];
        const float4 umn = make_float4(gmin_d(amn.x, bmn.x), gmin_d(amn.y, bmn.y), gmin_d(amn.z, bmn.z), 0.0f);
        const float4 umx = make_float4(gmax_d(amx.x, bmx.x), gmax_d(amx.y, bmx.y), gmax_d(amx.z, bmx.z), 0.0f);
        const float a = area_d(umn, umx);
        const int d = off < 0 ? -off : off;
        const int p = static_cast<int>((j < i ? j : i) & 1);
        // scanning j upwards, so on an equal (area, distance, parity) the lower j is already kept
        const bool better = a < best || (a == best && (d < bd || (d == bd && p < bp)));
        if (bj == i || better) {
            best = a;
            bd = d;
            bp = p;
            bj = j;
        }
    }
    nn[i] = static_cast<uint32_t>(bj);
}

// Mutual nearest neighbours i < j merge into a new node kept at i; j leaves the array.
__global__ void k_merge(const uint32_t* __restrict__ cur, uint32_t m, const uint32_t* __restrict__ nn, Nodes N,
                        uint32_t* __restrict__ alloc, uint32_t* __restrict__ next, uint32_t* __restrict__ keep) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
        const uint32_t j = nn[i];
        const bool mutual = j != i && nn[j] == i;
        if (mutual && i > j) {
            keep[i] = 0u;
            continue;
        }
        keep[i] = 1u;
        if (!mutual) {
            next[i] = cur[i];
            continue;
        }
        const uint32_t a = cur[i], b = cur[j];
        const uint32_t k = atomicAdd(alloc, 1u);
        const float4 amn = N.mn[a], amx = N.mx[a], bmn = N.mn[b], bmx = N.mx[b];
        N.mn[k] = make_float4(gmin_d(amn.x, bmn.x), gmin_d(amn.y, bmn.y), gmin_d(amn.z, bmn.z), 0.0f);
        N.mx[k] = make_float4(gmax_d(amx.x, bmx.x), gmax_d(amx.y, bmx.y), gmax_d(amx.z, bmx.z), 0.0f);
        N.child[k] = make_int2(static_cast<int>(a), static_cast<int>(b));
        next[i] = k;
    }
}

__global__ void k_compact(const uint32_t* __restrict__ next, const uint32_t* __restrict__ keep,
                          const uint32_t* __restrict__ pos, uint32_t m, uint32_t* __restrict__ out,
                          uint32_t* __restrict__ count) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
        if (keep[i]) out[pos[i]] = next[i];
        if (i == m - 1) *count = pos[i] + keep[i];
    }
}

// The nodes one clustering pass made, whose children all come from earlier passes: primitive count,
// SAH cost with the reference's constants (a node 2 x 1.2 plus its children's costs weighted by area
// ratio, a leaf 1 per primitive), and whether the subtree is emitted as one leaf (at most kMaxLeaf
// primitives, and no costlier than splitting).
__global__ void k_up(Nodes N, Tree T, uint32_t a, uint32_t b) {
    for (uint32_t v = a + blockIdx.x * blockDim.x + threadIdx.x; v < b; v += gridDim.x * blockDim.x) {
        const int2 c = N.child[v];
        const uint32_t l = static_cast<uint32_t>(c.x), r = static_cast<uint32_t>(c.y);
        const uint32_t cnt = T.cnt[l] + T.cnt[r];
        const float av = area_d(N.mn[v], N.mx[v]);
        const float al = area_d(N.mn[l], N.mx[l]), ar = area_d(N.mn[r], N.mx[r]);
        const float split = av > 0.0f ? 2.0f * 1.2f + (al / av) * T.cost[l] + (ar / av) * T.cost[r]
                                      : 2.0f * 1.2f + T.cost[l] + T.cost[r];
        const float leaf = static_cast<float>(cnt);
        const bool col = cnt <= kMaxLeaf && leaf <= split;
        T.cnt[v] = cnt;
        T.cost[v] = col ? leaf : split;
        T.col[v] = col ? 1u : 0u;
        T.outsize[v] = col ? 1u : 1u + T.outsize[l] + T.outsize[r];
    }
}

__global__ void k_root(Tree T, const uint32_t* __restrict__ cur) {
    const uint32_t r = cur[0];
    T.idx[r] = 0u;
    T.rb[r] = 0u;
    T.state[r] = T.col[r] ? 2u : 1u;
}

// One output node in the reference's layout; every box but the root's is inflated by 1e-3.
__device__ __forceinline__ void write_node(spt_bvh2_node* out, uint32_t i, float4 mn, float4 mx, uint32_t right,
                                           uint32_t count) {
    float4* o = reinterpret_cast<float4*>(out + i);
    if (i == 0) {
        o[0] = make_float4(mn.x, mn.y, mn.z, __uint_as_float(right));
        o[1] = make_float4(mx.x, mx.y, mx.z, __uint_as_float(count));
    } else {
        o[0] = make_float4(mn.x - 1e-3f, mn.y - 1e-3f, mn.z - 1e-3f, __uint_as_float(right));
        o[1] = make_float4(mx.x + 1e-3f, mx.y + 1e-3f, mx.z + 1e-3f, __uint_as_float(count));
    }
}

// The nodes of one pass, after every later pass (their parents): hand the children their output
// index (left right after the parent, right after the left subtree) and reference offset, and write
// the emitted nodes.
__global__ void k_down(Nodes N, Tree T, uint32_t a, uint32_t b, spt_bvh2_node* __restrict__ out) {
    for (uint32_t v = a + blockIdx.x * blockDim.x + threadIdx.x; v < b; v += gridDim.x * blockDim.x) {
        const int2 c = N.child[v];
        const uint32_t l = static_cast<uint32_t>(c.x), r = static_cast<uint32_t>(c.y);
        const uint8_t st = T.state[v];
        const uint32_t r0 = T.rb[v];
        T.rb[l] = r0;
        T.rb[r] = r0 + T.cnt[l];
        if (st == 1u) {
            const uint32_t i0 = T.idx[v];
            const uint32_t ir = i0 + 1u + T.outsize[l];
            T.idx[l] = i0 + 1u;
            T.idx[r] = ir;
            T.state[l] = T.col[l] ? 2u : 1u;
            T.state[r] = T.col[r] ? 2u : 1u;
            write_node(out, i0, N.mn[v], N.mx[v], ir, 0u);
        } else {
            T.state[l] = 0u;
            T.state[r] = 0u;
            if (st == 2u) write_node(out, T.idx[v], N.mn[v], N.mx[v], r0, T.cnt[v]);
        }
    }
}

__global__ void k_down_leaves(Nodes N, Tree T, uint32_t n, uint32_t* __restrict__ refs,
                              spt_bvh2_node* __restrict__ out) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        refs[T.rb[i]] = static_cast<uint32_t>(N.child[i].y);
        if (T.state[i] == 2u) write_node(out, T.idx[i], N.mn[i], N.mx[i], T.rb[i], 1u);
    }
}

// Bump layout of one build's buffers in one region, 256-byte aligned.  A pass with base 0 only sizes
// the region.
struct Bump {
    uintptr_t base;
    size_t off = 0;
    template <typename T>
    void take(T** p, size_t count) {
        off = (off + 255) & ~static_cast<size_t>(255);
        *p = reinterpret_cast<T*>(base + off);
        off += std::max<size_t>(count, 1) * sizeof(T);
    }
};

// The context's scratch slot that holds a build's buffers; it stays allocated, so later builds of
// no larger scenes allocate nothing (scenes of a batch are often built back to back).
constexpr int kBuildSlot = 10;

}  // namespace

spt_status build_ploc_tree(spt_context* ctx, const spt_scene_desc& d, HostBvh& out) {
    const auto t0 = std::chrono::steady_clock::now();
    out.nodes.clear();
    out.refs.clear();
    std::memset(&out.stats, 0, sizeof(out.stats));
    const uint32_t n = d.n_prims;
    if (n == 0) return SPT_OK;
    if (n > (1u << 30)) return fail(ctx, SPT_ERR_INVALID_ARGUMENT, "device BVH build: at most 2^30 primitives");
    cudaStream_t s = ctx->stream;
    float* prim;
    uint8_t* type;
    float4 *bmin, *bmax, *cen;
    uint32_t *cb, *vals, *vals2, *cur, *cur2, *nn, *next, *keep, *pos, *counters, *d_refs;
    uint64_t *keys, *keys2;
    spt_bvh2_node* d_out;
    char* temp;
    Nodes N;
    Tree T;
    const size_t n_nodes = 2ull * n - 1;
    // sort and scan scratch, sized for the largest call
    size_t sort_bytes = 0, scan_bytes = 0;
    SPT_CUDA(ctx, cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, static_cast<const uint64_t*>(nullptr),
                                                  static_cast<uint64_t*>(nullptr), static_cast<const uint32_t*>(nullptr),
                                                  static_cast<uint32_t*>(nullptr), static_cast<int>(n), 0, 63, s));
    SPT_CUDA(ctx, cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, static_cast<const uint32_t*>(nullptr),
                                                static_cast<uint32_t*>(nullptr), static_cast<int>(n), s));
    auto layout = [&](Bump& B) {
        B.take(&prim, 9ull * n);
        B.take(&type, n);
        B.take(&bmin, n);
        B.take(&bmax, n);
        B.take(&cen, n);
        B.take(&cb, 8);
        B.take(&keys, n);
        B.take(&keys2, n);
        B.take(&vals, n);
        B.take(&vals2, n);
        B.take(&cur, n);
        B.take(&cur2, n);
        B.take(&nn, n);
        B.take(&next, n);
        B.take(&keep, n);
        B.take(&pos, n);
        B.take(&counters, 2);
        B.take(&N.mn, n_nodes);
        B.take(&N.mx, n_nodes);
        B.take(&N.child, n_nodes);
        B.take(&T.cnt, n_nodes);
        B.take(&T.cost, n_nodes);
        B.take(&T.col, n_nodes);
        B.take(&T.outsize, n_nodes);
        B.take(&T.idx, n_nodes);
        B.take(&T.rb, n_nodes);
        B.take(&T.state, n_nodes);
        B.take(&d_out, n_nodes);
        B.take(&d_refs, n);
        B.take(&temp, std::max(sort_bytes, scan_bytes));
    };
    Bump sizing{0};
    layout(sizing);
    void* region;
    spt_status st = scratch(ctx, kBuildSlot, sizing.off, &region);
    if (st != SPT_OK) return st;
    Bump real{reinterpret_cast<uintptr_t>(region)};
    layout(real);

    SPT_CUDA(ctx, cudaMemcpyAsync(prim, d.prim_data, 9ull * n * sizeof(float), cudaMemcpyHostToDevice, s));
    SPT_CUDA(ctx, cudaMemcpyAsync(type, d.prim_type, n, cudaMemcpyHostToDevice, s));
    const uint32_t init[8] = {0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0u, 0u, 0u, 0u, 0u};
    SPT_CUDA(ctx, cudaMemcpyAsync(cb, init, sizeof(init), cudaMemcpyHostToDevice, s));
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
    const unsigned grid = static_cast<unsigned>(std::min<uint64_t>((n + 255) / 256, 8ull * sms));
    k_prim_boxes<<<grid, 256, 0, s>>>(prim, type, n, bmin, bmax, cen, cb);
    k_morton<<<grid, 256, 0, s>>>(cen, n, cb, keys, vals);
    size_t tb = std::max(sort_bytes, scan_bytes);
    SPT_CUDA(ctx, cub::DeviceRadixSort::SortPairs(temp, tb, keys, keys2, vals, vals2, static_cast<int>(n), 0, 63, s));
    k_leaves<<<grid, 256, 0, s>>>(vals2, n, bmin, bmax, N, T, cur);
    SPT_CUDA(ctx, cudaGetLastError());
    SPT_CUDA(ctx, cudaMemcpyAsync(counters, &n, sizeof(n), cudaMemcpyHostToDevice, s));  // next free node

    // clustering: every pass merges at least the globally closest mutual pair, so it ends
    uint32_t m = n;
    uint32_t passes = 0;
    uint32_t* h_count;
    if ((st = pinned(ctx, 2 * sizeof(uint32_t), reinterpret_cast<void**>(&h_count))) != SPT_OK) return st;
    std::vector<uint32_t> bounds{n};   // node ids created by pass p: [bounds[p], bounds[p + 1])
    while (m > 1) {
        if (++passes > n) return fail(ctx, SPT_ERR_INTERNAL, "device BVH build did not converge");
        const unsigned gm = static_cast<unsigned>(std::min<uint64_t>((m + 255) / 256, 8ull * sms));
        k_nearest<<<(m + kTile - 1) / kTile, kTile, 0, s>>>(cur, m, N, nn);
        k_merge<<<gm, 256, 0, s>>>(cur, m, nn, N, counters, next, keep);
        tb = std::max(sort_bytes, scan_bytes);
        SPT_CUDA(ctx, cub::DeviceScan::ExclusiveSum(temp, tb, keep, pos, static_cast<int>(m), s));
        k_compact<<<gm, 256, 0, s>>>(next, keep, pos, m, cur2, counters + 1);
        SPT_CUDA(ctx, cudaGetLastError());
        SPT_CUDA(ctx, cudaMemcpyAsync(h_count, counters, 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
        SPT_CUDA(ctx, cudaStreamSynchronize(s));
        if (h_count[1] >= m) return fail(ctx, SPT_ERR_INTERNAL, "device BVH build made no progress");
        m = h_count[1];
        bounds.push_back(h_count[0]);
        std::swap(cur, cur2);
    }
    // bottom-up over the passes in creation order (children before parents): counts, SAH costs,
    // collapse flags, emitted sizes; then top-down in reverse: output indices, reference offsets,
    // output nodes and the reference list
    uint32_t root = 0;
    SPT_CUDA(ctx, cudaMemcpyAsync(&root, cur, sizeof(root), cudaMemcpyDeviceToHost, s));
    for (size_t p = 0; p + 1 < bounds.size(); ++p) {
        const uint32_t a = bounds[p], b = bounds[p + 1];
        k_up<<<static_cast<unsigned>(std::min<uint64_t>((b - a + 255) / 256, 8ull * sms)), 256, 0, s>>>(N, T, a, b);
    }
    k_root<<<1, 1, 0, s>>>(T, cur);
    uint32_t n_out = 0;
    SPT_CUDA(ctx, cudaMemcpyAsync(&n_out, T.outsize + root, sizeof(n_out), cudaMemcpyDeviceToHost, s));
    SPT_CUDA(ctx, cudaStreamSynchronize(s));
    if (n_out == 0 || n_out > n_nodes) return fail(ctx, SPT_ERR_INTERNAL, "device BVH build: bad node count");
    for (size_t p = bounds.size() - 1; p-- > 0;) {
        const uint32_t a = bounds[p], b = bounds[p + 1];
        k_down<<<static_cast<unsigned>(std::min<uint64_t>((b - a + 255) / 256, 8ull * sms)), 256, 0, s>>>(N, T, a, b,
                                                                                                         d_out);
    }
    k_down_leaves<<<grid, 256, 0, s>>>(N, T, n, d_refs, d_out);
    SPT_CUDA(ctx, cudaGetLastError());
    out.nodes.resize(n_out);
    out.refs.resize(n);
    SPT_CUDA(ctx, cudaMemcpyAsync(out.nodes.data(), d_out, n_out * sizeof(spt_bvh2_node), cudaMemcpyDeviceToHost, s));
    SPT_CUDA(ctx, cudaMemcpyAsync(out.refs.data(), d_refs, n * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    SPT_CUDA(ctx, cudaStreamSynchronize(s));
    if (out.refs.size() != n) return fail(ctx, SPT_ERR_INTERNAL, "device BVH build lost primitives");
    tree_statistics(out);
    out.stats.build_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return SPT_OK;
}

}  // namespace spt
