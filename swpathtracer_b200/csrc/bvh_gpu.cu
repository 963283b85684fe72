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
//  4. on the host, a bottom-up SAH pass with the reference's constants (a node costs 2 x 1.2 plus its
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
constexpr uint32_t kMaxLeaf = 8;   // primitives per collapsed leaf

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

__global__ void k_leaves(const uint32_t* __restrict__ order, uint32_t n, const float4* __restrict__ bmin,
                         const float4* __restrict__ bmax, Nodes N, uint32_t* __restrict__ cur) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t p = order[i];
        N.mn[i] = bmin[p];
        N.mx[i] = bmax[p];
        N.child[i] = make_int2(-1, static_cast<int>(p));
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

// Device buffers of one build, freed on every exit path.
struct Scratch {
    std::vector<void*> ptrs;
    ~Scratch() {
        for (void* p : ptrs) cudaFree(p);
    }
    template <typename T>
    cudaError_t get(T** p, size_t count) {
        void* q = nullptr;
        const cudaError_t e = cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(T));
        if (e == cudaSuccess) ptrs.push_back(q);
        *p = static_cast<T*>(q);
        return e;
    }
};

float area_h(const float mn[3], const float mx[3]) {
    const float l = mx[0] - mn[0], m = mx[1] - mn[1], n = mx[2] - mn[2];
    return 2.0f * (l * (m + n) + m * n);
}

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
    Scratch S;
    float* prim;
    uint8_t* type;
    float4 *bmin, *bmax, *cen;
    uint32_t *cb, *vals, *vals2, *cur, *cur2, *nn, *next, *keep, *pos, *counters;
    uint64_t *keys, *keys2;
    Nodes N;
    const size_t n_nodes = 2ull * n - 1;
    SPT_CUDA(ctx, S.get(&prim, 9ull * n));
    SPT_CUDA(ctx, S.get(&type, n));
    SPT_CUDA(ctx, S.get(&bmin, n));
    SPT_CUDA(ctx, S.get(&bmax, n));
    SPT_CUDA(ctx, S.get(&cen, n));
    SPT_CUDA(ctx, S.get(&cb, 8));
    SPT_CUDA(ctx, S.get(&keys, n));
    SPT_CUDA(ctx, S.get(&keys2, n));
    SPT_CUDA(ctx, S.get(&vals, n));
    SPT_CUDA(ctx, S.get(&vals2, n));
    SPT_CUDA(ctx, S.get(&cur, n));
    SPT_CUDA(ctx, S.get(&cur2, n));
    SPT_CUDA(ctx, S.get(&nn, n));
    SPT_CUDA(ctx, S.get(&next, n));
    SPT_CUDA(ctx, S.get(&keep, n));
    SPT_CUDA(ctx, S.get(&pos, n));
    SPT_CUDA(ctx, S.get(&counters, 2));
    SPT_CUDA(ctx, S.get(&N.mn, n_nodes));
    SPT_CUDA(ctx, S.get(&N.mx, n_nodes));
    SPT_CUDA(ctx, S.get(&N.child, n_nodes));
    // sort and scan scratch, sized for the largest call
    size_t sort_bytes = 0, scan_bytes = 0;
    SPT_CUDA(ctx, cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, keys, keys2, vals, vals2,
                                                  static_cast<int>(n), 0, 63, s));
    SPT_CUDA(ctx, cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, keep, pos, static_cast<int>(n), s));
    void* temp;
    SPT_CUDA(ctx, S.get(reinterpret_cast<char**>(&temp), std::max(sort_bytes, scan_bytes)));

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
    k_leaves<<<grid, 256, 0, s>>>(vals2, n, bmin, bmax, N, cur);
    SPT_CUDA(ctx, cudaGetLastError());
    SPT_CUDA(ctx, cudaMemcpyAsync(counters, &n, sizeof(n), cudaMemcpyHostToDevice, s));  // next free node

    // clustering: every pass merges at least the globally closest mutual pair, so it ends
    uint32_t m = n;
    uint32_t passes = 0;
    uint32_t* h_count;
    SPT_CUDA(ctx, cudaMallocHost(&h_count, sizeof(uint32_t)));
    struct PinnedFree {
        uint32_t* p;
        ~PinnedFree() { cudaFreeHost(p); }
    } pin{h_count};
    while (m > 1) {
        if (++passes > n) return fail(ctx, SPT_ERR_INTERNAL, "device BVH build did not converge");
        const unsigned gm = static_cast<unsigned>(std::min<uint64_t>((m + 255) / 256, 8ull * sms));
        k_nearest<<<(m + kTile - 1) / kTile, kTile, 0, s>>>(cur, m, N, nn);
        k_merge<<<gm, 256, 0, s>>>(cur, m, nn, N, counters, next, keep);
        tb = std::max(sort_bytes, scan_bytes);
        SPT_CUDA(ctx, cub::DeviceScan::ExclusiveSum(temp, tb, keep, pos, static_cast<int>(m), s));
        k_compact<<<gm, 256, 0, s>>>(next, keep, pos, m, cur2, counters + 1);
        SPT_CUDA(ctx, cudaGetLastError());
        SPT_CUDA(ctx, cudaMemcpyAsync(h_count, counters + 1, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
        SPT_CUDA(ctx, cudaStreamSynchronize(s));
        if (*h_count >= m) return fail(ctx, SPT_ERR_INTERNAL, "device BVH build made no progress");
        m = *h_count;
        std::swap(cur, cur2);
    }
    uint32_t root = 0;
    SPT_CUDA(ctx, cudaMemcpyAsync(&root, cur, sizeof(root), cudaMemcpyDeviceToHost, s));
    std::vector<float4> hmn(n_nodes), hmx(n_nodes);
    std::vector<int2> hch(n_nodes);
    SPT_CUDA(ctx, cudaMemcpyAsync(hmn.data(), N.mn, n_nodes * sizeof(float4), cudaMemcpyDeviceToHost, s));
    SPT_CUDA(ctx, cudaMemcpyAsync(hmx.data(), N.mx, n_nodes * sizeof(float4), cudaMemcpyDeviceToHost, s));
    SPT_CUDA(ctx, cudaMemcpyAsync(hch.data(), N.child, n_nodes * sizeof(int2), cudaMemcpyDeviceToHost, s));
    SPT_CUDA(ctx, cudaStreamSynchronize(s));

    // bottom-up: primitive counts and SAH costs; collapse[v] marks subtrees emitted as one leaf
    std::vector<uint32_t> cnt(n_nodes, 1);
    std::vector<float> cost(n_nodes, 1.0f);
    std::vector<uint8_t> collapse(n_nodes, 1);
    {
        std::vector<uint32_t> st{root}, post;
        post.reserve(n_nodes);
        while (!st.empty()) {   // children before parents: reverse of a pre-order with right pushed last
            const uint32_t v = st.back();
            st.pop_back();
            post.push_back(v);
            if (hch[v].x >= 0) {
                st.push_back(static_cast<uint32_t>(hch[v].x));
                st.push_back(static_cast<uint32_t>(hch[v].y));
            }
        }
        for (size_t k = post.size(); k-- > 0;) {
            const uint32_t v = post[k];
            if (hch[v].x < 0) continue;
            const uint32_t a = static_cast<uint32_t>(hch[v].x), b = static_cast<uint32_t>(hch[v].y);
            cnt[v] = cnt[a] + cnt[b];
            const float mn[3] = {hmn[v].x, hmn[v].y, hmn[v].z}, mx[3] = {hmx[v].x, hmx[v].y, hmx[v].z};
            const float amn[3] = {hmn[a].x, hmn[a].y, hmn[a].z}, amx[3] = {hmx[a].x, hmx[a].y, hmx[a].z};
            const float bmn_[3] = {hmn[b].x, hmn[b].y, hmn[b].z}, bmx_[3] = {hmx[b].x, hmx[b].y, hmx[b].z};
            const float av = area_h(mn, mx);
            const float split = av > 0.0f ? 2.0f * 1.2f + (area_h(amn, amx) / av) * cost[a] + (area_h(bmn_, bmx_) / av) * cost[b]
                                          : 2.0f * 1.2f + cost[a] + cost[b];
            const float leaf = static_cast<float>(cnt[v]);
            collapse[v] = (cnt[v] <= kMaxLeaf && leaf <= split) ? 1 : 0;
            cost[v] = collapse[v] ? leaf : split;
        }
    }
    // depth-first, left-first flatten with the reference's box rule
    out.nodes.reserve(n_nodes);
    out.refs.reserve(n);
    struct Item {
        uint32_t v;
        int64_t parent;   // output index whose .right this node's index fills (-1: none)
    };
    std::vector<Item> st{{root, -1}};
    std::vector<uint32_t> sub;
    while (!st.empty()) {
        const Item it = st.back();
        st.pop_back();
        const uint32_t idx = static_cast<uint32_t>(out.nodes.size());
        if (it.parent >= 0) out.nodes[static_cast<size_t>(it.parent)].right = idx;
        spt_bvh2_node o{};
        const float4 a = hmn[it.v], b = hmx[it.v];
        const float inf = idx == 0 ? 0.0f : 1e-3f;
        o.min[0] = idx == 0 ? a.x : a.x - inf;
        o.min[1] = idx == 0 ? a.y : a.y - inf;
        o.min[2] = idx == 0 ? a.z : a.z - inf;
        o.max[0] = idx == 0 ? b.x : b.x + inf;
        o.max[1] = idx == 0 ? b.y : b.y + inf;
        o.max[2] = idx == 0 ? b.z : b.z + inf;
        if (collapse[it.v]) {
            o.right = static_cast<uint32_t>(out.refs.size());
            o.count = cnt[it.v];
            sub.assign(1, it.v);   // the subtree's primitives, left to right
            while (!sub.empty()) {
                const uint32_t u = sub.back();
                sub.pop_back();
                if (hch[u].x < 0) {
                    out.refs.push_back(static_cast<uint32_t>(hch[u].y));
                } else {
                    sub.push_back(static_cast<uint32_t>(hch[u].y));
                    sub.push_back(static_cast<uint32_t>(hch[u].x));
                }
            }
            out.nodes.push_back(o);
        } else {
            o.count = 0;
            out.nodes.push_back(o);
            st.push_back(Item{static_cast<uint32_t>(hch[it.v].y), static_cast<int64_t>(idx)});   // right, filled later
            st.push_back(Item{static_cast<uint32_t>(hch[it.v].x), -1});                          // left = idx + 1
        }
    }
    if (out.refs.size() != n) return fail(ctx, SPT_ERR_INTERNAL, "device BVH build lost primitives");
    tree_statistics(out);
    out.stats.build_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return SPT_OK;
}

}  // namespace spt
