// traverse_wide.cuh -- closest hit over the 8-wide quantized BVH (wide_build.h).
//
// Why the answer is still the reference's: every box of the reference tree below the root is its
// primitives' bounds inflated by 1e-3 (acceleration/sbvh.cpp:409-412), and the wide nodes' boxes
// contain those boxes (quantized outward).  A hit the reference keeps lies inside its leaf box
// (inside() below), hence at least ~1e-3 inside every ancestor box, so a conservative box test --
// here one FMA per plane on the quantized grid, with the interval clipped to [0, best t] -- can only
// visit more nodes than needed, never skip the node holding that hit.  The root box is tested with the
// reference's own slab test first, and every candidate is accepted by the reference's exact rules:
// Moller-Trumbore as in triangle.cpp, t > 0, the hit point inside the reference leaf box (+-1e-3), and
// the smallest (t, rank) with rank = the reference's depth-first leaf order.
#pragma once

#include "spt_internal.h"
#include "traverse.cuh"

namespace spt {

constexpr int kWideStack = 32;

__device__ __forceinline__ uint32_t byte_of(uint32_t lo, uint32_t hi, int j) {
    return ((j < 4 ? lo : hi) >> (8 * (j & 3))) & 0xFFu;
}

__device__ __forceinline__ float exp2i(int e) { return __int_as_float((e + 127) << 23); }

struct WideRay {
    V3 o;
    float ix, iy, iz;   // 1/d with zero components replaced by a tiny signed value
    uint32_t inv_oct;   // slot order key: slot ^ inv_oct, ascending = near to far
};

__device__ __forceinline__ float safe_inv(float d) {
    return 1.0f / (fabsf(d) > 1e-20f ? d : copysignf(1e-20f, d));
}

__device__ __forceinline__ void wide_node_hits(const DevScene& S, const WideRay& r, uint32_t idx, float best_t,
                                               uint32_t& g_base, uint32_t& g_hits, uint32_t& g_imask,
                                               uint32_t& t_base, uint32_t& t_mask) {
    const uint4* n = S.wnode + 5 * idx;
    const uint4 w0 = __ldg(n), w1 = __ldg(n + 1), w2 = __ldg(n + 2), w3 = __ldg(n + 3), w4 = __ldg(n + 4);
    const int ex = static_cast<int8_t>(w0.w & 0xFFu), ey = static_cast<int8_t>((w0.w >> 8) & 0xFFu),
              ez = static_cast<int8_t>((w0.w >> 16) & 0xFFu);
    const uint32_t imask = w0.w >> 24;
    const float sx = exp2i(ex) * r.ix, sy = exp2i(ey) * r.iy, sz = exp2i(ez) * r.iz;
    const float ox = (__uint_as_float(w0.x) - r.o.x) * r.ix;
    const float oy = (__uint_as_float(w0.y) - r.o.y) * r.iy;
    const float oz = (__uint_as_float(w0.z) - r.o.z) * r.iz;
    // The near plane is the low plane when 1/d >= 0.  The choice is made once per node on whole
    // words (four children's planes each), not per child and plane: 12 selects instead of 48.
    const bool nx = r.ix >= 0.0f, ny = r.iy >= 0.0f, nz = r.iz >= 0.0f;
    const uint32_t nx0 = nx ? w2.x : w3.z, nx1 = nx ? w2.y : w3.w, fx0 = nx ? w3.z : w2.x, fx1 = nx ? w3.w : w2.y;
    const uint32_t ny0 = ny ? w2.z : w4.x, ny1 = ny ? w2.w : w4.y, fy0 = ny ? w4.x : w2.z, fy1 = ny ? w4.y : w2.w;
    const uint32_t nz0 = nz ? w3.x : w4.z, nz1 = nz ? w3.y : w4.w, fz0 = nz ? w4.z : w3.x, fz1 = nz ? w4.w : w3.y;
    uint32_t hits = 0, tm = 0;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const uint32_t meta = byte_of(w1.z, w1.w, j);
        const bool inner = (imask >> j) & 1u;
        const float tnx = __fmaf_rn(static_cast<float>(byte_of(nx0, nx1, j)), sx, ox);
        const float tfx = __fmaf_rn(static_cast<float>(byte_of(fx0, fx1, j)), sx, ox);
        const float tny = __fmaf_rn(static_cast<float>(byte_of(ny0, ny1, j)), sy, oy);
        const float tfy = __fmaf_rn(static_cast<float>(byte_of(fy0, fy1, j)), sy, oy);
        const float tnz = __fmaf_rn(static_cast<float>(byte_of(nz0, nz1, j)), sz, oz);
        const float tfz = __fmaf_rn(static_cast<float>(byte_of(fz0, fz1, j)), sz, oz);
        const float tmin = fmaxf(fmaxf(tnx, tny), fmaxf(tnz, 0.0f));
        const float tmax = fminf(fminf(tfx, tfy), fminf(tfz, best_t));
        const bool hit = (inner || meta != 0u) && tmin <= tmax;
        if (hit) {
            if (inner) hits |= 1u << (j ^ r.inv_oct);
            else tm |= (meta >> 5) << (meta & 31u);
        }
    }
    g_base = w1.x;
    g_hits = hits;
    g_imask = imask;
    t_base = w1.y;
    t_mask = tm;
}

// One candidate triangle/sphere.  Without `exact`, the reference's inside-the-leaf-box test is
// deferred to the final hit (WideTraversal::finish / closest_hit_wide): a candidate that beats the
// current best on (t, rank) is kept either way, and if the final hit fails the test the ray is traced
// again with the test applied to every candidate.  Pruning with a best t that might later be rejected
// is safe because the final best, once it passes, is the minimum over all candidates with t > 0.
__device__ __forceinline__ void wide_candidate(const DevScene& S, uint32_t wslot, V3 o, V3 d, Hit1& h, bool exact) {
    const float4 a = __ldg(S.wtri + 3 * wslot);
    const float4 b = __ldg(S.wtri + 3 * wslot + 1);
    const float4 c = __ldg(S.wtri + 3 * wslot + 2);
    const uint32_t rank = __float_as_uint(a.w);
    float t, u = 0.0f, v = 0.0f;
    const bool sphere = __float_as_int(b.w) == SPT_PRIM_SPHERE;
    const bool ok = sphere ? sphere_test(f3v(a), c.x, o, d, t) : tri_test(f3v(a), f3v(b), f3v(c), o, d, t, u, v);
    if (!ok || !(t > 0.0f)) return;
    if (!(t < h.t || (h.found && t == h.t && rank < h.slot))) return;
    const uint32_t leaf = __float_as_uint(c.w);
    if (exact && !inside(S.leaf_box + 6 * leaf, hit_pos(sphere, o, d, t))) return;
    h.t = t;
    h.u = u;
    h.v = v;
    h.slot = rank;
    h.leaf = leaf;
    h.found = true;
}

// The deferred inside test of the final hit (o + d*t is the same float expression for both
// primitive kinds).
__device__ __forceinline__ bool final_inside(const DevScene& S, const Hit1& h, V3 o, V3 d) {
    return !h.found || inside(S.leaf_box + 6 * h.leaf, o + d * h.t);
}

__device__ __forceinline__ Hit1 closest_hit_wide_pass(const DevScene& S, V3 o, V3 d, uint32_t* overflow, bool exact) {
    Hit1 h;
    h.t = inf_f();
    h.u = h.v = 0.0f;
    h.slot = 0;
    h.leaf = 0;
    h.found = false;
    if (S.empty) return h;
    if (S.no_accel) {
        for (uint32_t s = 0; s < S.n_prims; ++s) prim_candidate(S, s, nullptr, o, d, false, h);
        return h;
    }
    {
        const RayInv ri = ray_inv(o, d);
        float t0, t1;
        if (!slab(ri, S.root_min[0], S.root_min[1], S.root_min[2], S.root_max[0], S.root_max[1], S.root_max[2], t0,
                  t1))
            return h;
    }
    WideRay r;
    r.o = o;
    r.ix = safe_inv(d.x);
    r.iy = safe_inv(d.y);
    r.iz = safe_inv(d.z);
    r.inv_oct = (r.ix >= 0.0f ? 0u : 1u) | (r.iy >= 0.0f ? 0u : 2u) | (r.iz >= 0.0f ? 0u : 4u);
    uint2 stack[kWideStack];
    int sp = 0;
    uint32_t g_base, g_hits, g_imask, t_base, t_mask;
    wide_node_hits(S, r, 0, h.t, g_base, g_hits, g_imask, t_base, t_mask);
    for (;;) {
        while (t_mask) {
            const int k = __ffs(t_mask) - 1;
            t_mask &= t_mask - 1;
            wide_candidate(S, t_base + k, o, d, h, exact);
        }
        if (!g_hits) {
            if (sp == 0) break;
            const uint2 e = stack[--sp];   // one 8-byte load
            g_base = e.x;
            g_hits = e.y & 0xFFu;
            g_imask = e.y >> 8;
        }
        const uint32_t key = __ffs(g_hits) - 1;
        g_hits &= g_hits - 1;
        const uint32_t s = key ^ r.inv_oct;
        const uint32_t child = g_base + __popc(g_imask & ((1u << s) - 1u));
        if (g_hits) {
            if (sp < kWideStack) {
                stack[sp] = make_uint2(g_base, g_hits | (g_imask << 8));
                ++sp;
            } else {
                atomicOr(overflow, 1u);
            }
        }
        wide_node_hits(S, r, child, h.t, g_base, g_hits, g_imask, t_base, t_mask);
    }
    return h;
}

__device__ __forceinline__ Hit1 closest_hit_wide(const DevScene& S, V3 o, V3 d, uint32_t* overflow) {
    Hit1 h = closest_hit_wide_pass(S, o, d, overflow, false);
    if (!final_inside(S, h, o, d)) h = closest_hit_wide_pass(S, o, d, overflow, true);
    return h;
}

// The same traversal as a resumable state, one node (and its triangles) per step, for kernels that
// keep a warp's lanes busy by giving a lane a new ray as soon as its ray is finished.
// A pop reads its 8-byte entry once (not its two halves in several loads): with that, the 48-register
// closest-hit kernel spills 16 bytes instead of 60 and runs 2,929 instead of 2,718 Mrays/s.
// REG_TOP keeps the most recent stack entry in registers, so a push followed by its pop touches no
// local memory.  The path tracer's extend kernel (no register bound) gains 2-5 % from it; the
// closest-hit kernel, held to 48 registers, would spill more and lose 9 %, so it keeps the plain
// stack.
// DEPTH is the compiled stack depth (entries per lane).  A traversal needs at most one entry per wide
// level below the root for the remaining children of an ancestor plus one per level for postponed
// triangles, 2 (H - 1) for a wide tree of H levels; wide_stack_bound() gives that bound per scene.
// step()'s `limit` (1 <= limit <= DEPTH) can hold a traversal to fewer entries; one that needs more
// sets the overflow status bit instead of writing past the limit.
// COUNT adds the lane's own work counters (node visits, primitive tests) over all of its rays.
template <bool REG_TOP, int DEPTH = kWideStack, bool COUNT = false>
struct WideTraversalT {
    static_assert(DEPTH >= 1 && DEPTH <= kWideStack, "stack depth out of range");
    V3 o, d;
    WideRay r;
    Hit1 h;
    uint2 stack[DEPTH];
    int sp;
    uint2 top;
    bool has_top;
    uint32_t g_base, g_hits, g_imask, t_base, t_mask;
    bool exact;
    uint32_t n_nodes = 0, n_prims = 0;   // COUNT only

    // entries in use: the local ones plus the register top
    __device__ __forceinline__ bool can_push(int limit) const {
        return sp + ((REG_TOP && has_top) ? 1 : 0) < limit && sp < DEPTH;
    }
    __device__ __forceinline__ void push(uint2 e) {
        if (!REG_TOP) {
            stack[sp++] = e;
            return;
        }
        if (has_top) stack[sp++] = top;
        top = e;
        has_top = true;
    }
    // With REG_TOP the register entry is the stack's top whenever the stack is not empty: a pop
    // returns it and at once loads the next entry from local memory into the register, so that load
    // has the whole next node visit to arrive before the following pop needs it.
    __device__ __forceinline__ bool empty() const { return REG_TOP ? !has_top : sp == 0; }
    __device__ __forceinline__ uint2 pop() {
        if (!REG_TOP) return stack[--sp];
        const uint2 r = top;
        if (sp > 0) top = stack[--sp];
        else has_top = false;
        return r;
    }

    // Returns false when the ray is already finished (empty scene or root box missed).  The root node
    // itself is visited by the first step(): a lane that takes a new ray while the rest of its warp
    // is mid-traversal then tests the root's children together with the other lanes' node visits,
    // not alone in the refill branch.
    __device__ __forceinline__ bool start(const DevScene& S, V3 o_, V3 d_, bool exact_ = false) {
        o = o_;
        d = d_;
        exact = exact_;
        h.t = inf_f();
        h.u = h.v = 0.0f;
        h.slot = 0;
        h.leaf = 0;
        h.found = false;
        sp = 0;
        has_top = false;
        if (S.empty) return false;
        const RayInv ri = ray_inv(o, d);
        float t0, t1;
        if (!slab(ri, S.root_min[0], S.root_min[1], S.root_min[2], S.root_max[0], S.root_max[1], S.root_max[2], t0, t1))
            return false;
        r.o = o;
        // safe_inv without dividing again: 1/d is already in ri unless |d| <= 1e-20
        r.ix = fabsf(d.x) > 1e-20f ? ri.inv.x : copysignf(1.0f / 1e-20f, d.x);
        r.iy = fabsf(d.y) > 1e-20f ? ri.inv.y : copysignf(1.0f / 1e-20f, d.y);
        r.iz = fabsf(d.z) > 1e-20f ? ri.inv.z : copysignf(1.0f / 1e-20f, d.z);
        r.inv_oct = (r.ix >= 0.0f ? 0u : 1u) | (r.iy >= 0.0f ? 0u : 2u) | (r.iz >= 0.0f ? 0u : 4u);
        // a pending visit of node 0: one hit child (slot 0, whose near-to-far key is inv_oct) of a
        // parent whose first child is node 0
        g_base = 0;
        g_imask = 1u;
        g_hits = 1u << r.inv_oct;
        t_base = 0;
        t_mask = 0;
        return true;
    }

    // One step: the pending triangles, then the next node.  Returns false once the ray is done.
    // When fewer than 1/8 of the warp's active lanes have triangles to test and this lane still has
    // nodes to visit, its triangles wait on the stack (tag bit 31 of .x) so the warp keeps traversing
    // together (after the triangle postponing of Ylitie et al., HPG 2017).  Measured on 2^24
    // incoherent rays: 2,103 -> 2,568 Mrays/s.  The order of the candidates does not change the
    // result, which is the minimum over (t, rank).  A popped triangle entry is tested at the next step
    // (no node work in hand), so every entry is postponed at most once.
    __device__ __forceinline__ bool step(const DevScene& S, uint32_t* overflow, int limit = DEPTH) {
        const unsigned act = __activemask();
        const unsigned tri = __ballot_sync(act, t_mask != 0u);
        if (t_mask && g_hits && can_push(limit) && 8 * __popc(tri) < __popc(act)) {
            push(make_uint2(t_base | 0x80000000u, t_mask));
            t_mask = 0;
        }
        while (t_mask) {
            const int k = __ffs(t_mask) - 1;
            t_mask &= t_mask - 1;
            wide_candidate(S, t_base + k, o, d, h, exact);
            if (COUNT) ++n_prims;
        }
        if (!g_hits) {
            if (empty()) return false;
            const uint2 e = pop();
            if (e.x & 0x80000000u) {   // postponed triangles
                t_base = e.x & 0x7FFFFFFFu;
                t_mask = e.y;
                return true;
            }
            g_base = e.x;
            g_hits = e.y & 0xFFu;
            g_imask = e.y >> 8;
        }
        const uint32_t key = __ffs(g_hits) - 1;
        g_hits &= g_hits - 1;
        const uint32_t s = key ^ r.inv_oct;
        const uint32_t child = g_base + __popc(g_imask & ((1u << s) - 1u));
        if (g_hits) {
            if (can_push(limit)) push(make_uint2(g_base, g_hits | (g_imask << 8)));
            else atomicOr(overflow, 1u);
        }
        wide_node_hits(S, r, child, h.t, g_base, g_hits, g_imask, t_base, t_mask);
        if (COUNT) ++n_nodes;
        return true;
    }

    // After step() returned false: true if the result is final; false if the final hit failed the
    // deferred inside test and the traversal restarted in exact mode (keep stepping).
    __device__ __forceinline__ bool finish(const DevScene& S) {
        if (exact || final_inside(S, h, o, d)) return true;
        start(S, o, d, true);
        return false;
    }
};

// Persistent warps with dynamic ray fetch (after Aila & Laine, "Understanding the Efficiency of Ray
// Traversal on GPUs", HPG 2009): a lane whose ray is finished takes the next ray at once instead of
// idling until the warp's longest ray ends.  Ray indices come from a warp-local pool refilled
// kChunk at a time from one global counter, so the counter sees one atomic per kChunk rays.  32 is
// the least that works (one refill may hand up to 32 lanes rays from a fresh chunk): against 64 it
// measured +0.6 % on the ordered incoherent queries and +4.6 % / +8.2 % on the box and layered path
// tracing (a shorter tail, and the ordered neighbours stay together); 128 lost 3 %.
// load(i, o, d) fetches ray i; store(i, h) writes its result.
constexpr uint32_t kChunk = 32;
static_assert(kChunk >= 32, "a refill takes up to 32 rays from one fresh chunk");
// Refill once this many lanes wait for a ray (or no lane is busy): the refill branch runs with only
// the waiting lanes, so batching it pays a little (2,674 -> 2,690 Mrays/s at 4; 2 and 8 gain less).
constexpr int kRefill = 4;

// COUNT: adds the kernel's own node visits and primitive tests to counts[0] / counts[1].
template <bool COUNT = false, typename Load, typename Store>
__device__ __forceinline__ void persistent_trace(const DevScene& S, uint64_t n, unsigned long long* next,
                                                 uint32_t* overflow, Load load, Store store,
                                                 unsigned long long* counts = nullptr) {
    const uint32_t lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    WideTraversalT<false, kWideStack, COUNT> tr;
    bool active = false, exhausted = false;
    uint64_t mine = 0;
    unsigned long long pool = 0, pool_end = 0;  // warp-uniform
    for (;;) {
        const unsigned need = __ballot_sync(0xFFFFFFFFu, !active && !exhausted);
        const unsigned busy = __ballot_sync(0xFFFFFFFFu, active);
        if (need && (__popc(need) >= kRefill || !busy)) {
            const uint32_t cnt = __popc(need), rank = __popc(need & lt);
            const unsigned long long have = pool_end - pool;
            unsigned long long fresh = 0;
            if (have < cnt) {
                if (lane == 0) fresh = atomicAdd(next, static_cast<unsigned long long>(kChunk));
                fresh = __shfl_sync(0xFFFFFFFFu, fresh, 0);
            }
            if (!active && !exhausted) {
                mine = rank < have ? pool + rank : fresh + (rank - have);
                if (mine >= n) {
                    exhausted = true;
                } else {
                    V3 o, d;
                    load(mine, o, d);
                    active = tr.start(S, o, d);
                    if (!active) store(mine, tr.h);
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
        if (active && !tr.step(S, overflow) && tr.finish(S)) {
            store(mine, tr.h);
            active = false;
        }
    }
    if (COUNT) {
        unsigned long long a = tr.n_nodes, b = tr.n_prims;
        for (int o = 16; o > 0; o >>= 1) {
            a += __shfl_xor_sync(0xFFFFFFFFu, a, o);
            b += __shfl_xor_sync(0xFFFFFFFFu, b, o);
        }
        if (lane == 0) {
            atomicAdd(counts, a);
            atomicAdd(counts + 1, b);
        }
    }
}

// Closest hit with the traversal the scene selected (a kernel template parameter, so each kernel
// carries one traversal's registers).
template <int TRAV>
__device__ __forceinline__ Hit1 trace_closest(const DevScene& S, V3 o, V3 d, uint32_t* overflow) {
    if (TRAV >= 1) return closest_hit_wide(S, o, d, overflow);
    return closest_hit<kStack>(S, o, d, overflow);
}

}  // namespace spt
