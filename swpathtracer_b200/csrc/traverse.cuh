// traverse.cuh -- ray/scene queries on the device.
//
// closest_hit(): ordered, t-pruned stack traversal of the binary SAH tree stored as 64-byte
//   "pair" nodes (both children's boxes in the parent), returning the reference's answer:
//   the reference (acceleration/sbvh.cpp:478-510) visits every node whose box passes the slab
//   test, depth first and left first, and keeps a hit iff t > 0, t < best and the hit point is
//   inside the leaf box (+-1e-3).  Its result is therefore the hit with the smallest t, ties going
//   to the leaf reference met first in depth-first order -- the smallest slot here.  The box test
//   is the reference's own (slab() in spt_device.cuh); visiting near child first and skipping
//   children with tmin > best t or tmax < 0 only drops subtrees that cannot hold a better hit:
//   every non-root box is its primitives' bounds inflated by 1e-3, so any hit inside one lies
//   at least 1e-3 / |d_axis| past the box's entry and before its exit.
//
// count_traverse(): the reference's traversal itself -- no ordering, no pruning -- over the
//   flattened binary tree, counting box and primitive tests and passes
//   (num_intersection_tests / num_intersections, sbvh.cpp:478-510), plus the hit it finds.
#pragma once

#include "spt_device.cuh"

namespace spt {

__device__ __forceinline__ float inf_f() { return __int_as_float(0x7f800000); }

struct Hit1 {
    float t, u, v;
    uint32_t slot;
    uint32_t leaf;   // reference leaf of the hit (wide traversal), for the deferred inside test
    bool found;
};

__device__ __forceinline__ void prim_candidate(const DevScene& S, uint32_t slot, const float* box, V3 o, V3 d,
                                               bool check_inside, Hit1& h) {
    const float4 a = __ldg(S.tri + 3 * slot);
    const float4 b = __ldg(S.tri + 3 * slot + 1);
    const float4 c = __ldg(S.tri + 3 * slot + 2);
    float t, u = 0.0f, v = 0.0f;
    bool sphere = __float_as_int(c.w) == SPT_PRIM_SPHERE;
    bool ok = sphere ? sphere_test(f3v(a), b.x, o, d, t) : tri_test(f3v(a), f3v(b), f3v(c), o, d, t, u, v);
    if (!ok || !(t > 0.0f)) return;
    if (!(t < h.t || (h.found && t == h.t && slot < h.slot))) return;
    if (check_inside && !inside(box, hit_pos(sphere, o, d, t))) return;
    h.t = t;
    h.u = u;
    h.v = v;
    h.slot = slot;
    h.found = true;
}

template <int STACK>
__device__ __forceinline__ Hit1 closest_hit(const DevScene& S, V3 o, V3 d, uint32_t* overflow) {
    Hit1 h;
    h.t = inf_f();
    h.u = h.v = 0.0f;
    h.slot = 0;
    h.leaf = 0;
    h.found = false;
    if (S.empty) return h;
    if (S.no_accel) {  // NoAccelStructure::intersect: every primitive, no box test, strict <
        for (uint32_t s = 0; s < S.n_prims; ++s) prim_candidate(S, s, nullptr, o, d, false, h);
        return h;
    }
    const RayInv r = ray_inv(o, d);
    float t0, t1;
    if (!slab(r, S.root_min[0], S.root_min[1], S.root_min[2], S.root_max[0], S.root_max[1], S.root_max[2], t0, t1))
        return h;
    if (S.root_is_leaf) {
        const int2 fc = __ldg(S.leaf);
        for (int k = 0; k < fc.y; ++k) prim_candidate(S, fc.x + k, S.leaf_box, o, d, true, h);
        return h;
    }
    int st_node[STACK];
    float st_t[STACK];
    int sp = 0;
    int node = 0;
    for (;;) {
        if (node >= 0) {
            const float4* p = S.pair + 4 * node;
            const float4 a = __ldg(p), b = __ldg(p + 1), c = __ldg(p + 2);
            const int4 refs = __ldg(reinterpret_cast<const int4*>(p + 3));
            float lmin, lmax, rmin, rmax;
            bool hl = slab(r, a.x, a.y, a.z, a.w, b.x, b.y, lmin, lmax) && !(lmin > h.t) && !(lmax < 0.0f);
            bool hr = slab(r, b.z, b.w, c.x, c.y, c.z, c.w, rmin, rmax) && !(rmin > h.t) && !(rmax < 0.0f);
            if (hl && hr) {
                int near = refs.x, far = refs.y;
                float far_t = rmin;
                if (rmin < lmin) {
                    near = refs.y;
                    far = refs.x;
                    far_t = lmin;
                }
                if (sp < STACK) {
                    st_node[sp] = far;
                    st_t[sp] = far_t;
                    ++sp;
                } else {
                    atomicOr(overflow, 1u);
                }
                node = near;
                continue;
            }
            if (hl) {
                node = refs.x;
                continue;
            }
            if (hr) {
                node = refs.y;
                continue;
            }
        } else {
            const int l = ~node;
            const int2 fc = __ldg(S.leaf + l);
            for (int k = 0; k < fc.y; ++k) prim_candidate(S, fc.x + k, S.leaf_box + 6 * l, o, d, true, h);
        }
        bool got = false;
        while (sp > 0) {
            --sp;
            if (!(st_t[sp] > h.t)) {
                node = st_node[sp];
                got = true;
                break;
            }
        }
        if (!got) break;
    }
    return h;
}

struct CountOut {
    uint32_t tests, hits, prim_tests;
};

template <int STACK>
__device__ __forceinline__ Hit1 count_traverse(const DevScene& S, V3 o, V3 d, CountOut& c, uint32_t* overflow) {
    Hit1 h;
    h.t = inf_f();
    h.u = h.v = 0.0f;
    h.slot = 0;
    h.leaf = 0;
    h.found = false;
    c.tests = c.hits = c.prim_tests = 0;
    if (S.empty) return h;
    if (S.no_accel) {
        for (uint32_t s = 0; s < S.n_prims; ++s) {
            ++c.tests;
            ++c.prim_tests;
            const float4 a = __ldg(S.tri + 3 * s), b = __ldg(S.tri + 3 * s + 1), cc = __ldg(S.tri + 3 * s + 2);
            float t, u = 0.0f, v = 0.0f;
            bool sphere = __float_as_int(cc.w) == SPT_PRIM_SPHERE;
            bool ok = sphere ? sphere_test(f3v(a), b.x, o, d, t) : tri_test(f3v(a), f3v(b), f3v(cc), o, d, t, u, v);
            if (!ok) continue;
            ++c.hits;
            if ((t < h.t) && (t > 0.0f)) {
                h.t = t; h.u = u; h.v = v; h.slot = s; h.found = true;
            }
        }
        return h;
    }
    const RayInv r = ray_inv(o, d);
    uint32_t stack[STACK];
    int sp = 0;
    stack[sp++] = 0;
    while (sp > 0) {
        const uint32_t i = stack[--sp];
        const spt_bvh2_node nd = S.node2[i];
        ++c.tests;
        float t0, t1;
        if (!slab(r, nd.min[0], nd.min[1], nd.min[2], nd.max[0], nd.max[1], nd.max[2], t0, t1)) continue;
        ++c.hits;
        if (nd.count) {
            for (uint32_t k = 0; k < nd.count; ++k) {
                const uint32_t s = nd.right + k;
                ++c.tests;
                ++c.prim_tests;
                const float4 a = __ldg(S.tri + 3 * s), b = __ldg(S.tri + 3 * s + 1), cc = __ldg(S.tri + 3 * s + 2);
                float t, u = 0.0f, v = 0.0f;
                bool sphere = __float_as_int(cc.w) == SPT_PRIM_SPHERE;
                bool ok = sphere ? sphere_test(f3v(a), b.x, o, d, t) : tri_test(f3v(a), f3v(b), f3v(cc), o, d, t, u, v);
                if (!ok) continue;
                ++c.hits;
                if ((t > 0.0f) && (t < h.t)) {
                    float bx[6] = {nd.min[0], nd.min[1], nd.min[2], nd.max[0], nd.max[1], nd.max[2]};
                    if (inside(bx, hit_pos(sphere, o, d, t))) {
                        h.t = t; h.u = u; h.v = v; h.slot = s; h.found = true;
                    }
                }
            }
        } else if (sp + 2 <= STACK) {
            stack[sp++] = nd.right;
            stack[sp++] = i + 1;
        } else {
            atomicOr(overflow, 1u);
        }
    }
    return h;
}

__device__ __forceinline__ uint32_t slot_prim(const DevScene& S, uint32_t slot) {
    return __float_as_uint(__ldg(S.tri + 3 * slot).w);
}

}  // namespace spt
