// bvh_build.cpp -- multithreaded host build of the reference's SAH tree (see bvh_build.h).
//
// Equality with the reference's tree rests on three facts:
//  * std::sort is deterministic: the permutation it produces depends only on the outcomes of the
//    comparisons it makes, so sorting a compact record keyed by the same centroid coordinate, from
//    the same starting order, yields the reference's order (sbvh_node.h:26-38).
//  * every float operation of the SAH sweep is done in the reference's order and precision
//    (aabb.cpp:11-16, sbvh.cpp:47-56, 76-110), on an FMA-free build (-ffp-contract=off).
//  * the recursion is left-first, so leaves cover consecutive ranges of the working array in
//    depth-first order, which is the order the reference's traversal meets them.
#include "bvh_build.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstring>
#include <limits>
#include <thread>

namespace spt {
namespace {

inline float gmin(float x, float y) { return (y < x) ? y : x; }  // glm::min
inline float gmax(float x, float y) { return (x < y) ? y : x; }  // glm::max

struct BRef {
    float c[3];
    uint32_t id;
    HostBox box;
};

inline void box_union(HostBox& acc, const HostBox& b) {  // AABB::operator+ (aabb.h:30-32)
    for (int k = 0; k < 3; ++k) {
        acc.mn[k] = gmin(acc.mn[k], b.mn[k]);
        acc.mx[k] = gmax(acc.mx[k], b.mx[k]);
    }
}

inline float box_area(const HostBox& b) {  // AABB::getArea (aabb.cpp:11-16)
    float l = b.mx[0] - b.mn[0], m = b.mx[1] - b.mn[1], n = b.mx[2] - b.mn[2];
    return 2.0f * (l * (m + n) + m * n);
}

struct TNode {
    HostBox box;
    int32_t left = -1, right = -1;
    uint32_t b = 0, e = 0;
};

const int kMaxDepth = 4096;

struct Builder {
    std::vector<BRef> refs;
    std::vector<TNode> pool;
    std::atomic<uint32_t> next{0};
    std::atomic<int> active{1};
    std::atomic<bool> too_deep{false};
    int max_threads = 1;

    void build(uint32_t node, uint32_t b, uint32_t e, int depth) {
        if (depth > kMaxDepth) {
            too_deep = true;
            return;
        }
        const uint32_t n = e - b;
        BRef* r = refs.data() + b;
        float best_cost = 1.0f * static_cast<float>(n);
        int best_axis = -1;
        long best_event = -1;
        thread_local std::vector<float> left_area;
        if (left_area.size() < n) left_area.resize(n);
        const float node_area = box_area(pool[node].box);
        for (int axis = 0; axis < 3; ++axis) {
            std::sort(r, r + n, [axis](const BRef& a, const BRef& c) { return a.c[axis] < c.c[axis]; });
            HostBox acc = r[0].box;
            for (uint32_t i = 0; i + 1 < n; ++i) {
                if (i) box_union(acc, r[i].box);
                left_area[i] = box_area(acc);
            }
            HostBox racc{};
            for (long i = static_cast<long>(n) - 2; i >= 0; --i) {
                if (i == static_cast<long>(n) - 2) racc = r[i + 1].box;
                else box_union(racc, r[i + 1].box);
                float ra = box_area(racc);
                float cost = 2.0f * 1.2f + ((left_area[i] / node_area) * static_cast<float>(i + 1) * 1.0f) +
                             ((ra / node_area) * static_cast<float>(n - 1 - i) * 1.0f);
                if (cost < best_cost) {
                    best_cost = cost;
                    best_event = i;
                    best_axis = axis;
                }
            }
        }
        if (best_axis == -1) {
            pool[node].b = b;
            pool[node].e = e;
            return;
        }
        std::sort(r, r + n, [best_axis](const BRef& a, const BRef& c) { return a.c[best_axis] < c.c[best_axis]; });
        const uint32_t mid = b + static_cast<uint32_t>(best_event) + 1;
        HostBox lb = r[0].box, rb = refs[mid].box;
        for (uint32_t i = b + 1; i < mid; ++i) box_union(lb, refs[i].box);
        for (uint32_t i = mid + 1; i < e; ++i) box_union(rb, refs[i].box);
        for (int k = 0; k < 3; ++k) {  // sbvh.cpp:409-412
            lb.mn[k] = lb.mn[k] - 1e-3f;
            lb.mx[k] = lb.mx[k] + 1e-3f;
            rb.mn[k] = rb.mn[k] - 1e-3f;
            rb.mx[k] = rb.mx[k] + 1e-3f;
        }
        const uint32_t ln = next.fetch_add(2), rn = ln + 1;
        pool[ln].box = lb;
        pool[rn].box = rb;
        pool[node].left = static_cast<int32_t>(ln);
        pool[node].right = static_cast<int32_t>(rn);
        if (n > 8192 && active.load() < max_threads) {
            ++active;
            std::thread t([this, ln, b, mid, depth] { build(ln, b, mid, depth + 1); });
            build(rn, mid, e, depth + 1);
            t.join();
            --active;
        } else {
            build(ln, b, mid, depth + 1);
            build(rn, mid, e, depth + 1);
        }
    }
};

}  // namespace

void prim_bounds(const spt_scene_desc& d, uint32_t i, HostBox& box, float c[3]) {
    const float* p = d.prim_data + 9ull * i;
    if (d.prim_type[i] == SPT_PRIM_SPHERE) {
        for (int k = 0; k < 3; ++k) {
            box.mn[k] = p[k] - p[3];
            box.mx[k] = p[k] + p[3];
            c[k] = p[k];
        }
        return;
    }
    for (int k = 0; k < 3; ++k) {
        box.mn[k] = gmin(gmin(p[k], p[3 + k]), p[6 + k]);
        box.mx[k] = gmax(gmax(p[k], p[3 + k]), p[6 + k]);
        c[k] = ((p[k] + p[3 + k]) + p[6 + k]) * (1.0f / 3.0f);
    }
}

bool build_sah_tree(const spt_scene_desc& d, int n_threads, HostBvh& out, const char** err) {
    auto t0 = std::chrono::steady_clock::now();
    out.nodes.clear();
    out.refs.clear();
    std::memset(&out.stats, 0, sizeof(out.stats));
    const uint32_t n = d.n_prims;
    if (n == 0) return true;
    Builder B;
    B.max_threads = n_threads > 0 ? n_threads : static_cast<int>(std::max(1u, std::thread::hardware_concurrency()));
    B.refs.resize(n);
    HostBox root{};
    for (uint32_t i = 0; i < n; ++i) {  // sbvh.cpp:17-24
        BRef& r = B.refs[i];
        r.id = i;
        prim_bounds(d, i, r.box, r.c);
        if (i == 0) root = r.box;
        else box_union(root, r.box);
    }
    B.pool.resize(2ull * n);
    B.next = 1;
    B.pool[0].box = root;
    B.build(0, 0, n, 0);
    if (B.too_deep) {
        *err = "SAH tree deeper than 4096 levels";
        return false;
    }
    // depth-first flatten (left first)
    const uint32_t count = B.next.load();
    out.nodes.resize(count);
    uint32_t emitted = 0;
    std::vector<uint32_t> slot_of(count);
    // iterative pre-order: output index = order of first visit
    std::vector<uint32_t> st{0};
    while (!st.empty()) {
        uint32_t pn = st.back();
        st.pop_back();
        slot_of[pn] = emitted++;
        const TNode& t = B.pool[pn];
        if (t.left >= 0) {
            st.push_back(static_cast<uint32_t>(t.right));
            st.push_back(static_cast<uint32_t>(t.left));
        }
    }
    for (uint32_t pn = 0; pn < count; ++pn) {
        const TNode& t = B.pool[pn];
        spt_bvh2_node& o = out.nodes[slot_of[pn]];
        for (int k = 0; k < 3; ++k) {
            o.min[k] = t.box.mn[k];
            o.max[k] = t.box.mx[k];
        }
        if (t.left >= 0) {
            o.right = slot_of[t.right];
            o.count = 0;
        } else {
            o.right = t.b;
            o.count = t.e - t.b;
        }
    }
    out.refs.resize(n);
    for (uint32_t i = 0; i < n; ++i) out.refs[i] = B.refs[i].id;
    tree_statistics(out);
    out.stats.build_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return true;
}

void tree_statistics(HostBvh& out) {
    // statistics as SBVH::collectTreeStatistics reports them (sbvh.cpp:517-575)
    spt_bvh_stats& s = out.stats;
    const double build_ms = s.build_ms;
    std::memset(&s, 0, sizeof(s));
    s.build_ms = build_ms;
    if (out.nodes.empty()) return;
    s.min_prims_leaf = std::numeric_limits<uint64_t>::max();
    std::vector<uint32_t> level{0}, nextl;
    uint64_t levels = 0;
    while (!level.empty()) {
        ++levels;
        nextl.clear();
        for (uint32_t i : level) {
            const spt_bvh2_node& nd = out.nodes[i];
            ++s.num_nodes;
            if (nd.count) {
                ++s.num_leaf_nodes;
                s.num_references += nd.count;
                s.min_prims_leaf = std::min<uint64_t>(s.min_prims_leaf, nd.count);
                s.max_prims_leaf = std::max<uint64_t>(s.max_prims_leaf, nd.count);
            } else {
                ++s.num_inner_nodes;
                nextl.push_back(i + 1);
                nextl.push_back(nd.right);
            }
        }
        level.swap(nextl);
    }
    s.tree_height = levels ? levels - 1 : 0;
    s.num_unreferenced = 0;  // every primitive lands in exactly one leaf of an object-split tree
}

}  // namespace spt
