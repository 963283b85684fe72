// Host-side check of the 8-wide collapse (swpathtracer_b200/csrc/wide_build.cpp) on one scene.
//
// Reads a scene dump (uint32 n, then n x 9 floats of triangle vertices), builds the reference's SAH
// tree (bvh_build.cpp) and its 8-wide collapse, and checks:
//   * every reference slot appears exactly once among the wide leaves' triangles;
//   * child and triangle indices stay in range, and children come after their parent
//     (breadth-first order);
//   * every child slot's dequantized box contains the reference leaf boxes of all the triangles
//     below it -- the property the wide traversal's exactness rests on;
//   * building twice gives the same bytes.
// Prints "ok <wide nodes> <triangles>" or the first violation, and exits non-zero on a violation.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "bvh_build.h"
#include "wide_build.h"

using namespace spt;

namespace {

struct Box {
    double mn[3], mx[3];
};

const std::vector<spt_bvh2_node>* g_bin;
const WideBvh* g_wide;
std::vector<int> g_leaf_of;   // reference slot -> binary leaf node
int g_bad = 0;

void fail(const char* what, size_t a, size_t b) {
    if (!g_bad) std::printf("violation: %s (%zu, %zu)\n", what, a, b);
    g_bad = 1;
}

Box leaf_box_of_slot(uint32_t slot) {
    const spt_bvh2_node& l = (*g_bin)[static_cast<size_t>(g_leaf_of[slot])];
    Box b;
    for (int k = 0; k < 3; ++k) {
        b.mn[k] = l.min[k];
        b.mx[k] = l.max[k];
    }
    return b;
}

void grow(Box& acc, const Box& b) {
    for (int k = 0; k < 3; ++k) {
        acc.mn[k] = std::fmin(acc.mn[k], b.mn[k]);
        acc.mx[k] = std::fmax(acc.mx[k], b.mx[k]);
    }
}

// the child box of slot s of node w, dequantized exactly (in double)
Box slot_box(const WideNode& w, int s) {
    const double p[3] = {w.px, w.py, w.pz};
    const int e[3] = {w.ex, w.ey, w.ez};
    Box b;
    for (int k = 0; k < 3; ++k) {
        b.mn[k] = p[k] + std::ldexp(static_cast<double>(w.qlo[k][s]), e[k]);
        b.mx[k] = p[k] + std::ldexp(static_cast<double>(w.qhi[k][s]), e[k]);
    }
    return b;
}

bool contains(const Box& outer, const Box& inner) {
    for (int k = 0; k < 3; ++k)
        if (!(outer.mn[k] <= inner.mn[k] && inner.mx[k] <= outer.mx[k])) return false;
    return true;
}

// union of the reference leaf boxes of every triangle below wide node i; checks the slots on the way
Box visit(uint32_t i, std::vector<int>& seen) {
    const std::vector<WideNode>& nodes = g_wide->nodes;
    const WideNode& w = nodes[i];
    Box all;
    for (int k = 0; k < 3; ++k) {
        all.mn[k] = INFINITY;
        all.mx[k] = -INFINITY;
    }
    for (int s = 0; s < 8; ++s) {
        Box below;
        bool any = false;
        if ((w.imask >> s) & 1u) {
            const uint32_t c = w.child_base + static_cast<uint32_t>(__builtin_popcount(w.imask & ((1u << s) - 1u)));
            if (c >= nodes.size() || c <= i) {
                fail("inner child index out of range or not after its parent", i, c);
                continue;
            }
            below = visit(c, seen);
            any = true;
        } else if (w.meta[s]) {
            const uint32_t off = w.meta[s] & 31u, mask = w.meta[s] >> 5;
            for (uint32_t t = 0; t < 3; ++t) {
                if (!((mask >> t) & 1u)) continue;
                const size_t k = static_cast<size_t>(w.tri_base) + off + t;
                if (k >= g_wide->tri_rank.size()) {
                    fail("triangle index out of range", i, k);
                    continue;
                }
                const uint32_t slot = g_wide->tri_rank[k];
                if (slot >= seen.size()) {
                    fail("reference slot out of range", k, slot);
                    continue;
                }
                ++seen[slot];
                const Box b = leaf_box_of_slot(slot);
                if (!any) below = b;
                else grow(below, b);
                any = true;
            }
        }
        if (!any) continue;
        if (!contains(slot_box(w, s), below)) fail("child box does not contain the boxes below it", i, static_cast<size_t>(s));
        grow(all, below);
    }
    return all;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 2) return 2;
    FILE* f = std::fopen(argv[1], "rb");
    if (!f) return 2;
    uint32_t n = 0;
    if (std::fread(&n, 4, 1, f) != 1) return 2;
    std::vector<float> data(9ull * n);
    if (n && std::fread(data.data(), 4, data.size(), f) != data.size()) return 2;
    std::fclose(f);
    std::vector<uint8_t> type(n, SPT_PRIM_TRIANGLE);
    std::vector<uint32_t> mat(n, 0);
    spt_scene_desc d{};
    d.n_prims = n;
    d.prim_type = type.data();
    d.prim_data = data.data();
    d.prim_material = mat.data();
    HostBvh tree;
    const char* err = nullptr;
    if (!build_sah_tree(d, 0, tree, &err)) {
        std::printf("violation: tree build failed\n");
        return 1;
    }
    WideBvh wide, again;
    build_wide(tree.nodes, wide);
    build_wide(tree.nodes, again);
    if (wide.nodes.size() != again.nodes.size() || wide.tri_rank != again.tri_rank ||
        std::memcmp(wide.nodes.data(), again.nodes.data(), wide.nodes.size() * sizeof(WideNode)) != 0)
        fail("two builds differ", wide.nodes.size(), again.nodes.size());
    g_bin = &tree.nodes;
    g_wide = &wide;
    g_leaf_of.assign(n, -1);
    for (size_t i = 0; i < tree.nodes.size(); ++i)
        if (tree.nodes[i].count)
            for (uint32_t k = 0; k < tree.nodes[i].count; ++k) g_leaf_of[tree.nodes[i].right + k] = static_cast<int>(i);
    std::vector<int> seen(n, 0);
    if (!wide.nodes.empty()) visit(0, seen);
    for (uint32_t s = 0; s < n; ++s)
        if (seen[s] != 1) {
            fail("reference slot not seen exactly once", s, static_cast<size_t>(seen[s]));
            break;
        }
    if (wide.tri_rank.size() != n) fail("triangle count differs", wide.tri_rank.size(), n);
    if (g_bad) return 1;
    std::printf("ok %zu %u\n", wide.nodes.size(), n);
    return 0;
}
