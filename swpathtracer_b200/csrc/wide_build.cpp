// wide_build.cpp -- collapse the reference binary tree into 8-wide quantized nodes (wide_build.h).
//
// Greedy collapse (the surface-area heuristic of wide-BVH literature, e.g. Ylitie, Karras, Laine,
// "Efficient Incoherent Ray Traversal on GPUs Through Compressed Wide BVHs", HPG 2017): starting from
// a binary node's two children, repeatedly open the inner child with the largest box area while the
// children still fit in 8 slots.  A binary leaf of k references takes ceil(k/3) slots (three
// triangles per slot); a leaf too large for the free slots becomes a wide node of its own.
// The boxes are the reference's boxes, quantized outward; triangles keep their reference slot
// ("rank") so that hits still resolve exactly as the reference's traversal order would.
// On the 1.31M-triangle mesh the collapse takes 65-86 ms on 8 host cores (360 ms before fixed-size
// item lists, a sort-free slot assignment and one thread per subtree of the root).
#include "wide_build.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <thread>

namespace spt {
namespace {

struct Box {
    float mn[3], mx[3];
};

inline Box node_box(const spt_bvh2_node& n) {
    Box b;
    for (int k = 0; k < 3; ++k) {
        b.mn[k] = n.min[k];
        b.mx[k] = n.max[k];
    }
    return b;
}

inline double area(const Box& b) {
    double l = double(b.mx[0]) - b.mn[0], m = double(b.mx[1]) - b.mn[1], n = double(b.mx[2]) - b.mn[2];
    return 2.0 * (l * (m + n) + m * n);
}

enum Kind { INNER, LEAF, LEAFNODE, CHUNK };

struct Item {
    Kind kind;
    uint32_t node;          // binary node (INNER / LEAF / LEAFNODE)
    uint32_t first, count;  // reference slots (LEAF / LEAFNODE / CHUNK)
    Box box;
};

inline int cost(const Item& it) { return it.kind == LEAF ? static_cast<int>((it.count + 2) / 3) : 1; }

// At most 8 items: every list below fills at most the 8 slots of one wide node (each item takes at
// least one), so fixed arrays replace per-node heap allocations.
struct Items {
    Item v[8];
    int n = 0;
    void push(const Item& it) { v[n++] = it; }
    int used() const {
        int u = 0;
        for (int k = 0; k < n; ++k) u += cost(v[k]);
        return u;
    }
};

struct Collapser {
    const std::vector<spt_bvh2_node>& bn;
    std::vector<WideNode>& out;
    std::vector<uint32_t>& rank;

    Item item_of(uint32_t i) const {
        const spt_bvh2_node& n = bn[i];
        Item it;
        it.node = i;
        it.box = node_box(n);
        if (n.count == 0) {
            it.kind = INNER;
            it.first = it.count = 0;
        } else {
            it.kind = (n.count + 2) / 3 <= 8 ? LEAF : LEAFNODE;
            it.first = n.right;
            it.count = n.count;
        }
        return it;
    }

    // children of an inner binary node, collapsed to at most 8 slots
    Items collapse(uint32_t i) const {
        Items items;
        items.push(item_of(i + 1));
        items.push(item_of(bn[i].right));
        // two big leaves may not fit together: turn the costliest into nodes of their own
        while (items.used() > 8) {
            int m = 0;   // the first item of the largest cost
            for (int k = 1; k < items.n; ++k)
                if (cost(items.v[m]) < cost(items.v[k])) m = k;
            items.v[m].kind = LEAFNODE;
        }
        int open_cost[8];   // slots an inner item's two children take, once known (-1: not yet)
        std::fill(open_cost, open_cost + 8, -1);
        for (;;) {
            int best = -1;
            double best_area = -1.0;
            const int u = items.used();
            for (int k = 0; k < items.n; ++k) {
                if (items.v[k].kind != INNER) continue;
                if (open_cost[k] < 0) {
                    const uint32_t n = items.v[k].node;
                    open_cost[k] = cost(item_of(n + 1)) + cost(item_of(bn[n].right));
                }
                if (u - 1 + open_cost[k] > 8) continue;
                double a = area(items.v[k].box);
                if (a > best_area) {
                    best_area = a;
                    best = k;
                }
            }
            if (best < 0) break;
            const uint32_t n = items.v[best].node;
            items.v[best] = item_of(n + 1);
            open_cost[best] = -1;
            open_cost[items.n] = -1;
            items.push(item_of(bn[n].right));
        }
        return items;
    }

    // children of a wide node that holds one large leaf's references
    Items leaf_children(uint32_t first, uint32_t count, const Box& box) const {
        Items items;
        if (count <= 24) {
            for (uint32_t s = 0; s < count; s += 3) items.push(Item{CHUNK, 0, first + s, std::min(3u, count - s), box});
        } else {
            const uint32_t per = (count + 7) / 8;
            for (uint32_t s = 0; s < count; s += per) items.push(Item{LEAFNODE, 0, first + s, std::min(per, count - s), box});
        }
        return items;
    }

    struct Kids {
        uint32_t idx[8];
        Items items[8];
        int n = 0;
    };

    // The wide node idx over `items`: written to out[idx], its leaf triangles appended to rank, its
    // inner children given consecutive slots at the end of out and returned with their items.
    void fill_node(uint32_t idx, const Items& items, Kids& kids) {
        // expand LEAF items into chunks of up to three triangles (items is never empty: a binary
        // node has two children and a leaf at least one reference)
        Items ch;
        ch.v[0] = items.v[0];
        for (int k = 0; k < items.n; ++k) {
            const Item& it = items.v[k];
            if (it.kind == LEAF)
                for (uint32_t s = 0; s < it.count; s += 3)
                    ch.push(Item{CHUNK, it.node, it.first + s, std::min(3u, it.count - s), it.box});
            else
                ch.push(it);
        }
        // node box and quantization grid
        Box nb = ch.v[0].box;
        for (int c = 0; c < ch.n; ++c)
            for (int k = 0; k < 3; ++k) {
                nb.mn[k] = std::min(nb.mn[k], ch.v[c].box.mn[k]);
                nb.mx[k] = std::max(nb.mx[k], ch.v[c].box.mx[k]);
            }
        WideNode w;
        std::memset(&w, 0, sizeof(w));
        w.px = nb.mn[0];
        w.py = nb.mn[1];
        w.pz = nb.mn[2];
        int e[3];
        for (int k = 0; k < 3; ++k) {
            double ext = double(nb.mx[k]) - double(nb.mn[k]);
            int ek = -125;
            if (ext > 0.0) ek = std::max(-125, static_cast<int>(std::ceil(std::log2(ext / 255.0))));
            while (std::ldexp(255.0, ek) < ext) ++ek;  // guard against log2 rounding
            e[k] = ek;
        }
        w.ex = static_cast<int8_t>(e[0]);
        w.ey = static_cast<int8_t>(e[1]);
        w.ez = static_cast<int8_t>(e[2]);
        // slot assignment by direction (greedy on the centre offsets): candidates by score, ties in
        // (child, slot) order
        double cx = 0.5 * (double(nb.mn[0]) + nb.mx[0]), cy = 0.5 * (double(nb.mn[1]) + nb.mx[1]),
               cz = 0.5 * (double(nb.mn[2]) + nb.mx[2]);
        struct Cand {
            double score;
            int child, slot;
        };
        Cand cand[64];
        int nc = 0;
        for (int c = 0; c < ch.n; ++c) {
            double dx = 0.5 * (double(ch.v[c].box.mn[0]) + ch.v[c].box.mx[0]) - cx;
            double dy = 0.5 * (double(ch.v[c].box.mn[1]) + ch.v[c].box.mx[1]) - cy;
            double dz = 0.5 * (double(ch.v[c].box.mn[2]) + ch.v[c].box.mx[2]) - cz;
            for (int s = 0; s < 8; ++s)
                cand[nc++] = Cand{((s & 1) ? dx : -dx) + ((s & 2) ? dy : -dy) + ((s & 4) ? dz : -dz), c, s};
        }
        // Scanning the candidates in that order and taking each whose child and slot are both free is
        // the same as taking, ch.n times, the best candidate whose child and slot are both free (a
        // skipped candidate stays blocked); the latter needs no sort.
        int slot_of[8], child_in[8];
        std::fill(slot_of, slot_of + 8, -1);
        std::fill(child_in, child_in + 8, -1);
        for (int round = 0; round < ch.n; ++round) {
            int best = -1;
            for (int k = 0; k < nc; ++k) {   // candidates are in (child, slot) order: '>' keeps the first
                const Cand& c = cand[k];
                if (slot_of[c.child] >= 0 || child_in[c.slot] >= 0) continue;
                if (best < 0 || c.score > cand[best].score) best = k;
            }
            slot_of[cand[best].child] = cand[best].slot;
            child_in[cand[best].slot] = cand[best].child;
        }
        // leaf triangles (consecutive, slot order) and inner children (consecutive, slot order)
        w.tri_base = static_cast<uint32_t>(rank.size());
        uint32_t n_inner = 0;
        for (int s = 0; s < 8; ++s)
            if (child_in[s] >= 0 && ch.v[child_in[s]].kind != CHUNK) ++n_inner;
        w.child_base = static_cast<uint32_t>(out.size());
        out.resize(out.size() + n_inner);
        int inner_child[8];
        int ni = 0;
        for (int s = 0; s < 8; ++s) {
            const int c = child_in[s];
            if (c < 0) continue;
            const Item& it = ch.v[c];
            for (int k = 0; k < 3; ++k) {
                double q0 = std::floor((double(it.box.mn[k]) - double(nb.mn[k])) / std::ldexp(1.0, e[k]));
                double q1 = std::ceil((double(it.box.mx[k]) - double(nb.mn[k])) / std::ldexp(1.0, e[k]));
                w.qlo[k][s] = static_cast<uint8_t>(std::min(255.0, std::max(0.0, q0)));
                w.qhi[k][s] = static_cast<uint8_t>(std::min(255.0, std::max(0.0, q1)));
            }
            if (it.kind == CHUNK) {
                const uint32_t off = static_cast<uint32_t>(rank.size()) - w.tri_base;
                w.meta[s] = static_cast<uint8_t>((((1u << it.count) - 1u) << 5) | off);
                for (uint32_t t = 0; t < it.count; ++t) rank.push_back(it.first + t);
            } else {
                w.imask |= static_cast<uint8_t>(1u << s);
                inner_child[ni++] = c;
            }
        }
        out[idx] = w;
        // the inner children, in slot order, at child_base + 0, 1, ...
        kids.n = ni;
        for (int k = 0; k < ni; ++k) {
            const Item& it = ch.v[inner_child[k]];
            kids.idx[k] = w.child_base + static_cast<uint32_t>(k);
            kids.items[k] = it.kind == INNER ? collapse(it.node) : leaf_children(it.first, it.count, it.box);
        }
    }

    // the subtree below idx, depth first: a node's children, then each child's subtree in slot order
    void fill(uint32_t idx, const Items& items) {
        Kids kids;
        fill_node(idx, items, kids);
        for (int k = 0; k < kids.n; ++k) fill(kids.idx[k], kids.items[k]);
    }
};

}  // namespace

void build_wide(const std::vector<spt_bvh2_node>& nodes, WideBvh& out) {
    out.nodes.clear();
    out.tri_rank.clear();
    if (nodes.empty()) return;
    std::vector<WideNode> built;
    Collapser c{nodes, built, out.tri_rank};
    built.resize(1);
    Collapser::Kids kids;
    c.fill_node(0, nodes[0].count ? c.leaf_children(nodes[0].right, nodes[0].count, node_box(nodes[0])) : c.collapse(0),
                kids);
    // The root's inner children's subtrees are independent: each is built on its own thread into
    // local arrays (its root at local 0), then spliced in slot order.  Sequentially each subtree's
    // triangles form one run, in slot order, so the triangle order is the same as a one-thread
    // build; node numbering does not matter because the breadth-first pass below renumbers.
    struct Sub {
        std::vector<WideNode> nodes;
        std::vector<uint32_t> rank;
    };
    std::vector<Sub> subs(kids.n);
    {
        auto build_sub = [&](int k) {
            Collapser ck{nodes, subs[k].nodes, subs[k].rank};
            subs[k].nodes.resize(1);
            ck.fill(0, kids.items[k]);
        };
        std::vector<std::thread> pool;
        for (int k = 0; k < kids.n; ++k) {
            if (nodes.size() >= 16384) pool.emplace_back(build_sub, k);   // small trees: no thread start-up
            else build_sub(k);
        }
        for (auto& t : pool) t.join();
    }
    for (int k = 0; k < kids.n; ++k) {
        const uint32_t tri_off = static_cast<uint32_t>(out.tri_rank.size());
        const uint32_t node_off = static_cast<uint32_t>(built.size()) - 1;   // local j >= 1 -> node_off + j
        for (size_t j = 0; j < subs[k].nodes.size(); ++j) {
            WideNode w = subs[k].nodes[j];
            w.tri_base += tri_off;
            w.child_base += node_off;   // children are never local 0 (a leaf-only node keeps the index
                                        // the next node would get, as in a one-thread build)
            if (j == 0) built[kids.idx[k]] = w;
            else built.push_back(w);
        }
        out.tri_rank.insert(out.tri_rank.end(), subs[k].rank.begin(), subs[k].rank.end());
    }
    // breadth-first order: the top levels, which every ray visits, share cache lines, and a node's
    // inner children stay consecutive
    std::vector<uint32_t> order;
    order.reserve(built.size());
    order.push_back(0);
    for (size_t q = 0; q < order.size(); ++q) {
        const WideNode& w = built[order[q]];
        const uint32_t n_inner = static_cast<uint32_t>(__builtin_popcount(w.imask));
        for (uint32_t k = 0; k < n_inner; ++k) order.push_back(w.child_base + k);
    }
    std::vector<uint32_t> new_id(built.size());
    for (size_t q = 0; q < order.size(); ++q) new_id[order[q]] = static_cast<uint32_t>(q);
    out.nodes.resize(built.size());
    for (size_t q = 0; q < order.size(); ++q) {
        WideNode w = built[order[q]];
        if (w.imask) w.child_base = new_id[w.child_base];
        out.nodes[q] = w;
    }
}

}  // namespace spt
