// wide_build.cpp -- collapse the reference binary tree into 8-wide quantized nodes (wide_build.h).
//
// Greedy collapse (the surface-area heuristic of wide-BVH literature, e.g. Ylitie, Karras, Laine,
// "Efficient Incoherent Ray Traversal on GPUs Through Compressed Wide BVHs", HPG 2017): starting from
// a binary node's two children, repeatedly open the inner child with the largest box area while the
// children still fit in 8 slots.  A binary leaf of k references takes ceil(k/3) slots (three
// triangles per slot); a leaf too large for the free slots becomes a wide node of its own.
// The boxes are the reference's boxes, quantized outward; triangles keep their reference slot
// ("rank") so that hits still resolve exactly as the reference's traversal order would.
#include "wide_build.h"

#include <algorithm>
#include <cmath>
#include <cstring>

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
    std::vector<Item> collapse(uint32_t i) const {
        std::vector<Item> items{item_of(i + 1), item_of(bn[i].right)};
        auto used = [&]() {
            int u = 0;
            for (const Item& it : items) u += cost(it);
            return u;
        };
        // two big leaves may not fit together: turn the costliest into nodes of their own
        while (used() > 8) {
            auto it = std::max_element(items.begin(), items.end(),
                                       [](const Item& a, const Item& b) { return cost(a) < cost(b); });
            it->kind = LEAFNODE;
        }
        for (;;) {
            int best = -1;
            double best_area = -1.0;
            const int u = used();
            for (size_t k = 0; k < items.size(); ++k) {
                if (items[k].kind != INNER) continue;
                const uint32_t n = items[k].node;
                Item l = item_of(n + 1), r = item_of(bn[n].right);
                if (u - 1 + cost(l) + cost(r) > 8) continue;
                double a = area(items[k].box);
                if (a > best_area) {
                    best_area = a;
                    best = static_cast<int>(k);
                }
            }
            if (best < 0) break;
            const uint32_t n = items[best].node;
            items[best] = item_of(n + 1);
            items.push_back(item_of(bn[n].right));
        }
        return items;
    }

    // children of a wide node that holds one large leaf's references
    std::vector<Item> leaf_children(uint32_t first, uint32_t count, const Box& box) const {
        std::vector<Item> items;
        if (count <= 24) {
            for (uint32_t s = 0; s < count; s += 3) items.push_back(Item{CHUNK, 0, first + s, std::min(3u, count - s), box});
        } else {
            const uint32_t per = (count + 7) / 8;
            for (uint32_t s = 0; s < count; s += per)
                items.push_back(Item{LEAFNODE, 0, first + s, std::min(per, count - s), box});
        }
        return items;
    }

    void fill(uint32_t idx, std::vector<Item> items) {
        // expand LEAF items into chunks of up to three triangles
        std::vector<Item> ch;
        for (const Item& it : items) {
            if (it.kind == LEAF)
                for (uint32_t s = 0; s < it.count; s += 3)
                    ch.push_back(Item{CHUNK, it.node, it.first + s, std::min(3u, it.count - s), it.box});
            else
                ch.push_back(it);
        }
        // node box and quantization grid
        Box nb = ch[0].box;
        for (const Item& it : ch)
            for (int k = 0; k < 3; ++k) {
                nb.mn[k] = std::min(nb.mn[k], it.box.mn[k]);
                nb.mx[k] = std::max(nb.mx[k], it.box.mx[k]);
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
        // slot assignment by direction (greedy on the centre offsets)
        double cx = 0.5 * (double(nb.mn[0]) + nb.mx[0]), cy = 0.5 * (double(nb.mn[1]) + nb.mx[1]),
               cz = 0.5 * (double(nb.mn[2]) + nb.mx[2]);
        struct Cand {
            double score;
            int child, slot;
        };
        std::vector<Cand> cand;
        for (size_t c = 0; c < ch.size(); ++c) {
            double dx = 0.5 * (double(ch[c].box.mn[0]) + ch[c].box.mx[0]) - cx;
            double dy = 0.5 * (double(ch[c].box.mn[1]) + ch[c].box.mx[1]) - cy;
            double dz = 0.5 * (double(ch[c].box.mn[2]) + ch[c].box.mx[2]) - cz;
            for (int s = 0; s < 8; ++s)
                cand.push_back(Cand{((s & 1) ? dx : -dx) + ((s & 2) ? dy : -dy) + ((s & 4) ? dz : -dz),
                                    static_cast<int>(c), s});
        }
        std::stable_sort(cand.begin(), cand.end(), [](const Cand& a, const Cand& b) { return a.score > b.score; });
        int slot_of[8], child_in[8];
        std::fill(slot_of, slot_of + 8, -1);
        std::fill(child_in, child_in + 8, -1);
        for (const Cand& c : cand)
            if (slot_of[c.child] < 0 && child_in[c.slot] < 0) {
                slot_of[c.child] = c.slot;
                child_in[c.slot] = c.child;
            }
        // leaf triangles (consecutive, slot order) and inner children (consecutive, slot order)
        w.tri_base = static_cast<uint32_t>(rank.size());
        std::vector<std::pair<uint32_t, std::vector<Item>>> inner;  // (node index, its items)
        uint32_t n_inner = 0;
        for (int s = 0; s < 8; ++s)
            if (child_in[s] >= 0 && ch[child_in[s]].kind != CHUNK) ++n_inner;
        w.child_base = static_cast<uint32_t>(out.size());
        out.resize(out.size() + n_inner);
        uint32_t next_inner = w.child_base;
        for (int s = 0; s < 8; ++s) {
            const int c = child_in[s];
            if (c < 0) continue;
            const Item& it = ch[c];
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
                if (it.kind == INNER)
                    inner.push_back({next_inner++, collapse(it.node)});
                else
                    inner.push_back({next_inner++, leaf_children(it.first, it.count, it.box)});
            }
        }
        out[idx] = w;
        for (auto& p : inner) fill(p.first, std::move(p.second));
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
    if (nodes[0].count) {
        c.fill(0, c.leaf_children(nodes[0].right, nodes[0].count, node_box(nodes[0])));
    } else {
        c.fill(0, c.collapse(0));
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
