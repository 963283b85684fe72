// bvh_build.h -- host build of the reference's full-sweep SAH binary tree.
#pragma once

#include <cstdint>
#include <vector>

#include "../../include/spt.h"

namespace spt {

struct HostBox {
    float mn[3], mx[3];
};

// The flattened tree: nodes in depth-first, left-first order (spt_bvh2_node semantics) and the
// primitive id of every leaf reference in leaf order.
struct HostBvh {
    std::vector<spt_bvh2_node> nodes;
    std::vector<uint32_t> refs;
    spt_bvh_stats stats{};
};

// Builds the tree the reference's SBVH::build makes for the same primitives
// (acceleration/sbvh.cpp:12-37, 58-421): per node, for axis x, y, z in turn, std::sort the
// references by centroid (each sort starting from the previous one's order), sweep prefix and
// suffix boxes, and keep the first split whose SAH cost 2*1.2 + (A_L/A)*N_L + (A_R/A)*N_R beats the
// leaf cost N; children are inflated by 1e-3.  Independent subtrees are built on worker threads;
// the result does not depend on the thread count.  Returns false on an input it cannot build.
bool build_sah_tree(const spt_scene_desc& desc, int n_threads, HostBvh& out, const char** err);

// Fills out.stats (all but build_ms) from out.nodes, as SBVH::collectTreeStatistics counts them.
void tree_statistics(HostBvh& out);

// Primitive bounds and centroid exactly as the reference computes them
// (primitives/triangle.cpp:76-87, primitives/sphere.cpp:48-60).
void prim_bounds(const spt_scene_desc& desc, uint32_t i, HostBox& box, float centroid[3]);

}  // namespace spt
