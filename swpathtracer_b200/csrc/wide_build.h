// wide_build.h -- collapse of the reference's binary SAH tree into an 8-wide, quantized BVH.
#pragma once

#include <cstdint>
#include <vector>

#include "../../include/spt.h"

namespace spt {

// One 80-byte node, five 16-byte words:
//   w0: origin p (3 floats), then 4 bytes: exponent x, y, z (int8) and the inner-child mask
//   w1: index of the first inner child node, index of the first leaf triangle, meta[8]
//   w2..w4: quantized child boxes, one byte per child: lo x, lo y, lo z, hi x, hi y, hi z
// Child j's box is p + 2^e * q (per axis), rounded outward, so it contains the reference box.
// Children sit in slots by direction: slot bit k set <=> the child's centre lies on the + side of the
// node centre along axis k; a ray visits hit children in the order slot ^ (7 - ray octant).
// Inner children are stored consecutively in slot order from the first-child index; a leaf child's
// meta byte is (mask of its 1..3 triangles << 5) | offset of its first triangle from the first leaf
// triangle (< 32); an empty slot has meta 0 and no inner bit.
struct WideNode {
    float px, py, pz;
    int8_t ex, ey, ez;
    uint8_t imask;
    uint32_t child_base;
    uint32_t tri_base;
    uint8_t meta[8];
    uint8_t qlo[3][8];
    uint8_t qhi[3][8];
};
static_assert(sizeof(WideNode) == 80, "WideNode must be 80 bytes");

struct WideBvh {
    std::vector<WideNode> nodes;
    std::vector<uint32_t> tri_rank;  // wide triangle order -> reference slot (depth-first leaf order)
};

// nodes/refs: the flattened reference tree (spt_bvh2_node, depth-first left-first).
void build_wide(const std::vector<spt_bvh2_node>& nodes, WideBvh& out);

}  // namespace spt
