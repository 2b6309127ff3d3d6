// An 8-wide BVH collapsed from the reference's BVH2 (crates/lightbaker/src/bvh.rs), compressed for the
// device: a node is 80 bytes, five 128-bit loads:
//   [0] origin p.xyz (f32), exponents ex, ey, ez (biased bytes) and the inner-child mask
//   [1] first inner child, first triangle, slot bytes 0..3 and 4..7 (a leaf slot: triangle offset from
//       the node's first triangle in bits 0..4, count - 1 in bits 5..6; 0xff: empty slot)
//   [2..4] child boxes quantized to 8 bits an axis: lo x, lo y, lo z, hi x, hi y, hi z (8 slots each)
// A child box dequantized in float (p + q * 2^e) contains the child's exact box (checked as built),
// so the walk visits every node the exact boxes would. Inner children of a node are stored one after
// another; the triangles of its leaf slots too, in a copy of the triangle array whose e2.w holds each
// triangle's index in the reference's array (the opacity coin, trace.wgsl:69-72, and the hit records
// use that index).
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "../../../include/lightbaker.h"

namespace lb {

struct Bvh8 {
    std::vector<uint32_t> nodes;  // 20 words a node
    std::vector<lb_tri> tris;     // leaf order; e2.w: the reference index's bits
    size_t n_nodes() const { return nodes.size() / 20; }
    static Bvh8 collapse(const lb_node *nodes, size_t n_nodes, const lb_tri *tris, size_t n_tris);
};

std::string bvh8_check(const Bvh8 &b, size_t n_tris, size_t &depth);

}  // namespace lb
