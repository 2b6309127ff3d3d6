// The BVH over the scene's casting triangles: crates/lightbaker/src/bvh.rs. Binned surface area
// heuristic (16 bins, leaves of at most 4), built on the CPU, flattened for the traversal.
#pragma once
#include <array>
#include <cstdint>
#include <functional>
#include <vector>

#include "../../../include/lightbaker.h"
#include "scene.h"

namespace lb {

struct Bvh {
    std::vector<lb_node> nodes;
    std::vector<lb_tri> tris;
    // each triangle's vertices as the scene holds them (9 floats, in `tris` order): v0 = tris[i].v0
    // exactly, while v0 + e1 and v0 + e2 may round; the watertight test reads these
    std::vector<float> verts;
    // each triangle's mesh and its index there, in `tris` order
    std::vector<std::array<uint32_t, 2>> source;
    // chart(mesh, triangle): the triangle's chart (0xffffffff: none); called from several threads at once
    static Bvh build(const Scene &scene, const std::function<uint32_t(size_t, size_t)> &chart);
    // the triangles' chart bits (e1.w) written again from chart(mesh, triangle): a BVH built before the layout
    // (the tree does not depend on them) gets the bits a build after it would have written
    void set_charts(const std::function<uint32_t(size_t, size_t)> &chart);
};

}  // namespace lb
