// The BVH over the scene's casting triangles: crates/lightbaker/src/bvh.rs. Binned surface area
// heuristic (16 bins, leaves of at most 4), built on the CPU, flattened for the traversal.
#pragma once
#include <cstdint>
#include <functional>
#include <vector>

#include "../../../include/lightbaker.h"
#include "scene.h"

namespace lb {

struct Bvh {
    std::vector<lb_node> nodes;
    std::vector<lb_tri> tris;
    // chart(mesh, triangle): the triangle's chart (0xffffffff: none)
    static Bvh build(const Scene &scene, const std::function<uint32_t(size_t, size_t)> &chart);
};

}  // namespace lb
