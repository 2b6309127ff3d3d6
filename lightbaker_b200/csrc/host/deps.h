// What a tile's light depends on, as one hash: crates/lightbaker/src/deps.rs. Its own surfaces, every
// casting triangle within reach of it or between that and the sun, the settings and BAKER_VERSION.
#pragma once
#include <array>
#include <string>
#include <vector>

#include "blake3.h"
#include "scene.h"

namespace lb {

constexpr uint32_t BAKER_VERSION = 11;  // deps.rs:10-11

struct Aabb {  // deps.rs:13-31
    Vec3 min = Vec3::splat(INFINITY), max = Vec3::splat(-INFINITY);
    void add(Vec3 p) {
        min = min.min(p);
        max = max.max(p);
    }
    Aabb grow(float r) const { return Aabb{min - r, max + r}; }
};

struct Boxes {  // deps.rs:33-57
    std::vector<std::vector<Aabb>> boxes;
    float top = -INFINITY;
    explicit Boxes(const Scene &scene);
};

using Hash = std::array<uint8_t, 32>;
Hash global_hash(const Scene &scene);  // deps.rs:59-68
// global_hash for a bake with the watertight triangle test (beyond the reference): its tiles and chunks
// are cached apart from the shader's
Hash watertight_hash(const Hash &global);
// deps.rs:70-96
Hash hash_reach(const Scene &scene, const Boxes &boxes, const Hash &global, const Aabb &own, float reach,
                const std::vector<uint8_t> &seed);
bool swept(const Aabb &zone, Vec3 sun, float top, const Aabb &b);  // deps.rs:98-121

}  // namespace lb
