// Where every lit surface sits in the lightmap: crates/lightbaker/src/layout.rs. Charts by region
// growing, each on its own plane; a tile packs its charts (skyline, quarter turns); tiles are shelved
// into the atlas on a 4-texel grid. The same scene always gives the same layout.
#pragma once
#include <array>
#include <cstdint>
#include <utility>
#include <vector>

#include "scene.h"
#include "vec.h"

namespace lb {

constexpr uint32_t ALIGN = 4;  // layout.rs:17-18
using TileKey = std::pair<int32_t, int32_t>;

struct Tile;

struct Chart {  // layout.rs:20-40
    uint32_t mesh;
    std::vector<uint32_t> tris;
    Vec3 normal, u, v;
    Vec2 min, max;
    TileKey tile;
    bool turned = false;
    uint32_t w = 0, h = 0, x = 0, y = 0;
    Vec2 local(Vec3 p, float density, uint32_t padding) const;                               // layout.rs:69-74
    std::array<std::array<float, 4>, 2> affine(const Tile &t, float density, uint32_t padding) const;  // :76-85
};

struct Tile {  // layout.rs:45-54
    TileKey key;
    std::vector<uint32_t> charts;
    uint32_t w = 0, h = 0, x = 0, y = 0;
};

struct Layout {  // layout.rs:56-66
    std::vector<Chart> charts;
    std::vector<Tile> tiles;
    uint32_t width = 0, height = 0;
    float density = 0;
    uint32_t padding = 0;
    std::vector<std::vector<uint32_t>> tri_chart;
    static Layout build(const Scene &scene);  // throws std::runtime_error when a tile is wider than the atlas
    std::vector<uint32_t> chart_tile() const;
};

Vec3 face_normal(const std::vector<Vec3> &pos, size_t t);  // layout.rs:333-335
Vec3 box_centre(const std::vector<Vec3> &pos, size_t t);   // :341-345
TileKey tile_of(Vec3 p, float size);                       // :347-349

}  // namespace lb
