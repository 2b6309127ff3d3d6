// A tile's texels: crates/lightbaker/src/raster.rs. Every texel whose centre a chart's triangle covers,
// then, conservatively, every texel a triangle only touches, sampled at the triangle's nearest point.
#pragma once
#include <vector>

#include "../../../include/lightbaker.h"
#include "layout.h"

namespace lb {

inline bool covered(const lb_texel &t) { return t.pos[3] > 0.5f; }
inline uint32_t texel_chart(const lb_texel &t) { return f2u(t.normal[3]); }

// The tile's texels, row by row in its own rectangle (tile.w x tile.h).
std::vector<lb_texel> rasterize(const Scene &scene, const Layout &layout, const Tile &tile);

}  // namespace lb

// One chart triangle of a tile as the rasteriser sets it up (raster.rs:48-67): its corners in chart
// space, their determinant, the corners in the world, the face normal, the world steps of one texel in
// x and y, its texel box (inclusive, clamped to the tile), its chart and the tile's index in a list of
// tiles. 128 bytes, for the device rasteriser (raster.cu).
struct RasterTri {
    float ua[2], ub[2], uc[2], det;
    float pa[3], pb[3], pc[3], n[3], dx[3], dy[3];
    int32_t x0, y0, x1, y1;
    uint32_t chart, tile, pad;
};
static_assert(sizeof(RasterTri) == 128, "a raster triangle is 128 bytes");

namespace lb {

// The tile's triangles in the order rasterize() visits them (charts in tile order, each chart's
// triangles in order), set up with the same arithmetic; degenerate ones (|det| < 1e-12) left out.
std::vector<RasterTri> raster_triangles(const Scene &scene, const Layout &layout, const Tile &tile, uint32_t tile_index);
// The same for several tiles, concatenated in list order (tile k's triangles carry tile index k): the work
// is split into equal runs of (chart, triangle) pairs across the tiles, set up by all host threads, so one
// large tile does not hold up the rest.
std::vector<RasterTri> raster_triangles(const Scene &scene, const Layout &layout, const std::vector<size_t> &tiles);

}  // namespace lb
