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
