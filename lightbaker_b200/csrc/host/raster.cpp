#include "raster.h"

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>

namespace lb {

namespace {
inline float signum(float x) { return std::isnan(x) ? x : std::copysign(1.0f, x); }
inline float clampf(float v, float lo, float hi) { return v < lo ? lo : (v > hi ? hi : v); }
inline int32_t as_i32(float f) {
    if (std::isnan(f)) return 0;
    if (f <= -2147483648.0f) return INT32_MIN;
    if (f >= 2147483647.0f) return INT32_MAX;
    return int32_t(f);
}

// raster.rs:102-114: the point of triangle (a, b, c) nearest p (2D)
Vec2 nearest(Vec2 p, Vec2 a, Vec2 b, Vec2 c) {
    auto side = [](Vec2 o, Vec2 e, Vec2 q) { return (e - o).perp_dot(q - o); };
    float s = signum(side(a, b, c));
    if (side(a, b, p) * s >= 0.0f && side(b, c, p) * s >= 0.0f && side(c, a, p) * s >= 0.0f) return p;
    auto seg = [&](Vec2 o, Vec2 e) {
        Vec2 d = e - o;
        return o + d * clampf((p - o).dot(d) / std::fmax(d.length_squared(), 1e-12f), 0.0f, 1.0f);
    };
    Vec2 cand[3] = {seg(a, b), seg(b, c), seg(c, a)};
    Vec2 best = cand[0];
    float bd = best.distance_squared(p);
    for (int k = 1; k < 3; k++) {
        float d = cand[k].distance_squared(p);
        if (d < bd) {  // the first of equals, as min_by
            bd = d;
            best = cand[k];
        }
    }
    return best;
}
}  // namespace

namespace {
// raster.rs:48-67: one chart triangle's set-up; false for a degenerate one
struct Setup {
    Vec2 ua, ub, uc;
    float det;
    Vec3 pa, pb, pc, n, dx, dy;
    int32_t x0, y0, x1, y1;
    void bary(Vec2 q, float &l1, float &l2, float &l3) const {
        l1 = ((ub.y - uc.y) * (q.x - uc.x) + (uc.x - ub.x) * (q.y - uc.y)) / det;
        l2 = ((uc.y - ua.y) * (q.x - uc.x) + (ua.x - uc.x) * (q.y - uc.y)) / det;
        l3 = 1.0f - l1 - l2;
    }
    Vec3 at(Vec2 q) const {
        float l1, l2, l3;
        bary(q, l1, l2, l3);
        return (pa * l1 + pb * l2) + pc * l3;
    }
};
bool setup(const Layout &layout, const Chart &c, const std::vector<Vec3> &pos, size_t t, int32_t w, int32_t h,
           Setup &s) {
    s.pa = pos[t * 3];
    s.pb = pos[t * 3 + 1];
    s.pc = pos[t * 3 + 2];
    s.ua = c.local(s.pa, layout.density, layout.padding);
    s.ub = c.local(s.pb, layout.density, layout.padding);
    s.uc = c.local(s.pc, layout.density, layout.padding);
    s.det = (s.ub.y - s.uc.y) * (s.ua.x - s.uc.x) + (s.uc.x - s.ub.x) * (s.ua.y - s.uc.y);
    if (std::fabs(s.det) < 1e-12f) return false;
    s.n = face_normal(pos, t);
    Vec3 o = s.at(Vec2(0, 0));
    s.dx = s.at(Vec2(1, 0)) - o;
    s.dy = s.at(Vec2(0, 1)) - o;
    Vec2 lo = s.ua.min(s.ub).min(s.uc).floor().max(Vec2(0, 0));
    Vec2 hi = s.ua.max(s.ub).max(s.uc).ceil().min(Vec2(float(w - 1), float(h - 1)));
    s.x0 = as_i32(lo.x);
    s.y0 = as_i32(lo.y);
    s.x1 = as_i32(hi.x);
    s.y1 = as_i32(hi.y);
    return true;
}
}  // namespace

std::vector<RasterTri> raster_triangles(const Scene &scene, const Layout &layout, const Tile &tile,
                                        uint32_t tile_index) {
    std::vector<RasterTri> out;
    for (uint32_t ci : tile.charts) {
        const Chart &c = layout.charts[ci];
        const std::vector<Vec3> &pos = scene.positions[c.mesh];
        for (uint32_t tt : c.tris) {
            Setup s;
            if (!setup(layout, c, pos, tt, int32_t(tile.w), int32_t(tile.h), s)) continue;
            out.push_back(RasterTri{{s.ua.x, s.ua.y}, {s.ub.x, s.ub.y}, {s.uc.x, s.uc.y}, s.det,
                                    {s.pa.x, s.pa.y, s.pa.z}, {s.pb.x, s.pb.y, s.pb.z}, {s.pc.x, s.pc.y, s.pc.z},
                                    {s.n.x, s.n.y, s.n.z}, {s.dx.x, s.dx.y, s.dx.z}, {s.dy.x, s.dy.y, s.dy.z},
                                    s.x0, s.y0, s.x1, s.y1, ci, tile_index, 0});
        }
    }
    return out;
}

std::vector<RasterTri> raster_triangles(const Scene &scene, const Layout &layout, const std::vector<size_t> &tiles) {
    // every (tile, chart) in order, with the count of (chart, triangle) pairs before it
    struct Span {
        uint32_t tile_k, chart;
        size_t first;
    };
    std::vector<Span> spans;
    size_t total = 0;
    for (size_t k = 0; k < tiles.size(); k++)
        for (uint32_t ci : layout.tiles[tiles[k]].charts) {
            spans.push_back(Span{uint32_t(k), ci, total});
            total += layout.charts[ci].tris.size();
        }
    const size_t RUN = 16384, runs = (total + RUN - 1) / RUN;
    std::vector<std::vector<RasterTri>> part(runs);
#pragma omp parallel for schedule(dynamic, 1)
    for (long long r = 0; r < (long long)runs; r++) {
        const size_t lo = size_t(r) * RUN, hi = std::min(total, lo + RUN);
        // the span holding pair `lo`, then on in order
        size_t si = size_t(std::upper_bound(spans.begin(), spans.end(), lo,
                                            [](size_t v, const Span &sp) { return v < sp.first; }) -
                           spans.begin()) -
                    1;
        std::vector<RasterTri> &out = part[size_t(r)];
        out.reserve(hi - lo);
        for (size_t at = lo; at < hi; si++) {
            const Span &sp = spans[si];
            const Tile &tile = layout.tiles[tiles[sp.tile_k]];
            const Chart &c = layout.charts[sp.chart];
            const std::vector<Vec3> &pos = scene.positions[c.mesh];
            for (size_t j = at - sp.first; j < c.tris.size() && at < hi; j++, at++) {
                Setup s;
                if (!setup(layout, c, pos, c.tris[j], int32_t(tile.w), int32_t(tile.h), s)) continue;
                out.push_back(RasterTri{{s.ua.x, s.ua.y}, {s.ub.x, s.ub.y}, {s.uc.x, s.uc.y}, s.det,
                                        {s.pa.x, s.pa.y, s.pa.z}, {s.pb.x, s.pb.y, s.pb.z}, {s.pc.x, s.pc.y, s.pc.z},
                                        {s.n.x, s.n.y, s.n.z}, {s.dx.x, s.dx.y, s.dx.z}, {s.dy.x, s.dy.y, s.dy.z},
                                        s.x0, s.y0, s.x1, s.y1, sp.chart, sp.tile_k, 0});
            }
        }
    }
    std::vector<size_t> first(runs + 1, 0);
    for (size_t r = 0; r < runs; r++) first[r + 1] = first[r] + part[r].size();
    std::vector<RasterTri> out(first.back());
#pragma omp parallel for schedule(dynamic, 1)
    for (long long r = 0; r < (long long)runs; r++)
        if (!part[size_t(r)].empty())
            std::memcpy(out.data() + first[size_t(r)], part[size_t(r)].data(), part[size_t(r)].size() * sizeof(RasterTri));
    return out;
}

// raster.rs:39-100
std::vector<lb_texel> rasterize(const Scene &scene, const Layout &layout, const Tile &tile) {
    int32_t w = int32_t(tile.w), h = int32_t(tile.h);
    std::vector<lb_texel> out(size_t(w) * size_t(h), lb_texel{});
    for (int conservative = 0; conservative < 2; conservative++) {
        for (uint32_t ci : tile.charts) {
            const Chart &c = layout.charts[ci];
            const std::vector<Vec3> &pos = scene.positions[c.mesh];
            for (uint32_t tt : c.tris) {
                Setup s;
                if (!setup(layout, c, pos, tt, w, h, s)) continue;
                const Vec2 ua = s.ua, ub = s.ub, uc = s.uc;
                const Vec3 pa = s.pa, pb = s.pb, pc = s.pc, n = s.n, dx = s.dx, dy = s.dy;
                auto bary = [&](Vec2 q, float &l1, float &l2, float &l3) { s.bary(q, l1, l2, l3); };
                for (int32_t y = s.y0; y <= s.y1; y++)
                    for (int32_t x = s.x0; x <= s.x1; x++) {
                        Vec2 centre(float(x) + 0.5f, float(y) + 0.5f);
                        size_t i = size_t(y) * size_t(w) + size_t(x);
                        if (covered(out[i])) continue;
                        Vec2 q = conservative ? nearest(centre, ua, ub, uc) : centre;
                        if (conservative && (std::fabs(q.x - centre.x) > 0.5f || std::fabs(q.y - centre.y) > 0.5f))
                            continue;
                        float l1, l2, l3;
                        bary(q, l1, l2, l3);
                        if (!conservative && (l1 < -1e-4f || l2 < -1e-4f || l3 < -1e-4f)) continue;
                        Vec3 p = (pa * l1 + pb * l2) + pc * l3;
                        out[i] = lb_texel{{p.x, p.y, p.z, 1.0f}, {n.x, n.y, n.z, u2f(ci)}, {dx.x, dx.y, dx.z, 0.0f},
                                          {dy.x, dy.y, dy.z, 0.0f}};
                    }
            }
        }
    }
    return out;
}

}  // namespace lb
