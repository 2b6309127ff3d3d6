#include "raster.h"

#include <climits>
#include <cmath>

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

// raster.rs:39-100
std::vector<lb_texel> rasterize(const Scene &scene, const Layout &layout, const Tile &tile) {
    int32_t w = int32_t(tile.w), h = int32_t(tile.h);
    std::vector<lb_texel> out(size_t(w) * size_t(h), lb_texel{});
    for (int conservative = 0; conservative < 2; conservative++) {
        for (uint32_t ci : tile.charts) {
            const Chart &c = layout.charts[ci];
            const std::vector<Vec3> &pos = scene.positions[c.mesh];
            for (uint32_t tt : c.tris) {
                size_t t = tt;
                Vec3 pa = pos[t * 3], pb = pos[t * 3 + 1], pc = pos[t * 3 + 2];
                Vec2 ua = c.local(pa, layout.density, layout.padding), ub = c.local(pb, layout.density, layout.padding),
                     uc = c.local(pc, layout.density, layout.padding);
                float det = (ub.y - uc.y) * (ua.x - uc.x) + (uc.x - ub.x) * (ua.y - uc.y);
                if (std::fabs(det) < 1e-12f) continue;
                auto bary = [&](Vec2 q, float &l1, float &l2, float &l3) {
                    l1 = ((ub.y - uc.y) * (q.x - uc.x) + (uc.x - ub.x) * (q.y - uc.y)) / det;
                    l2 = ((uc.y - ua.y) * (q.x - uc.x) + (ua.x - uc.x) * (q.y - uc.y)) / det;
                    l3 = 1.0f - l1 - l2;
                };
                auto at = [&](Vec2 q) {
                    float l1, l2, l3;
                    bary(q, l1, l2, l3);
                    return (pa * l1 + pb * l2) + pc * l3;
                };
                Vec3 n = face_normal(pos, t);
                Vec3 o = at(Vec2(0, 0));
                Vec3 dx = at(Vec2(1, 0)) - o, dy = at(Vec2(0, 1)) - o;
                Vec2 lo = ua.min(ub).min(uc).floor().max(Vec2(0, 0));
                Vec2 hi = ua.max(ub).max(uc).ceil().min(Vec2(float(w - 1), float(h - 1)));
                for (int32_t y = as_i32(lo.y); y <= as_i32(hi.y); y++)
                    for (int32_t x = as_i32(lo.x); x <= as_i32(hi.x); x++) {
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
