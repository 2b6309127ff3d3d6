// ORACLE — test infrastructure only (see oracle.h). The reference's CPU work between the GPU passes,
// restated from its Rust source with glam's operation order (every Vec3/Vec2 operation componentwise,
// dot products left to right, no fused multiply-add), sharing no code with the product:
//   or_raster_tile      crates/lightbaker/src/raster.rs:39-114 (with Chart::local, layout.rs:69-74, and
//                       face_normal, layout.rs:333-335)
//   or_chart_affine     layout.rs:76-85
//   or_tile_post        bake.rs:197-275 (inside test, sample point moves, occlusion curve, smoothing,
//                       the sun's field, direct light, fills, validity)
//   or_gather_select    bake.rs:286-298
//   or_bounce_tile      bake.rs:303-322
//   or_write_light      bake.rs:435-445
//   or_volume_fill      volume.rs:86-120
//   or_volume_fallback  bake.rs:337-359 with Volume::irradiance, volume.rs:125-147
//   or_composite        bake.rs:364-421
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <set>
#include <utility>
#include <vector>

#include "oracle.h"

namespace {

struct V2 {
    float x, y;
};
struct V3 {
    float x, y, z;
};
inline V3 v3(const float *p) { return {p[0], p[1], p[2]}; }
inline V3 add(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 mul(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
inline float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
// glam Vec3::cross
inline V3 cross(V3 a, V3 b) { return {a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y}; }
inline V2 sub2(V2 a, V2 b) { return {a.x - b.x, a.y - b.y}; }
inline V2 add2(V2 a, V2 b) { return {a.x + b.x, a.y + b.y}; }
inline V2 mul2(V2 a, float s) { return {a.x * s, a.y * s}; }
inline float dot2(V2 a, V2 b) { return a.x * b.x + a.y * b.y; }
inline float perp_dot(V2 a, V2 b) { return a.x * b.y - a.y * b.x; }
// Rust f32::signum: +1 for +0 and positives, -1 for -0 and negatives, NaN for NaN
inline float signum(float v) { return std::isnan(v) ? v : (std::signbit(v) ? -1.0f : 1.0f); }
// Rust f32::clamp (NaN stays NaN)
inline float clampf(float v, float lo, float hi) {
    if (v < lo) v = lo;
    if (v > hi) v = hi;
    return v;
}
// Rust f32::total_cmp's order as a key: a < b in total order iff key(a) < key(b)
inline int32_t total_key(float v) {
    int32_t b;
    std::memcpy(&b, &v, 4);
    return b ^ int32_t(uint32_t(b >> 31) >> 1);
}
inline uint32_t bits(float v) {
    uint32_t b;
    std::memcpy(&b, &v, 4);
    return b;
}
inline float from_bits(uint32_t b) {
    float v;
    std::memcpy(&v, &b, 4);
    return v;
}

constexpr uint32_t NONE = 0xffffffffu;
constexpr float PUSH = 0.03f;  // bake.rs:27
constexpr uint8_t V_NONE = 0, V_CENTRE = 1, V_OFFSET = 2, V_PUSHED = 3, V_FILLED = 4, V_VOLUME = 5;  // output.rs:29-40

// layout.rs:69-74
V2 chart_local(const or_chart *c, V3 p, float density, uint32_t padding) {
    V3 u = v3(c->u), v = v3(c->v);
    V2 a = mul2(sub2(V2{dot(p, u), dot(p, v)}, V2{c->min[0], c->min[1]}), density);
    if (c->turned) a = V2{a.y, a.x};
    float pad = float(padding) + 0.5f;
    return add2(add2(V2{float(c->x), float(c->y)}, V2{pad, pad}), a);
}

// raster.rs:117-129
V2 nearest(V2 p, V2 a, V2 b, V2 c) {
    auto side = [](V2 o, V2 e, V2 q) { return perp_dot(sub2(e, o), sub2(q, o)); };
    float s = signum(side(a, b, c));
    if (side(a, b, p) * s >= 0.0f && side(b, c, p) * s >= 0.0f && side(c, a, p) * s >= 0.0f) return p;
    auto seg = [&](V2 o, V2 e) {
        V2 d = sub2(e, o);
        float den = std::fmax(dot2(d, d), 1e-12f);  // f32::max: the larger, a NaN operand ignored
        return add2(o, mul2(d, clampf(dot2(sub2(p, o), d) / den, 0.0f, 1.0f)));
    };
    V2 cand[3] = {seg(a, b), seg(b, c), seg(c, a)};
    int best = 0;
    for (int k = 1; k < 3; k++) {  // min_by keeps the first of equal minima
        V2 dk = sub2(cand[k], p), db = sub2(cand[best], p);
        if (total_key(dot2(dk, dk)) < total_key(dot2(db, db))) best = k;
    }
    return cand[best];
}

}  // namespace

extern "C" {

void or_chart_affine(const or_chart *c, uint32_t tile_x, uint32_t tile_y, float density, uint32_t padding,
                     float out[8]) {
    float pad = float(padding) + 0.5f;
    V2 off = add2(V2{float(tile_x + c->x), float(tile_y + c->y)}, V2{pad, pad});
    V3 ax = c->turned ? v3(c->v) : v3(c->u), ay = c->turned ? v3(c->u) : v3(c->v);
    float mx = c->turned ? c->min[1] : c->min[0], my = c->turned ? c->min[0] : c->min[1];
    V3 cx = mul(ax, density), cy = mul(ay, density);
    float row[8] = {cx.x, cx.y, cx.z, off.x - mx * density, cy.x, cy.y, cy.z, off.y - my * density};
    std::memcpy(out, row, sizeof row);
}

void or_raster_tile(int w, int h, const or_chart *charts, size_t n_charts, const uint32_t *tri_start,
                    const float *pos, float density, uint32_t padding, lb_texel *out) {
    std::memset(out, 0, sizeof(lb_texel) * size_t(w) * h);
    for (int conservative = 0; conservative < 2; conservative++)
        for (size_t ci = 0; ci < n_charts; ci++) {
            const or_chart *c = &charts[ci];
            for (uint32_t t = tri_start[ci]; t < tri_start[ci + 1]; t++) {
                V3 pa = v3(pos + size_t(t) * 9), pb = v3(pos + size_t(t) * 9 + 3), pc = v3(pos + size_t(t) * 9 + 6);
                V2 ua = chart_local(c, pa, density, padding), ub = chart_local(c, pb, density, padding),
                   uc = chart_local(c, pc, density, padding);
                float det = (ub.y - uc.y) * (ua.x - uc.x) + (uc.x - ub.x) * (ua.y - uc.y);
                if (std::fabs(det) < 1e-12f) continue;
                auto bary = [&](V2 q, float &l1, float &l2, float &l3) {
                    l1 = ((ub.y - uc.y) * (q.x - uc.x) + (uc.x - ub.x) * (q.y - uc.y)) / det;
                    l2 = ((uc.y - ua.y) * (q.x - uc.x) + (ua.x - uc.x) * (q.y - uc.y)) / det;
                    l3 = 1.0f - l1 - l2;
                };
                auto at = [&](V2 q) {
                    float l1, l2, l3;
                    bary(q, l1, l2, l3);
                    return add(add(mul(pa, l1), mul(pb, l2)), mul(pc, l3));
                };
                // face_normal (layout.rs:333-335): (c - b) x (a - b), try_normalize or +y
                V3 n = cross(sub(pc, pb), sub(pa, pb));
                float rcp = 1.0f / std::sqrt(dot(n, n));
                n = (std::isfinite(rcp) && rcp > 0.0f) ? mul(n, rcp) : V3{0.0f, 1.0f, 0.0f};
                V3 o = at(V2{0.0f, 0.0f});
                V3 dx = sub(at(V2{1.0f, 0.0f}), o), dy = sub(at(V2{0.0f, 1.0f}), o);
                float lox = std::fmax(std::floor(std::fmin(std::fmin(ua.x, ub.x), uc.x)), 0.0f);
                float loy = std::fmax(std::floor(std::fmin(std::fmin(ua.y, ub.y), uc.y)), 0.0f);
                float hix = std::fmin(std::ceil(std::fmax(std::fmax(ua.x, ub.x), uc.x)), float(w - 1));
                float hiy = std::fmin(std::ceil(std::fmax(std::fmax(ua.y, ub.y), uc.y)), float(h - 1));
                for (int y = int(loy); y <= int(hiy); y++)
                    for (int x = int(lox); x <= int(hix); x++) {
                        V2 centre{float(x) + 0.5f, float(y) + 0.5f};
                        lb_texel &T = out[size_t(y) * w + x];
                        if (T.pos[3] > 0.5f) continue;
                        V2 q = conservative ? nearest(centre, ua, ub, uc) : centre;
                        if (conservative && (std::fabs(q.x - centre.x) > 0.5f || std::fabs(q.y - centre.y) > 0.5f))
                            continue;
                        float l1, l2, l3;
                        bary(q, l1, l2, l3);
                        if (!conservative && (l1 < -1e-4f || l2 < -1e-4f || l3 < -1e-4f)) continue;
                        V3 p = at(q);
                        float rec[16] = {p.x, p.y, p.z, 1.0f, n.x, n.y, n.z, from_bits(c->id),
                                         dx.x, dx.y, dx.z, 0.0f, dy.x, dy.y, dy.z, 0.0f};
                        std::memcpy(&T, rec, sizeof rec);
                    }
            }
        }
}

size_t or_tile_post(int w, int h, lb_texel *texels, const float *records, const or_post_settings *s,
                    uint8_t *valid, uint8_t *known, uint8_t *state, float *field, float *ao, float *direct) {
    size_t size = size_t(w) * h;
    std::vector<uint32_t> chart(size), hard(size, 0);
    std::vector<float> normal(size * 3), soft(size, 0.0f), ao_raw(size, 1.0f);
    for (size_t i = 0; i < size; i++) {
        const lb_texel &T = texels[i];
        bool cov = T.pos[3] > 0.5f;
        valid[i] = cov ? 1 : 0;
        chart[i] = cov ? bits(T.normal[3]) : NONE;
        for (int c = 0; c < 3; c++) normal[i * 3 + c] = T.normal[c];
        state[i] = V_NONE;
    }
    size_t k = 0;
    for (size_t i = 0; i < size; i++) {
        if (!valid[i]) continue;
        const float *r = records + 4 * k++;
        if (r[3] > s->inside_share) {
            valid[i] = 0;
            continue;
        }
        soft[i] = r[0];
        uint32_t b = bits(r[1]);
        hard[i] = b & 0x00ffffffu;
        uint32_t pick = b >> 24;
        state[i] = pick == 0 ? V_CENTRE : (pick == 9 ? V_PUSHED : V_OFFSET);
        lb_texel &T = texels[i];
        if (pick == 9) {
            for (int c = 0; c < 3; c++) T.pos[c] += T.normal[c] * PUSH;
        } else if (pick > 0) {
            // bake.rs:494-503 (trace.wgsl's offset)
            float cx, cy;
            if (pick <= 4) {
                cx = (pick & 1) ? 0.3f : -0.3f;
                cy = pick > 2 ? 0.3f : -0.3f;
            } else if (pick == 5) {
                cx = -0.45f, cy = 0.0f;
            } else if (pick == 6) {
                cx = 0.45f, cy = 0.0f;
            } else if (pick == 7) {
                cx = 0.0f, cy = -0.45f;
            } else {
                cx = 0.0f, cy = 0.45f;
            }
            for (int c = 0; c < 3; c++) T.pos[c] += T.dx[c] * cx + T.dy[c] * cy;
        }
        float a = std::fmax(1.0f - s->ao_strength * r[2], 0.0f);
        ao_raw[i] = std::fmax(std::pow(a, s->ao_contrast), s->ao_floor);
    }
    int rings = int(s->padding) + 4;
    or_smooth(w, h, chart.data(), normal.data(), ao_raw.data(), 1, valid, 1, ao);
    std::vector<float> soft_s(size);
    or_smooth(w, h, chart.data(), normal.data(), soft.data(), 1, valid, 1, soft_s.data());
    or_sun_field(w, h, chart.data(), normal.data(), hard.data(), valid, s->grid, s->sdf_radius, field);
    V3 irr = v3(s->sun_irradiance), sun = v3(s->sun_dir);
    for (size_t i = 0; i < size; i++) {
        V3 d = mul(mul(irr, std::fmax(dot(v3(&normal[i * 3]), sun), 0.0f)), soft_s[i]);
        direct[i * 3] = d.x, direct[i * 3 + 1] = d.y, direct[i * 3 + 2] = d.z;
    }
    std::vector<uint8_t> kn(valid, valid + size), tmp(valid, valid + size);
    or_fill(w, h, chart.data(), ao, 1, tmp.data(), rings);
    std::memcpy(tmp.data(), valid, size);
    or_fill(w, h, chart.data(), field, 1, tmp.data(), rings);
    or_fill(w, h, chart.data(), direct, 3, kn.data(), rings);
    for (size_t i = 0; i < size; i++) {
        if (texels[i].pos[3] > 0.5f && state[i] == V_NONE && kn[i]) state[i] = V_FILLED;
        known[i] = valid[i] ? 2 : kn[i];
    }
    return k;
}

void or_gather_select(int w, int h, const uint8_t *valid, const uint32_t *chart, uint32_t ds, uint8_t *gathered) {
    size_t size = size_t(w) * h, tw = size_t(w), bw = (tw + ds - 1) / ds;
    auto block = [&](size_t i) { return ((i / tw) / ds) * bw + (i % tw) / ds; };
    std::set<std::pair<size_t, uint32_t>> seen;
    for (size_t i = 0; i < size; i++) {
        gathered[i] = valid[i] && (i % tw) % ds == 0 && (i / tw) % ds == 0;
        if (gathered[i]) seen.insert({block(i), chart[i]});
    }
    for (size_t i = 0; i < size; i++)
        if (valid[i] && seen.insert({block(i), chart[i]}).second) gathered[i] = 1;
}

size_t or_bounce_tile(int w, int h, const uint32_t *chart, const float *normal, const uint8_t *gathered,
                      const float *records, uint32_t radius, uint32_t rings, float *e) {
    size_t size = size_t(w) * h, k = 0;
    std::vector<float> raw(size * 3, 0.0f);
    for (size_t i = 0; i < size; i++)
        if (gathered[i]) {
            for (int c = 0; c < 3; c++) raw[i * 3 + c] = records[4 * k + c];
            k++;
        }
    or_smooth(w, h, chart, normal, raw.data(), 3, gathered, int(radius), e);
    std::vector<uint8_t> g(gathered, gathered + size);
    or_fill(w, h, chart, e, 3, g.data(), int(rings));
    return k;
}

void or_write_light(uint32_t tx, uint32_t ty, int w, int h, uint32_t atlas_width, const uint8_t *known,
                    const float *direct, const float *indirect, float *light) {
    for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++) {
            size_t i = size_t(y) * w + x, a = (size_t(ty) + y) * atlas_width + tx + x;
            float *L = light + a * 4;
            if (known[i] >= 1) {
                for (int c = 0; c < 3; c++) L[c] = direct[i * 3 + c] + indirect[i * 3 + c];
                L[3] = 1.0f;
            } else {
                L[0] = L[1] = L[2] = L[3] = 0.0f;
            }
        }
}

void or_volume_fill(uint32_t nx, uint32_t ny, uint32_t nz, float *probes) {
    size_t n = size_t(nx) * ny * nz;
    std::vector<uint8_t> known(n), was(n);
    std::vector<float> src(n * 16);
    for (size_t k = 0; k < n; k++) known[k] = probes[k * 16 + 4 + 3] <= 0.5f;  // p[1][3] <= INSIDE
    static const int D[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
    for (int ring = 0; ring < 8; ring++) {
        was = known;
        std::memcpy(src.data(), probes, n * 16 * sizeof(float));
        for (size_t k = 0; k < n; k++) {
            if (was[k]) continue;
            int64_t x = int64_t(k % nx), z = int64_t((k / nx) % nz), y = int64_t(k / (size_t(nx) * nz));
            float sum[16] = {0};
            int c = 0;
            for (auto &d : D) {
                int64_t xx = x + d[0], yy = y + d[1], zz = z + d[2];
                if (xx < 0 || yy < 0 || zz < 0 || xx >= nx || yy >= ny || zz >= nz) continue;
                size_t j = (size_t(yy) * nz + size_t(zz)) * nx + size_t(xx);
                if (!was[j]) continue;
                for (int q = 0; q < 16; q++) sum[q] += src[j * 16 + q];
                c++;
            }
            if (c > 0) {
                for (int q = 0; q < 16; q++) probes[k * 16 + q] = sum[q] / float(c);
                known[k] = 1;
            }
        }
    }
}

size_t or_volume_fallback(int w, int h, const lb_texel *texels, const float *probes, uint32_t nx, uint32_t ny,
                          uint32_t nz, const float origin[3], float step, const float sun_irradiance[3],
                          const float sun_dir[3], uint8_t *known, uint8_t *state, float *field, float *ao,
                          float *direct, float *indirect) {
    const float PI = 3.14159265358979323846f;
    const float a0 = PI * 0.282095f, a1 = 2.0f * PI / 3.0f * 0.488603f;
    size_t fixed = 0;
    for (size_t i = 0; i < size_t(w) * h; i++) {
        const lb_texel &T = texels[i];
        if (!(T.pos[3] > 0.5f) || known[i] != 0) continue;
        V3 n = v3(T.normal);
        V3 p = add(v3(T.pos), mul(n, 0.15f));
        // Volume::irradiance (volume.rs:125-147)
        V3 f = sub(p, v3(origin));
        f = V3{f.x / step, f.y / step, f.z / step};
        float fx = clampf(f.x, 0.0f, float(nx - 1)), fy = clampf(f.y, 0.0f, float(ny - 1)),
              fz = clampf(f.z, 0.0f, float(nz - 1));
        size_t x0 = std::min<size_t>(size_t(fx), nx - 2), y0 = std::min<size_t>(size_t(fy), ny - 2),
               z0 = std::min<size_t>(size_t(fz), nz - 2);
        float tx = fx - float(x0), ty = fy - float(y0), tz = fz - float(z0);
        float p4[16] = {0};
        for (int k = 0; k < 8; k++) {
            int dx = k & 1, dy = (k >> 1) & 1, dz = (k >> 2) & 1;
            float wgt = (dx ? tx : 1.0f - tx) * (dy ? ty : 1.0f - ty) * (dz ? tz : 1.0f - tz);
            const float *q = probes + (((y0 + dy) * nz + (z0 + dz)) * nx + (x0 + dx)) * 16;
            for (int a = 0; a < 16; a++) p4[a] += q[a] * wgt;
        }
        float e[3];
        for (int c = 0; c < 3; c++) {
            float lobe = a0 * p4[c] + a1 * (p4[4 + c] * n.x + p4[8 + c] * n.y + p4[12 + c] * n.z);
            e[c] = 0.5f * a0 * p4[c] + 0.5f * std::fmax(lobe, 0.0f);
        }
        float sun = p4[3];
        V3 d = mul(mul(v3(sun_irradiance), std::fmax(dot(n, v3(sun_dir)), 0.0f)), sun);
        for (int c = 0; c < 3; c++) indirect[i * 3 + c] = e[c];
        direct[i * 3] = d.x, direct[i * 3 + 1] = d.y, direct[i * 3 + 2] = d.z;
        field[i] = sun > 0.5f ? 1.0f : 0.0f;
        ao[i] = 1.0f;
        known[i] = 1;
        state[i] = V_VOLUME;
        fixed++;
    }
    return fixed;
}

void or_composite(uint32_t aw, uint32_t ah, uint32_t ds, size_t n_tiles, const uint32_t *rects,
                  const uint8_t *const *known, const uint8_t *const *state, const float *const *field,
                  const float *const *ao, const float *const *indirect, float *direct_out, uint8_t *validity,
                  float *indirect_out) {
    size_t iw = (aw + ds - 1) / ds, ih = (ah + ds - 1) / ds;
    for (size_t a = 0; a < size_t(aw) * ah; a++) {
        direct_out[a * 2] = direct_out[a * 2 + 1] = 1.0f;
        validity[a] = V_NONE;
    }
    std::vector<float> sum(iw * ih * 4, 0.0f);
    for (size_t t = 0; t < n_tiles; t++) {
        uint32_t tx = rects[t * 4], ty = rects[t * 4 + 1], tw = rects[t * 4 + 2], th = rects[t * 4 + 3];
        for (uint32_t y = 0; y < th; y++)
            for (uint32_t x = 0; x < tw; x++) {
                size_t i = size_t(y) * tw + x;
                if (known[t][i] == 0) continue;
                size_t ax = tx + x, ay = ty + y, a = ay * aw + ax;
                direct_out[a * 2] = field[t][i];
                direct_out[a * 2 + 1] = ao[t][i];
                validity[a] = state[t][i];
                float k = known[t][i] == 2 ? 1.0f : 1e-3f;
                float *s = &sum[((ay / ds) * iw + ax / ds) * 4];
                for (int c = 0; c < 3; c++) s[c] += indirect[t][i * 3 + c] * k;
                s[3] += k;
            }
    }
    std::vector<uint8_t> has(iw * ih);
    for (size_t i = 0; i < iw * ih; i++) {
        const float *s = &sum[i * 4];
        has[i] = s[3] > 0.0f;
        for (int c = 0; c < 3; c++) indirect_out[i * 3 + c] = has[i] ? s[c] / s[3] : 0.0f;
    }
    std::vector<uint8_t> was;
    std::vector<float> src;
    for (int pass = 0; pass < 2; pass++) {
        was = has;
        src.assign(indirect_out, indirect_out + iw * ih * 3);
        for (size_t y = 0; y < ih; y++)
            for (size_t x = 0; x < iw; x++) {
                size_t i = y * iw + x;
                if (was[i]) continue;
                float acc[3] = {0, 0, 0};
                int n = 0;
                for (size_t yy = y > 0 ? y - 1 : 0; yy < std::min(y + 2, ih); yy++)
                    for (size_t xx = x > 0 ? x - 1 : 0; xx < std::min(x + 2, iw); xx++) {
                        size_t j = yy * iw + xx;
                        if (!was[j]) continue;
                        for (int c = 0; c < 3; c++) acc[c] += src[j * 3 + c];
                        n++;
                    }
                if (n > 0) {
                    for (int c = 0; c < 3; c++) indirect_out[i * 3 + c] = acc[c] / float(n);
                    has[i] = 1;
                }
            }
    }
}

}  // extern "C"
