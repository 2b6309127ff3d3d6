#include "layout.h"

#include <algorithm>
#include <climits>
#include <cmath>
#include <map>
#include <stdexcept>
#include <string>
#include <unordered_map>

namespace lb {

namespace {

uint32_t round_up(uint32_t v, uint32_t a) { return (v + a - 1) / a * a; }

// Rust's `f as u32` / `f as i32`: truncation, saturating, NaN to 0
uint32_t as_u32(float f) {
    if (!(f > 0.0f)) return 0;
    if (f >= 4294967295.0f) return 0xffffffffu;
    return uint32_t(f);
}
int32_t as_i32(float f) {
    if (std::isnan(f)) return 0;
    if (f <= -2147483648.0f) return INT32_MIN;
    if (f >= 2147483647.0f) return INT32_MAX;
    return int32_t(f);
}
long long as_i64(float f) {
    if (std::isnan(f)) return 0;
    if (f <= -9.2233720368547758e18f) return LLONG_MIN;
    if (f >= 9.2233720368547758e18f) return LLONG_MAX;
    return (long long)f;
}

struct Key3 {
    long long v[3];
    bool operator==(const Key3 &o) const { return v[0] == o.v[0] && v[1] == o.v[1] && v[2] == o.v[2]; }
};
struct Key3Hash {
    size_t operator()(const Key3 &k) const {
        uint64_t h = 1469598103934665603ull;
        for (long long x : k.v) {
            h ^= uint64_t(x);
            h *= 1099511628211ull;
        }
        return size_t(h);
    }
};

// layout.rs:129-171: charts by region growing across shared vertices, neighbours facing within `cos` of
// the seed and in its tile (by the centre of the triangle's box); each group in triangle order, the groups
// in the order of their seeds (each the lowest triangle not yet taken).
//
// A group never leaves its seed's tile, so the tiles are grown apart, in parallel: a tile's groups depend
// only on its own triangles (their seeds, in index order, are the ones the whole-mesh walk meets there),
// and each group's first triangle is its seed, so sorting all groups by their first triangle gives the
// whole-mesh walk's order.
std::vector<std::vector<uint32_t>> grow(const std::vector<Vec3> &pos, float cosv, float tile) {
    const size_t n = pos.size() / 3;
    std::vector<Vec3> normals(n);
    std::vector<TileKey> keys(n);
#pragma omp parallel for schedule(static)
    for (long long ti = 0; ti < (long long)n; ti++) {
        normals[ti] = face_normal(pos, size_t(ti));
        keys[ti] = tile_of(box_centre(pos, size_t(ti)), tile);
    }
    // the triangles of each tile, in index order
    std::map<TileKey, uint32_t> tile_id;
    std::vector<uint32_t> id_of(n), count;
    {
        TileKey last{INT32_MIN, INT32_MIN};
        uint32_t last_id = 0;
        for (size_t t = 0; t < n; t++) {
            if (t == 0 || keys[t] != last) {
                auto it = tile_id.emplace(keys[t], uint32_t(tile_id.size())).first;
                last = keys[t];
                last_id = it->second;
                if (last_id == count.size()) count.push_back(0);
            }
            id_of[t] = last_id;
            count[last_id]++;
        }
    }
    const size_t nt = count.size();
    std::vector<size_t> first(nt + 1, 0);
    for (size_t k = 0; k < nt; k++) first[k + 1] = first[k] + count[k];
    std::vector<uint32_t> members(n);
    {
        std::vector<size_t> at = first;
        for (size_t t = 0; t < n; t++) members[at[id_of[t]]++] = uint32_t(t);
    }
    auto key = [](Vec3 v) {
        return Key3{{as_i64(std::round(v.x * 1e4f)), as_i64(std::round(v.y * 1e4f)), as_i64(std::round(v.z * 1e4f))}};
    };
    // (a triangle is in one tile, so the tiles' threads write disjoint flags)
    std::vector<char> taken(n, 0);
    std::vector<std::vector<std::vector<uint32_t>>> per_tile(nt);
#pragma omp parallel for schedule(dynamic, 1)
    for (long long k = 0; k < (long long)nt; k++) {
        const uint32_t *tris = members.data() + first[k];
        const size_t m = first[k + 1] - first[k];
        std::unordered_map<Key3, std::vector<uint32_t>, Key3Hash> at;
        at.reserve(m * 2);
        for (size_t i = 0; i < m; i++)
            for (int c = 0; c < 3; c++) at[key(pos[size_t(tris[i]) * 3 + c])].push_back(tris[i]);
        auto &out = per_tile[k];
        for (size_t i = 0; i < m; i++) {
            const uint32_t seed = tris[i];
            if (taken[seed]) continue;
            taken[seed] = 1;
            std::vector<uint32_t> group{seed};
            Vec3 sn = normals[seed];
            TileKey sk = keys[seed];
            for (size_t j = 0; j < group.size(); j++) {
                size_t t = group[j];
                for (int c = 0; c < 3; c++) {
                    for (uint32_t o : at[key(pos[t * 3 + c])]) {
                        if (taken[o] || keys[o] != sk || normals[o].dot(sn) < cosv) continue;
                        taken[o] = 1;
                        group.push_back(o);
                    }
                }
            }
            std::sort(group.begin(), group.end());
            out.push_back(std::move(group));
        }
    }
    std::vector<std::vector<uint32_t>> out;
    for (auto &v : per_tile)
        for (auto &g : v) out.push_back(std::move(g));
    std::sort(out.begin(), out.end(), [](const std::vector<uint32_t> &a, const std::vector<uint32_t> &b) {
        return a[0] < b[0];
    });
    return out;
}

// layout.rs:173-196
Chart make_chart(const std::vector<Vec3> &pos, uint32_t mesh, std::vector<uint32_t> tris, float tile, float density,
                 uint32_t padding) {
    Vec3 sum(0, 0, 0);
    for (uint32_t t : tris) sum += (pos[t * 3 + 2] - pos[t * 3 + 1]).cross(pos[t * 3] - pos[t * 3 + 1]);
    Vec3 n;
    if (!sum.try_normalize(n)) n = face_normal(pos, tris[0]);
    Vec3 u = std::fabs(n.y) > 0.9f ? Vec3(1, 0, 0) : Vec3(0, 1, 0).cross(n);
    u = (u - n * u.dot(n)).normalize();
    Vec3 v = n.cross(u);
    Vec2 mn(INFINITY, INFINITY), mx(-INFINITY, -INFINITY);
    for (uint32_t t : tris)
        for (int k = 0; k < 3; k++) {
            Vec3 p = pos[t * 3 + k];
            Vec2 q(p.dot(u), p.dot(v));
            mn = mn.min(q);
            mx = mx.max(q);
        }
    auto size = [&](float e) { return as_u32(std::ceil(e * density)) + 1 + 2 * padding; };
    Chart c;
    c.mesh = mesh;
    c.normal = n;
    c.u = u;
    c.v = v;
    c.min = mn;
    c.max = mx;
    c.tile = tile_of(box_centre(pos, tris[0]), tile);
    c.turned = false;
    c.w = size(mx.x - mn.x);
    c.h = size(mx.y - mn.y);
    c.tris = std::move(tris);
    return c;
}

// layout.rs:263-331: the heights reached along a rectangle's width, as (x, width, top) segments
struct Skyline {
    std::vector<std::array<uint32_t, 3>> segs;
    uint32_t width;
    explicit Skyline(uint32_t w) : segs{{0, w, 0}}, width(w) {}
    bool find(uint32_t w, std::pair<uint32_t, uint32_t> &best) const {
        if (w > width) return false;
        bool have = false;
        for (size_t i = 0; i < segs.size(); i++) {
            uint32_t x = segs[i][0];
            if (x + w > width) break;
            uint32_t top = 0, reach = 0;
            for (size_t j = i; j < segs.size(); j++) {
                top = std::max(top, segs[j][2]);
                reach += segs[j][1];
                if (reach >= w) break;
            }
            if (!have || top < best.second) {
                best = {x, top};
                have = true;
            }
        }
        return have;
    }
    void place(uint32_t x, uint32_t y, uint32_t w, uint32_t h) {
        std::vector<std::array<uint32_t, 3>> next;
        next.reserve(segs.size() + 2);
        for (auto &s : segs) {
            uint32_t sx = s[0], sw = s[1], st = s[2], end = sx + sw;
            if (end <= x || sx >= x + w) {
                next.push_back(s);
                continue;
            }
            if (sx < x) next.push_back({sx, x - sx, st});
            if (end > x + w) next.push_back({x + w, end - x - w, st});
        }
        next.push_back({x, w, y + h});
        std::stable_sort(next.begin(), next.end(), [](auto &a, auto &b) { return a[0] < b[0]; });
        std::vector<std::array<uint32_t, 3>> merged;
        for (auto &s : next) {
            if (!merged.empty() && merged.back()[2] == s[2] && merged.back()[0] + merged.back()[1] == s[0])
                merged.back()[1] += s[1];
            else
                merged.push_back(s);
        }
        segs = std::move(merged);
    }
    uint32_t top() const {
        uint32_t t = 0;
        for (auto &s : segs) t = std::max(t, s[2]);
        return t;
    }
};

// layout.rs:198-238
Tile pack_tile(TileKey key, std::vector<uint32_t> ids, std::vector<Chart> &charts) {
    for (uint32_t i : ids) {
        Chart &c = charts[i];
        if (c.h > c.w) {
            c.turned = true;
            std::swap(c.w, c.h);
        }
    }
    std::vector<uint32_t> order = ids;
    std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) {
        const Chart &ca = charts[a], &cb = charts[b];
        if (cb.h != ca.h) return cb.h < ca.h;
        if (cb.w != ca.w) return cb.w < ca.w;
        return a < b;
    });
    uint64_t area = 0;
    uint32_t widest = 0;
    for (uint32_t i : ids) {
        area += uint64_t(charts[i].w) * charts[i].h;
        widest = std::max(widest, charts[i].w);
    }
    if (ids.empty()) widest = 1;
    uint32_t width = round_up(std::max(widest, uint32_t(std::ceil(std::sqrt(double(area) * 1.1)))), ALIGN);
    Skyline sky(width);
    for (uint32_t i : order) {
        Chart &c = charts[i];
        std::pair<uint32_t, uint32_t> a, b;
        bool flat = sky.find(c.w, a);
        bool up = (c.h <= width && c.w != c.h) ? sky.find(c.h, b) : false;
        uint32_t x, y;
        bool turn;
        if (flat && up && b.second + c.w < a.second + c.h) {
            x = b.first, y = b.second, turn = true;
        } else if (flat) {
            x = a.first, y = a.second, turn = false;
        } else if (up) {
            x = b.first, y = b.second, turn = true;
        } else {
            throw std::runtime_error("a chart no wider than its tile always fits");
        }
        if (turn) {
            c.turned = !c.turned;
            std::swap(c.w, c.h);
        }
        c.x = x;
        c.y = y;
        sky.place(x, y, c.w, c.h);
    }
    Tile t;
    t.key = key;
    t.charts = std::move(ids);
    t.w = width;
    t.h = round_up(std::max(sky.top(), 1u), ALIGN);
    return t;
}

// layout.rs:240-261
uint32_t shelve(std::vector<Tile> &tiles, uint32_t width) {
    std::vector<size_t> order(tiles.size());
    for (size_t i = 0; i < order.size(); i++) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) {
        if (tiles[b].h != tiles[a].h) return tiles[b].h < tiles[a].h;
        return tiles[a].key < tiles[b].key;
    });
    uint32_t x = 0, y = 0, row = 0;
    for (size_t i : order) {
        Tile &t = tiles[i];
        if (t.w > width)
            throw std::runtime_error("tile (" + std::to_string(t.key.first) + ", " + std::to_string(t.key.second) +
                                     ") is " + std::to_string(t.w) + " texels wide, the atlas " + std::to_string(width) +
                                     ": lower texelsPerMeter or tileSize, or widen the atlas");
        if (x + t.w > width) {
            x = 0;
            y += row;
            row = 0;
        }
        t.x = x;
        t.y = y;
        x += t.w;
        row = std::max(row, t.h);
    }
    return round_up(std::max(y + row, ALIGN), ALIGN);
}

}  // namespace

Vec2 Chart::local(Vec3 p, float density, uint32_t padding) const {
    Vec2 a = (Vec2(p.dot(u), p.dot(v)) - min) * density;
    if (turned) a = Vec2(a.y, a.x);
    return (Vec2(float(x), float(y)) + Vec2(float(padding) + 0.5f, float(padding) + 0.5f)) + a;
}

std::array<std::array<float, 4>, 2> Chart::affine(const Tile &tile, float density, uint32_t padding) const {
    float pad = float(padding) + 0.5f;
    Vec2 off = Vec2(float(tile.x + x), float(tile.y + y)) + Vec2(pad, pad);
    Vec3 ax = turned ? v : u, ay = turned ? u : v;
    float mx = turned ? min.y : min.x, my = turned ? min.x : min.y;
    auto row = [&](Vec3 axis, float mn, float o) {
        Vec3 c = axis * density;
        return std::array<float, 4>{c.x, c.y, c.z, o - mn * density};
    };
    return {row(ax, mx, off.x), row(ay, my, off.y)};
}

// layout.rs:89-115
Layout Layout::build(const Scene &scene) {
    const LightmapSettings &s = scene.header.lightmap;
    Layout L;
    L.density = s.texels_per_meter;
    L.padding = s.padding;
    float to_rad = s.chart_angle_deg * (3.14159265358979323846f / 180.0f);
    float cosv = std::cos(to_rad);
    L.tri_chart.resize(scene.positions.size());
    for (size_t m = 0; m < scene.positions.size(); m++) L.tri_chart[m].assign(scene.positions[m].size() / 3, 0xffffffffu);
    for (size_t mi = 0; mi < scene.header.meshes.size(); mi++) {
        const MeshInfo &m = scene.header.meshes[mi];
        if (!scene.header.materials[m.material].receives) continue;
        std::vector<std::vector<uint32_t>> groups = grow(scene.positions[mi], cosv, s.tile_size);
        // each group's chart on its own (in parallel), numbered in group order
        std::vector<Chart> made(groups.size());
#pragma omp parallel for schedule(dynamic, 64)
        for (long long g = 0; g < (long long)groups.size(); g++)
            made[g] = make_chart(scene.positions[mi], uint32_t(mi), std::move(groups[g]), s.tile_size, L.density,
                                 L.padding);
        for (Chart &c : made) {
            for (uint32_t t : c.tris) L.tri_chart[mi][t] = uint32_t(L.charts.size());
            L.charts.push_back(std::move(c));
        }
    }
    std::map<TileKey, std::vector<uint32_t>> by_tile;
    for (size_t i = 0; i < L.charts.size(); i++) by_tile[L.charts[i].tile].push_back(uint32_t(i));
    // the tiles packed apart (in parallel: a tile's packing reads and moves only its own charts), kept in
    // tile order
    std::vector<std::pair<TileKey, std::vector<uint32_t>>> todo(by_tile.begin(), by_tile.end());
    L.tiles.resize(todo.size());
    std::vector<std::string> failed(todo.size());
#pragma omp parallel for schedule(dynamic, 1)
    for (long long k = 0; k < (long long)todo.size(); k++) {
        try {
            L.tiles[k] = pack_tile(todo[k].first, todo[k].second, L.charts);
        } catch (const std::exception &e) {
            failed[k] = e.what();
        }
    }
    for (const std::string &f : failed)
        if (!f.empty()) throw std::runtime_error(f);
    L.height = shelve(L.tiles, s.atlas_width);
    L.width = s.atlas_width;
    return L;
}

std::vector<uint32_t> Layout::chart_tile() const {
    std::vector<uint32_t> out(charts.size(), 0);
    for (size_t ti = 0; ti < tiles.size(); ti++)
        for (uint32_t c : tiles[ti].charts) out[c] = uint32_t(ti);
    return out;
}

Vec3 face_normal(const std::vector<Vec3> &pos, size_t t) {
    Vec3 n;
    if ((pos[t * 3 + 2] - pos[t * 3 + 1]).cross(pos[t * 3] - pos[t * 3 + 1]).try_normalize(n)) return n;
    return Vec3(0, 1, 0);
}

Vec3 box_centre(const std::vector<Vec3> &pos, size_t t) {
    Vec3 a = pos[t * 3], b = pos[t * 3 + 1], c = pos[t * 3 + 2];
    return (a.min(b).min(c) + a.max(b).max(c)) * 0.5f;
}

TileKey tile_of(Vec3 p, float size) {
    return {as_i32(std::floor(p.x / size)), as_i32(std::floor(p.z / size))};
}

}  // namespace lb
