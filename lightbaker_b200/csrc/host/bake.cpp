#include "bake.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <exception>
#include <map>
#include <set>
#include <stdexcept>
#include <thread>

#include "cache.h"
#include "deps.h"
#include "filter.h"
#include "raster.h"

namespace lb {

namespace {
constexpr float F32_PI = 3.14159274101257324f;  // std::f32::consts::PI

double since(std::chrono::steady_clock::time_point t) {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t).count();
}
std::string fmt(const char *f, double a) {
    char b[128];
    snprintf(b, sizeof b, f, a);
    return b;
}
Vec3 v3(const std::array<float, 3> &a) { return Vec3(a[0], a[1], a[2]); }

// A tile being baked: its texels and the per-texel state the passes build up (bake.rs:82-92).
struct Work {
    size_t tile;
    std::vector<lb_texel> texels;
    std::vector<uint32_t> chart;
    std::vector<std::array<float, 3>> normal;
    std::vector<uint8_t> valid, gathered;
};

std::vector<size_t> offsets(const std::vector<size_t> &counts) {
    std::vector<size_t> out;
    size_t at = 0;
    for (size_t n : counts) {
        out.push_back(at);
        at += n;
    }
    return out;
}
}  // namespace

void texel_offset(uint32_t q, float &x, float &y) {
    switch (q) {
    case 1: case 2: case 3: case 4:
        x = (q & 1) == 1 ? 0.3f : -0.3f;
        y = q > 2 ? 0.3f : -0.3f;
        return;
    case 5: x = -0.45f, y = 0.0f; return;
    case 6: x = 0.45f, y = 0.0f; return;
    case 7: x = 0.0f, y = -0.45f; return;
    default: x = 0.0f, y = 0.45f; return;
    }
}

std::vector<uint8_t> TileLight::pack() const {
    Pack p;
    p.put(known).put(state).put(field).put(ao).put(direct).put(indirect);
    return p.bytes;
}

std::optional<TileLight> TileLight::unpack(const std::vector<uint8_t> &b, size_t size) {
    Unpack u{b.data(), b.size()};
    TileLight t;
    if (!u.take(t.known) || !u.take(t.state) || !u.take(t.field) || !u.take(t.ao) || !u.take(t.direct) ||
        !u.take(t.indirect))
        return std::nullopt;
    if (t.known.size() != size || t.state.size() != size || t.field.size() != size || t.ao.size() != size ||
        t.direct.size() != size || t.indirect.size() != size)
        return std::nullopt;
    return t;
}

Aabb tile_box(const Scene &scene, const Layout &layout, const std::vector<uint32_t> &charts) {
    Aabb b;
    for (uint32_t ci : charts) {
        const Chart &c = layout.charts[ci];
        for (uint32_t t : c.tris)
            for (int k = 0; k < 3; k++) b.add(scene.positions[c.mesh][size_t(t) * 3 + k]);
    }
    return b;
}

std::vector<uint8_t> tile_seed(const Scene &scene, const Layout &layout, TileKey key, const std::vector<uint32_t> &charts) {
    Blake3 k;
    int32_t a = key.first, b = key.second;
    k.update(&a, 4);
    k.update(&b, 4);
    for (uint32_t ci : charts) {
        const Chart &c = layout.charts[ci];
        k.update(&c.mesh, 4);
        k.update(&scene.header.meshes[c.mesh].material, 4);
        for (uint32_t t : c.tris) {
            k.update(&t, 4);
            k.update(&scene.positions[c.mesh][size_t(t) * 3], 36);
        }
    }
    std::vector<uint8_t> out(32);
    k.finalize(out.data());
    return out;
}

void write_light(const Layout &layout, size_t ti, const TileLight &l, std::vector<float> &light) {
    const Tile &t = layout.tiles[ti];
    for (size_t y = 0; y < t.h; y++)
        for (size_t x = 0; x < t.w; x++) {
            size_t i = y * t.w + x;
            size_t a = (t.y + y) * size_t(layout.width) + t.x + x;
            float *o = &light[a * 4];
            if (l.known[i] >= 1) {
                o[0] = l.direct[i][0] + l.indirect[i][0];
                o[1] = l.direct[i][1] + l.indirect[i][1];
                o[2] = l.direct[i][2] + l.indirect[i][2];
                o[3] = 1.0f;
            } else {
                o[0] = o[1] = o[2] = o[3] = 0.0f;
            }
        }
}

void Volume::irradiance(Vec3 p, Vec3 n, float e[3], float &sun) const {
    size_t nx = size[0], ny = size[1], nz = size[2];
    Vec3 f = (p - Vec3(origin[0], origin[1], origin[2])) / step;
    auto cl = [](float v, size_t n) { return std::min(std::max(v, 0.0f), float(n - 1)); };
    float fx = cl(f.x, nx), fy = cl(f.y, ny), fz = cl(f.z, nz);
    size_t x0 = std::min(size_t(fx), nx - 2), y0 = std::min(size_t(fy), ny - 2), z0 = std::min(size_t(fz), nz - 2);
    float tx = fx - float(x0), ty = fy - float(y0), tz = fz - float(z0);
    float p4[16] = {0};
    for (int k = 0; k < 8; k++) {
        int dx = k & 1, dy = (k >> 1) & 1, dz = (k >> 2) & 1;
        float w = ((dx ? tx : 1.0f - tx) * (dy ? ty : 1.0f - ty)) * (dz ? tz : 1.0f - tz);
        const auto &q = probes[((y0 + dy) * nz + (z0 + dz)) * nx + (x0 + dx)];
        for (int a = 0; a < 16; a++) p4[a] += q[a] * w;
    }
    float a0 = F32_PI * 0.282095f, a1 = 2.0f * F32_PI / 3.0f * 0.488603f;
    for (int c = 0; c < 3; c++)
        e[c] = 0.5f * a0 * p4[c] +
               0.5f * std::fmax(a0 * p4[c] + a1 * ((p4[4 + c] * n.x + p4[8 + c] * n.y) + p4[12 + c] * n.z), 0.0f);
    sun = p4[3];
}

Prepared prepare(const Scene &scene) {
    const SceneHeader &h = scene.header;
    const BakeSettings &b = h.bake;
    // The layout and the BVH at once: the tree's splits do not depend on the charts, so the BVH is built
    // beside the layout and the triangles' chart bits written in afterwards (the same bytes).
    Prepared P{Layout(), {}, {}, {}, {}, {}, {}, 0};
    std::exception_ptr layout_error;
    std::thread layout_thread([&]() {
        try {
            P.layout = Layout::build(scene);
        } catch (...) {
            layout_error = std::current_exception();
        }
    });
    try {
        P.bvh = Bvh::build(scene, [](size_t, size_t) { return 0xffffffffu; });
    } catch (...) {
        layout_thread.join();
        throw;
    }
    layout_thread.join();
    if (layout_error) std::rethrow_exception(layout_error);
    P.bvh.set_charts([&](size_t m, size_t t) { return P.layout.tri_chart[m][t]; });
    P.chart_tile = P.layout.chart_tile();
    for (size_t i = 0; i < P.layout.charts.size(); i++) {
        auto a = P.layout.charts[i].affine(P.layout.tiles[P.chart_tile[i]], P.layout.density, P.layout.padding);
        for (auto &r : a) P.affines.insert(P.affines.end(), r.begin(), r.end());
    }
    for (auto &m : h.materials) P.materials.insert(P.materials.end(), {m.albedo[0], m.albedo[1], m.albedo[2], m.opacity});
    P.sun = v3(h.sun.direction).normalize();
    P.g = uint32_t(std::sqrt(float(b.sun_samples)));
    Vec3 sky_avg = ((v3(h.sky.zenith) + v3(h.sky.horizon)) * 0.5f) * F32_PI;
    lb_params &p = P.params;
    std::memset(&p, 0, sizeof p);
    float rad = h.sun.radius_deg * (F32_PI / 180.0f);
    float sd[4] = {P.sun.x, P.sun.y, P.sun.z, std::tan(rad)};
    std::memcpy(p.sun_dir, sd, 16);
    for (int c = 0; c < 3; c++) {
        p.sun_irr[c] = h.sun.irradiance[c];
        p.zenith[c] = h.sky.zenith[c];
        p.horizon[c] = h.sky.horizon[c];
        p.ground[c] = h.sky.ground[c];
    }
    p.fallback[0] = sky_avg.x;
    p.fallback[1] = sky_avg.y;
    p.fallback[2] = sky_avg.z;
    p.ground[3] = std::fmin(INSIDE_REACH, b.ao_reach);
    p.counts[0] = P.g;
    p.counts[1] = b.ao_rays;
    p.counts[2] = b.gi_rays;
    p.counts[3] = 0;
    p.reach[0] = b.ao_reach;
    p.reach[1] = b.gi_reach;
    p.reach[2] = LIFT;
    p.reach[3] = 0.0f;
    p.atlas[0] = P.layout.width;
    p.atlas[1] = P.layout.height;
    p.atlas[2] = 0;
    p.atlas[3] = f2u(b.inside_share);
    return P;
}

namespace {

// volume.rs:34-120
Volume bake_volume(const Scene &scene, Tracer &gpu, lb_params params, const std::vector<float> &light,
                   const VolumeSettings &v, const Boxes &boxes, const Hash &global, const Cache &cache, Stats &stats,
                   const std::function<void(const std::string &)> &log, int rank, int world,
                   const std::function<void(void *, size_t)> &sum_words) {
    auto started = std::chrono::steady_clock::now();
    auto n = [&](int a) { return uint32_t(std::round((v.max[a] - v.min[a]) / v.step)) + 1; };
    std::array<uint32_t, 3> size = {std::max(n(0), 2u), std::max(n(1), 2u), std::max(n(2), 2u)};
    size_t nx = size[0], ny = size[1], nz = size[2], total = nx * ny * nz;
    auto at = [&](size_t k) {
        return Vec3(v.min[0] + float(k % nx) * v.step, v.min[1] + float(k / (nx * nz)) * v.step,
                    v.min[2] + float((k / nx) % nz) * v.step);
    };
    std::map<TileKey, std::vector<uint32_t>> chunks;
    for (size_t k = 0; k < total; k++) chunks[tile_of(at(k), scene.header.lightmap.tile_size)].push_back(uint32_t(k));
    Volume vol;
    vol.origin = v.min;
    vol.step = v.step;
    vol.size = size;
    vol.probes.assign(total, std::array<float, 16>{});
    std::vector<uint8_t> known(total, 0);
    std::vector<uint32_t> todo;
    std::vector<std::pair<Hash, std::vector<uint32_t>>> keys;
    std::string vjson = to_json(v).dump();
    for (auto &kv : chunks) {
        Aabb b;
        for (uint32_t k : kv.second) b.add(at(k));
        std::vector<uint8_t> seed(8);
        std::memcpy(seed.data(), &kv.first.first, 4);
        std::memcpy(seed.data() + 4, &kv.first.second, 4);
        seed.insert(seed.end(), vjson.begin(), vjson.end());
        Hash hash = hash_reach(scene, boxes, global, b, scene.header.bake.gi_reach, seed);
        auto got = cache.get("probes", hash);
        if (got && got->size() == kv.second.size() * 64) {
            for (size_t i = 0; i < kv.second.size(); i++) std::memcpy(vol.probes[kv.second[i]].data(), got->data() + i * 64, 64);
        } else {
            todo.insert(todo.end(), kv.second.begin(), kv.second.end());
            keys.emplace_back(hash, kv.second);
        }
    }
    // a bake split over ranks: this rank's contiguous run of the chunks to bake, balanced by probes (a probe's
    // keys are its own index, so any split keeps them); the others' probes arrive through the sum
    std::vector<uint64_t> chunk_cost;
    for (auto &kv : keys) chunk_cost.push_back(kv.second.size());
    const auto share = shard_range(chunk_cost, rank, world);
    size_t p0 = 0, p1 = 0;
    for (size_t c = 0; c < keys.size(); c++) {
        if (c < share.first) p0 += keys[c].second.size();
        if (c < share.second) p1 += keys[c].second.size();
    }
    std::vector<lb_texel> items(p1 - p0);
    for (size_t i = p0; i < p1; i++) {
        Vec3 p = at(todo[i]);
        items[i - p0] = lb_texel{{p.x, p.y, p.z, 1.0f}, {0.0f, 1.0f, 0.0f, u2f(todo[i])}, {0, 0, 0, 0}, {0, 0, 0, 0}};
    }
    params.counts[2] = v.rays;
    std::vector<float> res;
    stats.rays_volume += gpu.run(LB_PASS_VOLUME, params, items, light, res);
    if (world > 1) {
        std::vector<float> all(todo.size() * 16, 0.0f);
        std::memcpy(all.data() + p0 * 16, res.data(), (p1 - p0) * 64);
        sum_words(all.data(), all.size());
        res = std::move(all);
    }
    for (size_t i = 0; i < todo.size(); i++) std::memcpy(vol.probes[todo[i]].data(), &res[i * 16], 64);
    for (size_t c = share.first; c < share.second; c++) {
        auto &kv = keys[c];
        std::vector<uint8_t> bytes(kv.second.size() * 64);
        for (size_t i = 0; i < kv.second.size(); i++) std::memcpy(bytes.data() + i * 64, vol.probes[kv.second[i]].data(), 64);
        cache.put("probes", kv.first, bytes);
    }
    // inside solids: from the neighbours, a ring at a time
    for (size_t k = 0; k < total; k++) known[k] = vol.probes[k][7] <= VOLUME_INSIDE;
    for (int ring = 0; ring < 8; ring++) {
        std::vector<uint8_t> was = known;
        std::vector<std::array<float, 16>> src = vol.probes;
        for (size_t k = 0; k < total; k++) {
            if (was[k]) continue;
            long long x = k % nx, z = (k / nx) % nz, y = k / (nx * nz);
            float sum[16] = {0};
            int c = 0;
            static const int D[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
            for (auto &d : D) {
                long long xx = x + d[0], yy = y + d[1], zz = z + d[2];
                if (xx < 0 || yy < 0 || zz < 0 || xx >= (long long)nx || yy >= (long long)ny || zz >= (long long)nz) continue;
                size_t j = (size_t(yy) * nz + size_t(zz)) * nx + size_t(xx);
                if (was[j]) {
                    for (int q = 0; q < 16; q++) sum[q] += src[j][q];
                    c++;
                }
            }
            if (c > 0) {
                for (int q = 0; q < 16; q++) vol.probes[k][q] = sum[q] / float(c);
                known[k] = 1;
            }
        }
    }
    vol.chunks = chunks.size();
    vol.chunks_baked = keys.size();
    if (log)
        log("volume " + std::to_string(nx) + "x" + std::to_string(ny) + "x" + std::to_string(nz) + ": " +
            std::to_string(todo.size()) + " probes baked, " + fmt("%.1f s", since(started)));
    return vol;
}

}  // namespace

std::pair<size_t, size_t> shard_range(const std::vector<uint64_t> &cost, int rank, int world) {
    if (world <= 1) return {0, cost.size()};
    std::vector<uint64_t> prefix(cost.size() + 1, 0);
    for (size_t i = 0; i < cost.size(); i++) prefix[i + 1] = prefix[i] + cost[i];
    const uint64_t total = prefix.back();
    // boundary r: the item index whose prefix cost is nearest total * r / world (ties to the lower), never
    // before boundary r - 1
    auto boundary = [&](int r) {
        if (r <= 0) return size_t(0);
        if (r >= world) return cost.size();
        size_t k = 0;
        while (k < cost.size() && prefix[k] * uint64_t(world) < total * uint64_t(r)) k++;
        if (k > 0 && (prefix[k] * uint64_t(world) - total * uint64_t(r)) >
                         (total * uint64_t(r) - prefix[k - 1] * uint64_t(world)))
            k--;
        return k;
    };
    size_t a = 0;
    for (int r = 1; r <= rank; r++) a = std::max(a, boundary(r));
    size_t b = std::max(a, boundary(rank + 1));
    return {a, b};
}

Bake bake(const Scene &scene, Tracer &gpu, const Options &o) {
    auto started = std::chrono::steady_clock::now();
    auto log = [&](const std::string &s) {
        if (o.log) o.log(s);
    };
    const SceneHeader &h = scene.header;
    const BakeSettings &b = h.bake;
    const LightmapSettings &lm = h.lightmap;
    Prepared P = prepare(scene);
    Layout &layout = P.layout;
    size_t aw = layout.width, ah = layout.height;
    gpu.scene(P.bvh, P.materials, P.affines);
    if (o.watertight) gpu.watertight(P.bvh);
    const lb_params &params = P.params;
    Vec3 sun = P.sun;
    uint32_t g = P.g;
    Stats stats;
    stats.t_layout = since(started);
    log(std::to_string(scene.triangle_count()) + " triangles, " + std::to_string(layout.charts.size()) + " charts in " +
        std::to_string(layout.tiles.size()) + " tiles, atlas " + std::to_string(aw) + "x" + std::to_string(ah) +
        ", BVH " + std::to_string(P.bvh.nodes.size()) + " nodes (" + fmt("%.1f s)", since(started)));

    // which tiles the cache has (bake.rs:123-136)
    Cache cache(o.cache);
    Boxes boxes(scene);
    Hash global = global_hash(scene);
    if (o.watertight) global = watertight_hash(global);
    float reach = b.gi_bounces > 0 ? std::fmax(b.gi_reach, b.ao_reach) : b.ao_reach;
    size_t nt = layout.tiles.size();
    std::vector<Hash> hashes(nt);
    std::vector<std::optional<TileLight>> lights(nt);
#pragma omp parallel for schedule(dynamic, 1)
    for (long long ti = 0; ti < (long long)nt; ti++) {
        const Tile &t = layout.tiles[ti];
        hashes[ti] = hash_reach(scene, boxes, global, tile_box(scene, layout, t.charts), reach,
                                tile_seed(scene, layout, t.key, t.charts));
        if (auto bytes = cache.get("tile", hashes[ti])) lights[ti] = TileLight::unpack(*bytes, size_t(t.w) * t.h);
    }
    std::vector<size_t> dirty, cached;
    for (size_t i = 0; i < nt; i++) (lights[i] ? cached : dirty).push_back(i);
    log(std::to_string(dirty.size()) + " of " + std::to_string(nt) + " tiles to bake");

    // A bake split over ranks (beyond the reference): this rank bakes a contiguous run of the dirty tiles,
    // balanced by their texels, so its items are a contiguous run of each pass's whole list and keep their
    // keys (the index in that list) from one base; what the others bake arrives through sums of 32-bit words
    // in which every word has one writer. One rank: everything, and the sums are no-ops.
    const int world = (o.world > 1 && o.sum) ? o.world : 1, rank = world > 1 ? o.rank : 0;
    auto sum_words = [&](void *data, size_t words) {
        if (world > 1 && words) o.sum(data, words, false);
    };
    std::vector<uint64_t> tile_cost;
    for (size_t ti : dirty) tile_cost.push_back(uint64_t(layout.tiles[ti].w) * layout.tiles[ti].h);
    const auto shard = shard_range(tile_cost, rank, world);
    std::vector<size_t> mine(dirty.begin() + shard.first, dirty.begin() + shard.second);
    if (world > 1)
        log("rank " + std::to_string(rank) + " of " + std::to_string(world) + ": dirty tiles " +
            std::to_string(shard.first) + " to " + std::to_string(shard.second));
    // counts of every dirty tile from every rank: the bases of this rank's keys
    auto shared_counts = [&](const std::vector<size_t> &own, uint64_t &before, uint64_t &all) {
        std::vector<uint32_t> c(dirty.size(), 0);
        for (size_t k = 0; k < own.size(); k++) c[shard.first + k] = uint32_t(own[k]);
        sum_words(c.data(), c.size());
        before = all = 0;
        for (size_t k = 0; k < c.size(); k++) {
            if (k < shard.first) before += c[k];
            all += c[k];
        }
    };

    // the dirty tiles' texels (bake.rs:138-149)
    std::vector<Work> work(mine.size());
#pragma omp parallel for schedule(dynamic, 1)
    for (long long wi = 0; wi < (long long)mine.size(); wi++) {
        Work &w = work[wi];
        w.tile = mine[wi];
        w.texels = rasterize(scene, layout, layout.tiles[w.tile]);
        size_t n = w.texels.size();
        w.chart.resize(n);
        w.normal.resize(n);
        w.valid.resize(n);
        for (size_t i = 0; i < n; i++) {
            const lb_texel &t = w.texels[i];
            w.chart[i] = covered(t) ? texel_chart(t) : 0xffffffffu;
            w.normal[i] = {t.normal[0], t.normal[1], t.normal[2]};
            w.valid[i] = covered(t);
        }
    }
    std::vector<lb_texel> covered_list;
    std::vector<size_t> cov_counts;
    for (auto &w : work) {
        size_t c = 0;
        for (auto &t : w.texels)
            if (covered(t)) {
                covered_list.push_back(t);
                c++;
            }
        cov_counts.push_back(c);
    }
    uint64_t direct_base = 0, covered_all = 0;
    shared_counts(cov_counts, direct_base, covered_all);
    auto t0 = std::chrono::steady_clock::now();
    std::vector<float> direct;
    lb_params p_direct = params;
    p_direct.atlas[2] = uint32_t(direct_base);
    stats.rays_direct = gpu.run(LB_PASS_DIRECT, p_direct, covered_list, {}, direct);
    stats.t_direct = since(t0);
    log("sun and occlusion: " + std::to_string(covered_list.size()) + " texels, " + fmt("%.1f s", stats.t_direct));

    // materials much of whose surface lies inside solids (bake.rs:154-194)
    {
        std::vector<std::pair<size_t, size_t>> per(h.materials.size(), {0, 0});
        std::vector<std::pair<uint32_t, uint32_t>> chart(layout.charts.size(), {0, 0});
        size_t k = 0;
        for (auto &w : work)
            for (auto &t : w.texels) {
                if (!covered(t)) continue;
                uint32_t ci = texel_chart(t);
                size_t m = h.meshes[layout.charts[ci].mesh].material;
                bool ins = direct[k * 4 + 3] > b.inside_share;
                per[m].first++;
                per[m].second += ins;
                chart[ci].first++;
                chart[ci].second += ins;
                k++;
            }
        std::set<uint32_t> baked;
        for (auto &w : work)
            for (uint32_t c : layout.tiles[w.tile].charts) baked.insert(c);
        size_t empty = 0, inside = 0;
        for (uint32_t c : baked) {
            empty += chart[c].first == 0;
            inside += chart[c].first > 0 && chart[c].second == chart[c].first;
        }
        log("charts baked: " + std::to_string(baked.size()) + ", without a texel: " + std::to_string(empty) +
            ", all inside solids: " + std::to_string(inside));
        for (size_t m = 0; m < per.size(); m++)
            if (per[m].first > 2000 && per[m].second * 3 > per[m].first)
                log("warning: " + h.materials[m].name + ": " + std::to_string(per[m].second * 100 / per[m].first) +
                    "% of its " + std::to_string(per[m].first) +
                    " texels lie inside solids (hidden or overlapping faces, or faces turned inside out)");
    }

    // the sun's field, occlusion and the direct light, per tile (bake.rs:196-275)
    std::vector<size_t> counts;
    for (auto &w : work) counts.push_back(size_t(std::count(w.valid.begin(), w.valid.end(), 1)));
    std::vector<size_t> starts = offsets(counts);
    std::vector<TileLight> made(work.size());
    Vec3 irr = v3(h.sun.irradiance);
#pragma omp parallel for schedule(dynamic, 1)
    for (long long wi = 0; wi < (long long)work.size(); wi++) {
        Work &w = work[wi];
        const Tile &t = layout.tiles[w.tile];
        size_t size = size_t(t.w) * t.h;
        std::vector<uint8_t> state(size, V_NONE);
        std::vector<float> soft(size, 0.0f), ao(size, 1.0f);
        std::vector<uint32_t> hard(size, 0);
        size_t k = starts[wi];
        for (size_t i = 0; i < size; i++) {
            if (!w.valid[i]) continue;
            const float *r = &direct[k * 4];
            k++;
            if (r[3] > b.inside_share) {
                w.valid[i] = 0;
                continue;
            }
            soft[i] = r[0];
            uint32_t bits = f2u(r[1]);
            hard[i] = bits & 0x00ffffffu;
            uint32_t pick = bits >> 24;
            state[i] = pick == 0 ? V_CENTRE : pick == 9 ? V_PUSHED : V_OFFSET;
            lb_texel &tx = w.texels[i];
            if (pick == 9) {
                for (int c = 0; c < 3; c++) tx.pos[c] += tx.normal[c] * PUSH;
            } else if (pick > 0) {
                float cx, cy;
                texel_offset(pick, cx, cy);
                for (int c = 0; c < 3; c++) tx.pos[c] += tx.dx[c] * cx + tx.dy[c] * cy;
            }
            ao[i] = std::fmax(std::pow(std::fmax(1.0f - b.ao_strength * r[2], 0.0f), b.ao_contrast), b.ao_floor);
        }
        Surface s{t.w, t.h, w.chart.data(), w.normal.data()};
        size_t rings = lm.padding + 4;
        std::vector<float> aos = smooth(s, ao, 1, w.valid, 1);
        std::vector<float> softs = smooth(s, soft, 1, w.valid, 1);
        std::vector<float> field = sun_field(s, hard, w.valid, g, b.sdf_radius);
        std::vector<float> dl(size * 3);
        for (size_t i = 0; i < size; i++) {
            Vec3 n(w.normal[i][0], w.normal[i][1], w.normal[i][2]);
            Vec3 d = (irr * std::fmax(n.dot(sun), 0.0f)) * softs[i];
            dl[i * 3] = d.x;
            dl[i * 3 + 1] = d.y;
            dl[i * 3 + 2] = d.z;
        }
        std::vector<uint8_t> known = w.valid;
        {
            std::vector<uint8_t> k1 = known, k2 = known;
            fill(s, aos, 1, k1, rings);
            fill(s, field, 1, k2, rings);
        }
        fill(s, dl, 3, known, rings);
        for (size_t i = 0; i < size; i++)
            if (covered(w.texels[i]) && state[i] == V_NONE && known[i]) state[i] = V_FILLED;
        TileLight L;
        L.state = std::move(state);
        L.known.resize(size);
        for (size_t i = 0; i < size; i++) L.known[i] = w.valid[i] ? 2 : known[i];
        L.field = std::move(field);
        L.ao = std::move(aos);
        L.direct.resize(size);
        for (size_t i = 0; i < size; i++) L.direct[i] = {dl[i * 3], dl[i * 3 + 1], dl[i * 3 + 2]};
        L.indirect.assign(size, {0.0f, 0.0f, 0.0f});
        made[wi] = std::move(L);
    }
    for (size_t wi = 0; wi < work.size(); wi++) lights[work[wi].tile] = std::move(made[wi]);

    // the bounces, each gathering what the last left in the atlas (bake.rs:277-330): this rank's tiles'
    // light, the other ranks' through the sum, the cached tiles' (the same on every rank) after it
    std::vector<float> light(aw * ah * 4, 0.0f);
    auto share_light = [&]() {
        std::fill(light.begin(), light.end(), 0.0f);
        for (auto &w : work) write_light(layout, w.tile, *lights[w.tile], light);
        sum_words(light.data(), light.size());
        for (size_t ti : cached) write_light(layout, ti, *lights[ti], light);
    };
    share_light();
    size_t ds = lm.indirect_downscale;
    for (auto &w : work) {
        size_t tw = layout.tiles[w.tile].w;
        size_t bw = (tw + ds - 1) / ds;
        auto block = [&](size_t i) { return ((i / tw) / ds) * bw + (i % tw) / ds; };
        size_t n = w.valid.size();
        w.gathered.assign(n, 0);
        std::set<std::pair<size_t, uint32_t>> seen;
        for (size_t i = 0; i < n; i++)
            if (w.valid[i] && (i % tw) % ds == 0 && (i / tw) % ds == 0) {
                w.gathered[i] = 1;
                seen.insert({block(i), w.chart[i]});
            }
        for (size_t i = 0; i < n; i++)
            if (w.valid[i] && seen.insert({block(i), w.chart[i]}).second) w.gathered[i] = 1;
    }
    std::vector<lb_texel> gather;
    std::vector<size_t> gcounts;
    for (auto &w : work) {
        size_t c = 0;
        for (size_t i = 0; i < w.texels.size(); i++)
            if (w.gathered[i]) {
                gather.push_back(w.texels[i]);
                c++;
            }
        gcounts.push_back(c);
    }
    std::vector<size_t> gstarts = offsets(gcounts);
    uint64_t gather_base = 0, gathered_all = 0;
    shared_counts(gcounts, gather_base, gathered_all);
    lb_params p_gather = params;
    p_gather.atlas[2] = uint32_t(gather_base);
    auto tb = std::chrono::steady_clock::now();
    for (uint32_t bounce = 0; bounce < b.gi_bounces; bounce++) {
        auto t1 = std::chrono::steady_clock::now();
        std::vector<float> res;
        stats.rays_gather += gpu.run(LB_PASS_GATHER, p_gather, gather, light, res);
        std::vector<std::vector<float>> updated(work.size());
#pragma omp parallel for schedule(dynamic, 1)
        for (long long wi = 0; wi < (long long)work.size(); wi++) {
            Work &w = work[wi];
            const Tile &t = layout.tiles[w.tile];
            size_t size = size_t(t.w) * t.h;
            std::vector<float> e(size * 3, 0.0f);
            size_t k = gstarts[wi];
            for (size_t i = 0; i < size; i++)
                if (w.gathered[i]) {
                    e[i * 3] = res[k * 4];
                    e[i * 3 + 1] = res[k * 4 + 1];
                    e[i * 3 + 2] = res[k * 4 + 2];
                    k++;
                }
            Surface s{t.w, t.h, w.chart.data(), w.normal.data()};
            std::vector<float> sm = smooth(s, e, 3, w.gathered, size_t(b.gi_filter) * ds);
            std::vector<uint8_t> gk = w.gathered;
            fill(s, sm, 3, gk, lm.padding + 2 * ds + 2);
            updated[wi] = std::move(sm);
        }
        for (size_t wi = 0; wi < work.size(); wi++) {
            TileLight &l = *lights[work[wi].tile];
            for (size_t i = 0; i < l.indirect.size(); i++)
                l.indirect[i] = {updated[wi][i * 3], updated[wi][i * 3 + 1], updated[wi][i * 3 + 2]};
        }
        share_light();
        log("bounce " + std::to_string(bounce + 1) + ": " + std::to_string(gather.size()) + " texels x " +
            std::to_string(b.gi_rays) + " rays, " + fmt("%.1f s", since(t1)));
    }
    stats.t_bounces = since(tb);
    std::optional<Volume> volume;
    auto tv = std::chrono::steady_clock::now();
    if (h.volume)
        volume = bake_volume(scene, gpu, params, light, *h.volume, boxes, global, cache, stats, o.log, rank, world,
                             sum_words);
    stats.t_volume = since(tv);
    // texels left without light of their own take the volume's (bake.rs:335-359)
    auto tc = std::chrono::steady_clock::now();
    if (volume) {
        size_t fixed = 0;
        for (auto &w : work) {
            TileLight &l = *lights[w.tile];
            for (size_t i = 0; i < w.texels.size(); i++) {
                const lb_texel &t = w.texels[i];
                if (!covered(t) || l.known[i] != 0) continue;
                Vec3 n(t.normal[0], t.normal[1], t.normal[2]);
                float e[3], vs;
                volume->irradiance(Vec3(t.pos[0], t.pos[1], t.pos[2]) + n * 0.15f, n, e, vs);
                l.indirect[i] = {e[0], e[1], e[2]};
                Vec3 d = (irr * std::fmax(n.dot(sun), 0.0f)) * vs;
                l.direct[i] = {d.x, d.y, d.z};
                l.field[i] = vs > 0.5f ? 1.0f : 0.0f;
                l.ao[i] = 1.0f;
                l.known[i] = 1;
                l.state[i] = V_VOLUME;
                fixed++;
            }
        }
        if (fixed > 0) log(std::to_string(fixed) + " texels without light of their own lit from the volume");
    }
    for (auto &w : work) cache.put("tile", hashes[w.tile], lights[w.tile]->pack());

    // the atlas from every tile (bake.rs:364-421): this rank's tiles, the others' through the sums (each
    // ds x ds block lies in one tile: tiles start on a 4-texel grid and ds divides 4), then the cached tiles'
    Bake out;
    size_t iw = (aw + ds - 1) / ds, ih = (ah + ds - 1) / ds;
    std::vector<std::array<float, 2>> dpart(aw * ah, {0.0f, 0.0f});
    std::vector<uint8_t> vpart((aw * ah + 3) & ~size_t(3), 0), kpart((aw * ah + 3) & ~size_t(3), 0);
    std::vector<std::array<float, 4>> sum(iw * ih, {0, 0, 0, 0});
    auto put = [&](size_t ti) {
        const Tile &t = layout.tiles[ti];
        const TileLight &l = *lights[ti];
        for (size_t y = 0; y < t.h; y++)
            for (size_t x = 0; x < t.w; x++) {
                size_t i = y * t.w + x;
                if (l.known[i] == 0) continue;
                size_t ax = t.x + x, ay = t.y + y;
                dpart[ay * aw + ax] = {l.field[i], l.ao[i]};
                vpart[ay * aw + ax] = l.state[i];
                kpart[ay * aw + ax] = 1;
                float k = l.known[i] == 2 ? 1.0f : 1e-3f;
                auto &s = sum[(ay / ds) * iw + ax / ds];
                for (int c = 0; c < 3; c++) s[c] += l.indirect[i][c] * k;
                s[3] += k;
            }
    };
    for (auto &w : work) put(w.tile);
    sum_words(dpart.data(), dpart.size() * 2);
    sum_words(vpart.data(), vpart.size() / 4);
    sum_words(kpart.data(), kpart.size() / 4);
    sum_words(sum.data(), sum.size() * 4);
    for (size_t ti : cached) put(ti);
    out.direct.resize(aw * ah);
    out.validity.resize(aw * ah);
    for (size_t a = 0; a < aw * ah; a++) {
        out.direct[a] = kpart[a] ? dpart[a] : std::array<float, 2>{1.0f, 1.0f};
        out.validity[a] = vpart[a];
    }
    out.indirect.resize(iw * ih);
    std::vector<uint8_t> has(iw * ih);
    for (size_t i = 0; i < iw * ih; i++) {
        const auto &s = sum[i];
        if (s[3] > 0.0f) out.indirect[i] = {s[0] / s[3], s[1] / s[3], s[2] / s[3]};
        else out.indirect[i] = {0.0f, 0.0f, 0.0f};
        has[i] = s[3] > 0.0f;
    }
    for (int pass = 0; pass < 2; pass++) {
        std::vector<uint8_t> was = has;
        std::vector<std::array<float, 3>> src = out.indirect;
        for (size_t y = 0; y < ih; y++)
            for (size_t x = 0; x < iw; x++) {
                size_t i = y * iw + x;
                if (was[i]) continue;
                float acc[3] = {0, 0, 0};
                int n = 0;
                for (size_t yy = y > 0 ? y - 1 : 0; yy < std::min(y + 2, ih); yy++)
                    for (size_t xx = x > 0 ? x - 1 : 0; xx < std::min(x + 2, iw); xx++) {
                        size_t j = yy * iw + xx;
                        if (was[j]) {
                            for (int c = 0; c < 3; c++) acc[c] += src[j][c];
                            n++;
                        }
                    }
                if (n > 0) {
                    out.indirect[i] = {acc[0] / float(n), acc[1] / float(n), acc[2] / float(n)};
                    has[i] = 1;
                }
            }
    }
    stats.t_composite = since(tc);
    stats.tiles = nt;
    stats.tiles_baked = dirty.size();
    stats.texels_baked = covered_all;
    stats.chunks = volume ? volume->chunks : 0;
    stats.chunks_baked = volume ? volume->chunks_baked : 0;
    stats.seconds = since(started);
    out.layout = std::move(layout);
    out.iw = uint32_t(iw);
    out.ih = uint32_t(ih);
    out.volume = std::move(volume);
    out.stats = stats;
    return out;
}

}  // namespace lb
