// The device-resident bake (the batched mode): every dirty tile rebaked in one CUDA graph.
//
// The host does what only it can do cheaply before the first ray: read the scene, lay out the charts,
// build the BVH, hash the tiles against the cache and rasterise the dirty ones (the reference's steps,
// crates/lightbaker/src/bake.rs:94-149). Then one graph runs the rest on the device with no host round
// trip: the direct pass over every dirty texel at once (tiles of any size in one persistent launch), the
// texel passes, the gather selection and its compaction, every bounce (gather pass, smoothing, fill,
// the atlas rewritten), the volume and its fill, the fallback and the atlas composite. The graph is
// captured once per scene and can be replayed (a rebake of the same dirty set).
//
// Results equal the drop-in bake's (the host passes) record for record: the ray passes are the
// shader's arithmetic in its order, the texel passes the host's.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <string>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <stdexcept>
#include <vector>

#include "host/bake.h"
#include "host/cache.h"
#include "host/deps.h"
#include "host/handles.h"
#include "host/raster.h"
#include "lb_deps.h"
#include "lb_device.cuh"
#include "lb_kernels.h"
#include "lb_post.h"
#include "lb_runtime.h"
#include "plan.h"

using lbplan::ck;
using lbplan::DBuf;
using lbplan::gauss_weights;
using lbplan::since;

PostArgs lb_plan_post_args(lb_plan &p) {
    const lb::SceneHeader &h = p.scene.header;
    const lb::BakeSettings &b = h.bake;
    PostArgs a{};
    a.tiles = p.tiles_d.as<DTile>();
    a.n_tiles = int(p.dirty.size());
    a.n_texels = p.n_dirty_texels;
    a.tex = p.tex.as<float4>();
    a.cov_k = p.cov_k.as<uint32_t>();
    a.direct_out = p.direct_out.as<float4>();
    a.chart = p.chart.as<uint32_t>();
    a.valid = p.valid.as<uint8_t>();
    a.state = p.state.as<uint8_t>();
    a.known = p.known.as<uint8_t>();
    a.known_tmp = p.known_tmp.as<uint8_t>();
    a.gathered = p.gathered.as<uint8_t>();
    a.hard = p.hard.as<uint32_t>();
    a.gk = p.gk.as<uint32_t>();
    a.soft = p.soft.as<float>();
    a.ao_raw = p.ao_raw.as<float>();
    a.ao = p.ao.as<float>();
    a.field = p.field.as<float>();
    a.dl = p.dl.as<float4>();
    a.ind = p.ind.as<float4>();
    a.posg = p.posg.as<float4>();
    a.light = p.light.as<float4>();
    a.aw = p.aw;
    a.w1 = p.w1.as<float>();
    a.inside_share = b.inside_share;
    a.ao_strength = b.ao_strength;
    a.ao_contrast = b.ao_contrast;
    a.ao_floor = b.ao_floor;
    a.sdf_radius = b.sdf_radius;
    a.g = p.P.g;
    a.ds = p.ds;
    a.sun = make_float3(p.P.sun.x, p.P.sun.y, p.P.sun.z);
    a.irr = make_float3(h.sun.irradiance[0], h.sun.irradiance[1], h.sun.irradiance[2]);
    return a;
}

namespace {

// full occupancy for the kernel the pass launches with the plan's shape (walk, BVH, register cap)
int warp_blocks(const lb_plan &p, int pass) {
    lbd::Scene S = lb_scene_view(p.dscene);
    WarpPass w{};
    w.S = &S;
    w.pass = pass;
    w.sms = p.g->sms;
    const bool direct = pass == LB_PASS_DIRECT;
    w.bvh = direct ? p.bvh_direct : p.bvh_gather;
    w.refill = direct ? p.refill_direct : p.refill_gather;
    w.near = direct ? p.near_direct : p.near_gather;
    w.occ = direct ? p.occ_direct : p.occ_gather;
    return lb_warp_pass_blocks(w);
}

// A probe's position in the volume grid (volume.rs:36-37): x fastest, then z, then y.
lb::Vec3 probe_at(const lb::VolumeSettings &v, const std::array<uint32_t, 3> &size, size_t k) {
    size_t nx = size[0], nz = size[2];
    return lb::Vec3(v.min[0] + float(k % nx) * v.step, v.min[1] + float(k / (nx * nz)) * v.step,
                    v.min[2] + float((k / nx) % nz) * v.step);
}

// The volume's grid and its chunks, the probes of each ground-plan tile (volume.rs:34-41).
void volume_grid(const lb::VolumeSettings &v, float tile_size, std::array<uint32_t, 3> &size,
                 std::map<lb::TileKey, std::vector<uint32_t>> &chunks) {
    auto n = [&](int a) { return uint32_t(std::round((v.max[a] - v.min[a]) / v.step)) + 1; };
    size = {std::max(n(0), 2u), std::max(n(1), 2u), std::max(n(2), 2u)};
    chunks.clear();
    size_t np = size_t(size[0]) * size[1] * size[2];
    for (size_t k = 0; k < np; k++) chunks[lb::tile_of(probe_at(v, size, k), tile_size)].push_back(uint32_t(k));
}

// A chunk's seed (volume.rs:49-55): its key, then the volume's settings as JSON.
std::vector<uint8_t> chunk_seed(const lb::TileKey &key, const std::string &vjson) {
    std::vector<uint8_t> seed(8);
    std::memcpy(seed.data(), &key.first, 4);
    std::memcpy(seed.data() + 4, &key.second, 4);
    seed.insert(seed.end(), vjson.begin(), vjson.end());
    return seed;
}

// Every tile's and chunk's dependency hash (deps.rs:70-96, bake.rs:127-130, volume.rs:42-57), all on the
// device at once (deps.cu): the casting triangles concatenated here, the seeds hashed here.
void dependency_hashes(lb_gpu *g, const lb::Scene &scene, const lb::Layout &layout, const lb::Hash &global,
                       const std::map<lb::TileKey, std::vector<uint32_t>> *chunks, const std::array<uint32_t, 3> &vsize,
                       std::vector<lb::Hash> &tile_hashes, std::vector<lb::Hash> &chunk_hashes) {
    const lb::SceneHeader &h = scene.header;
    const lb::BakeSettings &b = h.bake;
    DepsInput in;
    std::vector<size_t> first(h.meshes.size() + 1, 0);
    for (size_t mi = 0; mi < h.meshes.size(); mi++) {
        bool casts = h.materials[h.meshes[mi].material].casts;
        first[mi + 1] = first[mi] + (casts ? scene.positions[mi].size() / 3 : 0);
    }
    std::vector<float> pos(first.back() * 9);
    in.tri_mesh.resize(first.back());
    in.mesh_start.push_back(0);
    std::vector<uint32_t> mesh_of(h.meshes.size(), 0);
    for (size_t mi = 0; mi < h.meshes.size(); mi++) {
        if (!h.materials[h.meshes[mi].material].casts) continue;
        mesh_of[mi] = uint32_t(in.mesh_id.size());
        in.mesh_id.push_back(uint32_t(mi));
        in.mesh_mat.push_back(h.meshes[mi].material);
        in.mesh_start.push_back(uint32_t(first[mi + 1]));
    }
    float top = -INFINITY;
#pragma omp parallel for schedule(dynamic, 16) reduction(max : top)
    for (long long mi = 0; mi < (long long)h.meshes.size(); mi++) {
        const std::vector<lb::Vec3> &P = scene.positions[mi];
        // the top of every triangle's box, casting or not (deps.rs:53)
        for (size_t t = 0; t + 2 < P.size(); t += 3)
            for (int k = 0; k < 3; k++) top = std::fmax(top, P[t + k].y);
        if (!h.materials[h.meshes[mi].material].casts) continue;
        float *dst = pos.data() + first[mi] * 9;
        for (size_t v = 0; v < P.size(); v++) {
            dst[v * 3] = P[v].x;
            dst[v * 3 + 1] = P[v].y;
            dst[v * 3 + 2] = P[v].z;
        }
        for (size_t t = first[mi]; t < first[mi + 1]; t++) in.tri_mesh[t] = mesh_of[mi];
    }
    in.pos = pos.data();
    in.n_tris = uint32_t(first.back());
    in.top = top;
    lb::Vec3 sun = lb::Vec3(h.sun.direction[0], h.sun.direction[1], h.sun.direction[2]).normalize();
    in.sun[0] = sun.x;
    in.sun[1] = sun.y;
    in.sun[2] = sun.z;
    // the queries: every tile (its surfaces' box, bake.rs:127-130), then every chunk (its probes' box)
    const size_t nt = layout.tiles.size(), nc = chunks ? chunks->size() : 0;
    std::vector<DepsQuery> qs(nt + nc);
    const float reach = b.gi_bounces > 0 ? std::fmax(b.gi_reach, b.ao_reach) : b.ao_reach;
#pragma omp parallel for schedule(dynamic, 1)
    for (long long ti = 0; ti < (long long)nt; ti++) {
        const lb::Tile &t = layout.tiles[ti];
        lb::Aabb own = lb::tile_box(scene, layout, t.charts);
        DepsQuery &q = qs[ti];
        q.min[0] = own.min.x, q.min[1] = own.min.y, q.min[2] = own.min.z;
        q.max[0] = own.max.x, q.max[1] = own.max.y, q.max[2] = own.max.z;
        q.reach = reach;
        std::vector<uint8_t> seed = lb::tile_seed(scene, layout, t.key, t.charts);
        q.prefix.assign(global.begin(), global.end());
        q.prefix.insert(q.prefix.end(), seed.begin(), seed.end());
    }
    if (chunks) {
        const lb::VolumeSettings &v = *h.volume;
        std::string vjson = lb::to_json(v).dump();
        size_t c = nt;
        for (auto &kv : *chunks) {
            lb::Aabb own;
            for (uint32_t k : kv.second) own.add(probe_at(v, vsize, k));
            DepsQuery &q = qs[c++];
            q.min[0] = own.min.x, q.min[1] = own.min.y, q.min[2] = own.min.z;
            q.max[0] = own.max.x, q.max[1] = own.max.y, q.max[2] = own.max.z;
            q.reach = b.gi_reach;
            std::vector<uint8_t> seed = chunk_seed(kv.first, vjson);
            q.prefix.assign(global.begin(), global.end());
            q.prefix.insert(q.prefix.end(), seed.begin(), seed.end());
        }
    }
    std::vector<std::array<uint8_t, 32>> out;
    lb_hash_reach_device(g, in, qs, out);
    tile_hashes.assign(out.begin(), out.begin() + nt);
    chunk_hashes.assign(out.begin() + nt, out.end());
}

void build(lb_plan &p) {
    auto t0 = std::chrono::steady_clock::now();
    const lb::SceneHeader &h = p.scene.header;
    const lb::BakeSettings &b = h.bake;
    const lb::LightmapSettings &lm = h.lightmap;
    p.P = lb::prepare(p.scene);
    auto mark = [&](const char *what) { p.build_phases += std::string(what) + " " + std::to_string(since(t0)) + " s; "; };
    mark("layout and BVH");
    lb::Layout &layout = p.P.layout;
    p.aw = layout.width;
    p.ah = layout.height;
    p.ds = lm.indirect_downscale;
    p.iw = (p.aw + p.ds - 1) / p.ds;
    p.ih = (p.ah + p.ds - 1) / p.ds;
    p.dscene = lb_scene_upload(p.g, p.P.bvh.nodes.data(), p.P.bvh.nodes.size(), p.P.bvh.tris.data(),
                               p.P.bvh.tris.size(), p.P.materials.data(), p.P.materials.size() / 4,
                               p.P.affines.data(), p.P.affines.size() / 8);
    if (!p.dscene) throw std::runtime_error(lb_last_error());
    if (p.opt.watertight &&
        lb_scene_set_vertices(p.g, p.dscene, p.P.bvh.verts.data(), p.P.bvh.tris.size()) != LB_OK)
        throw std::runtime_error(lb_last_error());

    // the cache (bake.rs:123-136); without a cache directory nothing is read or written, so the tiles' and
    // chunks' hashes (only ever cache keys) are not computed
    lb::Cache cache(p.opt.cache);
    const bool caching = !p.opt.cache.empty();
    if (h.volume) volume_grid(*h.volume, lm.tile_size, p.vsize, p.chunks);
    size_t nt = layout.tiles.size();
    p.hashes.resize(nt);
    p.lights.resize(nt);
    std::vector<lb::Hash> chunk_hashes;
    if (caching) {
        // every tile's and chunk's hash at once on the device
        lb::Hash global = lb::global_hash(p.scene);
        if (p.opt.watertight) global = lb::watertight_hash(global);
        dependency_hashes(p.g, p.scene, layout, global, h.volume ? &p.chunks : nullptr, p.vsize, p.hashes,
                          chunk_hashes);
        mark("dependency hashes");
#pragma omp parallel for schedule(dynamic, 1)
        for (long long ti = 0; ti < (long long)nt; ti++) {
            const lb::Tile &t = layout.tiles[ti];
            if (auto bytes = cache.get("tile", p.hashes[ti]))
                p.lights[ti] = lb::TileLight::unpack(*bytes, size_t(t.w) * t.h);
        }
    }
    for (size_t i = 0; i < nt; i++)
        if (!p.lights[i]) p.dirty.push_back(i);
    p.order = p.dirty;
    for (size_t i = 0; i < nt; i++)
        if (p.lights[i]) p.order.push_back(i);

    // device texel layout: dirty tiles first
    uint32_t off = 0;
    for (size_t k = 0; k < p.order.size(); k++) {
        const lb::Tile &t = layout.tiles[p.order[k]];
        p.tiles_all.push_back(DTile{t.x, t.y, t.w, t.h, off});
        off += t.w * t.h;
        if (k + 1 == p.dirty.size()) p.n_dirty_texels = off;
    }
    p.n_all = off;
    if (p.dirty.empty()) p.n_dirty_texels = 0;
    mark("upload and cache");

    // rasterise the dirty tiles (bake.rs:138-149) on the device: the host sets up each tile's triangles in
    // the host rasteriser's order (raster.rs:48-67), the device writes the texels (raster.cu), lists the
    // covered ones and counts the (block, chart) pairs that bound the gathered texels (bake.rs:286-297)
    cudaStream_t st = p.g->stream;
    const std::vector<RasterTri> rtris = lb::raster_triangles(p.scene, layout, p.dirty);
    mark("raster set-up");
    const size_t NT = p.n_dirty_texels ? p.n_dirty_texels : 1;
    p.tiles_d.alloc(std::max<size_t>(1, p.tiles_all.size()) * sizeof(DTile));
    p.tex.alloc(NT * 64);
    p.cov_idx.alloc(NT * 4);
    p.cov_k.alloc(NT * 4);
    DBuf rt, raster_temp, raster_counts;
    rt.alloc(std::max<size_t>(1, rtris.size()) * sizeof(RasterTri));
    raster_counts.alloc(16);
    const size_t raster_bytes = lb_raster_covered_temp(uint32_t(NT));
    raster_temp.alloc(raster_bytes);
    if (!p.tiles_all.empty())
        ck(cudaMemcpyAsync(p.tiles_d.p, p.tiles_all.data(), p.tiles_all.size() * sizeof(DTile), cudaMemcpyHostToDevice,
                           st),
           "upload");
    if (!rtris.empty())
        ck(cudaMemcpyAsync(rt.p, rtris.data(), rtris.size() * sizeof(RasterTri), cudaMemcpyHostToDevice, st), "upload");
    p.g->h2d += p.tiles_all.size() * sizeof(DTile) + rtris.size() * sizeof(RasterTri);
    mark("raster allocations and upload");
    unsigned long long *pairs_d = raster_counts.as<unsigned long long>();
    uint32_t *ncov_d = reinterpret_cast<uint32_t *>(pairs_d + 1);
    ck(lb_raster_tiles(rt.as<RasterTri>(), uint32_t(rtris.size()), p.tiles_d.as<DTile>(), uint32_t(p.dirty.size()),
                       p.n_dirty_texels, p.ds, p.tex.as<float4>(), p.cov_k.as<uint32_t>(), pairs_d, p.g->sms, st),
       "raster");
    ck(lb_raster_covered(p.tex.as<float4>(), p.n_dirty_texels, raster_temp.p, raster_bytes, p.cov_idx.as<uint32_t>(),
                         ncov_d, p.cov_k.as<uint32_t>(), p.g->sms, st),
       "covered texels");
    uint64_t counts[2] = {0, 0};
    ck(cudaMemcpyAsync(counts, raster_counts.p, 16, cudaMemcpyDeviceToHost, st), "raster counts");
    ck(cudaStreamSynchronize(st), "raster");
    p.max_gathered = p.n_dirty_texels ? counts[0] : 0;
    p.n_cov = p.n_dirty_texels ? uint32_t(counts[1] & 0xffffffffu) : 0;
    mark("raster");

    // cached tiles' light and the atlas the first bounce reads (all zero when no tile comes from the cache:
    // then cleared on the device instead); the atlas owner map is built on the device
    const bool any_cached = p.dirty.size() < p.order.size();
    const size_t n_cached = any_cached ? p.n_all : 0, n_atlas = any_cached ? size_t(p.aw) * p.ah : 0;
    std::vector<uint8_t> known(n_cached, 0), state(n_cached, 0);
    std::vector<float> field(n_cached, 0.0f), ao(n_cached, 0.0f);
    std::vector<float> dl(n_cached * 4, 0.0f), ind(n_cached * 4, 0.0f);
    std::vector<float> light(n_atlas * 4, 0.0f);
    for (size_t k = 0; k < p.order.size(); k++) {
        size_t ti = p.order[k];
        const DTile &t = p.tiles_all[k];
        if (!p.lights[ti]) continue;
        const lb::TileLight &l = *p.lights[ti];
        for (uint32_t i = 0; i < t.w * t.h; i++) {
            uint32_t d = t.off + i;
            known[d] = l.known[i];
            state[d] = l.state[i];
            field[d] = l.field[i];
            ao[d] = l.ao[i];
            for (int c = 0; c < 3; c++) {
                dl[size_t(d) * 4 + c] = l.direct[i][c];
                ind[size_t(d) * 4 + c] = l.indirect[i][c];
            }
        }
        lb::write_light(layout, ti, l, light);
    }

    // the volume's probes: cached chunks, the rest to bake (volume.rs:34-84)
    std::vector<float> probes_init;
    std::vector<lb_texel> probe_items;
    std::vector<uint32_t> probe_slot;
    if (h.volume) {
        const lb::VolumeSettings &v = *h.volume;
        p.has_volume = true;
        p.n_probes = p.vsize[0] * p.vsize[1] * p.vsize[2];
        auto at = [&](size_t k) { return probe_at(v, p.vsize, k); };
        probes_init.assign(size_t(p.n_probes) * 16, 0.0f);
        size_t ci = 0;
        for (auto &kv : p.chunks) {
            lb::Hash hash{};
            if (caching) hash = chunk_hashes[ci];
            ci++;
            auto got = caching ? cache.get("probes", hash) : std::nullopt;
            if (got && got->size() == kv.second.size() * 64) {
                for (size_t i = 0; i < kv.second.size(); i++)
                    std::memcpy(&probes_init[size_t(kv.second[i]) * 16], got->data() + i * 64, 64);
            } else {
                for (uint32_t k : kv.second) {
                    lb::Vec3 q = at(k);
                    probe_items.push_back(lb_texel{{q.x, q.y, q.z, 1.0f}, {0.0f, 1.0f, 0.0f, lb::u2f(k)}, {0, 0, 0, 0}, {0, 0, 0, 0}});
                    probe_slot.push_back(k);
                }
                p.chunk_keys.emplace_back(hash, kv.second);
            }
        }
        p.n_chunks = p.chunks.size();
        p.n_todo = uint32_t(probe_items.size());
    }

    mark("atlas and volume");
    // device memory
    size_t N = p.n_dirty_texels ? p.n_dirty_texels : 1, A = p.n_all ? p.n_all : 1;
    p.direct_out.alloc(std::max<size_t>(1, size_t(p.n_cov)) * 16);
    p.chart.alloc(A * 4);
    for (DBuf *d : {&p.valid, &p.known_tmp, &p.gathered}) d->alloc(N);
    for (DBuf *d : {&p.state, &p.known}) d->alloc(A);
    for (DBuf *d : {&p.hard, &p.gk, &p.soft, &p.ao_raw}) d->alloc(N * 4);
    for (DBuf *d : {&p.ao, &p.field}) d->alloc(A * 4);
    for (DBuf *d : {&p.dl, &p.ind}) d->alloc(A * 16);
    p.posg.alloc(N * 16);
    p.light.alloc(size_t(p.aw) * p.ah * 16);
    std::vector<float> w1 = gauss_weights(1), wr = gauss_weights(int(b.gi_filter * p.ds));
    p.w1.alloc(w1.size() * 4);
    p.wr.alloc(wr.size() * 4);
    p.gath_idx.alloc(N * 4);
    p.gath_count.alloc(16);
    p.gather_out.alloc(std::max<size_t>(1, size_t(p.n_cov)) * 16);
    p.select_bytes = lb_select_temp_bytes(uint32_t(N));
    p.select_temp.alloc(p.select_bytes);
    for (DBuf *d : {&p.s_ka, &p.s_kb}) d->alloc(N);
    for (DBuf *d : {&p.s_f1, &p.s_f2}) d->alloc(N * 4);
    for (DBuf *d : {&p.s_v4, &p.s_e0, &p.s_e1}) d->alloc(N * 16);
    size_t NP = p.n_probes ? p.n_probes : 1;
    p.probes.alloc(NP * 64);
    p.probes_init.alloc(NP * 64);
    p.probes_b.alloc(NP * 64);
    p.probe_items.alloc(std::max<size_t>(1, probe_items.size()) * 64);
    p.probe_slot.alloc(std::max<size_t>(1, probe_slot.size()) * 4);
    p.pk_a.alloc(NP);
    p.pk_b.alloc(NP);
    p.owner.alloc(size_t(p.aw) * p.ah * 4);
    p.direct_atlas.alloc(size_t(p.aw) * p.ah * 8);
    p.validity.alloc(size_t(p.aw) * p.ah);
    p.indirect.alloc(size_t(p.iw) * p.ih * 16);
    p.indirect_b.alloc(size_t(p.iw) * p.ih * 16);
    p.has.alloc(size_t(p.iw) * p.ih);
    p.has_b.alloc(size_t(p.iw) * p.ih);
    p.enc_bc5.alloc(size_t(p.aw) * p.ah);
    p.enc_rgb.alloc(size_t(p.iw) * p.ih * 4);
    p.enc_vol.alloc(NP * 16);
    p.enc_scale.alloc(4);
    p.counters.alloc(16 * 8);  // rays, nodes, tris, mats of each pass; then the passes' work counters
    // the first bounce's gather records, which the later bounces evaluate instead of tracing again (their
    // rays are the first bounce's: the keys depend on the gathered texel, not the bounce), and theta at the
    // scene's own values for that evaluation
    std::vector<float> theta;
    for (auto &m : h.materials) theta.insert(theta.end(), m.albedo.begin(), m.albedo.end());
    for (auto *c : {&h.sky.zenith, &h.sky.horizon, &h.sky.ground}) theta.insert(theta.end(), c->begin(), c->end());
    theta.push_back(1.0f);
    p.theta0.alloc(theta.size() * 4);
    bool recording = (p.reuse && b.gi_bounces > 1) || (p.keep_records && b.gi_bounces > 0);
    p.records.alloc(recording ? p.max_gathered * p.P.params.counts[2] * 8 : 16);
    const bool vrecording = p.keep_records && h.volume && p.n_todo;
    p.vrecords.alloc(vrecording ? size_t(p.n_todo) * h.volume->rays * 8 : 16);
    p.vraw.alloc(vrecording ? size_t(p.n_probes) * 64 : 16);

    mark("allocations");
    auto up = [&](DBuf &d, const void *src, size_t bytes) {
        if (bytes) {
            ck(cudaMemcpyAsync(d.p, src, bytes, cudaMemcpyHostToDevice, st), "upload");
            p.g->h2d += bytes;
        }
    };
    up(p.theta0, theta.data(), theta.size() * 4);
    if (any_cached) {
        up(p.known, known.data(), known.size());
        up(p.state, state.data(), state.size());
        up(p.field, field.data(), field.size() * 4);
        up(p.ao, ao.data(), ao.size() * 4);
        up(p.dl, dl.data(), dl.size() * 4);
        up(p.ind, ind.data(), ind.size() * 4);
        up(p.light, light.data(), light.size() * 4);
    } else {
        for (auto *d : {&p.known, &p.state}) ck(cudaMemsetAsync(d->p, 0, p.n_all, st), "clear");
        for (auto *d : {&p.field, &p.ao}) ck(cudaMemsetAsync(d->p, 0, size_t(p.n_all) * 4, st), "clear");
        for (auto *d : {&p.dl, &p.ind}) ck(cudaMemsetAsync(d->p, 0, size_t(p.n_all) * 16, st), "clear");
        ck(cudaMemsetAsync(p.light.p, 0, size_t(p.aw) * p.ah * 16, st), "clear");
    }
    ck(lb_owner_map(p.tiles_d.as<DTile>(), uint32_t(p.tiles_all.size()), p.aw, p.ah, p.owner.as<uint32_t>(), p.g->sms,
                    st),
       "owner map");
    up(p.w1, w1.data(), w1.size() * 4);
    up(p.wr, wr.data(), wr.size() * 4);
    up(p.probes_init, probes_init.data(), probes_init.size() * 4);
    up(p.probe_items, probe_items.data(), probe_items.size() * 64);
    up(p.probe_slot, probe_slot.data(), probe_slot.size() * 4);
    ck(cudaStreamSynchronize(st), "upload");
    p.blocks_direct = warp_blocks(p, LB_PASS_DIRECT);
    p.blocks_gather = warp_blocks(p, LB_PASS_GATHER);
    p.blocks_volume = warp_blocks(p, LB_PASS_VOLUME);
    mark("device arrays");
    p.t_prepare = since(t0);
}

// The autotuner: times the warp passes on a sample of this plan's covered texels (every k-th, up to
// 16384) for each ray order and persistent grid size, and keeps the fastest for the graph. Results do
// not depend on either choice.
void autotune(lb_plan &p) {
    if (p.n_cov == 0) return;
    cudaStream_t st = p.g->stream;
    lbd::Scene S = lb_scene_view(p.dscene);
    // a sample of texels spread over the map, large enough to keep every SM busy for a while (a small one
    // times the launch's tail, not its walk): 16 runs of consecutive covered texels, evenly spaced, so that
    // neighbouring warps work on neighbouring texels as in the whole pass (every n-th texel instead made
    // the shapes' times differ by under 1 % where the whole map's differed by 5 %)
    const uint32_t want = std::min<uint32_t>(p.n_cov, 65536), RUNS = 16;
    std::vector<uint32_t> sample;
    {
        std::vector<uint32_t> all(p.n_cov);
        ck(cudaMemcpy(all.data(), p.cov_idx.p, size_t(p.n_cov) * 4, cudaMemcpyDeviceToHost), "autotune");
        if (want == p.n_cov) {
            sample = all;
        } else {
            const uint32_t run = want / RUNS;
            for (uint32_t r = 0; r < RUNS; r++) {
                const uint64_t start = uint64_t(p.n_cov - run) * r / (RUNS - 1);
                sample.insert(sample.end(), all.begin() + start, all.begin() + start + run);
            }
        }
    }
    DBuf sidx, sout;
    sidx.alloc(sample.size() * 4);
    sout.alloc(sample.size() * 16);
    ck(cudaMemcpy(sidx.p, sample.data(), sample.size() * 4, cudaMemcpyHostToDevice), "autotune");
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int orders[] = {0, 8};
    struct Shape {
        int bvh, refill, near, occ;
    };
    // walks (the BVH2 with and without leaf lists) and register caps, each at full occupancy; lane refill
    // and the 8-wide BVH lost on every workload measured here and are left to the gpu handle's settings
    const Shape shapes[] = {{2, 0, 1, 0}, {2, 0, 1, 3}, {2, 0, 1, 4}, {2, 0, 0, 0}, {2, 0, 0, 3}, {2, 0, 0, 4}};
    std::string report;
    for (int pass : {LB_PASS_DIRECT, LB_PASS_GATHER}) {
        float best = 1e30f;
        int best_order = 8, best_blocks = 0, best_bvh = 2, best_refill = 0, best_near = 0, best_occ = 0, best_fetch = 0,
            best_ww = 0;
        for (const Shape &sh : shapes)
        for (int order : orders)
        for (int fetch : {0, 1})
        for (int ww : {0, 1}) {
            if (ww && pass != LB_PASS_DIRECT) continue;
            WarpPass probe{};
            probe.S = &S;
            probe.pass = pass;
            probe.sms = p.g->sms;
            probe.bvh = sh.bvh;
            probe.refill = sh.refill;
            probe.near = sh.near;
            probe.occ = sh.occ;
            int full = lb_warp_pass_blocks(probe);
            int per_sm = std::max(1, full / std::max(1, p.g->sms));
            for (int bps : {per_sm}) {
                WarpPass w{};
                w.pass = pass;
                w.S = &S;
                w.P = &p.P.params;
                w.tex = p.tex.as<float4>();
                w.idx = sidx.as<uint32_t>();
                w.n_host = uint32_t(sample.size());
                w.light = p.light.as<float4>();
                w.n_light = p.aw * p.ah;
                w.out = sout.as<float4>();
                w.counters = p.counters.as<unsigned long long>();
                w.sms = p.g->sms;
                w.blocks = bps * p.g->sms;
                w.group = order;
                w.bvh = sh.bvh;
                w.refill = sh.refill;
                w.near = sh.near;
                w.occ = sh.occ;
                w.work = fetch ? reinterpret_cast<unsigned int *>(p.counters.as<unsigned long long>() + 12) : nullptr;
                w.warp_walk = ww;
                float t = 0;
                for (int rep = 0; rep < 2; rep++) {
                    ck(cudaEventRecord(e0, st), "autotune");
                    ck(lb_launch_pass_warp(w, st), "autotune");
                    ck(cudaEventRecord(e1, st), "autotune");
                    ck(cudaEventSynchronize(e1), "autotune");
                    if (rep) cudaEventElapsedTime(&t, e0, e1);
                }
                if (t < best) {
                    best = t;
                    best_order = order;
                    best_blocks = bps * p.g->sms;
                    best_bvh = sh.bvh;
                    best_refill = sh.refill;
                    best_near = sh.near;
                    best_occ = sh.occ;
                    best_fetch = fetch;
                    best_ww = ww;
                }
            }
        }
        if (pass == LB_PASS_DIRECT) {
            p.group_direct = best_order;
            p.blocks_direct = best_blocks;
            p.bvh_direct = best_bvh;
            p.refill_direct = best_refill;
            p.near_direct = best_near;
            p.occ_direct = best_occ;
            p.fetch_direct = best_fetch;
            p.warp_walk = best_ww;
        } else {
            p.group_gather = best_order;
            p.blocks_gather = best_blocks;
            p.bvh_gather = best_bvh;
            p.refill_gather = best_refill;
            p.near_gather = best_near;
            p.occ_gather = best_occ;
            p.fetch_gather = best_fetch;
        }
        report += std::string(pass == LB_PASS_DIRECT ? "direct" : "gather") + ": bvh " + std::to_string(best_bvh) +
                  ", refill " + std::to_string(best_refill) + ", near " + std::to_string(best_near) + ", order " +
                  std::to_string(best_order) + ", register cap " + std::to_string(best_occ) + ", fetch " +
                  std::to_string(best_fetch) + (pass == LB_PASS_DIRECT ? ", warp walk " + std::to_string(best_ww) : "") +
                  ", " +
                  std::to_string(best_blocks / std::max(1, p.g->sms)) + " blocks/SM (" + std::to_string(best) +
                  " ms on " + std::to_string(sample.size()) + " texels); ";
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    p.tuned = report;
    if (p.opt.log) p.opt.log("autotune: " + report);
}

// The graph: everything from the direct pass to the atlas.
void capture(lb_plan &p) {
    const lb::SceneHeader &h = p.scene.header;
    const lb::BakeSettings &b = h.bake;
    cudaStream_t st = p.g->stream;
    lbd::Scene S = lb_scene_view(p.dscene);
    const lb_params &params = p.P.params;
    lb_params pvol = params;
    if (h.volume) pvol.counts[2] = h.volume->rays;
    PostArgs a = lb_plan_post_args(p);
    PostScratch s{p.s_ka.as<uint8_t>(), p.s_kb.as<uint8_t>(), p.s_f1.as<float>(), p.s_f2.as<float>(),
                  p.s_v4.as<float4>(), p.s_e0.as<float4>(), p.s_e1.as<float4>()};
    unsigned long long *cnt = p.counters.as<unsigned long long>();

    // a split bake: each pass takes this rank's share of its items, into outputs cleared first; the graph is
    // cut after the pass, where the launch sums the outputs over the ranks
    const bool split = p.world > 1;
    const uint32_t part = split ? uint32_t(p.rank) : 0, parts = split ? uint32_t(p.world) : 1;
    auto finish = [&](std::vector<std::pair<void *, size_t>> sums) {
        lb_plan::Piece pc;
        ck(cudaStreamEndCapture(st, &pc.graph), "end capture");
        pc.sums = std::move(sums);
        p.pieces.push_back(pc);
        ck(cudaGraphInstantiate(&p.pieces.back().exec, pc.graph, 0), "graph instantiate");
    };
    auto cut = [&](void *words, size_t count) {
        if (!split || !count) return;
        finish({{words, count}});
        ck(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "begin capture");
    };
    // the gather outputs a bounce's sum covers: every slot a gathered texel can take
    const size_t gather_slots = std::min<uint64_t>(p.max_gathered, p.n_cov);
    ck(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "begin capture");
    try {
        ck(cudaMemsetAsync(cnt, 0, 12 * 8, st), "counters");
        WarpPass w{};
        w.S = &S;
        w.sms = p.g->sms;
        w.full_count = false;
        w.part = part;
        w.parts = parts;
        if (p.n_cov && split) ck(cudaMemsetAsync(p.direct_out.p, 0, size_t(p.n_cov) * 16, st), "clear");
        if (p.n_cov) {
            w.pass = LB_PASS_DIRECT;
            w.P = &params;
            w.tex = p.tex.as<float4>();
            w.idx = p.cov_idx.as<uint32_t>();
            w.n_host = p.n_cov;
            w.out = p.direct_out.as<float4>();
            w.counters = cnt;
            w.blocks = p.blocks_direct;
            w.group = p.group_direct;
            w.bvh = p.bvh_direct;
            w.refill = p.refill_direct;
            w.near = p.near_direct;
            w.occ = p.occ_direct;
            w.work = p.fetch_direct ? reinterpret_cast<unsigned int *>(cnt + 12) : nullptr;
            w.warp_walk = p.warp_walk;
            ck(lb_launch_pass_warp(w, st), "direct pass");
            cut(p.direct_out.p, size_t(p.n_cov) * 4);
        }
        ck(lb_post_direct(a, int(h.lightmap.padding) + 4, s, st), "direct texel passes");
        ck(lb_select_gathered(a, p.select_temp.p, p.select_bytes, p.gath_idx.as<uint32_t>(), p.gath_count.as<uint32_t>(),
                              st),
           "gather selection");
        for (uint32_t bounce = 0; bounce < b.gi_bounces && p.n_dirty_texels; bounce++) {
            WarpPass gw{};
            gw.pass = LB_PASS_GATHER;
            gw.S = &S;
            gw.P = &params;
            gw.tex = p.tex.as<float4>();
            gw.idx = p.gath_idx.as<uint32_t>();
            gw.pos = p.posg.as<float4>();
            gw.n_dev = p.gath_count.as<uint32_t>();
            gw.light = p.light.as<float4>();
            gw.n_light = p.aw * p.ah;
            gw.out = p.gather_out.as<float4>();
            gw.counters = cnt + 4;
            gw.sms = p.g->sms;
            gw.blocks = p.blocks_gather;
            gw.group = p.group_gather;
            gw.bvh = p.bvh_gather;
            gw.refill = p.refill_gather;
            gw.near = p.near_gather;
            gw.occ = p.occ_gather;
            gw.work = p.fetch_gather ? reinterpret_cast<unsigned int *>(cnt + 13) : nullptr;
            gw.part = part;
            gw.parts = parts;
            bool replay = p.reuse && b.gi_bounces > 1, record = replay || p.keep_records;
            if (split && gather_slots)
                ck(cudaMemsetAsync(p.gather_out.p, 0, gather_slots * 16, st), "clear");
            if (replay && bounce > 0) {
                // the same rays met the same surfaces: evaluate the first bounce's records against this
                // bounce's atlas (the sums in ray order, as the pass sums them)
                ck(lb_eval_records(p.records.as<uint2>(), p.gath_count.as<uint32_t>(), 0, params.counts[2],
                                   p.light.as<float4>(), p.aw * p.ah, p.theta0.as<float>(),
                                   uint32_t(h.materials.size()), p.gather_out.as<float4>(), p.g->sms, st, part, parts),
                   "gather records");
            } else {
                gw.rec = record && bounce == 0 ? p.records.as<uint2>() : nullptr;
                ck(lb_launch_pass_warp(gw, st), "gather pass");
            }
            cut(p.gather_out.p, gather_slots * 4);
            ck(lb_post_bounce(a, p.gather_out.as<float4>(), int(b.gi_filter * p.ds), p.wr.as<float>(),
                              int(h.lightmap.padding + 2 * p.ds + 2), s, st),
               "bounce texel passes");
        }
        if (p.has_volume) {
            // the probes the cache holds, then the ones baked here (every launch starts from the same grid; in a
            // split bake rank 0 brings the cached probes and every rank its share of the rest, zero elsewhere)
            if (!split || p.rank == 0)
                ck(cudaMemcpyAsync(p.probes.p, p.probes_init.p, size_t(p.n_probes) * 64, cudaMemcpyDeviceToDevice,
                                   st),
                   "probes");
            else
                ck(cudaMemsetAsync(p.probes.p, 0, size_t(p.n_probes) * 64, st), "probes");
            if (p.n_todo) {
                WarpPass vw{};
                vw.pass = LB_PASS_VOLUME;
                vw.S = &S;
                vw.P = &pvol;
                vw.tex = p.probe_items.as<float4>();
                vw.n_host = p.n_todo;
                vw.light = p.light.as<float4>();
                vw.n_light = p.aw * p.ah;
                vw.out = p.probes.as<float4>();
                vw.slot = p.probe_slot.as<uint32_t>();
                vw.counters = cnt + 8;
                vw.sms = p.g->sms;
                vw.blocks = p.blocks_volume;
                vw.bvh = p.bvh_volume;
                vw.part = part;
                vw.parts = parts;
                vw.rec = p.keep_records ? p.vrecords.as<uint2>() : nullptr;
                ck(lb_launch_pass_warp(vw, st), "volume pass");
                cut(p.probes.p, size_t(p.n_probes) * 16);
                if (p.keep_records)
                    ck(cudaMemcpyAsync(p.vraw.p, p.probes.p, size_t(p.n_probes) * 64, cudaMemcpyDeviceToDevice, st),
                       "raw probes");
            }
            ck(lb_volume_fill(p.probes.as<float4>(), p.probes_b.as<float4>(), p.pk_a.as<uint8_t>(), p.pk_b.as<uint8_t>(),
                              p.vsize[0], p.vsize[1], p.vsize[2], 8, st),
               "volume fill");
            const lb::VolumeSettings &v = *h.volume;
            ck(lb_fallback(a, p.probes.as<float4>(), make_float3(v.min[0], v.min[1], v.min[2]), v.step, p.vsize[0],
                           p.vsize[1], p.vsize[2], st),
               "fallback");
        }
        CompositeArgs c{};
        c.owner = p.owner.as<uint32_t>();
        c.known = p.known.as<uint8_t>();
        c.state = p.state.as<uint8_t>();
        c.field = p.field.as<float>();
        c.ao = p.ao.as<float>();
        c.ind = p.ind.as<float4>();
        c.aw = p.aw;
        c.ah = p.ah;
        c.iw = p.iw;
        c.ih = p.ih;
        c.ds = p.ds;
        c.direct_out = p.direct_atlas.as<float2>();
        c.validity = p.validity.as<uint8_t>();
        c.indirect = p.indirect.as<float4>();
        c.has = p.has.as<uint8_t>();
        ck(lb_composite(c, p.indirect_b.as<float4>(), p.has_b.as<uint8_t>(), st), "composite");
        // the file's encodings, from the atlases just written (the file then needs only its compression);
        // BC5 takes whole 4 x 4 blocks (an atlas of another size is left to the host's writer, which refuses it)
        if (p.aw % 4 == 0 && p.ah % 4 == 0) {
            ck(lb_encode_bc5(p.direct_atlas.as<float2>(), p.aw, p.ah, p.enc_bc5.as<uint8_t>(), st), "BC5");
            ck(lb_encode_rgb9e5(p.indirect.as<float4>(), p.iw * p.ih, p.enc_rgb.as<uint32_t>(), st), "RGB9E5");
            if (p.has_volume)
                ck(lb_encode_volume(p.probes.as<float4>(), p.n_probes, p.enc_scale.as<unsigned int>(),
                                    p.enc_vol.as<uint8_t>(), st),
                   "volume bytes");
        }
        finish({});
    } catch (...) {
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        if (cudaStreamIsCapturing(st, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone) {
            cudaGraph_t g = nullptr;
            cudaStreamEndCapture(st, &g);
            if (g) cudaGraphDestroy(g);
        }
        throw;
    }
    p.kernel_nodes = 0;
    for (const lb_plan::Piece &pc : p.pieces) {
        size_t n_nodes = 0;
        ck(cudaGraphGetNodes(pc.graph, nullptr, &n_nodes), "graph nodes");
        std::vector<cudaGraphNode_t> nodes(n_nodes);
        ck(cudaGraphGetNodes(pc.graph, nodes.data(), &n_nodes), "graph nodes");
        for (auto nd : nodes) {
            cudaGraphNodeType t;
            if (cudaGraphNodeGetType(nd, &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) p.kernel_nodes++;
        }
    }
}

template <class T> std::vector<T> down(lb_plan &p, const DBuf &d, size_t n, size_t off = 0) {
    std::vector<T> v(n);
    if (n) {
        ck(cudaMemcpyAsync(v.data(), (const char *)d.p + off * sizeof(T), n * sizeof(T), cudaMemcpyDeviceToHost,
                           p.g->stream),
           "download");
        p.g->d2h += n * sizeof(T);
    }
    return v;
}

lb_plan *create_plan(lb_gpu *g, const uint8_t *scene, size_t len, const lb_bake_options *opts, bool keep_records) {
    if (!g || !scene) {
        lb_set_error("lb_plan_create: bad arguments");
        return nullptr;
    }
    try {
        ck(cudaSetDevice(g->device), "cudaSetDevice");
        lbplan::DBufScope spares(g);  // the plan's device buffers from (and back to) the handle's spares
        auto p = std::make_unique<lb_plan>();
        p->g = g;
        p->scene = lb::Scene::read(scene, len);
        if (opts && opts->cache_dir) p->opt.cache = opts->cache_dir;
        if (opts && opts->log) {
            auto fn = opts->log;
            void *ctx = opts->log_ctx;
            p->opt.log = [fn, ctx](const std::string &s) { fn(ctx, s.c_str()); };
        }
        p->opt.watertight = opts && opts->watertight;
        p->autotune = opts && opts->autotune;
        if (opts && opts->exchange && opts->exchange->world > 1) {
            const lb_exchange *ex = opts->exchange;
            if (!ex->sum || ex->rank < 0 || ex->rank >= ex->world)
                throw std::runtime_error("lb_exchange: bad rank or no sum");
            p->ex = *ex;
            p->rank = ex->rank;
            p->world = ex->world;
        }
        p->reuse = !(opts && opts->trace_every_bounce);
        p->keep_records = keep_records;
        p->group_direct = g->group_direct;
        p->group_gather = g->group_gather;
        p->bvh_direct = p->bvh_gather = p->bvh_volume = g->bvh;
        p->refill_direct = p->refill_gather = g->refill;
        p->near_direct = p->near_gather = g->near;
        p->fetch_direct = p->fetch_gather = g->fetch;
        p->warp_walk = g->warp_walk;
        // untuned shapes: with no register cap set on the handle, the direct pass runs the 4-block cap
        // without the sun rays' shared walk and the gathers the 3-block cap (on map_100m's whole direct pass
        // the 4-block cap takes 219 ms against 225 for the 3-block one; the compiler's budget with the
        // shared walk made the step 345 ms against 325)
        p->occ_direct = g->occ ? g->occ : 4;
        p->occ_gather = g->occ ? g->occ : 3;
        if (!g->occ) p->warp_walk = 0;
        auto t0 = std::chrono::steady_clock::now();
        build(*p);
        double t_build = since(t0);
        t0 = std::chrono::steady_clock::now();
        if (p->autotune) autotune(*p);
        double t_tune = since(t0);
        t0 = std::chrono::steady_clock::now();
        capture(*p);
        double t_capture = since(t0);
        if (p->opt.log) {
            if (p->world > 1)
                p->opt.log("rank " + std::to_string(p->rank) + " of " + std::to_string(p->world) +
                           ": its share of every pass's items, the outputs summed over the ranks after each pass");
            p->opt.log(std::to_string(p->dirty.size()) + " of " + std::to_string(p->P.layout.tiles.size()) +
                       " tiles to bake on the device, " + std::to_string(p->n_cov) + " texels, " +
                       std::to_string(p->n_todo) + " probes");
            p->opt.log("timing: build " + std::to_string(t_build) + " s, autotune " + std::to_string(t_tune) +
                       " s, capture " + std::to_string(t_capture) + " s");
            p->opt.log("timing of the build, cumulative: " + p->build_phases);
        }
        return p.release();
    } catch (const std::exception &e) {
        lb_set_error(e.what());
    }
    return nullptr;
}

}  // namespace

lb_plan *lb_plan_create_recording(lb_gpu *g, const uint8_t *scene, size_t len) {
    lb_bake_options o{};
    return create_plan(g, scene, len, &o, true);
}

extern "C" {

lb_plan *lb_plan_create(lb_gpu *g, const uint8_t *scene, size_t len, const lb_bake_options *opts) {
    return create_plan(g, scene, len, opts, false);
}

int lb_plan_launch(lb_plan *p) {
    if (!p) return LB_EINVAL;
    cudaError_t e = cudaSuccess;
    for (cudaEvent_t &ev : p->ev)
        if (!ev && e == cudaSuccess) e = cudaEventCreate(&ev);
    if (e == cudaSuccess) e = cudaEventRecord(p->ev[0], p->g->stream);
    for (const lb_plan::Piece &pc : p->pieces) {
        if (e == cudaSuccess) e = cudaGraphLaunch(pc.exec, p->g->stream);
        for (const auto &sum : pc.sums) {
            // the piece's outputs are complete before the ranks sum them, in place, on the device
            if (e == cudaSuccess) e = cudaStreamSynchronize(p->g->stream);
            if (e != cudaSuccess) break;
            if (p->ex.sum(p->ex.ctx, sum.first, sum.second, 1) != 0) {
                lb_set_error("lb_plan_launch: the exchange's sum failed");
                return LB_EEXCHANGE;
            }
        }
    }
    if (e == cudaSuccess) e = cudaEventRecord(p->ev[1], p->g->stream);
    if (e != cudaSuccess) return lb_cuda_fail(e, "lb_plan_launch");
    return LB_OK;
}

int lb_plan_rays(lb_plan *p, uint64_t rays[3]) {
    if (!p || !rays) return LB_EINVAL;
    unsigned long long c[12];
    cudaError_t e = cudaMemcpyAsync(c, p->counters.p, sizeof c, cudaMemcpyDeviceToHost, p->g->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(p->g->stream);
    if (e != cudaSuccess) return lb_cuda_fail(e, "lb_plan_rays");
    rays[0] = c[0];
    rays[1] = c[4];
    rays[2] = c[8];
    return LB_OK;
}

int lb_plan_kernels(const lb_plan *p) { return p ? p->kernel_nodes : 0; }

const char *lb_plan_tuning(const lb_plan *p) { return p ? p->tuned.c_str() : ""; }

void lb_plan_free(lb_plan *p) {
    if (p) {
        auto t0 = std::chrono::steady_clock::now();
        cudaStreamSynchronize(p->g->stream);
        auto log = p->opt.log;
        delete p;
        if (log) log("timing: plan freed in " + std::to_string(since(t0)) + " s");
    }
}

}  // extern "C"

const lb::Scene &lb_plan_scene(const lb_plan &p) { return p.scene; }

// The results of the last launch, as a bake (downloads, the cache writes).
lb::Bake lb_plan_collect(lb_plan &p) {
    const lb::SceneHeader &h = p.scene.header;
    auto t0 = std::chrono::steady_clock::now();
    ck(cudaStreamSynchronize(p.g->stream), "bake");
    const double t_wait = since(t0);
    float graph_ms = 0.0f;
    if (p.ev[0] && p.ev[1]) ck(cudaEventElapsedTime(&graph_ms, p.ev[0], p.ev[1]), "graph time");
    lb::Bake out;
    size_t A = size_t(p.aw) * p.ah;
    // the atlases and probes through the handle's pinned staging buffer (kept between bakes)
    const size_t n_ind = size_t(p.iw) * p.ih, n_pr = p.has_volume ? size_t(p.n_probes) * 16 : 0;
    auto up = [](size_t b) { return (b + 255) & ~size_t(255); };
    const size_t o_val = up(A * 8), o_ind = o_val + up(A), o_pr = o_ind + up(n_ind * 16), o_bc5 = o_pr + up(n_pr * 4),
                 o_rgb = o_bc5 + up(A), o_vb = o_rgb + up(n_ind * 4), o_sc = o_vb + up(p.has_volume ? size_t(p.n_probes) * 16 : 0),
                 total = o_sc + 4;
    if (lb_host_stage_reserve(p.g, total) != LB_OK) throw std::runtime_error(lb_last_error());
    char *stage = (char *)p.g->stage;
    auto fetch = [&](size_t off, const DBuf &d, size_t bytes) {
        if (!bytes) return;
        ck(cudaMemcpyAsync(stage + off, d.p, bytes, cudaMemcpyDeviceToHost, p.g->stream), "download");
        p.g->d2h += bytes;
    };
    fetch(0, p.direct_atlas, A * 8);
    fetch(o_val, p.validity, A);
    fetch(o_ind, p.indirect, n_ind * 16);
    if (p.has_volume) fetch(o_pr, p.probes, n_pr * 4);
    fetch(o_bc5, p.enc_bc5, A);
    fetch(o_rgb, p.enc_rgb, n_ind * 4);
    if (p.has_volume) {
        fetch(o_vb, p.enc_vol, size_t(p.n_probes) * 16);
        fetch(o_sc, p.enc_scale, 4);
    }
    uint64_t rays[3];
    if (lb_plan_rays(&p, rays) != LB_OK) throw std::runtime_error(lb_last_error());
    const double t_down = since(t0);
    const float *ind = (const float *)(stage + o_ind), *probes = (const float *)(stage + o_pr);
    // out of the staging buffer by all host threads (tens of MB: one thread's copy is the collection's
    // largest host cost)
    auto copy = [](void *dst, const void *src, size_t bytes) {
        const size_t piece = size_t(1) << 20, n = (bytes + piece - 1) / piece;
#pragma omp parallel for schedule(static) if (n > 4)
        for (long long k = 0; k < (long long)n; k++) {
            const size_t at = size_t(k) * piece;
            std::memcpy((char *)dst + at, (const char *)src + at, std::min(piece, bytes - at));
        }
    };
    out.direct.resize(A);
    copy(out.direct.data(), stage, A * 8);
    out.validity.resize(A);
    copy(out.validity.data(), stage + o_val, A);
    out.indirect.resize(n_ind);
    auto *oi = out.indirect.data();
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < (long long)n_ind; i++) oi[i] = {ind[i * 4], ind[i * 4 + 1], ind[i * 4 + 2]};
    out.iw = p.iw;
    out.ih = p.ih;
    if (p.aw % 4 == 0 && p.ah % 4 == 0) {
        lb::Encoded enc;
        enc.bc5.resize(A);
        copy(enc.bc5.data(), stage + o_bc5, A);
        enc.rgb9e5.resize(n_ind);
        copy(enc.rgb9e5.data(), stage + o_rgb, n_ind * 4);
        if (p.has_volume) {
            enc.volume.assign((const uint8_t *)stage + o_vb, (const uint8_t *)stage + o_vb + size_t(p.n_probes) * 16);
            std::memcpy(&enc.volume_scale, stage + o_sc, 4);
        }
        out.encoded = std::move(enc);
    }
    if (p.has_volume) {
        lb::Volume v;
        v.origin = h.volume->min;
        v.step = h.volume->step;
        v.size = p.vsize;
        v.probes.resize(p.n_probes);
        copy(v.probes.data(), probes, n_pr * 4);
        v.chunks = p.n_chunks;
        v.chunks_baked = p.chunk_keys.size();
        out.volume = std::move(v);
    }
    lb::Cache cache(p.opt.cache);
    if (!p.opt.cache.empty()) {
        // the dirty tiles' light for the cache (bake.rs:360-362), and the probe chunks (volume.rs:81-84)
        std::vector<uint8_t> kn = down<uint8_t>(p, p.known, p.n_dirty_texels), stt = down<uint8_t>(p, p.state, p.n_dirty_texels);
        std::vector<float> fd = down<float>(p, p.field, p.n_dirty_texels), ao = down<float>(p, p.ao, p.n_dirty_texels);
        std::vector<float> dl = down<float>(p, p.dl, size_t(p.n_dirty_texels) * 4),
                           id = down<float>(p, p.ind, size_t(p.n_dirty_texels) * 4);
        ck(cudaStreamSynchronize(p.g->stream), "download");
        // a split bake: every rank holds every tile's light, and writes its share of the tiles and chunks
        auto mine = [&](size_t k, size_t n) { return p.world <= 1 || k * size_t(p.world) / n == size_t(p.rank); };
        for (size_t k = 0; k < p.dirty.size(); k++) {
            if (!mine(k, p.dirty.size())) continue;
            const DTile &t = p.tiles_all[k];
            size_t n = size_t(t.w) * t.h;
            lb::TileLight l;
            l.known.assign(kn.begin() + t.off, kn.begin() + t.off + n);
            l.state.assign(stt.begin() + t.off, stt.begin() + t.off + n);
            l.field.assign(fd.begin() + t.off, fd.begin() + t.off + n);
            l.ao.assign(ao.begin() + t.off, ao.begin() + t.off + n);
            l.direct.resize(n);
            l.indirect.resize(n);
            for (size_t i = 0; i < n; i++) {
                size_t d = (t.off + i) * 4;
                l.direct[i] = {dl[d], dl[d + 1], dl[d + 2]};
                l.indirect[i] = {id[d], id[d + 1], id[d + 2]};
            }
            cache.put("tile", p.hashes[p.dirty[k]], l.pack());
        }
        if (p.has_volume)
            for (size_t c = 0; c < p.chunk_keys.size(); c++) {
                if (!mine(c, p.chunk_keys.size())) continue;
                auto &kv = p.chunk_keys[c];
                std::vector<uint8_t> bytes(kv.second.size() * 64);
                for (size_t i = 0; i < kv.second.size(); i++)
                    std::memcpy(bytes.data() + i * 64, &probes[size_t(kv.second[i]) * 16], 64);
                cache.put("probes", kv.first, bytes);
            }
    }
    out.layout = p.P.layout;
    lb::Stats &s = out.stats;
    s.tiles = p.P.layout.tiles.size();
    s.tiles_baked = p.dirty.size();
    s.texels_baked = p.n_cov;
    s.chunks = p.n_chunks;
    s.chunks_baked = p.chunk_keys.size();
    s.rays_direct = rays[0];
    s.rays_gather = rays[1];
    s.rays_volume = rays[2];
    s.t_layout = p.t_prepare;
    s.t_composite = since(t0);
    if (p.opt.log)
        p.opt.log("timing of the collection, cumulative: device " + std::to_string(t_wait) + " s (graph " +
                  std::to_string(graph_ms * 1e-3) + " s on the device); downloads " +
                  std::to_string(t_down) + " s; results and cache " + std::to_string(s.t_composite) + " s");
    return out;
}
