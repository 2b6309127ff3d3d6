// The C ABI's host side: prepared scenes, the bake entry point and the file writers.
#include <chrono>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <stdexcept>

#include "../lb_runtime.h"
#include "bake.h"
#include "blake3.h"
#include "bvh8.h"
#include "encode.h"
#include "handles.h"
#include "raster.h"

struct lb_prepared {
    lb::Scene scene;
    lb::Prepared prep;
};


namespace {

// The passes on the CUDA runtime (gpu/mod.rs:129-196 replaced by lb_scene_upload / lb_run).
class GpuTracer : public lb::Tracer {
  public:
    explicit GpuTracer(lb_gpu *g) : g_(g) {}
    ~GpuTracer() override { lb_scene_free(s_); }
    void scene(const lb::Bvh &bvh, const std::vector<float> &mats, const std::vector<float> &charts) override {
        lb_scene_free(s_);
        s_ = lb_scene_upload(g_, bvh.nodes.data(), bvh.nodes.size(), bvh.tris.data(), bvh.tris.size(), mats.data(),
                             mats.size() / 4, charts.data(), charts.size() / 8);
        if (!s_) throw std::runtime_error(lb_last_error());
    }
    void watertight(const lb::Bvh &bvh) override {
        if (!s_ || lb_scene_set_vertices(g_, s_, bvh.verts.data(), bvh.tris.size()) != LB_OK)
            throw std::runtime_error(lb_last_error());
    }
    uint64_t run(int pass, const lb_params &params, const std::vector<lb_texel> &items, const std::vector<float> &light,
                 std::vector<float> &out) override {
        size_t width = pass == LB_PASS_VOLUME ? 4 : 1;
        out.assign(items.size() * width * 4, 0.0f);
        if (items.empty()) return 0;
        int rc = lb_run(g_, s_, pass, &params, items.data(), items.size(), light.empty() ? nullptr : light.data(),
                        light.size() / 4, out.data());
        if (rc != LB_OK) throw std::runtime_error(std::string("GPU: ") + lb_last_error());
        lb_counters c;
        lb_get_counters(g_, &c);
        return c.rays;
    }

  private:
    lb_gpu *g_;
    lb_scene *s_ = nullptr;
};

// The passes on a caller's runner.
class CallbackTracer : public lb::Tracer {
  public:
    explicit CallbackTracer(const lb_tracer &t) : t_(t) {}
    void scene(const lb::Bvh &bvh, const std::vector<float> &mats, const std::vector<float> &charts) override {
        if (t_.scene(t_.ctx, bvh.nodes.data(), bvh.nodes.size(), bvh.tris.data(), bvh.tris.size(), mats.data(),
                     mats.size() / 4, charts.data(), charts.size() / 8) != 0)
            throw std::runtime_error("tracer: scene upload failed");
    }
    uint64_t run(int pass, const lb_params &params, const std::vector<lb_texel> &items, const std::vector<float> &light,
                 std::vector<float> &out) override {
        size_t width = pass == LB_PASS_VOLUME ? 4 : 1;
        out.assign(items.size() * width * 4, 0.0f);
        if (items.empty()) return 0;
        uint64_t rays = 0;
        if (t_.run(t_.ctx, pass, &params, items.data(), items.size(), light.empty() ? nullptr : light.data(),
                   light.size() / 4, out.data(), &rays) != 0)
            throw std::runtime_error("tracer: pass failed");
        return rays;
    }

  private:
    lb_tracer t_;
};

lb::Options options(const lb_bake_options *o) {
    lb::Options opt;
    if (o && o->cache_dir) opt.cache = o->cache_dir;
    if (o && o->log) {
        auto fn = o->log;
        void *ctx = o->log_ctx;
        opt.log = [fn, ctx](const std::string &s) { fn(ctx, s.c_str()); };
    }
    if (o) opt.watertight = o->watertight != 0;
    if (o && o->exchange && o->exchange->world > 1) {
        const lb_exchange *ex = o->exchange;
        if (!ex->sum || ex->rank < 0 || ex->rank >= ex->world) throw std::runtime_error("lb_exchange: bad rank or no sum");
        opt.rank = ex->rank;
        opt.world = ex->world;
        opt.sum = [ex](void *data, size_t words, bool device) {
            if (ex->sum(ex->ctx, data, words, device ? 1 : 0) != 0) throw std::runtime_error("lb_exchange: sum failed");
        };
    }
    return opt;
}

template <class F> auto guard(F f, decltype(f()) fail) -> decltype(f()) {
    try {
        return f();
    } catch (const std::exception &e) {
        lb_set_error(e.what());
    } catch (...) {
        lb_set_error("unknown error");
    }
    return fail;
}

}  // namespace

extern "C" {

lb_prepared *lb_prepare(const uint8_t *scene, size_t len) {
    return guard(
        [&]() -> lb_prepared * {
            if (!scene) throw std::runtime_error("lb_prepare: no scene");
            auto p = std::make_unique<lb_prepared>();
            p->scene = lb::Scene::read(scene, len);
            p->prep = lb::prepare(p->scene);
            return p.release();
        },
        nullptr);
}

void lb_prepared_free(lb_prepared *p) { delete p; }

int lb_prepared_get_info(const lb_prepared *p, lb_prepared_info *o) {
    if (!p || !o) return LB_EINVAL;
    std::memset(o, 0, sizeof *o);
    const lb::Prepared &P = p->prep;
    o->n_nodes = P.bvh.nodes.size();
    o->n_tris = P.bvh.tris.size();
    o->n_materials = P.materials.size() / 4;
    o->n_charts = P.affines.size() / 8;
    o->n_tiles = P.layout.tiles.size();
    o->n_triangles = p->scene.triangle_count();
    o->atlas_width = P.layout.width;
    o->atlas_height = P.layout.height;
    o->indirect_downscale = p->scene.header.lightmap.indirect_downscale;
    o->padding = P.layout.padding;
    o->gi_bounces = p->scene.header.bake.gi_bounces;
    o->has_volume = p->scene.header.volume.has_value();
    o->params = P.params;
    return LB_OK;
}

int lb_prepared_get_bvh(const lb_prepared *p, lb_node *nodes, lb_tri *tris) {
    if (!p || !nodes || !tris) return LB_EINVAL;
    std::memcpy(nodes, p->prep.bvh.nodes.data(), p->prep.bvh.nodes.size() * sizeof(lb_node));
    std::memcpy(tris, p->prep.bvh.tris.data(), p->prep.bvh.tris.size() * sizeof(lb_tri));
    return LB_OK;
}

int lb_prepared_get_vertices(const lb_prepared *p, float *verts) {
    if (!p || !verts) return LB_EINVAL;
    std::memcpy(verts, p->prep.bvh.verts.data(), p->prep.bvh.verts.size() * sizeof(float));
    return LB_OK;
}

int lb_prepared_get_materials(const lb_prepared *p, float *m) {
    if (!p || !m) return LB_EINVAL;
    std::memcpy(m, p->prep.materials.data(), p->prep.materials.size() * 4);
    return LB_OK;
}

int lb_prepared_get_charts(const lb_prepared *p, float *c) {
    if (!p || !c) return LB_EINVAL;
    std::memcpy(c, p->prep.affines.data(), p->prep.affines.size() * 4);
    return LB_OK;
}

int lb_prepared_get_tile(const lb_prepared *p, size_t t, uint32_t rect[4], int32_t key[2]) {
    if (!p || t >= p->prep.layout.tiles.size()) return LB_EINVAL;
    const lb::Tile &T = p->prep.layout.tiles[t];
    if (rect) {
        rect[0] = T.x;
        rect[1] = T.y;
        rect[2] = T.w;
        rect[3] = T.h;
    }
    if (key) {
        key[0] = T.key.first;
        key[1] = T.key.second;
    }
    return LB_OK;
}

size_t lb_prepared_get_tile_charts(const lb_prepared *p, size_t t, uint32_t *charts, size_t cap) {
    if (!p || t >= p->prep.layout.tiles.size()) return 0;
    const std::vector<uint32_t> &c = p->prep.layout.tiles[t].charts;
    if (charts) std::memcpy(charts, c.data(), std::min(cap, c.size()) * 4);
    return c.size();
}

size_t lb_prepared_get_chart(const lb_prepared *p, size_t c, lb_chart_frame *frame, uint32_t *tris, size_t cap) {
    if (!p || c >= p->prep.layout.charts.size()) return 0;
    const lb::Chart &C = p->prep.layout.charts[c];
    if (frame) {
        frame->mesh = C.mesh;
        frame->turned = C.turned ? 1u : 0u;
        frame->x = C.x;
        frame->y = C.y;
        frame->w = C.w;
        frame->h = C.h;
        const lb::Vec3 *axes[3] = {&C.normal, &C.u, &C.v};
        float *dst[3] = {frame->normal, frame->u, frame->v};
        for (int a = 0; a < 3; a++) {
            dst[a][0] = axes[a]->x;
            dst[a][1] = axes[a]->y;
            dst[a][2] = axes[a]->z;
        }
        frame->min[0] = C.min.x;
        frame->min[1] = C.min.y;
        frame->max[0] = C.max.x;
        frame->max[1] = C.max.y;
        frame->tile[0] = C.tile.first;
        frame->tile[1] = C.tile.second;
    }
    if (tris) std::memcpy(tris, C.tris.data(), std::min(cap, C.tris.size()) * 4);
    return C.tris.size();
}

int lb_prepared_rasterize(const lb_prepared *p, size_t t, lb_texel *out) {
    if (!p || !out || t >= p->prep.layout.tiles.size()) return LB_EINVAL;
    std::vector<lb_texel> v = lb::rasterize(p->scene, p->prep.layout, p->prep.layout.tiles[t]);
    std::memcpy(out, v.data(), v.size() * sizeof(lb_texel));
    return LB_OK;
}

lb_bake *lb_bake_run(lb_gpu *gpu, const uint8_t *scene, size_t len, const lb_bake_options *opts) {
    return guard(
        [&]() -> lb_bake * {
            if (!gpu || !scene) throw std::runtime_error("lb_bake_run: bad arguments");
            auto b = std::make_unique<lb_bake>();
            b->scene = lb::Scene::read(scene, len);
            GpuTracer tracer(gpu);
            b->bake = lb::bake(b->scene, tracer, options(opts));
            return b.release();
        },
        nullptr);
}

lb_bake *lb_bake_run_with(const lb_tracer *t, const uint8_t *scene, size_t len, const lb_bake_options *opts) {
    return guard(
        [&]() -> lb_bake * {
            if (!t || !t->scene || !t->run || !scene) throw std::runtime_error("lb_bake_run_with: bad arguments");
            auto b = std::make_unique<lb_bake>();
            b->scene = lb::Scene::read(scene, len);
            CallbackTracer tracer(*t);
            b->bake = lb::bake(b->scene, tracer, options(opts));
            return b.release();
        },
        nullptr);
}

void lb_bake_free(lb_bake *b) { delete b; }

lb_bake *lb_plan_result(lb_plan *p) {
    return guard(
        [&]() -> lb_bake * {
            if (!p) throw std::runtime_error("lb_plan_result: no plan");
            auto b = std::make_unique<lb_bake>();
            b->scene = lb_plan_scene(*p);
            b->bake = lb_plan_collect(*p);
            return b.release();
        },
        nullptr);
}

lb_bake *lb_bake_device(lb_gpu *gpu, const uint8_t *scene, size_t len, const lb_bake_options *opts) {
    auto t0 = std::chrono::steady_clock::now();
    lb_plan *p = lb_plan_create(gpu, scene, len, opts);
    if (!p) return nullptr;
    lb_bake *b = nullptr;
    if (lb_plan_launch(p) == LB_OK) b = lb_plan_result(p);
    lb_plan_free(p);
    if (b) b->bake.stats.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return b;
}

int lb_bake_get_info(const lb_bake *b, lb_bake_info *o) {
    if (!b || !o) return LB_EINVAL;
    std::memset(o, 0, sizeof *o);
    const lb::Bake &k = b->bake;
    o->width = k.layout.width;
    o->height = k.layout.height;
    o->indirect_width = k.iw;
    o->indirect_height = k.ih;
    if (k.volume) {
        o->has_volume = 1;
        for (int a = 0; a < 3; a++) {
            o->volume_size[a] = k.volume->size[a];
            o->volume_origin[a] = k.volume->origin[a];
        }
        o->volume_step = k.volume->step;
    }
    const lb::Stats &s = k.stats;
    o->tiles = s.tiles;
    o->tiles_baked = s.tiles_baked;
    o->texels_baked = s.texels_baked;
    o->chunks = s.chunks;
    o->chunks_baked = s.chunks_baked;
    o->seconds = s.seconds;
    o->rays_direct = s.rays_direct;
    o->rays_gather = s.rays_gather;
    o->rays_volume = s.rays_volume;
    o->t_layout = s.t_layout;
    o->t_direct = s.t_direct;
    o->t_bounces = s.t_bounces;
    o->t_volume = s.t_volume;
    o->t_composite = s.t_composite;
    o->n_charts = k.layout.charts.size();
    o->n_triangles = b->scene.triangle_count();
    return LB_OK;
}

int lb_bake_get_charts(const lb_bake *b, float *out) {
    if (!b || !out) return LB_EINVAL;
    const lb::Layout &l = b->bake.layout;
    std::vector<uint32_t> ct = l.chart_tile();
    for (size_t c = 0; c < l.charts.size(); c++) {
        auto a = l.charts[c].affine(l.tiles[ct[c]], l.density, l.padding);
        std::memcpy(out + c * 8, a[0].data(), 16);
        std::memcpy(out + c * 8 + 4, a[1].data(), 16);
    }
    return LB_OK;
}

int lb_bake_get_tri_charts(const lb_bake *b, uint32_t *out) {
    if (!b || !out) return LB_EINVAL;
    size_t k = 0;
    for (auto &m : b->bake.layout.tri_chart)
        for (uint32_t c : m) out[k++] = c;
    return LB_OK;
}

int lb_bake_get_direct(const lb_bake *b, float *out) {
    if (!b || !out) return LB_EINVAL;
    std::memcpy(out, b->bake.direct.data(), b->bake.direct.size() * 8);
    return LB_OK;
}

int lb_bake_get_indirect(const lb_bake *b, float *out) {
    if (!b || !out) return LB_EINVAL;
    std::memcpy(out, b->bake.indirect.data(), b->bake.indirect.size() * 12);
    return LB_OK;
}

int lb_bake_get_validity(const lb_bake *b, uint8_t *out) {
    if (!b || !out) return LB_EINVAL;
    std::memcpy(out, b->bake.validity.data(), b->bake.validity.size());
    return LB_OK;
}

int lb_bake_get_volume(const lb_bake *b, float *out) {
    if (!b || !out || !b->bake.volume) return LB_EINVAL;
    std::memcpy(out, b->bake.volume->probes.data(), b->bake.volume->probes.size() * 64);
    return LB_OK;
}

int lb_bake_device_encoded(const lb_bake *b) { return b && b->bake.encoded ? 1 : 0; }

int lb_bake_write(const lb_bake *b, uint8_t **out, size_t *len) {
    if (!b || !out || !len) return LB_EINVAL;
    return guard(
        [&]() -> int {
            std::vector<uint8_t> v = lb::write_bake(b->scene, b->bake);
            *out = (uint8_t *)malloc(v.size() ? v.size() : 1);
            if (!*out) throw std::runtime_error("out of host memory");
            std::memcpy(*out, v.data(), v.size());
            *len = v.size();
            return LB_OK;
        },
        LB_EIO);
}

void lb_free(void *p) { free(p); }

int lb_scene_encode(const char *header_json, const float *const *positions, const size_t *n_floats, size_t n_meshes,
                    uint8_t **out, size_t *len) {
    if (!header_json || !out || !len || (n_meshes && (!positions || !n_floats))) return LB_EINVAL;
    return guard(
        [&]() -> int {
            // the header as given, validated by reading the file back
            std::string head = header_json;
            std::vector<uint8_t> v{'L', 'B', 'S', 'C', 1, 0, 0, 0};
            uint32_t hl = uint32_t(head.size());
            v.insert(v.end(), (uint8_t *)&hl, (uint8_t *)&hl + 4);
            v.insert(v.end(), head.begin(), head.end());
            for (size_t m = 0; m < n_meshes; m++) {
                v.resize((v.size() + 3) & ~size_t(3), 0);
                const uint8_t *p = (const uint8_t *)positions[m];
                v.insert(v.end(), p, p + n_floats[m] * 4);
            }
            v.resize((v.size() + 3) & ~size_t(3), 0);
            lb::Scene::read(v.data(), v.size());
            *out = (uint8_t *)malloc(v.size());
            if (!*out) throw std::runtime_error("out of host memory");
            std::memcpy(*out, v.data(), v.size());
            *len = v.size();
            return LB_OK;
        },
        LB_EIO);
}

int lb_bvh8_check(const lb_node *nodes, size_t n_nodes, const lb_tri *tris, size_t n_tris, uint64_t *n_nodes8,
                  uint64_t *depth) {
    if (!nodes || !n_nodes || (n_tris && !tris)) return LB_EINVAL;
    return guard(
        [&]() -> int {
            lb::Bvh8 b = lb::Bvh8::collapse(nodes, n_nodes, tris, n_tris);
            size_t d = 0;
            // the reference's empty scene has one dummy triangle no leaf holds
            bool empty = nodes[0].count == 0 && n_nodes == 1;
            std::string err = lb::bvh8_check(b, empty ? 0 : n_tris, d);
            if (n_nodes8) *n_nodes8 = b.n_nodes();
            if (depth) *depth = d;
            if (!err.empty()) throw std::runtime_error("bvh8: " + err);
            return LB_OK;
        },
        LB_EINVAL);
}

int lb_bvh8_collapse(const lb_node *nodes, size_t n_nodes, const lb_tri *tris, size_t n_tris, uint32_t *nodes8,
                     lb_tri *tris8, uint64_t *n_nodes8, uint64_t *n_tris8) {
    if (!nodes || !n_nodes || !tris) return LB_EINVAL;
    return guard(
        [&]() -> int {
            lb::Bvh8 b = lb::Bvh8::collapse(nodes, n_nodes, tris, n_tris);
            if (n_nodes8) *n_nodes8 = b.n_nodes();
            if (n_tris8) *n_tris8 = b.tris.size();
            if (nodes8) std::memcpy(nodes8, b.nodes.data(), b.nodes.size() * 4);
            if (tris8) std::memcpy(tris8, b.tris.data(), b.tris.size() * sizeof(lb_tri));
            return LB_OK;
        },
        LB_EINVAL);
}

void lb_blake3(const uint8_t *data, size_t len, uint8_t out[32]) { lb::blake3_hash(data, len, out); }
uint32_t lb_rgb9e5(const float c[3]) { return lb::rgb9e5(c); }
void lb_rgb9e5_decode(uint32_t p, float out[3]) { lb::rgb9e5_decode(p, out); }
void lb_bc4_block(const uint8_t v[16], uint8_t out[8]) {
    auto b = lb::bc4_block(v);
    std::memcpy(out, b.data(), 8);
}

}  // extern "C"
