// The bake as it ships (.lbake): crates/lightbaker/src/output.rs and crates/lightbaker/src/encode.rs.
// `LBAK`, version 1, the JSON header, then 8-aligned chunks: direct (KTX2 BC5, zstd 19), indirect
// (KTX2 RGB9E5, zstd 19), charts, triangleCharts, validity and volume (raw deflate, best).
#include <zlib.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <stdexcept>

#include "bake.h"
#include "cache.h"
#include "encode.h"

namespace lb {

namespace {
std::vector<uint8_t> deflate_raw(const uint8_t *data, size_t len) {
    z_stream z;
    std::memset(&z, 0, sizeof z);
    if (deflateInit2(&z, 9, Z_DEFLATED, -15, 9, Z_DEFAULT_STRATEGY) != Z_OK) throw std::runtime_error("deflate init");
    std::vector<uint8_t> out(deflateBound(&z, uLong(len)) + 16);
    z.next_in = const_cast<Bytef *>(data);
    z.avail_in = uInt(len);
    z.next_out = out.data();
    z.avail_out = uInt(out.size());
    int rc = deflate(&z, Z_FINISH);
    deflateEnd(&z);
    if (rc != Z_STREAM_END) throw std::runtime_error("deflate");
    out.resize(z.total_out);
    return out;
}
template <class T> std::vector<uint8_t> bytes_of(const std::vector<T> &v) {
    const uint8_t *p = (const uint8_t *)v.data();
    return std::vector<uint8_t>(p, p + v.size() * sizeof(T));
}
uint8_t qbyte(float v) { return uint8_t(std::round(std::min(std::max(v, 0.0f), 1.0f) * 255.0f)); }

// output.rs:162-181
std::vector<uint8_t> volume_bytes(const std::vector<std::array<float, 16>> &probes, float scale) {
    const float SQRT3 = 1.7320508f;
    std::vector<uint8_t> out;
    out.reserve(probes.size() * 16);
    for (auto &p : probes) {
        for (int c = 0; c < 3; c++) out.push_back(qbyte(std::sqrt(std::fmax(p[c], 0.0f) / scale)));
        out.push_back(qbyte(p[3]));
        for (int axis = 1; axis < 4; axis++)
            for (int c = 0; c < 3; c++) {
                float r = p[c] > 1e-6f ? p[axis * 4 + c] / (p[c] * SQRT3) : 0.0f;
                out.push_back(qbyte(r * 0.5f + 0.5f));
            }
        out.insert(out.end(), {0, 0, 0});
    }
    return out;
}
Json jf3(const std::array<float, 3> &v) {
    Json a = Json::array();
    for (float x : v) a.arr.push_back(Json::f32(x));
    return a;
}
}  // namespace

// output.rs:95-154
std::vector<uint8_t> write_bake(const Scene &scene, const Bake &bake) {
    const Layout &l = bake.layout;
    size_t w = l.width, h = l.height;
    // the encodings: the device's when it made them (the same bits), else encoded here
    const Encoded *enc = bake.encoded ? &*bake.encoded : nullptr;
    std::vector<uint8_t> blocks;
    if (enc) {
        blocks = enc->bc5;
    } else {
        std::vector<uint8_t> rg(w * h * 2);
        for (size_t i = 0; i < w * h; i++) {
            rg[i * 2] = qbyte(bake.direct[i][0]);
            rg[i * 2 + 1] = qbyte(bake.direct[i][1]);
        }
        blocks = bc5(rg.data(), w, h);
    }
    std::vector<uint32_t> packed;
    if (enc) {
        packed = enc->rgb9e5;
    } else {
        packed.resize(bake.indirect.size());
        for (size_t i = 0; i < packed.size(); i++) packed[i] = rgb9e5(bake.indirect[i].data());
    }
    std::vector<float> charts;
    std::vector<uint32_t> ct = l.chart_tile();
    for (size_t c = 0; c < l.charts.size(); c++)
        for (auto &r : l.charts[c].affine(l.tiles[ct[c]], l.density, l.padding)) charts.insert(charts.end(), r.begin(), r.end());
    std::vector<uint32_t> tri;
    for (auto &m : l.tri_chart) tri.insert(tri.end(), m.begin(), m.end());
    std::vector<std::pair<std::string, std::vector<uint8_t>>> chunks;
    chunks.emplace_back("direct", ktx2(FORMAT_BC5, uint32_t(w), uint32_t(h), blocks));
    chunks.emplace_back("indirect", ktx2(FORMAT_RGB9E5, bake.iw, bake.ih, bytes_of(packed)));
    auto cb = bytes_of(charts);
    chunks.emplace_back("charts", deflate_raw(cb.data(), cb.size()));
    auto tb = bytes_of(tri);
    chunks.emplace_back("triangleCharts", deflate_raw(tb.data(), tb.size()));
    chunks.emplace_back("validity", deflate_raw(bake.validity.data(), bake.validity.size()));
    float scale = 1.0f;
    if (bake.volume && enc) {
        scale = enc->volume_scale;
        chunks.emplace_back("volume", deflate_raw(enc->volume.data(), enc->volume.size()));
    } else if (bake.volume) {
        scale = 1e-6f;
        for (auto &p : bake.volume->probes)
            for (int c = 0; c < 3; c++) scale = std::fmax(scale, p[c]);
        auto vb = volume_bytes(bake.volume->probes, scale);
        chunks.emplace_back("volume", deflate_raw(vb.data(), vb.size()));
    }
    const SceneHeader &sh = scene.header;
    Json head = Json::object();
    head.set("baker", Json::string("lightbaker 0.1.0"));
    head.set("scene", Json::string(to_hex(scene.hash.data(), 32)));
    head.set("user", sh.user);
    Json atlas = Json::object();
    atlas.set("width", Json::u32(l.width));
    atlas.set("height", Json::u32(l.height));
    atlas.set("texelsPerMeter", Json::f32(l.density));
    atlas.set("sdfRadius", Json::f32(sh.bake.sdf_radius));
    atlas.set("indirectWidth", Json::u32(bake.iw));
    atlas.set("indirectHeight", Json::u32(bake.ih));
    atlas.set("charts", Json::u32(uint32_t(l.charts.size())));
    head.set("atlas", atlas);
    const float PI = 3.14159274f;
    std::array<float, 3> sky;
    for (int c = 0; c < 3; c++) sky[c] = PI * (sh.sky.horizon[c] / 3.0f + 2.0f * sh.sky.zenith[c] / 3.0f);
    head.set("skyIrradiance", jf3(sky));
    Json meshes = Json::array();
    for (auto &m : sh.meshes) {
        Json o = Json::object();
        o.set("name", Json::string(m.name));
        o.set("triangles", Json::u32(m.triangles));
        meshes.arr.push_back(o);
    }
    head.set("meshes", meshes);
    if (bake.volume) {
        Json v = Json::object();
        v.set("origin", jf3(bake.volume->origin));
        v.set("step", Json::f32(bake.volume->step));
        Json sz = Json::array();
        for (uint32_t s : bake.volume->size) sz.arr.push_back(Json::u32(s));
        v.set("size", sz);
        v.set("scale", Json::f32(scale));
        head.set("volume", v);
    } else {
        head.set("volume", Json());
    }
    Json cj = Json::array();
    uint64_t at = 0;
    std::vector<uint64_t> offs;
    for (auto &c : chunks) {
        Json o = Json::object();
        o.set("name", Json::string(c.first));
        o.set("offset", Json::i64((long long)at));
        o.set("length", Json::i64((long long)c.second.size()));
        cj.arr.push_back(o);
        offs.push_back(at);
        at = (at + c.second.size() + 7) / 8 * 8;
    }
    head.set("chunks", cj);
    Json st = Json::object();
    st.set("tiles", Json::i64((long long)bake.stats.tiles));
    st.set("tilesBaked", Json::i64((long long)bake.stats.tiles_baked));
    st.set("texelsBaked", Json::i64((long long)bake.stats.texels_baked));
    st.set("chunks", Json::i64((long long)bake.stats.chunks));
    st.set("chunksBaked", Json::i64((long long)bake.stats.chunks_baked));
    Json sec;
    sec.kind = Json::Num;
    sec.num = bake.stats.seconds;
    char b[64];
    snprintf(b, sizeof b, "%.17g", bake.stats.seconds);
    sec.str = b;
    if (sec.str.find_first_of(".e") == std::string::npos) sec.str += ".0";
    st.set("seconds", sec);
    head.set("stats", st);
    std::string hs = head.dump();
    std::vector<uint8_t> out{'L', 'B', 'A', 'K'};
    uint32_t ver = 1, hl = uint32_t(hs.size());
    out.insert(out.end(), (uint8_t *)&ver, (uint8_t *)&ver + 4);
    out.insert(out.end(), (uint8_t *)&hl, (uint8_t *)&hl + 4);
    out.insert(out.end(), hs.begin(), hs.end());
    out.resize((out.size() + 7) / 8 * 8, 0);
    size_t base = out.size();
    for (size_t k = 0; k < chunks.size(); k++) {
        out.resize(base + offs[k], 0);
        out.insert(out.end(), chunks[k].second.begin(), chunks[k].second.end());
    }
    return out;
}

}  // namespace lb
