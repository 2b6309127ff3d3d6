#include "scene.h"

#include <cmath>
#include <cstring>
#include <set>
#include <stdexcept>

#include "blake3.h"

namespace lb {

namespace {
[[noreturn]] void bad(const std::string &m) { throw std::runtime_error(m); }

// serde's deny_unknown_fields (scene.rs:26 and every settings struct)
void only(const Json &j, const char *what, std::initializer_list<const char *> names) {
    if (j.kind != Json::Obj) bad(std::string("scene header: ") + what + " must be an object");
    std::set<std::string> ok(names.begin(), names.end());
    for (auto &kv : j.obj)
        if (!ok.count(kv.first)) bad(std::string("scene header: unknown field `") + kv.first + "` in " + what);
}
std::array<float, 3> f3(const Json &j) {
    if (j.kind != Json::Arr || j.arr.size() != 3) bad("scene header: expected three numbers");
    return {j.arr[0].as_f32(), j.arr[1].as_f32(), j.arr[2].as_f32()};
}
Json jf3(const std::array<float, 3> &v) {
    Json a = Json::array();
    for (float x : v) a.arr.push_back(Json::f32(x));
    return a;
}
uint32_t rd32(const uint8_t *p) {
    uint32_t v;
    std::memcpy(&v, p, 4);
    return v;
}
size_t align4(size_t n) { return (n + 3) & ~size_t(3); }
}  // namespace

size_t Scene::triangle_count() const {
    size_t n = 0;
    for (auto &p : positions) n += p.size() / 3;
    return n;
}

// scene.rs:140-161
Scene Scene::read(const uint8_t *bytes, size_t len) {
    if (len < 12 || std::memcmp(bytes, "LBSC", 4) != 0) bad("not a lightbaker scene");
    uint32_t version = rd32(bytes + 4);
    if (version != 1) bad("scene format " + std::to_string(version) + ", this baker reads 1");
    size_t hl = rd32(bytes + 8);
    if (12 + hl > len) bad("scene header cut short");
    Json j = Json::parse(std::string((const char *)bytes + 12, hl));
    only(j, "the header", {"sun", "sky", "materials", "meshes", "lightmap", "bake", "volume", "user"});
    Scene s;
    SceneHeader &h = s.header;
    const Json &sun = j.at("sun");
    only(sun, "sun", {"direction", "radiusDeg", "irradiance"});
    h.sun = Sun{f3(sun.at("direction")), sun.at("radiusDeg").as_f32(), f3(sun.at("irradiance"))};
    const Json &sky = j.at("sky");
    only(sky, "sky", {"zenith", "horizon", "ground"});
    h.sky = Sky{f3(sky.at("zenith")), f3(sky.at("horizon")), f3(sky.at("ground"))};
    const Json &mats = j.at("materials");
    if (mats.kind != Json::Arr) bad("scene header: materials must be an array");
    for (auto &m : mats.arr) {
        only(m, "a material", {"name", "albedo", "receives", "casts", "opacity"});
        Material mt;
        mt.name = m.at("name").as_str();
        mt.albedo = f3(m.at("albedo"));
        mt.receives = m.at("receives").as_bool();
        mt.casts = m.at("casts").as_bool();
        mt.opacity = m.has("opacity") ? m.at("opacity").as_f32() : 1.0f;  // scene.rs:72-79
        h.materials.push_back(mt);
    }
    const Json &meshes = j.at("meshes");
    if (meshes.kind != Json::Arr) bad("scene header: meshes must be an array");
    for (auto &m : meshes.arr) {
        only(m, "a mesh", {"name", "material", "triangles"});
        h.meshes.push_back(MeshInfo{m.at("name").as_str(), m.at("material").as_u32(), m.at("triangles").as_u32()});
    }
    const Json &lm = j.at("lightmap");
    only(lm, "lightmap", {"texelsPerMeter", "tileSize", "chartAngleDeg", "padding", "atlasWidth", "indirectDownscale"});
    h.lightmap = LightmapSettings{lm.at("texelsPerMeter").as_f32(), lm.at("tileSize").as_f32(),
                                  lm.at("chartAngleDeg").as_f32(), lm.at("padding").as_u32(),
                                  lm.at("atlasWidth").as_u32(), lm.at("indirectDownscale").as_u32()};
    const Json &b = j.at("bake");
    only(b, "bake", {"sunSamples", "aoRays", "aoReach", "aoStrength", "aoFloor", "aoContrast", "sdfRadius", "giRays",
                     "giBounces", "giReach", "insideShare", "giFilter"});
    h.bake = BakeSettings{b.at("sunSamples").as_u32(), b.at("aoRays").as_u32(),    b.at("aoReach").as_f32(),
                          b.at("aoStrength").as_f32(), b.at("aoFloor").as_f32(),   b.at("aoContrast").as_f32(),
                          b.at("sdfRadius").as_f32(),  b.at("giRays").as_u32(),    b.at("giBounces").as_u32(),
                          b.at("giReach").as_f32(),    b.at("insideShare").as_f32(), b.at("giFilter").as_u32()};
    if (const Json *v = j.get("volume"); v && v->kind != Json::Null) {
        only(*v, "volume", {"min", "max", "step", "rays"});
        h.volume = VolumeSettings{f3(v->at("min")), f3(v->at("max")), v->at("step").as_f32(), v->at("rays").as_u32()};
    }
    if (const Json *u = j.get("user")) h.user = *u;
    size_t at = align4(12 + hl);
    for (auto &m : h.meshes) {
        if (m.material >= h.materials.size())
            bad("mesh " + m.name + ": no material " + std::to_string(m.material));
        size_t n = size_t(m.triangles) * 9 * 4;
        if (at + n > len) bad("mesh " + m.name + ": positions cut short");
        std::vector<Vec3> p(size_t(m.triangles) * 3);
        for (size_t k = 0; k < p.size(); k++) {
            float v[3];
            std::memcpy(v, bytes + at + k * 12, 12);
            p[k] = Vec3(v[0], v[1], v[2]);
        }
        s.positions.push_back(std::move(p));
        at = align4(at + n);
    }
    if (at != len) bad("scene: " + std::to_string(len - at) + " bytes after the last mesh");
    // scene.rs:188-201
    const LightmapSettings &l = h.lightmap;
    if (!(l.texels_per_meter > 0.0f && l.tile_size > 0.0f)) bad("lightmap: texelsPerMeter and tileSize must be positive");
    if (!(l.atlas_width >= 64 && l.atlas_width % 4 == 0)) bad("lightmap: atlasWidth must be a multiple of 4, at least 64");
    if (!(l.indirect_downscale == 1 || l.indirect_downscale == 2 || l.indirect_downscale == 4))
        bad("lightmap: indirectDownscale 1, 2 or 4 (the tiles' grid)");
    uint32_t g = uint32_t(std::sqrt(float(h.bake.sun_samples)));
    if (!(g * g == h.bake.sun_samples && g >= 1)) bad("bake: sunSamples must be a square number");
    if (!(h.bake.ao_rays >= 1 && h.bake.gi_rays >= 1)) bad("bake: aoRays and giRays at least one");
    if (h.volume) {
        auto &v = *h.volume;
        if (!(v.step > 0.0f && v.max[0] >= v.min[0] && v.max[1] >= v.min[1] && v.max[2] >= v.min[2]))
            bad("volume: bad bounds or step");
    }
    blake3_hash(bytes, len, s.hash.data());
    return s;
}

// scene.rs:164-181
std::vector<uint8_t> Scene::write(const SceneHeader &h, const std::vector<std::vector<Vec3>> &positions) {
    if (h.meshes.size() != positions.size()) bad("one positions array a mesh");
    std::string head = to_json(h).dump();
    std::vector<uint8_t> out;
    out.insert(out.end(), {'L', 'B', 'S', 'C'});
    auto put32 = [&](uint32_t v) {
        uint8_t b[4];
        std::memcpy(b, &v, 4);
        out.insert(out.end(), b, b + 4);
    };
    put32(1);
    put32(uint32_t(head.size()));
    out.insert(out.end(), head.begin(), head.end());
    for (size_t m = 0; m < positions.size(); m++) {
        if (positions[m].size() != size_t(h.meshes[m].triangles) * 3)
            bad("mesh " + h.meshes[m].name + ": wrong vertex count");
        out.resize(align4(out.size()), 0);
        for (auto &v : positions[m]) {
            float f[3] = {v.x, v.y, v.z};
            const uint8_t *b = (const uint8_t *)f;
            out.insert(out.end(), b, b + 12);
        }
    }
    out.resize(align4(out.size()), 0);
    return out;
}

Json to_json(const Sun &s) {
    Json j = Json::object();
    j.set("direction", jf3(s.direction));
    j.set("radiusDeg", Json::f32(s.radius_deg));
    j.set("irradiance", jf3(s.irradiance));
    return j;
}
Json to_json(const Sky &s) {
    Json j = Json::object();
    j.set("zenith", jf3(s.zenith));
    j.set("horizon", jf3(s.horizon));
    j.set("ground", jf3(s.ground));
    return j;
}
Json to_json(const std::vector<Material> &ms) {
    Json a = Json::array();
    for (auto &m : ms) {
        Json j = Json::object();
        j.set("name", Json::string(m.name));
        j.set("albedo", jf3(m.albedo));
        j.set("receives", Json::boolean(m.receives));
        j.set("casts", Json::boolean(m.casts));
        j.set("opacity", Json::f32(m.opacity));
        a.arr.push_back(j);
    }
    return a;
}
Json to_json(const LightmapSettings &l) {
    Json j = Json::object();
    j.set("texelsPerMeter", Json::f32(l.texels_per_meter));
    j.set("tileSize", Json::f32(l.tile_size));
    j.set("chartAngleDeg", Json::f32(l.chart_angle_deg));
    j.set("padding", Json::u32(l.padding));
    j.set("atlasWidth", Json::u32(l.atlas_width));
    j.set("indirectDownscale", Json::u32(l.indirect_downscale));
    return j;
}
Json to_json(const BakeSettings &b) {
    Json j = Json::object();
    j.set("sunSamples", Json::u32(b.sun_samples));
    j.set("aoRays", Json::u32(b.ao_rays));
    j.set("aoReach", Json::f32(b.ao_reach));
    j.set("aoStrength", Json::f32(b.ao_strength));
    j.set("aoFloor", Json::f32(b.ao_floor));
    j.set("aoContrast", Json::f32(b.ao_contrast));
    j.set("sdfRadius", Json::f32(b.sdf_radius));
    j.set("giRays", Json::u32(b.gi_rays));
    j.set("giBounces", Json::u32(b.gi_bounces));
    j.set("giReach", Json::f32(b.gi_reach));
    j.set("insideShare", Json::f32(b.inside_share));
    j.set("giFilter", Json::u32(b.gi_filter));
    return j;
}
Json to_json(const VolumeSettings &v) {
    Json j = Json::object();
    j.set("min", jf3(v.min));
    j.set("max", jf3(v.max));
    j.set("step", Json::f32(v.step));
    j.set("rays", Json::u32(v.rays));
    return j;
}
Json to_json(const SceneHeader &h) {
    Json j = Json::object();
    j.set("sun", to_json(h.sun));
    j.set("sky", to_json(h.sky));
    j.set("materials", to_json(h.materials));
    Json ms = Json::array();
    for (auto &m : h.meshes) {
        Json o = Json::object();
        o.set("name", Json::string(m.name));
        o.set("material", Json::u32(m.material));
        o.set("triangles", Json::u32(m.triangles));
        ms.arr.push_back(o);
    }
    j.set("meshes", ms);
    j.set("lightmap", to_json(h.lightmap));
    j.set("bake", to_json(h.bake));
    j.set("volume", h.volume ? to_json(*h.volume) : Json());
    j.set("user", h.user);
    return j;
}

}  // namespace lb
