#include "deps.h"

#include <cmath>

namespace lb {

Boxes::Boxes(const Scene &scene) {
    for (auto &p : scene.positions) {
        std::vector<Aabb> v;
        v.reserve(p.size() / 3);
        for (size_t t = 0; t + 2 < p.size(); t += 3) {
            Aabb b;
            for (int k = 0; k < 3; k++) b.add(p[t + k]);
            v.push_back(b);
            top = std::fmax(top, b.max.y);
        }
        boxes.push_back(std::move(v));
    }
}

Hash global_hash(const Scene &scene) {
    const SceneHeader &h = scene.header;
    Blake3 k;
    uint32_t v = BAKER_VERSION;
    k.update(&v, 4);
    for (const Json &j : {to_json(h.sun), to_json(h.sky), to_json(h.materials), to_json(h.lightmap), to_json(h.bake)}) {
        std::string s = j.dump();
        k.update(s.data(), s.size());
    }
    Hash out;
    k.finalize(out.data());
    return out;
}

Hash watertight_hash(const Hash &global) {
    Blake3 k;
    k.update(global.data(), global.size());
    static const char tag[] = "watertight triangle test";
    k.update(tag, sizeof tag - 1);
    Hash out;
    k.finalize(out.data());
    return out;
}

bool swept(const Aabb &zone, Vec3 sun, float top, const Aabb &b) {
    float tmax = sun.y > 1e-4f ? std::fmax((top - zone.min.y) / sun.y, 0.0f) : 0.0f;
    float lo = 0.0f, hi = tmax;
    for (int a = 0; a < 3; a++) {
        float s = sun[a], zmin = zone.min[a], zmax = zone.max[a], bmin = b.min[a], bmax = b.max[a];
        if (std::fabs(s) < 1e-6f) {
            if (zmin > bmax || zmax < bmin) return false;
            continue;
        }
        float t1 = (bmax - zmin) / s, t2 = (bmin - zmax) / s;
        float a0 = s > 0.0f ? t2 : t1, a1 = s > 0.0f ? t1 : t2;
        lo = std::fmax(lo, a0);
        hi = std::fmin(hi, a1);
        if (lo > hi) return false;
    }
    return true;
}

Hash hash_reach(const Scene &scene, const Boxes &boxes, const Hash &global, const Aabb &own, float reach,
                const std::vector<uint8_t> &seed) {
    Aabb zone = own.grow(reach);
    Vec3 sun = Vec3(scene.header.sun.direction[0], scene.header.sun.direction[1], scene.header.sun.direction[2]).normalize();
    Blake3 k;
    k.update(global.data(), 32);
    k.update(seed.data(), seed.size());
    for (size_t mi = 0; mi < scene.header.meshes.size(); mi++) {
        const MeshInfo &m = scene.header.meshes[mi];
        if (!scene.header.materials[m.material].casts) continue;
        const std::vector<Aabb> &bx = boxes.boxes[mi];
        bool any = false;
        for (size_t t = 0; t < bx.size(); t++) {
            if (!swept(zone, sun, boxes.top, bx[t])) continue;
            if (!any) {
                uint32_t mm = uint32_t(mi);
                k.update(&mm, 4);
                k.update(&m.material, 4);
                any = true;
            }
            uint32_t tt = uint32_t(t);
            k.update(&tt, 4);
            k.update(&scene.positions[mi][t * 3], 36);
        }
    }
    Hash out;
    k.finalize(out.data());
    return out;
}

}  // namespace lb
