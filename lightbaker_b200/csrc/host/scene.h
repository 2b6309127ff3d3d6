// The scene a bake reads (.lbscene): crates/lightbaker/src/scene.rs. The magic `LBSC`, version 1
// (u32), the header's length (u32), the JSON header, then each mesh's positions (f32 x y z, three
// vertices a triangle), each array starting on a 4-byte boundary.
#pragma once
#include <array>
#include <cstdint>
#include <optional>
#include <string>
#include <vector>

#include "json.h"
#include "vec.h"

namespace lb {

using Rgb = std::array<float, 3>;

struct Sun {  // scene.rs:42-51
    std::array<float, 3> direction;
    float radius_deg;
    Rgb irradiance;
};
struct Sky {  // scene.rs:53-60
    Rgb zenith, horizon, ground;
};
struct Material {  // scene.rs:62-75
    std::string name;
    Rgb albedo;
    bool receives, casts;
    float opacity = 1.0f;
};
struct MeshInfo {  // scene.rs:81-87
    std::string name;
    uint32_t material, triangles;
};
struct LightmapSettings {  // scene.rs:89-103
    float texels_per_meter, tile_size, chart_angle_deg;
    uint32_t padding, atlas_width, indirect_downscale;
};
struct BakeSettings {  // scene.rs:105-126
    uint32_t sun_samples, ao_rays;
    float ao_reach, ao_strength, ao_floor, ao_contrast, sdf_radius;
    uint32_t gi_rays, gi_bounces;
    float gi_reach, inside_share;
    uint32_t gi_filter;
};
struct VolumeSettings {  // scene.rs:128-135
    std::array<float, 3> min, max;
    float step;
    uint32_t rays;
};
struct SceneHeader {  // scene.rs:25-40
    Sun sun;
    Sky sky;
    std::vector<Material> materials;
    std::vector<MeshInfo> meshes;
    LightmapSettings lightmap;
    BakeSettings bake;
    std::optional<VolumeSettings> volume;
    Json user;
};

struct Scene {
    SceneHeader header;
    std::vector<std::vector<Vec3>> positions;  // per mesh, three vertices a triangle
    std::array<uint8_t, 32> hash;              // blake3 of the whole file
    static Scene read(const uint8_t *bytes, size_t len);  // throws std::runtime_error
    static std::vector<uint8_t> write(const SceneHeader &h, const std::vector<std::vector<Vec3>> &positions);
    size_t triangle_count() const;
};

// serde_json's compact serialisation of each settings struct (field order and names as the reference).
Json to_json(const Sun &);
Json to_json(const Sky &);
Json to_json(const std::vector<Material> &);
Json to_json(const LightmapSettings &);
Json to_json(const BakeSettings &);
Json to_json(const VolumeSettings &);
Json to_json(const SceneHeader &);

}  // namespace lb
