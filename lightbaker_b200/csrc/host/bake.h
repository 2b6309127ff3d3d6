// A bake from start to end: crates/lightbaker/src/bake.rs and crates/lightbaker/src/volume.rs. The
// layout, the tiles' hashes, the dirty tiles traced (sun and occlusion, then the bounces, each
// reading every tile's light from the last), the texel passes, the volume, and the atlas.
#pragma once
#include <array>
#include <cstdint>
#include <functional>
#include <optional>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../../include/lightbaker.h"
#include "bvh.h"
#include "deps.h"
#include "layout.h"
#include "scene.h"

namespace lb {

constexpr float LIFT = 0.01f;          // bake.rs:24
constexpr float INSIDE_REACH = 0.3f;   // bake.rs:26
constexpr float PUSH = 0.03f;          // bake.rs:28
constexpr float VOLUME_INSIDE = 0.5f;  // volume.rs:20

// output.rs:29-40
enum Validity : uint8_t { V_NONE = 0, V_CENTRE = 1, V_OFFSET = 2, V_PUSHED = 3, V_FILLED = 4, V_VOLUME = 5 };

// The ray passes, as Gpu::scene and Gpu::run (gpu/mod.rs:129-196): the CUDA runtime in the product.
class Tracer {
  public:
    virtual ~Tracer() = default;
    virtual void scene(const Bvh &bvh, const std::vector<float> &materials, const std::vector<float> &charts) = 0;
    // out: n * width float4 records; returns the rays traced (every trace() call); throws std::runtime_error
    virtual uint64_t run(int pass, const lb_params &params, const std::vector<lb_texel> &items,
                     const std::vector<float> &light, std::vector<float> &out) = 0;
    // the watertight triangle test over the scene's exact vertices for the passes that follow (beyond
    // the reference); a tracer without one throws
    virtual void watertight(const Bvh &) { throw std::runtime_error("this tracer has no watertight triangle test"); }
};

struct Stats {  // bake.rs:49-58
    size_t tiles = 0, tiles_baked = 0, texels_baked = 0, chunks = 0, chunks_baked = 0;
    double seconds = 0;
    // beyond the reference: rays traced a pass (every trace() call), seconds a stage
    uint64_t rays_direct = 0, rays_gather = 0, rays_volume = 0;
    double t_layout = 0, t_direct = 0, t_bounces = 0, t_volume = 0, t_composite = 0;
};

struct TileLight {  // bake.rs:60-80
    std::vector<uint8_t> known, state;
    std::vector<float> field, ao;
    std::vector<std::array<float, 3>> direct, indirect;
    std::vector<uint8_t> pack() const;
    static std::optional<TileLight> unpack(const std::vector<uint8_t> &b, size_t size);
};

struct Volume {  // volume.rs:22-31
    std::array<float, 3> origin;
    float step;
    std::array<uint32_t, 3> size;
    std::vector<std::array<float, 16>> probes;  // [L0 rgb + sun, L1x rgb + back, L1y, L1z]
    size_t chunks = 0, chunks_baked = 0;
    void irradiance(Vec3 p, Vec3 n, float e[3], float &sun) const;  // volume.rs:125-147
};

// The file's encodings of a bake's atlases and probes, when the device made them (encode.cu): the BC5
// blocks of `direct`, the RGB9E5 words of `indirect`, the probes' bytes and their scale.
struct Encoded {
    std::vector<uint8_t> bc5;
    std::vector<uint32_t> rgb9e5;
    std::vector<uint8_t> volume;
    float volume_scale = 1.0f;
};

struct Bake {  // bake.rs:36-47
    Layout layout;
    std::vector<std::array<float, 2>> direct;
    std::vector<std::array<float, 3>> indirect;
    uint32_t iw = 0, ih = 0;
    std::vector<uint8_t> validity;
    std::optional<Volume> volume;
    Stats stats;
    std::optional<Encoded> encoded;  // beyond the reference: set by the device-resident bake
};

struct Options {  // bake.rs:30-34
    std::string cache;  // empty: none
    std::function<void(const std::string &)> log;
    bool watertight = false;  // beyond the reference: the watertight triangle test (Tracer::watertight)
    // beyond the reference: a bake split over `world` processes, this one rank `rank`. sum: the ranks'
    // element-wise sum of 32-bit words in place (data in host memory, or in device memory when `device`)
    int rank = 0, world = 1;
    std::function<void(void *data, size_t words, bool device)> sum;
};

// One rank's share of items with these costs: a contiguous range [first, last) of them, the ranges of
// ranks 0 .. world-1 following one another and splitting the total cost as evenly as whole items allow.
std::pair<size_t, size_t> shard_range(const std::vector<uint64_t> &cost, int rank, int world);

// The inputs every pass needs, built once per bake.
struct Prepared {
    Layout layout;
    std::vector<uint32_t> chart_tile;
    std::vector<float> affines;    // 8 a chart
    std::vector<float> materials;  // 4 a material
    Bvh bvh;
    lb_params params;
    Vec3 sun;
    uint32_t g;
};
Prepared prepare(const Scene &scene);

Bake bake(const Scene &scene, Tracer &gpu, const Options &o);

// bake.rs helpers shared with the device-resident bake
Aabb tile_box(const Scene &scene, const Layout &layout, const std::vector<uint32_t> &charts);
std::vector<uint8_t> tile_seed(const Scene &scene, const Layout &layout, TileKey key, const std::vector<uint32_t> &charts);
void write_light(const Layout &layout, size_t ti, const TileLight &l, std::vector<float> &light);
void texel_offset(uint32_t q, float &x, float &y);  // bake.rs:494-503

// .lbake writer: crates/lightbaker/src/output.rs
std::vector<uint8_t> write_bake(const Scene &scene, const Bake &bake);

}  // namespace lb
