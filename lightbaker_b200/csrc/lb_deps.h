// The tiles' and probe chunks' dependency hashes on the device (deps.cu; crates/lightbaker/src/deps.rs:70-121).
#pragma once
#include <array>
#include <cstdint>
#include <vector>

#include "lb_runtime.h"

// The scene as the swept-box test reads it: every casting mesh's triangles (9 floats each), concatenated in
// mesh order; per casting mesh its index in the scene, its material and its first triangle (n + 1 entries);
// per triangle its casting mesh; the sun's normalised direction and the top of every triangle's box.
struct DepsInput {
    const float *pos = nullptr;
    uint32_t n_tris = 0;
    std::vector<uint32_t> mesh_start, mesh_id, mesh_mat, tri_mesh;
    float sun[3] = {0, 0, 0};
    float top = 0;
};

// One hash: the box it is for, the reach round it, and the bytes hashed before the triangles (the global
// hash and the seed).
struct DepsQuery {
    float min[3], max[3];
    float reach;
    std::vector<uint8_t> prefix;
};

// BLAKE3 of each query's message (deps.rs:70-96), every query at once on the handle's stream; throws
// std::runtime_error on a CUDA error.
void lb_hash_reach_device(lb_gpu *g, const DepsInput &in, const std::vector<DepsQuery> &queries,
                          std::vector<std::array<uint8_t, 32>> &out);
