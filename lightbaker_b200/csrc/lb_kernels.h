// Launchers of the device code, for the runtime (runtime.cu) and the device-resident bake.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/lightbaker.h"

namespace lbd {
struct Scene;
}

// One ray pass over the BVH2, one thread an item. base: the index of items[0] in the whole list.
// counters (device, 4 x u64): rays always; nodes, triangles, materials when full_count.
cudaError_t lb_launch_pass_bvh2(int pass, const lbd::Scene &S, const lb_params &P, const float4 *items, uint32_t n,
                                uint32_t base, const float4 *light, uint32_t n_light, float4 *out,
                                unsigned long long *counters, bool full_count, cudaStream_t stream);

// A warp-per-item pass (passes_warp.cu). Items are tex[idx[k]] (or tex[k] without idx), k < *n_dev
// (or n_host); the gather pass may take positions from `pos` (indexed like tex records).
struct WarpPass {
    int pass;
    const lbd::Scene *S;
    const lb_params *P;
    const float4 *tex;        // 4 float4 a texel record
    const uint32_t *idx;      // optional
    const float4 *pos;        // optional (gather)
    const uint32_t *n_dev;    // optional (direct, gather)
    uint32_t n_host;
    uint32_t base;
    const float4 *light;
    uint32_t n_light;
    float4 *out;
    const uint32_t *slot;     // optional (volume): where probe k's records go
    unsigned long long *counters;
    bool full_count;
    int sms;
    int blocks;               // 0: as many as fit on the device at once
    int group;                // ray order within an item (passes_warp.cu): top index bits a round shares
    int bvh;                  // 2: the reference's BVH2; 8: the 8-wide BVH (S->nodes8)
    int refill;               // BVH2 occlusion and gather rays: a lane starts the item's next ray when its own ends
    int near;                 // BVH2 occlusion rays: test a leaf list gathered once an item (lb_device.cuh)
    int occ;                  // BVH2 direct and gather passes without counting: 3 or 4 caps registers so that
                              // this many 256-thread blocks fit an SM; else the compiler's own budget
    uint2 *rec;               // optional (gather, volume): every ray's outcome, [item][ray] (lb_device.cuh
                              // gather_record)
    unsigned int *work;       // optional (direct, gather): a counter the launch zeroes, from which warps take
                              // their next item as they free up; null: a static stride over the items
    int warp_walk;            // direct pass over the BVH2 without counting: a texel's sun rays walk the tree
                              // together (lb_device.cuh escapes_warp), when the tree is shallow enough
    uint32_t part, parts;     // a split bake: this rank takes share `part` of `parts` of the items (item_part in
                              // lb_device.cuh); parts 0 or 1: every item
};
// The gather records evaluated against a light atlas and theta (albedo 3 a material, zenith, horizon,
// ground, sun scale; transport.cu): each item's gather result, its terms summed in ray order, equal to
// what the gather pass gives for the same light.
// part, parts: only that share of the items (item_part), as the gather pass that recorded them.
cudaError_t lb_eval_records(const uint2 *rec, const uint32_t *n_dev, uint32_t n_host, uint32_t rays,
                            const float4 *light, uint32_t n_light, const float *theta, uint32_t n_mats, float4 *out,
                            int sms, cudaStream_t stream, uint32_t part = 0, uint32_t parts = 1);
cudaError_t lb_launch_pass_warp(const WarpPass &w, cudaStream_t stream);
// The persistent grid's size for a pass: SMs x resident blocks of 256 threads.
int lb_warp_pass_blocks(const WarpPass &w);
