// The C ABI's handles and the runtime helpers the host code shares.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "../../include/lightbaker.h"

// A device buffer kept by a handle and grown on demand.
struct lb_buffer {
    void *ptr = nullptr;
    size_t cap = 0;
};

struct lb_gpu {
    int device = 0;
    int sms = 0;
    char name[256] = {0};
    cudaStream_t stream = nullptr;
    bool counting = false;
    int kernel = 0;  // lb_run's kernels: 0 a thread an item, 1 a warp an item
    int group_direct = 0, group_gather = 0;  // the warp kernels' ray order (passes_warp.cu); 0: wedges of azimuth
    int bvh = 2;  // the warp kernels' BVH: 2 the reference's, 8 the 8-wide one
    int refill = 0;  // the warp kernels' lane refill (occlusion and gather rays over the BVH2)
    int near = 1;    // the warp kernels' leaf list for occlusion rays (BVH2)
    int occ = 0;     // the warp kernels' register cap (WarpPass::occ)
    int fetch = 1;   // the warp kernels take items from a work counter (WarpPass::work)
    int warp_walk = 1;  // the direct pass's sun rays walk the tree together (WarpPass::warp_walk)
    unsigned long long *counters = nullptr;       // device: rays, nodes, tris, mats
    unsigned long long *host_counters = nullptr;  // pinned copy, written by the stream
    lb_counters last = {};
    uint64_t h2d = 0, d2h = 0;  // bytes copied by this handle
    lb_buffer items, out, light, scratch;
    void *stage = nullptr;  // pinned host memory for downloads (lb_host_stage_reserve), kept between calls
    size_t stage_cap = 0;
    // device buffers a freed plan or transport gave back (plan.h DBuf), kept for the next one: no cudaFree,
    // which waits for the whole device, between bakes, and no cudaMalloc for a buffer a spare fits
    std::mutex spare_mu;
    std::vector<std::pair<void *, size_t>> spare;
    size_t spare_bytes = 0;
};

// The scene's buffers (gpu/mod.rs:65-71).
struct lb_scene {
    lb_gpu *gpu = nullptr;
    void *nodes = nullptr, *tris = nullptr, *mats = nullptr, *charts = nullptr;
    uint32_t n_nodes = 0, n_tris = 0, n_mats = 0, n_charts = 0;
    void *nodes8 = nullptr, *tris8 = nullptr;  // the 8-wide BVH collapsed from the BVH2 (bvh8_build.cu)
    uint32_t n_nodes8 = 0, n_tris8 = 0;
    uint32_t depth = 0xffffffffu;  // the most inner nodes on a root-to-leaf path of the BVH2
    void *verts = nullptr;  // exact vertices (lb_scene_set_vertices): the watertight triangle test
};

void lb_set_error(const std::string &msg);
// the device view of an uploaded scene (both BVHs)
namespace lbd {
struct Scene;
}
lbd::Scene lb_scene_view(const lb_scene *s);
int lb_cuda_fail(cudaError_t e, const char *what);
int lb_buffer_reserve(lb_buffer &b, size_t bytes);
int lb_host_stage_reserve(lb_gpu *g, size_t bytes);
// the scene's 8-wide BVH, built on the device from its BVH2 (bvh8_build.cu)
int lb_bvh8_build(lb_gpu *g, lb_scene *s);
void lb_buffer_free(lb_buffer &b);
int lb_run_device(lb_gpu *g, lb_scene *s, int pass, const lb_params &P, const float4 *items, uint32_t n, uint32_t base,
                  const float4 *light, uint32_t n_light, float4 *out);
void lb_collect_counters(lb_gpu *g);
// A spare buffer of at least `bytes` (and not more than twice that, plus 1 MiB) from the handle's spares,
// its size in *cap, or nullptr.
void *lb_spare_take(lb_gpu *g, size_t bytes, size_t *cap);
// Gives a buffer back to the handle's spares once the handle's stream has finished with it (it is
// synchronised here); when the spares would pass their limit the oldest are freed first (a buffer larger
// than the whole limit is freed at once).
void lb_spare_give(lb_gpu *g, void *p, size_t cap);
