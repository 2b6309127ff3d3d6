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
