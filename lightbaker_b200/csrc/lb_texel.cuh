// Texel helpers shared by the device bake's texel passes (post.cu) and the transport (transport.cu).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "lb_post.h"

namespace lbd {

// the tile holding texel i: tiles sorted by their first texel
__device__ __forceinline__ int find_tile(const DTile *tiles, int n, uint32_t i) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (tiles[mid].off <= i) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// filter.rs:13-18: two texels of one chart whose normals agree
__device__ __forceinline__ bool same(const uint32_t *chart, const float4 *tex, uint32_t i, uint32_t j) {
    if (chart[i] != chart[j]) return false;
    float4 a = tex[4 * i + 1], b = tex[4 * j + 1];
    return a.x * b.x + a.y * b.y + a.z * b.z >= 0.9f;
}

}  // namespace lbd
