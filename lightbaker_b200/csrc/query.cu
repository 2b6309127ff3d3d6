// Rays against an uploaded scene: lb_trace. The reference's walk (crates/lightbaker/src/gpu/trace.wgsl:83-130)
// is internal to its three passes; this entry point runs the same walk for rays a caller builds, one
// thread a ray, so a pass's rays can be checked one at a time (hit/miss masks, faces, distances) against
// the CPU oracle and between the two triangle tests.
#include <cuda_runtime.h>

#include <cstring>

#include "lb_device.cuh"
#include "lb_runtime.h"

namespace lbd {

template <int BVH, bool WT>
__global__ void __launch_bounds__(256) k_trace(Scene S, const lb_ray *rays, uint32_t n, int any, uint32_t seed,
                                               lb_hit *out) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 *r = (const float4 *)(rays + i);
        float4 a = __ldg(r), b = __ldg(r + 1);
        Count c;
        c.zero();
        Hit h = walk<BVH, false, WT>(S, mk(a.x, a.y, a.z), mk(b.x, b.y, b.z), a.w, any != 0, __float_as_uint(b.w), seed, c);
        ((uint4 *)out)[i] = make_uint4(__float_as_uint(h.t), h.tri, h.back ? 1u : 0u, 0u);
    }
}

}  // namespace lbd

extern "C" int lb_trace(lb_gpu *g, lb_scene *s, const lb_ray *rays, size_t n, int any, uint32_t seed, lb_hit *out) {
    static_assert(sizeof(lb_ray) == 32 && sizeof(lb_hit) == 16, "ray and hit records are two and one float4");
    if (!g || !s || s->gpu != g || (n && (!rays || !out))) {
        lb_set_error("lb_trace: bad arguments");
        return LB_EINVAL;
    }
    if (n == 0) return LB_OK;
    if (n > 0x7fffffffu) {
        lb_set_error("lb_trace: more than 2^31 rays in one call");
        return LB_EINVAL;
    }
    cudaError_t e = cudaSetDevice(g->device);
    if (e != cudaSuccess) return lb_cuda_fail(e, "cudaSetDevice");
    int rc;
    if ((rc = lb_buffer_reserve(g->items, n * sizeof(lb_ray))) != LB_OK) return rc;
    if ((rc = lb_buffer_reserve(g->out, n * sizeof(lb_hit))) != LB_OK) return rc;
    e = cudaMemcpyAsync(g->items.ptr, rays, n * sizeof(lb_ray), cudaMemcpyHostToDevice, g->stream);
    if (e != cudaSuccess) return lb_cuda_fail(e, "lb_trace: copy rays");
    g->h2d += n * sizeof(lb_ray);
    lbd::Scene S = lb_scene_view(s);
    uint32_t m = uint32_t(n);
    int blocks = int((m + 255u) / 256u);
    int cap = (g->sms > 0 ? g->sms : 148) * 8;
    if (blocks > cap) blocks = cap;
    const lb_ray *dr = (const lb_ray *)g->items.ptr;
    lb_hit *dh = (lb_hit *)g->out.ptr;
    const bool wt = S.verts != nullptr;
    if (g->bvh == 8) {
        if (!S.nodes8 || !S.tris8) {
            lb_set_error("lb_trace: the scene has no 8-wide BVH");
            return LB_EINVAL;
        }
        if (wt) lbd::k_trace<8, true><<<blocks, 256, 0, g->stream>>>(S, dr, m, any, seed, dh);
        else lbd::k_trace<8, false><<<blocks, 256, 0, g->stream>>>(S, dr, m, any, seed, dh);
    } else {
        if (wt) lbd::k_trace<2, true><<<blocks, 256, 0, g->stream>>>(S, dr, m, any, seed, dh);
        else lbd::k_trace<2, false><<<blocks, 256, 0, g->stream>>>(S, dr, m, any, seed, dh);
    }
    e = cudaGetLastError();
    if (e != cudaSuccess) return lb_cuda_fail(e, "lb_trace: launch");
    e = cudaMemcpyAsync(out, dh, n * sizeof(lb_hit), cudaMemcpyDeviceToHost, g->stream);
    if (e != cudaSuccess) return lb_cuda_fail(e, "lb_trace: copy hits");
    g->d2h += n * sizeof(lb_hit);
    e = cudaStreamSynchronize(g->stream);
    if (e != cudaSuccess) return lb_cuda_fail(e, "lb_trace");
    return LB_OK;
}
