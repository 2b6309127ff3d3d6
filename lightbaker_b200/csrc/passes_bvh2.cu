// The three ray passes over the reference's BVH2, one thread an item as the shader dispatches them
// (crates/lightbaker/src/gpu/trace.wgsl:170-324): direct (sun + occlusion + inside test), gather
// (bounced light), volume (L1 SH + the sun's share). Results match the shader's records exactly.
#include <cuda_runtime.h>

#include "lb_device.cuh"
#include "lb_kernels.h"

namespace lbd {

__device__ __forceinline__ float4 ld4(const float4 *p) { return __ldg(p); }

// trace.wgsl:159-168
template <bool COUNT, bool WT>
__device__ __forceinline__ bool inside(const Scene &S, const lb_params &P, uint32_t seed, float3 o, float3 n,
                                       uint32_t key, Count &c) {
    Frame f = frame(n);
    float back = 0.0f;
    for (uint32_t r = 0; r < 16u; r++) {
        float3 d = cosine((__uint2float_rn(r) + 0.5f) / 16.0f, radical(r), f);
        Hit h = trace<COUNT, WT>(S, o, d, P.ground[3], false, key + r + 7000u, seed, c);
        if (h.tri != NONE && h.back) back += 1.0f;
    }
    return back / 16.0f > __uint_as_float(P.atlas[3]);
}

// The warp's counts into the pass's counters: rays always, the walk's work when COUNT.
template <bool COUNT>
__device__ __forceinline__ void flush(Count &c, unsigned long long *counters) {
    for (int o = 16; o > 0; o >>= 1) {
        c.rays += __shfl_down_sync(0xffffffffu, c.rays, o);
        if (COUNT) {
            c.nodes += __shfl_down_sync(0xffffffffu, c.nodes, o);
            c.tris += __shfl_down_sync(0xffffffffu, c.tris, o);
            c.mats += __shfl_down_sync(0xffffffffu, c.mats, o);
        }
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&counters[0], (unsigned long long)c.rays);
        if (COUNT) {
            atomicAdd(&counters[1], (unsigned long long)c.nodes);
            atomicAdd(&counters[2], (unsigned long long)c.tris);
            atomicAdd(&counters[3], (unsigned long long)c.mats);
        }
    }
}

// trace.wgsl:170-243. `base` is the item index of items[0] in the whole list (the shader's
// P.atlas.z + i), which keys the sample sequence.
template <bool COUNT, bool WT>
__global__ void __launch_bounds__(128) direct_kernel(Scene S, lb_params P, const float4 *items, uint32_t n,
                                                     uint32_t base, float4 *out, unsigned long long *counters) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    Count c;
    c.zero();
    if (i < n) {
        uint32_t seed = __float_as_uint(P.reach[3]);
        float4 p4 = ld4(&items[4 * i]), n4 = ld4(&items[4 * i + 1]), dx4 = ld4(&items[4 * i + 2]), dy4 = ld4(&items[4 * i + 3]);
        float3 nrm = xyz(n4), pos = xyz(p4), dx = xyz(dx4), dy = xyz(dy4);
        uint32_t key = (base + i) * 7919u;
        uint32_t g = P.counts[0];
        float3 sun = xyz(P.sun_dir);
        float soft = 0.0f;
        uint32_t hard = 0u;
        float3 lift = scl(nrm, P.reach[2]);
        float3 at = pos;
        uint32_t pick = 0u;
        float span = 1.0f;
        if (inside<COUNT, WT>(S, P, seed, add(at, lift), nrm, key, c)) {
            for (uint32_t q = 1u; q < 9u; q++) {
                float2 cc = offset(q);
                float3 p = add(add(pos, scl(dx, cc.x)), scl(dy, cc.y));
                if (!inside<COUNT, WT>(S, P, seed, add(p, lift), nrm, key + q * 31u, c)) {
                    at = p;
                    pick = q;
                    span = 0.4f;
                    break;
                }
            }
            if (pick == 0u) {
                float3 p = add(pos, scl(nrm, PUSH));
                if (!inside<COUNT, WT>(S, P, seed, add(p, lift), nrm, key + 331u, c)) {
                    at = p;
                    pick = 9u;
                    span = 0.4f;
                }
            }
        }
        if (dot3(sun, nrm) > 0.0f) {
            Frame sf = frame(sun);
            uint32_t gg = g * g;
            float fg = __uint2float_rn(g), fgg = __uint2float_rn(gg);
            uint32_t turn = uint32_t(rnd(key, 17u, seed) * fgg);
            for (uint32_t s = 0u; s < gg; s++) {
                float cx = ((__uint2float_rn(s % g) + 0.5f) / fg - 0.5f) * span;
                float cy = ((__uint2float_rn(s / g) + 0.5f) / fg - 0.5f) * span;
                float3 o = add(add(add(at, scl(dx, cx)), scl(dy, cy)), lift);
                if (trace<COUNT, WT>(S, o, sun, FAR, true, key + s, seed, c).tri == NONE) hard |= 1u << (s & 31u);  // WGSL shifts modulo the bit width
                uint32_t k = (s + turn) % gg;
                float3 d = sun_disc(P, sf, k, gg);
                if (trace<COUNT, WT>(S, o, d, FAR, true, key + s + 1000u, seed, c).tri == NONE) soft += 1.0f;
            }
            soft /= fgg;
        }
        Frame f = frame(nrm);
        float3 o = add(at, lift);
        uint32_t rays = P.counts[1];
        float frays = __uint2float_rn(rays);
        float s1 = rnd(key, 3u, seed), s2 = rnd(key, 5u, seed);
        float occ = 0.0f, back = 0.0f;
        for (uint32_t r = 0u; r < rays; r++) {
            float3 d = cosine(fract((__uint2float_rn(r) + 0.5f) / frays + s1), fract(radical(r) + s2), f);
            Hit h = trace<COUNT, WT>(S, o, d, P.reach[0], false, key + r + 2000u, seed, c);
            if (h.tri == NONE) continue;
            float k = h.t / P.reach[0];
            occ += 1.0f - k * k;
            if (h.back && h.t < P.ground[3]) back += 1.0f;
        }
        out[i] = make_float4(soft, __uint_as_float(hard | (pick << 24u)), occ / frays, back / frays);
    }
    flush<COUNT>(c, counters);
}

// trace.wgsl:245-270
template <bool COUNT, bool WT>
__global__ void __launch_bounds__(128) gather_kernel(Scene S, lb_params P, const float4 *items, uint32_t n,
                                                     uint32_t base, const float4 *light, uint32_t n_light,
                                                     float4 *out, unsigned long long *counters) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    Count c;
    c.zero();
    if (i < n) {
        uint32_t seed = __float_as_uint(P.reach[3]);
        float4 p4 = ld4(&items[4 * i]), n4 = ld4(&items[4 * i + 1]), dx4 = ld4(&items[4 * i + 2]), dy4 = ld4(&items[4 * i + 3]);
        float3 nrm = xyz(n4), pos = xyz(p4), dx = xyz(dx4), dy = xyz(dy4);
        Frame f = frame(nrm);
        uint32_t key = (base + i) * 7919u;
        uint32_t rays = P.counts[2];
        float frays = __uint2float_rn(rays);
        float s1 = rnd(key, 11u, seed), s2 = rnd(key, 13u, seed);
        float3 sum = mk(0.f, 0.f, 0.f);
        float back = 0.0f;
        for (uint32_t r = 0u; r < rays; r++) {
            float jx = rnd(key + r, 19u, seed) - 0.5f, jy = rnd(key + r, 23u, seed) - 0.5f;
            float3 o = add(add(add(pos, scl(dx, jx)), scl(dy, jy)), scl(nrm, P.reach[2]));
            float3 d = cosine(fract((__uint2float_rn(r) + 0.5f) / frays + s1), fract(radical(r) + s2), f);
            Hit h = trace<COUNT, WT>(S, o, d, P.reach[1], false, key + r + 4000u, seed, c);
            if (h.tri == NONE) {
                sum = add(sum, sky(P, d));
                continue;
            }
            if (h.back) {
                back += 1.0f;
                continue;
            }
            sum = add(sum, bounced(S, P, light, n_light, o, d, h));
        }
        float3 e = scl(sum, PI);
        out[i] = make_float4(e.x / frays, e.y / frays, e.z / frays, back / frays);
    }
    flush<COUNT>(c, counters);
}

// trace.wgsl:272-324
template <bool COUNT, bool WT>
__global__ void __launch_bounds__(128) volume_kernel(Scene S, lb_params P, const float4 *items, uint32_t n,
                                                     const float4 *light, uint32_t n_light, float4 *out,
                                                     unsigned long long *counters) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    Count c;
    c.zero();
    if (i < n) {
        uint32_t seed = __float_as_uint(P.reach[3]);
        float4 p4 = ld4(&items[4 * i]), n4 = ld4(&items[4 * i + 1]);
        float3 o = xyz(p4);
        uint32_t key = __float_as_uint(n4.w) * 7919u + 77u;
        uint32_t rays = P.counts[2];
        float frays = __uint2float_rn(rays);
        float s1 = rnd(key, 29u, seed), s2 = rnd(key, 31u, seed);
        float3 l0 = mk(0.f, 0.f, 0.f), l1x = l0, l1y = l0, l1z = l0;
        float back = 0.0f;
        for (uint32_t r = 0u; r < rays; r++) {
            float u = fract((__uint2float_rn(r) + 0.5f) / frays + s1);
            float v = fract(radical(r) + s2);
            float z = 1.0f - 2.0f * u;
            float rr = sqrtf(fmaxf(0.0f, 1.0f - z * z));
            float a = v * 2.0f * PI;
            float sa, ca;
            sincos32(a, &sa, &ca);
            float3 d = mk(rr * ca, z, rr * sa);
            Hit h = trace<COUNT, WT>(S, o, d, P.reach[1], false, key + r, seed, c);
            float3 l = sky(P, d);
            if (h.tri != NONE) {
                if (h.back) back += 1.0f;
                l = h.back ? mk(0.f, 0.f, 0.f) : bounced(S, P, light, n_light, o, d, h);
            }
            l0 = add(l0, scl(l, 0.282095f));
            float3 lw = scl(l, 0.488603f);
            l1x = add(l1x, scl(lw, d.x));
            l1y = add(l1y, scl(lw, d.y));
            l1z = add(l1z, scl(lw, d.z));
        }
        float w = 4.0f * PI / frays;
        uint32_t g = P.counts[0], gg = g * g;
        Frame sf = frame(xyz(P.sun_dir));
        float sun = 0.0f;
        for (uint32_t s = 0u; s < gg; s++) {
            float3 d = sun_disc(P, sf, s, gg);
            if (trace<COUNT, WT>(S, o, d, FAR, true, key + s + 9000u, seed, c).tri == NONE) sun += 1.0f;
        }
        float3 a0 = scl(l0, w), ax = scl(l1x, w), ay = scl(l1y, w), az = scl(l1z, w);
        out[4 * i] = make_float4(a0.x, a0.y, a0.z, sun / __uint2float_rn(gg));
        out[4 * i + 1] = make_float4(ax.x, ax.y, ax.z, back / frays);
        out[4 * i + 2] = make_float4(ay.x, ay.y, ay.z, 0.0f);
        out[4 * i + 3] = make_float4(az.x, az.y, az.z, 0.0f);
    }
    flush<COUNT>(c, counters);
}

}  // namespace lbd

namespace {
template <bool COUNT, bool WT>
cudaError_t launch_bvh2(int pass, dim3 grid, int T, const lbd::Scene &S, const lb_params &P, const float4 *items,
                        uint32_t n, uint32_t base, const float4 *light, uint32_t n_light, float4 *out,
                        unsigned long long *counters, cudaStream_t stream) {
    switch (pass) {
    case LB_PASS_DIRECT:
        lbd::direct_kernel<COUNT, WT><<<grid, T, 0, stream>>>(S, P, items, n, base, out, counters);
        break;
    case LB_PASS_GATHER:
        lbd::gather_kernel<COUNT, WT><<<grid, T, 0, stream>>>(S, P, items, n, base, light, n_light, out, counters);
        break;
    case LB_PASS_VOLUME:
        lbd::volume_kernel<COUNT, WT><<<grid, T, 0, stream>>>(S, P, items, n, light, n_light, out, counters);
        break;
    default:
        return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}
}  // namespace

cudaError_t lb_launch_pass_bvh2(int pass, const lbd::Scene &S, const lb_params &P, const float4 *items, uint32_t n,
                                uint32_t base, const float4 *light, uint32_t n_light, float4 *out,
                                unsigned long long *counters, bool full_count, cudaStream_t stream) {
    if (n == 0) return cudaSuccess;
    const int T = 128;
    dim3 grid((n + T - 1) / T);
    const bool wt = S.verts != nullptr;  // the watertight kernels (lb_scene_set_vertices)
    if (full_count)
        return wt ? launch_bvh2<true, true>(pass, grid, T, S, P, items, n, base, light, n_light, out, counters, stream)
                  : launch_bvh2<true, false>(pass, grid, T, S, P, items, n, base, light, n_light, out, counters, stream);
    return wt ? launch_bvh2<false, true>(pass, grid, T, S, P, items, n, base, light, n_light, out, counters, stream)
              : launch_bvh2<false, false>(pass, grid, T, S, P, items, n, base, light, n_light, out, counters, stream);
}
