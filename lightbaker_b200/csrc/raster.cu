// The texel rasteriser on the device (crates/lightbaker/src/raster.rs:39-114), for the device-resident
// bake. The host lays out each triangle of each dirty tile's charts (its chart-space corners, the plane it
// spans and its texel box: the per-triangle set-up of raster.rs:48-67) in the order the host rasteriser
// visits them; the device does the per-texel work. In each of the two passes (texel centres inside the
// triangle, then the nearest point of the triangle within half a texel) a texel takes the first triangle
// in that order that claims it, as the host's "skip a covered texel" rule makes it: every triangle's
// claims are an atomic minimum on its index, then the winners write their texels. The arithmetic is the
// host's, in its order (built without contraction), so the texels equal the host's bit for bit.
#include <cuda_runtime.h>

#include <cub/cub.cuh>

#include "lb_post.h"

namespace lbd {
namespace {

constexpr uint32_t NOBODY = 0xffffffffu;

__device__ __forceinline__ float signum(float x) { return isnan(x) ? x : copysignf(1.0f, x); }
__device__ __forceinline__ float clampf(float v, float lo, float hi) { return v < lo ? lo : (v > hi ? hi : v); }

// raster.rs:102-114: the point of triangle (a, b, c) nearest p, in chart space
__device__ float2 nearest(float2 p, float2 a, float2 b, float2 c) {
    auto side = [](float2 o, float2 e, float2 q) {  // (e - o).perp_dot(q - o)
        float ex = e.x - o.x, ey = e.y - o.y, qx = q.x - o.x, qy = q.y - o.y;
        return ex * qy - ey * qx;
    };
    float s = signum(side(a, b, c));
    if (side(a, b, p) * s >= 0.0f && side(b, c, p) * s >= 0.0f && side(c, a, p) * s >= 0.0f) return p;
    auto seg = [&](float2 o, float2 e) {
        float dx = e.x - o.x, dy = e.y - o.y;
        float px = p.x - o.x, py = p.y - o.y;
        float k = clampf((px * dx + py * dy) / fmaxf(dx * dx + dy * dy, 1e-12f), 0.0f, 1.0f);
        return make_float2(o.x + dx * k, o.y + dy * k);
    };
    auto dist2 = [&](float2 q) {
        float x = q.x - p.x, y = q.y - p.y;
        return x * x + y * y;
    };
    float2 cand[3] = {seg(a, b), seg(b, c), seg(c, a)};
    float2 best = cand[0];
    float bd = dist2(best);
    for (int k = 1; k < 3; k++) {
        float d = dist2(cand[k]);
        if (d < bd) {  // the first of equals
            bd = d;
            best = cand[k];
        }
    }
    return best;
}

// raster.rs:55-58: barycentric weights of q
__device__ __forceinline__ void bary(const RasterTri &t, float2 q, float &l1, float &l2, float &l3) {
    l1 = ((t.ub[1] - t.uc[1]) * (q.x - t.uc[0]) + (t.uc[0] - t.ub[0]) * (q.y - t.uc[1])) / t.det;
    l2 = ((t.uc[1] - t.ua[1]) * (q.x - t.uc[0]) + (t.ua[0] - t.uc[0]) * (q.y - t.uc[1])) / t.det;
    l3 = 1.0f - l1 - l2;
}

// the point the texel samples in pass CONS (false: its centre, kept when inside; true: the nearest point
// of the triangle, kept within half a texel); false when the triangle does not claim it
template <bool CONS>
__device__ __forceinline__ bool sample(const RasterTri &t, int x, int y, float2 &q) {
    float2 centre = make_float2(float(x) + 0.5f, float(y) + 0.5f);
    if (CONS) {
        q = nearest(centre, make_float2(t.ua[0], t.ua[1]), make_float2(t.ub[0], t.ub[1]),
                    make_float2(t.uc[0], t.uc[1]));
        return !(fabsf(q.x - centre.x) > 0.5f || fabsf(q.y - centre.y) > 0.5f);
    }
    q = centre;
    float l1, l2, l3;
    bary(t, q, l1, l2, l3);
    return !(l1 < -1e-4f || l2 < -1e-4f || l3 < -1e-4f);
}

// One warp a triangle: each texel of its box that is not yet covered and that it claims takes the
// smallest claiming triangle index.
template <bool CONS>
__global__ void __launch_bounds__(256) k_claim(const RasterTri *tris, uint32_t n, const DTile *tiles,
                                               const float4 *tex, uint32_t *owner) {
    const int lane = threadIdx.x & 31;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t e = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; e < n; e += warps) {
        const RasterTri t = tris[e];
        const DTile tl = tiles[t.tile];
        const int bw = t.x1 - t.x0 + 1, bh = t.y1 - t.y0 + 1;
        if (bw <= 0 || bh <= 0) continue;
        const int cells = bw * bh;
        for (int c = lane; c < cells; c += 32) {
            const int x = t.x0 + c % bw, y = t.y0 + c / bw;
            const uint32_t i = tl.off + uint32_t(y) * tl.w + uint32_t(x);
            if (tex[4 * size_t(i)].w > 0.5f) continue;  // covered by an earlier pass
            float2 q;
            if (sample<CONS>(t, x, y, q)) atomicMin(&owner[i], e);
        }
    }
}

// One thread a texel: the winning triangle writes it (raster.rs:92-95) and the claim is cleared.
template <bool CONS>
__global__ void __launch_bounds__(256) k_write(const RasterTri *tris, const DTile *tiles, uint32_t n_texels,
                                               float4 *tex, uint32_t *owner) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n_texels; i += gridDim.x * blockDim.x) {
        const uint32_t e = owner[i];
        if (e == NOBODY) continue;
        owner[i] = NOBODY;
        const RasterTri t = tris[e];
        const DTile tl = tiles[t.tile];
        const uint32_t r = i - tl.off;
        float2 q;
        sample<CONS>(t, int(r % tl.w), int(r / tl.w), q);
        float l1, l2, l3;
        bary(t, q, l1, l2, l3);
        // (pa * l1 + pb * l2) + pc * l3
        float px = (t.pa[0] * l1 + t.pb[0] * l2) + t.pc[0] * l3;
        float py = (t.pa[1] * l1 + t.pb[1] * l2) + t.pc[1] * l3;
        float pz = (t.pa[2] * l1 + t.pb[2] * l2) + t.pc[2] * l3;
        float4 *o = tex + 4 * size_t(i);
        o[0] = make_float4(px, py, pz, 1.0f);
        o[1] = make_float4(t.n[0], t.n[1], t.n[2], __uint_as_float(t.chart));
        o[2] = make_float4(t.dx[0], t.dx[1], t.dx[2], 0.0f);
        o[3] = make_float4(t.dy[0], t.dy[1], t.dy[2], 0.0f);
    }
}

__global__ void k_fill_u32(uint32_t *p, uint32_t n, uint32_t v) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) p[i] = v;
}

// Covered texels that are the first of their chart in their ds x ds block (row-major within the block):
// the number of (block, chart) pairs, which bounds the gathered texels (bake.rs:286-297).
__global__ void k_first_of_chart(const DTile *tiles, uint32_t n_tiles, const float4 *tex, uint32_t ds,
                                 unsigned long long *count) {
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
    unsigned long long mine = 0;
    for (uint32_t k = 0; k < n_tiles; k++) {
        const DTile tl = tiles[k];
        const uint32_t n = tl.w * tl.h;
        for (uint32_t r = tid; r < n; r += stride) {
            const float4 *a = tex + 4 * (size_t(tl.off) + r);
            if (!(a[0].w > 0.5f)) continue;
            const uint32_t chart = __float_as_uint(a[1].w);
            const uint32_t x = r % tl.w, y = r / tl.w, bx = x / ds * ds, by = y / ds * ds;
            bool first = true;
            for (uint32_t yy = by; yy <= y && first; yy++)
                for (uint32_t xx = bx; xx < min(bx + ds, tl.w) && first; xx++) {
                    if (yy == y && xx >= x) break;
                    const float4 *b = tex + 4 * (size_t(tl.off) + yy * tl.w + xx);
                    if (b[0].w > 0.5f && __float_as_uint(b[1].w) == chart) first = false;
                }
            mine += first ? 1ull : 0ull;
        }
    }
    for (int o = 16; o > 0; o >>= 1) mine += __shfl_down_sync(0xffffffffu, mine, o);
    if ((threadIdx.x & 31) == 0 && mine) atomicAdd(count, mine);
}

__global__ void k_inverse_index(const uint32_t *idx, const uint32_t *count, uint32_t *inv) {
    const uint32_t n = *count;
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) inv[idx[j]] = j;
}

struct CoveredFlag {
    const float4 *tex;
    __device__ __forceinline__ uint8_t operator()(uint32_t i) const { return tex[4 * size_t(i)].w > 0.5f ? 1 : 0; }
};

// the atlas owner map: each tile texel's place in the concatenated texel arrays
__global__ void k_owner(const DTile *tiles, uint32_t n_tiles, uint32_t aw, uint32_t *owner) {
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
    for (uint32_t k = 0; k < n_tiles; k++) {
        const DTile tl = tiles[k];
        const uint32_t n = tl.w * tl.h;
        for (uint32_t r = tid; r < n; r += stride)
            owner[size_t(tl.y + r / tl.w) * aw + tl.x + r % tl.w] = tl.off + r;
    }
}

int grid_for(uint32_t n, int sms, int per_sm = 8) {
    int g = int((n + 255u) / 256u);
    int cap = (sms > 0 ? sms : 148) * per_sm;
    return g < 1 ? 1 : (g > cap ? cap : g);
}

}  // namespace
}  // namespace lbd

cudaError_t lb_raster_tiles(const RasterTri *tris, uint32_t n_tris, const DTile *tiles, uint32_t n_tiles,
                            uint32_t n_texels, uint32_t ds, float4 *tex, uint32_t *scratch,
                            unsigned long long *pairs, int sms, cudaStream_t st) {
    using namespace lbd;
    cudaError_t e = cudaMemsetAsync(tex, 0, size_t(n_texels) * 64, st);
    if (e != cudaSuccess || n_texels == 0) return e;
    k_fill_u32<<<grid_for(n_texels, sms), 256, 0, st>>>(scratch, n_texels, NOBODY);
    if (n_tris) {
        const int gw = grid_for(n_tris * 32u, sms);
        k_claim<false><<<gw, 256, 0, st>>>(tris, n_tris, tiles, tex, scratch);
        k_write<false><<<grid_for(n_texels, sms), 256, 0, st>>>(tris, tiles, n_texels, tex, scratch);
        k_claim<true><<<gw, 256, 0, st>>>(tris, n_tris, tiles, tex, scratch);
        k_write<true><<<grid_for(n_texels, sms), 256, 0, st>>>(tris, tiles, n_texels, tex, scratch);
    }
    e = cudaMemsetAsync(pairs, 0, sizeof(unsigned long long), st);
    if (e != cudaSuccess) return e;
    k_first_of_chart<<<grid_for(n_texels, sms), 256, 0, st>>>(tiles, n_tiles, tex, ds, pairs);
    return cudaGetLastError();
}

size_t lb_raster_covered_temp(uint32_t n_texels) {
    size_t bytes = 0;
    cub::CountingInputIterator<uint32_t> it(0);
    cub::TransformInputIterator<uint8_t, lbd::CoveredFlag, cub::CountingInputIterator<uint32_t>> flags(
        it, lbd::CoveredFlag{nullptr});
    cub::DeviceSelect::Flagged(nullptr, bytes, it, flags, (uint32_t *)nullptr, (uint32_t *)nullptr, int(n_texels));
    return bytes;
}

cudaError_t lb_raster_covered(const float4 *tex, uint32_t n_texels, void *temp, size_t temp_bytes, uint32_t *idx,
                              uint32_t *count, uint32_t *inverse, int sms, cudaStream_t st) {
    using namespace lbd;
    cudaError_t e = cudaMemsetAsync(count, 0, 4, st);
    if (e != cudaSuccess || n_texels == 0) return e;
    k_fill_u32<<<grid_for(n_texels, sms), 256, 0, st>>>(inverse, n_texels, NOBODY);
    cub::CountingInputIterator<uint32_t> it(0);
    cub::TransformInputIterator<uint8_t, CoveredFlag, cub::CountingInputIterator<uint32_t>> flags(it, CoveredFlag{tex});
    e = cub::DeviceSelect::Flagged(temp, temp_bytes, it, flags, idx, count, int(n_texels), st);
    if (e != cudaSuccess) return e;
    k_inverse_index<<<grid_for(n_texels, sms), 256, 0, st>>>(idx, count, inverse);
    return cudaGetLastError();
}

cudaError_t lb_owner_map(const DTile *tiles, uint32_t n_tiles, uint32_t aw, uint32_t ah, uint32_t *owner, int sms,
                         cudaStream_t st) {
    using namespace lbd;
    const uint32_t n = aw * ah;
    if (n == 0) return cudaSuccess;
    k_fill_u32<<<grid_for(n, sms), 256, 0, st>>>(owner, n, NOBODY);
    if (n_tiles) k_owner<<<grid_for(n, sms), 256, 0, st>>>(tiles, n_tiles, aw, owner);
    return cudaGetLastError();
}
