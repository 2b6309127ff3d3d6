// The bounce transport of a bake, and its adjoint.
//
// The bake's indirect light is a function of the scene's light parameters theta: every material's albedo,
// the sky's zenith, horizon and ground colours, and the sun's intensity (a scale s on its irradiance).
// Nothing else in the bake depends on them: visibility, the texel layout, the gather selection and every
// filter's weights are fixed by the geometry. So the transport records once what each gather ray met
// (trace.wgsl:245-270; the rays are the same in every bounce, their keys depend on the gathered texel's
// index and not on the bounce) and runs the bounces of bake.rs:300-329 as
//
//   light_0      = write_light(s * dl0)                           bake.rs:268-275 with write_light :434-444
//   res_b        = eval(records, light_b, theta)                  trace.wgsl:258-269, bounced :133-148
//   e_b          = fill(smooth(scatter(res_b)))                   bake.rs:309-323
//   light_{b+1}  = write_light(s * dl0 + e_b)                     bake.rs:324-328
//   probes       = fill(project(vrecords, light_B, theta))        trace.wgsl:272-324, volume.rs:88-121
//   fallback     = irradiance(probes) at the validity-5 texels    bake.rs:335-359, volume.rs:125-147
//   indirect     = dilate(dilate(composite(e_{B-1} | fallback)))  bake.rs:364-421
//
// where dl0 is the direct light at the scene's irradiance (linear in it: bake.rs:247-252 and the fills)
// and vrecords what each volume ray met (recorded once, as the gather rays). At theta0 (the scene's own
// values) every step is the device bake's own arithmetic on the same inputs, so the result is the bake's
// indirect atlas bit for bit. The volume's share runs only when some texel takes the fallback.
//
// The adjoint runs the steps transposed, the last bounce first. Every sum runs in a fixed order (no
// floating-point atomics; theta's sums in double), so a gradient is the same bits call after call and
// whatever the checkpointing. The forward keeps each bounce's light atlas when the checkpoint budget
// allows; with fewer checkpoints than bounces the backward recomputes the missing atlases from the
// nearest earlier checkpoint.
#include <cub/device/device_radix_sort.cuh>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <memory>
#include <vector>

#include "../../include/lightbaker.h"
#include "lb_device.cuh"
#include "lb_kernels.h"
#include "lb_post.h"
#include "lb_texel.cuh"
#include "plan.h"

using lbplan::ck;
using lbplan::DBuf;

namespace lbd {

// theta: albedo (3 a material), zenith, horizon, ground (3 each), the sun's scale
struct Theta {
    const float *t;
    uint32_t M;
    __device__ __forceinline__ float3 albedo(uint32_t m) const { return mk(t[3 * m], t[3 * m + 1], t[3 * m + 2]); }
    __device__ __forceinline__ float3 zenith() const { return mk(t[3 * M], t[3 * M + 1], t[3 * M + 2]); }
    __device__ __forceinline__ float3 horizon() const { return mk(t[3 * M + 3], t[3 * M + 4], t[3 * M + 5]); }
    __device__ __forceinline__ float3 ground() const { return mk(t[3 * M + 6], t[3 * M + 7], t[3 * M + 8]); }
    __device__ __forceinline__ float sun() const { return t[3 * M + 9]; }
    // the fallback light, as the host derives it from the sky (bake.rs:150-152)
    __device__ __forceinline__ float3 fallback() const {
        float3 z = zenith(), h = horizon();
        return mk(((z.x + h.x) * 0.5f) * PI, ((z.y + h.y) * 0.5f) * PI, ((z.z + h.z) * 0.5f) * PI);
    }
};

constexpr uint32_t LIT_NONE = 0xffffffffu, UNLIT = 0xfffffffeu;

// The records against the light and theta: each gathered texel's gather result, its terms summed in ray
// order as the gather pass sums them (trace.wgsl:258-269); a thread an item, reading its records in turn.
__global__ void k_eval(const uint2 *rec, const uint32_t *n_dev, uint32_t n_host, uint32_t rays, const float4 *light,
                       uint32_t n_light, Theta th, float4 *out, uint32_t part, uint32_t parts) {
    uint32_t lo, n;
    item_part(n_dev ? *n_dev : n_host, part, parts, lo, n);
    const float frays = __uint2float_rn(rays);
    const float3 zen = th.zenith(), hor = th.horizon(), gro = th.ground(), fb = th.fallback();
    for (uint32_t k = lo + blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const uint2 *rk = rec + size_t(k) * rays;
        float3 sum = mk(0.f, 0.f, 0.f);
        uint32_t nback = 0;
        for (uint32_t r = 0; r < rays; r++) {
            uint2 q = __ldg(&rk[r]);
            uint32_t kind = q.x >> 30;
            if (kind == KIND_SKY) {
                // trace.wgsl:63-66
                float y = __uint_as_float(q.y);
                sum = add(sum, y < 0.0f ? gro : add(scl(hor, 1.0f - y), scl(zen, y)));
            } else if (kind == KIND_BACK) {
                nback++;
            } else {
                uint32_t m = q.x & 0x3fffffffu;
                float3 al = m < th.M ? th.albedo(m) : mk(0.f, 0.f, 0.f);
                float3 e = fb;
                if (q.y < n_light) {
                    float4 l = __ldg(&light[q.y]);
                    if (l.w > 0.5f) e = mk(l.x, l.y, l.z);
                }
                sum = add(sum, mulv(mk(al.x / PI, al.y / PI, al.z / PI), e));
            }
        }
        float3 e = scl(sum, PI);
        out[k] = make_float4(e.x / frays, e.y / frays, e.z / frays, __uint2float_rn(nback) / frays);
    }
}

// write_light (bake.rs:434-444) with the direct light scaled by the sun's theta: the atlas holds a known
// texel's direct plus (after the first bounce) indirect light
__global__ void k_write_light(PostArgs a, const uint8_t *kb, const float4 *dl0, Theta th, const float4 *ind,
                              float4 *light) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n_texels) return;
    const DTile t = a.tiles[find_tile(a.tiles, a.n_tiles, i)];
    uint32_t li = i - t.off, x = li % t.w, y = li / t.w;
    float s = th.sun();
    float4 d0 = dl0[i];
    float4 d = make_float4(s * d0.x, s * d0.y, s * d0.z, 0.f);
    float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
    if (kb[i] >= 1) {
        if (ind) {
            float4 e = ind[i];
            v = make_float4(d.x + e.x, d.y + e.y, d.z + e.z, 1.0f);
        } else {
            v = make_float4(d.x, d.y, d.z, 1.0f);
        }
    }
    light[size_t(t.y + y) * a.aw + t.x + x] = v;
}

// the last bounce's light as the texels' indirect, the fallback texels' own kept
__global__ void k_final_ind(uint32_t n, const uint8_t *state, const float4 *e, const float4 *fixed_ind, float4 *ind) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    ind[i] = state[i] == 5 ? fixed_ind[i] : e ? e[i] : make_float4(0.f, 0.f, 0.f, 0.f);
}

// known during the bounces: the final flags less the fallback's
__global__ void k_known_bounce(uint32_t n, const uint8_t *known, const uint8_t *state, uint8_t *kb) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) kb[i] = state[i] == 5 ? 0 : known[i];
}

// ---- the records' order for the adjoint ----

// sort keys: a lit surface record by its atlas texel; one that takes the fallback, or sky, after them; back
// faces and unknown materials (no term) last
__global__ void k_record_keys(const uint2 *rec, uint64_t n_rec, const float4 *light, uint32_t n_light, uint32_t M,
                              uint32_t *keys, uint32_t *vals) {
    for (uint64_t r = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; r < n_rec; r += uint64_t(gridDim.x) * blockDim.x) {
        uint2 q = rec[r];
        uint32_t kind = q.x >> 30, key = LIT_NONE;
        if (kind == KIND_SKY) key = UNLIT;
        else if (kind == KIND_SURFACE && (q.x & 0x3fffffffu) < M)
            key = (q.y < n_light && light[q.y].w > 0.5f) ? q.y : UNLIT;
        keys[r] = key;
        vals[r] = uint32_t(r);
    }
}

// the sorted records: x = kind << 30 | item, y = material (surface) or the direction's y (sky)
__global__ void k_record_sorted(const uint2 *rec, const uint32_t *vals, uint64_t n, uint32_t rays, uint2 *sorted) {
    for (uint64_t q = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; q < n; q += uint64_t(gridDim.x) * blockDim.x) {
        uint32_t r = vals[q];
        uint2 v = rec[r];
        uint32_t kind = v.x >> 30;
        sorted[q] = make_uint2((kind << 30) | (r / rays), kind == KIND_SKY ? v.y : (v.x & 0x3fffffffu));
    }
}

// offs[l] = the first sorted record whose key is >= l, for l = 0..n_light, then the first UNLIT and the
// first LIT_NONE key
__global__ void k_record_offsets(const uint32_t *keys, uint64_t n, uint32_t n_light, uint64_t *offs) {
    uint32_t l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l > n_light + 2) return;
    uint32_t want = l <= n_light ? l : l == n_light + 1 ? UNLIT : LIT_NONE;
    uint64_t lo = 0, hi = n;
    while (lo < hi) {
        uint64_t mid = (lo + hi) >> 1;
        if (keys[mid] < want) lo = mid + 1;
        else hi = mid;
    }
    offs[l] = lo;
}

// ---- transposes: a thread writes its own texel's gradient, summing what it fed in a fixed order ----

// the composite's block average (bake.rs:364-391): a texel's share of its block's gradient; the fallback
// texels' share too when the volume is differentiated (`fallback`; k_vfallback_t takes it from there),
// else their light is fixed and gets none
__global__ void k_composite_t(PostArgs a, CompositeArgs c, const float4 *g_blocks, float4 *g_ind, int fallback) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n_texels) return;
    float4 g = make_float4(0.f, 0.f, 0.f, 0.f);
    if (c.known[i] != 0 && (c.state[i] != 5 || fallback)) {
        const DTile t = a.tiles[find_tile(a.tiles, a.n_tiles, i)];
        uint32_t li = i - t.off, ax = t.x + li % t.w, ay = t.y + li / t.w;
        uint32_t bx = ax / c.ds, by = ay / c.ds;
        float s3 = 0.0f;
        for (uint32_t y = by * c.ds; y < min((by + 1) * c.ds, c.ah); y++)
            for (uint32_t x = bx * c.ds; x < min((bx + 1) * c.ds, c.aw); x++) {
                uint32_t j = c.owner[size_t(y) * c.aw + x];
                if (j != NONE && c.known[j] != 0) s3 += c.known[j] == 2 ? 1.0f : 1e-3f;
            }
        float k = c.known[i] == 2 ? 1.0f : 1e-3f;
        float4 gb = g_blocks[by * c.iw + bx];
        g = make_float4(gb.x * k / s3, gb.y * k / s3, gb.z * k / s3, 0.f);
    }
    g_ind[i] = g;
}

__device__ __forceinline__ int flagged_around(const uint8_t *was, uint32_t i, uint32_t iw, uint32_t ih) {
    uint32_t x = i % iw, y = i / iw;
    int n = 0;
    for (uint32_t yy = y > 0 ? y - 1 : 0; yy < min(y + 2, ih); yy++)
        for (uint32_t xx = x > 0 ? x - 1 : 0; xx < min(x + 2, iw); xx++) n += was[yy * iw + xx] ? 1 : 0;
    return n;
}

// A texel's part in one dilation pass (bake.rs:394-421), from the pass's starting flags: 0x80 flagged, else
// the flagged neighbours it averages (0: none, it keeps its value)
__global__ void k_dilate_plan(const uint8_t *was, uint8_t *plan, uint32_t iw, uint32_t ih) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= iw * ih) return;
    plan[i] = was[i] ? 0x80 : uint8_t(flagged_around(was, i, iw, ih));
}

// one dilation pass transposed
__global__ void k_dilate_t(const uint8_t *plan, const float4 *g_out, float4 *g_in, uint32_t iw, uint32_t ih) {
    uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= iw * ih) return;
    float4 g = make_float4(0.f, 0.f, 0.f, 0.f);
    uint8_t pj = plan[j];
    if (pj & 0x80) {
        g = g_out[j];
        uint32_t x = j % iw, y = j / iw;
        for (uint32_t yy = y > 0 ? y - 1 : 0; yy < min(y + 2, ih); yy++)
            for (uint32_t xx = x > 0 ? x - 1 : 0; xx < min(x + 2, iw); xx++) {
                uint32_t i = yy * iw + xx;
                uint8_t pi = plan[i];
                if (pi & 0x80) continue;
                float f = float(pi);
                float4 go = g_out[i];
                g.x += go.x / f, g.y += go.y / f, g.z += go.z / f;
            }
    } else if (pj == 0) {
        g = g_out[j];
    }
    g_in[j] = g;
}

// the dilation's flags alone
__global__ void k_dilate_mask(const uint8_t *was, uint8_t *now, uint32_t iw, uint32_t ih) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= iw * ih) return;
    now[i] = was[i] || flagged_around(was, i, iw, ih) > 0;
}

// How a texel not yet filled fills in one ring (filter.rs:58-94): 1 from its own chart's flagged
// neighbours, 2 from any flagged neighbour (a texel of no chart), 0 not; n the neighbours averaged.
__device__ __forceinline__ int fill_mode(const PostArgs &a, const DTile &t, const uint8_t *was, uint32_t i, int x, int y,
                                         int &n) {
    uint32_t ci = a.chart[i];
    int no = 0, na = 0;
    for (int yy = y > 0 ? y - 1 : 0; yy < min(y + 2, int(t.h)); yy++)
        for (int xx = x > 0 ? x - 1 : 0; xx < min(x + 2, int(t.w)); xx++) {
            uint32_t q = t.off + uint32_t(yy) * t.w + uint32_t(xx);
            if (!was[q]) continue;
            if (ci != NONE && a.chart[q] == ci) no++;
            else na++;
        }
    if (no > 0) {
        n = no;
        return 1;
    }
    if (na > 0 && ci == NONE) {
        n = na;
        return 2;
    }
    n = 0;
    return 0;
}

// A texel's part in one fill ring, from the ring's starting flags: 0x80 flagged; else mode << 4 | n
// (fill_mode), and its flag for the next ring
__global__ void k_fill_plan(PostArgs a, const uint8_t *was, uint8_t *plan, uint8_t *now) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n_texels) return;
    if (was[i]) {
        plan[i] = 0x80;
        now[i] = 1;
        return;
    }
    const DTile t = a.tiles[find_tile(a.tiles, a.n_tiles, i)];
    int li = int(i - t.off), n;
    int mode = fill_mode(a, t, was, i, li % int(t.w), li / int(t.w), n);
    plan[i] = uint8_t((mode << 4) | n);
    now[i] = mode != 0;
}

// a flagged texel that a neighbour fills from in this ring gets 0x40 too (the others keep their value
// and feed nothing: the transpose copies them)
__global__ void k_fill_plan_mark(PostArgs a, uint8_t *plan) {
    uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= a.n_texels || !(plan[j] & 0x80)) return;
    const DTile t = a.tiles[find_tile(a.tiles, a.n_tiles, j)];
    int lj = int(j - t.off), x = lj % int(t.w), y = lj / int(t.w);
    bool feeds = false;
    for (int yy = y > 0 ? y - 1 : 0; yy < min(y + 2, int(t.h)); yy++)
        for (int xx = x > 0 ? x - 1 : 0; xx < min(x + 2, int(t.w)); xx++) {
            uint8_t pi = plan[t.off + uint32_t(yy) * t.w + uint32_t(xx)];
            if (!(pi & 0x80) && (pi >> 4) != 0) feeds = true;
        }
    if (feeds) plan[j] = 0xc0;
}

// one fill ring transposed
__global__ void k_fill_t(PostArgs a, const uint8_t *plan, const float4 *g_out, float4 *g_in) {
    uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= a.n_texels) return;
    float4 g = make_float4(0.f, 0.f, 0.f, 0.f);
    uint8_t pj = plan[j];
    if (pj == 0x80) {
        g = g_out[j];
    } else if (pj & 0x80) {
        g = g_out[j];
        const DTile t = a.tiles[find_tile(a.tiles, a.n_tiles, j)];
        int lj = int(j - t.off), x = lj % int(t.w), y = lj / int(t.w);
        uint32_t cj = a.chart[j];
        for (int yy = y > 0 ? y - 1 : 0; yy < min(y + 2, int(t.h)); yy++)
            for (int xx = x > 0 ? x - 1 : 0; xx < min(x + 2, int(t.w)); xx++) {
                uint32_t i = t.off + uint32_t(yy) * t.w + uint32_t(xx);
                uint8_t pi = plan[i];
                int mode = (pi & 0x80) ? 0 : pi >> 4;
                if (mode == 2 || (mode == 1 && cj == a.chart[i])) {
                    float4 go = g_out[i];
                    float f = float(pi & 15);
                    g.x += go.x / f, g.y += go.y / f, g.z += go.z / f;
                }
            }
    } else if ((pj >> 4) == 0) {
        g = g_out[j];
    }
    g_in[j] = g;
}

// the bounce smoothing's weight sums (filter.rs:20-53 over the gathered texels)
__global__ void k_smooth_wsum(PostArgs a, int r, const float *w, float *wsum) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n_texels) return;
    float s = 0.0f;
    if (a.gathered[i] && r > 0) {
        const DTile t = a.tiles[find_tile(a.tiles, a.n_tiles, i)];
        int li = int(i - t.off), x = li % int(t.w), y = li / int(t.w);
        for (int yy = y > r ? y - r : 0; yy < min(y + r + 1, int(t.h)); yy++)
            for (int xx = x > r ? x - r : 0; xx < min(x + r + 1, int(t.w)); xx++) {
                uint32_t j = t.off + uint32_t(yy) * t.w + uint32_t(xx);
                if (!a.gathered[j] || !same(a.chart, a.tex, i, j)) continue;
                s += w[(yy - y + r) * (2 * r + 1) + (xx - x + r)];
            }
    }
    wsum[i] = s;
}

// the bounce smoothing transposed (the Gaussian is symmetric: w(-d) = w(d))
__global__ void k_smooth_t(PostArgs a, const float4 *g_out, int r, const float *w, const float *wsum, float4 *g_in) {
    uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= a.n_texels) return;
    float4 g = make_float4(0.f, 0.f, 0.f, 0.f);
    if (!a.gathered[j] || r == 0) {
        g = g_out[j];
    } else {
        const DTile t = a.tiles[find_tile(a.tiles, a.n_tiles, j)];
        int lj = int(j - t.off), x = lj % int(t.w), y = lj / int(t.w);
        for (int yy = y > r ? y - r : 0; yy < min(y + r + 1, int(t.h)); yy++)
            for (int xx = x > r ? x - r : 0; xx < min(x + r + 1, int(t.w)); xx++) {
                uint32_t i = t.off + uint32_t(yy) * t.w + uint32_t(xx);
                if (!a.gathered[i] || !same(a.chart, a.tex, i, j)) continue;
                float f = w[(yy - y + r) * (2 * r + 1) + (xx - x + r)] / wsum[i];
                float4 go = g_out[i];
                g.x += go.x * f, g.y += go.y * f, g.z += go.z * f;
            }
    }
    g_in[j] = g;
}

// the scatter of gather results (bake.rs:309-316) transposed
__global__ void k_scatter_t(const uint32_t *idx, uint32_t n, const float4 *g_e, float4 *g_res) {
    uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) g_res[k] = g_e[idx[k]];
}

// write_light transposed: a known texel's atlas gradient goes to its direct light (summed over the
// bounces) and to the previous bounce's indirect
__global__ void k_light_t(PostArgs a, const uint8_t *kb, const float4 *g_light, float4 *g_dl, float4 *g_ind) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n_texels) return;
    float4 g = make_float4(0.f, 0.f, 0.f, 0.f);
    if (kb[i] >= 1) {
        const DTile t = a.tiles[find_tile(a.tiles, a.n_tiles, i)];
        uint32_t li = i - t.off;
        g = g_light[size_t(t.y + li / t.w) * a.aw + t.x + li % t.w];
    }
    float4 d = g_dl[i];
    g_dl[i] = make_float4(d.x + g.x, d.y + g.y, d.z + g.z, 0.f);
    if (g_ind) g_ind[i] = g;
}

// Theta's gradient slots in a block's partial sums: albedo (3 a material of this chunk), then zenith,
// horizon, ground and fallback (3 each).
constexpr int FIXED_SLOTS = 12;

// Theta's per-block partial sums: each warp adds into its own row of slots ([warp][3 mc]; one lane a
// component, the warp's staged values in lane order), then each slot is summed over the block's warps in
// warp order: the same bits every launch.
constexpr int TW = 8;  // warps a block in the adjoint's reduction kernels (256 threads)

__device__ __forceinline__ void warp_stage_add(double *row, uint32_t m0, uint32_t mc, const uint32_t *st_m,
                                               const double (*st_v)[3], int lane) {
    __syncwarp();
    if (lane < 3)
        for (int j = 0; j < 32; j++) {
            uint32_t m = st_m[j];
            if (m >= m0 && m < m0 + mc) row[3 * (m - m0) + lane] += st_v[j][lane];
        }
    __syncwarp();
}

__device__ __forceinline__ void block_rows_out(const double *acc, int S, const double *fixed, double *partial) {
    __syncthreads();
    const int slots = S + FIXED_SLOTS;
    for (int s = threadIdx.x; s < slots; s += blockDim.x) {
        double v = 0.0;
        if (s < S)
            for (int w = 0; w < TW; w++) v += acc[size_t(w) * S + s];
        else if (fixed)
            for (int l = 0; l < int(blockDim.x); l++) v += fixed[size_t(l) * FIXED_SLOTS + (s - S)];
        partial[size_t(blockIdx.x) * slots + s] = v;
    }
}

// The lit records, atlas texel by atlas texel (sorted; a lane a texel, 32 consecutive texels a warp): the
// atlas gradient (the texel's light fed each record's term al / pi * e) and the albedo gradients of the
// chunk's materials (the record's weight c = g / rays times its light). A texel's records are a chart's,
// so nearly always of one material: its weights are summed and multiplied by its light once; a texel
// with records of several materials is walked again record by record, lane by lane.
__global__ void __launch_bounds__(256) k_lit_t(const uint64_t *offs, const uint2 *sorted, uint32_t n_light,
                                               const float4 *light, Theta th, uint32_t m0, uint32_t mc, uint32_t rays,
                                               const float4 *g_res, float4 *g_light, int write_light,
                                               double *partial) {
    extern __shared__ double acc[];  // [TW][3 mc]
    __shared__ double st_v[TW][32][3];
    __shared__ uint32_t st_m[TW][32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, S = 3 * int(mc);
    double *row = acc + size_t(w) * S;
    for (int q = lane; q < S; q += 32) row[q] = 0.0;
    const float frays = __uint2float_rn(rays);
    const uint32_t stride = gridDim.x * TW * 32;
    for (uint32_t base = (blockIdx.x * TW + w) * 32; base < n_light; base += stride) {
        uint32_t l = base + lane, mfirst = NONE;
        bool mixed = false;
        double vx = 0.0, vy = 0.0, vz = 0.0;
        float4 L = make_float4(0.f, 0.f, 0.f, 0.f);
        uint64_t b = 0, e = 0;
        if (l < n_light) {
            b = offs[l];
            e = offs[l + 1];
            if (b < e) {
                L = light[l];
                uint32_t mr = __ldg(&sorted[b]).y;
                mfirst = mr;
                float3 al = th.albedo(mr);
                float gx = 0.f, gy = 0.f, gz = 0.f;
                for (uint64_t q = b; q < e; q++) {
                    uint2 sr = __ldg(&sorted[q]);
                    if (sr.y != mr) {
                        mixed = true;
                        mr = sr.y;
                        al = th.albedo(mr);
                    }
                    float4 g = __ldg(&g_res[sr.x & 0x3fffffffu]);
                    float cx = g.x / frays, cy = g.y / frays, cz = g.z / frays;
                    gx += cx * al.x, gy += cy * al.y, gz += cz * al.z;
                    vx += double(cx), vy += double(cy), vz += double(cz);
                }
                if (write_light) g_light[l] = make_float4(gx, gy, gz, 0.f);
            } else if (write_light) {
                g_light[l] = make_float4(0.f, 0.f, 0.f, 0.f);
            }
        }
        st_m[w][lane] = mixed ? NONE : mfirst;
        st_v[w][lane][0] = vx * double(L.x);
        st_v[w][lane][1] = vy * double(L.y);
        st_v[w][lane][2] = vz * double(L.z);
        warp_stage_add(row, m0, mc, st_m[w], st_v[w], lane);
        unsigned mx = __ballot_sync(0xffffffffu, mixed);
        while (mx) {
            int src = __ffs(mx) - 1;
            mx &= mx - 1;
            if (lane == src)
                for (uint64_t q = b; q < e; q++) {
                    uint2 sr = sorted[q];
                    uint32_t m = sr.y;
                    if (m < m0 || m >= m0 + mc) continue;
                    float4 g = g_res[sr.x & 0x3fffffffu];
                    double *d = row + 3 * (m - m0);
                    d[0] += double(g.x / frays) * double(L.x);
                    d[1] += double(g.y / frays) * double(L.y);
                    d[2] += double(g.z / frays) * double(L.z);
                }
            __syncwarp();
        }
    }
    block_rows_out(acc, S, nullptr, partial);
}

// The sky records and the surface records that take the fallback light (a lane a record): the sky's
// gradients and the fallback's in each thread's own registers, the albedo gradients of the chunk's
// materials lit by the fallback staged a warp at a time.
__global__ void __launch_bounds__(256) k_unlit_t(const uint2 *sorted, uint64_t n, Theta th, uint32_t m0, uint32_t mc,
                                                 uint32_t rays, const float4 *g_res, int fixed_slots, double *partial) {
    extern __shared__ double acc[];  // [TW][3 mc]
    __shared__ double st_v[TW][32][3];
    __shared__ uint32_t st_m[TW][32];
    __shared__ double fixed[256 * FIXED_SLOTS];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, S = 3 * int(mc);
    double *row = acc + size_t(w) * S;
    for (int q = lane; q < S; q += 32) row[q] = 0.0;
    const double frays = double(rays), qq = 3.14159265358979323846 / frays;
    const float3 fb = th.fallback();
    double f[FIXED_SLOTS] = {0};
    const uint64_t stride = uint64_t(gridDim.x) * TW * 32;
    for (uint64_t base = (uint64_t(blockIdx.x) * TW + w) * 32; base < n; base += stride) {
        uint64_t r = base + lane;
        uint32_t mst = NONE;
        double v0 = 0.0, v1 = 0.0, v2 = 0.0;
        if (r < n) {
            uint2 sr = __ldg(&sorted[r]);
            uint32_t kind = sr.x >> 30;
            float4 g = __ldg(&g_res[sr.x & 0x3fffffffu]);
            if (kind == KIND_SKY) {
                double y = double(__uint_as_float(sr.y));
                if (y < 0.0) {
                    f[6] += g.x * qq, f[7] += g.y * qq, f[8] += g.z * qq;
                } else {
                    f[0] += g.x * qq * y, f[1] += g.y * qq * y, f[2] += g.z * qq * y;
                    f[3] += g.x * qq * (1.0 - y), f[4] += g.y * qq * (1.0 - y), f[5] += g.z * qq * (1.0 - y);
                }
            } else {
                float3 al = th.albedo(sr.y);
                f[9] += g.x * double(al.x) / frays, f[10] += g.y * double(al.y) / frays;
                f[11] += g.z * double(al.z) / frays;
                mst = sr.y;
                v0 = g.x * double(fb.x) / frays, v1 = g.y * double(fb.y) / frays, v2 = g.z * double(fb.z) / frays;
            }
        }
        st_m[w][lane] = mst;
        st_v[w][lane][0] = v0;
        st_v[w][lane][1] = v1;
        st_v[w][lane][2] = v2;
        warp_stage_add(row, m0, mc, st_m[w], st_v[w], lane);
    }
    for (int c = 0; c < FIXED_SLOTS; c++) fixed[size_t(threadIdx.x) * FIXED_SLOTS + c] = fixed_slots ? f[c] : 0.0;
    block_rows_out(acc, S, fixed, partial);
}

// the sun's gradient: the direct light is s * dl0, so d/ds = sum over texels of g_dl . dl0
__global__ void k_sun_t(uint32_t n, const float4 *g_dl, const float4 *dl0, double *partial) {
    __shared__ double acc[256];
    double v = 0.0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float4 g = g_dl[i], d = dl0[i];
        v += double(g.x) * d.x + double(g.y) * d.y + double(g.z) * d.z;
    }
    acc[threadIdx.x] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int l = 0; l < int(blockDim.x); l++) t += acc[l];
        partial[blockIdx.x] = t;
    }
}

// Theta's gradient from the partial sums, in a fixed order: pass by pass (bounce, kind, material chunk),
// block by block.
struct PartialSet {
    const double *p;   // [blocks][slots]
    uint32_t m0, mc;   // the chunk's materials
    int fixed;         // holds the fixed slots
};

// A block an output: its threads take the (set, block) rows in a fixed stride, then a fixed tree.
__global__ void __launch_bounds__(256) k_theta_final(const PartialSet *sets, int n_sets, int blocks, const double *sun,
                                                     int sun_blocks, uint32_t M, float *g_theta) {
    __shared__ double part[256];
    // output j reads slot(s): albedo 3m+c; zenith/horizon/ground; the fallback feeds zenith and horizon;
    // the sun its own partials
    const uint32_t j = blockIdx.x;
    double v = 0.0;
    if (j == 3 * M + 9) {
        for (int b = threadIdx.x; b < sun_blocks; b += blockDim.x) v += sun[b];
    } else {
        const int rows = n_sets * blocks;
        for (int q = threadIdx.x; q < rows; q += blockDim.x) {
            const PartialSet &ps = sets[q / blocks];
            int b = q % blocks, slots = 3 * int(ps.mc) + FIXED_SLOTS;
            const double *row = ps.p + size_t(b) * slots;
            if (j < 3 * M) {
                uint32_t m = j / 3;
                if (m >= ps.m0 && m < ps.m0 + ps.mc) v += row[j - 3 * ps.m0];
            } else if (ps.fixed) {
                uint32_t c = j - 3 * M;  // 0..8: zenith, horizon, ground
                v += row[3 * ps.mc + c];
                if (c < 6) v += row[3 * ps.mc + 9 + c % 3] * (0.5 * 3.14159265358979323846);
            }
        }
    }
    part[threadIdx.x] = v;
    __syncthreads();
    for (int h = blockDim.x / 2; h > 0; h >>= 1) {
        if (int(threadIdx.x) < h) part[threadIdx.x] += part[threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0) g_theta[j] = float(part[0]);
}

// ---- the volume's share: the probes the fallback texels read (bake.rs:335-359, volume.rs:86-147) ----

// The volume records against the last bounce's light and theta: each probe's L1 harmonics, its terms
// summed in ray order as the volume pass sums them (trace.wgsl:272-324), a thread a probe; the sun's share
// and the back-face share (geometry alone) as the bake wrote them (`raw`).
__global__ void k_veval(const uint2 *rec, const float4 *items, const uint32_t *slot, uint32_t n, uint32_t rays,
                        uint32_t seed, const float4 *light, uint32_t n_light, Theta th, const float4 *raw,
                        float4 *probes) {
    const float frays = __uint2float_rn(rays);
    const float3 zen = th.zenith(), hor = th.horizon(), gro = th.ground(), fb = th.fallback();
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const uint32_t key = __float_as_uint(items[4 * k + 1].w) * 7919u + 77u;
        const float s1 = rnd(key, 29u, seed), s2 = rnd(key, 31u, seed);
        float3 l0 = mk(0.f, 0.f, 0.f), l1x = l0, l1y = l0, l1z = l0;
        const uint2 *rk = rec + size_t(k) * rays;
        for (uint32_t r = 0; r < rays; r++) {
            const float3 d = volume_ray(r, frays, s1, s2);
            const uint2 q = __ldg(&rk[r]);
            const uint32_t kind = q.x >> 30;
            float3 l = mk(0.f, 0.f, 0.f);
            if (kind == KIND_SKY) {
                l = d.y < 0.0f ? gro : add(scl(hor, 1.0f - d.y), scl(zen, d.y));  // trace.wgsl:63-66
            } else if (kind == KIND_SURFACE) {
                const uint32_t m = q.x & 0x3fffffffu;
                const float3 al = m < th.M ? th.albedo(m) : mk(0.f, 0.f, 0.f);
                float3 e = fb;
                if (q.y < n_light) {
                    const float4 L = __ldg(&light[q.y]);
                    if (L.w > 0.5f) e = mk(L.x, L.y, L.z);
                }
                l = mulv(mk(al.x / PI, al.y / PI, al.z / PI), e);  // trace.wgsl:133-148
            }
            const float3 lw = scl(l, 0.488603f);
            l0 = add(l0, scl(l, 0.282095f));
            l1x = add(l1x, scl(lw, d.x));
            l1y = add(l1y, scl(lw, d.y));
            l1z = add(l1z, scl(lw, d.z));
        }
        const float w = 4.0f * PI / frays;
        const uint32_t dst = slot[k];
        const float3 a[4] = {scl(l0, w), scl(l1x, w), scl(l1y, w), scl(l1z, w)};
        for (int c = 0; c < 4; c++)
            probes[4 * dst + c] = make_float4(a[c].x, a[c].y, a[c].z, raw[4 * dst + c].w);
    }
}

// The trilinear corners a fallback texel reads (volume.rs:125-137), as the fallback computes them.
struct VolumeGrid {
    float3 origin;
    float step;
    uint32_t nx, ny, nz;
};
__device__ __forceinline__ void fallback_corners(const PostArgs &a, uint32_t i, const VolumeGrid &v, uint32_t j[8],
                                                 float w[8]) {
    const float4 n4 = a.tex[4 * i + 1];
    float3 q = mk(a.posg[i].x + n4.x * 0.15f, a.posg[i].y + n4.y * 0.15f, a.posg[i].z + n4.z * 0.15f);
    float fx = (q.x - v.origin.x) / v.step, fy = (q.y - v.origin.y) / v.step, fz = (q.z - v.origin.z) / v.step;
    fx = fminf(fmaxf(fx, 0.0f), float(v.nx - 1));
    fy = fminf(fmaxf(fy, 0.0f), float(v.ny - 1));
    fz = fminf(fmaxf(fz, 0.0f), float(v.nz - 1));
    uint32_t x0 = min(uint32_t(fx), v.nx - 2), y0 = min(uint32_t(fy), v.ny - 2), z0 = min(uint32_t(fz), v.nz - 2);
    float tx = fx - float(x0), ty = fy - float(y0), tz = fz - float(z0);
    for (int k = 0; k < 8; k++) {
        int dx = k & 1, dy = (k >> 1) & 1, dz = (k >> 2) & 1;
        w[k] = ((dx ? tx : 1.0f - tx) * (dy ? ty : 1.0f - ty)) * (dz ? tz : 1.0f - tz);
        j[k] = ((y0 + dy) * v.nz + (z0 + dz)) * v.nx + (x0 + dx);
    }
}

// The fallback texels' light from the filled probes (bake.rs:337-359 through volume.rs:125-147), the
// arithmetic of the bake's own fallback, a thread a fallback texel.
__global__ void k_vfallback(PostArgs a, const uint32_t *f5, uint32_t n5, const float4 *probes, VolumeGrid v,
                            float4 *ind) {
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n5) return;
    const uint32_t i = f5[q];
    uint32_t j[8];
    float w[8];
    fallback_corners(a, i, v, j, w);
    float p4[16] = {0};
    for (int k = 0; k < 8; k++)
        for (int c = 0; c < 4; c++) {
            float4 pv = probes[4 * j[k] + c];
            p4[4 * c] += pv.x * w[k], p4[4 * c + 1] += pv.y * w[k], p4[4 * c + 2] += pv.z * w[k], p4[4 * c + 3] += pv.w * w[k];
        }
    const float4 n4 = a.tex[4 * i + 1];
    const float PI32 = 3.14159274101257324f;
    float a0 = PI32 * 0.282095f, a1 = 2.0f * PI32 / 3.0f * 0.488603f;
    float e[3];
    for (int c = 0; c < 3; c++)
        e[c] = 0.5f * a0 * p4[c] + 0.5f * fmaxf(a0 * p4[c] + a1 * ((p4[4 + c] * n4.x + p4[8 + c] * n4.y) + p4[12 + c] * n4.z), 0.0f);
    ind[i] = make_float4(e[0], e[1], e[2], 0.0f);
}

// The fallback transposed, a thread a fallback texel: its indirect's gradient (taken out of g_ind, where
// the composite's transpose left it) into the gradient of the four interpolated coefficients (rgb each),
// the cosine lobe's clamp at 0 read from the forward's probes.
__global__ void k_vfallback_t(PostArgs a, const uint32_t *f5, uint32_t n5, const float4 *probes, VolumeGrid v,
                              float4 *g_ind, float4 *gp) {
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n5) return;
    const uint32_t i = f5[q];
    const float4 g = g_ind[i];
    g_ind[i] = make_float4(0.f, 0.f, 0.f, 0.f);  // a fallback texel's light is not the bounces'
    uint32_t j[8];
    float w[8];
    fallback_corners(a, i, v, j, w);
    float p4[16] = {0};
    for (int k = 0; k < 8; k++)
        for (int c = 0; c < 4; c++) {
            float4 pv = probes[4 * j[k] + c];
            p4[4 * c] += pv.x * w[k], p4[4 * c + 1] += pv.y * w[k], p4[4 * c + 2] += pv.z * w[k], p4[4 * c + 3] += pv.w * w[k];
        }
    const float4 n4 = a.tex[4 * i + 1];
    const float PI32 = 3.14159274101257324f;
    const float a0 = PI32 * 0.282095f, a1 = 2.0f * PI32 / 3.0f * 0.488603f;
    const float gc[3] = {g.x, g.y, g.z};
    float o[4][3];
    for (int c = 0; c < 3; c++) {
        const float arg = a0 * p4[c] + a1 * ((p4[4 + c] * n4.x + p4[8 + c] * n4.y) + p4[12 + c] * n4.z);
        const float on = arg > 0.0f ? 1.0f : 0.0f;
        o[0][c] = gc[c] * (0.5f * a0 + on * 0.5f * a0);
        o[1][c] = gc[c] * on * 0.5f * a1 * n4.x;
        o[2][c] = gc[c] * on * 0.5f * a1 * n4.y;
        o[3][c] = gc[c] * on * 0.5f * a1 * n4.z;
    }
    for (int k = 0; k < 4; k++) gp[4 * size_t(q) + k] = make_float4(o[k][0], o[k][1], o[k][2], 0.f);
}

// The interpolation transposed, a thread a probe: the corner weights of the fallback texels that read it
// (listed at create, in texel order) times their coefficients' gradients.
__global__ void k_vprobe_t(const uint32_t *off, const uint32_t *who, const float *wt, uint32_t n_probes,
                           const float4 *gp, float4 *g_probes) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n_probes) return;
    float3 s[4] = {mk(0.f, 0.f, 0.f), mk(0.f, 0.f, 0.f), mk(0.f, 0.f, 0.f), mk(0.f, 0.f, 0.f)};
    for (uint32_t e = off[j]; e < off[j + 1]; e++) {
        const uint32_t q = who[e];
        const float w = wt[e];
        for (int k = 0; k < 4; k++) s[k] = add(s[k], scl(xyz(gp[4 * size_t(q) + k]), w));
    }
    for (int k = 0; k < 4; k++) g_probes[4 * size_t(j) + k] = make_float4(s[k].x, s[k].y, s[k].z, 0.f);
}

// One ring of the volume's fill (volume.rs:88-121) transposed, a thread a probe: a probe known before the
// ring keeps its own value and feeds each unknown neighbour that the ring fills (an average of its known
// neighbours); an unknown probe the ring leaves unknown keeps its own. `was`: the known flags before it.
__global__ void k_vfill_t(const uint8_t *was, const float4 *g_dst, float4 *g_src, uint32_t nx, uint32_t ny,
                          uint32_t nz) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t total = nx * ny * nz;
    if (j >= total) return;
    const int D[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
    auto neighbour = [&](uint32_t k, int d, uint32_t &out) {
        int x = int(k % nx), z = int((k / nx) % nz), y = int(k / (nx * nz));
        int xx = x + D[d][0], yy = y + D[d][1], zz = z + D[d][2];
        if (xx < 0 || yy < 0 || zz < 0 || xx >= int(nx) || yy >= int(ny) || zz >= int(nz)) return false;
        out = (uint32_t(yy) * nz + uint32_t(zz)) * nx + uint32_t(xx);
        return true;
    };
    auto known_count = [&](uint32_t k) {
        int c = 0;
        uint32_t m;
        for (int d = 0; d < 6; d++)
            if (neighbour(k, d, m) && was[m]) c++;
        return c;
    };
    float4 g[4];
    const bool keeps = was[j] || known_count(j) == 0;
    for (int q = 0; q < 4; q++) g[q] = keeps ? g_dst[4 * j + q] : make_float4(0.f, 0.f, 0.f, 0.f);
    if (was[j])
        for (int d = 0; d < 6; d++) {
            uint32_t k;
            if (!neighbour(j, d, k) || was[k]) continue;
            const int c = known_count(k);
            if (c == 0) continue;
            const float f = float(c);
            for (int q = 0; q < 4; q++) {
                float4 v = g_dst[4 * k + q];
                g[q] = make_float4(g[q].x + v.x / f, g[q].y + v.y / f, g[q].z + v.z / f, 0.f);
            }
        }
    for (int q = 0; q < 4; q++) g_src[4 * j + q] = g[q];
}

// The probes each fallback texel reads and their weights (8 a texel, corner order), for the per-probe lists.
__global__ void k_vcorners(PostArgs a, const uint32_t *f5, uint32_t n5, VolumeGrid v, uint32_t *j8, float *w8) {
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n5) return;
    fallback_corners(a, f5[q], v, j8 + 8 * size_t(q), w8 + 8 * size_t(q));
}

// The L1 projection transposed, a thread a volume ray: the gradient of the ray's radiance from its probe's
// coefficient gradients (w * basis(d)), divided by pi: as the gather's records weigh their terms (pi / rays),
// so the records' transposes (k_lit_t, k_unlit_t with one ray an item) give the volume rays' gradients.
__global__ void k_vrec_t(const float4 *items, const uint32_t *slot, uint32_t n, uint32_t rays, uint32_t seed,
                         const float4 *g_probes, float4 *vg) {
    const uint64_t total = uint64_t(n) * rays;
    const float frays = __uint2float_rn(rays), w = 4.0f * PI / frays;
    for (uint64_t q = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; q < total; q += uint64_t(gridDim.x) * blockDim.x) {
        const uint32_t k = uint32_t(q / rays), r = uint32_t(q % rays);
        const uint32_t key = __float_as_uint(items[4 * k + 1].w) * 7919u + 77u;
        const float3 d = volume_ray(r, frays, rnd(key, 29u, seed), rnd(key, 31u, seed));
        const uint32_t j = slot[k];
        const float3 g0 = xyz(g_probes[4 * j]), gx = xyz(g_probes[4 * j + 1]), gy = xyz(g_probes[4 * j + 2]),
                     gz = xyz(g_probes[4 * j + 3]);
        const float3 g1 = add(add(scl(gx, d.x), scl(gy, d.y)), scl(gz, d.z));
        const float3 gl = scl(add(scl(g0, 0.282095f), scl(g1, 0.488603f)), w / PI);
        vg[q] = make_float4(gl.x, gl.y, gl.z, 0.f);
    }
}

// write_light transposed for the last bounce's light, which only the volume reads: added to the direct
// light's gradient and to the last bounce's indirect's (the composite's transpose wrote it first).
__global__ void k_light_add_t(PostArgs a, const uint8_t *kb, const float4 *g_light, float4 *g_dl, float4 *g_ind) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n_texels || kb[i] < 1) return;
    const DTile t = a.tiles[find_tile(a.tiles, a.n_tiles, i)];
    uint32_t li = i - t.off;
    const float4 g = g_light[size_t(t.y + li / t.w) * a.aw + t.x + li % t.w];
    float4 d = g_dl[i];
    g_dl[i] = make_float4(d.x + g.x, d.y + g.y, d.z + g.z, 0.f);
    if (g_ind) {
        float4 e = g_ind[i];
        g_ind[i] = make_float4(e.x + g.x, e.y + g.y, e.z + g.z, 0.f);
    }
}

}  // namespace lbd

cudaError_t lb_eval_records(const uint2 *rec, const uint32_t *n_dev, uint32_t n_host, uint32_t rays,
                            const float4 *light, uint32_t n_light, const float *theta, uint32_t n_mats, float4 *out,
                            int sms, cudaStream_t stream, uint32_t part, uint32_t parts) {
    lbd::k_eval<<<sms * 16, 128, 0, stream>>>(rec, n_dev, n_host, rays, light, n_light, lbd::Theta{theta, n_mats}, out,
                                              part, parts);
    return cudaGetLastError();
}

namespace {

inline dim3 tg(uint64_t n) { return dim3(uint32_t((n + 255) / 256)); }

constexpr int T_THREADS = 32 * lbd::TW;  // threads of the adjoint's reduction kernels
constexpr size_t T_SMEM = 128 * 1024;    // their dynamic shared memory at most

}  // namespace

struct lb_transport {
    lb_plan *plan = nullptr;
    lb_gpu *g = nullptr;
    uint32_t M = 0, B = 0, n_gath = 0, rays = 0, n_light = 0, n_tex = 0, iw = 0, ih = 0;
    uint32_t K = 0;                      // checkpoints kept by the forward
    std::vector<uint32_t> ck_bounce;     // the bounce each checkpoint holds
    int rings = 0, r = 0, blocks = 0, sun_blocks = 0;
    uint32_t mc = 0;                     // materials a reduction pass covers
    uint64_t n_rec = 0, n_lit = 0, unlit0 = 0, n_unlit = 0;
    std::vector<float> theta0;
    PostArgs a{};
    CompositeArgs c{};
    const uint2 *records = nullptr;  // the plan's gather records, [item][ray]
    DBuf theta, sorted, offs, kb, dl0, fixed_ind, masks, wsum, has0, has1, ckpt, work, res, e0, e1, fk_a, fk_b,
        ind, out_atlas, out_tmp, out_has, out_has_b, out_direct, out_validity;
    DBuf g_in, g_blocks_a, g_blocks_b, g_ind, g_a, g_b, g_res, g_light, g_dl, partials, sun_partials, sets_d, g_theta;
    std::vector<lbd::PartialSet> sets;
    // the volume's share (a scene with a volume and texels it lights, state 5): the fallback texels' light
    // through the probes from the last bounce's light and theta (build())
    bool vol = false;
    uint32_t vrays = 0, n_vitems = 0, n_probes = 0, n5 = 0, vseed = 0;
    uint64_t n_vrec = 0, vunlit0 = 0, n_vunlit = 0;
    lbd::VolumeGrid grid{};
    static constexpr int VRINGS = 8;  // the fill's rings (bake_device.cu, volume.rs:88)
    DBuf light_last, vprobes, vprobes_b, vka, vkb, fb_ind, f5, vflags, vcsr_off, vcsr_who, vcsr_w, gp, g_vp_a, g_vp_b, vg,
        vsorted, voffs, g_vlight;
    cudaGraphExec_t fwd = nullptr, bwd = nullptr;
    bool forward_done = false;
    ~lb_transport() {
        if (fwd) cudaGraphExecDestroy(fwd);
        if (bwd) cudaGraphExecDestroy(bwd);
        if (plan) lb_plan_free(plan);
    }
    lbd::Theta th() const { return lbd::Theta{theta.as<float>(), M}; }
    float4 *slot(uint32_t j) const { return ckpt.as<float4>() + size_t(j) * n_light; }
};

namespace {

// the bounces' light after bounce b of the forward: res, filters, write (the atlas rewritten in place)
void bounce(lb_transport &t, float4 *light, uint32_t b, float4 *next, cudaStream_t st, float4 **filled) {
    ck(lb_eval_records(t.records, nullptr, t.n_gath, t.rays, light, t.n_light, t.theta.as<float>(), t.M,
                       t.res.as<float4>(), t.g->sms, st),
       "transport eval");
    ck(lb_bounce_filters(t.a, t.res.as<float4>(), t.r, t.plan->wr.as<float>(), t.rings, t.fk_a.as<uint8_t>(),
                         t.fk_b.as<uint8_t>(), t.e0.as<float4>(), t.e1.as<float4>(), filled, st),
       "transport filters");
    if (next && t.n_tex)
        lbd::k_write_light<<<tg(t.n_tex), 256, 0, st>>>(t.a, t.kb.as<uint8_t>(), t.dl0.as<float4>(), t.th(), *filled,
                                                        next);
    (void)b;
}

void light0(lb_transport &t, float4 *light, cudaStream_t st) {
    if (t.n_tex)
        lbd::k_write_light<<<tg(t.n_tex), 256, 0, st>>>(t.a, t.kb.as<uint8_t>(), t.dl0.as<float4>(), t.th(), nullptr,
                                                        light);
    ck(cudaGetLastError(), "transport light");
}

// the volume's share of the forward: the probes from the last bounce's light (the volume records), the
// fill, the fallback texels' light
void volume_forward(lb_transport &t, cudaStream_t st) {
    lb_plan &p = *t.plan;
    lbd::k_veval<<<tg(t.n_vitems), 256, 0, st>>>(p.vrecords.as<uint2>(), p.probe_items.as<float4>(),
                                                 p.probe_slot.as<uint32_t>(), t.n_vitems, t.vrays, t.vseed,
                                                 t.light_last.as<float4>(), t.n_light, t.th(), p.vraw.as<float4>(),
                                                 t.vprobes.as<float4>());
    ck(cudaGetLastError(), "volume records");
    ck(lb_volume_fill(t.vprobes.as<float4>(), t.vprobes_b.as<float4>(), t.vka.as<uint8_t>(), t.vkb.as<uint8_t>(),
                      t.grid.nx, t.grid.ny, t.grid.nz, lb_transport::VRINGS, st),
       "volume fill");
    lbd::k_vfallback<<<tg(t.n5), 256, 0, st>>>(t.a, t.f5.as<uint32_t>(), t.n5, t.vprobes.as<float4>(), t.grid,
                                               t.fb_ind.as<float4>());
    ck(cudaGetLastError(), "fallback");
}

// the volume's share of the adjoint (before the bounces'): the fallback texels' gradient into the probes,
// the fill and the projection transposed, the volume records as one-ray items, and the last bounce's light
// gradient into the direct light's and the last bounce's indirect's
void volume_backward(lb_transport &t, cudaStream_t st, size_t smem, int &set) {
    lb_plan &p = *t.plan;
    lbd::k_vfallback_t<<<tg(t.n5), 256, 0, st>>>(t.a, t.f5.as<uint32_t>(), t.n5, t.vprobes.as<float4>(), t.grid,
                                                 t.g_ind.as<float4>(), t.gp.as<float4>());
    lbd::k_vprobe_t<<<tg(t.n_probes), 256, 0, st>>>(t.vcsr_off.as<uint32_t>(), t.vcsr_who.as<uint32_t>(),
                                                    t.vcsr_w.as<float>(), t.n_probes, t.gp.as<float4>(),
                                                    t.g_vp_a.as<float4>());
    float4 *cur = t.g_vp_a.as<float4>(), *other = t.g_vp_b.as<float4>();
    for (int q = lb_transport::VRINGS - 1; q >= 0; q--) {
        lbd::k_vfill_t<<<tg(t.n_probes), 256, 0, st>>>(t.vflags.as<uint8_t>() + size_t(q) * t.n_probes, cur, other,
                                                       t.grid.nx, t.grid.ny, t.grid.nz);
        std::swap(cur, other);
    }
    lbd::k_vrec_t<<<t.g->sms * 8, 256, 0, st>>>(p.probe_items.as<float4>(), p.probe_slot.as<uint32_t>(), t.n_vitems,
                                                t.vrays, t.vseed, cur, t.vg.as<float4>());
    ck(cudaGetLastError(), "volume^T");
    for (uint32_t m0 = 0, first = 1; m0 < std::max(t.M, 1u); m0 += t.mc, first = 0) {
        uint32_t mc = std::min(t.mc, std::max(t.M, 1u) - m0);
        lbd::k_lit_t<<<t.blocks, T_THREADS, smem, st>>>(t.voffs.as<uint64_t>(), t.vsorted.as<uint2>(), t.n_light,
                                                        t.light_last.as<float4>(), t.th(), m0, mc, 1u, t.vg.as<float4>(),
                                                        t.g_vlight.as<float4>(), int(first),
                                                        const_cast<double *>(t.sets[set].p));
        set++;
        lbd::k_unlit_t<<<t.blocks, T_THREADS, smem, st>>>(t.vsorted.as<uint2>() + t.vunlit0, t.n_vunlit, t.th(), m0,
                                                          mc, 1u, t.vg.as<float4>(), int(first),
                                                          const_cast<double *>(t.sets[set].p));
        set++;
    }
    if (t.n_tex)
        lbd::k_light_add_t<<<tg(t.n_tex), 256, 0, st>>>(t.a, t.kb.as<uint8_t>(), t.g_vlight.as<float4>(),
                                                        t.g_dl.as<float4>(), t.B > 0 ? t.g_ind.as<float4>() : nullptr);
    ck(cudaGetLastError(), "volume records^T");
}

// the forward, from theta (on the device) to the indirect atlas in out_atlas
void record_forward(lb_transport &t, cudaStream_t st) {
    bool all = t.K >= t.B;
    float4 *filled = nullptr;
    if (t.B > 0) {
        float4 *cur = all ? t.slot(0) : t.work.as<float4>();
        light0(t, cur, st);
        uint32_t next_ck = 0;
        for (uint32_t b = 0; b < t.B; b++) {
            if (!all && next_ck < t.K && t.ck_bounce[next_ck] == b) {
                ck(cudaMemcpyAsync(t.slot(next_ck), cur, size_t(t.n_light) * 16, cudaMemcpyDeviceToDevice, st),
                   "checkpoint");
                next_ck++;
            }
            // the last bounce writes the light the volume reads
            float4 *nxt = b + 1 < t.B ? (all ? t.slot(b + 1) : cur) : t.vol ? t.light_last.as<float4>() : nullptr;
            bounce(t, cur, b, nxt, st, &filled);
            if (nxt) cur = nxt;
        }
    } else if (t.vol) {
        light0(t, t.light_last.as<float4>(), st);
    }
    if (t.vol) volume_forward(t, st);
    if (t.n_tex)
        lbd::k_final_ind<<<tg(t.n_tex), 256, 0, st>>>(t.n_tex, t.plan->state.as<uint8_t>(), filled,
                                                      t.vol ? t.fb_ind.as<float4>() : t.fixed_ind.as<float4>(),
                                                      t.ind.as<float4>());
    ck(lb_composite(t.c, t.out_tmp.as<float4>(), t.out_has_b.as<uint8_t>(), st), "transport composite");
}

// the adjoint, from the atlas gradient in g_in to theta's gradient in g_theta
void record_backward(lb_transport &t, cudaStream_t st) {
    const PostArgs &a = t.a;
    uint64_t nb = uint64_t(t.iw) * t.ih;
    ck(cudaMemsetAsync(t.g_dl.p, 0, t.g_dl.bytes, st), "memset");
    // the dilations transposed, last first, then the composite
    lbd::k_dilate_t<<<tg(nb), 256, 0, st>>>(t.has1.as<uint8_t>(), t.g_in.as<float4>(), t.g_blocks_a.as<float4>(), t.iw,
                                            t.ih);
    lbd::k_dilate_t<<<tg(nb), 256, 0, st>>>(t.has0.as<uint8_t>(), t.g_blocks_a.as<float4>(), t.g_blocks_b.as<float4>(),
                                            t.iw, t.ih);
    if (t.n_tex)
        lbd::k_composite_t<<<tg(t.n_tex), 256, 0, st>>>(a, t.c, t.g_blocks_b.as<float4>(), t.g_ind.as<float4>(),
                                                        int(t.vol));
    ck(cudaGetLastError(), "transport composite^T");
    bool all = t.K >= t.B;
    size_t smem = size_t(3 * t.mc) * lbd::TW * sizeof(double);
    int set = 0;
    if (t.vol) volume_backward(t, st, smem, set);
    for (int32_t b = int32_t(t.B) - 1; b >= 0; b--) {
        // the light this bounce read: kept, or recomputed from the nearest earlier checkpoint
        float4 *light;
        if (all) {
            light = t.slot(uint32_t(b));
        } else {
            uint32_t j = 0;
            while (j + 1 < t.K && t.ck_bounce[j + 1] <= uint32_t(b)) j++;
            light = t.work.as<float4>();
            ck(cudaMemcpyAsync(light, t.slot(j), size_t(t.n_light) * 16, cudaMemcpyDeviceToDevice, st), "restore");
            float4 *filled = nullptr;
            for (uint32_t bb = t.ck_bounce[j]; bb < uint32_t(b); bb++) bounce(t, light, bb, light, st, &filled);
        }
        if (t.n_tex) {
            // fill rings transposed (last ring first), the smoothing, the scatter
            float4 *outs[2] = {t.g_a.as<float4>(), t.g_b.as<float4>()};
            float4 *gw = t.g_ind.as<float4>();
            for (int q = t.rings - 1, o = 0; q >= 0; q--, o ^= 1) {
                lbd::k_fill_t<<<tg(t.n_tex), 256, 0, st>>>(a, t.masks.as<uint8_t>() + size_t(q) * t.n_tex, gw, outs[o]);
                gw = outs[o];
            }
            float4 *gs = gw == outs[0] ? outs[1] : outs[0];
            lbd::k_smooth_t<<<tg(t.n_tex), 256, 0, st>>>(a, gw, t.r, t.plan->wr.as<float>(), t.wsum.as<float>(), gs);
            if (t.n_gath)
                lbd::k_scatter_t<<<tg(t.n_gath), 256, 0, st>>>(t.plan->gath_idx.as<uint32_t>(), t.n_gath, gs,
                                                               t.g_res.as<float4>());
        }
        ck(cudaGetLastError(), "transport filters^T");
        // the records transposed: the atlas gradient and theta's partial sums, chunk by chunk of materials
        for (uint32_t m0 = 0, first = 1; m0 < std::max(t.M, 1u); m0 += t.mc, first = 0) {
            uint32_t mc = std::min(t.mc, std::max(t.M, 1u) - m0);
            lbd::k_lit_t<<<t.blocks, T_THREADS, smem, st>>>(
                t.offs.as<uint64_t>(), t.sorted.as<uint2>(), t.n_light, light, t.th(), m0, mc, t.rays, t.g_res.as<float4>(),
                t.g_light.as<float4>(), int(first), const_cast<double *>(t.sets[set].p));
            set++;
            lbd::k_unlit_t<<<t.blocks, T_THREADS, smem, st>>>(t.sorted.as<uint2>() + t.unlit0, t.n_unlit, t.th(), m0, mc,
                                                             t.rays, t.g_res.as<float4>(), int(first),
                                                             const_cast<double *>(t.sets[set].p));
            set++;
        }
        ck(cudaGetLastError(), "transport records^T");
        // write_light transposed: into the direct light, and the previous bounce's indirect
        if (t.n_tex)
            lbd::k_light_t<<<tg(t.n_tex), 256, 0, st>>>(a, t.kb.as<uint8_t>(), t.g_light.as<float4>(), t.g_dl.as<float4>(),
                                                        b > 0 ? t.g_ind.as<float4>() : nullptr);
    }
    lbd::k_sun_t<<<t.sun_blocks, 256, 0, st>>>(t.n_tex, t.g_dl.as<float4>(), t.dl0.as<float4>(),
                                              t.sun_partials.as<double>());
    uint32_t n_out = 3 * t.M + 10;
    lbd::k_theta_final<<<n_out, 256, 0, st>>>(t.sets_d.as<lbd::PartialSet>(), int(t.sets.size()), t.blocks,
                                                  t.sun_partials.as<double>(), t.sun_blocks, t.M, t.g_theta.as<float>());
    ck(cudaGetLastError(), "transport theta");
}

cudaGraphExec_t capture(lb_transport &t, void (*rec)(lb_transport &, cudaStream_t)) {
    cudaStream_t st = t.g->stream;
    ck(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "begin capture");
    try {
        rec(t, st);
    } catch (...) {
        cudaGraph_t gr = nullptr;
        cudaStreamEndCapture(st, &gr);
        if (gr) cudaGraphDestroy(gr);
        throw;
    }
    cudaGraph_t gr = nullptr;
    ck(cudaStreamEndCapture(st, &gr), "end capture");
    cudaGraphExec_t ex = nullptr;
    cudaError_t e = cudaGraphInstantiate(&ex, gr, 0);
    cudaGraphDestroy(gr);
    ck(e, "graph instantiate");
    return ex;
}

template <class T> void up(DBuf &d, const std::vector<T> &v, cudaStream_t st) {
    d.alloc(v.size() * sizeof(T));
    if (!v.empty()) ck(cudaMemcpyAsync(d.p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, st), "upload");
}

// The volume's share, when the bake lit texels from the volume (state 5): their list, the fill's known flags
// ring by ring, each probe's list of the fallback texels that read it (with the corner weights), the
// volume records in the adjoint's order (as the gather's, one ray an item) and the adjoint's arrays.
void volume_setup(lb_transport &t, cudaStream_t st) {
    lb_plan &p = *t.plan;
    t.vol = false;
    if (!p.has_volume || !p.n_todo || !t.n_tex) return;
    std::vector<uint8_t> state(t.n_tex);
    ck(cudaMemcpy(state.data(), p.state.p, t.n_tex, cudaMemcpyDeviceToHost), "state");
    std::vector<uint32_t> f5;
    for (uint32_t i = 0; i < t.n_tex; i++)
        if (state[i] == 5) f5.push_back(i);
    if (f5.empty()) return;
    const lb::VolumeSettings &v = *p.scene.header.volume;
    t.vol = true;
    t.n5 = uint32_t(f5.size());
    up(t.f5, f5, st);
    t.vrays = v.rays;
    t.n_vitems = p.n_todo;
    t.n_probes = p.n_probes;
    std::memcpy(&t.vseed, &p.P.params.reach[3], 4);
    t.n_vrec = uint64_t(t.n_vitems) * t.vrays;
    if (t.n_vrec >= (1ull << 30)) throw std::runtime_error("lb_transport_create: too many volume rays");
    t.grid = lbd::VolumeGrid{make_float3(v.min[0], v.min[1], v.min[2]), v.step, p.vsize[0], p.vsize[1], p.vsize[2]};
    if (t.grid.nx < 2 || t.grid.ny < 2 || t.grid.nz < 2)
        throw std::runtime_error("lb_transport_create: a volume needs two probes along each axis");
    const size_t N = std::max<size_t>(t.n_tex, 1);
    t.light_last.alloc(size_t(t.n_light) * 16);
    ck(cudaMemsetAsync(t.light_last.p, 0, t.light_last.bytes, st), "light");
    t.vprobes.alloc(size_t(t.n_probes) * 64);
    t.vprobes_b.alloc(size_t(t.n_probes) * 64);
    t.vka.alloc(t.n_probes);
    t.vkb.alloc(t.n_probes);
    t.fb_ind.alloc(N * 16);
    ck(cudaMemcpyAsync(t.fb_ind.p, t.fixed_ind.p, N * 16, cudaMemcpyDeviceToDevice, st), "fallback light");
    // the fill's known flags before each ring (volume.rs:88-121: known where the back-face share is at most
    // half, then every unknown probe with a known neighbour, ring by ring)
    {
        std::vector<float> raw(size_t(t.n_probes) * 16);
        ck(cudaMemcpy(raw.data(), p.vraw.p, raw.size() * 4, cudaMemcpyDeviceToHost), "raw probes");
        const uint32_t nx = t.grid.nx, ny = t.grid.ny, nz = t.grid.nz;
        std::vector<uint8_t> flags(size_t(lb_transport::VRINGS) * t.n_probes), was(t.n_probes);
        for (uint32_t k = 0; k < t.n_probes; k++) was[k] = raw[size_t(k) * 16 + 7] <= 0.5f;
        const int D[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
        for (int q = 0; q < lb_transport::VRINGS; q++) {
            std::copy(was.begin(), was.end(), flags.begin() + size_t(q) * t.n_probes);
            std::vector<uint8_t> now = was;
            for (uint32_t k = 0; k < t.n_probes; k++) {
                if (was[k]) continue;
                int x = int(k % nx), z = int((k / nx) % nz), y = int(k / (nx * nz));
                for (int d = 0; d < 6; d++) {
                    int xx = x + D[d][0], yy = y + D[d][1], zz = z + D[d][2];
                    if (xx < 0 || yy < 0 || zz < 0 || xx >= int(nx) || yy >= int(ny) || zz >= int(nz)) continue;
                    if (was[(uint32_t(yy) * nz + uint32_t(zz)) * nx + uint32_t(xx)]) {
                        now[k] = 1;
                        break;
                    }
                }
            }
            was.swap(now);
        }
        up(t.vflags, flags, st);
    }
    // each probe's fallback texels (index in f5) and weights, in texel order
    {
        DBuf j8, w8;
        j8.alloc(size_t(t.n5) * 8 * 4);
        w8.alloc(size_t(t.n5) * 8 * 4);
        lbd::k_vcorners<<<tg(t.n5), 256, 0, st>>>(t.a, t.f5.as<uint32_t>(), t.n5, t.grid, j8.as<uint32_t>(),
                                                  w8.as<float>());
        ck(cudaGetLastError(), "corners");
        std::vector<uint32_t> hj(size_t(t.n5) * 8);
        std::vector<float> hw(size_t(t.n5) * 8);
        ck(cudaMemcpy(hj.data(), j8.p, hj.size() * 4, cudaMemcpyDeviceToHost), "corners");
        ck(cudaMemcpy(hw.data(), w8.p, hw.size() * 4, cudaMemcpyDeviceToHost), "corners");
        std::vector<uint32_t> off(size_t(t.n_probes) + 1, 0), who(hj.size());
        std::vector<float> wt(hj.size());
        for (uint32_t j : hj) off[size_t(j) + 1]++;
        for (uint32_t k = 0; k < t.n_probes; k++) off[k + 1] += off[k];
        std::vector<uint32_t> at(off.begin(), off.end() - 1);
        for (size_t e = 0; e < hj.size(); e++) {
            uint32_t pos = at[hj[e]]++;
            who[pos] = uint32_t(e / 8);
            wt[pos] = hw[e];
        }
        up(t.vcsr_off, off, st);
        up(t.vcsr_who, who, st);
        up(t.vcsr_w, wt, st);
        ck(cudaStreamSynchronize(st), "corner lists");
    }
    // the volume records in the adjoint's order: lit by atlas texel (the bake's last light tells which texels
    // hold light), then sky and fallback-lit, then none
    t.vsorted.alloc(t.n_vrec * 8);
    t.voffs.alloc(size_t(t.n_light + 3) * 8);
    {
        DBuf keys, vals, keys2, vals2, temp;
        size_t n = std::max<uint64_t>(t.n_vrec, 1);
        keys.alloc(n * 4);
        vals.alloc(n * 4);
        keys2.alloc(n * 4);
        vals2.alloc(n * 4);
        lbd::k_record_keys<<<t.g->sms * 8, 256, 0, st>>>(p.vrecords.as<uint2>(), t.n_vrec, p.light.as<float4>(),
                                                        t.n_light, t.M, keys.as<uint32_t>(), vals.as<uint32_t>());
        size_t tb = 0;
        ck(cub::DeviceRadixSort::SortPairs(nullptr, tb, keys.as<uint32_t>(), keys2.as<uint32_t>(), vals.as<uint32_t>(),
                                           vals2.as<uint32_t>(), int(t.n_vrec), 0, 32, st),
           "sort size");
        temp.alloc(tb);
        ck(cub::DeviceRadixSort::SortPairs(temp.p, tb, keys.as<uint32_t>(), keys2.as<uint32_t>(), vals.as<uint32_t>(),
                                           vals2.as<uint32_t>(), int(t.n_vrec), 0, 32, st),
           "sort");
        lbd::k_record_sorted<<<t.g->sms * 8, 256, 0, st>>>(p.vrecords.as<uint2>(), vals2.as<uint32_t>(), t.n_vrec, 1u,
                                                          t.vsorted.as<uint2>());
        lbd::k_record_offsets<<<tg(t.n_light + 3), 256, 0, st>>>(keys2.as<uint32_t>(), t.n_vrec, t.n_light,
                                                                 t.voffs.as<uint64_t>());
        ck(cudaGetLastError(), "volume record order");
        std::vector<uint64_t> tail(3);
        ck(cudaMemcpyAsync(tail.data(), t.voffs.as<uint64_t>() + t.n_light, 24, cudaMemcpyDeviceToHost, st), "offsets");
        ck(cudaStreamSynchronize(st), "volume record order");
        t.vunlit0 = tail[0];
        t.n_vunlit = tail[2] - tail[0];
    }
    t.gp.alloc(size_t(t.n5) * 64);
    t.g_vp_a.alloc(size_t(t.n_probes) * 64);
    t.g_vp_b.alloc(size_t(t.n_probes) * 64);
    t.vg.alloc(std::max<uint64_t>(t.n_vrec, 1) * 16);
    t.g_vlight.alloc(size_t(t.n_light) * 16);
}

void build(lb_transport &t, uint32_t max_checkpoints) {
    lb_plan &p = *t.plan;
    cudaStream_t st = t.g->stream;
    const lb::SceneHeader &h = p.scene.header;
    if (p.n_dirty_texels != p.n_all)
        throw std::runtime_error("lb_transport_create: every tile must be baked (no cache)");
    // the bake at theta0: its arrays hold every fixed input
    if (lb_plan_launch(&p) != LB_OK) throw std::runtime_error(lb_last_error());
    ck(cudaStreamSynchronize(st), "bake");
    t.M = uint32_t(h.materials.size());
    t.B = h.bake.gi_bounces;
    t.rays = p.P.params.counts[2];
    t.n_light = p.aw * p.ah;
    t.n_tex = p.n_dirty_texels;
    t.iw = p.iw;
    t.ih = p.ih;
    t.r = int(h.bake.gi_filter * p.ds);
    t.rings = int(h.lightmap.padding + 2 * p.ds + 2);
    ck(cudaMemcpy(&t.n_gath, p.gath_count.p, 4, cudaMemcpyDeviceToHost), "gathered count");
    if (t.n_gath >= (1u << 30)) throw std::runtime_error("lb_transport_create: too many gathered texels");
    t.n_rec = uint64_t(t.n_gath) * t.rays;
    if (t.n_rec >= (1ull << 31)) throw std::runtime_error("lb_transport_create: more than 2^31 gather rays");
    // theta0: the scene's albedos and sky, the sun at its own irradiance
    t.theta0.clear();
    for (auto &m : h.materials) t.theta0.insert(t.theta0.end(), m.albedo.begin(), m.albedo.end());
    for (auto *c : {&h.sky.zenith, &h.sky.horizon, &h.sky.ground}) t.theta0.insert(t.theta0.end(), c->begin(), c->end());
    t.theta0.push_back(1.0f);
    up(t.theta, t.theta0, st);
    t.a = lb_plan_post_args(p);
    size_t N = std::max<size_t>(t.n_tex, 1);
    // fixed inputs: known during the bounces, the direct light at the scene's irradiance, the fallback
    // texels' light
    t.kb.alloc(N);
    t.dl0.alloc(N * 16);
    t.fixed_ind.alloc(N * 16);
    if (t.n_tex) {
        lbd::k_known_bounce<<<tg(t.n_tex), 256, 0, st>>>(t.n_tex, p.known.as<uint8_t>(), p.state.as<uint8_t>(),
                                                         t.kb.as<uint8_t>());
        ck(cudaMemcpyAsync(t.dl0.p, p.dl.p, size_t(t.n_tex) * 16, cudaMemcpyDeviceToDevice, st), "dl0");
        ck(cudaMemcpyAsync(t.fixed_ind.p, p.ind.p, size_t(t.n_tex) * 16, cudaMemcpyDeviceToDevice, st), "ind");
    }
    // the bounce fill's plan ring by ring (from the gathered flags on), the smoothing's weight sums
    t.masks.alloc(size_t(std::max(t.rings, 1)) * N);
    t.wsum.alloc(N * 4);
    if (t.n_tex) {
        DBuf fa, fb;
        fa.alloc(N);
        fb.alloc(N);
        ck(cudaMemcpyAsync(fa.p, p.gathered.p, t.n_tex, cudaMemcpyDeviceToDevice, st), "fill flags");
        uint8_t *was = fa.as<uint8_t>(), *now = fb.as<uint8_t>();
        for (int q = 0; q < t.rings; q++) {
            lbd::k_fill_plan<<<tg(t.n_tex), 256, 0, st>>>(t.a, was, t.masks.as<uint8_t>() + size_t(q) * t.n_tex, now);
            lbd::k_fill_plan_mark<<<tg(t.n_tex), 256, 0, st>>>(t.a, t.masks.as<uint8_t>() + size_t(q) * t.n_tex);
            std::swap(was, now);
        }
        lbd::k_smooth_wsum<<<tg(t.n_tex), 256, 0, st>>>(t.a, t.r, p.wr.as<float>(), t.wsum.as<float>());
        ck(cudaStreamSynchronize(st), "fill plan");
    }
    // the composite's arguments (its outputs in the transport's own arrays) and its dilation flags
    uint64_t nb = uint64_t(t.iw) * t.ih;
    t.ind.alloc(N * 16);
    t.out_atlas.alloc(nb * 16);
    t.out_tmp.alloc(nb * 16);
    t.out_has.alloc(nb);
    t.out_has_b.alloc(nb);
    t.out_direct.alloc(size_t(t.n_light) * 8);
    t.out_validity.alloc(t.n_light);
    t.c.owner = p.owner.as<uint32_t>();
    t.c.known = p.known.as<uint8_t>();
    t.c.state = p.state.as<uint8_t>();
    t.c.field = p.field.as<float>();
    t.c.ao = p.ao.as<float>();
    t.c.ind = t.ind.as<float4>();
    t.c.aw = p.aw;
    t.c.ah = p.ah;
    t.c.iw = p.iw;
    t.c.ih = p.ih;
    t.c.ds = p.ds;
    t.c.direct_out = t.out_direct.as<float2>();
    t.c.validity = t.out_validity.as<uint8_t>();
    t.c.indirect = t.out_atlas.as<float4>();
    t.c.has = t.out_has.as<uint8_t>();
    // the dilations' plans: from the composite's own flags (its block averages alone, run once), then
    // the first pass's
    t.has0.alloc(nb);
    t.has1.alloc(nb);
    if (nb) {
        DBuf f0, f1;
        f0.alloc(nb);
        f1.alloc(nb);
        CompositeArgs c0 = t.c;
        c0.ind = p.ind.as<float4>();
        c0.has = f0.as<uint8_t>();
        c0.indirect = t.out_tmp.as<float4>();
        ck(lb_composite_blocks(c0, st), "composite flags");
        lbd::k_dilate_plan<<<tg(nb), 256, 0, st>>>(f0.as<uint8_t>(), t.has0.as<uint8_t>(), t.iw, t.ih);
        lbd::k_dilate_mask<<<tg(nb), 256, 0, st>>>(f0.as<uint8_t>(), f1.as<uint8_t>(), t.iw, t.ih);
        lbd::k_dilate_plan<<<tg(nb), 256, 0, st>>>(f1.as<uint8_t>(), t.has1.as<uint8_t>(), t.iw, t.ih);
        ck(cudaStreamSynchronize(st), "dilation plan");
    }
    // every gather ray's outcome: the bake's first gather pass recorded them
    t.records = p.records.as<uint2>();
    t.res.alloc(std::max<size_t>(t.n_gath, 1) * 16);
    // the records sorted for the adjoint: lit ones by atlas texel, then sky and fallback-lit, then none
    t.sorted.alloc(t.n_rec * 8);
    t.offs.alloc(size_t(t.n_light + 3) * 8);
    {
        DBuf keys, vals, keys2, vals2, temp;
        size_t n = std::max<uint64_t>(t.n_rec, 1);
        keys.alloc(n * 4);
        vals.alloc(n * 4);
        keys2.alloc(n * 4);
        vals2.alloc(n * 4);
        if (t.n_rec) {
            lbd::k_record_keys<<<t.g->sms * 8, 256, 0, st>>>(t.records, t.n_rec, p.light.as<float4>(), t.n_light,
                                                            t.M, keys.as<uint32_t>(), vals.as<uint32_t>());
            size_t tb = 0;
            ck(cub::DeviceRadixSort::SortPairs(nullptr, tb, keys.as<uint32_t>(), keys2.as<uint32_t>(), vals.as<uint32_t>(),
                                               vals2.as<uint32_t>(), int(t.n_rec), 0, 32, st),
               "sort size");
            temp.alloc(tb);
            ck(cub::DeviceRadixSort::SortPairs(temp.p, tb, keys.as<uint32_t>(), keys2.as<uint32_t>(), vals.as<uint32_t>(),
                                               vals2.as<uint32_t>(), int(t.n_rec), 0, 32, st),
               "sort");
            lbd::k_record_sorted<<<t.g->sms * 8, 256, 0, st>>>(t.records, vals2.as<uint32_t>(), t.n_rec, t.rays,
                                                              t.sorted.as<uint2>());
        }
        lbd::k_record_offsets<<<tg(t.n_light + 3), 256, 0, st>>>(keys2.as<uint32_t>(), t.n_rec, t.n_light,
                                                                 t.offs.as<uint64_t>());
        ck(cudaGetLastError(), "record order");
        std::vector<uint64_t> tail(3);
        ck(cudaMemcpyAsync(tail.data(), t.offs.as<uint64_t>() + t.n_light, 24, cudaMemcpyDeviceToHost, st), "offsets");
        ck(cudaStreamSynchronize(st), "record order");
        t.n_lit = tail[0];
        t.unlit0 = tail[0];
        t.n_unlit = tail[2] - tail[0];
    }
    volume_setup(t, st);
    // checkpoints: every bounce's light when the budget allows, else K spread evenly (the first is bounce 0)
    t.K = max_checkpoints == 0 ? t.B : std::min(max_checkpoints, t.B);
    t.ck_bounce.clear();
    for (uint32_t j = 0; j < t.K; j++) t.ck_bounce.push_back(uint32_t(uint64_t(j) * t.B / t.K));
    t.ckpt.alloc(size_t(std::max(t.K, 1u)) * t.n_light * 16);
    ck(cudaMemsetAsync(t.ckpt.p, 0, t.ckpt.bytes, st), "checkpoints");
    t.work.alloc(size_t(t.n_light) * 16);
    ck(cudaMemsetAsync(t.work.p, 0, t.work.bytes, st), "work");
    t.e0.alloc(N * 16);
    t.e1.alloc(N * 16);
    t.fk_a.alloc(N);
    t.fk_b.alloc(N);
    // the adjoint's arrays and its fixed reduction grid
    t.g_in.alloc(nb * 16);
    t.g_blocks_a.alloc(nb * 16);
    t.g_blocks_b.alloc(nb * 16);
    t.g_ind.alloc(N * 16);
    t.g_a.alloc(N * 16);
    t.g_b.alloc(N * 16);
    t.g_dl.alloc(N * 16);
    t.g_res.alloc(std::max<size_t>(t.n_gath, 1) * 16);
    t.g_light.alloc(size_t(t.n_light) * 16);
    t.g_theta.alloc(size_t(3 * t.M + 10) * 4);
    t.blocks = t.g->sms * 4;
    t.sun_blocks = t.g->sms * 2;
    size_t per_mat = size_t(3) * lbd::TW * sizeof(double);
    t.mc = uint32_t(std::max<size_t>(1, T_SMEM / per_mat));
    t.mc = std::min(t.mc, std::max(t.M, 1u));
    size_t smem = size_t(3 * t.mc) * lbd::TW * sizeof(double);
    ck(cudaFuncSetAttribute(lbd::k_lit_t, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)), "smem");
    ck(cudaFuncSetAttribute(lbd::k_unlit_t, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)), "smem");
    uint32_t chunks = (std::max(t.M, 1u) + t.mc - 1) / t.mc;
    size_t per_set = size_t(t.blocks) * (3 * t.mc + lbd::FIXED_SLOTS);
    size_t n_sets = size_t(t.B + (t.vol ? 1 : 0)) * chunks * 2;
    t.partials.alloc(std::max<size_t>(n_sets, 1) * per_set * sizeof(double));
    t.sun_partials.alloc(size_t(t.sun_blocks) * sizeof(double));
    t.sets.clear();
    for (size_t s = 0; s < n_sets; s++) {
        uint32_t chunk = uint32_t((s / 2) % chunks);
        uint32_t m0 = chunk * t.mc, mc = std::min(t.mc, std::max(t.M, 1u) - m0);
        lbd::PartialSet ps{t.partials.as<double>() + s * per_set, m0, mc, int(chunk == 0)};
        t.sets.push_back(ps);
    }
    // a chunk's partial rows are laid out with its own slot count: give every set the chunk's mc
    up(t.sets_d, t.sets, st);
    ck(cudaStreamSynchronize(st), "transport arrays");
    t.fwd = capture(t, record_forward);
    t.bwd = capture(t, record_backward);
}

int fail(const std::exception &e) {
    lb_set_error(e.what());
    return LB_ECUDA;
}

}  // namespace

extern "C" {

lb_transport *lb_transport_create(lb_gpu *g, const uint8_t *scene, size_t len, uint32_t max_checkpoints) {
    if (!g || !scene) {
        lb_set_error("lb_transport_create: bad arguments");
        return nullptr;
    }
    lb_plan *p = lb_plan_create_recording(g, scene, len);
    if (!p) return nullptr;
    auto t = std::make_unique<lb_transport>();
    t->plan = p;
    t->g = g;
    try {
        lbplan::DBufScope spares(g);  // the transport's device buffers from (and back to) the handle's spares
        build(*t, max_checkpoints);
        return t.release();
    } catch (const std::exception &e) {
        lb_set_error(e.what());
    }
    return nullptr;
}

int lb_transport_info(const lb_transport *t, lb_transport_shape *info) {
    if (!t || !info) return LB_EINVAL;
    std::memset(info, 0, sizeof *info);
    info->n_materials = t->M;
    info->n_params = 3 * t->M + 10;
    info->bounces = t->B;
    info->checkpoints = t->K;
    info->indirect_width = t->iw;
    info->indirect_height = t->ih;
    info->gathered = t->n_gath;
    info->rays = t->rays;
    info->records = t->n_rec;
    info->lit_records = t->n_lit;
    info->unlit_records = t->n_unlit;
    info->checkpoint_bytes = uint64_t(std::max(t->K, 1u)) * t->n_light * 16;
    return LB_OK;
}

int lb_transport_theta0(const lb_transport *t, float *theta) {
    if (!t || !theta) return LB_EINVAL;
    std::memcpy(theta, t->theta0.data(), t->theta0.size() * 4);
    return LB_OK;
}

int lb_transport_forward_async(lb_transport *t, const float *d_theta, float *d_indirect) {
    if (!t || !d_theta || !d_indirect) return LB_EINVAL;
    cudaStream_t st = t->g->stream;
    cudaError_t e = cudaMemcpyAsync(t->theta.p, d_theta, t->theta.bytes, cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess) e = cudaGraphLaunch(t->fwd, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_indirect, t->out_atlas.p, size_t(t->iw) * t->ih * 16, cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) return lb_cuda_fail(e, "lb_transport_forward");
    t->forward_done = true;
    return LB_OK;
}

int lb_transport_backward_async(lb_transport *t, const float *d_g_indirect, float *d_g_theta) {
    if (!t || !d_g_indirect || !d_g_theta) return LB_EINVAL;
    if (!t->forward_done) {
        lb_set_error("lb_transport_backward: no forward to differentiate");
        return LB_EINVAL;
    }
    cudaStream_t st = t->g->stream;
    cudaError_t e = cudaMemcpyAsync(t->g_in.p, d_g_indirect, size_t(t->iw) * t->ih * 16, cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess) e = cudaGraphLaunch(t->bwd, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_g_theta, t->g_theta.p, t->g_theta.bytes, cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) return lb_cuda_fail(e, "lb_transport_backward");
    return LB_OK;
}

int lb_transport_forward(lb_transport *t, const float *theta, float *indirect) {
    if (!t || !theta || !indirect) return LB_EINVAL;
    cudaStream_t st = t->g->stream;
    cudaError_t e = cudaMemcpyAsync(t->theta.p, theta, t->theta.bytes, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaGraphLaunch(t->fwd, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(indirect, t->out_atlas.p, size_t(t->iw) * t->ih * 16, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return lb_cuda_fail(e, "lb_transport_forward");
    t->forward_done = true;
    return LB_OK;
}

int lb_transport_backward(lb_transport *t, const float *g_indirect, float *g_theta) {
    if (!t || !g_indirect || !g_theta) return LB_EINVAL;
    if (!t->forward_done) {
        lb_set_error("lb_transport_backward: no forward to differentiate");
        return LB_EINVAL;
    }
    cudaStream_t st = t->g->stream;
    cudaError_t e = cudaMemcpyAsync(t->g_in.p, g_indirect, size_t(t->iw) * t->ih * 16, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaGraphLaunch(t->bwd, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(g_theta, t->g_theta.p, t->g_theta.bytes, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return lb_cuda_fail(e, "lb_transport_backward");
    return LB_OK;
}

int lb_transport_bake_indirect(lb_transport *t, float *indirect) {
    if (!t || !indirect) return LB_EINVAL;
    cudaError_t e = cudaMemcpyAsync(indirect, t->plan->indirect.p, size_t(t->iw) * t->ih * 16, cudaMemcpyDeviceToHost,
                                    t->g->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(t->g->stream);
    if (e != cudaSuccess) return lb_cuda_fail(e, "lb_transport_bake_indirect");
    return LB_OK;
}

size_t lb_transport_export(lb_transport *t, const char *name, void *out, size_t cap) {
    // an empty array returns 0 too: the error text tells the two apart, so none is left from an earlier call
    lb_set_error("");
    if (!t || !name) {
        lb_set_error("lb_transport_export: bad arguments");
        return 0;
    }
    lb_plan &p = *t->plan;
    const void *src = nullptr;
    size_t bytes = 0;
    std::vector<uint8_t> host;
    std::string n = name;
    auto dev = [&](const DBuf &d, size_t b) {
        src = d.p;
        bytes = b;
    };
    if (n == "records") dev(p.records, t->n_rec * 8);
    else if (n == "gathered_index") dev(p.gath_idx, size_t(t->n_gath) * 4);
    else if (n == "texels") dev(p.tex, size_t(t->n_tex) * 64);
    else if (n == "sample_points") dev(p.posg, size_t(t->n_tex) * 16);
    else if (n == "chart") dev(p.chart, size_t(t->n_tex) * 4);
    else if (n == "gathered") dev(p.gathered, t->n_tex);
    else if (n == "known") dev(p.known, t->n_tex);
    else if (n == "known_bounce") dev(t->kb, t->n_tex);
    else if (n == "state") dev(p.state, t->n_tex);
    else if (n == "direct_light") dev(t->dl0, size_t(t->n_tex) * 16);
    else if (n == "fixed_indirect") dev(t->fixed_ind, size_t(t->n_tex) * 16);
    else if (n == "owner") dev(p.owner, size_t(t->n_light) * 4);
    // the bake's own arrays as it left them (the stages a test checks one by one)
    else if (n == "direct_records") dev(p.direct_out, size_t(p.n_cov) * 16);
    else if (n == "valid") dev(p.valid, t->n_tex);
    else if (n == "field") dev(p.field, size_t(t->n_tex) * 4);
    else if (n == "ao") dev(p.ao, size_t(t->n_tex) * 4);
    else if (n == "direct") dev(p.dl, size_t(t->n_tex) * 16);
    else if (n == "indirect_light") dev(p.ind, size_t(t->n_tex) * 16);
    else if (n == "gather_out") dev(p.gather_out, size_t(t->n_gath) * 16);
    else if (n == "light") dev(p.light, size_t(t->n_light) * 16);
    else if (n == "probes") dev(p.probes, p.has_volume ? size_t(p.n_probes) * 64 : 0);
    // the volume's share (empty when the transport does not differentiate the volume): every volume ray's
    // outcome, the probe items and their slots, the probes as the volume pass wrote them, the grid
    else if (n == "volume_records") dev(p.vrecords, t->vol ? t->n_vrec * 8 : 0);
    else if (n == "volume_items") dev(p.probe_items, t->vol ? size_t(t->n_vitems) * 64 : 0);
    else if (n == "volume_slots") dev(p.probe_slot, t->vol ? size_t(t->n_vitems) * 4 : 0);
    else if (n == "volume_raw") dev(p.vraw, t->vol ? size_t(t->n_probes) * 64 : 0);
    else if (n == "volume_grid") {
        // nx, ny, nz, rays, items, the sample seed (bits), origin xyz and step (bits); empty without the share
        if (t->vol) {
            uint32_t v[10] = {t->grid.nx, t->grid.ny, t->grid.nz, t->vrays, t->n_vitems, t->vseed, 0, 0, 0, 0};
            std::memcpy(&v[6], &t->grid.origin.x, 4);
            std::memcpy(&v[7], &t->grid.origin.y, 4);
            std::memcpy(&v[8], &t->grid.origin.z, 4);
            std::memcpy(&v[9], &t->grid.step, 4);
            host.resize(sizeof v);
            std::memcpy(host.data(), v, sizeof v);
            bytes = sizeof v;
        }
    }
    else if (n == "light_flags") {
        // the atlas's known flags (w of the light atlas)
        std::vector<float> l(size_t(t->n_light) * 4);
        if (cudaMemcpy(l.data(), p.light.p, l.size() * 4, cudaMemcpyDeviceToHost) != cudaSuccess) return 0;
        host.resize(t->n_light);
        for (size_t i = 0; i < t->n_light; i++) host[i] = l[4 * i + 3] > 0.5f;
        bytes = host.size();
    } else if (n == "tiles") {
        bytes = p.dirty.size() * sizeof(DTile);
        host.resize(bytes);
        std::memcpy(host.data(), p.tiles_all.data(), bytes);
    } else if (n == "smooth_weights") dev(p.wr, size_t(2 * t->r + 1) * (2 * t->r + 1) * 4);
    else if (n == "shape") {
        // aw, ah, iw, ih, ds, smoothing radius, fill rings, bounces, rays, gathered, texels, materials
        uint32_t v[12] = {p.aw, p.ah, p.iw, p.ih, p.ds, uint32_t(t->r), uint32_t(t->rings), t->B, t->rays, t->n_gath,
                          t->n_tex, t->M};
        host.resize(sizeof v);
        std::memcpy(host.data(), v, sizeof v);
        bytes = sizeof v;
    } else {
        lb_set_error("lb_transport_export: unknown array");
        return 0;
    }
    if (!out) return bytes;
    if (cap < bytes) {
        lb_set_error("lb_transport_export: buffer too small");
        return 0;
    }
    if (!host.empty()) std::memcpy(out, host.data(), bytes);
    else if (bytes && cudaMemcpy(out, src, bytes, cudaMemcpyDeviceToHost) != cudaSuccess) {
        lb_set_error("lb_transport_export: copy failed");
        return 0;
    }
    return bytes;
}

void lb_transport_free(lb_transport *t) {
    if (t) {
        cudaStreamSynchronize(t->g->stream);
        delete t;
    }
}

}  // extern "C"
