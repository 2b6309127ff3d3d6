// The texel passes of a bake on the device: what crates/lightbaker/src/bake.rs runs on the CPU between
// the ray passes (the per-tile work of :196-275, the gather selection of :282-298, the bounces' texel work
// of :303-328, the volume's inside fill volume.rs:86-117, the fallback :335-359 and the atlas :364-421),
// with the filters of crates/lightbaker/src/filter.rs. Every kernel runs over all dirty tiles at once:
// a thread a texel, the tile found from a table. Sums run in the reference's order and the Gaussian
// weights come from the host (as the host computes them), so results equal the host passes'.
#include <cub/device/device_select.cuh>
#include <thrust/iterator/counting_iterator.h>
#include <cuda_runtime.h>

#include "lb_device.cuh"
#include "lb_post.h"
#include "lb_texel.cuh"

namespace lbd {

// bake.rs:207-241: each covered texel's direct record unpacked; texels inside solids lose their own
// light; the AO curve; the sample point moved where the pass sampled off the centre.
__global__ void k_unpack(PostArgs a) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n_texels) return;
    float4 p = a.tex[4 * i], n = a.tex[4 * i + 1], dx = a.tex[4 * i + 2], dy = a.tex[4 * i + 3];
    bool cov = p.w > 0.5f;
    a.chart[i] = cov ? __float_as_uint(n.w) : NONE;
    uint8_t valid = cov, state = 0;
    float soft = 0.0f, ao = 1.0f;
    uint32_t hard = 0;
    float4 pg = p;
    if (cov) {
        float4 r = a.direct_out[a.cov_k[i]];
        if (r.w > a.inside_share) {
            valid = 0;
        } else {
            soft = r.x;
            uint32_t bits = __float_as_uint(r.y);
            hard = bits & 0x00ffffffu;
            uint32_t pick = bits >> 24;
            state = pick == 0 ? 1 : pick == 9 ? 3 : 2;
            if (pick == 9) {
                pg.x = p.x + n.x * PUSH;
                pg.y = p.y + n.y * PUSH;
                pg.z = p.z + n.z * PUSH;
            } else if (pick > 0) {
                float2 c = offset(pick);
                pg.x = p.x + (dx.x * c.x + dy.x * c.y);
                pg.y = p.y + (dx.y * c.x + dy.y * c.y);
                pg.z = p.z + (dx.z * c.x + dy.z * c.y);
            }
            float base = fmaxf(1.0f - a.ao_strength * r.z, 0.0f);
            // powf(x, 1) is x exactly on both sides; other contrasts round as CUDA's powf
            float curve = a.ao_contrast == 1.0f ? base : powf(base, a.ao_contrast);
            ao = fmaxf(curve, a.ao_floor);
        }
    }
    a.valid[i] = valid;
    a.state[i] = state;
    a.soft[i] = soft;
    a.ao_raw[i] = ao;
    a.hard[i] = hard;
    a.posg[i] = pg;
}

// filter.rs:20-53 on the occlusion and the soft sun (r = 1, their own weights), then the direct light
// from the smoothed sun (bake.rs:247-252)
__global__ void k_smooth_direct(PostArgs a) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n_texels) return;
    const DTile t = a.tiles[find_tile(a.tiles, a.n_tiles, i)];
    uint32_t li = i - t.off, x = li % t.w, y = li / t.w;
    float ao = a.ao_raw[i], soft = a.soft[i];
    if (a.valid[i]) {
        const int r = 1;
        float sa = 0.0f, ss = 0.0f, wsum = 0.0f;
        for (int yy = y > r ? int(y) - r : 0; yy < min(int(y) + r + 1, int(t.h)); yy++)
            for (int xx = x > r ? int(x) - r : 0; xx < min(int(x) + r + 1, int(t.w)); xx++) {
                uint32_t j = t.off + uint32_t(yy) * t.w + uint32_t(xx);
                if (!a.valid[j] || !same(a.chart, a.tex, i, j)) continue;
                float k = a.w1[(yy - int(y) + r) * (2 * r + 1) + (xx - int(x) + r)];
                sa += a.ao_raw[j] * k;
                ss += a.soft[j] * k;
                wsum += k;
            }
        ao = sa / wsum;
        soft = ss / wsum;
    }
    float4 n = a.tex[4 * i + 1];
    float d = fmaxf(n.x * a.sun.x + n.y * a.sun.y + n.z * a.sun.z, 0.0f);
    a.ao[i] = ao;
    a.dl[i] = make_float4(a.irr.x * d * soft, a.irr.y * d * soft, a.irr.z * d * soft, 0.0f);
}

// filter.rs:106-141: the sun's signed distance field from the hard sub-samples
__global__ void k_sun_field(PostArgs a) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n_texels) return;
    float out = -1.0f;
    if (a.valid[i]) {
        const DTile t = a.tiles[find_tile(a.tiles, a.n_tiles, i)];
        int li = int(i - t.off), x = li % int(t.w), y = li / int(t.w);
        int g = int(a.g), gg = g * g, reach = int(ceilf(a.sdf_radius)) + 1;
        bool lit = __popc(a.hard[i]) * 2 >= gg;
        float best = a.sdf_radius;
        float fg = float(g), half = 0.5f / fg;
        for (int yy = y > reach ? y - reach : 0; yy < min(y + reach + 1, int(t.h)); yy++)
            for (int xx = x > reach ? x - reach : 0; xx < min(x + reach + 1, int(t.w)); xx++) {
                uint32_t j = t.off + uint32_t(yy) * t.w + uint32_t(xx);
                if (!a.valid[j] || !same(a.chart, a.tex, i, j)) continue;
                uint32_t hj = a.hard[j];
                // cells of the other state only
                uint32_t other = lit ? ~hj : hj;
                if (gg < 32) other &= (1u << gg) - 1u;
                while (other) {
                    int c = __ffs(other) - 1;
                    other &= other - 1;
                    float px = float(xx) + (float(c % g) + 0.5f) / fg - (float(x) + 0.5f);
                    float py = float(yy) + (float(c / g) + 0.5f) / fg - (float(y) + 0.5f);
                    best = fminf(best, sqrtf(px * px + py * py) - half);
                }
            }
        float d = fminf(fmaxf(best, 0.0f), a.sdf_radius);
        out = 0.5f + 0.5f * (lit ? d : -d) / a.sdf_radius;
    }
    a.field[i] = out;
}

// filter.rs:58-94, one ring, on the occlusion, the field and the direct light at once (their three fills
// start from the same texels and grow alike: a texel's fill depends on its neighbours' flags only)
__global__ void k_fill5(PostArgs a, const uint8_t *was, uint8_t *now, const float *ao_in, float *ao_out,
                        const float *f_in, float *f_out, const float4 *dl_in, float4 *dl_out) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n_texels) return;
    float o_ao = ao_in[i], o_f = f_in[i];
    float4 o_dl = dl_in[i];
    uint8_t k = was[i];
    if (!was[i]) {
        const DTile t = a.tiles[find_tile(a.tiles, a.n_tiles, i)];
        int li = int(i - t.off), x = li % int(t.w), y = li / int(t.w);
        uint32_t ci = a.chart[i];
        float own[5] = {0, 0, 0, 0, 0}, any[5] = {0, 0, 0, 0, 0};
        int no = 0, na = 0;
        for (int yy = y > 0 ? y - 1 : 0; yy < min(y + 2, int(t.h)); yy++)
            for (int xx = x > 0 ? x - 1 : 0; xx < min(x + 2, int(t.w)); xx++) {
                uint32_t j = t.off + uint32_t(yy) * t.w + uint32_t(xx);
                if (!was[j]) continue;
                float4 d = dl_in[j];
                float v[5] = {ao_in[j], f_in[j], d.x, d.y, d.z};
                if (ci != NONE && a.chart[j] == ci) {
                    for (int c = 0; c < 5; c++) own[c] += v[c];
                    no++;
                } else {
                    for (int c = 0; c < 5; c++) any[c] += v[c];
                    na++;
                }
            }
        if (no > 0) {
            float fn = float(no);
            o_ao = own[0] / fn;
            o_f = own[1] / fn;
            o_dl = make_float4(own[2] / fn, own[3] / fn, own[4] / fn, 0.0f);
            k = 1;
        } else if (na > 0 && ci == NONE) {
            float fa = float(na);
            o_ao = any[0] / fa;
            o_f = any[1] / fa;
            o_dl = make_float4(any[2] / fa, any[3] / fa, any[4] / fa, 0.0f);
            k = 1;
        }
    }
    now[i] = k;
    ao_out[i] = o_ao;
    f_out[i] = o_f;
    dl_out[i] = o_dl;
}

// bake.rs:253-275 and write_light (:434-444): filled texels' state, known (2 own, 1 filled), no indirect
// yet; the tile's light into the atlas
__global__ void k_direct_final(PostArgs a) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n_texels) return;
    uint8_t kn = a.known_tmp[i];
    bool cov = a.tex[4 * i].w > 0.5f;
    if (cov && a.state[i] == 0 && kn) a.state[i] = 4;
    uint8_t known = a.valid[i] ? 2 : kn;
    a.known[i] = known;
    a.ind[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    const DTile t = a.tiles[find_tile(a.tiles, a.n_tiles, i)];
    uint32_t li = i - t.off, x = li % t.w, y = li / t.w;
    float4 d = a.dl[i];
    a.light[size_t(t.y + y) * a.aw + t.x + x] = known >= 1 ? make_float4(d.x, d.y, d.z, 1.0f) : make_float4(0.f, 0.f, 0.f, 0.f);
}

// bake.rs:286-297: a valid texel is gathered when it is the first valid texel of its chart in its
// smaller (ds x ds) texel, in row order (the grid texel, the block's first, included)
__global__ void k_gather_select(PostArgs a) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n_texels) return;
    uint8_t g = 0;
    if (a.valid[i]) {
        const DTile t = a.tiles[find_tile(a.tiles, a.n_tiles, i)];
        uint32_t li = i - t.off, x = li % t.w, y = li / t.w;
        uint32_t bx = x - x % a.ds, by = y - y % a.ds, ci = a.chart[i];
        g = 1;
        for (uint32_t yy = by; yy <= y && g; yy++)
            for (uint32_t xx = bx; xx < min(bx + a.ds, t.w); xx++) {
                if (yy == y && xx == x) break;
                uint32_t j = t.off + yy * t.w + xx;
                if (a.valid[j] && a.chart[j] == ci) {
                    g = 0;
                    break;
                }
            }
    }
    a.gathered[i] = g;
}

__global__ void k_inverse(const uint32_t *idx, const uint32_t *n, uint32_t *inv) {
    uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < *n) inv[idx[k]] = k;
}

// bake.rs:309-316: the gather results back into their texels, zero elsewhere
__global__ void k_scatter(PostArgs a, const float4 *res, float4 *e) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n_texels) return;
    float4 r = a.gathered[i] ? res[a.gk[i]] : make_float4(0.f, 0.f, 0.f, 0.f);
    e[i] = make_float4(r.x, r.y, r.z, 0.0f);
}

// filter.rs:20-53 on the bounced light (N = 3, radius giFilter * ds, valid: gathered)
__global__ void k_smooth3(PostArgs a, const float4 *in, float4 *out, int r, const float *w) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n_texels) return;
    float4 v = in[i];
    if (a.gathered[i] && r > 0) {
        const DTile t = a.tiles[find_tile(a.tiles, a.n_tiles, i)];
        int li = int(i - t.off), x = li % int(t.w), y = li / int(t.w);
        float sx = 0.f, sy = 0.f, sz = 0.f, wsum = 0.f;
        for (int yy = y > r ? y - r : 0; yy < min(y + r + 1, int(t.h)); yy++)
            for (int xx = x > r ? x - r : 0; xx < min(x + r + 1, int(t.w)); xx++) {
                uint32_t j = t.off + uint32_t(yy) * t.w + uint32_t(xx);
                if (!a.gathered[j] || !same(a.chart, a.tex, uint32_t(i), j)) continue;
                float k = w[(yy - y + r) * (2 * r + 1) + (xx - x + r)];
                float4 u = in[j];
                sx += u.x * k;
                sy += u.y * k;
                sz += u.z * k;
                wsum += k;
            }
        v = make_float4(sx / wsum, sy / wsum, sz / wsum, 0.0f);
    }
    out[i] = v;
}

// filter.rs:58-94, one ring, three channels
__global__ void k_fill3(PostArgs a, const uint8_t *was, uint8_t *now, const float4 *in, float4 *out) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n_texels) return;
    float4 o = in[i];
    uint8_t k = was[i];
    if (!k) {
        const DTile t = a.tiles[find_tile(a.tiles, a.n_tiles, i)];
        int li = int(i - t.off), x = li % int(t.w), y = li / int(t.w);
        uint32_t ci = a.chart[i];
        float own[3] = {0, 0, 0}, any[3] = {0, 0, 0};
        int no = 0, na = 0;
        for (int yy = y > 0 ? y - 1 : 0; yy < min(y + 2, int(t.h)); yy++)
            for (int xx = x > 0 ? x - 1 : 0; xx < min(x + 2, int(t.w)); xx++) {
                uint32_t j = t.off + uint32_t(yy) * t.w + uint32_t(xx);
                if (!was[j]) continue;
                float4 u = in[j];
                if (ci != NONE && a.chart[j] == ci) {
                    own[0] += u.x, own[1] += u.y, own[2] += u.z;
                    no++;
                } else {
                    any[0] += u.x, any[1] += u.y, any[2] += u.z;
                    na++;
                }
            }
        if (no > 0) {
            float f = float(no);
            o = make_float4(own[0] / f, own[1] / f, own[2] / f, 0.f);
            k = 1;
        } else if (na > 0 && ci == NONE) {
            float f = float(na);
            o = make_float4(any[0] / f, any[1] / f, any[2] / f, 0.f);
            k = 1;
        }
    }
    now[i] = k;
    out[i] = o;
}

// bake.rs:324-328: the bounce's light as the tile's indirect; the atlas rewritten
__global__ void k_bounce_final(PostArgs a, const float4 *e) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n_texels) return;
    float4 v = e[i];
    a.ind[i] = v;
    const DTile t = a.tiles[find_tile(a.tiles, a.n_tiles, i)];
    uint32_t li = i - t.off, x = li % t.w, y = li / t.w;
    float4 d = a.dl[i];
    a.light[size_t(t.y + y) * a.aw + t.x + x] =
        a.known[i] >= 1 ? make_float4(d.x + v.x, d.y + v.y, d.z + v.z, 1.0f) : make_float4(0.f, 0.f, 0.f, 0.f);
}

// volume.rs:86-117: one ring of the inside fill over the probe grid (x fastest, then z, then y)
__global__ void k_volume_fill(const uint8_t *was, uint8_t *now, const float4 *src, float4 *dst, uint32_t nx,
                              uint32_t ny, uint32_t nz) {
    uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t total = nx * ny * nz;
    if (k >= total) return;
    float4 o[4] = {src[4 * k], src[4 * k + 1], src[4 * k + 2], src[4 * k + 3]};
    uint8_t kn = was[k];
    if (!kn) {
        int x = k % nx, z = (k / nx) % nz, y = k / (nx * nz);
        const int D[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
        float s[16] = {0};
        int c = 0;
        for (int d = 0; d < 6; d++) {
            int xx = x + D[d][0], yy = y + D[d][1], zz = z + D[d][2];
            if (xx < 0 || yy < 0 || zz < 0 || xx >= int(nx) || yy >= int(ny) || zz >= int(nz)) continue;
            uint32_t j = (uint32_t(yy) * nz + uint32_t(zz)) * nx + uint32_t(xx);
            if (!was[j]) continue;
            for (int q = 0; q < 4; q++) {
                float4 v = src[4 * j + q];
                s[4 * q] += v.x, s[4 * q + 1] += v.y, s[4 * q + 2] += v.z, s[4 * q + 3] += v.w;
            }
            c++;
        }
        if (c > 0) {
            float f = float(c);
            for (int q = 0; q < 4; q++) o[q] = make_float4(s[4 * q] / f, s[4 * q + 1] / f, s[4 * q + 2] / f, s[4 * q + 3] / f);
            kn = 1;
        }
    }
    now[k] = kn;
    for (int q = 0; q < 4; q++) dst[4 * k + q] = o[q];
}

__global__ void k_volume_known(const float4 *probes, uint8_t *known, uint32_t total) {
    uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < total) known[k] = probes[4 * k + 1].w <= 0.5f;
}

// bake.rs:335-359 with Volume::irradiance (volume.rs:125-147)
__global__ void k_fallback(PostArgs a, const float4 *probes, float3 origin, float step, uint32_t nx, uint32_t ny,
                           uint32_t nz) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n_texels) return;
    float4 p = a.tex[4 * i], n4 = a.tex[4 * i + 1];
    if (!(p.w > 0.5f) || a.known[i] != 0) return;
    const float PI32 = 3.14159274101257324f;
    float3 q = mk(a.posg[i].x + n4.x * 0.15f, a.posg[i].y + n4.y * 0.15f, a.posg[i].z + n4.z * 0.15f);
    float fx = (q.x - origin.x) / step, fy = (q.y - origin.y) / step, fz = (q.z - origin.z) / step;
    fx = fminf(fmaxf(fx, 0.0f), float(nx - 1));
    fy = fminf(fmaxf(fy, 0.0f), float(ny - 1));
    fz = fminf(fmaxf(fz, 0.0f), float(nz - 1));
    uint32_t x0 = min(uint32_t(fx), nx - 2), y0 = min(uint32_t(fy), ny - 2), z0 = min(uint32_t(fz), nz - 2);
    float tx = fx - float(x0), ty = fy - float(y0), tz = fz - float(z0);
    float p4[16] = {0};
    for (int k = 0; k < 8; k++) {
        int dx = k & 1, dy = (k >> 1) & 1, dz = (k >> 2) & 1;
        float w = ((dx ? tx : 1.0f - tx) * (dy ? ty : 1.0f - ty)) * (dz ? tz : 1.0f - tz);
        uint32_t j = ((y0 + dy) * nz + (z0 + dz)) * nx + (x0 + dx);
        for (int c = 0; c < 4; c++) {
            float4 v = probes[4 * j + c];
            p4[4 * c] += v.x * w, p4[4 * c + 1] += v.y * w, p4[4 * c + 2] += v.z * w, p4[4 * c + 3] += v.w * w;
        }
    }
    float a0 = PI32 * 0.282095f, a1 = 2.0f * PI32 / 3.0f * 0.488603f;
    float e[3];
    for (int c = 0; c < 3; c++)
        e[c] = 0.5f * a0 * p4[c] + 0.5f * fmaxf(a0 * p4[c] + a1 * ((p4[4 + c] * n4.x + p4[8 + c] * n4.y) + p4[12 + c] * n4.z), 0.0f);
    float sun = p4[3];
    float d = fmaxf(n4.x * a.sun.x + n4.y * a.sun.y + n4.z * a.sun.z, 0.0f);
    a.ind[i] = make_float4(e[0], e[1], e[2], 0.0f);
    a.dl[i] = make_float4(a.irr.x * d * sun, a.irr.y * d * sun, a.irr.z * d * sun, 0.0f);
    a.field[i] = sun > 0.5f ? 1.0f : 0.0f;
    a.ao[i] = 1.0f;
    a.known[i] = 1;
    a.state[i] = 5;
}

// bake.rs:364-390: the direct atlas, validity, and each smaller texel's weighted light
__global__ void k_composite(CompositeArgs c) {
    uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= c.iw * c.ih) return;
    uint32_t bx = b % c.iw, by = b / c.iw;
    float s0 = 0.f, s1 = 0.f, s2 = 0.f, s3 = 0.f;
    for (uint32_t y = by * c.ds; y < min((by + 1) * c.ds, c.ah); y++)
        for (uint32_t x = bx * c.ds; x < min((bx + 1) * c.ds, c.aw); x++) {
            size_t a = size_t(y) * c.aw + x;
            uint32_t i = c.owner[a];
            float2 dout = make_float2(1.0f, 1.0f);
            uint8_t v = 0;
            if (i != NONE && c.known[i] != 0) {
                dout = make_float2(c.field[i], c.ao[i]);
                v = c.state[i];
                float k = c.known[i] == 2 ? 1.0f : 1e-3f;
                float4 e = c.ind[i];
                s0 += e.x * k;
                s1 += e.y * k;
                s2 += e.z * k;
                s3 += k;
            }
            c.direct_out[a] = dout;
            c.validity[a] = v;
        }
    c.has[b] = s3 > 0.0f;
    c.indirect[b] = s3 > 0.0f ? make_float4(s0 / s3, s1 / s3, s2 / s3, 0.f) : make_float4(0.f, 0.f, 0.f, 0.f);
}

// bake.rs:394-421: one dilation pass over the smaller atlas
__global__ void k_dilate(const uint8_t *was, uint8_t *now, const float4 *src, float4 *dst, uint32_t iw, uint32_t ih) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= iw * ih) return;
    float4 o = src[i];
    uint8_t h = was[i];
    if (!h) {
        uint32_t x = i % iw, y = i / iw;
        float acc[3] = {0, 0, 0};
        int n = 0;
        for (uint32_t yy = y > 0 ? y - 1 : 0; yy < min(y + 2, ih); yy++)
            for (uint32_t xx = x > 0 ? x - 1 : 0; xx < min(x + 2, iw); xx++) {
                uint32_t j = yy * iw + xx;
                if (was[j]) {
                    float4 v = src[j];
                    acc[0] += v.x, acc[1] += v.y, acc[2] += v.z;
                    n++;
                }
            }
        if (n > 0) {
            float f = float(n);
            o = make_float4(acc[0] / f, acc[1] / f, acc[2] / f, 0.f);
            h = 1;
        }
    }
    now[i] = h;
    dst[i] = o;
}

}  // namespace lbd

namespace {
inline dim3 grid_for(uint32_t n, int t = 256) { return dim3((n + t - 1) / t); }
}  // namespace

cudaError_t lb_post_direct(const PostArgs &a, int rings, PostScratch &s, cudaStream_t st) {
    if (a.n_texels == 0) return cudaSuccess;
    dim3 g = grid_for(a.n_texels);
    lbd::k_unpack<<<g, 256, 0, st>>>(a);
    lbd::k_smooth_direct<<<g, 256, 0, st>>>(a);
    lbd::k_sun_field<<<g, 256, 0, st>>>(a);
    // fills: ping-pong between (ao, field, dl, known) and the scratch copies
    cudaError_t e = cudaMemcpyAsync(s.known_a, a.valid, a.n_texels, cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) return e;
    uint8_t *kw = s.known_a, *kn = s.known_b;
    float *aw = a.ao, *an = s.f1, *fw = a.field, *fn = s.f2;
    float4 *dw = a.dl, *dn = s.v4;
    for (int r = 0; r < rings; r++) {
        lbd::k_fill5<<<g, 256, 0, st>>>(a, kw, kn, aw, an, fw, fn, dw, dn);
        std::swap(kw, kn);
        std::swap(aw, an);
        std::swap(fw, fn);
        std::swap(dw, dn);
    }
    if (aw != a.ao) {
        cudaMemcpyAsync(a.ao, aw, a.n_texels * 4, cudaMemcpyDeviceToDevice, st);
        cudaMemcpyAsync(a.field, fw, a.n_texels * 4, cudaMemcpyDeviceToDevice, st);
        cudaMemcpyAsync(a.dl, dw, a.n_texels * 16, cudaMemcpyDeviceToDevice, st);
    }
    if (kw != a.known_tmp) cudaMemcpyAsync(a.known_tmp, kw, a.n_texels, cudaMemcpyDeviceToDevice, st);
    lbd::k_direct_final<<<g, 256, 0, st>>>(a);
    lbd::k_gather_select<<<g, 256, 0, st>>>(a);
    return cudaGetLastError();
}

size_t lb_select_temp_bytes(uint32_t n) {
    size_t bytes = 0;
    thrust::counting_iterator<uint32_t> it(0);
    cub::DeviceSelect::Flagged(nullptr, bytes, it, (const uint8_t *)nullptr, (uint32_t *)nullptr, (uint32_t *)nullptr,
                               int(n));
    return bytes;
}

cudaError_t lb_select_gathered(const PostArgs &a, void *temp, size_t temp_bytes, uint32_t *idx, uint32_t *count,
                               cudaStream_t st) {
    if (a.n_texels == 0) return cudaMemsetAsync(count, 0, 4, st);
    thrust::counting_iterator<uint32_t> it(0);
    cudaError_t e = cub::DeviceSelect::Flagged(temp, temp_bytes, it, a.gathered, idx, count, int(a.n_texels), st);
    if (e != cudaSuccess) return e;
    lbd::k_inverse<<<grid_for(a.n_texels), 256, 0, st>>>(idx, count, a.gk);
    return cudaGetLastError();
}

cudaError_t lb_bounce_filters(const PostArgs &a, const float4 *res, int r, const float *w, int rings, uint8_t *ka,
                              uint8_t *kb, float4 *e0, float4 *e1, float4 **out, cudaStream_t st) {
    *out = e1;
    if (a.n_texels == 0) return cudaSuccess;
    dim3 g = grid_for(a.n_texels);
    lbd::k_scatter<<<g, 256, 0, st>>>(a, res, e0);
    lbd::k_smooth3<<<g, 256, 0, st>>>(a, e0, e1, r, w);
    cudaError_t e = cudaMemcpyAsync(ka, a.gathered, a.n_texels, cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) return e;
    uint8_t *kw = ka, *kn = kb;
    float4 *vw = e1, *vn = e0;
    for (int q = 0; q < rings; q++) {
        lbd::k_fill3<<<g, 256, 0, st>>>(a, kw, kn, vw, vn);
        std::swap(kw, kn);
        std::swap(vw, vn);
    }
    *out = vw;
    return cudaGetLastError();
}

cudaError_t lb_post_bounce(const PostArgs &a, const float4 *res, int r, const float *w, int rings, PostScratch &s,
                           cudaStream_t st) {
    if (a.n_texels == 0) return cudaSuccess;
    float4 *filled = nullptr;
    cudaError_t e = lb_bounce_filters(a, res, r, w, rings, s.known_a, s.known_b, s.e0, s.e1, &filled, st);
    if (e != cudaSuccess) return e;
    lbd::k_bounce_final<<<grid_for(a.n_texels), 256, 0, st>>>(a, filled);
    return cudaGetLastError();
}

cudaError_t lb_volume_fill(float4 *probes, float4 *scratch, uint8_t *ka, uint8_t *kb, uint32_t nx, uint32_t ny,
                           uint32_t nz, int rings, cudaStream_t st) {
    uint32_t total = nx * ny * nz;
    if (total == 0) return cudaSuccess;
    dim3 g = grid_for(total);
    lbd::k_volume_known<<<g, 256, 0, st>>>(probes, ka, total);
    float4 *pw = probes, *pn = scratch;
    uint8_t *kw = ka, *kn = kb;
    for (int r = 0; r < rings; r++) {
        lbd::k_volume_fill<<<g, 256, 0, st>>>(kw, kn, pw, pn, nx, ny, nz);
        std::swap(kw, kn);
        std::swap(pw, pn);
    }
    if (pw != probes) return cudaMemcpyAsync(probes, pw, size_t(total) * 64, cudaMemcpyDeviceToDevice, st);
    return cudaGetLastError();
}

cudaError_t lb_fallback(const PostArgs &a, const float4 *probes, float3 origin, float step, uint32_t nx, uint32_t ny,
                        uint32_t nz, cudaStream_t st) {
    if (a.n_texels == 0) return cudaSuccess;
    lbd::k_fallback<<<grid_for(a.n_texels), 256, 0, st>>>(a, probes, origin, step, nx, ny, nz);
    return cudaGetLastError();
}

cudaError_t lb_composite_blocks(const CompositeArgs &c, cudaStream_t st) {
    uint32_t n = c.iw * c.ih;
    if (n == 0) return cudaSuccess;
    lbd::k_composite<<<grid_for(n), 256, 0, st>>>(c);
    return cudaGetLastError();
}

cudaError_t lb_composite(const CompositeArgs &c, float4 *scratch, uint8_t *has_b, cudaStream_t st) {
    uint32_t n = c.iw * c.ih;
    if (n == 0) return cudaSuccess;
    lbd::k_composite<<<grid_for(n), 256, 0, st>>>(c);
    float4 *w = c.indirect, *nw = scratch;
    uint8_t *hw = c.has, *hn = has_b;
    for (int p = 0; p < 2; p++) {
        lbd::k_dilate<<<grid_for(n), 256, 0, st>>>(hw, hn, w, nw, c.iw, c.ih);
        std::swap(w, nw);
        std::swap(hw, hn);
    }
    // two passes: the result is back in c.indirect
    return cudaGetLastError();
}
