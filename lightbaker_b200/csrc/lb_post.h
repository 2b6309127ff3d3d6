// The device bake's per-texel state and the launchers of its texel passes (post.cu).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "host/raster.h"

// A tile in the device's texel arrays: its rectangle in the atlas and its first texel.
struct DTile {
    uint32_t x, y, w, h;
    uint32_t off;
};

// Arrays over the dirty tiles' texels (n_texels, the tiles in `tiles`, concatenated), and the atlas.
struct PostArgs {
    const DTile *tiles;
    int n_tiles;
    uint32_t n_texels;
    const float4 *tex;          // 4 float4 a texel (raster.rs Texel)
    const uint32_t *cov_k;      // a covered texel's index in the direct pass's list
    const float4 *direct_out;   // the direct pass's records
    uint32_t *chart;            // covered: its chart; else 0xffffffff
    uint8_t *valid, *state, *known, *known_tmp, *gathered;
    uint32_t *hard, *gk;
    float *soft, *ao_raw, *ao, *field;
    float4 *dl, *ind, *posg;
    float4 *light;              // the atlas the gathers read
    uint32_t aw;
    const float *w1;            // smooth weights, radius 1
    float inside_share, ao_strength, ao_contrast, ao_floor, sdf_radius;
    uint32_t g, ds;
    float3 sun, irr;
};

struct PostScratch {
    uint8_t *known_a, *known_b;
    float *f1, *f2;
    float4 *v4, *e0, *e1;
};

struct CompositeArgs {
    const uint32_t *owner;      // per atlas texel: its texel in the device arrays (all tiles), or none
    const uint8_t *known, *state;
    const float *field, *ao;
    const float4 *ind;
    uint32_t aw, ah, iw, ih, ds;
    float2 *direct_out;
    uint8_t *validity;
    float4 *indirect;
    uint8_t *has;
};

cudaError_t lb_post_direct(const PostArgs &a, int rings, PostScratch &s, cudaStream_t st);
size_t lb_select_temp_bytes(uint32_t n);
cudaError_t lb_select_gathered(const PostArgs &a, void *temp, size_t temp_bytes, uint32_t *idx, uint32_t *count,
                               cudaStream_t st);
// The bounce's texel work before the atlas write (bake.rs:309-323): the gather results scattered into their
// texels, smoothed and filled; *out is whichever of e0, e1 holds the filled light.
cudaError_t lb_bounce_filters(const PostArgs &a, const float4 *res, int r, const float *w, int rings, uint8_t *ka,
                              uint8_t *kb, float4 *e0, float4 *e1, float4 **out, cudaStream_t st);
cudaError_t lb_post_bounce(const PostArgs &a, const float4 *res, int r, const float *w, int rings, PostScratch &s,
                           cudaStream_t st);
cudaError_t lb_volume_fill(float4 *probes, float4 *scratch, uint8_t *ka, uint8_t *kb, uint32_t nx, uint32_t ny,
                           uint32_t nz, int rings, cudaStream_t st);
cudaError_t lb_fallback(const PostArgs &a, const float4 *probes, float3 origin, float step, uint32_t nx, uint32_t ny,
                        uint32_t nz, cudaStream_t st);
cudaError_t lb_composite(const CompositeArgs &c, float4 *scratch, uint8_t *has_b, cudaStream_t st);
// the composite's block averages alone, before its dilations
cudaError_t lb_composite_blocks(const CompositeArgs &c, cudaStream_t st);

// The output encodings (encode.cu; encode.rs:7-70, output.rs:162-181): the direct atlas as BC5 blocks (w, h
// multiples of 4; 16 bytes a 4 x 4 block), the indirect atlas as RGB9E5 words (float4 a texel in), the
// probes as 16 bytes each (4 float4 a probe in) with their scale (the largest L0 colour, >= 1e-6) as bits.
cudaError_t lb_encode_bc5(const float2 *direct, uint32_t w, uint32_t h, uint8_t *out, cudaStream_t st);
cudaError_t lb_encode_rgb9e5(const float4 *v, uint32_t n, uint32_t *out, cudaStream_t st);
cudaError_t lb_encode_volume(const float4 *probes, uint32_t n, unsigned int *scale_bits, uint8_t *out,
                             cudaStream_t st);

// The device rasteriser (raster.cu; raster.rs:39-114): the dirty tiles' texels (n_texels, the tiles in
// `tiles`, concatenated) from their triangles (RasterTri, in the host rasteriser's order), written into
// `tex` (64 bytes a texel, zero where uncovered); `scratch` holds n_texels claims; *pairs gets the number
// of (ds x ds block, chart) pairs over the covered texels (a bound on the gathered texels).
cudaError_t lb_raster_tiles(const RasterTri *tris, uint32_t n_tris, const DTile *tiles, uint32_t n_tiles,
                            uint32_t n_texels, uint32_t ds, float4 *tex, uint32_t *scratch,
                            unsigned long long *pairs, int sms, cudaStream_t st);
// The covered texels' indices in order (idx, *count) and each texel's place among them (inverse;
// 0xffffffff where not covered); temp: lb_raster_covered_temp(n_texels) bytes.
size_t lb_raster_covered_temp(uint32_t n_texels);
cudaError_t lb_raster_covered(const float4 *tex, uint32_t n_texels, void *temp, size_t temp_bytes, uint32_t *idx,
                              uint32_t *count, uint32_t *inverse, int sms, cudaStream_t st);
// The atlas owner map (aw x ah): each texel of a tile gets its place in the concatenated texel arrays,
// the rest 0xffffffff.
cudaError_t lb_owner_map(const DTile *tiles, uint32_t n_tiles, uint32_t aw, uint32_t ah, uint32_t *owner, int sms,
                         cudaStream_t st);

