/*
 * ORACLE — test infrastructure only. Nothing in the lightbaker_b200 package links, imports or calls
 * this; only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg do, as the checker.
 *
 * A scalar CPU restatement of the reference's bake passes:
 *   trace_ref.cpp   crates/lightbaker/src/gpu/trace.wgsl:41-324 (direct, gather, volume; trace()),
 *                   in FP32 with the shader's operation order, and the same walk in FP64
 *   filter_ref.cpp  crates/lightbaker/src/filter.rs:20-141 (smooth, fill, sun_field)
 *   bake_ref.cpp    the CPU work between the passes: raster.rs:39-114, layout.rs:69-85 (chart
 *                   coordinates), bake.rs:197-275 (per-tile post), :286-298 (gather selection),
 *                   :303-322 (bounce filters), :337-359 (volume fallback), :364-421 (composite),
 *                   :435-445 (write_light), volume.rs:86-147 (inside fill, irradiance)
 *   transport_ref.py  the bounce transport in float64 and its gradient (torch autograd)
 *   bvh_ref.cpp     crates/lightbaker/src/bvh.rs:50-162 (the binned SAH build, serial)
 *   bake_ref.py     a whole bake driven from these pieces (the layout and BVH as the product lays them
 *                   out; everything after, including the Params, restated)
 *
 * Parity status: the reference is Rust + wgpu and cannot run here (no Rust toolchain, no graphics
 * stack), and its tests hold no numeric golden vectors for these passes. The restatement is pinned by
 * the reference's own property tests (crates/lightbaker/tests/bake.rs:95-154, restated in
 * tests/test_bake_properties.py), its encode known-answer tests (encode.rs:150-180) and internal
 * consistency (FP64 twin); numeric parity with the WGSL is otherwise "parity unpinned".
 *
 * Build: oracle/build.py (g++ -O2 -ffp-contract=off -fopenmp): no fused multiply-add, so every
 * float operation rounds as the shader's source orders it.
 */
#ifndef LB_ORACLE_H
#define LB_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#include "../include/lightbaker.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Work the walk did, counted as lb_counters counts it on the device. */
typedef struct or_counters {
    uint64_t rays, nodes, tris, mats, overflows;
} or_counters;

/* One pass over n items, as Gpu::run: out gets n * width float4 records. threads <= 0: all cores. */
int or_run(int pass, const lb_node *nodes, size_t n_nodes, const lb_tri *tris, size_t n_tris,
           const float *materials, size_t n_materials, const float *charts, size_t n_charts,
           const lb_params *params, const lb_texel *items, size_t n, const float *light,
           size_t n_light, float *out, int threads, or_counters *counters);

/* or_run with the watertight triangle test over `verts` (9 floats a triangle, in tris order; NULL: the
 * shader's test), as lb_scene_set_vertices switches the kernels. */
int or_run_ex(int pass, const lb_node *nodes, size_t n_nodes, const lb_tri *tris, size_t n_tris,
              const float *materials, size_t n_materials, const float *charts, size_t n_charts,
              const lb_params *params, const lb_texel *items, size_t n, const float *light,
              size_t n_light, float *out, int threads, or_counters *counters, const float *verts);

/* One ray through the scene, in FP32 (precision 32) or FP64 (64); writes t, triangle
 * (0xffffffff: none), back face. `any`: the first accepted hit. */
int or_trace(int precision, const lb_node *nodes, size_t n_nodes, const lb_tri *tris, size_t n_tris,
             const float *materials, size_t n_materials, const lb_params *params, const float o[3],
             const float d[3], float tmax, int any, uint32_t ray, double *t, uint32_t *tri, int *back);
/* or_trace with the watertight test over `verts` for the FP32 walk (NULL: the shader's test). */
int or_trace_ex(int precision, const lb_node *nodes, size_t n_nodes, const lb_tri *tris, size_t n_tris,
                const float *materials, size_t n_materials, const lb_params *params, const float o[3],
                const float d[3], float tmax, int any, uint32_t ray, double *t, uint32_t *tri, int *back,
                const float *verts);

/* or_trace_ex over n rays (8 floats each, as lb_ray: o, tmax, d, key bits), in parallel. */
int or_trace_rays(int precision, const lb_node *nodes, size_t n_nodes, const lb_tri *tris, size_t n_tris,
                  const float *materials, size_t n_materials, const lb_params *params, const float *rays, size_t n,
                  int any, const float *verts, double *t, uint32_t *tri, int *back, int threads);
/* or_ray_ambiguous over n rays (as or_trace_rays), in parallel: out[i] 1 where ambiguous. */
int or_rays_ambiguous(const lb_node *nodes, size_t n_nodes, const lb_tri *tris, size_t n_tris,
                      const float *materials, size_t n_materials, const lb_params *params, const float *rays,
                      size_t n, double eps, int *out, int threads);

/* Is this ray within `eps` of deciding differently: does it pass, in FP64, within eps (barycentric)
 * of the edge of a triangle that stops it, or meet one within eps (relative) of 1e-4 or tmax? */
int or_ray_ambiguous(const lb_node *nodes, size_t n_nodes, const lb_tri *tris, size_t n_tris,
                     const float *materials, size_t n_materials, const lb_params *params,
                     const float o[3], const float d[3], float tmax, uint32_t ray, double eps);

/* The rays a pass casts for item i (origin, direction, tmax, any-hit flag, ray key), in the order the
 * shader casts them, for items whose outcome does not change the rays that follow: the sun and
 * occlusion rays of a direct item from its sample point (pick given), the gather rays, the volume's.
 * Returns the number of rays (at most cap). kind: 0 inside-test rays at the chosen point, 1 hard sun,
 * 2 soft sun, 3 occlusion, 4 gather, 5 volume sphere, 6 volume sun. */
size_t or_item_rays(int pass, const lb_params *params, const lb_texel *item, size_t index,
                    uint32_t pick, float *o, float *d, float *tmax, int *any, uint32_t *key,
                    int *kind, size_t cap);

/* Every gather ray's outcome for items[0..n) (4 words a ray, [item][ray]): kind (0 sky, 1 back face,
 * 2 surface), material, atlas texel of the hit (0xffffffff: none), bits of the direction's y. */
int or_gather_records(const lb_node *nodes, size_t n_nodes, const lb_tri *tris, size_t n_tris,
                      const float *materials, size_t n_materials, const float *charts, size_t n_charts,
                      const lb_params *params, const lb_texel *items, size_t n, size_t n_light,
                      uint32_t *records, int threads);

/* The shader's own helpers, for unit tests: pcg (trace.wgsl:41-45), rand (:46), radical (:49),
 * the sine and cosine both sides use. */
uint32_t or_pcg(uint32_t v);
float or_rand(uint32_t a, uint32_t b, uint32_t seed_bits);
float or_radical(uint32_t i);
void or_sincos(float a, float *s, float *c);

/* filter.rs restated (N channels interleaved). valid/known are bytes (0/1). */
void or_smooth(int w, int h, const uint32_t *chart, const float *normal /* 3 a texel */,
               const float *v, int channels, const uint8_t *valid, int r, float *out);
void or_fill(int w, int h, const uint32_t *chart, float *v, int channels, uint8_t *valid,
             int rings);
void or_sun_field(int w, int h, const uint32_t *chart, const float *normal, const uint32_t *hard,
                  const uint8_t *covered, int g, float radius, float *out);

/* ---- bake_ref.cpp: the reference's CPU work between the passes (bake.rs, raster.rs, volume.rs) ---- */

/* A chart as raster.rs reads it (layout.rs:20-40): plane axes, extent minimum, quarter turn, corner
 * in its tile, and its index in the layout (the texels' chart bits). */
typedef struct or_chart {
    float u[3], v[3], min[2];
    uint32_t turned, x, y, id;
} or_chart;

/* The bake settings the per-tile work reads (scene.rs BakeSettings, the sun, the layout's padding). */
typedef struct or_post_settings {
    float inside_share, ao_strength, ao_floor, ao_contrast, sdf_radius;
    float sun_irradiance[3], sun_dir[3] /* normalised */;
    int grid /* sqrt(sun_samples) */;
    uint32_t padding;
} or_post_settings;

/* layout.rs:76-85: the chart's map from a world point to atlas texels, two rows of 4. */
void or_chart_affine(const or_chart *c, uint32_t tile_x, uint32_t tile_y, float density, uint32_t padding,
                     float out[8]);
/* raster.rs:39-114: a w x h tile's texels from its charts (in the tile's order), chart ci's triangles
 * being pos[9 * tri_start[ci] .. 9 * tri_start[ci + 1]) (three vertices each). */
void or_raster_tile(int w, int h, const or_chart *charts, size_t n_charts, const uint32_t *tri_start,
                    const float *pos, float density, uint32_t padding, lb_texel *out);
/* bake.rs:197-275: one tile after the direct pass. `records` holds the pass's record of each covered
 * texel in row order; texels get their moved sample points. Writes valid (covered and not inside),
 * known (2 own light, 1 filled, 0 none), state (validity code), field, ao and direct (3 a texel).
 * Returns the records read. */
size_t or_tile_post(int w, int h, lb_texel *texels, const float *records, const or_post_settings *s,
                    uint8_t *valid, uint8_t *known, uint8_t *state, float *field, float *ao, float *direct);
/* bake.rs:286-298: where a tile's bounced light is gathered. */
void or_gather_select(int w, int h, const uint8_t *valid, const uint32_t *chart, uint32_t ds, uint8_t *gathered);
/* bake.rs:303-322: a tile's bounced light from the gather pass's records of its gathered texels (row
 * order): scattered, smoothed (radius gi_filter * ds) and filled (rings padding + 2 ds + 2). Returns
 * the records read. */
size_t or_bounce_tile(int w, int h, const uint32_t *chart, const float *normal, const uint8_t *gathered,
                      const float *records, uint32_t radius, uint32_t rings, float *e);
/* bake.rs:435-445: a tile's light into the atlas the gathers read (4 floats an atlas texel). */
void or_write_light(uint32_t tx, uint32_t ty, int w, int h, uint32_t atlas_width, const uint8_t *known,
                    const float *direct, const float *indirect, float *light);
/* volume.rs:86-120: probes inside solids filled from their neighbours, 8 rings (16 floats a probe). */
void or_volume_fill(uint32_t nx, uint32_t ny, uint32_t nz, float *probes);
/* bake.rs:337-359 with volume.rs:125-147: texels of a tile left without light lit from the volume.
 * Returns how many. */
size_t or_volume_fallback(int w, int h, const lb_texel *texels, const float *probes, uint32_t nx, uint32_t ny,
                          uint32_t nz, const float origin[3], float step, const float sun_irradiance[3],
                          const float sun_dir[3], uint8_t *known, uint8_t *state, float *field, float *ao,
                          float *direct, float *indirect);
/* bake.rs:364-421: the atlases from every tile (rects: x, y, w, h a tile; per-tile arrays): direct
 * (aw * ah * 2), validity (aw * ah), indirect (ceil(aw/ds) * ceil(ah/ds) * 3) with its 2 dilations. */
void or_composite(uint32_t aw, uint32_t ah, uint32_t ds, size_t n_tiles, const uint32_t *rects,
                  const uint8_t *const *known, const uint8_t *const *state, const float *const *field,
                  const float *const *ao, const float *const *indirect, float *direct_out, uint8_t *validity,
                  float *indirect_out);

/* ---- bvh_ref.cpp: the reference's BVH build (bvh.rs:50-162) ---- */

/* Bvh::build over every mesh's triangles (pos: 9 floats a triangle, meshes concatenated, mesh m's at
 * [mesh_first[m], mesh_first[m + 1])), skipping meshes whose material does not cast; tri_chart: each
 * triangle's chart (0xffffffff: none). Writes the nodes (when cap_nodes holds them all) and the triangles
 * (tris_out holds every triangle of the scene) and returns the node count. */
size_t or_bvh_build(const float *pos, const uint32_t *mesh_first, size_t n_meshes, const uint32_t *mesh_material,
                    const uint8_t *material_casts, const uint32_t *tri_chart, lb_node *nodes_out, size_t cap_nodes,
                    lb_tri *tris_out, size_t *n_tris_out);

#ifdef __cplusplus
}
#endif
#endif
