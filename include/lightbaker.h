/*
 * lightbaker-b200 C ABI.
 *
 * The drop-in seam for the bake passes of lightbaker: every function below replaces one piece of
 * the reference's `gpu::Gpu` boundary (crates/lightbaker/src/gpu/mod.rs) or of the bake entry point
 * built on it (crates/lightbaker/src/bake.rs, crates/lightbaker/src/lib.rs). Plain C types only:
 * pointers, sizes and the POD records the reference's shader reads, byte for byte.
 *
 * Conventions (mirroring the reference's anyhow::Result):
 *   - functions returning `int` give LB_OK (0) on success and a negative LB_E* code on failure;
 *     functions returning a handle give NULL on failure. Either way `lb_last_error()` holds a
 *     message for the calling thread.
 *   - the caller owns every host buffer passed in; it is only borrowed for the call.
 *   - a handle is used from one thread at a time (the reference drives its Gpu from the bake thread).
 */
#ifndef LIGHTBAKER_H
#define LIGHTBAKER_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- records the passes read and write (sizes and field order are the reference's) ---- */

/* BVH node, 32 bytes: crates/lightbaker/src/bvh.rs:12-22. count 0: inner node whose children are
 * `first` and `first + 1`; count > 0: leaf of `count` triangles from `first`. */
typedef struct lb_node {
    float min[3];
    uint32_t first;
    float max[3];
    uint32_t count;
} lb_node;

/* Triangle, 48 bytes: crates/lightbaker/src/bvh.rs:24-33. v0.w: material index bits;
 * e1.w: chart index bits (0xffffffff: none). */
typedef struct lb_tri {
    float v0[4];
    float e1[4];
    float e2[4];
} lb_tri;

/* Texel (or probe), 64 bytes: crates/lightbaker/src/raster.rs:11-22. pos.w: 1 where covered;
 * normal.w: chart index bits (a probe: its index in the volume). */
typedef struct lb_texel {
    float pos[4];
    float normal[4];
    float dx[4];
    float dy[4];
} lb_texel;

/* The passes' uniform block, 144 bytes: crates/lightbaker/src/gpu/mod.rs:11-23 and
 * crates/lightbaker/src/gpu/trace.wgsl:12-22. */
typedef struct lb_params {
    float sun_dir[4];   /* xyz towards the sun, w: tan of the disc's radius */
    float sun_irr[4];
    float zenith[4];
    float horizon[4];
    float ground[4];    /* w: reach of the inside-a-solid test (m) */
    float fallback[4];
    uint32_t counts[4]; /* sun grid side, ao rays, gather rays, items in this batch */
    float reach[4];     /* ao reach, gather reach, lift, seed bits */
    uint32_t atlas[4];  /* atlas width, height, first item, insideShare bits */
} lb_params;

/* crates/lightbaker/src/gpu/mod.rs:26-33; the result width is 1, 1 and 4 records a item. */
enum lb_pass { LB_PASS_DIRECT = 0, LB_PASS_GATHER = 1, LB_PASS_VOLUME = 2 };

enum lb_status {
    LB_OK = 0,
    LB_EINVAL = -1,    /* bad argument */
    LB_ENODEV = -2,    /* no CUDA device ("no GPU adapter", gpu/mod.rs:83) */
    LB_ECUDA = -3,     /* a CUDA call failed */
    LB_ENOMEM = -4,    /* device memory */
    /* -5 is not used: no kernel waits on another, and upload refuses a BVH2 a walk could loop in */
    LB_EIO = -6,       /* file or format error */
    LB_ESCRATCH = -7,  /* request larger than a fixed scratch area */
    LB_EEXCHANGE = -8  /* a split bake's sum (lb_exchange) failed */
};

typedef struct lb_gpu lb_gpu;
typedef struct lb_scene lb_scene;

/* Message for the last failure on this thread ("" if none). */
const char *lb_last_error(void);

/* Gpu::new (gpu/mod.rs:74-127): opens CUDA device `device` (an sm_100 part) and writes its name
 * (the reference's `pub adapter: String`, gpu/mod.rs:62) into name[0..cap). */
lb_gpu *lb_gpu_open(int device, char *name, size_t cap);
void lb_gpu_close(lb_gpu *gpu);

/* Gpu::scene (gpu/mod.rs:129-136): uploads the BVH, the materials (albedo rgb, opacity) and the
 * charts' affine rows (two float4 a chart). Empty charts: a one-chart dummy, as the reference. The
 * BVH must pass lb_bvh_check, or nothing is uploaded (NULL, the reason in lb_last_error). */
lb_scene *lb_scene_upload(lb_gpu *gpu, const lb_node *nodes, size_t n_nodes, const lb_tri *tris,
                          size_t n_tris, const float *materials /* 4 a material */, size_t n_materials,
                          const float *charts /* 8 a chart */, size_t n_charts);
void lb_scene_free(lb_scene *scene);
/* The checks lb_scene_upload makes of a BVH2 before anything reaches the device, on the host only:
 * every leaf inside the triangle array, and the nodes form a tree whose children follow their parent
 * as the reference allocates them (bvh.rs:93-101: an inner node's children at first > its own index,
 * no node with two parents; an inner node whose children lie past the array has none, the reference's
 * empty BVH). A cyclic or shared child would let a walk loop without end. LB_OK or LB_EINVAL. */
int lb_bvh_check(const lb_node *nodes, size_t n_nodes, size_t n_tris);
/* The triangles' exact vertices (9 floats a triangle: v0, v1, v2 of tris[i], in the uploaded order;
 * lb_prepared_get_vertices gives them for a prepared scene), or NULL and 0 to drop them. No counterpart in
 * the reference. With vertices every walk over this scene uses the watertight ray/triangle test (Woop,
 * Benthin and Wald, JCGT 2013) in place of the shader's Moller-Trumbore, and widens each box's exit by
 * 1 + 4e-7 so no box that holds a hit is culled: no ray passes between two triangles that share an
 * edge. Hit/miss, faces and t then differ from the shader's only for rays through an edge or a vertex
 * (within 1e-4 in barycentric terms), grazing a triangle, or ending within rounding of 1e-4 or tmax. */
int lb_scene_set_vertices(lb_gpu *gpu, lb_scene *scene, const float *verts, size_t n_tris);
/* The scene's 8-wide BVH (lb_set_bvh 8), which lb_scene_upload builds on the device from the BVH2: node
 * and triangle counts, and with non-NULL buffers the nodes (20 words each) and triangles (e2.w: the
 * triangle's index in the uploaded array). Equal byte for byte to lb_bvh8_collapse of the same BVH2.
 * No counterpart in the reference, whose walk uses the BVH2 only. */
int lb_scene_get_bvh8(lb_gpu *gpu, const lb_scene *scene, uint32_t *nodes8, lb_tri *tris8, uint64_t *n_nodes8,
                      uint64_t *n_tris8);

/* One ray for lb_trace: origin, maximum distance, direction, and its key (the ray number the shader's
 * opacity coin reads, trace.wgsl:69-72). */
typedef struct lb_ray {
    float o[3];
    float tmax;
    float d[3];
    uint32_t key;
} lb_ray;
/* Its hit: t (tmax when none), the triangle (its index in the uploaded order; 0xffffffff: none) and the
 * face (1: the ray met the back, the shader's det < 0). */
typedef struct lb_hit {
    float t;
    uint32_t tri;
    uint32_t back;
    uint32_t pad;
} lb_hit;
/* trace() (trace.wgsl:83-130) for each of n rays in host memory, with the handle's BVH (lb_set_bvh) and
 * the scene's triangle test: the nearest accepted hit, or with `any` the first accepted. seed: the bits
 * of params.reach[3], which the opacity coin mixes in. Blocking; results in the caller's `out`. No
 * counterpart in the reference (the shader's walk is internal to its passes); the passes' own rays
 * (oracle item rays) traced here give their hit/miss masks one ray at a time. */
int lb_trace(lb_gpu *gpu, lb_scene *scene, const lb_ray *rays, size_t n, int any, uint32_t seed, lb_hit *out);

/* Gpu::run (gpu/mod.rs:140-196): runs `pass` over `n` items, reading `light` (4 floats an atlas
 * texel; may be empty), writing n * width float4 records into the caller's `out` (width 4 for
 * LB_PASS_VOLUME, else 1). One launch over the list: item i is keyed as the shader keys it, by
 * params->atlas[2] + i (trace.wgsl:172-173). The bake's Params hold 0 there, as the reference's
 * Gpu::run gives its first batch; a caller running part of a longer list (one rank's shard of the
 * tiles) passes the index of its first item in the whole list, so every item keeps its key. */
int lb_run(lb_gpu *gpu, lb_scene *scene, int pass, const lb_params *params, const lb_texel *items,
           size_t n, const float *light, size_t n_light, float *out);

/* Rays traced and BVH work done by the last lb_run (or bake) on this handle, counted on the device
 * when counting is on (lb_set_counting). rays: every trace() call; nodes: node records fetched;
 * tris: triangles tested; mats: material records read by accepted candidates. */
typedef struct lb_counters {
    uint64_t rays, nodes, tris, mats;
} lb_counters;
int lb_set_counting(lb_gpu *gpu, int on);
int lb_get_counters(lb_gpu *gpu, lb_counters *out);

/* The handle's CUDA stream (a cudaStream_t), on which every pass is enqueued. No counterpart in the
 * reference (wgpu hides its queue); it lets a caller order its own work and events with the passes. */
void *lb_gpu_stream(lb_gpu *gpu);
/* Waits for the handle's stream, then moves the last pass's counters into lb_get_counters. */
int lb_gpu_sync(lb_gpu *gpu);
/* Gpu::run on items already in device memory: `items`, `light` and `out` are device pointers; the pass
 * is enqueued on the handle's stream and not waited for. `base` is the index of items[0] in the whole
 * list (it keys the sample sequence, as the shader's P.atlas.z + i). */
int lb_run_async(lb_gpu *gpu, lb_scene *scene, int pass, const lb_params *params, const lb_texel *items,
                 size_t n, uint32_t base, const float *light, size_t n_light, float *out);
/* Which kernels lb_run and lb_run_async use: 0 (default) one thread an item, as the shader is
 * dispatched; 1 one warp an item (the device-resident bake's kernels). Results are identical. */
int lb_set_pass_kernel(lb_gpu *gpu, int kind);
/* The warp kernels' ray order within an item: a warp's 32 rays of a round share the top `group` bits of
 * the ray index (and the bottom bits that remain): large values give the shader's order (bands of
 * elevation), 0 (the default) wedges of azimuth. Results are identical; speed is not (the device bake's
 * autotuner picks). */
int lb_set_ray_order(lb_gpu *gpu, int direct, int gather);
/* Leaf lists for the warp kernels' direct pass over the BVH2 (default on): a warp gathers once for a
 * texel the leaves within the occlusion reach (widened by its farthest candidate point) of its own point,
 * on its front side, nearest first, and its inside-test and occlusion rays test that list instead of
 * walking the tree. Same results: a ray whose list walk meets a tie the tree walk could settle another
 * way (an exact tie, or a near one where the hit's box entry rounds up to the hit) walks the tree. */
int lb_set_near(lb_gpu *gpu, int on);
/* Register cap of the warp kernels over the BVH2 (direct and gather, without counting): 0 (default) the
 * compiler's own budget; 3 or 4 registers capped so that this many 256-thread blocks share an SM (more
 * warps in flight, some values spilled). Same results. With 0, lb_bake_device and lb_plan_create without
 * autotuning use their own shapes: the 4-block cap without the shared sun walk (lb_set_warp_walk) for the
 * direct pass, the 3-block cap for the gathers; with 3 or 4 they use the handle's cap and walk. */
int lb_set_register_cap(lb_gpu *gpu, int blocks);
/* Lane refill in the warp kernels' occlusion and gather rays over the BVH2 (default off): a lane whose
 * ray has ended starts the item's next one instead of waiting for its round. Same results. */
int lb_set_refill(lb_gpu *gpu, int on);
/* Dynamic item fetch in the warp kernels' direct and gather passes and in lb_bake_device's untuned shapes
 * (default on): each warp takes its next item from a counter as soon as it is free, instead of a static
 * stride over the items, so warps behind heavy items no longer hold up the pass's end. Same results. */
int lb_set_fetch(lb_gpu *gpu, int on);
/* The warp kernels' direct pass over the BVH2 (default on): a texel's 32 sun rays (16 cells' hard and soft
 * rays, near-parallel, from within the texel) walk the tree together, one node at a time for the warp, each
 * lane testing its own ray; lanes leave subtrees their rays miss and the walk when their rays are stopped.
 * Used when the BVH2 has at most 48 inner nodes on any path (then no per-ray walk drops a child); the
 * same shadow bits, since whether a shadow ray is stopped does not depend on the order its triangles are
 * tested in. No counterpart in the reference. */
int lb_set_warp_walk(lb_gpu *gpu, int on);
/* The BVH the warp kernels walk: 2, the reference's (as uploaded); 8, the 8-wide BVH lb_scene_upload
 * collapses from it (80-byte nodes, 8-bit child boxes). Same hits, faces and records. */
int lb_set_bvh(lb_gpu *gpu, int width);
/* Bytes this handle copied host to device and device to host since the last reset. */
int lb_get_transfer(lb_gpu *gpu, uint64_t *h2d, uint64_t *d2h, int reset);


/* ---- the texel filters on the device (crates/lightbaker/src/filter.rs) ----
 * One tile of w x h texels, row by row; every array is in device memory; `channels` (1..4) floats a
 * texel, interleaved; chart: a texel's chart (0xffffffff: none); normal: 3 floats a texel. Enqueued on
 * the handle's stream (lb_gpu_sync waits). Results equal the reference's host functions. */
/* smooth (filter.rs:20-53): Gaussian mean (sigma = 0.75 r) of the valid texels on the same surface
 * (same chart, normals within n.n >= 0.9); radius 0..8. */
int lb_smooth(lb_gpu *gpu, uint32_t w, uint32_t h, const uint32_t *chart, const float *normal,
              const float *values, int channels, const uint8_t *valid, int radius, float *out);
/* fill (filter.rs:58-94): `rings` rings of filling texels without light from their neighbours, in place
 * (values and valid). Uses scratch the handle keeps (a ping-pong copy of the tile). */
int lb_fill(lb_gpu *gpu, uint32_t w, uint32_t h, const uint32_t *chart, float *values, int channels,
            uint8_t *valid, int rings);
/* lb_fill without allocating anything, for callers that cannot allocate device memory: a host
 * application that owns all of the GPU's memory through its own allocator (an engine or an editor
 * hosting the baker as a plugin), or a path where an allocation would synchronise the device while
 * other work is in flight. No counterpart in the reference. The fill's ping-pong copy lives in a
 * fixed 4.25 MiB device array that every GPU loading the library holds until exit; tiles of more
 * than 512 x 512 texels are rejected (LB_ESCRATCH). Arrays are device pointers as for lb_fill;
 * enqueued on `stream` (a cudaStream_t, NULL: the default stream) in the calling thread's current
 * CUDA context (the device's primary context unless the application made its own current). Each
 * context holds its own copy of the array at its own address: the first call in a context looks that
 * address up (cudaGetSymbolAddress) and caches it under the context's unique id, so make that first
 * call before any stream capture; made during a capture it is refused (LB_EINVAL) with nothing
 * launched. Calls share the array: calls that overlap on the GPU race. Nothing in it needs clearing:
 * each ring writes every texel of the copy it reads next. */
int lb_fill_fixed(void *stream, uint32_t w, uint32_t h, const uint32_t *chart, float *values, int channels,
                  uint8_t *valid, int rings);
/* sun_field (filter.rs:106-141): the sun's distance field from each texel's grid_side^2 hard bits
 * (grid side 1..5), 0.5 at a shadow's edge, 0 and 1 at `radius` texels; -1 where not covered. */
int lb_sun_field(lb_gpu *gpu, uint32_t w, uint32_t h, const uint32_t *chart, const float *normal,
                 const uint32_t *hard, const uint8_t *covered, uint32_t grid_side, float radius, float *out);

/* ---- the host pipeline (crates/lightbaker/src/bake.rs, lib.rs) ---- */

/* A scene read and laid out, with everything the passes read: the reference's steps before its
 * first Gpu::run (bake.rs:94-120): Scene::read (scene.rs:140-161), Layout::build, each chart's affine,
 * Bvh::build, the materials and the Params. */
typedef struct lb_prepared lb_prepared;
lb_prepared *lb_prepare(const uint8_t *scene, size_t len);
void lb_prepared_free(lb_prepared *p);

typedef struct lb_prepared_info {
    size_t n_nodes, n_tris, n_materials, n_charts, n_tiles, n_triangles;
    uint32_t atlas_width, atlas_height, indirect_downscale, padding;
    uint32_t gi_bounces, has_volume;
    lb_params params;
} lb_prepared_info;
int lb_prepared_get_info(const lb_prepared *p, lb_prepared_info *out);
/* Copies of the prepared arrays (caller-allocated, sized from the info). */
int lb_prepared_get_bvh(const lb_prepared *p, lb_node *nodes, lb_tri *tris);
int lb_prepared_get_materials(const lb_prepared *p, float *materials /* 4 a material */);
/* The BVH's triangles' vertices as the scene holds them (n_tris * 9 floats), for lb_scene_set_vertices. */
int lb_prepared_get_vertices(const lb_prepared *p, float *verts);
int lb_prepared_get_charts(const lb_prepared *p, float *charts /* 8 a chart */);
/* Tile t's rectangle (x, y, w, h in the atlas) and key. */
int lb_prepared_get_tile(const lb_prepared *p, size_t t, uint32_t rect[4], int32_t key[2]);
/* Tile t's charts, in the layout's order (layout.rs:45-54 `Tile::charts`): the count, and with a
 * buffer the first `cap` chart indices. */
size_t lb_prepared_get_tile_charts(const lb_prepared *p, size_t t, uint32_t *charts, size_t cap);
/* Chart c of the layout (layout.rs:20-40 `Chart`): its plane (normal, axes u and v, the extent min/max
 * on them), tile key, quarter turn, size and corner in its tile; the count of its triangles, and with
 * a buffer the first `cap` of them (indices into its mesh, in mesh order). */
typedef struct lb_chart_frame {
    uint32_t mesh, turned, x, y, w, h;
    int32_t tile[2];
    float normal[3], u[3], v[3], min[2], max[2];
} lb_chart_frame;
size_t lb_prepared_get_chart(const lb_prepared *p, size_t c, lb_chart_frame *frame, uint32_t *tris, size_t cap);
/* raster.rs:39-100: tile t's texels (w * h records, row by row). */
int lb_prepared_rasterize(const lb_prepared *p, size_t t, lb_texel *out);

/* A pass runner the bake can use in place of a device (the reference's `bake(scene, &Gpu, …)`
 * takes its device the same way): upload the scene, then run passes. Return 0 on success. */
typedef struct lb_tracer {
    void *ctx;
    int (*scene)(void *ctx, const lb_node *nodes, size_t n_nodes, const lb_tri *tris, size_t n_tris,
                 const float *materials, size_t n_materials, const float *charts, size_t n_charts);
    int (*run)(void *ctx, int pass, const lb_params *params, const lb_texel *items, size_t n,
               const float *light, size_t n_light, float *out, uint64_t *rays);
} lb_tracer;

/* How the ranks of a bake split over several processes (one a GPU) exchange what the others need (the
 * drop-in bake: the light atlas after each bounce, the probes, the atlases' pieces and some counts; the
 * device-resident bake: each ray pass's outputs, in device memory). No counterpart in the
 * reference (one process bakes everything). `sum` adds `count` 32-bit words at `data` element-wise over
 * every rank, in place, as unsigned integers: every exchanged word is written by one rank and zero on
 * the others, so the sum carries that rank's bits exactly (floats included). device: 0 host memory, 1
 * device memory (the library's stream is synchronised before the call). 0 on success. Every rank makes
 * the same calls in the same order. */
typedef struct lb_exchange {
    void *ctx;
    int rank, world;
    int (*sum)(void *ctx, void *data, size_t count, int device);
} lb_exchange;

typedef struct lb_bake_options {
    const char *cache_dir;                      /* NULL: no cache (bake.rs:30-34) */
    void (*log)(void *ctx, const char *line);   /* NULL: quiet */
    void *log_ctx;
    int autotune;                               /* device bake: time the passes' shapes on a sample first */
    int trace_every_bounce;                     /* device bake: trace the gather rays again in every bounce
                                                 * (default 0: the first bounce records each ray's outcome
                                                 * and later bounces evaluate the records; same results) */
    int watertight;                             /* the watertight triangle test (lb_scene_set_vertices) in
                                                 * every pass; such tiles are cached apart (default 0: the
                                                 * shader's test) */
    const lb_exchange *exchange;                /* NULL: one process bakes every tile. Else this rank bakes its
                                                 * share (lb_bake_run: of the dirty tiles, contiguous in tile
                                                 * order, balanced by their texels, and of the probe chunks;
                                                 * lb_bake_device / lb_plan_create: of every ray pass's items,
                                                 * contiguous, equal counts), and every rank returns the whole
                                                 * bake, equal to one process's bit for bit */
} lb_bake_options;

typedef struct lb_bake lb_bake;
/* bake() (bake.rs:94-432) with the passes on `gpu`. */
lb_bake *lb_bake_run(lb_gpu *gpu, const uint8_t *scene, size_t len, const lb_bake_options *opts);
/* The same with the passes on a caller's runner. */
lb_bake *lb_bake_run_with(const lb_tracer *tracer, const uint8_t *scene, size_t len, const lb_bake_options *opts);
void lb_bake_free(lb_bake *b);

typedef struct lb_bake_info {
    uint32_t width, height, indirect_width, indirect_height;
    uint32_t has_volume, volume_size[3];
    float volume_origin[3], volume_step;
    uint64_t tiles, tiles_baked, texels_baked, chunks, chunks_baked;
    double seconds;
    uint64_t rays_direct, rays_gather, rays_volume;
    double t_layout, t_direct, t_bounces, t_volume, t_composite;
    uint64_t n_charts, n_triangles;
} lb_bake_info;
int lb_bake_get_info(const lb_bake *b, lb_bake_info *out);
int lb_bake_get_direct(const lb_bake *b, float *out /* 2 an atlas texel: field, ao */);
int lb_bake_get_indirect(const lb_bake *b, float *out /* 3 a texel of the smaller atlas */);
int lb_bake_get_validity(const lb_bake *b, uint8_t *out);
int lb_bake_get_volume(const lb_bake *b, float *out /* 16 a probe */);
/* The layout the bake used: each chart's affine rows (8 floats a chart, layout.rs:76-85) and each
 * scene triangle's chart (meshes in order, 0xffffffff: none; layout.rs:64-65). */
int lb_bake_get_charts(const lb_bake *b, float *out);
int lb_bake_get_tri_charts(const lb_bake *b, uint32_t *out);
/* output::write (output.rs:95-154): the .lbake file. *out is malloc'd; free with lb_free. */
int lb_bake_write(const lb_bake *b, uint8_t **out, size_t *len);
/* 1 when the bake's file encodings (BC5 of `direct`, RGB9E5 of `indirect`, the probes' bytes) were made
 * on the device by lb_bake_device, which lb_bake_write then uses as they are (the same bytes the host's
 * encoders give); 0 when lb_bake_write encodes on the host. */
int lb_bake_device_encoded(const lb_bake *b);
void lb_free(void *p);

/* ---- the device-resident bake (the batched mode) ---- */

/* bake() with every dirty tile rebaked in one CUDA graph on `gpu`: the host lays out, builds the BVH,
 * hashes and rasterises (bake.rs:94-149); the device runs the ray passes over all dirty tiles at once,
 * the texel passes, the bounces, the volume and the atlas. Results equal lb_bake_run's. */
lb_bake *lb_bake_device(lb_gpu *gpu, const uint8_t *scene, size_t len, const lb_bake_options *opts);

/* The same in steps, for a caller that rebakes the same dirty set: create (host work, uploads, the
 * graph captured), launch (the graph enqueued on the handle's stream; may be repeated), result (waits,
 * downloads, writes the cache; a bake handle). lb_plan_rays gives the rays of the last launch a pass:
 * direct, gather (all bounces), volume (a split bake: this rank's). With an exchange the graph is cut
 * after each ray pass and lb_plan_launch returns once the last piece is enqueued, having synchronised
 * the stream and made the sums between the pieces (LB_EEXCHANGE when a sum fails). */
typedef struct lb_plan lb_plan;
lb_plan *lb_plan_create(lb_gpu *gpu, const uint8_t *scene, size_t len, const lb_bake_options *opts);
int lb_plan_launch(lb_plan *plan);
int lb_plan_rays(lb_plan *plan, uint64_t rays[3]);
lb_bake *lb_plan_result(lb_plan *plan);
/* Kernel launches in one launch of the plan's graph. */
int lb_plan_kernels(const lb_plan *plan);
/* What the autotuner chose for the plan ("" when it did not run). */
const char *lb_plan_tuning(const lb_plan *plan);
void lb_plan_free(lb_plan *plan);

/* The bounce transport and its adjoint: the bake's indirect atlas as a function of the scene's light
 * parameters theta, and the gradient of a loss on that atlas with respect to theta. No reference
 * counterpart: the reference bakes at the scene's own values only (bake.rs:300-421 is the function
 * differentiated here).
 *
 * theta (3 * n_materials + 10 floats): every material's albedo (rgb, scene.rs:62-75), the sky's zenith,
 * horizon and ground (rgb each, scene.rs:53-60), and the sun's intensity as a scale on its irradiance
 * (1 = the scene's own). lb_transport_theta0 gives the scene's own theta; forward at it gives the
 * device bake's indirect atlas bit for bit. Visibility does not depend on theta: create traces every
 * gather ray once and records what it met. Texels lit by the volume's fallback (validity 5,
 * bake.rs:335-359) take their light from the probes, which the transport evaluates from its own last
 * bounce's light and theta (create records every volume ray too), then fills and interpolates as the
 * bake does; the adjoint runs those steps transposed (the cosine lobe's clamp at 0 as in the forward).
 *
 * create bakes the scene once on the device (every tile, no cache) and keeps what the transport reads;
 * max_checkpoints bounds the light atlases the forward keeps for the backward (0: one a bounce); with
 * fewer than the bounces, backward recomputes the others from the nearest earlier one, and its result
 * is the same bits. forward / backward take and give host arrays and wait; the _async forms take device
 * pointers and only enqueue on the gpu handle's stream. backward differentiates the last forward: its
 * input is d(loss)/d(indirect) (indirect_width x indirect_height float4, w ignored), its output
 * d(loss)/d(theta). Gradients are deterministic (fixed-order sums, in double for theta). */
typedef struct lb_transport lb_transport;
typedef struct lb_transport_shape {
    uint32_t n_materials, n_params, bounces, checkpoints;
    uint32_t indirect_width, indirect_height, gathered, rays;
    uint64_t records, lit_records, unlit_records, checkpoint_bytes;
} lb_transport_shape;
lb_transport *lb_transport_create(lb_gpu *gpu, const uint8_t *scene, size_t len, uint32_t max_checkpoints);
int lb_transport_info(const lb_transport *t, lb_transport_shape *out);
int lb_transport_theta0(const lb_transport *t, float *theta);
int lb_transport_forward(lb_transport *t, const float *theta, float *indirect);
int lb_transport_backward(lb_transport *t, const float *g_indirect, float *g_theta);
int lb_transport_forward_async(lb_transport *t, const float *d_theta, float *d_indirect);
int lb_transport_backward_async(lb_transport *t, const float *d_g_indirect, float *d_g_theta);
/* The indirect atlas of the bake create ran (float4 a texel). */
int lb_transport_bake_indirect(lb_transport *t, float *indirect);
/* A copy of one of the transport's fixed arrays, for tests ("records", "gathered_index", "texels", "sample_points",
 * "chart", "gathered", "known", "known_bounce", "state", "direct_light", "fixed_indirect", "owner",
 * "light_flags", "tiles", "smooth_weights", "shape"; and the bake's arrays as it left them: "direct_records"
 * (the direct pass's record of each covered texel), "valid", "field", "ao", "direct" and "indirect_light"
 * (float4 a texel), "gather_out" (the last bounce's gather results), "light" (the last light atlas),
 * "probes"; and the volume's share, empty when no texel takes the fallback: "volume_records",
 * "volume_items", "volume_slots", "volume_raw" (the probes before the fill), "volume_grid"): its size in
 * bytes when out is NULL, else the bytes copied (0 on error, with lb_last_error set; 0 with it empty: an
 * empty array). */
size_t lb_transport_export(lb_transport *t, const char *name, void *out, size_t cap);
void lb_transport_free(lb_transport *t);

/* Scene::write (scene.rs:164-181) from a JSON header and positions: for tools and tests that make
 * scenes. header_json is the header as the file holds it. */
int lb_scene_encode(const char *header_json, const float *const *positions, const size_t *n_floats,
                    size_t n_meshes, uint8_t **out, size_t *len);
/* Collapses a BVH2 into the 8-wide BVH the device walks and checks it (every triangle in exactly one
 * leaf, every box inside its parent's slot): LB_OK, its node count and depth; for tests and tools. */
int lb_bvh8_check(const lb_node *nodes, size_t n_nodes, const lb_tri *tris, size_t n_tris, uint64_t *n_nodes8,
                  uint64_t *depth);
/* The same collapse on the host: counts, and with non-NULL buffers the nodes and triangles, as
 * lb_scene_get_bvh8 returns them; for tests of the device build. */
int lb_bvh8_collapse(const lb_node *nodes, size_t n_nodes, const lb_tri *tris, size_t n_tris, uint32_t *nodes8,
                     lb_tri *tris8, uint64_t *n_nodes8, uint64_t *n_tris8);
/* blake3 of a byte string (the hash the cache is keyed by), 32 bytes. */
void lb_blake3(const uint8_t *data, size_t len, uint8_t out[32]);
/* encode.rs: RGB9E5 and BC4 blocks, for format tests. */
uint32_t lb_rgb9e5(const float c[3]);
/* lb_rgb9e5 on the device over n float4 texels (rgb; w ignored) in device memory, into n words there,
 * enqueued on the handle's stream: the encoder the device-resident bake runs on its indirect atlas
 * (encode.cu), equal to lb_rgb9e5 bit for bit. No counterpart in the reference (encode.rs:53-70 runs on
 * the CPU). */
int lb_rgb9e5_device(lb_gpu *gpu, const float *rgba, size_t n, uint32_t *out);
void lb_rgb9e5_decode(uint32_t p, float out[3]);
void lb_bc4_block(const uint8_t v[16], uint8_t out[8]);

#ifdef __cplusplus
}
#endif
#endif
