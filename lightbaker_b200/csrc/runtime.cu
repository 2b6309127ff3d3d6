// The C ABI's device side: open a device, upload a scene, run a pass (crates/lightbaker/src/gpu/mod.rs).
//
// The reference runs a pass in batches of 65536 / 16384 / 8192 items, each with a new uniform buffer,
// result buffer and bind group, submitted and waited on before the next (gpu/mod.rs:140-196). Here a
// pass is one launch over every item: the shader keys its samples by P.atlas.z + i, the item's index
// in the whole list, so the batch split never changes a result, and there is no display watchdog to
// keep dispatches short for on a compute GPU. Device buffers are kept by the handle and grown, not
// allocated per call.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "lb_device.cuh"
#include "lb_kernels.h"
#include "lb_runtime.h"

static thread_local std::string g_error;

void lb_set_error(const std::string &msg) { g_error = msg; }

int lb_cuda_fail(cudaError_t e, const char *what) {
    char buf[512];
    snprintf(buf, sizeof buf, "%s: %s (%s)", what, cudaGetErrorString(e), cudaGetErrorName(e));
    g_error = buf;
    return e == cudaErrorMemoryAllocation ? LB_ENOMEM : LB_ECUDA;
}

#define LB_CUDA(call, what)                                          \
    do {                                                             \
        cudaError_t e_ = (call);                                     \
        if (e_ != cudaSuccess) return lb_cuda_fail(e_, what);        \
    } while (0)

int lb_buffer_reserve(lb_buffer &b, size_t bytes) {
    if (bytes <= b.cap) return LB_OK;
    if (b.ptr) cudaFree(b.ptr);
    b.ptr = nullptr;
    b.cap = 0;
    size_t want = bytes + bytes / 4;
    cudaError_t e = cudaMalloc(&b.ptr, want);
    if (e != cudaSuccess) {
        b.ptr = nullptr;
        return lb_cuda_fail(e, "cudaMalloc");
    }
    b.cap = want;
    return LB_OK;
}

int lb_host_stage_reserve(lb_gpu *g, size_t bytes) {
    if (bytes <= g->stage_cap) return LB_OK;
    cudaError_t e = cudaStreamSynchronize(g->stream);  // no copy into the old buffer is in flight
    if (e != cudaSuccess) return lb_cuda_fail(e, "lb_host_stage_reserve");
    if (g->stage) cudaFreeHost(g->stage);
    g->stage = nullptr;
    g->stage_cap = 0;
    size_t want = bytes + bytes / 4;
    e = cudaHostAlloc(&g->stage, want, cudaHostAllocDefault);
    if (e != cudaSuccess) {
        g->stage = nullptr;
        return lb_cuda_fail(e, "cudaHostAlloc");
    }
    g->stage_cap = want;
    return LB_OK;
}

void lb_buffer_free(lb_buffer &b) {
    if (b.ptr) cudaFree(b.ptr);
    b.ptr = nullptr;
    b.cap = 0;
}

namespace {
constexpr size_t SPARE_LIMIT = size_t(24) << 30;  // device memory the spares may hold
}  // namespace

void *lb_spare_take(lb_gpu *g, size_t bytes, size_t *cap) {
    std::lock_guard<std::mutex> lock(g->spare_mu);
    size_t best = g->spare.size();
    for (size_t i = 0; i < g->spare.size(); i++) {
        size_t c = g->spare[i].second;
        if (c >= bytes && c <= 2 * bytes + (size_t(1) << 20) && (best == g->spare.size() || c < g->spare[best].second))
            best = i;
    }
    if (best == g->spare.size()) return nullptr;
    void *p = g->spare[best].first;
    *cap = g->spare[best].second;
    g->spare_bytes -= *cap;
    g->spare.erase(g->spare.begin() + std::ptrdiff_t(best));  // the others keep their order, oldest first
    return p;
}

void lb_spare_give(lb_gpu *g, void *p, size_t cap) {
    if (!p) return;
    cudaStreamSynchronize(g->stream);
    if (cap > SPARE_LIMIT) {
        cudaFree(p);
        return;
    }
    // the newest buffer stays and the oldest spares go when the limit would be passed: a caller that bakes
    // again and again keeps its own buffers, whatever other work left spares before
    std::vector<void *> out;
    {
        std::lock_guard<std::mutex> lock(g->spare_mu);
        size_t k = 0;
        while (g->spare_bytes + cap > SPARE_LIMIT && k < g->spare.size()) {
            out.push_back(g->spare[k].first);
            g->spare_bytes -= g->spare[k].second;
            k++;
        }
        g->spare.erase(g->spare.begin(), g->spare.begin() + std::ptrdiff_t(k));
        g->spare.emplace_back(p, cap);
        g->spare_bytes += cap;
    }
    for (void *q : out) cudaFree(q);
}

extern "C" {

const char *lb_last_error(void) { return g_error.c_str(); }

lb_gpu *lb_gpu_open(int device, char *name, size_t cap) {
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0) {
        lb_set_error(std::string("no GPU adapter: ") + (e != cudaSuccess ? cudaGetErrorString(e) : "no CUDA device"));
        return nullptr;
    }
    if (device < 0 || device >= count) {
        lb_set_error("no GPU device " + std::to_string(device));
        return nullptr;
    }
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) {
        lb_set_error("no GPU device: cudaGetDeviceProperties failed");
        return nullptr;
    }
    if (prop.major != 10 || prop.minor != 0) {
        lb_set_error(std::string("no GPU device: ") + prop.name + " is sm_" + std::to_string(prop.major) +
                     std::to_string(prop.minor) + "; this build is for sm_100a (B200)");
        return nullptr;
    }
    if (cudaSetDevice(device) != cudaSuccess) {
        lb_set_error("no GPU device: cudaSetDevice failed");
        return nullptr;
    }
    lb_gpu *g = new lb_gpu();
    g->device = device;
    g->sms = prop.multiProcessorCount;
    snprintf(g->name, sizeof g->name, "%s (CUDA, sm_%d%d, %d SMs)", prop.name, prop.major, prop.minor, prop.multiProcessorCount);
    if (cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMalloc(&g->counters, 8 * sizeof(unsigned long long)) != cudaSuccess ||
        cudaMallocHost(&g->host_counters, 8 * sizeof(unsigned long long)) != cudaSuccess ||
        cudaMemset(g->counters, 0, 8 * sizeof(unsigned long long)) != cudaSuccess) {
        lb_set_error("no GPU device: stream or counter allocation failed");
        delete g;
        return nullptr;
    }
    if (name && cap) {
        strncpy(name, g->name, cap - 1);
        name[cap - 1] = 0;
    }
    return g;
}

void lb_gpu_close(lb_gpu *g) {
    if (!g) return;
    cudaSetDevice(g->device);
    cudaStreamSynchronize(g->stream);
    for (auto &s : g->spare) cudaFree(s.first);
    g->spare.clear();
    lb_buffer_free(g->items);
    lb_buffer_free(g->out);
    lb_buffer_free(g->light);
    lb_buffer_free(g->scratch);
    if (g->counters) cudaFree(g->counters);
    if (g->host_counters) cudaFreeHost(g->host_counters);
    if (g->stage) cudaFreeHost(g->stage);
    cudaStreamDestroy(g->stream);
    delete g;
}

int lb_bvh_check(const lb_node *nodes, size_t n_nodes, size_t n_tris) {
    if (!nodes || n_nodes == 0) {
        lb_set_error("lb_bvh_check: no nodes");
        return LB_EINVAL;
    }
    // every leaf inside the triangle array (an inner node whose children lie past the node array is the
    // reference's empty BVH: every walk and the 8-wide build treat it as having no children)
    for (size_t i = 0; i < n_nodes; i++)
        if (nodes[i].count > 0 && uint64_t(nodes[i].first) + nodes[i].count > n_tris) {
            lb_set_error("lb_bvh_check: BVH leaf " + std::to_string(i) + " reaches past the triangle array");
            return LB_EINVAL;
        }
    // A tree whose children come after their parent, as the reference allocates them (bvh.rs:93-101): each inner
    // node's children lie above its own index and no node has two parents. Every walk then visits each node at
    // most once a ray and ends; a cyclic or shared child would make a walk loop or repeat without bound.
    std::vector<uint8_t> parent(n_nodes, 0);
    for (size_t i = 0; i < n_nodes; i++) {
        if (nodes[i].count > 0 || uint64_t(nodes[i].first) + 1 >= n_nodes) continue;
        uint32_t c = nodes[i].first;
        if (c <= i || parent[c] || parent[c + 1]) {
            lb_set_error("lb_bvh_check: BVH node " + std::to_string(i) +
                         " is not a tree node (its children must follow it and have no other parent)");
            return LB_EINVAL;
        }
        parent[c] = parent[c + 1] = 1;
    }
    return LB_OK;
}

lb_scene *lb_scene_upload(lb_gpu *g, const lb_node *nodes, size_t n_nodes, const lb_tri *tris, size_t n_tris,
                          const float *materials, size_t n_materials, const float *charts, size_t n_charts) {
    if (!g || !nodes || n_nodes == 0 || (n_tris && !tris) || (n_materials && !materials) || (n_charts && !charts)) {
        lb_set_error("lb_scene_upload: bad arguments");
        return nullptr;
    }
    if (n_nodes > 0x7fffffffu || n_tris > 0x7fffffffu) {
        lb_set_error("lb_scene_upload: more than 2^31 nodes or triangles");
        return nullptr;
    }
    if (lb_bvh_check(nodes, n_nodes, n_tris) != LB_OK) return nullptr;
    cudaSetDevice(g->device);
    lb_scene *s = new lb_scene();
    s->gpu = g;
    // an empty list still gets one record, as the reference's dummy chart (gpu/mod.rs:134)
    static const float zero[8] = {0};
    struct Part {
        void **dst;
        const void *src;
        size_t bytes;
    } parts[4] = {
        {&s->nodes, nodes, n_nodes * sizeof(lb_node)},
        {&s->tris, n_tris ? (const void *)tris : zero, (n_tris ? n_tris : 1) * sizeof(lb_tri)},
        {&s->mats, n_materials ? (const void *)materials : zero, (n_materials ? n_materials : 1) * 16},
        {&s->charts, n_charts ? (const void *)charts : zero, (n_charts ? n_charts : 1) * 32},
    };
    static const lb_tri zero_tri = {};
    if (!n_tris) parts[1].src = &zero_tri;
    for (auto &p : parts) {
        cudaError_t e = cudaMalloc(p.dst, p.bytes);
        if (e == cudaSuccess) e = cudaMemcpy(*p.dst, p.src, p.bytes, cudaMemcpyHostToDevice);
        g->h2d += p.bytes;
        if (e != cudaSuccess) {
            lb_cuda_fail(e, "lb_scene_upload");
            lb_scene_free(s);
            return nullptr;
        }
    }
    s->n_nodes = uint32_t(n_nodes);
    s->n_tris = uint32_t(n_tris);
    s->n_mats = uint32_t(n_materials);
    s->n_charts = uint32_t(n_charts);
    {
        // the most inner nodes on a path (children follow their parent: lb_bvh_check), for the warp walks
        std::vector<uint32_t> d(n_nodes, 0);
        uint32_t most = 0;
        for (size_t i = 0; i < n_nodes; i++) {
            if (nodes[i].count > 0 || uint64_t(nodes[i].first) + 1 >= n_nodes) continue;
            uint32_t here = d[i] + 1;
            most = std::max(most, here);
            d[nodes[i].first] = d[nodes[i].first + 1] = here;
        }
        s->depth = most;
    }
    // the 8-wide BVH over the same triangles, collapsed on the device from the BVH2 just uploaded
    if (lb_bvh8_build(g, s) != LB_OK) {
        lb_scene_free(s);
        return nullptr;
    }
    return s;
}

}  // extern "C"

lbd::Scene lb_scene_view(const lb_scene *s) {
    lbd::Scene S{(const float4 *)s->nodes, (const float4 *)s->tris, (const float4 *)s->mats, (const float4 *)s->charts,
                 s->n_nodes, s->n_tris, s->n_mats, s->n_charts};
    S.nodes8 = (const uint4 *)s->nodes8;
    S.tris8 = (const float4 *)s->tris8;
    S.verts = (const float4 *)s->verts;
    S.grow = s->verts ? 1.0000004f : 1.0f;
    S.depth = s->depth;
    return S;
}

extern "C" {

void lb_scene_free(lb_scene *s) {
    if (!s) return;
    cudaSetDevice(s->gpu->device);
    for (void *p : {s->nodes, s->tris, s->mats, s->charts, s->nodes8, s->tris8, s->verts})
        if (p) cudaFree(p);
    delete s;
}

int lb_scene_set_vertices(lb_gpu *g, lb_scene *s, const float *verts, size_t n_tris) {
    if (!g || !s || s->gpu != g || (verts && n_tris != s->n_tris) || (!verts && n_tris)) {
        lb_set_error("lb_scene_set_vertices: bad arguments (one vertex triple for each uploaded triangle)");
        return LB_EINVAL;
    }
    LB_CUDA(cudaSetDevice(g->device), "cudaSetDevice");
    LB_CUDA(cudaStreamSynchronize(g->stream), "lb_scene_set_vertices");
    if (s->verts) {
        cudaFree(s->verts);
        s->verts = nullptr;
    }
    if (!verts || n_tris == 0) return LB_OK;
    std::vector<float> v4(n_tris * 12, 0.0f);
    for (size_t i = 0; i < n_tris * 3; i++)
        for (int k = 0; k < 3; k++) v4[i * 4 + k] = verts[i * 3 + k];
    size_t bytes = v4.size() * sizeof(float);
    void *p = nullptr;
    LB_CUDA(cudaMalloc(&p, bytes), "lb_scene_set_vertices");
    cudaError_t e = cudaMemcpy(p, v4.data(), bytes, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        cudaFree(p);
        return lb_cuda_fail(e, "lb_scene_set_vertices");
    }
    g->h2d += bytes;
    s->verts = p;
    return LB_OK;
}

int lb_scene_get_bvh8(lb_gpu *g, const lb_scene *s, uint32_t *nodes8, lb_tri *tris8, uint64_t *n_nodes8,
                      uint64_t *n_tris8) {
    if (!g || !s || s->gpu != g || !s->nodes8 || !s->tris8) {
        lb_set_error("lb_scene_get_bvh8: bad arguments");
        return LB_EINVAL;
    }
    if (n_nodes8) *n_nodes8 = s->n_nodes8;
    if (n_tris8) *n_tris8 = s->n_tris8;
    LB_CUDA(cudaSetDevice(g->device), "cudaSetDevice");
    LB_CUDA(cudaStreamSynchronize(g->stream), "lb_scene_get_bvh8");
    const size_t nb = size_t(s->n_nodes8) * 80, tb = size_t(s->n_tris8) * sizeof(lb_tri);
    if (nodes8) LB_CUDA(cudaMemcpy(nodes8, s->nodes8, nb, cudaMemcpyDeviceToHost), "lb_scene_get_bvh8");
    if (tris8) LB_CUDA(cudaMemcpy(tris8, s->tris8, tb, cudaMemcpyDeviceToHost), "lb_scene_get_bvh8");
    g->d2h += (nodes8 ? nb : 0) + (tris8 ? tb : 0);
    return LB_OK;
}

int lb_run(lb_gpu *g, lb_scene *s, int pass, const lb_params *params, const lb_texel *items, size_t n,
           const float *light, size_t n_light, float *out) {
    if (!g || !s || !params || pass < 0 || pass > 2 || (n && (!items || !out)) || (n_light && !light)) {
        lb_set_error("lb_run: bad arguments");
        return LB_EINVAL;
    }
    if (n == 0) return LB_OK;  // gpu/mod.rs:143-145
    if (n > 0xffffffffu / 8) {
        lb_set_error("lb_run: more than 2^29 items in one pass");
        return LB_EINVAL;
    }
    LB_CUDA(cudaSetDevice(g->device), "cudaSetDevice");
    size_t width = pass == LB_PASS_VOLUME ? 4 : 1;
    int rc;
    if ((rc = lb_buffer_reserve(g->items, n * sizeof(lb_texel))) != LB_OK) return rc;
    if ((rc = lb_buffer_reserve(g->out, n * width * 16)) != LB_OK) return rc;
    size_t nl = n_light ? n_light : 1;
    if ((rc = lb_buffer_reserve(g->light, nl * 16)) != LB_OK) return rc;
    LB_CUDA(cudaMemcpyAsync(g->items.ptr, items, n * sizeof(lb_texel), cudaMemcpyHostToDevice, g->stream), "copy items");
    g->h2d += n * sizeof(lb_texel);
    if (n_light) {
        LB_CUDA(cudaMemcpyAsync(g->light.ptr, light, n_light * 16, cudaMemcpyHostToDevice, g->stream), "copy light");
        g->h2d += n_light * 16;
    } else {
        LB_CUDA(cudaMemsetAsync(g->light.ptr, 0, 16, g->stream), "clear light");
    }
    lb_params P = *params;
    P.counts[3] = uint32_t(n);
    // one launch over the whole list: item i keyed by atlas.z + i (0 in the bake's Params; a shard passes its
    // first item's index in the whole list)
    const uint32_t base = params->atlas[2];
    rc = lb_run_device(g, s, pass, P, (const float4 *)g->items.ptr, uint32_t(n), base, (const float4 *)g->light.ptr,
                       uint32_t(nl), (float4 *)g->out.ptr);
    if (rc != LB_OK) return rc;
    LB_CUDA(cudaMemcpyAsync(out, g->out.ptr, n * width * 16, cudaMemcpyDeviceToHost, g->stream), "copy results");
    g->d2h += n * width * 16;
    LB_CUDA(cudaStreamSynchronize(g->stream), "lb_run");
    lb_collect_counters(g);
    return LB_OK;
}

void *lb_gpu_stream(lb_gpu *g) { return g ? (void *)g->stream : nullptr; }

int lb_gpu_sync(lb_gpu *g) {
    if (!g) return LB_EINVAL;
    LB_CUDA(cudaStreamSynchronize(g->stream), "lb_gpu_sync");
    lb_collect_counters(g);
    return LB_OK;
}

int lb_run_async(lb_gpu *g, lb_scene *s, int pass, const lb_params *params, const lb_texel *items, size_t n,
                 uint32_t base, const float *light, size_t n_light, float *out) {
    if (!g || !s || !params || pass < 0 || pass > 2 || (n && (!items || !out)) || !light || n_light == 0) {
        lb_set_error("lb_run_async: bad arguments (light must hold at least one record)");
        return LB_EINVAL;
    }
    if (n == 0) return LB_OK;
    if (n > 0xffffffffu / 8) {
        lb_set_error("lb_run_async: more than 2^29 items in one pass");
        return LB_EINVAL;
    }
    LB_CUDA(cudaSetDevice(g->device), "cudaSetDevice");
    lb_params P = *params;
    P.counts[3] = uint32_t(n);
    P.atlas[2] = base;
    return lb_run_device(g, s, pass, P, (const float4 *)items, uint32_t(n), base, (const float4 *)light,
                         uint32_t(n_light), (float4 *)out);
}

int lb_get_transfer(lb_gpu *g, uint64_t *h2d, uint64_t *d2h, int reset) {
    if (!g) return LB_EINVAL;
    if (h2d) *h2d = g->h2d;
    if (d2h) *d2h = g->d2h;
    if (reset) g->h2d = g->d2h = 0;
    return LB_OK;
}

int lb_set_pass_kernel(lb_gpu *g, int kind) {
    if (!g || kind < 0 || kind > 1) return LB_EINVAL;
    g->kernel = kind;
    return LB_OK;
}

int lb_set_near(lb_gpu *g, int on) {
    if (!g) return LB_EINVAL;
    g->near = on != 0;
    return LB_OK;
}

int lb_set_register_cap(lb_gpu *g, int blocks) {
    if (!g || !(blocks == 0 || blocks == 3 || blocks == 4)) return LB_EINVAL;
    g->occ = blocks;
    return LB_OK;
}

int lb_set_warp_walk(lb_gpu *g, int on) {
    if (!g) return LB_EINVAL;
    g->warp_walk = on != 0;
    return LB_OK;
}

int lb_set_fetch(lb_gpu *g, int on) {
    if (!g) return LB_EINVAL;
    g->fetch = on != 0;
    return LB_OK;
}

int lb_set_refill(lb_gpu *g, int on) {
    if (!g) return LB_EINVAL;
    g->refill = on != 0;
    return LB_OK;
}

int lb_set_bvh(lb_gpu *g, int width) {
    if (!g || (width != 2 && width != 8)) return LB_EINVAL;
    g->bvh = width;
    return LB_OK;
}

int lb_set_ray_order(lb_gpu *g, int direct, int gather) {
    if (!g || direct < 0 || gather < 0) return LB_EINVAL;
    g->group_direct = direct;
    g->group_gather = gather;
    return LB_OK;
}

int lb_set_counting(lb_gpu *g, int on) {
    if (!g) return LB_EINVAL;
    g->counting = on != 0;
    return LB_OK;
}

int lb_get_counters(lb_gpu *g, lb_counters *out) {
    if (!g || !out) return LB_EINVAL;
    *out = g->last;
    return LB_OK;
}

}  // extern "C"

// A pass over items already on the device, on the handle's stream. The pass's counters (rays always;
// the walk's work when counting is on) land in g->host_counters once the stream reaches them; call
// lb_collect_counters after a sync to move them into g->last.
int lb_run_device(lb_gpu *g, lb_scene *s, int pass, const lb_params &P, const float4 *items, uint32_t n, uint32_t base,
                  const float4 *light, uint32_t n_light, float4 *out) {
    lbd::Scene S = lb_scene_view(s);
    LB_CUDA(cudaMemsetAsync(g->counters, 0, 4 * sizeof(unsigned long long), g->stream), "counters");
    if (g->kernel == 1) {
        WarpPass w{};
        w.pass = pass;
        w.S = &S;
        w.P = &P;
        w.tex = items;
        w.n_host = n;
        w.base = base;
        w.light = light;
        w.n_light = n_light;
        w.out = out;
        w.counters = g->counters;
        w.full_count = g->counting;
        w.sms = g->sms;
        w.group = pass == LB_PASS_GATHER ? g->group_gather : g->group_direct;
        w.bvh = g->bvh;
        w.refill = g->refill;
        w.near = g->near;
        w.occ = g->occ;
        w.warp_walk = g->warp_walk;
        // the work counter: the handle's counter slot 4 (slots 4..7 of its 8 are otherwise unused)
        w.work = g->fetch ? reinterpret_cast<unsigned int *>(g->counters + 4) : nullptr;
        LB_CUDA(lb_launch_pass_warp(w, g->stream), "pass launch");
    } else {
        LB_CUDA(lb_launch_pass_bvh2(pass, S, P, items, n, base, light, n_light, out, g->counters, g->counting,
                                    g->stream),
                "pass launch");
    }
    LB_CUDA(cudaMemcpyAsync(g->host_counters, g->counters, 4 * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                            g->stream),
            "counters");
    return LB_OK;
}

void lb_collect_counters(lb_gpu *g) {
    g->last.rays = g->host_counters[0];
    g->last.nodes = g->host_counters[1];
    g->last.tris = g->host_counters[2];
    g->last.mats = g->host_counters[3];
}
