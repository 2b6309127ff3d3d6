// The 8-wide compressed BVH (host/bvh8.h has the node format) built on the device from the scene's BVH2,
// which is already in device memory: a breadth-first collapse, one level of nodes a step. A thread an
// item (a node to emit) finds the item's children with the host builder's own routine
// (host/bvh8_node.h) and counts its inner children and leaf triangles; a scan numbers them (inner
// children after every node of this and the earlier levels, in slot order; triangles after every
// triangle emitted before); a second launch writes the node (five 16-byte stores), its leaf triangles
// (each with its index in the BVH2's triangle array in e2.w) and the next level's items. The host
// collapse (host/bvh8.cpp) numbers nodes and triangles the same way, breadth first, so the two give the
// same bytes. The host reads two counts a level to size the next launch.
#include <cuda_runtime.h>

#include <cub/cub.cuh>

#include "host/bvh8_node.h"
#include "lb_runtime.h"

namespace {

__global__ void k_root(const lb_node *n2, lb8::Item *items) { items[0] = lb8::root_item(n2); }

// inner children (high word) and leaf triangles (low word) of each item
__global__ void __launch_bounds__(128) k_count(const lb8::Item *items, uint32_t n, const lb_node *n2, uint32_t nn2,
                                               unsigned long long *counts) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    lb8::Ref refs[8];
    const int m = lb8::refs_of(n2, nn2, items[i], refs);
    uint32_t tris;
    const uint32_t mask = lb8::inner_mask(refs, m, &tris);
    counts[i] = (unsigned long long)__popc(mask) << 32 | tris;
}

__global__ void __launch_bounds__(128) k_emit(const lb8::Item *items, uint32_t n, const lb_node *n2, uint32_t nn2,
                                              const lb_tri *t2, const unsigned long long *offsets, uint32_t node_base,
                                              uint32_t child_base, uint32_t tri_base, uint4 *nodes8, lb_tri *tris8,
                                              lb8::Item *next, int *err) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    lb8::Ref refs[8];
    const int m = lb8::refs_of(n2, nn2, items[i], refs);
    const unsigned long long o = offsets[i];
    const uint32_t kid0 = uint32_t(o >> 32), tri0 = tri_base + uint32_t(o);
    uint32_t w[lb8::WORDS];
    if (!lb8::node_words(refs, m, child_base + kid0, tri0, w)) atomicExch(err, 1);
    uint4 *dst = nodes8 + size_t(node_base + i) * (lb8::WORDS / 4);
    for (int k = 0; k < int(lb8::WORDS / 4); k++) dst[k] = make_uint4(w[4 * k], w[4 * k + 1], w[4 * k + 2], w[4 * k + 3]);
    const uint32_t mask = w[3] >> 24;
    uint32_t kids = 0, off = 0;
    for (int s = 0; s < m; s++) {
        if ((mask >> s) & 1u) {
            next[kid0 + kids++] = lb8::item_of(refs[s]);
            continue;
        }
        for (uint32_t t = 0; t < refs[s].count; t++) {
            const uint32_t orig = refs[s].first + t;
            const float4 *src = (const float4 *)(t2 + orig);
            float4 *d = (float4 *)(tris8 + tri0 + off + t);
            const float4 e2 = src[2];
            d[0] = src[0];
            d[1] = src[1];
            d[2] = make_float4(e2.x, e2.y, e2.z, __uint_as_float(orig));
        }
        off += refs[s].count;
    }
}

// grows a device buffer to at least `bytes`, keeping its first `keep` bytes
int grow(void *&p, size_t &cap, size_t bytes, size_t keep, cudaStream_t stream) {
    if (bytes <= cap) return LB_OK;
    size_t c = cap ? cap : 4096;
    while (c < bytes) c *= 2;
    void *q = nullptr;
    cudaError_t e = cudaMalloc(&q, c);
    if (e != cudaSuccess) return lb_cuda_fail(e, "bvh8 build: allocation");
    if (keep) {
        e = cudaMemcpyAsync(q, p, keep, cudaMemcpyDeviceToDevice, stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) {
            cudaFree(q);
            return lb_cuda_fail(e, "bvh8 build: copy");
        }
    }
    if (p) cudaFree(p);
    p = q;
    cap = c;
    return LB_OK;
}

struct Scratch {
    void *a = nullptr, *b = nullptr, *counts = nullptr, *offsets = nullptr, *temp = nullptr, *err = nullptr;
    size_t ca = 0, cb = 0, cc = 0, co = 0, ct = 0;
    ~Scratch() {
        for (void *p : {a, b, counts, offsets, temp, err})
            if (p) cudaFree(p);
    }
};

}  // namespace

// Builds s->nodes8 / s->tris8 from s->nodes / s->tris on the handle's stream; LB_OK or an error code.
int lb_bvh8_build(lb_gpu *g, lb_scene *s) {
    cudaStream_t st = g->stream;
    const uint32_t nn2 = s->n_nodes, n_tris = s->n_tris;
    const lb_node *n2 = (const lb_node *)s->nodes;
    const lb_tri *t2 = (const lb_tri *)s->tris;
    Scratch w;
    void *nodes8 = nullptr;
    size_t cap8 = 0;
    const size_t tri_cap = n_tris ? n_tris : 1;
    int rc = LB_OK;
    cudaError_t e;
    auto fail = [&](int code) {
        if (nodes8) cudaFree(nodes8);
        return code;
    };
    if ((e = cudaMalloc(&s->tris8, tri_cap * sizeof(lb_tri))) != cudaSuccess) return lb_cuda_fail(e, "bvh8 build");
    if ((e = cudaMalloc(&w.err, sizeof(int))) != cudaSuccess) return lb_cuda_fail(e, "bvh8 build");
    if ((e = cudaMemsetAsync(w.err, 0, sizeof(int), st)) != cudaSuccess) return lb_cuda_fail(e, "bvh8 build");
    const size_t NB = lb8::WORDS * 4;
    if ((rc = grow(nodes8, cap8, (size_t(nn2) / 4 + 64) * NB, 0, st)) != LB_OK) return fail(rc);
    if ((rc = grow(w.a, w.ca, sizeof(lb8::Item), 0, st)) != LB_OK) return fail(rc);
    k_root<<<1, 1, 0, st>>>(n2, (lb8::Item *)w.a);
    uint32_t node_base = 0, level = 1, total = 1;
    uint64_t tri_total = 0;
    while (level > 0) {
        if ((rc = grow(w.counts, w.cc, size_t(level) * 8, 0, st)) != LB_OK) return fail(rc);
        if ((rc = grow(w.offsets, w.co, size_t(level) * 8, 0, st)) != LB_OK) return fail(rc);
        const int blocks = int((level + 127) / 128);
        k_count<<<blocks, 128, 0, st>>>((const lb8::Item *)w.a, level, n2, nn2, (unsigned long long *)w.counts);
        size_t tb = 0;
        auto *cin = (unsigned long long *)w.counts, *cout = (unsigned long long *)w.offsets;
        if ((e = cub::DeviceScan::ExclusiveSum(nullptr, tb, cin, cout, int(level), st)) != cudaSuccess)
            return fail(lb_cuda_fail(e, "bvh8 build: scan size"));
        if ((rc = grow(w.temp, w.ct, tb, 0, st)) != LB_OK) return fail(rc);
        if ((e = cub::DeviceScan::ExclusiveSum(w.temp, tb, cin, cout, int(level), st)) != cudaSuccess)
            return fail(lb_cuda_fail(e, "bvh8 build: scan"));
        unsigned long long last[2];
        e = cudaMemcpyAsync(&last[0], cout + level - 1, 8, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(&last[1], cin + level - 1, 8, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return fail(lb_cuda_fail(e, "bvh8 build: level counts"));
        const unsigned long long sum = last[0] + last[1];
        const uint32_t kids = uint32_t(sum >> 32), tris = uint32_t(sum & 0xffffffffu);
        // an open item takes a BVH2 inner node no other item takes, and run items cut disjoint ranges of
        // leaf triangles, at most two a triangle: a tree gives at most nn2 + 2 n_tris + 1 nodes (a cycle
        // in a malformed BVH2 stops here)
        if (uint64_t(total) + kids > uint64_t(nn2) + 2 * uint64_t(n_tris) + 1 || tri_total + tris > tri_cap) {
            lb_set_error("bvh8 build: more nodes or triangles than the BVH2 allows");
            return fail(LB_EINVAL);
        }
        if ((rc = grow(nodes8, cap8, (size_t(total) + kids) * NB, size_t(total) * NB, st)) != LB_OK) return fail(rc);
        if ((rc = grow(w.b, w.cb, (size_t(kids) + 1) * sizeof(lb8::Item), 0, st)) != LB_OK) return fail(rc);
        k_emit<<<blocks, 128, 0, st>>>((const lb8::Item *)w.a, level, n2, nn2, t2, cout, node_base, total,
                                       uint32_t(tri_total), (uint4 *)nodes8, (lb_tri *)s->tris8, (lb8::Item *)w.b,
                                       (int *)w.err);
        if ((e = cudaGetLastError()) != cudaSuccess) return fail(lb_cuda_fail(e, "bvh8 build: launch"));
        std::swap(w.a, w.b);
        std::swap(w.ca, w.cb);
        node_base = total;
        total += kids;
        tri_total += tris;
        level = kids;
    }
    int err = 0;
    e = cudaMemcpyAsync(&err, w.err, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess && tri_total == 0) e = cudaMemsetAsync(s->tris8, 0, sizeof(lb_tri), st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return fail(lb_cuda_fail(e, "bvh8 build"));
    if (err) {
        lb_set_error("bvh8 build: cannot quantise a node's boxes");
        return fail(LB_EINVAL);
    }
    if (tri_total != n_tris && !(nn2 == 1 && tri_total == 0)) {  // one inner node: the reference's empty BVH
        lb_set_error("bvh8 build: the BVH2's leaves do not hold every triangle once");
        return fail(LB_EINVAL);
    }
    s->nodes8 = nodes8;
    s->n_nodes8 = total;
    s->n_tris8 = uint32_t(tri_total ? tri_total : 1);
    return LB_OK;
}
