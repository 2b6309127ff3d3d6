// What a tile's light depends on, hashed on the device (crates/lightbaker/src/deps.rs:70-121): for every
// query (a tile's surfaces' box, or a chunk of probes', with its reach and its prefix: the global hash and
// the seed) the casting triangles whose boxes meet the query's zone swept towards the sun, hashed with
// BLAKE3 in the reference's byte order:
//
//   global (32) | seed | per casting mesh with a hit, in mesh order: mesh (u32) material (u32)
//                        then per hit, in triangle order: triangle (u32) and its 9 floats
//
// All queries at once: a bit a (query, triangle) pair from the swept-box test (the reference's arithmetic,
// so the same triangles), a scan of the bits, each query's message written to device memory, and the
// BLAKE3 tree over every message: a thread a 1024-byte chunk, then the parent nodes level by level
// (pairing neighbours with the odd last carried up is BLAKE3's left-balanced tree). BLAKE3 is restated
// from its published specification (O'Connor, Aumasson, Neves, Wilcox-O'Hearn, 2020): the IV, message
// permutation, G function and flags are the specification's. The digests equal the host's
// (csrc/host/deps.cpp, blake3.cpp) byte for byte.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include <cub/device/device_scan.cuh>

#include "lb_deps.h"
#include "lb_runtime.h"

namespace lbd {

__constant__ uint32_t B3_IV[8] = {0x6A09E667u, 0xBB67AE85u, 0x3C6EF372u, 0xA54FF53Au,
                                  0x510E527Fu, 0x9B05688Cu, 0x1F83D9ABu, 0x5BE0CD19u};
__constant__ uint8_t B3_PERM[16] = {2, 6, 3, 10, 7, 0, 4, 13, 1, 11, 12, 5, 9, 14, 15, 8};
constexpr uint32_t CHUNK_START = 1, CHUNK_END = 2, PARENT = 4, ROOT = 8;

__device__ __forceinline__ uint32_t rotr(uint32_t x, int n) { return __funnelshift_r(x, x, n); }
__device__ __forceinline__ void g(uint32_t *s, int a, int b, int c, int d, uint32_t mx, uint32_t my) {
    s[a] = s[a] + s[b] + mx;
    s[d] = rotr(s[d] ^ s[a], 16);
    s[c] = s[c] + s[d];
    s[b] = rotr(s[b] ^ s[c], 12);
    s[a] = s[a] + s[b] + my;
    s[d] = rotr(s[d] ^ s[a], 8);
    s[c] = s[c] + s[d];
    s[b] = rotr(s[b] ^ s[c], 7);
}
// the compression function's first 8 output words (a chaining value, or the digest at the root)
__device__ void compress(const uint32_t cv[8], const uint32_t block[16], uint64_t counter, uint32_t len,
                         uint32_t flags, uint32_t out[8]) {
    uint32_t s[16], m[16], t[16];
    for (int i = 0; i < 8; i++) s[i] = cv[i];
    for (int i = 0; i < 4; i++) s[8 + i] = B3_IV[i];
    s[12] = uint32_t(counter);
    s[13] = uint32_t(counter >> 32);
    s[14] = len;
    s[15] = flags;
    for (int i = 0; i < 16; i++) m[i] = block[i];
    for (int r = 0; r < 7; r++) {
        g(s, 0, 4, 8, 12, m[0], m[1]);
        g(s, 1, 5, 9, 13, m[2], m[3]);
        g(s, 2, 6, 10, 14, m[4], m[5]);
        g(s, 3, 7, 11, 15, m[6], m[7]);
        g(s, 0, 5, 10, 15, m[8], m[9]);
        g(s, 1, 6, 11, 12, m[10], m[11]);
        g(s, 2, 7, 8, 13, m[12], m[13]);
        g(s, 3, 4, 9, 14, m[14], m[15]);
        if (r < 6) {
            for (int i = 0; i < 16; i++) t[i] = m[B3_PERM[i]];
            for (int i = 0; i < 16; i++) m[i] = t[i];
        }
    }
    for (int i = 0; i < 8; i++) out[i] = s[i] ^ s[i + 8];
}

// deps.rs:98-121
__device__ __forceinline__ bool swept(const float zmin[3], const float zmax[3], const float sun[3], float top,
                                      const float bmin[3], const float bmax[3]) {
    float tmax = sun[1] > 1e-4f ? fmaxf((top - zmin[1]) / sun[1], 0.0f) : 0.0f;
    float lo = 0.0f, hi = tmax;
    for (int a = 0; a < 3; a++) {
        float s = sun[a];
        if (fabsf(s) < 1e-6f) {
            if (zmin[a] > bmax[a] || zmax[a] < bmin[a]) return false;
            continue;
        }
        float t1 = (bmax[a] - zmin[a]) / s, t2 = (bmin[a] - zmax[a]) / s;
        float a0 = s > 0.0f ? t2 : t1, a1 = s > 0.0f ? t1 : t2;
        lo = fmaxf(lo, a0);
        hi = fminf(hi, a1);
        if (lo > hi) return false;
    }
    return true;
}

// A bit a (query, triangle): the triangle's box (deps.rs:33-57, componentwise min/max of its vertices)
// meets the query's zone (its box grown by the reach) swept towards the sun. Words [query][tri / 32].
__global__ void k_swept(const float *pos, uint32_t n_tris, const float *zones, uint32_t n_q, const float *sun3,
                        float top, uint32_t words, uint32_t *bits) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t q = blockIdx.y;
    bool in = false;
    if (i < n_tris) {
        const float *v = pos + size_t(i) * 9;
        float bmin[3], bmax[3];
        for (int a = 0; a < 3; a++) {
            bmin[a] = fminf(fminf(v[a], v[3 + a]), v[6 + a]);
            bmax[a] = fmaxf(fmaxf(v[a], v[3 + a]), v[6 + a]);
        }
        float sun[3] = {sun3[0], sun3[1], sun3[2]};
        in = swept(zones + size_t(q) * 6, zones + size_t(q) * 6 + 3, sun, top, bmin, bmax);
    }
    uint32_t m = __ballot_sync(0xffffffffu, in);
    if ((threadIdx.x & 31) == 0 && i < ((n_tris + 31) & ~31u)) bits[size_t(q) * words + (i >> 5)] = m;
}

__global__ void k_popc(const uint32_t *bits, size_t n, uint32_t *counts) {
    size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) counts[i] = __popc(bits[i]);
}

__global__ void k_row_starts(const uint32_t *scan, uint32_t words, uint32_t n_q, uint32_t *rs) {
    uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q < n_q) rs[q] = scan[size_t(q) * words];
}
__global__ void k_sub_rows(uint32_t *scan, uint32_t words, size_t n, const uint32_t *rs) {
    size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) scan[i] -= rs[i / words];
}

// hits of query q among triangles [0, x): the scan of the words' counts plus the bits below x in x's word
__device__ __forceinline__ uint32_t hits_below(const uint32_t *bits, const uint32_t *wscan, uint32_t words, uint32_t q,
                                               uint32_t x) {
    uint32_t w = x >> 5, r = x & 31u;
    uint32_t below = wscan[size_t(q) * words + w];
    if (r) below += __popc(bits[size_t(q) * words + w] & ((1u << r) - 1u));
    return below;
}

// per (query, casting mesh): its hits and the bytes it adds (8 + 40 a hit, 0 without a hit)
__global__ void k_mesh_bytes(const uint32_t *bits, const uint32_t *wscan, uint32_t words, const uint32_t *mesh_start,
                             uint32_t n_mesh, uint32_t n_q, uint32_t *hits, uint64_t *bytes) {
    size_t k = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= size_t(n_q) * n_mesh) return;
    uint32_t q = uint32_t(k / n_mesh), j = uint32_t(k % n_mesh);
    // wscan is exclusive within the query's row; the row's last word adds its own count at the end
    uint32_t a = mesh_start[j], b = mesh_start[j + 1];
    auto below = [&](uint32_t x) -> uint32_t {
        if (x >> 5 >= words) {
            uint32_t w = words - 1;
            return wscan[size_t(q) * words + w] + __popc(bits[size_t(q) * words + w]);
        }
        return hits_below(bits, wscan, words, q, x);
    };
    uint32_t h = below(b) - below(a);
    hits[k] = h;
    bytes[k] = h ? 8ull + 40ull * h : 0ull;
}

// writes every query's message: its prefix, each mesh's header, each hit's index and vertices
struct MsgArgs {
    const uint8_t *prefix;
    const uint64_t *prefix_off;
    const uint32_t *prefix_len;
    const uint64_t *msg_off;     // [q]
    const uint64_t *mesh_off;    // [q][j]: exclusive scan of the mesh bytes within the query (global scan minus row start)
    const uint64_t *mesh_row;    // [q]: the global scan at the row's start
    const uint32_t *mesh_start;  // [j] first triangle (in the concatenated casting triangles), n_mesh + 1
    const uint32_t *mesh_id, *mesh_mat;
    const uint32_t *tri_mesh;    // [i] the casting mesh of triangle i
    const uint32_t *bits, *wscan;
    uint32_t words, n_mesh, n_q, n_tris;
    const float *pos;
    uint8_t *msg;
};

__global__ void k_write_prefix(MsgArgs a) {
    uint32_t q = blockIdx.x;
    uint8_t *dst = a.msg + a.msg_off[q];
    for (uint32_t b = threadIdx.x; b < a.prefix_len[q]; b += blockDim.x) dst[b] = a.prefix[a.prefix_off[q] + b];
}

__device__ __forceinline__ void put32(uint8_t *p, uint32_t v) {
    p[0] = uint8_t(v);
    p[1] = uint8_t(v >> 8);
    p[2] = uint8_t(v >> 16);
    p[3] = uint8_t(v >> 24);
}

__global__ void k_write_headers(MsgArgs a, const uint32_t *hits) {
    size_t k = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= size_t(a.n_q) * a.n_mesh) return;
    if (!hits[k]) return;
    uint32_t q = uint32_t(k / a.n_mesh), j = uint32_t(k % a.n_mesh);
    uint8_t *p = a.msg + a.msg_off[q] + a.prefix_len[q] + (a.mesh_off[k] - a.mesh_row[q]);
    put32(p, a.mesh_id[j]);
    put32(p + 4, a.mesh_mat[j]);
}

__global__ void k_write_hits(MsgArgs a) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t q = blockIdx.y;
    if (i >= a.n_tris) return;
    if (!((a.bits[size_t(q) * a.words + (i >> 5)] >> (i & 31u)) & 1u)) return;
    uint32_t j = a.tri_mesh[i];
    uint32_t rank = hits_below(a.bits, a.wscan, a.words, q, i) - hits_below(a.bits, a.wscan, a.words, q, a.mesh_start[j]);
    size_t k = size_t(q) * a.n_mesh + j;
    uint8_t *p = a.msg + a.msg_off[q] + a.prefix_len[q] + (a.mesh_off[k] - a.mesh_row[q]) + 8 + 40ull * rank;
    put32(p, i - a.mesh_start[j]);
    const float *v = a.pos + size_t(i) * 9;
    for (int c = 0; c < 9; c++) put32(p + 4 + 4 * c, __float_as_uint(v[c]));
}

// BLAKE3 chunks: a thread a chunk of a message (chunk `c` of query q, counter c), its chaining value, or the
// digest when the message is one chunk long
__global__ void k_chunks(const uint8_t *msg, const uint64_t *msg_off, const uint64_t *msg_len,
                         const uint64_t *chunk_first, uint32_t n_q, uint64_t n_chunks, uint32_t *cvs, uint32_t *digest) {
    uint64_t ci = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (ci >= n_chunks) return;
    // the query this chunk belongs to: the last q with chunk_first[q] <= ci
    uint32_t lo = 0, hi = n_q;
    while (hi - lo > 1) {
        uint32_t mid = (lo + hi) / 2;
        if (chunk_first[mid] <= ci) lo = mid;
        else hi = mid;
    }
    uint32_t q = lo;
    uint64_t c = ci - chunk_first[q];
    uint64_t len = msg_len[q];
    uint64_t nch = len ? (len + 1023) / 1024 : 1;
    uint64_t start = c * 1024, clen = len > start ? (len - start < 1024 ? len - start : 1024) : 0;
    const uint8_t *src = msg + msg_off[q] + start;
    uint32_t nblocks = clen ? uint32_t((clen + 63) / 64) : 1;
    uint32_t cv[8];
    for (int i = 0; i < 8; i++) cv[i] = B3_IV[i];
    for (uint32_t b = 0; b < nblocks; b++) {
        uint32_t blen = uint32_t(clen - uint64_t(b) * 64 < 64 ? clen - uint64_t(b) * 64 : 64);
        if (!clen) blen = 0;
        uint32_t w[16];
        for (int i = 0; i < 16; i++) {
            uint32_t v = 0;
            for (int k = 0; k < 4; k++) {
                uint32_t o = uint32_t(i * 4 + k);
                if (o < blen) v |= uint32_t(src[uint64_t(b) * 64 + o]) << (8 * k);
            }
            w[i] = v;
        }
        uint32_t flags = (b == 0 ? CHUNK_START : 0u) | (b + 1 == nblocks ? CHUNK_END : 0u);
        if (b + 1 == nblocks && nch == 1) flags |= ROOT;
        compress(cv, w, c, blen, flags, cv);
    }
    for (int i = 0; i < 8; i++) cvs[ci * 8 + i] = cv[i];
    if (nch == 1)
        for (int i = 0; i < 8; i++) digest[size_t(q) * 8 + i] = cv[i];
}

// one level of parents: query q has cnt[q] values at src[first[q]..]; pairs become parents at dst[dfirst[q]..],
// an odd last moves up as it is; the pair that leaves one value is the root (the digest)
__global__ void k_parents(const uint32_t *src, const uint64_t *first, const uint32_t *cnt, uint32_t *dst,
                          const uint64_t *dfirst, const uint64_t *pair_first, uint32_t n_q, uint64_t n_pairs,
                          uint32_t *digest) {
    uint64_t pi = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (pi >= n_pairs) return;
    uint32_t lo = 0, hi = n_q;
    while (hi - lo > 1) {
        uint32_t mid = (lo + hi) / 2;
        if (pair_first[mid] <= pi) lo = mid;
        else hi = mid;
    }
    uint32_t q = lo;
    uint64_t k = pi - pair_first[q];  // output slot k of query q: the pair (2k, 2k+1), or the carried last
    uint32_t n = cnt[q];
    const uint32_t *a = src + (first[q] + 2 * k) * 8;
    uint32_t *out = dst + (dfirst[q] + k) * 8;
    if (2 * k + 1 >= n) {
        for (int i = 0; i < 8; i++) out[i] = a[i];
        return;
    }
    uint32_t block[16];
    for (int i = 0; i < 16; i++) block[i] = a[i];
    uint32_t iv[8];
    for (int i = 0; i < 8; i++) iv[i] = B3_IV[i];
    bool root = n == 2;
    compress(iv, block, 0, 64, PARENT | (root ? ROOT : 0u), out);
    if (root)
        for (int i = 0; i < 8; i++) digest[size_t(q) * 8 + i] = out[i];
}

}  // namespace lbd

namespace {
inline void ck(cudaError_t e, const char *what) {
    if (e != cudaSuccess) throw std::runtime_error(std::string("device hashing: ") + what + ": " + cudaGetErrorString(e));
}
struct Buf {
    void *p = nullptr;
    explicit Buf(size_t bytes) { ck(cudaMalloc(&p, bytes ? bytes : 16), "cudaMalloc"); }
    ~Buf() {
        if (p) cudaFree(p);
    }
    template <class T> T *as() const { return (T *)p; }
};
template <class T> void up(const Buf &b, const std::vector<T> &v, cudaStream_t st) {
    if (!v.empty()) ck(cudaMemcpyAsync(b.p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, st), "upload");
}
template <class T> size_t scan_temp(const T *in, T *out, size_t n) {
    size_t bytes = 0;
    ck(cub::DeviceScan::ExclusiveSum(nullptr, bytes, in, out, n), "scan size");
    return bytes;
}
}  // namespace

void lb_hash_reach_device(lb_gpu *g, const DepsInput &in, const std::vector<DepsQuery> &queries,
                          std::vector<std::array<uint8_t, 32>> &out) {
    cudaStream_t st = g->stream;
    const uint32_t n_q = uint32_t(queries.size());
    out.assign(n_q, {});
    if (!n_q) return;
    const uint32_t n_tris = in.n_tris, n_mesh = uint32_t(in.mesh_id.size());
    const uint32_t words = std::max<uint32_t>(1, (n_tris + 31) / 32);
    // the queries' zones (own box grown by the reach, deps.rs:28-30), prefixes
    std::vector<float> zones(size_t(n_q) * 6);
    std::vector<uint64_t> prefix_off(n_q);
    std::vector<uint32_t> prefix_len(n_q);
    std::vector<uint8_t> prefix;
    for (uint32_t q = 0; q < n_q; q++) {
        for (int a = 0; a < 3; a++) {
            zones[size_t(q) * 6 + a] = queries[q].min[a] - queries[q].reach;
            zones[size_t(q) * 6 + 3 + a] = queries[q].max[a] + queries[q].reach;
        }
        prefix_off[q] = prefix.size();
        prefix_len[q] = uint32_t(queries[q].prefix.size());
        prefix.insert(prefix.end(), queries[q].prefix.begin(), queries[q].prefix.end());
    }
    Buf d_pos(size_t(n_tris) * 36), d_zones(zones.size() * 4), d_sun(12), d_bits(size_t(n_q) * words * 4),
        d_wcnt(size_t(n_q) * words * 4), d_wscan(size_t(n_q) * words * 4);
    if (n_tris) ck(cudaMemcpyAsync(d_pos.p, in.pos, size_t(n_tris) * 36, cudaMemcpyHostToDevice, st), "positions");
    up(d_zones, zones, st);
    ck(cudaMemcpyAsync(d_sun.p, in.sun, 12, cudaMemcpyHostToDevice, st), "sun");
    g->h2d += size_t(n_tris) * 36 + zones.size() * 4;
    ck(cudaMemsetAsync(d_bits.p, 0, size_t(n_q) * words * 4, st), "bits");
    if (n_tris) {
        dim3 grid((n_tris + 255) / 256, n_q);
        lbd::k_swept<<<grid, 256, 0, st>>>(d_pos.as<float>(), n_tris, d_zones.as<float>(), n_q, d_sun.as<float>(),
                                           in.top, words, d_bits.as<uint32_t>());
        ck(cudaPeekAtLastError(), "swept");
    }
    // hits before each word, row by row (a row's scan restarts: scan every word, subtract the row's start)
    const size_t nw = size_t(n_q) * words;
    lbd::k_popc<<<(nw + 255) / 256, 256, 0, st>>>(d_bits.as<uint32_t>(), nw, d_wcnt.as<uint32_t>());
    ck(cudaPeekAtLastError(), "popc");
    {
        size_t tb = scan_temp(d_wcnt.as<uint32_t>(), d_wscan.as<uint32_t>(), nw);
        Buf t(tb);
        ck(cub::DeviceScan::ExclusiveSum(t.p, tb, d_wcnt.as<uint32_t>(), d_wscan.as<uint32_t>(), nw, st), "scan");
    }
    // each row's scan from 0: subtract the scan at the row's first word (unsigned wrap-around keeps the
    // difference exact: a row's hits are fewer than 2^32)
    {
        Buf rs(size_t(n_q) * 4);
        lbd::k_row_starts<<<(n_q + 255) / 256, 256, 0, st>>>(d_wscan.as<uint32_t>(), words, n_q, rs.as<uint32_t>());
        lbd::k_sub_rows<<<(nw + 255) / 256, 256, 0, st>>>(d_wscan.as<uint32_t>(), words, nw, rs.as<uint32_t>());
        ck(cudaPeekAtLastError(), "row scans");
        ck(cudaStreamSynchronize(st), "row scans");
    }
    // per (query, mesh) hits and bytes, and their scan
    Buf d_mstart((n_mesh + 1) * 4), d_mid(std::max<uint32_t>(1, n_mesh) * 4), d_mmat(std::max<uint32_t>(1, n_mesh) * 4),
        d_trimesh(size_t(std::max<uint32_t>(1, n_tris)) * 4);
    up(d_mstart, in.mesh_start, st);
    up(d_mid, in.mesh_id, st);
    up(d_mmat, in.mesh_mat, st);
    up(d_trimesh, in.tri_mesh, st);
    const size_t nqm = size_t(n_q) * n_mesh;
    Buf d_hits(std::max<size_t>(1, nqm) * 4), d_mbytes(std::max<size_t>(1, nqm) * 8), d_moff(std::max<size_t>(1, nqm) * 8);
    std::vector<uint64_t> mesh_row(n_q, 0), msg_len(n_q), msg_off(n_q);
    if (nqm) {
        lbd::k_mesh_bytes<<<(nqm + 255) / 256, 256, 0, st>>>(d_bits.as<uint32_t>(), d_wscan.as<uint32_t>(), words,
                                                            d_mstart.as<uint32_t>(), n_mesh, n_q, d_hits.as<uint32_t>(),
                                                            d_mbytes.as<uint64_t>());
        ck(cudaPeekAtLastError(), "mesh bytes");
        size_t tb = scan_temp(d_mbytes.as<uint64_t>(), d_moff.as<uint64_t>(), nqm);
        Buf t(tb);
        ck(cub::DeviceScan::ExclusiveSum(t.p, tb, d_mbytes.as<uint64_t>(), d_moff.as<uint64_t>(), nqm, st), "scan");
        std::vector<uint64_t> row_end(n_q);
        for (uint32_t q = 0; q < n_q; q++) {
            ck(cudaMemcpyAsync(&mesh_row[q], d_moff.as<uint64_t>() + size_t(q) * n_mesh, 8, cudaMemcpyDeviceToHost, st),
               "mesh rows");
        }
        uint64_t last_off = 0, last_bytes = 0;
        ck(cudaMemcpyAsync(&last_off, d_moff.as<uint64_t>() + nqm - 1, 8, cudaMemcpyDeviceToHost, st), "mesh total");
        ck(cudaMemcpyAsync(&last_bytes, d_mbytes.as<uint64_t>() + nqm - 1, 8, cudaMemcpyDeviceToHost, st), "mesh total");
        ck(cudaStreamSynchronize(st), "mesh rows");
        for (uint32_t q = 0; q < n_q; q++) row_end[q] = q + 1 < n_q ? mesh_row[q + 1] : last_off + last_bytes;
        for (uint32_t q = 0; q < n_q; q++) msg_len[q] = prefix_len[q] + (row_end[q] - mesh_row[q]);
    } else {
        for (uint32_t q = 0; q < n_q; q++) msg_len[q] = prefix_len[q];
    }
    uint64_t total = 0;
    for (uint32_t q = 0; q < n_q; q++) {
        msg_off[q] = total;
        total += msg_len[q];
    }
    Buf d_msg(total), d_prefix(prefix.size()), d_poff(n_q * 8), d_plen(n_q * 4), d_msgoff(n_q * 8), d_msglen(n_q * 8),
        d_mrow(n_q * 8);
    up(d_prefix, prefix, st);
    up(d_poff, prefix_off, st);
    up(d_plen, prefix_len, st);
    up(d_msgoff, msg_off, st);
    up(d_msglen, msg_len, st);
    up(d_mrow, mesh_row, st);
    lbd::MsgArgs a{};
    a.prefix = d_prefix.as<uint8_t>();
    a.prefix_off = d_poff.as<uint64_t>();
    a.prefix_len = d_plen.as<uint32_t>();
    a.msg_off = d_msgoff.as<uint64_t>();
    a.mesh_off = d_moff.as<uint64_t>();
    a.mesh_row = d_mrow.as<uint64_t>();
    a.mesh_start = d_mstart.as<uint32_t>();
    a.mesh_id = d_mid.as<uint32_t>();
    a.mesh_mat = d_mmat.as<uint32_t>();
    a.tri_mesh = d_trimesh.as<uint32_t>();
    a.bits = d_bits.as<uint32_t>();
    a.wscan = d_wscan.as<uint32_t>();
    a.words = words;
    a.n_mesh = n_mesh;
    a.n_q = n_q;
    a.n_tris = n_tris;
    a.pos = d_pos.as<float>();
    a.msg = d_msg.as<uint8_t>();
    lbd::k_write_prefix<<<n_q, 64, 0, st>>>(a);
    if (nqm) lbd::k_write_headers<<<(nqm + 255) / 256, 256, 0, st>>>(a, d_hits.as<uint32_t>());
    if (n_tris) lbd::k_write_hits<<<dim3((n_tris + 255) / 256, n_q), 256, 0, st>>>(a);
    ck(cudaPeekAtLastError(), "messages");
    // BLAKE3: chunks, then parents level by level
    std::vector<uint32_t> cnt(n_q);
    std::vector<uint64_t> first(n_q);
    uint64_t n_chunks = 0;
    for (uint32_t q = 0; q < n_q; q++) {
        cnt[q] = uint32_t(msg_len[q] ? (msg_len[q] + 1023) / 1024 : 1);
        first[q] = n_chunks;
        n_chunks += cnt[q];
    }
    Buf d_cv_a(n_chunks * 32), d_cv_b(n_chunks * 32), d_first(n_q * 8), d_cnt(n_q * 4), d_dfirst(n_q * 8),
        d_pfirst(n_q * 8), d_digest(size_t(n_q) * 32);
    up(d_first, first, st);
    lbd::k_chunks<<<(n_chunks + 127) / 128, 128, 0, st>>>(d_msg.as<uint8_t>(), d_msgoff.as<uint64_t>(),
                                                           d_msglen.as<uint64_t>(), d_first.as<uint64_t>(), n_q,
                                                           n_chunks, d_cv_a.as<uint32_t>(), d_digest.as<uint32_t>());
    ck(cudaPeekAtLastError(), "chunks");
    uint32_t *src = d_cv_a.as<uint32_t>(), *dst = d_cv_b.as<uint32_t>();
    for (;;) {
        uint32_t top = 0;
        for (uint32_t c : cnt) top = std::max(top, c);
        if (top <= 1) break;
        // this level: queries with more than one value pair them up; the rest keep theirs (1 slot)
        std::vector<uint64_t> dfirst(n_q), pfirst(n_q);
        std::vector<uint32_t> next(n_q);
        uint64_t slots = 0;
        for (uint32_t q = 0; q < n_q; q++) {
            next[q] = cnt[q] > 1 ? (cnt[q] + 1) / 2 : 1;
            dfirst[q] = slots;
            pfirst[q] = slots;
            slots += next[q];
        }
        up(d_cnt, cnt, st);
        up(d_dfirst, dfirst, st);
        up(d_pfirst, pfirst, st);
        ck(cudaStreamSynchronize(st), "level upload");
        lbd::k_parents<<<(slots + 127) / 128, 128, 0, st>>>(src, d_first.as<uint64_t>(), d_cnt.as<uint32_t>(), dst,
                                                             d_dfirst.as<uint64_t>(), d_pfirst.as<uint64_t>(), n_q,
                                                             slots, d_digest.as<uint32_t>());
        ck(cudaPeekAtLastError(), "parents");
        std::swap(src, dst);
        cnt = next;
        first = dfirst;
        up(d_first, first, st);
    }
    std::vector<uint32_t> dig(size_t(n_q) * 8);
    ck(cudaMemcpyAsync(dig.data(), d_digest.p, dig.size() * 4, cudaMemcpyDeviceToHost, st), "digests");
    ck(cudaStreamSynchronize(st), "digests");
    g->d2h += dig.size() * 4;
    for (uint32_t q = 0; q < n_q; q++)
        for (int i = 0; i < 8; i++) {
            uint32_t v = dig[size_t(q) * 8 + i];
            for (int k = 0; k < 4; k++) out[q][i * 4 + k] = uint8_t(v >> (8 * k));
        }
}
