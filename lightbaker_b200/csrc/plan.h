// The device-resident bake's state (bake_device.cu) and the transport built on it (transport.cu).
#pragma once
#include <cuda_runtime.h>

#include <array>
#include <chrono>
#include <cmath>
#include <map>
#include <optional>
#include <stdexcept>
#include <string>
#include <vector>

#include "host/bake.h"
#include "host/deps.h"
#include "lb_post.h"
#include "lb_runtime.h"

namespace lbplan {

inline void ck(cudaError_t e, const char *what) {
    if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

// The handle whose spare buffers DBufs allocated on this thread draw on (set by a DBufScope; none: plain
// cudaMalloc and cudaFree).
inline thread_local lb_gpu *g_dbuf_gpu = nullptr;
struct DBufScope {
    lb_gpu *prev;
    explicit DBufScope(lb_gpu *g) : prev(g_dbuf_gpu) { g_dbuf_gpu = g; }
    ~DBufScope() { g_dbuf_gpu = prev; }
    DBufScope(const DBufScope &) = delete;
    DBufScope &operator=(const DBufScope &) = delete;
};

// A device allocation freed with its owner: taken from, and given back to, its handle's spares when it was
// allocated inside a DBufScope (lb_spare_take / lb_spare_give), else cudaMalloc and cudaFree.
struct DBuf {
    void *p = nullptr;
    size_t bytes = 0, cap = 0;
    lb_gpu *owner = nullptr;
    DBuf() = default;
    DBuf(const DBuf &) = delete;
    DBuf &operator=(const DBuf &) = delete;
    void release() {
        if (!p) return;
        if (owner) lb_spare_give(owner, p, cap);
        else cudaFree(p);
        p = nullptr;
    }
    void alloc(size_t n) {
        release();
        bytes = n ? n : 16;
        owner = g_dbuf_gpu;
        if (owner && (p = lb_spare_take(owner, bytes, &cap)) != nullptr) return;
        ck(cudaMalloc(&p, bytes), "cudaMalloc");
        cap = bytes;
    }
    ~DBuf() { release(); }
    template <class T> T *as() const { return (T *)p; }
};

// filter.rs:28-41: exp(-(dx^2 + dy^2) / sigma2), sigma2 = 2 (0.75 r)^2, as the host computes it
inline std::vector<float> gauss_weights(int r) {
    std::vector<float> w(size_t(2 * r + 1) * (2 * r + 1), 0.0f);
    if (r == 0) return w;
    float q = float(r) * 0.75f;
    float sigma2 = 2.0f * (q * q);
    for (int dy = -r; dy <= r; dy++)
        for (int dx = -r; dx <= r; dx++) {
            float fx = float(dx), fy = float(dy);
            w[size_t(dy + r) * (2 * r + 1) + (dx + r)] = std::exp(-(fx * fx + fy * fy) / sigma2);
        }
    return w;
}

inline double since(std::chrono::steady_clock::time_point t) {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t).count();
}

}  // namespace lbplan

struct lb_plan {
    lb_gpu *g = nullptr;
    lb::Scene scene;
    lb::Prepared P;
    lb::Options opt;
    lb_scene *dscene = nullptr;
    std::vector<size_t> dirty, order;          // order: dirty tiles, then cached ones
    std::vector<lb::Hash> hashes;
    std::vector<std::optional<lb::TileLight>> lights;
    std::vector<DTile> tiles_all;              // in `order`
    uint32_t n_dirty_texels = 0, n_all = 0, n_cov = 0;
    std::vector<uint32_t> cov_counts;          // covered texels per dirty tile
    // volume
    bool has_volume = false;
    std::array<uint32_t, 3> vsize{};
    uint32_t n_probes = 0, n_todo = 0;
    std::map<lb::TileKey, std::vector<uint32_t>> chunks;
    std::vector<std::pair<lb::Hash, std::vector<uint32_t>>> chunk_keys;
    size_t n_chunks = 0;
    // device arrays
    lbplan::DBuf tiles_d, tex, cov_idx, cov_k, direct_out, chart, valid, state, known, known_tmp, gathered, hard, gk, soft,
        ao_raw, ao, field, dl, ind, posg, light, w1, wr, gath_idx, gath_count, gather_out, select_temp;
    lbplan::DBuf s_ka, s_kb, s_f1, s_f2, s_v4, s_e0, s_e1;
    lbplan::DBuf probes, probes_init, probes_b, probe_items, probe_slot, pk_a, pk_b;
    lbplan::DBuf owner, direct_atlas, validity, indirect, indirect_b, has, has_b, counters;
    lbplan::DBuf enc_bc5, enc_rgb, enc_vol, enc_scale;  // the output encodings (encode.cu)
    size_t select_bytes = 0;
    uint32_t aw = 0, ah = 0, iw = 0, ih = 0, ds = 1;
    int blocks_direct = 0, blocks_gather = 0, blocks_volume = 0;
    int kernel_nodes = 0;
    bool autotune = false;
    int group_direct = 8, group_gather = 8;  // ray order for the warp passes
    int bvh_direct = 2, bvh_gather = 2, bvh_volume = 2;  // BVH width for the warp passes
    int refill_direct = 0, refill_gather = 0;          // lane refill for the warp passes
    int near_direct = 1, near_gather = 1;              // leaf lists (direct: occlusion rays; gather: near hits)
    int occ_direct = 0, occ_gather = 0;                // register caps (WarpPass::occ)
    int fetch_direct = 1, fetch_gather = 1;            // items taken from a work counter (WarpPass::work)
    int warp_walk = 1;                                 // the direct pass's sun rays walk together (WarpPass)
    bool reuse = true;          // later bounces evaluate the first bounce's gather records
    bool keep_records = false;  // record the first bounce's gather rays whatever the bounce count
    uint64_t max_gathered = 0;  // a bound on the gathered texels (records are sized by it)
    lbplan::DBuf records, theta0;
    // with keep_records and a volume: every volume ray's outcome ([probe item][ray], gather_record) and the
    // probes as the volume pass wrote them, before the fill
    lbplan::DBuf vrecords, vraw;
    std::string tuned;  // what the autotuner picked
    std::string build_phases;  // the host build's phases, seconds since its start
    // a bake split over ranks (lb_exchange): every pass traces this rank's share of its items (item_part), and
    // the ranks sum the passes' outputs (one writer a word) before the texel passes that read them
    int rank = 0, world = 1;
    lb_exchange ex{};
    // the graph in pieces: one, or (world > 1) cut after each pass whose outputs the ranks sum; the sums
    // (device words) a launch makes after each piece
    struct Piece {
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
        std::vector<std::pair<void *, size_t>> sums;
    };
    std::vector<Piece> pieces;
    cudaEvent_t ev[2] = {nullptr, nullptr};  // around the last lb_plan_launch: the graph's device time
    double t_prepare = 0;
    lb::Stats stats;
    ~lb_plan() {
        for (cudaEvent_t e : ev)
            if (e) cudaEventDestroy(e);
        for (Piece &pc : pieces) {
            if (pc.exec) cudaGraphExecDestroy(pc.exec);
            if (pc.graph) cudaGraphDestroy(pc.graph);
        }
        if (dscene) lb_scene_free(dscene);
    }
};


// The plan's arguments for the texel passes over its dirty tiles.
PostArgs lb_plan_post_args(lb_plan &p);
// A plan of every tile (no cache) whose first gather pass records every ray's outcome in `records`.
lb_plan *lb_plan_create_recording(lb_gpu *g, const uint8_t *scene, size_t len);
