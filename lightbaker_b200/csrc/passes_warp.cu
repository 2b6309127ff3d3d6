// The three ray passes with a warp on each item (crates/lightbaker/src/gpu/trace.wgsl:170-324), for
// the device-resident bake. The shader runs an item's rays one after another in one thread; here the 32
// lanes of a warp trace 32 of the item's rays at once: the 16 rays of an inside test, the 16 hard and 16
// soft sun rays of a 4 x 4 grid, 32 occlusion or gather rays at a time. Rays of one item start at the
// same point (or within one texel) and their walks visit the same nodes, so a warp's loads coalesce
// and its lanes stay together far longer than with 32 items' rays. Sums the shader builds ray by ray
// (occlusion, bounced light, the L1 coefficients) are built in the same ray order here too (a lane
// adds its neighbours' terms in turn), so the records are bit-identical to the shader's.
//
// Persistent: a grid of (SMs x resident warps) walks the items with a stride. The item count may live
// in device memory (read at launch), so a pass can follow a device-side compaction in a CUDA graph.
#include <cuda_runtime.h>

#include "lb_device.cuh"
#include "lb_kernels.h"

namespace lbd {

constexpr unsigned FULL = 0xffffffffu;

// Adds the lanes' terms (those whose flag is set) to `sum` in lane order: the order a sequential loop
// over the rays would add them.
// (The loops stay rolled: fully unrolled twice in one kernel they make ptxas 12.9 fail register
// allocation on sm_100a.)
__device__ __forceinline__ float ordered_add(float sum, float term, bool on) {
    unsigned mask = __ballot_sync(FULL, on);
#pragma unroll 1
    for (int l = 0; l < 32; l++) {
        float v = __shfl_sync(FULL, term, l);
        if (mask & (1u << l)) sum += v;
    }
    return sum;
}
__device__ __forceinline__ float3 ordered_add3(float3 sum, float3 term, bool on) {
    unsigned mask = __ballot_sync(FULL, on);
#pragma unroll 1
    for (int l = 0; l < 32; l++) {
        float x = __shfl_sync(FULL, term.x, l), y = __shfl_sync(FULL, term.y, l), z = __shfl_sync(FULL, term.z, l);
        if (mask & (1u << l)) sum = add(sum, mk(x, y, z));
    }
    return sum;
}

// Ray order within an item. For a power-of-two ray count N = 2^L (32 <= N <= CAP), the warp's 32 rays
// of a round are those whose index shares its top `a` bits and its bottom `b` bits (a + b = L - 5):
// the Hammersley points (r / N, bitrev(r) / N) are a (0, m, 2)-net, so such a set fills one box of the
// unit square: a = L - 5 a band of elevations (the shader's order), a = 0 a wedge of azimuths, between
// them a patch of both. Rays of a patch head the same way and walk the same nodes. Each ray's term goes
// to shared memory at its index and the item's sum is then built in index order, as the shader's.
constexpr int WARPS = 8;     // warps a block (256 threads)
constexpr int AO_CAP = 512;  // largest grouped occlusion ray count
constexpr int GI_CAP = 256;  // largest grouped gather ray count

// The round-invariant parts of the index: the lane's bits, and how a round's number splits.
struct RayOrder {
    uint32_t lane_bits, b, top, lo_mask;
    bool grouped;
    __device__ __forceinline__ RayOrder(uint32_t n, uint32_t cap, int a, int lane) {
        int L = (n >= 32 && n <= cap && (n & (n - 1)) == 0) ? __ffs(n) - 1 : -1;
        grouped = L >= 0;
        if (!grouped) L = 5;
        a = max(0, min(a, L - 5));
        b = uint32_t(L - 5 - a);
        top = uint32_t(L - a);
        lo_mask = (1u << b) - 1u;
        lane_bits = grouped ? uint32_t(lane) << b : uint32_t(lane);
    }
    __device__ __forceinline__ uint32_t ray(uint32_t round) const {
        uint32_t r = grouped ? (((round >> b) << top) | lane_bits | (round & lo_mask)) : round * 32u + lane_bits;
        return r;
    }
    // the ray handed out seq-th (lane refill): the same order, round by round
    __device__ __forceinline__ uint32_t at(uint32_t seq) const {
        if (!grouped) return seq;
        uint32_t round = seq >> 5;
        return ((round >> b) << top) | ((seq & 31u) << b) | (round & lo_mask);
    }
};

// An item: its record (pos, normal, dx, dy), the position optionally taken from a second array
// (the texel's sample point moved by the direct pass, bake.rs:227-238).
struct Item {
    float4 pos, nrm, dx, dy;
};
__device__ __forceinline__ Item load_item(const float4 *tex, const uint32_t *idx, const float4 *pos_override,
                                          uint32_t k) {
    uint32_t t = idx ? __ldg(&idx[k]) : k;
    Item it;
    it.pos = pos_override ? __ldg(&pos_override[t]) : __ldg(&tex[4 * t]);
    it.nrm = __ldg(&tex[4 * t + 1]);
    it.dx = __ldg(&tex[4 * t + 2]);
    it.dy = __ldg(&tex[4 * t + 3]);
    return it;
}

// One ray of an inside test (trace.wgsl:159-168): ray r of the 16 from o about the normal n, and whether
// it meets a back face. Over the texel's leaf list when o may use it (`listed`; the ray starts within
// `shift` of the list's centre, heads into the same hemisphere and reaches no farther than the list),
// else the tree walk. Per lane: the two halves of a warp may test two points.
template <int BVH, bool COUNT, bool WT>
__device__ __forceinline__ bool inside_ray(const Scene &S, const lb_params &P, uint32_t seed, const uint32_t *list,
                                           const float *dist2, int nl, bool listed, float shift, float3 o, float3 n,
                                           uint32_t key, uint32_t r, Count &c) {
    Frame f = frame(n);
    float3 d = cosine((__uint2float_rn(r) + 0.5f) / 16.0f, radical(r), f);
    Hit h;
    if (listed) {
        bool tie;
        h = trace_list_t<COUNT, WT, TIE_INSIDE>(S, list, dist2, nl, o, d, P.ground[3], key + r + 7000u, seed, c,
                                                shift, tie);
        if (tie) {
            // nearly coincident faces: the tree walk's own order decides which is the hit (and its face)
            c.rays--;
            h = walk_apart<COUNT, WT>(S, o, d, P.ground[3], key + r + 7000u, seed, c);
        }
    } else {
        h = walk<BVH, COUNT, WT>(S, o, d, P.ground[3], false, key + r + 7000u, seed, c);
    }
    return h.tri != NONE && h.back;
}
// The test's verdict from the count of its 16 rays that met back faces: more than insideShare of them.
// The count is exact, as the shader's float sum of ones.
__device__ __forceinline__ bool inside_of(const lb_params &P, unsigned backs) {
    return __uint2float_rn(__popc(backs)) / 16.0f > __uint_as_float(P.atlas[3]);
}

// The item a warp takes next. With a work counter (zeroed before the launch) every warp takes the next item
// not yet taken as soon as it is free, so warps behind heavy items (texels whose inside tests retry, long
// escaping rays) no longer hold up the pass's end; without one, a static stride. Called by the whole warp.
// `lo`: the first item of the launch's share (item_part), where the counter's count starts.
__device__ __forceinline__ uint32_t take_item(unsigned int *work, uint32_t k, uint32_t step, uint32_t lo, int lane) {
    if (!work) return k + step;
    uint32_t v = 0;
    if (lane == 0) v = atomicAdd(work, 1u);
    return lo + __shfl_sync(FULL, v, 0);
}

template <bool COUNT>
__device__ __forceinline__ void flush_counts(Count &c, unsigned long long *counters) {
    for (int o = 16; o > 0; o >>= 1) {
        c.rays += __shfl_down_sync(FULL, c.rays, o);
        if (COUNT) {
            c.nodes += __shfl_down_sync(FULL, c.nodes, o);
            c.tris += __shfl_down_sync(FULL, c.tris, o);
            c.mats += __shfl_down_sync(FULL, c.mats, o);
        }
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&counters[0], (unsigned long long)c.rays);
        if (COUNT) {
            atomicAdd(&counters[1], (unsigned long long)c.nodes);
            atomicAdd(&counters[2], (unsigned long long)c.tris);
            atomicAdd(&counters[3], (unsigned long long)c.mats);
        }
    }
}

// trace.wgsl:170-243. OCC: blocks of 256 threads an SM must hold (1: the compiler's budget, capped at 128
// registers so that two blocks still fit).
template <int BVH, bool COUNT, int OCC = 1, int WALK = 0, bool WT = false>
__global__ void __launch_bounds__(256, (OCC < 2 ? 2 : OCC)) direct_warp(Scene S, lb_params P, const float4 *tex, const uint32_t *idx,
                                                   const uint32_t *n_dev, uint32_t n_host, uint32_t base, float4 *out,
                                                   unsigned long long *counters, int group, int refill, int near,
                                                   unsigned int *work, int warp_walk, uint32_t part,
                                                   uint32_t parts) {
    // each occlusion ray's term by ray index (0 for a miss: adding it to the sum changes no bit, as the sum
    // starts at +0 and every term is >= 0); before the rays, the ball query's scratch
    __shared__ float s_term[WARPS][AO_CAP];
    static_assert(sizeof(s_term[0]) >= 2 * BALL_FRONT * sizeof(uint32_t), "the ball query's scratch fits");
    __shared__ uint32_t s_list[WARPS][BALL_LEAVES];
    __shared__ float s_dist[WARPS][BALL_LEAVES];
    // the sun rays' shared walk (escapes_warp): its stack of kept children and their lanes
    constexpr int WW = (BVH == 2 && !COUNT) ? int(WARP_WALK_DEPTH) : 1;
    __shared__ uint32_t s_ww_node[WARPS][WW], s_ww_mask[WARPS][WW];
    // the leaf lists' occlusion rays left to the tree walk (near ties), by ray index
    constexpr int PW = (BVH == 2 && WALK == 1) ? WARPS : 1;
    __shared__ uint16_t s_pend[PW][AO_CAP];
    const int lane = threadIdx.x & 31;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    uint32_t lo, n;
    item_part(n_dev ? *n_dev : n_host, part, parts, lo, n);
    const uint32_t seed = __float_as_uint(P.reach[3]);
    const bool shared_sun = BVH == 2 && !COUNT && warp_walk && S.depth <= WARP_WALK_DEPTH;
    Count c;
    c.zero();
    const uint32_t first = work ? take_item(work, 0, 0, lo, lane) : lo + warp;
    for (uint32_t k = first; k < n; k = take_item(work, k, warps, lo, lane)) {
        Item it = load_item(tex, idx, nullptr, k);
        float3 nrm = xyz(it.nrm), pos = xyz(it.pos), dx = xyz(it.dx), dy = xyz(it.dy);
        uint32_t key = (base + k) * 7919u;
        uint32_t g = P.counts[0];
        float3 sun = xyz(P.sun_dir);
        float3 lift = scl(nrm, P.reach[2]);
        float3 at = pos;
        uint32_t pick = 0u;
        float span = 1.0f;
        const int wi = threadIdx.x >> 5;
        // The leaves around the texel's own point c0, gathered once, far enough for every ray of the inside
        // tests and the occlusion rays from any candidate point (reach plus the farthest candidate's
        // distance from c0). A ray from another point o uses the list when o is not behind c0's plane by
        // more than half the list's front margin (the list leaves out boxes wholly behind that plane, and
        // every ray here heads into the normal's hemisphere); its walk's early end counts |o - c0|.
        auto candidate = [&](uint32_t q) -> float3 {
            if (q == 9u) return add(pos, scl(nrm, PUSH));
            float2 cc = offset(q);
            return add(add(pos, scl(dx, cc.x)), scl(dy, cc.y));
        };
        const float3 c0 = add(pos, lift);
        int nl = -1;
        float rball = P.reach[0];
        const bool listed = BVH == 2 && WALK == 1 && near && P.counts[1] <= uint32_t(AO_CAP);
        if (listed) {
            float far_ = 0.0f;
            for (uint32_t q = 1u; q <= 9u; q++) far_ = fmaxf(far_, sqrtf(dot3(sub(add(candidate(q), lift), c0),
                                                                              sub(add(candidate(q), lift), c0))));
            rball = P.reach[0] + far_ * 1.001f + 1e-5f;
            uint32_t *scratch = reinterpret_cast<uint32_t *>(&s_term[wi][0]);
            nl = ball_leaves<COUNT>(S, c0, rball, nrm, scratch, scratch + BALL_FRONT, s_list[wi], s_dist[wi], lane, c);
        }
        const float front = -(rball * 1e-3f + 1e-4f) * 0.5f;
        auto listed_from = [&](float3 o, float &shift) -> bool {
            float3 v = sub(o, c0);
            shift = sqrtf(dot3(v, v)) * 1.001f + 1e-6f;
            return nl >= 0 && dot3(v, nrm) >= front;
        };
        // trace.wgsl:186-210: the texel's own point, then (when it is inside) the candidates 1..8 and the
        // pushed point 9 in order, until one is not inside. Points are tested two at a time, lanes 0..15
        // the first, 16..31 the next (a half warp is all one test takes): the first point not inside is the
        // sequential loop's, and a second point's test past it is not counted as traced. With COUNT one
        // point at a time (exact node and triangle counts). One call site, so the walks are inlined once.
        constexpr uint32_t STEP = COUNT ? 1u : 2u;
#pragma unroll 1
        for (uint32_t q = 0u; q <= 9u; q += STEP) {
            const uint32_t mine = q + (STEP == 2u ? uint32_t(lane >> 4) : 0u);
            bool back = false;
            if ((STEP == 2u || lane < 16) && mine <= 9u) {
                const float3 o = add(mine == 0u ? pos : candidate(mine), lift);
                const uint32_t k = mine == 0u ? key : (mine == 9u ? key + 331u : key + mine * 31u);
                float shift;
                const bool lst = listed_from(o, shift);
                back = inside_ray<BVH, COUNT, WT>(S, P, seed, s_list[wi], s_dist[wi], nl, lst, shift, o, nrm, k,
                                                  uint32_t(lane & 15), c);
            }
            const unsigned m = __ballot_sync(FULL, back);
            const bool in0 = inside_of(P, m & 0xffffu);
            const bool in1 = inside_of(P, m >> 16);
            // the point that is not inside, if any (10: both are)
            const uint32_t out = !in0 ? q : (STEP == 2u && q + 1u <= 9u && !in1 ? q + 1u : 10u);
            if (STEP == 2u && out == q && q + 1u <= 9u && lane >= 16) c.rays--;
            if (out == 0u) break;
            if (out <= 9u) {
                at = candidate(out);
                pick = out;
                span = 0.4f;
                break;
            }
        }
        float soft = 0.0f;
        uint32_t hard = 0u;
        if (dot3(sun, nrm) > 0.0f) {
            Frame sf = frame(sun);
            uint32_t gg = g * g;
            float fg = __uint2float_rn(g), fgg = __uint2float_rn(gg);
            uint32_t turn = uint32_t(rnd(key, 17u, seed) * fgg);
            uint32_t nsoft = 0;
            // a pair of rays a cell: lanes 0..15 the hard ray of cell s0 + lane, lanes 16..31 the soft one
            for (uint32_t s0 = 0; s0 < gg; s0 += 16) {
                uint32_t s = s0 + uint32_t(lane & 15);
                bool escaped = false;
                if (shared_sun) {
                    // the 32 rays (16 cells' hard and soft rays) start within the texel and head within the sun's
                    // disc: one walk of the BVH2 for the warp
                    const bool on = s < gg;
                    float3 o = at, d = sun;
                    uint32_t ray = key + s;
                    if (on) {
                        float cx = ((__uint2float_rn(s % g) + 0.5f) / fg - 0.5f) * span;
                        float cy = ((__uint2float_rn(s / g) + 0.5f) / fg - 0.5f) * span;
                        o = add(add(add(at, scl(dx, cx)), scl(dy, cy)), lift);
                        if (lane >= 16) {
                            d = sun_disc(P, sf, (s + turn) % gg, gg);
                            ray = key + s + 1000u;
                        }
                    }
                    const int wi2 = int(threadIdx.x >> 5);
                    escaped = escapes_warp<WT>(S, o, d, FAR, ray, seed, on, s_ww_node[wi2], s_ww_mask[wi2], lane, c);
                } else if (s < gg) {
                    float cx = ((__uint2float_rn(s % g) + 0.5f) / fg - 0.5f) * span;
                    float cy = ((__uint2float_rn(s / g) + 0.5f) / fg - 0.5f) * span;
                    float3 o = add(add(add(at, scl(dx, cx)), scl(dy, cy)), lift);
                    // lanes 0..15 the hard ray toward the sun, 16..31 the soft one (one walk call site)
                    const bool hard_ray = lane < 16;
                    const float3 d = hard_ray ? sun : sun_disc(P, sf, (s + turn) % gg, gg);
                    escaped = walk<BVH, COUNT, WT>(S, o, d, FAR, true, hard_ray ? key + s : key + s + 1000u, seed, c).tri ==
                              NONE;
                }
                unsigned m = __ballot_sync(FULL, escaped);
                hard |= (m & 0xffffu) << (s0 & 31u);  // the shader shifts modulo 32
                nsoft += __popc(m >> 16);
            }
            soft = __uint2float_rn(nsoft) / fgg;
        }
        Frame f = frame(nrm);
        float3 o = add(at, lift);
        uint32_t rays = P.counts[1];
        float frays = __uint2float_rn(rays);
        float s1 = rnd(key, 3u, seed), s2 = rnd(key, 5u, seed);
        float occ = 0.0f;
        uint32_t nback = 0;
        const RayOrder ord(rays, AO_CAP, group, lane);
        const int w = threadIdx.x >> 5;
        // the occlusion rays start at o: the texel's own list when it serves o, else o's own
        float ao_shift = 0.0f;
        if (pick != 0u && !listed_from(o, ao_shift)) {
            ao_shift = 0.0f;
            nl = -1;
            if (listed) {
                uint32_t *scratch = reinterpret_cast<uint32_t *>(&s_term[w][0]);
                nl = ball_leaves<COUNT>(S, o, P.reach[0], nrm, scratch, scratch + BALL_FRONT, s_list[w], s_dist[w], lane,
                                        c);
            }
        }
        if (pick == 0u) listed_from(o, ao_shift);
        if (nl >= 0) {
            uint32_t myback = 0, npend = 0;
            const unsigned below = (1u << lane) - 1u;
            auto term_of = [&](uint32_t r, const Hit &h) {
                float term = 0.0f;
                if (h.tri != NONE) {
                    float kk = h.t / P.reach[0];
                    term = 1.0f - kk * kk;
                    if (h.back && h.t < P.ground[3]) myback++;
                }
                s_term[w][r] = term;
            };
            auto dir_of = [&](uint32_t r) {
                return cosine(fract((__uint2float_rn(r) + 0.5f) / frays + s1), fract(radical(r) + s2), f);
            };
            for (uint32_t r0 = 0; r0 < rays; r0 += 32) {
                uint32_t r = ord.ray(r0 >> 5);
                bool pend = false;
                if (r < rays) {
                    bool tie;
                    Hit h = trace_list_t<COUNT, WT, TIE_OCC>(S, s_list[w], s_dist[w], nl, o, dir_of(r), P.reach[0],
                                                          key + r + 2000u, seed, c, ao_shift, tie);
                    if (tie) {
                        pend = true;
                        c.rays--;  // the tree walk counts it
                    } else {
                        term_of(r, h);
                    }
                }
                const unsigned pm = __ballot_sync(FULL, pend);
                if (pend) s_pend[PW == 1 ? 0 : w][npend + __popc(pm & below)] = uint16_t(r);
                npend += __popc(pm);
            }
            // nearly coincident faces: the tree walk's t (its box test may pass over the nearer face's box
            // when the entry rounds past the hit it holds), for the rays that met such a tie, 32 at a time
            __syncwarp();
            for (uint32_t b0 = 0; b0 < npend; b0 += 32) {
                const uint32_t i = b0 + uint32_t(lane);
                if (i < npend) {
                    const uint32_t r = s_pend[PW == 1 ? 0 : w][i];
                    term_of(r, walk_apart<COUNT, WT>(S, o, dir_of(r), P.reach[0], key + r + 2000u, seed, c));
                }
            }
            for (int ofs = 16; ofs > 0; ofs >>= 1) myback += __shfl_down_sync(FULL, myback, ofs);
            nback = __shfl_sync(FULL, myback, 0);
            __syncwarp();
            for (uint32_t r0 = 0; r0 < rays; r0 += 32) {
                uint32_t rr = r0 + uint32_t(lane);
                occ = ordered_add(occ, rr < rays ? s_term[w][rr] : 0.0f, rr < rays);
            }
            __syncwarp();
        } else if (BVH == 2 && WALK == 2 && refill && rays <= AO_CAP) {
            // lane refill: a lane takes the item's next ray as soon as its own has ended
            Walk2<COUNT, WT> wk;
            uint32_t seq = uint32_t(lane), next = 32, r = 0, myback = 0;
            bool have = seq < rays;
            if (have) {
                r = ord.at(seq);
                wk.start(S, o, cosine(fract((__uint2float_rn(r) + 0.5f) / frays + s1), fract(radical(r) + s2), f),
                         P.reach[0], false, key + r + 2000u, c);
            }
            while (__any_sync(FULL, have)) {
                if (have) wk.step(S, seed, c);
                bool fin = have && wk.done;
                if (fin) {
                    bool hit = wk.hit.tri != NONE;
                    float term = 0.0f;
                    if (hit) {
                        float kk = wk.hit.t / P.reach[0];
                        term = 1.0f - kk * kk;
                        if (wk.hit.back && wk.hit.t < P.ground[3]) myback++;
                    }
                    s_term[w][r] = term;
                }
                unsigned fm = __ballot_sync(FULL, fin);
                if (fin) {
                    seq = next + __popc(fm & ((1u << lane) - 1u));
                    have = seq < rays;
                    if (have) {
                        r = ord.at(seq);
                        wk.start(S, o,
                                 cosine(fract((__uint2float_rn(r) + 0.5f) / frays + s1), fract(radical(r) + s2), f),
                                 P.reach[0], false, key + r + 2000u, c);
                    }
                }
                next += __popc(fm);
            }
            for (int ofs = 16; ofs > 0; ofs >>= 1) myback += __shfl_down_sync(FULL, myback, ofs);
            nback = __shfl_sync(FULL, myback, 0);
            __syncwarp();
            for (uint32_t r0 = 0; r0 < rays; r0 += 32) {
                uint32_t rr = r0 + uint32_t(lane);
                occ = ordered_add(occ, rr < rays ? s_term[w][rr] : 0.0f, rr < rays);
            }
            __syncwarp();
        } else
        for (uint32_t r0 = 0; r0 < rays; r0 += 32) {
            uint32_t r = ord.ray(r0 >> 5);
            bool hit = false, bk = false;
            float term = 0.0f;
            if (r < rays) {
                float3 d = cosine(fract((__uint2float_rn(r) + 0.5f) / frays + s1), fract(radical(r) + s2), f);
                Hit h = walk<BVH, COUNT, WT>(S, o, d, P.reach[0], false, key + r + 2000u, seed, c);
                if (h.tri != NONE) {
                    hit = true;
                    float kk = h.t / P.reach[0];
                    term = 1.0f - kk * kk;
                    bk = h.back && h.t < P.ground[3];
                }
            }
            if (ord.grouped) {
                s_term[w][r] = term;
            } else {
                occ = ordered_add(occ, term, hit);
            }
            nback += __popc(__ballot_sync(FULL, bk));
        }
        if (nl < 0 && !(BVH == 2 && WALK == 2 && refill && rays <= AO_CAP) && ord.grouped) {
            __syncwarp();
            for (uint32_t r0 = 0; r0 < rays; r0 += 32) occ = ordered_add(occ, s_term[w][r0 + lane], true);
            __syncwarp();
        }
        if (lane == 0)
            out[k] = make_float4(soft, __uint_as_float(hard | (pick << 24u)), occ / frays, __uint2float_rn(nback) / frays);
    }
    flush_counts<COUNT>(c, counters);
}

// Gather rays that find a hit this close are resolved by the texel's leaf list (WALK 1); the others walk
// the tree. A speed parameter only: either way a ray gets the tree walk's hit.
constexpr float GATHER_NEAR = 2.0f;
// a queued gather ray's flag: its list walk met no accepted triangle
constexpr uint32_t PEND_MISSED = 0x8000u;
static_assert(GI_CAP <= int(PEND_MISSED), "ray indices leave the flag bit free");

// trace.wgsl:245-270. rec (optional): each ray's outcome ([item][ray], gather_record) for later bounces.
// WALK 1 (BVH2): the warp gathers the leaves within GATHER_NEAR (widened by the jitter's reach) of the
// texel's lifted point, and every ray first walks that list with its length cut to GATHER_NEAR; a hit
// there is the ray's nearest (any nearer triangle lies in the list too). The rays that found none, met a
// tie (which the tree walk settles in its own order) or start behind the list's plane queue up and walk
// the tree in full rounds of 32, so the long walks of rays that escape no longer hold up lanes whose rays
// ended nearby.
template <int BVH, bool COUNT, int OCC = 1, int WALK = 0, bool WT = false>
__global__ void __launch_bounds__(256, (OCC < 2 ? 2 : OCC)) gather_warp(
    Scene S, lb_params P, const float4 *tex, const uint32_t *idx, const float4 *pos_override, const uint32_t *n_dev,
    uint32_t n_host, uint32_t base, const float4 *light, uint32_t n_light, float4 *out, unsigned long long *counters,
    int group, int refill, uint2 *rec, unsigned int *work, uint32_t part, uint32_t parts) {
    constexpr int LW = (BVH == 2 && WALK == 1) ? WARPS : 1;  // the leaf lists' shared memory, when used
    __shared__ float3 s_term[WARPS][GI_CAP];
    __shared__ uint8_t s_on[WARPS][GI_CAP];
    __shared__ uint32_t s_list[LW][BALL_LEAVES];
    __shared__ float s_dist[LW][BALL_LEAVES];
    __shared__ uint16_t s_pend[LW][GI_CAP];
    const int lane = threadIdx.x & 31;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    uint32_t lo, n;
    item_part(n_dev ? *n_dev : n_host, part, parts, lo, n);
    const uint32_t seed = __float_as_uint(P.reach[3]);
    Count c;
    c.zero();
    const uint32_t first = work ? take_item(work, 0, 0, lo, lane) : lo + warp;
    for (uint32_t k = first; k < n; k = take_item(work, k, warps, lo, lane)) {
        Item it = load_item(tex, idx, pos_override, k);
        float3 nrm = xyz(it.nrm), pos = xyz(it.pos), dx = xyz(it.dx), dy = xyz(it.dy);
        Frame f = frame(nrm);
        uint32_t key = (base + k) * 7919u;
        uint32_t rays = P.counts[2];
        float frays = __uint2float_rn(rays);
        float s1 = rnd(key, 11u, seed), s2 = rnd(key, 13u, seed);
        float3 sum = mk(0.f, 0.f, 0.f);
        uint32_t nback = 0;
        const RayOrder ord(rays, GI_CAP, group, lane);
        const int w = threadIdx.x >> 5;
        const bool refilling = BVH == 2 && WALK == 2 && refill && rays <= GI_CAP;
        const bool listing = BVH == 2 && WALK == 1 && ord.grouped;
        // the ray's origin (jittered across the texel, lifted) and direction
        auto ray_of = [&](uint32_t rr, float3 &oo, float3 &dd) {
            float jx = rnd(key + rr, 19u, seed) - 0.5f, jy = rnd(key + rr, 23u, seed) - 0.5f;
            oo = add(add(add(pos, scl(dx, jx)), scl(dy, jy)), scl(nrm, P.reach[2]));
            dd = cosine(fract((__uint2float_rn(rr) + 0.5f) / frays + s1), fract(radical(rr) + s2), f);
        };
        // a ray's outcome into the item's terms (by ray index) and records
        auto finish = [&](uint32_t rr, float3 oo, float3 dd, const Hit &h, uint32_t &backs) {
            float3 term = mk(0.f, 0.f, 0.f);
            bool on = true;
            if (h.tri == NONE) term = sky(P, dd);
            else if (h.back) {
                on = false;
                backs++;
            } else term = bounced(S, P, light, n_light, oo, dd, h);
            s_term[w][rr] = term;
            s_on[w][rr] = on;
            if (rec) rec[size_t(k) * rays + rr] = gather_record(S, P, n_light, oo, dd, h);
        };
        if (listing) {
            const int lw = LW == 1 ? 0 : w;
            const float3 c0 = add(pos, scl(nrm, P.reach[2]));
            // every jittered origin lies within (|dx| + |dy|) / 2 of c0
            const float far_ = (sqrtf(dot3(dx, dx)) + sqrtf(dot3(dy, dy))) * 0.5f * 1.001f + 1e-5f;
            const float rnear = fminf(GATHER_NEAR, P.reach[1]), rball = rnear + far_;
            // the ball query's scratch (two levels of nodes) is the item's term array, not yet written
            static_assert(sizeof(s_term[0]) >= 2 * BALL_FRONT * sizeof(uint32_t), "scratch fits the terms");
            uint32_t *scratch = reinterpret_cast<uint32_t *>(&s_term[w][0]);
            const int nl = ball_leaves<COUNT>(S, c0, rball, nrm, scratch, scratch + BALL_FRONT, s_list[lw], s_dist[lw],
                                              lane, c);
            const float front = -(rball * 1e-3f + 1e-4f) * 0.5f;
            const unsigned below = (1u << lane) - 1u;
            uint32_t npend = 0, myback = 0;
            for (uint32_t r0 = 0; r0 < rays; r0 += 32) {
                const uint32_t r = ord.ray(r0 >> 5);
                float3 o, d;
                ray_of(r, o, d);
                bool done = false, missed = false;
                const float3 v = sub(o, c0);
                if (nl >= 0 && dot3(v, nrm) >= front) {
                    const float shift = sqrtf(dot3(v, v)) * 1.001f + 1e-6f;
                    bool tie;
                    Hit h = trace_list_t<COUNT, WT, TIE_GATHER>(S, s_list[lw], s_dist[lw], nl, o, d, rnear, key + r + 4000u,
                                                          seed, c, shift, tie);
                    if (h.tri != NONE && !tie) {
                        done = true;
                        finish(r, o, d, h, myback);
                    } else {
                        c.rays--;  // the tree walk counts it
                        missed = h.tri == NONE;
                    }
                }
                const unsigned pm = __ballot_sync(FULL, !done);
                if (!done) s_pend[lw][npend + __popc(pm & below)] = uint16_t(r | (missed ? PEND_MISSED : 0u));
                npend += __popc(pm);
            }
            // A ray whose list walk met no accepted triangle before rnear has none there at all (every
            // triangle it could meet that close lies in the list), so its tree walk passes over the boxes
            // it leaves before rnear, less a margin (1 %) far above the rounding of t and of the box test. Not
            // when counting (the reference walk's node counts), nor in a tree deeper than the walk's stack.
            const float skip = (!COUNT && S.depth <= uint32_t(STACK)) ? rnear * 0.99f - 1e-4f : 0.0f;
            __syncwarp();
            for (uint32_t b0 = 0; b0 < npend; b0 += 32) {
                const uint32_t i = b0 + uint32_t(lane);
                if (i < npend) {
                    const uint32_t e = s_pend[lw][i], r = e & ~PEND_MISSED;
                    float3 o, d;
                    ray_of(r, o, d);
                    Hit h = walk<BVH, COUNT, WT>(S, o, d, P.reach[1], false, key + r + 4000u, seed, c,
                                                 (e & PEND_MISSED) ? skip : 0.0f);
                    finish(r, o, d, h, myback);
                }
            }
            for (int ofs = 16; ofs > 0; ofs >>= 1) myback += __shfl_down_sync(FULL, myback, ofs);
            nback = __shfl_sync(FULL, myback, 0);
        } else if (refilling) {
            // lane refill: a lane takes the item's next ray as soon as its own has ended
            Walk2<COUNT, WT> wk;
            uint32_t seq = uint32_t(lane), next = 32, r = 0, myback = 0;
            bool have = seq < rays;
            auto begin = [&](uint32_t rr) {
                float jx = rnd(key + rr, 19u, seed) - 0.5f, jy = rnd(key + rr, 23u, seed) - 0.5f;
                float3 oo = add(add(add(pos, scl(dx, jx)), scl(dy, jy)), scl(nrm, P.reach[2]));
                float3 dd = cosine(fract((__uint2float_rn(rr) + 0.5f) / frays + s1), fract(radical(rr) + s2), f);
                wk.start(S, oo, dd, P.reach[1], false, key + rr + 4000u, c);
            };
            if (have) {
                r = ord.at(seq);
                begin(r);
            }
            while (__any_sync(FULL, have)) {
                if (have) wk.step(S, seed, c);
                bool fin = have && wk.done;
                if (fin) {
                    float3 term = mk(0.f, 0.f, 0.f);
                    bool on = true;
                    if (wk.hit.tri == NONE) term = sky(P, wk.d);
                    else if (wk.hit.back) {
                        on = false;
                        myback++;
                    } else term = bounced(S, P, light, n_light, wk.o, wk.d, wk.hit);
                    s_term[w][r] = term;
                    s_on[w][r] = on;
                    if (rec) rec[size_t(k) * rays + r] = gather_record(S, P, n_light, wk.o, wk.d, wk.hit);
                }
                unsigned fm = __ballot_sync(FULL, fin);
                if (fin) {
                    seq = next + __popc(fm & ((1u << lane) - 1u));
                    have = seq < rays;
                    if (have) {
                        r = ord.at(seq);
                        begin(r);
                    }
                }
                next += __popc(fm);
            }
            for (int ofs = 16; ofs > 0; ofs >>= 1) myback += __shfl_down_sync(FULL, myback, ofs);
            nback = __shfl_sync(FULL, myback, 0);
            __syncwarp();
            for (uint32_t r0 = 0; r0 < rays; r0 += 32) {
                uint32_t rr = r0 + uint32_t(lane);
                sum = ordered_add3(sum, rr < rays ? s_term[w][rr] : mk(0.f, 0.f, 0.f), rr < rays && s_on[w][rr]);
            }
            __syncwarp();
        } else
        for (uint32_t r0 = 0; r0 < rays; r0 += 32) {
            uint32_t r = ord.ray(r0 >> 5);
            bool on = false, bk = false;
            float3 term = mk(0.f, 0.f, 0.f);
            if (r < rays) {
                float jx = rnd(key + r, 19u, seed) - 0.5f, jy = rnd(key + r, 23u, seed) - 0.5f;
                float3 o = add(add(add(pos, scl(dx, jx)), scl(dy, jy)), scl(nrm, P.reach[2]));
                float3 d = cosine(fract((__uint2float_rn(r) + 0.5f) / frays + s1), fract(radical(r) + s2), f);
                Hit h = walk<BVH, COUNT, WT>(S, o, d, P.reach[1], false, key + r + 4000u, seed, c);
                if (h.tri == NONE) {
                    term = sky(P, d);
                    on = true;
                } else if (h.back) {
                    bk = true;
                } else {
                    term = bounced(S, P, light, n_light, o, d, h);
                    on = true;
                }
                if (rec) rec[size_t(k) * rays + r] = gather_record(S, P, n_light, o, d, h);
            }
            if (ord.grouped) {
                s_term[w][r] = term;
                s_on[w][r] = on;
            } else {
                sum = ordered_add3(sum, term, on);
            }
            nback += __popc(__ballot_sync(FULL, bk));
        }
        if (!refilling && ord.grouped) {
            __syncwarp();
            for (uint32_t r0 = 0; r0 < rays; r0 += 32) sum = ordered_add3(sum, s_term[w][r0 + lane], s_on[w][r0 + lane]);
            __syncwarp();
        }
        if (lane == 0) {
            float3 e = scl(sum, PI);
            out[k] = make_float4(e.x / frays, e.y / frays, e.z / frays, __uint2float_rn(nback) / frays);
        }
    }
    flush_counts<COUNT>(c, counters);
}

// trace.wgsl:272-324. `slot` (optional) scatters probe k's four records to 4 * slot[k].
template <int BVH, bool COUNT, bool WT = false>
__global__ void __launch_bounds__(256) volume_warp(Scene S, lb_params P, const float4 *tex, uint32_t n_all,
                                                   const float4 *light, uint32_t n_light, float4 *out,
                                                   const uint32_t *slot, unsigned long long *counters, uint32_t part,
                                                   uint32_t parts, uint2 *rec) {
    const int lane = threadIdx.x & 31;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    const uint32_t seed = __float_as_uint(P.reach[3]);
    Count c;
    c.zero();
    uint32_t lo, n;
    item_part(n_all, part, parts, lo, n);
    for (uint32_t k = lo + warp; k < n; k += warps) {
        float3 o = xyz(__ldg(&tex[4 * k]));
        uint32_t key = __float_as_uint(__ldg(&tex[4 * k + 1]).w) * 7919u + 77u;
        uint32_t rays = P.counts[2];
        float frays = __uint2float_rn(rays);
        float s1 = rnd(key, 29u, seed), s2 = rnd(key, 31u, seed);
        float3 l0 = mk(0.f, 0.f, 0.f), l1x = l0, l1y = l0, l1z = l0;
        uint32_t nback = 0;
        for (uint32_t r0 = 0; r0 < rays; r0 += 32) {
            uint32_t r = r0 + uint32_t(lane);
            bool on = r < rays, bk = false;
            float3 t0 = mk(0.f, 0.f, 0.f), tx = t0, ty = t0, tz = t0;
            if (on) {
                float3 d = volume_ray(r, frays, s1, s2);
                Hit h = walk<BVH, COUNT, WT>(S, o, d, P.reach[1], false, key + r, seed, c);
                float3 l = sky(P, d);
                if (h.tri != NONE) {
                    bk = h.back;
                    l = h.back ? mk(0.f, 0.f, 0.f) : bounced(S, P, light, n_light, o, d, h);
                }
                if (rec) rec[size_t(k) * rays + r] = gather_record(S, P, n_light, o, d, h);
                t0 = scl(l, 0.282095f);
                float3 lw = scl(l, 0.488603f);
                tx = scl(lw, d.x);
                ty = scl(lw, d.y);
                tz = scl(lw, d.z);
            }
            l0 = ordered_add3(l0, t0, on);
            l1x = ordered_add3(l1x, tx, on);
            l1y = ordered_add3(l1y, ty, on);
            l1z = ordered_add3(l1z, tz, on);
            nback += __popc(__ballot_sync(FULL, bk));
        }
        float w = 4.0f * PI / frays;
        uint32_t g = P.counts[0], gg = g * g;
        Frame sf = frame(xyz(P.sun_dir));
        uint32_t nsun = 0;
        for (uint32_t s0 = 0; s0 < gg; s0 += 32) {
            uint32_t s = s0 + uint32_t(lane);
            bool esc = false;
            if (s < gg) {
                float3 d = sun_disc(P, sf, s, gg);
                esc = walk<BVH, COUNT, WT>(S, o, d, FAR, true, key + s + 9000u, seed, c).tri == NONE;
            }
            nsun += __popc(__ballot_sync(FULL, esc));
        }
        if (lane < 4) {
            float3 a0 = scl(l0, w), ax = scl(l1x, w), ay = scl(l1y, w), az = scl(l1z, w);
            float4 rec;
            if (lane == 0) rec = make_float4(a0.x, a0.y, a0.z, __uint2float_rn(nsun) / __uint2float_rn(gg));
            else if (lane == 1) rec = make_float4(ax.x, ax.y, ax.z, __uint2float_rn(nback) / frays);
            else if (lane == 2) rec = make_float4(ay.x, ay.y, ay.z, 0.0f);
            else rec = make_float4(az.x, az.y, az.z, 0.0f);
            uint32_t dst = slot ? __ldg(&slot[k]) : k;
            out[4 * dst + lane] = rec;
        }
    }
    flush_counts<COUNT>(c, counters);
}

}  // namespace lbd

// The walk a pass's occlusion or gather rays take (a template parameter, so that each kernel carries only
// its own): 0 the tree walk, 1 leaf lists (BVH2; the tree walk when a list overflows), 2 lane refill (BVH2).
static int walk_of(const WarpPass &w) {
    if (w.bvh != 2 || w.pass == LB_PASS_VOLUME) return 0;
    if (w.refill) return 2;
    return w.near ? 1 : 0;
}

template <int BVH, bool COUNT, int OCC, int WALK, bool WT> int blocks_walk(int pass) {
    const int T = 256;
    int per_sm = 0;
    cudaError_t e;
    switch (pass) {
    case LB_PASS_DIRECT:
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, lbd::direct_warp<BVH, COUNT, OCC, WALK, WT>, T, 0);
        break;
    case LB_PASS_GATHER:
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, lbd::gather_warp<BVH, COUNT, OCC, WALK, WT>, T, 0);
        break;
    default:
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, lbd::volume_warp<BVH, COUNT, WT>, T, 0);
        break;
    }
    return (e != cudaSuccess || per_sm < 1) ? 1 : per_sm;
}

template <int BVH, bool COUNT, int OCC, int WALK, bool WT>
void launch_walk(const WarpPass &w, int blocks, cudaStream_t stream) {
    const int T = 256;
    switch (w.pass) {
    case LB_PASS_DIRECT:
        lbd::direct_warp<BVH, COUNT, OCC, WALK, WT><<<blocks, T, 0, stream>>>(
            *w.S, *w.P, w.tex, w.idx, w.n_dev, w.n_host, w.base, w.out, w.counters, w.group, w.refill, w.near, w.work,
            w.warp_walk, w.part, w.parts);
        break;
    case LB_PASS_GATHER:
        lbd::gather_warp<BVH, COUNT, OCC, WALK, WT><<<blocks, T, 0, stream>>>(
            *w.S, *w.P, w.tex, w.idx, w.pos, w.n_dev, w.n_host, w.base, w.light, w.n_light, w.out, w.counters, w.group,
            w.refill, w.rec, w.work, w.part, w.parts);
        break;
    default:
        lbd::volume_warp<BVH, COUNT, WT><<<blocks, T, 0, stream>>>(*w.S, *w.P, w.tex, w.n_host, w.light, w.n_light,
                                                                   w.out, w.slot, w.counters, w.part, w.parts, w.rec);
        break;
    }
}

// the watertight kernels: the scene has vertices (lb_scene_set_vertices); a pass sized before its scene
// is known is sized as the shader's test
static bool watertight(const WarpPass &w) { return w.S != nullptr && w.S->verts != nullptr; }

template <int BVH, bool COUNT, int OCC = 1> int blocks_for(const WarpPass &w) {
    if (watertight(w)) {
        switch (walk_of(w)) {
        case 1: return blocks_walk<BVH, COUNT, 1, 1, true>(w.pass);
        case 2: return blocks_walk<BVH, COUNT, 1, 2, true>(w.pass);
        default: return blocks_walk<BVH, COUNT, 1, 0, true>(w.pass);
        }
    }
    switch (walk_of(w)) {
    case 1: return blocks_walk<BVH, COUNT, OCC, 1, false>(w.pass);
    case 2: return blocks_walk<BVH, COUNT, OCC, 2, false>(w.pass);
    default: return blocks_walk<BVH, COUNT, OCC, 0, false>(w.pass);
    }
}

template <int BVH, bool COUNT, int OCC = 1> void launch(const WarpPass &w, int blocks, cudaStream_t stream) {
    if (watertight(w)) {
        switch (walk_of(w)) {
        case 1: launch_walk<BVH, COUNT, 1, 1, true>(w, blocks, stream); break;
        case 2: launch_walk<BVH, COUNT, 1, 2, true>(w, blocks, stream); break;
        default: launch_walk<BVH, COUNT, 1, 0, true>(w, blocks, stream); break;
        }
        return;
    }
    switch (walk_of(w)) {
    case 1: launch_walk<BVH, COUNT, OCC, 1, false>(w, blocks, stream); break;
    case 2: launch_walk<BVH, COUNT, OCC, 2, false>(w, blocks, stream); break;
    default: launch_walk<BVH, COUNT, OCC, 0, false>(w, blocks, stream); break;
    }
}

// the register-capped variants exist for the BVH2 walk without counting (the product's passes) with the
// shader's triangle test
static bool capped(const WarpPass &w) {
    return w.bvh == 2 && !w.full_count && w.pass != LB_PASS_VOLUME && (w.occ == 3 || w.occ == 4) && !watertight(w);
}

int lb_warp_pass_blocks(const WarpPass &w) {
    int per_sm;
    if (capped(w)) per_sm = w.occ == 3 ? blocks_for<2, false, 3>(w) : blocks_for<2, false, 4>(w);
    else
        per_sm = w.bvh == 8 ? (w.full_count ? blocks_for<8, true>(w) : blocks_for<8, false>(w))
                            : (w.full_count ? blocks_for<2, true>(w) : blocks_for<2, false>(w));
    return w.sms * per_sm;
}

cudaError_t lb_launch_pass_warp(const WarpPass &w, cudaStream_t stream) {
    const int T = 256;
    if (w.bvh == 8 && (w.S->nodes8 == nullptr || w.S->tris8 == nullptr)) return cudaErrorInvalidValue;
    int blocks = w.blocks > 0 ? w.blocks : lb_warp_pass_blocks(w);
    if (w.n_dev == nullptr) {
        // no more warps than the share's items
        const uint64_t parts = w.parts > 1 ? w.parts : 1, part = w.parts > 1 ? w.part : 0;
        const uint32_t mine = uint32_t(uint64_t(w.n_host) * (part + 1) / parts - uint64_t(w.n_host) * part / parts);
        uint32_t need = (mine + (T / 32) - 1) / (T / 32);
        if (need == 0) return cudaSuccess;
        if ((uint32_t)blocks > need) blocks = (int)need;
    }
    if (w.work && w.pass != LB_PASS_VOLUME) {
        cudaError_t e = cudaMemsetAsync(w.work, 0, sizeof(unsigned int), stream);
        if (e != cudaSuccess) return e;
    }
    if (capped(w)) {
        if (w.occ == 3) launch<2, false, 3>(w, blocks, stream);
        else launch<2, false, 4>(w, blocks, stream);
    } else if (w.bvh == 8) {
        if (w.full_count) launch<8, true>(w, blocks, stream);
        else launch<8, false>(w, blocks, stream);
    } else {
        if (w.full_count) launch<2, true>(w, blocks, stream);
        else launch<2, false>(w, blocks, stream);
    }
    return cudaGetLastError();
}
