// Device-side building blocks of the bake passes: the sample sequence, the ray frames, the sky, and
// the walk of the reference's BVH2 (crates/lightbaker/src/gpu/trace.wgsl:41-168). Every float
// operation is written in the shader's source order and this code is built with -fmad=false, so a
// result rounds exactly as the shader's source says (no contraction into fused multiply-adds).
#pragma once
#include <cstdint>

#include "../../include/lightbaker.h"

namespace lbd {

constexpr float PI = 3.14159265f;       // trace.wgsl:33
constexpr float FAR = 1e30f;            // :34
constexpr uint32_t NONE = 0xffffffffu;  // :35
constexpr float PUSH = 0.03f;           // :37
constexpr int STACK = 48;               // :86

// The scene as the kernels read it: float4 records, 16-byte aligned (node: 2, triangle: 3,
// material: 1, chart: 2).
struct Scene {
    const float4 *nodes;
    const float4 *tris;
    const float4 *mats;
    const float4 *charts;
    uint32_t n_nodes, n_tris, n_mats, n_charts;
    // the 8-wide BVH (host/bvh8.h): 5 uint4 a node, its triangle copy (e2.w: the reference index)
    const uint4 *nodes8 = nullptr;
    const float4 *tris8 = nullptr;
    // the triangles' exact vertices (3 float4 a triangle, BVH2 order): set, the walks use the watertight
    // triangle test and scale each box's exit distance by `grow` (1 + 4e-7, above the slab test's
    // rounding: Ize, "Robust BVH Ray Traversal", JCGT 2(2), 2013), so a box holding a hit is not missed;
    // 1 without vertices (the shader's tests, unchanged)
    const float4 *verts = nullptr;
    float grow = 1.0f;
    // the most inner nodes on any root-to-leaf path of the BVH2 (0xffffffff: not known)
    uint32_t depth = 0xffffffffu;
};

constexpr int STACK8 = 96;  // node groups the 8-wide walk can hold (depth x 7 at most)

// Work counters a thread keeps when counting is on (lb_counters).
struct Count {
    uint32_t rays, nodes, tris, mats;
    __device__ void zero() { rays = nodes = tris = mats = 0; }
};

// The share of a pass's items [0, n) that one rank of a split bake takes: [n part / parts, n (part + 1) /
// parts), contiguous, the shares covering every item once (parts 0 or 1: all of them). An item keeps its
// index, and so its key and its output slot, whichever rank takes it.
__device__ __forceinline__ void item_part(uint32_t n, uint32_t part, uint32_t parts, uint32_t &lo, uint32_t &hi) {
    if (parts <= 1) {
        lo = 0;
        hi = n;
        return;
    }
    lo = uint32_t(uint64_t(n) * part / parts);
    hi = uint32_t(uint64_t(n) * (part + 1) / parts);
}

__device__ __forceinline__ float3 mk(float x, float y, float z) { return make_float3(x, y, z); }
__device__ __forceinline__ float3 add(float3 a, float3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 sub(float3 a, float3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 scl(float3 a, float s) { return mk(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ float3 mulv(float3 a, float3 b) { return mk(a.x * b.x, a.y * b.y, a.z * b.z); }
__device__ __forceinline__ float dot3(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float3 cross3(float3 a, float3 b) {
    return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float3 norm3(float3 v) { return scl(v, 1.0f / sqrtf(dot3(v, v))); }
__device__ __forceinline__ float3 xyz(float4 v) { return mk(v.x, v.y, v.z); }
__device__ __forceinline__ float3 xyz(const float *p) { return mk(p[0], p[1], p[2]); }
__device__ __forceinline__ float fract(float x) { return x - floorf(x); }

// trace.wgsl:41-45
__device__ __forceinline__ uint32_t pcg(uint32_t v) {
    uint32_t s = v * 747796405u + 2891336453u;
    uint32_t w = ((s >> ((s >> 28u) + 4u)) ^ s) * 277803737u;
    return (w >> 22u) ^ w;
}
// trace.wgsl:46; u32 to f32 rounds to nearest, times 2^-32 (exact)
__device__ __forceinline__ float rnd(uint32_t a, uint32_t b, uint32_t seed) {
    return __uint2float_rn(pcg(a ^ pcg(b + seed))) * 0x1p-32f;
}
// trace.wgsl:49
__device__ __forceinline__ float radical(uint32_t i) { return __uint2float_rn(__brev(i)) * 0x1p-32f; }

// Sine and cosine of a (a >= 0), one algorithm for the kernels and the CPU oracle: Cody-Waite
// reduction by pi/2 (pi/2 split in three floats of 12, 12 and 24 significant bits), then Taylor
// polynomials of sin (to r^9) and cos (to r^10) on |r| <= pi/4 by Horner. Truncation < 3e-9.
__device__ __forceinline__ void sincos32(float a, float *s, float *c) {
    const float TWO_OVER_PI = 0x1.45f306p-1f;
    const float P1 = 0x1.92p+0f, P2 = 0x1.fb4p-12f, P3 = 0x1.4442d2p-24f;
    float k = rintf(a * TWO_OVER_PI);
    float r = ((a - k * P1) - k * P2) - k * P3;
    float r2 = r * r;
    float sp = r + r * r2 * (-0x1.555556p-3f + r2 * (0x1.111112p-7f + r2 * (-0x1.a01a02p-13f + r2 * 0x1.71de3ap-19f)));
    float cp = 1.0f + r2 * (-0.5f + r2 * (0x1.555556p-5f + r2 * (-0x1.6c16c2p-10f + r2 * (0x1.a01a02p-16f + r2 * -0x1.27e4fcp-22f))));
    int q = int(k) & 3;
    float ss = (q & 1) ? cp : sp, cc = (q & 1) ? sp : cp;
    *s = (q & 2) ? -ss : ss;
    *c = (q == 1 || q == 2) ? -cc : cc;
}

struct Frame {
    float3 t, b, n;
};
// trace.wgsl:51-55
__device__ __forceinline__ Frame frame(float3 n) {
    float3 a = fabsf(n.y) > 0.9f ? mk(1.0f, 0.0f, 0.0f) : mk(0.0f, 1.0f, 0.0f);
    float3 t = norm3(cross3(a, n));
    return Frame{t, cross3(n, t), n};
}
// mat3x3f(t, b, n) * (x, y, z), columns summed in order
__device__ __forceinline__ float3 apply(const Frame &f, float x, float y, float z) {
    return add(add(scl(f.t, x), scl(f.b, y)), scl(f.n, z));
}
// trace.wgsl:57-61
__device__ __forceinline__ float3 cosine(float u, float v, const Frame &f) {
    float r = sqrtf(u);
    float a = v * 2.0f * PI;
    float s, c;
    sincos32(a, &s, &c);
    return norm3(apply(f, r * c, r * s, sqrtf(fmaxf(0.0f, 1.0f - u))));
}
// trace.wgsl:63-66; mix(h, z, t) = h * (1 - t) + z * t
__device__ __forceinline__ float3 sky(const lb_params &P, float3 d) {
    if (d.y < 0.0f) return xyz(P.ground);
    return add(scl(xyz(P.horizon), 1.0f - d.y), scl(xyz(P.zenith), d.y));
}
// trace.wgsl:219-221 and :314-316: spiral sample k of gg on the sun's disc
__device__ __forceinline__ float3 sun_disc(const lb_params &P, const Frame &sf, uint32_t k, uint32_t gg) {
    float a = __uint2float_rn(k) * 2.399963f;
    float r = P.sun_dir[3] * sqrtf((__uint2float_rn(k) + 0.5f) / __uint2float_rn(gg));
    float s, c;
    sincos32(a, &s, &c);
    return norm3(add(add(xyz(P.sun_dir), scl(scl(sf.t, c), r)), scl(scl(sf.b, s), r)));
}
// trace.wgsl:289-295: volume ray r of a probe whose seeds are s1, s2 (of frays rays), uniform over the sphere
__device__ __forceinline__ float3 volume_ray(uint32_t r, float frays, float s1, float s2) {
    float u = fract((__uint2float_rn(r) + 0.5f) / frays + s1);
    float v = fract(radical(r) + s2);
    float z = 1.0f - 2.0f * u;
    float rr = sqrtf(fmaxf(0.0f, 1.0f - z * z));
    float a = v * 2.0f * PI;
    float sa, ca;
    sincos32(a, &sa, &ca);
    return mk(rr * ca, z, rr * sa);
}
// trace.wgsl:152-156
__device__ __forceinline__ float2 offset(uint32_t q) {
    if (q <= 4u) return make_float2((q & 1u) ? 0.3f : -0.3f, q > 2u ? 0.3f : -0.3f);
    switch (q) {
    case 5: return make_float2(-0.45f, 0.0f);
    case 6: return make_float2(0.45f, 0.0f);
    case 7: return make_float2(0.0f, -0.45f);
    default: return make_float2(0.0f, 0.45f);
    }
}

struct Hit {
    float t;
    uint32_t tri;
    bool back;
};

// trace.wgsl:69-72
template <bool COUNT>
__device__ __forceinline__ bool stops(const Scene &S, uint32_t tri, float v0w, uint32_t ray, uint32_t seed, Count &c) {
    if (COUNT) c.mats++;
    uint32_t m = __float_as_uint(v0w);
    float op = m < S.n_mats ? __ldg(&S.mats[m]).w : 1.0f;
    return op >= 1.0f || rnd(tri * 9781u, ray, seed) < op;
}

// ---- the triangle test ----
__device__ __forceinline__ float comp(float3 v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }

// The watertight test of Woop, Benthin and Wald ("Watertight Ray/Triangle Intersection", JCGT 2(1), 2013),
// restated: the ray's largest axis kz, the other two in the order that keeps the frame's handedness,
// the shear that takes d onto +z, then the three edge functions of the sheared vertices, each a
// difference of two rounded products (recomputed in FP64 when one is exactly zero). An edge two
// triangles share gives them edge functions that are exact negatives of each other, so a ray meets
// at least one of them and never passes between. The shear keeps orientation, so det's sign is the
// shader's det's sign. Returns (t, det) of a hit, t = -1 for a miss (every accepted t is above 1e-4).
static __device__ __noinline__ float2 watertight(const float4 *verts, uint32_t ref, float3 o, float3 d) {
    float ax = fabsf(d.x), ay = fabsf(d.y), az = fabsf(d.z);
    int kz = (ax >= ay && ax >= az) ? 0 : (ay >= az ? 1 : 2);
    int kx = kz == 2 ? 0 : kz + 1;
    int ky = kx == 2 ? 0 : kx + 1;
    float dz = comp(d, kz);
    if (dz < 0.0f) {
        int k = kx;
        kx = ky;
        ky = k;
    }
    float sx = comp(d, kx) / dz, sy = comp(d, ky) / dz, sz = 1.0f / dz;
    const float4 *v = verts + 3 * size_t(ref);
    float4 a4 = __ldg(v), b4 = __ldg(v + 1), c4 = __ldg(v + 2);
    float3 A = sub(xyz(a4), o), B = sub(xyz(b4), o), C = sub(xyz(c4), o);
    float Az = comp(A, kz), Bz = comp(B, kz), Cz = comp(C, kz);
    float Ax = comp(A, kx) - sx * Az, Ay = comp(A, ky) - sy * Az;
    float Bx = comp(B, kx) - sx * Bz, By = comp(B, ky) - sy * Bz;
    float Cx = comp(C, kx) - sx * Cz, Cy = comp(C, ky) - sy * Cz;
    float U = Cx * By - Cy * Bx, V = Ax * Cy - Ay * Cx, W = Bx * Ay - By * Ax;
    if (U == 0.0f || V == 0.0f || W == 0.0f) {
        // products of two floats are exact in FP64: the edge functions' signs are exact
        U = float(double(Cx) * double(By) - double(Cy) * double(Bx));
        V = float(double(Ax) * double(Cy) - double(Ay) * double(Cx));
        W = float(double(Bx) * double(Ay) - double(By) * double(Ax));
    }
    float2 miss = make_float2(-1.0f, 0.0f);
    if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return miss;
    float det = U + V + W;
    if (det == 0.0f) return miss;
    float T = U * (sz * Az) + V * (sz * Bz) + W * (sz * Cz);
    return make_float2(T / det, det);
}

// Whether the ray meets triangle `ref` (v0, e1, e2: its record), with its t and face (back: the shader's
// det < 0). WT false: Möller-Trumbore in the shader's arithmetic (trace.wgsl:105-121); true: the watertight
// test over the scene's vertices. The caller applies the window (1e-4, nearest so far). Each walk is
// built for both and picks once at its start, so the shader's test carries nothing of the other.
template <bool WT>
__device__ __forceinline__ bool tri_hit(const Scene &S, uint32_t ref, float4 v0, float4 e1, float4 e2, float3 o,
                                        float3 d, float &t, bool &back) {
    if (WT) {
        float2 r = watertight(S.verts, ref, o, d);
        t = r.x;
        back = r.y < 0.0f;
        return r.x >= 0.0f;
    }
    float3 p = cross3(d, xyz(e2));
    float det = dot3(xyz(e1), p);
    if (fabsf(det) < 1e-12f) return false;
    // 1 / det rounded to nearest: the same bits as the division (both are the correctly rounded reciprocal)
    float id = __frcp_rn(det);
    float3 s = sub(o, xyz(v0));
    float u = dot3(s, p) * id;
    if (u < 0.0f || u > 1.0f) return false;
    float3 q = cross3(s, xyz(e1));
    float v = dot3(d, q) * id;
    if (v < 0.0f || u + v > 1.0f) return false;
    t = dot3(xyz(e2), q) * id;
    back = det < 0.0f;
    return true;
}

// Three-way max and min in one instruction each (sm_100's three-source max.f32 / min.f32): the values
// of max(max(a, b), c) and min(min(a, b), c); only the sign of a zero result can differ, and the walk
// only compares these distances.
__device__ __forceinline__ float max3(float a, float b, float c) {
    float r;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}
__device__ __forceinline__ float min3(float a, float b, float c) {
    float r;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}

// trace.wgsl:74-80; the watertight walks (WT) scale the exit distance by `grow`
// `skip` > 0: a box the ray leaves before skip counts as missed (for a caller that knows no hit lies
// that close).
template <bool WT = false>
__device__ __forceinline__ float box(float3 o, float3 inv, float4 mn, float4 mx, float tmax, float grow = 1.0f,
                                     float skip = 0.0f) {
    float ax = (mn.x - o.x) * inv.x, ay = (mn.y - o.y) * inv.y, az = (mn.z - o.z) * inv.z;
    float bx = (mx.x - o.x) * inv.x, by = (mx.y - o.y) * inv.y, bz = (mx.z - o.z) * inv.z;
    float lo = max3(fminf(ax, bx), fminf(ay, by), fminf(az, bz));
    float hi = min3(fmaxf(ax, bx), fmaxf(ay, by), fmaxf(az, bz));
    if (WT) hi = hi * grow;
    float l0 = fmaxf(lo, 0.0f);
    if (skip > 0.0f && hi < skip) return FAR;
    return (hi >= l0 && lo < tmax) ? l0 : FAR;
}

// trace.wgsl:83-130: the nearest hit within tmax (any: the first accepted). A thread's own walk with
// a 48-entry stack; a far child that finds it full is dropped as in the shader. Child records are
// carried into the next step instead of being read again; a popped node is read once. The root's box
// is never tested (the shader starts at its children). An inner node whose children lie past the
// array ends the walk (the reference's one-node BVH of an empty scene). skip > 0 passes over the boxes the
// ray leaves before skip: for a ray known to have no accepted hit that close, in a tree no deeper than the
// stack (so no child is ever dropped), the walk opens the same other boxes in the same order and holds the
// same hits, so it returns the full walk's hit.
template <bool COUNT, bool WT>
__device__ __forceinline__ Hit trace_t(const Scene &S, float3 o, float3 d, float tmax, bool any, uint32_t ray,
                                       uint32_t seed, Count &c, float skip = 0.0f) {
    Hit hit{tmax, NONE, false};
    c.rays++;
    if (COUNT) c.nodes++;
    float3 dd = mk(fabsf(d.x) < 1e-12f ? 1e-12f : d.x, fabsf(d.y) < 1e-12f ? 1e-12f : d.y,
                   fabsf(d.z) < 1e-12f ? 1e-12f : d.z);
    float3 inv = mk(1.0f / dd.x, 1.0f / dd.y, 1.0f / dd.z);
    uint32_t stack[STACK];
    int sp = 0;
    float4 nlo = __ldg(&S.nodes[0]), nhi = __ldg(&S.nodes[1]);
    for (;;) {
        uint32_t first = __float_as_uint(nlo.w), count = __float_as_uint(nhi.w);
        bool moved = false;
        if (count > 0u) {
            for (uint32_t i = first; i < first + count; i++) {
                if (COUNT) c.tris++;
                float4 v0 = __ldg(&S.tris[3 * i]), e1 = __ldg(&S.tris[3 * i + 1]), e2 = __ldg(&S.tris[3 * i + 2]);
                float t;
                bool bk;
                if (!tri_hit<WT>(S, i, v0, e1, e2, o, d, t, bk)) continue;
                if (t > 1e-4f && t < hit.t && stops<COUNT>(S, i, v0.w, ray, seed, c)) {
                    hit = Hit{t, i, bk};
                    if (any) return hit;
                }
            }
        } else if (first + 1u < S.n_nodes) {
            if (COUNT) c.nodes += 2;
            float4 alo = __ldg(&S.nodes[2 * first]), ahi = __ldg(&S.nodes[2 * first + 1]);
            float4 blo = __ldg(&S.nodes[2 * first + 2]), bhi = __ldg(&S.nodes[2 * first + 3]);
            float ta = box<WT>(o, inv, alo, ahi, hit.t, S.grow, skip);
            float tb = box<WT>(o, inv, blo, bhi, hit.t, S.grow, skip);
            bool a_near = ta <= tb;
            float tn = fminf(ta, tb), tf = fmaxf(ta, tb);
            if (tn < FAR) {
                if (tf < FAR && sp < STACK) stack[sp++] = a_near ? first + 1u : first;
                nlo = a_near ? alo : blo;
                nhi = a_near ? ahi : bhi;
                moved = true;
            }
        }
        if (moved) continue;
        if (sp == 0) break;
        uint32_t n = stack[--sp];
        nlo = __ldg(&S.nodes[2 * n]);
        nhi = __ldg(&S.nodes[2 * n + 1]);
    }
    return hit;
}

// The BVH2 depth below which a per-ray walk never drops a child (its stack holds STACK entries and a walk
// pushes at most one a level): the warp walk below gives the per-ray walk's answers only then.
constexpr uint32_t WARP_WALK_DEPTH = STACK;

// Any-hit rays of a warp walked together: one traversal of the BVH2 shared by the warp's lanes, each lane
// with its own ray (`on`: it has one), a stack of (node, lanes) in shared memory (WARP_WALK_DEPTH entries).
// At an inner node every lane tests its own ray against both children's boxes (trace.wgsl:74-80, the same
// test as its own walk); the warp opens a child for the lanes whose rays enter it, the first child first,
// and keeps the other with its lanes. At a leaf each of those lanes tests the triangles for its own ray; a
// lane whose ray is stopped leaves the traversal. Returns whether the lane's ray escaped.
//
// The answer is each ray's own walk's (trace.wgsl:83-130 with `any`): both visit exactly the leaves whose
// boxes, all the way down, the ray enters (no child is ever dropped: the tree is no deeper than
// WARP_WALK_DEPTH, which the caller checks), and whether some triangle there stops the ray does not depend
// on the order they are tested in (the opacity coin is keyed by triangle and ray). Only the order and
// the work counters differ, so it runs without counting. For rays that start close together and head the
// same way (a texel's sun rays) the lanes' paths nearly coincide and the warp walks them in step.
template <bool WT>
__device__ __forceinline__ bool escapes_warp(const Scene &S, float3 o, float3 d, float tmax, uint32_t ray,
                                             uint32_t seed, bool on, uint32_t *st_node, uint32_t *st_mask, int lane,
                                             Count &c) {
    const unsigned me = 1u << lane;
    float3 dd = mk(fabsf(d.x) < 1e-12f ? 1e-12f : d.x, fabsf(d.y) < 1e-12f ? 1e-12f : d.y,
                   fabsf(d.z) < 1e-12f ? 1e-12f : d.z);
    float3 inv = mk(1.0f / dd.x, 1.0f / dd.y, 1.0f / dd.z);
    if (on) c.rays++;
    bool stopped = false;
    unsigned alive = __ballot_sync(0xffffffffu, on);  // lanes with a ray not yet stopped
    uint32_t node = 0;
    unsigned mask = alive;
    int sp = 0;
    while (alive) {
        const float4 nlo = __ldg(&S.nodes[2 * node]), nhi = __ldg(&S.nodes[2 * node + 1]);
        const uint32_t first = __float_as_uint(nlo.w), count = __float_as_uint(nhi.w);
        bool descend = false;
        if (count > 0u) {
            if ((mask & me) && !stopped) {
                for (uint32_t i = first; i < first + count; i++) {
                    float4 v0 = __ldg(&S.tris[3 * i]), e1 = __ldg(&S.tris[3 * i + 1]), e2 = __ldg(&S.tris[3 * i + 2]);
                    float t;
                    bool bk;
                    if (!tri_hit<WT>(S, i, v0, e1, e2, o, d, t, bk)) continue;
                    if (t > 1e-4f && t < tmax && stops<false>(S, i, v0.w, ray, seed, c)) {
                        stopped = true;
                        break;
                    }
                }
            }
            alive &= ~__ballot_sync(0xffffffffu, stopped);
        } else if (first + 1u < S.n_nodes) {
            const float4 alo = __ldg(&S.nodes[2 * first]), ahi = __ldg(&S.nodes[2 * first + 1]);
            const float4 blo = __ldg(&S.nodes[2 * first + 2]), bhi = __ldg(&S.nodes[2 * first + 3]);
            const bool in = (mask & me) && !stopped;
            const bool ha = in && box<WT>(o, inv, alo, ahi, tmax, S.grow) < FAR;
            const bool hb = in && box<WT>(o, inv, blo, bhi, tmax, S.grow) < FAR;
            const unsigned ma = __ballot_sync(0xffffffffu, ha), mb = __ballot_sync(0xffffffffu, hb);
            if (ma && mb) {
                if (sp < int(WARP_WALK_DEPTH)) {
                    if (lane == 0) {
                        st_node[sp] = first + 1u;
                        st_mask[sp] = mb;
                    }
                    sp++;
                }
                node = first;
                mask = ma;
                descend = true;
            } else if (ma | mb) {
                node = ma ? first : first + 1u;
                mask = ma ? ma : mb;
                descend = true;
            }
        }
        if (descend) continue;
        // the next kept child that still has a lane whose ray is not stopped
        __syncwarp();
        mask = 0;
        while (sp > 0 && !mask) {
            sp--;
            node = st_node[sp];
            mask = st_mask[sp] & alive;
        }
        __syncwarp();
        if (!mask) break;
    }
    return on && !stopped;
}

template <bool COUNT, bool WT = false>
__device__ __forceinline__ Hit trace(const Scene &S, float3 o, float3 d, float tmax, bool any, uint32_t ray,
                                     uint32_t seed, Count &c) {
    return trace_t<COUNT, WT>(S, o, d, tmax, any, ray, seed, c);
}

// trace() as a resumable walk: its state between nodes, so that a lane whose ray has ended can start
// another while its warp's other lanes go on. step() does what one pass of trace()'s loop does (one
// node: a leaf's triangles, or an inner node's two children, then a pop when there is nothing to
// descend to), so a ray visits the same nodes in the same order and ends with the same hit.
template <bool COUNT, bool WT = false>
struct Walk2 {
    float3 o, d, inv;
    uint32_t ray;
    bool any, done;
    Hit hit;
    float4 nlo, nhi;
    int sp;
    uint32_t stack[STACK];
    __device__ __forceinline__ void start(const Scene &S, float3 o_, float3 d_, float tmax, bool any_, uint32_t ray_,
                                          Count &c) {
        o = o_;
        d = d_;
        any = any_;
        ray = ray_;
        hit = Hit{tmax, NONE, false};
        c.rays++;
        if (COUNT) c.nodes++;
        float3 dd = mk(fabsf(d.x) < 1e-12f ? 1e-12f : d.x, fabsf(d.y) < 1e-12f ? 1e-12f : d.y,
                       fabsf(d.z) < 1e-12f ? 1e-12f : d.z);
        inv = mk(1.0f / dd.x, 1.0f / dd.y, 1.0f / dd.z);
        sp = 0;
        nlo = __ldg(&S.nodes[0]);
        nhi = __ldg(&S.nodes[1]);
        done = false;
    }
    __device__ __forceinline__ void step(const Scene &S, uint32_t seed, Count &c) {
        uint32_t first = __float_as_uint(nlo.w), count = __float_as_uint(nhi.w);
        if (count > 0u) {
            for (uint32_t i = first; i < first + count; i++) {
                if (COUNT) c.tris++;
                float4 v0 = __ldg(&S.tris[3 * i]), e1 = __ldg(&S.tris[3 * i + 1]), e2 = __ldg(&S.tris[3 * i + 2]);
                float t;
                bool bk;
                if (!tri_hit<WT>(S, i, v0, e1, e2, o, d, t, bk)) continue;
                if (t > 1e-4f && t < hit.t && stops<COUNT>(S, i, v0.w, ray, seed, c)) {
                    hit = Hit{t, i, bk};
                    if (any) {
                        done = true;
                        return;
                    }
                }
            }
        } else if (first + 1u < S.n_nodes) {
            if (COUNT) c.nodes += 2;
            float4 alo = __ldg(&S.nodes[2 * first]), ahi = __ldg(&S.nodes[2 * first + 1]);
            float4 blo = __ldg(&S.nodes[2 * first + 2]), bhi = __ldg(&S.nodes[2 * first + 3]);
            float ta = box<WT>(o, inv, alo, ahi, hit.t, S.grow);
            float tb = box<WT>(o, inv, blo, bhi, hit.t, S.grow);
            bool a_near = ta <= tb;
            float tn = fminf(ta, tb), tf = fmaxf(ta, tb);
            if (tn < FAR) {
                if (tf < FAR && sp < STACK) stack[sp++] = a_near ? first + 1u : first;
                nlo = a_near ? alo : blo;
                nhi = a_near ? ahi : bhi;
                return;
            }
        }
        if (sp == 0) {
            done = true;
            return;
        }
        uint32_t n = stack[--sp];
        nlo = __ldg(&S.nodes[2 * n]);
        nhi = __ldg(&S.nodes[2 * n + 1]);
    }
};

// ---- rays that end within a ball: occlusion rays (trace.wgsl:226-241) ----
// Every triangle a ray of length <= r from o can hit lies in a BVH2 leaf whose box comes within r of o,
// and, when the rays leave through the hemisphere about n (cosine rays: d.n >= 0), on the n side of o.
// A warp gathers those leaves once for an item; each of its rays then tests the same short list, a loop
// its lanes run together, instead of each walking the tree from the root on its own path.

constexpr int BALL_LEAVES = 192;  // leaves an item's list holds (more: the item walks the tree instead)
// nodes one level of the ball query holds; also the sort's scratch, so at least BALL_LEAVES
constexpr int BALL_FRONT = BALL_LEAVES;

__device__ __forceinline__ float box_dist2(float3 p, float4 mn, float4 mx) {
    float dx = fmaxf(fmaxf(mn.x - p.x, 0.0f), p.x - mx.x);
    float dy = fmaxf(fmaxf(mn.y - p.y, 0.0f), p.y - mx.y);
    float dz = fmaxf(fmaxf(mn.z - p.z, 0.0f), p.z - mx.z);
    return dx * dx + dy * dy + dz * dz;
}
// the largest (x - o).n over the box's corners
__device__ __forceinline__ float box_front(float3 o, float3 n, float4 mn, float4 mx) {
    float x = n.x >= 0.0f ? mx.x : mn.x, y = n.y >= 0.0f ? mx.y : mn.y, z = n.z >= 0.0f ? mx.z : mn.z;
    return (x - o.x) * n.x + (y - o.y) * n.y + (z - o.z) * n.z;
}

// A list entry: the leaf's node index, and in the top 4 bits which of its (at most 4) triangles the
// list's rays must test.
constexpr uint32_t LEAF_NODE = 0x0fffffffu;
constexpr int LEAF_MASK_SHIFT = 28;

// Warp-wide: the leaves within reach r of o on the n side (by a margin), into list (entries: node |
// triangle bits << 28, every triangle of the leaf), nearest first, with their boxes' squared distances
// from o in dist2. Returns their count, or -1 when a level or the list would overflow, a leaf holds more
// than 4 triangles or node indices need more than 28 bits. All lanes return the same value.
// (Dropping each leaf's triangles wholly behind o's plane from its bits was measured: testing them cost
// more than the triangle tests it saved.)
template <bool COUNT>
__device__ __noinline__ int ball_leaves(const Scene &S, float3 o, float r, float3 n, uint32_t *fa, uint32_t *fb,
                                        uint32_t *list, float *dist2, int lane, Count &c) {
    const unsigned FULLM = 0xffffffffu;
    float rr = r * 1.0001f + 1e-5f, r2 = rr * rr, margin = -(r * 1e-3f + 1e-4f);
    if (S.n_nodes > LEAF_NODE) return -1;
    float4 rlo = __ldg(&S.nodes[0]), rhi = __ldg(&S.nodes[1]);
    uint32_t rfirst = __float_as_uint(rlo.w), rcount = __float_as_uint(rhi.w);
    if (rcount > 0u) {
        if (rcount > 4u) return -1;
        if (lane == 0) {
            list[0] = ((1u << rcount) - 1u) << LEAF_MASK_SHIFT;
            dist2[0] = 0.0f;
        }
        __syncwarp();
        return 1;
    }
    if (rfirst + 1u >= S.n_nodes) return 0;
    if (lane < 2) fa[lane] = rfirst + uint32_t(lane);
    __syncwarp();
    int nf = 2, nl = 0;
    while (nf > 0) {
        int nn = 0;
        for (int base = 0; base < nf; base += 32) {
            int i = base + lane;
            bool leaf = false, inner = false, wide = false;
            uint32_t node = 0, first = 0, tris = 0;
            if (i < nf) {
                node = fa[i];
                float4 lo = __ldg(&S.nodes[2 * node]), hi = __ldg(&S.nodes[2 * node + 1]);
                if (COUNT) c.nodes++;
                if (box_dist2(o, lo, hi) <= r2 && box_front(o, n, lo, hi) >= margin) {
                    first = __float_as_uint(lo.w);
                    uint32_t count = __float_as_uint(hi.w);
                    if (count > 4u) {
                        wide = true;
                    } else if (count > 0u) {
                        leaf = true;
                        tris = count;
                    } else if (first + 1u < S.n_nodes) {
                        inner = true;
                    }
                }
            }
            if (__any_sync(FULLM, wide)) return -1;  // leaves of more than 4 triangles: the tree walk
            unsigned lm = __ballot_sync(FULLM, leaf), im = __ballot_sync(FULLM, inner);
            unsigned below = (1u << lane) - 1u;
            int lp = nl + __popc(lm & below), ip = nn + 2 * __popc(im & below);
            if (leaf && lp < BALL_LEAVES) list[lp] = node | (((1u << tris) - 1u) << LEAF_MASK_SHIFT);
            if (inner && ip + 1 < BALL_FRONT) {
                fb[ip] = first;
                fb[ip + 1] = first + 1u;
            }
            nl += __popc(lm);
            nn += 2 * __popc(im);
        }
        __syncwarp();
        if (nl > BALL_LEAVES || nn > BALL_FRONT) return -1;
        uint32_t *t = fa;
        fa = fb;
        fb = t;
        nf = nn;
    }
    // nearest first: rank by distance (ties by index), then place; keys in fb
    float *key = (float *)fb;
    for (int i = lane; i < nl; i += 32) {
        uint32_t node = list[i] & LEAF_NODE;
        key[i] = box_dist2(o, __ldg(&S.nodes[2 * node]), __ldg(&S.nodes[2 * node + 1]));
    }
    __syncwarp();
    uint32_t mine[BALL_LEAVES / 32];
    int rank[BALL_LEAVES / 32];
    float mykey[BALL_LEAVES / 32];
    for (int q = 0; q < BALL_LEAVES / 32; q++) {
        int i = q * 32 + lane;
        rank[q] = -1;
        if (i < nl) {
            float ki = key[i];
            int rk = 0;
            for (int j = 0; j < nl; j++) {
                float kj = key[j];
                rk += (kj < ki || (kj == ki && j < i)) ? 1 : 0;
            }
            rank[q] = rk;
            mine[q] = list[i];
            mykey[q] = ki;
        }
    }
    __syncwarp();
    for (int q = 0; q < BALL_LEAVES / 32; q++)
        if (rank[q] >= 0) {
            fa[rank[q]] = mine[q];
            dist2[rank[q]] = mykey[q];
        }
    __syncwarp();
    for (int i = lane; i < nl; i += 32) list[i] = fa[i];
    __syncwarp();
    return nl;
}

// trace() over a leaf list: the nearest accepted hit within tmax among the listed leaves' triangles (an
// entry's mask names the leaf's triangles the list keeps), with the walk's box test (culled by the nearest
// hit so far) and triangle test. The list is nearest first from its centre (dist2: each box's squared
// distance from it), and the ray starts within `shift` of that centre, so once a box lies farther than the
// nearest hit so far plus shift (by a relative margin far above the rounding of t, |d| and the distance),
// neither it nor any later box can hold a nearer hit and the walk ends: the same hit as the whole list.
//
// Near ties. The tree walk keeps the nearest hit among the boxes it opens, and it skips a box whose
// entry is not below the hit it holds. So its answer differs from the list's nearest hit t only when
// (a) another accepted triangle lies exactly at t (then the order boxes are opened in picks one), or
// (b) a box on the tree's path to the hit has an entry that rounds up to t or past it, and another accepted
// triangle lies just beyond t (the tree may hold that one first and skip the hit's box). Every box on that
// path contains the hit's leaf box, so its entry is at most the leaf box's (in exact arithmetic; computed,
// within a few units in the last place of it), and the triangle the tree holds instead lies between the
// hit and that entry. With TIES the walk also opens boxes entered up to tie_reach past the hit (the larger
// of the hit and its box's entry, widened by 1e-5), notes the accepted triangles there by facing, and sets
// `tie` when the case can change what the caller reads; the caller then walks the tree for that ray:
//   TIE_GATHER  the hit's triangle (material, chart, point): (a) any face, or (b) any face;
//   TIE_OCC     t and the facing: (a) another facing, or (b) any face (another t);
//   TIE_INSIDE  the facing alone: (a) or (b) with another facing.
// Without TIES the nearest triangle found wins (the first in list order at an exact tie).
constexpr int TIE_NONE = 0, TIE_GATHER = 1, TIE_OCC = 2, TIE_INSIDE = 3;
// how far past a hit at t, whose box the walk entered at e, a triangle may lie and still decide a tie
__device__ __forceinline__ float tie_reach(float t, float e) { return fmaxf(t, e) * 1.00001f; }
template <bool COUNT, bool WT, int TIES>
__device__ __forceinline__ Hit trace_list_t(const Scene &S, const uint32_t *list, const float *dist2, int nl, float3 o,
                                            float3 d, float tmax, uint32_t ray, uint32_t seed, Count &c, float shift,
                                            bool &tie) {
    Hit hit{tmax, NONE, false};
    // TIES: the nearest accepted t of each facing but the hit's, and the entry of the hit's box
    float of_front = FAR, of_back = FAR, e_hit = 0.0f;
    c.rays++;
    float3 dd = mk(fabsf(d.x) < 1e-12f ? 1e-12f : d.x, fabsf(d.y) < 1e-12f ? 1e-12f : d.y,
                   fabsf(d.z) < 1e-12f ? 1e-12f : d.z);
    float3 inv = mk(1.0f / dd.x, 1.0f / dd.y, 1.0f / dd.z);
    float lim = (tmax + shift) * 1.0001f + 1e-5f, lim2 = lim * lim;
    // boxes open while entered before `cull`: the nearest hit; TIES: tie_reach past it, so that boxes entered
    // just past the hit open too, to see the triangles near it
    float cull = tmax;
    for (int k = 0; k < nl; k++) {
        if (dist2[k] > lim2) break;
        const uint32_t entry = list[k], node = entry & LEAF_NODE;
        float4 lo = __ldg(&S.nodes[2 * node]), hi = __ldg(&S.nodes[2 * node + 1]);
        if (COUNT) c.nodes++;
        const float eb = box<WT>(o, inv, lo, hi, cull, S.grow);
        if (!(eb < FAR)) continue;
        const uint32_t first = __float_as_uint(lo.w);
        for (uint32_t m = entry >> LEAF_MASK_SHIFT; m; m &= m - 1u) {
            const uint32_t i = first + uint32_t(__ffs(int(m)) - 1);
            if (COUNT) c.tris++;
            float4 v0 = __ldg(&S.tris[3 * i]), e1 = __ldg(&S.tris[3 * i + 1]), e2 = __ldg(&S.tris[3 * i + 2]);
            float t;
            bool bk;
            if (!tri_hit<WT>(S, i, v0, e1, e2, o, d, t, bk)) continue;
            const bool nearer = t > 1e-4f && t < hit.t;
            const bool close = TIES && !nearer && hit.tri != NONE && t > 1e-4f && t <= tie_reach(hit.t, e_hit);
            if (!(nearer || close) || !stops<COUNT>(S, i, v0.w, ray, seed, c)) continue;
            if (nearer) {
                if (TIES && hit.tri != NONE) {
                    if (hit.back) of_back = fminf(of_back, hit.t);
                    else of_front = fminf(of_front, hit.t);
                }
                hit = Hit{t, i, bk};
                e_hit = eb;
                cull = TIES ? tie_reach(t, eb) : t;
                lim = (t + shift) * 1.0001f + 1e-5f;
                lim2 = lim * lim;
            } else if (bk) {
                of_back = fminf(of_back, t);
            } else {
                of_front = fminf(of_front, t);
            }
        }
    }
    tie = false;
    if (TIES != TIE_NONE && hit.tri != NONE) {
        const float same = hit.back ? of_back : of_front, other = hit.back ? of_front : of_back;
        // (b)'s first half: the hit's box entry, within rounding, at or past the hit
        const bool edge = e_hit * 1.00001f >= hit.t;
        const float w = tie_reach(hit.t, e_hit);
        if (TIES == TIE_GATHER) tie = same == hit.t || other == hit.t || (edge && fminf(same, other) <= w);
        else if (TIES == TIE_OCC) tie = other == hit.t || (edge && fminf(same, other) <= w);
        else tie = other == hit.t || (edge && other <= w);
    }
    return hit;
}
template <bool COUNT, bool WT = false>
__device__ __forceinline__ Hit trace_list(const Scene &S, const uint32_t *list, const float *dist2, int nl, float3 o,
                                          float3 d, float tmax, uint32_t ray, uint32_t seed, Count &c,
                                          float shift = 0.0f) {
    bool tie;
    return trace_list_t<COUNT, WT, TIE_NONE>(S, list, dist2, nl, o, d, tmax, ray, seed, c, shift, tie);
}

// The same query over the 8-wide BVH: the nearest accepted hit within tmax (any: the first accepted),
// the same triangle test in the same arithmetic, so every hit, its t and its face are the BVH2 walk's.
// A node's eight child boxes are tested at once; its leaf slots' triangles first, then its hit inner
// children nearest first (the rest pushed far to near with their entry distance, and skipped when
// popped beyond the nearest hit so far).
template <bool COUNT, bool WT>
__device__ __forceinline__ Hit trace8_t(const Scene &S, float3 o, float3 d, float tmax, bool any, uint32_t ray,
                                        uint32_t seed, Count &c) {
    Hit hit{tmax, NONE, false};
    c.rays++;
    float3 dd = mk(fabsf(d.x) < 1e-12f ? 1e-12f : d.x, fabsf(d.y) < 1e-12f ? 1e-12f : d.y,
                   fabsf(d.z) < 1e-12f ? 1e-12f : d.z);
    float3 inv = mk(1.0f / dd.x, 1.0f / dd.y, 1.0f / dd.z);
    uint32_t st_node[STACK8];
    float st_t[STACK8];
    int sp = 0;
    uint32_t n = 0;
    for (;;) {
        const uint4 *nd = S.nodes8 + 5 * size_t(n);
        uint4 a0 = __ldg(nd), a1 = __ldg(nd + 1), a2 = __ldg(nd + 2), a3 = __ldg(nd + 3), a4 = __ldg(nd + 4);
        if (COUNT) c.nodes++;
        float px = __uint_as_float(a0.x), py = __uint_as_float(a0.y), pz = __uint_as_float(a0.z);
        float sx = __uint_as_float((a0.w & 0xffu) << 23), sy = __uint_as_float(((a0.w >> 8) & 0xffu) << 23),
              sz = __uint_as_float(((a0.w >> 16) & 0xffu) << 23);
        uint32_t imask = a0.w >> 24;
        float tc[8];
        uint32_t leafmask = 0, innermask = 0;
#pragma unroll
        for (int s = 0; s < 8; s++) {
            uint32_t sh = uint32_t(s & 3) * 8u;
            uint32_t meta = ((s < 4 ? a1.z : a1.w) >> sh) & 0xffu;
            bool inner = (imask >> s) & 1u;
            if (!inner && meta == 0xffu) {
                tc[s] = FAR;
                continue;
            }
            float4 mn = make_float4(px + __uint2float_rn(((s < 4 ? a2.x : a2.y) >> sh) & 0xffu) * sx,
                                    py + __uint2float_rn(((s < 4 ? a2.z : a2.w) >> sh) & 0xffu) * sy,
                                    pz + __uint2float_rn(((s < 4 ? a3.x : a3.y) >> sh) & 0xffu) * sz, 0.0f);
            float4 mx = make_float4(px + __uint2float_rn(((s < 4 ? a3.z : a3.w) >> sh) & 0xffu) * sx,
                                    py + __uint2float_rn(((s < 4 ? a4.x : a4.y) >> sh) & 0xffu) * sy,
                                    pz + __uint2float_rn(((s < 4 ? a4.z : a4.w) >> sh) & 0xffu) * sz, 0.0f);
            float t = box<WT>(o, inv, mn, mx, hit.t, S.grow);
            tc[s] = t;
            if (t < FAR) {
                if (inner) innermask |= 1u << s;
                else leafmask |= 1u << s;
            }
        }
        while (leafmask) {
            int s = __ffs(leafmask) - 1;
            leafmask &= leafmask - 1;
            uint32_t meta = ((s < 4 ? a1.z : a1.w) >> (uint32_t(s & 3) * 8u)) & 0xffu;
            uint32_t first = a1.y + (meta & 31u), cnt = ((meta >> 5) & 3u) + 1u;
            for (uint32_t k = 0; k < cnt; k++) {
                if (COUNT) c.tris++;
                const float4 *tp = S.tris8 + 3 * size_t(first + k);
                float4 v0 = __ldg(tp), e1 = __ldg(tp + 1), e2 = __ldg(tp + 2);
                uint32_t orig = __float_as_uint(e2.w);
                float t;
                bool bk;
                if (!tri_hit<WT>(S, orig, v0, e1, e2, o, d, t, bk)) continue;
                if (t > 1e-4f && t < hit.t && stops<COUNT>(S, orig, v0.w, ray, seed, c)) {
                    hit = Hit{t, orig, bk};
                    if (any) return hit;
                }
            }
        }
        // inner children still nearer than the nearest hit: the nearest next, the rest on the stack
        uint32_t next = NONE;
        float tnext = FAR;
        uint32_t live = 0;
        for (uint32_t m = innermask; m; m &= m - 1) {
            int s = __ffs(m) - 1;
            if (tc[s] < hit.t) live |= 1u << s;
        }
        if (live) {
            // push far to near, keep the nearest
            while (live) {
                int far_s = -1;
                float tf = -1.0f;
                for (uint32_t m = live; m; m &= m - 1) {
                    int s = __ffs(m) - 1;
                    if (tc[s] >= tf) {
                        tf = tc[s];
                        far_s = s;
                    }
                }
                live &= ~(1u << far_s);
                uint32_t child = a1.x + __popc(imask & ((1u << far_s) - 1u));
                if (live == 0) {
                    next = child;
                    tnext = tf;
                } else if (sp < STACK8) {
                    st_node[sp] = child;
                    st_t[sp] = tf;
                    sp++;
                }
            }
        }
        if (next == NONE) {
            while (sp > 0) {
                sp--;
                if (st_t[sp] < hit.t) {
                    next = st_node[sp];
                    break;
                }
            }
            if (next == NONE) break;
        }
        (void)tnext;
        n = next;
    }
    return hit;
}
// The walk a pass uses: BVH 2 the reference's tree, 8 the 8-wide one; WT the watertight triangle test
// (the kernels are built for both and the launch picks by whether the scene has vertices).
template <int BVH, bool COUNT, bool WT = false>
__device__ __forceinline__ Hit walk(const Scene &S, float3 o, float3 d, float tmax, bool any, uint32_t ray,
                                    uint32_t seed, Count &c, float skip = 0.0f) {
    if (BVH == 8) return trace8_t<COUNT, WT>(S, o, d, tmax, any, ray, seed, c);
    return trace_t<COUNT, WT>(S, o, d, tmax, any, ray, seed, c, skip);
}
// The BVH2 walk for the rare ray a leaf list leaves to the tree (a near tie), as a call: one copy of the
// walk serves every such site instead of a copy inlined at each.
template <bool COUNT, bool WT>
__device__ __noinline__ Hit walk_apart(const Scene &S, float3 o, float3 d, float tmax, uint32_t ray, uint32_t seed,
                                       Count &c) {
    return trace_t<COUNT, WT>(S, o, d, tmax, false, ray, seed, c);
}

// A gather ray's outcome, all a bounce needs to evaluate it again against another light atlas:
// x = kind << 30 | material; y = the direction's y (sky, as bits) or the atlas texel the hit reads
// (surface; 0xffffffff when it reads none and takes the fallback), as bounced() finds it.
constexpr uint32_t KIND_SKY = 0u, KIND_BACK = 1u, KIND_SURFACE = 2u;
__device__ __forceinline__ uint2 gather_record(const Scene &S, const lb_params &P, uint32_t n_light, float3 o,
                                               float3 d, const Hit &h) {
    if (h.tri == NONE) return make_uint2(KIND_SKY << 30, __float_as_uint(d.y));
    if (h.back) return make_uint2(KIND_BACK << 30, 0u);
    float4 v0 = __ldg(&S.tris[3 * h.tri]), e1 = __ldg(&S.tris[3 * h.tri + 1]);
    uint32_t m = __float_as_uint(v0.w), ch = __float_as_uint(e1.w), li = NONE;
    if (ch != NONE && ch < S.n_charts) {
        float3 p = add(o, scl(d, h.t));
        float4 r0 = __ldg(&S.charts[2 * ch]), r1 = __ldg(&S.charts[2 * ch + 1]);
        float x = r0.x * p.x + r0.y * p.y + r0.z * p.z + r0.w * 1.0f;
        float y = r1.x * p.x + r1.y * p.y + r1.z * p.z + r1.w * 1.0f;
        int ix = min(max(int(floorf(x)), 0), int(P.atlas[0]) - 1);
        int iy = min(max(int(floorf(y)), 0), int(P.atlas[1]) - 1);
        uint32_t l = uint32_t(iy) * P.atlas[0] + uint32_t(ix);
        if (l < n_light) li = l;
    }
    return make_uint2((KIND_SURFACE << 30) | min(m, 0x3fffffffu), li);
}

// trace.wgsl:133-148
__device__ __forceinline__ float3 bounced(const Scene &S, const lb_params &P, const float4 *light, uint32_t n_light,
                                          float3 o, float3 d, const Hit &h) {
    float4 v0 = __ldg(&S.tris[3 * h.tri]), e1 = __ldg(&S.tris[3 * h.tri + 1]);
    uint32_t m = __float_as_uint(v0.w);
    float4 mat = m < S.n_mats ? __ldg(&S.mats[m]) : make_float4(0.f, 0.f, 0.f, 1.f);
    uint32_t ch = __float_as_uint(e1.w);
    float3 e = xyz(P.fallback);
    if (ch != NONE && ch < S.n_charts) {
        float3 p = add(o, scl(d, h.t));
        float4 r0 = __ldg(&S.charts[2 * ch]), r1 = __ldg(&S.charts[2 * ch + 1]);
        float x = r0.x * p.x + r0.y * p.y + r0.z * p.z + r0.w * 1.0f;
        float y = r1.x * p.x + r1.y * p.y + r1.z * p.z + r1.w * 1.0f;
        int ix = min(max(int(floorf(x)), 0), int(P.atlas[0]) - 1);
        int iy = min(max(int(floorf(y)), 0), int(P.atlas[1]) - 1);
        uint32_t li = uint32_t(iy) * P.atlas[0] + uint32_t(ix);
        if (li < n_light) {
            float4 l = __ldg(&light[li]);
            if (l.w > 0.5f) e = mk(l.x, l.y, l.z);
        }
    }
    return mulv(mk(mat.x / PI, mat.y / PI, mat.z / PI), e);
}

}  // namespace lbd
