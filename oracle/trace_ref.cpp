// ORACLE — test infrastructure only (see oracle.h). A scalar restatement of the reference's ray
// passes, crates/lightbaker/src/gpu/trace.wgsl, one function per shader function, each citing the
// lines it follows. The walk and the triangle test are templates on the scalar type: float is the
// shader's arithmetic in its source order (built without contraction), double is the FP64 twin.
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <type_traits>
#include <cstdint>
#include <cstring>
#include <vector>

#include "oracle.h"

namespace {

template <class T> struct V3 {
    T x, y, z;
};
template <class T> inline V3<T> mk(T x, T y, T z) { return V3<T>{x, y, z}; }
template <class T> inline V3<T> operator+(V3<T> a, V3<T> b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
template <class T> inline V3<T> operator-(V3<T> a, V3<T> b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
template <class T> inline V3<T> operator*(V3<T> a, T s) { return mk(a.x * s, a.y * s, a.z * s); }
template <class T> inline V3<T> mulv(V3<T> a, V3<T> b) { return mk(a.x * b.x, a.y * b.y, a.z * b.z); }
// WGSL dot and cross, summed left to right
template <class T> inline T dot(V3<T> a, V3<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class T> inline V3<T> cross(V3<T> a, V3<T> b) {
    return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
// normalize as v times the reciprocal of its length
template <class T> inline V3<T> normalize(V3<T> v) {
    T r = T(1) / std::sqrt(dot(v, v));
    return v * r;
}
template <class T> inline T vmin(T a, T b) { return std::fmin(a, b); }
template <class T> inline T vmax(T a, T b) { return std::fmax(a, b); }

inline V3<float> f3(const float *p) { return mk(p[0], p[1], p[2]); }
template <class T> inline V3<T> cvt(V3<float> v) { return mk(T(v.x), T(v.y), T(v.z)); }

const float PI = 3.14159265f;   // trace.wgsl:33
const float FAR = 1e30f;        // :34
const uint32_t NONE = 0xffffffffu;  // :35
const float PUSH = 0.03f;       // :37
const float INV_2_32 = 0x1p-32f;    // 1 / 4294967296, exact

inline uint32_t fbits(float f) { uint32_t u; std::memcpy(&u, &f, 4); return u; }
inline float bitsf(uint32_t u) { float f; std::memcpy(&f, &u, 4); return f; }

// trace.wgsl:41-45
inline uint32_t pcg(uint32_t v) {
    uint32_t s = v * 747796405u + 2891336453u;
    uint32_t w = ((s >> ((s >> 28u) + 4u)) ^ s) * 277803737u;
    return (w >> 22u) ^ w;
}
// trace.wgsl:46 (seed: bits of reach.w)
inline float rnd(uint32_t a, uint32_t b, uint32_t seed) { return float(pcg(a ^ pcg(b + seed))) * INV_2_32; }
inline uint32_t rev32(uint32_t v) {
    v = ((v >> 1) & 0x55555555u) | ((v & 0x55555555u) << 1);
    v = ((v >> 2) & 0x33333333u) | ((v & 0x33333333u) << 2);
    v = ((v >> 4) & 0x0f0f0f0fu) | ((v & 0x0f0f0f0fu) << 4);
    v = ((v >> 8) & 0x00ff00ffu) | ((v & 0x00ff00ffu) << 8);
    return (v >> 16) | (v << 16);
}
// trace.wgsl:49
inline float radical(uint32_t i) { return float(rev32(i)) * INV_2_32; }
inline float fract(float x) { return x - std::floor(x); }

// Sine and cosine, the same on both sides of the parity tests: Cody-Waite reduction by pi/2 (pi/2 split
// in three floats with 12, 12 and 24 significant bits), then the Taylor series of sin (to r^9) and cos
// (to r^10) on |r| <= pi/4, evaluated by Horner in float. Truncation error < 3e-9 on that range.
inline void sincos32(float a, float *s, float *c) {
    const float TWO_OVER_PI = 0x1.45f306p-1f;
    const float P1 = 0x1.92p+0f, P2 = 0x1.fb4p-12f, P3 = 0x1.4442d2p-24f;
    float k = std::rint(a * TWO_OVER_PI);
    float r = ((a - k * P1) - k * P2) - k * P3;
    float r2 = r * r;
    float sp = r + r * r2 * (-0x1.555556p-3f + r2 * (0x1.111112p-7f + r2 * (-0x1.a01a02p-13f + r2 * 0x1.71de3ap-19f)));
    float cp = 1.0f + r2 * (-0.5f + r2 * (0x1.555556p-5f + r2 * (-0x1.6c16c2p-10f + r2 * (0x1.a01a02p-16f + r2 * -0x1.27e4fcp-22f))));
    int q = int(k) & 3;
    switch (q) {
    case 0: *s = sp; *c = cp; break;
    case 1: *s = cp; *c = -sp; break;
    case 2: *s = -sp; *c = -cp; break;
    default: *s = -cp; *c = sp; break;
    }
}

struct Frame {
    V3<float> t, b, n;
};
// trace.wgsl:51-55
inline Frame frame(V3<float> n) {
    V3<float> a = std::fabs(n.y) > 0.9f ? mk(1.0f, 0.0f, 0.0f) : mk(0.0f, 1.0f, 0.0f);
    V3<float> t = normalize(cross(a, n));
    return Frame{t, cross(n, t), n};
}
// mat3x3f(t, b, n) * v, columns summed in order
inline V3<float> apply(const Frame &f, float x, float y, float z) { return (f.t * x + f.b * y) + f.n * z; }
// trace.wgsl:57-61
inline V3<float> cosine(float u, float v, const Frame &f) {
    float r = std::sqrt(u);
    float a = v * 2.0f * PI;
    float s, c;
    sincos32(a, &s, &c);
    return normalize(apply(f, r * c, r * s, std::sqrt(vmax(0.0f, 1.0f - u))));
}

struct Ctx {
    const lb_node *nodes;
    size_t n_nodes;
    const lb_tri *tris;
    size_t n_tris;
    const float *mats;
    size_t n_mats;
    const float *charts;
    size_t n_charts;
    const float *light;
    size_t n_light;
    const lb_params *P;
    uint32_t seed;
    or_counters *cnt;  // per thread
    // exact vertices (9 floats a triangle): the FP32 walk uses the watertight test and widens box exits
    const float *verts = nullptr;
};

// trace.wgsl:63-66 (mix(a, b, t) = a * (1 - t) + b * t)
inline V3<float> sky(const Ctx &C, V3<float> d) {
    if (d.y < 0.0f) return f3(C.P->ground);
    float u = 1.0f - d.y;
    return f3(C.P->horizon) * u + f3(C.P->zenith) * d.y;
}

inline float material_opacity(const Ctx &C, uint32_t tri) {
    uint32_t m = fbits(C.tris[tri].v0[3]);
    return m < C.n_mats ? C.mats[m * 4 + 3] : 1.0f;
}
// trace.wgsl:69-72
inline bool stops(const Ctx &C, uint32_t tri, uint32_t ray) {
    if (C.cnt) C.cnt->mats++;
    float op = material_opacity(C, tri);
    return op >= 1.0f || rnd(tri * 9781u, ray, C.seed) < op;
}

// trace.wgsl:74-80; grow (1 for the shader) scales the exit distance for the watertight walk
template <class T> inline T box(V3<T> o, V3<T> inv, V3<T> mn, V3<T> mx, T tmax, T far, T grow = T(1)) {
    V3<T> a = mulv(mn - o, inv);
    V3<T> b = mulv(mx - o, inv);
    T lo = vmax(vmax(vmin(a.x, b.x), vmin(a.y, b.y)), vmin(a.z, b.z));
    T hi = vmin(vmin(vmax(a.x, b.x), vmax(a.y, b.y)), vmax(a.z, b.z));
    T l0 = vmax(lo, T(0));
    return (hi * grow >= l0 && lo < tmax) ? l0 : far;
}

// The watertight ray/triangle test (Woop, Benthin and Wald, "Watertight Ray/Triangle Intersection", JCGT
// 2(1), 2013) in FP32: shear the ray's largest axis onto +z (the other two in the order that keeps the
// frame's handedness), then three edge functions of the sheared vertices, each a difference of two
// rounded products, recomputed in FP64 when one is exactly zero. Writes t and the face (det < 0: back).
inline float axis(V3<float> v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }
inline bool watertight(const float *verts, uint32_t i, V3<float> o, V3<float> d, float &t, bool &back) {
    float ax = std::fabs(d.x), ay = std::fabs(d.y), az = std::fabs(d.z);
    int kz = (ax >= ay && ax >= az) ? 0 : (ay >= az ? 1 : 2);
    int kx = kz == 2 ? 0 : kz + 1;
    int ky = kx == 2 ? 0 : kx + 1;
    float dz = axis(d, kz);
    if (dz < 0.0f) std::swap(kx, ky);
    float sx = axis(d, kx) / dz, sy = axis(d, ky) / dz, sz = 1.0f / dz;
    const float *v = verts + size_t(i) * 9;
    V3<float> A = mk(v[0], v[1], v[2]) - o, B = mk(v[3], v[4], v[5]) - o, Cv = mk(v[6], v[7], v[8]) - o;
    float Az = axis(A, kz), Bz = axis(B, kz), Cz = axis(Cv, kz);
    float Ax = axis(A, kx) - sx * Az, Ay = axis(A, ky) - sy * Az;
    float Bx = axis(B, kx) - sx * Bz, By = axis(B, ky) - sy * Bz;
    float Cx = axis(Cv, kx) - sx * Cz, Cy = axis(Cv, ky) - sy * Cz;
    float U = Cx * By - Cy * Bx, V = Ax * Cy - Ay * Cx, W = Bx * Ay - By * Ax;
    if (U == 0.0f || V == 0.0f || W == 0.0f) {
        U = float(double(Cx) * double(By) - double(Cy) * double(Bx));
        V = float(double(Ax) * double(Cy) - double(Ay) * double(Cx));
        W = float(double(Bx) * double(Ay) - double(By) * double(Ax));
    }
    if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return false;
    float det = U + V + W;
    if (det == 0.0f) return false;
    float T = U * (sz * Az) + V * (sz * Bz) + W * (sz * Cz);
    t = T / det;
    back = det < 0.0f;
    return true;
}
constexpr float WATERTIGHT_GROW = 1.0000004f;

template <class T> struct Hit {
    T t;
    uint32_t tri;
    bool back;
};

// trace.wgsl:83-130: the stack walk (48 entries; a far child that finds the stack full is dropped),
// near child first, Moller-Trumbore with |det| < 1e-12 rejected, hits with 1e-4 < t < nearest that the
// triangle's material stops. The root's own box is never tested, as in the shader. An inner node whose
// children lie past the node array (the reference's one-node BVH of an empty scene) ends the walk.
template <class T> Hit<T> trace(const Ctx &C, V3<T> o, V3<T> d, T tmax, bool any, uint32_t ray) {
    const T far = T(FAR);
    Hit<T> hit{tmax, NONE, false};
    if (C.cnt) { C.cnt->rays++; C.cnt->nodes++; }
    const T tiny = T(1e-12f);
    V3<T> dd = mk(std::fabs(d.x) < tiny ? tiny : d.x, std::fabs(d.y) < tiny ? tiny : d.y,
                  std::fabs(d.z) < tiny ? tiny : d.z);
    V3<T> inv = mk(T(1) / dd.x, T(1) / dd.y, T(1) / dd.z);
    uint32_t stack[48];
    uint32_t sp = 0, n = 0;
    for (;;) {
        const lb_node &node = C.nodes[n];
        if (node.count > 0u) {
            for (uint32_t i = node.first; i < node.first + node.count; i++) {
                if (C.cnt) C.cnt->tris++;
                if constexpr (std::is_same_v<T, float>) {
                    if (C.verts) {
                        float t;
                        bool bk;
                        if (!watertight(C.verts, i, o, d, t, bk)) continue;
                        if (t > 1e-4f && t < hit.t && stops(C, i, ray)) {
                            hit = Hit<T>{t, i, bk};
                            if (any) return hit;
                        }
                        continue;
                    }
                }
                const lb_tri &tr = C.tris[i];
                V3<T> e1 = cvt<T>(f3(tr.e1)), e2 = cvt<T>(f3(tr.e2)), v0 = cvt<T>(f3(tr.v0));
                V3<T> p = cross(d, e2);
                T det = dot(e1, p);
                if (std::fabs(det) < tiny) continue;
                T id = T(1) / det;
                V3<T> s = o - v0;
                T u = dot(s, p) * id;
                if (u < T(0) || u > T(1)) continue;
                V3<T> q = cross(s, e1);
                T v = dot(d, q) * id;
                if (v < T(0) || u + v > T(1)) continue;
                T t = dot(e2, q) * id;
                if (t > T(1e-4f) && t < hit.t && stops(C, i, ray)) {
                    hit = Hit<T>{t, i, det < T(0)};
                    if (any) return hit;
                }
            }
        } else if (size_t(node.first) + 1 < C.n_nodes) {
            const lb_node &a = C.nodes[node.first];
            const lb_node &b = C.nodes[node.first + 1u];
            if (C.cnt) C.cnt->nodes += 2;
            const T grow = (std::is_same_v<T, float> && C.verts) ? T(WATERTIGHT_GROW) : T(1);
            T ta = box(o, inv, cvt<T>(f3(a.min)), cvt<T>(f3(a.max)), hit.t, far, grow);
            T tb = box(o, inv, cvt<T>(f3(b.min)), cvt<T>(f3(b.max)), hit.t, far, grow);
            uint32_t near = ta <= tb ? node.first : node.first + 1u;
            uint32_t farc = ta <= tb ? node.first + 1u : node.first;
            T tn = vmin(ta, tb), tf = vmax(ta, tb);
            if (tn < far) {
                if (tf < far) {
                    if (sp < 48u) stack[sp++] = farc;
                    else if (C.cnt) C.cnt->overflows++;
                }
                n = near;
                continue;
            }
        }
        if (sp == 0u) break;
        sp--;
        n = stack[sp];
    }
    return hit;
}

// trace.wgsl:133-148
inline V3<float> bounced(const Ctx &C, V3<float> o, V3<float> d, const Hit<float> &h) {
    const lb_tri &tr = C.tris[h.tri];
    uint32_t m = fbits(tr.v0[3]);
    V3<float> albedo = m < C.n_mats ? mk(C.mats[m * 4], C.mats[m * 4 + 1], C.mats[m * 4 + 2]) : mk(0.f, 0.f, 0.f);
    uint32_t c = fbits(tr.e1[3]);
    V3<float> e = f3(C.P->fallback);
    if (c != NONE && c < C.n_charts) {
        V3<float> p = o + d * h.t;
        const float *r0 = C.charts + size_t(c) * 8, *r1 = r0 + 4;
        float x = r0[0] * p.x + r0[1] * p.y + r0[2] * p.z + r0[3] * 1.0f;
        float y = r1[0] * p.x + r1[1] * p.y + r1[2] * p.z + r1[3] * 1.0f;
        int aw = int(C.P->atlas[0]), ah = int(C.P->atlas[1]);
        int ix = std::min(std::max(int(std::floor(x)), 0), aw - 1);
        int iy = std::min(std::max(int(std::floor(y)), 0), ah - 1);
        size_t li = size_t(uint32_t(iy)) * C.P->atlas[0] + uint32_t(ix);
        if (li < C.n_light) {
            const float *l = C.light + li * 4;
            if (l[3] > 0.5f) e = mk(l[0], l[1], l[2]);
        }
    }
    return mulv(mk(albedo.x / PI, albedo.y / PI, albedo.z / PI), e);
}

// trace.wgsl:152-156
inline void offset(uint32_t q, float *x, float *y) {
    if (q <= 4u) {
        *x = (q & 1u) == 1u ? 0.3f : -0.3f;
        *y = q > 2u ? 0.3f : -0.3f;
        return;
    }
    static const float e[4][2] = {{-0.45f, 0.0f}, {0.45f, 0.0f}, {0.0f, -0.45f}, {0.0f, 0.45f}};
    *x = e[q - 5u][0];
    *y = e[q - 5u][1];
}

// trace.wgsl:159-168
inline bool inside(const Ctx &C, V3<float> o, V3<float> n, uint32_t key) {
    Frame f = frame(n);
    float back = 0.0f;
    for (uint32_t r = 0; r < 16u; r++) {
        V3<float> d = cosine((float(r) + 0.5f) / 16.0f, radical(r), f);
        Hit<float> h = trace<float>(C, o, d, C.P->ground[3], false, key + r + 7000u);
        if (h.tri != NONE && h.back) back += 1.0f;
    }
    return back / 16.0f > bitsf(C.P->atlas[3]);
}

// the sun disc's direction for spiral sample k of g*g (trace.wgsl:219-221, :314-316)
inline V3<float> sun_disc(const Ctx &C, const Frame &sf, uint32_t k, uint32_t gg) {
    V3<float> sun = f3(C.P->sun_dir);
    float a = float(k) * 2.399963f;
    float r = C.P->sun_dir[3] * std::sqrt((float(k) + 0.5f) / float(gg));
    float s, c;
    sincos32(a, &s, &c);
    return normalize((sun + sf.t * c * r) + sf.b * s * r);
}

// trace.wgsl:170-243
void direct_item(const Ctx &C, const lb_texel &tx, uint32_t index, float *out) {
    V3<float> n = f3(tx.normal);
    uint32_t key = index * 7919u;
    uint32_t g = C.P->counts[0];
    V3<float> sun = f3(C.P->sun_dir);
    Frame sf = frame(sun);
    float soft = 0.0f;
    uint32_t hard = 0u;
    V3<float> lift = n * C.P->reach[2];
    V3<float> pos = f3(tx.pos), dx = f3(tx.dx), dy = f3(tx.dy);
    V3<float> at = pos;
    uint32_t pick = 0u;
    float span = 1.0f;
    if (inside(C, at + lift, n, key)) {
        for (uint32_t q = 1u; q < 9u; q++) {
            float cx, cy;
            offset(q, &cx, &cy);
            V3<float> p = (pos + dx * cx) + dy * cy;
            if (!inside(C, p + lift, n, key + q * 31u)) {
                at = p;
                pick = q;
                span = 0.4f;
                break;
            }
        }
        if (pick == 0u) {
            V3<float> p = pos + n * PUSH;
            if (!inside(C, p + lift, n, key + 331u)) {
                at = p;
                pick = 9u;
                span = 0.4f;
            }
        }
    }
    if (dot(sun, n) > 0.0f) {
        uint32_t gg = g * g;
        for (uint32_t s = 0u; s < gg; s++) {
            float cx = ((float(s % g) + 0.5f) / float(g) - 0.5f) * span;
            float cy = ((float(s / g) + 0.5f) / float(g) - 0.5f) * span;
            V3<float> o = ((at + dx * cx) + dy * cy) + lift;
            if (trace<float>(C, o, sun, FAR, true, key + s).tri == NONE) hard |= 1u << (s & 31u);  // WGSL: the shift is taken modulo 32
            uint32_t k = (s + uint32_t(rnd(key, 17u, C.seed) * float(gg))) % gg;
            V3<float> d = sun_disc(C, sf, k, gg);
            if (trace<float>(C, o, d, FAR, true, key + s + 1000u).tri == NONE) soft += 1.0f;
        }
        soft /= float(gg);
    }
    Frame f = frame(n);
    V3<float> o = at + lift;
    uint32_t rays = C.P->counts[1];
    float s1 = rnd(key, 3u, C.seed), s2 = rnd(key, 5u, C.seed);
    float occ = 0.0f, back = 0.0f;
    for (uint32_t r = 0u; r < rays; r++) {
        V3<float> d = cosine(fract((float(r) + 0.5f) / float(rays) + s1), fract(radical(r) + s2), f);
        Hit<float> h = trace<float>(C, o, d, C.P->reach[0], false, key + r + 2000u);
        if (h.tri == NONE) continue;
        float k = h.t / C.P->reach[0];
        occ += 1.0f - k * k;
        if (h.back && h.t < C.P->ground[3]) back += 1.0f;
    }
    out[0] = soft;
    out[1] = bitsf(hard | (pick << 24u));
    out[2] = occ / float(rays);
    out[3] = back / float(rays);
}

// trace.wgsl:245-270
void gather_item(const Ctx &C, const lb_texel &tx, uint32_t index, float *out) {
    V3<float> n = f3(tx.normal);
    Frame f = frame(n);
    uint32_t key = index * 7919u;
    uint32_t rays = C.P->counts[2];
    float s1 = rnd(key, 11u, C.seed), s2 = rnd(key, 13u, C.seed);
    V3<float> sum = mk(0.f, 0.f, 0.f);
    float back = 0.0f;
    V3<float> pos = f3(tx.pos), dx = f3(tx.dx), dy = f3(tx.dy);
    for (uint32_t r = 0u; r < rays; r++) {
        float jx = rnd(key + r, 19u, C.seed) - 0.5f, jy = rnd(key + r, 23u, C.seed) - 0.5f;
        V3<float> o = ((pos + dx * jx) + dy * jy) + n * C.P->reach[2];
        V3<float> d = cosine(fract((float(r) + 0.5f) / float(rays) + s1), fract(radical(r) + s2), f);
        Hit<float> h = trace<float>(C, o, d, C.P->reach[1], false, key + r + 4000u);
        if (h.tri == NONE) { sum = sum + sky(C, d); continue; }
        if (h.back) { back += 1.0f; continue; }
        sum = sum + bounced(C, o, d, h);
    }
    V3<float> e = sum * PI;
    out[0] = e.x / float(rays);
    out[1] = e.y / float(rays);
    out[2] = e.z / float(rays);
    out[3] = back / float(rays);
}

// trace.wgsl:272-324
void volume_item(const Ctx &C, const lb_texel &probe, float *out) {
    V3<float> o = f3(probe.pos);
    uint32_t key = fbits(probe.normal[3]) * 7919u + 77u;
    uint32_t rays = C.P->counts[2];
    float s1 = rnd(key, 29u, C.seed), s2 = rnd(key, 31u, C.seed);
    V3<float> l0 = mk(0.f, 0.f, 0.f), l1x = l0, l1y = l0, l1z = l0;
    float back = 0.0f;
    for (uint32_t r = 0u; r < rays; r++) {
        float u = fract((float(r) + 0.5f) / float(rays) + s1);
        float v = fract(radical(r) + s2);
        float z = 1.0f - 2.0f * u;
        float rr = std::sqrt(vmax(0.0f, 1.0f - z * z));
        float a = v * 2.0f * PI;
        float sa, ca;
        sincos32(a, &sa, &ca);
        V3<float> d = mk(rr * ca, z, rr * sa);
        Hit<float> h = trace<float>(C, o, d, C.P->reach[1], false, key + r);
        V3<float> l = sky(C, d);
        if (h.tri != NONE) {
            if (h.back) back += 1.0f;
            l = h.back ? mk(0.f, 0.f, 0.f) : bounced(C, o, d, h);
        }
        l0 = l0 + l * 0.282095f;
        l1x = l1x + (l * 0.488603f) * d.x;
        l1y = l1y + (l * 0.488603f) * d.y;
        l1z = l1z + (l * 0.488603f) * d.z;
    }
    float w = 4.0f * PI / float(rays);
    uint32_t g = C.P->counts[0], gg = g * g;
    Frame sf = frame(f3(C.P->sun_dir));
    float sun = 0.0f;
    for (uint32_t s = 0u; s < gg; s++) {
        V3<float> d = sun_disc(C, sf, s, gg);
        if (trace<float>(C, o, d, FAR, true, key + s + 9000u).tri == NONE) sun += 1.0f;
    }
    V3<float> a0 = l0 * w, ax = l1x * w, ay = l1y * w, az = l1z * w;
    float rec[16] = {a0.x, a0.y, a0.z, sun / float(gg), ax.x, ax.y, ax.z, back / float(rays),
                     ay.x, ay.y, ay.z, 0.0f, az.x, az.y, az.z, 0.0f};
    std::memcpy(out, rec, sizeof rec);
}

Ctx make_ctx(const lb_node *nodes, size_t n_nodes, const lb_tri *tris, size_t n_tris, const float *mats,
             size_t n_mats, const float *charts, size_t n_charts, const lb_params *P, const float *light,
             size_t n_light) {
    Ctx C;
    C.nodes = nodes;
    C.n_nodes = n_nodes;
    C.tris = tris;
    C.n_tris = n_tris;
    C.mats = mats;
    C.n_mats = n_mats;
    C.charts = charts;
    C.n_charts = n_charts;
    C.light = light;
    C.n_light = n_light;
    C.P = P;
    C.seed = fbits(P->reach[3]);
    C.cnt = nullptr;
    return C;
}

}  // namespace

extern "C" {

int or_run(int pass, const lb_node *nodes, size_t n_nodes, const lb_tri *tris, size_t n_tris,
           const float *materials, size_t n_materials, const float *charts, size_t n_charts,
           const lb_params *params, const lb_texel *items, size_t n, const float *light,
           size_t n_light, float *out, int threads, or_counters *counters) {
    return or_run_ex(pass, nodes, n_nodes, tris, n_tris, materials, n_materials, charts, n_charts, params, items, n,
                     light, n_light, out, threads, counters, nullptr);
}

int or_run_ex(int pass, const lb_node *nodes, size_t n_nodes, const lb_tri *tris, size_t n_tris,
              const float *materials, size_t n_materials, const float *charts, size_t n_charts,
              const lb_params *params, const lb_texel *items, size_t n, const float *light,
              size_t n_light, float *out, int threads, or_counters *counters, const float *verts) {
    if (pass < 0 || pass > 2 || !params || (n && (!items || !out)) || !nodes || n_nodes == 0) return LB_EINVAL;
    Ctx base = make_ctx(nodes, n_nodes, tris, n_tris, materials, n_materials, charts, n_charts, params, light, n_light);
    base.verts = verts;
    size_t width = pass == LB_PASS_VOLUME ? 4 : 1;
    if (counters) std::memset(counters, 0, sizeof *counters);
#pragma omp parallel num_threads(threads > 0 ? threads : omp_get_max_threads())
    {
        or_counters local{};
        Ctx C = base;
        C.cnt = counters ? &local : nullptr;
#pragma omp for schedule(dynamic, 16)
        for (long long i = 0; i < (long long)n; i++) {
            float *o = out + size_t(i) * width * 4;
            // the shader keys item i of a dispatch by P.atlas.z + i (trace.wgsl:172-173): the item's index in the
            // whole list (Gpu::run sets atlas.z to each batch's first, gpu/mod.rs:160-166)
            uint32_t index = params->atlas[2] + uint32_t(i);
            if (pass == LB_PASS_DIRECT) direct_item(C, items[i], index, o);
            else if (pass == LB_PASS_GATHER) gather_item(C, items[i], index, o);
            else volume_item(C, items[i], o);
        }
        if (counters) {
#pragma omp critical
            {
                counters->rays += local.rays;
                counters->nodes += local.nodes;
                counters->tris += local.tris;
                counters->mats += local.mats;
                counters->overflows += local.overflows;
            }
        }
    }
    return LB_OK;
}

int or_trace(int precision, const lb_node *nodes, size_t n_nodes, const lb_tri *tris, size_t n_tris,
             const float *materials, size_t n_materials, const lb_params *params, const float o[3],
             const float d[3], float tmax, int any, uint32_t ray, double *t, uint32_t *tri, int *back) {
    return or_trace_ex(precision, nodes, n_nodes, tris, n_tris, materials, n_materials, params, o, d, tmax, any, ray,
                       t, tri, back, nullptr);
}

int or_trace_ex(int precision, const lb_node *nodes, size_t n_nodes, const lb_tri *tris, size_t n_tris,
                const float *materials, size_t n_materials, const lb_params *params, const float o[3],
                const float d[3], float tmax, int any, uint32_t ray, double *t, uint32_t *tri, int *back,
                const float *verts) {
    Ctx C = make_ctx(nodes, n_nodes, tris, n_tris, materials, n_materials, nullptr, 0, params, nullptr, 0);
    C.verts = verts;
    if (precision == 64) {
        Hit<double> h = trace<double>(C, mk<double>(o[0], o[1], o[2]), mk<double>(d[0], d[1], d[2]), double(tmax), any != 0, ray);
        *t = h.t; *tri = h.tri; *back = h.back;
    } else {
        Hit<float> h = trace<float>(C, mk(o[0], o[1], o[2]), mk(d[0], d[1], d[2]), tmax, any != 0, ray);
        *t = h.t; *tri = h.tri; *back = h.back;
    }
    return LB_OK;
}

int or_trace_rays(int precision, const lb_node *nodes, size_t n_nodes, const lb_tri *tris, size_t n_tris,
                  const float *materials, size_t n_materials, const lb_params *params, const float *rays, size_t n,
                  int any, const float *verts, double *t, uint32_t *tri, int *back, int threads) {
    Ctx base = make_ctx(nodes, n_nodes, tris, n_tris, materials, n_materials, nullptr, 0, params, nullptr, 0);
    base.verts = verts;
#pragma omp parallel for schedule(dynamic, 256) num_threads(threads > 0 ? threads : omp_get_max_threads())
    for (long long i = 0; i < (long long)n; i++) {
        const float *r = rays + size_t(i) * 8;
        uint32_t key;
        std::memcpy(&key, r + 7, 4);
        if (precision == 64) {
            Hit<double> h = trace<double>(base, mk<double>(r[0], r[1], r[2]), mk<double>(r[4], r[5], r[6]),
                                          double(r[3]), any != 0, key);
            t[i] = h.t; tri[i] = h.tri; back[i] = h.back;
        } else {
            Hit<float> h = trace<float>(base, mk(r[0], r[1], r[2]), mk(r[4], r[5], r[6]), r[3], any != 0, key);
            t[i] = h.t; tri[i] = h.tri; back[i] = h.back;
        }
    }
    return LB_OK;
}

int or_rays_ambiguous(const lb_node *nodes, size_t n_nodes, const lb_tri *tris, size_t n_tris,
                      const float *materials, size_t n_materials, const lb_params *params, const float *rays,
                      size_t n, double eps, int *out, int threads) {
#pragma omp parallel for schedule(dynamic, 256) num_threads(threads > 0 ? threads : omp_get_max_threads())
    for (long long i = 0; i < (long long)n; i++) {
        const float *r = rays + size_t(i) * 8;
        uint32_t key;
        std::memcpy(&key, r + 7, 4);
        out[i] = or_ray_ambiguous(nodes, n_nodes, tris, n_tris, materials, n_materials, params, r, r + 4, r[3], key,
                                  eps);
    }
    return LB_OK;
}

int or_ray_ambiguous(const lb_node *nodes, size_t n_nodes, const lb_tri *tris, size_t n_tris,
                     const float *materials, size_t n_materials, const lb_params *params,
                     const float of[3], const float df[3], float tmax, uint32_t ray, double eps) {
    Ctx C = make_ctx(nodes, n_nodes, tris, n_tris, materials, n_materials, nullptr, 0, params, nullptr, 0);
    V3<double> o = mk<double>(of[0], of[1], of[2]), d = mk<double>(df[0], df[1], df[2]);
    // every leaf whose box the ray passes within a margin of, every triangle in it
    double len = std::sqrt(dot(d, d));
    double margin = 1e-3;
    std::vector<uint32_t> st;
    st.push_back(0);
    while (!st.empty()) {
        uint32_t n = st.back();
        st.pop_back();
        const lb_node &node = nodes[n];
        if (node.count == 0) {
            if (size_t(node.first) + 1 >= n_nodes) continue;
            for (uint32_t c = node.first; c <= node.first + 1; c++) {
                const lb_node &b = nodes[c];
                double lo = 0, hi = double(tmax) * (1 + eps) + margin;
                bool ok = true;
                for (int a = 0; a < 3 && ok; a++) {
                    double oa = a == 0 ? o.x : a == 1 ? o.y : o.z, da = a == 0 ? d.x : a == 1 ? d.y : d.z;
                    double mn = double(b.min[a]) - margin, mx = double(b.max[a]) + margin;
                    if (std::fabs(da) < 1e-300) { ok = oa >= mn && oa <= mx; continue; }
                    double t1 = (mn - oa) / da, t2 = (mx - oa) / da;
                    if (t1 > t2) std::swap(t1, t2);
                    lo = std::max(lo, t1);
                    hi = std::min(hi, t2);
                    ok = lo <= hi;
                }
                if (ok) st.push_back(c);
            }
            continue;
        }
        for (uint32_t i = node.first; i < node.first + node.count; i++) {
            const lb_tri &tr = tris[i];
            V3<double> e1 = cvt<double>(f3(tr.e1)), e2 = cvt<double>(f3(tr.e2)), v0 = cvt<double>(f3(tr.v0));
            V3<double> p = cross(d, e2);
            double det = dot(e1, p);
            double scale = std::sqrt(dot(e1, e1)) * std::sqrt(dot(e2, e2)) * len;
            if (std::fabs(det) <= 1e-12 * (1 + eps) * 4 || std::fabs(det) < scale * 1e-7) {
                // grazing: decided by rounding on either side when the ray passes near the triangle
                V3<double> s = o - v0;
                double dist = std::fabs(dot(s, normalize(cross(e1, e2))));
                if (dist < 1e-4 * (1 + len)) return 1;
                continue;
            }
            double id = 1.0 / det;
            V3<double> s = o - v0;
            double u = dot(s, p) * id;
            V3<double> q = cross(s, e1);
            double v = dot(d, q) * id;
            double w = 1.0 - u - v;
            double t = dot(e2, q) * id;
            double m = std::min(u, std::min(v, w));
            bool in_t = t > 1e-4 * (1 - eps) - 1e-9 && t < double(tmax) * (1 + eps);
            if (!in_t) continue;
            bool near_t = std::fabs(t - 1e-4) <= 1e-4 * eps + 1e-9 || std::fabs(t - double(tmax)) <= double(tmax) * eps;
            if (m >= -eps && (m <= eps || near_t) && stops(C, i, ray)) return 1;
        }
    }
    return 0;
}

size_t or_item_rays(int pass, const lb_params *P, const lb_texel *item, size_t index, uint32_t pick,
                    float *o, float *d, float *tmax, int *any, uint32_t *key, int *kind, size_t cap) {
    Ctx C = make_ctx(nullptr, 0, nullptr, 0, nullptr, 0, nullptr, 0, P, nullptr, 0);
    size_t k = 0;
    auto put = [&](V3<float> oo, V3<float> dd, float tm, int an, uint32_t ky, int kd) {
        if (k < cap) {
            o[k * 3] = oo.x; o[k * 3 + 1] = oo.y; o[k * 3 + 2] = oo.z;
            d[k * 3] = dd.x; d[k * 3 + 1] = dd.y; d[k * 3 + 2] = dd.z;
            tmax[k] = tm; any[k] = an; key[k] = ky; kind[k] = kd;
        }
        k++;
    };
    const lb_texel &tx = *item;
    if (pass == LB_PASS_DIRECT) {
        V3<float> n = f3(tx.normal), sun = f3(P->sun_dir), pos = f3(tx.pos), dx = f3(tx.dx), dy = f3(tx.dy);
        uint32_t kk = uint32_t(index) * 7919u, g = P->counts[0], gg = g * g;
        V3<float> lift = n * P->reach[2], at = pos;
        float span = 1.0f;
        uint32_t ikey = kk;
        if (pick >= 1 && pick <= 8) {
            float cx, cy;
            offset(pick, &cx, &cy);
            at = (pos + dx * cx) + dy * cy;
            span = 0.4f;
            ikey = kk + pick * 31u;
        } else if (pick == 9) {
            at = pos + n * PUSH;
            span = 0.4f;
            ikey = kk + 331u;
        }
        Frame f = frame(n);
        for (uint32_t r = 0; r < 16u; r++)
            put(at + lift, cosine((float(r) + 0.5f) / 16.0f, radical(r), f), P->ground[3], 0, ikey + r + 7000u, 0);
        Frame sf = frame(sun);
        if (dot(sun, n) > 0.0f) {
            for (uint32_t s = 0; s < gg; s++) {
                float cx = ((float(s % g) + 0.5f) / float(g) - 0.5f) * span;
                float cy = ((float(s / g) + 0.5f) / float(g) - 0.5f) * span;
                V3<float> oo = ((at + dx * cx) + dy * cy) + lift;
                put(oo, sun, FAR, 1, kk + s, 1);
                uint32_t kd = (s + uint32_t(rnd(kk, 17u, C.seed) * float(gg))) % gg;
                put(oo, sun_disc(C, sf, kd, gg), FAR, 1, kk + s + 1000u, 2);
            }
        }
        uint32_t rays = P->counts[1];
        float s1 = rnd(kk, 3u, C.seed), s2 = rnd(kk, 5u, C.seed);
        for (uint32_t r = 0; r < rays; r++)
            put(at + lift, cosine(fract((float(r) + 0.5f) / float(rays) + s1), fract(radical(r) + s2), f), P->reach[0], 0, kk + r + 2000u, 3);
    } else if (pass == LB_PASS_GATHER) {
        V3<float> n = f3(tx.normal), pos = f3(tx.pos), dx = f3(tx.dx), dy = f3(tx.dy);
        Frame f = frame(n);
        uint32_t kk = uint32_t(index) * 7919u, rays = P->counts[2];
        float s1 = rnd(kk, 11u, C.seed), s2 = rnd(kk, 13u, C.seed);
        for (uint32_t r = 0; r < rays; r++) {
            float jx = rnd(kk + r, 19u, C.seed) - 0.5f, jy = rnd(kk + r, 23u, C.seed) - 0.5f;
            V3<float> oo = ((pos + dx * jx) + dy * jy) + n * P->reach[2];
            put(oo, cosine(fract((float(r) + 0.5f) / float(rays) + s1), fract(radical(r) + s2), f), P->reach[1], 0, kk + r + 4000u, 4);
        }
    } else {
        V3<float> o0 = f3(tx.pos);
        uint32_t kk = fbits(tx.normal[3]) * 7919u + 77u, rays = P->counts[2];
        float s1 = rnd(kk, 29u, C.seed), s2 = rnd(kk, 31u, C.seed);
        for (uint32_t r = 0; r < rays; r++) {
            float u = fract((float(r) + 0.5f) / float(rays) + s1), v = fract(radical(r) + s2);
            float z = 1.0f - 2.0f * u, rr = std::sqrt(vmax(0.0f, 1.0f - z * z)), a = v * 2.0f * PI, sa, ca;
            sincos32(a, &sa, &ca);
            put(o0, mk(rr * ca, z, rr * sa), P->reach[1], 0, kk + r, 5);
        }
        uint32_t g = P->counts[0], gg = g * g;
        Frame sf = frame(f3(P->sun_dir));
        for (uint32_t s = 0; s < gg; s++) put(o0, sun_disc(C, sf, s, gg), FAR, 1, kk + s + 9000u, 6);
    }
    return k;
}

// The outcome of every gather ray of every item (trace.wgsl:245-270): kind (0 sky, 1 back face, 2 a
// surface), for the sky the ray's direction y, for a surface its material and the atlas texel its chart
// maps the hit to (0xffffffff: none, the fallback). Records are [item][ray], 4 words each:
// kind, material, atlas index, bits of d.y.
int or_gather_records(const lb_node *nodes, size_t n_nodes, const lb_tri *tris, size_t n_tris, const float *materials,
                      size_t n_materials, const float *charts, size_t n_charts, const lb_params *P,
                      const lb_texel *items, size_t n, size_t n_light, uint32_t *rec, int threads) {
    Ctx base = make_ctx(nodes, n_nodes, tris, n_tris, materials, n_materials, charts, n_charts, P, nullptr, 0);
    uint32_t rays = P->counts[2];
#pragma omp parallel for schedule(dynamic, 16) num_threads(threads > 0 ? threads : omp_get_max_threads())
    for (long long k = 0; k < (long long)n; k++) {
        const Ctx &C = base;
        const lb_texel &tx = items[k];
        V3<float> nrm = f3(tx.normal), pos = f3(tx.pos), dx = f3(tx.dx), dy = f3(tx.dy);
        Frame f = frame(nrm);
        uint32_t key = (P->atlas[2] + uint32_t(k)) * 7919u;
        float s1 = rnd(key, 11u, C.seed), s2 = rnd(key, 13u, C.seed);
        for (uint32_t r = 0; r < rays; r++) {
            float jx = rnd(key + r, 19u, C.seed) - 0.5f, jy = rnd(key + r, 23u, C.seed) - 0.5f;
            V3<float> o = ((pos + dx * jx) + dy * jy) + nrm * C.P->reach[2];
            V3<float> d = cosine(fract((float(r) + 0.5f) / float(rays) + s1), fract(radical(r) + s2), f);
            Hit<float> h = trace<float>(C, o, d, C.P->reach[1], false, key + r + 4000u);
            uint32_t *w = rec + (size_t(k) * rays + r) * 4;
            w[0] = 0;
            w[1] = 0;
            w[2] = NONE;
            w[3] = fbits(d.y);
            if (h.tri == NONE) continue;
            if (h.back) {
                w[0] = 1;
                continue;
            }
            w[0] = 2;
            const lb_tri &tr = C.tris[h.tri];
            w[1] = fbits(tr.v0[3]);
            uint32_t c = fbits(tr.e1[3]);
            if (c != NONE && c < C.n_charts) {
                V3<float> p = o + d * h.t;
                const float *r0 = C.charts + size_t(c) * 8, *r1 = r0 + 4;
                float x = r0[0] * p.x + r0[1] * p.y + r0[2] * p.z + r0[3] * 1.0f;
                float y = r1[0] * p.x + r1[1] * p.y + r1[2] * p.z + r1[3] * 1.0f;
                int aw = int(C.P->atlas[0]), ah = int(C.P->atlas[1]);
                int ix = std::min(std::max(int(std::floor(x)), 0), aw - 1);
                int iy = std::min(std::max(int(std::floor(y)), 0), ah - 1);
                size_t li = size_t(uint32_t(iy)) * C.P->atlas[0] + uint32_t(ix);
                if (li < n_light) w[2] = uint32_t(li);
            }
        }
    }
    return LB_OK;
}

uint32_t or_pcg(uint32_t v) { return pcg(v); }
float or_rand(uint32_t a, uint32_t b, uint32_t seed_bits) { return rnd(a, b, seed_bits); }
float or_radical(uint32_t i) { return radical(i); }
void or_sincos(float a, float *s, float *c) { sincos32(a, s, c); }

}  // extern "C"
