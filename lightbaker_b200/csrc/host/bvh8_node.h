// One node of the 8-wide collapse (bvh8.h has the node format), shared by the host builder (bvh8.cpp)
// and the device builder (bvh8_build.cu) so that both emit the same bytes. A node to emit is an Item:
// either a BVH2 inner node opened (largest area first) until eight children, or a run of triangles of
// the BVH2 triangle array cut into slots of at most SLOT_TRIS. Everything here is plain float/double
// arithmetic with no contraction (the host compiles with -ffp-contract=off, the device with
// -fmad=false), floor/ceil/frexp/ldexpf (exact), and IEEE double division, so the host and the device
// agree bit for bit.
#pragma once
#include <cfloat>
#include <cmath>
#include <cstdint>

#include "../../../include/lightbaker.h"

#ifdef __CUDACC__
#define LB8_HD __host__ __device__ __forceinline__
#else
#define LB8_HD inline
#endif

namespace lb8 {

constexpr uint32_t SLOT_TRIS = 4;   // triangles a leaf slot holds
constexpr uint32_t NODE_TRIS = 32;  // triangles a node's leaf slots hold together (5-bit offsets)
constexpr uint32_t WORDS = 20;      // 32-bit words a node

// a child to place in a slot: a BVH2 inner node, or a run of triangles [first, first + count)
struct Ref {
    uint32_t leaf, node, first, count;
    float mn[3], mx[3];
};

// a node to emit: run == 0 opens BVH2 inner node `node`; run == 1 cuts [first, first + count) with box mn..mx
struct Item {
    uint32_t run, node, first, count;
    float mn[3], mx[3];
};

LB8_HD float area(const Ref &b) {
    float d[3];
    for (int a = 0; a < 3; a++) {
        float e = b.mx[a] - b.mn[a];
        d[a] = e > 0.0f ? e : 0.0f;
    }
    return d[0] * d[1] + d[1] * d[2] + d[2] * d[0];
}

LB8_HD Ref ref_of(const lb_node *n2, uint32_t i) {
    Ref r{};
    for (int a = 0; a < 3; a++) {
        r.mn[a] = n2[i].min[a];
        r.mx[a] = n2[i].max[a];
    }
    if (n2[i].count > 0) {
        r.leaf = 1;
        r.first = n2[i].first;
        r.count = n2[i].count;
    } else {
        r.node = i;
    }
    return r;
}

LB8_HD bool expandable(const lb_node *n2, size_t nn2, const Ref &r) {
    return !r.leaf && size_t(n2[r.node].first) + 1 < nn2;
}

// the children of an inner BVH2 node, opened (largest area first, the first at equal areas) until eight
LB8_HD int open(const lb_node *n2, size_t nn2, uint32_t i, Ref out[8]) {
    if (size_t(n2[i].first) + 1 >= nn2) return 0;  // the reference's empty one-node BVH
    int n = 2;
    out[0] = ref_of(n2, n2[i].first);
    out[1] = ref_of(n2, n2[i].first + 1);
    while (n < 8) {
        int best = -1;
        float ba = -1.0f;
        for (int k = 0; k < n; k++)
            if (expandable(n2, nn2, out[k]) && area(out[k]) > ba) {
                ba = area(out[k]);
                best = k;
            }
        if (best < 0) break;
        const uint32_t c = out[best].node;
        for (int k = n; k > best + 1; k--) out[k] = out[k - 1];
        out[best] = ref_of(n2, n2[c].first);
        out[best + 1] = ref_of(n2, n2[c].first + 1);
        n++;
    }
    return n;
}

// a run of triangles: runs of at most SLOT_TRIS, or (more than 32 triangles) eight runs cut again below
LB8_HD int split_run(const Ref &r, Ref out[8]) {
    const uint32_t chunks = (r.count + SLOT_TRIS - 1) / SLOT_TRIS;
    const uint32_t each = chunks <= 8 ? SLOT_TRIS : (r.count + 7) / 8;
    int n = 0;
    for (uint32_t k = 0; k < 8 && k * each < r.count; k++) {
        out[n] = r;
        out[n].first = r.first + k * each;
        out[n].count = r.count - k * each < each ? r.count - k * each : each;
        n++;
    }
    return n;
}

LB8_HD Item root_item(const lb_node *n2) {
    Item it{};
    if (n2[0].count > 0) {
        const Ref r = ref_of(n2, 0);
        it.run = 1;
        it.first = r.first;
        it.count = r.count;
        for (int a = 0; a < 3; a++) {
            it.mn[a] = r.mn[a];
            it.mx[a] = r.mx[a];
        }
    }
    return it;
}

LB8_HD int refs_of(const lb_node *n2, size_t nn2, const Item &it, Ref out[8]) {
    if (!it.run) return open(n2, nn2, it.node, out);
    Ref r{};
    r.leaf = 1;
    r.first = it.first;
    r.count = it.count;
    for (int a = 0; a < 3; a++) {
        r.mn[a] = it.mn[a];
        r.mx[a] = it.mx[a];
    }
    return split_run(r, out);
}

// the node a slot becomes when it cannot be a leaf slot of this node
LB8_HD Item item_of(const Ref &r) {
    Item it{};
    it.run = r.leaf;
    it.node = r.node;
    it.first = r.first;
    it.count = r.count;
    for (int a = 0; a < 3; a++) {
        it.mn[a] = r.mn[a];
        it.mx[a] = r.mx[a];
    }
    return it;
}

// slot s is an inner child: a BVH2 inner node, a run over SLOT_TRIS, or one past the node's 32 triangles
LB8_HD uint32_t inner_mask(const Ref *refs, int n, uint32_t *tris) {
    uint32_t mask = 0, off = 0;
    for (int s = 0; s < n; s++) {
        if (!refs[s].leaf || refs[s].count > SLOT_TRIS || off + refs[s].count > NODE_TRIS) mask |= 1u << s;
        else off += refs[s].count;
    }
    *tris = off;
    return mask;
}

// ceil(log2(y)) for y > 0, exactly: y = m 2^x with m in [0.5, 1)
LB8_HD int ceil_log2(double y) {
    int x;
    const double m = frexp(y, &x);
    return m > 0.5 ? x : x - 1;
}

// The node's words: origin, exponents and inner mask, first inner child, first triangle, slot bytes and
// the child boxes quantized to 8 bits an axis, each dequantized box (p + q 2^e in float) holding the
// child's exact box. False when no exponent up to 2^120 fits.
LB8_HD bool node_words(const Ref *refs, int n, uint32_t child_base, uint32_t tri_base, uint32_t w[WORDS]) {
    uint32_t tris;
    const uint32_t imask = inner_mask(refs, n, &tris);
    uint8_t meta[8];
    uint32_t off = 0;
    for (int s = 0; s < 8; s++) {
        meta[s] = 0xff;
        if (s < n && !((imask >> s) & 1u)) {
            meta[s] = uint8_t(off | ((refs[s].count - 1) << 5));
            off += refs[s].count;
        }
    }
    float amn[3], amx[3];
    for (int a = 0; a < 3; a++) {
        amn[a] = FLT_MAX;
        amx[a] = -FLT_MAX;
        for (int s = 0; s < n; s++) {
            amn[a] = refs[s].mn[a] < amn[a] ? refs[s].mn[a] : amn[a];
            amx[a] = amx[a] < refs[s].mx[a] ? refs[s].mx[a] : amx[a];
        }
        if (n == 0) amn[a] = amx[a] = 0.0f;
    }
    uint8_t q[6][8];
    for (int k = 0; k < 6; k++)
        for (int s = 0; s < 8; s++) q[k][s] = 0;
    uint32_t eb[3];
    for (int a = 0; a < 3; a++) {
        const float p = amn[a];
        const double extent = double(amx[a]) - double(p);
        int e = extent > 0 ? ceil_log2(extent / 255.0) : -100;
        e = e > -100 ? e : -100;
        for (;; e++) {
            const float scale = ldexpf(1.0f, e);
            bool ok = true;
            for (int s = 0; s < n && ok; s++) {
                double lo = floor((double(refs[s].mn[a]) - p) / scale);
                double hi = ceil((double(refs[s].mx[a]) - p) / scale);
                lo = lo < 0.0 ? 0.0 : lo;
                while (lo > 0 && p + float(lo) * scale > refs[s].mn[a]) lo -= 1;
                while (hi <= 255 && p + float(hi) * scale < refs[s].mx[a]) hi += 1;
                if (hi > 255 || p + float(lo) * scale > refs[s].mn[a]) {
                    ok = false;
                    break;
                }
                q[a][s] = uint8_t(lo);
                q[3 + a][s] = uint8_t(hi);
            }
            if (ok) break;
            if (e > 120) return false;
        }
        eb[a] = uint32_t(e + 127);
    }
    for (int s = n; s < 8; s++)  // empty slots: lo 1 > hi 0, a box no ray enters
        for (int a = 0; a < 3; a++) {
            q[a][s] = 1;
            q[3 + a][s] = 0;
        }
    for (int a = 0; a < 3; a++) {
        union {
            float f;
            uint32_t u;
        } b;
        b.f = amn[a];
        w[a] = b.u;
    }
    w[3] = eb[0] | (eb[1] << 8) | (eb[2] << 16) | (imask << 24);
    w[4] = child_base;
    w[5] = tri_base;
    w[6] = uint32_t(meta[0]) | uint32_t(meta[1]) << 8 | uint32_t(meta[2]) << 16 | uint32_t(meta[3]) << 24;
    w[7] = uint32_t(meta[4]) | uint32_t(meta[5]) << 8 | uint32_t(meta[6]) << 16 | uint32_t(meta[7]) << 24;
    for (int k = 0; k < 12; k++) {
        const int b0 = 4 * k;  // byte b of q (row-major [6][8]) is q[b / 8][b % 8]
        w[8 + k] = uint32_t(q[b0 / 8][b0 % 8]) | uint32_t(q[(b0 + 1) / 8][(b0 + 1) % 8]) << 8 |
                   uint32_t(q[(b0 + 2) / 8][(b0 + 2) % 8]) << 16 | uint32_t(q[(b0 + 3) / 8][(b0 + 3) % 8]) << 24;
    }
    return true;
}

}  // namespace lb8
