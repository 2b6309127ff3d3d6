// ORACLE — test infrastructure only (see oracle.h). The reference's BVH build restated from its Rust
// source (crates/lightbaker/src/bvh.rs:50-162: Bvh::build, bounds, area, best_split, partition), serially and
// in glam's operation order, sharing no code with the product's builder. The triangle order it produces is
// what the shader's opacity coin is keyed by (trace.wgsl:69-72), so the product's BVH must equal it byte for
// byte.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <utility>
#include <vector>

#include "oracle.h"

namespace {

struct V3 {
    float x, y, z;
    float operator[](int a) const { return a == 0 ? x : (a == 1 ? y : z); }
};
inline V3 vmin(V3 a, V3 b) { return {std::fmin(a.x, b.x), std::fmin(a.y, b.y), std::fmin(a.z, b.z)}; }
inline V3 vmax(V3 a, V3 b) { return {std::fmax(a.x, b.x), std::fmax(a.y, b.y), std::fmax(a.z, b.z)}; }
inline V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 cross(V3 a, V3 b) { return {a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y}; }
inline float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline float from_bits(uint32_t b) {
    float v;
    std::memcpy(&v, &b, 4);
    return v;
}

struct Prim {  // bvh.rs:40-46
    V3 min, max, centre;
    lb_tri tri;
};

const size_t BINS = 16, LEAF = 4;

// bvh.rs:108-110
struct Box {
    V3 lo{INFINITY, INFINITY, INFINITY}, hi{-INFINITY, -INFINITY, -INFINITY};
    void add(V3 a, V3 b) {
        lo = vmin(lo, a);
        hi = vmax(hi, b);
    }
};
// bvh.rs:112-115
float area(V3 mn, V3 mx) {
    V3 d = vmax(sub(mx, mn), V3{0.0f, 0.0f, 0.0f});
    return d.x * d.y + d.y * d.z + d.z * d.x;
}
// Rust's `as usize` from f32: truncation, saturating at 0 (and NaN to 0)
size_t to_usize(float v) { return v > 0.0f ? size_t(v) : 0; }

// bvh.rs:118-151
bool best_split(const Prim *p, size_t n, int &axis_out, float &at_out) {
    Box c, b;
    for (size_t i = 0; i < n; i++) {
        c.add(p[i].centre, p[i].centre);
        b.add(p[i].min, p[i].max);
    }
    float leaf_cost = float(n) * area(b.lo, b.hi);
    bool have = false;
    float best_cost = 0.0f, best_at = 0.0f;
    int best_axis = 0;
    for (int axis = 0; axis < 3; axis++) {
        float extent = c.hi[axis] - c.lo[axis];
        if (extent < 1e-6f) continue;
        Box bins[BINS];
        uint32_t cnt[BINS] = {0};
        for (size_t i = 0; i < n; i++) {
            size_t k = to_usize((p[i].centre[axis] - c.lo[axis]) / extent * float(BINS));
            if (k > BINS - 1) k = BINS - 1;
            bins[k].add(p[i].min, p[i].max);
            cnt[k]++;
        }
        for (size_t s = 1; s < BINS; s++) {
            uint32_t ln = 0, rn = 0;
            Box l, r;
            for (size_t k = 0; k < s; k++) {
                ln += cnt[k];
                l.add(bins[k].lo, bins[k].hi);
            }
            for (size_t k = s; k < BINS; k++) {
                rn += cnt[k];
                r.add(bins[k].lo, bins[k].hi);
            }
            if (ln == 0 || rn == 0) continue;
            float cost = float(ln) * area(l.lo, l.hi) + float(rn) * area(r.lo, r.hi);
            if (!have || cost < best_cost) {
                have = true;
                best_cost = cost;
                best_axis = axis;
                best_at = c.lo[axis] + extent * float(s) / float(BINS);
            }
        }
    }
    if (!have || !(best_cost < leaf_cost)) return false;
    axis_out = best_axis;
    at_out = best_at;
    return true;
}

}  // namespace

extern "C" size_t or_bvh_build(const float *pos, const uint32_t *mesh_first, size_t n_meshes, const uint32_t *mesh_material,
                               const uint8_t *material_casts, const uint32_t *tri_chart, lb_node *nodes_out,
                               size_t cap_nodes, lb_tri *tris_out, size_t *n_tris_out) {
    // bvh.rs:51-74: every casting triangle that is not degenerate, in mesh then triangle order
    std::vector<Prim> prims;
    for (size_t mi = 0; mi < n_meshes; mi++) {
        if (!material_casts[mesh_material[mi]]) continue;
        for (uint32_t t = mesh_first[mi]; t < mesh_first[mi + 1]; t++) {
            const float *v = pos + size_t(t) * 9;
            V3 a{v[0], v[1], v[2]}, b{v[3], v[4], v[5]}, c{v[6], v[7], v[8]};
            V3 e1 = sub(b, a), e2 = sub(c, a);
            V3 n = cross(e1, e2);
            if (dot(n, n) < 1e-14f) continue;
            Prim p;
            p.min = vmin(vmin(a, b), c);
            p.max = vmax(vmax(a, b), c);
            p.centre = V3{(a.x + b.x + c.x) / 3.0f, (a.y + b.y + c.y) / 3.0f, (a.z + b.z + c.z) / 3.0f};
            float rec[12] = {a.x, a.y, a.z, from_bits(mesh_material[mi]), e1.x, e1.y, e1.z, from_bits(tri_chart[t]),
                             e2.x, e2.y, e2.z, 0.0f};
            std::memcpy(&p.tri, rec, sizeof rec);
            prims.push_back(p);
        }
    }
    std::vector<lb_node> nodes(1);
    std::memset(nodes.data(), 0, sizeof(lb_node));
    if (prims.empty()) {
        // bvh.rs:75-79: one empty leaf, a box nothing reaches
        lb_node &r = nodes[0];
        for (int a = 0; a < 3; a++) {
            r.min[a] = 3.40282347e+38f;
            r.max[a] = -3.40282347e+38f;
        }
        r.first = 0;
        r.count = 0;
        if (cap_nodes >= 1) nodes_out[0] = r;
        std::memset(tris_out, 0, sizeof(lb_tri));
        *n_tris_out = 1;
        return 1;
    }
    struct Job {
        size_t ni, start, end;
    };
    std::vector<Job> stack{{0, 0, prims.size()}};
    auto leaf = [&](size_t ni, V3 lo, V3 hi, size_t start, size_t end) {
        lb_node &r = nodes[ni];
        r.min[0] = lo.x, r.min[1] = lo.y, r.min[2] = lo.z;
        r.max[0] = hi.x, r.max[1] = hi.y, r.max[2] = hi.z;
        r.first = uint32_t(start);
        r.count = uint32_t(end - start);
    };
    while (!stack.empty()) {
        Job j = stack.back();
        stack.pop_back();
        Prim *s = prims.data() + j.start;
        size_t n = j.end - j.start;
        Box bb;
        for (size_t i = 0; i < n; i++) bb.add(s[i].min, s[i].max);
        int axis = 0;
        float at = 0.0f;
        bool split = n > LEAF && best_split(s, n, axis, at);
        if (!split) {
            leaf(j.ni, bb.lo, bb.hi, j.start, j.end);
            continue;
        }
        // bvh.rs:153-162: move the primitives whose centre lies below the plane to the front
        size_t i = 0;
        for (size_t k = 0; k < n; k++)
            if (s[k].centre[axis] < at) {
                std::swap(s[i], s[k]);
                i++;
            }
        size_t mid = j.start + i;
        if (mid == j.start || mid == j.end) mid = j.start + n / 2;
        if (mid - j.start == 0 || j.end - mid == 0) {
            leaf(j.ni, bb.lo, bb.hi, j.start, j.end);
            continue;
        }
        size_t left = nodes.size();
        nodes.resize(nodes.size() + 2);
        std::memset(&nodes[left], 0, 2 * sizeof(lb_node));
        lb_node &r = nodes[j.ni];
        r.min[0] = bb.lo.x, r.min[1] = bb.lo.y, r.min[2] = bb.lo.z;
        r.max[0] = bb.hi.x, r.max[1] = bb.hi.y, r.max[2] = bb.hi.z;
        r.first = uint32_t(left);
        r.count = 0;
        stack.push_back({left + 1, mid, j.end});
        stack.push_back({left, j.start, mid});
    }
    if (nodes.size() <= cap_nodes) std::memcpy(nodes_out, nodes.data(), nodes.size() * sizeof(lb_node));
    for (size_t i = 0; i < prims.size(); i++) tris_out[i] = prims[i].tri;
    *n_tris_out = prims.size();
    return nodes.size();
}
