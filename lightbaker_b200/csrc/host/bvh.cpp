#include "bvh.h"

#include <cfloat>
#include <cmath>
#include <tuple>

namespace lb {

namespace {
constexpr size_t BINS = 16;  // bvh.rs:9
constexpr size_t LEAF = 4;   // bvh.rs:10

struct Prim {
    Vec3 min, max, centre;
    lb_tri tri;
};

// bvh.rs:109-111
void bounds_add(Vec3 &a, Vec3 &b, Vec3 lo, Vec3 hi) {
    a = a.min(lo);
    b = b.max(hi);
}
// bvh.rs:113-116
float area(Vec3 mn, Vec3 mx) {
    Vec3 d = (mx - mn).max(Vec3(0, 0, 0));
    return d.x * d.y + d.y * d.z + d.z * d.x;
}

// bvh.rs:119-151: the axis and plane of the cheapest binned split, if one beats a leaf
bool best_split(const Prim *p, size_t n, int &axis_out, float &at_out) {
    Vec3 cmin = Vec3::splat(INFINITY), cmax = Vec3::splat(-INFINITY), pmin = cmin, pmax = cmax;
    for (size_t i = 0; i < n; i++) {
        bounds_add(cmin, cmax, p[i].centre, p[i].centre);
        bounds_add(pmin, pmax, p[i].min, p[i].max);
    }
    float leaf_cost = float(n) * area(pmin, pmax);
    bool have = false;
    float best_cost = 0, best_at = 0;
    int best_axis = 0;
    for (int axis = 0; axis < 3; axis++) {
        float extent = cmax[axis] - cmin[axis];
        if (extent < 1e-6f) continue;
        Vec3 bmin[BINS], bmax[BINS];
        uint32_t bn[BINS];
        for (size_t b = 0; b < BINS; b++) {
            bmin[b] = Vec3::splat(INFINITY);
            bmax[b] = Vec3::splat(-INFINITY);
            bn[b] = 0;
        }
        for (size_t i = 0; i < n; i++) {
            float f = (p[i].centre[axis] - cmin[axis]) / extent * float(BINS);
            size_t b = f > 0.0f ? size_t(f) : 0;  // Rust `as usize`: truncation, saturating at 0
            if (b > BINS - 1) b = BINS - 1;
            bmin[b] = bmin[b].min(p[i].min);
            bmax[b] = bmax[b].max(p[i].max);
            bn[b]++;
        }
        for (size_t s = 1; s < BINS; s++) {
            uint32_t ln = 0, rn = 0;
            Vec3 lmin = Vec3::splat(INFINITY), lmax = Vec3::splat(-INFINITY), rmin = lmin, rmax = lmax;
            for (size_t b = 0; b < s; b++) {
                ln += bn[b];
                bounds_add(lmin, lmax, bmin[b], bmax[b]);
            }
            for (size_t b = s; b < BINS; b++) {
                rn += bn[b];
                bounds_add(rmin, rmax, bmin[b], bmax[b]);
            }
            if (ln == 0 || rn == 0) continue;
            float cost = float(ln) * area(lmin, lmax) + float(rn) * area(rmin, rmax);
            if (!have || cost < best_cost) {
                have = true;
                best_cost = cost;
                best_axis = axis;
                best_at = cmin[axis] + extent * float(s) / float(BINS);
            }
        }
    }
    if (!have || !(best_cost < leaf_cost)) return false;
    axis_out = best_axis;
    at_out = best_at;
    return true;
}

// bvh.rs:153-162: in place, the order a swap partition leaves
size_t partition(Prim *p, size_t n, int axis, float at) {
    size_t i = 0;
    for (size_t j = 0; j < n; j++)
        if (p[j].centre[axis] < at) {
            std::swap(p[i], p[j]);
            i++;
        }
    return i;
}
}  // namespace

// bvh.rs:50-106
Bvh Bvh::build(const Scene &scene, const std::function<uint32_t(size_t, size_t)> &chart) {
    std::vector<Prim> prims;
    for (size_t mi = 0; mi < scene.header.meshes.size(); mi++) {
        const MeshInfo &m = scene.header.meshes[mi];
        if (!scene.header.materials[m.material].casts) continue;
        const std::vector<Vec3> &p = scene.positions[mi];
        for (size_t t = 0; t < p.size() / 3; t++) {
            Vec3 a = p[t * 3], b = p[t * 3 + 1], c = p[t * 3 + 2];
            Vec3 e1 = b - a, e2 = c - a;
            if (e1.cross(e2).length_squared() < 1e-14f) continue;
            Prim q;
            q.min = a.min(b).min(c);
            q.max = a.max(b).max(c);
            q.centre = (a + b + c) / 3.0f;
            q.tri = lb_tri{{a.x, a.y, a.z, u2f(m.material)}, {e1.x, e1.y, e1.z, u2f(chart(mi, t))}, {e2.x, e2.y, e2.z, 0.0f}};
            prims.push_back(q);
        }
    }
    Bvh out;
    out.nodes.push_back(lb_node{});
    if (prims.empty()) {
        // one empty leaf, a box nothing reaches
        out.nodes[0] = lb_node{{FLT_MAX, FLT_MAX, FLT_MAX}, 0, {-FLT_MAX, -FLT_MAX, -FLT_MAX}, 0};
        out.tris.push_back(lb_tri{});
        return out;
    }
    auto set = [&](size_t ni, Vec3 mn, uint32_t first, Vec3 mx, uint32_t count) {
        out.nodes[ni] = lb_node{{mn.x, mn.y, mn.z}, first, {mx.x, mx.y, mx.z}, count};
    };
    std::vector<std::tuple<size_t, size_t, size_t>> stack{{0, 0, prims.size()}};
    while (!stack.empty()) {
        auto [ni, start, end] = stack.back();
        stack.pop_back();
        Prim *slice = prims.data() + start;
        size_t n = end - start;
        Vec3 bmin = Vec3::splat(INFINITY), bmax = Vec3::splat(-INFINITY);
        for (size_t i = 0; i < n; i++) bounds_add(bmin, bmax, slice[i].min, slice[i].max);
        int axis;
        float at;
        bool split = n > LEAF && best_split(slice, n, axis, at);
        if (!split) {
            set(ni, bmin, uint32_t(start), bmax, uint32_t(n));
            continue;
        }
        size_t mid = start + partition(slice, n, axis, at);
        if (mid == start || mid == end) mid = start + n / 2;
        if (mid - start == 0 || end - mid == 0) {
            set(ni, bmin, uint32_t(start), bmax, uint32_t(n));
            continue;
        }
        size_t left = out.nodes.size();
        out.nodes.push_back(lb_node{});
        out.nodes.push_back(lb_node{});
        set(ni, bmin, uint32_t(left), bmax, 0);
        stack.emplace_back(left + 1, mid, end);
        stack.emplace_back(left, start, mid);
    }
    out.tris.reserve(prims.size());
    for (auto &p : prims) out.tris.push_back(p.tri);
    return out;
}

}  // namespace lb
