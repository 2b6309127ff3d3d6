#include "bvh.h"

#include <omp.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <tuple>
#include <vector>

namespace lb {

namespace {
constexpr size_t BINS = 16;  // bvh.rs:9
constexpr size_t LEAF = 4;   // bvh.rs:10

// A primitive as the build moves it (40 bytes: the passes over a node's primitives and the partition's
// swaps touch only these); its triangle record and source are kept apart, by id.
struct Prim {
    Vec3 min, max, centre;
    uint32_t id;
};
struct Source {
    lb_tri tri;
    uint32_t mesh, index;  // where its vertices are in the scene
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

// Above this many primitives a node's bounds and bins are gathered by all threads, each over one
// contiguous run of the primitives, and the runs' results are merged in run order: fmin and fmax keep
// the first of equal values (so of -0 and +0 too), so the merge gives the serial fold's bits.
constexpr size_t PARALLEL_BINS = 1 << 15;
constexpr int MAX_PARTS = 64;  // runs a node's gathering is split into at most

// the contiguous run [lo, hi) of n items that part k of parts takes
inline void run_of(size_t n, int k, int parts, size_t &lo, size_t &hi) {
    lo = n * size_t(k) / size_t(parts);
    hi = n * size_t(k + 1) / size_t(parts);
}

// One axis's bins: bounds and counts.
struct Bins {
    Vec3 mn[BINS], mx[BINS];
    uint32_t n[BINS];
    void clear() {
        for (size_t b = 0; b < BINS; b++) {
            mn[b] = Vec3::splat(INFINITY);
            mx[b] = Vec3::splat(-INFINITY);
            n[b] = 0;
        }
    }
};

// A node's centres' bounds and its bounds over p[lo, hi), each folded in order (into locals: the callers'
// slots for several threads' runs share cache lines).
inline void gather_bounds(const Prim *p, size_t lo, size_t hi, Vec3 &cmin_out, Vec3 &cmax_out, Vec3 &pmin_out,
                          Vec3 &pmax_out) {
    Vec3 cmin = cmin_out, cmax = cmax_out, pmin = pmin_out, pmax = pmax_out;
    for (size_t i = lo; i < hi; i++) {
        bounds_add(cmin, cmax, p[i].centre, p[i].centre);
        bounds_add(pmin, pmax, p[i].min, p[i].max);
    }
    cmin_out = cmin, cmax_out = cmax, pmin_out = pmin, pmax_out = pmax;
}

// p[lo, hi) into the bins of every axis that is binned (use[axis]), in order (bvh.rs:127-133)
inline void gather_bins(const Prim *p, size_t lo, size_t hi, const bool use[3], const Vec3 &cmin, const float ext[3],
                        Bins out[3]) {
    Bins bins[3] = {out[0], out[1], out[2]};
    for (size_t i = lo; i < hi; i++) {
        for (int axis = 0; axis < 3; axis++) {
            if (!use[axis]) continue;
            float f = (p[i].centre[axis] - cmin[axis]) / ext[axis] * float(BINS);
            size_t b = f > 0.0f ? size_t(f) : 0;  // Rust `as usize`: truncation, saturating at 0
            if (b > BINS - 1) b = BINS - 1;
            Bins &q = bins[axis];
            q.mn[b] = q.mn[b].min(p[i].min);
            q.mx[b] = q.mx[b].max(p[i].max);
            q.n[b]++;
        }
    }
    for (int axis = 0; axis < 3; axis++) out[axis] = bins[axis];
}

// bvh.rs:119-151: the axis and plane of the cheapest binned split, if one beats a leaf, and the node's
// bounds (pmin, pmax: the fold bvh.rs:66-67 makes, the same bits, gathered here once). The three axes
// are binned in one pass over the primitives; from PARALLEL_BINS primitives on, every thread takes one
// contiguous run and the runs' bounds and bins are merged in run order. (The per-run arrays are sized to
// the runs: most calls are for nodes of a few primitives, for which clearing arrays sized for 64 runs
// cost more than the binning.)
bool best_split(const Prim *p, size_t n, int &axis_out, float &at_out, Vec3 &pmin, Vec3 &pmax) {
    Vec3 cmin = Vec3::splat(INFINITY), cmax = Vec3::splat(-INFINITY);
    pmin = cmin, pmax = cmax;
    const int parts = n >= PARALLEL_BINS ? std::max(1, std::min(omp_get_max_threads(), MAX_PARTS)) : 1;
    if (parts == 1) {
        gather_bounds(p, 0, n, cmin, cmax, pmin, pmax);
    } else {
        std::vector<Vec3> a(parts, Vec3::splat(INFINITY)), b(parts, Vec3::splat(-INFINITY)), c = a, d = b;
#pragma omp parallel for schedule(static, 1)
        for (int k = 0; k < parts; k++) {
            size_t lo, hi;
            run_of(n, k, parts, lo, hi);
            gather_bounds(p, lo, hi, a[k], b[k], c[k], d[k]);
        }
        for (int k = 0; k < parts; k++) {
            bounds_add(cmin, cmax, a[k], b[k]);
            bounds_add(pmin, pmax, c[k], d[k]);
        }
    }
    float leaf_cost = float(n) * area(pmin, pmax);
    bool use[3];
    float ext[3];
    for (int axis = 0; axis < 3; axis++) {
        ext[axis] = cmax[axis] - cmin[axis];
        use[axis] = !(ext[axis] < 1e-6f);
    }
    Bins bins[3];
    for (auto &q : bins) q.clear();
    if (parts == 1) {
        gather_bins(p, 0, n, use, cmin, ext, bins);
    } else {
        std::vector<Bins> runs(size_t(parts) * 3);
        for (auto &q : runs) q.clear();
#pragma omp parallel for schedule(static, 1)
        for (int k = 0; k < parts; k++) {
            size_t lo, hi;
            run_of(n, k, parts, lo, hi);
            gather_bins(p, lo, hi, use, cmin, ext, &runs[size_t(k) * 3]);
        }
        for (int k = 0; k < parts; k++)
            for (int axis = 0; axis < 3; axis++)
                for (size_t b = 0; b < BINS; b++) {
                    const Bins &r = runs[size_t(k) * 3 + axis];
                    bins[axis].mn[b] = bins[axis].mn[b].min(r.mn[b]);
                    bins[axis].mx[b] = bins[axis].mx[b].max(r.mx[b]);
                    bins[axis].n[b] += r.n[b];
                }
    }
    bool have = false;
    float best_cost = 0, best_at = 0;
    int best_axis = 0;
    for (int axis = 0; axis < 3; axis++) {
        if (!use[axis]) continue;
        const float extent = ext[axis];
        const Bins &q = bins[axis];
        // the bins' bounds and counts below and from each plane, swept once each way: min and max give the
        // reference's per-plane folds (bvh.rs:135-137) up to the sign of a zero, which no area changes
        // (max - min and its clamp at 0 are the same for either zero), so every cost compares the same
        Vec3 lo_min[BINS], lo_max[BINS], hi_min[BINS], hi_max[BINS];
        uint32_t lo_n[BINS], hi_n[BINS];
        {
            Vec3 mn = Vec3::splat(INFINITY), mx = Vec3::splat(-INFINITY);
            uint32_t c = 0;
            for (size_t b = 0; b < BINS; b++) {
                lo_min[b] = mn, lo_max[b] = mx, lo_n[b] = c;  // bins [0, b)
                bounds_add(mn, mx, q.mn[b], q.mx[b]);
                c += q.n[b];
            }
            mn = Vec3::splat(INFINITY), mx = Vec3::splat(-INFINITY), c = 0;
            for (size_t b = BINS; b-- > 0;) {
                bounds_add(mn, mx, q.mn[b], q.mx[b]);
                c += q.n[b];
                hi_min[b] = mn, hi_max[b] = mx, hi_n[b] = c;  // bins [b, BINS)
            }
        }
        for (size_t s = 1; s < BINS; s++) {
            uint32_t ln = lo_n[s], rn = hi_n[s];
            if (ln == 0 || rn == 0) continue;
            float cost = float(ln) * area(lo_min[s], lo_max[s]) + float(rn) * area(hi_min[s], hi_max[s]);
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
// bvh.rs:62-104 over prims[start, end) alone: its nodes in the order the walk allocates them, node 0 the
// range's root; an inner node's `first` is its left child's local index, a leaf's the global index of its
// first triangle.
void build_subtree(std::vector<Prim> &prims, size_t start0, size_t end0, std::vector<lb_node> &nodes) {
    nodes.assign(1, lb_node{});
    auto set = [&](size_t ni, Vec3 mn, uint32_t first, Vec3 mx, uint32_t count) {
        nodes[ni] = lb_node{{mn.x, mn.y, mn.z}, first, {mx.x, mx.y, mx.z}, count};
    };
    std::vector<std::tuple<size_t, size_t, size_t>> stack{{0, start0, end0}};
    while (!stack.empty()) {
        auto [ni, start, end] = stack.back();
        stack.pop_back();
        Prim *slice = prims.data() + start;
        size_t n = end - start;
        Vec3 bmin = Vec3::splat(INFINITY), bmax = Vec3::splat(-INFINITY);
        int axis;
        float at;
        bool split = false;
        if (n > LEAF) split = best_split(slice, n, axis, at, bmin, bmax);
        else
            for (size_t i = 0; i < n; i++) bounds_add(bmin, bmax, slice[i].min, slice[i].max);
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
        size_t left = nodes.size();
        nodes.push_back(lb_node{});
        nodes.push_back(lb_node{});
        set(ni, bmin, uint32_t(left), bmax, 0);
        stack.emplace_back(left + 1, mid, end);
        stack.emplace_back(left, start, mid);
    }
}
}  // namespace

// bvh.rs:50-106
Bvh Bvh::build(const Scene &scene, const std::function<uint32_t(size_t, size_t)> &chart) {
    // bvh.rs:51-74: every casting triangle that is not degenerate, in mesh and triangle order. Done in
    // parallel: each thread's contiguous run of the scene's triangles is counted, then written from the
    // count of the runs before it (the same order and ids as one pass).
    std::vector<size_t> mesh_first(scene.header.meshes.size() + 1, 0);
    for (size_t mi = 0; mi < scene.header.meshes.size(); mi++) {
        const MeshInfo &m = scene.header.meshes[mi];
        const size_t nt = scene.header.materials[m.material].casts ? scene.positions[mi].size() / 3 : 0;
        mesh_first[mi + 1] = mesh_first[mi] + nt;
    }
    const size_t n_all = mesh_first.back();
    auto locate = [&](size_t g, size_t &mi, size_t &t) {
        mi = size_t(std::upper_bound(mesh_first.begin(), mesh_first.end(), g) - mesh_first.begin()) - 1;
        t = g - mesh_first[mi];
    };
    auto keeps = [&](size_t mi, size_t t) {
        const std::vector<Vec3> &p = scene.positions[mi];
        Vec3 a = p[t * 3], b = p[t * 3 + 1], c = p[t * 3 + 2];
        return !((b - a).cross(c - a).length_squared() < 1e-14f);
    };
    const int runs_n = std::max(1, std::min(omp_get_max_threads() * 4, int((n_all + 4095) / 4096)));
    std::vector<size_t> kept(size_t(runs_n) + 1, 0);
#pragma omp parallel for schedule(dynamic, 1)
    for (int k = 0; k < runs_n; k++) {
        size_t lo, hi, mi, t, c = 0;
        run_of(n_all, k, runs_n, lo, hi);
        for (size_t g = lo; g < hi; g++) {
            locate(g, mi, t);
            c += keeps(mi, t) ? 1 : 0;
        }
        kept[size_t(k) + 1] = c;
    }
    for (int k = 0; k < runs_n; k++) kept[size_t(k) + 1] += kept[size_t(k)];
    std::vector<Prim> prims(kept.back());
    std::vector<Source> sources(kept.back());
#pragma omp parallel for schedule(dynamic, 1)
    for (int k = 0; k < runs_n; k++) {
        size_t lo, hi, mi, t, at = kept[size_t(k)];
        run_of(n_all, k, runs_n, lo, hi);
        for (size_t g = lo; g < hi; g++) {
            locate(g, mi, t);
            if (!keeps(mi, t)) continue;
            const MeshInfo &m = scene.header.meshes[mi];
            const std::vector<Vec3> &p = scene.positions[mi];
            Vec3 a = p[t * 3], b = p[t * 3 + 1], c = p[t * 3 + 2];
            Vec3 e1 = b - a, e2 = c - a;
            Prim &q = prims[at];
            q.min = a.min(b).min(c);
            q.max = a.max(b).max(c);
            q.centre = (a + b + c) / 3.0f;
            q.id = uint32_t(at);
            sources[at] = Source{lb_tri{{a.x, a.y, a.z, u2f(m.material)}, {e1.x, e1.y, e1.z, u2f(chart(mi, t))},
                                        {e2.x, e2.y, e2.z, 0.0f}},
                                 uint32_t(mi), uint32_t(t)};
            at++;
        }
    }
    Bvh out;
    out.nodes.push_back(lb_node{});
    if (prims.empty()) {
        // one empty leaf, a box nothing reaches
        out.nodes[0] = lb_node{{FLT_MAX, FLT_MAX, FLT_MAX}, 0, {-FLT_MAX, -FLT_MAX, -FLT_MAX}, 0};
        out.tris.push_back(lb_tri{});
        out.verts.assign(9, 0.0f);
        out.source.assign(1, {0xffffffffu, 0xffffffffu});
        return out;
    }
    // The serial walk below (bvh.rs:62-104) pops a node, decides it a leaf or splits its primitives in
    // place and allocates its two children next, then walks the left subtree before the right one. So
    // every subtree's nodes but its root come out as one contiguous run, in the order the same walk over
    // the subtree alone allocates them. Nodes of fewer than `cut` primitives become subtrees built on
    // their own (in parallel: their primitive ranges are disjoint); the top of the tree is walked first,
    // then walked again in the serial order, each subtree's run spliced in when its root is popped.
    // Indices, node bytes and triangle order are the serial build's.
    struct Top {
        size_t start, end;
        bool leaf = false, task = false;
        Vec3 bmin, bmax;
        int left = -1, right = -1;
        size_t task_id = 0;
    };
    const size_t cut = std::max<size_t>(2048, prims.size() / 32);
    std::vector<Top> top;
    std::vector<std::pair<size_t, size_t>> tasks;
    top.push_back(Top{0, prims.size()});
    std::vector<int> todo{0};
    while (!todo.empty()) {
        int id = todo.back();
        todo.pop_back();
        size_t start = top[id].start, end = top[id].end, n = end - start;
        if (n < cut) {
            top[id].task = true;
            top[id].task_id = tasks.size();
            tasks.emplace_back(start, end);
            continue;
        }
        Prim *slice = prims.data() + start;
        Vec3 bmin = Vec3::splat(INFINITY), bmax = Vec3::splat(-INFINITY);
        int axis;
        float at;
        bool split = false;
        if (n > LEAF) split = best_split(slice, n, axis, at, bmin, bmax);
        else
            for (size_t i = 0; i < n; i++) bounds_add(bmin, bmax, slice[i].min, slice[i].max);
        top[id].bmin = bmin;
        top[id].bmax = bmax;
        size_t mid = 0;
        if (split) {
            mid = start + partition(slice, n, axis, at);
            if (mid == start || mid == end) mid = start + n / 2;
            if (mid - start == 0 || end - mid == 0) split = false;
        }
        if (!split) {
            top[id].leaf = true;
            continue;
        }
        int l = int(top.size()), r = l + 1;
        top.push_back(Top{start, mid});
        top.push_back(Top{mid, end});
        top[id].left = l;
        top[id].right = r;
        todo.push_back(r);
        todo.push_back(l);
    }
    std::vector<std::vector<lb_node>> runs(tasks.size());
#pragma omp parallel for schedule(dynamic, 1)
    for (long long k = 0; k < (long long)tasks.size(); k++) build_subtree(prims, tasks[k].first, tasks[k].second, runs[k]);
    auto set = [&](size_t ni, Vec3 mn, uint32_t first, Vec3 mx, uint32_t count) {
        out.nodes[ni] = lb_node{{mn.x, mn.y, mn.z}, first, {mx.x, mx.y, mx.z}, count};
    };
    std::vector<std::pair<size_t, int>> stack{{0, 0}};
    while (!stack.empty()) {
        auto [ni, id] = stack.back();
        stack.pop_back();
        const Top &t = top[id];
        if (t.task) {
            const std::vector<lb_node> &run = runs[t.task_id];
            size_t base = out.nodes.size();
            // local node k (k >= 1) lands at base + k - 1; a leaf's first is already a triangle index
            auto place = [&](lb_node v) {
                if (v.count == 0) v.first = uint32_t(base + v.first - 1);
                return v;
            };
            out.nodes[ni] = place(run[0]);
            for (size_t k = 1; k < run.size(); k++) out.nodes.push_back(place(run[k]));
        } else if (t.leaf) {
            set(ni, t.bmin, uint32_t(t.start), t.bmax, uint32_t(t.end - t.start));
        } else {
            size_t left = out.nodes.size();
            out.nodes.push_back(lb_node{});
            out.nodes.push_back(lb_node{});
            set(ni, t.bmin, uint32_t(left), t.bmax, 0);
            stack.emplace_back(left + 1, t.right);
            stack.emplace_back(left, t.left);
        }
    }
    out.tris.resize(prims.size());
    out.source.resize(prims.size());
    out.verts.resize(prims.size() * 9);
#pragma omp parallel for schedule(static)
    for (long long ii = 0; ii < (long long)prims.size(); ii++) {
        const size_t i = size_t(ii);
        out.tris[i] = sources[prims[i].id].tri;
        const Source &src = sources[prims[i].id];
        out.source[i] = {src.mesh, src.index};
        const std::vector<Vec3> &p = scene.positions[src.mesh];
        for (int k = 0; k < 3; k++) {
            Vec3 v = p[size_t(src.index) * 3 + k];
            out.verts[i * 9 + k * 3] = v.x;
            out.verts[i * 9 + k * 3 + 1] = v.y;
            out.verts[i * 9 + k * 3 + 2] = v.z;
        }
    }
    return out;
}

void Bvh::set_charts(const std::function<uint32_t(size_t, size_t)> &chart) {
    for (size_t i = 0; i < tris.size(); i++)
        if (source[i][0] != 0xffffffffu) tris[i].e1[3] = u2f(chart(source[i][0], source[i][1]));
}

}  // namespace lb
