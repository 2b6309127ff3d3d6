#include "bvh8.h"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <deque>
#include <stdexcept>
#include <string>

namespace lb {

namespace {

struct Box {
    float mn[3], mx[3];
};

// a child to place in a slot: a BVH2 inner node, or a run of triangles of the BVH2 triangle array
struct Ref {
    bool leaf;
    uint32_t node;          // inner: BVH2 node index
    uint32_t first, count;  // leaf: triangles [first, first + count)
    Box box;
};

float area(const Box &b) {
    float d[3];
    for (int a = 0; a < 3; a++) d[a] = std::max(b.mx[a] - b.mn[a], 0.0f);
    return d[0] * d[1] + d[1] * d[2] + d[2] * d[0];
}

constexpr uint32_t SLOT_TRIS = 4;  // triangles a leaf slot holds
constexpr uint32_t NODE_TRIS = 32; // triangles a node's leaf slots hold together (5-bit offsets)

struct Builder {
    const lb_node *n2;
    size_t nn2;
    const lb_tri *t2;
    Bvh8 out;
    // a node to emit: its children; `synthetic` runs of more than SLOT_TRIS triangles become their own node
    std::deque<std::pair<uint32_t, std::vector<Ref>>> todo;

    Box node_box(uint32_t i) const {
        Box b;
        for (int a = 0; a < 3; a++) {
            b.mn[a] = n2[i].min[a];
            b.mx[a] = n2[i].max[a];
        }
        return b;
    }
    Ref ref_of(uint32_t i) const {
        Ref r{};
        r.box = node_box(i);
        if (n2[i].count > 0) {
            r.leaf = true;
            r.first = n2[i].first;
            r.count = n2[i].count;
        } else {
            r.leaf = false;
            r.node = i;
        }
        return r;
    }
    bool expandable(const Ref &r) const { return !r.leaf && size_t(n2[r.node].first) + 1 < nn2; }

    // the children of an inner BVH2 node, opened (largest area first) until eight
    std::vector<Ref> open(uint32_t i) const {
        std::vector<Ref> refs;
        if (size_t(n2[i].first) + 1 >= nn2) return refs;  // the reference's empty one-node BVH
        refs.push_back(ref_of(n2[i].first));
        refs.push_back(ref_of(n2[i].first + 1));
        while (refs.size() < 8) {
            int best = -1;
            float ba = -1.0f;
            for (size_t k = 0; k < refs.size(); k++)
                if (expandable(refs[k]) && area(refs[k].box) > ba) {
                    ba = area(refs[k].box);
                    best = int(k);
                }
            if (best < 0) break;
            uint32_t c = refs[best].node;
            refs[best] = ref_of(n2[c].first);
            refs.insert(refs.begin() + best + 1, ref_of(n2[c].first + 1));
        }
        return refs;
    }

    // children of a run of more than SLOT_TRIS triangles: runs of at most SLOT_TRIS, grouped eight to a node
    std::vector<Ref> split_run(const Ref &r) const {
        std::vector<Ref> parts;
        uint32_t per = SLOT_TRIS;
        uint32_t chunks = (r.count + per - 1) / per;
        if (chunks <= 8) {
            for (uint32_t k = 0; k < chunks; k++) {
                Ref c = r;
                c.first = r.first + k * per;
                c.count = std::min(per, r.count - k * per);
                parts.push_back(c);
            }
            return parts;
        }
        // more than 32 triangles: eight runs, each split again
        uint32_t each = (r.count + 7) / 8;
        for (uint32_t k = 0; k < 8 && k * each < r.count; k++) {
            Ref c = r;
            c.first = r.first + k * each;
            c.count = std::min(each, r.count - k * each);
            parts.push_back(c);
        }
        return parts;
    }

    void emit(uint32_t idx, std::vector<Ref> refs) {
        // a leaf slot over SLOT_TRIS triangles becomes a node of its own
        uint32_t *w = &out.nodes[size_t(idx) * 20];
        uint32_t imask = 0;
        uint8_t meta[8];
        std::memset(meta, 0xff, 8);
        uint32_t child_base = uint32_t(out.n_nodes());
        uint32_t tri_base = uint32_t(out.tris.size());
        uint32_t tri_off = 0;
        std::vector<std::pair<uint32_t, std::vector<Ref>>> kids;
        for (size_t s = 0; s < refs.size(); s++) {
            Ref &r = refs[s];
            bool as_node = !r.leaf || r.count > SLOT_TRIS || tri_off + r.count > NODE_TRIS;
            if (as_node) {
                imask |= 1u << s;
                std::vector<Ref> sub = r.leaf ? split_run(r) : open(r.node);
                kids.emplace_back(uint32_t(out.n_nodes() + kids.size()), std::move(sub));
            } else {
                meta[s] = uint8_t(tri_off | ((r.count - 1) << 5));
                for (uint32_t t = 0; t < r.count; t++) {
                    lb_tri tr = t2[r.first + t];
                    uint32_t orig = r.first + t;
                    std::memcpy(&tr.e2[3], &orig, 4);
                    out.tris.push_back(tr);
                }
                tri_off += r.count;
            }
        }
        // the node's box and quantisation
        Box all{{FLT_MAX, FLT_MAX, FLT_MAX}, {-FLT_MAX, -FLT_MAX, -FLT_MAX}};
        for (auto &r : refs)
            for (int a = 0; a < 3; a++) {
                all.mn[a] = std::min(all.mn[a], r.box.mn[a]);
                all.mx[a] = std::max(all.mx[a], r.box.mx[a]);
            }
        if (refs.empty())
            for (int a = 0; a < 3; a++) all.mn[a] = all.mx[a] = 0.0f;
        uint8_t q[6][8];
        std::memset(q, 0, sizeof q);
        uint32_t eb[3];
        for (int a = 0; a < 3; a++) {
            float p = all.mn[a];
            double extent = double(all.mx[a]) - double(p);
            int e = extent > 0 ? int(std::ceil(std::log2(extent / 255.0))) : -100;
            e = std::max(e, -100);
            for (;; e++) {
                float scale = std::ldexp(1.0f, e);
                bool ok = true;
                for (size_t s = 0; s < refs.size() && ok; s++) {
                    double lo = std::floor((double(refs[s].box.mn[a]) - p) / scale);
                    double hi = std::ceil((double(refs[s].box.mx[a]) - p) / scale);
                    lo = std::max(lo, 0.0);
                    // the device's float dequantisation must bound the child's box
                    while (lo > 0 && p + float(lo) * scale > refs[s].box.mn[a]) lo -= 1;
                    while (hi <= 255 && p + float(hi) * scale < refs[s].box.mx[a]) hi += 1;
                    if (hi > 255 || p + float(lo) * scale > refs[s].box.mn[a]) {
                        ok = false;
                        break;
                    }
                    q[a][s] = uint8_t(lo);
                    q[3 + a][s] = uint8_t(hi);
                }
                if (ok) break;
                if (e > 120) throw std::runtime_error("bvh8: cannot quantise a node's boxes");
            }
            eb[a] = uint32_t(e + 127);
        }
        // empty slots: lo 1 > hi 0, a box no ray enters
        for (size_t s = refs.size(); s < 8; s++)
            for (int a = 0; a < 3; a++) {
                q[a][s] = 1;
                q[3 + a][s] = 0;
            }
        float p3[3] = {all.mn[0], all.mn[1], all.mn[2]};
        std::memcpy(&w[0], p3, 12);
        w[3] = eb[0] | (eb[1] << 8) | (eb[2] << 16) | (imask << 24);
        w[4] = child_base;
        w[5] = tri_base;
        std::memcpy(&w[6], meta, 8);
        std::memcpy(&w[8], q, 48);
        // inner children follow, in slot order
        out.nodes.resize(out.nodes.size() + kids.size() * 20, 0);
        for (auto &k : kids) todo.push_back(std::move(k));
    }
};

}  // namespace

Bvh8 Bvh8::collapse(const lb_node *nodes, size_t n_nodes, const lb_tri *tris, size_t n_tris) {
    Builder b{nodes, n_nodes, tris, {}, {}};
    (void)n_tris;
    b.out.nodes.assign(20, 0);
    std::vector<Ref> root;
    if (nodes[0].count > 0) {
        Ref r = b.ref_of(0);
        root = r.count > SLOT_TRIS ? b.split_run(r) : std::vector<Ref>{r};
    } else {
        root = b.open(0);
    }
    b.todo.emplace_back(0, std::move(root));
    while (!b.todo.empty()) {
        auto [idx, refs] = std::move(b.todo.front());
        b.todo.pop_front();
        b.emit(idx, std::move(refs));
    }
    if (b.out.tris.empty()) b.out.tris.push_back(lb_tri{});
    return std::move(b.out);
}

}  // namespace lb

namespace lb {

// Structural checks of a collapse (for tests): every triangle reached once; children in range; each
// triangle's corners inside every box on its path from the root (what a correct walk needs; a child's
// box may reach past its parent's by a quantum, which does not matter).
std::string bvh8_check(const Bvh8 &b, size_t n_tris, size_t &depth) {
    struct Frame {
        size_t node, depth;
        float mn[3], mx[3];
    };
    auto slot_box = [&](const uint32_t *w, int s, float mn[3], float mx[3]) {
        float p[3];
        std::memcpy(p, w, 12);
        const uint8_t *q = (const uint8_t *)&w[8];
        for (int a = 0; a < 3; a++) {
            float scale;
            uint32_t bits = ((w[3] >> (8 * a)) & 0xffu) << 23;
            std::memcpy(&scale, &bits, 4);
            mn[a] = p[a] + float(q[a * 8 + s]) * scale;
            mx[a] = p[a] + float(q[(3 + a) * 8 + s]) * scale;
        }
    };
    std::vector<int> seen(n_tris, 0);
    std::vector<Frame> st{{0, 1, {-FLT_MAX, -FLT_MAX, -FLT_MAX}, {FLT_MAX, FLT_MAX, FLT_MAX}}};
    depth = 0;
    size_t visited = 0;
    while (!st.empty()) {
        Frame f = st.back();
        st.pop_back();
        depth = std::max(depth, f.depth);
        if (f.node >= b.n_nodes()) return "child index out of range";
        if (++visited > b.n_nodes()) return "a node reached twice";
        const uint32_t *w = &b.nodes[f.node * 20];
        uint32_t imask = w[3] >> 24, inner_rank = 0;
        const uint8_t *meta = (const uint8_t *)&w[6];
        for (int s = 0; s < 8; s++) {
            float mn[3], mx[3];
            slot_box(w, s, mn, mx);
            for (int a = 0; a < 3; a++) {
                mn[a] = std::max(mn[a], f.mn[a]);
                mx[a] = std::min(mx[a], f.mx[a]);
            }
            if ((imask >> s) & 1u) {
                Frame c{w[4] + inner_rank++, f.depth + 1, {mn[0], mn[1], mn[2]}, {mx[0], mx[1], mx[2]}};
                st.push_back(c);
            } else if (meta[s] != 0xff) {
                uint32_t first = w[5] + (meta[s] & 31u), cnt = ((meta[s] >> 5) & 3u) + 1u;
                for (uint32_t k = 0; k < cnt; k++) {
                    if (first + k >= b.tris.size()) return "triangle index out of range";
                    const lb_tri &t = b.tris[first + k];
                    uint32_t orig;
                    std::memcpy(&orig, &t.e2[3], 4);
                    if (orig >= n_tris) return "reference index out of range";
                    seen[orig]++;
                    for (int c3 = 0; c3 < 3; c3++)
                        for (int x = 0; x < 3; x++) {
                            float v = t.v0[x] + (c3 == 1 ? t.e1[x] : c3 == 2 ? t.e2[x] : 0.0f);
                            float tol = 1e-4f * (1.0f + std::fabs(v));
                            if (v < mn[x] - tol || v > mx[x] + tol) return "a triangle outside a box on its path";
                        }
                }
            }
        }
    }
    for (size_t i = 0; i < n_tris; i++)
        if (seen[i] != 1) return "triangle " + std::to_string(i) + " reached " + std::to_string(seen[i]) + " times";
    return "";
}

}  // namespace lb
