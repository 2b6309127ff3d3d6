#include "bvh8.h"

#include "bvh8_node.h"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <deque>
#include <stdexcept>
#include <string>

namespace lb {

// Breadth first, as the device builder (bvh8_build.cu) emits level by level: a node's inner children
// are numbered one after another in the order its slots list them, after every node emitted before it.
Bvh8 Bvh8::collapse(const lb_node *nodes, size_t n_nodes, const lb_tri *tris, size_t n_tris) {
    (void)n_tris;
    Bvh8 out;
    out.nodes.assign(lb8::WORDS, 0);
    std::deque<std::pair<uint32_t, lb8::Item>> todo;
    todo.emplace_back(0, lb8::root_item(nodes));
    while (!todo.empty()) {
        auto [idx, item] = todo.front();
        todo.pop_front();
        lb8::Ref refs[8];
        const int n = lb8::refs_of(nodes, n_nodes, item, refs);
        const uint32_t child_base = uint32_t(out.n_nodes()), tri_base = uint32_t(out.tris.size());
        uint32_t w[lb8::WORDS];
        if (!lb8::node_words(refs, n, child_base, tri_base, w))
            throw std::runtime_error("bvh8: cannot quantise a node's boxes");
        std::memcpy(&out.nodes[size_t(idx) * lb8::WORDS], w, sizeof w);
        const uint32_t imask = w[3] >> 24;
        uint32_t kids = 0;
        for (int s = 0; s < n; s++) {
            if ((imask >> s) & 1u) {
                todo.emplace_back(child_base + kids++, lb8::item_of(refs[s]));
                continue;
            }
            for (uint32_t t = 0; t < refs[s].count; t++) {
                lb_tri tr = tris[refs[s].first + t];
                const uint32_t orig = refs[s].first + t;
                std::memcpy(&tr.e2[3], &orig, 4);
                out.tris.push_back(tr);
            }
        }
        out.nodes.resize(out.nodes.size() + size_t(kids) * lb8::WORDS, 0);
    }
    if (out.tris.empty()) out.tris.push_back(lb_tri{});
    return out;
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
