// The CPU texel passes of the reference's bake, a tile at a time: crates/lightbaker/src/filter.rs.
// The plain (drop-in) bake runs them on the host between ray passes as the reference does; the
// device-resident bake runs the same passes as kernels (post.cu).
#pragma once
#include <array>
#include <cstdint>
#include <vector>

namespace lb {

struct Surface {  // filter.rs:4-18
    size_t w, h;
    const uint32_t *chart;
    const std::array<float, 3> *normal;
    bool same(size_t i, size_t j) const {
        const auto &a = normal[i], &b = normal[j];
        return chart[i] == chart[j] && a[0] * b[0] + a[1] * b[1] + a[2] * b[2] >= 0.9f;
    }
};

// filter.rs:20-53 (N channels a texel, interleaved)
std::vector<float> smooth(const Surface &s, const std::vector<float> &v, size_t N, const std::vector<uint8_t> &valid, size_t r);
// filter.rs:58-94
void fill(const Surface &s, std::vector<float> &v, size_t N, std::vector<uint8_t> &valid, size_t rings);
// filter.rs:106-141
std::vector<float> sun_field(const Surface &s, const std::vector<uint32_t> &hard, const std::vector<uint8_t> &covered,
                             size_t g, float radius);

}  // namespace lb
