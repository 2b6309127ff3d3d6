// ORACLE — test infrastructure only (see oracle.h). The reference's CPU texel passes restated:
// crates/lightbaker/src/filter.rs (smooth :20-53, fill :58-94, sun_field :106-141).
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "oracle.h"

namespace {
// filter.rs:13-18: same chart and normals within n.n >= 0.9
inline bool same(const uint32_t *chart, const float *normal, size_t i, size_t j) {
    const float *a = normal + i * 3, *b = normal + j * 3;
    return chart[i] == chart[j] && a[0] * b[0] + a[1] * b[1] + a[2] * b[2] >= 0.9f;
}
}  // namespace

extern "C" {

// filter.rs:20-53
void or_smooth(int w, int h, const uint32_t *chart, const float *normal, const float *v, int N,
               const uint8_t *valid, int r, float *out) {
    size_t size = size_t(w) * h;
    std::memcpy(out, v, size * N * sizeof(float));
    if (r == 0) return;
    float q = float(r) * 0.75f;
    float sigma2 = 2.0f * (q * q);
    std::vector<float> sum(N);
    for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++) {
            size_t i = size_t(y) * w + x;
            if (!valid[i]) continue;
            std::fill(sum.begin(), sum.end(), 0.0f);
            float wsum = 0.0f;
            for (int yy = y > r ? y - r : 0; yy < std::min(y + r + 1, h); yy++)
                for (int xx = x > r ? x - r : 0; xx < std::min(x + r + 1, w); xx++) {
                    size_t j = size_t(yy) * w + xx;
                    if (!valid[j] || !same(chart, normal, i, j)) continue;
                    float dx = float(xx) - float(x), dy = float(yy) - float(y);
                    float k = std::exp(-(dx * dx + dy * dy) / sigma2);
                    for (int c = 0; c < N; c++) sum[c] += v[j * N + c] * k;
                    wsum += k;
                }
            for (int c = 0; c < N; c++) out[i * N + c] = sum[c] / wsum;
        }
}

// filter.rs:58-94 (a ring at a time from a snapshot of the last one)
void or_fill(int w, int h, const uint32_t *chart, float *v, int N, uint8_t *valid, int rings) {
    size_t size = size_t(w) * h;
    std::vector<uint8_t> was(size);
    std::vector<float> src(size * N), own(N), any(N);
    for (int ring = 0; ring < rings; ring++) {
        std::memcpy(was.data(), valid, size);
        std::memcpy(src.data(), v, size * N * sizeof(float));
        for (int y = 0; y < h; y++)
            for (int x = 0; x < w; x++) {
                size_t i = size_t(y) * w + x;
                if (was[i]) continue;
                std::fill(own.begin(), own.end(), 0.0f);
                std::fill(any.begin(), any.end(), 0.0f);
                int no = 0, na = 0;
                for (int yy = y > 0 ? y - 1 : 0; yy < std::min(y + 2, h); yy++)
                    for (int xx = x > 0 ? x - 1 : 0; xx < std::min(x + 2, w); xx++) {
                        size_t j = size_t(yy) * w + xx;
                        if (!was[j]) continue;
                        if (chart[i] != 0xffffffffu && chart[j] == chart[i]) {
                            for (int c = 0; c < N; c++) own[c] += src[j * N + c];
                            no++;
                        } else {
                            for (int c = 0; c < N; c++) any[c] += src[j * N + c];
                            na++;
                        }
                    }
                if (no > 0) {
                    for (int c = 0; c < N; c++) v[i * N + c] = own[c] / float(no);
                    valid[i] = 1;
                } else if (na > 0 && chart[i] == 0xffffffffu) {
                    for (int c = 0; c < N; c++) v[i * N + c] = any[c] / float(na);
                    valid[i] = 1;
                }
            }
    }
}

// filter.rs:106-141
void or_sun_field(int w, int h, const uint32_t *chart, const float *normal, const uint32_t *hard,
                  const uint8_t *covered, int g, float radius, float *out) {
    int reach = int(std::ceil(radius)) + 1;
    for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++) {
            size_t i = size_t(y) * w + x;
            out[i] = -1.0f;
            if (!covered[i]) continue;
            bool lit = size_t(__builtin_popcount(hard[i])) * 2 >= size_t(g) * g;
            float best = radius;
            for (int yy = y > reach ? y - reach : 0; yy < std::min(y + reach + 1, h); yy++)
                for (int xx = x > reach ? x - reach : 0; xx < std::min(x + reach + 1, w); xx++) {
                    size_t j = size_t(yy) * w + xx;
                    if (!covered[j] || !same(chart, normal, i, j)) continue;
                    for (int c = 0; c < g * g; c++) {
                        bool bit = ((hard[j] >> c) & 1u) == 1u;
                        if (bit == lit) continue;
                        float px = float(xx) + (float(c % g) + 0.5f) / float(g) - (float(x) + 0.5f);
                        float py = float(yy) + (float(c / g) + 0.5f) / float(g) - (float(y) + 0.5f);
                        best = std::fmin(best, std::sqrt(px * px + py * py) - 0.5f / float(g));
                    }
                }
            float d = std::fmin(std::fmax(best, 0.0f), radius);
            out[i] = 0.5f + 0.5f * (lit ? d : -d) / radius;
        }
}

}  // extern "C"
