#include "filter.h"

#include <algorithm>
#include <cmath>

namespace lb {

std::vector<float> smooth(const Surface &s, const std::vector<float> &v, size_t N, const std::vector<uint8_t> &valid,
                          size_t r) {
    std::vector<float> out = v;
    if (r == 0) return out;
    float q = float(r) * 0.75f;
    float sigma2 = 2.0f * (q * q);
    std::vector<float> sum(N);
    for (size_t y = 0; y < s.h; y++)
        for (size_t x = 0; x < s.w; x++) {
            size_t i = y * s.w + x;
            if (!valid[i]) continue;
            std::fill(sum.begin(), sum.end(), 0.0f);
            float wsum = 0.0f;
            for (size_t yy = y > r ? y - r : 0; yy < std::min(y + r + 1, s.h); yy++)
                for (size_t xx = x > r ? x - r : 0; xx < std::min(x + r + 1, s.w); xx++) {
                    size_t j = yy * s.w + xx;
                    if (!valid[j] || !s.same(i, j)) continue;
                    float dx = float(xx) - float(x), dy = float(yy) - float(y);
                    float k = std::exp(-(dx * dx + dy * dy) / sigma2);
                    for (size_t c = 0; c < N; c++) sum[c] += v[j * N + c] * k;
                    wsum += k;
                }
            for (size_t c = 0; c < N; c++) out[i * N + c] = sum[c] / wsum;
        }
    return out;
}

void fill(const Surface &s, std::vector<float> &v, size_t N, std::vector<uint8_t> &valid, size_t rings) {
    std::vector<float> own(N), any(N);
    for (size_t ring = 0; ring < rings; ring++) {
        std::vector<uint8_t> was = valid;
        std::vector<float> src = v;
        for (size_t y = 0; y < s.h; y++)
            for (size_t x = 0; x < s.w; x++) {
                size_t i = y * s.w + x;
                if (was[i]) continue;
                std::fill(own.begin(), own.end(), 0.0f);
                std::fill(any.begin(), any.end(), 0.0f);
                int no = 0, na = 0;
                for (size_t yy = y > 0 ? y - 1 : 0; yy < std::min(y + 2, s.h); yy++)
                    for (size_t xx = x > 0 ? x - 1 : 0; xx < std::min(x + 2, s.w); xx++) {
                        size_t j = yy * s.w + xx;
                        if (!was[j]) continue;
                        if (s.chart[i] != 0xffffffffu && s.chart[j] == s.chart[i]) {
                            for (size_t c = 0; c < N; c++) own[c] += src[j * N + c];
                            no++;
                        } else {
                            for (size_t c = 0; c < N; c++) any[c] += src[j * N + c];
                            na++;
                        }
                    }
                if (no > 0) {
                    for (size_t c = 0; c < N; c++) v[i * N + c] = own[c] / float(no);
                    valid[i] = 1;
                } else if (na > 0 && s.chart[i] == 0xffffffffu) {
                    for (size_t c = 0; c < N; c++) v[i * N + c] = any[c] / float(na);
                    valid[i] = 1;
                }
            }
    }
}

std::vector<float> sun_field(const Surface &s, const std::vector<uint32_t> &hard, const std::vector<uint8_t> &covered,
                             size_t g, float radius) {
    size_t reach = size_t(std::ceil(radius)) + 1;
    std::vector<float> out(s.w * s.h, -1.0f);
    for (size_t y = 0; y < s.h; y++)
        for (size_t x = 0; x < s.w; x++) {
            size_t i = y * s.w + x;
            if (!covered[i]) continue;
            bool lit = size_t(__builtin_popcount(hard[i])) * 2 >= g * g;
            float best = radius;
            for (size_t yy = y > reach ? y - reach : 0; yy < std::min(y + reach + 1, s.h); yy++)
                for (size_t xx = x > reach ? x - reach : 0; xx < std::min(x + reach + 1, s.w); xx++) {
                    size_t j = yy * s.w + xx;
                    if (!covered[j] || !s.same(i, j)) continue;
                    for (size_t c = 0; c < g * g; c++) {
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
    return out;
}

}  // namespace lb
