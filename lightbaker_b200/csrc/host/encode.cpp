#include "encode.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <stdexcept>

#include "cache.h"

namespace lb {

std::array<uint8_t, 8> bc4_block(const uint8_t v[16]) {
    uint8_t hi = *std::max_element(v, v + 16), lo = *std::min_element(v, v + 16);
    std::array<uint8_t, 8> out{};
    out[0] = hi;
    out[1] = lo;
    if (hi == lo) return out;
    // hi > lo: index 0 is hi, 1 is lo, 2..7 from hi to lo in sevenths
    float pal[8];
    for (int i = 0; i < 8; i++)
        pal[i] = i == 0 ? float(hi) : i == 1 ? float(lo) : (float(8 - i) * float(hi) + float(i - 1) * float(lo)) / 7.0f;
    uint64_t bits = 0;
    for (int k = 0; k < 16; k++) {
        int best = 0;
        for (int i = 1; i < 8; i++)
            if (std::fabs(pal[i] - float(v[k])) < std::fabs(pal[best] - float(v[k]))) best = i;
        bits |= uint64_t(best) << (3 * k);
    }
    for (int b = 0; b < 6; b++) out[2 + b] = uint8_t(bits >> (8 * b));
    return out;
}

std::vector<uint8_t> bc5(const uint8_t *rg, size_t w, size_t h) {
    if (w % 4 || h % 4) throw std::runtime_error("bc5: size not a multiple of 4");
    std::vector<uint8_t> out;
    out.reserve(w * h);
    uint8_t block[16];
    for (size_t by = 0; by < h; by += 4)
        for (size_t bx = 0; bx < w; bx += 4)
            for (int c = 0; c < 2; c++) {
                for (int k = 0; k < 16; k++) block[k] = rg[((by + k / 4) * w + bx + k % 4) * 2 + c];
                auto b = bc4_block(block);
                out.insert(out.end(), b.begin(), b.end());
            }
    return out;
}

uint32_t rgb9e5(const float c[3]) {
    const float MAX = 65408.0f;
    float r = std::min(std::max(c[0], 0.0f), MAX), g = std::min(std::max(c[1], 0.0f), MAX),
          b = std::min(std::max(c[2], 0.0f), MAX);
    float m = std::fmax(std::fmax(r, g), b);
    if (m <= 0.0f) return 0;
    int e = std::max(int(std::floor(std::log2(m))), -16) + 1 + 15;
    float scale = std::ldexp(1.0f, e - 15 - 9);
    if (uint32_t(std::floor(m / scale + 0.5f)) == 512) {
        e += 1;
        scale *= 2.0f;
    }
    auto q = [&](float v) { return std::min(uint32_t(std::floor(v / scale + 0.5f)), 511u); };
    return q(r) | (q(g) << 9) | (q(b) << 18) | (uint32_t(e) << 27);
}

void rgb9e5_decode(uint32_t p, float out[3]) {
    float s = std::ldexp(1.0f, int(p >> 27) - 15 - 9);
    out[0] = float(p & 511) * s;
    out[1] = float((p >> 9) & 511) * s;
    out[2] = float((p >> 18) & 511) * s;
}

namespace {
void put32(std::vector<uint8_t> &o, uint32_t v) { o.insert(o.end(), (uint8_t *)&v, (uint8_t *)&v + 4); }
void put64(std::vector<uint8_t> &o, uint64_t v) { o.insert(o.end(), (uint8_t *)&v, (uint8_t *)&v + 8); }
void put16(std::vector<uint8_t> &o, uint16_t v) { o.insert(o.end(), (uint8_t *)&v, (uint8_t *)&v + 2); }

// encode.rs:128-148: the basic data format descriptor (Khronos Data Format 1.3), linear, BT.709
std::vector<uint8_t> dfd(Format f) {
    struct S {
        uint16_t off;
        uint8_t len, ch;
    };
    uint8_t model, bytes;
    std::array<uint8_t, 4> dims;
    std::vector<S> samples;
    if (f == FORMAT_BC5) {
        model = 133, dims = {3, 3, 0, 0}, bytes = 16, samples = {{0, 63, 0}, {64, 63, 1}};
    } else {
        model = 1, dims = {0, 0, 0, 0}, bytes = 4, samples = {{0, 8, 0}, {9, 8, 1}, {18, 8, 2}};
    }
    size_t block = 24 + 16 * samples.size();
    std::vector<uint8_t> d;
    put32(d, uint32_t(4 + block));
    put32(d, 0);
    put16(d, 2);
    put16(d, uint16_t(block));
    d.insert(d.end(), {model, 1, 1, 0});
    d.insert(d.end(), dims.begin(), dims.end());
    d.insert(d.end(), {bytes, 0, 0, 0, 0, 0, 0, 0});
    for (auto &s : samples) {
        put16(d, s.off);
        d.insert(d.end(), {s.len, s.ch});
        d.insert(d.end(), {0, 0, 0, 0});
        put32(d, 0);
        put32(d, 0xffffffffu);
    }
    return d;
}
}  // namespace

std::vector<uint8_t> ktx2(Format f, uint32_t w, uint32_t h, const std::vector<uint8_t> &data) {
    std::vector<uint8_t> packed = zstd_compress(data.data(), data.size(), 19);
    std::vector<uint8_t> d = dfd(f);
    const size_t HEADER = 12 + 9 * 4 + 4 * 4 + 2 * 8, LEVELS = 3 * 8;
    size_t dfd_at = HEADER + LEVELS;
    size_t data_at = (dfd_at + d.size() + 7) / 8 * 8;
    std::vector<uint8_t> out{0xAB, 0x4B, 0x54, 0x58, 0x20, 0x32, 0x30, 0xBB, 0x0D, 0x0A, 0x1A, 0x0A};
    uint32_t vk = f == FORMAT_BC5 ? 141 : 123, ts = f == FORMAT_BC5 ? 1 : 4;
    for (uint32_t v : {vk, ts, w, h, 0u, 0u, 1u, 1u, 2u}) put32(out, v);
    for (uint32_t v : {uint32_t(dfd_at), uint32_t(d.size()), 0u, 0u}) put32(out, v);
    put64(out, 0);
    put64(out, 0);
    for (uint64_t v : {uint64_t(data_at), uint64_t(packed.size()), uint64_t(data.size())}) put64(out, v);
    out.insert(out.end(), d.begin(), d.end());
    out.resize(data_at, 0);
    out.insert(out.end(), packed.begin(), packed.end());
    return out;
}

}  // namespace lb
