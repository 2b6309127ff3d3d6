#include "blake3.h"

#include <algorithm>
#include <array>
#include <cstring>
#include <vector>

namespace lb {

namespace {
const uint32_t IV[8] = {0x6A09E667u, 0xBB67AE85u, 0x3C6EF372u, 0xA54FF53Au,
                        0x510E527Fu, 0x9B05688Cu, 0x1F83D9ABu, 0x5BE0CD19u};
const uint8_t PERM[16] = {2, 6, 3, 10, 7, 0, 4, 13, 1, 11, 12, 5, 9, 14, 15, 8};
enum : uint32_t { CHUNK_START = 1, CHUNK_END = 2, PARENT = 4, ROOT = 8 };
const size_t CHUNK = 1024;

inline uint32_t rotr(uint32_t x, int n) { return (x >> n) | (x << (32 - n)); }
inline void g(uint32_t *s, int a, int b, int c, int d, uint32_t x, uint32_t y) {
    s[a] = s[a] + s[b] + x;
    s[d] = rotr(s[d] ^ s[a], 16);
    s[c] = s[c] + s[d];
    s[b] = rotr(s[b] ^ s[c], 12);
    s[a] = s[a] + s[b] + y;
    s[d] = rotr(s[d] ^ s[a], 8);
    s[c] = s[c] + s[d];
    s[b] = rotr(s[b] ^ s[c], 7);
}
// the compression function: 7 rounds of column then diagonal mixing, the message permuted between rounds
void compress(const uint32_t cv[8], const uint32_t block[16], uint64_t counter, uint32_t len, uint32_t flags,
              uint32_t out[16]) {
    uint32_t s[16] = {cv[0], cv[1], cv[2], cv[3], cv[4], cv[5], cv[6], cv[7], IV[0], IV[1], IV[2], IV[3],
                      uint32_t(counter), uint32_t(counter >> 32), len, flags};
    uint32_t m[16], t[16];
    std::memcpy(m, block, 64);
    for (int r = 0; r < 7; r++) {
        g(s, 0, 4, 8, 12, m[0], m[1]);
        g(s, 1, 5, 9, 13, m[2], m[3]);
        g(s, 2, 6, 10, 14, m[4], m[5]);
        g(s, 3, 7, 11, 15, m[6], m[7]);
        g(s, 0, 5, 10, 15, m[8], m[9]);
        g(s, 1, 6, 11, 12, m[10], m[11]);
        g(s, 2, 7, 8, 13, m[12], m[13]);
        g(s, 3, 4, 9, 14, m[14], m[15]);
        if (r < 6) {
            for (int k = 0; k < 16; k++) t[k] = m[PERM[k]];
            std::memcpy(m, t, 64);
        }
    }
    for (int k = 0; k < 8; k++) {
        out[k] = s[k] ^ s[k + 8];
        out[k + 8] = s[k + 8] ^ cv[k];
    }
}
void words(const uint8_t *b, uint32_t *w) {
    for (int k = 0; k < 16; k++)
        w[k] = uint32_t(b[4 * k]) | uint32_t(b[4 * k + 1]) << 8 | uint32_t(b[4 * k + 2]) << 16 | uint32_t(b[4 * k + 3]) << 24;
}
void parent_cv(const uint32_t l[8], const uint32_t r[8], uint32_t flags, uint32_t out[8]) {
    uint32_t block[16], o[16];
    std::memcpy(block, l, 32);
    std::memcpy(block + 8, r, 32);
    compress(IV, block, 0, 64, PARENT | flags, o);
    std::memcpy(out, o, 32);
}
}  // namespace

Blake3::Blake3() { std::memcpy(cv_, IV, 32); }

void Blake3::compress_chunk_block(bool last, uint32_t out_cv[8]) {
    uint32_t w[16], o[16];
    uint8_t b[64] = {0};
    std::memcpy(b, block_, block_len_);
    words(b, w);
    uint32_t flags = (blocks_compressed_ == 0 ? CHUNK_START : 0) | (last ? CHUNK_END : 0);
    compress(cv_, w, chunk_counter_, uint32_t(block_len_), flags, o);
    std::memcpy(out_cv, o, 32);
}

// merge completed subtrees: after chunk `total_chunks`, one merge a trailing zero bit of its count
void Blake3::push_chunk_cv(const uint32_t cv[8], uint64_t total) {
    uint32_t cur[8];
    std::memcpy(cur, cv, 32);
    while ((total & 1) == 0) {
        stack_len_--;
        parent_cv(stack_[stack_len_], cur, 0, cur);
        total >>= 1;
    }
    std::memcpy(stack_[stack_len_++], cur, 32);
}

void Blake3::update(const void *data, size_t len) {
    const uint8_t *p = (const uint8_t *)data;
    while (len > 0) {
        size_t chunk_bytes = blocks_compressed_ * 64 + block_len_;
        if (chunk_bytes == CHUNK) {
            // the chunk is complete and more input follows: its last block was held back; finish it
            uint32_t cv[8];
            compress_chunk_block(true, cv);
            push_chunk_cv(cv, chunk_counter_ + 1);
            chunk_counter_++;
            std::memcpy(cv_, IV, 32);
            blocks_compressed_ = 0;
            block_len_ = 0;
            continue;
        }
        if (block_len_ == 64) {
            uint32_t cv[8];
            compress_chunk_block(false, cv);
            std::memcpy(cv_, cv, 32);
            blocks_compressed_++;
            block_len_ = 0;
            continue;
        }
        size_t take = 64 - block_len_;
        if (take > len) take = len;
        std::memcpy(block_ + block_len_, p, take);
        block_len_ += take;
        p += take;
        len -= take;
    }
}

void Blake3::finalize(uint8_t out[32]) const {
    // the current chunk's output (the root when it is the only chunk), folded with the stack right to left
    uint32_t w[16], o[16];
    uint8_t b[64] = {0};
    std::memcpy(b, block_, block_len_);
    words(b, w);
    uint32_t flags = (blocks_compressed_ == 0 ? CHUNK_START : 0) | CHUNK_END;
    uint32_t in_cv[8];
    std::memcpy(in_cv, cv_, 32);
    uint64_t counter = chunk_counter_;
    uint32_t blen = uint32_t(block_len_);
    size_t n = stack_len_;
    while (n > 0) {
        // the node so far is a child: its chaining value, then its parent with the next stack entry
        uint32_t child[8];
        compress(in_cv, w, counter, blen, flags, o);
        std::memcpy(child, o, 32);
        n--;
        uint32_t block[16];
        std::memcpy(block, stack_[n], 32);
        std::memcpy(block + 8, child, 32);
        std::memcpy(w, block, 64);
        std::memcpy(in_cv, IV, 32);
        counter = 0;
        blen = 64;
        flags = PARENT;
    }
    compress(in_cv, w, counter, blen, flags | ROOT, o);
    for (int k = 0; k < 8; k++) {
        out[4 * k] = uint8_t(o[k]);
        out[4 * k + 1] = uint8_t(o[k] >> 8);
        out[4 * k + 2] = uint8_t(o[k] >> 16);
        out[4 * k + 3] = uint8_t(o[k] >> 24);
    }
}

std::string to_hex(const uint8_t *h, size_t n) {
    static const char *d = "0123456789abcdef";
    std::string s;
    for (size_t k = 0; k < n; k++) {
        s += d[h[k] >> 4];
        s += d[h[k] & 15];
    }
    return s;
}

std::string Blake3::hex() const {
    uint8_t h[32];
    finalize(h);
    return to_hex(h, 32);
}

namespace {
// chunk `index` of `data` (1 to 1024 bytes): its chaining value, or (root) the root output's first words
void chunk_cv(const uint8_t *p, size_t bytes, uint64_t index, bool root, uint32_t out[8]) {
    uint32_t cv[8], w[16], o[16];
    std::memcpy(cv, IV, 32);
    const size_t blocks = bytes == 0 ? 1 : (bytes + 63) / 64;
    for (size_t b = 0; b < blocks; b++) {
        const size_t blen = b + 1 < blocks ? 64 : bytes - b * 64;
        uint8_t block[64] = {0};
        std::memcpy(block, p + b * 64, blen);
        words(block, w);
        const uint32_t flags =
            (b == 0 ? CHUNK_START : 0) | (b + 1 == blocks ? CHUNK_END : 0) | (root && b + 1 == blocks ? ROOT : 0);
        compress(cv, w, index, uint32_t(blen), flags, o);
        std::memcpy(cv, o, 32);
    }
    std::memcpy(out, cv, 32);
}
}  // namespace

// One call over the whole input. From 64 KiB on, the chunks' chaining values are computed in parallel
// and merged pair by pair, level by level (an odd last node goes up as it is): that builds the same
// left-balanced tree the incremental hasher folds (every left subtree the largest power of two of chunks
// below the node's count), so the digest is the same.
void blake3_hash(const void *data, size_t len, uint8_t out[32]) {
    const size_t chunks = (len + CHUNK - 1) / CHUNK;
    if (len < (size_t(64) << 10) || chunks < 2) {
        Blake3 h;
        h.update(data, len);
        h.finalize(out);
        return;
    }
    const uint8_t *p = (const uint8_t *)data;
    std::vector<std::array<uint32_t, 8>> level(chunks);
#pragma omp parallel for schedule(static)
    for (long long c = 0; c < (long long)chunks; c++) {
        const size_t at = size_t(c) * CHUNK;
        chunk_cv(p + at, std::min(CHUNK, len - at), uint64_t(c), false, level[size_t(c)].data());
    }
    while (level.size() > 2) {
        std::vector<std::array<uint32_t, 8>> up((level.size() + 1) / 2);
#pragma omp parallel for schedule(static) if (level.size() > 4096)
        for (long long k = 0; k < (long long)(level.size() / 2); k++)
            parent_cv(level[2 * size_t(k)].data(), level[2 * size_t(k) + 1].data(), 0, up[size_t(k)].data());
        if (level.size() % 2) up.back() = level.back();
        level.swap(up);
    }
    uint32_t root[8];
    parent_cv(level[0].data(), level[1].data(), ROOT, root);
    for (int k = 0; k < 8; k++) {
        out[4 * k] = uint8_t(root[k]);
        out[4 * k + 1] = uint8_t(root[k] >> 8);
        out[4 * k + 2] = uint8_t(root[k] >> 16);
        out[4 * k + 3] = uint8_t(root[k] >> 24);
    }
}

}  // namespace lb
