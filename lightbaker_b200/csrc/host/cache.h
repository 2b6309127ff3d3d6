// Baked tiles and probe chunks kept by their hash: crates/lightbaker/src/cache.rs. `<kind>-<hex>.bin`,
// zstd-compressed (level 3), written to a temporary file and renamed; a missing or unreadable entry
// is a miss. zstd is the system's libzstd, opened at run time (no headers on this image).
#pragma once
#include <cstring>
#include <optional>
#include <string>
#include <vector>

#include "deps.h"

namespace lb {

struct Cache {
    std::string dir;  // empty: no cache
    explicit Cache(const std::string &d);
    std::optional<std::vector<uint8_t>> get(const std::string &kind, const Hash &h) const;
    void put(const std::string &kind, const Hash &h, const std::vector<uint8_t> &bytes) const;  // throws
};

// zstd through the system library (throws when it cannot be loaded)
std::vector<uint8_t> zstd_compress(const uint8_t *data, size_t len, int level);
std::optional<std::vector<uint8_t>> zstd_decompress(const uint8_t *data, size_t len);

// cache.rs:41-62: arrays end to end, each after its byte length (u64)
struct Pack {
    std::vector<uint8_t> bytes;
    template <class T> Pack &put(const std::vector<T> &v) {
        uint64_t n = v.size() * sizeof(T);
        const uint8_t *p = (const uint8_t *)&n;
        bytes.insert(bytes.end(), p, p + 8);
        const uint8_t *b = (const uint8_t *)v.data();
        bytes.insert(bytes.end(), b, b + n);
        return *this;
    }
};
struct Unpack {
    const uint8_t *p;
    size_t left;
    template <class T> bool take(std::vector<T> &out) {
        if (left < 8) return false;
        uint64_t n;
        std::memcpy(&n, p, 8);
        if (n > left - 8 || n % sizeof(T)) return false;
        out.resize(n / sizeof(T));
        std::memcpy(out.data(), p + 8, n);
        p += 8 + n;
        left -= 8 + n;
        return true;
    }
};

}  // namespace lb
