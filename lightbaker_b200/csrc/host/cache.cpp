#include "cache.h"

#include <dlfcn.h>
#include <sys/stat.h>

#include <cstdio>
#include <stdexcept>

namespace lb {

namespace {
// The handful of public zstd entry points used, declared here (names and signatures from zstd.h 1.5)
struct Zstd {
    size_t (*compressBound)(size_t);
    size_t (*compress)(void *, size_t, const void *, size_t, int);
    unsigned (*isError)(size_t);
    const char *(*getErrorName)(size_t);
    void *(*createDCtx)();
    size_t (*freeDCtx)(void *);
    size_t (*decompressStream)(void *, void *, void *);  // (ctx, ZSTD_outBuffer*, ZSTD_inBuffer*)
    bool ok = false;
};
struct InBuf {
    const void *src;
    size_t size, pos;
};
struct OutBuf {
    void *dst;
    size_t size, pos;
};
const Zstd &zstd() {
    static Zstd z = [] {
        Zstd z{};
        void *h = dlopen("libzstd.so.1", RTLD_NOW | RTLD_LOCAL);
        if (!h) return z;
        z.compressBound = (size_t(*)(size_t))dlsym(h, "ZSTD_compressBound");
        z.compress = (size_t(*)(void *, size_t, const void *, size_t, int))dlsym(h, "ZSTD_compress");
        z.isError = (unsigned (*)(size_t))dlsym(h, "ZSTD_isError");
        z.getErrorName = (const char *(*)(size_t))dlsym(h, "ZSTD_getErrorName");
        z.createDCtx = (void *(*)())dlsym(h, "ZSTD_createDCtx");
        z.freeDCtx = (size_t(*)(void *))dlsym(h, "ZSTD_freeDCtx");
        z.decompressStream = (size_t(*)(void *, void *, void *))dlsym(h, "ZSTD_decompressStream");
        z.ok = z.compressBound && z.compress && z.isError && z.getErrorName && z.createDCtx && z.freeDCtx &&
               z.decompressStream;
        return z;
    }();
    return z;
}
void mkdirs(const std::string &d) {
    std::string cur;
    for (size_t i = 0; i <= d.size(); i++) {
        if (i == d.size() || d[i] == '/') {
            if (!cur.empty()) mkdir(cur.c_str(), 0777);
        }
        if (i < d.size()) cur += d[i];
    }
    struct stat st;
    if (stat(d.c_str(), &st) != 0 || !S_ISDIR(st.st_mode)) throw std::runtime_error("cache: cannot create " + d);
}
}  // namespace

std::vector<uint8_t> zstd_compress(const uint8_t *data, size_t len, int level) {
    const Zstd &z = zstd();
    if (!z.ok) throw std::runtime_error("zstd: libzstd.so.1 not found");
    std::vector<uint8_t> out(z.compressBound(len));
    size_t n = z.compress(out.data(), out.size(), data, len, level);
    if (z.isError(n)) throw std::runtime_error(std::string("zstd: ") + z.getErrorName(n));
    out.resize(n);
    return out;
}

std::optional<std::vector<uint8_t>> zstd_decompress(const uint8_t *data, size_t len) {
    const Zstd &z = zstd();
    if (!z.ok) return std::nullopt;
    void *ctx = z.createDCtx();
    std::vector<uint8_t> out;
    std::vector<uint8_t> buf(1 << 17);
    InBuf in{data, len, 0};
    size_t last = 1;
    while (in.pos < in.size || last != 0) {
        OutBuf o{buf.data(), buf.size(), 0};
        size_t before = in.pos;
        last = z.decompressStream(ctx, &o, &in);
        if (z.isError(last)) {
            z.freeDCtx(ctx);
            return std::nullopt;
        }
        out.insert(out.end(), buf.begin(), buf.begin() + o.pos);
        if (o.pos == 0 && in.pos == before) {
            if (in.pos >= in.size) break;  // truncated frame
        }
    }
    z.freeDCtx(ctx);
    if (last != 0) return std::nullopt;
    return out;
}

Cache::Cache(const std::string &d) : dir(d) {
    if (!dir.empty()) mkdirs(dir);
}

std::optional<std::vector<uint8_t>> Cache::get(const std::string &kind, const Hash &h) const {
    if (dir.empty()) return std::nullopt;
    std::string f = dir + "/" + kind + "-" + to_hex(h.data(), 32) + ".bin";
    FILE *fp = fopen(f.c_str(), "rb");
    if (!fp) return std::nullopt;
    std::vector<uint8_t> raw;
    uint8_t b[1 << 16];
    size_t n;
    while ((n = fread(b, 1, sizeof b, fp)) > 0) raw.insert(raw.end(), b, b + n);
    fclose(fp);
    return zstd_decompress(raw.data(), raw.size());
}

void Cache::put(const std::string &kind, const Hash &h, const std::vector<uint8_t> &bytes) const {
    if (dir.empty()) return;
    std::string f = dir + "/" + kind + "-" + to_hex(h.data(), 32) + ".bin";
    std::string tmp = dir + "/" + kind + "-" + to_hex(h.data(), 32) + ".tmp";
    std::vector<uint8_t> z = zstd_compress(bytes.data(), bytes.size(), 3);
    FILE *fp = fopen(tmp.c_str(), "wb");
    if (!fp) throw std::runtime_error("cache: cannot write " + tmp);
    bool ok = fwrite(z.data(), 1, z.size(), fp) == z.size();
    ok = (fclose(fp) == 0) && ok;
    if (!ok || rename(tmp.c_str(), f.c_str()) != 0) throw std::runtime_error("cache: cannot write " + f);
}

}  // namespace lb
