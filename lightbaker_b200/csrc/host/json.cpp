#include "json.h"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <stdexcept>

namespace lb {

namespace {
struct Parser {
    const std::string &s;
    size_t i = 0;
    explicit Parser(const std::string &t) : s(t) {}
    [[noreturn]] void fail(const char *what) {
        throw std::runtime_error(std::string("scene header: ") + what + " at byte " + std::to_string(i));
    }
    void ws() {
        while (i < s.size() && (s[i] == ' ' || s[i] == '\t' || s[i] == '\n' || s[i] == '\r')) i++;
    }
    bool lit(const char *w) {
        size_t n = strlen(w);
        if (s.compare(i, n, w) == 0) {
            i += n;
            return true;
        }
        return false;
    }
    static void put_utf8(std::string &out, uint32_t cp) {
        if (cp < 0x80) out += char(cp);
        else if (cp < 0x800) {
            out += char(0xc0 | (cp >> 6));
            out += char(0x80 | (cp & 0x3f));
        } else if (cp < 0x10000) {
            out += char(0xe0 | (cp >> 12));
            out += char(0x80 | ((cp >> 6) & 0x3f));
            out += char(0x80 | (cp & 0x3f));
        } else {
            out += char(0xf0 | (cp >> 18));
            out += char(0x80 | ((cp >> 12) & 0x3f));
            out += char(0x80 | ((cp >> 6) & 0x3f));
            out += char(0x80 | (cp & 0x3f));
        }
    }
    uint32_t hex4() {
        if (i + 4 > s.size()) fail("short \\u escape");
        uint32_t v = 0;
        for (int k = 0; k < 4; k++) {
            char c = s[i++];
            v <<= 4;
            if (c >= '0' && c <= '9') v |= c - '0';
            else if (c >= 'a' && c <= 'f') v |= c - 'a' + 10;
            else if (c >= 'A' && c <= 'F') v |= c - 'A' + 10;
            else fail("bad \\u escape");
        }
        return v;
    }
    std::string string() {
        if (s[i] != '"') fail("expected a string");
        i++;
        std::string out;
        while (true) {
            if (i >= s.size()) fail("unterminated string");
            char c = s[i++];
            if (c == '"') break;
            if ((unsigned char)c < 0x20) fail("control character in string");
            if (c != '\\') {
                out += c;
                continue;
            }
            if (i >= s.size()) fail("unterminated escape");
            char e = s[i++];
            switch (e) {
            case '"': out += '"'; break;
            case '\\': out += '\\'; break;
            case '/': out += '/'; break;
            case 'b': out += '\b'; break;
            case 'f': out += '\f'; break;
            case 'n': out += '\n'; break;
            case 'r': out += '\r'; break;
            case 't': out += '\t'; break;
            case 'u': {
                uint32_t cp = hex4();
                if (cp >= 0xd800 && cp < 0xdc00 && i + 6 <= s.size() && s[i] == '\\' && s[i + 1] == 'u') {
                    i += 2;
                    uint32_t lo = hex4();
                    cp = 0x10000 + ((cp - 0xd800) << 10) + (lo - 0xdc00);
                }
                put_utf8(out, cp);
                break;
            }
            default: fail("bad escape");
            }
        }
        return out;
    }
    Json value(int depth) {
        if (depth > 128) fail("nesting too deep");
        ws();
        if (i >= s.size()) fail("unexpected end");
        Json j;
        char c = s[i];
        if (c == '{') {
            i++;
            j.kind = Json::Obj;
            ws();
            if (i < s.size() && s[i] == '}') {
                i++;
                return j;
            }
            while (true) {
                ws();
                std::string k = string();
                ws();
                if (i >= s.size() || s[i] != ':') fail("expected ':'");
                i++;
                j.obj.emplace_back(k, value(depth + 1));
                ws();
                if (i < s.size() && s[i] == ',') {
                    i++;
                    continue;
                }
                if (i < s.size() && s[i] == '}') {
                    i++;
                    break;
                }
                fail("expected ',' or '}'");
            }
        } else if (c == '[') {
            i++;
            j.kind = Json::Arr;
            ws();
            if (i < s.size() && s[i] == ']') {
                i++;
                return j;
            }
            while (true) {
                j.arr.push_back(value(depth + 1));
                ws();
                if (i < s.size() && s[i] == ',') {
                    i++;
                    continue;
                }
                if (i < s.size() && s[i] == ']') {
                    i++;
                    break;
                }
                fail("expected ',' or ']'");
            }
        } else if (c == '"') {
            j.kind = Json::Str;
            j.str = string();
        } else if (lit("true")) {
            j.kind = Json::Bool;
            j.b = true;
        } else if (lit("false")) {
            j.kind = Json::Bool;
            j.b = false;
        } else if (lit("null")) {
            j.kind = Json::Null;
        } else if (c == '-' || (c >= '0' && c <= '9')) {
            size_t st = i;
            if (s[i] == '-') i++;
            bool intlike = true;
            while (i < s.size() && ((s[i] >= '0' && s[i] <= '9') || s[i] == '.' || s[i] == 'e' || s[i] == 'E' ||
                                    s[i] == '+' || s[i] == '-')) {
                if (s[i] == '.' || s[i] == 'e' || s[i] == 'E') intlike = false;
                i++;
            }
            j.kind = Json::Num;
            j.str = s.substr(st, i - st);
            char *end = nullptr;
            j.num = strtod(j.str.c_str(), &end);
            if (!end || *end) fail("bad number");
            j.is_int = intlike;
        } else {
            fail("unexpected character");
        }
        return j;
    }
};

void escape(std::string &out, const std::string &s) {
    out += '"';
    for (unsigned char c : s) {
        switch (c) {
        case '"': out += "\\\""; break;
        case '\\': out += "\\\\"; break;
        case '\n': out += "\\n"; break;
        case '\r': out += "\\r"; break;
        case '\t': out += "\\t"; break;
        case '\b': out += "\\b"; break;
        case '\f': out += "\\f"; break;
        default:
            if (c < 0x20) {
                char b[8];
                snprintf(b, sizeof b, "\\u%04x", c);
                out += b;
            } else {
                out += char(c);
            }
        }
    }
    out += '"';
}

void dump_to(const Json &j, std::string &out) {
    switch (j.kind) {
    case Json::Null: out += "null"; break;
    case Json::Bool: out += j.b ? "true" : "false"; break;
    case Json::Num:
        if (j.is_f32) out += format_f32(float(j.num));
        else if (j.is_int) {
            char b[32];
            snprintf(b, sizeof b, "%lld", (long long)j.num);
            out += b;
        } else {
            out += j.str.empty() ? format_f32(float(j.num)) : j.str;
        }
        break;
    case Json::Str: escape(out, j.str); break;
    case Json::Arr:
        out += '[';
        for (size_t k = 0; k < j.arr.size(); k++) {
            if (k) out += ',';
            dump_to(j.arr[k], out);
        }
        out += ']';
        break;
    case Json::Obj:
        out += '{';
        for (size_t k = 0; k < j.obj.size(); k++) {
            if (k) out += ',';
            escape(out, j.obj[k].first);
            out += ':';
            dump_to(j.obj[k].second, out);
        }
        out += '}';
        break;
    }
}
}  // namespace

Json Json::parse(const std::string &text) {
    Parser p(text);
    Json j = p.value(0);
    p.ws();
    if (p.i != text.size()) p.fail("trailing characters");
    return j;
}

std::string Json::dump() const {
    std::string out;
    dump_to(*this, out);
    return out;
}

const Json *Json::get(const std::string &k) const {
    if (kind != Obj) return nullptr;
    for (auto &kv : obj)
        if (kv.first == k) return &kv.second;
    return nullptr;
}

const Json &Json::at(const std::string &k) const {
    const Json *j = get(k);
    if (!j) throw std::runtime_error("scene header: missing field `" + k + "`");
    return *j;
}

Json &Json::set(const std::string &k, Json v) {
    kind = Obj;
    for (auto &kv : obj)
        if (kv.first == k) {
            kv.second = std::move(v);
            return kv.second;
        }
    obj.emplace_back(k, std::move(v));
    return obj.back().second;
}

Json Json::f32(float v) {
    Json j;
    j.kind = Num;
    j.num = v;
    j.is_f32 = true;
    return j;
}
Json Json::u32(uint32_t v) {
    Json j;
    j.kind = Num;
    j.num = v;
    j.is_int = true;
    return j;
}
Json Json::i64(long long v) {
    Json j;
    j.kind = Num;
    j.num = double(v);
    j.is_int = true;
    return j;
}
Json Json::boolean(bool v) {
    Json j;
    j.kind = Bool;
    j.b = v;
    return j;
}
Json Json::string(const std::string &s) {
    Json j;
    j.kind = Str;
    j.str = s;
    return j;
}

float Json::as_f32() const {
    if (kind != Num) throw std::runtime_error("scene header: expected a number");
    return float(num);
}
uint32_t Json::as_u32() const {
    if (kind != Num || !is_int || num < 0 || num > 4294967295.0)
        throw std::runtime_error("scene header: expected an unsigned integer, got " + (kind == Num ? str : dump()));
    return uint32_t(num);
}
bool Json::as_bool() const {
    if (kind != Bool) throw std::runtime_error("scene header: expected a boolean");
    return b;
}
const std::string &Json::as_str() const {
    if (kind != Str) throw std::runtime_error("scene header: expected a string");
    return str;
}

std::string format_f32(float v) {
    if (std::isnan(v) || std::isinf(v)) return "null";  // serde_json writes non-finite floats as null
    if (v == 0.0f) return std::signbit(v) ? "-0.0" : "0.0";
    // shortest round-trip digits
    char buf[64];
    int prec = 1;
    for (; prec <= 9; prec++) {
        snprintf(buf, sizeof buf, "%.*e", prec - 1, double(v));
        if (strtof(buf, nullptr) == v) break;
    }
    std::string sgn;
    const char *p = buf;
    if (*p == '-') {
        sgn = "-";
        p++;
    }
    std::string digits;
    const char *e = p;
    for (; *e && *e != 'e'; e++)
        if (*e != '.') digits += *e;
    int exp10 = atoi(e + 1);
    while (digits.size() > 1 && digits.back() == '0') digits.pop_back();
    int length = int(digits.size());
    int kk = exp10 + 1;  // 10^(kk-1) <= v < 10^kk
    int k = kk - length;
    std::string out = sgn;
    if (0 <= k && kk <= 13) {
        out += digits + std::string(size_t(k), '0') + ".0";
    } else if (0 < kk && kk <= 13) {
        out += digits.substr(0, size_t(kk)) + "." + digits.substr(size_t(kk));
    } else if (-6 < kk && kk <= 0) {
        out += "0." + std::string(size_t(-kk), '0') + digits;
    } else if (length == 1) {
        out += digits + "e" + std::to_string(kk - 1);
    } else {
        out += digits.substr(0, 1) + "." + digits.substr(1) + "e" + std::to_string(kk - 1);
    }
    return out;
}

}  // namespace lb
