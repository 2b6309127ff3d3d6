// A small JSON value: parse (the scene header) and write compactly in the order fields were added
// (the reference hashes serde_json's compact output of its settings, crates/lightbaker/src/deps.rs:60-68).
#pragma once
#include <cstdint>
#include <map>
#include <memory>
#include <string>
#include <utility>
#include <vector>

namespace lb {

struct Json {
    enum Kind { Null, Bool, Num, Str, Arr, Obj } kind = Null;
    bool b = false;
    double num = 0;
    bool is_f32 = false;  // written as the shortest f32 (serde_json writes an f32 field that way)
    bool is_int = false;
    std::string str;  // Str; for Num, the source text
    std::vector<Json> arr;
    std::vector<std::pair<std::string, Json>> obj;  // in order

    static Json parse(const std::string &text);  // throws std::runtime_error
    std::string dump() const;                     // compact, serde_json style

    const Json *get(const std::string &k) const;
    bool has(const std::string &k) const { return get(k) != nullptr; }
    const Json &at(const std::string &k) const;  // throws when missing
    Json &set(const std::string &k, Json v);

    static Json f32(float v);
    static Json u32(uint32_t v);
    static Json i64(long long v);
    static Json boolean(bool v);
    static Json string(const std::string &s);
    static Json array() { Json j; j.kind = Arr; return j; }
    static Json object() { Json j; j.kind = Obj; return j; }

    float as_f32() const;
    uint32_t as_u32() const;
    bool as_bool() const;
    const std::string &as_str() const;
};

// The shortest decimal that reads back as v (as an f32), written as Rust's ryu does: "1.0", "0.25",
// "1e-7", "1.5e20".
std::string format_f32(float v);

}  // namespace lb
