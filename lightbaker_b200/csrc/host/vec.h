// Host vectors with the arithmetic of the reference's host math library (glam 0.34 Vec2/Vec3, scalar
// f32, no fused multiply-add): dot and length summed left to right, normalize as v * (1 / length).
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>
#if defined(__SSE2__)
#include <emmintrin.h>
#endif

namespace lb {

// std::fmin / std::fmax as the C library computes them (the non-NaN argument when one is NaN, the first
// of two equal values, so +0 or -0 as given), written out so that the compiler inlines them: the BVH
// build and the layout call them for every primitive of every node. On x86 the choice is made with
// SSE masks rather than branches (a box's bound moves with no pattern a branch predictor can follow).
#if defined(__SSE2__)
inline float fmin_(float a, float b) {
    const __m128 va = _mm_set_ss(a), vb = _mm_set_ss(b);
    const __m128 take_b = _mm_or_ps(_mm_cmplt_ss(vb, va), _mm_cmpunord_ss(va, va));
    return _mm_cvtss_f32(_mm_or_ps(_mm_and_ps(take_b, vb), _mm_andnot_ps(take_b, va)));
}
inline float fmax_(float a, float b) {
    const __m128 va = _mm_set_ss(a), vb = _mm_set_ss(b);
    const __m128 take_b = _mm_or_ps(_mm_cmpgt_ss(vb, va), _mm_cmpunord_ss(va, va));
    return _mm_cvtss_f32(_mm_or_ps(_mm_and_ps(take_b, vb), _mm_andnot_ps(take_b, va)));
}
#else
inline float fmin_(float a, float b) { return (b < a || a != a) ? b : a; }
inline float fmax_(float a, float b) { return (b > a || a != a) ? b : a; }
#endif

struct Vec2 {
    float x = 0, y = 0;
    Vec2() = default;
    Vec2(float a, float b) : x(a), y(b) {}
    Vec2 operator+(Vec2 o) const { return {x + o.x, y + o.y}; }
    Vec2 operator-(Vec2 o) const { return {x - o.x, y - o.y}; }
    Vec2 operator*(float s) const { return {x * s, y * s}; }
    float dot(Vec2 o) const { return x * o.x + y * o.y; }
    float perp_dot(Vec2 o) const { return x * o.y - y * o.x; }
    float length_squared() const { return dot(*this); }
    float distance_squared(Vec2 o) const { return (*this - o).length_squared(); }
    Vec2 min(Vec2 o) const { return {fmin_(x, o.x), fmin_(y, o.y)}; }
    Vec2 max(Vec2 o) const { return {fmax_(x, o.x), fmax_(y, o.y)}; }
    Vec2 floor() const { return {std::floor(x), std::floor(y)}; }
    Vec2 ceil() const { return {std::ceil(x), std::ceil(y)}; }
};

struct Vec3 {
    float x = 0, y = 0, z = 0;
    Vec3() = default;
    Vec3(float a, float b, float c) : x(a), y(b), z(c) {}
    static Vec3 splat(float v) { return {v, v, v}; }
    float operator[](int i) const { return i == 0 ? x : i == 1 ? y : z; }
    float &operator[](int i) { return i == 0 ? x : i == 1 ? y : z; }
    Vec3 operator+(Vec3 o) const { return {x + o.x, y + o.y, z + o.z}; }
    Vec3 operator-(Vec3 o) const { return {x - o.x, y - o.y, z - o.z}; }
    Vec3 operator-(float s) const { return {x - s, y - s, z - s}; }
    Vec3 operator+(float s) const { return {x + s, y + s, z + s}; }
    Vec3 operator*(float s) const { return {x * s, y * s, z * s}; }
    Vec3 operator/(float s) const { return {x / s, y / s, z / s}; }
    Vec3 &operator+=(Vec3 o) {
        x += o.x;
        y += o.y;
        z += o.z;
        return *this;
    }
    float dot(Vec3 o) const { return x * o.x + y * o.y + z * o.z; }
    Vec3 cross(Vec3 o) const { return {y * o.z - o.y * z, z * o.x - o.z * x, x * o.y - o.x * y}; }
    float length_squared() const { return dot(*this); }
    float length() const { return std::sqrt(dot(*this)); }
    Vec3 normalize() const { return *this * (1.0f / length()); }
    // glam try_normalize: None when 1/length is not finite and positive
    bool try_normalize(Vec3 &out) const {
        float r = 1.0f / length();
        if (std::isfinite(r) && r > 0.0f) {
            out = *this * r;
            return true;
        }
        return false;
    }
    Vec3 min(Vec3 o) const { return {fmin_(x, o.x), fmin_(y, o.y), fmin_(z, o.z)}; }
    Vec3 max(Vec3 o) const { return {fmax_(x, o.x), fmax_(y, o.y), fmax_(z, o.z)}; }
};

inline uint32_t f2u(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    return u;
}
inline float u2f(uint32_t u) {
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}

}  // namespace lb
