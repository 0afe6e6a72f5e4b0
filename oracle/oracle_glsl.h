// oracle_glsl.h - GLSL value semantics for the CPU oracle.
//
// TEST INFRASTRUCTURE ONLY. This directory is the CPU oracle of the hdcx
// integrator: a function-for-function C++ restatement of hdCodex's GLSL
// path tracer (src/gpu/vulkan_path_tracer.cpp:100-1891) and its host-side
// scene packing (:1961-2066, :2604-2993). Only the tests, the smoke check and
// the benchmark's CPU-baseline leg may load it, as the checker. The product
// (hdcodex_b200/) never includes, links or calls anything here.
//
// Arithmetic contract (shared with the CUDA integrator, which restates the same
// functions independently):
//   * every float operation is a single IEEE-754 binary32 operation in the
//     order the GLSL source writes it (left to right), with no fused
//     multiply-add: this file is compiled with -ffp-contract=off;
//   * dot(a, b) = (a.x*b.x + a.y*b.y) + a.z*b.z; length = sqrt(dot);
//     normalize(v) = v * (1 / sqrt(dot(v, v)));
//   * mix, clamp, smoothstep, reflect, refract and fract follow the GLSL 4.60
//     specification formulas;
//   * transcendentals (exp, log, pow, sin, cos, acos, atan) are the binary32
//     functions of hdcx/fpmath.h: fixed sequences of binary32 operations and
//     fused multiply-adds (fmaf), bit-identical on host and device; pow(x, 2)
//     is x * x and pow(x, 5) is x^5 in exact binary64 products.
#pragma once

#include <cmath>
#include <cstdint>

#include "hdcx/fpmath.h"

namespace oracle {

struct vec2 {
    float x, y;
};
struct vec3 {
    float x, y, z;
};
struct vec4 {
    float x, y, z, w;
};
struct ivec2 {
    int x, y;
};

inline vec2 V2(float x, float y) { return {x, y}; }
inline vec3 V3(float s) { return {s, s, s}; }
inline vec3 V3(float x, float y, float z) { return {x, y, z}; }
inline vec4 V4(float s) { return {s, s, s, s}; }
inline vec4 V4(float x, float y, float z, float w) { return {x, y, z, w}; }
inline vec4 V4(vec3 v, float w) { return {v.x, v.y, v.z, w}; }
inline vec3 xyz(vec4 v) { return {v.x, v.y, v.z}; }

inline vec2 operator+(vec2 a, vec2 b) { return {a.x + b.x, a.y + b.y}; }
inline vec2 operator-(vec2 a, vec2 b) { return {a.x - b.x, a.y - b.y}; }
inline vec2 operator*(vec2 a, float s) { return {a.x * s, a.y * s}; }
inline vec2 operator*(float s, vec2 a) { return {s * a.x, s * a.y}; }
inline vec2 operator*(vec2 a, vec2 b) { return {a.x * b.x, a.y * b.y}; }
inline vec2 operator/(vec2 a, vec2 b) { return {a.x / b.x, a.y / b.y}; }

inline vec3 operator+(vec3 a, vec3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline vec3 operator-(vec3 a, vec3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline vec3 operator-(vec3 a) { return {-a.x, -a.y, -a.z}; }
inline vec3 operator*(vec3 a, vec3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
inline vec3 operator*(vec3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
inline vec3 operator*(float s, vec3 a) { return {s * a.x, s * a.y, s * a.z}; }
inline vec3 operator/(vec3 a, vec3 b) { return {a.x / b.x, a.y / b.y, a.z / b.z}; }
inline vec3 operator/(vec3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
inline vec3& operator+=(vec3& a, vec3 b) { a = a + b; return a; }
inline vec3& operator*=(vec3& a, vec3 b) { a = a * b; return a; }
inline vec3& operator*=(vec3& a, float s) { a = a * s; return a; }
inline vec3& operator/=(vec3& a, float s) { a = a / s; return a; }

inline float dot(vec3 a, vec3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline float dot(vec2 a, vec2 b) { return a.x * b.x + a.y * b.y; }
inline vec3 cross(vec3 a, vec3 b)
{
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
inline float length(vec3 v) { return std::sqrt(dot(v, v)); }
inline float length(vec2 v) { return std::sqrt(dot(v, v)); }
inline vec3 normalize(vec3 v)
{
    const float inverse = 1.0f / std::sqrt(dot(v, v));
    return v * inverse;
}
inline vec2 normalize(vec2 v)
{
    const float inverse = 1.0f / std::sqrt(dot(v, v));
    return v * inverse;
}
inline float inversesqrt(float x) { return 1.0f / std::sqrt(x); }

// GLSL min/max/clamp: min(x, y) = y < x ? y : x, max(x, y) = x < y ? y : x.
inline float gmin(float x, float y) { return y < x ? y : x; }
inline float gmax(float x, float y) { return x < y ? y : x; }
inline float clampf(float x, float lo, float hi) { return gmin(gmax(x, lo), hi); }
inline vec3 gmax(vec3 a, vec3 b) { return {gmax(a.x, b.x), gmax(a.y, b.y), gmax(a.z, b.z)}; }
inline vec3 clamp3(vec3 v, vec3 lo, vec3 hi)
{
    return {clampf(v.x, lo.x, hi.x), clampf(v.y, lo.y, hi.y), clampf(v.z, lo.z, hi.z)};
}
inline vec2 clamp2(vec2 v, vec2 lo, vec2 hi)
{
    return {clampf(v.x, lo.x, hi.x), clampf(v.y, lo.y, hi.y)};
}
inline float absf(float x) { return std::fabs(x); }
inline vec3 abs3(vec3 v) { return {std::fabs(v.x), std::fabs(v.y), std::fabs(v.z)}; }
inline float fract(float x) { return x - std::floor(x); }
inline vec2 fract(vec2 v) { return {fract(v.x), fract(v.y)}; }
// mix(x, y, a) = x * (1 - a) + y * a
inline float mix(float x, float y, float a) { return x * (1.0f - a) + y * a; }
inline vec3 mix(vec3 x, vec3 y, float a) { return x * (1.0f - a) + y * a; }
inline float smoothstep(float e0, float e1, float x)
{
    const float t = clampf((x - e0) / (e1 - e0), 0.0f, 1.0f);
    return t * t * (3.0f - 2.0f * t);
}
// reflect(I, N) = I - 2 * dot(N, I) * N
inline vec3 reflect(vec3 i, vec3 n) { return i - 2.0f * dot(n, i) * n; }
// refract(I, N, eta): k = 1 - eta^2 (1 - dot(N, I)^2); k < 0 -> 0 else
// eta * I - (eta * dot(N, I) + sqrt(k)) * N
inline vec3 refract(vec3 i, vec3 n, float eta)
{
    const float d = dot(n, i);
    const float k = 1.0f - eta * eta * (1.0f - d * d);
    if (k < 0.0f) return V3(0.0f);
    return eta * i - (eta * d + std::sqrt(k)) * n;
}
inline bool anyGreaterThanZero(vec3 v) { return v.x > 0.0f || v.y > 0.0f || v.z > 0.0f; }
inline float radians(float degrees) { return degrees * 0.017453292519943295f; }

// Transcendentals: the binary32 functions of hdcx/fpmath.h (the device
// integrator calls the same functions, so both produce the same bits).
inline float gexp(float x) { return hdcx_fp_exp(x); }
inline float glog(float x) { return hdcx_fp_log(x); }
inline float gpow(float x, float y) { return hdcx_fp_pow(x, y); }
inline float gsin(float x) { return hdcx_fp_sin(x); }
inline float gcos(float x) { return hdcx_fp_cos(x); }
inline float gacos(float x) { return hdcx_fp_acos(x); }
inline float gatan2(float y, float x) { return hdcx_fp_atan2(y, x); }

inline float uintToFloat(uint32_t v) { return static_cast<float>(v); }

}  // namespace oracle
