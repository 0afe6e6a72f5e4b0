// ref_glsl_compat.h - GLSL 4.60 value semantics for compiling the reference
// integrator's own shader source as C++ on the CPU.
//
// TEST INFRASTRUCTURE ONLY (part of the oracle). oracle/ref_build.py extracts
// the GLSL of src/gpu/vulkan_path_tracer.cpp:31-1892 from the reference
// checkout, rewrites the few constructs C++ cannot express (parameter
// qualifiers, buffer blocks, swizzle methods, float literal suffixes, the
// entry point), and compiles it against this header and ref_harness.cpp into
// oracle/_ref/. Nothing of the reference's source is kept in this repository.
//
// Semantics: binary32 vector arithmetic component by component, in source
// order (compiled with -ffp-contract=off); transcendentals are the binary32
// functions of hdcx/fpmath.h (the same rule as the oracle);
// GLSL builtin formulas from the GLSL 4.60 specification.
#pragma once

#include <cstdint>
#include <cstring>
#include <algorithm>
#include <cmath>

#include "hdcx/fpmath.h"

namespace glsl {

typedef uint32_t uint;

struct uvec2;
struct ivec2;

struct vec2 {
    union { float x; float r; };
    union { float y; float g; };
    vec2() : x(0.0f), y(0.0f) {}
    explicit vec2(float s) : x(s), y(s) {}
    vec2(float a, float b) : x(a), y(b) {}
    explicit vec2(const uvec2& v);
    explicit vec2(const ivec2& v);
    float& operator[](int i) { return i == 0 ? x : y; }
    float operator[](int i) const { return i == 0 ? x : y; }
};

struct vec3 {
    union { float x; float r; };
    union { float y; float g; };
    union { float z; float b; };
    vec3() : x(0.0f), y(0.0f), z(0.0f) {}
    explicit vec3(float s) : x(s), y(s), z(s) {}
    vec3(float a, float b_, float c) : x(a), y(b_), z(c) {}
    float& operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
    float operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
    vec2 xy() const { return vec2(x, y); }
    vec2 yz() const { return vec2(y, z); }
    vec3 rgb() const { return *this; }
    vec3 xyz() const { return *this; }
};

struct vec4 {
    union { float x; float r; };
    union { float y; float g; };
    union { float z; float b; };
    union { float w; float a; };
    vec4() : x(0.0f), y(0.0f), z(0.0f), w(0.0f) {}
    explicit vec4(float s) : x(s), y(s), z(s), w(s) {}
    vec4(float a_, float b_, float c, float d) : x(a_), y(b_), z(c), w(d) {}
    vec4(const vec3& v, float d) : x(v.x), y(v.y), z(v.z), w(d) {}
    vec4(const vec2& v, float c, float d) : x(v.x), y(v.y), z(c), w(d) {}
    float& operator[](int i) { return i == 0 ? x : (i == 1 ? y : (i == 2 ? z : w)); }
    float operator[](int i) const { return i == 0 ? x : (i == 1 ? y : (i == 2 ? z : w)); }
    vec3 rgb() const { return vec3(x, y, z); }
    vec3 xyz() const { return vec3(x, y, z); }
    vec3 yzw() const { return vec3(y, z, w); }
    vec2 rg() const { return vec2(x, y); }
    vec2 xy() const { return vec2(x, y); }
};

struct uvec2 {
    uint x, y;
    uvec2() : x(0), y(0) {}
    uvec2(uint a, uint b) : x(a), y(b) {}
};
struct uvec3 {
    uint x, y, z;
    uvec2 xy() const { return uvec2(x, y); }
};
struct uvec4 {
    uint x, y, z, w;
    uvec2 xy() const { return uvec2(x, y); }
};
struct ivec2 {
    int x, y;
    ivec2() : x(0), y(0) {}
    explicit ivec2(int s) : x(s), y(s) {}
    ivec2(int a, int b) : x(a), y(b) {}
    explicit ivec2(const vec2& v) : x(static_cast<int>(v.x)), y(static_cast<int>(v.y)) {}
};
inline vec2::vec2(const uvec2& v) : x(static_cast<float>(v.x)), y(static_cast<float>(v.y)) {}
inline vec2::vec2(const ivec2& v) : x(static_cast<float>(v.x)), y(static_cast<float>(v.y)) {}

struct bvec3 {
    bool x, y, z;
};

// Arithmetic.
#define GLSL_VEC_OPS(V, N)                                                                                   \
    inline V operator+(const V& a, const V& b) { V r; for (int i = 0; i < N; ++i) r[i] = a[i] + b[i]; return r; } \
    inline V operator-(const V& a, const V& b) { V r; for (int i = 0; i < N; ++i) r[i] = a[i] - b[i]; return r; } \
    inline V operator*(const V& a, const V& b) { V r; for (int i = 0; i < N; ++i) r[i] = a[i] * b[i]; return r; } \
    inline V operator/(const V& a, const V& b) { V r; for (int i = 0; i < N; ++i) r[i] = a[i] / b[i]; return r; } \
    inline V operator+(const V& a, float s) { V r; for (int i = 0; i < N; ++i) r[i] = a[i] + s; return r; }       \
    inline V operator-(const V& a, float s) { V r; for (int i = 0; i < N; ++i) r[i] = a[i] - s; return r; }       \
    inline V operator*(const V& a, float s) { V r; for (int i = 0; i < N; ++i) r[i] = a[i] * s; return r; }       \
    inline V operator/(const V& a, float s) { V r; for (int i = 0; i < N; ++i) r[i] = a[i] / s; return r; }       \
    inline V operator+(float s, const V& a) { V r; for (int i = 0; i < N; ++i) r[i] = s + a[i]; return r; }       \
    inline V operator-(float s, const V& a) { V r; for (int i = 0; i < N; ++i) r[i] = s - a[i]; return r; }       \
    inline V operator*(float s, const V& a) { V r; for (int i = 0; i < N; ++i) r[i] = s * a[i]; return r; }       \
    inline V operator/(float s, const V& a) { V r; for (int i = 0; i < N; ++i) r[i] = s / a[i]; return r; }       \
    inline V operator-(const V& a) { V r; for (int i = 0; i < N; ++i) r[i] = -a[i]; return r; }                  \
    inline V& operator+=(V& a, const V& b) { a = a + b; return a; }                                              \
    inline V& operator-=(V& a, const V& b) { a = a - b; return a; }                                              \
    inline V& operator*=(V& a, const V& b) { a = a * b; return a; }                                              \
    inline V& operator/=(V& a, const V& b) { a = a / b; return a; }                                              \
    inline V& operator*=(V& a, float s) { a = a * s; return a; }                                                 \
    inline V& operator/=(V& a, float s) { a = a / s; return a; }                                                 \
    inline V& operator+=(V& a, float s) { a = a + s; return a; }
GLSL_VEC_OPS(vec2, 2)
GLSL_VEC_OPS(vec3, 3)
GLSL_VEC_OPS(vec4, 4)
#undef GLSL_VEC_OPS

inline ivec2 operator-(const ivec2& a, const ivec2& b) { return ivec2(a.x - b.x, a.y - b.y); }
inline ivec2 operator+(const ivec2& a, const ivec2& b) { return ivec2(a.x + b.x, a.y + b.y); }

// Builtins (GLSL 4.60 section 8).
inline float dot(const vec2& a, const vec2& b) { return a.x * b.x + a.y * b.y; }
inline float dot(const vec3& a, const vec3& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline vec3 cross(const vec3& a, const vec3& b)
{
    return vec3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
inline float sqrt(float x) { return std::sqrt(x); }
inline float inversesqrt(float x) { return 1.0f / std::sqrt(x); }
inline float length(const vec2& v) { return std::sqrt(dot(v, v)); }
inline float length(const vec3& v) { return std::sqrt(dot(v, v)); }
inline vec2 normalize(const vec2& v) { return v * (1.0f / std::sqrt(dot(v, v))); }
inline vec3 normalize(const vec3& v) { return v * (1.0f / std::sqrt(dot(v, v))); }
inline float abs(float x) { return std::fabs(x); }
inline vec3 abs(const vec3& v) { return vec3(std::fabs(v.x), std::fabs(v.y), std::fabs(v.z)); }
inline float floor(float x) { return std::floor(x); }
inline vec2 floor(const vec2& v) { return vec2(std::floor(v.x), std::floor(v.y)); }
inline float fract(float x) { return x - std::floor(x); }
inline vec2 fract(const vec2& v) { return vec2(fract(v.x), fract(v.y)); }
inline float round(float x) { return std::round(x); }
inline float min(float a, float b) { return b < a ? b : a; }
inline float max(float a, float b) { return a < b ? b : a; }
inline uint min(uint a, uint b) { return b < a ? b : a; }
inline uint max(uint a, uint b) { return a < b ? b : a; }
inline int min(int a, int b) { return b < a ? b : a; }
inline int max(int a, int b) { return a < b ? b : a; }
inline vec3 max(const vec3& a, const vec3& b) { return vec3(max(a.x, b.x), max(a.y, b.y), max(a.z, b.z)); }
inline vec3 min(const vec3& a, const vec3& b) { return vec3(min(a.x, b.x), min(a.y, b.y), min(a.z, b.z)); }
inline float clamp(float x, float lo, float hi) { return min(max(x, lo), hi); }
inline uint clamp(uint x, uint lo, uint hi) { return min(max(x, lo), hi); }
inline int clamp(int x, int lo, int hi) { return min(max(x, lo), hi); }
inline vec2 clamp(const vec2& v, const vec2& lo, const vec2& hi)
{
    return vec2(clamp(v.x, lo.x, hi.x), clamp(v.y, lo.y, hi.y));
}
inline vec3 clamp(const vec3& v, const vec3& lo, const vec3& hi)
{
    return vec3(clamp(v.x, lo.x, hi.x), clamp(v.y, lo.y, hi.y), clamp(v.z, lo.z, hi.z));
}
inline ivec2 clamp(const ivec2& v, const ivec2& lo, const ivec2& hi)
{
    return ivec2(clamp(v.x, lo.x, hi.x), clamp(v.y, lo.y, hi.y));
}
inline float mix(float x, float y, float a) { return x * (1.0f - a) + y * a; }
inline vec3 mix(const vec3& x, const vec3& y, float a) { return x * (1.0f - a) + y * a; }
inline float smoothstep(float e0, float e1, float x)
{
    const float t = clamp((x - e0) / (e1 - e0), 0.0f, 1.0f);
    return t * t * (3.0f - 2.0f * t);
}
inline vec3 reflect(const vec3& i, const vec3& n) { return i - 2.0f * dot(n, i) * n; }
inline vec3 refract(const vec3& i, const vec3& n, float eta)
{
    const float d = dot(n, i);
    const float k = 1.0f - eta * eta * (1.0f - d * d);
    if (k < 0.0f) return vec3(0.0f);
    return eta * i - (eta * d + std::sqrt(k)) * n;
}
inline float radians(float d) { return d * 0.017453292519943295f; }
// GLSL leaves the precision of these builtins to the implementation; this
// harness evaluates them with the binary32 functions of hdcx/fpmath.h.
inline float exp(float x) { return hdcx_fp_exp(x); }
inline float log(float x) { return hdcx_fp_log(x); }
inline float pow(float x, float y) { return hdcx_fp_pow(x, y); }
inline float sin(float x) { return hdcx_fp_sin(x); }
inline float cos(float x) { return hdcx_fp_cos(x); }
inline float acos(float x) { return hdcx_fp_acos(x); }
inline float atan(float y, float x) { return hdcx_fp_atan2(y, x); }
inline int bitCount(uint v) { return __builtin_popcount(v); }
inline bvec3 greaterThan(const vec3& a, const vec3& b) { return bvec3{a.x > b.x, a.y > b.y, a.z > b.z}; }
inline bool any(const bvec3& v) { return v.x || v.y || v.z; }
inline uint nonuniformEXT(uint i) { return i; }

// Combined image samplers: linear filter, REPEAT, one mip level (the
// reference's sampler, vulkan_path_tracer.cpp:2401-2423), texels decoded to
// linear float RGBA.
struct sampler2D {
    const float* texels = nullptr;
    int width = 0;
    int height = 0;
};
vec4 texture(const sampler2D& s, const vec2& uv);
vec4 texelFetch(const sampler2D& s, const ivec2& p, int lod);
inline ivec2 textureSize(const sampler2D& s, int) { return ivec2(s.width, s.height); }

// Ray queries (GL_EXT_ray_query), emulated by ref_harness.cpp.
struct accelerationStructureEXT {
    int unused = 0;
};
struct RayCandidate {
    uint primitive;
    float t;
    vec2 barycentrics;
};
struct rayQueryEXT {
    vec3 origin, direction;
    float tmin = 0.0f, tmax = 0.0f;
    uint flags = 0;
    bool started = false, done = false, opaque = false;
    int next = 0;
    int count = 0;
    RayCandidate candidates[256];
    bool overflow = false;
    RayCandidate current{};
    bool committed = false;
    RayCandidate committedHit{};
};
constexpr uint gl_RayFlagsNoneEXT = 0u;
constexpr uint gl_RayFlagsOpaqueEXT = 1u;
constexpr uint gl_RayFlagsTerminateOnFirstHitEXT = 4u;
constexpr uint gl_RayQueryCandidateIntersectionTriangleEXT = 0u;
constexpr uint gl_RayQueryCommittedIntersectionNoneEXT = 0u;
constexpr uint gl_RayQueryCommittedIntersectionTriangleEXT = 1u;

void rayQueryInitializeEXT(rayQueryEXT& q, const accelerationStructureEXT&, uint flags, uint mask, const vec3& origin,
                           float tmin, const vec3& direction, float tmax);
bool rayQueryProceedEXT(rayQueryEXT& q);
uint rayQueryGetIntersectionTypeEXT(rayQueryEXT& q, bool committed);
uint rayQueryGetIntersectionPrimitiveIndexEXT(rayQueryEXT& q, bool committed);
vec2 rayQueryGetIntersectionBarycentricsEXT(rayQueryEXT& q, bool committed);
float rayQueryGetIntersectionTEXT(rayQueryEXT& q, bool committed);
void rayQueryConfirmIntersectionEXT(rayQueryEXT& q);

extern thread_local uvec3 gl_GlobalInvocationID;

}  // namespace glsl
