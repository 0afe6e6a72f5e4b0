// common.cuh - device types and the arithmetic contract of the hdcx integrator.
//
// Arithmetic contract (the CPU oracle restates the same contract on its own):
//   * the integrator is compiled with -fmad=false: every float operation is a
//     single IEEE-754 binary32 operation, in the order the reference GLSL
//     (src/gpu/vulkan_path_tracer.cpp) writes it, left to right; division and
//     sqrt are IEEE (nvcc defaults -prec-div=true -prec-sqrt=true);
//   * dot(a, b) = (a.x*b.x + a.y*b.y) + a.z*b.z; normalize(v) = v * (1/sqrt(dot(v, v)));
//   * GLSL min/max/clamp/mix/smoothstep/reflect/refract/fract follow the GLSL
//     4.60 formulas;
//   * exp, log, pow, sin, cos, acos and atan2 are the binary32 functions of
//     hdcx/fpmath.h (fixed sequences of binary32 operations and fused
//     multiply-adds, so host and device evaluations agree bit for bit).
// Every vec3 the GLSL integrator carries per wavelength lane (throughput,
// radiance, colours after reflectanceSpectrum) holds one value in all three
// components, so the device code carries it as one float; luminance() of such
// a value is the three-term dot the GLSL evaluates.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "hdcx/fpmath.h"

namespace hdcx {

#define HDCX_D __device__ __forceinline__
#define HDCX_HD __host__ __device__ __forceinline__
#define HDCX_NOINLINE static __device__ __noinline__

constexpr uint32_t kMissingTexture = 0xffffffffu;
constexpr float kPi = 3.14159265359f;
constexpr float kTwoPi = 6.28318530718f;
constexpr uint32_t kInvalidPrimitive = 0xffffffffu;

// GpuMaterial / GpuLight device records (vulkan_path_tracer.cpp:42-86),
// byte-identical to the host packing.
struct __align__(16) GpuMaterial {
    float4 baseColorMetalness;
    float4 emissionRoughness;
    float4 transmissionOpacityIor;
    float4 transmissionColorThinWalled;
    float4 subsurfaceWeightScale;
    float4 subsurfaceColor;
    float4 subsurfaceRadius;
    float4 specularWeightColor;
    float4 coatWeightRoughnessIor;
    float4 coatColor;
    float4 transmissionMedium;
    float4 transmissionScatter;
    float4 sheenColorMode;
    float4 diffuseProperties;
    float4 translucentColorWeight;
    float4 baseColorTextureScale;
    float4 baseColorTextureBias;
    uint4 textureIndices0;
    uint4 textureIndices1;
    uint4 textureIndices2;
    uint4 textureIndices3;
    uint4 textureIndices4;
    uint4 textureIndices5;
};
static_assert(sizeof(GpuMaterial) == 368, "GpuMaterial is 23 x 16 bytes");

struct __align__(16) GpuLight {
    float4 colorIntensity;
    float4 controls;
    float4 position;
    float4 axisU;
    float4 axisV;
    float4 basisX;
    float4 basisY;
    float4 basisZ;
    float4 shaping;
    float4 focusTint;
    float4 shadow;
    float4 shadowColor;
    float4 geometry;
    uint4 textureInfo;
};
static_assert(sizeof(GpuLight) == 224, "GpuLight is 14 x 16 bytes");

// One device texture: texel array of an RGBA8 (UNORM or sRGB) or RGBA32F image.
struct TexDesc {
    const void* texels;
    uint32_t width;
    uint32_t height;
    uint32_t format;  // 0 RGBA8 UNORM, 1 RGBA8 sRGB, 2 RGBA32F
    uint32_t reserved;
    // Dome importance textures only (else null): the CDFs as compact floats
    // with every 32nd value repeated in skip arrays, in this order:
    //   marginal[h] (texel (0, row).y), marginalSkip[ceil(h/32)],
    //   conditional[h * w] (texel (col, row).x), conditionalSkip[h * ceil(w/32)],
    // where skip[k] = values[min(32k + 31, n - 1)].
    const float* cdf;
    // Texture LOD (hdcx_set_texture_lod): levels 1..levels-1 of the mip
    // pyramid as linear RGBA32F, level k (max(1, width >> k) x max(1, height >>
    // k) texels) after level k-1; null and levels 1 without a pyramid.
    const float4* mips;
    uint32_t levels;
    uint32_t pad;
};

// 8-wide BVH node with quantised child boxes (80 bytes). The layout is the
// compressed wide node of Ylitie, Karras and Laine, "Efficient Incoherent Ray
// Traversal on GPUs Through Compressed Wide BVHs", HPG 2017: origin p,
// power-of-two scale exponents, internal-child mask, base indices of the
// internal children and of the leaf triangles, one meta byte per slot (leaf
// children: unary triangle count << 5 | first triangle; internal and empty
// children: 0) and six quantised planes per child.
struct __align__(16) WideNode {
    float px, py, pz;
    uint8_t ex, ey, ez, imask;
    uint32_t childBase;
    uint32_t triBase;
    uint8_t meta[8];
    uint8_t qlox[8], qloy[8], qloz[8];
    uint8_t qhix[8], qhiy[8], qhiz[8];
};
static_assert(sizeof(WideNode) == 80, "wide node is 80 bytes");

// Two-level scenes (instancers): a bottom-level BVH per instanced mesh, in
// object space, plus one over the scene's other triangles in world space; the
// top-level BVH's leaves are instances.
struct BlasDesc {
    const WideNode* nodes;
    const float4* triVerts;  // leaf triangle copies; .w of the first: flattened id (world BLAS) or local index
    uint32_t nodeCount;
    uint32_t pad;
};

struct InstanceDesc {
    // World to object: object[j] = sum_i (world[i] - inv_i.w) * inv_i[j] for the
    // rows inv0..inv2 of the inverse of the instance's 3x3 (row vectors, the
    // translation in .w).
    float4 inv0, inv1, inv2;
    uint32_t blas;       // index into DeviceScene::blases
    uint32_t triBase;    // flattened id of the instance's first triangle
    uint32_t identity;   // 1: a world-space BLAS (ray and triangle ids used as they are)
    float margin;        // object-space widening of the boxes for the transformed ray's rounding
    float invNorm;       // max over j of sum_i |inverse[i][j]|: how much world lengths grow in object space
    float pad0, pad1, pad2;
};

// Traversal fault bits (a traversal's `fault` out-parameter; the kernels OR
// them into the render's counters[7], which the host reads back).
constexpr unsigned int kTraversalOverflow = 1u;  // a pending node group found the stack full and was dropped
constexpr unsigned int kTraversalBudget = 2u;    // a traversal visited more nodes than the BVH holds

// Scene as the kernels see it (device pointers).
struct DeviceScene {
    const float4* vertices;
    const uint32_t* indices;
    const uint32_t* triangleMaterials;
    const float2* texcoords;
    const float4* normals;
    const GpuMaterial* materials;
    const GpuLight* lights;
    const float4* emissive;
    const TexDesc* textures;
    const WideNode* nodes;
    const float4* triVerts;  // leaf-ordered triangles: 3 float4, primitive id in .w of the first
    uint32_t textureCount;
    uint32_t primitiveCount;
    uint32_t lightCount;     // authored lights, <= 64
    uint32_t opaque;
    uint32_t hasMeshLights;
    uint32_t nodeCount;
    uint32_t fullShading;    // 0: no material uses textures or layered lobes (see shadeKernel)
    uint32_t hasSubsurface;  // some material can take the subsurface random walk
    // Two-level scenes: instances, their BLASes; nodes/triVerts/nodeCount
    // are then the top-level BVH (its leaf "triangles" carry instance indices).
    const InstanceDesc* instances;  // null: single-level scene
    const BlasDesc* blases;
    uint32_t instanceCount;
};

// Per-render constants: the reference's CameraBlock (vulkan_path_tracer.cpp:91-98)
// with integer fields for the counts.
struct FrameConst {
    float3 origin;
    float3 lowerLeft;
    float3 horizontal;
    float3 vertical;
    uint32_t width;
    uint32_t height;
    uint32_t sampleIndex;
    uint32_t sampleCount;
    uint32_t maxBounces;
    uint32_t zUp;
    // Texture LOD: 0 off (every lookup at level 0, as the reference samples);
    // else the spread angle of a camera ray per unit distance (ray cones).
    float pixelSpread;
};

// ---------------------------------------------------------------------------
// float3 arithmetic with the contract's operation order.
// ---------------------------------------------------------------------------
HDCX_HD float3 f3(float s) { return make_float3(s, s, s); }
HDCX_HD float3 f3(float x, float y, float z) { return make_float3(x, y, z); }
HDCX_HD float3 xyz(float4 v) { return make_float3(v.x, v.y, v.z); }
HDCX_HD float3 operator+(float3 a, float3 b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }
HDCX_HD float3 operator-(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
HDCX_HD float3 operator-(float3 a) { return make_float3(-a.x, -a.y, -a.z); }
HDCX_HD float3 operator*(float3 a, float s) { return make_float3(a.x * s, a.y * s, a.z * s); }
HDCX_HD float3 operator*(float s, float3 a) { return make_float3(s * a.x, s * a.y, s * a.z); }
HDCX_HD float3 operator*(float3 a, float3 b) { return make_float3(a.x * b.x, a.y * b.y, a.z * b.z); }
HDCX_HD float3 operator/(float3 a, float s) { return make_float3(a.x / s, a.y / s, a.z / s); }
HDCX_HD float2 operator+(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
HDCX_HD float2 operator-(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
HDCX_HD float2 operator*(float2 a, float s) { return make_float2(a.x * s, a.y * s); }

#if defined(__CUDACC__)
HDCX_D float dot(float3 a, float3 b) { return __fadd_rn(__fadd_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)), __fmul_rn(a.z, b.z)); }
HDCX_D float3 cross(float3 a, float3 b)
{
    return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
HDCX_D float3 normalize(float3 v)
{
    const float inverse = 1.0f / sqrtf(dot(v, v));
    return v * inverse;
}
HDCX_D float2 normalize2(float2 v)
{
    const float inverse = 1.0f / sqrtf(v.x * v.x + v.y * v.y);
    return v * inverse;
}
HDCX_D float length2(float2 v) { return sqrtf(v.x * v.x + v.y * v.y); }
HDCX_D float inversesqrt(float x) { return 1.0f / sqrtf(x); }

// GLSL min(x, y) = y < x ? y : x ; max(x, y) = x < y ? y : x.
HDCX_D float gmin(float x, float y) { return y < x ? y : x; }
HDCX_D float gmax(float x, float y) { return x < y ? y : x; }
HDCX_D float clampf(float x, float lo, float hi) { return gmin(gmax(x, lo), hi); }
HDCX_D float fract(float x) { return x - floorf(x); }
HDCX_D float mix(float x, float y, float a) { return x * (1.0f - a) + y * a; }
HDCX_D float3 mix(float3 x, float3 y, float a) { return x * (1.0f - a) + y * a; }
HDCX_D float smoothstep(float e0, float e1, float x)
{
    const float t = clampf((x - e0) / (e1 - e0), 0.0f, 1.0f);
    return t * t * (3.0f - 2.0f * t);
}
HDCX_D float3 reflect(float3 i, float3 n) { return i - 2.0f * dot(n, i) * n; }
HDCX_D float3 refract(float3 i, float3 n, float eta)
{
    const float d = dot(n, i);
    const float k = 1.0f - eta * eta * (1.0f - d * d);
    if (k < 0.0f) return f3(0.0f);
    return eta * i - (eta * d + sqrtf(k)) * n;
}
HDCX_D float radians(float degrees) { return degrees * 0.017453292519943295f; }

// Transcendentals: the binary32 functions of hdcx/fpmath.h, bit-identical to
// the CPU evaluations of the integrator.
HDCX_D float gexp(float x) { return hdcx_fp_exp(x); }
HDCX_D float glog(float x) { return hdcx_fp_log(x); }
HDCX_D float gpow(float x, float y) { return hdcx_fp_pow(x, y); }
HDCX_D float gsin(float x) { return hdcx_fp_sin(x); }
HDCX_D float gcos(float x) { return hdcx_fp_cos(x); }
HDCX_D float gacos(float x) { return hdcx_fp_acos(x); }
HDCX_D float gatan2(float y, float x) { return hdcx_fp_atan2(y, x); }

#endif  // __CUDACC__

#if defined(__CUDACC__)
// pow(x, 2.0) and pow(x, 5.0) at call sites whose exponent is a constant:
// the same values hdcx_fp_pow returns for those exponents.
HDCX_D float gpow2(float x) { return x * x; }
HDCX_D float gpow5(float x) { return hdcx_fp_pow5(x); }
#endif

// lowbias32 integer hash and randomFloat (vulkan_path_tracer.cpp:100-113).
HDCX_HD uint32_t hashState(uint32_t value)
{
    value ^= value >> 16;
    value *= 0x7feb352du;
    value ^= value >> 15;
    value *= 0x846ca68bu;
    return value ^ (value >> 16);
}

#if defined(__CUDACC__)
HDCX_D float u2f(uint32_t v) { return __uint2float_rn(v); }
HDCX_D float randomFloat(uint32_t& state)
{
    state = hashState(state);
    return u2f(state) * (1.0f / 4294967296.0f);
}

// Order-independent confirmation threshold for a candidate of a non-opaque
// extension ray: a hash of the path's RNG state at ray start and the
// primitive, in randomFloat's [0, 1] mapping. The RNG is not advanced.
HDCX_D float anyHitThreshold(uint32_t rayRng, uint32_t primitive)
{
    return u2f(hashState(rayRng ^ hashState(primitive ^ 0x27d4eb2fu))) * (1.0f / 4294967296.0f);
}

// luminance of a lane value replicated in three components.
HDCX_D float luminance1(float s) { return s * 0.2126f + s * 0.7152f + s * 0.0722f; }
#endif  // __CUDACC__

}  // namespace hdcx
