// oracle_internal.h - packed scene, BVH and integrator declarations of the
// CPU oracle. TEST INFRASTRUCTURE ONLY (see oracle_glsl.h).
#pragma once

#include "oracle_glsl.h"

#include <array>
#include <cstdint>
#include <string>
#include <vector>

#include "hdcx.h"

namespace oracle {

constexpr uint32_t kMaxMaterialTextures = 256u;  // vulkan_path_tracer.cpp:22
constexpr uint32_t kMissingTexture = 0xffffffffu;  // :23
constexpr uint32_t kUdimTextureFlag = 0x80000000u;  // :24
constexpr uint32_t kUdimTileMask = 0x7fffffu;  // :25
constexpr uint32_t kMaxPathBounces = 12u;  // :26
constexpr uint32_t kMaxLights = 64u;  // :27

// GpuMaterial (vulkan_path_tracer.cpp:42-66 shader side, :1907-1933 host side).
struct GpuMaterial {
    vec4 baseColorMetalness;
    vec4 emissionRoughness;
    vec4 transmissionOpacityIor;
    vec4 transmissionColorThinWalled;
    vec4 subsurfaceWeightScale;
    vec4 subsurfaceColor;
    vec4 subsurfaceRadius;
    vec4 specularWeightColor;
    vec4 coatWeightRoughnessIor;
    vec4 coatColor;
    vec4 transmissionMedium;
    vec4 transmissionScatter;
    vec4 sheenColorMode;
    vec4 diffuseProperties;
    vec4 translucentColorWeight;
    vec4 baseColorTextureScale;
    vec4 baseColorTextureBias;
    std::array<uint32_t, 4> textureIndices0;
    std::array<uint32_t, 4> textureIndices1;
    std::array<uint32_t, 4> textureIndices2;
    std::array<uint32_t, 4> textureIndices3;
    std::array<uint32_t, 4> textureIndices4;
    std::array<uint32_t, 4> textureIndices5;
};
static_assert(sizeof(GpuMaterial) == 368, "GpuMaterial is 23 x 16 bytes");

// GpuLight (vulkan_path_tracer.cpp:71-86 shader side, :1935-1952 host side).
struct GpuLight {
    vec4 colorIntensity;
    vec4 controls;
    vec4 position;
    vec4 axisU;
    vec4 axisV;
    vec4 basisX;
    vec4 basisY;
    vec4 basisZ;
    vec4 shaping;
    vec4 focusTint;
    vec4 shadow;
    vec4 shadowColor;
    vec4 geometry;
    std::array<uint32_t, 4> textureInfo;
};
static_assert(sizeof(GpuLight) == 224, "GpuLight is 14 x 16 bytes");

// A device texture: the Vulkan image the reference creates from a
// SceneTexture (vulkan_path_tracer.cpp:2215-2221). Texels are kept decoded to
// linear float RGBA, which is what the sampler filters (an R8G8B8A8_SRGB
// image is decoded to linear before filtering; alpha stays linear).
struct Texture {
    uint32_t width{0};
    uint32_t height{0};
    uint32_t format{HDCX_TEXEL_RGBA8_UNORM};
    std::vector<uint8_t> bytes;   // raw RGBA8 (for the packing view)
    std::vector<float> floats;    // raw RGBA32F (for the packing view)
    std::vector<float> linear;    // decoded RGBA, width*height*4
};

// The scene as BuildScene leaves it on the device.
struct PackedScene {
    std::vector<vec4> vertices;
    std::vector<uint32_t> indices;
    std::vector<uint32_t> triangleMaterials;
    std::vector<vec2> texcoords;
    std::vector<vec4> normals;
    std::vector<GpuMaterial> materials;
    std::vector<GpuLight> lights;      // at least one record
    std::vector<vec4> emissive;        // cdf, probability/area, area, 0
    std::vector<Texture> textures;
    bool opaque{true};
    bool geometryReady{false};
    uint32_t lightCount{0};
    uint32_t primitiveCount{0};
};

// Restatement of Impl::BuildScene (vulkan_path_tracer.cpp:2604-2993).
PackedScene PackScene(const hdcx_scene_desc& scene);

// Linear value of an sRGB-encoded byte, as VK_FORMAT_R8G8B8A8_SRGB decodes it.
float SrgbByteToLinear(uint8_t value);

// ---------------------------------------------------------------------------
// Ray queries over a binary BVH with the watertight triangle test.
// ---------------------------------------------------------------------------
struct Hit {
    uint32_t primitive{0xffffffffu};
    float t{0.0f};
    vec2 barycentrics{0.0f, 0.0f};  // weights of vertex 1 and vertex 2
};

struct BvhNode {
    float lo[3];
    float hi[3];
    uint32_t left;   // internal: left child index; leaf: first primitive slot
    uint32_t count;  // 0 = internal (right child = left + 1 is NOT assumed); leaf size
    uint32_t right;
};

struct Bvh {
    std::vector<BvhNode> nodes;
    std::vector<uint32_t> primitives;
};

Bvh BuildBvh(const PackedScene& scene);

enum class AcceptMode {
    Opaque,       // every candidate is confirmed
    Stochastic,   // confirmed iff anyHitThreshold(rayRng, prim) <= opacity
    Threshold,    // confirmed iff opacity >= 0.5 (shadow rays)
};

// Closest confirmed hit with t in [tmin, tmax]; ties in t go to the smaller
// primitive index. Returns false on a miss.
bool TraceClosest(const PackedScene& scene, const Bvh& bvh, vec3 origin, vec3 direction,
                  float tmin, float tmax, AcceptMode mode, uint32_t rayRng, Hit* hit);
// Every triangle the watertight test hits with t in [tmin, tmax], in no
// particular order (the candidates a ray query reports).
void TraceAll(const PackedScene& scene, const Bvh& bvh, vec3 origin, vec3 direction, float tmin, float tmax,
              std::vector<Hit>* hits);
// Any confirmed hit with t in [tmin, tmax].
bool TraceAny(const PackedScene& scene, const Bvh& bvh, vec3 origin, vec3 direction,
              float tmin, float tmax, AcceptMode mode);

// Helpers the integrator and the traversal share.
uint32_t hashState(uint32_t value);
float anyHitThreshold(uint32_t rayRng, uint32_t primitive);
float surfaceOpacity(const PackedScene& scene, uint32_t primitive, vec2 barycentrics);

// ---------------------------------------------------------------------------
// Integrator
// ---------------------------------------------------------------------------
struct Camera {
    vec3 origin, lowerLeft, horizontal, vertical;
};

struct FrameParams {
    uint32_t width, height, sampleIndex, sampleCount, maxBounces;
    bool zUp;
};

struct Counters {
    uint64_t extensionRays{0};
    uint64_t shadowRays{0};
    uint64_t subsurfaceRays{0};
};

// One pixel of main() (vulkan_path_tracer.cpp:1189-1891): updates rgba[4]
// (running mean) and adds the FP64 XYZ of the batch into xyz[3].
void RenderPixel(const PackedScene& scene, const Bvh& bvh, const Camera& camera,
                 const FrameParams& frame, uint32_t x, uint32_t y, float* rgba, double* xyz,
                 Counters* counters);

}  // namespace oracle
