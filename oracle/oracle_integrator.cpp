// oracle_integrator.cpp - CPU restatement of hdCodex's spectral path tracer.
// TEST INFRASTRUCTURE ONLY (see oracle_glsl.h).
//
// One C++ function per GLSL function of src/gpu/vulkan_path_tracer.cpp
// (line ranges cited on each), with the same names, argument order and
// arithmetic order. The GLSL shader computes one pixel per invocation; here
// RenderPixel() is that invocation. Ray queries go through oracle_trace.cpp.
#include "oracle_internal.h"

#include <algorithm>
#include <cmath>

namespace oracle {
namespace {

constexpr float kPi = 3.14159265359f;
constexpr float kTwoPi = 6.28318530718f;

struct Ctx {
    const PackedScene* scene;
    const Bvh* bvh;
    // CameraBlock (vulkan_path_tracer.cpp:91-98)
    vec4 origin, lowerLeft, horizontal, vertical;
    uint32_t frame[4];
    Counters* counters;
};

float randomFloat(uint32_t& state)
{
    // vulkan_path_tracer.cpp:109-113
    state = hashState(state);
    return uintToFloat(state) * (1.0f / 4294967296.0f);
}

// ---------------------------------------------------------------------------
// Spectral functions (vulkan_path_tracer.cpp:115-179)
// ---------------------------------------------------------------------------
float reconstructRgb(vec3 rgb, float wavelength)
{
    const vec3 basis = V3(gexp(-0.5f * gpow((wavelength - 620.0f) / 30.0f, 2.0f)),
                          gexp(-0.5f * gpow((wavelength - 535.0f) / 25.0f, 2.0f)),
                          gexp(-0.5f * gpow((wavelength - 450.0f) / 20.0f, 2.0f)));
    return dot(gmax(rgb, V3(0.0f)), basis) / gmax(dot(V3(1.0f), basis), 1e-5f);
}

float reflectanceSpectrum(vec3 rgb, float wavelength)
{
    return clampf(reconstructRgb(rgb, wavelength), 0.0f, 1.0f);
}

float illuminantSpectrum(vec3 rgb, float wavelength)
{
    const float temperature = 6504.0f;
    const float c2 = 1.4387769e7f;
    const float referenceWavelength = 560.0f;
    const float planck = gpow(referenceWavelength / wavelength, 5.0f) *
                         (gexp(c2 / (referenceWavelength * temperature)) - 1.0f) /
                         gmax(gexp(c2 / (wavelength * temperature)) - 1.0f, 1e-5f);
    return gmax(reconstructRgb(rgb, wavelength) * planck, 0.0f);
}

vec3 cieXyz(float wavelength)
{
    const float tx1 = (wavelength - 442.0f) * (wavelength < 442.0f ? 0.0624f : 0.0374f);
    const float tx2 = (wavelength - 599.8f) * (wavelength < 599.8f ? 0.0264f : 0.0323f);
    const float tx3 = (wavelength - 501.1f) * (wavelength < 501.1f ? 0.0490f : 0.0382f);
    const float ty1 = (wavelength - 568.8f) * (wavelength < 568.8f ? 0.0213f : 0.0247f);
    const float ty2 = (wavelength - 530.9f) * (wavelength < 530.9f ? 0.0613f : 0.0322f);
    const float tz1 = (wavelength - 437.0f) * (wavelength < 437.0f ? 0.0845f : 0.0278f);
    const float tz2 = (wavelength - 459.0f) * (wavelength < 459.0f ? 0.0385f : 0.0725f);
    return V3(0.362f * gexp(-0.5f * tx1 * tx1) + 1.056f * gexp(-0.5f * tx2 * tx2) -
                  0.065f * gexp(-0.5f * tx3 * tx3),
              0.821f * gexp(-0.5f * ty1 * ty1) + 0.286f * gexp(-0.5f * ty2 * ty2),
              1.217f * gexp(-0.5f * tz1 * tz1) + 0.681f * gexp(-0.5f * tz2 * tz2));
}

vec3 sensorXyz(float wavelength) { return cieXyz(wavelength) * (400.0f / 106.856895f); }

vec3 spectralSensor(float wavelength)
{
    const vec3 x = sensorXyz(wavelength);
    return V3(3.2404542f * x.x - 1.5371385f * x.y - 0.4985314f * x.z,
              -0.9692660f * x.x + 1.8760108f * x.y + 0.0415560f * x.z,
              0.0556434f * x.x - 0.2040259f * x.y + 1.0572252f * x.z);
}

// ---------------------------------------------------------------------------
// Sampling and BSDF helpers (vulkan_path_tracer.cpp:183-471)
// ---------------------------------------------------------------------------
vec3 tangentFrameAxis(vec3 normal)
{
    return normalize(std::fabs(normal.z) < 0.999f ? cross(normal, V3(0.0f, 0.0f, 1.0f))
                                                  : cross(normal, V3(0.0f, 1.0f, 0.0f)));
}

vec3 cosineHemisphere(vec3 normal, uint32_t& state)
{
    // :183-195
    const float r1 = kTwoPi * randomFloat(state);
    const float r2 = randomFloat(state);
    const float r2s = std::sqrt(r2);
    const vec3 tangent = tangentFrameAxis(normal);
    const vec3 bitangent = cross(normal, tangent);
    return normalize(tangent * gcos(r1) * r2s + bitangent * gsin(r1) * r2s +
                     normal * std::sqrt(1.0f - r2));
}

float luminance(vec3 value) { return dot(value, V3(0.2126f, 0.7152f, 0.0722f)); }

vec3 fresnelSchlick(float cosTheta, vec3 f0)
{
    // :202-205
    return f0 + (V3(1.0f) - f0) * gpow(1.0f - clampf(cosTheta, 0.0f, 1.0f), 5.0f);
}

vec3 orthogonalTangent(vec3 normal, vec3 tangent)
{
    // :276-285
    vec3 result = tangent - normal * dot(normal, tangent);
    if (dot(result, result) < 1e-8f) {
        result = std::fabs(normal.z) < 0.999f ? cross(normal, V3(0.0f, 0.0f, 1.0f))
                                              : cross(normal, V3(0.0f, 1.0f, 0.0f));
    }
    return normalize(result);
}

float distributionGGXAnisotropic(vec3 halfway, vec3 normal, vec3 tangent, vec2 roughness)
{
    // :287-300
    const vec3 axisX = orthogonalTangent(normal, tangent);
    const vec3 axisY = cross(normal, axisX);
    const vec2 alpha = clamp2(roughness * roughness, V2(0.001f, 0.001f), V2(1.0f, 1.0f));
    const vec3 localHalf = V3(dot(halfway, axisX), dot(halfway, axisY), gmax(dot(halfway, normal), 0.0f));
    const float denominator = localHalf.x * localHalf.x / (alpha.x * alpha.x) +
                              localHalf.y * localHalf.y / (alpha.y * alpha.y) + localHalf.z * localHalf.z;
    return 1.0f / gmax(kPi * alpha.x * alpha.y * denominator * denominator, 1e-6f);
}

float geometryGGXAnisotropic(vec3 direction, vec3 normal, vec3 tangent, vec2 roughness)
{
    // :302-315
    const float nDotDirection = gmax(dot(normal, direction), 0.0f);
    if (nDotDirection <= 0.0f) return 0.0f;
    const vec3 axisX = orthogonalTangent(normal, tangent);
    const vec3 axisY = cross(normal, axisX);
    const vec2 alpha = clamp2(roughness * roughness, V2(0.001f, 0.001f), V2(1.0f, 1.0f));
    const float projected = gpow(alpha.x * dot(direction, axisX), 2.0f) +
                            gpow(alpha.y * dot(direction, axisY), 2.0f);
    const float lambda =
        (-1.0f + std::sqrt(1.0f + projected / gmax(nDotDirection * nDotDirection, 1e-8f))) * 0.5f;
    return 1.0f / (1.0f + lambda);
}

vec3 evaluateGGXAnisotropic(vec3 normal, vec3 tangent, vec3 viewDirection, vec3 lightDirection,
                            vec2 roughness, vec3 f0)
{
    // :317-332
    const vec3 halfway = normalize(viewDirection + lightDirection);
    const float nDotV = gmax(dot(normal, viewDirection), 0.0f);
    const float nDotL = gmax(dot(normal, lightDirection), 0.0f);
    const float vDotH = gmax(dot(viewDirection, halfway), 0.0f);
    if (nDotV <= 0.0f || nDotL <= 0.0f || vDotH <= 0.0f) return V3(0.0f);
    const float distribution = distributionGGXAnisotropic(halfway, normal, tangent, roughness);
    const float geometry = geometryGGXAnisotropic(viewDirection, normal, tangent, roughness) *
                           geometryGGXAnisotropic(lightDirection, normal, tangent, roughness);
    return distribution * geometry * fresnelSchlick(vDotH, f0) / gmax(4.0f * nDotV * nDotL, 1e-5f);
}

vec3 sampleGGXReflectionAnisotropic(vec3 incident, vec3 normal, vec3 tangent, vec2 roughness,
                                    uint32_t& state)
{
    // :334-350
    const vec3 axisX = orthogonalTangent(normal, tangent);
    const vec3 axisY = cross(normal, axisX);
    const vec2 alpha = clamp2(roughness * roughness, V2(0.001f, 0.001f), V2(1.0f, 1.0f));
    const float phi = kTwoPi * randomFloat(state);
    const float elevationSample = randomFloat(state);
    const float radius = std::sqrt(elevationSample / gmax(1.0f - elevationSample, 1e-6f));
    vec3 halfway = normalize(axisX * (alpha.x * radius * gcos(phi)) +
                             axisY * (alpha.y * radius * gsin(phi)) + normal);
    if (dot(halfway, -incident) < 0.0f) halfway = -halfway;
    const vec3 reflected = reflect(incident, halfway);
    return dot(reflected, normal) > 0.0f ? normalize(reflected) : normalize(reflect(incident, normal));
}

vec3 ggxSampleWeightAnisotropic(vec3 incident, vec3 outgoing, vec3 normal, vec3 tangent,
                                vec2 roughness, vec3 f0)
{
    // :352-367
    const vec3 viewDirection = normalize(-incident);
    const vec3 halfway = normalize(viewDirection + outgoing);
    const float nDotL = gmax(dot(normal, outgoing), 0.0f);
    const float nDotH = gmax(dot(normal, halfway), 0.0f);
    const float vDotH = gmax(dot(viewDirection, halfway), 0.0f);
    if (nDotL <= 0.0f || nDotH <= 0.0f || vDotH <= 0.0f) return V3(0.0f);
    const float distribution = distributionGGXAnisotropic(halfway, normal, tangent, roughness);
    const float pdf = distribution * nDotH / gmax(4.0f * vDotH, 1e-6f);
    return evaluateGGXAnisotropic(normal, tangent, viewDirection, outgoing, roughness, f0) * nDotL /
           gmax(pdf, 1e-6f);
}

float ggxReflectionPdfAnisotropic(vec3 normal, vec3 tangent, vec3 viewDirection, vec3 lightDirection,
                                  vec2 roughness)
{
    // :371-383
    if (dot(normal, viewDirection) <= 0.0f || dot(normal, lightDirection) <= 0.0f) return 0.0f;
    const vec3 halfway = normalize(viewDirection + lightDirection);
    const float nDotH = gmax(dot(normal, halfway), 0.0f);
    const float vDotH = gmax(dot(viewDirection, halfway), 0.0f);
    return distributionGGXAnisotropic(halfway, normal, tangent, roughness) * nDotH /
           gmax(4.0f * vDotH, 1e-6f);
}

float powerHeuristic(float firstPdf, float secondPdf)
{
    // :385-390
    const float firstSquared = firstPdf * firstPdf;
    const float secondSquared = secondPdf * secondPdf;
    return firstSquared / gmax(firstSquared + secondSquared, 1e-12f);
}

float surfaceReflectionPdf(vec3 normal, vec3 tangent, vec3 viewDirection, vec3 lightDirection,
                           vec2 roughness, vec2 coatRoughness, float sheenProbability,
                           float coatProbability, float specularProbability,
                           float translucentProbability)
{
    // :392-415
    const float reflectionCosinePdf = gmax(dot(normal, lightDirection), 0.0f) / kPi;
    const float transmissionCosinePdf = gmax(-dot(normal, lightDirection), 0.0f) / kPi;
    const float coatPdf = ggxReflectionPdfAnisotropic(normal, tangent, viewDirection, lightDirection,
                                                      coatRoughness);
    const float specularPdf =
        ggxReflectionPdfAnisotropic(normal, tangent, viewDirection, lightDirection, roughness);
    const float diffusePdf = mix(reflectionCosinePdf, transmissionCosinePdf, translucentProbability);
    const float basePdf = coatProbability * coatPdf +
                          (1.0f - coatProbability) *
                              (specularProbability * specularPdf + (1.0f - specularProbability) * diffusePdf);
    return sheenProbability * reflectionCosinePdf + (1.0f - sheenProbability) * basePdf;
}

float sheenDirectionalAlbedo(float nDotV, float roughness)
{
    // :419-429
    const float x = clampf(nDotV, 0.0f, 1.0f);
    const float y = clampf(roughness, 0.01f, 1.0f);
    const vec2 fit = V2(13.67300f, 1.0f) + V2(-68.78018f, 61.57746f) * x +
                     V2(799.08825f, 442.78211f) * y + V2(-905.00061f, 2597.49308f) * x * y +
                     V2(60.28956f, 121.81241f) * x * x + V2(1086.96473f, 3045.55075f) * y * y;
    return clampf(fit.x / gmax(fit.y, 1e-6f), 0.0f, 1.0f);
}

float sheenImageworksResponse(vec3 normal, vec3 viewDirection, vec3 lightDirection, float roughness)
{
    // :431-446
    const float nDotL = gmax(dot(normal, lightDirection), 0.0f);
    const float nDotV = gmax(dot(normal, viewDirection), 0.0f);
    if (nDotL <= 0.0f || nDotV <= 0.0f) return 0.0f;
    const vec3 halfway = normalize(viewDirection + lightDirection);
    const float nDotH = gmax(dot(normal, halfway), 0.0f);
    const float inverseRoughness = 1.0f / gmax(roughness, 0.005f);
    const float distribution = (2.0f + inverseRoughness) *
                               gpow(gmax(1.0f - nDotH * nDotH, 0.0f), inverseRoughness * 0.5f) /
                               (2.0f * kPi);
    const float brdf = distribution / gmax(4.0f * (nDotL + nDotV - nDotL * nDotV), 1e-6f);
    return brdf * nDotL;
}

float sheenZeltnerDirectionalAlbedo(float nDotV, float roughness)
{
    // :448-460
    const float x = clampf(nDotV, 0.0f, 1.0f);
    const float y = clampf(roughness, 0.01f, 1.0f);
    const float s = y * (0.0206607f + 1.58491f * y) / (0.0379424f + y * (1.32227f + y));
    const float m = y * (-0.193854f + y * (-1.14885f + y * (1.7932f - 0.95943f * y * y))) / (0.046391f + y);
    const float o = y * (0.000654023f + (-0.0207818f + 0.119681f * y) * y) / (1.26264f + y * (-1.92021f + y));
    return clampf(gexp(-0.5f * gpow((x - m) / gmax(s, 1e-6f), 2.0f)) /
                          (gmax(s, 1e-6f) * std::sqrt(2.0f * kPi)) + o,
                  0.0f, 1.0f);
}

float sheenResponse(vec3 normal, vec3 viewDirection, vec3 lightDirection, float roughness, bool zeltner)
{
    // :462-471
    if (!zeltner) return sheenImageworksResponse(normal, viewDirection, lightDirection, roughness);
    const float nDotL = gmax(dot(normal, lightDirection), 0.0f);
    const float nDotV = gmax(dot(normal, viewDirection), 0.0f);
    return sheenZeltnerDirectionalAlbedo(nDotV, roughness) * nDotL / kPi;
}

// ---------------------------------------------------------------------------
// Textures (the reference's sampler: linear filter, REPEAT, one mip level,
// vulkan_path_tracer.cpp:2401-2423). Bilinear weights follow the Vulkan
// formula in binary32; texel i covers [i, i+1) in texel space.
// ---------------------------------------------------------------------------
int WrapIndex(int i, int n)
{
    const int r = i % n;
    return r < 0 ? r + n : r;
}

float TexelCoordinate(float uv, uint32_t size)
{
    const float x = uv * static_cast<float>(size) - 0.5f;
    return std::fabs(x) < 16777216.0f ? x : 0.0f;  // also maps NaN to 0
}

vec4 TexelFetch(const Texture& t, int x, int y)
{
    const float* p = &t.linear[(static_cast<size_t>(y) * t.width + static_cast<size_t>(x)) * 4u];
    return V4(p[0], p[1], p[2], p[3]);
}

vec4 SampleBilinear(const Texture& t, vec2 uv)
{
    const float x = TexelCoordinate(uv.x, t.width);
    const float y = TexelCoordinate(uv.y, t.height);
    const float fx = std::floor(x), fy = std::floor(y);
    const float a = x - fx, b = y - fy;
    const int w = static_cast<int>(t.width), h = static_cast<int>(t.height);
    const int i0 = WrapIndex(static_cast<int>(fx), w);
    const int j0 = WrapIndex(static_cast<int>(fy), h);
    const int i1 = WrapIndex(i0 + 1, w);
    const int j1 = WrapIndex(j0 + 1, h);
    const vec4 t00 = TexelFetch(t, i0, j0), t10 = TexelFetch(t, i1, j0);
    const vec4 t01 = TexelFetch(t, i0, j1), t11 = TexelFetch(t, i1, j1);
    const float w00 = (1.0f - a) * (1.0f - b), w10 = a * (1.0f - b);
    const float w01 = (1.0f - a) * b, w11 = a * b;
    return V4(w00 * t00.x + w10 * t10.x + w01 * t01.x + w11 * t11.x,
              w00 * t00.y + w10 * t10.y + w01 * t01.y + w11 * t11.y,
              w00 * t00.z + w10 * t10.z + w01 * t01.z + w11 * t11.z,
              w00 * t00.w + w10 * t10.w + w01 * t01.w + w11 * t11.w);
}

vec4 textureSample(const Ctx& c, uint32_t index, vec2 uv)
{
    if (index >= c.scene->textures.size()) return V4(0.0f);
    return SampleBilinear(c.scene->textures[index], uv);
}

// ---------------------------------------------------------------------------
// Dome and environment (vulkan_path_tracer.cpp:473-569)
// ---------------------------------------------------------------------------
vec2 directionToVerticalCross(vec3 direction)
{
    const vec3 a = abs3(direction);
    vec2 faceUv;
    vec2 tile;
    if (a.x >= a.y && a.x >= a.z) {
        if (direction.x >= 0.0f) {
            faceUv = V2(-direction.z / a.x, direction.y / a.x);
            tile = V2(2.0f, 1.0f);
        } else {
            faceUv = V2(direction.z / a.x, direction.y / a.x);
            tile = V2(0.0f, 1.0f);
        }
    } else if (a.y >= a.z) {
        if (direction.y >= 0.0f) {
            faceUv = V2(direction.x / a.y, -direction.z / a.y);
            tile = V2(1.0f, 0.0f);
        } else {
            faceUv = V2(direction.x / a.y, direction.z / a.y);
            tile = V2(1.0f, 2.0f);
        }
    } else if (direction.z >= 0.0f) {
        faceUv = V2(direction.x / a.z, direction.y / a.z);
        tile = V2(1.0f, 1.0f);
    } else {
        faceUv = V2(-direction.x / a.z, direction.y / a.z);
        tile = V2(1.0f, 3.0f);
    }
    const vec2 q = tile + faceUv * 0.5f;
    return V2((q.x + 0.5f) / 3.0f, (q.y + 0.5f) / 4.0f);
}

vec2 domeTextureCoordinates(vec3 direction, uint32_t format)
{
    // :505-525
    if (format == 2u) {
        const float denominator =
            2.0f * std::sqrt(gmax(direction.x * direction.x + direction.y * direction.y +
                                      (direction.z + 1.0f) * (direction.z + 1.0f),
                                  1e-8f));
        return V2(direction.x / denominator + 0.5f, direction.y / denominator + 0.5f);
    }
    if (format == 3u) {
        const float radius = gacos(clampf(-direction.z, -1.0f, 1.0f)) / kPi;
        const vec2 dxy = V2(direction.x, direction.y);
        const vec2 radial = length(dxy) > 1e-6f ? normalize(dxy) : V2(0.0f, 0.0f);
        const float r = 0.5f * radius;
        return V2(0.5f + radial.x * r, 0.5f + radial.y * r);
    }
    if (format == 4u) return directionToVerticalCross(direction);
    return V2(fract(gatan2(direction.x, -direction.z) / (2.0f * kPi) + 1.0f),
              1.0f - gacos(clampf(direction.y, -1.0f, 1.0f)) / kPi);
}

vec3 sampleDome(const Ctx& c, const GpuLight& light, vec3 worldDirection)
{
    // :527-537
    const vec3 localDirection = normalize(V3(dot(worldDirection, xyz(light.basisX)),
                                             dot(worldDirection, xyz(light.basisY)),
                                             dot(worldDirection, xyz(light.basisZ))));
    const vec3 textureValue =
        light.textureInfo[0] == 0xffffffffu
            ? V3(1.0f)
            : xyz(textureSample(c, light.textureInfo[0], domeTextureCoordinates(localDirection, light.textureInfo[1])));
    return xyz(light.colorIntensity) * light.colorIntensity.w * textureValue;
}

uint32_t scenePrimitiveCount(const Ctx& c)
{
    // :539-542 reads float(primitiveCount) from lowerLeft.w; the count is an
    // integer here, so scenes past 2^24 triangles keep working.
    return c.scene->primitiveCount;
}

bool hasEmissiveTriangles(const Ctx& c)
{
    // :544-549
    const uint32_t n = scenePrimitiveCount(c);
    return n > 0u && c.scene->emissive[n - 1u].x > 0.0f;
}

uint32_t lightCountOf(const Ctx& c) { return (c.frame[3] >> 16u) & 0xffu; }

vec3 environment(const Ctx& c, vec3 direction)
{
    // :551-569
    vec3 result = V3(0.0f);
    const uint32_t lightCount = lightCountOf(c);
    if (lightCount == 0u) {
        if (hasEmissiveTriangles(c)) return V3(0.0f);
        const vec3 up = c.vertical.w > 0.5f ? V3(0.0f, 0.0f, 1.0f) : V3(0.0f, 1.0f, 0.0f);
        const float t = 0.5f * (dot(direction, up) + 1.0f);
        return mix(V3(0.035f, 0.045f, 0.065f), V3(0.38f, 0.55f, 0.85f), t);
    }
    for (uint32_t index = 0; index < lightCount; ++index) {
        const GpuLight& light = c.scene->lights[index];
        if (light.textureInfo[2] == 0u) result += sampleDome(c, light, direction);
    }
    return result;
}

vec3 latLongDirection(vec2 uv)
{
    // :571-579
    const float theta = kPi * (1.0f - uv.y);
    const float phi = 2.0f * kPi * uv.x;
    const float sineTheta = gsin(theta);
    return V3(sineTheta * gsin(phi), gcos(theta), -sineTheta * gcos(phi));
}

vec3 uniformSphere(uint32_t& state)
{
    // :1077-1083
    const float y = 1.0f - 2.0f * randomFloat(state);
    const float radius = std::sqrt(gmax(1.0f - y * y, 0.0f));
    const float phi = kTwoPi * randomFloat(state);
    return V3(radius * gcos(phi), y, radius * gsin(phi));
}

const Texture* importanceTexture(const Ctx& c, uint32_t index)
{
    return index < c.scene->textures.size() ? &c.scene->textures[index] : nullptr;
}

float domeLightPdf(const Ctx& c, const GpuLight& light, vec3 worldDirection)
{
    // :583-598
    const Texture* t = light.textureInfo[3] == 0xffffffffu ? nullptr : importanceTexture(c, light.textureInfo[3]);
    if (!t) return 1.0f / 12.5663706144f;
    const vec3 localDirection = normalize(V3(dot(worldDirection, xyz(light.basisX)),
                                             dot(worldDirection, xyz(light.basisY)),
                                             dot(worldDirection, xyz(light.basisZ))));
    const vec2 uv = domeTextureCoordinates(localDirection, light.textureInfo[1]);
    const int w = static_cast<int>(t->width), h = static_cast<int>(t->height);
    // ivec2(uv * dimensions) truncates toward zero; NaN maps to 0.
    const float fx = uv.x * static_cast<float>(w), fy = uv.y * static_cast<float>(h);
    int tx = std::fabs(fx) < 2147483520.0f ? static_cast<int>(fx) : 0;
    int ty = std::fabs(fy) < 2147483520.0f ? static_cast<int>(fy) : 0;
    tx = std::clamp(tx, 0, w - 1);
    ty = std::clamp(ty, 0, h - 1);
    return gmax(TexelFetch(*t, tx, ty).z, 0.0f);
}

void sampleDomeLight(const Ctx& c, const GpuLight& light, uint32_t& rng, vec3& worldDirection, float& pdf)
{
    // :600-650
    const Texture* t = light.textureInfo[3] == 0xffffffffu ? nullptr : importanceTexture(c, light.textureInfo[3]);
    if (!t) {
        worldDirection = uniformSphere(rng);
        pdf = 1.0f / 12.5663706144f;
        return;
    }
    const int w = static_cast<int>(t->width), h = static_cast<int>(t->height);
    const float rowTarget = randomFloat(rng);
    int low = 0;
    int high = h - 1;
    while (low < high) {
        const int middle = (low + high) / 2;
        const float cdf = TexelFetch(*t, 0, middle).y;
        if (rowTarget <= cdf) high = middle;
        else low = middle + 1;
    }
    const int row = low;
    const float columnTarget = randomFloat(rng);
    low = 0;
    high = w - 1;
    while (low < high) {
        const int middle = (low + high) / 2;
        const float cdf = TexelFetch(*t, middle, row).x;
        if (columnTarget <= cdf) high = middle;
        else low = middle + 1;
    }
    const int column = low;
    const float v0 = static_cast<float>(row) / static_cast<float>(h);
    const float v1 = static_cast<float>(row + 1) / static_cast<float>(h);
    const float cosine0 = gcos(kPi * (1.0f - v0));
    const float cosine1 = gcos(kPi * (1.0f - v1));
    const float cosineTheta = mix(cosine0, cosine1, randomFloat(rng));
    const float v = 1.0f - gacos(clampf(cosineTheta, -1.0f, 1.0f)) / kPi;
    const float u = (static_cast<float>(column) + randomFloat(rng)) / static_cast<float>(w);
    const vec3 localDirection = latLongDirection(V2(u, v));
    worldDirection = normalize(xyz(light.basisX) * localDirection.x + xyz(light.basisY) * localDirection.y +
                               xyz(light.basisZ) * localDirection.z);
    pdf = gmax(TexelFetch(*t, column, row).z, 0.0f);
}

float lightSelectionWeight(const GpuLight& light, vec3 position, vec3 normal, float diffuseEnergy,
                           float specularEnergy, float translucentEnergy)
{
    // :652-691
    const float power = gmax(light.geometry.w, 0.0f);
    if (power <= 0.0f) return 0.0f;
    const float diffuseResponse = gmax(diffuseEnergy, 0.0f) * light.controls.x;
    const float specularResponse = gmax(specularEnergy, 0.0f) * light.controls.y;
    const float transmissionResponse = gmax(translucentEnergy, 0.0f) * light.controls.x;
    const float minimumWeight = power * 0.01f;
    const uint32_t type = light.textureInfo[2];
    if (type == 0u) {
        return gmax(minimumWeight,
                    power * (0.5f * (diffuseResponse + transmissionResponse) + specularResponse));
    }
    vec3 direction;
    float geometryFactor = 1.0f;
    if (type == 5u) {
        direction = normalize(xyz(light.basisZ));
    } else {
        const vec3 toLight = xyz(light.position) - position;
        const float distanceSquared = gmax(dot(toLight, toLight), 1e-4f);
        direction = toLight * inversesqrt(distanceSquared);
        geometryFactor = 1.0f / distanceSquared;
        if (type == 1u || type == 2u) {
            const vec3 lightNormal = -normalize(xyz(light.basisZ));
            geometryFactor *= gmax(dot(lightNormal, -direction), 0.0f);
        } else if (type == 4u) {
            geometryFactor *= 0.5f;
        }
    }
    const float nDotL = dot(normal, direction);
    const float response = gmax(nDotL, 0.0f) * (diffuseResponse + specularResponse) +
                           gmax(-nDotL, 0.0f) * transmissionResponse;
    return gmax(minimumWeight, power * geometryFactor * response);
}

float totalAnalyticLightWeight(const Ctx& c, vec3 position, vec3 normal, float diffuseEnergy,
                               float specularEnergy, float translucentEnergy)
{
    // :693-705
    const uint32_t lightCount = lightCountOf(c);
    float total = 0.0f;
    for (uint32_t index = 0; index < lightCount; ++index) {
        total += lightSelectionWeight(c.scene->lights[index], position, normal, diffuseEnergy,
                                      specularEnergy, translucentEnergy);
    }
    return total;
}

void sampleAnalyticLight(const Ctx& c, vec3 position, vec3 normal, float diffuseEnergy,
                         float specularEnergy, float translucentEnergy, uint32_t& rng,
                         uint32_t& lightIndex, float& selectionPdf)
{
    // :707-737
    const uint32_t lightCount = lightCountOf(c);
    const float total =
        totalAnalyticLightWeight(c, position, normal, diffuseEnergy, specularEnergy, translucentEnergy);
    if (total <= 0.0f) {
        const float scaled = randomFloat(rng) * uintToFloat(lightCount);
        const uint32_t pick = scaled >= 4294967296.0f ? 0xffffffffu : static_cast<uint32_t>(scaled);
        lightIndex = std::min(pick, lightCount - 1u);
        selectionPdf = 1.0f / uintToFloat(lightCount);
        return;
    }
    const float target = randomFloat(rng) * total;
    float accumulated = 0.0f;
    lightIndex = lightCount - 1u;
    for (uint32_t index = 0; index < lightCount; ++index) {
        const float weight = lightSelectionWeight(c.scene->lights[index], position, normal, diffuseEnergy,
                                                  specularEnergy, translucentEnergy);
        accumulated += weight;
        if (target <= accumulated) {
            lightIndex = index;
            break;
        }
    }
    selectionPdf = lightSelectionWeight(c.scene->lights[lightIndex], position, normal, diffuseEnergy,
                                        specularEnergy, translucentEnergy) /
                   total;
}

float environmentLightPdf(const Ctx& c, vec3 position, vec3 normal, vec3 direction, float diffuseEnergy,
                          float specularEnergy, float translucentEnergy)
{
    // :739-758
    const uint32_t lightCount = lightCountOf(c);
    if (lightCount == 0u) return 0.0f;
    const float total =
        totalAnalyticLightWeight(c, position, normal, diffuseEnergy, specularEnergy, translucentEnergy);
    if (total <= 0.0f) return 0.0f;
    float pdf = 0.0f;
    for (uint32_t index = 0; index < lightCount; ++index) {
        const GpuLight& light = c.scene->lights[index];
        if (light.textureInfo[2] == 0u) {
            const float selectionPdf =
                lightSelectionWeight(light, position, normal, diffuseEnergy, specularEnergy, translucentEnergy) /
                total;
            pdf += selectionPdf * domeLightPdf(c, light, direction);
        }
    }
    return pdf;
}

// ---------------------------------------------------------------------------
// Surface attributes (vulkan_path_tracer.cpp:760-853)
// ---------------------------------------------------------------------------
vec4 sampleMaterialTexture(const Ctx& c, uint32_t textureIndex, vec2 uv, vec4 fallbackValue)
{
    // :760-775
    if (textureIndex == 0xffffffffu) return fallbackValue;
    if ((textureIndex & 0x80000000u) != 0u) {
        const float fu = std::floor(uv.x), fv = std::floor(uv.y);
        if (!(std::fabs(fu) < 1e6f) || !(std::fabs(fv) < 1e6f)) return fallbackValue;
        const int tileOffset = static_cast<int>(fu) + static_cast<int>(fv) * 10;
        if (tileOffset < 0 || tileOffset >= 23) return fallbackValue;
        const uint32_t presentTiles = (textureIndex >> 8u) & 0x7fffffu;
        const uint32_t tileBit = 1u << static_cast<uint32_t>(tileOffset);
        if ((presentTiles & tileBit) == 0u) return fallbackValue;
        const uint32_t descriptorIndex =
            (textureIndex & 0xffu) + static_cast<uint32_t>(__builtin_popcount(presentTiles & (tileBit - 1u)));
        if (descriptorIndex >= c.scene->textures.size()) return fallbackValue;
        return textureSample(c, descriptorIndex, fract(uv));
    }
    if (textureIndex >= c.scene->textures.size()) return fallbackValue;
    return textureSample(c, textureIndex, uv);
}

vec3 surfaceEmissionRgb(const Ctx& c, uint32_t primitive, vec2 uv)
{
    // :777-785
    const GpuMaterial& material = c.scene->materials[c.scene->triangleMaterials[primitive]];
    const float weight = gmax(material.transmissionOpacityIor.w, 0.0f);
    return material.textureIndices0[3] == 0xffffffffu
               ? xyz(material.emissionRoughness) * weight
               : xyz(sampleMaterialTexture(c, material.textureIndices0[3], uv, V4(0.0f))) * weight;
}

vec2 surfaceTextureCoordinates(const PackedScene& s, uint32_t primitive, vec2 barycentrics)
{
    // :787-795
    const vec3 b = V3(1.0f - barycentrics.x - barycentrics.y, barycentrics.x, barycentrics.y);
    const vec2 uv0 = s.texcoords[primitive * 3u + 0u];
    const vec2 uv1 = s.texcoords[primitive * 3u + 1u];
    const vec2 uv2 = s.texcoords[primitive * 3u + 2u];
    return uv0 * b.x + uv1 * b.y + uv2 * b.z;
}

vec3 applyNormalMap(const Ctx& c, uint32_t textureIndex, bool flipY, float scale, vec2 uv,
                    vec3 geometricNormal, vec3 p0, vec3 p1, vec3 p2, vec2 uv0, vec2 uv1, vec2 uv2)
{
    // :807-829
    if (textureIndex == 0xffffffffu) return geometricNormal;
    const vec2 deltaUv1 = uv1 - uv0;
    const vec2 deltaUv2 = uv2 - uv0;
    const float determinant = deltaUv1.x * deltaUv2.y - deltaUv1.y * deltaUv2.x;
    if (std::fabs(determinant) < 1e-8f) return geometricNormal;
    const vec3 edge1 = p1 - p0;
    const vec3 edge2 = p2 - p0;
    vec3 tangent = normalize((edge1 * deltaUv2.y - edge2 * deltaUv1.y) / determinant);
    tangent = normalize(tangent - geometricNormal * dot(geometricNormal, tangent));
    vec3 bitangent = normalize(cross(geometricNormal, tangent));
    if (determinant < 0.0f) bitangent = -bitangent;
    vec3 mapped = xyz(sampleMaterialTexture(c, textureIndex, uv, V4(0.5f, 0.5f, 1.0f, 1.0f)));
    mapped = mapped * 2.0f - V3(1.0f);
    if (flipY) mapped.y = -mapped.y;
    mapped.x *= scale;
    mapped.y *= scale;
    const vec3 result = normalize(tangent * mapped.x + bitangent * mapped.y + geometricNormal * mapped.z);
    return dot(result, geometricNormal) < 0.0f ? -result : result;
}

vec3 surfaceTangent(vec3 normal, vec3 p0, vec3 p1, vec3 p2, vec2 uv0, vec2 uv1, vec2 uv2)
{
    // :831-841
    const vec2 deltaUv1 = uv1 - uv0;
    const vec2 deltaUv2 = uv2 - uv0;
    const float determinant = deltaUv1.x * deltaUv2.y - deltaUv1.y * deltaUv2.x;
    if (std::fabs(determinant) < 1e-8f) return orthogonalTangent(normal, V3(1.0f, 0.0f, 0.0f));
    const vec3 tangent = ((p1 - p0) * deltaUv2.y - (p2 - p0) * deltaUv1.y) / determinant;
    return orthogonalTangent(normal, tangent);
}

vec3 surfaceShadingNormal(const PackedScene& s, uint32_t primitive, vec2 barycentrics, vec3 geometricNormal)
{
    // :843-853
    const vec3 b = V3(1.0f - barycentrics.x - barycentrics.y, barycentrics.x, barycentrics.y);
    vec3 result = xyz(s.normals[primitive * 3u + 0u]) * b.x + xyz(s.normals[primitive * 3u + 1u]) * b.y +
                  xyz(s.normals[primitive * 3u + 2u]) * b.z;
    if (dot(result, result) < 1e-12f) return geometricNormal;
    result = normalize(result);
    return dot(result, geometricNormal) < 0.0f ? -result : result;
}

// ---------------------------------------------------------------------------
// Visibility (vulkan_path_tracer.cpp:855-912)
// ---------------------------------------------------------------------------
bool sceneOpaque(const Ctx& c) { return (c.frame[3] & 0x100u) != 0u; }

vec3 shadowVisibility(const Ctx& c, vec3 origin, vec3 direction, float maximumDistance, const GpuLight& light)
{
    // :855-889
    if (light.shadow.x < 0.5f) return V3(1.0f);
    float traceDistance = maximumDistance;
    if (light.shadow.y >= 0.0f) traceDistance = gmin(traceDistance, light.shadow.y);
    if (traceDistance <= 0.001f) return V3(1.0f);
    c.counters->shadowRays++;
    const AcceptMode mode = sceneOpaque(c) ? AcceptMode::Opaque : AcceptMode::Threshold;
    const bool falloff = light.shadow.y >= 0.0f && light.shadow.z > 0.0f;
    float hitDistance = 0.0f;
    if (falloff) {
        // The shadow falloff reads the committed hit distance. With
        // TerminateOnFirstHit that is whichever candidate the driver found
        // first; here it is the closest confirmed hit, which is defined.
        Hit hit;
        if (!TraceClosest(*c.scene, *c.bvh, origin, direction, 0.001f, traceDistance, mode, 0u, &hit)) {
            return V3(1.0f);
        }
        hitDistance = hit.t;
    } else if (!TraceAny(*c.scene, *c.bvh, origin, direction, 0.001f, traceDistance, mode)) {
        return V3(1.0f);
    }
    float strength = 1.0f;
    if (falloff) {
        const float falloffDistance = gmin(light.shadow.z, gmax(light.shadow.y, 0.0f));
        strength = clampf((light.shadow.y - hitDistance) / gmax(falloffDistance, 1e-6f), 0.0f, 1.0f);
        strength = gpow(strength, gmax(light.shadow.w, 0.0f));
    }
    return mix(V3(1.0f), xyz(light.shadowColor), strength);
}

bool meshLightVisible(const Ctx& c, vec3 origin, vec3 direction, float maximumDistance)
{
    // :891-912
    if (maximumDistance <= 0.001f) return true;
    c.counters->shadowRays++;
    const AcceptMode mode = sceneOpaque(c) ? AcceptMode::Opaque : AcceptMode::Threshold;
    return !TraceAny(*c.scene, *c.bvh, origin, direction, 0.001f, maximumDistance, mode);
}

uint32_t sampleEmissiveTriangle(const Ctx& c, float target, uint32_t primitiveCount)
{
    // :914-924
    uint32_t low = 0u;
    uint32_t high = primitiveCount - 1u;
    while (low < high) {
        const uint32_t middle = low + (high - low) / 2u;
        if (target <= c.scene->emissive[middle].x) high = middle;
        else low = middle + 1u;
    }
    return low;
}

float emissiveTrianglePdf(const Ctx& c, uint32_t primitive, float distanceSquared, float emissionCosine)
{
    // :926-931
    if (emissionCosine <= 0.0f) return 0.0f;
    return c.scene->emissive[primitive].y * distanceSquared / emissionCosine;
}

// ---------------------------------------------------------------------------
// Diffuse and layered surface evaluation (vulkan_path_tracer.cpp:933-1069)
// ---------------------------------------------------------------------------
float eonDirectionalAlbedo(float nDotDirection, float roughness)
{
    const float c1 = 0.2877934092f;
    const float cosine = clampf(nDotDirection, 0.0f, 1.0f);
    const float sine = std::sqrt(gmax(1.0f - cosine * cosine, 0.0f));
    const float theta = gacos(cosine);
    const float sineCubed = sine * sine * sine;
    const float g = sine * (theta - sine * cosine) +
                    (2.0f / 3.0f) * (sine * (1.0f - sineCubed) / gmax(cosine, 1e-5f) - sine);
    const float a = 1.0f / (1.0f + c1 * roughness);
    return clampf(a + roughness * a * g / kPi, 0.0f, 1.0f);
}

vec3 evaluateDiffuseReflection(vec3 normal, vec3 viewDirection, vec3 lightDirection, vec3 diffuseColor,
                               float roughness, uint32_t model)
{
    // :946-1009
    const float nDotL = gmax(dot(normal, lightDirection), 0.0f);
    const float nDotV = gmax(dot(normal, viewDirection), 0.0f);
    if (nDotL <= 0.0f || nDotV <= 0.0f) return V3(0.0f);
    if (model == 1u) {
        const float sigma = clampf(roughness, 0.0f, 1.0f);
        const float sigmaSquared = sigma * sigma;
        const float a = 1.0f - 0.5f * sigmaSquared / (sigmaSquared + 0.33f);
        const float b = 0.45f * sigmaSquared / (sigmaSquared + 0.09f);
        const vec3 projectedLight = lightDirection - normal * nDotL;
        const vec3 projectedView = viewDirection - normal * nDotV;
        float azimuth = 0.0f;
        if (dot(projectedLight, projectedLight) > 1e-8f && dot(projectedView, projectedView) > 1e-8f) {
            azimuth = gmax(dot(normalize(projectedLight), normalize(projectedView)), 0.0f);
        }
        const float sinLight = std::sqrt(gmax(1.0f - nDotL * nDotL, 0.0f));
        const float sinView = std::sqrt(gmax(1.0f - nDotV * nDotV, 0.0f));
        const float sinAlpha = gmax(sinLight, sinView);
        const float tanBeta = gmin(sinLight / gmax(nDotL, 1e-5f), sinView / gmax(nDotV, 1e-5f));
        return V3(nDotL * (a + b * azimuth * sinAlpha * tanBeta) / kPi);
    }
    if (model == 2u) {
        const vec3 halfway = normalize(viewDirection + lightDirection);
        const float lDotH = gmax(dot(lightDirection, halfway), 0.0f);
        const float grazing = 0.5f + 2.0f * clampf(roughness, 0.0f, 1.0f) * lDotH * lDotH;
        const float lightScatter = 1.0f + (grazing - 1.0f) * gpow(1.0f - nDotL, 5.0f);
        const float viewScatter = 1.0f + (grazing - 1.0f) * gpow(1.0f - nDotV, 5.0f);
        return V3(nDotL * lightScatter * viewScatter / kPi);
    }
    if (model == 3u) {
        const float c1 = 0.2877934092f;
        const float c2 = 0.0726760455f;
        const float sigma = clampf(roughness, 0.0f, 1.0f);
        const float a = 1.0f / (1.0f + c1 * sigma);
        const float s = dot(lightDirection, viewDirection) - nDotL * nDotV;
        const float sOverT = s > 0.0f ? s / gmax(nDotL, nDotV) : s;
        const float singleScatter = a * (1.0f + sigma * sOverT);
        const float averageAlbedo = (1.0f + c2 * sigma) / (1.0f + c1 * sigma);
        const float outgoingAlbedo = eonDirectionalAlbedo(nDotV, sigma);
        const float incidentAlbedo = eonDirectionalAlbedo(nDotL, sigma);
        const float directionalFactor =
            (1.0f - outgoingAlbedo) * (1.0f - incidentAlbedo) / gmax(1.0f - averageAlbedo, 1e-5f);
        const vec3 rho = clamp3(diffuseColor, V3(0.0f), V3(0.9999f));
        const vec3 multipleScatterOverRho =
            rho * averageAlbedo / gmax(V3(1.0f) - rho * (1.0f - averageAlbedo), V3(1e-5f));
        return nDotL / kPi * (V3(singleScatter) + multipleScatterOverRho * directionalFactor);
    }
    return V3(nDotL / kPi);
}

struct SurfaceParams {
    vec3 diffuseColor;
    float transmission, subsurface, diffuseWeight, diffuseRoughness;
    uint32_t diffuseModel;
    float translucentWeight;
    vec3 translucentColor;
    float metalness;
    vec2 roughness;
    vec3 f0;
    float coat;
    vec2 coatRoughness;
    vec3 coatF0;
    float sheen;
    vec3 sheenColor;
    float sheenRoughness;
    bool sheenZeltner;
};

vec3 evaluateDirectSurface(vec3 normal, vec3 tangent, vec3 viewDirection, vec3 lightDirection,
                           const SurfaceParams& p, float diffuseScale, float specularScale)
{
    // :1013-1069
    const float signedNdotL = dot(normal, lightDirection);
    const float nDotL = gmax(signedNdotL, 0.0f);
    const float backNdotL = gmax(-signedNdotL, 0.0f);
    const float wrappedNdotL = gmax((signedNdotL + 0.5f * p.subsurface) / (1.0f + 0.5f * p.subsurface), 0.0f);
    if (wrappedNdotL <= 0.0f && nDotL <= 0.0f && backNdotL * p.translucentWeight <= 0.0f) return V3(0.0f);
    const vec3 halfway = nDotL > 0.0f ? normalize(viewDirection + lightDirection) : normal;
    const vec3 baseFresnel = fresnelSchlick(gmax(dot(viewDirection, halfway), 0.0f), p.f0);
    const vec3 diffuseResponse =
        mix(evaluateDiffuseReflection(normal, viewDirection, lightDirection, p.diffuseColor, p.diffuseRoughness,
                                      p.diffuseModel),
            V3(wrappedNdotL / kPi), p.subsurface);
    const vec3 diffuse = diffuseScale * (V3(1.0f) - baseFresnel) * p.diffuseWeight * (1.0f - p.translucentWeight) *
                         (1.0f - p.metalness) * p.diffuseColor * diffuseResponse * (1.0f - p.transmission);
    const vec3 viewFresnel = fresnelSchlick(gmax(dot(normal, viewDirection), 0.0f), p.f0);
    const vec3 translucent = diffuseScale * (V3(1.0f) - viewFresnel) * p.translucentWeight *
                             (1.0f - p.metalness) * p.translucentColor * (backNdotL / kPi) *
                             (1.0f - p.transmission);
    const vec3 specular = specularScale * nDotL *
                          evaluateGGXAnisotropic(normal, tangent, viewDirection, lightDirection, p.roughness, p.f0);
    vec3 coatFresnel = V3(0.0f);
    vec3 coatSpecular = V3(0.0f);
    if (p.coat > 0.0f) {
        coatFresnel = fresnelSchlick(gmax(dot(viewDirection, halfway), 0.0f), p.coatF0);
        coatSpecular = specularScale * p.coat * nDotL *
                       evaluateGGXAnisotropic(normal, tangent, viewDirection, lightDirection, p.coatRoughness,
                                              p.coatF0);
    }
    const vec3 baseLayer = (V3(1.0f) - p.coat * coatFresnel) * (diffuse + translucent + specular) + coatSpecular;
    const float sheenAlbedo = p.sheenZeltner
                                  ? sheenZeltnerDirectionalAlbedo(gmax(dot(normal, viewDirection), 0.0f), p.sheenRoughness)
                                  : sheenDirectionalAlbedo(gmax(dot(normal, viewDirection), 0.0f), p.sheenRoughness);
    const vec3 sheenLayer = specularScale * p.sheen * p.sheenColor *
                            sheenResponse(normal, viewDirection, lightDirection, p.sheenRoughness, p.sheenZeltner);
    return baseLayer * (1.0f - clampf(p.sheen * sheenAlbedo, 0.0f, 1.0f)) + sheenLayer;
}

vec3 offsetSurfaceOrigin(vec3 position, vec3 geometricNormal, vec3 direction)
{
    // :1071-1075
    const float side = dot(geometricNormal, direction) >= 0.0f ? 1.0f : -1.0f;
    return position + geometricNormal * (0.002f * side);
}

float shapingConeFactor(const GpuLight& light, float cosine)
{
    // :1085-1094
    const float angle = gacos(clampf(cosine, -1.0f, 1.0f));
    const float outer = radians(clampf(light.shaping.y, 0.0f, 180.0f));
    const float inner = outer * (1.0f - clampf(light.shaping.z, 0.0f, 1.0f));
    return outer >= 3.1415925f ? 1.0f
                               : (outer <= inner + 1e-6f ? (angle <= outer ? 1.0f : 0.0f)
                                                         : 1.0f - smoothstep(inner, outer, angle));
}

float dispersedIor(float iorAtD, float scale, float abbeNumber, float wavelength)
{
    // :1096-1110
    if (scale <= 0.0f || abbeNumber <= 1.0f) return iorAtD;
    const float lambdaF = 486.13f;
    const float lambdaD = 587.56f;
    const float lambdaC = 656.27f;
    const float reciprocalDelta = 1.0f / (lambdaF * lambdaF) - 1.0f / (lambdaC * lambdaC);
    const float b = (iorAtD - 1.0f) / gmax(abbeNumber * reciprocalDelta, 1e-8f);
    const float a = iorAtD - b / (lambdaD * lambdaD);
    const float cauchyIor = a + b / (wavelength * wavelength);
    return mix(iorAtD, cauchyIor, clampf(scale, 0.0f, 1.0f));
}

vec3 sampleHenyeyGreenstein(vec3 forward, float anisotropy, uint32_t& state)
{
    // :1112-1128
    const float g = clampf(anisotropy, -0.95f, 0.95f);
    const float u = randomFloat(state);
    const float cosine = std::fabs(g) < 1e-3f
                             ? 1.0f - 2.0f * u
                             : (1.0f + g * g - gpow((1.0f - g * g) / (1.0f - g + 2.0f * g * u), 2.0f)) / (2.0f * g);
    const float sine = std::sqrt(gmax(1.0f - cosine * cosine, 0.0f));
    const float phi = kTwoPi * randomFloat(state);
    const vec3 w = normalize(forward);
    const vec3 tangent = tangentFrameAxis(w);
    const vec3 bitangent = cross(w, tangent);
    return normalize(tangent * (gcos(phi) * sine) + bitangent * (gsin(phi) * sine) + w * cosine);
}

bool traceOpaqueBoundary(const Ctx& c, vec3 origin, vec3 direction, vec3& boundary, vec3& boundaryNormal,
                         float& boundaryDistance)
{
    // :1130-1151
    c.counters->subsurfaceRays++;
    Hit hit;
    if (!TraceClosest(*c.scene, *c.bvh, origin, direction, 0.001f, 10000.0f, AcceptMode::Opaque, 0u, &hit)) {
        return false;
    }
    const PackedScene& s = *c.scene;
    const uint32_t primitive = hit.primitive;
    const vec3 p0 = xyz(s.vertices[s.indices[primitive * 3u + 0u]]);
    const vec3 p1 = xyz(s.vertices[s.indices[primitive * 3u + 1u]]);
    const vec3 p2 = xyz(s.vertices[s.indices[primitive * 3u + 2u]]);
    boundaryDistance = hit.t;
    boundary = origin + direction * boundaryDistance;
    boundaryNormal = normalize(cross(p1 - p0, p2 - p0));
    if (dot(boundaryNormal, direction) > 0.0f) boundaryNormal = -boundaryNormal;
    return true;
}

bool randomWalkSubsurface(const Ctx& c, vec3 entry, vec3 outwardNormal, float meanFreePath, float albedo,
                          float anisotropy, uint32_t& state, vec3& exitOrigin, vec3& exitDirection,
                          float& attenuation)
{
    // :1153-1186
    const float radius = gmax(meanFreePath, 0.001f);
    const float sigmaS = 1.0f / radius;
    const float sigmaA = -glog(clampf(albedo, 0.001f, 0.9999f)) / radius;
    vec3 origin = entry - outwardNormal * 0.003f;
    vec3 direction = cosineHemisphere(-outwardNormal, state);
    attenuation = 1.0f;
    for (int step = 0; step < 8; ++step) {
        vec3 boundary;
        vec3 boundaryNormal;
        float boundaryDistance;
        if (!traceOpaqueBoundary(c, origin, direction, boundary, boundaryNormal, boundaryDistance)) return false;
        const float scatterDistance = -glog(gmax(1.0f - randomFloat(state), 1e-6f)) / sigmaS;
        const bool forceExit = step == 7;
        const float travel = forceExit ? boundaryDistance : gmin(scatterDistance, boundaryDistance);
        attenuation *= gexp(-sigmaA * travel);
        if (forceExit || scatterDistance >= boundaryDistance) {
            exitDirection = direction;
            exitOrigin = boundary + direction * 0.003f;
            return true;
        }
        origin += direction * scatterDistance;
        direction = sampleHenyeyGreenstein(direction, anisotropy, state);
    }
    return false;
}

// Returns the scalar radiance of one wavelength lane (vulkan_path_tracer.cpp:
// 1202-1880; the GLSL radiance vec3 holds the same value in every component).
float TraceLane(const Ctx& c, uint32_t index, uint32_t px, uint32_t py, uint32_t sampleNumber,
                uint32_t spectralLane, float* wavelengthOut)
{
    const PackedScene& s = *c.scene;
    uint32_t rng = hashState(index ^ (sampleNumber * 0x9e3779b9u) ^ 0xa511e9b3u);
    const float wavelengthShift = uintToFloat(hashState(index ^ 0x68bc21ebu)) * (1.0f / 4294967296.0f);
    const float wavelength =
        380.0f + 400.0f * fract(wavelengthShift + (uintToFloat(sampleNumber & 31u) + 0.5f) / 32.0f +
                                uintToFloat(spectralLane) / 3.0f);
    *wavelengthOut = wavelength;
    const float jx = randomFloat(rng);
    const float jy = randomFloat(rng);
    const vec2 uv = V2((uintToFloat(px) + jx) / uintToFloat(c.frame[0]), (uintToFloat(py) + jy) / uintToFloat(c.frame[1]));

    vec3 rayOrigin = xyz(c.origin);
    vec3 rayDirection = normalize(xyz(c.lowerLeft) + uv.x * xyz(c.horizontal) + uv.y * xyz(c.vertical) - rayOrigin);
    vec3 throughput = V3(1.0f);
    vec3 radiance = V3(0.0f);
    bool environmentOnMiss = true;
    bool previousWasDelta = true;
    float previousBsdfPdf = 0.0f;
    float previousEnvironmentLightPdf = 0.0f;
    bool insideMedium = false;
    float mediumAbsorption = 0.0f;
    float mediumScattering = 0.0f;
    float mediumAnisotropy = 0.0f;

    const int maxBounces = static_cast<int>(std::clamp(c.frame[3] & 0xffu, 1u, 12u));
    for (int bounce = 0; bounce < maxBounces; ++bounce) {
        c.counters->extensionRays++;
        Hit hit;
        const AcceptMode mode = sceneOpaque(c) ? AcceptMode::Opaque : AcceptMode::Stochastic;
        const bool found = TraceClosest(s, *c.bvh, rayOrigin, rayDirection, 0.001f, 10000.0f, mode, rng, &hit);
        if (!found) {
            if (environmentOnMiss) {
                const float misWeight =
                    previousWasDelta ? 1.0f : powerHeuristic(previousBsdfPdf, previousEnvironmentLightPdf);
                radiance += throughput * misWeight * V3(illuminantSpectrum(environment(c, rayDirection), wavelength));
            }
            break;
        }

        const uint32_t primitive = hit.primitive;
        const uint32_t i0 = s.indices[primitive * 3u + 0u];
        const uint32_t i1 = s.indices[primitive * 3u + 1u];
        const uint32_t i2 = s.indices[primitive * 3u + 2u];
        const vec3 p0 = xyz(s.vertices[i0]);
        const vec3 p1 = xyz(s.vertices[i1]);
        const vec3 p2 = xyz(s.vertices[i2]);
        const vec3 geometricNormal = normalize(cross(p1 - p0, p2 - p0));
        const bool frontFace = dot(geometricNormal, rayDirection) < 0.0f;
        const vec3 orientedGeometricNormal = frontFace ? geometricNormal : -geometricNormal;

        const vec2 barycentrics = hit.barycentrics;
        const vec3 authoredNormal = surfaceShadingNormal(s, primitive, barycentrics, geometricNormal);
        vec3 normal = frontFace ? authoredNormal : -authoredNormal;
        const vec2 uv0 = s.texcoords[primitive * 3u + 0u];
        const vec2 uv1 = s.texcoords[primitive * 3u + 1u];
        const vec2 uv2 = s.texcoords[primitive * 3u + 2u];
        const vec2 surfaceUv = surfaceTextureCoordinates(s, primitive, barycentrics);

        const float distance = hit.t;
        const vec3 hitPoint = rayOrigin + rayDirection * distance;
        if (insideMedium) {
            if (mediumScattering > 0.0f) {
                const float scatterDistance = -glog(gmax(1.0f - randomFloat(rng), 1e-6f)) / mediumScattering;
                if (scatterDistance < distance) {
                    throughput *= gexp(-mediumAbsorption * scatterDistance);
                    rayOrigin += rayDirection * scatterDistance;
                    rayDirection = sampleHenyeyGreenstein(rayDirection, mediumAnisotropy, rng);
                    environmentOnMiss = true;
                    previousWasDelta = true;
                    previousBsdfPdf = 0.0f;
                    continue;
                }
            }
            throughput *= gexp(-mediumAbsorption * distance);
        }
        const GpuMaterial& material = s.materials[s.triangleMaterials[primitive]];
        vec3 baseColorRgb = xyz(material.baseColorMetalness);
        if (material.textureIndices0[0] != 0xffffffffu) {
            const vec4 baseColorSample =
                sampleMaterialTexture(c, material.textureIndices0[0], surfaceUv, V4(baseColorRgb, 1.0f));
            const int channel = static_cast<int>(std::round(material.baseColorTextureScale.w));
            const float* comps = &baseColorSample.x;
            const vec3 sourceColor =
                channel < 0 ? xyz(baseColorSample) : V3(comps[std::clamp(channel, 0, 3)]);
            baseColorRgb = xyz(material.baseColorTextureBias) + xyz(material.baseColorTextureScale) * sourceColor;
        }
        const vec3 baseColor = V3(reflectanceSpectrum(baseColorRgb, wavelength));
        const float metalness = clampf(
            sampleMaterialTexture(c, material.textureIndices0[1], surfaceUv, V4(material.baseColorMetalness.w)).x,
            0.0f, 1.0f);
        const vec4 roughnessSample = sampleMaterialTexture(
            c, material.textureIndices0[2], surfaceUv,
            V4(material.emissionRoughness.w, material.subsurfaceColor.w, 0.0f, 1.0f));
        const vec2 roughness =
            clamp2(V2(roughnessSample.x, roughnessSample.y), V2(0.02f, 0.02f), V2(1.0f, 1.0f));
        const float diffuseRoughness = clampf(
            sampleMaterialTexture(c, material.textureIndices4[2], surfaceUv, V4(material.diffuseProperties.x)).x,
            0.0f, 1.0f);
        const float diffuseWeight = clampf(
            sampleMaterialTexture(c, material.textureIndices4[3], surfaceUv, V4(material.diffuseProperties.z)).x,
            0.0f, 1.0f);
        const uint32_t diffuseModel = static_cast<uint32_t>(material.diffuseProperties.y + 0.5f);
        normal = applyNormalMap(c, material.textureIndices1[1], material.coatWeightRoughnessIor.w > 0.5f,
                                material.subsurfaceWeightScale.w, surfaceUv, normal, p0, p1, p2, uv0, uv1, uv2);
        const vec3 tangent = surfaceTangent(normal, p0, p1, p2, uv0, uv1, uv2);
        const vec3 emissionRgb = surfaceEmissionRgb(c, primitive, surfaceUv);
        const vec3 emission = V3(illuminantSpectrum(emissionRgb, wavelength));
        float emissionMisWeight = 1.0f;
        if (!previousWasDelta && anyGreaterThanZero(emissionRgb)) {
            const float emissionCosine = std::fabs(dot(geometricNormal, -rayDirection));
            const float lightPdf = emissiveTrianglePdf(c, primitive, distance * distance, emissionCosine);
            emissionMisWeight = powerHeuristic(previousBsdfPdf, lightPdf);
        }
        radiance += throughput * emission * emissionMisWeight;

        const float transmission = clampf(material.transmissionOpacityIor.x, 0.0f, 1.0f);
        vec3 transmissionColorRgb = xyz(material.transmissionColorThinWalled);
        if (transmission > 0.0f) {
            transmissionColorRgb =
                xyz(sampleMaterialTexture(c, material.textureIndices1[2], surfaceUv, V4(transmissionColorRgb, 1.0f)));
        }
        const vec3 transmissionColor = V3(reflectanceSpectrum(transmissionColorRgb, wavelength));
        float subsurface = 0.0f;
        vec3 diffuseColor = baseColor;
        vec3 subsurfaceColorRgb = xyz(material.subsurfaceColor);
        vec3 subsurfaceRadiusRgb = gmax(xyz(material.subsurfaceRadius), V3(0.001f));
        if (material.subsurfaceWeightScale.x > 0.0f || material.textureIndices2[0] != 0xffffffffu) {
            subsurface = clampf(sampleMaterialTexture(c, material.textureIndices2[0], surfaceUv,
                                                      V4(material.subsurfaceWeightScale.x)).x,
                                0.0f, 1.0f);
            if (subsurface > 0.0f) {
                subsurfaceColorRgb = xyz(sampleMaterialTexture(c, material.textureIndices2[1], surfaceUv,
                                                               V4(xyz(material.subsurfaceColor), 1.0f)));
                subsurfaceRadiusRgb = gmax(xyz(sampleMaterialTexture(c, material.textureIndices2[2], surfaceUv,
                                                                     V4(xyz(material.subsurfaceRadius), 1.0f))),
                                           V3(0.001f));
                const vec3 subsurfaceColor = V3(reflectanceSpectrum(subsurfaceColorRgb, wavelength));
                diffuseColor = mix(baseColor, subsurfaceColor, subsurface);
            }
        }
        const float ior = dispersedIor(gmax(material.transmissionOpacityIor.z, 1.0001f), material.transmissionMedium.z,
                                       material.transmissionMedium.w, wavelength);
        const float specularWeight = clampf(
            sampleMaterialTexture(c, material.textureIndices3[0], surfaceUv, V4(material.specularWeightColor.x)).x,
            0.0f, 1.0f);
        const vec3 specularColorRgb = xyz(sampleMaterialTexture(
            c, material.textureIndices3[1], surfaceUv,
            V4(material.specularWeightColor.y, material.specularWeightColor.z, material.specularWeightColor.w, 1.0f)));
        const vec3 specularColor = V3(reflectanceSpectrum(specularColorRgb, wavelength));
        float dielectricReflectance = (ior - 1.0f) / (ior + 1.0f);
        dielectricReflectance *= dielectricReflectance;
        const vec3 f0 = mix(clamp3(V3(dielectricReflectance * specularWeight) * specularColor, V3(0.0f), V3(1.0f)),
                            baseColor, metalness);
        float coat = 0.0f;
        vec2 coatRoughness = V2(material.coatWeightRoughnessIor.y, material.subsurfaceRadius.w);
        vec3 coatF0 = V3(0.0f);
        if (material.coatWeightRoughnessIor.x > 0.0f || material.textureIndices3[2] != 0xffffffffu) {
            coat = clampf(sampleMaterialTexture(c, material.textureIndices3[2], surfaceUv,
                                                V4(material.coatWeightRoughnessIor.x)).x,
                          0.0f, 1.0f);
            if (coat > 0.0f) {
                const vec3 coatColorRgb = xyz(sampleMaterialTexture(c, material.textureIndices3[3], surfaceUv,
                                                                    V4(xyz(material.coatColor), 1.0f)));
                const vec3 coatColor = V3(reflectanceSpectrum(coatColorRgb, wavelength));
                const vec4 coatRoughnessSample = sampleMaterialTexture(
                    c, material.textureIndices4[0], surfaceUv, V4(coatRoughness.x, coatRoughness.y, 0.0f, 1.0f));
                coatRoughness = clamp2(V2(coatRoughnessSample.x, coatRoughnessSample.y), V2(0.02f, 0.02f),
                                       V2(1.0f, 1.0f));
                const float coatIor = gmax(material.coatWeightRoughnessIor.z, 1.0001f);
                float coatReflectance = (coatIor - 1.0f) / (coatIor + 1.0f);
                coatReflectance *= coatReflectance;
                coatF0 = clamp3(V3(coatReflectance) * coatColor, V3(0.0f), V3(1.0f));
            }
        }

        const float sheen = clampf(
            sampleMaterialTexture(c, material.textureIndices1[3], surfaceUv, V4(material.coatColor.w)).x, 0.0f, 1.0f);
        const vec3 sheenColorRgb = xyz(sampleMaterialTexture(c, material.textureIndices2[3], surfaceUv,
                                                             V4(xyz(material.sheenColorMode), 1.0f)));
        const vec3 sheenColor = V3(reflectanceSpectrum(sheenColorRgb, wavelength));
        const float sheenRoughness =
            clampf(sampleMaterialTexture(c, material.textureIndices4[1], surfaceUv, V4(material.transmissionScatter.w)).x,
                   0.01f, 1.0f);
        const bool sheenZeltner = material.sheenColorMode.w > 0.5f;
        const float translucentWeight =
            clampf(sampleMaterialTexture(c, material.textureIndices5[0], surfaceUv,
                                         V4(material.translucentColorWeight.w)).x,
                   0.0f, 1.0f);
        const vec3 translucentColorRgb = xyz(sampleMaterialTexture(
            c, material.textureIndices5[1], surfaceUv, V4(xyz(material.translucentColorWeight), 1.0f)));
        const vec3 translucentColor = V3(reflectanceSpectrum(translucentColorRgb, wavelength));

        const vec3 viewDirection = normalize(-rayDirection);
        const float sheenAlbedo = sheenZeltner
                                      ? sheenZeltnerDirectionalAlbedo(gmax(dot(normal, viewDirection), 0.0f), sheenRoughness)
                                      : sheenDirectionalAlbedo(gmax(dot(normal, viewDirection), 0.0f), sheenRoughness);
        const float sheenProbability = clampf(sheen * sheenAlbedo * luminance(sheenColor), 0.0f, 0.95f);
        const vec3 coatContribution =
            coat > 0.0f ? coat * fresnelSchlick(gmax(dot(normal, viewDirection), 0.0f), coatF0) : V3(0.0f);
        const float coatProbability = clampf(luminance(coatContribution), 0.0f, 0.95f);
        const vec3 baseFresnel = fresnelSchlick(gmax(dot(normal, viewDirection), 0.0f), f0);
        const vec3 specularContribution = baseFresnel;
        const vec3 diffuseContribution = (V3(1.0f) - baseFresnel) * diffuseWeight * (1.0f - translucentWeight) *
                                         (1.0f - metalness) * diffuseColor;
        const vec3 translucentContribution =
            (V3(1.0f) - baseFresnel) * translucentWeight * (1.0f - metalness) * translucentColor;
        const float specularEnergy = luminance(specularContribution);
        const float diffuseEnergy = luminance(diffuseContribution);
        const float translucentEnergy = luminance(translucentContribution);
        const float baseEnergy = diffuseEnergy + translucentEnergy;
        const float specularProbability =
            clampf(specularEnergy / gmax(specularEnergy + baseEnergy, 1e-5f), 0.05f, 0.95f);
        const float translucentProbability = baseEnergy > 1e-5f ? translucentEnergy / baseEnergy : 0.0f;
        const uint32_t lightCount = lightCountOf(c);
        const bool hasMeshLights = hasEmissiveTriangles(c);

        SurfaceParams sp;
        sp.diffuseColor = diffuseColor;
        sp.transmission = transmission;
        sp.subsurface = subsurface;
        sp.diffuseWeight = diffuseWeight;
        sp.diffuseRoughness = diffuseRoughness;
        sp.diffuseModel = diffuseModel;
        sp.translucentWeight = translucentWeight;
        sp.translucentColor = translucentColor;
        sp.metalness = metalness;
        sp.roughness = roughness;
        sp.f0 = f0;
        sp.coat = coat;
        sp.coatRoughness = coatRoughness;
        sp.coatF0 = coatF0;
        sp.sheen = sheen;
        sp.sheenColor = sheenColor;
        sp.sheenRoughness = sheenRoughness;
        sp.sheenZeltner = sheenZeltner;

        if (lightCount > 0u) {
            // :1469-1592
            const float directSpecularEnergy = specularEnergy + luminance(coatContribution) + sheenProbability;
            uint32_t lightIndex;
            float lightSelectionPdf;
            sampleAnalyticLight(c, hitPoint, normal, diffuseEnergy, directSpecularEnergy, translucentEnergy, rng,
                                lightIndex, lightSelectionPdf);
            const GpuLight& light = s.lights[lightIndex];
            vec3 lightDirection = V3(0.0f, 1.0f, 0.0f);
            vec3 lightRadiance = V3(0.0f);
            float inversePdf = 0.0f;
            float maximumShadowDistance = 10000.0f;
            if (light.textureInfo[2] == 0u) {
                float lightPdf = 0.0f;
                sampleDomeLight(c, light, rng, lightDirection, lightPdf);
                lightRadiance = sampleDome(c, light, lightDirection);
                inversePdf = lightPdf > 0.0f ? 1.0f / lightPdf : 0.0f;
            } else if (light.textureInfo[2] == 5u) {
                const float halfAngle = 0.5f * radians(clampf(light.geometry.z, 0.0f, 359.999f));
                if (halfAngle <= 1e-6f) {
                    lightDirection = normalize(xyz(light.basisZ));
                    inversePdf = 1.0f;
                } else {
                    const float cosineMaximum = gcos(halfAngle);
                    const float cosineTheta = mix(cosineMaximum, 1.0f, randomFloat(rng));
                    const float sineTheta = std::sqrt(gmax(1.0f - cosineTheta * cosineTheta, 0.0f));
                    const float phi = kTwoPi * randomFloat(rng);
                    lightDirection = normalize(xyz(light.basisX) * (gcos(phi) * sineTheta) +
                                               xyz(light.basisY) * (gsin(phi) * sineTheta) +
                                               xyz(light.basisZ) * cosineTheta);
                    inversePdf = 1.0f;
                }
                lightRadiance = xyz(light.colorIntensity) * light.colorIntensity.w;
            } else {
                const float lu = randomFloat(rng);
                const float lv = randomFloat(rng);
                const vec2 lightUv = V2(lu, lv);
                vec3 lightPosition = xyz(light.position);
                vec3 lightNormal = -normalize(xyz(light.basisZ));
                if (light.textureInfo[2] == 1u) {
                    lightPosition += (lightUv.x - 0.5f) * xyz(light.axisU) + (lightUv.y - 0.5f) * xyz(light.axisV);
                } else if (light.textureInfo[2] == 2u) {
                    const float diskRadius = std::sqrt(lightUv.x);
                    const float diskPhi = kTwoPi * lightUv.y;
                    lightPosition += diskRadius * (gcos(diskPhi) * xyz(light.axisU) + gsin(diskPhi) * xyz(light.axisV));
                } else if (light.textureInfo[2] == 3u) {
                    lightNormal = uniformSphere(rng);
                    lightPosition += light.geometry.x * lightNormal;
                } else if (light.textureInfo[2] == 4u) {
                    const float cylinderPhi = kTwoPi * lightUv.y;
                    lightNormal = normalize(gcos(cylinderPhi) * xyz(light.basisY) + gsin(cylinderPhi) * xyz(light.basisZ));
                    lightPosition += (lightUv.x - 0.5f) * xyz(light.axisU) + light.geometry.x * lightNormal;
                }
                const vec3 toLight = lightPosition - hitPoint;
                const float distanceSquared = dot(toLight, toLight);
                const float lightDistance = std::sqrt(gmax(distanceSquared, 1e-8f));
                lightDirection = toLight / lightDistance;
                const float emissionCosine = gmax(dot(lightNormal, -lightDirection), 0.0f);
                if (emissionCosine > 0.0f && light.controls.w > 0.0f) {
                    const float shapingCosine = gmax(dot(normalize(xyz(light.basisZ)), lightDirection), 0.0f);
                    const float focus = gpow(shapingCosine, gmax(light.shaping.x, 0.0f));
                    const vec3 focusColor = mix(xyz(light.focusTint), V3(1.0f), focus);
                    const vec3 textureValue =
                        light.textureInfo[2] != 1u || light.textureInfo[0] == 0xffffffffu
                            ? V3(1.0f)
                            : xyz(textureSample(c, light.textureInfo[0], lightUv));
                    lightRadiance = xyz(light.colorIntensity) * light.colorIntensity.w * textureValue * focusColor *
                                    shapingConeFactor(light, shapingCosine);
                    inversePdf = light.controls.w * emissionCosine / gmax(distanceSquared, 1e-8f);
                    maximumShadowDistance = gmax(lightDistance - 0.003f, 0.001f);
                }
            }
            if (inversePdf > 0.0f) {
                const vec3 direct = evaluateDirectSurface(normal, tangent, viewDirection, lightDirection, sp,
                                                          light.controls.x, light.controls.y);
                if (anyGreaterThanZero(direct)) {
                    const vec3 visibility =
                        shadowVisibility(c, offsetSurfaceOrigin(hitPoint, orientedGeometricNormal, lightDirection),
                                         lightDirection, maximumShadowDistance, light);
                    const vec3 spectralLight = V3(illuminantSpectrum(lightRadiance, wavelength));
                    const vec3 spectralVisibility = V3(reflectanceSpectrum(visibility, wavelength));
                    const float misWeight =
                        light.textureInfo[2] == 0u
                            ? powerHeuristic(environmentLightPdf(c, hitPoint, normal, lightDirection, diffuseEnergy,
                                                                 directSpecularEnergy, translucentEnergy),
                                             surfaceReflectionPdf(normal, tangent, viewDirection, lightDirection,
                                                                  roughness, coatRoughness, sheenProbability,
                                                                  coatProbability, specularProbability,
                                                                  translucentProbability))
                            : 1.0f;
                    radiance += throughput * direct * spectralLight * spectralVisibility * inversePdf * misWeight /
                                gmax(lightSelectionPdf, 1e-8f);
                }
            }
        } else if (!hasMeshLights) {
            // :1593-1668 fallback sun and sky
            const bool zUp = c.vertical.w > 0.5f;
            const vec3 up = zUp ? V3(0.0f, 0.0f, 1.0f) : V3(0.0f, 1.0f, 0.0f);
            const vec3 azimuth = zUp ? normalize(V3(1.0f, 1.0f, 0.0f)) : normalize(V3(1.0f, 0.0f, 1.0f));
            const vec3 sunDirection = normalize(up * 0.9659258f + azimuth * 0.2588190f);
            const vec3 direct = evaluateDirectSurface(normal, tangent, viewDirection, sunDirection, sp, 1.0f, 1.0f);
            if (anyGreaterThanZero(direct)) {
                const vec3 visibility =
                    shadowVisibility(c, offsetSurfaceOrigin(hitPoint, orientedGeometricNormal, sunDirection),
                                     sunDirection, 10000.0f, s.lights[0]);
                const vec3 sunRadiance = V3(3.45575f, 3.14159f, 2.82743f);
                const vec3 spectralSun = V3(illuminantSpectrum(sunRadiance, wavelength));
                const vec3 spectralVisibility = V3(reflectanceSpectrum(visibility, wavelength));
                radiance += throughput * direct * spectralSun * spectralVisibility;
            }
            const vec3 skyDirection = cosineHemisphere(normal, rng);
            const vec3 skyDirect = evaluateDirectSurface(normal, tangent, viewDirection, skyDirection, sp, 1.0f, 0.0f);
            if (anyGreaterThanZero(skyDirect)) {
                const vec3 visibility =
                    shadowVisibility(c, offsetSurfaceOrigin(hitPoint, orientedGeometricNormal, skyDirection),
                                     skyDirection, 10000.0f, s.lights[0]);
                const vec3 spectralSky = V3(illuminantSpectrum(environment(c, skyDirection), wavelength));
                const vec3 spectralVisibility = V3(reflectanceSpectrum(visibility, wavelength));
                radiance += throughput * skyDirect * spectralSky * spectralVisibility *
                            (kPi / gmax(dot(normal, skyDirection), 1e-4f));
            }
            if (translucentWeight > 0.0f) {
                const vec3 backSkyDirection = cosineHemisphere(-normal, rng);
                const vec3 backSkyDirect =
                    evaluateDirectSurface(normal, tangent, viewDirection, backSkyDirection, sp, 1.0f, 0.0f);
                if (anyGreaterThanZero(backSkyDirect)) {
                    const vec3 visibility = shadowVisibility(
                        c, offsetSurfaceOrigin(hitPoint, orientedGeometricNormal, backSkyDirection),
                        backSkyDirection, 10000.0f, s.lights[0]);
                    const vec3 spectralSky = V3(illuminantSpectrum(environment(c, backSkyDirection), wavelength));
                    const vec3 spectralVisibility = V3(reflectanceSpectrum(visibility, wavelength));
                    radiance += throughput * backSkyDirect * spectralSky * spectralVisibility *
                                (kPi / gmax(dot(-normal, backSkyDirection), 1e-4f));
                }
            }
        }

        if (hasMeshLights) {
            // :1670-1731
            const uint32_t primitiveCount = scenePrimitiveCount(c);
            const uint32_t lightPrimitive = sampleEmissiveTriangle(c, randomFloat(rng), primitiveCount);
            if (lightPrimitive != primitive && s.emissive[lightPrimitive].y > 0.0f) {
                const float root = std::sqrt(randomFloat(rng));
                const float second = randomFloat(rng);
                const vec3 barycentric = V3(1.0f - root, root * (1.0f - second), root * second);
                const vec3 lightP0 = xyz(s.vertices[s.indices[lightPrimitive * 3u + 0u]]);
                const vec3 lightP1 = xyz(s.vertices[s.indices[lightPrimitive * 3u + 1u]]);
                const vec3 lightP2 = xyz(s.vertices[s.indices[lightPrimitive * 3u + 2u]]);
                const vec3 lightPosition = lightP0 * barycentric.x + lightP1 * barycentric.y + lightP2 * barycentric.z;
                const vec3 lightNormal = normalize(cross(lightP1 - lightP0, lightP2 - lightP0));
                const vec3 toLight = lightPosition - hitPoint;
                const float distanceSquared = dot(toLight, toLight);
                const float lightDistance = std::sqrt(gmax(distanceSquared, 1e-8f));
                const vec3 lightDirection = toLight / lightDistance;
                const float emissionCosine = std::fabs(dot(lightNormal, -lightDirection));
                const float lightPdf = emissiveTrianglePdf(c, lightPrimitive, distanceSquared, emissionCosine);
                if (lightPdf > 0.0f) {
                    const vec3 direct =
                        evaluateDirectSurface(normal, tangent, viewDirection, lightDirection, sp, 1.0f, 1.0f);
                    if (anyGreaterThanZero(direct) &&
                        meshLightVisible(c, offsetSurfaceOrigin(hitPoint, orientedGeometricNormal, lightDirection),
                                         lightDirection, gmax(lightDistance - 0.003f, 0.001f))) {
                        const vec2 lightBary = V2(barycentric.y, barycentric.z);
                        const vec2 lightUv = surfaceTextureCoordinates(s, lightPrimitive, lightBary);
                        vec3 lightEmissionRgb = surfaceEmissionRgb(c, lightPrimitive, lightUv);
                        lightEmissionRgb *= surfaceOpacity(s, lightPrimitive, lightBary);
                        const vec3 spectralLight = V3(illuminantSpectrum(lightEmissionRgb, wavelength));
                        const float bsdfPdf = surfaceReflectionPdf(normal, tangent, viewDirection, lightDirection,
                                                                   roughness, coatRoughness, sheenProbability,
                                                                   coatProbability, specularProbability,
                                                                   translucentProbability);
                        const float misWeight = powerHeuristic(lightPdf, bsdfPdf);
                        radiance += throughput * direct * spectralLight * (misWeight / lightPdf);
                    }
                }
            }
        }

        if (randomFloat(rng) < transmission) {
            // :1735-1777
            const float eta = frontFace ? 1.0f / ior : ior;
            const float cosTheta = gmin(dot(-rayDirection, normal), 1.0f);
            float r0 = (1.0f - ior) / (1.0f + ior);
            r0 *= r0;
            const float fresnel = r0 + (1.0f - r0) * gpow(1.0f - cosTheta, 5.0f);
            const vec3 refracted = refract(rayDirection, normal, eta);
            const bool totalInternalReflection = dot(refracted, refracted) < 1e-8f;
            const bool thinWalled = material.transmissionColorThinWalled.w > 0.5f;
            bool refractedThroughBoundary = false;
            if (totalInternalReflection || randomFloat(rng) < fresnel) {
                rayDirection = reflect(rayDirection, normal);
            } else {
                rayDirection = thinWalled ? rayDirection : normalize(refracted);
                refractedThroughBoundary = !thinWalled;
            }
            const float transmissionDepth = gmax(material.transmissionMedium.x, 0.0f);
            throughput *= transmissionDepth > 0.0f ? V3(1.0f) : transmissionColor;
            if (refractedThroughBoundary) {
                if (frontFace) {
                    const float spectralTransmission = gmax(transmissionColor.x, 0.001f);
                    mediumAbsorption = transmissionDepth > 0.0f ? -glog(spectralTransmission) / transmissionDepth : 0.0f;
                    const float spectralScatter =
                        gmax(reconstructRgb(xyz(material.transmissionScatter), wavelength), 0.0f);
                    mediumScattering = transmissionDepth > 0.0f ? spectralScatter / transmissionDepth : spectralScatter;
                    mediumAnisotropy = material.transmissionMedium.y;
                    insideMedium = true;
                } else {
                    insideMedium = false;
                    mediumAbsorption = 0.0f;
                    mediumScattering = 0.0f;
                }
            }
            rayOrigin = hitPoint + rayDirection * 0.002f;
            environmentOnMiss = true;
            previousWasDelta = true;
            previousBsdfPdf = 0.0f;
            continue;
        }

        // :1779-1858 BSDF sampling chain
        environmentOnMiss = false;
        rayOrigin = hitPoint + orientedGeometricNormal * 0.002f;
        if (sheenProbability > 0.0f && randomFloat(rng) < sheenProbability) {
            rayDirection = cosineHemisphere(normal, rng);
            const float sheenPdf = gmax(dot(normal, rayDirection), 0.0f) / kPi;
            const float response = sheenResponse(normal, viewDirection, rayDirection, sheenRoughness, sheenZeltner);
            throughput *= sheen * sheenColor * response / gmax(sheenProbability * sheenPdf, 1e-6f);
            environmentOnMiss = true;
        } else {
            throughput *= (1.0f - sheen * sheenAlbedo) / gmax(1.0f - sheenProbability, 1e-4f);
            if (coatProbability > 0.0f && randomFloat(rng) < coatProbability) {
                const vec3 incident = rayDirection;
                rayDirection = sampleGGXReflectionAnisotropic(rayDirection, normal, tangent, coatRoughness, rng);
                throughput *= coat * ggxSampleWeightAnisotropic(incident, rayDirection, normal, tangent, coatRoughness,
                                                                coatF0) /
                              coatProbability;
                environmentOnMiss = gmax(coatRoughness.x, coatRoughness.y) < 0.2f;
            } else {
                throughput *= (V3(1.0f) - coatContribution) / gmax(1.0f - coatProbability, 1e-4f);
                if (randomFloat(rng) < specularProbability) {
                    const vec3 incident = rayDirection;
                    rayDirection = sampleGGXReflectionAnisotropic(rayDirection, normal, tangent, roughness, rng);
                    throughput *= ggxSampleWeightAnisotropic(incident, rayDirection, normal, tangent, roughness, f0) /
                                  specularProbability;
                    environmentOnMiss = gmax(roughness.x, roughness.y) < 0.2f;
                } else {
                    if (translucentProbability > 0.0f && randomFloat(rng) < translucentProbability) {
                        throughput *= translucentContribution /
                                      gmax((1.0f - specularProbability) * translucentProbability, 1e-4f);
                        rayDirection = cosineHemisphere(-normal, rng);
                        rayOrigin = offsetSurfaceOrigin(hitPoint, orientedGeometricNormal, rayDirection);
                    } else {
                        throughput *= diffuseContribution /
                                      gmax((1.0f - specularProbability) * (1.0f - translucentProbability), 1e-4f);
                        if (subsurface > 0.0f && randomFloat(rng) < subsurface) {
                            const float radius =
                                gmax(reconstructRgb(subsurfaceRadiusRgb, wavelength) *
                                         gmax(material.subsurfaceWeightScale.y, 0.0f),
                                     0.001f);
                            const float albedo = reflectanceSpectrum(subsurfaceColorRgb, wavelength);
                            vec3 exitOrigin;
                            vec3 exitDirection;
                            float attenuation;
                            if (randomWalkSubsurface(c, hitPoint, orientedGeometricNormal, radius, albedo,
                                                     material.subsurfaceWeightScale.z, rng, exitOrigin, exitDirection,
                                                     attenuation)) {
                                throughput *= attenuation;
                                rayOrigin = exitOrigin;
                                rayDirection = exitDirection;
                                environmentOnMiss = true;
                                previousWasDelta = true;
                                previousBsdfPdf = 0.0f;
                                continue;
                            }
                        }
                        rayDirection = cosineHemisphere(normal, rng);
                        const float lambertResponse = gmax(dot(normal, rayDirection), 0.0f) / kPi;
                        throughput *= evaluateDiffuseReflection(normal, viewDirection, rayDirection, diffuseColor,
                                                                diffuseRoughness, diffuseModel) /
                                      gmax(lambertResponse, 1e-6f);
                    }
                }
            }
        }
        if (lightCount > 0u || hasMeshLights) {
            // :1859-1874
            previousBsdfPdf = surfaceReflectionPdf(normal, tangent, viewDirection, rayDirection, roughness,
                                                   coatRoughness, sheenProbability, coatProbability,
                                                   specularProbability, translucentProbability);
            previousWasDelta = false;
            environmentOnMiss = true;
            previousEnvironmentLightPdf =
                lightCount > 0u
                    ? environmentLightPdf(c, hitPoint, normal, rayDirection, diffuseEnergy,
                                          specularEnergy + luminance(coatContribution) + sheenProbability,
                                          translucentEnergy)
                    : 0.0f;
        }
        if (bounce >= 2) {
            // :1875-1879 Russian roulette
            const float survival = clampf(gmax(throughput.x, gmax(throughput.y, throughput.z)), 0.1f, 0.95f);
            if (randomFloat(rng) > survival) break;
            throughput /= survival;
        }
    }
    return radiance.x;
}

}  // namespace

float surfaceOpacity(const PackedScene& scene, uint32_t primitive, vec2 barycentrics)
{
    // :797-803
    Ctx c{};
    c.scene = &scene;
    const GpuMaterial& material = scene.materials[scene.triangleMaterials[primitive]];
    const vec2 uv = surfaceTextureCoordinates(scene, primitive, barycentrics);
    return clampf(sampleMaterialTexture(c, material.textureIndices1[0], uv, V4(material.transmissionOpacityIor.y)).x,
                  0.0f, 1.0f);
}

void RenderPixel(const PackedScene& scene, const Bvh& bvh, const Camera& camera, const FrameParams& frame,
                 uint32_t x, uint32_t y, float* rgba, double* xyzSum, Counters* counters)
{
    Ctx c{};
    c.scene = &scene;
    c.bvh = &bvh;
    c.counters = counters;
    const uint32_t sampleCount = std::max(frame.sampleCount, 1u);
    // CameraUniform packing (vulkan_path_tracer.cpp:3242-3254)
    c.origin = V4(camera.origin, static_cast<float>(sampleCount));
    c.lowerLeft = V4(camera.lowerLeft, static_cast<float>(scene.primitiveCount));
    c.horizontal = V4(camera.horizontal, 0.0f);
    c.vertical = V4(camera.vertical, frame.zUp ? 1.0f : 0.0f);
    c.frame[0] = frame.width;
    c.frame[1] = frame.height;
    c.frame[2] = frame.sampleIndex;
    c.frame[3] = std::clamp(frame.maxBounces, 1u, kMaxPathBounces) | (scene.opaque ? (1u << 8) : 0u) |
                 (std::min(scene.lightCount, kMaxLights) << 16u);

    // main(): vulkan_path_tracer.cpp:1189-1891
    const uint32_t index = y * c.frame[0] + x;
    vec3 batchRadiance = V3(0.0f);
    double batchXyz[3] = {0.0, 0.0, 0.0};
    for (uint32_t sampleOffset = 0; sampleOffset < sampleCount; ++sampleOffset) {
        const uint32_t sampleNumber = c.frame[2] + sampleOffset;
        vec3 spectralSampleRadiance = V3(0.0f);
        double sampleXyz[3] = {0.0, 0.0, 0.0};
        for (uint32_t lane = 0; lane < 3u; ++lane) {
            float wavelength = 0.0f;
            const float radiance = TraceLane(c, index, x, y, sampleNumber, lane, &wavelength);
            spectralSampleRadiance += spectralSensor(wavelength) * radiance;
            const vec3 sensor = sensorXyz(wavelength);
            sampleXyz[0] += static_cast<double>(sensor.x) * radiance;
            sampleXyz[1] += static_cast<double>(sensor.y) * radiance;
            sampleXyz[2] += static_cast<double>(sensor.z) * radiance;
        }
        batchRadiance += spectralSampleRadiance / 3.0f;
        for (int k = 0; k < 3; ++k) batchXyz[k] += sampleXyz[k] / 3.0;
    }
    const vec3 previous = V3(rgba[0], rgba[1], rgba[2]);
    const float previousWeight = uintToFloat(c.frame[2]);
    const float totalWeight = previousWeight + uintToFloat(sampleCount);
    const vec3 result = (previous * previousWeight + batchRadiance) / totalWeight;
    rgba[0] = result.x;
    rgba[1] = result.y;
    rgba[2] = result.z;
    rgba[3] = 1.0f;
    for (int k = 0; k < 3; ++k) xyzSum[k] += batchXyz[k];
}

}  // namespace oracle
