// shading.cuh - device restatement of the reference integrator's shading
// functions (src/gpu/vulkan_path_tracer.cpp:115-1186), one function per GLSL
// function with the GLSL names. Lane-replicated vec3 values are scalars here
// (see common.cuh); vectors that really vary per component (directions, RGB
// inputs before spectral conversion) stay float3.
#pragma once

#include "common.cuh"

namespace hdcx {

__constant__ float cSrgbToLinear[256];

// ---------------------------------------------------------------------------
// Per-lane spectral constants. reconstructRgb's Gaussian basis and the Planck
// factor of illuminantSpectrum depend only on the wavelength, so each path
// computes them once (the same binary32 values the GLSL recomputes per call).
// ---------------------------------------------------------------------------
struct Spectrum {
    float wavelength;
    float br, bg, bb;   // basis (vulkan_path_tracer.cpp:120-123)
    float denominator;  // max(dot(vec3(1), basis), 1e-5)
    float planck;       // illuminantSpectrum's Planck ratio (:137-142)
};

HDCX_D Spectrum makeSpectrum(float wavelength)
{
    Spectrum s;
    s.wavelength = wavelength;
    s.br = gexp(-0.5f * gpow2((wavelength - 620.0f) / 30.0f));
    s.bg = gexp(-0.5f * gpow2((wavelength - 535.0f) / 25.0f));
    s.bb = gexp(-0.5f * gpow2((wavelength - 450.0f) / 20.0f));
    s.denominator = gmax(s.br + s.bg + s.bb, 1e-5f);
    const float temperature = 6504.0f;
    const float c2 = 1.4387769e7f;
    const float referenceWavelength = 560.0f;
    s.planck = gpow5(referenceWavelength / wavelength) *
               (gexp(c2 / (referenceWavelength * temperature)) - 1.0f) /
               gmax(gexp(c2 / (wavelength * temperature)) - 1.0f, 1e-5f);
    return s;
}

HDCX_D Spectrum spectrumFromBasis(float wavelength, float4 packed)
{
    Spectrum s;
    s.wavelength = wavelength;
    s.br = packed.x;
    s.bg = packed.y;
    s.bb = packed.z;
    s.planck = packed.w;
    s.denominator = gmax(s.br + s.bg + s.bb, 1e-5f);
    return s;
}

HDCX_D float reconstructRgb(float3 rgb, const Spectrum& s)
{
    // :118-126
    const float num = gmax(rgb.x, 0.0f) * s.br + gmax(rgb.y, 0.0f) * s.bg + gmax(rgb.z, 0.0f) * s.bb;
    return num / s.denominator;
}
HDCX_D float reflectanceSpectrum(float3 rgb, const Spectrum& s)
{
    return clampf(reconstructRgb(rgb, s), 0.0f, 1.0f);
}
HDCX_D float illuminantSpectrum(float3 rgb, const Spectrum& s)
{
    return gmax(reconstructRgb(rgb, s) * s.planck, 0.0f);
}

HDCX_D float3 cieXyz(float wavelength)
{
    // :146-170 (Wyman, Sloan and Shirley 2013 multi-lobe fit)
    const float tx1 = (wavelength - 442.0f) * (wavelength < 442.0f ? 0.0624f : 0.0374f);
    const float tx2 = (wavelength - 599.8f) * (wavelength < 599.8f ? 0.0264f : 0.0323f);
    const float tx3 = (wavelength - 501.1f) * (wavelength < 501.1f ? 0.0490f : 0.0382f);
    const float ty1 = (wavelength - 568.8f) * (wavelength < 568.8f ? 0.0213f : 0.0247f);
    const float ty2 = (wavelength - 530.9f) * (wavelength < 530.9f ? 0.0613f : 0.0322f);
    const float tz1 = (wavelength - 437.0f) * (wavelength < 437.0f ? 0.0845f : 0.0278f);
    const float tz2 = (wavelength - 459.0f) * (wavelength < 459.0f ? 0.0385f : 0.0725f);
    return f3(0.362f * gexp(-0.5f * tx1 * tx1) + 1.056f * gexp(-0.5f * tx2 * tx2) -
                  0.065f * gexp(-0.5f * tx3 * tx3),
              0.821f * gexp(-0.5f * ty1 * ty1) + 0.286f * gexp(-0.5f * ty2 * ty2),
              1.217f * gexp(-0.5f * tz1 * tz1) + 0.681f * gexp(-0.5f * tz2 * tz2));
}
HDCX_D float3 sensorXyz(float wavelength) { return cieXyz(wavelength) * (400.0f / 106.856895f); }
HDCX_D float3 spectralSensor(float wavelength)
{
    // :172-179
    const float3 x = sensorXyz(wavelength);
    return f3(3.2404542f * x.x - 1.5371385f * x.y - 0.4985314f * x.z,
              -0.9692660f * x.x + 1.8760108f * x.y + 0.0415560f * x.z,
              0.0556434f * x.x - 0.2040259f * x.y + 1.0572252f * x.z);
}

// ---------------------------------------------------------------------------
// Textures: linear filter, REPEAT, one mip (the reference's sampler,
// vulkan_path_tracer.cpp:2401-2423); sRGB images decode before filtering.
// ---------------------------------------------------------------------------
HDCX_D float4 texelFetch(const TexDesc& t, int x, int y)
{
    const size_t i = static_cast<size_t>(y) * t.width + static_cast<size_t>(x);
    if (t.format == 2u) return __ldg(reinterpret_cast<const float4*>(t.texels) + i);
    const uint32_t p = __ldg(reinterpret_cast<const uint32_t*>(t.texels) + i);
    const uint32_t r = p & 0xffu, g = (p >> 8) & 0xffu, b = (p >> 16) & 0xffu, a = p >> 24;
    if (t.format == 1u) {
        return make_float4(cSrgbToLinear[r], cSrgbToLinear[g], cSrgbToLinear[b], u2f(a) / 255.0f);
    }
    return make_float4(u2f(r) / 255.0f, u2f(g) / 255.0f, u2f(b) / 255.0f, u2f(a) / 255.0f);
}

HDCX_D int wrapIndex(int i, int n)
{
    const int r = i % n;
    return r < 0 ? r + n : r;
}

HDCX_D float texelCoordinate(float uv, uint32_t size)
{
    const float x = uv * u2f(size) - 0.5f;
    return fabsf(x) < 16777216.0f ? x : 0.0f;
}

HDCX_D float4 sampleBilinear(const TexDesc& t, float2 uv)
{
    const float x = texelCoordinate(uv.x, t.width);
    const float y = texelCoordinate(uv.y, t.height);
    const float fx = floorf(x), fy = floorf(y);
    const float a = x - fx, b = y - fy;
    const int w = static_cast<int>(t.width), h = static_cast<int>(t.height);
    const int i0 = wrapIndex(static_cast<int>(fx), w);
    const int j0 = wrapIndex(static_cast<int>(fy), h);
    const int i1 = wrapIndex(i0 + 1, w);
    const int j1 = wrapIndex(j0 + 1, h);
    const float4 t00 = texelFetch(t, i0, j0), t10 = texelFetch(t, i1, j0);
    const float4 t01 = texelFetch(t, i0, j1), t11 = texelFetch(t, i1, j1);
    const float w00 = (1.0f - a) * (1.0f - b), w10 = a * (1.0f - b);
    const float w01 = (1.0f - a) * b, w11 = a * b;
    return make_float4(w00 * t00.x + w10 * t10.x + w01 * t01.x + w11 * t11.x,
                       w00 * t00.y + w10 * t10.y + w01 * t01.y + w11 * t11.y,
                       w00 * t00.z + w10 * t10.z + w01 * t01.z + w11 * t11.z,
                       w00 * t00.w + w10 * t10.w + w01 * t01.w + w11 * t11.w);
}

HDCX_D float4 textureSample(const DeviceScene& s, uint32_t index, float2 uv)
{
    if (index >= s.textureCount) return make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    const TexDesc t = s.textures[index];
    return sampleBilinear(t, uv);
}

// Texture LOD (not in the reference, whose sampler has one mip level): the
// bilinear filter on mip level `level` >= 1 of the pyramid (REPEAT).
HDCX_D float4 sampleMipBilinear(const TexDesc& t, uint32_t level, float2 uv)
{
    const float4* m = t.mips;
    uint32_t w = t.width, h = t.height;
    for (uint32_t k = 1; k <= level; ++k) {
        const uint32_t nw = max(1u, w >> 1), nh = max(1u, h >> 1);
        if (k < level) m += size_t(nw) * nh;
        w = nw;
        h = nh;
    }
    const float x = texelCoordinate(uv.x, w), y = texelCoordinate(uv.y, h);
    const float fx = floorf(x), fy = floorf(y);
    const float a = x - fx, b = y - fy;
    const int i0 = wrapIndex(static_cast<int>(fx), static_cast<int>(w)), j0 = wrapIndex(static_cast<int>(fy), static_cast<int>(h));
    const int i1 = wrapIndex(i0 + 1, static_cast<int>(w)), j1 = wrapIndex(j0 + 1, static_cast<int>(h));
    const float4 t00 = __ldg(m + size_t(j0) * w + i0), t10 = __ldg(m + size_t(j0) * w + i1);
    const float4 t01 = __ldg(m + size_t(j1) * w + i0), t11 = __ldg(m + size_t(j1) * w + i1);
    const float w00 = (1.0f - a) * (1.0f - b), w10 = a * (1.0f - b), w01 = (1.0f - a) * b, w11 = a * b;
    return make_float4(w00 * t00.x + w10 * t10.x + w01 * t01.x + w11 * t11.x,
                       w00 * t00.y + w10 * t10.y + w01 * t01.y + w11 * t11.y,
                       w00 * t00.z + w10 * t10.z + w01 * t01.z + w11 * t11.z,
                       w00 * t00.w + w10 * t10.w + w01 * t01.w + w11 * t11.w);
}

// A lookup at level of detail lodBase + log2(sqrt(width * height)) (ray
// cones: lodBase holds the hit's texture-independent terms), trilinear
// between the two nearest levels; lodBase = -inf samples level 0 exactly as
// textureSample does.
HDCX_D float4 textureSampleLod(const DeviceScene& s, uint32_t index, float2 uv, float lodBase)
{
    if (index >= s.textureCount) return make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    const TexDesc t = s.textures[index];
    if (!(lodBase > -1e30f) || t.levels <= 1u || t.mips == nullptr) return sampleBilinear(t, uv);
    const float lod = fminf(fmaxf(lodBase + 0.5f * log2f(u2f(t.width) * u2f(t.height)), 0.0f), u2f(t.levels - 1u));
    const uint32_t l0 = static_cast<uint32_t>(lod);
    const float f = lod - u2f(l0);
    const float4 a = l0 == 0u ? sampleBilinear(t, uv) : sampleMipBilinear(t, l0, uv);
    if (f <= 0.0f || l0 + 1u >= t.levels) return a;
    const float4 b = sampleMipBilinear(t, l0 + 1u, uv);
    return make_float4(a.x + (b.x - a.x) * f, a.y + (b.y - a.y) * f, a.z + (b.z - a.z) * f, a.w + (b.w - a.w) * f);
}

HDCX_D float4 sampleMaterialTexture(const DeviceScene& s, uint32_t textureIndex, float2 uv, float4 fallbackValue,
                                    float lodBase = -INFINITY)
{
    // :760-775
    if (textureIndex == kMissingTexture) return fallbackValue;
    if ((textureIndex & 0x80000000u) != 0u) {
        const float fu = floorf(uv.x), fv = floorf(uv.y);
        if (!(fabsf(fu) < 1e6f) || !(fabsf(fv) < 1e6f)) return fallbackValue;
        const int tileOffset = static_cast<int>(fu) + static_cast<int>(fv) * 10;
        if (tileOffset < 0 || tileOffset >= 23) return fallbackValue;
        const uint32_t presentTiles = (textureIndex >> 8u) & 0x7fffffu;
        const uint32_t tileBit = 1u << static_cast<uint32_t>(tileOffset);
        if ((presentTiles & tileBit) == 0u) return fallbackValue;
        const uint32_t descriptorIndex = (textureIndex & 0xffu) + static_cast<uint32_t>(__popc(presentTiles & (tileBit - 1u)));
        if (descriptorIndex >= s.textureCount) return fallbackValue;
        return textureSampleLod(s, descriptorIndex, make_float2(fract(uv.x), fract(uv.y)), lodBase);
    }
    if (textureIndex >= s.textureCount) return fallbackValue;
    return textureSampleLod(s, textureIndex, uv, lodBase);
}

HDCX_D float4 f4(float v) { return make_float4(v, v, v, v); }
HDCX_D float4 f4(float3 v, float w) { return make_float4(v.x, v.y, v.z, w); }

HDCX_D float2 surfaceTextureCoordinates(const DeviceScene& s, uint32_t primitive, float b1, float b2)
{
    // :787-795
    const float b0 = 1.0f - b1 - b2;
    const float2 uv0 = __ldg(s.texcoords + primitive * 3u + 0u);
    const float2 uv1 = __ldg(s.texcoords + primitive * 3u + 1u);
    const float2 uv2 = __ldg(s.texcoords + primitive * 3u + 2u);
    return make_float2(uv0.x * b0 + uv1.x * b1 + uv2.x * b2, uv0.y * b0 + uv1.y * b1 + uv2.y * b2);
}

HDCX_D float surfaceOpacity(const DeviceScene& s, uint32_t primitive, float b1, float b2)
{
    // :797-803. Without an opacity texture the value is the material's
    // opacity, so the texture coordinates are not needed.
    const GpuMaterial* m = s.materials + __ldg(s.triangleMaterials + primitive);
    const uint32_t texture = m->textureIndices1.x;
    if (texture == kMissingTexture) return clampf(m->transmissionOpacityIor.y, 0.0f, 1.0f);
    const float2 uv = surfaceTextureCoordinates(s, primitive, b1, b2);
    return clampf(sampleMaterialTexture(s, texture, uv, f4(m->transmissionOpacityIor.y)).x, 0.0f, 1.0f);
}

HDCX_D float3 surfaceEmissionRgb(const DeviceScene& s, uint32_t primitive, float2 uv)
{
    // :777-785
    const GpuMaterial* m = s.materials + __ldg(s.triangleMaterials + primitive);
    const float weight = gmax(m->transmissionOpacityIor.w, 0.0f);
    if (m->textureIndices0.w == kMissingTexture) return xyz(m->emissionRoughness) * weight;
    const float4 t = sampleMaterialTexture(s, m->textureIndices0.w, uv, f4(0.0f));
    return f3(t.x, t.y, t.z) * weight;
}

// ---------------------------------------------------------------------------
// Sampling and BSDFs (vulkan_path_tracer.cpp:183-471, :933-1069)
// ---------------------------------------------------------------------------
HDCX_D float3 tangentFrameAxis(float3 normal)
{
    return normalize(fabsf(normal.z) < 0.999f ? cross(normal, f3(0.0f, 0.0f, 1.0f)) : cross(normal, f3(0.0f, 1.0f, 0.0f)));
}

HDCX_D float3 cosineHemisphere(float3 normal, uint32_t& state)
{
    // :183-195
    const float r1 = kTwoPi * randomFloat(state);
    const float r2 = randomFloat(state);
    const float r2s = sqrtf(r2);
    const float3 tangent = tangentFrameAxis(normal);
    const float3 bitangent = cross(normal, tangent);
    return normalize(tangent * gcos(r1) * r2s + bitangent * gsin(r1) * r2s + normal * sqrtf(1.0f - r2));
}

HDCX_D float fresnelSchlick(float cosTheta, float f0)
{
    // :202-205
    return f0 + (1.0f - f0) * gpow5(1.0f - clampf(cosTheta, 0.0f, 1.0f));
}

HDCX_D float3 orthogonalTangent(float3 normal, float3 tangent)
{
    // :276-285
    float3 result = tangent - normal * dot(normal, tangent);
    if (dot(result, result) < 1e-8f) {
        result = fabsf(normal.z) < 0.999f ? cross(normal, f3(0.0f, 0.0f, 1.0f)) : cross(normal, f3(0.0f, 1.0f, 0.0f));
    }
    return normalize(result);
}

HDCX_D float2 clampRoughness(float2 roughness)
{
    return make_float2(clampf(roughness.x * roughness.x, 0.001f, 1.0f), clampf(roughness.y * roughness.y, 0.001f, 1.0f));
}

HDCX_D float distributionGGXAnisotropic(float3 halfway, float3 normal, float3 tangent, float2 roughness)
{
    // :287-300
    const float3 axisX = orthogonalTangent(normal, tangent);
    const float3 axisY = cross(normal, axisX);
    const float2 alpha = clampRoughness(roughness);
    const float lx = dot(halfway, axisX), ly = dot(halfway, axisY), lz = gmax(dot(halfway, normal), 0.0f);
    const float denominator = lx * lx / (alpha.x * alpha.x) + ly * ly / (alpha.y * alpha.y) + lz * lz;
    return 1.0f / gmax(kPi * alpha.x * alpha.y * denominator * denominator, 1e-6f);
}

HDCX_D float geometryGGXAnisotropic(float3 direction, float3 normal, float3 tangent, float2 roughness)
{
    // :302-315
    const float nDotDirection = gmax(dot(normal, direction), 0.0f);
    if (nDotDirection <= 0.0f) return 0.0f;
    const float3 axisX = orthogonalTangent(normal, tangent);
    const float3 axisY = cross(normal, axisX);
    const float2 alpha = clampRoughness(roughness);
    const float projected = gpow2(alpha.x * dot(direction, axisX)) + gpow2(alpha.y * dot(direction, axisY));
    const float lambda = (-1.0f + sqrtf(1.0f + projected / gmax(nDotDirection * nDotDirection, 1e-8f))) * 0.5f;
    return 1.0f / (1.0f + lambda);
}

HDCX_D float evaluateGGXAnisotropic(float3 normal, float3 tangent, float3 viewDirection, float3 lightDirection,
                                    float2 roughness, float f0)
{
    // :317-332
    const float3 halfway = normalize(viewDirection + lightDirection);
    const float nDotV = gmax(dot(normal, viewDirection), 0.0f);
    const float nDotL = gmax(dot(normal, lightDirection), 0.0f);
    const float vDotH = gmax(dot(viewDirection, halfway), 0.0f);
    if (nDotV <= 0.0f || nDotL <= 0.0f || vDotH <= 0.0f) return 0.0f;
    const float distribution = distributionGGXAnisotropic(halfway, normal, tangent, roughness);
    const float geometry = geometryGGXAnisotropic(viewDirection, normal, tangent, roughness) *
                           geometryGGXAnisotropic(lightDirection, normal, tangent, roughness);
    return distribution * geometry * fresnelSchlick(vDotH, f0) / gmax(4.0f * nDotV * nDotL, 1e-5f);
}

HDCX_D float3 sampleGGXReflectionAnisotropic(float3 incident, float3 normal, float3 tangent, float2 roughness,
                                             uint32_t& state)
{
    // :334-350
    const float3 axisX = orthogonalTangent(normal, tangent);
    const float3 axisY = cross(normal, axisX);
    const float2 alpha = clampRoughness(roughness);
    const float phi = kTwoPi * randomFloat(state);
    const float elevationSample = randomFloat(state);
    const float radius = sqrtf(elevationSample / gmax(1.0f - elevationSample, 1e-6f));
    float3 halfway = normalize(axisX * (alpha.x * radius * gcos(phi)) + axisY * (alpha.y * radius * gsin(phi)) + normal);
    if (dot(halfway, -incident) < 0.0f) halfway = -halfway;
    const float3 reflected = reflect(incident, halfway);
    return dot(reflected, normal) > 0.0f ? normalize(reflected) : normalize(reflect(incident, normal));
}

HDCX_D float ggxSampleWeightAnisotropic(float3 incident, float3 outgoing, float3 normal, float3 tangent,
                                        float2 roughness, float f0)
{
    // :352-367
    const float3 viewDirection = normalize(-incident);
    const float3 halfway = normalize(viewDirection + outgoing);
    const float nDotL = gmax(dot(normal, outgoing), 0.0f);
    const float nDotH = gmax(dot(normal, halfway), 0.0f);
    const float vDotH = gmax(dot(viewDirection, halfway), 0.0f);
    if (nDotL <= 0.0f || nDotH <= 0.0f || vDotH <= 0.0f) return 0.0f;
    const float distribution = distributionGGXAnisotropic(halfway, normal, tangent, roughness);
    const float pdf = distribution * nDotH / gmax(4.0f * vDotH, 1e-6f);
    return evaluateGGXAnisotropic(normal, tangent, viewDirection, outgoing, roughness, f0) * nDotL / gmax(pdf, 1e-6f);
}

HDCX_D float ggxReflectionPdfAnisotropic(float3 normal, float3 tangent, float3 viewDirection, float3 lightDirection,
                                         float2 roughness)
{
    // :371-383
    if (dot(normal, viewDirection) <= 0.0f || dot(normal, lightDirection) <= 0.0f) return 0.0f;
    const float3 halfway = normalize(viewDirection + lightDirection);
    const float nDotH = gmax(dot(normal, halfway), 0.0f);
    const float vDotH = gmax(dot(viewDirection, halfway), 0.0f);
    return distributionGGXAnisotropic(halfway, normal, tangent, roughness) * nDotH / gmax(4.0f * vDotH, 1e-6f);
}

HDCX_D float powerHeuristic(float firstPdf, float secondPdf)
{
    // :385-390
    const float firstSquared = firstPdf * firstPdf;
    const float secondSquared = secondPdf * secondPdf;
    return firstSquared / gmax(firstSquared + secondSquared, 1e-12f);
}

HDCX_D float sheenDirectionalAlbedo(float nDotV, float roughness)
{
    // :419-429
    const float x = clampf(nDotV, 0.0f, 1.0f);
    const float y = clampf(roughness, 0.01f, 1.0f);
    const float fx = 13.67300f + -68.78018f * x + 799.08825f * y + -905.00061f * x * y + 60.28956f * x * x +
                     1086.96473f * y * y;
    const float fy = 1.0f + 61.57746f * x + 442.78211f * y + 2597.49308f * x * y + 121.81241f * x * x +
                     3045.55075f * y * y;
    return clampf(fx / gmax(fy, 1e-6f), 0.0f, 1.0f);
}

HDCX_D float sheenImageworksResponse(float3 normal, float3 viewDirection, float3 lightDirection, float roughness)
{
    // :431-446
    const float nDotL = gmax(dot(normal, lightDirection), 0.0f);
    const float nDotV = gmax(dot(normal, viewDirection), 0.0f);
    if (nDotL <= 0.0f || nDotV <= 0.0f) return 0.0f;
    const float3 halfway = normalize(viewDirection + lightDirection);
    const float nDotH = gmax(dot(normal, halfway), 0.0f);
    const float inverseRoughness = 1.0f / gmax(roughness, 0.005f);
    const float distribution =
        (2.0f + inverseRoughness) * gpow(gmax(1.0f - nDotH * nDotH, 0.0f), inverseRoughness * 0.5f) / (2.0f * kPi);
    const float brdf = distribution / gmax(4.0f * (nDotL + nDotV - nDotL * nDotV), 1e-6f);
    return brdf * nDotL;
}

HDCX_D float sheenZeltnerDirectionalAlbedo(float nDotV, float roughness)
{
    // :448-460
    const float x = clampf(nDotV, 0.0f, 1.0f);
    const float y = clampf(roughness, 0.01f, 1.0f);
    const float s = y * (0.0206607f + 1.58491f * y) / (0.0379424f + y * (1.32227f + y));
    const float m = y * (-0.193854f + y * (-1.14885f + y * (1.7932f - 0.95943f * y * y))) / (0.046391f + y);
    const float o = y * (0.000654023f + (-0.0207818f + 0.119681f * y) * y) / (1.26264f + y * (-1.92021f + y));
    return clampf(gexp(-0.5f * gpow2((x - m) / gmax(s, 1e-6f))) / (gmax(s, 1e-6f) * sqrtf(2.0f * kPi)) + o,
                  0.0f, 1.0f);
}

HDCX_D float sheenResponse(float3 normal, float3 viewDirection, float3 lightDirection, float roughness, bool zeltner)
{
    // :462-471
    if (!zeltner) return sheenImageworksResponse(normal, viewDirection, lightDirection, roughness);
    const float nDotL = gmax(dot(normal, lightDirection), 0.0f);
    const float nDotV = gmax(dot(normal, viewDirection), 0.0f);
    return sheenZeltnerDirectionalAlbedo(nDotV, roughness) * nDotL / kPi;
}

HDCX_D float eonDirectionalAlbedo(float nDotDirection, float roughness)
{
    // :933-944
    const float c1 = 0.2877934092f;
    const float cosine = clampf(nDotDirection, 0.0f, 1.0f);
    const float sine = sqrtf(gmax(1.0f - cosine * cosine, 0.0f));
    const float theta = gacos(cosine);
    const float sineCubed = sine * sine * sine;
    const float g = sine * (theta - sine * cosine) + (2.0f / 3.0f) * (sine * (1.0f - sineCubed) / gmax(cosine, 1e-5f) - sine);
    const float a = 1.0f / (1.0f + c1 * roughness);
    return clampf(a + roughness * a * g / kPi, 0.0f, 1.0f);
}

HDCX_D float evaluateDiffuseReflection(float3 normal, float3 viewDirection, float3 lightDirection, float diffuseColor,
                                       float roughness, uint32_t model)
{
    // :946-1009
    const float nDotL = gmax(dot(normal, lightDirection), 0.0f);
    const float nDotV = gmax(dot(normal, viewDirection), 0.0f);
    if (nDotL <= 0.0f || nDotV <= 0.0f) return 0.0f;
    if (model == 1u) {
        const float sigma = clampf(roughness, 0.0f, 1.0f);
        const float sigmaSquared = sigma * sigma;
        const float a = 1.0f - 0.5f * sigmaSquared / (sigmaSquared + 0.33f);
        const float b = 0.45f * sigmaSquared / (sigmaSquared + 0.09f);
        const float3 projectedLight = lightDirection - normal * nDotL;
        const float3 projectedView = viewDirection - normal * nDotV;
        float azimuth = 0.0f;
        if (dot(projectedLight, projectedLight) > 1e-8f && dot(projectedView, projectedView) > 1e-8f) {
            azimuth = gmax(dot(normalize(projectedLight), normalize(projectedView)), 0.0f);
        }
        const float sinLight = sqrtf(gmax(1.0f - nDotL * nDotL, 0.0f));
        const float sinView = sqrtf(gmax(1.0f - nDotV * nDotV, 0.0f));
        const float sinAlpha = gmax(sinLight, sinView);
        const float tanBeta = gmin(sinLight / gmax(nDotL, 1e-5f), sinView / gmax(nDotV, 1e-5f));
        return nDotL * (a + b * azimuth * sinAlpha * tanBeta) / kPi;
    }
    if (model == 2u) {
        const float3 halfway = normalize(viewDirection + lightDirection);
        const float lDotH = gmax(dot(lightDirection, halfway), 0.0f);
        const float grazing = 0.5f + 2.0f * clampf(roughness, 0.0f, 1.0f) * lDotH * lDotH;
        const float lightScatter = 1.0f + (grazing - 1.0f) * gpow5(1.0f - nDotL);
        const float viewScatter = 1.0f + (grazing - 1.0f) * gpow5(1.0f - nDotV);
        return nDotL * lightScatter * viewScatter / kPi;
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
        const float directionalFactor = (1.0f - outgoingAlbedo) * (1.0f - incidentAlbedo) / gmax(1.0f - averageAlbedo, 1e-5f);
        const float rho = clampf(diffuseColor, 0.0f, 0.9999f);
        const float multipleScatterOverRho = rho * averageAlbedo / gmax(1.0f - rho * (1.0f - averageAlbedo), 1e-5f);
        return nDotL / kPi * (singleScatter + multipleScatterOverRho * directionalFactor);
    }
    return nDotL / kPi;
}

// Material parameters of one shading point, per lane (the locals of main()).
struct SurfaceParams {
    float diffuseColor;
    float transmission, subsurface, diffuseWeight, diffuseRoughness;
    uint32_t diffuseModel;
    float translucentWeight;
    float translucentColor;
    float metalness;
    float2 roughness;
    float f0;
    float coat;
    float2 coatRoughness;
    float coatF0;
    float sheen;
    float sheenColor;
    float sheenRoughness;
    bool sheenZeltner;
};

HDCX_D float diffuseLayerSum(float diffuse, float translucent, float specular) { return diffuse + translucent + specular; }

HDCX_D float evaluateDirectSurface(float3 normal, float3 tangent, float3 viewDirection, float3 lightDirection,
                                   const SurfaceParams& p, float diffuseScale, float specularScale)
{
    // :1013-1069
    const float signedNdotL = dot(normal, lightDirection);
    const float nDotL = gmax(signedNdotL, 0.0f);
    const float backNdotL = gmax(-signedNdotL, 0.0f);
    const float wrappedNdotL = gmax((signedNdotL + 0.5f * p.subsurface) / (1.0f + 0.5f * p.subsurface), 0.0f);
    if (wrappedNdotL <= 0.0f && nDotL <= 0.0f && backNdotL * p.translucentWeight <= 0.0f) return 0.0f;
    const float3 halfway = nDotL > 0.0f ? normalize(viewDirection + lightDirection) : normal;
    const float baseFresnel = fresnelSchlick(gmax(dot(viewDirection, halfway), 0.0f), p.f0);
    const float diffuseResponse = mix(evaluateDiffuseReflection(normal, viewDirection, lightDirection, p.diffuseColor,
                                                                p.diffuseRoughness, p.diffuseModel),
                                      wrappedNdotL / kPi, p.subsurface);
    const float diffuse = diffuseScale * (1.0f - baseFresnel) * p.diffuseWeight * (1.0f - p.translucentWeight) *
                          (1.0f - p.metalness) * p.diffuseColor * diffuseResponse * (1.0f - p.transmission);
    const float viewFresnel = fresnelSchlick(gmax(dot(normal, viewDirection), 0.0f), p.f0);
    const float translucent = diffuseScale * (1.0f - viewFresnel) * p.translucentWeight * (1.0f - p.metalness) *
                              p.translucentColor * (backNdotL / kPi) * (1.0f - p.transmission);
    const float specular =
        specularScale * nDotL * evaluateGGXAnisotropic(normal, tangent, viewDirection, lightDirection, p.roughness, p.f0);
    float coatFresnel = 0.0f;
    float coatSpecular = 0.0f;
    if (p.coat > 0.0f) {
        coatFresnel = fresnelSchlick(gmax(dot(viewDirection, halfway), 0.0f), p.coatF0);
        coatSpecular = specularScale * p.coat * nDotL *
                       evaluateGGXAnisotropic(normal, tangent, viewDirection, lightDirection, p.coatRoughness, p.coatF0);
    }
    const float baseLayer = (1.0f - p.coat * coatFresnel) * (diffuseLayerSum(diffuse, translucent, specular)) + coatSpecular;
    // With sheen == 0 the sheen terms are exact zeros (the albedo and the
    // response are finite), leaving baseLayer * 1 + 0.
    if (p.sheen == 0.0f) return baseLayer;
    const float sheenAlbedo = p.sheenZeltner ? sheenZeltnerDirectionalAlbedo(gmax(dot(normal, viewDirection), 0.0f), p.sheenRoughness)
                                             : sheenDirectionalAlbedo(gmax(dot(normal, viewDirection), 0.0f), p.sheenRoughness);
    const float sheenLayer = specularScale * p.sheen * p.sheenColor *
                             sheenResponse(normal, viewDirection, lightDirection, p.sheenRoughness, p.sheenZeltner);
    return baseLayer * (1.0f - clampf(p.sheen * sheenAlbedo, 0.0f, 1.0f)) + sheenLayer;
}

// Not inlined: called from several sites of the shade kernel, one shared
// copy keeps the kernel's instruction footprint smaller (measured faster).
HDCX_NOINLINE float surfaceReflectionPdf(float3 normal, float3 tangent, float3 viewDirection, float3 lightDirection,
                                  float2 roughness, float2 coatRoughness, float sheenProbability, float coatProbability,
                                  float specularProbability, float translucentProbability)
{
    // :392-415
    const float reflectionCosinePdf = gmax(dot(normal, lightDirection), 0.0f) / kPi;
    const float transmissionCosinePdf = gmax(-dot(normal, lightDirection), 0.0f) / kPi;
    const float coatPdf = ggxReflectionPdfAnisotropic(normal, tangent, viewDirection, lightDirection, coatRoughness);
    const float specularPdf = ggxReflectionPdfAnisotropic(normal, tangent, viewDirection, lightDirection, roughness);
    const float diffusePdf = mix(reflectionCosinePdf, transmissionCosinePdf, translucentProbability);
    const float basePdf = coatProbability * coatPdf +
                          (1.0f - coatProbability) * (specularProbability * specularPdf + (1.0f - specularProbability) * diffusePdf);
    return sheenProbability * reflectionCosinePdf + (1.0f - sheenProbability) * basePdf;
}

HDCX_D float3 offsetSurfaceOrigin(float3 position, float3 geometricNormal, float3 direction)
{
    // :1071-1075
    const float side = dot(geometricNormal, direction) >= 0.0f ? 1.0f : -1.0f;
    return position + geometricNormal * (0.002f * side);
}

HDCX_D float3 uniformSphere(uint32_t& state)
{
    // :1077-1083
    const float y = 1.0f - 2.0f * randomFloat(state);
    const float radius = sqrtf(gmax(1.0f - y * y, 0.0f));
    const float phi = kTwoPi * randomFloat(state);
    return f3(radius * gcos(phi), y, radius * gsin(phi));
}

HDCX_D float shapingConeFactor(const GpuLight& light, float cosine)
{
    // :1085-1094
    const float angle = gacos(clampf(cosine, -1.0f, 1.0f));
    const float outer = radians(clampf(light.shaping.y, 0.0f, 180.0f));
    const float inner = outer * (1.0f - clampf(light.shaping.z, 0.0f, 1.0f));
    return outer >= 3.1415925f ? 1.0f
                               : (outer <= inner + 1e-6f ? (angle <= outer ? 1.0f : 0.0f) : 1.0f - smoothstep(inner, outer, angle));
}

HDCX_D float dispersedIor(float iorAtD, float scale, float abbeNumber, float wavelength)
{
    // :1096-1110 (Cauchy fit through the Abbe number)
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

HDCX_D float3 sampleHenyeyGreenstein(float3 forward, float anisotropy, uint32_t& state)
{
    // :1112-1128
    const float g = clampf(anisotropy, -0.95f, 0.95f);
    const float u = randomFloat(state);
    const float cosine = fabsf(g) < 1e-3f ? 1.0f - 2.0f * u
                                          : (1.0f + g * g - gpow2((1.0f - g * g) / (1.0f - g + 2.0f * g * u))) / (2.0f * g);
    const float sine = sqrtf(gmax(1.0f - cosine * cosine, 0.0f));
    const float phi = kTwoPi * randomFloat(state);
    const float3 w = normalize(forward);
    const float3 tangent = tangentFrameAxis(w);
    const float3 bitangent = cross(w, tangent);
    return normalize(tangent * (gcos(phi) * sine) + bitangent * (gsin(phi) * sine) + w * cosine);
}

// ---------------------------------------------------------------------------
// Dome, environment and light selection (vulkan_path_tracer.cpp:473-758)
// ---------------------------------------------------------------------------
HDCX_D float2 directionToVerticalCross(float3 d)
{
    const float ax = fabsf(d.x), ay = fabsf(d.y), az = fabsf(d.z);
    float2 faceUv;
    float2 tile;
    if (ax >= ay && ax >= az) {
        if (d.x >= 0.0f) { faceUv = make_float2(-d.z / ax, d.y / ax); tile = make_float2(2.0f, 1.0f); }
        else { faceUv = make_float2(d.z / ax, d.y / ax); tile = make_float2(0.0f, 1.0f); }
    } else if (ay >= az) {
        if (d.y >= 0.0f) { faceUv = make_float2(d.x / ay, -d.z / ay); tile = make_float2(1.0f, 0.0f); }
        else { faceUv = make_float2(d.x / ay, d.z / ay); tile = make_float2(1.0f, 2.0f); }
    } else if (d.z >= 0.0f) {
        faceUv = make_float2(d.x / az, d.y / az);
        tile = make_float2(1.0f, 1.0f);
    } else {
        faceUv = make_float2(-d.x / az, d.y / az);
        tile = make_float2(1.0f, 3.0f);
    }
    const float qx = tile.x + faceUv.x * 0.5f, qy = tile.y + faceUv.y * 0.5f;
    return make_float2((qx + 0.5f) / 3.0f, (qy + 0.5f) / 4.0f);
}

HDCX_D float2 domeTextureCoordinates(float3 direction, uint32_t format)
{
    // :505-525
    if (format == 2u) {
        const float denominator = 2.0f * sqrtf(gmax(direction.x * direction.x + direction.y * direction.y +
                                                         (direction.z + 1.0f) * (direction.z + 1.0f),
                                                     1e-8f));
        return make_float2(direction.x / denominator + 0.5f, direction.y / denominator + 0.5f);
    }
    if (format == 3u) {
        const float radius = gacos(clampf(-direction.z, -1.0f, 1.0f)) / kPi;
        const float2 dxy = make_float2(direction.x, direction.y);
        const float2 radial = length2(dxy) > 1e-6f ? normalize2(dxy) : make_float2(0.0f, 0.0f);
        const float r = 0.5f * radius;
        return make_float2(0.5f + radial.x * r, 0.5f + radial.y * r);
    }
    if (format == 4u) return directionToVerticalCross(direction);
    return make_float2(fract(gatan2(direction.x, -direction.z) / (2.0f * kPi) + 1.0f),
                       1.0f - gacos(clampf(direction.y, -1.0f, 1.0f)) / kPi);
}

HDCX_D float3 domeLocalDirection(const GpuLight& light, float3 worldDirection)
{
    return normalize(f3(dot(worldDirection, xyz(light.basisX)), dot(worldDirection, xyz(light.basisY)),
                        dot(worldDirection, xyz(light.basisZ))));
}

HDCX_D float3 sampleDome(const DeviceScene& s, const GpuLight& light, float3 worldDirection)
{
    // :527-537
    const float3 localDirection = domeLocalDirection(light, worldDirection);
    float3 textureValue = f3(1.0f);
    if (light.textureInfo.x != kMissingTexture) {
        const float4 t = textureSample(s, light.textureInfo.x, domeTextureCoordinates(localDirection, light.textureInfo.y));
        textureValue = f3(t.x, t.y, t.z);
    }
    return xyz(light.colorIntensity) * light.colorIntensity.w * textureValue;
}

HDCX_D float3 environment(const DeviceScene& s, const FrameConst& f, float3 direction)
{
    // :551-569
    float3 result = f3(0.0f);
    const uint32_t lightCount = s.lightCount;
    if (lightCount == 0u) {
        if (s.hasMeshLights) return f3(0.0f);
        const float3 up = f.zUp ? f3(0.0f, 0.0f, 1.0f) : f3(0.0f, 1.0f, 0.0f);
        const float t = 0.5f * (dot(direction, up) + 1.0f);
        return mix(f3(0.035f, 0.045f, 0.065f), f3(0.38f, 0.55f, 0.85f), t);
    }
    for (uint32_t index = 0; index < lightCount; ++index) {
        const GpuLight& light = s.lights[index];
        if (light.textureInfo.z == 0u) result = result + sampleDome(s, light, direction);
    }
    return result;
}

HDCX_D float3 latLongDirection(float u, float v)
{
    // :571-579
    const float theta = kPi * (1.0f - v);
    const float phi = 2.0f * kPi * u;
    const float sineTheta = gsin(theta);
    return f3(sineTheta * gsin(phi), gcos(theta), -sineTheta * gcos(phi));
}

HDCX_D const TexDesc* importanceTexture(const DeviceScene& s, uint32_t index)
{
    return (index == kMissingTexture || index >= s.textureCount) ? nullptr : s.textures + index;
}

HDCX_D float domeLightPdf(const DeviceScene& s, const GpuLight& light, float3 worldDirection)
{
    // :583-598
    const TexDesc* tp = importanceTexture(s, light.textureInfo.w);
    if (!tp) return 1.0f / 12.5663706144f;
    const TexDesc t = *tp;
    const float3 localDirection = domeLocalDirection(light, worldDirection);
    const float2 uv = domeTextureCoordinates(localDirection, light.textureInfo.y);
    const int w = static_cast<int>(t.width), h = static_cast<int>(t.height);
    const float fx = uv.x * u2f(t.width), fy = uv.y * u2f(t.height);
    int tx = fabsf(fx) < 2147483520.0f ? static_cast<int>(fx) : 0;
    int ty = fabsf(fy) < 2147483520.0f ? static_cast<int>(fy) : 0;
    tx = min(max(tx, 0), w - 1);
    ty = min(max(ty, 0), h - 1);
    return gmax(texelFetch(t, tx, ty).z, 0.0f);
}

// min(first i with target <= values[i], n - 1): the index the reference's
// binary search returns (:600-650), found through the skip array first (one
// 128-byte line per 32 values) and then inside one 32-value segment. Equal to
// the plain binary search when the values are non-decreasing, which the host
// checks before it builds the arrays.
HDCX_D int cdfSearch(const float* values, const float* skip, int n, float target)
{
    int low = 0;
    int high = (n + 31) / 32 - 1;
    while (low < high) {
        const int middle = (low + high) / 2;
        if (target <= __ldg(skip + middle)) high = middle;
        else low = middle + 1;
    }
    high = min(low * 32 + 31, n - 1);
    low = low * 32;
    while (low < high) {
        const int middle = (low + high) / 2;
        if (target <= __ldg(values + middle)) high = middle;
        else low = middle + 1;
    }
    return low;
}

HDCX_D void sampleDomeLight(const DeviceScene& s, const GpuLight& light, uint32_t& rng, float3& worldDirection, float& pdf)
{
    // :600-650
    const TexDesc* tp = importanceTexture(s, light.textureInfo.w);
    if (!tp) {
        worldDirection = uniformSphere(rng);
        pdf = 1.0f / 12.5663706144f;
        return;
    }
    const TexDesc t = *tp;
    const int w = static_cast<int>(t.width), h = static_cast<int>(t.height);
    const float4* texels = reinterpret_cast<const float4*>(t.texels);
    const float rowTarget = randomFloat(rng);
    int row, column;
    if (t.cdf) {
        const float* marginal = t.cdf;
        const float* marginalSkip = marginal + h;
        const float* conditional = marginalSkip + (h + 31) / 32;
        const int ws = (w + 31) / 32;
        const float* conditionalSkip = conditional + static_cast<size_t>(h) * w;
        row = cdfSearch(marginal, marginalSkip, h, rowTarget);
        const float columnTarget = randomFloat(rng);
        column = cdfSearch(conditional + static_cast<size_t>(row) * w, conditionalSkip + static_cast<size_t>(row) * ws, w,
                           columnTarget);
    } else {
        int low = 0;
        int high = h - 1;
        while (low < high) {
            const int middle = (low + high) / 2;
            const float cdf = __ldg(&texels[static_cast<size_t>(middle) * t.width].y);
            if (rowTarget <= cdf) high = middle;
            else low = middle + 1;
        }
        row = low;
        const float columnTarget = randomFloat(rng);
        low = 0;
        high = w - 1;
        const float4* rowTexels = texels + static_cast<size_t>(row) * t.width;
        while (low < high) {
            const int middle = (low + high) / 2;
            const float cdf = __ldg(&rowTexels[middle].x);
            if (columnTarget <= cdf) high = middle;
            else low = middle + 1;
        }
        column = low;
    }
    const float4* rowTexels = texels + static_cast<size_t>(row) * t.width;
    const float v0 = static_cast<float>(row) / static_cast<float>(h);
    const float v1 = static_cast<float>(row + 1) / static_cast<float>(h);
    const float cosine0 = gcos(kPi * (1.0f - v0));
    const float cosine1 = gcos(kPi * (1.0f - v1));
    const float cosineTheta = mix(cosine0, cosine1, randomFloat(rng));
    const float v = 1.0f - gacos(clampf(cosineTheta, -1.0f, 1.0f)) / kPi;
    const float u = (static_cast<float>(column) + randomFloat(rng)) / static_cast<float>(w);
    const float3 localDirection = latLongDirection(u, v);
    worldDirection = normalize(xyz(light.basisX) * localDirection.x + xyz(light.basisY) * localDirection.y +
                               xyz(light.basisZ) * localDirection.z);
    pdf = gmax(__ldg(&rowTexels[column].z), 0.0f);
}

HDCX_D float lightSelectionWeight(const GpuLight& light, float3 position, float3 normal, float diffuseEnergy,
                                  float specularEnergy, float translucentEnergy)
{
    // :652-691
    const float power = gmax(light.geometry.w, 0.0f);
    if (power <= 0.0f) return 0.0f;
    const float diffuseResponse = gmax(diffuseEnergy, 0.0f) * light.controls.x;
    const float specularResponse = gmax(specularEnergy, 0.0f) * light.controls.y;
    const float transmissionResponse = gmax(translucentEnergy, 0.0f) * light.controls.x;
    const float minimumWeight = power * 0.01f;
    const uint32_t type = light.textureInfo.z;
    if (type == 0u) {
        return gmax(minimumWeight, power * (0.5f * (diffuseResponse + transmissionResponse) + specularResponse));
    }
    float3 direction;
    float geometryFactor = 1.0f;
    if (type == 5u) {
        direction = normalize(xyz(light.basisZ));
    } else {
        const float3 toLight = xyz(light.position) - position;
        const float distanceSquared = gmax(dot(toLight, toLight), 1e-4f);
        direction = toLight * inversesqrt(distanceSquared);
        geometryFactor = 1.0f / distanceSquared;
        if (type == 1u || type == 2u) {
            const float3 lightNormal = -normalize(xyz(light.basisZ));
            geometryFactor = geometryFactor * gmax(dot(lightNormal, -direction), 0.0f);
        } else if (type == 4u) {
            geometryFactor = geometryFactor * 0.5f;
        }
    }
    const float nDotL = dot(normal, direction);
    const float response = gmax(nDotL, 0.0f) * (diffuseResponse + specularResponse) + gmax(-nDotL, 0.0f) * transmissionResponse;
    return gmax(minimumWeight, power * geometryFactor * response);
}

// `lights`: the scene's light records, s.lights or a shared-memory copy of them.
HDCX_D float totalAnalyticLightWeight(const DeviceScene& s, const GpuLight* lights, float3 position, float3 normal,
                                      float diffuseEnergy, float specularEnergy, float translucentEnergy)
{
    // :693-705
    float total = 0.0f;
    for (uint32_t index = 0; index < s.lightCount; ++index) {
        total += lightSelectionWeight(lights[index], position, normal, diffuseEnergy, specularEnergy, translucentEnergy);
    }
    return total;
}

HDCX_D void sampleAnalyticLight(const DeviceScene& s, const GpuLight* lights, float3 position, float3 normal,
                                float diffuseEnergy, float specularEnergy, float translucentEnergy, uint32_t& rng,
                                uint32_t& lightIndex, float& selectionPdf)
{
    // :707-737
    const uint32_t lightCount = s.lightCount;
    const float total = totalAnalyticLightWeight(s, lights, position, normal, diffuseEnergy, specularEnergy, translucentEnergy);
    if (total <= 0.0f) {
        const float scaled = randomFloat(rng) * u2f(lightCount);
        const uint32_t pick = scaled >= 4294967296.0f ? 0xffffffffu : static_cast<uint32_t>(scaled);
        lightIndex = min(pick, lightCount - 1u);
        selectionPdf = 1.0f / u2f(lightCount);
        return;
    }
    const float target = randomFloat(rng) * total;
    float accumulated = 0.0f;
    lightIndex = lightCount - 1u;
    for (uint32_t index = 0; index < lightCount; ++index) {
        const float weight = lightSelectionWeight(lights[index], position, normal, diffuseEnergy, specularEnergy, translucentEnergy);
        accumulated += weight;
        if (target <= accumulated) {
            lightIndex = index;
            break;
        }
    }
    selectionPdf = lightSelectionWeight(lights[lightIndex], position, normal, diffuseEnergy, specularEnergy, translucentEnergy) / total;
}

// Not inlined: called from several sites of the shade kernel, one shared
// copy keeps the kernel's instruction footprint smaller (measured faster).
HDCX_NOINLINE float environmentLightPdf(const DeviceScene& s, const GpuLight* lights, float3 position, float3 normal,
                                        float3 direction, float diffuseEnergy, float specularEnergy, float translucentEnergy)
{
    // :739-758
    if (s.lightCount == 0u) return 0.0f;
    const float total = totalAnalyticLightWeight(s, lights, position, normal, diffuseEnergy, specularEnergy, translucentEnergy);
    if (total <= 0.0f) return 0.0f;
    float pdf = 0.0f;
    for (uint32_t index = 0; index < s.lightCount; ++index) {
        const GpuLight& light = lights[index];
        if (light.textureInfo.z == 0u) {
            const float selectionPdf =
                lightSelectionWeight(light, position, normal, diffuseEnergy, specularEnergy, translucentEnergy) / total;
            pdf += selectionPdf * domeLightPdf(s, light, direction);
        }
    }
    return pdf;
}

// ---------------------------------------------------------------------------
// Surface frame (vulkan_path_tracer.cpp:807-853)
// ---------------------------------------------------------------------------
HDCX_D float3 applyNormalMap(const DeviceScene& s, uint32_t textureIndex, bool flipY, float scale, float2 uv,
                             float3 geometricNormal, float3 p0, float3 p1, float3 p2, float2 uv0, float2 uv1, float2 uv2)
{
    if (textureIndex == kMissingTexture) return geometricNormal;
    const float2 deltaUv1 = uv1 - uv0;
    const float2 deltaUv2 = uv2 - uv0;
    const float determinant = deltaUv1.x * deltaUv2.y - deltaUv1.y * deltaUv2.x;
    if (fabsf(determinant) < 1e-8f) return geometricNormal;
    const float3 edge1 = p1 - p0;
    const float3 edge2 = p2 - p0;
    float3 tangent = normalize((edge1 * deltaUv2.y - edge2 * deltaUv1.y) / determinant);
    tangent = normalize(tangent - geometricNormal * dot(geometricNormal, tangent));
    float3 bitangent = normalize(cross(geometricNormal, tangent));
    if (determinant < 0.0f) bitangent = -bitangent;
    const float4 t = sampleMaterialTexture(s, textureIndex, uv, make_float4(0.5f, 0.5f, 1.0f, 1.0f));
    float3 mapped = f3(t.x, t.y, t.z) * 2.0f - f3(1.0f);
    if (flipY) mapped.y = -mapped.y;
    mapped.x = mapped.x * scale;
    mapped.y = mapped.y * scale;
    const float3 result = normalize(tangent * mapped.x + bitangent * mapped.y + geometricNormal * mapped.z);
    return dot(result, geometricNormal) < 0.0f ? -result : result;
}

HDCX_D float3 surfaceTangent(float3 normal, float3 p0, float3 p1, float3 p2, float2 uv0, float2 uv1, float2 uv2)
{
    const float2 deltaUv1 = uv1 - uv0;
    const float2 deltaUv2 = uv2 - uv0;
    const float determinant = deltaUv1.x * deltaUv2.y - deltaUv1.y * deltaUv2.x;
    if (fabsf(determinant) < 1e-8f) return orthogonalTangent(normal, f3(1.0f, 0.0f, 0.0f));
    const float3 tangent = ((p1 - p0) * deltaUv2.y - (p2 - p0) * deltaUv1.y) / determinant;
    return orthogonalTangent(normal, tangent);
}

HDCX_D float3 surfaceShadingNormal(const DeviceScene& s, uint32_t primitive, float b1, float b2, float3 geometricNormal)
{
    const float b0 = 1.0f - b1 - b2;
    const float4 n0 = __ldg(s.normals + primitive * 3u + 0u);
    const float4 n1 = __ldg(s.normals + primitive * 3u + 1u);
    const float4 n2 = __ldg(s.normals + primitive * 3u + 2u);
    float3 result = xyz(n0) * b0 + xyz(n1) * b1 + xyz(n2) * b2;
    if (dot(result, result) < 1e-12f) return geometricNormal;
    result = normalize(result);
    return dot(result, geometricNormal) < 0.0f ? -result : result;
}

}  // namespace hdcx
