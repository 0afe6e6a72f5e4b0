// oracle_scene.cpp - CPU restatement of the reference's scene packing.
// TEST INFRASTRUCTURE ONLY (see oracle_glsl.h).
//
// Follows Impl::BuildScene (src/gpu/vulkan_path_tracer.cpp:2604-2993),
// TextureAverageLuminance (:1968-1996) and BuildLatLongImportanceTexture
// (:1998-2066). The input is the C scene description of include/hdcx.h, whose
// arrays stand for SceneSnapshot's vectors in their published order.
#include "oracle_internal.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>

namespace oracle {
namespace {

std::string Str(const char* s) { return s ? std::string(s) : std::string(); }

// SrgbToLinear (vulkan_path_tracer.cpp:1961-1966), binary32 with std::pow.
float SrgbToLinearFloat(float value)
{
    return value <= 0.04045F ? value / 12.92F : std::pow((value + 0.055F) / 1.055F, 2.4F);
}

// A texture the snapshot would hold: VersionedScene::UpsertTexture drops ids
// that are empty, zero-sized or whose pixel array has the wrong length
// (versioned_scene.h:355-364), so such entries never reach BuildScene.
bool TextureAccepted(const hdcx_texture_desc& t)
{
    if (!t.id || !t.id[0] || t.width == 0 || t.height == 0) return false;
    const uint64_t expected = uint64_t(t.width) * t.height * 4u;
    const bool bytesOk = t.rgba && t.rgba_count == expected;
    const bool floatsOk = t.rgba_float && t.rgba_float_count == expected;
    return bytesOk || floatsOk;
}

bool HasFloat(const hdcx_texture_desc& t)
{
    const uint64_t expected = uint64_t(t.width) * t.height * 4u;
    return t.rgba_float && t.rgba_float_count == expected;
}

Texture CreateTexture(const hdcx_texture_desc& source)
{
    Texture result;
    result.width = source.width;
    result.height = source.height;
    const size_t count = size_t(source.width) * source.height * 4u;
    result.linear.resize(count);
    if (HasFloat(source)) {
        result.format = HDCX_TEXEL_RGBA32F;
        result.floats.assign(source.rgba_float, source.rgba_float + count);
        std::memcpy(result.linear.data(), source.rgba_float, count * sizeof(float));
    } else {
        result.format = source.srgb ? HDCX_TEXEL_RGBA8_SRGB : HDCX_TEXEL_RGBA8_UNORM;
        result.bytes.assign(source.rgba, source.rgba + count);
        for (size_t i = 0; i < count; ++i) {
            const uint8_t b = source.rgba[i];
            const bool colour = (i & 3u) != 3u;
            result.linear[i] = (source.srgb && colour) ? SrgbByteToLinear(b)
                                                        : static_cast<float>(b) / 255.0f;
        }
    }
    return result;
}

Texture CreateFloatTexture(uint32_t w, uint32_t h, std::vector<float> rgba)
{
    Texture result;
    result.width = w;
    result.height = h;
    result.format = HDCX_TEXEL_RGBA32F;
    result.linear = rgba;
    result.floats = std::move(rgba);
    return result;
}

// TextureAverageLuminance (vulkan_path_tracer.cpp:1968-1996).
float TextureAverageLuminance(const hdcx_texture_desc& source)
{
    if (source.width == 0 || source.height == 0) return 0.0f;
    const size_t pixelCount = size_t(source.width) * source.height;
    const bool useFloat = source.rgba_float && source.rgba_float_count > 0;
    if ((useFloat && source.rgba_float_count < pixelCount * 4u) ||
        (!useFloat && (!source.rgba || source.rgba_count < pixelCount * 4u))) {
        return 0.0f;
    }
    double total = 0.0;
    for (size_t pixel = 0; pixel < pixelCount; ++pixel) {
        const size_t offset = pixel * 4u;
        float rgb[3];
        for (size_t c = 0; c < 3; ++c) {
            float value = useFloat ? source.rgba_float[offset + c]
                                   : static_cast<float>(source.rgba[offset + c]) / 255.0F;
            if (!useFloat && source.srgb) value = SrgbToLinearFloat(value);
            rgb[c] = std::isfinite(value) ? std::max(value, 0.0F) : 0.0F;
        }
        total += 0.2126 * rgb[0] + 0.7152 * rgb[1] + 0.0722 * rgb[2];
    }
    return static_cast<float>(total / static_cast<double>(pixelCount));
}

// BuildLatLongImportanceTexture (vulkan_path_tracer.cpp:1998-2066):
// R = conditional CDF of the row, G = marginal CDF of the row, B = pdf.
bool BuildLatLongImportance(const hdcx_texture_desc& source, Texture* out)
{
    if (source.width == 0 || source.height == 0) return false;
    const size_t pixelCount = size_t(source.width) * source.height;
    const bool useFloat = source.rgba_float && source.rgba_float_count > 0;
    std::vector<float> luminance(pixelCount, 0.0F);
    std::vector<double> weights(pixelCount, 0.0);
    std::vector<double> rowWeights(source.height, 0.0);
    constexpr double pi = 3.14159265358979323846;
    const double deltaPhi = 2.0 * pi / static_cast<double>(source.width);
    double totalWeight = 0.0;
    for (uint32_t y = 0; y < source.height; ++y) {
        const double v0 = static_cast<double>(y) / source.height;
        const double v1 = static_cast<double>(y + 1u) / source.height;
        const double cosine0 = std::cos(pi * (1.0 - v0));
        const double cosine1 = std::cos(pi * (1.0 - v1));
        const double solidAngle = deltaPhi * std::abs(cosine1 - cosine0);
        for (uint32_t x = 0; x < source.width; ++x) {
            const size_t pixel = size_t(y) * source.width + x;
            const size_t offset = pixel * 4u;
            float rgb[3];
            for (size_t c = 0; c < 3; ++c) {
                float value = useFloat ? source.rgba_float[offset + c]
                                       : static_cast<float>(source.rgba[offset + c]) / 255.0F;
                if (!useFloat && source.srgb) value = SrgbToLinearFloat(value);
                rgb[c] = std::isfinite(value) ? std::max(value, 0.0F) : 0.0F;
            }
            const float value = 0.2126F * rgb[0] + 0.7152F * rgb[1] + 0.0722F * rgb[2];
            luminance[pixel] = value;
            weights[pixel] = static_cast<double>(value) * solidAngle;
            rowWeights[y] += weights[pixel];
            totalWeight += weights[pixel];
        }
    }
    if (!(totalWeight > 0.0) || !std::isfinite(totalWeight)) return false;
    std::vector<float> rgba(pixelCount * 4u);
    double marginalCdf = 0.0;
    for (uint32_t y = 0; y < source.height; ++y) {
        marginalCdf += rowWeights[y] / totalWeight;
        double conditionalCdf = 0.0;
        for (uint32_t x = 0; x < source.width; ++x) {
            const size_t pixel = size_t(y) * source.width + x;
            conditionalCdf += rowWeights[y] > 0.0 ? weights[pixel] / rowWeights[y]
                                                  : 1.0 / static_cast<double>(source.width);
            const size_t offset = pixel * 4u;
            rgba[offset] = static_cast<float>(x + 1u == source.width ? 1.0 : conditionalCdf);
            rgba[offset + 1] = static_cast<float>(y + 1u == source.height ? 1.0 : marginalCdf);
            rgba[offset + 2] =
                static_cast<float>(static_cast<double>(luminance[pixel]) / totalWeight);
            rgba[offset + 3] = 1.0F;
        }
    }
    *out = CreateFloatTexture(source.width, source.height, std::move(rgba));
    return true;
}

vec4 F4(float x, float y, float z, float w) { return V4(x, y, z, w); }

GpuMaterial DefaultMaterial(const std::array<float, 3>& color)
{
    // vulkan_path_tracer.cpp:2768-2800
    GpuMaterial m;
    m.baseColorMetalness = F4(color[0], color[1], color[2], 0.0F);
    m.emissionRoughness = F4(0.0F, 0.0F, 0.0F, 0.5F);
    m.transmissionOpacityIor = F4(0.0F, 1.0F, 1.5F, 0.0F);
    m.transmissionColorThinWalled = F4(1.0F, 1.0F, 1.0F, 0.0F);
    m.subsurfaceWeightScale = F4(0.0F, 1.0F, 0.0F, 0.0F);
    m.subsurfaceColor = F4(color[0], color[1], color[2], 0.0F);
    m.subsurfaceRadius = F4(1.0F, 0.2F, 0.1F, 0.0F);
    m.specularWeightColor = F4(1.0F, 1.0F, 1.0F, 1.0F);
    m.coatWeightRoughnessIor = F4(0.0F, 0.1F, 1.5F, 0.0F);
    m.coatColor = F4(1.0F, 1.0F, 1.0F, 0.0F);
    m.transmissionMedium = F4(0.0F, 0.0F, 0.0F, 20.0F);
    m.transmissionScatter = F4(0.0F, 0.0F, 0.0F, 0.0F);
    m.sheenColorMode = F4(1.0F, 1.0F, 1.0F, 0.0F);
    m.diffuseProperties = F4(0.0F, 0.0F, 1.0F, 0.0F);
    m.translucentColorWeight = F4(1.0F, 1.0F, 1.0F, 0.0F);
    m.baseColorTextureScale = F4(1.0F, 1.0F, 1.0F, -1.0F);
    m.baseColorTextureBias = F4(0.0F, 0.0F, 0.0F, 0.0F);
    const std::array<uint32_t, 4> none{kMissingTexture, kMissingTexture, kMissingTexture,
                                       kMissingTexture};
    m.textureIndices0 = m.textureIndices1 = m.textureIndices2 = none;
    m.textureIndices3 = m.textureIndices4 = m.textureIndices5 = none;
    return m;
}

}  // namespace

float SrgbByteToLinear(uint8_t value)
{
    const double c = static_cast<double>(value) / 255.0;
    const double linear = c <= 0.04045 ? c / 12.92 : std::pow((c + 0.055) / 1.055, 2.4);
    return static_cast<float>(linear);
}

PackedScene PackScene(const hdcx_scene_desc& snapshot)
{
    PackedScene out;
    const auto materialsBegin = snapshot.materials;
    const auto materialsEnd = snapshot.materials + snapshot.material_count;
    // vulkan_path_tracer.cpp:2609-2612
    out.opaque = std::all_of(materialsBegin, materialsEnd, [](const hdcx_material_desc& m) {
        return m.opacity >= 0.999F && Str(m.opacity_texture).empty();
    });

    std::vector<const hdcx_texture_desc*> accepted;
    for (uint64_t i = 0; i < snapshot.texture_count; ++i) {
        if (TextureAccepted(snapshot.textures[i])) accepted.push_back(&snapshot.textures[i]);
    }

    // Textures and UDIM sets (vulkan_path_tracer.cpp:2622-2658).
    std::map<std::string, uint32_t, std::less<>> textureIndices;
    std::map<std::string, const hdcx_texture_desc*, std::less<>> textureSources;
    std::map<std::string, std::vector<const hdcx_texture_desc*>, std::less<>> udimSets;
    auto& textures = out.textures;
    for (const hdcx_texture_desc* texture : accepted) {
        const std::string setId = Str(texture->udim_set_id);
        if (!setId.empty() && texture->udim_tile != 0u) {
            udimSets[setId].push_back(texture);
            continue;
        }
        if (textures.size() >= kMaxMaterialTextures) continue;
        textureSources[Str(texture->id)] = texture;
        textureIndices[Str(texture->id)] = static_cast<uint32_t>(textures.size());
        textures.push_back(CreateTexture(*texture));
    }
    for (auto& [setId, tiles] : udimSets) {
        std::stable_sort(tiles.begin(), tiles.end(),
                         [](const hdcx_texture_desc* l, const hdcx_texture_desc* r) {
                             return l->udim_tile < r->udim_tile;
                         });
        const uint32_t base = static_cast<uint32_t>(textures.size());
        uint32_t presentTiles = 0u;
        for (const hdcx_texture_desc* tile : tiles) {
            if (textures.size() >= kMaxMaterialTextures) break;
            if (tile->udim_tile < 1001u || tile->udim_tile > 1023u) continue;
            presentTiles |= 1u << (tile->udim_tile - 1001u);
            textures.push_back(CreateTexture(*tile));
        }
        if (presentTiles != 0u) {
            textureIndices[setId] = kUdimTextureFlag | ((presentTiles & kUdimTileMask) << 8u) | base;
        }
    }
    const auto textureIndex = [&](const char* id) {
        const auto found = textureIndices.find(Str(id));
        return found == textureIndices.end() ? kMissingTexture : found->second;
    };
    std::map<std::string, float, std::less<>> luminanceCache;
    const auto textureAverageLuminance = [&](const std::string& id) {
        const auto cached = luminanceCache.find(id);
        if (cached != luminanceCache.end()) return cached->second;
        double total = 0.0;
        size_t count = 0;
        if (const auto source = textureSources.find(id); source != textureSources.end()) {
            total = TextureAverageLuminance(*source->second);
            count = 1;
        } else if (const auto tiles = udimSets.find(id); tiles != udimSets.end()) {
            for (const hdcx_texture_desc* tile : tiles->second) {
                total += TextureAverageLuminance(*tile);
                ++count;
            }
        }
        const float result = count > 0 ? static_cast<float>(total / static_cast<double>(count)) : 0.0F;
        luminanceCache.emplace(id, result);
        return result;
    };
    std::map<std::string, uint32_t, std::less<>> domeImportanceIndices;
    // vulkan_path_tracer.cpp:2681-2702
    const auto domeImportanceIndex = [&](const hdcx_light_desc& light) {
        if (light.type != HDCX_LIGHT_DOME ||
            (light.texture_format != HDCX_DOME_AUTOMATIC && light.texture_format != HDCX_DOME_LATLONG) ||
            textureIndex(light.texture) == kMissingTexture) {
            return kMissingTexture;
        }
        const std::string key = Str(light.texture);
        const auto cached = domeImportanceIndices.find(key);
        if (cached != domeImportanceIndices.end()) return cached->second;
        const auto source = textureSources.find(key);
        if (source == textureSources.end() || textures.size() >= kMaxMaterialTextures) {
            return kMissingTexture;
        }
        Texture importance;
        if (!BuildLatLongImportance(*source->second, &importance)) return kMissingTexture;
        const uint32_t index = static_cast<uint32_t>(textures.size());
        textures.push_back(std::move(importance));
        domeImportanceIndices.emplace(key, index);
        return index;
    };

    // Lights (vulkan_path_tracer.cpp:2704-2766).
    for (uint64_t i = 0; i < snapshot.light_count; ++i) {
        const hdcx_light_desc& light = snapshot.lights[i];
        if (!light.visible || out.lights.size() >= kMaxLights) continue;
        float radianceScale = light.intensity * std::exp2(light.exposure);
        if (light.type != HDCX_LIGHT_DOME && light.type != HDCX_LIGHT_DISTANT && light.normalize) {
            radianceScale /= std::max(light.area, 1e-8F);
        }
        const std::array<float, 3> emittedColor{light.color[0] * light.temperature_color[0],
                                                light.color[1] * light.temperature_color[1],
                                                light.color[2] * light.temperature_color[2]};
        float emittedLuminance = 0.2126F * std::max(emittedColor[0], 0.0F) +
                                 0.7152F * std::max(emittedColor[1], 0.0F) +
                                 0.0722F * std::max(emittedColor[2], 0.0F);
        if (!Str(light.texture).empty() &&
            (light.type == HDCX_LIGHT_DOME || light.type == HDCX_LIGHT_RECT)) {
            emittedLuminance *= textureAverageLuminance(Str(light.texture));
        }
        float emitterMeasure = 1.0F;
        if (light.type == HDCX_LIGHT_DOME) {
            emitterMeasure = 12.5663706144F;
        } else if (light.type != HDCX_LIGHT_DISTANT) {
            emitterMeasure = std::max(light.area, 0.0F);
        }
        float selectionPower =
            std::max(emittedLuminance * std::max(radianceScale, 0.0F) * emitterMeasure, 0.0F);
        if (!std::isfinite(selectionPower)) selectionPower = 0.0F;
        GpuLight g;
        g.colorIntensity = F4(emittedColor[0], emittedColor[1], emittedColor[2], radianceScale);
        g.controls = F4(light.diffuse, light.specular, static_cast<float>(light.type),
                        std::max(light.area, 0.0F));
        g.position = F4(light.position[0], light.position[1], light.position[2], 0.0F);
        g.axisU = F4(light.axis_u[0], light.axis_u[1], light.axis_u[2], 0.0F);
        g.axisV = F4(light.axis_v[0], light.axis_v[1], light.axis_v[2], 0.0F);
        g.basisX = F4(light.basis_x[0], light.basis_x[1], light.basis_x[2], 0.0F);
        g.basisY = F4(light.basis_y[0], light.basis_y[1], light.basis_y[2], 0.0F);
        g.basisZ = F4(light.basis_z[0], light.basis_z[1], light.basis_z[2], 0.0F);
        g.shaping = F4(light.shaping_focus, light.shaping_cone_angle, light.shaping_cone_softness, 0.0F);
        g.focusTint = F4(light.shaping_focus_tint[0], light.shaping_focus_tint[1],
                         light.shaping_focus_tint[2], 0.0F);
        g.shadow = F4(light.shadow_enable ? 1.0F : 0.0F, light.shadow_distance, light.shadow_falloff,
                      light.shadow_falloff_gamma);
        g.shadowColor = F4(light.shadow_color[0], light.shadow_color[1], light.shadow_color[2], 0.0F);
        g.geometry = F4(light.radius, light.length, light.angle, selectionPower);
        const uint32_t texIndex = textureIndex(light.texture);
        const uint32_t importance = domeImportanceIndex(light);
        g.textureInfo = {texIndex, light.texture_format, light.type, importance};
        out.lights.push_back(g);
    }
    out.lightCount = static_cast<uint32_t>(out.lights.size());
    if (out.lights.empty()) {
        GpuLight dummy{};
        dummy.shadow = F4(1.0F, -1.0F, -1.0F, 1.0F);
        out.lights.push_back(dummy);
    }

    // Materials (vulkan_path_tracer.cpp:2801-2881).
    auto& materials = out.materials;
    std::vector<float> materialEmissionPowers;
    materials.push_back(DefaultMaterial({0.8F, 0.8F, 0.8F}));
    materialEmissionPowers.push_back(0.0F);
    std::map<std::string, uint32_t, std::less<>> materialIndices;
    for (uint64_t i = 0; i < snapshot.material_count; ++i) {
        const hdcx_material_desc& m = snapshot.materials[i];
        const uint32_t index = static_cast<uint32_t>(materials.size());
        materialIndices[Str(m.id)] = index;
        GpuMaterial g;
        g.baseColorMetalness = F4(m.base_color[0], m.base_color[1], m.base_color[2], m.metalness);
        g.emissionRoughness = F4(m.emission[0], m.emission[1], m.emission[2], m.roughness);
        g.transmissionOpacityIor = F4(m.transmission, m.opacity, m.index_of_refraction, m.emission_weight);
        g.transmissionColorThinWalled = F4(m.transmission_color[0], m.transmission_color[1],
                                           m.transmission_color[2], m.thin_walled ? 1.0F : 0.0F);
        g.subsurfaceWeightScale = F4(m.subsurface, m.subsurface_scale,
                                     m.subsurface_scatter_anisotropy, m.normal_texture_scale);
        g.subsurfaceColor = F4(m.subsurface_color[0], m.subsurface_color[1], m.subsurface_color[2],
                               m.roughness_v);
        g.subsurfaceRadius = F4(m.subsurface_radius[0], m.subsurface_radius[1],
                                m.subsurface_radius[2], m.coat_roughness_v);
        g.specularWeightColor = F4(m.specular_weight, m.specular_color[0], m.specular_color[1],
                                   m.specular_color[2]);
        g.coatWeightRoughnessIor = F4(m.coat, m.coat_roughness, m.coat_index_of_refraction,
                                      m.normal_texture_flip_y ? 1.0F : 0.0F);
        g.coatColor = F4(m.coat_color[0], m.coat_color[1], m.coat_color[2], m.sheen);
        g.transmissionMedium = F4(m.transmission_depth, m.transmission_scatter_anisotropy,
                                  m.transmission_dispersion_scale,
                                  m.transmission_dispersion_abbe_number);
        g.transmissionScatter = F4(m.transmission_scatter[0], m.transmission_scatter[1],
                                   m.transmission_scatter[2], m.sheen_roughness);
        g.sheenColorMode = F4(m.sheen_color[0], m.sheen_color[1], m.sheen_color[2],
                              static_cast<float>(m.sheen_mode));
        g.diffuseProperties = F4(m.diffuse_roughness, static_cast<float>(m.diffuse_model),
                                 m.diffuse_weight, 0.0F);
        g.translucentColorWeight = F4(m.translucent_color[0], m.translucent_color[1],
                                      m.translucent_color[2], m.translucent_weight);
        g.baseColorTextureScale = F4(m.base_color_texture_scale[0], m.base_color_texture_scale[1],
                                     m.base_color_texture_scale[2],
                                     static_cast<float>(m.base_color_texture_channel));
        g.baseColorTextureBias = F4(m.base_color_texture_bias[0], m.base_color_texture_bias[1],
                                    m.base_color_texture_bias[2], 0.0F);
        g.textureIndices0 = {textureIndex(m.base_color_texture), textureIndex(m.metalness_texture),
                             textureIndex(m.roughness_texture), textureIndex(m.emission_texture)};
        g.textureIndices1 = {textureIndex(m.opacity_texture), textureIndex(m.normal_texture),
                             textureIndex(m.transmission_texture), textureIndex(m.sheen_texture)};
        g.textureIndices2 = {textureIndex(m.subsurface_texture), textureIndex(m.subsurface_color_texture),
                             textureIndex(m.subsurface_radius_texture),
                             textureIndex(m.sheen_color_texture)};
        g.textureIndices3 = {textureIndex(m.specular_texture), textureIndex(m.specular_color_texture),
                             textureIndex(m.coat_texture), textureIndex(m.coat_color_texture)};
        g.textureIndices4 = {textureIndex(m.coat_roughness_texture),
                             textureIndex(m.sheen_roughness_texture),
                             textureIndex(m.diffuse_roughness_texture),
                             textureIndex(m.diffuse_weight_texture)};
        g.textureIndices5 = {textureIndex(m.translucent_weight_texture),
                             textureIndex(m.translucent_color_texture), kMissingTexture,
                             kMissingTexture};
        materials.push_back(g);
        const float emissionLuminance =
            Str(m.emission_texture).empty()
                ? 0.2126F * std::max(m.emission[0], 0.0F) + 0.7152F * std::max(m.emission[1], 0.0F) +
                      0.0722F * std::max(m.emission[2], 0.0F)
                : textureAverageLuminance(Str(m.emission_texture));
        materialEmissionPowers.push_back(std::max(m.emission_weight, 0.0F) * emissionLuminance);
    }

    // Geometry flattening (vulkan_path_tracer.cpp:2882-2940).
    std::map<std::array<float, 3>, uint32_t> displayColorMaterials;
    for (uint64_t meshIndex = 0; meshIndex < snapshot.mesh_count; ++meshIndex) {
        const hdcx_mesh_desc& mesh = snapshot.meshes[meshIndex];
        const uint32_t base = static_cast<uint32_t>(out.vertices.size());
        for (uint64_t i = 0; i + 2 < mesh.position_count; i += 3) {
            out.vertices.push_back(V4(mesh.positions[i], mesh.positions[i + 1], mesh.positions[i + 2], 1.0F));
        }
        const std::string meshMaterial = Str(mesh.material_id);
        const auto foundMaterial = materialIndices.find(meshMaterial);
        uint32_t materialIndex = foundMaterial == materialIndices.end() ? 0u : foundMaterial->second;
        if (meshMaterial.empty()) {
            std::array<float, 3> color{mesh.display_color[0], mesh.display_color[1], mesh.display_color[2]};
            for (float& c : color) c = std::isfinite(c) ? std::clamp(c, 0.0F, 1.0F) : 0.5F;
            const auto found = displayColorMaterials.find(color);
            if (found != displayColorMaterials.end()) {
                materialIndex = found->second;
            } else {
                materialIndex = static_cast<uint32_t>(materials.size());
                displayColorMaterials.emplace(color, materialIndex);
                materials.push_back(DefaultMaterial(color));
                materialEmissionPowers.push_back(0.0F);
            }
        }
        const uint64_t localVertices = out.vertices.size() - base;
        for (uint64_t triangle = 0; triangle + 2 < mesh.index_count; triangle += 3) {
            const uint32_t i0 = mesh.indices[triangle];
            const uint32_t i1 = mesh.indices[triangle + 1];
            const uint32_t i2 = mesh.indices[triangle + 2];
            if (!(i0 < localVertices && i1 < localVertices && i2 < localVertices)) continue;
            out.indices.insert(out.indices.end(), {base + i0, base + i1, base + i2});
            const uint64_t triangleIndex = triangle / 3u;
            uint32_t triangleMaterialIndex = materialIndex;
            if (triangleIndex < mesh.triangle_material_id_count && mesh.triangle_material_ids) {
                const std::string id = Str(mesh.triangle_material_ids[triangleIndex]);
                if (id != meshMaterial) {
                    const auto f = materialIndices.find(id);
                    triangleMaterialIndex = f == materialIndices.end() ? 0u : f->second;
                }
            }
            out.triangleMaterials.push_back(triangleMaterialIndex);
            for (uint64_t corner = 0; corner < 3u; ++corner) {
                const uint64_t uvOffset = (triangle + corner) * 2u;
                out.texcoords.push_back(uvOffset + 1u < mesh.texcoord_count && mesh.texcoords
                                            ? V2(mesh.texcoords[uvOffset], mesh.texcoords[uvOffset + 1])
                                            : V2(0.0F, 0.0F));
                const uint64_t nOffset = (triangle + corner) * 3u;
                out.normals.push_back(nOffset + 2u < mesh.normal_count && mesh.normals
                                          ? V4(mesh.normals[nOffset], mesh.normals[nOffset + 1],
                                               mesh.normals[nOffset + 2], 0.0F)
                                          : V4(0.0F, 0.0F, 0.0F, 0.0F));
            }
        }
    }
    if (out.vertices.empty() || out.indices.empty()) {
        out.geometryReady = false;
        return out;
    }
    out.primitiveCount = static_cast<uint32_t>(out.triangleMaterials.size());

    // Emissive-triangle CDF in FP64 (vulkan_path_tracer.cpp:2944-2993).
    const size_t n = out.triangleMaterials.size();
    out.emissive.assign(n, V4(0.0F, 0.0F, 0.0F, 0.0F));
    std::vector<double> emissiveWeights(n, 0.0);
    std::vector<float> triangleAreas(n, 0.0F);
    double totalEmissiveWeight = 0.0;
    for (size_t primitive = 0; primitive < n; ++primitive) {
        const vec4& p0 = out.vertices[out.indices[primitive * 3]];
        const vec4& p1 = out.vertices[out.indices[primitive * 3 + 1]];
        const vec4& p2 = out.vertices[out.indices[primitive * 3 + 2]];
        const double e1x = static_cast<double>(p1.x) - p0.x;
        const double e1y = static_cast<double>(p1.y) - p0.y;
        const double e1z = static_cast<double>(p1.z) - p0.z;
        const double e2x = static_cast<double>(p2.x) - p0.x;
        const double e2y = static_cast<double>(p2.y) - p0.y;
        const double e2z = static_cast<double>(p2.z) - p0.z;
        const double cx = e1y * e2z - e1z * e2y;
        const double cy = e1z * e2x - e1x * e2z;
        const double cz = e1x * e2y - e1y * e2x;
        const float area = static_cast<float>(0.5 * std::sqrt(cx * cx + cy * cy + cz * cz));
        triangleAreas[primitive] = std::isfinite(area) ? area : 0.0F;
        const uint32_t materialIndex = out.triangleMaterials[primitive];
        const float power =
            materialIndex < materialEmissionPowers.size() ? materialEmissionPowers[materialIndex] : 0.0F;
        const double weight = static_cast<double>(triangleAreas[primitive]) * static_cast<double>(power);
        if (weight > 0.0 && std::isfinite(weight)) {
            emissiveWeights[primitive] = weight;
            totalEmissiveWeight += weight;
        }
    }
    if (totalEmissiveWeight > 0.0 && std::isfinite(totalEmissiveWeight)) {
        double cdf = 0.0;
        for (size_t primitive = 0; primitive < n; ++primitive) {
            const double probability = emissiveWeights[primitive] / totalEmissiveWeight;
            cdf += probability;
            const float area = triangleAreas[primitive];
            out.emissive[primitive] =
                V4(static_cast<float>(primitive + 1u == n ? 1.0 : cdf),
                   area > 0.0F ? static_cast<float>(probability) / area : 0.0F, area, 0.0F);
        }
    }
    out.geometryReady = true;
    return out;
}

}  // namespace oracle
