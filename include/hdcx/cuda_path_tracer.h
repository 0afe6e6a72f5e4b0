// cuda_path_tracer.h - drop-in replacement for hdcodex::VulkanPathTracer.
//
// hdcodex::CudaPathTracer has the methods of the reference's VulkanPathTracer
// (include/hdcodex/gpu/vulkan_path_tracer.h:26-52): SetScene, SetShadingMode,
// GetShadingMode, Render and HasGeometry, with the same argument meaning and
// the same error behaviour (std::runtime_error on a failed call,
// std::invalid_argument for the raster-preview mode). It is a header-only shim
// over the C ABI of hdcx.h, so it compiles against whichever SceneSnapshot the
// including translation unit sees: this project's include/hdcx/scene_snapshot.h
// by default, or the reference's versioned_scene.h when
// HDCX_USE_EXTERNAL_SCENE_ABI is defined. Construction takes a CUDA device
// ordinal where the reference takes (VulkanContext&, ShaderCache&).
#pragma once

#include <algorithm>
#include <array>
#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "hdcx.h"
#ifndef HDCX_USE_EXTERNAL_SCENE_ABI
#include "hdcx/scene_snapshot.h"
#endif

namespace hdcodex {

#ifndef HDCX_USE_EXTERNAL_SCENE_ABI
// PathTracerCamera (vulkan_path_tracer.h:16-23).
struct PathTracerCamera {
    std::array<float, 3> origin{};
    std::array<float, 3> lowerLeft{};
    std::array<float, 3> horizontal{};
    std::array<float, 3> vertical{};

    bool operator==(const PathTracerCamera&) const = default;
};
#endif

namespace hdcx_detail {

inline const char* Str(const std::string& s) { return s.empty() ? nullptr : s.c_str(); }

// Owns the C description of one snapshot; pointers refer into the snapshot,
// which the caller keeps alive for the duration of the call.
template <typename Snapshot>
struct SceneDescHolder {
    std::vector<hdcx_mesh_desc> meshes;
    std::vector<std::vector<const char*>> triangleIds;
    std::vector<hdcx_material_desc> materials;
    std::vector<hdcx_texture_desc> textures;
    std::vector<hdcx_light_desc> lights;
    hdcx_scene_desc desc{};

    explicit SceneDescHolder(const Snapshot& s)
    {
        meshes.reserve(s.meshes.size());
        triangleIds.reserve(s.meshes.size());
        for (const auto& m : s.meshes) {
            hdcx_mesh_desc d;
            hdcx_mesh_defaults(&d);
            d.id = Str(m.id);
            d.positions = m.positions.data();
            d.position_count = m.positions.size();
            d.indices = m.indices.data();
            d.index_count = m.indices.size();
            d.texcoords = m.texcoords.data();
            d.texcoord_count = m.texcoords.size();
            d.normals = m.normals.data();
            d.normal_count = m.normals.size();
            d.material_id = Str(m.materialId);
            auto& ids = triangleIds.emplace_back();
            for (const auto& id : m.triangleMaterialIds) ids.push_back(id.c_str());
            d.triangle_material_ids = ids.empty() ? nullptr : ids.data();
            d.triangle_material_id_count = ids.size();
            std::copy(m.displayColor.begin(), m.displayColor.end(), d.display_color);
            meshes.push_back(d);
        }
        for (const auto& m : s.materials) {
            hdcx_material_desc d;
            hdcx_material_defaults(&d);
            d.id = Str(m.id);
            auto c3 = [](float* dst, const std::array<float, 3>& src) { std::copy(src.begin(), src.end(), dst); };
            c3(d.base_color, m.baseColor);
            c3(d.base_color_texture_scale, m.baseColorTextureScale);
            c3(d.base_color_texture_bias, m.baseColorTextureBias);
            d.base_color_texture_channel = m.baseColorTextureChannel;
            c3(d.emission, m.emission);
            c3(d.transmission_color, m.transmissionColor);
            c3(d.transmission_scatter, m.transmissionScatter);
            c3(d.specular_color, m.specularColor);
            c3(d.coat_color, m.coatColor);
            c3(d.sheen_color, m.sheenColor);
            c3(d.translucent_color, m.translucentColor);
            c3(d.subsurface_color, m.subsurfaceColor);
            c3(d.subsurface_radius, m.subsurfaceRadius);
            d.diffuse_model = static_cast<uint32_t>(m.diffuseModel);
            d.diffuse_weight = m.diffuseWeight;
            d.diffuse_roughness = m.diffuseRoughness;
            d.metalness = m.metalness;
            d.roughness = m.roughness;
            d.roughness_v = m.roughnessV;
            d.opacity = m.opacity;
            d.emission_weight = m.emissionWeight;
            d.transmission = m.transmission;
            d.transmission_depth = m.transmissionDepth;
            d.transmission_scatter_anisotropy = m.transmissionScatterAnisotropy;
            d.transmission_dispersion_scale = m.transmissionDispersionScale;
            d.transmission_dispersion_abbe_number = m.transmissionDispersionAbbeNumber;
            d.index_of_refraction = m.indexOfRefraction;
            d.specular_weight = m.specularWeight;
            d.coat = m.coat;
            d.coat_roughness = m.coatRoughness;
            d.coat_roughness_v = m.coatRoughnessV;
            d.coat_index_of_refraction = m.coatIndexOfRefraction;
            d.sheen = m.sheen;
            d.sheen_roughness = m.sheenRoughness;
            d.sheen_mode = m.sheenMode;
            d.translucent_weight = m.translucentWeight;
            d.subsurface = m.subsurface;
            d.subsurface_scale = m.subsurfaceScale;
            d.subsurface_scatter_anisotropy = m.subsurfaceScatterAnisotropy;
            d.thin_walled = m.thinWalled ? 1 : 0;
            d.normal_texture_flip_y = m.normalTextureFlipY ? 1 : 0;
            d.normal_texture_scale = m.normalTextureScale;
            d.base_color_texture = Str(m.baseColorTexture);
            d.metalness_texture = Str(m.metalnessTexture);
            d.roughness_texture = Str(m.roughnessTexture);
            d.diffuse_weight_texture = Str(m.diffuseWeightTexture);
            d.diffuse_roughness_texture = Str(m.diffuseRoughnessTexture);
            d.emission_texture = Str(m.emissionTexture);
            d.opacity_texture = Str(m.opacityTexture);
            d.normal_texture = Str(m.normalTexture);
            d.transmission_texture = Str(m.transmissionTexture);
            d.specular_texture = Str(m.specularTexture);
            d.specular_color_texture = Str(m.specularColorTexture);
            d.coat_texture = Str(m.coatTexture);
            d.coat_color_texture = Str(m.coatColorTexture);
            d.coat_roughness_texture = Str(m.coatRoughnessTexture);
            d.sheen_texture = Str(m.sheenTexture);
            d.sheen_color_texture = Str(m.sheenColorTexture);
            d.sheen_roughness_texture = Str(m.sheenRoughnessTexture);
            d.translucent_weight_texture = Str(m.translucentWeightTexture);
            d.translucent_color_texture = Str(m.translucentColorTexture);
            d.subsurface_texture = Str(m.subsurfaceTexture);
            d.subsurface_color_texture = Str(m.subsurfaceColorTexture);
            d.subsurface_radius_texture = Str(m.subsurfaceRadiusTexture);
            materials.push_back(d);
        }
        for (const auto& t : s.textures) {
            hdcx_texture_desc d{};
            d.id = Str(t.id);
            d.udim_set_id = Str(t.udimSetId);
            d.udim_tile = t.udimTile;
            d.width = t.width;
            d.height = t.height;
            d.srgb = t.srgb ? 1 : 0;
            d.rgba = t.rgba.empty() ? nullptr : t.rgba.data();
            d.rgba_count = t.rgba.size();
            d.rgba_float = t.rgbaFloat.empty() ? nullptr : t.rgbaFloat.data();
            d.rgba_float_count = t.rgbaFloat.size();
            textures.push_back(d);
        }
        for (const auto& l : s.lights) {
            hdcx_light_desc d;
            hdcx_light_defaults(&d);
            auto c3 = [](float* dst, const std::array<float, 3>& src) { std::copy(src.begin(), src.end(), dst); };
            d.id = Str(l.id);
            d.type = static_cast<uint32_t>(l.type);
            d.visible = l.visible ? 1 : 0;
            c3(d.color, l.color);
            c3(d.temperature_color, l.temperatureColor);
            d.intensity = l.intensity;
            d.exposure = l.exposure;
            d.diffuse = l.diffuse;
            d.specular = l.specular;
            d.normalize = l.normalize ? 1 : 0;
            d.texture = Str(l.texture);
            d.texture_format = static_cast<uint32_t>(l.textureFormat);
            c3(d.basis_x, l.basisX);
            c3(d.basis_y, l.basisY);
            c3(d.basis_z, l.basisZ);
            c3(d.position, l.position);
            c3(d.axis_u, l.axisU);
            c3(d.axis_v, l.axisV);
            d.width = l.width;
            d.height = l.height;
            d.radius = l.radius;
            d.length = l.length;
            d.angle = l.angle;
            d.area = l.area;
            d.shaping_focus = l.shapingFocus;
            c3(d.shaping_focus_tint, l.shapingFocusTint);
            d.shaping_cone_angle = l.shapingConeAngle;
            d.shaping_cone_softness = l.shapingConeSoftness;
            d.shadow_enable = l.shadowEnable ? 1 : 0;
            c3(d.shadow_color, l.shadowColor);
            d.shadow_distance = l.shadowDistance;
            d.shadow_falloff = l.shadowFalloff;
            d.shadow_falloff_gamma = l.shadowFalloffGamma;
            lights.push_back(d);
        }
        desc.revision = s.revision;
        desc.meshes = meshes.data();
        desc.mesh_count = meshes.size();
        desc.materials = materials.data();
        desc.material_count = materials.size();
        desc.textures = textures.data();
        desc.texture_count = textures.size();
        desc.lights = lights.data();
        desc.light_count = lights.size();
    }
};

inline void Throw(hdcx_tracer* t, hdcx_status s, const char* operation)
{
    const std::string message = std::string(operation) + " failed: " + (t ? hdcx_last_error(t) : "") +
                                " (hdcx status " + std::to_string(static_cast<int>(s)) + ")";
    throw std::runtime_error(message);
}

}  // namespace hdcx_detail

// IsSupported probe of the renderer plugin (renderer_plugin.cpp:34-60):
// true when a CUDA device of compute capability 10.x is present.
inline bool IsCudaPathTracingSupported()
{
    int32_t supported = 0, count = 0;
    return hdcx_probe_devices(&supported, &count) == HDCX_OK && supported != 0;
}

class CudaPathTracer final {
public:
    explicit CudaPathTracer(int device = 0)
    {
        const hdcx_status s = hdcx_create(device, &_tracer);
        if (s != HDCX_OK) hdcx_detail::Throw(nullptr, s, "hdcx_create");
    }
    ~CudaPathTracer() { hdcx_destroy(_tracer); }
    CudaPathTracer(const CudaPathTracer&) = delete;
    CudaPathTracer& operator=(const CudaPathTracer&) = delete;

    template <typename Snapshot>
    void SetScene(const std::shared_ptr<Snapshot>& scene)
    {
        if (!scene) {
            const hdcx_status s = hdcx_set_scene(_tracer, nullptr);
            if (s != HDCX_OK) hdcx_detail::Throw(_tracer, s, "SetScene");
            return;
        }
        hdcx_detail::SceneDescHolder<std::remove_const_t<Snapshot>> holder(*scene);
        const hdcx_status s = hdcx_set_scene(_tracer, &holder.desc);
        if (s != HDCX_OK) hdcx_detail::Throw(_tracer, s, "SetScene");
    }

    void SetShadingMode(ShadingMode mode)
    {
        if (mode == ShadingMode::RasterPreview) {
            throw std::invalid_argument("raster preview requires the MaterialX graphics backend");
        }
        const hdcx_status s = hdcx_set_shading_mode(_tracer, static_cast<int32_t>(mode));
        if (s != HDCX_OK) hdcx_detail::Throw(_tracer, s, "SetShadingMode");
    }

    [[nodiscard]] ShadingMode GetShadingMode() const noexcept
    {
        return static_cast<ShadingMode>(hdcx_get_shading_mode(_tracer));
    }

    /// Traces a progressive sample batch per pixel and returns linear RGBA32F
    /// (the cumulative running mean), or an empty vector without geometry.
    [[nodiscard]] std::vector<float> Render(const PathTracerCamera& camera, std::uint32_t width, std::uint32_t height,
                                            std::uint32_t sampleIndex, std::uint32_t maxBounces = 8U,
                                            std::uint32_t sampleCount = 1U)
    {
        if (!HasGeometry() || width == 0 || height == 0) return {};
        hdcx_camera c{};
        std::copy(camera.origin.begin(), camera.origin.end(), c.origin);
        std::copy(camera.lowerLeft.begin(), camera.lowerLeft.end(), c.lower_left);
        std::copy(camera.horizontal.begin(), camera.horizontal.end(), c.horizontal);
        std::copy(camera.vertical.begin(), camera.vertical.end(), c.vertical);
        std::vector<float> pixels(static_cast<size_t>(width) * height * 4U);
        int32_t written = 0;
        const hdcx_status s =
            hdcx_render(_tracer, &c, width, height, sampleIndex, maxBounces, sampleCount, pixels.data(), &written);
        if (s != HDCX_OK) hdcx_detail::Throw(_tracer, s, "Render");
        if (!written) return {};
        return pixels;
    }

    [[nodiscard]] bool HasGeometry() const noexcept { return hdcx_has_geometry(_tracer) != 0; }

    [[nodiscard]] hdcx_tracer* Handle() const noexcept { return _tracer; }

private:
    hdcx_tracer* _tracer = nullptr;
};

}  // namespace hdcodex
