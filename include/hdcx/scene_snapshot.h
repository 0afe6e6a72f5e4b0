// scene_snapshot.h - the hdCodex scene ABI consumed by the CUDA tracer.
//
// Field-for-field the members that the path tracer reads from the reference's
// include/hdcodex/core/versioned_scene.h:17-274 (SceneMesh, the compact
// closure members of SceneMaterial, SceneTexture, SceneLight, SceneSnapshot)
// and ShadingMode (include/hdcodex/core/shading_mode.h:9-39), with the same
// names and defaults. A Hydra delegate that already has the reference's
// headers defines HDCX_USE_EXTERNAL_SCENE_ABI and uses its own types instead:
// cuda_path_tracer.h only touches the members declared here.
#pragma once

#include <array>
#include <cstdint>
#include <memory>
#include <optional>
#include <string>
#include <string_view>
#include <vector>

namespace hdcodex {

enum class ShadingMode {
    Fused,
    Modular,
    RasterPreview,
};

[[nodiscard]] constexpr std::string_view ShadingModeName(ShadingMode mode) noexcept
{
    switch (mode) {
    case ShadingMode::Fused: return "fused";
    case ShadingMode::Modular: return "modular";
    case ShadingMode::RasterPreview: return "raster";
    }
    return "fused";
}

[[nodiscard]] constexpr std::optional<ShadingMode> ParseShadingMode(std::string_view name) noexcept
{
    if (name == "fused" || name == "fused-specialized") return ShadingMode::Fused;
    if (name == "modular" || name == "instrumented") return ShadingMode::Modular;
    if (name == "raster" || name == "raster-preview") return ShadingMode::RasterPreview;
    return std::nullopt;
}

struct SceneMesh {
    std::string id;
    std::vector<float> positions;
    std::vector<std::uint32_t> indices;
    std::vector<float> texcoords;  // 2 per triangulated face corner
    std::vector<float> normals;    // 3 per face corner; zero = geometric normal
    std::string materialId;
    std::vector<std::string> triangleMaterialIds;
    std::array<float, 3> displayColor{0.5F, 0.5F, 0.5F};
};

struct SceneMaterial {
    enum class DiffuseModel : std::uint32_t {
        Lambert = 0U,
        OrenNayar = 1U,
        Burley = 2U,
        OrenNayarEnergyCompensated = 3U,
    };

    std::string id;
    std::string shaderNodeId;
    std::array<float, 3> baseColor{0.8F, 0.8F, 0.8F};
    std::array<float, 3> baseColorTextureScale{1.0F, 1.0F, 1.0F};
    std::array<float, 3> baseColorTextureBias{0.0F, 0.0F, 0.0F};
    int baseColorTextureChannel{-1};
    std::array<float, 3> emission{0.0F, 0.0F, 0.0F};
    std::array<float, 3> transmissionColor{1.0F, 1.0F, 1.0F};
    std::array<float, 3> transmissionScatter{0.0F, 0.0F, 0.0F};
    std::array<float, 3> specularColor{1.0F, 1.0F, 1.0F};
    std::array<float, 3> coatColor{1.0F, 1.0F, 1.0F};
    std::array<float, 3> sheenColor{1.0F, 1.0F, 1.0F};
    std::array<float, 3> translucentColor{1.0F, 1.0F, 1.0F};
    std::array<float, 3> subsurfaceColor{0.8F, 0.8F, 0.8F};
    std::array<float, 3> subsurfaceRadius{1.0F, 0.2F, 0.1F};
    DiffuseModel diffuseModel{DiffuseModel::Lambert};
    float diffuseWeight{1.0F};
    float diffuseRoughness{0.0F};
    float metalness{0.0F};
    float roughness{0.5F};
    float roughnessV{0.5F};
    float opacity{1.0F};
    float emissionWeight{0.0F};
    float transmission{0.0F};
    float transmissionDepth{0.0F};
    float transmissionScatterAnisotropy{0.0F};
    float transmissionDispersionScale{0.0F};
    float transmissionDispersionAbbeNumber{20.0F};
    float indexOfRefraction{1.5F};
    float specularWeight{1.0F};
    float coat{0.0F};
    float coatRoughness{0.1F};
    float coatRoughnessV{0.1F};
    float coatIndexOfRefraction{1.5F};
    float sheen{0.0F};
    float sheenRoughness{0.3F};
    std::uint32_t sheenMode{0U};
    float translucentWeight{0.0F};
    float subsurface{0.0F};
    float subsurfaceScale{1.0F};
    float subsurfaceScatterAnisotropy{0.0F};
    bool thinWalled{false};
    bool normalTextureFlipY{false};
    float normalTextureScale{1.0F};
    std::string baseColorTexture;
    std::string metalnessTexture;
    std::string roughnessTexture;
    std::string diffuseWeightTexture;
    std::string diffuseRoughnessTexture;
    std::string emissionTexture;
    std::string opacityTexture;
    std::string normalTexture;
    std::string transmissionTexture;
    std::string specularTexture;
    std::string specularColorTexture;
    std::string coatTexture;
    std::string coatColorTexture;
    std::string coatRoughnessTexture;
    std::string sheenTexture;
    std::string sheenColorTexture;
    std::string sheenRoughnessTexture;
    std::string translucentWeightTexture;
    std::string translucentColorTexture;
    std::string subsurfaceTexture;
    std::string subsurfaceColorTexture;
    std::string subsurfaceRadiusTexture;
};

struct SceneTexture {
    std::string id;
    std::string sourcePath;
    std::string udimSetId;
    std::uint32_t udimTile{0};
    std::uint32_t width{0};
    std::uint32_t height{0};
    bool srgb{false};
    std::vector<std::uint8_t> rgba;
    std::vector<float> rgbaFloat;
};

enum class SceneLightType : std::uint32_t {
    Dome,
    Rect,
    Disk,
    Sphere,
    Cylinder,
    Distant,
};

enum class DomeTextureFormat : std::uint32_t {
    Automatic,
    LatLong,
    MirroredBall,
    Angular,
    CubeMapVerticalCross,
};

struct SceneLight {
    std::string id;
    SceneLightType type{SceneLightType::Dome};
    bool visible{true};
    std::array<float, 3> color{1.0F, 1.0F, 1.0F};
    std::array<float, 3> temperatureColor{1.0F, 1.0F, 1.0F};
    float intensity{1.0F};
    float exposure{0.0F};
    float diffuse{1.0F};
    float specular{1.0F};
    bool normalize{false};
    std::string texture;
    DomeTextureFormat textureFormat{DomeTextureFormat::Automatic};
    std::array<float, 3> basisX{1.0F, 0.0F, 0.0F};
    std::array<float, 3> basisY{0.0F, 1.0F, 0.0F};
    std::array<float, 3> basisZ{0.0F, 0.0F, 1.0F};
    std::array<float, 3> position{0.0F, 0.0F, 0.0F};
    std::array<float, 3> axisU{1.0F, 0.0F, 0.0F};
    std::array<float, 3> axisV{0.0F, 1.0F, 0.0F};
    float width{1.0F};
    float height{1.0F};
    float radius{0.5F};
    float length{1.0F};
    float angle{0.53F};
    float area{1.0F};
    float shapingFocus{0.0F};
    std::array<float, 3> shapingFocusTint{0.0F, 0.0F, 0.0F};
    float shapingConeAngle{180.0F};
    float shapingConeSoftness{0.0F};
    bool shadowEnable{true};
    std::array<float, 3> shadowColor{0.0F, 0.0F, 0.0F};
    float shadowDistance{-1.0F};
    float shadowFalloff{-1.0F};
    float shadowFalloffGamma{1.0F};
};

struct SceneSnapshot {
    std::uint64_t revision{0};
    std::vector<SceneMesh> meshes;
    std::vector<SceneMaterial> materials;
    std::vector<SceneTexture> textures;
    std::vector<SceneLight> lights;
};

}  // namespace hdcodex
