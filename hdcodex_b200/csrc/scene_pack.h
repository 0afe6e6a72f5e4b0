// scene_pack.h - host packing of a scene snapshot into the device layout.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "hdcx.h"

namespace hdcx {

// One packed texture: raw texels as uploaded (RGBA8 bytes or RGBA32F floats).
struct PackedTexture {
    uint32_t width = 0;
    uint32_t height = 0;
    uint32_t format = HDCX_TEXEL_RGBA8_UNORM;
    std::vector<uint8_t> bytes;
    std::vector<float> floats;
};

// An instancer of the packed scene: its prototype in object space and where
// its instances' flattened triangles and vertices sit.
struct PackedInstancer {
    uint32_t mesh = 0;                    // index of the mesh in the snapshot
    std::vector<float> points;            // object space, xyzw per point
    std::vector<uint32_t> indices;        // the prototype's valid triangles (local point indices)
    std::vector<double> transforms;       // 16 per instance, as given
    uint32_t instanceCount = 0;
    uint32_t firstTriangle = 0;           // flattened id of instance 0's first triangle
    uint32_t firstVertex = 0;             // flattened index of instance 0's first vertex
    uint32_t triangles() const { return static_cast<uint32_t>(indices.size() / 3); }
    uint32_t pointCount() const { return static_cast<uint32_t>(points.size() / 4); }
};

// The flattened scene BuildScene produces (vulkan_path_tracer.cpp:2604-2993).
struct PackedSceneData {
    std::vector<float> vertices;            // xyzw per vertex
    std::vector<uint32_t> indices;          // 3 per triangle
    std::vector<uint32_t> triangleMaterials;
    std::vector<float> texcoords;           // 6 per triangle
    std::vector<float> normals;             // 12 per triangle
    std::vector<uint8_t> materials;         // 368 B records
    std::vector<uint8_t> lights;            // 224 B records, at least one
    std::vector<float> emissive;            // 4 per triangle
    std::vector<PackedTexture> textures;
    uint32_t lightCount = 0;
    bool opaque = true;
    bool geometryReady = false;
    std::vector<PackedInstancer> instancers;  // empty: a single-level scene
    std::vector<float> materialEmission;      // per material: emission weight x luminance (the CDF's power)

    uint32_t vertexCount() const { return static_cast<uint32_t>(vertices.size() / 4); }
    uint32_t triangleCount() const { return static_cast<uint32_t>(triangleMaterials.size()); }
    uint32_t materialCount() const { return static_cast<uint32_t>(materials.size() / HDCX_GPU_MATERIAL_BYTES); }
};

// Packs a snapshot with the reference's ordering and index rules. Meshes
// named by `instancers` are flattened first, as the reference's Hydra mesh
// adapter flattens an instanced mesh (flattenInstancer), and the packed
// scene records the instancers for a two-level BVH.
PackedSceneData packScene(const hdcx_scene_desc& scene, const hdcx_instancer_desc* instancers = nullptr,
                          uint64_t instancerCount = 0);

// World-space positions of every instance of `ins` (xyzw, instance-major):
// the flattened vertices, from its current object-space points.
std::vector<float> instancerWorldPoints(const PackedInstancer& ins);

// Recomputes the emissive-triangle CDF of `data` from its vertices (after
// an instancer's points moved).
void recomputeEmissive(PackedSceneData& data);

// Copies a caller-packed view into owned storage (validating counts).
PackedSceneData copyPackedView(const hdcx_packed_scene& view);

// Fills an hdcx_packed_scene view over `data` (texture views go to `textureViews`).
void makePackedView(const PackedSceneData& data, std::vector<hdcx_packed_texture>& textureViews,
                    hdcx_packed_scene* view);

// sRGB byte -> linear table the device sampler uses (binary64, rounded once).
void srgbTable(float table[256]);

}  // namespace hdcx
