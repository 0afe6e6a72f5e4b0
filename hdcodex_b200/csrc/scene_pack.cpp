// scene_pack.cpp - packs a SceneSnapshot into the integrator's device layout.
//
// Host-side restatement of Impl::BuildScene (src/gpu/vulkan_path_tracer.cpp:
// 2604-2993) and its helpers: texture and UDIM descriptor numbering
// (:2622-2658), average texture luminance (:1968-1996), the lat-long dome
// importance map (:1998-2066, R conditional CDF, G marginal CDF, B pdf),
// light records with their selection power (:2704-2766), the default and
// display-colour materials (:2768-2907), mesh flattening with per-triangle
// subsets (:2908-2940) and the FP64 emissive-triangle CDF (:2944-2993).
// GpuMaterial / GpuLight are written as the reference's 23 / 14 vec4 records.
#include "scene_pack.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <map>
#include <stdexcept>

namespace hdcx {
namespace {

constexpr uint32_t kMaxTextures = HDCX_MAX_TEXTURES;
constexpr uint32_t kMissing = HDCX_MISSING_TEXTURE;

std::string text(const char* s) { return s ? std::string(s) : std::string(); }

struct Vec4Writer {
    std::vector<uint8_t>& out;
    void f(float x, float y, float z, float w)
    {
        const float v[4] = {x, y, z, w};
        const auto* b = reinterpret_cast<const uint8_t*>(v);
        out.insert(out.end(), b, b + 16);
    }
    void u(uint32_t x, uint32_t y, uint32_t z, uint32_t w)
    {
        const uint32_t v[4] = {x, y, z, w};
        const auto* b = reinterpret_cast<const uint8_t*>(v);
        out.insert(out.end(), b, b + 16);
    }
};

float srgbToLinearF(float value)
{
    return value <= 0.04045F ? value / 12.92F : std::pow((value + 0.055F) / 1.055F, 2.4F);
}

uint64_t texelCount(const hdcx_texture_desc& t) { return uint64_t(t.width) * t.height * 4u; }

// VersionedScene::UpsertTexture admits only ids with a full pixel array
// (versioned_scene.h:355-364); other entries never reach BuildScene.
bool admitted(const hdcx_texture_desc& t)
{
    if (!t.id || !t.id[0] || t.width == 0 || t.height == 0) return false;
    const uint64_t n = texelCount(t);
    return (t.rgba && t.rgba_count == n) || (t.rgba_float && t.rgba_float_count == n);
}

bool isFloat(const hdcx_texture_desc& t) { return t.rgba_float && t.rgba_float_count == texelCount(t); }

PackedTexture upload(const hdcx_texture_desc& t)
{
    PackedTexture p;
    p.width = t.width;
    p.height = t.height;
    const size_t n = static_cast<size_t>(texelCount(t));
    if (isFloat(t)) {
        p.format = HDCX_TEXEL_RGBA32F;
        p.floats.assign(t.rgba_float, t.rgba_float + n);
    } else {
        p.format = t.srgb ? HDCX_TEXEL_RGBA8_SRGB : HDCX_TEXEL_RGBA8_UNORM;
        p.bytes.assign(t.rgba, t.rgba + n);
    }
    return p;
}

float linearChannel(const hdcx_texture_desc& t, bool useFloat, size_t i)
{
    float v = useFloat ? t.rgba_float[i] : static_cast<float>(t.rgba[i]) / 255.0F;
    if (!useFloat && t.srgb) v = srgbToLinearF(v);
    return std::isfinite(v) ? std::max(v, 0.0F) : 0.0F;
}

float averageLuminance(const hdcx_texture_desc& t)
{
    if (t.width == 0 || t.height == 0) return 0.0F;
    const size_t pixels = size_t(t.width) * t.height;
    const bool useFloat = t.rgba_float && t.rgba_float_count > 0;
    if ((useFloat && t.rgba_float_count < pixels * 4u) || (!useFloat && (!t.rgba || t.rgba_count < pixels * 4u))) {
        return 0.0F;
    }
    double total = 0.0;
    for (size_t px = 0; px < pixels; ++px) {
        const float r = linearChannel(t, useFloat, px * 4u), g = linearChannel(t, useFloat, px * 4u + 1u),
                    b = linearChannel(t, useFloat, px * 4u + 2u);
        total += 0.2126 * r + 0.7152 * g + 0.0722 * b;
    }
    return static_cast<float>(total / static_cast<double>(pixels));
}

bool latLongImportance(const hdcx_texture_desc& t, PackedTexture* out)
{
    if (t.width == 0 || t.height == 0) return false;
    const size_t pixels = size_t(t.width) * t.height;
    const bool useFloat = t.rgba_float && t.rgba_float_count > 0;
    std::vector<float> lum(pixels);
    std::vector<double> weight(pixels), rowWeight(t.height, 0.0);
    const double pi = 3.14159265358979323846;
    const double deltaPhi = 2.0 * pi / static_cast<double>(t.width);
    double total = 0.0;
    for (uint32_t y = 0; y < t.height; ++y) {
        const double v0 = static_cast<double>(y) / t.height, v1 = static_cast<double>(y + 1u) / t.height;
        const double solidAngle = deltaPhi * std::abs(std::cos(pi * (1.0 - v1)) - std::cos(pi * (1.0 - v0)));
        for (uint32_t x = 0; x < t.width; ++x) {
            const size_t px = size_t(y) * t.width + x;
            const float r = linearChannel(t, useFloat, px * 4u), g = linearChannel(t, useFloat, px * 4u + 1u),
                        b = linearChannel(t, useFloat, px * 4u + 2u);
            const float value = 0.2126F * r + 0.7152F * g + 0.0722F * b;
            lum[px] = value;
            weight[px] = static_cast<double>(value) * solidAngle;
            rowWeight[y] += weight[px];
            total += weight[px];
        }
    }
    if (!(total > 0.0) || !std::isfinite(total)) return false;
    out->width = t.width;
    out->height = t.height;
    out->format = HDCX_TEXEL_RGBA32F;
    out->floats.assign(pixels * 4u, 0.0F);
    double marginal = 0.0;
    for (uint32_t y = 0; y < t.height; ++y) {
        marginal += rowWeight[y] / total;
        double conditional = 0.0;
        for (uint32_t x = 0; x < t.width; ++x) {
            const size_t px = size_t(y) * t.width + x;
            conditional += rowWeight[y] > 0.0 ? weight[px] / rowWeight[y] : 1.0 / static_cast<double>(t.width);
            float* o = &out->floats[px * 4u];
            o[0] = static_cast<float>(x + 1u == t.width ? 1.0 : conditional);
            o[1] = static_cast<float>(y + 1u == t.height ? 1.0 : marginal);
            o[2] = static_cast<float>(static_cast<double>(lum[px]) / total);
            o[3] = 1.0F;
        }
    }
    return true;
}

void writeDefaultMaterial(std::vector<uint8_t>& out, const std::array<float, 3>& c)
{
    // vulkan_path_tracer.cpp:2768-2800
    Vec4Writer w{out};
    w.f(c[0], c[1], c[2], 0.0F);
    w.f(0.0F, 0.0F, 0.0F, 0.5F);
    w.f(0.0F, 1.0F, 1.5F, 0.0F);
    w.f(1.0F, 1.0F, 1.0F, 0.0F);
    w.f(0.0F, 1.0F, 0.0F, 0.0F);
    w.f(c[0], c[1], c[2], 0.0F);
    w.f(1.0F, 0.2F, 0.1F, 0.0F);
    w.f(1.0F, 1.0F, 1.0F, 1.0F);
    w.f(0.0F, 0.1F, 1.5F, 0.0F);
    w.f(1.0F, 1.0F, 1.0F, 0.0F);
    w.f(0.0F, 0.0F, 0.0F, 20.0F);
    w.f(0.0F, 0.0F, 0.0F, 0.0F);
    w.f(1.0F, 1.0F, 1.0F, 0.0F);
    w.f(0.0F, 0.0F, 1.0F, 0.0F);
    w.f(1.0F, 1.0F, 1.0F, 0.0F);
    w.f(1.0F, 1.0F, 1.0F, -1.0F);
    w.f(0.0F, 0.0F, 0.0F, 0.0F);
    for (int i = 0; i < 6; ++i) w.u(kMissing, kMissing, kMissing, kMissing);
}

// A flattened instanced mesh: owned arrays behind an hdcx_mesh_desc.
struct FlatMesh {
    std::vector<float> positions, texcoords, normals;
    std::vector<uint32_t> indices;
    std::vector<const char*> triangleMaterialIds;
    hdcx_mesh_desc desc{};
};

// Row-vector affine transform of a point in binary64 (mesh.cpp:964-969).
void transformPoint(const double* m, double x, double y, double z, double out[3])
{
    for (int j = 0; j < 3; ++j) out[j] = ((x * m[j] + y * m[4 + j]) + z * m[8 + j]) + m[12 + j];
}

// inverse(A) of the upper 3x3 (rows A[i] = m[4i..4i+2]) by cofactors.
void inverse3(const double* m, double inv[9])
{
    const double a00 = m[0], a01 = m[1], a02 = m[2];
    const double a10 = m[4], a11 = m[5], a12 = m[6];
    const double a20 = m[8], a21 = m[9], a22 = m[10];
    const double c00 = a11 * a22 - a12 * a21, c01 = a12 * a20 - a10 * a22, c02 = a10 * a21 - a11 * a20;
    const double det = (a00 * c00 + a01 * c01) + a02 * c02;
    inv[0] = c00 / det;
    inv[1] = (a02 * a21 - a01 * a22) / det;
    inv[2] = (a01 * a12 - a02 * a11) / det;
    inv[3] = c01 / det;
    inv[4] = (a00 * a22 - a02 * a20) / det;
    inv[5] = (a02 * a10 - a00 * a12) / det;
    inv[6] = c02 / det;
    inv[7] = (a01 * a20 - a00 * a21) / det;
    inv[8] = (a00 * a11 - a01 * a10) / det;
}

void checkAffine(const double* m)
{
    if (m[3] != 0.0 || m[7] != 0.0 || m[11] != 0.0 || m[15] != 1.0)
        throw std::invalid_argument("instancer: transforms must be affine (column 3 = 0, 0, 0, 1)");
}

// mesh.cpp:955-1004 for one instanced mesh.
void flattenInstancer(const hdcx_mesh_desc& m, const double* transforms, uint64_t count, FlatMesh& f)
{
    const uint64_t points = m.position_count / 3u;
    const uint64_t triangles = m.index_count / 3u;
    const uint64_t cornerNormals = m.normals ? m.normal_count / 3u : 0u;
    for (uint64_t inst = 0; inst < count; ++inst) {
        const double* T = transforms + 16u * inst;
        checkAffine(T);
        double inv[9];
        inverse3(T, inv);
        const uint32_t vertexBase = static_cast<uint32_t>(f.positions.size() / 3u);
        for (uint64_t p = 0; p < points; ++p) {
            double w[3];
            transformPoint(T, m.positions[3 * p], m.positions[3 * p + 1], m.positions[3 * p + 2], w);
            for (double c : w) f.positions.push_back(static_cast<float>(c));
        }
        for (uint64_t t = 0; t < triangles; ++t) {
            bool valid = true;
            for (int c = 0; c < 3; ++c) valid = valid && m.indices[3 * t + c] < points;
            if (!valid) continue;
            f.triangleMaterialIds.push_back(m.triangle_material_ids && t < m.triangle_material_id_count
                                                ? m.triangle_material_ids[t]
                                                : m.material_id);
            for (int c = 0; c < 3; ++c) {
                f.indices.push_back(vertexBase + m.indices[3 * t + c]);
                const uint64_t corner = 3 * t + c, uv = corner * 2u;
                const bool hasUv = m.texcoords && uv + 1u < m.texcoord_count;
                f.texcoords.push_back(hasUv ? m.texcoords[uv] : 0.0F);
                f.texcoords.push_back(hasUv ? m.texcoords[uv + 1] : 0.0F);
                double n[3] = {0.0, 0.0, 0.0};
                if (corner < cornerNormals) {
                    const double nx = m.normals[3 * corner], ny = m.normals[3 * corner + 1], nz = m.normals[3 * corner + 2];
                    for (int j = 0; j < 3; ++j) n[j] = (nx * inv[3 * j] + ny * inv[3 * j + 1]) + nz * inv[3 * j + 2];
                    const double length = std::sqrt((n[0] * n[0] + n[1] * n[1]) + n[2] * n[2]);
                    const double d = length > 1e-10 ? length : 1e-10;
                    for (double& x : n) x = length <= 1e-12 ? 0.0 : x / d;
                }
                for (double x : n) f.normals.push_back(static_cast<float>(x));
            }
        }
    }
    f.desc = m;
    f.desc.positions = f.positions.data();
    f.desc.position_count = f.positions.size();
    f.desc.indices = f.indices.data();
    f.desc.index_count = f.indices.size();
    f.desc.texcoords = f.texcoords.data();
    f.desc.texcoord_count = f.texcoords.size();
    f.desc.normals = f.normals.data();
    f.desc.normal_count = f.normals.size();
    f.desc.triangle_material_ids = f.triangleMaterialIds.data();
    f.desc.triangle_material_id_count = f.triangleMaterialIds.size();
}

// The emissive-triangle CDF (vulkan_path_tracer.cpp:2944-2993): binary64
// areas and weights, entry (cdf, probability / area, area, 0) per triangle.
void computeEmissive(PackedSceneData& out)
{
    const size_t n = out.triangleMaterials.size();
    out.emissive.assign(n * 4u, 0.0F);
    std::vector<double> weight(n, 0.0);
    std::vector<float> area(n, 0.0F);
    double total = 0.0;
    for (size_t p = 0; p < n; ++p) {
        const float* a = &out.vertices[size_t(out.indices[3 * p]) * 4u];
        const float* b = &out.vertices[size_t(out.indices[3 * p + 1]) * 4u];
        const float* c = &out.vertices[size_t(out.indices[3 * p + 2]) * 4u];
        const double e1x = static_cast<double>(b[0]) - a[0], e1y = static_cast<double>(b[1]) - a[1],
                     e1z = static_cast<double>(b[2]) - a[2];
        const double e2x = static_cast<double>(c[0]) - a[0], e2y = static_cast<double>(c[1]) - a[1],
                     e2z = static_cast<double>(c[2]) - a[2];
        const double cx = e1y * e2z - e1z * e2y, cy = e1z * e2x - e1x * e2z, cz = e1x * e2y - e1y * e2x;
        const float ar = static_cast<float>(0.5 * std::sqrt(cx * cx + cy * cy + cz * cz));
        area[p] = std::isfinite(ar) ? ar : 0.0F;
        const uint32_t mat = out.triangleMaterials[p];
        const float power = mat < out.materialEmission.size() ? out.materialEmission[mat] : 0.0F;
        const double w = static_cast<double>(area[p]) * static_cast<double>(power);
        if (w > 0.0 && std::isfinite(w)) {
            weight[p] = w;
            total += w;
        }
    }
    if (total > 0.0 && std::isfinite(total)) {
        double cdf = 0.0;
        for (size_t p = 0; p < n; ++p) {
            const double probability = weight[p] / total;
            cdf += probability;
            float* e = &out.emissive[p * 4u];
            e[0] = static_cast<float>(p + 1u == n ? 1.0 : cdf);
            e[1] = area[p] > 0.0F ? static_cast<float>(probability) / area[p] : 0.0F;
            e[2] = area[p];
            e[3] = 0.0F;
        }
    }
}

}  // namespace

std::vector<float> instancerWorldPoints(const PackedInstancer& ins)
{
    std::vector<float> out;
    out.reserve(size_t(ins.instanceCount) * ins.pointCount() * 4u);
    for (uint32_t inst = 0; inst < ins.instanceCount; ++inst) {
        const double* T = ins.transforms.data() + 16u * inst;
        for (uint32_t p = 0; p < ins.pointCount(); ++p) {
            double w[3];
            transformPoint(T, ins.points[4 * p], ins.points[4 * p + 1], ins.points[4 * p + 2], w);
            out.insert(out.end(), {static_cast<float>(w[0]), static_cast<float>(w[1]), static_cast<float>(w[2]), 1.0F});
        }
    }
    return out;
}

void recomputeEmissive(PackedSceneData& data) { computeEmissive(data); }

void srgbTable(float table[256])
{
    for (int i = 0; i < 256; ++i) {
        const double c = static_cast<double>(i) / 255.0;
        table[i] = static_cast<float>(c <= 0.04045 ? c / 12.92 : std::pow((c + 0.055) / 1.055, 2.4));
    }
}

PackedSceneData packScene(const hdcx_scene_desc& scene, const hdcx_instancer_desc* instancers, uint64_t instancerCount)
{
    PackedSceneData out;
    // Instanced meshes are flattened first; the rest of the packing sees the
    // flattened snapshot.
    hdcx_scene_desc snap = scene;
    std::vector<hdcx_mesh_desc> meshes;
    std::vector<FlatMesh> flat(instancerCount);
    std::vector<int> instancerOfMesh(scene.mesh_count, -1);
    if (instancerCount > 0) {
        if (!instancers) throw std::invalid_argument("instancer array is null");
        meshes.assign(scene.meshes, scene.meshes + scene.mesh_count);
        for (uint64_t k = 0; k < instancerCount; ++k) {
            const hdcx_instancer_desc& ins = instancers[k];
            if (ins.mesh_index >= scene.mesh_count) throw std::invalid_argument("instancer: mesh_index out of range");
            if (instancerOfMesh[ins.mesh_index] >= 0)
                throw std::invalid_argument("instancer: a mesh is instanced by more than one instancer");
            if (ins.instance_count > 0 && !ins.transforms) throw std::invalid_argument("instancer: transforms are null");
            instancerOfMesh[ins.mesh_index] = static_cast<int>(k);
            flattenInstancer(scene.meshes[ins.mesh_index], ins.transforms, ins.instance_count, flat[k]);
            meshes[ins.mesh_index] = flat[k].desc;
        }
        snap.meshes = meshes.data();
    }
    out.opaque = true;
    for (uint64_t i = 0; i < snap.material_count; ++i) {
        const hdcx_material_desc& m = snap.materials[i];
        if (!(m.opacity >= 0.999F && text(m.opacity_texture).empty())) out.opaque = false;
    }

    // Texture descriptors: plain textures in snapshot order, then UDIM sets
    // in set-id order with their tiles sorted by tile number.
    std::map<std::string, uint32_t, std::less<>> index;
    std::map<std::string, const hdcx_texture_desc*, std::less<>> plain;
    std::map<std::string, std::vector<const hdcx_texture_desc*>, std::less<>> udim;
    for (uint64_t i = 0; i < snap.texture_count; ++i) {
        const hdcx_texture_desc& t = snap.textures[i];
        if (!admitted(t)) continue;
        if (!text(t.udim_set_id).empty() && t.udim_tile != 0u) {
            udim[text(t.udim_set_id)].push_back(&t);
            continue;
        }
        if (out.textures.size() >= kMaxTextures) continue;
        plain[text(t.id)] = &t;
        index[text(t.id)] = static_cast<uint32_t>(out.textures.size());
        out.textures.push_back(upload(t));
    }
    for (auto& [setId, tiles] : udim) {
        std::stable_sort(tiles.begin(), tiles.end(),
                         [](const hdcx_texture_desc* a, const hdcx_texture_desc* b) { return a->udim_tile < b->udim_tile; });
        const uint32_t base = static_cast<uint32_t>(out.textures.size());
        uint32_t present = 0u;
        for (const hdcx_texture_desc* tile : tiles) {
            if (out.textures.size() >= kMaxTextures) break;
            if (tile->udim_tile < 1001u || tile->udim_tile > 1023u) continue;
            present |= 1u << (tile->udim_tile - 1001u);
            out.textures.push_back(upload(*tile));
        }
        if (present != 0u) index[setId] = HDCX_UDIM_TEXTURE_FLAG | ((present & HDCX_UDIM_TILE_MASK) << 8u) | base;
    }
    auto lookup = [&](const char* id) {
        const auto it = index.find(text(id));
        return it == index.end() ? kMissing : it->second;
    };
    std::map<std::string, float, std::less<>> luminanceCache;
    auto luminance = [&](const std::string& id) {
        if (auto c = luminanceCache.find(id); c != luminanceCache.end()) return c->second;
        double total = 0.0;
        size_t count = 0;
        if (auto p = plain.find(id); p != plain.end()) {
            total = averageLuminance(*p->second);
            count = 1;
        } else if (auto u = udim.find(id); u != udim.end()) {
            for (const hdcx_texture_desc* tile : u->second) {
                total += averageLuminance(*tile);
                ++count;
            }
        }
        const float r = count ? static_cast<float>(total / static_cast<double>(count)) : 0.0F;
        luminanceCache.emplace(id, r);
        return r;
    };
    std::map<std::string, uint32_t, std::less<>> importanceOf;
    auto importance = [&](const hdcx_light_desc& l) {
        if (l.type != HDCX_LIGHT_DOME || (l.texture_format != HDCX_DOME_AUTOMATIC && l.texture_format != HDCX_DOME_LATLONG) ||
            lookup(l.texture) == kMissing) {
            return kMissing;
        }
        const std::string key = text(l.texture);
        if (auto c = importanceOf.find(key); c != importanceOf.end()) return c->second;
        const auto src = plain.find(key);
        if (src == plain.end() || out.textures.size() >= kMaxTextures) return kMissing;
        PackedTexture map;
        if (!latLongImportance(*src->second, &map)) return kMissing;
        const uint32_t id = static_cast<uint32_t>(out.textures.size());
        out.textures.push_back(std::move(map));
        importanceOf.emplace(key, id);
        return id;
    };

    // Lights.
    Vec4Writer lw{out.lights};
    for (uint64_t i = 0; i < snap.light_count; ++i) {
        const hdcx_light_desc& l = snap.lights[i];
        if (!l.visible || out.lightCount >= HDCX_MAX_LIGHTS) continue;
        float scale = l.intensity * std::exp2(l.exposure);
        if (l.type != HDCX_LIGHT_DOME && l.type != HDCX_LIGHT_DISTANT && l.normalize) scale /= std::max(l.area, 1e-8F);
        const float cr = l.color[0] * l.temperature_color[0], cg = l.color[1] * l.temperature_color[1],
                    cb = l.color[2] * l.temperature_color[2];
        float emitted = 0.2126F * std::max(cr, 0.0F) + 0.7152F * std::max(cg, 0.0F) + 0.0722F * std::max(cb, 0.0F);
        if (!text(l.texture).empty() && (l.type == HDCX_LIGHT_DOME || l.type == HDCX_LIGHT_RECT)) {
            emitted *= luminance(text(l.texture));
        }
        float measure = 1.0F;
        if (l.type == HDCX_LIGHT_DOME) measure = 12.5663706144F;
        else if (l.type != HDCX_LIGHT_DISTANT) measure = std::max(l.area, 0.0F);
        float power = std::max(emitted * std::max(scale, 0.0F) * measure, 0.0F);
        if (!std::isfinite(power)) power = 0.0F;
        const uint32_t texIndex = lookup(l.texture);
        const uint32_t importanceIndex = importance(l);
        lw.f(cr, cg, cb, scale);
        lw.f(l.diffuse, l.specular, static_cast<float>(l.type), std::max(l.area, 0.0F));
        lw.f(l.position[0], l.position[1], l.position[2], 0.0F);
        lw.f(l.axis_u[0], l.axis_u[1], l.axis_u[2], 0.0F);
        lw.f(l.axis_v[0], l.axis_v[1], l.axis_v[2], 0.0F);
        lw.f(l.basis_x[0], l.basis_x[1], l.basis_x[2], 0.0F);
        lw.f(l.basis_y[0], l.basis_y[1], l.basis_y[2], 0.0F);
        lw.f(l.basis_z[0], l.basis_z[1], l.basis_z[2], 0.0F);
        lw.f(l.shaping_focus, l.shaping_cone_angle, l.shaping_cone_softness, 0.0F);
        lw.f(l.shaping_focus_tint[0], l.shaping_focus_tint[1], l.shaping_focus_tint[2], 0.0F);
        lw.f(l.shadow_enable ? 1.0F : 0.0F, l.shadow_distance, l.shadow_falloff, l.shadow_falloff_gamma);
        lw.f(l.shadow_color[0], l.shadow_color[1], l.shadow_color[2], 0.0F);
        lw.f(l.radius, l.length, l.angle, power);
        lw.u(texIndex, l.texture_format, l.type, importanceIndex);
        out.lightCount++;
    }
    if (out.lightCount == 0) {
        // An all-zero record with shadows on and no distance limit
        // (vulkan_path_tracer.cpp:2763-2766).
        for (int i = 0; i < 10; ++i) lw.f(0.0F, 0.0F, 0.0F, 0.0F);
        lw.f(1.0F, -1.0F, -1.0F, 1.0F);
        lw.f(0.0F, 0.0F, 0.0F, 0.0F);
        lw.f(0.0F, 0.0F, 0.0F, 0.0F);
        lw.u(0u, 0u, 0u, 0u);
    }

    // Materials: index 0 is the default, then the snapshot's materials.
    std::vector<float> emissionPower;
    writeDefaultMaterial(out.materials, {0.8F, 0.8F, 0.8F});
    emissionPower.push_back(0.0F);
    std::map<std::string, uint32_t, std::less<>> materialIndex;
    Vec4Writer mw{out.materials};
    for (uint64_t i = 0; i < snap.material_count; ++i) {
        const hdcx_material_desc& m = snap.materials[i];
        materialIndex[text(m.id)] = static_cast<uint32_t>(emissionPower.size());
        mw.f(m.base_color[0], m.base_color[1], m.base_color[2], m.metalness);
        mw.f(m.emission[0], m.emission[1], m.emission[2], m.roughness);
        mw.f(m.transmission, m.opacity, m.index_of_refraction, m.emission_weight);
        mw.f(m.transmission_color[0], m.transmission_color[1], m.transmission_color[2], m.thin_walled ? 1.0F : 0.0F);
        mw.f(m.subsurface, m.subsurface_scale, m.subsurface_scatter_anisotropy, m.normal_texture_scale);
        mw.f(m.subsurface_color[0], m.subsurface_color[1], m.subsurface_color[2], m.roughness_v);
        mw.f(m.subsurface_radius[0], m.subsurface_radius[1], m.subsurface_radius[2], m.coat_roughness_v);
        mw.f(m.specular_weight, m.specular_color[0], m.specular_color[1], m.specular_color[2]);
        mw.f(m.coat, m.coat_roughness, m.coat_index_of_refraction, m.normal_texture_flip_y ? 1.0F : 0.0F);
        mw.f(m.coat_color[0], m.coat_color[1], m.coat_color[2], m.sheen);
        mw.f(m.transmission_depth, m.transmission_scatter_anisotropy, m.transmission_dispersion_scale,
             m.transmission_dispersion_abbe_number);
        mw.f(m.transmission_scatter[0], m.transmission_scatter[1], m.transmission_scatter[2], m.sheen_roughness);
        mw.f(m.sheen_color[0], m.sheen_color[1], m.sheen_color[2], static_cast<float>(m.sheen_mode));
        mw.f(m.diffuse_roughness, static_cast<float>(m.diffuse_model), m.diffuse_weight, 0.0F);
        mw.f(m.translucent_color[0], m.translucent_color[1], m.translucent_color[2], m.translucent_weight);
        mw.f(m.base_color_texture_scale[0], m.base_color_texture_scale[1], m.base_color_texture_scale[2],
             static_cast<float>(m.base_color_texture_channel));
        mw.f(m.base_color_texture_bias[0], m.base_color_texture_bias[1], m.base_color_texture_bias[2], 0.0F);
        mw.u(lookup(m.base_color_texture), lookup(m.metalness_texture), lookup(m.roughness_texture), lookup(m.emission_texture));
        mw.u(lookup(m.opacity_texture), lookup(m.normal_texture), lookup(m.transmission_texture), lookup(m.sheen_texture));
        mw.u(lookup(m.subsurface_texture), lookup(m.subsurface_color_texture), lookup(m.subsurface_radius_texture),
             lookup(m.sheen_color_texture));
        mw.u(lookup(m.specular_texture), lookup(m.specular_color_texture), lookup(m.coat_texture), lookup(m.coat_color_texture));
        mw.u(lookup(m.coat_roughness_texture), lookup(m.sheen_roughness_texture), lookup(m.diffuse_roughness_texture),
             lookup(m.diffuse_weight_texture));
        mw.u(lookup(m.translucent_weight_texture), lookup(m.translucent_color_texture), kMissing, kMissing);
        const float emissionLuminance =
            text(m.emission_texture).empty()
                ? 0.2126F * std::max(m.emission[0], 0.0F) + 0.7152F * std::max(m.emission[1], 0.0F) +
                      0.0722F * std::max(m.emission[2], 0.0F)
                : luminance(text(m.emission_texture));
        emissionPower.push_back(std::max(m.emission_weight, 0.0F) * emissionLuminance);
    }

    // Meshes, in snapshot order.
    std::map<std::array<float, 3>, uint32_t> displayColorMaterial;
    for (uint64_t mi = 0; mi < snap.mesh_count; ++mi) {
        const hdcx_mesh_desc& mesh = snap.meshes[mi];
        const uint32_t base = out.vertexCount();
        if (instancerCount > 0 && instancerOfMesh[mi] >= 0) {
            const hdcx_instancer_desc& ins = instancers[instancerOfMesh[mi]];
            const hdcx_mesh_desc& proto = scene.meshes[mi];
            PackedInstancer pi;
            pi.mesh = static_cast<uint32_t>(mi);
            const uint64_t points = proto.position_count / 3u;
            for (uint64_t p = 0; p < points; ++p)
                pi.points.insert(pi.points.end(), {proto.positions[3 * p], proto.positions[3 * p + 1], proto.positions[3 * p + 2], 1.0F});
            for (uint64_t t = 0; t + 2 < proto.index_count; t += 3) {
                if (proto.indices[t] < points && proto.indices[t + 1] < points && proto.indices[t + 2] < points)
                    pi.indices.insert(pi.indices.end(), {proto.indices[t], proto.indices[t + 1], proto.indices[t + 2]});
            }
            pi.transforms.assign(ins.transforms, ins.transforms + 16u * ins.instance_count);
            pi.instanceCount = static_cast<uint32_t>(ins.instance_count);
            pi.firstTriangle = out.triangleCount();
            pi.firstVertex = base;
            if (pi.instanceCount > 0 && !pi.indices.empty()) out.instancers.push_back(std::move(pi));
        }
        for (uint64_t i = 0; i + 2 < mesh.position_count; i += 3) {
            out.vertices.insert(out.vertices.end(), {mesh.positions[i], mesh.positions[i + 1], mesh.positions[i + 2], 1.0F});
        }
        const std::string meshMaterial = text(mesh.material_id);
        uint32_t material = 0u;
        if (auto it = materialIndex.find(meshMaterial); it != materialIndex.end()) material = it->second;
        if (meshMaterial.empty()) {
            std::array<float, 3> c{mesh.display_color[0], mesh.display_color[1], mesh.display_color[2]};
            for (float& x : c) x = std::isfinite(x) ? std::clamp(x, 0.0F, 1.0F) : 0.5F;
            if (auto it = displayColorMaterial.find(c); it != displayColorMaterial.end()) {
                material = it->second;
            } else {
                material = static_cast<uint32_t>(emissionPower.size());
                displayColorMaterial.emplace(c, material);
                writeDefaultMaterial(out.materials, c);
                emissionPower.push_back(0.0F);
            }
        }
        const uint64_t local = out.vertexCount() - base;
        for (uint64_t tri = 0; tri + 2 < mesh.index_count; tri += 3) {
            const uint32_t i0 = mesh.indices[tri], i1 = mesh.indices[tri + 1], i2 = mesh.indices[tri + 2];
            if (!(i0 < local && i1 < local && i2 < local)) continue;
            out.indices.insert(out.indices.end(), {base + i0, base + i1, base + i2});
            uint32_t triMaterial = material;
            const uint64_t t = tri / 3u;
            if (mesh.triangle_material_ids && t < mesh.triangle_material_id_count) {
                const std::string id = text(mesh.triangle_material_ids[t]);
                if (id != meshMaterial) {
                    auto it = materialIndex.find(id);
                    triMaterial = it == materialIndex.end() ? 0u : it->second;
                }
            }
            out.triangleMaterials.push_back(triMaterial);
            for (uint64_t c = 0; c < 3; ++c) {
                const uint64_t uv = (tri + c) * 2u;
                if (mesh.texcoords && uv + 1u < mesh.texcoord_count) {
                    out.texcoords.insert(out.texcoords.end(), {mesh.texcoords[uv], mesh.texcoords[uv + 1]});
                } else {
                    out.texcoords.insert(out.texcoords.end(), {0.0F, 0.0F});
                }
                const uint64_t nn = (tri + c) * 3u;
                if (mesh.normals && nn + 2u < mesh.normal_count) {
                    out.normals.insert(out.normals.end(), {mesh.normals[nn], mesh.normals[nn + 1], mesh.normals[nn + 2], 0.0F});
                } else {
                    out.normals.insert(out.normals.end(), {0.0F, 0.0F, 0.0F, 0.0F});
                }
            }
        }
    }
    if (out.vertices.empty() || out.indices.empty()) {
        out.geometryReady = false;
        return out;
    }
    out.materialEmission = emissionPower;
    computeEmissive(out);
    out.geometryReady = true;
    return out;
}

PackedSceneData copyPackedView(const hdcx_packed_scene& v)
{
    PackedSceneData d;
    if (v.material_count == 0 || !v.materials) throw std::invalid_argument("packed scene: no materials");
    if (v.light_count > HDCX_MAX_LIGHTS) throw std::invalid_argument("packed scene: more than 64 lights");
    if (v.texture_count > HDCX_MAX_TEXTURES) throw std::invalid_argument("packed scene: more than 256 textures");
    d.vertices.assign(v.vertices, v.vertices + size_t(v.vertex_count) * 4u);
    d.indices.assign(v.indices, v.indices + size_t(v.triangle_count) * 3u);
    d.triangleMaterials.assign(v.triangle_materials, v.triangle_materials + v.triangle_count);
    d.texcoords.assign(v.texcoords, v.texcoords + size_t(v.triangle_count) * 6u);
    d.normals.assign(v.normals, v.normals + size_t(v.triangle_count) * 12u);
    const auto* mb = static_cast<const uint8_t*>(v.materials);
    d.materials.assign(mb, mb + size_t(v.material_count) * HDCX_GPU_MATERIAL_BYTES);
    const auto* lb = static_cast<const uint8_t*>(v.lights);
    d.lights.assign(lb, lb + size_t(std::max(1u, v.light_count)) * HDCX_GPU_LIGHT_BYTES);
    d.emissive.assign(v.emissive, v.emissive + size_t(v.triangle_count) * 4u);
    for (uint32_t i = 0; i < v.texture_count; ++i) {
        const hdcx_packed_texture& t = v.textures[i];
        PackedTexture p;
        p.width = t.width;
        p.height = t.height;
        p.format = t.format;
        const size_t n = size_t(t.width) * t.height * 4u;
        if (t.format == HDCX_TEXEL_RGBA32F) {
            p.floats.assign(static_cast<const float*>(t.texels), static_cast<const float*>(t.texels) + n);
        } else if (t.format == HDCX_TEXEL_RGBA8_UNORM || t.format == HDCX_TEXEL_RGBA8_SRGB) {
            p.bytes.assign(static_cast<const uint8_t*>(t.texels), static_cast<const uint8_t*>(t.texels) + n);
        } else {
            throw std::invalid_argument("packed scene: unknown texel format");
        }
        d.textures.push_back(std::move(p));
    }
    for (uint32_t m : d.triangleMaterials) {
        if (m >= v.material_count) throw std::invalid_argument("packed scene: triangle material index out of range");
    }
    for (uint32_t i : d.indices) {
        if (i >= v.vertex_count) throw std::invalid_argument("packed scene: vertex index out of range");
    }
    d.lightCount = v.light_count;
    d.opaque = v.opaque != 0u;
    d.geometryReady = v.vertex_count > 0 && v.triangle_count > 0;
    return d;
}

void makePackedView(const PackedSceneData& d, std::vector<hdcx_packed_texture>& textureViews, hdcx_packed_scene* v)
{
    std::memset(v, 0, sizeof(*v));
    textureViews.clear();
    for (const PackedTexture& t : d.textures) {
        hdcx_packed_texture tv{};
        tv.width = t.width;
        tv.height = t.height;
        tv.format = t.format;
        tv.texels = t.format == HDCX_TEXEL_RGBA32F ? static_cast<const void*>(t.floats.data())
                                                   : static_cast<const void*>(t.bytes.data());
        textureViews.push_back(tv);
    }
    v->vertex_count = d.vertexCount();
    v->triangle_count = d.triangleCount();
    v->material_count = d.materialCount();
    v->light_count = d.lightCount;
    v->texture_count = static_cast<uint32_t>(d.textures.size());
    v->opaque = d.opaque ? 1u : 0u;
    v->vertices = d.vertices.data();
    v->indices = d.indices.data();
    v->triangle_materials = d.triangleMaterials.data();
    v->texcoords = d.texcoords.data();
    v->normals = d.normals.data();
    v->materials = d.materials.data();
    v->lights = d.lights.data();
    v->emissive = d.emissive.data();
    v->textures = textureViews.data();
}

}  // namespace hdcx
