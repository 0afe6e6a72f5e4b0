// oracle_api.cpp - C interface of the CPU oracle. TEST INFRASTRUCTURE ONLY
// (see oracle_glsl.h). Mirrors the state handling of VulkanPathTracer::Impl
// (vulkan_path_tracer.cpp:3130-3160 output buffer, :3230-3306 Trace).
#include "hdcx_oracle.h"

#include "oracle_internal.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <functional>
#include <memory>
#include <thread>
#include <vector>

struct oracle_tracer {
    oracle::PackedScene scene;
    oracle::Bvh bvh;
    std::vector<hdcx_packed_texture> textureViews;
    std::vector<float> rgba;     // running mean of the current output size
    std::vector<double> xyz;     // FP64 XYZ sums
    uint32_t width = 0, height = 0;
    bool fallbackAxisInitialized = false;
    bool fallbackZUp = false;
};

namespace {

void ParallelRows(uint32_t y0, uint32_t y1, int threads, const std::function<void(uint32_t)>& body)
{
    unsigned n = threads > 0 ? static_cast<unsigned>(threads) : std::max(1u, std::thread::hardware_concurrency());
    n = std::min<unsigned>(n, std::max<uint32_t>(1u, y1 - y0));
    std::atomic<uint32_t> next{y0};
    auto worker = [&]() {
        for (;;) {
            const uint32_t y = next.fetch_add(1);
            if (y >= y1) break;
            body(y);
        }
    };
    std::vector<std::thread> pool;
    for (unsigned i = 1; i < n; ++i) pool.emplace_back(worker);
    worker();
    for (auto& t : pool) t.join();
}

oracle::Camera ToCamera(const hdcx_camera& c)
{
    oracle::Camera cam;
    cam.origin = oracle::V3(c.origin[0], c.origin[1], c.origin[2]);
    cam.lowerLeft = oracle::V3(c.lower_left[0], c.lower_left[1], c.lower_left[2]);
    cam.horizontal = oracle::V3(c.horizontal[0], c.horizontal[1], c.horizontal[2]);
    cam.vertical = oracle::V3(c.vertical[0], c.vertical[1], c.vertical[2]);
    return cam;
}

}  // namespace

extern "C" {

oracle_tracer* oracle_create(void) { return new oracle_tracer(); }

void oracle_destroy(oracle_tracer* tracer) { delete tracer; }

int oracle_set_scene(oracle_tracer* tracer, const hdcx_scene_desc* scene)
{
    if (!tracer) return 0;
    tracer->scene = oracle::PackedScene{};
    tracer->bvh = oracle::Bvh{};
    tracer->textureViews.clear();
    if (!scene) return 1;
    tracer->scene = oracle::PackScene(*scene);
    if (tracer->scene.geometryReady) tracer->bvh = oracle::BuildBvh(tracer->scene);
    for (const auto& t : tracer->scene.textures) {
        hdcx_packed_texture v{};
        v.width = t.width;
        v.height = t.height;
        v.format = t.format;
        v.texels = t.format == HDCX_TEXEL_RGBA32F ? static_cast<const void*>(t.floats.data())
                                                 : static_cast<const void*>(t.bytes.data());
        tracer->textureViews.push_back(v);
    }
    return 1;
}

int oracle_has_geometry(const oracle_tracer* tracer) { return tracer && tracer->scene.geometryReady ? 1 : 0; }

int oracle_packed_view(const oracle_tracer* tracer, hdcx_packed_scene* view)
{
    if (!tracer || !view) return 0;
    const auto& s = tracer->scene;
    std::memset(view, 0, sizeof(*view));
    view->vertex_count = static_cast<uint32_t>(s.vertices.size());
    view->triangle_count = static_cast<uint32_t>(s.triangleMaterials.size());
    view->material_count = static_cast<uint32_t>(s.materials.size());
    view->light_count = s.lightCount;
    view->texture_count = static_cast<uint32_t>(s.textures.size());
    view->opaque = s.opaque ? 1u : 0u;
    view->vertices = reinterpret_cast<const float*>(s.vertices.data());
    view->indices = s.indices.data();
    view->triangle_materials = s.triangleMaterials.data();
    view->texcoords = reinterpret_cast<const float*>(s.texcoords.data());
    view->normals = reinterpret_cast<const float*>(s.normals.data());
    view->materials = s.materials.data();
    view->lights = s.lights.data();
    view->emissive = reinterpret_cast<const float*>(s.emissive.data());
    view->textures = tracer->textureViews.data();
    return 1;
}

int oracle_render(oracle_tracer* tracer, const hdcx_camera* camera, uint32_t width, uint32_t height,
                  uint32_t sample_index, uint32_t max_bounces, uint32_t sample_count, uint32_t x0, uint32_t y0,
                  uint32_t x1, uint32_t y1, int32_t threads, float* rgba_out, double* xyz_out, uint64_t* counters)
{
    if (!tracer || !camera) return 0;
    if (!tracer->scene.geometryReady || width == 0 || height == 0) return 0;
    // EnsureOutput: a new size zero-fills the accumulation (:3130-3160).
    if (tracer->width != width || tracer->height != height) {
        tracer->width = width;
        tracer->height = height;
        tracer->rgba.assign(size_t(width) * height * 4u, 0.0f);
        tracer->xyz.assign(size_t(width) * height * 3u, 0.0);
    }
    if (sample_index == 0) std::fill(tracer->xyz.begin(), tracer->xyz.end(), 0.0);
    // Fallback up axis from the first render of this tracer (:3237-3241).
    if (!tracer->fallbackAxisInitialized) {
        tracer->fallbackZUp = std::fabs(camera->vertical[2]) > std::fabs(camera->vertical[1]);
        tracer->fallbackAxisInitialized = true;
    }
    if (x1 == 0 && y1 == 0) {
        x1 = width;
        y1 = height;
    }
    x1 = std::min(x1, width);
    y1 = std::min(y1, height);
    oracle::FrameParams frame{width, height, sample_index, sample_count, max_bounces, tracer->fallbackZUp};
    const oracle::Camera cam = ToCamera(*camera);
    std::atomic<uint64_t> ext{0}, sh{0}, ss{0};
    ParallelRows(y0, y1, threads, [&](uint32_t y) {
        oracle::Counters local;
        for (uint32_t x = x0; x < x1; ++x) {
            const size_t p = size_t(y) * width + x;
            oracle::RenderPixel(tracer->scene, tracer->bvh, cam, frame, x, y, &tracer->rgba[p * 4u],
                                &tracer->xyz[p * 3u], &local);
        }
        ext += local.extensionRays;
        sh += local.shadowRays;
        ss += local.subsurfaceRays;
    });
    if (rgba_out) std::memcpy(rgba_out, tracer->rgba.data(), tracer->rgba.size() * sizeof(float));
    if (xyz_out) std::memcpy(xyz_out, tracer->xyz.data(), tracer->xyz.size() * sizeof(double));
    if (counters) {
        counters[0] = ext.load();
        counters[1] = sh.load();
        counters[2] = ss.load();
    }
    return 1;
}

int oracle_trace_primary(oracle_tracer* tracer, const hdcx_camera* camera, uint32_t width, uint32_t height,
                         uint32_t sample_number, int32_t threads, uint32_t* primitive_out, float* distance_out)
{
    if (!tracer || !camera || !tracer->scene.geometryReady) return 0;
    const oracle::Camera cam = ToCamera(*camera);
    const bool opaque = tracer->scene.opaque;
    ParallelRows(0, height, threads, [&](uint32_t y) {
        for (uint32_t x = 0; x < width; ++x) {
            // Camera ray of main() (vulkan_path_tracer.cpp:1202-1213).
            const uint32_t index = y * width + x;
            uint32_t rng = oracle::hashState(index ^ (sample_number * 0x9e3779b9u) ^ 0xa511e9b3u);
            rng = oracle::hashState(rng);
            const float jx = oracle::uintToFloat(rng) * (1.0f / 4294967296.0f);
            rng = oracle::hashState(rng);
            const float jy = oracle::uintToFloat(rng) * (1.0f / 4294967296.0f);
            const float u = (oracle::uintToFloat(x) + jx) / oracle::uintToFloat(width);
            const float v = (oracle::uintToFloat(y) + jy) / oracle::uintToFloat(height);
            const oracle::vec3 dir =
                oracle::normalize(cam.lowerLeft + u * cam.horizontal + v * cam.vertical - cam.origin);
            oracle::Hit hit;
            const bool found = oracle::TraceClosest(tracer->scene, tracer->bvh, cam.origin, dir, 0.001f, 10000.0f,
                                                    opaque ? oracle::AcceptMode::Opaque : oracle::AcceptMode::Stochastic,
                                                    rng, &hit);
            primitive_out[index] = found ? hit.primitive : 0xffffffffu;
            if (distance_out) distance_out[index] = found ? hit.t : 0.0f;
        }
    });
    return 1;
}

}  // extern "C"
