// ref_harness.cpp - runs the reference integrator's own GLSL (compiled as C++
// by oracle/ref_build.py) on the CPU. TEST INFRASTRUCTURE ONLY.
//
// The harness provides what the Vulkan pipeline provides to the shader: the
// storage buffers and camera uniform of vulkan_path_tracer.cpp:37-98 (filled
// from the oracle's restatement of BuildScene), the combined image samplers,
// one invocation per pixel (gl_GlobalInvocationID), and GL_EXT_ray_query.
// Ray queries are emulated over the oracle's BVH with the oracle's watertight
// triangle test: opaque queries commit the closest hit (smallest t, ties to
// the smaller primitive); non-opaque queries report their candidates front to
// back (increasing t, then primitive index) and end at the first confirmed
// one - one of the traversal orders a driver may use.
#include "ref_glsl_compat.h"

#include <algorithm>
#include <atomic>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

#include "hdcx.h"
#include "oracle_internal.h"

namespace glsl {

thread_local uvec3 gl_GlobalInvocationID{0, 0, 0};

static const oracle::PackedScene* gScene = nullptr;
static const oracle::Bvh* gBvh = nullptr;
static bool gSceneOpaque = true;

static int wrapIndex(int i, int n)
{
    const int r = i % n;
    return r < 0 ? r + n : r;
}

static float texelCoordinate(float uv, int size)
{
    const float x = uv * static_cast<float>(size) - 0.5f;
    return std::fabs(x) < 16777216.0f ? x : 0.0f;
}

vec4 texelFetch(const sampler2D& s, const ivec2& p, int)
{
    if (!s.texels || p.x < 0 || p.y < 0 || p.x >= s.width || p.y >= s.height) return vec4(0.0f);
    const float* t = s.texels + (static_cast<size_t>(p.y) * s.width + p.x) * 4u;
    return vec4(t[0], t[1], t[2], t[3]);
}

vec4 texture(const sampler2D& s, const vec2& uv)
{
    if (!s.texels) return vec4(0.0f);
    const float x = texelCoordinate(uv.x, s.width), y = texelCoordinate(uv.y, s.height);
    const float fx = std::floor(x), fy = std::floor(y);
    const float a = x - fx, b = y - fy;
    const int i0 = wrapIndex(static_cast<int>(fx), s.width), j0 = wrapIndex(static_cast<int>(fy), s.height);
    const int i1 = wrapIndex(i0 + 1, s.width), j1 = wrapIndex(j0 + 1, s.height);
    const vec4 t00 = texelFetch(s, ivec2(i0, j0), 0), t10 = texelFetch(s, ivec2(i1, j0), 0);
    const vec4 t01 = texelFetch(s, ivec2(i0, j1), 0), t11 = texelFetch(s, ivec2(i1, j1), 0);
    const float w00 = (1.0f - a) * (1.0f - b), w10 = a * (1.0f - b), w01 = (1.0f - a) * b, w11 = a * b;
    vec4 r;
    for (int k = 0; k < 4; ++k) r[k] = w00 * t00[k] + w10 * t10[k] + w01 * t01[k] + w11 * t11[k];
    return r;
}

void rayQueryInitializeEXT(rayQueryEXT& q, const accelerationStructureEXT&, uint flags, uint, const vec3& origin,
                           float tmin, const vec3& direction, float tmax)
{
    q.origin = origin;
    q.direction = direction;
    q.tmin = tmin;
    q.tmax = tmax;
    q.flags = flags;
    q.started = false;
    q.done = false;
    q.next = 0;
    q.count = 0;
    q.overflow = false;
    q.committed = false;
}

static oracle::vec3 O3(const vec3& v) { return oracle::V3(v.x, v.y, v.z); }

bool rayQueryProceedEXT(rayQueryEXT& q)
{
    if (!q.started) {
        q.started = true;
        q.opaque = (q.flags & gl_RayFlagsOpaqueEXT) != 0u || gSceneOpaque;
        if (q.opaque) {
            oracle::Hit h;
            if (oracle::TraceClosest(*gScene, *gBvh, O3(q.origin), O3(q.direction), q.tmin, q.tmax,
                                     oracle::AcceptMode::Opaque, 0u, &h)) {
                q.committed = true;
                q.committedHit = RayCandidate{h.primitive, h.t, vec2(h.barycentrics.x, h.barycentrics.y)};
            }
            q.done = true;
            return false;
        }
        thread_local std::vector<oracle::Hit> hits;
        oracle::TraceAll(*gScene, *gBvh, O3(q.origin), O3(q.direction), q.tmin, q.tmax, &hits);
        std::sort(hits.begin(), hits.end(), [](const oracle::Hit& a, const oracle::Hit& b) {
            return a.t < b.t || (a.t == b.t && a.primitive < b.primitive);
        });
        const int cap = static_cast<int>(sizeof(q.candidates) / sizeof(q.candidates[0]));
        q.overflow = static_cast<int>(hits.size()) > cap;
        q.count = std::min(cap, static_cast<int>(hits.size()));
        for (int i = 0; i < q.count; ++i) {
            q.candidates[i] = RayCandidate{hits[i].primitive, hits[i].t, vec2(hits[i].barycentrics.x, hits[i].barycentrics.y)};
        }
    }
    if (q.done) return false;
    if (q.next < q.count) {
        q.current = q.candidates[q.next++];
        return true;
    }
    q.done = true;
    return false;
}

void rayQueryConfirmIntersectionEXT(rayQueryEXT& q)
{
    // Candidates arrive front to back, so nothing after a confirmed one is closer.
    q.committed = true;
    q.committedHit = q.current;
    q.done = true;
}

uint rayQueryGetIntersectionTypeEXT(rayQueryEXT& q, bool committed)
{
    if (committed) return q.committed ? gl_RayQueryCommittedIntersectionTriangleEXT : gl_RayQueryCommittedIntersectionNoneEXT;
    return gl_RayQueryCandidateIntersectionTriangleEXT;
}
uint rayQueryGetIntersectionPrimitiveIndexEXT(rayQueryEXT& q, bool committed)
{
    return committed ? q.committedHit.primitive : q.current.primitive;
}
vec2 rayQueryGetIntersectionBarycentricsEXT(rayQueryEXT& q, bool committed)
{
    return committed ? q.committedHit.barycentrics : q.current.barycentrics;
}
float rayQueryGetIntersectionTEXT(rayQueryEXT& q, bool committed) { return committed ? q.committedHit.t : q.current.t; }

#include "glsl_as_cpp.inc"

}  // namespace glsl

struct ref_tracer {
    oracle::PackedScene scene;
    oracle::Bvh bvh;
    std::vector<float> rgba;
    uint32_t width = 0, height = 0;
    bool fallbackAxisInitialized = false;
    bool fallbackZUp = false;
};

static std::mutex gRenderMutex;

extern "C" {

__attribute__((visibility("default"))) ref_tracer* ref_create(void) { return new ref_tracer(); }

__attribute__((visibility("default"))) void ref_destroy(ref_tracer* t) { delete t; }

__attribute__((visibility("default"))) int ref_set_scene(ref_tracer* t, const hdcx_scene_desc* desc)
{
    if (!t) return 0;
    t->scene = oracle::PackedScene{};
    t->bvh = oracle::Bvh{};
    if (!desc) return 1;
    t->scene = oracle::PackScene(*desc);
    if (t->scene.geometryReady) t->bvh = oracle::BuildBvh(t->scene);
    return 1;
}

// Render(camera, w, h, sampleIndex, maxBounces, sampleCount) over the pixel
// rectangle [x0, x1) x [y0, y1) (x1 = y1 = 0: whole image).
__attribute__((visibility("default"))) int ref_render(ref_tracer* t, const hdcx_camera* c, uint32_t width,
                                                      uint32_t height, uint32_t sampleIndex, uint32_t maxBounces,
                                                      uint32_t sampleCount, uint32_t x0, uint32_t y0, uint32_t x1,
                                                      uint32_t y1, int32_t threads, float* rgbaOut)
{
    if (!t || !c || !t->scene.geometryReady || width == 0 || height == 0) return 0;
    if (t->width != width || t->height != height) {
        t->width = width;
        t->height = height;
        t->rgba.assign(size_t(width) * height * 4u, 0.0f);
    }
    if (!t->fallbackAxisInitialized) {
        t->fallbackZUp = std::fabs(c->vertical[2]) > std::fabs(c->vertical[1]);
        t->fallbackAxisInitialized = true;
    }
    if (x1 == 0 && y1 == 0) {
        x1 = width;
        y1 = height;
    }
    std::lock_guard<std::mutex> lock(gRenderMutex);
    oracle::PackedScene& s = t->scene;
    using namespace glsl;
    gScene = &s;
    gBvh = &t->bvh;
    gSceneOpaque = s.opaque;
    positions = reinterpret_cast<vec4*>(s.vertices.data());
    indices = s.indices.data();
    triangleMaterials = s.triangleMaterials.data();
    materials = reinterpret_cast<GpuMaterial*>(s.materials.data());
    texcoords = reinterpret_cast<vec2*>(s.texcoords.data());
    shadingNormals = reinterpret_cast<vec4*>(s.normals.data());
    lights = reinterpret_cast<GpuLight*>(s.lights.data());
    emissiveTriangles = reinterpret_cast<vec4*>(s.emissive.data());
    pixels = reinterpret_cast<vec4*>(t->rgba.data());
    for (size_t i = 0; i < 256; ++i) materialTextures[i] = sampler2D{};
    for (size_t i = 0; i < s.textures.size() && i < 256; ++i) {
        materialTextures[i] = sampler2D{s.textures[i].linear.data(), static_cast<int>(s.textures[i].width),
                                        static_cast<int>(s.textures[i].height)};
    }
    const uint32_t sc = std::max(sampleCount, 1u);
    // CameraUniform packing (vulkan_path_tracer.cpp:3242-3254).
    camera.origin = vec4(c->origin[0], c->origin[1], c->origin[2], static_cast<float>(sc));
    camera.lowerLeft = vec4(c->lower_left[0], c->lower_left[1], c->lower_left[2], static_cast<float>(s.primitiveCount));
    camera.horizontal = vec4(c->horizontal[0], c->horizontal[1], c->horizontal[2], 0.0f);
    camera.vertical = vec4(c->vertical[0], c->vertical[1], c->vertical[2], t->fallbackZUp ? 1.0f : 0.0f);
    camera.frame = uvec4{width, height, sampleIndex,
                         std::clamp(maxBounces, 1u, 12u) | (s.opaque ? (1u << 8) : 0u) |
                             (std::min(s.lightCount, 64u) << 16)};
    const unsigned n = threads > 0 ? static_cast<unsigned>(threads) : std::max(1u, std::thread::hardware_concurrency());
    std::atomic<uint32_t> next{y0};
    auto worker = [&]() {
        for (;;) {
            const uint32_t y = next.fetch_add(1);
            if (y >= y1) break;
            for (uint32_t x = x0; x < x1; ++x) {
                gl_GlobalInvocationID = uvec3{x, y, 0};
                glsl_main();
            }
        }
    };
    std::vector<std::thread> pool;
    for (unsigned i = 1; i < n; ++i) pool.emplace_back(worker);
    worker();
    for (auto& th : pool) th.join();
    if (rgbaOut) std::memcpy(rgbaOut, t->rgba.data(), t->rgba.size() * sizeof(float));
    return 1;
}

}  // extern "C"
