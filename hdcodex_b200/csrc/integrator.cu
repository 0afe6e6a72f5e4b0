// integrator.cu - wavefront form of the reference's spectral path tracer.
//
// The reference runs one megakernel invocation per pixel (GLSL main(),
// src/gpu/vulkan_path_tracer.cpp:1189-1891): for every sample and each of the
// three wavelength lanes it loops over bounces, tracing, shading, sampling
// lights and the BSDF. Here every (pixel, sample, lane) is a path slot of a
// wave, and each bounce of a wave is four queue-driven kernels:
//   generate  - camera ray, RNG seed and wavelength of every slot (:1191-1213);
//   extend    - closest-hit traversal of the extension queue (:1228-1243);
//   shade     - miss/emission/medium/material/NEE/BSDF/roulette (:1245-1879),
//               appending surviving paths to the next extension queue and
//               light-sample rays to the shadow queue;
//   shadow    - any-hit visibility of the shadow queue (:855-912);
// and one accumulate kernel per wave adds the lane radiances through the
// sensor (:1882-1884). A path's radiance gets its contributions in the
// megakernel's order: light-sample contributions of bounce b are stored per
// shadow slot and added, in slot order, before anything of bounce b+1.
// Queues are compacted with warp-aggregated atomics; kernels loop over the
// device-side queue length, so a frame needs no host round trip.
#include "integrator.h"
#include "nrc.h"
#include "nvtx_range.h"

#include <cooperative_groups.h>

#include <algorithm>
#include <stdexcept>
#include <string>
#include <vector>

#include "device/shading.cuh"
#include "device/traverse.cuh"

namespace cg = cooperative_groups;

namespace hdcx {
namespace {

#define CUDA_OK(expr)                                                                                  \
    do {                                                                                               \
        cudaError_t err__ = (expr);                                                                    \
        if (err__ != cudaSuccess) throw std::runtime_error(std::string("render: ") + #expr + ": " +     \
                                                           cudaGetErrorString(err__));                 \
    } while (0)

constexpr uint32_t kFlagEnvironmentOnMiss = 1u;
constexpr uint32_t kFlagPreviousWasDelta = 2u;
constexpr uint32_t kFlagInsideMedium = 4u;
constexpr uint32_t kFlagTraining = 8u;  // radiance-cache mode: a full-length training path

enum ShadowKind : uint32_t {
    kShadowAnalytic = 0,
    kShadowSun = 1,
    kShadowSky = 2,
    kShadowMesh = 3,
};

struct WaveDesc {
    uint32_t sampleBase;   // first sample offset of the wave (relative to the render)
    uint32_t samples;      // samples per pixel in the wave
    uint32_t pixelBase;    // first pixel
    uint32_t pixels;       // pixels in the wave
    uint32_t count;        // samples * pixels * 3
};

// Light-sample slot k (0..2) of path `slot` in PathBuffers::contribution and
// ::contributionValid: the three slots of a path are adjacent, so a path's
// pending samples arrive in one memory sector, not three.
__device__ __forceinline__ uint32_t contributionIndex(uint32_t slot, uint32_t k) { return slot * 3u + k; }

__device__ __forceinline__ uint32_t appendIndex(uint32_t* counter)
{
    cg::coalesced_group g = cg::coalesced_threads();
    uint32_t base = 0;
    if (g.thread_rank() == 0) base = atomicAdd(counter, g.size());
    base = g.shfl(base, 0);
    return base + g.thread_rank();
}

__device__ __forceinline__ void slotToPath(const WaveDesc& w, const FrameConst& f, uint32_t slot, uint32_t& pixel,
                                           uint32_t& sampleNumber, uint32_t& lane)
{
    lane = slot % 3u;
    const uint32_t q = slot / 3u;
    pixel = w.pixelBase + q % w.pixels;
    sampleNumber = f.sampleIndex + w.sampleBase + q / w.pixels;
}

// ---------------------------------------------------------------------------
// generate: main() prologue (vulkan_path_tracer.cpp:1191-1223)
// ---------------------------------------------------------------------------
__global__ void generateKernel(FrameConst f, WaveDesc w, PathBuffers p)
{
    const uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot == 0) p.counters[0] = w.count;
    if (slot >= w.count) return;
    uint32_t pixel, sampleNumber, lane;
    slotToPath(w, f, slot, pixel, sampleNumber, lane);
    const uint32_t px = pixel % f.width, py = pixel / f.width;
    const uint32_t index = pixel;
    uint32_t rng = hashState(index ^ (sampleNumber * 0x9e3779b9u) ^ 0xa511e9b3u);
    const float wavelengthShift = u2f(hashState(index ^ 0x68bc21ebu)) * (1.0f / 4294967296.0f);
    const float wavelength =
        380.0f + 400.0f * fract(wavelengthShift + (u2f(sampleNumber & 31u) + 0.5f) / 32.0f + u2f(lane) / 3.0f);
    const float jx = randomFloat(rng);
    const float jy = randomFloat(rng);
    const float u = (u2f(px) + jx) / u2f(f.width);
    const float v = (u2f(py) + jy) / u2f(f.height);
    const float3 direction = normalize(f.lowerLeft + u * f.horizontal + v * f.vertical - f.origin);
    const Spectrum s = makeSpectrum(wavelength);
    p.rng[slot] = rng;
    p.wavelength[slot] = wavelength;
    p.spectrum[slot] = make_float4(s.br, s.bg, s.bb, s.planck);
    p.throughput[slot] = 1.0f;
    p.radiance[slot] = 0.0f;
    p.rayOrigin[slot] = make_float4(f.origin.x, f.origin.y, f.origin.z, 0.0f);
    p.rayDirection[slot] = make_float4(direction.x, direction.y, direction.z, 0.0f);
    uint32_t flags = kFlagEnvironmentOnMiss | kFlagPreviousWasDelta;
    if (p.cache.enabled) {
        // Training paths: a deterministic subset chosen by the path identity.
        const uint32_t key = hashState(pixel ^ hashState(sampleNumber * 0x9e3779b9u + lane * 0x85ebca6bu + 0x27d4eb2fu));
        if (key < p.cache.trainThreshold) {
            const uint32_t t = atomicAdd(p.cache.counters + 1, 1u);
            if (t < p.cache.trainCapacity) {
                flags |= kFlagTraining;
                p.cache.trainIndex[slot] = t;
                p.cache.trainSlot[t] = slot;
                p.cache.trainVertices[t] = 0u;
                for (uint32_t b = 0; b < kCacheMaxVertices; ++b)
                    p.cache.trainState[t * kCacheMaxVertices + b] = make_float2(-1.0f, 0.0f);
            }
        }
    }
    p.flags[slot] = flags;
    if (p.cone != nullptr) p.cone[slot] = make_float2(0.0f, f.pixelSpread);
    p.previousPdf[slot] = make_float2(0.0f, 0.0f);
    p.contributionValid[contributionIndex(slot, 0u)] = 0;
    p.contributionValid[contributionIndex(slot, 1u)] = 0;
    p.contributionValid[contributionIndex(slot, 2u)] = 0;
    p.queue[0][slot] = slot;
}

// ---------------------------------------------------------------------------
// extend: closest hit of every queued ray (vulkan_path_tracer.cpp:1228-1243)
// ---------------------------------------------------------------------------
// Resident blocks of 128 threads per SM the traversal kernels are compiled
// for (8: 64 registers per thread).
#ifndef HDCX_TRACE_MIN_BLOCKS
#define HDCX_TRACE_MIN_BLOCKS 8
#endif

// kInst (traversal kernels): 0 single-level scenes, 1 scenes with instancers.
template <Accept kMode, bool kCount, int kInst>
__global__ void __launch_bounds__(128, HDCX_TRACE_MIN_BLOCKS) extendKernel(DeviceScene s, PathBuffers p, const uint32_t* queue,
                                                    const uint32_t* count)
{
    const uint32_t n = *count;
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(p.stats + 0, static_cast<unsigned long long>(n));
    uint2 work = make_uint2(0u, 0u);
    uint32_t fault = 0u;  // traversal faults of this thread's rays
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t slot = queue[i];
        const float4 o = p.rayOrigin[slot];
        const float4 d = p.rayDirection[slot];
        HitRecord h;
        const bool found = traceRay<kMode, false, kCount, kInst>(s, xyz(o), xyz(d), 0.001f, 10000.0f, p.rng[slot], h, fault, &work);
        p.hit[slot] = found ? make_float4(h.t, __uint_as_float(h.primitive), h.b1, h.b2)
                            : make_float4(0.0f, __uint_as_float(kInvalidPrimitive), 0.0f, 0.0f);
        // Hits and misses go to separate queues, so that shading warps hold
        // only hits and the short environment path runs in its own kernel.
        if (found) p.hitQueue[appendIndex(p.counters + 4)] = slot;
        else p.missQueue[appendIndex(p.counters + 5)] = slot;
    }
    if (fault != 0u) atomicOr(reinterpret_cast<unsigned int*>(p.stats + 7), fault);
    if (kCount) {
        atomicAdd(p.stats + 3, static_cast<unsigned long long>(work.x));
        atomicAdd(p.stats + 4, static_cast<unsigned long long>(work.y));
    }
}

// ---------------------------------------------------------------------------
// shade
//
// shadeKernel<true> evaluates the whole closure. shadeKernel<false> serves
// scenes whose materials bind no textures and have no coat, sheen,
// transmission, subsurface or diffuse-transmission weight and use the Lambert
// diffuse model (DeviceScene::fullShading == 0): there those quantities are
// the constants the general kernel computes for them (fallback values, zero
// weights), so both kernels return the same bits and the specialised one
// carries far less code and state.
// ---------------------------------------------------------------------------
template <bool kFull>
HDCX_D float4 materialTexture(float lodBase, const DeviceScene& s, uint32_t index, float2 uv, float4 fallback)
{
    if (!kFull) return fallback;
    return sampleMaterialTexture(s, index, uv, fallback, lodBase);
}
struct ShadeCtx {
    const DeviceScene& s;
    const FrameConst& f;
    PathBuffers& p;
    uint32_t slot;
};

__device__ __forceinline__ void setContribution(PathBuffers& p, uint32_t slot, uint32_t k, float value)
{
    p.contribution[contributionIndex(slot, k)] = value;
    p.contributionValid[contributionIndex(slot, k)] = 1;
}

__device__ __forceinline__ void emitShadow(PathBuffers& p, uint32_t slot, uint32_t k, uint32_t kind, uint32_t light,
                                           float3 origin, float3 direction, float tmax, float a, float g1, float g2,
                                           float g3)
{
    const uint32_t j = appendIndex(p.counters + 2);
    p.shadowOrigin[j] = make_float4(origin.x, origin.y, origin.z, tmax);
    p.shadowDirection[j] = make_float4(direction.x, direction.y, direction.z, a);
    p.shadowFactors[j] = make_float4(g1, g2, g3, 0.0f);
    p.shadowSlot[j] = slot * 4u + k;
    p.shadowInfo[j] = kind | (light << 8);
    p.contributionValid[contributionIndex(slot, k)] = 1;
}

// Light-sample visibility that needs no ray: shadowVisibility's early returns
// (vulkan_path_tracer.cpp:858-861) give vec3(1.0).
__device__ __forceinline__ float analyticNeedsRay(const GpuLight& light, float maximumDistance, float& traceDistance)
{
    if (light.shadow.x < 0.5f) return 0.0f;
    traceDistance = maximumDistance;
    if (light.shadow.y >= 0.0f) traceDistance = gmin(traceDistance, light.shadow.y);
    if (traceDistance <= 0.001f) return 0.0f;
    return 1.0f;
}

// Analytic/sun/sky sample: value = contribution with visibility sv.
__device__ __forceinline__ float combineShadow(uint32_t kind, float a, float sv, float g1, float g2, float g3)
{
    if (kind == kShadowAnalytic) return a * sv * g1 * g2 / g3;
    if (kind == kShadowSun) return a * sv;
    return a * sv * g1;  // sky
}

__device__ void traceSurfaceLightSample(PathBuffers& p, const DeviceScene& s, const Spectrum& spec, uint32_t slot,
                                        uint32_t k, uint32_t kind, uint32_t lightIndex, const GpuLight& light,
                                        float3 origin, float3 direction, float maximumDistance, float a, float g1,
                                        float g2, float g3)
{
    float traceDistance = maximumDistance;
    if (analyticNeedsRay(light, maximumDistance, traceDistance) != 0.0f) {
        emitShadow(p, slot, k, kind, lightIndex, origin, direction, traceDistance, a, g1, g2, g3);
    } else {
        const float sv = reflectanceSpectrum(f3(1.0f), spec);
        setContribution(p, slot, k, combineShadow(kind, a, sv, g1, g2, g3));
    }
}

template <int kInst = -1>
__device__ bool traceOpaqueBoundary(const DeviceScene& s, PathBuffers& p, float3 origin, float3 direction,
                                    float3& boundary, float3& boundaryNormal, float& boundaryDistance)
{
    // :1130-1151
    atomicAdd(p.stats + 2, 1ull);
    HitRecord h;
    uint32_t fault = 0u;
    const bool found = traceRay<Accept::Opaque, false, false, kInst>(s, origin, direction, 0.001f, 10000.0f, 0u, h, fault);
    if (fault != 0u) atomicOr(reinterpret_cast<unsigned int*>(p.stats + 7), fault);
    if (!found) return false;
    const uint32_t primitive = h.primitive;
    const float3 p0 = xyz(__ldg(s.vertices + __ldg(s.indices + primitive * 3u + 0u)));
    const float3 p1 = xyz(__ldg(s.vertices + __ldg(s.indices + primitive * 3u + 1u)));
    const float3 p2 = xyz(__ldg(s.vertices + __ldg(s.indices + primitive * 3u + 2u)));
    boundaryDistance = h.t;
    boundary = origin + direction * boundaryDistance;
    boundaryNormal = normalize(cross(p1 - p0, p2 - p0));
    if (dot(boundaryNormal, direction) > 0.0f) boundaryNormal = -boundaryNormal;
    return true;
}

template <int kInst = -1>
__device__ bool randomWalkSubsurface(const DeviceScene& s, PathBuffers& p, float3 entry, float3 outwardNormal,
                                     float meanFreePath, float albedo, float anisotropy, uint32_t& state,
                                     float3& exitOrigin, float3& exitDirection, float& attenuation)
{
    // :1153-1186
    const float radius = gmax(meanFreePath, 0.001f);
    const float sigmaS = 1.0f / radius;
    const float sigmaA = -glog(clampf(albedo, 0.001f, 0.9999f)) / radius;
    float3 origin = entry - outwardNormal * 0.003f;
    float3 direction = cosineHemisphere(-outwardNormal, state);
    attenuation = 1.0f;
    for (int step = 0; step < 8; ++step) {
        float3 boundary, boundaryNormal;
        float boundaryDistance;
        if (!traceOpaqueBoundary<kInst>(s, p, origin, direction, boundary, boundaryNormal, boundaryDistance)) return false;
        const float scatterDistance = -glog(gmax(1.0f - randomFloat(state), 1e-6f)) / sigmaS;
        const bool forceExit = step == 7;
        const float travel = forceExit ? boundaryDistance : gmin(scatterDistance, boundaryDistance);
        attenuation = attenuation * gexp(-sigmaA * travel);
        if (forceExit || scatterDistance >= boundaryDistance) {
            exitDirection = direction;
            exitOrigin = boundary + direction * 0.003f;
            return true;
        }
        origin = origin + direction * scatterDistance;
        direction = sampleHenyeyGreenstein(direction, anisotropy, state);
    }
    return false;
}

// kLit: the scene has analytic or dome lights and no emissive triangles, so
// neither the fallback sun and sky (:1593-1668) nor emissive-triangle
// sampling (:1670-1731) can run; both are compiled out.
// kCache: radiance-cache mode (PathBuffers::cache): queries and training
// records at surface vertices; the plain kernels compile without it.
// The lit variants wait on memory most of the time (long-scoreboard stalls):
// the non-full ones are capped at 80 registers so that six blocks fit an SM
// instead of four, the full ones at 128 registers for four blocks instead of
// three; each costs a few spilled values and gains 4-6% of the kernel's time.
//
// kWalk: how a subsurface random walk (:1153-1186) runs.
//   kWalkInline - inside this kernel, nested in shading (renders without
//                 walk buffers);
//   kWalkDefer  - the walk's start (entry, normal, mean free path, albedo,
//                 anisotropy, RNG state, throughput) is recorded and the path
//                 handed to walkKernel, a traversal kernel; everything before
//                 it in the bounce (emission, the light sample, the radiance
//                 so far) is done. On the last bounce the walk cannot change
//                 the image and is not run;
//   kWalkReplay - re-shades a path whose deferred walk failed (a boundary ray
//                 escaped): the same bounce from its stored start, with the
//                 light sample and radiance writes of the first pass
//                 suppressed, taking the walk's RNG state after the failed
//                 walk at the walk's place and continuing with the diffuse
//                 lobe as the inline form does.
// All three give the same bits.
enum : int { kWalkInline = 0, kWalkDefer = 1, kWalkReplay = 2 };

// Light records a shade block copies into shared memory (3.5 KB).
constexpr uint32_t kStagedLights = 16;

template <bool kFull, bool kLit, bool kCache, int kWalk = kWalkInline>
__global__ void __launch_bounds__(128, kLit ? (kFull ? 4 : 6) : 1)
    shadeKernel(DeviceScene s, FrameConst f, PathBuffers p, uint32_t bounce, const uint32_t* queue,
                const uint32_t* count, uint32_t* nextQueue, uint32_t* nextCount)
{
    constexpr bool kReplay = kWalk == kWalkReplay;
    static_assert(kWalk == kWalkInline || kFull, "deferred walks are for the full kernels");
    const uint32_t n = *count;
    const bool lastBounce = bounce + 1u >= f.maxBounces;
    // Closure staging: with hits sorted by material (tuning sort_hits) a
    // block's consecutive hits mostly share one material. Its 368-byte
    // record is copied once per block iteration into shared memory, 16 bytes
    // per thread, and every thread whose hit uses it reads it from there;
    // other hits read theirs from global memory. Every thread of the block
    // runs the same iterations (the loop steps by block, not by thread).
    constexpr bool kStageable = kFull && !kReplay;
    const bool stage = kStageable && p.sortHits != 0u;
    __shared__ __align__(16) GpuMaterial stagedMaterial;
    __shared__ uint32_t stagedIndex;
    // The scene's light records, read two to three times over per shade
    // event by light selection and the environment pdf: copied once per
    // block into shared memory when there are at most kStagedLights of them.
    __shared__ __align__(16) GpuLight stagedLights[kStagedLights];
    const bool lightsStaged = s.lightCount <= kStagedLights;
    if (lightsStaged) {
        const uint32_t words = s.lightCount * static_cast<uint32_t>(sizeof(GpuLight) / sizeof(uint4));
        for (uint32_t w = threadIdx.x; w < words; w += blockDim.x)
            reinterpret_cast<uint4*>(stagedLights)[w] = __ldg(reinterpret_cast<const uint4*>(s.lights) + w);
    }
    __syncthreads();
    const GpuLight* lights = lightsStaged ? stagedLights : s.lights;
    for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
        if (stage) {
            __syncthreads();  // the previous iteration's reads of the staged record are done
            if (threadIdx.x == 0) {
                const uint32_t first = __float_as_uint(p.hit[queue[base]].y);
                stagedIndex = first == kInvalidPrimitive ? 0xffffffffu : __ldg(s.triangleMaterials + first);
            }
            __syncthreads();
            if (stagedIndex != 0xffffffffu && threadIdx.x < sizeof(GpuMaterial) / sizeof(uint4)) {
                reinterpret_cast<uint4*>(&stagedMaterial)[threadIdx.x] =
                    __ldg(reinterpret_cast<const uint4*>(s.materials + stagedIndex) + threadIdx.x);
            }
            __syncthreads();
        }
        const uint32_t i = base + threadIdx.x;
        if (i >= n) continue;
        const uint32_t slot = queue[i];
        float radiance = p.radiance[slot];
        // Light-sample contributions of the previous bounce, in slot order.
        // (A replay finds this bounce's own samples in the slots: they stay.)
        for (uint32_t k = 0; k < 3u && !kReplay; ++k) {
            uint8_t& valid = p.contributionValid[contributionIndex(slot, k)];
            if (valid) {
                radiance += p.contribution[contributionIndex(slot, k)];
                valid = 0;
            }
        }
        const Spectrum spec = spectrumFromBasis(p.wavelength[slot], p.spectrum[slot]);
        const float wavelength = spec.wavelength;
        uint32_t rng = p.rng[slot];
        float throughput = p.throughput[slot];
        uint32_t flags = p.flags[slot];
        bool environmentOnMiss = (flags & kFlagEnvironmentOnMiss) != 0u;
        bool previousWasDelta = (flags & kFlagPreviousWasDelta) != 0u;
        bool insideMedium = (flags & kFlagInsideMedium) != 0u;
        float2 previousPdf = p.previousPdf[slot];
        float previousBsdfPdf = previousPdf.x;
        float previousEnvironmentLightPdf = previousPdf.y;
        // The medium coefficients matter only inside a medium (entering one
        // sets all three), so paths outside one neither read nor write them.
        const float4 medium = insideMedium ? p.medium[slot] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        float mediumAbsorption = medium.x, mediumScattering = medium.y, mediumAnisotropy = medium.z;
        float3 rayOrigin = xyz(p.rayOrigin[slot]);
        float3 rayDirection = xyz(p.rayDirection[slot]);
        const float4 hitRec = p.hit[slot];
        const uint32_t primitive = __float_as_uint(hitRec.y);
        bool alive = true;
        bool deferred = false;  // kWalkDefer: walkKernel finishes this bounce
        // Ray cone (width, spread) of texture LOD; spread <= 0: level 0.
        const bool lodOn = kFull && f.pixelSpread > 0.0f && p.cone != nullptr;
        const float2 cone = lodOn ? p.cone[slot] : make_float2(0.0f, -1.0f);
        float coneWidth = 0.0f;
        bool coneKept = false;  // a smooth reflection or refraction keeps the cone

        if (primitive == kInvalidPrimitive) {
            // :1245-1255
            if (environmentOnMiss) {
                const float misWeight = previousWasDelta ? 1.0f : powerHeuristic(previousBsdfPdf, previousEnvironmentLightPdf);
                radiance += throughput * misWeight * illuminantSpectrum(environment(s, f, rayDirection), spec);
            }
            p.radiance[slot] = radiance;
            continue;
        }

        do {  // one bounce; `break` ends shading of this bounce
            const uint32_t i0 = __ldg(s.indices + primitive * 3u + 0u);
            const uint32_t i1 = __ldg(s.indices + primitive * 3u + 1u);
            const uint32_t i2 = __ldg(s.indices + primitive * 3u + 2u);
            const float3 p0 = xyz(__ldg(s.vertices + i0));
            const float3 p1 = xyz(__ldg(s.vertices + i1));
            const float3 p2 = xyz(__ldg(s.vertices + i2));
            const float3 geometricNormal = normalize(cross(p1 - p0, p2 - p0));
            const bool frontFace = dot(geometricNormal, rayDirection) < 0.0f;
            const float3 orientedGeometricNormal = frontFace ? geometricNormal : -geometricNormal;
            const float b1 = hitRec.z, b2 = hitRec.w;
            const float3 authoredNormal = surfaceShadingNormal(s, primitive, b1, b2, geometricNormal);
            float3 normal = frontFace ? authoredNormal : -authoredNormal;
            const float2 uv0 = __ldg(s.texcoords + primitive * 3u + 0u);
            const float2 uv1 = __ldg(s.texcoords + primitive * 3u + 1u);
            const float2 uv2 = __ldg(s.texcoords + primitive * 3u + 2u);
            const float2 surfaceUv = surfaceTextureCoordinates(s, primitive, b1, b2);
            const float distance = hitRec.x;
            // Texture LOD by ray cones (hdcx_set_texture_lod; Akenine-Moller et
            // al., "Texture Level of Detail Strategies for Real-Time Ray
            // Tracing", 2019): the cone's width at the hit, the triangle's
            // texel-to-world area ratio and the incidence give the
            // texture-independent part of the level; -inf samples level 0.
            float lodBase = -INFINITY;
            if (kFull && lodOn && cone.y > 0.0f) {
                coneWidth = cone.x + cone.y * distance;
                const float2 du = uv1 - uv0, dv = uv2 - uv0;
                const float uvArea = fabsf(du.x * dv.y - du.y * dv.x);
                const float3 c = cross(p1 - p0, p2 - p0);
                const float worldArea = sqrtf(dot(c, c));
                const float incidence = fmaxf(fabsf(dot(geometricNormal, rayDirection)), 1e-4f);
                if (uvArea > 0.0f && worldArea > 0.0f && coneWidth > 0.0f)
                    lodBase = 0.5f * log2f(uvArea / worldArea) + log2f(coneWidth / incidence);
            }
            const float3 hit = rayOrigin + rayDirection * distance;
            if (insideMedium) {
                // :1279-1295
                if (mediumScattering > 0.0f) {
                    const float scatterDistance = -glog(gmax(1.0f - randomFloat(rng), 1e-6f)) / mediumScattering;
                    if (scatterDistance < distance) {
                        throughput = throughput * gexp(-mediumAbsorption * scatterDistance);
                        rayOrigin = rayOrigin + rayDirection * scatterDistance;
                        rayDirection = sampleHenyeyGreenstein(rayDirection, mediumAnisotropy, rng);
                        environmentOnMiss = true;
                        previousWasDelta = true;
                        previousBsdfPdf = 0.0f;
                        break;
                    }
                }
                throughput = throughput * gexp(-mediumAbsorption * distance);
            }
            const uint32_t materialIndex = __ldg(s.triangleMaterials + primitive);
            const GpuMaterial* material =
                (stage && materialIndex == stagedIndex) ? &stagedMaterial : s.materials + materialIndex;
            float3 baseColorRgb = xyz(material->baseColorMetalness);
            if (kFull && material->textureIndices0.x != kMissingTexture) {
                const float4 sample = materialTexture<kFull>(lodBase, s, material->textureIndices0.x, surfaceUv, f4(baseColorRgb, 1.0f));
                const float scaleW = material->baseColorTextureScale.w;
                const int channel = static_cast<int>(roundf(scaleW));
                float3 sourceColor;
                if (channel < 0) {
                    sourceColor = f3(sample.x, sample.y, sample.z);
                } else {
                    const int c = min(channel, 3);
                    sourceColor = f3(c == 0 ? sample.x : (c == 1 ? sample.y : (c == 2 ? sample.z : sample.w)));
                }
                baseColorRgb = xyz(material->baseColorTextureBias) + xyz(material->baseColorTextureScale) * sourceColor;
            }
            const float baseColor = reflectanceSpectrum(baseColorRgb, spec);
            const float metalness = clampf(
                materialTexture<kFull>(lodBase, s, material->textureIndices0.y, surfaceUv, f4(material->baseColorMetalness.w)).x, 0.0f, 1.0f);
            const float4 roughnessSample = materialTexture<kFull>(
                lodBase, s, material->textureIndices0.z, surfaceUv,
                make_float4(material->emissionRoughness.w, material->subsurfaceColor.w, 0.0f, 1.0f));
            const float2 roughness = make_float2(clampf(roughnessSample.x, 0.02f, 1.0f), clampf(roughnessSample.y, 0.02f, 1.0f));
            const float diffuseRoughness = clampf(
                materialTexture<kFull>(lodBase, s, material->textureIndices4.z, surfaceUv, f4(material->diffuseProperties.x)).x, 0.0f, 1.0f);
            const float diffuseWeight = clampf(
                materialTexture<kFull>(lodBase, s, material->textureIndices4.w, surfaceUv, f4(material->diffuseProperties.z)).x, 0.0f, 1.0f);
            const uint32_t diffuseModel = kFull ? static_cast<uint32_t>(material->diffuseProperties.y + 0.5f) : 0u;
            if (kFull) normal = applyNormalMap(s, material->textureIndices1.y, material->coatWeightRoughnessIor.w > 0.5f,
                                    material->subsurfaceWeightScale.w, surfaceUv, normal, p0, p1, p2, uv0, uv1, uv2);
            const float3 tangent = surfaceTangent(normal, p0, p1, p2, uv0, uv1, uv2);
            // (A replay re-shades a bounce whose first pass went past this
            // point without ending the path and has recorded its vertex.)
            if (kCache && !kReplay) {
                const bool training = (flags & kFlagTraining) != 0u;
                bool terminate = bounce >= p.cache.prefixBounces;
                if (p.cache.spreadFactor > 0.0f) {
                    // Path spread (Mueller, Rousselle, Keller and Novak, "Real-time
                    // Neural Radiance Caching for Path Tracing", 2021, sec. 3.4):
                    // a(x1..xn) = (sum over i >= 2 of sqrt(|x(i-1) - xi|^2 /
                    // (p(wi) |cos(theta_i)|)))^2 against the primary footprint
                    // a0 = |x0 - x1|^2 / (4 pi |cos(theta_1)|); the path ends
                    // once a > c a0. A specular bounce (infinite pdf) adds nothing.
                    const float cosine = fmaxf(fabsf(dot(geometricNormal, rayDirection)), 1e-6f);
                    const float d2 = distance * distance;
                    float2 spread = bounce == 0u ? make_float2(d2 / (12.566370614f * cosine), 0.0f) : p.cache.spread[slot];
                    if (bounce > 0u && !previousWasDelta && previousBsdfPdf > 0.0f)
                        spread.y += sqrtf(d2 / (previousBsdfPdf * cosine));
                    p.cache.spread[slot] = spread;
                    terminate = terminate || spread.y * spread.y > p.cache.spreadFactor * spread.x;
                }
                if (training || terminate) {
                    const float3 qp = (hit - p.cache.sceneMin) * p.cache.sceneScale;
                    const float4 q0 = make_float4(qp.x, qp.y, qp.z, -rayDirection.x);
                    const float4 q1 = make_float4(-rayDirection.y, -rayDirection.z, normal.x, normal.y);
                    const float4 q2 = make_float4(normal.z, roughness.x, (wavelength - 380.0f) / 400.0f, 0.0f);
                    if (training) {
                        if (bounce < kCacheMaxVertices) {
                            const uint32_t r = p.cache.trainIndex[slot] * kCacheMaxVertices + bounce;
                            float4* rec = reinterpret_cast<float4*>(p.cache.trainRecords) + r * 3u;
                            rec[0] = q0;
                            rec[1] = q1;
                            rec[2] = q2;
                            p.cache.trainState[r] = make_float2(throughput, radiance);
                            p.cache.trainVertices[p.cache.trainIndex[slot]] = bounce + 1u;
                        }
                    } else {
                        // The cache replaces everything from this vertex on.
                        const uint32_t j = appendIndex(p.cache.counters + 0);
                        float4* rec = reinterpret_cast<float4*>(p.cache.queries) + static_cast<size_t>(j) * 3u;
                        rec[0] = q0;
                        rec[1] = q1;
                        rec[2] = q2;
                        p.cache.querySlot[j] = slot;
                        p.throughput[slot] = throughput;
                        alive = false;
                        break;
                    }
                }
            }
            const float3 emissionRgb = surfaceEmissionRgb(s, primitive, surfaceUv);
            const float emission = illuminantSpectrum(emissionRgb, spec);
            float emissionMisWeight = 1.0f;
            if (!previousWasDelta && (emissionRgb.x > 0.0f || emissionRgb.y > 0.0f || emissionRgb.z > 0.0f)) {
                const float emissionCosine = fabsf(dot(geometricNormal, -rayDirection));
                const float lightPdf = emissionCosine <= 0.0f
                                           ? 0.0f
                                           : __ldg(&s.emissive[primitive].y) * (distance * distance) / emissionCosine;
                emissionMisWeight = powerHeuristic(previousBsdfPdf, lightPdf);
            }
            radiance += throughput * emission * emissionMisWeight;

            const float transmission = kFull ? clampf(material->transmissionOpacityIor.x, 0.0f, 1.0f) : 0.0f;
            float3 transmissionColorRgb = xyz(material->transmissionColorThinWalled);
            if (transmission > 0.0f) {
                const float4 t = materialTexture<kFull>(lodBase, s, material->textureIndices1.z, surfaceUv, f4(transmissionColorRgb, 1.0f));
                transmissionColorRgb = f3(t.x, t.y, t.z);
            }
            const float transmissionColor = reflectanceSpectrum(transmissionColorRgb, spec);
            float subsurface = 0.0f;
            float diffuseColor = baseColor;
            float3 subsurfaceColorRgb = xyz(material->subsurfaceColor);
            float3 subsurfaceRadiusRgb = make_float3(gmax(material->subsurfaceRadius.x, 0.001f), gmax(material->subsurfaceRadius.y, 0.001f),
                                                     gmax(material->subsurfaceRadius.z, 0.001f));
            if (kFull && (material->subsurfaceWeightScale.x > 0.0f || material->textureIndices2.x != kMissingTexture)) {
                subsurface = clampf(materialTexture<kFull>(lodBase, s, material->textureIndices2.x, surfaceUv,
                                                          f4(material->subsurfaceWeightScale.x)).x, 0.0f, 1.0f);
                if (subsurface > 0.0f) {
                    const float4 c = materialTexture<kFull>(lodBase, s, material->textureIndices2.y, surfaceUv,
                                                           f4(xyz(material->subsurfaceColor), 1.0f));
                    subsurfaceColorRgb = f3(c.x, c.y, c.z);
                    const float4 r = materialTexture<kFull>(lodBase, s, material->textureIndices2.z, surfaceUv,
                                                           f4(xyz(material->subsurfaceRadius), 1.0f));
                    subsurfaceRadiusRgb = make_float3(gmax(r.x, 0.001f), gmax(r.y, 0.001f), gmax(r.z, 0.001f));
                    const float subsurfaceColor = reflectanceSpectrum(subsurfaceColorRgb, spec);
                    diffuseColor = mix(baseColor, subsurfaceColor, subsurface);
                }
            }
            const float ior = dispersedIor(gmax(material->transmissionOpacityIor.z, 1.0001f), material->transmissionMedium.z,
                                           material->transmissionMedium.w, wavelength);
            const float specularWeight = clampf(
                materialTexture<kFull>(lodBase, s, material->textureIndices3.x, surfaceUv, f4(material->specularWeightColor.x)).x, 0.0f, 1.0f);
            const float4 specularColorSample = materialTexture<kFull>(
                lodBase, s, material->textureIndices3.y, surfaceUv,
                make_float4(material->specularWeightColor.y, material->specularWeightColor.z, material->specularWeightColor.w, 1.0f));
            const float specularColor =
                reflectanceSpectrum(f3(specularColorSample.x, specularColorSample.y, specularColorSample.z), spec);
            float dielectricReflectance = (ior - 1.0f) / (ior + 1.0f);
            dielectricReflectance = dielectricReflectance * dielectricReflectance;
            const float f0 = mix(clampf(dielectricReflectance * specularWeight * specularColor, 0.0f, 1.0f), baseColor, metalness);
            float coat = 0.0f;
            float2 coatRoughness = make_float2(material->coatWeightRoughnessIor.y, material->subsurfaceRadius.w);
            float coatF0 = 0.0f;
            if (kFull && (material->coatWeightRoughnessIor.x > 0.0f || material->textureIndices3.z != kMissingTexture)) {
                coat = clampf(materialTexture<kFull>(lodBase, s, material->textureIndices3.z, surfaceUv,
                                                    f4(material->coatWeightRoughnessIor.x)).x, 0.0f, 1.0f);
                if (coat > 0.0f) {
                    const float4 cc = materialTexture<kFull>(lodBase, s, material->textureIndices3.w, surfaceUv, f4(xyz(material->coatColor), 1.0f));
                    const float coatColor = reflectanceSpectrum(f3(cc.x, cc.y, cc.z), spec);
                    const float4 cr = materialTexture<kFull>(lodBase, s, material->textureIndices4.x, surfaceUv,
                                                            make_float4(coatRoughness.x, coatRoughness.y, 0.0f, 1.0f));
                    coatRoughness = make_float2(clampf(cr.x, 0.02f, 1.0f), clampf(cr.y, 0.02f, 1.0f));
                    const float coatIor = gmax(material->coatWeightRoughnessIor.z, 1.0001f);
                    float coatReflectance = (coatIor - 1.0f) / (coatIor + 1.0f);
                    coatReflectance = coatReflectance * coatReflectance;
                    coatF0 = clampf(coatReflectance * coatColor, 0.0f, 1.0f);
                }
            }
            const float sheen =
                kFull ? clampf(materialTexture<kFull>(lodBase, s, material->textureIndices1.w, surfaceUv, f4(material->coatColor.w)).x, 0.0f, 1.0f)
                      : 0.0f;
            const float4 sheenColorSample = materialTexture<kFull>(lodBase, s, material->textureIndices2.w, surfaceUv,
                                                                  f4(xyz(material->sheenColorMode), 1.0f));
            const float sheenColor = reflectanceSpectrum(f3(sheenColorSample.x, sheenColorSample.y, sheenColorSample.z), spec);
            const float sheenRoughness = clampf(
                materialTexture<kFull>(lodBase, s, material->textureIndices4.y, surfaceUv, f4(material->transmissionScatter.w)).x, 0.01f, 1.0f);
            const bool sheenZeltner = material->sheenColorMode.w > 0.5f;
            const float translucentWeight = !kFull ? 0.0f : clampf(
                materialTexture<kFull>(lodBase, s, material->textureIndices5.x, surfaceUv, f4(material->translucentColorWeight.w)).x, 0.0f, 1.0f);
            const float4 translucentSample = materialTexture<kFull>(lodBase, s, material->textureIndices5.y, surfaceUv,
                                                                   f4(xyz(material->translucentColorWeight), 1.0f));
            const float translucentColor = reflectanceSpectrum(f3(translucentSample.x, translucentSample.y, translucentSample.z), spec);

            const float3 viewDirection = normalize(-rayDirection);
            const float nDotView = gmax(dot(normal, viewDirection), 0.0f);
            // sheenAlbedo only ever appears multiplied by sheen; with sheen == 0
            // those products are exact zeros for any finite albedo.
            const float sheenAlbedo = sheen == 0.0f ? 0.0f
                                      : (sheenZeltner ? sheenZeltnerDirectionalAlbedo(nDotView, sheenRoughness)
                                                      : sheenDirectionalAlbedo(nDotView, sheenRoughness));
            const float sheenProbability = clampf(sheen * sheenAlbedo * luminance1(sheenColor), 0.0f, 0.95f);
            const float coatContribution = coat > 0.0f ? coat * fresnelSchlick(nDotView, coatF0) : 0.0f;
            const float coatProbability = clampf(luminance1(coatContribution), 0.0f, 0.95f);
            const float baseFresnel = fresnelSchlick(nDotView, f0);
            const float specularContribution = baseFresnel;
            const float diffuseContribution =
                (1.0f - baseFresnel) * diffuseWeight * (1.0f - translucentWeight) * (1.0f - metalness) * diffuseColor;
            const float translucentContribution = (1.0f - baseFresnel) * translucentWeight * (1.0f - metalness) * translucentColor;
            const float specularEnergy = luminance1(specularContribution);
            const float diffuseEnergy = luminance1(diffuseContribution);
            const float translucentEnergy = luminance1(translucentContribution);
            const float baseEnergy = diffuseEnergy + translucentEnergy;
            const float specularProbability = clampf(specularEnergy / gmax(specularEnergy + baseEnergy, 1e-5f), 0.05f, 0.95f);
            const float translucentProbability = baseEnergy > 1e-5f ? translucentEnergy / baseEnergy : 0.0f;
            const uint32_t lightCount = kLit ? 1u : s.lightCount;
            const bool hasMeshLights = kLit ? false : s.hasMeshLights != 0u;

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
                // :1469-1592 analytic light sample
                const float directSpecularEnergy = specularEnergy + luminance1(coatContribution) + sheenProbability;
                uint32_t lightIndex;
                float lightSelectionPdf;
                sampleAnalyticLight(s, lights, hit, normal, diffuseEnergy, directSpecularEnergy, translucentEnergy, rng,
                                    lightIndex, lightSelectionPdf);
                const GpuLight& light = lights[lightIndex];
                float3 lightDirection = f3(0.0f, 1.0f, 0.0f);
                float3 lightRadiance = f3(0.0f);
                float inversePdf = 0.0f;
                float maximumShadowDistance = 10000.0f;
                const uint32_t type = light.textureInfo.z;
                if (type == 0u) {
                    float lightPdf = 0.0f;
                    sampleDomeLight(s, light, rng, lightDirection, lightPdf);
                    lightRadiance = sampleDome(s, light, lightDirection);
                    inversePdf = lightPdf > 0.0f ? 1.0f / lightPdf : 0.0f;
                } else if (type == 5u) {
                    const float halfAngle = 0.5f * radians(clampf(light.geometry.z, 0.0f, 359.999f));
                    if (halfAngle <= 1e-6f) {
                        lightDirection = normalize(xyz(light.basisZ));
                        inversePdf = 1.0f;
                    } else {
                        const float cosineMaximum = gcos(halfAngle);
                        const float cosineTheta = mix(cosineMaximum, 1.0f, randomFloat(rng));
                        const float sineTheta = sqrtf(gmax(1.0f - cosineTheta * cosineTheta, 0.0f));
                        const float phi = kTwoPi * randomFloat(rng);
                        lightDirection = normalize(xyz(light.basisX) * (gcos(phi) * sineTheta) +
                                                   xyz(light.basisY) * (gsin(phi) * sineTheta) + xyz(light.basisZ) * cosineTheta);
                        inversePdf = 1.0f;
                    }
                    lightRadiance = xyz(light.colorIntensity) * light.colorIntensity.w;
                } else {
                    const float lu = randomFloat(rng);
                    const float lv = randomFloat(rng);
                    float3 lightPosition = xyz(light.position);
                    float3 lightNormal = -normalize(xyz(light.basisZ));
                    if (type == 1u) {
                        lightPosition = lightPosition + ((lu - 0.5f) * xyz(light.axisU) + (lv - 0.5f) * xyz(light.axisV));
                    } else if (type == 2u) {
                        const float diskRadius = sqrtf(lu);
                        const float diskPhi = kTwoPi * lv;
                        lightPosition = lightPosition + diskRadius * (gcos(diskPhi) * xyz(light.axisU) + gsin(diskPhi) * xyz(light.axisV));
                    } else if (type == 3u) {
                        lightNormal = uniformSphere(rng);
                        lightPosition = lightPosition + light.geometry.x * lightNormal;
                    } else if (type == 4u) {
                        const float cylinderPhi = kTwoPi * lv;
                        lightNormal = normalize(gcos(cylinderPhi) * xyz(light.basisY) + gsin(cylinderPhi) * xyz(light.basisZ));
                        lightPosition = lightPosition + ((lu - 0.5f) * xyz(light.axisU) + light.geometry.x * lightNormal);
                    }
                    const float3 toLight = lightPosition - hit;
                    const float distanceSquared = dot(toLight, toLight);
                    const float lightDistance = sqrtf(gmax(distanceSquared, 1e-8f));
                    lightDirection = toLight / lightDistance;
                    const float emissionCosine = gmax(dot(lightNormal, -lightDirection), 0.0f);
                    if (emissionCosine > 0.0f && light.controls.w > 0.0f) {
                        const float shapingCosine = gmax(dot(normalize(xyz(light.basisZ)), lightDirection), 0.0f);
                        const float focus = gpow(shapingCosine, gmax(light.shaping.x, 0.0f));
                        const float3 focusColor = mix(xyz(light.focusTint), f3(1.0f), focus);
                        float3 textureValue = f3(1.0f);
                        if (!(type != 1u || light.textureInfo.x == kMissingTexture)) {
                            const float4 t = textureSample(s, light.textureInfo.x, make_float2(lu, lv));
                            textureValue = f3(t.x, t.y, t.z);
                        }
                        lightRadiance = xyz(light.colorIntensity) * light.colorIntensity.w * textureValue * focusColor *
                                        shapingConeFactor(light, shapingCosine);
                        inversePdf = light.controls.w * emissionCosine / gmax(distanceSquared, 1e-8f);
                        maximumShadowDistance = gmax(lightDistance - 0.003f, 0.001f);
                    }
                }
                if (inversePdf > 0.0f) {
                    const float direct = evaluateDirectSurface(normal, tangent, viewDirection, lightDirection, sp,
                                                               light.controls.x, light.controls.y);
                    if (direct > 0.0f) {
                        const float spectralLight = illuminantSpectrum(lightRadiance, spec);
                        const float misWeight =
                            type == 0u ? powerHeuristic(environmentLightPdf(s, lights, hit, normal, lightDirection, diffuseEnergy,
                                                                            directSpecularEnergy, translucentEnergy),
                                                        surfaceReflectionPdf(normal, tangent, viewDirection, lightDirection,
                                                                             roughness, coatRoughness, sheenProbability,
                                                                             coatProbability, specularProbability,
                                                                             translucentProbability))
                                       : 1.0f;
                        const float a = throughput * direct * spectralLight;
                        if (!kReplay) traceSurfaceLightSample(p, s, spec, slot, 0u, kShadowAnalytic, lightIndex, light,
                                                offsetSurfaceOrigin(hit, orientedGeometricNormal, lightDirection), lightDirection,
                                                maximumShadowDistance, a, inversePdf, misWeight, gmax(lightSelectionPdf, 1e-8f));
                    }
                }
            } else if (!kLit && !hasMeshLights) {
                // :1593-1668 fallback sun and sky
                const bool zUp = f.zUp != 0u;
                const float3 up = zUp ? f3(0.0f, 0.0f, 1.0f) : f3(0.0f, 1.0f, 0.0f);
                const float3 azimuth = zUp ? normalize(f3(1.0f, 1.0f, 0.0f)) : normalize(f3(1.0f, 0.0f, 1.0f));
                const float3 sunDirection = normalize(up * 0.9659258f + azimuth * 0.2588190f);
                const GpuLight& dummy = s.lights[0];
                const float direct = evaluateDirectSurface(normal, tangent, viewDirection, sunDirection, sp, 1.0f, 1.0f);
                if (direct > 0.0f) {
                    const float spectralSun = illuminantSpectrum(f3(3.45575f, 3.14159f, 2.82743f), spec);
                    if (!kReplay) traceSurfaceLightSample(p, s, spec, slot, 0u, kShadowSun, 0u, dummy,
                                            offsetSurfaceOrigin(hit, orientedGeometricNormal, sunDirection), sunDirection,
                                            10000.0f, throughput * direct * spectralSun, 0.0f, 0.0f, 0.0f);
                }
                const float3 skyDirection = cosineHemisphere(normal, rng);
                const float skyDirect = evaluateDirectSurface(normal, tangent, viewDirection, skyDirection, sp, 1.0f, 0.0f);
                if (skyDirect > 0.0f) {
                    const float spectralSky = illuminantSpectrum(environment(s, f, skyDirection), spec);
                    if (!kReplay) traceSurfaceLightSample(p, s, spec, slot, 1u, kShadowSky, 0u, dummy,
                                            offsetSurfaceOrigin(hit, orientedGeometricNormal, skyDirection), skyDirection,
                                            10000.0f, throughput * skyDirect * spectralSky,
                                            kPi / gmax(dot(normal, skyDirection), 1e-4f), 0.0f, 0.0f);
                }
                if (translucentWeight > 0.0f) {
                    const float3 backSkyDirection = cosineHemisphere(-normal, rng);
                    const float backSkyDirect =
                        evaluateDirectSurface(normal, tangent, viewDirection, backSkyDirection, sp, 1.0f, 0.0f);
                    if (backSkyDirect > 0.0f) {
                        const float spectralSky = illuminantSpectrum(environment(s, f, backSkyDirection), spec);
                        if (!kReplay) traceSurfaceLightSample(p, s, spec, slot, 2u, kShadowSky, 0u, dummy,
                                                offsetSurfaceOrigin(hit, orientedGeometricNormal, backSkyDirection),
                                                backSkyDirection, 10000.0f, throughput * backSkyDirect * spectralSky,
                                                kPi / gmax(dot(-normal, backSkyDirection), 1e-4f), 0.0f, 0.0f);
                    }
                }
            }

            if (!kLit && hasMeshLights) {
                // :1670-1731 emissive-triangle sample
                const uint32_t primitiveCount = s.primitiveCount;
                const float target = randomFloat(rng);
                uint32_t low = 0u, high = primitiveCount - 1u;
                while (low < high) {
                    const uint32_t middle = low + (high - low) / 2u;
                    if (target <= __ldg(&s.emissive[middle].x)) high = middle;
                    else low = middle + 1u;
                }
                const uint32_t lightPrimitive = low;
                if (lightPrimitive != primitive && __ldg(&s.emissive[lightPrimitive].y) > 0.0f) {
                    const float root = sqrtf(randomFloat(rng));
                    const float second = randomFloat(rng);
                    const float w0 = 1.0f - root, w1 = root * (1.0f - second), w2 = root * second;
                    const float3 lightP0 = xyz(__ldg(s.vertices + __ldg(s.indices + lightPrimitive * 3u + 0u)));
                    const float3 lightP1 = xyz(__ldg(s.vertices + __ldg(s.indices + lightPrimitive * 3u + 1u)));
                    const float3 lightP2 = xyz(__ldg(s.vertices + __ldg(s.indices + lightPrimitive * 3u + 2u)));
                    const float3 lightPosition = lightP0 * w0 + lightP1 * w1 + lightP2 * w2;
                    const float3 lightNormal = normalize(cross(lightP1 - lightP0, lightP2 - lightP0));
                    const float3 toLight = lightPosition - hit;
                    const float distanceSquared = dot(toLight, toLight);
                    const float lightDistance = sqrtf(gmax(distanceSquared, 1e-8f));
                    const float3 lightDirection = toLight / lightDistance;
                    const float emissionCosine = fabsf(dot(lightNormal, -lightDirection));
                    const float lightPdf =
                        emissionCosine <= 0.0f ? 0.0f : __ldg(&s.emissive[lightPrimitive].y) * distanceSquared / emissionCosine;
                    if (lightPdf > 0.0f) {
                        const float direct = evaluateDirectSurface(normal, tangent, viewDirection, lightDirection, sp, 1.0f, 1.0f);
                        if (direct > 0.0f) {
                            const float2 lightUv = surfaceTextureCoordinates(s, lightPrimitive, w1, w2);
                            float3 lightEmissionRgb = surfaceEmissionRgb(s, lightPrimitive, lightUv);
                            lightEmissionRgb = lightEmissionRgb * surfaceOpacity(s, lightPrimitive, w1, w2);
                            const float spectralLight = illuminantSpectrum(lightEmissionRgb, spec);
                            const float bsdfPdf = surfaceReflectionPdf(normal, tangent, viewDirection, lightDirection, roughness,
                                                                       coatRoughness, sheenProbability, coatProbability,
                                                                       specularProbability, translucentProbability);
                            const float misWeight = powerHeuristic(lightPdf, bsdfPdf);
                            const float a = throughput * direct * spectralLight;
                            const float maxDistance = gmax(lightDistance - 0.003f, 0.001f);
                            const float f1 = misWeight / lightPdf;
                            if (kReplay) {
                            } else if (maxDistance <= 0.001f) {
                                setContribution(p, slot, 1u, a * f1);
                            } else {
                                emitShadow(p, slot, 1u, kShadowMesh, 0u,
                                           offsetSurfaceOrigin(hit, orientedGeometricNormal, lightDirection), lightDirection,
                                           maxDistance, a, f1, 0.0f, 0.0f);
                            }
                        }
                    }
                }
            }

            if (randomFloat(rng) < transmission) {
                // :1735-1777
                const float eta = frontFace ? 1.0f / ior : ior;
                const float cosTheta = gmin(dot(-rayDirection, normal), 1.0f);
                float r0 = (1.0f - ior) / (1.0f + ior);
                r0 = r0 * r0;
                const float fresnel = r0 + (1.0f - r0) * gpow5(1.0f - cosTheta);
                const float3 refracted = refract(rayDirection, normal, eta);
                const bool totalInternalReflection = dot(refracted, refracted) < 1e-8f;
                const bool thinWalled = material->transmissionColorThinWalled.w > 0.5f;
                bool refractedThroughBoundary = false;
                if (totalInternalReflection || randomFloat(rng) < fresnel) {
                    rayDirection = reflect(rayDirection, normal);
                } else {
                    rayDirection = thinWalled ? rayDirection : normalize(refracted);
                    refractedThroughBoundary = !thinWalled;
                }
                const float transmissionDepth = gmax(material->transmissionMedium.x, 0.0f);
                throughput = throughput * (transmissionDepth > 0.0f ? 1.0f : transmissionColor);
                if (refractedThroughBoundary) {
                    if (frontFace) {
                        const float spectralTransmission = gmax(transmissionColor, 0.001f);
                        mediumAbsorption = transmissionDepth > 0.0f ? -glog(spectralTransmission) / transmissionDepth : 0.0f;
                        const float spectralScatter = gmax(reconstructRgb(xyz(material->transmissionScatter), spec), 0.0f);
                        mediumScattering = transmissionDepth > 0.0f ? spectralScatter / transmissionDepth : spectralScatter;
                        mediumAnisotropy = material->transmissionMedium.y;
                        insideMedium = true;
                    } else {
                        insideMedium = false;
                        mediumAbsorption = 0.0f;
                        mediumScattering = 0.0f;
                    }
                }
                rayOrigin = hit + rayDirection * 0.002f;
                environmentOnMiss = true;
                previousWasDelta = true;
                previousBsdfPdf = 0.0f;
                coneKept = true;
                break;
            }

            // :1779-1858 BSDF sampling chain
            environmentOnMiss = false;
            rayOrigin = hit + orientedGeometricNormal * 0.002f;
            if (sheenProbability > 0.0f && randomFloat(rng) < sheenProbability) {
                rayDirection = cosineHemisphere(normal, rng);
                const float sheenPdf = gmax(dot(normal, rayDirection), 0.0f) / kPi;
                const float response = sheenResponse(normal, viewDirection, rayDirection, sheenRoughness, sheenZeltner);
                throughput = throughput * (sheen * sheenColor * response / gmax(sheenProbability * sheenPdf, 1e-6f));
                environmentOnMiss = true;
            } else {
                throughput = throughput * ((1.0f - sheen * sheenAlbedo) / gmax(1.0f - sheenProbability, 1e-4f));
                if (coatProbability > 0.0f && randomFloat(rng) < coatProbability) {
                    const float3 incident = rayDirection;
                    rayDirection = sampleGGXReflectionAnisotropic(rayDirection, normal, tangent, coatRoughness, rng);
                    throughput = throughput * (coat * ggxSampleWeightAnisotropic(incident, rayDirection, normal, tangent,
                                                                                 coatRoughness, coatF0) / coatProbability);
                    environmentOnMiss = gmax(coatRoughness.x, coatRoughness.y) < 0.2f;
                } else {
                    throughput = throughput * ((1.0f - coatContribution) / gmax(1.0f - coatProbability, 1e-4f));
                    if (randomFloat(rng) < specularProbability) {
                        const float3 incident = rayDirection;
                        rayDirection = sampleGGXReflectionAnisotropic(rayDirection, normal, tangent, roughness, rng);
                        throughput = throughput * (ggxSampleWeightAnisotropic(incident, rayDirection, normal, tangent,
                                                                              roughness, f0) / specularProbability);
                        environmentOnMiss = gmax(roughness.x, roughness.y) < 0.2f;
                    } else {
                        if (translucentProbability > 0.0f && randomFloat(rng) < translucentProbability) {
                            throughput = throughput * (translucentContribution /
                                                       gmax((1.0f - specularProbability) * translucentProbability, 1e-4f));
                            rayDirection = cosineHemisphere(-normal, rng);
                            rayOrigin = offsetSurfaceOrigin(hit, orientedGeometricNormal, rayDirection);
                        } else {
                            throughput = throughput * (diffuseContribution /
                                                       gmax((1.0f - specularProbability) * (1.0f - translucentProbability), 1e-4f));
                            bool walked = false;
                            if (subsurface > 0.0f && randomFloat(rng) < subsurface) {
                                const float radius = gmax(reconstructRgb(subsurfaceRadiusRgb, spec) *
                                                              gmax(material->subsurfaceWeightScale.y, 0.0f),
                                                          0.001f);
                                const float albedo = reflectanceSpectrum(subsurfaceColorRgb, spec);
                                float3 exitOrigin, exitDirection;
                                float attenuation;
                                if (kWalk == kWalkDefer) {
                                    if (!lastBounce) {
                                        p.walkEntry[slot] = make_float4(hit.x, hit.y, hit.z, radius);
                                        p.walkNormal[slot] = make_float4(orientedGeometricNormal.x, orientedGeometricNormal.y,
                                                                         orientedGeometricNormal.z, albedo);
                                        p.walkState[slot] = make_float4(material->subsurfaceWeightScale.z,
                                                                        __uint_as_float(rng), throughput, 0.0f);
                                        // This bounce's extension queue has been traced: it holds the walks.
                                        uint32_t* walks = (bounce & 1u) ? p.queue[1] : p.queue[0];
                                        walks[appendIndex(p.counters + 6)] = slot;
                                    }
                                    deferred = true;
                                    break;
                                }
                                if (kWalk == kWalkReplay) {
                                    // The deferred walk failed; its RNG state after the walk.
                                    rng = __float_as_uint(p.walkState[slot].y);
                                } else if (randomWalkSubsurface(s, p, hit, orientedGeometricNormal, radius, albedo,
                                                                material->subsurfaceWeightScale.z, rng, exitOrigin,
                                                                exitDirection, attenuation)) {
                                    throughput = throughput * attenuation;
                                    rayOrigin = exitOrigin;
                                    rayDirection = exitDirection;
                                    environmentOnMiss = true;
                                    previousWasDelta = true;
                                    previousBsdfPdf = 0.0f;
                                    walked = true;
                                }
                            }
                            if (walked) break;
                            rayDirection = cosineHemisphere(normal, rng);
                            const float lambertResponse = gmax(dot(normal, rayDirection), 0.0f) / kPi;
                            throughput = throughput * (evaluateDiffuseReflection(normal, viewDirection, rayDirection, diffuseColor,
                                                                                 diffuseRoughness, diffuseModel) /
                                                       gmax(lambertResponse, 1e-6f));
                        }
                    }
                }
            }
            if (lightCount > 0u || hasMeshLights) {
                // :1859-1874
                previousBsdfPdf = surfaceReflectionPdf(normal, tangent, viewDirection, rayDirection, roughness, coatRoughness,
                                                       sheenProbability, coatProbability, specularProbability,
                                                       translucentProbability);
                previousWasDelta = false;
                environmentOnMiss = true;
                previousEnvironmentLightPdf =
                    lightCount > 0u ? environmentLightPdf(s, lights, hit, normal, rayDirection, diffuseEnergy,
                                                          specularEnergy + luminance1(coatContribution) + sheenProbability,
                                                          translucentEnergy)
                                    : 0.0f;
            }
            if (bounce >= 2u) {
                // :1875-1879 Russian roulette
                const float survival = clampf(throughput, 0.1f, 0.95f);
                if (randomFloat(rng) > survival) {
                    alive = false;
                    break;
                }
                throughput = throughput / survival;
            }
        } while (false);

        if (!kReplay) p.radiance[slot] = radiance;
        if (deferred || !alive || lastBounce) continue;
        p.rng[slot] = rng;
        p.throughput[slot] = throughput;
        p.flags[slot] = (environmentOnMiss ? kFlagEnvironmentOnMiss : 0u) | (previousWasDelta ? kFlagPreviousWasDelta : 0u) |
                        (insideMedium ? kFlagInsideMedium : 0u) | (kCache ? (flags & kFlagTraining) : 0u);
        p.previousPdf[slot] = make_float2(previousBsdfPdf, previousEnvironmentLightPdf);
        if (insideMedium) p.medium[slot] = make_float4(mediumAbsorption, mediumScattering, mediumAnisotropy, 0.0f);
        p.rayOrigin[slot] = make_float4(rayOrigin.x, rayOrigin.y, rayOrigin.z, 0.0f);
        p.rayDirection[slot] = make_float4(rayDirection.x, rayDirection.y, rayDirection.z, 0.0f);
        if (lodOn) p.cone[slot] = coneKept ? make_float2(coneWidth, cone.y) : make_float2(0.0f, -1.0f);
        nextQueue[appendIndex(nextCount)] = slot;
    }
}

// ---------------------------------------------------------------------------
// walk: the deferred subsurface random walks of one bounce (:1153-1186), a
// traversal kernel of its own instead of up to eight traversals nested in the
// full shade kernel. A walk that exits finishes the bounce as the inline form
// does (the exit ray is the path's next ray; no MIS bookkeeping, no roulette);
// a walk whose boundary ray escapes stores its RNG state and queues the path
// for shadeKernel<..., kWalkReplay>, which finishes the bounce the inline way.
// ---------------------------------------------------------------------------
template <int kInst>
__global__ void __launch_bounds__(128, HDCX_TRACE_MIN_BLOCKS)
    walkKernel(DeviceScene s, PathBuffers p, const uint32_t* walks, uint32_t* nextQueue, uint32_t* nextCount,
               uint32_t* replayQueue)
{
    const uint32_t n = p.counters[6];
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t slot = walks[i];
        const float4 entry = p.walkEntry[slot];
        const float4 outward = p.walkNormal[slot];
        const float4 state = p.walkState[slot];
        uint32_t rng = __float_as_uint(state.y);
        float3 exitOrigin, exitDirection;
        float attenuation;
        if (randomWalkSubsurface<kInst>(s, p, xyz(entry), xyz(outward), entry.w, outward.w, state.x, rng, exitOrigin,
                                 exitDirection, attenuation)) {
            p.rng[slot] = rng;
            p.throughput[slot] = state.z * attenuation;
            p.flags[slot] = kFlagEnvironmentOnMiss | kFlagPreviousWasDelta |
                            (p.flags[slot] & (kFlagInsideMedium | kFlagTraining));
            p.previousPdf[slot] = make_float2(0.0f, p.previousPdf[slot].y);
            p.rayOrigin[slot] = make_float4(exitOrigin.x, exitOrigin.y, exitOrigin.z, 0.0f);
            p.rayDirection[slot] = make_float4(exitDirection.x, exitDirection.y, exitDirection.z, 0.0f);
            if (p.cone != nullptr) p.cone[slot] = make_float2(0.0f, -1.0f);
            nextQueue[appendIndex(nextCount)] = slot;
        } else {
            p.walkState[slot] = make_float4(state.x, __uint_as_float(rng), state.z, 0.0f);
            replayQueue[appendIndex(p.counters + 7)] = slot;
        }
    }
}

// ---------------------------------------------------------------------------
// miss: environment on a miss (vulkan_path_tracer.cpp:1245-1255), the paths
// of extend's miss queue; the same steps as the top of shadeKernel
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128) missKernel(DeviceScene s, FrameConst f, PathBuffers p)
{
    const uint32_t n = p.counters[5];
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t slot = p.missQueue[i];
        float radiance = p.radiance[slot];
        // Light-sample contributions of the previous bounce, in slot order.
        for (uint32_t k = 0; k < 3u; ++k) {
            uint8_t& valid = p.contributionValid[contributionIndex(slot, k)];
            if (valid) {
                radiance += p.contribution[contributionIndex(slot, k)];
                valid = 0;
            }
        }
        const uint32_t flags = p.flags[slot];
        if ((flags & kFlagEnvironmentOnMiss) != 0u) {
            const Spectrum spec = spectrumFromBasis(p.wavelength[slot], p.spectrum[slot]);
            const float2 previousPdf = p.previousPdf[slot];
            const float misWeight =
                (flags & kFlagPreviousWasDelta) != 0u ? 1.0f : powerHeuristic(previousPdf.x, previousPdf.y);
            radiance += p.throughput[slot] * misWeight * illuminantSpectrum(environment(s, f, xyz(p.rayDirection[slot])), spec);
        }
        p.radiance[slot] = radiance;
    }
}

// ---------------------------------------------------------------------------
// shadow: visibility of light samples (vulkan_path_tracer.cpp:855-912)
// ---------------------------------------------------------------------------
template <bool kOpaque, bool kCount, int kInst>
__global__ void __launch_bounds__(128, HDCX_TRACE_MIN_BLOCKS) shadowKernel(DeviceScene s, PathBuffers p)
{
    const uint32_t n = p.counters[2];
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(p.stats + 1, static_cast<unsigned long long>(n));
    constexpr Accept kMode = kOpaque ? Accept::Opaque : Accept::Threshold;
    uint2 work = make_uint2(0u, 0u);
    uint32_t fault = 0u;  // traversal faults of this thread's rays
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        const float4 o = p.shadowOrigin[j];
        const float4 d = p.shadowDirection[j];
        const float4 fct = p.shadowFactors[j];
        const uint32_t slotK = p.shadowSlot[j];
        const uint32_t info = p.shadowInfo[j];
        const uint32_t slot = slotK >> 2, k = slotK & 3u;
        const uint32_t kind = info & 0xffu, lightIndex = info >> 8;
        const float3 origin = xyz(o), direction = xyz(d);
        const float tmax = o.w;
        HitRecord h;
        if (kind == kShadowMesh) {
            const bool occluded = traceRay<kMode, true, kCount, kInst>(s, origin, direction, 0.001f, tmax, 0u, h, fault, &work);
            if (occluded) p.contributionValid[contributionIndex(slot, k)] = 0;
            else p.contribution[contributionIndex(slot, k)] = d.w * fct.x;
            continue;
        }
        const GpuLight& light = s.lights[lightIndex];
        const bool falloff = light.shadow.y >= 0.0f && light.shadow.z > 0.0f;
        float3 visibility = f3(1.0f);
        bool hitSomething;
        float hitDistance = 0.0f;
        if (falloff) {
            hitSomething = traceRay<kMode, false, kCount, kInst>(s, origin, direction, 0.001f, tmax, 0u, h, fault, &work);
            hitDistance = h.t;
        } else {
            hitSomething = traceRay<kMode, true, kCount, kInst>(s, origin, direction, 0.001f, tmax, 0u, h, fault, &work);
        }
        if (hitSomething) {
            float strength = 1.0f;
            if (falloff) {
                const float falloffDistance = gmin(light.shadow.z, gmax(light.shadow.y, 0.0f));
                strength = clampf((light.shadow.y - hitDistance) / gmax(falloffDistance, 1e-6f), 0.0f, 1.0f);
                strength = gpow(strength, gmax(light.shadow.w, 0.0f));
            }
            visibility = mix(f3(1.0f), xyz(light.shadowColor), strength);
        }
        const Spectrum spec = spectrumFromBasis(p.wavelength[slot], p.spectrum[slot]);
        const float sv = reflectanceSpectrum(visibility, spec);
        p.contribution[contributionIndex(slot, k)] = combineShadow(kind, d.w, sv, fct.x, fct.y, fct.z);
    }
    if (fault != 0u) atomicOr(reinterpret_cast<unsigned int*>(p.stats + 7), fault);
    if (kCount) {
        atomicAdd(p.stats + 5, static_cast<unsigned long long>(work.x));
        atomicAdd(p.stats + 6, static_cast<unsigned long long>(work.y));
    }
}

// ---------------------------------------------------------------------------
// accumulate: sensor and per-pixel batch sums (vulkan_path_tracer.cpp:1882-1884)
// ---------------------------------------------------------------------------
__global__ void accumulateKernel(FrameConst f, WaveDesc w, PathBuffers p, float4* batch, double* batchXyz)
{
    const uint32_t local = blockIdx.x * blockDim.x + threadIdx.x;
    if (local >= w.pixels) return;
    const uint32_t pixel = w.pixelBase + local;
    float4 b = batch[pixel];
    double bx = batchXyz[3 * pixel + 0], by = batchXyz[3 * pixel + 1], bz = batchXyz[3 * pixel + 2];
    for (uint32_t sOff = 0; sOff < w.samples; ++sOff) {
        float3 spectral = f3(0.0f);
        double sx = 0.0, sy = 0.0, sz = 0.0;
        for (uint32_t lane = 0; lane < 3u; ++lane) {
            const uint32_t slot = (sOff * w.pixels + local) * 3u + lane;
            float radiance = p.radiance[slot];
            for (uint32_t k = 0; k < 3u; ++k) {
                if (p.contributionValid[contributionIndex(slot, k)]) radiance += p.contribution[contributionIndex(slot, k)];
            }
            const float wavelength = p.wavelength[slot];
            spectral = spectral + spectralSensor(wavelength) * radiance;
            const float3 x = sensorXyz(wavelength);
            sx = __dadd_rn(sx, __dmul_rn(static_cast<double>(x.x), static_cast<double>(radiance)));
            sy = __dadd_rn(sy, __dmul_rn(static_cast<double>(x.y), static_cast<double>(radiance)));
            sz = __dadd_rn(sz, __dmul_rn(static_cast<double>(x.z), static_cast<double>(radiance)));
        }
        b = make_float4(b.x + spectral.x / 3.0f, b.y + spectral.y / 3.0f, b.z + spectral.z / 3.0f, 0.0f);
        bx = __dadd_rn(bx, __ddiv_rn(sx, 3.0));
        by = __dadd_rn(by, __ddiv_rn(sy, 3.0));
        bz = __dadd_rn(bz, __ddiv_rn(sz, 3.0));
    }
    batch[pixel] = b;
    batchXyz[3 * pixel + 0] = bx;
    batchXyz[3 * pixel + 1] = by;
    batchXyz[3 * pixel + 2] = bz;
}

// pixels[index] = vec4((previous * previousWeight + batchRadiance) / totalWeight, 1.0)
// (vulkan_path_tracer.cpp:1886-1890); the FP64 XYZ sums add the batch.
__global__ void finalizeKernel(FrameConst f, FrameBuffers fb)
{
    const uint32_t pixel = blockIdx.x * blockDim.x + threadIdx.x;
    if (pixel >= f.width * f.height) return;
    // A restart (sampleIndex 0) gives the previous mean weight 0; it is not
    // read, so whatever the output buffer held (NaN included) cannot leak in.
    const float4 prev = f.sampleIndex == 0 ? make_float4(0.0f, 0.0f, 0.0f, 0.0f) : fb.rgba[pixel];
    const float4 b = fb.batch[pixel];
    const float previousWeight = u2f(f.sampleIndex);
    const float totalWeight = previousWeight + u2f(f.sampleCount);
    fb.rgba[pixel] = make_float4((prev.x * previousWeight + b.x) / totalWeight, (prev.y * previousWeight + b.y) / totalWeight,
                                 (prev.z * previousWeight + b.z) / totalWeight, 1.0f);
    for (int k = 0; k < 3; ++k) {
        const double base = f.sampleIndex == 0 ? 0.0 : fb.xyz[3 * pixel + k];
        fb.xyz[3 * pixel + k] = __dadd_rn(base, fb.batchXyz[3 * pixel + k]);
    }
}

__global__ void primaryKernel(DeviceScene s, FrameConst f, uint32_t sampleNumber, uint32_t* primitives, float* distances)
{
    const uint32_t pixel = blockIdx.x * blockDim.x + threadIdx.x;
    if (pixel >= f.width * f.height) return;
    const uint32_t px = pixel % f.width, py = pixel / f.width;
    uint32_t rng = hashState(pixel ^ (sampleNumber * 0x9e3779b9u) ^ 0xa511e9b3u);
    const float jx = randomFloat(rng);
    const float jy = randomFloat(rng);
    const float u = (u2f(px) + jx) / u2f(f.width);
    const float v = (u2f(py) + jy) / u2f(f.height);
    const float3 direction = normalize(f.lowerLeft + u * f.horizontal + v * f.vertical - f.origin);
    HitRecord h;
    uint32_t fault = 0u;  // primary hits of hdcx_trace_primary and the AOVs: a fault leaves the pixel a miss
    const bool found = s.opaque ? traceRay<Accept::Opaque, false>(s, f.origin, direction, 0.001f, 10000.0f, rng, h, fault)
                                : traceRay<Accept::Stochastic, false>(s, f.origin, direction, 0.001f, 10000.0f, rng, h, fault);
    primitives[pixel] = found ? h.primitive : kInvalidPrimitive;
    distances[pixel] = found ? h.t : 0.0f;
}

// ---------------------------------------------------------------------------
// radiance-cache mode: predictions into the terminated paths, suffix targets
// of the training paths
// ---------------------------------------------------------------------------
__global__ void cacheApplyKernel(PathBuffers p)
{
    const uint32_t n = p.cache.counters[0];
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        const uint32_t slot = p.cache.querySlot[j];
        p.radiance[slot] += p.throughput[slot] * fmaxf(p.cache.predictions[j], 0.0f);
    }
}

__global__ void cacheTargetsKernel(PathBuffers p)
{
    const uint32_t n = min(p.cache.counters[1], p.cache.trainCapacity);
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const uint32_t slot = p.cache.trainSlot[t];
        float total = p.radiance[slot];
        for (uint32_t k = 0; k < 3u; ++k) {
            if (p.contributionValid[contributionIndex(slot, k)]) total += p.contribution[contributionIndex(slot, k)];
        }
        const uint32_t vertices = min(p.cache.trainVertices[t], kCacheMaxVertices);
        for (uint32_t b = 0; b < vertices; ++b) {
            const uint32_t r = t * kCacheMaxVertices + b;
            const float2 st = p.cache.trainState[r];
            if (!(st.x > 0.0f)) continue;
            const float target = (total - st.y) / st.x;
            if (!(target >= 0.0f && target < 3.0e38f)) continue;
            const uint32_t j = atomicAdd(p.cache.counters + 2, 1u);
            const float4* src = reinterpret_cast<const float4*>(p.cache.trainRecords) + r * 3u;
            float4* dst = reinterpret_cast<float4*>(p.cache.sampleQueries) + static_cast<size_t>(j) * 3u;
            dst[0] = src[0];
            dst[1] = src[1];
            dst[2] = src[2];
            p.cache.sampleTargets[j] = target;
        }
    }
}

int gridFor(uint32_t maxItems, int perSm)
{
    int device = 0, sms = 148;
    cudaGetDevice(&device);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const int blocks = static_cast<int>((static_cast<uint64_t>(maxItems) + 127u) / 128u);
    return std::max(1, std::min(blocks, sms * perSm));
}

std::vector<WaveDesc> planWaves(uint32_t pixels, uint32_t samples, uint64_t capacity)
{
    std::vector<WaveDesc> waves;
    const uint64_t perSample = static_cast<uint64_t>(pixels) * 3u;
    if (perSample <= capacity) {
        const uint32_t k = static_cast<uint32_t>(std::max<uint64_t>(1u, std::min<uint64_t>(samples, capacity / perSample)));
        for (uint32_t s0 = 0; s0 < samples; s0 += k) {
            const uint32_t ks = std::min(k, samples - s0);
            waves.push_back({s0, ks, 0u, pixels, static_cast<uint32_t>(ks * perSample)});
        }
    } else {
        const uint32_t chunk = static_cast<uint32_t>(capacity / 3u);
        for (uint32_t s0 = 0; s0 < samples; ++s0) {
            for (uint32_t p0 = 0; p0 < pixels; p0 += chunk) {
                const uint32_t np = std::min(chunk, pixels - p0);
                waves.push_back({s0, 1u, p0, np, np * 3u});
            }
        }
    }
    return waves;
}

struct EventPair {
    cudaEvent_t start, stop;
    int stage;
};

}  // namespace

void uploadSrgbTable(const float* table256, cudaStream_t stream)
{
    CUDA_OK(cudaMemcpyToSymbolAsync(cSrgbToLinear, table256, 256 * sizeof(float), 0, cudaMemcpyHostToDevice, stream));
}

// ---------------------------------------------------------------------------
// hit sort: the hit queue in material order, so that a shading warp's lanes
// run the same material's code (scenes whose materials take very different
// paths: glass, subsurface walks, cut-out leaves). A counting sort over
// material bins: per-block shared histograms, one global reservation per bin
// and block iteration. Order within a bin is arbitrary; every path's result
// is independent of queue order.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t hitMaterialBin(const DeviceScene& s, const PathBuffers& p, uint32_t slot)
{
    const uint32_t primitive = __float_as_uint(p.hit[slot].y);
    return __ldg(s.triangleMaterials + primitive) % kHitBins;
}

__global__ void __launch_bounds__(256) countHitBinsKernel(DeviceScene s, PathBuffers p)
{
    __shared__ uint32_t histogram[kHitBins];
    for (uint32_t b = threadIdx.x; b < kHitBins; b += blockDim.x) histogram[b] = 0u;
    __syncthreads();
    const uint32_t n = p.counters[4];
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        atomicAdd(&histogram[hitMaterialBin(s, p, p.hitQueue[i])], 1u);
    __syncthreads();
    for (uint32_t b = threadIdx.x; b < kHitBins; b += blockDim.x)
        if (histogram[b] != 0u) atomicAdd(p.hitBins + b, histogram[b]);
}

// Exclusive prefix sum of the bin counts into the cursors (one warp).
__global__ void scanHitBinsKernel(PathBuffers p)
{
    constexpr uint32_t kPerLane = kHitBins / 32u;
    const uint32_t lane = threadIdx.x;
    uint32_t counts[kPerLane];
    uint32_t local = 0u;
    for (uint32_t k = 0; k < kPerLane; ++k) {
        counts[k] = p.hitBins[lane * kPerLane + k];
        local += counts[k];
    }
    uint32_t inclusive = local;
    for (uint32_t d = 1; d < 32u; d <<= 1) {
        const uint32_t v = __shfl_up_sync(0xffffffffu, inclusive, d);
        if (lane >= d) inclusive += v;
    }
    uint32_t offset = inclusive - local;
    for (uint32_t k = 0; k < kPerLane; ++k) {
        p.hitBins[kHitBins + lane * kPerLane + k] = offset;
        offset += counts[k];
    }
}

__global__ void __launch_bounds__(256) scatterHitsKernel(DeviceScene s, PathBuffers p)
{
    __shared__ uint32_t histogram[kHitBins];
    __shared__ uint32_t start[kHitBins];
    const uint32_t n = p.counters[4];
    // The loop bound is the same for every thread of the block (base is
    // per block), so the barriers inside are reached by all of them.
    for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
        for (uint32_t b = threadIdx.x; b < kHitBins; b += blockDim.x) histogram[b] = 0u;
        __syncthreads();
        const uint32_t i = base + threadIdx.x;
        const bool valid = i < n;
        const uint32_t slot = valid ? p.hitQueue[i] : 0u;
        const uint32_t bin = valid ? hitMaterialBin(s, p, slot) : 0u;
        const uint32_t rank = valid ? atomicAdd(&histogram[bin], 1u) : 0u;
        __syncthreads();
        for (uint32_t b = threadIdx.x; b < kHitBins; b += blockDim.x)
            if (histogram[b] != 0u) start[b] = atomicAdd(p.hitBins + kHitBins + b, histogram[b]);
        __syncthreads();
        if (valid) p.sortedHits[start[bin] + rank] = slot;
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// ray sort (tuning knob sort_rays): secondary extension rays are reordered
// within chunks of kRayChunk queue entries by a direction cell, so that a
// warp traces rays of similar direction. The queue's own order already keeps
// rays of nearby pixels, and so of nearby origins, close together: sorting
// within a chunk keeps that and adds directional coherence, with no global
// pass. Order within a cell is arbitrary; every path's result is independent
// of queue order.
// ---------------------------------------------------------------------------
constexpr uint32_t kRayChunk = 1024;  // queue entries per block iteration (256 threads x 4)
constexpr uint32_t kRayCells = 128;   // 6 cube faces x 4 x 4 cells (96 used)

__device__ __forceinline__ uint32_t directionCell(float4 d)
{
    const float ax = fabsf(d.x), ay = fabsf(d.y), az = fabsf(d.z);
    uint32_t face;
    float u, v, m;
    if (ax >= ay && ax >= az) {
        face = d.x < 0.0f ? 1u : 0u;
        u = d.y;
        v = d.z;
        m = ax;
    } else if (ay >= az) {
        face = d.y < 0.0f ? 3u : 2u;
        u = d.x;
        v = d.z;
        m = ay;
    } else {
        face = d.z < 0.0f ? 5u : 4u;
        u = d.x;
        v = d.y;
        m = az;
    }
    const float inv = m > 0.0f ? 2.0f / m : 0.0f;  // (u/m + 1) * 2 in [0, 4]
    const uint32_t cu = min(static_cast<uint32_t>(fmaxf(fmaf(u, inv, 2.0f), 0.0f)), 3u);
    const uint32_t cv = min(static_cast<uint32_t>(fmaxf(fmaf(v, inv, 2.0f), 0.0f)), 3u);
    return face * 16u + cu * 4u + cv;
}

__global__ void __launch_bounds__(256) sortRaysKernel(PathBuffers p, uint32_t* queue, const uint32_t* count)
{
    __shared__ uint32_t cursor[kRayCells];
    __shared__ uint32_t sorted[kRayChunk];
    const uint32_t n = *count;
    constexpr uint32_t kPer = kRayChunk / 256u;
    // The loop bound is the same for every thread of the block, so the
    // barriers inside are reached by all of them.
    for (uint32_t base = blockIdx.x * kRayChunk; base < n; base += gridDim.x * kRayChunk) {
        if (threadIdx.x < kRayCells) cursor[threadIdx.x] = 0u;
        __syncthreads();
        uint32_t slot[kPer], cell[kPer], rank[kPer];
#pragma unroll
        for (uint32_t k = 0; k < kPer; ++k) {
            const uint32_t i = base + k * 256u + threadIdx.x;
            slot[k] = i < n ? queue[i] : 0u;
            cell[k] = i < n ? directionCell(p.rayDirection[slot[k]]) : 0u;
            rank[k] = i < n ? atomicAdd(&cursor[cell[k]], 1u) : 0u;
        }
        __syncthreads();
        if (threadIdx.x < 32u) {
            // Exclusive prefix sum of the cell counts, four cells per lane.
            const uint32_t lane = threadIdx.x;
            uint32_t c[4], local = 0u;
#pragma unroll
            for (uint32_t k = 0; k < 4u; ++k) {
                c[k] = cursor[lane * 4u + k];
                local += c[k];
            }
            uint32_t inclusive = local;
#pragma unroll
            for (uint32_t d = 1; d < 32u; d <<= 1) {
                const uint32_t v = __shfl_up_sync(0xffffffffu, inclusive, d);
                if (lane >= d) inclusive += v;
            }
            uint32_t offset = inclusive - local;
#pragma unroll
            for (uint32_t k = 0; k < 4u; ++k) {
                cursor[lane * 4u + k] = offset;
                offset += c[k];
            }
        }
        __syncthreads();
#pragma unroll
        for (uint32_t k = 0; k < kPer; ++k) {
            if (base + k * 256u + threadIdx.x < n) sorted[cursor[cell[k]] + rank[k]] = slot[k];
        }
        __syncthreads();
#pragma unroll
        for (uint32_t k = 0; k < kPer; ++k) {
            const uint32_t i = base + k * 256u + threadIdx.x;
            if (i < n) queue[i] = sorted[k * 256u + threadIdx.x];
        }
        __syncthreads();
    }
}

template <int kInst>
void launchExtend(const DeviceScene& scene, PathBuffers& paths, const uint32_t* inQueue, const uint32_t* inCount,
                  bool count, int grid, cudaStream_t stream)
{
    if (count) {
        if (scene.opaque) extendKernel<Accept::Opaque, true, kInst><<<grid, 128, 0, stream>>>(scene, paths, inQueue, inCount);
        else extendKernel<Accept::Stochastic, true, kInst><<<grid, 128, 0, stream>>>(scene, paths, inQueue, inCount);
    } else {
        if (scene.opaque) extendKernel<Accept::Opaque, false, kInst><<<grid, 128, 0, stream>>>(scene, paths, inQueue, inCount);
        else extendKernel<Accept::Stochastic, false, kInst><<<grid, 128, 0, stream>>>(scene, paths, inQueue, inCount);
    }
}

template <int kInst>
void launchShadow(const DeviceScene& scene, PathBuffers& paths, bool count, int grid, cudaStream_t stream)
{
    if (count) {
        if (scene.opaque) shadowKernel<true, true, kInst><<<grid, 128, 0, stream>>>(scene, paths);
        else shadowKernel<false, true, kInst><<<grid, 128, 0, stream>>>(scene, paths);
    } else {
        if (scene.opaque) shadowKernel<true, false, kInst><<<grid, 128, 0, stream>>>(scene, paths);
        else shadowKernel<false, false, kInst><<<grid, 128, 0, stream>>>(scene, paths);
    }
}

// Whether the full shade kernels defer subsurface walks to walkKernel: path
// buffers with walk buffers (plain and radiance-cache mode alike).
bool deferWalks(const PathBuffers& paths)
{
    return paths.walkEntry != nullptr && paths.walkNormal != nullptr && paths.walkState != nullptr;
}

template <bool kCache>
void launchShade(const DeviceScene& scene, const FrameConst& frame, PathBuffers& paths, uint32_t bounce, const uint32_t* inQueue,
                 const uint32_t* inCount, uint32_t* outQueue, uint32_t* outCount, int grid, cudaStream_t stream)
{
    const bool lit = scene.lightCount > 0u && !scene.hasMeshLights;
    if (scene.fullShading) {
        if (deferWalks(paths)) {
            if (lit) shadeKernel<true, true, kCache, kWalkDefer><<<grid, 128, 0, stream>>>(scene, frame, paths, bounce, inQueue, inCount, outQueue, outCount);
            else shadeKernel<true, false, kCache, kWalkDefer><<<grid, 128, 0, stream>>>(scene, frame, paths, bounce, inQueue, inCount, outQueue, outCount);
        } else if (lit) {
            shadeKernel<true, true, kCache><<<grid, 128, 0, stream>>>(scene, frame, paths, bounce, inQueue, inCount, outQueue, outCount);
        } else {
            shadeKernel<true, false, kCache><<<grid, 128, 0, stream>>>(scene, frame, paths, bounce, inQueue, inCount, outQueue, outCount);
        }
    } else {
        if (lit) shadeKernel<false, true, kCache><<<grid, 128, 0, stream>>>(scene, frame, paths, bounce, inQueue, inCount, outQueue, outCount);
        else shadeKernel<false, false, kCache><<<grid, 128, 0, stream>>>(scene, frame, paths, bounce, inQueue, inCount, outQueue, outCount);
    }
}

void renderFrame(const DeviceScene& sceneIn, const FrameConst& frame, PathBuffers& paths, FrameBuffers& fb,
                 cudaStream_t stream, StageTimes* timing, bool countTraversal, uint64_t* launches, CacheRun* cacheRun)
{
    const DeviceScene& scene = sceneIn;
    const bool cacheMode = cacheRun != nullptr && cacheRun->cache != nullptr && paths.cache.enabled != 0u;
    if (!cacheMode) paths.cache.enabled = 0u;
    uint64_t launched = 0;
    const uint32_t pixels = frame.width * frame.height;
    CUDA_OK(cudaMemsetAsync(fb.batch, 0, sizeof(float4) * pixels, stream));
    CUDA_OK(cudaMemsetAsync(fb.batchXyz, 0, sizeof(double) * 3u * pixels, stream));
    const uint64_t wavePaths = paths.wavePaths ? std::min(paths.wavePaths, paths.capacity) : paths.capacity;
    const std::vector<WaveDesc> waves = planWaves(pixels, std::max(frame.sampleCount, 1u), wavePaths);
    const int traceGrid = gridFor(static_cast<uint32_t>(wavePaths), static_cast<int>(std::max(paths.traceBlocksPerSm, 1u)));
    const int shadeGrid = gridFor(static_cast<uint32_t>(wavePaths), static_cast<int>(std::max(paths.shadeBlocksPerSm, 1u)));
    const int missGrid = gridFor(static_cast<uint32_t>(wavePaths), 8);
    const bool sortHits = paths.sortHits != 0u && paths.sortedHits != nullptr && paths.hitBins != nullptr;
    const bool sortRays = paths.sortRays != 0u;
    // Subsurface walks in walkKernel (scenes that can take them).
    const bool walks = scene.fullShading && scene.hasSubsurface && deferWalks(paths);
    const int sortGrid = std::max(1, gridFor(static_cast<uint32_t>(wavePaths), 8) / 2);  // 256-thread blocks
    std::vector<EventPair> events;
    auto timed = [&](int stage, auto&& launch) {
        if (!timing) {
            launch();
            return;
        }
        EventPair e{};
        e.stage = stage;
        CUDA_OK(cudaEventCreate(&e.start));
        CUDA_OK(cudaEventCreate(&e.stop));
        CUDA_OK(cudaEventRecord(e.start, stream));
        launch();
        CUDA_OK(cudaEventRecord(e.stop, stream));
        events.push_back(e);
    };
    for (const WaveDesc& w : waves) {
        NvtxRange waveRange("hdcx wave");
        if (cacheMode) CUDA_OK(cudaMemsetAsync(paths.cache.counters, 0, 3 * sizeof(uint32_t), stream));
        generateKernel<<<(w.count + 255u) / 256u, 256, 0, stream>>>(frame, w, paths);
        CUDA_OK(cudaGetLastError());
        for (uint32_t bounce = 0; bounce < frame.maxBounces; ++bounce) {
            uint32_t* inQueue = paths.queue[bounce & 1u];
            uint32_t* outQueue = paths.queue[(bounce + 1u) & 1u];
            uint32_t* inCount = paths.counters + (bounce & 1u);
            uint32_t* outCount = paths.counters + ((bounce + 1u) & 1u);
            CUDA_OK(cudaMemsetAsync(paths.counters + 4, 0, 4 * sizeof(uint32_t), stream));
            if (sortRays && bounce > 0u) {
                sortRaysKernel<<<sortGrid, 256, 0, stream>>>(paths, inQueue, inCount);
                launched += 1;
            }
            timed(0, [&] {
                if (scene.instances) launchExtend<1>(scene, paths, inQueue, inCount, countTraversal, traceGrid, stream);
                else launchExtend<0>(scene, paths, inQueue, inCount, countTraversal, traceGrid, stream);
            });
            CUDA_OK(cudaGetLastError());
            CUDA_OK(cudaMemsetAsync(outCount, 0, sizeof(uint32_t), stream));
            CUDA_OK(cudaMemsetAsync(paths.counters + 2, 0, sizeof(uint32_t), stream));
            timed(1, [&] {
                const uint32_t* hits = paths.hitQueue;
                if (sortHits) {
                    CUDA_OK(cudaMemsetAsync(paths.hitBins, 0, 2 * kHitBins * sizeof(uint32_t), stream));
                    countHitBinsKernel<<<sortGrid, 256, 0, stream>>>(scene, paths);
                    scanHitBinsKernel<<<1, 32, 0, stream>>>(paths);
                    scatterHitsKernel<<<sortGrid, 256, 0, stream>>>(scene, paths);
                    hits = paths.sortedHits;
                }
                if (cacheMode) launchShade<true>(scene, frame, paths, bounce, hits, paths.counters + 4, outQueue, outCount, shadeGrid, stream);
                else launchShade<false>(scene, frame, paths, bounce, hits, paths.counters + 4, outQueue, outCount, shadeGrid, stream);
                missKernel<<<missGrid, 128, 0, stream>>>(scene, frame, paths);
                if (walks) {
                    // The deferred walks (in this bounce's traced extension
                    // queue), then the failed ones re-shaded (queued in the
                    // miss queue, which missKernel has consumed).
                    if (scene.instances) walkKernel<1><<<traceGrid, 128, 0, stream>>>(scene, paths, inQueue, outQueue, outCount, paths.missQueue);
                    else walkKernel<0><<<traceGrid, 128, 0, stream>>>(scene, paths, inQueue, outQueue, outCount, paths.missQueue);
                    const bool lit = scene.lightCount > 0u && !scene.hasMeshLights;
                    const uint32_t* replays = paths.missQueue;
                    const uint32_t* replayCount = paths.counters + 7;
                    if (cacheMode) {
                        if (lit) shadeKernel<true, true, true, kWalkReplay><<<missGrid, 128, 0, stream>>>(scene, frame, paths, bounce, replays, replayCount, outQueue, outCount);
                        else shadeKernel<true, false, true, kWalkReplay><<<missGrid, 128, 0, stream>>>(scene, frame, paths, bounce, replays, replayCount, outQueue, outCount);
                    } else {
                        if (lit) shadeKernel<true, true, false, kWalkReplay><<<missGrid, 128, 0, stream>>>(scene, frame, paths, bounce, replays, replayCount, outQueue, outCount);
                        else shadeKernel<true, false, false, kWalkReplay><<<missGrid, 128, 0, stream>>>(scene, frame, paths, bounce, replays, replayCount, outQueue, outCount);
                    }
                }
            });
            CUDA_OK(cudaGetLastError());
            timed(2, [&] {
                if (scene.instances) launchShadow<1>(scene, paths, countTraversal, traceGrid, stream);
                else launchShadow<0>(scene, paths, countTraversal, traceGrid, stream);
            });
            CUDA_OK(cudaGetLastError());
            launched += (sortHits ? 7 : 4) + (walks ? 2 : 0);
        }
        if (cacheMode) {
            // Predictions for the terminated paths, then one training round on
            // this wave's suffix samples (the next wave sees the update).
            uint32_t counts[3] = {0, 0, 0};
            CUDA_OK(cudaMemcpyAsync(counts, paths.cache.counters, sizeof counts, cudaMemcpyDeviceToHost, stream));
            CUDA_OK(cudaStreamSynchronize(stream));
            nrc::query(cacheRun->cache, paths.cache.queries, counts[0], paths.cache.predictions, stream);
            cacheApplyKernel<<<gridFor(std::max(counts[0], 1u), 8), 128, 0, stream>>>(paths);
            cacheTargetsKernel<<<gridFor(std::max(std::min(counts[1], paths.cache.trainCapacity), 1u), 8), 128, 0, stream>>>(paths);
            CUDA_OK(cudaGetLastError());
            CUDA_OK(cudaMemcpyAsync(counts, paths.cache.counters, sizeof counts, cudaMemcpyDeviceToHost, stream));
            CUDA_OK(cudaStreamSynchronize(stream));
            cacheRun->queries += counts[0];
            cacheRun->samples += counts[2];
            if (counts[2] > 0u) {
                cacheRun->lastLoss = nrc::train(cacheRun->cache, paths.cache.sampleQueries, paths.cache.sampleTargets, counts[2],
                                                cacheRun->trainSteps, stream);
            }
            launched += 2;
        }
        launched += 2;
        accumulateKernel<<<(w.pixels + 255u) / 256u, 256, 0, stream>>>(frame, w, paths, fb.batch, fb.batchXyz);
        CUDA_OK(cudaGetLastError());
    }
    finalizeKernel<<<(pixels + 255u) / 256u, 256, 0, stream>>>(frame, fb);
    CUDA_OK(cudaGetLastError());
    launched += 1;
    if (launches) *launches = launched;
    if (timing) {
        CUDA_OK(cudaStreamSynchronize(stream));
        timing->waves = static_cast<uint32_t>(waves.size());
        for (EventPair& e : events) {
            float ms = 0.0f;
            CUDA_OK(cudaEventElapsedTime(&ms, e.start, e.stop));
            if (e.stage == 0) {
                timing->extendMs += ms;
                timing->extendLaunches++;
            } else if (e.stage == 1) {
                timing->shadeMs += ms;
            } else {
                timing->shadowMs += ms;
            }
            cudaEventDestroy(e.start);
            cudaEventDestroy(e.stop);
        }
    }
}

__global__ void upscaleNearestKernel(const float4* src, uint32_t srcWidth, uint32_t srcHeight, float4* dst,
                                     uint32_t width, uint32_t height)
{
    const uint64_t pixel = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (pixel >= uint64_t(width) * height) return;
    const uint32_t x = static_cast<uint32_t>(pixel % width), y = static_cast<uint32_t>(pixel / width);
    // render_pass.cpp:55-60: source = min(size - 1, destination * size / destinationSize).
    const uint32_t sy = static_cast<uint32_t>(min(uint64_t(srcHeight - 1u), uint64_t(y) * srcHeight / height));
    const uint32_t sx = static_cast<uint32_t>(min(uint64_t(srcWidth - 1u), uint64_t(x) * srcWidth / width));
    dst[pixel] = src[uint64_t(sy) * srcWidth + sx];
}

void launchUpscaleNearest(const float4* src, uint32_t srcWidth, uint32_t srcHeight, float4* dst, uint32_t width,
                          uint32_t height, cudaStream_t stream)
{
    const uint64_t pixels = uint64_t(width) * height;
    if (pixels == 0 || srcWidth == 0 || srcHeight == 0) return;
    upscaleNearestKernel<<<static_cast<unsigned>((pixels + 255u) / 256u), 256, 0, stream>>>(src, srcWidth, srcHeight, dst,
                                                                                          width, height);
    CUDA_OK(cudaGetLastError());
}

// One level of a texture's mip pyramid: each texel the mean of the 2x2
// texels below it (the last row / column reused for odd sizes), level 0
// decoded to linear RGBA (sRGB through the sampler's table).
__global__ void mipLevelKernel(TexDesc t, const float4* below, uint32_t bw, uint32_t bh, float4* out, uint32_t w, uint32_t h)
{
    const uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= uint64_t(w) * h) return;
    const uint32_t x = static_cast<uint32_t>(i % w), y = static_cast<uint32_t>(i / w);
    const uint32_t x0 = min(2u * x, bw - 1u), x1 = min(2u * x + 1u, bw - 1u);
    const uint32_t y0 = min(2u * y, bh - 1u), y1 = min(2u * y + 1u, bh - 1u);
    float4 a, b, c, d;
    if (below == nullptr) {
        a = texelFetch(t, static_cast<int>(x0), static_cast<int>(y0));
        b = texelFetch(t, static_cast<int>(x1), static_cast<int>(y0));
        c = texelFetch(t, static_cast<int>(x0), static_cast<int>(y1));
        d = texelFetch(t, static_cast<int>(x1), static_cast<int>(y1));
    } else {
        a = below[size_t(y0) * bw + x0];
        b = below[size_t(y0) * bw + x1];
        c = below[size_t(y1) * bw + x0];
        d = below[size_t(y1) * bw + x1];
    }
    out[i] = make_float4(((a.x + b.x) + (c.x + d.x)) * 0.25f, ((a.y + b.y) + (c.y + d.y)) * 0.25f,
                         ((a.z + b.z) + (c.z + d.z)) * 0.25f, ((a.w + b.w) + (c.w + d.w)) * 0.25f);
}

uint64_t mipTexels(uint32_t width, uint32_t height, uint32_t& levels)
{
    uint64_t total = 0;
    levels = 1;
    uint32_t w = width, h = height;
    while (w > 1u || h > 1u) {
        w = std::max(1u, w >> 1);
        h = std::max(1u, h >> 1);
        total += uint64_t(w) * h;
        ++levels;
    }
    return total;
}

void buildMips(TexDesc& desc, float4* mips, cudaStream_t stream)
{
    uint32_t levels = 1;
    mipTexels(desc.width, desc.height, levels);
    uint32_t bw = desc.width, bh = desc.height;
    const float4* below = nullptr;
    float4* out = mips;
    for (uint32_t k = 1; k < levels; ++k) {
        const uint32_t w = std::max(1u, bw >> 1), h = std::max(1u, bh >> 1);
        const uint64_t n = uint64_t(w) * h;
        mipLevelKernel<<<static_cast<unsigned>((n + 255u) / 256u), 256, 0, stream>>>(desc, below, bw, bh, out, w, h);
        CUDA_OK(cudaGetLastError());
        below = out;
        out += n;
        bw = w;
        bh = h;
    }
    desc.mips = mips;
    desc.levels = levels;
}

void tracePrimary(const DeviceScene& scene, const FrameConst& frame, uint32_t sampleNumber, uint32_t* primitives,
                  float* distances, cudaStream_t stream)
{
    const uint32_t pixels = frame.width * frame.height;
    primaryKernel<<<(pixels + 127u) / 128u, 128, 0, stream>>>(scene, frame, sampleNumber, primitives, distances);
    CUDA_OK(cudaGetLastError());
}

}  // namespace hdcx
