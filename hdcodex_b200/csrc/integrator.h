// integrator.h - host interface of the wavefront integrator.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "device/common.cuh"

namespace hdcx {

// Radiance-cache mode (device side): paths that are not training paths stop
// at the first surface vertex after `prefixBounces` bounces and record a cache
// query there; a sparse, deterministic set of training paths runs the full
// bounce budget and records every vertex (query features, throughput and
// radiance on arrival) for the suffix targets.
constexpr uint32_t kCacheMaxVertices = 12;  // HDCX_MAX_PATH_BOUNCES
struct CacheDevice {
    uint32_t enabled = 0;
    uint32_t prefixBounces = 2;   // paths end at this bounce at the latest
    float spreadFactor = 0.0f;    // > 0: also end once the path's spread exceeds it x the primary footprint
    float2* spread = nullptr;     // per path: primary footprint a0, sum of sqrt spread terms
    uint32_t trainThreshold = 0;  // a path trains when its identity hash < this
    uint32_t trainCapacity = 0;   // training paths per wave
    float3 sceneMin{};            // query positions are (hit - sceneMin) * sceneScale, in [0, 1]
    float3 sceneScale{};
    float* queries = nullptr;          // wave capacity x 12: termination queries
    uint32_t* querySlot = nullptr;     // path slot of each query
    uint32_t* trainIndex = nullptr;    // per path: its training record block
    uint32_t* trainSlot = nullptr;     // per training path: its path slot
    uint32_t* trainVertices = nullptr; // per training path: vertices recorded
    float* trainRecords = nullptr;     // trainCapacity x kCacheMaxVertices x 12
    float2* trainState = nullptr;      // (throughput, radiance) on arrival at each recorded vertex
    float* sampleQueries = nullptr;    // compacted training batch: trainCapacity x kCacheMaxVertices x 12
    float* sampleTargets = nullptr;
    float* predictions = nullptr;      // wave capacity
    uint32_t* counters = nullptr;      // [0] queries, [1] training paths, [2] training samples
};

// Material bins of the hit sort (material index modulo kHitBins).
constexpr uint32_t kHitBins = 256;

// Device buffers of one wave of paths (structure of arrays, 16-byte records).
struct PathBuffers {
    uint64_t capacity = 0;          // paths the buffers hold (the stride of the per-slot arrays)
    uint64_t wavePaths = 0;         // paths per wave, at most capacity (0: capacity)
    uint32_t shadowPerPath = 0;     // shadow-ray slots per path per bounce
    uint32_t* rng = nullptr;
    float* wavelength = nullptr;
    float4* spectrum = nullptr;     // basis r, g, b and Planck factor of the lane
    float* throughput = nullptr;
    float* radiance = nullptr;
    float4* rayOrigin = nullptr;
    float4* rayDirection = nullptr;
    uint32_t* flags = nullptr;
    float2* previousPdf = nullptr;  // previousBsdfPdf, previousEnvironmentLightPdf
    float4* medium = nullptr;       // absorption, scattering, anisotropy
    float4* hit = nullptr;          // t, primitive (bits), b1, b2
    float* contribution = nullptr;  // 3 * capacity: path slot s, light-sample slot k at 3 s + k
    uint8_t* contributionValid = nullptr;  // same indexing as contribution
    uint32_t* queue[2] = {nullptr, nullptr};
    uint32_t* hitQueue = nullptr;       // extend's output: paths whose ray hit (shaded)
    uint32_t* missQueue = nullptr;      // extend's output: paths whose ray missed (environment)
    float4* shadowOrigin = nullptr;     // xyz, tmax
    float4* shadowDirection = nullptr;  // xyz, partial product
    float4* shadowFactors = nullptr;    // f1, f2, f3
    uint32_t* shadowSlot = nullptr;     // path slot * 4 + k
    uint32_t* shadowInfo = nullptr;     // kind | light << 8
    // [0], [1] extension queues, [2] shadow queue, [4] hits, [5] misses,
    // [6] deferred subsurface walks, [7] failed walks to re-shade (8 entries)
    uint32_t* counters = nullptr;
    // extension, shadow, subsurface rays; extension node visits and triangle
    // tests; shadow node visits and triangle tests (counting mode)
    unsigned long long* stats = nullptr;
    CacheDevice cache;
    // Launch shape (host side): blocks of 128 threads per SM of the traversal
    // and shade kernels (the autotuner's knobs; results do not depend on them).
    uint32_t traceBlocksPerSm = 16;
    uint32_t shadeBlocksPerSm = 8;
    // Hits shaded in material order (sortHits = 1): the hit queue is counted
    // and scattered into sortedHits by material bin; hitBins holds the bins'
    // counts, then their cursors (2 x kHitBins).
    uint32_t sortHits = 0;
    uint32_t* sortedHits = nullptr;
    uint32_t* hitBins = nullptr;
    // Secondary extension rays traced in direction order (sortRays = 1): each
    // chunk of 1024 queue entries is sorted in place by a direction cell.
    uint32_t sortRays = 0;
    // Deferred subsurface walks (all three set, else walks run inside the
    // shade kernel): per path slot, the walk's entry point and mean free path,
    // outward normal and albedo, and (anisotropy, RNG state, throughput).
    float4* walkEntry = nullptr;
    float4* walkNormal = nullptr;
    float4* walkState = nullptr;
    // Texture LOD: per path the ray cone (width at the last vertex, spread
    // angle; spread <= 0 once the cone is no longer tracked). Null: no LOD.
    float2* cone = nullptr;
};

// Per-pixel accumulation buffers of the current output size.
struct FrameBuffers {
    uint32_t width = 0, height = 0;
    float4* rgba = nullptr;        // running mean (the reference's output buffer)
    double* xyz = nullptr;         // FP64 XYZ sums, 3 per pixel
    float4* batch = nullptr;       // batchRadiance of the current render
    double* batchXyz = nullptr;    // FP64 XYZ of the current render, 3 per pixel
};

struct StageTimes {
    double extendMs = 0, shadeMs = 0, shadowMs = 0;
    uint32_t waves = 0;
    uint32_t extendLaunches = 0;
};

void uploadSrgbTable(const float* table256, cudaStream_t stream);

// Renders sampleCount samples per pixel into fb (running mean update).
// `timing` non-null records per-stage device times with CUDA events.
// countTraversal selects the traversal kernels that count node visits and
// triangle tests (into paths.stats[3..6]); *launches gets the kernel count.
namespace nrc {
struct Cache;
}

// Host side of the radiance-cache mode: the cache and its training schedule.
struct CacheRun {
    nrc::Cache* cache = nullptr;
    uint32_t trainSteps = 1;  // Adam steps per wave on the wave's suffix samples
    float lastLoss = 0.0f;
    uint64_t queries = 0, samples = 0;
};

void renderFrame(const DeviceScene& scene, const FrameConst& frame, PathBuffers& paths, FrameBuffers& fb,
                 cudaStream_t stream, StageTimes* timing, bool countTraversal, uint64_t* launches,
                 CacheRun* cacheRun = nullptr);

// dst (width x height) = src (srcWidth x srcHeight) upscaled by nearest
// neighbour: the reference's UpscaleNearest (render_pass.cpp:45-68).
void launchUpscaleNearest(const float4* src, uint32_t srcWidth, uint32_t srcHeight, float4* dst, uint32_t width,
                          uint32_t height, cudaStream_t stream);

// Texels of the mip levels 1.. of a width x height texture (`levels` gets
// the level count, level 0 included).
uint64_t mipTexels(uint32_t width, uint32_t height, uint32_t& levels);
// Builds the mip pyramid of `desc` into `mips` (mipTexels float4) on
// `stream` and records it in desc.mips / desc.levels.
void buildMips(TexDesc& desc, float4* mips, cudaStream_t stream);

// Primary-hit ids and distances of sample `sampleNumber` (device outputs).
void tracePrimary(const DeviceScene& scene, const FrameConst& frame, uint32_t sampleNumber, uint32_t* primitives,
                  float* distances, cudaStream_t stream);

}  // namespace hdcx
