// hdcx_api.cpp - the C ABI of include/hdcx.h.
//
// One hdcx_tracer owns everything the reference's VulkanPathTracer::Impl owns
// (vulkan_path_tracer.cpp:2082-3346): the device scene (flattened buffers,
// textures, the BVH), the RGBA32F running-mean buffer of the last render size
// and the fallback up axis fixed by its first render. Every entry point turns
// exceptions and CUDA errors into a status code plus hdcx_last_error().
#include "hdcx.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstddef>
#include <memory>
#include <mutex>
#include <cmath>
#include <cstring>
#include <new>
#include <stdexcept>
#include <string>
#include <vector>

#include "batch_plan.h"
#include "bvh_build.h"
#include "device_memory.h"
#include "integrator.h"
#include "nrc.h"
#include "nvtx_range.h"
#include "render_static.h"
#include "scene_pack.h"

namespace {

using namespace hdcx;

struct StatusError : std::runtime_error {
    hdcx_status status;
    StatusError(hdcx_status s, const std::string& m) : std::runtime_error(m), status(s) {}
};

void check(cudaError_t e, const char* what)
{
    if (e == cudaSuccess) return;
    const hdcx_status s = e == cudaErrorMemoryAllocation ? HDCX_ERROR_OUT_OF_MEMORY : HDCX_ERROR_CUDA;
    throw StatusError(s, std::string(what) + ": " + cudaGetErrorString(e));
}

// Device allocation tracked by the tracer.
struct DeviceBuffer {
    void* ptr = nullptr;
    size_t bytes = 0;
    DeviceBuffer() = default;
    DeviceBuffer(const DeviceBuffer&) = delete;
    DeviceBuffer& operator=(const DeviceBuffer&) = delete;
    ~DeviceBuffer() { reset(); }
    void reset()
    {
        deviceFree(ptr);
        ptr = nullptr;
        bytes = 0;
    }
    void allocate(size_t n)
    {
        reset();
        ptr = deviceMalloc(n);
        bytes = n;
    }
    template <typename T>
    T* as() const
    {
        return static_cast<T*>(ptr);
    }
};

// Path state of one wave of up to paths.capacity paths and the device
// buffers behind it.
struct PathStore {
    std::vector<DeviceBuffer*> buffers;
    PathBuffers paths;
    PathStore() = default;
    PathStore(const PathStore&) = delete;
    PathStore& operator=(const PathStore&) = delete;
    ~PathStore() { release(); }
    void release()
    {
        for (DeviceBuffer* b : buffers) delete b;
        buffers.clear();
        paths = PathBuffers{};
    }
    template <typename T>
    T* alloc(size_t count)
    {
        auto* b = new DeviceBuffer();
        buffers.push_back(b);
        b->allocate(count * sizeof(T));
        return b->as<T>();
    }
    // Replaces the buffers by buffers of `n` paths; the GPU must be done with the old ones.
    void allocate(uint64_t n, uint32_t shadowPerPath)
    {
        release();
        PathBuffers& p = paths;
        const uint64_t ns = n * shadowPerPath;
        p.capacity = n;
        p.wavePaths = n;
        p.shadowPerPath = shadowPerPath;
        p.rng = alloc<uint32_t>(n);
        p.wavelength = alloc<float>(n);
        p.spectrum = alloc<float4>(n);
        p.throughput = alloc<float>(n);
        p.radiance = alloc<float>(n);
        p.rayOrigin = alloc<float4>(n);
        p.rayDirection = alloc<float4>(n);
        p.flags = alloc<uint32_t>(n);
        p.previousPdf = alloc<float2>(n);
        p.medium = alloc<float4>(n);
        p.hit = alloc<float4>(n);
        p.contribution = alloc<float>(3 * n);
        p.contributionValid = alloc<uint8_t>(3 * n);
        p.queue[0] = alloc<uint32_t>(n);
        p.queue[1] = alloc<uint32_t>(n);
        p.hitQueue = alloc<uint32_t>(n);
        p.missQueue = alloc<uint32_t>(n);
        p.shadowOrigin = alloc<float4>(ns);
        p.shadowDirection = alloc<float4>(ns);
        p.shadowFactors = alloc<float4>(ns);
        p.shadowSlot = alloc<uint32_t>(ns);
        p.shadowInfo = alloc<uint32_t>(ns);
        p.counters = alloc<uint32_t>(8);
        p.sortedHits = alloc<uint32_t>(n);
        p.hitBins = alloc<uint32_t>(2 * kHitBins);
        p.walkEntry = alloc<float4>(n);
        p.walkNormal = alloc<float4>(n);
        p.walkState = alloc<float4>(n);
        p.cone = alloc<float2>(n);
    }
};

// ---------------------------------------------------------------------------
// Path arenas
//
// A render needs the path state of its waves (about 359 bytes per path) only
// while it runs, so path state belongs to a per-device pool of arenas rather
// than to tracers: hdcx_render and hdcx_autotune check an arena out for the
// call, hdcx_render_batch one per lane until the batch's work has finished.
// Many tracers on one device then share a few large buffers instead of each
// holding its own. An arena grows to the largest wave asked of it and keeps
// its buffers until the last tracer of its device is destroyed. A device has
// at most kMaxArenas arenas; a render that finds them all busy waits for one.
// (A tracer in radiance-cache mode renders on path buffers of its own, sized
// together with its cache buffers.)
// ---------------------------------------------------------------------------
constexpr int kArenaDevices = 64;
constexpr size_t kMaxArenas = 8;

struct PathArena {
    std::mutex busy;  // held by the render or batch lane that uses the arena
    PathStore store;
};

struct ArenaPool {
    std::mutex lock;
    std::vector<std::unique_ptr<PathArena>> arenas;
    size_t next = 0;
    int tracers = 0;
};

ArenaPool& arenaPool(int device)
{
    // Never destroyed: the arenas go with their device's last tracer, not at
    // process exit, when the CUDA runtime may already be gone.
    static ArenaPool* pools = new ArenaPool[kArenaDevices];
    if (device < 0 || device >= kArenaDevices) throw std::runtime_error("device ordinal out of range");
    return pools[device];
}

struct ArenaLease {
    PathArena* arena = nullptr;
    std::unique_lock<std::mutex> hold;
};

// A free arena of `device`, or a new one while the device has fewer than
// kMaxArenas. When all are busy: with `wait`, waits for one of them (round
// robin); without, returns an empty lease.
ArenaLease checkoutArena(int device, bool wait)
{
    ArenaPool& pool = arenaPool(device);
    PathArena* busy = nullptr;
    {
        std::lock_guard<std::mutex> guard(pool.lock);
        for (auto& a : pool.arenas) {
            std::unique_lock<std::mutex> hold(a->busy, std::try_to_lock);
            if (hold.owns_lock()) return ArenaLease{a.get(), std::move(hold)};
        }
        if (pool.arenas.size() < kMaxArenas) {
            pool.arenas.push_back(std::make_unique<PathArena>());
            PathArena* a = pool.arenas.back().get();
            return ArenaLease{a, std::unique_lock<std::mutex>(a->busy)};
        }
        if (!wait) return ArenaLease{};
        busy = pool.arenas[pool.next++ % pool.arenas.size()].get();
    }
    return ArenaLease{busy, std::unique_lock<std::mutex>(busy->busy)};
}

// Frames of hdcx_render_async in flight (defined with the render helpers).
struct AsyncFrames;

// A scene with instancers: the bottom-level BVHs (index 0: the scene's
// non-instanced triangles in world space, when it has any; then one per
// instancer, in object space), the top-level BVH over the instances, the
// device tables behind DeviceScene::instances / blases, and the packed scene
// kept on the host for hdcx_update_instancer_points.
struct TwoLevel {
    std::vector<WideBvh> blases;
    std::vector<int> blasOfInstancer;  // per instancer: its index in blases
    WideBvh top;
    std::vector<DeviceBuffer*> buffers;
    std::vector<float4*> objectPoints;      // per instancer, device
    std::vector<uint32_t*> objectIndices;   // per instancer, device
    std::vector<float> objectScale;         // per instancer: the BLAS's quantisation floor
    std::vector<InstanceDesc> instances;
    std::vector<BlasDesc> blasTable;
    InstanceDesc* instancesDevice = nullptr;
    BlasDesc* blasDevice = nullptr;
    uint32_t plainInstance = 0;             // 1 when instance 0 is the world-space BLAS
    PackedSceneData host;
    TwoLevel() = default;
    TwoLevel(const TwoLevel&) = delete;
    TwoLevel& operator=(const TwoLevel&) = delete;
    ~TwoLevel()
    {
        for (WideBvh& b : blases) freeWideBvh(b);
        freeWideBvh(top);
        for (DeviceBuffer* b : buffers) delete b;
    }
    template <typename T>
    T* upload(const std::vector<T>& data, cudaStream_t stream)
    {
        auto* b = new DeviceBuffer();
        buffers.push_back(b);
        b->allocate(std::max<size_t>(1, data.size()) * sizeof(T));
        if (!data.empty()) check(cudaMemcpyAsync(b->ptr, data.data(), data.size() * sizeof(T), cudaMemcpyHostToDevice, stream), "upload");
        return b->as<T>();
    }
};

}  // namespace

struct hdcx_nrc {
    int device = 0;
    cudaStream_t stream = nullptr;
    hdcx::nrc::Cache* cache = nullptr;
    std::string lastError;
    ~hdcx_nrc()
    {
        if (stream) cudaStreamSynchronize(stream);
        hdcx::nrc::destroy(cache);
        if (stream) cudaStreamDestroy(stream);
    }
};

struct hdcx_tracer {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string lastError;
    int32_t shadingMode = HDCX_SHADING_FUSED;
    bool geometryReady = false;
    bool fallbackAxisInitialized = false;
    bool fallbackZUp = false;
    uint64_t wavePaths = 0;  // 0 = automatic
    uint32_t traceBlocksPerSm = 16;
    uint32_t shadeBlocksPerSm = 8;
    uint32_t sortHits = 0;   // shade hits in material order
    uint32_t sortRays = 0;   // trace secondary rays in direction order
    uint32_t profiling = 0;  // HDCX_PROFILE_* bits
    // Scene.
    std::vector<DeviceBuffer*> sceneBuffers;
    DeviceBuffer texDescs;
    DeviceScene scene{};
    WideBvh bvh;
    // Path state of radiance-cache renders (other renders use the arenas).
    PathStore own;
    DeviceBuffer rgba, xyz, batch, batchXyz;
    // Device AOVs (hdcx_set_aovs): primary hit and distance of the first
    // sample of every render, per pixel of the render's size.
    uint32_t aovFlags = 0;
    DeviceBuffer aovIds, aovDepth;
    uint32_t aovWidth = 0, aovHeight = 0;
    DeviceBuffer preview;  // hdcx_render_preview's upscaled image
    // Frames of hdcx_render_async in flight (created on first use).
    AsyncFrames* async = nullptr;
    // Two-level scenes (hdcx_set_scene_instanced); null for single-level ones.
    std::unique_ptr<TwoLevel> twoLevel;
    double sceneBuildMs = 0.0;  // host wall time of the last set_scene
    uint32_t textureLod = 0;    // hdcx_set_texture_lod
    std::vector<TexDesc> texDescHost;  // the device table's host copy (mip pyramids added on demand)
    double bvhBuildMs = 0.0;    // of which building the BVHs
    DeviceBuffer statsBuffer;  // this tracer's ray counters (8 x u64), whichever path buffers it renders with
    FrameBuffers fb;
    uint64_t xyzSamples = 0;
    hdcx_render_stats stats{};
    cudaEvent_t start = nullptr, stop = nullptr;
    // Radiance-cache mode (hdcx_set_radiance_cache).
    hdcx_nrc* radianceCache = nullptr;
    uint32_t cachePrefix = 2;
    float cacheSpread = 0.0F;  // hdcx_set_radiance_cache_spread
    uint32_t cacheTrainingPaths = 1u << 14;
    std::vector<DeviceBuffer*> cacheBuffers;
    CacheDevice cacheDevice;
    uint64_t cacheCapacity = 0;
    CacheRun cacheRun;
    float3 sceneMin{}, sceneScale{};

    ~hdcx_tracer()
    {
        if (stream) cudaStreamSynchronize(stream);
        clearScene();
        own.release();
        clearCache();
        if (start) cudaEventDestroy(start);
        if (stop) cudaEventDestroy(stop);
        if (stream) cudaStreamDestroy(stream);
    }
    void clearScene()
    {
        for (DeviceBuffer* b : sceneBuffers) delete b;
        sceneBuffers.clear();
        texDescs.reset();
        freeWideBvh(bvh);
        twoLevel.reset();
        scene = DeviceScene{};
        geometryReady = false;
    }
    void clearCache()
    {
        for (DeviceBuffer* b : cacheBuffers) delete b;
        cacheBuffers.clear();
        cacheDevice = CacheDevice{};
        cacheCapacity = 0;
    }
    template <typename T>
    T* cacheAlloc(size_t count)
    {
        auto* b = new DeviceBuffer();
        cacheBuffers.push_back(b);
        b->allocate(count * sizeof(T));
        return b->as<T>();
    }
    template <typename T>
    T* upload(const std::vector<T>& host)
    {
        auto* b = new DeviceBuffer();
        sceneBuffers.push_back(b);
        b->allocate(host.size() * sizeof(T));
        if (!host.empty()) check(cudaMemcpyAsync(b->ptr, host.data(), host.size() * sizeof(T), cudaMemcpyHostToDevice, stream), "upload");
        return b->as<T>();
    }
};

struct hdcx_packing {
    PackedSceneData data;
    std::vector<hdcx_packed_texture> textureViews;
    hdcx_packed_scene view{};
};

namespace {

hdcx_status fail(hdcx_tracer* t, hdcx_status s, const std::string& message)
{
    if (t) t->lastError = message;
    return s;
}

template <typename F>
hdcx_status guarded(hdcx_tracer* t, F&& body)
{
    try {
        if (t) {
            t->lastError.clear();
            check(cudaSetDevice(t->device), "cudaSetDevice");
        }
        body();
        return HDCX_OK;
    } catch (const StatusError& e) {
        return fail(t, e.status, e.what());
    } catch (const OutOfDeviceMemory& e) {
        return fail(t, HDCX_ERROR_OUT_OF_MEMORY, e.what());
    } catch (const std::invalid_argument& e) {
        return fail(t, HDCX_ERROR_INVALID_ARGUMENT, e.what());
    } catch (const std::bad_alloc&) {
        return fail(t, HDCX_ERROR_OUT_OF_MEMORY, "host allocation failed");
    } catch (const std::exception& e) {
        return fail(t, HDCX_ERROR_CUDA, e.what());
    }
}

// Whether any material uses a texture, a layered lobe (coat, sheen,
// transmission, subsurface, diffuse transmission) or a non-Lambert diffuse
// model; scenes without these run the specialised shade kernel.
bool needsFullShading(const PackedSceneData& d)
{
    const size_t n = d.materials.size() / HDCX_GPU_MATERIAL_BYTES;
    for (size_t i = 0; i < n; ++i) {
        GpuMaterial m;
        std::memcpy(&m, d.materials.data() + i * HDCX_GPU_MATERIAL_BYTES, sizeof m);
        const uint32_t* tex = &m.textureIndices0.x;
        for (int k = 0; k < 24; ++k) {
            if (tex[k] != HDCX_MISSING_TEXTURE) return true;
        }
        if (m.transmissionOpacityIor.x > 0.0F || m.subsurfaceWeightScale.x > 0.0F || m.coatWeightRoughnessIor.x > 0.0F ||
            m.coatColor.w > 0.0F || m.translucentColorWeight.w > 0.0F ||
            static_cast<uint32_t>(m.diffuseProperties.y + 0.5F) != 0u) {
            return true;
        }
        if (!(m.transmissionOpacityIor.x <= 0.0F) || !(m.coatColor.w <= 0.0F) || !(m.translucentColorWeight.w <= 0.0F)) {
            return true;  // NaN weights take the general kernel
        }
    }
    return false;
}

// Whether any material can take the subsurface walk: a subsurface weight
// above zero (or NaN) or a subsurface-weight texture.
bool hasSubsurfaceMaterial(const PackedSceneData& d)
{
    const size_t n = d.materials.size() / HDCX_GPU_MATERIAL_BYTES;
    for (size_t i = 0; i < n; ++i) {
        GpuMaterial m;
        std::memcpy(&m, d.materials.data() + i * HDCX_GPU_MATERIAL_BYTES, sizeof m);
        if (!(m.subsurfaceWeightScale.x <= 0.0F) || m.textureIndices2.x != HDCX_MISSING_TEXTURE) return true;
    }
    return false;
}

// Per-triangle opacity hints for the BVH's leaf copies: the opacity that
// surfaceOpacity returns for a triangle whose material has no opacity texture
// (the material's opacity clamped to [0, 1] as GLSL clamps, a NaN kept), -1
// for the others, whose opacity the traversal samples from the texture.
std::vector<float> opacityHints(const PackedSceneData& d)
{
    const size_t materialCount = d.materials.size() / HDCX_GPU_MATERIAL_BYTES;
    std::vector<float> perMaterial(materialCount, -1.0F);
    for (size_t i = 0; i < materialCount; ++i) {
        GpuMaterial m;
        std::memcpy(&m, d.materials.data() + i * HDCX_GPU_MATERIAL_BYTES, sizeof m);
        if (m.textureIndices1.x != HDCX_MISSING_TEXTURE) continue;
        float x = m.transmissionOpacityIor.y;
        x = x < 0.0F ? 0.0F : x;
        x = 1.0F < x ? 1.0F : x;
        perMaterial[i] = x;
    }
    std::vector<float> hints(d.triangleMaterials.size(), -1.0F);
    for (size_t t = 0; t < hints.size(); ++t) {
        const uint32_t m = d.triangleMaterials[t];
        if (m < materialCount) hints[t] = perMaterial[m];
    }
    return hints;
}

// The arrays behind TexDesc::cdf for a dome importance texture (R: the
// row's conditional CDF, G at column 0: the marginal CDF). Returns false, and
// the device keeps the plain binary search, unless every CDF is finite and
// non-decreasing: only then does the two-level search find the same index.
bool buildCdfArrays(const PackedTexture& pt, std::vector<float>& block)
{
    const size_t w = pt.width, h = pt.height;
    if (w == 0 || h == 0 || pt.floats.size() < w * h * 4u) return false;
    const size_t hs = (h + 31) / 32, ws = (w + 31) / 32;
    block.assign(h + hs + w * h + h * ws, 0.0F);
    float* marginal = block.data();
    float* marginalSkip = marginal + h;
    float* conditional = marginalSkip + hs;
    float* conditionalSkip = conditional + w * h;
    auto monotone = [](const float* v, size_t n) {
        for (size_t i = 0; i < n; ++i) {
            if (!std::isfinite(v[i]) || (i > 0 && v[i] < v[i - 1])) return false;
        }
        return true;
    };
    for (size_t row = 0; row < h; ++row) {
        marginal[row] = pt.floats[(row * w) * 4u + 1u];
        for (size_t col = 0; col < w; ++col) conditional[row * w + col] = pt.floats[(row * w + col) * 4u + 0u];
        if (!monotone(conditional + row * w, w)) return false;
        for (size_t k = 0; k < ws; ++k) conditionalSkip[row * ws + k] = conditional[row * w + std::min(32 * k + 31, w - 1)];
    }
    if (!monotone(marginal, h)) return false;
    for (size_t k = 0; k < hs; ++k) marginalSkip[k] = marginal[std::min(32 * k + 31, h - 1)];
    return true;
}

// The mip pyramids of every texture without one (texture LOD), built on the
// GPU into scene buffers; updates the host copy of the descriptor table.
void buildTextureMips(hdcx_tracer* t)
{
    for (TexDesc& td : t->texDescHost) {
        if (td.mips != nullptr || td.width == 0u || td.height == 0u) continue;
        uint32_t levels = 1;
        const uint64_t n = mipTexels(td.width, td.height, levels);
        if (n == 0) continue;
        auto* b = new DeviceBuffer();
        t->sceneBuffers.push_back(b);
        b->allocate(n * sizeof(float4));
        buildMips(td, b->as<float4>(), t->stream);
    }
}

// Object-space scale of a point set (max |coordinate|, max extent): the
// quantisation floor of its BVH.
float pointScale(const float* xyzw, size_t count)
{
    float scale = 0.0F;
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (size_t i = 0; i < count; ++i) {
        for (int k = 0; k < 3; ++k) {
            const float v = xyzw[4 * i + k];
            if (!std::isfinite(v)) continue;
            lo[k] = std::min(lo[k], v);
            hi[k] = std::max(hi[k], v);
            scale = std::max(scale, std::fabs(v));
        }
    }
    for (int k = 0; k < 3; ++k)
        if (hi[k] >= lo[k]) scale = std::max(scale, hi[k] - lo[k]);
    return std::max(scale, 1e-20F);
}

// World boxes of the instances (over their flattened vertices) as the
// degenerate triangles (lo, hi, lo) the top-level build takes, and the
// instances' margins; then the top-level BVH.
void buildTopLevel(hdcx_tracer* t, TwoLevel& tl, const PackedSceneData& d, const std::vector<uint32_t>& plainVertices)
{
    std::vector<float> boxes;
    std::vector<uint32_t> boxIndices;
    auto addBox = [&](const float* xyzw, const uint32_t* which, size_t count) {
        float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
        float mag = 0.0F;
        for (size_t i = 0; i < count; ++i) {
            const float* v = xyzw + 4 * size_t(which ? which[i] : i);
            for (int k = 0; k < 3; ++k) {
                if (!std::isfinite(v[k])) continue;
                lo[k] = std::min(lo[k], v[k]);
                hi[k] = std::max(hi[k], v[k]);
                mag = std::max(mag, std::fabs(v[k]));
            }
        }
        const uint32_t b = static_cast<uint32_t>(boxes.size() / 4);
        boxes.insert(boxes.end(), {lo[0], lo[1], lo[2], 1.0F, hi[0], hi[1], hi[2], 1.0F});
        boxIndices.insert(boxIndices.end(), {b, b + 1u, b});
        return mag;
    };
    size_t inst = 0;
    if (tl.plainInstance) {
        addBox(d.vertices.data(), plainVertices.data(), plainVertices.size());
        inst = 1;
    }
    for (size_t k = 0; k < d.instancers.size(); ++k) {
        const PackedInstancer& pi = d.instancers[k];
        float objectMag = 0.0F;
        for (size_t i = 0; i < pi.points.size(); i += 4)
            for (int c = 0; c < 3; ++c)
                if (std::isfinite(pi.points[i + c])) objectMag = std::max(objectMag, std::fabs(pi.points[i + c]));
        for (uint32_t j = 0; j < pi.instanceCount; ++j, ++inst) {
            const float worldMag = addBox(d.vertices.data() + 4 * (size_t(pi.firstVertex) + size_t(j) * pi.pointCount()), nullptr,
                                          pi.pointCount());
            InstanceDesc& I = tl.instances[inst];
            const float translation = std::max({std::fabs(I.inv0.w), std::fabs(I.inv1.w), std::fabs(I.inv2.w)});
            // 2^-20 of every magnitude that enters the transformed ray and the
            // world vertices, taken to object space.
            I.margin = 9.5367432e-7F * (objectMag + (worldMag + translation) * I.invNorm);
        }
    }
    float* boxDev = tl.upload(boxes, t->stream);
    uint32_t* boxIdxDev = tl.upload(boxIndices, t->stream);
    freeWideBvh(tl.top);
    tl.top = buildWideBvh(reinterpret_cast<const float4*>(boxDev), boxIdxDev, static_cast<uint32_t>(boxIndices.size() / 3),
                          pointScale(boxes.data(), boxes.size() / 4), t->stream);
    check(cudaMemcpyAsync(tl.instancesDevice, tl.instances.data(), tl.instances.size() * sizeof(InstanceDesc),
                          cudaMemcpyHostToDevice, t->stream),
          "upload instances");
}

// The two-level form of a scene with instancers (see TwoLevel).
void buildTwoLevel(hdcx_tracer* t, const PackedSceneData& d, DeviceScene& s, float worldScale)
{
    auto tl = std::make_unique<TwoLevel>();
    tl->host = d;
    const size_t n = d.triangleCount();
    std::vector<uint8_t> instanced(n, 0u);
    for (const PackedInstancer& pi : d.instancers) {
        const size_t end = size_t(pi.firstTriangle) + size_t(pi.instanceCount) * pi.triangles();
        for (size_t p = pi.firstTriangle; p < end; ++p) instanced[p] = 1u;
    }
    std::vector<uint32_t> plainIds, plainIndices, plainVertices;
    for (size_t p = 0; p < n; ++p) {
        if (instanced[p]) continue;
        plainIds.push_back(static_cast<uint32_t>(p));
        for (int c = 0; c < 3; ++c) {
            plainIndices.push_back(d.indices[3 * p + c]);
            plainVertices.push_back(d.indices[3 * p + c]);
        }
    }
    if (!plainIds.empty()) {
        uint32_t* idsDev = tl->upload(plainIds, t->stream);
        uint32_t* idxDev = tl->upload(plainIndices, t->stream);
        tl->blases.push_back(buildWideBvh(s.vertices, idxDev, static_cast<uint32_t>(plainIds.size()), worldScale, t->stream,
                                          idsDev));
        tl->plainInstance = 1;
        InstanceDesc I{};
        I.inv0 = make_float4(1.0F, 0.0F, 0.0F, 0.0F);
        I.inv1 = make_float4(0.0F, 1.0F, 0.0F, 0.0F);
        I.inv2 = make_float4(0.0F, 0.0F, 1.0F, 0.0F);
        I.blas = 0;
        I.identity = 1;
        I.invNorm = 1.0F;
        tl->instances.push_back(I);
    }
    for (const PackedInstancer& pi : d.instancers) {
        const uint32_t blas = static_cast<uint32_t>(tl->blases.size());
        tl->blasOfInstancer.push_back(static_cast<int>(blas));
        float4* pts = reinterpret_cast<float4*>(tl->upload(pi.points, t->stream));
        uint32_t* idx = tl->upload(pi.indices, t->stream);
        tl->objectPoints.push_back(pts);
        tl->objectIndices.push_back(idx);
        tl->objectScale.push_back(pointScale(pi.points.data(), pi.pointCount()));
        tl->blases.push_back(buildWideBvh(pts, idx, pi.triangles(), tl->objectScale.back(), t->stream));
        for (uint32_t j = 0; j < pi.instanceCount; ++j) {
            const double* T = pi.transforms.data() + 16u * j;
            // inverse(A) by cofactors, as the flattening computes it.
            const double a00 = T[0], a01 = T[1], a02 = T[2], a10 = T[4], a11 = T[5], a12 = T[6], a20 = T[8], a21 = T[9],
                         a22 = T[10];
            const double c00 = a11 * a22 - a12 * a21, c01 = a12 * a20 - a10 * a22, c02 = a10 * a21 - a11 * a20;
            const double det = (a00 * c00 + a01 * c01) + a02 * c02;
            const double inv[9] = {c00 / det,
                                   (a02 * a21 - a01 * a22) / det,
                                   (a01 * a12 - a02 * a11) / det,
                                   c01 / det,
                                   (a00 * a22 - a02 * a20) / det,
                                   (a02 * a10 - a00 * a12) / det,
                                   c02 / det,
                                   (a01 * a20 - a00 * a21) / det,
                                   (a00 * a11 - a01 * a10) / det};
            InstanceDesc I{};
            I.inv0 = make_float4(float(inv[0]), float(inv[1]), float(inv[2]), float(T[12]));
            I.inv1 = make_float4(float(inv[3]), float(inv[4]), float(inv[5]), float(T[13]));
            I.inv2 = make_float4(float(inv[6]), float(inv[7]), float(inv[8]), float(T[14]));
            I.blas = blas;
            I.triBase = pi.firstTriangle + j * pi.triangles();
            I.identity = 0;
            float norm = 0.0F;
            for (int c = 0; c < 3; ++c)
                norm = std::max(norm, float(std::fabs(inv[c]) + std::fabs(inv[3 + c]) + std::fabs(inv[6 + c])));
            if (!std::isfinite(norm) || !std::isfinite(det) || det == 0.0)
                throw std::invalid_argument("instancer: a transform is singular or not finite");
            I.invNorm = norm;
            tl->instances.push_back(I);
        }
    }
    for (const WideBvh& b : tl->blases) tl->blasTable.push_back(BlasDesc{b.nodes, b.triVerts, b.nodeCount, 0u});
    tl->blasDevice = tl->upload(tl->blasTable, t->stream);
    tl->instancesDevice = tl->upload(tl->instances, t->stream);
    buildTopLevel(t, *tl, d, plainVertices);
    s.nodes = tl->top.nodes;
    s.triVerts = tl->top.triVerts;
    s.nodeCount = tl->top.nodeCount;
    s.instances = tl->instancesDevice;
    s.blases = tl->blasDevice;
    s.instanceCount = static_cast<uint32_t>(tl->instances.size());
    t->twoLevel = std::move(tl);
}

void uploadScene(hdcx_tracer* t, const PackedSceneData& d)
{
    check(cudaStreamSynchronize(t->stream), "cudaStreamSynchronize");
    t->clearScene();
    if (!d.geometryReady) return;
    DeviceScene s{};
    s.vertices = reinterpret_cast<const float4*>(t->upload(d.vertices));
    s.indices = t->upload(d.indices);
    s.triangleMaterials = t->upload(d.triangleMaterials);
    s.texcoords = reinterpret_cast<const float2*>(t->upload(d.texcoords));
    s.normals = reinterpret_cast<const float4*>(t->upload(d.normals));
    s.materials = reinterpret_cast<const GpuMaterial*>(t->upload(d.materials));
    s.lights = reinterpret_cast<const GpuLight*>(t->upload(d.lights));
    s.emissive = reinterpret_cast<const float4*>(t->upload(d.emissive));
    std::vector<TexDesc> descs;
    for (const PackedTexture& pt : d.textures) {
        TexDesc td{};
        td.width = pt.width;
        td.height = pt.height;
        td.format = pt.format;
        td.texels = pt.format == HDCX_TEXEL_RGBA32F ? static_cast<const void*>(t->upload(pt.floats))
                                                    : static_cast<const void*>(t->upload(pt.bytes));
        descs.push_back(td);
    }
    // Dome importance textures get the compact CDF arrays of TexDesc::cdf.
    for (uint32_t l = 0; l < d.lightCount && (size_t(l) + 1) * sizeof(GpuLight) <= d.lights.size(); ++l) {
        GpuLight light;
        std::memcpy(&light, d.lights.data() + size_t(l) * sizeof(GpuLight), sizeof(GpuLight));
        const uint32_t index = light.textureInfo.w;
        if (light.textureInfo.z != 0u || index >= descs.size() || descs[index].cdf) continue;
        const PackedTexture& pt = d.textures[index];
        std::vector<float> block;
        if (pt.format == HDCX_TEXEL_RGBA32F && buildCdfArrays(pt, block)) {
            descs[index].cdf = t->upload(block);
        }
    }
    for (TexDesc& td : descs) td.levels = 1u;
    t->texDescHost = descs;
    if (t->textureLod) buildTextureMips(t);
    descs = t->texDescHost;
    t->texDescs.allocate(std::max<size_t>(1, descs.size()) * sizeof(TexDesc));
    if (!descs.empty()) {
        check(cudaMemcpyAsync(t->texDescs.ptr, descs.data(), descs.size() * sizeof(TexDesc), cudaMemcpyHostToDevice, t->stream),
              "upload textures");
    }
    s.textures = t->texDescs.as<TexDesc>();
    s.textureCount = static_cast<uint32_t>(descs.size());
    s.primitiveCount = d.triangleCount();
    s.lightCount = std::min(d.lightCount, static_cast<uint32_t>(HDCX_MAX_LIGHTS));
    s.opaque = d.opaque ? 1u : 0u;
    s.fullShading = needsFullShading(d) ? 1u : 0u;
    s.hasSubsurface = hasSubsurfaceMaterial(d) ? 1u : 0u;
    s.hasMeshLights = (d.triangleCount() > 0 && d.emissive[(size_t(d.triangleCount()) - 1) * 4u] > 0.0F) ? 1u : 0u;
    {
        // Scene box (padded by 0.1% per side) for the radiance-cache positions.
        float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
        for (size_t v = 0; v < d.vertices.size() / 4; ++v) {
            for (int a = 0; a < 3; ++a) {
                const float x = d.vertices[v * 4 + a];
                if (std::isfinite(x)) {
                    lo[a] = std::min(lo[a], x);
                    hi[a] = std::max(hi[a], x);
                }
            }
        }
        float extent[3];
        for (int a = 0; a < 3; ++a) {
            if (!(hi[a] >= lo[a])) lo[a] = hi[a] = 0.0F;
            extent[a] = std::max(hi[a] - lo[a], 1e-6F);
            lo[a] -= 1e-3F * extent[a];
            extent[a] *= 1.002F;
        }
        t->sceneMin = make_float3(lo[0], lo[1], lo[2]);
        t->sceneScale = make_float3(1.0F / extent[0], 1.0F / extent[1], 1.0F / extent[2]);
    }
    // Padding floor of the BVH quantisation: the scene's coordinate scale.
    float scale = 0.0F;
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (size_t i = 0; i < d.vertices.size(); i += 4) {
        for (int k = 0; k < 3; ++k) {
            const float v = d.vertices[i + k];
            if (!std::isfinite(v)) continue;
            lo[k] = std::min(lo[k], v);
            hi[k] = std::max(hi[k], v);
            scale = std::max(scale, std::fabs(v));
        }
    }
    for (int k = 0; k < 3; ++k) {
        if (hi[k] >= lo[k]) scale = std::max(scale, hi[k] - lo[k]);
    }
    const auto bvhStart = std::chrono::steady_clock::now();
    NvtxRange bvhRange("hdcx bvh build");
    if (d.instancers.empty()) {
        const std::vector<float> hostHints = opacityHints(d);
        const float* hints = t->upload(hostHints);
        t->bvh = buildWideBvh(s.vertices, s.indices, s.primitiveCount, std::max(scale, 1e-20F), t->stream, nullptr, hints);
        s.nodes = t->bvh.nodes;
        s.triVerts = t->bvh.triVerts;
        s.nodeCount = t->bvh.nodeCount;
    } else {
        buildTwoLevel(t, d, s, std::max(scale, 1e-20F));
    }
    check(cudaStreamSynchronize(t->stream), "scene upload");
    t->bvhBuildMs = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - bvhStart).count();
    t->scene = s;
    t->geometryReady = true;
}

void ensureOutput(hdcx_tracer* t, uint32_t w, uint32_t h)
{
    if (t->fb.width == w && t->fb.height == h && t->fb.rgba) return;
    // EnsureOutput (vulkan_path_tracer.cpp:3130-3160): a new size gets a
    // zero-filled accumulation buffer.
    check(cudaStreamSynchronize(t->stream), "cudaStreamSynchronize");
    const size_t pixels = size_t(w) * h;
    t->rgba.allocate(pixels * sizeof(float4));
    t->xyz.allocate(pixels * 3u * sizeof(double));
    t->batch.allocate(pixels * sizeof(float4));
    t->batchXyz.allocate(pixels * 3u * sizeof(double));
    check(cudaMemsetAsync(t->rgba.ptr, 0, pixels * sizeof(float4), t->stream), "clear output");
    check(cudaMemsetAsync(t->xyz.ptr, 0, pixels * 3u * sizeof(double), t->stream), "clear xyz");
    t->fb.width = w;
    t->fb.height = h;
    t->fb.rgba = t->rgba.as<float4>();
    t->fb.xyz = t->xyz.as<double>();
    t->fb.batch = t->batch.as<float4>();
    t->fb.batchXyz = t->batchXyz.as<double>();
    t->xyzSamples = 0;
}

constexpr uint64_t kAutomaticWavePaths = 12ull << 20;  // ~12.6M paths per wave
// Device bytes of path state per path (PathBuffers with three shadow slots
// and the deferred subsurface-walk records).
constexpr uint64_t kPathStateBytes = 143 + 48 + 8 + 3 * 56;

// Smallest wave an automatic wave is shrunk to when device memory is short.
constexpr uint64_t kMinimumAutomaticWave = 1ull << 16;

// Sizes the wave of a render of `needed` paths on `store` and grows the store
// to it; returns the wave. The wave is the tracer's own wave size if it set
// one, else min(needed, `capOverride` or the automatic wave). A wave the
// tracer did not set is also bounded by device memory: its path state takes
// at most three quarters of what is free plus what the store already holds
// (the wave size does not change the image). Buffers larger than the wave are
// kept, but the wave is this call's, since it decides the launch shape.
// `fixed`: the store is not grown; the wave is bounded by its capacity.
uint64_t ensureStore(hdcx_tracer* t, PathStore& store, uint64_t needed, uint64_t capOverride, bool fixed)
{
    constexpr uint32_t kShadowSlots = 3;
    const uint64_t cap = t->wavePaths ? t->wavePaths : (capOverride ? capOverride : kAutomaticWavePaths);
    uint64_t capacity = std::max<uint64_t>(3, std::min(needed, cap));
    if (fixed) return std::min(capacity, store.paths.capacity);
    if (t->wavePaths == 0) {
        size_t freeBytes = 0, totalBytes = 0;
        check(cudaMemGetInfo(&freeBytes, &totalBytes), "cudaMemGetInfo");
        const uint64_t held = store.paths.capacity * (143ull + 56ull * store.paths.shadowPerPath);
        uint64_t fit = (static_cast<uint64_t>(freeBytes) + held) / 4 * 3 / (143ull + 56ull * kShadowSlots);
        if (store.paths.shadowPerPath >= kShadowSlots) fit = std::max(fit, store.paths.capacity);  // held buffers serve as is
        capacity = std::min(capacity, std::max(fit, std::min(capacity, kMinimumAutomaticWave)));
    }
    if (store.paths.capacity < capacity || store.paths.shadowPerPath < kShadowSlots) {
        check(cudaStreamSynchronize(t->stream), "cudaStreamSynchronize");
        store.allocate(capacity, kShadowSlots);
    }
    return capacity;
}

unsigned long long* tracerStats(hdcx_tracer* t)
{
    if (!t->statsBuffer.ptr) t->statsBuffer.allocate(8 * sizeof(unsigned long long));
    return t->statsBuffer.as<unsigned long long>();
}

// Buffers of the radiance-cache mode for waves of up to `capacity` paths.
void ensureCacheBuffers(hdcx_tracer* t, uint64_t capacity)
{
    const uint64_t trainCapacity = 2ull * t->cacheTrainingPaths;
    if (t->cacheCapacity >= capacity && t->cacheDevice.trainCapacity == trainCapacity && t->cacheDevice.queries) return;
    check(cudaStreamSynchronize(t->stream), "cudaStreamSynchronize");
    t->clearCache();
    CacheDevice& c = t->cacheDevice;
    const uint64_t records = trainCapacity * kCacheMaxVertices;
    c.queries = t->cacheAlloc<float>(capacity * 12u);
    c.querySlot = t->cacheAlloc<uint32_t>(capacity);
    c.predictions = t->cacheAlloc<float>(capacity);
    c.trainIndex = t->cacheAlloc<uint32_t>(capacity);
    c.spread = t->cacheAlloc<float2>(capacity);
    c.trainSlot = t->cacheAlloc<uint32_t>(trainCapacity);
    c.trainVertices = t->cacheAlloc<uint32_t>(trainCapacity);
    c.trainRecords = t->cacheAlloc<float>(records * 12u);
    c.trainState = t->cacheAlloc<float2>(records);
    c.sampleQueries = t->cacheAlloc<float>(records * 12u);
    c.sampleTargets = t->cacheAlloc<float>(records);
    c.counters = t->cacheAlloc<uint32_t>(4);
    c.trainCapacity = static_cast<uint32_t>(trainCapacity);
    t->cacheCapacity = capacity;
}

FrameConst makeFrame(const hdcx_tracer* t, const hdcx_camera& c, uint32_t w, uint32_t h, uint32_t sampleIndex,
                     uint32_t maxBounces, uint32_t sampleCount)
{
    FrameConst f{};
    f.origin = make_float3(c.origin[0], c.origin[1], c.origin[2]);
    f.lowerLeft = make_float3(c.lower_left[0], c.lower_left[1], c.lower_left[2]);
    f.horizontal = make_float3(c.horizontal[0], c.horizontal[1], c.horizontal[2]);
    f.vertical = make_float3(c.vertical[0], c.vertical[1], c.vertical[2]);
    f.width = w;
    f.height = h;
    f.sampleIndex = sampleIndex;
    f.sampleCount = std::max(sampleCount, 1u);
    f.maxBounces = std::clamp(maxBounces, 1u, HDCX_MAX_PATH_BOUNCES);
    f.zUp = t->fallbackZUp ? 1u : 0u;
    if (t->textureLod) {
        // Spread angle of a camera ray per pixel: the image's vertical extent
        // over its height in pixels, at the distance of the image plane.
        const double cx = double(f.lowerLeft.x) + 0.5 * f.horizontal.x + 0.5 * f.vertical.x - f.origin.x;
        const double cy = double(f.lowerLeft.y) + 0.5 * f.horizontal.y + 0.5 * f.vertical.y - f.origin.y;
        const double cz = double(f.lowerLeft.z) + 0.5 * f.horizontal.z + 0.5 * f.vertical.z - f.origin.z;
        const double distance = std::sqrt(cx * cx + cy * cy + cz * cz);
        const double extent = std::sqrt(double(f.vertical.x) * f.vertical.x + double(f.vertical.y) * f.vertical.y +
                                        double(f.vertical.z) * f.vertical.z);
        if (distance > 0.0 && h > 0u) f.pixelSpread = static_cast<float>(extent / (double(h) * distance));
    }
    return f;
}

// hdcx_render_async's frames (defined with the render helpers below).
void drainAsync(hdcx_tracer* t);
void destroyAsync(hdcx_tracer* t);

}  // namespace

extern "C" {

HDCX_API uint32_t hdcx_abi_version(void) { return HDCX_ABI_VERSION; }

HDCX_API uint32_t hdcx_abi_struct_sizes(uint64_t* sizes, uint32_t capacity)
{
    const uint64_t all[] = {sizeof(hdcx_camera),         sizeof(hdcx_mesh_desc),  sizeof(hdcx_material_desc),
                            sizeof(hdcx_texture_desc),   sizeof(hdcx_light_desc), sizeof(hdcx_scene_desc),
                            sizeof(hdcx_packed_texture), sizeof(hdcx_packed_scene), sizeof(hdcx_render_stats),
                            sizeof(hdcx_batch_job), sizeof(hdcx_nrc_config), sizeof(hdcx_tuning),
                            sizeof(hdcx_instancer_desc), sizeof(hdcx_scene_info)};
    const uint32_t n = static_cast<uint32_t>(sizeof(all) / sizeof(all[0]));
    for (uint32_t i = 0; i < std::min(n, capacity); ++i) sizes[i] = all[i];
    return n;
}

HDCX_API void hdcx_material_defaults(hdcx_material_desc* m)
{
    if (!m) return;
    std::memset(m, 0, sizeof(*m));
    auto set3 = [](float* d, float a, float b, float c) { d[0] = a; d[1] = b; d[2] = c; };
    set3(m->base_color, 0.8F, 0.8F, 0.8F);
    set3(m->base_color_texture_scale, 1.0F, 1.0F, 1.0F);
    m->base_color_texture_channel = -1;
    set3(m->transmission_color, 1.0F, 1.0F, 1.0F);
    set3(m->specular_color, 1.0F, 1.0F, 1.0F);
    set3(m->coat_color, 1.0F, 1.0F, 1.0F);
    set3(m->sheen_color, 1.0F, 1.0F, 1.0F);
    set3(m->translucent_color, 1.0F, 1.0F, 1.0F);
    set3(m->subsurface_color, 0.8F, 0.8F, 0.8F);
    set3(m->subsurface_radius, 1.0F, 0.2F, 0.1F);
    m->diffuse_weight = 1.0F;
    m->roughness = 0.5F;
    m->roughness_v = 0.5F;
    m->opacity = 1.0F;
    m->transmission_dispersion_abbe_number = 20.0F;
    m->index_of_refraction = 1.5F;
    m->specular_weight = 1.0F;
    m->coat_roughness = 0.1F;
    m->coat_roughness_v = 0.1F;
    m->coat_index_of_refraction = 1.5F;
    m->sheen_roughness = 0.3F;
    m->subsurface_scale = 1.0F;
    m->normal_texture_scale = 1.0F;
}

HDCX_API void hdcx_light_defaults(hdcx_light_desc* l)
{
    if (!l) return;
    std::memset(l, 0, sizeof(*l));
    auto set3 = [](float* d, float a, float b, float c) { d[0] = a; d[1] = b; d[2] = c; };
    l->visible = 1;
    set3(l->color, 1.0F, 1.0F, 1.0F);
    set3(l->temperature_color, 1.0F, 1.0F, 1.0F);
    l->intensity = 1.0F;
    l->diffuse = 1.0F;
    l->specular = 1.0F;
    set3(l->basis_x, 1.0F, 0.0F, 0.0F);
    set3(l->basis_y, 0.0F, 1.0F, 0.0F);
    set3(l->basis_z, 0.0F, 0.0F, 1.0F);
    set3(l->axis_u, 1.0F, 0.0F, 0.0F);
    set3(l->axis_v, 0.0F, 1.0F, 0.0F);
    l->width = 1.0F;
    l->height = 1.0F;
    l->radius = 0.5F;
    l->length = 1.0F;
    l->angle = 0.53F;
    l->area = 1.0F;
    l->shaping_cone_angle = 180.0F;
    l->shadow_enable = 1;
    l->shadow_distance = -1.0F;
    l->shadow_falloff = -1.0F;
    l->shadow_falloff_gamma = 1.0F;
}

HDCX_API void hdcx_mesh_defaults(hdcx_mesh_desc* m)
{
    if (!m) return;
    std::memset(m, 0, sizeof(*m));
    m->display_color[0] = m->display_color[1] = m->display_color[2] = 0.5F;
}

HDCX_API hdcx_status hdcx_probe_devices(int32_t* supported, int32_t* deviceCount)
{
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess) count = 0;
    int ok = 0;
    for (int d = 0; d < count; ++d) {
        cudaDeviceProp prop{};
        if (cudaGetDeviceProperties(&prop, d) == cudaSuccess && prop.major == 10) ok = 1;
    }
    if (supported) *supported = ok;
    if (deviceCount) *deviceCount = count;
    return HDCX_OK;
}

HDCX_API hdcx_status hdcx_set_device_memory_limit(int32_t device, uint64_t bytes)
{
    if (device < 0 || device >= 64) return HDCX_ERROR_INVALID_ARGUMENT;
    setDeviceMemoryLimit(device, bytes);
    return HDCX_OK;
}

HDCX_API hdcx_status hdcx_get_device_memory_usage(int32_t device, uint64_t* inUse, uint64_t* limit)
{
    if (device < 0 || device >= 64) return HDCX_ERROR_INVALID_ARGUMENT;
    if (inUse) *inUse = deviceMemoryInUse(device);
    if (limit) *limit = deviceMemoryLimit(device);
    return HDCX_OK;
}

HDCX_API hdcx_status hdcx_test_break_bvh(hdcx_tracer* t)
{
    if (!t) return HDCX_ERROR_INVALID_ARGUMENT;
    if (!t->geometryReady || t->scene.nodes == nullptr || t->scene.nodeCount < 8u)
        return fail(t, HDCX_ERROR_INVALID_ARGUMENT, "hdcx_test_break_bvh: needs a BVH of at least 8 nodes");
    return guarded(t, [&] {
        // WideNode::childBase of node 0: the root's internal children become nodes 0..7.
        static_assert(offsetof(WideNode, childBase) == 16, "WideNode layout");
        const uint32_t zero = 0;
        auto* field = reinterpret_cast<char*>(const_cast<WideNode*>(t->scene.nodes)) + offsetof(WideNode, childBase);
        check(cudaMemcpyAsync(field, &zero, sizeof zero, cudaMemcpyHostToDevice, t->stream), "break BVH");
        check(cudaStreamSynchronize(t->stream), "break BVH");
    });
}

HDCX_API hdcx_status hdcx_create(int32_t device, hdcx_tracer** out)
{
    if (!out) return HDCX_ERROR_INVALID_ARGUMENT;
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) return HDCX_ERROR_NO_DEVICE;
    if (device < 0 || device >= count) return HDCX_ERROR_INVALID_ARGUMENT;
    cudaDeviceProp prop{};
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return HDCX_ERROR_CUDA;
    if (prop.major != 10) return HDCX_ERROR_UNSUPPORTED;  // kernels are built for sm_100a only
    auto* t = new (std::nothrow) hdcx_tracer();
    if (!t) return HDCX_ERROR_OUT_OF_MEMORY;
    t->device = device;
    const hdcx_status s = guarded(t, [&] {
        check(cudaStreamCreateWithFlags(&t->stream, cudaStreamNonBlocking), "cudaStreamCreate");
        check(cudaEventCreate(&t->start), "cudaEventCreate");
        check(cudaEventCreate(&t->stop), "cudaEventCreate");
        float table[256];
        srgbTable(table);
        uploadSrgbTable(table, t->stream);
        check(cudaStreamSynchronize(t->stream), "init");
    });
    if (s != HDCX_OK) {
        delete t;
        return s;
    }
    if (device >= kArenaDevices) {
        delete t;
        return HDCX_ERROR_UNSUPPORTED;
    }
    {
        ArenaPool& pool = arenaPool(device);
        std::lock_guard<std::mutex> guard(pool.lock);
        ++pool.tracers;
    }
    *out = t;
    return HDCX_OK;
}

HDCX_API void hdcx_destroy(hdcx_tracer* t)
{
    if (!t) return;
    const int device = t->device;
    cudaSetDevice(device);
    destroyAsync(t);
    delete t;
    // The device's last tracer takes the path arenas with it.
    ArenaPool& pool = arenaPool(device);
    std::lock_guard<std::mutex> guard(pool.lock);
    if (--pool.tracers == 0) pool.arenas.clear();
}

HDCX_API const char* hdcx_last_error(const hdcx_tracer* t) { return t ? t->lastError.c_str() : ""; }

HDCX_API hdcx_status hdcx_set_scene(hdcx_tracer* t, const hdcx_scene_desc* desc)
{
    return hdcx_set_scene_instanced(t, desc, nullptr, 0);
}

HDCX_API hdcx_status hdcx_set_scene_instanced(hdcx_tracer* t, const hdcx_scene_desc* desc,
                                              const hdcx_instancer_desc* instancers, uint64_t instancerCount)
{
    if (!t) return HDCX_ERROR_INVALID_ARGUMENT;
    return guarded(t, [&] {
        drainAsync(t);
        if (!desc) {
            check(cudaStreamSynchronize(t->stream), "cudaStreamSynchronize");
            t->clearScene();
            return;
        }
        NvtxRange range("hdcx set_scene");
        const auto start = std::chrono::steady_clock::now();
        PackedSceneData d;
        {
            NvtxRange packRange("hdcx pack_scene");
            d = packScene(*desc, instancers, instancerCount);
        }
        uploadScene(t, d);
        t->sceneBuildMs = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - start).count();
    });
}

HDCX_API hdcx_status hdcx_update_instancer_points(hdcx_tracer* t, uint64_t instancer, const float* positions,
                                                  uint64_t positionCount)
{
    if (!t || !positions) return HDCX_ERROR_INVALID_ARGUMENT;
    if (!t->twoLevel || instancer >= t->twoLevel->host.instancers.size())
        return fail(t, HDCX_ERROR_INVALID_ARGUMENT, "hdcx_update_instancer_points: no such instancer in the scene");
    TwoLevel& tl = *t->twoLevel;
    PackedInstancer& pi = tl.host.instancers[instancer];
    if (positionCount != 3u * uint64_t(pi.pointCount()))
        return fail(t, HDCX_ERROR_INVALID_ARGUMENT,
                    "hdcx_update_instancer_points: position_count must be 3 x the mesh's point count (" +
                        std::to_string(3u * uint64_t(pi.pointCount())) + ")");
    return guarded(t, [&] {
        drainAsync(t);
        check(cudaStreamSynchronize(t->stream), "cudaStreamSynchronize");
        for (uint32_t p = 0; p < pi.pointCount(); ++p)
            for (int c = 0; c < 3; ++c) pi.points[4 * p + c] = positions[3 * p + c];
        // The flattened world vertices of every instance and the emissive CDF.
        const std::vector<float> world = instancerWorldPoints(pi);
        std::copy(world.begin(), world.end(), tl.host.vertices.begin() + 4 * size_t(pi.firstVertex));
        recomputeEmissive(tl.host);
        auto* vertices = const_cast<float4*>(t->scene.vertices);
        check(cudaMemcpyAsync(vertices + pi.firstVertex, world.data(), world.size() * sizeof(float), cudaMemcpyHostToDevice,
                              t->stream),
              "update vertices");
        check(cudaMemcpyAsync(const_cast<float4*>(t->scene.emissive), tl.host.emissive.data(),
                              tl.host.emissive.size() * sizeof(float), cudaMemcpyHostToDevice, t->stream),
              "update emissive");
        // Refit of the instancer's bottom level in object space, then a new
        // top level over the moved instances.
        check(cudaMemcpyAsync(tl.objectPoints[instancer], pi.points.data(), pi.points.size() * sizeof(float),
                              cudaMemcpyHostToDevice, t->stream),
              "update object points");
        tl.objectScale[instancer] = pointScale(pi.points.data(), pi.pointCount());
        WideBvh& blas = tl.blases[tl.blasOfInstancer[instancer]];
        refitWideBvh(blas, tl.objectPoints[instancer], tl.objectIndices[instancer], tl.objectScale[instancer], t->stream);
        std::vector<uint32_t> plainVertices;
        if (tl.plainInstance) {
            std::vector<uint8_t> instanced(tl.host.triangleCount(), 0u);
            for (const PackedInstancer& q : tl.host.instancers) {
                const size_t end = size_t(q.firstTriangle) + size_t(q.instanceCount) * q.triangles();
                for (size_t p = q.firstTriangle; p < end; ++p) instanced[p] = 1u;
            }
            for (size_t p = 0; p < instanced.size(); ++p)
                if (!instanced[p])
                    for (int c = 0; c < 3; ++c) plainVertices.push_back(tl.host.indices[3 * p + c]);
        }
        buildTopLevel(t, tl, tl.host, plainVertices);
        check(cudaStreamSynchronize(t->stream), "update instancer");
        t->scene.nodes = tl.top.nodes;
        t->scene.triVerts = tl.top.triVerts;
        t->scene.nodeCount = tl.top.nodeCount;
        const size_t nt = tl.host.triangleCount();
        t->scene.hasMeshLights = (nt > 0 && tl.host.emissive[(nt - 1) * 4u] > 0.0F) ? 1u : 0u;
    });
}

HDCX_API hdcx_status hdcx_set_texture_lod(hdcx_tracer* t, uint32_t mode)
{
    if (!t) return HDCX_ERROR_INVALID_ARGUMENT;
    if (mode > 1u) return fail(t, HDCX_ERROR_INVALID_ARGUMENT, "hdcx_set_texture_lod: mode must be 0 or 1");
    return guarded(t, [&] {
        drainAsync(t);
        t->textureLod = mode;
        if (mode && t->geometryReady && !t->texDescHost.empty()) {
            check(cudaStreamSynchronize(t->stream), "cudaStreamSynchronize");
            buildTextureMips(t);
            check(cudaMemcpyAsync(t->texDescs.ptr, t->texDescHost.data(), t->texDescHost.size() * sizeof(TexDesc),
                                  cudaMemcpyHostToDevice, t->stream),
                  "upload textures");
            check(cudaStreamSynchronize(t->stream), "texture LOD");
        }
    });
}

HDCX_API hdcx_status hdcx_read_texture_level(hdcx_tracer* t, uint32_t texture, uint32_t level, float* rgba,
                                             uint64_t floatCount, uint32_t* width, uint32_t* height)
{
    if (!t) return HDCX_ERROR_INVALID_ARGUMENT;
    if (texture >= t->texDescHost.size())
        return fail(t, HDCX_ERROR_INVALID_ARGUMENT, "hdcx_read_texture_level: no such texture");
    const TexDesc& td = t->texDescHost[texture];
    if (level == 0u || level >= td.levels || td.mips == nullptr)
        return fail(t, HDCX_ERROR_INVALID_ARGUMENT, "hdcx_read_texture_level: no such mip level (levels " +
                                                        std::to_string(td.levels) + "; level 0 is the texture itself)");
    uint32_t w = td.width, h = td.height;
    uint64_t offset = 0;
    for (uint32_t k = 1; k <= level; ++k) {
        const uint32_t nw = std::max(1u, w >> 1), nh = std::max(1u, h >> 1);
        if (k < level) offset += uint64_t(nw) * nh;
        w = nw;
        h = nh;
    }
    if (width) *width = w;
    if (height) *height = h;
    if (!rgba) return HDCX_OK;
    if (floatCount < uint64_t(w) * h * 4u) return fail(t, HDCX_ERROR_INVALID_ARGUMENT, "hdcx_read_texture_level: output too small");
    return guarded(t, [&] {
        check(cudaMemcpyAsync(rgba, td.mips + offset, uint64_t(w) * h * sizeof(float4), cudaMemcpyDefault, t->stream),
              "read mip level");
        check(cudaStreamSynchronize(t->stream), "read mip level");
    });
}

HDCX_API hdcx_status hdcx_get_scene_info(const hdcx_tracer* t, hdcx_scene_info* info)
{
    if (!t || !info) return HDCX_ERROR_INVALID_ARGUMENT;
    *info = hdcx_scene_info{};
    if (!t->geometryReady) return HDCX_OK;
    auto bvhBytes = [](const WideBvh& b) {
        return uint64_t(b.nodeCount) * sizeof(WideNode) + uint64_t(b.triangleCount) * 3u * sizeof(float4);
    };
    info->triangles = t->scene.primitiveCount;
    uint64_t sceneBytes = 0;
    for (const DeviceBuffer* b : t->sceneBuffers) sceneBytes += b->bytes;
    if (t->twoLevel) {
        const TwoLevel& tl = *t->twoLevel;
        info->instances = tl.instances.size();
        info->bottom_levels = tl.blases.size();
        info->bvh_bytes = bvhBytes(tl.top);
        for (const WideBvh& b : tl.blases) info->bvh_bytes += bvhBytes(b);
        for (const DeviceBuffer* b : tl.buffers) sceneBytes += b->bytes;
    } else {
        info->bvh_bytes = bvhBytes(t->bvh);
    }
    info->scene_bytes = sceneBytes + info->bvh_bytes;
    info->build_ms = t->sceneBuildMs;
    info->bvh_build_ms = t->bvhBuildMs;
    return HDCX_OK;
}

HDCX_API hdcx_status hdcx_set_scene_packed(hdcx_tracer* t, const hdcx_packed_scene* view)
{
    if (!t || !view) return HDCX_ERROR_INVALID_ARGUMENT;
    return guarded(t, [&] {
        drainAsync(t);
        uploadScene(t, copyPackedView(*view));
    });
}

HDCX_API hdcx_status hdcx_pack_scene(const hdcx_scene_desc* desc, hdcx_packing** out)
{
    return hdcx_pack_scene_instanced(desc, nullptr, 0, out);
}

HDCX_API hdcx_status hdcx_pack_scene_instanced(const hdcx_scene_desc* desc, const hdcx_instancer_desc* instancers,
                                               uint64_t instancerCount, hdcx_packing** out)
{
    if (!desc || !out) return HDCX_ERROR_INVALID_ARGUMENT;
    *out = nullptr;
    try {
        auto p = std::make_unique<hdcx_packing>();
        p->data = packScene(*desc, instancers, instancerCount);
        makePackedView(p->data, p->textureViews, &p->view);
        *out = p.release();
        return HDCX_OK;
    } catch (const std::bad_alloc&) {
        return HDCX_ERROR_OUT_OF_MEMORY;
    } catch (const std::exception&) {
        return HDCX_ERROR_INVALID_ARGUMENT;
    }
}

HDCX_API const hdcx_packed_scene* hdcx_packing_view(const hdcx_packing* p) { return p ? &p->view : nullptr; }

HDCX_API void hdcx_packing_destroy(hdcx_packing* p) { delete p; }

HDCX_API int32_t hdcx_has_geometry(const hdcx_tracer* t) { return t && t->geometryReady ? 1 : 0; }

HDCX_API hdcx_status hdcx_set_shading_mode(hdcx_tracer* t, int32_t mode)
{
    if (!t) return HDCX_ERROR_INVALID_ARGUMENT;
    if (mode == HDCX_SHADING_RASTER_PREVIEW) {
        return fail(t, HDCX_ERROR_UNSUPPORTED, "raster preview requires the MaterialX graphics backend");
    }
    if (mode != HDCX_SHADING_FUSED && mode != HDCX_SHADING_MODULAR) {
        return fail(t, HDCX_ERROR_INVALID_ARGUMENT, "unknown shading mode");
    }
    t->shadingMode = mode;
    t->lastError.clear();
    return HDCX_OK;
}

HDCX_API int32_t hdcx_get_shading_mode(const hdcx_tracer* t) { return t ? t->shadingMode : HDCX_SHADING_FUSED; }

HDCX_API hdcx_status hdcx_set_profiling(hdcx_tracer* t, uint32_t flags)
{
    if (!t) return HDCX_ERROR_INVALID_ARGUMENT;
    t->profiling = flags;
    return HDCX_OK;
}

HDCX_API hdcx_status hdcx_set_wave_size(hdcx_tracer* t, uint64_t paths)
{
    if (!t) return HDCX_ERROR_INVALID_ARGUMENT;
    if (paths != 0 && paths < 3) return fail(t, HDCX_ERROR_INVALID_ARGUMENT, "a wave holds at least 3 paths");
    t->wavePaths = paths;
    return HDCX_OK;
}

}  // extern "C"

namespace {

void enqueueAovs(hdcx_tracer* t, const FrameConst& frame);

// One render in three phases. prepare: output and path buffers, the fallback
// axis, counters cleared (may allocate and synchronise the tracer's stream).
// enqueue: the kernels and the optional read-back, asynchronous on the
// tracer's stream. finish: wait for the stream, fill the counters.
// hdcx_render runs the phases back to back; hdcx_render_batch runs every
// job's prepare, then every enqueue, then every finish, so that the jobs'
// kernels overlap on the GPU.
struct RenderCall {
    FrameConst frame{};
    PathBuffers paths;  // the buffers this call renders with: the tracer's own, or a batch lane's
    uint64_t pathsNeeded = 0;
    StageTimes times;
    uint64_t launches = 0;
    bool stageTiming = false;
    bool counting = false;
    bool active = false;
};

void prepareRender(hdcx_tracer* t, const hdcx_camera& camera, uint32_t width, uint32_t height, uint32_t sampleIndex,
                   uint32_t maxBounces, uint32_t sampleCount, uint64_t waveCap, bool allowStageTiming,
                   RenderCall& call, PathArena* arena = nullptr, bool fixedArena = false)
{
    ensureOutput(t, width, height);
    if (!t->fallbackAxisInitialized) {
        t->fallbackZUp = std::fabs(camera.vertical[2]) > std::fabs(camera.vertical[1]);
        t->fallbackAxisInitialized = true;
    }
    call.frame = makeFrame(t, camera, width, height, sampleIndex, maxBounces, sampleCount);
    call.pathsNeeded = uint64_t(width) * height * 3u * call.frame.sampleCount;
    // Radiance-cache renders keep path state of their own; the others use the
    // arena checked out for the call (a batch lane's arena is `fixed`).
    PathStore& store = (t->radianceCache || !arena) ? t->own : arena->store;
    const bool fixed = fixedArena && &store != &t->own;
    const uint64_t wave = ensureStore(t, store, call.pathsNeeded, waveCap, fixed);
    call.paths = store.paths;
    call.paths.wavePaths = wave;
    call.paths.stats = tracerStats(t);
    call.paths.traceBlocksPerSm = t->traceBlocksPerSm;
    call.paths.shadeBlocksPerSm = t->shadeBlocksPerSm;
    call.paths.sortHits = t->sortHits;
    call.paths.sortRays = t->sortRays;
    check(cudaMemsetAsync(call.paths.stats, 0, 8 * sizeof(unsigned long long), t->stream), "clear stats");
    call.paths.cache = CacheDevice{};
    if (t->radianceCache) {
        ensureCacheBuffers(t, call.paths.capacity);
        CacheDevice c = t->cacheDevice;
        c.enabled = 1u;
        c.prefixBounces = t->cachePrefix;
        c.spreadFactor = t->cacheSpread;
        const double wave = static_cast<double>(std::min<uint64_t>(call.pathsNeeded, call.paths.wavePaths));
        c.trainThreshold = static_cast<uint32_t>(std::min(4294967295.0, double(t->cacheTrainingPaths) / wave * 4294967296.0));
        c.sceneMin = t->sceneMin;
        c.sceneScale = t->sceneScale;
        call.paths.cache = c;
        t->cacheRun.cache = t->radianceCache->cache;
    }
    call.stageTiming = allowStageTiming && (t->profiling & HDCX_PROFILE_STAGE_TIMES) != 0u;
    call.counting = (t->profiling & HDCX_PROFILE_COUNT_TRAVERSAL) != 0u;
    call.active = true;
}

// `pathsDone` (optional) is recorded once the kernels no longer use the path
// buffers, before the read-back: the next job of a batch lane waits on it.
void enqueueRender(hdcx_tracer* t, RenderCall& call, float* rgbaOut, bool timeEvents = true,
                   cudaEvent_t pathsDone = nullptr)
{
    if (timeEvents) check(cudaEventRecord(t->start, t->stream), "cudaEventRecord");
    renderFrame(t->scene, call.frame, call.paths, t->fb, t->stream, call.stageTiming ? &call.times : nullptr,
                call.counting, &call.launches, t->radianceCache ? &t->cacheRun : nullptr);
    enqueueAovs(t, call.frame);
    if (timeEvents) check(cudaEventRecord(t->stop, t->stream), "cudaEventRecord");
    if (pathsDone) check(cudaEventRecord(pathsDone, t->stream), "cudaEventRecord");
    if (rgbaOut) {
        check(cudaMemcpyAsync(rgbaOut, t->fb.rgba, size_t(call.frame.width) * call.frame.height * sizeof(float4),
                              cudaMemcpyDeviceToHost, t->stream),
              "read back");
    }
}

// The render's traversal fault word (counter 7 of the render's statistics,
// which every traversal kernel ORs its threads' fault bits into): a dropped node
// group or an exhausted node budget means hits may have been lost, so the
// image is not trusted.
void throwOnTraversalFault(unsigned long long word)
{
    const unsigned int bits = static_cast<unsigned int>(word);
    if (bits == 0u) return;
    std::string what = "render: traversal fault:";
    if (bits & kTraversalOverflow) what += " a pending node group found the traversal stack full;";
    if (bits & kTraversalBudget) what += " a ray visited more nodes than the BVH holds (malformed node array);";
    what += " the image may have lost hits";
    throw StatusError(HDCX_ERROR_INTERNAL, what);
}

// `graphMs` >= 0: the render ran inside a batch graph, which measured its device time.
void finishRender(hdcx_tracer* t, RenderCall& call, float graphMs = -1.0F)
{
    {
        NvtxRange range("hdcx wait for render");
        check(cudaStreamSynchronize(t->stream), "render");
    }
    t->xyzSamples = (call.frame.sampleIndex == 0 ? 0 : t->xyzSamples) + call.frame.sampleCount;
    unsigned long long counters[8];
    check(cudaMemcpy(counters, call.paths.stats, sizeof counters, cudaMemcpyDeviceToHost), "read stats");
    throwOnTraversalFault(counters[7]);
    float ms = graphMs;
    if (graphMs < 0.0F) check(cudaEventElapsedTime(&ms, t->start, t->stop), "cudaEventElapsedTime");
    t->stats = hdcx_render_stats{};
    t->stats.spectral_paths = call.pathsNeeded;
    t->stats.extension_rays = counters[0];
    t->stats.shadow_rays = counters[1];
    t->stats.subsurface_rays = counters[2];
    t->stats.render_ms = ms;
    t->stats.extend_ms = call.times.extendMs;
    t->stats.shade_ms = call.times.shadeMs;
    t->stats.shadow_ms = call.times.shadowMs;
    t->stats.waves = call.times.waves;
    t->stats.extend_launches = call.times.extendLaunches;
    t->stats.kernel_launches = call.launches;
    t->stats.extension_node_visits = counters[3];
    t->stats.extension_triangle_tests = counters[4];
    t->stats.shadow_node_visits = counters[5];
    t->stats.shadow_triangle_tests = counters[6];
}

// Device AOVs of a render: the primary hit of the call's first sample (the
// hdcx_trace_primary result for sample `sampleIndex`), when hdcx_set_aovs
// enabled them.
void enqueueAovs(hdcx_tracer* t, const FrameConst& frame)
{
    if (t->aovFlags == 0u) return;
    const size_t pixels = size_t(frame.width) * frame.height;
    if (t->aovWidth != frame.width || t->aovHeight != frame.height || !t->aovIds.ptr) {
        check(cudaStreamSynchronize(t->stream), "cudaStreamSynchronize");
        t->aovIds.allocate(pixels * sizeof(uint32_t));
        t->aovDepth.allocate(pixels * sizeof(float));
        t->aovWidth = frame.width;
        t->aovHeight = frame.height;
    }
    tracePrimary(t->scene, frame, frame.sampleIndex, t->aovIds.as<uint32_t>(), t->aovDepth.as<float>(), t->stream);
}

// ---------------------------------------------------------------------------
// hdcx_render_async: two frames in flight per tracer. A frame renders on the
// tracer's stream, copies its running mean and counters to device staging
// there (so the next frame may overwrite the accumulation), and a second
// stream copies the staging to pinned host memory while the next frame
// renders. Frames complete in ticket order.
// ---------------------------------------------------------------------------
struct AsyncSlot {
    uint64_t ticket = 0;
    bool pending = false;  // enqueued, not yet completed
    bool held = false;     // completed; its host image is valid
    int32_t written = 0;
    ArenaLease lease;
    RenderCall call;
    DeviceBuffer staging, stats;
    float* host = nullptr;  // pinned
    size_t hostBytes = 0;
    unsigned long long* hostStats = nullptr;  // pinned, 8 counters
    cudaEvent_t start = nullptr, stop = nullptr, staged = nullptr, copied = nullptr;
};

struct AsyncFrames {
    cudaStream_t copyStream = nullptr;
    AsyncSlot slot[2];
    uint64_t next = 0;
    ~AsyncFrames()
    {
        if (copyStream) cudaStreamSynchronize(copyStream);
        for (AsyncSlot& s : slot) {
            if (s.host) cudaFreeHost(s.host);
            if (s.hostStats) cudaFreeHost(s.hostStats);
            for (cudaEvent_t e : {s.start, s.stop, s.staged, s.copied})
                if (e) cudaEventDestroy(e);
        }
        if (copyStream) cudaStreamDestroy(copyStream);
    }
};

AsyncFrames& asyncFrames(hdcx_tracer* t)
{
    if (!t->async) {
        auto a = std::make_unique<AsyncFrames>();
        check(cudaStreamCreateWithFlags(&a->copyStream, cudaStreamNonBlocking), "cudaStreamCreate");
        for (AsyncSlot& s : a->slot) {
            check(cudaEventCreate(&s.start), "cudaEventCreate");
            check(cudaEventCreate(&s.stop), "cudaEventCreate");
            check(cudaEventCreateWithFlags(&s.staged, cudaEventDisableTiming), "cudaEventCreate");
            check(cudaEventCreateWithFlags(&s.copied, cudaEventDisableTiming), "cudaEventCreate");
            check(cudaHostAlloc(reinterpret_cast<void**>(&s.hostStats), 8 * sizeof(unsigned long long),
                                cudaHostAllocDefault),
                  "cudaHostAlloc");
        }
        t->async = a.release();
    }
    return *t->async;
}

// Waits for a pending frame and takes its counters and device time into the
// tracer's stats, as finishRender does for hdcx_render.
void completeAsync(hdcx_tracer* t, AsyncSlot& s)
{
    if (!s.pending) return;
    s.pending = false;
    s.held = true;
    if (!s.written) return;
    const cudaError_t e = cudaEventSynchronize(s.copied);
    s.lease = ArenaLease{};
    check(e, "hdcx_render_async frame");
    t->xyzSamples = (s.call.frame.sampleIndex == 0 ? 0 : t->xyzSamples) + s.call.frame.sampleCount;
    float ms = 0.0F;
    check(cudaEventElapsedTime(&ms, s.start, s.stop), "cudaEventElapsedTime");
    const unsigned long long* c = s.hostStats;
    t->stats = hdcx_render_stats{};
    t->stats.spectral_paths = s.call.pathsNeeded;
    t->stats.extension_rays = c[0];
    t->stats.shadow_rays = c[1];
    t->stats.subsurface_rays = c[2];
    t->stats.render_ms = ms;
    t->stats.kernel_launches = s.call.launches;
    t->stats.extension_node_visits = c[3];
    t->stats.extension_triangle_tests = c[4];
    t->stats.shadow_node_visits = c[5];
    t->stats.shadow_triangle_tests = c[6];
    throwOnTraversalFault(c[7]);
}

// Completes every pending frame with a ticket up to `last`, oldest first.
void completeAsyncUpTo(hdcx_tracer* t, uint64_t last)
{
    if (!t->async) return;
    for (;;) {
        AsyncSlot* oldest = nullptr;
        for (AsyncSlot& s : t->async->slot)
            if (s.pending && s.ticket <= last && (!oldest || s.ticket < oldest->ticket)) oldest = &s;
        if (!oldest) return;
        completeAsync(t, *oldest);
    }
}

void drainAsync(hdcx_tracer* t) { completeAsyncUpTo(t, ~0ull); }

void destroyAsync(hdcx_tracer* t)
{
    if (!t->async) return;
    try {
        drainAsync(t);
    } catch (const std::exception&) {
    }
    delete t->async;
    t->async = nullptr;
}

void enqueueAsync(hdcx_tracer* t, const hdcx_camera& camera, uint32_t width, uint32_t height, uint32_t sampleIndex,
                  uint32_t maxBounces, uint32_t sampleCount, uint64_t* ticket)
{
    AsyncFrames& a = asyncFrames(t);
    AsyncSlot& s = a.slot[a.next % 2u];
    // The slot's previous frame (two tickets back) completes, and its host
    // image is given up, before this frame takes the slot.
    completeAsyncUpTo(t, s.ticket);
    s.held = false;
    s.written = 0;
    s.ticket = a.next++;
    s.call = RenderCall{};
    if (t->geometryReady && width > 0 && height > 0) {
        ArenaLease lease;
        if (!t->radianceCache) lease = checkoutArena(t->device, true);
        prepareRender(t, camera, width, height, sampleIndex, maxBounces, sampleCount, 0, false, s.call, lease.arena);
        const size_t bytes = size_t(width) * height * sizeof(float4);
        if (s.hostBytes < bytes) {
            if (s.host) check(cudaFreeHost(s.host), "cudaFreeHost");
            s.host = nullptr;
            s.hostBytes = 0;
            check(cudaHostAlloc(reinterpret_cast<void**>(&s.host), bytes, cudaHostAllocDefault), "cudaHostAlloc");
            s.hostBytes = bytes;
        }
        if (s.staging.bytes < bytes) s.staging.allocate(bytes);
        if (!s.stats.ptr) s.stats.allocate(8 * sizeof(unsigned long long));
        check(cudaEventRecord(s.start, t->stream), "cudaEventRecord");
        enqueueRender(t, s.call, nullptr, false);
        check(cudaEventRecord(s.stop, t->stream), "cudaEventRecord");
        check(cudaMemcpyAsync(s.staging.ptr, t->fb.rgba, bytes, cudaMemcpyDeviceToDevice, t->stream), "stage frame");
        check(cudaMemcpyAsync(s.stats.ptr, s.call.paths.stats, 8 * sizeof(unsigned long long), cudaMemcpyDeviceToDevice,
                              t->stream),
              "stage counters");
        check(cudaEventRecord(s.staged, t->stream), "cudaEventRecord");
        check(cudaStreamWaitEvent(a.copyStream, s.staged, 0), "cudaStreamWaitEvent");
        check(cudaMemcpyAsync(s.host, s.staging.ptr, bytes, cudaMemcpyDeviceToHost, a.copyStream), "read back frame");
        check(cudaMemcpyAsync(s.hostStats, s.stats.ptr, 8 * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                              a.copyStream),
              "read back counters");
        check(cudaEventRecord(s.copied, a.copyStream), "cudaEventRecord");
        s.lease = std::move(lease);
        s.written = 1;
    }
    s.pending = true;
    *ticket = s.ticket;
}

// Nearest-neighbour upscale of the interactive preview: the reference's
// UpscaleNearest (render_pass.cpp:45-68) on the device.
void upscalePreview(hdcx_tracer* t, uint32_t traceWidth, uint32_t traceHeight, uint32_t width, uint32_t height)
{
    const size_t bytes = size_t(width) * height * sizeof(float4);
    if (t->preview.bytes < bytes) {
        check(cudaStreamSynchronize(t->stream), "cudaStreamSynchronize");
        t->preview.allocate(bytes);
    }
    launchUpscaleNearest(t->fb.rgba, traceWidth, traceHeight, t->preview.as<float4>(), width, height, t->stream);
}

}  // namespace

extern "C" {

HDCX_API hdcx_status hdcx_render(hdcx_tracer* t, const hdcx_camera* camera, uint32_t width, uint32_t height,
                                 uint32_t sampleIndex, uint32_t maxBounces, uint32_t sampleCount, float* rgbaOut,
                                 int32_t* written)
{
    if (!t || !camera) return HDCX_ERROR_INVALID_ARGUMENT;
    if (written) *written = 0;
    if (!t->geometryReady || width == 0 || height == 0) return HDCX_OK;
    if (uint64_t(width) * height > (1ull << 28)) return fail(t, HDCX_ERROR_INVALID_ARGUMENT, "image larger than 2^28 pixels");
    return guarded(t, [&] {
        drainAsync(t);
        NvtxRange range("hdcx render");
        // The arena stays checked out until the render's work has finished.
        ArenaLease lease;
        if (!t->radianceCache) lease = checkoutArena(t->device, true);
        RenderCall call;
        prepareRender(t, *camera, width, height, sampleIndex, maxBounces, sampleCount, 0, true, call, lease.arena);
        enqueueRender(t, call, rgbaOut);
        finishRender(t, call);
        if (written) *written = 1;
    });
}

HDCX_API hdcx_status hdcx_render_preview(hdcx_tracer* t, const hdcx_camera* camera, uint32_t width, uint32_t height,
                                         float* rgbaOut, int32_t* written)
{
    if (!t || !camera) return HDCX_ERROR_INVALID_ARGUMENT;
    if (written) *written = 0;
    if (!t->geometryReady || width == 0 || height == 0) return HDCX_OK;
    if (uint64_t(width) * height > (1ull << 28)) return fail(t, HDCX_ERROR_INVALID_ARGUMENT, "image larger than 2^28 pixels");
    // render_pass.cpp:191-208: half resolution (rounded up), sample 0, two
    // bounces, one sample, upscaled by nearest neighbour.
    constexpr uint32_t kScale = 2u, kBounces = 2u;
    const uint32_t traceWidth = std::max(1u, (width + kScale - 1u) / kScale);
    const uint32_t traceHeight = std::max(1u, (height + kScale - 1u) / kScale);
    return guarded(t, [&] {
        drainAsync(t);
        ArenaLease lease;
        if (!t->radianceCache) lease = checkoutArena(t->device, true);
        RenderCall call;
        prepareRender(t, *camera, traceWidth, traceHeight, 0u, kBounces, 1u, 0, true, call, lease.arena);
        enqueueRender(t, call, nullptr);
        upscalePreview(t, traceWidth, traceHeight, width, height);
        if (rgbaOut) {
            check(cudaMemcpyAsync(rgbaOut, t->preview.ptr, size_t(width) * height * sizeof(float4), cudaMemcpyDefault,
                                  t->stream),
                  "read back preview");
        }
        finishRender(t, call);
        if (written) *written = 1;
    });
}

HDCX_API hdcx_status hdcx_device_preview(hdcx_tracer* t, const float** device)
{
    if (!t || !device) return HDCX_ERROR_INVALID_ARGUMENT;
    *device = t->preview.as<float>();
    return HDCX_OK;
}

HDCX_API hdcx_status hdcx_render_async(hdcx_tracer* t, const hdcx_camera* camera, uint32_t width, uint32_t height,
                                       uint32_t sampleIndex, uint32_t maxBounces, uint32_t sampleCount, uint64_t* ticket)
{
    if (!t || !camera || !ticket) return HDCX_ERROR_INVALID_ARGUMENT;
    if (uint64_t(width) * height > (1ull << 28)) return fail(t, HDCX_ERROR_INVALID_ARGUMENT, "image larger than 2^28 pixels");
    return guarded(t, [&] { enqueueAsync(t, *camera, width, height, sampleIndex, maxBounces, sampleCount, ticket); });
}

HDCX_API hdcx_status hdcx_wait_render(hdcx_tracer* t, uint64_t ticket, const float** hostRgba, int32_t* written)
{
    if (!t) return HDCX_ERROR_INVALID_ARGUMENT;
    if (hostRgba) *hostRgba = nullptr;
    if (written) *written = 0;
    AsyncSlot* slot = nullptr;
    if (t->async) {
        for (AsyncSlot& s : t->async->slot)
            if ((s.pending || s.held) && s.ticket == ticket) slot = &s;
    }
    if (!slot) return fail(t, HDCX_ERROR_INVALID_ARGUMENT, "hdcx_wait_render: the ticket is not held (a frame's image is "
                                                          "kept until the call two tickets later)");
    return guarded(t, [&] {
        completeAsyncUpTo(t, ticket);
        if (hostRgba && slot->written) *hostRgba = slot->host;
        if (written) *written = slot->written;
    });
}

HDCX_API hdcx_status hdcx_set_aovs(hdcx_tracer* t, uint32_t flags)
{
    if (!t) return HDCX_ERROR_INVALID_ARGUMENT;
    if ((flags & ~(HDCX_AOV_PRIMITIVE_ID | HDCX_AOV_DEPTH)) != 0u)
        return fail(t, HDCX_ERROR_INVALID_ARGUMENT, "hdcx_set_aovs: unknown AOV flags");
    t->aovFlags = flags;
    return HDCX_OK;
}

HDCX_API hdcx_status hdcx_read_aovs(hdcx_tracer* t, uint32_t* primitiveOut, float* depthOut, uint64_t pixelCount)
{
    if (!t) return HDCX_ERROR_INVALID_ARGUMENT;
    return guarded(t, [&] {
        drainAsync(t);
        const uint64_t n = uint64_t(t->aovWidth) * t->aovHeight;
        if (n == 0 || !t->aovIds.ptr) throw std::invalid_argument("hdcx_read_aovs: no render has written AOVs");
        if (pixelCount < n) throw std::invalid_argument("hdcx_read_aovs: output smaller than width*height");
        if (primitiveOut)
            check(cudaMemcpyAsync(primitiveOut, t->aovIds.ptr, n * sizeof(uint32_t), cudaMemcpyDefault, t->stream), "read ids");
        if (depthOut)
            check(cudaMemcpyAsync(depthOut, t->aovDepth.ptr, n * sizeof(float), cudaMemcpyDefault, t->stream), "read depth");
        check(cudaStreamSynchronize(t->stream), "read AOVs");
    });
}

HDCX_API hdcx_status hdcx_render_batch(hdcx_batch_job* jobs, uint32_t count, uint64_t pathBudget)
{
    return hdcx_render_batch_ex(jobs, count, pathBudget, 0u);
}

}  // extern "C"

namespace {

// A batch renders the jobs of each device in up to kBatchLanes lanes that run
// concurrently. The jobs of a lane run one after another on the lane's path
// buffers, which belong to the lane's first tracer and hold up to
// kBatchLaneWave paths: waves as large as a single render's, where one set of
// buffers per job would split the device memory among all the jobs.
constexpr uint32_t kBatchLanes = 4;
constexpr uint64_t kBatchLaneWave = 48ull << 20;

struct BatchPlan {
    std::vector<uint32_t> order;     // jobs in enqueue order, lane by lane
    std::vector<int> lane;           // per job: its lane, or -1 (the tracer's own path state)
    std::vector<ArenaLease> leases;  // per lane: its arena, held until the batch's work has finished
};

// Deals the jobs that can share path state (geometry, a non-empty image, no
// radiance cache) to lanes, largest first onto the lane with the fewest paths,
// and sizes each lane's arena: its largest job's paths, at most kBatchLaneWave
// and at most an equal share of the budget (`pathBudget` paths per device, 0:
// half the device's free memory), never below 1,048,576 paths (planLanes,
// batch_plan.h, holds these rules). Lanes take the
// arenas that are free; only a batch that holds none yet waits for one, so
// concurrent batches cannot wait on each other. Jobs left without a lane (no
// arena, or its buffers could not be allocated) render on their own path state.
BatchPlan planBatch(hdcx_batch_job* jobs, uint32_t count, uint64_t pathBudget)
{
    BatchPlan plan;
    plan.lane.assign(count, -1);
    auto need = [&](uint32_t j) {
        const hdcx_batch_job& b = jobs[j];
        return uint64_t(b.width) * b.height * 3u * std::max(b.sample_count, 1u);
    };
    std::vector<int> devices;
    for (uint32_t j = 0; j < count; ++j) {
        if (std::find(devices.begin(), devices.end(), jobs[j].tracer->device) == devices.end())
            devices.push_back(jobs[j].tracer->device);
    }
    for (int device : devices) {
        std::vector<uint32_t> eligible;
        for (uint32_t j = 0; j < count; ++j) {
            const hdcx_batch_job& b = jobs[j];
            const hdcx_tracer* t = b.tracer;
            if (t->device == device && t->geometryReady && !t->radianceCache && b.width > 0 && b.height > 0 &&
                uint64_t(b.width) * b.height <= (1ull << 28))
                eligible.push_back(j);
        }
        if (eligible.empty() || cudaSetDevice(device) != cudaSuccess) continue;
        std::vector<ArenaLease> leases;
        const size_t wanted = std::min<size_t>(kBatchLanes, eligible.size());
        try {
            while (leases.size() < wanted) {
                ArenaLease lease = checkoutArena(device, false);
                if (!lease.arena) break;
                leases.push_back(std::move(lease));
            }
            if (leases.empty() && plan.leases.empty()) leases.push_back(checkoutArena(device, true));
        } catch (const std::exception&) {
        }
        if (leases.empty()) continue;
        const uint32_t lanes = static_cast<uint32_t>(leases.size());
        uint64_t budget = pathBudget;
        if (budget == 0) {
            size_t freeBytes = 0, totalBytes = 0;
            if (cudaMemGetInfo(&freeBytes, &totalBytes) != cudaSuccess) freeBytes = 0;
            uint64_t held = 0;
            for (const ArenaLease& l : leases) held += l.arena->store.paths.capacity * kPathStateBytes;
            budget = (freeBytes + held) / 2 / kPathStateBytes;
        }
        std::vector<uint64_t> paths;
        for (uint32_t j : eligible) paths.push_back(need(j));
        const LanePlan lanePlan = planLanes(paths, lanes, budget, kBatchLaneWave, 1ull << 20);
        for (uint32_t l = 0; l < lanes; ++l) {
            std::vector<uint32_t> members;
            for (uint32_t k : lanePlan.members[l]) members.push_back(eligible[k]);
            const uint64_t capacity = lanePlan.capacity[l];
            PathStore& store = leases[l].arena->store;
            bool ready = true;
            try {
                if (store.paths.capacity < capacity || store.paths.shadowPerPath < 3u) store.allocate(capacity, 3u);
            } catch (const std::exception&) {
                store.release();
                cudaGetLastError();
                ready = false;
            }
            if (!ready) {
                for (uint32_t j : members) plan.order.push_back(j);
                continue;
            }
            const int index = static_cast<int>(plan.leases.size());
            plan.leases.push_back(std::move(leases[l]));
            for (uint32_t j : members) {
                plan.lane[j] = index;
                plan.order.push_back(j);
            }
        }
    }
    for (uint32_t j = 0; j < count; ++j) {
        if (std::find(plan.order.begin(), plan.order.end(), j) == plan.order.end()) plan.order.push_back(j);
    }
    return plan;
}

// Events of one batch call, destroyed with it.
struct BatchEvents {
    std::vector<cudaEvent_t> events;
    explicit BatchEvents(uint32_t count) : events(count, nullptr) {}
    BatchEvents(const BatchEvents&) = delete;
    BatchEvents& operator=(const BatchEvents&) = delete;
    ~BatchEvents()
    {
        for (cudaEvent_t e : events)
            if (e) cudaEventDestroy(e);
    }
    cudaEvent_t make(uint32_t j)
    {
        if (!events[j]) check(cudaEventCreateWithFlags(&events[j], cudaEventDisableTiming), "cudaEventCreate");
        return events[j];
    }
};

// The batch graph of a device, kept between calls: the executable graph of
// the last batch (updated in place with cudaGraphExecUpdate when the next
// batch has the same launch topology, instantiated anew otherwise), the
// capture stream and the events the graph records. One batch at a time per
// device uses it.
struct BatchGraphCache {
    std::mutex lock;
    cudaGraphExec_t exec = nullptr;
    cudaStream_t stream = nullptr;
    cudaEvent_t fork = nullptr, start = nullptr, stop = nullptr;
    std::vector<cudaEvent_t> jobStart, jobStop;  // timing events per job slot (event-record nodes of the graph)
    std::vector<cudaEvent_t> jobDone;            // per job slot: ordering only (lane order, the join)
    uint64_t instantiations = 0, updates = 0;
};

BatchGraphCache& batchGraphCache(int device)
{
    static BatchGraphCache* caches = new BatchGraphCache[kArenaDevices];  // never destroyed, like the arenas
    return caches[device];
}

// Captures the kernels of every active job (each on its own tracer's stream,
// forked from and joined into one capture stream) into a CUDA graph, brings
// the device's cached executable graph up to date with it (or instantiates
// one), launches it, then queues the read-backs. Returns the graph's device
// time and, in jobMs, each job's device time from its first to its last
// kernel (events recorded inside the graph; jobs overlap, so these do not add
// up to the graph's time); a negative value (nothing launched) when the batch
// cannot be captured: jobs on several devices, a job in radiance-cache mode
// (it synchronises with the host per wave) or a capture error. A launch,
// synchronisation or read-back error after instantiation sets the affected
// jobs' status to HDCX_ERROR_CUDA and takes them out of the batch.
float enqueueBatchGraph(hdcx_batch_job* jobs, uint32_t count, std::vector<RenderCall>& calls, const BatchPlan& plan,
                        std::vector<float>& jobMs)
{
    int device = -1;
    for (uint32_t j = 0; j < count; ++j) {
        if (!calls[j].active) continue;
        hdcx_tracer* t = jobs[j].tracer;
        if (t->radianceCache || (device >= 0 && t->device != device)) return -1.0F;
        device = t->device;
    }
    if (device < 0 || device >= kArenaDevices || cudaSetDevice(device) != cudaSuccess) return -1.0F;
    // The prepare phase queued clears on the tracers' streams; the graph runs
    // on its own stream, so they must have finished.
    for (uint32_t j = 0; j < count; ++j) {
        if (calls[j].active && cudaStreamSynchronize(jobs[j].tracer->stream) != cudaSuccess) return -1.0F;
    }
    BatchGraphCache& cache = batchGraphCache(device);
    std::lock_guard<std::mutex> hold(cache.lock);
    if (!cache.stream) {
        if (cudaStreamCreateWithFlags(&cache.stream, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&cache.fork, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreate(&cache.start) != cudaSuccess || cudaEventCreate(&cache.stop) != cudaSuccess) {
            cudaGetLastError();
            return -1.0F;
        }
    }
    while (cache.jobStart.size() < count) {
        cudaEvent_t a = nullptr, b = nullptr, c = nullptr;
        if (cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&b) != cudaSuccess ||
            cudaEventCreateWithFlags(&c, cudaEventDisableTiming) != cudaSuccess) {
            if (a) cudaEventDestroy(a);
            if (b) cudaEventDestroy(b);
            cudaGetLastError();
            return -1.0F;
        }
        cache.jobStart.push_back(a);
        cache.jobStop.push_back(b);
        cache.jobDone.push_back(c);
    }
    bool captured = cudaStreamBeginCapture(cache.stream, cudaStreamCaptureModeRelaxed) == cudaSuccess;
    try {
        if (captured) {
            check(cudaEventRecord(cache.fork, cache.stream), "fork");
            // A job starts after the fork, or after the previous job of its
            // lane (its stop event, recorded after its last kernel).
            std::vector<int> laneLast(plan.leases.size(), -1);
            for (uint32_t j : plan.order) {
                if (!calls[j].active) continue;
                hdcx_tracer* t = jobs[j].tracer;
                const int lane = plan.lane[j];
                const bool afterLane = lane >= 0 && laneLast[lane] >= 0;
                check(cudaStreamWaitEvent(t->stream, afterLane ? cache.jobDone[laneLast[lane]] : cache.fork, 0),
                      "join the capture");
                // Timing events become event-record nodes of the graph (a
                // plain record inside a capture only orders the streams).
                check(cudaEventRecordWithFlags(cache.jobStart[j], t->stream, cudaEventRecordExternal), "job start");
                enqueueRender(t, calls[j], nullptr, false);
                check(cudaEventRecordWithFlags(cache.jobStop[j], t->stream, cudaEventRecordExternal), "job stop");
                check(cudaEventRecord(cache.jobDone[j], t->stream), "job done");
                check(cudaStreamWaitEvent(cache.stream, cache.jobDone[j], 0), "join");
                if (lane >= 0) laneLast[lane] = static_cast<int>(j);
            }
        }
    } catch (const std::exception&) {
        captured = false;
    }
    cudaGraph_t graph = nullptr;
    const cudaError_t end = cudaStreamEndCapture(cache.stream, &graph);
    bool ready = captured && end == cudaSuccess && graph != nullptr;
    if (ready && cache.exec) {
        cudaGraphExecUpdateResultInfo info{};
        if (cudaGraphExecUpdate(cache.exec, graph, &info) == cudaSuccess) {
            cache.updates++;
        } else {
            cudaGetLastError();
            cudaGraphExecDestroy(cache.exec);
            cache.exec = nullptr;
        }
    }
    if (ready && !cache.exec) {
        if (cudaGraphInstantiate(&cache.exec, graph, 0) == cudaSuccess) {
            cache.instantiations++;
        } else {
            cache.exec = nullptr;
            ready = false;
        }
    }
    if (graph) cudaGraphDestroy(graph);
    if (!ready) {
        cudaGetLastError();
        return -1.0F;
    }
    // Once the graph is launched the jobs' work is committed to it: a failure
    // from here on fails every job of the graph (its images are not valid),
    // and is not retried on the streams.
    float ms = -1.0F;
    cudaError_t err = cudaEventRecord(cache.start, cache.stream);
    if (err == cudaSuccess) err = cudaGraphLaunch(cache.exec, cache.stream);
    if (err == cudaSuccess) err = cudaEventRecord(cache.stop, cache.stream);
    if (err == cudaSuccess) err = cudaStreamSynchronize(cache.stream);
    if (err == cudaSuccess) err = cudaEventElapsedTime(&ms, cache.start, cache.stop);
    jobMs.assign(count, 0.0F);
    for (uint32_t j = 0; j < count; ++j) {
        if (!calls[j].active) continue;
        hdcx_tracer* t = jobs[j].tracer;
        cudaError_t jobErr = err;
        if (jobErr == cudaSuccess) jobErr = cudaEventElapsedTime(&jobMs[j], cache.jobStart[j], cache.jobStop[j]);
        if (jobErr == cudaSuccess && jobs[j].rgba_out) {
            jobErr = cudaMemcpyAsync(jobs[j].rgba_out, t->fb.rgba,
                                     size_t(calls[j].frame.width) * calls[j].frame.height * sizeof(float4),
                                     cudaMemcpyDeviceToHost, t->stream);
        }
        if (jobErr != cudaSuccess) {
            jobs[j].status = fail(t, HDCX_ERROR_CUDA, std::string("hdcx_render_batch (CUDA graph): ") +
                                                           cudaGetErrorString(jobErr));
            calls[j].active = false;
            cudaGetLastError();
        }
    }
    if (err != cudaSuccess) cudaGetLastError();
    return ms < 0.0F ? 0.0F : ms;
}

}  // namespace

extern "C" {

HDCX_API hdcx_status hdcx_get_batch_graph_stats(int32_t device, uint64_t* instantiations, uint64_t* updates)
{
    if (device < 0 || device >= kArenaDevices) return HDCX_ERROR_INVALID_ARGUMENT;
    BatchGraphCache& cache = batchGraphCache(device);
    std::lock_guard<std::mutex> hold(cache.lock);
    if (instantiations) *instantiations = cache.instantiations;
    if (updates) *updates = cache.updates;
    return HDCX_OK;
}

HDCX_API hdcx_status hdcx_render_batch_ex(hdcx_batch_job* jobs, uint32_t count, uint64_t pathBudget, uint32_t flags)
{
    if (count == 0) return HDCX_OK;
    if (!jobs) return HDCX_ERROR_INVALID_ARGUMENT;
    for (uint32_t j = 0; j < count; ++j) {
        jobs[j].status = HDCX_OK;
        jobs[j].written = 0;
        jobs[j].render_ms = 0.0;
        if (!jobs[j].tracer) return HDCX_ERROR_INVALID_ARGUMENT;
        for (uint32_t k = 0; k < j; ++k) {
            if (jobs[k].tracer == jobs[j].tracer) {
                return fail(jobs[j].tracer, HDCX_ERROR_INVALID_ARGUMENT,
                            "hdcx_render_batch: a tracer appears in more than one job of the batch");
            }
        }
    }
    for (uint32_t j = 0; j < count; ++j) {
        hdcx_tracer* t = jobs[j].tracer;
        if (t->async) {
            const hdcx_status drained = guarded(t, [&] { drainAsync(t); });
            if (drained != HDCX_OK) return drained;
        }
    }
    NvtxRange range("hdcx render_batch");
    std::vector<RenderCall> calls(count);
    auto record = [&](uint32_t j, hdcx_status status) {
        if (status != HDCX_OK) {
            jobs[j].status = status;
            calls[j].active = false;
        }
    };
    const BatchPlan plan = planBatch(jobs, count, pathBudget);
    for (uint32_t j : plan.order) {
        hdcx_batch_job& b = jobs[j];
        hdcx_tracer* t = b.tracer;
        if (!t->geometryReady || b.width == 0 || b.height == 0) continue;
        if (uint64_t(b.width) * b.height > (1ull << 28)) {
            record(j, fail(t, HDCX_ERROR_INVALID_ARGUMENT, "image larger than 2^28 pixels"));
            continue;
        }
        PathArena* arena = plan.lane[j] >= 0 ? plan.leases[plan.lane[j]].arena : nullptr;
        const uint64_t laneWave = arena ? arena->store.paths.capacity : 0;
        record(j, guarded(t, [&] {
            prepareRender(t, b.camera, b.width, b.height, b.sample_index, b.max_bounces, b.sample_count, laneWave,
                          false, calls[j], arena, true);
        }));
    }
    BatchEvents events(count);
    std::vector<float> jobMs;
    const float graphMs = (flags & HDCX_BATCH_CUDA_GRAPH) ? enqueueBatchGraph(jobs, count, calls, plan, jobMs) : -1.0F;
    if (graphMs < 0.0F) {
        // Lane by lane: a job waits until the previous job of its lane no
        // longer uses the lane's path buffers.
        std::vector<cudaEvent_t> laneDone(plan.leases.size(), nullptr);
        for (uint32_t j : plan.order) {
            if (!calls[j].active) continue;
            hdcx_tracer* t = jobs[j].tracer;
            const int lane = plan.lane[j];
            cudaEvent_t done = nullptr;
            const hdcx_status st = guarded(t, [&] {
                if (lane >= 0) {
                    done = events.make(j);
                    if (laneDone[lane]) check(cudaStreamWaitEvent(t->stream, laneDone[lane], 0), "lane order");
                }
                enqueueRender(t, calls[j], jobs[j].rgba_out, true, done);
            });
            if (lane >= 0 && done) {
                // A job that failed part-way may have launched kernels on the
                // arena: the lane's next job waits for its stream all the same.
                if (st != HDCX_OK) cudaEventRecord(done, t->stream);
                laneDone[lane] = done;
            }
            record(j, st);
        }
    }
    hdcx_status overall = HDCX_OK;
    for (uint32_t j = 0; j < count; ++j) {
        if (calls[j].active) {
            record(j, guarded(jobs[j].tracer, [&] {
                finishRender(jobs[j].tracer, calls[j], graphMs < 0.0F ? -1.0F : jobMs[j]);
                jobs[j].written = 1;
                jobs[j].render_ms = jobs[j].tracer->stats.render_ms;
            }));
        }
        if (overall == HDCX_OK && jobs[j].status != HDCX_OK) overall = jobs[j].status;
    }
    return overall;
}

HDCX_API hdcx_status hdcx_render_static(hdcx_tracer* t, const hdcx_camera* camera, uint32_t width, uint32_t height,
                                        uint32_t sampleIndex, uint32_t maxBounces, uint32_t sampleCount,
                                        float* rgbaDevice, int32_t* written)
{
    if (!t || !camera || !rgbaDevice) return HDCX_ERROR_INVALID_ARGUMENT;
    if (written) *written = 0;
    if (t->async) {
        const hdcx_status drained = guarded(t, [&] { drainAsync(t); });
        if (drained != HDCX_OK) return drained;
    }
    if (!t->geometryReady || width == 0 || height == 0) return HDCX_OK;
    if (uint64_t(width) * height > kStaticMaxPixels) {
        return fail(t, HDCX_ERROR_INVALID_ARGUMENT,
                    "hdcx_render_static: width*height = " + std::to_string(uint64_t(width) * height) +
                        " exceeds its maximum of " + std::to_string(kStaticMaxPixels) + " pixels");
    }
    if (reinterpret_cast<uintptr_t>(rgbaDevice) % 16u != 0u)
        return fail(t, HDCX_ERROR_INVALID_ARGUMENT, "hdcx_render_static: rgba_device must be 16-byte aligned");
    if (t->radianceCache) {
        return fail(t, HDCX_ERROR_INVALID_ARGUMENT,
                    "hdcx_render_static: the tracer has a radiance cache attached; the static render has no cache "
                    "mode (detach it with hdcx_set_radiance_cache(tracer, NULL, ...) or use hdcx_render)");
    }
    return guarded(t, [&] {
        if (!t->fallbackAxisInitialized) {
            t->fallbackZUp = std::fabs(camera->vertical[2]) > std::fabs(camera->vertical[1]);
            t->fallbackAxisInitialized = true;
        }
        const FrameConst f = makeFrame(t, *camera, width, height, sampleIndex, maxBounces, sampleCount);
        throwOnTraversalFault(renderStatic(t->scene, f, reinterpret_cast<float4*>(rgbaDevice), t->stream));
        if (written) *written = 1;
    });
}

HDCX_API hdcx_status hdcx_read_rgba(hdcx_tracer* t, float* out, uint64_t count)
{
    if (!t || !out) return HDCX_ERROR_INVALID_ARGUMENT;
    return guarded(t, [&] {
        const uint64_t n = uint64_t(t->fb.width) * t->fb.height * 4u;
        if (count < n || !t->fb.rgba) throw std::invalid_argument("output buffer smaller than width*height*4");
        check(cudaMemcpyAsync(out, t->fb.rgba, n * sizeof(float), cudaMemcpyDeviceToHost, t->stream), "read rgba");
        check(cudaStreamSynchronize(t->stream), "read rgba");
    });
}

HDCX_API hdcx_status hdcx_read_xyz(hdcx_tracer* t, double* out, uint64_t count, uint64_t* samples)
{
    if (!t || !out) return HDCX_ERROR_INVALID_ARGUMENT;
    return guarded(t, [&] {
        const uint64_t n = uint64_t(t->fb.width) * t->fb.height * 3u;
        if (count < n || !t->fb.xyz) throw std::invalid_argument("output buffer smaller than width*height*3");
        check(cudaMemcpyAsync(out, t->fb.xyz, n * sizeof(double), cudaMemcpyDeviceToHost, t->stream), "read xyz");
        check(cudaStreamSynchronize(t->stream), "read xyz");
        if (samples) *samples = t->xyzSamples;
    });
}

HDCX_API hdcx_status hdcx_device_rgba(hdcx_tracer* t, const float** device)
{
    if (!t || !device) return HDCX_ERROR_INVALID_ARGUMENT;
    *device = reinterpret_cast<const float*>(t->fb.rgba);
    return HDCX_OK;
}

HDCX_API hdcx_status hdcx_trace_primary(hdcx_tracer* t, const hdcx_camera* camera, uint32_t width, uint32_t height,
                                        uint32_t sampleNumber, uint32_t* primitiveOut, float* distanceOut)
{
    if (!t || !camera || !primitiveOut) return HDCX_ERROR_INVALID_ARGUMENT;
    if (!t->geometryReady) return fail(t, HDCX_ERROR_INVALID_ARGUMENT, "no geometry");
    if (width == 0 || height == 0) return HDCX_OK;
    return guarded(t, [&] {
        const size_t pixels = size_t(width) * height;
        DeviceBuffer prims, dists;
        prims.allocate(pixels * sizeof(uint32_t));
        dists.allocate(pixels * sizeof(float));
        const FrameConst f = makeFrame(t, *camera, width, height, 0u, 1u, 1u);
        tracePrimary(t->scene, f, sampleNumber, prims.as<uint32_t>(), dists.as<float>(), t->stream);
        check(cudaMemcpyAsync(primitiveOut, prims.ptr, pixels * sizeof(uint32_t), cudaMemcpyDeviceToHost, t->stream), "read ids");
        if (distanceOut) {
            check(cudaMemcpyAsync(distanceOut, dists.ptr, pixels * sizeof(float), cudaMemcpyDeviceToHost, t->stream), "read t");
        }
        check(cudaStreamSynchronize(t->stream), "trace primary");
    });
}

HDCX_API hdcx_status hdcx_get_stats(const hdcx_tracer* t, hdcx_render_stats* stats)
{
    if (!t || !stats) return HDCX_ERROR_INVALID_ARGUMENT;
    *stats = t->stats;
    return HDCX_OK;
}


// ---------------------------------------------------------------------------
// Neural radiance cache
// ---------------------------------------------------------------------------
}  // extern "C"

namespace {

template <typename F>
hdcx_status nrcGuarded(hdcx_nrc* n, F&& body)
{
    try {
        n->lastError.clear();
        check(cudaSetDevice(n->device), "cudaSetDevice");
        body();
        return HDCX_OK;
    } catch (const StatusError& e) {
        n->lastError = e.what();
        return e.status;
    } catch (const std::invalid_argument& e) {
        n->lastError = e.what();
        return HDCX_ERROR_INVALID_ARGUMENT;
    } catch (const std::bad_alloc&) {
        n->lastError = "host allocation failed";
        return HDCX_ERROR_OUT_OF_MEMORY;
    } catch (const std::exception& e) {
        n->lastError = e.what();
        const bool timeout = std::strstr(e.what(), "timed out") != nullptr;
        const bool oom = std::strstr(e.what(), "out of memory") != nullptr;
        return timeout ? HDCX_ERROR_TIMEOUT : (oom ? HDCX_ERROR_OUT_OF_MEMORY : HDCX_ERROR_CUDA);
    }
}

}  // namespace

extern "C" {

HDCX_API void hdcx_nrc_defaults(hdcx_nrc_config* c)
{
    if (!c) return;
    const hdcx::nrc::Config d;
    c->log2_table_size = d.log2TableSize;
    c->base_resolution = d.baseResolution;
    c->finest_resolution = d.finestResolution;
    c->learning_rate = d.learningRate;
    c->beta1 = d.beta1;
    c->beta2 = d.beta2;
    c->epsilon = d.epsilon;
    c->seed = d.seed;
}

HDCX_API hdcx_status hdcx_nrc_create(int32_t device, const hdcx_nrc_config* config, hdcx_nrc** out)
{
    if (!out) return HDCX_ERROR_INVALID_ARGUMENT;
    *out = nullptr;
    int supported = 0, count = 0;
    hdcx_probe_devices(&supported, &count);
    if (!supported || device < 0 || device >= count) return HDCX_ERROR_NO_DEVICE;
    auto* n = new (std::nothrow) hdcx_nrc();
    if (!n) return HDCX_ERROR_OUT_OF_MEMORY;
    n->device = device;
    const hdcx_status s = nrcGuarded(n, [&] {
        hdcx::nrc::Config c;
        if (config) {
            c.log2TableSize = config->log2_table_size;
            c.baseResolution = config->base_resolution;
            c.finestResolution = config->finest_resolution;
            c.learningRate = config->learning_rate;
            c.beta1 = config->beta1;
            c.beta2 = config->beta2;
            c.epsilon = config->epsilon;
            c.seed = config->seed;
        }
        check(cudaStreamCreateWithFlags(&n->stream, cudaStreamNonBlocking), "cudaStreamCreate");
        n->cache = hdcx::nrc::create(device, c);
    });
    if (s != HDCX_OK) {
        delete n;
        return s;
    }
    *out = n;
    return HDCX_OK;
}

HDCX_API void hdcx_nrc_destroy(hdcx_nrc* n)
{
    if (!n) return;
    cudaSetDevice(n->device);
    delete n;
}

HDCX_API const char* hdcx_nrc_last_error(const hdcx_nrc* n) { return n ? n->lastError.c_str() : "null cache"; }

HDCX_API uint64_t hdcx_nrc_grid_parameter_count(const hdcx_nrc* n) { return n ? hdcx::nrc::gridParameterCount(n->cache) : 0; }

HDCX_API hdcx_status hdcx_nrc_resolutions(const hdcx_nrc* n, uint32_t* r)
{
    if (!n || !r) return HDCX_ERROR_INVALID_ARGUMENT;
    for (int l = 0; l < hdcx::nrc::kLevels; ++l) r[l] = hdcx::nrc::resolution(n->cache, l);
    return HDCX_OK;
}

HDCX_API hdcx_status hdcx_nrc_query(hdcx_nrc* n, const float* queries, uint32_t count, float* radiance)
{
    if (!n || (count && (!queries || !radiance))) return HDCX_ERROR_INVALID_ARGUMENT;
    return nrcGuarded(n, [&] { hdcx::nrc::query(n->cache, queries, count, radiance, n->stream); });
}

HDCX_API hdcx_status hdcx_nrc_train(hdcx_nrc* n, const float* queries, const float* targets, uint32_t count, uint32_t steps,
                                    float* meanLoss)
{
    if (!n || (count && (!queries || !targets))) return HDCX_ERROR_INVALID_ARGUMENT;
    return nrcGuarded(n, [&] {
        const float loss = hdcx::nrc::train(n->cache, queries, targets, count, steps, n->stream);
        if (meanLoss) *meanLoss = loss;
    });
}

HDCX_API hdcx_status hdcx_nrc_gradients(hdcx_nrc* n, const float* queries, const float* targets, uint32_t count,
                                        float* mlpGradient, float* gridGradient)
{
    if (!n || (count && (!queries || !targets))) return HDCX_ERROR_INVALID_ARGUMENT;
    return nrcGuarded(n, [&] { hdcx::nrc::gradients(n->cache, queries, targets, count, mlpGradient, gridGradient, n->stream); });
}

HDCX_API hdcx_status hdcx_nrc_check_wait_timeout(hdcx_nrc* n, uint32_t polls)
{
    if (!n || polls == 0) return HDCX_ERROR_INVALID_ARGUMENT;
    return nrcGuarded(n, [&] { hdcx::nrc::checkWaitTimeout(n->cache, polls, n->stream); });
}

HDCX_API hdcx_status hdcx_nrc_get_parameters(hdcx_nrc* n, float* mlp, float* grid)
{
    if (!n) return HDCX_ERROR_INVALID_ARGUMENT;
    return nrcGuarded(n, [&] { hdcx::nrc::getParameters(n->cache, mlp, grid); });
}

HDCX_API hdcx_status hdcx_nrc_set_parameters(hdcx_nrc* n, const float* mlp, const float* grid)
{
    if (!n || !mlp || !grid) return HDCX_ERROR_INVALID_ARGUMENT;
    return nrcGuarded(n, [&] { hdcx::nrc::setParameters(n->cache, mlp, grid); });
}

HDCX_API hdcx_status hdcx_get_tuning(const hdcx_tracer* t, hdcx_tuning* out)
{
    if (!t || !out) return HDCX_ERROR_INVALID_ARGUMENT;
    *out = hdcx_tuning{};
    out->wave_paths = t->wavePaths;
    out->trace_blocks_per_sm = t->traceBlocksPerSm;
    out->shade_blocks_per_sm = t->shadeBlocksPerSm;
    out->sort_hits = t->sortHits;
    out->sort_rays = t->sortRays;
    return HDCX_OK;
}

HDCX_API hdcx_status hdcx_set_tuning(hdcx_tracer* t, const hdcx_tuning* in)
{
    if (!t || !in) return HDCX_ERROR_INVALID_ARGUMENT;
    if ((in->wave_paths != 0 && in->wave_paths < 3) || in->trace_blocks_per_sm < 1 || in->trace_blocks_per_sm > 64 ||
        in->shade_blocks_per_sm < 1 || in->shade_blocks_per_sm > 64 || in->sort_hits > 1 || in->sort_rays > 1)
        return fail(t, HDCX_ERROR_INVALID_ARGUMENT,
                    "tuning out of range (wave >= 3 paths or 0, 1..64 blocks per SM, sort_hits and sort_rays 0 or 1)");
    t->wavePaths = in->wave_paths;
    t->traceBlocksPerSm = in->trace_blocks_per_sm;
    t->shadeBlocksPerSm = in->shade_blocks_per_sm;
    t->sortHits = in->sort_hits;
    t->sortRays = in->sort_rays;
    return HDCX_OK;
}

}  // extern "C"

namespace {

struct TuningKey {
    int device;
    uint32_t triangles, width, height, samples, bounces, full, lit, opaque;
    bool operator==(const TuningKey& o) const
    {
        return device == o.device && triangles == o.triangles && width == o.width && height == o.height &&
               samples == o.samples && bounces == o.bounces && full == o.full && lit == o.lit && opaque == o.opaque;
    }
};

std::mutex gTuningLock;
std::vector<std::pair<TuningKey, hdcx_tuning>> gTunings;

}  // namespace

extern "C" {

HDCX_API hdcx_status hdcx_autotune(hdcx_tracer* t, const hdcx_camera* camera, uint32_t width, uint32_t height,
                                   uint32_t maxBounces, uint32_t sampleCount, hdcx_tuning* result)
{
    if (!t || !camera || width == 0 || height == 0) return HDCX_ERROR_INVALID_ARGUMENT;
    if (!t->geometryReady) return fail(t, HDCX_ERROR_INVALID_ARGUMENT, "no geometry");
    if (t->radianceCache) return fail(t, HDCX_ERROR_INVALID_ARGUMENT, "detach the radiance cache before tuning");
    NvtxRange range("hdcx autotune");
    const TuningKey key{t->device, t->scene.primitiveCount, width, height, std::max(sampleCount, 1u),
                        std::clamp(maxBounces, 1u, HDCX_MAX_PATH_BOUNCES), t->scene.fullShading,
                        (t->scene.lightCount > 0u && !t->scene.hasMeshLights) ? 1u : 0u, t->scene.opaque};
    {
        std::lock_guard<std::mutex> lock(gTuningLock);
        for (const auto& entry : gTunings) {
            if (entry.first == key) {
                hdcx_tuning cached = entry.second;
                cached.candidates = 0;
                t->wavePaths = cached.wave_paths;
                t->traceBlocksPerSm = cached.trace_blocks_per_sm;
                t->shadeBlocksPerSm = cached.shade_blocks_per_sm;
                t->sortHits = cached.sort_hits;
                t->sortRays = cached.sort_rays;
                if (result) *result = cached;
                return HDCX_OK;
            }
        }
    }
    hdcx_tuning best{};
    return guarded(t, [&] {
        const uint32_t savedProfiling = t->profiling;
        t->profiling = 0;
        ArenaLease lease = checkoutArena(t->device, true);  // one arena for every timed render
        // Best of two device-timed renders of one configuration.
        auto measure = [&](uint64_t wave, uint32_t trace, uint32_t shade, uint32_t sort = 0, uint32_t rays = 0) {
            t->wavePaths = wave;
            t->traceBlocksPerSm = trace;
            t->shadeBlocksPerSm = shade;
            t->sortHits = sort;
            t->sortRays = rays;
            double ms = 1e30;
            for (int rep = 0; rep < 2; ++rep) {
                RenderCall call;
                prepareRender(t, *camera, width, height, 0, maxBounces, sampleCount, 0, false, call, lease.arena);
                enqueueRender(t, call, nullptr);
                finishRender(t, call);
                ms = std::min(ms, t->stats.render_ms);
            }
            return ms;
        };
        const uint64_t needed = uint64_t(width) * height * 3u * key.samples;
        best.wave_paths = 0;
        best.trace_blocks_per_sm = 16;
        best.shade_blocks_per_sm = 8;
        best.default_milliseconds = measure(0, 16, 8);
        best.milliseconds = best.default_milliseconds;
        best.candidates = 1;
        auto consider = [&](uint64_t wave, uint32_t trace, uint32_t shade, uint32_t sort, uint32_t rays = 0) {
            const double ms = measure(wave, trace, shade, sort, rays);
            ++best.candidates;
            if (ms < best.milliseconds) {
                best.milliseconds = ms;
                best.wave_paths = wave;
                best.trace_blocks_per_sm = trace;
                best.shade_blocks_per_sm = shade;
                best.sort_hits = sort;
                best.sort_rays = rays;
            }
        };
        // The hit sort first: whether it pays depends on how differently the
        // scene's materials shade, which the other knobs hardly change.
        consider(0, 16, 8, 1u);
        const uint32_t sort = best.sort_hits;
        // Waves above the automatic size shorten the launches' tails; they are
        // tried while their path state stays within half the device memory
        // that is free or already held by the arena.
        size_t freeBytes = 0, totalBytes = 0;
        check(cudaMemGetInfo(&freeBytes, &totalBytes), "cudaMemGetInfo");
        const uint64_t pathBytesLimit = (freeBytes + lease.arena->store.paths.capacity * kPathStateBytes) / 2;
        for (uint64_t wave : {48ull << 20, 32ull << 20, 24ull << 20, 16ull << 20, 8ull << 20, 4ull << 20, 2ull << 20,
                              1ull << 20}) {
            if (wave < needed && wave * kPathStateBytes <= pathBytesLimit)
                consider(wave, best.trace_blocks_per_sm, best.shade_blocks_per_sm, sort);
        }
        for (uint32_t trace : {8u, 32u, 64u}) consider(best.wave_paths, trace, best.shade_blocks_per_sm, sort);
        for (uint32_t shade : {2u, 4u, 16u}) consider(best.wave_paths, best.trace_blocks_per_sm, shade, sort);
        // The sort again, the other way, at the chosen launch shape.
        consider(best.wave_paths, best.trace_blocks_per_sm, best.shade_blocks_per_sm, best.sort_hits ^ 1u);
        // The ray sort, at the chosen launch shape and hit sort.
        consider(best.wave_paths, best.trace_blocks_per_sm, best.shade_blocks_per_sm, best.sort_hits, 1u);
        // Arena buffers grown for a larger candidate than the one chosen are
        // released; the next render allocates the chosen wave.
        const uint64_t chosen = std::max<uint64_t>(3, std::min(needed, best.wave_paths ? best.wave_paths : kAutomaticWavePaths));
        if (lease.arena->store.paths.capacity > chosen) {
            check(cudaStreamSynchronize(t->stream), "cudaStreamSynchronize");
            lease.arena->store.release();
        }
        t->wavePaths = best.wave_paths;
        t->traceBlocksPerSm = best.trace_blocks_per_sm;
        t->shadeBlocksPerSm = best.shade_blocks_per_sm;
        t->sortHits = best.sort_hits;
        t->sortRays = best.sort_rays;
        t->profiling = savedProfiling;
        {
            std::lock_guard<std::mutex> lock(gTuningLock);
            gTunings.emplace_back(key, best);
        }
        if (result) *result = best;
    });
}

HDCX_API hdcx_status hdcx_set_radiance_cache(hdcx_tracer* t, hdcx_nrc* cache, uint32_t prefixBounces,
                                             uint32_t trainingPaths, uint32_t trainSteps)
{
    if (!t) return HDCX_ERROR_INVALID_ARGUMENT;
    if (!cache) {
        t->radianceCache = nullptr;
        return HDCX_OK;
    }
    if (cache->device != t->device) return fail(t, HDCX_ERROR_INVALID_ARGUMENT, "the radiance cache lives on another device");
    if (prefixBounces < 1 || prefixBounces >= HDCX_MAX_PATH_BOUNCES)
        return fail(t, HDCX_ERROR_INVALID_ARGUMENT, "prefix_bounces must be in [1, 11]");
    if (trainingPaths < 128 || trainingPaths > (1u << 20))
        return fail(t, HDCX_ERROR_INVALID_ARGUMENT, "training_paths must be in [128, 2^20]");
    t->radianceCache = cache;
    t->cachePrefix = prefixBounces;
    t->cacheTrainingPaths = trainingPaths;
    t->cacheRun = CacheRun{};
    t->cacheRun.trainSteps = std::max(trainSteps, 1u);
    return HDCX_OK;
}

HDCX_API hdcx_status hdcx_set_radiance_cache_spread(hdcx_tracer* t, float factor)
{
    if (!t) return HDCX_ERROR_INVALID_ARGUMENT;
    if (!(factor >= 0.0F && factor <= 1e6F)) return fail(t, HDCX_ERROR_INVALID_ARGUMENT, "spread factor must be in [0, 1e6]");
    t->cacheSpread = factor;
    return HDCX_OK;
}

HDCX_API hdcx_status hdcx_get_radiance_cache_stats(const hdcx_tracer* t, uint64_t* queries, uint64_t* samples, float* loss)
{
    if (!t) return HDCX_ERROR_INVALID_ARGUMENT;
    if (queries) *queries = t->cacheRun.queries;
    if (samples) *samples = t->cacheRun.samples;
    if (loss) *loss = t->cacheRun.lastLoss;
    return HDCX_OK;
}

}  // extern "C"
