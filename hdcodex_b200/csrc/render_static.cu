// render_static.cu - the wavefront render with its scratch in a static device
// array, for hdcx_render_static (include/hdcx.h).
//
// Some callers cannot allocate device memory while they render: a plugin
// inside a host application that reserves the GPU's memory for itself and
// gives plugins no allocator, or an interactive loop that must not pay the
// device-wide synchronisation cudaFree (and often cudaMalloc) implies. The
// ordinary render allocates its per-wave path state and per-pixel sums on its
// first call and again whenever the image size grows. This variant runs the
// same kernels with that scratch carved out of one file-scope __device__ array
// of fixed size instead, and calls no allocator of any kind.
//
// Limits (compile-time, checked by the entry point): images up to
// kStaticMaxPixels pixels; waves of kStaticWavePaths paths (a frame needs more
// waves than the ordinary render, whose waves hold up to ~12.6M paths, so this
// variant is slower on large frames). Every GPU that loads the library keeps
// the array, kStaticScratchBytes (about 62 MB), until the process exits.
//
// The array's device address is looked up once per device with
// cudaGetSymbolAddress, by the first call on that device (with that device
// current). All calls on a device share the one array and it keeps the last
// call's contents, so calls whose GPU work overlapped would race: each call
// therefore holds a per-device lock until its work on the GPU has finished.
#include "render_static.h"

#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <stdexcept>
#include <string>

namespace hdcx {
namespace {

constexpr uint64_t kAlign = 256;
constexpr uint64_t alignUp(uint64_t v) { return (v + kAlign - 1) / kAlign * kAlign; }

// Bytes of every scratch region, in carve order.
constexpr uint64_t kN = kStaticWavePaths;
constexpr uint64_t kShadow = kN * kStaticShadowPerPath;
constexpr uint64_t kRegionBytes[] = {
    4 * kN,                        // rng
    4 * kN,                        // wavelength
    16 * kN,                       // spectrum
    4 * kN,                        // throughput
    4 * kN,                        // radiance
    16 * kN,                       // rayOrigin
    16 * kN,                       // rayDirection
    4 * kN,                        // flags
    8 * kN,                        // previousPdf
    16 * kN,                       // medium
    16 * kN,                       // hit
    4 * 3 * kN,                    // contribution (3 slots)
    3 * kN,                        // contributionValid
    4 * kN,                        // queue[0]
    4 * kN,                        // queue[1]
    4 * kN,                        // hitQueue
    4 * kN,                        // missQueue
    16 * kShadow,                  // shadowOrigin
    16 * kShadow,                  // shadowDirection
    16 * kShadow,                  // shadowFactors
    4 * kShadow,                   // shadowSlot
    4 * kShadow,                   // shadowInfo
    4 * 8,                         // counters
    8 * 8,                         // stats
    16 * kStaticMaxPixels,         // batch (float4 per pixel)
    24 * kStaticMaxPixels,         // batchXyz (3 doubles per pixel)
};
constexpr int kRegions = static_cast<int>(sizeof(kRegionBytes) / sizeof(kRegionBytes[0]));

constexpr uint64_t totalBytes()
{
    uint64_t total = 0;
    for (int i = 0; i < kRegions; ++i) total += alignUp(kRegionBytes[i]);
    return total;
}

static_assert(totalBytes() == kStaticScratchBytes, "kStaticScratchBytes must match the carve layout");

// The scratch: path state of one wave and the per-pixel sums of one frame.
static __device__ __align__(256) unsigned char gStaticScratch[kStaticScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex gDeviceLocks[kMaxDevices];
std::mutex gSetupLock;
unsigned char* gScratchAddress[kMaxDevices] = {};

// Device address of gStaticScratch on `device`, which must be current.
unsigned char* scratchAddress(int device)
{
    std::lock_guard<std::mutex> lock(gSetupLock);
    if (!gScratchAddress[device]) {
        void* ptr = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&ptr, gStaticScratch);
        if (e != cudaSuccess || ptr == nullptr)
            throw std::runtime_error(std::string("static scratch: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        gScratchAddress[device] = static_cast<unsigned char*>(ptr);
    }
    return gScratchAddress[device];
}

void ok(cudaError_t e, const char* what)
{
    if (e != cudaSuccess) throw std::runtime_error(std::string("static render: ") + what + ": " + cudaGetErrorString(e));
}

}  // namespace

unsigned int renderStatic(const DeviceScene& scene, const FrameConst& frame, float4* rgba, cudaStream_t stream)
{
    const uint64_t pixels = static_cast<uint64_t>(frame.width) * frame.height;
    if (pixels > kStaticMaxPixels) throw std::invalid_argument("image larger than the static scratch maximum");
    int device = 0;
    ok(cudaGetDevice(&device), "cudaGetDevice");
    if (device < 0 || device >= kMaxDevices) throw std::runtime_error("static render: device ordinal out of range");
    std::lock_guard<std::mutex> deviceLock(gDeviceLocks[device]);
    unsigned char* base = scratchAddress(device);

    unsigned char* region[kRegions];
    uint64_t offset = 0;
    for (int i = 0; i < kRegions; ++i) {
        region[i] = base + offset;
        offset += alignUp(kRegionBytes[i]);
    }
    PathBuffers p;
    p.capacity = kN;
    p.wavePaths = kN;
    p.shadowPerPath = kStaticShadowPerPath;
    p.rng = reinterpret_cast<uint32_t*>(region[0]);
    p.wavelength = reinterpret_cast<float*>(region[1]);
    p.spectrum = reinterpret_cast<float4*>(region[2]);
    p.throughput = reinterpret_cast<float*>(region[3]);
    p.radiance = reinterpret_cast<float*>(region[4]);
    p.rayOrigin = reinterpret_cast<float4*>(region[5]);
    p.rayDirection = reinterpret_cast<float4*>(region[6]);
    p.flags = reinterpret_cast<uint32_t*>(region[7]);
    p.previousPdf = reinterpret_cast<float2*>(region[8]);
    p.medium = reinterpret_cast<float4*>(region[9]);
    p.hit = reinterpret_cast<float4*>(region[10]);
    p.contribution = reinterpret_cast<float*>(region[11]);
    p.contributionValid = reinterpret_cast<uint8_t*>(region[12]);
    p.queue[0] = reinterpret_cast<uint32_t*>(region[13]);
    p.queue[1] = reinterpret_cast<uint32_t*>(region[14]);
    p.hitQueue = reinterpret_cast<uint32_t*>(region[15]);
    p.missQueue = reinterpret_cast<uint32_t*>(region[16]);
    p.shadowOrigin = reinterpret_cast<float4*>(region[17]);
    p.shadowDirection = reinterpret_cast<float4*>(region[18]);
    p.shadowFactors = reinterpret_cast<float4*>(region[19]);
    p.shadowSlot = reinterpret_cast<uint32_t*>(region[20]);
    p.shadowInfo = reinterpret_cast<uint32_t*>(region[21]);
    p.counters = reinterpret_cast<uint32_t*>(region[22]);
    p.stats = reinterpret_cast<unsigned long long*>(region[23]);

    FrameBuffers fb;
    fb.width = frame.width;
    fb.height = frame.height;
    fb.rgba = rgba;
    fb.batch = reinterpret_cast<float4*>(region[24]);
    fb.batchXyz = reinterpret_cast<double*>(region[25]);
    // The frame's FP64 XYZ running sums are not kept by this variant: the
    // finalize pass adds them into the batch sums of the same pixel (each
    // thread reads and writes only its own pixel), which the next call clears.
    fb.xyz = fb.batchXyz;

    // The array keeps the previous call's contents: the queue counters and
    // ray statistics must start at zero (renderFrame clears the batch sums).
    ok(cudaMemsetAsync(p.counters, 0, 8 * sizeof(uint32_t), stream), "clear counters");
    ok(cudaMemsetAsync(p.stats, 0, 8 * sizeof(unsigned long long), stream), "clear stats");
    renderFrame(scene, frame, p, fb, stream, nullptr, false, nullptr);
    // The lock covers the GPU work too: the next call may reuse the array.
    ok(cudaStreamSynchronize(stream), "render");
    unsigned long long faults = 0;  // renderFrame's traversal fault word
    ok(cudaMemcpy(&faults, p.stats + 7, sizeof faults, cudaMemcpyDeviceToHost), "read the traversal fault word");
    return static_cast<unsigned int>(faults);
}

}  // namespace hdcx
