// nrc.cu - neural radiance cache kernels (hash-grid encoding, tcgen05 MLP
// forward and backward, Adam) and their host driver.
//
// Network (one query = one path vertex and one wavelength lane):
//   input (64): 16 hash-grid levels x 2 features of the position (Mueller et
//   al., "Instant Neural Graphics Primitives with a Multiresolution Hash
//   Encoding", SIGGRAPH 2022: trilinear interpolation of FP16 features at the
//   8 cell corners, dense indexing while (N+1)^3 fits the level, else the
//   spatial hash x ^ 2654435761 y ^ 805459861 z), then direction (3), shading
//   normal (3), roughness, wavelength, zeros;
//   layers: 64->64 (x4, ReLU), 64->16 (output 0 = radiance), no biases;
//   loss: relative L2, (p - y)^2 / (p^2 + 0.01) with p held constant in the
//   denominator (Mueller et al., "Real-time Neural Radiance Caching for Path
//   Tracing", SIGGRAPH 2021).
//
// Tensor cores: every GEMM is a 128-row tile issued as tcgen05.mma kind::f16
// (BF16 x BF16 -> FP32 in tensor memory) by one thread, completion tracked by
// tcgen05.commit on an mbarrier. Operands sit in shared memory in one
// core-matrix tiling (8x8 BF16 blocks of 128 bytes, no swizzle) which serves
// as K-major or MN-major operand by the descriptor alone:
//   forward      Z_l  = X_l W_l^T      A = X_l (K-major),  B = W_l (K-major)
//   backward     dA_l = dZ_l W_l       A = dZ_l (K-major), B = W_l (MN-major)
//   weight grad  dW_l += dZ_l^T X_l    A = dZ_l (MN-major, padded to 128 rows),
//                                      B = X_l (MN-major), accumulated in
//                                      tensor memory over all tiles of a CTA.
// Activations and output gradients are rounded to BF16 before each GEMM.
// Waits on the mbarrier are bounded: on expiry the kernel records an error,
// waits (bounded) for the MMA in flight, frees its tensor memory and returns.
#include "nrc.h"

#include "device_memory.h"

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

namespace hdcx {
namespace nrc {
namespace {

#define NRC_OK(expr)                                                                                              \
    do {                                                                                                          \
        cudaError_t err__ = (expr);                                                                               \
        if (err__ != cudaSuccess) throw std::runtime_error(std::string("nrc: ") + #expr + ": " + cudaGetErrorString(err__)); \
    } while (0)

constexpr uint32_t kErrorTimeout = 1u;
// The drain wait after a timeout also ran out: an MMA may still have been in
// flight when the kernel freed its tensor memory. Freeing is still the lesser
// hazard: a CTA that exits holding tensor memory leaves the next CTA's
// tcgen05.alloc on that SM waiting for columns that never come back.
constexpr uint32_t kErrorDrain = 2u;
constexpr uint32_t kWaitLimit = 1u << 22;  // mbarrier polls before a wait gives up

struct DeviceParams {
    const __nv_bfloat16* weights;  // tiled BF16 weights of the five layers
    const __half2* grid;           // FP16 features, [level][entry]
    uint32_t resolution[kLevels];
    uint32_t tableMask;
    uint32_t log2Table;
};

// ---------------------------------------------------------------------------
// PTX wrappers
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smemAddress(const void* p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

// Shared-memory matrix descriptor, no swizzle: start address, leading and
// stride byte offsets (all in 16-byte units), descriptor version 1.
__device__ __forceinline__ uint64_t matrixDescriptor(uint32_t address, uint32_t leadingBytes, uint32_t strideBytes)
{
    return static_cast<uint64_t>((address >> 4) & 0x3FFFu) | (static_cast<uint64_t>((leadingBytes >> 4) & 0x3FFFu) << 16) |
           (static_cast<uint64_t>((strideBytes >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B,
// K-major (0) or MN-major (1) operands, N >> 3 and M >> 4.
__host__ __device__ constexpr uint32_t instructionDescriptor(int m, int n, bool aMnMajor, bool bMnMajor)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((aMnMajor ? 1u : 0u) << 15) | ((bMnMajor ? 1u : 0u) << 16) |
           (static_cast<uint32_t>(n >> 3) << 17) | (static_cast<uint32_t>(m >> 4) << 24);
}

__device__ __forceinline__ void mma(uint32_t dTmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate)
{
    const uint32_t zero = 0u;
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}\n" ::"r"(dTmem),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate), "r"(zero));
}

__device__ __forceinline__ void commitTo(uint64_t* bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smemAddress(bar))
                 : "memory");
}

__device__ __forceinline__ void barrierInit(uint64_t* bar)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smemAddress(bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Bounded wait for the phase `parity` of `bar`; false if the limit ran out.
__device__ __forceinline__ bool barrierWait(uint64_t* bar, uint32_t parity, uint32_t limit = kWaitLimit)
{
    const uint32_t address = smemAddress(bar);
    for (uint32_t i = 0; i < limit; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(address), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void fenceBeforeSync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fenceAfterSync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fenceProxyAsync() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 16 consecutive FP32 columns of this thread's tensor-memory lane.
__device__ __forceinline__ void tmemLoad16(uint32_t address, float* v)
{
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(address));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ uint32_t tmemAllocate(uint32_t* slot, uint32_t columns)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smemAddress(slot)), "r"(columns)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    return 0;
}

__device__ __forceinline__ void tmemFree(uint32_t address, uint32_t columns)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(address), "r"(columns) : "memory");
}

// ---------------------------------------------------------------------------
// Encoding
// ---------------------------------------------------------------------------
__device__ __forceinline__ void levelCorners(const DeviceParams& p, int level, float3 pos, uint32_t index[8], float weight[8])
{
    const uint32_t n = p.resolution[level];
    const float fn = static_cast<float>(n);
    float sx = fminf(fmaxf(pos.x, 0.0f), 1.0f) * fn, sy = fminf(fmaxf(pos.y, 0.0f), 1.0f) * fn,
          sz = fminf(fmaxf(pos.z, 0.0f), 1.0f) * fn;
    const uint32_t cx = min(static_cast<uint32_t>(sx), n - 1u), cy = min(static_cast<uint32_t>(sy), n - 1u),
                   cz = min(static_cast<uint32_t>(sz), n - 1u);
    const float fx = sx - static_cast<float>(cx), fy = sy - static_cast<float>(cy), fz = sz - static_cast<float>(cz);
    const uint64_t side = static_cast<uint64_t>(n) + 1u;
    const bool dense = side * side * side <= static_cast<uint64_t>(p.tableMask) + 1u;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        const uint32_t x = cx + (c & 1), y = cy + ((c >> 1) & 1), z = cz + ((c >> 2) & 1);
        const uint32_t h = dense ? static_cast<uint32_t>(x + side * (y + side * z))
                                 : (x ^ (y * 2654435761u) ^ (z * 805459861u));
        index[c] = (static_cast<uint32_t>(level) << p.log2Table) + (h & p.tableMask);
        weight[c] = ((c & 1) ? fx : 1.0f - fx) * (((c >> 1) & 1) ? fy : 1.0f - fy) * (((c >> 2) & 1) ? fz : 1.0f - fz);
    }
}

// The 64 network inputs of query record q (zeros for a missing query).
__device__ void encodeQuery(const DeviceParams& p, const float* q, float in[kWidth])
{
#pragma unroll
    for (int i = 0; i < kWidth; ++i) in[i] = 0.0f;
    if (!q) return;
    const float3 pos = make_float3(q[0], q[1], q[2]);
    for (int level = 0; level < kLevels; ++level) {
        uint32_t index[8];
        float weight[8];
        levelCorners(p, level, pos, index, weight);
        float f0 = 0.0f, f1 = 0.0f;
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            const float2 v = __half22float2(p.grid[index[c]]);
            f0 = fmaf(weight[c], v.x, f0);
            f1 = fmaf(weight[c], v.y, f1);
        }
        in[2 * level] = f0;
        in[2 * level + 1] = f1;
    }
#pragma unroll
    for (int i = 0; i < 9; ++i) in[32 + i] = q[3 + i];
}

// Writes 64 values of row `row` as BF16 into a tile with `colGroups` column groups.
__device__ __forceinline__ void storeRow(__nv_bfloat16* tile, uint32_t row, const float* v, uint32_t colGroups, int count)
{
    for (int c = 0; c < count; c += 8) {
        __align__(16) __nv_bfloat16 b[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) b[i] = __float2bfloat16_rn(v[c + i]);
        *reinterpret_cast<uint4*>(tile + tiled(row, static_cast<uint32_t>(c), colGroups)) = *reinterpret_cast<const uint4*>(b);
    }
}

__device__ __forceinline__ void loadWeights(__nv_bfloat16* dst, const __nv_bfloat16* src)
{
    const uint4* s = reinterpret_cast<const uint4*>(src);
    uint4* d = reinterpret_cast<uint4*>(dst);
    for (uint32_t i = threadIdx.x; i < kWeightCount / 8u; i += blockDim.x) d[i] = s[i];
}

// Issues Z = X W_l^T for a 128-row tile: X has 8 column groups, K = 64.
__device__ __forceinline__ void issueForward(uint32_t dTmem, const __nv_bfloat16* x, const __nv_bfloat16* w, int layer)
{
    const uint32_t idesc = instructionDescriptor(kTile, layerRows(layer), false, false);
    const uint32_t xa = smemAddress(x), wa = smemAddress(w + layerOffset(layer));
#pragma unroll
    for (uint32_t k = 0; k < 4; ++k) {
        mma(dTmem, matrixDescriptor(xa + k * 256u, 128u, 1024u), matrixDescriptor(wa + k * 256u, 128u, 1024u), idesc, k > 0u);
    }
}

// ---------------------------------------------------------------------------
// Kernels
// ---------------------------------------------------------------------------
constexpr uint32_t kQuerySmem = kWeightCount * 2u + kTile * kWidth * 2u + 16u;

__global__ void __launch_bounds__(128) queryKernel(DeviceParams p, const float* queries, uint32_t count, float* out,
                                                   uint32_t* error)
{
    extern __shared__ __align__(16) uint8_t smem[];
    __nv_bfloat16* w = reinterpret_cast<__nv_bfloat16*>(smem);
    __nv_bfloat16* x = w + kWeightCount;
    uint64_t* bar = reinterpret_cast<uint64_t*>(x + kTile * kWidth);
    uint32_t* slot = reinterpret_cast<uint32_t*>(bar + 1);
    const uint32_t warp = threadIdx.x >> 5;
    loadWeights(w, p.weights);
    if (threadIdx.x == 0) barrierInit(bar);
    if (warp == 0) tmemAllocate(slot, 64u);
    fenceProxyAsync();
    fenceBeforeSync();
    __syncthreads();
    fenceAfterSync();
    const uint32_t tmem = *slot;
    const uint32_t laneBase = tmem + ((warp * 32u) << 16);
    uint32_t phase = 0;
    bool failed = false;
    for (uint32_t base = blockIdx.x * kTile; base < count && !failed; base += gridDim.x * kTile) {
        const uint32_t row = threadIdx.x;
        const uint32_t q = base + row;
        float v[kWidth];
        encodeQuery(p, q < count ? queries + static_cast<size_t>(q) * kQueryFloats : nullptr, v);
        storeRow(x, row, v, 8u, kWidth);
        for (int layer = 0; layer < kLayers; ++layer) {
            fenceProxyAsync();
            fenceBeforeSync();
            __syncthreads();
            fenceAfterSync();
            if (threadIdx.x == 0) {
                issueForward(tmem, x, w, layer);
                commitTo(bar);
            }
            // Every thread takes the same decision, so that no barrier or
            // warp-collective tensor-memory load is reached by only some.
            if (__syncthreads_or(barrierWait(bar, phase) ? 0 : 1)) {
                failed = true;
                break;
            }
            phase ^= 1u;
            fenceAfterSync();
            if (layer < kLayers - 1) {
                for (int c = 0; c < kWidth; c += 16) tmemLoad16(laneBase + static_cast<uint32_t>(c), v + c);
#pragma unroll
                for (int i = 0; i < kWidth; ++i) v[i] = fmaxf(v[i], 0.0f);
                storeRow(x, row, v, 8u, kWidth);
            } else {
                tmemLoad16(laneBase, v);
                if (q < count) out[q] = v[0];
            }
            fenceBeforeSync();
        }
    }
    if (failed) {
        // Bounded: lets an MMA still in flight finish before the memory is freed.
        const bool drained = barrierWait(bar, phase);
        if (threadIdx.x == 0) atomicOr(error, drained ? kErrorTimeout : (kErrorTimeout | kErrorDrain));
    }
    __syncthreads();
    fenceAfterSync();
    if (warp == 0) tmemFree(tmem, 64u);
}

// Forward and backward of every tile of 128 training records; weight
// gradients accumulate in tensor memory and are added to `mlpGrad` at the
// end; hash-grid gradients are scattered with atomics into `gridGrad`.
constexpr uint32_t kTrainSmem = kWeightCount * 2u + 5u * kTile * kWidth * 2u + kTile * 128u * 2u + 16u;

__global__ void __launch_bounds__(128) trainKernel(DeviceParams p, const float* queries, const float* targets, uint32_t count,
                                                   float gradientScale, float* mlpGrad, float* gridGrad, float* lossSum,
                                                   uint32_t* error)
{
    extern __shared__ __align__(16) uint8_t smem[];
    __nv_bfloat16* w = reinterpret_cast<__nv_bfloat16*>(smem);
    __nv_bfloat16* xs = w + kWeightCount;             // X_0 .. X_4, 128 x 64 each
    __nv_bfloat16* g = xs + 5 * kTile * kWidth;       // dZ, 128 x 128 (columns past the layer width stay zero)
    uint64_t* bar = reinterpret_cast<uint64_t*>(g + kTile * 128);
    uint32_t* slot = reinterpret_cast<uint32_t*>(bar + 1);
    const uint32_t warp = threadIdx.x >> 5;
    loadWeights(w, p.weights);
    for (uint32_t i = threadIdx.x; i < kTile * 128u / 8u; i += blockDim.x) reinterpret_cast<uint4*>(g)[i] = make_uint4(0, 0, 0, 0);
    if (threadIdx.x == 0) barrierInit(bar);
    if (warp == 0) tmemAllocate(slot, 512u);
    fenceProxyAsync();
    fenceBeforeSync();
    __syncthreads();
    fenceAfterSync();
    const uint32_t tmem = *slot;
    const uint32_t laneOffset = (warp * 32u) << 16;
    // Tensor memory columns: [0, 64) Z / dA of the current GEMM, [64 + 64 l, 128 + 64 l) dW_l.
    uint32_t phase = 0;
    bool failed = false;
    bool accumulated = false;
    float lossPart = 0.0f;
    const uint32_t row = threadIdx.x;
    for (uint32_t base = blockIdx.x * kTile; base < count && !failed; base += gridDim.x * kTile) {
        const uint32_t q = base + row;
        const bool valid = q < count;
        const float* record = valid ? queries + static_cast<size_t>(q) * kQueryFloats : nullptr;
        float v[kWidth];
        encodeQuery(p, record, v);
        storeRow(xs, row, v, 8u, kWidth);
        float prediction = 0.0f;
        // Forward, keeping X_0 .. X_4.
        for (int layer = 0; layer < kLayers && !failed; ++layer) {
            fenceProxyAsync();
            fenceBeforeSync();
            __syncthreads();
            fenceAfterSync();
            if (threadIdx.x == 0) {
                issueForward(tmem, xs + layer * kTile * kWidth, w, layer);
                commitTo(bar);
            }
            // Every thread takes the same decision, so that no barrier or
            // warp-collective tensor-memory load is reached by only some.
            if (__syncthreads_or(barrierWait(bar, phase) ? 0 : 1)) {
                failed = true;
                break;
            }
            phase ^= 1u;
            fenceAfterSync();
            if (layer < kLayers - 1) {
                for (int c = 0; c < kWidth; c += 16) tmemLoad16(tmem + laneOffset + static_cast<uint32_t>(c), v + c);
#pragma unroll
                for (int i = 0; i < kWidth; ++i) v[i] = fmaxf(v[i], 0.0f);
                storeRow(xs + (layer + 1) * kTile * kWidth, row, v, 8u, kWidth);
            } else {
                tmemLoad16(tmem + laneOffset, v);
                prediction = v[0];
            }
            fenceBeforeSync();
        }
        if (failed) break;
        // Output gradient of the relative L2 loss.
        float outGrad[16];
#pragma unroll
        for (int i = 0; i < 16; ++i) outGrad[i] = 0.0f;
        if (valid) {
            const float target = targets[q];
            const float denominator = prediction * prediction + 0.01f;
            const float diff = prediction - target;
            lossPart += diff * diff / denominator;
            outGrad[0] = 2.0f * diff / denominator * gradientScale;
        }
        storeRow(g, row, outGrad, 16u, 16);
        // Backward, layer 4 down to 0.
        for (int layer = kLayers - 1; layer >= 0; --layer) {
            fenceProxyAsync();
            fenceBeforeSync();
            __syncthreads();
            fenceAfterSync();
            if (threadIdx.x == 0) {
                const uint32_t ga = smemAddress(g);
                const uint32_t wa = smemAddress(w + layerOffset(layer));
                const uint32_t xa = smemAddress(xs + layer * kTile * kWidth);
                // dA = dZ W_l: A = dZ K-major (K = rows of W_l), B = W_l MN-major.
                const uint32_t kSteps = static_cast<uint32_t>(layerRows(layer)) / 16u;
                const uint32_t idescA = instructionDescriptor(kTile, kWidth, false, true);
                for (uint32_t k = 0; k < kSteps; ++k) {
                    mma(tmem, matrixDescriptor(ga + k * 256u, 128u, 2048u), matrixDescriptor(wa + k * 2048u, 1024u, 128u),
                        idescA, k > 0u);
                }
                // dW_l += dZ^T X_l: A = dZ MN-major (128 rows, zero past the layer width), B = X_l MN-major, K = 128.
                const uint32_t idescW = instructionDescriptor(kTile, kWidth, true, true);
                const uint32_t dw = tmem + 64u + 64u * static_cast<uint32_t>(layer);
                for (uint32_t k = 0; k < 8; ++k) {
                    mma(dw, matrixDescriptor(ga + k * 4096u, 2048u, 128u), matrixDescriptor(xa + k * 2048u, 1024u, 128u), idescW,
                        (accumulated || k > 0u) ? 1u : 0u);
                }
                commitTo(bar);
            }
            // Every thread takes the same decision, so that no barrier or
            // warp-collective tensor-memory load is reached by only some.
            if (__syncthreads_or(barrierWait(bar, phase) ? 0 : 1)) {
                failed = true;
                break;
            }
            phase ^= 1u;
            fenceAfterSync();
            for (int c = 0; c < kWidth; c += 16) tmemLoad16(tmem + laneOffset + static_cast<uint32_t>(c), v + c);
            if (layer > 0) {
                // dZ_{l-1} = dA_l where X_l > 0.
                const __nv_bfloat16* xl = xs + layer * kTile * kWidth;
#pragma unroll
                for (int i = 0; i < kWidth; ++i) {
                    if (!(__bfloat162float(xl[tiled(row, static_cast<uint32_t>(i), 8u)]) > 0.0f)) v[i] = 0.0f;
                }
                storeRow(g, row, v, 16u, kWidth);
            } else if (valid) {
                // Hash-grid gradients: input columns 0..31.
                const float3 pos = make_float3(record[0], record[1], record[2]);
                for (int level = 0; level < kLevels; ++level) {
                    uint32_t index[8];
                    float weight[8];
                    levelCorners(p, level, pos, index, weight);
                    const float d0 = v[2 * level], d1 = v[2 * level + 1];
                    if (d0 == 0.0f && d1 == 0.0f) continue;
#pragma unroll
                    for (int c = 0; c < 8; ++c) {
                        atomicAdd(gridGrad + 2u * index[c], weight[c] * d0);
                        atomicAdd(gridGrad + 2u * index[c] + 1u, weight[c] * d1);
                    }
                }
            }
            fenceBeforeSync();
        }
        accumulated = true;
    }
    if (failed) {
        // Bounded: lets an MMA still in flight finish before the memory is freed.
        const bool drained = barrierWait(bar, phase);
        if (threadIdx.x == 0) atomicOr(error, drained ? kErrorTimeout : (kErrorTimeout | kErrorDrain));
    }
    fenceBeforeSync();
    __syncthreads();
    fenceAfterSync();
    // Weight gradients: tensor-memory lanes 0..63 hold rows 0..63 of dW_l.
    // Whole warps load (the load is warp-collective); only real rows are added.
    if (!failed && accumulated && warp < 2) {
        const uint32_t r = warp * 32u + (threadIdx.x & 31u);
        for (int layer = 0; layer < kLayers; ++layer) {
            float d[kWidth];
            for (int c = 0; c < kWidth; c += 16) tmemLoad16(tmem + laneOffset + 64u + 64u * layer + static_cast<uint32_t>(c), d + c);
            if (r < static_cast<uint32_t>(layerRows(layer))) {
                float* dst = mlpGrad + layerOffset(layer) + r * kWidth;
                for (int c = 0; c < kWidth; ++c) atomicAdd(dst + c, d[c]);
            }
        }
    }
    if (lossPart != 0.0f) atomicAdd(lossSum, lossPart);
    fenceBeforeSync();
    __syncthreads();
    fenceAfterSync();
    if (warp == 0) tmemFree(tmem, 512u);
}

// The kernels' bounded wait on an mbarrier that nothing arrives at: the wait
// runs out, the kernel records the timeout and returns (the host reads the
// error flag; the context stays usable). Used by hdcx_nrc_check_wait_timeout.
__global__ void waitTimeoutKernel(uint32_t limit, uint32_t* error)
{
    __shared__ uint64_t bar;
    if (threadIdx.x == 0) barrierInit(&bar);
    __syncthreads();
    if (__syncthreads_or(barrierWait(&bar, 0u, limit) ? 0 : 1) && threadIdx.x == 0) atomicOr(error, kErrorTimeout);
}

// Adam on `n` FP32 parameters; refreshes the BF16 tiled weights (mlp) or the
// FP16 table (grid) and clears the gradients.
__global__ void adamKernel(float* params, float* grad, float* m, float* v, uint32_t n, float lr, float beta1, float beta2,
                           float epsilon, float correction1, float correction2, __nv_bfloat16* tiledWeights, __half* table)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float gi = grad[i];
        const float mi = beta1 * m[i] + (1.0f - beta1) * gi;
        const float vi = beta2 * v[i] + (1.0f - beta2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float pi = params[i] - lr * (mi / correction1) / (sqrtf(vi / correction2) + epsilon);
        params[i] = pi;
        grad[i] = 0.0f;
        if (tiledWeights) {
            const uint32_t layer = i < 16384u ? i / 4096u : 4u;
            const uint32_t local = i - layerOffset(static_cast<int>(layer));
            tiledWeights[layerOffset(static_cast<int>(layer)) + tiled(local / 64u, local % 64u, 8u)] = __float2bfloat16_rn(pi);
        }
        if (table) table[i] = __float2half_rn(pi);
    }
}

__global__ void refreshKernel(const float* params, uint32_t n, __nv_bfloat16* tiledWeights, __half* table)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (tiledWeights) {
            const uint32_t layer = i < 16384u ? i / 4096u : 4u;
            const uint32_t local = i - layerOffset(static_cast<int>(layer));
            tiledWeights[layerOffset(static_cast<int>(layer)) + tiled(local / 64u, local % 64u, 8u)] = __float2bfloat16_rn(params[i]);
        }
        if (table) table[i] = __float2half_rn(params[i]);
    }
}

template <typename T>
T* deviceAlloc(size_t count)
{
    return static_cast<T*>(deviceMalloc(std::max<size_t>(count, 1) * sizeof(T)));
}

}  // namespace

struct Cache {
    int device = 0;
    Config config;
    uint32_t resolution[kLevels] = {};
    uint64_t gridCount = 0;  // FP32 parameters of the table (levels x entries x 2)
    float* mlp = nullptr;
    float* mlpGrad = nullptr;
    float* mlpM = nullptr;
    float* mlpV = nullptr;
    __nv_bfloat16* mlpTiled = nullptr;
    float* grid = nullptr;
    float* gridGrad = nullptr;
    float* gridM = nullptr;
    float* gridV = nullptr;
    __half* gridHalf = nullptr;
    float* loss = nullptr;
    uint32_t* error = nullptr;
    uint64_t step = 0;
    int sms = 148;

    DeviceParams params() const
    {
        DeviceParams p{};
        p.weights = mlpTiled;
        p.grid = reinterpret_cast<const __half2*>(gridHalf);
        for (int i = 0; i < kLevels; ++i) p.resolution[i] = resolution[i];
        p.log2Table = config.log2TableSize;
        p.tableMask = (1u << config.log2TableSize) - 1u;
        return p;
    }
};

namespace {

void checkError(Cache* c, cudaStream_t stream)
{
    uint32_t e = 0;
    NRC_OK(cudaMemcpyAsync(&e, c->error, sizeof e, cudaMemcpyDeviceToHost, stream));
    NRC_OK(cudaStreamSynchronize(stream));
    if (e != 0u) {
        NRC_OK(cudaMemsetAsync(c->error, 0, sizeof(uint32_t), stream));
        throw std::runtime_error((e & kErrorDrain) != 0u
                                     ? "nrc: a tensor-core wait timed out, and so did the wait for the MMA in flight "
                                       "before tensor memory was freed"
                                     : "nrc: a tensor-core wait timed out");
    }
}

void runTrainKernel(Cache* c, const float* queries, const float* targets, uint32_t count, cudaStream_t stream)
{
    const int blocks = static_cast<int>(std::min<uint32_t>((count + kTile - 1) / kTile, static_cast<uint32_t>(c->sms)));
    trainKernel<<<blocks, 128, kTrainSmem, stream>>>(c->params(), queries, targets, count, 1.0f / static_cast<float>(count),
                                                     c->mlpGrad, c->gridGrad, c->loss, c->error);
    NRC_OK(cudaGetLastError());
}

}  // namespace

Cache* create(int device, const Config& config)
{
    if (config.log2TableSize < 10 || config.log2TableSize > 24) throw std::invalid_argument("nrc: log2 table size out of [10, 24]");
    if (config.baseResolution < 2 || config.finestResolution < config.baseResolution)
        throw std::invalid_argument("nrc: resolutions out of range");
    NRC_OK(cudaSetDevice(device));
    int major = 0;
    NRC_OK(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device));
    if (major != 10) throw std::runtime_error("nrc: needs an sm_100 device");
    auto* c = new Cache();
    c->device = device;
    c->config = config;
    NRC_OK(cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, device));
    const double growth = std::exp((std::log(double(config.finestResolution)) - std::log(double(config.baseResolution))) /
                                   double(kLevels - 1));
    for (int l = 0; l < kLevels; ++l)
        c->resolution[l] = static_cast<uint32_t>(std::floor(double(config.baseResolution) * std::pow(growth, double(l))));
    c->gridCount = static_cast<uint64_t>(kLevels) * (1ull << config.log2TableSize) * kFeatures;
    c->mlp = deviceAlloc<float>(kWeightCount);
    c->mlpGrad = deviceAlloc<float>(kWeightCount);
    c->mlpM = deviceAlloc<float>(kWeightCount);
    c->mlpV = deviceAlloc<float>(kWeightCount);
    c->mlpTiled = deviceAlloc<__nv_bfloat16>(kWeightCount);
    c->grid = deviceAlloc<float>(c->gridCount);
    c->gridGrad = deviceAlloc<float>(c->gridCount);
    c->gridM = deviceAlloc<float>(c->gridCount);
    c->gridV = deviceAlloc<float>(c->gridCount);
    c->gridHalf = deviceAlloc<__half>(c->gridCount);
    c->loss = deviceAlloc<float>(1);
    c->error = deviceAlloc<uint32_t>(1);
    NRC_OK(cudaFuncSetAttribute(queryKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kQuerySmem));
    NRC_OK(cudaFuncSetAttribute(trainKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kTrainSmem));
    // Initialisation: weights uniform in +-sqrt(6 / (fan_in + fan_out)), table uniform in +-1e-4.
    std::mt19937 rng(config.seed);
    std::vector<float> mlp(kWeightCount, 0.0f);
    for (int layer = 0; layer < kLayers; ++layer) {
        const int rows = layer == kLayers - 1 ? 1 : layerRows(layer);  // padded output rows stay zero
        const float bound = std::sqrt(6.0f / float(kWidth + layerRows(layer)));
        std::uniform_real_distribution<float> u(-bound, bound);
        for (int r = 0; r < rows; ++r)
            for (int k = 0; k < kWidth; ++k) mlp[layerOffset(layer) + r * kWidth + k] = u(rng);
    }
    std::vector<float> grid(c->gridCount);
    std::uniform_real_distribution<float> ug(-1e-4f, 1e-4f);
    for (float& x : grid) x = ug(rng);
    setParameters(c, mlp.data(), grid.data());
    return c;
}

void destroy(Cache* c)
{
    if (!c) return;
    cudaSetDevice(c->device);
    for (void* p : {static_cast<void*>(c->mlp), static_cast<void*>(c->mlpGrad), static_cast<void*>(c->mlpM),
                    static_cast<void*>(c->mlpV), static_cast<void*>(c->mlpTiled), static_cast<void*>(c->grid),
                    static_cast<void*>(c->gridGrad), static_cast<void*>(c->gridM), static_cast<void*>(c->gridV),
                    static_cast<void*>(c->gridHalf), static_cast<void*>(c->loss), static_cast<void*>(c->error)})
        deviceFree(p);
    delete c;
}

void setParameters(Cache* c, const float* mlp, const float* grid)
{
    NRC_OK(cudaSetDevice(c->device));
    NRC_OK(cudaMemcpy(c->mlp, mlp, kWeightCount * sizeof(float), cudaMemcpyHostToDevice));
    NRC_OK(cudaMemcpy(c->grid, grid, c->gridCount * sizeof(float), cudaMemcpyHostToDevice));
    NRC_OK(cudaMemset(c->mlpGrad, 0, kWeightCount * sizeof(float)));
    NRC_OK(cudaMemset(c->mlpM, 0, kWeightCount * sizeof(float)));
    NRC_OK(cudaMemset(c->mlpV, 0, kWeightCount * sizeof(float)));
    NRC_OK(cudaMemset(c->gridGrad, 0, c->gridCount * sizeof(float)));
    NRC_OK(cudaMemset(c->gridM, 0, c->gridCount * sizeof(float)));
    NRC_OK(cudaMemset(c->gridV, 0, c->gridCount * sizeof(float)));
    NRC_OK(cudaMemset(c->error, 0, sizeof(uint32_t)));
    refreshKernel<<<64, 256>>>(c->mlp, kWeightCount, c->mlpTiled, nullptr);
    refreshKernel<<<c->sms * 4, 256>>>(c->grid, static_cast<uint32_t>(c->gridCount), nullptr, c->gridHalf);
    NRC_OK(cudaGetLastError());
    NRC_OK(cudaDeviceSynchronize());
    c->step = 0;
}

void getParameters(Cache* c, float* mlp, float* grid)
{
    NRC_OK(cudaSetDevice(c->device));
    NRC_OK(cudaDeviceSynchronize());
    if (mlp) NRC_OK(cudaMemcpy(mlp, c->mlp, kWeightCount * sizeof(float), cudaMemcpyDeviceToHost));
    if (grid) NRC_OK(cudaMemcpy(grid, c->grid, c->gridCount * sizeof(float), cudaMemcpyDeviceToHost));
}

void checkWaitTimeout(Cache* c, uint32_t polls, cudaStream_t stream)
{
    waitTimeoutKernel<<<1, 128, 0, stream>>>(polls, c->error);
    NRC_OK(cudaGetLastError());
    checkError(c, stream);
}

uint64_t gridParameterCount(const Cache* c) { return c->gridCount; }
uint32_t resolution(const Cache* c, int level) { return c->resolution[level]; }

void query(Cache* c, const float* queries, uint32_t count, float* out, cudaStream_t stream)
{
    if (count == 0) return;
    const int blocks = static_cast<int>(std::min<uint32_t>((count + kTile - 1) / kTile, static_cast<uint32_t>(c->sms) * 4u));
    queryKernel<<<blocks, 128, kQuerySmem, stream>>>(c->params(), queries, count, out, c->error);
    NRC_OK(cudaGetLastError());
    checkError(c, stream);
}

float train(Cache* c, const float* queries, const float* targets, uint32_t count, uint32_t steps, cudaStream_t stream)
{
    if (count == 0 || steps == 0) return 0.0f;
    float lossValue = 0.0f;
    for (uint32_t s = 0; s < steps; ++s) {
        NRC_OK(cudaMemsetAsync(c->loss, 0, sizeof(float), stream));
        runTrainKernel(c, queries, targets, count, stream);
        ++c->step;
        const float b1 = 1.0f - std::pow(c->config.beta1, float(c->step));
        const float b2 = 1.0f - std::pow(c->config.beta2, float(c->step));
        adamKernel<<<64, 256, 0, stream>>>(c->mlp, c->mlpGrad, c->mlpM, c->mlpV, kWeightCount, c->config.learningRate,
                                           c->config.beta1, c->config.beta2, c->config.epsilon, b1, b2, c->mlpTiled, nullptr);
        adamKernel<<<c->sms * 8, 256, 0, stream>>>(c->grid, c->gridGrad, c->gridM, c->gridV, static_cast<uint32_t>(c->gridCount),
                                                   c->config.learningRate, c->config.beta1, c->config.beta2,
                                                   c->config.epsilon, b1, b2, nullptr, c->gridHalf);
        NRC_OK(cudaGetLastError());
    }
    NRC_OK(cudaMemcpyAsync(&lossValue, c->loss, sizeof(float), cudaMemcpyDeviceToHost, stream));
    checkError(c, stream);
    return lossValue / static_cast<float>(count);
}

void gradients(Cache* c, const float* queries, const float* targets, uint32_t count, float* mlpGrad, float* gridGrad,
               cudaStream_t stream)
{
    NRC_OK(cudaMemsetAsync(c->mlpGrad, 0, kWeightCount * sizeof(float), stream));
    NRC_OK(cudaMemsetAsync(c->gridGrad, 0, c->gridCount * sizeof(float), stream));
    NRC_OK(cudaMemsetAsync(c->loss, 0, sizeof(float), stream));
    if (count > 0) runTrainKernel(c, queries, targets, count, stream);
    checkError(c, stream);
    if (mlpGrad) NRC_OK(cudaMemcpy(mlpGrad, c->mlpGrad, kWeightCount * sizeof(float), cudaMemcpyDeviceToHost));
    if (gridGrad) NRC_OK(cudaMemcpy(gridGrad, c->gridGrad, c->gridCount * sizeof(float), cudaMemcpyDeviceToHost));
    NRC_OK(cudaMemsetAsync(c->mlpGrad, 0, kWeightCount * sizeof(float), stream));
    NRC_OK(cudaMemsetAsync(c->gridGrad, 0, c->gridCount * sizeof(float), stream));
    NRC_OK(cudaStreamSynchronize(stream));
}

}  // namespace nrc
}  // namespace hdcx
