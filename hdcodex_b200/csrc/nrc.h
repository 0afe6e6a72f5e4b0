// nrc.h - the neural radiance cache: multiresolution hash-grid encoding and a
// 64-wide, 4-hidden-layer ReLU MLP whose forward and backward passes run on
// the sm_100a tensor cores (tcgen05.mma, BF16 operands, FP32 accumulation in
// tensor memory), trained online with FP32 Adam.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "hdcx.h"

namespace hdcx {
namespace nrc {

constexpr int kTile = 128;        // queries per MMA tile (M)
constexpr int kWidth = 64;        // input and hidden width
constexpr int kOut = 16;          // output width of the last layer (output 0 is the radiance)
constexpr int kLayers = 5;        // 64->64, three 64->64, 64->16
constexpr int kLevels = 16;       // hash-grid levels
constexpr int kFeatures = 2;      // features per level
constexpr int kQueryFloats = 12;  // query record: position (3, in [0, 1]), direction (3), normal (3), roughness, wavelength, 0
constexpr uint32_t kWeightCount = 4u * 64u * 64u + 16u * 64u;

__host__ __device__ constexpr uint32_t layerOffset(int layer) { return layer < 4 ? static_cast<uint32_t>(layer) * 4096u : 16384u; }
__host__ __device__ constexpr int layerRows(int layer) { return layer < 4 ? 64 : 16; }

// Element (r, c) of a matrix with `colGroups` groups of eight columns in the
// core-matrix tiling the tensor-core descriptors read: 8x8 blocks of 128
// bytes, row groups outermost, each block row-major.
__host__ __device__ inline uint32_t tiled(uint32_t r, uint32_t c, uint32_t colGroups)
{
    return ((r >> 3) * colGroups + (c >> 3)) * 64u + (r & 7u) * 8u + (c & 7u);
}

struct Config {
    uint32_t log2TableSize = 19;
    uint32_t baseResolution = 16;
    uint32_t finestResolution = 2048;
    float learningRate = 1e-2f;
    float beta1 = 0.9f;
    float beta2 = 0.99f;
    float epsilon = 1e-8f;
    uint32_t seed = 1337;
};

struct Cache;  // device state (nrc.cu)

Cache* create(int device, const Config& config);
void destroy(Cache* cache);
// Radiance predictions (one float per query) for `count` device query records.
void query(Cache* cache, const float* queries, uint32_t count, float* out, cudaStream_t stream);
// `steps` Adam steps on the relative L2 loss against `targets`; returns the
// mean loss of the last step.
float train(Cache* cache, const float* queries, const float* targets, uint32_t count, uint32_t steps, cudaStream_t stream);
// Gradients of the mean loss without an update (host outputs, FP32).
void gradients(Cache* cache, const float* queries, const float* targets, uint32_t count, float* mlpGrad, float* gridGrad,
               cudaStream_t stream);
// Runs the kernels' bounded mbarrier wait on a barrier nothing arrives at, for
// at most `polls` polls; throws the timeout error the host then reads.
void checkWaitTimeout(Cache* cache, uint32_t polls, cudaStream_t stream);
uint64_t gridParameterCount(const Cache* cache);
void getParameters(Cache* cache, float* mlp, float* grid);
void setParameters(Cache* cache, const float* mlp, const float* grid);
uint32_t resolution(const Cache* cache, int level);

}  // namespace nrc
}  // namespace hdcx
