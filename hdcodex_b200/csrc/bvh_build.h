// bvh_build.h - on-GPU construction of the 8-wide compressed BVH.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "device/common.cuh"

namespace hdcx {

struct WideBvh {
    WideNode* nodes = nullptr;
    float4* triVerts = nullptr;  // 3 float4 per leaf-ordered triangle
    uint32_t nodeCount = 0;
    uint32_t depth = 0;
    uint32_t triangleCount = 0;
};

// Builds the BVH of `triangleCount` triangles given as device vertex (xyzw)
// and index arrays. sceneScale = max(|coordinate|, scene extent) bounds the
// quantisation step from below. Synchronous on `stream`; throws
// std::runtime_error on a CUDA failure.
WideBvh buildWideBvh(const float4* vertices, const uint32_t* indices, uint32_t triangleCount, float sceneScale,
                     cudaStream_t stream);
void freeWideBvh(WideBvh& bvh);

}  // namespace hdcx
