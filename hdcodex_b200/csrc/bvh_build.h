// bvh_build.h - on-GPU construction of the 8-wide compressed BVH.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>
#include <vector>

#include "device/common.cuh"

namespace hdcx {

struct WideBvh {
    WideNode* nodes = nullptr;
    float4* triVerts = nullptr;  // 3 float4 per leaf-ordered triangle
    uint32_t nodeCount = 0;
    uint32_t depth = 0;
    uint32_t triangleCount = 0;
    float sceneScale = 0.0f;            // the quantisation floor it was built (or last refitted) with
    std::vector<uint32_t> levelStart;   // nodes of level d: [levelStart[d], levelStart[d+1])
    float4* nodeBoxes = nullptr;        // refit scratch: each node's box (lo, hi), allocated by the first refit
};

// Builds the BVH of `triangleCount` triangles given as device vertex (xyzw)
// and index arrays. sceneScale = max(|coordinate|, scene extent) bounds the
// quantisation step from below. The id stored with each leaf triangle is
// primIds[position] (null: its position in the list). The leaf copy's
// second vertex carries opacityHint[position] in .w (null: -1): a triangle's
// constant opacity when its material has no opacity texture, else -1 (the
// traversal then samples the texture). Synchronous on `stream`; throws
// std::runtime_error on a CUDA failure.
WideBvh buildWideBvh(const float4* vertices, const uint32_t* indices, uint32_t triangleCount, float sceneScale,
                     cudaStream_t stream, const uint32_t* primIds = nullptr, const float* opacityHint = nullptr);

// Refits a BVH built without primIds to moved vertices (same triangles, same
// indices): leaf triangle copies, then every node's child boxes level by
// level from the leaves up, quantised as the build quantises them. The tree
// keeps its topology. Synchronous on `stream`.
void refitWideBvh(WideBvh& bvh, const float4* vertices, const uint32_t* indices, float sceneScale, cudaStream_t stream);
void freeWideBvh(WideBvh& bvh);

}  // namespace hdcx
