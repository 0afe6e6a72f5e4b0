// render_static.h - the allocation-free render behind hdcx_render_static.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "integrator.h"

namespace hdcx {

// Largest image (width * height) the static scratch holds per-pixel sums for.
constexpr uint64_t kStaticMaxPixels = 1ull << 20;
// Paths per wave in the static scratch, and shadow-ray slots per path.
constexpr uint64_t kStaticWavePaths = 1ull << 16;
constexpr uint32_t kStaticShadowPerPath = 3;
// Size of the static scratch array (checked against its layout at compile time).
constexpr uint64_t kStaticScratchBytes = 62063104ull;

// Renders like renderFrame into the caller's running-mean buffer `rgba`
// (width * height float4, device memory) with all scratch taken from the
// static array; returns once the GPU work has finished, with the render's
// traversal fault bits (kTraversalOverflow, kTraversalBudget; 0: none), which
// the traversal kernels OR into the render statistics. Allocates nothing.
unsigned int renderStatic(const DeviceScene& scene, const FrameConst& frame, float4* rgba, cudaStream_t stream);

}  // namespace hdcx
