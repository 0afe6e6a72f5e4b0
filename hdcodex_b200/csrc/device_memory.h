// device_memory.h - every device allocation of the library, counted per
// device against an optional budget (hdcx_set_device_memory_limit).
//
// Path arenas, scene buffers, the BVH build's temporaries and the radiance
// cache all allocate here, so a host application can bound what the tracer
// takes of a GPU it shares, and an allocation past the budget fails the same
// way an exhausted device does: with OutOfDeviceMemory, which the C ABI
// reports as HDCX_ERROR_OUT_OF_MEMORY, and nothing launched.
#pragma once

#include <cstddef>
#include <cstdint>
#include <stdexcept>

namespace hdcx {

// Thrown when the budget or the device has no room; the message contains
// "out of memory".
struct OutOfDeviceMemory : std::runtime_error {
    using std::runtime_error::runtime_error;
};

// cudaMalloc of `bytes` (at least 16) on the current device, counted against
// that device's budget. Other CUDA errors throw std::runtime_error.
void* deviceMalloc(size_t bytes);
// Frees memory from deviceMalloc; null is ignored.
void deviceFree(void* p);

// Budget of `device` in bytes (0: none); allocations already made stay.
void setDeviceMemoryLimit(int device, uint64_t bytes);
uint64_t deviceMemoryLimit(int device);
// Bytes the library holds on `device` (deviceMalloc minus deviceFree).
uint64_t deviceMemoryInUse(int device);

}  // namespace hdcx
