// device_memory.cpp - counted device allocations (see device_memory.h).
#include "device_memory.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <string>
#include <unordered_map>
#include <utility>

namespace hdcx {
namespace {

constexpr int kDevices = 64;

struct Ledger {
    std::mutex lock;
    uint64_t limit[kDevices] = {};
    uint64_t inUse[kDevices] = {};
    std::unordered_map<void*, std::pair<int, uint64_t>> blocks;
};

Ledger& ledger()
{
    // Never destroyed: buffers may be freed after static destructors ran.
    static Ledger* l = new Ledger();
    return *l;
}

int checkedDevice(int device)
{
    if (device < 0 || device >= kDevices) throw std::invalid_argument("device ordinal out of range");
    return device;
}

}  // namespace

void* deviceMalloc(size_t bytes)
{
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) throw std::runtime_error(std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    checkedDevice(device);
    const uint64_t size = std::max<uint64_t>(bytes, 16);
    Ledger& l = ledger();
    {
        std::lock_guard<std::mutex> guard(l.lock);
        if (l.limit[device] != 0 && l.inUse[device] + size > l.limit[device]) {
            throw OutOfDeviceMemory("device " + std::to_string(device) + " out of memory: an allocation of " +
                                    std::to_string(size) + " bytes exceeds the library's budget of " +
                                    std::to_string(l.limit[device]) + " bytes (" + std::to_string(l.inUse[device]) +
                                    " in use)");
        }
        l.inUse[device] += size;  // reserved before the call, so concurrent allocations respect the budget
    }
    void* p = nullptr;
    e = cudaMalloc(&p, size);
    std::lock_guard<std::mutex> guard(l.lock);
    if (e != cudaSuccess) {
        l.inUse[device] -= size;
        cudaGetLastError();
        if (e == cudaErrorMemoryAllocation) {
            throw OutOfDeviceMemory("device " + std::to_string(device) + " out of memory: cudaMalloc of " +
                                    std::to_string(size) + " bytes failed");
        }
        throw std::runtime_error(std::string("cudaMalloc: ") + cudaGetErrorString(e));
    }
    l.blocks[p] = {device, size};
    return p;
}

void deviceFree(void* p)
{
    if (!p) return;
    Ledger& l = ledger();
    {
        std::lock_guard<std::mutex> guard(l.lock);
        auto it = l.blocks.find(p);
        if (it != l.blocks.end()) {
            l.inUse[it->second.first] -= it->second.second;
            l.blocks.erase(it);
        }
    }
    cudaFree(p);
}

void setDeviceMemoryLimit(int device, uint64_t bytes)
{
    Ledger& l = ledger();
    std::lock_guard<std::mutex> guard(l.lock);
    l.limit[checkedDevice(device)] = bytes;
}

uint64_t deviceMemoryLimit(int device)
{
    Ledger& l = ledger();
    std::lock_guard<std::mutex> guard(l.lock);
    return l.limit[checkedDevice(device)];
}

uint64_t deviceMemoryInUse(int device)
{
    Ledger& l = ledger();
    std::lock_guard<std::mutex> guard(l.lock);
    return l.inUse[checkedDevice(device)];
}

}  // namespace hdcx
