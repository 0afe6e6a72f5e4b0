// nvtx_range.h - named host ranges for profilers, in an "hdcx" NVTX domain.
//
// NVTX v3 is header-only: until a tool (Nsight Systems, Nsight Compute's
// range filters) injects itself, each push/pop is one call through a table
// of no-op entries, so the ranges stay compiled in. They mark the stages a
// profile of a Hydra render pass wants to see beside the kernels: scene
// packing, the BVH build, each render call and its waves, batches, the
// autotuner and the read-back.
#pragma once

#include <nvtx3/nvToolsExt.h>

namespace hdcx {

inline nvtxDomainHandle_t nvtxDomain()
{
    static const nvtxDomainHandle_t domain = nvtxDomainCreateA("hdcx");
    return domain;
}

class NvtxRange {
public:
    explicit NvtxRange(const char* name)
    {
        nvtxEventAttributes_t a{};
        a.version = NVTX_VERSION;
        a.size = NVTX_EVENT_ATTRIB_STRUCT_SIZE;
        a.messageType = NVTX_MESSAGE_TYPE_ASCII;
        a.message.ascii = name;
        nvtxDomainRangePushEx(nvtxDomain(), &a);
    }
    ~NvtxRange() { nvtxDomainRangePop(nvtxDomain()); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

}  // namespace hdcx
