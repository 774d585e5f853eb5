// er_nvtx.h -- NVTX ranges around the library's phases (upload, grid, batch,
// Widom, pocket blocking, server jobs). NVTX v3 is header-only: without a
// profiler attached a range costs a branch on an unset function pointer.
#pragma once
#include <nvtx3/nvToolsExt.h>

namespace er {

struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

}  // namespace er
