// Host-side NVTX ranges of the library's phases, in the domain "ndt_b200"
// (NVTX3, header only: without a tool attached a range costs a pointer
// test).  ncu selects kernels by range, e.g. (always with
// --clock-control none, so that ncu leaves the GPU clocks alone, and a small
// capture count):
//   ncu --nvtx --nvtx-include "ndt_b200@rounds/" --clock-control none \
//       --metrics gpu__time_duration.sum -c 60 ...
#pragma once

#include <nvtx3/nvToolsExt.h>

namespace ndt {

inline nvtxDomainHandle_t nvtx_domain() {
    static nvtxDomainHandle_t d = nvtxDomainCreateA("ndt_b200");
    return d;
}

// Pushes a named range for the life of the object.
class NvtxRange {
public:
    explicit NvtxRange(const char *name) {
        nvtxEventAttributes_t a = {};
        a.version = NVTX_VERSION;
        a.size = NVTX_EVENT_ATTRIB_STRUCT_SIZE;
        a.messageType = NVTX_MESSAGE_TYPE_ASCII;
        a.message.ascii = name;
        nvtxDomainRangePushEx(nvtx_domain(), &a);
    }
    ~NvtxRange() { nvtxDomainRangePop(nvtx_domain()); }
    NvtxRange(const NvtxRange &) = delete;
    NvtxRange &operator=(const NvtxRange &) = delete;
};

}  // namespace ndt
