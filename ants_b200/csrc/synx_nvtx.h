// NVTX ranges for the library's host-side phases (the CUDA toolkit's header-only NVTX3).
#pragma once

#include <nvtx3/nvToolsExt.h>

namespace synx {

// An NVTX range over a host-side phase (level setup, iteration, readback, batch step), labelled
// with its name and a number (the level, or the number of contexts): it shows the stage's structure
// on a profiler timeline and costs nothing unless a profiler attaches.
struct NvtxRange {
  NvtxRange(const char* name, long long value) {
    nvtxEventAttributes_t a = {};
    a.version = NVTX_VERSION;
    a.size = NVTX_EVENT_ATTRIB_STRUCT_SIZE;
    a.messageType = NVTX_MESSAGE_TYPE_ASCII;
    a.message.ascii = name;
    a.payloadType = NVTX_PAYLOAD_TYPE_INT64;
    a.payload.llValue = value;
    nvtxRangePushEx(&a);
  }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

}  // namespace synx
