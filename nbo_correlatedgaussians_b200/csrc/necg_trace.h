// necg_trace.h -- NVTX ranges over the library's entry points, so a timeline
// tool (Nsight Systems, or ncu --nvtx filters) shows which call enqueued which
// kernels.  NVTX is header-only and costs a few nanoseconds per range when no
// tool is attached.
#pragma once
#include <nvtx3/nvToolsExt.h>

namespace necg {

struct TraceRange {
    explicit TraceRange(const char *name) { nvtxRangePushA(name); }
    ~TraceRange() { nvtxRangePop(); }
    TraceRange(const TraceRange &) = delete;
    TraceRange &operator=(const TraceRange &) = delete;
};

}  // namespace necg
