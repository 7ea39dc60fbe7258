// sr_trace.hpp — NVTX ranges around the host-side phases of the library's
// calls (validation and compile, subtree detection, uploads, launch shape
// tuning, launches, read-backs), so that a timeline tool shows where a
// generation's host time goes.  The reference marks one phase the same way
// (nvtxRangePush "CPU: Parse & Split Trees", src/cleaned/cl_gpu_eval.cu:369-381).
// NVTX 3 is header-only; with no tool attached a range costs a few
// nanoseconds.
#pragma once
#include <nvtx3/nvToolsExt.h>

namespace sr {

class TraceRange {
 public:
  explicit TraceRange(const char *name) { nvtxRangePushA(name); }
  ~TraceRange() { nvtxRangePop(); }
  TraceRange(const TraceRange &) = delete;
  TraceRange &operator=(const TraceRange &) = delete;
};

}  // namespace sr

#define SR_TRACE_CAT2(a, b) a##b
#define SR_TRACE_CAT(a, b) SR_TRACE_CAT2(a, b)
#define SR_TRACE(name) ::sr::TraceRange SR_TRACE_CAT(sr_trace_, __LINE__)(name)
