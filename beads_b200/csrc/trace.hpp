// Named NVTX ranges around the engine's host-side phases (run, eval,
// minimize, autotune, adjoint sweeps, execute), so a timeline profiler shows
// them by name.  NVTX 3 is header-only: with no tool attached a range costs a
// branch on a null function pointer.
#pragma once

#include <nvtx3/nvToolsExt.h>

namespace bb {

class TraceRange {
 public:
  explicit TraceRange(const char* name) { nvtxRangePushA(name); }
  ~TraceRange() { nvtxRangePop(); }
  TraceRange(const TraceRange&) = delete;
  TraceRange& operator=(const TraceRange&) = delete;
};

}  // namespace bb
