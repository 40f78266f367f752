// NVTX ranges around the library's entry points and phases (header-only NVTX3): a profiler
// such as Nsight Systems shows them on the host timeline beside the kernels they enqueue;
// without a tool attached each push/pop is a check of one pointer.
#pragma once
#include <nvtx3/nvToolsExt.h>

namespace tsvm {

class TraceRange {
 public:
  explicit TraceRange(const char *name) { nvtxRangePushA(name); }
  ~TraceRange() { nvtxRangePop(); }
  TraceRange(const TraceRange &) = delete;
  TraceRange &operator=(const TraceRange &) = delete;
};

// Consecutive phases of one call: next() closes the open range and opens the next; the
// destructor closes the last, so an early return leaves the ranges balanced.
class TracePhases {
 public:
  TracePhases() = default;
  void next(const char *name) {
    if (open_) nvtxRangePop();
    nvtxRangePushA(name);
    open_ = true;
  }
  ~TracePhases() {
    if (open_) nvtxRangePop();
  }
  TracePhases(const TracePhases &) = delete;
  TracePhases &operator=(const TracePhases &) = delete;

 private:
  bool open_ = false;
};

}  // namespace tsvm
