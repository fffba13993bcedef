// NVTX ranges over the library's host-side phases (a step, a batched run,
// the adjoint, a freeze-out surface), so that profilers that record NVTX
// (ncu --nvtx with --nvtx-include, nsys) can select their kernels by name.
// NVTX 3 is header-only: without such a tool attached a push/pop pair only
// checks a function pointer.
#pragma once
#include <nvtx3/nvToolsExt.h>

struct VhNvtxRange {
  explicit VhNvtxRange(const char* name) { nvtxRangePushA(name); }
  ~VhNvtxRange() { nvtxRangePop(); }
  VhNvtxRange(const VhNvtxRange&) = delete;
  VhNvtxRange& operator=(const VhNvtxRange&) = delete;
};
