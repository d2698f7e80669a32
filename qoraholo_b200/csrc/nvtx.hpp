// Named ranges on the host timeline (NVTX) around each stage's launches, so that a profiler can show
// the stages and filter kernels by stage (ncu --nvtx --nvtx-include "qhk:solve/"). Without a tool
// attached a range costs one check of an unset function pointer. NVTX 3 is header-only.
#pragma once

#include <nvtx3/nvToolsExt.h>

namespace qhk {

class NvtxRange {
 public:
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

}  // namespace qhk
