// Device-side bounds checks of the debug build (compiled with QHK_DEBUG: `python qoraholo_b200/_build.py
// --debug` writes qoraholo_b200/debug/libqhk.so).
//
// QHK_CHECK(cond) guards one access or one queue item: in the release build it is the constant `true` and
// the compiler removes it; in the debug build a false condition is recorded -- a count, and the source
// line of the first one seen -- and the caller skips the access it guards, so a bad index shows up as a
// record the host reads (qhk_debug_violations) instead of a memory fault, and the context stays usable.
// Nothing traps. A skipped tile load leaves its mbarrier short of bytes, so the bounded wait on it ends
// and reports a timeout as well.
//
// The record is a static device variable, one per translation unit that includes this header (the
// library is built without relocatable device code); each such unit registers a reader of its own
// record with debug.cu at load time.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>

namespace qhk {
namespace debug {

struct Record {
  unsigned long long count;  // failed checks
  int line;                  // source line of the first failed check (0: none)
  int pad;
};

// Register a reader of one translation unit's record (debug.cu). `reset` clears it.
using RecordReader = int (*)(Record* out, bool reset);
bool register_reader(const char* unit, RecordReader reader);

// True in the debug build. violations(): failed checks of all registered units since the last reset
// (cleared when `reset`), with "file:line" of one unit's first failure in *first when there was one.
bool enabled();
std::uint64_t violations(bool reset, std::string* first);

#ifdef QHK_DEBUG

namespace {
__device__ Record g_record;

__device__ __noinline__ void record_failure(int line) {
  if (atomicAdd(&g_record.count, 1ull) == 0ull) atomicExch(&g_record.line, line);
}

int read_record(Record* out, bool reset) {
  cudaError_t e = cudaMemcpyFromSymbol(out, g_record, sizeof(Record));
  if (e == cudaSuccess && reset) {
    const Record zero{};
    e = cudaMemcpyToSymbol(g_record, &zero, sizeof(Record));
  }
  return e == cudaSuccess ? 0 : static_cast<int>(e);
}

const bool g_registered = register_reader(__FILE__, read_record);
}  // namespace

__device__ __forceinline__ bool check(bool ok, int line) {
  if (!ok) record_failure(line);
  return ok;
}

#define QHK_CHECK(...) (::qhk::debug::check(static_cast<bool>(__VA_ARGS__), __LINE__))

#else

#define QHK_CHECK(...) true

#endif

// Bytes of dynamic shared memory this launch was given (for layout checks).
__device__ __forceinline__ unsigned dynamic_smem_bytes() {
  unsigned v;
  asm("mov.u32 %0, %%dynamic_smem_size;" : "=r"(v));
  return v;
}

}  // namespace debug
}  // namespace qhk
