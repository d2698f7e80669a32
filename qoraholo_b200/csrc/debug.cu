// Registry of the per-translation-unit bounds-check records of the debug build (debug.cuh), and the
// totals behind qhk_debug_violations. In the release build no unit registers and the totals are zero.
#include <mutex>
#include <string>
#include <vector>

#include "debug.cuh"
#include "qhk_util.cuh"

namespace qhk {
namespace debug {

namespace {
struct Unit {
  const char* file;
  RecordReader read;
};
std::mutex& registry_mutex() {
  static std::mutex m;
  return m;
}
std::vector<Unit>& registry() {
  static std::vector<Unit> units;
  return units;
}
}  // namespace

bool register_reader(const char* unit, RecordReader reader) {
  std::lock_guard<std::mutex> lock(registry_mutex());
  registry().push_back({unit, reader});
  return true;
}

bool enabled() {
#ifdef QHK_DEBUG
  return true;
#else
  return false;
#endif
}

std::uint64_t violations(bool reset, std::string* first) {
  std::lock_guard<std::mutex> lock(registry_mutex());
  std::uint64_t total = 0;
  for (const Unit& u : registry()) {
    Record r{};
    const int e = u.read(&r, reset);
    if (e != 0) throw Error(kCudaError, std::string("debug record of ") + u.file + ": " +
                                            cudaGetErrorString(static_cast<cudaError_t>(e)));
    if (r.count != 0 && first != nullptr && first->empty()) {
      const std::string f = u.file;
      *first = f.substr(f.find_last_of('/') + 1) + ":" + std::to_string(r.line);
    }
    total += r.count;
  }
  return total;
}

}  // namespace debug
}  // namespace qhk
