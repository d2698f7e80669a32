// Shared helpers of the host C++ layer: argument checks with the reference's exception types and
// the mapping of C ABI status codes back to them.
#pragma once

#include <stdexcept>
#include <string>

#include "qoraholo/backend.hpp"
#include "qoraholo_b200.h"

namespace qoraholo::host {

inline void require(bool ok, const std::string& what) {
  if (!ok) throw std::invalid_argument(what);
}

// Throws the exception class of a QHK_* status (include/qoraholo_b200.h).
inline void check(int status) {
  if (status == QHK_OK) return;
  const std::string msg = qhk_last_error();
  if (status == QHK_INVALID_ARGUMENT) throw std::invalid_argument(msg);
  if (status == QHK_LOGIC_ERROR) throw std::logic_error(msg);
  throw std::runtime_error(msg);
}

// This build has one backend; `cpu` fails loudly rather than falling back to host code.
inline void require_cuda(Backend backend) {
  if (backend != Backend::cuda) {
    throw std::runtime_error("qoraholo-b200 runs on CUDA devices only: use Backend::cuda");
  }
  if (!qhk_device_present()) throw std::runtime_error("no CUDA device available");
}

inline void require_even_square(int ny, int nx, const char* who) {
  require(ny == nx && nx >= 4 && nx % 2 == 0, std::string(who) + ": images must be square with an even side");
}

}  // namespace qoraholo::host
