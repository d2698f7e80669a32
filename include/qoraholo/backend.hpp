// Device selection of the public API. This build runs every stage on a CUDA device (B200,
// sm_100a); `cuda` is the default everywhere, and `cpu` is rejected with std::runtime_error --
// there is no host fallback.
#pragma once

namespace qoraholo {

enum class Backend { cpu, cuda };

// True when a CUDA device is visible.
[[nodiscard]] bool cuda_available();

}  // namespace qoraholo
