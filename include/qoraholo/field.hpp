// Off-axis holography: sideband search and field retrieval. Declarations as in the reference's
// include/qoraholo/field.hpp; the default backend is CUDA.
#pragma once

#include <array>
#include <optional>

#include "qoraholo/array.hpp"
#include "qoraholo/backend.hpp"

namespace qoraholo {

// +1 sideband peak relative to DC in pixels: integer bin and sub-pixel estimate.
struct Sideband {
  int iy = 0;
  int ix = 0;
  float y = 0;
  float x = 0;
  float magnitude = 0;
};

struct FieldOptions {
  std::optional<std::array<float, 2>> center;  // {y, x} from DC; empty: search the first hologram
  float radius = 0;                            // crop radius; <= 0: |center| / 3
  float dc_exclusion = 0;                      // DC radius skipped by the search; <= 0: N / 8
  int output_size = 0;                         // field side; 0: the hologram side
};

[[nodiscard]] Sideband find_sideband(const Array3<float>& holograms, float dc_exclusion = 0);

// Square holograms with an even side -> fields (count, m, m); field pixel = hologram pixel * N / m.
[[nodiscard]] Array3<cfloat> extract_fields(const Array3<float>& holograms,
                                            const FieldOptions& options = {},
                                            Backend backend = Backend::cuda);

// sample / background pixel by pixel; background holds one field or one per sample field.
[[nodiscard]] Array3<cfloat> field_ratio(const Array3<cfloat>& sample,
                                         const Array3<cfloat>& background);

}  // namespace qoraholo
