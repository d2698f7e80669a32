// Least-squares phase unwrapping and the complex Rytov phase. Declarations as in the reference's
// include/qoraholo/unwrap.hpp; the default backend is CUDA.
#pragma once

#include "qoraholo/array.hpp"
#include "qoraholo/backend.hpp"

namespace qoraholo {

// Unweighted least-squares unwrap of each image (even sides), congruent to the input mod 2 pi.
[[nodiscard]] Array3<float> unwrap(const Array3<float>& wrapped, Backend backend = Backend::cuda);

// log|r| + i unwrap(arg r), shifted by a multiple of 2 pi so that the border mean is in (-pi, pi].
[[nodiscard]] Array3<cfloat> rytov(const Array3<cfloat>& ratio, Backend backend = Backend::cuda);

}  // namespace qoraholo
