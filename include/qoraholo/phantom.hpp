// Synthetic test objects and holograms (fixture generators). Declarations as in the reference's
// include/qoraholo/phantom.hpp.
#pragma once

#include <array>
#include <cstdint>
#include <span>

#include "qoraholo/array.hpp"
#include "qoraholo/odt.hpp"

namespace qoraholo {

// Uniform sphere centred (z, y, x) micrometres from the volume centre; painted in order, each
// entirely inside or outside every earlier one.
struct Sphere {
  float z = 0;
  float y = 0;
  float x = 0;
  float radius = 1;
  float n = 1.38f;
};

enum class ScatteringModel { born, rytov, exact };

[[nodiscard]] Array3<float> render_phantom(std::span<const Sphere> spheres,
                                           const Geometry& geometry, int nz, int n);

[[nodiscard]] Array3<cfloat> forward_fields(std::span<const Sphere> spheres,
                                            std::span<const Illumination> illuminations,
                                            const Geometry& geometry, int n,
                                            ScatteringModel model = ScatteringModel::rytov);

struct HologramOptions {
  std::array<float, 2> carrier{5.0f, 5.0f};  // reference tilt {fy, fx}, cycles per micrometre
  float reference_amplitude = 1;
  float noise = 0;  // standard deviation of additive Gaussian noise
  std::uint64_t seed = 1;
};

[[nodiscard]] Array3<float> synthesize_holograms(const Array3<cfloat>& ratio,
                                                 std::span<const Illumination> illuminations,
                                                 const Geometry& geometry,
                                                 const HologramOptions& options = {});

}  // namespace qoraholo
