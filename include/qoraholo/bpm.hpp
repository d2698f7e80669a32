// Multi-slice beam propagation: forward model and gradient inversion. Declarations as in the
// reference's include/qoraholo/bpm.hpp; the default backend is CUDA.
#pragma once

#include <span>
#include <vector>

#include "qoraholo/array.hpp"
#include "qoraholo/backend.hpp"
#include "qoraholo/odt.hpp"

namespace qoraholo {

struct BpmOptions {
  // Weight the scattered part of each slice by the obliquity of the scattered wave (capped at the
  // detection NA), which makes the weak-object limit the first Born approximation at every angle.
  bool obliquity = true;
  Backend backend = Backend::cuda;
};

// Refractive index (nz, n, n) -> field ratios at z = 0, (count, n, n).
[[nodiscard]] Array3<cfloat> bpm_forward(const Array3<float>& ri,
                                         std::span<const Illumination> illuminations,
                                         const Geometry& geometry, const BpmOptions& options = {});

struct BpmSolveOptions {
  int iterations = 20;
  int batch = 0;          // illuminations per step; 0 or count: all, with FISTA momentum
  float step = 1.0f;      // multiple of 1 / L
  float tv_weight = 0.0f; // weight of TV(n - n_medium); 0: n >= n_medium only
  int tv_inner = 10;
  bool obliquity = true;
  Backend backend = Backend::cuda;
};

struct BpmResult {
  Array3<float> ri;
  std::vector<double> loss;  // 0.5 / count * sum |bpm(x) - fields|^2 per iteration
};

[[nodiscard]] BpmResult bpm_reconstruct(const Array3<cfloat>& fields,
                                        std::span<const Illumination> illuminations,
                                        const Geometry& geometry, const Array3<float>& initial,
                                        const BpmSolveOptions& options = {});

}  // namespace qoraholo
