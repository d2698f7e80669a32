// Optical diffraction tomography: Rytov fields -> refractive-index volume by the Fourier
// diffraction theorem, with an optional missing-cone solver. Declarations as in the reference's
// include/qoraholo/odt.hpp; defaults select the CUDA backend.
#pragma once

#include <span>
#include <vector>

#include "qoraholo/array.hpp"
#include "qoraholo/backend.hpp"

namespace qoraholo {

// Micrometres and cycles per micrometre.
struct Geometry {
  float wavelength = 0.532f;  // in vacuum
  float n_medium = 1.337f;
  float na = 1.2f;            // detection numerical aperture
  float pixel = 0.1f;         // field pixel in the sample plane, also the voxel side
};

// Lateral frequency (fy, fx) of an incident plane wave; |f| < n_medium / wavelength.
struct Illumination {
  float fy = 0;
  float fx = 0;
};

// Both run the same deterministic mapping on the device (one owner per voxel, illumination
// order, no atomics); the names are kept for source compatibility.
enum class Mapping { gather, scatter };

enum class Solver {
  gerchberg_papoulis,  // n >= n_medium in real space, measured voxels restored in k-space
  tv,                  // FISTA on the data term plus tv_weight * k0^2 * TV, x >= 0
};

// Gerchberg-Papoulis on half spectra (real potential) or on full complex spectra.
enum class GpTransform { r2c, c2c };

struct OdtOptions {
  int nz = 0;          // axial voxels; 0: the field side
  int iterations = 0;  // solver iterations; 0: plain Rytov ODT
  Solver solver = Solver::gerchberg_papoulis;
  GpTransform gp_transform = GpTransform::r2c;
  float tv_weight = 1e-2f;  // on n^2 - n_medium^2, independent of the wavelength
  int tv_inner = 10;        // FGP steps of each TV proximal step
  Mapping mapping = Mapping::gather;
  Backend backend = Backend::cuda;
};

struct OdtResult {
  Array3<float> ri;   // (nz, n, n), centre-origin
  double filled = 0;  // fraction of k-space voxels that received data
};

[[nodiscard]] OdtResult reconstruct(const Array3<cfloat>& rytov_fields,
                                    std::span<const Illumination> illuminations,
                                    const Geometry& geometry, const OdtOptions& options = {});

// Normal incidence, then count - 1 directions evenly spaced on a circle at na_illumination.
[[nodiscard]] std::vector<Illumination> circular_scan(int count, float na_illumination,
                                                      const Geometry& geometry);

}  // namespace qoraholo
