// Fixture generators of the public API (include/qoraholo/phantom.hpp). The rendered phantom and the
// analytic fields are computed on the device (qhk_render_phantom, qhk_forward_fields; csrc/synth.cu).
// Hologram synthesis stays on the host because its noise must be the reference's stream: draws of
// std::normal_distribution<float> from one std::mt19937_64 seeded with `seed`, taken view by view and
// row by row (src/phantom.cpp:193-221), so that seeded inputs are the reference's inputs.
#include <cmath>
#include <complex>
#include <numbers>
#include <random>
#include <vector>

#include "host_common.hpp"
#include "qoraholo/phantom.hpp"

namespace qoraholo {

namespace {

qhk_geometry c_geometry(const Geometry& g) { return {g.wavelength, g.n_medium, g.na, g.pixel}; }

std::vector<float> sphere_rows(std::span<const Sphere> spheres) {
  std::vector<float> rows;
  rows.reserve(5 * spheres.size());
  for (const Sphere& s : spheres) rows.insert(rows.end(), {s.z, s.y, s.x, s.radius, s.n});
  return rows;
}

// e^{i 2 pi f r_j} for the centred coordinates r_j = (j - n / 2) * pixel of one axis.
std::vector<std::complex<double>> axis_phases(double f, int n, double pixel) {
  std::vector<std::complex<double>> w(n);
  for (int j = 0; j < n; ++j) w[j] = std::polar(1.0, 2.0 * std::numbers::pi * f * ((j - n / 2) * pixel));
  return w;
}

}  // namespace

Array3<float> render_phantom(std::span<const Sphere> spheres, const Geometry& geometry, int nz, int n) {
  host::require(nz >= 1 && n >= 1, "render_phantom: empty shape");
  host::require_cuda(Backend::cuda);
  Array3<float> out(nz, n, n);
  const auto rows = sphere_rows(spheres);
  const qhk_geometry g = c_geometry(geometry);
  host::check(qhk_render_phantom(rows.data(), static_cast<int>(spheres.size()), &g, nz, n, out.data.data()));
  return out;
}

Array3<cfloat> forward_fields(std::span<const Sphere> spheres, std::span<const Illumination> illuminations,
                              const Geometry& geometry, int n, ScatteringModel model) {
  host::require(n >= 4 && n % 2 == 0, "forward_fields: n must be even");
  host::require(model != ScatteringModel::exact || spheres.size() == 1,
                "forward_fields: the exact model takes exactly one sphere");
  host::require_cuda(Backend::cuda);
  const int count = static_cast<int>(illuminations.size());
  Array3<cfloat> out(count, n, n);
  if (count == 0) return out;
  std::vector<float> il(2 * illuminations.size());
  for (std::size_t a = 0; a < illuminations.size(); ++a) {
    il[2 * a] = illuminations[a].fy;
    il[2 * a + 1] = illuminations[a].fx;
  }
  const auto rows = sphere_rows(spheres);
  const qhk_geometry g = c_geometry(geometry);
  const int m = model == ScatteringModel::born ? QHK_MODEL_BORN : model == ScatteringModel::rytov ? QHK_MODEL_RYTOV
                                                                                                   : QHK_MODEL_EXACT;
  host::check(qhk_forward_fields(rows.data(), static_cast<int>(spheres.size()), il.data(), count, &g, n, m,
                                 out.data.data()));
  return out;
}

Array3<float> synthesize_holograms(const Array3<cfloat>& ratio, std::span<const Illumination> illuminations,
                                   const Geometry& geometry, const HologramOptions& options) {
  if (static_cast<std::size_t>(ratio.nz) != illuminations.size()) {
    throw std::invalid_argument("synthesize_holograms: need one illumination per field");
  }
  // |R + u_in r|^2 = A^2 + |r|^2 + 2 A Re(e^{i 2 pi ((fy + cy) y + (fx + cx) x)} r) with the reference wave
  // R = A e^{-i 2 pi (cy y + cx x)} and the incident wave u_in = e^{i 2 pi (fy y + fx x)}: the phase
  // factor separates into one row and one column factor per view.
  Array3<float> out(ratio.nz, ratio.ny, ratio.nx);
  std::mt19937_64 rng(options.seed);
  std::normal_distribution<float> noise(0.0f, options.noise);
  const double amp = options.reference_amplitude;
  const double pixel = geometry.pixel;
  for (int a = 0; a < ratio.nz; ++a) {
    const auto wy = axis_phases(double(illuminations[a].fy) + options.carrier[0], ratio.ny, pixel);
    const auto wx = axis_phases(double(illuminations[a].fx) + options.carrier[1], ratio.nx, pixel);
    for (int y = 0; y < ratio.ny; ++y) {
      for (int x = 0; x < ratio.nx; ++x) {
        const std::complex<double> r(ratio(a, y, x));
        const double cross = (wy[y] * wx[x] * r).real();
        float v = static_cast<float>(amp * amp + std::norm(r) + 2.0 * amp * cross);
        if (options.noise > 0) v += noise(rng);
        out(a, y, x) = v;
      }
    }
  }
  return out;
}

}  // namespace qoraholo
