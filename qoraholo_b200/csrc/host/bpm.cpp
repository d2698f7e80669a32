// BPM forward model and gradient inversion of the public API (include/qoraholo/bpm.hpp) over the
// C ABI. Validation as the reference's dispatch (src/api.cpp:141-201).
#include <string>

#include "host_common.hpp"
#include "qoraholo/bpm.hpp"

namespace qoraholo {

namespace {

void checked_bpm(int nz, int n, int count, std::span<const Illumination> il, const Geometry& g, Backend backend,
                 const char* who) {
  const std::string w(who);
  host::require(n >= 4 && n % 2 == 0 && nz >= 1, w + ": volume must be (nz, n, n) with an even n");
  host::require(count >= 1 && static_cast<std::size_t>(count) == il.size(), w + ": need one illumination per field");
  host::require(g.wavelength > 0 && g.pixel > 0 && g.n_medium > 0 && g.na > 0, w + ": geometry values must be positive");
  const float fm = g.n_medium / g.wavelength;
  for (const auto& v : il) {
    host::require(v.fy * v.fy + v.fx * v.fx < fm * fm, w + ": illumination frequency beyond n_medium / wavelength");
  }
  host::require_cuda(backend);
}

}  // namespace

Array3<cfloat> bpm_forward(const Array3<float>& ri, std::span<const Illumination> illuminations,
                           const Geometry& geometry, const BpmOptions& options) {
  host::require(ri.ny == ri.nx, "bpm_forward: volume must be (nz, n, n)");
  const int count = static_cast<int>(illuminations.size());
  checked_bpm(ri.nz, ri.nx, count, illuminations, geometry, options.backend, "bpm_forward");
  const qhk_geometry g{geometry.wavelength, geometry.n_medium, geometry.na, geometry.pixel};
  Array3<cfloat> out(count, ri.nx, ri.nx);
  host::check(qhk_bpm_forward(ri.data.data(), ri.nz, ri.nx, reinterpret_cast<const float*>(illuminations.data()),
                              count, &g, options.obliquity ? 1 : 0, out.data.data()));
  return out;
}

BpmResult bpm_reconstruct(const Array3<cfloat>& fields, std::span<const Illumination> illuminations,
                          const Geometry& geometry, const Array3<float>& initial, const BpmSolveOptions& options) {
  host::require(initial.ny == initial.nx && fields.ny == initial.ny && fields.nx == initial.nx,
                "bpm_reconstruct: fields (count, n, n) and initial (nz, n, n) must share n");
  host::require(options.iterations >= 0 && options.step > 0 && options.tv_weight >= 0 && options.tv_inner >= 1,
                "bpm_reconstruct: invalid solver options");
  checked_bpm(initial.nz, initial.nx, fields.nz, illuminations, geometry, options.backend, "bpm_reconstruct");
  const qhk_geometry g{geometry.wavelength, geometry.n_medium, geometry.na, geometry.pixel};
  const qhk_bpm_solve_options o{options.iterations, options.batch, options.step, options.tv_weight, options.tv_inner,
                                options.obliquity ? 1 : 0};
  BpmResult r;
  r.ri = Array3<float>(initial.nz, initial.ny, initial.nx);
  r.loss.resize(options.iterations);
  host::check(qhk_bpm_reconstruct(fields.data.data(), fields.nz, fields.nx,
                                  reinterpret_cast<const float*>(illuminations.data()), &g, initial.data.data(),
                                  initial.nz, &o, r.ri.data.data(), r.loss.data()));
  return r;
}

}  // namespace qoraholo
