// Free functions of the public C++ API (include/qoraholo/*.hpp) over the C ABI of libqhk.so.
// Argument validation follows the reference's dispatch layer (src/api.cpp:13-137) so that the
// same calls raise the same exception types; the computation runs on the device.
#include <cmath>
#include <numbers>
#include <string>

#include "host_common.hpp"
#include "qoraholo/qoraholo.hpp"

namespace qoraholo {

using host::check;
using host::require;

bool cuda_available() { return qhk_device_present() != 0; }

Sideband find_sideband(const Array3<float>& holograms, float dc_exclusion) {
  const int n = holograms.nx;
  require(holograms.nz >= 1 && n == holograms.ny && n % 2 == 0 && n >= 4,
          "find_sideband: holograms must be square with an even side");
  host::require_cuda(Backend::cuda);
  Sideband s;
  check(qhk_find_sideband(holograms.data.data(), n, dc_exclusion, &s.iy, &s.ix, &s.y, &s.x, &s.magnitude));
  return s;
}

namespace {

// crop_plan validation (src/api.cpp:52-60) ahead of the device call.
int checked_output(const FieldOptions& o, std::array<float, 2> c, int n) {
  const int out = o.output_size > 0 ? o.output_size : n;
  float radius = o.radius;
  if (radius <= 0) radius = std::hypot(c[0], c[1]) / 3.0f;
  require(out % 2 == 0 && out <= n, "extract_fields: output_size must be even and <= N");
  require(radius > 0 && radius <= static_cast<float>(out) / 2.0f,
          "extract_fields: crop radius must fit in the output window");
  return out;
}

}  // namespace

Array3<cfloat> extract_fields(const Array3<float>& holograms, const FieldOptions& options, Backend backend) {
  host::require_even_square(holograms.ny, holograms.nx, "extract_fields");
  require(holograms.nz >= 1, "extract_fields: empty stack");
  host::require_cuda(backend);
  std::array<float, 2> c{};
  if (options.center) {
    c = *options.center;
  } else {
    const Sideband s = find_sideband(holograms, options.dc_exclusion);
    c = {static_cast<float>(s.iy), static_cast<float>(s.ix)};
  }
  const int m = checked_output(options, c, holograms.nx);
  Array3<cfloat> out(holograms.nz, m, m);
  check(qhk_extract_fields(holograms.data.data(), holograms.nz, holograms.nx, c[0], c[1], options.radius,
                           options.output_size, out.data.data()));
  return out;
}

Array3<cfloat> field_ratio(const Array3<cfloat>& sample, const Array3<cfloat>& background) {
  if (sample.ny != background.ny || sample.nx != background.nx ||
      (background.nz != 1 && background.nz != sample.nz)) {
    throw std::invalid_argument("field_ratio: background shape does not match");
  }
  host::require_cuda(Backend::cuda);
  Array3<cfloat> out(sample.nz, sample.ny, sample.nx);
  if (sample.size() == 0) return out;
  check(qhk_field_ratio(sample.data.data(), sample.nz, sample.ny, sample.nx, background.data.data(), background.nz,
                        out.data.data()));
  return out;
}

Array3<float> unwrap(const Array3<float>& wrapped, Backend backend) {
  require(wrapped.ny % 2 == 0 && wrapped.nx % 2 == 0 && wrapped.ny >= 2 && wrapped.nx >= 2,
          "unwrap: image sides must be even");
  host::require_cuda(backend);
  Array3<float> out(wrapped.nz, wrapped.ny, wrapped.nx);
  if (wrapped.nz == 0) return out;
  check(qhk_unwrap(wrapped.data.data(), wrapped.nz, wrapped.ny, wrapped.nx, out.data.data()));
  return out;
}

Array3<cfloat> rytov(const Array3<cfloat>& ratio, Backend backend) {
  require(ratio.ny % 2 == 0 && ratio.nx % 2 == 0 && ratio.ny >= 4 && ratio.nx >= 4,
          "rytov: image sides must be even");
  host::require_cuda(backend);
  Array3<cfloat> out(ratio.nz, ratio.ny, ratio.nx);
  if (ratio.nz == 0) return out;
  check(qhk_rytov(ratio.data.data(), ratio.nz, ratio.ny, ratio.nx, out.data.data()));
  return out;
}

namespace host {

qhk_odt_options odt_options(const OdtOptions& o) {
  return qhk_odt_options{o.nz,
                         o.iterations,
                         o.solver == Solver::tv ? QHK_SOLVER_TV : QHK_SOLVER_GP,
                         o.gp_transform == GpTransform::c2c ? QHK_GP_C2C : QHK_GP_R2C,
                         o.tv_weight,
                         o.tv_inner,
                         o.mapping == Mapping::scatter ? QHK_MAPPING_SCATTER : QHK_MAPPING_GATHER};
}

// odt_grid validation (src/api.cpp:107-123); returns nz.
int checked_odt(int n, int count, std::span<const Illumination> il, const Geometry& g, const OdtOptions& o) {
  host::require_even_square(n, n, "reconstruct");
  require(count >= 1 && static_cast<std::size_t>(count) == il.size(), "reconstruct: need one illumination per field");
  require(g.wavelength > 0 && g.pixel > 0 && g.n_medium > 0 && g.na > 0,
          "reconstruct: geometry values must be positive");
  const int nz = o.nz > 0 ? o.nz : n;
  require(nz % 2 == 0, "reconstruct: nz must be even");
  const float fm = g.n_medium / g.wavelength;
  for (const auto& v : il) {
    require(v.fy * v.fy + v.fx * v.fx < fm * fm, "reconstruct: illumination frequency beyond n_medium / wavelength");
  }
  host::require_cuda(o.backend);
  return nz;
}

}  // namespace host

OdtResult reconstruct(const Array3<cfloat>& rytov_fields, std::span<const Illumination> illuminations,
                      const Geometry& geometry, const OdtOptions& options) {
  require(rytov_fields.ny == rytov_fields.nx, "reconstruct: images must be square");
  const int n = rytov_fields.nx;
  const int nz = host::checked_odt(n, rytov_fields.nz, illuminations, geometry, options);
  const qhk_geometry g{geometry.wavelength, geometry.n_medium, geometry.na, geometry.pixel};
  const qhk_odt_options o = host::odt_options(options);
  OdtResult r;
  r.ri = Array3<float>(nz, n, n);
  check(qhk_reconstruct(rytov_fields.data.data(), rytov_fields.nz, n,
                        reinterpret_cast<const float*>(illuminations.data()), &g, &o, r.ri.data.data(), &r.filled));
  return r;
}

std::vector<Illumination> circular_scan(int count, float na_illumination, const Geometry& geometry) {
  require(count >= 1, "circular_scan: count must be positive");
  require(na_illumination >= 0 && na_illumination < geometry.n_medium,
          "circular_scan: na_illumination must be below n_medium");
  std::vector<Illumination> out(count);
  const float f = na_illumination / geometry.wavelength;
  for (int i = 1; i < count; ++i) {
    const float phi =
        2.0f * std::numbers::pi_v<float> * static_cast<float>(i - 1) / static_cast<float>(count - 1);
    out[i] = {f * std::sin(phi), f * std::cos(phi)};
  }
  return out;
}

}  // namespace qoraholo
