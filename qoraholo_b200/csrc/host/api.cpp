// Free functions of the public C++ API (include/qoraholo/*.hpp) over the C ABI of libqhk.so.
// Argument validation follows the reference's dispatch layer (src/api.cpp:13-137) so that the
// same calls raise the same exception types; the computation runs on the device.
#include <cmath>
#include <numbers>
#include <string>

#include "host_common.hpp"
#include "raw.hpp"
#include "qoraholo/qoraholo.hpp"

namespace qoraholo {

using host::check;
using host::require;

bool cuda_available() { return qhk_device_present() != 0; }

namespace raw {

Sideband find_sideband(const float* holograms, int count, int ny, int nx, float dc_exclusion) {
  const int n = nx;
  require(count >= 1 && n == ny && n % 2 == 0 && n >= 4, "find_sideband: holograms must be square with an even side");
  host::require_cuda(Backend::cuda);
  Sideband s;
  check(qhk_find_sideband(holograms, n, dc_exclusion, &s.iy, &s.ix, &s.y, &s.x, &s.magnitude));
  return s;
}

}  // namespace raw

Sideband find_sideband(const Array3<float>& holograms, float dc_exclusion) {
  return raw::find_sideband(holograms.data.data(), holograms.nz, holograms.ny, holograms.nx, dc_exclusion);
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

namespace raw {

FieldCall extract_fields_check(const float* holograms, int count, int ny, int nx, const FieldOptions& options,
                               Backend backend) {
  host::require_even_square(ny, nx, "extract_fields");
  require(count >= 1, "extract_fields: empty stack");
  host::require_cuda(backend);
  FieldCall call;
  if (options.center) {
    call.center = *options.center;
  } else {
    const Sideband s = find_sideband(holograms, count, ny, nx, options.dc_exclusion);
    call.center = {static_cast<float>(s.iy), static_cast<float>(s.ix)};
  }
  call.out = checked_output(options, call.center, nx);
  return call;
}

void extract_fields_run(const float* holograms, int count, int n, const FieldOptions& options, const FieldCall& call,
                        cfloat* out) {
  check(qhk_extract_fields(holograms, count, n, call.center[0], call.center[1], options.radius, options.output_size,
                           out));
}

void field_ratio_check(int count, int ny, int nx, int bcount, int bny, int bnx) {
  if (ny != bny || nx != bnx || (bcount != 1 && bcount != count)) {
    throw std::invalid_argument("field_ratio: background shape does not match");
  }
  host::require_cuda(Backend::cuda);
}

void field_ratio_run(const cfloat* sample, int count, int ny, int nx, const cfloat* background, int bcount,
                     cfloat* out) {
  if (static_cast<std::size_t>(count) * ny * nx == 0) return;
  check(qhk_field_ratio(sample, count, ny, nx, background, bcount, out));
}

void unwrap_check(int ny, int nx, Backend backend) {
  require(ny % 2 == 0 && nx % 2 == 0 && ny >= 2 && nx >= 2, "unwrap: image sides must be even");
  host::require_cuda(backend);
}

void unwrap_run(const float* wrapped, int count, int ny, int nx, float* out) {
  if (count == 0) return;
  check(qhk_unwrap(wrapped, count, ny, nx, out));
}

void rytov_check(int ny, int nx, Backend backend) {
  require(ny % 2 == 0 && nx % 2 == 0 && ny >= 4 && nx >= 4, "rytov: image sides must be even");
  host::require_cuda(backend);
}

void rytov_run(const cfloat* ratio, int count, int ny, int nx, cfloat* out) {
  if (count == 0) return;
  check(qhk_rytov(ratio, count, ny, nx, out));
}

}  // namespace raw

Array3<cfloat> extract_fields(const Array3<float>& holograms, const FieldOptions& options, Backend backend) {
  const raw::FieldCall call =
      raw::extract_fields_check(holograms.data.data(), holograms.nz, holograms.ny, holograms.nx, options, backend);
  Array3<cfloat> out(holograms.nz, call.out, call.out);
  raw::extract_fields_run(holograms.data.data(), holograms.nz, holograms.nx, options, call, out.data.data());
  return out;
}

Array3<cfloat> field_ratio(const Array3<cfloat>& sample, const Array3<cfloat>& background) {
  raw::field_ratio_check(sample.nz, sample.ny, sample.nx, background.nz, background.ny, background.nx);
  Array3<cfloat> out(sample.nz, sample.ny, sample.nx);
  raw::field_ratio_run(sample.data.data(), sample.nz, sample.ny, sample.nx, background.data.data(), background.nz,
                       out.data.data());
  return out;
}

Array3<float> unwrap(const Array3<float>& wrapped, Backend backend) {
  raw::unwrap_check(wrapped.ny, wrapped.nx, backend);
  Array3<float> out(wrapped.nz, wrapped.ny, wrapped.nx);
  raw::unwrap_run(wrapped.data.data(), wrapped.nz, wrapped.ny, wrapped.nx, out.data.data());
  return out;
}

Array3<cfloat> rytov(const Array3<cfloat>& ratio, Backend backend) {
  raw::rytov_check(ratio.ny, ratio.nx, backend);
  Array3<cfloat> out(ratio.nz, ratio.ny, ratio.nx);
  raw::rytov_run(ratio.data.data(), ratio.nz, ratio.ny, ratio.nx, out.data.data());
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

namespace raw {

int reconstruct_check(int count, int ny, int nx, std::span<const Illumination> illuminations, const Geometry& geometry,
                      const OdtOptions& options) {
  require(ny == nx, "reconstruct: images must be square");
  return host::checked_odt(nx, count, illuminations, geometry, options);
}

double reconstruct_run(const cfloat* fields, int count, int n, std::span<const Illumination> illuminations,
                       const Geometry& geometry, const OdtOptions& options, float* out) {
  const qhk_geometry g{geometry.wavelength, geometry.n_medium, geometry.na, geometry.pixel};
  const qhk_odt_options o = host::odt_options(options);
  double filled = 0;
  check(qhk_reconstruct(fields, count, n, reinterpret_cast<const float*>(illuminations.data()), &g, &o, out, &filled));
  return filled;
}

}  // namespace raw

OdtResult reconstruct(const Array3<cfloat>& rytov_fields, std::span<const Illumination> illuminations,
                      const Geometry& geometry, const OdtOptions& options) {
  const int nz =
      raw::reconstruct_check(rytov_fields.nz, rytov_fields.ny, rytov_fields.nx, illuminations, geometry, options);
  const int n = rytov_fields.nx;
  OdtResult r;
  r.ri = Array3<float>(nz, n, n);
  r.filled = raw::reconstruct_run(rytov_fields.data.data(), rytov_fields.nz, n, illuminations, geometry, options,
                                  r.ri.data.data());
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
