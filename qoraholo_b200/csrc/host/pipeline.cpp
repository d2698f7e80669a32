// qoraholo::Pipeline over the qhk_pipeline handle of the C ABI. Constructor validation as the
// reference's (src/pipeline.cpp:72-91); process() before set_background() is a logic_error.
#include "qoraholo/pipeline.hpp"

#include <algorithm>
#include <chrono>
#include <cmath>

#include "host_common.hpp"

namespace qoraholo {

namespace host {
qhk_odt_options odt_options(const OdtOptions& o);
int checked_odt(int n, int count, std::span<const Illumination> il, const Geometry& g, const OdtOptions& o);
}  // namespace host

class Pipeline::Impl {
 public:
  ~Impl() {
    if (handle) qhk_pipeline_destroy(handle);
  }
  qhk_pipeline* handle = nullptr;
  PipelineTimings timings;
  double filled = 0;
  double setup_ms = 0;
  std::size_t input_size = 0;
  std::array<int, 3> shape{};
  bool has_background = false;
};

Pipeline::Pipeline(PipelineOptions options) : impl_(std::make_unique<Impl>()) {
  const auto t0 = std::chrono::steady_clock::now();
  const int n = options.hologram_size;
  host::require(options.count >= 1, "Pipeline: count must be positive");
  host::require(n >= 4 && n % 2 == 0, "Pipeline: hologram_size must be even");
  host::require(options.field.center.has_value(), "Pipeline: field.center (the carrier) is required");
  host::require(options.upload_chunks >= 1 && options.upload_chunks <= options.count,
                "Pipeline: upload_chunks must be between 1 and count");
  const auto c = *options.field.center;
  const int out = options.field.output_size > 0 ? options.field.output_size : n;
  float radius = options.field.radius > 0 ? options.field.radius : std::hypot(c[0], c[1]) / 3.0f;
  host::require(out % 2 == 0 && out <= n, "extract_fields: output_size must be even and <= N");
  host::require(radius > 0 && radius <= static_cast<float>(out) / 2.0f,
                "extract_fields: crop radius must fit in the output window");
  const int nz = host::checked_odt(out, options.count, options.illuminations, options.geometry, options.odt);
  qhk_pipeline_options o{};
  o.count = options.count;
  o.hologram_size = n;
  o.center_y = c[0];
  o.center_x = c[1];
  o.radius = options.field.radius;
  o.output_size = options.field.output_size;
  o.upload_chunks = options.upload_chunks;
  o.odt = host::odt_options(options.odt);
  const qhk_geometry g{options.geometry.wavelength, options.geometry.n_medium, options.geometry.na,
                       options.geometry.pixel};
  host::check(qhk_pipeline_create(&impl_->handle, &o, reinterpret_cast<const float*>(options.illuminations.data()),
                                  &g));
  impl_->input_size = static_cast<std::size_t>(options.count) * n * n;
  impl_->shape = {nz, out, out};
  impl_->setup_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

Pipeline::~Pipeline() = default;
Pipeline::Pipeline(Pipeline&&) noexcept = default;
Pipeline& Pipeline::operator=(Pipeline&&) noexcept = default;

void Pipeline::set_background(const Array3<float>& backgrounds) {
  host::require(backgrounds.size() == impl_->input_size && backgrounds.ny == backgrounds.nx,
                "Pipeline::set_background: shape must be (count, N, N)");
  host::check(qhk_pipeline_set_background(impl_->handle, backgrounds.data.data()));
  impl_->has_background = true;
}

std::span<float> Pipeline::input() { return {qhk_pipeline_input(impl_->handle), impl_->input_size}; }

void Pipeline::process() {
  if (!impl_->has_background) throw std::logic_error("Pipeline: set_background() first");
  host::check(qhk_pipeline_process(impl_->handle));
  qhk_pipeline_timings t{};
  host::check(qhk_pipeline_result(impl_->handle, &impl_->filled, &t));
  impl_->timings = PipelineTimings{t.upload, t.fields, t.rytov,  t.fft2,     t.clear, t.mapping,
                                   t.normalize, t.solve, t.finish, t.download, t.total};
}

std::span<const float> Pipeline::output() const {
  const auto [nz, ny, nx] = impl_->shape;
  return {qhk_pipeline_output(impl_->handle), static_cast<std::size_t>(nz) * ny * nx};
}

double Pipeline::filled() const { return impl_->filled; }

void Pipeline::run(std::span<const float> holograms, std::span<float> index) {
  const auto [nz, ny, nx] = impl_->shape;
  host::require(holograms.size() == impl_->input_size, "Pipeline::run: shape must be (count, N, N)");
  host::require(index.size() == static_cast<std::size_t>(nz) * ny * nx, "Pipeline::run: output must be (nz, n, n)");
  if (!impl_->has_background) throw std::logic_error("Pipeline: set_background() first");
  host::check(qhk_pipeline_run(impl_->handle, holograms.data(), index.data()));
  qhk_pipeline_timings t{};
  host::check(qhk_pipeline_result(impl_->handle, &impl_->filled, &t));
  impl_->timings = PipelineTimings{t.upload, t.fields, t.rytov,  t.fft2,     t.clear, t.mapping,
                                   t.normalize, t.solve, t.finish, t.download, t.total};
}

void Pipeline::run_stream(std::span<const float> holograms, std::span<float> index, int items) {
  const auto [nz, ny, nx] = impl_->shape;
  const std::size_t volume = static_cast<std::size_t>(nz) * ny * nx;
  host::require(items >= 1 && holograms.size() == items * impl_->input_size,
                "Pipeline::run_stream: shape must be (items, count, N, N)");
  host::require(index.size() == items * volume, "Pipeline::run_stream: output must be (items, nz, n, n)");
  if (!impl_->has_background) throw std::logic_error("Pipeline: set_background() first");
  host::check(qhk_pipeline_run_stream(impl_->handle, holograms.data(), items, index.data()));
  qhk_pipeline_timings t{};
  host::check(qhk_pipeline_result(impl_->handle, &impl_->filled, &t));
  impl_->timings = PipelineTimings{t.upload, t.fields, t.rytov,  t.fft2,     t.clear, t.mapping,
                                   t.normalize, t.solve, t.finish, t.download, t.total};
}

OdtResult Pipeline::run(const Array3<float>& holograms) {
  host::require(holograms.ny == holograms.nx, "Pipeline::run: shape must be (count, N, N)");
  const auto [nz, ny, nx] = impl_->shape;
  OdtResult r{Array3<float>(nz, ny, nx), 0.0};
  run(std::span<const float>(holograms.data), std::span<float>(r.ri.data));
  r.filled = impl_->filled;
  return r;
}

const PipelineTimings& Pipeline::timings() const { return impl_->timings; }
double Pipeline::setup_ms() const { return impl_->setup_ms; }
std::size_t Pipeline::device_bytes() const { return qhk_pipeline_device_bytes(impl_->handle); }
std::array<int, 3> Pipeline::output_shape() const { return impl_->shape; }

}  // namespace qoraholo
