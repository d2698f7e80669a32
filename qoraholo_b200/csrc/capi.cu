// extern "C" entry points of libqhk.so (include/qoraholo_b200.h). Every function validates its
// arguments, converts exceptions into a status code and records the message for qhk_last_error().
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <numbers>
#include <string>

#include "../../include/qoraholo_b200.h"
#include <complex>
#include <deque>
#include <vector>

#include "autotune.hpp"
#include "bpm.hpp"
#include "debug.cuh"
#include "field.hpp"
#include "odt.hpp"
#include "pipeline.hpp"
#include "server.hpp"
#include "synth.hpp"
#include "unwrap.hpp"

namespace {

thread_local std::string g_last_error;

template <class F>
int guard(F&& f) {
  try {
    f();
    return qhk::kOk;
  } catch (const qhk::Error& e) {
    g_last_error = e.what();
    return e.status;
  } catch (const std::bad_alloc& e) {
    g_last_error = e.what();
    return qhk::kOutOfMemory;
  } catch (const std::exception& e) {
    g_last_error = e.what();
    return qhk::kInternal;
  }
}

cudaStream_t as_stream(void* s) { return static_cast<cudaStream_t>(s); }

// Validation of the reconstruct() arguments (src/api.cpp:107-123) and the solver configuration.
qhk::OdtConfig odt_config(int n, int count, const float* il, const qhk_geometry* g, const qhk_odt_options* o) {
  using qhk::require;
  require(g != nullptr && o != nullptr && il != nullptr, "reconstruct: null argument");
  require(n >= 4 && n % 2 == 0, "reconstruct: images must be square with an even side");
  require(count >= 1, "reconstruct: need one illumination per field");
  require(g->wavelength > 0 && g->pixel > 0 && g->n_medium > 0 && g->na > 0,
          "reconstruct: geometry values must be positive");
  const int nz = o->nz > 0 ? o->nz : n;
  require(nz % 2 == 0, "reconstruct: nz must be even");
  const float fm = g->n_medium / g->wavelength;
  for (int a = 0; a < count; ++a) {
    const float fy = il[2 * a], fx = il[2 * a + 1];
    require(fy * fy + fx * fx < fm * fm, "reconstruct: illumination frequency beyond n_medium / wavelength");
  }
  require(o->iterations >= 0, "reconstruct: iterations must be non-negative");
  require(o->solver == QHK_SOLVER_GP || o->solver == QHK_SOLVER_TV, "reconstruct: unknown solver");
  require(o->gp_transform == QHK_GP_R2C || o->gp_transform == QHK_GP_C2C, "reconstruct: unknown gp_transform");
  require(o->mapping == QHK_MAPPING_GATHER || o->mapping == QHK_MAPPING_SCATTER, "reconstruct: unknown mapping");
  const bool tv = o->iterations > 0 && o->solver == QHK_SOLVER_TV;
  require(!tv || (o->tv_inner >= 0 && o->tv_weight > 0), "reconstruct: TV needs tv_weight > 0 and tv_inner >= 0");
  qhk::OdtConfig c;
  c.grid = qhk::make_grid(n, nz, g->wavelength, g->n_medium, g->na, g->pixel);
  c.count = count;
  c.iterations = o->iterations;
  c.tv = tv;
  c.r2c = o->gp_transform == QHK_GP_R2C;
  const float k0 = 2.0f * std::numbers::pi_v<float> / g->wavelength;
  c.lambda = o->tv_weight * k0 * k0;
  c.tv_inner = o->tv_inner;
  c.nm2 = g->n_medium * g->n_medium;
  c.inv_k02 = 1.0f / (k0 * k0);
  return c;
}

// Reads an ODT plan's wait counter after the work queued on `s` (synchronises `s`) and fails with a
// timeout status if a bounded device wait of the plan ran out since `seen`.
void check_plan_waits(const qhk::OdtPlan& plan, unsigned long long& seen, cudaStream_t s, const char* what) {
  unsigned long long n = 0;
  qhk::check(cudaMemcpyAsync(&n, plan.wait_count(), sizeof n, cudaMemcpyDeviceToHost, s), "download wait count");
  qhk::check(cudaStreamSynchronize(s), what);
  if (n != seen) {
    seen = n;
    qhk::fail(qhk::kTimeout, qhk::wait_timeout_message(what));
  }
}

}  // namespace

struct qhk_odt {
  qhk::OdtPlan plan;
  unsigned long long waits_seen = 0;  // the plan's wait counter at the last check
};

struct qhk_pipeline {
  qhk::PipelinePlan plan;
};

extern "C" {

const char* qhk_last_error(void) { return g_last_error.c_str(); }

int qhk_device_present(void) {
  int count = 0;
  return cudaGetDeviceCount(&count) == cudaSuccess && count > 0 ? 1 : 0;
}

int qhk_odt_create(qhk_odt** plan, int n, int count, const float* illum_fyfx, const qhk_geometry* geometry,
                   const qhk_odt_options* options) {
  return guard([&] {
    qhk::require(plan != nullptr, "qhk_odt_create: null plan");
    const qhk::OdtConfig c = odt_config(n, count, illum_fyfx, geometry, options);
    *plan = new qhk_odt{qhk::OdtPlan(c, illum_fyfx)};
  });
}

int qhk_odt_run(qhk_odt* plan, void* d_fields, float* d_index, void* stream) {
  return guard([&] {
    qhk::require(plan && d_fields && d_index, "qhk_odt_run: null argument");
    plan->plan.run(static_cast<float2*>(d_fields), d_index, as_stream(stream));
  });
}

int qhk_odt_filled(qhk_odt* plan, void* stream, double* filled) {
  return guard([&] {
    qhk::require(plan && filled, "qhk_odt_filled: null argument");
    unsigned long long v = 0;
    qhk::check(cudaMemcpyAsync(&v, plan->plan.filled(), sizeof v, cudaMemcpyDeviceToHost, as_stream(stream)),
               "download filled");
    check_plan_waits(plan->plan, plan->waits_seen, as_stream(stream), "qhk_odt_filled");
    *filled = static_cast<double>(v) / static_cast<double>(plan->plan.volume());
  });
}

int qhk_odt_shape(const qhk_odt* plan, int* nz, int* n) {
  return guard([&] {
    qhk::require(plan && nz && n, "qhk_odt_shape: null argument");
    *nz = plan->plan.config().grid.nz;
    *n = plan->plan.config().grid.n;
  });
}

size_t qhk_odt_device_bytes(const qhk_odt* plan) { return plan ? plan->plan.device_bytes() : 0; }

int qhk_odt_destroy(qhk_odt* plan) {
  return guard([&] { delete plan; });
}

int qhk_reconstruct(const void* fields, int count, int n, const float* illum_fyfx, const qhk_geometry* geometry,
                    const qhk_odt_options* options, float* out, double* filled) {
  return guard([&] {
    qhk::require(fields && out, "reconstruct: null argument");
    const qhk::OdtConfig c = odt_config(n, count, illum_fyfx, geometry, options);
    qhk::OdtPlan plan(c, illum_fyfx);
    qhk::Stream stream;
    const std::size_t nf = static_cast<std::size_t>(count) * n * n;
    qhk::DevBuf<float2> d_fields(nf);
    qhk::DevBuf<float> d_index(plan.volume());
    qhk::upload(d_fields.get(), fields, nf * sizeof(float2), stream.get());
    plan.run(d_fields.get(), d_index.get(), stream.get());
    qhk::download(out, d_index.get(), plan.volume() * sizeof(float), stream.get());
    unsigned long long v = 0;
    qhk::check(cudaMemcpyAsync(&v, plan.filled(), sizeof v, cudaMemcpyDeviceToHost, stream.get()), "download filled");
    unsigned long long waits = 0;
    check_plan_waits(plan, waits, stream.get(), "reconstruct");
    if (filled) *filled = static_cast<double>(v) / static_cast<double>(plan.volume());
  });
}

int qhk_ewald_map(const void* d_spectra, int count, int n, int nz, const float* illum_fyfx,
                  const qhk_geometry* geometry, int half, void* d_data, uint8_t* d_hits,
                  unsigned long long* d_filled, void* stream) {
  return guard([&] {
    qhk::require(d_spectra && d_data && d_hits && d_filled, "ewald_map: null argument");
    qhk_odt_options o{nz, 0, QHK_SOLVER_GP, QHK_GP_R2C, 1e-2f, 10, QHK_MAPPING_GATHER};
    const qhk::OdtConfig c = odt_config(n, count, illum_fyfx, geometry, &o);
    const auto table = qhk::illumination_table(c.grid, illum_fyfx, count);
    qhk::DevBuf<float4> il(count);
    const cudaStream_t s = as_stream(stream);
    qhk::check(cudaMemcpyAsync(il.get(), table.data(), count * sizeof(float4), cudaMemcpyHostToDevice, s),
               "upload illuminations");
    const auto* spectra = static_cast<const float2*>(d_spectra);
    if (half) {
      qhk::map_half(spectra, il.get(), count, c.grid, static_cast<float2*>(d_data), d_hits, d_filled, s);
    } else {
      qhk::map_full(spectra, il.get(), count, c.grid, static_cast<float2*>(d_data), nullptr, d_hits, d_filled, s);
    }
    qhk::check(cudaStreamSynchronize(s), "ewald_map");
  });
}

int qhk_tv_prox(const float* d_b, float* d_x, float* d_dual, int nz, int ny, int nx, float lambda, int inner,
                void* stream) {
  return guard([&] {
    qhk::require(d_b && d_x && d_dual, "tv_prox: null argument");
    qhk::require(nz >= 1 && ny >= 1 && nx >= 1 && lambda > 0 && inner >= 0, "tv_prox: invalid arguments");
    const std::size_t v = static_cast<std::size_t>(nz) * ny * nx;
    const cudaStream_t s = as_stream(stream);
    qhk::DevBuf<float> scratch(9 * v);
    qhk::DevBuf<unsigned long long> waits(1);
    qhk::check(cudaMemsetAsync(waits.get(), 0, sizeof(unsigned long long), s), "cudaMemset");
    qhk::TvBuffers t;
    for (int c = 0; c < 3; ++c) {
      t.v[0][c] = d_dual + c * v;
      for (int i = 1; i < 4; ++i) t.v[i][c] = scratch.get() + (3 * (i - 1) + c) * v;
    }
    t.p_index = 0;
    t.wait_status = waits.get();
    qhk::tv_prox(d_b, t, nz, ny, nx, lambda, inner, qhk::TvFinal::plain, 0.0f, nullptr, d_x, 0, 0, s);
    if (t.p_index != 0) {
      qhk::check(cudaMemcpyAsync(d_dual, t.v[t.p_index][0], 3 * v * sizeof(float), cudaMemcpyDeviceToDevice, s),
                 "copy dual");
    }
    // The scratch buffer is freed on return; wait for the kernels that use it.
    unsigned long long n = 0;
    qhk::check(cudaMemcpyAsync(&n, waits.get(), sizeof n, cudaMemcpyDeviceToHost, s), "download wait count");
    qhk::check(cudaStreamSynchronize(s), "tv_prox");
    if (n != 0) qhk::fail(qhk::kTimeout, qhk::wait_timeout_message("tv_prox"));
  });
}

int qhk_tv_prox_device(const float* d_b, float* d_x, float* d_dual, int nz, int ny, int nx, float lambda, int inner,
                       void* stream) {
  return guard([&] {
    qhk::require(d_b && d_x && d_dual, "tv_prox: null argument");
    qhk::require(nz >= 1 && ny >= 1 && nx >= 1 && lambda > 0 && inner >= 0, "tv_prox: invalid arguments");
    const std::size_t v = static_cast<std::size_t>(nz) * ny * nx;
    const cudaStream_t s = as_stream(stream);
    qhk::TvBuffers t;
    for (int i = 0; i < 3; ++i)
      for (int c = 0; c < 3; ++c) t.v[i][c] = d_dual + (3 * i + c) * v;
    t.p_index = 0;
    qhk::tv_prox(d_b, t, nz, ny, nx, lambda, inner, qhk::TvFinal::plain, 0.0f, nullptr, d_x, 0, 0, s);
    if (t.p_index != 0) {
      qhk::check(cudaMemcpyAsync(d_dual, t.v[t.p_index][0], 3 * v * sizeof(float), cudaMemcpyDeviceToDevice, s),
                 "copy dual");
    }
  });
}

int qhk_tv_prox_workspace(const float* d_b, float* d_x, float* d_work, int work_volumes, int nz, int ny, int nx,
                          float lambda, int inner, void* stream) {
  return guard([&] {
    qhk::require(d_b && d_x && d_work, "tv_prox: null argument");
    qhk::require(work_volumes == 9 || work_volumes == 12, "tv_prox: work_volumes must be 9 or 12");
    qhk::require(nz >= 1 && ny >= 1 && nx >= 1 && lambda > 0 && inner >= 0, "tv_prox: invalid arguments");
    const std::size_t v = static_cast<std::size_t>(nz) * ny * nx;
    const cudaStream_t s = as_stream(stream);
    qhk::TvBuffers t;
    for (int i = 0; i < work_volumes / 3; ++i)
      for (int c = 0; c < 3; ++c) t.v[i][c] = d_work + (3 * i + c) * v;
    t.p_index = 0;
    qhk::tv_prox(d_b, t, nz, ny, nx, lambda, inner, qhk::TvFinal::plain, 0.0f, nullptr, d_x, 0, 0, s);
    if (t.p_index != 0) {
      for (int c = 0; c < 3; ++c) {
        qhk::check(cudaMemcpyAsync(d_work + c * v, t.v[t.p_index][c], v * sizeof(float), cudaMemcpyDeviceToDevice, s),
                   "copy dual");
      }
    }
  });
}

int qhk_pinned_alloc(size_t bytes, void** ptr) {
  return guard([&] {
    qhk::require(ptr != nullptr && bytes > 0, "pinned_alloc: null pointer or zero size");
    *ptr = nullptr;
    qhk::check(cudaMallocHost(ptr, bytes), "cudaMallocHost");
  });
}

int qhk_pinned_free(void* ptr) {
  return guard([&] {
    if (ptr) qhk::check(cudaFreeHost(ptr), "cudaFreeHost");
  });
}

int qhk_wait_timeouts(uint64_t* count) {
  return guard([&] {
    qhk::require(count != nullptr, "wait_timeouts: null argument");
    *count = qhk::tv_wait_timeouts();
  });
}

int qhk_debug_enabled(void) { return qhk::debug::enabled() ? 1 : 0; }

int qhk_debug_violations(uint64_t* count, int reset) {
  return guard([&] {
    qhk::require(count != nullptr, "debug_violations: null argument");
    if (qhk::debug::enabled()) qhk::check(cudaDeviceSynchronize(), "debug_violations");
    std::string first;
    *count = qhk::debug::violations(reset != 0, &first);
    g_last_error = first.empty() ? std::string() : "first failed bounds check at " + first;
  });
}

uint64_t qhk_kernel_launches(void) { return qhk::g_launches.load(std::memory_order_relaxed); }

int qhk_fft2d(void* d_data, int count, int n, int forward, float scale, void* stream) {
  return guard([&] {
    qhk::require(d_data && count >= 1 && n >= 1, "fft2d: invalid arguments");
    qhk::fft2d(static_cast<float2*>(d_data), count, n, forward != 0, scale, as_stream(stream));
  });
}

int qhk_rfft3(const float* d_x, void* d_half, int nz, int ny, int nx, void* stream) {
  return guard([&] {
    qhk::require(d_x && d_half && nz >= 1 && ny >= 1 && nx >= 2 && nx % 2 == 0, "rfft3: invalid arguments");
    const int h = nx / 2 + 1;
    const std::size_t nh = static_cast<std::size_t>(ny) * h;
    auto* e = static_cast<float2*>(d_half);
    const cudaStream_t s = as_stream(stream);
    qhk::rows_r2c(d_x, e, static_cast<std::size_t>(nz) * ny, nx, false, s);
    qhk::axis_pass(e, nz, nh, ny, h, h, true, qhk::AxisMode::plain, 1.0f, {}, s);
    qhk::axis_pass(e, ny, h, nz, nh, h, true, qhk::AxisMode::plain, 1.0f, {}, s);
  });
}

int qhk_irfft3(void* d_half, float* d_x, int nz, int ny, int nx, float scale, void* stream) {
  return guard([&] {
    qhk::require(d_x && d_half && nz >= 1 && ny >= 1 && nx >= 2 && nx % 2 == 0, "irfft3: invalid arguments");
    const int h = nx / 2 + 1;
    const std::size_t nh = static_cast<std::size_t>(ny) * h;
    auto* e = static_cast<float2*>(d_half);
    const cudaStream_t s = as_stream(stream);
    qhk::axis_pass(e, ny, h, nz, nh, h, false, qhk::AxisMode::plain, scale, {}, s);
    qhk::axis_pass(e, nz, nh, ny, h, h, false, qhk::AxisMode::plain, 1.0f, {}, s);
    qhk::rows_c2r(e, d_x, static_cast<std::size_t>(nz) * ny, nx, qhk::C2rMode::store, 0, 0, s);
  });
}

int qhk_extract_fields(const float* holo, int count, int n, float cy, float cx, float radius, int output_size,
                       void* out) {
  return guard([&] {
    qhk::require(holo && out, "extract_fields: null argument");
    qhk::require(n >= 4 && n % 2 == 0, "extract_fields: images must be square with an even side");
    qhk::require(count >= 1, "extract_fields: empty stack");
    const qhk::CropPlan crop = qhk::make_crop(n, cy, cx, radius, output_size);
    qhk::FieldPlan plan(crop, count);
    qhk::Stream stream;
    const std::size_t nin = static_cast<std::size_t>(count) * n * n;
    const std::size_t nout = static_cast<std::size_t>(count) * crop.out * crop.out;
    qhk::DevBuf<float> d_holo(nin);
    qhk::DevBuf<float2> d_out(nout);
    qhk::upload(d_holo.get(), holo, nin * sizeof(float), stream.get());
    plan.fields(d_holo.get(), d_out.get(), stream.get());
    qhk::download(out, d_out.get(), nout * sizeof(float2), stream.get());
  });
}

int qhk_field_ratio(const void* sample, int count, int ny, int nx, const void* background, int bcount, void* out) {
  return guard([&] {
    qhk::require(sample && background && out, "field_ratio: null argument");
    qhk::require(count >= 1 && ny >= 1 && nx >= 1 && (bcount == 1 || bcount == count),
                 "field_ratio: background shape does not match");
    qhk::Stream stream;
    const cudaStream_t s = stream.get();
    const std::size_t plane = static_cast<std::size_t>(ny) * nx;
    const std::size_t total = plane * count;
    qhk::DevBuf<float2> ds(total), db(plane * bcount);
    qhk::upload(ds.get(), sample, ds.bytes(), s);
    qhk::upload(db.get(), background, db.bytes(), s);
    qhk::field_ratio(ds.get(), db.get(), plane, bcount == count && count > 1, total, ds.get(), s);
    qhk::download(out, ds.get(), ds.bytes(), s);
  });
}

int qhk_find_sideband(const float* holo, int n, float dc_exclusion, int* iy, int* ix, float* y, float* x,
                      float* magnitude) {
  return guard([&] {
    qhk::require(holo && iy && ix && y && x && magnitude, "find_sideband: null argument");
    qhk::require(n >= 4 && n % 2 == 0, "find_sideband: holograms must be square with an even side");
    if (dc_exclusion <= 0) dc_exclusion = static_cast<float>(n) / 8.0f;
    const int h = n / 2 + 1;
    qhk::Stream stream;
    const cudaStream_t s = stream.get();
    qhk::DevBuf<float> d_holo(static_cast<std::size_t>(n) * n);
    qhk::DevBuf<float2> d_half(static_cast<std::size_t>(n) * h);
    qhk::DevBuf<float> d_mag(1);
    qhk::DevBuf<int> d_idx(1);
    qhk::check(cudaMemcpyAsync(d_holo.get(), holo, d_holo.bytes(), cudaMemcpyHostToDevice, s), "upload hologram");
    qhk::sideband_peak(d_holo.get(), n, dc_exclusion, d_half.get(), d_mag.get(), d_idx.get(), s);
    std::vector<float2> half(static_cast<std::size_t>(n) * h);
    float mag = 0;
    int idx = -1;
    qhk::check(cudaMemcpyAsync(half.data(), d_half.get(), d_half.bytes(), cudaMemcpyDeviceToHost, s), "download");
    qhk::check(cudaMemcpyAsync(&mag, d_mag.get(), sizeof mag, cudaMemcpyDeviceToHost, s), "download");
    qhk::check(cudaMemcpyAsync(&idx, d_idx.get(), sizeof idx, cudaMemcpyDeviceToHost, s), "download");
    qhk::check(cudaStreamSynchronize(s), "find_sideband");
    if (idx < 0 || mag == 0.0f) qhk::fail(qhk::kCudaError, "find_sideband: no peak outside the DC region");
    const int c = n / 2;
    // Centred spectrum S[yy][xx] = H(yy - c, xx - c); H(fy, fx < 0) = conj H(-fy, -fx).
    const auto spec = [&](int yy, int xx) {
      int fy = yy - c, fx = xx - c;
      bool conj = false;
      if (fx < 0) {
        fy = -fy;
        fx = -fx;
        conj = true;
      }
      const float2 v = half[static_cast<std::size_t>((fy % n + n) % n) * h + fx];
      return std::complex<float>(v.x, conj ? -v.y : v.y);
    };
    // Jacobsen's three-bin estimator with Candan's bias correction (src/cpu/field.cpp:15-22).
    const auto refine = [&](std::complex<float> lo, std::complex<float> mid, std::complex<float> hi) {
      const std::complex<float> den = 2.0f * mid - lo - hi;
      if (std::abs(den) == 0.0f) return 0.0f;
      const float cc = std::numbers::pi_v<float> / static_cast<float>(n);
      const float d = ((lo - hi) / den).real() * std::tan(cc) / cc;
      return std::clamp(d, -0.5f, 0.5f);
    };
    const int py = idx / n, px = idx % n;
    *iy = py - c;
    *ix = px - c;
    *y = static_cast<float>(*iy) + refine(spec(py - 1, px), spec(py, px), spec(py + 1, px));
    *x = static_cast<float>(*ix) + refine(spec(py, px - 1), spec(py, px), spec(py, px + 1));
    *magnitude = mag;
  });
}

int qhk_unwrap(const float* wrapped, int count, int ny, int nx, float* out) {
  return guard([&] {
    qhk::require(wrapped && out, "unwrap: null argument");
    qhk::UnwrapPlan plan(count, ny, nx);
    qhk::Stream stream;
    const std::size_t total = static_cast<std::size_t>(count) * ny * nx;
    qhk::DevBuf<float> psi(total), phi(total);
    qhk::upload(psi.get(), wrapped, total * sizeof(float), stream.get());
    plan.unwrap(psi.get(), phi.get(), stream.get());
    qhk::download(out, phi.get(), total * sizeof(float), stream.get());
  });
}

int qhk_unwrap_noalloc(const float* d_wrapped, float* d_unwrapped, int count, int ny, int nx, void* stream) {
  return guard([&] { qhk::unwrap_noalloc(d_wrapped, d_unwrapped, count, ny, nx, as_stream(stream)); });
}

int qhk_rytov(const void* ratio, int count, int ny, int nx, void* out) {
  return guard([&] {
    qhk::require(ratio && out, "rytov: null argument");
    qhk::require(ny >= 4 && nx >= 4, "rytov: image sides must be even");
    qhk::UnwrapPlan plan(count, ny, nx);
    qhk::Stream stream;
    const cudaStream_t s = stream.get();
    const std::size_t total = static_cast<std::size_t>(count) * ny * nx;
    qhk::DevBuf<float2> r(total);
    qhk::DevBuf<float> psi(total), logamp(total), phi(total);
    qhk::upload(r.get(), ratio, total * sizeof(float2), s);
    qhk::split_ratio(r.get(), total, psi.get(), logamp.get(), s);
    plan.rytov(psi.get(), logamp.get(), phi.get(), r.get(), s);
    qhk::download(out, r.get(), total * sizeof(float2), s);
  });
}

int qhk_pipeline_create(qhk_pipeline** pipeline, const qhk_pipeline_options* o, const float* illum_fyfx,
                        const qhk_geometry* geometry) {
  return guard([&] {
    qhk::require(pipeline && o, "Pipeline: null argument");
    const int n = o->hologram_size;
    qhk::require(o->count >= 1, "Pipeline: count must be positive");
    qhk::require(n >= 4 && n % 2 == 0, "Pipeline: hologram_size must be even");
    qhk::require(o->upload_chunks >= 1 && o->upload_chunks <= o->count,
                 "Pipeline: upload_chunks must be between 1 and count");
    const qhk::CropPlan crop = qhk::make_crop(n, o->center_y, o->center_x, o->radius, o->output_size);
    const qhk::OdtConfig c = odt_config(crop.out, o->count, illum_fyfx, geometry, &o->odt);
    *pipeline = new qhk_pipeline{qhk::PipelinePlan(crop, o->count, o->upload_chunks, c, illum_fyfx)};
  });
}

int qhk_pipeline_create_batched(qhk_pipeline** pipeline, const qhk_pipeline_options* o, const float* illum_fyfx,
                                const qhk_geometry* geometry, int batch) {
  return guard([&] {
    qhk::require(pipeline && o, "Pipeline: null argument");
    qhk::require(batch >= 1, "Pipeline: batch must be positive");
    const int n = o->hologram_size;
    qhk::require(o->count >= 1, "Pipeline: count must be positive");
    qhk::require(n >= 4 && n % 2 == 0, "Pipeline: hologram_size must be even");
    const qhk::CropPlan crop = qhk::make_crop(n, o->center_y, o->center_x, o->radius, o->output_size);
    qhk::OdtConfig c = odt_config(crop.out, o->count, illum_fyfx, geometry, &o->odt);
    c.batch = batch;
    qhk::require(o->upload_chunks >= 1 && o->upload_chunks <= o->count * batch,
                 "Pipeline: upload_chunks must be between 1 and count * batch");
    *pipeline = new qhk_pipeline{qhk::PipelinePlan(crop, o->count, o->upload_chunks, c, illum_fyfx)};
  });
}

int qhk_pipeline_process_device_graph(qhk_pipeline* p, const float* d_holo, float* d_index, void* stream) {
  return guard([&] {
    qhk::require(p && d_holo && d_index, "Pipeline: null argument");
    p->plan.process_device_graph(d_holo, d_index, as_stream(stream));
  });
}

int qhk_pipeline_filled_batch(qhk_pipeline* p, void* stream, double* filled) {
  return guard([&] {
    qhk::require(p && filled, "Pipeline: null argument");
    const int b = p->plan.batch();
    std::vector<unsigned long long> v(b);
    qhk::check(cudaMemcpyAsync(v.data(), p->plan.odt().filled(), b * sizeof(unsigned long long),
                               cudaMemcpyDeviceToHost, as_stream(stream)),
               "download filled");
    p->plan.check_device_waits(as_stream(stream));
    for (int i = 0; i < b; ++i) filled[i] = static_cast<double>(v[i]) / static_cast<double>(p->plan.odt().volume());
  });
}

int qhk_pipeline_set_background(qhk_pipeline* p, const float* backgrounds) {
  return guard([&] {
    qhk::require(p && backgrounds, "Pipeline::set_background: null argument");
    p->plan.set_background(backgrounds);
  });
}

float* qhk_pipeline_input(qhk_pipeline* p) { return p ? p->plan.input() : nullptr; }
const float* qhk_pipeline_output(const qhk_pipeline* p) { return p ? p->plan.output() : nullptr; }

int qhk_pipeline_process(qhk_pipeline* p) {
  return guard([&] {
    qhk::require(p != nullptr, "Pipeline: null pipeline");
    p->plan.process();
  });
}

int qhk_pipeline_run(qhk_pipeline* p, const float* holograms, float* index) {
  return guard([&] {
    qhk::require(p && holograms && index, "Pipeline: null argument");
    p->plan.process_host(holograms, index);
  });
}

int qhk_pipeline_run_stream(qhk_pipeline* p, const float* holograms, int items, float* index) {
  return guard([&] {
    qhk::require(p && holograms && index, "Pipeline: null argument");
    p->plan.process_stream(holograms, index, items);
  });
}

int qhk_pipeline_process_device(qhk_pipeline* p, const float* d_holo, float* d_index, void* stream) {
  return guard([&] {
    qhk::require(p && d_holo && d_index, "Pipeline: null argument");
    p->plan.process_device(d_holo, d_index, as_stream(stream));
  });
}

int qhk_pipeline_result(const qhk_pipeline* p, double* filled, qhk_pipeline_timings* t) {
  return guard([&] {
    qhk::require(p != nullptr, "Pipeline: null pipeline");
    if (filled) *filled = p->plan.filled();
    if (t) {
      const qhk::PipelineTimes& v = p->plan.timings();
      *t = qhk_pipeline_timings{v.upload, v.fields, v.rytov,  v.fft2,     v.clear, v.mapping,
                                v.normalize, v.solve, v.finish, v.download, v.total};
    }
  });
}

int qhk_pipeline_filled(qhk_pipeline* p, void* stream, double* filled) {
  return guard([&] {
    qhk::require(p && filled, "Pipeline: null argument");
    unsigned long long v = 0;
    qhk::check(cudaMemcpyAsync(&v, p->plan.odt().filled(), sizeof v, cudaMemcpyDeviceToHost, as_stream(stream)),
               "download filled");
    p->plan.check_device_waits(as_stream(stream));
    *filled = static_cast<double>(v) / static_cast<double>(p->plan.odt().volume());
  });
}

int qhk_pipeline_check_waits(qhk_pipeline* p, void* stream) {
  return guard([&] {
    qhk::require(p != nullptr, "Pipeline: null pipeline");
    p->plan.check_device_waits(as_stream(stream));
  });
}

int qhk_pipeline_time_prox(qhk_pipeline* p, int enable) {
  return guard([&] {
    qhk::require(p != nullptr, "Pipeline: null pipeline");
    p->plan.odt().enable_prox_timing(enable != 0);
  });
}

int qhk_pipeline_prox_time(qhk_pipeline* p, double* ms, uint64_t* launches) {
  return guard([&] {
    qhk::require(p && ms && launches, "Pipeline: null argument");
    const auto [t, n] = p->plan.odt().prox_timing();
    *ms = t;
    *launches = n;
  });
}

int qhk_pipeline_wait_probe(qhk_pipeline* p, int polls) {
  return guard([&] {
    qhk::require(p != nullptr, "Pipeline: null pipeline");
    p->plan.wait_probe(polls);
  });
}

int qhk_pipeline_shape(const qhk_pipeline* p, int* nz, int* ny, int* nx) {
  return guard([&] {
    qhk::require(p && nz && ny && nx, "Pipeline: null argument");
    *nz = p->plan.odt().config().grid.nz;
    *ny = *nx = p->plan.odt().config().grid.n;
  });
}

size_t qhk_pipeline_device_bytes(const qhk_pipeline* p) { return p ? p->plan.device_bytes() : 0; }

int qhk_pipeline_destroy(qhk_pipeline* p) {
  return guard([&] { delete p; });
}

int qhk_fft2d_host(void* data, int count, int n, int forward, float scale) {
  return guard([&] {
    qhk::require(data && count >= 1 && n >= 1, "fft2d: invalid arguments");
    qhk::Stream stream;
    const std::size_t total = static_cast<std::size_t>(count) * n * n;
    qhk::DevBuf<float2> d(total);
    qhk::check(cudaMemcpyAsync(d.get(), data, total * sizeof(float2), cudaMemcpyHostToDevice, stream.get()), "upload");
    qhk::fft2d(d.get(), count, n, forward != 0, scale, stream.get());
    qhk::check(cudaMemcpyAsync(data, d.get(), total * sizeof(float2), cudaMemcpyDeviceToHost, stream.get()),
               "download");
    qhk::check(cudaStreamSynchronize(stream.get()), "fft2d");
  });
}

namespace {

qhk::BpmTablesHost checked_tables(int nz, int n, int count, const float* il, const qhk_geometry* g, bool obliquity) {
  qhk::require(il && g, "bpm: null argument");
  qhk::require(n >= 4 && n % 2 == 0 && nz >= 1, "bpm: volume must be (nz, n, n) with an even n");
  qhk::require(count >= 1, "bpm: need one illumination per field");
  qhk::require(g->wavelength > 0 && g->pixel > 0 && g->n_medium > 0 && g->na > 0, "bpm: geometry values must be positive");
  const float fm = g->n_medium / g->wavelength;
  for (int a = 0; a < count; ++a) {
    qhk::require(il[2 * a] * il[2 * a] + il[2 * a + 1] * il[2 * a + 1] < fm * fm,
                 "bpm: illumination frequency beyond n_medium / wavelength");
  }
  return qhk::bpm_tables(n, nz, il, count, g->wavelength, g->n_medium, g->na, g->pixel, obliquity);
}

}  // namespace

int qhk_bpm_forward(const float* ri, int nz, int n, const float* illum_fyfx, int count, const qhk_geometry* geometry,
                    int obliquity, void* out) {
  return guard([&] {
    qhk::require(ri && out, "bpm_forward: null argument");
    const auto t = checked_tables(nz, n, count, illum_fyfx, geometry, obliquity != 0);
    qhk::Stream stream;
    const cudaStream_t s = stream.get();
    const std::size_t vol = static_cast<std::size_t>(nz) * n * n;
    qhk::DevBuf<float> d_ri(vol), d_x(vol);
    qhk::check(cudaMemcpyAsync(d_ri.get(), ri, vol * sizeof(float), cudaMemcpyHostToDevice, s), "upload volume");
    qhk::contrast(d_ri.get(), geometry->n_medium, vol, d_x.get(), false, s);
    qhk::BpmPlan plan(t, count, false);
    plan.forward(d_x.get(), 0, count, s);
    qhk::check(cudaMemcpyAsync(out, plan.fields(), static_cast<std::size_t>(count) * n * n * sizeof(float2),
                               cudaMemcpyDeviceToHost, s),
               "download fields");
    qhk::check(cudaStreamSynchronize(s), "bpm_forward");
  });
}

int qhk_bpm_vjp(const float* x, int nz, int n, const void* r, const float* illum_fyfx, int count,
                const qhk_geometry* geometry, int obliquity, float* out) {
  return guard([&] {
    qhk::require(x && r && out, "bpm_vjp: null argument");
    const auto t = checked_tables(nz, n, count, illum_fyfx, geometry, obliquity != 0);
    qhk::Stream stream;
    const cudaStream_t s = stream.get();
    const std::size_t vol = static_cast<std::size_t>(nz) * n * n;
    const std::size_t nf = static_cast<std::size_t>(count) * n * n;
    qhk::DevBuf<float> d_x(vol), d_grad(vol);
    qhk::DevBuf<float2> d_r(nf);
    qhk::check(cudaMemcpyAsync(d_x.get(), x, vol * sizeof(float), cudaMemcpyHostToDevice, s), "upload volume");
    qhk::check(cudaMemcpyAsync(d_r.get(), r, nf * sizeof(float2), cudaMemcpyHostToDevice, s), "upload residual");
    qhk::check(cudaMemsetAsync(d_grad.get(), 0, vol * sizeof(float), s), "cudaMemset");
    qhk::BpmPlan plan(t, count, true);
    plan.forward(d_x.get(), 0, count, s);
    plan.adjoint(d_x.get(), d_r.get(), 0, count, 1.0f, d_grad.get(), s);
    qhk::check(cudaMemcpyAsync(out, d_grad.get(), vol * sizeof(float), cudaMemcpyDeviceToHost, s), "download");
    qhk::check(cudaStreamSynchronize(s), "bpm_vjp");
  });
}

struct qhk_bpm_plan {
  qhk::BpmTablesHost tables;
  float n_medium = 0;
  int chunk = 0;
  qhk::DevBuf<float> x;
  std::unique_ptr<qhk::BpmPlan> plan;
};

int qhk_bpm_plan_create(qhk_bpm_plan** plan, int nz, int n, const float* illum_fyfx, int count,
                        const qhk_geometry* geometry, int obliquity, int chunk, int checkpoint_every) {
  return guard([&] {
    qhk::require(plan != nullptr, "bpm: null argument");
    qhk::require(chunk >= 0 && checkpoint_every >= 0, "bpm: chunk and checkpoint_every must be non-negative");
    auto p = std::make_unique<qhk_bpm_plan>();
    p->tables = checked_tables(nz, n, count, illum_fyfx, geometry, obliquity != 0);
    p->n_medium = geometry->n_medium;
    p->chunk = chunk > 0 ? std::min(chunk, count) : count;
    p->x.reset(static_cast<std::size_t>(nz) * n * n);
    p->plan = std::make_unique<qhk::BpmPlan>(p->tables, p->chunk, checkpoint_every == 0, checkpoint_every);
    *plan = p.release();
  });
}

int qhk_bpm_plan_forward(qhk_bpm_plan* p, const float* d_ri, void* d_fields, void* stream) {
  return guard([&] {
    qhk::require(p && d_ri && d_fields, "bpm: null argument");
    qhk::require(p->plan->checkpoint_every() > 0 || p->chunk == p->tables.count,
                 "bpm: without checkpoints the plan must take all illuminations in one chunk");
    const cudaStream_t s = as_stream(stream);
    const auto& t = p->tables;
    const std::size_t plane = static_cast<std::size_t>(t.n) * t.n;
    qhk::contrast(d_ri, p->n_medium, plane * t.nz, p->x.get(), false, s);
    for (int first = 0; first < t.count; first += p->chunk) {
      const int nb = std::min(p->chunk, t.count - first);
      p->plan->forward(p->x.get(), first, nb, s);
      qhk::check(cudaMemcpyAsync(static_cast<float2*>(d_fields) + first * plane, p->plan->fields(),
                                 nb * plane * sizeof(float2), cudaMemcpyDeviceToDevice, s),
                 "bpm fields");
    }
  });
}

int qhk_bpm_plan_vjp(qhk_bpm_plan* p, const float* d_ri, const void* d_grad_fields, float* d_grad_ri, void* stream) {
  return guard([&] {
    qhk::require(p && d_ri && d_grad_fields && d_grad_ri, "bpm: null argument");
    const cudaStream_t s = as_stream(stream);
    const auto& t = p->tables;
    const std::size_t plane = static_cast<std::size_t>(t.n) * t.n;
    const std::size_t vol = plane * t.nz;
    qhk::contrast(d_ri, p->n_medium, vol, p->x.get(), false, s);
    qhk::check(cudaMemsetAsync(d_grad_ri, 0, vol * sizeof(float), s), "cudaMemset");
    const auto* g = static_cast<const float2*>(d_grad_fields);
    for (int first = 0; first < t.count; first += p->chunk) {
      const int nb = std::min(p->chunk, t.count - first);
      if (p->plan->checkpoint_every() == 0) p->plan->forward(p->x.get(), first, nb, s);  // envelopes of this chunk
      p->plan->adjoint(p->x.get(), g + first * plane, first, nb, 1.0f, d_grad_ri, s);
    }
  });
}

size_t qhk_bpm_plan_device_bytes(const qhk_bpm_plan* p) { return p ? p->plan->device_bytes() + p->x.bytes() : 0; }

int qhk_bpm_plan_destroy(qhk_bpm_plan* p) {
  return guard([&] { delete p; });
}

int qhk_bpm_reconstruct(const void* fields, int count, int n, const float* illum_fyfx, const qhk_geometry* geometry,
                        const float* initial, int nz, const qhk_bpm_solve_options* o, float* out, double* loss) {
  return guard([&] {
    qhk::require(fields && initial && out && o, "bpm_reconstruct: null argument");
    qhk::require(o->iterations >= 0 && o->step > 0 && o->tv_weight >= 0 && o->tv_inner >= 1,
                 "bpm_reconstruct: invalid solver options");
    qhk::require(o->iterations == 0 || loss != nullptr, "bpm_reconstruct: null loss");
    const auto t = checked_tables(nz, n, count, illum_fyfx, geometry, o->obliquity != 0);
    qhk::Stream stream;
    const cudaStream_t s = stream.get();
    const std::size_t vol = static_cast<std::size_t>(nz) * n * n;
    const std::size_t nf = static_cast<std::size_t>(count) * n * n;
    qhk::DevBuf<float> d_ri(vol), d_x(vol);
    qhk::DevBuf<float2> d_f(nf);
    qhk::DevBuf<double> d_loss(std::max(o->iterations, 1));
    qhk::DevBuf<unsigned long long> d_waits(1);
    qhk::check(cudaMemsetAsync(d_waits.get(), 0, sizeof(unsigned long long), s), "cudaMemset");
    qhk::check(cudaMemcpyAsync(d_ri.get(), initial, vol * sizeof(float), cudaMemcpyHostToDevice, s), "upload");
    qhk::check(cudaMemcpyAsync(d_f.get(), fields, nf * sizeof(float2), cudaMemcpyHostToDevice, s), "upload");
    qhk::check(cudaMemsetAsync(d_loss.get(), 0, d_loss.bytes(), s), "cudaMemset");
    qhk::contrast(d_ri.get(), geometry->n_medium, vol, d_x.get(), true, s);
    qhk::bpm_solve(t, d_f.get(), d_x.get(), o->iterations, o->batch, o->step, o->tv_weight, o->tv_inner, d_loss.get(),
                   s, d_waits.get());
    qhk::add_medium(d_x.get(), geometry->n_medium, vol, d_ri.get(), s);
    qhk::check(cudaMemcpyAsync(out, d_ri.get(), vol * sizeof(float), cudaMemcpyDeviceToHost, s), "download");
    if (o->iterations > 0) {
      qhk::check(cudaMemcpyAsync(loss, d_loss.get(), o->iterations * sizeof(double), cudaMemcpyDeviceToHost, s),
                 "download loss");
    }
    unsigned long long waits = 0;
    qhk::check(cudaMemcpyAsync(&waits, d_waits.get(), sizeof waits, cudaMemcpyDeviceToHost, s), "download wait count");
    qhk::check(cudaStreamSynchronize(s), "bpm_reconstruct");
    if (waits != 0) qhk::fail(qhk::kTimeout, qhk::wait_timeout_message("bpm_reconstruct"));
    for (int i = 0; i < o->iterations; ++i) loss[i] *= 0.5 / count;
  });
}


int qhk_tv_form(int form) {
  return guard([&] { qhk::set_tv_form(form); });
}

int qhk_autotune_enable(int enabled) {
  return guard([&] { qhk::set_autotune_enabled(enabled != 0); });
}

int qhk_autotune_radix(int enabled) {
  return guard([&] { qhk::set_radix_tuning(enabled != 0); });
}

int qhk_selftest_rcp_sqrt(uint64_t* mismatches, uint32_t* first_bad) {
  return guard([&] {
    qhk::require(mismatches && first_bad, "selftest_rcp_sqrt: null argument");
    unsigned long long n = 0;
    unsigned b = 0;
    qhk::selftest_rcp_sqrt(&n, &b);
    *mismatches = n;
    *first_bad = b;
  });
}

int qhk_fft_axis_engine(int engine) {
  return guard([&] {
    qhk::require(engine >= -1 && engine <= 2, "fft_axis_engine: -1, 0, 1 or 2");
    qhk::force_axis_engine(engine);
  });
}

size_t qhk_autotune_report(char* buf, size_t size) {
  const std::string r = qhk::autotune_report();
  if (buf && size > 0) {
    const std::size_t n = std::min(size - 1, r.size());
    std::memcpy(buf, r.data(), n);
    buf[n] = '\0';
  }
  return r.size();
}

struct qhk_unwrap_batch {
  qhk::UnwrapBatchPlan plan;
};

int qhk_unwrap_batch_create(qhk_unwrap_batch** plan, const int* ny, const int* nx, int count) {
  return guard([&] {
    qhk::require(plan != nullptr, "unwrap batch: null argument");
    *plan = new qhk_unwrap_batch{qhk::UnwrapBatchPlan(ny, nx, count)};
  });
}

size_t qhk_unwrap_batch_offset(const qhk_unwrap_batch* p, int image) {
  return p && image >= 0 && image < p->plan.count() ? p->plan.offset(image) : 0;
}

size_t qhk_unwrap_batch_total(const qhk_unwrap_batch* p) { return p ? p->plan.total() : 0; }

int qhk_unwrap_batch_run(qhk_unwrap_batch* p, const float* d_wrapped, float* d_unwrapped, int use_graph,
                         void* stream) {
  return guard([&] {
    qhk::require(p && d_wrapped && d_unwrapped, "unwrap batch: null argument");
    if (use_graph) {
      p->plan.unwrap_graph(d_wrapped, d_unwrapped, as_stream(stream));
    } else {
      p->plan.unwrap(d_wrapped, d_unwrapped, as_stream(stream));
    }
  });
}

size_t qhk_unwrap_batch_device_bytes(const qhk_unwrap_batch* p) { return p ? p->plan.device_bytes() : 0; }

int qhk_unwrap_batch_destroy(qhk_unwrap_batch* p) {
  return guard([&] { delete p; });
}

int qhk_synthesize_holograms_device(const void* d_ratio, int count, int n, const float* illum_fyfx, double pixel,
                                    double carrier_y, double carrier_x, double amplitude, float noise, uint64_t seed,
                                    float* d_out, void* stream) {
  return guard([&] {
    qhk::synthesize_holograms_device(static_cast<const float2*>(d_ratio), illum_fyfx, count, n, pixel, carrier_y,
                                     carrier_x, amplitude, noise, seed, d_out, as_stream(stream));
  });
}

int qhk_render_phantom(const float* spheres, int k, const qhk_geometry* geometry, int nz, int n, float* out) {
  return guard([&] {
    qhk::require(geometry && out, "render_phantom: null argument");
    qhk::require(nz >= 1 && n >= 1, "render_phantom: empty shape");
    qhk::Stream stream;
    const std::size_t total = static_cast<std::size_t>(nz) * n * n;
    qhk::DevBuf<float> d(total);
    qhk::render_spheres_device(spheres, k, geometry->n_medium, geometry->pixel, nz, n, d.get(), stream.get());
    qhk::download(out, d.get(), total * sizeof(float), stream.get());
    qhk::check(cudaStreamSynchronize(stream.get()), "render_phantom");
  });
}

int qhk_forward_fields(const float* spheres, int k, const float* illum_fyfx, int count, const qhk_geometry* geometry,
                       int n, int model, void* out) {
  return guard([&] {
    qhk::require(geometry && out, "forward_fields: null argument");
    qhk::Stream stream;
    const std::size_t total = static_cast<std::size_t>(std::max(count, 0)) * n * n;
    qhk::DevBuf<float2> d(std::max<std::size_t>(total, 1));
    qhk::sphere_fields_device(spheres, k, illum_fyfx, count, geometry->wavelength, geometry->n_medium, geometry->na,
                              geometry->pixel, n, model, d.get(), stream.get());
    qhk::download(out, d.get(), total * sizeof(float2), stream.get());
    qhk::check(cudaStreamSynchronize(stream.get()), "forward_fields");
  });
}

struct qhk_server {
  qhk::Server server;
};

int qhk_server_create(qhk_server** server, size_t hbm_budget_bytes, int max_inflight, int use_graphs) {
  return guard([&] {
    qhk::require(server != nullptr, "Server: null argument");
    // QHK_SERVER_STAGERS: host threads that stage pageable inputs and outputs (default 2).
    const char* e = std::getenv("QHK_SERVER_STAGERS");
    const int stagers = e && std::atoi(e) > 0 ? std::atoi(e) : 2;
    *server = new qhk_server{qhk::Server(hbm_budget_bytes, max_inflight, use_graphs != 0, stagers)};
  });
}

int qhk_server_add_geometry(qhk_server* sv, const qhk_pipeline_options* o, const float* illum_fyfx,
                            const qhk_geometry* geometry, const float* backgrounds, int* geometry_id) {
  return guard([&] {
    qhk::require(sv && o && backgrounds && geometry_id, "Server: null argument");
    const int n = o->hologram_size;
    qhk::require(o->count >= 1, "Server: count must be positive");
    qhk::require(n >= 4 && n % 2 == 0, "Server: hologram_size must be even");
    const qhk::CropPlan crop = qhk::make_crop(n, o->center_y, o->center_x, o->radius, o->output_size);
    const qhk::OdtConfig c = odt_config(crop.out, o->count, illum_fyfx, geometry, &o->odt);
    *geometry_id = sv->server.add_geometry(crop, o->count, c, illum_fyfx, backgrounds);
  });
}

int qhk_server_remove_geometry(qhk_server* sv, int geometry_id) {
  return guard([&] {
    qhk::require(sv != nullptr, "Server: null server");
    sv->server.remove_geometry(geometry_id);
  });
}

int qhk_server_volume_shape(qhk_server* sv, int geometry_id, int* nz, int* n) {
  return guard([&] {
    qhk::require(sv && nz && n, "Server: null argument");
    sv->server.volume_shape(geometry_id, nz, n);
  });
}

int qhk_server_submit(qhk_server* sv, int geometry_id, const float* holograms, float* index_out, uint64_t* ticket) {
  return guard([&] {
    qhk::require(sv && ticket, "Server: null argument");
    *ticket = sv->server.submit(geometry_id, holograms, index_out);
  });
}

int qhk_server_done(qhk_server* sv, uint64_t ticket, int* done) {
  return guard([&] {
    qhk::require(sv && done, "Server: null argument");
    *done = sv->server.done(ticket) ? 1 : 0;
  });
}

int qhk_server_cancel(qhk_server* sv, uint64_t ticket, int* cancelled) {
  return guard([&] {
    qhk::require(sv && cancelled, "Server: null argument");
    *cancelled = sv->server.cancel(ticket) ? 1 : 0;
  });
}

int qhk_server_wait(qhk_server* sv, uint64_t ticket, double* filled, qhk_request_times* times) {
  return guard([&] {
    qhk::require(sv != nullptr, "Server: null server");
    qhk::RequestTimes t;
    sv->server.wait(ticket, filled, &t);
    if (times) *times = qhk_request_times{t.queue, t.service, t.total, t.gpu};
  });
}

int qhk_server_stats(qhk_server* sv, qhk_server_counters* out) {
  return guard([&] {
    qhk::require(sv && out, "Server: null argument");
    const qhk::ServerStats s = sv->server.stats();
    *out = qhk_server_counters{s.submitted,          s.completed,      s.failed,         s.cancelled,
                               s.workspaces_created, s.workspaces_evicted, s.graph_launches, s.passed_over,
                               s.budget,             s.used,           s.peak_used,      s.geometries,
                               s.inflight,           s.peak_inflight};
  });
}

int qhk_server_destroy(qhk_server* sv) {
  return guard([&] { delete sv; });
}

int qhk_admission_simulate(size_t budget, int max_inflight, int max_pass, int n_geometries, const size_t* resident,
                           const size_t* workspace, const int* ops, int n_ops, int* admitted, int* action,
                           size_t* used, int* n_admitted) {
  return guard([&] {
    qhk::require(n_geometries >= 1 && resident && workspace && n_admitted && (n_ops == 0 || ops),
                 "admission: null argument");
    qhk::require(n_ops == 0 || (admitted && action && used), "admission: null output");
    qhk::Admission a(budget, max_inflight, max_pass);
    int next_ws = 0;
    for (int g = 0; g < n_geometries; ++g) {
      qhk::require(a.add_geometry(resident[g], workspace[g]) == g, "admission: geometry does not fit the budget");
      (void)a.make_room(workspace[g]);
      a.add_idle(g, next_ws++);
    }
    std::deque<std::pair<int, int>> pending;  // (submission index, geometry)
    std::deque<int> running;                  // workspaces, oldest first
    int submitted = 0, count = 0;
    for (int k = 0; k < n_ops; ++k) {
      if (ops[k] >= 0) {
        qhk::require(ops[k] < n_geometries, "admission: unknown geometry in ops");
        pending.emplace_back(submitted++, ops[k]);
      } else if (!running.empty()) {
        a.release(running.front());
        running.pop_front();
      }
      for (;;) {
        std::vector<int> order;
        for (const auto& p : pending) order.push_back(p.second);
        const auto d = a.choose(order);
        if (!d) break;
        const int wid = d->action == qhk::Admission::Action::reuse ? d->workspace : next_ws++;
        a.commit(*d, wid);
        qhk::require(count < n_ops, "admission: more admissions than ops");
        admitted[count] = pending[d->position].first;
        action[count] = d->action == qhk::Admission::Action::reuse ? 0 : (d->evict.empty() ? 1 : 2);
        used[count] = a.used();
        ++count;
        pending.erase(pending.begin() + static_cast<std::ptrdiff_t>(d->position));
        running.push_back(wid);
      }
    }
    *n_admitted = count;
  });
}

}  // extern "C"
