// extern "C" entry points of libqhk.so (include/qoraholo_b200.h). Every function validates its
// arguments, converts exceptions into a status code and records the message for qhk_last_error().
#include <cmath>
#include <cstring>
#include <numbers>
#include <string>

#include "../../include/qoraholo_b200.h"
#include "odt.hpp"

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

}  // namespace

struct qhk_odt {
  qhk::OdtPlan plan;
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
    qhk::check(cudaStreamSynchronize(as_stream(stream)), "qhk_odt_filled");
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
    qhk::check(cudaMemcpyAsync(d_fields.get(), fields, nf * sizeof(float2), cudaMemcpyHostToDevice, stream.get()),
               "upload fields");
    plan.run(d_fields.get(), d_index.get(), stream.get());
    qhk::check(cudaMemcpyAsync(out, d_index.get(), plan.volume() * sizeof(float), cudaMemcpyDeviceToHost,
                               stream.get()),
               "download index");
    unsigned long long v = 0;
    qhk::check(cudaMemcpyAsync(&v, plan.filled(), sizeof v, cudaMemcpyDeviceToHost, stream.get()), "download filled");
    qhk::check(cudaStreamSynchronize(stream.get()), "reconstruct");
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
    qhk::DevBuf<float> scratch(6 * v);
    qhk::TvBuffers t;
    for (int c = 0; c < 3; ++c) {
      t.v[0][c] = d_dual + c * v;
      t.v[1][c] = scratch.get() + c * v;
      t.v[2][c] = scratch.get() + (3 + c) * v;
    }
    t.p_index = 0;
    qhk::tv_prox(d_b, t, nz, ny, nx, lambda, inner, qhk::TvFinal::plain, 0.0f, nullptr, d_x, 0, 0, s);
    if (t.p_index != 0) {
      qhk::check(cudaMemcpyAsync(d_dual, t.v[t.p_index][0], 3 * v * sizeof(float), cudaMemcpyDeviceToDevice, s),
                 "copy dual");
    }
    // The scratch buffer is freed on return; wait for the kernels that use it.
    qhk::check(cudaStreamSynchronize(s), "tv_prox");
  });
}

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

}  // extern "C"
