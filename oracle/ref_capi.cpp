// Test infrastructure only. A flat C interface over the reference's own C++ API (its public
// headers include/qoraholo/*.hpp and the CPU backend in src/cpu/*.cpp), compiled together with the
// reference sources into oracle/_ref/libqhref.so by oracle/build_ref.py. The tests and the CPU
// baseline call it through ctypes (oracle/refimpl.py) to pin the numpy restatement and the CUDA
// path against the reference itself. Nothing in the product links it.
//
// Arrays are dense row-major float32 / interleaved complex64. Every function returns 0 or an
// error class: 1 invalid_argument, 2 runtime_error, 3 logic_error, 4 other; the message is
// available from ref_last_error().

#include <algorithm>
#include <chrono>
#include <complex>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "backends.hpp"
#include "cpu/fft.hpp"
#include "cpu/tv.hpp"
#include "pocketfft_hdronly.h"
#include "qoraholo/qoraholo.hpp"

using namespace qoraholo;

namespace {

thread_local std::string g_error;

template <class F>
int guard(F&& f) {
  try {
    f();
    return 0;
  } catch (const std::invalid_argument& e) {
    g_error = e.what();
    return 1;
  } catch (const std::logic_error& e) {
    g_error = e.what();
    return 3;
  } catch (const std::runtime_error& e) {
    g_error = e.what();
    return 2;
  } catch (const std::exception& e) {
    g_error = e.what();
    return 4;
  }
}

Geometry geometry(const float* g) { return Geometry{g[0], g[1], g[2], g[3]}; }

std::vector<Illumination> illum(const float* il, int count) {
  std::vector<Illumination> out(count);
  for (int i = 0; i < count; ++i) out[i] = {il[2 * i], il[2 * i + 1]};
  return out;
}

template <class T>
Array3<T> load(const void* p, int nz, int ny, int nx) {
  Array3<T> a(nz, ny, nx);
  std::memcpy(a.data.data(), p, a.size() * sizeof(T));
  return a;
}

template <class T>
void store(const Array3<T>& a, void* p) {
  std::memcpy(p, a.data.data(), a.size() * sizeof(T));
}

std::vector<Sphere> spheres(const float* s, int k) {
  std::vector<Sphere> out(k);
  for (int i = 0; i < k; ++i) out[i] = {s[5 * i], s[5 * i + 1], s[5 * i + 2], s[5 * i + 3], s[5 * i + 4]};
  return out;
}

// Backend of the ODT options built below: the CPU one, or the reference's CUDA backend in the
// library built with it (ref_use_cuda).
Backend g_backend = Backend::cpu;

OdtOptions odt_options(int nz, int iterations, int solver, int gp_transform, float tv_weight,
                       int tv_inner) {
  OdtOptions o;
  o.backend = g_backend;
  o.nz = nz;
  o.iterations = iterations;
  o.solver = solver ? Solver::tv : Solver::gerchberg_papoulis;
  o.gp_transform = gp_transform ? GpTransform::c2c : GpTransform::r2c;
  o.tv_weight = tv_weight;
  o.tv_inner = tv_inner;
  return o;
}

}  // namespace

extern "C" {

// Selects the reference's CUDA backend (1) or its CPU backend (0) for reconstruct and the Pipeline;
// error 2 when this library was built without the CUDA backend.
int ref_use_cuda(int on) {
  return guard([&] {
#ifdef QORAHOLO_HAS_CUDA
    g_backend = on ? Backend::cuda : Backend::cpu;
#else
    if (on) throw std::runtime_error("reference built without its CUDA backend");
    g_backend = Backend::cpu;
#endif
  });
}

const char* ref_last_error() { return g_error.c_str(); }

int ref_threads() { return cpu::threads(); }

int ref_circular_scan(int count, float na_ill, const float* geom, float* out) {
  return guard([&] {
    const auto il = circular_scan(count, na_ill, geometry(geom));
    for (int i = 0; i < count; ++i) {
      out[2 * i] = il[i].fy;
      out[2 * i + 1] = il[i].fx;
    }
  });
}

int ref_find_sideband(const float* h, int nz, int n, float dc_excl, int* iy, int* ix, float* fyx_mag) {
  return guard([&] {
    const Sideband s = find_sideband(load<float>(h, nz, n, n), dc_excl);
    *iy = s.iy;
    *ix = s.ix;
    fyx_mag[0] = s.y;
    fyx_mag[1] = s.x;
    fyx_mag[2] = s.magnitude;
  });
}

int ref_extract_fields(const float* h, int nz, int n, int has_center, float cy, float cx,
                       float radius, float dc_excl, int out_size, void* out) {
  return guard([&] {
    FieldOptions o;
    if (has_center) o.center = std::array<float, 2>{cy, cx};
    o.radius = radius;
    o.dc_exclusion = dc_excl;
    o.output_size = out_size;
    store(extract_fields(load<float>(h, nz, n, n), o), out);
  });
}

int ref_field_ratio(const void* s, int nz, int ny, int nx, const void* b, int bnz, void* out) {
  return guard([&] {
    store(field_ratio(load<cfloat>(s, nz, ny, nx), load<cfloat>(b, bnz, ny, nx)), out);
  });
}

int ref_unwrap(const float* w, int nz, int ny, int nx, float* out) {
  return guard([&] { store(unwrap(load<float>(w, nz, ny, nx)), out); });
}

int ref_rytov(const void* r, int nz, int ny, int nx, void* out) {
  return guard([&] { store(rytov(load<cfloat>(r, nz, ny, nx)), out); });
}

int ref_dct2(float* a, int nz, int ny, int nx, int axis, int inverse) {
  return guard([&] {
    auto arr = load<float>(a, nz, ny, nx);
    if (inverse) {
      cpu::idct2(arr, axis);
    } else {
      cpu::dct2(arr, axis);
    }
    store(arr, a);
  });
}

int ref_pocketfft_dct2(const float* a, int nz, int ny, int nx, int axis, float fct, float* out) {
  return guard([&] {
    const pocketfft::shape_t shape{std::size_t(nz), std::size_t(ny), std::size_t(nx)};
    const pocketfft::stride_t stride{std::ptrdiff_t(ny * nx * sizeof(float)),
                                     std::ptrdiff_t(nx * sizeof(float)), sizeof(float)};
    pocketfft::dct(shape, stride, stride, {std::size_t(axis)}, 2, a, out, fct, false);
  });
}

int ref_reconstruct(const void* fields, int count, int n, const float* il, const float* geom,
                    int nz, int iterations, int solver, int gp_transform, float tv_weight,
                    int tv_inner, float* out, double* filled, double* stage_ms) {
  return guard([&] {
    const Geometry g = geometry(geom);
    const auto ill = illum(il, count);
    const OdtOptions o = odt_options(nz, iterations, solver, gp_transform, tv_weight, tv_inner);
    const auto f = load<cfloat>(fields, count, n, n);
    const auto grid = odt_grid(n, count, ill, g, o);
    OdtTimings t;
    const OdtResult r = cpu::reconstruct(f, ill, grid, g, o, &t);
    store(r.ri, out);
    *filled = r.filled;
    if (stage_ms) {
      stage_ms[0] = t.fft2;
      stage_ms[1] = t.mapping;
      stage_ms[2] = t.normalize;
      stage_ms[3] = t.solve;
      stage_ms[4] = t.finish;
    }
  });
}

// The Ewald mapping of cpu::reconstruct (src/cpu/odt.cpp:137-171) on given spectra, followed by the
// Hermitian half data of src/cpu/odt.cpp:37-62: the grid from the reference's make_grid
// (src/api.cpp:32-42), every bin from its detail::ewald_target, the sign from detail::parity, and
// the half data from detail::hermitian_data and detail::negative_bin (src/common.hpp), so the
// indices, hit counts and sums are the reference's own. The loop is the reference's (one k_z column
// per iteration, illuminations in order, fiz in float). Outputs: a (nz, n, n/2+1) complex, hits
// (nz, n, n/2+1) in {0, 1, 2}, and the filled-voxel count.
int ref_ewald_half(const void* spectra, int count, int n, int nz, const float* il, const float* geom, void* a_out,
                   unsigned char* hits_out, long long* filled) {
  return guard([&] {
    const Geometry gm = geometry(geom);
    const detail::OdtGrid g = make_grid(n, nz, gm);
    const auto ill = illum(il, count);
    const auto* s = static_cast<const cfloat*>(spectra);
    const std::size_t plane = static_cast<std::size_t>(n) * n;
    std::vector<float> fiz(count);
    for (int a = 0; a < count; ++a) {
      fiz[a] = std::sqrt(g.fm2 - ill[a].fy * ill[a].fy - ill[a].fx * ill[a].fx);
    }
    std::vector<cfloat> pot(static_cast<std::size_t>(nz) * plane);
    std::vector<float> weight(pot.size(), 0.0f);
    for (int col = 0; col < static_cast<int>(plane); ++col) {
      const int ky = col / n;
      const int kx = col % n;
      for (int a = 0; a < count; ++a) {
        detail::EwaldTarget t{};
        if (!detail::ewald_target(g, ky, kx, ill[a].fy, ill[a].fx, fiz[a], t)) continue;
        const cfloat v = cfloat(0.0f, -g.gain * t.nuz) * s[a * plane + col];
        const std::size_t i = t.kz * plane + col;
        pot[i] += detail::parity(t.kz) * v;
        weight[i] += 1.0f;
      }
    }
    long long count_filled = 0;
    for (std::size_t i = 0; i < pot.size(); ++i) {
      if (weight[i] > 0) {
        pot[i] /= weight[i];
        ++count_filled;
      }
    }
    const int h = n / 2 + 1;
    auto* a = static_cast<cfloat*>(a_out);
    for (int kz = 0; kz < nz; ++kz) {
      const int mz = detail::negative_bin(kz, nz);
      for (int ky = 0; ky < n; ++ky) {
        const int my = detail::negative_bin(ky, n);
        for (int kx = 0; kx < h; ++kx) {
          const std::size_t i = (std::size_t(kz) * n + ky) * n + kx;
          const std::size_t j = (std::size_t(mz) * n + my) * n + detail::negative_bin(kx, n);
          const std::size_t o = (std::size_t(kz) * n + ky) * h + kx;
          float re = 0, im = 0;
          detail::hermitian_data(pot[i].real(), pot[i].imag(), pot[j].real(), pot[j].imag(), re, im);
          a[o] = {re, im};
          hits_out[o] = static_cast<unsigned char>((weight[i] > 0) + (weight[j] > 0));
        }
      }
    }
    *filled = count_filled;
  });
}

int ref_tv_prox(const float* b, float* x, float* dual_p, int nz, int ny, int nx, float lambda,
                int inner) {
  return guard([&] {
    const std::size_t size = std::size_t(nz) * ny * nx;
    cpu::Dual d(size);
    for (int a = 0; a < 3; ++a) std::memcpy(d.p[a].data(), dual_p + a * size, size * sizeof(float));
    const detail::Volume v{nz, ny, nx, nx};
    cpu::tv_prox(b, x, d, v, lambda, inner);
    for (int a = 0; a < 3; ++a) std::memcpy(dual_p + a * size, d.p[a].data(), size * sizeof(float));
  });
}

int ref_bpm_tables(int n, int nz, const float* il, int count, const float* geom, int obliquity,
                   void* step, void* last, float* q, float* phase_lipschitz) {
  return guard([&] {
    const BpmTables t = bpm_tables(n, nz, illum(il, count), geometry(geom), obliquity != 0);
    std::memcpy(step, t.step.data(), t.step.size() * sizeof(cfloat));
    std::memcpy(last, t.last.data(), t.last.size() * sizeof(cfloat));
    std::memcpy(q, t.q.data(), t.q.size() * sizeof(float));
    phase_lipschitz[0] = t.phase;
    phase_lipschitz[1] = t.lipschitz;
  });
}

int ref_bpm_forward(const float* ri, int nz, int n, const float* il, int count, const float* geom,
                    int obliquity, void* out) {
  return guard([&] {
    BpmOptions o;
    o.obliquity = obliquity != 0;
    store(bpm_forward(load<float>(ri, nz, n, n), illum(il, count), geometry(geom), o), out);
  });
}

// x: contrast n - n_medium; r: (count, n, n) residual.
int ref_bpm_vjp(const float* x, int nz, int n, const void* r, const float* il, int count,
                const float* geom, int obliquity, float* out) {
  return guard([&] {
    const BpmTables t = bpm_tables(n, nz, illum(il, count), geometry(geom), obliquity != 0);
    store(cpu::bpm_vjp(load<float>(x, nz, n, n), load<cfloat>(r, count, n, n), t), out);
  });
}

int ref_bpm_jvp(const float* x, const float* h, int nz, int n, const float* il, int count,
                const float* geom, int obliquity, void* out) {
  return guard([&] {
    const BpmTables t = bpm_tables(n, nz, illum(il, count), geometry(geom), obliquity != 0);
    store(cpu::bpm_jvp(load<float>(x, nz, n, n), load<float>(h, nz, n, n), t), out);
  });
}

int ref_bpm_reconstruct(const void* fields, int count, int n, const float* il, const float* geom,
                        const float* initial, int nz, int iterations, int batch, float step,
                        float tv_weight, int tv_inner, int obliquity, float* out, double* loss) {
  return guard([&] {
    BpmSolveOptions o;
    o.iterations = iterations;
    o.batch = batch;
    o.step = step;
    o.tv_weight = tv_weight;
    o.tv_inner = tv_inner;
    o.obliquity = obliquity != 0;
    const BpmResult r = bpm_reconstruct(load<cfloat>(fields, count, n, n), illum(il, count),
                                        geometry(geom), load<float>(initial, nz, n, n), o);
    store(r.ri, out);
    std::copy(r.loss.begin(), r.loss.end(), loss);
  });
}

int ref_render_phantom(const float* s, int k, const float* geom, int nz, int n, float* out) {
  return guard([&] { store(render_phantom(spheres(s, k), geometry(geom), nz, n), out); });
}

int ref_forward_fields(const float* s, int k, const float* il, int count, const float* geom, int n,
                       int model, void* out) {
  return guard([&] {
    const ScatteringModel m = model == 0   ? ScatteringModel::born
                              : model == 1 ? ScatteringModel::rytov
                                           : ScatteringModel::exact;
    store(forward_fields(spheres(s, k), illum(il, count), geometry(geom), n, m), out);
  });
}

int ref_synthesize_holograms(const void* ratio, int count, int ny, int nx, const float* il,
                             const float* geom, float cy, float cx, float amplitude, float noise,
                             unsigned long long seed, float* out) {
  return guard([&] {
    const HologramOptions o{{cy, cx}, amplitude, noise, seed};
    store(synthesize_holograms(load<cfloat>(ratio, count, ny, nx), illum(il, count), geometry(geom), o),
          out);
  });
}

// Pipeline on the CPU backend: constructor, set_background, then `runs` calls of run(). The
// result of the last run goes to out; ms[0] = setup, ms[1] = set_background, ms[2] = last run,
// ms[3..] = the stage timings of the last run (fields, rytov, fft2, mapping, normalize, solve,
// finish, total).
int ref_pipeline(const float* holo, const float* bg, int count, int n, float cy, float cx,
                 float radius, int out_size, const float* il, const float* geom, int nz,
                 int iterations, int solver, int gp_transform, float tv_weight, int tv_inner,
                 int runs, float* out, double* filled, double* ms) {
  return guard([&] {
    PipelineOptions po;
    po.count = count;
    po.hologram_size = n;
    po.field.center = std::array<float, 2>{cy, cx};
    po.field.radius = radius;
    po.field.output_size = out_size;
    po.illuminations = illum(il, count);
    po.geometry = geometry(geom);
    po.odt = odt_options(nz, iterations, solver, gp_transform, tv_weight, tv_inner);
    Pipeline p(po);
    const auto t0 = std::chrono::steady_clock::now();
    p.set_background(load<float>(bg, count, n, n));
    const double t_bg =
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    const auto h = load<float>(holo, count, n, n);
    OdtResult r;
    double t_run = 0;
    for (int i = 0; i < std::max(runs, 1); ++i) {
      const auto t1 = std::chrono::steady_clock::now();
      r = p.run(h);
      t_run = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t1).count();
    }
    store(r.ri, out);
    *filled = r.filled;
    const PipelineTimings& t = p.timings();
    const double v[] = {p.setup_ms(), t_bg,      t_run,   t.fields, t.rytov,  t.fft2,
                        t.mapping,    t.normalize, t.solve, t.finish, t.total};
    std::copy(std::begin(v), std::end(v), ms);
  });
}

// Checks that the Pipeline rejects process() before set_background() (logic_error) and a
// missing carrier (invalid_argument): returns the two error classes in codes[0..1].
int ref_pipeline_errors(int count, int n, const float* il, const float* geom, int* codes) {
  PipelineOptions po;
  po.count = count;
  po.hologram_size = n;
  po.field.center = std::array<float, 2>{float(n) / 4, float(n) / 4};
  po.field.output_size = n / 2;
  po.illuminations = illum(il, count);
  po.geometry = geometry(geom);
  codes[0] = guard([&] {
    Pipeline p(po);
    p.process();
  });
  po.field.center.reset();
  codes[1] = guard([&] { Pipeline p(po); });
  return 0;
}

}  // extern "C"
