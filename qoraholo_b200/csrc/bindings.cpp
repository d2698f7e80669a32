// Python module `_core`: the reference's binding surface (python/bindings.cpp of QoraHolo,
// nanobind) restated with pybind11 over the C++ API of this library. Names, argument names,
// defaults and return types are the reference's, except that `backend` defaults to "cuda" (the
// only backend of this build). The GIL is released around device work.
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <optional>
#include <stdexcept>
#include <string>
#include <vector>

#include "qoraholo/qoraholo.hpp"
#include "qoraholo_b200.h"
#include "host/raw.hpp"

namespace py = pybind11;
using namespace qoraholo;

namespace {

template <class T>
using In = py::array_t<T, py::array::c_style | py::array::forcecast>;

// (count, ny, nx) of a 3D array, as to_array validates it.
template <class T>
std::array<int, 3> dims3(const In<T>& a) {
  if (a.ndim() != 3) throw std::invalid_argument("expected a 3D array (count, ny, nx)");
  return {static_cast<int>(a.shape(0)), static_cast<int>(a.shape(1)), static_cast<int>(a.shape(2))};
}

template <class T>
Array3<T> to_array(const In<T>& a) {
  if (a.ndim() != 3) throw std::invalid_argument("expected a 3D array (count, ny, nx)");
  Array3<T> out(static_cast<int>(a.shape(0)), static_cast<int>(a.shape(1)), static_cast<int>(a.shape(2)));
  std::copy(a.data(), a.data() + a.size(), out.data.begin());
  return out;
}

// Page-locked buffers for Pipeline.run results, recycled when their arrays are released (a couple of
// free buffers per size are kept; the rest are freed). Never destroyed: at exit the CUDA runtime may
// already be gone.
struct PooledBuffer {
  float* data;
  std::size_t size;
};

class PinnedPool {
 public:
  float* take(std::size_t n) {
    {
      std::lock_guard<std::mutex> lk(mu_);
      auto& v = free_[n];
      if (!v.empty()) {
        float* p = v.back();
        v.pop_back();
        return p;
      }
    }
    void* p = nullptr;
    if (qhk_pinned_alloc(n * sizeof(float), &p) != QHK_OK) throw std::runtime_error(qhk_last_error());
    return static_cast<float*>(p);
  }
  void give(float* p, std::size_t n) {
    {
      std::lock_guard<std::mutex> lk(mu_);
      auto& v = free_[n];
      if (v.size() < kKeep) {
        v.push_back(p);
        return;
      }
    }
    qhk_pinned_free(p);
  }

 private:
  static constexpr std::size_t kKeep = 2;
  std::mutex mu_;
  std::map<std::size_t, std::vector<float*>> free_;
};

PinnedPool& pinned_pool() {
  static auto* pool = new PinnedPool;
  return *pool;
}

template <class T>
py::array_t<T> to_numpy(Array3<T>&& a) {
  auto* owner = new std::vector<T>(std::move(a.data));
  py::capsule free(owner, [](void* p) { delete static_cast<std::vector<T>*>(p); });
  return py::array_t<T>({static_cast<py::ssize_t>(a.nz), static_cast<py::ssize_t>(a.ny), static_cast<py::ssize_t>(a.nx)},
                        owner->data(), free);
}

std::vector<Illumination> to_illum(const In<float>& a) {
  if (a.ndim() != 2 || a.shape(1) != 2) throw std::invalid_argument("illuminations must have shape (count, 2)");
  std::vector<Illumination> out(a.shape(0));
  for (py::ssize_t i = 0; i < a.shape(0); ++i) out[i] = {a.at(i, 0), a.at(i, 1)};
  return out;
}

Backend parse_backend(const std::string& s) {
  if (s == "cpu") return Backend::cpu;
  if (s == "cuda") return Backend::cuda;
  throw std::invalid_argument("backend must be 'cpu' or 'cuda'");
}

Solver parse_solver(const std::string& s) {
  if (s == "gp") return Solver::gerchberg_papoulis;
  if (s == "tv") return Solver::tv;
  throw std::invalid_argument("solver must be 'gp' or 'tv'");
}

GpTransform parse_transform(const std::string& s) {
  if (s == "r2c") return GpTransform::r2c;
  if (s == "c2c") return GpTransform::c2c;
  throw std::invalid_argument("gp_transform must be 'r2c' or 'c2c'");
}

Mapping parse_mapping(const std::string& s) {
  if (s == "gather") return Mapping::gather;
  if (s == "scatter") return Mapping::scatter;
  throw std::invalid_argument("mapping must be 'gather' or 'scatter'");
}

OdtOptions odt_options(int nz, int iterations, const std::string& solver, const std::string& gp_transform,
                       float tv_weight, int tv_inner, const std::string& mapping, const std::string& backend) {
  OdtOptions o;
  o.nz = nz;
  o.iterations = iterations;
  o.solver = parse_solver(solver);
  o.gp_transform = parse_transform(gp_transform);
  o.tv_weight = tv_weight;
  o.tv_inner = tv_inner;
  o.mapping = parse_mapping(mapping);
  o.backend = parse_backend(backend);
  return o;
}

}  // namespace

PYBIND11_MODULE(_core, m) {
  m.def("cuda_available", &cuda_available);

  py::class_<Geometry>(m, "Geometry")
      .def(py::init<>())
      .def(py::init([](float wavelength, float n_medium, float na, float pixel) {
             return Geometry{wavelength, n_medium, na, pixel};
           }),
           py::arg("wavelength"), py::arg("n_medium"), py::arg("na"), py::arg("pixel"))
      .def_readwrite("wavelength", &Geometry::wavelength)
      .def_readwrite("n_medium", &Geometry::n_medium)
      .def_readwrite("na", &Geometry::na)
      .def_readwrite("pixel", &Geometry::pixel)
      .def("__repr__", [](const Geometry& g) {
        return "Geometry(wavelength=" + std::to_string(g.wavelength) + ", n_medium=" + std::to_string(g.n_medium) +
               ", na=" + std::to_string(g.na) + ", pixel=" + std::to_string(g.pixel) + ")";
      });

  py::class_<Sphere>(m, "Sphere")
      .def(py::init([](float z, float y, float x, float radius, float n) { return Sphere{z, y, x, radius, n}; }),
           py::arg("z"), py::arg("y"), py::arg("x"), py::arg("radius"), py::arg("n"))
      .def_readwrite("z", &Sphere::z)
      .def_readwrite("y", &Sphere::y)
      .def_readwrite("x", &Sphere::x)
      .def_readwrite("radius", &Sphere::radius)
      .def_readwrite("n", &Sphere::n);

  py::class_<Sideband>(m, "Sideband")
      .def_readonly("iy", &Sideband::iy)
      .def_readonly("ix", &Sideband::ix)
      .def_readonly("y", &Sideband::y)
      .def_readonly("x", &Sideband::x)
      .def_readonly("magnitude", &Sideband::magnitude);

  // The per-call functions run on the numpy buffers themselves (raw.hpp): no copies into owning
  // arrays, outputs allocated uninitialised and written by the device transfer.
  m.def(
      "find_sideband",
      [](In<float> holograms, float dc_exclusion) {
        const auto [nz, ny, nx] = dims3(holograms);
        py::gil_scoped_release release;
        return raw::find_sideband(holograms.data(), nz, ny, nx, dc_exclusion);
      },
      py::arg("holograms"), py::arg("dc_exclusion") = 0.0f);

  m.def(
      "extract_fields",
      [](In<float> holograms, std::optional<std::array<float, 2>> center, float radius, float dc_exclusion,
         int output_size, const std::string& backend) {
        const auto [nz, ny, nx] = dims3(holograms);
        const FieldOptions opt{center, radius, dc_exclusion, output_size};
        const Backend b = parse_backend(backend);
        raw::FieldCall call;
        {
          py::gil_scoped_release release;
          call = raw::extract_fields_check(holograms.data(), nz, ny, nx, opt, b);
        }
        py::array_t<cfloat> out({nz, call.out, call.out});
        {
          py::gil_scoped_release release;
          raw::extract_fields_run(holograms.data(), nz, nx, opt, call, out.mutable_data());
        }
        return out;
      },
      py::arg("holograms"), py::arg("center") = py::none(), py::arg("radius") = 0.0f, py::arg("dc_exclusion") = 0.0f,
      py::arg("output_size") = 0, py::arg("backend") = "cuda");

  m.def(
      "field_ratio",
      [](In<cfloat> sample, In<cfloat> background) {
        const auto [nz, ny, nx] = dims3(sample);
        const auto [bz, by, bx] = dims3(background);
        raw::field_ratio_check(nz, ny, nx, bz, by, bx);
        py::array_t<cfloat> out({nz, ny, nx});
        {
          py::gil_scoped_release release;
          raw::field_ratio_run(sample.data(), nz, ny, nx, background.data(), bz, out.mutable_data());
        }
        return out;
      },
      py::arg("sample"), py::arg("background"));

  m.def(
      "unwrap",
      [](In<float> wrapped, const std::string& backend) {
        const auto [nz, ny, nx] = dims3(wrapped);
        raw::unwrap_check(ny, nx, parse_backend(backend));
        py::array_t<float> out({nz, ny, nx});
        {
          py::gil_scoped_release release;
          raw::unwrap_run(wrapped.data(), nz, ny, nx, out.mutable_data());
        }
        return out;
      },
      py::arg("wrapped"), py::arg("backend") = "cuda");

  m.def(
      "rytov",
      [](In<cfloat> ratio, const std::string& backend) {
        const auto [nz, ny, nx] = dims3(ratio);
        raw::rytov_check(ny, nx, parse_backend(backend));
        py::array_t<cfloat> out({nz, ny, nx});
        {
          py::gil_scoped_release release;
          raw::rytov_run(ratio.data(), nz, ny, nx, out.mutable_data());
        }
        return out;
      },
      py::arg("ratio"), py::arg("backend") = "cuda");

  m.def(
      "reconstruct",
      [](In<cfloat> fields, In<float> illuminations, const Geometry& geometry, int nz, int iterations,
         const std::string& solver, const std::string& gp_transform, float tv_weight, int tv_inner,
         const std::string& mapping, const std::string& backend) {
        const auto [count, ny, nx] = dims3(fields);
        const auto il = to_illum(illuminations);
        const OdtOptions opt = odt_options(nz, iterations, solver, gp_transform, tv_weight, tv_inner, mapping, backend);
        const int depth = raw::reconstruct_check(count, ny, nx, il, geometry, opt);
        py::array_t<float> out({depth, nx, nx});
        double filled = 0;
        {
          py::gil_scoped_release release;
          filled = raw::reconstruct_run(fields.data(), count, nx, il, geometry, opt, out.mutable_data());
        }
        return py::make_tuple(out, filled);
      },
      py::arg("fields"), py::arg("illuminations"), py::arg("geometry"), py::arg("nz") = 0, py::arg("iterations") = 0,
      py::arg("solver") = "gp", py::arg("gp_transform") = "r2c", py::arg("tv_weight") = OdtOptions{}.tv_weight,
      py::arg("tv_inner") = OdtOptions{}.tv_inner, py::arg("mapping") = "gather", py::arg("backend") = "cuda");

  py::class_<Pipeline>(m, "Pipeline")
      .def(py::init([](int count, int hologram_size, std::array<float, 2> center, float radius, int output_size,
                       In<float> illuminations, const Geometry& geometry, int nz, int iterations,
                       const std::string& solver, const std::string& gp_transform, float tv_weight, int tv_inner,
                       const std::string& mapping, const std::string& backend, int upload_chunks) {
             PipelineOptions o;
             o.count = count;
             o.hologram_size = hologram_size;
             o.field.center = center;
             o.field.radius = radius;
             o.field.output_size = output_size;
             o.illuminations = to_illum(illuminations);
             o.geometry = geometry;
             o.odt = odt_options(nz, iterations, solver, gp_transform, tv_weight, tv_inner, mapping, backend);
             o.upload_chunks = upload_chunks;
             return new Pipeline(std::move(o));
           }),
           py::arg("count"), py::arg("hologram_size"), py::arg("center"), py::arg("radius"), py::arg("output_size"),
           py::arg("illuminations"), py::arg("geometry"), py::arg("nz"), py::arg("iterations"), py::arg("solver"),
           py::arg("gp_transform"), py::arg("tv_weight"), py::arg("tv_inner"), py::arg("mapping"), py::arg("backend"),
           py::arg("upload_chunks"))
      .def(
          "set_background",
          [](Pipeline& p, In<float> backgrounds) {
            auto b = to_array(backgrounds);
            py::gil_scoped_release release;
            p.set_background(b);
          },
          py::arg("backgrounds"))
      .def(
          "run",
          [](Pipeline& p, In<float> holograms) {
            if (static_cast<std::size_t>(holograms.size()) != p.input().size() || holograms.ndim() != 3 ||
                holograms.shape(1) != holograms.shape(2)) {
              throw std::invalid_argument("Pipeline.run: shape must be (count, N, N)");
            }
            const auto [nz, ny, nx] = p.output_shape();
            // The result lives in a page-locked buffer of the pool, so the device writes it directly;
            // the buffer goes back to the pool when the array is released.
            const std::size_t n = static_cast<std::size_t>(nz) * ny * nx;
            auto* owner = new PooledBuffer{pinned_pool().take(n), n};
            py::capsule release_buffer(owner, [](void* o) {
              auto* b = static_cast<PooledBuffer*>(o);
              pinned_pool().give(b->data, b->size);
              delete b;
            });
            py::array_t<float> out({nz, ny, nx}, owner->data, release_buffer);
            std::span<const float> in(holograms.data(), static_cast<std::size_t>(holograms.size()));
            std::span<float> dst(owner->data, n);
            {
              py::gil_scoped_release release;
              p.run(in, dst);
            }
            return out;
          },
          py::arg("holograms"))
      .def(
          "run_stream",
          [](Pipeline& p, In<float> holograms) {
            if (holograms.ndim() != 4 || holograms.shape(0) < 1 ||
                static_cast<std::size_t>(holograms.size()) != holograms.shape(0) * p.input().size() ||
                holograms.shape(2) != holograms.shape(3)) {
              throw std::invalid_argument("Pipeline.run_stream: shape must be (items, count, N, N)");
            }
            const auto [nz, ny, nx] = p.output_shape();
            const int items = static_cast<int>(holograms.shape(0));
            const std::size_t n = static_cast<std::size_t>(items) * nz * ny * nx;
            auto* owner = new PooledBuffer{pinned_pool().take(n), n};
            py::capsule release_buffer(owner, [](void* o) {
              auto* b = static_cast<PooledBuffer*>(o);
              pinned_pool().give(b->data, b->size);
              delete b;
            });
            py::array_t<float> out({items, nz, ny, nx}, owner->data, release_buffer);
            std::span<const float> in(holograms.data(), static_cast<std::size_t>(holograms.size()));
            std::span<float> dst(owner->data, n);
            {
              py::gil_scoped_release release;
              p.run_stream(in, dst, items);
            }
            return out;
          },
          py::arg("holograms"))
      .def_property_readonly("filled", &Pipeline::filled)
      .def_property_readonly("setup_ms", &Pipeline::setup_ms)
      .def_property_readonly("device_bytes", &Pipeline::device_bytes)
      .def_property_readonly("timings", [](const Pipeline& p) {
        const PipelineTimings& t = p.timings();
        py::dict d;
        d["upload"] = t.upload;
        d["fields"] = t.fields;
        d["rytov"] = t.rytov;
        d["fft2"] = t.fft2;
        d["clear"] = t.clear;
        d["mapping"] = t.mapping;
        d["normalize"] = t.normalize;
        d["solve"] = t.solve;
        d["finish"] = t.finish;
        d["download"] = t.download;
        d["total"] = t.total;
        return d;
      });

  m.def(
      "circular_scan",
      [](int count, float na_illumination, const Geometry& geometry) {
        const auto il = circular_scan(count, na_illumination, geometry);
        Array3<float> out(1, count, 2);
        for (int i = 0; i < count; ++i) {
          out.data[2 * i] = il[i].fy;
          out.data[2 * i + 1] = il[i].fx;
        }
        return to_numpy(std::move(out));
      },
      py::arg("count"), py::arg("na_illumination"), py::arg("geometry"));

  m.def(
      "render_phantom",
      [](const std::vector<Sphere>& spheres, const Geometry& geometry, int nz, int n) {
        return to_numpy(render_phantom(spheres, geometry, nz, n));
      },
      py::arg("spheres"), py::arg("geometry"), py::arg("nz"), py::arg("n"));

  m.def(
      "forward_fields",
      [](const std::vector<Sphere>& spheres, In<float> illuminations, const Geometry& geometry, int n,
         const std::string& model) {
        ScatteringModel sm{};
        if (model == "rytov") {
          sm = ScatteringModel::rytov;
        } else if (model == "born") {
          sm = ScatteringModel::born;
        } else if (model == "exact") {
          sm = ScatteringModel::exact;
        } else {
          throw std::invalid_argument("model must be 'rytov', 'born' or 'exact'");
        }
        const auto il = to_illum(illuminations);
        Array3<cfloat> out;
        {
          py::gil_scoped_release release;
          out = forward_fields(spheres, il, geometry, n, sm);
        }
        return to_numpy(std::move(out));
      },
      py::arg("spheres"), py::arg("illuminations"), py::arg("geometry"), py::arg("n"), py::arg("model") = "rytov");

  m.def(
      "bpm_forward",
      [](In<float> ri, In<float> illuminations, const Geometry& geometry, bool obliquity, const std::string& backend) {
        auto v = to_array(ri);
        const auto il = to_illum(illuminations);
        const BpmOptions opt{obliquity, parse_backend(backend)};
        Array3<cfloat> out;
        {
          py::gil_scoped_release release;
          out = bpm_forward(v, il, geometry, opt);
        }
        return to_numpy(std::move(out));
      },
      py::arg("ri"), py::arg("illuminations"), py::arg("geometry"), py::arg("obliquity") = true,
      py::arg("backend") = "cuda");

  m.def(
      "bpm_reconstruct",
      [](In<cfloat> fields, In<float> illuminations, const Geometry& geometry, In<float> initial, int iterations,
         int batch, float step, float tv_weight, int tv_inner, bool obliquity, const std::string& backend) {
        auto f = to_array(fields);
        auto init = to_array(initial);
        const auto il = to_illum(illuminations);
        BpmSolveOptions opt;
        opt.iterations = iterations;
        opt.batch = batch;
        opt.step = step;
        opt.tv_weight = tv_weight;
        opt.tv_inner = tv_inner;
        opt.obliquity = obliquity;
        opt.backend = parse_backend(backend);
        BpmResult r;
        {
          py::gil_scoped_release release;
          r = bpm_reconstruct(f, il, geometry, init, opt);
        }
        return py::make_tuple(to_numpy(std::move(r.ri)), r.loss);
      },
      py::arg("fields"), py::arg("illuminations"), py::arg("geometry"), py::arg("initial"), py::arg("iterations"),
      py::arg("batch"), py::arg("step"), py::arg("tv_weight"), py::arg("tv_inner"), py::arg("obliquity"),
      py::arg("backend"));

  m.def(
      "synthesize_holograms",
      [](In<cfloat> ratio, In<float> illuminations, const Geometry& geometry, std::array<float, 2> carrier,
         float reference_amplitude, float noise, std::uint64_t seed) {
        const HologramOptions opt{carrier, reference_amplitude, noise, seed};
        return to_numpy(synthesize_holograms(to_array(ratio), to_illum(illuminations), geometry, opt));
      },
      py::arg("ratio"), py::arg("illuminations"), py::arg("geometry"),
      py::arg("carrier") = std::array<float, 2>{5.0f, 5.0f}, py::arg("reference_amplitude") = 1.0f,
      py::arg("noise") = 0.0f, py::arg("seed") = 1);
}
