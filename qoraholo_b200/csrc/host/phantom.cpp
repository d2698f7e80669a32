// Fixture generators of the public API (include/qoraholo/phantom.hpp): spheres rendered at voxel
// centres, analytic scattered fields (first Born / Rytov sphere spectra on the Ewald caps, or the
// exact scalar partial-wave solution for one sphere), and off-axis holograms with Gaussian noise.
// Host code in double precision, like the reference's generators (src/phantom.cpp); the final
// inverse 2D FFT of forward_fields runs on the device.
#include <cmath>
#include <complex>
#include <numbers>
#include <random>
#include <vector>

#include "host_common.hpp"
#include "qoraholo/phantom.hpp"

namespace qoraholo {

namespace {

constexpr double kPi = std::numbers::pi;

// Index under painter's order of the first `count` spheres at (z, y, x).
double index_at(std::span<const Sphere> spheres, std::size_t count, double n_medium, double z, double y, double x) {
  double n = n_medium;
  for (std::size_t i = 0; i < count; ++i) {
    const Sphere& s = spheres[i];
    const double dz = z - s.z, dy = y - s.y, dx = x - s.x;
    if (dz * dz + dy * dy + dx * dx <= double(s.radius) * s.radius) n = s.n;
  }
  return n;
}

// Fourier transform of the unit ball normalised to 1 at q = 0: 3 (sin x - x cos x) / x^3.
double ball(double x) {
  return x < 1e-3 ? 1.0 - x * x / 10.0 : 3.0 * (std::sin(x) - x * std::cos(x)) / (x * x * x);
}

// Scattering coefficients c_l of a homogeneous sphere (scalar Helmholtz, size parameter x = k R,
// relative index m): continuity of u and du/dr at r = R with spherical Bessel / Hankel functions,
// ratios j_l / j_{l-1} from a downward continued fraction for stability.
std::vector<std::complex<double>> sphere_coefficients(double x, double m) {
  const int lmax = static_cast<int>(x + 4.0 * std::cbrt(x) + 10.0);
  const auto ratios = [&](double z) {
    std::vector<double> rho(lmax + 1);
    double r = 0;
    for (int l = lmax + 60; l >= 1; --l) {
      r = 1.0 / ((2.0 * l + 1.0) / z - r);
      if (l <= lmax) rho[l] = r;
    }
    return rho;
  };
  const auto rx = ratios(x);
  const auto rm = ratios(m * x);
  std::vector<std::complex<double>> c(lmax + 1);
  double jm1 = std::cos(x) / x, j = std::sin(x) / x;
  double ym1 = std::sin(x) / x, y = -std::cos(x) / x;
  for (int l = 0; l <= lmax; ++l) {
    if (l > 0) {
      const double yn = (2.0 * l - 1.0) / x * y - ym1;
      ym1 = y;
      y = yn;
      jm1 = j;
      j = rx[l] * j;
    }
    const std::complex<double> h(j, y), hm1(jm1, ym1);
    const double dj = jm1 - (l + 1.0) / x * j;
    const std::complex<double> dh = hm1 - (l + 1.0) / x * h;
    const double d = (l == 0 ? 1.0 / std::tan(m * x) : 1.0 / rm[l]) - (l + 1.0) / (m * x);
    c[l] = (m * d * j - dj) / (dh - m * d * h);
  }
  return c;
}

}  // namespace

Array3<float> render_phantom(std::span<const Sphere> spheres, const Geometry& geometry, int nz, int n) {
  if (nz < 1 || n < 1) throw std::invalid_argument("render_phantom: empty shape");
  Array3<float> out(nz, n, n);
  const double d = geometry.pixel;
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < n; ++i)
        out(k, j, i) = static_cast<float>(
            index_at(spheres, spheres.size(), geometry.n_medium, (k - nz / 2) * d, (j - n / 2) * d, (i - n / 2) * d));
  return out;
}

Array3<cfloat> forward_fields(std::span<const Sphere> spheres, std::span<const Illumination> illuminations,
                              const Geometry& geometry, int n, ScatteringModel model) {
  if (n < 4 || n % 2 != 0) throw std::invalid_argument("forward_fields: n must be even");
  if (model == ScatteringModel::exact && spheres.size() != 1) {
    throw std::invalid_argument("forward_fields: the exact model takes exactly one sphere");
  }
  const double k0 = 2.0 * kPi / geometry.wavelength;
  const double nm = geometry.n_medium;
  const double fm2 = nm * nm / (double(geometry.wavelength) * geometry.wavelength);
  const double fna2 = double(geometry.na) * geometry.na / (double(geometry.wavelength) * geometry.wavelength);
  const double d = geometry.pixel;
  const double df = 1.0 / (n * d);
  const double km = k0 * nm;
  const auto waves = model == ScatteringModel::exact ? sphere_coefficients(km * spheres[0].radius, spheres[0].n / nm)
                                                     : std::vector<std::complex<double>>{};
  // Potential step of each sphere over the index it is painted on, times its volume.
  std::vector<double> step(spheres.size());
  for (std::size_t i = 0; i < spheres.size(); ++i) {
    const Sphere& s = spheres[i];
    const double parent = index_at(spheres, i, nm, s.z, s.y, s.x);
    step[i] = k0 * k0 * (double(s.n) * s.n - parent * parent) * (4.0 / 3.0 * kPi * double(s.radius) * s.radius * s.radius);
  }
  const int count = static_cast<int>(illuminations.size());
  Array3<cfloat> out(count, n, n);
  for (int a = 0; a < count; ++a) {
    const double fiy = illuminations[a].fy, fix = illuminations[a].fx;
    if (fiy * fiy + fix * fix >= fm2) {
      throw std::invalid_argument("forward_fields: illumination beyond n_medium / wavelength");
    }
    const double fiz = std::sqrt(fm2 - fiy * fiy - fix * fix);
    for (int ky = 0; ky < n; ++ky) {
      for (int kx = 0; kx < n; ++kx) {
        const double my = (ky < n / 2 ? ky : ky - n) * df;
        const double mx = (kx < n / 2 ? kx : kx - n) * df;
        const double fy = my + fiy, fx = mx + fix;
        const double rho2 = fy * fy + fx * fx;
        std::complex<double> u = 0;
        if (rho2 <= fna2 && rho2 < fm2) {
          const double nuz = std::sqrt(fm2 - rho2);
          const double qz = nuz - fiz;
          std::complex<double> o = 0;  // 3D spectrum of the scattering potential at q
          if (model == ScatteringModel::exact) {
            const Sphere& s = spheres[0];
            const double ct = (fy * fiy + fx * fix + nuz * fiz) / fm2;
            std::complex<double> sum = 0;
            double pm1 = 0, p = 1;  // Legendre P_{l-1}, P_l
            for (std::size_t l = 0; l < waves.size(); ++l) {
              const double w = 2.0 * double(l) + 1.0;
              sum += w * waves[l] * p;
              const double pn = (w * ct * p - double(l) * pm1) / (double(l) + 1.0);
              pm1 = p;
              p = pn;
            }
            o = 4.0 * kPi * std::complex<double>(0.0, -1.0 / km) * sum *
                std::polar(1.0, -2.0 * kPi * (qz * s.z + my * s.y + mx * s.x));
          } else {
            const double q = 2.0 * kPi * std::sqrt(qz * qz + my * my + mx * mx);
            for (std::size_t i = 0; i < spheres.size(); ++i) {
              const Sphere& s = spheres[i];
              o += step[i] * ball(q * s.radius) * std::polar(1.0, -2.0 * kPi * (qz * s.z + my * s.y + mx * s.x));
            }
          }
          // Fourier diffraction theorem U = i o / (4 pi nu_z); centre-origin DFT: (-1)^(ky+kx) / d^2.
          u = std::complex<double>(0.0, 1.0 / (4.0 * kPi * nuz)) * o * (((ky + kx) & 1) ? -1.0 : 1.0) / (d * d);
        }
        out(a, ky, kx) = cfloat(u);
      }
    }
  }
  host::require_cuda(Backend::cuda);
  host::check(qhk_fft2d_host(out.data.data(), count, n, 0, 1.0f / static_cast<float>(n * n)));
  for (auto& v : out.data) v = model == ScatteringModel::rytov ? std::exp(v) : 1.0f + v;
  return out;
}

Array3<float> synthesize_holograms(const Array3<cfloat>& ratio, std::span<const Illumination> illuminations,
                                   const Geometry& geometry, const HologramOptions& options) {
  if (static_cast<std::size_t>(ratio.nz) != illuminations.size()) {
    throw std::invalid_argument("synthesize_holograms: need one illumination per field");
  }
  Array3<float> out(ratio.nz, ratio.ny, ratio.nx);
  std::mt19937_64 rng(options.seed);
  std::normal_distribution<float> noise(0.0f, options.noise);
  const double d = geometry.pixel;
  for (int a = 0; a < ratio.nz; ++a) {
    for (int y = 0; y < ratio.ny; ++y) {
      for (int x = 0; x < ratio.nx; ++x) {
        const double ry = (y - ratio.ny / 2) * d, rx = (x - ratio.nx / 2) * d;
        const auto incident = std::polar(1.0, 2.0 * kPi * (illuminations[a].fy * ry + illuminations[a].fx * rx));
        const auto reference = std::polar(double(options.reference_amplitude),
                                          -2.0 * kPi * (options.carrier[0] * ry + options.carrier[1] * rx));
        float v = static_cast<float>(std::norm(reference + incident * std::complex<double>(ratio(a, y, x))));
        if (options.noise > 0) v += noise(rng);
        out(a, y, x) = v;
      }
    }
  }
  return out;
}

}  // namespace qoraholo
