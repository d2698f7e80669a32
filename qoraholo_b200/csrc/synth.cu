// Off-axis hologram synthesis on the device: |R + u_in * ratio|^2 + Gaussian noise, the formula of
// the reference's synthesize_holograms (src/phantom.cpp:193-221), for generating request streams
// without a host round trip. The intensity is formed in double as on the host, so noise-free
// holograms agree with the host's to float rounding. The noise comes from a counter-based generator
// (a 64-bit mix of (seed, pixel) and the Box-Muller transform), not from std::mt19937_64: the draws
// differ from the host's, their distribution (zero mean, standard deviation `noise`) is the same,
// and a seed gives the same holograms on every run and device.
#include <algorithm>
#include <cmath>
#include <complex>
#include <numbers>
#include <vector>

#include "qhk_internal.hpp"
#include "synth.hpp"

namespace qhk {

namespace {

__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
  // splitmix64 finaliser (Steele, Lea and Flood 2014)
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

__global__ void k_synthesize(const float2* __restrict__ ratio, const double2* __restrict__ illum, int count, int n,
                             double pixel, double carrier_y, double carrier_x, double amplitude, float noise,
                             unsigned long long seed, float* __restrict__ out) {
  const std::size_t plane = static_cast<std::size_t>(n) * n;
  const std::size_t total = plane * count;
  const double two_pi = 2.0 * 3.14159265358979323846;
  for (std::size_t i = blockIdx.x * static_cast<std::size_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<std::size_t>(gridDim.x) * blockDim.x) {
    const int a = static_cast<int>(i / plane);
    const std::size_t p = i - static_cast<std::size_t>(a) * plane;
    const int y = static_cast<int>(p / n);
    const int x = static_cast<int>(p - static_cast<std::size_t>(y) * n);
    const double ry = (y - n / 2) * pixel, rx = (x - n / 2) * pixel;
    const double2 il = illum[a];
    double si, ci, sr, cr;
    sincos(two_pi * (il.x * ry + il.y * rx), &si, &ci);
    sincos(-two_pi * (carrier_y * ry + carrier_x * rx), &sr, &cr);
    const float2 r = ratio[i];
    // reference + incident * ratio
    const double re = amplitude * cr + (ci * r.x - si * r.y);
    const double im = amplitude * sr + (ci * r.y + si * r.x);
    float v = static_cast<float>(re * re + im * im);
    if (noise > 0.0f) {
      const unsigned long long h1 = mix64(seed ^ mix64(2 * i));
      const unsigned long long h2 = mix64(seed ^ mix64(2 * i + 1));
      const double u1 = (static_cast<double>(h1 >> 11) + 1.0) * (1.0 / 9007199254740992.0);  // (0, 1]
      const double u2 = static_cast<double>(h2 >> 11) * (1.0 / 9007199254740992.0);          // [0, 1)
      v += noise * static_cast<float>(sqrt(-2.0 * log(u1)) * cos(two_pi * u2));
    }
    out[i] = v;
  }
}

// ---- Spheres: rendered index and analytic fields (include/qoraholo/phantom.hpp) ------------------
// One thread per voxel / per spectrum sample, in double precision like the reference's host
// generators (src/phantom.cpp:84-191), with products and sums rounded separately (no fused
// multiply-add) where a comparison decides the result, so that the rendered index equals the host
// evaluation bit for bit.

// Index at voxel centres: painter's order, i.e. the last sphere (in the given order) that contains
// the centre decides, found by scanning the spheres backwards and stopping at the first hit.
__global__ void k_render_spheres(const double4* __restrict__ sph, const double* __restrict__ index, int k,
                                 double n_medium, int nz, int n, double pixel, float* __restrict__ out) {
  const std::size_t plane = static_cast<std::size_t>(n) * n;
  const std::size_t total = plane * nz;
  for (std::size_t i = blockIdx.x * static_cast<std::size_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<std::size_t>(gridDim.x) * blockDim.x) {
    const int z = static_cast<int>(i / plane);
    const std::size_t p = i - static_cast<std::size_t>(z) * plane;
    const int y = static_cast<int>(p / n);
    const int x = static_cast<int>(p - static_cast<std::size_t>(y) * n);
    const double pz = __dmul_rn(static_cast<double>(z - nz / 2), pixel);
    const double py = __dmul_rn(static_cast<double>(y - n / 2), pixel);
    const double px = __dmul_rn(static_cast<double>(x - n / 2), pixel);
    double v = n_medium;
    for (int s = k - 1; s >= 0; --s) {
      const double4 c = sph[s];  // centre z, y, x and squared radius
      const double dz = __dsub_rn(pz, c.x), dy = __dsub_rn(py, c.y), dx = __dsub_rn(px, c.z);
      const double d2 = __dadd_rn(__dadd_rn(__dmul_rn(dz, dz), __dmul_rn(dy, dy)), __dmul_rn(dx, dx));
      if (d2 <= c.w) {
        v = index[s];
        break;
      }
    }
    out[i] = static_cast<float>(v);
  }
}

struct SpectrumGrid {
  double fm2, fna2, df, pixel;
  double km;  // 2 pi n_medium / wavelength
  int n, count, k;
  int waves;  // partial-wave terms of the exact model, 0 for the first-order models
};

// The scattered field's 2D spectrum at bin (ky, kx) of view a, on the centre-origin grid (the
// (-1)^(ky + kx) / pixel^2 factor makes the plain inverse DFT land on it): the Fourier diffraction
// theorem U = i O(q) / (4 pi nu_z) on the Ewald cap, q = (nu_z - fiz, my, mx), zero outside the
// pupil. O(q) is the sum of the spheres' first Born spectra (potential step times volume times the
// ball's form factor, phase of the centre) or, for one sphere, its exact scalar far field (partial
// waves c_l summed against Legendre polynomials of the scattering angle).
__global__ void k_sphere_spectra(const double2* __restrict__ illum, const double4* __restrict__ sph,
                                 const double* __restrict__ step, const double2* __restrict__ waves, SpectrumGrid g,
                                 float2* __restrict__ out) {
  const double two_pi = 2.0 * 3.14159265358979323846;
  const std::size_t plane = static_cast<std::size_t>(g.n) * g.n;
  const std::size_t total = plane * g.count;
  for (std::size_t i = blockIdx.x * static_cast<std::size_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<std::size_t>(gridDim.x) * blockDim.x) {
    const int a = static_cast<int>(i / plane);
    const std::size_t p = i - static_cast<std::size_t>(a) * plane;
    const int ky = static_cast<int>(p / g.n);
    const int kx = static_cast<int>(p - static_cast<std::size_t>(ky) * g.n);
    const double my = (ky < g.n / 2 ? ky : ky - g.n) * g.df;
    const double mx = (kx < g.n / 2 ? kx : kx - g.n) * g.df;
    const double2 il = illum[a];
    const double fy = my + il.x, fx = mx + il.y;
    const double rho2 = fy * fy + fx * fx;
    float2 u = make_float2(0.0f, 0.0f);
    if (rho2 <= g.fna2 && rho2 < g.fm2) {
      const double fiz = sqrt(g.fm2 - il.x * il.x - il.y * il.y);
      const double nuz = sqrt(g.fm2 - rho2);
      const double qz = nuz - fiz;
      double ore = 0.0, oim = 0.0;  // O(q)
      if (g.waves > 0) {
        // exact: O = 4 pi (-i / k_m) sum_l (2l + 1) c_l P_l(cos theta) e^{-2 pi i q.c}
        const double ct = (fy * il.x + fx * il.y + nuz * fiz) / g.fm2;
        double sre = 0.0, sim = 0.0, pl = 1.0, plm1 = 0.0;
        for (int l = 0; l < g.waves; ++l) {
          const double w = 2.0 * l + 1.0;
          sre += w * waves[l].x * pl;
          sim += w * waves[l].y * pl;
          const double pn = (w * ct * pl - l * plm1) / (l + 1.0);
          plm1 = pl;
          pl = pn;
        }
        const double4 c = sph[0];
        double sn, cs;
        sincos(-two_pi * (qz * c.x + my * c.y + mx * c.z), &sn, &cs);
        const double f = 4.0 * 3.14159265358979323846 / g.km;  // times -i
        const double tre = f * sim, tim = -f * sre;         // -i f (sre + i sim)
        ore = tre * cs - tim * sn;
        oim = tre * sn + tim * cs;
      } else {
        const double q = two_pi * sqrt(qz * qz + my * my + mx * mx);
        for (int s = 0; s < g.k; ++s) {
          const double4 c = sph[s];
          const double x = q * sqrt(c.w);
          const double ball = x < 1e-3 ? 1.0 - x * x / 10.0 : 3.0 * (sin(x) - x * cos(x)) / (x * x * x);
          double sn, cs;
          sincos(-two_pi * (qz * c.x + my * c.y + mx * c.z), &sn, &cs);
          ore += step[s] * ball * cs;
          oim += step[s] * ball * sn;
        }
      }
      // U = i O / (4 pi nu_z) * (-1)^(ky + kx) / pixel^2
      const double sgn = ((ky + kx) & 1) ? -1.0 : 1.0;
      const double f = sgn / (4.0 * 3.14159265358979323846 * nuz * g.pixel * g.pixel);
      u = make_float2(static_cast<float>(-oim * f), static_cast<float>(ore * f));
    }
    out[i] = u;
  }
}

// After the inverse DFT: the Rytov field e^v, or the Born / exact field 1 + v, in complex float.
__global__ void k_finish_fields(float2* __restrict__ v, std::size_t total, int rytov) {
  for (std::size_t i = blockIdx.x * static_cast<std::size_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<std::size_t>(gridDim.x) * blockDim.x) {
    const float2 a = v[i];
    if (rytov) {
      float sn, cs;
      sincosf(a.y, &sn, &cs);
      const float m = expf(a.x);
      v[i] = make_float2(m * cs, m * sn);
    } else {
      v[i] = make_float2(1.0f + a.x, a.y);
    }
  }
}

unsigned grid_of(std::size_t total) {
  return static_cast<unsigned>(std::min<std::size_t>((total + 255) / 256, 148u * 32u));
}

}  // namespace

std::vector<std::complex<double>> partial_wave_coefficients(double x, double m) {
  // l_max after Wiscombe (1980); the log derivative D_l(m x) = j_l'(m x) / j_l(m x) by its downward
  // recurrence D_l(z) = l / z - 1 / (D_{l+1}(z) + (l + 2) / z), started well above l_max (stable);
  // j_l(x) by Miller's downward recurrence j_{l-1} = (2l + 1) / x j_l - j_{l+1}, normalised to
  // j_0 = sin x / x; y_l(x) upwards from y_0 = -cos x / x, y_1 = y_0 / x - sin x / x (stable); the
  // derivatives f_l' = l / x f_l - f_{l+1}; then continuity of the field and its radial derivative
  // at the surface: c_l = (m D_l j_l - j_l') / (h_l' - m D_l h_l), h_l = j_l + i y_l.
  require(x > 0 && m > 0, "forward_fields: sphere radius and index must be positive");
  const int lmax = static_cast<int>(x + 4.05 * std::cbrt(x) + 2.0) + 1;
  const int start = lmax + 16 + static_cast<int>(std::sqrt(40.0 * x));
  const double mx = m * x;
  std::vector<double> d(lmax + 2, 0.0);
  double dl = 0.0;
  for (int l = start; l >= 0; --l) {
    dl = l / mx - 1.0 / (dl + (l + 2.0) / mx);
    if (l <= lmax + 1) d[l] = dl;
  }
  std::vector<double> j(lmax + 2), y(lmax + 2);
  double jp1 = 0.0, jl = 1e-300;
  for (int l = start; l >= 0; --l) {
    const double jm1 = (2.0 * l + 1.0) / x * jl - jp1;
    if (l <= lmax + 1) j[l] = jl;
    jp1 = jl;
    jl = jm1;
    if (std::abs(jl) > 1e250) {  // rescale to stay in range
      jl *= 1e-250;
      jp1 *= 1e-250;
      for (int t = l; t <= lmax + 1 && t >= 0; ++t) j[t] *= 1e-250;
    }
  }
  const double norm = (std::sin(x) / x) / j[0];
  for (double& v : j) v *= norm;
  y[0] = -std::cos(x) / x;
  y[1] = y[0] / x - std::sin(x) / x;
  for (int l = 1; l <= lmax; ++l) y[l + 1] = (2.0 * l + 1.0) / x * y[l] - y[l - 1];
  std::vector<std::complex<double>> c(lmax + 1);
  for (int l = 0; l <= lmax; ++l) {
    const std::complex<double> h(j[l], y[l]), h1(j[l + 1], y[l + 1]);
    const double dj = l / x * j[l] - j[l + 1];
    const std::complex<double> dh = l / x * h - h1;
    const double md = m * d[l];
    c[l] = (md * j[l] - dj) / (dh - md * h);
  }
  return c;
}

void render_spheres_device(const float* spheres, int k, double n_medium, double pixel, int nz, int n, float* out,
                           cudaStream_t s) {
  require(nz >= 1 && n >= 1, "render_phantom: empty shape");
  require(k >= 0 && (k == 0 || spheres != nullptr) && out != nullptr, "render_phantom: null argument");
  std::vector<double4> sph(std::max(k, 1));
  std::vector<double> index(std::max(k, 1));
  for (int i = 0; i < k; ++i) {
    const float* v = spheres + 5 * i;
    sph[i] = make_double4(v[0], v[1], v[2], static_cast<double>(v[3]) * v[3]);
    index[i] = v[4];
  }
  DevBuf<double4> d_sph(sph.size());
  DevBuf<double> d_index(index.size());
  check(cudaMemcpyAsync(d_sph.get(), sph.data(), sph.size() * sizeof(double4), cudaMemcpyHostToDevice, s), "upload");
  check(cudaMemcpyAsync(d_index.get(), index.data(), index.size() * sizeof(double), cudaMemcpyHostToDevice, s),
        "upload");
  const std::size_t total = static_cast<std::size_t>(nz) * n * n;
  k_render_spheres<<<grid_of(total), 256, 0, s>>>(d_sph.get(), d_index.get(), k, n_medium, nz, n, pixel, out);
  check_launch("render phantom");
  check(cudaStreamSynchronize(s), "render phantom");  // the tables go out of scope
}

void sphere_fields_device(const float* spheres, int k, const float* illum_fyfx, int count, double wavelength,
                          double n_medium, double na, double pixel, int n, int model, float2* out, cudaStream_t s) {
  require(n >= 4 && n % 2 == 0, "forward_fields: n must be even");
  require(model >= 0 && model <= 2, "forward_fields: unknown model");
  require(model != 2 || k == 1, "forward_fields: the exact model takes exactly one sphere");
  require(count >= 1 && illum_fyfx != nullptr && out != nullptr && (k == 0 || spheres != nullptr),
          "forward_fields: null argument");
  const double fm2 = n_medium * n_medium / (wavelength * wavelength);
  SpectrumGrid g{};
  g.fm2 = fm2;
  g.fna2 = na * na / (wavelength * wavelength);
  g.df = 1.0 / (n * pixel);
  g.pixel = pixel;
  g.km = 2.0 * std::numbers::pi / wavelength * n_medium;
  g.n = n;
  g.count = count;
  g.k = k;
  std::vector<double2> il(count);
  for (int a = 0; a < count; ++a) {
    const double fy = illum_fyfx[2 * a], fx = illum_fyfx[2 * a + 1];
    require(fy * fy + fx * fx < fm2, "forward_fields: illumination beyond n_medium / wavelength");
    il[a] = make_double2(fy, fx);
  }
  // Spheres as (centre, radius^2) plus, for the first-order models, the potential step of each over
  // the index it is painted on (the index of the earlier spheres at its centre) times its volume.
  const double k0 = 2.0 * std::numbers::pi / wavelength;
  std::vector<double4> sph(std::max(k, 1));
  std::vector<double> step(std::max(k, 1));
  for (int i = 0; i < k; ++i) {
    const float* v = spheres + 5 * i;
    sph[i] = make_double4(v[0], v[1], v[2], static_cast<double>(v[3]) * v[3]);
    double parent = n_medium;
    for (int e = i - 1; e >= 0; --e) {
      const float* w = spheres + 5 * e;
      const double dz = double(v[0]) - w[0], dy = double(v[1]) - w[1], dx = double(v[2]) - w[2];
      if (dz * dz + dy * dy + dx * dx <= double(w[3]) * w[3]) {
        parent = w[4];
        break;
      }
    }
    const double r = v[3];
    step[i] = k0 * k0 * (double(v[4]) * v[4] - parent * parent) * (4.0 / 3.0 * std::numbers::pi * r * r * r);
  }
  std::vector<double2> waves(1);
  if (model == 2) {
    const auto c = partial_wave_coefficients(g.km * spheres[3], spheres[4] / n_medium);
    waves.resize(c.size());
    for (std::size_t l = 0; l < c.size(); ++l) waves[l] = make_double2(c[l].real(), c[l].imag());
    g.waves = static_cast<int>(c.size());
  }
  DevBuf<double2> d_il(count), d_waves(waves.size());
  DevBuf<double4> d_sph(sph.size());
  DevBuf<double> d_step(step.size());
  check(cudaMemcpyAsync(d_il.get(), il.data(), il.size() * sizeof(double2), cudaMemcpyHostToDevice, s), "upload");
  check(cudaMemcpyAsync(d_sph.get(), sph.data(), sph.size() * sizeof(double4), cudaMemcpyHostToDevice, s), "upload");
  check(cudaMemcpyAsync(d_step.get(), step.data(), step.size() * sizeof(double), cudaMemcpyHostToDevice, s),
        "upload");
  check(cudaMemcpyAsync(d_waves.get(), waves.data(), waves.size() * sizeof(double2), cudaMemcpyHostToDevice, s),
        "upload");
  const std::size_t total = static_cast<std::size_t>(count) * n * n;
  k_sphere_spectra<<<grid_of(total), 256, 0, s>>>(d_il.get(), d_sph.get(), d_step.get(), d_waves.get(), g, out);
  check_launch("sphere spectra");
  fft2d(out, count, n, false, 1.0f / static_cast<float>(n * n), s);
  k_finish_fields<<<grid_of(total), 256, 0, s>>>(out, total, model == 1 ? 1 : 0);
  check_launch("finish fields");
  check(cudaStreamSynchronize(s), "forward fields");  // the tables go out of scope
}

void synthesize_holograms_device(const float2* ratio, const float* illum_fyfx, int count, int n, double pixel,
                                 double carrier_y, double carrier_x, double amplitude, float noise,
                                 unsigned long long seed, float* out, cudaStream_t s) {
  require(ratio && illum_fyfx && out, "synthesize_holograms: null argument");
  require(count >= 1 && n >= 1, "synthesize_holograms: empty stack");
  require(pixel > 0 && noise >= 0, "synthesize_holograms: pixel must be positive and noise non-negative");
  std::vector<double2> il(count);
  for (int a = 0; a < count; ++a) il[a] = make_double2(illum_fyfx[2 * a], illum_fyfx[2 * a + 1]);
  DevBuf<double2> d_il(count);
  check(cudaMemcpyAsync(d_il.get(), il.data(), count * sizeof(double2), cudaMemcpyHostToDevice, s),
        "upload illuminations");
  const std::size_t total = static_cast<std::size_t>(count) * n * n;
  const unsigned grid = static_cast<unsigned>(std::min<std::size_t>((total + 255) / 256, 148u * 32u));
  k_synthesize<<<grid, 256, 0, s>>>(ratio, d_il.get(), count, n, pixel, carrier_y, carrier_x, amplitude, noise, seed,
                                    out);
  check_launch("synthesize holograms");
  check(cudaStreamSynchronize(s), "synthesize holograms");  // d_il goes out of scope
}

}  // namespace qhk
