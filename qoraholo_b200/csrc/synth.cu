// Off-axis hologram synthesis on the device: |R + u_in * ratio|^2 + Gaussian noise, the formula of
// the reference's synthesize_holograms (src/phantom.cpp:193-221), for generating request streams
// without a host round trip. The intensity is formed in double as on the host, so noise-free
// holograms agree with the host's to float rounding. The noise comes from a counter-based generator
// (a 64-bit mix of (seed, pixel) and the Box-Muller transform), not from std::mt19937_64: the draws
// differ from the host's, their distribution (zero mean, standard deviation `noise`) is the same,
// and a seed gives the same holograms on every run and device.
#include <cmath>
#include <numbers>
#include <vector>

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

}  // namespace

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
