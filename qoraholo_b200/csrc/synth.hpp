// Hologram synthesis on the device (synth.cu).
#pragma once

#include <complex>
#include <vector>

#include "qhk_util.cuh"

namespace qhk {

// ratio: (count, n, n) complex64 field ratios on the device -> out: (count, n, n) float32 holograms
// on the device; illum_fyfx on the host. Returns when done.
void synthesize_holograms_device(const float2* ratio, const float* illum_fyfx, int count, int n, double pixel,
                                 double carrier_y, double carrier_x, double amplitude, float noise,
                                 unsigned long long seed, float* out, cudaStream_t s);

// Spheres as rows of (z, y, x, radius, index), micrometres from the volume centre, painted in order.
// Index at the voxel centres of an (nz, n, n) volume of `pixel` spacing -> out (device). Synchronous.
void render_spheres_device(const float* spheres, int k, double n_medium, double pixel, int nz, int n, float* out,
                           cudaStream_t s);
// Analytic fields of the spheres at z = 0 for each illumination -> out (count, n, n) complex (device):
// model 0 first Born (1 + v), 1 Rytov (e^v), 2 exact partial waves of one sphere (1 + v). Synchronous.
void sphere_fields_device(const float* spheres, int k, const float* illum_fyfx, int count, double wavelength,
                          double n_medium, double na, double pixel, int n, int model, float2* out, cudaStream_t s);
// Scattering coefficients c_l, l = 0..l_max, of a homogeneous sphere of size parameter x = k_m R and
// relative index m for the scalar Helmholtz equation.
std::vector<std::complex<double>> partial_wave_coefficients(double x, double m);

}  // namespace qhk
