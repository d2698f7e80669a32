// BPM plan of the CUDA backend (bpm.cu).
#pragma once

#include <vector>

#include "qhk_internal.hpp"

namespace qhk {

// Per-illumination tables (count, n, n), lateral bins in FFT order, computed in double on the
// host and rounded to float: propagator over one voxel, back-propagator times the detection
// pupil for the last slice, obliquity weight; and the screen phase per unit contrast and the
// Lipschitz constant of the data term (the reference's bpm_tables, src/bpm.cpp:10-60).
struct BpmTablesHost {
  int n = 0, nz = 0, count = 0;
  float phase = 0;
  float lipschitz = 0;
  std::vector<float2> step, last;
  std::vector<float> q;
};

BpmTablesHost bpm_tables(int n, int nz, const float* illum_fyfx, int count, float wavelength, float n_medium,
                         float na, float pixel, bool obliquity);

class BpmPlan {
 public:
  // chunk: illuminations per device pass; store: keep the envelope in front of every screen for
  // the adjoint. checkpoint_every = K > 0 instead keeps only the spectrum entering every K-th
  // slice, for every illumination (ceil(nz / K) planes per illumination); the adjoint then
  // recomputes each segment's K envelopes from its checkpoint before sweeping it backwards.
  BpmPlan(const BpmTablesHost& t, int chunk, bool store, int checkpoint_every = 0);

  // Envelopes at z = 0 of illuminations first .. first + nb - 1 for contrast x (device), left in
  // fields() (normalised).
  void forward(const float* x, int first, int nb, cudaStream_t s);
  // fields() <- fields() - data[first ..], and *d_loss += sum |.|^2 (double, on the device).
  double residual(const float2* data, int first, int nb, double* d_loss, cudaStream_t s);
  // grad += gscale * J^T r for the chunk of the last forward(); r is fields() (after residual())
  // or `residual` when given (device, nb planes).
  void adjoint(const float* x, const float2* residual, int first, int nb, float gscale, float* grad, cudaStream_t s);

  [[nodiscard]] float2* fields() const { return w_.get(); }
  [[nodiscard]] std::size_t device_bytes() const;
  [[nodiscard]] int checkpoint_every() const { return every_; }

 private:
  void fft2(const float2* src, float2* dst, bool forward, int nb, int mode, const void* args, cudaStream_t s);
  // Envelopes of slices k0 .. k1-1 of the chunk into env_, from the checkpoint of slice k0.
  void recompute(const float* x, int first, int nb, int k0, int k1, cudaStream_t s);

  const BpmTablesHost& t_;
  int chunk_;
  bool store_on_;
  std::size_t plane_ = 0;
  DevBuf<float2> step_, last_;
  DevBuf<float> q_;
  DevBuf<float2> s_, w_, stored_;
  DevBuf<double> partial_;
  int every_ = 0;
  DevBuf<float2> ckpt_, env_, rs_, rw_;  // checkpoint mode
  DevBuf<float> gpart_;                   // gradient sums per group of views (adjoint, register engine)
};

// x = ri - n_medium (optionally clamped at 0), and back.
void contrast(const float* ri, float n_medium, std::size_t total, float* x, bool clamp, cudaStream_t s);
void add_medium(const float* x, float n_medium, std::size_t total, float* ri, cudaStream_t s);

// Proximal gradient inversion (FISTA over all illuminations, or passes over batches) of the
// contrast d_x (device, updated in place); d_loss[it] receives sum |bpm(x) - fields|^2 of each
// iteration (unscaled); bounded device waits of its TV steps that run out are counted in the device
// word *d_waits (may be null: the library-wide counter). Synchronises the stream.
void bpm_solve(const BpmTablesHost& t, const float2* d_fields, float* d_x, int iterations, int batch, float step,
               float tv_weight, int tv_inner, double* d_loss, cudaStream_t s,
               unsigned long long* d_waits = nullptr);

}  // namespace qhk
