// Unwrap / Rytov plan of the CUDA backend (unwrap.cu).
#pragma once

#include "qhk_internal.hpp"

namespace qhk {

class UnwrapPlan {
 public:
  UnwrapPlan(int count, int ny, int nx);

  // psi (count, ny, nx) wrapped phase -> phi, congruent to psi modulo 2 pi (cpu::unwrap).
  void unwrap(const float* psi, float* phi, cudaStream_t s);
  // Rytov field logamp + i (unwrap(psi) - 2 pi m) into out; phi_scratch holds count*ny*nx floats.
  void rytov(const float* psi, const float* logamp, float* phi_scratch, float2* out, cudaStream_t s);

  [[nodiscard]] std::size_t device_bytes() const;

 private:
  // Least-squares solve into phi (without the constant) and the per-image constants.
  void solve(const float* psi, float* phi, cudaStream_t s);

  int count_, ny_, nx_;
  int rows_ = 16;
  int nblk_ = 1;
  DevBuf<float2> dtw_y_, dtw_x_;
  DevBuf<float> cos_y_, cos_x_;
  DevBuf<float> d1_;
  DevBuf<double> partial_;
  DevBuf<float2> consts_;  // (congruence constant, 2 pi shift) per image
};

// Least-squares unwrap of count images (ny, nx) from psi into phi (both on the device) with no
// allocation: scratch and tables live in a file-scope device array (unwrap.cu); at most 4096 images
// of at most 1024 x 1024 and 4194304 pixels per call. Asynchronous on `s`; calls that overlap on the
// GPU share the scratch and race.
void unwrap_noalloc(const float* psi, float* phi, int count, int ny, int nx, cudaStream_t s);

// out = sample / background (background: one image, or one per image when per_image).
void field_ratio(const float2* sample, const float2* bg, std::size_t plane, bool per_image, std::size_t total,
                 float2* out, cudaStream_t s);

// psi = arg(r), logamp = log |r| of a formed ratio.
void split_ratio(const float2* ratio, std::size_t total, float* psi, float* logamp, cudaStream_t s);

}  // namespace qhk
