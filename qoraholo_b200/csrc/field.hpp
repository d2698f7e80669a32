// Field-extraction plan of the CUDA backend (field.cu).
#pragma once

#include "qhk_internal.hpp"

namespace qhk {

// Integer crop centre, radius and output side (the reference's CropPlan, src/backends.hpp:20-25,
// resolved as crop_plan does, src/api.cpp:52-60), plus the hologram side n.
struct CropPlan {
  int n = 0;
  int cy = 0;
  int cx = 0;
  float radius = 0;
  int out = 0;
};

CropPlan make_crop(int n, float cy, float cx, float radius, int output_size);

class FieldPlan {
 public:
  FieldPlan(const CropPlan& plan, int count);

  // Passes 1-2 for holograms first .. first + valid - 1; `holo` points at hologram `first`.
  void spectra(const float* holo, int first, int valid, cudaStream_t s);
  // Pass 3 for all holograms: mode 0 writes demodulated fields (count, m, m); mode 1 writes the
  // phase and log-amplitude of the ratio to the background fields `bg`.
  // bg_count > 0: `bg` holds that many images and image i uses background i % bg_count (a stack of
  // several requests of one geometry). images > 0: only the first `images` images.
  void finish(int mode, float2* field, const float2* bg, float* psi, float* logamp, cudaStream_t s,
              int bg_count = 0, int images = 0);
  // All three passes, demodulated fields.
  void fields(const float* holo, float2* out, cudaStream_t s);

  [[nodiscard]] const CropPlan& plan() const { return plan_; }
  [[nodiscard]] int count() const { return count_; }
  [[nodiscard]] std::size_t device_bytes() const;

 private:
  CropPlan plan_;
  int count_;
  float r2_ = 0;
  int dxlo_ = 0;
  int W_ = 0;
  DevBuf<float2> t1_;
  DevBuf<float2> t2_;
};

// Sideband search of find_sideband (src/cpu/field.cpp:25-60) on hologram `holo` (n x n, device):
// its half spectrum into `half` (n x (n/2+1)), and the peak magnitude and index y * n + x of the
// centred spectrum into d_mag / d_idx (-1 when nothing lies outside the DC disc).
void sideband_peak(const float* holo, int n, float dc_exclusion, float2* half, float* d_mag, int* d_idx,
                   cudaStream_t s);

}  // namespace qhk
