// Unwrap / Rytov plan of the CUDA backend (unwrap.cu).
#pragma once

#include <vector>

#include "graph.hpp"
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

// Least-squares unwrap of an uneven batch: `count` images, image i of its own (even) size ny[i] x
// nx[i], packed one after another in the input and output buffers (image i starts at offset(i) =
// the pixel count of images 0 .. i-1). Each of the five passes is ONE launch for the whole batch:
// persistent CTAs (as many as are resident at once) take (image, tile) items off a device queue,
// largest images first, and run the tile code of the stacked plan above for that image's size, so
// every image's result is bitwise the one UnwrapPlan gives for it. unwrap_graph replays the five
// launches as one captured CUDA graph.
class UnwrapBatchPlan {
 public:
  UnwrapBatchPlan(const int* ny, const int* nx, int count);
  ~UnwrapBatchPlan();
  UnwrapBatchPlan(const UnwrapBatchPlan&) = delete;
  UnwrapBatchPlan& operator=(const UnwrapBatchPlan&) = delete;

  void unwrap(const float* psi, float* phi, cudaStream_t s);
  void unwrap_graph(const float* psi, float* phi, cudaStream_t s);

  [[nodiscard]] int count() const { return static_cast<int>(offsets_.size()); }
  [[nodiscard]] std::size_t offset(int i) const { return offsets_.at(i); }
  [[nodiscard]] std::size_t total() const { return total_; }
  [[nodiscard]] std::size_t device_bytes() const;
  [[nodiscard]] std::uint64_t graph_replays() const { return graph_.replays(); }

 private:
  struct Pass {
    void* items = nullptr;  // int2 (image, tile) on the device
    int n = 0;
    std::size_t smem = 0;
    unsigned grid = 0;
  };
  std::vector<std::size_t> offsets_;
  std::size_t total_ = 0;
  std::vector<DevBuf<float2>> dtw_;  // per distinct side length
  std::vector<DevBuf<float>> cos_;
  DevBuf<unsigned char> images_;     // per-image descriptors
  DevBuf<int2> items_;               // all passes' items, concatenated
  DevBuf<int> counters_;             // one queue head per pass
  DevBuf<float> d1_;
  DevBuf<double> partial_;
  DevBuf<float2> consts_;
  // Passes 1-5 (staged tiles for passes 1-3), then passes 1-3 of the images whose lines run on the
  // register engine: each has its own queue, so that each kernel holds only its own tiles' registers.
  Pass pass_[8];
  CapturedWork graph_;
  bool warmed_ = false;
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
