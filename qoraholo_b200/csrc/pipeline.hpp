// Device side of qoraholo::Pipeline (pipeline.cu).
#pragma once

#include "field.hpp"
#include "odt.hpp"
#include "unwrap.hpp"

namespace qhk {

// Stage times of the last process() in milliseconds (qoraholo::PipelineTimings).
struct PipelineTimes {
  double upload = 0, fields = 0, rytov = 0, fft2 = 0, clear = 0, mapping = 0, normalize = 0, solve = 0,
         finish = 0, download = 0, total = 0;
};

class PipelinePlan {
 public:
  PipelinePlan(const CropPlan& crop, int count, int upload_chunks, const OdtConfig& odt, const float* illum_fyfx);

  // Background holograms (count, N, N) on the host; their fields stay on the device.
  void set_background(const float* host_bg);
  // Page-locked input (count, N, N) and output (nz, n, n) buffers.
  [[nodiscard]] float* input() const { return input_.get(); }
  [[nodiscard]] const float* output() const { return output_.get(); }
  // input() -> output(), synchronous, with stage timings.
  void process();
  // Holograms already on the device -> index on the device, asynchronous on `s` (no host copies).
  void process_device(const float* d_holo, float* d_index, cudaStream_t s);

  [[nodiscard]] double filled() const { return filled_; }
  [[nodiscard]] const PipelineTimes& timings() const { return timings_; }
  [[nodiscard]] std::size_t device_bytes() const;
  [[nodiscard]] bool has_background() const { return has_background_; }
  [[nodiscard]] const OdtPlan& odt() const { return odt_; }
  [[nodiscard]] const CropPlan& crop() const { return crop_; }
  [[nodiscard]] int count() const { return count_; }

 private:
  enum { kStart, kFields, kRytov, kDownloaded = kRytov + 1 + OdtPlan::kMarks, kMarks };
  void compute(const float* d_holo, bool chunked_upload, float* d_index, cudaStream_t s);

  CropPlan crop_;
  int count_;
  int chunk_;
  int chunks_;
  Stream compute_;
  Stream copy_;
  FieldPlan field_;
  UnwrapPlan unwrap_;
  OdtPlan odt_;
  PinnedBuf<float> input_;
  PinnedBuf<float> output_;
  PinnedBuf<unsigned long long> filled_host_;
  DevBuf<float> holo_;
  DevBuf<float2> background_;
  DevBuf<float2> fields_;
  DevBuf<float> psi_;
  DevBuf<float> logamp_;
  DevBuf<float> phi_;
  DevBuf<float> index_;
  std::vector<Event> chunk_done_;
  StageClock clock_;
  PipelineTimes timings_;
  double filled_ = 0;
  bool has_background_ = false;
};

}  // namespace qhk
