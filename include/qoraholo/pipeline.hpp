// Holograms -> refractive index with all device state allocated once. Declarations as in the
// reference's include/qoraholo/pipeline.hpp.
#pragma once

#include <array>
#include <cstddef>
#include <memory>
#include <span>
#include <vector>

#include "qoraholo/array.hpp"
#include "qoraholo/field.hpp"
#include "qoraholo/odt.hpp"

namespace qoraholo {

struct PipelineOptions {
  int count = 0;          // holograms per stack
  int hologram_size = 0;  // side N
  FieldOptions field;     // field.center (the reference carrier) is required
  std::vector<Illumination> illuminations;
  Geometry geometry;      // field pixel, also the voxel side
  OdtOptions odt;
  int upload_chunks = 1;  // parts of the host -> device copy that overlap field extraction
};

// Milliseconds of each stage of the last process(); device event intervals except `total`.
struct PipelineTimings {
  double upload = 0;
  double fields = 0;
  double rytov = 0;
  double fft2 = 0;
  double clear = 0;
  double mapping = 0;
  double normalize = 0;
  double solve = 0;
  double finish = 0;
  double download = 0;
  double total = 0;
};

class Pipeline {
 public:
  explicit Pipeline(PipelineOptions options);
  ~Pipeline();
  Pipeline(Pipeline&&) noexcept;
  Pipeline& operator=(Pipeline&&) noexcept;

  void set_background(const Array3<float>& backgrounds);
  // Page-locked (count, N, N) input buffer.
  [[nodiscard]] std::span<float> input();
  void process();  // needs set_background() first
  // Page-locked (nz, n, n) result of the last process().
  [[nodiscard]] std::span<const float> output() const;
  [[nodiscard]] double filled() const;
  [[nodiscard]] OdtResult run(const Array3<float>& holograms);
  // The same into caller memory: holograms (count, N, N) -> index (nz, n, n), no intermediate
  // host buffers of the caller's size (qhk_pipeline_run).
  void run(std::span<const float> holograms, std::span<float> index);
  // `items` stacks back to back -> `items` volumes back to back, the transfers of one stack
  // overlapping the solve of the next (qhk_pipeline_run_stream). filled() is the last stack's.
  void run_stream(std::span<const float> holograms, std::span<float> index, int items);

  [[nodiscard]] const PipelineTimings& timings() const;
  [[nodiscard]] double setup_ms() const;
  [[nodiscard]] std::size_t device_bytes() const;
  [[nodiscard]] std::array<int, 3> output_shape() const;

  class Impl;

 private:
  std::unique_ptr<Impl> impl_;
};

}  // namespace qoraholo
