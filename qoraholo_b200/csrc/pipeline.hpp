// Device side of qoraholo::Pipeline (pipeline.cu).
#pragma once

#include "field.hpp"
#include "graph.hpp"
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
  // `own_io`: allocate the page-locked input / output buffers and the resident background fields
  // (the Pipeline form). Without them the plan is a serving workspace: device buffers only, with the
  // background fields passed to enqueue().
  PipelinePlan(const CropPlan& crop, int count, int upload_chunks, const OdtConfig& odt, const float* illum_fyfx,
               bool own_io = true);

  // Background holograms (count, N, N) on the host; their fields stay on the device.
  void set_background(const float* host_bg);
  // Page-locked input (batch * count, N, N) and output (batch, nz, n, n) buffers.
  [[nodiscard]] float* input() const { return input_.get(); }
  [[nodiscard]] const float* output() const { return output_.get(); }
  // input() -> output(), synchronous, with stage timings.
  void process();
  // Caller memory (pageable or page-locked) holograms (batch * count, N, N) -> caller memory
  // volume(s) (batch, nz, n, n), synchronous, with stage timings. Each upload chunk is copied into
  // the page-locked input by the host copy threads just before its transfer is queued, so the copy
  // of chunk k overlaps the transfer and field passes of the chunks before it; the pages of
  // `index` are faulted in while the solver runs, and the volume comes back in kOutParts parts,
  // each copied out as soon as it has landed while the next part is in flight. Page-locked caller
  // buffers are transferred directly, without staging or host copies. Either pointer may be null:
  // the input is then taken from input(), the volume left in output().
  void process_host(const float* holograms, float* index);
  // `items` inputs of process_host back to back -> `items` outputs back to back, caller memory,
  // synchronous. Streamed: the upload of input i + 1 and the download of output i - 1 run while
  // input i is solved (two device volumes alternate, the downloads on their own stream), and the host
  // stages the next input and copies out the previous output meanwhile. Each output is bitwise that
  // of process_host on its input; timings() then holds only the total.
  void process_stream(const float* holograms, float* index, int items);
  // Holograms already on the device -> index on the device, asynchronous on `s` (no host copies).
  void process_device(const float* d_holo, float* d_index, cudaStream_t s);
  // The same replayed as one CUDA graph (captured on the second call for these buffers; the first
  // call runs directly so that lazy setup happens outside the capture). No stage timings.
  void process_device_graph(const float* d_holo, float* d_index, cudaStream_t s);

  // Serving-workspace forms, asynchronous on `s`, no stage marks (so they can be graph-captured):
  // background holograms (device) -> demodulated background fields `bg_out` (count, m, m); and
  // holograms (device) -> index (device) against background fields `bg`. The filled-voxel count of
  // the last enqueue is odt().filled().
  void enqueue_background(const float* d_bg_holo, float2* bg_out, cudaStream_t s);
  void enqueue(const float* d_holo, const float2* bg, float* d_index, cudaStream_t s);
  // The plan's own stream, and the device buffers the serving loop copies into / out of.
  [[nodiscard]] cudaStream_t stream() const { return compute_.get(); }
  [[nodiscard]] float* holo_buffer() const { return holo_.get(); }
  [[nodiscard]] float* index_buffer() const { return index_.get(); }
  // Of one request (one stack of `count` holograms / fields).
  [[nodiscard]] std::size_t hologram_floats() const {
    return static_cast<std::size_t>(count_) * crop_.n * crop_.n;
  }
  [[nodiscard]] std::size_t field_elems() const { return static_cast<std::size_t>(count_) * crop_.out * crop_.out; }

  [[nodiscard]] double filled() const { return filled_; }
  // Fails with kTimeout if a bounded device wait of this plan ran out since the last check (reads
  // the plan's wait counter; synchronises `s`). The host runs check after their own synchronise;
  // callers of the device forms call this when they want to know.
  void check_device_waits(cudaStream_t s);
  // Test hook: a bounded wait that nothing completes, counted in this plan's wait counter on its
  // own stream (the form of every wait of the two-step FGP kernel), then check_device_waits.
  void wait_probe(int polls);
  [[nodiscard]] const PipelineTimes& timings() const { return timings_; }
  [[nodiscard]] std::size_t device_bytes() const;
  [[nodiscard]] bool has_background() const { return has_background_; }
  [[nodiscard]] const OdtPlan& odt() const { return odt_; }
  OdtPlan& odt() { return odt_; }
  [[nodiscard]] const CropPlan& crop() const { return crop_; }
  [[nodiscard]] int count() const { return count_; }
  // Requests of this geometry per run (OdtConfig::batch): inputs, fields and volumes are that many
  // stacks one after another; the background fields are one stack.
  [[nodiscard]] int batch() const { return batch_; }

 private:
  enum { kStart, kFields, kRytov, kDownloaded = kRytov + 1 + OdtPlan::kMarks, kMarks };
  static constexpr int kOutParts = 8;
  // chunked_upload: the holograms come from input_ in chunks on the copy stream, each first
  // copied there from `host_src` when that is given (or transferred straight from it when it is
  // page-locked). solve_slot >= 0 (process_stream's volume slot, without marks): the reconstruction
  // from the fields runs as that slot's CUDA graph, directly on the slot's first use.
  void compute(const float* d_holo, bool chunked_upload, const float2* bg, float* d_index, cudaStream_t s,
               bool marks, const float* host_src = nullptr, bool host_src_locked = false, int solve_slot = -1);

  CropPlan crop_;
  int count_;
  int batch_;
  int chunk_;
  int chunks_;
  Stream compute_;
  Stream copy_;
  FieldPlan field_;
  UnwrapPlan unwrap_;
  OdtPlan odt_;
  PinnedBuf<float> input_;
  PinnedBuf<float> output_;
  PinnedBuf<unsigned long long> filled_host_;  // batch_ filled counts, then the plan's wait counter
  unsigned long long waits_seen_ = 0;            // the wait counter at the last check
  DevBuf<float> holo_;
  DevBuf<float2> background_;
  DevBuf<float2> fields_;
  DevBuf<float> psi_;
  DevBuf<float> logamp_;
  DevBuf<float> phi_;
  DevBuf<float> index_;
  DevBuf<float> index_alt_;  // the second device volume of process_stream, allocated by its first call
  Stream down_;              // process_stream's downloads
  Event holo_free_;          // on compute_: the field passes have read holo_ (the next upload may start)
  Event solved_[2];          // process_stream: volume slot k written
  Event downloaded_[2];      // process_stream: volume slot k read back
  std::vector<Event> chunk_done_;
  std::vector<Event> part_done_;
  StageClock clock_;
  CapturedWork graph_;
  bool graph_warm_ = false;
  CapturedWork solve_graph_[2];  // process_stream: the solve into volume slot k, replayed
  bool solve_warm_[2] = {false, false};
  PipelineTimes timings_;
  double filled_ = 0;
  bool has_background_ = false;
};

}  // namespace qhk
