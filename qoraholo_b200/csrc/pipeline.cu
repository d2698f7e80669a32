// Holograms -> refractive index with everything allocated once: the device side of
// qoraholo::Pipeline. Replaces the reference's CudaPipeline (src/cuda/pipeline.cu:12-147).
//
// process(): the sample holograms go host -> device in `upload_chunks` parts on a copy stream;
// the field passes of each part start as soon as its copy has landed (event wait), so the copy
// overlaps field extraction. The last field pass forms the ratio to the resident background
// fields and its phase / log-amplitude directly; then the unwrap passes, the Rytov assembly,
// the ODT plan, and the device -> host copy of the volume into page-locked memory in parts.
// process_host() does the same from and into caller memory: the host copy threads fill each
// upload chunk's staging just before its transfer, and copy each downloaded part out as it lands.
// Stage times are event intervals on the compute stream, read after it finishes (the upload time
// then includes the host staging of the chunks).
#include <chrono>
#include <exception>

#include "host_copy.hpp"
#include "pipeline.hpp"
#include "nvtx.hpp"

namespace qhk {

namespace {

int checked_chunk(int count, int upload_chunks) {
  require(count >= 1, "Pipeline: count must be positive");
  require(upload_chunks >= 1 && upload_chunks <= count, "Pipeline: upload_chunks must be between 1 and count");
  return (count + upload_chunks - 1) / upload_chunks;
}

// Waits for every stream of a host-buffer run when an exception leaves the run, so that no transfer
// queued into or out of caller memory or the page-locked staging is still in flight once the caller
// gets control back (and may free or reuse that memory). Errors of the waits themselves are dropped:
// the exception in flight already reports the failure.
class DrainOnThrow {
 public:
  DrainOnThrow(cudaStream_t a, cudaStream_t b, cudaStream_t c)
      : streams_{a, b, c}, pending_(std::uncaught_exceptions()) {}
  DrainOnThrow(const DrainOnThrow&) = delete;
  DrainOnThrow& operator=(const DrainOnThrow&) = delete;
  ~DrainOnThrow() {
    if (std::uncaught_exceptions() <= pending_) return;
    for (cudaStream_t st : streams_) {
      if (st != nullptr) (void)cudaStreamSynchronize(st);
    }
  }

 private:
  cudaStream_t streams_[3];
  int pending_;
};

}  // namespace

PipelinePlan::PipelinePlan(const CropPlan& crop, int count, int upload_chunks, const OdtConfig& odt,
                           const float* illum_fyfx, bool own_io)
    : crop_(crop),
      count_(count),
      batch_(odt.batch),
      chunk_(checked_chunk(count * odt.batch, upload_chunks)),
      chunks_((count * odt.batch + chunk_ - 1) / chunk_),
      field_(crop, count * odt.batch),
      unwrap_(count * odt.batch, crop.out, crop.out),
      odt_(odt, illum_fyfx),
      clock_(kMarks) {
  require(odt.grid.n == crop.out, "Pipeline: volume side must equal the field side");
  const std::size_t image = static_cast<std::size_t>(crop.n) * crop.n;
  const std::size_t field = static_cast<std::size_t>(count) * crop.out * crop.out;
  const std::size_t b = batch_;
  if (own_io) {
    input_ = PinnedBuf<float>(b * count * image);
    output_ = PinnedBuf<float>(b * odt_.volume());
    filled_host_ = PinnedBuf<unsigned long long>(b + 1);
    background_.reset(field);
  }
  holo_.reset(b * count * image);
  fields_.reset(b * field);
  psi_.reset(b * field);
  logamp_.reset(b * field);
  phi_.reset(b * field);
  index_.reset(b * odt_.volume());
  for (int k = 0; k < chunks_; ++k) chunk_done_.emplace_back();
  for (int k = 0; k < kOutParts; ++k) part_done_.emplace_back();
}

std::size_t PipelinePlan::device_bytes() const {
  return field_.device_bytes() + unwrap_.device_bytes() + odt_.device_bytes() + holo_.bytes() + background_.bytes() +
         fields_.bytes() + psi_.bytes() + logamp_.bytes() + phi_.bytes() + index_.bytes();
}

void PipelinePlan::set_background(const float* host_bg) {
  require(background_.get() != nullptr, "Pipeline: serving workspaces take their background fields per call");
  const cudaStream_t s = compute_.get();
  const std::size_t image = static_cast<std::size_t>(crop_.n) * crop_.n;
  check(cudaMemcpyAsync(holo_.get(), host_bg, count_ * image * sizeof(float), cudaMemcpyHostToDevice, s),
        "upload backgrounds");
  field_.spectra(holo_.get(), 0, count_, s);
  field_.finish(0, background_.get(), nullptr, nullptr, nullptr, s, 0, count_);
  check(cudaStreamSynchronize(s), "set_background");
  has_background_ = true;
}

void PipelinePlan::enqueue_background(const float* d_bg_holo, float2* bg_out, cudaStream_t s) {
  field_.spectra(d_bg_holo, 0, count_, s);
  field_.finish(0, bg_out, nullptr, nullptr, nullptr, s, 0, count_);
}

void PipelinePlan::enqueue(const float* d_holo, const float2* bg, float* d_index, cudaStream_t s) {
  compute(d_holo, false, bg, d_index, s, false);
}

void PipelinePlan::compute(const float* d_holo, bool chunked_upload, const float2* bg, float* d_index, cudaStream_t s,
                           bool marks, const float* host_src, bool host_src_locked, int solve_slot) {
  const std::size_t image = static_cast<std::size_t>(crop_.n) * crop_.n;
  if (marks) clock_.mark(kStart, s);
  const int images = count_ * batch_;
  if (chunked_upload) {
    const cudaStream_t c = copy_.get();
    // holo_ is free once the field passes of the previous input have read it.
    check(cudaStreamWaitEvent(c, holo_free_.get(), 0), "cudaStreamWaitEvent");
    for (int k = 0; k < chunks_; ++k) {
      const int first = k * chunk_;
      const int valid = std::min(chunk_, images - first);
      float* dst = holo_.get() + first * image;
      const float* src = input_.get() + first * image;
      if (host_src && host_src_locked) {
        src = host_src + first * image;  // page-locked caller memory: transferred directly
      } else if (host_src) {
        chunk_done_[k].synchronize();  // the previous input's transfer out of this staging chunk
        HostCopier::shared().copy(input_.get() + first * image, host_src + first * image, valid * image * sizeof(float));
      }
      check(cudaMemcpyAsync(dst, src, valid * image * sizeof(float), cudaMemcpyHostToDevice, c), "upload holograms");
      chunk_done_[k].record(c);
      check(cudaStreamWaitEvent(s, chunk_done_[k].get(), 0), "cudaStreamWaitEvent");
      field_.spectra(dst, first, valid, s);
    }
    holo_free_.record(s);
  } else {
    field_.spectra(d_holo, 0, images, s);
  }
  {
    const NvtxRange r("qhk:fields");
    field_.finish(1, nullptr, bg, psi_.get(), logamp_.get(), s, count_);
  }
  if (marks) clock_.mark(kFields, s);
  {
    const NvtxRange r("qhk:rytov");
    unwrap_.rytov(psi_.get(), logamp_.get(), phi_.get(), fields_.get(), s);
  }
  if (marks) clock_.mark(kRytov, s);
  if (marks) {
    odt_.run_marked(fields_.get(), d_index, s, &clock_, kRytov + 1);
  } else if (solve_slot >= 0 && solve_warm_[solve_slot]) {
    // The same launches as odt_.run, replayed as one graph: about 2 us of launch overhead saved per
    // kernel, some 200 kernels per reconstruction.
    solve_graph_[solve_slot].run({fields_.get(), d_index}, s,
                                 [&](cudaStream_t c) { odt_.run(fields_.get(), d_index, c); });
  } else {
    odt_.run(fields_.get(), d_index, s);  // a slot's first solve also runs any tuning outside capture
    if (solve_slot >= 0) solve_warm_[solve_slot] = true;
  }
}

void PipelinePlan::process() { process_host(nullptr, nullptr); }

void PipelinePlan::process_host(const float* holograms, float* index) {
  if (!has_background_) fail(kLogicError, "Pipeline: set_background() first");
  const auto t0 = std::chrono::steady_clock::now();
  const cudaStream_t s = compute_.get();
  const DrainOnThrow drain(copy_.get(), s, down_.get());
  const std::size_t image = static_cast<std::size_t>(crop_.n) * crop_.n;
  const float* src = holograms == input_.get() ? nullptr : holograms;
  const bool src_locked = src && is_page_locked(src, static_cast<std::size_t>(batch_) * count_ * image * sizeof(float));
  compute(nullptr, true, background_.get(), index_.get(), s, true, src, src_locked);
  const std::size_t total = static_cast<std::size_t>(batch_) * odt_.volume();
  // Page-locked caller output: the device writes it directly (no staging, no host copy).
  const bool dst_locked = index && index != output_.get() && is_page_locked(index, total * sizeof(float));
  float* const down = dst_locked ? index : output_.get();
  const std::size_t part = (total + kOutParts - 1) / kOutParts;
  const auto part_len = [&](int j) {
    const std::size_t off = j * part;
    return off < total ? std::min(part, total - off) : std::size_t{0};
  };
  for (int j = 0; j < kOutParts; ++j) {
    if (part_len(j) > 0) {
      check(cudaMemcpyAsync(down + j * part, index_.get() + j * part, part_len(j) * sizeof(float),
                            cudaMemcpyDeviceToHost, s),
            "download index");
    }
    part_done_[j].record(s);
  }
  check(cudaMemcpyAsync(filled_host_.get(), odt_.filled(), batch_ * sizeof(unsigned long long),
                        cudaMemcpyDeviceToHost, s),
        "download filled");
  check(cudaMemcpyAsync(filled_host_.get() + batch_, odt_.wait_count(), sizeof(unsigned long long),
                        cudaMemcpyDeviceToHost, s),
        "download wait count");
  clock_.mark(kDownloaded, s);
  if (index != nullptr && index != output_.get() && !dst_locked) {
    HostCopier& copier = HostCopier::shared();
    copier.touch(index, total * sizeof(float));  // while the device works
    for (int j = 0; j < kOutParts; ++j) {
      part_done_[j].synchronize();
      copier.copy(index + j * part, output_.get() + j * part, part_len(j) * sizeof(float));
    }
  }
  check(cudaStreamSynchronize(s), "process");
  if (filled_host_.get()[batch_] != waits_seen_) {
    waits_seen_ = filled_host_.get()[batch_];
    fail(kTimeout, wait_timeout_message("Pipeline"));
  }
  filled_ = static_cast<double>(*filled_host_.get()) / static_cast<double>(odt_.volume());
  const int o = kRytov + 1;
  timings_.upload = chunk_done_.back().since_event(clock_.event(kStart));
  timings_.fields = clock_.ms(kStart, kFields);
  timings_.rytov = clock_.ms(kFields, kRytov);
  timings_.fft2 = clock_.ms(kRytov, o + OdtPlan::kMarkFft2);
  timings_.clear = clock_.ms(o + OdtPlan::kMarkFft2, o + OdtPlan::kMarkClear);
  timings_.mapping = clock_.ms(o + OdtPlan::kMarkClear, o + OdtPlan::kMarkMapping);
  timings_.normalize = clock_.ms(o + OdtPlan::kMarkMapping, o + OdtPlan::kMarkNormalize);
  timings_.solve = clock_.ms(o + OdtPlan::kMarkNormalize, o + OdtPlan::kMarkSolve);
  timings_.finish = clock_.ms(o + OdtPlan::kMarkSolve, o + OdtPlan::kMarkFinish);
  timings_.download = clock_.ms(o + OdtPlan::kMarkFinish, kDownloaded);
  timings_.total = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

void PipelinePlan::process_stream(const float* holograms, float* index, int items) {
  if (!has_background_) fail(kLogicError, "Pipeline: set_background() first");
  require(input_.get() != nullptr, "Pipeline: serving workspaces have no host stream");
  require(holograms != nullptr && index != nullptr && items >= 1, "Pipeline: stream needs inputs and outputs");
  const auto t0 = std::chrono::steady_clock::now();
  const cudaStream_t s = compute_.get();
  const cudaStream_t d = down_.get();
  const DrainOnThrow drain(copy_.get(), s, d);
  const std::size_t in_item = static_cast<std::size_t>(batch_) * count_ * crop_.n * crop_.n;
  const std::size_t out_item = static_cast<std::size_t>(batch_) * odt_.volume();
  const bool src_locked = is_page_locked(holograms, items * in_item * sizeof(float));
  const bool dst_locked = is_page_locked(index, items * out_item * sizeof(float));
  if (index_alt_.get() == nullptr) index_alt_.reset(out_item);
  float* const slot[2] = {index_.get(), index_alt_.get()};
  const std::size_t part = (out_item + kOutParts - 1) / kOutParts;
  const auto part_len = [&](int j) {
    const std::size_t off = j * part;
    return off < out_item ? std::min(part, out_item - off) : std::size_t{0};
  };
  HostCopier& copier = HostCopier::shared();
  // Output i from the page-locked staging into the caller's memory, part by part as each lands.
  const auto collect = [&](int i) {
    if (dst_locked) return;
    float* const dst = index + i * out_item;
    for (int j = 0; j < kOutParts; ++j) {
      part_done_[j].synchronize();
      copier.copy(dst + j * part, output_.get() + j * part, part_len(j) * sizeof(float));
    }
  };
  for (int i = 0; i < items; ++i) {
    const int k = i % 2;
    // Slot k was last read back by the download of output i - 2.
    if (i >= 2) check(cudaStreamWaitEvent(s, downloaded_[k].get(), 0), "cudaStreamWaitEvent");
    compute(nullptr, true, background_.get(), slot[k], s, false, holograms + i * in_item, src_locked, k);
    check(cudaMemcpyAsync(filled_host_.get(), odt_.filled(), batch_ * sizeof(unsigned long long),
                          cudaMemcpyDeviceToHost, s),
          "download filled");
    solved_[k].record(s);
    // While the device solves input i: the host copies out output i - 1 (downloaded meanwhile), and
    // faults in the pages of output i. Output i's download reuses the staging only after that.
    if (i >= 1) collect(i - 1);
    if (!dst_locked) copier.touch(index + i * out_item, out_item * sizeof(float));
    check(cudaStreamWaitEvent(d, solved_[k].get(), 0), "cudaStreamWaitEvent");
    float* const down = dst_locked ? index + i * out_item : output_.get();
    for (int j = 0; j < kOutParts; ++j) {
      if (part_len(j) > 0) {
        check(cudaMemcpyAsync(down + j * part, slot[k] + j * part, part_len(j) * sizeof(float),
                              cudaMemcpyDeviceToHost, d),
              "download index");
      }
      part_done_[j].record(d);
    }
    downloaded_[k].record(d);
  }
  check(cudaMemcpyAsync(filled_host_.get() + batch_, odt_.wait_count(), sizeof(unsigned long long),
                        cudaMemcpyDeviceToHost, s),
        "download wait count");
  collect(items - 1);
  check(cudaStreamSynchronize(d), "stream download");
  check(cudaStreamSynchronize(s), "stream");
  if (filled_host_.get()[batch_] != waits_seen_) {
    waits_seen_ = filled_host_.get()[batch_];
    fail(kTimeout, wait_timeout_message("Pipeline stream"));
  }
  filled_ = static_cast<double>(*filled_host_.get()) / static_cast<double>(odt_.volume());
  timings_ = PipelineTimes{};
  timings_.total = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

void PipelinePlan::check_device_waits(cudaStream_t s) {
  unsigned long long n = 0;
  check(cudaMemcpyAsync(&n, odt_.wait_count(), sizeof n, cudaMemcpyDeviceToHost, s), "download wait count");
  check(cudaStreamSynchronize(s), "wait count");
  if (n != waits_seen_) {
    waits_seen_ = n;
    fail(kTimeout, wait_timeout_message("Pipeline"));
  }
}

void PipelinePlan::wait_probe(int polls) {
  require(polls >= 1 && polls <= (1 << 20), "wait_probe: polls must be between 1 and 2^20");
  bounded_wait_probe(const_cast<unsigned long long*>(odt_.wait_count()), polls, compute_.get());
  check_device_waits(compute_.get());
}

void PipelinePlan::process_device(const float* d_holo, float* d_index, cudaStream_t s) {
  if (!has_background_) fail(kLogicError, "Pipeline: set_background() first");
  compute(d_holo, false, background_.get(), d_index, s, true);
}

void PipelinePlan::process_device_graph(const float* d_holo, float* d_index, cudaStream_t s) {
  if (!has_background_) fail(kLogicError, "Pipeline: set_background() first");
  if (!graph_warm_) {
    enqueue(d_holo, background_.get(), d_index, s);
    graph_warm_ = true;
    return;
  }
  graph_.run({d_holo, d_index}, s, [&](cudaStream_t c) { enqueue(d_holo, background_.get(), d_index, c); });
}

}  // namespace qhk
