// Host-side copies between caller memory and page-locked staging, split over a few persistent
// threads. One thread's memcpy reaches a fraction of the host's memory bandwidth, and the first
// write to a freshly allocated (not yet faulted) buffer costs a page fault per 4 KB page; both
// scale with threads. Used by the Pipeline's host-buffer run and by the serving loop's stagers.
#pragma once

#include <condition_variable>
#include <cstddef>
#include <cstdint>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

namespace qhk {

// Whether [p, p + bytes) is page-locked host memory (both ends lie in page-locked allocations, so
// the device can transfer it directly without a staging copy).
bool is_page_locked(const void* p, std::size_t bytes);

// Host <-> device transfers of caller memory for one-shot calls: page-locked memory goes directly;
// pageable memory streams through two page-locked staging buffers of kChunk bytes (kept for the
// process), the host copy of one chunk overlapping the transfer of the other, on the shared copy
// threads (a download writes every page of its destination first: its contents are unspecified
// until it returns). Synchronous with respect to the host buffer: upload returns when the source may be
// reused, download when the destination holds the data (both wait for `s`). One transfer at a time
// per process (a mutex); the device side is ordered on `s`.
void upload(void* d_dst, const void* host_src, std::size_t bytes, cudaStream_t s);
void download(void* host_dst, const void* d_src, std::size_t bytes, cudaStream_t s);

class HostCopier {
 public:
  // `threads` in total, the calling thread included (so threads - 1 workers).
  explicit HostCopier(int threads);
  ~HostCopier();
  HostCopier(const HostCopier&) = delete;
  HostCopier& operator=(const HostCopier&) = delete;

  // memcpy of `bytes`, in parts of kPart bytes taken by the workers and the caller.
  void copy(void* dst, const void* src, std::size_t bytes);
  // Writes one zero byte into every page of [dst, dst + bytes), so that the page faults of memory
  // that is about to be overwritten are taken now (for example while the device computes). Only
  // for memory whose contents do not matter.
  void touch(void* dst, std::size_t bytes);
  [[nodiscard]] int threads() const { return static_cast<int>(workers_.size()) + 1; }

  // The process-wide copier: QHK_COPY_THREADS threads (default min(8, hardware threads)).
  static HostCopier& shared();

  static constexpr std::size_t kPart = std::size_t{1} << 20;

 private:
  struct Job {
    const std::function<void(std::size_t)>* fn = nullptr;
    std::size_t parts = 0;
    std::size_t next = 0;  // next part to hand out, under mu_
    std::size_t done = 0;  // parts finished, under mu_
    int active = 0;        // workers inside this job, under mu_
  };
  // Runs fn(0 .. parts-1) on the workers and the caller; returns when all are done. Jobs from
  // several callers run one after another.
  void run(std::size_t parts, const std::function<void(std::size_t)>& fn);
  void drain(Job& job);
  void worker();

  std::mutex job_mu_;  // one job at a time
  std::mutex mu_;
  std::condition_variable wake_;
  std::condition_variable finished_;
  Job* job_ = nullptr;
  std::uint64_t generation_ = 0;
  bool stop_ = false;
  std::vector<std::thread> workers_;
};

}  // namespace qhk
