// HostCopier: persistent threads for large host copies and page pre-faulting.
#include <unistd.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <string>
#include <stdexcept>
#include <mutex>

#include <cuda_runtime.h>

#include "host_copy.hpp"

namespace qhk {

namespace {

bool locked(const void* p) {
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();  // not a pointer the runtime knows: pageable
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

}  // namespace

bool is_page_locked(const void* p, std::size_t bytes) {
  if (p == nullptr || bytes == 0) return false;
  return locked(p) && locked(static_cast<const char*>(p) + bytes - 1);
}

namespace {

constexpr std::size_t kChunk = std::size_t{32} << 20;

// Two page-locked staging buffers and their "transfer done" events, created on first use and kept
// for the process (never freed: at exit the CUDA runtime may already be gone).
struct Staging {
  std::mutex mu;
  void* buf[2] = {};
  cudaEvent_t done[2] = {};
  int device = -1;
};

Staging& staging() {
  static auto* st = new Staging;
  return *st;
}

// Buffers of the current device (recreated if the calling thread's device changed).
void ensure_staging(Staging& st) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) throw std::runtime_error("transfer: cudaGetDevice failed");
  if (st.device == dev && st.buf[0]) return;
  for (int i = 0; i < 2; ++i) {
    if (!st.buf[i] && cudaMallocHost(&st.buf[i], kChunk) != cudaSuccess) {
      throw std::runtime_error("transfer: cudaMallocHost failed");
    }
    if (st.done[i]) cudaEventDestroy(st.done[i]);
    if (cudaEventCreateWithFlags(&st.done[i], cudaEventDisableTiming) != cudaSuccess) {
      throw std::runtime_error("transfer: cudaEventCreate failed");
    }
  }
  st.device = dev;
}

void ok(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

}  // namespace

void upload(void* d_dst, const void* host_src, std::size_t bytes, cudaStream_t s) {
  if (bytes == 0) return;
  if (is_page_locked(host_src, bytes)) {
    ok(cudaMemcpyAsync(d_dst, host_src, bytes, cudaMemcpyHostToDevice, s), "upload");
    ok(cudaStreamSynchronize(s), "upload");
    return;
  }
  Staging& st = staging();
  std::lock_guard<std::mutex> lk(st.mu);
  ensure_staging(st);
  HostCopier& copier = HostCopier::shared();
  for (std::size_t off = 0, k = 0; off < bytes; off += kChunk, ++k) {
    const int b = static_cast<int>(k & 1);
    const std::size_t len = std::min(kChunk, bytes - off);
    if (k >= 2) ok(cudaEventSynchronize(st.done[b]), "upload");  // buffer b's previous transfer
    copier.copy(st.buf[b], static_cast<const char*>(host_src) + off, len);
    ok(cudaMemcpyAsync(static_cast<char*>(d_dst) + off, st.buf[b], len, cudaMemcpyHostToDevice, s), "upload");
    ok(cudaEventRecord(st.done[b], s), "upload");
  }
  ok(cudaStreamSynchronize(s), "upload");
}

void download(void* host_dst, const void* d_src, std::size_t bytes, cudaStream_t s) {
  if (bytes == 0) return;
  if (is_page_locked(host_dst, bytes)) {
    ok(cudaMemcpyAsync(host_dst, d_src, bytes, cudaMemcpyDeviceToHost, s), "download");
    ok(cudaStreamSynchronize(s), "download");
    return;
  }
  Staging& st = staging();
  std::lock_guard<std::mutex> lk(st.mu);
  ensure_staging(st);
  HostCopier& copier = HostCopier::shared();
  const std::size_t chunks = (bytes + kChunk - 1) / kChunk;
  const auto issue = [&](std::size_t k) {
    const int b = static_cast<int>(k & 1);
    const std::size_t off = k * kChunk;
    ok(cudaMemcpyAsync(st.buf[b], static_cast<const char*>(d_src) + off, std::min(kChunk, bytes - off),
                       cudaMemcpyDeviceToHost, s),
       "download");
    ok(cudaEventRecord(st.done[b], s), "download");
  };
  issue(0);
  // The destination's page faults (a fresh array) are taken while the device finishes the work
  // queued before this call and the first chunk is in flight.
  copier.touch(host_dst, bytes);
  for (std::size_t k = 0; k < chunks; ++k) {
    const int b = static_cast<int>(k & 1);
    ok(cudaEventSynchronize(st.done[b]), "download");
    if (k + 1 < chunks) issue(k + 1);  // the next chunk lands while this one is copied out
    const std::size_t off = k * kChunk;
    copier.copy(static_cast<char*>(host_dst) + off, st.buf[b], std::min(kChunk, bytes - off));
  }
}

HostCopier::HostCopier(int threads) {
  for (int i = 1; i < std::max(threads, 1); ++i) workers_.emplace_back([this] { worker(); });
}

HostCopier::~HostCopier() {
  {
    std::lock_guard<std::mutex> lk(mu_);
    stop_ = true;
  }
  wake_.notify_all();
  for (auto& t : workers_) t.join();
}

HostCopier& HostCopier::shared() {
  static HostCopier copier([] {
    const char* e = std::getenv("QHK_COPY_THREADS");
    if (e && std::atoi(e) > 0) return std::atoi(e);
    return static_cast<int>(std::min(8u, std::max(1u, std::thread::hardware_concurrency())));
  }());
  return copier;
}

void HostCopier::drain(Job& job) {
  for (;;) {
    std::size_t i;
    {
      std::lock_guard<std::mutex> lk(mu_);
      if (job.next >= job.parts) return;
      i = job.next++;
    }
    (*job.fn)(i);
    std::lock_guard<std::mutex> lk(mu_);
    if (++job.done == job.parts) finished_.notify_all();
  }
}

void HostCopier::worker() {
  std::uint64_t seen = 0;
  for (;;) {
    Job* job;
    {
      std::unique_lock<std::mutex> lk(mu_);
      wake_.wait(lk, [&] { return stop_ || (job_ != nullptr && generation_ != seen); });
      if (stop_) return;
      seen = generation_;
      job = job_;
      ++job->active;
    }
    drain(*job);
    std::lock_guard<std::mutex> lk(mu_);
    if (--job->active == 0) finished_.notify_all();
  }
}

void HostCopier::run(std::size_t parts, const std::function<void(std::size_t)>& fn) {
  if (parts == 0) return;
  if (parts == 1 || workers_.empty()) {
    for (std::size_t i = 0; i < parts; ++i) fn(i);
    return;
  }
  std::lock_guard<std::mutex> one(job_mu_);
  Job job;
  job.fn = &fn;
  job.parts = parts;
  {
    std::lock_guard<std::mutex> lk(mu_);
    job_ = &job;
    ++generation_;
  }
  wake_.notify_all();
  drain(job);
  std::unique_lock<std::mutex> lk(mu_);
  job_ = nullptr;  // workers that have not joined yet no longer can; `job` lives until those inside leave
  finished_.wait(lk, [&] { return job.done == job.parts && job.active == 0; });
}

void HostCopier::copy(void* dst, const void* src, std::size_t bytes) {
  if (bytes == 0 || dst == src) return;
  const std::size_t parts = (bytes + kPart - 1) / kPart;
  const std::function<void(std::size_t)> fn = [&](std::size_t i) {
    const std::size_t off = i * kPart;
    std::memcpy(static_cast<char*>(dst) + off, static_cast<const char*>(src) + off, std::min(kPart, bytes - off));
  };
  run(parts, fn);
}

void HostCopier::touch(void* dst, std::size_t bytes) {
  if (bytes == 0) return;
  static const std::size_t page = [] {
    const long p = sysconf(_SC_PAGESIZE);
    return p > 0 ? static_cast<std::size_t>(p) : std::size_t{4096};
  }();
  const std::size_t parts = (bytes + kPart - 1) / kPart;
  char* base = static_cast<char*>(dst);
  const std::function<void(std::size_t)> fn = [&](std::size_t i) {
    const std::size_t begin = i * kPart, end = std::min(begin + kPart, bytes);
    // the first byte of the part, then every page boundary inside it
    const auto addr = reinterpret_cast<std::uintptr_t>(base + begin);
    std::size_t off = begin;
    for (;;) {
      *reinterpret_cast<volatile char*>(base + off) = 0;
      const std::size_t next = ((addr - begin + off) / page + 1) * page - (addr - begin);
      if (next >= end) break;
      off = next;
    }
  };
  run(parts, fn);
}

}  // namespace qhk
