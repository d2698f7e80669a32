// Host-side utilities of the CUDA backend: error reporting, device buffers, streams, events.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstddef>
#include <cstdint>
#include <mutex>
#include <set>
#include <stdexcept>
#include <string>
#include <utility>

namespace qhk {

// Error classes of the C ABI (include/qoraholo_b200.h): the host layer maps them back to the
// exception types of the reference API (invalid_argument, runtime_error, logic_error).
enum Status : int {
  kOk = 0,
  kInvalidArgument = 1,
  kCudaError = 2,
  kLogicError = 3,
  kOutOfMemory = 4,
  kTimeout = 5,
  kInternal = 6,
};

struct Error : std::runtime_error {
  Status status;
  Error(Status s, const std::string& what) : std::runtime_error(what), status(s) {}
};

inline void fail(Status s, const std::string& what) { throw Error(s, what); }
inline void require(bool ok, const std::string& what) {
  if (!ok) throw Error(kInvalidArgument, what);
}

inline void check(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return;
  const Status s = e == cudaErrorMemoryAllocation ? kOutOfMemory : kCudaError;
  throw Error(s, std::string(what) + ": " + cudaGetErrorString(e));
}

// Kernels launched by this library since load (every launch site calls check_launch once).
inline std::atomic<std::uint64_t> g_launches{0};

inline void check_launch(const char* what) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  check(cudaGetLastError(), what);
}

template <class T>
class DevBuf {
 public:
  DevBuf() = default;
  explicit DevBuf(std::size_t n) { reset(n); }
  ~DevBuf() { release(); }
  DevBuf(DevBuf&& o) noexcept : p_(std::exchange(o.p_, nullptr)), n_(std::exchange(o.n_, 0)) {}
  DevBuf& operator=(DevBuf&& o) noexcept {
    std::swap(p_, o.p_);
    std::swap(n_, o.n_);
    return *this;
  }
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;

  void reset(std::size_t n) {
    release();
    if (n > 0) check(cudaMalloc(&p_, n * sizeof(T)), "cudaMalloc");
    n_ = n;
  }
  void release() {
    if (p_) cudaFree(p_);
    p_ = nullptr;
    n_ = 0;
  }
  [[nodiscard]] T* get() const { return p_; }
  [[nodiscard]] std::size_t size() const { return n_; }
  [[nodiscard]] std::size_t bytes() const { return n_ * sizeof(T); }

 private:
  T* p_ = nullptr;
  std::size_t n_ = 0;
};

template <class T>
class PinnedBuf {
 public:
  PinnedBuf() = default;
  explicit PinnedBuf(std::size_t n) {
    if (n > 0) check(cudaMallocHost(&p_, n * sizeof(T)), "cudaMallocHost");
    n_ = n;
  }
  ~PinnedBuf() {
    if (p_) cudaFreeHost(p_);
  }
  PinnedBuf(PinnedBuf&& o) noexcept : p_(std::exchange(o.p_, nullptr)), n_(std::exchange(o.n_, 0)) {}
  PinnedBuf& operator=(PinnedBuf&& o) noexcept {
    std::swap(p_, o.p_);
    std::swap(n_, o.n_);
    return *this;
  }
  PinnedBuf(const PinnedBuf&) = delete;
  PinnedBuf& operator=(const PinnedBuf&) = delete;
  [[nodiscard]] T* get() const { return p_; }
  [[nodiscard]] std::size_t size() const { return n_; }

 private:
  T* p_ = nullptr;
  std::size_t n_ = 0;
};

class Stream {
 public:
  Stream() { check(cudaStreamCreateWithFlags(&s_, cudaStreamNonBlocking), "cudaStreamCreate"); }
  ~Stream() {
    if (s_) cudaStreamDestroy(s_);
  }
  Stream(const Stream&) = delete;
  Stream& operator=(const Stream&) = delete;
  [[nodiscard]] cudaStream_t get() const { return s_; }

 private:
  cudaStream_t s_{};
};

class Event {
 public:
  Event() { check(cudaEventCreate(&e_), "cudaEventCreate"); }
  ~Event() {
    if (e_) cudaEventDestroy(e_);
  }
  Event(const Event&) = delete;
  Event& operator=(const Event&) = delete;
  Event(Event&& o) noexcept : e_(std::exchange(o.e_, nullptr)) {}
  [[nodiscard]] cudaEvent_t get() const { return e_; }
  void record(cudaStream_t s) { check(cudaEventRecord(e_, s), "cudaEventRecord"); }
  void synchronize() const { check(cudaEventSynchronize(e_), "cudaEventSynchronize"); }
  [[nodiscard]] float since(const Event& start) const { return since_event(start.get()); }
  [[nodiscard]] float since_event(cudaEvent_t start) const {
    float ms = 0;
    check(cudaEventElapsedTime(&ms, start, e_), "cudaEventElapsedTime");
    return ms;
  }

 private:
  cudaEvent_t e_{};
};

// Raises a kernel's dynamic shared memory limit to the device maximum, once per (device, kernel).
// Launches of any size then succeed as long as dynamic plus static shared memory fit the SM.
template <class K>
void ensure_smem(K kernel) {
  static std::mutex mutex;
  static std::set<std::pair<int, const void*>> done;
  int dev = 0;
  check(cudaGetDevice(&dev), "cudaGetDevice");
  std::lock_guard<std::mutex> lock(mutex);
  const auto key = std::make_pair(dev, reinterpret_cast<const void*>(kernel));
  if (done.count(key)) return;
  cudaFuncAttributes attr{};
  check(cudaFuncGetAttributes(&attr, kernel), "cudaFuncGetAttributes");
  int optin = 0;
  check(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev), "cudaDeviceGetAttribute");
  check(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             optin - static_cast<int>(attr.sharedSizeBytes)),
        "cudaFuncSetAttribute");
  done.insert(key);
}

inline unsigned blocks_for(std::size_t n, unsigned threads) {
  return static_cast<unsigned>((n + threads - 1) / threads);
}

// Number of SMs of the current device, for grid sizing.
int sm_count();

}  // namespace qhk
