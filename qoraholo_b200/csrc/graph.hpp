// CUDA-graph replay of a fixed sequence of launches (host side).
#pragma once

#include <cstdint>
#include <functional>
#include <vector>

#include "qhk_util.cuh"

namespace qhk {

// Runs the work that `enqueue` puts on the stream it is handed as one CUDA graph: captured on the
// first call (and again whenever `key` -- the buffers the work touches -- changes), replayed on
// the following calls. The graph runs on an internal stream, ordered after earlier work on `s`,
// and later work on `s` waits for it, so `s` may be any stream including the legacy default one.
// `enqueue` must be capturable: launches, memsets and device copies only, nothing that allocates
// or synchronises (run it once outside a graph first so that lazy setup happens outside capture).
class CapturedWork {
 public:
  CapturedWork() = default;
  CapturedWork(const CapturedWork&) = delete;
  CapturedWork& operator=(const CapturedWork&) = delete;
  ~CapturedWork() { reset(); }

  void run(const std::vector<const void*>& key, cudaStream_t s, const std::function<void(cudaStream_t)>& enqueue) {
    if (!exec_ || key != key_) capture(key, enqueue);
    ready_.record(s);
    check(cudaStreamWaitEvent(stream_.get(), ready_.get(), 0), "cudaStreamWaitEvent");
    check(cudaGraphLaunch(exec_, stream_.get()), "cudaGraphLaunch");
    g_launches.fetch_add(kernels_);
    done_.record(stream_.get());
    check(cudaStreamWaitEvent(s, done_.get(), 0), "cudaStreamWaitEvent");
    ++replays_;
  }

  [[nodiscard]] std::uint64_t kernels() const { return kernels_; }
  [[nodiscard]] std::uint64_t replays() const { return replays_; }

 private:
  void reset() {
    if (exec_) cudaGraphExecDestroy(exec_);
    exec_ = nullptr;
  }

  void capture(const std::vector<const void*>& key, const std::function<void(cudaStream_t)>& enqueue) {
    reset();
    const cudaStream_t c = stream_.get();
    cudaGraph_t graph = nullptr;
    check(cudaStreamBeginCapture(c, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
    try {
      enqueue(c);
    } catch (...) {
      cudaStreamEndCapture(c, &graph);
      if (graph) cudaGraphDestroy(graph);
      throw;
    }
    check(cudaStreamEndCapture(c, &graph), "cudaStreamEndCapture");
    std::size_t nodes = 0;
    check(cudaGraphGetNodes(graph, nullptr, &nodes), "cudaGraphGetNodes");
    std::vector<cudaGraphNode_t> list(nodes);
    check(cudaGraphGetNodes(graph, list.data(), &nodes), "cudaGraphGetNodes");
    std::uint64_t kernels = 0;
    for (cudaGraphNode_t n : list) {
      cudaGraphNodeType t{};
      check(cudaGraphNodeGetType(n, &t), "cudaGraphNodeGetType");
      kernels += t == cudaGraphNodeTypeKernel;
    }
    const cudaError_t e = cudaGraphInstantiate(&exec_, graph, 0);
    cudaGraphDestroy(graph);
    check(e, "cudaGraphInstantiate");
    g_launches.fetch_sub(kernels);  // captured, not run: counted at each replay
    kernels_ = kernels;
    key_ = key;
  }

  Stream stream_;
  Event ready_, done_;
  cudaGraphExec_t exec_ = nullptr;
  std::vector<const void*> key_;
  std::uint64_t kernels_ = 0;
  std::uint64_t replays_ = 0;
};

}  // namespace qhk
