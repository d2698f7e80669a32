// Serving loop: continuous batching of reconstruction requests of several geometries on one GPU,
// against a fixed device-memory budget (server.cu). No counterpart in the reference, whose nearest
// form is one Pipeline per geometry used by one caller at a time (src/cuda/pipeline.cu:12-147).
#pragma once

#include "host_copy.hpp"

#include <chrono>
#include <condition_variable>
#include <cstddef>
#include <cstdint>
#include <deque>
#include <list>
#include <map>
#include <memory>
#include <mutex>
#include <optional>
#include <string>
#include <thread>
#include <vector>

#include "pipeline.hpp"

namespace qhk {

// Admission policy, host bookkeeping only (no CUDA calls, so it is tested on the CPU).
//
// Device memory = the resident state of every registered geometry (its background fields) plus
// the workspaces (one PipelinePlan each) that requests run in. A workspace belongs to one geometry
// and is kept after its request completes (idle), so the next request of that geometry reuses it
// with no allocation. A pending request is admitted when an execution slot is free and
//   1. an idle workspace of its geometry exists (reuse), or
//   2. a new workspace fits the budget (allocate), or
//   3. it fits after releasing idle workspaces of other geometries, least recently used first
//      (evict, then allocate).
// Requests are considered in arrival order; one that cannot be admitted yet is passed over so that
// later, smaller requests fill the memory and slots that are free (continuous batching), but the
// oldest request can be passed over at most `max_pass` times: after that nothing is admitted
// until it fits.
class Admission {
 public:
  enum class Action { reuse, allocate };
  struct Decision {
    std::size_t position = 0;       // index into the pending queue
    int geometry = -1;
    Action action = Action::reuse;
    int workspace = -1;             // reuse: the idle workspace taken
    std::vector<int> evict;         // workspaces to release first (idle, other geometries)
  };

  Admission(std::size_t budget, int max_inflight, int max_pass = 8);

  // Registers a geometry; its resident bytes are held from now on. Returns the geometry id, or -1
  // when resident + one workspace cannot fit the budget even with every idle workspace released
  // (nothing is changed then).
  int add_geometry(std::size_t resident, std::size_t workspace);
  // Releases the resident bytes of a geometry with no busy workspace; returns the idle workspaces
  // the caller must destroy.
  std::vector<int> remove_geometry(int geometry);

  // Chooses the next request to admit from `pending` (geometry ids in arrival order), or nothing.
  // The caller must apply the decision with commit() before asking again.
  [[nodiscard]] std::optional<Decision> choose(const std::vector<int>& pending) const;
  // Applies a decision: evicted workspaces are forgotten, a reused one becomes busy, an allocated
  // one is recorded as `new_workspace` (busy).
  void commit(const Decision& d, int new_workspace);
  // A request's workspace finished: it becomes idle (most recently used).
  void release(int workspace);
  // A workspace that failed to allocate or whose request failed is dropped.
  void drop(int workspace);
  // Registers an idle workspace created outside choose() (the first one of a geometry).
  void add_idle(int geometry, int workspace);
  // Forgets idle workspaces, least recently used first, until `bytes` more fit the budget; returns
  // them for the caller to destroy.
  std::vector<int> make_room(std::size_t bytes);

  [[nodiscard]] std::size_t used() const { return used_; }
  [[nodiscard]] std::size_t budget() const { return budget_; }
  [[nodiscard]] int inflight() const { return inflight_; }
  [[nodiscard]] int head_passed() const { return head_passed_; }
  [[nodiscard]] std::size_t workspace_bytes(int geometry) const { return geoms_.at(geometry).workspace; }
  [[nodiscard]] int geometry_of(int workspace) const { return owner_.at(workspace); }

 private:
  struct Geometry {
    std::size_t resident = 0;
    std::size_t workspace = 0;
    int busy = 0;
    bool live = false;
  };
  std::size_t budget_;
  int max_inflight_;
  int max_pass_;
  std::size_t used_ = 0;
  int inflight_ = 0;
  int head_passed_ = 0;
  std::vector<Geometry> geoms_;
  std::map<int, int> owner_;   // workspace -> geometry
  std::list<int> idle_;        // idle workspaces, least recently used first
};

// Per-request host timings in milliseconds.
struct RequestTimes {
  double queue = 0;    // submit -> admitted
  double service = 0;  // admitted -> completion seen by the host
  double total = 0;    // submit -> completion seen by the host
  double gpu = 0;      // device time of the request (events around its copies and kernels)
};

struct ServerStats {
  std::uint64_t submitted = 0, completed = 0, failed = 0, cancelled = 0;
  std::uint64_t workspaces_created = 0, workspaces_evicted = 0, graph_launches = 0, passed_over = 0;
  std::size_t budget = 0, used = 0, peak_used = 0;
  int geometries = 0, inflight = 0, peak_inflight = 0;
};

class Server {
 public:
  Server(std::size_t hbm_budget, int max_inflight, bool use_graphs = true, int stagers = 2);
  ~Server();
  Server(const Server&) = delete;
  Server& operator=(const Server&) = delete;

  // Registers a geometry: builds its first workspace, computes the background fields from the host
  // background holograms (count, N, N) and keeps them resident. Synchronous. Returns its id.
  int add_geometry(const CropPlan& crop, int count, const OdtConfig& odt, const float* illum_fyfx,
                   const float* host_bg);
  // Frees a geometry's resident state and idle workspaces; QHK_LOGIC_ERROR while requests of it are
  // pending or running.
  void remove_geometry(int geometry);
  // Queues one request: holograms (count, N, N) on the host -> index (nz, n, n) into `host_out`.
  // Both may be pageable (staged through the workspace's page-locked buffers by the server's stager
  // threads) or page-locked (copied directly). Both must stay valid until wait() returns; the contents
  // of a pageable `host_out` are unspecified until then (its pages are faulted in while the request
  // runs). Returns a ticket.
  std::uint64_t submit(int geometry, const float* host_holo, float* host_out);
  // Blocks until the request is done; its filled fraction and timings. Throws the request's error.
  void wait(std::uint64_t ticket, double* filled, RequestTimes* times);
  // True when the request has completed (wait() will not block).
  bool done(std::uint64_t ticket);
  // Withdraws a request that has not been admitted yet: it completes with QHK_LOGIC_ERROR ("cancelled")
  // and takes no device time. Returns false (and changes nothing) once it runs or has finished.
  bool cancel(std::uint64_t ticket);
  [[nodiscard]] ServerStats stats();
  void volume_shape(int geometry, int* nz, int* n);

 private:
  using Clock = std::chrono::steady_clock;
  struct Geometry {
    CropPlan crop{};
    int count = 0;
    OdtConfig odt{};
    std::vector<float> illum;
    DevBuf<float2> background;
    std::size_t holo_floats = 0, volume = 0;
    int pending = 0;  // requests not yet waited for
  };
  struct Workspace {
    int geometry = -1;
    std::unique_ptr<PipelinePlan> plan;
    cudaGraphExec_t graph = nullptr;
    std::uint64_t graph_kernels = 0;
    bool warmed = false;
    Event start, stop;
    PinnedBuf<unsigned long long> filled{2};  // the filled count, then the plan's wait counter
    unsigned long long waits_seen = 0;         // the wait counter after the previous request
    PinnedBuf<float> in, out;  // staging for pageable callers, allocated on first use
    ~Workspace();
  };
  struct Request {
    std::uint64_t ticket = 0;
    int geometry = -1;
    const float* caller_in = nullptr;
    float* caller_out = nullptr;
    bool in_pinned = false, out_pinned = false;
    bool started = false;  // the start job is done with caller_out (its pages faulted in): drain may copy
    Clock::time_point submitted, admitted, finished;
    int workspace = -1;
    bool fresh_workspace = false;  // admitted with a workspace still to be allocated
    bool done = false;
    double filled = 0;
    float gpu_ms = 0;
    std::string error;
    Status error_status = kOk;
  };
  struct Completion {
    Server* server;
    std::uint64_t ticket;
  };
  // Work for the stager threads: stage a request's input and enqueue its device work, or copy its
  // result out of the workspace's staging buffer.
  struct Job {
    enum Kind { start, drain } kind;
    std::uint64_t ticket;
  };

  static void CUDART_CB on_complete(void* data);
  void loop();
  void stager(HostCopier& copier);
  void start_request(std::uint64_t ticket, HostCopier& copier);
  void drain_request(std::uint64_t ticket, HostCopier& copier);
  void launch(const Request& r, Workspace& w, const Geometry& g);
  void fail_request(Request& r, const std::string& error, Status status);
  static std::unique_ptr<Workspace> make_workspace(const Geometry& g);
  static bool is_pinned(const void* p);

  std::mutex mu_;
  std::condition_variable wake_;   // scheduler: submissions, completions, released workspaces, stop
  std::condition_variable done_;   // waiters
  std::condition_variable jobs_cv_;  // stagers
  std::condition_variable started_;  // drains waiting for their request's start job
  int device_ = 0;
  bool use_graphs_;
  bool exclusive_ = false;  // serialise the requests' kernels (copies still overlap)
  std::mutex compute_mu_;
  Event compute_tail_;      // recorded after the last enqueued request's kernels
  bool stop_ = false;
  bool stop_stagers_ = false;
  bool kick_ = false;  // something the scheduler acts on changed since it last looked
  Admission admission_;
  std::vector<std::unique_ptr<Geometry>> geoms_;
  std::map<int, std::unique_ptr<Workspace>> workspaces_;
  int next_workspace_ = 0;
  std::deque<std::uint64_t> pending_;
  std::map<std::uint64_t, std::unique_ptr<Request>> requests_;
  std::vector<std::uint64_t> completed_;
  std::deque<Job> jobs_;
  std::uint64_t next_ticket_ = 1;
  ServerStats stats_;
  std::thread thread_;
  std::vector<std::unique_ptr<HostCopier>> copiers_;  // one per stager
  std::vector<std::thread> stagers_;
};

}  // namespace qhk
