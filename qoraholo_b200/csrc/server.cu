// Serving loop: continuous batching of reconstruction requests of several geometries on one GPU.
//
// A scheduler thread owns the device work. Requests wait in arrival order; whenever an execution
// slot and device memory are free (Admission, below), the next admissible request is given a
// workspace of its geometry -- an idle one is reused, otherwise one is allocated, releasing idle
// workspaces of other geometries first if the budget requires it -- and its whole pass is enqueued
// on the workspace's stream: host -> device copy of the holograms, the pipeline (field extraction
// against the geometry's resident background fields, Rytov, Ewald mapping, GP / FISTA-TV), device
// -> host copy of the index volume and of the filled count, and a host callback. Requests of
// different workspaces run concurrently on the GPU: their copies overlap other requests' kernels,
// and small requests fill the SMs that large ones leave idle between launches. From its second
// request on, a workspace replays its pipeline as one CUDA graph captured from the same enqueue
// code, so a request costs a handful of host calls instead of hundreds of launches.
//
// Results do not depend on what runs beside them: each request computes in its own workspace with
// the same deterministic kernels, so a request's volume is bitwise the same alone and in a mix.
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <thread>

#include "nvtx.hpp"
#include "server.hpp"

namespace qhk {

// ---------------------------------------------------------------------------------------------
// Admission

Admission::Admission(std::size_t budget, int max_inflight, int max_pass)
    : budget_(budget), max_inflight_(max_inflight), max_pass_(max_pass) {
  require(budget > 0, "Server: the device-memory budget must be positive");
  require(max_inflight >= 1, "Server: max_inflight must be at least 1");
  require(max_pass >= 0, "Server: max_pass must be non-negative");
}

int Admission::add_geometry(std::size_t resident, std::size_t workspace) {
  std::size_t idle_bytes = 0;
  for (int w : idle_) idle_bytes += geoms_[owner_.at(w)].workspace;
  if (used_ - idle_bytes + resident + workspace > budget_) return -1;
  geoms_.push_back(Geometry{resident, workspace, 0, true});
  used_ += resident;
  return static_cast<int>(geoms_.size()) - 1;
}

std::vector<int> Admission::remove_geometry(int geometry) {
  Geometry& g = geoms_.at(geometry);
  require(g.live, "Server: unknown geometry");
  if (g.busy > 0) fail(kLogicError, "Server: geometry has running requests");
  std::vector<int> out;
  for (auto it = idle_.begin(); it != idle_.end();) {
    if (owner_.at(*it) == geometry) {
      out.push_back(*it);
      used_ -= g.workspace;
      owner_.erase(*it);
      it = idle_.erase(it);
    } else {
      ++it;
    }
  }
  used_ -= g.resident;
  g.live = false;
  return out;
}

std::optional<Admission::Decision> Admission::choose(const std::vector<int>& pending) const {
  if (inflight_ >= max_inflight_) return std::nullopt;
  for (std::size_t i = 0; i < pending.size(); ++i) {
    const int g = pending[i];
    const Geometry& G = geoms_.at(g);
    Decision d;
    d.position = i;
    d.geometry = g;
    // Reuse the most recently used idle workspace of this geometry.
    for (auto it = idle_.rbegin(); it != idle_.rend(); ++it) {
      if (owner_.at(*it) == g) {
        d.action = Action::reuse;
        d.workspace = *it;
        return d;
      }
    }
    d.action = Action::allocate;
    if (used_ + G.workspace <= budget_) return d;
    std::size_t freed = 0;
    for (int w : idle_) {
      if (used_ - freed + G.workspace <= budget_) break;
      d.evict.push_back(w);
      freed += geoms_[owner_.at(w)].workspace;
    }
    if (used_ - freed + G.workspace <= budget_) return d;
    if (i == 0 && head_passed_ >= max_pass_) return std::nullopt;
  }
  return std::nullopt;
}

void Admission::commit(const Decision& d, int new_workspace) {
  for (int w : d.evict) {
    idle_.remove(w);
    used_ -= geoms_[owner_.at(w)].workspace;
    owner_.erase(w);
  }
  Geometry& g = geoms_.at(d.geometry);
  if (d.action == Action::reuse) {
    idle_.remove(d.workspace);
  } else {
    owner_[new_workspace] = d.geometry;
    used_ += g.workspace;
  }
  ++g.busy;
  ++inflight_;
  head_passed_ = d.position == 0 ? 0 : head_passed_ + 1;
}

void Admission::release(int workspace) {
  Geometry& g = geoms_.at(owner_.at(workspace));
  --g.busy;
  --inflight_;
  idle_.push_back(workspace);
}

void Admission::drop(int workspace) {
  const auto it = owner_.find(workspace);
  if (it == owner_.end()) return;
  Geometry& g = geoms_.at(it->second);
  const auto idle = std::find(idle_.begin(), idle_.end(), workspace);
  if (idle != idle_.end()) {
    idle_.erase(idle);
  } else {
    --g.busy;
    --inflight_;
  }
  used_ -= g.workspace;
  owner_.erase(it);
}

void Admission::add_idle(int geometry, int workspace) {
  owner_[workspace] = geometry;
  used_ += geoms_.at(geometry).workspace;
  idle_.push_back(workspace);
}

std::vector<int> Admission::make_room(std::size_t bytes) {
  std::vector<int> out;
  while (used_ + bytes > budget_ && !idle_.empty()) {
    const int w = idle_.front();
    idle_.pop_front();
    used_ -= geoms_[owner_.at(w)].workspace;
    owner_.erase(w);
    out.push_back(w);
  }
  return out;
}

// ---------------------------------------------------------------------------------------------
// Server

namespace {

double ms_between(std::chrono::steady_clock::time_point a, std::chrono::steady_clock::time_point b) {
  return std::chrono::duration<double, std::milli>(b - a).count();
}

}  // namespace

Server::Workspace::~Workspace() {
  if (graph) cudaGraphExecDestroy(graph);
}

Server::Server(std::size_t hbm_budget, int max_inflight, bool use_graphs, int stagers)
    : use_graphs_(use_graphs), admission_(hbm_budget, max_inflight) {
  const char* e = std::getenv("QHK_SERVER_EXCLUSIVE");
  exclusive_ = e && e[0] == '1';
  require(stagers >= 1, "Server: need at least one stager thread");
  check(cudaGetDevice(&device_), "cudaGetDevice");
  stats_.budget = hbm_budget;
  thread_ = std::thread([this] { loop(); });
  // Each stager copies with its own threads (the staging copies are host-bandwidth bound and one core
  // reaches a fraction of it), so two stagers' copies proceed side by side.
  const int hw = static_cast<int>(std::max(1u, std::thread::hardware_concurrency()));
  for (int i = 0; i < stagers; ++i) copiers_.push_back(std::make_unique<HostCopier>(std::clamp(hw / stagers, 1, 8)));
  for (int i = 0; i < stagers; ++i) stagers_.emplace_back([this, i] { stager(*copiers_[i]); });
}

Server::~Server() {
  {
    std::lock_guard<std::mutex> lk(mu_);
    stop_ = true;
  }
  wake_.notify_all();
  if (thread_.joinable()) thread_.join();  // returns once nothing is in flight
  {
    std::lock_guard<std::mutex> lk(mu_);
    stop_stagers_ = true;
  }
  jobs_cv_.notify_all();
  for (auto& t : stagers_) t.join();
  cudaSetDevice(device_);
  workspaces_.clear();
  geoms_.clear();
}

bool Server::is_pinned(const void* p) {
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

std::unique_ptr<Server::Workspace> Server::make_workspace(const Geometry& g) {
  auto w = std::make_unique<Workspace>();
  w->plan = std::make_unique<PipelinePlan>(g.crop, g.count, 1, g.odt, g.illum.data(), false);
  return w;
}

int Server::add_geometry(const CropPlan& crop, int count, const OdtConfig& odt, const float* illum_fyfx,
                         const float* host_bg) {
  require(illum_fyfx != nullptr && host_bg != nullptr, "Server: null argument");
  check(cudaSetDevice(device_), "cudaSetDevice");
  auto g = std::make_unique<Geometry>();
  g->crop = crop;
  g->count = count;
  g->odt = odt;
  g->illum.assign(illum_fyfx, illum_fyfx + 2 * static_cast<std::size_t>(count));
  g->holo_floats = static_cast<std::size_t>(count) * crop.n * crop.n;
  g->volume = static_cast<std::size_t>(odt.grid.nz) * odt.grid.n * odt.grid.n;
  auto w = make_workspace(*g);
  g->background.reset(w->plan->field_elems());
  const cudaStream_t s = w->plan->stream();
  check(cudaMemcpyAsync(w->plan->holo_buffer(), host_bg, g->holo_floats * sizeof(float), cudaMemcpyHostToDevice, s),
        "Server: upload backgrounds");
  w->plan->enqueue_background(w->plan->holo_buffer(), g->background.get(), s);
  check(cudaStreamSynchronize(s), "Server: background fields");
  const std::size_t resident = g->background.bytes();
  const std::size_t ws_bytes = w->plan->device_bytes();

  std::vector<std::unique_ptr<Workspace>> dead;
  int id = -1;
  {
    std::lock_guard<std::mutex> lk(mu_);
    id = admission_.add_geometry(resident, ws_bytes);
    if (id >= 0) {
      for (int e : admission_.make_room(ws_bytes)) {
        dead.push_back(std::move(workspaces_.at(e)));
        workspaces_.erase(e);
        ++stats_.workspaces_evicted;
      }
      w->geometry = id;
      geoms_.push_back(std::move(g));
      const int wid = next_workspace_++;
      workspaces_[wid] = std::move(w);
      admission_.add_idle(id, wid);
      ++stats_.workspaces_created;
      ++stats_.geometries;
      stats_.used = admission_.used();
      stats_.peak_used = std::max(stats_.peak_used, stats_.used);
    }
  }
  if (id < 0) {
    fail(kInvalidArgument, "Server: geometry does not fit the device-memory budget (" + std::to_string(resident) +
                               " resident + " + std::to_string(ws_bytes) + " per workspace bytes)");
  }
  return id;
}

void Server::remove_geometry(int geometry) {
  std::vector<std::unique_ptr<Workspace>> dead;
  std::unique_ptr<Geometry> gone;
  {
    std::lock_guard<std::mutex> lk(mu_);
    require(geometry >= 0 && geometry < static_cast<int>(geoms_.size()) && geoms_[geometry],
            "Server: unknown geometry");
    if (geoms_[geometry]->pending > 0) fail(kLogicError, "Server: geometry has queued or running requests");
    for (int e : admission_.remove_geometry(geometry)) {
      dead.push_back(std::move(workspaces_.at(e)));
      workspaces_.erase(e);
    }
    gone = std::move(geoms_[geometry]);
    --stats_.geometries;
    stats_.used = admission_.used();
  }
  check(cudaSetDevice(device_), "cudaSetDevice");
}

void Server::volume_shape(int geometry, int* nz, int* n) {
  std::lock_guard<std::mutex> lk(mu_);
  require(geometry >= 0 && geometry < static_cast<int>(geoms_.size()) && geoms_[geometry],
          "Server: unknown geometry");
  *nz = geoms_[geometry]->odt.grid.nz;
  *n = geoms_[geometry]->odt.grid.n;
}

std::uint64_t Server::submit(int geometry, const float* host_holo, float* host_out) {
  require(host_holo != nullptr && host_out != nullptr, "Server: null argument");
  auto r = std::make_unique<Request>();
  r->submitted = Clock::now();
  r->geometry = geometry;
  r->caller_in = host_holo;
  r->caller_out = host_out;
  r->in_pinned = is_pinned(host_holo);
  r->out_pinned = is_pinned(host_out);
  std::uint64_t ticket = 0;
  {
    std::lock_guard<std::mutex> lk(mu_);
    require(!stop_, "Server: closed");
    require(geometry >= 0 && geometry < static_cast<int>(geoms_.size()) && geoms_[geometry],
            "Server: unknown geometry");
    ++geoms_[geometry]->pending;  // keeps the geometry alive until this request is waited for
    ticket = next_ticket_++;
    r->ticket = ticket;
    requests_[ticket] = std::move(r);
    pending_.push_back(ticket);
    ++stats_.submitted;
    kick_ = true;
  }
  wake_.notify_one();
  return ticket;
}

bool Server::done(std::uint64_t ticket) {
  std::lock_guard<std::mutex> lk(mu_);
  const auto it = requests_.find(ticket);
  require(it != requests_.end(), "Server: unknown ticket");
  return it->second->done;
}

bool Server::cancel(std::uint64_t ticket) {
  std::lock_guard<std::mutex> lk(mu_);
  const auto it = requests_.find(ticket);
  require(it != requests_.end(), "Server: unknown ticket");
  const auto q = std::find(pending_.begin(), pending_.end(), ticket);
  if (q == pending_.end()) return false;
  pending_.erase(q);
  Request& r = *it->second;
  r.error = "Server: request cancelled before it ran";
  r.error_status = kLogicError;
  r.admitted = r.finished = Clock::now();
  r.done = true;
  ++stats_.cancelled;
  kick_ = true;  // a passed-over head may be gone
  wake_.notify_one();
  done_.notify_all();
  return true;
}

void Server::wait(std::uint64_t ticket, double* filled, RequestTimes* times) {
  std::unique_ptr<Request> r;
  {
    std::unique_lock<std::mutex> lk(mu_);
    const auto it = requests_.find(ticket);
    require(it != requests_.end(), "Server: unknown ticket");
    Request* p = it->second.get();
    done_.wait(lk, [p] { return p->done; });
    r = std::move(it->second);
    requests_.erase(it);
    --geoms_[r->geometry]->pending;
  }
  if (!r->error.empty()) throw Error(r->error_status, r->error);
  if (filled) *filled = r->filled;
  if (times) {
    times->queue = ms_between(r->submitted, r->admitted);
    times->service = ms_between(r->admitted, r->finished);
    times->total = ms_between(r->submitted, r->finished);
    times->gpu = r->gpu_ms;
  }
}

ServerStats Server::stats() {
  std::lock_guard<std::mutex> lk(mu_);
  ServerStats s = stats_;
  s.used = admission_.used();
  s.inflight = admission_.inflight();
  return s;
}

void CUDART_CB Server::on_complete(void* data) {
  // Runs on the CUDA callback thread: no CUDA calls here, only the hand-over to the scheduler.
  auto* c = static_cast<Completion*>(data);
  Server* sv = c->server;
  const std::uint64_t ticket = c->ticket;
  delete c;
  // Notify under the lock: once it is released the scheduler may finish and the server go away.
  std::lock_guard<std::mutex> lk(sv->mu_);
  sv->completed_.push_back(ticket);
  sv->wake_.notify_one();
}

void Server::launch(const Request& r, Workspace& w, const Geometry& g) {
  const cudaStream_t s = w.plan->stream();
  const float* in = r.in_pinned ? r.caller_in : w.in.get();
  float* out = r.out_pinned ? r.caller_out : w.out.get();
  w.start.record(s);
  check(cudaMemcpyAsync(w.plan->holo_buffer(), in, g.holo_floats * sizeof(float), cudaMemcpyHostToDevice, s),
        "Server: upload holograms");
  const float2* bg = g.background.get();
  // Serialised compute (QHK_SERVER_EXCLUSIVE=1): each request's kernels wait for the previous
  // request's kernels, in the order they are enqueued, while copies still overlap.
  std::unique_lock<std::mutex> ck(compute_mu_, std::defer_lock);
  const auto begin_compute = [&] {
    if (!exclusive_) return;
    ck.lock();
    check(cudaStreamWaitEvent(s, compute_tail_.get(), 0), "cudaStreamWaitEvent");
  };
  const auto end_compute = [&] {
    if (!exclusive_) return;
    compute_tail_.record(s);
    ck.unlock();
  };
  if (!w.warmed || !use_graphs_) {
    // First request of a workspace: eager launches, which also make every lazy per-device setup
    // (twiddle tables, shared-memory limits) happen outside any capture.
    begin_compute();
    w.plan->enqueue(w.plan->holo_buffer(), bg, w.plan->index_buffer(), s);
    end_compute();
    w.warmed = true;
  } else {
    if (!w.graph) {
      cudaGraph_t graph = nullptr;
      check(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "Server: begin capture");
      try {
        w.plan->enqueue(w.plan->holo_buffer(), bg, w.plan->index_buffer(), s);
      } catch (...) {
        cudaStreamEndCapture(s, &graph);
        if (graph) cudaGraphDestroy(graph);
        throw;
      }
      check(cudaStreamEndCapture(s, &graph), "Server: end capture");
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
      const cudaError_t e = cudaGraphInstantiate(&w.graph, graph, 0);
      cudaGraphDestroy(graph);
      check(e, "Server: instantiate graph");
      // Captured launches did not run; they are counted when the graph is launched.
      g_launches.fetch_sub(kernels);
      w.graph_kernels = kernels;
    }
    begin_compute();
    check(cudaGraphLaunch(w.graph, s), "Server: graph launch");
    end_compute();
    g_launches.fetch_add(w.graph_kernels);
    std::lock_guard<std::mutex> lk(mu_);
    ++stats_.graph_launches;
  }
  check(cudaMemcpyAsync(out, w.plan->index_buffer(), g.volume * sizeof(float), cudaMemcpyDeviceToHost, s),
        "Server: download index");
  check(cudaMemcpyAsync(w.filled.get(), w.plan->odt().filled(), sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                        s),
        "Server: download filled");
  check(cudaMemcpyAsync(w.filled.get() + 1, w.plan->odt().wait_count(), sizeof(unsigned long long),
                        cudaMemcpyDeviceToHost, s),
        "Server: download wait count");
  w.stop.record(s);
  auto* c = new Completion{this, r.ticket};
  const cudaError_t e = cudaLaunchHostFunc(s, &Server::on_complete, c);
  if (e != cudaSuccess) {
    delete c;
    check(e, "Server: completion callback");
  }
}

void Server::fail_request(Request& r, const std::string& error, Status status) {
  // Called with the lock held. The workspace (if any) is dropped: its state is unknown.
  r.error = error;
  r.error_status = status;
  r.done = true;
  ++stats_.failed;
  if (r.workspace >= 0) admission_.drop(r.workspace);
  kick_ = true;
  wake_.notify_one();
  done_.notify_all();
}

// Stager: stage the input into the workspace (pageable callers), allocate the workspace if it is
// new, and enqueue the request's device work.
void Server::start_request(std::uint64_t ticket, HostCopier& copier) {
  const NvtxRange range("qhk:serve_request");
  Request* r = nullptr;
  Workspace* w = nullptr;
  const Geometry* g = nullptr;
  {
    std::lock_guard<std::mutex> lk(mu_);
    r = requests_.at(ticket).get();
    g = geoms_[r->geometry].get();
    if (!r->fresh_workspace) w = workspaces_.at(r->workspace).get();
  }
  try {
    std::unique_ptr<Workspace> fresh;
    if (!w) {
      fresh = make_workspace(*g);
      fresh->geometry = r->geometry;
      w = fresh.get();
    }
    if (!r->in_pinned) {
      if (!w->in.get()) w->in = PinnedBuf<float>(g->holo_floats);
      copier.copy(w->in.get(), r->caller_in, g->holo_floats * sizeof(float));
    }
    if (!r->out_pinned && !w->out.get()) w->out = PinnedBuf<float>(g->volume);
    if (fresh) {
      std::lock_guard<std::mutex> lk(mu_);
      workspaces_[r->workspace] = std::move(fresh);
      ++stats_.workspaces_created;
    }
    launch(*r, *w, *g);
    // While the device works: the page faults of a fresh output buffer (its contents are unspecified
    // until wait returns) are taken now instead of during the copy out, which waits for this.
    if (!r->out_pinned) copier.touch(r->caller_out, g->volume * sizeof(float));
    {
      std::lock_guard<std::mutex> lk(mu_);
      r->started = true;
    }
    started_.notify_all();
  } catch (const std::exception& e) {
    std::unique_ptr<Workspace> failed;
    {
      std::lock_guard<std::mutex> lk(mu_);
      if (const auto it = workspaces_.find(r->workspace); it != workspaces_.end()) {
        failed = std::move(it->second);
        workspaces_.erase(it);
      }
      const auto* qe = dynamic_cast<const Error*>(&e);
      fail_request(*r, e.what(), qe ? qe->status : kInternal);
      r->started = true;  // no drain may wait on it
    }
    started_.notify_all();
    // Freeing device memory waits for the device, including other requests' completion callbacks,
    // which take the lock: it is released first.
    failed.reset();
  }
}

// Stager: copy a finished request's volume out of the workspace's staging buffer, then release the
// workspace.
void Server::drain_request(std::uint64_t ticket, HostCopier& copier) {
  Request* r = nullptr;
  const Workspace* w = nullptr;
  std::size_t bytes = 0;
  {
    std::unique_lock<std::mutex> lk(mu_);
    r = requests_.at(ticket).get();
    w = workspaces_.at(r->workspace).get();
    bytes = geoms_[r->geometry]->volume * sizeof(float);
    started_.wait(lk, [r] { return r->started; });  // the start job may still be faulting caller_out in
  }
  copier.copy(r->caller_out, w->out.get(), bytes);
  std::lock_guard<std::mutex> lk(mu_);
  r->finished = Clock::now();
  r->done = true;
  admission_.release(r->workspace);
  ++stats_.completed;
  kick_ = true;
  wake_.notify_one();
  done_.notify_all();
}

void Server::stager(HostCopier& copier) {
  cudaSetDevice(device_);
  std::unique_lock<std::mutex> lk(mu_);
  for (;;) {
    jobs_cv_.wait(lk, [this] { return stop_stagers_ || !jobs_.empty(); });
    if (jobs_.empty()) return;  // stopping, nothing left
    const Job job = jobs_.front();
    jobs_.pop_front();
    lk.unlock();
    if (job.kind == Job::start) {
      start_request(job.ticket, copier);
    } else {
      drain_request(job.ticket, copier);
    }
    lk.lock();
  }
}

void Server::loop() {
  cudaSetDevice(device_);
  std::unique_lock<std::mutex> lk(mu_);
  for (;;) {
    // Completions: device work done. Pageable outputs go to a stager; the rest are done here.
    bool any_done = false;
    for (const std::uint64_t t : completed_) {
      Request& r = *requests_.at(t);
      Workspace& w = *workspaces_.at(r.workspace);
      try {
        r.gpu_ms = w.stop.since(w.start);
      } catch (const Error&) {
        r.gpu_ms = 0;
      }
      r.filled = static_cast<double>(*w.filled.get()) / static_cast<double>(geoms_[r.geometry]->volume);
      if (w.filled.get()[1] != w.waits_seen) {  // a bounded device wait ran out: the volume is not valid
        w.waits_seen = w.filled.get()[1];
        fail_request(r, wait_timeout_message("Server"), kTimeout);
        continue;
      }
      if (r.out_pinned) {
        r.finished = Clock::now();
        r.done = true;
        admission_.release(r.workspace);
        ++stats_.completed;
        any_done = true;
      } else {
        jobs_.push_back(Job{Job::drain, t});
        jobs_cv_.notify_one();
      }
    }
    completed_.clear();
    if (any_done) done_.notify_all();

    if (stop_) {
      for (const std::uint64_t t : pending_) {
        Request& r = *requests_.at(t);
        r.error = "Server: closed before the request ran";
        r.error_status = kLogicError;
        r.done = true;
        ++stats_.failed;
      }
      pending_.clear();
      done_.notify_all();
      if (admission_.inflight() == 0) break;
    }

    // Admit as many pending requests as slots and memory allow; stagers take them from here.
    while (!stop_ && !pending_.empty()) {
      std::vector<int> order;
      const std::size_t look = std::min<std::size_t>(pending_.size(), 64);
      for (std::size_t i = 0; i < look; ++i) order.push_back(requests_.at(pending_[i])->geometry);
      const auto d = admission_.choose(order);
      if (!d) break;
      std::vector<std::unique_ptr<Workspace>> dead;
      for (int e : d->evict) {
        dead.push_back(std::move(workspaces_.at(e)));
        workspaces_.erase(e);
        ++stats_.workspaces_evicted;
      }
      const bool reuse = d->action == Admission::Action::reuse;
      const int wid = reuse ? d->workspace : next_workspace_++;
      admission_.commit(*d, wid);
      if (d->position > 0) ++stats_.passed_over;
      const std::uint64_t t = pending_[d->position];
      pending_.erase(pending_.begin() + static_cast<std::ptrdiff_t>(d->position));
      Request& r = *requests_.at(t);
      r.admitted = Clock::now();
      r.workspace = wid;
      r.fresh_workspace = !reuse;
      stats_.used = admission_.used();
      stats_.peak_used = std::max(stats_.peak_used, stats_.used);
      stats_.peak_inflight = std::max(stats_.peak_inflight, admission_.inflight());
      jobs_.push_back(Job{Job::start, t});
      jobs_cv_.notify_one();
      if (!dead.empty()) {
        lk.unlock();
        dead.clear();  // frees device memory (waits for the device): never under the lock
        lk.lock();
      }
    }
    if (stop_ && admission_.inflight() == 0) continue;
    wake_.wait(lk, [this] { return stop_ || !completed_.empty() || kick_; });
    kick_ = false;
  }
}

}  // namespace qhk
