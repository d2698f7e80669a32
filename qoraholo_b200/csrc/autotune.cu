// Launch-shape autotuner (autotune.hpp).
#include <algorithm>
#include <cstdlib>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>

#include "autotune.hpp"

namespace qhk {

namespace {

struct Entry {
  int choice = 0;
  std::vector<std::pair<int, float>> timings;  // (candidate, microseconds)
};

std::mutex g_tune_mutex;
std::map<TuneKey, Entry> g_tuned;

int initial_enabled() {
  const char* v = std::getenv("QHK_AUTOTUNE");
  return (v && v[0] == '0') ? 0 : 1;
}
std::atomic<int> g_enabled{initial_enabled()};

const char* family_name(TuneFamily f) {
  switch (f) {
    case TuneFamily::axis: return "axis_cols";
    case TuneFamily::fgp: return "fgp_rows";
    default: return "axis_engine";
  }
}

// Optional table of choices shared between runs (QHK_AUTOTUNE_FILE): one line per key, "family s0 ..
// s5 choice". Keys found there are not timed again; new choices are appended. A profiled run can so
// reuse the shapes a plain run of the same command chose, instead of timing them under the profiler.
const char* table_path() {
  const char* p = std::getenv("QHK_AUTOTUNE_FILE");
  return (p && p[0]) ? p : nullptr;
}

bool g_table_loaded = false;  // guarded by g_tune_mutex

void load_table(int device) {
  if (g_table_loaded) return;
  g_table_loaded = true;
  const char* path = table_path();
  if (!path) return;
  std::ifstream in(path);
  std::string fam;
  while (in >> fam) {
    TuneKey k;
    k.device = device;
    k.family = fam == "fgp_rows" ? TuneFamily::fgp : fam == "axis_engine" ? TuneFamily::axis_engine : TuneFamily::axis;
    for (long long& v : k.shape) in >> v;
    Entry e;
    in >> e.choice;
    if (!in) break;
    g_tuned.emplace(k, std::move(e));
  }
}

void append_table(const TuneKey& k, int choice) {
  const char* path = table_path();
  if (!path) return;
  std::ofstream out(path, std::ios::app);
  out << family_name(k.family);
  for (const long long v : k.shape) out << ' ' << v;
  out << ' ' << choice << '\n';
}

}  // namespace

bool TuneKey::operator<(const TuneKey& o) const {
  if (device != o.device) return device < o.device;
  if (family != o.family) return family < o.family;
  return shape < o.shape;
}

TuneKey tune_key(TuneFamily family, std::array<long long, 6> shape) {
  TuneKey k;
  check(cudaGetDevice(&k.device), "cudaGetDevice");
  k.family = family;
  k.shape = shape;
  return k;
}

int tuned_choice(const TuneKey& key, int fallback) {
  if (!autotune_enabled()) return fallback;
  std::lock_guard<std::mutex> lk(g_tune_mutex);
  load_table(key.device);
  const auto it = g_tuned.find(key);
  return it == g_tuned.end() ? fallback : it->second.choice;
}

bool is_tuned(const TuneKey& key) {
  std::lock_guard<std::mutex> lk(g_tune_mutex);
  load_table(key.device);
  return g_tuned.count(key) != 0;
}

bool autotune_enabled() { return g_enabled.load() != 0; }
void set_autotune_enabled(bool on) { g_enabled.store(on ? 1 : 0); }

int autotune(const TuneKey& key, const std::vector<int>& candidates, int fallback,
             const std::function<void(int)>& run, cudaStream_t s, int reps) {
  if (!autotune_enabled() || candidates.size() < 2) return tuned_choice(key, fallback);
  if (is_tuned(key)) return tuned_choice(key, fallback);
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  check(cudaStreamIsCapturing(s, &cap), "cudaStreamIsCapturing");
  if (cap != cudaStreamCaptureStatusNone) return tuned_choice(key, fallback);
  Event start, stop;
  Entry e;
  float best = 0;
  for (const int c : candidates) {
    run(c);
    run(c);
    start.record(s);
    for (int r = 0; r < reps; ++r) run(c);
    stop.record(s);
    check(cudaEventSynchronize(stop.get()), "autotune");
    const float us = 1000.0f * stop.since(start) / static_cast<float>(reps);
    e.timings.emplace_back(c, us);
    if (e.timings.size() == 1 || us < best) {
      best = us;
      e.choice = c;
    }
  }
  std::lock_guard<std::mutex> lk(g_tune_mutex);
  const auto ins = g_tuned.emplace(key, std::move(e));
  if (ins.second) append_table(key, ins.first->second.choice);
  return ins.first->second.choice;
}

std::string autotune_report() {
  std::lock_guard<std::mutex> lk(g_tune_mutex);
  std::ostringstream out;
  for (const auto& [k, e] : g_tuned) {
    out << family_name(k.family) << " device " << k.device << " shape";
    for (const long long v : k.shape) out << ' ' << v;
    out << " -> " << e.choice << " (";
    for (std::size_t i = 0; i < e.timings.size(); ++i) {
      out << (i ? ", " : "") << e.timings[i].first << ": " << e.timings[i].second << " us";
    }
    out << ")\n";
  }
  return out.str();
}

}  // namespace qhk
