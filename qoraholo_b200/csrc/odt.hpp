// ODT solver plan of the CUDA backend (odt.cu): holds the device buffers for one geometry and
// runs fields -> index on a stream.
#pragma once

#include <utility>
#include <vector>

#include "qhk_internal.hpp"

namespace qhk {

// Events recorded at stage boundaries on one stream, read after the stream has finished.
class StageClock {
 public:
  explicit StageClock(int marks) : events_(marks) {}
  void mark(int i, cudaStream_t s) { events_.at(i).record(s); }
  [[nodiscard]] double ms(int from, int to) const { return events_.at(to).since(events_.at(from)); }
  [[nodiscard]] cudaEvent_t event(int i) const { return events_.at(i).get(); }

 private:
  std::vector<Event> events_;
};

Grid make_grid(int n, int nz, float wavelength, float n_medium, float na, float pixel);

// Per-illumination (fy, fx, fiz, 0), fiz = sqrt(fm2 - fy^2 - fx^2) in float as the host computes it.
std::vector<float4> illumination_table(const Grid& g, const float* illum_fyfx, int count);

// Ewald mapping of `count` spectra (count, n, n): half-spectrum data and hit counts (nz, n, n/2+1)
// for the real solvers, or the full normalised potential and mask (nz, n, n) for the complex one
// (`measured`, optional, gets a copy). `filled` is incremented by the number of voxels with data.
// `batch` volumes at once: volume b maps spectra b * count .. into its own arrays and filled[b].
void map_half(const float2* spectra, const float4* illum, int count, const Grid& g, float2* a, std::uint8_t* hits,
              unsigned long long* filled, cudaStream_t s, int batch = 1);
void map_full(const float2* spectra, const float4* illum, int count, const Grid& g, float2* pot, float2* measured,
              std::uint8_t* mask, unsigned long long* filled, cudaStream_t s, int batch = 1);

struct OdtConfig {
  Grid grid{};
  int count = 0;       // fields (illuminations)
  int iterations = 0;  // missing-cone iterations; 0: plain Rytov ODT
  bool tv = false;     // FISTA-TV instead of Gerchberg-Papoulis
  bool r2c = true;     // GP on half spectra (the TV solver always is)
  float lambda = 0;    // TV weight times k0^2
  int tv_inner = 10;
  float nm2 = 0;       // n_medium^2
  float inv_k02 = 0;   // 1 / k0^2
  int batch = 1;       // independent reconstructions of this geometry per run (not with TV)
};

// Two CUDA events owned together (start and end of a timed span); destroyed with their owner.
class EventPair {
 public:
  EventPair() {
    check(cudaEventCreate(&a_), "cudaEventCreate");
    check(cudaEventCreate(&b_), "cudaEventCreate");
  }
  ~EventPair() {
    if (a_) cudaEventDestroy(a_);
    if (b_) cudaEventDestroy(b_);
  }
  EventPair(EventPair&& o) noexcept : a_(std::exchange(o.a_, nullptr)), b_(std::exchange(o.b_, nullptr)) {}
  EventPair& operator=(EventPair&& o) noexcept {
    std::swap(a_, o.a_);
    std::swap(b_, o.b_);
    return *this;
  }
  EventPair(const EventPair&) = delete;
  EventPair& operator=(const EventPair&) = delete;
  [[nodiscard]] cudaEvent_t start() const { return a_; }
  [[nodiscard]] cudaEvent_t end() const { return b_; }

 private:
  cudaEvent_t a_ = nullptr, b_ = nullptr;
};

class OdtPlan {
 public:
  // Stage marks recorded by run() when a clock is given, in this order.
  enum Mark { kMarkFft2, kMarkClear, kMarkMapping, kMarkNormalize, kMarkSolve, kMarkFinish, kMarks };

  // illum_fyfx: count (fy, fx) pairs on the host.
  OdtPlan(const OdtConfig& cfg, const float* illum_fyfx);

  // fields: (batch * count, n, n) Rytov fields on the device, overwritten by their spectra. index:
  // (batch, nz, n, n) output on the device. Clock marks are `first + Mark`.
  void run(float2* fields, float* index, cudaStream_t s, StageClock* clock = nullptr);
  void run_marked(float2* fields, float* index, cudaStream_t s, StageClock* clock, int first) {
    first_mark_ = first;
    run(fields, index, s, clock);
    first_mark_ = 0;
  }

  // Voxels that received data in the last run, on the device (one count per volume of the batch).
  [[nodiscard]] const unsigned long long* filled() const { return filled_.get(); }
  // Device counter of the plan's bounded waits that ran out, over its whole life (never reset):
  // a caller compares it before and after its runs.
  [[nodiscard]] const unsigned long long* wait_count() const { return waits_.get(); }
  [[nodiscard]] std::size_t volume() const { return vol_; }  // of one reconstruction
  [[nodiscard]] std::size_t device_bytes() const;
  [[nodiscard]] const OdtConfig& config() const { return cfg_; }

  // Device time of the FISTA-TV proximal steps inside runs (every outer iteration's but the last, which
  // also writes the index): CUDA events on the run's stream around each step, from enable_prox_timing(true)
  // on, in runs launched directly (not under stream capture). prox_timing() waits for the events and returns
  // the milliseconds and the kernel launches they cover, and starts a new count.
  void enable_prox_timing(bool on);
  std::pair<double, std::uint64_t> prox_timing();

 private:
  void mark(StageClock* clock, int m, cudaStream_t s) const;
  void tune();
  void solve_real(float* index, float inv, cudaStream_t s);
  void solve_complex(float* index, float inv, cudaStream_t s);

  OdtConfig cfg_;
  bool real_ = false;
  std::size_t half_ = 0;
  std::size_t vol_ = 0;
  int first_mark_ = 0;
  DevBuf<float4> illum_;
  DevBuf<unsigned long long> filled_;
  DevBuf<unsigned long long> waits_;
  DevBuf<float2> a_;
  DevBuf<std::uint8_t> hits_;
  DevBuf<float2> e_;
  DevBuf<float> x_;
  DevBuf<float> xprev_;
  DevBuf<float> dual_;
  std::vector<TvBuffers> tv_;  // per volume of a batch (FISTA-TV)
  bool prox_timing_ = false;
  std::vector<EventPair> prox_events_;
  std::uint64_t prox_launches_ = 0;
  DevBuf<float2> pot_;
  DevBuf<std::uint8_t> mask_;
  DevBuf<float2> measured_;
};

}  // namespace qhk
