// Launch-shape autotuner: times candidate tile shapes of a kernel family on the device and keeps the
// fastest per (device, family, shape), for the rest of the process.
//
// Tuning runs when a plan is built (never inside a stream capture): each candidate is launched on
// the plan's own scratch buffers, twice to warm up and then `reps` times between CUDA events, and
// the candidate with the smallest time wins. Kernels then read their shape from the table, falling
// back to a fixed heuristic when a shape was never tuned (or tuning is off: QHK_AUTOTUNE=0). With
// QHK_AUTOTUNE_FILE set, choices are also read from and appended to that file, so that another run
// (a profiled one, say) uses the same shapes without timing them again. The tile-shape choices only
// change how work is tiled, never the arithmetic of any output element, so results are bitwise the same
// whichever shape wins. The FFT decomposition of the axis passes (family axis_engine) does change the
// rounding, so it is timed only when radix tuning is switched on (QHK_AUTOTUNE_RADIX=1,
// qhk_autotune_radix): results then stay within the oracle's tolerance but depend on which variant won.
#pragma once

#include <array>
#include <functional>
#include <string>
#include <vector>

#include "qhk_util.cuh"

namespace qhk {

enum class TuneFamily : int {
  axis = 0,         // FFT axis pass: columns per CTA
  fgp = 1,          // FGP step: rows per CTA
  axis_engine = 2,  // FFT axis pass: decomposition (register variants, staged engine); opt-in
};

struct TuneKey {
  int device = 0;
  TuneFamily family = TuneFamily::axis;
  std::array<long long, 6> shape{};
  bool operator<(const TuneKey& o) const;
};

TuneKey tune_key(TuneFamily family, std::array<long long, 6> shape);

// The tuned choice for `key`, or `fallback` when there is none or tuning is off.
int tuned_choice(const TuneKey& key, int fallback);
// True when `key` has a tuned choice.
bool is_tuned(const TuneKey& key);
// Autotuning on (default) unless QHK_AUTOTUNE=0 or qhk_autotune_enable(0).
bool autotune_enabled();
void set_autotune_enabled(bool on);

// Times run(c) for every candidate c on stream s and records the fastest for `key` (once per key:
// a tuned key is not timed again). No-op, returning the fallback, when tuning is off, the key has
// a single candidate or s is capturing. Returns the choice in effect.
int autotune(const TuneKey& key, const std::vector<int>& candidates, int fallback,
             const std::function<void(int)>& run, cudaStream_t s, int reps = 3);

// One line per tuned key: family, shape, choice, and the time of every candidate in microseconds.
std::string autotune_report();

}  // namespace qhk
