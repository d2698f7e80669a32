// Hologram synthesis on the device (synth.cu).
#pragma once

#include "qhk_util.cuh"

namespace qhk {

// ratio: (count, n, n) complex64 field ratios on the device -> out: (count, n, n) float32 holograms
// on the device; illum_fyfx on the host. Returns when done.
void synthesize_holograms_device(const float2* ratio, const float* illum_fyfx, int count, int n, double pixel,
                                 double carrier_y, double carrier_x, double amplitude, float noise,
                                 unsigned long long seed, float* out, cudaStream_t s);

}  // namespace qhk
