// Device self-checks of arithmetic helpers that restate IEEE operations with other instructions: every
// input of the helper's domain is run through it and through the IEEE intrinsics it replaces, and the
// mismatches are counted (qhk_selftest_rcp_sqrt).
#include <cstdint>

#include "qhk_internal.hpp"

namespace qhk {

namespace {

__global__ void k_check_rcp_sqrt(std::uint32_t first, std::uint32_t last, unsigned long long* bad,
                                 unsigned* first_bad) {
  const std::uint32_t stride = gridDim.x * blockDim.x;
  for (std::uint32_t b = first + blockIdx.x * blockDim.x + threadIdx.x; b < last; b += stride) {
    const float x = __uint_as_float(b);
    const float want = __frcp_rn(__fsqrt_rn(x));
    const float got = rcp_sqrt_rn(x);
    if (__float_as_uint(want) != __float_as_uint(got)) {
      atomicAdd(bad, 1ull);
      atomicMin(first_bad, b);
    }
  }
}

}  // namespace

void selftest_rcp_sqrt(unsigned long long* mismatches, unsigned* first_bad) {
  DevBuf<unsigned long long> bad(1);
  DevBuf<unsigned> first(1);
  check(cudaMemset(bad.get(), 0, sizeof(unsigned long long)), "cudaMemset");
  check(cudaMemset(first.get(), 0xff, sizeof(unsigned)), "cudaMemset");
  // Every float in [1, 2^126): the helper's fast domain (1 itself for the branch-free projection).
  const std::uint32_t lo = 0x3f800000u, hi = 0x7e800000u;
  int sms = 0;
  check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0), "cudaDeviceGetAttribute");
  k_check_rcp_sqrt<<<sms * 8, 256>>>(lo, hi, bad.get(), first.get());
  check_launch("selftest rcp_sqrt");
  check(cudaMemcpy(mismatches, bad.get(), sizeof(unsigned long long), cudaMemcpyDeviceToHost), "cudaMemcpy");
  check(cudaMemcpy(first_bad, first.get(), sizeof(unsigned), cudaMemcpyDeviceToHost), "cudaMemcpy");
}

}  // namespace qhk
