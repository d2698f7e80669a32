// Device self-checks of arithmetic helpers that restate IEEE operations with other instructions: every
// input of the helper's domain is run through it and through the IEEE intrinsics it replaces, and the
// mismatches are counted (qhk_selftest_rcp_sqrt).
#include <cstdint>

#include "qhk_internal.hpp"
#include "rcp_sqrt2.cuh"

namespace qhk {

namespace {

// The scalar form, and the packed form with the input in either lane (the other lane's input the next
// float), against the IEEE pair. neg_zero is -0 from the launch, as the FGP kernels pass it.
__global__ void k_check_rcp_sqrt(std::uint32_t first, std::uint32_t last, float neg_zero, unsigned long long* bad,
                                 unsigned* first_bad) {
  const std::uint32_t stride = gridDim.x * blockDim.x;
  const float2 nz = make_float2(neg_zero, neg_zero);
  for (std::uint32_t b = first + blockIdx.x * blockDim.x + threadIdx.x; b < last; b += stride) {
    const float x = __uint_as_float(b);
    const float x1 = __uint_as_float(b + 1 < last ? b + 1 : first);
    const unsigned want = __float_as_uint(__frcp_rn(__fsqrt_rn(x)));
    const float2 lo = rcp_sqrt_rn2(make_float2(x, x1), nz);
    const float2 hi = rcp_sqrt_rn2(make_float2(x1, x), nz);
    if (__float_as_uint(rcp_sqrt_rn(x)) != want || __float_as_uint(lo.x) != want || __float_as_uint(hi.y) != want) {
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
  k_check_rcp_sqrt<<<sms * 8, 256>>>(lo, hi, -0.0f, bad.get(), first.get());
  check_launch("selftest rcp_sqrt");
  check(cudaMemcpy(mismatches, bad.get(), sizeof(unsigned long long), cudaMemcpyDeviceToHost), "cudaMemcpy");
  check(cudaMemcpy(first_bad, first.get(), sizeof(unsigned), cudaMemcpyDeviceToHost), "cudaMemcpy");
}

}  // namespace qhk
