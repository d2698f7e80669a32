// Tensor-memory-accelerator (TMA) loads of volume tiles into shared memory, completed on an
// mbarrier: the host encodes a 3-D tensor map of a dense (nz, ny, nx) float volume, and one thread
// of a CTA issues cp.async.bulk.tensor loads of (box_y rows x box_x floats) boxes that land in
// shared memory and count their bytes on the slot's mbarrier; the consumers wait on its phase.
// Loads only, from this GPU's own memory, and without cluster multicast. Boxes that reach outside
// the volume (negative or too large y, x beyond nx) are filled with zeros by the hardware. The box's
// x coordinate is always 0 (16-byte aligned); box_x * 4 bytes must be a multiple of 16 and the
// shared destination 128-byte aligned.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "debug.cuh"

namespace qhk {

// Tensor map of the volume at `base` (dense nz x ny x nx floats, 16-byte aligned, nx % 4 == 0)
// with boxes of box_x floats by box_y rows by one plane.
CUtensorMap volume_tensor_map(const float* base, int nx, int ny, int nz, int box_x, int box_y);

namespace tma {

__device__ __forceinline__ std::uint32_t smem_addr(const void* p) {
  return static_cast<std::uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(std::uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

// The issuing thread's arrival, announcing `bytes` of transactions that complete the phase.
__device__ __forceinline__ void mbar_expect(std::uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}

// Orders this thread's earlier shared-memory accesses (generic proxy) before the async-proxy
// writes of TMA loads it issues next.
__device__ __forceinline__ void fence_async_shared() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

// Box at (x, y, z) of `map` into dst, completing on `bar`. The debug build skips (and records) a box
// whose x is not on a 16-byte boundary or whose destination or mbarrier is misaligned.
__device__ __forceinline__ void load_3d(void* dst, const CUtensorMap* map, int x, int y, int z, std::uint64_t* bar) {
  if (!QHK_CHECK((x & 3) == 0 && (smem_addr(dst) & 127u) == 0 && (smem_addr(bar) & 7u) == 0)) return;
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];\n" ::"r"(smem_addr(dst)),
      "l"(reinterpret_cast<std::uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_addr(bar))
      : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(std::uint64_t* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait for the phase `parity` of `bar`: false, and *timeouts incremented, if it has not
// completed after `limit` polls (each suspends the thread for at most a short hardware-defined
// time), so that a load that never lands ends the wait with an error the host can read.
constexpr int kWaitLimit = 1 << 20;
__device__ __forceinline__ bool mbar_wait(std::uint64_t* bar, unsigned parity, unsigned long long* timeouts,
                                          int limit = kWaitLimit) {
  for (int i = 0; i < limit; ++i) {
    if (mbar_try_wait(bar, parity)) return true;
  }
  atomicAdd(timeouts, 1ull);
  return false;
}

}  // namespace tma

}  // namespace qhk
