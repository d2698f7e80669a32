// Host side of the TMA loads: tensor maps of dense float volumes, encoded by the driver's
// cuTensorMapEncodeTiled (reached through the runtime's driver entry point, so that the library
// does not link libcuda itself).
#include <mutex>

#include "qhk_internal.hpp"
#include "tma.cuh"

namespace qhk {

namespace {

using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                 const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled encoder() {
  static EncodeTiled fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult status{};
    check(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &status),
          "cudaGetDriverEntryPoint(cuTensorMapEncodeTiled)");
    require(status == cudaDriverEntryPointSuccess && p != nullptr, "tma: cuTensorMapEncodeTiled is not available");
    fn = reinterpret_cast<EncodeTiled>(p);
  });
  return fn;
}

// One thread waits on an mbarrier that nothing arrives at, with the bounded wait of the TMA
// kernels: the wait runs out after `polls` polls and is counted in *counter. No load is in flight,
// so the CTA can leave at once.
__global__ void k_wait_probe(unsigned long long* counter, int polls) {
  __shared__ __align__(8) std::uint64_t bar;
  tma::mbar_init(&bar, 1);
  tma::mbar_wait(&bar, 0, counter, polls);
}

}  // namespace

void bounded_wait_probe(unsigned long long* counter, int polls, cudaStream_t s) {
  require(counter != nullptr && polls >= 1, "wait_probe: invalid arguments");
  k_wait_probe<<<1, 1, 0, s>>>(counter, polls);
  check_launch("wait probe");
}

CUtensorMap volume_tensor_map(const float* base, int nx, int ny, int nz, int box_x, int box_y) {
  require(base != nullptr && reinterpret_cast<std::uintptr_t>(base) % 16 == 0, "tma: volume must be 16-byte aligned");
  require(nx % 4 == 0 && nx >= 4 && ny >= 1 && nz >= 1, "tma: rows must be a multiple of 4 floats");
  require(box_x >= 4 && box_x <= 256 && box_x % 4 == 0 && box_y >= 1 && box_y <= 256, "tma: box out of range");
  CUtensorMap map{};
  const cuuint64_t dims[3] = {static_cast<cuuint64_t>(nx), static_cast<cuuint64_t>(ny), static_cast<cuuint64_t>(nz)};
  const cuuint64_t strides[2] = {static_cast<cuuint64_t>(nx) * sizeof(float),
                                 static_cast<cuuint64_t>(nx) * ny * sizeof(float)};
  const cuuint32_t box[3] = {static_cast<cuuint32_t>(box_x), static_cast<cuuint32_t>(box_y), 1};
  const cuuint32_t elem[3] = {1, 1, 1};
  const CUresult r = encoder()(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float*>(base), dims, strides, box,
                               elem, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                               CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  require(r == CUDA_SUCCESS, "tma: cuTensorMapEncodeTiled failed");
  return map;
}

}  // namespace qhk
