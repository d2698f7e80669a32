// rcp_sqrt_rn (qhk_math.cuh) on a pair of lanes with Blackwell's packed FP32 instructions: each lane goes
// through exactly the operations of the scalar form -- the products as fma.rn.f32x2 with an addend of -0
// that the caller passes in from a kernel argument (so that the compiler cannot fold the addend and fuse
// the product with a neighbouring add), the refinements as fma.rn.f32x2 -- so each lane's result is the
// scalar one bit for bit (checked exhaustively on the device with the scalar form, qhk_selftest_rcp_sqrt).
#pragma once

#include <cuda_runtime.h>

#include "qhk_math.cuh"

namespace qhk {

__device__ __forceinline__ unsigned long long rsq2_pack(float2 v) {
  return (static_cast<unsigned long long>(__float_as_uint(v.y)) << 32) | __float_as_uint(v.x);
}
__device__ __forceinline__ float2 rsq2_unpack(unsigned long long d) {
  return make_float2(__uint_as_float(static_cast<unsigned>(d)), __uint_as_float(static_cast<unsigned>(d >> 32)));
}
__device__ __forceinline__ float2 rsq2_fma(float2 a, float2 b, float2 c) {
  unsigned long long d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(rsq2_pack(a)), "l"(rsq2_pack(b)), "l"(rsq2_pack(c)));
  return rsq2_unpack(d);
}

// -a on both lanes as one packed subtraction from -0: (-0) - a = -a for every a, signed zeros included
// ((-0) - (+0) = -0, (-0) - (-0) = +0), where negating each lane on its own costs an instruction per lane.
__device__ __forceinline__ float2 rsq2_neg(float2 a, float2 neg_zero) {
  unsigned long long d;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(rsq2_pack(neg_zero)), "l"(rsq2_pack(a)));
  return rsq2_unpack(d);
}

// Both lanes in [1, 2^126) take the packed path; otherwise each lane runs the scalar form.
__device__ __forceinline__ float2 rcp_sqrt_rn2(float2 x, float2 neg_zero) {
  if (!(x.x < 0x1p126f && x.y < 0x1p126f)) return make_float2(rcp_sqrt_rn(x.x), rcp_sqrt_rn(x.y));
  float2 y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y.x) : "f"(x.x));
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y.y) : "f"(x.y));
  const float2 g = rsq2_fma(x, y, neg_zero);                                   // x y
  const float2 r = rsq2_fma(rsq2_neg(g, neg_zero), g, x);                      // x - g^2
  const float2 h = rsq2_fma(make_float2(0.5f, 0.5f), y, neg_zero);             // y / 2
  const float2 s = rsq2_fma(r, h, g);
  float2 z;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(z.x) : "f"(s.x));
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(z.y) : "f"(s.y));
  const float2 e = rsq2_fma(rsq2_neg(s, neg_zero), z, make_float2(1.0f, 1.0f));  // 1 - s z
  return rsq2_fma(e, z, z);
}

}  // namespace qhk
