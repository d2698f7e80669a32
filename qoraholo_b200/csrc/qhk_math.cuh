// Device restatement of the index and physics expressions the reference evaluates on both of its
// backends (src/common.hpp). Every float operation that decides a result bit for bit -- the
// Ewald-sphere indices, the FGP dual step, the accumulation order of the mapping -- is written
// with round-to-nearest intrinsics (__fadd_rn, __fmul_rn, ...), which nvcc never contracts into
// fused multiply-adds, so the device evaluates exactly the IEEE operations of the host code.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace qhk {

constexpr float kPiF = 3.14159265358979323846f;

__host__ __device__ __forceinline__ float parity(int i) { return (i & 1) ? -1.0f : 1.0f; }
__host__ __device__ __forceinline__ int signed_bin(int k, int n) { return k < n / 2 ? k : k - n; }
__host__ __device__ __forceinline__ int negative_bin(int k, int n) { return k == 0 ? 0 : n - k; }
// Makhoul reordering of a DCT-II of length n: x[i] goes to v[dct_position(i, n)].
__host__ __device__ __forceinline__ int dct_position(int i, int n) {
  return (i & 1) ? n - 1 - (i >> 1) : (i >> 1);
}

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b)
__device__ __forceinline__ float2 cmulc(float2 a, float2 b) {
  return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
__device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }

// p - 2 pi floor((p + pi) / 2 pi) in the host's operation order. For x = p + pi in (-3, 12) -- every
// difference of two phases in [-pi, pi] -- the floor of the correctly rounded quotient x / 2pi is -1, 0
// or 1, and since that quotient is monotonic in x it is decided by comparisons: it is 1 exactly from
// x = 2pi on (x just below 2pi gives a quotient one or two units below 1 in the last place, which rounds
// below 1), and below 0 exactly for x < 0 (x is then at least 2^-23 in magnitude, p and pi being floats
// near pi, so the quotient does not round to -0). Outside that range the division runs. Either way the
// result is bitwise that of the division.
__device__ __forceinline__ float wrap_phase(float p) {
  const float two_pi = __fmul_rn(2.0f, kPiF);
  const float x = __fadd_rn(p, kPiF);
  float f;
  if (x > -3.0f && x < 12.0f) {
    f = x < 0.0f ? -1.0f : (x >= two_pi ? 1.0f : 0.0f);
  } else {
    f = floorf(__fdiv_rn(x, two_pi));
  }
  return __fsub_rn(p, __fmul_rn(two_pi, f));
}

// k-space grid of the Ewald mapping: lateral side n, axial side nz; frequencies in cycles/um.
struct Grid {
  int n;
  int nz;
  float df;    // 1 / (n * pixel)
  float dfz;   // 1 / (nz * pixel)
  float fm2;   // (n_medium / wavelength)^2
  float fna2;  // (na / wavelength)^2
  float gain;  // 4 pi / pixel
};

// Axial bin (wrapped to [0, nz)) and nu_z of lateral bin (ky, kx) for an illumination
// (fiy, fix, fiz); false outside the detection pupil, the medium or the grid. The operations are
// those of the reference's ewald_target, one IEEE operation each.
__device__ __forceinline__ bool ewald_target(const Grid& g, int ky, int kx, float fiy, float fix,
                                             float fiz, int& kz, float& nuz) {
  const float fy = __fadd_rn(__fmul_rn(static_cast<float>(signed_bin(ky, g.n)), g.df), fiy);
  const float fx = __fadd_rn(__fmul_rn(static_cast<float>(signed_bin(kx, g.n)), g.df), fix);
  const float rho2 = __fadd_rn(__fmul_rn(fy, fy), __fmul_rn(fx, fx));
  if (rho2 > g.fna2 || rho2 >= g.fm2) return false;
  nuz = __fsqrt_rn(__fsub_rn(g.fm2, rho2));
  const int k = static_cast<int>(floorf(__fadd_rn(__fdiv_rn(__fsub_rn(nuz, fiz), g.dfz), 0.5f)));
  if (k < -g.nz / 2 || k >= g.nz / 2) return false;
  kz = k < 0 ? k + g.nz : k;
  return true;
}

// 1 / sqrt(x) with the two roundings of the host's 1.0f / std::sqrt(x) -- RN(1 / RN(sqrt(x))) -- for
// x >= 1 (the dual projection's factor), from the hardware's approximate reciprocal square root and
// reciprocal refined with fused multiply-adds after Markstein (P. Markstein, "IA-64 and Elementary
// Functions", 2000, the Newton-Raphson refinements with an exactly computed residual): the root as g = x y
// from y ~ 1 / sqrt(x), corrected by the residual x - g^2 times y / 2; its reciprocal from z ~ 1 / s
// refined once by z + z (1 - s z). Equal to __frcp_rn(__fsqrt_rn(x)) for every float in [1, 2^126),
// checked exhaustively on the device (qhk_selftest_rcp_sqrt); above that, and for NaN, the IEEE intrinsics
// run. (Further refinements of y and z were checked exhaustively too; none changes a single result.)
__device__ __forceinline__ float rcp_sqrt_rn(float x) {
  if (!(x < 0x1p126f)) return __frcp_rn(__fsqrt_rn(x));
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  const float g = __fmul_rn(x, y);
  const float r = __fmaf_rn(-g, g, x);
  const float s = __fmaf_rn(r, __fmul_rn(0.5f, y), g);
  float z;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(z) : "f"(s));
  return __fmaf_rn(__fmaf_rn(-s, z, 1.0f), z, z);
}

// One FGP dual step at a voxel (Beck & Teboulle's FGP on the TV dual): q = r + step g,
// projection onto the unit ball, momentum. Same operation order as the host, unfused.
__device__ __forceinline__ void tv_dual_step(const float g[3], float step, float momentum,
                                             float p[3], float r[3]) {
  float q[3];
  float norm2 = 0.0f;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    q[a] = __fadd_rn(r[a], __fmul_rn(step, g[a]));
    norm2 = __fadd_rn(norm2, __fmul_rn(q[a], q[a]));
  }
  // 1 / sqrt(norm2) with two roundings as the host's 1.0f / std::sqrt(norm2) where norm2 > 1, else 1:
  // rcp_sqrt_rn(max(norm2, 1)), without a branch (exactly 1 at 1; max(NaN, 1) = 1).
  const float scale = rcp_sqrt_rn(fmaxf(norm2, 1.0f));
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const float next = __fmul_rn(q[a], scale);
    r[a] = __fadd_rn(next, __fmul_rn(momentum, __fsub_rn(next, p[a])));
    p[a] = next;
  }
}

// The projection part of tv_dual_step alone: p = proj(r + step g), the same operations.
__device__ __forceinline__ void tv_dual_project(const float g[3], float step, const float r[3], float p[3]) {
  float q[3];
  float norm2 = 0.0f;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    q[a] = __fadd_rn(r[a], __fmul_rn(step, g[a]));
    norm2 = __fadd_rn(norm2, __fmul_rn(q[a], q[a]));
  }
  // 1 / sqrt(norm2) with two roundings as the host's 1.0f / std::sqrt(norm2) where norm2 > 1, else 1:
  // rcp_sqrt_rn(max(norm2, 1)), without a branch (exactly 1 at 1; max(NaN, 1) = 1).
  const float scale = rcp_sqrt_rn(fmaxf(norm2, 1.0f));
#pragma unroll
  for (int a = 0; a < 3; ++a) p[a] = __fmul_rn(q[a], scale);
}

// Primal point max(b - lambda adj, 0).
__device__ __forceinline__ float tv_primal(float b, float lambda, float adj) {
  const float x = __fsub_rn(b, __fmul_rn(lambda, adj));
  return x > 0.0f ? x : 0.0f;
}

// Real part of the principal sqrt(n_m^2 + O / k0^2).
__device__ __forceinline__ float index_from_potential(float re, float im, float nm2, float inv_k02) {
  const float a = __fadd_rn(nm2, __fmul_rn(re, inv_k02));
  const float b = __fmul_rn(im, inv_k02);
  return __fsqrt_rn(__fmul_rn(0.5f, __fadd_rn(hypotf(a, b), a)));
}

}  // namespace qhk
