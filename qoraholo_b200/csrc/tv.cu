// Total-variation proximal step by FGP on the dual (Beck & Teboulle 2009), the dominant cost of
// the FISTA-TV reconstruction (it follows the reference's tv_prox, src/cuda/tv.cu:256-293, and
// its CPU form src/cpu/tv.cpp:7-44, with the per-voxel math of src/common.hpp:107-153).
//
// One FGP step is one kernel of exactly one wave of CTAs. The (y-tile, z) plane units -- TY full
// rows (all x) of one plane -- are split evenly over the CTAs in y-tile-major order, and a CTA
// marches along z through its units (one march per y-tile it touches). Shared memory holds a
// three-plane ring of the input dual r (rows y0-1 .. y0+TY, three components), filled by cp.async
// one plane ahead, and the primal point z = max(b - lambda L(r), 0) for two planes (rows y0 ..
// y0+TY): z of plane k+1 is computed once from the ring and reused as plane k of the next step, so
// z is never written to HBM, and each r value is read from HBM once (the one-row halos come from
// L2). Per step the HBM traffic is b, r_in (3), p (3) read and p (3), r_out (3) written -- 13
// volumes; the first step reads p as r (10 volumes) and the last writes no r (10 volumes).
//
// Two steps per pass (k_fgp2, for float4 rows of at most 256 x values): a CTA also computes the first
// step's primal and dual on the rows beyond its tile that the second step reads, so one pass moves 13
// volumes for two steps. r, b and p arrive as TMA box loads counted on mbarriers (bounded waits), the
// arithmetic runs on pairs of x points with the packed FP32 instructions, and 256^3 volumes run an
// instantiation with the sizes compiled in.
//
// All arithmetic uses the round-to-nearest intrinsics in the reference's operation order, so the
// device iterates are bit-identical to the CPU's.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <mutex>
#include <set>
#include <vector>

#include "autotune.hpp"
#include "qhk_internal.hpp"
#include "rcp_sqrt2.cuh"
#include "tma.cuh"

namespace qhk {

namespace {

struct FgpArgs {
  const float* b;
  const float* rin[3];
  const float* pin[3];
  float* pout[3];
  float* rout[3];
  int nz, ny, nx;
  int ytiles;  // ceil(ny / TY)
  float lambda, step, momentum;
};

template <int VEC>
struct Vec;
template <>
struct Vec<4> {
  using T = float4;
  __device__ static void load(const float* p, float* v) {
    const float4 t = *reinterpret_cast<const float4*>(p);
    v[0] = t.x, v[1] = t.y, v[2] = t.z, v[3] = t.w;
  }
  __device__ static void store(float* p, const float* v) {
    *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
  }
};
template <>
struct Vec<1> {
  __device__ static void load(const float* p, float* v) { v[0] = *p; }
  __device__ static void store(float* p, const float* v) { *p = v[0]; }
};

// Asynchronous 16-byte (VEC = 4) or 4-byte (VEC = 1) global -> shared copies (cp.async), grouped
// per plane so that plane z+2 streams in while plane z+1's primal point and plane z's dual step are
// computed.
template <int VEC>
__device__ __forceinline__ void copy_async(float* dst, const float* src) {
  const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
  if constexpr (VEC == 4) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src));
  } else {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(src));
  }
}
__device__ __forceinline__ void copy_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void copy_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

template <int VEC, bool FIRST, bool LAST>
__global__ void __launch_bounds__(256, 3) k_fgp(FgpArgs A) {
  extern __shared__ __align__(16) float sm[];
  const int nx = A.nx, ny = A.ny, nz = A.nz;
  const int TY = static_cast<int>(blockDim.y);
  const int tx = static_cast<int>(threadIdx.x);
  const int ty = static_cast<int>(threadIdx.y);
  const int x0 = tx * VEC;
  const int ring_rows = TY + 2;
  const std::size_t plane_sz = static_cast<std::size_t>(3) * ring_rows * nx;
  const std::size_t zb_sz = static_cast<std::size_t>(TY + 1) * nx;
  // Ring of r planes: plane z lives in slot (z - z0 + 1) % 3 (plane z0 - 1 in slot 0).
  float* R = sm;
  float* Z = sm + 3 * plane_sz;  // primal of plane z in slot (z - z0) & 1
  float* Bs = Z + 2 * zb_sz;     // b of plane z in slot (z - z0) & 1
  const std::size_t nxy = static_cast<std::size_t>(nx) * ny;
  // This CTA's share of the (y-tile, z) plane units, y-tile major: an even split over a grid that
  // is exactly one wave, walked as one z-march per y-tile it touches.
  const long long units = static_cast<long long>(A.ytiles) * nz;
  const long long u_end = units * (blockIdx.x + 1) / gridDim.x;
  for (long long u = units * blockIdx.x / gridDim.x; u < u_end;) {
    const int y0 = static_cast<int>(u / nz) * TY;
    const int z0 = static_cast<int>(u % nz);
    const int z1 = static_cast<int>(min(static_cast<long long>(nz), z0 + (u_end - u)));
    u += z1 - z0;
    const int zlast = min(z1, nz - 1);  // last plane whose dual r is needed (for the primal of z1)
    const auto rslot = [&](int z) { return R + static_cast<std::size_t>((z - z0 + 1) % 3) * plane_sz; };
    const auto zslot = [&](int z) { return Z + static_cast<std::size_t>((z - z0) & 1) * zb_sz; };
    const auto bslot = [&](int z) { return Bs + static_cast<std::size_t>((z - z0) & 1) * zb_sz; };

    // Rows outside the volume are never read by the arithmetic below (the boundary terms drop
    // them), so they are not copied.
    const auto issue_r = [&](int z, int comps) {
      float* dst = rslot(z);
      for (int rc = ty; rc < comps * ring_rows; rc += TY) {
        const int c = rc / ring_rows;
        const int rr = rc - c * ring_rows;
        const int y = y0 - 1 + rr;
        if (y < 0 || y >= ny) continue;
        copy_async<VEC>(dst + (static_cast<std::size_t>(c) * ring_rows + rr) * nx + x0,
                        A.rin[c] + static_cast<std::size_t>(z) * nxy + static_cast<std::size_t>(y) * nx + x0);
      }
    };
    const auto issue_b = [&](int z) {
      float* dst = bslot(z);
      for (int rr = ty; rr < TY + 1; rr += TY) {
        const int y = y0 + rr;
        if (y >= ny) continue;
        copy_async<VEC>(dst + static_cast<std::size_t>(rr) * nx + x0,
                        A.b + static_cast<std::size_t>(z) * nxy + static_cast<std::size_t>(y) * nx + x0);
      }
    };
    // z on plane z (rows y0 .. y0+TY) from r of that plane and of the plane below. Every thread runs
    // the same number of row iterations so that all lanes reach the shuffles; with VEC = 4 a thread
    // reads its four x values as one float4 and gets x - 1 from the lane on its left.
    const int linear = static_cast<int>(threadIdx.y * blockDim.x + threadIdx.x);
    const int lane = linear & 31;
    // Lanes that exist in this thread's warp (the block's last warp may be partial).
    const int warp_threads = min(32, static_cast<int>(blockDim.x * blockDim.y) - (linear & ~31));
    const unsigned lanes = warp_threads >= 32 ? 0xffffffffu : ((1u << warp_threads) - 1u);
    // One primal value from the ring: sum of the r differences in the host's order, then tv_primal.
    const auto primal_value = [&](int z, int y, int x, float vz, float vzb, float vy, float vym, float vx,
                                  float left, float vb) {
      float sacc = 0.0f;
      if (z < nz - 1) sacc = __fadd_rn(sacc, vz);
      if (z > 0) sacc = __fsub_rn(sacc, vzb);
      if (y < ny - 1) sacc = __fadd_rn(sacc, vy);
      if (y > 0) sacc = __fsub_rn(sacc, vym);
      if (x < nx - 1) sacc = __fadd_rn(sacc, vx);
      if (x > 0) sacc = __fsub_rn(sacc, left);
      return tv_primal(vb, A.lambda, sacc);
    };
    const auto primal = [&](int z) {
      const float* Rc = rslot(z);
      const float* Rb = rslot(z - 1);
      const float* B = bslot(z);
      float* Zd = zslot(z);
      {  // rows y0 .. y0 + TY - 1: one row per thread row, VEC values per thread
        const int rr = ty;
        const int y = y0 + rr;
        const float* rz = Rc + (0 * static_cast<std::size_t>(ring_rows) + rr + 1) * nx;
        const float* rzb = Rb + (0 * static_cast<std::size_t>(ring_rows) + rr + 1) * nx;
        const float* ry = Rc + (1 * static_cast<std::size_t>(ring_rows) + rr + 1) * nx;
        const float* rym = Rc + (1 * static_cast<std::size_t>(ring_rows) + rr) * nx;
        const float* rx = Rc + (2 * static_cast<std::size_t>(ring_rows) + rr + 1) * nx;
        float vz[VEC], vzb[VEC], vy[VEC], vym[VEC], vx[VEC], vb[VEC];
        Vec<VEC>::load(rz + x0, vz);
        Vec<VEC>::load(rzb + x0, vzb);
        Vec<VEC>::load(ry + x0, vy);
        Vec<VEC>::load(rym + x0, vym);
        Vec<VEC>::load(rx + x0, vx);
        Vec<VEC>::load(B + static_cast<std::size_t>(rr) * nx + x0, vb);
        float left;
        if constexpr (VEC == 4) {
          const float from_lane = __shfl_up_sync(lanes, vx[3], 1);
          left = (x0 > 0 && lane == 0) ? rx[x0 - 1] : from_lane;
        } else {
          left = x0 > 0 ? rx[x0 - 1] : 0.0f;
        }
        float out[VEC];
#pragma unroll
        for (int i = 0; i < VEC; ++i) {
          const int x = x0 + i;
          out[i] = y < ny ? primal_value(z, y, x, vz[i], vzb[i], vy[i], vym[i], vx[i],
                                         i == 0 ? left : vx[i > 0 ? i - 1 : 0], vb[i])
                          : 0.0f;
        }
        Vec<VEC>::store(Zd + static_cast<std::size_t>(rr) * nx + x0, out);
      }
      {  // row y0 + TY (the next tile's first row, needed for this tile's y gradient): spread over
         // all threads, one value each, so that no thread row waits for another.
        const int rr = TY;
        const int y = y0 + rr;
        if (y < ny) {
          const float* rz = Rc + (0 * static_cast<std::size_t>(ring_rows) + rr + 1) * nx;
          const float* rzb = Rb + (0 * static_cast<std::size_t>(ring_rows) + rr + 1) * nx;
          const float* ry = Rc + (1 * static_cast<std::size_t>(ring_rows) + rr + 1) * nx;
          const float* rym = Rc + (1 * static_cast<std::size_t>(ring_rows) + rr) * nx;
          const float* rx = Rc + (2 * static_cast<std::size_t>(ring_rows) + rr + 1) * nx;
          const float* vb = B + static_cast<std::size_t>(rr) * nx;
          float* out = Zd + static_cast<std::size_t>(rr) * nx;
          const int nthreads = static_cast<int>(blockDim.x * blockDim.y);
          for (int x = linear; x < nx; x += nthreads) {
            out[x] = primal_value(z, y, x, rz[x], rzb[x], ry[x], rym[x], rx[x], x > 0 ? rx[x - 1] : 0.0f, vb[x]);
          }
        }
      }
    };

  // Prologue: planes z0 - 1 (z component only), z0 (and b) in one group, z0 + 1 in the next.
    if (z0 > 0) issue_r(z0 - 1, 1);
    issue_r(z0, 3);
    issue_b(z0);
    copy_commit();
    const bool second = z0 + 1 <= zlast;
    if (second) {
      issue_r(z0 + 1, 3);
      issue_b(z0 + 1);
      copy_commit();
      copy_wait<1>();
    } else {
      copy_wait<0>();
    }
    __syncthreads();
    primal(z0);
    __syncthreads();

    const int y = y0 + ty;
    for (int z = z0; z < z1; ++z) {
      // Two barriers per plane: after the first every thread is past the previous plane's dual
      // step, so the ring slot and b slot of plane z + 2 (those of z - 1 and z) are free for the
      // prefetch, which then streams in during this plane's primal and dual steps.
      const std::size_t at = static_cast<std::size_t>(z) * nxy + static_cast<std::size_t>(y) * nx + x0;
      float pv[3][VEC];
      if (!FIRST && y < ny) {
#pragma unroll
        for (int c = 0; c < 3; ++c) Vec<VEC>::load(A.pin[c] + at, pv[c]);
      }
      copy_wait<0>();  // plane z + 1
      __syncthreads();
      if (z + 2 <= zlast) {
        issue_r(z + 2, 3);
        issue_b(z + 2);
        copy_commit();
      }
      if (z + 1 < nz) primal(z + 1);
      __syncthreads();
      {
        const float* Rc = rslot(z);
        float rv[3][VEC];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          Vec<VEC>::load(Rc + (static_cast<std::size_t>(c) * ring_rows + ty + 1) * nx + x0, rv[c]);
          if (FIRST) {
#pragma unroll
            for (int i = 0; i < VEC; ++i) pv[c][i] = rv[c][i];
          }
        }
        const float* zcp = zslot(z) + static_cast<std::size_t>(ty) * nx;
        float zc[VEC], zy[VEC], zz[VEC];
        Vec<VEC>::load(zcp + x0, zc);
        Vec<VEC>::load(zslot(z) + static_cast<std::size_t>(ty + 1) * nx + x0, zy);
        Vec<VEC>::load(zslot(z + 1) + static_cast<std::size_t>(ty) * nx + x0, zz);
        float right;
        if constexpr (VEC == 4) {
          const float from_lane = __shfl_down_sync(lanes, zc[0], 1);
          right = (x0 + VEC < nx && (lane == 31 || lane == warp_threads - 1)) ? zcp[x0 + VEC] : from_lane;
        } else {
          right = x0 + 1 < nx ? zcp[x0 + 1] : 0.0f;
        }
        if (y < ny) {
#pragma unroll
          for (int i = 0; i < VEC; ++i) {
            const int x = x0 + i;
            const float c = zc[i];
            float g[3];
            g[0] = z < nz - 1 ? __fsub_rn(c, zz[i]) : 0.0f;
            g[1] = y < ny - 1 ? __fsub_rn(c, zy[i]) : 0.0f;
            g[2] = x < nx - 1 ? __fsub_rn(c, i == VEC - 1 ? right : zc[i < VEC - 1 ? i + 1 : 0]) : 0.0f;
            float p[3] = {pv[0][i], pv[1][i], pv[2][i]};
            float r[3] = {rv[0][i], rv[1][i], rv[2][i]};
            tv_dual_step(g, A.step, A.momentum, p, r);
#pragma unroll
            for (int c2 = 0; c2 < 3; ++c2) {
              pv[c2][i] = p[c2];
              rv[c2][i] = r[c2];
            }
          }
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            Vec<VEC>::store(A.pout[c] + at, pv[c]);
            if (!LAST) Vec<VEC>::store(A.rout[c] + at, rv[c]);
          }
        }
      }
    }
    __syncthreads();  // the next march's prologue reuses the ring
  }
}

// The same FGP step without a stored extrapolated point: r_k = p_k + m (p_k - p_{k-1}) (the
// formula of the step above, the same float operations on the same stored values, so bitwise the
// same r) is recomputed where it is needed from the two previous duals. A step then reads b, p_k
// (3) and p_{k-1} (3) and writes p_{k+1} (3) -- 10 volumes instead of 13 (the first step, r_0 =
// p_0, reads b and p_0 and writes p_1: 7). The ring holds r: plane z+2's p_k lands in its ring
// slot and its p_{k-1} in a staging plane by cp.async, and each thread turns its own copied
// elements into r once they land. It is an autotuner candidate: on B200 at 256^3 it loses (274 vs
// 156 us per step), because the one-row halos of two duals are re-read from DRAM (709 MB read
// against 470 MB algorithmic) and the staging plane halves the resident CTAs.
struct FgpPArgs {
  const float* b;
  const float* pk[3];    // p_k; on the first step p_0 = r_0
  const float* pkm1[3];  // p_{k-1} (not read on the first step)
  float* pout[3];        // p_{k+1}
  int nz, ny, nx;
  int ytiles;
  float lambda, step;
  float momentum;  // m_{k-1}: r_k = p_k + m_{k-1} (p_k - p_{k-1})
};

template <int VEC, bool FIRST>
__global__ void __launch_bounds__(256, 2) k_fgp_p(FgpPArgs A) {
  extern __shared__ __align__(16) float sm[];
  const int nx = A.nx, ny = A.ny, nz = A.nz;
  const int TY = static_cast<int>(blockDim.y);
  const int tx = static_cast<int>(threadIdx.x);
  const int ty = static_cast<int>(threadIdx.y);
  const int x0 = tx * VEC;
  const int ring_rows = TY + 2;
  const std::size_t plane_sz = static_cast<std::size_t>(3) * ring_rows * nx;
  const std::size_t zb_sz = static_cast<std::size_t>(TY + 1) * nx;
  float* R = sm;                                // 3 slots: r of planes z, z+1; p_k of plane z+2
  float* S = R + 3 * plane_sz;                  // p_{k-1} of the plane in flight
  float* Z = S + (FIRST ? 0 : plane_sz);        // primal of plane z in slot (z - z0) & 1
  float* Bs = Z + 2 * zb_sz;                    // b of plane z in slot (z - z0) & 1
  const std::size_t nxy = static_cast<std::size_t>(nx) * ny;
  const int linear = static_cast<int>(threadIdx.y * blockDim.x + threadIdx.x);
  const int lane = linear & 31;
  const int warp_threads = min(32, static_cast<int>(blockDim.x * blockDim.y) - (linear & ~31));
  const unsigned lanes = warp_threads >= 32 ? 0xffffffffu : ((1u << warp_threads) - 1u);
  const float m = A.momentum;

  const long long units = static_cast<long long>(A.ytiles) * nz;
  const long long u_end = units * (blockIdx.x + 1) / gridDim.x;
  for (long long u = units * blockIdx.x / gridDim.x; u < u_end;) {
    const int y0 = static_cast<int>(u / nz) * TY;
    const int z0 = static_cast<int>(u % nz);
    const int z1 = static_cast<int>(min(static_cast<long long>(nz), z0 + (u_end - u)));
    u += z1 - z0;
    const int zlast = min(z1, nz - 1);  // last plane whose r is needed (for the primal of z1)
    const auto rslot = [&](int z) { return R + static_cast<std::size_t>((z - z0 + 1) % 3) * plane_sz; };
    const auto zslot = [&](int z) { return Z + static_cast<std::size_t>((z - z0) & 1) * zb_sz; };
    const auto bslot = [&](int z) { return Bs + static_cast<std::size_t>((z - z0) & 1) * zb_sz; };

    // Each thread copies, and later converts, the same elements: row-components rc = ty, ty + TY,
    // ... of the ring, x0 .. x0 + VEC - 1. Rows outside the volume are neither copied nor read.
    const auto issue_p = [&](int z, int comps) {
      float* dst = rslot(z);
      for (int rc = ty; rc < comps * ring_rows; rc += TY) {
        const int c = rc / ring_rows;
        const int rr = rc - c * ring_rows;
        const int y = y0 - 1 + rr;
        if (y < 0 || y >= ny) continue;
        const std::size_t off = static_cast<std::size_t>(z) * nxy + static_cast<std::size_t>(y) * nx + x0;
        const std::size_t at = (static_cast<std::size_t>(c) * ring_rows + rr) * nx + x0;
        copy_async<VEC>(dst + at, A.pk[c] + off);
        if (!FIRST) copy_async<VEC>(S + at, A.pkm1[c] + off);
      }
    };
    const auto convert = [&](int z, int comps) {
      if (FIRST) return;
      float* dst = rslot(z);
      for (int rc = ty; rc < comps * ring_rows; rc += TY) {
        const int c = rc / ring_rows;
        const int rr = rc - c * ring_rows;
        const int y = y0 - 1 + rr;
        if (y < 0 || y >= ny) continue;
        const std::size_t at = (static_cast<std::size_t>(c) * ring_rows + rr) * nx + x0;
        float pkv[VEC], pmv[VEC];
        Vec<VEC>::load(dst + at, pkv);
        Vec<VEC>::load(S + at, pmv);
#pragma unroll
        for (int i = 0; i < VEC; ++i) pkv[i] = __fadd_rn(pkv[i], __fmul_rn(m, __fsub_rn(pkv[i], pmv[i])));
        Vec<VEC>::store(dst + at, pkv);
      }
    };
    const auto issue_b = [&](int z) {
      float* dst = bslot(z);
      for (int rr = ty; rr < TY + 1; rr += TY) {
        const int y = y0 + rr;
        if (y >= ny) continue;
        copy_async<VEC>(dst + static_cast<std::size_t>(rr) * nx + x0,
                        A.b + static_cast<std::size_t>(z) * nxy + static_cast<std::size_t>(y) * nx + x0);
      }
    };
    // z on plane z (rows y0 .. y0+TY) from r of that plane and of the plane below (as k_fgp).
    const auto primal = [&](int z) {
      const float* Rc = rslot(z);
      const float* Rb = rslot(z - 1);
      const float* B = bslot(z);
      float* Zd = zslot(z);
      for (int it = 0; it < 2; ++it) {
        const int rr = ty + it * TY;
        const bool active = rr < TY + 1;
        const int rrc = active ? rr : 0;
        const int y = y0 + rrc;
        const float* rz = Rc + (0 * static_cast<std::size_t>(ring_rows) + rrc + 1) * nx;
        const float* rzb = Rb + (0 * static_cast<std::size_t>(ring_rows) + rrc + 1) * nx;
        const float* ry = Rc + (1 * static_cast<std::size_t>(ring_rows) + rrc + 1) * nx;
        const float* rym = Rc + (1 * static_cast<std::size_t>(ring_rows) + rrc) * nx;
        const float* rx = Rc + (2 * static_cast<std::size_t>(ring_rows) + rrc + 1) * nx;
        float vz[VEC], vzb[VEC], vy[VEC], vym[VEC], vx[VEC], vb[VEC];
        Vec<VEC>::load(rz + x0, vz);
        Vec<VEC>::load(rzb + x0, vzb);
        Vec<VEC>::load(ry + x0, vy);
        Vec<VEC>::load(rym + x0, vym);
        Vec<VEC>::load(rx + x0, vx);
        Vec<VEC>::load(B + static_cast<std::size_t>(rrc) * nx + x0, vb);
        float left;
        if constexpr (VEC == 4) {
          const float from_lane = __shfl_up_sync(lanes, vx[3], 1);
          left = (x0 > 0 && lane == 0) ? rx[x0 - 1] : from_lane;
        } else {
          left = x0 > 0 ? rx[x0 - 1] : 0.0f;
        }
        if (!active) continue;
        float out[VEC];
#pragma unroll
        for (int i = 0; i < VEC; ++i) {
          const int x = x0 + i;
          float zv = 0.0f;
          if (y < ny) {
            float sacc = 0.0f;
            if (z < nz - 1) sacc = __fadd_rn(sacc, vz[i]);
            if (z > 0) sacc = __fsub_rn(sacc, vzb[i]);
            if (y < ny - 1) sacc = __fadd_rn(sacc, vy[i]);
            if (y > 0) sacc = __fsub_rn(sacc, vym[i]);
            if (x < nx - 1) sacc = __fadd_rn(sacc, vx[i]);
            if (x > 0) sacc = __fsub_rn(sacc, i == 0 ? left : vx[i > 0 ? i - 1 : 0]);
            zv = tv_primal(vb[i], A.lambda, sacc);
          }
          out[i] = zv;
        }
        Vec<VEC>::store(Zd + static_cast<std::size_t>(rr) * nx + x0, out);
      }
    };

    // Prologue: plane z0 - 1 (z component only) and z0 landed and converted, z0 + 1 in flight.
    if (z0 > 0) {
      issue_p(z0 - 1, 1);
      copy_commit();
      copy_wait<0>();
      convert(z0 - 1, 1);
    }
    issue_p(z0, 3);
    issue_b(z0);
    copy_commit();
    copy_wait<0>();
    convert(z0, 3);
    if (z0 + 1 <= zlast) {
      issue_p(z0 + 1, 3);
      issue_b(z0 + 1);
      copy_commit();
    }
    __syncthreads();
    primal(z0);
    __syncthreads();

    const int y = y0 + ty;
    for (int z = z0; z < z1; ++z) {
      // Plane z + 1 (copied during the previous iteration): land and convert this thread's share,
      // then start plane z + 2 into the free ring slot and the staging plane.
      copy_wait<0>();
      if (z + 1 <= zlast) convert(z + 1, 3);
      if (z + 2 <= zlast) {
        issue_p(z + 2, 3);
        issue_b(z + 2);
        copy_commit();
      }
      __syncthreads();
      if (z + 1 < nz) primal(z + 1);
      __syncthreads();
      {
        const float* Rc = rslot(z);
        float rv[3][VEC];
#pragma unroll
        for (int c = 0; c < 3; ++c) Vec<VEC>::load(Rc + (static_cast<std::size_t>(c) * ring_rows + ty + 1) * nx + x0, rv[c]);
        const float* zcp = zslot(z) + static_cast<std::size_t>(ty) * nx;
        float zc[VEC], zy[VEC], zz[VEC];
        Vec<VEC>::load(zcp + x0, zc);
        Vec<VEC>::load(zslot(z) + static_cast<std::size_t>(ty + 1) * nx + x0, zy);
        Vec<VEC>::load(zslot(z + 1) + static_cast<std::size_t>(ty) * nx + x0, zz);
        float right;
        if constexpr (VEC == 4) {
          const float from_lane = __shfl_down_sync(lanes, zc[0], 1);
          right = (x0 + VEC < nx && (lane == 31 || lane == warp_threads - 1)) ? zcp[x0 + VEC] : from_lane;
        } else {
          right = x0 + 1 < nx ? zcp[x0 + 1] : 0.0f;
        }
        if (y < ny) {
          float pv[3][VEC];
#pragma unroll
          for (int i = 0; i < VEC; ++i) {
            const int x = x0 + i;
            const float c = zc[i];
            float g[3];
            g[0] = z < nz - 1 ? __fsub_rn(c, zz[i]) : 0.0f;
            g[1] = y < ny - 1 ? __fsub_rn(c, zy[i]) : 0.0f;
            g[2] = x < nx - 1 ? __fsub_rn(c, i == VEC - 1 ? right : zc[i < VEC - 1 ? i + 1 : 0]) : 0.0f;
            const float r[3] = {rv[0][i], rv[1][i], rv[2][i]};
            float p[3];
            tv_dual_project(g, A.step, r, p);
#pragma unroll
            for (int c2 = 0; c2 < 3; ++c2) pv[c2][i] = p[c2];
          }
          const std::size_t at = static_cast<std::size_t>(z) * nxy + static_cast<std::size_t>(y) * nx + x0;
#pragma unroll
          for (int c = 0; c < 3; ++c) Vec<VEC>::store(A.pout[c] + at, pv[c]);
        }
      }
      __syncthreads();
    }
  }
}

// Final primal point x = max(b - lambda L(p), 0), VEC voxels of one row per thread, and its use.
template <int VEC, int Mode>
__global__ void __launch_bounds__(256)
    k_tv_final(const float* b, const float* pz, const float* py, const float* px, int nz, int ny, int nx,
               float lambda, float momentum, float* xprev, float* out, float nm2, float inv_k02) {
  const std::size_t nxy = static_cast<std::size_t>(nx) * ny;
  const std::size_t total = nxy * nz / VEC;
  for (std::size_t t = blockIdx.x * static_cast<std::size_t>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<std::size_t>(gridDim.x) * blockDim.x) {
    const std::size_t i0 = t * VEC;
    const int x0 = static_cast<int>(i0 % nx);
    const int y = static_cast<int>((i0 / nx) % ny);
    const int z = static_cast<int>(i0 / nxy);
    float bv[VEC], cz[VEC], cy[VEC], cx[VEC], bz[VEC], by[VEC];
    Vec<VEC>::load(b + i0, bv);
    Vec<VEC>::load(pz + i0, cz);
    Vec<VEC>::load(py + i0, cy);
    Vec<VEC>::load(px + i0, cx);
    if (z > 0) Vec<VEC>::load(pz + i0 - nxy, bz);
    if (y > 0) Vec<VEC>::load(py + i0 - nx, by);
    const float left = x0 > 0 ? px[i0 - 1] : 0.0f;
    float xv[VEC];
#pragma unroll
    for (int i = 0; i < VEC; ++i) {
      const int x = x0 + i;
      float s = 0.0f;
      if (z < nz - 1) s = __fadd_rn(s, cz[i]);
      if (z > 0) s = __fsub_rn(s, bz[i]);
      if (y < ny - 1) s = __fadd_rn(s, cy[i]);
      if (y > 0) s = __fsub_rn(s, by[i]);
      if (x < nx - 1) s = __fadd_rn(s, cx[i]);
      if (x > 0) s = __fsub_rn(s, i == 0 ? left : cx[i > 0 ? i - 1 : 0]);
      xv[i] = tv_primal(bv[i], lambda, s);
    }
    if constexpr (Mode == static_cast<int>(TvFinal::plain)) {
      Vec<VEC>::store(out + i0, xv);
    } else if constexpr (Mode == static_cast<int>(TvFinal::momentum)) {
      float pv[VEC], yv[VEC];
      Vec<VEC>::load(xprev + i0, pv);
#pragma unroll
      for (int i = 0; i < VEC; ++i) yv[i] = __fadd_rn(xv[i], __fmul_rn(momentum, __fsub_rn(xv[i], pv[i])));
      Vec<VEC>::store(xprev + i0, xv);
      Vec<VEC>::store(out + i0, yv);
    } else {
#pragma unroll
      for (int i = 0; i < VEC; ++i) xv[i] = index_from_potential(xv[i], 0.0f, nm2, inv_k02);
      Vec<VEC>::store(out + i0, xv);
    }
  }
}

// Two FGP steps (k and k + 1) in one pass over the volume, so that a pair of steps moves the HBM
// traffic of one: b, r_k (3) and p_k (3) read, p_{k+2} (3) and r_{k+2} (3) written -- 13 volumes
// for two steps (the first pair reads p_0 as r_0: 10; the last writes no r: 10). The march and the
// split of the (y-tile, z) units over one wave of CTAs are those of k_fgp; the rows of step k are
// widened by the halo that step k + 1 needs and recomputed by both neighbouring tiles:
//   z_k        rows y0-1 .. y0+TY+1   from r_k rows y0-2 .. y0+TY+1 and b
//   r_{k+1}    rows y0-1 .. y0+TY     (dual step k; p_{k+1} only on the tile's own rows)
//   z_{k+1}    rows y0   .. y0+TY
//   p, r_{k+2} rows y0   .. y0+TY-1   (dual step k + 1, to HBM)
// In z the march runs three planes ahead of its output. Iteration q computes z_k of plane q+2,
// dual step k of plane q+1, z_{k+1} of plane q+1 and dual step k+1 of plane q. The inputs arrive as
// TMA box loads: r_k and b of plane q+3 into the ring slot of plane q at the iteration's first
// barrier (a whole plane ahead of their use), p_k of plane q+2 at its second barrier (used by the
// next iteration's dual step k). Shared memory, in rows of the pitch (nx rounded up to 32 floats):
// r_k ring (3 planes x 3 components x TY+4 rows), b ring (3 x TY+3), z_k (2 x TY+3), the parts of
// r_{k+1} that other threads read (its y component, TY+2 rows; its z component of row y0+TY for
// two planes and its x component of that row; each thread's last own x value), z_{k+1}
// (2 x TY+1), p_k (3 x TY+2): 20 TY + 64 rows and ceil(threads / pitch) rows. The own rows of
// every phase belong to one thread row each (four x values per thread), and the halo rows of z_k
// and of dual step k are spread over all threads with the same point -> thread map in both phases,
// so the step-k dual reads only z_k values that its own thread wrote in this iteration or that a
// barrier separates from their writer: two barriers per plane. p_{k+1} and r_{k+1} of the thread's
// own points stay in registers from dual step k to the z_{k+1} phase and dual step k + 1. The per-point operations are those of k_fgp in
// the same order, so the iterates are bit-identical.
struct Fgp2Args {
  const float* pin[3];  // p_k (not read on the first step)
  float* pout[3];       // p_{k+2}
  float* rout[3];       // r_{k+2} (not written when step k + 1 is the last)
  int nz, ny, nx;
  int pitch;  // shared-memory row length: nx rounded up to 32 floats (the box width)
  int ytiles;
  float lambda, step;
  float m1, m2;     // momenta of steps k and k + 1
  float neg_zero;  // -0.0f, the addend of the packed products (a value the compiler cannot see)
  unsigned long long* timeouts;  // bounded waits that ran out are counted here (null: g_fgp2_timeouts)
};
// Box-load maps of r_k (on the first step p_0), boxes of (pitch x TY+4 rows), and of b (pitch x TY+3).
struct Fgp2Maps {
  CUtensorMap r[3];
  CUtensorMap b;
  CUtensorMap p[3];  // p_k, boxes of (pitch x TY+2 rows); not read on the first step
};

// Waits of k_fgp2 that ran out (a box load that never completed) in calls that pass no counter of
// their own; read by tv_wait_timeouts().
__device__ unsigned long long g_fgp2_timeouts = 0;

// The same two operations on a pair of neighbouring x points with Blackwell's packed FP32 add and
// multiply (two correctly rounded operations per instruction, each as the scalar __fadd_rn /
// __fmul_rn). A term a guard drops is added as -0.0 or subtracted as +0.0 instead, which leaves
// every value (signed zeros included) unchanged, so the pair results equal the scalar ones bit for
// bit. z and y guards are the same for both points; x guards come as the points' own flags.
//
// Products must round on their own: ptxas contracts a packed multiply followed by a packed add into
// one FMA even when both carry explicit rounding modes, and also when the product is written as an
// FMA with a literal -0.0 addend (it folds that back into a multiply); measured on this toolkit, it
// changes results in the last bit. So a product is an FMA whose -0.0 addend (`nz`) comes from a
// kernel argument: RN(a b + -0) = RN(a b) for every a b, signed zeros included, and an FMA result
// is never fused into a later add.
__device__ __forceinline__ unsigned long long pack2(float2 a) {
  unsigned long long v;
  asm("mov.b64 %0, {%1, %2};" : "=l"(v) : "f"(a.x), "f"(a.y));
  return v;
}
__device__ __forceinline__ float2 unpack2(unsigned long long v) {
  float2 a;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(a.x), "=f"(a.y) : "l"(v));
  return a;
}
__device__ __forceinline__ float2 add2(float2 a, float2 b) {
  unsigned long long d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(pack2(a)), "l"(pack2(b)));
  return unpack2(d);
}
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return add2(a, make_float2(-b.x, -b.y)); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b, float2 nz) {
  unsigned long long d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(pack2(a)), "l"(pack2(b)), "l"(pack2(nz)));
  return unpack2(d);
}

// Primal points of x and x+1: vxm is the x component of the dual at x-1 and x (dropped where the
// point is x = 0); last_x1 marks x+1 = nx-1 (its +x term dropped).
__device__ __forceinline__ float2 fgp_primal_pair(bool zhi, bool zlo, bool yhi, bool ylo, bool first_x0,
                                                  bool last_x1, float2 vz, float2 vzb, float2 vy, float2 vym,
                                                  float2 vx, float2 vxm, float2 vb, float lambda, float2 nz) {
  float2 sacc = make_float2(0.0f, 0.0f);
  if (zhi) sacc = add2(sacc, vz);   // z < nz - 1
  if (zlo) sacc = sub2(sacc, vzb);  // z > 0
  if (yhi) sacc = add2(sacc, vy);   // y < ny - 1
  if (ylo) sacc = sub2(sacc, vym);  // y > 0
  if (last_x1) vx.y = -0.0f;        // x + 1 == nx - 1
  sacc = add2(sacc, vx);
  if (first_x0) vxm.x = 0.0f;  // x == 0
  sacc = sub2(sacc, vxm);
  const float2 t = sub2(vb, mul2(make_float2(lambda, lambda), sacc, nz));
  return make_float2(t.x > 0.0f ? t.x : 0.0f, t.y > 0.0f ? t.y : 0.0f);
}

// Dual steps at x and x+1 (tv_dual_step on each point, the same operations).
__device__ __forceinline__ void fgp_dual_pair(float2 c, float2 cz, float2 cy, float2 cx, bool zhi, bool yhi,
                                              bool last_x1, float step, float momentum, float2 p[3], float2 r[3],
                                              float2 nz) {
  float2 g[3];
  g[0] = zhi ? sub2(c, cz) : make_float2(0.0f, 0.0f);
  g[1] = yhi ? sub2(c, cy) : make_float2(0.0f, 0.0f);
  g[2] = sub2(c, cx);
  if (last_x1) g[2].y = 0.0f;
  const float2 st = make_float2(step, step);
  float2 q[3];
  float2 norm2 = make_float2(0.0f, 0.0f);
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    q[a] = add2(r[a], mul2(st, g[a], nz));
    norm2 = add2(norm2, mul2(q[a], q[a], nz));
  }
  // 1 / sqrt(norm2) per point where norm2 > 1, else 1, as tv_dual_step: computed for every point, without
  // a branch, as rcp_sqrt_rn(max(norm2, 1)) -- exactly 1 at 1 (the self-check covers [1, 2^126)), and
  // max(NaN, 1) = 1 as the host's comparison gives.
  const float2 scale = rcp_sqrt_rn2(make_float2(fmaxf(norm2.x, 1.0f), fmaxf(norm2.y, 1.0f)), nz);
  const float2 m = make_float2(momentum, momentum);
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const float2 next = mul2(q[a], scale, nz);
    r[a] = add2(next, mul2(m, sub2(next, p[a]), nz));
    p[a] = next;
  }
}

// Rows of the two-step kernel's shared memory, apart from the rows that hold each thread's last own
// x value (ceil(threads / pitch)).
constexpr std::size_t fgp2_rows(int ty) { return 20 * static_cast<std::size_t>(ty) + 64; }
// Threads per CTA the two-step kernel is compiled for (nx / 4 x TY must stay within it).
constexpr int fgp2_threads(int ty) { return ty == 8 ? 512 : 256; }

// CUBE > 0: compiled for a CUBE^3 volume (the sizes, the pitch and the block shape are constants, so
// shared-memory and global addresses fold into immediate offsets); 0: any size, from the arguments.
template <int TY, bool FIRST, bool LAST, int CUBE = 0>
__global__ void __launch_bounds__(fgp2_threads(TY), 1) k_fgp2(Fgp2Args A, const __grid_constant__ Fgp2Maps M) {
  extern __shared__ __align__(128) float smem2[];
  constexpr int VEC = 4;
  constexpr int RK_ROWS = TY + 4, B_ROWS = TY + 3, R1_ROWS = TY + 2, Z1_ROWS = TY + 1;
  constexpr int HALO = (8 + TY - 1) / TY;  // halo pair slots per thread: 2 nx over nx / 4 * TY threads
  constexpr bool kFullWarps = CUBE > 0 && (CUBE / VEC * TY) % 32 == 0;
  const int nx = CUBE > 0 ? CUBE : A.nx, ny = CUBE > 0 ? CUBE : A.ny, nz = CUBE > 0 ? CUBE : A.nz;
  const int bx = CUBE > 0 ? CUBE / VEC : static_cast<int>(blockDim.x);
  const int tx = static_cast<int>(threadIdx.x);
  const int ty = static_cast<int>(threadIdx.y);
  const int x0 = tx * VEC;
  const int nthreads = bx * TY;
  const int linear = ty * bx + tx;
  const int lane = linear & 31;
  const int warp_threads = kFullWarps ? 32 : min(32, nthreads - (linear & ~31));
  const unsigned lanes = warp_threads >= 32 ? 0xffffffffu : ((1u << warp_threads) - 1u);
  const std::size_t nxy = static_cast<std::size_t>(nx) * ny;
  // Shared memory in floats, rows of P floats (A.pitch: nx rounded up to 128 bytes; the columns
  // from nx on hold the zeros the box loads fill in): slot strides and buffer bases (32-bit offsets
  // from smem2), then the mbarriers. r_{k+1} keeps in shared memory only what other threads read:
  // its y component (rows y0-1 .. y0+TY), its z component of row y0+TY for two planes, its x
  // component of row y0+TY, and each thread's last own x value (the left neighbour of the next
  // thread's first point); the rest the z_{k+1} phase takes from the registers of its own thread.
  const int P = CUBE > 0 ? (CUBE + 31) / 32 * 32 : A.pitch;
  const int RKP = RK_ROWS * P, BP = B_ROWS * P, R1P = R1_ROWS * P, Z1P = Z1_ROWS * P;
  const int EDGE_ROWS = (nthreads + P - 1) / P;
  const int OB = 9 * RKP, OZ = OB + 3 * BP, ORY = OZ + 2 * BP, ORZH = ORY + R1P, ORXH = ORZH + 2 * P,
            OEDGE = ORXH + P, OZ1 = OEDGE + EDGE_ROWS * P, OPK = OZ1 + 2 * Z1P;
  // mbarriers: 0-2 for the plane loads (r_k and b) into ring slots 0-2, 3 for p_k.
  std::uint64_t* const bars = reinterpret_cast<std::uint64_t*>(smem2 + OPK + 3 * R1P);
  // Own-row offsets within a slot: r_k row ty+2 (rows start at y0-2); b, z_k, r_{k+1} row ty+1
  // (rows start at y0-1); z_{k+1} row ty (rows start at y0).
  const int own_rk = (ty + 2) * P + x0;
  const int own_b = (ty + 1) * P + x0;
  const int own_z1 = ty * P + x0;
  // The thread's four own points run as two pairs of packed operations; x guards per point.
  const bool x_first = x0 == 0;       // point 0 is x = 0
  const bool x_last = x0 + VEC == nx;  // point 3 is x = nx - 1
  const auto f2 = [](float a, float b) { return make_float2(a, b); };
  const float2 nzero = make_float2(A.neg_zero, A.neg_zero);
  // Primal points of the own row of plane z (y given); left = x component of the dual at x0-1.
  const auto primal4 = [&](int z, int yy, const float* vz, const float* vzb, const float* vy, const float* vym,
                           const float* vx, float left, const float* vb, float* out) {
    const bool zhi = z < nz - 1, zlo = z > 0, yhi = yy < ny - 1, ylo = yy > 0;
    const auto pairs = [&](bool zh, bool zl, bool yh, bool yl) {
      const float2 o0 = fgp_primal_pair(zh, zl, yh, yl, x_first, false, f2(vz[0], vz[1]), f2(vzb[0], vzb[1]),
                                        f2(vy[0], vy[1]), f2(vym[0], vym[1]), f2(vx[0], vx[1]), f2(left, vx[0]),
                                        f2(vb[0], vb[1]), A.lambda, nzero);
      const float2 o1 = fgp_primal_pair(zh, zl, yh, yl, false, x_last, f2(vz[2], vz[3]), f2(vzb[2], vzb[3]),
                                        f2(vy[2], vy[3]), f2(vym[2], vym[3]), f2(vx[2], vx[3]), f2(vx[1], vx[2]),
                                        f2(vb[2], vb[3]), A.lambda, nzero);
      out[0] = o0.x, out[1] = o0.y, out[2] = o1.x, out[3] = o1.y;
    };
    // Interior rows (warp-uniform: a warp holds part of one row of one plane) with the guards as
    // constants, so that the pair code has no branches; the boundary rows with the guards.
    if (zhi && zlo && yhi && ylo) {
      pairs(true, true, true, true);
    } else {
      pairs(zhi, zlo, yhi, ylo);
    }
  };
  // Dual steps of the own points (row yy) of plane z from primal values c, +z (cz), +y (cy) and the
  // primal value right of the last point; p and r updated in place.
  const auto dual4 = [&](int z, int yy, const float* c, const float* cz, const float* cy, float right,
                         float momentum, float (*pv)[VEC], float (*rv)[VEC]) {
    const bool zhi = z < nz - 1, yhi = yy < ny - 1;
    const auto pairs = [&](bool zh, bool yh) {
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int k0 = 2 * h;
        float2 pp[3], rr[3];
#pragma unroll
        for (int cc = 0; cc < 3; ++cc) {
          pp[cc] = f2(pv[cc][k0], pv[cc][k0 + 1]);
          rr[cc] = f2(rv[cc][k0], rv[cc][k0 + 1]);
        }
        fgp_dual_pair(f2(c[k0], c[k0 + 1]), f2(cz[k0], cz[k0 + 1]), f2(cy[k0], cy[k0 + 1]),
                      f2(c[k0 + 1], h == 0 ? c[2] : right), zh, yh, h == 1 && x_last, A.step, momentum, pp, rr,
                      nzero);
#pragma unroll
        for (int cc = 0; cc < 3; ++cc) {
          pv[cc][k0] = pp[cc].x, pv[cc][k0 + 1] = pp[cc].y;
          rv[cc][k0] = rr[cc].x, rv[cc][k0 + 1] = rr[cc].y;
        }
      }
    };
    if (zhi && yhi) {  // interior rows: guards as constants, as in primal4
      pairs(true, true);
    } else {
      pairs(zhi, yhi);
    }
  };
  // The layout, mbarriers included, must fit the shared memory the launch was given (CTA-uniform).
  if (!QHK_CHECK(static_cast<std::size_t>(OPK + 3 * R1P) * sizeof(float) + 4 * sizeof(std::uint64_t) <=
                 debug::dynamic_smem_bytes())) {
    return;
  }
  if (linear == 0) {
    for (int i = 0; i < 4; ++i) tma::mbar_init(bars + i, 1);
  }
  __syncthreads();
  unsigned long long* const timeouts = A.timeouts != nullptr ? A.timeouts : &g_fgp2_timeouts;
  unsigned phases = 0;  // bit i: parity of the next completion of mbarrier i
  // Thread 0 (the only issuer): bit i of `armed` is set while mbarrier i has a load in flight whose
  // completion no wait has seen yet; bit i of `armed_par` is that completion's parity. An early exit
  // waits for those loads (bounded) before the CTA's shared memory can be handed to another CTA.
  unsigned armed = 0, armed_par = 0;
  const auto arm = [&](int i) {
    armed |= 1u << i;
    armed_par = (armed_par & ~(1u << i)) | (phases & (1u << i));
  };
  const auto drain = [&]() {
    if (linear != 0) return;
    for (int i = 0; i < 4; ++i) {
      if ((armed >> i) & 1u) tma::mbar_wait(bars + i, (armed_par >> i) & 1u, timeouts);
    }
  };
  // Halo rows as pairs of points (x, x+1), x even: 2 nx pair slots, slot u = linear + j nthreads.
  // Slots below 3 nx / 2 are the z_k halo rows y0-1 (side 0), y0+TY (1), y0+TY+1 (2) -- z_k / b row
  // 0, TY+1, TY+2 -- of which those below nx are also the dual-k halo rows, so each such pair's z_k is
  // its own thread's write; the rest (side 3) are row y0+TY of z_{k+1}.
  const int half = nx / 2;
  int hz_side[HALO], hz_x[HALO];
#pragma unroll
  for (int j = 0; j < HALO; ++j) {
    const int u = linear + j * nthreads;
    hz_side[j] = u < 2 * nx ? u / half : -1;
    hz_x[j] = 2 * (u - max(hz_side[j], 0) * half);
  }
  const auto ld2 = [](const float* p) { return *reinterpret_cast<const float2*>(p); };
  const auto st2 = [](float* p, float2 v) { *reinterpret_cast<float2*>(p) = v; };

  const long long units = static_cast<long long>(CUBE > 0 ? (CUBE + TY - 1) / TY : A.ytiles) * nz;
  const long long u_end = units * (blockIdx.x + 1) / gridDim.x;
  for (long long u = units * blockIdx.x / gridDim.x; u < u_end;) {
    const int y0 = static_cast<int>(u / nz) * TY;
    const int z0 = static_cast<int>(u % nz);
    if (!QHK_CHECK(y0 < ny && u < units)) break;  // CTA-uniform
    const int zend = static_cast<int>(min(static_cast<long long>(nz), z0 + (u_end - u)));
    u += zend - z0;
    const int zmax = min(zend + 1, nz - 1);  // last plane of r_k and b read
    const int y = y0 + ty;
    const bool own = y < ny;
    const std::size_t own_g = static_cast<std::size_t>(y) * nx + x0;  // within a plane

    // Box loads by thread 0, counted on an mbarrier. A plane z into ring slot s (z mod 3): r_k rows
    // y0-2 .. y0+TY+1 (`comps` components) and b rows y0-1 .. y0+TY+1, on mbarrier s; p_k of plane
    // z, rows y0-1 .. y0+TY, into the p_k slot on mbarrier 3. Rows outside the volume arrive as
    // zeros and are never read.
    const auto issue = [&](int z, int s, int comps, bool with_b) {
      if (!QHK_CHECK(z >= 0 && z < nz && s >= 0 && s < 3)) return;
      tma::fence_async_shared();
      std::uint64_t* bar = bars + s;
      arm(s);
      tma::mbar_expect(bar, static_cast<unsigned>((comps * RK_ROWS + (with_b ? B_ROWS : 0)) * P * 4));
      for (int c = 0; c < comps; ++c) tma::load_3d(smem2 + (s * 3 + c) * RKP, &M.r[c], 0, y0 - 2, z, bar);
      if (with_b) tma::load_3d(smem2 + OB + s * BP, &M.b, 0, y0 - 1, z, bar);
    };
    const auto issue_pk = [&](int z) {
      if (!QHK_CHECK(z >= 0 && z < nz)) return;
      tma::fence_async_shared();
      arm(3);
      tma::mbar_expect(bars + 3, static_cast<unsigned>(3 * R1_ROWS * P * 4));
      for (int c = 0; c < 3; ++c) tma::load_3d(smem2 + OPK + c * R1P, &M.p[c], 0, y0 - 1, z, bars + 3);
    };
    // Bounded wait on mbarrier i (every thread), then its phase bit flips.
    const auto wait_bar = [&](int i) {
      const bool done = tma::mbar_wait(bars + i, (phases >> i) & 1u, timeouts);
      if (done) armed &= ~(1u << i);
      phases ^= 1u << i;
      return done;
    };
    const auto mod3 = [](int z) { return ((z % 3) + 3) % 3; };
    // Iteration q needs r_k and b of planes up to q+2 (the z component of q+1 for z_k of q+2).
    if (linear == 0) {
      if (z0 >= 2) issue(z0 - 2, mod3(z0 - 2), 1, false);
      if (z0 >= 1) issue(z0 - 1, mod3(z0 - 1), 3, true);
    }
    bool ok = true;
    if (z0 >= 2) ok = wait_bar(mod3(z0 - 2)) && ok;

    float cr[3][VEC] = {}, cp[3][VEC] = {};  // r_{k+1}, p_{k+1} of this thread's points of plane q
    float nr[3][VEC] = {}, np[3][VEC] = {};  // the same of plane q+1
    int m0 = mod3(z0 - 3);                   // ring slot of plane q (and of q+3)
    for (int q = z0 - 3; q < zend; ++q, m0 = m0 == 2 ? 0 : m0 + 1) {
      const int a2 = q + 2, a1 = q + 1;
      const int m1 = m0 == 2 ? 0 : m0 + 1;  // ring slot of q+1
      const int m2 = m0 == 0 ? 2 : m0 - 1;  // ring slot of q+2
      const int par = q & 1;                // parity of q and q+2 (z_k, z_{k+1}, r_{k+1} row); q+1 has par ^ 1
      const bool do_a = a2 >= 0 && a2 < nz;                  // z_k of plane a2
      const bool do_b = a1 >= 0 && a1 >= z0 - 1 && a1 < nz;  // dual step k on plane a1
      const bool do_c = a1 >= z0 && a1 < nz;                 // z_{k+1} of plane a1
      const bool do_d = q >= z0;                             // dual step k+1 on plane q
      const bool wait_plane = a2 >= 0 && a2 <= zmax;  // plane a2, loaded one iteration ago
      if (wait_plane) ok = wait_bar(m2) && ok;
      if (__syncthreads_or(!ok)) {
        // A load never completed: leave with the timeout counted (every thread takes this exit),
        // after a bounded wait for each load still in flight (the plane of slot m2, p_k of a1).
        drain();
        return;
      }
      // Slot m0 held plane q, last read one iteration ago: plane q+3 streams in for a whole plane.
      if (linear == 0 && q + 3 <= zmax) issue(q + 3, m0, 3, true);

      // z_k of plane a2 that this thread computes and the dual step k below reads again: own row, halo pairs.
      float zk_own[VEC] = {};
      float2 hz_own[HALO];
#pragma unroll
      for (int j = 0; j < HALO; ++j) hz_own[j] = f2(0.0f, 0.0f);
      if (do_a) {
        const int a = a2;
        const float* Rz = smem2 + (m2 * 3 + 0) * RKP;
        const float* Rzb = smem2 + (m1 * 3 + 0) * RKP;  // plane a-1; not read on plane 0
        const float* Ry = smem2 + (m2 * 3 + 1) * RKP;
        const float* Rx = smem2 + (m2 * 3 + 2) * RKP;
        const float* B = smem2 + OB + m2 * BP;
        float* Z = smem2 + OZ + par * BP;
        {
          float vz[VEC], vzb[VEC], vy[VEC], vym[VEC], vx[VEC], vb[VEC];
          Vec<VEC>::load(Rz + own_rk, vz);
          Vec<VEC>::load(Rzb + own_rk, vzb);
          Vec<VEC>::load(Ry + own_rk, vy);
          Vec<VEC>::load(Ry + own_rk - P, vym);
          Vec<VEC>::load(Rx + own_rk, vx);
          Vec<VEC>::load(B + own_b, vb);
          const float from_lane = __shfl_up_sync(lanes, vx[3], 1);
          const float left = (x0 > 0 && lane == 0) ? Rx[own_rk - 1] : from_lane;
          if (own) primal4(a, y, vz, vzb, vy, vym, vx, left, vb, zk_own);
          Vec<VEC>::store(Z + own_b, zk_own);
        }
#pragma unroll
        for (int j = 0; j < HALO; ++j) {
          const int side = hz_side[j];
          const int x = hz_x[j];
          const int zi = side == 0 ? 0 : TY + side;
          const int yy = y0 - 1 + zi;
          if (side >= 0 && side <= 2 && yy >= 0 && yy < ny) {
            const int i = (zi + 1) * P + x;  // r_k row of yy
            const float2 vx = ld2(Rx + i);
            const float2 o = fgp_primal_pair(a < nz - 1, a > 0, yy < ny - 1, yy > 0, x == 0, x + 1 == nx - 1,
                                             ld2(Rz + i), ld2(Rzb + i), ld2(Ry + i), ld2(Ry + i - P), vx,
                                             f2(x > 0 ? Rx[i - 1] : 0.0f, vx.x), ld2(B + zi * P + x), A.lambda, nzero);
            st2(Z + zi * P + x, o);
            hz_own[j] = o;
          }
        }
      }

      // p_k of plane a1, loaded during the previous iteration.
      const bool wait_pk = !FIRST && do_b;
      if (wait_pk) ok = wait_bar(3) && ok;
      const float* PK = smem2 + OPK;
      if (do_b) {
        const int a = a1;
        const float* Zc = smem2 + OZ + (par ^ 1) * BP;
        const float* R = smem2 + (m1 * 3) * RKP;
        float* Ry1 = smem2 + ORY;
        float* RzH = smem2 + ORZH + (par ^ 1) * P;  // z component of row y0+TY, plane a1
        float* RxH = smem2 + ORXH;                  // x component of row y0+TY
        {
          float zc[VEC], zy[VEC], zz[VEC];
          Vec<VEC>::load(Zc + own_b, zc);
          Vec<VEC>::load(Zc + own_b + P, zy);
#pragma unroll
          for (int k = 0; k < VEC; ++k) zz[k] = zk_own[k];
          const float from_lane = __shfl_down_sync(lanes, zc[0], 1);
          const float right =
              (x0 + VEC < nx && (lane == 31 || lane == warp_threads - 1)) ? Zc[own_b + VEC] : from_lane;
          float rv[3][VEC], pk[3][VEC];
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            Vec<VEC>::load(R + c * RKP + own_rk, rv[c]);
            if (!FIRST) Vec<VEC>::load(PK + c * R1P + own_b, pk[c]);
          }
          if (own) {
#pragma unroll
            for (int c = 0; c < 3; ++c)
#pragma unroll
              for (int k = 0; k < VEC; ++k) {
                nr[c][k] = rv[c][k];
                np[c][k] = FIRST ? rv[c][k] : pk[c][k];
              }
            dual4(a, y, zc, zz, zy, right, A.m1, np, nr);
            Vec<VEC>::store(Ry1 + own_b, nr[1]);
          }
          smem2[OEDGE + linear] = nr[2][3];  // the left neighbour of the next thread's first point
        }
        // halo rows y0-1 and y0+TY: the points this thread took in the z_k phase, so their z_k of
        // plane a+1 is this thread's own write.
#pragma unroll
        for (int h = 0; h < HALO; ++h) {
          const int side = hz_side[h];
          const int x = hz_x[h];
          const int zi = side == 0 ? 0 : TY + 1;
          const int yy = y0 - 1 + zi;
          if ((side == 0 || side == 1) && yy >= 0 && yy < ny) {
            const int i = zi * P + x;
            const float2 c0 = ld2(Zc + i);
            const float2 cz = a < nz - 1 ? hz_own[h] : f2(0.0f, 0.0f);  // this thread's write above
            const float2 cy = yy < ny - 1 ? ld2(Zc + i + P) : f2(0.0f, 0.0f);
            const float2 cx = f2(c0.y, x + 2 < nx ? Zc[i + 2] : 0.0f);
            float2 p[3], r[3];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
              r[c] = ld2(R + c * RKP + i + P);
              p[c] = FIRST ? r[c] : ld2(PK + c * R1P + i);
            }
            fgp_dual_pair(c0, cz, cy, cx, a < nz - 1, yy < ny - 1, x + 1 == nx - 1, A.step, A.m1, p, r, nzero);
            st2(Ry1 + i, r[1]);
            if (side == 1) {
              st2(RzH + x, r[0]);
              st2(RxH + x, r[2]);
            }
          }
        }
      }
      if (__syncthreads_or(!ok)) {  // r_{k+1} of plane a1 complete
        drain();  // p_k of a1 if its wait ran out, and plane q+3 issued into slot m0 above
        return;
      }
      // Every thread is past dual step k of a1: the p_k slot is free for p_k of a2, exactly the
      // planes whose dual step k the next iteration runs (and waits for): do_b of q+1.
      if (linear == 0 && !FIRST && a2 >= 0 && a2 >= z0 - 1 && a2 < nz && a2 <= zend) issue_pk(a2);

      float zn[VEC] = {};  // z_{k+1} of this thread's points of plane a1
      if (do_c) {
        const int a = a1;
        const float* RzH = smem2 + ORZH + (par ^ 1) * P;  // row y0+TY, plane a
        const float* RzbH = smem2 + ORZH + par * P;       // row y0+TY, plane a-1; not read on plane 0
        const float* Ry = smem2 + ORY;
        const float* RxH = smem2 + ORXH;
        const float* B = smem2 + OB + m1 * BP;
        float* Z = smem2 + OZ1 + (par ^ 1) * Z1P;
        {
          // Own points: r_{k+1} of planes a (nr) and a-1 (cr, before the dual step k+1 below
          // updates it) from this thread's registers; the y component of the row below and the x
          // component left of the first point from shared memory.
          float vym[VEC], vb[VEC];
          Vec<VEC>::load(Ry + own_b - P, vym);
          Vec<VEC>::load(B + own_b, vb);
          const float from_lane = __shfl_up_sync(lanes, nr[2][3], 1);
          const float left = (x0 > 0 && lane == 0) ? smem2[OEDGE + linear - 1] : from_lane;
          if (own) primal4(a, y, nr[0], cr[0], nr[1], vym, nr[2], left, vb, zn);
          Vec<VEC>::store(Z + own_z1, zn);
        }
        if (y0 + TY < ny) {  // row y0+TY: the pair slots of side 3
          const int yy = y0 + TY;
#pragma unroll
          for (int j = 0; j < HALO; ++j) {
            const int x = hz_x[j];
            if (hz_side[j] == 3) {
              const int i = (TY + 1) * P + x;
              const float2 vx = ld2(RxH + x);
              const float2 o = fgp_primal_pair(a < nz - 1, a > 0, yy < ny - 1, yy > 0, x == 0, x + 1 == nx - 1,
                                               ld2(RzH + x), ld2(RzbH + x), ld2(Ry + i), ld2(Ry + i - P), vx,
                                               f2(x > 0 ? RxH[x - 1] : 0.0f, vx.x), ld2(B + i), A.lambda, nzero);
              st2(Z + TY * P + x, o);
            }
          }
        }
      }

      if (do_d) {  // own row: z_{k+1} of plane q row ty (row ty+1 below it), of plane q+1 in zn
        const float* Zc = smem2 + OZ1 + par * Z1P;
        float zc[VEC], zy[VEC];
        Vec<VEC>::load(Zc + own_z1, zc);
        Vec<VEC>::load(Zc + own_z1 + P, zy);
        const float from_lane = __shfl_down_sync(lanes, zc[0], 1);
        const float right = (x0 + VEC < nx && (lane == 31 || lane == warp_threads - 1)) ? Zc[own_z1 + VEC] : from_lane;
        if (own) {
          dual4(q, y, zc, zn, zy, right, A.m2, cp, cr);
          const std::size_t at = q * nxy + own_g;
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            Vec<VEC>::store(A.pout[c] + at, cp[c]);
            if (!LAST) Vec<VEC>::store(A.rout[c] + at, cr[c]);
          }
        }
      }
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int k = 0; k < VEC; ++k) {
          cr[c][k] = nr[c][k];
          cp[c][k] = np[c][k];
        }
    }
    __syncthreads();  // the next march's prologue reuses the rings
  }
}

// Rows per CTA for an (nz, ny, nx) volume (TY rows of full x extent) and the grid: every CTA
// resident at once (a partial second wave would double the time of the step), with an even share of
// the plane units each.
struct FgpShape {
  int ty;
  int grid;
  std::size_t smem;
  int variant = 0;  // 0: r stored (k_fgp), 1: r recomputed (k_fgp_p), 2: two steps per pass (k_fgp2)
};

// Shared memory of the two-step form (rows of the 128-byte-aligned pitch, then 3 mbarriers), and
// the largest a CTA may take on this part.
int fgp2_pitch(int nx) { return (nx + 31) / 32 * 32; }
std::size_t fgp2_smem(int nx, int ty) {
  const std::size_t pitch = fgp2_pitch(nx);
  const std::size_t edge_rows = ((nx / 4) * static_cast<std::size_t>(ty) + pitch - 1) / pitch;
  return (fgp2_rows(ty) + edge_rows) * pitch * sizeof(float) + 4 * sizeof(std::uint64_t);
}
constexpr std::size_t kSmemOptin = 227 * 1024;

// Box loads take at most 256 floats per row.
bool fgp2_fits(int nx, int ty) {
  return nx % 4 == 0 && nx <= 256 && (nx / 4) * ty <= fgp2_threads(ty) && fgp2_smem(nx, ty) <= kSmemOptin;
}

// Shared memory of the r-recomputing step: 3 ring slots + 1 staging plane of 3 components x TY + 2
// rows, 2 primal and 2 b planes of TY + 1 rows (no staging on the first step).
std::size_t fgp_p_smem(int nx, int ty, bool first) {
  return ((first ? 3 : 4) * static_cast<std::size_t>(3) * (ty + 2) + 4 * static_cast<std::size_t>(ty + 1)) * nx *
         sizeof(float);
}

// Autotuner choices: variant * 16 + rows per CTA.
constexpr int kFgpVariantScale = 16;

std::size_t fgp_smem(int nx, int ty) {
  return (3 * static_cast<std::size_t>(3) * (ty + 2) + 4 * static_cast<std::size_t>(ty + 1)) * nx * sizeof(float);
}

// Rows per CTA that a CTA of this volume can take: tx * ty <= 256 threads and the shared memory
// within the SM's limit (the two-step form: float4 rows, 512 threads and the opt-in limit, and only
// where the caller has the fourth dual triplet); the default is the tallest of at most 4 rows of
// the one-step form within 110 KiB.
template <int VEC>
std::vector<int> fgp_rows_candidates(int nx, bool two_step) {
  std::vector<int> out;
  const int tx = nx / VEC;
  if (VEC == 4 && two_step) {
    for (const int ty : {8, 4, 2})
      if (fgp2_fits(nx, ty)) out.push_back(2 * kFgpVariantScale + ty);
  }
  for (const int variant : {1, 0}) {
    for (const int ty : {8, 4, 2, 1}) {
      const std::size_t smem = variant == 1 ? fgp_p_smem(nx, ty, false) : fgp_smem(nx, ty);
      if (tx * ty <= 256 && smem <= 200 * 1024) out.push_back(variant * kFgpVariantScale + ty);
    }
  }
  return out;
}

template <int VEC>
int fgp_rows_default(int nx) {
  const int tx = nx / VEC;
  int ty = 4;
  while (ty > 1 && (tx * ty > 256 || fgp_smem(nx, ty) > 110 * 1024)) --ty;
  require(tx * ty <= 256 && fgp_smem(nx, ty) <= 200 * 1024,
          "tv: volume rows too long for the FGP kernel (at most 1024 float4-aligned or 256 other x values)");
  return ty;
}

template <int VEC>
TuneKey fgp_key(int nz, int ny, int nx) {
  return tune_key(TuneFamily::fgp, {nz, ny, nx, VEC, 0, 0});
}

template <int VEC>
FgpShape fgp_shape_rows(int nz, int ny, int nx, int choice) {
  const int variant = choice / kFgpVariantScale;
  const int ty = choice % kFgpVariantScale;
  const std::size_t smem =
      variant == 2 ? fgp2_smem(nx, ty) : variant == 1 ? fgp_p_smem(nx, ty, false) : fgp_smem(nx, ty);
  int per_sm = 0;
  if (variant == 2) {
    const auto occupancy = [&](auto kernel) {
      ensure_smem(kernel);
      check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, (nx / 4) * ty, smem), "cudaOccupancy");
    };
    if (ty == 8) {
      occupancy(k_fgp2<8, false, false>);
    } else if (ty == 4) {
      occupancy(k_fgp2<4, false, false>);
    } else {
      occupancy(k_fgp2<2, false, false>);
    }
  } else if (variant == 1) {
    auto kernel = k_fgp_p<VEC, false>;
    ensure_smem(kernel);
    check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, (nx / VEC) * ty, smem), "cudaOccupancy");
  } else {
    auto kernel = k_fgp<VEC, false, false>;
    ensure_smem(kernel);
    check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, (nx / VEC) * ty, smem), "cudaOccupancy");
  }
  const long long slots = static_cast<long long>(sm_count()) * std::max(per_sm, 1);
  const long long units = static_cast<long long>((ny + ty - 1) / ty) * nz;
  FgpShape sh{ty, static_cast<int>(std::min(slots, units)), smem, variant};
  return sh;
}

// Forced FGP form (qhk_tv_form): 0 the tuned / default one, 1 stored r, 2 recomputed r, 3 two
// steps per pass, 16 + rows two steps per pass with that many rows per CTA (2, 4 or 8).
std::atomic<int> g_fgp_form{0};

// The tuned (or forced) shape; the two-step form only with VEC = 4 and a fourth dual triplet, else
// the stored-r form with its default rows.
template <int VEC>
FgpShape fgp_shape(int nz, int ny, int nx, bool two_step) {
  const int form = g_fgp_form.load();
  const int fallback = fgp_rows_default<VEC>(nx);
  int choice = tuned_choice(fgp_key<VEC>(nz, ny, nx), fallback);
  if (form == 3) {
    choice = fallback;
    for (const int ty : {8, 4, 2}) {
      if (fgp2_fits(nx, ty)) {
        choice = 2 * kFgpVariantScale + ty;
        break;
      }
    }
  } else if (form >= 16) {  // two steps per pass with form - 16 rows, where that fits
    choice = fgp2_fits(nx, form - 16) ? 2 * kFgpVariantScale + (form - 16) : fallback;
  } else if (form == 1 || form == 2) {
    const int ty = choice / kFgpVariantScale == 2 ? fallback : choice % kFgpVariantScale;
    choice = (form - 1) * kFgpVariantScale + ty;
    const std::size_t smem = form == 2 ? fgp_p_smem(nx, ty, false) : fgp_smem(nx, ty);
    if (smem > 200 * 1024) choice = (form - 1) * kFgpVariantScale + 1;
  }
  if (choice / kFgpVariantScale == 2 && (VEC != 4 || !two_step || !fgp2_fits(nx, choice % kFgpVariantScale))) {
    choice = fallback;
  }
  return fgp_shape_rows<VEC>(nz, ny, nx, choice);
}

template <int VEC, bool FIRST, bool LAST>
void launch_fgp(const FgpArgs& a, const FgpShape& sh, cudaStream_t s) {
  auto kernel = k_fgp<VEC, FIRST, LAST>;
  ensure_smem(kernel);
  const dim3 block(a.nx / VEC, sh.ty);
  kernel<<<sh.grid, block, sh.smem, s>>>(a);
  check_launch("fgp step");
}

// The first step of the r-recomputing form needs no staging plane: its smem is smaller.
template <int VEC, bool FIRST>
void launch_fgp_p(const FgpPArgs& a, const FgpShape& sh, cudaStream_t s) {
  auto kernel = k_fgp_p<VEC, FIRST>;
  ensure_smem(kernel);
  const dim3 block(a.nx / VEC, sh.ty);
  const std::size_t smem = fgp_p_smem(a.nx, sh.ty, FIRST);
  kernel<<<sh.grid, block, smem, s>>>(a);
  check_launch("fgp step");
}

template <int TY, bool FIRST, bool LAST, int CUBE>
void launch_fgp2_t(const Fgp2Args& a, const float* const rin[3], const float* b, int grid, cudaStream_t s) {
  auto kernel = k_fgp2<TY, FIRST, LAST, CUBE>;
  ensure_smem(kernel);
  Fgp2Maps maps;
  for (int c = 0; c < 3; ++c) maps.r[c] = volume_tensor_map(rin[c], a.nx, a.ny, a.nz, a.pitch, TY + 4);
  maps.b = volume_tensor_map(b, a.nx, a.ny, a.nz, a.pitch, TY + 3);
  for (int c = 0; c < 3; ++c) maps.p[c] = FIRST ? maps.r[c] : volume_tensor_map(a.pin[c], a.nx, a.ny, a.nz, a.pitch, TY + 2);
  kernel<<<grid, dim3(a.nx / 4, TY), fgp2_smem(a.nx, TY), s>>>(a, maps);
  check_launch("fgp two steps");
}

template <int TY, int CUBE = 0>
void launch_fgp2_rows(bool first, bool last, const Fgp2Args& a, const float* const rin[3], const float* b, int grid,
                      cudaStream_t s) {
  if (first && last) {
    launch_fgp2_t<TY, true, true, CUBE>(a, rin, b, grid, s);
  } else if (first) {
    launch_fgp2_t<TY, true, false, CUBE>(a, rin, b, grid, s);
  } else if (last) {
    launch_fgp2_t<TY, false, true, CUBE>(a, rin, b, grid, s);
  } else {
    launch_fgp2_t<TY, false, false, CUBE>(a, rin, b, grid, s);
  }
}

// rin: r_k (p_0 on the first step), b: the point the prox is taken at.
void launch_fgp2(bool first, bool last, Fgp2Args a, const float* const rin[3], const float* b, const FgpShape& sh,
                 cudaStream_t s) {
  require(fgp2_fits(a.nx, sh.ty), "tv: two-step FGP shape out of range");
  a.pitch = fgp2_pitch(a.nx);
  a.neg_zero = -0.0f;
  if (sh.ty == 8 && a.nx == 256 && a.ny == 256 && a.nz == 256) {  // the 256^3 volumes, sizes compiled in
    launch_fgp2_rows<8, 256>(first, last, a, rin, b, sh.grid, s);
  } else if (sh.ty == 8) {
    launch_fgp2_rows<8>(first, last, a, rin, b, sh.grid, s);
  } else if (sh.ty == 4) {
    launch_fgp2_rows<4>(first, last, a, rin, b, sh.grid, s);
  } else {
    require(sh.ty == 2, "tv: two-step FGP rows must be 2, 4 or 8");
    launch_fgp2_rows<2>(first, last, a, rin, b, sh.grid, s);
  }
}

template <int VEC>
void launch_fgp_any(bool first, bool last, const FgpArgs& a, const FgpShape& sh, cudaStream_t s) {
  if (first && last) {
    launch_fgp<VEC, true, true>(a, sh, s);
  } else if (first) {
    launch_fgp<VEC, true, false>(a, sh, s);
  } else if (last) {
    launch_fgp<VEC, false, true>(a, sh, s);
  } else {
    launch_fgp<VEC, false, false>(a, sh, s);
  }
}

template <int VEC>
void launch_final(TvFinal mode, const float* b, float* const p[3], int nz, int ny, int nx, float lambda,
                  float momentum, float* xprev, float* out, float nm2, float inv_k02, cudaStream_t s) {
  const std::size_t total = static_cast<std::size_t>(nz) * ny * nx / VEC;
  const unsigned grid = static_cast<unsigned>(std::min<std::size_t>((total + 255) / 256, 148u * 16u));
  switch (mode) {
    case TvFinal::plain:
      k_tv_final<VEC, 0><<<grid, 256, 0, s>>>(b, p[0], p[1], p[2], nz, ny, nx, lambda, momentum, xprev, out, nm2,
                                               inv_k02);
      break;
    case TvFinal::momentum:
      k_tv_final<VEC, 1><<<grid, 256, 0, s>>>(b, p[0], p[1], p[2], nz, ny, nx, lambda, momentum, xprev, out, nm2,
                                               inv_k02);
      break;
    case TvFinal::index:
      k_tv_final<VEC, 2><<<grid, 256, 0, s>>>(b, p[0], p[1], p[2], nz, ny, nx, lambda, momentum, xprev, out, nm2,
                                               inv_k02);
      break;
  }
  check_launch("tv final primal");
}

}  // namespace

float fista_t(float t) { return 0.5f * (1.0f + std::sqrt(1.0f + 4.0f * t * t)); }

unsigned long long tv_wait_timeouts() {
  unsigned long long n = 0;
  check(cudaMemcpyFromSymbol(&n, g_fgp2_timeouts, sizeof(n)), "read wait timeouts");
  return n;
}

std::string wait_timeout_message(const char* what) {
  return std::string(what) +
         ": a bounded device wait ran out (a TMA load of the two-step FGP kernel never completed); "
         "the result is not valid";
}

void set_tv_form(int form) {
  require((form >= 0 && form <= 3) || form == 18 || form == 20 || form == 24,
          "tv: form must be 0 (tuned), 1 (stored r), 2 (recomputed r), 3 (two steps per pass) or 16 + rows "
          "(two steps per pass with 2, 4 or 8 rows per CTA)");
  g_fgp_form.store(form);
}

void tv_prox(const float* b, TvBuffers& t, int nz, int ny, int nx, float lambda, int inner, TvFinal final_mode,
             float momentum, float* xprev, float* out, float nm2, float inv_k02, cudaStream_t s) {
  require(nz >= 1 && ny >= 1 && nx >= 1, "tv: empty volume");
  // float4 rows need nx % 4 == 0 and 16-byte aligned volumes.
  bool aligned = nx % 4 == 0 && reinterpret_cast<std::uintptr_t>(b) % 16 == 0 &&
                 reinterpret_cast<std::uintptr_t>(out) % 16 == 0 &&
                 (xprev == nullptr || reinterpret_cast<std::uintptr_t>(xprev) % 16 == 0);
  for (int i = 0; i < 3; ++i)
    for (int c = 0; c < 3; ++c) aligned = aligned && reinterpret_cast<std::uintptr_t>(t.v[i][c]) % 16 == 0;
  if (t.has_fourth()) {
    for (int c = 0; c < 3; ++c) aligned = aligned && reinterpret_cast<std::uintptr_t>(t.v[3][c]) % 16 == 0;
  }
  const int vec = aligned ? 4 : 1;
  const FgpShape sh = vec == 4 ? fgp_shape<4>(nz, ny, nx, t.has_fourth()) : fgp_shape<1>(nz, ny, nx, false);
  const float step = 1.0f / (12.0f * lambda);
  float tk = 1.0f;
  if (sh.variant != 2 && t.p_index == 3) {
    // The one-step forms rotate among the first three triplets: bring p there (only after the form
    // changed between two calls on the same buffers).
    const std::size_t vbytes = static_cast<std::size_t>(nz) * ny * nx * sizeof(float);
    for (int c = 0; c < 3; ++c)
      check(cudaMemcpyAsync(t.v[0][c], t.v[3][c], vbytes, cudaMemcpyDeviceToDevice, s), "copy dual");
    t.p_index = 0;
  }
  if (sh.variant == 2) {
    // Pairs of steps: (p, r) in two triplets -> (p, r) in two others; the first pair reads p_0 as
    // r_0. An odd last step runs the one-step kernel (stored-r form of the same shape family).
    int pc = t.p_index, rc = t.p_index;
    const auto free_pair = [&](int& f0, int& f1) {
      int n = 0;
      for (int i = 0; i < 4 && n < 2; ++i) {
        if (i == pc || i == rc) continue;
        (n++ == 0 ? f0 : f1) = i;
      }
    };
    int k = 0;
    for (; k + 2 <= inner; k += 2) {
      const float t1 = fista_t(tk);
      const float t2 = fista_t(t1);
      Fgp2Args a{};
      a.timeouts = t.wait_status;
      a.nz = nz, a.ny = ny, a.nx = nx;
      a.ytiles = (ny + sh.ty - 1) / sh.ty;
      a.lambda = lambda, a.step = step;
      a.m1 = (tk - 1.0f) / t1;
      a.m2 = (t1 - 1.0f) / t2;
      int f0 = 0, f1 = 0;
      free_pair(f0, f1);
      const float* rin[3];
      for (int c = 0; c < 3; ++c) {
        rin[c] = t.v[rc][c];
        a.pin[c] = t.v[pc][c];
        a.pout[c] = t.v[f0][c];
        a.rout[c] = t.v[f1][c];
      }
      launch_fgp2(k == 0, k + 2 == inner, a, rin, b, sh, s);
      pc = f0, rc = f1;
      tk = t2;
    }
    if (k < inner) {  // the last step alone
      const FgpShape one = fgp_shape_rows<4>(nz, ny, nx, fgp_rows_default<4>(nx));
      const float tn = fista_t(tk);
      FgpArgs a{};
      a.b = b;
      a.nz = nz, a.ny = ny, a.nx = nx;
      a.ytiles = (ny + one.ty - 1) / one.ty;
      a.lambda = lambda, a.step = step, a.momentum = (tk - 1.0f) / tn;
      int f0 = 0, f1 = 0;
      free_pair(f0, f1);
      const int po = k == 0 ? f0 : pc;  // the first step may not update p_0 = r_0 in place
      for (int c = 0; c < 3; ++c) {
        a.rin[c] = t.v[rc][c];
        a.pin[c] = t.v[pc][c];
        a.pout[c] = t.v[po][c];
        a.rout[c] = t.v[f1][c];
      }
      launch_fgp_any<4>(k == 0, true, a, one, s);
      pc = po;
      tk = tn;
    }
    t.p_index = pc;
  } else if (sh.variant == 1) {
    // p_k lives in triplet (i0 + k) % 3; step k reads p_k and p_{k-1}, writes p_{k+1} over p_{k-2}.
    const int i0 = t.p_index;
    float m_prev = 0.0f;
    for (int k = 0; k < inner; ++k) {
      FgpPArgs a{};
      a.b = b;
      a.nz = nz, a.ny = ny, a.nx = nx;
      a.ytiles = (ny + sh.ty - 1) / sh.ty;
      a.lambda = lambda, a.step = step, a.momentum = m_prev;
      for (int c = 0; c < 3; ++c) {
        a.pk[c] = t.v[(i0 + k) % 3][c];
        a.pkm1[c] = t.v[(i0 + k + 2) % 3][c];
        a.pout[c] = t.v[(i0 + k + 1) % 3][c];
      }
      if (vec == 4) {
        k == 0 ? launch_fgp_p<4, true>(a, sh, s) : launch_fgp_p<4, false>(a, sh, s);
      } else {
        k == 0 ? launch_fgp_p<1, true>(a, sh, s) : launch_fgp_p<1, false>(a, sh, s);
      }
      const float tn = fista_t(tk);
      m_prev = (tk - 1.0f) / tn;
      tk = tn;
    }
    if (inner > 0) t.p_index = (i0 + inner) % 3;
  } else {
    const int ip = t.p_index;
    const int ia = (ip + 1) % 3;
    int cur_r = ip;
    for (int k = 0; k < inner; ++k) {
      const float tn = fista_t(tk);
      const float m = (tk - 1.0f) / tn;
      FgpArgs a{};
      a.b = b;
      a.nz = nz, a.ny = ny, a.nx = nx;
      a.ytiles = (ny + sh.ty - 1) / sh.ty;
      a.lambda = lambda, a.step = step, a.momentum = m;
      const int rout = k == 0 ? (ip + 2) % 3 : 3 - ia - cur_r;
      for (int c = 0; c < 3; ++c) {
        a.rin[c] = t.v[cur_r][c];
        a.pin[c] = t.v[k == 0 ? ip : ia][c];
        a.pout[c] = t.v[ia][c];
        a.rout[c] = t.v[rout][c];
      }
      if (vec == 4) {
        launch_fgp_any<4>(k == 0, k == inner - 1, a, sh, s);
      } else {
        launch_fgp_any<1>(k == 0, k == inner - 1, a, sh, s);
      }
      cur_r = rout;
      tk = tn;
    }
    if (inner > 0) t.p_index = ia;
  }
  if (final_mode == TvFinal::none) return;
  float* const* p = t.v[t.p_index];
  if (vec == 4) {
    launch_final<4>(final_mode, b, p, nz, ny, nx, lambda, momentum, xprev, out, nm2, inv_k02, s);
  } else {
    launch_final<1>(final_mode, b, p, nz, ny, nx, lambda, momentum, xprev, out, nm2, inv_k02, s);
  }
}

namespace {

// Deterministic pseudo-random values in [lo, hi) (tuning inputs only).
__global__ void k_fill_hash(float* p, std::size_t n, float lo, float hi, unsigned seed) {
  for (std::size_t i = blockIdx.x * static_cast<std::size_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<std::size_t>(gridDim.x) * blockDim.x) {
    unsigned h = static_cast<unsigned>(i) * 0x9E3779B1u + seed;
    h ^= h >> 15;
    h *= 0x85EBCA77u;
    h ^= h >> 13;
    p[i] = lo + (hi - lo) * static_cast<float>(h >> 8) * (1.0f / 16777216.0f);
  }
}

template <int VEC>
void tune_fgp_rows(float* b, TvBuffers& t, int nz, int ny, int nx, float lambda, cudaStream_t s) {
  // Two middle steps of each form (one launch of the two-step form, two of the others): r (or p_k)
  // from triplet 0, p (or p_{k-1}) from triplet 1, outputs into triplets 1 and 2 (the two-step
  // form: 2 and 3), so that the inputs each run reads are never written.
  FgpArgs a{};
  a.b = b;
  a.nz = nz, a.ny = ny, a.nx = nx;
  a.lambda = lambda, a.step = 1.0f / (12.0f * lambda), a.momentum = 0.5f;
  FgpPArgs q{};
  q.b = b;
  q.nz = nz, q.ny = ny, q.nx = nx;
  q.lambda = a.lambda, q.step = a.step, q.momentum = 0.5f;
  for (int c = 0; c < 3; ++c) {
    a.rin[c] = t.v[0][c];
    a.pin[c] = t.v[1][c];
    a.pout[c] = t.v[1][c];
    a.rout[c] = t.v[2][c];
    q.pk[c] = t.v[0][c];
    q.pkm1[c] = t.v[1][c];
    q.pout[c] = t.v[2][c];
  }
  Fgp2Args w{};
  w.nz = nz, w.ny = ny, w.nx = nx;
  w.lambda = a.lambda, w.step = a.step, w.m1 = 0.5f, w.m2 = 0.5f;
  const float* w_rin[3] = {};
  if (t.has_fourth()) {
    for (int c = 0; c < 3; ++c) {
      w_rin[c] = t.v[0][c];
      w.pin[c] = t.v[1][c];
      w.pout[c] = t.v[2][c];
      w.rout[c] = t.v[3][c];
    }
  }
  autotune(fgp_key<VEC>(nz, ny, nx), fgp_rows_candidates<VEC>(nx, t.has_fourth()), fgp_rows_default<VEC>(nx),
           [&](int choice) {
             const FgpShape sh = fgp_shape_rows<VEC>(nz, ny, nx, choice);
             if (sh.variant == 2) {
               w.ytiles = (ny + sh.ty - 1) / sh.ty;
               launch_fgp2(false, false, w, w_rin, b, sh, s);
             } else if (sh.variant == 1) {
               q.ytiles = (ny + sh.ty - 1) / sh.ty;
               launch_fgp_p<VEC, false>(q, sh, s);
               launch_fgp_p<VEC, false>(q, sh, s);
             } else {
               a.ytiles = (ny + sh.ty - 1) / sh.ty;
               launch_fgp<VEC, false, false>(a, sh, s);
               launch_fgp<VEC, false, false>(a, sh, s);
             }
           },
           s);
}

}  // namespace

void tune_tv(float* b, TvBuffers& t, int nz, int ny, int nx, float lambda, cudaStream_t s) {
  require(nz >= 1 && ny >= 1 && nx >= 1, "tv: empty volume");
  if (!autotune_enabled()) return;
  const std::size_t vol = static_cast<std::size_t>(nz) * ny * nx;
  const unsigned grid = static_cast<unsigned>(std::min<std::size_t>((vol + 255) / 256, 148u * 16u));
  // Representative inputs: b in [0, 2), r in [-1, 1) (about half the dual points get projected),
  // p = 0. All of them are scratch of the caller.
  k_fill_hash<<<grid, 256, 0, s>>>(b, vol, 0.0f, 2.0f, 1u);
  check_launch("tv tune fill");
  for (int c = 0; c < 3; ++c) {
    k_fill_hash<<<grid, 256, 0, s>>>(t.v[0][c], vol, -1.0f, 1.0f, 2u + c);
    check_launch("tv tune fill");
    check(cudaMemsetAsync(t.v[1][c], 0, vol * sizeof(float), s), "cudaMemset");
  }
  bool aligned = nx % 4 == 0 && reinterpret_cast<std::uintptr_t>(b) % 16 == 0;
  for (int i = 0; i < (t.has_fourth() ? 4 : 3); ++i)
    for (int c = 0; c < 3; ++c) aligned = aligned && reinterpret_cast<std::uintptr_t>(t.v[i][c]) % 16 == 0;
  if (aligned) {
    tune_fgp_rows<4>(b, t, nz, ny, nx, lambda, s);
  } else {
    tune_fgp_rows<1>(b, t, nz, ny, nx, lambda, s);
  }
}

}  // namespace qhk
