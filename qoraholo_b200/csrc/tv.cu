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
// All arithmetic uses the round-to-nearest intrinsics in the reference's operation order, so the
// device iterates are bit-identical to the CPU's.
#include <algorithm>
#include <cmath>
#include <mutex>
#include <set>
#include <vector>

#include "autotune.hpp"
#include "qhk_internal.hpp"

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
            float s = 0.0f;
            if (z < nz - 1) s = __fadd_rn(s, vz[i]);
            if (z > 0) s = __fsub_rn(s, vzb[i]);
            if (y < ny - 1) s = __fadd_rn(s, vy[i]);
            if (y > 0) s = __fsub_rn(s, vym[i]);
            if (x < nx - 1) s = __fadd_rn(s, vx[i]);
            if (x > 0) s = __fsub_rn(s, i == 0 ? left : vx[i > 0 ? i - 1 : 0]);
            zv = tv_primal(vb[i], A.lambda, s);
          }
          out[i] = zv;
        }
        Vec<VEC>::store(Zd + static_cast<std::size_t>(rr) * nx + x0, out);
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
      const bool prefetch = z + 2 <= zlast;
      if (prefetch) {
        issue_r(z + 2, 3);
        issue_b(z + 2);
        copy_commit();
      }
      const std::size_t at = static_cast<std::size_t>(z) * nxy + static_cast<std::size_t>(y) * nx + x0;
      float pv[3][VEC];
      if (!FIRST && y < ny) {
#pragma unroll
        for (int c = 0; c < 3; ++c) Vec<VEC>::load(A.pin[c] + at, pv[c]);
      }
      if (prefetch) {
        copy_wait<1>();
      } else {
        copy_wait<0>();
      }
      __syncthreads();
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

// Rows per CTA for an (nz, ny, nx) volume (TY rows of full x extent) and the grid: every CTA
// resident at once (a partial second wave would double the time of the step), with an even share of
// the plane units each.
struct FgpShape {
  int ty;
  int grid;
  std::size_t smem;
};

std::size_t fgp_smem(int nx, int ty) {
  return (3 * static_cast<std::size_t>(3) * (ty + 2) + 4 * static_cast<std::size_t>(ty + 1)) * nx * sizeof(float);
}

// Rows per CTA that a CTA of this volume can take: tx * ty <= 256 threads and the shared memory
// within the SM's limit; the default is the tallest of at most 4 rows within 110 KiB.
template <int VEC>
std::vector<int> fgp_rows_candidates(int nx) {
  std::vector<int> out;
  const int tx = nx / VEC;
  for (const int ty : {8, 4, 2, 1}) {
    if (tx * ty <= 256 && fgp_smem(nx, ty) <= 200 * 1024) out.push_back(ty);
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
FgpShape fgp_shape_rows(int nz, int ny, int nx, int ty) {
  const std::size_t smem = fgp_smem(nx, ty);
  auto kernel = k_fgp<VEC, false, false>;
  ensure_smem(kernel);
  int per_sm = 0;
  check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, (nx / VEC) * ty, smem), "cudaOccupancy");
  const long long slots = static_cast<long long>(sm_count()) * std::max(per_sm, 1);
  const long long units = static_cast<long long>((ny + ty - 1) / ty) * nz;
  return {ty, static_cast<int>(std::min(slots, units)), smem};
}

template <int VEC>
FgpShape fgp_shape(int nz, int ny, int nx) {
  const int ty = tuned_choice(fgp_key<VEC>(nz, ny, nx), fgp_rows_default<VEC>(nx));
  return fgp_shape_rows<VEC>(nz, ny, nx, ty);
}

template <int VEC, bool FIRST, bool LAST>
void launch_fgp(const FgpArgs& a, const FgpShape& sh, cudaStream_t s) {
  auto kernel = k_fgp<VEC, FIRST, LAST>;
  ensure_smem(kernel);
  const dim3 block(a.nx / VEC, sh.ty);
  kernel<<<sh.grid, block, sh.smem, s>>>(a);
  check_launch("fgp step");
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

void tv_prox(const float* b, TvBuffers& t, int nz, int ny, int nx, float lambda, int inner, TvFinal final_mode,
             float momentum, float* xprev, float* out, float nm2, float inv_k02, cudaStream_t s) {
  require(nz >= 1 && ny >= 1 && nx >= 1, "tv: empty volume");
  // float4 rows need nx % 4 == 0 and 16-byte aligned volumes.
  bool aligned = nx % 4 == 0 && reinterpret_cast<std::uintptr_t>(b) % 16 == 0 &&
                 reinterpret_cast<std::uintptr_t>(out) % 16 == 0 &&
                 (xprev == nullptr || reinterpret_cast<std::uintptr_t>(xprev) % 16 == 0);
  for (int i = 0; i < 3; ++i)
    for (int c = 0; c < 3; ++c) aligned = aligned && reinterpret_cast<std::uintptr_t>(t.v[i][c]) % 16 == 0;
  const int vec = aligned ? 4 : 1;
  const FgpShape sh = vec == 4 ? fgp_shape<4>(nz, ny, nx) : fgp_shape<1>(nz, ny, nx);
  const float step = 1.0f / (12.0f * lambda);
  float tk = 1.0f;
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
  FgpArgs a{};
  a.b = b;
  a.nz = nz, a.ny = ny, a.nx = nx;
  a.lambda = lambda, a.step = 1.0f / (12.0f * lambda), a.momentum = 0.5f;
  for (int c = 0; c < 3; ++c) {
    a.rin[c] = t.v[0][c];
    a.pin[c] = t.v[1][c];
    a.pout[c] = t.v[1][c];
    a.rout[c] = t.v[2][c];
  }
  autotune(fgp_key<VEC>(nz, ny, nx), fgp_rows_candidates<VEC>(nx), fgp_rows_default<VEC>(nx),
           [&](int ty) {
             a.ytiles = (ny + ty - 1) / ty;
             launch_fgp<VEC, false, false>(a, fgp_shape_rows<VEC>(nz, ny, nx, ty), s);
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
  for (int i = 0; i < 3; ++i)
    for (int c = 0; c < 3; ++c) aligned = aligned && reinterpret_cast<std::uintptr_t>(t.v[i][c]) % 16 == 0;
  if (aligned) {
    tune_fgp_rows<4>(b, t, nz, ny, nx, lambda, s);
  } else {
    tune_fgp_rows<1>(b, t, nz, ny, nx, lambda, s);
  }
}

}  // namespace qhk
