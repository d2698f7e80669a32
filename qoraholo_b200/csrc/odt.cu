// Rytov fields -> refractive index on the device: 2D FFT of the fields, Ewald-sphere mapping into
// 3D k-space, and the missing-cone solver (Gerchberg-Papoulis on half or full spectra, FISTA-TV).
// Replaces the reference's OdtSolver (src/cuda/odt.cu:170-349; CPU form src/cpu/odt.cpp:124-242).
//
// Mapping. Each voxel of k-space receives the sum, in illumination order, of the spectrum values
// whose Ewald target it is, divided by their count. A thread owns K consecutive axial bins of one
// lateral column and walks all illuminations, recomputing the target bin with the reference's
// float operations (qhk_math.cuh: ewald_target), and accumulates the hits that fall in its bins
// in registers. Every voxel therefore has exactly one writer, sums in the CPU's order and needs
// no atomics; indices and hit counts are bit-identical to the CPU's, and so are the sums given the
// same spectra. For the real (R2C) solvers the same thread also walks the mirrored column -k and
// writes the half-spectrum data a = (P(k) + conj P(-k)) / 2 and hits = M(k) + M(-k) directly
// (src/common.hpp:72-87), so neither the full complex potential nor the weights are ever stored.
// The filled-voxel count is an integer reduction.
#include <algorithm>
#include <cmath>
#include <numbers>
#include <vector>

#include "autotune.hpp"
#include "debug.cuh"
#include "odt.hpp"
#include "nvtx.hpp"

namespace qhk {

namespace {

constexpr int kMapK = 8;  // axial bins per thread

__device__ __forceinline__ void accumulate(float (&re)[kMapK], float (&im)[kMapK], float (&w)[kMapK], int slot,
                                           float vr, float vi) {
#pragma unroll
  for (int i = 0; i < kMapK; ++i) {
    if (slot == i) {
      re[i] = __fadd_rn(re[i], vr);
      im[i] = __fadd_rn(im[i], vi);
      w[i] = __fadd_rn(w[i], 1.0f);
    }
  }
}

// Mapped value of spectrum s at axial bin kz: parity(kz) * (0, -gain nu_z) * s, as the host
// computes it: (0*sr - f*si, 0*si + f*sr) with f = -gain*nu_z, then the sign.
__device__ __forceinline__ void mapped(const Grid& g, float nuz, int kz, float2 s, float& vr, float& vi) {
  const float f = __fmul_rn(-g.gain, nuz);
  const float p = parity(kz);
  vr = __fmul_rn(p, -__fmul_rn(f, s.y));
  vi = __fmul_rn(p, __fmul_rn(f, s.x));
}

__device__ __forceinline__ unsigned long long warp_sum(unsigned long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// Half-spectrum mapping, one warp per lateral column (ky, kx) of the half spectrum (kx <= n/2), kMapCols
// columns per block, consecutive in the flattened (ky, kx) order, so that the block's output rows are
// contiguous. Each warp accumulates its column in shared memory: the sums and hit counts of side P (the
// column itself) and side N (its mirror (-ky, -kx), whose bin kz lands on -kz here). Lane l computes the
// targets of illuminations l, l + 32, ... once each and adds its own value; lanes of one round that hit
// the same bin (found with __match_any_sync) add one after another in lane order, i.e. in illumination
// order, so every bin's sum has the CPU's order and no atomics are used. Then the lanes turn the
// column into half data a = (P + conj N) / 2 and hits, and the block writes its columns out coalesced.
// Row pitch (float2 elements) of a column of the mapping's output tile: at least nz, congruent to 4
// modulo 16, so that 8 consecutive columns at 4 consecutive bins fill the 16 two-bank slots twice.
__host__ __device__ constexpr int map_pitch(int nz) { return (nz + 15) / 16 * 16 + 4; }

// Adds `value` to acc[bin] and one to cnt[bin] for every lane with `bin` >= 0, lanes with equal bins in
// increasing lane order.
__device__ __forceinline__ void ordered_add(float2* acc, std::uint16_t* cnt, int bin, float2 value, int lane) {
  unsigned pend = __ballot_sync(0xffffffffu, bin >= 0);
  const unsigned same = __match_any_sync(0xffffffffu, bin);
  while (pend) {
    const unsigned mine = same & pend;
    const bool leader = ((pend >> lane) & 1u) && (__ffs(mine) - 1 == lane);
    if (leader) {
      const float2 a = acc[bin];
      acc[bin] = make_float2(__fadd_rn(a.x, value.x), __fadd_rn(a.y, value.y));
      cnt[bin] = static_cast<std::uint16_t>(cnt[bin] + 1);
    }
    __syncwarp();
    pend &= ~__ballot_sync(0xffffffffu, leader);
  }
}

template <int kMapCols>  // columns (warps) per block
__global__ void __launch_bounds__(32 * kMapCols)
    k_map_half(const float2* __restrict__ spectra, const float4* __restrict__ illum, int count, Grid g,
               float2* __restrict__ a, std::uint8_t* __restrict__ hits, unsigned long long* __restrict__ filled) {
  extern __shared__ __align__(16) unsigned char map_smem[];
  const int n = g.n, nz = g.nz, h = n / 2 + 1;
  const std::size_t plane = static_cast<std::size_t>(n) * n;  // one spectrum
  const std::size_t hplane = static_cast<std::size_t>(n) * h;  // one kz plane of the half spectrum
  {  // volume blockIdx.y of a batch: its own spectra, k-space arrays and filled count
    const std::size_t v = blockIdx.y;
    spectra += v * count * plane;
    a += v * nz * hplane;
    hits += v * nz * hplane;
    filled += v;
  }
  const int lane = static_cast<int>(threadIdx.x) & 31;
  const int warp = static_cast<int>(threadIdx.x) >> 5;
  // Shared memory: the block's output tile, one padded row per column (a_tile[col][pitch]: a warp writes
  // its own row, and the read-out, consecutive threads on consecutive columns, falls on distinct banks),
  // then per warp the column sums accP[nz], accN[nz]; then per warp the counts cntP[nz], cntN[nz]; then
  // the tile's hits h_tile[col][pitch].
  const int pitch = map_pitch(nz);
  // The layout must fit the launch's shared memory (block-uniform).
  if (!QHK_CHECK(static_cast<std::size_t>(kMapCols) * (pitch * (sizeof(float2) + 1) + 2 * nz * (sizeof(float2) + 2)) <=
                 debug::dynamic_smem_bytes())) {
    return;
  }
  auto* a_tile = reinterpret_cast<float2*>(map_smem);
  float2* accP = a_tile + pitch * kMapCols + 2 * warp * nz;
  float2* accN = accP + nz;
  auto* cnt0 = reinterpret_cast<std::uint16_t*>(a_tile + pitch * kMapCols + 2 * kMapCols * nz);
  std::uint16_t* cntP = cnt0 + 2 * warp * nz;
  std::uint16_t* cntN = cntP + nz;
  auto* h_tile = reinterpret_cast<std::uint8_t*>(cnt0 + 2 * kMapCols * nz);
  const std::size_t col0 = static_cast<std::size_t>(blockIdx.x) * kMapCols;
  const std::size_t col = col0 + warp;
  unsigned long long cnt = 0;
  if (col < hplane) {  // warp-uniform
    const int ky = static_cast<int>(col / h);
    const int kx = static_cast<int>(col - static_cast<std::size_t>(ky) * h);
    const int myk = negative_bin(ky, n);
    const int mkx = negative_bin(kx, n);
    for (int k = lane; k < nz; k += 32) {
      accP[k] = make_float2(0.0f, 0.0f);
      accN[k] = make_float2(0.0f, 0.0f);
      cntP[k] = 0;
      cntN[k] = 0;
    }
    __syncwarp();
    for (int base = 0; base < count; base += 32) {
      const int ai = base + lane;
      int kp = -1, kn = -1;  // target bins of side P and side N (already negated), -1: none
      float2 vp = make_float2(0.0f, 0.0f), vn = make_float2(0.0f, 0.0f);
      if (ai < count) {
        const float4 il = __ldg(illum + ai);
        int kz;
        float nuz;
        if (ewald_target(g, ky, kx, il.x, il.y, il.z, kz, nuz)) {
          mapped(g, nuz, kz, spectra[ai * plane + static_cast<std::size_t>(ky) * n + kx], vp.x, vp.y);
          kp = kz;
        }
        if (ewald_target(g, myk, mkx, il.x, il.y, il.z, kz, nuz)) {
          mapped(g, nuz, kz, spectra[ai * plane + static_cast<std::size_t>(myk) * n + mkx], vn.x, vn.y);
          kn = negative_bin(kz, nz);
        }
      }
      if (!QHK_CHECK(kp < nz && kn < nz)) kp = kn = -1;  // a target bin outside the column
      ordered_add(accP, cntP, kp, vp, lane);
      ordered_add(accN, cntN, kn, vn, lane);
    }
    const bool mirror_is_full_only = kx >= 1 && kx <= n / 2 - 1;
    for (int kz = lane; kz < nz; kz += 32) {
      float2 p = accP[kz], m = accN[kz];
      const float pw = static_cast<float>(cntP[kz]), nw = static_cast<float>(cntN[kz]);
      if (pw > 0.0f) p = make_float2(__fdiv_rn(p.x, pw), __fdiv_rn(p.y, pw));
      if (nw > 0.0f) m = make_float2(__fdiv_rn(m.x, nw), __fdiv_rn(m.y, nw));
      a_tile[warp * pitch + kz] = make_float2(__fmul_rn(0.5f, __fadd_rn(p.x, m.x)), __fmul_rn(0.5f, __fsub_rn(p.y, m.y)));
      h_tile[warp * pitch + kz] = static_cast<std::uint8_t>((pw > 0.0f) + (nw > 0.0f));
      cnt += (pw > 0.0f) + (mirror_is_full_only && nw > 0.0f);
    }
  }
  __syncthreads();
  // Out: kz rows of the block's columns, consecutive threads on consecutive columns.
  const int ncols = static_cast<int>(min(static_cast<std::size_t>(kMapCols), hplane - min(col0, hplane)));
  for (int i = static_cast<int>(threadIdx.x); i < nz * kMapCols; i += 32 * kMapCols) {
    const int kz = i / kMapCols, c = i - kz * kMapCols;
    if (c < ncols) {
      const std::size_t o = kz * hplane + col0 + c;
      a[o] = a_tile[c * pitch + kz];
      hits[o] = h_tile[c * pitch + kz];
    }
  }
  cnt = warp_sum(cnt);
  if (lane == 0 && cnt) atomicAdd(filled, cnt);
}

// Full complex potential (normalised) and the measured mask, for the complex solver and the plain
// Rytov reconstruction. `measured` (optional) receives a second copy of the potential.
__global__ void __launch_bounds__(256)
    k_map_full(const float2* __restrict__ spectra, const float4* __restrict__ illum, int count, Grid g,
               float2* __restrict__ pot, float2* __restrict__ measured, std::uint8_t* __restrict__ mask,
               unsigned long long* __restrict__ filled) {
  const int n = g.n, nz = g.nz;
  {  // volume blockIdx.y of a batch
    const std::size_t v = blockIdx.y;
    const std::size_t vol = nz * static_cast<std::size_t>(n) * n;
    spectra += v * count * static_cast<std::size_t>(n) * n;
    pot += v * vol;
    if (measured) measured += v * vol;
    mask += v * vol;
    filled += v;
  }
  const int chunks = (nz + kMapK - 1) / kMapK;
  const std::size_t total = static_cast<std::size_t>(chunks) * n * n;
  const std::size_t t = blockIdx.x * static_cast<std::size_t>(blockDim.x) + threadIdx.x;
  unsigned long long cnt = 0;
  if (t < total) {
    const int kx = static_cast<int>(t % n);
    const std::size_t rest = t / n;
    const int ky = static_cast<int>(rest % n);
    const int k0 = static_cast<int>(rest / n) * kMapK;
    const std::size_t plane = static_cast<std::size_t>(n) * n;
    float pre[kMapK] = {}, pim[kMapK] = {}, pw[kMapK] = {};
    for (int ai = 0; ai < count; ++ai) {
      const float4 il = __ldg(illum + ai);
      int kz;
      float nuz;
      if (ewald_target(g, ky, kx, il.x, il.y, il.z, kz, nuz) && kz >= k0 && kz < k0 + kMapK) {
        float vr, vi;
        mapped(g, nuz, kz, spectra[ai * plane + static_cast<std::size_t>(ky) * n + kx], vr, vi);
        accumulate(pre, pim, pw, kz - k0, vr, vi);
      }
    }
#pragma unroll
    for (int i = 0; i < kMapK; ++i) {
      const int kz = k0 + i;
      if (kz >= nz) break;
      float pr = pre[i], pi = pim[i];
      if (pw[i] > 0.0f) {
        pr = __fdiv_rn(pr, pw[i]);
        pi = __fdiv_rn(pi, pw[i]);
      }
      const std::size_t o = (static_cast<std::size_t>(kz) * n + ky) * n + kx;
      pot[o] = make_float2(pr, pi);
      if (measured) measured[o] = make_float2(pr, pi);
      mask[o] = pw[i] > 0.0f;
      cnt += pw[i] > 0.0f;
    }
  }
  cnt = warp_sum(cnt);
  if ((threadIdx.x & 31) == 0 && cnt) atomicAdd(filled, cnt);
}

}  // namespace

void map_half(const float2* spectra, const float4* illum, int count, const Grid& g, float2* a, std::uint8_t* hits,
              unsigned long long* filled, cudaStream_t s, int batch) {
  require(batch >= 1 && batch <= 65535, "ewald mapping: invalid batch");
  require(g.nz >= 1 && g.nz <= 1024, "ewald mapping: nz must be at most 1024");
  require(count <= 65535, "ewald mapping: at most 65535 illuminations");
  const std::size_t columns = static_cast<std::size_t>(g.n) * (g.n / 2 + 1);
  const auto launch = [&](auto kernel, int cols) {
    // Output tile, per-warp column sums and counts, tile hits, as laid out in k_map_half.
    const std::size_t smem = static_cast<std::size_t>(cols) *
                             (map_pitch(g.nz) * (sizeof(float2) + 1) + g.nz * (2 * sizeof(float2) + 2 * sizeof(std::uint16_t)));
    ensure_smem(kernel);
    kernel<<<dim3(blocks_for(columns, cols), batch), 32 * cols, smem, s>>>(spectra, illum, count, g, a, hits, filled);
  };
  // About 59 KB of shared memory per block: three blocks per SM.
  if (g.nz <= 256) {
    launch(k_map_half<8>, 8);
  } else if (g.nz <= 512) {
    launch(k_map_half<4>, 4);
  } else {
    launch(k_map_half<2>, 2);
  }
  check_launch("ewald mapping");
}

void map_full(const float2* spectra, const float4* illum, int count, const Grid& g, float2* pot, float2* measured,
              std::uint8_t* mask, unsigned long long* filled, cudaStream_t s, int batch) {
  require(batch >= 1 && batch <= 65535, "ewald mapping: invalid batch");
  const int chunks = (g.nz + kMapK - 1) / kMapK;
  const std::size_t threads = static_cast<std::size_t>(chunks) * g.n * g.n;
  k_map_full<<<dim3(blocks_for(threads, 256), batch), 256, 0, s>>>(spectra, illum, count, g, pot, measured, mask,
                                                                   filled);
  check_launch("ewald mapping");
}

std::vector<float4> illumination_table(const Grid& g, const float* illum_fyfx, int count) {
  std::vector<float4> il(count);
  for (int a = 0; a < count; ++a) {
    const float fy = illum_fyfx[2 * a];
    const float fx = illum_fyfx[2 * a + 1];
    il[a] = make_float4(fy, fx, std::sqrt(g.fm2 - fy * fy - fx * fx), 0.0f);
  }
  return il;
}

Grid make_grid(int n, int nz, float wavelength, float n_medium, float na, float pixel) {
  const float fm = n_medium / wavelength;
  const float fna = na / wavelength;
  return Grid{n,
              nz,
              1.0f / (static_cast<float>(n) * pixel),
              1.0f / (static_cast<float>(nz) * pixel),
              fm * fm,
              fna * fna,
              4.0f * std::numbers::pi_v<float> / pixel};
}

OdtPlan::OdtPlan(const OdtConfig& cfg, const float* illum_fyfx) : cfg_(cfg) {
  const Grid& g = cfg_.grid;
  const int n = g.n, nz = g.nz, h = n / 2 + 1;
  require(n >= 4 && n % 2 == 0 && nz >= 2 && nz % 2 == 0, "odt: invalid grid");
  require(cfg_.count >= 1, "odt: need at least one field");
  require(cfg_.batch >= 1 && cfg_.batch <= 65535 && static_cast<long long>(cfg_.batch) * nz <= 65535,
          "odt: batches of reconstructions need batch * nz <= 65535");
  real_ = cfg_.iterations > 0 && (cfg_.tv || cfg_.r2c);
  half_ = static_cast<std::size_t>(nz) * n * h;
  vol_ = static_cast<std::size_t>(nz) * n * n;
  const std::size_t b = cfg_.batch;
  const std::vector<float4> il = illumination_table(g, illum_fyfx, cfg_.count);
  illum_.reset(cfg_.count);
  check(cudaMemcpy(illum_.get(), il.data(), il.size() * sizeof(float4), cudaMemcpyHostToDevice), "upload illuminations");
  filled_.reset(b);
  waits_.reset(1);
  check(cudaMemset(waits_.get(), 0, waits_.bytes()), "cudaMemset");
  if (real_) {
    a_.reset(b * half_);
    hits_.reset(b * half_);
    e_.reset(b * half_);
    if (cfg_.tv) {  // GP keeps its real rows on chip (rows_c2r_r2c)
      // Per volume: the real volume, x_prev and four dual triplets (the proximal step runs volume by
      // volume; the k-space passes span the batch).
      x_.reset(b * vol_);
      xprev_.reset(b * vol_);
      dual_.reset(12 * b * vol_);
      tv_.resize(b);
      for (std::size_t v = 0; v < b; ++v) {
        tv_[v].wait_status = waits_.get();
        for (int i = 0; i < 4; ++i)
          for (int c = 0; c < 3; ++c) tv_[v].v[i][c] = dual_.get() + (12 * v + 3 * i + c) * vol_;
      }
    }
  } else {
    pot_.reset(b * vol_);
    mask_.reset(b * vol_);
    if (cfg_.iterations > 0) measured_.reset(b * vol_);
  }
  tune();
}

// Autotunes the launch shapes of this plan's passes on its own buffers (scratch at this point):
// the axis passes' tile widths and the FGP tile height (autotune.hpp). Results do not depend on
// the shapes chosen.
void OdtPlan::tune() {
  if (!autotune_enabled()) return;
  const Grid& g = cfg_.grid;
  const int n = g.n, nz = g.nz, h = n / 2 + 1;
  const std::size_t nh = static_cast<std::size_t>(n) * h;
  const std::size_t nn = static_cast<std::size_t>(n) * n;
  Stream stream;
  const cudaStream_t s = stream.get();
  const int b = cfg_.batch;
  float2* scratch = real_ ? e_.get() : pot_.get();
  const std::size_t room = static_cast<std::size_t>(b) * (real_ ? half_ : vol_);
  if (static_cast<std::size_t>(cfg_.count) * b * nn <= room) {  // the 2D FFT of the fields
    tune_axis_pass(scratch, cfg_.count * b, nn, n, static_cast<std::size_t>(n), n, true, AxisMode::plain, 1.0f,
                   AxisAux{}, s);
  }
  if (real_) {
    const AxisAux aux{a_.get(), hits_.get()};
    check(cudaMemsetAsync(a_.get(), 0, a_.bytes(), s), "cudaMemset");
    check(cudaMemsetAsync(hits_.get(), 0, hits_.bytes(), s), "cudaMemset");
    for (const bool fwd : {true, false}) {
      tune_axis_pass(scratch, b * nz, nh, n, h, h, fwd, AxisMode::plain, 1.0f, AxisAux{}, s);
    }
    tune_axis_pass(scratch, n, h, nz, nh, h, false, AxisMode::from_data, 1.0f, aux, s, b, half_);
    tune_axis_pass(scratch, n, h, nz, nh, h, true, AxisMode::restore_half, 1.0f, aux, s, b, half_);
    if (cfg_.tv) tune_tv(x_.get(), tv_[0], nz, n, n, cfg_.lambda, s);
  } else {
    for (const bool fwd : {true, false}) {
      tune_axis_pass(scratch, b * nz, nn, n, static_cast<std::size_t>(n), n, fwd, AxisMode::plain, 1.0f, AxisAux{},
                     s);
      tune_axis_pass(scratch, n, static_cast<std::size_t>(n), nz, nn, n, fwd, AxisMode::plain, 1.0f, AxisAux{}, s,
                     b, vol_);
    }
    if (cfg_.iterations > 0) {
      check(cudaMemsetAsync(mask_.get(), 0, mask_.bytes(), s), "cudaMemset");
      tune_axis_pass(scratch, n, static_cast<std::size_t>(n), nz, nn, n, true, AxisMode::restore_mask, 1.0f,
                     AxisAux{measured_.get(), mask_.get()}, s, b, vol_);
    }
  }
  check(cudaStreamSynchronize(s), "autotune");
}

std::size_t OdtPlan::device_bytes() const {
  return illum_.bytes() + filled_.bytes() + a_.bytes() + hits_.bytes() + e_.bytes() + x_.bytes() + xprev_.bytes() +
         dual_.bytes() + pot_.bytes() + mask_.bytes() + measured_.bytes();
}

void OdtPlan::mark(StageClock* clock, int m, cudaStream_t s) const {
  if (clock) clock->mark(first_mark_ + m, s);
}

void OdtPlan::run(float2* fields, float* index, cudaStream_t s, StageClock* clock) {
  const Grid& g = cfg_.grid;
  const int n = g.n, nz = g.nz, h = n / 2 + 1;
  const std::size_t nh = static_cast<std::size_t>(n) * h;
  const std::size_t nn = static_cast<std::size_t>(n) * n;
  const float inv = 1.0f / (static_cast<float>(nz) * static_cast<float>(n) * static_cast<float>(n));

  {
    const NvtxRange r("qhk:fft2");
    fft2d(fields, cfg_.count * cfg_.batch, n, true, 1.0f, s);
  }
  mark(clock, kMarkFft2, s);
  check(cudaMemsetAsync(filled_.get(), 0, filled_.bytes(), s), "cudaMemset");
  mark(clock, kMarkClear, s);
  if (real_) {
    const NvtxRange r("qhk:mapping");
    map_half(fields, illum_.get(), cfg_.count, g, a_.get(), hits_.get(), filled_.get(), s, cfg_.batch);
  } else {
    const NvtxRange r("qhk:mapping");
    map_full(fields, illum_.get(), cfg_.count, g, pot_.get(), measured_.get(), mask_.get(), filled_.get(), s,
             cfg_.batch);
  }
  mark(clock, kMarkMapping, s);
  mark(clock, kMarkNormalize, s);

  const NvtxRange r("qhk:solve");
  if (real_) {
    solve_real(index, inv, s);
  } else {
    solve_complex(index, inv, s);
  }
  mark(clock, kMarkSolve, s);
  mark(clock, kMarkFinish, s);
}

// Half-spectrum loops (src/cpu/odt.cpp:76-120). x = irfft3(a) inv first; the k-space step is the
// z pass (forward, restore, inverse); FISTA-TV then runs the proximal step on the C2R output.
void OdtPlan::solve_real(float* index, float inv, cudaStream_t s) {
  const Grid& g = cfg_.grid;
  const int n = g.n, nz = g.nz, h = n / 2 + 1;
  const std::size_t nh = static_cast<std::size_t>(n) * h;
  const int b = cfg_.batch;  // volumes, one after another: y passes and rows span the batch
  const std::size_t rows = static_cast<std::size_t>(b) * nz * n;
  float2* e = e_.get();
  const AxisAux aux{a_.get(), hits_.get()};
  // E = a * inv, inverse along z, then y, then C2R along x.
  axis_pass(e, n, h, nz, nh, h, false, AxisMode::from_data, inv, aux, s, b, half_);
  axis_pass(e, b * nz, nh, n, h, h, false, AxisMode::plain, 1.0f, AxisAux{}, s);
  if (!cfg_.tv) {
    // GP: x = C2R(E); each step clamps x, R2C, y, z restore, y, C2R. The C2R, the clamp and the next
    // R2C run as one row pass, so x stays on chip between steps; the last C2R writes the index.
    for (int it = 0; it < cfg_.iterations; ++it) {
      rows_c2r_r2c(e, rows, n, s);
      axis_pass(e, b * nz, nh, n, h, h, true, AxisMode::plain, 1.0f, AxisAux{}, s);
      axis_pass(e, n, h, nz, nh, h, true, AxisMode::restore_half, inv, aux, s, b, half_);
      axis_pass(e, b * nz, nh, n, h, h, false, AxisMode::plain, 1.0f, AxisAux{}, s);
    }
    rows_c2r(e, index, rows, n, C2rMode::index, cfg_.nm2, cfg_.inv_k02, s);
    return;
  }
  rows_c2r(e, x_.get(), rows, n, C2rMode::store, cfg_.nm2, cfg_.inv_k02, s);
  const auto kspace_step = [&](const float* in, bool clamp, float* out, C2rMode mode) {
    rows_r2c(in, e, rows, n, clamp, s);
    axis_pass(e, b * nz, nh, n, h, h, true, AxisMode::plain, 1.0f, AxisAux{}, s);
    axis_pass(e, n, h, nz, nh, h, true, AxisMode::restore_half, inv, aux, s, b, half_);
    axis_pass(e, b * nz, nh, n, h, h, false, AxisMode::plain, 1.0f, AxisAux{}, s);
    rows_c2r(e, out, rows, n, mode, cfg_.nm2, cfg_.inv_k02, s);
  };
  // FISTA-TV: y lives in x_ (it is also b, the C2R output), x_prev in xprev_, the dual in dual_; volume v
  // of a batch at offset v * vol_ of x_, xprev_ and the index, its half spectrum at v * half_ of E.
  const std::size_t vbytes = vol_ * sizeof(float);
  check(cudaMemcpyAsync(xprev_.get(), x_.get(), b * vbytes, cudaMemcpyDeviceToDevice, s), "copy x");
  for (int v = 0; v < b; ++v) {
    check(cudaMemsetAsync(tv_[v].v[0][0], 0, 3 * vbytes, s), "cudaMemset");
    tv_[v].p_index = 0;
  }
  float t = 1.0f;
  // Between iterations the final primal, the momentum point y and y's R2C run as one row pass
  // (rows_tv_final_r2c), so y is never written: the next k-space step starts from its spectra.
  for (int it = 0; it < cfg_.iterations; ++it) {
    const bool last = it == cfg_.iterations - 1;
    if (it == 0) {
      const NvtxRange r("qhk:kspace");
      kspace_step(x_.get(), false, x_.get(), C2rMode::store);
    } else {
      const NvtxRange r("qhk:kspace");
      axis_pass(e, b * nz, nh, n, h, h, true, AxisMode::plain, 1.0f, AxisAux{}, s);
      axis_pass(e, n, h, nz, nh, h, true, AxisMode::restore_half, inv, aux, s, b, half_);
      axis_pass(e, b * nz, nh, n, h, h, false, AxisMode::plain, 1.0f, AxisAux{}, s);
      rows_c2r(e, x_.get(), rows, n, C2rMode::store, cfg_.nm2, cfg_.inv_k02, s);
    }
    const float tn = fista_t(t);
    const float m = (t - 1.0f) / tn;
    const NvtxRange r("qhk:tv_prox");
    cudaStreamCaptureStatus capturing = cudaStreamCaptureStatusNone;
    check(cudaStreamIsCapturing(s, &capturing), "cudaStreamIsCapturing");
    const bool timed = prox_timing_ && !last && capturing == cudaStreamCaptureStatusNone;
    const std::uint64_t launches0 = g_launches.load(std::memory_order_relaxed);
    if (timed) {
      prox_events_.emplace_back();
      check(cudaEventRecord(prox_events_.back().start(), s), "cudaEventRecord");
    }
    for (int v = 0; v < b; ++v) {
      float* xv = x_.get() + v * vol_;
      float* pv = xprev_.get() + v * vol_;
      if (last) {
        tv_prox(xv, tv_[v], nz, n, n, cfg_.lambda, cfg_.tv_inner, TvFinal::index, m, pv, index + v * vol_, cfg_.nm2,
                cfg_.inv_k02, s);
      } else {
        tv_prox(xv, tv_[v], nz, n, n, cfg_.lambda, cfg_.tv_inner, TvFinal::none, m, pv, xv, cfg_.nm2, cfg_.inv_k02,
                s);
      }
    }
    if (timed) {  // the proximal steps only: the fused row passes below are not FGP work
      check(cudaEventRecord(prox_events_.back().end(), s), "cudaEventRecord");
      prox_launches_ += g_launches.load(std::memory_order_relaxed) - launches0;
    }
    if (!last) {
      for (int v = 0; v < b; ++v) {
        const TvBuffers& tb = tv_[v];
        rows_tv_final_r2c(x_.get() + v * vol_, tb.v[tb.p_index], nz, n, n, cfg_.lambda, m, xprev_.get() + v * vol_,
                          e + v * half_, s);
      }
    }
    t = tn;
  }
}

void OdtPlan::enable_prox_timing(bool on) {
  prox_timing_ = on && cfg_.tv;
  prox_timing();  // drops what an earlier count recorded
}

std::pair<double, std::uint64_t> OdtPlan::prox_timing() {
  double ms = 0.0;
  for (const EventPair& e : prox_events_) {
    float t = 0.0f;
    check(cudaEventSynchronize(e.end()), "cudaEventSynchronize");
    check(cudaEventElapsedTime(&t, e.start(), e.end()), "cudaEventElapsedTime");
    ms += t;
  }
  prox_events_.clear();
  const std::uint64_t n = prox_launches_;
  prox_launches_ = 0;
  return {ms, n};
}

// Full complex spectra (src/cpu/odt.cpp:208-240): plain Rytov ODT, or GP with the C2C transforms.
void OdtPlan::solve_complex(float* index, float inv, cudaStream_t s) {
  const Grid& g = cfg_.grid;
  const int n = g.n, nz = g.nz;
  const std::size_t nn = static_cast<std::size_t>(n) * n;
  const int b = cfg_.batch;
  const std::size_t rows = static_cast<std::size_t>(b) * nz * n;
  float2* p = pot_.get();
  const AxisAux aux{measured_.get(), mask_.get()};
  axis_pass(p, n, n, nz, nn, n, false, AxisMode::plain, 1.0f, AxisAux{}, s, b, vol_);
  axis_pass(p, b * nz, nn, n, n, n, false, AxisMode::plain, 1.0f, AxisAux{}, s);
  for (int it = 0; it < cfg_.iterations; ++it) {
    rows_c2c(p, rows, n, false, RowMode::inv_clamp_fwd, inv, nullptr, 0, 0, s);
    axis_pass(p, b * nz, nn, n, n, n, true, AxisMode::plain, 1.0f, AxisAux{}, s);
    axis_pass(p, n, n, nz, nn, n, true, AxisMode::restore_mask, 1.0f, aux, s, b, vol_);
    axis_pass(p, b * nz, nn, n, n, n, false, AxisMode::plain, 1.0f, AxisAux{}, s);
  }
  rows_c2c(p, rows, n, false, RowMode::inv_index, inv, index, cfg_.nm2, cfg_.inv_k02, s);
}

}  // namespace qhk
