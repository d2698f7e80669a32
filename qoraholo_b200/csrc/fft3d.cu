// FFT passes over HBM-resident volumes and image stacks, built on the shared-memory engine
// (fft_engine.cuh). One kernel launch is one pass over the data along one axis: a CTA stages a
// tile of lines, transforms it on chip and writes it back, with the pointwise step that precedes
// or follows the transform folded into the load or the store:
//   * axis passes along y or z of (outer, pos, inner) data, tiles of COLS contiguous columns;
//     the z pass of the Gerchberg-Papoulis / FISTA loop runs forward transform, k-space restore
//     and inverse transform in one launch (the restore touches every voxel exactly there);
//   * real rows <-> half spectra by a half-length complex FFT (two real samples per complex
//     value) with the split / merge step in shared memory;
//   * complex rows, with the clamp of the complex GP loop between its inverse and forward row
//     transforms, or the refractive index as the epilogue of the last inverse.
#include <atomic>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <set>

#include "autotune.hpp"
#include "qhk_internal.hpp"

namespace qhk {

int sm_count() {
  int dev = 0;
  check(cudaGetDevice(&dev), "cudaGetDevice");
  int n = 0;
  check(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev), "cudaDeviceGetAttribute");
  return n;
}

FftLen make_fft_len(int n) {
  require(n >= 1, "fft: length must be positive");
  FftLen L;
  L.n = n;
  int m = n;
  const auto push = [&](int r) {
    if (L.passes >= kMaxPasses) fail(kInternal, "fft: too many passes");
    L.radix[L.passes++] = r;
    m /= r;
  };
  while (m % 8 == 0) push(8);
  if (m % 4 == 0) push(4);
  if (m % 2 == 0) push(2);
  while (m % 3 == 0) push(3);
  while (m % 5 == 0) push(5);
  for (int p = 7; m > 1; p += 2) {
    while (m % p == 0) push(p);
  }
  return L;
}

namespace {

struct TwiddleEntry {
  FftLen len;
  DevBuf<float2> table;
};

std::mutex g_tw_mutex;
std::map<std::pair<int, int>, std::unique_ptr<TwiddleEntry>> g_tw;

template <class K>
void allow_smem(K kernel, std::size_t) {
  ensure_smem(kernel);
}

constexpr int kThreads = 256;
constexpr int kBatch = 8;  // loads in flight per thread in the strided passes

// ---- axis passes ------------------------------------------------------------------------------

template <bool Fwd, int Mode, int COLS>
__global__ void __launch_bounds__(kThreads)
    k_axis(float2* __restrict__ data, std::size_t so, std::size_t sp, int ni, FftLen L, float scale,
           const float2* __restrict__ aux_a, const std::uint8_t* __restrict__ aux_h, std::size_t sb) {
  extern __shared__ float2 sm[];
  const int n = L.n;
  float2* A = sm;
  float2* B = sm + static_cast<std::size_t>(n) * COLS;
  const int c0 = static_cast<int>(blockIdx.x) * COLS;
  const int cols = min(COLS, ni - c0);
  // Volume blockIdx.z of a batch starts sb elements after the previous one (data and aux alike).
  const std::size_t base = static_cast<std::size_t>(blockIdx.z) * sb + static_cast<std::size_t>(blockIdx.y) * so + c0;
  const int tid = static_cast<int>(threadIdx.x);
  const int nth = static_cast<int>(blockDim.x);
  constexpr int kFrom = static_cast<int>(AxisMode::from_data);
  constexpr int kHalf = static_cast<int>(AxisMode::restore_half);
  constexpr int kMask = static_cast<int>(AxisMode::restore_mask);

  // Loads are issued kBatch at a time per thread before any is used, so that a CTA keeps
  // kBatch * blockDim loads in flight (the columns are strided lines; a load-use loop is
  // latency bound).
  const int total = n * COLS;
  for (int i0 = tid; i0 < total; i0 += nth * kBatch) {
    float2 v[kBatch];
#pragma unroll
    for (int b = 0; b < kBatch; ++b) {
      const int idx = i0 + b * nth;
      const int pos = idx / COLS;
      const int col = idx - pos * COLS;
      v[b] = make_float2(0.0f, 0.0f);
      if (idx < total && col < cols) {
        const std::size_t g = base + pos * sp + col;
        v[b] = Mode == kFrom ? cscale(aux_a[g], scale) : data[g];
      }
    }
#pragma unroll
    for (int b = 0; b < kBatch; ++b) {
      const int idx = i0 + b * nth;
      if (idx < total) A[idx] = v[b];
    }
  }
  __syncthreads();

  float2* res;
  if constexpr (Mode == kHalf || Mode == kMask) {
    res = smem_fft_cols<true, COLS>(A, B, COLS, L, tid, nth);
    float2* other = res == A ? B : A;
    for (int i0 = tid; i0 < total; i0 += nth * kBatch) {
      float2 av[kBatch];
      std::uint8_t hv[kBatch];
#pragma unroll
      for (int b = 0; b < kBatch; ++b) {
        const int idx = i0 + b * nth;
        const int pos = idx / COLS;
        const int col = idx - pos * COLS;
        av[b] = make_float2(0.0f, 0.0f);
        hv[b] = 0;
        if (idx < total && col < cols) {
          const std::size_t g = base + pos * sp + col;
          av[b] = aux_a[g];
          hv[b] = aux_h[g];
        }
      }
#pragma unroll
      for (int b = 0; b < kBatch; ++b) {
        const int idx = i0 + b * nth;
        const int pos = idx / COLS;
        const int col = idx - pos * COLS;
        if (idx >= total || col >= cols) continue;
        float2 v = res[idx];
        if constexpr (Mode == kHalf) {
          const float2 a = av[b];
          const float w = 1.0f - 0.5f * static_cast<float>(hv[b]);
          v = make_float2((a.x + w * v.x) * scale, (a.y + w * v.y) * scale);
        } else {
          if (hv[b]) v = av[b];
        }
        res[idx] = v;
      }
    }
    __syncthreads();
    res = smem_fft_cols<false, COLS>(res, other, COLS, L, tid, nth);
  } else {
    res = smem_fft_cols<Fwd, COLS>(A, B, COLS, L, tid, nth);
  }

  for (int idx = tid; idx < n * COLS; idx += nth) {
    const int pos = idx / COLS;
    const int col = idx - pos * COLS;
    if (col >= cols) continue;
    float2 v = res[idx];
    if (Mode == static_cast<int>(AxisMode::plain) && scale != 1.0f) v = cscale(v, scale);
    data[base + pos * sp + col] = v;
  }
}

template <bool Fwd, int Mode, int COLS>
void launch_axis(float2* data, int n_outer, std::size_t so, int n, std::size_t sp, int ni, float scale,
                 const AxisAux& aux, int batch, std::size_t sb, cudaStream_t s) {
  const FftLen& L = fft_len(n);
  const std::size_t smem = 2 * static_cast<std::size_t>(n) * COLS * sizeof(float2);
  auto kernel = k_axis<Fwd, Mode, COLS>;
  allow_smem(kernel, smem);
  const dim3 grid((ni + COLS - 1) / COLS, n_outer, batch);
  kernel<<<grid, kThreads, smem, s>>>(data, so, sp, ni, L, scale, aux.a, aux.hits, sb);
  check_launch("fft axis pass");
}

template <int Mode, int COLS>
void axis_dispatch_dir(bool forward, float2* data, int n_outer, std::size_t so, int n, std::size_t sp,
                       int ni, float scale, const AxisAux& aux, int batch, std::size_t sb, cudaStream_t s) {
  if (forward) {
    launch_axis<true, Mode, COLS>(data, n_outer, so, n, sp, ni, scale, aux, batch, sb, s);
  } else {
    launch_axis<false, Mode, COLS>(data, n_outer, so, n, sp, ni, scale, aux, batch, sb, s);
  }
}

template <int COLS>
void axis_dispatch(float2* data, int n_outer, std::size_t so, int n, std::size_t sp, int ni, bool forward,
                   AxisMode mode, float scale, const AxisAux& aux, int batch, std::size_t sb, cudaStream_t s) {
  switch (mode) {
    case AxisMode::plain:
      axis_dispatch_dir<0, COLS>(forward, data, n_outer, so, n, sp, ni, scale, aux, batch, sb, s);
      break;
    case AxisMode::restore_half:
      launch_axis<true, 1, COLS>(data, n_outer, so, n, sp, ni, scale, aux, batch, sb, s);
      break;
    case AxisMode::restore_mask:
      launch_axis<true, 2, COLS>(data, n_outer, so, n, sp, ni, scale, aux, batch, sb, s);
      break;
    case AxisMode::from_data:
      launch_axis<false, 3, COLS>(data, n_outer, so, n, sp, ni, scale, aux, batch, sb, s);
      break;
  }
}

// Row transforms with the length known at compile time (MC > 0) or at run time (MC = 0): with
// MC the index arithmetic of the staging loops is by constants, not runtime divisions.
template <bool Fwd, int COLS, int MC>
__device__ __forceinline__ float2* row_fft(float2* a, float2* b, int cp, const FftLen& L, int tid, int nth) {
  if constexpr (MC > 0) {
    return fftdev::passes_fixed<MC, 0, 1, Fwd, COLS>(a, b, cp, L.tw, tid, nth);
  } else {
    return smem_fft_cols<Fwd, COLS>(a, b, cp, L, tid, nth);
  }
}

// ---- real rows <-> half spectra -----------------------------------------------------------------

template <bool Clamp, int COLS, int MC>
__global__ void __launch_bounds__(kThreads)
    k_rows_r2c(const float* __restrict__ x, float2* __restrict__ e, std::size_t rows, int nx, FftLen Lm,
               const float2* __restrict__ twn) {
  extern __shared__ float2 sm[];
  constexpr int cp = COLS + 1;
  const int M = MC > 0 ? MC : Lm.n;
  const int h = M + 1;
  float2* A = sm;
  float2* B = sm + static_cast<std::size_t>(h) * cp;
  const std::size_t r0 = static_cast<std::size_t>(blockIdx.x) * COLS;
  const int nr = static_cast<int>(min(static_cast<std::size_t>(COLS), rows - r0));
  const int tid = static_cast<int>(threadIdx.x);
  const int nth = static_cast<int>(blockDim.x);

  for (int idx = tid; idx < M * COLS; idx += nth) {
    const int row = idx / M;
    const int m = idx - row * M;
    float2 v = make_float2(0.0f, 0.0f);
    if (row < nr) {
      v = *reinterpret_cast<const float2*>(x + (r0 + row) * nx + 2 * m);
      if (Clamp) v = make_float2(fmaxf(v.x, 0.0f), fmaxf(v.y, 0.0f));
    }
    A[m * cp + row] = v;
  }
  __syncthreads();
  const float2* res = row_fft<true, COLS, MC>(A, B, cp, Lm, tid, nth);

  for (int idx = tid; idx < h * COLS; idx += nth) {
    const int row = idx / h;
    const int k = idx - row * h;
    if (row >= nr) continue;
    const float2 zk = res[(k == M ? 0 : k) * cp + row];
    const float2 zm = res[(k == 0 ? 0 : M - k) * cp + row];
    const float2 ev = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
    const float2 d = make_float2(zk.x - zm.x, zk.y + zm.y);  // zk - conj(zm)
    const float2 od = make_float2(0.5f * d.y, -0.5f * d.x);   // d / (2i)
    const float2 w = __ldg(twn + k);
    e[(r0 + row) * h + k] = cadd(ev, cmul(w, od));
  }
}

template <int Mode, int COLS, int MC>
__global__ void __launch_bounds__(kThreads)
    k_rows_c2r(const float2* __restrict__ e, float* __restrict__ x, std::size_t rows, int nx, FftLen Lm,
               const float2* __restrict__ twn, float nm2, float inv_k02) {
  extern __shared__ float2 sm[];
  constexpr int cp = COLS + 1;
  const int M = MC > 0 ? MC : Lm.n;
  const int h = M + 1;
  float2* A = sm;
  float2* B = sm + static_cast<std::size_t>(h) * cp;
  const std::size_t r0 = static_cast<std::size_t>(blockIdx.x) * COLS;
  const int nr = static_cast<int>(min(static_cast<std::size_t>(COLS), rows - r0));
  const int tid = static_cast<int>(threadIdx.x);
  const int nth = static_cast<int>(blockDim.x);

  for (int idx = tid; idx < h * COLS; idx += nth) {
    const int row = idx / h;
    const int k = idx - row * h;
    A[k * cp + row] = row < nr ? e[(r0 + row) * h + k] : make_float2(0.0f, 0.0f);
  }
  __syncthreads();
  for (int idx = tid; idx < M * COLS; idx += nth) {
    const int k = idx / COLS;
    const int row = idx - k * COLS;
    float2 xk = A[k * cp + row];
    float2 xm = A[(M - k) * cp + row];
    if (k == 0) {  // a real signal has real bins 0 and M; their imaginary parts drop out
      xk.y = 0.0f;
      xm.y = 0.0f;
    }
    const float2 sv = make_float2(xk.x + xm.x, xk.y - xm.y);  // xk + conj(xm)
    const float2 d = make_float2(xk.x - xm.x, xk.y + xm.y);   // xk - conj(xm)
    const float2 w = __ldg(twn + k);
    const float2 t = cmulc(d, w);                              // d * e^{+2 pi i k / nx}
    B[k * cp + row] = make_float2(sv.x - t.y, sv.y + t.x);     // sv + i t
  }
  __syncthreads();
  const float2* res = row_fft<false, COLS, MC>(B, A, cp, Lm, tid, nth);

  for (int idx = tid; idx < M * COLS; idx += nth) {
    const int row = idx / M;
    const int m = idx - row * M;
    if (row >= nr) continue;
    float2 z = res[m * cp + row];
    if (Mode == static_cast<int>(C2rMode::index)) {
      z = make_float2(index_from_potential(z.x, 0.0f, nm2, inv_k02), index_from_potential(z.y, 0.0f, nm2, inv_k02));
    }
    *reinterpret_cast<float2*>(x + (r0 + row) * nx + 2 * m) = z;
  }
}

// One boundary between two Gerchberg-Papoulis steps on rows, in place: the C2R of the half spectra,
// the real-space constraint max(x, 0) and the R2C of the constrained rows, without the real rows
// going through HBM. The operations are those of k_rows_c2r (store) followed by k_rows_r2c (Clamp)
// on the same values, so the half spectra are bitwise the same. Each CTA reads all its rows before
// it writes any, so `e` is updated in place.
template <int COLS, int MC>
__global__ void __launch_bounds__(kThreads)
    k_rows_c2r_r2c(float2* __restrict__ e, std::size_t rows, FftLen Lm, const float2* __restrict__ twn) {
  extern __shared__ float2 sm[];
  constexpr int cp = COLS + 1;
  const int M = MC > 0 ? MC : Lm.n;
  const int h = M + 1;
  float2* A = sm;
  float2* B = sm + static_cast<std::size_t>(h) * cp;
  const std::size_t r0 = static_cast<std::size_t>(blockIdx.x) * COLS;
  const int nr = static_cast<int>(min(static_cast<std::size_t>(COLS), rows - r0));
  const int tid = static_cast<int>(threadIdx.x);
  const int nth = static_cast<int>(blockDim.x);

  for (int idx = tid; idx < h * COLS; idx += nth) {
    const int row = idx / h;
    const int k = idx - row * h;
    A[k * cp + row] = row < nr ? e[(r0 + row) * h + k] : make_float2(0.0f, 0.0f);
  }
  __syncthreads();
  for (int idx = tid; idx < M * COLS; idx += nth) {
    const int k = idx / COLS;
    const int row = idx - k * COLS;
    float2 xk = A[k * cp + row];
    float2 xm = A[(M - k) * cp + row];
    if (k == 0) {  // a real signal has real bins 0 and M; their imaginary parts drop out
      xk.y = 0.0f;
      xm.y = 0.0f;
    }
    const float2 sv = make_float2(xk.x + xm.x, xk.y - xm.y);  // xk + conj(xm)
    const float2 d = make_float2(xk.x - xm.x, xk.y + xm.y);   // xk - conj(xm)
    const float2 w = __ldg(twn + k);
    const float2 t = cmulc(d, w);                              // d * e^{+2 pi i k / nx}
    B[k * cp + row] = make_float2(sv.x - t.y, sv.y + t.x);     // sv + i t
  }
  __syncthreads();
  float2* real = row_fft<false, COLS, MC>(B, A, cp, Lm, tid, nth);  // real samples 2m, 2m+1 of each row
  for (int idx = tid; idx < M * COLS; idx += nth) {
    const int row = idx / M;
    const int m = idx - row * M;
    float2 v = make_float2(0.0f, 0.0f);
    if (row < nr) {
      v = real[m * cp + row];
      v = make_float2(fmaxf(v.x, 0.0f), fmaxf(v.y, 0.0f));
    }
    real[m * cp + row] = v;
  }
  __syncthreads();
  const float2* res = row_fft<true, COLS, MC>(real, real == A ? B : A, cp, Lm, tid, nth);

  for (int idx = tid; idx < h * COLS; idx += nth) {
    const int row = idx / h;
    const int k = idx - row * h;
    if (row >= nr) continue;
    const float2 zk = res[(k == M ? 0 : k) * cp + row];
    const float2 zm = res[(k == 0 ? 0 : M - k) * cp + row];
    const float2 ev = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
    const float2 d = make_float2(zk.x - zm.x, zk.y + zm.y);  // zk - conj(zm)
    const float2 od = make_float2(0.5f * d.y, -0.5f * d.x);   // d / (2i)
    const float2 w = __ldg(twn + k);
    e[(r0 + row) * h + k] = cadd(ev, cmul(w, od));
  }
}

// The end of one FISTA-TV iteration and the start of the next on rows: the final primal of the
// proximal step x = max(b - lambda div p, 0) (as k_tv_final: the same additions in the same order),
// the FISTA point y = x + m (x - xprev), xprev <- x, and the R2C of y's rows into the half spectra e,
// y itself never written to HBM. Each row r = z * ny + y of the volume (dense (nz, ny, 2M)) is one
// column of the tile; its divergence reads p_z of plane z - 1 and p_y of row y - 1 from HBM (L2).
template <int COLS, int MC>
__global__ void __launch_bounds__(kThreads)
    k_rows_tv_final_r2c(const float* __restrict__ b, const float* __restrict__ pz, const float* __restrict__ py,
                        const float* __restrict__ px, int nz, int ny, float lambda, float momentum,
                        float* __restrict__ xprev, float2* __restrict__ e, std::size_t rows, FftLen Lm,
                        const float2* __restrict__ twn) {
  extern __shared__ float2 sm[];
  constexpr int cp = COLS + 1;
  const int M = MC > 0 ? MC : Lm.n;
  const int h = M + 1;
  const int nx = 2 * M;
  const std::size_t nxy = static_cast<std::size_t>(nx) * ny;
  float2* A = sm;
  float2* B = sm + static_cast<std::size_t>(h) * cp;
  const std::size_t r0 = static_cast<std::size_t>(blockIdx.x) * COLS;
  const int nr = static_cast<int>(min(static_cast<std::size_t>(COLS), rows - r0));
  const int tid = static_cast<int>(threadIdx.x);
  const int nth = static_cast<int>(blockDim.x);
  // Plane and image row of the tile's first volume row, by one division; those of the others by
  // counting on from it (a 64-bit division per loaded item cost more than the item's arithmetic).
  const int y_first = static_cast<int>(r0 % static_cast<std::size_t>(ny));
  const int z_first = static_cast<int>(r0 / static_cast<std::size_t>(ny));

  for (int idx = tid; idx < M * COLS; idx += nth) {
    const int row = idx / M;
    const int m = idx - row * M;
    float2 v = make_float2(0.0f, 0.0f);
    if (row < nr) {
      const std::size_t r = r0 + row;
      int y = y_first + row, z = z_first;
      while (y >= ny) y -= ny, ++z;  // row < COLS: at most ceil(COLS / ny) steps
      const std::size_t i0 = r * nx + 2 * m;
      const float2 bv = *reinterpret_cast<const float2*>(b + i0);
      const float2 cz = *reinterpret_cast<const float2*>(pz + i0);
      const float2 cy = *reinterpret_cast<const float2*>(py + i0);
      const float2 cx = *reinterpret_cast<const float2*>(px + i0);
      const float2 pv = *reinterpret_cast<const float2*>(xprev + i0);
      float2 bz = make_float2(0.0f, 0.0f), by = make_float2(0.0f, 0.0f);
      if (z > 0) bz = *reinterpret_cast<const float2*>(pz + i0 - nxy);
      if (y > 0) by = *reinterpret_cast<const float2*>(py + i0 - nx);
      const float left = m > 0 ? px[i0 - 1] : 0.0f;
      const float bb[2] = {bv.x, bv.y}, czz[2] = {cz.x, cz.y}, cyy[2] = {cy.x, cy.y}, cxx[2] = {cx.x, cx.y};
      const float bzz[2] = {bz.x, bz.y}, byy[2] = {by.x, by.y}, pvv[2] = {pv.x, pv.y};
      float xv[2], yv[2];
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const int x = 2 * m + i;
        float sdiv = 0.0f;
        if (z < nz - 1) sdiv = __fadd_rn(sdiv, czz[i]);
        if (z > 0) sdiv = __fsub_rn(sdiv, bzz[i]);
        if (y < ny - 1) sdiv = __fadd_rn(sdiv, cyy[i]);
        if (y > 0) sdiv = __fsub_rn(sdiv, byy[i]);
        if (x < nx - 1) sdiv = __fadd_rn(sdiv, cxx[i]);
        if (x > 0) sdiv = __fsub_rn(sdiv, i == 0 ? left : cxx[0]);
        xv[i] = tv_primal(bb[i], lambda, sdiv);
        yv[i] = __fadd_rn(xv[i], __fmul_rn(momentum, __fsub_rn(xv[i], pvv[i])));
      }
      *reinterpret_cast<float2*>(xprev + i0) = make_float2(xv[0], xv[1]);
      v = make_float2(yv[0], yv[1]);
    }
    A[m * cp + row] = v;
  }
  __syncthreads();
  const float2* res = row_fft<true, COLS, MC>(A, B, cp, Lm, tid, nth);

  for (int idx = tid; idx < h * COLS; idx += nth) {
    const int row = idx / h;
    const int k = idx - row * h;
    if (row >= nr) continue;
    const float2 zk = res[(k == M ? 0 : k) * cp + row];
    const float2 zm = res[(k == 0 ? 0 : M - k) * cp + row];
    const float2 ev = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
    const float2 d = make_float2(zk.x - zm.x, zk.y + zm.y);  // zk - conj(zm)
    const float2 od = make_float2(0.5f * d.y, -0.5f * d.x);   // d / (2i)
    const float2 w = __ldg(twn + k);
    e[(r0 + row) * h + k] = cadd(ev, cmul(w, od));
  }
}

// ---- complex rows -----------------------------------------------------------------------------------

template <bool Fwd, int Mode, int COLS, int NC>
__global__ void __launch_bounds__(kThreads)
    k_rows_c2c(float2* __restrict__ data, std::size_t rows, FftLen L, float scale, float* __restrict__ index,
               float nm2, float inv_k02) {
  extern __shared__ float2 sm[];
  constexpr int cp = COLS + 1;
  const int n = NC > 0 ? NC : L.n;
  float2* A = sm;
  float2* B = sm + static_cast<std::size_t>(n) * cp;
  const std::size_t r0 = static_cast<std::size_t>(blockIdx.x) * COLS;
  const int nr = static_cast<int>(min(static_cast<std::size_t>(COLS), rows - r0));
  const int tid = static_cast<int>(threadIdx.x);
  const int nth = static_cast<int>(blockDim.x);

  for (int idx = tid; idx < n * COLS; idx += nth) {
    const int row = idx / n;
    const int pos = idx - row * n;
    A[pos * cp + row] = row < nr ? data[(r0 + row) * n + pos] : make_float2(0.0f, 0.0f);
  }
  __syncthreads();
  float2* res;
  if constexpr (Mode == static_cast<int>(RowMode::plain)) {
    res = row_fft<Fwd, COLS, NC>(A, B, cp, L, tid, nth);
  } else {
    res = row_fft<false, COLS, NC>(A, B, cp, L, tid, nth);
    if constexpr (Mode == static_cast<int>(RowMode::inv_clamp_fwd)) {
      float2* other = res == A ? B : A;
      for (int idx = tid; idx < n * COLS; idx += nth) {
        const int pos = idx / COLS;
        const int row = idx - pos * COLS;
        const float2 v = res[pos * cp + row];
        res[pos * cp + row] = make_float2(fmaxf(v.x * scale, 0.0f), 0.0f);
      }
      __syncthreads();
      res = row_fft<true, COLS, NC>(res, other, cp, L, tid, nth);
    }
  }
  for (int idx = tid; idx < n * COLS; idx += nth) {
    const int row = idx / n;
    const int pos = idx - row * n;
    if (row >= nr) continue;
    const float2 v = res[pos * cp + row];
    if constexpr (Mode == static_cast<int>(RowMode::inv_index)) {
      index[(r0 + row) * n + pos] = index_from_potential(v.x * scale, v.y * scale, nm2, inv_k02);
    } else if constexpr (Mode == static_cast<int>(RowMode::plain)) {
      data[(r0 + row) * n + pos] = scale != 1.0f ? cscale(v, scale) : v;
    } else {
      data[(r0 + row) * n + pos] = v;
    }
  }
}

// Rows per CTA: as many as fit a 64 KiB double buffer, at most 16.
constexpr int rows_per_cta(int n) {
  int c = 16;
  while (c > 1 && 2 * static_cast<std::size_t>(n + 1) * (c + 1) * sizeof(float2) > 64 * 1024) c /= 2;
  return c;
}

template <int COLS, int MC>
void launch_r2c(const float* x, float2* e, std::size_t rows, int nx, bool clamp, cudaStream_t s) {
  const int M = nx / 2;
  const FftLen& Lm = fft_len(M);
  const FftLen& Ln = fft_len(nx);
  const std::size_t smem = 2 * static_cast<std::size_t>(M + 1) * (COLS + 1) * sizeof(float2);
  const unsigned grid = static_cast<unsigned>((rows + COLS - 1) / COLS);
  if (clamp) {
    allow_smem(k_rows_r2c<true, COLS, MC>, smem);
    k_rows_r2c<true, COLS, MC><<<grid, kThreads, smem, s>>>(x, e, rows, nx, Lm, Ln.tw);
  } else {
    allow_smem(k_rows_r2c<false, COLS, MC>, smem);
    k_rows_r2c<false, COLS, MC><<<grid, kThreads, smem, s>>>(x, e, rows, nx, Lm, Ln.tw);
  }
  check_launch("rows r2c");
}

template <int COLS, int MC>
void launch_tv_final_r2c(const float* b, const float* const p[3], int nz, int ny, int nx, float lambda,
                         float momentum, float* xprev, float2* e, cudaStream_t s) {
  const int M = nx / 2;
  const FftLen& Lm = fft_len(M);
  const FftLen& Ln = fft_len(nx);
  const std::size_t rows = static_cast<std::size_t>(nz) * ny;
  const std::size_t smem = 2 * static_cast<std::size_t>(M + 1) * (COLS + 1) * sizeof(float2);
  const unsigned grid = static_cast<unsigned>((rows + COLS - 1) / COLS);
  allow_smem(k_rows_tv_final_r2c<COLS, MC>, smem);
  k_rows_tv_final_r2c<COLS, MC><<<grid, kThreads, smem, s>>>(b, p[0], p[1], p[2], nz, ny, lambda, momentum, xprev,
                                                              e, rows, Lm, Ln.tw);
  check_launch("rows tv final r2c");
}

template <int COLS, int MC>
void launch_c2r_r2c(float2* e, std::size_t rows, int nx, cudaStream_t s) {
  const int M = nx / 2;
  const FftLen& Lm = fft_len(M);
  const FftLen& Ln = fft_len(nx);
  const std::size_t smem = 2 * static_cast<std::size_t>(M + 1) * (COLS + 1) * sizeof(float2);
  const unsigned grid = static_cast<unsigned>((rows + COLS - 1) / COLS);
  allow_smem(k_rows_c2r_r2c<COLS, MC>, smem);
  k_rows_c2r_r2c<COLS, MC><<<grid, kThreads, smem, s>>>(e, rows, Lm, Ln.tw);
  check_launch("rows c2r r2c");
}

template <int COLS, int MC>
void launch_c2r(const float2* e, float* x, std::size_t rows, int nx, C2rMode mode, float nm2, float inv_k02,
                cudaStream_t s) {
  const int M = nx / 2;
  const FftLen& Lm = fft_len(M);
  const FftLen& Ln = fft_len(nx);
  const std::size_t smem = 2 * static_cast<std::size_t>(M + 1) * (COLS + 1) * sizeof(float2);
  const unsigned grid = static_cast<unsigned>((rows + COLS - 1) / COLS);
  if (mode == C2rMode::index) {
    allow_smem(k_rows_c2r<1, COLS, MC>, smem);
    k_rows_c2r<1, COLS, MC><<<grid, kThreads, smem, s>>>(e, x, rows, nx, Lm, Ln.tw, nm2, inv_k02);
  } else {
    allow_smem(k_rows_c2r<0, COLS, MC>, smem);
    k_rows_c2r<0, COLS, MC><<<grid, kThreads, smem, s>>>(e, x, rows, nx, Lm, Ln.tw, nm2, inv_k02);
  }
  check_launch("rows c2r");
}

template <bool Fwd, int Mode, int COLS, int NC>
void launch_c2c_rows(float2* data, std::size_t rows, int nx, float scale, float* index, float nm2,
                     float inv_k02, cudaStream_t s) {
  const FftLen& L = fft_len(nx);
  const std::size_t smem = 2 * static_cast<std::size_t>(nx) * (COLS + 1) * sizeof(float2);
  auto kernel = k_rows_c2c<Fwd, Mode, COLS, NC>;
  allow_smem(kernel, smem);
  const unsigned grid = static_cast<unsigned>((rows + COLS - 1) / COLS);
  kernel<<<grid, kThreads, smem, s>>>(data, rows, L, scale, index, nm2, inv_k02);
  check_launch("rows c2c");
}

template <int COLS, int NC>
void c2c_rows_dispatch(float2* data, std::size_t rows, int nx, bool forward, RowMode mode, float scale,
                       float* index, float nm2, float inv_k02, cudaStream_t s) {
  switch (mode) {
    case RowMode::plain:
      if (forward) {
        launch_c2c_rows<true, 0, COLS, NC>(data, rows, nx, scale, index, nm2, inv_k02, s);
      } else {
        launch_c2c_rows<false, 0, COLS, NC>(data, rows, nx, scale, index, nm2, inv_k02, s);
      }
      break;
    case RowMode::inv_clamp_fwd:
      launch_c2c_rows<false, 1, COLS, NC>(data, rows, nx, scale, index, nm2, inv_k02, s);
      break;
    case RowMode::inv_index:
      launch_c2c_rows<false, 2, COLS, NC>(data, rows, nx, scale, index, nm2, inv_k02, s);
      break;
  }
}

}  // namespace

std::size_t axis_smem_budget() {
  // QHK_FFT_AXIS_KIB overrides the shared-memory budget of an axis-pass tile (tuning).
  static const std::size_t budget = [] {
    const char* e = std::getenv("QHK_FFT_AXIS_KIB");
    const long v = e ? std::atol(e) : 0;
    return static_cast<std::size_t>(v > 0 ? v : 72) * 1024;
  }();
  return budget;
}

const FftLen& fft_len(int n) {
  int dev = 0;
  check(cudaGetDevice(&dev), "cudaGetDevice");
  std::lock_guard<std::mutex> lock(g_tw_mutex);
  auto& slot = g_tw[{dev, n}];
  if (!slot) {
    auto entry = std::make_unique<TwiddleEntry>();
    entry->len = make_fft_len(n);
    std::vector<float2> host(n);
    const double two_pi = 6.283185307179586476925286766559;
    for (int k = 0; k < n; ++k) {
      const double a = two_pi * static_cast<double>(k) / static_cast<double>(n);
      host[k] = make_float2(static_cast<float>(std::cos(a)), static_cast<float>(-std::sin(a)));
    }
    entry->table.reset(n);
    check(cudaMemcpy(entry->table.get(), host.data(), n * sizeof(float2), cudaMemcpyHostToDevice),
          "upload twiddles");
    entry->len.tw = entry->table.get();
    slot = std::move(entry);
  }
  return slot->len;
}

namespace {

void axis_cols(int cols, float2* data, int n_outer, std::size_t so, int n, std::size_t sp, int ni, bool forward,
               AxisMode mode, float scale, const AxisAux& aux, int batch, std::size_t sb, cudaStream_t s) {
  switch (cols) {
    case 16: axis_dispatch<16>(data, n_outer, so, n, sp, ni, forward, mode, scale, aux, batch, sb, s); break;
    case 8: axis_dispatch<8>(data, n_outer, so, n, sp, ni, forward, mode, scale, aux, batch, sb, s); break;
    case 4: axis_dispatch<4>(data, n_outer, so, n, sp, ni, forward, mode, scale, aux, batch, sb, s); break;
    default: axis_dispatch<1>(data, n_outer, so, n, sp, ni, forward, mode, scale, aux, batch, sb, s); break;
  }
}

// Tile widths whose double buffer fits a CTA, widest first, and the default: the widest whose
// buffer fits `axis_smem_budget()`.
std::vector<int> axis_candidates(int n) {
  std::vector<int> out;
  for (const int c : {16, 8, 4}) {
    if (2 * static_cast<std::size_t>(n) * c * sizeof(float2) <= 200 * 1024) out.push_back(c);
  }
  return out;
}

int axis_default(int n) {
  for (const int c : {16, 8, 4}) {
    if (2 * static_cast<std::size_t>(n) * c * sizeof(float2) <= axis_smem_budget()) return c;
  }
  return 1;
}

TuneKey axis_key(int n_outer, std::size_t so, int n, std::size_t sp, int ni, bool forward, AxisMode mode,
                 int batch) {
  return tune_key(TuneFamily::axis, {n, ni, n_outer, static_cast<long long>(so), static_cast<long long>(sp),
                                     2 * static_cast<long long>(mode) + (forward ? 1 : 0) + 16LL * batch});
}

}  // namespace

namespace {

// Engine of an axis pass (FFT decomposition): 1 and 2 the register engine's variants, 0 the staged
// engine with its own tile width.
TuneKey engine_key(int n_outer, std::size_t so, int n, std::size_t sp, int ni, bool forward, AxisMode mode,
                   int batch) {
  return tune_key(TuneFamily::axis_engine,
                  {n, ni, n_outer, static_cast<long long>(so), static_cast<long long>(sp),
                   2 * static_cast<long long>(mode) + (forward ? 1 : 0) + 16LL * batch});
}

std::atomic<int> g_radix_tuning{-1};  // -1: from the environment
std::atomic<int> g_axis_engine{-1};   // -1: the tuned or default decomposition; else forced

}  // namespace

void force_axis_engine(int engine) { g_axis_engine.store(engine, std::memory_order_relaxed); }

bool radix_tuning_enabled() {
  int v = g_radix_tuning.load(std::memory_order_relaxed);
  if (v < 0) {
    const char* e = std::getenv("QHK_AUTOTUNE_RADIX");
    v = e && std::strcmp(e, "1") == 0 ? 1 : 0;
    g_radix_tuning.store(v, std::memory_order_relaxed);
  }
  return v == 1;
}

void set_radix_tuning(bool on) { g_radix_tuning.store(on ? 1 : 0, std::memory_order_relaxed); }

void axis_pass(float2* data, int n_outer, std::size_t so, int n, std::size_t sp, int ni, bool forward,
               AxisMode mode, float scale, const AxisAux& aux, cudaStream_t s, int batch, std::size_t sb) {
  require(n_outer >= 1 && n_outer <= 65535 && batch >= 1 && batch <= 65535,
          "fft: too many lines in the outer dimension");
  const int forced = g_axis_engine.load(std::memory_order_relaxed);
  int engine = 1;
  if (forced >= 0 && forced <= axis_reg_variants(n)) {
    engine = forced;
  } else if (axis_reg_variants(n) > 0 && radix_tuning_enabled()) {
    engine = tuned_choice(engine_key(n_outer, so, n, sp, ni, forward, mode, batch), 1);
  }
  if (engine != 0 && axis_pass_reg(data, n_outer, so, n, sp, ni, forward, mode, scale, aux, s, batch, sb, engine)) {
    return;
  }
  require(static_cast<std::size_t>(n) * 2 * sizeof(float2) <= 200 * 1024, "fft: transform length too large");
  const int cols = tuned_choice(axis_key(n_outer, so, n, sp, ni, forward, mode, batch), axis_default(n));
  axis_cols(cols, data, n_outer, so, n, sp, ni, forward, mode, scale, aux, batch, sb, s);
}

void tune_axis_pass(float2* data, int n_outer, std::size_t so, int n, std::size_t sp, int ni, bool forward,
                    AxisMode mode, float scale, const AxisAux& aux, cudaStream_t s, int batch, std::size_t sb) {
  require(n_outer >= 1 && n_outer <= 65535 && batch >= 1 && batch <= 65535,
          "fft: too many lines in the outer dimension");
  if (const int variants = axis_reg_variants(n); variants > 0) {
    // The register engine covers n: its decomposition is fixed unless radix tuning is on, in which case
    // its variants and the staged engine (at its default tile width) are timed against each other.
    if (!radix_tuning_enabled()) return;
    std::vector<int> candidates{1};
    if (variants > 1) candidates.push_back(2);
    if (static_cast<std::size_t>(n) * 2 * sizeof(float2) <= 200 * 1024) candidates.push_back(0);
    autotune(engine_key(n_outer, so, n, sp, ni, forward, mode, batch), candidates, 1,
             [&](int c) {
               if (c == 0) {
                 axis_cols(axis_default(n), data, n_outer, so, n, sp, ni, forward, mode, scale, aux, batch, sb, s);
               } else {
                 axis_pass_reg(data, n_outer, so, n, sp, ni, forward, mode, scale, aux, s, batch, sb, c);
               }
             },
             s);
    return;
  }
  autotune(axis_key(n_outer, so, n, sp, ni, forward, mode, batch), axis_candidates(n), axis_default(n),
           [&](int c) { axis_cols(c, data, n_outer, so, n, sp, ni, forward, mode, scale, aux, batch, sb, s); }, s);
}

// Lengths with compile-time row kernels (the common volume and image sides); others run the
// runtime-length kernels.
#define QHK_FIXED_LENGTHS(X) X(32) X(64) X(96) X(128) X(192) X(256) X(384) X(512)

void rows_r2c(const float* x, float2* e, std::size_t rows, int nx, bool clamp, cudaStream_t s) {
  require(nx >= 2 && nx % 2 == 0, "rfft: row length must be even");
  if (rows_r2c_reg(x, e, rows, nx, clamp, s)) return;
  switch (nx / 2) {
#define QHK_R2C(M)                                                \
  case M:                                                         \
    launch_r2c<rows_per_cta(M), M>(x, e, rows, nx, clamp, s);     \
    return;
    QHK_FIXED_LENGTHS(QHK_R2C)
#undef QHK_R2C
    default: break;
  }
  switch (rows_per_cta(nx / 2)) {
    case 16: launch_r2c<16, 0>(x, e, rows, nx, clamp, s); break;
    case 8: launch_r2c<8, 0>(x, e, rows, nx, clamp, s); break;
    case 4: launch_r2c<4, 0>(x, e, rows, nx, clamp, s); break;
    case 2: launch_r2c<2, 0>(x, e, rows, nx, clamp, s); break;
    default: launch_r2c<1, 0>(x, e, rows, nx, clamp, s); break;
  }
}

void rows_c2r(const float2* e, float* x, std::size_t rows, int nx, C2rMode mode, float nm2, float inv_k02,
              cudaStream_t s) {
  require(nx >= 2 && nx % 2 == 0, "irfft: row length must be even");
  if (rows_c2r_reg(e, x, rows, nx, mode, nm2, inv_k02, s)) return;
  switch (nx / 2) {
#define QHK_C2R(M)                                                          \
  case M:                                                                   \
    launch_c2r<rows_per_cta(M), M>(e, x, rows, nx, mode, nm2, inv_k02, s);  \
    return;
    QHK_FIXED_LENGTHS(QHK_C2R)
#undef QHK_C2R
    default: break;
  }
  switch (rows_per_cta(nx / 2)) {
    case 16: launch_c2r<16, 0>(e, x, rows, nx, mode, nm2, inv_k02, s); break;
    case 8: launch_c2r<8, 0>(e, x, rows, nx, mode, nm2, inv_k02, s); break;
    case 4: launch_c2r<4, 0>(e, x, rows, nx, mode, nm2, inv_k02, s); break;
    case 2: launch_c2r<2, 0>(e, x, rows, nx, mode, nm2, inv_k02, s); break;
    default: launch_c2r<1, 0>(e, x, rows, nx, mode, nm2, inv_k02, s); break;
  }
}

void rows_c2r_r2c(float2* e, std::size_t rows, int nx, cudaStream_t s) {
  require(nx >= 2 && nx % 2 == 0, "rfft: row length must be even");
  if (rows_c2r_r2c_reg(e, rows, nx, s)) return;
  switch (nx / 2) {
#define QHK_C2R_R2C(M)                                    \
  case M:                                                 \
    launch_c2r_r2c<rows_per_cta(M), M>(e, rows, nx, s);   \
    return;
    QHK_FIXED_LENGTHS(QHK_C2R_R2C)
#undef QHK_C2R_R2C
    default: break;
  }
  switch (rows_per_cta(nx / 2)) {
    case 16: launch_c2r_r2c<16, 0>(e, rows, nx, s); break;
    case 8: launch_c2r_r2c<8, 0>(e, rows, nx, s); break;
    case 4: launch_c2r_r2c<4, 0>(e, rows, nx, s); break;
    case 2: launch_c2r_r2c<2, 0>(e, rows, nx, s); break;
    default: launch_c2r_r2c<1, 0>(e, rows, nx, s); break;
  }
}

void rows_tv_final_r2c(const float* b, const float* const p[3], int nz, int ny, int nx, float lambda, float momentum,
                       float* xprev, float2* e, cudaStream_t s) {
  require(nx >= 2 && nx % 2 == 0 && nz >= 1 && ny >= 1, "rfft: row length must be even");
  switch (nx / 2) {
#define QHK_TVF_R2C(M)                                                                           \
  case M:                                                                                        \
    launch_tv_final_r2c<rows_per_cta(M), M>(b, p, nz, ny, nx, lambda, momentum, xprev, e, s);    \
    return;
    QHK_FIXED_LENGTHS(QHK_TVF_R2C)
#undef QHK_TVF_R2C
    default: break;
  }
  switch (rows_per_cta(nx / 2)) {
    case 16: launch_tv_final_r2c<16, 0>(b, p, nz, ny, nx, lambda, momentum, xprev, e, s); break;
    case 8: launch_tv_final_r2c<8, 0>(b, p, nz, ny, nx, lambda, momentum, xprev, e, s); break;
    case 4: launch_tv_final_r2c<4, 0>(b, p, nz, ny, nx, lambda, momentum, xprev, e, s); break;
    case 2: launch_tv_final_r2c<2, 0>(b, p, nz, ny, nx, lambda, momentum, xprev, e, s); break;
    default: launch_tv_final_r2c<1, 0>(b, p, nz, ny, nx, lambda, momentum, xprev, e, s); break;
  }
}

void rows_c2c(float2* data, std::size_t rows, int nx, bool forward, RowMode mode, float scale, float* index,
              float nm2, float inv_k02, cudaStream_t s) {
  switch (nx) {
#define QHK_C2C(N)                                                                                        \
  case N:                                                                                                 \
    c2c_rows_dispatch<rows_per_cta(N), N>(data, rows, nx, forward, mode, scale, index, nm2, inv_k02, s);  \
    return;
    QHK_FIXED_LENGTHS(QHK_C2C)
#undef QHK_C2C
    default: break;
  }
  switch (rows_per_cta(nx)) {
    case 16: c2c_rows_dispatch<16, 0>(data, rows, nx, forward, mode, scale, index, nm2, inv_k02, s); break;
    case 8: c2c_rows_dispatch<8, 0>(data, rows, nx, forward, mode, scale, index, nm2, inv_k02, s); break;
    case 4: c2c_rows_dispatch<4, 0>(data, rows, nx, forward, mode, scale, index, nm2, inv_k02, s); break;
    case 2: c2c_rows_dispatch<2, 0>(data, rows, nx, forward, mode, scale, index, nm2, inv_k02, s); break;
    default: c2c_rows_dispatch<1, 0>(data, rows, nx, forward, mode, scale, index, nm2, inv_k02, s); break;
  }
}

#undef QHK_FIXED_LENGTHS

void fft2d(float2* data, int count, int n, bool forward, float scale, cudaStream_t s) {
  rows_c2c(data, static_cast<std::size_t>(count) * n, n, forward, RowMode::plain, 1.0f, nullptr, 0, 0, s);
  axis_pass(data, count, static_cast<std::size_t>(n) * n, n, static_cast<std::size_t>(n), n, forward,
            AxisMode::plain, scale, AxisAux{}, s);
}

}  // namespace qhk
