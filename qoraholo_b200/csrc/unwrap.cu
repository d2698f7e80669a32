// Least-squares phase unwrapping (Ghiglia & Romero 1994) and Rytov assembly on the device.
// Replaces the reference's Unwrapper (src/cuda/unwrap.cu, src/cuda/stages.cuh:57-80) and follows
// cpu::unwrap / cpu::rytov (src/cpu/unwrap.cpp:11-82, DCT by Makhoul, src/cpu/fft.cpp:101-133).
//
// Three passes over a stack of images, each a batched launch over all images:
//   1. rows: divergence of the wrapped differences (the Neumann Poisson right-hand side, with
//      the host's float operations, so bit-identical) and its DCT-II along x;
//   2. columns: DCT-II along y, division by the eigenvalue of the 5-point Neumann Laplacian,
//      inverse DCT along y -- the whole spectral solve in one launch;
//   3. rows: inverse DCT along x, and per-CTA partial sums of exp(i (psi - phi)) in double.
// A small per-image kernel then reduces the partial sums in a fixed order (no atomics) to the
// congruence constant and forms the border mean, in the host's summation order, for the 2 pi
// shift of the Rytov phase.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <map>
#include <numbers>
#include <vector>

#include "debug.cuh"
#include "fft_reg.cuh"
#include "nvtx.hpp"
#include "unwrap.hpp"

namespace qhk {

namespace {

constexpr int kThreads = 256;

template <class K>
void allow(K kernel, std::size_t) {
  ensure_smem(kernel);
}

// Each pass is written as the work of one tile (a CTA's share) of one image, so that the stacked
// launches below (grid = tiles x images of one size) and the uneven-batch launches (persistent
// CTAs draining an (image, tile) queue) run the same code. `psi`, `d1`, `phi` point at the image.

// Pass 1: COLS rows y0 .. y0 + COLS - 1 of one image.
template <int COLS>
__device__ __forceinline__ void div_dctx_tile(const float* __restrict__ psi, float* __restrict__ d1, int ny, int nx,
                                              const FftLen& L, const float2* __restrict__ dtw, int y0, float2* sm) {
  constexpr int cp = COLS + 1;
  float2* A = sm;
  float2* B = A + static_cast<std::size_t>(nx) * cp;
  float* P = reinterpret_cast<float*>(B + static_cast<std::size_t>(nx) * cp);  // rows y0-1 .. y0+COLS
  constexpr std::size_t img = 0;
  const int tid = static_cast<int>(threadIdx.x), nth = static_cast<int>(blockDim.x);
  for (int idx = tid; idx < (COLS + 2) * nx; idx += nth) {
    const int rr = idx / nx;
    const int x = idx - rr * nx;
    const int y = y0 - 1 + rr;
    P[idx] = (y >= 0 && y < ny) ? psi[img + static_cast<std::size_t>(y) * nx + x] : 0.0f;
  }
  __syncthreads();
  for (int idx = tid; idx < COLS * nx; idx += nth) {
    const int row = idx / nx;
    const int x = idx - row * nx;
    const int y = y0 + row;
    float r = 0.0f;
    if (y < ny) {
      const float* c = P + static_cast<std::size_t>(row + 1) * nx;
      const float p = c[x];
      if (x + 1 < nx) r = __fadd_rn(r, wrap_phase(__fsub_rn(c[x + 1], p)));
      if (x > 0) r = __fsub_rn(r, wrap_phase(__fsub_rn(p, c[x - 1])));
      if (y + 1 < ny) r = __fadd_rn(r, wrap_phase(__fsub_rn(c[x + nx], p)));
      if (y > 0) r = __fsub_rn(r, wrap_phase(__fsub_rn(p, c[x - nx])));
    }
    A[dct_position(x, nx) * cp + row] = make_float2(r, 0.0f);
  }
  __syncthreads();
  const float2* res = smem_fft_cols<true, COLS>(A, B, cp, L, tid, nth);
  for (int idx = tid; idx < COLS * nx; idx += nth) {
    const int row = idx / nx;
    const int k = idx - row * nx;
    if (y0 + row >= ny) continue;
    const float2 v = res[k * cp + row];
    const float2 w = __ldg(dtw + k);
    d1[img + static_cast<std::size_t>(y0 + row) * nx + k] = w.x * v.x - w.y * v.y;
  }
}

template <int COLS>
__global__ void __launch_bounds__(kThreads)
    k_div_dctx(const float* __restrict__ psi, float* __restrict__ d1, int ny, int nx, FftLen L,
               const float2* __restrict__ dtw) {
  extern __shared__ __align__(16) float2 sm[];
  const std::size_t img = static_cast<std::size_t>(blockIdx.y) * ny * nx;
  div_dctx_tile<COLS>(psi + img, d1 + img, ny, nx, L, dtw, static_cast<int>(blockIdx.x) * COLS, sm);
}

// Pass 2: COLS columns c0 .. c0 + COLS - 1 of one image: DCT-II along y, divide, inverse DCT
// along y.
template <int COLS>
__device__ __forceinline__ void dcty_solve_tile(const float* __restrict__ d1, float* __restrict__ d2, int ny, int nx,
                                                const FftLen& L, const float2* __restrict__ dtw,
                                                const float* __restrict__ cos_y, const float* __restrict__ cos_x,
                                                int c0, float2* sm) {
  float2* A = sm;
  float2* B = A + static_cast<std::size_t>(ny) * COLS;
  float* Cf = reinterpret_cast<float*>(B + static_cast<std::size_t>(ny) * COLS);
  const int cols = min(COLS, nx - c0);
  constexpr std::size_t img = 0;
  const int tid = static_cast<int>(threadIdx.x), nth = static_cast<int>(blockDim.x);
  for (int idx = tid; idx < ny * COLS; idx += nth) {
    const int y = idx / COLS;
    const int col = idx - y * COLS;
    const float v = col < cols ? d1[img + static_cast<std::size_t>(y) * nx + c0 + col] : 0.0f;
    A[dct_position(y, ny) * COLS + col] = make_float2(v, 0.0f);
  }
  __syncthreads();
  float2* res = smem_fft_cols<true, COLS>(A, B, COLS, L, tid, nth);
  float2* other = res == A ? B : A;
  for (int idx = tid; idx < ny * COLS; idx += nth) {
    const int k = idx / COLS;
    const int col = idx - k * COLS;
    const int kx = c0 + col;
    const float2 v = res[idx];
    const float2 w = __ldg(dtw + k);
    const float c = w.x * v.x - w.y * v.y;
    float out = 0.0f;
    if (col < cols && !(k == 0 && kx == 0)) {
      const float ev = __fsub_rn(__fadd_rn(__ldg(cos_y + k), __ldg(cos_x + kx)), 4.0f);
      out = __fdiv_rn(c, ev);
    }
    Cf[idx] = out;
  }
  __syncthreads();
  for (int idx = tid; idx < ny * COLS; idx += nth) {
    const int k = idx / COLS;
    const int col = idx - k * COLS;
    const float a = Cf[idx];
    const float mirror = k == 0 ? 0.0f : Cf[(ny - k) * COLS + col];
    const float2 w = __ldg(dtw + k);  // e^{-i pi k / 2n}; the inverse uses its conjugate
    other[idx] = cmulc(make_float2(a, -mirror), w);
  }
  __syncthreads();
  const float2* out = smem_fft_cols<false, COLS>(other, res, COLS, L, tid, nth);
  const float inv = 1.0f / static_cast<float>(ny);
  for (int idx = tid; idx < ny * COLS; idx += nth) {
    const int y = idx / COLS;
    const int col = idx - y * COLS;
    if (col >= cols) continue;
    d2[img + static_cast<std::size_t>(y) * nx + c0 + col] = out[dct_position(y, ny) * COLS + col].x * inv;
  }
}

template <int COLS>
__global__ void __launch_bounds__(kThreads)
    k_dcty_solve(const float* __restrict__ d1, float* __restrict__ d2, int ny, int nx, FftLen L,
                 const float2* __restrict__ dtw, const float* __restrict__ cos_y, const float* __restrict__ cos_x) {
  extern __shared__ __align__(16) float2 sm[];
  const std::size_t img = static_cast<std::size_t>(blockIdx.y) * ny * nx;
  dcty_solve_tile<COLS>(d1 + img, d2 + img, ny, nx, L, dtw, cos_y, cos_x, static_cast<int>(blockIdx.x) * COLS, sm);
}

// Pass 3: inverse DCT along x of COLS rows y0 .. y0 + COLS - 1 (in place), and the congruence
// partial sums over those rows: pair[0] = sum cos(psi - phi), pair[1] = sum sin(psi - phi).
// `red` is the CTA's shared reduction buffer of 2 x kThreads doubles.
template <int COLS>
__device__ __forceinline__ void idctx_tile(float* __restrict__ phi, const float* __restrict__ psi, int ny, int nx,
                                           const FftLen& L, const float2* __restrict__ dtw, int y0,
                                           double* __restrict__ pair, float2* sm, double (*red)[kThreads]) {
  constexpr int cp = COLS + 1;
  float2* A = sm;
  float2* B = A + static_cast<std::size_t>(nx) * cp;
  float* F = reinterpret_cast<float*>(B + static_cast<std::size_t>(nx) * cp);
  constexpr std::size_t img = 0;
  const int tid = static_cast<int>(threadIdx.x), nth = static_cast<int>(blockDim.x);
  for (int idx = tid; idx < COLS * nx; idx += nth) {
    const int row = idx / nx;
    const int k = idx - row * nx;
    F[idx] = y0 + row < ny ? phi[img + static_cast<std::size_t>(y0 + row) * nx + k] : 0.0f;
  }
  __syncthreads();
  for (int idx = tid; idx < COLS * nx; idx += nth) {
    const int row = idx / nx;
    const int k = idx - row * nx;
    const float a = F[idx];
    const float mirror = k == 0 ? 0.0f : F[row * nx + nx - k];
    A[k * cp + row] = cmulc(make_float2(a, -mirror), __ldg(dtw + k));
  }
  __syncthreads();
  const float2* res = smem_fft_cols<false, COLS>(A, B, cp, L, tid, nth);
  const float inv = 1.0f / static_cast<float>(nx);
  double sc = 0.0, ss = 0.0;
  for (int idx = tid; idx < COLS * nx; idx += nth) {
    const int row = idx / nx;
    const int x = idx - row * nx;
    if (y0 + row >= ny) continue;
    const std::size_t g = img + static_cast<std::size_t>(y0 + row) * nx + x;
    const float v = res[dct_position(x, nx) * cp + row].x * inv;
    phi[g] = v;
    double s, c;
    sincos(static_cast<double>(__fsub_rn(psi[g], v)), &s, &c);
    sc += c;
    ss += s;
  }
  red[0][tid] = sc;
  red[1][tid] = ss;
  __syncthreads();
  for (int h = nth / 2; h > 0; h >>= 1) {
    if (tid < h) {
      red[0][tid] += red[0][tid + h];
      red[1][tid] += red[1][tid + h];
    }
    __syncthreads();
  }
  if (tid == 0) {
    pair[0] = red[0][0];
    pair[1] = red[1][0];
  }
}

// Stacked form: partial[(image * gridDim.x + blockIdx.x) * 2 + {0, 1}].
template <int COLS>
__global__ void __launch_bounds__(kThreads)
    k_idctx(float* __restrict__ phi, const float* __restrict__ psi, int ny, int nx, FftLen L,
            const float2* __restrict__ dtw, double* __restrict__ partial) {
  extern __shared__ __align__(16) float2 sm[];
  __shared__ double red[2][kThreads];
  const std::size_t img = static_cast<std::size_t>(blockIdx.y) * ny * nx;
  idctx_tile<COLS>(phi + img, psi + img, ny, nx, L, dtw, static_cast<int>(blockIdx.x) * COLS,
                   partial + (static_cast<std::size_t>(blockIdx.y) * gridDim.x + blockIdx.x) * 2, sm, red);
}

// ---- The same three passes on the register-resident engine (fft_reg.cuh), lines of n = 128, 256, 384, 512.
// The DCT-II of a line of n reals (Makhoul: v[p] = r[x(p)], X[k] = Re(e^{-i pi k / 2n} V[k]), V = FFT_n(v)) runs
// as a complex FFT of half length h = n / 2 of z[m] = v[2m] + i v[2m + 1], then the split
//   V[k] = (Z[k] + conj Z[h-k]) / 2 + W_n^k (Z[k] - conj Z[h-k]) / 2i, k = 0..h, with V[n-k] = conj V[k],
// so X[k] = Re(w_k V[k]) and X[n-k] = -Im(w_k V[k]) (w_k = e^{-i pi k / 2n}). The inverse DCT takes the
// Hermitian A[k] = (a[k] - i a[n-k]) conj(w_k) (a[n] = 0) through the half-length inverse FFT of
//   B[k] = A[k] + conj A[h-k] + i (A[k] - conj A[h-k]) e^{2 pi i k / n},
// whose outputs z[m] are the real samples 2m (real part) and 2m + 1 (imaginary part). T threads per line
// hold V = h / T values; W_n^k comes from the length-n table, whose even entries are the half length's.

// Position in the line of the Makhoul-reordered sample p (the inverse of dct_position).
__device__ __forceinline__ int makhoul_x(int p, int n) { return p < n / 2 ? 2 * p : 2 * (n - 1 - p) + 1; }

// X[k] and X[n - k] of the DCT-II from the half-length spectrum Z in natural order (zs[m * zp], m < h).
__device__ __forceinline__ void dct_pair(const float2* zs, int zp, int k, int h, const float2* __restrict__ twn,
                                         const float2* __restrict__ dtw, float& xk, float& xnk) {
  const float2 zk = zs[(k == h ? 0 : k) * zp];
  const float2 zm = zs[(k == 0 ? 0 : h - k) * zp];
  const float2 ev = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
  const float2 d = make_float2(zk.x - zm.x, zk.y + zm.y);  // zk - conj(zm)
  const float2 od = make_float2(0.5f * d.y, -0.5f * d.x);   // d / 2i
  const float2 vk = cadd(ev, cmul(__ldg(twn + k), od));
  const float2 w = __ldg(dtw + k);
  xk = w.x * vk.x - w.y * vk.y;
  xnk = -(w.x * vk.y + w.y * vk.x);
}

// B[k] of the half-length inverse from A[k] and A[h - k] (A[0], A[h] real).
__device__ __forceinline__ float2 idct_merge(float2 ak, float2 am, int k, const float2* __restrict__ twn) {
  if (k == 0) {
    ak.y = 0.0f;
    am.y = 0.0f;
  }
  const float2 sv = make_float2(ak.x + am.x, ak.y - am.y);  // ak + conj(am)
  const float2 d = make_float2(ak.x - am.x, ak.y + am.y);   // ak - conj(am)
  const float2 tt = cmulc(d, __ldg(twn + k));                // d e^{2 pi i k / n}
  return make_float2(sv.x - tt.y, sv.y + tt.x);              // sv + i tt
}

// Row pitch (float2) of the natural-order staging of a pass-1 row tile: T V + 8, or T V + 4 for T = 4, so
// that a warp's rows (4 of 8 threads, 2 of 16, 8 of 4) fall on distinct two-bank slots.
template <int T, int V>
__host__ __device__ constexpr int reg_row_pitch() {
  return T * V + (T == 4 ? 4 : 8);
}

// Shared memory of the register row tiles (passes 1 and 3): first an area of float2 for the transform's
// exchange, the natural-order spectrum and (pass 1) the divergence tile, rounded to 16 bytes; then a row
// buffer of (R + 2) n floats for the tile's input rows and its output rows. Pass 2's column tiles use
// one area for the exchange and the spectrum.
template <int T, int V>
__host__ __device__ constexpr std::size_t reg_rows_area() {
  using Tile = regfft::RowTile<T>;
  const std::size_t xs = static_cast<std::size_t>(V) * Tile::A,
                    zs = static_cast<std::size_t>(Tile::R) * reg_row_pitch<T, V>(),
                    dv = (static_cast<std::size_t>(Tile::R) * (2 * T * V + 1) + 1) / 2;
  const std::size_t m = xs > zs ? (xs > dv ? xs : dv) : (zs > dv ? zs : dv);
  return (m + 1) / 2 * 2;
}
// Floats of the row buffer: pass 1's input rows y0 - 1 .. y0 + R (pitch n) and either pass's output rows
// (pitch at most n + 2 T).
template <int T, int V>
__host__ __device__ constexpr std::size_t reg_rows_buf() {
  constexpr std::size_t R = regfft::RowTile<T>::R, n = 2 * T * V;
  return R * n + (2 * n > 2 * R * T ? 2 * n : 2 * R * T);
}
template <int T, int V>
__host__ __device__ constexpr std::size_t reg_rows_smem() {
  return reg_rows_area<T, V>() * sizeof(float2) + reg_rows_buf<T, V>() * sizeof(float);
}
template <int T, int V>
__host__ __device__ constexpr std::size_t reg_cols_smem() {
  return static_cast<std::size_t>(T * V + 1) * (kThreads / T) * sizeof(float2);
}

// Four consecutive floats of global memory: one 16-byte access when `vec` (the address 16-byte aligned),
// else four 4-byte ones -- the images of an uneven batch are packed densely, so their rows need not be
// aligned. ldg4 reads through the read-only cache (data the kernel does not write).
__device__ __forceinline__ bool aligned16(const void* p) { return (reinterpret_cast<std::uintptr_t>(p) & 15u) == 0; }
__device__ __forceinline__ float4 ld4(const float* p, bool vec) {
  return vec ? *reinterpret_cast<const float4*>(p) : make_float4(p[0], p[1], p[2], p[3]);
}
__device__ __forceinline__ float4 ldg4(const float* p, bool vec) {
  return vec ? __ldg(reinterpret_cast<const float4*>(p)) : make_float4(__ldg(p), __ldg(p + 1), __ldg(p + 2), __ldg(p + 3));
}
__device__ __forceinline__ void st4(float* p, float4 v, bool vec) {
  if (vec) {
    *reinterpret_cast<float4*>(p) = v;
  } else {
    p[0] = v.x, p[1] = v.y, p[2] = v.z, p[3] = v.w;
  }
}

// Pass 1: rows y0 .. y0 + R - 1 (R = 256 / T) of one image of width n = 2 T V. The rows y0 - 1 .. y0 + R
// of psi come in coalesced; the divergence of the wrapped differences is formed in natural order in shared
// memory and read by the transform in the half-length DCT's order; the DCT rows leave coalesced.
template <int T, int V>
__device__ __forceinline__ void div_dctx_tile_reg(const float* __restrict__ psi, float* __restrict__ d1, int ny,
                                                  const float2* __restrict__ twn, const float2* __restrict__ dtw,
                                                  int y0, float2* sm) {
  if (!QHK_CHECK(reg_rows_smem<T, V>() <= debug::dynamic_smem_bytes() && y0 >= 0 && y0 < ny)) return;
  using Tile = regfft::RowTile<T>;
  constexpr int h = T * V, n = 2 * h, R = Tile::R, P = reg_row_pitch<T, V>();
  constexpr int Q = n / 4;   // float4 per row
  constexpr int DP = n + 1;  // divergence row pitch: the strided reads below spread over the banks
  constexpr int OP = n + T;  // output row pitch: a warp's rows start on distinct banks
  static_assert(static_cast<std::size_t>(R) * OP <= reg_rows_buf<T, V>(), "output rows");
  const int tid = static_cast<int>(threadIdx.x);
  const int t = tid % T, r = tid / T;
  float* rows = reinterpret_cast<float*>(sm + reg_rows_area<T, V>());
  float* dv = reinterpret_cast<float*>(sm);
  const bool vec = aligned16(psi) && aligned16(d1);  // n is a multiple of 4: every row alike
  for (int i = tid; i < (R + 2) * Q; i += kThreads) {  // rows outside the image are never read
    const int rr = i / Q, yy = y0 - 1 + rr;
    if (yy >= 0 && yy < ny) {
      reinterpret_cast<float4*>(rows)[i] = ldg4(psi + static_cast<std::size_t>(yy) * n + 4 * (i - rr * Q), vec);
    }
  }
  __syncthreads();
  for (int i = tid; i < R * n; i += kThreads) {
    const int rr = i / n, x = i - rr * n, y = y0 + rr;
    const float* c = rows + (rr + 1) * n;
    float acc = 0.0f;
    if (y < ny) {
      const float p = c[x];
      if (x + 1 < n) acc = __fadd_rn(acc, wrap_phase(__fsub_rn(c[x + 1], p)));
      if (x > 0) acc = __fsub_rn(acc, wrap_phase(__fsub_rn(p, c[x - 1])));
      if (y + 1 < ny) acc = __fadd_rn(acc, wrap_phase(__fsub_rn(c[x + n], p)));
      if (y > 0) acc = __fsub_rn(acc, wrap_phase(__fsub_rn(p, c[x - n])));
    }
    dv[rr * DP + x] = acc;
  }
  __syncthreads();
  float2 v[V];
#pragma unroll
  for (int j = 0; j < V; ++j) {
    const int m = t + T * j;
    v[j] = make_float2(dv[r * DP + makhoul_x(2 * m, n)], dv[r * DP + makhoul_x(2 * m + 1, n)]);
  }
  __syncthreads();  // the exchange overwrites the divergence tile
  regfft::line_fft<T, V, true>(v, t, sm + r, Tile::A, Tile::B, twn, 2);
  __syncthreads();
  float2* zs = sm + r * P;
#pragma unroll
  for (int j = 0; j < V; ++j) zs[t + T * j] = v[j];
  __syncthreads();
  float* out = rows + r * OP;
#pragma unroll
  for (int j = 0; j <= V; ++j) {
    if (j == V && t != 0) break;
    const int k = j < V ? t + T * j : h;
    float xk, xnk;
    dct_pair(zs, 1, k, h, twn, dtw, xk, xnk);
    out[k] = xk;
    if (k > 0 && k < h) out[n - k] = xnk;
  }
  __syncthreads();
  for (int i = tid; i < R * Q; i += kThreads) {
    const int rr = i / Q, yy = y0 + rr;
    if (yy < ny) {
      st4(d1 + static_cast<std::size_t>(yy) * n + 4 * (i - rr * Q),
          reinterpret_cast<const float4*>(rows + rr * OP)[i - rr * Q], vec);
    }
  }
}

// Pass 2: columns c0 .. c0 + COLS - 1 (COLS = 256 / T) of one image of height n = 2 T V: DCT-II along y,
// divide by the Neumann eigenvalue, inverse DCT along y.
template <int T, int V>
__device__ __forceinline__ void dcty_solve_tile_reg(const float* __restrict__ d1, float* __restrict__ d2, int nx,
                                                    const float2* __restrict__ twn, const float2* __restrict__ dtw,
                                                    const float* __restrict__ cos_y, const float* __restrict__ cos_x,
                                                    int c0, float2* sm) {
  if (!QHK_CHECK(reg_cols_smem<T, V>() <= debug::dynamic_smem_bytes() && c0 >= 0 && c0 < nx)) return;
  constexpr int h = T * V, n = 2 * h, COLS = kThreads / T;
  const int c = static_cast<int>(threadIdx.x) % COLS, t = static_cast<int>(threadIdx.x) / COLS;
  const int col = c0 + c;
  const bool live = col < nx;
  const float* in = d1 + (live ? col : 0);
  float2 v[V];
#pragma unroll
  for (int j = 0; j < V; ++j) {
    const int m = t + T * j;
    v[j] = live ? make_float2(in[static_cast<std::size_t>(makhoul_x(2 * m, n)) * nx],
                              in[static_cast<std::size_t>(makhoul_x(2 * m + 1, n)) * nx])
                : make_float2(0.0f, 0.0f);
  }
  regfft::line_fft<T, V, true>(v, t, sm + c, T * COLS, COLS, twn, 2);
  __syncthreads();
#pragma unroll
  for (int j = 0; j < V; ++j) sm[(t + T * j) * COLS + c] = v[j];  // Z, natural order
  __syncthreads();
  // a = X / eigenvalue at k and n - k, then A[k] for the thread's bins k = t + T j (and k = h for t = 0).
  float2 av[V + 1];
#pragma unroll
  for (int j = 0; j <= V; ++j) {
    const int k = j < V ? t + T * j : h;
    float xk = 0.0f, xnk = 0.0f;
    if (j < V || t == 0) dct_pair(sm + c, COLS, k, h, twn, dtw, xk, xnk);
    const float ex = __ldg(cos_x + (live ? col : 0));
    float ak = 0.0f, ank = 0.0f;
    if (live && !(k == 0 && col == 0)) ak = __fdiv_rn(xk, __fsub_rn(__fadd_rn(__ldg(cos_y + k), ex), 4.0f));
    if (live && k > 0 && k < h) ank = __fdiv_rn(xnk, __fsub_rn(__fadd_rn(__ldg(cos_y + n - k), ex), 4.0f));
    if (k == h) ank = ak;  // a[n - h] = a[h]
    av[j] = cmulc(make_float2(ak, k == 0 ? 0.0f : -ank), __ldg(dtw + k));
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j <= V; ++j) {
    if (j < V || t == 0) sm[(j < V ? t + T * j : h) * COLS + c] = av[j];  // A[k], k = 0..h
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < V; ++j) {
    const int k = t + T * j;
    v[j] = idct_merge(sm[k * COLS + c], sm[(h - k) * COLS + c], k, twn);
  }
  __syncthreads();  // the exchange of the inverse reuses the buffer
  regfft::line_fft<T, V, false>(v, t, sm + c, T * COLS, COLS, twn, 2);
  if (!live) return;
  const float inv = 1.0f / static_cast<float>(n);
  float* out = d2 + col;
#pragma unroll
  for (int j = 0; j < V; ++j) {
    const int m = t + T * j;
    out[static_cast<std::size_t>(makhoul_x(2 * m, n)) * nx] = v[j].x * inv;
    out[static_cast<std::size_t>(makhoul_x(2 * m + 1, n)) * nx] = v[j].y * inv;
  }
}

// Pass 3: inverse DCT along x of rows y0 .. y0 + R - 1 (in place) and the congruence partial sums of the
// tile, as idctx_tile. The phi rows come in and leave coalesced; the transform's output, in the
// half-length DCT's order, is staged in shared memory and read back in natural order for the store and
// for the congruence sums against psi.
template <int T, int V>
__device__ __forceinline__ void idctx_tile_reg(float* __restrict__ phi, const float* __restrict__ psi, int ny,
                                               const float2* __restrict__ twn, const float2* __restrict__ dtw, int y0,
                                               double* __restrict__ pair, float2* sm, double (*red)[kThreads]) {
  if (!QHK_CHECK(reg_rows_smem<T, V>() <= debug::dynamic_smem_bytes() && y0 >= 0 && y0 < ny)) return;
  using Tile = regfft::RowTile<T>;
  constexpr int h = T * V, n = 2 * h, R = Tile::R, Q = n / 4;
  constexpr int IP = n + T;      // input row pitch: a warp's rows start on distinct banks
  constexpr int OQ = n + 2 * T;  // staged output row pitch (float2 pitch h + T: conflict-free pair stores)
  static_assert(static_cast<std::size_t>(R) * OQ <= reg_rows_buf<T, V>(), "output rows");
  const int tid = static_cast<int>(threadIdx.x), nth = static_cast<int>(blockDim.x);
  const int t = tid % T, r = tid / T;
  float* rows = reinterpret_cast<float*>(sm + reg_rows_area<T, V>());
  const bool vec = aligned16(phi) && aligned16(psi);  // n is a multiple of 4: every row alike
  for (int i = tid; i < R * Q; i += kThreads) {
    const int rr = i / Q, yy = y0 + rr;
    const float4 a = yy < ny ? ld4(phi + static_cast<std::size_t>(yy) * n + 4 * (i - rr * Q), vec)
                             : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    reinterpret_cast<float4*>(rows + rr * IP)[i - rr * Q] = a;
  }
  __syncthreads();
  const float* row = rows + r * IP;
  const auto avalue = [&](int k) {  // A[k] = (a[k] - i a[n-k]) conj(w_k), a[n] = 0
    return cmulc(make_float2(row[k], k == 0 ? 0.0f : -row[n - k]), __ldg(dtw + k));
  };
  float2 v[V];
#pragma unroll
  for (int j = 0; j < V; ++j) {
    const int k = t + T * j;
    v[j] = idct_merge(avalue(k), avalue(h - k), k, twn);
  }
  // Every thread has read its rows before the exchange's barrier, so the row buffer is free afterwards.
  regfft::line_fft<T, V, false>(v, t, sm + r, Tile::A, Tile::B, twn, 2);
  const float inv = 1.0f / static_cast<float>(n);
  float2* q = reinterpret_cast<float2*>(rows + r * OQ);  // q[m] = values at half-length positions 2m, 2m + 1
#pragma unroll
  for (int j = 0; j < V; ++j) q[t + T * j] = make_float2(v[j].x * inv, v[j].y * inv);
  __syncthreads();
  // Natural order: x even is half-length position x / 2, x odd is n - 1 - (x - 1) / 2.
  double sc = 0.0, ss = 0.0;
  for (int i = tid; i < R * Q; i += kThreads) {
    const int rr = i / Q, yy = y0 + rr;
    if (yy >= ny) continue;
    const int x0 = 4 * (i - rr * Q);
    const float* qr = rows + rr * OQ;
    const float2 ev = *reinterpret_cast<const float2*>(qr + x0 / 2);          // x0, x0 + 2
    const float2 od = *reinterpret_cast<const float2*>(qr + n - 2 - x0 / 2);  // x0 + 3, x0 + 1
    const float4 val = make_float4(ev.x, od.y, ev.y, od.x);
    const std::size_t g = static_cast<std::size_t>(yy) * n + x0;
    st4(phi + g, val, vec);
    const float4 ps = ldg4(psi + g, vec);
    const float d[4] = {__fsub_rn(ps.x, val.x), __fsub_rn(ps.y, val.y), __fsub_rn(ps.z, val.z),
                        __fsub_rn(ps.w, val.w)};
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      double sn, cs;
      sincos(static_cast<double>(d[e]), &sn, &cs);
      sc += cs;
      ss += sn;
    }
  }
  red[0][tid] = sc;
  red[1][tid] = ss;
  __syncthreads();
  for (int hh = nth / 2; hh > 0; hh >>= 1) {
    if (tid < hh) {
      red[0][tid] += red[0][tid + hh];
      red[1][tid] += red[1][tid + hh];
    }
    __syncthreads();
  }
  if (tid == 0) {
    pair[0] = red[0][0];
    pair[1] = red[1][0];
  }
}

template <int T, int V>
__global__ void __launch_bounds__(kThreads)
    k_div_dctx_reg(const float* __restrict__ psi, float* __restrict__ d1, int ny, const float2* __restrict__ twn,
                   const float2* __restrict__ dtw) {
  extern __shared__ __align__(16) float2 sm[];
  const std::size_t img = static_cast<std::size_t>(blockIdx.y) * ny * (2 * T * V);
  div_dctx_tile_reg<T, V>(psi + img, d1 + img, ny, twn, dtw, static_cast<int>(blockIdx.x) * (kThreads / T), sm);
}

template <int T, int V>
__global__ void __launch_bounds__(kThreads)
    k_dcty_solve_reg(const float* __restrict__ d1, float* __restrict__ d2, int nx, const float2* __restrict__ twn,
                     const float2* __restrict__ dtw, const float* __restrict__ cos_y, const float* __restrict__ cos_x) {
  extern __shared__ __align__(16) float2 sm[];
  const std::size_t img = static_cast<std::size_t>(blockIdx.y) * (2 * T * V) * nx;
  dcty_solve_tile_reg<T, V>(d1 + img, d2 + img, nx, twn, dtw, cos_y, cos_x,
                            static_cast<int>(blockIdx.x) * (kThreads / T), sm);
}

template <int T, int V>
__global__ void __launch_bounds__(kThreads)
    k_idctx_reg(float* __restrict__ phi, const float* __restrict__ psi, int ny, const float2* __restrict__ twn,
                const float2* __restrict__ dtw, double* __restrict__ partial) {
  extern __shared__ __align__(16) float2 sm[];
  __shared__ double red[2][kThreads];
  const std::size_t img = static_cast<std::size_t>(blockIdx.y) * ny * (2 * T * V);
  idctx_tile_reg<T, V>(phi + img, psi + img, ny, twn, dtw, static_cast<int>(blockIdx.x) * (kThreads / T),
                       partial + (static_cast<std::size_t>(blockIdx.y) * gridDim.x + blockIdx.x) * 2, sm, red);
}

// Calls f.template operator()<T, V>() when the register engine takes lines of length n; false otherwise.
template <class F>
bool with_unwrap_line(int n, F&& f) {
  if (!fft_reg_engine_enabled()) return false;
  switch (n) {
    case 128: f.template operator()<8, 8>(); return true;
    case 192: f.template operator()<4, 24>(); return true;
    case 256: f.template operator()<8, 16>(); return true;
    case 384: f.template operator()<8, 24>(); return true;
    case 512: f.template operator()<16, 16>(); return true;
    default: return false;
  }
}

// Threads per line of the register engine for lines of length n, 0 when the staged engine runs them.
int unwrap_line_threads(int n) {
  int t = 0;
  with_unwrap_line(n, [&]<int T, int V>() { t = T; });
  return t;
}

// Rows of a pass-1 / pass-3 tile and columns of a pass-2 tile for lines of length n: the register
// engine's R = 256 / T where it runs, else the staged tiles'. Every path (planned, batched, without
// allocation) tiles alike, so that the congruence partial sums, and with them the results, agree.
int rows_per_cta(int len, std::size_t extra_per_row);

int unwrap_tile_rows(int nx) {
  const int t = unwrap_line_threads(nx);
  return t ? kThreads / t : rows_per_cta(nx, static_cast<std::size_t>(nx) * sizeof(float));
}


// Per image: congruence constant c = arg(sum exp(i (psi - phi))) from the image's nblk partial
// pairs, then the 2 pi multiple of the border mean of phi + c, summed in the host's order.
__device__ __forceinline__ void rytov_consts_image(const float* __restrict__ phi, int ny, int nx,
                                                   const double* __restrict__ partial, int nblk,
                                                   float2* __restrict__ out, float* pairs) {
  __shared__ double red[2][kThreads];
  __shared__ float cshared;
  constexpr std::size_t img = 0;
  const int tid = static_cast<int>(threadIdx.x), nth = static_cast<int>(blockDim.x);
  double sc = 0.0, ss = 0.0;
  for (int b = tid; b < nblk; b += nth) {
    sc += partial[2 * b];
    ss += partial[2 * b + 1];
  }
  red[0][tid] = sc;
  red[1][tid] = ss;
  __syncthreads();
  for (int h = nth / 2; h > 0; h >>= 1) {
    if (tid < h) {
      red[0][tid] += red[0][tid + h];
      red[1][tid] += red[1][tid + h];
    }
    __syncthreads();
  }
  if (tid == 0) cshared = static_cast<float>(atan2(red[1][0], red[0][0]));
  __syncthreads();
  const float c = cshared;
  // pairs: x = 0..nx-1 -> phase(0, x) + phase(ny-1, x); then y = 1..ny-2 -> phase(y, 0) + phase(y, nx-1)
  const int npairs = nx + ny - 2;
  for (int i = tid; i < npairs; i += nth) {
    float a, b;
    if (i < nx) {
      a = __fadd_rn(phi[img + i], c);
      b = __fadd_rn(phi[img + static_cast<std::size_t>(ny - 1) * nx + i], c);
    } else {
      const int y = i - nx + 1;
      a = __fadd_rn(phi[img + static_cast<std::size_t>(y) * nx], c);
      b = __fadd_rn(phi[img + static_cast<std::size_t>(y) * nx + nx - 1], c);
    }
    pairs[i] = __fadd_rn(a, b);
  }
  __syncthreads();
  if (tid == 0) {
    double sum = 0.0;
    for (int i = 0; i < npairs; ++i) sum = __dadd_rn(sum, static_cast<double>(pairs[i]));
    const double mean = sum / (2.0 * nx + 2.0 * (ny - 2));
    const double two_pi = 2.0 * 3.14159265358979323846;
    *out = make_float2(c, static_cast<float>(two_pi * round(mean / two_pi)));
  }
}

__global__ void __launch_bounds__(kThreads)
    k_rytov_consts(const float* __restrict__ phi, int ny, int nx, const double* __restrict__ partial, int nblk,
                   float2* __restrict__ consts) {
  extern __shared__ float pairs[];
  const std::size_t img = static_cast<std::size_t>(blockIdx.x) * ny * nx;
  rytov_consts_image(phi + img, ny, nx, partial + static_cast<std::size_t>(blockIdx.x) * nblk * 2, nblk,
                     consts + blockIdx.x, pairs);
}

// out = logamp + i ((phi + c) - shift), or phi_out = phi + c when logamp is null.
__global__ void k_rytov_assemble(const float* __restrict__ phi, const float* __restrict__ logamp,
                                 const float2* __restrict__ consts, std::size_t plane, std::size_t total,
                                 float2* __restrict__ out, float* __restrict__ phi_out) {
  for (std::size_t i = blockIdx.x * static_cast<std::size_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<std::size_t>(gridDim.x) * blockDim.x) {
    const float2 k = consts[i / plane];
    const float v = __fadd_rn(phi[i], k.x);
    if (logamp) {
      out[i] = make_float2(logamp[i], __fsub_rn(v, k.y));
    } else {
      phi_out[i] = v;
    }
  }
}

__global__ void k_split_ratio(const float2* __restrict__ ratio, std::size_t total, float* __restrict__ psi,
                              float* __restrict__ logamp) {
  for (std::size_t i = blockIdx.x * static_cast<std::size_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<std::size_t>(gridDim.x) * blockDim.x) {
    const float2 r = ratio[i];
    psi[i] = atan2f(r.y, r.x);
    logamp[i] = logf(hypotf(r.x, r.y));
  }
}

// out = sample / background; background holds one image (bplane == 0 offset) or one per image.
__global__ void k_ratio(const float2* __restrict__ sample, const float2* __restrict__ bg, std::size_t plane,
                        bool per_image, std::size_t total, float2* __restrict__ out) {
  for (std::size_t i = blockIdx.x * static_cast<std::size_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<std::size_t>(gridDim.x) * blockDim.x) {
    const float2 u = sample[i];
    const float2 v = bg[per_image ? i : i % plane];
    const float d = 1.0f / (v.x * v.x + v.y * v.y);
    out[i] = make_float2((u.x * v.x + u.y * v.y) * d, (u.y * v.x - u.x * v.y) * d);
  }
}

int rows_per_cta(int len, std::size_t extra_per_row) {
  int c = 16;
  while (c > 1 && 2 * static_cast<std::size_t>(len) * (c + 1) * sizeof(float2) + (c + 2) * extra_per_row > 64 * 1024)
    c /= 2;
  return c;
}

// 2 cos(pi k / n) of the Neumann eigenvalue (src/common.hpp:28-31): the argument in float as the
// reference forms it, its cosine evaluated in double and rounded once to float -- the correctly
// rounded value in all but vanishingly rare cases, so that host-built and device-built tables agree
// (the C library's single-precision cosine is off by an ulp for about 1 % of these arguments).
float eigen_cos2(int k, int n) {
  const float a = kPiF * static_cast<float>(k) / static_cast<float>(n);
  return 2.0f * static_cast<float>(std::cos(static_cast<double>(a)));
}

unsigned grid_for(std::size_t total) {
  return static_cast<unsigned>(std::min<std::size_t>((total + kThreads - 1) / kThreads, 148u * 32u));
}

}  // namespace

UnwrapPlan::UnwrapPlan(int count, int ny, int nx) : count_(count), ny_(ny), nx_(nx) {
  require(count >= 1 && count <= 65535 && ny >= 2 && nx >= 2 && ny % 2 == 0 && nx % 2 == 0,
          "unwrap: image sides must be even");
  const auto dct_table = [](int n) {
    std::vector<float2> w(n);
    for (int k = 0; k < n; ++k) {
      const double a = -std::numbers::pi * k / (2.0 * n);
      w[k] = make_float2(static_cast<float>(std::cos(a)), static_cast<float>(std::sin(a)));
    }
    return w;
  };
  const auto cos_table = [](int n) {
    std::vector<float> c(n);
    for (int k = 0; k < n; ++k) c[k] = eigen_cos2(k, n);
    return c;
  };
  const auto up = [](auto& buf, const auto& host) {
    buf.reset(host.size());
    check(cudaMemcpy(buf.get(), host.data(), host.size() * sizeof(host[0]), cudaMemcpyHostToDevice), "upload table");
  };
  up(dtw_y_, dct_table(ny));
  up(dtw_x_, dct_table(nx));
  up(cos_y_, cos_table(ny));
  up(cos_x_, cos_table(nx));
  rows_ = unwrap_tile_rows(nx);
  nblk_ = (ny + rows_ - 1) / rows_;
  d1_.reset(static_cast<std::size_t>(count) * ny * nx);
  partial_.reset(static_cast<std::size_t>(count) * nblk_ * 2);
  consts_.reset(count);
}

std::size_t UnwrapPlan::device_bytes() const {
  return d1_.bytes() + partial_.bytes() + consts_.bytes() + dtw_y_.bytes() + dtw_x_.bytes() + cos_y_.bytes() +
         cos_x_.bytes();
}

void UnwrapPlan::solve(const float* psi, float* phi, cudaStream_t s) {
  const int ny = ny_, nx = nx_;
  const FftLen& Lx = fft_len(nx);
  const FftLen& Ly = fft_len(ny);
  const int c = rows_;
  const bool reg_rows = with_unwrap_line(nx, [&]<int T, int V>() {
    const std::size_t smem = reg_rows_smem<T, V>();
    ensure_smem(k_div_dctx_reg<T, V>);
    k_div_dctx_reg<T, V><<<dim3(nblk_, count_), kThreads, smem, s>>>(psi, d1_.get(), ny, Lx.tw, dtw_x_.get());
    check_launch("unwrap pass 1");
  });
  if (!reg_rows) {
    const std::size_t smem = 2 * static_cast<std::size_t>(nx) * (c + 1) * sizeof(float2) + (c + 2) * nx * sizeof(float);
    const dim3 grid(nblk_, count_);
#define QHK_U1(C)                                                                                \
  case C:                                                                                        \
    allow(k_div_dctx<C>, smem);                                                                  \
    k_div_dctx<C><<<grid, kThreads, smem, s>>>(psi, d1_.get(), ny, nx, Lx, dtw_x_.get());         \
    break;
    switch (c) {
      QHK_U1(16)
      QHK_U1(8)
      QHK_U1(4)
      QHK_U1(2)
      QHK_U1(1)
    }
#undef QHK_U1
    check_launch("unwrap pass 1");
  }
  const bool reg_cols = with_unwrap_line(ny, [&]<int T, int V>() {
    const std::size_t smem = reg_cols_smem<T, V>();
    const dim3 grid((nx + kThreads / T - 1) / (kThreads / T), count_);
    ensure_smem(k_dcty_solve_reg<T, V>);
    k_dcty_solve_reg<T, V><<<grid, kThreads, smem, s>>>(d1_.get(), phi, nx, Ly.tw, dtw_y_.get(), cos_y_.get(),
                                                        cos_x_.get());
    check_launch("unwrap pass 2");
  });
  if (!reg_cols) {
    int cc = 16;
    const auto smem_of = [&](int k) {
      return 2 * static_cast<std::size_t>(ny) * k * sizeof(float2) + static_cast<std::size_t>(ny) * k * sizeof(float);
    };
    while (cc > 1 && smem_of(cc) > 80 * 1024) cc /= 2;
    const std::size_t smem = smem_of(cc);
    const dim3 grid((nx + cc - 1) / cc, count_);
#define QHK_U2(C)                                                                                                \
  case C:                                                                                                        \
    allow(k_dcty_solve<C>, smem);                                                                                \
    k_dcty_solve<C><<<grid, kThreads, smem, s>>>(d1_.get(), phi, ny, nx, Ly, dtw_y_.get(), cos_y_.get(),        \
                                                 cos_x_.get());                                                  \
    break;
    switch (cc) {
      QHK_U2(16)
      QHK_U2(8)
      QHK_U2(4)
      QHK_U2(2)
      QHK_U2(1)
    }
#undef QHK_U2
    check_launch("unwrap pass 2");
  }
  if (reg_rows) {
    with_unwrap_line(nx, [&]<int T, int V>() {
      const std::size_t smem = reg_rows_smem<T, V>();
      ensure_smem(k_idctx_reg<T, V>);
      k_idctx_reg<T, V><<<dim3(nblk_, count_), kThreads, smem, s>>>(phi, psi, ny, Lx.tw, dtw_x_.get(), partial_.get());
      check_launch("unwrap pass 3");
    });
  } else {
    const std::size_t smem = 2 * static_cast<std::size_t>(nx) * (c + 1) * sizeof(float2) + c * nx * sizeof(float);
    const dim3 grid(nblk_, count_);
#define QHK_U3(C)                                                                                    \
  case C:                                                                                            \
    allow(k_idctx<C>, smem);                                                                         \
    k_idctx<C><<<grid, kThreads, smem, s>>>(phi, psi, ny, nx, Lx, dtw_x_.get(), partial_.get());     \
    break;
    switch (c) {
      QHK_U3(16)
      QHK_U3(8)
      QHK_U3(4)
      QHK_U3(2)
      QHK_U3(1)
    }
#undef QHK_U3
    check_launch("unwrap pass 3");
  }
  const std::size_t smem = static_cast<std::size_t>(nx + ny) * sizeof(float);
  k_rytov_consts<<<count_, kThreads, smem, s>>>(phi, ny, nx, partial_.get(), nblk_, consts_.get());
  check_launch("rytov constants");
}

void UnwrapPlan::unwrap(const float* psi, float* phi, cudaStream_t s) {
  solve(psi, phi, s);
  const std::size_t total = static_cast<std::size_t>(count_) * ny_ * nx_;
  k_rytov_assemble<<<grid_for(total), kThreads, 0, s>>>(phi, nullptr, consts_.get(),
                                                        static_cast<std::size_t>(ny_) * nx_, total, nullptr, phi);
  check_launch("unwrap constant");
}

void UnwrapPlan::rytov(const float* psi, const float* logamp, float* phi_scratch, float2* out, cudaStream_t s) {
  solve(psi, phi_scratch, s);
  const std::size_t total = static_cast<std::size_t>(count_) * ny_ * nx_;
  k_rytov_assemble<<<grid_for(total), kThreads, 0, s>>>(phi_scratch, logamp, consts_.get(),
                                                        static_cast<std::size_t>(ny_) * nx_, total, out, nullptr);
  check_launch("rytov assemble");
}

// ---- Uneven batches --------------------------------------------------------------------------

namespace {

// One image of an uneven batch, as the batch kernels see it.
struct BatchImage {
  std::size_t offset;  // first pixel in the packed buffers
  int ny, nx;
  int rows;            // rows per tile of passes 1 and 3 (as UnwrapPlan for this size)
  int cols;            // columns per tile of pass 2
  int nblk;            // row tiles
  int reg_x, reg_y;    // rows (passes 1, 3) / columns (pass 2) on the register engine
  int partial;         // first congruence partial pair of this image
  FftLen Lx, Ly;
  const float2* dtw_x;
  const float2* dtw_y;
  const float* cos_x;
  const float* cos_y;
};

constexpr int kAssembleChunk = 16384;  // pixels per item of the last pass

// One pass's work queue: `n` (image, tile) items drained through `counter`, over `images` images
// packed in buffers of `total` pixels.
struct BatchQueue {
  const BatchImage* imgs;
  const int2* items;
  int n;
  int images;
  std::size_t total;
  int* counter;
};

// Debug-build checks of a queue item (CTA-uniform): the image index, the image inside the packed
// buffers, and the tile index below tiles(image). The release build compiles this to `true`.
template <class Tiles>
__device__ __forceinline__ bool item_in_bounds(const BatchQueue& Q, int2 w, Tiles tiles) {
  if (!QHK_CHECK(w.x >= 0 && w.x < Q.images)) return false;
  const BatchImage& im = Q.imgs[w.x];
  return QHK_CHECK(im.offset + static_cast<std::size_t>(im.ny) * im.nx <= Q.total && w.y >= 0 && w.y < tiles(im));
}
__device__ __forceinline__ int row_tiles(const BatchImage& im) { return im.nblk; }
__device__ __forceinline__ int col_tiles(const BatchImage& im) { return (im.nx + im.cols - 1) / im.cols; }

// Next queue item for the whole CTA (thread 0 takes it, everyone reads it).
__device__ __forceinline__ int next_item(int* counter) {
  __shared__ int item;
  if (threadIdx.x == 0) item = atomicAdd(counter, 1);
  __syncthreads();
  const int it = item;
  __syncthreads();
  return it;
}

// The register tiles by line length (the lengths of with_unwrap_line).
#define QHK_REG_SWITCH(N, CALL) \
  switch (N) {                  \
    case 128: CALL(8, 8); break;  \
    case 192: CALL(4, 24); break; \
    case 256: CALL(8, 16); break; \
    case 384: CALL(8, 24); break; \
    default: CALL(16, 16); break; \
  }

#define QHK_ROWS_SWITCH(R, CALL) \
  switch (R) {                   \
    case 16: CALL(16); break;    \
    case 8: CALL(8); break;      \
    case 4: CALL(4); break;      \
    case 2: CALL(2); break;      \
    default: CALL(1); break;     \
  }

template <bool Reg>
__global__ void __launch_bounds__(kThreads, Reg ? 2 : 1)
    k_batch_pass1(const float* __restrict__ psi, float* __restrict__ d1, const BatchQueue Q) {
  extern __shared__ __align__(16) float2 sm[];
  for (int it = next_item(Q.counter); it < Q.n; it = next_item(Q.counter)) {
    const int2 w = Q.items[it];
    if (!item_in_bounds(Q, w, row_tiles)) continue;
    const BatchImage& im = Q.imgs[w.x];
#define QHK_R1(T, V)                                                                                      \
  div_dctx_tile_reg<T, V>(psi + im.offset, d1 + im.offset, im.ny, im.Lx.tw, im.dtw_x, w.y * (kThreads / T), sm)
#define QHK_P1(C) div_dctx_tile<C>(psi + im.offset, d1 + im.offset, im.ny, im.nx, im.Lx, im.dtw_x, w.y * (C), sm)
    if constexpr (Reg) {
      QHK_REG_SWITCH(im.nx, QHK_R1)
    } else {
      QHK_ROWS_SWITCH(im.rows, QHK_P1)
    }
#undef QHK_P1
#undef QHK_R1
    __syncthreads();
  }
}

template <bool Reg>
__global__ void __launch_bounds__(kThreads, Reg ? 2 : 1)
    k_batch_pass2(const float* __restrict__ d1, float* __restrict__ phi, const BatchQueue Q) {
  extern __shared__ __align__(16) float2 sm[];
  for (int it = next_item(Q.counter); it < Q.n; it = next_item(Q.counter)) {
    const int2 w = Q.items[it];
    if (!item_in_bounds(Q, w, col_tiles)) continue;
    const BatchImage& im = Q.imgs[w.x];
#define QHK_R2(T, V)                                                                                       \
  dcty_solve_tile_reg<T, V>(d1 + im.offset, phi + im.offset, im.nx, im.Ly.tw, im.dtw_y, im.cos_y, im.cos_x, \
                            w.y * (kThreads / T), sm)
#define QHK_P2(C)                                                                                                  \
  dcty_solve_tile<C>(d1 + im.offset, phi + im.offset, im.ny, im.nx, im.Ly, im.dtw_y, im.cos_y, im.cos_x, w.y * (C), \
                     sm)
    if constexpr (Reg) {
      QHK_REG_SWITCH(im.ny, QHK_R2)
    } else {
      QHK_ROWS_SWITCH(im.cols, QHK_P2)
    }
#undef QHK_P2
#undef QHK_R2
    __syncthreads();
  }
}

template <bool Reg>
__global__ void __launch_bounds__(kThreads, Reg ? 2 : 1)
    k_batch_pass3(float* __restrict__ phi, const float* __restrict__ psi, double* __restrict__ partial,
                  const BatchQueue Q) {
  extern __shared__ __align__(16) float2 sm[];
  __shared__ double red[2][kThreads];
  for (int it = next_item(Q.counter); it < Q.n; it = next_item(Q.counter)) {
    const int2 w = Q.items[it];
    if (!item_in_bounds(Q, w, row_tiles)) continue;
    const BatchImage& im = Q.imgs[w.x];
    double* pair = partial + 2 * (static_cast<std::size_t>(im.partial) + w.y);
#define QHK_R3(T, V) \
  idctx_tile_reg<T, V>(phi + im.offset, psi + im.offset, im.ny, im.Lx.tw, im.dtw_x, w.y * (kThreads / T), pair, sm, red)
#define QHK_P3(C) \
  idctx_tile<C>(phi + im.offset, psi + im.offset, im.ny, im.nx, im.Lx, im.dtw_x, w.y * (C), pair, sm, red)
    if constexpr (Reg) {
      QHK_REG_SWITCH(im.nx, QHK_R3)
    } else {
      QHK_ROWS_SWITCH(im.rows, QHK_P3)
    }
#undef QHK_P3
#undef QHK_R3
    __syncthreads();
  }
}

__global__ void __launch_bounds__(kThreads)
    k_batch_pass4(const float* __restrict__ phi, const double* __restrict__ partial, float2* __restrict__ consts,
                  const BatchQueue Q) {
  extern __shared__ float pairs[];
  for (int it = next_item(Q.counter); it < Q.n; it = next_item(Q.counter)) {
    const int2 w = Q.items[it];
    if (!item_in_bounds(Q, w, [](const BatchImage&) { return 1; })) continue;
    const BatchImage& im = Q.imgs[w.x];
    rytov_consts_image(phi + im.offset, im.ny, im.nx, partial + 2 * static_cast<std::size_t>(im.partial), im.nblk,
                       consts + w.x, pairs);
    __syncthreads();
  }
}

__global__ void __launch_bounds__(kThreads)
    k_batch_pass5(float* __restrict__ phi, const float2* __restrict__ consts, const BatchQueue Q) {
  for (int it = next_item(Q.counter); it < Q.n; it = next_item(Q.counter)) {
    const int2 w = Q.items[it];
    const auto chunks = [](const BatchImage& im) {
      return static_cast<int>((static_cast<std::size_t>(im.ny) * im.nx + kAssembleChunk - 1) / kAssembleChunk);
    };
    if (!item_in_bounds(Q, w, chunks)) continue;
    const BatchImage& im = Q.imgs[w.x];
    const float c = consts[w.x].x;
    const std::size_t pixels = static_cast<std::size_t>(im.ny) * im.nx;
    const std::size_t a = static_cast<std::size_t>(w.y) * kAssembleChunk;
    const std::size_t b = min(pixels, a + kAssembleChunk);
    float* img = phi + im.offset;
    if (aligned16(img) && (b - a) % 4 == 0) {
      // Four points per access, four accesses in flight per thread (a chunk of an even-sided image is a
      // multiple of 4 points, starting on a multiple of 4).
      float4* v = reinterpret_cast<float4*>(img + a);
      const int n4 = static_cast<int>((b - a) / 4);
      for (int i = static_cast<int>(threadIdx.x); i < n4; i += 4 * kThreads) {
        float4 q[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          if (i + u * kThreads < n4) q[u] = v[i + u * kThreads];
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          if (i + u * kThreads < n4) {
            v[i + u * kThreads] = make_float4(__fadd_rn(q[u].x, c), __fadd_rn(q[u].y, c), __fadd_rn(q[u].z, c),
                                              __fadd_rn(q[u].w, c));
          }
        }
      }
    } else {
      for (std::size_t i = a + threadIdx.x; i < b; i += blockDim.x) img[i] = __fadd_rn(img[i], c);
    }
  }
}

#undef QHK_ROWS_SWITCH
#undef QHK_REG_SWITCH

int solve_cols(int ny) {
  int cc = 16;
  const auto smem_of = [&](int k) {
    return 2 * static_cast<std::size_t>(ny) * k * sizeof(float2) + static_cast<std::size_t>(ny) * k * sizeof(float);
  };
  while (cc > 1 && smem_of(cc) > 80 * 1024) cc /= 2;
  return cc;
}

template <class K>
unsigned persistent_grid(K kernel, std::size_t smem, int items) {
  ensure_smem(kernel);
  int per_sm = 0;
  check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kThreads, smem), "cudaOccupancy");
  const long long slots = static_cast<long long>(sm_count()) * std::max(per_sm, 1);
  return static_cast<unsigned>(std::max<long long>(1, std::min<long long>(slots, items)));
}

}  // namespace

UnwrapBatchPlan::UnwrapBatchPlan(const int* ny, const int* nx, int count) {
  require(ny && nx && count >= 1, "unwrap batch: need at least one image");
  std::vector<BatchImage> im(count);
  std::map<int, int> side;  // side length -> table index
  const auto table = [&](int n) {
    const auto it = side.find(n);
    if (it != side.end()) return it->second;
    std::vector<float2> w(n);
    std::vector<float> c(n);
    for (int k = 0; k < n; ++k) {
      const double a = -std::numbers::pi * k / (2.0 * n);
      w[k] = make_float2(static_cast<float>(std::cos(a)), static_cast<float>(std::sin(a)));
      c[k] = eigen_cos2(k, n);
    }
    dtw_.emplace_back(n);
    cos_.emplace_back(n);
    check(cudaMemcpy(dtw_.back().get(), w.data(), n * sizeof(float2), cudaMemcpyHostToDevice), "upload table");
    check(cudaMemcpy(cos_.back().get(), c.data(), n * sizeof(float), cudaMemcpyHostToDevice), "upload table");
    side[n] = static_cast<int>(dtw_.size()) - 1;
    return side[n];
  };
  int partial = 0;
  std::size_t smem[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int i = 0; i < count; ++i) {
    require(ny[i] >= 2 && nx[i] >= 2 && ny[i] % 2 == 0 && nx[i] % 2 == 0, "unwrap: image sides must be even");
    BatchImage& b = im[i];
    b.offset = total_;
    offsets_.push_back(total_);
    total_ += static_cast<std::size_t>(ny[i]) * nx[i];
    b.ny = ny[i];
    b.nx = nx[i];
    b.reg_x = unwrap_line_threads(b.nx) != 0;
    b.reg_y = unwrap_line_threads(b.ny) != 0;
    b.rows = unwrap_tile_rows(b.nx);
    b.cols = b.reg_y ? kThreads / unwrap_line_threads(b.ny) : solve_cols(b.ny);
    b.nblk = (b.ny + b.rows - 1) / b.rows;
    b.partial = partial;
    partial += b.nblk;
    b.Lx = fft_len(b.nx);
    b.Ly = fft_len(b.ny);
    const int tx = table(b.nx), ty = table(b.ny);
    b.dtw_x = dtw_[tx].get();
    b.cos_x = cos_[tx].get();
    b.dtw_y = dtw_[ty].get();
    b.cos_y = cos_[ty].get();
    const std::size_t row_buf = 2 * static_cast<std::size_t>(b.nx) * (b.rows + 1) * sizeof(float2);
    if (!with_unwrap_line(b.nx, [&]<int T, int V>() {
          smem[5] = std::max(smem[5], reg_rows_smem<T, V>());
          smem[7] = std::max(smem[7], reg_rows_smem<T, V>());
        })) {
      smem[0] = std::max(smem[0], row_buf + (b.rows + 2) * static_cast<std::size_t>(b.nx) * sizeof(float));
      smem[2] = std::max(smem[2], row_buf + b.rows * static_cast<std::size_t>(b.nx) * sizeof(float));
    }
    if (!with_unwrap_line(b.ny, [&]<int T, int V>() { smem[6] = std::max(smem[6], reg_cols_smem<T, V>()); })) {
      smem[1] = std::max(smem[1], 2 * static_cast<std::size_t>(b.ny) * b.cols * sizeof(float2) +
                                      static_cast<std::size_t>(b.ny) * b.cols * sizeof(float));
    }
    smem[3] = std::max(smem[3], static_cast<std::size_t>(b.nx + b.ny) * sizeof(float));
  }
  // Items, largest images first so that the queue ends with small tiles.
  std::vector<int> order(count);
  for (int i = 0; i < count; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
    return static_cast<std::size_t>(im[a].ny) * im[a].nx > static_cast<std::size_t>(im[b].ny) * im[b].nx;
  });
  std::vector<int2> items[8];
  for (const int i : order) {
    const BatchImage& b = im[i];
    for (int t = 0; t < b.nblk; ++t) items[b.reg_x ? 5 : 0].push_back(make_int2(i, t));
    for (int t = 0; t < (b.nx + b.cols - 1) / b.cols; ++t) items[b.reg_y ? 6 : 1].push_back(make_int2(i, t));
    items[3].push_back(make_int2(i, 0));
    const std::size_t pixels = static_cast<std::size_t>(b.ny) * b.nx;
    for (std::size_t t = 0; t * kAssembleChunk < pixels; ++t) items[4].push_back(make_int2(i, static_cast<int>(t)));
  }
  items[2] = items[0];
  items[7] = items[5];
  std::vector<int2> all;
  std::size_t at[8];
  for (int p = 0; p < 8; ++p) {
    at[p] = all.size();
    all.insert(all.end(), items[p].begin(), items[p].end());
  }
  items_.reset(all.size());
  check(cudaMemcpy(items_.get(), all.data(), all.size() * sizeof(int2), cudaMemcpyHostToDevice), "upload items");
  images_.reset(count * sizeof(BatchImage));
  check(cudaMemcpy(images_.get(), im.data(), count * sizeof(BatchImage), cudaMemcpyHostToDevice), "upload images");
  counters_.reset(8);
  d1_.reset(total_);
  partial_.reset(2 * static_cast<std::size_t>(partial));
  consts_.reset(count);
  for (int p = 0; p < 8; ++p) {
    pass_[p].items = items_.get() + at[p];
    pass_[p].n = static_cast<int>(items[p].size());
    pass_[p].smem = smem[p];
  }
  pass_[0].grid = persistent_grid(k_batch_pass1<false>, smem[0], pass_[0].n);
  pass_[1].grid = persistent_grid(k_batch_pass2<false>, smem[1], pass_[1].n);
  pass_[2].grid = persistent_grid(k_batch_pass3<false>, smem[2], pass_[2].n);
  pass_[5].grid = persistent_grid(k_batch_pass1<true>, smem[5], pass_[5].n);
  pass_[6].grid = persistent_grid(k_batch_pass2<true>, smem[6], pass_[6].n);
  pass_[7].grid = persistent_grid(k_batch_pass3<true>, smem[7], pass_[7].n);
  pass_[3].grid = persistent_grid(k_batch_pass4, smem[3], pass_[3].n);
  pass_[4].grid = persistent_grid(k_batch_pass5, 0, pass_[4].n);
}

UnwrapBatchPlan::~UnwrapBatchPlan() = default;

std::size_t UnwrapBatchPlan::device_bytes() const {
  std::size_t t = images_.bytes() + items_.bytes() + counters_.bytes() + d1_.bytes() + partial_.bytes() +
                  consts_.bytes();
  for (const auto& d : dtw_) t += d.bytes();
  for (const auto& c : cos_) t += c.bytes();
  return t;
}

void UnwrapBatchPlan::unwrap(const float* psi, float* phi, cudaStream_t s) {
  const NvtxRange r("qhk:unwrap_batch");
  const auto* imgs = reinterpret_cast<const BatchImage*>(images_.get());
  int* q = counters_.get();
  const auto queue = [&](int p) {
    return BatchQueue{imgs, static_cast<const int2*>(pass_[p].items), pass_[p].n, count(), total_, q + p};
  };
  check(cudaMemsetAsync(q, 0, 8 * sizeof(int), s), "cudaMemset");
  // Each of passes 1-3 runs as up to two persistent launches: the images whose lines the register engine
  // takes (pass_[5 + p]) and the others (pass_[p]).
  for (const bool reg : {false, true}) {
    const int p = reg ? 5 : 0;
    if (pass_[p].n == 0) continue;
    if (reg) {
      k_batch_pass1<true><<<pass_[p].grid, kThreads, pass_[p].smem, s>>>(psi, d1_.get(), queue(p));
    } else {
      k_batch_pass1<false><<<pass_[p].grid, kThreads, pass_[p].smem, s>>>(psi, d1_.get(), queue(p));
    }
    check_launch("unwrap batch pass 1");
  }
  for (const bool reg : {false, true}) {
    const int p = reg ? 6 : 1;
    if (pass_[p].n == 0) continue;
    if (reg) {
      k_batch_pass2<true><<<pass_[p].grid, kThreads, pass_[p].smem, s>>>(d1_.get(), phi, queue(p));
    } else {
      k_batch_pass2<false><<<pass_[p].grid, kThreads, pass_[p].smem, s>>>(d1_.get(), phi, queue(p));
    }
    check_launch("unwrap batch pass 2");
  }
  for (const bool reg : {false, true}) {
    const int p = reg ? 7 : 2;
    if (pass_[p].n == 0) continue;
    if (reg) {
      k_batch_pass3<true><<<pass_[p].grid, kThreads, pass_[p].smem, s>>>(phi, psi, partial_.get(), queue(p));
    } else {
      k_batch_pass3<false><<<pass_[p].grid, kThreads, pass_[p].smem, s>>>(phi, psi, partial_.get(), queue(p));
    }
    check_launch("unwrap batch pass 3");
  }
  k_batch_pass4<<<pass_[3].grid, kThreads, pass_[3].smem, s>>>(phi, partial_.get(), consts_.get(), queue(3));
  check_launch("unwrap batch constants");
  k_batch_pass5<<<pass_[4].grid, kThreads, 0, s>>>(phi, consts_.get(), queue(4));
  check_launch("unwrap batch constant");
}

void UnwrapBatchPlan::unwrap_graph(const float* psi, float* phi, cudaStream_t s) {
  if (!warmed_) {  // lazy per-device setup happens here, outside any capture
    unwrap(psi, phi, s);
    warmed_ = true;
    return;
  }
  graph_.run({psi, phi}, s, [&](cudaStream_t c) { unwrap(psi, phi, c); });
}

void field_ratio(const float2* sample, const float2* bg, std::size_t plane, bool per_image, std::size_t total,
                 float2* out, cudaStream_t s) {
  k_ratio<<<grid_for(total), kThreads, 0, s>>>(sample, bg, plane, per_image, total, out);
  check_launch("field ratio");
}

void split_ratio(const float2* ratio, std::size_t total, float* psi, float* logamp, cudaStream_t s) {
  k_split_ratio<<<grid_for(total), kThreads, 0, s>>>(ratio, total, psi, logamp);
  check_launch("split ratio");
}

}  // namespace qhk

// ---- Unwrap with no allocation -----------------------------------------------------------------
// The least-squares unwrap above, for callers that cannot allocate device memory: all scratch (the
// DCT intermediate, the congruence partial sums, the per-image constants and every twiddle /
// eigenvalue table, including the FFT twiddles that the planned path keeps in a cudaMalloc'd cache)
// lives in one file-scope device array, sized for at most kNoAllocPixels pixels per call.

namespace qhk {

namespace {

constexpr std::size_t kNoAllocPixels = std::size_t(1) << 22;  // count * ny * nx, 16 MiB of float
constexpr int kNoAllocMaxSide = 1024;                           // ny, nx
constexpr int kNoAllocMaxImages = 4096;                         // count
constexpr std::size_t kNoAllocPartials = std::size_t(1) << 16;  // (image, row block) pairs
// Layout in floats; every region starts on a 256-byte boundary.
constexpr std::size_t kOffD1 = 0;
constexpr std::size_t kOffPartial = kOffD1 + kNoAllocPixels;                   // 2 doubles per pair
constexpr std::size_t kOffConsts = kOffPartial + 4 * kNoAllocPartials;         // float2 per image
constexpr std::size_t kOffTables = kOffConsts + 2 * kNoAllocMaxImages;
constexpr std::size_t kTableFloats = 4 * 2 * kNoAllocMaxSide + 2 * kNoAllocMaxSide;  // 4 float2 + 2 float tables
constexpr std::size_t kNoAllocFloats = kOffTables + kTableFloats;

}  // namespace

// File-scope scratch of unwrap_noalloc, about 17.8 MB on every device that loads the library.
static __device__ __align__(256) float g_unwrap_scratch[kNoAllocFloats];

namespace {

// The current device's address of g_unwrap_scratch. In host code the array's name is only a
// host-side stand-in, so kernels get this address instead. It is looked up on every call (a cheap
// query that allocates nothing) rather than cached, so that a device or primary-context reset
// cannot leave a stale address behind. The first lookup on a device is the one that may load this
// file's module there (lazy module loading) and with it reserve the array.
float* scratch_base() {
  void* p = nullptr;
  check(cudaGetSymbolAddress(&p, g_unwrap_scratch), "cudaGetSymbolAddress");
  return static_cast<float*>(p);
}

// DCT twiddles e^{-i pi k / 2n}, 2 cos(pi k / n) and FFT twiddles e^{-2 pi i k / n} for one side.
__global__ void k_side_tables(int n, float2* dtw, float* cos2, float2* fftw) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    double s, c;
    sincos(-3.141592653589793238462643 * k / (2.0 * n), &s, &c);
    dtw[k] = make_float2(static_cast<float>(c), static_cast<float>(s));
    // The host tables' value (eigen_cos2): the float argument, its cosine in double, rounded once.
    cos2[k] = 2.0f * static_cast<float>(cos(static_cast<double>(kPiF * static_cast<float>(k) / static_cast<float>(n))));
    sincos(6.283185307179586476925287 * k / n, &s, &c);
    fftw[k] = make_float2(static_cast<float>(c), static_cast<float>(-s));
  }
}

}  // namespace

void unwrap_noalloc(const float* psi, float* phi, int count, int ny, int nx, cudaStream_t s) {
  require(psi && phi, "unwrap_noalloc: null argument");
  require(count >= 1 && ny >= 2 && nx >= 2 && ny % 2 == 0 && nx % 2 == 0, "unwrap: image sides must be even");
  require(ny <= kNoAllocMaxSide && nx <= kNoAllocMaxSide && count <= kNoAllocMaxImages &&
              static_cast<std::size_t>(count) * ny * nx <= kNoAllocPixels,
          "unwrap_noalloc: at most 4096 images of at most 1024 x 1024 and 4194304 pixels per call");
  const int rows = unwrap_tile_rows(nx);
  const int nblk = (ny + rows - 1) / rows;
  require(static_cast<std::size_t>(count) * nblk <= kNoAllocPartials,
          "unwrap_noalloc: too many images for the partial-sum scratch");
  float* base = scratch_base();
  float* d1 = base + kOffD1;
  auto* partial = reinterpret_cast<double*>(base + kOffPartial);
  auto* consts = reinterpret_cast<float2*>(base + kOffConsts);
  float* t = base + kOffTables;
  auto* dtw_y = reinterpret_cast<float2*>(t);
  auto* dtw_x = reinterpret_cast<float2*>(t + 2 * kNoAllocMaxSide);
  auto* fft_y = reinterpret_cast<float2*>(t + 4 * kNoAllocMaxSide);
  auto* fft_x = reinterpret_cast<float2*>(t + 6 * kNoAllocMaxSide);
  float* cos_y = t + 8 * kNoAllocMaxSide;
  float* cos_x = t + 9 * kNoAllocMaxSide;
  k_side_tables<<<4, 256, 0, s>>>(ny, dtw_y, cos_y, fft_y);
  check_launch("unwrap_noalloc tables");
  k_side_tables<<<4, 256, 0, s>>>(nx, dtw_x, cos_x, fft_x);
  check_launch("unwrap_noalloc tables");
  FftLen Ly = make_fft_len(ny);
  FftLen Lx = make_fft_len(nx);
  Ly.tw = fft_y;
  Lx.tw = fft_x;
  // The tiles and kernels of the planned path (UnwrapPlan::solve) on the static tables.
  const bool reg_rows = with_unwrap_line(nx, [&]<int T, int V>() {
    ensure_smem(k_div_dctx_reg<T, V>);
    k_div_dctx_reg<T, V><<<dim3(nblk, count), kThreads, reg_rows_smem<T, V>(), s>>>(psi, d1, ny, fft_x, dtw_x);
    check_launch("unwrap_noalloc pass 1");
  });
  if (!reg_rows) {
    const std::size_t smem = 2 * static_cast<std::size_t>(nx) * (rows + 1) * sizeof(float2) + (rows + 2) * nx * sizeof(float);
    const dim3 grid(nblk, count);
#define QHK_S1(C)                                                                   \
  case C:                                                                           \
    allow(k_div_dctx<C>, smem);                                                     \
    k_div_dctx<C><<<grid, kThreads, smem, s>>>(psi, d1, ny, nx, Lx, dtw_x);         \
    break;
    switch (rows) {
      QHK_S1(16)
      QHK_S1(8)
      QHK_S1(4)
      QHK_S1(2)
      QHK_S1(1)
    }
#undef QHK_S1
    check_launch("unwrap_noalloc pass 1");
  }
  const bool reg_cols = with_unwrap_line(ny, [&]<int T, int V>() {
    const dim3 grid((nx + kThreads / T - 1) / (kThreads / T), count);
    ensure_smem(k_dcty_solve_reg<T, V>);
    k_dcty_solve_reg<T, V><<<grid, kThreads, reg_cols_smem<T, V>(), s>>>(d1, phi, nx, fft_y, dtw_y, cos_y, cos_x);
    check_launch("unwrap_noalloc pass 2");
  });
  if (!reg_cols) {
    int cc = 16;
    const auto smem_of = [&](int k) {
      return 2 * static_cast<std::size_t>(ny) * k * sizeof(float2) + static_cast<std::size_t>(ny) * k * sizeof(float);
    };
    while (cc > 1 && smem_of(cc) > 80 * 1024) cc /= 2;
    const std::size_t smem = smem_of(cc);
    const dim3 grid((nx + cc - 1) / cc, count);
#define QHK_S2(C)                                                                                        \
  case C:                                                                                                \
    allow(k_dcty_solve<C>, smem);                                                                        \
    k_dcty_solve<C><<<grid, kThreads, smem, s>>>(d1, phi, ny, nx, Ly, dtw_y, cos_y, cos_x);            \
    break;
    switch (cc) {
      QHK_S2(16)
      QHK_S2(8)
      QHK_S2(4)
      QHK_S2(2)
      QHK_S2(1)
    }
#undef QHK_S2
    check_launch("unwrap_noalloc pass 2");
  }
  if (reg_rows) {
    with_unwrap_line(nx, [&]<int T, int V>() {
      ensure_smem(k_idctx_reg<T, V>);
      k_idctx_reg<T, V><<<dim3(nblk, count), kThreads, reg_rows_smem<T, V>(), s>>>(phi, psi, ny, fft_x, dtw_x, partial);
      check_launch("unwrap_noalloc pass 3");
    });
  } else {
    const std::size_t smem = 2 * static_cast<std::size_t>(nx) * (rows + 1) * sizeof(float2) + rows * nx * sizeof(float);
    const dim3 grid(nblk, count);
#define QHK_S3(C)                                                                              \
  case C:                                                                                      \
    allow(k_idctx<C>, smem);                                                                   \
    k_idctx<C><<<grid, kThreads, smem, s>>>(phi, psi, ny, nx, Lx, dtw_x, partial);             \
    break;
    switch (rows) {
      QHK_S3(16)
      QHK_S3(8)
      QHK_S3(4)
      QHK_S3(2)
      QHK_S3(1)
    }
#undef QHK_S3
    check_launch("unwrap_noalloc pass 3");
  }
  k_rytov_consts<<<count, kThreads, static_cast<std::size_t>(nx + ny) * sizeof(float), s>>>(phi, ny, nx, partial,
                                                                                           nblk, consts);
  check_launch("unwrap_noalloc constants");
  const std::size_t total = static_cast<std::size_t>(count) * ny * nx;
  k_rytov_assemble<<<grid_for(total), kThreads, 0, s>>>(phi, nullptr, consts, static_cast<std::size_t>(ny) * nx, total,
                                                        nullptr, phi);
  check_launch("unwrap_noalloc constant");
}

}  // namespace qhk
