// Multi-slice beam propagation (BPM) on the device: forward model, its adjoint, and the proximal
// gradient inversion. Replaces the reference's Bpm class and bpm_reconstruct (src/cuda/bpm.cu:126-349)
// and follows the CPU form (src/cpu/bpm.cpp:18-243) and the tables of src/bpm.cpp:10-60.
//
// A pass of the model processes a chunk of nb illuminations at once, all planes (nb, n, n). Each
// slice is two 2D FFTs. For n = 64, 128, 256 (the register-resident engine) a slice is two passes, each
// keeping a line of every plane on chip across a transform, the pointwise step and the opposite transform:
//   forward:  columns [FFT (completing FFT(w)), S = c (q W + (1 - q) S), IFFT] ->
//             rows [IFFT (completing IFFT(S)), x 1/n^2, store envelope, times the screen e^{i phase x_k},
//             FFT]                                                        (2 launches per slice)
//   adjoint:  rows [IFFT, x 1/n^2, gradient terms summed per pixel in view order within groups of views,
//             conj(screen) b, FFT] + the groups' sums in order -> columns [FFT, U = conj(c)(g + back),
//             g = (1 - q) U, b = q U, IFFT]                               (3 launches per slice)
// Other sides use the staged engine with the pointwise work folded into the column pass epilogues
// (4 launches per forward slice, 5 per adjoint slice: a separate gradient kernel with one thread per
// pixel summing the views in order). The gradient has a fixed summation order; the data term is summed
// in double per CTA and reduced in order.
#include <algorithm>
#include <cmath>
#include <complex>
#include <numbers>
#include <vector>

#include "bpm.hpp"
#include "fft_reg.cuh"
#include "nvtx.hpp"

namespace qhk {

namespace {

constexpr int kThreads = 256;

template <class K>
void allow(K kernel, std::size_t) {
  ensure_smem(kernel);
}

// Rows of length n, src -> dst (may alias), COLS rows per CTA.
template <bool Fwd, int COLS>
__global__ void __launch_bounds__(kThreads)
    k_rows(const float2* __restrict__ src, float2* __restrict__ dst, std::size_t rows, FftLen L) {
  extern __shared__ float2 sm[];
  constexpr int cp = COLS + 1;
  const int n = L.n;
  float2* A = sm;
  float2* B = sm + static_cast<std::size_t>(n) * cp;
  const std::size_t r0 = static_cast<std::size_t>(blockIdx.x) * COLS;
  const int nr = static_cast<int>(min(static_cast<std::size_t>(COLS), rows - r0));
  const int tid = static_cast<int>(threadIdx.x), nth = static_cast<int>(blockDim.x);
  for (int idx = tid; idx < n * COLS; idx += nth) {
    const int row = idx / n;
    const int pos = idx - row * n;
    A[pos * cp + row] = row < nr ? src[(r0 + row) * n + pos] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  const float2* res = smem_fft_cols<Fwd, COLS>(A, B, cp, L, tid, nth);
  for (int idx = tid; idx < n * COLS; idx += nth) {
    const int row = idx / n;
    const int pos = idx - row * n;
    if (row < nr) dst[(r0 + row) * n + pos] = res[pos * cp + row];
  }
}

enum ColMode : int { kScreen = 0, kPropagate = 1, kScale = 2, kSplit = 3 };

struct ColArgs {
  float2* data;         // (nb, n, n), transformed in place (kPropagate: read only)
  float2* s;            // kPropagate: spectrum S, updated; kSplit: g, updated
  float2* store;        // kScreen: envelope store of this slice (nb, n, n) or null
  const float* x;       // kScreen: contrast of this slice (n, n)
  const float2* coef;   // kPropagate / kSplit: propagator table of the chunk (nb, n, n)
  const float* q;       // obliquity weights (nb, n, n)
  float phase;          // screen phase per unit contrast
  float inv;            // 1 / n^2
  int has_back;         // kSplit: add data (the back-propagated screen term) to g
  // kSplitInv: also finish the previous slice's gradient (the first plane's blocks, one pixel per thread
  // position): grad += gscale phase (part[0] + part[1] + ...), when grad is set.
  const float* part;
  int groups;
  float gscale;
  float* grad;
};

template <bool Fwd, int Mode, int COLS>
__global__ void __launch_bounds__(kThreads) k_cols(ColArgs a, FftLen L) {
  extern __shared__ float2 sm[];
  const int n = L.n;
  float2* A = sm;
  float2* B = sm + static_cast<std::size_t>(n) * COLS;
  const int c0 = static_cast<int>(blockIdx.x) * COLS;
  const int cols = min(COLS, n - c0);
  const std::size_t base = static_cast<std::size_t>(blockIdx.y) * n * n + c0;
  const int tid = static_cast<int>(threadIdx.x), nth = static_cast<int>(blockDim.x);
  for (int idx = tid; idx < n * COLS; idx += nth) {
    const int pos = idx / COLS;
    const int col = idx - pos * COLS;
    A[idx] = col < cols ? a.data[base + static_cast<std::size_t>(pos) * n + col] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  const float2* res = smem_fft_cols<Fwd, COLS>(A, B, COLS, L, tid, nth);
  for (int idx = tid; idx < n * COLS; idx += nth) {
    const int pos = idx / COLS;
    const int col = idx - pos * COLS;
    if (col >= cols) continue;
    const std::size_t g = base + static_cast<std::size_t>(pos) * n + col;
    const float2 v = res[idx];
    if constexpr (Mode == kScreen) {
      const float2 w = cscale(v, a.inv);
      if (a.store) a.store[g] = w;
      float sn, cs;
      sincosf(a.phase * a.x[static_cast<std::size_t>(pos) * n + c0 + col], &sn, &cs);
      a.data[g] = cmul(make_float2(cs, sn), w);
    } else if constexpr (Mode == kPropagate) {
      const float2 c = a.coef[g];
      const float q = a.q[g];
      const float2 s = a.s[g];
      const float tre = q * v.x + (1.0f - q) * s.x;
      const float tim = q * v.y + (1.0f - q) * s.y;
      a.s[g] = make_float2(c.x * tre - c.y * tim, c.x * tim + c.y * tre);
    } else if constexpr (Mode == kScale) {
      a.data[g] = cscale(v, a.inv);
    } else {
      float2 gi = a.s[g];
      if (a.has_back) gi = cadd(gi, v);
      else gi = v;
      const float2 c = a.coef[g];
      const float q = a.q[g];
      const float ure = c.x * gi.x + c.y * gi.y;
      const float uim = c.x * gi.y - c.y * gi.x;
      a.data[g] = make_float2(q * ure, q * uim);
      a.s[g] = make_float2((1.0f - q) * ure, (1.0f - q) * uim);
    }
  }
}

// The same two passes on the register-resident engine (fft_reg.cuh) for n = 64, 128, 256: rows with
// R = 256 / T rows per CTA, T threads per row; columns with COLS = 256 / T columns per CTA, T threads
// per column, the epilogue of k_cols applied to the positions each thread holds.
template <bool Fwd, int T, int V>
__global__ void __launch_bounds__(kThreads)
    k_rows_reg(const float2* __restrict__ src, float2* __restrict__ dst, std::size_t rows, const float2* tw) {
  using Tile = regfft::RowTile<T>;
  constexpr int N = T * V;
  extern __shared__ float2 sm[];
  const int t = static_cast<int>(threadIdx.x) % T, r = static_cast<int>(threadIdx.x) / T;
  const std::size_t row = static_cast<std::size_t>(blockIdx.x) * Tile::R + r;
  const bool live = row < rows;
  float2 v[V];
#pragma unroll
  for (int j = 0; j < V; ++j) v[j] = live ? src[row * N + t + T * j] : make_float2(0.f, 0.f);
  regfft::line_fft<T, V, Fwd>(v, t, sm + r, Tile::A, Tile::B, tw);  // every row read before any write
  if (live) {
#pragma unroll
    for (int j = 0; j < V; ++j) dst[row * N + t + T * j] = v[j];
  }
}

template <bool Fwd, int Mode, int T, int V>
__global__ void __launch_bounds__(kThreads) k_cols_reg(ColArgs a, const float2* tw) {
  constexpr int N = T * V, COLS = kThreads / T;
  extern __shared__ float2 sm[];
  const int c = static_cast<int>(threadIdx.x) % COLS, t = static_cast<int>(threadIdx.x) / COLS;
  const int col = static_cast<int>(blockIdx.x) * COLS + c;
  const bool live = col < N;
  const std::size_t base = static_cast<std::size_t>(blockIdx.y) * N * N + (live ? col : 0);
  float2 v[V];
#pragma unroll
  for (int j = 0; j < V; ++j) v[j] = live ? a.data[base + static_cast<std::size_t>(t + T * j) * N] : make_float2(0.f, 0.f);
  regfft::line_fft<T, V, Fwd>(v, t, sm + c, T * COLS, COLS, tw);
  if (!live) return;
#pragma unroll
  for (int j = 0; j < V; ++j) {
    const int pos = t + T * j;
    const std::size_t g = base + static_cast<std::size_t>(pos) * N;
    const float2 vv = v[j];
    if constexpr (Mode == kScreen) {
      const float2 w = cscale(vv, a.inv);
      if (a.store) a.store[g] = w;
      float sn, cs;
      sincosf(a.phase * a.x[static_cast<std::size_t>(pos) * N + col], &sn, &cs);
      a.data[g] = cmul(make_float2(cs, sn), w);
    } else if constexpr (Mode == kPropagate) {
      const float2 cc = a.coef[g];
      const float q = a.q[g];
      const float2 sv = a.s[g];
      const float tre = q * vv.x + (1.0f - q) * sv.x;
      const float tim = q * vv.y + (1.0f - q) * sv.y;
      a.s[g] = make_float2(cc.x * tre - cc.y * tim, cc.x * tim + cc.y * tre);
    } else if constexpr (Mode == kScale) {
      a.data[g] = cscale(vv, a.inv);
    } else {
      float2 gi = a.s[g];
      if (a.has_back) gi = cadd(gi, vv);
      else gi = vv;
      const float2 cc = a.coef[g];
      const float q = a.q[g];
      const float ure = cc.x * gi.x + cc.y * gi.y;
      const float uim = cc.x * gi.y - cc.y * gi.x;
      a.data[g] = make_float2(q * ure, q * uim);
      a.s[g] = make_float2((1.0f - q) * ure, (1.0f - q) * uim);
    }
  }
}

template <int T, int V>
void fft2_reg(const float2* src, float2* dst, bool forward, int nb, int mode, const ColArgs& args, cudaStream_t s) {
  constexpr int N = T * V;
  const float2* tw = fft_len(N).tw;
  const std::size_t rows = static_cast<std::size_t>(nb) * N;
  {
    using Tile = regfft::RowTile<T>;
    const std::size_t smem = static_cast<std::size_t>(V) * Tile::A * sizeof(float2);
    const unsigned grid = static_cast<unsigned>((rows + Tile::R - 1) / Tile::R);
    const auto launch = [&](auto kernel) {
      ensure_smem(kernel);
      kernel<<<grid, kThreads, smem, s>>>(src, dst, rows, tw);
    };
    if (forward) {
      launch(k_rows_reg<true, T, V>);
    } else {
      launch(k_rows_reg<false, T, V>);
    }
    check_launch("bpm rows");
  }
  ColArgs a = args;
  a.data = dst;
  constexpr int COLS = kThreads / T;
  const std::size_t smem = static_cast<std::size_t>(N) * COLS * sizeof(float2);
  const dim3 grid((N + COLS - 1) / COLS, nb);
  const auto launch = [&](auto kernel) {
    ensure_smem(kernel);
    kernel<<<grid, kThreads, smem, s>>>(a, tw);
  };
  switch (mode) {
    case kScreen: launch(k_cols_reg<false, kScreen, T, V>); break;
    case kPropagate: launch(k_cols_reg<true, kPropagate, T, V>); break;
    case kScale: launch(k_cols_reg<false, kScale, T, V>); break;
    default: launch(k_cols_reg<true, kSplit, T, V>); break;
  }
  check_launch("bpm cols");
}

// One slice of the forward sweep as two passes on the register engine, each keeping a line of every
// plane on chip across a transform, the pointwise step and the opposite transform:
//   column pass (kPropInv): the forward column transform of the row-transformed envelope completes its
//     2D FFT W; S = c (q W + (1 - q) S) (as the kPropagate epilogue) is stored; the inverse column
//     transform of S starts the next inverse 2D FFT. kInvOnly applies only the inverse column transform to
//     S (the first slice of a recomputed segment).
//   row pass (kScreenFwd): the inverse row transform completes IFFT(S); x 1/n^2, store the envelope, times
//     the screen (as the kScreen epilogue), then the forward row transform of the next slice's FFT.
//     kScaleOut ends the sweep: inverse rows and x 1/n^2 only.
// The inverse 2D FFT thus runs columns first and the forward one rows first; the recomputed segments use
// the same two passes, so their envelopes are bitwise the forward sweep's.
enum SliceMode : int { kPropInv = 0, kInvOnly = 1, kScreenFwd = 2, kScaleOut = 3, kSplitInv = 4 };

template <int Mode, int T, int V>
__global__ void __launch_bounds__(kThreads) k_slice_cols(ColArgs a, const float2* tw) {
  constexpr int N = T * V, COLS = kThreads / T;
  extern __shared__ float2 sm[];
  const int c = static_cast<int>(threadIdx.x) % COLS, t = static_cast<int>(threadIdx.x) / COLS;
  const int col = static_cast<int>(blockIdx.x) * COLS + c;
  const bool live = col < N;
  const std::size_t base = static_cast<std::size_t>(blockIdx.y) * N * N + (live ? col : 0);
  float2 v[V];
  if constexpr (Mode == kPropInv) {
#pragma unroll
    for (int j = 0; j < V; ++j) v[j] = live ? a.data[base + static_cast<std::size_t>(t + T * j) * N] : make_float2(0.f, 0.f);
    regfft::line_fft<T, V, true>(v, t, sm + c, T * COLS, COLS, tw);
#pragma unroll
    for (int j = 0; j < V; ++j) {
      if (!live) continue;
      const std::size_t g = base + static_cast<std::size_t>(t + T * j) * N;
      const float2 vv = v[j];
      const float2 cc = a.coef[g];
      const float q = a.q[g];
      const float2 sv = a.s[g];
      const float tre = q * vv.x + (1.0f - q) * sv.x;
      const float tim = q * vv.y + (1.0f - q) * sv.y;
      v[j] = make_float2(cc.x * tre - cc.y * tim, cc.x * tim + cc.y * tre);
      a.s[g] = v[j];
    }
    __syncthreads();  // the inverse transform reuses the exchange buffer
  } else if constexpr (Mode == kSplitInv) {
    // Adjoint: the forward column transform completes FFT(w); U = conj(c)(g + back) (as the kSplit
    // epilogue), g = (1 - q) U is stored, b = q U goes on to the inverse column transform.
    if (a.grad && blockIdx.y == 0 && live) {  // the previous slice's per-group sums, in group order
      constexpr std::size_t plane = static_cast<std::size_t>(N) * N;
#pragma unroll
      for (int j = 0; j < V; ++j) {
        const std::size_t p = static_cast<std::size_t>(t + T * j) * N + col;
        float acc = a.part[p];
        for (int g = 1; g < a.groups; ++g) acc += a.part[g * plane + p];
        a.grad[p] += a.gscale * a.phase * acc;
      }
    }
#pragma unroll
    for (int j = 0; j < V; ++j) v[j] = live ? a.data[base + static_cast<std::size_t>(t + T * j) * N] : make_float2(0.f, 0.f);
    regfft::line_fft<T, V, true>(v, t, sm + c, T * COLS, COLS, tw);
#pragma unroll
    for (int j = 0; j < V; ++j) {
      if (!live) continue;
      const std::size_t g = base + static_cast<std::size_t>(t + T * j) * N;
      const float2 vv = v[j];
      float2 gi = a.s[g];
      if (a.has_back) gi = cadd(gi, vv);
      else gi = vv;
      const float2 cc = a.coef[g];
      const float q = a.q[g];
      const float ure = cc.x * gi.x + cc.y * gi.y;
      const float uim = cc.x * gi.y - cc.y * gi.x;
      v[j] = make_float2(q * ure, q * uim);
      a.s[g] = make_float2((1.0f - q) * ure, (1.0f - q) * uim);
    }
    __syncthreads();
  } else {
#pragma unroll
    for (int j = 0; j < V; ++j) v[j] = live ? a.s[base + static_cast<std::size_t>(t + T * j) * N] : make_float2(0.f, 0.f);
  }
  regfft::line_fft<T, V, false>(v, t, sm + c, T * COLS, COLS, tw);
  if (!live) return;
#pragma unroll
  for (int j = 0; j < V; ++j) a.data[base + static_cast<std::size_t>(t + T * j) * N] = v[j];
}

// Row pass for image row y (blockIdx.x) of one group of R = 256 / T illuminations (blockIdx.y), one row
// each, so that the group shares the screen factors of row y (computed once, in shared memory).
template <int Mode, int T, int V>
__global__ void __launch_bounds__(kThreads) k_slice_rows(ColArgs a, int nb, const float2* tw) {
  using Tile = regfft::RowTile<T>;
  constexpr int N = T * V, R = Tile::R;
  extern __shared__ float2 sm[];
  float2* screen = sm + static_cast<std::size_t>(V) * Tile::A;  // (cos, sin) of row y
  const int tid = static_cast<int>(threadIdx.x);
  const int t = tid % T, r = tid / T;
  const int y = static_cast<int>(blockIdx.x);
  const int view = static_cast<int>(blockIdx.y) * R + r;
  const bool live = view < nb;
  const std::size_t row = (static_cast<std::size_t>(live ? view : 0) * N + y) * N;
  if (Mode == kScreenFwd && tid < N) {
    float sn, cs;
    sincosf(a.phase * a.x[static_cast<std::size_t>(y) * N + tid], &sn, &cs);
    screen[tid] = make_float2(cs, sn);
  }
  float2 v[V];
#pragma unroll
  for (int j = 0; j < V; ++j) v[j] = live ? a.data[row + t + T * j] : make_float2(0.f, 0.f);
  regfft::line_fft<T, V, false>(v, t, sm + r, Tile::A, Tile::B, tw);  // its barrier also publishes `screen`
#pragma unroll
  for (int j = 0; j < V; ++j) {
    const int pos = t + T * j;
    float2 w = cscale(v[j], a.inv);
    if constexpr (Mode == kScreenFwd) {
      if (live && a.store) a.store[row + pos] = w;
      w = cmul(screen[pos], w);
    }
    v[j] = w;
  }
  if constexpr (Mode == kScreenFwd) {
    __syncthreads();  // the forward transform reuses the exchange buffer
    regfft::line_fft<T, V, true>(v, t, sm + r, Tile::A, Tile::B, tw);
  }
  if (!live) return;
#pragma unroll
  for (int j = 0; j < V; ++j) a.data[row + t + T * j] = v[j];
}

// Adjoint row pass of slice k for image row y (blockIdx.x) of one group of R = 256 / T illuminations
// (blockIdx.y), one row each: the inverse row transform completes IFFT(b); x 1/n^2; each view's term of the
// gradient, Im(conj(t w_k) b) with t = e^{i phase x_k}, goes to shared memory, and one thread per pixel adds
// the group's terms in view order into part[group, y, :]; b <- conj(t) b, then (kForward) the forward row
// transform of the next slice's FFT. k_gradient_groups adds the groups in order into the gradient.
template <bool kForward, int T, int V>
__global__ void __launch_bounds__(kThreads)
    k_slice_gradient(float2* __restrict__ data, const float2* __restrict__ env, const float* __restrict__ x,
                     float phase, float inv, int nb, float* __restrict__ part, const float2* tw) {
  using Tile = regfft::RowTile<T>;
  constexpr int N = T * V, R = Tile::R;
  extern __shared__ float2 sm[];
  float* terms = reinterpret_cast<float*>(sm + static_cast<std::size_t>(V) * Tile::A);  // R views x N pixels
  float2* screen = reinterpret_cast<float2*>(terms + R * N);                            // (cos, sin) of row y
  const int tid = static_cast<int>(threadIdx.x);
  const int t = tid % T, r = tid / T;
  const int y = static_cast<int>(blockIdx.x);
  const int v0 = static_cast<int>(blockIdx.y) * R;
  if (tid < N) {  // the screen of row y, the same for every view
    float sn, cs;
    sincosf(phase * x[static_cast<std::size_t>(y) * N + tid], &sn, &cs);
    screen[tid] = make_float2(cs, sn);
  }
  const int view = v0 + r;
  const bool live = view < nb;
  const std::size_t row = (static_cast<std::size_t>(live ? view : 0) * N + y) * N;
  float2 v[V];
#pragma unroll
  for (int j = 0; j < V; ++j) v[j] = live ? data[row + t + T * j] : make_float2(0.f, 0.f);
  regfft::line_fft<T, V, false>(v, t, sm + r, Tile::A, Tile::B, tw);  // its barrier also publishes `screen`
#pragma unroll
  for (int j = 0; j < V; ++j) {
    const int pos = t + T * j;
    const float cs = screen[pos].x, sn = screen[pos].y;
    const float2 bv = cscale(v[j], inv);
    float term = 0.0f;
    if (live) {
      const float2 w = cmul(make_float2(cs, sn), env[row + pos]);
      term = w.x * bv.y - w.y * bv.x;
    }
    terms[r * N + pos] = term;
    v[j] = cmul(make_float2(cs, -sn), bv);
  }
  __syncthreads();
  if (tid < N) {
    float acc = 0.0f;
    for (int i = 0; i < R && v0 + i < nb; ++i) acc += terms[i * N + tid];
    part[(static_cast<std::size_t>(blockIdx.y) * N + y) * N + tid] = acc;
  }
  if constexpr (kForward) regfft::line_fft<T, V, true>(v, t, sm + r, Tile::A, Tile::B, tw);
  if (!live) return;
#pragma unroll
  for (int j = 0; j < V; ++j) data[row + t + T * j] = v[j];
}

// grad += gscale phase (part[0] + part[1] + ...), the groups added in order, per pixel.
__global__ void k_gradient_groups(const float* __restrict__ part, int groups, std::size_t plane, float gscale,
                                  float phase, float* __restrict__ grad) {
  for (std::size_t p = blockIdx.x * static_cast<std::size_t>(blockDim.x) + threadIdx.x; p < plane;
       p += static_cast<std::size_t>(gridDim.x) * blockDim.x) {
    float acc = part[p];
    for (int g = 1; g < groups; ++g) acc += part[g * plane + p];
    grad[p] += gscale * phase * acc;
  }
}

// Calls f.template operator()<T, V>() for the plane sides the slice passes cover; false otherwise.
template <class F>
bool with_slice_shape(int n, F&& f) {
  if (!fft_reg_engine_enabled()) return false;
  switch (n) {
    case 64: f.template operator()<8, 8>(); return true;
    case 128: f.template operator()<8, 16>(); return true;
    case 256: f.template operator()<16, 16>(); return true;
    default: return false;
  }
}

template <int T, int V>
void slice_cols(int mode, const ColArgs& a, int nb, cudaStream_t s) {
  constexpr int N = T * V, COLS = kThreads / T;
  const std::size_t smem = static_cast<std::size_t>(N) * COLS * sizeof(float2);
  const dim3 grid((N + COLS - 1) / COLS, nb);
  const float2* tw = fft_len(N).tw;
  const auto launch = [&](auto kernel) {
    ensure_smem(kernel);
    kernel<<<grid, kThreads, smem, s>>>(a, tw);
  };
  if (mode == kPropInv) {
    launch(k_slice_cols<kPropInv, T, V>);
  } else if (mode == kSplitInv) {
    launch(k_slice_cols<kSplitInv, T, V>);
  } else {
    launch(k_slice_cols<kInvOnly, T, V>);
  }
  check_launch("bpm slice columns");
}

template <int T, int V>
void slice_rows(int mode, const ColArgs& a, int nb, cudaStream_t s) {
  using Tile = regfft::RowTile<T>;
  constexpr int N = T * V;
  const std::size_t smem = static_cast<std::size_t>(V) * Tile::A * sizeof(float2) + static_cast<std::size_t>(N) * sizeof(float2);
  const dim3 grid(N, (nb + Tile::R - 1) / Tile::R);
  const float2* tw = fft_len(N).tw;
  const auto launch = [&](auto kernel) {
    ensure_smem(kernel);
    kernel<<<grid, kThreads, smem, s>>>(a, nb, tw);
  };
  if (mode == kScreenFwd) {
    launch(k_slice_rows<kScreenFwd, T, V>);
  } else {
    launch(k_slice_rows<kScaleOut, T, V>);
  }
  check_launch("bpm slice rows");
}

template <int T, int V>
void slice_gradient(bool forward, float2* data, const float2* env, const float* x, float phase, float inv, int nb,
                    float gscale, float* part, float* grad, cudaStream_t s) {
  using Tile = regfft::RowTile<T>;
  constexpr int N = T * V;
  const int groups = (nb + Tile::R - 1) / Tile::R;
  const std::size_t smem = static_cast<std::size_t>(V) * Tile::A * sizeof(float2) +
                           static_cast<std::size_t>(Tile::R) * N * sizeof(float) + static_cast<std::size_t>(N) * sizeof(float2);
  const float2* tw = fft_len(N).tw;
  const dim3 grid(N, groups);
  const auto launch = [&](auto kernel) {
    ensure_smem(kernel);
    kernel<<<grid, kThreads, smem, s>>>(data, env, x, phase, inv, nb, part, tw);
  };
  if (forward) {
    launch(k_slice_gradient<true, T, V>);
  } else {
    launch(k_slice_gradient<false, T, V>);
  }
  check_launch("bpm slice gradient");
  if (grad) {  // else the next column pass adds the groups (ColArgs::grad)
    const std::size_t plane = static_cast<std::size_t>(N) * N;
    k_gradient_groups<<<static_cast<unsigned>((plane + kThreads - 1) / kThreads), kThreads, 0, s>>>(
        part, groups, plane, gscale, phase, grad);
    check_launch("bpm gradient groups");
  }
}

// Forward rows only (the envelope of the first slice entering the sweep).
template <int T, int V>
void rows_forward(float2* data, int nb, cudaStream_t s) {
  using Tile = regfft::RowTile<T>;
  constexpr int N = T * V;
  const std::size_t rows = static_cast<std::size_t>(nb) * N;
  const std::size_t smem = static_cast<std::size_t>(V) * Tile::A * sizeof(float2);
  const unsigned grid = static_cast<unsigned>((rows + Tile::R - 1) / Tile::R);
  ensure_smem(k_rows_reg<true, T, V>);
  k_rows_reg<true, T, V><<<grid, kThreads, smem, s>>>(data, data, rows, fft_len(N).tw);
  check_launch("bpm rows");
}

// Spectrum of the unit envelope: n^2 at the zero bin of every plane.
__global__ void k_unit_spectrum(float2* s, std::size_t plane, std::size_t total) {
  for (std::size_t i = blockIdx.x * static_cast<std::size_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<std::size_t>(gridDim.x) * blockDim.x) {
    s[i] = make_float2(i % plane == 0 ? static_cast<float>(plane) : 0.0f, 0.0f);
  }
}

// First slice: the envelope is 1; store it and apply the screen of slice 0.
__global__ void k_first_screen(float2* w, float2* store, const float* x, float phase, std::size_t plane,
                               std::size_t total) {
  for (std::size_t i = blockIdx.x * static_cast<std::size_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<std::size_t>(gridDim.x) * blockDim.x) {
    if (store) store[i] = make_float2(1.0f, 0.0f);
    float sn, cs;
    sincosf(phase * x[i % plane], &sn, &cs);
    w[i] = make_float2(cs, sn);
  }
}

// r = y - data in place, and per-CTA sums of |r|^2 in double.
__global__ void __launch_bounds__(kThreads)
    k_residual(float2* y, const float2* __restrict__ data, std::size_t total, double* partial) {
  __shared__ double red[kThreads];
  double acc = 0.0;
  for (std::size_t i = blockIdx.x * static_cast<std::size_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<std::size_t>(gridDim.x) * blockDim.x) {
    const float2 v = csub(y[i], data[i]);
    y[i] = v;
    acc += static_cast<double>(v.x) * v.x + static_cast<double>(v.y) * v.y;
  }
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int h = blockDim.x / 2; h > 0; h >>= 1) {
    if (static_cast<int>(threadIdx.x) < h) red[threadIdx.x] += red[threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
}

// Sums `n` partials in order and adds the result to *out.
__global__ void k_sum_partials(const double* partial, int n, double* out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double s = 0.0;
    for (int i = 0; i < n; ++i) s += partial[i];
    *out += s;
  }
}

// One thread per pixel of slice k: grad += gscale * phase * sum_a Im(conj(t w_a) b_a), and
// b_a <- conj(t) b_a, t = e^{i phase x}.
__global__ void k_gradient(float2* b, const float2* __restrict__ store, const float* __restrict__ x, float phase,
                           int nb, std::size_t plane, float gscale, float* grad) {
  for (std::size_t p = blockIdx.x * static_cast<std::size_t>(blockDim.x) + threadIdx.x; p < plane;
       p += static_cast<std::size_t>(gridDim.x) * blockDim.x) {
    float sn, cs;
    sincosf(phase * x[p], &sn, &cs);
    float acc = 0.0f;
    for (int j = 0; j < nb; ++j) {
      const std::size_t o = j * plane + p;
      const float2 bv = b[o];
      const float2 v = cmul(make_float2(cs, sn), store[o]);
      acc += v.x * bv.y - v.y * bv.x;
      b[o] = cmul(make_float2(cs, -sn), bv);
    }
    grad[p] += gscale * phase * acc;
  }
}

__global__ void k_axpy_clamp(const float* point, const float* grad, float alpha, std::size_t total, float* z,
                             float* out) {
  for (std::size_t i = blockIdx.x * static_cast<std::size_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<std::size_t>(gridDim.x) * blockDim.x) {
    const float v = point[i] - alpha * grad[i];
    if (z) z[i] = v;
    if (out) out[i] = fmaxf(v, 0.0f);
  }
}

__global__ void k_extrapolate(const float* next, float* x, float momentum, std::size_t total, float* y) {
  for (std::size_t i = blockIdx.x * static_cast<std::size_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<std::size_t>(gridDim.x) * blockDim.x) {
    const float nv = next[i];
    y[i] = nv + momentum * (nv - x[i]);
    x[i] = nv;
  }
}

__global__ void k_contrast(const float* ri, float nm, std::size_t total, float* x, bool clamp) {
  for (std::size_t i = blockIdx.x * static_cast<std::size_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<std::size_t>(gridDim.x) * blockDim.x) {
    const float v = __fsub_rn(ri[i], nm);
    x[i] = clamp ? fmaxf(v, 0.0f) : v;
  }
}

__global__ void k_add_medium(const float* x, float nm, std::size_t total, float* ri) {
  for (std::size_t i = blockIdx.x * static_cast<std::size_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<std::size_t>(gridDim.x) * blockDim.x) {
    ri[i] = __fadd_rn(x[i], nm);
  }
}

unsigned grid_for(std::size_t total) {
  return static_cast<unsigned>(std::min<std::size_t>((total + kThreads - 1) / kThreads, 148u * 32u));
}

int rows_cols(int n) {
  int c = 16;
  while (c > 1 && 2 * static_cast<std::size_t>(n) * (c + 1) * sizeof(float2) > 72 * 1024) c /= 2;
  return c;
}

}  // namespace

// Per-view tables of the multi-slice model (the quantities of src/bpm.cpp:10-60), on the lateral DFT
// grid in transform order. For a scattered plane wave of lateral frequency (fy, fx) = bin + illumination
// that propagates in the medium (fy^2 + fx^2 < fm^2), with axial frequency nu = sqrt(fm^2 - fy^2 - fx^2):
//   step  e^{i 2 pi (nu - fiz) dz}: one slice of propagation of the envelope (the carrier e^{i 2 pi fiz z}
//         of the illumination factored out), dz = pixel;
//   last  e^{i 2 pi (nu - fiz) z_back}: from the last slice back to the volume's central plane, where the
//         fields are recorded, kept only inside the pupil (fy^2 + fx^2 <= fna^2);
//   q     the obliquity fm / nu of the thin-screen update, with nu bounded below by
//         sqrt(max(fm^2 - fna^2, fm^2 / 100)); 1 without obliquity and for evanescent bins.
// Evanescent bins propagate nothing (step = last = 0). The Lipschitz constant of the data term's
// gradient is nz (k0 dz)^2 times the mean over views of q^2 at the view's own direction (bin 0).
// Computed in double, stored in float.
BpmTablesHost bpm_tables(int n, int nz, const float* il, int count, float wavelength, float n_medium, float na,
                         float pixel, bool obliquity) {
  const double two_pi = 2.0 * std::numbers::pi;
  const double fm2 = (double(n_medium) / wavelength) * (double(n_medium) / wavelength);
  const double fna2 = (double(na) / wavelength) * (double(na) / wavelength);
  const double dz = pixel;
  const double df = 1.0 / (n * dz);
  const double nu_floor = std::sqrt(std::max(fm2 - fna2, 0.01 * fm2));
  const double z_back = -(nz - 1 - nz / 2) * dz;  // central plane, seen from the last slice
  const auto unit = [](double angle) {
    const std::complex<double> w = std::exp(std::complex<double>(0.0, angle));
    return make_float2(static_cast<float>(w.real()), static_cast<float>(w.imag()));
  };
  const auto obliquity_of = [&](double nu) { return obliquity ? std::sqrt(fm2) / std::max(nu, nu_floor) : 1.0; };

  BpmTablesHost t;
  t.n = n;
  t.nz = nz;
  t.count = count;
  t.phase = static_cast<float>(two_pi / wavelength * dz);
  const std::size_t plane = static_cast<std::size_t>(n) * n;
  t.step.assign(plane * count, make_float2(0, 0));
  t.last.assign(plane * count, make_float2(0, 0));
  t.q.assign(plane * count, 1.0f);
  double mean_q2 = 0;
  for (int a = 0; a < count; ++a) {
    const double fiy = il[2 * a], fix = il[2 * a + 1];
    const double fiz = std::sqrt(fm2 - fiy * fiy - fix * fix);
    float2* step = t.step.data() + a * plane;
    float2* last = t.last.data() + a * plane;
    float* q = t.q.data() + a * plane;
    for (int ky = 0; ky < n; ++ky) {
      const double fy = signed_bin(ky, n) * df + fiy;
      for (int kx = 0; kx < n; ++kx) {
        const double fx = signed_bin(kx, n) * df + fix;
        const double rho2 = fy * fy + fx * fx;
        if (rho2 >= fm2) continue;  // evanescent
        const std::size_t b = static_cast<std::size_t>(ky) * n + kx;
        const double nu = std::sqrt(fm2 - rho2);
        step[b] = unit(two_pi * (nu - fiz) * dz);
        if (rho2 <= fna2) last[b] = unit(two_pi * (nu - fiz) * z_back);
        q[b] = static_cast<float>(obliquity_of(nu));
      }
    }
    mean_q2 += static_cast<double>(q[0]) * q[0] / count;
  }
  t.lipschitz = static_cast<float>(nz * static_cast<double>(t.phase) * t.phase * mean_q2);
  return t;
}

BpmPlan::BpmPlan(const BpmTablesHost& t, int chunk, bool store, int checkpoint_every)
    : t_(t), chunk_(chunk), store_on_(store && checkpoint_every <= 0), every_(std::max(checkpoint_every, 0)) {
  require(t.n >= 4 && t.n % 2 == 0 && t.nz >= 1 && t.count >= 1, "bpm: invalid tables");
  require(chunk >= 1 && chunk <= t.count && chunk <= 65535, "bpm: invalid chunk");
  plane_ = static_cast<std::size_t>(t.n) * t.n;
  const std::size_t all = plane_ * t.count;
  step_.reset(all);
  last_.reset(all);
  q_.reset(all);
  check(cudaMemcpy(step_.get(), t.step.data(), step_.bytes(), cudaMemcpyHostToDevice), "upload tables");
  check(cudaMemcpy(last_.get(), t.last.data(), last_.bytes(), cudaMemcpyHostToDevice), "upload tables");
  check(cudaMemcpy(q_.get(), t.q.data(), q_.bytes(), cudaMemcpyHostToDevice), "upload tables");
  s_.reset(plane_ * chunk);
  w_.reset(plane_ * chunk);
  if (store_on_) stored_.reset(plane_ * chunk * t.nz);
  if (every_ > 0) {
    const int segments = (t.nz + every_ - 1) / every_;
    ckpt_.reset(plane_ * t.count * segments);
    env_.reset(plane_ * chunk * std::min(every_, t.nz));
    rs_.reset(plane_ * chunk);
    rw_.reset(plane_ * chunk);
  }
  partial_.reset(4096);
  gpart_.reset(plane_ * ((chunk + 15) / 16));  // per-group gradient sums (groups of at least 16 views)
}

std::size_t BpmPlan::device_bytes() const {
  return step_.bytes() + last_.bytes() + q_.bytes() + s_.bytes() + w_.bytes() + stored_.bytes() + partial_.bytes() +
         ckpt_.bytes() + env_.bytes() + rs_.bytes() + rw_.bytes() + gpart_.bytes();
}

void BpmPlan::fft2(const float2* src, float2* dst, bool forward, int nb, int mode, const void* args_v,
                   cudaStream_t s) {
  const int n = t_.n;
  if (fft_reg_engine_enabled() && (n == 64 || n == 128 || n == 256)) {
    const ColArgs& args = *static_cast<const ColArgs*>(args_v);
    if (n == 64) {
      fft2_reg<8, 8>(src, dst, forward, nb, mode, args, s);
    } else if (n == 128) {
      fft2_reg<8, 16>(src, dst, forward, nb, mode, args, s);
    } else {
      fft2_reg<16, 16>(src, dst, forward, nb, mode, args, s);
    }
    return;
  }
  const FftLen& L = fft_len(n);
  const int c = rows_cols(n);
  const std::size_t rows = static_cast<std::size_t>(nb) * n;
  {
    const std::size_t smem = 2 * static_cast<std::size_t>(n) * (c + 1) * sizeof(float2);
    const unsigned grid = static_cast<unsigned>((rows + c - 1) / c);
#define QHK_ROWS(C)                                                      \
  case C:                                                                \
    if (forward) {                                                       \
      allow(k_rows<true, C>, smem);                                      \
      k_rows<true, C><<<grid, kThreads, smem, s>>>(src, dst, rows, L);   \
    } else {                                                             \
      allow(k_rows<false, C>, smem);                                     \
      k_rows<false, C><<<grid, kThreads, smem, s>>>(src, dst, rows, L);  \
    }                                                                    \
    break;
    switch (c) {
      QHK_ROWS(16)
      QHK_ROWS(8)
      QHK_ROWS(4)
      QHK_ROWS(2)
      QHK_ROWS(1)
    }
#undef QHK_ROWS
    check_launch("bpm rows");
  }
  ColArgs a = *static_cast<const ColArgs*>(args_v);
  a.data = dst;
  const std::size_t smem = 2 * static_cast<std::size_t>(n) * c * sizeof(float2);
  const dim3 grid((n + c - 1) / c, nb);
#define QHK_COLS(C)                                                                                   \
  case C:                                                                                             \
    switch (mode) {                                                                                   \
      case kScreen: allow(k_cols<false, kScreen, C>, smem); k_cols<false, kScreen, C><<<grid, kThreads, smem, s>>>(a, L); break; \
      case kPropagate: allow(k_cols<true, kPropagate, C>, smem); k_cols<true, kPropagate, C><<<grid, kThreads, smem, s>>>(a, L); break; \
      case kScale: allow(k_cols<false, kScale, C>, smem); k_cols<false, kScale, C><<<grid, kThreads, smem, s>>>(a, L); break; \
      default: allow(k_cols<true, kSplit, C>, smem); k_cols<true, kSplit, C><<<grid, kThreads, smem, s>>>(a, L); break; \
    }                                                                                                 \
    break;
  switch (c) {
    QHK_COLS(16)
    QHK_COLS(8)
    QHK_COLS(4)
    QHK_COLS(2)
    QHK_COLS(1)
  }
#undef QHK_COLS
  check_launch("bpm columns");
}

void BpmPlan::forward(const float* x, int first, int nb, cudaStream_t s) {
  const NvtxRange r("qhk:bpm_forward");
  const int nz = t_.nz;
  const std::size_t total = plane_ * nb;
  const std::size_t off = plane_ * first;
  const float inv = 1.0f / static_cast<float>(plane_);
  k_unit_spectrum<<<grid_for(total), kThreads, 0, s>>>(s_.get(), plane_, total);
  check_launch("bpm start");
  k_first_screen<<<grid_for(total), kThreads, 0, s>>>(w_.get(), store_on_ ? stored_.get() : nullptr, x, t_.phase,
                                                      plane_, total);
  check_launch("bpm start");
  // Two passes per slice on the register engine (k_slice_cols / k_slice_rows).
  if (with_slice_shape(t_.n, [&]<int T, int V>() {
        rows_forward<T, V>(w_.get(), nb, s);
        for (int k = 0; k < nz; ++k) {
          if (every_ > 0 && k % every_ == 0) {
            float2* ck = ckpt_.get() + (static_cast<std::size_t>(k / every_) * t_.count + first) * plane_;
            check(cudaMemcpyAsync(ck, s_.get(), total * sizeof(float2), cudaMemcpyDeviceToDevice, s),
                  "bpm checkpoint");
          }
          ColArgs c{};
          c.data = w_.get();
          c.s = s_.get();
          c.coef = (k == nz - 1 ? last_.get() : step_.get()) + off;
          c.q = q_.get() + off;
          slice_cols<T, V>(kPropInv, c, nb, s);
          ColArgs w{};
          w.data = w_.get();
          w.inv = inv;
          if (k + 1 < nz) {
            w.store = store_on_ ? stored_.get() + (k + 1) * total : nullptr;
            w.x = x + (k + 1) * plane_;
            w.phase = t_.phase;
            slice_rows<T, V>(kScreenFwd, w, nb, s);
          } else {
            slice_rows<T, V>(kScaleOut, w, nb, s);  // envelopes at z = 0 in w
          }
        }
      })) {
    return;
  }
  for (int k = 0; k < nz; ++k) {
    if (every_ > 0 && k % every_ == 0) {
      // Spectrum entering slice k of illuminations first .. first + nb - 1.
      float2* ck = ckpt_.get() + (static_cast<std::size_t>(k / every_) * t_.count + first) * plane_;
      check(cudaMemcpyAsync(ck, s_.get(), total * sizeof(float2), cudaMemcpyDeviceToDevice, s), "bpm checkpoint");
    }
    if (k > 0) {
      ColArgs a{};
      a.store = store_on_ ? stored_.get() + k * total : nullptr;
      a.x = x + k * plane_;
      a.phase = t_.phase;
      a.inv = inv;
      fft2(s_.get(), w_.get(), false, nb, kScreen, &a, s);
    }
    ColArgs a{};
    a.s = s_.get();
    a.coef = (k == nz - 1 ? last_.get() : step_.get()) + off;
    a.q = q_.get() + off;
    fft2(w_.get(), w_.get(), true, nb, kPropagate, &a, s);
  }
  ColArgs a{};
  a.inv = inv;
  fft2(s_.get(), w_.get(), false, nb, kScale, &a, s);  // envelopes at z = 0 in w
}

void BpmPlan::adjoint(const float* x, const float2* residual_or_null, int first, int nb, float gscale, float* grad,
                      cudaStream_t s) {
  const NvtxRange r("qhk:bpm_adjoint");
  const int nz = t_.nz;
  const std::size_t total = plane_ * nb;
  const std::size_t off = plane_ * first;
  const float inv = 1.0f / static_cast<float>(plane_);
  // w holds the residual r (or it is copied in); g = FFT(r), split at the last slice.
  if (residual_or_null) {
    check(cudaMemcpyAsync(w_.get(), residual_or_null, total * sizeof(float2), cudaMemcpyDeviceToDevice, s),
          "copy residual");
  }
  require(store_on_ || every_ > 0, "bpm: the plan keeps no envelopes for an adjoint");
  const auto envelope = [&](int k) -> const float2* {
    if (every_ > 0) {
      const int k0 = (k / every_) * every_;
      if (k == nz - 1 || k % every_ == every_ - 1) recompute(x, first, nb, k0, std::min(k0 + every_, nz), s);
      return env_.get() + (k - k0) * total;
    }
    return stored_.get() + k * total;
  };
  // Two passes per slice on the register engine: k_slice_gradient (inverse rows, gradient, conj(screen),
  // forward rows) and k_slice_cols<kSplitInv> (forward columns, split, inverse columns).
  if (with_slice_shape(t_.n, [&]<int T, int V>() {
        const int groups = (nb + regfft::RowTile<T>::R - 1) / regfft::RowTile<T>::R;
        const auto split = [&](const float2* coef, int has_back, float* slice_grad) {
          ColArgs c{};
          c.data = w_.get();
          c.s = s_.get();
          c.coef = coef + off;
          c.q = q_.get() + off;
          c.has_back = has_back;
          c.part = gpart_.get();
          c.groups = groups;
          c.gscale = gscale;
          c.phase = t_.phase;
          c.grad = slice_grad;
          slice_cols<T, V>(kSplitInv, c, nb, s);
        };
        rows_forward<T, V>(w_.get(), nb, s);
        split(last_.get(), 0, nullptr);
        for (int k = nz - 1; k >= 0; --k) {
          const float2* env = envelope(k);
          // Slice k's gradient groups are added by the next column pass, or here for the last slice.
          slice_gradient<T, V>(k > 0, w_.get(), env, x + k * plane_, t_.phase, inv, nb, gscale, gpart_.get(),
                               k > 0 ? nullptr : grad, s);
          if (k > 0) split(step_.get(), 1, grad + k * plane_);
        }
      })) {
    return;
  }
  ColArgs a{};
  a.s = s_.get();
  a.coef = last_.get() + off;
  a.q = q_.get() + off;
  a.has_back = 0;
  fft2(w_.get(), w_.get(), true, nb, kSplit, &a, s);
  for (int k = nz - 1; k >= 0; --k) {
    const float2* env = envelope(k);
    ColArgs b{};
    b.inv = inv;
    fft2(w_.get(), w_.get(), false, nb, kScale, &b, s);
    k_gradient<<<grid_for(plane_), kThreads, 0, s>>>(w_.get(), env, x + k * plane_, t_.phase, nb, plane_, gscale,
                                                     grad + k * plane_);
    check_launch("bpm gradient");
    if (k > 0) {
      ColArgs c{};
      c.s = s_.get();
      c.coef = step_.get() + off;
      c.q = q_.get() + off;
      c.has_back = 1;
      fft2(w_.get(), w_.get(), true, nb, kSplit, &c, s);
    }
  }
}

void BpmPlan::recompute(const float* x, int first, int nb, int k0, int k1, cudaStream_t s) {
  const std::size_t total = plane_ * nb;
  const std::size_t off = plane_ * first;
  const float inv = 1.0f / static_cast<float>(plane_);
  const float2* ck = ckpt_.get() + (static_cast<std::size_t>(k0 / every_) * t_.count + first) * plane_;
  check(cudaMemcpyAsync(rs_.get(), ck, total * sizeof(float2), cudaMemcpyDeviceToDevice, s), "bpm restore");
  // The forward sweep's two passes per slice (register engine), so the envelopes are bitwise its own.
  if (with_slice_shape(t_.n, [&]<int T, int V>() {
        const auto screen = [&](int k) {  // rw_ holds C^-1(S) of slice k: envelope k, then its row FFT
          ColArgs w{};
          w.data = rw_.get();
          w.inv = inv;
          w.store = env_.get() + (k - k0) * total;
          w.x = x + k * plane_;
          w.phase = t_.phase;
          slice_rows<T, V>(kScreenFwd, w, nb, s);
        };
        if (k0 == 0) {
          k_first_screen<<<grid_for(total), kThreads, 0, s>>>(rw_.get(), env_.get(), x, t_.phase, plane_, total);
          check_launch("bpm recompute");
          rows_forward<T, V>(rw_.get(), nb, s);
        } else {
          ColArgs c{};
          c.data = rw_.get();
          c.s = rs_.get();
          slice_cols<T, V>(kInvOnly, c, nb, s);
          screen(k0);
        }
        for (int k = k0; k + 1 < k1; ++k) {  // the spectrum entering k + 1, then envelope k + 1
          ColArgs c{};
          c.data = rw_.get();
          c.s = rs_.get();
          c.coef = step_.get() + off;
          c.q = q_.get() + off;
          slice_cols<T, V>(kPropInv, c, nb, s);
          screen(k + 1);
        }
      })) {
    return;
  }
  for (int k = k0; k < k1; ++k) {
    float2* env = env_.get() + (k - k0) * total;
    if (k == 0) {
      k_first_screen<<<grid_for(total), kThreads, 0, s>>>(rw_.get(), env, x, t_.phase, plane_, total);
      check_launch("bpm recompute");
    } else {
      ColArgs a{};
      a.store = env;
      a.x = x + k * plane_;
      a.phase = t_.phase;
      a.inv = inv;
      fft2(rs_.get(), rw_.get(), false, nb, kScreen, &a, s);
    }
    if (k + 1 < k1) {  // the spectrum entering slice k + 1 (slices k1 .. have their own checkpoint)
      ColArgs a{};
      a.s = rs_.get();
      a.coef = step_.get() + off;
      a.q = q_.get() + off;
      fft2(rw_.get(), rw_.get(), true, nb, kPropagate, &a, s);
    }
  }
}

double BpmPlan::residual(const float2* data, int first, int nb, double* d_loss, cudaStream_t s) {
  const std::size_t total = plane_ * nb;
  const unsigned blocks = std::min<unsigned>(grid_for(total), 4096);
  k_residual<<<blocks, kThreads, 0, s>>>(w_.get(), data + plane_ * first, total, partial_.get());
  check_launch("bpm residual");
  k_sum_partials<<<1, 32, 0, s>>>(partial_.get(), static_cast<int>(blocks), d_loss);
  check_launch("bpm residual");
  return 0.0;
}

void contrast(const float* ri, float n_medium, std::size_t total, float* x, bool clamp, cudaStream_t s) {
  k_contrast<<<grid_for(total), kThreads, 0, s>>>(ri, n_medium, total, x, clamp);
  check_launch("contrast");
}

void add_medium(const float* x, float n_medium, std::size_t total, float* ri, cudaStream_t s) {
  k_add_medium<<<grid_for(total), kThreads, 0, s>>>(x, n_medium, total, ri);
  check_launch("add medium");
}

void bpm_solve(const BpmTablesHost& t, const float2* d_fields, float* d_x, int iterations, int batch, float step,
               float tv_weight, int tv_inner, double* d_loss, cudaStream_t s, unsigned long long* d_waits) {
  const int count = t.count;
  batch = batch <= 0 || batch >= count ? count : batch;
  const bool fista = batch == count;
  const float alpha = step / t.lipschitz;
  const bool tv = tv_weight > 0;
  const std::size_t size = static_cast<std::size_t>(t.nz) * t.n * t.n;
  BpmPlan plan(t, batch, true);
  DevBuf<float> vols(4 * size);
  float* y = vols.get();
  float* next = y + size;
  float* grad = y + 2 * size;
  float* z = y + 3 * size;
  DevBuf<float> dual(tv ? 12 * size : 0);
  TvBuffers tvb;
  tvb.wait_status = d_waits;
  if (tv) {
    check(cudaMemsetAsync(dual.get(), 0, 3 * size * sizeof(float), s), "cudaMemset");
    for (int i = 0; i < 4; ++i)
      for (int c = 0; c < 3; ++c) tvb.v[i][c] = dual.get() + (3 * i + c) * size;
  }
  check(cudaMemcpyAsync(y, d_x, size * sizeof(float), cudaMemcpyDeviceToDevice, s), "copy x");
  const auto gradient = [&](const float* point, int first, int last, double* loss) {
    check(cudaMemsetAsync(grad, 0, size * sizeof(float), s), "cudaMemset");
    plan.forward(point, first, last - first, s);
    plan.residual(d_fields, first, last - first, loss, s);
    plan.adjoint(point, nullptr, first, last - first, 1.0f / static_cast<float>(last - first), grad, s);
  };
  const auto prox = [&](const float* point, float* out) {
    if (tv) {
      k_axpy_clamp<<<grid_for(size), kThreads, 0, s>>>(point, grad, alpha, size, z, nullptr);
      check_launch("gradient step");
      tv_prox(z, tvb, t.nz, t.n, t.n, alpha * tv_weight, tv_inner, TvFinal::plain, 0.0f, nullptr, out, 0, 0, s);
    } else {
      k_axpy_clamp<<<grid_for(size), kThreads, 0, s>>>(point, grad, alpha, size, nullptr, out);
      check_launch("gradient step");
    }
  };
  float tk = 1.0f;
  for (int it = 0; it < iterations; ++it) {
    if (fista) {
      gradient(y, 0, count, d_loss + it);
      prox(y, next);
      const float tn = fista_t(tk);
      k_extrapolate<<<grid_for(size), kThreads, 0, s>>>(next, d_x, (tk - 1.0f) / tn, size, y);
      check_launch("extrapolate");
      tk = tn;
    } else {
      for (int first = 0; first < count; first += batch) {
        gradient(d_x, first, std::min(first + batch, count), d_loss + it);
        prox(d_x, d_x);
      }
    }
  }
  check(cudaStreamSynchronize(s), "bpm_reconstruct");
}

}  // namespace qhk
