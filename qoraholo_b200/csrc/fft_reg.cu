// FFT axis passes on the register-resident engine (fft_reg.cuh) for the lengths it covers: 64, 128,
// 192, 256 and 512. A CTA takes COLS lines (consecutive inner columns) of one outer slice, T threads per
// line holding V = n / T values each; loads and stores are rows of COLS consecutive complex values.
// The modes are those of the staged kernels (fft3d.cu k_axis): plain transform with a scale, the
// k-space restore between a forward and an inverse transform (half-spectrum data or a mask), and an
// inverse transform of aux data times a scale.
#include <cstdlib>
#include <cstring>

#include "fft_reg.cuh"
#include "qhk_internal.hpp"

namespace qhk {

namespace {

constexpr int kRegThreads = 256;

// Resident CTAs per SM, so that their loads overlap each other's transforms: for V <= 16 values per
// thread, three for one transform (at most 85 registers) and two for the restore modes, which hold two
// transforms' state (at most 128); longer per-thread DFTs keep the registers they need (no bound).
constexpr bool restore_mode(int mode) {
  return mode == static_cast<int>(AxisMode::restore_half) || mode == static_cast<int>(AxisMode::restore_mask);
}
constexpr int axis_min_blocks(int mode, int V) { return V >= 24 ? 1 : restore_mode(mode) ? 2 : 3; }

template <bool Fwd, int Mode, int T, int V>
__global__ void __launch_bounds__(kRegThreads, axis_min_blocks(Mode, V))
    k_axis_reg(float2* __restrict__ data, std::size_t so, std::size_t sp, int ni, const float2* __restrict__ tw,
               float scale, const float2* __restrict__ aux_a, const std::uint8_t* __restrict__ aux_h,
               std::size_t sb) {
  constexpr int COLS = kRegThreads / T;
  extern __shared__ float2 xs[];  // T * V * COLS exchange values
  constexpr int kFrom = static_cast<int>(AxisMode::from_data);
  constexpr int kHalf = static_cast<int>(AxisMode::restore_half);
  constexpr int kMask = static_cast<int>(AxisMode::restore_mask);
  constexpr std::size_t kSmem = (static_cast<std::size_t>(T) * V * COLS + (Mode == kHalf || Mode == kMask ? V * kRegThreads : 0)) * sizeof(float2);
  if (!QHK_CHECK(kSmem <= debug::dynamic_smem_bytes() && blockDim.x == kRegThreads)) return;  // block-uniform
  const int c = static_cast<int>(threadIdx.x) % COLS;
  const int t = static_cast<int>(threadIdx.x) / COLS;
  const int col = static_cast<int>(blockIdx.x) * COLS + c;
  const bool live = col < ni;
  const std::size_t base =
      static_cast<std::size_t>(blockIdx.z) * sb + static_cast<std::size_t>(blockIdx.y) * so + (live ? col : 0);
  float2 v[V];
#pragma unroll
  for (int j = 0; j < V; ++j) {
    const std::size_t g = base + static_cast<std::size_t>(t + T * j) * sp;
    v[j] = live ? (Mode == kFrom ? cscale(aux_a[g], scale) : data[g]) : make_float2(0.0f, 0.0f);
  }
  if constexpr (Mode == kHalf || Mode == kMask) {
    // The restore's data a streams into shared memory (cp.async, each thread its own positions, read
    // back by the same thread) while the forward transform runs; the hit counts, one byte each, are
    // packed four to a register. Neither occupies the transform's registers.
    float2* as = xs + static_cast<std::size_t>(T) * V * COLS + threadIdx.x;  // as[j * blockDim]
    unsigned hp[(V + 3) / 4] = {};
#pragma unroll
    for (int j = 0; j < V; ++j) {
      const std::size_t g = base + static_cast<std::size_t>(t + T * j) * sp;
      if (live) {
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(static_cast<unsigned>(
                         __cvta_generic_to_shared(as + j * kRegThreads))),
                     "l"(aux_a + g)
                     : "memory");
        hp[j / 4] |= static_cast<unsigned>(aux_h[g]) << (8 * (j % 4));
      } else {
        as[j * kRegThreads] = make_float2(0.0f, 0.0f);
      }
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    regfft::line_fft<T, V, true>(v, t, xs + c, T * COLS, COLS, tw);
    asm volatile("cp.async.wait_all;\n" ::: "memory");
#pragma unroll
    for (int j = 0; j < V; ++j) {
      const float2 a = as[j * kRegThreads];
      const unsigned h = (hp[j / 4] >> (8 * (j % 4))) & 0xffu;
      if constexpr (Mode == kHalf) {
        const float w = 1.0f - 0.5f * static_cast<float>(h);
        v[j] = make_float2((a.x + w * v[j].x) * scale, (a.y + w * v[j].y) * scale);
      } else {
        if (h) v[j] = a;
      }
    }
    __syncthreads();  // every thread has read the exchange buffer of the forward transform
    regfft::line_fft<T, V, false>(v, t, xs + c, T * COLS, COLS, tw);
  } else {
    regfft::line_fft<T, V, Fwd>(v, t, xs + c, T * COLS, COLS, tw);
    if (Mode == static_cast<int>(AxisMode::plain) && scale != 1.0f) {
#pragma unroll
      for (int j = 0; j < V; ++j) v[j] = cscale(v[j], scale);
    }
  }
  if (live) {
#pragma unroll
    for (int j = 0; j < V; ++j) data[base + static_cast<std::size_t>(t + T * j) * sp] = v[j];
  }
}

template <bool Fwd, int Mode, int T, int V>
void launch_axis_reg(float2* data, int n_outer, std::size_t so, std::size_t sp, int ni, float scale,
                     const AxisAux& aux, int batch, std::size_t sb, cudaStream_t s) {
  constexpr int COLS = kRegThreads / T;
  // The exchange buffer, and for the restore modes the staged restore data (V values per thread).
  const bool restore = Mode == static_cast<int>(AxisMode::restore_half) || Mode == static_cast<int>(AxisMode::restore_mask);
  const std::size_t smem = (static_cast<std::size_t>(T) * V * COLS + (restore ? V * kRegThreads : 0)) * sizeof(float2);
  auto kernel = k_axis_reg<Fwd, Mode, T, V>;
  ensure_smem(kernel);
  const dim3 grid((ni + COLS - 1) / COLS, n_outer, batch);
  kernel<<<grid, kRegThreads, smem, s>>>(data, so, sp, ni, fft_len(T * V).tw, scale, aux.a, aux.hits, sb);
  check_launch("fft axis pass");
}

template <int T, int V>
void axis_reg_mode(float2* data, int n_outer, std::size_t so, std::size_t sp, int ni, bool forward, AxisMode mode,
                   float scale, const AxisAux& aux, int batch, std::size_t sb, cudaStream_t s) {
  switch (mode) {
    case AxisMode::plain:
      if (forward) {
        launch_axis_reg<true, 0, T, V>(data, n_outer, so, sp, ni, scale, aux, batch, sb, s);
      } else {
        launch_axis_reg<false, 0, T, V>(data, n_outer, so, sp, ni, scale, aux, batch, sb, s);
      }
      break;
    case AxisMode::restore_half:
      launch_axis_reg<true, 1, T, V>(data, n_outer, so, sp, ni, scale, aux, batch, sb, s);
      break;
    case AxisMode::restore_mask:
      launch_axis_reg<true, 2, T, V>(data, n_outer, so, sp, ni, scale, aux, batch, sb, s);
      break;
    case AxisMode::from_data:
      launch_axis_reg<false, 3, T, V>(data, n_outer, so, sp, ni, scale, aux, batch, sb, s);
      break;
  }
}

// ---- real rows <-> half spectra ---------------------------------------------------------------------
// Rows of nx = 2M real values as M complex values (the pairs 2m, 2m + 1), a length-M transform on the
// register engine (the R2C, C2R and GP-step-boundary passes; the FISTA-TV final-primal pass stays on the
// staged engine, whose flat loads of its seven operands measured faster), and the split / merge of the half spectrum with the same formulas as the staged row
// kernels (fft3d.cu k_rows_*): e[k] = (Z[k] + conj Z[M-k]) / 2 + W_nx^k (Z[k] - conj Z[M-k]) / (2i),
// k = 0..M. A CTA takes R = 256 / T rows, T threads per row (consecutive threads on consecutive
// positions of a row), for half lengths 64, 128, 192 and 256. The exchange buffer has strides A, B of
// the row-tile layout (conflict-free in
// both exchange phases); the split stages Z in natural order, rows kRowPitch(M) apart.

using regfft::RowTile;

template <int M>
constexpr int row_pitch() {
  return M + 8;
}

template <int T, int V>
constexpr std::size_t row_smem() {
  constexpr std::size_t xs = static_cast<std::size_t>(V) * RowTile<T>::A;
  constexpr std::size_t zs = static_cast<std::size_t>(RowTile<T>::R) * row_pitch<T * V>();
  return (xs > zs ? xs : zs) * sizeof(float2);
}

// The half spectrum of the row from Z (natural order in zs, this row's start), positions k = t + T j and,
// for t = 0, k = M; written to e_row[k].
template <int T, int V>
__device__ __forceinline__ void split_store(const float2* zs, int t, const float2* __restrict__ twn,
                                            float2* __restrict__ e_row) {
  constexpr int M = T * V;
#pragma unroll
  for (int j = 0; j <= V; ++j) {
    const int k = j < V ? t + T * j : M;
    if (j == V && t != 0) break;
    const float2 zk = zs[k == M ? 0 : k];
    const float2 zm = zs[k == 0 ? 0 : M - k];
    const float2 ev = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
    const float2 d = make_float2(zk.x - zm.x, zk.y + zm.y);  // zk - conj(zm)
    const float2 od = make_float2(0.5f * d.y, -0.5f * d.x);   // d / (2i)
    e_row[k] = cadd(ev, cmul(__ldg(twn + k), od));
  }
}

// The merge before a C2R: from e_row[m] and e_row[M - m], the value whose inverse transform gives the
// pairs (2m, 2m + 1), for m = t + T j.
template <int T, int V>
__device__ __forceinline__ void merge_load(const float2* __restrict__ e_row, int t, const float2* __restrict__ twn,
                                           float2 (&v)[V]) {
  constexpr int M = T * V;
  float2 xk[V], xm[V];
#pragma unroll
  for (int j = 0; j < V; ++j) {
    const int m = t + T * j;
    xk[j] = e_row[m];
    xm[j] = e_row[M - m];
  }
#pragma unroll
  for (int j = 0; j < V; ++j) {
    const int m = t + T * j;
    float2 a = xk[j], b = xm[j];
    if (m == 0) {  // a real signal has real bins 0 and M; their imaginary parts drop out
      a.y = 0.0f;
      b.y = 0.0f;
    }
    const float2 sv = make_float2(a.x + b.x, a.y - b.y);  // xk + conj(xm)
    const float2 d = make_float2(a.x - b.x, a.y + b.y);   // xk - conj(xm)
    const float2 tt = cmulc(d, __ldg(twn + m));            // d * e^{+2 pi i m / nx}
    v[j] = make_float2(sv.x - tt.y, sv.y + tt.x);         // sv + i tt
  }
}

template <bool Clamp, int T, int V>
__global__ void __launch_bounds__(kRegThreads)
    k_rows_r2c_reg(const float* __restrict__ x, float2* __restrict__ e, std::size_t rows,
                   const float2* __restrict__ tw, const float2* __restrict__ twn) {
  if (!QHK_CHECK(row_smem<T, V>() <= debug::dynamic_smem_bytes() && blockDim.x == kRegThreads)) return;
  using Tile = RowTile<T>;
  constexpr int M = T * V, h = M + 1, P = row_pitch<M>();
  extern __shared__ float2 sm[];
  const int t = static_cast<int>(threadIdx.x) % T, r = static_cast<int>(threadIdx.x) / T;
  const std::size_t row = static_cast<std::size_t>(blockIdx.x) * Tile::R + r;
  const bool live = row < rows;
  float2 v[V];
#pragma unroll
  for (int j = 0; j < V; ++j) {
    float2 a = live ? *reinterpret_cast<const float2*>(x + row * (2 * M) + 2 * (t + T * j)) : make_float2(0.0f, 0.0f);
    if (Clamp) a = make_float2(fmaxf(a.x, 0.0f), fmaxf(a.y, 0.0f));
    v[j] = a;
  }
  regfft::line_fft<T, V, true>(v, t, sm + r, Tile::A, Tile::B, tw);
  __syncthreads();  // the exchange buffer becomes the natural-order staging
#pragma unroll
  for (int j = 0; j < V; ++j) sm[r * P + t + T * j] = v[j];
  __syncthreads();
  if (live) split_store<T, V>(sm + r * P, t, twn, e + row * h);
}

template <int Mode, int T, int V>
__global__ void __launch_bounds__(kRegThreads)
    k_rows_c2r_reg(const float2* __restrict__ e, float* __restrict__ x, std::size_t rows, const float2* __restrict__ tw,
                   const float2* __restrict__ twn, float nm2, float inv_k02) {
  if (!QHK_CHECK(row_smem<T, V>() <= debug::dynamic_smem_bytes() && blockDim.x == kRegThreads)) return;
  using Tile = RowTile<T>;
  constexpr int M = T * V, h = M + 1;
  extern __shared__ float2 sm[];
  const int t = static_cast<int>(threadIdx.x) % T, r = static_cast<int>(threadIdx.x) / T;
  const std::size_t row = static_cast<std::size_t>(blockIdx.x) * Tile::R + r;
  const bool live = row < rows;
  float2 v[V];
  merge_load<T, V>(e + (live ? row : 0) * h, t, twn, v);
  regfft::line_fft<T, V, false>(v, t, sm + r, Tile::A, Tile::B, tw);
  if (live) {
#pragma unroll
    for (int j = 0; j < V; ++j) {
      float2 z = v[j];
      if (Mode == static_cast<int>(C2rMode::index)) {
        z = make_float2(index_from_potential(z.x, 0.0f, nm2, inv_k02), index_from_potential(z.y, 0.0f, nm2, inv_k02));
      }
      *reinterpret_cast<float2*>(x + row * (2 * M) + 2 * (t + T * j)) = z;
    }
  }
}

// One Gerchberg-Papoulis step boundary on rows, in place: C2R, max(x, 0), R2C (the operations of
// k_rows_c2r_reg then k_rows_r2c_reg<true>), the real rows never leaving the chip.
template <int T, int V>
__global__ void __launch_bounds__(kRegThreads)
    k_rows_c2r_r2c_reg(float2* __restrict__ e, std::size_t rows, const float2* __restrict__ tw,
                       const float2* __restrict__ twn) {
  if (!QHK_CHECK(row_smem<T, V>() <= debug::dynamic_smem_bytes() && blockDim.x == kRegThreads)) return;
  using Tile = RowTile<T>;
  constexpr int M = T * V, h = M + 1, P = row_pitch<M>();
  extern __shared__ float2 sm[];
  const int t = static_cast<int>(threadIdx.x) % T, r = static_cast<int>(threadIdx.x) / T;
  const std::size_t row = static_cast<std::size_t>(blockIdx.x) * Tile::R + r;
  const bool live = row < rows;
  float2 v[V];
  merge_load<T, V>(e + (live ? row : 0) * h, t, twn, v);
  regfft::line_fft<T, V, false>(v, t, sm + r, Tile::A, Tile::B, tw);
#pragma unroll
  for (int j = 0; j < V; ++j) v[j] = live ? make_float2(fmaxf(v[j].x, 0.0f), fmaxf(v[j].y, 0.0f)) : make_float2(0.0f, 0.0f);
  __syncthreads();
  regfft::line_fft<T, V, true>(v, t, sm + r, Tile::A, Tile::B, tw);
  __syncthreads();
#pragma unroll
  for (int j = 0; j < V; ++j) sm[r * P + t + T * j] = v[j];
  __syncthreads();
  if (live) split_store<T, V>(sm + r * P, t, twn, e + row * h);
}

template <class K>
void row_smem_attr(K kernel, std::size_t smem) {
  ensure_smem(kernel);
}

// Calls f.template operator()<T, V>() for the half-spectrum length M the register engine covers;
// false when it does not.
template <class F>
bool with_row_shape(int M, F&& f) {
  if (!fft_reg_engine_enabled()) return false;
  switch (M) {
    case 64: f.template operator()<8, 8>(); return true;
    case 128: f.template operator()<8, 16>(); return true;
    case 192: f.template operator()<8, 24>(); return true;
    case 256: f.template operator()<16, 16>(); return true;
    default: return false;
  }
}

}  // namespace

bool rows_r2c_reg(const float* x, float2* e, std::size_t rows, int nx, bool clamp, cudaStream_t s) {
  return with_row_shape(nx / 2, [&]<int T, int V>() {
    const std::size_t smem = row_smem<T, V>();
    const unsigned grid = static_cast<unsigned>((rows + RowTile<T>::R - 1) / RowTile<T>::R);
    const float2* tw = fft_len(T * V).tw;
    const float2* twn = fft_len(nx).tw;
    if (clamp) {
      row_smem_attr(k_rows_r2c_reg<true, T, V>, smem);
      k_rows_r2c_reg<true, T, V><<<grid, kRegThreads, smem, s>>>(x, e, rows, tw, twn);
    } else {
      row_smem_attr(k_rows_r2c_reg<false, T, V>, smem);
      k_rows_r2c_reg<false, T, V><<<grid, kRegThreads, smem, s>>>(x, e, rows, tw, twn);
    }
    check_launch("rows r2c");
  });
}

bool rows_c2r_reg(const float2* e, float* x, std::size_t rows, int nx, C2rMode mode, float nm2, float inv_k02,
                  cudaStream_t s) {
  return with_row_shape(nx / 2, [&]<int T, int V>() {
    const std::size_t smem = row_smem<T, V>();
    const unsigned grid = static_cast<unsigned>((rows + RowTile<T>::R - 1) / RowTile<T>::R);
    const float2* tw = fft_len(T * V).tw;
    const float2* twn = fft_len(nx).tw;
    if (mode == C2rMode::index) {
      row_smem_attr(k_rows_c2r_reg<1, T, V>, smem);
      k_rows_c2r_reg<1, T, V><<<grid, kRegThreads, smem, s>>>(e, x, rows, tw, twn, nm2, inv_k02);
    } else {
      row_smem_attr(k_rows_c2r_reg<0, T, V>, smem);
      k_rows_c2r_reg<0, T, V><<<grid, kRegThreads, smem, s>>>(e, x, rows, tw, twn, nm2, inv_k02);
    }
    check_launch("rows c2r");
  });
}

bool rows_c2r_r2c_reg(float2* e, std::size_t rows, int nx, cudaStream_t s) {
  return with_row_shape(nx / 2, [&]<int T, int V>() {
    const std::size_t smem = row_smem<T, V>();
    const unsigned grid = static_cast<unsigned>((rows + RowTile<T>::R - 1) / RowTile<T>::R);
    row_smem_attr(k_rows_c2r_r2c_reg<T, V>, smem);
    k_rows_c2r_r2c_reg<T, V><<<grid, kRegThreads, smem, s>>>(e, rows, fft_len(T * V).tw, fft_len(nx).tw);
    check_launch("rows c2r r2c");
  });
}

bool fft_reg_engine_enabled() {
  // QHK_FFT_ENGINE=staged keeps every pass on the staged shared-memory engine (for comparisons).
  static const bool on = [] {
    const char* e = std::getenv("QHK_FFT_ENGINE");
    return !(e && std::strcmp(e, "staged") == 0);
  }();
  return on;
}

int axis_reg_variants(int n) {
  if (!fft_reg_engine_enabled()) return 0;
  switch (n) {
    case 64: case 128: case 256: return 2;
    case 192: case 512: return 1;
    default: return 0;
  }
}

// Variant 1 (the default) and variant 2 (fewer threads per line, longer per-thread DFTs) of the register
// engine's decomposition N = T V for each length it covers.
bool axis_pass_reg(float2* data, int n_outer, std::size_t so, int n, std::size_t sp, int ni, bool forward,
                   AxisMode mode, float scale, const AxisAux& aux, cudaStream_t s, int batch, std::size_t sb,
                   int variant) {
  if (variant < 1 || variant > axis_reg_variants(n)) return false;
  const bool alt = variant == 2;
  switch (n) {
    case 64:
      if (alt) {
        axis_reg_mode<4, 16>(data, n_outer, so, sp, ni, forward, mode, scale, aux, batch, sb, s);
      } else {
        axis_reg_mode<8, 8>(data, n_outer, so, sp, ni, forward, mode, scale, aux, batch, sb, s);
      }
      return true;
    case 128:
      if (alt) {
        axis_reg_mode<4, 32>(data, n_outer, so, sp, ni, forward, mode, scale, aux, batch, sb, s);
      } else {
        axis_reg_mode<8, 16>(data, n_outer, so, sp, ni, forward, mode, scale, aux, batch, sb, s);
      }
      return true;
    case 192: axis_reg_mode<8, 24>(data, n_outer, so, sp, ni, forward, mode, scale, aux, batch, sb, s); return true;
    case 256:
      if (alt) {
        axis_reg_mode<8, 32>(data, n_outer, so, sp, ni, forward, mode, scale, aux, batch, sb, s);
      } else {
        axis_reg_mode<16, 16>(data, n_outer, so, sp, ni, forward, mode, scale, aux, batch, sb, s);
      }
      return true;
    case 512: axis_reg_mode<16, 32>(data, n_outer, so, sp, ni, forward, mode, scale, aux, batch, sb, s); return true;
    default: return false;
  }
}

}  // namespace qhk
