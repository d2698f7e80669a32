// Register-resident FFT of lines of length N = T * V held by T threads with V values each.
//
// Thread t of a line owns positions t + T j, j = 0 .. V-1, before and after the transform, so the
// caller loads and stores the same pattern (consecutive threads on consecutive lines at one position:
// coalesced rows of a tile of lines). With n = t + T j and k = k1 + V k2 (k1 < V, k2 < T):
//
//   X[k1 + V k2] = sum_t W_T^{t k2} W_N^{t k1} sum_j W_V^{j k1} x[t + T j]
//
// step 1: each thread a length-V DFT over its own values (j -> k1), then the twiddle W_N^{t k1};
// exchange: through shared memory, after which every thread holds, for its V / T bins k1 = t + T i,
// the values of all T threads of the line;
// step 2: each thread V / T length-T DFTs (t -> k2), whose output X[k1 + V k2] is position
// t + T (i + (V / T) k2) -- the thread's own positions again. V must be a multiple of T.
//
// One shared-memory round trip and one barrier per transform, against a write and a read of shared
// memory per radix pass in the staged Stockham engine (fft_engine.cuh). Forward sign e^{-2 pi i / N};
// the inverse is unnormalised.
#pragma once

#include <cuda_runtime.h>

#include "debug.cuh"
#include "fft_engine.cuh"

namespace qhk {
namespace regfft {

// cos(2 pi q / 32) and -sin(2 pi q / 32), q = 0..31 (e^{-2 pi i q / 32}); q is a constant after unrolling,
// so the lookup folds to an immediate.
__device__ __forceinline__ float w32_re(int q) {
  constexpr float c[8] = {1.0f, 0.98078528040323044913f, 0.92387953251128675613f, 0.83146961230254523708f,
                          0.70710678118654752440f, 0.55557023301960222474f, 0.38268343236508977173f,
                          0.19509032201612826785f};
  // cos(2 pi q / 32) from the first octant by the symmetries of the circle.
  q &= 31;
  if (q == 8 || q == 24) return 0.0f;
  if (q < 8) return c[q];
  if (q <= 16) return -c[16 - q];
  if (q < 24) return -c[q - 16];
  return c[32 - q];
}
__device__ __forceinline__ float w32_im(int q) { return -w32_re(q + 24); }  // -sin(a) = cos(a + 3 pi / 2)

// cos(2 pi q / 24), q = 0..23, from the quarter wave (0, 15, ..., 90 degrees) by symmetry.
__device__ __forceinline__ float w24_re(int q) {
  constexpr float c[7] = {1.0f, 0.96592582628906828675f, 0.86602540378443864676f, 0.70710678118654752440f,
                          0.5f, 0.25881904510252076235f, 0.0f};
  q %= 24;
  if (q <= 6) return c[q];
  if (q <= 12) return -c[12 - q];
  if (q <= 18) return -c[q - 12];
  return c[24 - q];
}
__device__ __forceinline__ float w24_im(int q) { return -w24_re(q + 18); }  // -sin(a) = cos(a + 3 pi / 2)

// v * W_R^m, W_R = e^{-2 pi i / R} (its conjugate for the inverse), R a divisor of 32 or of 24. Called
// with R and m constant after unrolling, so the factors 1, -i, -1, i cost no multiplication and the
// others are immediates.
template <bool Fwd>
__device__ __forceinline__ float2 wmul(float2 v, int R, int m) {
  const bool of32 = 32 % R == 0;
  const int L = of32 ? 32 : 24;
  const int q = (m % R) * (L / R);  // the same root as a power of W_L
  if (q == 0) return v;
  if (2 * q == L) return make_float2(-v.x, -v.y);
  if (4 * q == L) return Fwd ? make_float2(v.y, -v.x) : make_float2(-v.y, v.x);
  if (4 * q == 3 * L) return Fwd ? make_float2(-v.y, v.x) : make_float2(v.y, -v.x);
  const float c = of32 ? w32_re(q) : w24_re(q);
  const float s = (Fwd ? 1.0f : -1.0f) * (of32 ? w32_im(q) : w24_im(q));
  return make_float2(v.x * c - v.y * s, v.x * s + v.y * c);
}

template <int R, bool Fwd>
__device__ __forceinline__ void dft(float2* v);

// Length N1 * N2 as N2-point DFTs over n2 (n = n1 + N1 n2), twiddles W_N^{n1 k1}, N1-point DFTs over
// n1; output k = k1 + N2 k2 in place.
template <int N1, int N2, bool Fwd>
__device__ __forceinline__ void dft_split(float2* v) {
  constexpr int N = N1 * N2;
  float2 a[N1][N2];
#pragma unroll
  for (int n1 = 0; n1 < N1; ++n1) {
#pragma unroll
    for (int n2 = 0; n2 < N2; ++n2) a[n1][n2] = v[n1 + N1 * n2];
    dft<N2, Fwd>(a[n1]);
  }
#pragma unroll
  for (int k1 = 0; k1 < N2; ++k1) {
    float2 b[N1];
#pragma unroll
    for (int n1 = 0; n1 < N1; ++n1) b[n1] = wmul<Fwd>(a[n1][k1], N, n1 * k1);
    dft<N1, Fwd>(b);
#pragma unroll
    for (int k2 = 0; k2 < N1; ++k2) v[k1 + N2 * k2] = b[k2];
  }
}

template <int R, bool Fwd>
__device__ __forceinline__ void dft(float2* v) {
  if constexpr (R == 1) {
  } else if constexpr (R == 2) {
    fftdev::dft2<Fwd>(v);
  } else if constexpr (R == 3) {
    fftdev::dft3<Fwd>(v);
  } else if constexpr (R == 4) {
    fftdev::dft4<Fwd>(v[0], v[1], v[2], v[3]);
  } else if constexpr (R == 8) {
    fftdev::dft8<Fwd>(v);
  } else if constexpr (R == 16) {
    dft_split<4, 4, Fwd>(v);
  } else if constexpr (R == 24) {
    dft_split<3, 8, Fwd>(v);
  } else {
    static_assert(R == 32, "register DFT lengths: 1, 2, 3, 4, 8, 16, 24, 32");
    dft_split<4, 8, Fwd>(v);
  }
}

// The transform of one line, T threads of V values (see the header comment). `v` holds x[t + T j] on
// entry and X[t + T j] on return. `xs` is this line's exchange buffer: element (k1, s) -- bin k1 of
// thread s -- at xs[k1 * A + s * B]; lines of a tile interleave (the caller offsets `xs` per line), and
// A, B are chosen per tile shape so that the writes (k1 fixed) and the reads (s fixed) of a warp fall
// on distinct banks. tw[i * tws] is e^{-2 pi i i / N}, i < N (tws = 2 reads a length-2N table, whose
// even entries are exactly those of the length-N one). All threads of the CTA call it together: it
// synchronises before the exchange reads, and the caller must synchronise before writing `xs` again.
template <int T, int V, bool Fwd>
__device__ __forceinline__ void line_fft(float2 (&v)[V], int t, float2* xs, int A, int B, const float2* tw,
                                         int tws = 1) {
  static_assert(V % T == 0, "register FFT: V must be a multiple of T");
  constexpr int N = T * V;
  dft<V, Fwd>(v);
#pragma unroll
  for (int k1 = 1; k1 < V; ++k1) {
    const float2 w = __ldg(tw + ((t * k1) % N) * tws);
    v[k1] = cmul(v[k1], Fwd ? w : make_float2(w.x, -w.y));
  }
#pragma unroll
  for (int k1 = 0; k1 < V; ++k1) xs[k1 * A + t * B] = v[k1];
  __syncthreads();
  constexpr int P = V / T;
#pragma unroll
  for (int i = 0; i < P; ++i) {
    float2 u[T];
    const int k1 = t + T * i;
#pragma unroll
    for (int s = 0; s < T; ++s) u[s] = xs[k1 * A + s * B];
    dft<T, Fwd>(u);
#pragma unroll
    for (int k2 = 0; k2 < T; ++k2) v[i + P * k2] = u[k2];
  }
}

// Exchange strides for tiles of rows: 256 threads, T per row (consecutive threads on consecutive positions
// of a row), R = 256 / T rows. A 64-bit shared-memory access is served per half-warp, 16 threads over the
// 16 two-bank slots: with T = 4 a half-warp spans 4 threads of 4 rows, with T = 8 8 threads of 2 rows,
// with T = 16 16 threads of one row. B (per thread) and A (per bin) are chosen so that t * B + r and
// t * A + r fall on 16 distinct slots within every half-warp, in the writes and in the reads of the
// exchange (B and A congruent to 16 / T times an odd number modulo 16, rows r0 .. r0 + 16 / T - 1 with r0 a
// multiple of 16 / T), and so that B >= R and A >= T * B (the (bin, thread, row) elements do not overlap).
// True when t * S + r lands on 16 distinct two-bank slots over one half-warp: T threads of 16 / T rows.
constexpr bool half_warp_distinct(int T, int S) {
  bool seen[16] = {};
  for (int t = 0; t < T; ++t) {
    for (int r = 0; r < 16 / T; ++r) {
      const int slot = (t * S + r) % 16;
      if (seen[slot]) return false;
      seen[slot] = true;
    }
  }
  return true;
}

template <int T>
struct RowTile {
  static_assert(T == 4 || T == 8 || T == 16, "row tiles of 4, 8 or 16 threads per row");
  static constexpr int R = 256 / T;
  static constexpr int B = T == 4 ? 68 : T == 8 ? 34 : 17;
  static constexpr int A = T == 4 ? 4 * 68 + 4 : T == 8 ? 8 * 34 + 2 : 16 * 17 + 1;
  static_assert(B >= R && A >= T * B, "row tile exchange elements overlap");
  static_assert(half_warp_distinct(T, B) && half_warp_distinct(T, A), "row tile exchange has bank conflicts");
};

}  // namespace regfft
}  // namespace qhk
