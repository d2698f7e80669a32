// Shared-memory FFT engine: mixed-radix Stockham autosort (decimation in time) over lines held in
// shared memory. A CTA stages a tile of lines from HBM, runs every pass in shared memory and
// writes the tile back, so each HBM pass of a transform reads and writes its data once; the
// callers fuse their pointwise neighbours (crop, clamp, k-space restore, demodulation, Rytov
// assembly) into that load and store.
//
// Layout in shared memory: element `pos` of line `col` at a[pos * cp + col], so the threads of a
// warp touch consecutive columns (bank-conflict free for cp = COLS or an odd pitch).
// Pass (ns, R) maps butterfly j (k = j mod ns) from positions j + q n/R to (j - k) R + k + q ns,
// twiddled by W_n^{k q n/(ns R)}, with W_n = e^{-2 pi i / n} for the forward sign. Radix 8, 4, 2,
// 3, 5 have straight-line butterflies; any other prime factor uses a direct DFT.
#pragma once

#include <cuda_runtime.h>

#include "qhk_math.cuh"

namespace qhk {

constexpr int kMaxPasses = 16;

// One transform length: its radix sequence and the twiddle table e^{-2 pi i k / n}, k < n.
struct FftLen {
  int n = 0;
  int passes = 0;
  int radix[kMaxPasses] = {};
  const float2* tw = nullptr;
};

// Radix sequence for n: 8s first, then one 4 or 2, then 3, 5 and any other primes.
FftLen make_fft_len(int n);

namespace fftdev {

template <bool Fwd>
__device__ __forceinline__ float2 twiddle(const float2* tw, int idx) {
  const float2 w = __ldg(tw + idx);
  return Fwd ? w : make_float2(w.x, -w.y);
}

// i * s * v with s = -1 forward, +1 inverse.
template <bool Fwd>
__device__ __forceinline__ float2 rot(float2 v) {
  return Fwd ? make_float2(v.y, -v.x) : make_float2(-v.y, v.x);
}

template <bool Fwd>
__device__ __forceinline__ void dft2(float2* v) {
  const float2 a = v[0], b = v[1];
  v[0] = cadd(a, b);
  v[1] = csub(a, b);
}

template <bool Fwd>
__device__ __forceinline__ void dft4(float2& x0, float2& x1, float2& x2, float2& x3) {
  const float2 a0 = cadd(x0, x2), a1 = csub(x0, x2);
  const float2 b0 = cadd(x1, x3), b1 = rot<Fwd>(csub(x1, x3));
  x0 = cadd(a0, b0);
  x2 = csub(a0, b0);
  x1 = cadd(a1, b1);
  x3 = csub(a1, b1);
}

template <bool Fwd>
__device__ __forceinline__ void dft8(float2* v) {
  // Radix-2 split of a length-8 DFT into two length-4 DFTs of the even and odd samples.
  float2 e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
  float2 o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
  dft4<Fwd>(e0, e1, e2, e3);
  dft4<Fwd>(o0, o1, o2, o3);
  const float h = 0.70710678118654752440f;
  // w8^1 o1, w8^2 o2, w8^3 o3 with w8 = e^{-/+ i pi / 4}
  const float2 t1 = Fwd ? make_float2(h * (o1.x + o1.y), h * (o1.y - o1.x))
                        : make_float2(h * (o1.x - o1.y), h * (o1.y + o1.x));
  const float2 t2 = rot<Fwd>(o2);
  const float2 t3 = Fwd ? make_float2(h * (o3.y - o3.x), -h * (o3.x + o3.y))
                        : make_float2(-h * (o3.x + o3.y), h * (o3.x - o3.y));
  v[0] = cadd(e0, o0);
  v[4] = csub(e0, o0);
  v[1] = cadd(e1, t1);
  v[5] = csub(e1, t1);
  v[2] = cadd(e2, t2);
  v[6] = csub(e2, t2);
  v[3] = cadd(e3, t3);
  v[7] = csub(e3, t3);
}

template <bool Fwd>
__device__ __forceinline__ void dft3(float2* v) {
  const float sn = 0.86602540378443864676f;
  const float2 t1 = cadd(v[1], v[2]);
  const float2 t2 = make_float2(v[0].x - 0.5f * t1.x, v[0].y - 0.5f * t1.y);
  const float2 t3 = rot<Fwd>(csub(v[1], v[2]));
  const float2 t4 = cscale(t3, sn);
  v[0] = cadd(v[0], t1);
  v[1] = cadd(t2, t4);
  v[2] = csub(t2, t4);
}

template <bool Fwd>
__device__ __forceinline__ void dft5(float2* v) {
  const float c1 = 0.30901699437494742410f, c2 = -0.80901699437494742410f;
  const float s1 = 0.95105651629515357212f, s2 = 0.58778525229247312917f;
  const float2 t1 = cadd(v[1], v[4]), t2 = cadd(v[2], v[3]);
  const float2 t3 = csub(v[1], v[4]), t4 = csub(v[2], v[3]);
  const float2 b1 = make_float2(v[0].x + c1 * t1.x + c2 * t2.x, v[0].y + c1 * t1.y + c2 * t2.y);
  const float2 b2 = make_float2(v[0].x + c2 * t1.x + c1 * t2.x, v[0].y + c2 * t1.y + c1 * t2.y);
  // i s (s1 t3 + s2 t4) and i s (s2 t3 - s1 t4)
  const float2 d1 = rot<Fwd>(make_float2(s1 * t3.x + s2 * t4.x, s1 * t3.y + s2 * t4.y));
  const float2 d2 = rot<Fwd>(make_float2(s2 * t3.x - s1 * t4.x, s2 * t3.y - s1 * t4.y));
  v[0] = cadd(v[0], cadd(t1, t2));
  v[1] = cadd(b1, d1);
  v[4] = csub(b1, d1);
  v[2] = cadd(b2, d2);
  v[3] = csub(b2, d2);
}

template <int R, bool Fwd>
__device__ __forceinline__ void dft(float2* v) {
  if constexpr (R == 2) {
    dft2<Fwd>(v);
  } else if constexpr (R == 3) {
    dft3<Fwd>(v);
  } else if constexpr (R == 4) {
    dft4<Fwd>(v[0], v[1], v[2], v[3]);
  } else if constexpr (R == 5) {
    dft5<Fwd>(v);
  } else {
    dft8<Fwd>(v);
  }
}

// One Stockham pass of radix R over `cols` lines: src -> dst.
template <int R, bool Fwd>
__device__ __forceinline__ void pass(const float2* src, float2* dst, int cp, int cols, int n, int ns,
                                     const float2* tw, int tid, int nth) {
  const int m = n / R;
  const int tws = n / (ns * R);
  const int total = m * cols;
  for (int t = tid; t < total; t += nth) {
    const int col = t % cols;
    const int j = t / cols;
    const int k = j % ns;
    float2 v[R];
#pragma unroll
    for (int q = 0; q < R; ++q) v[q] = src[(j + q * m) * cp + col];
    if (k) {
#pragma unroll
      for (int q = 1; q < R; ++q) v[q] = cmul(v[q], twiddle<Fwd>(tw, k * q * tws));
    }
    dft<R, Fwd>(v);
    const int base = (j - k) * R + k;
#pragma unroll
    for (int q = 0; q < R; ++q) dst[(base + q * ns) * cp + col] = v[q];
  }
}

// A pass with a prime radix R not handled above: direct DFT reading its inputs from src.
template <bool Fwd>
__device__ void pass_generic(const float2* src, float2* dst, int cp, int cols, int n, int ns, int R,
                             const float2* tw, int tid, int nth) {
  const int m = n / R;
  const int tws = n / (ns * R);
  const int total = m * cols;
  for (int t = tid; t < total; t += nth) {
    const int col = t % cols;
    const int j = t / cols;
    const int k = j % ns;
    const int base = (j - k) * R + k;
    for (int o = 0; o < R; ++o) {
      float2 acc = make_float2(0.0f, 0.0f);
      for (int q = 0; q < R; ++q) {
        float2 x = src[(j + q * m) * cp + col];
        if (k && q) x = cmul(x, twiddle<Fwd>(tw, k * q * tws));
        acc = cadd(acc, cmul(x, twiddle<Fwd>(tw, ((q * o) % R) * m)));
      }
      dst[(base + o * ns) * cp + col] = acc;
    }
  }
}

}  // namespace fftdev

// Transforms `cols` lines of length L.n held in `a` (pitch cp), using `b` as the other buffer of
// the ping-pong. All threads of the CTA take part; the caller synchronises before the call
// (after staging) and the function synchronises after every pass. Returns the buffer that holds
// the result (a or b).
template <bool Fwd>
__device__ float2* smem_fft(float2* a, float2* b, int cp, int cols, const FftLen& L, int tid, int nth) {
  int ns = 1;
  for (int s = 0; s < L.passes; ++s) {
    const int R = L.radix[s];
    switch (R) {
      case 8: fftdev::pass<8, Fwd>(a, b, cp, cols, L.n, ns, L.tw, tid, nth); break;
      case 4: fftdev::pass<4, Fwd>(a, b, cp, cols, L.n, ns, L.tw, tid, nth); break;
      case 2: fftdev::pass<2, Fwd>(a, b, cp, cols, L.n, ns, L.tw, tid, nth); break;
      case 3: fftdev::pass<3, Fwd>(a, b, cp, cols, L.n, ns, L.tw, tid, nth); break;
      case 5: fftdev::pass<5, Fwd>(a, b, cp, cols, L.n, ns, L.tw, tid, nth); break;
      default: fftdev::pass_generic<Fwd>(a, b, cp, cols, L.n, ns, R, L.tw, tid, nth); break;
    }
    __syncthreads();
    float2* t = a;
    a = b;
    b = t;
    ns *= R;
  }
  return a;
}

// ---- Compile-time lengths -----------------------------------------------------------------------
// The same passes with the length, the radix sequence and every pass's stride known at compile
// time, so all index arithmetic is by constants. Used for the common lengths; others take the
// runtime engine above.

struct RadixSeq {
  int r[kMaxPasses] = {};
  int count = 0;
};

constexpr RadixSeq radix_seq(int n) {
  RadixSeq s{};
  int m = n;
  while (m % 8 == 0) {
    s.r[s.count++] = 8;
    m /= 8;
  }
  if (m % 4 == 0) {
    s.r[s.count++] = 4;
    m /= 4;
  }
  if (m % 2 == 0) {
    s.r[s.count++] = 2;
    m /= 2;
  }
  while (m % 3 == 0) {
    s.r[s.count++] = 3;
    m /= 3;
  }
  while (m % 5 == 0) {
    s.r[s.count++] = 5;
    m /= 5;
  }
  return s;
}

namespace fftdev {

template <int N, int R, int NS, bool Fwd, int COLS>
__device__ __forceinline__ void pass_fixed(const float2* src, float2* dst, int cp, const float2* tw, int tid,
                                           int nth) {
  constexpr int m = N / R;
  constexpr int tws = N / (NS * R);
  constexpr int total = m * COLS;
  for (int t = tid; t < total; t += nth) {
    const int col = t % COLS;
    const int j = t / COLS;
    const int k = j % NS;
    float2 v[R];
#pragma unroll
    for (int q = 0; q < R; ++q) v[q] = src[(j + q * m) * cp + col];
    if (NS > 1 && k) {
#pragma unroll
      for (int q = 1; q < R; ++q) v[q] = cmul(v[q], twiddle<Fwd>(tw, k * q * tws));
    }
    dft<R, Fwd>(v);
    const int base = (j - k) * R + k;
#pragma unroll
    for (int q = 0; q < R; ++q) dst[(base + q * NS) * cp + col] = v[q];
  }
}

template <int N, int S, int NS, bool Fwd, int COLS>
__device__ __forceinline__ float2* passes_fixed(float2* a, float2* b, int cp, const float2* tw, int tid, int nth) {
  constexpr RadixSeq seq = radix_seq(N);
  if constexpr (S == seq.count) {
    return a;
  } else {
    constexpr int R = seq.r[S];
    pass_fixed<N, R, NS, Fwd, COLS>(a, b, cp, tw, tid, nth);
    __syncthreads();
    return passes_fixed<N, S + 1, NS * R, Fwd, COLS>(b, a, cp, tw, tid, nth);
  }
}

}  // namespace fftdev

// Lines of length L.n in `a` (pitch cp, COLS lines), result buffer returned; specialised for the
// common lengths.
template <bool Fwd, int COLS>
__device__ float2* smem_fft_cols(float2* a, float2* b, int cp, const FftLen& L, int tid, int nth) {
  switch (L.n) {
    case 64: return fftdev::passes_fixed<64, 0, 1, Fwd, COLS>(a, b, cp, L.tw, tid, nth);
    case 128: return fftdev::passes_fixed<128, 0, 1, Fwd, COLS>(a, b, cp, L.tw, tid, nth);
    case 192: return fftdev::passes_fixed<192, 0, 1, Fwd, COLS>(a, b, cp, L.tw, tid, nth);
    case 256: return fftdev::passes_fixed<256, 0, 1, Fwd, COLS>(a, b, cp, L.tw, tid, nth);
    case 384: return fftdev::passes_fixed<384, 0, 1, Fwd, COLS>(a, b, cp, L.tw, tid, nth);
    case 512: return fftdev::passes_fixed<512, 0, 1, Fwd, COLS>(a, b, cp, L.tw, tid, nth);
    case 1024: return fftdev::passes_fixed<1024, 0, 1, Fwd, COLS>(a, b, cp, L.tw, tid, nth);
    default: return smem_fft<Fwd>(a, b, cp, COLS, L, tid, nth);
  }
}

}  // namespace qhk
