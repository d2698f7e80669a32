// Off-axis hologram -> complex field on the device: FFT, circular crop around the sideband
// centre, inverse FFT at the output size. Replaces the reference's FieldStage (src/cuda/field.cu,
// src/cuda/stages.cuh:19-47) and follows cpu::extract_fields (src/cpu/field.cpp:78-121).
//
// Only the spectrum inside the crop disc is ever needed, so the forward transform is pruned:
//   1. rows: real rows -> half spectra by a half-length complex FFT; only the W columns of the
//      crop window are written (a negative kx is read as the conjugate of +kx, which is exact for
//      the row transform of real data);
//   2. columns: N-point forward FFT along y of those W columns, the disc mask and the
//      centre-origin sign, then the m-point inverse FFT along y, in one launch;
//   3. rows: m-point inverse FFT along x of the W nonzero columns, then (-1)^(x+y) / N^2
//      (demodulation), or -- for the Pipeline -- the ratio to the resident background field and its
//      phase and log-amplitude.
#include <cmath>

#include "field.hpp"

namespace qhk {

namespace {

constexpr int kThreads = 256;

// Pass 1. Rows of real holograms (length N), COLS rows per CTA; writes t1[row][j] = H_row(fx),
// fx = cx + dxlo + j, for j < W (zero if fx is outside [-N/2, N/2)).
template <int COLS>
__global__ void __launch_bounds__(kThreads)
    k_holo_rows(const float* __restrict__ holo, float2* __restrict__ t1, std::size_t rows, int N, FftLen Lm,
                const float2* __restrict__ twn, int fx0, int W) {
  extern __shared__ float2 sm[];
  constexpr int cp = COLS + 1;
  const int M = Lm.n;
  float2* A = sm;
  float2* B = sm + static_cast<std::size_t>(M + 1) * cp;
  const std::size_t r0 = static_cast<std::size_t>(blockIdx.x) * COLS;
  const int nr = static_cast<int>(min(static_cast<std::size_t>(COLS), rows - r0));
  const int tid = static_cast<int>(threadIdx.x), nth = static_cast<int>(blockDim.x);
  for (int idx = tid; idx < M * COLS; idx += nth) {
    const int row = idx / M;
    const int m = idx - row * M;
    A[m * cp + row] = row < nr ? *reinterpret_cast<const float2*>(holo + (r0 + row) * N + 2 * m) : make_float2(0.f, 0.f);
  }
  __syncthreads();
  const float2* res = smem_fft_cols<true, COLS>(A, B, cp, Lm, tid, nth);
  for (int idx = tid; idx < W * COLS; idx += nth) {
    const int row = idx / W;
    const int j = idx - row * W;
    if (row >= nr) continue;
    const int fx = fx0 + j;
    float2 v = make_float2(0.0f, 0.0f);
    if (fx >= -N / 2 && fx < N / 2) {
      const int k = fx >= 0 ? fx : -fx;
      const float2 zk = res[(k == M ? 0 : k) * cp + row];
      const float2 zm = res[(k == 0 ? 0 : M - k) * cp + row];
      const float2 ev = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
      const float2 d = make_float2(zk.x - zm.x, zk.y + zm.y);
      const float2 od = make_float2(0.5f * d.y, -0.5f * d.x);
      v = cadd(ev, cmul(__ldg(twn + k), od));
      if (fx < 0) v.y = -v.y;
    }
    t1[(r0 + row) * W + j] = v;
  }
}

// Pass 2. Columns of t1 (N along y, W columns per image), COLS columns per CTA: forward N-point
// FFT, crop (rows dy in [dylo, dyhi] at output row m/2 + dy), inverse m-point FFT; t2 is
// (count, m, W).
template <int COLS>
__global__ void __launch_bounds__(kThreads)
    k_holo_cols(const float2* __restrict__ t1, float2* __restrict__ t2, int N, int m, int W, FftLen Ln, FftLen Lmo,
                int cy, int cx, int dxlo, float r2, float sign) {
  extern __shared__ float2 sm[];
  const int big = N > m ? N : m;
  float2* A = sm;
  float2* B = sm + static_cast<std::size_t>(big) * COLS;
  const int c0 = static_cast<int>(blockIdx.x) * COLS;
  const int cols = min(COLS, W - c0);
  const std::size_t img = blockIdx.y;
  const int tid = static_cast<int>(threadIdx.x), nth = static_cast<int>(blockDim.x);
  const float2* src = t1 + img * N * W + c0;
  for (int idx = tid; idx < N * COLS; idx += nth) {
    const int pos = idx / COLS;
    const int col = idx - pos * COLS;
    A[idx] = col < cols ? src[static_cast<std::size_t>(pos) * W + col] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  float2* res = smem_fft_cols<true, COLS>(A, B, COLS, Ln, tid, nth);
  float2* C = res == A ? B : A;
  for (int idx = tid; idx < m * COLS; idx += nth) {
    const int jy = idx / COLS;
    const int col = idx - jy * COLS;
    const int dy = jy - m / 2;
    const int dx = dxlo + c0 + col;
    const int fy = cy + dy;
    const int fx = cx + dx;
    float2 v = make_float2(0.0f, 0.0f);
    if (col < cols && static_cast<float>(dy * dy + dx * dx) <= r2 && fy >= -N / 2 && fy < N / 2 && fx >= -N / 2 &&
        fx < N / 2) {
      v = cscale(res[((fy + N) % N) * COLS + col], sign);
    }
    C[idx] = v;
  }
  __syncthreads();
  const float2* out = smem_fft_cols<false, COLS>(C, res, COLS, Lmo, tid, nth);
  float2* dst = t2 + img * m * W + c0;
  for (int idx = tid; idx < m * COLS; idx += nth) {
    const int pos = idx / COLS;
    const int col = idx - pos * COLS;
    if (col < cols) dst[static_cast<std::size_t>(pos) * W + col] = out[idx];
  }
}

// Pass 3. Output rows (count * m rows of m), COLS rows per CTA: place the W columns at
// m/2 + dxlo + j, inverse m-point FFT along x, then the epilogue of `Mode`.
//   0: field = v * (-1)^(x+y) / N^2
//   1: ratio to `bg` (a demodulated field; stacks of several requests reuse the bg_rows rows of one
//      geometry's backgrounds) -> psi = arg, logamp = log |.|
template <int Mode, int COLS>
__global__ void __launch_bounds__(kThreads)
    k_field_rows(const float2* __restrict__ t2, std::size_t rows, int m, int W, int x0, FftLen Lmo, float inv_nn,
                 float2* __restrict__ field, const float2* __restrict__ bg, float* __restrict__ psi,
                 float* __restrict__ logamp, std::size_t bg_rows) {
  extern __shared__ float2 sm[];
  constexpr int cp = COLS + 1;
  float2* A = sm;
  float2* B = sm + static_cast<std::size_t>(m) * cp;
  const std::size_t r0 = static_cast<std::size_t>(blockIdx.x) * COLS;
  const int nr = static_cast<int>(min(static_cast<std::size_t>(COLS), rows - r0));
  const int tid = static_cast<int>(threadIdx.x), nth = static_cast<int>(blockDim.x);
  __shared__ std::size_t bg_row[COLS];  // first background element of each row
  if (Mode == 1 && tid < COLS) bg_row[tid] = ((r0 + tid) % bg_rows) * m;
  for (int idx = tid; idx < m * COLS; idx += nth) A[idx + idx / COLS] = make_float2(0.f, 0.f);  // pitch cp
  __syncthreads();
  for (int idx = tid; idx < W * COLS; idx += nth) {
    const int row = idx / W;
    const int j = idx - row * W;
    if (row < nr) A[(x0 + j) * cp + row] = t2[(r0 + row) * W + j];
  }
  __syncthreads();
  const float2* res = smem_fft_cols<false, COLS>(A, B, cp, Lmo, tid, nth);
  for (int idx = tid; idx < m * COLS; idx += nth) {
    const int row = idx / m;
    const int x = idx - row * m;
    if (row >= nr) continue;
    const std::size_t g = (r0 + row) * m + x;
    const int y = static_cast<int>((r0 + row) % m);
    const float2 v = cscale(res[x * cp + row], inv_nn * parity(x + y));
    if constexpr (Mode == 0) {
      field[g] = v;
    } else {
      const float2 b = bg[bg_row[row] + x];  // the background stack repeats every bg_rows rows
      const float d = 1.0f / (b.x * b.x + b.y * b.y);
      const float re = (v.x * b.x + v.y * b.y) * d;
      const float im = (v.y * b.x - v.x * b.y) * d;
      psi[g] = atan2f(im, re);
      logamp[g] = logf(hypotf(re, im));
    }
  }
}

int rows_per_cta(int len) {
  int c = 16;
  while (c > 1 && 2 * static_cast<std::size_t>(len + 1) * (c + 1) * sizeof(float2) > 64 * 1024) c /= 2;
  return c;
}

template <class K>
void allow(K kernel, std::size_t) {
  ensure_smem(kernel);
}

}  // namespace

CropPlan make_crop(int n, float cy, float cx, float radius, int output_size) {
  CropPlan p;
  p.n = n;
  p.cy = static_cast<int>(std::lround(cy));
  p.cx = static_cast<int>(std::lround(cx));
  p.radius = radius;
  p.out = output_size > 0 ? output_size : n;
  if (p.radius <= 0) p.radius = std::hypot(cy, cx) / 3.0f;
  require(p.out % 2 == 0 && p.out <= n, "extract_fields: output_size must be even and <= N");
  require(p.radius > 0 && p.radius <= static_cast<float>(p.out) / 2.0f,
          "extract_fields: crop radius must fit in the output window");
  return p;
}

FieldPlan::FieldPlan(const CropPlan& plan, int count) : plan_(plan), count_(count) {
  const int N = plan.n, m = plan.out;
  require(N >= 4 && N % 2 == 0, "extract_fields: images must be square with an even side");
  require(count >= 1 && count <= 65535, "extract_fields: invalid number of holograms");
  r2_ = plan.radius * plan.radius;
  // Largest |d| with d^2 <= r^2 in float, clipped to the output window.
  int d = 0;
  while (static_cast<float>((d + 1) * (d + 1)) <= r2_) ++d;
  dxlo_ = std::max(-m / 2, -d);
  const int dxhi = std::min(m / 2 - 1, d);
  W_ = dxhi - dxlo_ + 1;
  t1_.reset(static_cast<std::size_t>(count) * N * W_);
  t2_.reset(static_cast<std::size_t>(count) * m * W_);
}

std::size_t FieldPlan::device_bytes() const { return t1_.bytes() + t2_.bytes(); }

void FieldPlan::spectra(const float* holo, int first, int valid, cudaStream_t s) {
  const int N = plan_.n, m = plan_.out;
  const FftLen& Lm = fft_len(N / 2);
  const FftLen& Ln = fft_len(N);
  const FftLen& Lo = fft_len(m);
  const std::size_t rows = static_cast<std::size_t>(valid) * N;
  float2* t1 = t1_.get() + static_cast<std::size_t>(first) * N * W_;
  {
    const int c = rows_per_cta(N / 2);
    const std::size_t smem = 2 * static_cast<std::size_t>(N / 2 + 1) * (c + 1) * sizeof(float2);
    const unsigned grid = static_cast<unsigned>((rows + c - 1) / c);
    const int fx0 = plan_.cx + dxlo_;
#define QHK_ROWS(C)                                                                      \
  case C:                                                                                \
    allow(k_holo_rows<C>, smem);                                                         \
    k_holo_rows<C><<<grid, kThreads, smem, s>>>(holo, t1, rows, N, Lm, Ln.tw, fx0, W_); \
    break;
    switch (c) {
      QHK_ROWS(16)
      QHK_ROWS(8)
      QHK_ROWS(4)
      QHK_ROWS(2)
      QHK_ROWS(1)
    }
#undef QHK_ROWS
    check_launch("field rows");
  }
  {
    const int big = std::max(N, m);
    int c = 16;
    while (c > 1 && 2 * static_cast<std::size_t>(big) * c * sizeof(float2) > 72 * 1024) c /= 2;
    const std::size_t smem = 2 * static_cast<std::size_t>(big) * c * sizeof(float2);
    const dim3 grid((W_ + c - 1) / c, valid);
    float2* t2 = t2_.get() + static_cast<std::size_t>(first) * m * W_;
    const float sign = parity(plan_.cy + plan_.cx);
#define QHK_COLS(C)                                                                                          \
  case C:                                                                                                    \
    allow(k_holo_cols<C>, smem);                                                                             \
    k_holo_cols<C><<<grid, kThreads, smem, s>>>(t1, t2, N, m, W_, Ln, Lo, plan_.cy, plan_.cx, dxlo_, r2_, sign); \
    break;
    switch (c) {
      QHK_COLS(16)
      QHK_COLS(8)
      QHK_COLS(4)
      QHK_COLS(2)
      QHK_COLS(1)
    }
#undef QHK_COLS
    check_launch("field columns");
  }
}

void FieldPlan::finish(int mode, float2* field, const float2* bg, float* psi, float* logamp, cudaStream_t s,
                       int bg_count, int images) {
  const int N = plan_.n, m = plan_.out;
  const std::size_t bg_rows = static_cast<std::size_t>(bg_count > 0 ? bg_count : count_) * m;
  const FftLen& Lo = fft_len(m);
  require(images >= 0 && images <= count_, "fields: image count beyond the plan");
  const std::size_t rows = static_cast<std::size_t>(images > 0 ? images : count_) * m;
  const int c = rows_per_cta(m);
  const std::size_t smem = 2 * static_cast<std::size_t>(m) * (c + 1) * sizeof(float2);
  const unsigned grid = static_cast<unsigned>((rows + c - 1) / c);
  const int x0 = m / 2 + dxlo_;
  const float inv_nn = 1.0f / static_cast<float>(static_cast<std::size_t>(N) * N);
#define QHK_FIN(C)                                                                                        \
  case C:                                                                                                 \
    if (mode == 0) {                                                                                      \
      allow(k_field_rows<0, C>, smem);                                                                    \
      k_field_rows<0, C><<<grid, kThreads, smem, s>>>(t2_.get(), rows, m, W_, x0, Lo, inv_nn, field, bg, psi, \
                                                       logamp, bg_rows);                                    \
    } else {                                                                                              \
      allow(k_field_rows<1, C>, smem);                                                                    \
      k_field_rows<1, C><<<grid, kThreads, smem, s>>>(t2_.get(), rows, m, W_, x0, Lo, inv_nn, field, bg, psi, \
                                                       logamp, bg_rows);                                    \
    }                                                                                                     \
    break;
  switch (c) {
    QHK_FIN(16)
    QHK_FIN(8)
    QHK_FIN(4)
    QHK_FIN(2)
    QHK_FIN(1)
  }
#undef QHK_FIN
  check_launch("field inverse rows");
}

void FieldPlan::fields(const float* holo, float2* out, cudaStream_t s) {
  spectra(holo, 0, count_, s);
  finish(0, out, nullptr, nullptr, nullptr, s);
}

}  // namespace qhk

namespace qhk {

namespace {

// Peak of |H| over the +1 half plane of the centred spectrum outside the DC disc, in the host's
// scan order (rows y = 1 .. n-2, then columns x = n/2 .. n-2; the first strict maximum wins), from
// the half spectrum `half` (n x (n/2+1)) of one hologram. One CTA.
__global__ void __launch_bounds__(1024)
    k_sideband_argmax(const float2* __restrict__ half, int n, float dc2, float* best_mag, int* best_idx) {
  __shared__ float sm_mag[1024];
  __shared__ int sm_idx[1024];
  const int h = n / 2 + 1, c = n / 2;
  const int wx = n - 1 - c;  // columns c .. n-2
  const int total = (n - 2) * wx;
  float bm = 0.0f;
  int bi = -1;
  for (int t = threadIdx.x; t < total; t += blockDim.x) {
    const int y = 1 + t / wx;
    const int x = c + t % wx;
    const int dy = y - c, dx = x - c;
    if (dx == 0 && dy <= 0) continue;
    if (static_cast<float>(dy * dy + dx * dx) <= dc2) continue;
    const float2 v = half[static_cast<std::size_t>((dy + n) % n) * h + dx];
    const float m = hypotf(v.x, v.y);
    if (m > bm) {
      bm = m;
      bi = y * n + x;
    }
  }
  sm_mag[threadIdx.x] = bm;
  sm_idx[threadIdx.x] = bi;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      const float om = sm_mag[threadIdx.x + s];
      const int oi = sm_idx[threadIdx.x + s];
      const float mm = sm_mag[threadIdx.x];
      const int mi = sm_idx[threadIdx.x];
      if (om > mm || (om == mm && oi >= 0 && (mi < 0 || oi < mi))) {
        sm_mag[threadIdx.x] = om;
        sm_idx[threadIdx.x] = oi;
      }
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    *best_mag = sm_mag[0];
    *best_idx = sm_idx[0];
  }
}

}  // namespace

void sideband_peak(const float* holo, int n, float dc_exclusion, float2* half, float* d_mag, int* d_idx,
                   cudaStream_t s) {
  const int h = n / 2 + 1;
  rows_r2c(holo, half, static_cast<std::size_t>(n), n, false, s);
  axis_pass(half, 1, static_cast<std::size_t>(n) * h, n, static_cast<std::size_t>(h), h, true, AxisMode::plain, 1.0f,
            AxisAux{}, s);
  k_sideband_argmax<<<1, 1024, 0, s>>>(half, n, dc_exclusion * dc_exclusion, d_mag, d_idx);
  check_launch("sideband peak");
}

}  // namespace qhk
