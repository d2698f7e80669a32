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
#include <map>
#include <numbers>
#include <vector>

#include "unwrap.hpp"
#include "nvtx.hpp"

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
  extern __shared__ float2 sm[];
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
  extern __shared__ float2 sm[];
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
  extern __shared__ float2 sm[];
  __shared__ double red[2][kThreads];
  const std::size_t img = static_cast<std::size_t>(blockIdx.y) * ny * nx;
  idctx_tile<COLS>(phi + img, psi + img, ny, nx, L, dtw, static_cast<int>(blockIdx.x) * COLS,
                   partial + (static_cast<std::size_t>(blockIdx.y) * gridDim.x + blockIdx.x) * 2, sm, red);
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
  rows_ = rows_per_cta(nx, static_cast<std::size_t>(nx) * sizeof(float));
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
  {
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
  {
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
  {
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
  int partial;         // first congruence partial pair of this image
  FftLen Lx, Ly;
  const float2* dtw_x;
  const float2* dtw_y;
  const float* cos_x;
  const float* cos_y;
};

constexpr int kAssembleChunk = 16384;  // pixels per item of the last pass

// Next queue item for the whole CTA (thread 0 takes it, everyone reads it).
__device__ __forceinline__ int next_item(int* counter) {
  __shared__ int item;
  if (threadIdx.x == 0) item = atomicAdd(counter, 1);
  __syncthreads();
  const int it = item;
  __syncthreads();
  return it;
}

#define QHK_ROWS_SWITCH(R, CALL) \
  switch (R) {                   \
    case 16: CALL(16); break;    \
    case 8: CALL(8); break;      \
    case 4: CALL(4); break;      \
    case 2: CALL(2); break;      \
    default: CALL(1); break;     \
  }

__global__ void __launch_bounds__(kThreads)
    k_batch_pass1(const float* __restrict__ psi, float* __restrict__ d1, const BatchImage* __restrict__ imgs,
                  const int2* __restrict__ items, int n, int* counter) {
  extern __shared__ float2 sm[];
  for (int it = next_item(counter); it < n; it = next_item(counter)) {
    const int2 w = items[it];
    const BatchImage& im = imgs[w.x];
#define QHK_P1(C) div_dctx_tile<C>(psi + im.offset, d1 + im.offset, im.ny, im.nx, im.Lx, im.dtw_x, w.y * (C), sm)
    QHK_ROWS_SWITCH(im.rows, QHK_P1)
#undef QHK_P1
    __syncthreads();
  }
}

__global__ void __launch_bounds__(kThreads)
    k_batch_pass2(const float* __restrict__ d1, float* __restrict__ phi, const BatchImage* __restrict__ imgs,
                  const int2* __restrict__ items, int n, int* counter) {
  extern __shared__ float2 sm[];
  for (int it = next_item(counter); it < n; it = next_item(counter)) {
    const int2 w = items[it];
    const BatchImage& im = imgs[w.x];
#define QHK_P2(C)                                                                                                  \
  dcty_solve_tile<C>(d1 + im.offset, phi + im.offset, im.ny, im.nx, im.Ly, im.dtw_y, im.cos_y, im.cos_x, w.y * (C), \
                     sm)
    QHK_ROWS_SWITCH(im.cols, QHK_P2)
#undef QHK_P2
    __syncthreads();
  }
}

__global__ void __launch_bounds__(kThreads)
    k_batch_pass3(float* __restrict__ phi, const float* __restrict__ psi, double* __restrict__ partial,
                  const BatchImage* __restrict__ imgs, const int2* __restrict__ items, int n, int* counter) {
  extern __shared__ float2 sm[];
  __shared__ double red[2][kThreads];
  for (int it = next_item(counter); it < n; it = next_item(counter)) {
    const int2 w = items[it];
    const BatchImage& im = imgs[w.x];
    double* pair = partial + 2 * (static_cast<std::size_t>(im.partial) + w.y);
#define QHK_P3(C) \
  idctx_tile<C>(phi + im.offset, psi + im.offset, im.ny, im.nx, im.Lx, im.dtw_x, w.y * (C), pair, sm, red)
    QHK_ROWS_SWITCH(im.rows, QHK_P3)
#undef QHK_P3
    __syncthreads();
  }
}

__global__ void __launch_bounds__(kThreads)
    k_batch_pass4(const float* __restrict__ phi, const double* __restrict__ partial, float2* __restrict__ consts,
                  const BatchImage* __restrict__ imgs, const int2* __restrict__ items, int n, int* counter) {
  extern __shared__ float pairs[];
  for (int it = next_item(counter); it < n; it = next_item(counter)) {
    const int2 w = items[it];
    const BatchImage& im = imgs[w.x];
    rytov_consts_image(phi + im.offset, im.ny, im.nx, partial + 2 * static_cast<std::size_t>(im.partial), im.nblk,
                       consts + w.x, pairs);
    __syncthreads();
  }
}

__global__ void __launch_bounds__(kThreads)
    k_batch_pass5(float* __restrict__ phi, const float2* __restrict__ consts, const BatchImage* __restrict__ imgs,
                  const int2* __restrict__ items, int n, int* counter) {
  for (int it = next_item(counter); it < n; it = next_item(counter)) {
    const int2 w = items[it];
    const BatchImage& im = imgs[w.x];
    const float c = consts[w.x].x;
    const std::size_t pixels = static_cast<std::size_t>(im.ny) * im.nx;
    const std::size_t a = static_cast<std::size_t>(w.y) * kAssembleChunk;
    const std::size_t b = min(pixels, a + kAssembleChunk);
    for (std::size_t i = a + threadIdx.x; i < b; i += blockDim.x) {
      phi[im.offset + i] = __fadd_rn(phi[im.offset + i], c);
    }
  }
}

#undef QHK_ROWS_SWITCH

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
  std::size_t smem[5] = {0, 0, 0, 0, 0};
  for (int i = 0; i < count; ++i) {
    require(ny[i] >= 2 && nx[i] >= 2 && ny[i] % 2 == 0 && nx[i] % 2 == 0, "unwrap: image sides must be even");
    BatchImage& b = im[i];
    b.offset = total_;
    offsets_.push_back(total_);
    total_ += static_cast<std::size_t>(ny[i]) * nx[i];
    b.ny = ny[i];
    b.nx = nx[i];
    b.rows = rows_per_cta(b.nx, static_cast<std::size_t>(b.nx) * sizeof(float));
    b.cols = solve_cols(b.ny);
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
    smem[0] = std::max(smem[0], row_buf + (b.rows + 2) * static_cast<std::size_t>(b.nx) * sizeof(float));
    smem[1] = std::max(smem[1], 2 * static_cast<std::size_t>(b.ny) * b.cols * sizeof(float2) +
                                    static_cast<std::size_t>(b.ny) * b.cols * sizeof(float));
    smem[2] = std::max(smem[2], row_buf + b.rows * static_cast<std::size_t>(b.nx) * sizeof(float));
    smem[3] = std::max(smem[3], static_cast<std::size_t>(b.nx + b.ny) * sizeof(float));
  }
  // Items, largest images first so that the queue ends with small tiles.
  std::vector<int> order(count);
  for (int i = 0; i < count; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
    return static_cast<std::size_t>(im[a].ny) * im[a].nx > static_cast<std::size_t>(im[b].ny) * im[b].nx;
  });
  std::vector<int2> items[5];
  for (const int i : order) {
    const BatchImage& b = im[i];
    for (int t = 0; t < b.nblk; ++t) items[0].push_back(make_int2(i, t));
    for (int t = 0; t < (b.nx + b.cols - 1) / b.cols; ++t) items[1].push_back(make_int2(i, t));
    items[3].push_back(make_int2(i, 0));
    const std::size_t pixels = static_cast<std::size_t>(b.ny) * b.nx;
    for (std::size_t t = 0; t * kAssembleChunk < pixels; ++t) items[4].push_back(make_int2(i, static_cast<int>(t)));
  }
  items[2] = items[0];
  std::vector<int2> all;
  std::size_t at[5];
  for (int p = 0; p < 5; ++p) {
    at[p] = all.size();
    all.insert(all.end(), items[p].begin(), items[p].end());
  }
  items_.reset(all.size());
  check(cudaMemcpy(items_.get(), all.data(), all.size() * sizeof(int2), cudaMemcpyHostToDevice), "upload items");
  images_.reset(count * sizeof(BatchImage));
  check(cudaMemcpy(images_.get(), im.data(), count * sizeof(BatchImage), cudaMemcpyHostToDevice), "upload images");
  counters_.reset(5);
  d1_.reset(total_);
  partial_.reset(2 * static_cast<std::size_t>(partial));
  consts_.reset(count);
  for (int p = 0; p < 5; ++p) {
    pass_[p].items = items_.get() + at[p];
    pass_[p].n = static_cast<int>(items[p].size());
    pass_[p].smem = smem[p];
  }
  pass_[0].grid = persistent_grid(k_batch_pass1, smem[0], pass_[0].n);
  pass_[1].grid = persistent_grid(k_batch_pass2, smem[1], pass_[1].n);
  pass_[2].grid = persistent_grid(k_batch_pass3, smem[2], pass_[2].n);
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
  const auto items = [&](int p) { return static_cast<const int2*>(pass_[p].items); };
  check(cudaMemsetAsync(q, 0, 5 * sizeof(int), s), "cudaMemset");
  k_batch_pass1<<<pass_[0].grid, kThreads, pass_[0].smem, s>>>(psi, d1_.get(), imgs, items(0), pass_[0].n, q);
  check_launch("unwrap batch pass 1");
  k_batch_pass2<<<pass_[1].grid, kThreads, pass_[1].smem, s>>>(d1_.get(), phi, imgs, items(1), pass_[1].n, q + 1);
  check_launch("unwrap batch pass 2");
  k_batch_pass3<<<pass_[2].grid, kThreads, pass_[2].smem, s>>>(phi, psi, partial_.get(), imgs, items(2),
                                                               pass_[2].n, q + 2);
  check_launch("unwrap batch pass 3");
  k_batch_pass4<<<pass_[3].grid, kThreads, pass_[3].smem, s>>>(phi, partial_.get(), consts_.get(), imgs, items(3),
                                                               pass_[3].n, q + 3);
  check_launch("unwrap batch constants");
  k_batch_pass5<<<pass_[4].grid, kThreads, 0, s>>>(phi, consts_.get(), imgs, items(4), pass_[4].n, q + 4);
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
  const int rows = rows_per_cta(nx, static_cast<std::size_t>(nx) * sizeof(float));
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
  {
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
  {
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
  {
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
