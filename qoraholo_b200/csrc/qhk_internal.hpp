// Internal interfaces shared by the CUDA translation units of the backend. The public boundary is
// the C ABI in include/qoraholo_b200.h (capi.cu); these declarations are not exported.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "fft_engine.cuh"
#include "qhk_math.cuh"
#include "qhk_util.cuh"

namespace qhk {

// Cached transform description (radices + device twiddle table) of length n on the current
// device. Thread safe; tables live until the process exits.
const FftLen& fft_len(int n);

// ---- FFT passes (fft3d.cu) ------------------------------------------------------------------
// Data viewed as [outer][pos][inner], element (o, p, i) at o * so + p * sp + i, inner contiguous.
// Transforms along pos for every (o, i) with i < ni.
enum class AxisMode : int {
  plain,          // transform, times scale
  restore_half,   // forward, e = a + (1 - hits / 2) e, times scale, inverse (GP/FISTA k-space step)
  restore_mask,   // forward, e = mask ? measured : e, inverse (complex GP k-space step)
  from_data,      // loads aux (a) times scale instead of data, inverse transform
};
struct AxisAux {
  const float2* a = nullptr;        // half-spectrum data, or measured spectrum
  const std::uint8_t* hits = nullptr;  // hits (0..2) or mask (0/1)
};
// Shared-memory budget of one axis-pass tile (bytes); QHK_FFT_AXIS_KIB overrides it.
std::size_t axis_smem_budget();
// `batch` arrays of that layout, each sb elements after the previous (data and aux alike).
void axis_pass(float2* data, int n_outer, std::size_t so, int n, std::size_t sp, int ni, bool forward,
               AxisMode mode, float scale, const AxisAux& aux, cudaStream_t s, int batch = 1, std::size_t sb = 0);
// The same pass on the register-resident engine (fft_reg.cu) when it covers length n (64, 128, 192,
// 256, 512) in decomposition `variant` (1: the default; 2: fewer threads per line with longer
// per-thread DFTs, for 64, 128, 256); false otherwise, or when QHK_FFT_ENGINE=staged.
bool axis_pass_reg(float2* data, int n_outer, std::size_t so, int n, std::size_t sp, int ni, bool forward,
                   AxisMode mode, float scale, const AxisAux& aux, cudaStream_t s, int batch, std::size_t sb,
                   int variant = 1);
// Register-engine decompositions of length n (0: not covered).
int axis_reg_variants(int n);
// Whether plans also time the FFT decomposition of their axis passes (register variants against the
// staged engine): off by default, since the decompositions round differently and the choice would make
// results depend on timing (QHK_AUTOTUNE_RADIX=1 or qhk_autotune_radix(1)).
bool radix_tuning_enabled();
void set_radix_tuning(bool on);
// Forces the decomposition of every axis pass the register engine covers (0: staged engine; 1, 2: the
// register variants, where the length has them); -1 restores the tuned or default one. For tests.
void force_axis_engine(int engine);

// Runs rcp_sqrt_rn (qhk_math.cuh) against __frcp_rn(__fsqrt_rn(x)) for every float x in [1, 2^126) on
// the current device: the number of mismatches and the bits of the smallest mismatching x (all ones
// when there is none). Synchronous.
void selftest_rcp_sqrt(unsigned long long* mismatches, unsigned* first_bad);
bool fft_reg_engine_enabled();

// Times the tile widths of this axis pass on `data` (scratch: it is overwritten) and keeps the
// fastest for later axis_pass calls of the same shape. Never inside a stream capture.
void tune_axis_pass(float2* data, int n_outer, std::size_t so, int n, std::size_t sp, int ni, bool forward,
                    AxisMode mode, float scale, const AxisAux& aux, cudaStream_t s, int batch = 1,
                    std::size_t sb = 0);

// Rows of real length nx <-> half spectra of nx / 2 + 1 bins (rows dense, row pitches nx and
// nx / 2 + 1). R2C optionally clamps its input at 0 (Gerchberg-Papoulis). C2R writes the real
// rows, or the refractive index of the potential (last iteration).
void rows_r2c(const float* x, float2* e, std::size_t rows, int nx, bool clamp, cudaStream_t s);
enum class C2rMode : int { store, index };
void rows_c2r(const float2* e, float* x, std::size_t rows, int nx, C2rMode mode, float nm2, float inv_k02,
              cudaStream_t s);
// rows_c2r (store) then the real-space constraint max(x, 0) and rows_r2c of the constrained rows, in
// place on the half spectra `e`, the real rows never written out (one GP step boundary).
void rows_c2r_r2c(float2* e, std::size_t rows, int nx, cudaStream_t s);
// The final primal of a proximal TV step with FISTA momentum (tv_prox's TvFinal::momentum on dual p),
// then rows_r2c (no clamp) of the extrapolated point into `e`, without writing it: xprev <- x,
// e <- R2C(x + momentum (x - xprev)). Volumes dense (nz, ny, nx), nx even, 8-byte aligned.
void rows_tv_final_r2c(const float* b, const float* const p[3], int nz, int ny, int nx, float lambda, float momentum,
                       float* xprev, float2* e, cudaStream_t s);
// R2C, C2R and the GP step boundary on the register-resident engine (fft_reg.cu) when it covers the
// half length nx / 2 (64, 128, 192, 256); false otherwise. The staged functions call them first.
bool rows_r2c_reg(const float* x, float2* e, std::size_t rows, int nx, bool clamp, cudaStream_t s);
bool rows_c2r_reg(const float2* e, float* x, std::size_t rows, int nx, C2rMode mode, float nm2, float inv_k02,
                  cudaStream_t s);
bool rows_c2r_r2c_reg(float2* e, std::size_t rows, int nx, cudaStream_t s);

// Complex rows of length nx (dense). Modes for the complex Gerchberg-Papoulis loop.
enum class RowMode : int {
  plain,            // transform (forward or inverse), times scale
  inv_clamp_fwd,    // inverse times scale, (max(re, 0), 0), forward
  inv_index,        // inverse times scale, refractive index of (re, im) into `index`
};
void rows_c2c(float2* data, std::size_t rows, int nx, bool forward, RowMode mode, float scale, float* index,
              float nm2, float inv_k02, cudaStream_t s);

// 2D FFT of `count` images of n x n (dense), in place.
void fft2d(float2* data, int count, int n, bool forward, float scale, cudaStream_t s);

// ---- TV proximal step (tv.cu) -----------------------------------------------------------------
// Three triplets of dual volumes (z, y, x components). The dual p lives in v[p_index]; an FGP
// step reads the previous dual r from one triplet and writes the next r to another, and the
// first step of a call moves p to a free triplet (neighbouring CTAs still read the old p as r),
// so the three rotate and p_index is updated by tv_prox.
// Dual triplets (three volumes each) of the FGP iteration: p lives in v[p_index]. The fourth
// triplet is optional; with it the two-step form (k_fgp2) can run, which reads the duals of the
// neighbouring tiles' rows and so cannot update p or r in place.
struct TvBuffers {
  float* v[4][3] = {};
  int p_index = 0;
  // Device counter of this caller's bounded waits that ran out (a TMA box load of the two-step FGP
  // kernel that never completed); null counts them in the library-wide counter (tv_wait_timeouts).
  unsigned long long* wait_status = nullptr;
  [[nodiscard]] bool has_fourth() const { return v[3][0] != nullptr; }
};
enum class TvFinal : int {
  plain,     // out = argmin
  momentum,  // x = argmin; y = x + m (x - xprev); xprev <- x; out <- y
  index,     // out = refractive index of argmin
  none,      // no primal: the dual is left in t.v[t.p_index] (rows_tv_final_r2c takes it from there)
};
// `inner` FGP steps on the dual started from p, then the final primal. b and all volumes are dense
// (nz, ny, nx). For `momentum` the primal goes to xprev (in place) and the extrapolated point to out
// (which may alias b).
void tv_prox(const float* b, TvBuffers& t, int nz, int ny, int nx, float lambda, int inner,
             TvFinal final_mode, float momentum, float* xprev, float* out, float nm2, float inv_k02,
             cudaStream_t s);

// t_{k+1} of FISTA and FGP, 0.5 (1 + sqrt(1 + 4 t^2)) in float (host).
float fista_t(float t);

// FGP step form: 0 the autotuned one (untuned default: r stored), 1 the extrapolated point r
// stored between steps, 2 r recomputed from the two previous duals. Results are bitwise the same.
void set_tv_form(int form);

// Times the FGP tile heights on this volume's shape and keeps the fastest for later tv_prox calls.
// b and all three dual triplets of t are scratch (overwritten). Never inside a stream capture.
void tune_tv(float* b, TvBuffers& t, int nz, int ny, int nx, float lambda, cudaStream_t s);
// Bounded waits of the FGP kernels that ran out since the library was loaded, in calls whose
// TvBuffers carry no wait_status of their own (0 unless a box load never completed).
unsigned long long tv_wait_timeouts();
// Message of the error raised when a bounded device wait ran out in `what`.
std::string wait_timeout_message(const char* what);
// One bounded mbarrier wait that nothing completes, counted in the device word *counter (tma.cu).
void bounded_wait_probe(unsigned long long* counter, int polls, cudaStream_t s);

}  // namespace qhk
