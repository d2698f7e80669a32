/* C ABI of the QoraHolo B200 backend (libqhk.so).
 *
 * This is the drop-in boundary that replaces the reference's CUDA seam, the `namespace cuda`
 * functions and Pipeline::Impl declared in src/backends.hpp:75-126 of QoraHolo. Each entry point
 * names the reference interface it replaces. Plain C: device and host pointers, element counts,
 * `void*` streams (cudaStream_t; NULL = the legacy default stream), int status.
 *
 * Conventions (the reference's, README.md:268-277): arrays are dense row-major (z, y, x) with x
 * fastest; complex values are interleaved float32 pairs (complex64); images are square with an
 * even side; the centre of an image is pixel n/2; lengths in micrometres, frequencies in cycles
 * per micrometre. Illuminations are `count` (fy, fx) float pairs.
 *
 * Status: 0 on success, otherwise a QHK_* error class; qhk_last_error() returns the message of
 * the last failure on the calling thread. The host C++ layer maps the classes back to the
 * reference's exceptions: QHK_INVALID_ARGUMENT -> std::invalid_argument (src/api.cpp:13-28),
 * QHK_LOGIC_ERROR -> std::logic_error (src/pipeline.cpp:107-110), others -> std::runtime_error
 * (src/cuda/util.cuh:16-26).
 */
#ifndef QORAHOLO_B200_H_
#define QORAHOLO_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  QHK_OK = 0,
  QHK_INVALID_ARGUMENT = 1,
  QHK_CUDA_ERROR = 2,
  QHK_LOGIC_ERROR = 3,
  QHK_OUT_OF_MEMORY = 4,
  QHK_TIMEOUT = 5,
  QHK_INTERNAL = 6
};

enum { QHK_SOLVER_GP = 0, QHK_SOLVER_TV = 1 };          /* qoraholo::Solver (include/qoraholo/odt.hpp:25-32) */
enum { QHK_GP_R2C = 0, QHK_GP_C2C = 1 };                /* qoraholo::GpTransform (odt.hpp:38) */
enum { QHK_MAPPING_GATHER = 0, QHK_MAPPING_SCATTER = 1 }; /* qoraholo::Mapping (odt.hpp:22); both run the
                                                            same deterministic owner-computes mapping */

/* qoraholo::Geometry (include/qoraholo/odt.hpp:12-17). */
typedef struct qhk_geometry {
  float wavelength;
  float n_medium;
  float na;
  float pixel;
} qhk_geometry;

/* qoraholo::OdtOptions without the backend field (include/qoraholo/odt.hpp:40-51). */
typedef struct qhk_odt_options {
  int nz;           /* axial voxels; 0: field side */
  int iterations;   /* missing-cone iterations; 0: plain Rytov ODT */
  int solver;       /* QHK_SOLVER_* */
  int gp_transform; /* QHK_GP_* */
  float tv_weight;  /* TV weight for n^2 - n_medium^2 */
  int tv_inner;     /* FGP steps per proximal step */
  int mapping;      /* QHK_MAPPING_* */
} qhk_odt_options;

/* Message of the last failure on this thread ("" if none). */
const char* qhk_last_error(void);

/* 1 when a CUDA device is visible. Replaces cuda::device_present (src/cuda/runtime.cu:6-9). */
int qhk_device_present(void);

/* ---- ODT solver plan: replaces cuda::OdtSolver (src/cuda/stages.cuh:84-137, src/cuda/odt.cu:170-349).
 * A plan owns the device buffers of one geometry (n, nz, count, options) and runs Rytov fields ->
 * refractive index on a stream with no allocation. Validation follows odt_grid (src/api.cpp:107-123). */
typedef struct qhk_odt qhk_odt;
int qhk_odt_create(qhk_odt** plan, int n, int count, const float* illum_fyfx, const qhk_geometry* geometry,
                   const qhk_odt_options* options);
/* d_fields: (count, n, n) complex64 on the device, overwritten with their spectra.
 * d_index: (nz, n, n) float32 on the device. Asynchronous on `stream`. */
int qhk_odt_run(qhk_odt* plan, void* d_fields, float* d_index, void* stream);
/* Fraction of k-space voxels that received data in the last run (OdtResult::filled); waits for `stream`. */
int qhk_odt_filled(qhk_odt* plan, void* stream, double* filled);
int qhk_odt_shape(const qhk_odt* plan, int* nz, int* n);
size_t qhk_odt_device_bytes(const qhk_odt* plan);
int qhk_odt_destroy(qhk_odt* plan);

/* Per-call reconstruction, host in / host out: replaces cuda::reconstruct (src/cuda/odt.cu:359-406,
 * declared src/backends.hpp:113-116). fields: (count, n, n) complex64; out: (nz, n, n) float32 with
 * nz = options->nz or n. filled may be NULL. Allocates a plan for the call, like the reference. */
int qhk_reconstruct(const void* fields, int count, int n, const float* illum_fyfx, const qhk_geometry* geometry,
                    const qhk_odt_options* options, float* out, double* filled);

/* Ewald-sphere mapping alone: replaces map_gather / map_scatter, normalize_hits and
 * hermitian_hits / hermitian_data (src/cuda/odt.cu:22-131). d_spectra: (count, n, n) complex64
 * spectra of the Rytov fields. half != 0: d_data receives the half-spectrum data
 * a = (P(k) + conj P(-k)) / 2, (nz, n, n/2+1) complex64, and d_hits = M(k) + M(-k) (uint8);
 * half == 0: the normalised potential (nz, n, n) complex64 and the mask M (uint8). *d_filled (one
 * uint64 on the device) is incremented by the number of voxels that received data. The result does
 * not depend on the launch configuration: indices, counts and sums are those of the CPU mapping
 * (src/cpu/odt.cpp:147-173), summed in illumination order, with no atomics on floats. */
int qhk_ewald_map(const void* d_spectra, int count, int n, int nz, const float* illum_fyfx,
                  const qhk_geometry* geometry, int half, void* d_data, uint8_t* d_hits,
                  unsigned long long* d_filled, void* stream);

/* ---- TV proximal step: replaces cuda::tv_prox (src/cuda/tv.cuh:31-33, src/cuda/tv.cu:256-293).
 * x = argmin 0.5 |x - b|^2 + lambda TV(x), x >= 0, by `inner` FGP steps warm-started from the dual
 * d_dual (3 volumes: z, y, x components), which is updated. All on the device, (nz, ny, nx) dense. */
int qhk_tv_prox(const float* d_b, float* d_x, float* d_dual, int nz, int ny, int nx, float lambda, int inner,
                void* stream);

/* ---- FFTs on the device (the transforms the reference ran through cuFFT, src/cuda/util.cuh:137-174).
 * Unnormalised; results times `scale`. */
int qhk_fft2d(void* d_data, int count, int n, int forward, float scale, void* stream);
/* Real (nz, ny, nx) -> half spectrum (nz, ny, nx/2+1), and back (d_half is overwritten). */
int qhk_rfft3(const float* d_x, void* d_half, int nz, int ny, int nx, void* stream);
int qhk_irfft3(void* d_half, float* d_x, int nz, int ny, int nx, float scale, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* QORAHOLO_B200_H_ */
