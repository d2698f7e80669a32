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

/* The same proximal step with no allocation: d_dual holds 9 volumes -- the dual p (3 volumes, warm
 * start, updated in place) followed by 6 volumes of scratch. Asynchronous on `stream`. With 9
 * volumes it runs the one-step FGP forms (qhk_tv_prox, with 9 volumes of its own scratch, can run
 * two steps per pass). */
int qhk_tv_prox_device(const float* d_b, float* d_x, float* d_dual, int nz, int ny, int nx, float lambda, int inner,
                       void* stream);

/* The same with a caller workspace of `work_volumes` volumes: the dual p (3 volumes, warm start,
 * updated in place) followed by 6 (work_volumes 9: the one-step FGP forms) or 9 volumes of scratch
 * (work_volumes 12: also the two-step form). No allocation; asynchronous on `stream`. */
int qhk_tv_prox_workspace(const float* d_b, float* d_x, float* d_work, int work_volumes, int nz, int ny, int nx,
                          float lambda, int inner, void* stream);

/* Page-locked host memory (no counterpart in the reference): qhk_pipeline_run transfers page-locked
 * holograms and volumes directly, without staging copies, so callers that reuse buffers across runs
 * can allocate them here. */
int qhk_pinned_alloc(size_t bytes, void** ptr);
int qhk_pinned_free(void* ptr);

/* Bounded device waits (no counterpart in the reference, whose kernels have no device-side waits):
 * the two-step FGP kernel waits for its box loads (TMA) on mbarriers with an iteration limit; a wait
 * that gives up is counted and ends the kernel early, after a bounded wait for every load it still
 * has in flight, so the context stays usable but that result is invalid. Pipelines, ODT plans, the
 * server and qhk_tv_prox count in a counter of their own and turn a wait that ran out into
 * QHK_TIMEOUT (std::runtime_error in C++, RuntimeError in Python) from the call that synchronises
 * on the work: qhk_pipeline_process / run / run_stream, qhk_reconstruct, qhk_tv_prox, the server's
 * result, and for device-form runs qhk_pipeline_filled / filled_batch / check_waits and
 * qhk_odt_filled, qhk_bpm_reconstruct. qhk_wait_timeouts returns the count of the calls that have no
 * counter of their own (qhk_tv_prox_device, qhk_tv_prox_workspace): 0 in every correct run. It reads
 * the counter without waiting for work queued on other streams. */
int qhk_wait_timeouts(uint64_t* count);

/* Bounds checks of the debug build (compiled with QHK_DEBUG: `python qoraholo_b200/_build.py --debug`
 * writes qoraholo_b200/debug/libqhk.so, the same ABI). Its tile loaders, work-queue items, line indices
 * and shared-memory layouts check themselves and skip an access that would leave its buffer, recording
 * it instead of faulting; a skipped tile load also ends its bounded wait (QHK_TIMEOUT). No counterpart
 * in the reference, which has no device checks. qhk_debug_enabled: 1 in the debug build, else 0.
 * qhk_debug_violations: failed checks since the last reset (reset != 0 clears them), after waiting
 * for the device; when there were some, qhk_last_error names the source line of a first one. Always 0
 * in the release build. */
int qhk_debug_enabled(void);
int qhk_debug_violations(uint64_t* count, int reset);

/* Number of kernels this library has launched since it was loaded (for launch accounting). */
uint64_t qhk_kernel_launches(void);

/* ---- FFTs on the device (the transforms the reference ran through cuFFT, src/cuda/util.cuh:137-174).
 * Unnormalised; results times `scale`. */
int qhk_fft2d(void* d_data, int count, int n, int forward, float scale, void* stream);
/* Real (nz, ny, nx) -> half spectrum (nz, ny, nx/2+1), and back (d_half is overwritten). */
int qhk_rfft3(const float* d_x, void* d_half, int nz, int ny, int nx, void* stream);
int qhk_irfft3(void* d_half, float* d_x, int nz, int ny, int nx, float scale, void* stream);

/* ---- Field retrieval: replaces cuda::extract_fields / FieldStage (src/cuda/field.cu:121-135,
 * src/cuda/stages.cuh:19-47). Host in / host out. holo: (count, n, n) float32; the crop follows
 * crop_plan (src/api.cpp:52-60): centre (cy, cx) pixels from DC rounded to integers, radius <= 0
 * means |centre| / 3, output_size 0 means n. out: (count, m, m) complex64, m the output side. */
int qhk_extract_fields(const float* holo, int count, int n, float cy, float cx, float radius, int output_size,
                       void* out);

/* sample / background pixel by pixel (field_ratio, src/cpu/field.cpp:62-74; host-only in the reference).
 * sample: (count, ny, nx) complex64, background: bcount == 1 or bcount == count images. Host in / out. */
int qhk_field_ratio(const void* sample, int count, int ny, int nx, const void* background, int bcount, void* out);

/* Peak of the +1 sideband of hologram `holo` (n x n, host): find_sideband (src/cpu/field.cpp:25-60),
 * integer peak and the Jacobsen / Candan sub-pixel refinement. dc_exclusion <= 0 means n / 8. */
int qhk_find_sideband(const float* holo, int n, float dc_exclusion, int* iy, int* ix, float* y, float* x,
                      float* magnitude);

/* ---- Unwrap and Rytov: replaces cuda::unwrap / cuda::rytov / Unwrapper (src/cuda/unwrap.cu:156-263).
 * Host in / host out, (count, ny, nx) with even sides. */
int qhk_unwrap(const float* wrapped, int count, int ny, int nx, float* out);
int qhk_rytov(const void* ratio, int count, int ny, int nx, void* out);

/* Unwrap with no allocation -- no counterpart in the reference. The same least-squares unwrap as
 * qhk_unwrap, device in / device out: d_wrapped and d_unwrapped are (count, ny, nx) float32 buffers on
 * the device, owned by the caller; the function calls no cudaMalloc, cudaFree or other allocating
 * routine. It exists for callers that cannot allocate device memory during a run: a serving process
 * whose device memory is already reserved by its own allocator or HBM budget (where a library
 * allocation would fail or evict cached state), and real-time loops that must not pay for, or
 * synchronise on, allocation and release. All scratch lives in one static device array of about
 * 17.8 MB that a GPU holds from the moment the library's module is loaded on it until exit. With lazy
 * module loading (CUDA's default) that moment can be the first qhk_unwrap_noalloc call on the device,
 * so a caller that sizes its own reservation to what is left should first make one warm-up call (or
 * set CUDA_MODULE_LOADING=EAGER), and make that first call before any stream capture. Every call looks
 * up the array's address on the current device (cudaGetSymbolAddress, which allocates nothing), so the
 * function stays usable after a device reset. Limits: even sides, ny and nx <= 1024, count <= 4096,
 * count * ny * nx <= 4194304 pixels; larger requests return QHK_INVALID_ARGUMENT. Every call writes
 * all the scratch it reads (nothing must start at zero), asynchronously on `stream`; calls that overlap
 * on the GPU share the array and race, so serialise them (one stream, or events). */
int qhk_unwrap_noalloc(const float* d_wrapped, float* d_unwrapped, int count, int ny, int nx, void* stream);

/* ---- Launch-shape autotuner (no counterpart in the reference, which uses cuFFT plans and fixed
 * launch shapes). Plans time the candidate tile shapes of their FFT axis passes (columns per CTA)
 * and of the FGP step (rows per CTA) on their own buffers when they are built, and keep the fastest
 * per (device, shape) for the process; results are bitwise the same for every shape. On by default
 * (environment QHK_AUTOTUNE=0 turns it off). */
int qhk_autotune_enable(int enabled);
/* Also time the FFT decomposition of the axis passes (the register engine's variants T x V and the
 * staged radix engine) when plans are built, and keep the fastest. Off by default (environment
 * QHK_AUTOTUNE_RADIX=1 turns it on): the decompositions round differently, so with it on results stay
 * within the oracle's tolerance but depend on which variant won -- runs are no longer bitwise
 * reproducible across processes, nor batches bitwise equal to single requests. */
int qhk_autotune_radix(int enabled);
/* Forces the FFT decomposition of the axis passes the register engine covers, for tests and comparisons:
 * 0 the staged radix engine, 1 and 2 the register variants (2 where the length has one: 64, 128, 256);
 * -1 (the default) the tuned or default choice. */
int qhk_fft_axis_engine(int engine);

/* Self-check of the FGP dual projection's factor 1 / sqrt(x) (no counterpart in the reference): the
 * library computes it from approximate hardware results refined with fused multiply-adds, and this runs
 * it against the IEEE square root and reciprocal (the reference's 1.0f / std::sqrt) for every float in
 * [1, 2^126) on the current device. `mismatches` receives their number (0 when the two agree
 * everywhere), `first_bad` the bits of the smallest mismatching input. Synchronous. */
int qhk_selftest_rcp_sqrt(uint64_t* mismatches, uint32_t* first_bad);
/* FGP step form of tv_prox (bitwise the same results): 0 the tuned one, 1 the extrapolated point
 * stored between steps (13 volumes of traffic per step), 2 recomputed from the two previous duals
 * (10 volumes), 3 two steps per pass (13 volumes per two steps; needs rows of a multiple of 4
 * floats, at most 256, and a fourth dual triplet, so qhk_tv_prox_device runs form 1 instead),
 * 16 + rows: two steps per pass with 2, 4 or 8 rows per CTA (where the volume allows it). */
int qhk_tv_form(int form);
/* The tuned choices, one line each, into `buf` (NUL-terminated, truncated to `size`); returns the
 * full length. */
size_t qhk_autotune_report(char* buf, size_t size);

/* ---- Uneven unwrap batches (no counterpart in the reference, whose Unwrapper runs one image size per
 * call and loops over images for the y transform, src/cuda/unwrap.cu:156-234). `count` images of
 * their own even sizes ny[i] x nx[i], packed one after another on the device (image i starts at
 * qhk_unwrap_batch_offset(plan, i) floats); each of the five passes is one persistent launch over the
 * whole batch whose CTAs drain an (image, tile) queue. Every image's result is bitwise what
 * qhk_unwrap gives for it alone. `use_graph` != 0 replays the five launches as one CUDA graph (the
 * first call runs them directly). */
typedef struct qhk_unwrap_batch qhk_unwrap_batch;
int qhk_unwrap_batch_create(qhk_unwrap_batch** plan, const int* ny, const int* nx, int count);
size_t qhk_unwrap_batch_offset(const qhk_unwrap_batch* plan, int image);
size_t qhk_unwrap_batch_total(const qhk_unwrap_batch* plan);
int qhk_unwrap_batch_run(qhk_unwrap_batch* plan, const float* d_wrapped, float* d_unwrapped, int use_graph,
                         void* stream);
size_t qhk_unwrap_batch_device_bytes(const qhk_unwrap_batch* plan);
int qhk_unwrap_batch_destroy(qhk_unwrap_batch* plan);

/* Off-axis hologram synthesis on the device: synthesize_holograms (src/phantom.cpp:193-221, host-only in
 * the reference), |R + u_in ratio|^2 + noise, R = amplitude e^{-2 pi i carrier . r}, u_in = e^{2 pi i
 * (fy y + fx x)}. d_ratio (count, n, n) complex64 and d_out (count, n, n) float32 on the device,
 * illuminations on the host; `pixel` is the hologram pixel. Noise-free holograms equal the host's to
 * float rounding; the noise is N(0, noise^2) from a counter-based generator seeded by `seed` (other
 * draws than the host's std::mt19937_64). Synchronous. */
int qhk_synthesize_holograms_device(const void* d_ratio, int count, int n, const float* illum_fyfx, double pixel,
                                    double carrier_y, double carrier_x, double amplitude, float noise, uint64_t seed,
                                    float* d_out, void* stream);

/* Fixture generators of include/qoraholo/phantom.hpp, computed on the device (the reference computes
 * them on the host: render_phantom src/phantom.cpp:84-100, forward_fields src/phantom.cpp:102-191).
 * `spheres` are k rows of (z, y, x, radius, index) floats, micrometres from the volume centre, painted
 * in order (each entirely inside or outside every earlier one). Host in, host out, synchronous.
 * qhk_render_phantom: the index at the voxel centres of an (nz, n, n) volume of the geometry's pixel,
 * bitwise the reference's double-precision evaluation. qhk_forward_fields: field ratios
 * (count, n, n) complex64 at z = 0 for each illumination, model QHK_MODEL_BORN (1 + v),
 * QHK_MODEL_RYTOV (e^v) or QHK_MODEL_EXACT (the scalar partial-wave solution of exactly one sphere,
 * 1 + v); errors as the reference's (std::invalid_argument). */
enum { QHK_MODEL_BORN = 0, QHK_MODEL_RYTOV = 1, QHK_MODEL_EXACT = 2 }; /* qoraholo::ScatteringModel */
int qhk_render_phantom(const float* spheres, int k, const qhk_geometry* geometry, int nz, int n, float* out);
int qhk_forward_fields(const float* spheres, int k, const float* illum_fyfx, int count, const qhk_geometry* geometry,
                       int n, int model, void* out);

/* ---- Pipeline: replaces cuda::make_pipeline and Pipeline::Impl (src/backends.hpp:75-89,
 * src/cuda/pipeline.cu:12-161). Validation of the Pipeline constructor (src/pipeline.cpp:72-91). */
typedef struct qhk_pipeline_options {
  int count;          /* holograms per stack */
  int hologram_size;  /* side N */
  float center_y;     /* reference carrier, pixels from DC */
  float center_x;
  float radius;       /* crop radius; <= 0: |centre| / 3 */
  int output_size;    /* field side m; 0: N */
  int upload_chunks;  /* 1 .. count */
  qhk_odt_options odt;
} qhk_pipeline_options;

/* qoraholo::PipelineTimings (include/qoraholo/pipeline.hpp:31-43), milliseconds. */
typedef struct qhk_pipeline_timings {
  double upload, fields, rytov, fft2, clear, mapping, normalize, solve, finish, download, total;
} qhk_pipeline_timings;

typedef struct qhk_pipeline qhk_pipeline;
int qhk_pipeline_create(qhk_pipeline** pipeline, const qhk_pipeline_options* options, const float* illum_fyfx,
                        const qhk_geometry* geometry);
/* Background holograms (count, N, N), host. Their fields stay on the device. */
int qhk_pipeline_set_background(qhk_pipeline* pipeline, const float* backgrounds);
/* Page-locked input (count, N, N) float32 and output (nz, m, m) float32 buffers owned by the pipeline. */
float* qhk_pipeline_input(qhk_pipeline* pipeline);
const float* qhk_pipeline_output(const qhk_pipeline* pipeline);
/* input -> output; QHK_LOGIC_ERROR before set_background. Synchronous. */
int qhk_pipeline_process(qhk_pipeline* pipeline);
/* Pipeline::run (src/pipeline.cpp:116-129, run(holograms) -> OdtResult) on caller memory:
 * holograms (count, N, N) float32 -> index (nz, m, m) float32, both host memory, pageable or
 * page-locked (batched pipelines: batch stacks in, batch volumes out). Synchronous; the result
 * (filled, timings) as after process(). The staging copies run on QHK_COPY_THREADS host threads
 * (default min(8, hardware threads)), each upload chunk's copy overlapping the transfer and field
 * passes of the chunks before it; the pages of `index` are written (faulted in) while the device
 * solves, then the volume is copied out part by part as it arrives. Page-locked buffers (such as
 * qhk_pinned_alloc's) are transferred directly instead, without staging or host copies. `input` and
 * `output` serve as the staging for pageable buffers and then hold this call's data. */
int qhk_pipeline_run(qhk_pipeline* pipeline, const float* holograms, float* index);
/* A stream of `items` runs (no counterpart in the reference, which reconstructs one stack per
 * Pipeline::run): holograms (items, count, N, N) -> index (items, nz, m, m), host memory as for
 * qhk_pipeline_run, synchronous. The upload of stack i + 1 and the download of volume i - 1 overlap
 * the solve of stack i, so a stream costs about the device time of its stacks rather than that plus
 * the transfers; each volume is bitwise what qhk_pipeline_run gives for its stack. From each of the
 * two device volumes' second use on (within a call or across calls), the solve into it is replayed
 * as a captured CUDA graph instead of being launched kernel by kernel. Afterwards `filled` is that of
 * the last stack and the timings hold only `total`. One more device volume, and two graphs. */
int qhk_pipeline_run_stream(qhk_pipeline* pipeline, const float* holograms, int items, float* index);
/* Device-resident variant: d_holo (count, N, N) and d_index (nz, m, m) on the device, asynchronous on
 * `stream`, no host copies (for serving loops and benchmarks). */
int qhk_pipeline_process_device(qhk_pipeline* pipeline, const float* d_holo, float* d_index, void* stream);
/* filled fraction and stage timings of the last process(). */
int qhk_pipeline_result(const qhk_pipeline* pipeline, double* filled, qhk_pipeline_timings* timings);
/* Filled fraction after process_device (waits for `stream`); QHK_TIMEOUT if a bounded device wait of
 * the pipeline ran out since its last check (qhk_wait_timeouts). */
int qhk_pipeline_filled(qhk_pipeline* pipeline, void* stream, double* filled);
/* Waits for `stream` and returns QHK_TIMEOUT if a bounded device wait of the pipeline ran out since
 * its last check (after device-form runs, which cannot report it themselves). */
int qhk_pipeline_check_waits(qhk_pipeline* pipeline, void* stream);
/* Test hook of the timeout path: one bounded wait (`polls` polls, 1 .. 2^20) on an mbarrier that
 * nothing arrives at -- the form of the FGP kernel's waits -- counted in the pipeline's counter, on
 * the pipeline's own stream; returns QHK_TIMEOUT as a run whose wait ran out does. No load is in
 * flight, so the pipeline stays usable. */
int qhk_pipeline_wait_probe(qhk_pipeline* pipeline, int polls);
/* Device time of the FISTA-TV proximal steps inside the pipeline's runs (no counterpart in the
 * reference; for measurement): after qhk_pipeline_time_prox(pipeline, 1), runs launched directly (not
 * under stream capture) record CUDA events on their stream around the proximal step of every outer
 * iteration but the last; qhk_pipeline_prox_time waits for them and returns their total milliseconds
 * and the kernel launches inside them (the FGP launches), and starts a new count. */
int qhk_pipeline_time_prox(qhk_pipeline* pipeline, int enable);
int qhk_pipeline_prox_time(qhk_pipeline* pipeline, double* ms, uint64_t* launches);
int qhk_pipeline_shape(const qhk_pipeline* pipeline, int* nz, int* ny, int* nx);
/* Batched pipeline (no counterpart in the reference): `batch` requests of this geometry per run, each
 * pass one launch for all of them (FISTA-TV: the k-space passes span the batch, the TV proximal steps
 * run volume by volume). Input (batch * count, N, N), output (batch, nz, m, m); the background
 * holograms stay one stack (count, N, N). Every solver; each volume bitwise its single run. */
int qhk_pipeline_create_batched(qhk_pipeline** pipeline, const qhk_pipeline_options* options, const float* illum_fyfx,
                                const qhk_geometry* geometry, int batch);
/* process_device replayed as one CUDA graph (the first call for a pair of buffers runs directly). */
int qhk_pipeline_process_device_graph(qhk_pipeline* pipeline, const float* d_holo, float* d_index, void* stream);
/* Filled fraction of each of the batch's volumes after process_device (waits for `stream`). */
int qhk_pipeline_filled_batch(qhk_pipeline* pipeline, void* stream, double* filled);
size_t qhk_pipeline_device_bytes(const qhk_pipeline* pipeline);
int qhk_pipeline_destroy(qhk_pipeline* pipeline);

/* ---- Serving loop (no counterpart in the reference; its nearest form is one Pipeline per geometry,
 * src/cuda/pipeline.cu:12-147, used by one caller at a time). One scheduler thread per server admits
 * reconstruction requests of registered geometries as execution slots and device memory free up
 * (continuous batching against `hbm_budget_bytes`), keeps each geometry's background fields resident,
 * reuses per-geometry workspaces, runs requests of different workspaces concurrently on their own
 * streams and replays each workspace's pipeline as a CUDA graph from its second request on
 * (`use_graphs`). A request's result is bitwise the same alone and in any mix. Thread-safe: submit
 * and wait may be called from any threads. */
typedef struct qhk_server qhk_server;

/* Host timings of one request, milliseconds. */
typedef struct qhk_request_times {
  double queue_ms;    /* submit -> admitted */
  double service_ms;  /* admitted -> completion seen by the host */
  double total_ms;    /* submit -> completion seen by the host */
  double gpu_ms;      /* device time of the request (its copies and kernels) */
} qhk_request_times;

typedef struct qhk_server_counters {
  uint64_t submitted, completed, failed, cancelled;
  uint64_t workspaces_created, workspaces_evicted, graph_launches, passed_over;
  size_t budget, used, peak_used;
  int geometries, inflight, peak_inflight;
} qhk_server_counters;

/* The environment variable QHK_SERVER_STAGERS sets the number of host threads that stage pageable
 * inputs and outputs through the workspaces' page-locked buffers (default 2). QHK_SERVER_EXCLUSIVE=1
 * runs the requests' kernels one request at a time, in admission order, while their copies still
 * overlap: a lower tail latency at moderate load, less throughput at saturation (requests that run
 * together fill each other's idle SMs). */
int qhk_server_create(qhk_server** server, size_t hbm_budget_bytes, int max_inflight, int use_graphs);
/* Registers a geometry, validated as qhk_pipeline_create (`upload_chunks` is ignored), with its
 * background holograms (count, N, N) on the host. Synchronous. QHK_INVALID_ARGUMENT when its
 * background fields plus one workspace cannot fit the budget. */
int qhk_server_add_geometry(qhk_server* server, const qhk_pipeline_options* options, const float* illum_fyfx,
                            const qhk_geometry* geometry, const float* backgrounds, int* geometry_id);
/* QHK_LOGIC_ERROR while requests of the geometry are queued or running. */
int qhk_server_remove_geometry(qhk_server* server, int geometry_id);
int qhk_server_volume_shape(qhk_server* server, int geometry_id, int* nz, int* n);
/* Queues holograms (count, N, N) float32 -> index (nz, n, n) float32 into `index_out`. Host buffers,
 * pageable (staged by the server's threads) or page-locked (copied directly); both must stay valid
 * until qhk_server_wait returns, and a pageable `index_out` holds unspecified values until then. */
int qhk_server_submit(qhk_server* server, int geometry_id, const float* holograms, float* index_out,
                      uint64_t* ticket);
/* *done = 1 once the request has completed. */
int qhk_server_done(qhk_server* server, uint64_t ticket, int* done);
/* Withdraws a request not admitted yet (*cancelled = 1): it then completes with QHK_LOGIC_ERROR and uses
 * no device time. *cancelled = 0 once it runs or has finished. */
int qhk_server_cancel(qhk_server* server, uint64_t ticket, int* cancelled);
/* Blocks until the request is done; `filled` and `times` may be NULL. Returns the request's error. */
int qhk_server_wait(qhk_server* server, uint64_t ticket, double* filled, qhk_request_times* times);
int qhk_server_stats(qhk_server* server, qhk_server_counters* stats);
/* Drains running requests (queued ones fail with QHK_LOGIC_ERROR) and frees everything. */
int qhk_server_destroy(qhk_server* server);

/* The server's admission policy run on the host alone, for tests and capacity planning (no device
 * work). Geometries g = 0..n_geometries-1 hold resident[g] bytes and workspace[g] bytes per workspace
 * (one workspace each is created at registration). ops: g >= 0 submits a request of geometry g; -1
 * completes the oldest running request. After every op as many requests as possible are admitted;
 * each admission appends the request's submission index to admitted[], its action to action[] (0
 * reuse, 1 allocate, 2 allocate after evicting idle workspaces) and the budget in use after it to
 * used[] (arrays of n_ops entries). *n_admitted receives the count. */
int qhk_admission_simulate(size_t budget, int max_inflight, int max_pass, int n_geometries, const size_t* resident,
                           const size_t* workspace, const int* ops, int n_ops, int* admitted, int* action,
                           size_t* used, int* n_admitted);

/* ---- Beam propagation: replaces cuda::bpm_forward / bpm_vjp / bpm_reconstruct (src/backends.hpp:117-124,
 * src/cuda/bpm.cu:236-349), tables as bpm_tables (src/bpm.cpp:10-60). Host in / host out. */
/* ri: (nz, n, n) refractive index -> out: (count, n, n) complex64 field ratios at z = 0. */
int qhk_bpm_forward(const float* ri, int nz, int n, const float* illum_fyfx, int count, const qhk_geometry* geometry,
                    int obliquity, void* out);
/* x: (nz, n, n) contrast n - n_medium, r: (count, n, n) complex64 -> out = J^T r (nz, n, n). */
int qhk_bpm_vjp(const float* x, int nz, int n, const void* r, const float* illum_fyfx, int count,
                const qhk_geometry* geometry, int obliquity, float* out);

/* qoraholo::BpmSolveOptions without the backend field (include/qoraholo/bpm.hpp:29-41). */
/* Device-level BPM plan for gradient-based inversion (autograd): the forward model on device
 * buffers, and its vector-Jacobian product with slice checkpointing. Replaces the Bpm class of the
 * reference's CUDA backend (src/cuda/bpm.cu:126-199; forward and adjoint sweeps, envelopes stored
 * for every slice) with a plan that keeps, per illumination, only the spectrum entering every
 * `checkpoint_every`-th slice (0: every envelope, as the reference) and recomputes each segment of
 * slices before sweeping it backwards. `chunk` illuminations run per device pass (0: all). */
typedef struct qhk_bpm_plan qhk_bpm_plan;
int qhk_bpm_plan_create(qhk_bpm_plan** plan, int nz, int n, const float* illum_fyfx, int count,
                        const qhk_geometry* geometry, int obliquity, int chunk, int checkpoint_every);
/* d_ri (nz, n, n) float32 -> d_fields (count, n, n) complex64, the field ratios at z = 0; keeps the
 * checkpoints of this volume for a following qhk_bpm_plan_vjp. Asynchronous on `stream`. */
int qhk_bpm_plan_forward(qhk_bpm_plan* plan, const float* d_ri, void* d_fields, void* stream);
/* d_grad_ri (nz, n, n) = Re(J^H g) for g = d_grad_fields (count, n, n) complex64, J the Jacobian of
 * the forward model at d_ri, which must be the volume of the last qhk_bpm_plan_forward. For
 * g = forward(ri) - data this is the gradient of 1/2 |forward(ri) - data|^2 (src/cuda/bpm.cu:250-272). */
int qhk_bpm_plan_vjp(qhk_bpm_plan* plan, const float* d_ri, const void* d_grad_fields, float* d_grad_ri, void* stream);
size_t qhk_bpm_plan_device_bytes(const qhk_bpm_plan* plan);
int qhk_bpm_plan_destroy(qhk_bpm_plan* plan);

typedef struct qhk_bpm_solve_options {
  int iterations;
  int batch;
  float step;
  float tv_weight;
  int tv_inner;
  int obliquity;
} qhk_bpm_solve_options;

/* fields (count, n, n) complex64, initial (nz, n, n) index -> out (nz, n, n) index; loss receives
 * `iterations` doubles (the data term per iteration, BpmResult::loss). */
int qhk_bpm_reconstruct(const void* fields, int count, int n, const float* illum_fyfx, const qhk_geometry* geometry,
                        const float* initial, int nz, const qhk_bpm_solve_options* options, float* out, double* loss);

/* Host in / host out 2D FFT of `count` n x n images (used by the fixture generators). */
int qhk_fft2d_host(void* data, int count, int n, int forward, float scale);

#ifdef __cplusplus
}
#endif

#endif /* QORAHOLO_B200_H_ */
