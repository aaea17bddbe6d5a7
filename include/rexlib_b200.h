/*
 * rexlib_b200: a B200 (sm_100a) backend for rexlib's em reconstruction path.
 *
 * The C-ABI boundary of librexlib_b200.so. Every entry point takes plain
 * device pointers, element counts and a cudaStream_t passed as void*; no C++
 * or framework type crosses it. Each one replaces the work a rexlib program
 * builder's program does when the eager dispatcher submits the operation
 * named beside it, so a rexlib plugin's program launch() (the pattern of
 * plugins/cuda/src/hardware/stream_program.hpp:49) forwards its buffers here.
 *
 * Conventions.
 * - Complex arrays are interleaved (re, im) float32, rexlib's complex_float32.
 * - Arrays are row-major. The core axes of every operand are contiguous; the
 *   batch of a per-slice operand is addressed by two strides, in units of
 *   its core: element (v, p) starts at v * volume_stride + p * particle_stride
 *   cores. A stride of 0 broadcasts, as rexlib's batch broadcasting does.
 * - Calls are stream-ordered and asynchronous. A return of
 *   REXLIB_B200_OK means the work was enqueued; rexlib_b200_last_error()
 *   returns the calling thread's last message otherwise.
 * - Invalid arguments are refused with REXLIB_B200_INVALID_ARGUMENT (the
 *   reference throws std::invalid_argument at the same points); shapes or
 *   types the backend does not run are refused with REXLIB_B200_UNSUPPORTED
 *   (a rexlib program builder answers backend_priority::unsupported).
 */
#ifndef REXLIB_B200_H
#define REXLIB_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define REXLIB_B200_ABI_VERSION 2

#if defined(__GNUC__)
#define REXLIB_B200_API __attribute__((visibility("default")))
#else
#define REXLIB_B200_API
#endif

typedef enum rexlib_b200_status
{
	REXLIB_B200_OK = 0,
	REXLIB_B200_INVALID_ARGUMENT = 1,
	REXLIB_B200_UNSUPPORTED = 2,
	REXLIB_B200_CUDA_ERROR = 3,
	REXLIB_B200_WORKSPACE_TOO_SMALL = 4
} rexlib_b200_status;

/* em::gridding_profile (include/rexlib/em/ops/parameters/gridding_window.hpp). */
typedef enum rexlib_b200_gridding_profile
{
	REXLIB_B200_WINDOW_BOX = 0,
	REXLIB_B200_WINDOW_TRIANGLE = 1,
	REXLIB_B200_WINDOW_KAISER_BESSEL = 2
} rexlib_b200_gridding_profile;

/* em::gridding_window: nearest() = {BOX, 0.5, 0}, linear() =
 * {TRIANGLE, 1, 0}, kaiser_bessel(w, beta) = {KAISER_BESSEL, w, beta}
 * (src/em/ops/parameters/gridding_window.cpp). */
typedef struct rexlib_b200_gridding_window
{
	int32_t profile;
	double half_width;
	double shape;
} rexlib_b200_gridding_window;

/* em::ctf_optics (include/rexlib/em/ops/parameters/ctf_optics.hpp): the
 * voltage in kV, Cs in mm, amplitude contrast in [0, 1). */
typedef struct rexlib_b200_ctf_optics
{
	double voltage;
	double spherical_aberration;
	double amplitude_contrast;
} rexlib_b200_ctf_optics;

/* How the insertion sums. THROUGHPUT: FP32 sums whose order varies between
 * runs. DETERMINISTIC: every voxel sums its contributions in one fixed order
 * (slice, then sample order), so runs are bit-identical and a batch split
 * across calls gives the bits of one call; every window, slice extents up to
 * 1024, fewer than 65,536 volumes. */
typedef enum rexlib_b200_insert_mode
{
	REXLIB_B200_INSERT_THROUGHPUT = 0,
	REXLIB_B200_INSERT_DETERMINISTIC = 1
} rexlib_b200_insert_mode;

/* Element types: rexlib's float32, float64, complex_float32 and
 * complex_float64 (interleaved re, im). An insertion names its real type
 * (FLOAT32 or FLOAT64); its complex operands hold pairs of it. */
typedef enum rexlib_b200_element_type
{
	REXLIB_B200_FLOAT32 = 0,
	REXLIB_B200_FLOAT64 = 1,
	REXLIB_B200_COMPLEX64 = 2,
	REXLIB_B200_COMPLEX128 = 3
} rexlib_b200_element_type;

/* Batch strides of a per-slice operand, in cores (0 broadcasts). */
typedef struct rexlib_b200_batch_strides
{
	int64_t volume;
	int64_t particle;
} rexlib_b200_batch_strides;

/*
 * The operands of one insertion call: V accumulators of extent N, each
 * receiving P slices of extent n.
 *
 *   numerator_in/out    (V, N, N, N/2+1) complex
 *   denominator_in/out  (V, N, N, N/2+1) real
 *   slices              core (n, n/2+1) complex
 *   transforms          core (3, 4) real, [A | t]
 *   radial_weights      core (n/2+1) real
 *
 * Every operand holds element_type: FLOAT32 (the default of a zeroed
 * descriptor; complex operands complex64) or FLOAT64 (complex128), one type
 * for all, as slice_insertion_rules.hpp:86-90 requires. FLOAT64 runs in the
 * throughput mode (the deterministic mode returns REXLIB_B200_UNSUPPORTED),
 * with Kaiser-Bessel half-widths up to 3.
 *
 * The outputs are the inputs plus the insertions. Passing the same pointer
 * for an input and its output updates in place; the inputs are copied to
 * the outputs first otherwise (insert_slices_operation.hpp:50-52). The
 * workspace is device memory of rexlib_b200_insertion_workspace_size() bytes,
 * 256-byte aligned (the program's scratch requirement,
 * include/rexlib/core/hardware/program.hpp:63). It holds, besides the work
 * plan, one numerator tile per resident CTA, so its size depends on the
 * current device's SM count: query it with the device of the call current.
 */
typedef struct rexlib_b200_insertion
{
	void *numerator_out;
	void *denominator_out;
	const void *numerator_in;
	const void *denominator_in;
	const void *slices;
	const void *transforms;
	const void *radial_weights;
	rexlib_b200_batch_strides slice_strides;
	rexlib_b200_batch_strides transform_strides;
	rexlib_b200_batch_strides radial_strides;
	int64_t volume_count;      /* V */
	int64_t slices_per_volume; /* P */
	int64_t slice_extent;      /* n */
	int64_t volume_extent;     /* N */
	rexlib_b200_gridding_window window;
	int32_t mode;              /* rexlib_b200_insert_mode */
	void *workspace;
	size_t workspace_bytes;
	int32_t element_type;      /* rexlib_b200_element_type: FLOAT32 or FLOAT64 */
} rexlib_b200_insertion;

/* The calling thread's last error message ("" if none). */
REXLIB_B200_API const char *rexlib_b200_last_error(void);

/* REXLIB_B200_ABI_VERSION of the library. */
REXLIB_B200_API int32_t rexlib_b200_abi_version(void);

/* Device scratch an insertion call needs, in bytes (0 when none). */
REXLIB_B200_API int32_t rexlib_b200_insertion_workspace_size(const rexlib_b200_insertion *insertion, size_t *bytes);

/* Kernels of this library an insertion call launches (its accumulator copy
 * for distinct outputs is a device copy, not a kernel). No counterpart in
 * the reference: it lets a caller count the library's launches. */
REXLIB_B200_API int32_t rexlib_b200_insertion_launches(const rexlib_b200_insertion *insertion, int32_t *count);

/*
 * The on-chip rates the tiled insertion's accumulation runs into, for its
 * roofline beside HBM (no counterpart in the reference). Each call launches
 * blocks x threads threads doing per_thread operations; the caller times it.
 *   l2_reduction_run: red.global.add.v4.f32 of one 16-byte slot a lane, the
 *     slots pseudo-random over `region` (device, `bytes`, 16-byte aligned):
 *     the numerator's vector reductions into its L2 scratch;
 *   shared_atomic_run: FP32 shared-memory atomics at pseudo-random words of a
 *     48 KB tile (bank conflicts included), one float added to *sink at the
 *     end: the denominator's taps, in lane operations.
 */
REXLIB_B200_API int32_t rexlib_b200_l2_reduction_run(void *region, int64_t bytes, int32_t blocks, int32_t threads,
	int32_t per_thread, uint32_t seed, void *stream);
REXLIB_B200_API int32_t rexlib_b200_shared_atomic_run(float *sink, int32_t blocks, int32_t threads,
	int32_t per_thread, uint32_t seed, void *stream);

/*
 * em::insert_slices (src/em/functional/reconstruction.cpp:49-77; operation
 * include/rexlib/em/ops/reconstruction/insert_slices_operation.hpp:40-114):
 *   numerator[g]   += kappa(g - K) r v exp(-2 pi i g.C/N)
 *   denominator[g] += kappa(g - K) r
 */
REXLIB_B200_API int32_t rexlib_b200_insert_slices(const rexlib_b200_insertion *insertion, void *stream);

/*
 * em::insert_weighted_slices (src/em/functional/reconstruction.cpp:79-105;
 * insert_weighted_slices_operation.hpp:33-46): the denominator receives
 * kappa r W(k). weights: core (n, n/2+1) of the insertion's real type.
 */
REXLIB_B200_API int32_t rexlib_b200_insert_weighted_slices(
	const rexlib_b200_insertion *insertion,
	const void *weights,
	rexlib_b200_batch_strides weight_strides,
	void *stream);

/*
 * em::insert_ctf_slices (src/em/functional/reconstruction.cpp:107-138;
 * insert_ctf_slices_operation.hpp:33-67): the numerator receives
 * kappa r c(k) v, the denominator kappa r c(k)^2. ctf: core (4) of the
 * insertion's real type: defocus U, defocus V (angstroms), astigmatism
 * angle, phase shift (radians).
 */
REXLIB_B200_API int32_t rexlib_b200_insert_ctf_slices(
	const rexlib_b200_insertion *insertion,
	const void *ctf,
	rexlib_b200_batch_strides ctf_strides,
	rexlib_b200_ctf_optics optics,
	double pixel_size,
	void *stream);

/*
 * insert_ctf_slices without any device allocation. No counterpart in the
 * reference: it serves callers that cannot call cudaMalloc, such as a rexlib
 * program launching on a queue that must not synchronize the device (as a
 * cudaMalloc or cudaFree does), or a caller whose device memory is budgeted
 * up front. The operands, their checks and the results are those of
 * rexlib_b200_insert_ctf_slices; the descriptor's workspace fields are
 * ignored, and the scratch is instead a fixed 8 MiB array inside the
 * library, present on every device that loads the library until the
 * process exits.
 * - A call whose scratch would exceed 8 MiB is refused with
 *   REXLIB_B200_INVALID_ARGUMENT and a message giving both sizes; insert
 *   such batches in several calls. In the throughput mode the scratch is
 *   104 bytes per slice and volume, plus 4 bytes per tile and volume, plus
 *   16 bytes per work item, of which there are tiles x (1 + ceil(P / 320))
 *   per volume (each part rounded up to 256 bytes, plus 256). Its tiles keep
 *   the whole tile in shared memory: 1,440 tiles for a 256^3 volume with the
 *   linear window, so about 47,000 slices of 256^2 into one 256^3 volume
 *   fit; the nearest window has fewer tiles, while Kaiser-Bessel windows and
 *   odd volume extents have more and fit fewer slices. The deterministic
 *   mode needs 104 bytes per slice and volume plus 4 bytes per 16^3 tile.
 * - Every call looks up the array's device address in the current context
 *   (the lookup allocates nothing). The first call in a context loads the
 *   library's device code there, so make that first call before any stream
 *   capture.
 * - Every call shares the one array and leaves its contents behind; calls
 *   that overlap on the GPU (other streams, other host threads) race on it,
 *   so order them on one stream or serialize them.
 */
REXLIB_B200_API int32_t rexlib_b200_insert_ctf_slices_fixed_scratch(
	const rexlib_b200_insertion *insertion,
	const void *ctf,
	rexlib_b200_batch_strides ctf_strides,
	rexlib_b200_ctf_optics optics,
	double pixel_size,
	void *stream);

/*
 * Batched reconstructions: many insertions of uneven box size and particle
 * count (classes, half-maps) in one set of launches, their work items
 * claimed by one persistent insertion launch. No operation of the reference
 * covers it (a rexlib caller runs one insert_*_slices per reconstruction);
 * the results are those of one rexlib_b200_insert_* call per job: the bits
 * of those calls in the deterministic mode, within the FP32 sum order in
 * the throughput mode.
 *
 * Each job is an rexlib_b200_insertion (its accumulators, slices, batch
 * strides and extents) with its weights (WEIGHTED: core (n, n/2+1)) or CTF
 * parameters (CTF: core (4)) in `extra`. The call's window, mode and element
 * type are those of jobs[0] (every job must agree; float32 only); the jobs'
 * workspace fields are ignored. At most 64 jobs a call; the jobs travel by
 * value in the kernels' parameters, so a call reads no host memory on the
 * GPU and captures into a CUDA graph.
 *
 * Throughput mode: the tile size and the run lengths of the work items are
 * chosen by an online tuner, per job set (the jobs' boxes and particle
 * counts in powers of two). The first calls of a new job set each try one
 * candidate (timed with CUDA events, results exact whatever the candidate);
 * once all are timed, later calls take the fastest. REXLIB_B200_TUNE_CACHE
 * names a file where chosen settings persist across processes. A call made
 * during stream capture takes the chosen setting or the default and times
 * nothing, so tune before capturing.
 */
typedef enum rexlib_b200_insertion_kind
{
	REXLIB_B200_KIND_PLAIN = 0,    /* insert_slices */
	REXLIB_B200_KIND_CTF = 1,      /* insert_ctf_slices */
	REXLIB_B200_KIND_WEIGHTED = 2  /* insert_weighted_slices */
} rexlib_b200_insertion_kind;

typedef struct rexlib_b200_insertion_job
{
	rexlib_b200_insertion insertion;
	const void *extra;
	rexlib_b200_batch_strides extra_strides;
} rexlib_b200_insertion_job;

/* A throughput tile setting: the cells of a tile and the shortest and
 * longest run of hits a work item takes. */
typedef struct rexlib_b200_tile_config
{
	int32_t cells;
	int32_t min_hits;
	int32_t max_hits;
} rexlib_b200_tile_config;

/* Device scratch a batched call needs (whatever setting the tuner picks),
 * 256-byte aligned. No counterpart in the reference. */
REXLIB_B200_API int32_t rexlib_b200_batched_insertion_workspace_size(const rexlib_b200_insertion_job *jobs,
	int32_t job_count, int32_t kind, size_t *bytes);

/* The batched insertion (see above). optics and pixel_size serve the CTF
 * kind. No counterpart in the reference. */
REXLIB_B200_API int32_t rexlib_b200_batched_insert(const rexlib_b200_insertion_job *jobs, int32_t job_count,
	int32_t kind, rexlib_b200_ctf_optics optics, double pixel_size, void *workspace, size_t workspace_bytes,
	void *stream);

/* The tuner's state for this job set: *tuned 1 with the chosen setting in
 * *config, or 0 (still trying candidates; *config the default). No
 * counterpart in the reference. */
REXLIB_B200_API int32_t rexlib_b200_batched_tuning(const rexlib_b200_insertion_job *jobs, int32_t job_count,
	int32_t kind, int32_t *tuned, rexlib_b200_tile_config *config);

/* Kernels of this library a batched call launches (besides accumulator
 * copies for distinct outputs). */
REXLIB_B200_API int32_t rexlib_b200_batched_insertion_launches(int32_t mode, int32_t *count);

/*
 * Background standardization of `batch` float32 images of rank 2 or 3
 * (contiguous, row-major; extents[0..rank-1]). Consecutive runs of
 * images_per_key images share one uint64 key: image b draws from
 * keys[b / images_per_key] at counters continuing from
 * (b % images_per_key) * image size, so 1 gives every image its own key and
 * `batch` makes one key serve all. statistics: optional device array
 * (batch, 2) receiving each image's second-pass mean and scale.
 */
typedef struct rexlib_b200_standardization
{
	float *result;
	const float *value;
	const uint64_t *keys;
	int64_t images_per_key;
	int64_t batch;
	int32_t rank;
	int64_t extents[3];
	double radius;
	double lower_bound;
	double upper_bound;
	double *statistics;
} rexlib_b200_standardization;

/*
 * em::standardize_background{,_2d,_3d} (src/em/functional/preprocessing.cpp:40-62;
 * operation include/rexlib/em/ops/preprocessing/standardize_background_operation.hpp:18-66):
 * the mean and standard deviation of the finite background (squared
 * distance from the centre above radius^2), again over the elements within
 * the bounds, then (x - mean) / std with out-of-bounds or non-finite elements
 * replaced by Philox4x32-10 Box-Muller draws.
 */
REXLIB_B200_API int32_t rexlib_b200_standardize_background(const rexlib_b200_standardization *standardization,
	void *stream);

/*
 * CTF epilogue of an R2C: mode 1 multiplies frequency k of image b by its
 * CTF c(k) (the expression of insert_ctf_slices_operation.hpp:40-55, with
 * k_y in fftfreq order) and writes c(k)^2 to `weights` when given; mode 2
 * multiplies by the sign of c(k) (a phase flip) and writes |c(k)|. ctf holds
 * (defocus U, defocus V, astigmatism angle, phase shift) per image at a
 * stride of ctf_stride floats (0 shares one set); `voltage` optionally gives
 * each image its own voltage in kV, else optics.voltage serves all.
 */
typedef struct rexlib_b200_ctf_epilogue
{
	int32_t mode;
	const float *ctf;
	int64_t ctf_stride;
	const float *voltage;
	rexlib_b200_ctf_optics optics;
	double pixel_size;
	float *weights;
} rexlib_b200_ctf_epilogue;

/*
 * rfft2 (include/rexlib/ops/fourier/rfft_operation.hpp; CPU:
 * src/backends/cpu/kernels/pocketfft_fourier_transform.cpp:129): the
 * unnormalised R2C of `batch` float images (n, n) into complex (n, n/2+1),
 * optionally followed by the CTF epilogue (NULL or mode 0: none). n in
 * {32, 64, 96, 128, 160, 192, 200, 256}.
 */
REXLIB_B200_API int32_t rexlib_b200_rfft2(void *out, const float *in, int64_t batch, int64_t n,
	const rexlib_b200_ctf_epilogue *epilogue, void *stream);

/*
 * standardize_background_2d followed by rfft2 with its CTF epilogue, in one
 * pass over the images: no reference operation fuses them (the reference
 * runs standardize_background_operation and then rfft_operation). The
 * standardization descriptor's value, keys, bounds, radius and statistics
 * mean what they mean for rexlib_b200_standardize_background; its result may
 * be NULL, in which case the standardized images are not written at all.
 * The spectra (and the epilogue's weights) are bit-identical to those of the
 * two calls. Square 2D images of 64, 128 or 256 only, 16-byte aligned;
 * other shapes return REXLIB_B200_UNSUPPORTED.
 */
REXLIB_B200_API int32_t rexlib_b200_standardize_rfft2(void *out, const rexlib_b200_standardization *standardization,
	const rexlib_b200_ctf_epilogue *epilogue, void *stream);

/*
 * irfft2 (include/rexlib/ops/fourier/irfft_operation.hpp; CPU:
 * pocketfft_fourier_transform.cpp:152): the C2R of complex (n, n/2+1) half
 * spectra into float (n, n), scaled by 1/n^2 (backward normalisation). n in
 * {32, 64, 96, 128, 160, 192, 200}.
 */
REXLIB_B200_API int32_t rexlib_b200_irfft2(float *out, const void *in, int64_t batch, int64_t n, void *stream);

/* Device scratch rexlib_b200_irfft3 and rexlib_b200_wiener_irfft3 need for
 * a volume of extent N, in bytes. */
REXLIB_B200_API int32_t rexlib_b200_irfft3_workspace_size(int64_t extent, size_t *bytes);

/*
 * irfft3: the C2R of a complex (N, N, N/2+1) half spectrum into a float
 * (N, N, N) volume, scaled by 1/N^3. N in {32, 64, 96, 128, 160, 192, 200, 256}.
 */
REXLIB_B200_API int32_t rexlib_b200_irfft3(float *out, const void *in, int64_t extent, void *workspace,
	size_t workspace_bytes, void *stream);

/* How the Wiener step divides: REGULARIZED gives X = N / (D + c) for every
 * voxel; THRESHOLD gives X = N / D where D > c and 0 elsewhere (the divide of
 * tests/integration/src/em/functional/test_cpu_reconstruction.cpp:457-464). */
typedef enum rexlib_b200_wiener_mode
{
	REXLIB_B200_WIENER_REGULARIZED = 0,
	REXLIB_B200_WIENER_THRESHOLD = 1
} rexlib_b200_wiener_mode;

/*
 * The Wiener divide of an insertion's accumulators followed by irfft3, the
 * divide fused into the first pass: volume = irfft3(numerator / denominator)
 * with the divide of `mode` and the constant c. The reference has no
 * operation for the divide; its test composes divide and irfft3
 * (test_cpu_reconstruction.cpp:457-470).
 */
REXLIB_B200_API int32_t rexlib_b200_wiener_irfft3(float *out, const void *numerator, const float *denominator,
	int64_t extent, int32_t mode, double constant, void *workspace, size_t workspace_bytes, void *stream);

/*
 * rfft3 (include/rexlib/ops/fourier/rfft_operation.hpp over three axes;
 * CPU: pocketfft_fourier_transform.cpp:129): the unnormalised R2C of a float
 * (N, N, N) volume into its complex (N, N, N/2+1) half spectrum, N in
 * {32, 64, 128, 256}.
 */
REXLIB_B200_API int32_t rexlib_b200_rfft3(void *out, const float *in, int64_t extent, void *stream);

/*
 * The learned prior's reconstruction loop (no counterpart in the reference):
 * - fsc: the Fourier shell correlation sums of two half spectra (N, N, N/2+1):
 *   sums[s], sums[S + s], sums[2 S + s] (S = N/2 + 1 shells, s = round |k|)
 *   receive sum Re(a conj b), sum |a|^2 and sum |b|^2 over the full spectrum;
 *   the correlation of shell s is the first over the root of the others.
 * - prior_wiener: out = (numerator + c prior) / (denominator + c), the data
 *   of an insertion's accumulators combined with a prior's spectrum.
 * - blob_spectrum: the half spectrum of sum_b a exp(-|p - N/2 - c|^2 / 2 s^2)
 *   over blobs (a, s, c_x, c_y, c_z), 5 floats each, zero beyond the shell
 *   `cutoff` (none when negative).
 * - phantom_slices: `slices` noisy central slices (n, n/2+1) of such a
 *   phantom (1 to 4096 blobs): for slice p, c(k) F(k_x A0 + k_y A1) + noise,
 *   F written for an image centred at n/2, A0 and A1 the first two rows of
 *   transforms (P, 3, 4), c the CTF of ctf (P, 4) (defocus U, V, angle,
 *   phase shift) as insert_ctf_slices evaluates it, the noise complex
 *   Gaussian of standard deviation `noise` per component (Philox keyed by
 *   seed + p).
 */
REXLIB_B200_API int32_t rexlib_b200_fsc(const void *a, const void *b, int64_t extent, double *sums, void *stream);
REXLIB_B200_API int32_t rexlib_b200_prior_wiener(void *out, const void *numerator, const float *denominator,
	const void *prior, int64_t extent, double constant, void *stream);
REXLIB_B200_API int32_t rexlib_b200_blob_spectrum(void *out, const float *blobs, int32_t count, int64_t extent,
	double cutoff, void *stream);
REXLIB_B200_API int32_t rexlib_b200_phantom_slices(void *out, const float *blobs, int32_t count, int64_t slices,
	int64_t extent, const float *transforms, const float *ctf, rexlib_b200_ctf_optics optics, double pixel_size,
	double noise, uint64_t seed, void *stream);

/*
 * fill (ops::fill_operation, include/rexlib/ops/assignment/fill_operation.hpp:33-42;
 * the zeros, ones, full and fill of src/functional/creation.cpp:301-346 and
 * 473-480): every element of the contiguous destination of `count` elements
 * of `type` set to *value, one element of that type in host memory.
 */
REXLIB_B200_API int32_t rexlib_b200_fill(void *destination, int32_t type, int64_t count, const void *value,
	void *stream);

/*
 * add and divide (ops::add_operation, ops::divide_operation,
 * include/rexlib/ops/arithmetic/add_operation.hpp:20-28 and
 * divide_operation.hpp:20-29; the CPU's elementwise kernels,
 * src/backends/cpu/builders/arithmetic/add_program_builder.cpp:22 and
 * divide_program_builder.cpp:22): result[i] = x[i] + y[i] or x[i] / y[i] over
 * `count` contiguous elements of one `type` (binary_homogeneous_rule). An
 * input of one element (x_count or y_count 1) is broadcast; otherwise its
 * count must be the result's. The result may be one of the inputs; partial
 * overlaps are not supported. Real division is IEEE. Complex division
 * gives the reference's results bit for bit as g++ compiles its
 * std::complex division: complex64 in double precision, complex128 by
 * Smith's method (away from the float64 overflow and underflow limits),
 * both with C's Annex G recovery of NaN quotients (x / 0 is infinite).
 */
REXLIB_B200_API int32_t rexlib_b200_add(void *result, const void *x, int64_t x_count, const void *y, int64_t y_count,
	int32_t type, int64_t count, void *stream);
REXLIB_B200_API int32_t rexlib_b200_divide(void *result, const void *x, int64_t x_count, const void *y,
	int64_t y_count, int32_t type, int64_t count, void *stream);

/*
 * The learned prior (a 3D U-Net regularising the reconstruction). No
 * counterpart in the reference: these entry points serve the prior only.
 *
 * 3x3x3 convolution, stride 1, zero padding 1, of channels-last BF16 volumes
 * (D, H, W, C) on the tcgen05 tensor cores, FP32 accumulation:
 *   out[v, o] = epilogue(bias[o] + sum over taps t and input channels i of
 *               in[v + t - 1, i] w[o, t, i])
 * with tap t = (dz * 3 + dy) * 3 + dx. The input channels are those of one
 * volume or of two concatenated (inputs[0] then inputs[1]); the weights are
 * BF16 (C_out, 27, C_in) over the concatenated channels. Epilogue 0 stores
 * the sum, 1 its ReLU, 2 the sum where masks[...] > 0 and 0 elsewhere (the
 * ReLU of a backward pass). The output channels may be split between two
 * volumes (outputs[0] takes the first output_split). D, H and W are powers
 * of two; every source has 16, 32 or a multiple of 64 channels (at most
 * 256); 16 to 128 output channels, a multiple of 16. Strides count
 * elements between voxels (multiples of 8), addresses are 16-byte aligned.
 * `error` (device, optional) receives a nonzero code if a wait inside the
 * kernel ran out of time. `wait_limit_ns` bounds each wait of the kernel's
 * pipeline (0: two seconds); a limit under a microsecond tests the barrier
 * once without waiting (a caller can make the waits run out on purpose to
 * check the error path). After a wait runs out the kernel stops issuing,
 * waits (at most two seconds each) for its copies and tensor-core
 * operations in flight, frees its tensor memory and returns.
 */
typedef struct rexlib_b200_conv3d_args
{
	int32_t sources;
	const void *inputs[2];
	int32_t input_channels[2];
	int32_t input_strides[2];
	int32_t depth, height, width;
	const void *weights;
	const float *bias;
	int32_t output_channels;
	int32_t epilogue;
	void *outputs[2];
	int32_t output_strides[2];
	int32_t output_split;
	const void *masks[2];
	int32_t mask_strides[2];
	int32_t *error;
	int64_t wait_limit_ns;
} rexlib_b200_conv3d_args;

REXLIB_B200_API int32_t rexlib_b200_conv3d(const rexlib_b200_conv3d_args *args, void *stream);

/*
 * Weight and bias gradients of rexlib_b200_conv3d, on the tcgen05 tensor
 * cores. For the output gradient g (voxels x output_channels BF16, rows of
 * output_grad_stride elements) and the convolution's input sources (their
 * channels concatenated, i running over all of them):
 *   weight_grad[o][t][i] += sum_v g[v][o] x[v + offset(t)][i]
 *   bias_grad[o]         += sum_v g[v][o]
 * in FP32, added to what the arrays hold (zero padding outside the volume;
 * tap t = 9 (dz + 1) + 3 (dy + 1) + (dx + 1), the weights' order).
 * bias_grad may be null. The same rules on extents, channels, strides and
 * alignment as the convolution, and a width of at least 16; output_channels
 * 16 to 128, a multiple of 16. The sums are taken in an unspecified order
 * (FP32 reductions from many CTAs). `error` and `wait_limit_ns` as for the
 * convolution.
 */
typedef struct rexlib_b200_conv3d_wgrad_args
{
	int32_t sources;
	const void *inputs[2];
	int32_t input_channels[2];
	int32_t input_strides[2];
	int32_t depth, height, width;
	const void *output_grad;
	int32_t output_channels;
	int32_t output_grad_stride;
	float *weight_grad;
	float *bias_grad;
	int32_t *error;
	int64_t wait_limit_ns;
} rexlib_b200_conv3d_wgrad_args;

REXLIB_B200_API int32_t rexlib_b200_conv3d_wgrad(const rexlib_b200_conv3d_wgrad_args *args, void *stream);

/*
 * The U-Net prior itself, for cubic volumes of extent N (16 to 512, a power
 * of two): four levels of 16, 32, 64 and 128 channels, two 3x3x3
 * convolutions with ReLU a level, 2x2x2 mean pooling, 2x2x2 stride-2
 * transposed convolutions, skip tensors concatenated in the decoder, a
 * 1x1x1 head added to the input (about 1.4 million FP32 parameters, Adam).
 * The network owns its device buffers (allocated at creation). Volumes are
 * FP32 (N, N, N) on the device; calls are stream-ordered.
 *   forward:  output = input + head(U-Net(input))
 *   backward: after a forward, adds the gradients of
 *             0.5 mean((output - target)^2) to the parameters' gradients
 *             and the loss to *loss (device FP32)
 *   adam_step: Adam (0.9, 0.999, 1e-8) at the learning rate, gradients
 *             cleared
 *   copy:     the FP32 parameters and gradients out, parameters in (to
 *             save or load a network)
 *   layer:    where a layer's weights and bias start in them, and its kind
 *             (0 first, 1 3x3x3, 2 transposed, 3 head) and channels
 */
typedef struct rexlib_b200_unet rexlib_b200_unet;
REXLIB_B200_API int32_t rexlib_b200_unet_create(int32_t extent, uint64_t seed, rexlib_b200_unet **net);
REXLIB_B200_API int32_t rexlib_b200_unet_destroy(rexlib_b200_unet *net);
REXLIB_B200_API int32_t rexlib_b200_unet_parameter_count(const rexlib_b200_unet *net, int64_t *count);
/* Copies the FP32 parameters and/or their gradients out (device or host
 * buffers of parameter_count floats), and/or new parameters in. */
REXLIB_B200_API int32_t rexlib_b200_unet_copy(rexlib_b200_unet *net, float *parameters_out, float *gradients_out,
	const float *parameters_in, void *stream);
/* Copies the BF16 output of layer `layer` (which 0) or its gradient
 * (which 1) after a forward (backward) pass, channels last; the head's
 * output is the forward's output. For tests and inspection. */
REXLIB_B200_API int32_t rexlib_b200_unet_tensor(rexlib_b200_unet *net, int32_t which, int32_t layer, void *out,
	void *stream);
REXLIB_B200_API int32_t rexlib_b200_unet_layer(const rexlib_b200_unet *net, int32_t layer, int64_t *weight_offset,
	int64_t *bias_offset, int32_t *shape);
REXLIB_B200_API int32_t rexlib_b200_unet_forward(rexlib_b200_unet *net, const float *input, float *output,
	void *stream);
REXLIB_B200_API int32_t rexlib_b200_unet_backward(rexlib_b200_unet *net, const float *target, float *loss,
	void *stream);
REXLIB_B200_API int32_t rexlib_b200_unet_adam_step(rexlib_b200_unet *net, float learning_rate, void *stream);
/* The device error word of the network's convolutions (nonzero: a wait ran
 * out of time); synchronizes. */
REXLIB_B200_API int32_t rexlib_b200_unet_error(rexlib_b200_unet *net, int32_t *code);

#ifdef __cplusplus
}
#endif

#endif /* REXLIB_B200_H */
