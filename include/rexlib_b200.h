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

#define REXLIB_B200_ABI_VERSION 1

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
 * (slice, then sample order), so runs are bit-identical. */
typedef enum rexlib_b200_insert_mode
{
	REXLIB_B200_INSERT_THROUGHPUT = 0,
	REXLIB_B200_INSERT_DETERMINISTIC = 1
} rexlib_b200_insert_mode;

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
 *   denominator_in/out  (V, N, N, N/2+1) float
 *   slices              core (n, n/2+1) complex
 *   transforms          core (3, 4) float, [A | t]
 *   radial_weights      core (n/2+1) float
 *
 * The outputs are the inputs plus the insertions. Passing the same pointer
 * for an input and its output updates in place; the inputs are copied to
 * the outputs first otherwise (insert_slices_operation.hpp:50-52). The
 * workspace is device memory of rexlib_b200_insertion_workspace_size() bytes
 * (the program's scratch requirement, include/rexlib/core/hardware/program.hpp:63).
 */
typedef struct rexlib_b200_insertion
{
	void *numerator_out;
	float *denominator_out;
	const void *numerator_in;
	const float *denominator_in;
	const void *slices;
	const float *transforms;
	const float *radial_weights;
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
} rexlib_b200_insertion;

/* The calling thread's last error message ("" if none). */
REXLIB_B200_API const char *rexlib_b200_last_error(void);

/* REXLIB_B200_ABI_VERSION of the library. */
REXLIB_B200_API int32_t rexlib_b200_abi_version(void);

/* Device scratch an insertion call needs, in bytes (0 when none). */
REXLIB_B200_API int32_t rexlib_b200_insertion_workspace_size(const rexlib_b200_insertion *insertion, size_t *bytes);

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
 * kappa r W(k). weights: core (n, n/2+1) float.
 */
REXLIB_B200_API int32_t rexlib_b200_insert_weighted_slices(
	const rexlib_b200_insertion *insertion,
	const float *weights,
	rexlib_b200_batch_strides weight_strides,
	void *stream);

/*
 * em::insert_ctf_slices (src/em/functional/reconstruction.cpp:107-138;
 * insert_ctf_slices_operation.hpp:33-67): the numerator receives
 * kappa r c(k) v, the denominator kappa r c(k)^2. ctf: core (4) float:
 * defocus U, defocus V (angstroms), astigmatism angle, phase shift (radians).
 */
REXLIB_B200_API int32_t rexlib_b200_insert_ctf_slices(
	const rexlib_b200_insertion *insertion,
	const float *ctf,
	rexlib_b200_batch_strides ctf_strides,
	rexlib_b200_ctf_optics optics,
	double pixel_size,
	void *stream);

#ifdef __cplusplus
}
#endif

#endif /* REXLIB_B200_H */
