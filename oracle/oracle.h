/*
 * Oracle: a plain-C restatement of the reference CPU backend's em
 * reconstruction path. TEST INFRASTRUCTURE ONLY: tests, the smoke check and
 * the bench's CPU-baseline leg load it as the checker; the product never
 * links, loads or calls it.
 *
 * Pinned against (a) the reference's own CPU functors compiled from its
 * sources (oracle/ref, libref_strict.so: bit-identical float32 and float64
 * results expected) and (b) the known answers of the reference's tests
 * (Philox4x32-10 vectors, uniform/normal draws, CTF at k = 0), committed as
 * fixtures under tests/golden.
 *
 * Layouts (row-major, contiguous):
 *   numerator   (V, N, N, H) complex (re, im interleaved), H = N / 2 + 1
 *   denominator (V, N, N, H) real
 *   slices      (P, n, h) complex, or (V, P, n, h) with slices_per_volume
 *   transforms  (V, P, 3, 4)
 *   radial      (h), or (P, h) with radial_per_particle
 *   ctf         (4) or (V, P, 4) with extra_per_particle   [kind 1]
 *   weight      (n, h) or (P, n, h) with extra_per_particle [kind 2]
 */
#ifndef REXLIB_B200_ORACLE_H
#define REXLIB_B200_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* kind: 0 insert_slices, 1 insert_ctf_slices, 2 insert_weighted_slices.
 * profile: 0 nearest (box), 1 linear (triangle), 2 Kaiser-Bessel.
 * Accumulates into numerator/denominator in place. Returns 0. */
int oracle_insert_f32(
	int kind, float *numerator, float *denominator, const float *slices,
	const float *extra, const float *transforms, const float *radial,
	long volumes, long particles, long n, long big,
	int slices_per_volume, int radial_per_particle, int extra_per_particle,
	int profile, double half_width, double shape,
	double voltage, double cs, double amplitude_contrast, double pixel_size);

int oracle_insert_f64(
	int kind, double *numerator, double *denominator, const double *slices,
	const double *extra, const double *transforms, const double *radial,
	long volumes, long particles, long n, long big,
	int slices_per_volume, int radial_per_particle, int extra_per_particle,
	int profile, double half_width, double shape,
	double voltage, double cs, double amplitude_contrast, double pixel_size);

/* Philox4x32-10 block. */
void oracle_philox4x32_10(const uint32_t counter[4], const uint32_t key[2], uint32_t out[4]);

/* Box-Muller pair of the draw block `block` under `key`. */
void oracle_standard_normal_pair(uint64_t key, uint64_t block, double out[2]);

/* uniform_open_closed of 64 random bits. */
double oracle_uniform_open_closed(uint64_t bits);

/* derive_key(key, data): word pair 0 of the key-derivation block. */
uint64_t oracle_derive_key(uint64_t key, uint64_t data);

/* CTF c(k) evaluated in float32 the way the insertion does. */
float oracle_ctf_f32(double voltage, double cs, double amplitude_contrast,
	double pixel_size, long extent, double defocus_u, double defocus_v,
	double angle, double phase_shift, float k_x, float k_y);

/* Background standardization of `batch` images of rank `rank` (2 or 3),
 * extents dims[0..rank-1]. keys holds `batch` keys when key_per_image,
 * else one key shared by every image. statistics (optional, 2 * batch
 * doubles) receives the second-pass mean and scale of each image. */
int oracle_standardize_f32(
	float *result, const float *value, const uint64_t *keys,
	long batch, int rank, const long *dims, int key_per_image,
	double radius, double lower_bound, double upper_bound,
	double *statistics);

int oracle_standardize_f64(
	double *result, const double *value, const uint64_t *keys,
	long batch, int rank, const long *dims, int key_per_image,
	double radius, double lower_bound, double upper_bound,
	double *statistics);

/* Background mask of one image: 1 where background. */
void oracle_background_mask(uint8_t *mask, int rank, const long *dims, double radius);

#ifdef __cplusplus
}
#endif

#endif
