/*
 * Oracle (test infrastructure only): background standardization restated in
 * C from the reference CPU backend.
 *
 *  - background: squared integer distance from the centre extent/2 above
 *    radius^2 (builders/em/preprocessing/background_geometry.inl:41-100);
 *  - moments: count, sum and sum of squares in FP64 over the background
 *    elements that are finite and whose standardized value lies within the
 *    bounds; pass 0 with mean 0, scale 1 and unbounded, pass 1 with the pass-0
 *    statistics and the bounds (background_moments_kernel.inl:60-215,
 *    standardize_background_kernel.inl:26-50);
 *  - finalize: mean = S/c, variance = Q/c - mean^2, scale = 1/sqrt(variance)
 *    or 1, and (0, 1) without a valid element (background_moments_kernel.inl:125-145);
 *  - map: (x - mean) * scale in the element type; an element that is not
 *    finite or lies outside the bounds is replaced by
 *    standard_normal_pair(key, c / 2)[c % 2], with c the row-major position
 *    among the elements sharing the key (standardization_map_kernel.inl:46-132,
 *    standardize_background_operation.hpp:37-60).
 * The FP64 sums run in the reference's order: per row, four lanes over the
 * runs either side of the excluded disc, lanes merged in order.
 */
#include "oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>

typedef struct
{
	double mean, scale, lower, upper;
} moments_bounds;

static int is_valid(double x, const moments_bounds *b)
{
	const double z = (x - b->mean) * b->scale;
	return (fabs(x) <= DBL_MAX) & (z >= b->lower) & (z <= b->upper);
}

/* Half-width of the excluded run along the inner axis at squared distance
 * d2 over the other axes (compute_half_width). */
static long excluded_half_width(long d2, long extent, double r2)
{
	const long widest = extent;
	if ((double)(d2 + widest * widest) <= r2)
		return extent;
	long result = (long)sqrt(r2 - (double)d2);
	result = result < widest ? result : widest;
	while (result > 0 && !((double)(d2 + result * result) <= r2))
		--result;
	while (result < widest && (double)(d2 + (result + 1) * (result + 1)) <= r2)
		++result;
	return result;
}

#define DEFINE_STANDARDIZE(SUFFIX, T, TMAX)                                                          \
	static void fold_##SUFFIX(const T *row, long first, long last, const moments_bounds *b,         \
		long *total, double *sum, double *sq)                                                        \
	{                                                                                                \
		long counts[4] = { 0, 0, 0, 0 };                                                             \
		double sums[4] = { 0, 0, 0, 0 }, squares[4] = { 0, 0, 0, 0 };                               \
		long position = first;                                                                       \
		for (; position + 4 <= last; position += 4)                                                  \
			for (int lane = 0; lane < 4; ++lane)                                                     \
			{                                                                                        \
				const double x = (double)row[position + lane];                                       \
				const int valid = is_valid(x, b);                                                    \
				const double kept = valid ? x : 0.0;                                                 \
				counts[lane] += valid ? 1 : 0;                                                       \
				sums[lane] += kept;                                                                  \
				squares[lane] += kept * kept;                                                        \
			}                                                                                        \
		for (; position < last; ++position)                                                          \
		{                                                                                            \
			const double x = (double)row[position];                                                  \
			const int valid = is_valid(x, b);                                                        \
			const double kept = valid ? x : 0.0;                                                     \
			counts[0] += valid ? 1 : 0;                                                              \
			sums[0] += kept;                                                                         \
			squares[0] += kept * kept;                                                               \
		}                                                                                            \
		for (int lane = 0; lane < 4; ++lane)                                                         \
		{                                                                                            \
			*total += counts[lane];                                                                  \
			*sum += sums[lane];                                                                      \
			*sq += squares[lane];                                                                    \
		}                                                                                            \
	}                                                                                                \
                                                                                                     \
	int oracle_standardize_##SUFFIX(T *result, const T *value, const uint64_t *keys, long batch,     \
		int rank, const long *dims, int key_per_image, double radius, double lower_bound,            \
		double upper_bound, double *statistics)                                                      \
	{                                                                                                \
		const double r2 = radius * radius;                                                           \
		long size = 1;                                                                               \
		for (int a = 0; a < rank; ++a)                                                               \
			size *= dims[a];                                                                         \
		const long width = dims[rank - 1];                                                           \
		const long rows = size / width;                                                              \
		for (long b = 0; b < batch; ++b)                                                             \
		{                                                                                            \
			const T *img = value + (size_t)b * size;                                                 \
			T *out = result + (size_t)b * size;                                                      \
			double mean = 0.0, scl = 1.0;                                                            \
			for (int pass = 0; pass < 2; ++pass)                                                     \
			{                                                                                        \
				moments_bounds bounds;                                                               \
				if (pass == 0)                                                                       \
				{                                                                                    \
					bounds.mean = 0.0;                                                               \
					bounds.scale = 1.0;                                                              \
					bounds.lower = -INFINITY;                                                        \
					bounds.upper = INFINITY;                                                         \
				}                                                                                    \
				else                                                                                 \
				{                                                                                    \
					bounds.mean = mean;                                                              \
					bounds.scale = scl;                                                              \
					bounds.lower = lower_bound;                                                      \
					bounds.upper = upper_bound;                                                      \
				}                                                                                    \
				long total = 0;                                                                      \
				double sum = 0.0, sq = 0.0;                                                          \
				for (long r = 0; r < rows; ++r)                                                      \
				{                                                                                    \
					long rem = r, d2 = 0;                                                            \
					for (int a = rank - 2; a >= 0; --a)                                              \
					{                                                                                \
						const long i = rem % dims[a];                                                \
						rem /= dims[a];                                                              \
						const long d = i - dims[a] / 2;                                              \
						d2 += d * d;                                                                 \
					}                                                                                \
					long ex_first = 0, ex_second = 0;                                                \
					if (!((double)d2 > r2))                                                          \
					{                                                                                \
						const long hw = excluded_half_width(d2, width, r2);                          \
						const long c = width / 2;                                                    \
						long lo = c - hw, hi = c + hw + 1;                                           \
						lo = lo < 0 ? 0 : (lo > width ? width : lo);                                 \
						hi = hi < 0 ? 0 : (hi > width ? width : hi);                                 \
						ex_first = lo;                                                               \
						ex_second = hi;                                                              \
					}                                                                                \
					const T *row = img + (size_t)r * width;                                          \
					fold_##SUFFIX(row, 0, ex_first, &bounds, &total, &sum, &sq);                     \
					fold_##SUFFIX(row, ex_second, width, &bounds, &total, &sum, &sq);              \
				}                                                                                    \
				if (total == 0)                                                                      \
				{                                                                                    \
					mean = 0.0;                                                                      \
					scl = 1.0;                                                                       \
				}                                                                                    \
				else                                                                                 \
				{                                                                                    \
					const double t = (double)total;                                                  \
					mean = sum / t;                                                                  \
					const double variance = sq / t - mean * mean;                                    \
					scl = variance > 0.0 ? 1.0 / sqrt(variance) : 1.0;                               \
				}                                                                                    \
			}                                                                                        \
			if (statistics)                                                                          \
			{                                                                                        \
				statistics[2 * b] = mean;                                                            \
				statistics[2 * b + 1] = scl;                                                         \
			}                                                                                        \
			const T m = (T)mean, s = (T)scl, lo = (T)lower_bound, hi = (T)upper_bound;               \
			const uint64_t key = key_per_image ? keys[b] : keys[0];                                  \
			const uint64_t counter0 = key_per_image ? 0 : (uint64_t)b * (uint64_t)size;              \
			for (long i = 0; i < size; ++i)                                                          \
			{                                                                                        \
				const T z = ((T)img[i] - m) * s;                                                     \
				const T az = z < (T)0 ? -z : z;                                                      \
				const int kept = (z >= lo) & (z <= hi) & (az <= TMAX);                               \
				if (kept)                                                                            \
				{                                                                                    \
					out[i] = z;                                                                      \
				}                                                                                    \
				else                                                                                 \
				{                                                                                    \
					const uint64_t c = counter0 + (uint64_t)i;                                       \
					double pair[2];                                                                  \
					oracle_standard_normal_pair(key, c / 2, pair);                                   \
					out[i] = (T)pair[c % 2];                                                         \
				}                                                                                    \
			}                                                                                        \
		}                                                                                            \
		return 0;                                                                                    \
	}

DEFINE_STANDARDIZE(f32, float, FLT_MAX)
DEFINE_STANDARDIZE(f64, double, DBL_MAX)

void oracle_background_mask(uint8_t *mask, int rank, const long *dims, double radius)
{
	const double r2 = radius * radius;
	long size = 1;
	for (int a = 0; a < rank; ++a)
		size *= dims[a];
	for (long i = 0; i < size; ++i)
	{
		long rem = i, d2 = 0;
		for (int a = rank - 1; a >= 0; --a)
		{
			const long j = rem % dims[a];
			rem /= dims[a];
			const long d = j - dims[a] / 2;
			d2 += d * d;
		}
		mask[i] = (double)d2 > r2 ? 1 : 0;
	}
}
