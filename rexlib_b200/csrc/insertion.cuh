// Fourier-slice insertion: shared definitions of the insertion kernels.
//
// Semantics follow the reference CPU backend (all paths relative to the
// reference's src/backends/cpu): rows and columns of a slice from
// builders/em/reconstruction/slice_insertion_functor.inl:339-393, sample
// preparation from row_insertion_kernel.inl:139-285, the scatter from
// row_insertion_kernel.inl:288-360, windows from kernels/*_window.inl, the
// CTF from kernels/contrast_transfer_function.inl:26-87.
#pragma once

#include "common.cuh"

namespace rexlib_b200
{

// Largest Kaiser-Bessel table a launch carries by value (1024 entries per
// voxel of half-width, plus three): half-widths up to 7 in float, up to 3 in
// double (the table is held in the element type, as the CPU holds it, and a
// kernel's parameters are limited to 32 KB).
constexpr int kb_table_capacity = 7 * 1024 + 3;
constexpr int kb_table_capacity_f64 = 3 * 1024 + 3;
constexpr int max_taps = 15;

template <typename T>
struct complex_of;
template <>
struct complex_of<float>
{
	using type = float2;
};
template <>
struct complex_of<double>
{
	using type = double2;
};
template <typename T>
using complex_t = typename complex_of<T>::type;

enum class weight_kind : int
{
	unit = 0,
	ctf = 1,
	spectrum = 2
};

template <typename T, int CAPACITY>
struct kb_table_of
{
	T half_width;
	T scale;
	int step_count;
	int tap_count;
	T values[CAPACITY];
};
using kb_table = kb_table_of<float, kb_table_capacity>;
// The table of a batched call (half-widths up to 2), small enough to travel
// in the kernels' parameters beside the jobs.
constexpr int kb_table_capacity_batch = 2056;
using kb_table_batch = kb_table_of<float, kb_table_capacity_batch>;
using kb_table_f64 = kb_table_of<double, kb_table_capacity_f64>;

// Per-launch operands and constants of an insertion whose operands hold
// elements of T (float or double; complex ones as pairs of T).
template <typename T>
struct insertion_launch_of
{
	complex_t<T> *numerator;
	T *denominator;
	const complex_t<T> *slices;
	const T *transforms;
	const T *radial;
	const T *extra;
	int64_t slice_stride_v, slice_stride_p;
	int64_t transform_stride_v, transform_stride_p;
	int64_t radial_stride_v, radial_stride_p;
	int64_t extra_stride_v, extra_stride_p;
	int64_t volumes, particles;
	int n, h, big, big_h;
	int profile;
	int tap_count;
	// CTF constants of the launch, FP64 (ctf_weight / contrast_transfer_function).
	double ctf_wavelength;
	double ctf_aberration;   // Cs in angstroms
	double ctf_phase_offset; // asin(Q)
	double ctf_frequency_scale_sq;
};
using insertion_launch = insertion_launch_of<float>;

// What the batched calls' tuner varies: the cells of a throughput tile
// (its L2 numerator) and the shortest and longest run of hits a work item
// takes. Zero fields keep the defaults.
struct tile_config
{
	int cells;
	int min_hits;
	int max_hits;
};

// floor(c) as an int: one conversion rounding toward minus infinity.
__device__ __forceinline__ int floor_int(float c) { return __float2int_rd(c); }
__device__ __forceinline__ int floor_int(double c) { return __double2int_rd(c); }
__device__ __forceinline__ float magnitude(float x) { return fabsf(x); }
__device__ __forceinline__ double magnitude(double x) { return fabs(x); }

// Round-half-up shell of |k| by the integer test of
// row_insertion_kernel.inl:195-219: (s + 1/2)^2 <= |k|^2 moves to s + 1.
// For integer m = |k|^2 the shell s satisfies s^2 - s < m <= s^2 + s, and
// sqrt(m) stays at least 1/(8 s + 4) away from every half-integer, far more
// than float's rounding for m < 2^22; so floor(sqrt(m) + 1/2) in float is
// exact there. Larger m (beyond any supported slice) take the integer test.
__device__ __forceinline__ int shell_of(int kx, int ky)
{
	const int m = kx * kx + ky * ky;
	int s = static_cast<int>(sqrtf(static_cast<float>(m)) + 0.5f);
	if (m >= (1 << 22))
	{
		while (s > 0 && 4 * (s - 1) * (s - 1) + 4 * (s - 1) + 1 > 4 * m)
			--s;
		while (4 * s * s + 4 * s + 1 <= 4 * m)
			++s;
	}
	return s;
}

// Window placement on one axis (kernels/box_window.inl:18-33,
// kernels/triangle_window.inl:18-35, kernels/kaiser_bessel_window.inl:80-136),
// in the element type T.
template <int PROFILE, typename T, typename KB>
__device__ __forceinline__ int place(T c, T *w, const KB *kb)
{
	if constexpr (PROFILE == REXLIB_B200_WINDOW_BOX)
	{
		const T half = c < T(0) ? T(-0.5) : T(0.5);
		w[0] = T(1);
		return static_cast<int>(fadd(c, half));
	}
	else if constexpr (PROFILE == REXLIB_B200_WINDOW_TRIANGLE)
	{
		const int below = floor_int(c); // floor(c)
		const T fraction = fsub(c, static_cast<T>(below));
		w[0] = fsub(T(1), fraction);
		w[1] = fraction;
		return below;
	}
	else
	{
		const int first = floor_int(fsub(c, kb->half_width)) + 1; // floor(c - w) + 1
		for (int t = 0; t < kb->tap_count; ++t)
		{
			const T distance = magnitude(fsub(static_cast<T>(first + t), c));
			const T position = fmul(distance, kb->scale);
			const int step = static_cast<int>(position);
			const int index = step < kb->step_count ? step : kb->step_count + 1;
			const T fraction = fsub(position, static_cast<T>(index));
			const T below = kb->values[index];
			w[t] = fadd(below, fmul(fraction, fsub(kb->values[index + 1], below)));
		}
		return first;
	}
}

template <int PROFILE, typename KB>
__device__ __forceinline__ int taps_of(const KB *kb)
{
	if constexpr (PROFILE == REXLIB_B200_WINDOW_BOX)
		return 1;
	else if constexpr (PROFILE == REXLIB_B200_WINDOW_TRIANGLE)
		return 2;
	else
		return kb->tap_count;
}

template <int PROFILE>
constexpr int weight_capacity()
{
	return PROFILE == REXLIB_B200_WINDOW_BOX ? 1 : (PROFILE == REXLIB_B200_WINDOW_TRIANGLE ? 2 : max_taps);
}

// Host-side launch entries of the scatter kernels.
void launch_insert_scatter(const insertion_launch &launch, weight_kind kind, const kb_table *kb,
	bool odd_volume, cudaStream_t stream);
void launch_insert_scatter(const insertion_launch_of<double> &launch, weight_kind kind, const kb_table_f64 *kb,
	bool odd_volume, cudaStream_t stream);

} // namespace rexlib_b200
