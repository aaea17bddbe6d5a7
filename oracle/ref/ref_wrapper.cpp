// Test infrastructure only: a C entry layer over the reference's own CPU
// implementation of the em reconstruction path, compiled from the reference
// sources where they lie (see oracle/ref/Makefile). Nothing in the product
// links this; tests and the bench's reference arm load it as the checker and
// the CPU baseline.
//
// The functors called here are the reference CPU backend's:
// - slice_insertion_functor<T, SampleWeight>
//   (src/backends/cpu/builders/em/reconstruction/slice_insertion_functor.inl:52-290)
//   with the plan of slice_insertion_layout_plan
//   (src/backends/cpu/plans/slice_insertion_layout_plan.cpp:81-185);
// - standardize_background_kernel with background_moments_kernel and
//   standardization_map_kernel
//   (src/backends/cpu/builders/em/preprocessing/*.inl), driven per image the
//   way batch_reduce_map_program_builder.inl:176-197 drives them;
// - philox4x32_10 and standard_normal_pair (src/backends/cpu/kernels/).

#include <backends/cpu/builders/em/reconstruction/ctf_weight.hpp>
#include <backends/cpu/builders/em/reconstruction/slice_insertion_functor.hpp>
#include <backends/cpu/builders/em/reconstruction/spectrum_weight.hpp>
#include <backends/cpu/builders/em/reconstruction/unit_weight.hpp>
#include <backends/cpu/builders/em/preprocessing/standardize_background_kernel.hpp>
#include <backends/cpu/kernels/contrast_transfer_function.hpp>
#include <backends/cpu/kernels/philox.hpp>
#include <backends/cpu/kernels/standard_normal.hpp>
#include <backends/cpu/loops/linear_index_run.hpp>
#include <backends/cpu/loops/multidimensional_index.hpp>

#include <rexlib/backends/cpu/thread_pool.hpp>
#include <rexlib/core/dispatch/operand_descriptor.hpp>
#include <rexlib/core/layout/strided_layout.hpp>
#include <rexlib/em/ops/parameters/ctf_optics.hpp>
#include <rexlib/em/ops/parameters/gridding_window.hpp>

#include <complex>
#include <cstdint>
#include <cstring>
#include <exception>
#include <memory>
#include <string>
#include <tuple>
#include <vector>

using namespace rexlib;

namespace
{

thread_local std::string last_error;

std::unique_ptr<cpu::thread_pool> &pool_slot()
{
	static std::unique_ptr<cpu::thread_pool> pool;
	return pool;
}

cpu::thread_pool &get_pool(int threads)
{
	auto &pool = pool_slot();
	const auto wanted = static_cast<std::size_t>(threads < 1 ? 1 : threads);
	if (!pool || pool->get_size() != wanted)
	{
		pool.reset();
		pool.reset(new cpu::thread_pool(wanted));
	}
	return *pool;
}

operand_descriptor describe(std::vector<std::size_t> extents, numerical_type type)
{
	return operand_descriptor(
		strided_layout::make_contiguous_layout(make_span(extents)),
		type
	);
}

em::gridding_window make_window(int profile, double half_width, double shape)
{
	switch (profile)
	{
	case 0:
		return em::gridding_window::nearest();
	case 1:
		return em::gridding_window::linear();
	default:
		return em::gridding_window::kaiser_bessel(half_width, shape);
	}
}

// The inputs of each variant, in the order of its operation's operands.
template <typename T>
void call_functor(
	const cpu::slice_insertion_functor<T, cpu::unit_weight> &functor,
	std::complex<T> *numerator, T *denominator, const std::complex<T> *slices,
	const T *, const T *transforms, const T *radial, cpu::thread_pool &pool)
{
	functor(
		std::make_tuple(numerator, denominator),
		std::make_tuple(
			static_cast<const std::complex<T>*>(numerator),
			static_cast<const T*>(denominator), slices, transforms, radial),
		std::tuple<>(), pool);
}

template <typename T>
void call_functor(
	const cpu::slice_insertion_functor<T, cpu::ctf_weight> &functor,
	std::complex<T> *numerator, T *denominator, const std::complex<T> *slices,
	const T *ctf, const T *transforms, const T *radial, cpu::thread_pool &pool)
{
	functor(
		std::make_tuple(numerator, denominator),
		std::make_tuple(
			static_cast<const std::complex<T>*>(numerator),
			static_cast<const T*>(denominator), slices, transforms, ctf, radial),
		std::tuple<>(), pool);
}

template <typename T>
void call_functor(
	const cpu::slice_insertion_functor<T, cpu::spectrum_weight> &functor,
	std::complex<T> *numerator, T *denominator, const std::complex<T> *slices,
	const T *weight, const T *transforms, const T *radial, cpu::thread_pool &pool)
{
	functor(
		std::make_tuple(numerator, denominator),
		std::make_tuple(
			static_cast<const std::complex<T>*>(numerator),
			static_cast<const T*>(denominator), slices, weight, transforms, radial),
		std::tuple<>(), pool);
}

// Shapes: accumulators (V, 1, N, N, H); slices (P, n, h) shared by every
// volume or (V, P, n, h); transforms (V, P, 3, 4); radial (h) or (P, h);
// ctf (P, 4) or (V, P, 4); weights like the slices.
template <typename T, typename SampleWeight>
int run_insertion(
	const typename SampleWeight::parameters_type &parameters,
	int kind,
	std::complex<T> *numerator,
	T *denominator,
	const std::complex<T> *slices,
	const T *extra,
	const T *transforms,
	const T *radial,
	long volumes,
	long particles,
	long n,
	long big,
	int slices_per_volume,
	int radial_per_particle,
	int extra_per_particle,
	int profile,
	double half_width,
	double shape,
	int threads
)
{
	const auto type = sizeof(T) == 4 ? numerical_type::float32 : numerical_type::float64;
	const auto ctype = sizeof(T) == 4 ? numerical_type::complex_float32 : numerical_type::complex_float64;
	const std::size_t V = static_cast<std::size_t>(volumes);
	const std::size_t P = static_cast<std::size_t>(particles);
	const std::size_t h = static_cast<std::size_t>(n / 2 + 1);
	const std::size_t N = static_cast<std::size_t>(big);
	const std::size_t H = N / 2 + 1;
	const std::size_t sn = static_cast<std::size_t>(n);

	std::vector<operand_descriptor> outs;
	outs.push_back(describe({V, 1, N, N, H}, ctype));
	outs.push_back(describe({V, 1, N, N, H}, type));

	std::vector<operand_descriptor> ins;
	ins.push_back(describe({V, 1, N, N, H}, ctype));
	ins.push_back(describe({V, 1, N, N, H}, type));
	if (slices_per_volume)
		ins.push_back(describe({V, P, sn, h}, ctype));
	else
		ins.push_back(describe({P, sn, h}, ctype));
	std::vector<std::size_t> ranks = {3, 3, 2};
	if (kind == 2)
	{
		// weighted: weight after slice
		if (extra_per_particle)
			ins.push_back(describe({P, sn, h}, type));
		else
			ins.push_back(describe({sn, h}, type));
		ranks.push_back(2);
	}
	ins.push_back(describe({V, P, 3, 4}, type));
	ranks.push_back(2);
	if (kind == 1)
	{
		if (extra_per_particle)
			ins.push_back(describe({V, P, 4}, type));
		else
			ins.push_back(describe({4}, type));
		ranks.push_back(1);
	}
	if (radial_per_particle)
		ins.push_back(describe({P, h}, type));
	else
		ins.push_back(describe({h}, type));
	ranks.push_back(1);

	cpu::slice_insertion_layout_plan plan(
		make_span(outs), make_span(ins), make_span(ranks)
	);
	cpu::slice_insertion_functor<T, SampleWeight> functor(
		std::move(plan),
		make_window(profile, half_width, shape),
		parameters,
		cpu::slice_insertion_tuning()
	);
	auto &pool = get_pool(threads);
	call_functor(functor, numerator, denominator, slices, extra, transforms, radial, pool);
	return 0;
}

template <typename T>
int run_insert_any(
	int kind,
	void *numerator, void *denominator, const void *slices, const void *extra,
	const void *transforms, const void *radial,
	long volumes, long particles, long n, long big,
	int slices_per_volume, int radial_per_particle, int extra_per_particle,
	int profile, double half_width, double shape,
	double voltage, double cs, double q, double pixel_size, int threads)
{
	auto *num = static_cast<std::complex<T>*>(numerator);
	auto *den = static_cast<T*>(denominator);
	const auto *sl = static_cast<const std::complex<T>*>(slices);
	const auto *ex = static_cast<const T*>(extra);
	const auto *tr = static_cast<const T*>(transforms);
	const auto *ra = static_cast<const T*>(radial);
	if (kind == 0)
		return run_insertion<T, cpu::unit_weight>(
			cpu::unit_weight::parameters_type(), 0, num, den, sl, ex, tr, ra,
			volumes, particles, n, big, slices_per_volume, radial_per_particle,
			extra_per_particle, profile, half_width, shape, threads);
	if (kind == 1)
		return run_insertion<T, cpu::ctf_weight>(
			cpu::ctf_weight::parameters_type(em::ctf_optics(voltage, cs, q), pixel_size),
			1, num, den, sl, ex, tr, ra,
			volumes, particles, n, big, slices_per_volume, radial_per_particle,
			extra_per_particle, profile, half_width, shape, threads);
	return run_insertion<T, cpu::spectrum_weight>(
		cpu::spectrum_weight::parameters_type(), 2, num, den, sl, ex, tr, ra,
		volumes, particles, n, big, slices_per_volume, radial_per_particle,
		extra_per_particle, profile, half_width, shape, threads);
}

// One image through the reference's standardization kernels: two moment
// passes over rows (the inner axis) and the map over the image as one run,
// as batch_reduce_map_program_builder.inl:176-197 sequences them.
template <typename T>
void standardize_image(
	const cpu::standardize_background_kernel &kernel,
	T *out, const T *in, std::uint64_t key, std::size_t counter,
	int rank, const long *dims, double *statistics)
{
	std::size_t size = 1;
	for (int a = 0; a < rank; ++a)
		size *= static_cast<std::size_t>(dims[a]);
	const std::size_t width = static_cast<std::size_t>(dims[rank - 1]);
	const std::size_t rows = size / width;
	cpu::standardize_background_kernel::statistics_type stats = {{ 0.0, 1.0 }};
	for (std::size_t pass = 0; pass < 2; ++pass)
	{
		const auto reduction = kernel.make_reduction(pass, stats);
		std::size_t count = 0;
		double sum = 0.0, squares = 0.0;
		std::vector<std::ptrdiff_t> coordinates(static_cast<std::size_t>(rank), 0);
		for (std::size_t r = 0; r < rows; ++r)
		{
			std::size_t rem = r;
			for (int a = rank - 2; a >= 0; --a)
			{
				coordinates[static_cast<std::size_t>(a)] =
					static_cast<std::ptrdiff_t>(rem % static_cast<std::size_t>(dims[a]));
				rem /= static_cast<std::size_t>(dims[a]);
			}
			coordinates[static_cast<std::size_t>(rank - 1)] = 0;
			const auto index = cpu::multidimensional_index(
				static_cast<std::size_t>(rank), static_cast<std::size_t>(rank - 1)
			).rebased(coordinates.data());
			reduction.combine_run(
				std::make_tuple(&count, &sum, &squares),
				std::make_tuple(in + r * width),
				std::make_tuple(std::ptrdiff_t(1)),
				width,
				index
			);
		}
		reduction.finalize(&stats[0], &stats[1], count, sum, squares, size);
	}
	if (statistics)
	{
		statistics[0] = stats[0];
		statistics[1] = stats[1];
	}
	const std::uint64_t *key_pointer = &key;
	const auto map = kernel.make_map(stats, std::make_tuple(in, key_pointer), counter);
	map(
		std::make_tuple(out, in),
		std::make_tuple(std::ptrdiff_t(1), std::ptrdiff_t(1)),
		size,
		cpu::linear_index_run<std::ptrdiff_t>(0, 1)
	);
}

} // anonymous namespace

extern "C" {

// Background standardization of `batch` images (rank 2 or 3) through the
// reference kernels. keys: one per image, or one shared (counter continues).
int ref_standardize(
	int dtype, void *result, const void *value, const uint64_t *keys,
	long batch, int rank, const long *dims, int key_per_image,
	double radius, double lower, double upper, double *statistics)
{
	try
	{
		std::vector<std::size_t> extents;
		std::size_t size = 1;
		for (int a = 0; a < rank; ++a)
		{
			extents.push_back(static_cast<std::size_t>(dims[a]));
			size *= extents.back();
		}
		const cpu::standardize_background_kernel kernel(
			cpu::background_geometry(make_span(extents), radius), lower, upper);
		for (long b = 0; b < batch; ++b)
		{
			const auto key = key_per_image ? keys[b] : keys[0];
			const std::size_t counter = key_per_image ? 0 : static_cast<std::size_t>(b) * size;
			double *stats = statistics ? statistics + 2 * b : nullptr;
			if (dtype == 8)
				standardize_image<double>(kernel,
					static_cast<double*>(result) + b * size,
					static_cast<const double*>(value) + b * size,
					key, counter, rank, dims, stats);
			else
				standardize_image<float>(kernel,
					static_cast<float*>(result) + b * size,
					static_cast<const float*>(value) + b * size,
					key, counter, rank, dims, stats);
		}
		return 0;
	}
	catch (const std::exception &e)
	{
		last_error = e.what();
		return 1;
	}
}


const char *ref_last_error(void) { return last_error.c_str(); }

// kind: 0 insert_slices, 1 insert_ctf_slices (extra = ctf), 2 insert_weighted_slices (extra = weight).
// dtype: 4 float32, 8 float64. Accumulates in place into numerator/denominator.
int ref_insert(
	int kind, int dtype,
	void *numerator, void *denominator, const void *slices, const void *extra,
	const void *transforms, const void *radial,
	long volumes, long particles, long n, long big,
	int slices_per_volume, int radial_per_particle, int extra_per_particle,
	int profile, double half_width, double shape,
	double voltage, double cs, double q, double pixel_size, int threads)
{
	try
	{
		if (dtype == 8)
			return run_insert_any<double>(kind, numerator, denominator, slices, extra,
				transforms, radial, volumes, particles, n, big, slices_per_volume,
				radial_per_particle, extra_per_particle, profile, half_width, shape,
				voltage, cs, q, pixel_size, threads);
		return run_insert_any<float>(kind, numerator, denominator, slices, extra,
			transforms, radial, volumes, particles, n, big, slices_per_volume,
			radial_per_particle, extra_per_particle, profile, half_width, shape,
			voltage, cs, q, pixel_size, threads);
	}
	catch (const std::exception &e)
	{
		last_error = e.what();
		return 1;
	}
}

void ref_philox4x32_10(const uint32_t counter[4], const uint32_t key[2], uint32_t out[4])
{
	const auto result = cpu::philox4x32_10(
		{{ counter[0], counter[1], counter[2], counter[3] }},
		{{ key[0], key[1] }}
	);
	for (int i = 0; i < 4; ++i)
		out[i] = result[i];
}

void ref_standard_normal_pair(uint64_t key, uint64_t block, double out[2])
{
	const auto pair = cpu::standard_normal_pair(key, block);
	out[0] = pair[0];
	out[1] = pair[1];
}

// CTF c(k) at (k_x, k_y) in float32, as the insertion evaluates it.
float ref_ctf(double voltage, double cs, double q, double pixel_size, long extent,
	double du, double dv, double angle, double shift, float kx, float ky)
{
	const cpu::contrast_transfer_function<float> f(
		em::ctf_optics(voltage, cs, q), pixel_size,
		static_cast<std::size_t>(extent), du, dv, angle, shift);
	return f(kx, ky);
}

} // extern "C"
