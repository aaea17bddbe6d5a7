// The array operations that callers of the reconstruction path run on the
// device arrays between its steps: fill (ops::fill_operation,
// include/rexlib/ops/assignment/fill_operation.hpp; the zeros of
// src/functional/creation.cpp), add and divide (ops::add_operation,
// ops::divide_operation, include/rexlib/ops/arithmetic/; the CPU's
// elementwise kernels, src/backends/cpu/builders/arithmetic/
// add_program_builder.cpp and divide_program_builder.cpp).
//
// Every operand has one element type (binary_homogeneous_rule): float32,
// float64, complex64 or complex128. Operands are contiguous; an input of one
// element is broadcast over the result, the one form of broadcasting served
// here (a plugin answers backend_priority::unsupported for the others).
// Division is IEEE for the real types. Complex division reproduces what the
// reference's std::complex division compiles to with g++ (libgcc's complex
// division): complex64 in double precision, complex128 by Smith's method
// (R. L. Smith, "Algorithm 116: Complex division", CACM 5(8), 1962), both
// followed by C's Annex G recovery of NaN quotients. For complex128 operands
// near the float64 overflow and underflow limits libgcc also rescales them
// and reorders the products; that is not reproduced, so the last bits there
// may differ.
//
// The work is bound by HBM bandwidth. A grid-stride loop over packs of
// 16 bytes (4, 2, 2 or 1 elements) runs when every array operand is 16-byte
// aligned, with the last count mod pack elements done one by one; otherwise
// the loop goes element by element.
#include "common.cuh"

#include <algorithm>
#include <cstring>

namespace rexlib_b200
{
namespace
{

constexpr int array_threads = 256;
#ifndef REXLIB_B200_DIVIDE_DEPTH
#define REXLIB_B200_DIVIDE_DEPTH 2
#endif
constexpr int array_divide_depth = REXLIB_B200_DIVIDE_DEPTH;

enum class binary_op
{
	add,
	divide
};

// The recovery of C's Annex G (ISO/IEC 9899, G.5.1) for a quotient whose
// parts both came out NaN: a zero divisor gives infinities, an infinite
// dividend over a finite divisor infinities, and a finite dividend over an
// infinite divisor zeros.
template <typename R>
__device__ __forceinline__ void recover_nan_quotient(R a, R b, R c, R d, R &x, R &y)
{
	if (!(isnan(x) && isnan(y)))
		return;
	const R inf = R(INFINITY);
	if (c == R(0) && d == R(0) && (!isnan(a) || !isnan(b)))
	{
		x = copysign(inf, c) * a;
		y = copysign(inf, c) * b;
	}
	else if ((isinf(a) || isinf(b)) && isfinite(c) && isfinite(d))
	{
		a = copysign(isinf(a) ? R(1) : R(0), a);
		b = copysign(isinf(b) ? R(1) : R(0), b);
		x = inf * (a * c + b * d);
		y = inf * (b * c - a * d);
	}
	else if ((isinf(c) || isinf(d)) && isfinite(a) && isfinite(b))
	{
		c = copysign(isinf(c) ? R(1) : R(0), c);
		d = copysign(isinf(d) ? R(1) : R(0), d);
		x = R(0) * (a * c + b * d);
		y = R(0) * (b * c - a * d);
	}
}

// complex64: (ac + bd, bc - ad) / (c^2 + d^2) evaluated in double precision
// (the products of two floats are exact there), each part rounded to float
// once at the end. This is how the host compiler's runtime divides the
// std::complex<float> values of the reference's kernel, bit for bit.
__device__ __forceinline__ float2 complex_divide(float2 p, float2 q)
{
	const double a = p.x, b = p.y, c = q.x, d = q.y;
	const double denom = __dadd_rn(__dmul_rn(c, c), __dmul_rn(d, d));
	float x = __double2float_rn(__ddiv_rn(__dadd_rn(__dmul_rn(a, c), __dmul_rn(b, d)), denom));
	float y = __double2float_rn(__ddiv_rn(__dsub_rn(__dmul_rn(b, c), __dmul_rn(a, d)), denom));
	recover_nan_quotient(p.x, p.y, q.x, q.y, x, y);
	return make_float2(x, y);
}

// complex128: Smith's method, dividing through by the larger part of the
// divisor, every operation rounded as written.
__device__ __forceinline__ double2 complex_divide(double2 p, double2 q)
{
	const double a = p.x, b = p.y, c = q.x, d = q.y;
	double x, y;
	if (fabs(c) >= fabs(d))
	{
		const double r = __ddiv_rn(d, c), den = __dadd_rn(c, __dmul_rn(d, r));
		x = __ddiv_rn(__dadd_rn(a, __dmul_rn(b, r)), den);
		y = __ddiv_rn(__dsub_rn(b, __dmul_rn(a, r)), den);
	}
	else
	{
		const double r = __ddiv_rn(c, d), den = __dadd_rn(__dmul_rn(c, r), d);
		x = __ddiv_rn(__dadd_rn(__dmul_rn(a, r), b), den);
		y = __ddiv_rn(__dsub_rn(__dmul_rn(b, r), a), den);
	}
	recover_nan_quotient(a, b, c, d, x, y);
	return make_double2(x, y);
}

template <binary_op OP>
__device__ __forceinline__ float apply(float a, float b)
{
	return OP == binary_op::add ? __fadd_rn(a, b) : __fdiv_rn(a, b);
}

template <binary_op OP>
__device__ __forceinline__ double apply(double a, double b)
{
	return OP == binary_op::add ? __dadd_rn(a, b) : __ddiv_rn(a, b);
}

template <binary_op OP>
__device__ __forceinline__ float2 apply(float2 a, float2 b)
{
	if constexpr (OP == binary_op::add)
		return make_float2(__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y));
	else
		return complex_divide(a, b);
}

template <binary_op OP>
__device__ __forceinline__ double2 apply(double2 a, double2 b)
{
	if constexpr (OP == binary_op::add)
		return make_double2(__dadd_rn(a.x, b.x), __dadd_rn(a.y, b.y));
	else
		return complex_divide(a, b);
}

// A pack of 16 bytes.
template <typename T>
struct alignas(16) pack
{
	static constexpr int size = 16 / sizeof(T);
	T v[size];
};

// DEPTH packs a thread are loaded before any is computed: the division's
// double-precision chain would otherwise hold back the next loads and leave
// too few bytes in flight to keep HBM busy.
template <typename T, binary_op OP, int DEPTH>
__global__ void __launch_bounds__(array_threads) binary_packed_kernel(T *out, const T *x, const T *y,
	int64_t packs, bool x_scalar, bool y_scalar)
{
	using P = pack<T>;
	const T xs = x_scalar ? x[0] : T{};
	const T ys = y_scalar ? y[0] : T{};
	const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
	for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < packs; i += DEPTH * stride)
	{
		P a[DEPTH], b[DEPTH];
#pragma unroll
		for (int u = 0; u < DEPTH; ++u)
		{
			if (i + u * stride < packs)
			{
				if (!x_scalar)
					a[u] = reinterpret_cast<const P *>(x)[i + u * stride];
				if (!y_scalar)
					b[u] = reinterpret_cast<const P *>(y)[i + u * stride];
			}
		}
#pragma unroll
		for (int u = 0; u < DEPTH; ++u)
		{
			if (i + u * stride < packs)
			{
				P r;
#pragma unroll
				for (int e = 0; e < P::size; ++e)
					r.v[e] = apply<OP>(x_scalar ? xs : a[u].v[e], y_scalar ? ys : b[u].v[e]);
				reinterpret_cast<P *>(out)[i + u * stride] = r;
			}
		}
	}
}

template <typename T, binary_op OP>
__global__ void __launch_bounds__(array_threads) binary_kernel(T *out, const T *x, const T *y, int64_t first,
	int64_t count, bool x_scalar, bool y_scalar)
{
	const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
	for (int64_t i = first + static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < count; i += stride)
		out[i] = apply<OP>(x[x_scalar ? 0 : i], y[y_scalar ? 0 : i]);
}

template <typename T>
__global__ void __launch_bounds__(array_threads) fill_packed_kernel(T *out, T value, int64_t packs)
{
	using P = pack<T>;
	P p;
#pragma unroll
	for (int e = 0; e < P::size; ++e)
		p.v[e] = value;
	const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
	for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < packs; i += stride)
		reinterpret_cast<P *>(out)[i] = p;
}

template <typename T>
__global__ void __launch_bounds__(array_threads) fill_kernel(T *out, T value, int64_t first, int64_t count)
{
	const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
	for (int64_t i = first + static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < count; i += stride)
		out[i] = value;
}

// As many CTAs of KERNEL as are resident at once on all SMs (one wave of
// the grid-stride loop), fewer when the work is small. The occupancy is
// looked up once per kernel.
template <auto KERNEL>
unsigned grid_for(int64_t items)
{
	static const int resident = [] {
		int blocks = 0;
		check_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, KERNEL, array_threads, 0),
			"occupancy query");
		return std::max(blocks, 1);
	}();
	int device = 0, sms = 0;
	check_cuda(cudaGetDevice(&device), "device query");
	check_cuda(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "device query");
	const int64_t wanted = (items + array_threads - 1) / array_threads;
	return static_cast<unsigned>(
		std::max<int64_t>(1, std::min<int64_t>(wanted, static_cast<int64_t>(sms) * resident)));
}

bool aligned16(const void *p) { return reinterpret_cast<uintptr_t>(p) % 16 == 0; }

template <typename T, binary_op OP>
void launch_binary(void *result, const void *x, int64_t x_count, const void *y, int64_t y_count, int64_t count,
	cudaStream_t stream)
{
	T *out = static_cast<T *>(result);
	const T *a = static_cast<const T *>(x);
	const T *b = static_cast<const T *>(y);
	const bool x_scalar = x_count == 1 && count != 1;
	const bool y_scalar = y_count == 1 && count != 1;
	int64_t done = 0;
	if (aligned16(out) && (x_scalar || aligned16(a)) && (y_scalar || aligned16(b)))
	{
		const int64_t packs = count / pack<T>::size;
		if (packs > 0)
		{
			constexpr int depth = OP == binary_op::divide ? array_divide_depth : 1;
			constexpr auto kernel = binary_packed_kernel<T, OP, depth>;
			kernel<<<grid_for<kernel>((packs + depth - 1) / depth), array_threads, 0, stream>>>(out, a, b, packs,
				x_scalar, y_scalar);
			check_cuda(cudaGetLastError(), "elementwise launch");
		}
		done = packs * pack<T>::size;
	}
	if (done < count)
	{
		constexpr auto kernel = binary_kernel<T, OP>;
		kernel<<<grid_for<kernel>(count - done), array_threads, 0, stream>>>(out, a, b, done, count, x_scalar,
			y_scalar);
		check_cuda(cudaGetLastError(), "elementwise launch");
	}
}

template <typename T>
void launch_fill(void *destination, const void *value, int64_t count, cudaStream_t stream)
{
	T *out = static_cast<T *>(destination);
	T v;
	std::memcpy(&v, value, sizeof(T));
	int64_t done = 0;
	if (aligned16(out))
	{
		const int64_t packs = count / pack<T>::size;
		if (packs > 0)
		{
			constexpr auto kernel = fill_packed_kernel<T>;
			kernel<<<grid_for<kernel>(packs), array_threads, 0, stream>>>(out, v, packs);
			check_cuda(cudaGetLastError(), "fill launch");
		}
		done = packs * pack<T>::size;
	}
	if (done < count)
	{
		constexpr auto kernel = fill_kernel<T>;
		kernel<<<grid_for<kernel>(count - done), array_threads, 0, stream>>>(out, v, done, count);
		check_cuda(cudaGetLastError(), "fill launch");
	}
}

void check_type(int32_t type)
{
	if (type != REXLIB_B200_FLOAT32 && type != REXLIB_B200_FLOAT64 && type != REXLIB_B200_COMPLEX64 &&
		type != REXLIB_B200_COMPLEX128)
		fail(REXLIB_B200_UNSUPPORTED, "element type not served: float32, float64, complex64 and complex128 are");
}

template <binary_op OP>
void run_binary(void *result, const void *x, int64_t x_count, const void *y, int64_t y_count, int32_t type,
	int64_t count, void *stream)
{
	check_type(type);
	require(count >= 0, "negative element count");
	require(x_count == count || x_count == 1, "the dividend or augend must have the result's count or one element");
	require(y_count == count || y_count == 1, "the divisor or addend must have the result's count or one element");
	if (count == 0)
		return;
	require(result && x && y, "null operand");
	const cudaStream_t s = as_stream(stream);
	switch (type)
	{
	case REXLIB_B200_FLOAT32:
		launch_binary<float, OP>(result, x, x_count, y, y_count, count, s);
		break;
	case REXLIB_B200_FLOAT64:
		launch_binary<double, OP>(result, x, x_count, y, y_count, count, s);
		break;
	case REXLIB_B200_COMPLEX64:
		launch_binary<float2, OP>(result, x, x_count, y, y_count, count, s);
		break;
	default:
		launch_binary<double2, OP>(result, x, x_count, y, y_count, count, s);
		break;
	}
}

} // anonymous namespace
} // namespace rexlib_b200

using namespace rexlib_b200;

extern "C" int32_t rexlib_b200_fill(void *destination, int32_t type, int64_t count, const void *value, void *stream)
{
	return guarded([&] {
		check_type(type);
		require(count >= 0, "negative element count");
		require(value != nullptr, "null fill value");
		if (count == 0)
			return;
		require(destination != nullptr, "null destination");
		const cudaStream_t s = as_stream(stream);
		switch (type)
		{
		case REXLIB_B200_FLOAT32:
			launch_fill<float>(destination, value, count, s);
			break;
		case REXLIB_B200_FLOAT64:
			launch_fill<double>(destination, value, count, s);
			break;
		case REXLIB_B200_COMPLEX64:
			launch_fill<float2>(destination, value, count, s);
			break;
		default:
			launch_fill<double2>(destination, value, count, s);
			break;
		}
	});
}

extern "C" int32_t rexlib_b200_add(void *result, const void *x, int64_t x_count, const void *y, int64_t y_count,
	int32_t type, int64_t count, void *stream)
{
	return guarded([&] { run_binary<binary_op::add>(result, x, x_count, y, y_count, type, count, stream); });
}

extern "C" int32_t rexlib_b200_divide(void *result, const void *x, int64_t x_count, const void *y, int64_t y_count,
	int32_t type, int64_t count, void *stream)
{
	return guarded([&] { run_binary<binary_op::divide>(result, x, x_count, y, y_count, type, count, stream); });
}
