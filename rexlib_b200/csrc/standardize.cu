// Background standardization: one CTA per image.
//
// Follows the reference CPU backend (src/backends/cpu/builders/em/preprocessing):
//  - background: the squared integer distance from the centre extent/2
//    exceeds radius^2 (background_geometry.inl:41-100);
//  - two moment passes in FP64 over the finite background elements: pass 0
//    unbounded, pass 1 keeping the elements whose standardized value (with
//    the pass-0 statistics) lies within the bounds
//    (background_moments_kernel.inl:149-215, standardize_background_kernel.inl:26-50);
//  - finalize: mean = S/c, variance = Q/c - mean^2, scale = 1/sqrt(variance),
//    or 1 when the variance is not positive, and (0, 1) with no element
//    (background_moments_kernel.inl:125-145);
//  - map: (x - mean) * scale in float; an element that is not finite or
//    falls outside the bounds takes the Box-Muller draw of the Philox4x32-10
//    block (key, c / 2), cosine branch for even c
//    (standardization_map_kernel.inl:46-132, kernels/philox.inl:15-110,
//    kernels/standard_normal.inl:19-50).
// The image is read from HBM once: the second pass and the map re-read it
// from L2. The moment sums use a tree order, so the statistics match the
// CPU's to FP64 rounding rather than bit for bit.
#include "common.cuh"

#include <cfloat>
#include <cmath>

namespace rexlib_b200
{
namespace
{

constexpr int standardize_threads = 256;

struct standardize_launch
{
	float *result;
	const float *value;
	const uint64_t *keys;
	int64_t images_per_key;
	int64_t batch;
	int rank;
	int dims[3];
	int64_t size;
	int64_t radius_squared_floor; // floor(radius^2), capped
	double lower, upper;
	double *statistics;
};

__device__ __forceinline__ void philox_round(uint32_t c[4], uint32_t k0, uint32_t k1)
{
	const uint64_t p0 = static_cast<uint64_t>(0xD2511F53u) * c[0];
	const uint64_t p1 = static_cast<uint64_t>(0xCD9E8D57u) * c[2];
	const uint32_t n0 = static_cast<uint32_t>(p1 >> 32) ^ c[1] ^ k0;
	const uint32_t n2 = static_cast<uint32_t>(p0 >> 32) ^ c[3] ^ k1;
	c[0] = n0;
	c[1] = static_cast<uint32_t>(p1);
	c[2] = n2;
	c[3] = static_cast<uint32_t>(p0);
}

// Box-Muller pair of the draw block `block` under `key`.
__device__ __forceinline__ double2 normal_pair(uint64_t key, uint64_t block)
{
	uint32_t c[4] = {static_cast<uint32_t>(block), static_cast<uint32_t>(block >> 32), 0u, 0u};
	uint32_t k0 = static_cast<uint32_t>(key), k1 = static_cast<uint32_t>(key >> 32);
	philox_round(c, k0, k1);
	for (int round = 1; round < 10; ++round)
	{
		k0 += 0x9E3779B9u;
		k1 += 0xBB67AE85u;
		philox_round(c, k0, k1);
	}
	const uint64_t h0 = (static_cast<uint64_t>(c[1]) << 32) | c[0];
	const uint64_t h1 = (static_cast<uint64_t>(c[3]) << 32) | c[2];
	const double u0 = static_cast<double>((h0 >> 11) + 1) * (1.0 / 9007199254740992.0);
	const double u1 = static_cast<double>((h1 >> 11) + 1) * (1.0 / 9007199254740992.0);
	const double radius = sqrt(-2.0 * log(u0));
	double s, co;
	sincos(6.283185307179586476925 * u1, &s, &co);
	return make_double2(radius * co, radius * s);
}

struct moments
{
	double count, sum, squares;
};

__device__ __forceinline__ moments block_sum(moments m, double *scratch)
{
	for (int o = 16; o > 0; o >>= 1)
	{
		m.count += __shfl_xor_sync(0xffffffffu, m.count, o);
		m.sum += __shfl_xor_sync(0xffffffffu, m.sum, o);
		m.squares += __shfl_xor_sync(0xffffffffu, m.squares, o);
	}
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	const int warps = blockDim.x >> 5;
	__syncthreads();
	if (lane == 0)
	{
		scratch[3 * warp] = m.count;
		scratch[3 * warp + 1] = m.sum;
		scratch[3 * warp + 2] = m.squares;
	}
	__syncthreads();
	moments t{0.0, 0.0, 0.0};
	for (int w = 0; w < warps; ++w)
	{
		t.count += scratch[3 * w];
		t.sum += scratch[3 * w + 1];
		t.squares += scratch[3 * w + 2];
	}
	return t;
}

__device__ __forceinline__ void finalize(const moments &m, double &mean, double &scale)
{
	if (m.count == 0.0)
	{
		mean = 0.0;
		scale = 1.0;
		return;
	}
	mean = m.sum / m.count;
	const double variance = m.squares / m.count - mean * mean;
	scale = variance > 0.0 ? 1.0 / sqrt(variance) : 1.0;
}

// The image walked row by row (a row runs along the last axis): warps take
// rows, lanes take the elements of a row, so no element index is divided.
// An element is background when its integer squared distance d2 from the
// centre exceeds radius^2; for an integer d2 that is d2 > floor(radius^2).
template <typename Visit>
__device__ __forceinline__ void for_each_element(const standardize_launch &L, Visit &&visit)
{
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	const int warps = blockDim.x >> 5;
	const int width = L.dims[L.rank - 1];
	const int height = L.dims[L.rank - 2];
	const int depth = L.rank == 3 ? L.dims[0] : 1;
	const int cx = width / 2, cy = height / 2, cz = depth / 2;
	const int rows = height * depth;
	for (int r = warp; r < rows; r += warps)
	{
		const int z = r / height;
		const int y = r - z * height;
		const int64_t row_d2 = static_cast<int64_t>(y - cy) * (y - cy) +
			(L.rank == 3 ? static_cast<int64_t>(z - cz) * (z - cz) : 0);
		const int64_t base = static_cast<int64_t>(r) * width;
		for (int x = lane; x < width; x += 32)
		{
			const int64_t d2 = row_d2 + static_cast<int64_t>(x - cx) * (x - cx);
			visit(base + x, d2 > L.radius_squared_floor);
		}
	}
}

__global__ void __launch_bounds__(standardize_threads) standardize_kernel(const standardize_launch L)
{
	__shared__ double scratch[3 * (standardize_threads / 32)];
	const int64_t image = blockIdx.x;
	const float *in = L.value + image * L.size;
	float *out = L.result + image * L.size;

	double mean = 0.0, scale = 1.0;
	for (int pass = 0; pass < 2; ++pass)
	{
		const double lower = pass == 0 ? -INFINITY : L.lower;
		const double upper = pass == 0 ? INFINITY : L.upper;
		moments m{0.0, 0.0, 0.0};
		for_each_element(L, [&](int64_t i, bool background) {
			if (!background)
				return;
			const double x = static_cast<double>(__ldg(in + i));
			const double z = (x - mean) * scale;
			if ((fabs(x) <= DBL_MAX) && (z >= lower) && (z <= upper))
			{
				m.count += 1.0;
				m.sum += x;
				m.squares += x * x;
			}
		});
		const moments t = block_sum(m, scratch);
		finalize(t, mean, scale);
	}
	if (L.statistics && threadIdx.x == 0)
	{
		L.statistics[2 * image] = mean;
		L.statistics[2 * image + 1] = scale;
	}

	const float mean_f = static_cast<float>(mean), scale_f = static_cast<float>(scale);
	const float lower_f = static_cast<float>(L.lower), upper_f = static_cast<float>(L.upper);
	const uint64_t key = L.keys[image / L.images_per_key];
	const uint64_t counter0 = static_cast<uint64_t>(image % L.images_per_key) * static_cast<uint64_t>(L.size);
	for (int64_t i = threadIdx.x; i < L.size; i += blockDim.x)
	{
		const float z = __fmul_rn(__fsub_rn(__ldg(in + i), mean_f), scale_f);
		const bool kept = (z >= lower_f) & (z <= upper_f) & (fabsf(z) <= FLT_MAX);
		if (kept)
		{
			out[i] = z;
		}
		else
		{
			const uint64_t c = counter0 + static_cast<uint64_t>(i);
			const double2 pair = normal_pair(key, c >> 1);
			out[i] = static_cast<float>((c & 1) ? pair.y : pair.x);
		}
	}
}

} // anonymous namespace
} // namespace rexlib_b200

using namespace rexlib_b200;

extern "C" int32_t rexlib_b200_standardize_background(const rexlib_b200_standardization *s, void *stream)
{
	return guarded([&] {
		require(s != nullptr, "null standardization descriptor");
		require(s->rank == 2 || s->rank == 3, "images must have 2 or 3 axes");
		require(s->batch >= 0, "negative batch");
		// standardize_background_operation.cpp:17-39.
		require(s->radius >= 0.0, "standardize_background: the radius must be 0 or more");
		require(s->lower_bound < 0.0 && s->upper_bound > 0.0,
			"standardize_background: the bounds must lie on either side of 0");
		require(s->images_per_key >= 1, "images_per_key must be 1 or more");
		standardize_launch L{};
		L.size = 1;
		for (int a = 0; a < s->rank; ++a)
		{
			require(s->extents[a] >= 1 && s->extents[a] <= (1 << 20), "image extents must lie in [1, 2^20]");
			L.dims[a] = static_cast<int>(s->extents[a]);
			L.size *= s->extents[a];
		}
		if (s->batch == 0 || L.size == 0)
			return;
		require(s->result && s->value && s->keys, "null operand");
		require(s->batch <= 0x7fffffffLL, "too many images in one call");
		L.result = s->result;
		L.value = s->value;
		L.keys = s->keys;
		L.images_per_key = s->images_per_key;
		L.batch = s->batch;
		L.rank = s->rank;
		// An integer d2 exceeds radius^2 exactly when it exceeds floor(radius^2).
		const double r2 = s->radius * s->radius;
		L.radius_squared_floor = r2 >= 9.0e18 ? INT64_MAX : static_cast<int64_t>(std::floor(r2));
		L.lower = s->lower_bound;
		L.upper = s->upper_bound;
		L.statistics = s->statistics;
		standardize_kernel<<<static_cast<unsigned>(s->batch), standardize_threads, 0, as_stream(stream)>>>(L);
		check_cuda(cudaGetLastError(), "standardization launch");
	});
}
