// Background standardization: the device code shared by the standardization
// kernels (standardize.cu) and the R2C kernels that standardize an image they
// have staged in shared memory before transforming it (fft2.cu).
//
// Follows the reference CPU backend (src/backends/cpu/builders/em/preprocessing):
// background_geometry.inl:41-100 (the background test),
// background_moments_kernel.inl:125-215 and standardize_background_kernel.inl:26-50
// (the two FP64 moment passes and their finalize),
// standardization_map_kernel.inl:46-132 (the map and its draws),
// kernels/philox.inl:15-110 and kernels/standard_normal.inl:19-50 (the draws).
#pragma once

#include "common.cuh"

#include <cfloat>
#include <cmath>

namespace rexlib_b200
{

// Threads of every CTA that runs the resident standardization.
constexpr int resident_threads = 256;

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

// Shape of a resident image: 16-byte chunks of 4 elements, w4 chunks a row.
// A thread takes chunks tid, tid + 256, ...; between its chunks the row
// advances by step_rows and the chunk column by step_cols (256 = step_rows *
// w4 + step_cols), so no chunk index is divided.
// Chunk j = row * w4 + col of the image sits at chunk row * pitch + col of
// the staging buffer: pitch = w4 for a contiguous copy, more for a buffer
// whose rows are padded (the R2C kernels' spectrum rows).
struct resident_shape
{
	int chunks, w4, step_rows, step_cols;
	int cx, cy;
	int radius_squared; // floor(radius^2) capped at INT_MAX; every d2 here is below it
	int pitch;
};

// Moments of the finite background elements of a resident image; with
// BOUNDED, only those whose value standardized with (mean, scale) lies in
// [lower, upper]. The bound test runs in FP32 first, with a margin of 2^-18
// of the magnitudes involved (far above the few roundings between the FP32
// and FP64 values); only an element within that margin of a bound takes the
// FP64 test, which decides exactly as the CPU does.
// The chunks [first, end) of the image, chunk j at s_image[row * pitch + col - first].
template <bool BOUNDED>
__device__ __forceinline__ moments resident_moments(const float4 *s_image, const resident_shape &R, int first,
	int end, double mean, double scale, double lower, double upper)
{
	const float mean_f = static_cast<float>(mean), scale_f = static_cast<float>(scale);
	const float lower_f = static_cast<float>(lower), upper_f = static_cast<float>(upper);
	int count = 0;
	double sum = 0.0, squares = 0.0;
	const int start = first + static_cast<int>(threadIdx.x);
	int row = start / R.w4, col = start - row * R.w4;
	// Unrolled so that a thread's chunk loads are in flight together: the
	// fused 256 R2C walks its share straight from global memory.
#pragma unroll 16
	for (int j = start; j < end; j += resident_threads)
	{
		const float4 q = s_image[row * R.pitch + col - first];
		const float e[4] = {q.x, q.y, q.z, q.w};
		const int dy = row - R.cy;
#pragma unroll
		for (int u = 0; u < 4; ++u)
		{
			const int dx = 4 * col + u - R.cx;
			if (dy * dy + dx * dx <= R.radius_squared || !(fabsf(e[u]) <= FLT_MAX))
				continue;
			if constexpr (BOUNDED)
			{
				const float z = (e[u] - mean_f) * scale_f;
				const float margin = ((fabsf(e[u]) + fabsf(mean_f)) * scale_f + fabsf(z)) * 3.814697265625e-6f;
				bool inside;
				if (z - margin >= lower_f && z + margin <= upper_f)
					inside = true;
				else if (z + margin < lower_f || z - margin > upper_f)
					inside = false;
				else
				{
					const double zd = (static_cast<double>(e[u]) - mean) * scale;
					inside = zd >= lower && zd <= upper;
				}
				if (!inside)
					continue;
			}
			const double x = static_cast<double>(e[u]);
			++count;
			sum += x;
			squares += x * x;
		}
		row += R.step_rows;
		col += R.step_cols;
		if (col >= R.w4)
		{
			col -= R.w4;
			++row;
		}
	}
	return moments{static_cast<double>(count), sum, squares};
}

// Standardizes a 2D image staged whole in shared memory by this CTA
// (resident_threads threads): both moment passes, the statistics when asked
// for, and the map. Each mapped chunk is streamed to `out` when it is not
// null and, with IN_PLACE, written back over the staged chunk.
template <bool IN_PLACE>
__device__ __forceinline__ void standardize_resident(const standardize_launch &L, const resident_shape &R,
	float4 *s_image, int64_t image, double *scratch, float4 *out)
{
	// Pass 0 over every finite background element; pass 1 keeps those within
	// the bounds, which is pass 0 again when the bounds are infinite.
	double mean = 0.0, scale = 1.0;
	finalize(block_sum(resident_moments<false>(s_image, R, 0, R.chunks, 0.0, 1.0, 0.0, 0.0), scratch), mean, scale);
	if (L.lower != -INFINITY || L.upper != INFINITY)
		finalize(block_sum(resident_moments<true>(s_image, R, 0, R.chunks, mean, scale, L.lower, L.upper), scratch), mean,
			scale);
	if (L.statistics && threadIdx.x == 0)
	{
		L.statistics[2 * image] = mean;
		L.statistics[2 * image + 1] = scale;
	}

	const float mean_f = static_cast<float>(mean), scale_f = static_cast<float>(scale);
	const float lower_f = static_cast<float>(L.lower), upper_f = static_cast<float>(L.upper);
	const uint64_t key = L.keys[image / L.images_per_key];
	const uint64_t counter0 = static_cast<uint64_t>(image % L.images_per_key) * static_cast<uint64_t>(L.size);
	int row = static_cast<int>(threadIdx.x) / R.w4, col = static_cast<int>(threadIdx.x) - row * R.w4;
	for (int j = threadIdx.x; j < R.chunks; j += resident_threads)
	{
		float4 *slot = s_image + row * R.pitch + col;
		const float4 q = *slot;
		float e[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
		for (int u = 0; u < 4; ++u)
		{
			const float z = __fmul_rn(__fsub_rn(e[u], mean_f), scale_f);
			const bool kept = (z >= lower_f) & (z <= upper_f) & (fabsf(z) <= FLT_MAX);
			if (kept)
			{
				e[u] = z;
			}
			else
			{
				const uint64_t c = counter0 + 4 * static_cast<uint64_t>(j) + u;
				const double2 pair = normal_pair(key, c >> 1);
				e[u] = static_cast<float>((c & 1) ? pair.y : pair.x);
			}
		}
		const float4 r = make_float4(e[0], e[1], e[2], e[3]);
		if (out)
			__stcs(out + j, r);
		if constexpr (IN_PLACE)
			*slot = r;
		row += R.step_rows;
		col += R.step_cols;
		if (col >= R.w4)
		{
			col -= R.w4;
			++row;
		}
	}
}

// The moments of every CTA's share of an image held by a cluster of C CTAs,
// summed in rank order, so every CTA of the cluster gets the same bits: each
// CTA writes its share into slot `rank` of every CTA's `slots` (distributed
// shared memory), and after a cluster barrier sums the C slots. `slots`
// holds C sets of (count, sum, squares) for this pass.
template <int C, typename Cluster>
__device__ __forceinline__ moments cluster_moments(Cluster &cluster, double (*slots)[3], int rank,
	const moments &share)
{
	if (threadIdx.x < C)
	{
		double *slot = cluster.map_shared_rank(&slots[rank][0], static_cast<int>(threadIdx.x));
		slot[0] = share.count;
		slot[1] = share.sum;
		slot[2] = share.squares;
	}
	cluster.sync();
	moments t{0.0, 0.0, 0.0};
	for (int r = 0; r < C; ++r)
	{
		t.count += slots[r][0];
		t.sum += slots[r][1];
		t.squares += slots[r][2];
	}
	return t;
}

// Element c of an image standardized with (mean, scale) in float, or, when
// it is not finite or falls outside [lower, upper], the Box-Muller draw of
// the Philox block (key, c / 2) (cosine branch for even c), for the pair of
// elements 2 i, 2 i + 1 whose counter of the first is `c_even`.
__device__ __forceinline__ float2 standardize_pair(float2 q, float mean_f, float scale_f, float lower_f, float upper_f,
	uint64_t key, uint64_t c_even)
{
	float z0 = __fmul_rn(__fsub_rn(q.x, mean_f), scale_f);
	float z1 = __fmul_rn(__fsub_rn(q.y, mean_f), scale_f);
	const bool kept0 = (z0 >= lower_f) & (z0 <= upper_f) & (fabsf(z0) <= FLT_MAX);
	const bool kept1 = (z1 >= lower_f) & (z1 <= upper_f) & (fabsf(z1) <= FLT_MAX);
	if (!(kept0 && kept1))
	{
		const double2 pair = normal_pair(key, c_even >> 1);
		if (!kept0)
			z0 = static_cast<float>(pair.x);
		if (!kept1)
			z1 = static_cast<float>(pair.y);
	}
	return make_float2(z0, z1);
}

// The launch of a standardization descriptor, checked as the reference's
// operation checks it (standardize_background_operation.cpp:17-39). Returns
// false when there is nothing to do (an empty batch or image).
bool standardize_plan(const rexlib_b200_standardization *s, standardize_launch &L);

// The resident shape of a 2D image of L, staged with `pitch` chunks a row.
resident_shape resident_shape_of(const standardize_launch &L, int pitch);

} // namespace rexlib_b200
