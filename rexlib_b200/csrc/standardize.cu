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
// A 2D image of up to 96 KB whose rows are a multiple of 4 elements stays
// resident: the CTA stages it in shared memory with 16-byte cp.async copies,
// runs both passes and the map from there and streams the result out, so
// HBM sees one read and one write per element. A larger 2D image (up to
// 768 KB, 256^2 among them) stays resident on a cluster of 2, 4 or 8 CTAs:
// each stages a contiguous share of it, and the moments of the shares meet
// through distributed shared memory. Other images (3D, wider) are walked
// from global memory: the second pass and the map re-read them from L2. The
// moment sums use a tree order, so the statistics match the CPU's to FP64
// rounding rather than bit for bit.
#include "standardize.cuh"

#include <algorithm>
#include <cfloat>
#include <climits>
#include <cmath>

#include <cooperative_groups.h>

namespace rexlib_b200
{
namespace
{

constexpr int standardize_threads = 256;
constexpr size_t resident_max_bytes = 96 * 1024;

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

__global__ void __launch_bounds__(resident_threads) standardize_resident_kernel(const standardize_launch L,
	const resident_shape R)
{
	extern __shared__ float4 s_image[];
	__shared__ double scratch[3 * (resident_threads / 32)];
	const int64_t image = blockIdx.x;
	const float4 *in = reinterpret_cast<const float4 *>(L.value + image * L.size);
	float4 *out = reinterpret_cast<float4 *>(L.result + image * L.size);
	for (int j = threadIdx.x; j < R.chunks; j += resident_threads)
	{
		const unsigned dst = static_cast<unsigned>(__cvta_generic_to_shared(s_image + j));
		asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(in + j) : "memory");
	}
	asm volatile("cp.async.wait_all;" ::: "memory");
	__syncthreads();

	standardize_resident<false>(L, R, s_image, image, scratch, out);
}

// A 2D image resident on a cluster of C CTAs: CTA r stages chunks
// [r chunks / C, (r + 1) chunks / C). Each pass, every CTA adds its share's
// moments, writes them into every CTA's slot r, and after a cluster barrier
// sums the C slots in rank order, so all CTAs hold the same statistics.
template <int C>
__global__ void __cluster_dims__(C, 1, 1) __launch_bounds__(resident_threads) standardize_cluster_kernel(
	const standardize_launch L, const resident_shape R)
{
	namespace cg = cooperative_groups;
	extern __shared__ float4 s_share[];
	__shared__ double scratch[3 * (resident_threads / 32)];
	__shared__ double slots[2][C][3]; // per pass, per rank: count, sum, squares
	cg::cluster_group cluster = cg::this_cluster();
	const int rank = static_cast<int>(cluster.block_rank());
	const int64_t image = blockIdx.x / C;
	const int first = static_cast<int>(static_cast<int64_t>(rank) * R.chunks / C);
	const int end = static_cast<int>(static_cast<int64_t>(rank + 1) * R.chunks / C);
	const float4 *in = reinterpret_cast<const float4 *>(L.value + image * L.size);
	float4 *out = reinterpret_cast<float4 *>(L.result + image * L.size);
	for (int j = first + threadIdx.x; j < end; j += resident_threads)
	{
		const unsigned dst = static_cast<unsigned>(__cvta_generic_to_shared(s_share + (j - first)));
		asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(in + j) : "memory");
	}
	asm volatile("cp.async.wait_all;" ::: "memory");
	__syncthreads();
	// Every CTA of the cluster runs before any writes into another's slots.
	cluster.sync();

	auto combine = [&](const moments &share, int pass) { return cluster_moments<C>(cluster, slots[pass], rank, share); };
	double mean = 0.0, scale = 1.0;
	finalize(combine(block_sum(resident_moments<false>(s_share, R, first, end, 0.0, 1.0, 0.0, 0.0), scratch), 0), mean,
		scale);
	if (L.lower != -INFINITY || L.upper != INFINITY)
		finalize(combine(block_sum(resident_moments<true>(s_share, R, first, end, mean, scale, L.lower, L.upper),
							 scratch),
					 1),
			mean, scale);
	if (L.statistics && rank == 0 && threadIdx.x == 0)
	{
		L.statistics[2 * image] = mean;
		L.statistics[2 * image + 1] = scale;
	}

	const float mean_f = static_cast<float>(mean), scale_f = static_cast<float>(scale);
	const float lower_f = static_cast<float>(L.lower), upper_f = static_cast<float>(L.upper);
	const uint64_t key = L.keys[image / L.images_per_key];
	const uint64_t counter0 = static_cast<uint64_t>(image % L.images_per_key) * static_cast<uint64_t>(L.size);
	for (int j = first + threadIdx.x; j < end; j += resident_threads)
	{
		const float4 q = s_share[j - first];
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
		__stcs(out + j, make_float4(e[0], e[1], e[2], e[3]));
	}
}

template <int C>
void launch_cluster(const standardize_launch &L, const resident_shape &R, cudaStream_t stream)
{
	const size_t share = sizeof(float4) * static_cast<size_t>((R.chunks + C - 1) / C);
	check_cuda(cudaFuncSetAttribute(standardize_cluster_kernel<C>, cudaFuncAttributeMaxDynamicSharedMemorySize,
				   static_cast<int>(resident_max_bytes)),
		"standardization attributes");
	standardize_cluster_kernel<C><<<static_cast<unsigned>(C * L.batch), resident_threads, share, stream>>>(L, R);
}

} // anonymous namespace
} // namespace rexlib_b200

using namespace rexlib_b200;

bool rexlib_b200::standardize_plan(const rexlib_b200_standardization *s, standardize_launch &L)
{
	require(s != nullptr, "null standardization descriptor");
	require(s->rank == 2 || s->rank == 3, "images must have 2 or 3 axes");
	require(s->batch >= 0, "negative batch");
	// standardize_background_operation.cpp:17-39.
	require(s->radius >= 0.0, "standardize_background: the radius must be 0 or more");
	require(s->lower_bound < 0.0 && s->upper_bound > 0.0,
		"standardize_background: the bounds must lie on either side of 0");
	require(s->images_per_key >= 1, "images_per_key must be 1 or more");
	L = standardize_launch{};
	L.size = 1;
	for (int a = 0; a < s->rank; ++a)
	{
		require(s->extents[a] >= 1 && s->extents[a] <= (1 << 20), "image extents must lie in [1, 2^20]");
		L.dims[a] = static_cast<int>(s->extents[a]);
		L.size *= s->extents[a];
	}
	if (s->batch == 0 || L.size == 0)
		return false;
	require(s->value && s->keys, "null operand");
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
	return true;
}

resident_shape rexlib_b200::resident_shape_of(const standardize_launch &L, int pitch)
{
	const int width = L.dims[L.rank - 1];
	resident_shape R{};
	R.chunks = static_cast<int>(L.size / 4);
	R.w4 = width / 4;
	R.step_rows = resident_threads / R.w4;
	R.step_cols = resident_threads % R.w4;
	R.cx = width / 2;
	R.cy = L.dims[0] / 2;
	R.radius_squared = static_cast<int>(std::min<int64_t>(L.radius_squared_floor, INT32_MAX));
	R.pitch = pitch;
	return R;
}

extern "C" int32_t rexlib_b200_standardize_background(const rexlib_b200_standardization *s, void *stream)
{
	return guarded([&] {
		standardize_launch L;
		if (!standardize_plan(s, L))
			return;
		require(L.result != nullptr, "null operand");
		const int width = L.dims[L.rank - 1];
		const size_t bytes = static_cast<size_t>(L.size) * sizeof(float);
		const bool stageable = L.rank == 2 && width % 4 == 0 && reinterpret_cast<uintptr_t>(L.value) % 16 == 0 &&
			reinterpret_cast<uintptr_t>(L.result) % 16 == 0;
		const bool resident = stageable && bytes <= resident_max_bytes;
		// The cluster size that keeps each share within the resident budget.
		const int cluster = !stageable || resident ? 0
			: bytes <= 2 * resident_max_bytes   ? 2
			: bytes <= 4 * resident_max_bytes   ? 4
			: bytes <= 8 * resident_max_bytes   ? 8
												: 0;
		if (resident || (cluster > 0 && s->batch <= 0x7fffffffLL / cluster))
		{
			const resident_shape R = resident_shape_of(L, width / 4);
			if (cluster == 2)
				launch_cluster<2>(L, R, as_stream(stream));
			else if (cluster == 4)
				launch_cluster<4>(L, R, as_stream(stream));
			else if (cluster == 8)
				launch_cluster<8>(L, R, as_stream(stream));
			else
			{
				check_cuda(cudaFuncSetAttribute(standardize_resident_kernel,
							   cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(resident_max_bytes)),
					"standardization attributes");
				standardize_resident_kernel<<<static_cast<unsigned>(s->batch), resident_threads, bytes,
					as_stream(stream)>>>(L, R);
			}
		}
		else
		{
			standardize_kernel<<<static_cast<unsigned>(s->batch), standardize_threads, 0, as_stream(stream)>>>(L);
		}
		check_cuda(cudaGetLastError(), "standardization launch");
	});
}
