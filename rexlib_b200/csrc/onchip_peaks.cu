// The on-chip rates the tiled insertion's accumulation runs into, measured
// on the device it runs on (the insertion's roofline beside HBM):
// - vector FP32 reductions into L2 (red.global.add.v4.f32), one 16-byte slot
//   a lane, slots pseudo-random over an L2-resident region the size of the
//   insertion's numerator scratch: the rate of the numerator's tap pairs;
// - FP32 shared-memory atomics at pseudo-random words of a 48 KB tile (bank
//   conflicts included): the rate of the denominator's taps, in lane
//   operations.
// Each launch runs `per_thread` operations a thread over `blocks` x
// `threads`; the caller times it. No counterpart in the reference.
#include "common.cuh"

namespace rexlib_b200
{
namespace
{

__global__ void l2_reduction_kernel(float4 *__restrict__ region, uint32_t slots, int per_thread, uint32_t seed)
{
	uint32_t x = (blockIdx.x * blockDim.x + threadIdx.x) * 2654435761u ^ seed;
	for (int i = 0; i < per_thread; ++i)
	{
		x = x * 1664525u + 1013904223u;
		float4 *p = region + (x % slots);
		asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(p), "f"(1.0f), "f"(1.0f), "f"(1.0f),
					 "f"(1.0f)
					 : "memory");
	}
}

constexpr int shared_words = 12288; // 48 KB

__global__ void shared_atomic_kernel(float *__restrict__ sink, int per_thread, uint32_t seed)
{
	__shared__ float tile[shared_words];
	for (int i = threadIdx.x; i < shared_words; i += blockDim.x)
		tile[i] = 0.0f;
	__syncthreads();
	uint32_t x = (blockIdx.x * blockDim.x + threadIdx.x) * 2654435761u ^ seed;
	for (int i = 0; i < per_thread; ++i)
	{
		x = x * 1664525u + 1013904223u;
		atomicAdd(tile + (x >> 8) % shared_words, 1.0f);
	}
	__syncthreads();
	if (threadIdx.x == 0)
		atomicAdd(sink, tile[seed % shared_words]);
}

} // anonymous namespace
} // namespace rexlib_b200

using namespace rexlib_b200;

extern "C" int32_t rexlib_b200_l2_reduction_run(void *region, int64_t bytes, int32_t blocks, int32_t threads,
	int32_t per_thread, uint32_t seed, void *stream)
{
	return guarded([&] {
		require(region != nullptr && reinterpret_cast<uintptr_t>(region) % 16 == 0, "the region must be 16-byte aligned");
		require(bytes >= 16 && bytes / 16 <= 0xFFFFFFFFll, "region of 16 bytes to 64 GiB");
		require(blocks > 0 && threads > 0 && threads <= 1024 && per_thread > 0, "positive launch sizes");
		l2_reduction_kernel<<<blocks, threads, 0, as_stream(stream)>>>(static_cast<float4 *>(region),
			static_cast<uint32_t>(bytes / 16), per_thread, seed);
		check_cuda(cudaGetLastError(), "L2 reduction launch");
	});
}

extern "C" int32_t rexlib_b200_shared_atomic_run(float *sink, int32_t blocks, int32_t threads, int32_t per_thread,
	uint32_t seed, void *stream)
{
	return guarded([&] {
		require(sink != nullptr, "null sink");
		require(blocks > 0 && threads > 0 && threads <= 1024 && per_thread > 0, "positive launch sizes");
		shared_atomic_kernel<<<blocks, threads, 0, as_stream(stream)>>>(sink, per_thread, seed);
		check_cuda(cudaGetLastError(), "shared atomic launch");
	});
}
