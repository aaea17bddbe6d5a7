// 3x3x3 convolution of channels-last BF16 volumes on the tcgen05 tensor
// cores: an implicit GEMM whose rows (M) are 128 output voxels and whose
// columns (N) are the output channels, accumulated in FP32 in tensor memory
// over K = 27 taps x input channels.
//
// Operands reach shared memory by TMA. A tap's A tile is one 4D box of the
// input volume (channels, x, y, z) shifted by the tap, with out-of-volume
// voxels zero-filled by the TMA unit itself (the padding of 1); its B tile
// is one box of the weights (channels, tap, output channel). Both are K-major
// and swizzled to the width of their channel chunk (16, 32 or 64 channels:
// 32, 64 or 128 bytes a row), which is the canonical layout the MMA reads.
// The input may be two volumes whose channels are concatenated (a U-Net
// decoder's upsampled and skip tensors), read in turn without copying.
//
// Warp roles in a persistent CTA (one per SM): warp 0 issues the TMA loads
// into a ring of stages, warp 1 owns the tensor memory and issues the MMAs
// (one thread), warps 2-5 drain each finished tile from tensor memory (one
// lane of TMEM per thread), add the bias, apply ReLU or the ReLU mask of a
// backward pass, convert to BF16 and store. Two accumulators in TMEM let the
// MMAs of the next tile run while the last one drains. Every wait on an
// mbarrier is bounded in time; a wait that runs out records an error word
// the host reads, instead of hanging. After a failure every role stops
// issuing; the producer waits (bounded) for the copies it has in flight and
// the MMA thread for its tensor-core operations, so that no copy or MMA
// outlives the CTA's shared and tensor memory, which is then freed.
#include "common.cuh"
#include "tcgen05.cuh"

#include <cuda.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>

namespace rexlib_b200
{
namespace
{

using namespace sm100;

constexpr int conv_threads = 192;
constexpr int conv_max_stages = 8;
constexpr size_t conv_smem_budget = 200 * 1024;

struct alignas(64) conv_source
{
	CUtensorMap volume;  // (channels, x, y, z), box (chunk, wb, hb, db)
	CUtensorMap weights; // (input channels of all sources, 27, output channels), box (chunk, 1, output channels)
	int chunk;           // channels a stage takes (16, 32 or 64)
	int chunks;          // channel chunks of this source
	int weight_channel;  // this source's first input channel in the weights
	int pad;
};

struct alignas(64) conv_params
{
	conv_source source[2];
	int sources;
	int depth, height, width;
	int wb, hb, db, rows; // tile box and its voxels
	int tiles_x, tiles_y, tiles;
	int cout;
	int k_iterations; // stages a tile takes: 27 x chunks of every source
	int stage_stride; // bytes of one stage (A then B), 1024-aligned
	int b_offset;     // bytes from a stage's start to its B tile
	int stages;
	uint32_t tmem_columns;
	int epilogue;           // 0: plain, 1: ReLU, 2: multiply by (mask > 0)
	const float *bias;      // FP32 per output channel, or null
	__nv_bfloat16 *out0;    // output channels [0, split)
	__nv_bfloat16 *out1;    // output channels [split, cout)
	const __nv_bfloat16 *mask0;
	const __nv_bfloat16 *mask1;
	int split;
	int out0_stride, out1_stride; // elements between voxels
	int mask0_stride, mask1_stride;
	int *error;       // set when a bounded wait runs out
	uint64_t wait_ns; // bound on each pipeline wait
};

__device__ __forceinline__ void tile_origin(const conv_params &p, int tile, int &x0, int &y0, int &z0)
{
	x0 = (tile % p.tiles_x) * p.wb;
	y0 = ((tile / p.tiles_x) % p.tiles_y) * p.hb;
	z0 = (tile / (p.tiles_x * p.tiles_y)) * p.db;
}

__device__ __forceinline__ void report(const conv_params &p, int code)
{
	if (p.error != nullptr)
		atomicCAS(p.error, 0, code);
}

__global__ void __launch_bounds__(conv_threads, 1) conv3d_kernel(const __grid_constant__ conv_params p)
{
	extern __shared__ __align__(1024) unsigned char smem_raw[];
	unsigned char *smem = reinterpret_cast<unsigned char *>(
		(reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
	__shared__ uint64_t full[conv_max_stages], empty[conv_max_stages], tmem_full[2], tmem_empty[2], drained;
	__shared__ uint32_t tmem_base;
	__shared__ int failed;

	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	volatile int *stop = &failed;
	if (threadIdx.x == 0)
	{
		for (int s = 0; s < p.stages; ++s)
		{
			mbarrier_init(&full[s], 1);
			mbarrier_init(&empty[s], 1);
		}
		for (int b = 0; b < 2; ++b)
		{
			mbarrier_init(&tmem_full[b], 1);
			mbarrier_init(&tmem_empty[b], 4);
		}
		mbarrier_init(&drained, 1);
		failed = 0;
		fence_barrier_init();
	}
	if (warp == 0 && lane == 0)
		for (int i = 0; i < p.sources; ++i)
		{
			prefetch_tensor_map(&p.source[i].volume);
			prefetch_tensor_map(&p.source[i].weights);
		}
	if (warp == 1)
		tmem_allocate(&tmem_base, p.tmem_columns);
	tcgen05_fence_before();
	__syncthreads();
	tcgen05_fence_after();
	const uint32_t tmem = tmem_base;

	if (warp == 0)
	{
		// TMA producer.
		if (lane == 0)
		{
			int s = 0;
			uint32_t phase = 0;
			uint32_t issued = 0;       // stages that have taken a load
			uint32_t issued_phase = 0; // bit s: the phase parity of stage s's last load
			for (int tile = blockIdx.x; tile < p.tiles && !*stop; tile += gridDim.x)
			{
				int x0, y0, z0;
				tile_origin(p, tile, x0, y0, z0);
				for (int tap = 0; tap < 27 && !*stop; ++tap)
				{
					const int dz = tap / 9 - 1, dy = (tap / 3) % 3 - 1, dx = tap % 3 - 1;
					for (int src = 0; src < p.sources; ++src)
					{
						const conv_source &S = p.source[src];
						for (int c = 0; c < S.chunks; ++c)
						{
							if (*stop || !mbarrier_wait(&empty[s], phase ^ 1, p.wait_ns))
							{
								if (!*stop)
									report(p, 1);
								*stop = 1;
								break;
							}
							unsigned char *stage = smem + s * p.stage_stride;
							const uint32_t bytes = static_cast<uint32_t>((p.rows + p.cout) * S.chunk * 2);
							mbarrier_expect_tx(&full[s], bytes);
							tma_load_4d(stage, &S.volume, &full[s], c * S.chunk, x0 + dx, y0 + dy, z0 + dz);
							tma_load_3d(stage + p.b_offset, &S.weights, &full[s], S.weight_channel + c * S.chunk, tap, 0);
							issued |= 1u << s;
							issued_phase = (issued_phase & ~(1u << s)) | (phase << s);
							if (++s == p.stages)
							{
								s = 0;
								phase ^= 1;
							}
						}
						if (*stop)
							break;
					}
				}
			}
			// After a failure, the loads still landing: each stage's last
			// one completes its phase (at once where the MMAs consumed it).
			if (*stop)
				for (int t = 0; t < p.stages; ++t)
					if ((issued >> t) & 1u)
						mbarrier_wait(&full[t], (issued_phase >> t) & 1u);
		}
	}
	else if (warp == 1)
	{
		// MMA issuer.
		if (lane == 0)
		{
			const uint32_t idesc = bf16_idesc(128, static_cast<uint32_t>(p.cout));
			int s = 0;
			uint32_t phase = 0;
			int local = 0;
			for (int tile = blockIdx.x; tile < p.tiles && !*stop; tile += gridDim.x, ++local)
			{
				const int buffer = local & 1;
				if (!mbarrier_wait(&tmem_empty[buffer], ((local >> 1) & 1) ^ 1, p.wait_ns))
				{
					if (!*stop)
						report(p, 2);
					*stop = 1;
					break;
				}
				tcgen05_fence_after();
				const uint32_t d = tmem + static_cast<uint32_t>(buffer * p.cout);
				int k = 0;
				for (int tap = 0; tap < 27 && !*stop; ++tap)
					for (int src = 0; src < p.sources && !*stop; ++src)
					{
						const conv_source &S = p.source[src];
						const uint32_t row_bytes = static_cast<uint32_t>(S.chunk * 2);
						for (int c = 0; c < S.chunks; ++c, ++k)
						{
							if (*stop || !mbarrier_wait(&full[s], phase, p.wait_ns))
							{
								if (!*stop)
									report(p, 3);
								*stop = 1;
								break;
							}
							tcgen05_fence_after();
							const uint32_t a_addr = smem_address(smem + s * p.stage_stride);
							const uint32_t b_addr = a_addr + static_cast<uint32_t>(p.b_offset);
							for (int kk = 0; kk < S.chunk / 16; ++kk)
								mma_f16(d, kmajor_descriptor(a_addr + kk * 32, row_bytes),
									kmajor_descriptor(b_addr + kk * 32, row_bytes), idesc, (k > 0 || kk > 0) ? 1u : 0u);
							mma_commit(&empty[s]); // the stage is free once these MMAs have read it
							if (++s == p.stages)
							{
								s = 0;
								phase ^= 1;
							}
						}
					}
				mma_commit(&tmem_full[buffer]); // the accumulator is complete
			}
			// Every MMA issued has completed before the memory they use is
			// freed (immediate after a normal run, whose epilogue waited).
			mma_commit(&drained);
			mbarrier_wait(&drained, 0);
		}
	}
	else
	{
		// Epilogue: warps 2-5; warp w drains TMEM lanes 32 (w % 4) onward.
		const int quarter = warp & 3;
		const int row = quarter * 32 + lane;
		int local = 0;
		for (int tile = blockIdx.x; tile < p.tiles; tile += gridDim.x, ++local)
		{
			const int buffer = local & 1;
			if (*stop || !mbarrier_wait(&tmem_full[buffer], (local >> 1) & 1, p.wait_ns))
			{
				if (!*stop)
					report(p, 4);
				*stop = 1;
				break;
			}
			tcgen05_fence_after();
			int x0, y0, z0;
			tile_origin(p, tile, x0, y0, z0);
			const bool valid = row < p.rows;
			const int x = x0 + row % p.wb, y = y0 + (row / p.wb) % p.hb, z = z0 + row / (p.wb * p.hb);
			const int64_t voxel = (static_cast<int64_t>(z) * p.height + y) * p.width + x;
			for (int g = 0; g < p.cout / 16; ++g)
			{
				float v[16];
				tmem_load16(tmem + (static_cast<uint32_t>(quarter * 32) << 16) + static_cast<uint32_t>(buffer * p.cout + g * 16),
					v);
				if (!valid)
					continue;
				const int c0 = g * 16;
				const bool first = c0 < p.split;
				__nv_bfloat16 *out = first ? p.out0 + voxel * p.out0_stride + c0
										   : p.out1 + voxel * p.out1_stride + (c0 - p.split);
				if (p.bias != nullptr)
#pragma unroll
					for (int i = 0; i < 16; ++i)
						v[i] += __ldg(p.bias + c0 + i);
				if (p.epilogue == 1)
				{
#pragma unroll
					for (int i = 0; i < 16; ++i)
						v[i] = fmaxf(v[i], 0.0f);
				}
				else if (p.epilogue == 2)
				{
					const __nv_bfloat16 *mask = first ? p.mask0 + voxel * p.mask0_stride + c0
													  : p.mask1 + voxel * p.mask1_stride + (c0 - p.split);
					if (mask != nullptr && (first ? p.mask0 : p.mask1) != nullptr)
					{
						const uint4 m0 = *reinterpret_cast<const uint4 *>(mask);
						const uint4 m1 = *reinterpret_cast<const uint4 *>(mask + 8);
						const __nv_bfloat16 *mb0 = reinterpret_cast<const __nv_bfloat16 *>(&m0);
						const __nv_bfloat16 *mb1 = reinterpret_cast<const __nv_bfloat16 *>(&m1);
#pragma unroll
						for (int i = 0; i < 8; ++i)
						{
							if (!(__bfloat162float(mb0[i]) > 0.0f))
								v[i] = 0.0f;
							if (!(__bfloat162float(mb1[i]) > 0.0f))
								v[8 + i] = 0.0f;
						}
					}
				}
				uint4 packed[2];
				__nv_bfloat162 *h = reinterpret_cast<__nv_bfloat162 *>(packed);
#pragma unroll
				for (int i = 0; i < 8; ++i)
					h[i] = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);
				reinterpret_cast<uint4 *>(out)[0] = packed[0];
				reinterpret_cast<uint4 *>(out)[1] = packed[1];
			}
			tcgen05_fence_before();
			__syncwarp();
			if (lane == 0)
				mbarrier_arrive(&tmem_empty[buffer]);
		}
	}
	tcgen05_fence_before();
	__syncthreads();
	if (warp == 1)
	{
		tcgen05_fence_after();
		tmem_free(tmem, p.tmem_columns);
	}
}

// ---------------------------------------------------------------------------
// Host side

using encode_tiled_t = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
	const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
	CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

encode_tiled_t encode_tiled()
{
	static encode_tiled_t fn = nullptr;
	static std::once_flag once;
	std::call_once(once, [] {
		void *p = nullptr;
		cudaDriverEntryPointQueryResult q{};
		if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) ==
				cudaSuccess &&
			q == cudaDriverEntryPointSuccess)
			fn = reinterpret_cast<encode_tiled_t>(p);
	});
	require(fn != nullptr, "the driver has no cuTensorMapEncodeTiled");
	return fn;
}

CUtensorMapSwizzle swizzle_of(int row_bytes)
{
	return row_bytes == 128 ? CU_TENSOR_MAP_SWIZZLE_128B
		: row_bytes == 64   ? CU_TENSOR_MAP_SWIZZLE_64B
							: CU_TENSOR_MAP_SWIZZLE_32B;
}

void encode(CUtensorMap *map, const void *base, int rank, const cuuint64_t *dims, const cuuint64_t *strides_bytes,
	const cuuint32_t *box, int row_bytes)
{
	cuuint32_t element_strides[5] = {1, 1, 1, 1, 1};
	const CUresult r = encode_tiled()(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, static_cast<cuuint32_t>(rank),
		const_cast<void *>(base), dims, strides_bytes, box, element_strides, CU_TENSOR_MAP_INTERLEAVE_NONE,
		swizzle_of(row_bytes), CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
	if (r != CUDA_SUCCESS)
		fail(REXLIB_B200_INVALID_ARGUMENT, "a tensor map of the convolution was refused (code " + std::to_string(r) + ")");
}

int sm_count()
{
	int device = 0, sms = 0;
	check_cuda(cudaGetDevice(&device), "device query");
	check_cuda(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "device query");
	return sms;
}

} // anonymous namespace
} // namespace rexlib_b200

using namespace rexlib_b200;

extern "C" int32_t rexlib_b200_conv3d(const rexlib_b200_conv3d_args *a, void *stream)
{
	return guarded([&] {
		require(a != nullptr, "null convolution arguments");
		require(a->sources == 1 || a->sources == 2, "a convolution reads one or two input volumes");
		require(a->depth >= 1 && a->height >= 1 && a->width >= 1, "volume extents must be positive");
		const int D = a->depth, H = a->height, W = a->width;
		auto pow2 = [](int v) { return v > 0 && (v & (v - 1)) == 0; };
		if (!pow2(D) || !pow2(H) || !pow2(W))
			fail(REXLIB_B200_UNSUPPORTED, "the convolution takes volume extents that are powers of two");
		if (a->output_channels < 16 || a->output_channels > 128 || a->output_channels % 16 != 0)
			fail(REXLIB_B200_UNSUPPORTED, "the convolution takes 16 to 128 output channels, a multiple of 16");
		conv_params p{};
		p.sources = a->sources;
		p.depth = D;
		p.height = H;
		p.width = W;
		p.wb = std::min(W, 128);
		p.hb = std::min(H, 128 / p.wb);
		p.db = std::min(D, 128 / (p.wb * p.hb));
		p.rows = p.wb * p.hb * p.db;
		p.tiles_x = W / p.wb;
		p.tiles_y = H / p.hb;
		p.tiles = p.tiles_x * p.tiles_y * (D / p.db);
		p.cout = a->output_channels;
		int total_in = 0;
		for (int i = 0; i < a->sources; ++i)
			total_in += a->input_channels[i];
		int max_chunk = 16;
		int k_iterations = 0;
		for (int i = 0; i < a->sources; ++i)
		{
			const int c = a->input_channels[i];
			if (!(c == 16 || c == 32 || c % 64 == 0) || c > 256)
				fail(REXLIB_B200_UNSUPPORTED, "the convolution takes 16, 32 or a multiple of 64 input channels a source");
			require(a->inputs[i] != nullptr, "null input volume");
			require(a->input_strides[i] >= c && a->input_strides[i] % 8 == 0, "input rows must hold their channels, "
				"a multiple of 8");
			require(reinterpret_cast<uintptr_t>(a->inputs[i]) % 16 == 0, "input volumes must be 16-byte aligned");
			conv_source &S = p.source[i];
			S.chunk = std::min(c, 64);
			S.chunks = c / S.chunk;
			S.weight_channel = i == 0 ? 0 : a->input_channels[0];
			max_chunk = std::max(max_chunk, S.chunk);
			k_iterations += 27 * S.chunks;
			const cuuint64_t vdims[4] = {static_cast<cuuint64_t>(c), static_cast<cuuint64_t>(W),
				static_cast<cuuint64_t>(H), static_cast<cuuint64_t>(D)};
			const cuuint64_t row = static_cast<cuuint64_t>(a->input_strides[i]) * 2;
			const cuuint64_t vstrides[3] = {row, row * W, row * W * H};
			const cuuint32_t vbox[4] = {static_cast<cuuint32_t>(S.chunk), static_cast<cuuint32_t>(p.wb),
				static_cast<cuuint32_t>(p.hb), static_cast<cuuint32_t>(p.db)};
			encode(&S.volume, a->inputs[i], 4, vdims, vstrides, vbox, S.chunk * 2);
			const cuuint64_t wdims[3] = {static_cast<cuuint64_t>(total_in), 27, static_cast<cuuint64_t>(p.cout)};
			const cuuint64_t wstrides[2] = {static_cast<cuuint64_t>(total_in) * 2,
				static_cast<cuuint64_t>(total_in) * 2 * 27};
			const cuuint32_t wbox[3] = {static_cast<cuuint32_t>(S.chunk), 1, static_cast<cuuint32_t>(p.cout)};
			encode(&S.weights, a->weights, 3, wdims, wstrides, wbox, S.chunk * 2);
		}
		require(reinterpret_cast<uintptr_t>(a->weights) % 16 == 0, "weights must be 16-byte aligned");
		p.k_iterations = k_iterations;
		const int a_bytes = 128 * max_chunk * 2;
		p.b_offset = a_bytes;
		p.stage_stride = (a_bytes + p.cout * max_chunk * 2 + 1023) / 1024 * 1024;
		p.stages = static_cast<int>(std::min<size_t>(conv_max_stages, conv_smem_budget / p.stage_stride));
		p.tmem_columns = 32;
		while (p.tmem_columns < static_cast<uint32_t>(2 * p.cout))
			p.tmem_columns *= 2;
		p.epilogue = a->epilogue;
		p.bias = a->bias;
		require(a->outputs[0] != nullptr, "null output volume");
		p.split = a->output_split > 0 ? a->output_split : p.cout;
		require(p.split % 16 == 0 && p.split <= p.cout, "the output split falls on a multiple of 16 channels");
		require(p.split == p.cout || a->outputs[1] != nullptr, "null second output volume");
		p.out0 = static_cast<__nv_bfloat16 *>(a->outputs[0]);
		p.out1 = static_cast<__nv_bfloat16 *>(a->outputs[1]);
		p.out0_stride = a->output_strides[0];
		p.out1_stride = a->output_strides[1];
		p.mask0 = static_cast<const __nv_bfloat16 *>(a->masks[0]);
		p.mask1 = static_cast<const __nv_bfloat16 *>(a->masks[1]);
		p.mask0_stride = a->mask_strides[0];
		p.mask1_stride = a->mask_strides[1];
		for (int i = 0; i < 2; ++i)
		{
			require(reinterpret_cast<uintptr_t>(a->outputs[i]) % 16 == 0 && a->output_strides[i] % 8 == 0 &&
					reinterpret_cast<uintptr_t>(a->masks[i]) % 16 == 0 && a->mask_strides[i] % 8 == 0,
				"outputs and masks must be 16-byte aligned, their rows a multiple of 8 channels");
		}
		require(p.epilogue >= 0 && p.epilogue <= 2, "unknown epilogue");
		p.error = a->error;
		p.wait_ns = a->wait_limit_ns > 0 ? static_cast<uint64_t>(a->wait_limit_ns) : default_wait_ns;
		const size_t smem = static_cast<size_t>(p.stages) * p.stage_stride + 1024;
		check_cuda(cudaFuncSetAttribute(conv3d_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)),
			"convolution attributes");
		const int grid = std::min(p.tiles, sm_count());
		conv3d_kernel<<<grid, conv_threads, smem, as_stream(stream)>>>(p);
		check_cuda(cudaGetLastError(), "convolution launch");
	});
}
