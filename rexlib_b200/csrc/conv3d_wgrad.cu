// Weight and bias gradients of the 3x3x3 convolution on the tcgen05 tensor
// cores: for the output gradient g and the convolution's input x,
//   dw[o][t][i] = sum_v g[v][o] x[v + offset(t)][i],   db[o] = sum_v g[v][o].
//
// As a GEMM, D[(t, i), o] = sum over K = voxels of A[(t, i), v] B[v, o]: the
// rows (M) are taps x input channels, the columns (N) output channels, and K
// runs over the voxels, so both operands are MN-major (their M or N index is
// the contiguous one in memory). The accumulators stay in tensor memory for
// all the voxels a CTA takes, and are added to dw once at the end.
//
// The sum over voxels is split by the input line's x position j rather than
// by the output voxel: for tap (dx, dy, dz),
//   sum_v x[v + t] g[v] = sum over rows (y, z), and j, of x[z + dz - 1][y + dy - 1][j] g[z][y][j - dx + 1],
// so a stage is one x-segment j = x0 .. x0 + xs - 1 (up to 128, K) at (y, z):
// - the input lines of all nine (dy, dz) taps as ONE 5D TMA box (8 channels,
//   xs, 3, 3, K8 pieces of 8 channels) of the volume viewed as (8 channels,
//   x, y, z, pieces), zero-filled outside the volume. It lands as piece p,
//   line (dz, dy), voxel r at 16 ((9 p + 3 dz + dy) xs + r) bytes: the 9 K8
//   groups of 8 channels (p, dz, dy) sit at one stride, so one MMA of
//   M = 128 takes 16 consecutive groups;
// - g's row at x0 + 1 - dx .. for dx = 0, 1, 2: three 5D boxes (8 channels,
//   xs, 1, 1, CO / 8), zero-filled outside the volume, one after another, so
//   that their 3 CO / 8 groups of 8 channels (dx, piece) also sit at one
//   stride: one MMA of N = 3 CO takes the three x taps at once.
// The M tiles cover the groups 16 at a time; the last one starts at group
// 9 K8 - 16 so that no MMA reads past the lines (its rows that repeat the
// previous tile's groups are dropped by the epilogue). A K step of 16
// positions issues one MMA of 128 x 3 CO x 16 per tile, into columns
// (dx, output channel) of the tile's accumulator.
//
// With 64 output channels (CO = 64) the three copies of g would leave room
// for two stages only, which measured slower; there the sum is split by the
// output voxel instead: the lines carry an x halo (xs + 2 voxels, from
// x0 - 1), one copy of g is loaded, and the tap dx is the same line groups
// read from voxel dx on (a start address 16 dx bytes further; the no-swizzle
// layout allows any 16-byte start), 3 x tiles MMAs of N = CO a K step.
//
// A CTA takes one chunk of K8 x 8 input channels, one chunk of CO output
// channels and a range of segments. Warp roles: warp 0 issues the TMA loads,
// warp 1 owns the tensor memory and issues the MMAs (one thread), warps 2-5
// first sum g over the CTA's segments for the bias gradient (CTAs of the
// first input chunk), then drain the accumulators into dw with FP32
// reductions. Every mbarrier wait is bounded in time; one that runs out
// records an error word, every role stops issuing, the copies and MMAs in
// flight are waited for (bounded) and the tensor memory is freed.
#include "common.cuh"
#include "tcgen05.cuh"
#include "tensor_map.cuh"

#include <cuda.h>
#include <cuda_bf16.h>

#include <algorithm>

namespace rexlib_b200
{
namespace
{

using namespace sm100;

constexpr int wgrad_tc_threads = 192;
constexpr int wgrad_max_stages = 8;
constexpr int wgrad_max_chunks = 64;
constexpr size_t wgrad_smem_budget = 200 * 1024;
// Shared memory asked for at least: one CTA an SM, so that CTAs never wait
// on one another for tensor memory.
constexpr size_t wgrad_smem_floor = 120 * 1024;

struct alignas(64) wgrad_params
{
	CUtensorMap line[2]; // per source: (8 channels, x, y, z, pieces of 8), box (8, xs (xs + 2 at CO = 64), 3, 3, K8)
	CUtensorMap grad;    // g as (8 channels, x, y, z, pieces of 8), box (8, xs, 1, 1, CO / 8)
	int height, width;
	int xs;           // voxels of a segment: min(W, 128)
	int segments;     // segments of an x-row
	int rows;         // segments of the volume
	int rows_per_cta; // segments of a CTA (the last CTA may take fewer)
	int cin;          // input channels of all sources
	int a_bytes, b_bytes, b_offset, stage_stride, stages; // b_bytes: one of the three copies of g
	uint32_t tmem_columns;
	const __nv_bfloat16 *g;
	int g_stride;
	float *dw, *db;
	int *error;
	uint64_t wait_ns;
	int chunk_source[wgrad_max_chunks];  // per input chunk: its source,
	int chunk_piece[wgrad_max_chunks];   // its first piece of 8 channels there,
	int chunk_channel[wgrad_max_chunks]; // and its first channel among all sources
};

__device__ __forceinline__ void report(const wgrad_params &p, int code)
{
	if (p.error != nullptr)
		atomicCAS(p.error, 0, code);
}

__device__ __forceinline__ void epilogue_barrier() { asm volatile("bar.sync 1, 128;" ::: "memory"); }

template <int K8, int CO>
__global__ void __launch_bounds__(wgrad_tc_threads, 1) conv3d_wgrad_kernel(const __grid_constant__ wgrad_params p)
{
	constexpr bool WIDE = CO <= 32; // the x taps in N (three copies of g)
	constexpr int GROUPS = 9 * K8;            // groups of 8 channels in a stage's lines: (piece, dz, dy)
	constexpr int TILES = (GROUPS + 15) / 16; // M tiles of 16 groups
	static_assert(GROUPS >= 16, "a tile takes 16 groups");

	extern __shared__ __align__(1024) unsigned char smem_raw[];
	unsigned char *smem = reinterpret_cast<unsigned char *>(
		(reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
	__shared__ uint64_t full[wgrad_max_stages], empty[wgrad_max_stages], tmem_full, drained;
	__shared__ uint32_t tmem_base;
	__shared__ int failed;
	__shared__ float bias_sum[CO];

	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	volatile int *stop = &failed;
	const int chunk = blockIdx.y, co_chunk = blockIdx.z;
	const int r_begin = blockIdx.x * p.rows_per_cta;
	const int r_end = min(p.rows, r_begin + p.rows_per_cta);
	if (threadIdx.x == 0)
	{
		for (int s = 0; s < p.stages; ++s)
		{
			mbarrier_init(&full[s], 1);
			mbarrier_init(&empty[s], 1);
		}
		mbarrier_init(&tmem_full, 1);
		mbarrier_init(&drained, 1);
		failed = 0;
		fence_barrier_init();
	}
	if (threadIdx.x < CO)
		bias_sum[threadIdx.x] = 0.0f;
	if (warp == 0 && lane == 0)
	{
		prefetch_tensor_map(&p.line[p.chunk_source[chunk]]);
		prefetch_tensor_map(&p.grad);
	}
	if (warp == 1)
		tmem_allocate(&tmem_base, p.tmem_columns);
	tcgen05_fence_before();
	__syncthreads();
	tcgen05_fence_after();
	const uint32_t tmem = tmem_base;
	const int H = p.height, W = p.width, xs = p.xs;

	if (warp == 0)
	{
		// TMA producer.
		if (lane == 0)
		{
			const CUtensorMap *line = &p.line[p.chunk_source[chunk]];
			const int piece = p.chunk_piece[chunk];
			const int co_piece = co_chunk * (CO / 8);
			const uint32_t bytes = static_cast<uint32_t>(p.a_bytes + (WIDE ? 3 : 1) * p.b_bytes);
			int s = 0;
			uint32_t phase = 0;
			uint32_t issued = 0;       // stages that have taken loads
			uint32_t issued_phase = 0; // bit s: the phase parity of stage s's last loads
			for (int r = r_begin; r < r_end && !*stop; ++r)
			{
				if (!mbarrier_wait(&empty[s], phase ^ 1, p.wait_ns))
				{
					if (!*stop)
						report(p, 1);
					*stop = 1;
					break;
				}
				const int x0 = (r % p.segments) * xs;
				const int y = (r / p.segments) % H, z = r / (p.segments * H);
				unsigned char *stage = smem + s * p.stage_stride;
				mbarrier_expect_tx(&full[s], bytes);
				if constexpr (WIDE)
				{
					tma_load_5d(stage, line, &full[s], 0, x0, y - 1, z - 1, piece);
					for (int dx = 0; dx < 3; ++dx)
						tma_load_5d(stage + p.b_offset + dx * p.b_bytes, &p.grad, &full[s], 0, x0 + 1 - dx, y, z, co_piece);
				}
				else
				{
					tma_load_5d(stage, line, &full[s], 0, x0 - 1, y - 1, z - 1, piece);
					tma_load_5d(stage + p.b_offset, &p.grad, &full[s], 0, x0, y, z, co_piece);
				}
				issued |= 1u << s;
				issued_phase = (issued_phase & ~(1u << s)) | (phase << s);
				if (++s == p.stages)
				{
					s = 0;
					phase ^= 1;
				}
			}
			// After a failure, the loads still landing: each stage's last
			// ones complete its phase (at once where the MMAs consumed it).
			if (*stop)
				for (int t = 0; t < p.stages; ++t)
					if ((issued >> t) & 1u)
						mbarrier_wait(&full[t], (issued_phase >> t) & 1u);
		}
	}
	else if (warp == 1)
	{
		// MMA issuer: A and B MN-major (instruction descriptor bits 15, 16).
		if (lane == 0)
		{
			constexpr uint32_t idesc = bf16_idesc(128, WIDE ? 3 * CO : CO) | (1u << 15) | (1u << 16);
			const uint32_t smem_base = smem_address(smem);
			const uint32_t group_stride = static_cast<uint32_t>(WIDE ? xs : xs + 2) * 16; // between groups of the lines
			const uint32_t piece_stride = static_cast<uint32_t>(xs) * 16; // between groups of g's copies
			const int ksteps = xs / 16;
			uint32_t tile_start[TILES]; // 16-byte units from a stage's start to tile t's first group
#pragma unroll
			for (int t = 0; t < TILES; ++t)
				tile_start[t] = static_cast<uint32_t>(min(16 * t, GROUPS - 16)) * group_stride >> 4;
			int s = 0;
			uint32_t phase = 0;
			bool first = true;
			for (int r = r_begin; r < r_end && !*stop; ++r)
			{
				if (!mbarrier_wait(&full[s], phase, p.wait_ns))
				{
					if (!*stop)
						report(p, 3);
					*stop = 1;
					break;
				}
				tcgen05_fence_after();
				// Descriptors of the stage's operands: core matrices of 8
				// voxels (K) x 8 channels, 128 contiguous bytes; 128 bytes
				// between core matrices along K, the group (or piece) stride
				// along M (or N). The others differ in the start address only
				// (addresses below 256 KB: the 14-bit field takes the sum).
				const uint32_t a_addr = smem_base + static_cast<uint32_t>(s * p.stage_stride);
				const uint64_t a0 = interleaved_descriptor(a_addr, 128, group_stride);
				const uint64_t b0 = interleaved_descriptor(a_addr + static_cast<uint32_t>(p.b_offset), 128, piece_stride);
				for (int ks = 0; ks < ksteps; ++ks)
				{
					const uint32_t k = static_cast<uint32_t>(ks * 16); // 16 voxels of 16 bytes
					const uint32_t accumulate = first && ks == 0 ? 0u : 1u;
					if constexpr (WIDE)
					{
#pragma unroll
						for (int t = 0; t < TILES; ++t)
							mma_f16(tmem + static_cast<uint32_t>(t * 3 * CO), a0 + (tile_start[t] + k), b0 + k, idesc,
								accumulate);
					}
					else
					{
#pragma unroll
						for (int t = 0; t < TILES; ++t)
#pragma unroll
							for (int dx = 0; dx < 3; ++dx)
								mma_f16(tmem + static_cast<uint32_t>((t * 3 + dx) * CO), a0 + (tile_start[t] + k + dx), b0 + k,
									idesc, accumulate);
					}
				}
				first = false;
				mma_commit(&empty[s]); // the stage is free once these MMAs have read it
				if (++s == p.stages)
				{
					s = 0;
					phase ^= 1;
				}
			}
			mma_commit(&tmem_full);
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
		const int et = threadIdx.x - 64;
		if (p.db != nullptr && chunk == 0)
		{
			// The bias gradient of the CTA's segments, from g in global memory
			// while the MMAs run: thread et sums piece et % (CO / 8) of every
			// (128 / (CO / 8))-th voxel.
			constexpr int PIECES = CO / 8;
			const int piece = et % PIECES;
			float acc[8] = {};
			for (int r = r_begin; r < r_end && !*stop; ++r)
			{
				const int x0 = (r % p.segments) * xs;
				const int y = (r / p.segments) % H, z = r / (p.segments * H);
				const int64_t v0 = (static_cast<int64_t>(z) * H + y) * W + x0;
				for (int x = et / PIECES; x < xs; x += 128 / PIECES)
				{
					const uint4 q = __ldg(
						reinterpret_cast<const uint4 *>(p.g + (v0 + x) * p.g_stride + co_chunk * CO + piece * 8));
					const __nv_bfloat162 *h = reinterpret_cast<const __nv_bfloat162 *>(&q);
#pragma unroll
					for (int i = 0; i < 4; ++i)
					{
						const float2 f = __bfloat1622float2(h[i]);
						acc[2 * i] += f.x;
						acc[2 * i + 1] += f.y;
					}
				}
			}
#pragma unroll
			for (int i = 0; i < 8; ++i)
				atomicAdd(&bias_sum[piece * 8 + i], acc[i]);
			epilogue_barrier();
			if (et < CO && !*stop)
				atomicAdd(p.db + co_chunk * CO + et, bias_sum[et]);
		}
		if (r_begin < r_end)
		{
			bool ok = !*stop && mbarrier_wait(&tmem_full, 0, p.wait_ns);
			// The TMEM loads take the whole warp: one decision for all lanes.
			ok = __all_sync(0xffffffffu, ok);
			if (!ok)
			{
				if (lane == 0 && !*stop)
					report(p, 4);
				*stop = 1;
			}
			else
			{
				tcgen05_fence_after();
				const int row = quarter * 32 + lane; // M row of every tile: group row / 8, channel row % 8
				const int64_t tap_stride = p.cin;
				const int64_t out_stride = 27 * tap_stride;
#pragma unroll
				for (int t = 0; t < TILES; ++t)
				{
					const int j = min(16 * t, GROUPS - 16) + row / 8;
					const bool keep = j >= 16 * t; // rows a previous tile already took are dropped
					const int pc = j / 9, line = j % 9;
					const int ci = p.chunk_channel[chunk] + pc * 8 + row % 8;
#pragma unroll
					for (int dx = 0; dx < 3; ++dx)
					{
						const int tap = (line / 3) * 9 + (line % 3) * 3 + dx;
						float *out = p.dw + static_cast<int64_t>(co_chunk * CO) * out_stride + tap * tap_stride + ci;
#pragma unroll
						for (int c = 0; c < CO / 16; ++c)
						{
							float v[16];
							tmem_load16(tmem + (static_cast<uint32_t>(quarter * 32) << 16) +
									static_cast<uint32_t>((t * 3 + dx) * CO + c * 16),
								v);
							if (keep)
#pragma unroll
								for (int i = 0; i < 16; ++i)
									atomicAdd(out + (c * 16 + i) * out_stride, v[i]);
						}
					}
				}
			}
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

} // anonymous namespace
} // namespace rexlib_b200

namespace rexlib_b200
{
namespace
{

uint32_t wgrad_tmem_columns(int columns)
{
	uint32_t c = 32;
	while (c < static_cast<uint32_t>(columns))
		c *= 2;
	return c;
}

void launch_wgrad(const rexlib_b200_conv3d_wgrad_args *a, cudaStream_t stream)
{
	wgrad_params p{};
	const int D = a->depth, H = a->height, W = a->width;
	p.height = H;
	p.width = W;
	p.xs = std::min(W, 128);
	p.segments = W / p.xs;
	p.rows = D * H * p.segments;
	const int cout = a->output_channels;
	// Output chunks of up to 64 channels; input chunks of 32 channels where
	// every source divides into them and the accumulators (9 tiles x CO
	// columns) fit, of 16 otherwise (6 tiles x CO).
	const int co = std::min(cout, 64);
	bool by32 = co <= 32;
	int cin = 0;
	for (int i = 0; i < a->sources; ++i)
	{
		cin += a->input_channels[i];
		by32 = by32 && a->input_channels[i] % 32 == 0;
	}
	const int ci = by32 ? 32 : 16;
	const int k8 = ci / 8;
	p.cin = cin;
	int chunks = 0;
	for (int i = 0; i < a->sources; ++i)
		for (int c0 = 0; c0 < a->input_channels[i]; c0 += ci)
		{
			require(chunks < wgrad_max_chunks, "too many input channels for the weight gradient");
			p.chunk_source[chunks] = i;
			p.chunk_piece[chunks] = c0 / 8;
			p.chunk_channel[chunks] = (i == 0 ? 0 : a->input_channels[0]) + c0;
			++chunks;
		}
	for (int i = 0; i < a->sources; ++i)
	{
		const int c = a->input_channels[i];
		const cuuint64_t row = static_cast<cuuint64_t>(a->input_strides[i]) * 2;
		const cuuint64_t dims[5] = {8, static_cast<cuuint64_t>(W), static_cast<cuuint64_t>(H),
			static_cast<cuuint64_t>(D), static_cast<cuuint64_t>(c / 8)};
		const cuuint64_t strides[4] = {row, row * W, row * W * H, 16};
		// With up to 32 output channels the lines are xs voxels from x0; with
		// 64 they carry the x halo, xs + 2 from x0 - 1.
		const cuuint32_t box[5] = {8, static_cast<cuuint32_t>(co <= 32 ? p.xs : p.xs + 2), 3, 3, static_cast<cuuint32_t>(k8)};
		encode(&p.line[i], a->inputs[i], 5, dims, strides, box, 0);
	}
	{
		const cuuint64_t row = static_cast<cuuint64_t>(a->output_grad_stride) * 2;
		const cuuint64_t dims[5] = {8, static_cast<cuuint64_t>(W), static_cast<cuuint64_t>(H),
			static_cast<cuuint64_t>(D), static_cast<cuuint64_t>(cout / 8)};
		const cuuint64_t strides[4] = {row, row * W, row * W * H, 16};
		const cuuint32_t box[5] = {8, static_cast<cuuint32_t>(p.xs), 1, 1, static_cast<cuuint32_t>(co / 8)};
		encode(&p.grad, a->output_grad, 5, dims, strides, box, 0);
	}
	const bool wide = co <= 32;
	p.a_bytes = 16 * (wide ? p.xs : p.xs + 2) * 9 * k8;
	p.b_bytes = 16 * p.xs * (co / 8);
	p.b_offset = (p.a_bytes + 1023) / 1024 * 1024;
	p.stage_stride = (p.b_offset + (wide ? 3 : 1) * p.b_bytes + 1023) / 1024 * 1024;
	p.stages = static_cast<int>(std::min<size_t>(wgrad_max_stages, wgrad_smem_budget / p.stage_stride));
	require(p.stages >= 2, "the weight gradient's stages do not fit in shared memory");
	const int tiles = (9 * k8 + 15) / 16;
	p.tmem_columns = wgrad_tmem_columns(tiles * 3 * co);
	require(p.tmem_columns <= 512, "the weight gradient's accumulators do not fit in tensor memory");
	p.g = static_cast<const __nv_bfloat16 *>(a->output_grad);
	p.g_stride = a->output_grad_stride;
	p.dw = a->weight_grad;
	p.db = a->bias_grad;
	p.error = a->error;
	p.wait_ns = a->wait_limit_ns > 0 ? static_cast<uint64_t>(a->wait_limit_ns) : default_wait_ns;
	// About one wave: the (input chunk, output chunk) pairs share the SMs,
	// each pair's segments split evenly over its CTAs.
	const int co_chunks = cout / co;
	const int pairs = chunks * co_chunks;
	const int per_pair = std::max(1, std::min(p.rows, sm_count() / pairs));
	p.rows_per_cta = (p.rows + per_pair - 1) / per_pair;
	const int ctas = (p.rows + p.rows_per_cta - 1) / p.rows_per_cta;
	const size_t smem = std::max(wgrad_smem_floor, static_cast<size_t>(p.stages) * p.stage_stride + 1024);
	const dim3 grid(static_cast<unsigned>(ctas), static_cast<unsigned>(chunks), static_cast<unsigned>(co_chunks));
	auto run = [&](auto kernel) {
		check_cuda(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)),
			"weight gradient attributes");
		kernel<<<grid, wgrad_tc_threads, smem, stream>>>(p);
	};
	if (k8 == 4)
		co == 16 ? run(conv3d_wgrad_kernel<4, 16>) : run(conv3d_wgrad_kernel<4, 32>);
	else
		co == 16 ? run(conv3d_wgrad_kernel<2, 16>) : co == 32 ? run(conv3d_wgrad_kernel<2, 32>)
													  : run(conv3d_wgrad_kernel<2, 64>);
	check_cuda(cudaGetLastError(), "weight gradient launch");
}

} // anonymous namespace
} // namespace rexlib_b200

using namespace rexlib_b200;

extern "C" int32_t rexlib_b200_conv3d_wgrad(const rexlib_b200_conv3d_wgrad_args *a, void *stream)
{
	return guarded([&] {
		require(a != nullptr, "null weight gradient arguments");
		require(a->sources == 1 || a->sources == 2, "a convolution reads one or two input volumes");
		require(a->depth >= 1 && a->height >= 1 && a->width >= 1, "volume extents must be positive");
		auto pow2 = [](int v) { return v > 0 && (v & (v - 1)) == 0; };
		if (!pow2(a->depth) || !pow2(a->height) || !pow2(a->width) || a->width < 16)
			fail(REXLIB_B200_UNSUPPORTED, "the weight gradient takes volume extents that are powers of two, a width "
				"of at least 16");
		if (a->output_channels < 16 || a->output_channels > 128 || a->output_channels % 16 != 0)
			fail(REXLIB_B200_UNSUPPORTED, "the weight gradient takes 16 to 128 output channels, a multiple of 16");
		for (int i = 0; i < a->sources; ++i)
		{
			const int c = a->input_channels[i];
			if (!(c == 16 || c == 32 || c % 64 == 0) || c > 256)
				fail(REXLIB_B200_UNSUPPORTED, "the weight gradient takes 16, 32 or a multiple of 64 input channels a "
					"source");
			require(a->inputs[i] != nullptr, "null input volume");
			require(a->input_strides[i] >= c && a->input_strides[i] % 8 == 0, "input rows must hold their channels, "
				"a multiple of 8");
			require(reinterpret_cast<uintptr_t>(a->inputs[i]) % 16 == 0, "input volumes must be 16-byte aligned");
		}
		require(a->output_grad != nullptr && reinterpret_cast<uintptr_t>(a->output_grad) % 16 == 0,
			"the output gradient must be 16-byte aligned");
		require(a->output_grad_stride >= a->output_channels && a->output_grad_stride % 8 == 0,
			"output gradient rows must hold their channels, a multiple of 8");
		require(a->weight_grad != nullptr, "null weight gradient");
		launch_wgrad(a, as_stream(stream));
	});
}
