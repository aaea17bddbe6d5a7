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
// Two kernels. The x-row kernel below (an input line copied once serves the
// three taps along x) runs widths of 16 to 256 with up to 64 output
// channels in its wide form, and other widths that are multiples of 128
// with its x halo. The box kernel, whose 128-voxel tiles are boxes of the
// volume, runs the rest, and the 2x2x2 stride-2 transposed convolution as
// a single tap (conv3d.cuh).
//
// Box kernel. Warp roles in a persistent CTA (one per SM): warp 0 issues the TMA loads
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
#include "tensor_map.cuh"
#include "conv3d.cuh"

#include <cuda.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>

namespace rexlib_b200
{
namespace
{

using namespace sm100;

constexpr int conv_threads = 192;
constexpr int conv_max_stages = 12;
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

// What the epilogue does with a finished tile: bias, ReLU or a backward
// pass's ReLU mask, BF16 stores into one or two output volumes.
struct conv_output
{
	int cout;
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
	// A 2x2x2 stride-2 transposed convolution (one tap): the cout columns
	// are (sub-position, channel) pairs of up_cout channels from sub-position
	// sub_base on, written to out0 at voxel 2 v + s of the volume twice the
	// input's extents (rows of up_cout channels). 0: a plain convolution.
	int up_cout;
	int sub_base;
};

struct alignas(64) conv_params
{
	conv_source source[2];
	int sources;
	int depth, height, width;
	int wb, hb, db, rows; // tile box and its voxels
	int tiles_x, tiles_y, tiles;
	int cout;
	int k_iterations; // stages a tile takes: taps x chunks of every source
	int taps;         // 27, or 1 for a transposed convolution's single product
	int stage_stride; // bytes of one stage (A then B), 1024-aligned
	int b_offset;     // bytes from a stage's start to its B tile
	int stages;
	uint32_t tmem_columns;
	conv_output o;
};

__device__ __forceinline__ void tile_origin(const conv_params &p, int tile, int &x0, int &y0, int &z0)
{
	x0 = (tile % p.tiles_x) * p.wb;
	y0 = ((tile / p.tiles_x) % p.tiles_y) * p.hb;
	z0 = (tile / (p.tiles_x * p.tiles_y)) * p.db;
}

__device__ __forceinline__ void report(const conv_output &o, int code)
{
	if (o.error != nullptr)
		atomicCAS(o.error, 0, code);
}

// The end of the epilogue for 16 output channels (16 g on) of one voxel:
// bias, ReLU or a backward pass's ReLU mask, and BF16 conversion.
__device__ __forceinline__ void epilogue16(const conv_output &o, int64_t voxel, int g, float (&v)[16], uint4 (&packed)[2])
{
	const int c0 = g * 16;
	const bool first = c0 < o.split;
	if (o.bias != nullptr)
#pragma unroll
		for (int i = 0; i < 16; ++i)
			v[i] += __ldg(o.bias + c0 + i);
	if (o.epilogue == 1)
	{
#pragma unroll
		for (int i = 0; i < 16; ++i)
			v[i] = fmaxf(v[i], 0.0f);
	}
	else if (o.epilogue == 2)
	{
		const __nv_bfloat16 *mask_base = first ? o.mask0 : o.mask1;
		if (mask_base != nullptr)
		{
			const __nv_bfloat16 *mask = first ? o.mask0 + voxel * o.mask0_stride + c0
											  : o.mask1 + voxel * o.mask1_stride + (c0 - o.split);
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
	__nv_bfloat162 *h = reinterpret_cast<__nv_bfloat162 *>(packed);
#pragma unroll
	for (int i = 0; i < 8; ++i)
		h[i] = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);
}

// The same, stored to the voxel's output row.
__device__ __forceinline__ void finish16(const conv_output &o, int64_t voxel, int g, float (&v)[16])
{
	uint4 packed[2];
	epilogue16(o, voxel, g, v, packed);
	const int c0 = g * 16;
	__nv_bfloat16 *out = c0 < o.split ? o.out0 + voxel * o.out0_stride + c0 : o.out1 + voxel * o.out1_stride + (c0 - o.split);
	reinterpret_cast<uint4 *>(out)[0] = packed[0];
	reinterpret_cast<uint4 *>(out)[1] = packed[1];
}

// The epilogue of one TMEM lane (one output voxel) of a finished tile: its
// cout FP32 sums from columns `column` on, 16 at a time, summed over
// `accumulators` partial accumulators cout columns apart. Every lane of the
// warp takes part in the TMEM loads; `valid` false skips the stores.
__device__ __forceinline__ void drain_voxel(const conv_output &o, uint32_t tmem_lane_base, uint32_t column,
	int64_t voxel, bool valid, int accumulators = 1)
{
	for (int g = 0; g < o.cout / 16; ++g)
	{
		float v[16];
		tmem_load16(tmem_lane_base + column + static_cast<uint32_t>(g * 16), v);
		for (int j = 1; j < accumulators; ++j)
		{
			float t[16];
			tmem_load16(tmem_lane_base + column + static_cast<uint32_t>(j * o.cout + g * 16), t);
#pragma unroll
			for (int i = 0; i < 16; ++i)
				v[i] += t[i];
		}
		if (valid)
			finish16(o, voxel, g, v);
	}
}

// The epilogue of one TMEM lane for a transposed convolution: input voxel
// (x, y, z) of a W x H volume, its cout columns 16 at a time, each group one
// sub-position's channels: bias, BF16, stored at output voxel 2 v + s.
__device__ __forceinline__ void drain_transposed(const conv_output &o, uint32_t tmem_lane_base, uint32_t column, int x,
	int y, int z, int W, int H, bool valid)
{
	for (int g = 0; g < o.cout / 16; ++g)
	{
		float v[16];
		tmem_load16(tmem_lane_base + column + static_cast<uint32_t>(g * 16), v);
		if (!valid)
			continue;
		const int n0 = g * 16;
		const int sub = o.sub_base + n0 / o.up_cout, c0 = n0 % o.up_cout;
		const int64_t u = (static_cast<int64_t>(2 * z + (sub >> 2)) * (2 * H) + 2 * y + ((sub >> 1) & 1)) * (2 * W) +
			2 * x + (sub & 1);
		if (o.bias != nullptr)
#pragma unroll
			for (int i = 0; i < 16; ++i)
				v[i] += __ldg(o.bias + c0 + i);
		uint4 packed[2];
		__nv_bfloat162 *h = reinterpret_cast<__nv_bfloat162 *>(packed);
#pragma unroll
		for (int i = 0; i < 8; ++i)
			h[i] = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);
		uint4 *out = reinterpret_cast<uint4 *>(o.out0 + u * o.up_cout + c0);
		out[0] = packed[0];
		out[1] = packed[1];
	}
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
				for (int tap = 0; tap < p.taps && !*stop; ++tap)
				{
					// One tap: the input voxel itself (a transposed convolution).
					const bool one = p.taps == 1;
					const int dz = one ? 0 : tap / 9 - 1, dy = one ? 0 : (tap / 3) % 3 - 1, dx = one ? 0 : tap % 3 - 1;
					for (int src = 0; src < p.sources; ++src)
					{
						const conv_source &S = p.source[src];
						for (int c = 0; c < S.chunks; ++c)
						{
							if (*stop || !mbarrier_wait(&empty[s], phase ^ 1, p.o.wait_ns))
							{
								if (!*stop)
									report(p.o, 1);
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
				if (!mbarrier_wait(&tmem_empty[buffer], ((local >> 1) & 1) ^ 1, p.o.wait_ns))
				{
					if (!*stop)
						report(p.o, 2);
					*stop = 1;
					break;
				}
				tcgen05_fence_after();
				const uint32_t d = tmem + static_cast<uint32_t>(buffer * p.cout);
				int k = 0;
				for (int tap = 0; tap < p.taps && !*stop; ++tap)
					for (int src = 0; src < p.sources && !*stop; ++src)
					{
						const conv_source &S = p.source[src];
						const uint32_t row_bytes = static_cast<uint32_t>(S.chunk * 2);
						for (int c = 0; c < S.chunks; ++c, ++k)
						{
							if (*stop || !mbarrier_wait(&full[s], phase, p.o.wait_ns))
							{
								if (!*stop)
									report(p.o, 3);
								*stop = 1;
								break;
							}
							tcgen05_fence_after();
							const uint32_t a_addr = smem_address(smem + s * p.stage_stride);
							const uint64_t a0 = kmajor_descriptor(a_addr, row_bytes);
							const uint64_t b0 = kmajor_descriptor(a_addr + static_cast<uint32_t>(p.b_offset), row_bytes);
							for (int kk = 0; kk < S.chunk / 16; ++kk) // K steps of 32 bytes: 2 in the address field
								mma_f16(d, a0 + 2 * kk, b0 + 2 * kk, idesc, (k > 0 || kk > 0) ? 1u : 0u);
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
			if (*stop || !mbarrier_wait(&tmem_full[buffer], (local >> 1) & 1, p.o.wait_ns))
			{
				if (!*stop)
					report(p.o, 4);
				*stop = 1;
				break;
			}
			tcgen05_fence_after();
			int x0, y0, z0;
			tile_origin(p, tile, x0, y0, z0);
			const bool valid = row < p.rows;
			const int x = x0 + row % p.wb, y = y0 + (row / p.wb) % p.hb, z = z0 + row / (p.wb * p.hb);
			const int64_t voxel = (static_cast<int64_t>(z) * p.height + y) * p.width + x;
			if (p.o.up_cout > 0)
				drain_transposed(p.o, tmem + (static_cast<uint32_t>(quarter * 32) << 16),
					static_cast<uint32_t>(buffer * p.cout), x, y, z, p.width, p.height, valid);
			else
				drain_voxel(p.o, tmem + (static_cast<uint32_t>(quarter * 32) << 16), static_cast<uint32_t>(buffer * p.cout),
					voxel, valid);
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
// The same convolution over x-rows of 128 voxels (W a multiple of 128), with
// each input line fetched once for the three taps along x.
//
// A tile is one x-row of 128 output voxels. For each (dz, dy) one TMA load
// brings the input line x0 - 1 .. x0 + 128 of row (y + dy, z + dz) (130
// voxels; zeros outside the volume, filled by the TMA unit) into shared
// memory in the interleaved K-major layout: the tensor map views the volume
// as (8 channels, x, y, z, channel pieces of 8), so the box lands as piece
// k of halo voxel r at 16 (130 k + r) bytes. In that layout a tile may start
// at any row, so the taps dx = -1, 0, +1 are the same line read from rows
// 0, 1 and 2: one load serves three taps (the box kernel fetches every tap's
// 128 voxels again), and the L2-to-SM traffic of the input falls threefold.
//
// Every source takes chunks of one width (CHUNK). A stage holds LINES
// input lines (3, one dz, for chunks of 16 or 32 channels; 1 for 64),
// loaded as one 5D box (lines consecutive in y), and the weights of their
// 3 LINES taps as one 3D box over a (channels, outputs, taps) view, which
// lands tap-major, each tap a whole B operand: two TMA instructions a
// stage, which feeds 9 to 18 MMAs. The MMAs of a tile chain on NACC partial
// accumulators (by tap column dx), which the epilogue sums. The MMA loop is
// flat, its operand geometry fixed at compile time: one thread issues every
// MMA, and the instructions between them are what its issue rate pays for.
// Warp roles as in the box kernel: warp 0 loads, warp 1 issues the MMAs,
// warps 2-5 drain the accumulators.
//
// The wide form (HALVES 1 or 2; widths of 16 to 256, up to 64 output
// channels): a tile is T = 128 HALVES voxels, R = T / W consecutive rows
// y0 .. y0 + R - 1 at z (one row of 256 for W = 256), and a stage's box
// holds the rows y0 - 1 + dy of its lines, R + LINES - 1 rows of W voxels
// without an x halo, consecutive in shared memory. One MMA of N = 3 cout
// takes the three x taps of a line at once: A is the line's run of 128
// positions (unshifted; a half's second run 128 positions on) and B the
// three taps' weight boxes, consecutive in the stage, so that
//   D[m][dx cout + o] = sum_i x[position m][i] w[(dz, dy, dx)][o][i]
// and the output is y[m] = D[m - 1][dx = 0] + D[m][dx = 1] + D[m + 1][dx = 2],
// the first term left out at x = 0 and the last at x = W - 1 (the padding).
// A third as many MMAs as the tap-by-tap form, each no slower at these
// widths. The epilogue takes the neighbouring TMEM lanes' terms by warp
// shuffles, and across the warps' 32-lane blocks through shared memory,
// behind an mbarrier whose waits are bounded like every other.
constexpr int rows_threads = 192;
constexpr int rows_halo = 130;
constexpr int rows_piece_bytes = rows_halo * 16; // one 8-channel piece of a line

struct alignas(64) rows_source
{
	CUtensorMap line;    // (8 channels, x, y, z, pieces of 8), box (8, 130, 1, 1, chunk / 8), no swizzle
	CUtensorMap weights; // (input channels of all sources, 27, output channels), box (chunk, 1, output channels)
	int chunk;           // channels a stage takes (16, 32 or 64)
	int chunks;
	int weight_channel;  // this source's first input channel in the weights
	int line_bytes;      // bytes of a stage's lines
};

struct alignas(64) rows_params
{
	rows_source source[2];
	int sources;
	int depth, height, width;
	int tiles_x, tiles;
	int rows_per_tile; // R: rows of W voxels a tile takes (1 where W is a multiple of 128)
	int tiles_y;       // H / R
	int cout;
	int stage_stride; // bytes of one stage: the input lines, then a weight box per tap
	int b_offset;     // bytes from a stage's start to its first weight box
	int b_box;        // bytes between weight boxes (cout x the widest chunk x 2: whole swizzle atoms)
	int stages;
	uint32_t tmem_columns;
	conv_output o;
};

// HALVES 0: rows of 128 with the x halo, NACC partial accumulators by tap
// column; HALVES 1 or 2: the wide form (NACC unused).
// LINES: the (dz, dy) lines a stage holds: 1 (64-channel chunks), 3 (one
// dz), or 9 (all three dz planes, one box of z extent 3; wide form with
// 16-channel chunks, where three such stages fit).
template <int CHUNK, int NACC, int HALVES, int LINES>
__global__ void __launch_bounds__(rows_threads, 1) conv3d_rows_kernel(const __grid_constant__ rows_params p)
{
	constexpr bool HALO = HALVES == 0;
	// Every source takes chunks of CHUNK channels, a K step 16 of them.
	constexpr int KSTEPS = CHUNK / 16;

	extern __shared__ __align__(1024) unsigned char smem_raw[];
	unsigned char *smem = reinterpret_cast<unsigned char *>(
		(reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
	__shared__ uint64_t full[conv_max_stages], empty[conv_max_stages], tmem_full[2], tmem_empty[2], drained;
	__shared__ uint32_t tmem_base;
	__shared__ int failed;
	// The wide form's exchange between the epilogue warps' lane blocks:
	// [round parity][to the next block (dx = 0 term of its last lane), to
	// the previous one (dx = 2 term of its first lane)][block][16 channels].
	constexpr int BLOCKS = HALVES > 0 ? 4 * HALVES : 4; // the epilogue warps' 32-lane blocks of a tile
	__shared__ float4 edge[2][2][BLOCKS][4];
	__shared__ uint64_t edge_ready;

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
		mbarrier_init(&edge_ready, 4);
		failed = 0;
		fence_barrier_init();
	}
	if (warp == 0 && lane == 0)
		for (int i = 0; i < p.sources; ++i)
		{
			prefetch_tensor_map(&p.source[i].line);
			prefetch_tensor_map(&p.source[i].weights);
		}
	if (warp == 1)
		tmem_allocate(&tmem_base, p.tmem_columns);
	tcgen05_fence_before();
	__syncthreads();
	tcgen05_fence_after();
	const uint32_t tmem = tmem_base;
	const int H = p.height, W = p.width;
	constexpr int groups = 9 / LINES; // stages of a tile per source chunk

	if (warp == 0)
	{
		// TMA producer.
		if (lane == 0)
		{
			int s = 0;
			uint32_t phase = 0;
			uint32_t issued = 0;       // stages that have taken loads
			uint32_t issued_phase = 0; // bit s: the phase parity of stage s's last loads
			for (int tile = blockIdx.x; tile < p.tiles && !*stop; tile += gridDim.x)
			{
				int x0 = 0, y, z; // without the halo y is the tile's first row y0
				if constexpr (HALO)
				{
					x0 = (tile % p.tiles_x) * 128;
					y = (tile / p.tiles_x) % H;
					z = tile / (p.tiles_x * H);
				}
				else
				{
					y = (tile % p.tiles_y) * p.rows_per_tile;
					z = tile / p.tiles_y;
				}
				for (int g = 0; g < groups && !*stop; ++g)
					for (int src = 0; src < p.sources && !*stop; ++src)
					{
						const rows_source &S = p.source[src];
						const int k8 = S.chunk / 8;
						for (int c = 0; c < S.chunks; ++c)
						{
							if (*stop || !mbarrier_wait(&empty[s], phase ^ 1, p.o.wait_ns))
							{
								if (!*stop)
									report(p.o, 1);
								*stop = 1;
								break;
							}
							unsigned char *stage = smem + s * p.stage_stride;
							const int first_tap = g * 3 * LINES; // (dz, dy) of the stage's first line, times 3
							const int line_index = first_tap / 3;  // (dz + 1) * 3 + dy + 1 of that line
							mbarrier_expect_tx(&full[s], static_cast<uint32_t>(S.line_bytes + 3 * LINES * p.cout * S.chunk * 2));
							// The stage's LINES lines (consecutive in y) in one box,
							// the weights of its 3 LINES taps in another.
							if constexpr (HALO)
								tma_load_5d(stage, &S.line, &full[s], 0, x0 - 1, y + line_index % 3 - 1, z + line_index / 3 - 1,
									c * k8);
							else
								tma_load_4d(stage, &S.line, &full[s], c * S.chunk, 0, y + line_index % 3 - 1,
									z + line_index / 3 - 1);
							tma_load_3d(stage + p.b_offset, &S.weights, &full[s], S.weight_channel + c * S.chunk, 0,
								first_tap);
							issued |= 1u << s;
							issued_phase = (issued_phase & ~(1u << s)) | (phase << s);
							if (++s == p.stages)
							{
								s = 0;
								phase ^= 1;
							}
						}
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
		// MMA issuer.
		if (lane == 0)
		{
			const uint32_t idesc = bf16_idesc(128, static_cast<uint32_t>(HALO ? p.cout : 3 * p.cout));
			const uint32_t smem_base = smem_address(smem);
			const uint32_t stage_stride = static_cast<uint32_t>(p.stage_stride);
			const uint32_t b_offset = static_cast<uint32_t>(p.b_offset);
			const uint32_t box_step = static_cast<uint32_t>(p.b_box) >> 4;
			// With the halo: bytes between pieces (the K-direction core
			// matrices), and 16-byte steps between lines and between K steps.
			constexpr uint32_t lead = LINES * rows_piece_bytes;
			constexpr uint32_t line_step = rows_piece_bytes >> 4;
			constexpr uint32_t kstep = 2 * lead >> 4;
			// The wide form: 16-byte units between its lines (rows of W voxels).
			const uint32_t row_units = static_cast<uint32_t>(p.width) * (CHUNK / 8);
			// ... and between its dz planes when a stage holds all nine lines.
			const uint32_t plane_units = static_cast<uint32_t>(p.rows_per_tile + 2) * row_units;
			int stages_per_tile = 0;
			for (int src = 0; src < p.sources; ++src)
				stages_per_tile += groups * p.source[src].chunks;
			int s = 0;
			uint32_t phase = 0;
			int local = 0;
			for (int tile = blockIdx.x; tile < p.tiles && !*stop; tile += gridDim.x, ++local)
			{
				const int buffer = local & 1;
				if (!mbarrier_wait(&tmem_empty[buffer], ((local >> 1) & 1) ^ 1, p.o.wait_ns))
				{
					if (!*stop)
						report(p.o, 2);
					*stop = 1;
					break;
				}
				tcgen05_fence_after();
				// NACC partial accumulators, by tap column dx: consecutive
				// MMAs chain on different accumulators. The stages of a tile
				// are consumed in order whatever source and chunk they carry
				// (the producer knows), so the loop is flat, with the
				// operand geometry fixed at compile time: the instructions
				// between MMAs are what this thread's issue rate pays for.
				const uint32_t d = tmem + static_cast<uint32_t>(buffer * (HALO ? NACC : 3 * HALVES) * p.cout);
				for (int st = 0; st < stages_per_tile; ++st)
				{
					if (*stop || !mbarrier_wait(&full[s], phase, p.o.wait_ns))
					{
						if (!*stop)
							report(p.o, 3);
						*stop = 1;
						break;
					}
					tcgen05_fence_after();
					// Descriptors of the stage's first operands; the others differ
					// in the start address field only (addresses below 256 KB: the
					// 14-bit field takes the sum). Tap column dx starts dx rows (16 dx
					// bytes) into a line; a K step of 16 is two pieces further.
					const uint32_t a_addr = smem_base + static_cast<uint32_t>(s) * stage_stride;
					const uint64_t a0 = interleaved_descriptor(a_addr, lead, 128);
					const uint64_t b0 = kmajor_descriptor(a_addr + b_offset, CHUNK * 2);
					const bool tile_start = st == 0;
					if constexpr (HALO)
					{
#pragma unroll
						for (int l = 0; l < LINES; ++l)
#pragma unroll
							for (int dx = 0; dx < 3; ++dx)
#pragma unroll
								for (int kk = 0; kk < KSTEPS; ++kk)
								{
									const bool fresh = tile_start && l == 0 && kk == 0 && dx < NACC;
									mma_f16(d + static_cast<uint32_t>((dx % NACC) * p.cout),
										a0 + (l * line_step + kk * kstep + dx),
										b0 + ((l * 3 + dx) * box_step + kk * 2), idesc, fresh ? 0u : 1u);
								}
					}
					else
					{
						// One MMA of N = 3 cout a (line, K step, half): A is the
						// line's run of positions as K-major rows of CHUNK
						// channels, swizzled to their width (every start a whole
						// number of 8-row atoms on: W is 16 or more), a K step 32
						// bytes into the row; B spans the line's three tap boxes.
						const uint64_t as = kmajor_descriptor(a_addr, CHUNK * 2);
#pragma unroll
						for (int l = 0; l < LINES; ++l)
#pragma unroll
							for (int kk = 0; kk < KSTEPS; ++kk)
#pragma unroll
								for (int h = 0; h < HALVES; ++h)
								{
									const bool fresh = tile_start && l == 0 && kk == 0;
									mma_f16(d + static_cast<uint32_t>(h * 3 * p.cout),
										as + ((l / 3) * plane_units + (l % 3) * row_units + h * (128 * CHUNK / 8) + kk * 2),
										b0 + (l * 3 * box_step + kk * 2), idesc, fresh ? 0u : 1u);
								}
					}
					mma_commit(&empty[s]); // the stage is free once these MMAs have read it
					if (++s == p.stages)
					{
						s = 0;
						phase ^= 1;
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
		const uint32_t lane_base = tmem + (static_cast<uint32_t>(quarter * 32) << 16);
		int local = 0;
		uint32_t round = 0; // exchanges of the wide form so far
		for (int tile = blockIdx.x; tile < p.tiles; tile += gridDim.x, ++local)
		{
			const int buffer = local & 1;
			// One decision for the whole warp: the TMEM loads take every lane.
			const bool ready = __all_sync(0xffffffffu, !*stop && mbarrier_wait(&tmem_full[buffer], (local >> 1) & 1,
																	 p.o.wait_ns));
			if (!ready)
			{
				if (lane == 0 && !*stop)
					report(p.o, 4);
				*stop = 1;
				break;
			}
			tcgen05_fence_after();
			if constexpr (HALO)
			{
				const int x0 = (tile % p.tiles_x) * 128;
				const int y = (tile / p.tiles_x) % H, z = tile / (p.tiles_x * H);
				const int64_t voxel = (static_cast<int64_t>(z) * H + y) * W + x0 + row;
				drain_voxel(p.o, lane_base, static_cast<uint32_t>(buffer * NACC * p.cout), voxel, true, NACC);
			}
			else
			{
				// Lane block k = 4 h + quarter holds positions 32 k .. 32 k + 31
				// of the tile: the neighbours' terms by shuffles within it,
				// and from blocks k - 1 and k + 1 through `edge`.
				const int y0 = (tile % p.tiles_y) * p.rows_per_tile, z = tile / p.tiles_y;
				const int64_t base = (static_cast<int64_t>(z) * H + y0) * W;
				const uint32_t column = static_cast<uint32_t>(buffer * 3 * HALVES * p.cout);
				bool ok = true;
				if constexpr (HALVES > 2)
				{
					// Four halves: the three terms of every half do not fit in
					// registers at once, so the exchange takes two passes over
					// TMEM: the boundary terms of every half first, then each
					// half's three terms again for the sums.
					for (int g = 0; g < p.cout / 16; ++g, ++round)
					{
						const int par = static_cast<int>(round & 1u);
#pragma unroll
						for (int h = 0; h < HALVES; ++h)
						{
							uint32_t r0[16], r2[16];
							const uint32_t c = lane_base + column + static_cast<uint32_t>(h * 3 * p.cout + g * 16);
							tmem_load16_async(c, r0);
							tmem_load16_async(c + static_cast<uint32_t>(2 * p.cout), r2);
							tmem_wait_loads();
							tmem_loaded(r0);
							tmem_loaded(r2);
							const int k = h * 4 + quarter;
							if (lane == 31)
#pragma unroll
								for (int i = 0; i < 4; ++i)
									edge[par][0][k][i] = make_float4(__uint_as_float(r0[4 * i]), __uint_as_float(r0[4 * i + 1]),
										__uint_as_float(r0[4 * i + 2]), __uint_as_float(r0[4 * i + 3]));
							if (lane == 0)
#pragma unroll
								for (int i = 0; i < 4; ++i)
									edge[par][1][k][i] = make_float4(__uint_as_float(r2[4 * i]), __uint_as_float(r2[4 * i + 1]),
										__uint_as_float(r2[4 * i + 2]), __uint_as_float(r2[4 * i + 3]));
						}
						__syncwarp();
						if (lane == 0)
							mbarrier_arrive(&edge_ready);
						ok = __all_sync(0xffffffffu, mbarrier_wait(&edge_ready, round & 1u, p.o.wait_ns));
						if (!ok)
						{
							if (lane == 0 && !*stop)
								report(p.o, 5);
							*stop = 1;
							break;
						}
#pragma unroll 1
						for (int h = 0; h < HALVES; ++h)
						{
							uint32_t r0[16], r1[16], r2[16];
							const uint32_t c = lane_base + column + static_cast<uint32_t>(h * 3 * p.cout + g * 16);
							tmem_load16_async(c, r0);
							tmem_load16_async(c + static_cast<uint32_t>(p.cout), r1);
							tmem_load16_async(c + static_cast<uint32_t>(2 * p.cout), r2);
							tmem_wait_loads();
							tmem_loaded(r0);
							tmem_loaded(r1);
							tmem_loaded(r2);
							const int k = h * 4 + quarter;
							const int m = k * 32 + lane;
							const int x = m & (W - 1);
							float from_prev[16], from_next[16];
#pragma unroll
							for (int i = 0; i < 16; ++i)
								from_prev[i] = from_next[i] = 0.0f;
							if (lane == 0 && k > 0)
#pragma unroll
								for (int i = 0; i < 4; ++i)
								{
									const float4 e = edge[par][0][k - 1][i];
									from_prev[4 * i] = e.x;
									from_prev[4 * i + 1] = e.y;
									from_prev[4 * i + 2] = e.z;
									from_prev[4 * i + 3] = e.w;
								}
							if (lane == 31 && k < 4 * HALVES - 1)
#pragma unroll
								for (int i = 0; i < 4; ++i)
								{
									const float4 e = edge[par][1][k + 1][i];
									from_next[4 * i] = e.x;
									from_next[4 * i + 1] = e.y;
									from_next[4 * i + 2] = e.z;
									from_next[4 * i + 3] = e.w;
								}
							float v[16];
#pragma unroll
							for (int i = 0; i < 16; ++i)
							{
								float left = __shfl_up_sync(0xffffffffu, __uint_as_float(r0[i]), 1);
								float right = __shfl_down_sync(0xffffffffu, __uint_as_float(r2[i]), 1);
								if (lane == 0)
									left = from_prev[i];
								if (lane == 31)
									right = from_next[i];
								v[i] = __uint_as_float(r1[i]) + (x > 0 ? left : 0.0f) + (x < W - 1 ? right : 0.0f);
							}
							finish16(p.o, base + m, g, v);
						}
					}
				}
				else
				for (int g = 0; g < p.cout / 16; ++g, ++round)
				{
					// The dx = 0, 1, 2 terms of both halves: six loads in flight,
					// one wait.
					uint32_t r0[HALVES][16], r1[HALVES][16], r2[HALVES][16];
#pragma unroll
					for (int h = 0; h < HALVES; ++h)
					{
						const uint32_t c = lane_base + column + static_cast<uint32_t>(h * 3 * p.cout + g * 16);
						tmem_load16_async(c, r0[h]);
						tmem_load16_async(c + static_cast<uint32_t>(p.cout), r1[h]);
						tmem_load16_async(c + static_cast<uint32_t>(2 * p.cout), r2[h]);
					}
					tmem_wait_loads();
					float t0[HALVES][16], t1[HALVES][16], t2[HALVES][16];
#pragma unroll
					for (int h = 0; h < HALVES; ++h)
					{
						tmem_loaded(r0[h]);
						tmem_loaded(r1[h]);
						tmem_loaded(r2[h]);
#pragma unroll
						for (int i = 0; i < 16; ++i)
						{
							t0[h][i] = __uint_as_float(r0[h][i]);
							t1[h][i] = __uint_as_float(r1[h][i]);
							t2[h][i] = __uint_as_float(r2[h][i]);
						}
					}
					const int par = static_cast<int>(round & 1u);
#pragma unroll
					for (int h = 0; h < HALVES; ++h)
					{
						const int k = h * 4 + quarter;
						// 16-byte shared accesses: the epilogue's shared memory traffic
						// competes with the tensor cores' operand reads.
						if (lane == 31)
#pragma unroll
							for (int i = 0; i < 4; ++i)
								edge[par][0][k][i] = make_float4(t0[h][4 * i], t0[h][4 * i + 1], t0[h][4 * i + 2], t0[h][4 * i + 3]);
						if (lane == 0)
#pragma unroll
							for (int i = 0; i < 4; ++i)
								edge[par][1][k][i] = make_float4(t2[h][4 * i], t2[h][4 * i + 1], t2[h][4 * i + 2], t2[h][4 * i + 3]);
					}
					__syncwarp();
					if (lane == 0)
						mbarrier_arrive(&edge_ready);
					ok = __all_sync(0xffffffffu, mbarrier_wait(&edge_ready, round & 1u, p.o.wait_ns));
					if (!ok)
					{
						if (lane == 0 && !*stop)
							report(p.o, 5);
						*stop = 1;
						break;
					}
#pragma unroll
					for (int h = 0; h < HALVES; ++h)
					{
						const int k = h * 4 + quarter;
						const int m = k * 32 + lane;
						const int x = m & (W - 1);
						// The neighbouring blocks' terms, for lanes 0 and 31.
						float from_prev[16], from_next[16];
#pragma unroll
						for (int i = 0; i < 16; ++i)
							from_prev[i] = from_next[i] = 0.0f;
						if (lane == 0 && k > 0)
#pragma unroll
							for (int i = 0; i < 4; ++i)
							{
								const float4 e = edge[par][0][k - 1][i];
								from_prev[4 * i] = e.x;
								from_prev[4 * i + 1] = e.y;
								from_prev[4 * i + 2] = e.z;
								from_prev[4 * i + 3] = e.w;
							}
						if (lane == 31 && k < 4 * HALVES - 1)
#pragma unroll
							for (int i = 0; i < 4; ++i)
							{
								const float4 e = edge[par][1][k + 1][i];
								from_next[4 * i] = e.x;
								from_next[4 * i + 1] = e.y;
								from_next[4 * i + 2] = e.z;
								from_next[4 * i + 3] = e.w;
							}
						float v[16];
#pragma unroll
						for (int i = 0; i < 16; ++i)
						{
							float left = __shfl_up_sync(0xffffffffu, t0[h][i], 1);
							float right = __shfl_down_sync(0xffffffffu, t2[h][i], 1);
							if (lane == 0)
								left = from_prev[i];
							if (lane == 31)
								right = from_next[i];
							v[i] = t1[h][i] + (x > 0 ? left : 0.0f) + (x < W - 1 ? right : 0.0f);
						}
						finish16(p.o, base + m, g, v);
					}
				}
				if (!ok)
					break;
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

} // anonymous namespace
} // namespace rexlib_b200

using namespace rexlib_b200;

namespace rexlib_b200
{
namespace
{

conv_output output_of(const rexlib_b200_conv3d_args *a)
{
	conv_output o{};
	o.cout = a->output_channels;
	o.epilogue = a->epilogue;
	require(o.epilogue >= 0 && o.epilogue <= 2, "unknown epilogue");
	o.bias = a->bias;
	require(a->outputs[0] != nullptr, "null output volume");
	o.split = a->output_split > 0 ? a->output_split : o.cout;
	require(o.split % 16 == 0 && o.split <= o.cout, "the output split falls on a multiple of 16 channels");
	require(o.split == o.cout || a->outputs[1] != nullptr, "null second output volume");
	o.out0 = static_cast<__nv_bfloat16 *>(a->outputs[0]);
	o.out1 = static_cast<__nv_bfloat16 *>(a->outputs[1]);
	o.out0_stride = a->output_strides[0];
	o.out1_stride = a->output_strides[1];
	o.mask0 = static_cast<const __nv_bfloat16 *>(a->masks[0]);
	o.mask1 = static_cast<const __nv_bfloat16 *>(a->masks[1]);
	o.mask0_stride = a->mask_strides[0];
	o.mask1_stride = a->mask_strides[1];
	for (int i = 0; i < 2; ++i)
		require(reinterpret_cast<uintptr_t>(a->outputs[i]) % 16 == 0 && a->output_strides[i] % 8 == 0 &&
				reinterpret_cast<uintptr_t>(a->masks[i]) % 16 == 0 && a->mask_strides[i] % 8 == 0,
			"outputs and masks must be 16-byte aligned, their rows a multiple of 8 channels");
	o.error = a->error;
	o.wait_ns = a->wait_limit_ns > 0 ? static_cast<uint64_t>(a->wait_limit_ns) : default_wait_ns;
	return o;
}

// The weights' tensor map of source i: (all input channels, 27, cout), box
// (chunk, 1, cout), swizzled to the chunk's width.
void encode_weights(CUtensorMap *map, const rexlib_b200_conv3d_args *a, int total_in, int chunk)
{
	const cuuint64_t wdims[3] = {static_cast<cuuint64_t>(total_in), 27, static_cast<cuuint64_t>(a->output_channels)};
	const cuuint64_t wstrides[2] = {static_cast<cuuint64_t>(total_in) * 2, static_cast<cuuint64_t>(total_in) * 2 * 27};
	const cuuint32_t wbox[3] = {static_cast<cuuint32_t>(chunk), 1, static_cast<cuuint32_t>(a->output_channels)};
	encode(map, a->weights, 3, wdims, wstrides, wbox, chunk * 2);
}

uint32_t tmem_columns_for(int cout)
{
	uint32_t columns = 32;
	while (columns < static_cast<uint32_t>(2 * cout))
		columns *= 2;
	return columns;
}

// The wide form's halves a tile (1 or 2), or 0 where it does not apply:
// tiles of 256 voxels where two buffers of 6 cout accumulator columns fit
// in TMEM (cout up to 32), of 128 up to 64 output channels; a tile holds
// whole rows (W at most the tile, 16 or more) and whole tiles fill H.
int wide_halves(const rexlib_b200_conv3d_args *a)
{
	const int W = a->width, H = a->height, cout = a->output_channels;
	// Four halves (tiles of 512 voxels, two buffers of 12 cout columns) at 16
	// output channels and widths of 128 or 256: fewer input rows loaded per
	// output row, more MMAs per stage.
	if (cout <= 16 && W >= 128 && W <= 256 && H % (512 / W) == 0)
		return 4;
	const int halves = cout <= 32 ? 2 : cout <= 64 ? 1 : 0;
	if (halves == 0 || W < 16 || W > 128 * halves)
		return 0;
	return H % (128 * halves / W) == 0 ? halves : 0;
}

void launch_rows(const rexlib_b200_conv3d_args *a, int total_in, cudaStream_t stream)
{
	rows_params p{};
	p.sources = a->sources;
	p.depth = a->depth;
	p.height = a->height;
	p.width = a->width;
	const int W = a->width, H = a->height, D = a->depth;
	// The wide form where it applies (R = 128 halves / W rows a tile, no x
	// halo); otherwise rows of 128 voxels with the halo (W a multiple of 128).
	const int halves = wide_halves(a);
	const bool halo = halves == 0;
	const int R = halo ? 1 : 128 * halves / W;
	p.tiles_x = halo ? W / 128 : 1;
	p.rows_per_tile = R;
	p.tiles_y = H / R;
	p.tiles = halo ? p.tiles_x * H * D : p.tiles_y * D;
	p.cout = a->output_channels;
	int line_bytes = 0, max_chunk = 16;
	// One chunk width for every source: the narrowest source's (a wider
	// source is read in more chunks).
	max_chunk = 64;
	for (int i = 0; i < a->sources; ++i)
		max_chunk = std::min(max_chunk, std::min(a->input_channels[i], 64));
	// Three lines a stage for chunks of 16 or 32 channels (whose MMAs are
	// small), one for 64; all nine in the wide form with 16-channel chunks
	// where three such stages (three planes of R + 2 rows and 27 weight
	// boxes) fit, which pays the stage's barrier round trip once for all of
	// a tile's MMAs (with two stages the copies no longer hide: slower).
	int lines = max_chunk <= 32 ? 3 : 1;
	if (!halo && halves < 4 && max_chunk == 16)
	{
		const size_t planes = static_cast<size_t>(3) * (R + 2) * W * 16 * 2;
		const size_t stage = ((planes + 1023) / 1024 * 1024 + 27 * static_cast<size_t>(p.cout) * 16 * 2 + 1023) / 1024 * 1024;
		if (3 * stage <= conv_smem_budget)
			lines = 9;
	}
	const int planes = lines == 9 ? 3 : 1;
	for (int i = 0; i < a->sources; ++i)
	{
		rows_source &S = p.source[i];
		const int c = a->input_channels[i];
		S.chunk = max_chunk;
		S.chunks = c / S.chunk;
		S.weight_channel = i == 0 ? 0 : a->input_channels[0];
		// With the halo: the volume as (8 channels, x, y, z, pieces of 8
		// channels), a box of `lines` consecutive lines of 130 voxels landing
		// as piece k, line l at 2080 (lines k + l) bytes. The wide form: the
		// volume as (channels, x, y, z), a box of R + lines - 1 rows of W
		// voxels landing as K-major rows of the chunk's channels, swizzled to
		// their width, position r of row j at row (W j + r).
		const cuuint64_t row = static_cast<cuuint64_t>(a->input_strides[i]) * 2;
		if (halo)
		{
			S.line_bytes = (S.chunk / 8) * lines * rows_piece_bytes;
			const cuuint64_t ldims[5] = {8, static_cast<cuuint64_t>(W), static_cast<cuuint64_t>(H),
				static_cast<cuuint64_t>(D), static_cast<cuuint64_t>(c / 8)};
			const cuuint64_t lstrides[4] = {row, row * W, row * W * H, 16};
			const cuuint32_t lbox[5] = {8, rows_halo, static_cast<cuuint32_t>(lines), 1,
				static_cast<cuuint32_t>(S.chunk / 8)};
			encode(&S.line, a->inputs[i], 5, ldims, lstrides, lbox, 0);
		}
		else
		{
			const int box_rows = R + (lines == 9 ? 2 : lines - 1);
			S.line_bytes = planes * box_rows * W * S.chunk * 2;
			const cuuint64_t ldims[4] = {static_cast<cuuint64_t>(c), static_cast<cuuint64_t>(W),
				static_cast<cuuint64_t>(H), static_cast<cuuint64_t>(D)};
			const cuuint64_t lstrides[3] = {row, row * W, row * W * H};
			const cuuint32_t lbox[4] = {static_cast<cuuint32_t>(S.chunk), static_cast<cuuint32_t>(W),
				static_cast<cuuint32_t>(box_rows), static_cast<cuuint32_t>(planes)};
			encode(&S.line, a->inputs[i], 4, ldims, lstrides, lbox, S.chunk * 2);
		}
		line_bytes = std::max(line_bytes, S.line_bytes);
		// The weights as (input channels, output channels, 27 taps): a box
		// of 3 lines taps lands tap-major, each tap a whole B operand.
		const cuuint64_t wdims[3] = {static_cast<cuuint64_t>(total_in), static_cast<cuuint64_t>(p.cout), 27};
		const cuuint64_t wstrides[2] = {static_cast<cuuint64_t>(total_in) * 2 * 27, static_cast<cuuint64_t>(total_in) * 2};
		const cuuint32_t wbox[3] = {static_cast<cuuint32_t>(S.chunk), static_cast<cuuint32_t>(p.cout),
			static_cast<cuuint32_t>(3 * lines)};
		encode(&S.weights, a->weights, 3, wdims, wstrides, wbox, S.chunk * 2);
	}
	p.b_offset = (line_bytes + 1023) / 1024 * 1024;
	p.b_box = p.cout * max_chunk * 2;
	p.stage_stride = (p.b_offset + 3 * lines * p.b_box + 1023) / 1024 * 1024;
	p.stages = static_cast<int>(std::min<size_t>(conv_max_stages, conv_smem_budget / p.stage_stride));
	require(p.stages >= 2, "the convolution's stages do not fit in shared memory");
	// With the halo, partial accumulators by tap column: three where two
	// buffers of them fit in the 512 TMEM columns, two otherwise. The wide
	// form: 3 cout columns a half.
	const int accumulators = p.cout <= 64 ? 3 : 2;
	p.tmem_columns = tmem_columns_for((halo ? accumulators : 3 * halves) * p.cout);
	p.o = output_of(a);
	const size_t smem = static_cast<size_t>(p.stages) * p.stage_stride + 1024;
	const int grid = std::min(p.tiles, sm_count());
	auto run = [&](auto kernel) {
		check_cuda(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)),
			"convolution attributes");
		kernel<<<grid, rows_threads, smem, stream>>>(p);
	};
	if (halves == 4)
		switch (max_chunk)
		{
		case 16: run(conv3d_rows_kernel<16, 1, 4, 3>); break;
		case 32: run(conv3d_rows_kernel<32, 1, 4, 3>); break;
		default: run(conv3d_rows_kernel<64, 1, 4, 1>); break;
		}
	else if (halves == 2)
		switch (max_chunk)
		{
		case 16: lines == 9 ? run(conv3d_rows_kernel<16, 1, 2, 9>) : run(conv3d_rows_kernel<16, 1, 2, 3>); break;
		case 32: run(conv3d_rows_kernel<32, 1, 2, 3>); break;
		default: run(conv3d_rows_kernel<64, 1, 2, 1>); break;
		}
	else if (halves == 1)
		switch (max_chunk)
		{
		case 16: lines == 9 ? run(conv3d_rows_kernel<16, 1, 1, 9>) : run(conv3d_rows_kernel<16, 1, 1, 3>); break;
		case 32: run(conv3d_rows_kernel<32, 1, 1, 3>); break;
		default: run(conv3d_rows_kernel<64, 1, 1, 1>); break;
		}
	else
		switch (max_chunk)
		{
		case 16:
			accumulators == 3 ? run(conv3d_rows_kernel<16, 3, 0, 3>) : run(conv3d_rows_kernel<16, 2, 0, 3>);
			break;
		case 32:
			accumulators == 3 ? run(conv3d_rows_kernel<32, 3, 0, 3>) : run(conv3d_rows_kernel<32, 2, 0, 3>);
			break;
		default:
			accumulators == 3 ? run(conv3d_rows_kernel<64, 3, 0, 1>) : run(conv3d_rows_kernel<64, 2, 0, 1>);
			break;
		}
	check_cuda(cudaGetLastError(), "convolution launch");
}

void launch_boxes(const rexlib_b200_conv3d_args *a, int total_in, cudaStream_t stream)
{
	const int D = a->depth, H = a->height, W = a->width;
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
	int max_chunk = 16;
	int k_iterations = 0;
	for (int i = 0; i < a->sources; ++i)
	{
		const int c = a->input_channels[i];
		conv_source &S = p.source[i];
		S.chunk = std::min(c, 64);
		S.chunks = c / S.chunk;
		S.weight_channel = i == 0 ? 0 : a->input_channels[0];
		max_chunk = std::max(max_chunk, S.chunk);
		k_iterations += 27 * S.chunks;
		const cuuint64_t vdims[4] = {static_cast<cuuint64_t>(c), static_cast<cuuint64_t>(W), static_cast<cuuint64_t>(H),
			static_cast<cuuint64_t>(D)};
		const cuuint64_t row = static_cast<cuuint64_t>(a->input_strides[i]) * 2;
		const cuuint64_t vstrides[3] = {row, row * W, row * W * H};
		const cuuint32_t vbox[4] = {static_cast<cuuint32_t>(S.chunk), static_cast<cuuint32_t>(p.wb),
			static_cast<cuuint32_t>(p.hb), static_cast<cuuint32_t>(p.db)};
		encode(&S.volume, a->inputs[i], 4, vdims, vstrides, vbox, S.chunk * 2);
		encode_weights(&S.weights, a, total_in, S.chunk);
	}
	p.k_iterations = k_iterations;
	p.taps = 27;
	const int a_bytes = 128 * max_chunk * 2;
	p.b_offset = a_bytes;
	p.stage_stride = (a_bytes + p.cout * max_chunk * 2 + 1023) / 1024 * 1024;
	p.stages = static_cast<int>(std::min<size_t>(conv_max_stages, conv_smem_budget / p.stage_stride));
	p.tmem_columns = tmem_columns_for(p.cout);
	p.o = output_of(a);
	const size_t smem = static_cast<size_t>(p.stages) * p.stage_stride + 1024;
	check_cuda(cudaFuncSetAttribute(conv3d_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)),
		"convolution attributes");
	const int grid = std::min(p.tiles, sm_count());
	conv3d_kernel<<<grid, conv_threads, smem, stream>>>(p);
	check_cuda(cudaGetLastError(), "convolution launch");
}

} // anonymous namespace
} // namespace rexlib_b200

namespace rexlib_b200
{

void conv3d_transposed2(const void *x, int cin, int D, int H, int W, const void *weights, const float *bias, int cout,
	void *out, int *error, cudaStream_t stream)
{
	require(cin == 16 || cin == 32 || (cin % 64 == 0 && cin <= 256), "the transposed convolution takes 16, 32 or a "
		"multiple of 64 input channels");
	require(cout % 16 == 0 && cout >= 16 && cout <= 256, "the transposed convolution takes 16 to 256 output channels, "
		"a multiple of 16");
	require(reinterpret_cast<uintptr_t>(x) % 16 == 0 && reinterpret_cast<uintptr_t>(weights) % 16 == 0 &&
			reinterpret_cast<uintptr_t>(out) % 16 == 0,
		"the transposed convolution's volumes and weights must be 16-byte aligned");
	// The 8 cout columns (sub-position, channel) in parts of at most 256:
	// whole sub-positions a part.
	const int per_part = std::max(1, 256 / cout); // sub-positions a part
	for (int sub0 = 0; sub0 < 8; sub0 += per_part)
	{
		const int subs = std::min(per_part, 8 - sub0);
		conv_params p{};
		p.sources = 1;
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
		p.cout = subs * cout;
		p.taps = 1;
		conv_source &S = p.source[0];
		S.chunk = std::min(cin, 64);
		S.chunks = cin / S.chunk;
		S.weight_channel = 0;
		p.k_iterations = S.chunks;
		const cuuint64_t vdims[4] = {static_cast<cuuint64_t>(cin), static_cast<cuuint64_t>(W), static_cast<cuuint64_t>(H),
			static_cast<cuuint64_t>(D)};
		const cuuint64_t row = static_cast<cuuint64_t>(cin) * 2;
		const cuuint64_t vstrides[3] = {row, row * W, row * W * H};
		const cuuint32_t vbox[4] = {static_cast<cuuint32_t>(S.chunk), static_cast<cuuint32_t>(p.wb),
			static_cast<cuuint32_t>(p.hb), static_cast<cuuint32_t>(p.db)};
		encode(&S.volume, x, 4, vdims, vstrides, vbox, S.chunk * 2);
		// This part's weights [s][o][i], s from sub0: (cin, 1 tap, its columns).
		const void *w = static_cast<const __nv_bfloat16 *>(weights) + static_cast<int64_t>(sub0) * cout * cin;
		const cuuint64_t wdims[3] = {static_cast<cuuint64_t>(cin), 1, static_cast<cuuint64_t>(p.cout)};
		const cuuint64_t wstrides[2] = {row, row};
		const cuuint32_t wbox[3] = {static_cast<cuuint32_t>(S.chunk), 1, static_cast<cuuint32_t>(p.cout)};
		encode(&S.weights, w, 3, wdims, wstrides, wbox, S.chunk * 2);
		const int a_bytes = 128 * S.chunk * 2;
		p.b_offset = a_bytes;
		p.stage_stride = (a_bytes + p.cout * S.chunk * 2 + 1023) / 1024 * 1024;
		p.stages = static_cast<int>(std::min<size_t>(conv_max_stages, conv_smem_budget / p.stage_stride));
		require(p.stages >= 2, "the transposed convolution's stages do not fit in shared memory");
		p.tmem_columns = tmem_columns_for(p.cout);
		p.o.cout = p.cout;
		p.o.epilogue = 0;
		p.o.bias = bias;
		p.o.out0 = static_cast<__nv_bfloat16 *>(out);
		p.o.split = p.cout;
		p.o.error = error;
		p.o.wait_ns = default_wait_ns;
		p.o.up_cout = cout;
		p.o.sub_base = sub0;
		const size_t smem = static_cast<size_t>(p.stages) * p.stage_stride + 1024;
		check_cuda(cudaFuncSetAttribute(conv3d_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)),
			"transposed convolution attributes");
		const int grid = std::min(p.tiles, sm_count());
		conv3d_kernel<<<grid, conv_threads, smem, stream>>>(p);
		check_cuda(cudaGetLastError(), "transposed convolution launch");
	}
}

} // namespace rexlib_b200

extern "C" int32_t rexlib_b200_conv3d(const rexlib_b200_conv3d_args *a, void *stream)
{
	return guarded([&] {
		require(a != nullptr, "null convolution arguments");
		require(a->sources == 1 || a->sources == 2, "a convolution reads one or two input volumes");
		require(a->depth >= 1 && a->height >= 1 && a->width >= 1, "volume extents must be positive");
		auto pow2 = [](int v) { return v > 0 && (v & (v - 1)) == 0; };
		if (!pow2(a->depth) || !pow2(a->height) || !pow2(a->width))
			fail(REXLIB_B200_UNSUPPORTED, "the convolution takes volume extents that are powers of two");
		if (a->output_channels < 16 || a->output_channels > 128 || a->output_channels % 16 != 0)
			fail(REXLIB_B200_UNSUPPORTED, "the convolution takes 16 to 128 output channels, a multiple of 16");
		int total_in = 0;
		for (int i = 0; i < a->sources; ++i)
		{
			const int c = a->input_channels[i];
			if (!(c == 16 || c == 32 || c % 64 == 0) || c > 256)
				fail(REXLIB_B200_UNSUPPORTED, "the convolution takes 16, 32 or a multiple of 64 input channels a source");
			require(a->inputs[i] != nullptr, "null input volume");
			require(a->input_strides[i] >= c && a->input_strides[i] % 8 == 0, "input rows must hold their channels, "
				"a multiple of 8");
			require(reinterpret_cast<uintptr_t>(a->inputs[i]) % 16 == 0, "input volumes must be 16-byte aligned");
			total_in += c;
		}
		require(a->weights != nullptr && reinterpret_cast<uintptr_t>(a->weights) % 16 == 0,
			"weights must be 16-byte aligned");
		// The x-row kernel (each input line read once for its three x taps)
		// in its wide form or, for widths that are multiples of 128, with
		// the x halo; boxes of 128 voxels otherwise.
		const bool rows = a->width % 128 == 0 || wide_halves(a) > 0;
		if (rows && std::getenv("REXLIB_B200_CONV_BOXES") == nullptr)
			launch_rows(a, total_in, as_stream(stream));
		else
			launch_boxes(a, total_in, as_stream(stream));
	});
}
