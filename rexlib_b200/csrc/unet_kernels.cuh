// The learned prior's kernels besides the tensor-core convolution: the
// first convolution (one input channel), the weight gradients of the 3x3x3
// convolutions, mean pooling, the 2x2x2 stride-2 transposed convolution,
// the 1x1x1 head with its residual, the loss and the Adam step. Volumes are
// channels-last BF16 (D, H, W, C); parameters and their gradients FP32.
#pragma once

#include "common.cuh"

#include <cuda_bf16.h>

namespace rexlib_b200
{
namespace unet
{

using bf16 = __nv_bfloat16;

__device__ __forceinline__ float f(bf16 v) { return __bfloat162float(v); }

struct volume_shape
{
	int d, h, w;
	__device__ __forceinline__ int64_t voxels() const { return static_cast<int64_t>(d) * h * w; }
};

// The voxel of linear index v shifted by tap t (-1, 0 or +1 per axis); -1
// when that falls outside the volume.
__device__ __forceinline__ int64_t tap_neighbour(const volume_shape &s, int64_t v, int t)
{
	const int x = static_cast<int>(v % s.w), y = static_cast<int>((v / s.w) % s.h), z = static_cast<int>(v / (static_cast<int64_t>(s.w) * s.h));
	const int zz = z + t / 9 - 1, yy = y + (t / 3) % 3 - 1, xx = x + t % 3 - 1;
	if (zz < 0 || zz >= s.d || yy < 0 || yy >= s.h || xx < 0 || xx >= s.w)
		return -1;
	return (static_cast<int64_t>(zz) * s.h + yy) * s.w + xx;
}

// The coordinates of linear voxel v (32-bit: volumes hold under 2^31 voxels).
__device__ __forceinline__ void voxel_xyz(const volume_shape &s, int v, int &x, int &y, int &z)
{
	x = v % s.w;
	y = (v / s.w) % s.h;
	z = v / (s.w * s.h);
}

// Eight BF16 values of one 16-byte load, as floats.
__device__ __forceinline__ void unpack8(const uint4 &q, float *out)
{
	const __nv_bfloat162 *h = reinterpret_cast<const __nv_bfloat162 *>(&q);
#pragma unroll
	for (int j = 0; j < 4; ++j)
	{
		const float2 t = __bfloat1622float2(h[j]);
		out[2 * j] = t.x;
		out[2 * j + 1] = t.y;
	}
}

__device__ __forceinline__ uint4 pack8(const float *v)
{
	uint4 q;
	__nv_bfloat162 *h = reinterpret_cast<__nv_bfloat162 *>(&q);
#pragma unroll
	for (int j = 0; j < 4; ++j)
		h[j] = __floats2bfloat162_rn(v[2 * j], v[2 * j + 1]);
	return q;
}

// First convolution: one FP32 input channel, 16 outputs with bias and ReLU.
// The weights sit in shared memory tap-major ([t][16]) so that a tap's 16
// weights are four broadcast 16-byte loads; a thread takes two voxels
// neighbouring in x (each weight load feeds both, and they share the input
// line's middle values), and each output sums its taps in order from the
// bias.
__global__ void __launch_bounds__(256) first_conv_kernel(volume_shape s, const float *__restrict__ x,
	const float *__restrict__ w, const float *__restrict__ bias, bf16 *__restrict__ out)
{
	__shared__ __align__(16) float sw[27 * 16];
	for (int i = threadIdx.x; i < 16 * 27; i += blockDim.x)
		sw[(i % 27) * 16 + i / 27] = w[i];
	float b[16];
#pragma unroll
	for (int c = 0; c < 16; ++c)
		b[c] = __ldg(bias + c);
	__syncthreads();
	const int pairs = static_cast<int>(s.voxels() / 2); // voxel pairs (2 p, 2 p + 1): W is even
	for (int pair = blockIdx.x * blockDim.x + threadIdx.x; pair < pairs; pair += gridDim.x * blockDim.x)
	{
		const int v = 2 * pair;
		int x0, y0, z0;
		voxel_xyz(s, v, x0, y0, z0);
		float acc[2][16];
#pragma unroll
		for (int c = 0; c < 16; ++c)
			acc[0][c] = acc[1][c] = b[c];
#pragma unroll
		for (int dz = 0; dz < 3; ++dz)
#pragma unroll
			for (int dy = 0; dy < 3; ++dy)
			{
				const int zz = z0 + dz - 1, yy = y0 + dy - 1;
				const bool row_inside = zz >= 0 && zz < s.d && yy >= 0 && yy < s.h;
				// The line's values at x0 - 1 .. x0 + 2 (zeros outside).
				float line[4];
#pragma unroll
				for (int j = 0; j < 4; ++j)
				{
					const int xx = x0 - 1 + j;
					line[j] = row_inside && xx >= 0 && xx < s.w ? __ldg(x + (zz * s.h + yy) * s.w + xx) : 0.0f;
				}
#pragma unroll
				for (int dx = 0; dx < 3; ++dx)
				{
					const float4 *wt = reinterpret_cast<const float4 *>(sw + (dz * 9 + dy * 3 + dx) * 16);
#pragma unroll
					for (int q = 0; q < 4; ++q)
					{
						const float4 ww = wt[q];
#pragma unroll
						for (int e = 0; e < 2; ++e)
						{
							const float xin = line[dx + e];
							acc[e][4 * q] = fmaf(xin, ww.x, acc[e][4 * q]);
							acc[e][4 * q + 1] = fmaf(xin, ww.y, acc[e][4 * q + 1]);
							acc[e][4 * q + 2] = fmaf(xin, ww.z, acc[e][4 * q + 2]);
							acc[e][4 * q + 3] = fmaf(xin, ww.w, acc[e][4 * q + 3]);
						}
					}
				}
			}
#pragma unroll
		for (int e = 0; e < 2; ++e)
		{
#pragma unroll
			for (int c = 0; c < 16; ++c)
				acc[e][c] = fmaxf(acc[e][c], 0.0f);
			uint4 *dst = reinterpret_cast<uint4 *>(out + static_cast<int64_t>(v + e) * 16);
			dst[0] = pack8(acc[e]);
			dst[1] = pack8(acc[e] + 8);
		}
	}
}

// Its weight gradient: dw[c][t] = sum_v g[v][c] x[v + t], db[c] = sum_v g[v][c].
// A warp takes 32 consecutive voxels at a time and four output channels
// (warp % 4): each lane reads its voxel's 27 neighbours of x (the warp's
// reads are consecutive floats) and its four g values, and keeps the 27 x 4
// sums in registers. At the end the warp's sums are reduced by shuffles and
// added to the gradient once. Launch: first_grad_threads threads, a grid of
// a few blocks an SM.
constexpr int first_grad_threads = 256;

__global__ void __launch_bounds__(first_grad_threads) first_conv_grad_kernel(volume_shape s,
	const float *__restrict__ x, const bf16 *__restrict__ g, float *__restrict__ dw, float *__restrict__ db)
{
	constexpr int voxel_warps = first_grad_threads / 128; // warps of one channel group in a block
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	const int cg = warp & 3;
	float acc[27][4] = {};
	float bias[4] = {};
	const int64_t voxels = s.voxels();
	const int hw = s.h * s.w;
	const int64_t step = static_cast<int64_t>(gridDim.x) * voxel_warps * 32;
	for (int64_t v = (static_cast<int64_t>(blockIdx.x) * voxel_warps + (warp >> 2)) * 32 + lane; v < voxels; v += step)
	{
		const int vi = static_cast<int>(v); // volumes hold under 2^31 voxels
		const int x0 = vi % s.w, y0 = (vi / s.w) % s.h, z0 = vi / hw;
		const uint2 q = __ldg(reinterpret_cast<const uint2 *>(g + v * 16 + cg * 4));
		const float2 g01 = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(&q.x));
		const float2 g23 = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(&q.y));
		const float gv[4] = {g01.x, g01.y, g23.x, g23.y};
#pragma unroll
		for (int c = 0; c < 4; ++c)
			bias[c] += gv[c];
#pragma unroll
		for (int dz = 0; dz < 3; ++dz)
		{
			const int z = z0 + dz - 1;
#pragma unroll
			for (int dy = 0; dy < 3; ++dy)
			{
				const int y = y0 + dy - 1;
				const bool inside = z >= 0 && z < s.d && y >= 0 && y < s.h;
				const float *row = x + (static_cast<int64_t>(z) * s.h + y) * s.w;
#pragma unroll
				for (int dx = 0; dx < 3; ++dx)
				{
					const int xx = x0 + dx - 1;
					const float xv = inside && xx >= 0 && xx < s.w ? __ldg(row + xx) : 0.0f;
#pragma unroll
					for (int c = 0; c < 4; ++c)
						acc[dz * 9 + dy * 3 + dx][c] = fmaf(gv[c], xv, acc[dz * 9 + dy * 3 + dx][c]);
				}
			}
		}
	}
#pragma unroll
	for (int t = 0; t < 28; ++t)
#pragma unroll
		for (int c = 0; c < 4; ++c)
		{
			float value = t < 27 ? acc[t][c] : bias[c];
#pragma unroll
			for (int offset = 16; offset > 0; offset >>= 1)
				value += __shfl_xor_sync(0xffffffffu, value, offset);
			if (lane == 0)
				atomicAdd(t < 27 ? dw + (cg * 4 + c) * 27 + t : db + cg * 4 + c, value);
		}
}

// Weight gradients as GEMMs over voxels on the CUDA cores:
// - a 3x3x3 convolution (UP false; ROWS = cout):
//     dw[o][n] += sum_v g[v][o] col[v][n],  col[v][t cin + i] = x[v + t][i],
//     db[o] += sum_v g[v][o],
//   x the concatenated sources (zero outside the volume);
// - a 2x2x2 stride-2 transposed convolution (UP true; ROWS = 8 cout, rows
//   (s, o) for the sub-positions s = 4 sz + 2 sy + sx), over the voxels v of
//   its input x (shape `s`):
//     dw[s][o][i] += sum_v g[2 v + s][o] x[v][i],  db[o] += sum_v,s g[2 v + s][o].
// A block takes a range of voxels, 64 at a time, and `cols` of the columns
// n (blockIdx.y selects them); it stages the chunk's rows and columns as
// FP32 in shared memory, and each thread accumulates a 4 x 4 tile of (row,
// n) sums in registers: two 16-byte shared loads feed 16 FMAs. The next
// chunk's 16-byte global loads are issued before the current chunk's sums,
// so their latency hides under the arithmetic. The tiles are added to the
// gradient once, at the end.
constexpr int wgrad_threads = 256;
constexpr int wgrad_chunk = 64;

template <int ROWS, bool UP = false>
__global__ void __launch_bounds__(wgrad_threads) wgrad_kernel(volume_shape s, const bf16 *__restrict__ xa, int ca,
	int sa, const bf16 *__restrict__ xb, int cb, int sb, const bf16 *__restrict__ g, float *__restrict__ dw,
	float *__restrict__ db, int64_t voxels_per_block)
{
	constexpr int cols = 4 * wgrad_threads / (ROWS / 4); // columns a block covers: (ROWS / 4) x (cols / 4) threads
	constexpr int g_items = (wgrad_chunk * (ROWS / 8) + wgrad_threads - 1) / wgrad_threads; // 16-byte loads a thread
	constexpr int c_items = (wgrad_chunk * (cols / 8) + wgrad_threads - 1) / wgrad_threads;
	constexpr int cout = UP ? ROWS / 8 : ROWS; // channels of a g voxel
	extern __shared__ float4 wgrad_smem[];
	float *sg = reinterpret_cast<float *>(wgrad_smem); // chunk x ROWS
	float *scol = sg + wgrad_chunk * ROWS;              // chunk x cols
	const int cin = ca + cb;
	const int ncols = UP ? cin : 27 * cin;
	const int n_first = blockIdx.y * cols;
	const int og = threadIdx.x % (ROWS / 4), ng = threadIdx.x / (ROWS / 4);
	const int o0 = og * 4, n0 = ng * 4;
	const bool active = n_first + n0 < ncols;
	const bool bias_thread = blockIdx.y == 0 && ng == 0;
	float acc[4][4] = {};
	float bias_acc[4] = {};
	const int64_t voxels = s.voxels();
	const int64_t v_begin = static_cast<int64_t>(blockIdx.x) * voxels_per_block;
	const int64_t v_end = min(voxels, v_begin + voxels_per_block);
	const int hw = s.h * s.w;
	uint4 pg[g_items], pc[c_items];

	// The 16-byte loads of the chunk at v0 into registers (zeros outside).
	auto fetch = [&](int64_t v0) {
#pragma unroll
		for (int j = 0; j < g_items; ++j)
		{
			const int k = threadIdx.x + j * wgrad_threads;
			pg[j] = make_uint4(0, 0, 0, 0);
			if (k < wgrad_chunk * (ROWS / 8))
			{
				const int local = k / (ROWS / 8), part = k % (ROWS / 8);
				const int64_t v = v0 + local;
				if (v < v_end)
				{
					int64_t u = v;
					int piece = part;
					if constexpr (UP)
					{
						// Row piece `part`: sub-position part / (cout / 8), channels
						// 8 (part % (cout / 8)) on, of fine voxel 2 v + s.
						const int sub = part / (cout / 8);
						piece = part % (cout / 8);
						const int vi = static_cast<int>(v);
						const int x = vi % s.w, y = (vi / s.w) % s.h, z = vi / hw;
						u = (static_cast<int64_t>(2 * z + (sub >> 2)) * (2 * s.h) + 2 * y + ((sub >> 1) & 1)) * (2 * s.w) +
							2 * x + (sub & 1);
					}
					pg[j] = __ldg(reinterpret_cast<const uint4 *>(g + u * cout) + piece);
				}
			}
		}
#pragma unroll
		for (int j = 0; j < c_items; ++j)
		{
			const int k = threadIdx.x + j * wgrad_threads;
			pc[j] = make_uint4(0, 0, 0, 0);
			if (k >= wgrad_chunk * (cols / 8))
				continue;
			const int local = k / (cols / 8), part = k % (cols / 8);
			const int n = n_first + part * 8;
			const int64_t v = v0 + local;
			if (v < v_end && n < ncols)
			{
				if constexpr (UP)
					pc[j] = __ldg(reinterpret_cast<const uint4 *>(xa + v * sa + n));
				else
				{
					const int t = n / cin, i = n - t * cin;
					const int vi = static_cast<int>(v); // volumes hold under 2^31 voxels
					const int x = vi % s.w + t % 3 - 1, y = (vi / s.w) % s.h + (t / 3) % 3 - 1, z = vi / hw + t / 9 - 1;
					if (x >= 0 && x < s.w && y >= 0 && y < s.h && z >= 0 && z < s.d)
					{
						const int64_t u = (static_cast<int64_t>(z) * s.h + y) * s.w + x;
						const bf16 *src = i < ca ? xa + u * sa + i : xb + u * sb + (i - ca);
						pc[j] = __ldg(reinterpret_cast<const uint4 *>(src));
					}
				}
			}
		}
	};
	auto store = [&]() {
#pragma unroll
		for (int j = 0; j < g_items; ++j)
		{
			const int k = threadIdx.x + j * wgrad_threads;
			if (k < wgrad_chunk * (ROWS / 8))
			{
				float vals[8];
				unpack8(pg[j], vals);
				float4 *dst = reinterpret_cast<float4 *>(sg + (k / (ROWS / 8)) * ROWS + (k % (ROWS / 8)) * 8);
				dst[0] = make_float4(vals[0], vals[1], vals[2], vals[3]);
				dst[1] = make_float4(vals[4], vals[5], vals[6], vals[7]);
			}
		}
#pragma unroll
		for (int j = 0; j < c_items; ++j)
		{
			const int k = threadIdx.x + j * wgrad_threads;
			if (k < wgrad_chunk * (cols / 8))
			{
				float vals[8];
				unpack8(pc[j], vals);
				float4 *dst = reinterpret_cast<float4 *>(scol + (k / (cols / 8)) * cols + (k % (cols / 8)) * 8);
				dst[0] = make_float4(vals[0], vals[1], vals[2], vals[3]);
				dst[1] = make_float4(vals[4], vals[5], vals[6], vals[7]);
			}
		}
	};

	if (v_begin < v_end)
		fetch(v_begin);
	for (int64_t v0 = v_begin; v0 < v_end; v0 += wgrad_chunk)
	{
		__syncthreads(); // the previous chunk is consumed
		store();
		__syncthreads();
		if (v0 + wgrad_chunk < v_end)
			fetch(v0 + wgrad_chunk); // in flight during the sums below
		if (!active)
			continue;
#pragma unroll 4
		for (int v = 0; v < wgrad_chunk; ++v)
		{
			const float4 a = *reinterpret_cast<const float4 *>(sg + v * ROWS + o0);
			const float4 b = *reinterpret_cast<const float4 *>(scol + v * cols + n0);
			const float av[4] = {a.x, a.y, a.z, a.w};
			const float bv[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
			for (int r = 0; r < 4; ++r)
#pragma unroll
				for (int c = 0; c < 4; ++c)
					acc[r][c] = fmaf(av[r], bv[c], acc[r][c]);
			if (bias_thread)
#pragma unroll
				for (int r = 0; r < 4; ++r)
					bias_acc[r] += av[r];
		}
	}
	if (active)
	{
		const int n = n_first + n0;
#pragma unroll
		for (int r = 0; r < 4; ++r)
#pragma unroll
			for (int c = 0; c < 4; ++c)
				if (n + c < ncols)
					atomicAdd(dw + static_cast<int64_t>(o0 + r) * ncols + n + c, acc[r][c]);
		if (bias_thread)
#pragma unroll
			for (int r = 0; r < 4; ++r)
				atomicAdd(db + (o0 + r) % cout, bias_acc[r]);
	}
}

// The flipped, transposed weights of the backward-data convolution:
// wt[i][26 - t][o] = w[o][t][i] (BF16 from the FP32 master copy).
__global__ void flip_weights_kernel(const float *__restrict__ w, int cout, int cin, bf16 *__restrict__ wt)
{
	const int64_t n = static_cast<int64_t>(cout) * 27 * cin;
	for (int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; k < n;
		 k += static_cast<int64_t>(gridDim.x) * blockDim.x)
	{
		const int i = static_cast<int>(k % cin), t = static_cast<int>((k / cin) % 27), o = static_cast<int>(k / (27 * cin));
		wt[(static_cast<int64_t>(i) * 27 + (26 - t)) * cout + o] = __float2bfloat16(w[k]);
	}
}

// 2x2x2 mean pooling of x (D, H, W, C) into out (D/2, H/2, W/2, C): a
// thread takes 8 channels of one output voxel (16-byte loads), summing the
// eight children in order.
__global__ void __launch_bounds__(256) pool_kernel(volume_shape s, int c, const bf16 *__restrict__ x,
	bf16 *__restrict__ out)
{
	const int groups = c / 8;
	const int n = static_cast<int>(s.voxels() / 8) * groups;
	const int ow = s.w / 2, oh = s.h / 2;
	for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
	{
		const int g = k % groups, v = k / groups;
		const int x0 = (v % ow) * 2, y0 = ((v / ow) % oh) * 2, z0 = v / (ow * oh) * 2;
		float sum[8] = {};
#pragma unroll
		for (int i = 0; i < 8; ++i)
		{
			const int64_t child = (static_cast<int64_t>(z0 + (i >> 2)) * s.h + y0 + ((i >> 1) & 1)) * s.w + x0 + (i & 1);
			float t[8];
			unpack8(__ldg(reinterpret_cast<const uint4 *>(x + child * c) + g), t);
#pragma unroll
			for (int j = 0; j < 8; ++j)
				sum[j] += t[j];
		}
#pragma unroll
		for (int j = 0; j < 8; ++j)
			sum[j] *= 0.125f;
		reinterpret_cast<uint4 *>(out + static_cast<int64_t>(v) * c)[g] = pack8(sum);
	}
}

// Gradient into a skip tensor that was also pooled: where the forward
// activation is positive, the skip gradient plus an eighth of the pooled
// volume's gradient at the parent voxel; 0 elsewhere (the ReLU's mask).
// Eight channels a thread.
__global__ void __launch_bounds__(256) skip_pool_grad_kernel(volume_shape s, int c, const bf16 *__restrict__ activation,
	const bf16 *__restrict__ skip_grad, const bf16 *__restrict__ pooled_grad, bf16 *__restrict__ out)
{
	const int groups = c / 8;
	const int n = static_cast<int>(s.voxels()) * groups;
	const int ow = s.w / 2, oh = s.h / 2;
	for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
	{
		const int g = k % groups, v = k / groups;
		int x, y, z;
		voxel_xyz(s, v, x, y, z);
		const int64_t parent = (static_cast<int64_t>(z / 2) * oh + y / 2) * ow + x / 2;
		float a[8], sg[8], pg[8], r[8];
		unpack8(__ldg(reinterpret_cast<const uint4 *>(activation) + k), a);
		unpack8(__ldg(reinterpret_cast<const uint4 *>(skip_grad) + k), sg);
		unpack8(__ldg(reinterpret_cast<const uint4 *>(pooled_grad + parent * c) + g), pg);
#pragma unroll
		for (int j = 0; j < 8; ++j)
			r[j] = a[j] > 0.0f ? sg[j] + 0.125f * pg[j] : 0.0f;
		reinterpret_cast<uint4 *>(out)[k] = pack8(r);
	}
}

// The 2x2x2 stride-2 transposed convolution's input gradient (its forward
// runs on the tensor cores, conv3d.cuh), masked by the forward input's ReLU:
// dx[v][i] = (x[v][i] > 0) sum_s sum_o g[2v + s][o] w[s][o][i].
// Block (voxel range, 16 input channels): the weights of those channels sit
// in shared memory as [s][o][16]; a thread takes one voxel and sums over s
// then o in order, the output gradient read 8 channels at a time.
__global__ void __launch_bounds__(256) up_grad_input_kernel(volume_shape s, int cin, int cout,
	const bf16 *__restrict__ x, const float *__restrict__ w, const bf16 *__restrict__ g, bf16 *__restrict__ dx)
{
	extern __shared__ float4 up_smem[];
	float *sw = reinterpret_cast<float *>(up_smem); // 8 x cout x 16
	const int i0 = blockIdx.y * 16;
	for (int k = threadIdx.x; k < 8 * cout * 16; k += blockDim.x)
		sw[k] = w[static_cast<int64_t>(k / 16) * cin + i0 + k % 16];
	__syncthreads();
	const int W2 = 2 * s.w, H2 = 2 * s.h;
	const int voxels = static_cast<int>(s.voxels());
	for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < voxels; v += gridDim.x * blockDim.x)
	{
		int xx, yy, zz;
		voxel_xyz(s, v, xx, yy, zz);
		float acc[16] = {};
		for (int sub = 0; sub < 8; ++sub)
		{
			const int64_t u = (static_cast<int64_t>(2 * zz + (sub >> 2)) * H2 + 2 * yy + ((sub >> 1) & 1)) * W2 + 2 * xx + (sub & 1);
			const uint4 *gr = reinterpret_cast<const uint4 *>(g + u * cout);
			for (int o0 = 0; o0 < cout; o0 += 8)
			{
				float go[8];
				unpack8(__ldg(gr + o0 / 8), go);
#pragma unroll
				for (int j = 0; j < 8; ++j)
				{
					const float4 *wr = reinterpret_cast<const float4 *>(sw + (sub * cout + o0 + j) * 16);
#pragma unroll
					for (int q = 0; q < 4; ++q)
					{
						const float4 ww = wr[q];
						acc[4 * q] = fmaf(go[j], ww.x, acc[4 * q]);
						acc[4 * q + 1] = fmaf(go[j], ww.y, acc[4 * q + 1]);
						acc[4 * q + 2] = fmaf(go[j], ww.z, acc[4 * q + 2]);
						acc[4 * q + 3] = fmaf(go[j], ww.w, acc[4 * q + 3]);
					}
				}
			}
		}
		const uint4 *xm = reinterpret_cast<const uint4 *>(x + static_cast<int64_t>(v) * cin + i0);
		float m[8];
		unpack8(__ldg(xm), m);
#pragma unroll
		for (int j = 0; j < 8; ++j)
			acc[j] = m[j] > 0.0f ? acc[j] : 0.0f;
		unpack8(__ldg(xm + 1), m);
#pragma unroll
		for (int j = 0; j < 8; ++j)
			acc[8 + j] = m[j] > 0.0f ? acc[8 + j] : 0.0f;
		uint4 *dst = reinterpret_cast<uint4 *>(dx + static_cast<int64_t>(v) * cin + i0);
		dst[0] = pack8(acc);
		dst[1] = pack8(acc + 8);
	}
}

// The 1x1x1 head and the residual: y[v] = x[v] + b + sum_i h[v][i] w[i]
// (16 channels, two 16-byte loads a voxel).
__global__ void __launch_bounds__(256) head_kernel(int64_t voxels, int c, const bf16 *__restrict__ h,
	const float *__restrict__ w, const float *__restrict__ bias, const float *__restrict__ x, float *__restrict__ y)
{
	float wr[16];
#pragma unroll
	for (int i = 0; i < 16; ++i)
		wr[i] = __ldg(w + i);
	const float b = __ldg(bias);
	for (int64_t v = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; v < voxels;
		 v += static_cast<int64_t>(gridDim.x) * blockDim.x)
	{
		float hv[16];
		const uint4 *hr = reinterpret_cast<const uint4 *>(h + v * 16);
		unpack8(__ldg(hr), hv);
		unpack8(__ldg(hr + 1), hv + 8);
		float acc = b;
#pragma unroll
		for (int i = 0; i < 16; ++i)
			acc = fmaf(hv[i], wr[i], acc);
		y[v] = x[v] + acc;
	}
}

// The loss 0.5 mean (y - t)^2 (added to *loss), its gradient g = (y - t) / V
// through the head: dh[v][i] = (h > 0) g w[i]; dw[i] += sum g h[v][i],
// db += sum g.
__global__ void head_loss_grad_kernel(int64_t voxels, int c, const bf16 *__restrict__ h, const float *__restrict__ w,
	const float *__restrict__ y, const float *__restrict__ target, bf16 *__restrict__ dh, float *__restrict__ dw,
	float *__restrict__ db, float *__restrict__ loss)
{
	__shared__ float part[32][18];
	float lw[16] = {};
	float lb = 0.0f, ll = 0.0f;
	const float inv = 1.0f / static_cast<float>(voxels);
	for (int64_t v = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; v < voxels;
		 v += static_cast<int64_t>(gridDim.x) * blockDim.x)
	{
		const float d = y[v] - target[v];
		ll += 0.5f * d * d * inv;
		const float g = d * inv;
		lb += g;
		for (int i = 0; i < c; ++i)
		{
			const float hv = f(h[v * c + i]);
			lw[i] = fmaf(g, hv, lw[i]);
			dh[v * c + i] = __float2bfloat16(hv > 0.0f ? g * w[i] : 0.0f);
		}
	}
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	for (int o = 16; o > 0; o >>= 1)
	{
		ll += __shfl_xor_sync(0xffffffffu, ll, o);
		lb += __shfl_xor_sync(0xffffffffu, lb, o);
		for (int i = 0; i < 16; ++i)
			lw[i] += __shfl_xor_sync(0xffffffffu, lw[i], o);
	}
	if (lane == 0)
	{
		for (int i = 0; i < 16; ++i)
			part[warp][i] = lw[i];
		part[warp][16] = lb;
		part[warp][17] = ll;
	}
	__syncthreads();
	if (threadIdx.x < 18)
	{
		float sum = 0.0f;
		for (int k = 0; k < static_cast<int>(blockDim.x >> 5); ++k)
			sum += part[k][threadIdx.x];
		if (threadIdx.x < c)
			atomicAdd(dw + threadIdx.x, sum);
		else if (threadIdx.x == 16)
			atomicAdd(db, sum);
		else if (threadIdx.x == 17)
			atomicAdd(loss, sum);
	}
}

// Adam (beta1 0.9, beta2 0.999, eps 1e-8) on the FP32 master parameters,
// then their BF16 copies for the tensor-core convolutions (where given);
// the gradients are cleared for the next step.
__global__ void adam_kernel(int64_t n, float *__restrict__ p, float *__restrict__ grad, float *__restrict__ m,
	float *__restrict__ v, float lr, float bias1, float bias2)
{
	for (int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; k < n;
		 k += static_cast<int64_t>(gridDim.x) * blockDim.x)
	{
		const float g = grad[k];
		const float mk = 0.9f * m[k] + 0.1f * g;
		const float vk = 0.999f * v[k] + 0.001f * g * g;
		m[k] = mk;
		v[k] = vk;
		p[k] -= lr * (mk / bias1) / (sqrtf(vk / bias2) + 1e-8f);
		grad[k] = 0.0f;
	}
}

__global__ void to_bf16_kernel(int64_t n, const float *__restrict__ x, bf16 *__restrict__ y)
{
	for (int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; k < n;
		 k += static_cast<int64_t>(gridDim.x) * blockDim.x)
		y[k] = __float2bfloat16(x[k]);
}

} // namespace unet
} // namespace rexlib_b200
