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

// First convolution: one FP32 input channel, 16 outputs with bias and ReLU.
__global__ void first_conv_kernel(volume_shape s, const float *__restrict__ x, const float *__restrict__ w,
	const float *__restrict__ bias, bf16 *__restrict__ out)
{
	__shared__ float sw[16 * 27];
	__shared__ float sb[16];
	for (int i = threadIdx.x; i < 16 * 27; i += blockDim.x)
		sw[i] = w[i];
	if (threadIdx.x < 16)
		sb[threadIdx.x] = bias[threadIdx.x];
	__syncthreads();
	for (int64_t v = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; v < s.voxels();
		 v += static_cast<int64_t>(gridDim.x) * blockDim.x)
	{
		float xin[27];
#pragma unroll
		for (int t = 0; t < 27; ++t)
		{
			const int64_t n = tap_neighbour(s, v, t);
			xin[t] = n >= 0 ? x[n] : 0.0f;
		}
		__align__(16) bf16 o[16];
#pragma unroll
		for (int c = 0; c < 16; ++c)
		{
			float acc = sb[c];
#pragma unroll
			for (int t = 0; t < 27; ++t)
				acc = fmaf(xin[t], sw[c * 27 + t], acc);
			o[c] = __float2bfloat16(fmaxf(acc, 0.0f));
		}
		uint4 *dst = reinterpret_cast<uint4 *>(out + v * 16);
		dst[0] = reinterpret_cast<const uint4 *>(o)[0];
		dst[1] = reinterpret_cast<const uint4 *>(o)[1];
	}
}

// Its weight gradient: dw[c][t] = sum_v g[v][c] x[v + t], db[c] = sum_v g[v][c].
// One block per voxel chunk; partial sums reduced in shared memory, then
// added to the FP32 gradient.
__global__ void first_conv_grad_kernel(volume_shape s, const float *__restrict__ x, const bf16 *__restrict__ g,
	float *__restrict__ dw, float *__restrict__ db)
{
	__shared__ float acc[16 * 28];
	for (int i = threadIdx.x; i < 16 * 28; i += blockDim.x)
		acc[i] = 0.0f;
	__syncthreads();
	float local[28];
	const int c = threadIdx.x & 15;
	for (int i = 0; i < 28; ++i)
		local[i] = 0.0f;
	for (int64_t v = (blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x) / 16; v < s.voxels();
		 v += static_cast<int64_t>(gridDim.x) * blockDim.x / 16)
	{
		const float gv = f(g[v * 16 + c]);
		if (gv == 0.0f)
			continue;
#pragma unroll
		for (int t = 0; t < 27; ++t)
		{
			const int64_t n = tap_neighbour(s, v, t);
			if (n >= 0)
				local[t] = fmaf(gv, x[n], local[t]);
		}
		local[27] += gv;
	}
	for (int i = 0; i < 28; ++i)
		atomicAdd(&acc[c * 28 + i], local[i]);
	__syncthreads();
	for (int i = threadIdx.x; i < 16 * 28; i += blockDim.x)
	{
		const int cc = i / 28, t = i % 28;
		if (t < 27)
			atomicAdd(dw + cc * 27 + t, acc[i]);
		else
			atomicAdd(db + cc, acc[i]);
	}
}

// Weight gradient of a 3x3x3 convolution: dw[o][t][i] = sum_v g[v][o] x[v + t][i]
// over the concatenated input channels (source a then source b), and
// db[o] = sum_v g[v][o] (tap 0's blocks only). Block = (range of voxels,
// tap), walked in chunks staged in shared memory; a thread owns an 8 x 8
// block of (o, i) (groups of threads split each chunk's voxels when the
// channels leave threads over) and adds its sums to the gradient once.
constexpr int grad_threads = 256;
constexpr int grad_chunk = 64;

__global__ void __launch_bounds__(grad_threads) conv_grad_kernel(volume_shape s, const bf16 *__restrict__ xa, int ca,
	int sa, const bf16 *__restrict__ xb, int cb, int sb, const bf16 *__restrict__ g, int cout, float *__restrict__ dw,
	float *__restrict__ db)
{
	extern __shared__ float smem[];
	const int cin = ca + cb;
	float *sg = smem;                    // grad_chunk x cout
	float *sx = sg + grad_chunk * cout;  // grad_chunk x cin
	const int tap = blockIdx.y;
	const int tiles_i = cin / 8;
	const int tiles = (cout / 8) * tiles_i;
	const int groups = grad_threads / tiles > 0 ? grad_threads / tiles : 1;
	const bool working = threadIdx.x < tiles * groups;
	const int tile = threadIdx.x % tiles, group = threadIdx.x / tiles;
	const int o0 = (tile / tiles_i) * 8, i0 = (tile % tiles_i) * 8;
	float acc[8][8] = {};
	float bias_acc[8] = {};
	const int64_t voxels = s.voxels();
	for (int64_t v0 = static_cast<int64_t>(blockIdx.x) * grad_chunk; v0 < voxels;
		 v0 += static_cast<int64_t>(gridDim.x) * grad_chunk)
	{
		__syncthreads(); // the previous chunk is consumed
		for (int i = threadIdx.x; i < grad_chunk * cout; i += blockDim.x)
		{
			const int64_t v = v0 + i / cout;
			sg[i] = v < voxels ? f(g[v * cout + i % cout]) : 0.0f;
		}
		for (int i = threadIdx.x; i < grad_chunk * cin; i += blockDim.x)
		{
			const int64_t v = v0 + i / cin;
			const int ch = i % cin;
			float value = 0.0f;
			if (v < voxels)
			{
				const int64_t n = tap_neighbour(s, v, tap);
				if (n >= 0)
					value = ch < ca ? f(xa[n * sa + ch]) : f(xb[n * sb + ch - ca]);
			}
			sx[i] = value;
		}
		__syncthreads();
		if (!working)
			continue;
		for (int v = group; v < grad_chunk; v += groups)
		{
			float go[8], xi[8];
#pragma unroll
			for (int a = 0; a < 8; ++a)
			{
				go[a] = sg[v * cout + o0 + a];
				xi[a] = sx[v * cin + i0 + a];
			}
#pragma unroll
			for (int a = 0; a < 8; ++a)
			{
				bias_acc[a] += go[a];
#pragma unroll
				for (int b = 0; b < 8; ++b)
					acc[a][b] = fmaf(go[a], xi[b], acc[a][b]);
			}
		}
	}
	if (!working)
		return;
#pragma unroll
	for (int a = 0; a < 8; ++a)
	{
#pragma unroll
		for (int b = 0; b < 8; ++b)
			atomicAdd(dw + (static_cast<int64_t>(o0 + a) * 27 + tap) * cin + i0 + b, acc[a][b]);
		if (tap == 0 && i0 == 0)
			atomicAdd(db + o0 + a, bias_acc[a]);
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

// 2x2x2 mean pooling of x (D, H, W, C) into out (D/2, H/2, W/2, C).
__global__ void pool_kernel(volume_shape s, int c, const bf16 *__restrict__ x, bf16 *__restrict__ out)
{
	const int64_t n = s.voxels() / 8 * c;
	const int ow = s.w / 2, oh = s.h / 2;
	for (int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; k < n;
		 k += static_cast<int64_t>(gridDim.x) * blockDim.x)
	{
		const int ch = static_cast<int>(k % c);
		const int64_t v = k / c;
		const int x0 = static_cast<int>(v % ow) * 2, y0 = static_cast<int>((v / ow) % oh) * 2, z0 = static_cast<int>(v / (static_cast<int64_t>(ow) * oh)) * 2;
		float sum = 0.0f;
#pragma unroll
		for (int i = 0; i < 8; ++i)
			sum += f(x[((static_cast<int64_t>(z0 + (i >> 2)) * s.h + y0 + ((i >> 1) & 1)) * s.w + x0 + (i & 1)) * c + ch]);
		out[k] = __float2bfloat16(0.125f * sum);
	}
}

// Gradient into a skip tensor that was also pooled: where the forward
// activation is positive, the skip gradient plus an eighth of the pooled
// volume's gradient at the parent voxel; 0 elsewhere (the ReLU's mask).
__global__ void skip_pool_grad_kernel(volume_shape s, int c, const bf16 *__restrict__ activation,
	const bf16 *__restrict__ skip_grad, const bf16 *__restrict__ pooled_grad, bf16 *__restrict__ out)
{
	const int64_t n = s.voxels() * c;
	const int ow = s.w / 2, oh = s.h / 2;
	for (int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; k < n;
		 k += static_cast<int64_t>(gridDim.x) * blockDim.x)
	{
		const int ch = static_cast<int>(k % c);
		const int64_t v = k / c;
		const int x = static_cast<int>(v % s.w), y = static_cast<int>((v / s.w) % s.h), z = static_cast<int>(v / (static_cast<int64_t>(s.w) * s.h));
		const int64_t parent = ((static_cast<int64_t>(z / 2) * oh + y / 2) * ow + x / 2) * c + ch;
		const float value = f(skip_grad[k]) + 0.125f * f(pooled_grad[parent]);
		out[k] = __float2bfloat16(f(activation[k]) > 0.0f ? value : 0.0f);
	}
}

// 2x2x2 stride-2 transposed convolution: out[2v + s][o] = b[o] + sum_i x[v][i] w[s][o][i]
// (sub-position s = (a * 2 + b) * 2 + c); out has extents 2 (D, H, W).
__global__ void up_kernel(volume_shape s, int cin, int cout, const bf16 *__restrict__ x, const float *__restrict__ w,
	const float *__restrict__ bias, bf16 *__restrict__ out)
{
	const float *__restrict__ sw = w; // 8 x cout x cin, read through the cache
	const int W2 = 2 * s.w, H2 = 2 * s.h;
	const int64_t n = s.voxels() * 8 * cout;
	for (int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; k < n;
		 k += static_cast<int64_t>(gridDim.x) * blockDim.x)
	{
		const int o = static_cast<int>(k % cout);
		const int64_t u = k / cout; // output voxel
		const int X = static_cast<int>(u % W2), Y = static_cast<int>((u / W2) % H2), Z = static_cast<int>(u / (static_cast<int64_t>(W2) * H2));
		const int sub = ((Z & 1) * 2 + (Y & 1)) * 2 + (X & 1);
		const int64_t v = (static_cast<int64_t>(Z >> 1) * s.h + (Y >> 1)) * s.w + (X >> 1);
		const float *wr = sw + (sub * cout + o) * cin;
		const bf16 *xr = x + v * cin;
		float acc = bias[o];
		for (int i = 0; i < cin; ++i)
			acc = fmaf(f(xr[i]), wr[i], acc);
		out[k] = __float2bfloat16(acc);
	}
}

// Its input gradient, masked by the forward input's ReLU:
// dx[v][i] = (x[v][i] > 0) sum_s sum_o g[2v + s][o] w[s][o][i].
__global__ void up_grad_input_kernel(volume_shape s, int cin, int cout, const bf16 *__restrict__ x,
	const float *__restrict__ w, const bf16 *__restrict__ g, bf16 *__restrict__ dx)
{
	const float *__restrict__ sw = w;
	const int W2 = 2 * s.w, H2 = 2 * s.h;
	const int64_t n = s.voxels() * cin;
	for (int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; k < n;
		 k += static_cast<int64_t>(gridDim.x) * blockDim.x)
	{
		const int i = static_cast<int>(k % cin);
		const int64_t v = k / cin;
		if (!(f(x[k]) > 0.0f))
		{
			dx[k] = __float2bfloat16(0.0f);
			continue;
		}
		const int xx = static_cast<int>(v % s.w), yy = static_cast<int>((v / s.w) % s.h), zz = static_cast<int>(v / (static_cast<int64_t>(s.w) * s.h));
		float acc = 0.0f;
		for (int sub = 0; sub < 8; ++sub)
		{
			const int64_t u = (static_cast<int64_t>(2 * zz + (sub >> 2)) * H2 + 2 * yy + ((sub >> 1) & 1)) * W2 + 2 * xx + (sub & 1);
			const bf16 *gr = g + u * cout;
			for (int o = 0; o < cout; ++o)
				acc = fmaf(f(gr[o]), sw[(sub * cout + o) * cin + i], acc);
		}
		dx[k] = __float2bfloat16(acc);
	}
}

// Its weight gradient: dw[s][o][i] = sum_v g[2v + s][o] x[v][i], db[o] = sum g[.][o].
// Block: a range of input voxels; a thread owns entries of (s, o, i) and
// adds its sum once.
__global__ void up_grad_weight_kernel(volume_shape s, int cin, int cout, const bf16 *__restrict__ x,
	const bf16 *__restrict__ g, float *__restrict__ dw, float *__restrict__ db)
{
	const int W2 = 2 * s.w, H2 = 2 * s.h;
	const int entries = 8 * cout * cin;
	const int64_t voxels = s.voxels();
	const int64_t per_block = (voxels + gridDim.x - 1) / gridDim.x;
	const int64_t v_begin = blockIdx.x * per_block, v_end = v_begin + per_block < voxels ? v_begin + per_block : voxels;
	for (int e = threadIdx.x; e < entries + cout; e += blockDim.x)
	{
		float acc = 0.0f;
		if (e < entries)
		{
			const int i = e % cin, o = (e / cin) % cout, sub = e / (cin * cout);
			for (int64_t v = v_begin; v < v_end; ++v)
			{
				const int xx = static_cast<int>(v % s.w), yy = static_cast<int>((v / s.w) % s.h), zz = static_cast<int>(v / (static_cast<int64_t>(s.w) * s.h));
				const int64_t u = (static_cast<int64_t>(2 * zz + (sub >> 2)) * H2 + 2 * yy + ((sub >> 1) & 1)) * W2 + 2 * xx + (sub & 1);
				acc = fmaf(f(g[u * cout + o]), f(x[v * cin + i]), acc);
			}
			atomicAdd(dw + e, acc);
		}
		else
		{
			const int o = e - entries;
			for (int64_t v = v_begin; v < v_end; ++v)
			{
				const int xx = static_cast<int>(v % s.w), yy = static_cast<int>((v / s.w) % s.h), zz = static_cast<int>(v / (static_cast<int64_t>(s.w) * s.h));
				for (int sub = 0; sub < 8; ++sub)
				{
					const int64_t u = (static_cast<int64_t>(2 * zz + (sub >> 2)) * H2 + 2 * yy + ((sub >> 1) & 1)) * W2 + 2 * xx + (sub & 1);
					acc += f(g[u * cout + o]);
				}
			}
			atomicAdd(db + o, acc);
		}
	}
}

// The 1x1x1 head and the residual: y[v] = x[v] + b + sum_i h[v][i] w[i].
__global__ void head_kernel(int64_t voxels, int c, const bf16 *__restrict__ h, const float *__restrict__ w,
	const float *__restrict__ bias, const float *__restrict__ x, float *__restrict__ y)
{
	for (int64_t v = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; v < voxels;
		 v += static_cast<int64_t>(gridDim.x) * blockDim.x)
	{
		float acc = bias[0];
		for (int i = 0; i < c; ++i)
			acc = fmaf(f(h[v * c + i]), w[i], acc);
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
