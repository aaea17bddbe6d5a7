// Complex FFT of one line held in registers by a group of lanes.
//
// A line of length L = M * W is spread over W consecutive lanes (W a power
// of two up to 32); lane j holds the M elements x[W * n1 + j], n1 < M. The
// transform is the four-step decomposition L = M x W: a length-M DFT in each
// lane's registers over n1, the twiddles exp(s 2 pi i j k1 / L), then a
// radix-2 decimation-in-frequency FFT of length W across the lanes (shuffles)
// for every k1. Afterwards lane j holds X[k1 + M * bitrev(j)] in register k1.
// s = -1 is the forward (unnormalised) transform, s = +1 the inverse.
//
// Twiddles come from sincospif of exact rationals, so each is correct to a
// unit or so in the last place; no table lives in memory.
#pragma once

#include <cuda_runtime.h>

namespace rexlib_b200
{

__device__ __forceinline__ float2 c_add(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 c_sub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 c_mul(float2 a, float2 b)
{
	return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 c_conj(float2 a) { return make_float2(a.x, -a.y); }

// exp(sign * 2 pi i * num / den) for integers with 0 <= num < den.
__device__ __forceinline__ float2 unit_root(int num, int den, int sign)
{
	float s, c;
	sincospif(2.0f * static_cast<float>(num) / static_cast<float>(den), &s, &c);
	return make_float2(c, sign < 0 ? -s : s);
}

__device__ __forceinline__ int bit_reverse(int v, int bits) { return static_cast<int>(__brev(static_cast<unsigned>(v)) >> (32 - bits)); }

template <int W>
constexpr int log2_of()
{
	return W == 1 ? 0 : 1 + log2_of<W / 2>();
}

template <int M, int W>
struct line_fft
{
	static constexpr int length = M * W;
	static constexpr int bits = log2_of<W>();

	// v: the M values of this lane; j: the lane's index within its group.
	__device__ __forceinline__ static void run(float2 (&v)[M], int j, int sign)
	{
		// Length-M DFT over n1 in registers.
		if constexpr (M > 1)
		{
			float2 root[M];
#pragma unroll
			for (int t = 0; t < M; ++t)
				root[t] = unit_root(t, M, sign);
			float2 y[M];
#pragma unroll
			for (int k1 = 0; k1 < M; ++k1)
			{
				float2 acc = v[0];
#pragma unroll
				for (int n1 = 1; n1 < M; ++n1)
				{
					const float2 t = c_mul(v[n1], root[(n1 * k1) % M]);
					acc = c_add(acc, t);
				}
				y[k1] = acc;
			}
			// Twiddles exp(sign 2 pi i j k1 / L).
#pragma unroll
			for (int k1 = 0; k1 < M; ++k1)
				v[k1] = k1 == 0 ? y[0] : c_mul(y[k1], unit_root((j * k1) % length, length, sign));
		}
		// Radix-2 DIF across the W lanes.
#pragma unroll
		for (int s = W / 2; s >= 1; s >>= 1)
		{
			const bool upper = (j & s) != 0;
			const float2 w = unit_root(j & (s - 1), 2 * s, sign);
#pragma unroll
			for (int k1 = 0; k1 < M; ++k1)
			{
				const float2 own = v[k1];
				float2 other;
				other.x = __shfl_xor_sync(0xffffffffu, own.x, s, W);
				other.y = __shfl_xor_sync(0xffffffffu, own.y, s, W);
				v[k1] = upper ? c_mul(c_sub(other, own), w) : c_add(own, other);
			}
		}
	}

	// The output index held by lane j in register k1.
	__device__ __forceinline__ static int output_index(int k1, int j)
	{
		if constexpr (bits == 0)
			return k1;
		else
			return k1 + M * bit_reverse(j, bits);
	}
};

} // namespace rexlib_b200
