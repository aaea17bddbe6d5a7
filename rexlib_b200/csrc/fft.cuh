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
// unit or so in the last place. A lane builds them once into a plan and
// reuses it for every line it transforms.
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

// In-register DFT of length M with roots exp(sign 2 pi i t / M): radix-2
// butterflies for M = 2, 4, 8 and 16, the direct sum with precomputed roots
// for the other lengths.
template <int M>
struct small_dft
{
	float2 root[M > 8 || M == 1 || M == 2 || M == 4 || M == 8 || M == 16 ? 1 : M];

	__device__ __forceinline__ explicit small_dft(int sign)
	{
		if constexpr (!(M > 8 || M == 1 || M == 2 || M == 4 || M == 8 || M == 16))
		{
#pragma unroll
			for (int t = 0; t < M; ++t)
				root[t] = unit_root(t, M, sign);
		}
	}

	// x * (sign i)
	__device__ __forceinline__ static float2 rotate(float2 x, int sign)
	{
		return sign < 0 ? make_float2(x.y, -x.x) : make_float2(-x.y, x.x);
	}

	__device__ __forceinline__ static void dft4(float2 &v0, float2 &v1, float2 &v2, float2 &v3, int sign)
	{
		const float2 a = c_add(v0, v2), b = c_sub(v0, v2);
		const float2 c = c_add(v1, v3), d = rotate(c_sub(v1, v3), sign);
		v0 = c_add(a, c);
		v2 = c_sub(a, c);
		v1 = c_add(b, d);
		v3 = c_sub(b, d);
	}

	// The radix-2 DFT of 8 on its own, for the halves of a DFT of 16.
	__device__ __forceinline__ static void run8(float2 (&v)[8], int sign)
	{
		float2 e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
		float2 o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
		dft4(e0, e1, e2, e3, sign);
		dft4(o0, o1, o2, o3, sign);
		constexpr float h = 0.70710678118654752f;
		o1 = c_mul(o1, make_float2(h, sign * h));
		o2 = rotate(o2, sign);
		o3 = c_mul(o3, make_float2(-h, sign * h));
		v[0] = c_add(e0, o0);
		v[4] = c_sub(e0, o0);
		v[1] = c_add(e1, o1);
		v[5] = c_sub(e1, o1);
		v[2] = c_add(e2, o2);
		v[6] = c_sub(e2, o2);
		v[3] = c_add(e3, o3);
		v[7] = c_sub(e3, o3);
	}

	__device__ __forceinline__ void run(float2 (&v)[M], int sign) const
	{
		if constexpr (M == 1)
			return;
		else if constexpr (M == 2)
		{
			const float2 a = v[0];
			v[0] = c_add(a, v[1]);
			v[1] = c_sub(a, v[1]);
		}
		else if constexpr (M == 4)
			dft4(v[0], v[1], v[2], v[3], sign);
		else if constexpr (M == 16)
		{
			float2 e[8], o[8];
#pragma unroll
			for (int i = 0; i < 8; ++i)
			{
				e[i] = v[2 * i];
				o[i] = v[2 * i + 1];
			}
			small_dft<8>::run8(e, sign);
			small_dft<8>::run8(o, sign);
			// o_k * exp(sign 2 pi i k / 16), k = 1..7.
			constexpr float c1 = 0.92387953251128674f, s1 = 0.38268343236508977f, h = 0.70710678118654752f;
			o[1] = c_mul(o[1], make_float2(c1, sign * s1));
			o[2] = c_mul(o[2], make_float2(h, sign * h));
			o[3] = c_mul(o[3], make_float2(s1, sign * c1));
			o[4] = rotate(o[4], sign);
			o[5] = c_mul(o[5], make_float2(-s1, sign * c1));
			o[6] = c_mul(o[6], make_float2(-h, sign * h));
			o[7] = c_mul(o[7], make_float2(-c1, sign * s1));
#pragma unroll
			for (int k = 0; k < 8; ++k)
			{
				v[k] = c_add(e[k], o[k]);
				v[k + 8] = c_sub(e[k], o[k]);
			}
		}
		else if constexpr (M == 8)
			run8(v, sign);
		else
		{
			float2 y[M];
#pragma unroll
			for (int k1 = 0; k1 < M; ++k1)
			{
				float2 acc = v[0];
#pragma unroll
				for (int n1 = 1; n1 < M; ++n1)
				{
					float2 w;
					if constexpr (M > 8)
						w = unit_root((n1 * k1) % M, M, sign);
					else
						w = root[(n1 * k1) % M];
					acc = c_add(acc, c_mul(v[n1], w));
				}
				y[k1] = acc;
			}
#pragma unroll
			for (int k1 = 0; k1 < M; ++k1)
				v[k1] = y[k1];
		}
	}
};

template <int M, int W>
struct line_fft
{
	static constexpr int length = M * W;
	static constexpr int bits = log2_of<W>();

	// What a lane needs for every line it transforms, built once: the
	// four-step twiddles exp(sign 2 pi i j k1 / L) and the twiddle of each
	// cross-lane radix-2 stage.
	struct plan
	{
		int j;
		int sign;
		small_dft<M> dft;
		float2 twiddle[M];
		float2 stage[bits > 0 ? bits : 1];

		__device__ __forceinline__ plan(int lane, int s) : j(lane), sign(s), dft(s)
		{
#pragma unroll
			for (int k1 = 0; k1 < M; ++k1)
				twiddle[k1] = unit_root((j * k1) % length, length, sign);
			int t = 0;
#pragma unroll
			for (int st = W / 2; st >= 1; st >>= 1)
				stage[t++] = unit_root(j & (st - 1), 2 * st, sign);
		}
	};

	// v: the M values of this lane.
	__device__ __forceinline__ static void run(float2 (&v)[M], const plan &p)
	{
		if constexpr (M > 1)
		{
			p.dft.run(v, p.sign);
#pragma unroll
			for (int k1 = 1; k1 < M; ++k1)
				v[k1] = c_mul(v[k1], p.twiddle[k1]);
		}
		// Radix-2 DIF across the W lanes.
		int t = 0;
#pragma unroll
		for (int s = W / 2; s >= 1; s >>= 1)
		{
			const bool upper = (p.j & s) != 0;
			const float2 w = p.stage[t++];
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
