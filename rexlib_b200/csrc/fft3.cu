// 3D C2R of a half spectrum (N, N, N/2+1) into a volume (N, N, N), with the
// Wiener divide of an insertion's accumulators fused into its first pass.
//
// irfft3 (include/rexlib/ops/fourier/irfft_operation.hpp; the CPU runs
// pocketfft's c2r, src/backends/cpu/kernels/pocketfft_fourier_transform.cpp:152)
// with the backward normalisation (1/N^3), in three passes over HBM:
//  1. inverse complex lines along z, one CTA per (y, block of 32 x): the
//     tile (N z) x (32 x) is read with coalesced rows, transformed in shared
//     memory and written to the workspace; the Wiener variant reads the
//     numerator and denominator here and divides on the way in;
//  2. inverse complex lines along y, likewise, in place in the workspace;
//  3. the C2R along x, one complex line of N/2 per (z, y) row, written as
//     the N reals of the row.
// The divide (no rexlib operation; the reference test divides, then calls
// irfft3, test_cpu_reconstruction.cpp:457-470): REGULARIZED X = N / (D + c),
// THRESHOLD X = N / D where D > c, else 0.
#include "common.cuh"
#include "fft.cuh"

#include <algorithm>
#include <cmath>
#include <string>

namespace rexlib_b200
{
namespace
{

constexpr int volume_threads = 256;
constexpr int x_block = 32;

struct volume_launch
{
	const float2 *in;       // spectrum (z pass of irfft3)
	const float2 *numerator; // Wiener inputs (z pass)
	const float *denominator;
	float2 *work;            // (N, N, H) intermediate
	float *out;              // (N, N, N)
	int big, H;
	int wiener_mode;         // -1: plain irfft3
	float constant;
};

// Pass 1 and 2: lines along z (axis 0) or y (axis 1) of the (N, N, H) array.
template <int M, int W, int AXIS>
__global__ void __launch_bounds__(volume_threads) volume_lines_kernel(const volume_launch P)
{
	extern __shared__ float2 tile[]; // N x x_block
	const int big = P.big, H = P.H;
	const int fixed = blockIdx.y; // y for the z pass, z for the y pass
	const int x0 = blockIdx.x * x_block;
	const int xw = min(x_block, H - x0);
	// Element (line index l, x) of the tile lives at l * x_block + x.
	auto global_offset = [&](int l, int x) -> int64_t {
		return AXIS == 0 ? ((int64_t)l * big + fixed) * H + x0 + x : ((int64_t)fixed * big + l) * H + x0 + x;
	};
	for (int i = threadIdx.x; i < big * x_block; i += blockDim.x)
	{
		const int l = i / x_block, x = i % x_block;
		float2 value = make_float2(0.0f, 0.0f);
		if (x < xw)
		{
			const int64_t o = global_offset(l, x);
			if (AXIS == 0 && P.wiener_mode >= 0)
			{
				const float2 num = P.numerator[o];
				const float den = P.denominator[o];
				if (P.wiener_mode == REXLIB_B200_WIENER_REGULARIZED)
				{
					const float inv = 1.0f / (den + P.constant);
					value = make_float2(num.x * inv, num.y * inv);
				}
				else if (den > P.constant)
				{
					value = make_float2(num.x / den, num.y / den);
				}
			}
			else
			{
				value = AXIS == 0 ? P.in[o] : P.work[o];
			}
		}
		tile[i] = value;
	}
	__syncthreads();
	constexpr int G = 32 / W;
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	const int group = warp * G + lane / W;
	const int j = lane % W;
	const typename line_fft<M, W>::plan line_plan(j, 1);
	for (int base = 0; base < x_block; base += (volume_threads / 32) * G)
	{
		const int x = base + group;
		const bool active = x < xw;
		float2 v[M];
#pragma unroll
		for (int n1 = 0; n1 < M; ++n1)
			v[n1] = active ? tile[(W * n1 + j) * x_block + x] : make_float2(0.0f, 0.0f);
		line_fft<M, W>::run(v, line_plan);
		if (active)
		{
#pragma unroll
			for (int k1 = 0; k1 < M; ++k1)
				tile[line_fft<M, W>::output_index(k1, j) * x_block + x] = v[k1];
		}
	}
	__syncthreads();
	for (int i = threadIdx.x; i < big * x_block; i += blockDim.x)
	{
		const int l = i / x_block, x = i % x_block;
		if (x < xw)
			P.work[global_offset(l, x)] = tile[i];
	}
}

// Pass 3: the C2R of each row along x (as irfft2's rows), W lanes a row; a
// grid-stride loop over the rows so each lane builds its plan once.
template <int M, int W>
__global__ void __launch_bounds__(volume_threads) volume_rows_kernel(const volume_launch P)
{
	__shared__ float2 split_twiddle[129]; // exp(2 pi i k / N), k < N/2
	const int big = P.big, H = P.H, L = big / 2;
	for (int k = threadIdx.x; k < L; k += blockDim.x)
		split_twiddle[k] = unit_root(k, big, 1);
	__syncthreads();
	constexpr int G = 32 / W;
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	const int j = lane % W;
	const typename line_fft<M, W>::plan row_plan(j, 1);
	const float scale = 1.0f / (static_cast<float>(big) * static_cast<float>(big) * static_cast<float>(L));
	const int64_t rows = static_cast<int64_t>(big) * big;
	const int64_t stride = static_cast<int64_t>(gridDim.x) * (volume_threads / 32) * G;
	// Every lane of a warp runs the same number of iterations (the shuffles
	// need the whole warp); a group past the last row computes on zeros.
	for (int64_t base = (static_cast<int64_t>(blockIdx.x) * (volume_threads / 32) + warp) * G; base < rows;
		 base += stride)
	{
		const int64_t row = base + lane / W;
		const bool active = row < rows;
		const float2 *in = P.work + (active ? row : 0) * H;
		float2 v[M];
#pragma unroll
		for (int n1 = 0; n1 < M; ++n1)
		{
			const int k = W * n1 + j;
			float2 r = make_float2(0.0f, 0.0f);
			if (active)
			{
				float2 a = in[k];
				float2 b = in[L - k];
				if (k == 0)
				{
					a.y = 0.0f;
					b.y = 0.0f;
				}
				const float2 bc = c_conj(b);
				const float2 e = make_float2(0.5f * (a.x + bc.x), 0.5f * (a.y + bc.y));
				const float2 d = make_float2(0.5f * (a.x - bc.x), 0.5f * (a.y - bc.y));
				const float2 o = c_mul(d, split_twiddle[k]);
				r = make_float2(e.x - o.y, e.y + o.x);
			}
			v[n1] = r;
		}
		line_fft<M, W>::run(v, row_plan);
		if (active)
		{
			float *out = P.out + row * big;
#pragma unroll
			for (int k1 = 0; k1 < M; ++k1)
			{
				const int idx = line_fft<M, W>::output_index(k1, j);
				*reinterpret_cast<float2 *>(out + 2 * idx) = make_float2(v[k1].x * scale, v[k1].y * scale);
			}
		}
	}
}

// Register-and-shared-memory forms of the three passes for N = 64, 128 and
// 256 (lines of N = R1 x R2 with R1 >= R2).
//  - Lines along z or y, 32 x per CTA: a line is R2 threads t of one x
//    (lanes run over x, so a warp's loads and stores are 32 consecutive
//    complex). Each thread loads its R1 elements x[R2 n1 + t] straight from
//    HBM, takes their DFT of R1 in registers and the twiddle
//    exp(2 pi i t k1 / N), writes them to a shared (N x 32) exchange in a
//    skewed order (element (k1, n2) at line position R2 k1 + (n2 + k1) mod
//    R2), and after a barrier takes the DFTs of R2 over n2 for k1 = t + R2 b
//    and stores the results straight to HBM.
//  - Rows along x: a line of N/2 = R1 x R2 per R2 threads, the C2R split
//    computed on the way in from the workspace, the exchange through a row
//    scratch padded to a half-warp's worth of banks.
template <int R1, int R2, int AXIS>
__global__ void __launch_bounds__(32 * R2, 1024 / (32 * R2)) volume_lines_fast_kernel(const volume_launch P)
{
	constexpr int N = R1 * R2, B = R1 / R2;
	static_assert(R1 % R2 == 0, "R2 divides R1");
	extern __shared__ float2 tile[]; // N x x_block: the exchange
	__shared__ float2 tw[N];         // exp(2 pi i m / N)
	const int H = P.H;
	const int x = threadIdx.x & 31;
	const int t = threadIdx.x >> 5;
	// H = N/2 + 1 = 32 q + 1. Blocks 0..q-1 take 32 x each at one fixed
	// coordinate (blockIdx.y); block q takes the last plane x = N/2, its
	// lanes running over 32 fixed coordinates (blockIdx.y < N/32; the rest
	// of that column of blocks has nothing to do).
	const bool last_plane = blockIdx.x == (H - 1) / x_block;
	if (last_plane && static_cast<int>(blockIdx.y) >= N / x_block)
		return;
	const int fixed = last_plane ? static_cast<int>(blockIdx.y) * x_block + x : static_cast<int>(blockIdx.y);
	const int xg = last_plane ? H - 1 : static_cast<int>(blockIdx.x) * x_block + x;
	auto global_offset = [&](int l) -> int64_t {
		return AXIS == 0 ? ((int64_t)l * N + fixed) * H + xg : ((int64_t)fixed * N + l) * H + xg;
	};
	for (int m = threadIdx.x; m < N; m += blockDim.x)
		tw[m] = unit_root(m, N, 1);
	// Step 1 straight from HBM: this thread's R1 elements x[R2 n1 + t], all
	// loads issued before any is used.
	float2 v[R1];
	if (AXIS == 0 && P.wiener_mode >= 0)
	{
		float den[R1];
#pragma unroll
		for (int n1 = 0; n1 < R1; ++n1)
		{
			v[n1] = P.numerator[global_offset(R2 * n1 + t)];
			den[n1] = P.denominator[global_offset(R2 * n1 + t)];
		}
#pragma unroll
		for (int n1 = 0; n1 < R1; ++n1)
		{
			if (P.wiener_mode == REXLIB_B200_WIENER_REGULARIZED)
			{
				const float inv = 1.0f / (den[n1] + P.constant);
				v[n1] = make_float2(v[n1].x * inv, v[n1].y * inv);
			}
			else
			{
				v[n1] = den[n1] > P.constant ? make_float2(v[n1].x / den[n1], v[n1].y / den[n1]) : make_float2(0.0f, 0.0f);
			}
		}
	}
	else
	{
		const float2 *src = AXIS == 0 ? P.in : P.work;
#pragma unroll
		for (int n1 = 0; n1 < R1; ++n1)
			v[n1] = src[global_offset(R2 * n1 + t)];
	}
	__syncthreads(); // the twiddle table
	{
		const small_dft<R1> dft(1);
		dft.run(v, 1);
#pragma unroll
		for (int k1 = 1; k1 < R1; ++k1)
			v[k1] = c_mul(v[k1], tw[(t * k1) & (N - 1)]);
#pragma unroll
		for (int k1 = 0; k1 < R1; ++k1)
			tile[(R2 * k1 + ((t + k1) & (R2 - 1))) * x_block + x] = v[k1];
	}
	__syncthreads();
	// Step 2 and the result straight to HBM: X[k1 + R1 k2] for k1 = t + R2 b.
	const small_dft<R2> dft(1);
#pragma unroll
	for (int b = 0; b < B; ++b)
	{
		const int k1 = t + R2 * b;
		float2 u[R2];
#pragma unroll
		for (int n2 = 0; n2 < R2; ++n2)
			u[n2] = tile[(R2 * k1 + ((n2 + k1) & (R2 - 1))) * x_block + x];
		dft.run(u, 1);
#pragma unroll
		for (int k2 = 0; k2 < R2; ++k2)
			P.work[global_offset(k1 + R1 * k2)] = u[k2];
	}
}

template <int R1, int R2>
__global__ void __launch_bounds__(volume_threads) volume_rows_fast_kernel(const volume_launch P)
{
	constexpr int L = R1 * R2, N = 2 * L, H = L + 1, B = R1 / R2;
	constexpr int rows_per_pass = volume_threads / R2;
	constexpr int stride = L + 8; // two rows of a half-warp 16 banks apart
	static_assert(R1 % R2 == 0, "R2 divides R1");
	__shared__ float2 scratch[rows_per_pass * stride];
	__shared__ float2 tw[N]; // exp(2 pi i m / N)
	for (int m = threadIdx.x; m < N; m += blockDim.x)
		tw[m] = unit_root(m, N, 1);
	__syncthreads();
	const int t = threadIdx.x % R2;
	const int local = threadIdx.x / R2;
	float2 *line = scratch + local * stride;
	const float scale = 1.0f / (static_cast<float>(N) * static_cast<float>(N) * static_cast<float>(L));
	const small_dft<R1> dft1(1);
	const small_dft<R2> dft2(1);
	const int64_t rows = static_cast<int64_t>(N) * N;
	for (int64_t base = static_cast<int64_t>(blockIdx.x) * rows_per_pass; base < rows;
		 base += static_cast<int64_t>(gridDim.x) * rows_per_pass)
	{
		const int64_t row = base + local;
		const float2 *in = P.work + row * H;
		// Z[k] = E[k] + i O[k]: E = (X[k] + conj X[L-k]) / 2,
		// O = (X[k] - conj X[L-k]) / 2 * exp(2 pi i k / N); the imaginary
		// parts of X[0] and X[L] are ignored, as a C2R does.
		float2 v[R1];
#pragma unroll
		for (int n1 = 0; n1 < R1; ++n1)
		{
			const int k = R2 * n1 + t;
			float2 a = in[k];
			float2 b = in[L - k];
			if (k == 0)
			{
				a.y = 0.0f;
				b.y = 0.0f;
			}
			const float2 bc = c_conj(b);
			const float2 e = make_float2(0.5f * (a.x + bc.x), 0.5f * (a.y + bc.y));
			const float2 o = c_mul(make_float2(0.5f * (a.x - bc.x), 0.5f * (a.y - bc.y)), tw[k]);
			v[n1] = make_float2(e.x - o.y, e.y + o.x);
		}
		dft1.run(v, 1);
#pragma unroll
		for (int k1 = 1; k1 < R1; ++k1)
			v[k1] = c_mul(v[k1], tw[(2 * t * k1) & (N - 1)]);
		__syncwarp();
#pragma unroll
		for (int k1 = 0; k1 < R1; ++k1)
			line[R2 * k1 + ((t + k1) & (R2 - 1))] = v[k1];
		__syncwarp();
		float *out = P.out + row * N;
#pragma unroll
		for (int b = 0; b < B; ++b)
		{
			const int k1 = t + R2 * b;
			float2 u[R2];
#pragma unroll
			for (int n2 = 0; n2 < R2; ++n2)
				u[n2] = line[R2 * k1 + ((n2 + k1) & (R2 - 1))];
			dft2.run(u, 1);
#pragma unroll
			for (int k2 = 0; k2 < R2; ++k2)
				*reinterpret_cast<float2 *>(out + 2 * (k1 + R1 * k2)) =
					make_float2(u[k2].x * scale, u[k2].y * scale);
		}
	}
}

template <int R1, int R2, int RR1, int RR2>
void run_volume_fast(const volume_launch &P, cudaStream_t stream)
{
	const size_t smem = sizeof(float2) * static_cast<size_t>(P.big) * x_block;
	const dim3 grid((P.H + x_block - 1) / x_block, P.big);
	auto z_pass = volume_lines_fast_kernel<R1, R2, 0>;
	auto y_pass = volume_lines_fast_kernel<R1, R2, 1>;
	check_cuda(cudaFuncSetAttribute(z_pass, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)),
		"irfft3 attributes");
	check_cuda(cudaFuncSetAttribute(y_pass, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)),
		"irfft3 attributes");
	z_pass<<<grid, 32 * R2, smem, stream>>>(P);
	check_cuda(cudaGetLastError(), "irfft3 z pass");
	y_pass<<<grid, 32 * R2, smem, stream>>>(P);
	check_cuda(cudaGetLastError(), "irfft3 y pass");
	int device = 0, sms = 0;
	check_cuda(cudaGetDevice(&device), "device query");
	check_cuda(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "device query");
	const int64_t rows = static_cast<int64_t>(P.big) * P.big;
	const int64_t rows_per_pass = volume_threads / RR2;
	const int64_t blocks = std::min<int64_t>(rows / rows_per_pass, static_cast<int64_t>(sms) * 8);
	volume_rows_fast_kernel<RR1, RR2><<<static_cast<unsigned>(blocks), volume_threads, 0, stream>>>(P);
	check_cuda(cudaGetLastError(), "irfft3 x pass");
}

template <int CM, int CW, int RM, int RW>
void run_volume(const volume_launch &P, cudaStream_t stream)
{
	const size_t smem = sizeof(float2) * static_cast<size_t>(P.big) * x_block;
	const dim3 grid((P.H + x_block - 1) / x_block, P.big);
	auto z_pass = volume_lines_kernel<CM, CW, 0>;
	auto y_pass = volume_lines_kernel<CM, CW, 1>;
	check_cuda(cudaFuncSetAttribute(z_pass, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)),
		"irfft3 attributes");
	check_cuda(cudaFuncSetAttribute(y_pass, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)),
		"irfft3 attributes");
	z_pass<<<grid, volume_threads, smem, stream>>>(P);
	check_cuda(cudaGetLastError(), "irfft3 z pass");
	y_pass<<<grid, volume_threads, smem, stream>>>(P);
	check_cuda(cudaGetLastError(), "irfft3 y pass");
	const int64_t rows = static_cast<int64_t>(P.big) * P.big;
	const int64_t rows_per_block = (volume_threads / 32) * (32 / RW);
	int device = 0, sms = 0;
	check_cuda(cudaGetDevice(&device), "device query");
	check_cuda(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "device query");
	const int64_t blocks = std::min<int64_t>((rows + rows_per_block - 1) / rows_per_block, static_cast<int64_t>(sms) * 8);
	volume_rows_kernel<RM, RW><<<static_cast<unsigned>(blocks), volume_threads, 0, stream>>>(P);
	check_cuda(cudaGetLastError(), "irfft3 x pass");
}

bool run_for_extent(const volume_launch &P, cudaStream_t stream)
{
	switch (P.big)
	{
	case 32:
		run_volume<1, 32, 1, 16>(P, stream);
		return true;
	case 64:
		run_volume_fast<8, 8, 8, 4>(P, stream);
		return true;
	case 96:
		run_volume<3, 32, 3, 16>(P, stream);
		return true;
	case 128:
		run_volume_fast<16, 8, 8, 8>(P, stream);
		return true;
	case 160:
		run_volume<5, 32, 5, 16>(P, stream);
		return true;
	case 192:
		run_volume<6, 32, 3, 32>(P, stream);
		return true;
	case 200:
		run_volume<25, 8, 25, 4>(P, stream);
		return true;
	case 256:
		run_volume_fast<16, 16, 16, 8>(P, stream);
		return true;
	default:
		return false;
	}
}

bool supported_volume(int64_t big)
{
	return big == 32 || big == 64 || big == 96 || big == 128 || big == 160 || big == 192 || big == 200 || big == 256;
}

size_t volume_workspace(int64_t big) { return sizeof(float2) * static_cast<size_t>(big) * big * (big / 2 + 1); }

void run_checked(volume_launch &P, int64_t extent, void *workspace, size_t workspace_bytes, void *stream)
{
	if (!supported_volume(extent))
		fail(REXLIB_B200_UNSUPPORTED, "irfft3 runs volumes of 32, 64, 96, 128, 160, 192, 200 or 256");
	require(P.out != nullptr, "null output");
	const size_t need = volume_workspace(extent);
	if (workspace == nullptr || workspace_bytes < need)
		fail(REXLIB_B200_WORKSPACE_TOO_SMALL, "irfft3 needs " + std::to_string(need) + " bytes of workspace");
	P.big = static_cast<int>(extent);
	P.H = P.big / 2 + 1;
	P.work = static_cast<float2 *>(workspace);
	run_for_extent(P, as_stream(stream));
}

} // anonymous namespace
} // namespace rexlib_b200

using namespace rexlib_b200;

extern "C" int32_t rexlib_b200_irfft3_workspace_size(int64_t extent, size_t *bytes)
{
	return guarded([&] {
		require(bytes != nullptr, "null result pointer");
		if (!supported_volume(extent))
			fail(REXLIB_B200_UNSUPPORTED, "irfft3 runs volumes of 32, 64, 96, 128, 160, 192, 200 or 256");
		*bytes = volume_workspace(extent);
	});
}

extern "C" int32_t rexlib_b200_irfft3(float *out, const void *in, int64_t extent, void *workspace,
	size_t workspace_bytes, void *stream)
{
	return guarded([&] {
		require(in != nullptr, "null input");
		volume_launch P{};
		P.in = static_cast<const float2 *>(in);
		P.out = out;
		P.wiener_mode = -1;
		run_checked(P, extent, workspace, workspace_bytes, stream);
	});
}

extern "C" int32_t rexlib_b200_wiener_irfft3(float *out, const void *numerator, const float *denominator,
	int64_t extent, int32_t mode, double constant, void *workspace, size_t workspace_bytes, void *stream)
{
	return guarded([&] {
		require(numerator != nullptr && denominator != nullptr, "null accumulator");
		require(mode == REXLIB_B200_WIENER_REGULARIZED || mode == REXLIB_B200_WIENER_THRESHOLD, "unknown Wiener mode");
		require(std::isfinite(constant), "the Wiener constant must be finite");
		volume_launch P{};
		P.numerator = static_cast<const float2 *>(numerator);
		P.denominator = denominator;
		P.out = out;
		P.wiener_mode = mode;
		P.constant = static_cast<float>(constant);
		run_checked(P, extent, workspace, workspace_bytes, stream);
	});
}
