// Volume tools of the learned prior's reconstruction loop:
// - rfft3: the unnormalised 3D R2C of a real (N, N, N) volume into its half
//   spectrum (N, N, N/2+1) (rfft_operation over three axes; the CPU runs
//   pocketfft's r2c, src/backends/cpu/kernels/pocketfft_fourier_transform.cpp:129),
//   N in {32, 64, 128, 256}: rows along x (an N/2 complex FFT of the packed
//   reals, then the real split), then lines along y and z;
// - the Fourier shell correlation of two half spectra;
// - the prior-regularised Wiener combination (N + c P) / (D + c);
// - the analytic spectrum of a phantom of Gaussian blobs (optionally low-
//   passed), and its noisy CTF-modulated central slices: the synthetic data
//   the prior is trained on and judged with.
#include "common.cuh"
#include "fft.cuh"
#include "standardize.cuh"

#include <algorithm>
#include <cmath>
#include <string>

namespace rexlib_b200
{
namespace
{

constexpr int tool_threads = 256;
constexpr int tile_x = 32;

// Rows: the R2C of each row of N reals, W lanes a row (N/2 = M x W).
template <int M, int W>
__global__ void __launch_bounds__(tool_threads) rows_r2c_kernel(const float *__restrict__ in, float2 *__restrict__ out,
	int big)
{
	constexpr int L = M * W; // N / 2
	constexpr int G = tool_threads / W;
	__shared__ float2 z[G][L + 1];
	__shared__ float2 twiddle[L];
	const int H = big / 2 + 1;
	for (int k = threadIdx.x; k < L; k += blockDim.x)
		twiddle[k] = unit_root(k, big, -1); // exp(-2 pi i k / N)
	const int g = threadIdx.x / W, j = threadIdx.x % W;
	const typename line_fft<M, W>::plan plan(j, -1);
	const int64_t rows = static_cast<int64_t>(big) * big;
	__syncthreads();
	for (int64_t base = static_cast<int64_t>(blockIdx.x) * G; base < rows; base += static_cast<int64_t>(gridDim.x) * G)
	{
		const int64_t row = base + g;
		const bool active = row < rows;
		const float2 *src = reinterpret_cast<const float2 *>(in + (active ? row : 0) * big);
		float2 v[M];
#pragma unroll
		for (int n1 = 0; n1 < M; ++n1)
			v[n1] = active ? src[W * n1 + j] : make_float2(0.0f, 0.0f);
		line_fft<M, W>::run(v, plan);
#pragma unroll
		for (int k1 = 0; k1 < M; ++k1)
			z[g][line_fft<M, W>::output_index(k1, j)] = v[k1];
		__syncthreads();
		if (active)
		{
			float2 *dst = out + row * H;
			for (int k = j; k < H; k += W)
			{
				// X[k] = (Z[k] + conj Z[L-k]) / 2 - i exp(-2 pi i k / N) (Z[k] - conj Z[L-k]) / 2.
				const float2 a = z[g][k % L];
				const float2 b = c_conj(z[g][(L - k) % L]);
				const float2 e = make_float2(0.5f * (a.x + b.x), 0.5f * (a.y + b.y));
				const float2 d = make_float2(0.5f * (a.x - b.x), 0.5f * (a.y - b.y));
				const float2 t = c_mul(d, k < L ? twiddle[k] : make_float2(-1.0f, 0.0f));
				dst[k] = make_float2(e.x + t.y, e.y - t.x);
			}
		}
		__syncthreads();
	}
}

// Lines along z (AXIS 0) or y (AXIS 1) of a (N, N, H) complex array, 32 x a
// block, forward (unnormalised), from src into dst (which may be src).
template <int M, int AXIS>
__global__ void __launch_bounds__(tool_threads) lines_forward_kernel(const float2 *src, float2 *dst, int big)
{
	extern __shared__ float2 tile[]; // N x tile_x
	const int H = big / 2 + 1;
	const int fixed = blockIdx.y;
	const int x0 = blockIdx.x * tile_x;
	const int xw = min(tile_x, H - x0);
	auto offset = [&](int l, int x) -> int64_t {
		return AXIS == 0 ? (static_cast<int64_t>(l) * big + fixed) * H + x0 + x : (static_cast<int64_t>(fixed) * big + l) * H + x0 + x;
	};
	for (int i = threadIdx.x; i < big * tile_x; i += blockDim.x)
	{
		const int l = i / tile_x, x = i % tile_x;
		tile[i] = x < xw ? src[offset(l, x)] : make_float2(0.0f, 0.0f);
	}
	__syncthreads();
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	const typename line_fft<M, 32>::plan plan(lane, -1);
	for (int x = warp; x < tile_x; x += tool_threads / 32)
	{
		float2 v[M];
#pragma unroll
		for (int n1 = 0; n1 < M; ++n1)
			v[n1] = tile[(32 * n1 + lane) * tile_x + x];
		line_fft<M, 32>::run(v, plan);
		__syncwarp();
#pragma unroll
		for (int k1 = 0; k1 < M; ++k1)
			tile[line_fft<M, 32>::output_index(k1, lane) * tile_x + x] = v[k1];
	}
	__syncthreads();
	for (int i = threadIdx.x; i < big * tile_x; i += blockDim.x)
	{
		const int l = i / tile_x, x = i % tile_x;
		if (x < xw)
			dst[offset(l, x)] = tile[i];
	}
}

template <int RM, int RW, int CM>
void run_rfft3(const float *in, float2 *out, int big, cudaStream_t stream)
{
	const int64_t rows = static_cast<int64_t>(big) * big;
	const int groups = tool_threads / RW;
	const unsigned blocks = static_cast<unsigned>(std::min<int64_t>((rows + groups - 1) / groups, 148 * 8));
	rows_r2c_kernel<RM, RW><<<blocks, tool_threads, 0, stream>>>(in, out, big);
	check_cuda(cudaGetLastError(), "rfft3 x pass");
	const size_t smem = sizeof(float2) * static_cast<size_t>(big) * tile_x;
	const dim3 grid((big / 2 + 1 + tile_x - 1) / tile_x, big);
	auto y_pass = lines_forward_kernel<CM, 1>;
	auto z_pass = lines_forward_kernel<CM, 0>;
	check_cuda(cudaFuncSetAttribute(y_pass, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)),
		"rfft3 attributes");
	check_cuda(cudaFuncSetAttribute(z_pass, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)),
		"rfft3 attributes");
	y_pass<<<grid, tool_threads, smem, stream>>>(out, out, big);
	check_cuda(cudaGetLastError(), "rfft3 y pass");
	z_pass<<<grid, tool_threads, smem, stream>>>(out, out, big);
	check_cuda(cudaGetLastError(), "rfft3 z pass");
}

} // anonymous namespace
} // namespace rexlib_b200

namespace rexlib_b200
{
namespace
{

__device__ __forceinline__ int signed_frequency(int s, int big) { return s <= big / 2 ? s : s - big; }

// Fourier shell correlation sums of two half spectra, per shell
// round(|k|) <= N/2: sum Re(a conj b), sum |a|^2, sum |b|^2, each stored
// frequency counted twice but for the planes x = 0 and x = N/2 (even N),
// which hold their own conjugates.
__global__ void __launch_bounds__(tool_threads) fsc_kernel(const float2 *__restrict__ a, const float2 *__restrict__ b,
	int big, double *__restrict__ sums)
{
	extern __shared__ double acc[]; // 3 x shells
	const int H = big / 2 + 1, shells = big / 2 + 1;
	for (int i = threadIdx.x; i < 3 * shells; i += blockDim.x)
		acc[i] = 0.0;
	__syncthreads();
	const int64_t n = static_cast<int64_t>(big) * big * H;
	for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
		 i += static_cast<int64_t>(gridDim.x) * blockDim.x)
	{
		const int x = static_cast<int>(i % H), y = static_cast<int>((i / H) % big), z = static_cast<int>(i / (static_cast<int64_t>(H) * big));
		const int ky = signed_frequency(y, big), kz = signed_frequency(z, big);
		const double r = sqrt(static_cast<double>(x) * x + static_cast<double>(ky) * ky + static_cast<double>(kz) * kz);
		const int shell = static_cast<int>(r + 0.5);
		if (shell >= shells)
			continue;
		const double w = (x == 0 || (big % 2 == 0 && x == big / 2)) ? 1.0 : 2.0;
		const float2 u = a[i], v = b[i];
		atomicAdd(&acc[shell], w * (static_cast<double>(u.x) * v.x + static_cast<double>(u.y) * v.y));
		atomicAdd(&acc[shells + shell], w * (static_cast<double>(u.x) * u.x + static_cast<double>(u.y) * u.y));
		atomicAdd(&acc[2 * shells + shell], w * (static_cast<double>(v.x) * v.x + static_cast<double>(v.y) * v.y));
	}
	__syncthreads();
	for (int i = threadIdx.x; i < 3 * shells; i += blockDim.x)
		if (acc[i] != 0.0)
			atomicAdd(sums + i, acc[i]);
}

// out = (numerator + c prior) / (denominator + c), voxel by voxel.
__global__ void prior_wiener_kernel(int64_t n, const float2 *__restrict__ num, const float *__restrict__ den,
	const float2 *__restrict__ prior, float c, float2 *__restrict__ out)
{
	for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
		 i += static_cast<int64_t>(gridDim.x) * blockDim.x)
	{
		const float inv = 1.0f / (den[i] + c);
		const float2 p = prior[i], q = num[i];
		out[i] = make_float2((q.x + c * p.x) * inv, (q.y + c * p.y) * inv);
	}
}

// A phantom: blob b has amplitude, sigma (voxels) and centre (x, y, z)
// relative to the volume centre N/2, stored as 5 floats.
// The half spectrum of the volume sum_b a exp(-|p - N/2 - c|^2 / (2 s^2)):
// a (2 pi)^(3/2) s^3 exp(-2 pi^2 s^2 |k|^2 / N^2) exp(-2 pi i k.(N/2 + c) / N),
// zero beyond the shell `cutoff` (|k| > cutoff; cutoff < 0 keeps all).
__global__ void blob_spectrum_kernel(const float *__restrict__ blobs, int count, int big, double cutoff,
	float2 *__restrict__ out)
{
	const int H = big / 2 + 1;
	const int64_t n = static_cast<int64_t>(big) * big * H;
	for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
		 i += static_cast<int64_t>(gridDim.x) * blockDim.x)
	{
		const int x = static_cast<int>(i % H), y = static_cast<int>((i / H) % big), z = static_cast<int>(i / (static_cast<int64_t>(H) * big));
		const double kx = x, ky = signed_frequency(y, big), kz = signed_frequency(z, big);
		const double k2 = kx * kx + ky * ky + kz * kz;
		double re = 0.0, im = 0.0;
		if (cutoff < 0.0 || k2 <= cutoff * cutoff)
		{
			const double half = 0.5 * big;
			for (int b = 0; b < count; ++b)
			{
				const float *p = blobs + 5 * b;
				const double s = p[1];
				const double mag = p[0] * 15.749609945722419 * s * s * s * exp(-2.0 * pi * pi * s * s * k2 / (double(big) * big));
				const double phase = -2.0 * pi * (kx * (half + p[2]) + ky * (half + p[3]) + kz * (half + p[4])) / big;
				double sn, cs;
				sincos(phase, &sn, &cs);
				re += mag * cs;
				im += mag * sn;
			}
		}
		out[i] = make_float2(static_cast<float>(re), static_cast<float>(im));
	}
}

// Noisy CTF-modulated central slices of a blob phantom: slice p at
// frequency (kx, ky) holds c(k) F(kx A0 + ky A1) + noise, F the phantom's
// spectrum above written for an image centred at n/2 (the DFT of the
// projection along A2), A0 and A1 the first two rows of transform p, c the
// CTF of the slice (the reference's expression, contrast_transfer_function.inl:
// 26-80, with defocus U, V, angle and phase shift of row p of `ctf`), and
// the noise complex Gaussian of standard deviation `noise` per component
// (Philox draws keyed by `seed`). One CTA a slice; per blob, the separable
// factors along kx and ky come from shared tables, `chunk` blobs at a time
// (the partial sums of a slice wait in its output between chunks).
constexpr int slice_blobs_max = 4096;

__global__ void __launch_bounds__(tool_threads) phantom_slices_kernel(const float *__restrict__ blobs, int count,
	int chunk, int n, const float *__restrict__ transforms, const float *__restrict__ ctf, double wavelength,
	double cs_angstrom, double phase_offset, double frequency_scale_sq, float noise, uint64_t seed,
	float2 *__restrict__ out)
{
	extern __shared__ float2 table[]; // chunk x (h + n): row factors then column factors
	const int h = n / 2 + 1;
	const int p = blockIdx.x;
	const float *tr = transforms + 12 * p;
	const double half = 0.5 * n;
	float2 *dst = out + static_cast<int64_t>(p) * n * h;
	for (int b0 = 0; b0 < count; b0 += chunk)
	{
	const int nb = min(chunk, count - b0);
	__syncthreads(); // the previous chunk's tables are consumed
	for (int i = threadIdx.x; i < nb * (h + n); i += blockDim.x)
	{
		const int b = i / (h + n), j = i % (h + n);
		const float *bl = blobs + 5 * (b0 + b);
		const double s = bl[1];
		const double alpha = 2.0 * pi * pi * s * s / (double(n) * n);
		// Offset of the blob's centre along the slice's axes A0 (x) and A1 (y).
		const double u = tr[0] * bl[2] + tr[1] * bl[3] + tr[2] * bl[4];
		const double v = tr[4] * bl[2] + tr[5] * bl[3] + tr[6] * bl[4];
		double k, shift, scale;
		if (j < h)
		{
			k = j;
			shift = half + u;
			scale = bl[0] * 15.749609945722419 * s * s * s;
		}
		else
		{
			k = signed_frequency(j - h, n);
			shift = half + v;
			scale = 1.0;
		}
		double sn, cs;
		sincos(-2.0 * pi * k * shift / n, &sn, &cs);
		const double g = scale * exp(-alpha * k * k);
		table[i] = make_float2(static_cast<float>(g * cs), static_cast<float>(g * sn));
	}
	__syncthreads();
	const bool last = b0 + nb >= count;
	// CTF coefficients of the slice (as the insertion settles them).
	const double du = ctf[4 * p], dv = ctf[4 * p + 1], angle = ctf[4 * p + 2], shift = ctf[4 * p + 3];
	const double dscale = pi * wavelength * frequency_scale_sq;
	const double hd = 0.5 * (du - dv);
	const double c0 = dscale * 0.5 * (du + dv), c1 = dscale * hd * cos(2.0 * angle), c2 = 2.0 * dscale * hd * sin(2.0 * angle);
	const double c3 = 0.5 * pi * cs_angstrom * wavelength * wavelength * wavelength * frequency_scale_sq * frequency_scale_sq;
	const double c4 = shift + phase_offset;
	for (int i = threadIdx.x; i < n * h; i += blockDim.x)
	{
		const int row = i / h, kx = i % h;
		const double ky = signed_frequency(row, n);
		float2 acc = b0 > 0 ? dst[i] : make_float2(0.0f, 0.0f);
		for (int b = 0; b < nb; ++b)
		{
			const float2 tx = table[b * (h + n) + kx];
			const float2 ty = table[b * (h + n) + h + row];
			acc.x += tx.x * ty.x - tx.y * ty.y;
			acc.y += tx.x * ty.y + tx.y * ty.x;
		}
		if (!last)
		{
			dst[i] = acc;
			continue;
		}
		const double xx = double(kx) * kx, yy = ky * ky, sq = xx + yy;
		const double phase = c0 * sq + c1 * (xx - yy) + c2 * (kx * ky) - c3 * sq * sq + c4;
		const float c = static_cast<float>(sin(phase));
		float2 value = make_float2(c * acc.x, c * acc.y);
		if (noise > 0.0f)
		{
			const double2 z = normal_pair(seed + static_cast<uint64_t>(p), static_cast<uint64_t>(i));
			value.x += noise * static_cast<float>(z.x);
			value.y += noise * static_cast<float>(z.y);
		}
		dst[i] = value;
	}
	}
}

} // anonymous namespace
} // namespace rexlib_b200

using namespace rexlib_b200;

extern "C" int32_t rexlib_b200_rfft3(void *out, const float *in, int64_t extent, void *stream)
{
	return guarded([&] {
		require(in != nullptr && out != nullptr, "null volume");
		const cudaStream_t s = as_stream(stream);
		float2 *o = static_cast<float2 *>(out);
		switch (extent)
		{
		case 32:
			run_rfft3<2, 8, 1>(in, o, 32, s);
			break;
		case 64:
			run_rfft3<4, 8, 2>(in, o, 64, s);
			break;
		case 128:
			run_rfft3<8, 8, 4>(in, o, 128, s);
			break;
		case 256:
			run_rfft3<16, 8, 8>(in, o, 256, s);
			break;
		default:
			fail(REXLIB_B200_UNSUPPORTED, "rfft3 runs volumes of 32, 64, 128 or 256");
		}
	});
}

extern "C" int32_t rexlib_b200_fsc(const void *a, const void *b, int64_t extent, double *sums, void *stream)
{
	return guarded([&] {
		require(a != nullptr && b != nullptr && sums != nullptr, "null operand");
		require(extent >= 2 && extent <= 2048, "volume extents from 2 to 2048");
		const int shells = static_cast<int>(extent / 2 + 1);
		const cudaStream_t s = as_stream(stream);
		check_cuda(cudaMemsetAsync(sums, 0, sizeof(double) * 3 * shells, s), "shell sums");
		fsc_kernel<<<148 * 4, tool_threads, sizeof(double) * 3 * shells, s>>>(static_cast<const float2 *>(a),
			static_cast<const float2 *>(b), static_cast<int>(extent), sums);
		check_cuda(cudaGetLastError(), "shell correlation launch");
	});
}

extern "C" int32_t rexlib_b200_prior_wiener(void *out, const void *numerator, const float *denominator,
	const void *prior, int64_t extent, double constant, void *stream)
{
	return guarded([&] {
		require(out && numerator && denominator && prior, "null operand");
		require(std::isfinite(constant) && constant > 0.0, "the constant must be finite and positive");
		const int64_t n = extent * extent * (extent / 2 + 1);
		prior_wiener_kernel<<<148 * 8, tool_threads, 0, as_stream(stream)>>>(n, static_cast<const float2 *>(numerator),
			denominator, static_cast<const float2 *>(prior), static_cast<float>(constant), static_cast<float2 *>(out));
		check_cuda(cudaGetLastError(), "prior Wiener launch");
	});
}

extern "C" int32_t rexlib_b200_blob_spectrum(void *out, const float *blobs, int32_t count, int64_t extent,
	double cutoff, void *stream)
{
	return guarded([&] {
		require(out && (count == 0 || blobs), "null operand");
		require(extent >= 2 && extent <= 2048, "volume extents from 2 to 2048");
		blob_spectrum_kernel<<<148 * 8, tool_threads, 0, as_stream(stream)>>>(blobs, count, static_cast<int>(extent),
			cutoff, static_cast<float2 *>(out));
		check_cuda(cudaGetLastError(), "blob spectrum launch");
	});
}

extern "C" int32_t rexlib_b200_phantom_slices(void *out, const float *blobs, int32_t count, int64_t slices,
	int64_t extent, const float *transforms, const float *ctf, rexlib_b200_ctf_optics optics, double pixel_size,
	double noise, uint64_t seed, void *stream)
{
	return guarded([&] {
		require(out && blobs && transforms && ctf, "null operand");
		if (count < 1 || count > slice_blobs_max)
			fail(REXLIB_B200_UNSUPPORTED, "phantom slices take 1 to 4096 blobs");
		require(extent >= 8 && extent <= 512 && slices >= 0 && slices < (1LL << 31), "extents from 8 to 512");
		const int n = static_cast<int>(extent);
		const size_t per_blob = sizeof(float2) * (n / 2 + 1 + n);
		const int chunk = static_cast<int>(std::min<size_t>(64, std::min<size_t>(count, 200 * 1024 / per_blob)));
		const size_t smem = per_blob * chunk;
		check_cuda(cudaFuncSetAttribute(phantom_slices_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
					   static_cast<int>(smem)),
			"phantom slices attributes");
		const double volts = optics.voltage * 1e3;
		const double wavelength = 12.2643247 / std::sqrt(volts * (1.0 + 0.978466e-6 * volts));
		const double fs = 1.0 / (static_cast<double>(n) * pixel_size);
		if (slices > 0)
			phantom_slices_kernel<<<static_cast<unsigned>(slices), tool_threads, smem, as_stream(stream)>>>(blobs, count,
				chunk, n, transforms, ctf, wavelength, optics.spherical_aberration * 1e7, std::asin(optics.amplitude_contrast),
				fs * fs, static_cast<float>(noise), seed, static_cast<float2 *>(out));
		check_cuda(cudaGetLastError(), "phantom slices launch");
	});
}
