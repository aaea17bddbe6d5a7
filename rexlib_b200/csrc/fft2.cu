// Batched 2D real FFTs of square images, one CTA per image.
//
// rfft2: the forward, unnormalised R2C of (n, n) float images into
// (n, n/2+1) complex half spectra, rows k_y in numpy.fft.fftfreq order and
// columns k_x >= 0 (rexlib's rfft2 layout, include/rexlib/ops/fourier/
// rfft_operation.hpp; the CPU runs pocketfft's r2c,
// src/backends/cpu/kernels/pocketfft_fourier_transform.cpp:129). Each row
// packs its reals in pairs into a complex line of n/2 (x[2j] + i x[2j+1]),
// transforms it, and splits it into the n/2+1 outputs; the columns are then
// transformed in shared memory. An epilogue can multiply every frequency by
// the image's CTF c(k) (or its sign, a phase flip) and write c(k)^2 beside
// it: the slice and the weight that insert_weighted_slices takes.
//
// irfft2: the exact inverse (the backward normalisation, 1/n^2), columns
// first, then each row's half spectrum recombined into a complex line of n/2
// and inverted; the imaginary parts of the k_x = 0 and k_x = n/2 columns are
// ignored, as a C2R does.
//
// Sizes: n in {32, 64, 96, 128, 160, 192, 200, 256} for rfft2 and the same
// up to 200 for irfft2 (their lines factor as M x W with W a power of two).
// A 256 spectrum does not fit in one CTA's shared memory: rfft2 at 256 runs
// on a cluster of CTAs that split the columns (rfft2_256_kernel). The
// general kernel, which then runs its columns in two halves and transforms
// the rows twice, remains for inputs that are not 8-byte aligned.
//
// standardize_rfft2: at n = 64 and 128 the R2C kernels can standardize the
// image they have staged in shared memory (background statistics, map and
// draws, standardize.cuh) before transforming it, so the standardized image
// never travels through HBM. The spectra are the same bits as those of the
// standardization followed by rfft2.
#include "common.cuh"
#include "fft.cuh"
#include "standardize.cuh"

#include <cmath>

#include <cooperative_groups.h>

namespace rexlib_b200
{
namespace
{

constexpr int fft_threads = 256;
constexpr int max_half_spectrum = 129; // h at the largest extent, 256
constexpr size_t fft_smem_budget = 220 * 1024;

struct rfft2_launch
{
	const float *in;
	float2 *out;
	float *weights;
	int64_t batch;
	int n, h, L;
	int ncols;
	int ctf_mode;
	const float *ctf;
	int64_t ctf_stride;
	const float *voltage;
	double voltage_default;
	double aberration;   // Cs in angstroms
	double phase_offset; // asin(Q)
	double frequency_scale_sq;
};

__device__ __forceinline__ double wavelength_of(double kv)
{
	const double volts = kv * 1e3;
	return 12.2643247 / sqrt(volts * (1.0 + 0.978466e-6 * volts));
}

// CTF coefficients of contrast_transfer_function.inl:26-65 for one image:
// radial, axial, diagonal, aberration and the phase offset.
__device__ __forceinline__ void ctf_coefficients(const rfft2_launch &P, int64_t image, float *coef)
{
	const float *c = P.ctf + image * P.ctf_stride;
	const double du = c[0], dv = c[1], angle = c[2], shift = c[3];
	const double wl = wavelength_of(P.voltage ? static_cast<double>(P.voltage[image]) : P.voltage_default);
	const double dscale = pi * wl * P.frequency_scale_sq;
	const double hd = 0.5 * (du - dv);
	double s2, c2;
	sincos(2.0 * angle, &s2, &c2);
	coef[0] = static_cast<float>(dscale * 0.5 * (du + dv));
	coef[1] = static_cast<float>(dscale * hd * c2);
	coef[2] = static_cast<float>(2.0 * dscale * hd * s2);
	coef[3] = static_cast<float>(0.5 * pi * P.aberration * wl * wl * wl * P.frequency_scale_sq * P.frequency_scale_sq);
	coef[4] = static_cast<float>(shift + P.phase_offset);
}

// Columns [c0, c1) of the half spectrum, held in shared memory with row
// stride `stride` (column c0 first), through the CTF epilogue to the output.
// The CTA walks the (row, k_x) pairs in output order, so every lane has work
// and consecutive threads store consecutive outputs. The row of pair i is
// (i + 1/2) / width in float: exact, since the quotient stays at least
// 1/(2 width) from an integer while its rounding error is below 2^-24 i/width.
__device__ __forceinline__ void ctf_epilogue_store(const rfft2_launch &P, int64_t image, const float2 *buf,
	int stride, int c0, int c1, const float *coef)
{
	const int n = P.n, h = P.h;
	const int width = c1 - c0;
	const float inv_width = 1.0f / static_cast<float>(width);
	float2 *out = P.out + image * static_cast<int64_t>(n) * h;
	float *wout = P.weights ? P.weights + image * static_cast<int64_t>(n) * h : nullptr;
	for (int i = threadIdx.x; i < n * width; i += blockDim.x)
	{
		const int row = static_cast<int>((static_cast<float>(i) + 0.5f) * inv_width);
		const int cw = i - row * width;
		const int col = c0 + cw;
		float2 X = buf[static_cast<size_t>(row) * stride + cw];
		if (P.ctf_mode != 0)
		{
			// k_y in numpy.fft.fftfreq order: the row n/2 is -n/2.
			const float ky = static_cast<float>(row < n / 2 ? row : row - n);
			const float kx = static_cast<float>(col);
			const float xx = kx * kx, yy = ky * ky, sq = xx + yy;
			const float ph = coef[0] * sq + coef[1] * (xx - yy) + coef[2] * (kx * ky) - coef[3] * (sq * sq) + coef[4];
			const float c = sin_reduced(ph);
			const float f = P.ctf_mode == 1 ? c : (c < 0.0f ? -1.0f : 1.0f);
			X.x *= f;
			X.y *= f;
			if (wout)
				wout[static_cast<int64_t>(row) * h + col] = P.ctf_mode == 1 ? c * c : fabsf(c);
		}
		out[static_cast<int64_t>(row) * h + col] = X;
	}
}

template <int RM, int RW, int CM, int CW>
__global__ void __launch_bounds__(fft_threads) rfft2_kernel(const rfft2_launch P)
{
	extern __shared__ float2 smem[];
	__shared__ float coef[5];
	__shared__ float2 split_twiddle[max_half_spectrum]; // exp(-2 pi i k / n), k < h
	constexpr int RG = 32 / RW, CG = 32 / CW;
	const int n = P.n, h = P.h, L = P.L, ncols = P.ncols;
	for (int k = threadIdx.x; k < h; k += blockDim.x)
		split_twiddle[k] = unit_root(k == n ? 0 : k, n, -1);
	float2 *buf = smem;
	float2 *zbuf = buf + static_cast<size_t>(n) * ncols;
	const int64_t image = blockIdx.x;
	const float *x = P.in + image * static_cast<int64_t>(n) * n;
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	const int warps = blockDim.x >> 5;

	if (P.ctf_mode != 0 && threadIdx.x == 0)
		ctf_coefficients(P, image, coef);
	__syncthreads(); // the split twiddles and the CTF coefficients

	for (int c0 = 0; c0 < h; c0 += ncols)
	{
		const int c1 = min(h, c0 + ncols);
		const int width = c1 - c0;
		// Rows: R2C by a packed complex line of n/2 and the split.
		{
			const int group = warp * RG + lane / RW;
			const int j = lane % RW;
			const typename line_fft<RM, RW>::plan row_plan(j, -1);
			float2 *z = zbuf + static_cast<size_t>(group) * L;
			for (int base = 0; base < n; base += warps * RG)
			{
				const int row = base + group;
				const bool active = row < n;
				float2 v[RM];
#pragma unroll
				for (int n1 = 0; n1 < RM; ++n1)
				{
					const int idx = RW * n1 + j;
					v[n1] = active ? *reinterpret_cast<const float2 *>(x + static_cast<int64_t>(row) * n + 2 * idx)
								   : make_float2(0.0f, 0.0f);
				}
				line_fft<RM, RW>::run(v, row_plan);
				if (active)
				{
#pragma unroll
					for (int k1 = 0; k1 < RM; ++k1)
						z[line_fft<RM, RW>::output_index(k1, j)] = v[k1];
				}
				__syncwarp();
				if (active)
				{
					for (int k = c0 + j; k < c1; k += RW)
					{
						const float2 zk = z[k == L ? 0 : k];
						const float2 zl = c_conj(z[k == 0 ? 0 : L - k]);
						const float2 e = make_float2(0.5f * (zk.x + zl.x), 0.5f * (zk.y + zl.y));
						const float2 d = c_sub(zk, zl);
						const float2 o = make_float2(0.5f * d.y, -0.5f * d.x); // (zk - conj zl) / 2i
						buf[static_cast<size_t>(row) * ncols + (k - c0)] = c_add(e, c_mul(split_twiddle[k], o));
					}
				}
				__syncwarp();
			}
		}
		__syncthreads();
		// Columns: complex lines of n over k_y.
		{
			const int group = warp * CG + lane / CW;
			const int j = lane % CW;
			const typename line_fft<CM, CW>::plan column_plan(j, -1);
			for (int base = 0; base < width; base += warps * CG)
			{
				const int col = base + group;
				const bool active = col < width;
				float2 v[CM];
#pragma unroll
				for (int n1 = 0; n1 < CM; ++n1)
					v[n1] = active ? buf[static_cast<size_t>(CW * n1 + j) * ncols + col] : make_float2(0.0f, 0.0f);
				line_fft<CM, CW>::run(v, column_plan);
				if (active)
				{
#pragma unroll
					for (int k1 = 0; k1 < CM; ++k1)
						buf[static_cast<size_t>(line_fft<CM, CW>::output_index(k1, j)) * ncols + col] = v[k1];
				}
			}
		}
		__syncthreads();
		ctf_epilogue_store(P, image, buf, ncols, c0, c1, coef);
		__syncthreads();
	}
}

// rfft2 at n = 128 with the whole half spectrum in shared memory (128 rows
// of 66 complex; the stride of 66 = 2 mod 16 keeps the column accesses of 8
// threads x 2 columns in a half-warp on distinct banks, and puts rows 4
// apart 16 banks apart).
//  - Rows: the packed complex line of 64 (x[2j] + i x[2j+1]) as 8 x 8, eight
//    threads a row: a DFT of 8 in registers over x[8 n1 + t], the twiddle
//    exp(-2 pi i t k1 / 64), an exchange through the row's own storage in a
//    skewed layout (element (k1, n2) at 8 k1 + (n2 + k1) mod 8, so neither
//    side of the exchange repeats a bank), a DFT of 8, then the split into
//    the 65 outputs.
//  - Columns: the outputs of k_x = 0 and k_x = 64 are real, so their two
//    columns travel as one complex column (DC + i Nyquist) in slot 0; the 64
//    column lines of 128 then run as 8 x 16, eight threads a column in two
//    passes of 32 columns, with the same skewed exchange, and slot 0 is
//    unpacked into k_x = 0 and 64 after.
//  - The CTF epilogue and the store as in the general kernel.
constexpr int r128_stride = 66;

template <bool STANDARDIZE>
__global__ void __launch_bounds__(fft_threads, 3) rfft2_128_kernel(const rfft2_launch P, const standardize_launch S,
	const resident_shape R)
{
	constexpr int n = 128, h = 65, RS = r128_stride;
	extern __shared__ float2 spec[]; // n x RS
	__shared__ float2 tw[n];         // exp(-2 pi i m / 128)
	__shared__ float coef[5];
	__shared__ double moment_scratch[3 * (fft_threads / 32)];
	const int64_t image = blockIdx.x;
	const float *x = P.in + image * static_cast<int64_t>(n) * n;
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	// The image into the rows of the spectrum buffer (row r at r * RS; 64
	// complex of 66), all of it in flight at once.
	for (int i = threadIdx.x; i < n * (n / 4); i += blockDim.x)
	{
		const int row = i >> 5, chunk = i & 31;
		const unsigned dst = static_cast<unsigned>(__cvta_generic_to_shared(spec + row * RS + 2 * chunk));
		asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(x + row * n + 4 * chunk) : "memory");
	}
	for (int m = threadIdx.x; m < n; m += blockDim.x)
		tw[m] = unit_root(m, n, -1);
	if (P.ctf_mode != 0 && threadIdx.x == 0)
		ctf_coefficients(P, image, coef);
	asm volatile("cp.async.wait_all;" ::: "memory");
	__syncthreads();
	if constexpr (STANDARDIZE)
	{
		// The image's rows are 33 chunks of 16 bytes apart in the buffer.
		standardize_resident<true>(S, R, reinterpret_cast<float4 *>(spec), image, moment_scratch,
			S.result ? reinterpret_cast<float4 *>(S.result + image * S.size) : nullptr);
		__syncthreads();
	}

	// Rows, 32 a pass: the two rows of a half-warp sit 4 apart (16 banks
	// apart): warp w, group g takes row (w mod 4) + 4 (g mod 2) + 8 (g / 2)
	// + 16 (w / 4).
	{
		const int t = lane & 7;
		const int g = lane >> 3;
		const int offset = (warp & 3) + 4 * (g & 1) + 8 * (g >> 1) + 16 * (warp >> 2);
		float2 tw_row[8];
#pragma unroll
		for (int k1 = 0; k1 < 8; ++k1)
			tw_row[k1] = tw[(2 * t * k1) & (n - 1)];
		for (int base = 0; base < n; base += 32)
		{
			const int row = base + offset;
			float2 *line = spec + row * RS;
			float2 v[8];
#pragma unroll
			for (int n1 = 0; n1 < 8; ++n1)
				v[n1] = line[8 * n1 + t];
			__syncwarp();
			small_dft<8>::run8(v, -1);
#pragma unroll
			for (int k1 = 1; k1 < 8; ++k1)
				v[k1] = c_mul(v[k1], tw_row[k1]);
#pragma unroll
			for (int k1 = 0; k1 < 8; ++k1)
				line[8 * k1 + ((t + k1) & 7)] = v[k1];
			__syncwarp();
#pragma unroll
			for (int n2 = 0; n2 < 8; ++n2)
				v[n2] = line[8 * t + ((n2 + t) & 7)];
			small_dft<8>::run8(v, -1); // v[k2] = Z[t + 8 k2]
			__syncwarp();
#pragma unroll
			for (int k2 = 0; k2 < 8; ++k2)
				line[t + 8 * k2] = v[k2];
			__syncwarp();
			// The split: out[k] = (Z[k] + conj Z[64-k]) / 2 + w^k (Z[k] - conj Z[64-k]) / 2i.
			float2 o[8];
#pragma unroll
			for (int m = 0; m < 8; ++m)
			{
				const int k = t + 8 * m;
				const float2 zk = line[k];
				const float2 zl = c_conj(line[(64 - k) & 63]);
				const float2 e = make_float2(0.5f * (zk.x + zl.x), 0.5f * (zk.y + zl.y));
				const float2 d = c_sub(zk, zl);
				o[m] = c_add(e, c_mul(tw[k], make_float2(0.5f * d.y, -0.5f * d.x)));
			}
			__syncwarp();
#pragma unroll
			for (int m = 0; m < 8; ++m)
				line[t + 8 * m] = o[m];
			if (t == 0)
			{
				// Slot 0: DC + i Nyquist, both real (Re Z0 + Im Z0, Re Z0 - Im Z0).
				const float2 z0 = v[0];
				line[0] = make_float2(z0.x + z0.y, z0.x - z0.y);
			}
			__syncwarp();
		}
	}
	__syncthreads();

	// Columns 0..63 as lines of 128 = 8 x 16, eight threads a column, two
	// passes of 32 columns.
	{
		const int t = lane & 7;
		const small_dft<16> dft16(-1);
#pragma unroll 1
		for (int pass = 0; pass < 2; ++pass)
		{
			const int col = 32 * pass + 4 * warp + (lane >> 3);
			float2 *c = spec + col;
			{
				float2 v[2][8];
#pragma unroll
				for (int a = 0; a < 2; ++a)
#pragma unroll
					for (int n1 = 0; n1 < 8; ++n1)
						v[a][n1] = c[(16 * n1 + t + 8 * a) * RS];
#pragma unroll
				for (int a = 0; a < 2; ++a)
				{
					small_dft<8>::run8(v[a], -1);
#pragma unroll
					for (int k1 = 1; k1 < 8; ++k1)
						v[a][k1] = c_mul(v[a][k1], tw[((t + 8 * a) * k1) & (n - 1)]);
				}
				__syncwarp();
#pragma unroll
				for (int a = 0; a < 2; ++a)
#pragma unroll
					for (int k1 = 0; k1 < 8; ++k1)
						c[(16 * k1 + ((t + 8 * a + k1) & 15)) * RS] = v[a][k1];
			}
			__syncwarp();
			float2 u[16];
#pragma unroll
			for (int n2 = 0; n2 < 16; ++n2)
				u[n2] = c[(16 * t + ((n2 + t) & 15)) * RS];
			dft16.run(u, -1);
			__syncwarp();
#pragma unroll
			for (int k2 = 0; k2 < 16; ++k2)
				c[(t + 8 * k2) * RS] = u[k2];
		}
	}
	__syncthreads();

	// Unpack slot 0: W = D + i Y, D[k] = (W[k] + conj W[-k]) / 2,
	// Y[k] = (W[k] - conj W[-k]) / 2i; D and Y are spectra of real columns,
	// so D[-k] = conj D[k]. Each thread takes the pair (k, 128 - k).
	for (int k = threadIdx.x; k <= n / 2; k += blockDim.x)
	{
		const int m = (n - k) & (n - 1);
		const float2 wk = spec[k * RS], wm = c_conj(spec[m * RS]);
		const float2 dk = make_float2(0.5f * (wk.x + wm.x), 0.5f * (wk.y + wm.y));
		const float2 diff = c_sub(wk, wm);
		const float2 yk = make_float2(0.5f * diff.y, -0.5f * diff.x);
		spec[k * RS] = dk;
		spec[k * RS + 64] = yk;
		if (m != k)
		{
			spec[m * RS] = c_conj(dk);
			spec[m * RS + 64] = c_conj(yk);
		}
	}
	__syncthreads();
	ctf_epilogue_store(P, image, spec, RS, 0, h, coef);
}

// rfft2 at n = 64 with the whole half spectrum in shared memory (64 rows of
// 34 complex: 16-byte aligned rows for the staging copies), the pattern of
// the n = 128 kernel at half the size:
//  - Rows: the packed complex line of 32 as 8 x 4, four threads a row: a DFT
//    of 8 in registers over x[4 n1 + t], the twiddle exp(-2 pi i t k1 / 32),
//    an exchange through the row's storage (element (k1, t) at
//    4 k1 + (t + k1) mod 4), two DFTs of 4 per thread, then the split into
//    the 33 outputs with k_x = 0 and 32 packed in slot 0.
//  - Columns: 32 lines of 64 as 8 x 8, eight threads a column, with the
//    skewed exchange; slot 0 is unpacked into k_x = 0 and 32 after.
//  - The CTF epilogue and the store as in the general kernel.
// At 40 registers six CTAs share an SM (48 warps); eight would spill.
constexpr int r64_stride = 34;

template <bool STANDARDIZE>
__global__ void __launch_bounds__(fft_threads, 6) rfft2_64_kernel(const rfft2_launch P, const standardize_launch S,
	const resident_shape R)
{
	constexpr int n = 64, h = 33, RS = r64_stride;
	__shared__ __align__(16) float2 spec[n * RS];
	__shared__ float2 tw[n]; // exp(-2 pi i m / 64)
	__shared__ float coef[5];
	__shared__ double moment_scratch[3 * (fft_threads / 32)];
	const int64_t image = blockIdx.x;
	const float *x = P.in + image * static_cast<int64_t>(n) * n;
	// The image into the rows of the spectrum buffer (row r at r * RS: 32
	// complex of 34), 16 bytes a copy.
	for (int i = threadIdx.x; i < n * (n / 4); i += blockDim.x)
	{
		const int row = i >> 4, chunk = i & 15;
		const unsigned dst = static_cast<unsigned>(__cvta_generic_to_shared(spec + row * RS + 2 * chunk));
		asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(x + row * n + 4 * chunk) : "memory");
	}
	for (int m = threadIdx.x; m < n; m += blockDim.x)
		tw[m] = unit_root(m, n, -1);
	if (P.ctf_mode != 0 && threadIdx.x == 0)
		ctf_coefficients(P, image, coef);
	asm volatile("cp.async.wait_all;" ::: "memory");
	__syncthreads();
	if constexpr (STANDARDIZE)
	{
		// The image's rows are 17 chunks of 16 bytes apart in the buffer.
		standardize_resident<true>(S, R, reinterpret_cast<float4 *>(spec), image, moment_scratch,
			S.result ? reinterpret_cast<float4 *>(S.result + image * S.size) : nullptr);
		__syncthreads();
	}

	// Rows: 64 rows x four threads, one pass.
	{
		const int t = threadIdx.x & 3;
		const int row = threadIdx.x >> 2;
		float2 *line = spec + row * RS;
		float2 v[8];
#pragma unroll
		for (int n1 = 0; n1 < 8; ++n1)
			v[n1] = line[4 * n1 + t];
		__syncwarp();
		small_dft<8>::run8(v, -1);
#pragma unroll
		for (int k1 = 1; k1 < 8; ++k1)
			v[k1] = c_mul(v[k1], tw[(2 * t * k1) & (n - 1)]);
#pragma unroll
		for (int k1 = 0; k1 < 8; ++k1)
			line[4 * k1 + ((t + k1) & 3)] = v[k1];
		__syncwarp();
		// Thread t takes k1 = t and t + 4: element (k1, t') at 4 k1 + (t' + k1) mod 4.
		float2 a[4], b[4];
#pragma unroll
		for (int tp = 0; tp < 4; ++tp)
		{
			a[tp] = line[4 * t + ((tp + t) & 3)];
			b[tp] = line[4 * (t + 4) + ((tp + t + 4) & 3)];
		}
		small_dft<4>::dft4(a[0], a[1], a[2], a[3], -1); // a[k2] = Z[t + 8 k2]
		small_dft<4>::dft4(b[0], b[1], b[2], b[3], -1); // b[k2] = Z[t + 4 + 8 k2]
		__syncwarp();
#pragma unroll
		for (int k2 = 0; k2 < 4; ++k2)
		{
			line[t + 8 * k2] = a[k2];
			line[t + 4 + 8 * k2] = b[k2];
		}
		__syncwarp();
		// The split: out[k] = (Z[k] + conj Z[32-k]) / 2 + w^k (Z[k] - conj Z[32-k]) / 2i, k = t + 4 m.
		float2 o[8];
#pragma unroll
		for (int m = 0; m < 8; ++m)
		{
			const int k = t + 4 * m;
			const float2 zk = line[k];
			if (k == 0)
				o[m] = make_float2(zk.x + zk.y, zk.x - zk.y); // slot 0: DC + i Nyquist
			else
			{
				const float2 zl = c_conj(line[32 - k]);
				const float2 e = make_float2(0.5f * (zk.x + zl.x), 0.5f * (zk.y + zl.y));
				const float2 d = c_sub(zk, zl);
				o[m] = c_add(e, c_mul(tw[k], make_float2(0.5f * d.y, -0.5f * d.x)));
			}
		}
		__syncwarp();
#pragma unroll
		for (int m = 0; m < 8; ++m)
			line[t + 4 * m] = o[m];
	}
	__syncthreads();

	// Columns 0..31 as lines of 64 = 8 x 8, eight threads a column, one pass.
	{
		const int t = threadIdx.x & 7;
		const int col = threadIdx.x >> 3;
		float2 *c = spec + col;
		float2 u[8];
#pragma unroll
		for (int n1 = 0; n1 < 8; ++n1)
			u[n1] = c[(8 * n1 + t) * RS];
		small_dft<8>::run8(u, -1);
#pragma unroll
		for (int k1 = 1; k1 < 8; ++k1)
			u[k1] = c_mul(u[k1], tw[(t * k1) & (n - 1)]);
		__syncwarp();
#pragma unroll
		for (int k1 = 0; k1 < 8; ++k1)
			c[(8 * k1 + ((t + k1) & 7)) * RS] = u[k1];
		__syncwarp();
#pragma unroll
		for (int n2 = 0; n2 < 8; ++n2)
			u[n2] = c[(8 * t + ((n2 + t) & 7)) * RS];
		small_dft<8>::run8(u, -1);
		__syncwarp();
#pragma unroll
		for (int k2 = 0; k2 < 8; ++k2)
			c[(t + 8 * k2) * RS] = u[k2];
	}
	__syncthreads();

	// Unpack slot 0 into k_x = 0 (slot 0) and k_x = 32 (slot 32), as at 128.
	for (int k = threadIdx.x; k <= n / 2; k += blockDim.x)
	{
		const int m = (n - k) & (n - 1);
		const float2 wk = spec[k * RS], wm = c_conj(spec[m * RS]);
		const float2 dk = make_float2(0.5f * (wk.x + wm.x), 0.5f * (wk.y + wm.y));
		const float2 diff = c_sub(wk, wm);
		const float2 yk = make_float2(0.5f * diff.y, -0.5f * diff.x);
		spec[k * RS] = dk;
		spec[k * RS + 32] = yk;
		if (m != k)
		{
			spec[m * RS] = c_conj(dk);
			spec[m * RS + 32] = c_conj(yk);
		}
	}
	__syncthreads();
	ctf_epilogue_store(P, image, spec, RS, 0, h, coef);
}

// rfft2 at n = 256 on a cluster of C CTAs (C = 4: 256 threads and about
// 104 KB each, two CTAs an SM). The half spectrum (256 x 129 complex,
// 264 KB) does not fit one CTA's shared memory; the CTAs of a cluster each
// hold 128 / C of its columns and exchange the row outputs through
// distributed shared memory, so every image is read once and written once.
//  - Rows: CTA r transforms image rows [256 r / C, 256 (r + 1) / C) as packed
//    complex lines of 128 (x[2j] + i x[2j+1]), 16 x 8 with eight threads a
//    line: a DFT of 16 in registers over x[8 n1 + t], the twiddle
//    exp(-2 pi i t k1 / 128), an exchange through the group's scratch in a
//    skewed layout, two DFTs of 8, then the split into the 129 outputs with
//    k_x = 0 and 128 (both real) packed as one complex value in slot 0.
//    Slot k goes to CTA k / (128 / C).
//  - A cluster barrier; then each CTA transforms its columns of 256 as
//    16 x 16 lines, sixteen threads a column (a half-warp), in place with
//    the skewed exchange. The row stride 128 / C + 1 (odd) keeps the sixteen
//    rows a half-warp touches on distinct banks.
//  - CTA 0 unpacks slot 0 into k_x = 0 (slot 0) and k_x = 128 (its padding slot).
//  - Each CTA stores its columns through the CTF epilogue.
template <int C>
struct r256_shape
{
	static constexpr int threads = 1024 / C;
	static constexpr int cols = 128 / C;        // column slots a CTA owns
	static constexpr int stride = cols + 1;     // column buffer row stride (complex), odd
	static constexpr int groups = threads / 8;  // rows in flight: eight threads each
	static constexpr int rows = 256 / C;        // image rows a CTA transforms, in two passes
	static constexpr int group_stride = 136;    // row scratch per group (complex): groups of a half-warp 16 banks apart
	static constexpr size_t smem = sizeof(float2) * (256 * stride + groups * group_stride);
	static_assert(rows == 2 * groups, "two passes of rows");
};

template <int C>
__device__ __forceinline__ void rfft2_256_store(const rfft2_launch &P, int64_t image, int rank, const float2 *buf,
	const float *coef)
{
	constexpr int n = 256, h = 129;
	using S = r256_shape<C>;
	// CTA r: k_x in [r cols, (r + 1) cols); CTA 0 also k_x = 128 (slot cols).
	const int width = rank == 0 ? S::cols + 1 : S::cols;
	const float inv_width = 1.0f / static_cast<float>(width);
	float2 *out = P.out + image * static_cast<int64_t>(n) * h;
	float *wout = P.weights ? P.weights + image * static_cast<int64_t>(n) * h : nullptr;
	for (int i = threadIdx.x; i < n * width; i += blockDim.x)
	{
		// The row of pair i: exact, as in ctf_epilogue_store.
		const int row = static_cast<int>((static_cast<float>(i) + 0.5f) * inv_width);
		const int slot = i - row * width;
		const int col = rank == 0 ? (slot < S::cols ? slot : 128) : rank * S::cols + slot;
		float2 X = buf[row * S::stride + slot];
		if (P.ctf_mode != 0)
		{
			const float ky = static_cast<float>(row < n / 2 ? row : row - n);
			const float kx = static_cast<float>(col);
			const float xx = kx * kx, yy = ky * ky, sq = xx + yy;
			const float ph = coef[0] * sq + coef[1] * (xx - yy) + coef[2] * (kx * ky) - coef[3] * (sq * sq) + coef[4];
			const float c = sin_reduced(ph);
			const float f = P.ctf_mode == 1 ? c : (c < 0.0f ? -1.0f : 1.0f);
			X.x *= f;
			X.y *= f;
			if (wout)
				wout[static_cast<int64_t>(row) * h + col] = P.ctf_mode == 1 ? c * c : fabsf(c);
		}
		out[static_cast<int64_t>(row) * h + col] = X;
	}
}

template <int C, bool STANDARDIZE>
__global__ void __cluster_dims__(C, 1, 1) __launch_bounds__(1024 / C, C / 2) rfft2_256_kernel(const rfft2_launch P,
	const standardize_launch SL, const resident_shape R)
{
	namespace cg = cooperative_groups;
	using S = r256_shape<C>;
	constexpr int n = 256;
	extern __shared__ float2 r256_smem[];
	float2 *colbuf = r256_smem;                  // 256 rows x S::stride
	float2 *scratch = colbuf + n * S::stride;    // S::groups x S::group_stride
	__shared__ float2 tw[n];                     // exp(-2 pi i m / 256)
	__shared__ float coef[5];
	__shared__ double moment_scratch[3 * (1024 / C / 32)];
	__shared__ double slots[2][C][3]; // per moment pass, per rank: count, sum, squares
	cg::cluster_group cluster = cg::this_cluster();
	const int rank = static_cast<int>(cluster.block_rank());
	const int64_t image = blockIdx.x / C;
	const float *x = P.in + image * static_cast<int64_t>(n) * n;
	for (int m = threadIdx.x; m < n; m += blockDim.x)
		tw[m] = unit_root(m, n, -1);
	if (P.ctf_mode != 0 && threadIdx.x == 0)
		ctf_coefficients(P, image, coef);
	float2 *owner[C];
#pragma unroll
	for (int r = 0; r < C; ++r)
		owner[r] = cluster.map_shared_rank(colbuf, r);
	// Every CTA runs before any writes into another's shared memory.
	cluster.sync();

	// The standardization of the image: CTA r takes the moments of its own
	// rows [64 r, 64 r + 64) straight from global memory, in the thread and
	// chunk order of the standardization's cluster kernel, and the shares
	// meet in rank order; the rows are then standardized as they are loaded.
	float mean_f = 0.0f, scale_f = 1.0f, lower_f = 0.0f, upper_f = 0.0f;
	uint64_t key = 0, counter0 = 0;
	float2 *std_out = nullptr;
	if constexpr (STANDARDIZE)
	{
		const int first = static_cast<int>(static_cast<int64_t>(rank) * R.chunks / C);
		const int end = static_cast<int>(static_cast<int64_t>(rank + 1) * R.chunks / C);
		const float4 *share = reinterpret_cast<const float4 *>(x) + first;
		double mean = 0.0, scale = 1.0;
		finalize(cluster_moments<C>(cluster, slots[0], rank,
					 block_sum(resident_moments<false>(share, R, first, end, 0.0, 1.0, 0.0, 0.0), moment_scratch)),
			mean, scale);
		if (SL.lower != -INFINITY || SL.upper != INFINITY)
			finalize(cluster_moments<C>(cluster, slots[1], rank,
						 block_sum(resident_moments<true>(share, R, first, end, mean, scale, SL.lower, SL.upper),
							 moment_scratch)),
				mean, scale);
		if (SL.statistics && rank == 0 && threadIdx.x == 0)
		{
			SL.statistics[2 * image] = mean;
			SL.statistics[2 * image + 1] = scale;
		}
		mean_f = static_cast<float>(mean);
		scale_f = static_cast<float>(scale);
		lower_f = static_cast<float>(SL.lower);
		upper_f = static_cast<float>(SL.upper);
		key = SL.keys[image / SL.images_per_key];
		counter0 = static_cast<uint64_t>(image % SL.images_per_key) * static_cast<uint64_t>(SL.size);
		if (SL.result)
			std_out = reinterpret_cast<float2 *>(SL.result + image * SL.size);
	}

	// Rows: S::groups groups of eight threads, two passes.
	{
		const int g = threadIdx.x >> 3, t = threadIdx.x & 7;
		float2 *sc = scratch + g * S::group_stride;
		const small_dft<16> dft16(-1);
#pragma unroll 1
		for (int pass = 0; pass < 2; ++pass)
		{
			const int row = S::rows * rank + S::groups * pass + g;
			const float2 *line = reinterpret_cast<const float2 *>(x + static_cast<int64_t>(row) * n);
			float2 v[16];
#pragma unroll
			for (int n1 = 0; n1 < 16; ++n1)
				v[n1] = line[8 * n1 + t];
			if constexpr (STANDARDIZE)
			{
#pragma unroll
				for (int n1 = 0; n1 < 16; ++n1)
				{
					const int pair = row * (n / 2) + 8 * n1 + t; // elements 2 pair and 2 pair + 1
					v[n1] = standardize_pair(v[n1], mean_f, scale_f, lower_f, upper_f, key,
						counter0 + 2 * static_cast<uint64_t>(pair));
					if (std_out)
						__stcs(std_out + pair, v[n1]);
				}
			}
			dft16.run(v, -1);
#pragma unroll
			for (int k1 = 1; k1 < 16; ++k1)
				v[k1] = c_mul(v[k1], tw[(2 * t * k1) & (n - 1)]);
#pragma unroll
			for (int k1 = 0; k1 < 16; ++k1)
				sc[8 * k1 + ((t + k1) & 7)] = v[k1];
			__syncwarp();
			// Thread t takes k1 = t and t + 8: element (k1, t') sits at 8 k1 + (t' + k1) mod 8.
			float2 a[8], b[8];
#pragma unroll
			for (int tp = 0; tp < 8; ++tp)
			{
				a[tp] = sc[8 * t + ((tp + t) & 7)];
				b[tp] = sc[8 * (t + 8) + ((tp + t + 8) & 7)];
			}
			small_dft<8>::run8(a, -1); // a[k2] = Z[t + 16 k2]
			small_dft<8>::run8(b, -1); // b[k2] = Z[t + 8 + 16 k2]
			__syncwarp();
#pragma unroll
			for (int k2 = 0; k2 < 8; ++k2)
			{
				sc[t + 16 * k2] = a[k2];
				sc[t + 8 + 16 * k2] = b[k2];
			}
			__syncwarp();
			// The split: out[k] = (Z[k] + conj Z[128-k]) / 2 + w^k (Z[k] - conj Z[128-k]) / 2i,
			// k = t + 8 m; slot 0 holds DC + i Nyquist. Slot k belongs to CTA m / (16 / C).
#pragma unroll
			for (int m = 0; m < 16; ++m)
			{
				const int k = t + 8 * m;
				const float2 zk = sc[k];
				float2 o;
				if (k == 0)
					o = make_float2(zk.x + zk.y, zk.x - zk.y);
				else
				{
					const float2 zl = c_conj(sc[128 - k]);
					const float2 e = make_float2(0.5f * (zk.x + zl.x), 0.5f * (zk.y + zl.y));
					const float2 d = c_sub(zk, zl);
					o = c_add(e, c_mul(tw[k], make_float2(0.5f * d.y, -0.5f * d.x)));
				}
				owner[m / (16 / C)][row * S::stride + (k % S::cols)] = o;
			}
			__syncwarp(); // the group's scratch is reused by the next pass
		}
	}
	// Every row output has landed in its owner's buffer.
	cluster.sync();

	// Columns: S::cols lines of 256 = 16 x 16, sixteen threads a column, two passes.
	{
		const int t = threadIdx.x & 15;
		const small_dft<16> dft16(-1);
#pragma unroll 1
		for (int pass = 0; pass < 2; ++pass)
		{
			const int col = (S::cols / 2) * pass + (threadIdx.x >> 4);
			float2 *c = colbuf + col;
			float2 u[16];
#pragma unroll
			for (int n1 = 0; n1 < 16; ++n1)
				u[n1] = c[(16 * n1 + t) * S::stride];
			dft16.run(u, -1);
#pragma unroll
			for (int k1 = 1; k1 < 16; ++k1)
				u[k1] = c_mul(u[k1], tw[(t * k1) & (n - 1)]);
			__syncwarp();
#pragma unroll
			for (int k1 = 0; k1 < 16; ++k1)
				c[(16 * k1 + ((t + k1) & 15)) * S::stride] = u[k1];
			__syncwarp();
#pragma unroll
			for (int n2 = 0; n2 < 16; ++n2)
				u[n2] = c[(16 * t + ((n2 + t) & 15)) * S::stride];
			dft16.run(u, -1);
			__syncwarp();
#pragma unroll
			for (int k2 = 0; k2 < 16; ++k2)
				c[(t + 16 * k2) * S::stride] = u[k2];
		}
	}
	__syncthreads();

	if (rank == 0)
	{
		// Unpack slot 0: W = D + i Y with D, Y the spectra of the real columns
		// k_x = 0 and 128: D[k] = (W[k] + conj W[-k]) / 2, Y[k] = (W[k] - conj W[-k]) / 2i.
		for (int k = threadIdx.x; k <= n / 2; k += blockDim.x)
		{
			const int m = (n - k) & (n - 1);
			const float2 wk = colbuf[k * S::stride], wm = c_conj(colbuf[m * S::stride]);
			const float2 dk = make_float2(0.5f * (wk.x + wm.x), 0.5f * (wk.y + wm.y));
			const float2 diff = c_sub(wk, wm);
			const float2 yk = make_float2(0.5f * diff.y, -0.5f * diff.x);
			colbuf[k * S::stride] = dk;
			colbuf[k * S::stride + S::cols] = yk;
			if (m != k)
			{
				colbuf[m * S::stride] = c_conj(dk);
				colbuf[m * S::stride + S::cols] = c_conj(yk);
			}
		}
		__syncthreads();
	}
	rfft2_256_store<C>(P, image, rank, colbuf, coef);
}

// The cluster size of the 256 R2C.
constexpr int r256_cluster = 4;

struct irfft2_launch
{
	const float2 *in;
	float *out;
	int64_t batch;
	int n, h, L;
};

template <int RM, int RW, int CM, int CW>
__global__ void __launch_bounds__(fft_threads) irfft2_kernel(const irfft2_launch P)
{
	extern __shared__ float2 smem[];
	__shared__ float2 split_twiddle[max_half_spectrum]; // exp(2 pi i k / n), k < h
	constexpr int RG = 32 / RW, CG = 32 / CW;
	const int n = P.n, h = P.h, L = P.L;
	float2 *buf = smem; // n x h
	for (int k = threadIdx.x; k < h; k += blockDim.x)
		split_twiddle[k] = unit_root(k == n ? 0 : k, n, 1);
	const int64_t image = blockIdx.x;
	const float2 *in = P.in + image * static_cast<int64_t>(n) * h;
	float *out = P.out + image * static_cast<int64_t>(n) * n;
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	const int warps = blockDim.x >> 5;
	for (int i = threadIdx.x; i < n * h; i += blockDim.x)
		buf[i] = in[i];
	__syncthreads();
	// Columns: inverse complex lines of n.
	{
		const int group = warp * CG + lane / CW;
		const int j = lane % CW;
		const typename line_fft<CM, CW>::plan column_plan(j, 1);
		for (int base = 0; base < h; base += warps * CG)
		{
			const int col = base + group;
			const bool active = col < h;
			float2 v[CM];
#pragma unroll
			for (int n1 = 0; n1 < CM; ++n1)
				v[n1] = active ? buf[static_cast<size_t>(CW * n1 + j) * h + col] : make_float2(0.0f, 0.0f);
			line_fft<CM, CW>::run(v, column_plan);
			if (active)
			{
#pragma unroll
				for (int k1 = 0; k1 < CM; ++k1)
					buf[static_cast<size_t>(line_fft<CM, CW>::output_index(k1, j)) * h + col] = v[k1];
			}
		}
	}
	__syncthreads();
	// Rows: C2R. Z[k] = E[k] + i O[k] with E = (X[k] + conj X[L-k]) / 2 and
	// O = (X[k] - conj X[L-k]) / 2 * exp(2 pi i k / n); the line of n/2 is
	// inverted and its parts are the even and odd reals.
	{
		const int group = warp * RG + lane / RW;
		const int j = lane % RW;
		const typename line_fft<RM, RW>::plan row_plan(j, 1);
		const float scale = 1.0f / (static_cast<float>(n) * static_cast<float>(L));
		for (int base = 0; base < n; base += warps * RG)
		{
			const int row = base + group;
			const bool active = row < n;
			float2 v[RM];
#pragma unroll
			for (int n1 = 0; n1 < RM; ++n1)
			{
				const int k = RW * n1 + j;
				float2 r = make_float2(0.0f, 0.0f);
				if (active)
				{
					float2 a = buf[static_cast<size_t>(row) * h + k];
					float2 b = buf[static_cast<size_t>(row) * h + (L - k)];
					if (k == 0)
					{
						a.y = 0.0f;
						b.y = 0.0f;
					}
					const float2 bc = c_conj(b);
					const float2 e = make_float2(0.5f * (a.x + bc.x), 0.5f * (a.y + bc.y));
					const float2 d = make_float2(0.5f * (a.x - bc.x), 0.5f * (a.y - bc.y));
					const float2 o = c_mul(d, split_twiddle[k]);
					r = make_float2(e.x - o.y, e.y + o.x); // E + i O
				}
				v[n1] = r;
			}
			line_fft<RM, RW>::run(v, row_plan);
			if (active)
			{
#pragma unroll
				for (int k1 = 0; k1 < RM; ++k1)
				{
					const int idx = line_fft<RM, RW>::output_index(k1, j);
					*reinterpret_cast<float2 *>(out + static_cast<int64_t>(row) * n + 2 * idx) =
						make_float2(v[k1].x * scale, v[k1].y * scale);
				}
			}
		}
	}
}

// The 256 R2C on its cluster, with or without the standardization of the image.
template <bool STANDARDIZE>
void launch_rfft2_256(const rfft2_launch &P, const standardize_launch &SL, const resident_shape &R,
	cudaStream_t stream)
{
	using S = r256_shape<r256_cluster>;
	constexpr auto kernel = rfft2_256_kernel<r256_cluster, STANDARDIZE>;
	check_cuda(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(S::smem)),
		"rfft2 attributes");
	kernel<<<static_cast<unsigned>(r256_cluster * P.batch), S::threads, S::smem, stream>>>(P, SL, R);
	check_cuda(cudaGetLastError(), "rfft2 launch");
}

// The R2C kernels that hold a whole 64 or 128 image in shared memory, with
// or without the standardization of the staged image.
template <bool STANDARDIZE>
void launch_resident_rfft2(const rfft2_launch &P, const standardize_launch &S, const resident_shape &R,
	cudaStream_t stream)
{
	if (P.n == 128)
	{
		const size_t smem = sizeof(float2) * 128 * r128_stride;
		check_cuda(cudaFuncSetAttribute(rfft2_128_kernel<STANDARDIZE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
					   static_cast<int>(smem)),
			"rfft2 attributes");
		rfft2_128_kernel<STANDARDIZE><<<static_cast<unsigned>(P.batch), fft_threads, smem, stream>>>(P, S, R);
	}
	else
	{
		rfft2_64_kernel<STANDARDIZE><<<static_cast<unsigned>(P.batch), fft_threads, 0, stream>>>(P, S, R);
	}
	check_cuda(cudaGetLastError(), "rfft2 launch");
}

struct rfft2_sizes
{
	template <int RM, int RW, int CM, int CW>
	static void launch(const rfft2_launch &P, cudaStream_t stream)
	{
		if (P.n == 128 && reinterpret_cast<uintptr_t>(P.in) % 16 == 0)
		{
			launch_resident_rfft2<false>(P, standardize_launch{}, resident_shape{}, stream);
			return;
		}
		if (P.n == 64 && reinterpret_cast<uintptr_t>(P.in) % 16 == 0)
		{
			launch_resident_rfft2<false>(P, standardize_launch{}, resident_shape{}, stream);
			return;
		}
		if (P.n == 256 && reinterpret_cast<uintptr_t>(P.in) % 8 == 0 && P.batch <= (1LL << 29))
		{
			launch_rfft2_256<false>(P, standardize_launch{}, resident_shape{}, stream);
			return;
		}
		const size_t smem = sizeof(float2) * (static_cast<size_t>(P.n) * P.ncols +
			static_cast<size_t>(fft_threads / 32) * (32 / RW) * P.L);
		auto kernel = rfft2_kernel<RM, RW, CM, CW>;
		check_cuda(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)),
			"rfft2 attributes");
		kernel<<<static_cast<unsigned>(P.batch), fft_threads, smem, stream>>>(P);
		check_cuda(cudaGetLastError(), "rfft2 launch");
	}
};

struct irfft2_sizes
{
	template <int RM, int RW, int CM, int CW>
	static void launch(const irfft2_launch &P, cudaStream_t stream)
	{
		const size_t smem = sizeof(float2) * static_cast<size_t>(P.n) * P.h;
		auto kernel = irfft2_kernel<RM, RW, CM, CW>;
		check_cuda(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)),
			"irfft2 attributes");
		kernel<<<static_cast<unsigned>(P.batch), fft_threads, smem, stream>>>(P);
		check_cuda(cudaGetLastError(), "irfft2 launch");
	}
};

template <typename Sizes, typename Launch>
bool launch_for_extent(int n, const Launch &P, cudaStream_t stream)
{
	switch (n)
	{
	case 32:
		Sizes::template launch<1, 16, 1, 32>(P, stream);
		return true;
	case 64:
		Sizes::template launch<1, 32, 2, 32>(P, stream);
		return true;
	case 96:
		Sizes::template launch<3, 16, 3, 32>(P, stream);
		return true;
	case 128:
		Sizes::template launch<2, 32, 4, 32>(P, stream);
		return true;
	case 160:
		Sizes::template launch<5, 16, 5, 32>(P, stream);
		return true;
	case 192:
		Sizes::template launch<3, 32, 6, 32>(P, stream);
		return true;
	case 200:
		Sizes::template launch<25, 4, 25, 8>(P, stream);
		return true;
	case 256:
		Sizes::template launch<4, 32, 8, 32>(P, stream);
		return true;
	default:
		return false;
	}
}

bool supported_extent(int64_t n)
{
	switch (n)
	{
	case 32:
	case 64:
	case 96:
	case 128:
	case 160:
	case 192:
	case 200:
	case 256:
		return true;
	default:
		return false;
	}
}

int row_lanes(int n)
{
	switch (n)
	{
	case 32:
	case 96:
	case 160:
		return 16;
	case 200:
		return 4;
	default:
		return 32;
	}
}

} // anonymous namespace
} // namespace rexlib_b200

using namespace rexlib_b200;

namespace
{

// The launch of an rfft2 of `batch` checked images of n (a supported extent),
// with the epilogue checked as the reference checks ctf_optics and the pixel
// size.
rfft2_launch rfft2_plan(void *out, const float *in, int64_t batch, int64_t n,
	const rexlib_b200_ctf_epilogue *epilogue)
{
	rfft2_launch P{};
	P.in = in;
	P.out = static_cast<float2 *>(out);
	P.batch = batch;
	P.n = static_cast<int>(n);
	P.h = P.n / 2 + 1;
	P.L = P.n / 2;
	const size_t zbytes = sizeof(float2) * static_cast<size_t>(fft_threads / 32) * (32 / row_lanes(P.n)) * P.L;
	const int max_cols = static_cast<int>((fft_smem_budget - zbytes) / (sizeof(float2) * P.n));
	const int phases = (P.h + max_cols - 1) / max_cols;
	P.ncols = (P.h + phases - 1) / phases;
	if (epilogue && epilogue->mode != 0)
	{
		require(epilogue->mode == 1 || epilogue->mode == 2, "unknown CTF epilogue mode");
		require(epilogue->ctf != nullptr, "null ctf parameters");
		require(epilogue->ctf_stride >= 0, "negative ctf stride");
		const auto &o = epilogue->optics;
		require(std::isfinite(o.voltage) && o.voltage > 0.0, "ctf_optics: the voltage must be finite and positive");
		require(std::isfinite(o.spherical_aberration), "ctf_optics: the spherical aberration must be finite");
		require(o.amplitude_contrast >= 0.0 && o.amplitude_contrast < 1.0,
			"ctf_optics: the amplitude contrast must lie in [0, 1)");
		require(std::isfinite(epilogue->pixel_size) && epilogue->pixel_size > 0.0,
			"the pixel size must be finite and positive");
		P.ctf_mode = epilogue->mode;
		P.ctf = epilogue->ctf;
		P.ctf_stride = epilogue->ctf_stride;
		P.voltage = epilogue->voltage;
		P.voltage_default = o.voltage;
		P.aberration = o.spherical_aberration * 1e7;
		P.phase_offset = std::asin(o.amplitude_contrast);
		const double fs = 1.0 / (static_cast<double>(n) * epilogue->pixel_size);
		P.frequency_scale_sq = fs * fs;
		P.weights = epilogue->weights;
	}
	return P;
}

} // anonymous namespace

extern "C" int32_t rexlib_b200_rfft2(void *out, const float *in, int64_t batch, int64_t n,
	const rexlib_b200_ctf_epilogue *epilogue, void *stream)
{
	return guarded([&] {
		require(batch >= 0, "negative batch");
		if (!supported_extent(n))
			fail(REXLIB_B200_UNSUPPORTED, "rfft2 runs square images of 32, 64, 96, 128, 160, 192, 200 or 256");
		if (batch == 0)
			return;
		require(out && in, "null operand");
		require(reinterpret_cast<uintptr_t>(in) % 8 == 0 && reinterpret_cast<uintptr_t>(out) % 8 == 0,
			"operands must be 8-byte aligned");
		require(batch <= 0x7fffffffLL, "too many images in one call");
		const rfft2_launch P = rfft2_plan(out, in, batch, n, epilogue);
		launch_for_extent<rfft2_sizes>(P.n, P, as_stream(stream));
	});
}

extern "C" int32_t rexlib_b200_standardize_rfft2(void *out, const rexlib_b200_standardization *standardization,
	const rexlib_b200_ctf_epilogue *epilogue, void *stream)
{
	return guarded([&] {
		standardize_launch S;
		if (!standardize_plan(standardization, S))
			return;
		if (S.rank != 2 || S.dims[0] != S.dims[1] || (S.dims[0] != 64 && S.dims[0] != 128 && S.dims[0] != 256))
			fail(REXLIB_B200_UNSUPPORTED, "standardize_rfft2 runs square 2D images of 64, 128 or 256");
		require(out != nullptr, "null operand");
		require(reinterpret_cast<uintptr_t>(S.value) % 16 == 0 && reinterpret_cast<uintptr_t>(S.result) % 16 == 0,
			"the images and the standardized images must be 16-byte aligned");
		require(reinterpret_cast<uintptr_t>(out) % 8 == 0, "the spectra must be 8-byte aligned");
		const int n = S.dims[0];
		const rfft2_launch P = rfft2_plan(out, S.value, S.batch, n, epilogue);
		if (n == 256)
		{
			require(S.batch <= (1LL << 29), "too many images in one call");
			// The image's rows are 64 chunks of 16 bytes apart in global memory.
			launch_rfft2_256<true>(P, S, resident_shape_of(S, n / 4), as_stream(stream));
		}
		else
		{
			launch_resident_rfft2<true>(P, S, resident_shape_of(S, (n == 128 ? r128_stride : r64_stride) / 2),
				as_stream(stream));
		}
	});
}

extern "C" int32_t rexlib_b200_irfft2(float *out, const void *in, int64_t batch, int64_t n, void *stream)
{
	return guarded([&] {
		require(batch >= 0, "negative batch");
		if (!supported_extent(n) || n > 200)
			fail(REXLIB_B200_UNSUPPORTED, "irfft2 runs square images of 32, 64, 96, 128, 160, 192 or 200");
		if (batch == 0)
			return;
		require(out && in, "null operand");
		require(reinterpret_cast<uintptr_t>(in) % 8 == 0 && reinterpret_cast<uintptr_t>(out) % 8 == 0,
			"operands must be 8-byte aligned");
		require(batch <= 0x7fffffffLL, "too many images in one call");
		irfft2_launch P{};
		P.in = static_cast<const float2 *>(in);
		P.out = out;
		P.batch = batch;
		P.n = static_cast<int>(n);
		P.h = P.n / 2 + 1;
		P.L = P.n / 2;
		launch_for_extent<irfft2_sizes>(P.n, P, as_stream(stream));
	});
}
