// Slice-parallel insertion: one CTA settles one slice and scatters each of
// its samples straight into the accumulators with global reductions.
//
// It runs every window, both volume parities and every sample weight, and
// serves shapes the tiled kernel does not take (odd N, Kaiser-Bessel,
// non-square scaling) and the float64 insertions (slice_insertion_rules.hpp:
// 86-90 admits float32 and float64, one type for every operand). Per-
// contribution values are computed with the reference's operations in the
// element type T and in the reference's order (row_insertion_kernel.inl:
// 139-360), so results differ from the CPU only by the order of the sums.
#include "insertion.cuh"

namespace rexlib_b200
{
namespace
{

__device__ __forceinline__ void red_add2(float2 *address, float re, float im)
{
	asm volatile("red.global.add.v2.f32 [%0], {%1, %2};" ::"l"(address), "f"(re), "f"(im) : "memory");
}

__device__ __forceinline__ void red_add(float *address, float value)
{
	asm volatile("red.global.add.f32 [%0], %1;" ::"l"(address), "f"(value) : "memory");
}

__device__ __forceinline__ void red_add2(double2 *address, double re, double im)
{
	asm volatile("red.global.add.f64 [%0], %1;" ::"l"(&address->x), "d"(re) : "memory");
	asm volatile("red.global.add.f64 [%0], %1;" ::"l"(&address->y), "d"(im) : "memory");
}

__device__ __forceinline__ void red_add(double *address, double value)
{
	asm volatile("red.global.add.f64 [%0], %1;" ::"l"(address), "d"(value) : "memory");
}

__device__ __forceinline__ float sine(float x) { return sinf(x); }
__device__ __forceinline__ double sine(double x) { return sin(x); }

template <typename T>
__device__ __forceinline__ complex_t<T> make_complex(double re, double im);
template <>
__device__ __forceinline__ float2 make_complex<float>(double re, double im)
{
	return make_float2(static_cast<float>(re), static_cast<float>(im));
}
template <>
__device__ __forceinline__ double2 make_complex<double>(double re, double im)
{
	return make_double2(re, im);
}

template <typename T>
struct slice_settled
{
	double xs[3];
	double ys[3];
	T c_radial, c_axial, c_diag, c_aberr, c_phase;
	int last_shell;
};

template <typename T, typename KB, int PROFILE, int KIND, bool ODD>
__global__ void __launch_bounds__(256) insert_scatter_kernel(
	const insertion_launch_of<T> L, const __grid_constant__ KB kb_by_value)
{
	using C = complex_t<T>;
	extern __shared__ double4 shared_raw[];
	C *x_phase = reinterpret_cast<C *>(shared_raw);
	C *y_phase = x_phase + L.h;
	C *volume_phase = y_phase + L.n;                      // N entries when ODD
	T *radial = reinterpret_cast<T *>(volume_phase + (ODD ? L.big : 0));
	__shared__ slice_settled<T> settled;
	__shared__ int last_shell_shared;

	const KB *kb = &kb_by_value;
	const int64_t index = blockIdx.x;
	const int64_t v = index / L.particles;
	const int64_t p = index % L.particles;
	const int n = L.n, h = L.h;
	const C *slice = L.slices + (v * L.slice_stride_v + p * L.slice_stride_p) * (int64_t)n * h;
	const T *tr = L.transforms + (v * L.transform_stride_v + p * L.transform_stride_p) * 12;
	const T *rad = L.radial + (v * L.radial_stride_v + p * L.radial_stride_p) * h;

	// Settle the slice (slice_insertion_functor.inl:161-270).
	if (threadIdx.x == 0)
		last_shell_shared = -1;
	__syncthreads();
	for (int s = threadIdx.x; s < h; s += blockDim.x)
	{
		const T r = rad[s];
		radial[s] = r;
		if (r != T(0))
			atomicMax(&last_shell_shared, s);
	}
	const double centre = static_cast<double>(n / 2);
	{
		const double sx = 2.0 * pi * (centre + static_cast<double>(tr[3])) / static_cast<double>(n);
		for (int j = threadIdx.x; j < h; j += blockDim.x)
		{
			double sn, cs;
			sincos(sx * static_cast<double>(j), &sn, &cs);
			x_phase[j] = make_complex<T>(cs, sn);
		}
		const double sy = 2.0 * pi * (centre + static_cast<double>(tr[7])) / static_cast<double>(n);
		for (int j = threadIdx.x; j < n; j += blockDim.x)
		{
			const double f = j <= n / 2 ? static_cast<double>(j) : static_cast<double>(j - n);
			double sn, cs;
			sincos(sy * f, &sn, &cs);
			y_phase[j] = make_complex<T>(cs, sn);
		}
	}
	if constexpr (ODD)
	{
		const int half = L.big / 2;
		const double s = 2.0 * pi * (-static_cast<double>(half)) / static_cast<double>(L.big);
		for (int j = threadIdx.x; j < L.big; j += blockDim.x)
		{
			const double f = j <= half ? static_cast<double>(j) : static_cast<double>(j - L.big);
			double sn, cs;
			sincos(s * f, &sn, &cs);
			volume_phase[j] = make_complex<T>(cs, sn);
		}
	}
	if (threadIdx.x == 0)
	{
		const double scale = static_cast<double>(L.big) / static_cast<double>(n);
		for (int a = 0; a < 3; ++a)
		{
			settled.xs[a] = static_cast<double>(tr[a]) * scale;
			settled.ys[a] = static_cast<double>(tr[4 + a]) * scale;
		}
		if constexpr (KIND == static_cast<int>(weight_kind::ctf))
		{
			const T *ctf = L.extra + (v * L.extra_stride_v + p * L.extra_stride_p) * 4;
			const double du = ctf[0], dv = ctf[1], angle = ctf[2], shift = ctf[3];
			const double dscale = pi * L.ctf_wavelength * L.ctf_frequency_scale_sq;
			const double hd = 0.5 * (du - dv);
			double s2, c2;
			sincos(2.0 * angle, &s2, &c2);
			settled.c_phase = static_cast<T>(shift + L.ctf_phase_offset);
			settled.c_radial = static_cast<T>(dscale * 0.5 * (du + dv));
			settled.c_axial = static_cast<T>(dscale * hd * c2);
			settled.c_diag = static_cast<T>(2.0 * dscale * hd * s2);
			const double wl = L.ctf_wavelength;
			settled.c_aberr = static_cast<T>(0.5 * pi * L.ctf_aberration * wl * wl * wl *
				L.ctf_frequency_scale_sq * L.ctf_frequency_scale_sq);
		}
	}
	__syncthreads();
	const int last_shell = last_shell_shared;
	if (last_shell < 0)
		return;

	const T *weights = nullptr;
	if constexpr (KIND == static_cast<int>(weight_kind::spectrum))
		weights = L.extra + (v * L.extra_stride_v + p * L.extra_stride_p) * (int64_t)n * h;

	C *num = L.numerator + v * (int64_t)L.big * L.big * L.big_h;
	T *den = L.denominator + v * (int64_t)L.big * L.big * L.big_h;
	const int half = L.big / 2;
	const int big = L.big;
	const int H = L.big_h;

	// Rows and columns (slice_insertion_functor.inl:339-393).
	const double radius = static_cast<double>(last_shell) + 0.5;
	const int last_column = h - (n % 2 == 0 ? 2 : 1);
	const int widest = min(last_column, static_cast<int>(radius));
	const int highest_row = n % 2 == 0 ? n / 2 - 1 : n / 2;
	const int first_row = max(-highest_row, -widest);
	const int last_row = min(highest_row, widest);
	bool finite = true;
	for (int a = 0; a < 3; ++a)
		finite = finite && isfinite(settled.xs[a]) && isfinite(settled.ys[a]);
	if (!finite)
		return;
	const T step[3] = {static_cast<T>(settled.xs[0]), static_cast<T>(settled.xs[1]), static_cast<T>(settled.xs[2])};

	const int warp = threadIdx.x >> 5;
	const int lane = threadIdx.x & 31;
	const int warps = blockDim.x >> 5;
	const int taps = taps_of<PROFILE>(kb);
	constexpr int WC = weight_capacity<PROFILE>();

	for (int ky = first_row + warp; ky <= last_row; ky += warps)
	{
		const double kyv = static_cast<double>(ky);
		const double reach = radius * radius - kyv * kyv;
		if (reach < 0.0)
			continue;
		const int last = min(widest, static_cast<int>(sqrt(reach)));
		const T base[3] = {static_cast<T>(kyv * settled.ys[0]), static_cast<T>(kyv * settled.ys[1]),
			static_cast<T>(kyv * settled.ys[2])};
		const int srow = ky < 0 ? ky + n : ky;
		const C yph = y_phase[srow];
		const C *row = slice + (int64_t)srow * h;
		for (int kx = lane; kx <= last; kx += 32)
		{
			const int shell = shell_of(kx, ky);
			const T r = shell <= last_shell ? radial[shell] : T(0);
			if (r == T(0))
				continue;
			T wnum = T(1), wden = T(1);
			if constexpr (KIND == static_cast<int>(weight_kind::ctf))
			{
				const T kxt = static_cast<T>(kx), kyt = static_cast<T>(ky);
				const T xx = fmul(kxt, kxt);
				const T yy = fmul(kyt, kyt);
				const T sq = fadd(xx, yy);
				T ph = fmul(settled.c_radial, sq);
				ph = fadd(ph, fmul(settled.c_axial, fsub(xx, yy)));
				ph = fadd(ph, fmul(settled.c_diag, fmul(kxt, kyt)));
				ph = fsub(ph, fmul(settled.c_aberr, fmul(sq, sq)));
				ph = fadd(ph, settled.c_phase);
				wnum = sine(ph);
				wden = fmul(wnum, wnum);
			}
			else if constexpr (KIND == static_cast<int>(weight_kind::spectrum))
			{
				wden = weights[(int64_t)srow * h + kx];
			}
			const C sample = row[kx];
			const C xph = x_phase[kx];
			const T shre = fsub(fmul(sample.x, xph.x), fmul(sample.y, xph.y));
			const T shim = fadd(fmul(sample.x, xph.y), fmul(sample.y, xph.x));
			const T vre0 = fsub(fmul(shre, yph.x), fmul(shim, yph.y));
			const T vim0 = fadd(fmul(shre, yph.y), fmul(shim, yph.x));
			const T sc = fmul(r, wnum);
			const T count = fmul(r, wden);
			const T kxf = static_cast<T>(kx);
			const T cpos[3] = {fadd(base[0], fmul(kxf, step[0])), fadd(base[1], fmul(kxf, step[1])),
				fadd(base[2], fmul(kxf, step[2]))};

			for (int sgn = 0; sgn < (kx >= 1 ? 2 : 1); ++sgn)
			{
				// The partner -k lands on -K: the coordinates negate exactly.
				const T cx = sgn ? -cpos[0] : cpos[0];
				T wx[WC], wy[WC], wz[WC];
				const int fx = place<PROFILE>(cx, wx, kb);
				if (fx > half || fx + taps - 1 < 0)
					continue;
				const int fy = place<PROFILE>(sgn ? -cpos[1] : cpos[1], wy, kb);
				const int fz = place<PROFILE>(sgn ? -cpos[2] : cpos[2], wz, kb);
				const T vre = fmul(vre0, sc);
				const T vim = fmul(sgn ? -vim0 : vim0, sc);
				for (int tz = 0; tz < taps; ++tz)
				{
					const int z = fz + tz;
					if (z < -half || z > half)
						continue;
					const int sz = z < 0 ? z + big : z;
					for (int ty = 0; ty < taps; ++ty)
					{
						const int y = fy + ty;
						if (y < -half || y > half)
							continue;
						const int sy = y < 0 ? y + big : y;
						const T wzy = fmul(wz[tz], wy[ty]);
						const int64_t row_offset = ((int64_t)sz * big + sy) * H;
						for (int tx = 0; tx < taps; ++tx)
						{
							const int x = fx + tx;
							if (x < 0 || x > half)
								continue;
							const T w = fmul(wzy, wx[tx]);
							T are = fmul(vre, w), aim = fmul(vim, w);
							if constexpr (!ODD)
							{
								if ((x + sy + sz) & 1)
								{
									are = -are;
									aim = -aim;
								}
							}
							else
							{
								const C px = volume_phase[x], py = volume_phase[sy], pz = volume_phase[sz];
								const T bre = fsub(fmul(are, px.x), fmul(aim, px.y));
								const T bim = fadd(fmul(are, px.y), fmul(aim, px.x));
								const T cre = fsub(fmul(bre, py.x), fmul(bim, py.y));
								const T cim = fadd(fmul(bre, py.y), fmul(bim, py.x));
								are = fsub(fmul(cre, pz.x), fmul(cim, pz.y));
								aim = fadd(fmul(cre, pz.y), fmul(cim, pz.x));
							}
							red_add2(num + row_offset + x, are, aim);
							red_add(den + row_offset + x, fmul(count, w));
						}
					}
				}
			}
		}
	}
}

template <typename T, typename KB, int PROFILE, int KIND>
void launch_kind(const insertion_launch_of<T> &L, const KB *kb, bool odd, cudaStream_t stream)
{
	const int64_t grid = L.volumes * L.particles;
	const size_t smem = sizeof(complex_t<T>) * (L.h + L.n + (odd ? L.big : 0)) + sizeof(T) * L.h + 16;
	if (odd)
	{
		auto kernel = insert_scatter_kernel<T, KB, PROFILE, KIND, true>;
		check_cuda(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
			"insertion kernel attributes");
		kernel<<<(unsigned)grid, 256, smem, stream>>>(L, *kb);
	}
	else
	{
		auto kernel = insert_scatter_kernel<T, KB, PROFILE, KIND, false>;
		check_cuda(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
			"insertion kernel attributes");
		kernel<<<(unsigned)grid, 256, smem, stream>>>(L, *kb);
	}
	check_cuda(cudaGetLastError(), "insertion kernel launch");
}

template <typename T, typename KB, int PROFILE>
void launch_profile(const insertion_launch_of<T> &L, weight_kind kind, const KB *kb, bool odd, cudaStream_t s)
{
	switch (kind)
	{
	case weight_kind::unit:
		launch_kind<T, KB, PROFILE, 0>(L, kb, odd, s);
		break;
	case weight_kind::ctf:
		launch_kind<T, KB, PROFILE, 1>(L, kb, odd, s);
		break;
	case weight_kind::spectrum:
		launch_kind<T, KB, PROFILE, 2>(L, kb, odd, s);
		break;
	}
}

template <typename T, typename KB>
void launch_scatter(const insertion_launch_of<T> &launch, weight_kind kind, const KB *kb, bool odd_volume,
	cudaStream_t stream)
{
	if (launch.volumes * launch.particles == 0)
		return;
	require(launch.volumes * launch.particles <= 0x7fffffffLL, "too many slices in one call");
	switch (launch.profile)
	{
	case REXLIB_B200_WINDOW_BOX:
		launch_profile<T, KB, REXLIB_B200_WINDOW_BOX>(launch, kind, kb, odd_volume, stream);
		break;
	case REXLIB_B200_WINDOW_TRIANGLE:
		launch_profile<T, KB, REXLIB_B200_WINDOW_TRIANGLE>(launch, kind, kb, odd_volume, stream);
		break;
	default:
		launch_profile<T, KB, REXLIB_B200_WINDOW_KAISER_BESSEL>(launch, kind, kb, odd_volume, stream);
		break;
	}
}

} // anonymous namespace

void launch_insert_scatter(const insertion_launch &launch, weight_kind kind, const kb_table *kb, bool odd_volume,
	cudaStream_t stream)
{
	launch_scatter(launch, kind, kb, odd_volume, stream);
}

void launch_insert_scatter(const insertion_launch_of<double> &launch, weight_kind kind, const kb_table_f64 *kb,
	bool odd_volume, cudaStream_t stream)
{
	launch_scatter(launch, kind, kb, odd_volume, stream);
}

} // namespace rexlib_b200
