/*
 * Oracle (test infrastructure only): Fourier-slice insertion restated in C
 * from the reference CPU backend, in float32 and float64, in the same
 * per-voxel order of additions and with the same float operations, so that a
 * build with -ffp-contract=off is bit-identical to the reference functor
 * built the same way.
 *
 * Followed, by step:
 *  - settle_slices: frame = (N / n) rows 0 and 1 of A; last shell with a
 *    nonzero radial weight; x and y shift phases from FP64 cos/sin
 *    (slice_insertion_functor.inl:161-270, kernels/slice_frame.cpp:10,
 *    kernels/axis_phase.inl:16-35).
 *  - rows and columns: highest row n/2-1 for even n, radius last_shell + 1/2,
 *    widest column h-2 (even) or h-1 (odd), per-row reach sqrt(r^2 - k_y^2)
 *    (slice_insertion_functor.inl:339-393); sign +1 from column 0, sign -1
 *    from column 1 (the Hermitian partner).
 *  - per-voxel order: the reference visits, per slice and sign, the z then
 *    the y frequency intervals of a tile (plans/volume_tile.cpp:68-105); for
 *    an even N the stored index N/2 holds -N/2 (first interval) and +N/2
 *    (last), so the passes below visit frequency -N/2 before the rest.
 *  - prepare: sample weights (unit_weight.inl, ctf_weight.inl:74-103,
 *    spectrum_weight.inl:53-71); coordinates base + k * step in T
 *    (row_insertion_kernel.inl:139-178); windows (kernels/triangle_window.inl,
 *    box_window.inl, kaiser_bessel_window.inl, bessel_i0.cpp); radial shell
 *    round-half-up by the integer test (row_insertion_kernel.inl:188-226);
 *    values (row_insertion_kernel.inl:229-285).
 *  - scatter: taps z, y, x with the frequency bounds, skip r == 0,
 *    num += phase(value * w), den += count * w (row_insertion_kernel.inl:288-360)
 *    with the volume phase (-1)^(x+y+z) for even N (alternating_sign.inl:19)
 *    or the tabulated phase for odd N (tabulated_phase.inl:26-36).
 *  - CTF coefficients (kernels/contrast_transfer_function.inl:26-87,
 *    em/ops/parameters/ctf_optics.cpp:84 for the wavelength).
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define ORACLE_PI 3.141592653589793238462643383279502884

static double bessel_i0(double x)
{
	const double quarter_square = 0.25 * x * x;
	double sum = 1.0, term = 1.0;
	for (double k = 1.0;; k += 1.0)
	{
		term *= quarter_square / (k * k);
		sum += term;
		if (term <= 2.220446049250313e-16 * sum)
			return sum;
	}
}

static double wavelength_of(double voltage_kv)
{
	const double volts = voltage_kv * 1e3;
	return 12.2643247 / sqrt(volts * (1.0 + 0.978466e-6 * volts));
}

/* Stored index of a signed frequency: k < 0 wraps by the extent. */
static long stored_of(long f, long extent) { return f < 0 ? f + extent : f; }

/* Round-half-up of |k| for integer k, by 4s^2+4s+1 <= 4|k|^2. */
static long shell_of(long kx, long ky)
{
	const long m = kx * kx + ky * ky;
	long s = (long)floor(sqrt((double)m) + 0.5);
	while (s > 0 && 4 * (s - 1) * (s - 1) + 4 * (s - 1) + 1 > 4 * m)
		--s;
	while (4 * s * s + 4 * s + 1 <= 4 * m)
		++s;
	return s;
}

#define DEFINE_INSERT(SUFFIX, T, SINFN, TO_INT)                                                      \
	typedef struct                                                                                   \
	{                                                                                                \
		T half_width;                                                                                \
		T scale;                                                                                     \
		int step_count;                                                                              \
		int tap_count;                                                                               \
		T *table;                                                                                    \
	} kb_##SUFFIX;                                                                                   \
                                                                                                     \
	/* Place a sample on one axis: first voxel and tap weights. */                                  \
	static void place_##SUFFIX(int profile, const kb_##SUFFIX *kb, T c, int *first, T *w)            \
	{                                                                                                \
		if (profile == 0)                                                                            \
		{                                                                                            \
			const T half = c < (T)0 ? (T)-0.5 : (T)0.5;                                              \
			*first = (int)(c + half);                                                                \
			w[0] = (T)1;                                                                             \
		}                                                                                            \
		else if (profile == 1)                                                                       \
		{                                                                                            \
			const int truncated = (int)c;                                                            \
			const int below = truncated - (c < (T)truncated ? 1 : 0);                                \
			const T fraction = c - (T)below;                                                         \
			*first = below;                                                                          \
			w[0] = (T)1 - fraction;                                                                  \
			w[1] = fraction;                                                                         \
		}                                                                                            \
		else                                                                                         \
		{                                                                                            \
			const T low = c - kb->half_width;                                                        \
			const int truncated = (int)low;                                                          \
			*first = truncated - (low < (T)truncated ? 1 : 0) + 1;                                   \
			for (int t = 0; t < kb->tap_count; ++t)                                                  \
			{                                                                                        \
				T distance = (T)(*first + t) - c;                                                    \
				distance = distance < (T)0 ? -distance : distance;                                   \
				const T position = distance * kb->scale;                                             \
				const int step = (int)position;                                                      \
				const int index = step < kb->step_count ? step : kb->step_count + 1;                 \
				const T fraction = position - (T)index;                                              \
				const T below = kb->table[index];                                                    \
				w[t] = below + fraction * (kb->table[index + 1] - below);                            \
			}                                                                                        \
		}                                                                                            \
	}                                                                                                \
                                                                                                     \
	int oracle_insert_##SUFFIX(                                                                      \
		int kind, T *numerator, T *denominator, const T *slices, const T *extra,                     \
		const T *transforms, const T *radial, long volumes, long particles, long n, long big,        \
		int slices_per_volume, int radial_per_particle, int extra_per_particle, int profile,         \
		double half_width, double shape, double voltage, double cs, double amplitude_contrast,       \
		double pixel_size)                                                                           \
	{                                                                                                \
		const long h = n / 2 + 1;                                                                    \
		const long H = big / 2 + 1;                                                                  \
		const long half = big / 2;                                                                   \
		const double scale = (double)big / (double)n;                                                \
		const double centre = (double)(n / 2);                                                       \
		const int even_big = big % 2 == 0;                                                           \
		const long last_column = h - (n % 2 == 0 ? 2 : 1);                                           \
		const long highest_row = n % 2 == 0 ? n / 2 - 1 : n / 2;                                     \
                                                                                                     \
		kb_##SUFFIX kb;                                                                              \
		memset(&kb, 0, sizeof(kb));                                                                  \
		int tap_count = profile == 0 ? 1 : 2;                                                        \
		if (profile == 2)                                                                            \
		{                                                                                            \
			const double norm = 1.0 / bessel_i0(shape);                                              \
			const long count = (long)ceil(half_width * 1024.0);                                      \
			kb.half_width = (T)half_width;                                                           \
			kb.tap_count = (int)ceil(2.0 * half_width);                                              \
			kb.scale = (T)((double)count / half_width);                                              \
			kb.step_count = (int)count;                                                              \
			kb.table = (T *)calloc((size_t)count + 3, sizeof(T));                                    \
			for (long i = 0; i <= count; ++i)                                                        \
			{                                                                                        \
				const double ratio = (double)i / (double)count;                                      \
				kb.table[i] = (T)(bessel_i0(shape * sqrt(1.0 - ratio * ratio)) * norm);             \
			}                                                                                        \
			tap_count = kb.tap_count;                                                                \
		}                                                                                            \
                                                                                                     \
		/* Volume phase table for odd N: exp(-2 pi i f C / N) by stored index. */                    \
		T *vol_phase = NULL;                                                                         \
		if (!even_big)                                                                               \
		{                                                                                            \
			vol_phase = (T *)malloc(sizeof(T) * 2 * (size_t)big);                                    \
			const double s = 2.0 * ORACLE_PI * (-(double)half) / (double)big;                        \
			for (long j = 0; j < big; ++j)                                                           \
			{                                                                                        \
				const double f = j <= half ? (double)j : (double)j - (double)big;                    \
				vol_phase[2 * j] = (T)cos(s * f);                                                    \
				vol_phase[2 * j + 1] = (T)sin(s * f);                                                \
			}                                                                                        \
		}                                                                                            \
                                                                                                     \
		T *x_phase = (T *)malloc(sizeof(T) * 2 * (size_t)h);                                         \
		T *y_phase = (T *)malloc(sizeof(T) * 2 * (size_t)n);                                         \
		T *wz = (T *)malloc(sizeof(T) * 16), *wy = (T *)malloc(sizeof(T) * 16);                      \
		T *wx = (T *)malloc(sizeof(T) * 16);                                                         \
		const double wavelength = wavelength_of(voltage);                                            \
                                                                                                     \
		for (long v = 0; v < volumes; ++v)                                                           \
		{                                                                                            \
			T *num = numerator + (size_t)v * big * big * H * 2;                                      \
			T *den = denominator + (size_t)v * big * big * H;                                        \
			for (long p = 0; p < particles; ++p)                                                     \
			{                                                                                        \
				const long index = v * particles + p;                                                \
				const T *tr = transforms + (size_t)index * 12;                                       \
				const T *slice = slices + (size_t)(slices_per_volume ? index : p) * n * h * 2;       \
				const T *rad = radial + (size_t)(radial_per_particle ? p : 0) * h;                   \
				long last_shell = -1;                                                                \
				for (long s = 0; s < h; ++s)                                                         \
					if (rad[s] != (T)0)                                                              \
						last_shell = s;                                                              \
				if (last_shell < 0)                                                                  \
					continue;                                                                        \
				double xs[3], ys[3];                                                                 \
				for (int a = 0; a < 3; ++a)                                                          \
				{                                                                                    \
					xs[a] = (double)tr[a] * scale;                                                   \
					ys[a] = (double)tr[4 + a] * scale;                                               \
				}                                                                                    \
				{                                                                                    \
					const double sx = 2.0 * ORACLE_PI * (centre + (double)tr[3]) / (double)n;        \
					for (long j = 0; j < h; ++j)                                                     \
					{                                                                                \
						const double f = j <= n / 2 ? (double)j : (double)j - (double)n;             \
						x_phase[2 * j] = (T)cos(sx * f);                                             \
						x_phase[2 * j + 1] = (T)sin(sx * f);                                         \
					}                                                                                \
					const double sy = 2.0 * ORACLE_PI * (centre + (double)tr[7]) / (double)n;        \
					for (long j = 0; j < n; ++j)                                                     \
					{                                                                                \
						const double f = j <= n / 2 ? (double)j : (double)j - (double)n;             \
						y_phase[2 * j] = (T)cos(sy * f);                                             \
						y_phase[2 * j + 1] = (T)sin(sy * f);                                         \
					}                                                                                \
				}                                                                                    \
				/* CTF coefficients, FP64 then T. */                                                 \
				T c_radial = 0, c_axial = 0, c_diag = 0, c_aberr = 0, c_phase = 0;                   \
				const T *ctf = NULL;                                                                 \
				const T *weight = NULL;                                                              \
				if (kind == 1)                                                                       \
				{                                                                                    \
					ctf = extra + (extra_per_particle ? (size_t)index * 4 : 0);                      \
					const double du = (double)ctf[0], dv = (double)ctf[1];                           \
					const double angle = (double)ctf[2], shift = (double)ctf[3];                     \
					const double aberration = cs * 1e7;                                              \
					const double fs = 1.0 / ((double)n * pixel_size);                                \
					const double fs2 = fs * fs;                                                      \
					const double dscale = ORACLE_PI * wavelength * fs2;                              \
					const double hd = 0.5 * (du - dv);                                               \
					c_phase = (T)(shift + asin(amplitude_contrast));                                 \
					c_radial = (T)(dscale * 0.5 * (du + dv));                                        \
					c_axial = (T)(dscale * hd * cos(2.0 * angle));                                   \
					c_diag = (T)(2.0 * dscale * hd * sin(2.0 * angle));                              \
					c_aberr = (T)(0.5 * ORACLE_PI * aberration * wavelength * wavelength *           \
						wavelength * fs2 * fs2);                                                     \
				}                                                                                    \
				else if (kind == 2)                                                                  \
				{                                                                                    \
					weight = extra + (extra_per_particle ? (size_t)p * n * h : 0);                   \
				}                                                                                    \
				const double radius = (double)last_shell + 0.5;                                      \
				const long widest = last_column < (long)radius ? last_column : (long)radius;         \
				const long first_row = -highest_row > -widest ? -highest_row : -widest;              \
				const long last_row = highest_row < widest ? highest_row : widest;                   \
                                                                                                     \
				for (int sign = 1; sign >= -1; sign -= 2)                                            \
				{                                                                                    \
					const long first = sign < 0 ? 1 : 0;                                             \
					double step[3], ystep[3];                                                        \
					int finite = 1;                                                                  \
					for (int a = 0; a < 3; ++a)                                                      \
					{                                                                                \
						step[a] = (double)sign * xs[a];                                              \
						ystep[a] = (double)sign * ys[a];                                             \
						finite = finite && isfinite(step[a]) && isfinite(ystep[a]);                  \
					}                                                                                \
					if (!finite)                                                                     \
						continue;                                                                    \
					const T step_t[3] = { (T)step[0], (T)step[1], (T)step[2] };                      \
					/* Passes over the z then y frequency -N/2 (even N) before the rest. */         \
					const int passes = even_big ? 2 : 1;                                             \
					for (int zpass = 0; zpass < passes; ++zpass)                                     \
					for (int ypass = 0; ypass < passes; ++ypass)                                     \
					for (long ky = first_row; ky <= last_row; ++ky)                                  \
					{                                                                                \
						const double kyv = (double)ky;                                               \
						const double reach = radius * radius - kyv * kyv;                            \
						if (reach < 0.0)                                                             \
							continue;                                                                \
						long last = (long)sqrt(reach);                                               \
						last = widest < last ? widest : last;                                        \
						if (first > last)                                                            \
							continue;                                                                \
						const T base_t[3] = { (T)(kyv * ystep[0]), (T)(kyv * ystep[1]),              \
							(T)(kyv * ystep[2]) };                                                   \
						const long srow = ky < 0 ? ky + n : ky;                                      \
						const T *row = slice + (size_t)srow * h * 2;                                 \
						const T yre = y_phase[2 * srow], yim = y_phase[2 * srow + 1];                \
						const T sgn = sign < 0 ? (T)-1 : (T)1;                                       \
						for (long kx = first; kx <= last; ++kx)                                      \
						{                                                                            \
							const long shell = shell_of(kx, ky);                                     \
							const T r = shell <= last_shell ? rad[shell] : (T)0;                     \
							if (r == (T)0)                                                           \
								continue;                                                            \
							T wnum = (T)1, wden = (T)1;                                              \
							if (kind == 1)                                                           \
							{                                                                        \
								const T kxt = (T)kx, kyt = (T)ky;                                    \
								const T xx = kxt * kxt;                                              \
								const T yy = kyt * kyt;                                              \
								const T sq = xx + yy;                                                \
								const T ph = c_radial * sq + c_axial * (xx - yy) +                   \
									c_diag * (kxt * kyt) - c_aberr * (sq * sq) + c_phase;            \
								wnum = SINFN(ph);                                                    \
								wden = wnum * wnum;                                                  \
							}                                                                        \
							else if (kind == 2)                                                      \
							{                                                                        \
								wden = weight[(size_t)srow * h + kx];                                \
							}                                                                        \
							const T sre = row[2 * kx], sim = row[2 * kx + 1];                        \
							const T xre = x_phase[2 * kx], xim = x_phase[2 * kx + 1];                \
							const T shre = sre * xre - sim * xim;                                    \
							const T shim = sre * xim + sim * xre;                                    \
							const T vre0 = shre * yre - shim * yim;                                  \
							const T vim0 = shre * yim + shim * yre;                                  \
							const T sc = r * wnum;                                                   \
							const T vre = vre0 * sc;                                                 \
							const T vim = sgn * vim0 * sc;                                           \
							const T count = r * wden;                                                \
							int fz, fy, fx;                                                          \
							const T kxt = (T)kx;                                                     \
							place_##SUFFIX(profile, &kb, base_t[2] + kxt * step_t[2], &fz, wz);      \
							place_##SUFFIX(profile, &kb, base_t[1] + kxt * step_t[1], &fy, wy);      \
							place_##SUFFIX(profile, &kb, base_t[0] + kxt * step_t[0], &fx, wx);      \
							for (int tz = 0; tz < tap_count; ++tz)                                   \
							{                                                                        \
								const long z = (long)fz + tz;                                        \
								if (z < -half || z > half)                                           \
									continue;                                                        \
								if (even_big && ((zpass == 0) != (z == -half)))                      \
									continue;                                                        \
								const long sz = stored_of(z, big);                                   \
								const T wzt = wz[tz];                                                \
								for (int ty = 0; ty < tap_count; ++ty)                               \
								{                                                                    \
									const long y = (long)fy + ty;                                    \
									if (y < -half || y > half)                                       \
										continue;                                                    \
									if (even_big && ((ypass == 0) != (y == -half)))                  \
										continue;                                                    \
									const long sy = stored_of(y, big);                               \
									const T wzy = wzt * wy[ty];                                      \
									T *nrow = num + ((size_t)sz * big + sy) * H * 2;                 \
									T *drow = den + ((size_t)sz * big + sy) * H;                     \
									for (int tx = 0; tx < tap_count; ++tx)                           \
									{                                                                \
										const long x = (long)fx + tx;                                \
										if (x < 0 || x > half)                                       \
											continue;                                                \
										const T w = wzy * wx[tx];                                    \
										T are = vre * w, aim = vim * w;                              \
										if (even_big)                                                \
										{                                                            \
											if ((x + sy + sz) % 2 != 0)                              \
											{                                                        \
												are = -are;                                          \
												aim = -aim;                                          \
											}                                                        \
										}                                                            \
										else                                                         \
										{                                                            \
											const T *px = vol_phase + 2 * x;                         \
											const T *py = vol_phase + 2 * sy;                        \
											const T *pz = vol_phase + 2 * sz;                        \
											T bre = are * px[0] - aim * px[1];                       \
											T bim = are * px[1] + aim * px[0];                       \
											T cre = bre * py[0] - bim * py[1];                       \
											T cim = bre * py[1] + bim * py[0];                       \
											are = cre * pz[0] - cim * pz[1];                         \
											aim = cre * pz[1] + cim * pz[0];                         \
										}                                                            \
										nrow[2 * x] += are;                                          \
										nrow[2 * x + 1] += aim;                                      \
										drow[x] += count * w;                                        \
									}                                                                \
								}                                                                    \
							}                                                                        \
						}                                                                            \
					}                                                                                \
				}                                                                                    \
			}                                                                                        \
		}                                                                                            \
		free(kb.table);                                                                              \
		free(vol_phase);                                                                             \
		free(x_phase);                                                                               \
		free(y_phase);                                                                               \
		free(wz);                                                                                    \
		free(wy);                                                                                    \
		free(wx);                                                                                    \
		return 0;                                                                                    \
	}

DEFINE_INSERT(f32, float, sinf, 0)
DEFINE_INSERT(f64, double, sin, 0)

float oracle_ctf_f32(double voltage, double cs, double amplitude_contrast, double pixel_size,
	long extent, double defocus_u, double defocus_v, double angle, double phase_shift,
	float k_x, float k_y)
{
	const double wavelength = wavelength_of(voltage);
	const double aberration = cs * 1e7;
	const double fs = 1.0 / ((double)extent * pixel_size);
	const double fs2 = fs * fs;
	const double dscale = ORACLE_PI * wavelength * fs2;
	const double hd = 0.5 * (defocus_u - defocus_v);
	const float c_phase = (float)(phase_shift + asin(amplitude_contrast));
	const float c_radial = (float)(dscale * 0.5 * (defocus_u + defocus_v));
	const float c_axial = (float)(dscale * hd * cos(2.0 * angle));
	const float c_diag = (float)(2.0 * dscale * hd * sin(2.0 * angle));
	const float c_aberr = (float)(0.5 * ORACLE_PI * aberration * wavelength * wavelength * wavelength * fs2 * fs2);
	const float xx = k_x * k_x;
	const float yy = k_y * k_y;
	const float sq = xx + yy;
	return sinf(c_radial * sq + c_axial * (xx - yy) + c_diag * (k_x * k_y) - c_aberr * (sq * sq) + c_phase);
}
