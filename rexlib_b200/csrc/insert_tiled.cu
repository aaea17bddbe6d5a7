// Tile-major insertion for the nearest and linear windows.
//
// The volume's frequency box is cut into tiles of anchor voxels. A sample
// belongs to the one tile that holds its anchor (floor(K) per axis for the
// linear window, the rounded K for the nearest), and every tap it spreads
// lands in that tile or in the one-voxel halo past its upper faces. A CTA
// keeps one tile (with its halo) on chip, inserts into it every sample of a
// run of slices that it owns, and flushes the tile into the accumulators with
// vector global reductions, applying the volume phase exp(-2 pi i g.C/N) per
// voxel on the way (the phase of a voxel is common to all its contributions,
// so it factors out of the sum; row_insertion_kernel.inl:354 applies it per
// contribution).
//
// The tile's denominator sits in shared memory (FP32 atomics). Its numerator
// sits in a private L2-resident scratch per CTA that the taps reach with
// red.global.add.v2.f32: that moves two thirds of the tap traffic off the
// shared-memory pipe, which the bank conflicts of pseudo-random voxel
// addresses otherwise saturate, onto the otherwise idle L2 atomic units. A
// caller without room for the scratch gets the same kernel with all three
// arrays in shared memory.
//
// Work is balanced by a device-side plan: a first pass counts, per tile, the
// slices whose plane can reach it; the plan kernel cuts the slices of each
// tile into runs of about the same number of hits, so the tiles near the
// origin, which every plane crosses, are split over many CTAs; a persistent
// kernel then claims the runs from a device counter. The run length is the
// total hit count over about 16 runs per CTA, kept within [320, 2560]: long
// runs flush a tile less often, and enough runs per CTA keep the last
// claimed run from holding up the grid.
//
// The samples of a slice follow the reference's rows and columns
// (slice_insertion_functor.inl:339-393), bounded per tile with the row and
// column clipping of kernels/row_interval.cpp:34-135; the contribution
// values follow row_insertion_kernel.inl:139-285 with the reference's float
// operations (coordinates, windows, CTF phase polynomial, products).
#include "insertion.cuh"

#include <algorithm>
#include <cmath>
#include <cstdlib>

namespace rexlib_b200
{
namespace
{

constexpr int insert_threads = 512;
constexpr int insert_warps = insert_threads / 32;
constexpr int insert_blocks_per_sm = 2;
constexpr int count_threads = 256;
constexpr size_t insert_smem_budget = 88 * 1024;  // throughput tiles: two CTAs per SM, besides their row records
constexpr size_t l2_numerator_cells = 12000;      // tile cells when the numerator is in L2 (denominator: 48 KB)

struct tile_plan
{
	int lo[3];      // lowest anchor per axis (z, y, x)
	int extent[3];  // anchors per tile per axis
	int tiles[3];   // tiles per axis
	int box[3];     // shared-memory cells per axis: extent + halo
	int tile_count; // tiles per volume
	int min_hits;   // the shortest and longest run (hits per item)
	int max_hits;
	int target_items; // runs the plan aims for: about 16 per CTA
	int item_capacity;
	bool l2_numerator; // numerator tile in the L2 scratch, denominator in shared memory
	int64_t scratch_per_cta; // float2 units of L2 scratch a CTA holds
};

struct work_item
{
	int volume;
	int tile;
	int first;
	int last;
};

// Workspace layout (bytes): the settled slices (V*P), counts (V*T int), the
// item count and the work counter, then the items.
struct settled_slice;
struct workspace_view
{
	settled_slice *settled;
	int *counts;
	int *item_count;
	int *work_counter;
	work_item *items;
	float2 *scratch; // per-CTA numerator tiles (L2 numerator only)
};

size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

constexpr size_t settled_bytes = 104;

workspace_view view_workspace(void *base, int64_t volumes, int64_t particles, const tile_plan &plan)
{
	char *p = static_cast<char *>(base);
	workspace_view w{};
	w.settled = reinterpret_cast<settled_slice *>(p);
	p += align_up(settled_bytes * volumes * particles, 256);
	w.counts = reinterpret_cast<int *>(p);
	p += align_up(sizeof(int) * volumes * plan.tile_count, 256);
	w.item_count = reinterpret_cast<int *>(p);
	w.work_counter = w.item_count + 1;
	p += 256;
	w.items = reinterpret_cast<work_item *>(p);
	p += align_up(sizeof(work_item) * static_cast<size_t>(plan.item_capacity), 256);
	w.scratch = reinterpret_cast<float2 *>(p);
	return w;
}

int insert_grid()
{
	int device = 0, sms = 0;
	check_cuda(cudaGetDevice(&device), "device query");
	check_cuda(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "device query");
	return sms * insert_blocks_per_sm;
}

size_t workspace_bytes(int64_t volumes, int64_t particles, const tile_plan &plan)
{
	return align_up(settled_bytes * volumes * particles, 256) + align_up(sizeof(int) * volumes * plan.tile_count, 256) +
		256 + align_up(sizeof(work_item) * static_cast<size_t>(plan.item_capacity), 256) +
		(plan.l2_numerator ? static_cast<size_t>(plan.scratch_per_cta) * sizeof(float2) * insert_grid() : 0);
}

// ---------------------------------------------------------------------------
// Pass 0: settle every slice once (slice_insertion_functor.inl:161-270)

// What the passes need of a slice, computed once per slice.
struct settled_slice
{
	double ys[3];      // (N/n) * row 1 of A in FP64: row bases are ky * ys rounded to float
	double qx, qy;     // (n/2 + t) / n per image axis: the shift phase exp(2 pi i k q)
	float step[3];     // float((N/n) * row 0 of A): the volume step per column
	float normal[3];   // unit normal of the slice's plane
	float ctf[5];      // radial, axial, diagonal, aberration, phase offset of the CTF phase
	float disc;        // bound on |K| over the inserted samples
	int last_shell;    // last shell with a nonzero radial weight; -1: nothing to insert
	float sigma_min;   // least singular value of the map k -> K (1 for a rotation and N = n)
	float rotor[2];    // exp(2 pi i qx): the x shift phase of one column step
};
static_assert(sizeof(settled_slice) == settled_bytes, "settled_slice layout");

constexpr int settle_threads = 256;

__global__ void __launch_bounds__(settle_threads) settle_kernel(const insertion_launch L, settled_slice *out,
	int kind)
{
	const int64_t index = (static_cast<int64_t>(blockIdx.x) * settle_threads + threadIdx.x) >> 5;
	const int lane = threadIdx.x & 31;
	if (index >= L.volumes * L.particles)
		return;
	const int64_t v = index / L.particles, p = index % L.particles;
	const int n = L.n, h = L.h;
	const float *rad = L.radial + (v * L.radial_stride_v + p * L.radial_stride_p) * h;
	int last_shell = -1;
	for (int s = lane; s < h; s += 32)
		if (__ldg(rad + s) != 0.0f)
			last_shell = s;
	for (int o = 16; o > 0; o >>= 1)
		last_shell = max(last_shell, __shfl_xor_sync(0xffffffffu, last_shell, o));
	if (lane != 0)
		return;
	const float *tr = L.transforms + (v * L.transform_stride_v + p * L.transform_stride_p) * 12;
	const double scale = static_cast<double>(L.big) / static_cast<double>(n);
	settled_slice r{};
	double xs[3];
	bool finite = true;
	for (int a = 0; a < 3; ++a)
	{
		xs[a] = static_cast<double>(__ldg(tr + a)) * scale;
		r.ys[a] = static_cast<double>(__ldg(tr + 4 + a)) * scale;
		r.step[a] = static_cast<float>(xs[a]);
		finite = finite && isfinite(xs[a]) && isfinite(r.ys[a]);
	}
	const double centre = static_cast<double>(n / 2);
	r.qx = (centre + static_cast<double>(__ldg(tr + 3))) / static_cast<double>(n);
	r.qy = (centre + static_cast<double>(__ldg(tr + 7))) / static_cast<double>(n);
	{
		double sn, cs;
		sincospi(2.0 * (r.qx - rint(r.qx)), &sn, &cs);
		r.rotor[0] = static_cast<float>(cs);
		r.rotor[1] = static_cast<float>(sn);
	}
	const double nx = xs[1] * r.ys[2] - xs[2] * r.ys[1];
	const double ny = xs[2] * r.ys[0] - xs[0] * r.ys[2];
	const double nz = xs[0] * r.ys[1] - xs[1] * r.ys[0];
	const double norm = sqrt(nx * nx + ny * ny + nz * nz);
	if (!(finite && isfinite(norm)))
		last_shell = -1;
	if (norm > 0.0)
	{
		r.normal[0] = static_cast<float>(nx / norm);
		r.normal[1] = static_cast<float>(ny / norm);
		r.normal[2] = static_cast<float>(nz / norm);
	}
	else
	{
		r.normal[0] = r.normal[1] = r.normal[2] = 0.0f; // a degenerate frame: no plane test
	}
	const double x2 = xs[0] * xs[0] + xs[1] * xs[1] + xs[2] * xs[2];
	const double y2 = r.ys[0] * r.ys[0] + r.ys[1] * r.ys[1] + r.ys[2] * r.ys[2];
	{
		// Singular values of the map k -> K = k_x xs + k_y ys.
		const double xy = xs[0] * r.ys[0] + xs[1] * r.ys[1] + xs[2] * r.ys[2];
		const double mean = 0.5 * (x2 + y2);
		const double spread = sqrt(0.25 * (x2 - y2) * (x2 - y2) + xy * xy);
		r.sigma_min = static_cast<float>(sqrt(fmax(0.0, mean - spread)));
		// Inserted samples have |k| <= last_shell + 1/2; their taps reach a
		// voxel further. Two voxels of margin.
		r.disc = static_cast<float>((static_cast<double>(max(last_shell, 0)) + 0.5) * sqrt(mean + spread) + 2.0);
	}
	if (kind == static_cast<int>(weight_kind::ctf))
	{
		const float *ctf = L.extra + (v * L.extra_stride_v + p * L.extra_stride_p) * 4;
		const double du = __ldg(ctf), dv = __ldg(ctf + 1), angle = __ldg(ctf + 2), shift = __ldg(ctf + 3);
		const double dscale = pi * L.ctf_wavelength * L.ctf_frequency_scale_sq;
		const double hd = 0.5 * (du - dv);
		double s2, c2;
		sincos(2.0 * angle, &s2, &c2);
		const double wl = L.ctf_wavelength;
		r.ctf[0] = static_cast<float>(dscale * 0.5 * (du + dv));
		r.ctf[1] = static_cast<float>(dscale * hd * c2);
		r.ctf[2] = static_cast<float>(2.0 * dscale * hd * s2);
		r.ctf[3] = static_cast<float>(0.5 * pi * L.ctf_aberration * wl * wl * wl * L.ctf_frequency_scale_sq *
			L.ctf_frequency_scale_sq);
		r.ctf[4] = static_cast<float>(shift + L.ctf_phase_offset);
	}
	r.last_shell = last_shell;
	out[index] = r;
}

// The K-space box whose samples a tile owns, widened by a voxel on each side
// so that rounding in the plane and row tests never drops a sample; axis
// order (x, y, z) as in the reference's frequency_bounds.
struct k_bounds
{
	float lower[3];
	float upper[3];
};

__device__ __forceinline__ k_bounds tile_bounds(const tile_plan &plan, int tile, int *lo)
{
	const int tz = tile / (plan.tiles[1] * plan.tiles[2]);
	const int ty = (tile / plan.tiles[2]) % plan.tiles[1];
	const int tx = tile % plan.tiles[2];
	lo[0] = plan.lo[0] + tz * plan.extent[0];
	lo[1] = plan.lo[1] + ty * plan.extent[1];
	lo[2] = plan.lo[2] + tx * plan.extent[2];
	k_bounds b;
	b.lower[0] = lo[2] - 1.0f;
	b.upper[0] = lo[2] + plan.extent[2] + 1.0f;
	b.lower[1] = lo[1] - 1.0f;
	b.upper[1] = lo[1] + plan.extent[1] + 1.0f;
	b.lower[2] = lo[0] - 1.0f;
	b.upper[2] = lo[0] + plan.extent[0] + 1.0f;
	return b;
}

// Can the plane of the slice reach the box? The box's support along the
// normal must cover the origin's plane, and the box must lie within the
// disc's reach. Both tests carry a margin for float rounding.
__device__ __forceinline__ bool plane_reaches(const settled_slice &s, const k_bounds &b)
{
	if (s.last_shell < 0)
		return false;
	float along = 0.0f, support = 0.0f, d2 = 0.0f;
	for (int a = 0; a < 3; ++a)
	{
		const float c = 0.5f * (b.lower[a] + b.upper[a]);
		const float hw = 0.5f * (b.upper[a] - b.lower[a]);
		along += s.normal[a] * c;
		support += fabsf(s.normal[a]) * hw;
		const float d = fmaxf(0.0f, fmaxf(b.lower[a], -b.upper[a]));
		d2 += d * d;
	}
	return fabsf(along) <= support + 0.05f && d2 <= s.disc * s.disc;
}

// ---------------------------------------------------------------------------
// Pass 1: hits per (volume, tile)

__global__ void __launch_bounds__(count_threads) count_hits_kernel(const insertion_launch L, const tile_plan plan,
	const settled_slice *settled, int *counts)
{
	const int tile = blockIdx.x;
	const int64_t v = blockIdx.y;
	int lo[3];
	const k_bounds b = tile_bounds(plan, tile, lo);
	int hits = 0;
	for (int64_t p = threadIdx.x; p < L.particles; p += blockDim.x)
		hits += plane_reaches(settled[v * L.particles + p], b) ? 1 : 0;
	__shared__ int partial[count_threads / 32];
	for (int o = 16; o > 0; o >>= 1)
		hits += __shfl_xor_sync(0xffffffffu, hits, o);
	if ((threadIdx.x & 31) == 0)
		partial[threadIdx.x >> 5] = hits;
	__syncthreads();
	if (threadIdx.x == 0)
	{
		int total = 0;
		for (int w = 0; w < count_threads / 32; ++w)
			total += partial[w];
		counts[v * plan.tile_count + tile] = total;
	}
}

// ---------------------------------------------------------------------------
// Pass 2: runs of slices per tile

__global__ void __launch_bounds__(1024) plan_items_kernel(const tile_plan plan, int64_t volumes, int64_t particles,
	const int *counts, int *item_count, int *work_counter, work_item *items)
{
	__shared__ int running;
	__shared__ int warp_sums[32];
	__shared__ unsigned long long total_hits;
	if (threadIdx.x == 0)
	{
		running = 0;
		total_hits = 0;
	}
	__syncthreads();
	const int64_t cells = volumes * plan.tile_count;
	// The run length from the total hit count.
	unsigned long long mine = 0;
	for (int64_t i = threadIdx.x; i < cells; i += blockDim.x)
		mine += static_cast<unsigned long long>(counts[i]);
	for (int o = 16; o > 0; o >>= 1)
		mine += __shfl_xor_sync(0xffffffffu, mine, o);
	if ((threadIdx.x & 31) == 0)
		atomicAdd(&total_hits, mine);
	__syncthreads();
	const unsigned long long wanted = (total_hits + plan.target_items - 1) / plan.target_items;
	const int hits_per_item = wanted < static_cast<unsigned long long>(plan.min_hits) ? plan.min_hits
		: wanted > static_cast<unsigned long long>(plan.max_hits)                  ? plan.max_hits
																				   : static_cast<int>(wanted);
	for (int64_t base = 0; base < cells; base += blockDim.x)
	{
		const int64_t i = base + threadIdx.x;
		int runs = 0;
		if (i < cells)
		{
			const int c = counts[i];
			runs = c == 0 ? 0 : (c + hits_per_item - 1) / hits_per_item;
			runs = static_cast<int>(runs < particles ? runs : particles);
		}
		// Block-wide exclusive scan of runs.
		int x = runs;
		const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
		for (int o = 1; o < 32; o <<= 1)
		{
			const int y = __shfl_up_sync(0xffffffffu, x, o);
			if (lane >= o)
				x += y;
		}
		if (lane == 31)
			warp_sums[warp] = x;
		__syncthreads();
		if (warp == 0)
		{
			int s = lane < (int)(blockDim.x >> 5) ? warp_sums[lane] : 0;
			for (int o = 1; o < 32; o <<= 1)
			{
				const int y = __shfl_up_sync(0xffffffffu, s, o);
				if (lane >= o)
					s += y;
			}
			warp_sums[lane] = s;
		}
		__syncthreads();
		const int before = running + (warp > 0 ? warp_sums[warp - 1] : 0) + x - runs;
		if (i < cells && runs > 0)
		{
			const int volume = static_cast<int>(i / plan.tile_count);
			const int tile = static_cast<int>(i % plan.tile_count);
			const int64_t span = (particles + runs - 1) / runs;
			for (int r = 0; r < runs; ++r)
			{
				const int64_t first = r * span;
				const int64_t last = first + span < particles ? first + span : particles;
				if (before + r < plan.item_capacity)
					items[before + r] = work_item{volume, tile, static_cast<int>(first), static_cast<int>(last)};
			}
		}
		__syncthreads();
		if (threadIdx.x == blockDim.x - 1)
			running = before + runs;
		__syncthreads();
	}
	if (threadIdx.x == 0)
	{
		*item_count = min(running, plan.item_capacity);
		*work_counter = 0;
	}
}

// ---------------------------------------------------------------------------
// Pass 3: insertion

// The row and column clipping of kernels/row_interval.cpp:84-136
// (bound_rows) and 34-82 (clip_row) in float, with a slack that keeps the
// ranges conservative under float rounding; the tile's anchor test decides
// ownership exactly.
__device__ __forceinline__ void bound_rows(const float *x_step, const float *y_step, const k_bounds &b,
	int first_x, int last_x, int first_y, int last_y, int &begin, int &end)
{
	float low = static_cast<float>(first_y), high = static_cast<float>(last_y);
	for (int a = 0; a < 3; ++a)
	{
		const float at_first = first_x * x_step[a];
		const float at_last = last_x * x_step[a];
		const float lower = b.lower[a] - fmaxf(at_first, at_last);
		const float upper = b.upper[a] - fminf(at_first, at_last);
		if (fabsf(y_step[a]) < 1e-6f)
		{
			if (!(lower <= 0.01f && -0.01f <= upper))
			{
				begin = end = first_y;
				return;
			}
			continue;
		}
		const float inv = 1.0f / y_step[a];
		const float at_lower = lower * inv;
		const float at_upper = upper * inv;
		low = fmaxf(low, fminf(at_lower, at_upper));
		high = fminf(high, fmaxf(at_lower, at_upper));
	}
	if (low > high + 0.01f)
	{
		begin = end = first_y;
		return;
	}
	begin = max(static_cast<int>(floorf(low - 0.01f)), first_y);
	end = min(static_cast<int>(ceilf(high + 0.01f)) + 1, last_y + 1);
}

__device__ __forceinline__ void clip_row(const float *base, const float *inv_step, const float *step,
	const k_bounds &b, int first, int last, int &begin, int &end)
{
	float low = static_cast<float>(first), high = static_cast<float>(last);
	for (int a = 0; a < 3; ++a)
	{
		if (fabsf(step[a]) < 1e-6f)
		{
			if (!(b.lower[a] - 0.01f <= base[a] && base[a] <= b.upper[a] + 0.01f))
			{
				begin = end = first;
				return;
			}
			continue;
		}
		const float at_lower = (b.lower[a] - base[a]) * inv_step[a];
		const float at_upper = (b.upper[a] - base[a]) * inv_step[a];
		low = fmaxf(low, fminf(at_lower, at_upper));
		high = fminf(high, fmaxf(at_lower, at_upper));
	}
	if (low > high + 0.01f)
	{
		begin = end = first;
		return;
	}
	begin = max(static_cast<int>(floorf(low - 0.01f)), first);
	end = min(static_cast<int>(ceilf(high + 0.01f)) + 1, last + 1);
}

// exp(2 pi i q k) with the argument reduced exactly in FP64 first.
__device__ __forceinline__ float2 shift_phase(double q, int k)
{
	const double t = q * static_cast<double>(k);
	const float u = static_cast<float>(t - rint(t));
	float s, c;
	sincospif(2.0f * u, &s, &c);
	return make_float2(c, s);
}

__device__ __forceinline__ float2 cmul(float2 a, float2 b)
{
	return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// Per-row record a warp shares through shared memory: two 16-byte words,
// {base x, base y, base z, y phase re} and {y phase im, k_y, k_x of the
// row's candidate 0 minus its index, unused}.
struct __align__(16) row_record
{
	float4 lo, hi;
};
static_assert(sizeof(row_record) == 32, "row_record layout");

template <int PROFILE>
__device__ __forceinline__ int anchor_of(float c)
{
	if constexpr (PROFILE == REXLIB_B200_WINDOW_BOX)
	{
		const float half = c < 0.0f ? -0.5f : 0.5f;
		return static_cast<int>(fadd(c, half));
	}
	else
	{
		const int truncated = static_cast<int>(c);
		return truncated - (c < static_cast<float>(truncated) ? 1 : 0);
	}
}

// One tap: the numerator into the L2 scratch (L2_NUM) or shared memory, the
// denominator into shared memory.
template <bool L2_NUM>
__device__ __forceinline__ void add_tap(float2 *g_num, float *s_re, float *s_im, float *s_den, int c, float re,
	float im, float d)
{
	if constexpr (L2_NUM)
		asm volatile("red.global.add.v2.f32 [%0], {%1, %2};" ::"l"(g_num + c), "f"(re), "f"(im) : "memory");
	else
	{
		atomicAdd(s_re + c, re);
		atomicAdd(s_im + c, im);
	}
	atomicAdd(s_den + c, d);
}

template <int PROFILE, int KIND, bool L2_NUM>
__global__ void __launch_bounds__(insert_threads, insert_blocks_per_sm) insert_tiled_kernel(const insertion_launch L,
	const tile_plan plan, const settled_slice *settled, const int *item_count, int *work_counter,
	const work_item *items, float2 *scratch)
{
	constexpr int TAPS = PROFILE == REXLIB_B200_WINDOW_BOX ? 1 : 2;
	constexpr int shared_arrays = L2_NUM ? 1 : 3;
	extern __shared__ float4 smem_raw[];
	const int cells = plan.box[0] * plan.box[1] * plan.box[2];
	const bool odd = (L.big & 1) != 0;
	// Row records first (16-byte aligned), then the volume phase table (odd
	// N), then the accumulators.
	row_record *warp_rows = reinterpret_cast<row_record *>(smem_raw);
	float2 *s_volume_phase = reinterpret_cast<float2 *>(warp_rows + insert_warps * 32);
	float *s_den = reinterpret_cast<float *>(s_volume_phase + (odd ? L.big : 0));
	float *s_re = s_den + cells; // shared numerator (!L2_NUM)
	float *s_im = s_re + cells;
	// L2 numerator: float2 cells (nearest), or the two paired float4 layouts
	// (linear): g_even slot j of a row holds x = 2j and 2j+1, g_odd slot j
	// holds 2j+1 and 2j+2.
	constexpr bool PAIRED = L2_NUM && TAPS == 2;
	const int sx = plan.box[2] / 2 + 1;
	float2 *g_num = L2_NUM ? scratch + static_cast<int64_t>(blockIdx.x) * plan.scratch_per_cta : nullptr;
	float4 *g_even = reinterpret_cast<float4 *>(g_num);
	float4 *g_odd = g_even + static_cast<int64_t>(plan.box[0]) * plan.box[1] * sx;
	if constexpr (L2_NUM)
		for (int64_t i = threadIdx.x; i < plan.scratch_per_cta; i += blockDim.x)
			__stcg(g_num + i, make_float2(0.0f, 0.0f));
	__shared__ int s_item;
	__shared__ int s_next_particle;

	const int lane = threadIdx.x & 31;
	const int warp = threadIdx.x >> 5;
	const int n = L.n, h = L.h, big = L.big, H = L.big_h;
	const int half = big / 2;
	const int bx = plan.box[2], by = plan.box[1];
	const int plane = by * bx;
	const int last_column = h - (n % 2 == 0 ? 2 : 1);
	const int highest_row = n % 2 == 0 ? n / 2 - 1 : n / 2;

	if (odd)
	{
		const double s = 2.0 * pi * (-static_cast<double>(half)) / static_cast<double>(big);
		for (int j = threadIdx.x; j < big; j += blockDim.x)
		{
			const double f = j <= half ? static_cast<double>(j) : static_cast<double>(j - big);
			double sn, cs;
			sincos(s * f, &sn, &cs);
			s_volume_phase[j] = make_float2(static_cast<float>(cs), static_cast<float>(sn));
		}
	}

	const int total_items = *item_count;
	for (;;)
	{
		if (threadIdx.x == 0)
		{
			s_item = atomicAdd(work_counter, 1);
			s_next_particle = 0;
		}
		for (int i = threadIdx.x; i < shared_arrays * cells; i += blockDim.x)
			s_den[i] = 0.0f;
		__syncthreads();
		const int item_index = s_item;
		if (item_index >= total_items)
			break;
		const work_item item = items[item_index];
		const int64_t v = item.volume;
		int lo[3];
		const k_bounds bounds = tile_bounds(plan, item.tile, lo);
		// The K region the tile owns, with a margin far above float rounding:
		// [lo, lo + extent) for the linear window (anchor floor(K)), half a
		// voxel lower for the nearest (anchor round(K)). Rows and columns are
		// clipped to it; the anchor test then decides exactly.
		k_bounds owned;
		{
			const float shift = TAPS == 1 ? 0.5f : 0.0f;
			const int order[3] = {2, 1, 0};
			for (int a = 0; a < 3; ++a)
			{
				owned.lower[a] = lo[order[a]] - shift - 0.02f;
				owned.upper[a] = lo[order[a]] + plan.extent[order[a]] - shift + 0.02f;
			}
		}

		// Slices of the run, claimed 32 at a time by the warps: each lane tests
		// one against the tile, then the warp inserts the hits one by one.
		for (;;)
		{
			int claimed = 0;
			if (lane == 0)
				claimed = atomicAdd(&s_next_particle, 32);
			claimed = __shfl_sync(0xffffffffu, claimed, 0);
			if (item.first + claimed >= item.last)
				break;
			const int64_t mine = item.first + claimed + lane;
			const bool hit = mine < item.last && plane_reaches(settled[v * L.particles + mine], bounds);
			unsigned hits = __ballot_sync(0xffffffffu, hit);
			while (hits)
			{
			const int bit = __ffs(hits) - 1;
			hits &= hits - 1;
			const int64_t p = item.first + claimed + bit;
			const settled_slice S = settled[v * L.particles + p];
			const int last_shell = S.last_shell;
			const float *rad = L.radial + (v * L.radial_stride_v + p * L.radial_stride_p) * h;
			const float *weights = nullptr;
			if constexpr (KIND == static_cast<int>(weight_kind::spectrum))
				weights = L.extra + (v * L.extra_stride_v + p * L.extra_stride_p) * (int64_t)n * h;
			const float2 *slice = L.slices + (v * L.slice_stride_v + p * L.slice_stride_p) * (int64_t)n * h;

			const float radius = static_cast<float>(last_shell) + 0.5f;
			const int widest = min(last_column, last_shell);
			const int first_row = max(-highest_row, -widest);
			const int last_row = min(highest_row, widest);

			for (int sgn = 0; sgn < 2; ++sgn)
			{
				const float sign = sgn ? -1.0f : 1.0f;
				const int first = sgn;
				const float step[3] = {sign * S.step[0], sign * S.step[1], sign * S.step[2]};
				const float ystep_f[3] = {sign * static_cast<float>(S.ys[0]), sign * static_cast<float>(S.ys[1]),
					sign * static_cast<float>(S.ys[2])};
				const float inv_step[3] = {1.0f / step[0], 1.0f / step[1], 1.0f / step[2]};
				int row_begin, row_end;
				bound_rows(step, ystep_f, owned, first, widest, first_row, last_row, row_begin, row_end);
				for (int r0 = row_begin; r0 < row_end; r0 += 32)
				{
					// Lane j prepares row r0 + j; the rows with candidates are
					// compacted into shared memory in order.
					const int ky = r0 + lane;
					int b = 0, e = 0;
					float base[3] = {0.0f, 0.0f, 0.0f};
					if (ky < row_end)
					{
						// reach = radius^2 - ky^2 is an integer plus 1/4: exact in float.
						const float reach = radius * radius - static_cast<float>(ky * ky);
						if (reach >= 0.0f)
						{
							const int last = min(widest, static_cast<int>(sqrtf(reach)));
							if (first <= last)
							{
								// Row bases ky * ys in FP64 rounded to float, as the CPU.
								const double kyv = static_cast<double>(ky) * (sgn ? -1.0 : 1.0);
								base[0] = static_cast<float>(kyv * S.ys[0]);
								base[1] = static_cast<float>(kyv * S.ys[1]);
								base[2] = static_cast<float>(kyv * S.ys[2]);
								clip_row(base, inv_step, step, owned, first, last, b, e);
							}
						}
					}
					const int count = max(0, e - b);
					int prefix = count;
					for (int o = 1; o < 32; o <<= 1)
					{
						const int y = __shfl_up_sync(0xffffffffu, prefix, o);
						if (lane >= o)
							prefix += y;
					}
					const int total = __shfl_sync(0xffffffffu, prefix, 31);
					if (total == 0)
						continue;
					const int before = prefix - count; // candidates of the earlier rows
					const bool filled = count > 0;
					const unsigned filled_rows = __ballot_sync(0xffffffffu, filled);
					row_record *rows = warp_rows + warp * 32;
					if (filled)
					{
						const float2 y_phase = shift_phase(S.qy, ky);
						row_record rec;
						rec.lo = make_float4(base[0], base[1], base[2], y_phase.x);
						rec.hi = make_float4(y_phase.y, __int_as_float(ky), __int_as_float(b - before), 0.0f);
						rows[__popc(filled_rows & ((1u << lane) - 1u))] = rec;
					}
					__syncwarp();

					// One candidate sample per lane per round. The row of
					// candidate c0 + lane: the filled rows that start at or
					// before c0, then the row starts among c0 + 1 .. c0 + lane.
					for (int c0 = 0; c0 < total; c0 += 32)
					{
						const int at = before - c0;
						const unsigned started = __ballot_sync(0xffffffffu, filled && at <= 0);
						const unsigned starts = __reduce_or_sync(0xffffffffu, filled && at > 0 && at < 32 ? 1u << at : 0u);
						const int cand = c0 + lane;
						if (cand >= total)
							break;
						const int row_index = __popc(started) - 1 + __popc(starts & ((2u << lane) - 1u));
						const float4 rlo = rows[row_index].lo;
						const float4 rhi = rows[row_index].hi;
						const int kx = cand + __float_as_int(rhi.z);
						const int rky = __float_as_int(rhi.y);
						const float2 row_y_phase = make_float2(rlo.w, rhi.x);
						const float kxf = static_cast<float>(kx);
						const float cx = fadd(rlo.x, fmul(kxf, step[0]));
						const float cy = fadd(rlo.y, fmul(kxf, step[1]));
						const float cz = fadd(rlo.z, fmul(kxf, step[2]));
						const int ax = anchor_of<PROFILE>(cx) - lo[2];
						const int ay = anchor_of<PROFILE>(cy) - lo[1];
						const int az = anchor_of<PROFILE>(cz) - lo[0];
						if (static_cast<unsigned>(ax) >= static_cast<unsigned>(plan.extent[2]) ||
							static_cast<unsigned>(ay) >= static_cast<unsigned>(plan.extent[1]) ||
							static_cast<unsigned>(az) >= static_cast<unsigned>(plan.extent[0]))
							continue;
						const int shell = shell_of(kx, rky);
						const float r = shell <= last_shell ? __ldg(rad + shell) : 0.0f;
						if (r == 0.0f)
							continue;
						const int srow = rky < 0 ? rky + n : rky;
						float wnum = 1.0f, wden = 1.0f;
						if constexpr (KIND == static_cast<int>(weight_kind::ctf))
						{
							const float kyt = static_cast<float>(rky);
							const float xx = fmul(kxf, kxf);
							const float yy = fmul(kyt, kyt);
							const float sq = fadd(xx, yy);
							float ph = fmul(S.ctf[0], sq);
							ph = fadd(ph, fmul(S.ctf[1], fsub(xx, yy)));
							ph = fadd(ph, fmul(S.ctf[2], fmul(kxf, kyt)));
							ph = fsub(ph, fmul(S.ctf[3], fmul(sq, sq)));
							ph = fadd(ph, S.ctf[4]);
							wnum = sin_reduced(ph);
							wden = wnum * wnum;
						}
						else if constexpr (KIND == static_cast<int>(weight_kind::spectrum))
						{
							wden = __ldg(weights + (int64_t)srow * h + kx);
						}
						const float2 sample = __ldg(slice + (int64_t)srow * h + kx);
						const float2 value = cmul(cmul(sample, shift_phase(S.qx, kx)), row_y_phase);
						const float sc = r * wnum;
						const float vre = value.x * sc;
						const float vim = (sgn ? -value.y : value.y) * sc;
						const float cnt = r * wden;
						const int cell = (az * by + ay) * bx + ax;
						if constexpr (TAPS == 1)
						{
							add_tap<L2_NUM>(g_num, s_re, s_im, s_den, cell, vre, vim, cnt);
						}
						else
						{
							const float fx = fsub(cx, static_cast<float>(ax + lo[2]));
							const float fy = fsub(cy, static_cast<float>(ay + lo[1]));
							const float fz = fsub(cz, static_cast<float>(az + lo[0]));
							const float wx[2] = {fsub(1.0f, fx), fx};
							const float wy[2] = {fsub(1.0f, fy), fy};
							const float wz[2] = {fsub(1.0f, fz), fz};
#pragma unroll
							for (int dz = 0; dz < 2; ++dz)
#pragma unroll
								for (int dy = 0; dy < 2; ++dy)
								{
									const float wzy = fmul(wz[dz], wy[dy]);
									if constexpr (PAIRED)
									{
										const float w0 = fmul(wzy, wx[0]), w1 = fmul(wzy, wx[1]);
										const int c = cell + dz * plane + dy * bx;
										float4 *slot = ((ax & 1) ? g_odd : g_even) + ((az + dz) * by + (ay + dy)) * sx + (ax >> 1);
										asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(slot), "f"(vre * w0),
													 "f"(vim * w0), "f"(vre * w1), "f"(vim * w1)
													 : "memory");
										atomicAdd(s_den + c, cnt * w0);
										atomicAdd(s_den + c + 1, cnt * w1);
									}
									else
									{
#pragma unroll
										for (int dx = 0; dx < 2; ++dx)
										{
											const float w = fmul(wzy, wx[dx]);
											const int c = cell + dz * plane + dy * bx + dx;
											add_tap<L2_NUM>(g_num, s_re, s_im, s_den, c, vre * w, vim * w, cnt * w);
										}
									}
								}
						}
					}
					__syncwarp();
				}
			}
			}
		}
		__syncthreads();

		// Flush the tile and its halo, with the volume phase.
		float2 *num = L.numerator + v * (int64_t)big * big * H;
		float *den = L.denominator + v * (int64_t)big * big * H;
		for (int i = threadIdx.x; i < cells; i += blockDim.x)
		{
			const int cz = i / plane;
			const int cy = (i / bx) % by;
			const int cx = i % bx;
			float re, im;
			const float d = s_den[i];
			if constexpr (PAIRED)
			{
				// x = cx is half cx & 1 of even slot cx >> 1 and, from x = 1,
				// half (cx - 1) & 1 of odd slot (cx - 1) >> 1.
				const int64_t row = (static_cast<int64_t>(cz) * by + cy) * 2 * sx;
				float2 *e = reinterpret_cast<float2 *>(g_even) + row + cx;
				const float2 a = __ldcg(e);
				re = a.x;
				im = a.y;
				if (re != 0.0f || im != 0.0f)
					__stcg(e, make_float2(0.0f, 0.0f));
				if (cx >= 1)
				{
					float2 *o = reinterpret_cast<float2 *>(g_odd) + row + cx - 1;
					const float2 b = __ldcg(o);
					if (b.x != 0.0f || b.y != 0.0f)
					{
						re += b.x;
						im += b.y;
						__stcg(o, make_float2(0.0f, 0.0f));
					}
				}
			}
			else if constexpr (L2_NUM)
			{
				const float2 a = __ldcg(g_num + i);
				re = a.x;
				im = a.y;
				if (re != 0.0f || im != 0.0f)
					__stcg(g_num + i, make_float2(0.0f, 0.0f));
			}
			else
			{
				re = s_re[i];
				im = s_im[i];
			}
			if (re == 0.0f && im == 0.0f && d == 0.0f)
				continue;
			const int fz = lo[0] + cz, fy = lo[1] + cy, fx = lo[2] + cx;
			if (fz < -half || fz > half || fy < -half || fy > half || fx < 0 || fx > half)
				continue;
			const int sz = fz < 0 ? fz + big : fz;
			const int sy = fy < 0 ? fy + big : fy;
			float are = re, aim = im;
			if (!odd)
			{
				if ((fx + sy + sz) & 1)
				{
					are = -are;
					aim = -aim;
				}
			}
			else
			{
				const float2 px = s_volume_phase[fx], py = s_volume_phase[sy], pz = s_volume_phase[sz];
				const float bre = px.x * are - px.y * aim;
				const float bim = px.y * are + px.x * aim;
				const float cre = py.x * bre - py.y * bim;
				const float cim = py.y * bre + py.x * bim;
				are = pz.x * cre - pz.y * cim;
				aim = pz.y * cre + pz.x * cim;
			}
			const int64_t offset = ((int64_t)sz * big + sy) * H + fx;
			asm volatile("red.global.add.v2.f32 [%0], {%1, %2};" ::"l"(num + offset), "f"(are), "f"(aim) : "memory");
			asm volatile("red.global.add.f32 [%0], %1;" ::"l"(den + offset), "f"(d) : "memory");
		}
		__syncthreads();
	}
}

// ---------------------------------------------------------------------------
// Deterministic mode: a gather in the CPU's order.
//
// Tiles of 16^3 stored voxels (z, y in [0, N), x in [0, N/2]); a CTA owns a
// tile, starts from the accumulator's values and walks the slices in index
// order, as the CPU's insert_tile does (slice_insertion_functor.inl:274-466):
// for each slice, sign (+k, then -k), pair of z and y frequency intervals
// of the tile (plans/volume_tile.cpp:68-105; with an even N the stored N/2
// holds -N/2 and +N/2) and row k_y in ascending order, the samples k_x in
// ascending order. Each voxel therefore sums its contributions in exactly
// the CPU's order, whatever the scheduling, and a batch split across calls
// gives the bits of one call.
//
// Per (slice, sign, interval pair) the rows are taken in batches of at most
// 32 rows and 1,024 samples: a warp prepares the rows (the reach and
// clipping of the CPU's bound_rows / clip_row), all threads compute the
// batch's sample positions K and values into shared memory, then every
// thread gathers for the voxels of one pillar of the tile along the axis
// the slice's normal leans on most. A voxel g can only receive from samples
// with |K - g| < sqrt(3) (the nearest window: sqrt(3)/2), i.e. k within
// sqrt(3) / sigma_min of the least-squares k* = (M^T M)^-1 M^T g of the
// frame M = [x step, y step]; those candidates are tested exactly (the
// anchor of the CPU's window place) in row, then column, order. Pillars
// are disjoint, so the read-modify-writes of a batch never race, and
// barriers separate the batches.

struct det_plan
{
	int extent[3]; // stored voxels per tile (z, y, x)
	int tiles[3];
	int tile_count;
};

constexpr int det_threads = 512;
constexpr int det_edge = 16;       // tile edge: det_edge^2 pillars, two threads each
constexpr int det_capacity = 768;  // samples in a batch
constexpr int det_batch_rows = 32; // rows in a batch (one warp prepares them)
static_assert(2 * det_edge * det_edge == det_threads, "two threads a pillar");

__device__ __forceinline__ int det_intervals(int begin, int end, int extent, int *lower, int *upper)
{
	// list_stored_frequencies of plans/volume_tile.cpp:68-105.
	const int half = extent / 2;
	const int first = begin, last = end - 1;
	const bool both = extent % 2 == 0 && first <= half && half <= last;
	int count = 0;
	if (last > half)
	{
		lower[count] = both ? -half : max(first, half + 1) - extent;
		upper[count] = last - extent;
		++count;
	}
	else if (both)
	{
		lower[count] = -half;
		upper[count] = -half;
		++count;
	}
	if (first <= half)
	{
		lower[count] = first;
		upper[count] = min(last, half);
		++count;
	}
	return count;
}

// The frequency of stored index s within the interval [lo, hi], or a
// sentinel above any frequency when it has none there.
__device__ __forceinline__ int frequency_in(int s, int lo, int hi, int extent)
{
	const int half = extent / 2;
	const int f = s > half ? s - extent : s;
	if (f >= lo && f <= hi)
		return f;
	if (extent % 2 == 0 && s == half && -half >= lo && -half <= hi)
		return -half;
	return 1 << 30;
}

// A batch row: the CPU's clipped interval [b, e) of k_x, the batch index of
// its first sample, its y phase and its base (k_y times the y step).
struct det_row
{
	int b, e, off;
	float2 y_phase;
	float base[3];
};

template <int PROFILE, int KIND>
__global__ void __launch_bounds__(det_threads, 1) insert_deterministic_kernel(const insertion_launch L,
	const det_plan plan, const settled_slice *settled, const int *tile_order)
{
	constexpr int TAPS = PROFILE == REXLIB_B200_WINDOW_BOX ? 1 : 2;
	constexpr int cells = det_edge * det_edge * det_edge;
	extern __shared__ float4 smem_raw[];
	float4 *s_key = smem_raw;                 // K of batch sample i; w = 1 when it inserts
	float4 *s_val = s_key + det_capacity;     // (re, im, weight of the denominator, -)
	float *s_re = reinterpret_cast<float *>(s_val + det_capacity);
	float *s_im = s_re + cells;
	float *s_den = s_im + cells;
	float2 *s_volume_phase = reinterpret_cast<float2 *>(s_den + cells); // odd N
	__shared__ det_row rows[det_batch_rows];
	__shared__ int s_hits[det_threads];
	__shared__ int s_warp_hits[det_threads / 32];
	__shared__ int s_hit_count, s_rows, s_total;
	__shared__ settled_slice s_slice;

	const int n = L.n, h = L.h, big = L.big, H = L.big_h;
	const int half = big / 2;
	const int last_column = h - (n % 2 == 0 ? 2 : 1);
	const int highest_row = n % 2 == 0 ? n / 2 - 1 : n / 2;
	const bool odd = (big & 1) != 0;
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	const int64_t v = blockIdx.y;
	const int tile = tile_order[blockIdx.x];
	const int tz = tile / (plan.tiles[1] * plan.tiles[2]);
	const int ty = (tile / plan.tiles[2]) % plan.tiles[1];
	const int tx = tile % plan.tiles[2];
	const int z0 = tz * det_edge, y0 = ty * det_edge, x0 = tx * det_edge;
	const int z1 = min(z0 + det_edge, big), y1 = min(y0 + det_edge, big), x1 = min(x0 + det_edge, H);

	if (odd)
	{
		const double s = 2.0 * pi * (-static_cast<double>(half)) / static_cast<double>(big);
		for (int j = threadIdx.x; j < big; j += blockDim.x)
		{
			const double f = j <= half ? static_cast<double>(j) : static_cast<double>(j - big);
			double sn, cs;
			sincos(s * f, &sn, &cs);
			s_volume_phase[j] = make_float2(static_cast<float>(cs), static_cast<float>(sn));
		}
	}
	float2 *num = L.numerator + v * (int64_t)big * big * H;
	float *den = L.denominator + v * (int64_t)big * big * H;
	for (int i = threadIdx.x; i < cells; i += blockDim.x)
	{
		const int sz = z0 + i / (det_edge * det_edge), sy = y0 + (i / det_edge) % det_edge, x = x0 + i % det_edge;
		float2 a = make_float2(0.0f, 0.0f);
		float d = 0.0f;
		if (sz < z1 && sy < y1 && x < x1)
		{
			const int64_t offset = ((int64_t)sz * big + sy) * H + x;
			a = num[offset];
			d = den[offset];
		}
		s_re[i] = a.x;
		s_im[i] = a.y;
		s_den[i] = d;
	}

	int zl[2], zu[2], yl[2], yu[2];
	const int zcount = det_intervals(z0, z1, big, zl, zu);
	const int ycount = det_intervals(y0, y1, big, yl, yu);
	// The K region whose taps can reach any voxel of the tile: a sample
	// reaches voxel g when its K lies in g + [-1, 1) per axis (the nearest
	// window: [-1/2, 1/2]); 0.05 more for rounding.
	constexpr float margin = (PROFILE == REXLIB_B200_WINDOW_BOX ? 0.5f : 1.0f) + 0.05f;
	k_bounds whole;
	whole.lower[0] = x0 - margin;
	whole.upper[0] = x1 - 1 + margin;
	whole.lower[1] = fminf(yl[0], yl[ycount - 1]) - margin;
	whole.upper[1] = fmaxf(yu[0], yu[ycount - 1]) + margin;
	whole.lower[2] = fminf(zl[0], zl[zcount - 1]) - margin;
	whole.upper[2] = fmaxf(zu[0], zu[zcount - 1]) + margin;
	// Pillar (p1, p2); the pillar's two threads take alternate voxels of it.
	const int pillar = threadIdx.x % (det_edge * det_edge), half_of = threadIdx.x / (det_edge * det_edge);
	const int p1 = pillar / det_edge, p2 = pillar % det_edge;

	for (int64_t chunk = 0; chunk < L.particles; chunk += det_threads)
	{
		// The slices of the chunk that reach the tile, in index order.
		const int64_t mine = chunk + threadIdx.x;
		const bool hit = mine < L.particles && plane_reaches(settled[v * L.particles + mine], whole);
		const unsigned hits = __ballot_sync(0xffffffffu, hit);
		__syncthreads(); // the previous chunk's hit list is done with
		if (lane == 0)
			s_warp_hits[warp] = __popc(hits);
		__syncthreads();
		int before = 0;
		for (int w = 0; w < warp; ++w)
			before += s_warp_hits[w];
		if (hit)
			s_hits[before + __popc(hits & ((1u << lane) - 1u))] = threadIdx.x;
		if (threadIdx.x == det_threads - 1)
			s_hit_count = before + __popc(hits);
		__syncthreads();
		const int hit_count = s_hit_count;

		for (int hi = 0; hi < hit_count; ++hi)
		{
			const int64_t p = chunk + s_hits[hi];
			__syncthreads(); // the previous slice is done with s_slice
			if (threadIdx.x < static_cast<int>(sizeof(settled_slice) / 4))
				reinterpret_cast<int *>(&s_slice)[threadIdx.x] =
					reinterpret_cast<const int *>(settled + v * L.particles + p)[threadIdx.x];
			__syncthreads();
			const settled_slice &S = s_slice;
			const int last_shell = S.last_shell;
			const float *rad = L.radial + (v * L.radial_stride_v + p * L.radial_stride_p) * h;
			const float *weights = nullptr;
			if constexpr (KIND == static_cast<int>(weight_kind::spectrum))
				weights = L.extra + (v * L.extra_stride_v + p * L.extra_stride_p) * (int64_t)n * h;
			const float2 *slice = L.slices + (v * L.slice_stride_v + p * L.slice_stride_p) * (int64_t)n * h;
			const float radius = static_cast<float>(last_shell) + 0.5f;
			const int widest = min(last_column, last_shell);
			const int first_row = max(-highest_row, -widest);
			const int last_row = min(highest_row, widest);
			// The pillar axis: the one the normal leans on most (0 x, 1 y, 2 z).
			const float nx = fabsf(S.normal[0]), ny = fabsf(S.normal[1]), nz = fabsf(S.normal[2]);
			const int axis = nz >= ny && nz >= nx ? 2 : (ny >= nx ? 1 : 0);
			const float slab = (TAPS == 2 ? 1.0f : 0.5f) * (nx + ny + nz) + 0.02f;
			// A sample reaches voxel g when its K lies in g + [-cube, cube) per axis.
			constexpr float cube = TAPS == 2 ? 1.0f : 0.5f;
			// Candidates lie within this k distance of k*.
			const float reach_k = fminf((TAPS == 2 ? 1.7320508f : 0.8660254f) / fmaxf(S.sigma_min, 1e-6f) + 0.02f, 1.0e6f);

			for (int sgn = 0; sgn < 2; ++sgn)
			{
				const float sign = sgn ? -1.0f : 1.0f;
				const int first = sgn;
				const float step[3] = {sign * S.step[0], sign * S.step[1], sign * S.step[2]};
				const float ystep_f[3] = {sign * static_cast<float>(S.ys[0]), sign * static_cast<float>(S.ys[1]),
					sign * static_cast<float>(S.ys[2])};
				const float inv_step[3] = {1.0f / step[0], 1.0f / step[1], 1.0f / step[2]};
				// k* = (M^T M)^-1 M^T g for M = [step, ystep].
				const float g11 = step[0] * step[0] + step[1] * step[1] + step[2] * step[2];
				const float g12 = step[0] * ystep_f[0] + step[1] * ystep_f[1] + step[2] * ystep_f[2];
				const float g22 = ystep_f[0] * ystep_f[0] + ystep_f[1] * ystep_f[1] + ystep_f[2] * ystep_f[2];
				const float det = g11 * g22 - g12 * g12;
				const float inv_det = det != 0.0f ? 1.0f / det : 0.0f;
				float pu[3], pv[3];
				for (int a = 0; a < 3; ++a)
				{
					pu[a] = (g22 * step[a] - g12 * ystep_f[a]) * inv_det;
					pv[a] = (g11 * ystep_f[a] - g12 * step[a]) * inv_det;
				}

				for (int zi = 0; zi < zcount; ++zi)
					for (int yi = 0; yi < ycount; ++yi)
					{
						k_bounds bounds;
						bounds.lower[0] = x0 - margin;
						bounds.upper[0] = x1 - 1 + margin;
						bounds.lower[1] = yl[yi] - margin;
						bounds.upper[1] = yu[yi] + margin;
						bounds.lower[2] = zl[zi] - margin;
						bounds.upper[2] = zu[zi] + margin;
						if (!plane_reaches(S, bounds))
							continue;
						int row_begin, row_end;
						bound_rows(step, ystep_f, bounds, first, widest, first_row, last_row, row_begin, row_end);

						// This thread's pillar in the interval pair: the two fixed
						// frequencies, the frequency range along the axis.
						int fz = 1 << 30, fy = 1 << 30, fx = 1 << 30, lo_t = 0, hi_t = -1;
						{
							const int sz_p = z0 + p1, sy_p = (axis == 2 ? y0 + p1 : y0 + p2), x_p = x0 + p2;
							if (axis == 2)
							{
								fy = sy_p < y1 ? frequency_in(sy_p, yl[yi], yu[yi], big) : 1 << 30;
								fx = x_p < x1 ? x_p : 1 << 30;
								lo_t = zl[zi];
								hi_t = zu[zi];
							}
							else if (axis == 1)
							{
								fz = sz_p < z1 ? frequency_in(sz_p, zl[zi], zu[zi], big) : 1 << 30;
								fx = x_p < x1 ? x_p : 1 << 30;
								lo_t = yl[yi];
								hi_t = yu[yi];
							}
							else
							{
								fz = sz_p < z1 ? frequency_in(sz_p, zl[zi], zu[zi], big) : 1 << 30;
								fy = sy_p < y1 ? frequency_in(sy_p, yl[yi], yu[yi], big) : 1 << 30;
								lo_t = x0;
								hi_t = x1 - 1;
							}
							const bool fixed_ok = (axis == 2 || fz != (1 << 30)) && (axis == 1 || fy != (1 << 30)) &&
								(axis == 0 || fx != (1 << 30));
							if (!fixed_ok)
								hi_t = lo_t - 1;
							else
							{
								// |n . g| <= slab along the pillar.
								const float na = S.normal[axis];
								const float rest = (axis == 0 ? 0.0f : S.normal[0] * fx) +
									(axis == 1 ? 0.0f : S.normal[1] * fy) + (axis == 2 ? 0.0f : S.normal[2] * fz);
								const float ta = (-rest - slab) / na, tb = (-rest + slab) / na;
								lo_t = max(lo_t, static_cast<int>(floorf(fminf(ta, tb))));
								hi_t = min(hi_t, static_cast<int>(ceilf(fmaxf(ta, tb))));
							}
						}

						for (int r0 = row_begin; r0 < row_end;)
						{
							__syncthreads(); // the previous batch is done with the rows and the table
							if (warp == 0)
							{
								const int ky = r0 + lane;
								int b = 0, e = 0;
								det_row rec{};
								if (ky < row_end)
								{
									const float reach = radius * radius - static_cast<float>(ky * ky);
									if (reach >= 0.0f)
									{
										const int last = min(widest, static_cast<int>(sqrtf(reach)));
										if (first <= last)
										{
											const double kyv = static_cast<double>(ky) * (sgn ? -1.0 : 1.0);
											rec.base[0] = static_cast<float>(kyv * S.ys[0]);
											rec.base[1] = static_cast<float>(kyv * S.ys[1]);
											rec.base[2] = static_cast<float>(kyv * S.ys[2]);
											clip_row(rec.base, inv_step, step, bounds, first, last, b, e);
										}
									}
								}
								const int count = max(0, e - b);
								int prefix = count;
								for (int o = 1; o < 32; o <<= 1)
								{
									const int y = __shfl_up_sync(0xffffffffu, prefix, o);
									if (lane >= o)
										prefix += y;
								}
								// The batch: the rows whose samples fit (at least one row).
								const unsigned fits = __ballot_sync(0xffffffffu, ky < row_end && prefix <= det_capacity);
								const int nb = max(1, __popc(fits));
								if (count > 0)
									rec.y_phase = shift_phase(S.qy, ky);
								rec.b = b;
								rec.e = max(b, e);
								rec.off = prefix - count;
								rows[lane] = rec;
								if (lane == nb - 1)
								{
									s_rows = nb;
									s_total = prefix;
								}
							}
							__syncthreads();
							const int nb = s_rows, total = s_total;

							// The batch's sample positions and values, as the CPU's prepare.
							for (int i = threadIdx.x; i < total; i += blockDim.x)
							{
								int lo_r = 0;
								for (int bit = 16; bit > 0; bit >>= 1)
									if (lo_r + bit < nb && rows[lo_r + bit].off <= i)
										lo_r += bit;
								const det_row &row = rows[lo_r];
								const int kx = row.b + (i - row.off);
								const int rky = r0 + lo_r;
								const float kxf = static_cast<float>(kx);
								const float cx = fadd(row.base[0], fmul(kxf, step[0]));
								const float cy = fadd(row.base[1], fmul(kxf, step[1]));
								const float cz = fadd(row.base[2], fmul(kxf, step[2]));
								const int shell = shell_of(kx, rky);
								const float r = shell <= last_shell ? __ldg(rad + shell) : 0.0f;
								float vre = 0.0f, vim = 0.0f, cnt = 0.0f;
								if (r != 0.0f)
								{
									const int srow = rky < 0 ? rky + n : rky;
									float wnum = 1.0f, wden = 1.0f;
									if constexpr (KIND == static_cast<int>(weight_kind::ctf))
									{
										const float kyt = static_cast<float>(rky);
										const float xx = fmul(kxf, kxf);
										const float yy = fmul(kyt, kyt);
										const float sq = fadd(xx, yy);
										float ph = fmul(S.ctf[0], sq);
										ph = fadd(ph, fmul(S.ctf[1], fsub(xx, yy)));
										ph = fadd(ph, fmul(S.ctf[2], fmul(kxf, kyt)));
										ph = fsub(ph, fmul(S.ctf[3], fmul(sq, sq)));
										ph = fadd(ph, S.ctf[4]);
										wnum = sinf(ph);
										wden = fmul(wnum, wnum);
									}
									else if constexpr (KIND == static_cast<int>(weight_kind::spectrum))
									{
										wden = __ldg(weights + (int64_t)srow * h + kx);
									}
									const float2 sample = __ldg(slice + (int64_t)srow * h + kx);
									const float2 xph = shift_phase(S.qx, kx);
									const float2 yph = row.y_phase;
									const float shre = fsub(fmul(sample.x, xph.x), fmul(sample.y, xph.y));
									const float shim = fadd(fmul(sample.x, xph.y), fmul(sample.y, xph.x));
									const float vre0 = fsub(fmul(shre, yph.x), fmul(shim, yph.y));
									const float vim0 = fadd(fmul(shre, yph.y), fmul(shim, yph.x));
									const float sc = fmul(r, wnum);
									vre = fmul(vre0, sc);
									vim = fmul(sgn ? -vim0 : vim0, sc);
									cnt = fmul(r, wden);
								}
								s_key[i] = make_float4(cx, cy, cz, r != 0.0f ? 1.0f : 0.0f);
								s_val[i] = make_float4(vre, vim, cnt, 0.0f);
							}
							__syncthreads();

							// The gather: this pillar's voxels near the plane, each summing
							// its samples of the batch in row, then column, order.
							for (int t = lo_t + half_of; t <= hi_t; t += 2)
							{
								const int gx = axis == 0 ? t : fx, gy = axis == 1 ? t : fy, gz = axis == 2 ? t : fz;
								const int sy = gy < 0 ? gy + big : gy, sz = gz < 0 ? gz + big : gz;
								const int cell = ((sz - z0) * det_edge + (sy - y0)) * det_edge + (gx - x0);
								const float gxf = static_cast<float>(gx), gyf = static_cast<float>(gy),
											gzf = static_cast<float>(gz);
								const float u = fminf(fmaxf(pu[0] * gxf + pu[1] * gyf + pu[2] * gzf, -1.0e7f), 1.0e7f);
								const float w = fminf(fmaxf(pv[0] * gxf + pv[1] * gyf + pv[2] * gzf, -1.0e7f), 1.0e7f);
								const int ky_lo = max(r0, static_cast<int>(ceilf(w - reach_k)));
								const int ky_hi = min(r0 + nb - 1, static_cast<int>(floorf(w + reach_k)));
								const int kx_lo = static_cast<int>(ceilf(u - reach_k));
								const int kx_hi = static_cast<int>(floorf(u + reach_k));
								if (ky_lo > ky_hi)
									continue;
								float acc_re = s_re[cell], acc_im = s_im[cell], acc_den = s_den[cell];
								bool touched = false;
								const float gv[3] = {gxf, gyf, gzf};
								for (int ky = ky_lo; ky <= ky_hi; ++ky)
								{
									const det_row &row = rows[ky - r0];
									// k_x whose K lies in g + [-reach, reach) on every axis (a
									// margin of 0.02 in k_x; the anchor test below decides).
									float lo = static_cast<float>(max(row.b, kx_lo)), hi = static_cast<float>(min(row.e - 1, kx_hi));
#pragma unroll
									for (int a = 0; a < 3; ++a)
									{
										if (fabsf(step[a]) < 1e-6f)
											continue;
										const float t1 = (gv[a] - cube - row.base[a]) * inv_step[a];
										const float t2 = (gv[a] + cube - row.base[a]) * inv_step[a];
										lo = fmaxf(lo, fminf(t1, t2) - 0.02f);
										hi = fminf(hi, fmaxf(t1, t2) + 0.02f);
									}
									const int b = static_cast<int>(ceilf(lo)), e = static_cast<int>(floorf(hi));
									for (int kx = b; kx <= e; ++kx)
									{
										const int i = row.off + kx - row.b;
										const float4 key = s_key[i];
										if (key.w == 0.0f)
											continue;
										const int ax = anchor_of<PROFILE>(key.x), ay = anchor_of<PROFILE>(key.y),
												  az = anchor_of<PROFILE>(key.z);
										const int ox = gx - ax, oy = gy - ay, oz = gz - az;
										if (static_cast<unsigned>(ox) >= static_cast<unsigned>(TAPS) ||
											static_cast<unsigned>(oy) >= static_cast<unsigned>(TAPS) ||
											static_cast<unsigned>(oz) >= static_cast<unsigned>(TAPS))
											continue;
										const float4 val = s_val[i];
										float wgt = 1.0f;
										if constexpr (TAPS == 2)
										{
											const float fxr = fsub(key.x, static_cast<float>(ax));
											const float fyr = fsub(key.y, static_cast<float>(ay));
											const float fzr = fsub(key.z, static_cast<float>(az));
											const float wx = ox ? fxr : fsub(1.0f, fxr);
											const float wy = oy ? fyr : fsub(1.0f, fyr);
											const float wz = oz ? fzr : fsub(1.0f, fzr);
											wgt = fmul(fmul(wz, wy), wx);
										}
										float are = fmul(val.x, wgt), aim = fmul(val.y, wgt);
										if (!odd)
										{
											if ((gx + sy + sz) & 1)
											{
												are = -are;
												aim = -aim;
											}
										}
										else
										{
											const float2 px = s_volume_phase[gx], py = s_volume_phase[sy];
											const float2 pz = s_volume_phase[sz];
											const float bre = fsub(fmul(are, px.x), fmul(aim, px.y));
											const float bim = fadd(fmul(are, px.y), fmul(aim, px.x));
											const float cre = fsub(fmul(bre, py.x), fmul(bim, py.y));
											const float cim = fadd(fmul(bre, py.y), fmul(bim, py.x));
											are = fsub(fmul(cre, pz.x), fmul(cim, pz.y));
											aim = fadd(fmul(cre, pz.y), fmul(cim, pz.x));
										}
										acc_re = fadd(acc_re, are);
										acc_im = fadd(acc_im, aim);
										acc_den = fadd(acc_den, fmul(val.z, wgt));
										touched = true;
									}
								}
								if (touched)
								{
									s_re[cell] = acc_re;
									s_im[cell] = acc_im;
									s_den[cell] = acc_den;
								}
							}
							r0 += nb;
						}
					}
			}
		}
	}
	__syncthreads();

	// Write back: this CTA alone owns these voxels.
	for (int i = threadIdx.x; i < cells; i += blockDim.x)
	{
		const int sz = z0 + i / (det_edge * det_edge), sy = y0 + (i / det_edge) % det_edge, x = x0 + i % det_edge;
		if (sz >= z1 || sy >= y1 || x >= x1)
			continue;
		const int64_t offset = ((int64_t)sz * big + sy) * H + x;
		num[offset] = make_float2(s_re[i], s_im[i]);
		den[offset] = s_den[i];
	}
}

// The tiles nearest the origin first (the planes cross those most): a
// counting sort of the tiles by their distance from it, in units of 8.
__global__ void __launch_bounds__(1024) det_order_kernel(const det_plan plan, int big, int *order)
{
	__shared__ int counts[128];
	__shared__ int starts[128];
	for (int i = threadIdx.x; i < 128; i += blockDim.x)
		counts[i] = 0;
	__syncthreads();
	auto key_of = [&](int t) {
		const int tz = t / (plan.tiles[1] * plan.tiles[2]);
		const int ty = (t / plan.tiles[2]) % plan.tiles[1];
		const int tx = t % plan.tiles[2];
		auto axis_distance = [&](int s0, int s1) {
			// Least |frequency| over stored indices [s0, s1).
			if (s0 == 0)
				return 0;
			const int half = big / 2;
			if (s0 <= half && half < s1)
				return min(s0, big - (s1 - 1));
			return s1 - 1 <= half ? s0 : big - (s1 - 1);
		};
		const int dz = axis_distance(tz * det_edge, min(tz * det_edge + det_edge, big));
		const int dy = axis_distance(ty * det_edge, min(ty * det_edge + det_edge, big));
		const int dx = tx * det_edge;
		const float d = sqrtf(static_cast<float>(dz * dz + dy * dy + dx * dx));
		return min(127, static_cast<int>(d / 8.0f));
	};
	for (int t = threadIdx.x; t < plan.tile_count; t += blockDim.x)
		atomicAdd(&counts[key_of(t)], 1);
	__syncthreads();
	if (threadIdx.x == 0)
	{
		int run = 0;
		for (int k = 0; k < 128; ++k)
		{
			starts[k] = run;
			run += counts[k];
		}
	}
	__syncthreads();
	// Within one distance the order is arbitrary: it changes no result.
	for (int t = threadIdx.x; t < plan.tile_count; t += blockDim.x)
		order[atomicAdd(&starts[key_of(t)], 1)] = t;
}

det_plan make_det_plan(const insertion_launch &L)
{
	const int H = L.big / 2 + 1;
	det_plan plan{};
	plan.extent[0] = plan.extent[1] = plan.extent[2] = det_edge;
	plan.tiles[0] = (L.big + det_edge - 1) / det_edge;
	plan.tiles[1] = (L.big + det_edge - 1) / det_edge;
	plan.tiles[2] = (H + det_edge - 1) / det_edge;
	plan.tile_count = plan.tiles[0] * plan.tiles[1] * plan.tiles[2];
	return plan;
}

size_t det_workspace_bytes(const insertion_launch &L)
{
	return align_up(settled_bytes * L.volumes * L.particles, 256) +
		align_up(sizeof(int) * static_cast<size_t>(make_det_plan(L).tile_count), 256);
}

template <int PROFILE, int KIND>
void launch_deterministic(const insertion_launch &L, const settled_slice *settled, int *order, cudaStream_t stream)
{
	const det_plan plan = make_det_plan(L);
	det_order_kernel<<<1, 1024, 0, stream>>>(plan, L.big, order);
	check_cuda(cudaGetLastError(), "deterministic tile order launch");
	auto kernel = insert_deterministic_kernel<PROFILE, KIND>;
	const size_t smem = sizeof(float4) * 2 * det_capacity + sizeof(float) * 3 * det_edge * det_edge * det_edge +
		(L.big % 2 ? static_cast<size_t>(L.big) * 8 : 0);
	check_cuda(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)),
		"deterministic insertion attributes");
	kernel<<<dim3(plan.tile_count, static_cast<unsigned>(L.volumes)), det_threads, smem, stream>>>(L, plan, settled,
		order);
	check_cuda(cudaGetLastError(), "deterministic insertion launch");
}

// ---------------------------------------------------------------------------
// Host side

int env_int(const char *name, int fallback)
{
	const char *v = std::getenv(name);
	if (!v || !*v)
		return fallback;
	const int x = std::atoi(v);
	return x > 0 ? x : fallback;
}

tile_plan make_plan(const insertion_launch &L, bool l2_numerator)
{
	const int taps = L.profile == REXLIB_B200_WINDOW_BOX ? 1 : 2;
	const int half = L.big / 2;
	// Anchors that can put a tap on a stored voxel: z and y frequencies in
	// [-N/2, N/2], x in [0, N/2].
	const int lo_zy = taps == 2 ? -half - 1 : -half;
	const int count_zy = half - lo_zy + 1;
	const int lo_x = taps == 2 ? -1 : 0;
	const int count_x = half - lo_x + 1;
	const int halo = taps - 1;
	// Shared bytes per cell: the denominator, plus the numerator when it is not in L2.
	const size_t cell_bytes = l2_numerator ? 4 : 12;
	const size_t smem_cells = insert_smem_budget / cell_bytes - (L.big % 2 ? (L.big * 8 + cell_bytes - 1) / cell_bytes : 0);
	const size_t l2_cells = static_cast<size_t>(std::max(512, env_int("REXLIB_B200_TILE_CELLS", static_cast<int>(l2_numerator_cells))));
	const size_t max_cells = l2_numerator ? std::min(smem_cells, l2_cells) : smem_cells;

	tile_plan best{};
	long best_score = -1;
	for (int e_zy = 4; e_zy <= count_zy; ++e_zy)
	{
		for (int e_x = 4; e_x <= count_x; ++e_x)
		{
			const size_t cells = static_cast<size_t>(e_zy + halo) * (e_zy + halo) * (e_x + halo);
			if (cells > max_cells)
				break;
			const int t_zy = (count_zy + e_zy - 1) / e_zy;
			const int t_x = (count_x + e_x - 1) / e_x;
			// Fewest tiles; then the least padding.
			const long tiles = static_cast<long>(t_zy) * t_zy * t_x;
			const long padding = static_cast<long>(t_zy * e_zy - count_zy) + (t_x * e_x - count_x);
			const long score = tiles * 100000 + padding;
			if (best_score < 0 || score < best_score)
			{
				best_score = score;
				best.extent[0] = best.extent[1] = e_zy;
				best.extent[2] = e_x;
				best.tiles[0] = best.tiles[1] = t_zy;
				best.tiles[2] = t_x;
			}
		}
	}
	best.lo[0] = best.lo[1] = lo_zy;
	best.lo[2] = lo_x;
	for (int a = 0; a < 3; ++a)
		best.box[a] = best.extent[a] + halo;
	best.tile_count = best.tiles[0] * best.tiles[1] * best.tiles[2];
	// REXLIB_B200_TILE_HITS fixes the run length; by default it follows the
	// total hit count.
	const int fixed_hits = env_int("REXLIB_B200_TILE_HITS", 0);
	best.min_hits = fixed_hits > 0 ? fixed_hits : 320;
	best.max_hits = fixed_hits > 0 ? fixed_hits : 2560;
	best.target_items = insert_grid() * 16;
	const int64_t runs_per_tile = 1 + std::min<int64_t>(L.particles, (L.particles + best.min_hits - 1) /
		best.min_hits);
	const int64_t capacity = L.volumes * best.tile_count * runs_per_tile;
	best.item_capacity = static_cast<int>(std::min<int64_t>(capacity, 1LL << 30));
	best.l2_numerator = l2_numerator;
	// The linear window's numerator tile is held twice, as x pairs (2j, 2j+1)
	// and (2j+1, 2j+2) of float4 slots, so a tap pair is one reduction
	// whatever the parity of its anchor; the nearest window's as float2 cells.
	const int64_t rows_zy = static_cast<int64_t>(best.box[0]) * best.box[1];
	best.scratch_per_cta = !l2_numerator ? 0
		: taps == 2                      ? 2 * rows_zy * (best.box[2] / 2 + 1) * 2
										 : rows_zy * best.box[2];
	return best;
}

template <int PROFILE, int KIND, bool L2_NUM>
void launch_storage(const insertion_launch &L, const tile_plan &plan, const workspace_view &w, cudaStream_t stream)
{
	auto kernel = insert_tiled_kernel<PROFILE, KIND, L2_NUM>;
	const size_t smem = sizeof(row_record) * insert_warps * 32 + (L.big % 2 ? static_cast<size_t>(L.big) * 8 : 0) +
		static_cast<size_t>(plan.box[0]) * plan.box[1] * plan.box[2] * (L2_NUM ? 4 : 12);
	check_cuda(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)),
		"tiled insertion attributes");
	kernel<<<insert_grid(), insert_threads, smem, stream>>>(L, plan, w.settled, w.item_count, w.work_counter,
		w.items, w.scratch);
	check_cuda(cudaGetLastError(), "tiled insertion launch");
}

template <int PROFILE, int KIND>
void launch_kind(const insertion_launch &L, const tile_plan &plan, const workspace_view &w, cudaStream_t stream)
{
	if (plan.l2_numerator)
		launch_storage<PROFILE, KIND, true>(L, plan, w, stream);
	else
		launch_storage<PROFILE, KIND, false>(L, plan, w, stream);
}

} // anonymous namespace

bool tiled_insertion_applies(const insertion_launch &launch, weight_kind, int mode)
{
	if (mode == REXLIB_B200_INSERT_DETERMINISTIC)
		return (launch.profile == REXLIB_B200_WINDOW_BOX || launch.profile == REXLIB_B200_WINDOW_TRIANGLE) &&
			launch.volumes * launch.particles > 0 && launch.volumes < 65536 && launch.n <= 1024;
	if (launch.profile != REXLIB_B200_WINDOW_BOX && launch.profile != REXLIB_B200_WINDOW_TRIANGLE)
		return false;
	if (std::getenv("REXLIB_B200_SCATTER_ONLY"))
		return false;
	return launch.big >= 16 && launch.n <= 1024 && launch.volumes * launch.particles > 0 &&
		launch.particles < (1LL << 30) && launch.volumes < 65536;
}

size_t tiled_insertion_workspace(const insertion_launch &launch, weight_kind, int mode, bool shared_tiles)
{
	if (mode == REXLIB_B200_INSERT_DETERMINISTIC)
		return det_workspace_bytes(launch);
	return workspace_bytes(launch.volumes, launch.particles, make_plan(launch, !shared_tiles));
}

void launch_insert_tiled(const insertion_launch &L, weight_kind kind, int mode, bool shared_tiles, void *workspace,
	size_t, cudaStream_t stream)
{
	if (mode == REXLIB_B200_INSERT_DETERMINISTIC)
	{
		settled_slice *settled = static_cast<settled_slice *>(workspace);
		int *order = reinterpret_cast<int *>(static_cast<char *>(workspace) +
			align_up(settled_bytes * L.volumes * L.particles, 256));
		const int64_t slices = L.volumes * L.particles;
		settle_kernel<<<static_cast<unsigned>((slices + settle_threads / 32 - 1) / (settle_threads / 32)),
			settle_threads, 0, stream>>>(L, settled, static_cast<int>(kind));
		check_cuda(cudaGetLastError(), "settle launch");
		const bool box = L.profile == REXLIB_B200_WINDOW_BOX;
		switch (kind)
		{
		case weight_kind::unit:
			box ? launch_deterministic<REXLIB_B200_WINDOW_BOX, 0>(L, settled, order, stream)
				: launch_deterministic<REXLIB_B200_WINDOW_TRIANGLE, 0>(L, settled, order, stream);
			break;
		case weight_kind::ctf:
			box ? launch_deterministic<REXLIB_B200_WINDOW_BOX, 1>(L, settled, order, stream)
				: launch_deterministic<REXLIB_B200_WINDOW_TRIANGLE, 1>(L, settled, order, stream);
			break;
		case weight_kind::spectrum:
			box ? launch_deterministic<REXLIB_B200_WINDOW_BOX, 2>(L, settled, order, stream)
				: launch_deterministic<REXLIB_B200_WINDOW_TRIANGLE, 2>(L, settled, order, stream);
			break;
		}
		return;
	}
	const tile_plan plan = make_plan(L, !shared_tiles);
	const workspace_view w = view_workspace(workspace, L.volumes, L.particles, plan);
	const int64_t slices = L.volumes * L.particles;
	settle_kernel<<<static_cast<unsigned>((slices + settle_threads / 32 - 1) / (settle_threads / 32)), settle_threads,
		0, stream>>>(L, w.settled, static_cast<int>(kind));
	check_cuda(cudaGetLastError(), "settle launch");
	count_hits_kernel<<<dim3(plan.tile_count, static_cast<unsigned>(L.volumes)), count_threads, 0, stream>>>(
		L, plan, w.settled, w.counts);
	check_cuda(cudaGetLastError(), "hit count launch");
	plan_items_kernel<<<1, 1024, 0, stream>>>(plan, L.volumes, L.particles, w.counts, w.item_count, w.work_counter,
		w.items);
	check_cuda(cudaGetLastError(), "plan launch");
	const bool box = L.profile == REXLIB_B200_WINDOW_BOX;
	switch (kind)
	{
	case weight_kind::unit:
		box ? launch_kind<REXLIB_B200_WINDOW_BOX, 0>(L, plan, w, stream)
			: launch_kind<REXLIB_B200_WINDOW_TRIANGLE, 0>(L, plan, w, stream);
		break;
	case weight_kind::ctf:
		box ? launch_kind<REXLIB_B200_WINDOW_BOX, 1>(L, plan, w, stream)
			: launch_kind<REXLIB_B200_WINDOW_TRIANGLE, 1>(L, plan, w, stream);
		break;
	case weight_kind::spectrum:
		box ? launch_kind<REXLIB_B200_WINDOW_BOX, 2>(L, plan, w, stream)
			: launch_kind<REXLIB_B200_WINDOW_TRIANGLE, 2>(L, plan, w, stream);
		break;
	}
}

// Throughput: settle, count, plan, insert; deterministic: settle, tile order, insert.
int tiled_insertion_launches(int mode) { return mode == REXLIB_B200_INSERT_DETERMINISTIC ? 3 : 4; }

} // namespace rexlib_b200
