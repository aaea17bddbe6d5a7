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
#include <type_traits>

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
	float k_shift;     // K offset of the region a tile's anchors own: w - 1 for the Kaiser-Bessel window (its
					   // first tap is floor(K - w) + 1), 0 otherwise
};

struct work_item
{
	int volume; // the volume; in a batched call, the job in its bits 16 and up
	int tile;
	int first;
	int last;
};

// The deterministic mode's tiles: 16^3 stored voxels (the gather below).
struct det_plan
{
	int extent[3]; // stored voxels per tile (z, y, x)
	int tiles[3];
	int tile_count;
};

// A batched call: many reconstructions (jobs) of uneven box size and
// particle count in one set of launches, one persistent insertion launch
// claiming the work items of every job. The jobs travel by value in the
// kernels' parameters (CUDA 12.1 and later take up to 32,764 bytes of them),
// so a call reads nothing from the host and captures into a CUDA graph.
constexpr int max_batch_jobs = 64;
constexpr int batch_job_bits = 16; // a work item's volume: job << 16 | volume

struct batch_job
{
	insertion_launch launch;
	tile_plan plan;         // throughput mode
	det_plan dplan;         // deterministic mode
	int64_t settled_offset; // the job's first settled slice
	int64_t cell_offset;    // the job's first (volume, tile) cell
};

struct batch_param
{
	int job_count;
	int64_t slices; // settled slices of all jobs
	int64_t cells;  // (volume, tile) cells of all jobs
	batch_job jobs[max_batch_jobs];
};
static_assert(sizeof(batch_param) <= 30000, "the jobs must fit a kernel's parameters");

struct no_batch
{
};
template <bool BATCHED>
using batch_arg = typename std::conditional<BATCHED, batch_param, no_batch>::type;

// The job holding settled slice `index` (or (volume, tile) cell `index`):
// the last whose first one is at or below it.
__device__ __forceinline__ int job_of_slice(const batch_param &b, int64_t index)
{
	int j = 0;
	while (j + 1 < b.job_count && b.jobs[j + 1].settled_offset <= index)
		++j;
	return j;
}

__device__ __forceinline__ int job_of_cell(const batch_param &b, int64_t index)
{
	int j = 0;
	while (j + 1 < b.job_count && b.jobs[j + 1].cell_offset <= index)
		++j;
	return j;
}

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

// Settles slice p of volume v into *out, with the 32 lanes of a warp.
__device__ __forceinline__ void settle_slice(const insertion_launch &L, int64_t v, int64_t p, int lane,
	settled_slice *out, int kind)
{
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
	*out = r;
}

__global__ void __launch_bounds__(settle_threads) settle_kernel(const insertion_launch L, settled_slice *out,
	int kind)
{
	const int64_t index = (static_cast<int64_t>(blockIdx.x) * settle_threads + threadIdx.x) >> 5;
	if (index >= L.volumes * L.particles)
		return;
	settle_slice(L, index / L.particles, index % L.particles, threadIdx.x & 31, out + index, kind);
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
	b.lower[0] = lo[2] - 1.0f + plan.k_shift;
	b.upper[0] = lo[2] + plan.extent[2] + 1.0f + plan.k_shift;
	b.lower[1] = lo[1] - 1.0f + plan.k_shift;
	b.upper[1] = lo[1] + plan.extent[1] + 1.0f + plan.k_shift;
	b.lower[2] = lo[0] - 1.0f + plan.k_shift;
	b.upper[2] = lo[0] + plan.extent[0] + 1.0f + plan.k_shift;
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

// The slices of volume v whose plane can reach `tile`, counted by the CTA
// into *count.
__device__ __forceinline__ void count_tile_hits(const insertion_launch &L, const tile_plan &plan,
	const settled_slice *settled, int64_t v, int tile, int *count)
{
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
		*count = total;
	}
}

__global__ void __launch_bounds__(count_threads) count_hits_kernel(const insertion_launch L, const tile_plan plan,
	const settled_slice *settled, int *counts)
{
	const int tile = blockIdx.x;
	const int64_t v = blockIdx.y;
	count_tile_hits(L, plan, settled, v, tile, counts + v * plan.tile_count + tile);
}

// The batched forms of passes 0 and 1: one launch each over every job's
// slices and (volume, tile) cells.
__global__ void __launch_bounds__(settle_threads) settle_batch_kernel(const __grid_constant__ batch_param b,
	settled_slice *out, int kind)
{
	const int64_t index = (static_cast<int64_t>(blockIdx.x) * settle_threads + threadIdx.x) >> 5;
	if (index >= b.slices)
		return;
	const batch_job &job = b.jobs[job_of_slice(b, index)];
	const int64_t local = index - job.settled_offset;
	settle_slice(job.launch, local / job.launch.particles, local % job.launch.particles, threadIdx.x & 31,
		out + index, kind);
}

__global__ void __launch_bounds__(count_threads) count_hits_batch_kernel(const __grid_constant__ batch_param b,
	const settled_slice *settled, int *counts)
{
	const int64_t cell = blockIdx.x;
	const batch_job &job = b.jobs[job_of_cell(b, cell)];
	const int64_t local = cell - job.cell_offset;
	count_tile_hits(job.launch, job.plan, settled + job.settled_offset, local / job.plan.tile_count,
		static_cast<int>(local % job.plan.tile_count), counts + cell);
}

// ---------------------------------------------------------------------------
// Pass 2: runs of slices per tile

// In a batched call `plan` holds the run lengths and capacities common to
// the jobs, and every (volume, tile) cell of every job is planned.
template <bool BATCHED>
__global__ void __launch_bounds__(1024) plan_items_kernel(const tile_plan plan, int64_t volumes, int64_t particles,
	const int *counts, int *item_count, int *work_counter, work_item *items, const __grid_constant__ batch_arg<BATCHED> b)
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
	int64_t cells = volumes * plan.tile_count;
	if constexpr (BATCHED)
		cells = b.cells;
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
		// The cell's volume (a batched call: job << 16 | volume), tile and slices.
		int volume = 0, tile = 0;
		int64_t cell_particles = particles;
		if (i < cells)
		{
			if constexpr (BATCHED)
			{
				const int j = job_of_cell(b, i);
				const batch_job &job = b.jobs[j];
				const int64_t local = i - job.cell_offset;
				volume = (j << batch_job_bits) | static_cast<int>(local / job.plan.tile_count);
				tile = static_cast<int>(local % job.plan.tile_count);
				cell_particles = job.launch.particles;
			}
			else
			{
				volume = static_cast<int>(i / plan.tile_count);
				tile = static_cast<int>(i % plan.tile_count);
			}
			const int c = counts[i];
			runs = c == 0 ? 0 : (c + hits_per_item - 1) / hits_per_item;
			runs = static_cast<int>(runs < cell_particles ? runs : cell_particles);
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
			const int64_t span = (cell_particles + runs - 1) / runs;
			for (int r = 0; r < runs; ++r)
			{
				const int64_t first = r * span;
				const int64_t last = first + span < cell_particles ? first + span : cell_particles;
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

// The shift phase exp(i a f) of signed frequency f as the CPU tabulates it
// (kernels/axis_phase.inl:16-35): the angle a f in FP64, its cosine and sine
// in FP64, each rounded to float. `a` is 2 pi (n/2 + t) / n, evaluated in
// that order. The FP64 cosine and sine here and in the CPU's libm are both
// within two units of the last FP64 place, so their float roundings agree
// unless the value lies within that distance of a float rounding boundary.
__device__ __forceinline__ float2 exact_shift_phase(double angle_step, int f)
{
	double s, c;
	sincos(angle_step * static_cast<double>(f), &s, &c);
	return make_float2(static_cast<float>(c), static_cast<float>(s));
}

__device__ __forceinline__ float2 cmul(float2 a, float2 b)
{
	return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// a b as two packed FP32 operations: (a.x b.x, a.x b.y) + (-a.y b.y, a.y b.x).
__device__ __forceinline__ float2 cmul2(float2 a, float2 b)
{
	return __ffma2_rn(make_float2(-a.y, a.y), make_float2(b.y, b.x), __fmul2_rn(make_float2(a.x, a.x), b));
}

// An L2 policy that keeps lines past the streaming data: the numerator
// scratch of a CTA is reduced into and re-read at every flush, while the
// slices stream through L2 once.
__device__ __forceinline__ uint64_t evict_last_policy()
{
	uint64_t policy;
	asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(policy));
	return policy;
}

__device__ __forceinline__ float2 load_scratch(const float2 *p, uint64_t policy)
{
	float2 v;
	asm volatile("ld.global.cg.L2::cache_hint.v2.f32 {%0, %1}, [%2], %3;" : "=f"(v.x), "=f"(v.y) : "l"(p), "l"(policy));
	return v;
}

__device__ __forceinline__ void store_scratch(float2 *p, float2 v, uint64_t policy)
{
	asm volatile("st.global.cg.L2::cache_hint.v2.f32 [%0], {%1, %2}, %3;" ::"l"(p), "f"(v.x), "f"(v.y), "l"(policy)
				 : "memory");
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
		// floor(c): one conversion rounding toward minus infinity (0 for NaN, as truncation gives).
		return __float2int_rd(c);
	}
}

// The Kaiser-Bessel window of one tap at `distance` from K, by the table
// lerp of kernels/kaiser_bessel_window.inl:80-136 (as `place` computes it).
__device__ __forceinline__ float kb_weight(float distance, float scale, int step_count, const float *values)
{
	const float position = fmul(distance, scale);
	const int step = static_cast<int>(position);
	const int index = step < step_count ? step : step_count + 1;
	const float fraction = fsub(position, static_cast<float>(index));
	const float below = values[index];
	return fadd(below, fmul(fraction, fsub(values[index + 1], below)));
}

// The first tap of the Kaiser-Bessel window at c: floor(c - w) + 1.
__device__ __forceinline__ int kb_first(float c, float half_width)
{
	return __float2int_rd(fsub(c, half_width)) + 1;
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

// What a window adds to the tiled kernel's parameters: the Kaiser-Bessel
// table (by value, like the scatter kernel's), nothing for the others.
template <int PROFILE, typename TABLE = kb_table>
struct window_param
{
};
template <typename TABLE>
struct window_param<REXLIB_B200_WINDOW_KAISER_BESSEL, TABLE>
{
	TABLE kb;
};

// The Kaiser-Bessel table of one call, or of a batched call.
template <bool BATCHED>
using kb_table_for = typename std::conditional<BATCHED, kb_table_batch, kb_table>::type;

// The volume phase table exp(-2 pi i f (-N/2) / N) of an odd N, by stored
// index (tabulated_phase.inl:26-36), filled by the CTA.
__device__ __forceinline__ void fill_volume_phase(float2 *table, int big)
{
	const int half = big / 2;
	const double s = 2.0 * pi * (-static_cast<double>(half)) / static_cast<double>(big);
	for (int j = threadIdx.x; j < big; j += blockDim.x)
	{
		const double f = j <= half ? static_cast<double>(j) : static_cast<double>(j - big);
		double sn, cs;
		sincos(s * f, &sn, &cs);
		table[j] = make_float2(static_cast<float>(cs), static_cast<float>(sn));
	}
}

// A launch's (or a batched call's job's) operands and tile plan.
template <bool BATCHED>
__device__ __forceinline__ const insertion_launch &launch_of(const insertion_launch &call, const batch_arg<BATCHED> &b,
	int job)
{
	if constexpr (BATCHED)
		return b.jobs[job].launch;
	else
		return call;
}

template <bool BATCHED>
__device__ __forceinline__ const tile_plan &plan_of(const tile_plan &call, const batch_arg<BATCHED> &b, int job)
{
	if constexpr (BATCHED)
		return b.jobs[job].plan;
	else
		return call;
}

template <bool BATCHED>
__device__ __forceinline__ const det_plan &det_plan_of(const det_plan &call, const batch_arg<BATCHED> &b, int job)
{
	if constexpr (BATCHED)
		return b.jobs[job].dplan;
	else
		return call;
}

// In a batched call (BATCHED), L_call and plan_call hold what the CTA sizes
// its storage by over all jobs: L_call.big the largest odd volume extent (0
// when none), plan_call.box the largest tile box and scratch_per_cta the
// largest numerator tile; each work item then takes its job's operands and
// plan from `b`.
template <int PROFILE, int KIND, bool L2_NUM, bool BATCHED>
__global__ void __launch_bounds__(insert_threads, insert_blocks_per_sm) insert_tiled_kernel(const insertion_launch L_call,
	const tile_plan plan_call, const settled_slice *settled_call, const int *item_count, int *work_counter,
	const work_item *items, float2 *scratch, const __grid_constant__ window_param<PROFILE, kb_table_for<BATCHED>> wp,
	const __grid_constant__ batch_arg<BATCHED> b)
{
	constexpr bool KB = PROFILE == REXLIB_B200_WINDOW_KAISER_BESSEL;
	constexpr int TAPS = PROFILE == REXLIB_B200_WINDOW_BOX ? 1 : 2; // the nearest and linear windows' taps
	constexpr int shared_arrays = L2_NUM ? 1 : 3;
	extern __shared__ float4 smem_raw[];
	const int max_cells = plan_call.box[0] * plan_call.box[1] * plan_call.box[2];
	const int table_big = (L_call.big & 1) ? L_call.big : 0;
	// Row records first (16-byte aligned), then the volume phase table (odd
	// N), then the accumulators.
	row_record *warp_rows = reinterpret_cast<row_record *>(smem_raw);
	float2 *s_volume_phase = reinterpret_cast<float2 *>(warp_rows + insert_warps * 32);
	float *s_kb = reinterpret_cast<float *>(s_volume_phase + table_big); // Kaiser-Bessel table
	int kb_floats = 0;
	if constexpr (KB)
		kb_floats = wp.kb.step_count + 3;
	float *s_den = s_kb + kb_floats;
	float *s_re = s_den + max_cells; // shared numerator (!L2_NUM)
	float *s_im = s_re + max_cells;
	// L2 numerator: float2 cells (nearest), or the two paired float4 layouts
	// (linear): g_even slot j of a row holds x = 2j and 2j+1, g_odd slot j
	// holds 2j+1 and 2j+2.
	constexpr bool PAIRED = L2_NUM && (PROFILE == REXLIB_B200_WINDOW_TRIANGLE || KB);
	float2 *g_num = L2_NUM ? scratch + static_cast<int64_t>(blockIdx.x) * plan_call.scratch_per_cta : nullptr;
	const uint64_t keep = evict_last_policy();
	if constexpr (L2_NUM)
		for (int64_t i = threadIdx.x; i < plan_call.scratch_per_cta; i += blockDim.x)
			store_scratch(g_num + i, make_float2(0.0f, 0.0f), keep);
	__shared__ int s_item;
	__shared__ int s_next_particle;

	const int lane = threadIdx.x & 31;
	const int warp = threadIdx.x >> 5;

	// The extent the phase table holds (a batched call refills it when a job
	// of another odd extent comes).
	int table_of = 0;
	if (!BATCHED && table_big > 0)
	{
		fill_volume_phase(s_volume_phase, table_big);
		table_of = table_big;
	}
	if constexpr (KB)
		for (int j = threadIdx.x; j < kb_floats; j += blockDim.x)
			s_kb[j] = wp.kb.values[j];

	const int total_items = *item_count;
	for (;;)
	{
		if (threadIdx.x == 0)
		{
			s_item = atomicAdd(work_counter, 1);
			s_next_particle = 0;
		}
		for (int i = threadIdx.x; i < shared_arrays * max_cells; i += blockDim.x)
			s_den[i] = 0.0f;
		__syncthreads();
		const int item_index = s_item;
		if (item_index >= total_items)
			break;
		const work_item item = items[item_index];
		int job = 0;
		int64_t v = item.volume;
		if constexpr (BATCHED)
		{
			job = item.volume >> batch_job_bits;
			v = item.volume & ((1 << batch_job_bits) - 1);
		}
		const insertion_launch &L = launch_of<BATCHED>(L_call, b, job);
		const tile_plan &plan = plan_of<BATCHED>(plan_call, b, job);
		const settled_slice *settled = settled_call;
		if constexpr (BATCHED)
			settled += b.jobs[job].settled_offset;
		const int n = L.n, h = L.h, big = L.big, H = L.big_h;
		const int half = big / 2;
		const bool odd = (big & 1) != 0;
		const int cells = plan.box[0] * plan.box[1] * plan.box[2];
		const int bx = plan.box[2], by = plan.box[1];
		const int plane = by * bx;
		const int last_column = h - (n % 2 == 0 ? 2 : 1);
		const int highest_row = n % 2 == 0 ? n / 2 - 1 : n / 2;
		const int sx = plan.box[2] / 2 + 1;
		float4 *g_even = reinterpret_cast<float4 *>(g_num);
		float4 *g_odd = g_even + static_cast<int64_t>(plan.box[0]) * plan.box[1] * sx;
		if (BATCHED && odd && table_of != big)
		{
			// Every thread agrees on the job; the barrier before the next
			// item's claim keeps the table until this item's flush is done.
			fill_volume_phase(s_volume_phase, big);
			table_of = big;
			__syncthreads();
		}
		int lo[3];
		const k_bounds bounds = tile_bounds(plan, item.tile, lo);
		// The K region the tile owns, with a margin far above float rounding:
		// [lo, lo + extent) for the linear window (anchor floor(K)), half a
		// voxel lower for the nearest (anchor round(K)). Rows and columns are
		// clipped to it; the anchor test then decides exactly.
		k_bounds owned;
		{
			const float shift = KB ? -plan.k_shift : (TAPS == 1 ? 0.5f : 0.0f);
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
						int ax, ay, az;
						if constexpr (KB)
						{
							ax = kb_first(cx, wp.kb.half_width) - lo[2];
							ay = kb_first(cy, wp.kb.half_width) - lo[1];
							az = kb_first(cz, wp.kb.half_width) - lo[0];
						}
						else
						{
							ax = anchor_of<PROFILE>(cx) - lo[2];
							ay = anchor_of<PROFILE>(cy) - lo[1];
							az = anchor_of<PROFILE>(cz) - lo[0];
						}
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
						const float2 value = cmul2(cmul2(sample, shift_phase(S.qx, kx)), row_y_phase);
						const float sc = r * wnum;
						const float2 v2 = __fmul2_rn(value, make_float2(sc, sgn ? -sc : sc));
						const float vre = v2.x;
						const float vim = v2.y;
						const float cnt = r * wden;
						const int cell = (az * by + ay) * bx + ax;
						if constexpr (KB)
						{
							// Taps first .. first + taps - 1 per axis (taps <= 4 on this
							// path), each weighted by the table lerp at its distance from
							// K; (w_z w_y) w_x as the CPU.
							const int taps = wp.kb.tap_count;
							const float scale = wp.kb.scale;
							const int steps = wp.kb.step_count;
							float wx[4], wy[4], wz[4];
#pragma unroll
							for (int t = 0; t < 4; ++t)
							{
								wx[t] = t < taps ? kb_weight(fabsf(fsub(static_cast<float>(ax + lo[2] + t), cx)), scale, steps, s_kb) : 0.0f;
								wy[t] = t < taps ? kb_weight(fabsf(fsub(static_cast<float>(ay + lo[1] + t), cy)), scale, steps, s_kb) : 0.0f;
								wz[t] = t < taps ? kb_weight(fabsf(fsub(static_cast<float>(az + lo[0] + t), cz)), scale, steps, s_kb) : 0.0f;
							}
#pragma unroll
							for (int dz = 0; dz < 4; ++dz)
							{
								if (dz >= taps)
									break;
#pragma unroll
								for (int dy = 0; dy < 4; ++dy)
								{
									if (dy >= taps)
										break;
									const float wzy = fmul(wz[dz], wy[dy]);
									const int c = cell + dz * plane + dy * bx;
									if constexpr (PAIRED)
									{
										// x taps (0, 1) and (2, 3) as pairs, a third one alone: all
										// start at the parity of ax, so one layout takes them.
										const int64_t row = static_cast<int64_t>((az + dz) * by + (ay + dy)) * sx;
										float4 *slots = ((ax & 1) ? g_odd : g_even) + row + (ax >> 1);
#pragma unroll
										for (int dx = 0; dx < 4; dx += 2)
										{
											if (dx >= taps)
												break;
											const float w0 = fmul(wzy, wx[dx]);
											atomicAdd(s_den + c + dx, cnt * w0);
											if (dx + 1 < taps)
											{
												const float w1 = fmul(wzy, wx[dx + 1]);
												asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(slots + dx / 2),
															 "f"(vre * w0), "f"(vim * w0), "f"(vre * w1), "f"(vim * w1)
															 : "memory");
												atomicAdd(s_den + c + dx + 1, cnt * w1);
											}
											else
											{
												// x = ax + dx alone: its half of the even layout.
												float2 *half_slot = reinterpret_cast<float2 *>(g_even) + 2 * row + ax + dx;
												asm volatile("red.global.add.v2.f32 [%0], {%1, %2};" ::"l"(half_slot), "f"(vre * w0),
															 "f"(vim * w0) : "memory");
											}
										}
									}
									else
									{
#pragma unroll
										for (int dx = 0; dx < 4; ++dx)
										{
											if (dx >= taps)
												break;
											const float w = fmul(wzy, wx[dx]);
											add_tap<L2_NUM>(g_num, s_re, s_im, s_den, c + dx, vre * w, vim * w, cnt * w);
										}
									}
								}
							}
						}
						else if constexpr (TAPS == 1)
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
							// The tap weights and contributions as packed FP32 pairs
							// (two lanes of one instruction on sm_100).
							const float2 wy2 = make_float2(wy[0], wy[1]);
							const float2 wx2 = make_float2(wx[0], wx[1]);
							const float2 cc = make_float2(cnt, cnt);
#pragma unroll
							for (int dz = 0; dz < 2; ++dz)
#pragma unroll
								for (int dy = 0; dy < 2; ++dy)
								{
									const float2 wzy2 = __fmul2_rn(make_float2(wz[dz], wz[dz]), wy2);
									const float wzy = dy ? wzy2.y : wzy2.x;
									if constexpr (PAIRED)
									{
										const float2 w = __fmul2_rn(make_float2(wzy, wzy), wx2);
										const float2 a0 = __fmul2_rn(v2, make_float2(w.x, w.x));
										const float2 a1 = __fmul2_rn(v2, make_float2(w.y, w.y));
										const float2 dd = __fmul2_rn(cc, w);
										const int c = cell + dz * plane + dy * bx;
										float4 *slot = ((ax & 1) ? g_odd : g_even) + ((az + dz) * by + (ay + dy)) * sx + (ax >> 1);
										asm volatile("red.global.add.L2::cache_hint.v4.f32 [%0], {%1, %2, %3, %4}, %5;" ::"l"(slot),
													 "f"(a0.x), "f"(a0.y), "f"(a1.x), "f"(a1.y), "l"(keep)
													 : "memory");
										atomicAdd(s_den + c, dd.x);
										atomicAdd(s_den + c + 1, dd.y);
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
				const float2 a = load_scratch(e, keep);
				re = a.x;
				im = a.y;
				if (re != 0.0f || im != 0.0f)
					store_scratch(e, make_float2(0.0f, 0.0f), keep);
				if (cx >= 1)
				{
					float2 *o = reinterpret_cast<float2 *>(g_odd) + row + cx - 1;
					const float2 b = load_scratch(o, keep);
					if (b.x != 0.0f || b.y != 0.0f)
					{
						re += b.x;
						im += b.y;
						store_scratch(o, make_float2(0.0f, 0.0f), keep);
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
// The work comes in stages of up to 8 slices, 512 rows and 2,048 samples; a
// stage may end inside a slice, at a row boundary, and the next one resumes
// there. A stage computes, each step parallel over the whole stage:
// - its units (slice, sign, interval pair): the rows that reach the tile
//   (bound_rows of kernels/row_interval.cpp:84-136);
// - its rows: the columns that reach the tile (clip_row, :34-82), the row
//   base and y phase;
// - its samples: K, the window's anchor and fractions, the value and the
//   denominator weight, as the CPU's prepare (row_insertion_kernel.inl:139-285).
// Then every thread gathers for its pillar of the tile, along the axis the
// slice's normal leans on most, its half of the voxels (alternate stored
// indices). A sample reaches a voxel of the pillar only when its K lies
// within the window of the pillar's two fixed coordinates, so the pillar
// visits the few rows whose line crosses that 2x2 cross-section, and in each
// the few columns that do; the anchor test decides exactly. Rows ascend and
// columns ascend, so every voxel adds its contributions in the CPU's order.
// Units of one pillar axis share the voxel owners, so the gather of a stage
// needs a barrier only where the axis changes.

constexpr int det_threads = 512;
constexpr int det_edge = 16;                              // tile edge: det_edge^2 pillars, two threads each
constexpr int det_stage_slices = 8;                       // slices a stage takes at most
constexpr int det_unit_combos = 8;                        // units per slice at most: 2 signs x 2 x 2 interval pairs
constexpr int det_stage_units = det_stage_slices * det_unit_combos;
constexpr int det_stage_rows = det_threads;               // rows a stage holds: one thread each
constexpr int det_stage_samples = 2048;                   // samples a stage holds (a row has at most n/2 + 1)
static_assert(2 * det_edge * det_edge == det_threads, "two threads a pillar");
static_assert(det_stage_units <= 64, "the unit scan covers two entries a lane");

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

// A unit of a stage: (slice, sign, interval pair) and its rows there.
struct det_unit
{
	int slice, sgn, zi, yi;
	int row_begin; // k_y of the unit's first row in the stage
	int rows;      // its rows in the stage
	int row_first; // index of its first row in the stage's row table
	int axis;      // pillar axis (0 x, 1 y, 2 z): the one the normal leans on most
	float step[3], inv_step[3];
	float step_b, inv_b, step_c, inv_c; // the step along the pillar's lower (b) and higher (c) fixed axes
	float ky_b, ky_c, ky_half;          // a pillar's rows: k_y* = ky_b F_b + ky_c F_c, within ky_half
};

// A tile cell: x swizzled by y, so that the pillars of a warp, along any
// axis, meet few bank conflicts.
__device__ __forceinline__ int det_cell(int z, int y, int x)
{
	return (z * det_edge + y) * det_edge + (x ^ (y & (det_edge - 1)));
}

// In a batched call (BATCHED) tile_order lists the (volume, tile) cells of
// every job, and the CTA takes its job's operands and plan from `b`.
template <int PROFILE, int KIND, bool BATCHED>
__global__ void __launch_bounds__(det_threads, 1) insert_deterministic_kernel(const insertion_launch L_call,
	const det_plan plan_call, const settled_slice *settled_call, const int *tile_order,
	const __grid_constant__ kb_table_for<BATCHED> kb, const __grid_constant__ batch_arg<BATCHED> b)
{
	int job = 0;
	int64_t v = blockIdx.y;
	int tile = 0;
	if constexpr (BATCHED)
	{
		const int64_t cell = tile_order[blockIdx.x];
		job = job_of_cell(b, cell);
		const int64_t local = cell - b.jobs[job].cell_offset;
		v = local / b.jobs[job].dplan.tile_count;
		tile = static_cast<int>(local % b.jobs[job].dplan.tile_count);
	}
	else
	{
		tile = tile_order[blockIdx.x];
	}
	const insertion_launch &L = launch_of<BATCHED>(L_call, b, job);
	const det_plan &plan = det_plan_of<BATCHED>(plan_call, b, job);
	const settled_slice *settled = settled_call;
	if constexpr (BATCHED)
		settled += b.jobs[job].settled_offset;
	constexpr bool KB = PROFILE == REXLIB_B200_WINDOW_KAISER_BESSEL;
	constexpr int TAPS = PROFILE == REXLIB_B200_WINDOW_BOX ? 1 : 2; // taps of the nearest and linear windows
	const int taps = KB ? kb.tap_count : TAPS;
	constexpr int cells = det_edge * det_edge * det_edge;
	// A sample reaches voxel g when its K lies in g + [-cube, cube) per axis:
	// within a voxel (linear), half a voxel (nearest), or for the
	// Kaiser-Bessel window of half-width w, with g at or past the first tap
	// floor(K - w) + 1 and within the taps after it: w + 1 bounds both.
	const float cube = KB ? kb.half_width + 1.0f : (TAPS == 2 ? 1.0f : 0.5f);
	const float margin = cube + 0.05f;
	extern __shared__ float4 smem_raw[];
	// Per sample: the anchor (the first tap per axis), fractions past it (the
	// Kaiser-Bessel window: K itself), the denominator weight, the value.
	float4 *s_frac = smem_raw;                                                 // fractions (or K) x, y, z; denominator weight
	float2 *s_val = reinterpret_cast<float2 *>(s_frac + det_stage_samples);    // numerator value
	short4 *s_anchor = reinterpret_cast<short4 *>(s_val + det_stage_samples); // anchor x, y, z; w = 1 when it inserts
	float2 *s_num = reinterpret_cast<float2 *>(s_anchor + det_stage_samples);
	float *s_den = reinterpret_cast<float *>(s_num + cells);
	float2 *s_volume_phase = reinterpret_cast<float2 *>(s_den + cells); // odd N
	float *s_kb = reinterpret_cast<float *>(s_volume_phase + ((L.big & 1) ? L.big : 0)); // Kaiser-Bessel table
	__shared__ int4 s_row_i[det_stage_rows];   // first and end column, first sample, k_y
	__shared__ float4 s_row_f[det_stage_rows]; // base x, y, z; unit
	__shared__ float2 s_row_phase[det_stage_rows];
	__shared__ det_unit s_units[det_stage_units];
	__shared__ settled_slice s_slices[det_stage_slices];
	__shared__ long long s_particle[det_stage_slices];
	__shared__ double2 s_angle[det_stage_slices]; // the x and y shift phases' angle steps
	__shared__ int s_hits[det_threads];
	__shared__ int s_scan[det_threads / 32];
	__shared__ int s_hit_count, s_all_rows, s_stage_samples, s_next[3];

	const int n = L.n, h = L.h, big = L.big, H = L.big_h;
	const int half = big / 2;
	const int last_column = h - (n % 2 == 0 ? 2 : 1);
	const int highest_row = n % 2 == 0 ? n / 2 - 1 : n / 2;
	const bool odd = (big & 1) != 0;
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	const int tz = tile / (plan.tiles[1] * plan.tiles[2]);
	const int ty = (tile / plan.tiles[2]) % plan.tiles[1];
	const int tx = tile % plan.tiles[2];
	const int z0 = tz * det_edge, y0 = ty * det_edge, x0 = tx * det_edge;
	const int z1 = min(z0 + det_edge, big), y1 = min(y0 + det_edge, big), x1 = min(x0 + det_edge, H);

	if (odd)
		fill_volume_phase(s_volume_phase, big);
	if constexpr (KB)
		for (int i = threadIdx.x; i < kb.step_count + 3; i += blockDim.x)
			s_kb[i] = kb.values[i];
	float2 *num = L.numerator + v * (int64_t)big * big * H;
	float *den = L.denominator + v * (int64_t)big * big * H;
	for (int i = threadIdx.x; i < cells; i += blockDim.x)
	{
		const int lz = i / (det_edge * det_edge), ly = (i / det_edge) % det_edge, lx = i % det_edge;
		float2 a = make_float2(0.0f, 0.0f);
		float d = 0.0f;
		if (z0 + lz < z1 && y0 + ly < y1 && x0 + lx < x1)
		{
			const int64_t offset = ((int64_t)(z0 + lz) * big + (y0 + ly)) * H + (x0 + lx);
			a = num[offset];
			d = den[offset];
		}
		s_num[det_cell(lz, ly, lx)] = a;
		s_den[det_cell(lz, ly, lx)] = d;
	}

	int zl[2], zu[2], yl[2], yu[2];
	const int zcount = det_intervals(z0, z1, big, zl, zu);
	const int ycount = det_intervals(y0, y1, big, yl, yu);
	const int combos = 2 * zcount * ycount; // units a slice has
	// The K region whose taps can reach any voxel of the tile.
	k_bounds whole;
	whole.lower[0] = x0 - margin;
	whole.upper[0] = x1 - 1 + margin;
	whole.lower[1] = fminf(yl[0], yl[ycount - 1]) - margin;
	whole.upper[1] = fmaxf(yu[0], yu[ycount - 1]) + margin;
	whole.lower[2] = fminf(zl[0], zl[zcount - 1]) - margin;
	whole.upper[2] = fmaxf(zu[0], zu[zcount - 1]) + margin;
	auto unit_bounds = [&](int zi, int yi) {
		k_bounds b;
		b.lower[0] = x0 - margin;
		b.upper[0] = x1 - 1 + margin;
		b.lower[1] = (yi ? yl[1] : yl[0]) - margin;
		b.upper[1] = (yi ? yu[1] : yu[0]) + margin;
		b.lower[2] = (zi ? zl[1] : zl[0]) - margin;
		b.upper[2] = (zi ? zu[1] : zu[0]) + margin;
		return b;
	};
	// Pillar (p1, p2): p2 along the lower fixed axis, p1 along the higher;
	// the pillar's two threads take the stored indices of parity half_of.
	const int pillar = threadIdx.x % (det_edge * det_edge), half_of = threadIdx.x / (det_edge * det_edge);
	const int p1 = pillar / det_edge, p2 = pillar % det_edge;

	for (int64_t chunk = 0; chunk < L.particles; chunk += det_threads)
	{
		// The slices of the chunk that reach the tile, in index order.
		const int64_t mine = chunk + threadIdx.x;
		const bool hit = mine < L.particles && plane_reaches(settled[v * L.particles + mine], whole);
		const unsigned hits = __ballot_sync(0xffffffffu, hit);
		__syncthreads(); // the previous chunk is done with the hit list
		if (lane == 0)
			s_scan[warp] = __popc(hits);
		__syncthreads();
		int before = 0;
		for (int w = 0; w < warp; ++w)
			before += s_scan[w];
		if (hit)
			s_hits[before + __popc(hits & ((1u << lane) - 1u))] = threadIdx.x;
		if (threadIdx.x == det_threads - 1)
			s_hit_count = before + __popc(hits);
		__syncthreads();
		const int hit_count = s_hit_count;

		// The stage cursor: hit index, unit of that slice, rows of the unit done.
		int cursor_slice = 0, cursor_combo = 0, cursor_row = 0;
		while (cursor_slice < hit_count)
		{
			const int G = min(det_stage_slices, hit_count - cursor_slice);
			const int units = G * combos;
			__syncthreads(); // the previous stage is done with every table
			for (int w = threadIdx.x; w < G * static_cast<int>(sizeof(settled_slice) / 4); w += det_threads)
			{
				const int g = w / static_cast<int>(sizeof(settled_slice) / 4);
				const int word = w % static_cast<int>(sizeof(settled_slice) / 4);
				const int64_t p = chunk + s_hits[cursor_slice + g];
				reinterpret_cast<int *>(&s_slices[g])[word] = reinterpret_cast<const int *>(settled + v * L.particles + p)[word];
				if (word == 0)
				{
					s_particle[g] = p;
					const float *tr = L.transforms + (v * L.transform_stride_v + p * L.transform_stride_p) * 12;
					const double centre = static_cast<double>(n / 2);
					s_angle[g] = make_double2(2.0 * pi * (centre + static_cast<double>(__ldg(tr + 3))) / static_cast<double>(n),
						2.0 * pi * (centre + static_cast<double>(__ldg(tr + 7))) / static_cast<double>(n));
				}
			}
			__syncthreads();

			// Units: the rows of (slice, sign, interval pair) that reach the tile.
			if (threadIdx.x < units)
			{
				const int u = threadIdx.x;
				const int g = u / combos, combo = u % combos;
				const int sgn = combo / (zcount * ycount), zi = (combo / ycount) % zcount, yi = combo % ycount;
				const settled_slice &S = s_slices[g];
				det_unit U;
				U.slice = g;
				U.sgn = sgn;
				U.zi = zi;
				U.yi = yi;
				const float sign = sgn ? -1.0f : 1.0f;
				float ystep_f[3];
				for (int a = 0; a < 3; ++a)
				{
					U.step[a] = sign * S.step[a];
					U.inv_step[a] = 1.0f / U.step[a];
					ystep_f[a] = sign * static_cast<float>(S.ys[a]);
				}
				const float nx = fabsf(S.normal[0]), ny = fabsf(S.normal[1]), nz = fabsf(S.normal[2]);
				const int axis = nz >= ny && nz >= nx ? 2 : (ny >= nx ? 1 : 0);
				U.axis = axis;
				// The fixed axes: b = y for an x pillar, else x; c = y for a z pillar, else z.
				U.step_b = axis == 0 ? U.step[1] : U.step[0];
				U.inv_b = axis == 0 ? U.inv_step[1] : U.inv_step[0];
				U.step_c = axis == 2 ? U.step[1] : U.step[2];
				U.inv_c = axis == 2 ? U.inv_step[1] : U.inv_step[2];
				const float ystep_b = axis == 0 ? ystep_f[1] : ystep_f[0];
				const float ystep_c = axis == 2 ? ystep_f[1] : ystep_f[2];
				// k_y where K's fixed coordinates are (F_b, F_c): (F_c s_b - F_b s_c) / D.
				const float D = U.step_b * ystep_c - U.step_c * ystep_b;
				if (fabsf(D) > 1e-6f)
				{
					U.ky_c = U.step_b / D;
					U.ky_b = -U.step_c / D;
					U.ky_half = (cube + 0.01f) * (fabsf(U.step_b) + fabsf(U.step_c)) / fabsf(D) + 0.05f;
				}
				else
				{
					U.ky_b = U.ky_c = 0.0f;
					U.ky_half = 1.0e7f;
				}
				int rb = 0, re = 0;
				const k_bounds bounds = unit_bounds(zi, yi);
				if (plane_reaches(S, bounds))
				{
					const int widest = min(last_column, S.last_shell);
					const int first_row = max(-highest_row, -widest);
					const int last_row = min(highest_row, widest);
					bound_rows(U.step, ystep_f, bounds, sgn, widest, first_row, last_row, rb, re);
				}
				if (g == 0 && combo < cursor_combo)
					re = rb;
				else if (g == 0 && combo == cursor_combo)
					rb = min(re, rb + cursor_row);
				U.row_begin = rb;
				U.rows = max(0, re - rb);
				s_units[u] = U;
			}
			__syncthreads();
			if (warp == 0)
			{
				// Exclusive scan of the units' rows: two units a lane.
				const int ra = lane < units ? s_units[lane].rows : 0;
				const int rb = lane + 32 < units ? s_units[lane + 32].rows : 0;
				int ia = ra, ib = rb;
				for (int o = 1; o < 32; o <<= 1)
				{
					const int ya = __shfl_up_sync(0xffffffffu, ia, o);
					const int yb = __shfl_up_sync(0xffffffffu, ib, o);
					if (lane >= o)
					{
						ia += ya;
						ib += yb;
					}
				}
				const int total_a = __shfl_sync(0xffffffffu, ia, 31);
				if (lane < units)
					s_units[lane].row_first = ia - ra;
				if (lane + 32 < units)
					s_units[lane + 32].row_first = total_a + ib - rb;
				const int total = total_a + __shfl_sync(0xffffffffu, ib, 31);
				if (lane == 0)
					s_all_rows = total;
			}
			__syncthreads();
			const int all_rows = s_all_rows;
			const int rows_here = min(all_rows, det_stage_rows);
			// The unit holding stage row r: the last with row_first <= r.
			auto unit_of = [&](int r) {
				int lo = 0;
				for (int bit = 32; bit > 0; bit >>= 1)
					if (lo + bit < units && s_units[lo + bit].row_first <= r)
						lo += bit;
				return lo;
			};

			// Rows: the CPU's reach and column clipping, base and y phase.
			int count = 0;
			if (threadIdx.x < rows_here)
			{
				const int r = threadIdx.x;
				const int u = unit_of(r);
				const det_unit &U = s_units[u];
				const settled_slice &S = s_slices[U.slice];
				const int ky = U.row_begin + (r - U.row_first);
				const float radius = static_cast<float>(S.last_shell) + 0.5f;
				const int widest = min(last_column, S.last_shell);
				int b = 0, e = 0;
				float base[3] = {0.0f, 0.0f, 0.0f};
				const float reach = radius * radius - static_cast<float>(ky * ky);
				if (reach >= 0.0f)
				{
					const int last = min(widest, static_cast<int>(sqrtf(reach)));
					if (U.sgn <= last)
					{
						const double kyv = static_cast<double>(ky) * (U.sgn ? -1.0 : 1.0);
						base[0] = static_cast<float>(kyv * S.ys[0]);
						base[1] = static_cast<float>(kyv * S.ys[1]);
						base[2] = static_cast<float>(kyv * S.ys[2]);
						clip_row(base, U.inv_step, U.step, unit_bounds(U.zi, U.yi), U.sgn, last, b, e);
					}
				}
				count = max(0, e - b);
				s_row_i[r] = make_int4(b, max(b, e), 0, ky);
				s_row_f[r] = make_float4(base[0], base[1], base[2], __int_as_float(u));
				s_row_phase[r] = count > 0 ? exact_shift_phase(s_angle[U.slice].y, ky) : make_float2(0.0f, 0.0f);
			}
			// Exclusive scan of the rows' samples.
			int inclusive = count;
			for (int o = 1; o < 32; o <<= 1)
			{
				const int y = __shfl_up_sync(0xffffffffu, inclusive, o);
				if (lane >= o)
					inclusive += y;
			}
			if (lane == 31)
				s_scan[warp] = inclusive;
			__syncthreads();
			if (warp == 0)
			{
				int s = lane < det_threads / 32 ? s_scan[lane] : 0;
				for (int o = 1; o < 32; o <<= 1)
				{
					const int y = __shfl_up_sync(0xffffffffu, s, o);
					if (lane >= o)
						s += y;
				}
				if (lane < det_threads / 32)
					s_scan[lane] = s;
			}
			__syncthreads();
			inclusive += warp > 0 ? s_scan[warp - 1] : 0;
			if (threadIdx.x < rows_here)
				s_row_i[threadIdx.x].z = inclusive - count;
			// The stage ends at the last row whose samples fit.
			const int r_cut =
				__syncthreads_count(threadIdx.x < rows_here && inclusive <= det_stage_samples);
			if (r_cut > 0 && threadIdx.x == r_cut - 1)
				s_stage_samples = inclusive;
			if (r_cut == 0 && threadIdx.x == 0)
				s_stage_samples = 0;
			if (threadIdx.x == 0)
			{
				if (r_cut >= all_rows)
				{
					s_next[0] = cursor_slice + G;
					s_next[1] = 0;
					s_next[2] = 0;
				}
				else
				{
					const int u = unit_of(r_cut);
					const int g = s_units[u].slice, combo = u - g * combos;
					s_next[0] = cursor_slice + g;
					s_next[1] = combo;
					s_next[2] = (r_cut - s_units[u].row_first) + (g == 0 && combo == cursor_combo ? cursor_row : 0);
				}
			}
			__syncthreads();
			const int stage_samples = min(s_stage_samples, det_stage_samples);

			// Samples: K, anchor and fractions, value and weights.
			for (int i = threadIdx.x; i < stage_samples; i += det_threads)
			{
				int r = 0;
				for (int bit = det_stage_rows / 2; bit > 0; bit >>= 1)
					if (r + bit < r_cut && s_row_i[r + bit].z <= i)
						r += bit;
				const int4 ri = s_row_i[r];
				const float4 rf = s_row_f[r];
				const det_unit &U = s_units[__float_as_int(rf.w)];
				const settled_slice &S = s_slices[U.slice];
				const int64_t p = s_particle[U.slice];
				const int kx = ri.x + (i - ri.z);
				const int rky = ri.w;
				const float kxf = static_cast<float>(kx);
				const float cx = fadd(rf.x, fmul(kxf, U.step[0]));
				const float cy = fadd(rf.y, fmul(kxf, U.step[1]));
				const float cz = fadd(rf.z, fmul(kxf, U.step[2]));
				int ax, ay, az;
				if constexpr (KB)
				{
					ax = kb_first(cx, kb.half_width);
					ay = kb_first(cy, kb.half_width);
					az = kb_first(cz, kb.half_width);
				}
				else
				{
					ax = anchor_of<PROFILE>(cx);
					ay = anchor_of<PROFILE>(cy);
					az = anchor_of<PROFILE>(cz);
				}
				const int shell = shell_of(kx, rky);
				const float *rad = L.radial + (v * L.radial_stride_v + p * L.radial_stride_p) * h;
				const float r_w = shell <= S.last_shell ? __ldg(rad + shell) : 0.0f;
				float vre = 0.0f, vim = 0.0f, cnt = 0.0f;
				if (r_w != 0.0f)
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
						const float *weights = L.extra + (v * L.extra_stride_v + p * L.extra_stride_p) * (int64_t)n * h;
						wden = __ldg(weights + (int64_t)srow * h + kx);
					}
					const float2 *slice = L.slices + (v * L.slice_stride_v + p * L.slice_stride_p) * (int64_t)n * h;
					const float2 sample = __ldg(slice + (int64_t)srow * h + kx);
					const float2 xph = exact_shift_phase(s_angle[U.slice].x, kx);
					const float2 yph = s_row_phase[r];
					const float shre = fsub(fmul(sample.x, xph.x), fmul(sample.y, xph.y));
					const float shim = fadd(fmul(sample.x, xph.y), fmul(sample.y, xph.x));
					const float vre0 = fsub(fmul(shre, yph.x), fmul(shim, yph.y));
					const float vim0 = fadd(fmul(shre, yph.y), fmul(shim, yph.x));
					const float sc = fmul(r_w, wnum);
					vre = fmul(vre0, sc);
					vim = fmul(U.sgn ? -vim0 : vim0, sc);
					cnt = fmul(r_w, wden);
				}
				s_anchor[i] = make_short4(static_cast<short>(ax), static_cast<short>(ay), static_cast<short>(az),
					static_cast<short>(r_w != 0.0f ? 1 : 0));
				if constexpr (KB)
					s_frac[i] = make_float4(cx, cy, cz, cnt);
				else
					s_frac[i] = make_float4(fsub(cx, static_cast<float>(ax)), fsub(cy, static_cast<float>(ay)),
						fsub(cz, static_cast<float>(az)), cnt);
				s_val[i] = make_float2(vre, vim);
			}
			__syncthreads();

			// The gather, unit by unit in the CPU's order.
			int previous_axis = -1;
			for (int u = 0; u < units; ++u)
			{
				const det_unit &U = s_units[u];
				const int rows = min(U.rows, r_cut - U.row_first);
				if (rows <= 0)
					continue;
				const int a = U.axis;
				if (a != previous_axis)
				{
					if (previous_axis >= 0)
						__syncthreads(); // the voxels change owners
					previous_axis = a;
				}
				// The pillar's stored coordinates and fixed frequencies.
				const int zlo = U.zi ? zl[1] : zl[0], zhi = U.zi ? zu[1] : zu[0];
				const int ylo = U.yi ? yl[1] : yl[0], yhi = U.yi ? yu[1] : yu[0];
				int sb, sc, fb, fc, lo_a, hi_a;
				if (a == 2)
				{
					sb = x0 + p2;
					sc = y0 + p1;
					fb = sb < x1 ? sb : 1 << 30;
					fc = sc < y1 ? frequency_in(sc, ylo, yhi, big) : 1 << 30;
					lo_a = zlo;
					hi_a = zhi;
				}
				else if (a == 1)
				{
					sb = x0 + p2;
					sc = z0 + p1;
					fb = sb < x1 ? sb : 1 << 30;
					fc = sc < z1 ? frequency_in(sc, zlo, zhi, big) : 1 << 30;
					lo_a = ylo;
					hi_a = yhi;
				}
				else
				{
					sb = y0 + p2;
					sc = z0 + p1;
					fb = sb < y1 ? frequency_in(sb, ylo, yhi, big) : 1 << 30;
					fc = sc < z1 ? frequency_in(sc, zlo, zhi, big) : 1 << 30;
					lo_a = x0;
					hi_a = x1 - 1;
				}
				if (fb == (1 << 30) || fc == (1 << 30))
					continue;
				const float fbf = static_cast<float>(fb), fcf = static_cast<float>(fc);
				const float kys = fminf(fmaxf(U.ky_b * fbf + U.ky_c * fcf, -1.0e7f), 1.0e7f);
				const int ky_lo = max(U.row_begin, static_cast<int>(ceilf(kys - U.ky_half)));
				const int ky_hi = min(U.row_begin + rows - 1, static_cast<int>(floorf(fminf(kys + U.ky_half, 1.0e7f))));
				for (int ky = ky_lo; ky <= ky_hi; ++ky)
				{
					const int r = U.row_first + (ky - U.row_begin);
					const int4 ri = s_row_i[r];
					if (ri.y <= ri.x)
						continue;
					const float4 rf = s_row_f[r];
					// The columns whose K lies within the window of (F_b, F_c), with a
					// margin of 0.01 in K and 0.02 in k_x; the anchor test decides.
					float lo = static_cast<float>(ri.x), hi = static_cast<float>(ri.y - 1);
					const float base_b = a == 0 ? rf.y : rf.x;
					const float base_c = a == 2 ? rf.y : rf.z;
					bool crosses = true;
					if (fabsf(U.step_b) < 1e-6f)
						crosses = fbf - cube - 0.01f <= base_b && base_b <= fbf + cube + 0.01f;
					else
					{
						const float t1 = (fbf - cube - 0.01f - base_b) * U.inv_b;
						const float t2 = (fbf + cube + 0.01f - base_b) * U.inv_b;
						lo = fmaxf(lo, fminf(t1, t2) - 0.02f);
						hi = fminf(hi, fmaxf(t1, t2) + 0.02f);
					}
					if (fabsf(U.step_c) < 1e-6f)
						crosses = crosses && fcf - cube - 0.01f <= base_c && base_c <= fcf + cube + 0.01f;
					else
					{
						const float t1 = (fcf - cube - 0.01f - base_c) * U.inv_c;
						const float t2 = (fcf + cube + 0.01f - base_c) * U.inv_c;
						lo = fmaxf(lo, fminf(t1, t2) - 0.02f);
						hi = fminf(hi, fmaxf(t1, t2) + 0.02f);
					}
					if (!crosses || lo > hi)
						continue;
					const int k_first = static_cast<int>(ceilf(lo)), k_last = static_cast<int>(floorf(hi));
					for (int kx = k_first; kx <= k_last; ++kx)
					{
						const int i = ri.z + (kx - ri.x);
						const short4 an = s_anchor[i];
						if (an.w == 0)
							continue;
						const int anchor_a = a == 0 ? an.x : (a == 1 ? an.y : an.z);
						const int ob = fb - (a == 0 ? an.y : an.x);
						const int oc = fc - (a == 2 ? an.y : an.z);
						if (static_cast<unsigned>(ob) >= static_cast<unsigned>(taps) ||
							static_cast<unsigned>(oc) >= static_cast<unsigned>(taps))
							continue;
#pragma unroll
						for (int d = 0; d < taps; ++d)
						{
							const int t = anchor_a + d;
							if (t < lo_a || t > hi_a)
								continue;
							const int st = a == 0 ? t : (t < 0 ? t + big : t);
							if ((st & 1) != half_of)
								continue;
							const int gx = a == 0 ? st : sb;
							const int sy = a == 1 ? st : (a == 0 ? sb : sc);
							const int sz = a == 2 ? st : sc;
							const float4 fr = s_frac[i];
							const float2 val = s_val[i];
							float wgt = 1.0f;
							if constexpr (KB)
							{
								// The voxel's frequencies; the window of each axis at its
								// distance from K; (w_z w_y) w_x as the CPU.
								const int gfx = a == 0 ? t : fb;
								const int gfy = a == 1 ? t : (a == 0 ? fb : fc);
								const int gfz = a == 2 ? t : fc;
								const float wx = kb_weight(fabsf(fsub(static_cast<float>(gfx), fr.x)), kb.scale, kb.step_count, s_kb);
								const float wy = kb_weight(fabsf(fsub(static_cast<float>(gfy), fr.y)), kb.scale, kb.step_count, s_kb);
								const float wz = kb_weight(fabsf(fsub(static_cast<float>(gfz), fr.z)), kb.scale, kb.step_count, s_kb);
								wgt = fmul(fmul(wz, wy), wx);
							}
							else if constexpr (TAPS == 2)
							{
								const int ox = a == 0 ? d : ob;
								const int oy = a == 1 ? d : (a == 0 ? ob : oc);
								const int oz = a == 2 ? d : oc;
								const float wx = ox ? fr.x : fsub(1.0f, fr.x);
								const float wy = oy ? fr.y : fsub(1.0f, fr.y);
								const float wz = oz ? fr.z : fsub(1.0f, fr.z);
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
							const int cell = det_cell(sz - z0, sy - y0, gx - x0);
							float2 acc = s_num[cell];
							acc.x = fadd(acc.x, are);
							acc.y = fadd(acc.y, aim);
							s_num[cell] = acc;
							s_den[cell] = fadd(s_den[cell], fmul(fr.w, wgt));
						}
					}
				}
			}
			cursor_slice = s_next[0];
			cursor_combo = s_next[1];
			cursor_row = s_next[2];
		}
	}
	__syncthreads();

	// Write back: this CTA alone owns these voxels.
	for (int i = threadIdx.x; i < cells; i += blockDim.x)
	{
		const int lz = i / (det_edge * det_edge), ly = (i / det_edge) % det_edge, lx = i % det_edge;
		if (z0 + lz >= z1 || y0 + ly >= y1 || x0 + lx >= x1)
			continue;
		const int64_t offset = ((int64_t)(z0 + lz) * big + (y0 + ly)) * H + (x0 + lx);
		num[offset] = s_num[det_cell(lz, ly, lx)];
		den[offset] = s_den[det_cell(lz, ly, lx)];
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
void launch_deterministic(const insertion_launch &L, const settled_slice *settled, int *order, const kb_table &kb,
	cudaStream_t stream)
{
	const det_plan plan = make_det_plan(L);
	det_order_kernel<<<1, 1024, 0, stream>>>(plan, L.big, order);
	check_cuda(cudaGetLastError(), "deterministic tile order launch");
	auto kernel = insert_deterministic_kernel<PROFILE, KIND, false>;
	// The stage's samples (fractions and weight, value, anchor), the tile's
	// accumulators, the volume phase table (odd N), the Kaiser-Bessel table.
	const size_t smem = (sizeof(float4) + sizeof(float2) + sizeof(short4)) * det_stage_samples +
		(sizeof(float2) + sizeof(float)) * det_edge * det_edge * det_edge +
		((L.big & 1) ? static_cast<size_t>(L.big) * 8 : 0) +
		(PROFILE == REXLIB_B200_WINDOW_KAISER_BESSEL ? sizeof(float) * (kb.step_count + 3) : 0);
	check_cuda(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)),
		"deterministic insertion attributes");
	kernel<<<dim3(plan.tile_count, static_cast<unsigned>(L.volumes)), det_threads, smem, stream>>>(L, plan, settled,
		order, kb, no_batch{});
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

tile_plan make_plan(const insertion_launch &L, bool l2_numerator, const tile_config *config = nullptr)
{
	const int taps = L.tap_count;
	const int half = L.big / 2;
	// Anchors that can put a tap on a stored voxel: z and y frequencies in
	// [-N/2, N/2], x in [0, N/2].
	// A window's first tap sits up to taps - 1 below the lowest voxel it reaches.
	const int lo_zy = -half - (taps - 1);
	const int count_zy = half - lo_zy + 1;
	const int lo_x = -(taps - 1);
	const int count_x = half - lo_x + 1;
	const int halo = taps - 1;
	// Shared bytes per cell: the denominator, plus the numerator when it is not in L2.
	const size_t cell_bytes = l2_numerator ? 4 : 12;
	// Less the volume phase table (odd N) and the Kaiser-Bessel table (at most
	// 512 floats per tap, plus three).
	const size_t table_bytes = (L.big % 2 ? static_cast<size_t>(L.big) * 8 : 0) +
		(L.profile == REXLIB_B200_WINDOW_KAISER_BESSEL ? (512 * static_cast<size_t>(std::max(taps, 2)) + 3) * 4 : 0);
	const size_t smem_cells = (insert_smem_budget - table_bytes) / cell_bytes;
	const size_t l2_cells = static_cast<size_t>(std::max(512, config != nullptr && config->cells > 0 ? config->cells
		: env_int("REXLIB_B200_TILE_CELLS", static_cast<int>(l2_numerator_cells))));
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
	if (config != nullptr && config->min_hits > 0 && config->max_hits >= config->min_hits)
	{
		best.min_hits = config->min_hits;
		best.max_hits = config->max_hits;
	}
	best.target_items = insert_grid() * 16;
	const int64_t runs_per_tile = 1 + std::min<int64_t>(L.particles, (L.particles + best.min_hits - 1) /
		best.min_hits);
	const int64_t capacity = L.volumes * best.tile_count * runs_per_tile;
	best.item_capacity = static_cast<int>(std::min<int64_t>(capacity, 1LL << 30));
	best.l2_numerator = l2_numerator;
	// The linear and Kaiser-Bessel windows' numerator tile is held twice, as x
	// pairs (2j, 2j+1) and (2j+1, 2j+2) of float4 slots, so a tap pair is one
	// reduction whatever the parity of its first x; the nearest window's as
	// float2 cells.
	const int64_t rows_zy = static_cast<int64_t>(best.box[0]) * best.box[1];
	const bool paired = L.profile == REXLIB_B200_WINDOW_TRIANGLE || L.profile == REXLIB_B200_WINDOW_KAISER_BESSEL;
	best.scratch_per_cta = !l2_numerator ? 0 : paired ? 2 * rows_zy * (best.box[2] / 2 + 1) * 2 : rows_zy * best.box[2];
	best.k_shift = 0.0f;
	return best;
}

template <int PROFILE, int KIND, bool L2_NUM>
void launch_storage(const insertion_launch &L, const tile_plan &plan, const workspace_view &w, const kb_table &kb,
	cudaStream_t stream)
{
	auto kernel = insert_tiled_kernel<PROFILE, KIND, L2_NUM, false>;
	window_param<PROFILE> wp{};
	size_t table_bytes = 0;
	if constexpr (PROFILE == REXLIB_B200_WINDOW_KAISER_BESSEL)
	{
		wp.kb = kb;
		table_bytes = sizeof(float) * (kb.step_count + 3);
	}
	const size_t smem = sizeof(row_record) * insert_warps * 32 + (L.big % 2 ? static_cast<size_t>(L.big) * 8 : 0) +
		table_bytes + static_cast<size_t>(plan.box[0]) * plan.box[1] * plan.box[2] * (L2_NUM ? 4 : 12);
	check_cuda(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)),
		"tiled insertion attributes");
	kernel<<<insert_grid(), insert_threads, smem, stream>>>(L, plan, w.settled, w.item_count, w.work_counter,
		w.items, w.scratch, wp, no_batch{});
	check_cuda(cudaGetLastError(), "tiled insertion launch");
}

template <int PROFILE, int KIND>
void launch_kind(const insertion_launch &L, const tile_plan &plan, const workspace_view &w, const kb_table &kb,
	cudaStream_t stream)
{
	if (plan.l2_numerator)
		launch_storage<PROFILE, KIND, true>(L, plan, w, kb, stream);
	else
		launch_storage<PROFILE, KIND, false>(L, plan, w, kb, stream);
}

template <int KIND>
void launch_window(const insertion_launch &L, const tile_plan &plan, const workspace_view &w, const kb_table &kb,
	cudaStream_t stream)
{
	if (L.profile == REXLIB_B200_WINDOW_BOX)
		launch_kind<REXLIB_B200_WINDOW_BOX, KIND>(L, plan, w, kb, stream);
	else if (L.profile == REXLIB_B200_WINDOW_TRIANGLE)
		launch_kind<REXLIB_B200_WINDOW_TRIANGLE, KIND>(L, plan, w, kb, stream);
	else
		launch_kind<REXLIB_B200_WINDOW_KAISER_BESSEL, KIND>(L, plan, w, kb, stream);
}

} // anonymous namespace

bool tiled_insertion_applies(const insertion_launch &launch, weight_kind, int mode)
{
	if (mode == REXLIB_B200_INSERT_DETERMINISTIC)
		return launch.volumes * launch.particles > 0 && launch.volumes < 65536 && launch.n <= 1024;
	// The Kaiser-Bessel window with up to 4 taps an axis (half-width up to 2);
	// wider windows take the scatter kernel.
	if (launch.profile == REXLIB_B200_WINDOW_KAISER_BESSEL && launch.tap_count > 4)
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

namespace
{

template <int KIND>
void launch_deterministic_window(const insertion_launch &L, const settled_slice *settled, int *order,
	const kb_table &kb, cudaStream_t stream)
{
	if (L.profile == REXLIB_B200_WINDOW_BOX)
		launch_deterministic<REXLIB_B200_WINDOW_BOX, KIND>(L, settled, order, kb, stream);
	else if (L.profile == REXLIB_B200_WINDOW_TRIANGLE)
		launch_deterministic<REXLIB_B200_WINDOW_TRIANGLE, KIND>(L, settled, order, kb, stream);
	else
		launch_deterministic<REXLIB_B200_WINDOW_KAISER_BESSEL, KIND>(L, settled, order, kb, stream);
}

} // anonymous namespace

void launch_insert_tiled(const insertion_launch &L, weight_kind kind, int mode, bool shared_tiles, void *workspace,
	size_t, const kb_table *kb, cudaStream_t stream)
{
	if (mode == REXLIB_B200_INSERT_DETERMINISTIC)
	{
		require(L.profile != REXLIB_B200_WINDOW_KAISER_BESSEL || kb != nullptr, "the window table is missing");
		static const kb_table no_table{};
		const kb_table &table = kb ? *kb : no_table;
		settled_slice *settled = static_cast<settled_slice *>(workspace);
		int *order = reinterpret_cast<int *>(static_cast<char *>(workspace) +
			align_up(settled_bytes * L.volumes * L.particles, 256));
		const int64_t slices = L.volumes * L.particles;
		settle_kernel<<<static_cast<unsigned>((slices + settle_threads / 32 - 1) / (settle_threads / 32)),
			settle_threads, 0, stream>>>(L, settled, static_cast<int>(kind));
		check_cuda(cudaGetLastError(), "settle launch");
		switch (kind)
		{
		case weight_kind::unit:
			launch_deterministic_window<0>(L, settled, order, table, stream);
			break;
		case weight_kind::ctf:
			launch_deterministic_window<1>(L, settled, order, table, stream);
			break;
		case weight_kind::spectrum:
			launch_deterministic_window<2>(L, settled, order, table, stream);
			break;
		}
		return;
	}
	require(L.profile != REXLIB_B200_WINDOW_KAISER_BESSEL || kb != nullptr, "the window table is missing");
	static const kb_table no_table{};
	const kb_table &table = kb ? *kb : no_table;
	tile_plan plan = make_plan(L, !shared_tiles);
	if (L.profile == REXLIB_B200_WINDOW_KAISER_BESSEL)
		plan.k_shift = table.half_width - 1.0f;
	const workspace_view w = view_workspace(workspace, L.volumes, L.particles, plan);
	const int64_t slices = L.volumes * L.particles;
	settle_kernel<<<static_cast<unsigned>((slices + settle_threads / 32 - 1) / (settle_threads / 32)), settle_threads,
		0, stream>>>(L, w.settled, static_cast<int>(kind));
	check_cuda(cudaGetLastError(), "settle launch");
	count_hits_kernel<<<dim3(plan.tile_count, static_cast<unsigned>(L.volumes)), count_threads, 0, stream>>>(
		L, plan, w.settled, w.counts);
	check_cuda(cudaGetLastError(), "hit count launch");
	plan_items_kernel<false><<<1, 1024, 0, stream>>>(plan, L.volumes, L.particles, w.counts, w.item_count,
		w.work_counter, w.items, no_batch{});
	check_cuda(cudaGetLastError(), "plan launch");
	switch (kind)
	{
	case weight_kind::unit:
		launch_window<0>(L, plan, w, table, stream);
		break;
	case weight_kind::ctf:
		launch_window<1>(L, plan, w, table, stream);
		break;
	case weight_kind::spectrum:
		launch_window<2>(L, plan, w, table, stream);
		break;
	}
}

// Throughput: settle, count, plan, insert; deterministic: settle, tile order, insert.
int tiled_insertion_launches(int mode) { return mode == REXLIB_B200_INSERT_DETERMINISTIC ? 3 : 4; }

// ---------------------------------------------------------------------------
// Batched calls

namespace
{

// The tiles of every job nearest the origin first, as det_order_kernel
// orders one call's: a counting sort of all (volume, tile) cells by their
// tile's distance from the origin, in units of 8.
__global__ void __launch_bounds__(1024) det_order_batch_kernel(const __grid_constant__ batch_param b, int *order)
{
	__shared__ int counts[128];
	__shared__ int starts[128];
	for (int i = threadIdx.x; i < 128; i += blockDim.x)
		counts[i] = 0;
	__syncthreads();
	auto key_of = [&](int64_t cell) {
		const batch_job &job = b.jobs[job_of_cell(b, cell)];
		const det_plan &plan = job.dplan;
		const int big = job.launch.big;
		const int t = static_cast<int>((cell - job.cell_offset) % plan.tile_count);
		const int tz = t / (plan.tiles[1] * plan.tiles[2]);
		const int ty = (t / plan.tiles[2]) % plan.tiles[1];
		const int tx = t % plan.tiles[2];
		auto axis_distance = [&](int s0, int s1) {
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
	for (int64_t c = threadIdx.x; c < b.cells; c += blockDim.x)
		atomicAdd(&counts[key_of(c)], 1);
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
	for (int64_t c = threadIdx.x; c < b.cells; c += blockDim.x)
		order[atomicAdd(&starts[key_of(c)], 1)] = static_cast<int>(c);
}

struct batch_layout
{
	batch_param param;
	tile_plan envelope;      // largest tile and numerator scratch, common run lengths (throughput)
	insertion_launch shape;  // largest odd volume extent (big), for the phase table
	size_t smem;             // dynamic shared memory of the insertion launch
	size_t settled, counts, items, scratch, order; // workspace offsets
	size_t bytes;
};

batch_layout plan_batch(const insertion_launch *jobs, int count, weight_kind, int mode, const tile_config &config,
	const kb_table &kb)
{
	require(count >= 1 && count <= max_batch_jobs, "a batched call takes 1 to 64 jobs");
	batch_layout out{};
	batch_param &b = out.param;
	b.job_count = count;
	const bool det = mode == REXLIB_B200_INSERT_DETERMINISTIC;
	int64_t slices = 0, cells = 0, capacity = 0, max_cells = 0, max_scratch = 0;
	int odd_big = 0, max_big = 0;
	size_t det_smem = 0;
	for (int j = 0; j < count; ++j)
	{
		batch_job &job = b.jobs[j];
		job.launch = jobs[j];
		job.settled_offset = slices;
		job.cell_offset = cells;
		slices += jobs[j].volumes * jobs[j].particles;
		if ((jobs[j].big & 1) && jobs[j].big > odd_big)
			odd_big = jobs[j].big;
		max_big = std::max(max_big, jobs[j].big);
		if (det)
		{
			job.dplan = make_det_plan(jobs[j]);
			cells += jobs[j].volumes * job.dplan.tile_count;
		}
		else
		{
			job.plan = make_plan(jobs[j], true, &config);
			if (jobs[j].profile == REXLIB_B200_WINDOW_KAISER_BESSEL)
				job.plan.k_shift = kb.half_width - 1.0f;
			cells += jobs[j].volumes * job.plan.tile_count;
			const int64_t runs_per_tile = 1 + std::min<int64_t>(jobs[j].particles,
				(jobs[j].particles + job.plan.min_hits - 1) / job.plan.min_hits);
			capacity += jobs[j].volumes * job.plan.tile_count * runs_per_tile;
			max_cells = std::max<int64_t>(max_cells, static_cast<int64_t>(job.plan.box[0]) * job.plan.box[1] *
				job.plan.box[2]);
			max_scratch = std::max<int64_t>(max_scratch, job.plan.scratch_per_cta);
		}
	}
	require(capacity < (1LL << 30) && cells < (1LL << 31), "the batched call is too large");
	b.slices = slices;
	b.cells = cells;
	out.shape = jobs[0];
	out.shape.big = odd_big;
	if (!det)
	{
		out.envelope = b.jobs[0].plan;
		out.envelope.box[0] = static_cast<int>(max_cells);
		out.envelope.box[1] = out.envelope.box[2] = 1;
		out.envelope.scratch_per_cta = max_scratch;
		out.envelope.item_capacity = static_cast<int>(capacity);
		out.envelope.target_items = insert_grid() * 16;
		const size_t table_bytes = jobs[0].profile == REXLIB_B200_WINDOW_KAISER_BESSEL
			? sizeof(float) * (kb.step_count + 3) : 0;
		out.smem = sizeof(row_record) * insert_warps * 32 + static_cast<size_t>(odd_big) * 8 + table_bytes +
			static_cast<size_t>(max_cells) * 4;
	}
	else
	{
		det_smem = (sizeof(float4) + sizeof(float2) + sizeof(short4)) * det_stage_samples +
			(sizeof(float2) + sizeof(float)) * det_edge * det_edge * det_edge + static_cast<size_t>(odd_big) * 8 +
			(jobs[0].profile == REXLIB_B200_WINDOW_KAISER_BESSEL ? sizeof(float) * (kb.step_count + 3) : 0);
		out.smem = det_smem;
	}
	size_t at = 0;
	out.settled = at;
	at += align_up(settled_bytes * static_cast<size_t>(slices), 256);
	out.counts = at;
	at += align_up(sizeof(int) * static_cast<size_t>(cells), 256) + 256; // counts (or the order), then two counters
	if (!det)
	{
		out.items = at;
		at += align_up(sizeof(work_item) * static_cast<size_t>(capacity), 256);
		out.scratch = at;
		at += static_cast<size_t>(max_scratch) * sizeof(float2) * insert_grid();
	}
	out.order = out.counts;
	out.bytes = at;
	return out;
}

template <int PROFILE, int KIND>
void launch_batch_kernels(const batch_layout &layout, int mode, const kb_table &table, char *w, cudaStream_t stream)
{
	const batch_param &b = layout.param;
	kb_table_batch kb{};
	kb.half_width = table.half_width;
	kb.scale = table.scale;
	kb.step_count = table.step_count;
	kb.tap_count = table.tap_count;
	if constexpr (PROFILE == REXLIB_B200_WINDOW_KAISER_BESSEL)
	{
		require(table.step_count + 3 <= kb_table_capacity_batch,
			"batched calls take Kaiser-Bessel half-widths up to 2");
		for (int i = 0; i < table.step_count + 3; ++i)
			kb.values[i] = table.values[i];
	}
	settled_slice *settled = reinterpret_cast<settled_slice *>(w + layout.settled);
	settle_batch_kernel<<<static_cast<unsigned>((b.slices + settle_threads / 32 - 1) / (settle_threads / 32)),
		settle_threads, 0, stream>>>(b, settled, KIND);
	check_cuda(cudaGetLastError(), "batched settle launch");
	if (mode == REXLIB_B200_INSERT_DETERMINISTIC)
	{
		int *order = reinterpret_cast<int *>(w + layout.order);
		det_order_batch_kernel<<<1, 1024, 0, stream>>>(b, order);
		check_cuda(cudaGetLastError(), "batched tile order launch");
		auto kernel = insert_deterministic_kernel<PROFILE, KIND, true>;
		check_cuda(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
					   static_cast<int>(layout.smem)),
			"batched deterministic insertion attributes");
		insertion_launch shape = layout.shape;
		kernel<<<static_cast<unsigned>(b.cells), det_threads, layout.smem, stream>>>(shape, b.jobs[0].dplan, settled,
			order, kb, b);
		check_cuda(cudaGetLastError(), "batched deterministic insertion launch");
		return;
	}
	int *counts = reinterpret_cast<int *>(w + layout.counts);
	int *item_count = reinterpret_cast<int *>(w + layout.counts + align_up(sizeof(int) * b.cells, 256));
	int *work_counter = item_count + 1;
	work_item *items = reinterpret_cast<work_item *>(w + layout.items);
	float2 *scratch = reinterpret_cast<float2 *>(w + layout.scratch);
	count_hits_batch_kernel<<<static_cast<unsigned>(b.cells), count_threads, 0, stream>>>(b, settled, counts);
	check_cuda(cudaGetLastError(), "batched hit count launch");
	plan_items_kernel<true><<<1, 1024, 0, stream>>>(layout.envelope, 0, 0, counts, item_count, work_counter, items, b);
	check_cuda(cudaGetLastError(), "batched plan launch");
	auto kernel = insert_tiled_kernel<PROFILE, KIND, true, true>;
	window_param<PROFILE, kb_table_batch> wp{};
	if constexpr (PROFILE == REXLIB_B200_WINDOW_KAISER_BESSEL)
		wp.kb = kb;
	check_cuda(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(layout.smem)),
		"batched insertion attributes");
	kernel<<<insert_grid(), insert_threads, layout.smem, stream>>>(layout.shape, layout.envelope, settled, item_count,
		work_counter, items, scratch, wp, b);
	check_cuda(cudaGetLastError(), "batched insertion launch");
}

template <int KIND>
void launch_batch_window(const batch_layout &layout, int profile, int mode, const kb_table &kb, char *w,
	cudaStream_t stream)
{
	if (profile == REXLIB_B200_WINDOW_BOX)
		launch_batch_kernels<REXLIB_B200_WINDOW_BOX, KIND>(layout, mode, kb, w, stream);
	else if (profile == REXLIB_B200_WINDOW_TRIANGLE)
		launch_batch_kernels<REXLIB_B200_WINDOW_TRIANGLE, KIND>(layout, mode, kb, w, stream);
	else
		launch_batch_kernels<REXLIB_B200_WINDOW_KAISER_BESSEL, KIND>(layout, mode, kb, w, stream);
}

} // anonymous namespace

size_t batched_insertion_workspace(const insertion_launch *jobs, int count, weight_kind kind, int mode,
	const tile_config &config, const kb_table &kb)
{
	return plan_batch(jobs, count, kind, mode, config, kb).bytes;
}

void launch_batched_insertion(const insertion_launch *jobs, int count, weight_kind kind, int mode,
	const tile_config &config, const kb_table &kb, void *workspace, size_t workspace_bytes, cudaStream_t stream)
{
	const batch_layout layout = plan_batch(jobs, count, kind, mode, config, kb);
	if (layout.bytes > workspace_bytes || (layout.bytes > 0 && workspace == nullptr))
		fail(REXLIB_B200_WORKSPACE_TOO_SMALL, "the batched insertion needs " + std::to_string(layout.bytes) +
			" bytes of workspace");
	char *w = static_cast<char *>(workspace);
	switch (kind)
	{
	case weight_kind::unit:
		launch_batch_window<0>(layout, jobs[0].profile, mode, kb, w, stream);
		break;
	case weight_kind::ctf:
		launch_batch_window<1>(layout, jobs[0].profile, mode, kb, w, stream);
		break;
	case weight_kind::spectrum:
		launch_batch_window<2>(layout, jobs[0].profile, mode, kb, w, stream);
		break;
	}
}

// Settle, count, plan, insert (throughput); settle, tile order, insert (deterministic).
int batched_insertion_launches(int mode) { return mode == REXLIB_B200_INSERT_DETERMINISTIC ? 3 : 4; }

} // namespace rexlib_b200
