// C entry points of the insertions: argument checks (the shape and type
// rules of include/rexlib/em/ops/reconstruction/slice_insertion_rules.hpp
// and the parameter checks of src/em/ops/parameters/*.cpp), the copy of the
// accumulators into distinct outputs, and the choice of kernel.
#include "insertion.cuh"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>
#include <string>
#include <type_traits>
#include <vector>

namespace rexlib_b200
{

// Tiled-kernel entry points (insert_tiled.cu).
bool tiled_insertion_applies(const insertion_launch &launch, weight_kind kind, int mode);
// shared_tiles: keep the whole tile in shared memory (no L2 numerator scratch).
size_t tiled_insertion_workspace(const insertion_launch &launch, weight_kind kind, int mode, bool shared_tiles);
// kb: the Kaiser-Bessel table (the deterministic mode with that window; null otherwise).
void launch_insert_tiled(const insertion_launch &launch, weight_kind kind, int mode, bool shared_tiles,
	void *workspace, size_t workspace_bytes, const kb_table *kb, cudaStream_t stream);
int tiled_insertion_launches(int mode);
// Batched calls (insert_tiled.cu).
size_t batched_insertion_workspace(const insertion_launch *jobs, int count, weight_kind kind, int mode,
	const tile_config &config, const kb_table &kb);
void launch_batched_insertion(const insertion_launch *jobs, int count, weight_kind kind, int mode,
	const tile_config &config, const kb_table &kb, void *workspace, size_t workspace_bytes, cudaStream_t stream);
int batched_insertion_launches(int mode);

namespace
{

double bessel_i0(double x)
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

void check_window(const rexlib_b200_gridding_window &w)
{
	switch (w.profile)
	{
	case REXLIB_B200_WINDOW_BOX:
	case REXLIB_B200_WINDOW_TRIANGLE:
		return;
	case REXLIB_B200_WINDOW_KAISER_BESSEL:
		require(std::isfinite(w.half_width) && w.half_width > 0.0,
			"gridding_window: the half-width of a Kaiser-Bessel window must be finite and positive");
		require(std::isfinite(w.shape) && w.shape >= 0.0,
			"gridding_window: the shape of a Kaiser-Bessel window must be finite and 0 or more");
		if (w.half_width > 7.0)
			fail(REXLIB_B200_UNSUPPORTED, "Kaiser-Bessel half-widths above 7 are not supported");
		return;
	default:
		require(false, "unknown gridding profile");
	}
}

// The window table of kaiser_bessel_window.inl:18-49 (1024 samples per
// voxel of half-width, two zeros past the end), in the element type T.
template <typename T, int CAPACITY>
void fill_kb_table(const rexlib_b200_gridding_window &w, kb_table_of<T, CAPACITY> &kb)
{
	kb.half_width = static_cast<T>(w.half_width);
	kb.tap_count = static_cast<int>(std::ceil(2.0 * w.half_width));
	if (w.profile != REXLIB_B200_WINDOW_KAISER_BESSEL)
	{
		kb.tap_count = w.profile == REXLIB_B200_WINDOW_BOX ? 1 : 2;
		kb.scale = T(0);
		kb.step_count = 0;
		return;
	}
	const double normalization = 1.0 / bessel_i0(w.shape);
	const long count = static_cast<long>(std::ceil(w.half_width * 1024.0));
	require(count + 3 <= CAPACITY, "Kaiser-Bessel table too large for the element type");
	kb.scale = static_cast<T>(static_cast<double>(count) / w.half_width);
	kb.step_count = static_cast<int>(count);
	for (long i = 0; i < CAPACITY; ++i)
		kb.values[i] = T(0);
	for (long i = 0; i <= count; ++i)
	{
		const double ratio = static_cast<double>(i) / static_cast<double>(count);
		kb.values[i] = static_cast<T>(bessel_i0(w.shape * std::sqrt(1.0 - ratio * ratio)) * normalization);
	}
}

constexpr const char *deterministic_limits =
	"the deterministic mode takes slice extents up to 1024 and fewer than 65,536 volumes";

// The window table of this call, filled in this thread's own storage (no
// allocation per call); only the Kaiser-Bessel window and the scatter kernel
// read it.
const kb_table *window_table(const rexlib_b200_gridding_window &w)
{
	thread_local kb_table table;
	fill_kb_table(w, table);
	return &table;
}

const kb_table_f64 *window_table_f64(const rexlib_b200_gridding_window &w)
{
	thread_local kb_table_f64 table;
	fill_kb_table(w, table);
	return &table;
}

void check_strides(const rexlib_b200_batch_strides &s, const char *name)
{
	require(s.volume >= 0 && s.particle >= 0, std::string(name) + ": batch strides must be 0 or more");
}

template <typename T>
insertion_launch_of<T> prepare(const rexlib_b200_insertion *a)
{
	require(a != nullptr, "null insertion descriptor");
	require(a->volume_count >= 0 && a->slices_per_volume >= 0, "negative batch extents");
	require(a->slice_extent >= 1 && a->volume_extent >= 1, "extents must be positive");
	if (a->slice_extent > 1024 || a->volume_extent > 2048)
		fail(REXLIB_B200_UNSUPPORTED, "slice extents above 1024 or volume extents above 2048 are not supported");
	check_window(a->window);
	check_strides(a->slice_strides, "slices");
	check_strides(a->transform_strides, "transforms");
	check_strides(a->radial_strides, "radial weights");
	require(a->mode == REXLIB_B200_INSERT_THROUGHPUT || a->mode == REXLIB_B200_INSERT_DETERMINISTIC,
		"unknown insertion mode");
	const bool empty = a->volume_count == 0;
	require(empty || (a->numerator_out && a->denominator_out && a->numerator_in && a->denominator_in),
		"null accumulator");
	require(empty || a->slices_per_volume == 0 || (a->slices && a->transforms && a->radial_weights),
		"null slice operand");
	constexpr size_t align = sizeof(complex_t<T>);
	require((reinterpret_cast<uintptr_t>(a->numerator_out) % align) == 0 &&
			(reinterpret_cast<uintptr_t>(a->numerator_in) % align) == 0 &&
			(reinterpret_cast<uintptr_t>(a->slices) % align) == 0,
		align == 8 ? "complex operands must be 8-byte aligned" : "complex operands must be 16-byte aligned");
	if (sizeof(T) == 8 && a->window.profile == REXLIB_B200_WINDOW_KAISER_BESSEL && a->window.half_width > 3.0)
		fail(REXLIB_B200_UNSUPPORTED, "float64 insertions take Kaiser-Bessel half-widths up to 3");

	insertion_launch_of<T> L{};
	L.numerator = static_cast<complex_t<T> *>(a->numerator_out);
	L.denominator = static_cast<T *>(a->denominator_out);
	L.slices = static_cast<const complex_t<T> *>(a->slices);
	L.transforms = static_cast<const T *>(a->transforms);
	L.radial = static_cast<const T *>(a->radial_weights);
	L.slice_stride_v = a->slice_strides.volume;
	L.slice_stride_p = a->slice_strides.particle;
	L.transform_stride_v = a->transform_strides.volume;
	L.transform_stride_p = a->transform_strides.particle;
	L.radial_stride_v = a->radial_strides.volume;
	L.radial_stride_p = a->radial_strides.particle;
	L.volumes = a->volume_count;
	L.particles = a->slices_per_volume;
	L.n = static_cast<int>(a->slice_extent);
	L.h = L.n / 2 + 1;
	L.big = static_cast<int>(a->volume_extent);
	L.big_h = L.big / 2 + 1;
	L.profile = a->window.profile;
	L.tap_count = a->window.profile == REXLIB_B200_WINDOW_BOX
		? 1
		: (a->window.profile == REXLIB_B200_WINDOW_TRIANGLE ? 2 : static_cast<int>(std::ceil(2.0 * a->window.half_width)));
	return L;
}

// Outputs = inputs + insertions: copy the inputs over distinct outputs
// (real elements of `real_bytes`).
void copy_accumulators(const rexlib_b200_insertion *a, size_t real_bytes, cudaStream_t stream)
{
	const size_t voxels = static_cast<size_t>(a->volume_count) * a->volume_extent * a->volume_extent *
		(a->volume_extent / 2 + 1);
	if (voxels == 0)
		return;
	if (a->numerator_out != a->numerator_in)
		check_cuda(cudaMemcpyAsync(a->numerator_out, a->numerator_in, voxels * 2 * real_bytes,
					   cudaMemcpyDeviceToDevice, stream),
			"copy of the numerator");
	if (a->denominator_out != a->denominator_in)
		check_cuda(cudaMemcpyAsync(a->denominator_out, a->denominator_in, voxels * real_bytes,
					   cudaMemcpyDeviceToDevice, stream),
			"copy of the denominator");
}

// The descriptor's element type: calls body(L) with the launch of that type.
template <typename Body>
void with_element_type(const rexlib_b200_insertion *a, Body &&body)
{
	require(a != nullptr, "null insertion descriptor");
	if (a->element_type == REXLIB_B200_FLOAT32)
		body(prepare<float>(a));
	else if (a->element_type == REXLIB_B200_FLOAT64)
		body(prepare<double>(a));
	else
		fail(REXLIB_B200_UNSUPPORTED, "insertions run float32 or float64 operands");
}

constexpr const char *float64_modes = "float64 insertions run in the throughput mode only";

// The float64 insertions: the slice-parallel kernel in double.
void run(const rexlib_b200_insertion *a, insertion_launch_of<double> &L, weight_kind kind, void *stream_handle)
{
	const cudaStream_t stream = as_stream(stream_handle);
	if (L.volumes * L.particles > 0 && a->mode == REXLIB_B200_INSERT_DETERMINISTIC)
		fail(REXLIB_B200_UNSUPPORTED, float64_modes);
	copy_accumulators(a, sizeof(double), stream);
	if (L.volumes * L.particles == 0)
		return;
	launch_insert_scatter(L, kind, window_table_f64(a->window), L.big % 2 != 0, stream);
}

void run(const rexlib_b200_insertion *a, insertion_launch &L, weight_kind kind, void *stream_handle)
{
	const cudaStream_t stream = as_stream(stream_handle);
	copy_accumulators(a, sizeof(float), stream);
	if (L.volumes * L.particles == 0)
		return;
	const bool kaiser_bessel = a->window.profile == REXLIB_B200_WINDOW_KAISER_BESSEL;
	if (tiled_insertion_applies(L, kind, a->mode))
	{
		const size_t need = tiled_insertion_workspace(L, kind, a->mode, false);
		if (need > a->workspace_bytes || (need > 0 && a->workspace == nullptr))
			fail(REXLIB_B200_WORKSPACE_TOO_SMALL,
				"the insertion needs " + std::to_string(need) + " bytes of workspace");
		if (reinterpret_cast<uintptr_t>(a->workspace) % 256 != 0)
			fail(REXLIB_B200_INVALID_ARGUMENT, "the workspace must be 256-byte aligned");
		launch_insert_tiled(L, kind, a->mode, false, a->workspace, a->workspace_bytes,
			kaiser_bessel ? window_table(a->window) : nullptr, stream);
		return;
	}
	if (a->mode == REXLIB_B200_INSERT_DETERMINISTIC)
		fail(REXLIB_B200_UNSUPPORTED, deterministic_limits);
	launch_insert_scatter(L, kind, window_table(a->window), L.big % 2 != 0, stream);
}

// Scratch for callers that cannot allocate device memory (see
// rexlib_b200_insert_ctf_slices_fixed_scratch in include/rexlib_b200.h): a
// fixed array in the library's device image, 8 MiB on every device that
// loads the library, held until the process exits.
constexpr size_t fixed_scratch_bytes = size_t(8) << 20;
static __device__ __align__(256) unsigned char fixed_scratch[fixed_scratch_bytes];

// The device address of the fixed scratch in the current context. The host
// name of the array is only a stand-in for it. The address belongs to the
// context that loaded the library's module, and a cudaDeviceReset or another
// context made current loads it again elsewhere, so it is looked up on every
// call rather than cached: the lookup allocates nothing. The first call in a
// context loads the module there, which is why that call should come before
// any stream capture.
void *fixed_scratch_in_current_context()
{
	void *address = nullptr;
	check_cuda(cudaGetSymbolAddress(&address, fixed_scratch), "address of the fixed insertion scratch");
	require(address != nullptr, "the fixed insertion scratch has no device address");
	return address;
}

// insert_ctf_slices with the fixed scratch in place of a caller's workspace:
// the float64 path needs no scratch.
void run_fixed_scratch(const rexlib_b200_insertion *a, insertion_launch_of<double> &L, void *stream_handle)
{
	run(a, L, weight_kind::ctf, stream_handle);
}

void run_fixed_scratch(const rexlib_b200_insertion *a, insertion_launch &L, void *stream_handle)
{
	const cudaStream_t stream = as_stream(stream_handle);
	const bool tiled = L.volumes * L.particles > 0 && tiled_insertion_applies(L, weight_kind::ctf, a->mode);
	if (tiled)
	{
		const size_t need = tiled_insertion_workspace(L, weight_kind::ctf, a->mode, true);
		if (need > fixed_scratch_bytes)
			fail(REXLIB_B200_INVALID_ARGUMENT,
				"this insertion needs " + std::to_string(need) + " bytes of scratch, more than the " +
					std::to_string(fixed_scratch_bytes) +
					" bytes the fixed-scratch entry point holds; insert the slices in smaller batches");
	}
	else if (L.volumes * L.particles > 0 && a->mode == REXLIB_B200_INSERT_DETERMINISTIC)
	{
		fail(REXLIB_B200_UNSUPPORTED, deterministic_limits);
	}
	copy_accumulators(a, sizeof(float), stream);
	if (L.volumes * L.particles == 0)
		return;
	const bool kaiser_bessel = a->window.profile == REXLIB_B200_WINDOW_KAISER_BESSEL;
	if (tiled)
	{
		// Every kernel of the call writes the scratch before reading it (the
		// plan pass also resets the work counter), so nothing needs clearing.
		// The tiles stay whole in shared memory: the L2 numerator tiles
		// (about 100 KB per CTA) would not fit.
		launch_insert_tiled(L, weight_kind::ctf, a->mode, true, fixed_scratch_in_current_context(),
			fixed_scratch_bytes, kaiser_bessel ? window_table(a->window) : nullptr, stream);
		return;
	}
	launch_insert_scatter(L, weight_kind::ctf, window_table(a->window), L.big % 2 != 0, stream);
}

// The CTF operand and constants of insert_ctf_slices: the ctf_optics checks
// (src/em/ops/parameters/ctf_optics.cpp:17-51) and the pixel size check of
// insert_ctf_slices_operation.cpp:17-39, then the wavelength, Cs in
// angstroms, asin(Q) and the squared frequency scale in FP64.
template <typename T>
void set_ctf(insertion_launch_of<T> &L, const rexlib_b200_insertion *a, const void *ctf,
	const rexlib_b200_batch_strides &ctf_strides, const rexlib_b200_ctf_optics &optics, double pixel_size)
{
	check_strides(ctf_strides, "ctf");
	require(std::isfinite(optics.voltage) && optics.voltage > 0.0,
		"ctf_optics: the voltage must be finite and positive");
	require(std::isfinite(optics.spherical_aberration), "ctf_optics: the spherical aberration must be finite");
	require(optics.amplitude_contrast >= 0.0 && optics.amplitude_contrast < 1.0,
		"ctf_optics: the amplitude contrast must lie in [0, 1)");
	require(std::isfinite(pixel_size) && pixel_size > 0.0, "the pixel size must be finite and positive");
	require(a->volume_count * a->slices_per_volume == 0 || ctf != nullptr, "null ctf");
	L.extra = static_cast<const T *>(ctf);
	L.extra_stride_v = ctf_strides.volume;
	L.extra_stride_p = ctf_strides.particle;
	const double volts = optics.voltage * 1e3;
	L.ctf_wavelength = 12.2643247 / std::sqrt(volts * (1.0 + 0.978466e-6 * volts));
	L.ctf_aberration = optics.spherical_aberration * 1e7;
	L.ctf_phase_offset = std::asin(optics.amplitude_contrast);
	const double fs = 1.0 / (static_cast<double>(a->slice_extent) * pixel_size);
	L.ctf_frequency_scale_sq = fs * fs;
}

// ---------------------------------------------------------------------------
// Batched calls: argument checks, the online tuner of the throughput mode.

weight_kind kind_of(int32_t kind)
{
	switch (kind)
	{
	case REXLIB_B200_KIND_PLAIN:
		return weight_kind::unit;
	case REXLIB_B200_KIND_CTF:
		return weight_kind::ctf;
	case REXLIB_B200_KIND_WEIGHTED:
		return weight_kind::spectrum;
	default:
		fail(REXLIB_B200_INVALID_ARGUMENT, "unknown insertion kind");
	}
}

// The jobs' launches, checked as one insertion each, with their extra
// operand and the CTF constants.
std::vector<insertion_launch> prepare_jobs(const rexlib_b200_insertion_job *jobs, int32_t count, int32_t kind,
	const rexlib_b200_ctf_optics *optics, double pixel_size)
{
	require(jobs != nullptr, "null job list");
	if (count < 1 || count > 64)
		fail(REXLIB_B200_UNSUPPORTED, "a batched call takes 1 to 64 jobs");
	const rexlib_b200_insertion &first = jobs[0].insertion;
	std::vector<insertion_launch> out;
	out.reserve(static_cast<size_t>(count));
	const weight_kind k = kind_of(kind);
	for (int32_t j = 0; j < count; ++j)
	{
		const rexlib_b200_insertion &a = jobs[j].insertion;
		if (a.element_type != REXLIB_B200_FLOAT32)
			fail(REXLIB_B200_UNSUPPORTED, "batched insertions run float32 operands");
		require(a.mode == first.mode && a.window.profile == first.window.profile &&
				a.window.half_width == first.window.half_width && a.window.shape == first.window.shape,
			"the jobs of a batched call share one window and one mode");
		insertion_launch L = prepare<float>(&a);
		require(L.volumes * L.particles > 0, "every job of a batched call inserts slices");
		if (L.profile == REXLIB_B200_WINDOW_KAISER_BESSEL && a.window.half_width > 2.0)
			fail(REXLIB_B200_UNSUPPORTED, "batched calls take Kaiser-Bessel half-widths up to 2");
		if (first.mode == REXLIB_B200_INSERT_THROUGHPUT)
		{
			if (L.big < 16)
				fail(REXLIB_B200_UNSUPPORTED, "batched throughput calls take volume extents of 16 and more");
		}
		if (k != weight_kind::unit)
		{
			check_strides(jobs[j].extra_strides, k == weight_kind::ctf ? "ctf" : "weights");
			require(jobs[j].extra != nullptr, k == weight_kind::ctf ? "null ctf" : "null weights");
			L.extra = static_cast<const float *>(jobs[j].extra);
			L.extra_stride_v = jobs[j].extra_strides.volume;
			L.extra_stride_p = jobs[j].extra_strides.particle;
		}
		if (k == weight_kind::ctf)
			set_ctf(L, &a, jobs[j].extra, jobs[j].extra_strides, *optics, pixel_size);
		out.push_back(L);
	}
	return out;
}

// Candidate settings the tuner times, the default first.
const tile_config tune_candidates[] = {
	{12000, 320, 2560}, {8000, 320, 2560}, {16000, 320, 2560},
	{12000, 320, 640},  {12000, 640, 5120}, {12000, 160, 1280},
};
constexpr int tune_count = static_cast<int>(sizeof(tune_candidates) / sizeof(tune_candidates[0]));

struct tune_state
{
	int chosen = -1; // index into tune_candidates, or -1 while tuning
	int next = 0;    // the next candidate to try
	cudaEvent_t begin[tune_count] = {};
	cudaEvent_t end[tune_count] = {};
	float ms[tune_count] = {};
	bool timed[tune_count] = {};
};

std::mutex tune_mutex;
std::map<std::string, tune_state> tune_states;
bool tune_cache_read = false;

// A job set: the kind, window and every job's extents, volumes and
// particle count rounded to a power of two.
std::string signature(const std::vector<insertion_launch> &L, int32_t kind, const rexlib_b200_gridding_window &w)
{
	std::ostringstream o;
	o << "k" << kind << "w" << w.profile << ":" << w.half_width << ":" << w.shape;
	for (const auto &j : L)
	{
		int bucket = 0;
		while ((int64_t(1) << (bucket + 1)) <= j.particles)
			++bucket;
		o << "|" << j.n << "," << j.big << "," << j.volumes << "," << bucket;
	}
	return o.str();
}

const char *tune_cache_path()
{
	const char *p = std::getenv("REXLIB_B200_TUNE_CACHE");
	return p != nullptr && *p != '\0' ? p : nullptr;
}

// Lines of the cache file: signature, cells, min_hits, max_hits, ms.
void read_tune_cache_locked()
{
	if (tune_cache_read)
		return;
	tune_cache_read = true;
	const char *path = tune_cache_path();
	if (path == nullptr)
		return;
	std::ifstream in(path);
	std::string line;
	while (std::getline(in, line))
	{
		std::istringstream fields(line);
		std::string key;
		tile_config c{};
		float ms = 0.0f;
		if (!(fields >> key >> c.cells >> c.min_hits >> c.max_hits >> ms))
			continue;
		for (int i = 0; i < tune_count; ++i)
			if (tune_candidates[i].cells == c.cells && tune_candidates[i].min_hits == c.min_hits &&
				tune_candidates[i].max_hits == c.max_hits)
				tune_states[key].chosen = i;
	}
}

void write_tune_cache_locked(const std::string &key, int chosen, float ms)
{
	const char *path = tune_cache_path();
	if (path == nullptr)
		return;
	std::ofstream out(path, std::ios::app);
	const tile_config &c = tune_candidates[chosen];
	out << key << " " << c.cells << " " << c.min_hits << " " << c.max_hits << " " << ms << "\n";
}

// Collects the candidates' timings whose events have completed; chooses
// the fastest once every candidate is timed.
void settle_tuning_locked(const std::string &key, tune_state &t)
{
	if (t.chosen >= 0)
		return;
	int timed = 0;
	for (int i = 0; i < t.next; ++i)
	{
		if (!t.timed[i] && cudaEventQuery(t.end[i]) == cudaSuccess)
		{
			cudaEventElapsedTime(&t.ms[i], t.begin[i], t.end[i]);
			t.timed[i] = true;
		}
		timed += t.timed[i] ? 1 : 0;
	}
	cudaGetLastError(); // a query of an unfinished event is not an error
	if (timed < tune_count)
		return;
	int best = 0;
	for (int i = 1; i < tune_count; ++i)
		if (t.ms[i] < t.ms[best])
			best = i;
	t.chosen = best;
	for (int i = 0; i < tune_count; ++i)
	{
		cudaEventDestroy(t.begin[i]);
		cudaEventDestroy(t.end[i]);
	}
	write_tune_cache_locked(key, best, t.ms[best]);
}

} // anonymous namespace
} // namespace rexlib_b200

using namespace rexlib_b200;

extern "C" {

int32_t rexlib_b200_abi_version(void) { return REXLIB_B200_ABI_VERSION; }

int32_t rexlib_b200_insertion_workspace_size(const rexlib_b200_insertion *insertion, size_t *bytes)
{
	return guarded([&] {
		require(bytes != nullptr, "null result pointer");
		*bytes = 0;
		with_element_type(insertion, [&](auto L) {
			if constexpr (std::is_same_v<decltype(L), insertion_launch>)
				if (tiled_insertion_applies(L, weight_kind::unit, insertion->mode))
					*bytes = tiled_insertion_workspace(L, weight_kind::unit, insertion->mode, false);
		});
	});
}

int32_t rexlib_b200_insertion_launches(const rexlib_b200_insertion *insertion, int32_t *count)
{
	return guarded([&] {
		require(count != nullptr, "null result pointer");
		with_element_type(insertion, [&](auto L) {
			if (L.volumes * L.particles == 0)
				*count = 0;
			else
				*count = 1;
			if constexpr (std::is_same_v<decltype(L), insertion_launch>)
				if (L.volumes * L.particles > 0 && tiled_insertion_applies(L, weight_kind::unit, insertion->mode))
					*count = tiled_insertion_launches(insertion->mode);
		});
	});
}

int32_t rexlib_b200_insert_slices(const rexlib_b200_insertion *insertion, void *stream)
{
	return guarded([&] { with_element_type(insertion, [&](auto L) { run(insertion, L, weight_kind::unit, stream); }); });
}

int32_t rexlib_b200_insert_weighted_slices(const rexlib_b200_insertion *insertion, const void *weights,
	rexlib_b200_batch_strides weight_strides, void *stream)
{
	return guarded([&] {
		with_element_type(insertion, [&](auto L) {
			check_strides(weight_strides, "weights");
			require(insertion->volume_count * insertion->slices_per_volume == 0 || weights != nullptr,
				"null weights");
			L.extra = static_cast<decltype(L.extra)>(weights);
			L.extra_stride_v = weight_strides.volume;
			L.extra_stride_p = weight_strides.particle;
			run(insertion, L, weight_kind::spectrum, stream);
		});
	});
}

int32_t rexlib_b200_insert_ctf_slices(const rexlib_b200_insertion *insertion, const void *ctf,
	rexlib_b200_batch_strides ctf_strides, rexlib_b200_ctf_optics optics, double pixel_size, void *stream)
{
	return guarded([&] {
		with_element_type(insertion, [&](auto L) {
			set_ctf(L, insertion, ctf, ctf_strides, optics, pixel_size);
			run(insertion, L, weight_kind::ctf, stream);
		});
	});
}

} // extern "C"

extern "C" int32_t rexlib_b200_insert_ctf_slices_fixed_scratch(const rexlib_b200_insertion *insertion,
	const void *ctf, rexlib_b200_batch_strides ctf_strides, rexlib_b200_ctf_optics optics, double pixel_size,
	void *stream)
{
	return guarded([&] {
		with_element_type(insertion, [&](auto L) {
			set_ctf(L, insertion, ctf, ctf_strides, optics, pixel_size);
			run_fixed_scratch(insertion, L, stream);
		});
	});
}

extern "C" int32_t rexlib_b200_batched_insertion_workspace_size(const rexlib_b200_insertion_job *jobs,
	int32_t job_count, int32_t kind, size_t *bytes)
{
	return guarded([&] {
		require(bytes != nullptr, "null result pointer");
		const rexlib_b200_ctf_optics optics{300.0, 2.7, 0.1};
		const std::vector<insertion_launch> L = prepare_jobs(jobs, job_count, kind, &optics, 1.0);
		const kb_table *kb = window_table(jobs[0].insertion.window);
		size_t most = 0;
		const int mode = jobs[0].insertion.mode;
		for (int i = 0; i < (mode == REXLIB_B200_INSERT_DETERMINISTIC ? 1 : tune_count); ++i)
			most = std::max(most, batched_insertion_workspace(L.data(), job_count, kind_of(kind), mode,
				tune_candidates[i], *kb));
		*bytes = most;
	});
}

extern "C" int32_t rexlib_b200_batched_insert(const rexlib_b200_insertion_job *jobs, int32_t job_count,
	int32_t kind, rexlib_b200_ctf_optics optics, double pixel_size, void *workspace, size_t workspace_bytes,
	void *stream_handle)
{
	return guarded([&] {
		const cudaStream_t stream = as_stream(stream_handle);
		const std::vector<insertion_launch> L = prepare_jobs(jobs, job_count, kind, &optics, pixel_size);
		if (reinterpret_cast<uintptr_t>(workspace) % 256 != 0)
			fail(REXLIB_B200_INVALID_ARGUMENT, "the workspace must be 256-byte aligned");
		const kb_table *kb = window_table(jobs[0].insertion.window);
		const int mode = jobs[0].insertion.mode;
		for (int32_t j = 0; j < job_count; ++j)
			copy_accumulators(&jobs[j].insertion, sizeof(float), stream);
		tile_config config = tune_candidates[0];
		int timing = -1;
		std::string key;
		cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
		check_cuda(cudaStreamIsCapturing(stream, &capture), "capture query");
		if (mode == REXLIB_B200_INSERT_THROUGHPUT)
		{
			key = signature(L, kind, jobs[0].insertion.window);
			std::lock_guard<std::mutex> lock(tune_mutex);
			read_tune_cache_locked();
			tune_state &t = tune_states[key];
			settle_tuning_locked(key, t);
			if (t.chosen >= 0)
				config = tune_candidates[t.chosen];
			else if (capture == cudaStreamCaptureStatusNone && t.next < tune_count)
			{
				timing = t.next++;
				config = tune_candidates[timing];
				check_cuda(cudaEventCreate(&t.begin[timing]), "tuning event");
				check_cuda(cudaEventCreate(&t.end[timing]), "tuning event");
				check_cuda(cudaEventRecord(t.begin[timing], stream), "tuning event");
			}
		}
		launch_batched_insertion(L.data(), job_count, kind_of(kind), mode, config, *kb, workspace, workspace_bytes,
			stream);
		if (timing >= 0)
		{
			std::lock_guard<std::mutex> lock(tune_mutex);
			check_cuda(cudaEventRecord(tune_states[key].end[timing], stream), "tuning event");
		}
	});
}

extern "C" int32_t rexlib_b200_batched_tuning(const rexlib_b200_insertion_job *jobs, int32_t job_count,
	int32_t kind, int32_t *tuned, rexlib_b200_tile_config *config)
{
	return guarded([&] {
		require(tuned != nullptr && config != nullptr, "null result pointer");
		const rexlib_b200_ctf_optics optics{300.0, 2.7, 0.1};
		const std::vector<insertion_launch> L = prepare_jobs(jobs, job_count, kind, &optics, 1.0);
		const std::string key = signature(L, kind, jobs[0].insertion.window);
		std::lock_guard<std::mutex> lock(tune_mutex);
		read_tune_cache_locked();
		tune_state &t = tune_states[key];
		settle_tuning_locked(key, t);
		const tile_config &c = tune_candidates[t.chosen >= 0 ? t.chosen : 0];
		*tuned = t.chosen >= 0 ? 1 : 0;
		config->cells = c.cells;
		config->min_hits = c.min_hits;
		config->max_hits = c.max_hits;
	});
}

extern "C" int32_t rexlib_b200_batched_insertion_launches(int32_t mode, int32_t *count)
{
	return guarded([&] {
		require(count != nullptr, "null result pointer");
		*count = batched_insertion_launches(mode);
	});
}
