// C entry points of the insertions: argument checks (the shape and type
// rules of include/rexlib/em/ops/reconstruction/slice_insertion_rules.hpp
// and the parameter checks of src/em/ops/parameters/*.cpp), the copy of the
// accumulators into distinct outputs, and the choice of kernel.
#include "insertion.cuh"

#include <array>
#include <cmath>
#include <mutex>
#include <string>

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
// voxel of half-width, two zeros past the end).
void fill_kb_table(const rexlib_b200_gridding_window &w, kb_table &kb)
{
	kb.half_width = static_cast<float>(w.half_width);
	kb.tap_count = static_cast<int>(std::ceil(2.0 * w.half_width));
	if (w.profile != REXLIB_B200_WINDOW_KAISER_BESSEL)
	{
		kb.tap_count = w.profile == REXLIB_B200_WINDOW_BOX ? 1 : 2;
		kb.scale = 0.0f;
		kb.step_count = 0;
		return;
	}
	const double normalization = 1.0 / bessel_i0(w.shape);
	const long count = static_cast<long>(std::ceil(w.half_width * 1024.0));
	kb.scale = static_cast<float>(static_cast<double>(count) / w.half_width);
	kb.step_count = static_cast<int>(count);
	for (long i = 0; i < kb_table_capacity; ++i)
		kb.values[i] = 0.0f;
	for (long i = 0; i <= count; ++i)
	{
		const double ratio = static_cast<double>(i) / static_cast<double>(count);
		kb.values[i] = static_cast<float>(bessel_i0(w.shape * std::sqrt(1.0 - ratio * ratio)) * normalization);
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

void check_strides(const rexlib_b200_batch_strides &s, const char *name)
{
	require(s.volume >= 0 && s.particle >= 0, std::string(name) + ": batch strides must be 0 or more");
}

insertion_launch prepare(const rexlib_b200_insertion *a)
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
	require((reinterpret_cast<uintptr_t>(a->numerator_out) % 8) == 0 &&
			(reinterpret_cast<uintptr_t>(a->numerator_in) % 8) == 0 &&
			(reinterpret_cast<uintptr_t>(a->slices) % 8) == 0,
		"complex operands must be 8-byte aligned");

	insertion_launch L{};
	L.numerator = static_cast<float2 *>(a->numerator_out);
	L.denominator = a->denominator_out;
	L.slices = static_cast<const float2 *>(a->slices);
	L.transforms = a->transforms;
	L.radial = a->radial_weights;
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

// Outputs = inputs + insertions: copy the inputs over distinct outputs.
void copy_accumulators(const rexlib_b200_insertion *a, cudaStream_t stream)
{
	const size_t voxels = static_cast<size_t>(a->volume_count) * a->volume_extent * a->volume_extent *
		(a->volume_extent / 2 + 1);
	if (voxels == 0)
		return;
	if (a->numerator_out != a->numerator_in)
		check_cuda(cudaMemcpyAsync(a->numerator_out, a->numerator_in, voxels * 8, cudaMemcpyDeviceToDevice, stream),
			"copy of the numerator");
	if (a->denominator_out != a->denominator_in)
		check_cuda(cudaMemcpyAsync(a->denominator_out, a->denominator_in, voxels * 4, cudaMemcpyDeviceToDevice,
					   stream),
			"copy of the denominator");
}

void run(const rexlib_b200_insertion *a, insertion_launch &L, weight_kind kind, void *stream_handle)
{
	const cudaStream_t stream = as_stream(stream_handle);
	copy_accumulators(a, stream);
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

std::mutex fixed_scratch_mutex;
std::array<void *, 256> fixed_scratch_address{};

// The device address of the fixed scratch on the current device. The host
// name of the array is only a stand-in for it; the address is looked up once
// per device, with that device current, on the first call there.
void *fixed_scratch_on_current_device()
{
	int device = -1;
	check_cuda(cudaGetDevice(&device), "current device");
	require(device >= 0 && device < static_cast<int>(fixed_scratch_address.size()), "device index out of range");
	std::lock_guard<std::mutex> lock(fixed_scratch_mutex);
	if (fixed_scratch_address[device] == nullptr)
	{
		void *address = nullptr;
		check_cuda(cudaGetSymbolAddress(&address, fixed_scratch), "address of the fixed insertion scratch");
		fixed_scratch_address[device] = address;
	}
	return fixed_scratch_address[device];
}

// insert_ctf_slices with the fixed scratch in place of a caller's workspace.
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
	copy_accumulators(a, stream);
	if (L.volumes * L.particles == 0)
		return;
	const bool kaiser_bessel = a->window.profile == REXLIB_B200_WINDOW_KAISER_BESSEL;
	if (tiled)
	{
		// Every kernel of the call writes the scratch before reading it (the
		// plan pass also resets the work counter), so nothing needs clearing.
		// The tiles stay whole in shared memory: the L2 numerator tiles
		// (about 100 KB per CTA) would not fit.
		launch_insert_tiled(L, weight_kind::ctf, a->mode, true, fixed_scratch_on_current_device(),
			fixed_scratch_bytes, kaiser_bessel ? window_table(a->window) : nullptr, stream);
		return;
	}
	launch_insert_scatter(L, weight_kind::ctf, window_table(a->window), L.big % 2 != 0, stream);
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
		insertion_launch L = prepare(insertion);
		*bytes = tiled_insertion_applies(L, weight_kind::unit, insertion->mode)
			? tiled_insertion_workspace(L, weight_kind::unit, insertion->mode, false)
			: 0;
	});
}

int32_t rexlib_b200_insertion_launches(const rexlib_b200_insertion *insertion, int32_t *count)
{
	return guarded([&] {
		require(count != nullptr, "null result pointer");
		insertion_launch L = prepare(insertion);
		if (L.volumes * L.particles == 0)
			*count = 0;
		else if (tiled_insertion_applies(L, weight_kind::unit, insertion->mode))
			*count = tiled_insertion_launches(insertion->mode);
		else
			*count = 1;
	});
}

int32_t rexlib_b200_insert_slices(const rexlib_b200_insertion *insertion, void *stream)
{
	return guarded([&] {
		insertion_launch L = prepare(insertion);
		run(insertion, L, weight_kind::unit, stream);
	});
}

int32_t rexlib_b200_insert_weighted_slices(const rexlib_b200_insertion *insertion, const float *weights,
	rexlib_b200_batch_strides weight_strides, void *stream)
{
	return guarded([&] {
		insertion_launch L = prepare(insertion);
		check_strides(weight_strides, "weights");
		require(insertion->volume_count * insertion->slices_per_volume == 0 || weights != nullptr, "null weights");
		L.extra = weights;
		L.extra_stride_v = weight_strides.volume;
		L.extra_stride_p = weight_strides.particle;
		run(insertion, L, weight_kind::spectrum, stream);
	});
}

int32_t rexlib_b200_insert_ctf_slices(const rexlib_b200_insertion *insertion, const float *ctf,
	rexlib_b200_batch_strides ctf_strides, rexlib_b200_ctf_optics optics, double pixel_size, void *stream)
{
	return guarded([&] {
		insertion_launch L = prepare(insertion);
		check_strides(ctf_strides, "ctf");
		// ctf_optics checks (src/em/ops/parameters/ctf_optics.cpp:17-51) and
		// the pixel size check of insert_ctf_slices_operation.cpp:17-39.
		require(std::isfinite(optics.voltage) && optics.voltage > 0.0,
			"ctf_optics: the voltage must be finite and positive");
		require(std::isfinite(optics.spherical_aberration), "ctf_optics: the spherical aberration must be finite");
		require(optics.amplitude_contrast >= 0.0 && optics.amplitude_contrast < 1.0,
			"ctf_optics: the amplitude contrast must lie in [0, 1)");
		require(std::isfinite(pixel_size) && pixel_size > 0.0, "the pixel size must be finite and positive");
		require(insertion->volume_count * insertion->slices_per_volume == 0 || ctf != nullptr, "null ctf");
		L.extra = ctf;
		L.extra_stride_v = ctf_strides.volume;
		L.extra_stride_p = ctf_strides.particle;
		const double volts = optics.voltage * 1e3;
		L.ctf_wavelength = 12.2643247 / std::sqrt(volts * (1.0 + 0.978466e-6 * volts));
		L.ctf_aberration = optics.spherical_aberration * 1e7;
		L.ctf_phase_offset = std::asin(optics.amplitude_contrast);
		const double fs = 1.0 / (static_cast<double>(insertion->slice_extent) * pixel_size);
		L.ctf_frequency_scale_sq = fs * fs;
		run(insertion, L, weight_kind::ctf, stream);
	});
}

} // extern "C"

extern "C" int32_t rexlib_b200_insert_ctf_slices_fixed_scratch(const rexlib_b200_insertion *insertion,
	const float *ctf, rexlib_b200_batch_strides ctf_strides, rexlib_b200_ctf_optics optics, double pixel_size,
	void *stream)
{
	return guarded([&] {
		insertion_launch L = prepare(insertion);
		check_strides(ctf_strides, "ctf");
		require(std::isfinite(optics.voltage) && optics.voltage > 0.0,
			"ctf_optics: the voltage must be finite and positive");
		require(std::isfinite(optics.spherical_aberration), "ctf_optics: the spherical aberration must be finite");
		require(optics.amplitude_contrast >= 0.0 && optics.amplitude_contrast < 1.0,
			"ctf_optics: the amplitude contrast must lie in [0, 1)");
		require(std::isfinite(pixel_size) && pixel_size > 0.0, "the pixel size must be finite and positive");
		require(insertion->volume_count * insertion->slices_per_volume == 0 || ctf != nullptr, "null ctf");
		L.extra = ctf;
		L.extra_stride_v = ctf_strides.volume;
		L.extra_stride_p = ctf_strides.particle;
		const double volts = optics.voltage * 1e3;
		L.ctf_wavelength = 12.2643247 / std::sqrt(volts * (1.0 + 0.978466e-6 * volts));
		L.ctf_aberration = optics.spherical_aberration * 1e7;
		L.ctf_phase_offset = std::asin(optics.amplitude_contrast);
		const double fs = 1.0 / (static_cast<double>(insertion->slice_extent) * pixel_size);
		L.ctf_frequency_scale_sq = fs * fs;
		run_fixed_scratch(insertion, L, stream);
	});
}
