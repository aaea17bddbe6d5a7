// Test driver: rexlib itself (librexlib.so, the reference's core compiled
// from its sources by oracle/ref's `make core`) loading the B200 plugin
// through its plugin manager and running the em operations through
// execute() and the eager dispatcher, as a rexlib user's program would. The
// tests call these C functions through ctypes and compare the results with
// the C-ABI path and the oracle.
//
// Test infrastructure only: the product is the plugin; this is its caller.
#include <rexlib/core/dispatch/dispatcher.hpp>
#include <rexlib/core/dispatch/execution_context.hpp>
#include <rexlib/core/dispatch/program_service.hpp>
#include <rexlib/core/hardware/buffer.hpp>
#include <rexlib/core/hardware/device_context.hpp>
#include <rexlib/core/hardware/device_index.hpp>
#include <rexlib/core/hardware/device_service.hpp>
#include <rexlib/core/hardware/memory_resource_affinity.hpp>
#include <rexlib/core/layout/strided_layout.hpp>
#include <rexlib/core/ndarray/access_hazard_tracker.hpp>
#include <rexlib/core/ndarray/array.hpp>
#include <rexlib/core/ndarray/array_descriptor.hpp>
#include <rexlib/core/ndarray/const_array_ref.hpp>
#include <rexlib/core/numerical/numerical_type.hpp>
#include <rexlib/core/plugin.hpp>
#include <rexlib/core/plugin_manager.hpp>
#include <rexlib/core/service_catalog.hpp>
#include <rexlib/core/span.hpp>
#include <rexlib/em/functional/preprocessing.hpp>
#include <rexlib/em/functional/reconstruction.hpp>
#include <rexlib/em/ops/parameters/ctf_optics.hpp>
#include <rexlib/em/ops/parameters/gridding_window.hpp>
#include <rexlib/functional/creation.hpp>
#include <rexlib/functional/fourier.hpp>
#include <rexlib/functional/transfer.hpp>

#include "../../rexlib_b200/plugin/batch_plan.hpp"

#include <cstdint>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace
{

struct session
{
	rexlib::service_catalog catalog{false};
	rexlib::plugin_manager plugins;
	rexlib::execution_context context;
	bool has_context = false;
};

std::unique_ptr<session> g_session;
std::string g_error;

template <typename F>
int32_t guarded(F &&f)
{
	try
	{
		g_error.clear();
		return f();
	}
	catch (const std::exception &e)
	{
		g_error = e.what();
		return -1;
	}
	catch (...)
	{
		g_error = "unknown exception";
		return -1;
	}
}

// An operand passed from Python: host data, its type and extents.
struct driver_array
{
	void *data;
	int32_t dtype; // 0 float32, 1 float64, 2 complex64, 3 complex128, 4 uint64
	int32_t rank;
	int64_t extents[8];
};

rexlib::numerical_type type_of(int32_t code)
{
	switch (code)
	{
	case 0:
		return rexlib::numerical_type::float32;
	case 1:
		return rexlib::numerical_type::float64;
	case 2:
		return rexlib::numerical_type::complex_float32;
	case 3:
		return rexlib::numerical_type::complex_float64;
	case 4:
		return rexlib::numerical_type::uint64;
	default:
		throw std::invalid_argument("unknown type code");
	}
}

std::size_t bytes_of(int32_t code)
{
	static const std::size_t bytes[] = {4, 8, 8, 16, 8};
	return bytes[code];
}

std::vector<std::size_t> extents_of(const driver_array &a)
{
	return std::vector<std::size_t>(a.extents, a.extents + a.rank);
}

std::size_t count_of(const driver_array &a)
{
	std::size_t n = 1;
	for (int i = 0; i < a.rank; ++i)
		n *= static_cast<std::size_t>(a.extents[i]);
	return n;
}

rexlib::array_descriptor descriptor_of(const driver_array &a)
{
	const auto e = extents_of(a);
	return rexlib::array_descriptor(rexlib::strided_layout::make_contiguous_layout(rexlib::make_span(e)),
		type_of(a.dtype));
}

const rexlib::execution_context &context()
{
	if (!g_session || !g_session->has_context)
		throw std::logic_error("no b200 execution context: call driver_open_device first");
	return g_session->context;
}

// A host array from the context's host allocator (the plugin's pinned
// memory) holding a copy of `a`.
rexlib::array host_array(const driver_array &a)
{
	rexlib::array h = rexlib::empty(descriptor_of(a), rexlib::memory_resource_affinity::host, context());
	h.get_access_hazard_tracker()->wait(rexlib::read_write);
	void *p = h.get_storage()->get_host_ptr();
	if (p == nullptr)
		throw std::runtime_error("the host allocator gave memory the host cannot reach");
	std::memcpy(p, a.data, count_of(a) * bytes_of(a.dtype));
	return h;
}

rexlib::array device_array(const driver_array &a)
{
	rexlib::array h = host_array(a);
	return rexlib::to_device_copy(h, context());
}

void read_back(rexlib::array &device, driver_array &a)
{
	rexlib::array h = rexlib::to_host_copy(device, context());
	h.get_access_hazard_tracker()->wait(rexlib::read_only);
	std::memcpy(a.data, h.get_storage()->get_host_ptr(), count_of(a) * bytes_of(a.dtype));
}

rexlib::em::gridding_window window_of(int32_t profile, double half_width, double shape)
{
	if (profile == 0)
		return rexlib::em::gridding_window::nearest();
	if (profile == 1)
		return rexlib::em::gridding_window::linear();
	return rexlib::em::gridding_window::kaiser_bessel(half_width, shape);
}

} // anonymous namespace

extern "C" {

const char *driver_error(void) { return g_error.c_str(); }

// A fresh catalog (no built-in backends) with the plugin at `path` loaded by
// rexlib's plugin manager and registered.
int32_t driver_open(const char *path)
{
	return guarded([&] {
		g_session.reset();
		auto s = std::make_unique<session>();
		s->plugins.load_plugin(path);
		rexlib::register_all_plugins_at(s->plugins, s->catalog);
		g_session = std::move(s);
		return 0;
	});
}

void driver_close(void) { g_session.reset(); }

// The backends the device service knows, comma-separated.
int32_t driver_backends(char *out, int64_t capacity)
{
	return guarded([&] {
		std::vector<std::string> names;
		g_session->catalog.get_service<rexlib::device_service>()->enumerate_backends(names);
		std::string joined;
		for (const auto &n : names)
			joined += (joined.empty() ? "" : ",") + n;
		std::strncpy(out, joined.c_str(), static_cast<std::size_t>(capacity));
		return 0;
	});
}

// Devices the "b200" backend enumerates.
int32_t driver_device_count(void)
{
	return guarded([&] {
		std::vector<rexlib::device_index> indices;
		g_session->catalog.get_service<rexlib::device_service>()->enumerate_devices(indices);
		int32_t n = 0;
		for (const auto &i : indices)
			n += i.get_backend_name() == "b200" ? 1 : 0;
		return n;
	});
}

// An execution context on b200 device `id` with an eager dispatcher.
int32_t driver_open_device(int32_t id)
{
	return guarded([&] {
		auto devices = g_session->catalog.get_service<rexlib::device_service>();
		auto session = devices->create_device_session(rexlib::device_index("b200", static_cast<std::size_t>(id)));
		g_session->context = rexlib::execution_context(rexlib::device_context(session),
			rexlib::make_eager_dispatcher(g_session->catalog.get_service<rexlib::program_service>()));
		g_session->has_context = true;
		return 0;
	});
}

// em::insert_{,weighted_,ctf_}slices (kind 0, 1, 2) on the b200 device: the
// operands copied to the device with to_device_copy, the accumulators
// updated in place, read back with to_host_copy into numerator and
// denominator. host_input names one input (2: slices) left in host memory,
// strided_slices views the slices with a stride of 2 in their last axis (the
// slices array then holds twice the columns); both should find no program.
int32_t driver_insert(int32_t kind, int32_t profile, double half_width, double shape, const double *optics,
	double pixel_size, driver_array *numerator, driver_array *denominator, const driver_array *slices,
	const driver_array *transforms, const driver_array *extra, const driver_array *radial, int32_t host_input,
	int32_t strided_slices)
{
	return guarded([&] {
		rexlib::array num = device_array(*numerator);
		rexlib::array den = device_array(*denominator);
		rexlib::array sl = host_input == 2 ? host_array(*slices) : device_array(*slices);
		if (strided_slices)
		{
			auto e = extents_of(*slices);
			std::vector<std::ptrdiff_t> strides(e.size());
			std::ptrdiff_t s = 1;
			for (std::size_t i = e.size(); i-- > 0;)
			{
				strides[i] = s;
				s *= static_cast<std::ptrdiff_t>(e[i]);
			}
			e.back() /= 2;
			strides.back() = 2;
			sl = rexlib::array(sl.share_storage(), rexlib::array_descriptor(rexlib::strided_layout::make_custom_layout(
				rexlib::make_span(e), rexlib::make_span(strides)), type_of(slices->dtype)));
		}
		rexlib::array tr = device_array(*transforms);
		rexlib::array ra = device_array(*radial);
		const auto window = window_of(profile, half_width, shape);
		if (kind == 0)
		{
			rexlib::em::insert_slices(num, den, sl, tr, ra, window, context(), &num, &den);
		}
		else if (kind == 1)
		{
			rexlib::array w = device_array(*extra);
			rexlib::em::insert_weighted_slices(num, den, sl, w, tr, ra, window, context(), &num, &den);
		}
		else
		{
			rexlib::array c = device_array(*extra);
			rexlib::em::insert_ctf_slices(num, den, sl, tr, c, ra, window,
				rexlib::em::ctf_optics(optics[0], optics[1], optics[2]), pixel_size, context(), &num, &den);
		}
		read_back(num, *numerator);
		read_back(den, *denominator);
		return 0;
	});
}

// zeros on the device, read back (the fill program).
int32_t driver_zeros(driver_array *out)
{
	return guarded([&] {
		rexlib::array z = rexlib::zeros(descriptor_of(*out), rexlib::memory_resource_affinity::device, context());
		read_back(z, *out);
		return 0;
	});
}

// em::standardize_background over the trailing `axes` axes of `value`.
int32_t driver_standardize(const driver_array *value, const driver_array *keys, int32_t axes, double radius,
	double lower, double upper, driver_array *result)
{
	return guarded([&] {
		rexlib::array v = device_array(*value);
		rexlib::array k = device_array(*keys);
		std::vector<std::ptrdiff_t> list;
		for (int32_t i = value->rank - axes; i < value->rank; ++i)
			list.push_back(i);
		rexlib::array r = rexlib::em::standardize_background(v, k, rexlib::make_span(list), radius, lower, upper,
			context());
		read_back(r, *result);
		return 0;
	});
}

// rfft over the last two axes, then irfft back: both spectra and images.
int32_t driver_rfft2(const driver_array *images, driver_array *spectra, driver_array *restored)
{
	return guarded([&] {
		rexlib::array x = device_array(*images);
		const std::ptrdiff_t axes[2] = {images->rank - 2, images->rank - 1};
		rexlib::array f = rexlib::rfft(x, rexlib::make_span(axes, 2), context());
		read_back(f, *spectra);
		rexlib::array y = rexlib::irfft(f, rexlib::make_span(axes, 2),
			static_cast<std::size_t>(images->extents[images->rank - 1]), context());
		read_back(y, *restored);
		return 0;
	});
}

// The plugin's batch plan: volumes, particles and the (volume, particle)
// strides in cores of an operand, for the CPU tests.
int32_t driver_plan(const int64_t *acc, int32_t acc_rank, const int64_t *in, int32_t in_rank, const int64_t *in_strides,
	int64_t core, int64_t *out)
{
	return guarded([&] {
		rexlib_b200::plugin::batch_plan plan;
		std::string why;
		std::vector<std::size_t> a(acc, acc + acc_rank), e(in, in + in_rank);
		std::vector<std::ptrdiff_t> s(in_strides, in_strides + in_rank);
		if (!rexlib_b200::plugin::plan_batches(a, {e}, plan, why))
			throw std::invalid_argument(why);
		int64_t sv = 0, sp = 0;
		const bool flat = rexlib_b200::plugin::batch_strides(plan, e, s, core, sv, sp);
		out[0] = plan.volumes;
		out[1] = plan.particles;
		out[2] = flat ? 1 : 0;
		out[3] = sv;
		out[4] = sp;
		return 0;
	});
}

} // extern "C"
