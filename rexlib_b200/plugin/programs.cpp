// The B200 backend's program builders: one per operation declaration the
// backend serves, each answering the program service's suitability query
// (include/rexlib/core/dispatch/program_builder.hpp:47-97) and building a
// program that forwards its buffers to the C-ABI of librexlib_b200.so.
//
// A builder answers backend_priority::unsupported, without throwing, unless
// the queue is this backend's, every operand lives where the program can
// reach it (this backend's device memory; a copy may also read or write
// host-accessible memory), the types are those the kernels take and the
// layouts are ones the kernels address (contiguous cores; batch axes that
// flatten to one stride each). The CPU backend then serves what is left.
#include "batch_plan.hpp"
#include "hardware.hpp"
#include "registry.hpp"

#include <rexlib_b200.h>

#include <rexlib/core/backend_priority.hpp>
#include <rexlib/core/dispatch/operand_descriptor.hpp>
#include <rexlib/core/dispatch/program_builder.hpp>
#include <rexlib/core/dispatch/program_builder_registration.hpp>
#include <rexlib/core/hardware/memory_resource.hpp>
#include <rexlib/core/hardware/memory_resource_kind.hpp>
#include <rexlib/core/layout/strided_layout.hpp>
#include <rexlib/core/numerical/numerical_type.hpp>
#include <rexlib/core/numerical/scalar_value.hpp>
#include <rexlib/core/operation/operation.hpp>
#include <rexlib/core/operation/operation_cast.hpp>
#include <rexlib/core/operation/operation_id.hpp>
#include <rexlib/em/ops/parameters/ctf_optics.hpp>
#include <rexlib/em/ops/parameters/gridding_profile.hpp>
#include <rexlib/em/ops/parameters/gridding_window.hpp>
#include <rexlib/em/ops/preprocessing/standardize_background_operation.hpp>
#include <rexlib/em/ops/reconstruction/insert_ctf_slices_operation.hpp>
#include <rexlib/em/ops/reconstruction/insert_slices_operation.hpp>
#include <rexlib/em/ops/reconstruction/insert_weighted_slices_operation.hpp>
#include <rexlib/ops/arithmetic/add_operation.hpp>
#include <rexlib/ops/arithmetic/divide_operation.hpp>
#include <rexlib/ops/assignment/copy_operation.hpp>
#include <rexlib/ops/assignment/fill_operation.hpp>
#include <rexlib/ops/fourier/fourier_normalization.hpp>
#include <rexlib/ops/fourier/irfft_operation.hpp>
#include <rexlib/ops/fourier/rfft_operation.hpp>

#include <complex>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

namespace rexlib_b200
{
namespace plugin
{

namespace
{

using rexlib::backend_priority;
using rexlib::numerical_type;
using descriptors = rexlib::span<const rexlib::operand_descriptor>;
using out_buffers = rexlib::span<const std::shared_ptr<rexlib::buffer>>;
using in_buffers = rexlib::span<const std::shared_ptr<const rexlib::buffer>>;

void require_ok(int32_t status)
{
	if (status == REXLIB_B200_OK)
		return;
	const std::string message = rexlib_b200_last_error();
	if (status == REXLIB_B200_INVALID_ARGUMENT)
		throw std::invalid_argument(message);
	throw std::runtime_error(message);
}

// REXLIB_B200_TRACE set: a builder that refuses an operation says why on
// stderr (rexlib's own logging is compiled out of a release build).
void trace_refusal(const char *operation, const std::string &why)
{
	static const bool on = std::getenv("REXLIB_B200_TRACE") != nullptr;
	if (on)
		std::fprintf(stderr, "rexlib_b200: %s: not run on the b200 backend: %s\n", operation, why.c_str());
}

const command_queue *our_queue(rexlib::command_queue &queue) noexcept
{
	return dynamic_cast<const command_queue *>(&queue);
}

// On this backend's device memory, of the queue's device?
bool on_device(const rexlib::operand_descriptor &d, const command_queue &q) noexcept
{
	const memory_resource *m = device_memory_of(d.get_memory_resource());
	return m != nullptr && m->device() == q.device();
}

bool host_accessible(const rexlib::operand_descriptor &d) noexcept
{
	const auto *r = d.get_memory_resource();
	return r != nullptr && rexlib::is_host_accessible(r->get_kind());
}

std::size_t element_bytes(numerical_type t) noexcept
{
	switch (t)
	{
	case numerical_type::float32:
		return 4;
	case numerical_type::float64:
	case numerical_type::complex_float32:
	case numerical_type::int64:
	case numerical_type::uint64:
		return 8;
	case numerical_type::complex_float64:
		return 16;
	default:
		return 0;
	}
}

int32_t element_code(numerical_type t) noexcept
{
	switch (t)
	{
	case numerical_type::float32:
		return REXLIB_B200_FLOAT32;
	case numerical_type::float64:
		return REXLIB_B200_FLOAT64;
	case numerical_type::complex_float32:
		return REXLIB_B200_COMPLEX64;
	case numerical_type::complex_float64:
		return REXLIB_B200_COMPLEX128;
	default:
		return -1;
	}
}

struct layout_of
{
	std::vector<std::size_t> extents;
	std::vector<std::ptrdiff_t> strides;
	std::ptrdiff_t offset = 0;
	std::size_t count = 1;

	explicit layout_of(const rexlib::operand_descriptor &d)
	{
		const auto &l = d.get_layout();
		l.get_extents(extents);
		l.get_strides(strides);
		offset = l.get_offset();
		count = l.compute_element_count();
	}
	bool contiguous() const { return core_is_contiguous(extents, strides, extents.size()); }
	std::vector<std::size_t> batch(std::size_t core_rank) const
	{
		return std::vector<std::size_t>(extents.begin(), extents.end() - static_cast<std::ptrdiff_t>(core_rank));
	}
	std::vector<std::ptrdiff_t> batch_strides(std::size_t core_rank) const
	{
		return std::vector<std::ptrdiff_t>(strides.begin(), strides.end() - static_cast<std::ptrdiff_t>(core_rank));
	}
};

// The byte address of an operand's first element in its buffer.
void *operand_address(rexlib::buffer &b, std::ptrdiff_t offset_bytes)
{
	char *base = static_cast<char *>(address_of(b));
	if (base == nullptr)
		throw std::invalid_argument("rexlib_b200: an operand's buffer is not reachable by the b200 backend");
	return base + offset_bytes;
}

const void *operand_address(const rexlib::buffer &b, std::ptrdiff_t offset_bytes)
{
	const char *base = static_cast<const char *>(address_of(b));
	if (base == nullptr)
		throw std::invalid_argument("rexlib_b200: an operand's buffer is not reachable by the b200 backend");
	return base + offset_bytes;
}

// REXLIB_B200_DETERMINISTIC (unset, "", "0" or "false": throughput mode),
// read when a program is built.
int32_t insertion_mode()
{
	const char *v = std::getenv("REXLIB_B200_DETERMINISTIC");
	if (v == nullptr || *v == '\0' || std::strcmp(v, "0") == 0 || std::strcmp(v, "false") == 0)
		return REXLIB_B200_INSERT_THROUGHPUT;
	return REXLIB_B200_INSERT_DETERMINISTIC;
}

// ---------------------------------------------------------------------------
// Insertions: insert_slices, insert_weighted_slices, insert_ctf_slices.

enum class insertion_kind
{
	plain,
	weighted,
	ctf
};

// Inputs: numerator, denominator, slice, [weight], transform, [ctf], radial.
struct insertion_operands
{
	int slice = 2;
	int extra = -1; // weight or ctf
	int transform = 3;
	int radial = 4;
	std::size_t extra_core = 0;
};

insertion_operands operands_of(insertion_kind kind)
{
	insertion_operands o;
	if (kind == insertion_kind::weighted)
	{
		o.extra = 3;
		o.transform = 4;
		o.radial = 5;
		o.extra_core = 2;
	}
	else if (kind == insertion_kind::ctf)
	{
		o.transform = 3;
		o.extra = 4;
		o.radial = 5;
		o.extra_core = 1;
	}
	return o;
}

rexlib_b200_gridding_window window_of(const rexlib::em::gridding_window &w)
{
	rexlib_b200_gridding_window c{};
	switch (w.get_profile())
	{
	case rexlib::em::gridding_profile::box:
		c.profile = REXLIB_B200_WINDOW_BOX;
		break;
	case rexlib::em::gridding_profile::triangle:
		c.profile = REXLIB_B200_WINDOW_TRIANGLE;
		break;
	default:
		c.profile = REXLIB_B200_WINDOW_KAISER_BESSEL;
	}
	c.half_width = w.get_half_width();
	c.shape = w.get_shape();
	return c;
}

// What the insertion program needs, planned from the descriptors; `ok`
// false (with the reason) when the kernels cannot take the call.
struct insertion_plan
{
	bool ok = false;
	std::string why;
	rexlib_b200_insertion desc{};
	rexlib_b200_batch_strides extra_strides{};
	std::ptrdiff_t offsets[8] = {}; // bytes: outputs 0-1, then inputs at 2 + index
	std::size_t workspace = 0;
};

insertion_plan plan_insertion(insertion_kind kind, const rexlib::em::gridding_window &window, descriptors outs,
	descriptors ins, const command_queue &queue)
{
	insertion_plan p;
	const insertion_operands o = operands_of(kind);
	const std::size_t n_in = kind == insertion_kind::plain ? 5 : 6;
	if (outs.size() != 2 || ins.size() != n_in)
	{
		p.why = "operand counts";
		return p;
	}
	for (const auto &d : outs)
		if (!on_device(d, queue))
		{
			p.why = "an accumulator is not in the b200 device's memory";
			return p;
		}
	for (const auto &d : ins)
		if (!on_device(d, queue))
		{
			p.why = "an input is not in the b200 device's memory";
			return p;
		}
	const numerical_type complex_type = outs[0].get_data_type();
	const numerical_type real_type = outs[1].get_data_type();
	const bool f32 = complex_type == numerical_type::complex_float32 && real_type == numerical_type::float32;
	const bool f64 = complex_type == numerical_type::complex_float64 && real_type == numerical_type::float64;
	if (!f32 && !f64)
	{
		p.why = "element types";
		return p;
	}
	const layout_of num_out(outs[0]), den_out(outs[1]), num_in(ins[0]), den_in(ins[1]);
	const layout_of slice(ins[o.slice]), transform(ins[o.transform]), radial(ins[o.radial]);
	if (num_out.extents.size() < 3 || slice.extents.size() < 2 || transform.extents.size() < 2 ||
		radial.extents.size() < 1)
	{
		p.why = "ranks";
		return p;
	}
	const std::size_t N = num_out.extents[num_out.extents.size() - 3];
	const std::size_t n = slice.extents[slice.extents.size() - 2];
	// Accumulators: contiguous, one after the other.
	for (const layout_of *acc : {&num_out, &den_out, &num_in, &den_in})
		if (!acc->contiguous())
		{
			p.why = "the accumulators are not contiguous";
			return p;
		}
	struct core
	{
		const layout_of *l;
		std::size_t rank;
	};
	std::vector<core> cores = {{&slice, 2}, {&transform, 2}, {&radial, 1}};
	const layout_of *extra = nullptr;
	if (o.extra >= 0)
	{
		extra = new layout_of(ins[o.extra]);
		cores.push_back({extra, o.extra_core});
	}
	std::unique_ptr<const layout_of> extra_owner(extra);
	for (const auto &c : cores)
		if (c.l->extents.size() < c.rank || !core_is_contiguous(c.l->extents, c.l->strides, c.rank))
		{
			p.why = "an operand's core axes are not contiguous";
			return p;
		}
	batch_plan plan;
	std::vector<std::vector<std::size_t>> batches;
	for (const auto &c : cores)
		batches.push_back(c.l->batch(c.rank));
	if (!plan_batches(num_out.batch(3), batches, plan, p.why))
		return p;
	auto strides_of = [&](const layout_of &l, std::size_t rank, rexlib_b200_batch_strides &s) {
		std::size_t core = 1;
		for (std::size_t i = 0; i < rank; ++i)
			core *= l.extents[l.extents.size() - 1 - i];
		int64_t sv = 0, sp = 0;
		if (!batch_strides(plan, l.batch(rank), l.batch_strides(rank), static_cast<int64_t>(core), sv, sp))
			return false;
		s.volume = sv;
		s.particle = sp;
		return true;
	};
	rexlib_b200_insertion &d = p.desc;
	rexlib_b200_batch_strides acc{};
	if (!strides_of(num_out, 3, acc) || !(plan.volumes <= 1 || acc.volume == 1) ||
		!strides_of(slice, 2, d.slice_strides) || !strides_of(transform, 2, d.transform_strides) ||
		!strides_of(radial, 1, d.radial_strides) || (extra && !strides_of(*extra, o.extra_core, p.extra_strides)))
	{
		p.why = "batch axes that do not flatten to one stride each";
		return p;
	}
	d.volume_count = plan.volumes;
	d.slices_per_volume = plan.particles;
	d.slice_extent = static_cast<int64_t>(n);
	d.volume_extent = static_cast<int64_t>(N);
	d.window = window_of(window);
	d.mode = insertion_mode();
	d.element_type = f32 ? REXLIB_B200_FLOAT32 : REXLIB_B200_FLOAT64;
	const std::size_t cb = element_bytes(complex_type), rb = element_bytes(real_type);
	p.offsets[0] = num_out.offset * static_cast<std::ptrdiff_t>(cb);
	p.offsets[1] = den_out.offset * static_cast<std::ptrdiff_t>(rb);
	for (std::size_t i = 0; i < n_in; ++i)
	{
		const std::size_t bytes = element_bytes(ins[i].get_data_type());
		p.offsets[2 + i] = ins[i].get_layout().get_offset() * static_cast<std::ptrdiff_t>(bytes);
	}
	// The kernels' own checks (sizes, windows) decide whether the call is
	// one they run; the workspace is sized with the queue's device current.
	// The buffers are bound at launch: the query sees stand-in addresses,
	// aligned as the buffers are, which it checks but never reads.
	device_scope scope(queue.device());
	rexlib_b200_insertion query = d;
	void *stand_in = reinterpret_cast<void *>(static_cast<uintptr_t>(256));
	query.numerator_out = query.denominator_out = stand_in;
	query.numerator_in = query.denominator_in = query.slices = query.transforms = query.radial_weights = stand_in;
	size_t bytes = 0;
	const int32_t status = rexlib_b200_insertion_workspace_size(&query, &bytes);
	if (status != REXLIB_B200_OK)
	{
		p.why = rexlib_b200_last_error();
		return p;
	}
	p.workspace = bytes;
	p.ok = true;
	return p;
}

class insertion_program final : public program
{
public:
	insertion_program(insertion_kind kind, const insertion_plan &plan, const rexlib::em::ctf_optics *optics,
		double pixel_size)
		: m_kind(kind), m_plan(plan), m_pixel_size(pixel_size)
	{
		if (optics != nullptr)
			m_optics = {optics->get_voltage(), optics->get_spherical_aberration(), optics->get_amplitude_contrast()};
		if (plan.workspace > 0)
			m_scratch.emplace_back(plan.workspace, 256, rexlib::memory_resource_affinity::device);
	}

	void launch(out_buffers outputs, in_buffers inputs, rexlib::span<const std::shared_ptr<rexlib::buffer>> scratch,
		cudaStream_t stream) const override
	{
		const insertion_operands o = operands_of(m_kind);
		rexlib_b200_insertion d = m_plan.desc;
		d.numerator_out = operand_address(*outputs[0], m_plan.offsets[0]);
		d.denominator_out = operand_address(*outputs[1], m_plan.offsets[1]);
		d.numerator_in = operand_address(*inputs[0], m_plan.offsets[2]);
		d.denominator_in = operand_address(*inputs[1], m_plan.offsets[3]);
		d.slices = operand_address(*inputs[o.slice], m_plan.offsets[2 + o.slice]);
		d.transforms = operand_address(*inputs[o.transform], m_plan.offsets[2 + o.transform]);
		d.radial_weights = operand_address(*inputs[o.radial], m_plan.offsets[2 + o.radial]);
		if (m_plan.workspace > 0)
		{
			d.workspace = address_of(*scratch[0]);
			d.workspace_bytes = scratch[0]->get_size();
		}
		switch (m_kind)
		{
		case insertion_kind::plain:
			require_ok(rexlib_b200_insert_slices(&d, stream));
			break;
		case insertion_kind::weighted:
			require_ok(rexlib_b200_insert_weighted_slices(&d, operand_address(*inputs[o.extra],
				m_plan.offsets[2 + o.extra]), m_plan.extra_strides, stream));
			break;
		case insertion_kind::ctf:
			require_ok(rexlib_b200_insert_ctf_slices(&d, operand_address(*inputs[o.extra], m_plan.offsets[2 + o.extra]),
				m_plan.extra_strides, m_optics, m_pixel_size, stream));
			break;
		}
	}

private:
	insertion_kind m_kind;
	insertion_plan m_plan;
	rexlib_b200_ctf_optics m_optics{};
	double m_pixel_size;
};

template <typename Op, insertion_kind KIND>
class insertion_builder final : public rexlib::program_builder
{
public:
	rexlib::operation_id get_operation_id() const noexcept override { return rexlib::operation_id::of<Op>(); }

	backend_priority get_suitability(const rexlib::operation &op, descriptors outs, descriptors ins,
		rexlib::command_queue &queue) const override
	{
		try
		{
			const command_queue *q = our_queue(queue);
			if (q == nullptr)
				return backend_priority::unsupported;
			const auto &typed = rexlib::operation_cast<Op>(op);
			const insertion_plan plan = plan_insertion(KIND, typed.get_window(), outs, ins, *q);
			if (!plan.ok)
				trace_refusal("insertion", plan.why);
			return plan.ok ? backend_priority::optimal : backend_priority::unsupported;
		}
		catch (...)
		{
			return backend_priority::unsupported;
		}
	}

	std::shared_ptr<rexlib::program> build(const rexlib::operation &op, descriptors outs, descriptors ins,
		rexlib::command_queue &queue, rexlib::program_cache *) const override
	{
		const command_queue *q = our_queue(queue);
		if (q == nullptr)
			throw std::invalid_argument("rexlib_b200: not a b200 queue");
		const auto &typed = rexlib::operation_cast<Op>(op);
		const insertion_plan plan = plan_insertion(KIND, typed.get_window(), outs, ins, *q);
		if (!plan.ok)
			throw std::invalid_argument("rexlib_b200: the insertion cannot run on the b200 backend: " + plan.why);
		if constexpr (KIND == insertion_kind::ctf)
			return std::make_shared<insertion_program>(KIND, plan, &typed.get_optics(), typed.get_pixel_size());
		else
			return std::make_shared<insertion_program>(KIND, plan, nullptr, 1.0);
	}
};

const rexlib::program_builder_registration<
	insertion_builder<rexlib::em::insert_slices_operation, insertion_kind::plain>>
	register_insert_slices(get_program_builder_registry());
const rexlib::program_builder_registration<
	insertion_builder<rexlib::em::insert_weighted_slices_operation, insertion_kind::weighted>>
	register_insert_weighted_slices(get_program_builder_registry());
const rexlib::program_builder_registration<
	insertion_builder<rexlib::em::insert_ctf_slices_operation, insertion_kind::ctf>>
	register_insert_ctf_slices(get_program_builder_registry());

// ---------------------------------------------------------------------------
// fill (zeros, ones, full): contiguous float32, float64, complex64 and
// complex128 destinations on the device.

class fill_program final : public program
{
public:
	fill_program(int32_t type, std::size_t count, std::ptrdiff_t offset, const unsigned char *value, std::size_t bytes)
		: m_type(type), m_count(count), m_offset(offset)
	{
		std::memcpy(m_value, value, bytes);
	}
	void launch(out_buffers outputs, in_buffers, rexlib::span<const std::shared_ptr<rexlib::buffer>>,
		cudaStream_t stream) const override
	{
		require_ok(rexlib_b200_fill(operand_address(*outputs[0], m_offset), m_type, static_cast<int64_t>(m_count),
			m_value, stream));
	}

private:
	int32_t m_type;
	std::size_t m_count;
	std::ptrdiff_t m_offset;
	alignas(16) unsigned char m_value[16] = {};
};

class fill_builder final : public rexlib::program_builder
{
public:
	rexlib::operation_id get_operation_id() const noexcept override
	{
		return rexlib::operation_id::of<rexlib::ops::fill_operation>();
	}
	backend_priority get_suitability(const rexlib::operation &, descriptors outs, descriptors,
		rexlib::command_queue &queue) const override
	{
		const command_queue *q = our_queue(queue);
		if (q == nullptr || outs.size() != 1 || !on_device(outs[0], *q) || element_code(outs[0].get_data_type()) < 0)
			return backend_priority::unsupported;
		return layout_of(outs[0]).contiguous() ? backend_priority::optimal : backend_priority::unsupported;
	}
	std::shared_ptr<rexlib::program> build(const rexlib::operation &op, descriptors outs, descriptors,
		rexlib::command_queue &, rexlib::program_cache *) const override
	{
		const auto &fill = rexlib::operation_cast<rexlib::ops::fill_operation>(op);
		const numerical_type t = outs[0].get_data_type();
		const layout_of l(outs[0]);
		unsigned char value[16] = {};
		switch (t)
		{
		case numerical_type::float32:
		{
			const float v = rexlib::scalar_value_cast<float>(fill.get_fill_value());
			std::memcpy(value, &v, sizeof v);
			break;
		}
		case numerical_type::float64:
		{
			const double v = rexlib::scalar_value_cast<double>(fill.get_fill_value());
			std::memcpy(value, &v, sizeof v);
			break;
		}
		case numerical_type::complex_float32:
		{
			const std::complex<float> v = rexlib::scalar_value_cast<std::complex<float>>(fill.get_fill_value());
			std::memcpy(value, &v, sizeof v);
			break;
		}
		default:
		{
			const std::complex<double> v = rexlib::scalar_value_cast<std::complex<double>>(fill.get_fill_value());
			std::memcpy(value, &v, sizeof v);
		}
		}
		return std::make_shared<fill_program>(element_code(t), l.count,
			l.offset * static_cast<std::ptrdiff_t>(element_bytes(t)), value, element_bytes(t));
	}
};

const rexlib::program_builder_registration<fill_builder> register_fill(get_program_builder_registry());

// ---------------------------------------------------------------------------
// copy (to_device, to_host, copies on the device): one contiguous block of
// bytes between this backend's device memory and device or host-accessible
// memory, of one element type.

class copy_program final : public program
{
public:
	copy_program(std::size_t bytes, std::ptrdiff_t out_offset, std::ptrdiff_t in_offset)
		: m_bytes(bytes), m_out(out_offset), m_in(in_offset)
	{
	}
	void launch(out_buffers outputs, in_buffers inputs, rexlib::span<const std::shared_ptr<rexlib::buffer>>,
		cudaStream_t stream) const override
	{
		if (m_bytes == 0)
			return;
		check(cudaMemcpyAsync(operand_address(*outputs[0], m_out), operand_address(*inputs[0], m_in), m_bytes,
				  cudaMemcpyDefault, stream),
			"copy");
	}

private:
	std::size_t m_bytes;
	std::ptrdiff_t m_out, m_in;
};

class copy_builder final : public rexlib::program_builder
{
public:
	rexlib::operation_id get_operation_id() const noexcept override
	{
		return rexlib::operation_id::of<rexlib::ops::copy_operation>();
	}
	backend_priority get_suitability(const rexlib::operation &, descriptors outs, descriptors ins,
		rexlib::command_queue &queue) const override
	{
		const command_queue *q = our_queue(queue);
		if (q == nullptr || outs.size() != 1 || ins.size() != 1)
			return backend_priority::unsupported;
		const bool out_ok = on_device(outs[0], *q) || host_accessible(outs[0]);
		const bool in_ok = on_device(ins[0], *q) || host_accessible(ins[0]);
		// One side at least in this device's memory; the same type and
		// extents on both, each one contiguous block.
		if (!out_ok || !in_ok || !(on_device(outs[0], *q) || on_device(ins[0], *q)))
			return backend_priority::unsupported;
		if (outs[0].get_data_type() != ins[0].get_data_type() || element_bytes(outs[0].get_data_type()) == 0)
			return backend_priority::unsupported;
		const layout_of a(outs[0]), b(ins[0]);
		if (a.extents != b.extents || !a.contiguous() || !b.contiguous())
			return backend_priority::unsupported;
		return backend_priority::optimal;
	}
	std::shared_ptr<rexlib::program> build(const rexlib::operation &, descriptors outs, descriptors ins,
		rexlib::command_queue &, rexlib::program_cache *) const override
	{
		const std::size_t e = element_bytes(outs[0].get_data_type());
		const layout_of a(outs[0]), b(ins[0]);
		return std::make_shared<copy_program>(a.count * e, a.offset * static_cast<std::ptrdiff_t>(e),
			b.offset * static_cast<std::ptrdiff_t>(e));
	}
};

const rexlib::program_builder_registration<copy_builder> register_copy(get_program_builder_registry());

// ---------------------------------------------------------------------------
// add and divide: contiguous operands of one type, each input the result's
// extents or one element.

template <bool DIVIDE>
class binary_program final : public program
{
public:
	binary_program(int32_t type, int64_t count, int64_t x_count, int64_t y_count, const std::ptrdiff_t offsets[3])
		: m_type(type), m_count(count), m_x(x_count), m_y(y_count)
	{
		for (int i = 0; i < 3; ++i)
			m_offsets[i] = offsets[i];
	}
	void launch(out_buffers outputs, in_buffers inputs, rexlib::span<const std::shared_ptr<rexlib::buffer>>,
		cudaStream_t stream) const override
	{
		void *r = operand_address(*outputs[0], m_offsets[0]);
		const void *x = operand_address(*inputs[0], m_offsets[1]);
		const void *y = operand_address(*inputs[1], m_offsets[2]);
		require_ok(DIVIDE ? rexlib_b200_divide(r, x, m_x, y, m_y, m_type, m_count, stream)
						  : rexlib_b200_add(r, x, m_x, y, m_y, m_type, m_count, stream));
	}

private:
	int32_t m_type;
	int64_t m_count, m_x, m_y;
	std::ptrdiff_t m_offsets[3] = {};
};

template <typename Op, bool DIVIDE>
class binary_builder final : public rexlib::program_builder
{
public:
	rexlib::operation_id get_operation_id() const noexcept override { return rexlib::operation_id::of<Op>(); }
	backend_priority get_suitability(const rexlib::operation &, descriptors outs, descriptors ins,
		rexlib::command_queue &queue) const override
	{
		const command_queue *q = our_queue(queue);
		if (q == nullptr || outs.size() != 1 || ins.size() != 2)
			return backend_priority::unsupported;
		const numerical_type t = outs[0].get_data_type();
		if (element_code(t) < 0 || ins[0].get_data_type() != t || ins[1].get_data_type() != t)
			return backend_priority::unsupported;
		if (!on_device(outs[0], *q) || !on_device(ins[0], *q) || !on_device(ins[1], *q))
			return backend_priority::unsupported;
		const layout_of r(outs[0]), x(ins[0]), y(ins[1]);
		if (!r.contiguous() || !x.contiguous() || !y.contiguous())
			return backend_priority::unsupported;
		if ((x.count != r.count && x.count != 1) || (y.count != r.count && y.count != 1))
			return backend_priority::unsupported;
		return backend_priority::optimal;
	}
	std::shared_ptr<rexlib::program> build(const rexlib::operation &, descriptors outs, descriptors ins,
		rexlib::command_queue &, rexlib::program_cache *) const override
	{
		const numerical_type t = outs[0].get_data_type();
		const std::ptrdiff_t e = static_cast<std::ptrdiff_t>(element_bytes(t));
		const layout_of r(outs[0]), x(ins[0]), y(ins[1]);
		const std::ptrdiff_t offsets[3] = {r.offset * e, x.offset * e, y.offset * e};
		return std::make_shared<binary_program<DIVIDE>>(element_code(t), static_cast<int64_t>(r.count),
			static_cast<int64_t>(x.count), static_cast<int64_t>(y.count), offsets);
	}
};

const rexlib::program_builder_registration<binary_builder<rexlib::ops::add_operation, false>> register_add(
	get_program_builder_registry());
const rexlib::program_builder_registration<binary_builder<rexlib::ops::divide_operation, true>> register_divide(
	get_program_builder_registry());

// ---------------------------------------------------------------------------
// rfft over the last two axes (float32 images of the sizes the kernels
// take) and irfft over the last two or three (complex64 half spectra),
// backward normalisation (unnormalised forward, 1/n^d inverse).

bool trailing_axes(rexlib::span<const std::size_t> axes, std::size_t rank, std::size_t count)
{
	if (axes.size() != count)
		return false;
	for (std::size_t i = 0; i < count; ++i)
		if (axes[i] != rank - count + i)
			return false;
	return true;
}

class fft_program final : public program
{
public:
	enum class kind
	{
		r2c2,
		c2r2,
		c2r3
	};
	fft_program(kind k, int64_t batch, int64_t n, std::ptrdiff_t out_offset, std::ptrdiff_t in_offset,
		std::size_t workspace)
		: m_kind(k), m_batch(batch), m_n(n), m_out(out_offset), m_in(in_offset)
	{
		if (workspace > 0)
			m_scratch.emplace_back(workspace, 256, rexlib::memory_resource_affinity::device);
	}
	void launch(out_buffers outputs, in_buffers inputs, rexlib::span<const std::shared_ptr<rexlib::buffer>> scratch,
		cudaStream_t stream) const override
	{
		void *out = operand_address(*outputs[0], m_out);
		const void *in = operand_address(*inputs[0], m_in);
		switch (m_kind)
		{
		case kind::r2c2:
			require_ok(rexlib_b200_rfft2(out, static_cast<const float *>(in), m_batch, m_n, nullptr, stream));
			break;
		case kind::c2r2:
			require_ok(rexlib_b200_irfft2(static_cast<float *>(out), in, m_batch, m_n, stream));
			break;
		case kind::c2r3:
		{
			const std::size_t volume = static_cast<std::size_t>(m_n) * m_n * (m_n / 2 + 1);
			for (int64_t b = 0; b < m_batch; ++b)
				require_ok(rexlib_b200_irfft3(static_cast<float *>(out) + b * m_n * m_n * m_n,
					static_cast<const char *>(in) + b * volume * 8, m_n, address_of(*scratch[0]), scratch[0]->get_size(),
					stream));
		}
		}
	}

private:
	kind m_kind;
	int64_t m_batch, m_n;
	std::ptrdiff_t m_out, m_in;
};

bool square_trailing(const layout_of &l, std::size_t axes, std::size_t last)
{
	const std::size_t r = l.extents.size();
	if (r < axes)
		return false;
	for (std::size_t i = r - axes; i + 1 < r; ++i)
		if (l.extents[i] != l.extents[r - axes])
			return false;
	return l.extents[r - 1] == last;
}

class rfft_builder final : public rexlib::program_builder
{
public:
	rexlib::operation_id get_operation_id() const noexcept override
	{
		return rexlib::operation_id::of<rexlib::ops::rfft_operation>();
	}
	backend_priority get_suitability(const rexlib::operation &op, descriptors outs, descriptors ins,
		rexlib::command_queue &queue) const override
	{
		const command_queue *q = our_queue(queue);
		if (q == nullptr || outs.size() != 1 || ins.size() != 1 || !on_device(outs[0], *q) || !on_device(ins[0], *q))
			return backend_priority::unsupported;
		const auto &fft = rexlib::operation_cast<rexlib::ops::rfft_operation>(op);
		const layout_of out(outs[0]), in(ins[0]);
		if (ins[0].get_data_type() != numerical_type::float32 ||
			outs[0].get_data_type() != numerical_type::complex_float32 || !out.contiguous() || !in.contiguous())
			return backend_priority::unsupported;
		if (fft.get_normalization() != rexlib::ops::fourier_normalization::backward ||
			!trailing_axes(fft.get_parameters().get_axes(), in.extents.size(), 2))
			return backend_priority::unsupported;
		const std::size_t n = in.extents.back();
		if (!square_trailing(in, 2, n) || !square_trailing(out, 2, n / 2 + 1))
			return backend_priority::unsupported;
		switch (n)
		{
		case 32: case 64: case 96: case 128: case 160: case 192: case 200: case 256:
			return backend_priority::optimal;
		default:
			return backend_priority::unsupported;
		}
	}
	std::shared_ptr<rexlib::program> build(const rexlib::operation &, descriptors outs, descriptors ins,
		rexlib::command_queue &, rexlib::program_cache *) const override
	{
		const layout_of out(outs[0]), in(ins[0]);
		const int64_t n = static_cast<int64_t>(in.extents.back());
		return std::make_shared<fft_program>(fft_program::kind::r2c2, static_cast<int64_t>(in.count) / (n * n), n,
			out.offset * 8, in.offset * 4, 0);
	}
};

class irfft_builder final : public rexlib::program_builder
{
public:
	rexlib::operation_id get_operation_id() const noexcept override
	{
		return rexlib::operation_id::of<rexlib::ops::irfft_operation>();
	}
	backend_priority get_suitability(const rexlib::operation &op, descriptors outs, descriptors ins,
		rexlib::command_queue &queue) const override
	{
		const command_queue *q = our_queue(queue);
		if (q == nullptr || outs.size() != 1 || ins.size() != 1 || !on_device(outs[0], *q) || !on_device(ins[0], *q))
			return backend_priority::unsupported;
		const auto &fft = rexlib::operation_cast<rexlib::ops::irfft_operation>(op);
		const layout_of out(outs[0]), in(ins[0]);
		if (ins[0].get_data_type() != numerical_type::complex_float32 ||
			outs[0].get_data_type() != numerical_type::float32 || !out.contiguous() || !in.contiguous())
			return backend_priority::unsupported;
		if (fft.get_normalization() != rexlib::ops::fourier_normalization::backward)
			return backend_priority::unsupported;
		const auto axes = fft.get_parameters().get_axes();
		const std::size_t d = axes.size();
		if ((d != 2 && d != 3) || !trailing_axes(axes, out.extents.size(), d))
			return backend_priority::unsupported;
		const std::size_t n = out.extents.back();
		if (fft.get_parameters().get_extent() != n || !square_trailing(out, d, n) || !square_trailing(in, d, n / 2 + 1))
			return backend_priority::unsupported;
		if (d == 2)
		{
			switch (n)
			{
			case 32: case 64: case 96: case 128: case 160: case 192: case 200:
				return backend_priority::optimal;
			default:
				return backend_priority::unsupported;
			}
		}
		switch (n)
		{
		case 32: case 64: case 96: case 128: case 160: case 192: case 200: case 256:
			return backend_priority::optimal;
		default:
			return backend_priority::unsupported;
		}
	}
	std::shared_ptr<rexlib::program> build(const rexlib::operation &op, descriptors outs, descriptors ins,
		rexlib::command_queue &queue, rexlib::program_cache *) const override
	{
		const auto &fft = rexlib::operation_cast<rexlib::ops::irfft_operation>(op);
		const layout_of out(outs[0]), in(ins[0]);
		const int64_t n = static_cast<int64_t>(out.extents.back());
		const std::size_t d = fft.get_parameters().get_axes().size();
		if (d == 2)
			return std::make_shared<fft_program>(fft_program::kind::c2r2, static_cast<int64_t>(out.count) / (n * n), n,
				out.offset * 4, in.offset * 8, 0);
		size_t workspace = 0;
		{
			device_scope scope(our_queue(queue)->device());
			require_ok(rexlib_b200_irfft3_workspace_size(n, &workspace));
		}
		return std::make_shared<fft_program>(fft_program::kind::c2r3, static_cast<int64_t>(out.count) / (n * n * n), n,
			out.offset * 4, in.offset * 8, workspace);
	}
};

const rexlib::program_builder_registration<rfft_builder> register_rfft(get_program_builder_registry());
const rexlib::program_builder_registration<irfft_builder> register_irfft(get_program_builder_registry());

// ---------------------------------------------------------------------------
// standardize_background over the trailing 2 or 3 axes of contiguous
// float32 images, uint64 keys: one per image, or one per run of images
// (a key whose trailing batch axes are broadcast).

class standardize_program final : public program
{
public:
	standardize_program(const rexlib_b200_standardization &d, std::ptrdiff_t out_offset, std::ptrdiff_t value_offset,
		std::ptrdiff_t key_offset)
		: m_desc(d), m_out(out_offset), m_value(value_offset), m_key(key_offset)
	{
	}
	void launch(out_buffers outputs, in_buffers inputs, rexlib::span<const std::shared_ptr<rexlib::buffer>>,
		cudaStream_t stream) const override
	{
		rexlib_b200_standardization d = m_desc;
		d.result = static_cast<float *>(operand_address(*outputs[0], m_out));
		d.value = static_cast<const float *>(operand_address(*inputs[0], m_value));
		d.keys = static_cast<const uint64_t *>(operand_address(*inputs[1], m_key));
		require_ok(rexlib_b200_standardize_background(&d, stream));
	}

private:
	rexlib_b200_standardization m_desc;
	std::ptrdiff_t m_out, m_value, m_key;
};

// The descriptor for the call, or false when the kernels cannot take it.
bool plan_standardize(const rexlib::em::standardize_background_operation &op, descriptors outs, descriptors ins,
	rexlib_b200_standardization &d)
{
	const layout_of out(outs[0]), value(ins[0]), key(ins[1]);
	const auto axes = op.get_parameters().get_axes();
	const std::size_t rank = value.extents.size();
	const std::size_t d_axes = axes.size();
	if ((d_axes != 2 && d_axes != 3) || !trailing_axes(axes, rank, d_axes))
		return false;
	if (!out.contiguous() || !value.contiguous() || out.extents != value.extents)
		return false;
	const std::size_t batch_rank = rank - d_axes;
	std::vector<std::size_t> batch(value.extents.begin(), value.extents.begin() + static_cast<std::ptrdiff_t>(batch_rank));
	// The key: the batch axes, the trailing ones possibly broadcast (1).
	std::vector<std::size_t> k = key.extents;
	if (k.size() > batch_rank)
		return false;
	k.insert(k.begin(), batch_rank - k.size(), 1);
	std::size_t trailing = batch_rank;
	while (trailing > 0 && k[trailing - 1] == 1)
		--trailing;
	int64_t images_per_key = 1;
	for (std::size_t i = 0; i < batch_rank; ++i)
	{
		if (i < trailing && k[i] != batch[i])
			return false;
		if (i >= trailing)
			images_per_key *= static_cast<int64_t>(batch[i]);
	}
	if (!key.contiguous())
		return false;
	int64_t images = 1;
	for (std::size_t e : batch)
		images *= static_cast<int64_t>(e);
	d = rexlib_b200_standardization{};
	d.images_per_key = images_per_key > 0 ? images_per_key : 1;
	d.batch = images;
	d.rank = static_cast<int32_t>(d_axes);
	for (std::size_t i = 0; i < d_axes; ++i)
		d.extents[i] = static_cast<int64_t>(value.extents[batch_rank + i]);
	d.radius = op.get_radius();
	d.lower_bound = op.get_lower_bound();
	d.upper_bound = op.get_upper_bound();
	return true;
}

class standardize_builder final : public rexlib::program_builder
{
public:
	rexlib::operation_id get_operation_id() const noexcept override
	{
		return rexlib::operation_id::of<rexlib::em::standardize_background_operation>();
	}
	backend_priority get_suitability(const rexlib::operation &op, descriptors outs, descriptors ins,
		rexlib::command_queue &queue) const override
	{
		try
		{
			const command_queue *q = our_queue(queue);
			if (q == nullptr || outs.size() != 1 || ins.size() != 2)
				return backend_priority::unsupported;
			if (!on_device(outs[0], *q) || !on_device(ins[0], *q) || !on_device(ins[1], *q))
				return backend_priority::unsupported;
			if (outs[0].get_data_type() != numerical_type::float32 || ins[0].get_data_type() != numerical_type::float32 ||
				ins[1].get_data_type() != numerical_type::uint64)
				return backend_priority::unsupported;
			rexlib_b200_standardization d{};
			return plan_standardize(rexlib::operation_cast<rexlib::em::standardize_background_operation>(op), outs, ins,
					   d)
				? backend_priority::optimal
				: backend_priority::unsupported;
		}
		catch (...)
		{
			return backend_priority::unsupported;
		}
	}
	std::shared_ptr<rexlib::program> build(const rexlib::operation &op, descriptors outs, descriptors ins,
		rexlib::command_queue &, rexlib::program_cache *) const override
	{
		rexlib_b200_standardization d{};
		if (!plan_standardize(rexlib::operation_cast<rexlib::em::standardize_background_operation>(op), outs, ins, d))
			throw std::invalid_argument("rexlib_b200: the standardization cannot run on the b200 backend");
		return std::make_shared<standardize_program>(d, outs[0].get_layout().get_offset() * 4,
			ins[0].get_layout().get_offset() * 4, ins[1].get_layout().get_offset() * 8);
	}
};

const rexlib::program_builder_registration<standardize_builder> register_standardize(get_program_builder_registry());

} // anonymous namespace

} // namespace plugin
} // namespace rexlib_b200
