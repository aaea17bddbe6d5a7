// The B200 backend's device, memory, queue and token objects (hardware.hpp).
#include "hardware.hpp"

#include <rexlib/core/hardware/device_properties.hpp>
#include <rexlib/core/hardware/device_type.hpp>
#include <rexlib/core/hardware/memory_resource_affinity.hpp>
#include <rexlib/core/version.hpp>

#include <new>
#include <stdexcept>

namespace rexlib_b200
{
namespace plugin
{

void check(cudaError_t status, const char *what)
{
	if (status != cudaSuccess)
		throw std::runtime_error(std::string("rexlib_b200: ") + what + ": " + cudaGetErrorString(status));
}

device_scope::device_scope(int device)
{
	check(cudaGetDevice(&m_previous), "current device");
	if (m_previous != device)
	{
		check(cudaSetDevice(device), "set device");
		m_switched = true;
	}
}

device_scope::~device_scope()
{
	if (m_switched)
		cudaSetDevice(m_previous);
}

// ---------------------------------------------------------------------------
// Memory

memory_resource::memory_resource(int device, rexlib::memory_resource_kind kind) noexcept : m_device(device), m_kind(kind)
{
}

rexlib::memory_resource_kind memory_resource::get_kind() const noexcept { return m_kind; }

std::shared_ptr<rexlib::memory_allocator> memory_resource::create_allocator() const
{
	return std::make_shared<allocator>(*this);
}

const memory_resource *device_memory_of(const rexlib::memory_resource *resource) noexcept
{
	const auto *ours = dynamic_cast<const memory_resource *>(resource);
	return ours != nullptr && !ours->on_host() ? ours : nullptr;
}

buffer::buffer(const memory_resource &resource, void *data, std::size_t size) noexcept
	: m_resource(resource), m_data(data), m_size(size)
{
}

buffer::~buffer()
{
	if (m_data == nullptr)
		return;
	int previous = -1;
	cudaGetDevice(&previous);
	cudaSetDevice(m_resource.device());
	if (m_resource.on_host())
		cudaFreeHost(m_data);
	else
		cudaFree(m_data);
	if (previous >= 0)
		cudaSetDevice(previous);
}

void *buffer::get_host_ptr() noexcept { return m_resource.on_host() ? m_data : nullptr; }
const void *buffer::get_host_ptr() const noexcept { return m_resource.on_host() ? m_data : nullptr; }
std::size_t buffer::get_size() const noexcept { return m_size; }
const rexlib::memory_resource &buffer::get_memory_resource() const noexcept { return m_resource; }

const void *address_of(const rexlib::buffer &b) noexcept
{
	if (const auto *ours = dynamic_cast<const buffer *>(&b))
		return ours->data();
	return b.get_host_ptr();
}

void *address_of(rexlib::buffer &b) noexcept
{
	if (auto *ours = dynamic_cast<buffer *>(&b))
		return ours->data();
	return b.get_host_ptr();
}

allocator::allocator(const memory_resource &resource) noexcept : m_resource(resource) {}

const rexlib::memory_resource &allocator::get_memory_resource() const noexcept { return m_resource; }

// cudaMalloc returns 256-byte aligned memory; pinned host pages are 4 KiB.
std::size_t allocator::get_max_alignment() const noexcept { return 256; }

std::shared_ptr<rexlib::buffer> allocator::allocate(std::size_t size, std::size_t alignment, rexlib::command_queue *,
	rexlib::command_token &)
{
	if (alignment > get_max_alignment() || (alignment & (alignment - 1)) != 0)
		throw std::invalid_argument("rexlib_b200: alignments are powers of two up to 256 bytes");
	device_scope scope(m_resource.device());
	void *data = nullptr;
	const std::size_t bytes = size > 0 ? size : 1;
	const cudaError_t status = m_resource.on_host() ? cudaMallocHost(&data, bytes) : cudaMalloc(&data, bytes);
	if (status == cudaErrorMemoryAllocation)
	{
		cudaGetLastError();
		throw std::bad_alloc();
	}
	check(status, m_resource.on_host() ? "pinned host allocation" : "device allocation");
	return std::make_shared<buffer>(m_resource, data, size);
}

// ---------------------------------------------------------------------------
// Tokens and queues

timeline::timeline(int device) noexcept : m_device(device) {}

timeline::~timeline()
{
	int previous = -1;
	cudaGetDevice(&previous);
	cudaSetDevice(m_device);
	m_events.clear();
	if (previous >= 0)
		cudaSetDevice(previous);
}

void timeline::retire_locked() const
{
	while (!m_events.empty() && cudaEventQuery(m_events.front().get()) == cudaSuccess)
	{
		m_events.pop_front();
		++m_first;
	}
}

std::size_t timeline::record(cudaStream_t stream)
{
	cudaEvent_t raw = nullptr;
	check(cudaEventCreateWithFlags(&raw, cudaEventDisableTiming), "event creation");
	std::shared_ptr<CUevent_st> e(raw, [](cudaEvent_t x) { cudaEventDestroy(x); });
	check(cudaEventRecord(e.get(), stream), "event record");
	std::lock_guard<std::mutex> lock(m_mutex);
	retire_locked();
	m_events.push_back(std::move(e));
	return m_first + m_events.size() - 1;
}

void timeline::wait(std::size_t id) const
{
	std::shared_ptr<CUevent_st> e;
	{
		std::lock_guard<std::mutex> lock(m_mutex);
		if (id < m_first)
			return;
		if (id - m_first >= m_events.size())
			throw std::out_of_range("rexlib_b200: unknown command token");
		e = m_events[id - m_first];
	}
	check(cudaEventSynchronize(e.get()), "command wait");
}

bool timeline::is_complete(std::size_t id) const
{
	std::lock_guard<std::mutex> lock(m_mutex);
	retire_locked();
	return id < m_first;
}

void timeline::make_wait(cudaStream_t stream, std::size_t id) const
{
	std::lock_guard<std::mutex> lock(m_mutex);
	if (id < m_first)
		return;
	if (id - m_first >= m_events.size())
		throw std::out_of_range("rexlib_b200: unknown command token");
	check(cudaStreamWaitEvent(stream, m_events[id - m_first].get(), 0), "stream wait");
}

rexlib::span<const rexlib::program_scratch_requirement> program::get_scratch_requirements() const
{
	return rexlib::span<const rexlib::program_scratch_requirement>(m_scratch.data(), m_scratch.size());
}

command_queue::command_queue(int device) : m_device(device), m_timeline(std::make_shared<timeline>(device))
{
	device_scope scope(device);
	check(cudaStreamCreateWithFlags(&m_stream, cudaStreamNonBlocking), "stream creation");
}

command_queue::~command_queue()
{
	int previous = -1;
	cudaGetDevice(&previous);
	cudaSetDevice(m_device);
	cudaStreamSynchronize(m_stream);
	m_in_flight.clear();
	cudaStreamDestroy(m_stream);
	if (previous >= 0)
		cudaSetDevice(previous);
}

rexlib::command_token command_queue::submit(rexlib::command cmd)
{
	const auto *prog = dynamic_cast<const program *>(cmd.get_program().get());
	if (prog == nullptr)
		throw std::invalid_argument("rexlib_b200: the b200 queue runs the programs of the b200 backend only");
	device_scope scope(m_device);
	std::lock_guard<std::mutex> lock(m_mutex);
	for (const auto &dependency : cmd.get_dependencies())
	{
		if (dependency.is_empty())
			continue;
		const auto *other = dynamic_cast<const timeline *>(dependency.get_timeline().get());
		if (other == m_timeline.get())
			continue; // stream order
		if (other != nullptr)
			other->make_wait(m_stream, dependency.get_id());
		else
			dependency.wait();
	}
	prog->launch(cmd.get_outputs(), cmd.get_inputs(), cmd.get_scratch(), m_stream);
	const cudaError_t launched = cudaGetLastError();
	if (launched != cudaSuccess)
	{
		cudaStreamSynchronize(m_stream);
		check(launched, "program launch");
	}
	const std::size_t id = m_timeline->record(m_stream);
	// Release the commands (and their buffers) whose work has completed.
	while (!m_in_flight.empty() && m_timeline->is_complete(m_in_flight.front().first))
		m_in_flight.pop_front();
	m_in_flight.emplace_back(id, std::move(cmd));
	return rexlib::command_token(m_timeline, id);
}

// ---------------------------------------------------------------------------
// Devices

device::device(int id)
	: m_id(id)
	, m_device_memory(id, rexlib::memory_resource_kind::device_local)
	, m_pinned_memory(id, rexlib::memory_resource_kind::host_staging)
{
}

const rexlib::memory_resource &device::get_memory_resource(rexlib::memory_resource_affinity affinity) const
{
	switch (affinity)
	{
	case rexlib::memory_resource_affinity::device:
		return m_device_memory;
	case rexlib::memory_resource_affinity::host:
		return m_pinned_memory;
	default:
		throw std::invalid_argument("rexlib_b200: unknown memory affinity");
	}
}

std::shared_ptr<rexlib::command_queue> device::create_command_queue() const
{
	return std::make_shared<command_queue>(m_id);
}

std::string device_backend::get_name() const { return "b200"; }

rexlib::version device_backend::get_version() const { return rexlib::version(0, 2, 0); }

// Every CUDA device of compute capability 10.0 (sm_100a code only); none
// when the runtime finds no device.
void device_backend::enumerate_devices(std::vector<std::size_t> &ids) const
{
	ids.clear();
	int count = 0;
	if (cudaGetDeviceCount(&count) != cudaSuccess)
	{
		cudaGetLastError();
		return;
	}
	for (int d = 0; d < count; ++d)
	{
		cudaDeviceProp p{};
		if (cudaGetDeviceProperties(&p, d) == cudaSuccess && p.major == 10 && p.minor == 0)
			ids.push_back(static_cast<std::size_t>(d));
	}
}

bool device_backend::get_device_properties(std::size_t id, rexlib::device_properties &properties) const
{
	std::vector<std::size_t> ids;
	enumerate_devices(ids);
	bool found = false;
	for (std::size_t i : ids)
		found = found || i == id;
	if (!found)
		return false;
	cudaDeviceProp p{};
	check(cudaGetDeviceProperties(&p, static_cast<int>(id)), "device properties");
	properties.set_type(rexlib::device_type::gpu);
	properties.set_name(p.name);
	properties.set_total_memory_bytes(p.totalGlobalMem);
	properties.set_optimal_data_alignment(256);
	char location[32] = {};
	if (cudaDeviceGetPCIBusId(location, sizeof(location), static_cast<int>(id)) == cudaSuccess)
		properties.set_physical_location(location);
	return true;
}

std::shared_ptr<rexlib::device> device_backend::create_device(std::size_t id) const
{
	rexlib::device_properties properties;
	if (!get_device_properties(id, properties))
		throw std::invalid_argument("rexlib_b200: no B200 (compute capability 10.0) device numbered " +
			std::to_string(id));
	return std::make_shared<device>(static_cast<int>(id));
}

} // namespace plugin
} // namespace rexlib_b200
