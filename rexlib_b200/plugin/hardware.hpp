// The B200 device as rexlib's hardware abstraction sees it: a device
// backend named "b200" (one device per CUDA device), memory resources for
// device memory and pinned host memory, their allocators and buffers, and a
// command queue over one CUDA stream whose command tokens are CUDA events.
//
// Interfaces implemented: include/rexlib/core/hardware/device_backend.hpp,
// device.hpp, memory_resource.hpp, memory_allocator.hpp, buffer.hpp,
// command_queue.hpp (submit, :55) and command_timeline.hpp. The queue keeps
// every submitted command, and so its buffers, alive until the command's
// event has completed, which is what plugins/cuda/src/hardware/
// cuda_command_queue.cpp:195-215 does with its record_use.
#pragma once

#include <rexlib/core/hardware/buffer.hpp>
#include <rexlib/core/hardware/command.hpp>
#include <rexlib/core/hardware/command_queue.hpp>
#include <rexlib/core/hardware/command_timeline.hpp>
#include <rexlib/core/hardware/command_token.hpp>
#include <rexlib/core/hardware/device.hpp>
#include <rexlib/core/hardware/device_backend.hpp>
#include <rexlib/core/hardware/memory_allocator.hpp>
#include <rexlib/core/hardware/memory_resource.hpp>
#include <rexlib/core/hardware/program.hpp>
#include <rexlib/core/hardware/program_scratch_requirement.hpp>

#include <cuda_runtime_api.h>

#include <cstddef>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

namespace rexlib_b200
{
namespace plugin
{

// Throws std::runtime_error naming `what` when `status` is not cudaSuccess.
void check(cudaError_t status, const char *what);

// Makes `device` current for the scope and restores the previous device.
class device_scope
{
public:
	explicit device_scope(int device);
	~device_scope();
	device_scope(const device_scope &) = delete;
	device_scope &operator=(const device_scope &) = delete;

private:
	int m_previous = -1;
	bool m_switched = false;
};

// Memory of one CUDA device (device_local) or pinned host memory that the
// device reaches by DMA (host_staging, host accessible).
class memory_resource final : public rexlib::memory_resource
{
public:
	memory_resource(int device, rexlib::memory_resource_kind kind) noexcept;
	rexlib::memory_resource_kind get_kind() const noexcept override;
	std::shared_ptr<rexlib::memory_allocator> create_allocator() const override;
	int device() const noexcept { return m_device; }
	bool on_host() const noexcept { return m_kind == rexlib::memory_resource_kind::host_staging; }

private:
	int m_device;
	rexlib::memory_resource_kind m_kind;
};

// Is the memory resource one of this backend's device memories?
const memory_resource *device_memory_of(const rexlib::memory_resource *resource) noexcept;

class buffer final : public rexlib::buffer
{
public:
	buffer(const memory_resource &resource, void *data, std::size_t size) noexcept;
	~buffer() override;
	void *get_host_ptr() noexcept override;
	const void *get_host_ptr() const noexcept override;
	std::size_t get_size() const noexcept override;
	const rexlib::memory_resource &get_memory_resource() const noexcept override;
	void *data() const noexcept { return m_data; }

private:
	const memory_resource &m_resource;
	void *m_data;
	std::size_t m_size;
};

// The address of a buffer's bytes for a kernel or a copy: the device
// address of this backend's buffers, the host address of host-accessible
// ones; null when neither.
const void *address_of(const rexlib::buffer &b) noexcept;
void *address_of(rexlib::buffer &b) noexcept;

// cudaMalloc / cudaMallocHost per buffer; the memory is ready when the call
// returns, so `pending` stays empty. Freeing synchronizes the device (what
// cudaFree does), so a buffer is never reused under a kernel still reading
// it.
class allocator final : public rexlib::memory_allocator
{
public:
	explicit allocator(const memory_resource &resource) noexcept;
	const rexlib::memory_resource &get_memory_resource() const noexcept override;
	std::size_t get_max_alignment() const noexcept override;
	std::shared_ptr<rexlib::buffer> allocate(std::size_t size, std::size_t alignment, rexlib::command_queue *queue_hint,
		rexlib::command_token &pending) override;

private:
	const memory_resource &m_resource;
};

// Command tokens of one queue: token i is the CUDA event recorded after
// command i. Events of completed commands are retired in order; a retired
// id counts as complete.
class timeline final : public rexlib::command_timeline
{
public:
	explicit timeline(int device) noexcept;
	~timeline() override;
	std::size_t record(cudaStream_t stream);
	void wait(std::size_t id) const override;
	bool is_complete(std::size_t id) const override;
	// Makes `stream` wait for command `id` on the device (no host wait).
	void make_wait(cudaStream_t stream, std::size_t id) const;

private:
	int m_device;
	mutable std::mutex m_mutex;
	// ids m_first .. m_first + size - 1; shared so that a wait keeps its
	// event alive while another thread retires it.
	mutable std::deque<std::shared_ptr<CUevent_st>> m_events;
	mutable std::size_t m_first = 0;
	void retire_locked() const;
};

// A program of this backend: launch() enqueues its work on the queue's
// stream, with the buffers bound to the command.
class program : public rexlib::program
{
public:
	rexlib::span<const rexlib::program_scratch_requirement> get_scratch_requirements() const override;
	virtual void launch(rexlib::span<const std::shared_ptr<rexlib::buffer>> outputs,
		rexlib::span<const std::shared_ptr<const rexlib::buffer>> inputs,
		rexlib::span<const std::shared_ptr<rexlib::buffer>> scratch, cudaStream_t stream) const = 0;

protected:
	std::vector<rexlib::program_scratch_requirement> m_scratch;
};

class command_queue final : public rexlib::command_queue
{
public:
	explicit command_queue(int device);
	~command_queue() override;
	rexlib::command_token submit(rexlib::command cmd) override;
	int device() const noexcept { return m_device; }
	cudaStream_t stream() const noexcept { return m_stream; }

private:
	int m_device;
	cudaStream_t m_stream = nullptr;
	std::shared_ptr<timeline> m_timeline;
	std::mutex m_mutex;
	std::deque<std::pair<std::size_t, rexlib::command>> m_in_flight;
};

class device final : public rexlib::device
{
public:
	explicit device(int id);
	const rexlib::memory_resource &get_memory_resource(rexlib::memory_resource_affinity affinity) const override;
	std::shared_ptr<rexlib::command_queue> create_command_queue() const override;

private:
	int m_id;
	memory_resource m_device_memory;
	memory_resource m_pinned_memory;
};

class device_backend final : public rexlib::device_backend
{
public:
	std::string get_name() const override;
	rexlib::version get_version() const override;
	void enumerate_devices(std::vector<std::size_t> &ids) const override;
	bool get_device_properties(std::size_t id, rexlib::device_properties &properties) const override;
	std::shared_ptr<rexlib::device> create_device(std::size_t id) const override;
};

} // namespace plugin
} // namespace rexlib_b200
