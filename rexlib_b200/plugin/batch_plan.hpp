// Batch planning of the insertions, on the host, in C++: which batch axes
// the accumulators keep (their own axes, extent above 1) and which the
// insertion sums over (every other broadcast axis), and each operand's
// (volume, particle) strides in whole cores over that plan. It is the step
// slice_insertion_layout_plan takes on the CPU
// (src/backends/cpu/plans/slice_insertion_layout_plan.cpp:81-185); the
// kernels take a plan as V accumulators receiving P slices each, an operand
// element (v, p) starting v * volume + p * particle cores in.
//
// No rexlib or CUDA type appears here, so the plan is tested on its own.
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

namespace rexlib_b200
{
namespace plugin
{

struct batch_plan
{
	std::vector<std::size_t> shape; // the broadcast batch shape
	std::vector<int> kept;          // axes of `shape` the accumulators own
	std::vector<int> reduced;       // axes summed over
	std::int64_t volumes = 1;       // product of the kept extents
	std::int64_t particles = 1;     // product of the reduced extents
};

// Plans from the accumulators' batch extents and every input's batch
// extents (right-aligned, numpy broadcasting). False, with the reason, when
// they do not broadcast.
bool plan_batches(const std::vector<std::size_t> &accumulators,
	const std::vector<std::vector<std::size_t>> &inputs, batch_plan &plan, std::string &why);

// The (volume, particle) strides, in cores of `core_elements` elements, of
// an operand whose batch axes have `extents` and `strides` (in elements;
// right-aligned to the plan, a missing or unit axis broadcasting). False
// when the kept axes, or the reduced ones, do not step through the operand
// by one stride each (a layout the kernels cannot address), or when a
// stride is not a whole number of cores.
bool batch_strides(const batch_plan &plan, const std::vector<std::size_t> &extents,
	const std::vector<std::ptrdiff_t> &strides, std::int64_t core_elements, std::int64_t &volume_stride,
	std::int64_t &particle_stride);

// Are the last `core_rank` axes of a layout row-major contiguous?
bool core_is_contiguous(const std::vector<std::size_t> &extents, const std::vector<std::ptrdiff_t> &strides,
	std::size_t core_rank);

} // namespace plugin
} // namespace rexlib_b200
