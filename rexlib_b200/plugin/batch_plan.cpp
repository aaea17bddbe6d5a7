// Batch planning of the insertions (batch_plan.hpp).
#include "batch_plan.hpp"

namespace rexlib_b200
{
namespace plugin
{

namespace
{

// The extent of `axis` of the broadcast shape of rank `rank` in an operand
// of batch extents `extents` (1 where the operand has no such axis).
std::size_t aligned_extent(const std::vector<std::size_t> &extents, std::size_t rank, std::size_t axis)
{
	const std::size_t missing = rank - extents.size();
	return axis < missing ? 1 : extents[axis - missing];
}

// One stride for the flattened index over `axes` (outermost first): every
// non-trivial axis, inner to outer, must step by the stride times the
// product of the inner extents. A broadcast axis (operand extent 1) steps
// by 0, which only a stride of 0 allows.
bool flatten(const batch_plan &plan, const std::vector<int> &axes, const std::vector<std::size_t> &extents,
	const std::vector<std::ptrdiff_t> &strides, std::int64_t core, std::int64_t &stride)
{
	const std::size_t rank = plan.shape.size();
	const std::size_t missing = rank - extents.size();
	bool first = true;
	std::int64_t unit = 0;
	std::int64_t inner = 1;
	for (auto it = axes.rbegin(); it != axes.rend(); ++it)
	{
		const std::size_t axis = static_cast<std::size_t>(*it);
		const std::size_t extent = plan.shape[axis];
		if (extent == 1)
			continue;
		const bool broadcast = aligned_extent(extents, rank, axis) == 1;
		const std::int64_t step = broadcast ? 0 : static_cast<std::int64_t>(strides[axis - missing]);
		if (first)
		{
			unit = step;
			first = false;
		}
		else if (step != unit * inner)
		{
			return false;
		}
		inner *= static_cast<std::int64_t>(extent);
	}
	if (unit % core != 0)
		return false;
	stride = unit / core;
	return true;
}

} // anonymous namespace

bool plan_batches(const std::vector<std::size_t> &accumulators,
	const std::vector<std::vector<std::size_t>> &inputs, batch_plan &plan, std::string &why)
{
	std::size_t rank = accumulators.size();
	for (const auto &e : inputs)
		rank = e.size() > rank ? e.size() : rank;
	plan = batch_plan{};
	plan.shape.assign(rank, 1);
	auto merge = [&](const std::vector<std::size_t> &e) {
		for (std::size_t axis = 0; axis < rank; ++axis)
		{
			const std::size_t x = aligned_extent(e, rank, axis);
			std::size_t &s = plan.shape[axis];
			if (x == s || x == 1)
				continue;
			if (s != 1)
			{
				why = "the batch axes of the operands do not broadcast";
				return false;
			}
			s = x;
		}
		return true;
	};
	if (!merge(accumulators))
		return false;
	for (const auto &e : inputs)
		if (!merge(e))
			return false;
	for (std::size_t axis = 0; axis < rank; ++axis)
	{
		if (aligned_extent(accumulators, rank, axis) != 1)
		{
			plan.kept.push_back(static_cast<int>(axis));
			plan.volumes *= static_cast<std::int64_t>(plan.shape[axis]);
		}
		else
		{
			plan.reduced.push_back(static_cast<int>(axis));
			plan.particles *= static_cast<std::int64_t>(plan.shape[axis]);
		}
	}
	return true;
}

bool batch_strides(const batch_plan &plan, const std::vector<std::size_t> &extents,
	const std::vector<std::ptrdiff_t> &strides, std::int64_t core_elements, std::int64_t &volume_stride,
	std::int64_t &particle_stride)
{
	if (extents.size() > plan.shape.size() || strides.size() != extents.size() || core_elements <= 0)
		return false;
	volume_stride = particle_stride = 0;
	return flatten(plan, plan.kept, extents, strides, core_elements, volume_stride) &&
		flatten(plan, plan.reduced, extents, strides, core_elements, particle_stride) && volume_stride >= 0 &&
		particle_stride >= 0;
}

bool core_is_contiguous(const std::vector<std::size_t> &extents, const std::vector<std::ptrdiff_t> &strides,
	std::size_t core_rank)
{
	if (extents.size() < core_rank || strides.size() != extents.size())
		return false;
	std::ptrdiff_t expected = 1;
	for (std::size_t i = 0; i < core_rank; ++i)
	{
		const std::size_t axis = extents.size() - 1 - i;
		if (extents[axis] != 1 && strides[axis] != expected)
			return false;
		expected *= static_cast<std::ptrdiff_t>(extents[axis]);
	}
	return true;
}

} // namespace plugin
} // namespace rexlib_b200
