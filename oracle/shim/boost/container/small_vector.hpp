// Stand-in for boost::container::small_vector, used only to build the
// reference CPU path as test infrastructure: a std::vector with the same
// template shape (the inline capacity is ignored).
#pragma once
#include <cstddef>
#include <vector>

namespace boost
{
namespace container
{

template <typename T, std::size_t N, typename Allocator = void, typename Options = void>
class small_vector : public std::vector<T>
{
public:
	using std::vector<T>::vector;
	small_vector() = default;
};

} // namespace container
} // namespace boost
