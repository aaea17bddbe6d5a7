// Stand-in for boost/functional/hash.hpp, used only to build the reference
// CPU path as test infrastructure: hash_value via std::hash and the usual
// golden-ratio combine.
#pragma once
#include <cstddef>
#include <functional>

namespace boost
{

template <typename T>
std::size_t hash_value(const T &value)
{
	return std::hash<T>()(value);
}

template <typename T>
void hash_combine(std::size_t &seed, const T &value)
{
	seed ^= hash_value(value) + 0x9e3779b97f4a7c15ULL + (seed << 6) + (seed >> 2);
}

inline void hash_combine(std::size_t &seed, std::size_t value)
{
	seed ^= value + 0x9e3779b97f4a7c15ULL + (seed << 6) + (seed >> 2);
}

} // namespace boost
