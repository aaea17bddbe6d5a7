// Oracle for the elementwise divide of complex arrays (test infrastructure
// only). The reference's CPU kernel (src/backends/cpu/builders/arithmetic/
// divide_program_builder.cpp:19-22) stores load(x) / load(y), and load/store
// are the identity for std::complex<float> and std::complex<double>
// (src/backends/cpu/load_store.hpp): the quotient is std::complex's
// operator/, which g++ lowers to its runtime's complex division. This file
// performs that same division, compiled by the same compiler with the
// reference's floating-point flags (no fast-math), so it is the reference's
// arithmetic rather than a restatement of it.
#include <complex>
#include <cstdint>

extern "C" void oracle_divide_complex64(std::complex<float> *out, const std::complex<float> *x, int64_t x_count,
	const std::complex<float> *y, int64_t y_count, int64_t count)
{
	for (int64_t i = 0; i < count; ++i)
		out[i] = x[x_count == 1 ? 0 : i] / y[y_count == 1 ? 0 : i];
}

extern "C" void oracle_divide_complex128(std::complex<double> *out, const std::complex<double> *x,
	int64_t x_count, const std::complex<double> *y, int64_t y_count, int64_t count)
{
	for (int64_t i = 0; i < count; ++i)
		out[i] = x[x_count == 1 ? 0 : i] / y[y_count == 1 ? 0 : i];
}
