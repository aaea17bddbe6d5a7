// Shared device helpers and the error plumbing of the C-ABI layer.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <stdexcept>
#include <string>

#include "rexlib_b200.h"

namespace rexlib_b200
{

// An error carrying the status the C entry point returns.
class status_error : public std::runtime_error
{
public:
	status_error(rexlib_b200_status status, const std::string &message)
		: std::runtime_error(message), m_status(status)
	{
	}
	rexlib_b200_status status() const noexcept { return m_status; }

private:
	rexlib_b200_status m_status;
};

[[noreturn]] inline void fail(rexlib_b200_status status, const std::string &message)
{
	throw status_error(status, message);
}

inline void require(bool condition, const std::string &message)
{
	if (!condition)
		fail(REXLIB_B200_INVALID_ARGUMENT, message);
}

// sin(x) for |x| up to about 1e5: Cody-Waite reduction by 2 pi with a
// three-part constant (2 pi = 6.28125 + 1.93530717e-3 + 1.02531317e-11;
// the first part has 8 significant bits, so k * part stays exact), then the
// hardware sine on [-pi, pi] (absolute error below 2^-21).
__device__ __forceinline__ float sin_reduced(float x)
{
	const float k = rintf(x * 0.159154937f);
	float r = fmaf(-k, 6.28125f, x);
	r = fmaf(-k, 1.93530717e-3f, r);
	r = fmaf(-k, 1.02531317e-11f, r);
	return __sinf(r);
}

inline void check_cuda(cudaError_t error, const char *what)
{
	if (error != cudaSuccess)
		fail(REXLIB_B200_CUDA_ERROR, std::string(what) + ": " + cudaGetErrorString(error));
}

// Runs `body`, turning exceptions into a status and the thread's message.
void set_last_error(const std::string &message);

template <typename Body>
int32_t guarded(Body &&body) noexcept
{
	try
	{
		set_last_error("");
		body();
		return REXLIB_B200_OK;
	}
	catch (const status_error &e)
	{
		set_last_error(e.what());
		return e.status();
	}
	catch (const std::bad_alloc &)
	{
		set_last_error("out of host memory");
		return REXLIB_B200_CUDA_ERROR;
	}
	catch (const std::exception &e)
	{
		set_last_error(e.what());
		return REXLIB_B200_INVALID_ARGUMENT;
	}
	catch (...)
	{
		set_last_error("unknown error");
		return REXLIB_B200_INVALID_ARGUMENT;
	}
}

inline cudaStream_t as_stream(void *stream) { return static_cast<cudaStream_t>(stream); }

// Round-to-nearest float and double operations that the compiler may not
// contract into fused multiply-adds: the CPU backend's results are reproduced
// operation for operation.
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double fmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double fadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double fsub(double a, double b) { return __dsub_rn(a, b); }

constexpr double pi = 3.141592653589793238462643383279502884;

} // namespace rexlib_b200
