// Host helpers for TMA tensor maps of BF16 volumes: the driver's
// cuTensorMapEncodeTiled (reached through the runtime, so that the library
// links no libcuda), the swizzle matching a K-major operand row, and the
// device's SM count for persistent grids.
#pragma once

#include "common.cuh"

#include <cuda.h>

#include <mutex>
#include <string>

namespace rexlib_b200
{

using encode_tiled_t = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
	const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
	CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

inline encode_tiled_t encode_tiled()
{
	static encode_tiled_t fn = nullptr;
	static std::once_flag once;
	std::call_once(once, [] {
		void *p = nullptr;
		cudaDriverEntryPointQueryResult q{};
		if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) ==
				cudaSuccess &&
			q == cudaDriverEntryPointSuccess)
			fn = reinterpret_cast<encode_tiled_t>(p);
	});
	require(fn != nullptr, "the driver has no cuTensorMapEncodeTiled");
	return fn;
}

// The swizzle matching a K-major operand's row width; 0: none (the
// interleaved layout).
inline CUtensorMapSwizzle swizzle_of(int row_bytes)
{
	return row_bytes == 128 ? CU_TENSOR_MAP_SWIZZLE_128B
		: row_bytes == 64   ? CU_TENSOR_MAP_SWIZZLE_64B
		: row_bytes == 32   ? CU_TENSOR_MAP_SWIZZLE_32B
							: CU_TENSOR_MAP_SWIZZLE_NONE;
}

inline void encode(CUtensorMap *map, const void *base, int rank, const cuuint64_t *dims, const cuuint64_t *strides_bytes,
	const cuuint32_t *box, int row_bytes)
{
	cuuint32_t element_strides[5] = {1, 1, 1, 1, 1};
	const CUresult r = encode_tiled()(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, static_cast<cuuint32_t>(rank),
		const_cast<void *>(base), dims, strides_bytes, box, element_strides, CU_TENSOR_MAP_INTERLEAVE_NONE,
		swizzle_of(row_bytes), CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
	if (r != CUDA_SUCCESS)
		fail(REXLIB_B200_INVALID_ARGUMENT, "a tensor map of the convolution was refused (code " + std::to_string(r) + ")");
}

inline int sm_count()
{
	int device = 0, sms = 0;
	check_cuda(cudaGetDevice(&device), "device query");
	check_cuda(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "device query");
	return sms;
}

} // namespace rexlib_b200
