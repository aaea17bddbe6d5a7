// The 2x2x2 stride-2 transposed convolution of the U-Net prior on the
// tcgen05 tensor cores, through the convolution's box kernel with one tap:
//   out[2 v + s][o] = bias[o] + sum_i x[v][i] w[s][o][i]
// for sub-positions s = 4 sz + 2 sy + sx, x channels-last BF16 of extents
// (D, H, W) with cin channels a voxel, w BF16 [8][cout][cin], out BF16 of
// extents (2D, 2H, 2W) with cout channels a voxel. The GEMM's columns are
// (sub-position, channel) pairs, at most 256 a launch; the epilogue writes
// each group of 16 to its output voxel. Launches on `stream`; throws the
// library's status error on an argument it refuses. `error` (device,
// optional) receives a nonzero code if a wait inside the kernel ran out.
#pragma once

#include <cuda_runtime.h>

namespace rexlib_b200
{

void conv3d_transposed2(const void *x, int cin, int D, int H, int W, const void *weights, const float *bias, int cout,
	void *out, int *error, cudaStream_t stream);

} // namespace rexlib_b200
