// Tile-major insertion (shared-memory accumulation). Placeholder: no shape
// is taken yet, so every call goes to the slice-parallel kernel.
#include "insertion.cuh"

namespace rexlib_b200
{

bool tiled_insertion_applies(const insertion_launch &, weight_kind, int) { return false; }

size_t tiled_insertion_workspace(const insertion_launch &, weight_kind, int) { return 0; }

void launch_insert_tiled(const insertion_launch &, weight_kind, int, void *, size_t, cudaStream_t)
{
	fail(REXLIB_B200_UNSUPPORTED, "tiled insertion unavailable");
}

} // namespace rexlib_b200
