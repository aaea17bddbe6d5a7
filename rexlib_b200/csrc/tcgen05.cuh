// Blackwell (sm_100a) primitives in inline PTX: mbarriers with bounded
// waits, TMA tiled loads (no multicast: one CTA, this GPU's memory), the
// tcgen05 tensor-core MMA with its accumulator in tensor memory (TMEM),
// TMEM allocation and loads, and the shared-memory matrix descriptors.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace rexlib_b200
{
namespace sm100
{

__device__ __forceinline__ uint32_t smem_address(const void *p)
{
	return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbarrier_init(uint64_t *bar, uint32_t count)
{
	asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_address(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_barrier_init()
{
	asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbarrier_arrive(uint64_t *bar)
{
	asm volatile("{\n\t.reg .b64 state;\n\tmbarrier.arrive.shared::cta.b64 state, [%0];\n\t}" ::"r"(smem_address(bar))
				 : "memory");
}

__device__ __forceinline__ void mbarrier_expect_tx(uint64_t *bar, uint32_t bytes)
{
	asm volatile("{\n\t.reg .b64 state;\n\tmbarrier.arrive.expect_tx.shared::cta.b64 state, [%0], %1;\n\t}" ::"r"(
					 smem_address(bar)),
		"r"(bytes)
				 : "memory");
}

__device__ __forceinline__ uint64_t global_timer_ns()
{
	uint64_t t;
	asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
	return t;
}

// True once the phase of `parity` has completed; never waits.
__device__ __forceinline__ bool mbarrier_test(uint64_t *bar, uint32_t parity)
{
	uint32_t done = 0;
	asm volatile("{\n\t.reg .pred p;\n\tmbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, "
				 "p;\n\t}"
				 : "=r"(done)
				 : "r"(smem_address(bar)), "r"(parity)
				 : "memory");
	return done != 0;
}

constexpr uint64_t default_wait_ns = 2000000000ull;

// One potentially blocking test of the phase of `parity`: the thread may be
// suspended (issuing nothing) until the phase completes or about
// `suspend_ns` pass. True once the phase has completed.
__device__ __forceinline__ bool mbarrier_try_wait(uint32_t bar_address, uint32_t parity, uint32_t suspend_ns)
{
	uint32_t done = 0;
	asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\tselp.u32 %0, 1, 0, "
				 "p;\n\t}"
				 : "=r"(done)
				 : "r"(bar_address), "r"(parity), "r"(suspend_ns)
				 : "memory");
	return done != 0;
}

// Waits for the phase of `parity` to complete, for at most `budget_ns` of
// wall time (two seconds by default; a budget under a microsecond tests the
// barrier once). The waiting thread is suspended between tests rather than
// spinning, so that it leaves the issue slots to the warps doing the work.
// False when the budget ran out: the caller records the failure and leaves
// instead of waiting forever.
__device__ __forceinline__ bool mbarrier_wait(uint64_t *bar, uint32_t parity, uint64_t budget_ns = default_wait_ns)
{
	if (budget_ns < 1000)
		return mbarrier_test(bar, parity);
	constexpr uint32_t suspend_ns = 20000;
	const uint32_t a = smem_address(bar);
	if (mbarrier_try_wait(a, parity, suspend_ns))
		return true;
	const uint64_t start = global_timer_ns();
	for (;;)
	{
		if (mbarrier_try_wait(a, parity, suspend_ns))
			return true;
		if (global_timer_ns() - start > budget_ns)
			return false;
	}
}

// A TMA tiled load of a 4D box into shared memory, completing `bytes` on
// the mbarrier. The innermost coordinate must start on a 16-byte boundary.
__device__ __forceinline__ void tma_load_4d(void *dst, const void *tensor_map, uint64_t *bar, int c0, int c1, int c2,
	int c3)
{
	asm volatile("cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, "
				 "%4, %5}], [%6];" ::"r"(smem_address(dst)),
		"l"(tensor_map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_address(bar))
				 : "memory");
}

__device__ __forceinline__ void tma_load_5d(void *dst, const void *tensor_map, uint64_t *bar, int c0, int c1, int c2,
	int c3, int c4)
{
	asm volatile("cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, "
				 "%4, %5, %6}], [%7];" ::"r"(smem_address(dst)),
		"l"(tensor_map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(smem_address(bar))
				 : "memory");
}

__device__ __forceinline__ void tma_load_3d(void *dst, const void *tensor_map, uint64_t *bar, int c0, int c1, int c2)
{
	asm volatile("cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, "
				 "%4}], [%5];" ::"r"(smem_address(dst)),
		"l"(tensor_map), "r"(c0), "r"(c1), "r"(c2), "r"(smem_address(bar))
				 : "memory");
}

__device__ __forceinline__ void prefetch_tensor_map(const void *tensor_map)
{
	asm volatile("prefetch.tensormap [%0];" ::"l"(tensor_map) : "memory");
}

// TMEM: `columns` (a power of two, 32 to 512) allocated by one whole warp;
// the address lands in *slot (shared memory).
__device__ __forceinline__ void tmem_allocate(uint32_t *slot, uint32_t columns)
{
	asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_address(slot)),
		"r"(columns)
				 : "memory");
	asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_free(uint32_t address, uint32_t columns)
{
	asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(address), "r"(columns) : "memory");
}

__device__ __forceinline__ void tcgen05_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tcgen05_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }

// D (TMEM, FP32) = A * B^T (+ D when accumulate): A and B from shared
// memory through their descriptors, BF16 or F16 operands of one type.
__device__ __forceinline__ void mma_f16(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
	uint32_t accumulate)
{
	asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\ttcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, "
				 "p;\n\t}" ::"r"(d_tmem),
		"l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate)
				 : "memory");
}

// Arrives on the mbarrier once every tcgen05 operation this thread issued
// before has completed.
__device__ __forceinline__ void mma_commit(uint64_t *bar)
{
	asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_address(bar))
				 : "memory");
}

// 16 consecutive FP32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_load16(uint32_t address, float (&v)[16])
{
	uint32_t r[16];
	asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
				 "%14, %15}, [%16];"
				 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
				 "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
				 : "r"(address));
	asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
	for (int i = 0; i < 16; ++i)
		v[i] = __uint_as_float(r[i]);
}

// 16 consecutive FP32 columns of this thread's TMEM lane into raw registers,
// without waiting: several loads in flight, then one tmem_wait_loads()
// before the registers are read.
__device__ __forceinline__ void tmem_load16_async(uint32_t address, uint32_t (&r)[16])
{
	asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
				 "%14, %15}, [%16];"
				 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
				 "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
				 : "r"(address));
}

__device__ __forceinline__ void tmem_wait_loads() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// After tmem_wait_loads(): ties the registers of one load to a point after
// the wait, so that no use of them is scheduled before it.
__device__ __forceinline__ void tmem_loaded(uint32_t (&r)[16])
{
	asm volatile(""
				 : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]),
				 "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]), "+r"(r[15]));
}

// Shared-memory matrix descriptor of a K-major operand tile whose rows (M
// or N) are `row_bytes` (32, 64 or 128) of K, swizzled to that width, rows
// 8 at a time in atoms of 8 x row_bytes: the start address (16-byte units),
// the stride between atoms of 8 rows, the SM100 descriptor version and the
// swizzle mode (128B: 2, 64B: 4, 32B: 6).
__device__ __forceinline__ uint64_t kmajor_descriptor(uint32_t smem_addr, uint32_t row_bytes)
{
	const uint32_t layout = row_bytes == 128 ? 2u : row_bytes == 64 ? 4u : 6u;
	uint64_t d = 0;
	d |= static_cast<uint64_t>((smem_addr >> 4) & 0x3FFFu);
	d |= static_cast<uint64_t>(1u) << 16;                               // leading byte offset: unused when swizzled
	d |= static_cast<uint64_t>(((8u * row_bytes) >> 4) & 0x3FFFu) << 32; // stride byte offset: one atom of 8 rows
	d |= static_cast<uint64_t>(1u) << 46;                               // version (SM100)
	d |= static_cast<uint64_t>(layout) << 61;
	return d;
}

// Shared-memory matrix descriptor of a K-major operand without swizzle (the
// interleaved canonical layout): core matrices of 8 rows x 16 bytes, each
// 128 contiguous bytes (row r of a core matrix at +16 r); `k_stride` bytes
// between core matrices adjacent in K, `row_group_stride` bytes between
// groups of 8 rows. Any 16-byte aligned start is valid, so a tile may start
// at any row of a larger block.
__device__ __forceinline__ uint64_t interleaved_descriptor(uint32_t smem_addr, uint32_t k_stride,
	uint32_t row_group_stride)
{
	uint64_t d = 0;
	d |= static_cast<uint64_t>((smem_addr >> 4) & 0x3FFFu);
	d |= static_cast<uint64_t>((k_stride >> 4) & 0x3FFFu) << 16;         // leading (K) byte offset
	d |= static_cast<uint64_t>((row_group_stride >> 4) & 0x3FFFu) << 32; // stride (M or N) byte offset
	d |= static_cast<uint64_t>(1u) << 46;                               // version (SM100); swizzle 0: none
	return d;
}

// 16 bytes from global into shared memory, asynchronously; `bytes` 0 writes
// zeros and reads nothing.
__device__ __forceinline__ void copy16_async(uint32_t smem_dst, const void *src, uint32_t bytes)
{
	asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_dst), "l"(src), "r"(bytes) : "memory");
}

__device__ __forceinline__ void copy_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }

// Waits until at most `N` of this thread's committed copy groups are pending.
template <int N>
__device__ __forceinline__ void copy_async_wait()
{
	asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Orders this thread's generic-proxy shared-memory writes (completed copies
// included) before later async-proxy reads (the tensor cores').
__device__ __forceinline__ void fence_proxy_async_shared()
{
	asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B,
// both K-major, M x N.
__host__ __device__ constexpr uint32_t bf16_idesc(uint32_t m, uint32_t n)
{
	return (1u << 4) | (1u << 7) | (1u << 10) | ((n >> 3) << 17) | ((m >> 4) << 24);
}

} // namespace sm100
} // namespace rexlib_b200
