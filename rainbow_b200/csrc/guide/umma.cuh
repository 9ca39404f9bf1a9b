// Blackwell (sm_100a) building blocks for the guiding network kernels:
// shared-memory matrix descriptors, the tcgen05 BF16 MMA with FP32 accumulators
// in tensor memory, TMEM allocation and loads, mbarriers with time-bounded waits
// and the bulk (non-tensor) global -> shared copy. Everything is inline PTX.
//
// Operand layout ("canonical, no swizzle"): a matrix is stored as 8-row x
// 16-byte core matrices (8 rows of 8 bf16, each row 16 contiguous bytes).
//  - K-major operand (rows = M or N, 8 consecutive K elements per core row):
//    the descriptor's LBO is the byte distance between the two core matrices
//    that make up K = 16, SBO the distance between consecutive 8-row groups.
//  - MN-major operand (8 consecutive M/N elements per core row, 8 K rows per
//    core matrix): SBO is the distance between consecutive 8-element M/N
//    groups, LBO the distance between consecutive 8-row K groups.
// No load in this file uses cluster multicast.
#pragma once

#include <cstdint>

namespace rb {
namespace guide {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
	return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// ------------------------------------------------------------ descriptors
// Shared-memory matrix descriptor: start address, leading / stride byte
// offsets (all >> 4), descriptor version 1 (bits 46-47), base offset 0,
// no swizzle (bits 61-63 = 0).
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
	return static_cast<uint64_t>((saddr >> 4) & 0x3FFFu)
		| (static_cast<uint64_t>((lbo_bytes >> 4) & 0x3FFFu) << 16)
		| (static_cast<uint64_t>((sbo_bytes >> 4) & 0x3FFFu) << 32)
		| (1ull << 46);
}

// Instruction descriptor of kind::f16 with BF16 A and B and an FP32
// accumulator: c_format (bits 4-5) = F32, a_format (7-9) = b_format (10-12) =
// BF16, a_major (15) / b_major (16) = 0 for K-major, 1 for MN-major,
// N >> 3 at bits 17-22, M >> 4 at bits 24-28.
__host__ __device__ constexpr uint32_t idesc_bf16(uint32_t m, uint32_t n, bool a_mn, bool b_mn) {
	return (1u << 4) | (1u << 7) | (1u << 10) | ((a_mn ? 1u : 0u) << 15) | ((b_mn ? 1u : 0u) << 16)
		| ((n >> 3) << 17) | ((m >> 4) << 24);
}

// ------------------------------------------------------------ fences
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void named_barrier(uint32_t id, uint32_t threads) {
	asm volatile("bar.sync %0, %1;" :: "r"(id), "r"(threads) : "memory");
}

// ------------------------------------------------------------ mbarrier
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
	asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
	asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
	uint32_t ok;
	asm volatile(
		"{\n\t.reg .pred p;\n\t"
		"mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
		"selp.u32 %0, 1, 0, p;\n\t}"
		: "=r"(ok) : "r"(smem_u32(bar)), "r"(parity) : "memory");
	return ok != 0u;
}

__device__ __forceinline__ uint64_t global_timer_ns() {
	uint64_t t;
	asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
	return t;
}

// Waits for phase `parity` of `bar` to complete. Gives up after `limit_ns`
// nanoseconds of wall time (each try_wait returns by itself after a
// hardware-defined suspend time) and returns false then.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint64_t limit_ns) {
	if (mbar_try_wait(bar, parity)) return true;
	const uint64_t t0 = global_timer_ns();
	for (;;) {
		if (mbar_try_wait(bar, parity)) return true;
		if (global_timer_ns() - t0 > limit_ns) return false;
	}
}

// ------------------------------------------------------------ bulk copy
// Global -> shared copy by the bulk-copy engine, completing on `bar` with a
// transaction count of `bytes`. Both addresses 16-byte aligned, bytes a
// multiple of 16. Plain (non-multicast) form.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
	asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
		:: "r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar)) : "memory");
}

// ------------------------------------------------------------ TMEM
// Allocation / release by one full warp. ncols: power of two in [32, 512].
__device__ __forceinline__ void tmem_alloc(uint32_t* dst_smem, uint32_t ncols) {
	asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
		:: "r"(smem_u32(dst_smem)), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
	asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
	asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(taddr), "r"(ncols) : "memory");
}

// D[tmem] (+)= A[smem] * B[smem]^T for one K = 16 step, issued by one thread.
__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t accumulate) {
	asm volatile(
		"{\n\t.reg .pred p;\n\t"
		"setp.ne.b32 p, %4, 0;\n\t"
		"tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
		:: "r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate) : "memory");
}

// Arrives on `bar` once all MMAs issued so far by this thread have completed.
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
	asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
		:: "r"(smem_u32(bar)) : "memory");
}

// 16 consecutive FP32 columns of this thread's TMEM lane (32x32b shape: warp
// w of a warpgroup reads lanes 32w..32w+31, one lane per thread). The load and
// its wait are one statement so no register is read before it has arrived.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
	uint32_t r[16];
	asm volatile(
		"tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n\t"
		"tcgen05.wait::ld.sync.aligned;"
		: "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
		  "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
		: "r"(taddr) : "memory");
#pragma unroll
	for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

// 32 columns: two loads, one wait.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float* v) {
	uint32_t r[32];
	asm volatile(
		"tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%32];\n\t"
		"tcgen05.ld.sync.aligned.32x32b.x16.b32 {%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%33];\n\t"
		"tcgen05.wait::ld.sync.aligned;"
		: "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
		  "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
		  "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
		  "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
		: "r"(taddr), "r"(taddr + 16u) : "memory");
#pragma unroll
	for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}

} // namespace guide
} // namespace rb
