// PTX helpers shared by the table-driven Legendre kernels: mbarriers with
// bounded waits and plain (non-multicast) bulk copies into shared memory.
#pragma once

#include <cstdint>

namespace shtb_ptx {

// every mbarrier wait of the table kernels gives up after this long
constexpr uint64_t WAIT_NS = 1000000000ull;

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
	asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ uint64_t global_ns()
{
	uint64_t t;
	asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
	return t;
}

__device__ __forceinline__ bool mbar_try(uint32_t a, uint32_t parity)
{
	uint32_t done;
	asm volatile("{\n\t.reg .pred p;\n\t"
	             "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
	             "selp.u32 %0, 1, 0, p;\n\t}"
	             : "=r"(done) : "r"(a), "r"(parity) : "memory");
	return done != 0;
}

// bounded wait for the phase of parity `parity`; false when the time limit
// passes (the CTA's abort flag is then set) or another thread set the flag
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, volatile int* abort_flag)
{
	const uint32_t a = smem_u32(bar);
	const uint64_t t0 = global_ns();
	for (int it = 0;; it++) {
		if (mbar_try(a, parity)) return true;
		if ((it & 255) == 255) {
			if (*abort_flag) return false;
			if (global_ns() - t0 > WAIT_NS) { *abort_flag = 1; return false; }
		}
	}
}

// the same wait without the flag (clean-up), bounded
__device__ __forceinline__ void mbar_wait_quiet(uint64_t* bar, uint32_t parity)
{
	const uint32_t a = smem_u32(bar);
	const uint64_t t0 = global_ns();
	for (int it = 0;; it++) {
		if (mbar_try(a, parity)) return;
		if ((it & 255) == 255 && global_ns() - t0 > WAIT_NS) return;
	}
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes)
{
	asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar)
{
	asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" :: "r"(smem_u32(bar)) : "memory");
}

// plain bulk copy global -> this CTA's shared memory (16-byte aligned, size a
// multiple of 16), completion counted in bytes on the mbarrier
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint64_t* bar)
{
	asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
	             :: "r"(dst), "l"(src), "r"(bytes), "r"(smem_u32(bar)) : "memory");
}

} // namespace shtb_ptx
