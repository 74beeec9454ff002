// Bulk-copy (TMA) and mbarrier helpers, inline PTX for sm_100a.
//
// Only untiled bulk copies from this GPU's own global memory into the
// issuing CTA's shared memory are used (no cluster multicast).  Every wait on
// an mbarrier is bounded: after `limit` polls (a kernel argument, set per
// process by blasfeo_b200_set_wait_limit, default BF_WAIT_LIMIT, about one
// second) it gives up and reports a timeout to the caller, which records
// info = -3 and returns.  Before returning, a kernel whose copies may still be
// in flight waits for them once more with the fixed BF_DRAIN_LIMIT (about four
// seconds), so that no copy lands in the shared memory of an exited block
// unless it is stuck for that long too: the drain is best effort, bounded like
// every other wait.
#pragma once
#include <stdint.h>

#define BF_WAIT_LIMIT (1u << 24)
#define BF_DRAIN_LIMIT (1u << 26)

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
	asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
	asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

// global -> shared bulk copy completing on bar (dst, src 16-byte aligned, bytes % 16 == 0)
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
	asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
	                 smem_u32(dst)),
	             "l"(src), "r"(bytes), "r"(smem_u32(bar))
	             : "memory");
}

// order earlier generic-proxy accesses of shared memory before later async-proxy (bulk copy) writes
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
	uint32_t ok;
	asm volatile(
	    "{\n\t.reg .pred p;\n\t"
	    "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
	    "selp.u32 %0, 1, 0, p;\n\t}"
	    : "=r"(ok)
	    : "r"(smem_u32(bar)), "r"(parity)
	    : "memory");
	return ok != 0;
}

// bounded wait for phase `parity` of bar; false after `limit` polls
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, uint32_t limit) {
	for (uint32_t it = 0; it < limit; it++) {
		if (mbar_try_wait(bar, parity)) return true;
		if (it > 64) __nanosleep(64);
	}
	return false;
}
