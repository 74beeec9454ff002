// Self-check of the bounded mbarrier wait that every bulk-copy kernel uses
// (chain.cu, riccati.cu, posv_tc.cu): one warp arms an mbarrier for 16 bytes
// of bulk-copy data and issues no copy, so the wait can only run out.  The
// kernel then reports the timeout status the other kernels report (-3) and
// returns; nothing is in flight, so nothing can land after the block exits.
#include "common.cuh"
#include "tma.cuh"

namespace {

__global__ void k_wait_timeout_check(uint32_t limit, int *out) {
	__shared__ __align__(8) uint64_t bar;
	if (threadIdx.x == 0) {
		mbar_init(&bar, 1);
		mbar_fence_init();
	}
	__syncwarp();
	if (threadIdx.x == 0) mbar_arrive_expect_tx(&bar, 16);  // 16 bytes that never come
	__syncwarp();
	const bool ok = __all_sync(0xffffffffu, mbar_wait(&bar, 0u, limit));
	if (threadIdx.x == 0) out[0] = ok ? 0 : -3;
}

}  // namespace

extern "C" int blasfeo_b200_check_wait_timeout(int *status, void *stream) {
	if (!status) return BLASFEO_B200_EINVAL;
	k_wait_timeout_check<<<1, 32, 0, (cudaStream_t)stream>>>(bf::wait_limit(), status);
	return bf::check_launch();
}
