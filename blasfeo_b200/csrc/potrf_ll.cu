// FP64 potrf_l for instances whose lower triangle does not fit in shared
// memory: one CTA per instance, left-looking 16-column panels with the
// updates on the FP64 tensor cores (chol_ll.cuh).
#include "chol_ll.cuh"
#include "kernels.cuh"

namespace {

// 128 threads, POTRF_LL_MINB resident CTAs per SM: the serial panel chain of
// one instance is hidden behind the other instances on the SM, so occupancy
// pays for a few spilled registers; POTRF_LL_FR fragment rows per warp in the
// panel update
#ifndef POTRF_LL_MINB
#define POTRF_LL_MINB 6
#endif
#ifndef POTRF_LL_FR
#define POTRF_LL_FR 1
#endif
constexpr int LL_NT = 128;

__global__ void __launch_bounds__(LL_NT, POTRF_LL_MINB)
    k_potrf_ll(SizeArg sz, MatArg<double> C, MatArg<double> D, int *info, int min_n, int max_n) {
	extern __shared__ __align__(16) double ll_smem[];
	__shared__ int s_bad;
	const int b = blockIdx.x;
	const int n = sz.M(b);
	if (n <= min_n || n > max_n) return;
	if (threadIdx.x == 0) s_bad = 0;
	__syncthreads();
	chol_ll<LL_NT, POTRF_LL_FR>(C.get(b), D.get(b), n, ll_smem, &s_bad);
	if (info && threadIdx.x == 0) info[b] = s_bad;
}

}  // namespace

namespace bf {

// largest n the blocked global-memory kernel takes (its panel lives in shared memory)
int dpotrf_ll_max_n() {
	static int lim = 0;
	if (!lim)
		for (int v = 16; v <= 8192; v += 16)
			if (ll_smem_bytes(v) <= max_smem_optin()) lim = v;
	return lim;
}

// instances with min_n < n <= max_m
int dpotrf_ll_launch(int batch, SizeArg sz, int min_n, int max_m, MatArg<double> C, MatArg<double> D, int *info,
                     cudaStream_t s) {
	if (batch <= 0 || max_m <= min_n) return BLASFEO_B200_OK;
	if (max_m > dpotrf_ll_max_n()) return BLASFEO_B200_ENOTSUP;
	const size_t smem = ll_smem_bytes(max_m);
	bf::smem_optin(k_potrf_ll, smem);
	k_potrf_ll<<<batch, LL_NT, smem, s>>>(sz, C, D, info, min_n, max_m);
	return check_launch();
}

}  // namespace bf
