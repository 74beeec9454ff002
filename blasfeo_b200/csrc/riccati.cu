// Batched Riccati recursion (LQR backward factorization), one warp per
// problem, the whole recursion in one persistent kernel.
//
// Per problem (examples/example_d_riccati_recursion.c:115-143,
// d_back_ric_trf_libstr):
//   L_N = chol(Q_N)                                   (blasfeo_dpotrf_l)
//   for k = N-1 .. 0:
//     W   = BAbt_k * Lxx_{k+1}                        (blasfeo_dtrmm_rlnn)
//     L_k = chol(RSQ_k + W W^T)                       (blasfeo_dsyrk_dpotrf_ln)
// with BAbt_k = [B_k^T; A_k^T] ((nu+nx) x nx), RSQ_k = [[R, S],[S^T, Q]]
// ((nu+nx) x (nu+nx), lower triangle used) and Lxx_{k+1} the lower-right
// nx x nx block of L_{k+1} (the whole L_N for k = N-1).  Stage N stores Q_N
// in the top-left nx x nx block of its (nu+nx)^2 slot and L_N there too, as
// the reference example does with nu_N = 0.
//
// The factor of stage k+1 never leaves the chip: it is kept in shared memory
// (FP64) and consumed by stage k.  Each stage's BAbt_k and RSQ_k are bulk
// copied (TMA) into a double buffer so the next stage's inputs arrive while
// the current stage computes; L_k (lower triangle) and its inverse diagonal
// are the only writes.  nu + nx <= 16: lane i owns row i; the 16x16 factor
// runs in FP64 registers (DiagCol, chol.cuh).  T = float gives the
// single-precision variant (FP32 storage and FP32 trmm/syrk products; the
// pivots and rank-1 updates of the diagonal factor stay FP64).
#include "chol.cuh"
#include "common.cuh"
#include "tma.cuh"

namespace {

constexpr int RM = 16;
constexpr int RIC_WARPS = 8;
constexpr int R_LD = 17;

template <typename T>
struct RicLayout {
	int ba_el, rsq_el, buf_el, warp_bytes;
};

template <typename T>
__host__ __device__ inline RicLayout<T> ric_layout(int nx) {
	RicLayout<T> l;
	const int cnx = (nx + 3) / 4 * 4;
	l.ba_el = RM * cnx;
	l.rsq_el = RM * RM;
	l.buf_el = l.ba_el + l.rsq_el;
	int bytes = 2 * l.buf_el * (int)sizeof(T);
	bytes = (bytes + 15) / 16 * 16;
	bytes += 2 * RM * R_LD * 8 + RM * 8 + 16 + 16;
	l.warp_bytes = (bytes + 127) / 128 * 128;
	return l;
}

__device__ __forceinline__ int pm_idx(int i, int j, int cn) { return (i & ~3) * cn + 4 * j + (i & 3); }

template <typename T>
__global__ void __launch_bounds__(RIC_WARPS * 32) k_ric_trf(int batch, int N, int nx, int nu, const T *__restrict__ pBA,
                                                           long long sba, const T *__restrict__ pRSQ, long long srsq,
                                                           T *pL, T *pLd, long long sl, int *info, uint32_t wait_limit) {
	extern __shared__ __align__(128) unsigned char smem[];
	const RicLayout<T> lay = ric_layout<T>(nx);
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	unsigned char *base = smem + (size_t)warp * lay.warp_bytes;
	T *buf[2] = {(T *)base, (T *)base + lay.buf_el};
	double *Lp = (double *)(base + ((2 * lay.buf_el * (int)sizeof(T) + 15) / 16 * 16));
	double *Wm = Lp + RM * R_LD;
	double *dv = Wm + RM * R_LD;
	uint64_t *bar = (uint64_t *)(dv + RM);
	int *bad = (int *)(bar + 2);
	const int M = nu + nx;
	const int cnx = (nx + 3) / 4 * 4;
	const uint32_t ba_bytes = (uint32_t)(lay.ba_el * sizeof(T)), rsq_bytes = (uint32_t)(lay.rsq_el * sizeof(T));

	const long long gw = (long long)blockIdx.x * RIC_WARPS + warp;
	const long long nw = (long long)gridDim.x * RIC_WARPS;
	if (lane == 0) {
		mbar_init(&bar[0], 1);
		mbar_init(&bar[1], 1);
		mbar_fence_init();
	}
	__syncwarp();
	uint32_t phase[2] = {0u, 0u};
	// stage k of problem b into buffer slot (stage N has no BAbt)
	auto issue = [&](long long b, int k, int slot) {
		T *d = buf[slot];
		const bool has_ba = k < N;
		mbar_arrive_expect_tx(&bar[slot], rsq_bytes + (has_ba ? ba_bytes : 0u));
		if (has_ba) bulk_g2s(d, pBA + sba * (b * N + k), ba_bytes, &bar[slot]);
		bulk_g2s(d + lay.ba_el, pRSQ + srsq * (b * (N + 1) + k), rsq_bytes, &bar[slot]);
	};
	int slot = 0;
	if (gw < batch && lane == 0) issue(gw, N, 0);
	for (long long b = gw; b < batch; b += nw) {
		if (lane == 0) *bad = 0;
		for (int k = N; k >= 0; k--, slot ^= 1) {
			// prefetch the next stage (or the first stage of the next problem)
			if (lane == 0) {
				fence_proxy_async_smem();
				if (k > 0)
					issue(b, k - 1, slot ^ 1);
				else if (b + nw < batch)
					issue(b + nw, N, slot ^ 1);
			}
			if (!mbar_wait(&bar[slot], phase[slot], wait_limit)) {
				if (lane == 0 && info) info[b] = -3;
				// drain both slots' copies before the warp leaves
				mbar_wait(&bar[slot], phase[slot], BF_DRAIN_LIMIT);
				mbar_wait(&bar[slot ^ 1], phase[slot ^ 1], BF_DRAIN_LIMIT);
				return;
			}
			phase[slot] ^= 1u;
			const T *BA = buf[slot];
			const T *RSQ = buf[slot] + lay.ba_el;
			const int m = (k == N) ? nx : M;    // size of this stage's factor
			const int off = (k + 1 == N) ? 0 : nu;  // Lxx offset inside L_{k+1}
			double r[RM];
			if (k == N) {
#pragma unroll
				for (int l = 0; l < RM; l++)
					r[l] = (lane < m && l <= lane) ? (l < m ? (double)RSQ[pm_idx(lane, l, RM)] : 0.0) : (l == lane ? 1.0 : 0.0);
			} else {
				// W = BAbt_k * Lxx_{k+1}: lane i owns row i (j < nx), products in T
				T w[RM];
#pragma unroll
				for (int j = 0; j < RM; j++) {
					T s = T(0);
					if (lane < M && j < nx) {
#pragma unroll
						for (int l = j; l < RM; l++)
							if (l < nx) s = fma(BA[pm_idx(lane, l, cnx)], (T)Lp[(off + l) * R_LD + off + j], s);
					}
					w[j] = s;
				}
				if (lane < RM) {
#pragma unroll
					for (int j = 0; j < RM; j++) Wm[lane * R_LD + j] = w[j];
				}
				__syncwarp();
				// S = RSQ_k + W W^T (lower), row i in FP64 registers
#pragma unroll
				for (int j = 0; j < RM; j++) {
					T s;
					if (lane < M && j <= lane) {
						s = RSQ[pm_idx(lane, j, RM)];
#pragma unroll
						for (int l = 0; l < RM; l++)
							if (l < nx) s = fma(w[l], (T)Wm[j * R_LD + l], s);
					} else {
						s = (j == lane) ? T(1) : T(0);
					}
					r[j] = (double)s;
				}
			}
			DiagCol<0>::run(r, lane, m, 0, dv, bad);
			__syncwarp();
			// keep L_k on chip for stage k-1, write its lower triangle and inverse diagonal
			if (lane < RM) {
#pragma unroll
				for (int l = 0; l < RM; l++) Lp[lane * R_LD + l] = (l <= lane) ? r[l] : 0.0;
			}
			T *gL = pL + sl * (b * (N + 1) + k);
			if (lane < m) {
#pragma unroll
				for (int l = 0; l < RM; l++)
					if (l <= lane && l < m) gL[pm_idx(lane, l, RM)] = (T)r[l];
				(pLd + sl * (b * (N + 1) + k))[lane] = (T)dv[lane];
			}
			if (lane == 0 && *bad && info && info[b] == 0) info[b] = (N - k) * RM + *bad;
			if (lane == 0) *bad = 0;
			__syncwarp();
		}
	}
}

template <typename T, typename BT>
int ric_run(int batch, int N, int nx, int nu, BT *sBA, BT *sRSQ, BT *sL, int *info, void *stream) {
	if (batch < 0 || N < 0 || nx < 1 || nu < 0 || !sRSQ || !sL || (N > 0 && !sBA)) return BLASFEO_B200_EINVAL;
	if (batch == 0) return BLASFEO_B200_OK;
	const int M = nu + nx;
	if (M > RM) return BLASFEO_B200_ENOTSUP;
	if (sRSQ->m != RM || sRSQ->n != RM || sL->m != RM || sL->n != RM) return BLASFEO_B200_ENOTSUP;
	if ((long long)sRSQ->batch < (long long)batch * (N + 1) || (long long)sL->batch < (long long)batch * (N + 1))
		return BLASFEO_B200_EINVAL;
	if (N > 0 && (sBA->m != RM || sBA->n != nx || (long long)sBA->batch < (long long)batch * N))
		return BLASFEO_B200_EINVAL;
	if (((uintptr_t)sRSQ->pA & 15) || ((sRSQ->stride * sizeof(T)) & 15)) return BLASFEO_B200_EINVAL;
	if (N > 0 && (((uintptr_t)sBA->pA & 15) || ((sBA->stride * sizeof(T)) & 15))) return BLASFEO_B200_EINVAL;
	if (info) cudaMemsetAsync(info, 0, sizeof(int) * batch, (cudaStream_t)stream);
	sL->use_dA = 0;
	const RicLayout<T> lay = ric_layout<T>(nx);
	const size_t smem = (size_t)lay.warp_bytes * RIC_WARPS;
	cudaFuncSetAttribute(k_ric_trf<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
	int per_sm = 0;
	cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_ric_trf<T>, RIC_WARPS * 32, smem);
	if (per_sm < 1) per_sm = 1;
	long long grid = (long long)bf::num_sms() * per_sm;
	const long long need = (batch + RIC_WARPS - 1) / RIC_WARPS;
	if (grid > need) grid = need;
	k_ric_trf<T><<<(unsigned)grid, RIC_WARPS * 32, smem, (cudaStream_t)stream>>>(
	    batch, N, nx, nu, N > 0 ? sBA->pA : nullptr, N > 0 ? sBA->stride : 0, sRSQ->pA, sRSQ->stride, sL->pA, sL->dA,
	    sL->stride, info, bf::wait_limit());
	return bf::check_launch();
}

}  // namespace

extern "C" {

int blasfeo_dric_trf_batch(int batch, int N, int nx, int nu, struct blasfeo_dmat_batch *sBAbt,
                           struct blasfeo_dmat_batch *sRSQ, struct blasfeo_dmat_batch *sL, int *info, void *stream) {
	return ric_run<double>(batch, N, nx, nu, sBAbt, sRSQ, sL, info, stream);
}

int blasfeo_sric_trf_batch(int batch, int N, int nx, int nu, struct blasfeo_smat_batch *sBAbt,
                           struct blasfeo_smat_batch *sRSQ, struct blasfeo_smat_batch *sL, int *info, void *stream) {
	return ric_run<float>(batch, N, nx, nu, sBAbt, sRSQ, sL, info, stream);
}

}  // extern "C"
