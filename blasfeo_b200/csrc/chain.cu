// Fused uniform-batch chain, one warp per instance (m = 16):
//   S = A A^T + shift*I          (blasfeo_dsyrk_ln + blasfeo_ddiare)
//   L = chol(S)                  (blasfeo_dpotrf_l, inverse diagonal kept)
//   X = R L^{-T}                 (blasfeo_dtrsm_rltn)
//   D = C - X G^T                (blasfeo_dgemm_nt)
// The composition mirrors the reference calls it replaces
// (blasfeo_hp_pm/d_blas3_lib4.c:5400, :4123, :727; d_lapack_lib4.c:918).
//
// The chain is HBM-bound (about 1.5 flop per byte), so the design is about
// bytes: each warp streams its instances' inputs (A, R, C, G: 10 KB for
// k = 32, contiguous panel-major slabs) into shared memory with bulk copies
// (TMA) on an mbarrier; every intermediate (S, L, X) stays on chip; L (lower
// triangle), X and D are written once.  Persistent grid: each warp walks the
// batch with a stride of the total warp count.  Memory-level parallelism
// comes from 16 resident warps per SM, each with one instance in flight
// (CHAIN_NBUF = 2 double-buffers instead, with fewer warps; measured slower:
// 0.89 ms vs 0.67 ms for 100k instances).
#include "chol.cuh"
#include "common.cuh"
#include "tma.cuh"

#ifndef CHAIN_WARPS
#define CHAIN_WARPS 8
#endif
#ifndef CHAIN_NBUF
#define CHAIN_NBUF 1
#endif

namespace {

constexpr int CM = 16;                 // chain size m
constexpr int CH_WARPS = CHAIN_WARPS;   // warps per CTA
constexpr int W_LD = 17;               // row stride of the FP64 work matrix

struct ChainLayout {
	int a_dbl;     // doubles of the A slab (16 x cnA)
	int buf_dbl;   // A + R + C + G
	int warp_bytes;
};

__host__ __device__ inline ChainLayout chain_layout(int k) {
	ChainLayout l;
	const int cna = (k + 3) / 4 * 4;
	l.a_dbl = CM * cna;
	l.buf_dbl = l.a_dbl + 3 * CM * CM;
	// input buffer(s), the work matrix, reciprocal pivots, mbarriers
	l.warp_bytes = CHAIN_NBUF * l.buf_dbl * 8 + CM * W_LD * 8 + CM * 8 + 16 + 16;
	l.warp_bytes = (l.warp_bytes + 127) / 128 * 128;
	return l;
}

__device__ __forceinline__ int pm_idx16(int i, int j) { return (i & ~3) * CM + 4 * j + (i & 3); }

__global__ void __launch_bounds__(CH_WARPS * 32) k_chain16(int batch, int k, double shift, const double *__restrict__ pA,
                                                           long long sa, const double *__restrict__ pR, long long sr,
                                                           const double *__restrict__ pC, long long sc,
                                                           const double *__restrict__ pG, long long sg, double *pL,
                                                           double *pLd, long long sl, double *pX, long long sx,
                                                           double *pD, long long sd, int *info) {
	extern __shared__ __align__(128) unsigned char smem[];
	const ChainLayout lay = chain_layout(k);
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	unsigned char *base = smem + (size_t)warp * lay.warp_bytes;
	double *buf[2] = {(double *)base, (double *)base + (CHAIN_NBUF - 1) * lay.buf_dbl};
	double *W = (double *)base + CHAIN_NBUF * lay.buf_dbl;
	double *dv = W + CM * W_LD;
	uint64_t *bar = (uint64_t *)(dv + CM);
	int *bad = (int *)(bar + 2);
	const int cna = (k + 3) / 4 * 4;
	const uint32_t a_bytes = (uint32_t)lay.a_dbl * 8, m_bytes = CM * CM * 8;
	const uint32_t tx = a_bytes + 3 * m_bytes;

	const long long gw = (long long)blockIdx.x * CH_WARPS + warp;
	const long long nw = (long long)gridDim.x * CH_WARPS;
	if (lane == 0) {
		mbar_init(&bar[0], 1);
		mbar_init(&bar[1], 1);
		mbar_fence_init();
	}
	__syncwarp();
	auto issue = [&](long long b, int slot) {
		double *d = buf[slot];
		mbar_arrive_expect_tx(&bar[slot], tx);
		bulk_g2s(d, pA + sa * b, a_bytes, &bar[slot]);
		bulk_g2s(d + lay.a_dbl, pR + sr * b, m_bytes, &bar[slot]);
		bulk_g2s(d + lay.a_dbl + CM * CM, pC + sc * b, m_bytes, &bar[slot]);
		bulk_g2s(d + lay.a_dbl + 2 * CM * CM, pG + sg * b, m_bytes, &bar[slot]);
	};
	if (gw < batch && lane == 0) issue(gw, 0);
	uint32_t phase[2] = {0u, 0u};
	int slot = 0;
	for (long long b = gw; b < batch; b += nw, slot ^= (CHAIN_NBUF - 1)) {
		const long long nb = b + nw;
		if (CHAIN_NBUF == 1 && b != gw && lane == 0) {
			// single buffer: refill it for this instance (its last readers finished at the loop end)
			fence_proxy_async_smem();
			issue(b, slot);
		}
		if (CHAIN_NBUF == 2 && nb < batch && lane == 0) {
			// the other buffer was last read by generic loads (previous instance)
			fence_proxy_async_smem();
			issue(nb, slot ^ 1);
		}
		if (!mbar_wait(&bar[slot], phase[slot])) {
			if (lane == 0 && info) info[b] = -3;  // bulk copy did not complete in time
			mbar_wait(&bar[slot], phase[slot]);
			if (CHAIN_NBUF == 2 && nb < batch) mbar_wait(&bar[slot ^ 1], phase[slot ^ 1]);
			return;
		}
		phase[slot] ^= 1u;
		const double *A = buf[slot];
		double *R = buf[slot] + lay.a_dbl;
		double *Cm = R + CM * CM;
		const double *G = Cm + CM * CM;

		// 1. S = A A^T + shift I: lanes 0..19 own half 4x4 tiles (rows of tile ti, 2 columns of tile tj)
		if (lane < 20) {
			int ti, tj;
			tri_index(lane >> 1, ti, tj);
			const int q = lane & 1;
			double acc[8];
#pragma unroll
			for (int e = 0; e < 8; e++) acc[e] = 0.0;
			const double *ai = A + ti * 4 * cna, *aj = A + tj * 4 * cna + 2 * q;
			for (int kk = 0; kk < k; kk++) {
				const double2 x01 = *(const double2 *)(ai + 4 * kk), x23 = *(const double2 *)(ai + 4 * kk + 2);
				const double2 y = *(const double2 *)(aj + 4 * kk);
				acc[0] = fma(x01.x, y.x, acc[0]); acc[1] = fma(x01.y, y.x, acc[1]);
				acc[2] = fma(x23.x, y.x, acc[2]); acc[3] = fma(x23.y, y.x, acc[3]);
				acc[4] = fma(x01.x, y.y, acc[4]); acc[5] = fma(x01.y, y.y, acc[5]);
				acc[6] = fma(x23.x, y.y, acc[6]); acc[7] = fma(x23.y, y.y, acc[7]);
			}
#pragma unroll
			for (int c = 0; c < 2; c++)
#pragma unroll
				for (int r = 0; r < 4; r++) {
					const int i = 4 * ti + r, j = 4 * tj + 2 * q + c;
					W[i * W_LD + j] = acc[4 * c + r] + (i == j ? shift : 0.0);
				}
		}
		if (lane == 0) *bad = 0;
		__syncwarp();
		// 2. L = chol(S): lane i holds row i in FP64 registers
		{
			double r[CM];
#pragma unroll
			for (int l = 0; l < CM; l++) r[l] = (lane < CM && l <= lane) ? W[lane * W_LD + l] : (l == lane ? 1.0 : 0.0);
			DiagCol<0>::run(r, lane, CM, 0, dv, bad);
			if (lane < CM) {
#pragma unroll
				for (int l = 0; l < CM; l++) W[lane * W_LD + l] = (l <= lane) ? r[l] : 0.0;
			}
		}
		__syncwarp();
		// 3./4. X = R L^{-T} and D = C - X G^T, lane i owns row i
		if (lane < CM) {
			const int i = lane;
			double x[CM];
#pragma unroll
			for (int j = 0; j < CM; j++) {
				double s = R[pm_idx16(i, j)];
#pragma unroll
				for (int l = 0; l < j; l++) s = fma(-x[l], W[j * W_LD + l], s);
				x[j] = s * dv[j];
			}
#pragma unroll
			for (int j = 0; j < CM; j++) {
				double s = 0.0;
#pragma unroll
				for (int l = 0; l < CM; l++) s = fma(x[l], G[pm_idx16(j, l)], s);
				Cm[pm_idx16(i, j)] = Cm[pm_idx16(i, j)] - s;
			}
#pragma unroll
			for (int j = 0; j < CM; j++) R[pm_idx16(i, j)] = x[j];
		}
		__syncwarp();
		// 5. outputs: L lower triangle (and its inverse diagonal), X, D
		double *gL = pL + sl * b, *gX = pX + sx * b, *gD = pD + sd * b;
		for (int e = lane; e < CM * CM; e += 32) {
			const int j = (e & 63) >> 2, i = ((e >> 6) << 2) | (e & 3);
			if (j <= i) gL[e] = W[i * W_LD + j];
		}
		if (lane < CM) (pLd + sl * b)[lane] = dv[lane];
		for (int e = 2 * lane; e < CM * CM; e += 64) {
			*(double2 *)(gX + e) = *(const double2 *)(R + e);
			*(double2 *)(gD + e) = *(const double2 *)(Cm + e);
		}
		if (lane == 0 && info) info[b] = *bad;
		__syncwarp();
	}
}

}  // namespace

extern "C" {

int blasfeo_dsyrk_dpotrf_dtrsm_dgemm_batch(int batch, int m, int k, double shift, struct blasfeo_dmat_batch *sA,
                                           struct blasfeo_dmat_batch *sR, struct blasfeo_dmat_batch *sC,
                                           struct blasfeo_dmat_batch *sG, struct blasfeo_dmat_batch *sL,
                                           struct blasfeo_dmat_batch *sX, struct blasfeo_dmat_batch *sD, int *info,
                                           void *stream) {
	if (batch < 0 || !sA || !sR || !sC || !sG || !sL || !sX || !sD) return BLASFEO_B200_EINVAL;
	if (batch == 0) return BLASFEO_B200_OK;
	if (m != CM || k < 1 || k > 64) return BLASFEO_B200_ENOTSUP;
	const struct blasfeo_dmat_batch *mm[] = {sR, sC, sG, sL, sX, sD};
	for (auto p : mm)
		if (p->m != CM || p->n != CM || p->batch < batch) return BLASFEO_B200_EINVAL;
	if (sA->m != CM || sA->n < k || sA->batch < batch) return BLASFEO_B200_EINVAL;
	// bulk copies need 16-byte aligned sources
	const struct blasfeo_dmat_batch *all[] = {sA, sR, sC, sG};
	for (auto p : all)
		if (((uintptr_t)p->pA & 15) || ((p->stride * 8) & 15)) return BLASFEO_B200_EINVAL;
	if (sA->cn != (k + 3) / 4 * 4) return BLASFEO_B200_EINVAL;
	sL->use_dA = CM;
	sX->use_dA = 0;
	sD->use_dA = 0;
	const ChainLayout lay = chain_layout(k);
	const size_t smem = (size_t)lay.warp_bytes * CH_WARPS;
	cudaFuncSetAttribute(k_chain16, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
	int per_sm = 0;
	cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_chain16, CH_WARPS * 32, smem);
	if (per_sm < 1) per_sm = 1;
	long long grid = (long long)bf::num_sms() * per_sm;
	long long need = (batch + CH_WARPS - 1) / CH_WARPS;
	if (grid > need) grid = need;
	k_chain16<<<(unsigned)grid, CH_WARPS * 32, smem, (cudaStream_t)stream>>>(
	    batch, k, shift, sA->pA, sA->stride, sR->pA, sR->stride, sC->pA, sC->stride, sG->pA, sG->stride, sL->pA,
	    sL->dA, sL->stride, sX->pA, sX->stride, sD->pA, sD->stride, info);
	return bf::check_launch();
}

}  // extern "C"
