// Fused uniform-batch chain, two instances per warp (m = 16; one per
// half-warp, lane i of a half owns row i):
//   S = A A^T + shift*I          (blasfeo_dsyrk_ln + blasfeo_ddiare)
//   L = chol(S)                  (blasfeo_dpotrf_l, inverse diagonal kept)
//   X = R L^{-T}                 (blasfeo_dtrsm_rltn)
//   D = C - X G^T                (blasfeo_dgemm_nt)
// The composition mirrors the reference calls it replaces
// (blasfeo_hp_pm/d_blas3_lib4.c:5400, :4123, :727; d_lapack_lib4.c:918).
//
// The chain is HBM-bound (about 1.5 flop per byte), so the design is about
// bytes and issue slots: each half-warp streams its instance's inputs (A, R,
// C, G: 10 KB for k = 32, contiguous panel-major slabs) into shared memory
// with bulk copies (TMA) on its own mbarrier; every intermediate (S, L, X)
// stays on chip; L (lower triangle), X and D are written once.  A 16 x 16
// instance has 16 rows, so a whole warp per instance would leave half of its
// lanes idle in every row-parallel phase; two instances per warp halve the
// instructions issued per instance.  Persistent grid: each warp walks the
// batch in pairs with a stride of the total warp count.
#include "chol.cuh"
#include "common.cuh"
#include "tma.cuh"

namespace {

constexpr int CM = 16;       // chain size m
constexpr int CH_WARPS = 4;  // warps per CTA (8 instances in flight)
constexpr int W_LD = 17;     // row stride of the FP64 work matrix

struct ChainLayout {
	int a_dbl;      // doubles of the A slab (16 x cnA)
	int buf_dbl;    // A + R + C + G
	int half_bytes; // one instance slot: inputs, work matrix, pivots, mbarrier, flags
};

__host__ __device__ inline ChainLayout chain_layout(int k) {
	ChainLayout l;
	const int cna = (k + 3) / 4 * 4;
	l.a_dbl = CM * cna;
	l.buf_dbl = l.a_dbl + 3 * CM * CM;
	l.half_bytes = l.buf_dbl * 8 + CM * W_LD * 8 + CM * 8 + 16 + 16;
	l.half_bytes = (l.half_bytes + 127) / 128 * 128;
	return l;
}

__device__ __forceinline__ int pm_idx16(int i, int j) { return (i & ~3) * CM + 4 * j + (i & 3); }

__global__ void __launch_bounds__(CH_WARPS * 32) k_chain16(int batch, int k, double shift, const double *__restrict__ pA,
                                                           long long sa, const double *__restrict__ pR, long long sr,
                                                           const double *__restrict__ pC, long long sc,
                                                           const double *__restrict__ pG, long long sg, double *pL,
                                                           double *pLd, long long sl, double *pX, long long sx,
                                                           double *pD, long long sd, int *info, uint32_t wait_limit) {
	extern __shared__ __align__(128) unsigned char smem[];
	const ChainLayout lay = chain_layout(k);
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	const int h = lane >> 4, li = lane & 15;
	unsigned char *base = smem + (size_t)(2 * warp + h) * lay.half_bytes;
	double *buf = (double *)base;
	double *W = buf + lay.buf_dbl;
	double *dv = W + CM * W_LD;
	uint64_t *bar = (uint64_t *)(dv + CM);
	int *bad = (int *)(bar + 1);
	const int cna = (k + 3) / 4 * 4;
	const uint32_t a_bytes = (uint32_t)lay.a_dbl * 8, m_bytes = CM * CM * 8;
	const uint32_t tx = a_bytes + 3 * m_bytes;

	const long long gw = (long long)blockIdx.x * CH_WARPS + warp;
	const long long nw = (long long)gridDim.x * CH_WARPS;
	const long long npairs = ((long long)batch + 1) / 2;
	if (li == 0) {
		mbar_init(bar, 1);
		mbar_fence_init();
	}
	__syncwarp();
	uint32_t phase = 0u;
	for (long long p = gw; p < npairs; p += nw) {  // warp-uniform loop
		const long long b = 2 * p + h;
		const bool act = b < batch;  // the second half of the last pair may be empty
		if (act && li == 0) {
			// (the slot's generic accesses by the previous pair were fenced at its end)
			mbar_arrive_expect_tx(bar, tx);
			bulk_g2s(buf, pA + sa * b, a_bytes, bar);
			bulk_g2s(buf + lay.a_dbl, pR + sr * b, m_bytes, bar);
			bulk_g2s(buf + lay.a_dbl + CM * CM, pC + sc * b, m_bytes, bar);
			bulk_g2s(buf + lay.a_dbl + 2 * CM * CM, pG + sg * b, m_bytes, bar);
		}
		bool ok = true;
		if (act) {
			ok = mbar_wait(bar, phase, wait_limit);
			phase ^= 1u;
		}
		if (!__all_sync(0xffffffffu, ok)) {  // a bulk copy did not complete in time
			if (act && li == 0 && info) info[b] = -3;
			// drain the copy still in flight (again bounded): best effort -- if
			// this wait also runs out, the block returns with the copy possibly
			// still landing in its shared memory; info = -3 reports the run
			if (act) mbar_wait(bar, phase ^ 1u, BF_DRAIN_LIMIT);
			return;
		}
		const double *A = buf;
		double *R = buf + lay.a_dbl;
		double *Cm = R + CM * CM;
		const double *G = Cm + CM * CM;

		// 1. S = A A^T + shift I: lanes 0..9 of the half own one 4x4 tile (ti, tj) of the lower part
		if (li < 10) {
			int ti, tj;
			tri_index(li, ti, tj);
			double acc[16];
#pragma unroll
			for (int e = 0; e < 16; e++) acc[e] = 0.0;
			const double *ai = A + ti * 4 * cna, *aj = A + tj * 4 * cna;
			for (int kk = 0; kk < k; kk++) {
				const double2 x01 = *(const double2 *)(ai + 4 * kk), x23 = *(const double2 *)(ai + 4 * kk + 2);
				const double2 y01 = *(const double2 *)(aj + 4 * kk), y23 = *(const double2 *)(aj + 4 * kk + 2);
				const double x[4] = {x01.x, x01.y, x23.x, x23.y}, y[4] = {y01.x, y01.y, y23.x, y23.y};
#pragma unroll
				for (int c = 0; c < 4; c++)
#pragma unroll
					for (int r = 0; r < 4; r++) acc[4 * c + r] = fma(x[r], y[c], acc[4 * c + r]);
			}
#pragma unroll
			for (int c = 0; c < 4; c++)
#pragma unroll
				for (int r = 0; r < 4; r++) {
					const int i = 4 * ti + r, j = 4 * tj + c;
					W[i * W_LD + j] = acc[4 * c + r] + (i == j ? shift : 0.0);
				}
		}
		if (li == 0) *bad = 0;
		__syncwarp();
		// 2. L = chol(S): lane i of the half holds row i in FP64 registers
		{
			double r[CM];
#pragma unroll
			for (int l = 0; l < CM; l++) r[l] = (l <= li) ? W[li * W_LD + l] : 0.0;
			DiagCol<0, double, 16>::run(r, li, CM, 0, dv, bad);
#pragma unroll
			for (int l = 0; l < CM; l++) W[li * W_LD + l] = (l <= li) ? r[l] : 0.0;
		}
		__syncwarp();
		// 3./4. X = R L^{-T} and D = C - X G^T, lane i owns row i; G read four
		// rows (one panel column) at a time
		{
			const int i = li;
			double x[CM];
#pragma unroll
			for (int j = 0; j < CM; j++) {
				double s = R[pm_idx16(i, j)];
#pragma unroll
				for (int l = 0; l < j; l++) s = fma(-x[l], W[j * W_LD + l], s);
				x[j] = s * dv[j];
			}
#pragma unroll
			for (int jp = 0; jp < CM / 4; jp++) {
				double s[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
				for (int l = 0; l < CM; l++) {
					const double2 g01 = *(const double2 *)(G + jp * 4 * CM + 4 * l);
					const double2 g23 = *(const double2 *)(G + jp * 4 * CM + 4 * l + 2);
					s[0] = fma(x[l], g01.x, s[0]);
					s[1] = fma(x[l], g01.y, s[1]);
					s[2] = fma(x[l], g23.x, s[2]);
					s[3] = fma(x[l], g23.y, s[3]);
				}
#pragma unroll
				for (int q = 0; q < 4; q++) Cm[pm_idx16(i, 4 * jp + q)] -= s[q];
			}
#pragma unroll
			for (int j = 0; j < CM; j++) R[pm_idx16(i, j)] = x[j];
		}
		__syncwarp();
		// 5. outputs: L lower triangle (and its inverse diagonal), X, D
		if (act) {
			double *gL = pL + sl * b, *gX = pX + sx * b, *gD = pD + sd * b;
			for (int e = li; e < CM * CM; e += 16) {
				const int j = (e & 63) >> 2, i = ((e >> 6) << 2) | (e & 3);
				if (j <= i) gL[e] = W[i * W_LD + j];
			}
			(pLd + sl * b)[li] = dv[li];
			for (int e = 2 * li; e < CM * CM; e += 32) {
				*(double2 *)(gX + e) = *(const double2 *)(R + e);
				*(double2 *)(gD + e) = *(const double2 *)(Cm + e);
			}
			if (li == 0 && info) info[b] = *bad;
		}
		// this pair's generic accesses to the slot are ordered before the next
		// pair's bulk copies into it
		fence_proxy_async_smem();
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
	const size_t smem = (size_t)lay.half_bytes * 2 * CH_WARPS;
	cudaFuncSetAttribute(k_chain16, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
	int per_sm = 0;
	cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_chain16, CH_WARPS * 32, smem);
	if (per_sm < 1) per_sm = 1;
	long long grid = (long long)bf::num_sms() * per_sm;
	long long need = ((long long)batch + 2 * CH_WARPS - 1) / (2 * CH_WARPS);
	if (grid > need) grid = need;
	k_chain16<<<(unsigned)grid, CH_WARPS * 32, smem, (cudaStream_t)stream>>>(
	    batch, k, shift, sA->pA, sA->stride, sR->pA, sR->stride, sC->pA, sC->stride, sG->pA, sG->stride, sL->pA,
	    sL->dA, sL->stride, sX->pA, sX->stride, sD->pA, sD->stride, info, bf::wait_limit());
	return bf::check_launch();
}

}  // extern "C"
