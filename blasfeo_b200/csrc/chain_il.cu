// The fused n = 16 chain (blasfeo_dsyrk_dpotrf_dtrsm_dgemm_batch, chain.cu)
// on batch-interleaved slabs (interleave.cu): a quad of lanes per instance,
// 8 instances per warp, every load and store one element of 8 consecutive
// instances (a contiguous 64-byte run of the interleaved layout).
//
// Lane q of the quad owns the rows i = q + 4s (s = 0..3) of S / L, of X and
// of D.  Per instance (the reference sequence blasfeo_dsyrk_ln
// (d_blas3_lib4.c:5400) + blasfeo_ddiare + blasfeo_dpotrf_l
// (d_lapack_lib4.c:918) + blasfeo_dtrsm_rltn (d_blas3_lib4.c:4123) +
// blasfeo_dgemm_nt (d_blas3_lib4.c:727)):
//   S = A A^T + shift I   in registers, rank-1 updates of the lane's rows by
//                         column l of A, read from shared memory that
//                         cp.async fills 8 columns at a time, double-buffered
//                         (the copies hold no registers);
//   L = chol(S)           column by column in registers, pivot rule of
//                         kernel/generic/kernel_dgemm_4x4_lib4.c:5700-5710
//                         (c > 0 -> sqrt(c) and 1/sqrt(c), else 0 and 0), the
//                         pivot column passed around the quad by shuffles;
//                         then L's strictly lower part and inverse pivots
//                         parked in shared memory, which frees S's registers;
//   X = R L^{-T}          the lane's 4 rows of R in registers, column by
//                         column, d_ij = (r_ij - sum_{l<j} d_il L_jl) *
//                         (1/L_jj) as the reference's trsm, each L_jl read
//                         once from shared memory for the 4 rows;
//   D = C - X G^T         G staged the same way, rows 0..7 issued before the
//                         factorization so that they land under it, rows
//                         8..15 under the first half of D.
// Each load or copy moves one element of 8 consecutive instances (64 bytes).
// Loads that a warp waits on one at a time leave it latency-bound, so the
// kernel keeps copies in flight and 12 warps per SM (168 registers, 16.5 KB
// of shared memory per warp).
// L's lower triangle and inverse diagonal, X and D are written once.
#include "quad.cuh"

namespace {

using namespace quad;

struct ChainIlArgs {
	int batch, k;
	double shift;
	const double *A, *R, *C, *G;
	double *L, *X, *D;
	long long ga, g16;  // group strides (elements) of the 16 x k and 16 x 16 slabs
	int cna;            // panel stride of A (k rounded up to 4)
	int *info;
};

constexpr int WPB = 4;                // warps per block
constexpr int LSLOTS = 120 + 16;      // strictly lower L, then the inverse diagonal
constexpr int BSLOTS = 128;           // staging buffer: 128 elements of 8 instances

// 128 elements (i, c) of the warp's 8 instances, i in [r0, r0 + nr), c in
// [c0, c0 + nc) (nr * nc = 128) of a panel-major slab with panel stride cn,
// columns >= ncol skipped, into stage[nc (i - r0) + (c - c0)][t]: each element
// of 8 instances is one 64-byte run in HBM, copied as four 16-byte pieces; 16
// pieces per lane, none held in registers.
__device__ __forceinline__ void stage_128(double (*stage)[QPW], const double *grp, int cn, int r0, int c0, int nc,
                                          int ncol, int lane) {
#pragma unroll 4
	for (int r = 0; r < 16; r++) {
		const int p = lane + 32 * r;
		const int el = p >> 2, part = p & 3;
		const int i = r0 + el / nc, c = c0 + el % nc;
		if (c < ncol) cpa16(&stage[el][2 * part], grp + pme(i, c, cn) * IL + 2 * part);
	}
}

template <int N>
__device__ __forceinline__ void cpa_wait() {
	asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

__global__ void __launch_bounds__(WPB * 32, 3) k_chain16_il(ChainIlArgs a) {
	// per warp: L_jl (l < j) of its 8 instances at lw[tri(j) + l][t], the
	// inverse pivots at lw[120 + j][t]; a 128-element staging buffer st.  A is
	// staged 8 columns at a time, alternately into st and into lw (free until
	// the factorization), so the next chunk's copies run under the current
	// chunk's products; G rows 0..7 go to st before the factorization, rows
	// 8..15 to lw after the solve.  The 8 quads of a warp read 8 consecutive
	// doubles, no bank conflict.
	extern __shared__ __align__(16) double dsm[];
	const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
	double(*lw)[QPW] = (double(*)[QPW])(dsm + (size_t)w * (LSLOTS + BSLOTS) * QPW);
	double(*st)[QPW] = lw + LSLOTS;
	const int q = lane & 3, t = lane >> 2;
	const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	if (gw * QPW >= a.batch) return;  // a whole warp past the batch (no block barrier follows)
	const long long b = gw * QPW + t;
	const bool act = b < a.batch;
	// the warp's 8 instances: half of group gw / 2 (the slab holds whole
	// groups, so the copies of a partial last group stay inside it)
	const long long g = gw >> 1;
	const int sl0 = (int)(gw & 1) * QPW;
	const double *Ag = a.A + g * a.ga + sl0;
	const double *Gg = a.G + g * a.g16 + sl0;
	const double *Rm = a.R + g * a.g16 + sl0 + t;
	const double *Cm = a.C + g * a.g16 + sl0 + t;
	double *Lg = a.L + g * a.g16 + sl0 + t;
	double *Xg = a.X + g * a.g16 + sl0 + t;
	double *Dg = a.D + g * a.g16 + sl0 + t;

	// 1. S = A A^T + shift I (rows q + 4s), A staged 8 columns at a time,
	// double-buffered
	double S[4][16];
#pragma unroll
	for (int s = 0; s < 4; s++)
#pragma unroll
		for (int j = 0; j < 16; j++) S[s][j] = 0.0;
	const int nch = (a.k + 7) / 8;
	stage_128(st, Ag, a.cna, 0, 0, 8, a.k, lane);
	cpa_commit();
	for (int ch = 0; ch < nch; ch++) {
		double(*cur)[QPW] = (ch & 1) ? lw : st;
		if (ch + 1 < nch) {
			stage_128((ch & 1) ? st : lw, Ag, a.cna, 0, 8 * (ch + 1), 8, a.k, lane);
			cpa_commit();
			cpa_wait<1>();
		} else {
			cpa_wait<0>();
		}
		__syncwarp();
		const int nc = min(8, a.k - 8 * ch);
#pragma unroll 2
		for (int c = 0; c < nc; c++) {
			double col[16];
#pragma unroll
			for (int i = 0; i < 16; i++) col[i] = cur[8 * i + c][t];
#pragma unroll
			for (int s = 0; s < 4; s++) {
				const double ai =
				    (q == 0) ? col[4 * s] : (q == 1) ? col[4 * s + 1] : (q == 2) ? col[4 * s + 2] : col[4 * s + 3];
#pragma unroll
				for (int j = 0; j < 16; j++)
					if (j <= 4 * s + 3) S[s][j] = fma(ai, col[j], S[s][j]);
			}
		}
		__syncwarp();
	}
	// G rows 0..7: copies run under the factorization and the solve
	stage_128(st, Gg, 16, 0, 0, 16, 16, lane);
	cpa_commit();
	// shift on the diagonal; entries right of it (computed with the others,
	// never used) cleared
	clear_upper(S, q, a.shift);

	// 2. L = chol(S); L to HBM (lower triangle and dA slots after the 16 x 16
	// panel block) and its strictly lower part to shared memory
	int bad = 0;
	QCol<0, true>::run(S, q, lane, 16, &lw[120][t], Lg + 256LL * IL, act, bad);
#pragma unroll
	for (int s = 0; s < 4; s++) {
		const int i = q + 4 * s;
#pragma unroll
		for (int j = 0; j < 16; j++) {
			if (j <= 4 * s + 3 && j <= i) {
				if (act) Lg[pme(i, j, 16) * IL] = S[s][j];
				if (j < i) lw[tri(i) + j][t] = S[s][j];
			}
		}
	}
	if (act && q == 0 && a.info) a.info[b] = bad;
	__syncwarp();

	// 3. X = R L^{-T}: the lane's four rows together, L_jl broadcast to the quad
	double x[4][16];
#pragma unroll
	for (int s = 0; s < 4; s++)
#pragma unroll
		for (int j = 0; j < 16; j++) x[s][j] = Rm[pme(q + 4 * s, j, 16) * IL];
#pragma unroll
	for (int j = 0; j < 16; j++) {
#pragma unroll
		for (int l = 0; l < j; l++) {
			const double ljl = lw[tri(j) + l][t];
#pragma unroll
			for (int s = 0; s < 4; s++) x[s][j] = fma(-x[s][l], ljl, x[s][j]);
		}
		const double iv = lw[120 + j][t];
#pragma unroll
		for (int s = 0; s < 4; s++) x[s][j] *= iv;
	}
	if (act) {
#pragma unroll
		for (int s = 0; s < 4; s++)
#pragma unroll
			for (int j = 0; j < 16; j++) Xg[pme(q + 4 * s, j, 16) * IL] = x[s][j];
	}

	// 4. D = C - X G^T: G rows 8..15 staged into lw (the solve is done with
	// it), columns 0..7 of D from st meanwhile
	__syncwarp();
	stage_128(lw, Gg, 16, 8, 0, 16, 16, lane);
	cpa_commit();
	cpa_wait<1>();
	__syncwarp();
#pragma unroll 1
	for (int h = 0; h < 2; h++) {
		if (h == 1) {
			cpa_wait<0>();
			__syncwarp();
		}
		double(*gs)[QPW] = h ? lw : st;
#pragma unroll 2
		for (int jj = 0; jj < 8; jj++) {
			const int j = 8 * h + jj;
			double cv[4];
#pragma unroll
			for (int s = 0; s < 4; s++) cv[s] = Cm[pme(q + 4 * s, j, 16) * IL];
#pragma unroll
			for (int l = 0; l < 16; l++) {
				const double gv = gs[16 * jj + l][t];
#pragma unroll
				for (int s = 0; s < 4; s++) cv[s] = fma(-x[s][l], gv, cv[s]);
			}
			if (act) {
#pragma unroll
				for (int s = 0; s < 4; s++) Dg[pme(q + 4 * s, j, 16) * IL] = cv[s];
			}
		}
	}
}

template <typename BT>
bool il_ok(const BT *s, int m, int n, int batch) {
	return s && s->mem && s->m == m && s->n == n && s->batch >= batch && s->il == IL;
}

}  // namespace

extern "C" int blasfeo_dsyrk_dpotrf_dtrsm_dgemm_batch_il(int batch, int m, int k, double shift,
                                                         struct blasfeo_dmat_batch_il *sA,
                                                         struct blasfeo_dmat_batch_il *sR,
                                                         struct blasfeo_dmat_batch_il *sC,
                                                         struct blasfeo_dmat_batch_il *sG,
                                                         struct blasfeo_dmat_batch_il *sL,
                                                         struct blasfeo_dmat_batch_il *sX,
                                                         struct blasfeo_dmat_batch_il *sD, int *info, void *stream) {
	if (batch < 0 || !sA) return BLASFEO_B200_EINVAL;
	if (batch == 0) return BLASFEO_B200_OK;
	if (m != 16 || k < 1) return BLASFEO_B200_ENOTSUP;
	// the staging copies move 16-byte pieces: slabs on 16-byte boundaries
	if (!il_ok(sA, 16, k, batch) || ((uintptr_t)sA->mem & 15)) return BLASFEO_B200_EINVAL;
	const struct blasfeo_dmat_batch_il *sq[] = {sR, sC, sG, sL, sX, sD};
	for (auto p : sq)
		if (!il_ok(p, 16, 16, batch) || p->gstride != sR->gstride || ((uintptr_t)p->mem & 15))
			return BLASFEO_B200_EINVAL;
	ChainIlArgs a;
	a.batch = batch;
	a.k = k;
	a.shift = shift;
	a.A = sA->mem;
	a.R = sR->mem;
	a.C = sC->mem;
	a.G = sG->mem;
	a.L = sL->mem;
	a.X = sX->mem;
	a.D = sD->mem;
	a.ga = sA->gstride;
	a.g16 = sR->gstride;
	a.cna = sA->cn;
	a.info = info;
	const long long warps = (batch + QPW - 1) / QPW;
	const long long blocks = (warps + WPB - 1) / WPB;
	const int smem = WPB * (LSLOTS + BSLOTS) * QPW * (int)sizeof(double);
	cudaFuncSetAttribute(k_chain16_il, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
	k_chain16_il<<<(unsigned)blocks, WPB * 32, smem, (cudaStream_t)stream>>>(a);
	return bf::check_launch();
}
