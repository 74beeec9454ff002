// Batched Riccati factorization (riccati.cu's recursion) on batch-interleaved
// slabs: a group of G lanes per problem (G = 4 by default: a quad), 32 / G
// problems per warp.
//
// Per problem (examples/example_d_riccati_recursion.c:115-143,
// d_back_ric_trf_libstr):
//   L_N = chol(Q_N)                                   (blasfeo_dpotrf_l)
//   for k = N-1 .. 0:
//     W   = BAbt_k * Lxx_{k+1}                        (blasfeo_dtrmm_rlnn)
//     L_k = chol(RSQ_k + W W^T)                       (blasfeo_dsyrk_dpotrf_ln)
// with Lxx_{k+1} the lower-right nx x nx block of L_{k+1} (all of L_N).
//
// Slabs are stage-major so that the problems of a warp are consecutive
// instances at every stage: stage k of problem b is instance k * bs + b,
// bs = batch rounded up to a multiple of 16.  Each element of the warp's
// problems is one contiguous run in HBM (64 bytes for G = 4), copied by
// cp.async (16-byte pieces that hold no registers) into the warp's stage
// buffer; the copies of stage k-1 are issued before stage k's factorization
// and land under it.
//
// Lane o of the group owns rows o + G s of W, of RSQ_k + W W^T and of L_k; the
// previous factor is kept in shared memory (lower triangle with the diagonal)
// and read broadcast to the group; BAbt_k and W are staged column-major, so a
// lane's own entries and a column read by all lanes are both free of bank
// conflicts.  The products are FP64 in the reference's order:
// W_ij = sum_{l=j}^{nx-1} BAbt_il L_lj ascending in l, then
// RSQ_ij + sum_l W_il W_jl ascending in l; the 16 x 16 factor runs in
// registers (quad::GCol, the reference's pivot rule).
#include "quad.cuh"

namespace {

using namespace quad;

constexpr int LP_SLOTS = 136;          // previous factor, lower triangle with the diagonal
constexpr int BW_SLOTS = 256;          // BAbt_k column-major, overwritten row by row by W
constexpr int RQ_SLOTS = 136;          // lower triangle of RSQ_k
constexpr int WARP_SLOTS = LP_SLOTS + BW_SLOTS + RQ_SLOTS;
constexpr int RIC_THREADS = 64;
#ifndef RIC_G
#define RIC_G 4                        // lanes per problem (4, 8, 16 measured: 4 fastest)
#endif

struct RicIlArgs {
	int batch, N, nx, nu;
	long long bs;                      // instances per stage
	const double *BA, *RSQ;
	double *L;
	long long gba, g16;                // group strides (elements) of the 16 x nx and 16 x 16 slabs
	int cnx;                           // panel stride of BAbt
	int *info;
};

// stage k's inputs of the warp's P problems (group gb of a stage, first slot
// sl0): each element of the P problems is P doubles in HBM, copied as P / 2
// pieces of 16 bytes
template <int P>
__device__ __forceinline__ void stage_inputs(const RicIlArgs &a, int k, long long gb, int sl0, double (*bw)[P],
                                             double (*rq)[P], int lane) {
	constexpr int PC = P / 2;          // pieces per element
	const long long gk = (long long)k * (a.bs / IL) + gb;
	const double *R = a.RSQ + gk * a.g16 + sl0;
#pragma unroll 4
	for (int p = lane; p < 256 * PC; p += 32) {
		const int el = p / PC, part = p % PC;
		const int i = el >> 4, j = el & 15;
		if (j <= i) cpa16(&rq[tri_d(i) + j][2 * part], R + pme(i, j, 16) * IL + 2 * part);
	}
	if (k < a.N) {
		const double *B = a.BA + gk * a.gba + sl0;
#pragma unroll 4
		for (int p = lane; p < 256 * PC; p += 32) {
			const int el = p / PC, part = p % PC;
			const int i = el & 15, l = el >> 4;
			if (l < a.nx) cpa16(&bw[16 * l + i][2 * part], B + pme(i, l, a.cnx) * IL + 2 * part);
		}
	}
}

// G lanes per problem, P = 32 / G problems per warp
template <int G>
__global__ void __launch_bounds__(RIC_THREADS) k_ric_trf_il(RicIlArgs a) {
	constexpr int P = 32 / G, R = 16 / G;
	extern __shared__ __align__(16) double dsm[];
	const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
	double(*lp)[P] = (double(*)[P])(dsm + (size_t)w * WARP_SLOTS * P);
	double(*bw)[P] = lp + LP_SLOTS;
	double(*rq)[P] = bw + BW_SLOTS;
	const int o = lane % G, t = lane / G;
	const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	if (gw * P >= a.batch) return;  // a whole warp past the batch (no block barrier follows)
	const long long b = gw * P + t;
	const bool act = b < a.batch;
	const long long gb = (gw * P) / IL;
	const int sl0 = (int)((gw * P) % IL);
	const int M = a.nu + a.nx;
	int first = 0;

	stage_inputs<P>(a, a.N, gb, sl0, bw, rq, lane);
	cpa_commit();
	for (int k = a.N; k >= 0; k--) {
		cpa_wait_all();
		__syncwarp();
		const int m = (k == a.N) ? a.nx : M;  // size of this stage's factor
		// S = RSQ_k on the lane's rows, rows and columns >= m an identity block
		double S[R][16];
#pragma unroll
		for (int s = 0; s < R; s++) {
			const int i = o + G * s;
#pragma unroll
			for (int j = 0; j < 16; j++) {
				const double v = (j <= i && i < m) ? rq[tri_d(i) + j][t] : 0.0;
				S[s][j] = (i >= m && j == i) ? 1.0 : v;
			}
		}
		if (k < a.N) {
			const int off = (k + 1 == a.N) ? 0 : a.nu;  // Lxx inside L_{k+1}
			// W = BAbt_k * Lxx_{k+1}, the lane's rows, written over them
#pragma unroll 1
			for (int s = 0; s < R; s++) {
				const int i = o + G * s;
				double ba[16], wr[16];
#pragma unroll
				for (int l = 0; l < 16; l++) ba[l] = bw[16 * l + i][t];
#pragma unroll
				for (int j = 0; j < 16; j++) {
					double acc = 0.0;
#pragma unroll
					for (int l = j; l < 16; l++)
						if (l < a.nx) acc = fma(ba[l], lp[tri_d(off + l) + off + j][t], acc);
					wr[j] = acc;
				}
#pragma unroll
				for (int j = 0; j < 16; j++)
					if (j < a.nx) bw[16 * j + i][t] = wr[j];
			}
			__syncwarp();
			// + W W^T over the first M rows
			syrk_rows_cm<G, P>(S, bw, a.nx, M, o, t);
		}
		clear_upper_g<G>(S, o, 0.0);
		__syncwarp();
		// stage k-1's inputs land under this stage's factorization
		if (k > 0) {
			stage_inputs<P>(a, k - 1, gb, sl0, bw, rq, lane);
			cpa_commit();
		}
		const long long idx = (long long)k * a.bs + b;
		double *Lg = a.L + (idx / IL) * a.g16 + idx % IL;
		int bad = 0;
		GCol<G, 0, false>::run(S, o, lane, m, nullptr, Lg + 256LL * IL, act, bad);
		if (bad && first == 0) first = (a.N - k) * 16 + bad;
		// L_k: rows < m to HBM; the whole lower triangle kept for stage k-1
#pragma unroll
		for (int s = 0; s < R; s++) {
			const int i = o + G * s;
#pragma unroll
			for (int j = 0; j < 16; j++) {
				if (j <= G * s + G - 1 && j <= i) {
					if (act && i < m) Lg[pme(i, j, 16) * IL] = S[s][j];
					lp[tri_d(i) + j][t] = S[s][j];
				}
			}
		}
		__syncwarp();
	}
	if (act && o == 0 && a.info) a.info[b] = first;
}

template <int G>
int launch_ric_il(const RicIlArgs &a, cudaStream_t s) {
	constexpr int P = 32 / G;
	const long long warps = (a.batch + P - 1) / P;
	const long long blocks = (warps * 32 + RIC_THREADS - 1) / RIC_THREADS;
	const int smem = (RIC_THREADS / 32) * WARP_SLOTS * P * (int)sizeof(double);
	cudaFuncSetAttribute(k_ric_trf_il<G>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
	k_ric_trf_il<G><<<(unsigned)blocks, RIC_THREADS, smem, s>>>(a);
	return bf::check_launch();
}

bool il16(const struct blasfeo_dmat_batch_il *s, int n, long long need) {
	return s && s->mem && s->m == 16 && s->n == n && (long long)s->batch >= need && s->il == IL &&
	       !((uintptr_t)s->mem & 15);
}

}  // namespace

extern "C" int blasfeo_dric_trf_batch_il(int batch, int N, int nx, int nu, struct blasfeo_dmat_batch_il *sBAbt,
                                         struct blasfeo_dmat_batch_il *sRSQ, struct blasfeo_dmat_batch_il *sL,
                                         int *info, void *stream) {
	if (batch < 0 || N < 0 || nx < 1 || nu < 0) return BLASFEO_B200_EINVAL;
	if (batch == 0) return BLASFEO_B200_OK;
	if (nu + nx > 16) return BLASFEO_B200_ENOTSUP;
	const long long bs = (batch + IL - 1) / IL * IL;
	if (!il16(sRSQ, 16, (N + 1) * bs) || !il16(sL, 16, (N + 1) * bs) || sRSQ->gstride != sL->gstride)
		return BLASFEO_B200_EINVAL;
	if (N > 0 && !il16(sBAbt, nx, N * bs)) return BLASFEO_B200_EINVAL;
	RicIlArgs a;
	a.batch = batch;
	a.N = N;
	a.nx = nx;
	a.nu = nu;
	a.bs = bs;
	a.BA = N > 0 ? sBAbt->mem : nullptr;
	a.RSQ = sRSQ->mem;
	a.L = sL->mem;
	a.gba = N > 0 ? sBAbt->gstride : 0;
	a.g16 = sRSQ->gstride;
	a.cnx = N > 0 ? sBAbt->cn : 4;
	a.info = info;
	return launch_ric_il<RIC_G>(a, (cudaStream_t)stream);
}
