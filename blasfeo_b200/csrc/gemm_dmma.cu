// FP64 gemm_nt / syrk_ln on the FP64 tensor cores (DMMA, mma.sync m8n8k4
// f64): D = beta*C + alpha*A*B^T, syrk writing only the lower triangle
// (blasfeo_hp_pm/d_blas3_lib4.c:727 gemm_nt, :5400 syrk_ln).
//
// One CTA computes a BM x BN output tile of one instance; every warp owns a
// 32 x 32 sub-tile as 4 x 4 fragments of 8 x 8 (two FP64 accumulators per
// thread and fragment).  K is walked in BK = 16 slices through a 3-stage
// cp.async pipeline.  The staging copies BLASFEO's panel layout as it is: the
// BK columns of one 4-row panel are one contiguous run of 4*BK doubles in
// global memory and land as one contiguous run in shared memory, so every
// 16-byte copy is fully used.  An m8n8k4 operand fragment (8 rows x 4 k:
// lane l holds row l/4, k l%4) is then two 4x4 tiles of two panels, i.e. two
// contiguous 128-byte runs: conflict-free shared-memory loads.
//
// Out-of-range rows of a partial tile only feed output rows/columns that are
// never stored; columns k >= K are zero-filled in both operands.  C is read
// only when beta != 0 (as the HP kernels do).  Instances whose row offset is
// not a multiple of 4, or whose panels are not 16-byte aligned, are copied
// element by element (8-byte cp.async) with the same arithmetic.
#include "common.cuh"
#include "kernels.cuh"

namespace {

constexpr int DM_BK = 16;
constexpr int DM_STAGES = 3;

__device__ __forceinline__ void cp_async16(uint32_t dst, const void *src, uint32_t src_bytes) {
	asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async8(uint32_t dst, const void *src, uint32_t src_bytes) {
	asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(dst), "l"(src), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
	asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

__device__ __forceinline__ void dmma(double &d0, double &d1, double a, double b) {
	asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
	             : "+d"(d0), "+d"(d1)
	             : "d"(a), "d"(b));
}

// Stage the ROWS x BK slice (rows r0.., columns k0..) of one operand into
// shared memory `dst` (panel-major: panel p at p*4*BK, column kk at 4*kk).
// Chunk c (16 bytes, two rows of one column) of the slice sits at dst + 2c.
template <int ROWS, int NT>
__device__ __forceinline__ void stage_operand(double *dst, const PMat<double> &a, int rows, int kdim, int r0,
                                              int k0, bool fast) {
	const uint32_t sdst = (uint32_t)__cvta_generic_to_shared(dst);
	if (fast) {
		constexpr int CH = ROWS * DM_BK / 2;
#pragma unroll
		for (int c = threadIdx.x; c < CH; c += NT) {
			const int p = c / (2 * DM_BK), w = c % (2 * DM_BK);
			const int kk = w >> 1;
			const bool ok = (r0 + 4 * p < rows) && (k0 + kk < kdim);
			const double *src = ok ? a.addr(r0 + 4 * p + 2 * (w & 1), k0 + kk) : a.p;
			cp_async16(sdst + 16u * c, src, ok ? 16u : 0u);
		}
	} else {
		constexpr int EL = ROWS * DM_BK;
		for (int e = threadIdx.x; e < EL; e += NT) {
			const int p = e / (4 * DM_BK), w = e % (4 * DM_BK);
			const int kk = w >> 2, r = r0 + 4 * p + (w & 3);
			const bool ok = (r < rows) && (k0 + kk < kdim);
			const double *src = ok ? a.addr(r, k0 + kk) : a.p;
			cp_async8(sdst + 8u * e, src, ok ? 8u : 0u);
		}
	}
}

template <int BM, int BN, bool LOWER>
__global__ void __launch_bounds__((BM / 32) * (BN / 32) * 32)
    k_dgemm_nt_dmma(SizeArg sz, double alpha, MatArg<double> A, MatArg<double> B, double beta, MatArg<double> C,
                    MatArg<double> D, int tiles_n, int tiles_mn) {
	constexpr int WN = BN / 32;
	constexpr int NT = (BM / 32) * WN * 32;
	constexpr int SA = BM * DM_BK, SB = BN * DM_BK;  // doubles per stage
	extern __shared__ __align__(128) double dm_smem[];
	double *sA = dm_smem;
	double *sB = dm_smem + DM_STAGES * SA;

	// one-dimensional grid with the output tiles of one instance consecutive:
	// the CTAs that share an instance's A and B slices run together and meet in L2
	const int b = (int)(blockIdx.x / (unsigned)tiles_mn);
	const int tile = (int)(blockIdx.x % (unsigned)tiles_mn);
	const int m = sz.M(b), n = sz.N(b), k = sz.K(b);
	const int tmi = tile / tiles_n, tni = tile % tiles_n;
	const int i0 = tmi * BM, j0 = tni * BN;
	if (i0 >= m || j0 >= n) return;
	if (LOWER && j0 > i0 + BM - 1) return;
	const PMat<double> a = A.get(b), bm = B.get(b), c = C.get(b), d = D.get(b);
	// the 16-byte copies need panel-aligned rows and 16-byte aligned panels
	const bool fast_a = ((a.ri & 3) == 0) && ((((uintptr_t)a.p) & 15) == 0);
	const bool fast_b = ((bm.ri & 3) == 0) && ((((uintptr_t)bm.p) & 15) == 0);

	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	const int wm0 = (warp / WN) * 32, wn0 = (warp % WN) * 32;
	const int fr = lane >> 2, fk = lane & 3;

	double acc[4][4][2];
#pragma unroll
	for (int i = 0; i < 4; i++)
#pragma unroll
		for (int j = 0; j < 4; j++) acc[i][j][0] = acc[i][j][1] = 0.0;

	const int KT = (k + DM_BK - 1) / DM_BK;
#pragma unroll
	for (int s = 0; s < DM_STAGES - 1; s++) {
		if (s < KT) {
			stage_operand<BM, NT>(sA + s * SA, a, m, k, i0, s * DM_BK, fast_a);
			stage_operand<BN, NT>(sB + s * SB, bm, n, k, j0, s * DM_BK, fast_b);
		}
		cp_async_commit();
	}
	for (int kt = 0; kt < KT; kt++) {
		cp_async_wait<DM_STAGES - 2>();
		__syncthreads();
		{
			const int ks = kt + DM_STAGES - 1;
			if (ks < KT) {
				const int buf = ks % DM_STAGES;
				stage_operand<BM, NT>(sA + buf * SA, a, m, k, i0, ks * DM_BK, fast_a);
				stage_operand<BN, NT>(sB + buf * SB, bm, n, k, j0, ks * DM_BK, fast_b);
			}
			cp_async_commit();
		}
		const double *tA = sA + (kt % DM_STAGES) * SA;
		const double *tB = sB + (kt % DM_STAGES) * SB;
#pragma unroll
		for (int kq = 0; kq < DM_BK / 4; kq++) {
			double av[4], bv[4];
#pragma unroll
			for (int i = 0; i < 4; i++) {
				const int lr = wm0 + 8 * i + fr;
				av[i] = tA[(lr >> 2) * (4 * DM_BK) + (4 * kq + fk) * 4 + (lr & 3)];
			}
#pragma unroll
			for (int j = 0; j < 4; j++) {
				const int lc = wn0 + 8 * j + fr;
				bv[j] = tB[(lc >> 2) * (4 * DM_BK) + (4 * kq + fk) * 4 + (lc & 3)];
			}
#pragma unroll
			for (int i = 0; i < 4; i++)
#pragma unroll
				for (int j = 0; j < 4; j++) dmma(acc[i][j][0], acc[i][j][1], av[i], bv[j]);
		}
	}
	cp_async_wait<0>();

	// epilogue: fragment (i,j), thread holds row 8i + lane/4, columns 8j + 2(lane%4) + {0,1}
#pragma unroll
	for (int i = 0; i < 4; i++) {
		const int gi = i0 + wm0 + 8 * i + fr;
		if (gi >= m) continue;
#pragma unroll
		for (int j = 0; j < 4; j++) {
#pragma unroll
			for (int h = 0; h < 2; h++) {
				const int gj = j0 + wn0 + 8 * j + 2 * fk + h;
				if (gj >= n) continue;
				if (LOWER && gj > gi) continue;
				double v = alpha * acc[i][j][h];
				if (beta != 0.0) v = fma(beta, c.at(gi, gj), v);
				d.at(gi, gj) = v;
			}
		}
	}
}

template <int BM, int BN, bool LOWER>
int launch_dmma(int batch, SizeArg sz, int max_m, int max_n, double alpha, MatArg<double> A, MatArg<double> B,
                double beta, MatArg<double> C, MatArg<double> D, cudaStream_t s) {
	constexpr int NT = (BM / 32) * (BN / 32) * 32;
	const size_t smem = (size_t)DM_STAGES * (BM + BN) * DM_BK * sizeof(double);
	auto kern = k_dgemm_nt_dmma<BM, BN, LOWER>;
	bf::smem_optin(kern, smem);
	const int tm = cdiv(max_m, BM), tn = cdiv(max_n, BN);
	const long long ctas = (long long)batch * tm * tn;
	if (ctas > 0x7fffffffLL) return BLASFEO_B200_ENOTSUP;
	kern<<<(unsigned)ctas, NT, smem, s>>>(sz, alpha, A, B, beta, C, D, tn, tm * tn);
	return bf::check_launch();
}

}  // namespace

namespace bf {

// FP64 tensor-core gemm_nt / syrk_ln: tile 0 = 64 x 64 (4 warps), 1 = 32 x 32 (1 warp)
template <bool LOWER>
int dgemm_nt_dmma_launch(int batch, SizeArg sz, int max_m, int max_n, double alpha, MatArg<double> A,
                         MatArg<double> B, double beta, MatArg<double> C, MatArg<double> D, cudaStream_t s,
                         int tile) {
	if (tile == 0) return launch_dmma<64, 64, LOWER>(batch, sz, max_m, max_n, alpha, A, B, beta, C, D, s);
	return launch_dmma<32, 32, LOWER>(batch, sz, max_m, max_n, alpha, A, B, beta, C, D, s);
}
template int dgemm_nt_dmma_launch<false>(int, SizeArg, int, int, double, MatArg<double>, MatArg<double>, double,
                                         MatArg<double>, MatArg<double>, cudaStream_t, int);
template int dgemm_nt_dmma_launch<true>(int, SizeArg, int, int, double, MatArg<double>, MatArg<double>, double,
                                        MatArg<double>, MatArg<double>, cudaStream_t, int);

}  // namespace bf
