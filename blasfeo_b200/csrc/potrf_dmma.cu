// FP64 Cholesky potrf_l (blasfeo_hp_pm/d_lapack_lib4.c:918) for instances with
// n <= 64: one warp per instance, the whole lower triangle in registers, the
// trailing updates on the FP64 tensor cores (DMMA, mma.sync m8n8k4 f64).
//
// The matrix is a grid of 8 x 8 blocks; block (I,J), J <= I, is held as an
// m8n8 accumulator fragment: lane l keeps row 8I + l/4, columns 8J + 2(l%4)
// and 8J + 2(l%4) + 1.  Unfactored blocks are kept NEGATED (F = -A), so the
// rank-8 trailing update A_IJ -= L_IK L_JK^T is a plain accumulate,
// F_IJ += L_IK L_JK^T, two m8n8k4 DMMAs per block.  Both operand fragments of
// that product (8 rows x 4 k, lane l: row l/4, k l%4) are the same shuffle of
// the factored panel block, so one fragment pair per block row serves as A
// and as B.
//
// Right-looking by 8-column panels K:
//   panel:   column by column, the FP64 pivot is broadcast by a shuffle, its
//            reciprocal square root taken (pivot rule of
//            kernel/generic/kernel_dgemm_4x4_lib4.c:5700-5710: c > 0 ->
//            L_jj = c * rsqrt(c), dA_j = rsqrt(c); else 0 and 0), the column
//            scaled and the rest of the panel updated with FMAs;
//   trailing: every block right of the panel, two DMMAs each.
// Everything is unrolled over the compile-time block grid (N8 = ceil(n/8)), so
// the fragments never leave registers; rows and columns n..8*N8-1 hold the
// identity.  The instance arrives through shared memory (16-byte cp.async
// copies of the lower panels, all in flight together).  HBM traffic: one read
// and one write of the lower triangle.
#include "common.cuh"
#include "kernels.cuh"

namespace {

constexpr unsigned FULL = 0xffffffffu;

__device__ __forceinline__ void dmma_acc(double &d0, double &d1, double a, double b) {
	asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
	             : "+d"(d0), "+d"(d1)
	             : "d"(a), "d"(b));
}

__host__ __device__ constexpr int blk(int i, int j) { return i * (i + 1) / 2 + j; }

__device__ __forceinline__ void cp_async16(uint32_t dst, const void *src) {
	asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}

// doubles of the compact lower panels of an n8 x n8 matrix (panel p keeps its
// columns 0..4p+3 at offset 8p(p+1), the global panel layout cut at the
// diagonal tile)
__host__ __device__ constexpr int lower_panels(int n8) { return 8 * (n8 / 4) * (n8 / 4 + 1); }

template <int N8, int WPC, int MINB>
__global__ void __launch_bounds__(32 * WPC, MINB) k_potrf_dmma(int batch, SizeArg sz, MatArg<double> C,
                                                               MatArg<double> D, int *info) {
	constexpr int NB = N8 * (N8 + 1) / 2;
	const int lane = threadIdx.x & 31;
	const int b = blockIdx.x * WPC + (threadIdx.x >> 5);
	if (b >= batch) return;
	const int n = sz.M(b);
	if (n <= 0 || n > 8 * N8) return;
	const PMat<double> c = C.get(b), d = D.get(b);
	const int r = lane >> 2, q = lane & 3;

	// Stage the lower panels in shared memory with 16-byte asynchronous copies
	// (one wait for the whole instance: every copy is in flight at once), then
	// fill the fragments from there.  Rows not starting a panel, or panels not
	// 16-byte aligned, are read element by element from global memory.
	extern __shared__ __align__(16) double pot_smem[];
	double *S = pot_smem + (threadIdx.x >> 5) * lower_panels(8 * N8);
	const bool staged = ((c.ri & 3) == 0) && ((((uintptr_t)c.p) & 15) == 0);
	if (staged) {
		const uint32_t sbase = (uint32_t)__cvta_generic_to_shared(S);
		const int P = (n + 3) >> 2;
		for (int p = 0; p < P; p++) {
			const double *g = c.addr(4 * p, 0);
			for (int ch = lane; ch < 8 * (p + 1); ch += 32)
				cp_async16(sbase + 8u * (uint32_t)(8 * p * (p + 1) + 2 * ch), g + 2 * ch);
		}
		asm volatile("cp.async.wait_all;" ::: "memory");
		__syncwarp();
	}

	// fragments (negated), identity in the padding, zeros above the diagonal
	double F[NB][2];
#pragma unroll
	for (int I = 0; I < N8; I++)
#pragma unroll
		for (int J = 0; J <= I; J++)
#pragma unroll
			for (int h = 0; h < 2; h++) {
				const int gi = 8 * I + r, gj = 8 * J + 2 * q + h;
				double v;
				if (gi < n && gj < n) {
					if (gj > gi)
						v = 0.0;
					else
						v = -(staged ? S[8 * (gi >> 2) * ((gi >> 2) + 1) + 4 * gj + (gi & 3)] : *c.addr(gi, gj));
				} else {
					v = (gi == gj) ? -1.0 : 0.0;
				}
				F[blk(I, J)][h] = v;
			}

	int bad = 0;
#pragma unroll
	for (int K = 0; K < N8; K++) {
		const int KK = blk(K, K);
		// ---- panel K, column by column ----
#pragma unroll
		for (int cc = 0; cc < 8; cc++) {
			const int e = cc & 1, src = cc >> 1;
			const double cv = -__shfl_sync(FULL, F[KK][e], (cc << 2) | src);
			const bool ok = cv > 0.0;
			const double inv = ok ? rsqrt(cv) : 0.0;
			const double lcc = ok ? cv * inv : 0.0;
			if (!ok && bad == 0) bad = 8 * K + cc + 1;
			if (lane == 0 && 8 * K + cc < n) d.d[8 * K + cc] = inv;
			// scale column cc (held by the lanes with q == cc/2, element cc&1)
			if (q == src) {
#pragma unroll
				for (int I = K; I < N8; I++) {
					double &x = F[blk(I, K)][e];
					if (I > K || r > cc)
						x = -x * inv;
					else if (r == cc)
						x = lcc;
				}
			}
			if (cc < 7) {
				// update columns cc+1..7 of the panel: F(i,c') += L(i,cc) L(8K+c',cc)
				const double lk0 = __shfl_sync(FULL, F[KK][e], ((2 * q) << 2) | src);
				const double lk1 = __shfl_sync(FULL, F[KK][e], ((2 * q + 1) << 2) | src);
#pragma unroll
				for (int I = K; I < N8; I++) {
					const double li = __shfl_sync(FULL, F[blk(I, K)][e], (lane & ~3) | src);
					if (2 * q > cc && (I > K || r >= 2 * q)) F[blk(I, K)][0] = fma(li, lk0, F[blk(I, K)][0]);
					if (2 * q + 1 > cc && (I > K || r >= 2 * q + 1))
						F[blk(I, K)][1] = fma(li, lk1, F[blk(I, K)][1]);
				}
			}
		}
		if (K + 1 == N8) continue;
		// ---- operand fragments of the factored panel: a0 = L(8I+r, 8K+q), a1 = L(8I+r, 8K+4+q) ----
		double a0[N8], a1[N8];
#pragma unroll
		for (int I = K + 1; I < N8; I++) {
			const int s0 = (lane & ~3) | (q >> 1), s1 = (lane & ~3) | (2 + (q >> 1));
			const double t00 = __shfl_sync(FULL, F[blk(I, K)][0], s0);
			const double t01 = __shfl_sync(FULL, F[blk(I, K)][1], s0);
			const double t10 = __shfl_sync(FULL, F[blk(I, K)][0], s1);
			const double t11 = __shfl_sync(FULL, F[blk(I, K)][1], s1);
			a0[I] = (q & 1) ? t01 : t00;
			a1[I] = (q & 1) ? t11 : t10;
		}
		// ---- trailing update, next panel's column first ----
#pragma unroll
		for (int J = K + 1; J < N8; J++)
#pragma unroll
			for (int I = J; I < N8; I++) {
				dmma_acc(F[blk(I, J)][0], F[blk(I, J)][1], a0[I], a0[J]);
				dmma_acc(F[blk(I, J)][0], F[blk(I, J)][1], a1[I], a1[J]);
			}
	}

	// store the lower triangle of L
#pragma unroll
	for (int I = 0; I < N8; I++)
#pragma unroll
		for (int J = 0; J <= I; J++)
#pragma unroll
			for (int h = 0; h < 2; h++) {
				const int gi = 8 * I + r, gj = 8 * J + 2 * q + h;
				if (gi < n && gj <= gi) *d.addr(gi, gj) = F[blk(I, J)][h];
			}
	if (info && lane == 0) info[b] = bad;
}

template <int N8>
void launch_n8(int batch, SizeArg sz, MatArg<double> C, MatArg<double> D, int *info, cudaStream_t s) {
	constexpr int WPC = N8 <= 4 ? 4 : (N8 <= 6 ? 2 : 1);
	// n in 49..56: 168 registers (the fragments still fit) for 12 resident
	// warps per SM instead of 8 (measured 3.7 -> 4.4 TF/s at n = 56); at
	// n = 64 the same cap spills fragments and loses (4.4 -> 2.9 TF/s)
	constexpr int MINB = N8 == 7 ? 12 : 1;
	const size_t smem = (size_t)WPC * lower_panels(8 * N8) * sizeof(double);
	k_potrf_dmma<N8, WPC, MINB><<<(batch + WPC - 1) / WPC, 32 * WPC, smem, s>>>(batch, sz, C, D, info);
}

}  // namespace

namespace bf {

// FP64 potrf_l, one warp per instance, for max_m <= 64
int dpotrf_dmma_launch(int batch, SizeArg sz, int max_m, MatArg<double> C, MatArg<double> D, int *info,
                       cudaStream_t s) {
	if (max_m <= 0 || batch <= 0) return BLASFEO_B200_OK;
	switch ((max_m + 7) / 8) {
	case 1: launch_n8<1>(batch, sz, C, D, info, s); break;
	case 2: launch_n8<2>(batch, sz, C, D, info, s); break;
	case 3: launch_n8<3>(batch, sz, C, D, info, s); break;
	case 4: launch_n8<4>(batch, sz, C, D, info, s); break;
	case 5: launch_n8<5>(batch, sz, C, D, info, s); break;
	case 6: launch_n8<6>(batch, sz, C, D, info, s); break;
	case 7: launch_n8<7>(batch, sz, C, D, info, s); break;
	case 8: launch_n8<8>(batch, sz, C, D, info, s); break;
	default: return BLASFEO_B200_ENOTSUP;
	}
	return check_launch();
}

}  // namespace bf
