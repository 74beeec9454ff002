// FP64 Cholesky of one matrix per CTA whose lower triangle does not fit in
// shared memory (the reference's dpotrf_l, blasfeo_hp_pm/d_lapack_lib4.c:918,
// for n beyond the shared-memory kernels), and the two triangular solves of
// the factor+solve chain (dtrsv_lnn / dtrsv_ltn) on the result.
//
// Left-looking by 16-column panels K (columns c0 = 16K .. c0+15):
//   update:  the panel (rows c0..n-1) starts from C and receives
//            -L(rows, 0:c0) L(c0:c0+16, 0:c0)^T on the FP64 tensor cores
//            (DMMA m8n8k4; every warp owns 8-row fragment rows, the operand
//            fragments are read from the factored columns in global memory --
//            two 128-byte runs each in the panel layout, L2-resident while the
//            CTA works on the matrix);
//   factor:  warp 0 factors the 16 x 16 diagonal block in FP64 registers
//            (DiagCol of chol.cuh: pivot rule of
//            kernel/generic/kernel_dgemm_4x4_lib4.c:5700-5710), the rows below
//            solve their 16 entries against it (one thread per row,
//            reciprocal-pivot multiply);
//   store:   the finished panel goes to D once, 1/L_jj to D's dA.
// Every element of L is written once and read back only by later panels'
// updates, so D may alias C.  Rows and columns n..16*ceil(n/16)-1 act as the
// identity.
#pragma once
#include "chol.cuh"
#include "common.cuh"

constexpr int LL_PSTR = 17;  // shared-memory panel row stride (doubles)

// shared memory of chol_ll for matrices up to max_n: the panel, the 16x17
// diagonal factor with its reciprocal pivots
__host__ __device__ inline size_t ll_smem_bytes(int max_n) {
	return ((size_t)(max_n + 8) * LL_PSTR + 16 * 17) * sizeof(double);
}

__device__ __forceinline__ void ll_dmma(double &d0, double &d1, double a, double b) {
	asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
	             : "+d"(d0), "+d"(d1)
	             : "d"(a), "d"(b));
}

// L(i, k) of the factored columns, 0 for rows beyond n
__device__ __forceinline__ double ll_ld(const PMat<double> &d, int i, int k, int n) {
	return i < n ? *d.addr(i, k) : 0.0;
}

// Factor the n x n lower triangle of c into d (lower triangle of L, 1/L_jj in
// d.d[j]); *bad (shared, zeroed by the caller) receives the first
// non-positive pivot j+1.  All NT threads of the CTA call it.  FR: fragment
// rows a warp updates at a time (its accumulators: 8 FR doubles per lane).
template <int NT, int FR = 4>
__device__ void chol_ll(const PMat<double> &c, const PMat<double> &d, int n, double *smem, int *bad) {
	constexpr int NW = NT / 32;
	double *pan = smem;
	double *Lt = smem + (size_t)(n + 8) * LL_PSTR;
	const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
	const int r = lane >> 2, q = lane & 3;
	const int NBK = (n + 15) >> 4;
	for (int K = 0; K < NBK; K++) {
		const int c0 = 16 * K;
		const int m = n - c0;
		const int R = (m + 7) >> 3;
		// ---- panel update: up to FR fragment rows per warp at a time ----
		for (int f0 = warp; f0 < R; f0 += FR * NW) {
			double acc[FR][2][2];
#pragma unroll
			for (int u = 0; u < FR; u++) {
				const int row = c0 + 8 * (f0 + u * NW) + r;
#pragma unroll
				for (int fc = 0; fc < 2; fc++)
#pragma unroll
					for (int h = 0; h < 2; h++) {
						const int col = c0 + 8 * fc + 2 * q + h;
						double v = 0.0;
						if (f0 + u * NW < R) {
							if (row < n && col < n)
								v = (col <= row) ? -*c.addr(row, col) : 0.0;
							else
								v = (row == col) ? -1.0 : 0.0;
						}
						acc[u][fc][h] = v;
					}
			}
#pragma unroll 2
			for (int k = 0; k < c0; k += 8) {
				double a0[FR], a1[FR];
				const double b00 = ll_ld(d, c0 + r, k + q, n), b01 = ll_ld(d, c0 + 8 + r, k + q, n);
				const double b10 = ll_ld(d, c0 + r, k + 4 + q, n), b11 = ll_ld(d, c0 + 8 + r, k + 4 + q, n);
#pragma unroll
				for (int u = 0; u < FR; u++) {
					const int row = c0 + 8 * (f0 + u * NW) + r;
					const bool act = f0 + u * NW < R;
					a0[u] = act ? ll_ld(d, row, k + q, n) : 0.0;
					a1[u] = act ? ll_ld(d, row, k + 4 + q, n) : 0.0;
				}
#pragma unroll
				for (int u = 0; u < FR; u++) {
					if (f0 + u * NW < R) {  // warp-uniform
						ll_dmma(acc[u][0][0], acc[u][0][1], a0[u], b00);
						ll_dmma(acc[u][1][0], acc[u][1][1], a0[u], b01);
						ll_dmma(acc[u][0][0], acc[u][0][1], a1[u], b10);
						ll_dmma(acc[u][1][0], acc[u][1][1], a1[u], b11);
					}
				}
			}
#pragma unroll
			for (int u = 0; u < FR; u++) {
				const int pr = 8 * (f0 + u * NW) + r;  // panel row
				if (f0 + u * NW < R) {
#pragma unroll
					for (int fc = 0; fc < 2; fc++)
#pragma unroll
						for (int h = 0; h < 2; h++) pan[pr * LL_PSTR + 8 * fc + 2 * q + h] = -acc[u][fc][h];
				}
			}
		}
		__syncthreads();
		// ---- diagonal block (warp 0, FP64 registers) ----
		const int nbk = m < 16 ? m : 16;
		if (warp == 0) {
			double rv[CHOL_NB];
#pragma unroll
			for (int l = 0; l < CHOL_NB; l++) rv[l] = (lane < CHOL_NB && l <= lane) ? pan[lane * LL_PSTR + l] : 0.0;
			DiagCol<0, double>::run(rv, lane, nbk, c0, d.d, bad);
			if (lane < CHOL_NB) {
#pragma unroll
				for (int l = 0; l < CHOL_NB; l++) Lt[lane * 17 + l] = (l <= lane) ? rv[l] : 0.0;
				// the lane that computed pivot `lane` wrote d.d[c0 + lane]
				Lt[lane * 17 + 16] = (lane < nbk) ? d.d[c0 + lane] : 1.0;
			}
		}
		__syncthreads();
		// ---- rows below the diagonal block: x = a L_KK^{-T} ----
		for (int i = 16 + tid; i < m; i += NT) {
			double x[16];
#pragma unroll
			for (int cc = 0; cc < 16; cc++) x[cc] = pan[i * LL_PSTR + cc];
#pragma unroll
			for (int cc = 0; cc < 16; cc++) {
				double s = x[cc];
#pragma unroll
				for (int l = 0; l < cc; l++) s = fma(-x[l], Lt[cc * 17 + l], s);
				x[cc] = s * Lt[cc * 17 + 16];
			}
#pragma unroll
			for (int cc = 0; cc < 16; cc++) pan[i * LL_PSTR + cc] = x[cc];
		}
		__syncthreads();
		// ---- store the panel: 4-row x 16-column runs of the panel layout ----
		for (int e = tid; e < 16 * ((m + 3) & ~3); e += NT) {
			const int p = e >> 6, w = e & 63;
			const int i = 4 * p + (w & 3), j = w >> 2;  // panel-relative row, column
			const int gi = c0 + i, gj = c0 + j;
			if (gi < n && gj < n && (i >= 16 || j <= i))
				*d.addr(gi, gj) = (i < 16) ? Lt[i * 17 + j] : pan[i * LL_PSTR + j];
		}
		__syncthreads();
	}
}

// y := L^{-1} y and y := L^{-T} y for the factor in d (global memory), y in
// shared memory (n doubles); one thread per row, 16-row blocks solved by warp
// 0 with shuffles (reciprocal pivots from d.d).
template <int NT>
__device__ void trsv_ll_fwd(const PMat<double> &d, int n, double *y) {
	const int tid = threadIdx.x, lane = tid & 31;
	for (int c0 = 0; c0 < n; c0 += 16) {
		const int nbk = n - c0 < 16 ? n - c0 : 16;
		if (tid < 32) {
			double v = (lane < nbk) ? y[c0 + lane] : 0.0;
			for (int k = 0; k < nbk; k++) {
				const double yk = __shfl_sync(0xffffffffu, v, k) * d.d[c0 + k];
				if (lane == k) v = yk;
				if (lane > k && lane < nbk) v = fma(-*d.addr(c0 + lane, c0 + k), yk, v);
			}
			if (lane < nbk) y[c0 + lane] = v;
		}
		__syncthreads();
		for (int i = c0 + 16 + tid; i < n; i += NT) {
			double s = y[i];
			for (int k = 0; k < nbk; k++) s = fma(-*d.addr(i, c0 + k), y[c0 + k], s);
			y[i] = s;
		}
		__syncthreads();
	}
}

template <int NT>
__device__ void trsv_ll_bwd(const PMat<double> &d, int n, double *y) {
	const int tid = threadIdx.x, lane = tid & 31;
	for (int c0 = (n - 1) & ~15; c0 >= 0; c0 -= 16) {
		const int nbk = n - c0 < 16 ? n - c0 : 16;
		if (tid < 32) {
			double v = (lane < nbk) ? y[c0 + lane] : 0.0;
			for (int k = nbk - 1; k >= 0; k--) {
				const double xk = __shfl_sync(0xffffffffu, v, k) * d.d[c0 + k];
				if (lane == k) v = xk;
				if (lane < k) v = fma(-*d.addr(c0 + k, c0 + lane), xk, v);
			}
			if (lane < nbk) y[c0 + lane] = v;
		}
		__syncthreads();
		for (int j = tid; j < c0; j += NT) {
			double s = y[j];
			for (int k = 0; k < nbk; k++) s = fma(-*d.addr(c0 + k, j), y[c0 + k], s);
			y[j] = s;
		}
		__syncthreads();
	}
}
