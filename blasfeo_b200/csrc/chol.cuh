// CTA-level Cholesky of a matrix held in shared memory, used by potrf_l and by
// the fused factor+solve kernels.
//
// Shared-memory layout ("lower panels"): the lower triangle of an n x n matrix
// as P = ceil(n/4) row panels; panel p (rows 4p..4p+3) keeps columns
// 0..4p+3, column-major inside the panel (4 consecutive elements per column),
// i.e. the BLASFEO panel layout with everything right of the diagonal tile
// dropped.  Panel p starts at element 8p(p+1); a 4x4 tile and a 4-row column
// slice are contiguous.  Padding rows/columns (n..4P-1) hold the identity so
// they factor to the identity and never touch real entries.
//
// Algorithm: right-looking, 16 columns (4 panels) per block step.
//   1. one warp factors the 16x16 diagonal block in FP64 registers (pivot rule
//      of kernel/generic/kernel_dgemm_4x4_lib4.c:5700-5710: c>0 -> sqrt(c) and
//      its reciprocal, else 0 and 0) and forms the explicit inverse of that
//      block, also in FP64;
//   2. the panel below is solved as a product with that inverse
//      (L_IK = A_IK * inv(L_KK)^T), one thread per row;
//   3. the trailing lower triangle gets the rank-16 update, one 4x4 tile per
//      thread (loads are 16-byte vectors from the contiguous tiles).
// Three __syncthreads per 16 columns.
#pragma once
#include "common.cuh"

#define CHOL_NB 16

__host__ __device__ __forceinline__ int lp_off(int p) { return 8 * p * (p + 1); }
__host__ __device__ __forceinline__ int lp_size(int n) {
	int P = (n + 3) / 4;
	return 8 * P * (P + 1);
}
template <typename T>
__device__ __forceinline__ T &lp_at(T *S, int i, int j) {
	return S[lp_off(i >> 2) + 4 * j + (i & 3)];
}

// 4-element vector type per precision
template <typename T> struct V4;
template <> struct V4<float> { typedef float4 type; };
template <> struct V4<double> { typedef double4 type; };

template <typename T>
__device__ __forceinline__ void ld4(const T *p, T &a, T &b, T &c, T &d);
template <>
__device__ __forceinline__ void ld4<float>(const float *p, float &a, float &b, float &c, float &d) {
	float4 v = *(const float4 *)p;
	a = v.x; b = v.y; c = v.z; d = v.w;
}
template <>
__device__ __forceinline__ void ld4<double>(const double *p, double &a, double &b, double &c, double &d) {
	double2 v0 = *(const double2 *)p, v1 = *(const double2 *)(p + 2);
	a = v0.x; b = v0.y; c = v1.x; d = v1.y;
}
template <typename T>
__device__ __forceinline__ void st4(T *p, T a, T b, T c, T d);
template <>
__device__ __forceinline__ void st4<float>(float *p, float a, float b, float c, float d) {
	*(float4 *)p = make_float4(a, b, c, d);
}
template <>
__device__ __forceinline__ void st4<double>(double *p, double a, double b, double c, double d) {
	*(double2 *)p = make_double2(a, b);
	*(double2 *)(p + 2) = make_double2(c, d);
}

// map a linear index over the lower-triangular tile set {(ti,tj): 0<=tj<=ti<R}
__device__ __forceinline__ void tri_index(int t, int &ti, int &tj) {
	int r = (int)((sqrtf(8.0f * (float)t + 1.0f) - 1.0f) * 0.5f);
	while ((r + 1) * (r + 2) / 2 <= t) r++;
	while (r * (r + 1) / 2 > t) r--;
	ti = r;
	tj = t - r * (r + 1) / 2;
}

// Factor the 16x16 diagonal block at column c0 (nbk <= 16 real columns) with
// warp 0.  Writes L_KK back into S (type T), 1/L_jj into dinv[c0+j] (FP64 in
// shared memory), the explicit inverse of L_KK (row-major 16x16, FP64 math,
// stored as T) into invL, and the first bad pivot (j+1) into *bad.
template <typename T>
__device__ void chol_diag_block(T *S, int c0, int nbk, double *dinv, T *invL, double *scratch, int *bad) {
	const int lane = threadIdx.x & 31;
	// lane i (< 16) holds row c0+i of the block in FP64
	double v[CHOL_NB];
#pragma unroll
	for (int l = 0; l < CHOL_NB; l++) {
		double x = 0.0;
		if (lane < CHOL_NB && l <= lane) {
			if (lane < nbk && l < nbk)
				x = (double)lp_at(S, c0 + lane, c0 + l);
			else if (l == lane)
				x = 1.0;
		}
		v[l] = x;
	}
#pragma unroll
	for (int j = 0; j < CHOL_NB; j++) {
		double d = 0.0, inv = 0.0;
		if (lane == j) {
			chol_pivot(v[j], d, inv);
			if (!(v[j] > 0.0) && j < nbk && *bad == 0) *bad = c0 + j + 1;
			v[j] = d;
		}
		inv = __shfl_sync(0xffffffffu, inv, j);
		if (lane > j) v[j] *= inv;
		if (lane == j && j < nbk) dinv[c0 + j] = inv;
#pragma unroll
		for (int l = j + 1; l < CHOL_NB; l++) {
			double t = __shfl_sync(0xffffffffu, v[j], l);
			if (lane >= l) v[l] = fma(-v[j], t, v[l]);
		}
	}
	// L_KK -> scratch (FP64, row-major 16x17, column 16 = inverse pivot) and back into S
	if (lane < CHOL_NB) {
		double dd = 0.0;
#pragma unroll
		for (int l = 0; l < CHOL_NB; l++)
			if (l == lane) dd = v[l];
		scratch[lane * 17 + 16] = (dd != 0.0) ? 1.0 / dd : 0.0;
#pragma unroll
		for (int l = 0; l < CHOL_NB; l++) scratch[lane * 17 + l] = (l <= lane) ? v[l] : 0.0;
		if (lane < nbk) {
#pragma unroll
			for (int l = 0; l < CHOL_NB; l++)
				if (l <= lane && l < nbk) lp_at(S, c0 + lane, c0 + l) = (T)v[l];
		}
	}
	__syncwarp();
	// explicit inverse: lane c computes column c of inv(L_KK) by forward substitution
	if (lane < CHOL_NB) {
		const int c = lane;
		double x[CHOL_NB];
#pragma unroll
		for (int i = 0; i < CHOL_NB; i++) {
			double s = (i == c) ? 1.0 : 0.0;
#pragma unroll
			for (int l = 0; l < i; l++) s = fma(-scratch[i * 17 + l], x[l], s);
			x[i] = (i < c) ? 0.0 : s * scratch[i * 17 + 16];
		}
#pragma unroll
		for (int i = 0; i < CHOL_NB; i++) invL[i * CHOL_NB + c] = (T)x[i];
	}
}

// Full factorization of the n x n lower-panel matrix S by the whole CTA.
// dinv: FP64 shared array of >= 4P entries; invL_all: per block step 256
// entries (row-major inverse of each diagonal block; pass stride 0 to reuse
// one 256-entry buffer); scratch: 16*17 doubles; bad: shared int (0 on entry).
template <typename T>
__device__ void chol_smem(T *S, int n, double *dinv, T *invL_all, int invL_stride, double *scratch, int *bad) {
	const int P = (n + 3) >> 2;
	const int tid = threadIdx.x, nt = blockDim.x;
	for (int k0 = 0; k0 < P; k0 += 4) {
		const int c0 = 4 * k0;
		const int nbk = min(CHOL_NB, n - c0);
		T *invL = invL_all + (size_t)(k0 >> 2) * invL_stride;
		if (tid < 32) chol_diag_block<T>(S, c0, nbk, dinv, invL, scratch, bad);
		__syncthreads();
		// panel: rows r in [c0+16, 4P) : L[r][c0..c0+15] = A[r][c0..] * invL^T
		const int r0 = c0 + CHOL_NB;
		const int nrow = 4 * P - r0;
		for (int t = tid; t < nrow; t += nt) {
			const int r = r0 + t;
			T a[CHOL_NB];
#pragma unroll
			for (int l = 0; l < CHOL_NB; l++) a[l] = lp_at(S, r, c0 + l);
#pragma unroll
			for (int c = 0; c < CHOL_NB; c++) {
				T s = T(0);
#pragma unroll
				for (int l = 0; l <= c; l++) s = fma(a[l], invL[c * CHOL_NB + l], s);
				lp_at(S, r, c0 + c) = s;
			}
		}
		__syncthreads();
		// trailing update of tiles (ti,tj), k0+4 <= tj <= ti < P
		const int R = P - (k0 + 4);
		if (R > 0) {
			const int ntiles = R * (R + 1) / 2;
			for (int t = tid; t < ntiles; t += nt) {
				int ti, tj;
				tri_index(t, ti, tj);
				ti += k0 + 4;
				tj += k0 + 4;
				T *tile = S + lp_off(ti) + 16 * tj;
				T acc[16];
#pragma unroll
				for (int q = 0; q < 4; q++) ld4<T>(tile + 4 * q, acc[4 * q], acc[4 * q + 1], acc[4 * q + 2], acc[4 * q + 3]);
				const T *li = S + lp_off(ti) + 4 * c0;
				const T *lj = S + lp_off(tj) + 4 * c0;
#pragma unroll 4
				for (int c = 0; c < CHOL_NB; c++) {
					T a0, a1, a2, a3, b0, b1, b2, b3;
					ld4<T>(li + 4 * c, a0, a1, a2, a3);
					ld4<T>(lj + 4 * c, b0, b1, b2, b3);
					// acc[4*q + r] is element (row r of ti, column q of tj)
					acc[0] = fma(-a0, b0, acc[0]); acc[1] = fma(-a1, b0, acc[1]);
					acc[2] = fma(-a2, b0, acc[2]); acc[3] = fma(-a3, b0, acc[3]);
					acc[4] = fma(-a0, b1, acc[4]); acc[5] = fma(-a1, b1, acc[5]);
					acc[6] = fma(-a2, b1, acc[6]); acc[7] = fma(-a3, b1, acc[7]);
					acc[8] = fma(-a0, b2, acc[8]); acc[9] = fma(-a1, b2, acc[9]);
					acc[10] = fma(-a2, b2, acc[10]); acc[11] = fma(-a3, b2, acc[11]);
					acc[12] = fma(-a0, b3, acc[12]); acc[13] = fma(-a1, b3, acc[13]);
					acc[14] = fma(-a2, b3, acc[14]); acc[15] = fma(-a3, b3, acc[15]);
				}
#pragma unroll
				for (int q = 0; q < 4; q++) st4<T>(tile + 4 * q, acc[4 * q], acc[4 * q + 1], acc[4 * q + 2], acc[4 * q + 3]);
			}
		}
		__syncthreads();
	}
}
