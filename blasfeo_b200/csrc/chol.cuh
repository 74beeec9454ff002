// CTA-level Cholesky of a matrix held in shared memory, used by potrf_l and by
// the fused factor+solve kernels.
//
// Shared-memory layout ("lower panels"): the lower triangle of an n x n matrix
// as P = ceil(n/4) row panels; panel p (rows 4p..4p+3) keeps the 4x4 tiles
// 0..p, i.e. the BLASFEO panel layout with everything right of the diagonal
// tile dropped.  Panel p starts at element 8p(p+1); tile (p,q) is 16
// contiguous elements, column-major inside the tile.  Inside a tile the
// 16-byte chunks are XOR-swizzled with (p+q): threads that read different
// tiles of one tile row or one tile column then hit different banks (every
// tile starts on a 128-byte (FP64) / 64-byte (FP32) boundary, so without the
// swizzle all of them would collide on the same banks).
// Padding rows/columns (n..4P-1) hold the identity so they factor to the
// identity and never touch real entries.
//
// Algorithm: right-looking, 16 columns (4 panels) per block step, two
// __syncthreads per step:
//   A. all threads: panel of block column K by substitution with the
//      factored diagonal block (one row per thread, the reciprocal pivots
//      multiplied in);
//   B. warp 0 (critical path): rank-16 update of the 16x16 diagonal block K+1
//      and its factorization in FP64 registers (pivot rule of
//      kernel/generic/kernel_dgemm_4x4_lib4.c:5700-5710: c>0 -> sqrt(c) and its
//      reciprocal, else 0 and 0); the warps on the other three schedulers:
//      rank-16 update of the rest of the trailing matrix (8 x 4 tile blocks
//      per warp), which hides the serial diagonal work.
// With inv_diag the diagonal blocks are replaced at the end by their explicit
// inverses (FP64 arithmetic, all blocks in parallel) for the blocked
// triangular solves of the factor+solve kernels.
#pragma once
#include "common.cuh"

#define CHOL_NB 16

__host__ __device__ __forceinline__ int lp_off(int p) { return 8 * p * (p + 1); }
__host__ __device__ __forceinline__ int lp_size(int n) {
	int P = (n + 3) / 4;
	return 8 * P * (P + 1);
}

// physical index of element (i,j) (j <= 4*(i/4)+3) in the swizzled lower panels
template <typename T>
__device__ __forceinline__ int lp_idx(int i, int j);
template <>
__device__ __forceinline__ int lp_idx<double>(int i, int j) {
	const int p = i >> 2, q = j >> 2;
	const int e = ((j & 3) << 2) | (i & 3);
	return lp_off(p) + 16 * q + ((((e >> 1) ^ ((p + q) & 7)) << 1) | (e & 1));
}
template <>
__device__ __forceinline__ int lp_idx<float>(int i, int j) {
	const int p = i >> 2, q = j >> 2;
	return lp_off(p) + 16 * q + ((((j & 3) ^ ((p + q) & 3)) << 2) | (i & 3));
}
template <typename T>
__device__ __forceinline__ T &lp_at(T *S, int i, int j) {
	return S[lp_idx<T>(i, j)];
}
template <typename T>
__device__ __forceinline__ const T &lp_at(const T *S, int i, int j) {
	return S[lp_idx<T>(i, j)];
}

// column c (0..3) of tile (p,q): the 4 rows as a, b, c, d
template <typename T>
__device__ __forceinline__ void tile_col_ld(const T *S, int p, int q, int c, T &a0, T &a1, T &a2, T &a3);
template <>
__device__ __forceinline__ void tile_col_ld<double>(const double *S, int p, int q, int c, double &a0, double &a1,
                                                    double &a2, double &a3) {
	const double *t = S + lp_off(p) + 16 * q;
	const int s = (p + q) & 7;
	double2 v0 = *(const double2 *)(t + (((2 * c) ^ s) << 1));
	double2 v1 = *(const double2 *)(t + (((2 * c + 1) ^ s) << 1));
	a0 = v0.x; a1 = v0.y; a2 = v1.x; a3 = v1.y;
}
template <>
__device__ __forceinline__ void tile_col_ld<float>(const float *S, int p, int q, int c, float &a0, float &a1,
                                                   float &a2, float &a3) {
	const float *t = S + lp_off(p) + 16 * q;
	float4 v = *(const float4 *)(t + ((c ^ ((p + q) & 3)) << 2));
	a0 = v.x; a1 = v.y; a2 = v.z; a3 = v.w;
}
template <typename T>
__device__ __forceinline__ void tile_col_st(T *S, int p, int q, int c, T a0, T a1, T a2, T a3);
template <>
__device__ __forceinline__ void tile_col_st<double>(double *S, int p, int q, int c, double a0, double a1, double a2,
                                                    double a3) {
	double *t = S + lp_off(p) + 16 * q;
	const int s = (p + q) & 7;
	*(double2 *)(t + (((2 * c) ^ s) << 1)) = make_double2(a0, a1);
	*(double2 *)(t + (((2 * c + 1) ^ s) << 1)) = make_double2(a2, a3);
}
template <>
__device__ __forceinline__ void tile_col_st<float>(float *S, int p, int q, int c, float a0, float a1, float a2,
                                                   float a3) {
	float *t = S + lp_off(p) + 16 * q;
	*(float4 *)(t + ((c ^ ((p + q) & 3)) << 2)) = make_float4(a0, a1, a2, a3);
}

// map a linear index over the lower-triangular tile set {(ti,tj): 0<=tj<=ti<R}
__device__ __forceinline__ void tri_index(int t, int &ti, int &tj) {
	int r = (int)((sqrtf(8.0f * (float)t + 1.0f) - 1.0f) * 0.5f);
	while ((r + 1) * (r + 2) / 2 <= t) r++;
	while (r * (r + 1) / 2 > t) r--;
	ti = r;
	tj = t - r * (r + 1) / 2;
}

// Cholesky pivot through one reciprocal square root: inv = 1/sqrt(c),
// d = c*inv (= sqrt(c)); non-positive c -> 0, 0.
__device__ __forceinline__ void chol_pivot_rsqrt(double c, double &d, double &inv) {
	if (c > 0.0) {
		inv = rsqrt(c);
		d = c * inv;
	} else {
		d = 0.0;
		inv = 0.0;
	}
}

// One column J of the 16x16 diagonal-block factorization; lane i holds row i
// of the block in r[] (compile-time indices only, so r stays in registers).
// The pivot is broadcast by a shuffle and every lane computes its reciprocal
// square root in FP64 (T = float: FP32 entries and updates, FP64 pivots);
// column J reaches the other rows by shuffles.  The pivot rule is applied
// without branches so the compiler can overlap the column update with the
// next pivot.  The terminal step records the first non-positive pivot
// (c0 + j + 1) in *bad by one ballot over the rows.
// WIDTH = 16 factors two independent blocks per warp, one per half-warp:
// `lane` is then the lane within the half (0..15), the shuffles stay inside
// the half, and each half records its own dinv / bad (the caller passes the
// half's pointers).  The whole warp executes the call.
template <int J, typename T = double, int WIDTH = 32>
struct DiagCol {
	static __device__ __forceinline__ void run(T (&r)[CHOL_NB], int lane, int nbk, int c0, double *dinv, int *bad) {
		const double cj = (double)__shfl_sync(0xffffffffu, r[J], J, WIDTH);
		const bool ok = cj > 0.0;
		const double inv = ok ? rsqrt(cj) : 0.0;
		r[J] = (lane == J) ? (T)(ok ? cj * inv : 0.0) : r[J] * (T)inv;
		if (lane == J && J < nbk) dinv[c0 + J] = inv;
#pragma unroll
		for (int l = J + 1; l < CHOL_NB; l++) {
			const T t = __shfl_sync(0xffffffffu, r[J], l, WIDTH);
			if (lane >= l) r[l] = fma(-r[J], t, r[l]);
		}
		DiagCol<J + 1, T, WIDTH>::run(r, lane, nbk, c0, dinv, bad);
	}
};
template <typename T, int WIDTH>
struct DiagCol<CHOL_NB, T, WIDTH> {
	static __device__ __forceinline__ void run(T (&r)[CHOL_NB], int lane, int nbk, int c0, double *, int *bad) {
		T d = T(1);
#pragma unroll
		for (int l = 0; l < CHOL_NB; l++)
			if (l == lane) d = r[l];
		unsigned m = __ballot_sync(0xffffffffu, lane < nbk && !(d > T(0)));
		if (WIDTH == 16) m = (m >> (threadIdx.x & 16)) & 0xffffu;  // this half-warp's rows
		if (m && lane == 0 && *bad == 0) *bad = c0 + __ffs(m);
	}
};

// FP32 data: the 16 x 16 lower block, staged row-major in blk (16 rows of 17),
// is factored by every lane of the warp at once, each holding the whole lower
// triangle in registers, so the pivot chain issues no shuffles: under the
// trailing update of the other warps, which keeps the shared-memory / shuffle
// unit busy, each of the 16 pivot steps of DiagCol waited for that unit
// several times (clock64 probe of the n = 256 solver: 11.7k cycles per block).
// Same operations in the same order as DiagCol (pivot rule of
// kernel/generic/kernel_dgemm_4x4_lib4.c:5700-5710 with FP64 pivots and
// reciprocals, column scaling, then the rank-1 update of the trailing columns
// in column order), so the factor is bitwise the same.  Lane i < 16 receives
// row i of L in r; lane i < nbk writes dinv[c0 + i]; the first non-positive
// pivot (c0 + j + 1) goes to *bad.
template <typename T>
__device__ __forceinline__ void diag_factor_rep(const T *blk, int nbk, int c0, double *dinv, int *bad,
                                                T (&r)[CHOL_NB], int lane) {
	T a[CHOL_NB * (CHOL_NB + 1) / 2];  // packed lower triangle, (i, j) at i (i + 1) / 2 + j
#pragma unroll
	for (int i = 0; i < CHOL_NB; i++)
#pragma unroll
		for (int j = 0; j <= i; j++) a[i * (i + 1) / 2 + j] = blk[i * 17 + j];
	double inv_all[CHOL_NB];
	int first_bad = 0;
#pragma unroll
	for (int J = 0; J < CHOL_NB; J++) {
		const double cj = (double)a[J * (J + 1) / 2 + J];
		const bool ok = cj > 0.0;
		const double inv = ok ? rsqrt(cj) : 0.0;
		inv_all[J] = inv;
		if (!ok && J < nbk && first_bad == 0) first_bad = J + 1;
		a[J * (J + 1) / 2 + J] = (T)(ok ? cj * inv : 0.0);
#pragma unroll
		for (int i = J + 1; i < CHOL_NB; i++) a[i * (i + 1) / 2 + J] = a[i * (i + 1) / 2 + J] * (T)inv;
#pragma unroll
		for (int l = J + 1; l < CHOL_NB; l++)
#pragma unroll
			for (int i = l; i < CHOL_NB; i++)
				a[i * (i + 1) / 2 + l] = fma(-a[i * (i + 1) / 2 + J], a[l * (l + 1) / 2 + J], a[i * (i + 1) / 2 + l]);
	}
#pragma unroll
	for (int l = 0; l < CHOL_NB; l++) r[l] = T(0);
#pragma unroll
	for (int i = 0; i < CHOL_NB; i++)
		if (lane == i) {
#pragma unroll
			for (int l = 0; l <= i; l++) r[l] = a[i * (i + 1) / 2 + l];
			if (i < nbk) dinv[c0 + i] = inv_all[i];
		}
	if (lane == 0 && first_bad && *bad == 0) *bad = c0 + first_bad;
}

// Write the factored diagonal block (lane i: row i in r) back into S and into
// the row-major Lt (reciprocal pivots, from the FP64 dinv, in column 16).
template <typename T>
__device__ __forceinline__ void chol_diag_store(T *S, int c0, int nbk, const double *dinv, T *Lt, const T (&r)[CHOL_NB],
                                                int lane) {
	if (lane < CHOL_NB) {
#pragma unroll
		for (int l = 0; l < CHOL_NB; l++) Lt[lane * 17 + l] = (l <= lane) ? r[l] : T(0);
		if (lane < nbk) {
#pragma unroll
			for (int l = 0; l < CHOL_NB; l++)
				if (l <= lane) lp_at(S, c0 + lane, c0 + l) = r[l];
		}
	}
	__syncwarp();
	if (lane < CHOL_NB) Lt[lane * 17 + 16] = (lane < nbk) ? (T)dinv[c0 + lane] : T(1);
	__syncwarp();
}

// Warp 0: factor the diagonal block at column c0 (nbk <= 16 real columns; the
// padding is the identity) in FP64 registers; write L_KK back into S, 1/L_jj
// into dinv[c0+j] (FP64), the first bad pivot (j+1) into *bad, and for the
// panel solve a row-major 16x17 copy Lt of L_KK in the working precision with
// the reciprocal pivots in column 16.
template <typename T, bool REP = false>
__device__ void chol_diag_factor(T *S, int c0, int nbk, double *dinv, T *Lt, int *bad) {
	const int lane = threadIdx.x & 31;
	T r[CHOL_NB];
#pragma unroll
	for (int l = 0; l < CHOL_NB; l++) {
		T x = T(0);
		if (lane < CHOL_NB && l <= lane) {
			if (lane < nbk && l < nbk)
				x = lp_at(S, c0 + lane, c0 + l);
			else if (l == lane)
				x = T(1);
		}
		r[l] = x;
	}
	if constexpr (REP && sizeof(T) == 4) {
		if (lane < CHOL_NB) {
#pragma unroll
			for (int l = 0; l < CHOL_NB; l++) Lt[lane * 17 + l] = r[l];
		}
		__syncwarp();
		diag_factor_rep<T>(Lt, nbk, c0, dinv, bad, r, lane);
		__syncwarp();  // every lane has read the staged block before it is overwritten
	} else {
		DiagCol<0, T>::run(r, lane, nbk, c0, dinv, bad);
	}
	chol_diag_store<T>(S, c0, nbk, dinv, Lt, r, lane);
}

// Warp 0, look-ahead step: the rank-16 update of diagonal block K+1 (columns
// c0n..c0n+15) with the panel of block column K (columns c0..c0+15, already
// solved), fused with its factorization.  Lane i (and lane i+16) own row i of
// the block; the two half-warps take 8 of the 16 panel columns each, reading
// the panel rows of the block as broadcast tile-column loads, and their
// partial sums meet by one shuffle.  The update runs in the working precision
// T, the factorization in FP64 registers (DiagCol).  Outputs as
// chol_diag_factor.
template <typename T, bool REP = false>
__device__ void chol_diag_update_factor(T *S, int c0n, int nbk, int c0, double *dinv, T *Lt, int *bad) {
	const int lane = threadIdx.x & 31;
	const int i = lane & 15, h = lane >> 4;
	const int pn = c0n >> 2, kb = c0 >> 2;
	T u[CHOL_NB];
#pragma unroll
	for (int l = 0; l < CHOL_NB; l++) u[l] = (h == 0 && l <= i && i < nbk && l < nbk) ? lp_at(S, c0n + i, c0n + l) : T(0);
	// row i of the panel block, the half-warp's 8 columns
	T pr[8];
#pragma unroll
	for (int l = 0; l < 8; l++) pr[l] = (i < nbk) ? lp_at(S, c0n + i, c0 + 8 * h + l) : T(0);
#pragma unroll
	for (int jq = 0; jq < 4; jq++) {
		if (4 * jq >= nbk) break;  // row panels past the end of the matrix
#pragma unroll
		for (int l = 0; l < 8; l++) {
			const int col = 8 * h + l;
			T v0, v1, v2, v3;
			tile_col_ld<T>(S, pn + jq, kb + (col >> 2), col & 3, v0, v1, v2, v3);
			u[4 * jq] = fma(-pr[l], v0, u[4 * jq]);
			u[4 * jq + 1] = fma(-pr[l], v1, u[4 * jq + 1]);
			u[4 * jq + 2] = fma(-pr[l], v2, u[4 * jq + 2]);
			u[4 * jq + 3] = fma(-pr[l], v3, u[4 * jq + 3]);
		}
	}
	T r[CHOL_NB];
#pragma unroll
	for (int l = 0; l < CHOL_NB; l++) {
		const T s = u[l] + __shfl_xor_sync(0xffffffffu, u[l], 16);
		// real entries of the lower triangle; identity in the padding
		r[l] = (l <= i && i < nbk && l < nbk) ? s : ((l == i && i >= nbk) ? T(1) : T(0));
	}
	if constexpr (REP && sizeof(T) == 4) {
		if (lane < CHOL_NB) {
#pragma unroll
			for (int l = 0; l < CHOL_NB; l++) Lt[lane * 17 + l] = r[l];
		}
		__syncwarp();
		diag_factor_rep<T>(Lt, nbk, c0n, dinv, bad, r, lane);
		__syncwarp();  // every lane has read the staged block before it is overwritten
	} else {
		DiagCol<0, T>::run(r, lane, nbk, c0n, dinv, bad);
	}
	chol_diag_store<T>(S, c0n, nbk, dinv, Lt, r, lane);
}

// panel of block column c0, rows r in [rbeg, rend): substitution with the
// diagonal block, L[r][c0+c] = (A[r][c0+c] - sum_{l<c} L[r][c0+l] L_KK[c][l]) * inv_c
template <typename T>
__device__ __forceinline__ void chol_panel_rows(T *S, int c0, int rbeg, int rend, int tid0, int nthr, const T *Lt) {
	const int kb = c0 >> 2;
	for (int r = rbeg + tid0; r < rend; r += nthr) {
		const int p = r >> 2, ri = r & 3;
		T *row = S + lp_off(p) + 16 * kb;
		int idx[CHOL_NB];
#pragma unroll
		for (int l = 0; l < CHOL_NB; l++) {
			const int qq = l >> 2, e = ((l & 3) << 2) | ri;
			idx[l] = 16 * qq + (sizeof(T) == 4 ? ((((l & 3) ^ ((p + kb + qq) & 3)) << 2) | ri)
			                                   : ((((e >> 1) ^ ((p + kb + qq) & 7)) << 1) | (e & 1)));
		}
		T a[CHOL_NB];
#pragma unroll
		for (int l = 0; l < CHOL_NB; l++) a[l] = row[idx[l]];
#pragma unroll
		for (int c = 0; c < CHOL_NB; c++) {
			T s = a[c];
#pragma unroll
			for (int l = 0; l < c; l++) s = fma(-a[l], Lt[c * 17 + l], s);
			a[c] = s * Lt[c * 17 + 16];
		}
#pragma unroll
		for (int l = 0; l < CHOL_NB; l++) row[idx[l]] = a[l];
	}
}

// Explicit inverse of diagonal block K (row-major 16x16, stored as T) from the
// factor in S and the FP64 reciprocal pivots; lane c computes column c.
template <typename T>
__device__ void chol_block_inverse(const T *S, int n, int K, const double *dinv, T *invL, int lane) {
	const int c0 = 16 * K;
	const int nbk = min(CHOL_NB, n - c0);
	const int c = lane;
	if (c >= CHOL_NB) return;
	double x[CHOL_NB];
#pragma unroll
	for (int i = 0; i < CHOL_NB; i++) {
		double s = (i == c) ? 1.0 : 0.0;
#pragma unroll
		for (int l = 0; l < i; l++) {
			const double lil = (i < nbk && l < nbk) ? (double)lp_at(S, c0 + i, c0 + l) : 0.0;
			s = fma(-lil, x[l], s);
		}
		const double di = (i < nbk) ? dinv[c0 + i] : 1.0;
		x[i] = (i < c) ? 0.0 : s * di;
	}
#pragma unroll
	for (int i = 0; i < CHOL_NB; i++) invL[i * CHOL_NB + c] = (T)x[i];
}

// Diagonal block K of the factor in S replaced by its inverse (lower
// triangular, same tiles, working precision), from the factor in S and the
// FP64 reciprocal pivots; lane c computes column c.  Only the real rows and
// columns (< n) are written; the whole warp calls it.
template <typename T>
__device__ void chol_block_inverse_inplace(T *S, int n, int K, const double *dinv, int lane) {
	const int c0 = 16 * K;
	const int nbk = min(CHOL_NB, n - c0);
	const int c = lane & 15;
	double x[CHOL_NB];
#pragma unroll
	for (int i = 0; i < CHOL_NB; i++) {
		double s = (i == c) ? 1.0 : 0.0;
#pragma unroll
		for (int l = 0; l < i; l++) {
			const double lil = (i < nbk && l < nbk) ? (double)lp_at(S, c0 + i, c0 + l) : 0.0;
			s = fma(-lil, x[l], s);
		}
		const double di = (i < nbk) ? dinv[c0 + i] : 1.0;
		x[i] = (i < c) ? 0.0 : s * di;
	}
	__syncwarp();  // every lane has read the block before any lane overwrites it
	if (lane < CHOL_NB && c < nbk) {
#pragma unroll
		for (int i = 0; i < CHOL_NB; i++)
			if (i >= c && i < nbk) lp_at(S, c0 + i, c0 + c) = (T)x[i];
	}
	__syncwarp();
}

// rank-16 update of tile (ti,tj) with the panel at block column c0
template <typename T>
__device__ __forceinline__ void chol_tile_update(T *S, int ti, int tj, int c0) {
	T acc[16];
	const int kb = c0 >> 2;
#pragma unroll
	for (int q = 0; q < 4; q++) tile_col_ld<T>(S, ti, tj, q, acc[4 * q], acc[4 * q + 1], acc[4 * q + 2], acc[4 * q + 3]);
	const T *pa = S + lp_off(ti) + 16 * kb;
	const T *pb = S + lp_off(tj) + 16 * kb;
#pragma unroll
	for (int qq = 0; qq < 4; qq++) {
		// tile kb+qq of row panels ti and tj; column slices with the tile swizzle
		const T *ta = pa + 16 * qq, *tb = pb + 16 * qq;
		const int sa = ti + kb + qq, sb = tj + kb + qq;
#pragma unroll
		for (int c = 0; c < 4; c++) {
			T a0, a1, a2, a3, b0, b1, b2, b3;
			if (sizeof(T) == 4) {
				float4 va = *(const float4 *)(ta + ((c ^ (sa & 3)) << 2));
				float4 vb = *(const float4 *)(tb + ((c ^ (sb & 3)) << 2));
				a0 = (T)va.x; a1 = (T)va.y; a2 = (T)va.z; a3 = (T)va.w;
				b0 = (T)vb.x; b1 = (T)vb.y; b2 = (T)vb.z; b3 = (T)vb.w;
			} else {
				double2 va0 = *(const double2 *)(ta + (((2 * c) ^ (sa & 7)) << 1));
				double2 va1 = *(const double2 *)(ta + (((2 * c + 1) ^ (sa & 7)) << 1));
				double2 vb0 = *(const double2 *)(tb + (((2 * c) ^ (sb & 7)) << 1));
				double2 vb1 = *(const double2 *)(tb + (((2 * c + 1) ^ (sb & 7)) << 1));
				a0 = (T)va0.x; a1 = (T)va0.y; a2 = (T)va1.x; a3 = (T)va1.y;
				b0 = (T)vb0.x; b1 = (T)vb0.y; b2 = (T)vb1.x; b3 = (T)vb1.y;
			}
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
	}
#pragma unroll
	for (int q = 0; q < 4; q++) tile_col_st<T>(S, ti, tj, q, acc[4 * q], acc[4 * q + 1], acc[4 * q + 2], acc[4 * q + 3]);
}

// Full factorization of the n x n lower-panel matrix S by the whole CTA
// (blockDim.x >= 64).  dinv: FP64 shared array of >= 4P entries; Lt: 16*17
// entries of T; bad: shared int (0 on entry).  With inv_diag the diagonal
// blocks of the factor are replaced at the end by their explicit inverses
// (all blocks in parallel), for the blocked triangular solves; the blocks
// below the diagonal keep L.
// REP (FP32 only, kernels with registers to spare): the diagonal blocks are
// factored by diag_factor_rep instead of DiagCol.
template <typename T, bool REP = false>
__device__ void chol_smem(T *S, int n, double *dinv, T *Lt, int *bad, bool inv_diag) {
	const int P = (n + 3) >> 2;
	const int NB = (n + 15) >> 4;
	const int tid = threadIdx.x, nt = blockDim.x;
	const int warp = tid >> 5, lane = tid & 31;
	if (warp == 0) chol_diag_factor<T, REP>(S, 0, min(CHOL_NB, n), dinv, Lt, bad);
	__syncthreads();
	for (int K = 0; K < NB; K++) {
		const int c0 = 16 * K, k0 = 4 * K;
		// A. panel rows below the diagonal block
		chol_panel_rows<T>(S, c0, c0 + CHOL_NB, 4 * P, tid, nt, Lt);
		__syncthreads();
		if (K + 1 >= NB) break;
		// B. trailing tiles (ti,tj), k0+4 <= tj <= ti < P; the 10 of the
		// diagonal block K+1 belong to warp 0, which then factors that block
		const int R = P - (k0 + 4);
		if (warp == 0) {
			chol_diag_update_factor<T, REP>(S, c0 + CHOL_NB, min(CHOL_NB, n - c0 - CHOL_NB), c0, dinv, Lt, bad);
		} else if (warp & 3) {
			// warps 4, 8, ... share warp 0's scheduler (warp w issues from
			// sub-partition w % 4): they sit the update out so that the serial
			// diagonal chain keeps its issue slots
			// A warp takes an 8 x 4 block of tiles (8 tile rows, 4 tile columns;
			// lane l: row l / 4, column l % 4): each tile column slice of the
			// panel is then read by 4 lanes and each tile row slice by 8 lanes
			// at once (broadcast), 12 distinct 16-byte loads per 32 tile
			// updates instead of 33 for 32 tiles of one tile row.  Shared-memory
			// bandwidth bounds this update, and its traffic also delays the
			// diagonal warp's loads and shuffles.  Tiles above the diagonal or
			// past the matrix are skipped; the tiles of block K+1 (rows < 4)
			// belong to warp 0.
			const int nuw = (nt >> 5) - ((nt >> 5) + 3) / 4;
			const int uw = warp - (warp >> 2) - 1;
			const int scmax = (R + 3) >> 2, sr = (R + 7) >> 3;
			int si = 0, base = 0, cnt = scmax < 2 ? scmax : 2;
			for (int sidx = uw;; sidx += nuw) {
				while (si < sr && sidx >= base + cnt) {
					base += cnt;
					si++;
					cnt = (2 * si + 2 < scmax) ? 2 * si + 2 : scmax;
				}
				if (si >= sr) break;
				const int ti = 8 * si + (lane >> 2), tj = 4 * (sidx - base) + (lane & 3);
				if (ti < R && ti >= 4 && tj <= ti) chol_tile_update<T>(S, ti + k0 + 4, tj + k0 + 4, c0);
			}
		}
		__syncthreads();
	}
	if (inv_diag) {
		const int nw = nt >> 5;
		for (int K = warp; K < NB; K += nw) chol_block_inverse_inplace<T>(S, n, K, dinv, lane);
		__syncthreads();
	}
}

// Panel index of 4-element chunk ch of the lower panels (panel p holds
// 4(p+1) chunks; chunks before panel p: 2p(p+1)).
__device__ __forceinline__ int lp_chunk_panel(int ch) {
	int p = (int)((sqrtf(2.0f * (float)ch + 1.0f) - 1.0f) * 0.5f);
	while (2 * (p + 1) * (p + 2) <= ch) p++;
	while (2 * p * (p + 1) > ch) p--;
	return p;
}

// Load the lower triangle of an n x n panel-major matrix (row offset a
// multiple of 4: panel p of the lower triangle is the contiguous run
// src[4p*cn .. 4p*cn + 16(p+1)) ) into swizzled lower panels of type TD,
// identity in the padding.  Each thread moves 4-element column slices,
// UNR of them in flight.  slot (optional): unswizzled FP64 copy.
template <typename TD, typename TS, int UNR>
__device__ void load_lp_vec(TD *S, int n, const TS *__restrict__ src, int cn, double *slot) {
	const int P = (n + 3) >> 2;
	const int nch = 2 * P * (P + 1);
	const int tid = threadIdx.x, nt = blockDim.x;
	for (int base = tid; base < nch; base += UNR * nt) {
		TS v[UNR][4];
		int pp[UNR], cc[UNR];
#pragma unroll
		for (int u = 0; u < UNR; u++) {
			const int ch = base + u * nt;
			pp[u] = -1;
			if (ch < nch) {
				const int p = lp_chunk_panel(ch);
				const int col = ch - 2 * p * (p + 1);
				pp[u] = p;
				cc[u] = col;
				const TS *g = src + (size_t)(4 * p) * cn + 4 * col;
				if (sizeof(TS) == 8) {
					double2 x0 = __ldg((const double2 *)g), x1 = __ldg((const double2 *)g + 1);
					v[u][0] = (TS)x0.x; v[u][1] = (TS)x0.y; v[u][2] = (TS)x1.x; v[u][3] = (TS)x1.y;
				} else {
					float4 x = __ldg((const float4 *)g);
					v[u][0] = (TS)x.x; v[u][1] = (TS)x.y; v[u][2] = (TS)x.z; v[u][3] = (TS)x.w;
				}
			}
		}
#pragma unroll
		for (int u = 0; u < UNR; u++) {
			const int p = pp[u];
			if (p < 0) continue;
			const int j = cc[u];
			TD o[4];
			double d[4];
#pragma unroll
			for (int r = 0; r < 4; r++) {
				const int i = 4 * p + r;
				double x;
				if (i < n && j < n)
					x = (j <= i) ? (double)v[u][r] : 0.0;
				else
					x = (i == j) ? 1.0 : 0.0;
				d[r] = x;
				o[r] = (TD)x;
			}
			tile_col_st<TD>(S, p, j >> 2, j & 3, o[0], o[1], o[2], o[3]);
			if (slot) {
				double *sd = slot + lp_off(p) + 4 * j;
				*(double2 *)sd = make_double2(d[0], d[1]);
				*(double2 *)(sd + 2) = make_double2(d[2], d[3]);
			}
		}
	}
}

// Store the lower triangle (j <= i < n) of swizzled lower panels into a
// panel-major matrix with panel-aligned row offset (see load_lp_vec).
template <typename T, int UNR>
__device__ void store_lp_vec(const T *S, int n, T *dst, int cn) {
	const int P = (n + 3) >> 2;
	const int nch = 2 * P * (P + 1);
	const int tid = threadIdx.x, nt = blockDim.x;
	for (int base = tid; base < nch; base += UNR * nt) {
#pragma unroll
		for (int u = 0; u < UNR; u++) {
			const int ch = base + u * nt;
			if (ch >= nch) continue;
			const int p = lp_chunk_panel(ch);
			const int j = ch - 2 * p * (p + 1);
			if (j >= n) continue;
			T o0, o1, o2, o3;
			tile_col_ld<T>(S, p, j >> 2, j & 3, o0, o1, o2, o3);
			T *g = dst + (size_t)(4 * p) * cn + 4 * j;
			if (j < 4 * p && 4 * p + 3 < n) {
				if (sizeof(T) == 8) {
					*(double2 *)g = make_double2((double)o0, (double)o1);
					*((double2 *)g + 1) = make_double2((double)o2, (double)o3);
				} else {
					*(float4 *)g = make_float4((float)o0, (float)o1, (float)o2, (float)o3);
				}
			} else {
				const T o[4] = {o0, o1, o2, o3};
#pragma unroll
				for (int r = 0; r < 4; r++)
					if (4 * p + r < n && j <= 4 * p + r) g[r] = o[r];
			}
		}
	}
}
