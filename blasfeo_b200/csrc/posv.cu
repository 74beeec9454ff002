// Fused factor + solve for variable-size batches of SPD systems A x = b.
//
// The chain being fused is the reference's dpotrf_l followed by dtrsv_lnn and
// dtrsv_ltn (blasfeo_hp_pm/d_lapack_lib4.c:918; blasfeo_hp_pm/d_blas2_lib4.c).
// One CTA solves one system at a time and is persistent: it pulls systems from
// a list sorted by decreasing n (largest first), one list per size class, each
// class launched with the shared memory its largest member needs.
//
//   plain (T = double): lower triangle -> shared memory (lower panels, one HBM
//     read), chol_smem, blocked forward/backward substitution (16x16 diagonal
//     blocks by warp shuffles), x written once.  Matrices whose FP64 lower
//     panels do not fit shared memory take the global-memory path
//     (k_posv_global) instead.
//   mixed (T = float): lower triangle converted to FP32 in shared memory,
//     chol_smem with FP64 diagonal blocks (pivots, reciprocals, block
//     inverses), then iterative refinement: residual r = b - A x in FP64 from
//     the FP64 matrix in global memory (L2-resident while the CTA works on
//     it), correction solves in FP32 with the stored block inverses, x += d in
//     FP64, stopping when ||r||_inf <= tol * ||A||_inf * ||x||_inf.
#include <climits>

#include "chol.cuh"
#include "chol_ll.cuh"
#include "common.cuh"
#include "kernels.cuh"
#include "posv.cuh"

namespace {

__host__ __device__ inline size_t a16(size_t x) { return (x + 15) / 16 * 16; }

// Sort systems by decreasing n (counting sort over n) and split into classes.
// Single CTA.
__global__ void k_posv_classify(int batch, const int *__restrict__ nvec, int max_n, ClassTable ct, PosvWs ws) {
	extern __shared__ int sh[];
	int *hist = sh;               // max_n + 2 buckets
	int *off = sh + (max_n + 2);  // max_n + 2
	const int tid = threadIdx.x, nt = blockDim.x;
	for (int i = tid; i < max_n + 2; i += nt) hist[i] = 0;
	__syncthreads();
	for (int i = tid; i < batch; i += nt) {
		int n = nvec[i];
		n = n < 0 ? 0 : (n > max_n ? max_n + 1 : n);
		atomicAdd(&hist[n], 1);
	}
	__syncthreads();
	if (tid == 0) {
		// descending n: bucket max_n+1 (oversize) first ... bucket 0 last
		int acc = 0;
		for (int v = max_n + 1; v >= 0; v--) {
			off[v] = acc;
			acc += hist[v];
		}
		for (int c = 0; c < ct.nclass; c++) {
			int lo = (c == 0) ? 1 : ct.upper[c - 1] + 1;
			int hi = ct.upper[c];
			if (c == ct.nclass - 1) hi = max_n + 1;  // last class takes oversize too (kernel rejects)
			int s = INT_MAX, cnt = 0;
			for (int v = hi; v >= lo; v--) {
				if (hist[v]) {
					if (off[v] < s) s = off[v];
					cnt += hist[v];
				}
			}
			ws.start[c] = (cnt ? s : 0);
			ws.count[c] = cnt;
			ws.counter[c] = 0;
		}
	}
	__syncthreads();
	for (int i = tid; i < batch; i += nt) {
		int n = nvec[i];
		n = n < 0 ? 0 : (n > max_n ? max_n + 1 : n);
		int pos = atomicAdd(&off[n], 1);
		ws.list[pos] = i;
	}
}

// shared-memory plan of the posv kernel
struct PosvPlan {
	size_t S_off, dinv_off, scr_off, w_off, x_off, r_off, ybuf_off, asum_off, misc_off, total;
};
// CTA size of a size class (largest n of the class).  The mixed kernel's
// shared memory (FP32 lower panels: 63 KB at n = 176, 102 KB at n = 224,
// 133 KB at n = 256) lets three 128-thread CTAs share an SM up to n = 176,
// two up to n = 224, and one 256-thread CTA runs above (thread counts
// measured: the work per system is latency-bound, and fewer threads make the
// barriers cheaper, as long as the trailing updates keep enough warps)
__host__ __device__ inline int posv_threads(int upper) {
	return upper <= 64 ? 64 : (upper <= 224 ? 128 : 256);
}
// Shared memory of one CTA: the lower panels S (the mixed solver overwrites
// their diagonal blocks with the blocks' inverses after the factorization),
// FP64 reciprocal pivots, the factorization's scratch (row-major copy of the
// diagonal block; the mixed solver's first residual pass reuses it for the
// row sums of |A|), the right-hand side / correction w in T and, for the
// mixed solver, the FP64 solution x and residual r.
template <typename T, bool MIXED>
__host__ __device__ inline PosvPlan posv_plan(int max_n, int nt) {
	(void)nt;
	PosvPlan p;
	const int P = (max_n + 3) / 4;
	const int NB = (max_n + 15) / 16;
	const int nv = NB * 16;
	const size_t scr = (16 * 17 + 64) * sizeof(double);
	const size_t asum = MIXED ? (size_t)nv * sizeof(double) : 0;
	p.S_off = 0;
	p.dinv_off = p.S_off + a16((size_t)lp_size(max_n) * sizeof(T));
	p.scr_off = p.dinv_off + a16((size_t)4 * P * sizeof(double));
	p.asum_off = p.scr_off;
	p.w_off = p.scr_off + a16(scr > asum ? scr : asum);
	p.x_off = p.w_off + a16((size_t)nv * sizeof(T));
	p.r_off = p.x_off + (MIXED ? a16((size_t)nv * sizeof(double)) : 0);
	p.ybuf_off = p.r_off + (MIXED ? a16((size_t)nv * sizeof(double)) : 0);
	p.misc_off = p.ybuf_off + a16(16 * sizeof(T));
	p.total = p.misc_off + 64 * sizeof(double);
	return p;
}

// Forward substitution w := L^{-1} w on the lower panels, 16-row blocks.
// With inv_diag the diagonal blocks of S hold their inverses (chol_smem) and
// the diagonal step is a 16x16 product; otherwise warp 0 substitutes with the
// FP64 reciprocal pivots.
template <typename T>
__device__ void trsv_fwd(const T *S, int n, bool inv_diag, const double *dinv, T *w, T *ybuf) {
	const int tid = threadIdx.x, nt = blockDim.x;
	const int NB = (n + 15) >> 4;
	for (int K = 0; K < NB; K++) {
		const int c0 = 16 * K;
		const int nbk = min(16, n - c0);
		if (inv_diag) {
			if (tid < 16) {
				// all 16 entries of row tid of the block are read (the lower
				// panels of a class hold 16 * NB rows and columns) and the ones
				// outside the lower triangle masked by a select, so the loads
				// need no branches
				T s = T(0);
#pragma unroll
				for (int l = 0; l < 16; l++) {
					const T v = lp_at(S, c0 + tid, c0 + l);
					s = fma((l <= tid) ? v : T(0), w[c0 + l], s);
				}
				ybuf[tid] = (tid < nbk) ? s : T(0);
			}
		} else if (tid < 32) {
			const int lane = tid;
			T v = (lane < nbk) ? w[c0 + lane] : T(0);
			for (int k = 0; k < nbk; k++) {
				T yk = __shfl_sync(0xffffffffu, v, k) * (T)dinv[c0 + k];
				if (lane == k) v = yk;
				if (lane > k && lane < nbk) v = fma(-lp_at(S, c0 + lane, c0 + k), yk, v);
			}
			if (lane < 16) ybuf[lane] = (lane < nbk) ? v : T(0);
		}
		__syncthreads();
		// rows below the block, one 4-row panel per thread: each column of a
		// tile comes in one vector load (rows n.. of the last panel hold zeros
		// below the diagonal and stay zero)
		const int kb = c0 >> 2, P = (n + 3) >> 2;
		for (int p = kb + 4 + tid; p < P; p += nt) {
			T s0 = w[4 * p], s1 = w[4 * p + 1], s2 = w[4 * p + 2], s3 = w[4 * p + 3];
#pragma unroll
			for (int q = 0; q < 4; q++)
#pragma unroll
				for (int c = 0; c < 4; c++) {
					T a0, a1, a2, a3;
					tile_col_ld<T>(S, p, kb + q, c, a0, a1, a2, a3);
					const T y = ybuf[4 * q + c];
					s0 = fma(-a0, y, s0);
					s1 = fma(-a1, y, s1);
					s2 = fma(-a2, y, s2);
					s3 = fma(-a3, y, s3);
				}
			w[4 * p] = s0;
			w[4 * p + 1] = s1;
			w[4 * p + 2] = s2;
			w[4 * p + 3] = s3;
		}
		if (tid < nbk) w[c0 + tid] = ybuf[tid];
		__syncthreads();
	}
}

// Backward substitution w := L^{-T} w (inv_diag as trsv_fwd).
template <typename T>
__device__ void trsv_bwd(const T *S, int n, bool inv_diag, const double *dinv, T *w, T *ybuf) {
	const int tid = threadIdx.x, nt = blockDim.x;
	const int NB = (n + 15) >> 4;
	for (int K = NB - 1; K >= 0; K--) {
		const int c0 = 16 * K;
		const int nbk = min(16, n - c0);
		if (inv_diag) {
			if (tid < 16) {
				T s = T(0);
#pragma unroll
				for (int l = 0; l < 16; l++) {
					const T v = lp_at(S, c0 + l, c0 + tid);
					s = fma((l >= tid && l < nbk) ? v : T(0), w[c0 + l], s);
				}
				ybuf[tid] = (tid < nbk) ? s : T(0);
			}
		} else if (tid < 32) {
			const int lane = tid;
			T v = (lane < nbk) ? w[c0 + lane] : T(0);
			for (int k = nbk - 1; k >= 0; k--) {
				T xk = __shfl_sync(0xffffffffu, v, k) * (T)dinv[c0 + k];
				if (lane == k) v = xk;
				if (lane < k) v = fma(-lp_at(S, c0 + k, c0 + lane), xk, v);
			}
			if (lane < 16) ybuf[lane] = (lane < nbk) ? v : T(0);
		}
		__syncthreads();
		// columns left of the block: for column j the 16 rows of block row K
		// are column slices of four tiles (one vector load each); the panels
		// of the block row past the matrix (q with kb + q >= P) are skipped,
		// rows n.. of the last real panel hold zeros left of the diagonal
		const int kb = c0 >> 2, P = (n + 3) >> 2;
		for (int j = tid; j < c0; j += nt) {
			T s = w[j];
#pragma unroll
			for (int q = 0; q < 4; q++) {
				if (kb + q >= P) break;
				T a0, a1, a2, a3;
				tile_col_ld<T>(S, kb + q, j >> 2, j & 3, a0, a1, a2, a3);
				s = fma(-a0, ybuf[4 * q], s);
				s = fma(-a1, ybuf[4 * q + 1], s);
				s = fma(-a2, ybuf[4 * q + 2], s);
				s = fma(-a3, ybuf[4 * q + 3], s);
			}
			w[j] = s;
		}
		if (tid < nbk) w[c0 + tid] = ybuf[tid];
		__syncthreads();
	}
}

template <typename T>
__device__ double block_max(double v, double *red) {
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
	for (int off = 16; off > 0; off >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, off));
	if (lane == 0) red[warp] = v;
	__syncthreads();
	if (threadIdx.x == 0) {
		double m = 0.0;
		for (int w = 0; w < nw; w++) m = fmax(m, red[w]);
		red[32] = m;
	}
	__syncthreads();
	double r = red[32];
	__syncthreads();
	return r;
}

// CTA-wide maxima of N <= 3 values at once (one reduction, two barriers for
// all); red: 51 doubles, up to 16 warps
template <int N>
__device__ void block_max_n(double (&v)[N], double *red) {
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
	for (int off = 16; off > 0; off >>= 1)
#pragma unroll
		for (int e = 0; e < N; e++) v[e] = fmax(v[e], __shfl_down_sync(0xffffffffu, v[e], off));
	if (lane == 0)
#pragma unroll
		for (int e = 0; e < N; e++) red[16 * e + warp] = v[e];
	__syncthreads();
	if (threadIdx.x < N) {
		double m = 0.0;
		for (int w = 0; w < nw; w++) m = fmax(m, red[16 * threadIdx.x + w]);
		red[48 + threadIdx.x] = m;
	}
	__syncthreads();
#pragma unroll
	for (int e = 0; e < N; e++) v[e] = red[48 + e];
	__syncthreads();
}

// r = b - A x (FP64), A symmetric given by its lower triangle, in one pass
// over the lower triangle (every element read once).
// LP = false: A in BLASFEO panel-major storage (tile row ti at base + 4*ti*cn);
// LP = true: A in lower panels (tile row ti at base + lp_off(ti)).
// Either way the tiles 0..ti of tile row ti are 128 (ti+1) contiguous bytes,
// tile (ti,tj) column-major.  Warp w takes tile rows ti = w, w + NW, ...
// and reads a row as contiguous 512-byte pieces, one 16-byte load per lane:
// piece k, lane l holds rows 2(l&1), 2(l&1)+1 of column 16k + jl of the
// row, jl = 4(l>>3) + ((l&7)>>1), so every load instruction of the warp
// covers four whole cache lines.  A lane's column set {16k + jl} is the same
// in every row, so the transposed contributions (A^T x for the strictly lower
// part) accumulate per lane in registers (cacc[k]) over all rows of the
// warp; the row contributions (A x for the lower part with the diagonal) are
// reduced over the lanes of equal parity by shuffles after each row.  After
// all rows the warps subtract their column sums one after the other in warp
// order, so the result does not depend on timing.  KMAX = pieces of the
// longest row (tile rows <= 4 KMAX, n <= 16 KMAX).
// RES: the residual into r; NORM: the row sums of |A| into asum.
template <bool LP>
__device__ __forceinline__ const double *res_row(const double *base, int cn, int ti) {
	return LP ? base + lp_off(ti) : base + (size_t)(4 * ti) * cn;
}

template <bool LP, bool RES, bool NORM, int KMAX>
__device__ void sym_residual(const double *base, int cn, int n, const double *b, const double *x, double *r,
                             double *asum) {
	const int tid = threadIdx.x, nt = blockDim.x;
	const int lane = tid & 31, warp = tid >> 5, nw = nt >> 5;
	const int P = (n + 3) >> 2;
	const int a0 = 2 * (lane & 1);                           // first of the lane's two rows in a tile
	const int jl = 4 * (lane >> 3) + ((lane & 7) >> 1);      // the lane's column in a 16-column piece
	double cacc[KMAX], cabs[KMAX];
#pragma unroll
	for (int k = 0; k < KMAX; k++) cacc[k] = cabs[k] = 0.0;
	for (int ti = warp; ti < P; ti += nw) {
		const double *row = res_row<LP>(base, cn, ti) + 2 * lane;
		const int kr = (ti + 4) >> 2;       // pieces of this row
		const int kl = ti - (lane >> 3);    // the lane's tile 4k + (lane>>3) is in the row iff 4k <= kl
		const int gi0 = 4 * ti + a0;
		// every load of the row first (L2 only: the per-CTA copy (LP) is
		// written by this kernel); slots past the row stay zero
		double2 v[KMAX];
#pragma unroll
		for (int k = 0; k < KMAX; k++) {
			v[k] = make_double2(0.0, 0.0);
			if (k < kr && 4 * k <= kl) v[k] = __ldcg((const double2 *)(row + 64 * k));
		}
		const double xr0 = x[gi0], xr1 = x[gi0 + 1];
		double r0 = 0.0, r1 = 0.0, s0 = 0.0, s1 = 0.0;
#pragma unroll
		for (int k = 0; k < KMAX; k++) {
			if (k < kr) {
				const int gj = 16 * k + jl;
				const bool ok = 4 * k <= kl && gj < n;
				const double xj = x[gj];
				// row part: j <= i; column part: j < i
				const double e0 = ok && gi0 < n && gj <= gi0 ? v[k].x : 0.0;
				const double e1 = ok && gi0 + 1 < n && gj <= gi0 + 1 ? v[k].y : 0.0;
				const double c0 = gj < gi0 ? e0 : 0.0;
				const double c1 = gj < gi0 + 1 ? e1 : 0.0;
				if (RES) {
					r0 = fma(e0, xj, r0);
					r1 = fma(e1, xj, r1);
					cacc[k] = fma(c0, xr0, fma(c1, xr1, cacc[k]));
				}
				if (NORM) {
					s0 += fabs(e0);
					s1 += fabs(e1);
					cabs[k] += fabs(c0) + fabs(c1);
				}
			}
		}
#pragma unroll
		for (int off = 2; off < 32; off <<= 1) {
			if (RES) {
				r0 += __shfl_xor_sync(0xffffffffu, r0, off);
				r1 += __shfl_xor_sync(0xffffffffu, r1, off);
			}
			if (NORM) {
				s0 += __shfl_xor_sync(0xffffffffu, s0, off);
				s1 += __shfl_xor_sync(0xffffffffu, s1, off);
			}
		}
		if (lane < 2) {
			if (RES) {
				r[gi0] = (gi0 < n ? b[gi0] : 0.0) - r0;
				r[gi0 + 1] = (gi0 + 1 < n ? b[gi0 + 1] : 0.0) - r1;
			}
			if (NORM) {
				asum[gi0] = s0;
				asum[gi0 + 1] = s1;
			}
		}
	}
	// the two lanes of a column (rows 0,1 and 2,3 of each tile) combined
#pragma unroll
	for (int k = 0; k < KMAX; k++) {
		if (RES) cacc[k] += __shfl_xor_sync(0xffffffffu, cacc[k], 1);
		if (NORM) cabs[k] += __shfl_xor_sync(0xffffffffu, cabs[k], 1);
	}
	__syncthreads();
	// column parts: subtracted from r (added to asum) one warp after the
	// other, in warp order
	for (int wv = 0; wv < nw; wv++) {
		if (warp == wv && !(lane & 1)) {
#pragma unroll
			for (int k = 0; k < KMAX; k++) {
				const int J = 16 * k + jl;
				if (J < 4 * P) {
					if (RES) r[J] -= cacc[k];
					if (NORM) asum[J] += cabs[k];
				}
			}
		}
		__syncthreads();
	}
}

// pieces of the longest tile row the kernel variant takes (its largest n)
template <int NT, int MINB>
struct ResShape {
	static constexpr int KMAX = NT == 64 ? 4 : (MINB == 4 ? 8 : (MINB == 3 ? 11 : (MINB == 2 ? 14 : 16)));
};

template <typename T, bool MIXED, int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB) k_posv(int cls, int max_n, PosvWs ws, const int *__restrict__ nvec,
                                              const DevDesc<double> *__restrict__ sA,
                                              const DevVec<double> *__restrict__ sb,
                                              const DevVec<double> *__restrict__ sx, int max_iter, double tol,
                                              int *iters, double *berr, int *info, double *slots) {
	static_assert(NT % 32 == 0 && NT <= 512, "block_max_n keeps up to 16 warps' partial maxima");
	extern __shared__ __align__(16) unsigned char smem[];
	const PosvPlan pl = posv_plan<T, MIXED>(max_n, NT);
	// per-CTA FP64 copy of the lower panels (refinement residuals read it from
	// L2 instead of the caller's matrix, which may sit in host memory)
	double *slot = slots ? slots + (size_t)blockIdx.x * lp_size(max_n) : nullptr;
	double *asum = (double *)(smem + pl.asum_off);
	T *S = (T *)(smem + pl.S_off);
	double *dinv = (double *)(smem + pl.dinv_off);
	double *scratch = (double *)(smem + pl.scr_off);
	T *w = (T *)(smem + pl.w_off);
	double *xs = (double *)(smem + pl.x_off);
	double *rs = (double *)(smem + pl.r_off);
	T *ybuf = (T *)(smem + pl.ybuf_off);
	double *misc = (double *)(smem + pl.misc_off);
	int *s_bad = (int *)(misc + 60);
	int *s_item = (int *)(misc + 61);
	const int tid = threadIdx.x, nt = blockDim.x;
	const int start = ws.start[cls], count = ws.count[cls];

	for (;;) {
		if (tid == 0) {
			int k = atomicAdd(&ws.counter[cls], 1);
			*s_item = (k < count) ? ws.list[start + k] : -1;
			*s_bad = 0;
		}
		__syncthreads();
		const int sys = *s_item;
		if (sys < 0) break;
		const int n = nvec[sys];
		if (n <= 0 || n > max_n) {
			if (tid == 0) {
				if (info) info[sys] = (n <= 0) ? 0 : -2;
				if (iters) iters[sys] = 0;
			}
			__syncthreads();
			continue;
		}
		PMat<double> a;
		a.p = sA[sys].pA;
		a.d = sA[sys].dA;
		a.cn = sA[sys].cn;
		a.ri = 0;
		a.cj = 0;
		const double *bg = sb[sys].pa;
		double *xg = sx[sys].pa;
		const int nv = ((n + 15) >> 4) * 16;

		// lower triangle -> lower panels (converted to T), identity padding; the
		// mixed path with refinement slots also keeps an FP64 copy there
		// one CTA per SM (the largest classes) keeps more loads in flight per thread
		if (MINB <= 2)
			load_lp_vec<T, double, 4>(S, n, a.p, a.cn, MIXED ? slot : nullptr);
		else
			load_lp_vec<T, double, 2>(S, n, a.p, a.cn, MIXED ? slot : nullptr);
		for (int i = tid; i < nv; i += nt) w[i] = (i < n) ? (T)bg[i] : T(0);
		if (MIXED)
			for (int i = tid; i < nv; i += nt) xs[i] = 0.0;
		__syncthreads();
		chol_smem<T>(S, n, dinv, (T *)scratch, s_bad, MIXED);

		if (!MIXED) {
			trsv_fwd<T>(S, n, false, dinv, w, ybuf);
			trsv_bwd<T>(S, n, false, dinv, w, ybuf);
			for (int i = tid; i < n; i += nt) xg[i] = (double)w[i];
			if (tid == 0) {
				if (info) info[sys] = *s_bad;
				if (iters) iters[sys] = 0;
			}
			__syncthreads();
			continue;
		}

		// mixed: refinement loop; the first pass solves with r = b
		double anorm = 0.0, bnorm_res = 0.0;
		int it = 0;
		bool conv = false;
		double scale = 1.0;
		{
			double m = 0.0;
			for (int i = tid; i < n; i += nt) m = fmax(m, fabs(bg[i]));
			m = block_max<T>(m, misc);
			scale = (m > 0.0) ? 1.0 / m : 1.0;
			for (int i = tid; i < nv; i += nt) w[i] = (i < n) ? (T)(bg[i] * scale) : T(0);
			__syncthreads();
		}
		for (;;) {
			trsv_fwd<T>(S, n, true, dinv, w, ybuf);
			trsv_bwd<T>(S, n, true, dinv, w, ybuf);
			for (int i = tid; i < n; i += nt) xs[i] += (double)w[i] / scale;
			__syncthreads();
			// ||A||_inf (row sums of |A|) once, before the first residual
			// (the first pass also accumulates the row sums of |A|: one read of A)
			constexpr int KM = ResShape<NT, MINB>::KMAX;
			if (slot) {
				if (it == 0)
					sym_residual<true, true, true, KM>(slot, 0, n, bg, xs, rs, asum);
				else
					sym_residual<true, true, false, KM>(slot, 0, n, bg, xs, rs, asum);
			} else {
				if (it == 0)
					sym_residual<false, true, true, KM>(a.p, a.cn, n, bg, xs, rs, asum);
				else
					sym_residual<false, true, false, KM>(a.p, a.cn, n, bg, xs, rs, asum);
			}
			// norms (on the first pass also ||A||_inf from the row sums of |A|
			// that the residual accumulated), reduced together
			double rm, xm;
			{
				double m3[3] = {0.0, 0.0, 0.0};
				for (int i = tid; i < n; i += nt) {
					m3[0] = fmax(m3[0], fabs(rs[i]));
					m3[1] = fmax(m3[1], fabs(xs[i]));
					if (it == 0) m3[2] = fmax(m3[2], asum[i]);
				}
				if (it == 0) {
					block_max_n<3>(m3, misc);
					anorm = m3[2];
				} else {
					double m2[2] = {m3[0], m3[1]};
					block_max_n<2>(m2, misc);
					m3[0] = m2[0];
					m3[1] = m2[1];
				}
				rm = m3[0];
				xm = m3[1];
			}
			it++;
			bnorm_res = (anorm > 0.0 && xm > 0.0) ? rm / (anorm * xm) : (rm == 0.0 ? 0.0 : INFINITY);
			if (bnorm_res <= tol) {
				conv = true;
				break;
			}
			if (it > max_iter) break;
			scale = (rm > 0.0) ? 1.0 / rm : 1.0;
			for (int i = tid; i < nv; i += nt) w[i] = (i < n) ? (T)(rs[i] * scale) : T(0);
			__syncthreads();
		}
		for (int i = tid; i < n; i += nt) xg[i] = xs[i];
		if (tid == 0) {
			if (iters) iters[sys] = it - 1;
			if (berr) berr[sys] = bnorm_res;
			if (info) info[sys] = *s_bad ? *s_bad : (conv ? 0 : -1);
		}
		__syncthreads();
	}
}

// Systems whose FP64 lower panels exceed shared memory: the factor goes to a
// per-CTA workspace slot (panel layout, blocked left-looking with FP64
// tensor-core updates, chol_ll.cuh), then the two blocked triangular solves
// read it from there (L2-resident), the right-hand side in shared memory.
__host__ __device__ inline size_t posv_slot_elems(int max_n) {
	const size_t p4 = (size_t)(max_n + 3) / 4 * 4;
	return p4 * p4 + (size_t)(max_n + 15) / 16 * 16;
}
constexpr int POSV_GLOBAL_NT = 128;
// fragment rows per warp in the factorization's panel updates
#ifndef POSV_GLOBAL_FR
#define POSV_GLOBAL_FR 1
#endif
__global__ void __launch_bounds__(POSV_GLOBAL_NT, 4)
    k_posv_global(int cls, int max_n, PosvWs ws, const int *__restrict__ nvec, const DevDesc<double> *__restrict__ sA,
                  const DevVec<double> *__restrict__ sb, const DevVec<double> *__restrict__ sx, double *slots,
                  int *info) {
	extern __shared__ __align__(16) double pg_smem[];
	__shared__ int s_item, s_bad;
	const int tid = threadIdx.x;
	const int start = ws.start[cls], count = ws.count[cls];
	double *y = pg_smem + ll_smem_bytes(max_n) / sizeof(double);
	PMat<double> L;
	L.p = slots + posv_slot_elems(max_n) * blockIdx.x;
	L.cn = (max_n + 3) / 4 * 4;
	L.d = L.p + (size_t)L.cn * L.cn;
	L.ri = L.cj = 0;
	for (;;) {
		if (tid == 0) {
			int k = atomicAdd(&ws.counter[cls], 1);
			s_item = (k < count) ? ws.list[start + k] : -1;
			s_bad = 0;
		}
		__syncthreads();
		const int sys = s_item;
		if (sys < 0) break;
		const int n = nvec[sys];
		if (n <= 0 || n > max_n) {
			if (tid == 0 && info) info[sys] = (n <= 0) ? 0 : -2;
			__syncthreads();
			continue;
		}
		PMat<double> a;
		a.p = sA[sys].pA;
		a.d = nullptr;
		a.cn = sA[sys].cn;
		a.ri = a.cj = 0;
		const double *bg = sb[sys].pa;
		for (int i = tid; i < n; i += POSV_GLOBAL_NT) y[i] = bg[i];
		chol_ll<POSV_GLOBAL_NT, POSV_GLOBAL_FR>(a, L, n, pg_smem, &s_bad);
		trsv_ll_fwd<POSV_GLOBAL_NT>(L, n, y);
		trsv_ll_bwd<POSV_GLOBAL_NT>(L, n, y);
		double *xg = sx[sys].pa;
		for (int i = tid; i < n; i += POSV_GLOBAL_NT) xg[i] = y[i];
		if (tid == 0 && info) info[sys] = s_bad;
		__syncthreads();
	}
}

struct PosvClassCfg {
	int upper;
	int threads;
};

template <typename T, bool MIXED, int NT, int MINB>
int launch_posv(int c, int upper, size_t smem, int batch, int rslots, PosvWs ws, const int *n, const void *sA,
                const void *sb, const void *sx, int max_iter, double tol, int *iters, double *berr, int *info,
                double *rs, cudaStream_t s) {
	auto kern = k_posv<T, MIXED, NT, MINB>;
	bf::smem_optin(kern, smem);
	int per_sm = 0;
	cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, NT, smem);
	if (per_sm < 1) per_sm = 1;
	int grid = bf::num_sms() * per_sm;
	if (grid > batch) grid = batch;
	if (rslots && grid > rslots) grid = rslots;
	kern<<<grid, NT, smem, s>>>(c, upper, ws, n, (const DevDesc<double> *)sA, (const DevVec<double> *)sb,
	                            (const DevVec<double> *)sx, max_iter, tol, iters, berr, info, rs);
	return bf::check_launch();
}

// the mixed solver's engine for n <= 256 (tensor cores unless SIMT is asked for)
inline bool tensor_engine() {
	const int e = bf::posv_engine();
	return e == BLASFEO_B200_POSV_TENSOR || (e == BLASFEO_B200_POSV_DEFAULT && POSV_TENSOR_DEFAULT);
}

// size classes and workspace layout of one call
struct PosvLayout {
	ClassTable ct;
	PosvClassCfg cfg[POSV_MAX_CLASSES];
	int nc;
	bool need_global;
	int gslots, rslots;
	size_t need, slots_off, rslots_off;
};

template <typename T, bool MIXED>
PosvLayout posv_layout(int batch, int max_n, bool use_slots) {
	PosvLayout L;
	// size classes: shared memory and CTA size follow the largest member
	const size_t smem_cap = bf::max_smem_optin();
	const int uppers[] = {16, 32, 64, 96, 128, 160, 176, 192, 224, 256};
	int nc = 0;
	int smem_limit_n = 0;  // largest n the shared-memory kernel takes
	for (int v = 4; v <= 4096; v += 4)
		if (posv_plan<T, MIXED>(v, posv_threads(v)).total <= smem_cap) smem_limit_n = v;
	// plain FP64: above n = 128 the blocked kernel with FP64 tensor-core
	// updates (L2-resident factor, 4 systems per SM) beats the shared-memory one
	if (!MIXED && smem_limit_n > 128) smem_limit_n = 128;
	for (int u : uppers) {
		if (nc >= POSV_MAX_CLASSES - 1) break;
		int uu = u < smem_limit_n ? u : smem_limit_n;
		if (nc > 0 && uu <= L.cfg[nc - 1].upper) continue;
		L.cfg[nc].upper = uu;
		L.cfg[nc].threads = posv_threads(uu);
		nc++;
		if (uu >= max_n) break;
	}
	L.need_global = max_n > L.cfg[nc - 1].upper;
	if (L.need_global) {
		L.cfg[nc].upper = max_n;
		L.cfg[nc].threads = POSV_GLOBAL_NT;
		nc++;
	}
	L.nc = nc;
	L.ct.nclass = nc;
	for (int c = 0; c < nc; c++) L.ct.upper[c] = L.cfg[c].upper;
	// workspace: work list and class tables, global-path factor slots,
	// mapped-path refinement slots
	L.gslots = L.need_global ? 4 * bf::num_sms() : 0;
	L.need = posv_list_bytes((size_t)batch);
	L.slots_off = L.need;
	L.need += (size_t)L.gslots * posv_slot_elems(max_n) * sizeof(double);
	L.rslots_off = a16(L.need);
	L.rslots = 0;
	if (MIXED && use_slots) {
		const int per_sm = 16;  // upper bound of resident CTAs per SM over all classes
		L.rslots = bf::num_sms() * per_sm;
		// one set per stream of the class rotation (two streams)
		L.need = L.rslots_off + 2 * (size_t)L.rslots * lp_size(max_n) * sizeof(double);
	}
	return L;
}

template <typename T, bool MIXED>
int posv_run(int batch, const int *n, int max_n, const void *sA, const void *sb, const void *sx, int max_iter,
             double tol, int *iters, double *berr, int *info, void *work, size_t work_bytes, cudaStream_t s,
             bool use_slots, bool one_stream = false) {
	if (batch < 0 || !n || !sA || !sb || !sx || max_n < 0) return BLASFEO_B200_EINVAL;
	if (batch == 0 || max_n == 0) return BLASFEO_B200_OK;
	const PosvLayout lay = posv_layout<T, MIXED>(batch, max_n, use_slots);
	const PosvClassCfg *cfg = lay.cfg;
	const ClassTable ct = lay.ct;
	const int nc = lay.nc;
	const bool need_global = lay.need_global;
	if (need_global && max_n > bf::dpotrf_ll_max_n()) return BLASFEO_B200_ENOTSUP;
	const int gslots = lay.gslots, rslots = lay.rslots;
	const size_t need = lay.need, slots_off = lay.slots_off, rslots_off = lay.rslots_off;
	char *wsp = (char *)work;
	if (!wsp) {
		wsp = (char *)bf::workspace(need, s);
		if (!wsp) return BLASFEO_B200_ENOMEM;
	} else if (work_bytes < need) {
		return BLASFEO_B200_ENOMEM;
	}
	PosvWs ws;
	ws.list = (int *)wsp;
	char *q = wsp + a16((size_t)batch * sizeof(int));
	ws.start = (int *)q;
	q += a16(POSV_MAX_CLASSES * sizeof(int));
	ws.count = (int *)q;
	q += a16(POSV_MAX_CLASSES * sizeof(int));
	ws.counter = (int *)q;
	q += a16(POSV_MAX_CLASSES * sizeof(int));
	ws.hist = (int *)q;
	k_posv_classify<<<1, 1024, 2 * (max_n + 2) * sizeof(int), s>>>(batch, n, max_n, ct, ws);
	if (bf::check_launch()) return BLASFEO_B200_ECUDA;
	const int sms = bf::num_sms();
	// the size classes are independent: they alternate between the caller's
	// stream and a second one (forked after the classification, joined at the
	// end), so a class's CTAs start on the SMs that the previous class's last
	// systems leave idle (mixed solver, 20,000 systems: 10.5 -> 9.8 ms)
	cudaStream_t side = nullptr;
	cudaEvent_t fork = nullptr, join = nullptr;
	// (the mapped path's per-CTA refinement slots: one set per stream)
	// (one_stream: the caller's stream only; the second stream and its events
	// are created on a host thread's first call, which can take device memory)
	const bool two = !one_stream && nc > 1 && bf::side_stream(&side, &fork, &join);
	if (two) {
		cudaEventRecord(fork, s);
		cudaStreamWaitEvent(side, fork, 0);
	}
	const cudaStream_t s0 = s;
	int status = BLASFEO_B200_OK;
	for (int ci = 0; ci < nc && status == BLASFEO_B200_OK; ci++) {
		// order (measured): the plain solver largest class first; the mixed
		// one its largest class first (one CTA per SM, the longest), then the
		// others smallest first on alternating streams, which fill the SMs
		// that the largest class's last systems leave idle (20,000 systems:
		// 8.88 -> 8.75 ms against smallest first throughout)
		const int c = !MIXED ? nc - 1 - ci : (ci == 0 ? nc - 1 : ci - 1);
		const cudaStream_t s = (two && (ci & 1)) ? side : s0;
		const bool glob = need_global && c == nc - 1;
		if (glob) {
			const size_t gsm = ll_smem_bytes(max_n) + (size_t)max_n * sizeof(double);
			bf::smem_optin(k_posv_global, gsm);
			k_posv_global<<<gslots, POSV_GLOBAL_NT, gsm, s>>>(c, max_n, ws, n, (const DevDesc<double> *)sA,
			                                                  (const DevVec<double> *)sb, (const DevVec<double> *)sx,
			                                                  (double *)(wsp + slots_off), info);
		} else if (MIXED && !use_slots && cfg[c].upper <= 256 && tensor_engine()) {
			const int st = bf::posv_tc_launch(c, cfg[c].upper, batch, ws, n, sA, sb, sx, max_iter, tol, iters, berr,
			                                  info, s);
			if (st) {
				status = st;
				break;
			}
		} else {
			PosvPlan pl = posv_plan<T, MIXED>(cfg[c].upper, cfg[c].threads);
			double *rs = rslots ? (double *)(wsp + rslots_off) + (s != s0 ? (size_t)rslots * lp_size(max_n) : 0)
			                    : nullptr;
			int st;
			if (cfg[c].upper <= 64)
				st = launch_posv<T, MIXED, 64, 8>(c, cfg[c].upper, pl.total, batch, rslots, ws, n, sA, sb, sx, max_iter,
				                                  tol, iters, berr, info, rs, s);
			else if (cfg[c].upper <= 128)
				st = launch_posv<T, MIXED, 128, 4>(c, cfg[c].upper, pl.total, batch, rslots, ws, n, sA, sb, sx,
				                                   max_iter, tol, iters, berr, info, rs, s);
			else if (cfg[c].upper <= 176)
				st = launch_posv<T, MIXED, 128, 3>(c, cfg[c].upper, pl.total, batch, rslots, ws, n, sA, sb, sx,
				                                   max_iter, tol, iters, berr, info, rs, s);
			else if (cfg[c].upper <= 224)
				st = launch_posv<T, MIXED, 128, 2>(c, cfg[c].upper, pl.total, batch, rslots, ws, n, sA, sb, sx,
				                                   max_iter, tol, iters, berr, info, rs, s);
			else
				st = launch_posv<T, MIXED, 256, 1>(c, cfg[c].upper, pl.total, batch, rslots, ws, n, sA, sb, sx,
				                                   max_iter, tol, iters, berr, info, rs, s);
			if (st) {
				status = st;
				break;
			}
		}
		if (bf::check_launch()) status = BLASFEO_B200_ECUDA;
	}
	// joined on every path, errors included (a fork left open would break a
	// stream capture of the call)
	if (two) {
		cudaEventRecord(join, side);
		cudaStreamWaitEvent(s, join, 0);
	}
	return status;
}

}  // namespace

extern "C" {

size_t blasfeo_dposv_worksize(int batch) {
	// list + class tables (enough for every system that takes a shared-memory kernel)
	return posv_list_bytes((size_t)(batch > 0 ? batch : 0));
}

size_t blasfeo_dposv_worksize_n(int batch, int max_n, int mixed) {
	if (batch < 0 || max_n <= 0) return blasfeo_dposv_worksize(batch);
	return mixed ? posv_layout<float, true>(batch, max_n, false).need : posv_layout<double, false>(batch, max_n, false).need;
}

int blasfeo_dposv_l_vbatch(int batch, const int *n, int max_n, const struct blasfeo_dmat *sA,
                           const struct blasfeo_dvec *sb, const struct blasfeo_dvec *sx, int *info, void *work,
                           size_t work_bytes, void *stream) {
	return posv_run<double, false>(batch, n, max_n, sA, sb, sx, 0, 0.0, nullptr, nullptr, info, work, work_bytes,
	                               (cudaStream_t)stream, false);
}

int blasfeo_dsposv_l_vbatch(int batch, const int *n, int max_n, const struct blasfeo_dmat *sA,
                            const struct blasfeo_dvec *sb, const struct blasfeo_dvec *sx, int max_iter, double tol,
                            int *iters, double *berr, int *info, void *work, size_t work_bytes, void *stream) {
	return posv_run<float, true>(batch, n, max_n, sA, sb, sx, max_iter, tol, iters, berr, info, work, work_bytes,
	                             (cudaStream_t)stream, false);
}

int blasfeo_dsposv_l_vbatch_mapped(int batch, const int *n, int max_n, const struct blasfeo_dmat *sA,
                                   const struct blasfeo_dvec *sb, const struct blasfeo_dvec *sx, int max_iter,
                                   double tol, int *iters, double *berr, int *info, void *work, size_t work_bytes,
                                   void *stream) {
	return posv_run<float, true>(batch, n, max_n, sA, sb, sx, max_iter, tol, iters, berr, info, work, work_bytes,
	                             (cudaStream_t)stream, true);
}

}  // extern "C"

namespace bf {

// the mixed solver on the caller's stream alone (no per-thread second stream)
// with a caller-provided workspace: the allocation-free entry point's path
int dsposv_one_stream(int batch, const int *n, int max_n, const void *sA, const void *sb, const void *sx, int max_iter,
                      double tol, int *iters, double *berr, int *info, void *work, size_t work_bytes,
                      cudaStream_t stream) {
	return posv_run<float, true>(batch, n, max_n, sA, sb, sx, max_iter, tol, iters, berr, info, work, work_bytes,
	                             stream, false, true);
}

}  // namespace bf
