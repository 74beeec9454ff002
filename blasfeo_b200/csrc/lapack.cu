// LAPACK-level routines on panel-major device matrices: potrf_l,
// syrk_dpotrf_ln, getrf_rp, geqrf (single, uniform batch, variable batch).
// One CTA factors one instance.
//
// potrf_l (blasfeo_hp_pm/d_lapack_lib4.c:918): when the lower triangle fits in
// shared memory the matrix is loaded once (coalesced 4-row panel runs),
// factored there by chol_smem (chol.cuh) and written back once: HBM traffic is
// one read and one write of the lower triangle.  Larger matrices use an
// unblocked right-looking factorization directly in global memory (L1/L2
// resident for BLASFEO-sized problems).
//
// getrf_rp (blasfeo_hp_pm/d_lapack_lib4.c:2396): right-looking LU with row
// pivoting; per column a CTA-wide argmax (first index of the largest |a|,
// kernel/generic/kernel_dgetrf_pivot_lib4.c:84), a full-row swap, scaling by
// the reciprocal pivot (0 for a zero pivot) and a rank-1 update.  The
// element-wise operation order equals the reference's (one subtraction per
// earlier column, in column order).
//
// geqrf (blasfeo_hp_pm/d_lapack_lib4.c:3444): Householder QR, one reflector
// per column with LAPACK dlarfg signs (kernel/generic/kernel_dgeqrf_4_lib4.c:
// 80-96); the column norm is a CTA reduction in the working precision, the
// reflector is applied to every trailing column by one thread per column.
#include <climits>

#include "chol.cuh"
#include "common.cuh"
#include "kernels.cuh"

namespace {

__host__ __device__ inline size_t align16(size_t x) { return (x + 15) / 16 * 16; }

// shared-memory plan of the potrf kernel for matrices up to max_n
// (lower panels, FP64 reciprocal pivots, the 16x17 row-major copy of the
// diagonal block that chol_smem's panel solve reads, the bad-pivot flag)
struct PotrfSmem {
	size_t s_bytes, dinv_off, lt_off, bad_off, total;
};
template <typename T>
__host__ __device__ inline PotrfSmem potrf_smem_plan(int max_n) {
	PotrfSmem p;
	int P = (max_n + 3) / 4;
	p.s_bytes = align16((size_t)lp_size(max_n) * sizeof(T));
	p.dinv_off = p.s_bytes;
	p.lt_off = p.dinv_off + align16((size_t)4 * P * sizeof(double));
	p.bad_off = p.lt_off + align16(16 * 17 * sizeof(T));
	p.total = p.bad_off + 16;
	return p;
}

// load the lower triangle of C (n x n at the view's offsets) into lower panels,
// identity in the padding
template <typename T>
__device__ void load_lower_panels(T *S, int n, const PMat<T> &c) {
	const int P = (n + 3) >> 2;
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
	for (int p = warp; p < P; p += nw) {
		const int cnt = 16 * (p + 1);
		for (int e = lane; e < cnt; e += 32) {
			int i = 4 * p + (e & 3), j = e >> 2;
			T v;
			if (i < n && j < n)
				v = (j <= i) ? c.at(i, j) : T(0);
			else
				v = (i == j) ? T(1) : T(0);
			S[lp_idx<T>(i, j)] = v;
		}
	}
}

// write the lower triangle (j <= i < n) of the lower panels into D
template <typename T>
__device__ void store_lower_panels(const T *S, int n, const PMat<T> &d) {
	const int P = (n + 3) >> 2;
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
	for (int p = warp; p < P; p += nw) {
		const int cnt = 16 * (p + 1);
		for (int e = lane; e < cnt; e += 32) {
			int i = 4 * p + (e & 3), j = e >> 2;
			if (i < n && j <= i) d.at(i, j) = S[lp_idx<T>(i, j)];
		}
	}
}

// Instances with n <= max_n are factored here; larger ones of a
// variable-size batch are left to the global-memory kernel.
template <typename T, int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB)
    k_potrf_smem(SizeArg sz, MatArg<T> C, MatArg<T> D, int *info, int max_n, int min_n) {
	extern __shared__ __align__(16) unsigned char smem[];
	const int b = blockIdx.x;
	const int n = sz.M(b);
	if (n <= 0 || n > max_n || n <= min_n) return;
	PotrfSmem pl = potrf_smem_plan<T>(max_n);
	T *S = (T *)smem;
	double *dinv = (double *)(smem + pl.dinv_off);
	T *Lt = (T *)(smem + pl.lt_off);
	int *bad = (int *)(smem + pl.bad_off);
	const PMat<T> c = C.get(b), d = D.get(b);
	if (threadIdx.x == 0) *bad = 0;
	if ((c.ri & 3) == 0)
		load_lp_vec<T, T, 4>(S, n, c.p + (size_t)c.ri * c.cn + 4 * c.cj, c.cn, nullptr);
	else
		load_lower_panels<T>(S, n, c);
	__syncthreads();
	chol_smem<T>(S, n, dinv, Lt, bad, false);
	if ((d.ri & 3) == 0)
		store_lp_vec<T, 4>(S, n, d.p + (size_t)d.ri * d.cn + 4 * d.cj, d.cn);
	else
		store_lower_panels<T>(S, n, d);
	for (int j = threadIdx.x; j < n; j += blockDim.x) d.d[j] = (T)dinv[j];
	if (info && threadIdx.x == 0) info[b] = *bad;
}

// unblocked right-looking Cholesky in global memory (any size)
template <typename T>
__global__ void __launch_bounds__(256) k_potrf_global(SizeArg sz, MatArg<T> C, MatArg<T> D, int *info, int min_n) {
	__shared__ double s_inv;
	__shared__ int s_bad;
	const int b = blockIdx.x;
	const int n = sz.M(b);
	if (n <= 0 || n <= min_n) return;
	const PMat<T> c = C.get(b), d = D.get(b);
	const int tid = threadIdx.x, nt = blockDim.x;
	const int warp = tid >> 5, lane = tid & 31, nw = nt >> 5;
	for (int j = warp; j < n; j += nw)
		for (int i = j + lane; i < n; i += 32) d.at(i, j) = c.at(i, j);
	if (tid == 0) s_bad = 0;
	__syncthreads();
	for (int j = 0; j < n; j++) {
		if (tid == 0) {
			double dd, inv;
			double cc = (double)d.at(j, j);
			chol_pivot(cc, dd, inv);
			if (!(cc > 0.0) && s_bad == 0) s_bad = j + 1;
			d.at(j, j) = (T)dd;
			d.d[j] = (T)inv;
			s_inv = inv;
		}
		__syncthreads();
		const T inv = (T)s_inv;
		for (int i = j + 1 + tid; i < n; i += nt) d.at(i, j) *= inv;
		__syncthreads();
		for (int l = j + 1 + warp; l < n; l += nw) {
			const T djl = d.at(l, j);
			for (int i = l + lane; i < n; i += 32) d.at(i, l) = fma(-d.at(i, j), djl, d.at(i, l));
		}
		__syncthreads();
	}
	if (info && tid == 0) info[b] = s_bad;
}

// Cholesky of the m x n lower trapezoid (potrf_l_mn, blasfeo_hp_pm/
// d_lapack_lib4.c:1155; blasfeo_ref/x_lapack_ref.c:185): the first n columns of
// chol, rows n..m-1 of them solved against the n x n factor; same pivot rule
// and inverse diagonal as potrf_l.  One CTA per instance, right-looking in
// global memory (L1/L2 resident at these sizes).
template <typename T>
__global__ void __launch_bounds__(256) k_potrf_mn(SizeArg sz, MatArg<T> C, MatArg<T> D, int *info) {
	__shared__ double s_inv;
	__shared__ int s_bad;
	const int b = blockIdx.x;
	const int m = sz.M(b);
	const int n = sz.N(b) < m ? sz.N(b) : m;
	if (m <= 0 || n <= 0) return;
	const PMat<T> c = C.get(b), d = D.get(b);
	const int tid = threadIdx.x, nt = blockDim.x;
	const int warp = tid >> 5, lane = tid & 31, nw = nt >> 5;
	for (int j = warp; j < n; j += nw)
		for (int i = j + lane; i < m; i += 32) d.at(i, j) = c.at(i, j);
	if (tid == 0) s_bad = 0;
	__syncthreads();
	for (int j = 0; j < n; j++) {
		if (tid == 0) {
			double dd, inv;
			double cc = (double)d.at(j, j);
			chol_pivot(cc, dd, inv);
			if (!(cc > 0.0) && s_bad == 0) s_bad = j + 1;
			d.at(j, j) = (T)dd;
			d.d[j] = (T)inv;
			s_inv = inv;
		}
		__syncthreads();
		const T inv = (T)s_inv;
		for (int i = j + 1 + tid; i < m; i += nt) d.at(i, j) *= inv;
		__syncthreads();
		for (int l = j + 1 + warp; l < n; l += nw) {
			const T djl = d.at(l, j);
			for (int i = l + lane; i < m; i += 32) d.at(i, l) = fma(-d.at(i, j), djl, d.at(i, l));
		}
		__syncthreads();
	}
	if (info && tid == 0) info[b] = s_bad;
}

// CTA-wide argmax of |x| with first-index tie-break; returns index (valid in all threads)
template <typename T>
__device__ int block_argmax_first(T v, int idx, int *s_idx, T *s_val) {
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
	for (int off = 16; off > 0; off >>= 1) {
		T ov = __shfl_down_sync(0xffffffffu, v, off);
		int oi = __shfl_down_sync(0xffffffffu, idx, off);
		if (ov > v || (ov == v && oi < idx)) {
			v = ov;
			idx = oi;
		}
	}
	if (lane == 0) {
		s_val[warp] = v;
		s_idx[warp] = idx;
	}
	__syncthreads();
	if (threadIdx.x == 0) {
		T bv = s_val[0];
		int bi = s_idx[0];
		for (int w = 1; w < nw; w++)
			if (s_val[w] > bv || (s_val[w] == bv && s_idx[w] < bi)) {
				bv = s_val[w];
				bi = s_idx[w];
			}
		s_idx[32] = bi;
	}
	__syncthreads();
	int r = s_idx[32];
	__syncthreads();
	return r;
}

// block_argmax_first with one barrier: every thread reduces the per-warp
// results itself.  Two calls must be separated by a __syncthreads (the
// per-warp slots are reused).
template <typename T>
__device__ int block_argmax_first1(T v, int idx, int *s_idx, T *s_val) {
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
	for (int off = 16; off > 0; off >>= 1) {
		T ov = __shfl_down_sync(0xffffffffu, v, off);
		int oi = __shfl_down_sync(0xffffffffu, idx, off);
		if (ov > v || (ov == v && oi < idx)) {
			v = ov;
			idx = oi;
		}
	}
	if (lane == 0) {
		s_val[warp] = v;
		s_idx[warp] = idx;
	}
	__syncthreads();
	T bv = s_val[0];
	int bi = s_idx[0];
	for (int w = 1; w < nw; w++)
		if (s_val[w] > bv || (s_val[w] == bv && s_idx[w] < bi)) {
			bv = s_val[w];
			bi = s_idx[w];
		}
	return bi;
}

// LU with row pivoting of one instance per CTA.  SMEM: the instance's m x n
// block is copied into shared memory (panel-major), factored there and
// copied back; only instances whose block fits in smem_cap bytes are taken.
// Global: factored in place in D; with smem_cap >= 0 only the instances that
// do not fit are taken (the other kernel of the launch has the rest).
template <typename T, int NT, bool SMEM>
__global__ void __launch_bounds__(NT) k_getrf(SizeArg sz, MatArg<T> C, MatArg<T> D, int *ipiv, long long ipiv_stride,
                                               int *info, int smem_cap, bool piv_on) {
	extern __shared__ __align__(16) unsigned char smem_raw[];
	__shared__ int s_idx[33];
	__shared__ T s_val[32];
	__shared__ int s_bad;
	const int b = blockIdx.x;
	const int m = sz.M(b), n = sz.N(b);
	if (m <= 0 || n <= 0) return;
	const bool fits = (size_t)((m + 3) / 4 * 4) * ((n + 3) / 4 * 4) * sizeof(T) <= (size_t)(smem_cap < 0 ? 0 : smem_cap);
	if (SMEM ? !fits : (smem_cap >= 0 && fits)) return;
	const PMat<T> c = C.get(b), dg = D.get(b);
	PMat<T> d = dg;
	if (SMEM) {
		d.p = (T *)smem_raw;
		d.cn = (n + 3) / 4 * 4;
		d.ri = d.cj = 0;
	}
	const int tid = threadIdx.x;
	int *piv = piv_on ? ipiv + ipiv_stride * b : nullptr;
	const int warp = tid >> 5, lane = tid & 31, nw = NT >> 5;
	for (int j = warp; j < n; j += nw)
		for (int i = lane; i < m; i += 32) d.at(i, j) = c.at(i, j);
	if (tid == 0) s_bad = 0;
	__syncthreads();
	const int mn = m < n ? m : n;
	for (int j = 0; j < mn; j++) {
		int ip = j;
		if (piv_on) {
			// pivot search over rows j..m-1
			T best = T(-1);
			int bi = INT_MAX;
			for (int i = j + tid; i < m; i += NT) {
				T a = dev_abs(d.at(i, j));
				if (a > best) {
					best = a;
					bi = i;
				}
			}
			ip = block_argmax_first<T>(best, bi, s_idx, s_val);
			if (ip >= m) ip = j;  // no candidate compared above -1: a column of NaNs
			if (ip != j)
				for (int l = tid; l < n; l += NT) {
					T t = d.at(j, l);
					d.at(j, l) = d.at(ip, l);
					d.at(ip, l) = t;
				}
		}
		__syncthreads();
		const T p = d.at(j, j);
		// getrf_rp: a zero pivot gives inverse 0; getrf_np divides as the
		// reference does (blasfeo_ref/x_lapack_ref.c, REF_GETRF_NOPIVOT: 1.0/d_00)
		const T inv = piv_on ? ((p != T(0)) ? T(1) / p : T(0)) : T(1) / p;
		if (tid == 0) {
			if (piv_on) piv[j] = ip;
			dg.d[j] = inv;
			if (p == T(0) && s_bad == 0) s_bad = j + 1;
		}
		for (int i = j + 1 + tid; i < m; i += NT) d.at(i, j) *= inv;
		__syncthreads();
		for (int l = j + 1 + warp; l < n; l += nw) {
			const T ujl = d.at(j, l);
			for (int i = j + 1 + lane; i < m; i += 32) d.at(i, l) = fma(-d.at(i, j), ujl, d.at(i, l));
		}
		__syncthreads();
	}
	if (SMEM) {
		for (int j = warp; j < n; j += nw)
			for (int i = lane; i < m; i += 32) dg.at(i, j) = d.at(i, j);
	}
	if (info && tid == 0) info[b] = s_bad;
}

// D = A B + D on the FP64 tensor cores (mma.sync m8n8k4 f64): per lane one
// element of A (row lane/4, column lane%4), one of B (row lane%4, column
// lane/4) and two of D (row lane/4, columns 2 (lane%4) and 2 (lane%4) + 1)
__device__ __forceinline__ void lu_dmma(double &d0, double &d1, double a, double b) {
	asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
	             : "+d"(d0), "+d"(d1)
	             : "d"(a), "d"(b));
}

// 4 consecutive elements at an address aligned to 4 elements (a panel-layout
// column run of 4 rows), as vector accesses
__device__ __forceinline__ void ld_run4(const double *p, double &a, double &b, double &c, double &d) {
	const double2 x = *reinterpret_cast<const double2 *>(p), y = *reinterpret_cast<const double2 *>(p + 2);
	a = x.x;
	b = x.y;
	c = y.x;
	d = y.y;
}
__device__ __forceinline__ void ld_run4(const float *p, float &a, float &b, float &c, float &d) {
	const float4 x = *reinterpret_cast<const float4 *>(p);
	a = x.x;
	b = x.y;
	c = x.z;
	d = x.w;
}
__device__ __forceinline__ void st_run4(double *p, double a, double b, double c, double d) {
	*reinterpret_cast<double2 *>(p) = make_double2(a, b);
	*reinterpret_cast<double2 *>(p + 2) = make_double2(c, d);
}
__device__ __forceinline__ void st_run4(float *p, float a, float b, float c, float d) {
	*reinterpret_cast<float4 *>(p) = make_float4(a, b, c, d);
}

// LU with row pivoting of one instance per CTA whose block stays in global
// memory (L2), blocked by 16-column panels (the reference's HP driver is
// blocked too: kernel_dgetrf_pivot panels and kernel_dgemm_nn corrections,
// blasfeo_hp_pm/d_lapack_lib4.c:2396-3431).  Per panel c0:
//   a. the panel (rows c0..m-1, 16 columns) is staged in shared memory;
//   b. it is factored there column by column: pivot = first row of the largest
//      |a| (kernel/generic/kernel_dgetrf_pivot_lib4.c:84-165), row swap inside
//      the panel, scaling by the reciprocal pivot (0 for a zero pivot;
//      getrf_np divides), rank-1 update of the panel's later columns -- two
//      barriers per column, each thread scaling and updating its own rows and
//      finding their candidate for the next pivot;
//   c. the panel goes back to global memory;
//   d. its row swaps, in order, are one permutation of at most 32 rows,
//      applied to the columns outside the panel (one thread per column, all
//      loads before the stores);
//   e. U12 = L11^{-1} A12 for the columns right of the panel (one thread per
//      column, unit lower L11 from shared memory), kept in shared memory;
//   f. A22 -= L21 U12 as 4 x 4 register tiles (rank-16 update, 4-row tiles of
//      the panel layout, consecutive threads on consecutive column tiles, the
//      next tile's loads in flight under the current tile's products).
// Shared memory: (m + 4) x 17 panel, 16 x (n + 4) U12, m + 4 ints.  MINB
// blocks per SM cap the registers (the variants differ in it).
template <typename T, int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB) k_getrf_blk(SizeArg sz, MatArg<T> C, MatArg<T> D, int *ipiv,
                                                   long long ipiv_stride, int *info, int smem_cap, int max_m,
                                                   bool piv_on) {
	extern __shared__ __align__(16) unsigned char smem_raw[];
	__shared__ int s_idx[33];
	__shared__ T s_val[32];
	__shared__ int s_bad;
	__shared__ int s_piv[16];
	__shared__ int s_rows[32], s_from[32], s_nmv;
	const int b = blockIdx.x;
	const int m = sz.M(b), n = sz.N(b);
	if (m <= 0 || n <= 0) return;
	// instances whose whole block fits the shared-memory kernel are its work
	const bool fits = (size_t)((m + 3) / 4 * 4) * ((n + 3) / 4 * 4) * sizeof(T) <= (size_t)(smem_cap < 0 ? 0 : smem_cap);
	if (smem_cap >= 0 && fits) return;
	const PMat<T> c = C.get(b), d = D.get(b);
	const int tid = threadIdx.x;
	int *piv = piv_on ? ipiv + ipiv_stride * b : nullptr;
	T *P = (T *)smem_raw;                        // panel: row r at P + 17 r
	// U12: row k at Us + k * usld, its column l at slot (l % 4) * q4 + l / 4, so
	// that the update's threads (consecutive 4-column tiles) read consecutive
	// slots for each of a tile's 4 columns (no bank conflict)
	T *Us = P + (size_t)(max_m + 4) * 17;
	const int usld = n + 4, q4 = usld / 4;
	int *cont = (int *)(Us + (size_t)16 * usld);  // row permutation of a panel (max_m + 4 ints)
	// D = C first (in place afterwards)
	if (c.p != d.p || c.ri != d.ri || c.cj != d.cj) {
		for (int e = tid; e < m * n; e += NT) {
			const int i = e % m, j = e / m;
			d.at(i, j) = c.at(i, j);
		}
	}
	if (tid == 0) s_bad = 0;
	__syncthreads();
	const int mn = m < n ? m : n;
	for (int c0 = 0; c0 < mn; c0 += 16) {
		const int w = mn - c0 < 16 ? mn - c0 : 16;
		const int pr = m - c0;
		// a. stage the panel
		for (int e = tid; e < pr * 16; e += NT) {
			const int r = e >> 4, j = e & 15;
			P[r * 17 + j] = (j < w) ? d.at(c0 + r, c0 + j) : T(0);
		}
		__syncthreads();
		// b. factor it: per column one barrier for the pivot search and one
		// after the row swap; each thread scales and updates its own rows
		// (r = j+1+tid, +NT, ...) against the pivot row and tracks their
		// largest |entry| of the next column for the next pivot search
		T best = T(-1);
		int bi = INT_MAX;
		if (piv_on)
			for (int r = tid; r < pr; r += NT) {
				const T a = dev_abs(P[r * 17]);
				if (a > best) {
					best = a;
					bi = r;
				}
			}
		for (int j = 0; j < w; j++) {
			int ip = j;
			if (piv_on) {
				ip = block_argmax_first1<T>(best, bi, s_idx, s_val);
				if (ip >= pr) ip = j;  // no candidate compared above -1: a column of NaNs
				if (ip != j && tid < 16) {
					const T t = P[j * 17 + tid];
					P[j * 17 + tid] = P[ip * 17 + tid];
					P[ip * 17 + tid] = t;
				}
			}
			if (tid == 0) s_piv[j] = c0 + ip;
			__syncthreads();
			const T pv = P[j * 17 + j];
			const T inv = piv_on ? ((pv != T(0)) ? T(1) / pv : T(0)) : T(1) / pv;
			if (tid == 0) {
				if (piv_on) piv[c0 + j] = c0 + ip;
				d.d[c0 + j] = inv;
				if (pv == T(0) && s_bad == 0) s_bad = c0 + j + 1;
			}
			T urow[16];
#pragma unroll
			for (int l = 0; l < 16; l++) urow[l] = (l > j && l < w) ? P[j * 17 + l] : T(0);
			best = T(-1);
			bi = INT_MAX;
			for (int r = j + 1 + tid; r < pr; r += NT) {
				T *row = P + r * 17;
				const T lj = row[j] * inv;
				row[j] = lj;
#pragma unroll
				for (int l = 0; l < 16; l++)
					if (l > j && l < w) row[l] = fma(-lj, urow[l], row[l]);
				if (j + 1 < w) {
					const T a = dev_abs(row[j + 1]);
					if (a > best) {
						best = a;
						bi = r;
					}
				}
			}
		}
		__syncthreads();
		// c. panel back to global memory
		for (int e = tid; e < pr * w; e += NT) {
			const int r = e / w, j = e % w;
			d.at(c0 + r, c0 + j) = P[r * 17 + j];
		}
		// d. the panel's row swaps on the other columns: the 16 swaps in order
		// make one permutation of at most 32 rows.  cont[r] (shared, one int
		// per panel row) starts as r; thread 0 runs the swaps on it; the rows
		// that received another row's content (s_rows[k] gets the old row
		// s_from[k]) are collected in parallel; each column thread then
		// loads all of them before it stores any.
		if (piv_on) {
			for (int r = tid; r < pr; r += NT) cont[r] = r;
			if (tid == 0) s_nmv = 0;
			__syncthreads();
			if (tid == 0) {
				for (int j = 0; j < w; j++) {
					const int r2 = s_piv[j] - c0;
					if (r2 == j) continue;
					const int t = cont[j];
					cont[j] = cont[r2];
					cont[r2] = t;
				}
			}
			__syncthreads();
			if (tid < 2 * w) {
				// candidates: the panel rows, and the pivot rows below them
				// (each once: the first j that names it)
				int r = -1;
				if (tid < w) {
					r = tid;
				} else {
					const int r2 = s_piv[tid - w] - c0;
					bool first = r2 >= w;
					for (int j = 0; j < tid - w && first; j++)
						if (s_piv[j] - c0 == r2) first = false;
					if (first) r = r2;
				}
				if (r >= 0 && cont[r] != r) {
					const int k = atomicAdd(&s_nmv, 1);
					s_rows[k] = c0 + r;
					s_from[k] = c0 + cont[r];
				}
			}
			__syncthreads();
			const int nmv = s_nmv;
			for (int l = tid; l < n; l += NT) {
				if (l >= c0 && l < c0 + w) continue;
				T v[32];
#pragma unroll
				for (int k = 0; k < 32; k++)
					if (k < nmv) v[k] = d.at(s_from[k], l);
#pragma unroll
				for (int k = 0; k < 32; k++)
					if (k < nmv) d.at(s_rows[k], l) = v[k];
			}
		}
		__syncthreads();
		// e. U12 = L11^{-1} A12 (unit lower L11)
		const int nr = n - c0 - w;
		// a full panel's 16 rows of a column are 4 aligned runs of 4 when the
		// panel starts on a panel boundary: vector accesses then
		const bool vecu = w == 16 && ((d.ri + c0) & 3) == 0 && ((uintptr_t)d.p & 15) == 0;
		for (int l = tid; l < nr; l += NT) {
			T u[16];
			if (vecu) {
#pragma unroll
				for (int k = 0; k < 16; k += 4) ld_run4(d.addr(c0 + k, c0 + w + l), u[k], u[k + 1], u[k + 2], u[k + 3]);
			} else {
#pragma unroll
				for (int k = 0; k < 16; k++) u[k] = (k < w) ? d.at(c0 + k, c0 + w + l) : T(0);
			}
#pragma unroll
			for (int k = 1; k < 16; k++)
#pragma unroll
				for (int kk = 0; kk < k; kk++) u[k] = fma(-P[k * 17 + kk], u[kk], u[k]);
			if (vecu) {
#pragma unroll
				for (int k = 0; k < 16; k += 4) st_run4(d.addr(c0 + k, c0 + w + l), u[k], u[k + 1], u[k + 2], u[k + 3]);
			}
#pragma unroll
			for (int k = 0; k < 16; k++) {
				if (!vecu && k < w) d.at(c0 + k, c0 + w + l) = u[k];
				Us[k * usld + (l & 3) * q4 + (l >> 2)] = (k < w) ? u[k] : T(0);
			}
		}
		__syncthreads();
		// f. A22 -= L21 U12 (rows c0 + w.., columns c0 + w..).  FP64: a 32 x 32
		// tile per warp as 4 x 4 DMMA fragments, L21 from the panel and U12 from
		// shared memory (one fragment load per 256 products), C from and back
		// to global memory.  FP32: a 4 x 4 tile per thread and step; the next
		// tile's loads are issued before this one's products, so a thread
		// always has one tile's L2 round trip in flight
		const int rows = pr - w;
		if constexpr (sizeof(T) == 8) {
			if (rows > 0 && nr > 0) {
				const int nrt = (rows + 31) >> 5, nct = (nr + 31) >> 5;
				const int lane = tid & 31, warp = tid >> 5, nw = NT >> 5;
				const int g = lane >> 2, tq = lane & 3;
				for (int t = warp; t < nrt * nct; t += nw) {
					const int r0 = w + 32 * (t / nct), l0 = 32 * (t % nct);
					double acc[4][4][2];
#pragma unroll
					for (int rb = 0; rb < 4; rb++) {
						const int row = r0 + 8 * rb + g;
#pragma unroll
						for (int cb = 0; cb < 4; cb++) {
							const int col = l0 + 8 * cb + 2 * tq;
							acc[rb][cb][0] = (row < pr && col < nr) ? d.at(c0 + row, c0 + w + col) : 0.0;
							acc[rb][cb][1] = (row < pr && col + 1 < nr) ? d.at(c0 + row, c0 + w + col + 1) : 0.0;
						}
					}
#pragma unroll
					for (int ks = 0; ks < 4; ks++) {
						double a[4], bb[4];
#pragma unroll
						for (int rb = 0; rb < 4; rb++) {
							const int row = r0 + 8 * rb + g;
							a[rb] = (row < pr) ? -(double)P[row * 17 + 4 * ks + tq] : 0.0;
						}
#pragma unroll
						for (int cb = 0; cb < 4; cb++) {
							const int col = l0 + 8 * cb + g;
							bb[cb] = (col < nr) ? (double)Us[(4 * ks + tq) * usld + (col & 3) * q4 + (col >> 2)] : 0.0;
						}
#pragma unroll
						for (int rb = 0; rb < 4; rb++)
#pragma unroll
							for (int cb = 0; cb < 4; cb++) lu_dmma(acc[rb][cb][0], acc[rb][cb][1], a[rb], bb[cb]);
					}
#pragma unroll
					for (int rb = 0; rb < 4; rb++) {
						const int row = r0 + 8 * rb + g;
#pragma unroll
						for (int cb = 0; cb < 4; cb++) {
							const int col = l0 + 8 * cb + 2 * tq;
							if (row < pr && col < nr) d.at(c0 + row, c0 + w + col) = (T)acc[rb][cb][0];
							if (row < pr && col + 1 < nr) d.at(c0 + row, c0 + w + col + 1) = (T)acc[rb][cb][1];
						}
					}
				}
			}
		} else if (rows > 0 && nr > 0) {
			const int ntr = (rows + 3) >> 2, ntc = (nr + 3) >> 2, ntt = ntr * ntc;
			// a tile's 4 rows of one column are one aligned 4-element run of the
			// panel layout when its first row is on a panel boundary (tile rows
			// start at c0 + w + 4 ti) and pA is 16-byte aligned: vector loads
			// and stores then (full tiles), element by element otherwise
			const bool vec = ((d.ri + c0 + w) & 3) == 0 && ((uintptr_t)d.p & 15) == 0;
			auto load_tile = [&](int t, T (&v)[4][4]) {
				const int ti = t / ntc, tj = t % ntc;
				const int r0 = w + 4 * ti, l0 = 4 * tj;
				if (vec && r0 + 4 <= pr) {
#pragma unroll
					for (int q = 0; q < 4; q++) {
						if (l0 + q < nr)
							ld_run4(d.addr(c0 + r0, c0 + w + l0 + q), v[0][q], v[1][q], v[2][q], v[3][q]);
						else
							v[0][q] = v[1][q] = v[2][q] = v[3][q] = T(0);
					}
					return;
				}
#pragma unroll
				for (int a = 0; a < 4; a++)
#pragma unroll
					for (int q = 0; q < 4; q++)
						v[a][q] = (r0 + a < pr && l0 + q < nr) ? d.at(c0 + r0 + a, c0 + w + l0 + q) : T(0);
			};
			T nxt[4][4];
			if (tid < ntt) load_tile(tid, nxt);
			for (int t = tid; t < ntt; t += NT) {
				const int ti = t / ntc, tj = t % ntc;
				const int r0 = w + 4 * ti, l0 = 4 * tj;
				T acc[4][4];
#pragma unroll
				for (int a = 0; a < 4; a++)
#pragma unroll
					for (int q = 0; q < 4; q++) acc[a][q] = nxt[a][q];
				if (t + NT < ntt) load_tile(t + NT, nxt);
#pragma unroll
				for (int k = 0; k < 16; k++) {
					T av[4], bv[4];
#pragma unroll
					for (int a = 0; a < 4; a++) av[a] = (r0 + a < pr) ? P[(r0 + a) * 17 + k] : T(0);
#pragma unroll
					for (int q = 0; q < 4; q++) bv[q] = Us[k * usld + q * q4 + tj];
#pragma unroll
					for (int a = 0; a < 4; a++)
#pragma unroll
						for (int q = 0; q < 4; q++) acc[a][q] = fma(-av[a], bv[q], acc[a][q]);
				}
				if (vec && r0 + 4 <= pr) {
#pragma unroll
					for (int q = 0; q < 4; q++)
						if (l0 + q < nr) st_run4(d.addr(c0 + r0, c0 + w + l0 + q), acc[0][q], acc[1][q], acc[2][q], acc[3][q]);
				} else {
#pragma unroll
					for (int a = 0; a < 4; a++)
#pragma unroll
						for (int q = 0; q < 4; q++)
							if (r0 + a < pr && l0 + q < nr) d.at(c0 + r0 + a, c0 + w + l0 + q) = acc[a][q];
				}
			}
		}
		__syncthreads();
	}
	if (info && tid == 0) info[b] = s_bad;
}

template <typename T>
__device__ T block_sum(T v, T *s_red) {
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
	for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
	if (lane == 0) s_red[warp] = v;
	__syncthreads();
	if (threadIdx.x == 0) {
		T s = T(0);
		for (int w = 0; w < nw; w++) s += s_red[w];
		s_red[32] = s;
	}
	__syncthreads();
	T r = s_red[32];
	__syncthreads();
	return r;
}

// Householder QR of one instance per CTA (shared or global memory, as k_getrf).
template <typename T, int NT, bool SMEM>
__global__ void __launch_bounds__(NT) k_geqrf(SizeArg sz, MatArg<T> C, MatArg<T> D, int smem_cap) {
	extern __shared__ __align__(16) unsigned char smem_raw[];
	__shared__ T s_red[33];
	__shared__ T s_tau, s_sc, s_beta;
	const int b = blockIdx.x;
	const int m = sz.M(b), n = sz.N(b);
	if (m <= 0 || n <= 0) return;
	const bool fits = (size_t)((m + 3) / 4 * 4) * ((n + 3) / 4 * 4) * sizeof(T) <= (size_t)(smem_cap < 0 ? 0 : smem_cap);
	if (SMEM ? !fits : (smem_cap >= 0 && fits)) return;
	const PMat<T> c = C.get(b), dg = D.get(b);
	PMat<T> d = dg;
	if (SMEM) {
		d.p = (T *)smem_raw;
		d.cn = (n + 3) / 4 * 4;
		d.ri = d.cj = 0;
	}
	T *tau = dg.d + dg.ri;
	const int tid = threadIdx.x;
	const int warp = tid >> 5, lane = tid & 31, nw = NT >> 5;
	for (int j = warp; j < n; j += nw)
		for (int i = lane; i < m; i += 32) d.at(i, j) = c.at(i, j);
	__syncthreads();
	const int kmax = m < n ? m : n;
	for (int j = 0; j < kmax; j++) {
		T part = T(0);
		for (int i = j + 1 + tid; i < m; i += NT) {
			T x = d.at(i, j);
			part = fma(x, x, part);
		}
		const T s = block_sum<T>(part, s_red);
		if (tid == 0) {
			if (s == T(0)) {
				s_tau = T(0);
				s_sc = T(1);
				s_beta = d.at(j, j);
			} else {
				T alpha = d.at(j, j);
				T beta = sqrt(fma(alpha, alpha, s));
				if (alpha > T(0)) beta = -beta;
				s_tau = (beta - alpha) / beta;
				s_sc = T(1) / (alpha - beta);
				s_beta = beta;
			}
			tau[j] = s_tau;
		}
		__syncthreads();
		const T t = s_tau;
		if (s != T(0)) {
			for (int i = j + 1 + tid; i < m; i += NT) d.at(i, j) *= s_sc;
			if (tid == 0) d.at(j, j) = s_beta;
		}
		__syncthreads();
		// apply the reflector: one warp per trailing column, lanes over rows
		for (int col = j + 1 + warp; col < n; col += nw) {
			T w = T(0);
			for (int i = j + 1 + lane; i < m; i += 32) w = fma(d.at(i, j), d.at(i, col), w);
#pragma unroll
			for (int off = 16; off > 0; off >>= 1) w += __shfl_xor_sync(0xffffffffu, w, off);
			w = -t * (w + d.at(j, col));
			for (int i = j + 1 + lane; i < m; i += 32) d.at(i, col) = fma(w, d.at(i, j), d.at(i, col));
			__syncwarp();
			if (lane == 0) d.at(j, col) += w;
		}
		__syncthreads();
	}
	if (SMEM) {
		for (int j = warp; j < n; j += nw)
			for (int i = lane; i < m; i += 32) dg.at(i, j) = d.at(i, j);
	}
}

// shared memory of the blocked QR: the panel, then (FP64) the V^T C buffer
__host__ __device__ inline size_t qr_panel_bytes(int max_m, size_t esz) {
	return ((size_t)(max_m + 4) * 17 * esz + 15) / 16 * 16;
}
// the trailing columns are updated in chunks of at most QR_CHUNK_CB 32-column
// blocks, so the buffer stays bounded for wide matrices
constexpr int QR_CHUNK_CB = 8;
__host__ __device__ inline int qr_w_slots(int nt, int max_n) {
	const int nw = nt / 32, ncb0 = (max_n + 31) / 32;
	const int ncb = ncb0 < QR_CHUNK_CB ? ncb0 : QR_CHUNK_CB;
	return 512 * (nw > ncb ? nw : ncb);
}

// V(r, k) of the panel's unit lower trapezoidal reflector block (P: rows of 17)
__device__ __forceinline__ double qr_v(const double *P, int r, int k) {
	return (r > k) ? P[r * 17 + k] : ((r == k) ? 1.0 : 0.0);
}

// C = C - V T^T (V^T C) on the FP64 tensor cores for the trailing columns of
// a 16-column panel (rows c0.. of the panel layout, columns c0 + w ..):
// P holds V (pr rows), Tm the 16 x 16 upper triangular T, Wsm the partial
// sums.  Every thread of the CTA calls it; it ends with a barrier.
__device__ __noinline__ void qr_update_dmma(const PMat<double> &d, const double *P, const double *Tm, double *Wsm, int c0, int w,
                               int pr, int nr_all, int NT) {
	const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = NT >> 5;
	const int g = lane >> 2, tq = lane & 3;
	for (int cc = 0; cc < nr_all; cc += 32 * QR_CHUNK_CB) {
		// this chunk's columns: c0 + wc .. (wc = w + cc), nr of them
		const int nr = min(32 * QR_CHUNK_CB, nr_all - cc), wc = w + cc;
		const int ncb = (nr + 31) >> 5;
		const int nsplit = nw / ncb > 1 ? nw / ncb : 1;
		// rows per split, a multiple of 4 (the DMMA k step)
		const int rsz = ((pr + nsplit - 1) / nsplit + 3) & ~3;
		const int wld = 32 * ncb;  // row stride of one 16 x wld partial block
		// e1. partial W blocks: task (cb, sp) -> rows [sp rsz, (sp+1) rsz), columns [32 cb, 32 cb + 32)
		for (int task = warp; task < ncb * nsplit; task += nw) {
			const int cb = task % ncb, sp = task / ncb;
			const int l0 = 32 * cb, rb0 = sp * rsz, rb1 = min(pr, rb0 + rsz);
			double acc[2][4][2];
	#pragma unroll
			for (int mb = 0; mb < 2; mb++)
	#pragma unroll
				for (int nb = 0; nb < 4; nb++) acc[mb][nb][0] = acc[mb][nb][1] = 0.0;
	#pragma unroll 2
			for (int r = rb0; r < rb1; r += 4) {
				const int row = r + tq;
				double a[2], b[4];
	#pragma unroll
				for (int mb = 0; mb < 2; mb++) a[mb] = (row < pr) ? qr_v(P, row, 8 * mb + g) : 0.0;
	#pragma unroll
				for (int nb = 0; nb < 4; nb++) {
					const int col = l0 + 8 * nb + g;
					b[nb] = (row < pr && col < nr) ? d.at(c0 + row, c0 + wc + col) : 0.0;
				}
	#pragma unroll
				for (int mb = 0; mb < 2; mb++)
	#pragma unroll
					for (int nb = 0; nb < 4; nb++) lu_dmma(acc[mb][nb][0], acc[mb][nb][1], a[mb], b[nb]);
			}
			double *wp = Wsm + (size_t)sp * 16 * wld;
	#pragma unroll
			for (int mb = 0; mb < 2; mb++)
	#pragma unroll
				for (int nb = 0; nb < 4; nb++) {
					const int k = 8 * mb + g, col = l0 + 8 * nb + 2 * tq;
					wp[k * wld + col] = acc[mb][nb][0];
					wp[k * wld + col + 1] = acc[mb][nb][1];
				}
		}
		__syncthreads();
		// e2. W = sum of the partials (split order), then W <- T^T W, a thread per column
		for (int col = tid; col < nr; col += NT) {
			double wv[16];
	#pragma unroll
			for (int k = 0; k < 16; k++) {
				double sacc = Wsm[k * wld + col];
				for (int sp = 1; sp < nsplit; sp++) sacc += Wsm[(size_t)sp * 16 * wld + k * wld + col];
				wv[k] = sacc;
			}
	#pragma unroll
			for (int k = 15; k >= 0; k--) {
				double z = 0.0;
	#pragma unroll
				for (int q = 0; q <= k; q++) z = fma(Tm[q * 17 + k], wv[q], z);
				wv[k] = z;
			}
	#pragma unroll
			for (int k = 0; k < 16; k++) Wsm[k * wld + col] = wv[k];
		}
		__syncthreads();
		// e3. C -= V W, 32 x 32 tiles
		const int nrt = (pr + 31) >> 5;
		for (int t = warp; t < nrt * ncb; t += nw) {
			const int r0 = 32 * (t / ncb), l0 = 32 * (t % ncb);
			double acc[4][4][2];
	#pragma unroll
			for (int rb = 0; rb < 4; rb++) {
				const int row = r0 + 8 * rb + g;
	#pragma unroll
				for (int cb = 0; cb < 4; cb++) {
					const int col = l0 + 8 * cb + 2 * tq;
					acc[rb][cb][0] = (row < pr && col < nr) ? d.at(c0 + row, c0 + wc + col) : 0.0;
					acc[rb][cb][1] = (row < pr && col + 1 < nr) ? d.at(c0 + row, c0 + wc + col + 1) : 0.0;
				}
			}
	#pragma unroll
			for (int ks = 0; ks < 4; ks++) {
				double a[4], b[4];
	#pragma unroll
				for (int rb = 0; rb < 4; rb++) {
					const int row = r0 + 8 * rb + g;
					a[rb] = (row < pr) ? -qr_v(P, row, 4 * ks + tq) : 0.0;
				}
	#pragma unroll
				for (int cb = 0; cb < 4; cb++) {
					const int col = l0 + 8 * cb + g;
					b[cb] = (col < nr) ? Wsm[(4 * ks + tq) * wld + col] : 0.0;
				}
	#pragma unroll
				for (int rb = 0; rb < 4; rb++)
	#pragma unroll
					for (int cb = 0; cb < 4; cb++) lu_dmma(acc[rb][cb][0], acc[rb][cb][1], a[rb], b[cb]);
			}
	#pragma unroll
			for (int rb = 0; rb < 4; rb++) {
				const int row = r0 + 8 * rb + g;
	#pragma unroll
				for (int cb = 0; cb < 4; cb++) {
					const int col = l0 + 8 * cb + 2 * tq;
					if (row < pr && col < nr) d.at(c0 + row, c0 + wc + col) = acc[rb][cb][0];
					if (row < pr && col + 1 < nr) d.at(c0 + row, c0 + wc + col + 1) = acc[rb][cb][1];
				}
			}
		}
		__syncthreads();
	}
}

// Householder QR of one instance per CTA whose block stays in global memory
// (L2), blocked by 16-column panels with the compact WY form of the panel's
// reflectors (the reference's HP driver applies 4-column blocks with
// kernel_dlarf_t_4_lib4, blasfeo_hp_pm/d_lapack_lib4.c:3444 and
// kernel/generic/kernel_dgeqrf_4_lib4.c:1030).  Per panel c0:
//   a. the panel (rows c0..m-1, 16 columns) is staged in shared memory;
//   b. it is factored there column by column with the reflector convention of
//      dlarfg (kernel/generic/kernel_dgeqrf_4_lib4.c:80-96: beta = -sign(alpha)
//      ||(alpha, x)||, tau = (beta - alpha) / beta, v = x / (alpha - beta);
//      tau = 0 when x = 0), each reflector applied to the panel's later columns;
//   c. panel and tau go back to global memory;
//   d. T (upper triangular, H_0 H_1 .. H_15 = I - V T V^T) from V^T V:
//      T_jj = tau_j, T_{0:j,j} = -tau_j T_{0:j,0:j} (V^T v_j)_{0:j};
//      (lane k of warp 0 computes row k of T: the rows are independent);
//   e. the trailing columns C = A(c0:m, c0+16:n) become Q^T C = C - V T^T (V^T C),
//      a warp per pair of columns with its lanes over the rows (V^T C by
//      butterfly sums; the update's next rows loaded before the current ones
//      are stored).
// Shared memory: (m + 4) x 17 panel, 16 x 17 T and V^T V.
// DMMA: the trailing update on the FP64 tensor cores (FP64 only; needs the
// V^T C buffer and more registers, so it pays from ~128 x 256 blocks on)
// FP64 with DMMA at 256 threads: 128 registers (a few spilled) for 2 CTAs per
// SM: 2.18 -> 2.90 TF/s at 256 x 128, 3.29 -> 3.87 at 384 x 192 against the
// 512-thread variant that the size rule took before
template <typename T, int NT, bool DMMA>
__global__ void __launch_bounds__(NT, (DMMA && NT == 256 && sizeof(T) == 8) ? 2 : 1) k_geqrf_blk(SizeArg sz, MatArg<T> C, MatArg<T> D, int smem_cap, int max_m,
                                                   int max_n) {
	extern __shared__ __align__(16) unsigned char smem_raw[];
	__shared__ T s_red[33];
	__shared__ T s_tau, s_sc, s_beta;
	__shared__ T Tm[16 * 17];
	__shared__ T G[16 * 17];
	const int b = blockIdx.x;
	const int m = sz.M(b), n = sz.N(b);
	if (m <= 0 || n <= 0) return;
	const bool fits = (size_t)((m + 3) / 4 * 4) * ((n + 3) / 4 * 4) * sizeof(T) <= (size_t)(smem_cap < 0 ? 0 : smem_cap);
	if (smem_cap >= 0 && fits) return;
	const PMat<T> c = C.get(b), d = D.get(b);
	T *tau = d.d + d.ri;
	const int tid = threadIdx.x;
	const int warp = tid >> 5, lane = tid & 31, nw = NT >> 5;
	T *P = (T *)smem_raw;  // panel: row r at P + 17 r
	// FP64: V^T C partial sums (qr_w_slots(NT, max_n) doubles) after the panel
	double *Wsm = (double *)(smem_raw + qr_panel_bytes(max_m, sizeof(T)));
	if (c.p != d.p || c.ri != d.ri || c.cj != d.cj) {
		for (int e = tid; e < m * n; e += NT) {
			const int i = e % m, j = e / m;
			d.at(i, j) = c.at(i, j);
		}
	}
	__syncthreads();
	const int kmax = m < n ? m : n;
	for (int c0 = 0; c0 < kmax; c0 += 16) {
		const int w = kmax - c0 < 16 ? kmax - c0 : 16;
		const int pr = m - c0;
		// a. stage the panel
		for (int e = tid; e < pr * 16; e += NT) {
			const int r = e >> 4, j = e & 15;
			P[r * 17 + j] = (j < w) ? d.at(c0 + r, c0 + j) : T(0);
		}
		__syncthreads();
		// b. factor it
		for (int j = 0; j < w; j++) {
			T part = T(0);
			for (int r = j + 1 + tid; r < pr; r += NT) {
				const T x = P[r * 17 + j];
				part = fma(x, x, part);
			}
			const T sq = block_sum<T>(part, s_red);
			if (tid == 0) {
				if (sq == T(0)) {
					s_tau = T(0);
					s_sc = T(1);
					s_beta = P[j * 17 + j];
				} else {
					const T alpha = P[j * 17 + j];
					T beta = sqrt(fma(alpha, alpha, sq));
					if (alpha > T(0)) beta = -beta;
					s_tau = (beta - alpha) / beta;
					s_sc = T(1) / (alpha - beta);
					s_beta = beta;
				}
				tau[c0 + j] = s_tau;
			}
			__syncthreads();
			const T t = s_tau;
			if (sq != T(0)) {
				for (int r = j + 1 + tid; r < pr; r += NT) P[r * 17 + j] *= s_sc;
				if (tid == 0) P[j * 17 + j] = s_beta;
			}
			__syncthreads();
			for (int col = j + 1 + warp; col < w; col += nw) {
				T wv = T(0);
				for (int r = j + 1 + lane; r < pr; r += 32) wv = fma(P[r * 17 + j], P[r * 17 + col], wv);
#pragma unroll
				for (int off = 16; off > 0; off >>= 1) wv += __shfl_xor_sync(0xffffffffu, wv, off);
				wv = -t * (wv + P[j * 17 + col]);
				for (int r = j + 1 + lane; r < pr; r += 32) P[r * 17 + col] = fma(wv, P[r * 17 + j], P[r * 17 + col]);
				__syncwarp();
				if (lane == 0) P[j * 17 + col] += wv;
			}
			__syncthreads();
		}
		// c. panel back to global memory
		for (int e = tid; e < pr * w; e += NT) {
			const int r = e / w, j = e % w;
			d.at(c0 + r, c0 + j) = P[r * 17 + j];
		}
		const int nr = n - c0 - w;
		if (nr > 0) {
			// d. G = V^T V (strictly upper part), V unit lower trapezoidal in P:
			// a warp per column j, its lanes over the rows r >= j, all k < j at
			// once, butterfly sums
			for (int j = 1 + warp; j < w; j += nw) {
				T g[16];
#pragma unroll
				for (int k = 0; k < 16; k++) g[k] = T(0);
				for (int r = j + lane; r < pr; r += 32) {
					const T vj = (r == j) ? T(1) : P[r * 17 + j];
#pragma unroll
					for (int k = 0; k < 16; k++)
						if (k < j) g[k] = fma(P[r * 17 + k], vj, g[k]);
				}
#pragma unroll
				for (int k = 0; k < 16; k++)
#pragma unroll
					for (int off = 16; off > 0; off >>= 1) g[k] += __shfl_xor_sync(0xffffffffu, g[k], off);
				if (lane == 0) {
#pragma unroll
					for (int k = 0; k < 16; k++)
						if (k < j) G[k * 17 + j] = g[k];
				}
			}
			__syncthreads();
			// T row by row: lane k of warp 0 owns row k (T_kj for j >= k
			// depends only on row k and on G), so the 16 rows are independent
			if (tid < 16) {
				const int k = tid;
				T t[16];
#pragma unroll
				for (int j = 0; j < 16; j++) {
					const T tj = (j < w) ? tau[c0 + j] : T(0);
					T z = T(0);
#pragma unroll
					for (int q = 0; q < j; q++)
						if (q >= k) z = fma(t[q], G[q * 17 + j], z);
					// columns j >= w hold no reflector: exact zeros (G there is stale)
					t[j] = (j >= w || j < k) ? T(0) : ((j == k) ? tj : -tj * z);
				}
#pragma unroll
				for (int j = 0; j < 16; j++) Tm[k * 17 + j] = t[j];
			}
			__syncthreads();
			// e. C = C - V T^T (V^T C).  FP64 on the tensor cores (DMMA):
			//   e1. W = V^T C (16 x nr): a warp per 32-column block and row
			//       chunk (the rows split so that every warp has a task),
			//       partial sums in shared memory, added in a fixed order;
			//   e2. W <- T^T W, a thread per column;
			//   e3. C -= V W as 32 x 32 tiles per warp.
			// FP32: a warp per pair of trailing columns, its lanes over the
			// rows; w = V^T c by butterfly sums, then w <- T^T w in place, then
			// c -= V w with the next rows' loads issued before the current
			// rows' stores.
			if constexpr (sizeof(T) == 8 && DMMA) {
				qr_update_dmma(d, P, Tm, Wsm, c0, w, pr, nr, NT);
			} else
			for (int l0 = 2 * warp; l0 < nr; l0 += 2 * nw) {
				const bool two = l0 + 1 < nr;
				const int col0 = c0 + w + l0, col1 = col0 + (two ? 1 : 0);
				T w0[16], w1[16];
#pragma unroll
				for (int k = 0; k < 16; k++) w0[k] = w1[k] = T(0);
#pragma unroll 2
				for (int r = lane; r < pr; r += 32) {
					const T a0 = d.at(c0 + r, col0), a1 = d.at(c0 + r, col1);
#pragma unroll
					for (int k = 0; k < 16; k++) {
						// V(r, k): 1 on the diagonal, the stored vector below, 0 above
						const T v = (r > k) ? P[r * 17 + k] : ((r == k) ? T(1) : T(0));
						w0[k] = fma(v, a0, w0[k]);
						w1[k] = fma(v, a1, w1[k]);
					}
				}
#pragma unroll
				for (int k = 0; k < 16; k++)
#pragma unroll
					for (int off = 16; off > 0; off >>= 1) {
						w0[k] += __shfl_xor_sync(0xffffffffu, w0[k], off);
						w1[k] += __shfl_xor_sync(0xffffffffu, w1[k], off);
					}
#pragma unroll
				for (int k = 15; k >= 0; k--) {
					T z0 = T(0), z1 = T(0);
#pragma unroll
					for (int q = 0; q <= k; q++) {
						const T tq = Tm[q * 17 + k];
						z0 = fma(tq, w0[q], z0);
						z1 = fma(tq, w1[q], z1);
					}
					w0[k] = z0;
					w1[k] = z1;
				}
				int r = lane;
				T a0 = T(0), a1 = T(0);
				if (r < pr) {
					a0 = d.at(c0 + r, col0);
					a1 = d.at(c0 + r, col1);
				}
				while (r < pr) {
					const int rn = r + 32;
					T n0 = T(0), n1 = T(0);
					if (rn < pr) {
						n0 = d.at(c0 + rn, col0);
						n1 = d.at(c0 + rn, col1);
					}
#pragma unroll
					for (int k = 0; k < 16; k++) {
						const T v = (r > k) ? P[r * 17 + k] : ((r == k) ? T(1) : T(0));
						a0 = fma(-v, w0[k], a0);
						a1 = fma(-v, w1[k], a1);
					}
					d.at(c0 + r, col0) = a0;
					if (two) d.at(c0 + r, col1) = a1;
					a0 = n0;
					a1 = n1;
					r = rn;
				}
			}
		}
		__syncthreads();
	}
}

}  // namespace

namespace {
template <typename T, int NT, int MINB>
void launch_potrf_smem(int batch, SizeArg sz, int max_m, size_t smem, MatArg<T> C, MatArg<T> D, int *info,
                       cudaStream_t s, int min_n = 0) {
	auto kern = k_potrf_smem<T, NT, MINB>;
	bf::smem_optin(kern, smem);
	kern<<<batch, NT, smem, s>>>(sz, C, D, info, max_m, min_n);
}
}  // namespace

namespace bf {

// variant: -1 auto; 0..3: shared memory with 64/128/256/512 threads for the
// instances that fit (the others in global memory, a second launch);
// 4: everything in global memory (FP64: blocked, FP64 tensor-core updates);
// 5 (FP64, max_m <= 64): one warp per instance on the FP64 tensor cores
// (potrf_dmma.cu).  FP64 auto: 5 for n <= 64, 1 for 64 < n <= 128, the
// blocked global-memory kernel above.
template <typename T>
int potrf_launch(int batch, SizeArg sz, int max_m, MatArg<T> C, MatArg<T> D, int *info, cudaStream_t s, int variant) {
	if (batch <= 0 || max_m <= 0) return BLASFEO_B200_OK;
	if constexpr (sizeof(T) == 8) {
		if (max_m <= 64 && (variant < 0 || variant == 5)) return dpotrf_dmma_launch(batch, sz, max_m, C, D, info, s);
		if (variant < 0 && max_m <= dpotrf_ll_max_n()) {
			// by size (measured fastest per range, uniform batches n = 32..384):
			// n <= 64 one warp on the FP64 tensor cores, larger n blocked from
			// L2 with FP64 tensor-core updates (at n = 128 0.11 ms against
			// 0.15 ms for the shared-memory kernel); one launch per range, each
			// kernel skips the instances of the other range
			int st = dpotrf_dmma_launch(batch, sz, 64, C, D, info, s);
			if (st || max_m <= 64) return st;
			return dpotrf_ll_launch(batch, sz, 64, max_m, C, D, info, s);
		}
	}
	if (variant == 5) variant = -1;
	static int limit_cache[2] = {0, 0};
	int &lim = limit_cache[sizeof(T) == 8];
	if (!lim)
		for (int v = 4; v <= 1024; v += 4)
			if (potrf_smem_plan<T>(v).total <= max_smem_optin()) lim = v;
	const int smax = max_m < lim ? max_m : lim;
	PotrfSmem pl = potrf_smem_plan<T>(smax);
	if (variant < 0) variant = smax <= 64 ? 0 : (smax <= 128 ? 1 : 3);
	switch (variant) {
	case 0: launch_potrf_smem<T, 64, 8>(batch, sz, smax, pl.total, C, D, info, s); break;
	case 1: launch_potrf_smem<T, 128, 4>(batch, sz, smax, pl.total, C, D, info, s); break;
	case 2: launch_potrf_smem<T, 256, 2>(batch, sz, smax, pl.total, C, D, info, s); break;
	case 3: launch_potrf_smem<T, 512, 1>(batch, sz, smax, pl.total, C, D, info, s); break;
	default: break;
	}
	if (variant >= 4 || max_m > smax) {
		const int min_n = variant >= 4 ? 0 : smax;
		if constexpr (sizeof(T) == 8) {
			// FP64 beyond shared memory: blocked, FP64 tensor-core updates
			if (max_m <= dpotrf_ll_max_n()) return dpotrf_ll_launch(batch, sz, min_n, max_m, C, D, info, s);
		}
		k_potrf_global<T><<<batch, 256, 0, s>>>(sz, C, D, info, min_n);
	}
	return check_launch();
}
template int potrf_launch<double>(int, SizeArg, int, MatArg<double>, MatArg<double>, int *, cudaStream_t, int);
template int potrf_launch<float>(int, SizeArg, int, MatArg<float>, MatArg<float>, int *, cudaStream_t, int);

}  // namespace bf

namespace {

template <typename T, typename S>
void potrf_single(int m, S *sC, int ci, int cj, S *sD, int di, int dj) {
	if (m <= 0) return;
	sD->use_dA = (di == 0 && dj == 0) ? m : 0;
	bf::potrf_launch<T>(1, uniform_sizes(m, m, 0), m, single_arg<T>(sC, ci, cj), single_arg<T>(sD, di, dj), nullptr,
	                    bf::cur_stream(), -1);
	bf::finish_single();
}

template <typename T, typename BT>
int potrf_batch(int batch, int m, BT *sC, int ci, int cj, BT *sD, int di, int dj, int *info, void *stream) {
	if (batch < 0 || !sC || !sD) return BLASFEO_B200_EINVAL;
	if (m <= 0 || batch == 0) return BLASFEO_B200_OK;
	sD->use_dA = (di == 0 && dj == 0) ? m : 0;
	return bf::potrf_launch<T>(batch, uniform_sizes(m, m, 0), m, batch_arg<T>(sC, ci, cj), batch_arg<T>(sD, di, dj),
	                           info, (cudaStream_t)stream, -1);
}

template <typename T, typename S>
void syrk_potrf_single(int m, int k, S *sA, int ai, int aj, S *sB, int bi, int bj, S *sC, int ci, int cj, S *sD,
                       int di, int dj) {
	if (m <= 0) return;
	cudaStream_t s = bf::cur_stream();
	MatArg<T> D = single_arg<T>(sD, di, dj);
	bf::gemm_nt_launch<T, true>(1, uniform_sizes(m, m, k), m, m, k, T(1), single_arg<T>(sA, ai, aj),
	                            single_arg<T>(sB, bi, bj), T(1), single_arg<T>(sC, ci, cj), D, s, -1);
	sD->use_dA = (di == 0 && dj == 0) ? m : 0;
	bf::potrf_launch<T>(1, uniform_sizes(m, m, 0), m, D, D, nullptr, s, -1);
	bf::finish_single();
}

template <typename T, typename BT>
int syrk_potrf_batch(int batch, int m, int k, BT *sA, int ai, int aj, BT *sB, int bi, int bj, BT *sC, int ci, int cj,
                     BT *sD, int di, int dj, int *info, void *stream) {
	if (batch < 0 || !sA || !sB || !sC || !sD) return BLASFEO_B200_EINVAL;
	if (m <= 0 || batch == 0) return BLASFEO_B200_OK;
	cudaStream_t s = (cudaStream_t)stream;
	MatArg<T> D = batch_arg<T>(sD, di, dj);
	int st = bf::gemm_nt_launch<T, true>(batch, uniform_sizes(m, m, k), m, m, k, T(1), batch_arg<T>(sA, ai, aj),
	                                     batch_arg<T>(sB, bi, bj), T(1), batch_arg<T>(sC, ci, cj), D, s, -1);
	if (st) return st;
	sD->use_dA = (di == 0 && dj == 0) ? m : 0;
	return bf::potrf_launch<T>(batch, uniform_sizes(m, m, 0), m, D, D, info, s, -1);
}

// variant: -1 auto; 0..2: the blocked global-memory kernels (getrf: 128
// threads with 4 or 2 blocks per SM, 256 threads; geqrf: 256 threads with the
// SIMT trailing update, 256 and 512 threads with the DMMA one); 3..5: the
// instances whose block fits in shared memory there (128/256/512 threads),
// the others in the blocked global-memory kernel (a second launch).
template <typename T, int NT, bool SMEM>
void launch_getrf(int batch, SizeArg sz, int cap, size_t smem, MatArg<T> C, MatArg<T> D, int *ipiv,
                  long long ipiv_stride, int *info, cudaStream_t s, bool piv = true) {
	auto kern = k_getrf<T, NT, SMEM>;
	bf::smem_optin(kern, smem);
	kern<<<batch, NT, smem, s>>>(sz, C, D, ipiv, ipiv_stride, info, cap, piv);
}

// blocked global-memory LU (k_getrf_blk) for the instances that do not fit
// shared memory (cap >= 0) or for all of them (cap < 0)
template <typename T, int NT, int MINB>
void launch_getrf_blk(int batch, SizeArg sz, int cap, int max_m, int max_n, MatArg<T> C, MatArg<T> D, int *ipiv,
                      long long ipiv_stride, int *info, cudaStream_t s, bool piv = true) {
	auto kern = k_getrf_blk<T, NT, MINB>;
	const size_t smem = ((size_t)(max_m + 4) * 17 + (size_t)16 * (max_n + 4)) * sizeof(T) + (size_t)(max_m + 4) * sizeof(int);
	if (smem > bf::max_smem_optin()) {
		// panel and U12 beyond shared memory (blocks of more than ~1,500 rows):
		// the unblocked global-memory kernel
		launch_getrf<T, 512, false>(batch, sz, cap, 0, C, D, ipiv, ipiv_stride, info, s, piv);
		return;
	}
	bf::smem_optin(kern, smem);
	kern<<<batch, NT, smem, s>>>(sz, C, D, ipiv, ipiv_stride, info, cap, max_m, piv);
}
template <typename T, int NT, bool SMEM>
void launch_geqrf(int batch, SizeArg sz, int cap, size_t smem, MatArg<T> C, MatArg<T> D, cudaStream_t s) {
	auto kern = k_geqrf<T, NT, SMEM>;
	bf::smem_optin(kern, smem);
	kern<<<batch, NT, smem, s>>>(sz, C, D, cap);
}

// blocked global-memory QR (k_geqrf_blk) for the instances that do not fit
// shared memory (cap >= 0) or for all of them (cap < 0)
template <typename T, int NT, bool DMMA>
void launch_geqrf_blk(int batch, SizeArg sz, int cap, int max_m, int max_n, MatArg<T> C, MatArg<T> D,
                      cudaStream_t s) {
	auto kern = k_geqrf_blk<T, NT, DMMA>;
	const size_t smem = qr_panel_bytes(max_m, sizeof(T)) +
	                    (sizeof(T) == 8 && DMMA ? (size_t)qr_w_slots(NT, max_n) * sizeof(double) : 0);
	if (smem > bf::max_smem_optin()) {
		// a panel beyond shared memory (more than ~1,500 rows): the unblocked kernel
		launch_geqrf<T, 512, false>(batch, sz, cap, 0, C, D, s);
		return;
	}
	bf::smem_optin(kern, smem);
	kern<<<batch, NT, smem, s>>>(sz, C, D, cap, max_m, max_n);
}

inline size_t lu_smem_bytes(int max_m, int max_n, size_t esz) {
	return (size_t)((max_m + 3) / 4 * 4) * ((max_n + 3) / 4 * 4) * esz;
}

// built-in rule for getrf (qr = false) and geqrf (qr = true), from uniform
// batches timed on the B200 at n = 32..384: the shared-memory kernel with 128
// threads for small blocks, the blocked global-memory kernels above (getrf:
// 128 threads with 4 blocks per SM up to n = 96, with 3 up to 288, then 256
// threads; geqrf: shared memory up to 64 rows, then the DMMA update with
// 256 threads at 2 CTAs per SM)
inline int pick_lu_variant(int variant, int max_m, int max_n, bool qr = false) {
	if (variant < 0) {
		const int mx = max_m > max_n ? max_m : max_n;
		if (mx <= 48)
			variant = 3;
		else if (!qr)
			variant = mx <= 96 ? 0 : (mx <= 288 ? 1 : 2);
		else
			variant = mx <= 64 ? 3 : 1;
	}
	return variant;
}

template <typename T>
int getrf_launch(int batch, SizeArg sz, MatArg<T> C, MatArg<T> D, int *ipiv, long long ipiv_stride, int *info,
                 cudaStream_t s, int max_m, int max_n, int variant = -1, bool piv = true) {
	const size_t cap_full = bf::max_smem_optin() - 1024;
	const size_t need = lu_smem_bytes(max_m, max_n, sizeof(T));
	const size_t smem = need < cap_full ? need : cap_full;
	const int cap = (int)smem;
	variant = pick_lu_variant(variant, max_m, max_n);
	switch (variant) {
	// blocked: 128 threads with 4 or 3 blocks per SM (register cap; FP64 variant 1
	// spills a little at 3, faster than 2: n = 224 2.25 -> 2.65 TF/s), 256 threads
	case 0: launch_getrf_blk<T, 128, 4>(batch, sz, -1, max_m, max_n, C, D, ipiv, ipiv_stride, info, s, piv); break;
	case 1:
		// FP64: 3 CTAs per SM up to n = 288 (the size rule's range), 2 above:
		// batches that mix sizes up to 384 ran faster with 2 (mixed-op stream,
		// LU share 348 -> 329 ms)
		if (sizeof(T) == 8 && (max_m > 288 || max_n > 288))
			launch_getrf_blk<T, 128, 2>(batch, sz, -1, max_m, max_n, C, D, ipiv, ipiv_stride, info, s, piv);
		else
			launch_getrf_blk<T, 128, sizeof(T) == 8 ? 3 : 2>(batch, sz, -1, max_m, max_n, C, D, ipiv, ipiv_stride,
			                                                   info, s, piv);
		break;
	case 2: launch_getrf_blk<T, 256, 1>(batch, sz, -1, max_m, max_n, C, D, ipiv, ipiv_stride, info, s, piv); break;
	case 3: launch_getrf<T, 128, true>(batch, sz, cap, smem, C, D, ipiv, ipiv_stride, info, s, piv); break;
	case 4: launch_getrf<T, 256, true>(batch, sz, cap, smem, C, D, ipiv, ipiv_stride, info, s, piv); break;
	default: launch_getrf<T, 512, true>(batch, sz, cap, smem, C, D, ipiv, ipiv_stride, info, s, piv); break;
	}
	if (variant >= 3 && need > smem)
		launch_getrf_blk<T, 256, 1>(batch, sz, cap, max_m, max_n, C, D, ipiv, ipiv_stride, info, s, piv);
	return bf::check_launch();
}

template <typename T>
int geqrf_launch(int batch, SizeArg sz, MatArg<T> C, MatArg<T> D, cudaStream_t s, int max_m, int max_n,
                 int variant = -1) {
	const size_t cap_full = bf::max_smem_optin() - 1024;
	const size_t need = lu_smem_bytes(max_m, max_n, sizeof(T));
	const size_t smem = need < cap_full ? need : cap_full;
	const int cap = (int)smem;
	variant = pick_lu_variant(variant, max_m, max_n, true);
	switch (variant) {
	// blocked: 256 threads with the SIMT update, 256 or 512 threads with the DMMA update
	case 0: launch_geqrf_blk<T, 256, false>(batch, sz, -1, max_m, max_n, C, D, s); break;
	case 1: launch_geqrf_blk<T, 256, true>(batch, sz, -1, max_m, max_n, C, D, s); break;
	case 2: launch_geqrf_blk<T, 512, true>(batch, sz, -1, max_m, max_n, C, D, s); break;
	case 3: launch_geqrf<T, 128, true>(batch, sz, cap, smem, C, D, s); break;
	case 4: launch_geqrf<T, 256, true>(batch, sz, cap, smem, C, D, s); break;
	default: launch_geqrf<T, 512, true>(batch, sz, cap, smem, C, D, s); break;
	}
	if (variant >= 3 && need > smem) launch_geqrf_blk<T, 512, true>(batch, sz, cap, max_m, max_n, C, D, s);
	return bf::check_launch();
}

template <typename T, typename S>
void getrf_single(int m, int n, S *sC, int ci, int cj, S *sD, int di, int dj, int *ipiv) {
	if (m <= 0 || n <= 0) return;
	if (!ipiv) {
		bf::set_error(BLASFEO_B200_EINVAL);
		return;
	}
	sD->use_dA = (di == 0 && dj == 0) ? 1 : 0;
	cudaStream_t s = bf::cur_stream();
	int mn = m < n ? m : n;
	int *dpiv = (int *)bf::workspace(mn * sizeof(int), s);
	if (!dpiv) {
		bf::set_error(BLASFEO_B200_ENOMEM);
		return;
	}
	getrf_launch<T>(1, uniform_sizes(m, n, 0), single_arg<T>(sC, ci, cj), single_arg<T>(sD, di, dj), dpiv, 0, nullptr, s,
	                m, n);
	if (bf::check_launch() != BLASFEO_B200_OK) return;
	// the pivot vector is a host array in the reference API: always complete the copy
	if (cudaMemcpyAsync(ipiv, dpiv, mn * sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
	    cudaStreamSynchronize(s) != cudaSuccess)
		bf::set_error(BLASFEO_B200_ECUDA);
}

template <typename T, typename BT>
int getrf_batch(int batch, int m, int n, BT *sC, int ci, int cj, BT *sD, int di, int dj, int *ipiv, int *info,
                void *stream) {
	if (batch < 0 || !sC || !sD || !ipiv) return BLASFEO_B200_EINVAL;
	if (m <= 0 || n <= 0 || batch == 0) return BLASFEO_B200_OK;
	sD->use_dA = (di == 0 && dj == 0) ? 1 : 0;
	int mn = m < n ? m : n;
	return getrf_launch<T>(batch, uniform_sizes(m, n, 0), batch_arg<T>(sC, ci, cj), batch_arg<T>(sD, di, dj), ipiv, mn,
	                       info, (cudaStream_t)stream, m, n);
}

// LU without pivoting (getrf_np, blasfeo_hp_pm/d_lapack_lib4.c:2078)
template <typename T, typename S>
void getrf_np_single(int m, int n, S *sC, int ci, int cj, S *sD, int di, int dj) {
	if (m <= 0 || n <= 0) return;
	sD->use_dA = (di == 0 && dj == 0) ? 1 : 0;
	getrf_launch<T>(1, uniform_sizes(m, n, 0), single_arg<T>(sC, ci, cj), single_arg<T>(sD, di, dj), nullptr, 0, nullptr,
	                bf::cur_stream(), m, n, -1, false);
	bf::finish_single();
}

template <typename T, typename BT>
int getrf_np_batch(int batch, int m, int n, BT *sC, int ci, int cj, BT *sD, int di, int dj, int *info, void *stream) {
	if (batch < 0 || !sC || !sD) return BLASFEO_B200_EINVAL;
	if (m <= 0 || n <= 0 || batch == 0) return BLASFEO_B200_OK;
	sD->use_dA = (di == 0 && dj == 0) ? 1 : 0;
	return getrf_launch<T>(batch, uniform_sizes(m, n, 0), batch_arg<T>(sC, ci, cj), batch_arg<T>(sD, di, dj), nullptr, 0,
	                       info, (cudaStream_t)stream, m, n, -1, false);
}

// potrf_l_mn: use_dA = 1 with zero offsets, as blasfeo_hp_dpotrf_l_mn sets it
// (blasfeo_hp_pm/d_lapack_lib4.c:1184-1187)
template <typename T, typename S>
void potrf_mn_single(int m, int n, S *sC, int ci, int cj, S *sD, int di, int dj) {
	if (m <= 0 || n <= 0) return;
	sD->use_dA = (di == 0 && dj == 0) ? 1 : 0;
	k_potrf_mn<T><<<1, 256, 0, bf::cur_stream()>>>(uniform_sizes(m, n, 0), single_arg<T>(sC, ci, cj),
	                                                single_arg<T>(sD, di, dj), nullptr);
	bf::finish_single();
}

template <typename T, typename BT>
int potrf_mn_batch(int batch, int m, int n, BT *sC, int ci, int cj, BT *sD, int di, int dj, int *info, void *stream) {
	if (batch < 0 || !sC || !sD) return BLASFEO_B200_EINVAL;
	if (m <= 0 || n <= 0 || batch == 0) return BLASFEO_B200_OK;
	sD->use_dA = (di == 0 && dj == 0) ? 1 : 0;
	k_potrf_mn<T><<<batch, 256, 0, (cudaStream_t)stream>>>(uniform_sizes(m, n, 0), batch_arg<T>(sC, ci, cj),
	                                                         batch_arg<T>(sD, di, dj), info);
	return bf::check_launch();
}

template <typename T, typename S>
void geqrf_single(int m, int n, S *sC, int ci, int cj, S *sD, int di, int dj) {
	if (m <= 0 || n <= 0) return;
	sD->use_dA = 0;
	geqrf_launch<T>(1, uniform_sizes(m, n, 0), single_arg<T>(sC, ci, cj), single_arg<T>(sD, di, dj), bf::cur_stream(), m,
	                n);
	bf::finish_single();
}

template <typename T, typename BT>
int geqrf_batch(int batch, int m, int n, BT *sC, int ci, int cj, BT *sD, int di, int dj, void *stream) {
	if (batch < 0 || !sC || !sD) return BLASFEO_B200_EINVAL;
	if (m <= 0 || n <= 0 || batch == 0) return BLASFEO_B200_OK;
	sD->use_dA = 0;
	return geqrf_launch<T>(batch, uniform_sizes(m, n, 0), batch_arg<T>(sC, ci, cj), batch_arg<T>(sD, di, dj),
	                       (cudaStream_t)stream, m, n);
}

// geqrf work size of the HP reference (blasfeo_hp_pm/d_lapack_lib4.c:3433-3440)
template <typename T>
int geqrf_ws(int m, int n) {
	int cm = (m + 3) / 4 * 4;
	int cn = (n + 3) / 4 * 4;
	return 4 * (cm + cn) * (int)sizeof(T);
}

}  // namespace

extern "C" {

void blasfeo_dpotrf_l(int m, struct blasfeo_dmat *sC, int ci, int cj, struct blasfeo_dmat *sD, int di, int dj) {
	potrf_single<double>(m, sC, ci, cj, sD, di, dj);
}
void blasfeo_spotrf_l(int m, struct blasfeo_smat *sC, int ci, int cj, struct blasfeo_smat *sD, int di, int dj) {
	potrf_single<float>(m, sC, ci, cj, sD, di, dj);
}
void blasfeo_dsyrk_dpotrf_ln(int m, int k, struct blasfeo_dmat *sA, int ai, int aj, struct blasfeo_dmat *sB, int bi,
                             int bj, struct blasfeo_dmat *sC, int ci, int cj, struct blasfeo_dmat *sD, int di, int dj) {
	syrk_potrf_single<double>(m, k, sA, ai, aj, sB, bi, bj, sC, ci, cj, sD, di, dj);
}
void blasfeo_ssyrk_spotrf_ln(int m, int k, struct blasfeo_smat *sA, int ai, int aj, struct blasfeo_smat *sB, int bi,
                             int bj, struct blasfeo_smat *sC, int ci, int cj, struct blasfeo_smat *sD, int di, int dj) {
	syrk_potrf_single<float>(m, k, sA, ai, aj, sB, bi, bj, sC, ci, cj, sD, di, dj);
}
void blasfeo_dgetrf_rp(int m, int n, struct blasfeo_dmat *sC, int ci, int cj, struct blasfeo_dmat *sD, int di, int dj,
                       int *ipiv) {
	getrf_single<double>(m, n, sC, ci, cj, sD, di, dj, ipiv);
}
void blasfeo_sgetrf_rp(int m, int n, struct blasfeo_smat *sC, int ci, int cj, struct blasfeo_smat *sD, int di, int dj,
                       int *ipiv) {
	getrf_single<float>(m, n, sC, ci, cj, sD, di, dj, ipiv);
}
int blasfeo_dgeqrf_worksize(int m, int n) { return geqrf_ws<double>(m, n); }
int blasfeo_sgeqrf_worksize(int m, int n) { return geqrf_ws<float>(m, n); }
void blasfeo_dgeqrf(int m, int n, struct blasfeo_dmat *sC, int ci, int cj, struct blasfeo_dmat *sD, int di, int dj,
                    void *work) {
	(void)work;
	geqrf_single<double>(m, n, sC, ci, cj, sD, di, dj);
}
void blasfeo_sgeqrf(int m, int n, struct blasfeo_smat *sC, int ci, int cj, struct blasfeo_smat *sD, int di, int dj,
                    void *work) {
	(void)work;
	geqrf_single<float>(m, n, sC, ci, cj, sD, di, dj);
}

void blasfeo_dpotrf_l_mn(int m, int n, struct blasfeo_dmat *sC, int ci, int cj, struct blasfeo_dmat *sD, int di, int dj) {
	potrf_mn_single<double>(m, n, sC, ci, cj, sD, di, dj);
}
void blasfeo_spotrf_l_mn(int m, int n, struct blasfeo_smat *sC, int ci, int cj, struct blasfeo_smat *sD, int di, int dj) {
	potrf_mn_single<float>(m, n, sC, ci, cj, sD, di, dj);
}
void blasfeo_dgetrf_np(int m, int n, struct blasfeo_dmat *sC, int ci, int cj, struct blasfeo_dmat *sD, int di, int dj) {
	getrf_np_single<double>(m, n, sC, ci, cj, sD, di, dj);
}
void blasfeo_sgetrf_np(int m, int n, struct blasfeo_smat *sC, int ci, int cj, struct blasfeo_smat *sD, int di, int dj) {
	getrf_np_single<float>(m, n, sC, ci, cj, sD, di, dj);
}
int blasfeo_dpotrf_l_mn_batch(int batch, int m, int n, struct blasfeo_dmat_batch *sC, int ci, int cj,
                              struct blasfeo_dmat_batch *sD, int di, int dj, int *info, void *stream) {
	return potrf_mn_batch<double>(batch, m, n, sC, ci, cj, sD, di, dj, info, stream);
}
int blasfeo_spotrf_l_mn_batch(int batch, int m, int n, struct blasfeo_smat_batch *sC, int ci, int cj,
                              struct blasfeo_smat_batch *sD, int di, int dj, int *info, void *stream) {
	return potrf_mn_batch<float>(batch, m, n, sC, ci, cj, sD, di, dj, info, stream);
}
int blasfeo_dgetrf_np_batch(int batch, int m, int n, struct blasfeo_dmat_batch *sC, int ci, int cj,
                            struct blasfeo_dmat_batch *sD, int di, int dj, int *info, void *stream) {
	return getrf_np_batch<double>(batch, m, n, sC, ci, cj, sD, di, dj, info, stream);
}
int blasfeo_sgetrf_np_batch(int batch, int m, int n, struct blasfeo_smat_batch *sC, int ci, int cj,
                            struct blasfeo_smat_batch *sD, int di, int dj, int *info, void *stream) {
	return getrf_np_batch<float>(batch, m, n, sC, ci, cj, sD, di, dj, info, stream);
}

int blasfeo_dpotrf_l_batch(int batch, int m, struct blasfeo_dmat_batch *sC, int ci, int cj,
                           struct blasfeo_dmat_batch *sD, int di, int dj, int *info, void *stream) {
	return potrf_batch<double>(batch, m, sC, ci, cj, sD, di, dj, info, stream);
}
int blasfeo_spotrf_l_batch(int batch, int m, struct blasfeo_smat_batch *sC, int ci, int cj,
                           struct blasfeo_smat_batch *sD, int di, int dj, int *info, void *stream) {
	return potrf_batch<float>(batch, m, sC, ci, cj, sD, di, dj, info, stream);
}
int blasfeo_dsyrk_dpotrf_ln_batch(int batch, int m, int k, struct blasfeo_dmat_batch *sA, int ai, int aj,
                                  struct blasfeo_dmat_batch *sB, int bi, int bj, struct blasfeo_dmat_batch *sC, int ci,
                                  int cj, struct blasfeo_dmat_batch *sD, int di, int dj, int *info, void *stream) {
	return syrk_potrf_batch<double>(batch, m, k, sA, ai, aj, sB, bi, bj, sC, ci, cj, sD, di, dj, info, stream);
}
int blasfeo_ssyrk_spotrf_ln_batch(int batch, int m, int k, struct blasfeo_smat_batch *sA, int ai, int aj,
                                  struct blasfeo_smat_batch *sB, int bi, int bj, struct blasfeo_smat_batch *sC, int ci,
                                  int cj, struct blasfeo_smat_batch *sD, int di, int dj, int *info, void *stream) {
	return syrk_potrf_batch<float>(batch, m, k, sA, ai, aj, sB, bi, bj, sC, ci, cj, sD, di, dj, info, stream);
}
int blasfeo_dgetrf_rp_batch(int batch, int m, int n, struct blasfeo_dmat_batch *sC, int ci, int cj,
                            struct blasfeo_dmat_batch *sD, int di, int dj, int *ipiv, int *info, void *stream) {
	return getrf_batch<double>(batch, m, n, sC, ci, cj, sD, di, dj, ipiv, info, stream);
}
int blasfeo_sgetrf_rp_batch(int batch, int m, int n, struct blasfeo_smat_batch *sC, int ci, int cj,
                            struct blasfeo_smat_batch *sD, int di, int dj, int *ipiv, int *info, void *stream) {
	return getrf_batch<float>(batch, m, n, sC, ci, cj, sD, di, dj, ipiv, info, stream);
}
int blasfeo_dgeqrf_batch(int batch, int m, int n, struct blasfeo_dmat_batch *sC, int ci, int cj,
                         struct blasfeo_dmat_batch *sD, int di, int dj, void *stream) {
	return geqrf_batch<double>(batch, m, n, sC, ci, cj, sD, di, dj, stream);
}
int blasfeo_sgeqrf_batch(int batch, int m, int n, struct blasfeo_smat_batch *sC, int ci, int cj,
                         struct blasfeo_smat_batch *sD, int di, int dj, void *stream) {
	return geqrf_batch<float>(batch, m, n, sC, ci, cj, sD, di, dj, stream);
}

int blasfeo_dpotrf_l_vbatch_variant(int batch, const int *m, int max_m, const struct blasfeo_dmat *sC,
                                    const struct blasfeo_dmat *sD, int *info, int variant, void *stream) {
	if (batch < 0 || !m || !sC || !sD || max_m < 0 || variant > 5) return BLASFEO_B200_EINVAL;
	if (batch == 0 || max_m == 0) return BLASFEO_B200_OK;
	if (variant < 0) variant = bf::dispatch_pick(1, batch, m, m, m, max_m, max_m, max_m, (cudaStream_t)stream);
	return bf::potrf_launch<double>(batch, var_sizes(m, m, nullptr), max_m, vbatch_arg<double>(sC),
	                                vbatch_arg<double>(sD), info, (cudaStream_t)stream, variant);
}
int blasfeo_dpotrf_l_vbatch(int batch, const int *m, int max_m, const struct blasfeo_dmat *sC,
                            const struct blasfeo_dmat *sD, int *info, void *stream) {
	return blasfeo_dpotrf_l_vbatch_variant(batch, m, max_m, sC, sD, info, -1, stream);
}
int blasfeo_dgetrf_rp_vbatch_variant(int batch, const int *m, const int *n, int max_m, int max_n,
                                     const struct blasfeo_dmat *sC, const struct blasfeo_dmat *sD, int *ipiv,
                                     int ipiv_stride, int *info, int variant, void *stream) {
	if (batch < 0 || !m || !n || !sC || !sD || !ipiv || max_m < 0 || max_n < 0 || variant > 5) return BLASFEO_B200_EINVAL;
	if (batch == 0 || max_m == 0 || max_n == 0) return BLASFEO_B200_OK;
	if (variant < 0) variant = bf::dispatch_pick(2, batch, m, n, n, max_m, max_n, max_n, (cudaStream_t)stream);
	return getrf_launch<double>(batch, var_sizes(m, n, nullptr), vbatch_arg<double>(sC), vbatch_arg<double>(sD), ipiv,
	                            ipiv_stride, info, (cudaStream_t)stream, max_m, max_n, variant);
}
int blasfeo_dgetrf_rp_vbatch(int batch, const int *m, const int *n, int max_m, int max_n,
                             const struct blasfeo_dmat *sC, const struct blasfeo_dmat *sD, int *ipiv, int ipiv_stride,
                             int *info, void *stream) {
	return blasfeo_dgetrf_rp_vbatch_variant(batch, m, n, max_m, max_n, sC, sD, ipiv, ipiv_stride, info, -1, stream);
}
int blasfeo_dgeqrf_vbatch_variant(int batch, const int *m, const int *n, int max_m, int max_n,
                                  const struct blasfeo_dmat *sC, const struct blasfeo_dmat *sD, int variant,
                                  void *stream) {
	if (batch < 0 || !m || !n || !sC || !sD || max_m < 0 || max_n < 0 || variant > 5) return BLASFEO_B200_EINVAL;
	if (batch == 0 || max_m == 0 || max_n == 0) return BLASFEO_B200_OK;
	if (variant < 0) variant = bf::dispatch_pick(3, batch, m, n, n, max_m, max_n, max_n, (cudaStream_t)stream);
	return geqrf_launch<double>(batch, var_sizes(m, n, nullptr), vbatch_arg<double>(sC), vbatch_arg<double>(sD),
	                            (cudaStream_t)stream, max_m, max_n, variant);
}
int blasfeo_dgeqrf_vbatch(int batch, const int *m, const int *n, int max_m, int max_n, const struct blasfeo_dmat *sC,
                          const struct blasfeo_dmat *sD, void *stream) {
	return blasfeo_dgeqrf_vbatch_variant(batch, m, n, max_m, max_n, sC, sD, -1, stream);
}

}  // extern "C"
