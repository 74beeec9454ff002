// Column-major drop-in: the blasfeo_cm_* routines of the reference on the
// hot path (include/blasfeo_d_blasfeo_api.h:321,324,342,389,391 and
// include/blasfeo_s_blasfeo_api.h:282,295,305; implementation
// blasfeo_hp_cm/dgemm.c:3821, dsyrk.c:3022, dtrsm.c:5245, dpotrf.c:564,
// dgetrf.c:85) for device-resident column-major matrices.
//
// struct blasfeo_cm_dmat has the reference layout (include/blasfeo_common.h:
// 220-229): pA is a column-major array whose leading dimension is the
// descriptor's m, element (i,j) at pA[i + j*m] (the BLAS API wrappers set m to
// lda, blas_api/xpotrf_ref.c).  Like the reference's column-major routines,
// these neither read nor write dA / use_dA.
//
// Each call stages the sub-blocks it reads into panel-major scratch (one
// gather kernel per operand, coalesced column reads), runs this library's
// panel-major routine on them (the same kernels, hence the same arithmetic
// as the panel-major drop-ins), and scatters the result block back: the
// whole block for gemm / trsm / getrf, the lower triangle (diagonal included)
// for syrk_ln / potrf_l, the part the reference writes.  The scratch is a
// library-owned device buffer of its own (the panel-major routines use the
// other one for their pivots).
#include "common.cuh"

namespace {

// column-major block (m x n at A, leading dimension lda) -> panel-major
// scratch with panel stride cn; padding rows/columns (up to 4-row panels and
// cn columns) zeroed
template <typename T>
__global__ void k_cm_gather(int m, int n, int pm, int cn, const T *__restrict__ A, int lda, T *__restrict__ P) {
	const size_t total = (size_t)pm * cn;
	for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
		const int i = (int)(e % pm), j = (int)(e / pm);  // consecutive threads: consecutive rows of a column
		const T v = (i < m && j < n) ? A[(size_t)i + (size_t)j * lda] : T(0);
		P[(size_t)(i & ~3) * cn + 4 * j + (i & 3)] = v;
	}
}

// panel-major scratch (m x n, panel stride cn) -> column-major block at D
// (leading dimension ldd); lower: only i >= j
template <typename T>
__global__ void k_cm_scatter(int m, int n, int cn, const T *__restrict__ P, T *__restrict__ D, int ldd, int lower) {
	const size_t total = (size_t)m * n;
	for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
		const int i = (int)(e % m), j = (int)(e / m);
		if (lower && i < j) continue;
		D[(size_t)i + (size_t)j * ldd] = P[(size_t)(i & ~3) * cn + 4 * j + (i & 3)];
	}
}

inline int grid_for(size_t total) {
	size_t g = (total + 255) / 256;
	const size_t cap = (size_t)bf::num_sms() * 8;
	return (int)(g < 1 ? 1 : (g > cap ? cap : g));
}

template <typename T>
struct CmT;
template <>
struct CmT<double> {
	typedef struct blasfeo_cm_dmat cm;
	typedef struct blasfeo_dmat pm;
};
template <>
struct CmT<float> {
	typedef struct blasfeo_cm_smat cm;
	typedef struct blasfeo_smat pm;
};

// panel-major staging matrices of one call, carved from the column-major
// scratch buffer: pA (pm x cn) then dA (min(m,n) rounded up to 16)
template <typename T>
struct Stage {
	typedef typename CmT<T>::pm PM;
	PM mat[4];
	int count = 0;
	size_t bytes = 0;
	static size_t need(int m, int n) {
		const size_t pm = (size_t)(m + 3) / 4 * 4, cn = (size_t)(n + 3) / 4 * 4;
		const size_t mn = (size_t)(m < n ? m : n);
		return ((pm * cn + (mn + 15) / 16 * 16) * sizeof(T) + 255) / 256 * 256;
	}
	void add(int m, int n) {
		PM &d = mat[count++];
		d.m = m;
		d.n = n;
		d.pm = (m + 3) / 4 * 4;
		d.cn = (n + 3) / 4 * 4;
		d.use_dA = 0;
		d.memsize = (int)need(m, n);
		d.mem = (T *)(uintptr_t)bytes;  // offset until bind()
		bytes += need(m, n);
	}
	bool bind(cudaStream_t s) {
		char *base = (char *)bf::workspace_cm(bytes, s);
		if (!base) return false;
		for (int i = 0; i < count; i++) {
			PM &d = mat[i];
			T *p = (T *)(base + (uintptr_t)d.mem);
			d.mem = p;
			d.pA = p;
			d.dA = p + (size_t)d.pm * d.cn;
		}
		return true;
	}
};

template <typename T>
void gather(const typename CmT<T>::cm *A, int ai, int aj, const typename CmT<T>::pm &P, cudaStream_t s) {
	const size_t total = (size_t)P.pm * P.cn;
	k_cm_gather<T><<<grid_for(total), 256, 0, s>>>(P.m, P.n, P.pm, P.cn,
	                                              A->pA + (size_t)ai + (size_t)aj * A->m, A->m, P.pA);
}

template <typename T>
void scatter(const typename CmT<T>::pm &P, typename CmT<T>::cm *D, int di, int dj, bool lower, cudaStream_t s) {
	const size_t total = (size_t)P.m * P.n;
	k_cm_scatter<T><<<grid_for(total), 256, 0, s>>>(P.m, P.n, P.cn, P.pA, D->pA + (size_t)di + (size_t)dj * D->m,
	                                               D->m, lower ? 1 : 0);
}

template <typename M>
bool bad(const M *a) {
	return !a || !a->pA || a->m < 0;
}

// the r x c block at (i, j) lies inside the descriptor's m x n matrix (m is
// the leading dimension, so this also keeps every column inside its stride):
// an out-of-range block would make the gather read, and the scatter write,
// outside the caller's buffer
template <typename M>
bool bad_block(const M *a, int i, int j, int r, int c) {
	return bad(a) || a->n < 0 || i < 0 || j < 0 || r < 0 || c < 0 || (long long)i + r > a->m ||
	       (long long)j + c > a->n;
}

// the panel-major drop-ins, by precision
inline void pm_gemm_nt(int m, int n, int k, double al, blasfeo_dmat *A, blasfeo_dmat *B, double be, blasfeo_dmat *C) {
	blasfeo_dgemm_nt(m, n, k, al, A, 0, 0, B, 0, 0, be, C, 0, 0, C, 0, 0);
}
inline void pm_gemm_nt(int m, int n, int k, float al, blasfeo_smat *A, blasfeo_smat *B, float be, blasfeo_smat *C) {
	blasfeo_sgemm_nt(m, n, k, al, A, 0, 0, B, 0, 0, be, C, 0, 0, C, 0, 0);
}
inline void pm_syrk_ln(int m, int k, double al, blasfeo_dmat *A, blasfeo_dmat *B, double be, blasfeo_dmat *C) {
	blasfeo_dsyrk_ln(m, k, al, A, 0, 0, B, 0, 0, be, C, 0, 0, C, 0, 0);
}
inline void pm_syrk_ln(int m, int k, float al, blasfeo_smat *A, blasfeo_smat *B, float be, blasfeo_smat *C) {
	blasfeo_ssyrk_ln(m, k, al, A, 0, 0, B, 0, 0, be, C, 0, 0, C, 0, 0);
}
inline void pm_trsm_rltn(int m, int n, double al, blasfeo_dmat *A, blasfeo_dmat *B) {
	blasfeo_dtrsm_rltn(m, n, al, A, 0, 0, B, 0, 0, B, 0, 0);
}
inline void pm_trsm_rltn(int m, int n, float al, blasfeo_smat *A, blasfeo_smat *B) {
	blasfeo_strsm_rltn(m, n, al, A, 0, 0, B, 0, 0, B, 0, 0);
}
inline void pm_potrf_l(int m, blasfeo_dmat *C) { blasfeo_dpotrf_l(m, C, 0, 0, C, 0, 0); }
inline void pm_potrf_l(int m, blasfeo_smat *C) { blasfeo_spotrf_l(m, C, 0, 0, C, 0, 0); }
inline void pm_getrf_rp(int m, int n, blasfeo_dmat *C, int *ipiv) { blasfeo_dgetrf_rp(m, n, C, 0, 0, C, 0, 0, ipiv); }

// D = beta C + alpha A B^T; syrk: the lower triangle of the m x m result
template <typename T>
void cm_gemm(int m, int n, int k, T alpha, typename CmT<T>::cm *sA, int ai, int aj, typename CmT<T>::cm *sB, int bi,
             int bj, T beta, typename CmT<T>::cm *sC, int ci, int cj, typename CmT<T>::cm *sD, int di, int dj,
             bool syrk) {
	if (m <= 0 || n <= 0) return;
	if (k < 0 || bad_block(sA, ai, aj, m, k) || bad_block(sB, bi, bj, n, k) ||
	    (beta != T(0) && bad_block(sC, ci, cj, m, n)) || (beta == T(0) && bad(sC)) || bad_block(sD, di, dj, m, n)) {
		bf::set_error(BLASFEO_B200_EINVAL);
		return;
	}
	cudaStream_t s = bf::cur_stream();
	const int kk = k > 0 ? k : 1;
	Stage<T> st;
	st.add(m, kk);  // A
	st.add(n, kk);  // B
	st.add(m, n);   // C, overwritten by the result
	if (!st.bind(s)) {
		bf::set_error(BLASFEO_B200_ENOMEM);
		return;
	}
	if (k > 0) {
		gather<T>(sA, ai, aj, st.mat[0], s);
		gather<T>(sB, bi, bj, st.mat[1], s);
	}
	// C is read only when beta != 0, as in the panel-major routine
	if (beta != T(0)) gather<T>(sC, ci, cj, st.mat[2], s);
	if (bf::check_launch() != BLASFEO_B200_OK) return;
	if (syrk)
		pm_syrk_ln(m, k, alpha, &st.mat[0], &st.mat[1], beta, &st.mat[2]);
	else
		pm_gemm_nt(m, n, k, alpha, &st.mat[0], &st.mat[1], beta, &st.mat[2]);
	scatter<T>(st.mat[2], sD, di, dj, syrk, s);
	bf::finish_single();
}

// D = alpha B A^{-T}, A n x n lower, non-unit
template <typename T>
void cm_trsm_rltn(int m, int n, T alpha, typename CmT<T>::cm *sA, int ai, int aj, typename CmT<T>::cm *sB, int bi,
                  int bj, typename CmT<T>::cm *sD, int di, int dj) {
	if (m <= 0 || n <= 0) return;
	if (bad_block(sA, ai, aj, n, n) || bad_block(sB, bi, bj, m, n) || bad_block(sD, di, dj, m, n)) {
		bf::set_error(BLASFEO_B200_EINVAL);
		return;
	}
	cudaStream_t s = bf::cur_stream();
	Stage<T> st;
	st.add(n, n);  // A
	st.add(m, n);  // B, overwritten by the result
	if (!st.bind(s)) {
		bf::set_error(BLASFEO_B200_ENOMEM);
		return;
	}
	gather<T>(sA, ai, aj, st.mat[0], s);
	gather<T>(sB, bi, bj, st.mat[1], s);
	if (bf::check_launch() != BLASFEO_B200_OK) return;
	pm_trsm_rltn(m, n, alpha, &st.mat[0], &st.mat[1]);
	scatter<T>(st.mat[1], sD, di, dj, false, s);
	bf::finish_single();
}

// lower Cholesky factor of the m x m block of C into the lower triangle of D
template <typename T>
void cm_potrf_l(int m, typename CmT<T>::cm *sC, int ci, int cj, typename CmT<T>::cm *sD, int di, int dj) {
	if (m <= 0) return;
	if (bad_block(sC, ci, cj, m, m) || bad_block(sD, di, dj, m, m)) {
		bf::set_error(BLASFEO_B200_EINVAL);
		return;
	}
	cudaStream_t s = bf::cur_stream();
	Stage<T> st;
	st.add(m, m);
	if (!st.bind(s)) {
		bf::set_error(BLASFEO_B200_ENOMEM);
		return;
	}
	gather<T>(sC, ci, cj, st.mat[0], s);
	if (bf::check_launch() != BLASFEO_B200_OK) return;
	pm_potrf_l(m, &st.mat[0]);
	scatter<T>(st.mat[0], sD, di, dj, true, s);
	bf::finish_single();
}

// P C = L U of the m x n block of C into D; ipiv: host array of min(m,n)
// 0-based absolute row indices (blasfeo_hp_cm/dgetrf.c:263)
void cm_dgetrf_rp(int m, int n, blasfeo_cm_dmat *sC, int ci, int cj, blasfeo_cm_dmat *sD, int di, int dj, int *ipiv) {
	if (m <= 0 || n <= 0) return;
	if (bad_block(sC, ci, cj, m, n) || bad_block(sD, di, dj, m, n) || !ipiv) {
		bf::set_error(BLASFEO_B200_EINVAL);
		return;
	}
	cudaStream_t s = bf::cur_stream();
	Stage<double> st;
	st.add(m, n);
	if (!st.bind(s)) {
		bf::set_error(BLASFEO_B200_ENOMEM);
		return;
	}
	gather<double>(sC, ci, cj, st.mat[0], s);
	if (bf::check_launch() != BLASFEO_B200_OK) return;
	pm_getrf_rp(m, n, &st.mat[0], ipiv);
	scatter<double>(st.mat[0], sD, di, dj, false, s);
	bf::finish_single();
}

template <typename T, typename M>
size_t cm_memsize(int m, int n) {
	if (m < 0 || n < 0) return 0;
	const int mn = m < n ? m : n;
	return ((size_t)m * n + mn) * sizeof(T);
}

template <typename T, typename M>
void cm_create(int m, int n, M *sA, void *memory) {
	T *p = (T *)memory;
	const int mn = m < n ? m : n;
	sA->mem = p;
	sA->pA = p;
	sA->dA = p + (size_t)m * n;
	sA->m = m;
	sA->n = n;
	sA->use_dA = 0;
	sA->memsize = (int)(((size_t)m * n + mn) * sizeof(T));
}

}  // namespace

extern "C" {

size_t blasfeo_cm_memsize_dmat(int m, int n) { return cm_memsize<double, blasfeo_cm_dmat>(m, n); }
size_t blasfeo_cm_memsize_smat(int m, int n) { return cm_memsize<float, blasfeo_cm_smat>(m, n); }
void blasfeo_cm_create_dmat(int m, int n, struct blasfeo_cm_dmat *sA, void *memory) {
	cm_create<double>(m, n, sA, memory);
}
void blasfeo_cm_create_smat(int m, int n, struct blasfeo_cm_smat *sA, void *memory) {
	cm_create<float>(m, n, sA, memory);
}

void blasfeo_cm_dgemm_nt(int m, int n, int k, double alpha, struct blasfeo_cm_dmat *sA, int ai, int aj,
                         struct blasfeo_cm_dmat *sB, int bi, int bj, double beta, struct blasfeo_cm_dmat *sC, int ci,
                         int cj, struct blasfeo_cm_dmat *sD, int di, int dj) {
	cm_gemm<double>(m, n, k, alpha, sA, ai, aj, sB, bi, bj, beta, sC, ci, cj, sD, di, dj, false);
}
void blasfeo_cm_sgemm_nt(int m, int n, int k, float alpha, struct blasfeo_cm_smat *sA, int ai, int aj,
                         struct blasfeo_cm_smat *sB, int bi, int bj, float beta, struct blasfeo_cm_smat *sC, int ci,
                         int cj, struct blasfeo_cm_smat *sD, int di, int dj) {
	cm_gemm<float>(m, n, k, alpha, sA, ai, aj, sB, bi, bj, beta, sC, ci, cj, sD, di, dj, false);
}
void blasfeo_cm_dsyrk_ln(int m, int k, double alpha, struct blasfeo_cm_dmat *sA, int ai, int aj,
                         struct blasfeo_cm_dmat *sB, int bi, int bj, double beta, struct blasfeo_cm_dmat *sC, int ci,
                         int cj, struct blasfeo_cm_dmat *sD, int di, int dj) {
	cm_gemm<double>(m, m, k, alpha, sA, ai, aj, sB, bi, bj, beta, sC, ci, cj, sD, di, dj, true);
}
void blasfeo_cm_dtrsm_rltn(int m, int n, double alpha, struct blasfeo_cm_dmat *sA, int ai, int aj,
                           struct blasfeo_cm_dmat *sB, int bi, int bj, struct blasfeo_cm_dmat *sD, int di, int dj) {
	cm_trsm_rltn<double>(m, n, alpha, sA, ai, aj, sB, bi, bj, sD, di, dj);
}
void blasfeo_cm_strsm_rltn(int m, int n, float alpha, struct blasfeo_cm_smat *sA, int ai, int aj,
                           struct blasfeo_cm_smat *sB, int bi, int bj, struct blasfeo_cm_smat *sD, int di, int dj) {
	cm_trsm_rltn<float>(m, n, alpha, sA, ai, aj, sB, bi, bj, sD, di, dj);
}
void blasfeo_cm_dpotrf_l(int m, struct blasfeo_cm_dmat *sC, int ci, int cj, struct blasfeo_cm_dmat *sD, int di,
                         int dj) {
	cm_potrf_l<double>(m, sC, ci, cj, sD, di, dj);
}
void blasfeo_cm_spotrf_l(int m, struct blasfeo_cm_smat *sC, int ci, int cj, struct blasfeo_cm_smat *sD, int di,
                         int dj) {
	cm_potrf_l<float>(m, sC, ci, cj, sD, di, dj);
}
void blasfeo_cm_dgetrf_rp(int m, int n, struct blasfeo_cm_dmat *sC, int ci, int cj, struct blasfeo_cm_dmat *sD, int di,
                          int dj, int *ipiv) {
	cm_dgetrf_rp(m, n, sC, ci, cj, sD, di, dj, ipiv);
}

}  // extern "C"
