/*
 * blasfeo_b200 -- BLASFEO's level-3 / LAPACK hot path for NVIDIA B200 (sm_100a).
 *
 * C ABI of libblasfeo_b200.so.  Plain C types only: pointers, sizes, and the
 * BLASFEO descriptor structs.  CUDA streams are passed as `void *` (a
 * cudaStream_t; NULL = the legacy default stream).
 *
 * Drop-in part: the functions named blasfeo_d* / blasfeo_s* below keep the
 * names, argument lists and argument meanings of BLASFEO 0.1.4.2's BLASFEO API
 * (panel-major, LA=HIGH_PERFORMANCE), with one difference: the memory handed
 * to blasfeo_create_dmat / blasfeo_create_dvec is DEVICE memory (cudaMalloc),
 * so pA / dA / pa point into HBM.  The descriptor structs live in host memory
 * and have the reference's exact field layout.  Citations name the reference
 * prototype each entry point replaces (paths relative to the BLASFEO tree).
 *
 * Semantics kept from the reference:
 *   - panel-major storage with panel size 4 for both precisions: element (i,j)
 *     at pA[(i - i%4)*cn + 4*j + i%4]  (include/blasfeo_common.h:112);
 *   - pA followed by dA in the buffer, 64-byte rounded memsize;
 *   - dA holds the inverse diagonal after potrf/getrf (use_dA set), the cached
 *     inverse diagonal that trsm_rltn reuses, and tau after geqrf;
 *   - non-positive Cholesky pivot -> L_jj = 0, inverse 0, no error;
 *     zero LU pivot -> inverse 0; pivot = first row of the largest |a|;
 *     ipiv 0-based absolute row indices.
 * Differences: no exit(1) on unsupported offsets -- every offset is supported;
 * the single-instance calls synchronise their stream before returning unless
 * blasfeo_b200_set_sync(0) is in effect; errors are recorded and readable with
 * blasfeo_b200_last_error().
 *
 * Batched part (no reference counterpart; the reference is single-instance):
 *   *_batch   uniform batch, all instances the same size, stored as a strided
 *             slab (struct blasfeo_dmat_batch); asynchronous on `stream`.
 *   *_vbatch  variable-size batch: device arrays of per-instance sizes and of
 *             per-instance descriptors (struct blasfeo_dmat in device memory,
 *             pA/dA pointing to device memory); asynchronous on `stream`.
 * Batched calls return a status code (0 = launched) and, where given, write a
 * per-instance info[] (device memory): 0 = ok, j+1 = first bad pivot at j.
 */
#ifndef BLASFEO_B200_H_
#define BLASFEO_B200_H_

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BLASFEO_B200_PS 4

/* ---- descriptors: include/blasfeo_common.h:67-110 (identical layout) ---- */
struct blasfeo_dmat {
	double *mem;  /* device memory passed to create */
	double *pA;   /* device: pm*cn panel-major doubles */
	double *dA;   /* device: inverse diagonal / tau, min(m,n) rounded to 16 */
	int m, n, pm, cn;
	int use_dA;   /* host-side flag: dA holds a valid inverse diagonal for use_dA columns */
	int memsize;
};
struct blasfeo_smat {
	float *mem; float *pA; float *dA;
	int m, n, pm, cn;
	int use_dA;
	int memsize;
};
struct blasfeo_dvec { double *mem; double *pa; int m, pm, memsize; };
struct blasfeo_svec { float *mem; float *pa; int m, pm, memsize; };

/* uniform batch: `batch` consecutive instances, instance b's storage starts at
 * mem + b*stride elements and is laid out exactly as blasfeo_create_dmat lays
 * out one matrix (pA, then dA). */
struct blasfeo_dmat_batch {
	double *mem; double *pA; double *dA;
	int m, n, pm, cn;
	int use_dA;
	int batch;
	long long stride;   /* elements between instances */
	size_t memsize;     /* bytes of the whole slab */
};
struct blasfeo_smat_batch {
	float *mem; float *pA; float *dA;
	int m, n, pm, cn;
	int use_dA;
	int batch;
	long long stride;
	size_t memsize;
};

/* batch-interleaved uniform batch (no reference counterpart): instances in
 * groups of il (16); element slot e of the panel layout (element (i,j) at
 * e = (i - i%4)*cn + 4*j + i%4, then the inverse diagonal at e = pm*cn + k)
 * of instance b at mem[(b / il) * gstride + e * il + b % il], so one element of
 * 16 consecutive instances is one contiguous 128-byte run. */
struct blasfeo_dmat_batch_il {
	double *mem;
	int m, n, pm, cn;
	int batch;
	int il;
	long long gstride;  /* elements per group of il instances */
	size_t memsize;     /* bytes of the whole slab */
};

/* column-major descriptors, include/blasfeo_common.h:220-229 (same fields and
 * order): pA is a column-major array in DEVICE memory whose leading dimension
 * is m, element (i,j) at pA[i + j*m] (the reference's BLAS API sets m = lda). */
struct blasfeo_cm_dmat {
	double *mem; double *pA; double *dA;
	int m, n;
	int use_dA;
	int memsize;
};
struct blasfeo_cm_smat {
	float *mem; float *pA; float *dA;
	int m, n;
	int use_dA;
	int memsize;
};

/* status codes */
#define BLASFEO_B200_OK 0
#define BLASFEO_B200_EINVAL 1      /* bad argument (size, NULL pointer, out of range) */
#define BLASFEO_B200_ECUDA 2       /* a CUDA call failed */
#define BLASFEO_B200_ENOMEM 3      /* workspace too small / allocation failed */
#define BLASFEO_B200_ENOTSUP 4     /* size beyond what the kernel supports */

/* ---- library state ---- */
int blasfeo_b200_last_error(void);                  /* last status of a void entry point, then cleared */
const char *blasfeo_b200_error_string(int status);
void blasfeo_b200_set_stream(void *stream);         /* stream of the single-instance entry points (per host thread) */
void *blasfeo_b200_get_stream(void);
void blasfeo_b200_set_sync(int sync);               /* 1 (default): single-instance calls synchronise before return */
int blasfeo_b200_version(void);
/* measured FMA throughput (GFLOP/s) of the current device, prec 'd' or 's';
 * the roofline denominator of the SIMT kernels (no reference counterpart) */
double blasfeo_b200_measure_fma_peak(char prec, int iters);
/* Polls of every bounded mbarrier wait of the kernels that use bulk copies
 * (the fused n=16 chain, the batched Riccati factorization, the tensor-memory
 * engine of the mixed solver), process-wide; 0 restores the default (2^24
 * polls, about one second).  A wait that runs out sets the instance's
 * info = -3 and the kernel returns after draining its copies (no reference
 * counterpart: the reference has no asynchronous copies). */
void blasfeo_b200_set_wait_limit(unsigned int polls);
unsigned int blasfeo_b200_get_wait_limit(void);
/* Self-check of that timeout path: one warp waits, with the current limit, on
 * an mbarrier armed for data that no copy delivers; *status (device int)
 * receives -3 when the wait ran out (0 if it did not).  Asynchronous on
 * `stream`. */
int blasfeo_b200_check_wait_timeout(int *status, void *stream);

/* ---- storage: auxiliary/d_aux_lib4.c:1519,1548,1575,1588 / include/blasfeo_d_aux.h ---- */
size_t blasfeo_memsize_dmat(int m, int n);
size_t blasfeo_memsize_diag_dmat(int m, int n);
void blasfeo_create_dmat(int m, int n, struct blasfeo_dmat *sA, void *memory);
size_t blasfeo_memsize_dvec(int m);
void blasfeo_create_dvec(int m, struct blasfeo_dvec *sa, void *memory);
size_t blasfeo_memsize_smat(int m, int n);
size_t blasfeo_memsize_diag_smat(int m, int n);
void blasfeo_create_smat(int m, int n, struct blasfeo_smat *sA, void *memory);
size_t blasfeo_memsize_svec(int m);
void blasfeo_create_svec(int m, struct blasfeo_svec *sa, void *memory);

/* host column-major A (lda) <-> device panel-major sA: auxiliary/d_aux_lib4.c:1607 (pack), :2238 (unpack) */
void blasfeo_pack_dmat(int m, int n, double *A, int lda, struct blasfeo_dmat *sA, int ai, int aj);
void blasfeo_unpack_dmat(int m, int n, struct blasfeo_dmat *sA, int ai, int aj, double *A, int lda);
/* transposed: auxiliary/d_aux_lib4.c:2086 (pack_tran: sA's n x m block at
 * (ai,aj) = A^T, A m x n column-major), :2360 (unpack_tran: A n x m = block^T) */
void blasfeo_pack_tran_dmat(int m, int n, double *A, int lda, struct blasfeo_dmat *sA, int ai, int aj);
void blasfeo_unpack_tran_dmat(int m, int n, struct blasfeo_dmat *sA, int ai, int aj, double *A, int lda);
void blasfeo_pack_tran_smat(int m, int n, float *A, int lda, struct blasfeo_smat *sA, int ai, int aj);
void blasfeo_unpack_tran_smat(int m, int n, struct blasfeo_smat *sA, int ai, int aj, float *A, int lda);
void blasfeo_pack_dvec(int m, double *x, int xi, struct blasfeo_dvec *sa, int ai);
void blasfeo_unpack_dvec(int m, struct blasfeo_dvec *sa, int ai, double *x, int xi);
void blasfeo_pack_smat(int m, int n, float *A, int lda, struct blasfeo_smat *sA, int ai, int aj);
void blasfeo_unpack_smat(int m, int n, struct blasfeo_smat *sA, int ai, int aj, float *A, int lda);

/* ---- column-major drop-in (device-resident column-major matrices) ----
 * storage: auxiliary/d_aux_common.c:111,121 (m*n elements, then min(m,n) for
 * dA; the reference declares create with a struct blasfeo_pm_dmat pointer,
 * include/blasfeo_d_aux.h:237, these take the column-major descriptor).
 * Routines: include/blasfeo_d_blasfeo_api.h:321 (gemm_nt), :324 (syrk_ln,
 * lower triangle of D written), :342 (trsm_rltn), :389 (potrf_l, lower
 * triangle of D written), :391 (getrf_rp, ipiv: host array of min(m,n)
 * 0-based absolute row indices); include/blasfeo_s_blasfeo_api.h:282, :295,
 * :305.  Same arguments and results as the panel-major routines of the same
 * name; dA / use_dA are neither read nor written (as in blasfeo_hp_cm/).
 * Single-instance semantics as the panel-major drop-ins (stream, sync, last
 * error). */
size_t blasfeo_cm_memsize_dmat(int m, int n);
void blasfeo_cm_create_dmat(int m, int n, struct blasfeo_cm_dmat *sA, void *memory);
size_t blasfeo_cm_memsize_smat(int m, int n);
void blasfeo_cm_create_smat(int m, int n, struct blasfeo_cm_smat *sA, void *memory);
void blasfeo_cm_dgemm_nt(int m, int n, int k, double alpha, struct blasfeo_cm_dmat *sA, int ai, int aj,
                         struct blasfeo_cm_dmat *sB, int bi, int bj, double beta, struct blasfeo_cm_dmat *sC, int ci,
                         int cj, struct blasfeo_cm_dmat *sD, int di, int dj);
void blasfeo_cm_dsyrk_ln(int m, int k, double alpha, struct blasfeo_cm_dmat *sA, int ai, int aj,
                         struct blasfeo_cm_dmat *sB, int bi, int bj, double beta, struct blasfeo_cm_dmat *sC, int ci,
                         int cj, struct blasfeo_cm_dmat *sD, int di, int dj);
void blasfeo_cm_dtrsm_rltn(int m, int n, double alpha, struct blasfeo_cm_dmat *sA, int ai, int aj,
                           struct blasfeo_cm_dmat *sB, int bi, int bj, struct blasfeo_cm_dmat *sD, int di, int dj);
void blasfeo_cm_dpotrf_l(int m, struct blasfeo_cm_dmat *sC, int ci, int cj, struct blasfeo_cm_dmat *sD, int di, int dj);
void blasfeo_cm_dgetrf_rp(int m, int n, struct blasfeo_cm_dmat *sC, int ci, int cj, struct blasfeo_cm_dmat *sD, int di,
                          int dj, int *ipiv);
void blasfeo_cm_sgemm_nt(int m, int n, int k, float alpha, struct blasfeo_cm_smat *sA, int ai, int aj,
                         struct blasfeo_cm_smat *sB, int bi, int bj, float beta, struct blasfeo_cm_smat *sC, int ci,
                         int cj, struct blasfeo_cm_smat *sD, int di, int dj);
void blasfeo_cm_strsm_rltn(int m, int n, float alpha, struct blasfeo_cm_smat *sA, int ai, int aj,
                           struct blasfeo_cm_smat *sB, int bi, int bj, struct blasfeo_cm_smat *sD, int di, int dj);
void blasfeo_cm_spotrf_l(int m, struct blasfeo_cm_smat *sC, int ci, int cj, struct blasfeo_cm_smat *sD, int di, int dj);
void blasfeo_pack_svec(int m, float *x, int xi, struct blasfeo_svec *sa, int ai);
void blasfeo_unpack_svec(int m, struct blasfeo_svec *sa, int ai, float *x, int xi);
/* include/blasfeo_d_aux.h:115 dgecp, :141 ddiare, :162 drowsw */
void blasfeo_dgecp(int m, int n, struct blasfeo_dmat *sA, int ai, int aj, struct blasfeo_dmat *sB, int bi, int bj);
void blasfeo_ddiare(int kmax, double alpha, struct blasfeo_dmat *sA, int ai, int aj);
void blasfeo_drowsw(int kmax, struct blasfeo_dmat *sA, int ai, int aj, struct blasfeo_dmat *sC, int ci, int cj);
void blasfeo_sgecp(int m, int n, struct blasfeo_smat *sA, int ai, int aj, struct blasfeo_smat *sB, int bi, int bj);
void blasfeo_sdiare(int kmax, float alpha, struct blasfeo_smat *sA, int ai, int aj);
void blasfeo_srowsw(int kmax, struct blasfeo_smat *sA, int ai, int aj, struct blasfeo_smat *sC, int ci, int cj);

/* ---- level 3: include/blasfeo_d_blasfeo_api.h:143 (gemm_nt), :149 (syrk_ln), :222 (trsm_rltn), :186 (trmm_rlnn) ---- */
void blasfeo_dgemm_nt(int m, int n, int k, double alpha, struct blasfeo_dmat *sA, int ai, int aj,
	struct blasfeo_dmat *sB, int bi, int bj, double beta, struct blasfeo_dmat *sC, int ci, int cj,
	struct blasfeo_dmat *sD, int di, int dj);
void blasfeo_dsyrk_ln(int m, int k, double alpha, struct blasfeo_dmat *sA, int ai, int aj,
	struct blasfeo_dmat *sB, int bi, int bj, double beta, struct blasfeo_dmat *sC, int ci, int cj,
	struct blasfeo_dmat *sD, int di, int dj);
void blasfeo_dtrsm_rltn(int m, int n, double alpha, struct blasfeo_dmat *sA, int ai, int aj,
	struct blasfeo_dmat *sB, int bi, int bj, struct blasfeo_dmat *sD, int di, int dj);
void blasfeo_dtrmm_rlnn(int m, int n, double alpha, struct blasfeo_dmat *sA, int ai, int aj,
	struct blasfeo_dmat *sB, int bi, int bj, struct blasfeo_dmat *sD, int di, int dj);
/* include/blasfeo_s_blasfeo_api.h (same lines, single precision) */
void blasfeo_sgemm_nt(int m, int n, int k, float alpha, struct blasfeo_smat *sA, int ai, int aj,
	struct blasfeo_smat *sB, int bi, int bj, float beta, struct blasfeo_smat *sC, int ci, int cj,
	struct blasfeo_smat *sD, int di, int dj);
void blasfeo_ssyrk_ln(int m, int k, float alpha, struct blasfeo_smat *sA, int ai, int aj,
	struct blasfeo_smat *sB, int bi, int bj, float beta, struct blasfeo_smat *sC, int ci, int cj,
	struct blasfeo_smat *sD, int di, int dj);
void blasfeo_strsm_rltn(int m, int n, float alpha, struct blasfeo_smat *sA, int ai, int aj,
	struct blasfeo_smat *sB, int bi, int bj, struct blasfeo_smat *sD, int di, int dj);
void blasfeo_strmm_rlnn(int m, int n, float alpha, struct blasfeo_smat *sA, int ai, int aj,
	struct blasfeo_smat *sB, int bi, int bj, struct blasfeo_smat *sD, int di, int dj);

/* ---- LAPACK: include/blasfeo_d_blasfeo_api.h:280 (potrf_l), :286 (syrk_dpotrf_ln), :291 (getrf_rp), :293-294 (geqrf) ---- */
void blasfeo_dpotrf_l(int m, struct blasfeo_dmat *sC, int ci, int cj, struct blasfeo_dmat *sD, int di, int dj);
void blasfeo_dsyrk_dpotrf_ln(int m, int k, struct blasfeo_dmat *sA, int ai, int aj, struct blasfeo_dmat *sB, int bi, int bj,
	struct blasfeo_dmat *sC, int ci, int cj, struct blasfeo_dmat *sD, int di, int dj);
/* ipiv: HOST array of min(m,n) ints, as in the reference */
void blasfeo_dgetrf_rp(int m, int n, struct blasfeo_dmat *sC, int ci, int cj, struct blasfeo_dmat *sD, int di, int dj, int *ipiv);
int blasfeo_dgeqrf_worksize(int m, int n);
/* work: unused by the device kernels (may be NULL); kept for the signature */
void blasfeo_dgeqrf(int m, int n, struct blasfeo_dmat *sC, int ci, int cj, struct blasfeo_dmat *sD, int di, int dj, void *work);
void blasfeo_spotrf_l(int m, struct blasfeo_smat *sC, int ci, int cj, struct blasfeo_smat *sD, int di, int dj);
void blasfeo_ssyrk_spotrf_ln(int m, int k, struct blasfeo_smat *sA, int ai, int aj, struct blasfeo_smat *sB, int bi, int bj,
	struct blasfeo_smat *sC, int ci, int cj, struct blasfeo_smat *sD, int di, int dj);
void blasfeo_sgetrf_rp(int m, int n, struct blasfeo_smat *sC, int ci, int cj, struct blasfeo_smat *sD, int di, int dj, int *ipiv);
int blasfeo_sgeqrf_worksize(int m, int n);
void blasfeo_sgeqrf(int m, int n, struct blasfeo_smat *sC, int ci, int cj, struct blasfeo_smat *sD, int di, int dj, void *work);

/* ---- adjacent variants: include/blasfeo_d_blasfeo_api.h:150 (syrk_ln_mn), :224 (trsm_rltu),
 *      :281 (potrf_l_mn), :289 (getrf_np); s twins include/blasfeo_s_blasfeo_api.h:146, :208, :242, :249 ----
 * syrk_ln_mn: lower trapezoid (m x n, j <= i) of D = beta*C + alpha*A*B^T.
 * trsm_rltu:  D = alpha * B * A^{-T}, A lower with unit diagonal (not read).
 * potrf_l_mn: Cholesky of the m x n lower trapezoid (n clamped to m): the n x n
 *             factor and the rows below solved against it; 1/L_jj in dA,
 *             use_dA = 1 with zero offsets (as the reference sets it).
 * getrf_np:   LU without pivoting, unit L below and U on/above the diagonal of
 *             D, 1/U_jj in dA (a zero pivot divides by zero, as the reference). */
void blasfeo_dsyrk_ln_mn(int m, int n, int k, double alpha, struct blasfeo_dmat *sA, int ai, int aj,
	struct blasfeo_dmat *sB, int bi, int bj, double beta, struct blasfeo_dmat *sC, int ci, int cj,
	struct blasfeo_dmat *sD, int di, int dj);
void blasfeo_dtrsm_rltu(int m, int n, double alpha, struct blasfeo_dmat *sA, int ai, int aj,
	struct blasfeo_dmat *sB, int bi, int bj, struct blasfeo_dmat *sD, int di, int dj);
void blasfeo_dpotrf_l_mn(int m, int n, struct blasfeo_dmat *sC, int ci, int cj, struct blasfeo_dmat *sD, int di, int dj);
void blasfeo_dgetrf_np(int m, int n, struct blasfeo_dmat *sC, int ci, int cj, struct blasfeo_dmat *sD, int di, int dj);
void blasfeo_ssyrk_ln_mn(int m, int n, int k, float alpha, struct blasfeo_smat *sA, int ai, int aj,
	struct blasfeo_smat *sB, int bi, int bj, float beta, struct blasfeo_smat *sC, int ci, int cj,
	struct blasfeo_smat *sD, int di, int dj);
void blasfeo_strsm_rltu(int m, int n, float alpha, struct blasfeo_smat *sA, int ai, int aj,
	struct blasfeo_smat *sB, int bi, int bj, struct blasfeo_smat *sD, int di, int dj);
void blasfeo_spotrf_l_mn(int m, int n, struct blasfeo_smat *sC, int ci, int cj, struct blasfeo_smat *sD, int di, int dj);
void blasfeo_sgetrf_np(int m, int n, struct blasfeo_smat *sC, int ci, int cj, struct blasfeo_smat *sD, int di, int dj);

/* ---- level 2 used by the solve chains: include/blasfeo_d_blasfeo_api.h:85 (gemv_n), :93 (trsv_lnn), :97 (trsv_ltn) ---- */
void blasfeo_dgemv_n(int m, int n, double alpha, struct blasfeo_dmat *sA, int ai, int aj, struct blasfeo_dvec *sx, int xi,
	double beta, struct blasfeo_dvec *sy, int yi, struct blasfeo_dvec *sz, int zi);
void blasfeo_dtrsv_lnn(int m, struct blasfeo_dmat *sA, int ai, int aj, struct blasfeo_dvec *sx, int xi, struct blasfeo_dvec *sz, int zi);
void blasfeo_dtrsv_ltn(int m, struct blasfeo_dmat *sA, int ai, int aj, struct blasfeo_dvec *sx, int xi, struct blasfeo_dvec *sz, int zi);

/* ---- uniform batches (no reference counterpart) ---- */
size_t blasfeo_memsize_dmat_batch(int m, int n, int batch);
void blasfeo_create_dmat_batch(int m, int n, int batch, struct blasfeo_dmat_batch *sA, void *memory);
void blasfeo_dmat_batch_instance(struct blasfeo_dmat_batch *sA, int b, struct blasfeo_dmat *out);
/* batch-interleaved slabs (no reference counterpart): size, creation, and
 * conversion from / to the back-to-back slab of the same m x n (on `stream`;
 * EINVAL for mismatched sizes or a source with fewer instances). */
size_t blasfeo_memsize_dmat_batch_il(int m, int n, int batch);
void blasfeo_create_dmat_batch_il(int m, int n, int batch, struct blasfeo_dmat_batch_il *sA, void *memory);
int blasfeo_dmat_batch_to_il(const struct blasfeo_dmat_batch *src, struct blasfeo_dmat_batch_il *dst, void *stream);
int blasfeo_dmat_batch_from_il(const struct blasfeo_dmat_batch_il *src, struct blasfeo_dmat_batch *dst, void *stream);
/* Host column-major batch (instance b at A + b*strideA, leading dimension lda,
 * the batched form of blasfeo_pack_dmat / blasfeo_unpack_dmat,
 * auxiliary/d_aux_lib4.c:1607,2238) <-> the top-left m x n block of an
 * interleaved slab: one host copy and one conversion kernel; returns when the
 * copy is complete. */
int blasfeo_pack_dmat_batch_il(int batch, int m, int n, const double *A, int lda, long long strideA,
	struct blasfeo_dmat_batch_il *sB, void *stream);
int blasfeo_unpack_dmat_batch_il(int batch, int m, int n, const struct blasfeo_dmat_batch_il *sB, double *A, int lda,
	long long strideA, void *stream);
/* potrf_l (include/blasfeo_d_blasfeo_api.h:280, one instance per lane pair)
 * on interleaved slabs of equal geometry, m <= 16 (else ENOTSUP): the m x m
 * lower factor of each instance of sC into sD with the inverse diagonal in its
 * dA slots; info[b] as for blasfeo_dpotrf_l_batch. */
int blasfeo_dpotrf_l_batch_il(int batch, int m, struct blasfeo_dmat_batch_il *sC, struct blasfeo_dmat_batch_il *sD,
	int *info, void *stream);
/* The fused chain blasfeo_dsyrk_dpotrf_dtrsm_dgemm_batch on interleaved slabs
 * (one instance per quad of lanes): m = 16 only (else ENOTSUP), sA 16 x k with
 * k >= 1, sR, sC, sG, sL, sX, sD 16 x 16 of one group stride; results equal to
 * the back-to-back call's, info[b] as there (never -3: no bulk copies). */
int blasfeo_dsyrk_dpotrf_dtrsm_dgemm_batch_il(int batch, int m, int k, double shift,
	struct blasfeo_dmat_batch_il *sA, struct blasfeo_dmat_batch_il *sR, struct blasfeo_dmat_batch_il *sC,
	struct blasfeo_dmat_batch_il *sG, struct blasfeo_dmat_batch_il *sL, struct blasfeo_dmat_batch_il *sX,
	struct blasfeo_dmat_batch_il *sD, int *info, void *stream);
/* The Riccati factorization blasfeo_dric_trf_batch on interleaved slabs (one
 * problem per quad of lanes), nu + nx <= 16 (else ENOTSUP).  Stage-major
 * slabs: stage k of problem b is instance k * bs + b, bs = batch rounded up
 * to a multiple of 16 (so the problems of a group sit side by side at every
 * stage); sBAbt 16 x nx with >= N * bs instances, sRSQ and sL 16 x 16 with
 * >= (N+1) * bs instances, all on 16-byte boundaries (else EINVAL).  Outputs
 * and info[b] as blasfeo_dric_trf_batch (never -3: no bulk-copy waits). */
int blasfeo_dric_trf_batch_il(int batch, int N, int nx, int nu, struct blasfeo_dmat_batch_il *sBAbt,
	struct blasfeo_dmat_batch_il *sRSQ, struct blasfeo_dmat_batch_il *sL, int *info, void *stream);

/* Host column-major batch <-> uniform-batch slab (no reference counterpart;
 * the batched form of blasfeo_pack_dmat / blasfeo_unpack_dmat): instance b of
 * the host array starts at A + b*strideA (ld lda) and maps to the m x n block
 * at (bi, bj) of slab instance b.  One host<->device copy of the whole batch
 * (a single 2-D copy when strideA == lda*n) through the library staging
 * buffer, one conversion kernel; returns after the copies completed on
 * `stream`.  BLASFEO_B200_EINVAL for out-of-range sizes or offsets. */
int blasfeo_pack_dmat_batch(int batch, int m, int n, const double *A, int lda, long long strideA,
	struct blasfeo_dmat_batch *sB, int bi, int bj, void *stream);
int blasfeo_unpack_dmat_batch(int batch, int m, int n, struct blasfeo_dmat_batch *sB, int bi, int bj, double *A,
	int lda, long long strideA, void *stream);
int blasfeo_pack_smat_batch(int batch, int m, int n, const float *A, int lda, long long strideA,
	struct blasfeo_smat_batch *sB, int bi, int bj, void *stream);
int blasfeo_unpack_smat_batch(int batch, int m, int n, struct blasfeo_smat_batch *sB, int bi, int bj, float *A,
	int lda, long long strideA, void *stream);
size_t blasfeo_memsize_smat_batch(int m, int n, int batch);
void blasfeo_create_smat_batch(int m, int n, int batch, struct blasfeo_smat_batch *sA, void *memory);
void blasfeo_smat_batch_instance(struct blasfeo_smat_batch *sA, int b, struct blasfeo_smat *out);

int blasfeo_dgemm_nt_batch(int batch, int m, int n, int k, double alpha, struct blasfeo_dmat_batch *sA, int ai, int aj,
	struct blasfeo_dmat_batch *sB, int bi, int bj, double beta, struct blasfeo_dmat_batch *sC, int ci, int cj,
	struct blasfeo_dmat_batch *sD, int di, int dj, void *stream);
int blasfeo_dsyrk_ln_batch(int batch, int m, int k, double alpha, struct blasfeo_dmat_batch *sA, int ai, int aj,
	struct blasfeo_dmat_batch *sB, int bi, int bj, double beta, struct blasfeo_dmat_batch *sC, int ci, int cj,
	struct blasfeo_dmat_batch *sD, int di, int dj, void *stream);
int blasfeo_dtrsm_rltn_batch(int batch, int m, int n, double alpha, struct blasfeo_dmat_batch *sA, int ai, int aj,
	struct blasfeo_dmat_batch *sB, int bi, int bj, struct blasfeo_dmat_batch *sD, int di, int dj, void *stream);
int blasfeo_dpotrf_l_batch(int batch, int m, struct blasfeo_dmat_batch *sC, int ci, int cj,
	struct blasfeo_dmat_batch *sD, int di, int dj, int *info, void *stream);
int blasfeo_dsyrk_dpotrf_ln_batch(int batch, int m, int k, struct blasfeo_dmat_batch *sA, int ai, int aj,
	struct blasfeo_dmat_batch *sB, int bi, int bj, struct blasfeo_dmat_batch *sC, int ci, int cj,
	struct blasfeo_dmat_batch *sD, int di, int dj, int *info, void *stream);
/* ipiv: device array, batch * min(m,n) ints */
int blasfeo_dgetrf_rp_batch(int batch, int m, int n, struct blasfeo_dmat_batch *sC, int ci, int cj,
	struct blasfeo_dmat_batch *sD, int di, int dj, int *ipiv, int *info, void *stream);
int blasfeo_dgeqrf_batch(int batch, int m, int n, struct blasfeo_dmat_batch *sC, int ci, int cj,
	struct blasfeo_dmat_batch *sD, int di, int dj, void *stream);

int blasfeo_sgemm_nt_batch(int batch, int m, int n, int k, float alpha, struct blasfeo_smat_batch *sA, int ai, int aj,
	struct blasfeo_smat_batch *sB, int bi, int bj, float beta, struct blasfeo_smat_batch *sC, int ci, int cj,
	struct blasfeo_smat_batch *sD, int di, int dj, void *stream);
int blasfeo_ssyrk_ln_batch(int batch, int m, int k, float alpha, struct blasfeo_smat_batch *sA, int ai, int aj,
	struct blasfeo_smat_batch *sB, int bi, int bj, float beta, struct blasfeo_smat_batch *sC, int ci, int cj,
	struct blasfeo_smat_batch *sD, int di, int dj, void *stream);
int blasfeo_strsm_rltn_batch(int batch, int m, int n, float alpha, struct blasfeo_smat_batch *sA, int ai, int aj,
	struct blasfeo_smat_batch *sB, int bi, int bj, struct blasfeo_smat_batch *sD, int di, int dj, void *stream);
int blasfeo_spotrf_l_batch(int batch, int m, struct blasfeo_smat_batch *sC, int ci, int cj,
	struct blasfeo_smat_batch *sD, int di, int dj, int *info, void *stream);
int blasfeo_ssyrk_spotrf_ln_batch(int batch, int m, int k, struct blasfeo_smat_batch *sA, int ai, int aj,
	struct blasfeo_smat_batch *sB, int bi, int bj, struct blasfeo_smat_batch *sC, int ci, int cj,
	struct blasfeo_smat_batch *sD, int di, int dj, int *info, void *stream);
int blasfeo_sgetrf_rp_batch(int batch, int m, int n, struct blasfeo_smat_batch *sC, int ci, int cj,
	struct blasfeo_smat_batch *sD, int di, int dj, int *ipiv, int *info, void *stream);
int blasfeo_sgeqrf_batch(int batch, int m, int n, struct blasfeo_smat_batch *sC, int ci, int cj,
	struct blasfeo_smat_batch *sD, int di, int dj, void *stream);
/* uniform batches of the adjacent variants (info: first bad pivot + 1, or 0) */
int blasfeo_dsyrk_ln_mn_batch(int batch, int m, int n, int k, double alpha, struct blasfeo_dmat_batch *sA, int ai, int aj,
	struct blasfeo_dmat_batch *sB, int bi, int bj, double beta, struct blasfeo_dmat_batch *sC, int ci, int cj,
	struct blasfeo_dmat_batch *sD, int di, int dj, void *stream);
int blasfeo_dtrsm_rltu_batch(int batch, int m, int n, double alpha, struct blasfeo_dmat_batch *sA, int ai, int aj,
	struct blasfeo_dmat_batch *sB, int bi, int bj, struct blasfeo_dmat_batch *sD, int di, int dj, void *stream);
int blasfeo_dpotrf_l_mn_batch(int batch, int m, int n, struct blasfeo_dmat_batch *sC, int ci, int cj,
	struct blasfeo_dmat_batch *sD, int di, int dj, int *info, void *stream);
int blasfeo_dgetrf_np_batch(int batch, int m, int n, struct blasfeo_dmat_batch *sC, int ci, int cj,
	struct blasfeo_dmat_batch *sD, int di, int dj, int *info, void *stream);
int blasfeo_ssyrk_ln_mn_batch(int batch, int m, int n, int k, float alpha, struct blasfeo_smat_batch *sA, int ai, int aj,
	struct blasfeo_smat_batch *sB, int bi, int bj, float beta, struct blasfeo_smat_batch *sC, int ci, int cj,
	struct blasfeo_smat_batch *sD, int di, int dj, void *stream);
int blasfeo_strsm_rltu_batch(int batch, int m, int n, float alpha, struct blasfeo_smat_batch *sA, int ai, int aj,
	struct blasfeo_smat_batch *sB, int bi, int bj, struct blasfeo_smat_batch *sD, int di, int dj, void *stream);
int blasfeo_spotrf_l_mn_batch(int batch, int m, int n, struct blasfeo_smat_batch *sC, int ci, int cj,
	struct blasfeo_smat_batch *sD, int di, int dj, int *info, void *stream);
int blasfeo_sgetrf_np_batch(int batch, int m, int n, struct blasfeo_smat_batch *sC, int ci, int cj,
	struct blasfeo_smat_batch *sD, int di, int dj, int *info, void *stream);

/* ---- variable-size batches (no reference counterpart) ----
 * Size arrays (m, n, k) and descriptor arrays (sA, ...) are DEVICE arrays of
 * `batch` entries; max_* are upper bounds of the sizes (used for grid and
 * shared-memory sizing).  All offsets are zero. */
int blasfeo_dgemm_nt_vbatch(int batch, const int *m, const int *n, const int *k, int max_m, int max_n, int max_k,
	double alpha, const struct blasfeo_dmat *sA, const struct blasfeo_dmat *sB, double beta,
	const struct blasfeo_dmat *sC, const struct blasfeo_dmat *sD, void *stream);
int blasfeo_dpotrf_l_vbatch(int batch, const int *m, int max_m, const struct blasfeo_dmat *sC,
	const struct blasfeo_dmat *sD, int *info, void *stream);
/* ipiv: device array, instance b uses ipiv[b*ipiv_stride ...] */
int blasfeo_dgetrf_rp_vbatch(int batch, const int *m, const int *n, int max_m, int max_n,
	const struct blasfeo_dmat *sC, const struct blasfeo_dmat *sD, int *ipiv, int ipiv_stride, int *info, void *stream);
int blasfeo_dgeqrf_vbatch(int batch, const int *m, const int *n, int max_m, int max_n,
	const struct blasfeo_dmat *sC, const struct blasfeo_dmat *sD, void *stream);

/* Kernel-variant selection for the variable-size batches (used by the
 * autotuner and the learned cost model; variant -1 = built-in heuristic).
 * op 0 gemm_nt: 0..3 SIMT tile shapes; 4 = 64x64 and 5 = 32x32 tiles on the
 *   FP64 tensor cores (the s-twin runs 4 and 5 as SIMT tiles);
 * op 1 potrf_l: 0..3 shared memory with 64/128/256/512 threads, 4 global
 *   memory, 5 one warp per instance on the FP64 tensor cores (max_m <= 64;
 *   larger batches take the heuristic);
 * op 2 getrf_rp: 0..2 blocked in global memory (128 threads with 4 or 3
 *   blocks per SM (2 when the largest matrix exceeds 288), 256 threads), 3..5
 *   shared memory with 128/256/512 threads;
 * op 3 geqrf: 0..2 blocked in global memory (256 threads with the SIMT
 *   trailing update, 256 threads (2 per SM) and 512 threads with the FP64
 *   tensor-core update), 3..5
 *   shared memory with 128/256/512 threads.
 * Variants change the schedule and, through the summation order of the dot
 * products, the rounding of an element; every variant meets the routine's
 * tolerance against the reference (pivot choices of getrf are identical). */
int blasfeo_b200_num_variants(int op);
int blasfeo_dgemm_nt_vbatch_variant(int batch, const int *m, const int *n, const int *k, int max_m, int max_n, int max_k,
	double alpha, const struct blasfeo_dmat *sA, const struct blasfeo_dmat *sB, double beta,
	const struct blasfeo_dmat *sC, const struct blasfeo_dmat *sD, int variant, void *stream);
int blasfeo_dpotrf_l_vbatch_variant(int batch, const int *m, int max_m, const struct blasfeo_dmat *sC,
	const struct blasfeo_dmat *sD, int *info, int variant, void *stream);
int blasfeo_dgetrf_rp_vbatch_variant(int batch, const int *m, const int *n, int max_m, int max_n,
	const struct blasfeo_dmat *sC, const struct blasfeo_dmat *sD, int *ipiv, int ipiv_stride, int *info, int variant,
	void *stream);
int blasfeo_dgeqrf_vbatch_variant(int batch, const int *m, const int *n, int max_m, int max_n,
	const struct blasfeo_dmat *sC, const struct blasfeo_dmat *sD, int variant, void *stream);

/* Learned dispatch (no reference counterpart).  With a cost model installed,
 * the four *_vbatch_variant routines called with variant -1 (and the plain
 * *_vbatch routines, which pass -1) take the variant the model predicts
 * fastest instead of the built-in rule.  The model is the MLP of the
 * blasfeo_b200_mlp_* kernels with nin = blasfeo_b200_cost_model_nfeat() inputs:
 *   [op one-hot (gemm_nt, potrf_l, getrf_rp, geqrf), log2(batch)/13,
 *    mean/9, max/9 and std/4 of log2 of the per-instance m, n and k,
 *    variant one-hot (6)]
 * (potrf_l: m = n = k = the sizes; getrf_rp, geqrf: k = n), trained to
 * predict the log run time.  A pick runs the feature and MLP kernels on the
 * launch's stream and synchronises it once to read the predictions; picks are
 * cached per (device, op, batch, max_m, max_n, max_k), so a repeated launch
 * shape dispatches without the model.  A stream under capture never runs the
 * model (a cached pick, else the built-in rule).  set copies the parameters
 * (blasfeo_b200_mlp_param_count(nin, hidden) floats, host memory) and clears
 * the cache; EINVAL for a wrong nin.  dispatch_pick returns the variant a
 * launch would take (-1: the built-in rule; -2: bad arguments). */
int blasfeo_b200_cost_model_nfeat(void);
int blasfeo_b200_set_cost_model(int nin, int hidden, const float *params);
void blasfeo_b200_clear_cost_model(void);
int blasfeo_b200_dispatch_pick(int op, int batch, const int *m, const int *n, const int *k, int max_m, int max_n,
	int max_k, void *stream);

/* ---- fused solvers (no reference counterpart; built from dpotrf_l + dtrsv_lnn + dtrsv_ltn) ----
 * Solve A x = b for a variable-size batch of SPD systems; A is read from the
 * lower triangle of each descriptor (full storage, upper part ignored).
 *   dposv:  plain FP64 factor and solve (x written to sx).
 *   dsposv: FP32 factor (FP64 diagonal blocks, FP64 pivots), FP64 residual and
 *           iterative refinement until ||b-Ax||_inf <= tol*||A||_inf*||x||_inf
 *           or max_iter refinement steps; iters[b] / berr[b] (device, may be NULL)
 *           receive the step count and final backward error; info[b] = -1 when
 *           refinement did not reach tol.
 * work/work_bytes: device workspace; NULL uses a library-owned workspace (one
 * per host thread and device, like the stream of the single-instance calls).
 * blasfeo_dposv_worksize_n(batch, max_n, mixed) gives its size for a call
 * (mixed = 1: dsposv); blasfeo_dposv_worksize(batch) is the size when every
 * system fits a shared-memory kernel (dsposv with n <= 256, dposv with
 * n <= 128); larger plain systems also need per-CTA factor slots. */
size_t blasfeo_dposv_worksize(int batch);
size_t blasfeo_dposv_worksize_n(int batch, int max_n, int mixed);
int blasfeo_dposv_l_vbatch(int batch, const int *n, int max_n, const struct blasfeo_dmat *sA,
	const struct blasfeo_dvec *sb, const struct blasfeo_dvec *sx, int *info,
	void *work, size_t work_bytes, void *stream);
int blasfeo_dsposv_l_vbatch(int batch, const int *n, int max_n, const struct blasfeo_dmat *sA,
	const struct blasfeo_dvec *sb, const struct blasfeo_dvec *sx, int max_iter, double tol,
	int *iters, double *berr, int *info, void *work, size_t work_bytes, void *stream);

/* Engine of blasfeo_dsposv_l_vbatch for systems with n <= 256 (per calling
 * host thread; larger systems always take the SIMT/global-memory kernels):
 *   SIMT:   FP32 Cholesky with FP32 FMA trailing updates in shared memory;
 *   TENSOR: trailing matrix in tensor memory, rank-16 trailing updates as
 *           3xTF32 tcgen05.mma with FP32 accumulation (same FP64 diagonal
 *           blocks, residual and refinement).
 * DEFAULT is the engine the library measured fastest on the uneven-size
 * workload.  set returns BLASFEO_B200_EINVAL for an unknown engine. */
#define BLASFEO_B200_POSV_DEFAULT 0
#define BLASFEO_B200_POSV_SIMT 1
#define BLASFEO_B200_POSV_TENSOR 2
int blasfeo_b200_set_posv_engine(int engine);
int blasfeo_b200_get_posv_engine(void);

/* Fused per-instance chain on a uniform batch (m = 16, 1 <= k <= 64; all
 * slabs from blasfeo_create_dmat_batch, zero offsets), replacing the sequence
 * blasfeo_dsyrk_ln (d_blas3_lib4.c:5400) + blasfeo_ddiare + blasfeo_dpotrf_l
 * (d_lapack_lib4.c:918) + blasfeo_dtrsm_rltn (d_blas3_lib4.c:4123) +
 * blasfeo_dgemm_nt (d_blas3_lib4.c:727):
 *   S = A A^T + shift*I,  L = chol(S) (lower, inverse diagonal in L's dA),
 *   X = R L^{-T},  D = C - X G^T.
 * One launch; info[b] as for dpotrf_l (-3: a bulk copy timed out). */
int blasfeo_dsyrk_dpotrf_dtrsm_dgemm_batch(int batch, int m, int k, double shift, struct blasfeo_dmat_batch *sA,
	struct blasfeo_dmat_batch *sR, struct blasfeo_dmat_batch *sC, struct blasfeo_dmat_batch *sG,
	struct blasfeo_dmat_batch *sL, struct blasfeo_dmat_batch *sX, struct blasfeo_dmat_batch *sD, int *info,
	void *stream);

/* Batched Riccati factorization (LQR backward pass), the recursion of
 * examples/example_d_riccati_recursion.c:115-143 (blasfeo_dpotrf_l, then per
 * stage blasfeo_dtrmm_rlnn + blasfeo_dsyrk_dpotrf_ln) for `batch` independent
 * problems with horizon N, nx states, nu inputs, nu + nx <= 16, in one launch.
 * Slabs (zero offsets): sBAbt batch*N instances of 16 x nx (problem b, stage k
 * at b*N + k; rows 0..nu-1 = B_k^T, rows nu.. = A_k^T), sRSQ and sL
 * batch*(N+1) instances of 16 x 16 (problem b, stage k at b*(N+1) + k; stage N
 * holds Q_N / L_N in its top-left nx x nx block).  Outputs: L_k (lower
 * triangle) and its inverse diagonal in sL's dA; info[b] = 16*(N-k) + j + 1
 * for the first non-positive pivot j of stage k, -3 on a copy timeout. */
int blasfeo_dric_trf_batch(int batch, int N, int nx, int nu, struct blasfeo_dmat_batch *sBAbt,
	struct blasfeo_dmat_batch *sRSQ, struct blasfeo_dmat_batch *sL, int *info, void *stream);
int blasfeo_sric_trf_batch(int batch, int N, int nx, int nu, struct blasfeo_smat_batch *sBAbt,
	struct blasfeo_smat_batch *sRSQ, struct blasfeo_smat_batch *sL, int *info, void *stream);

/* Batched Riccati solve (no reference counterpart for the batch; per problem
 * the sequence d_back_ric_trs_libstr of examples/example_d_riccati_recursion.c:203-270:
 * blasfeo_dtrmv_ltn / dtrmv_lnn / dgemv_n / dtrsv_lnn_mn backward, dtrsv_ltn_mn /
 * dgemv_t / dtrmv_ltn / dtrmv_lnn forward) on the factors of
 * blasfeo_dric_trf_batch: the LQ problem
 *   min sum_k 1/2 [u;x]_k^T RSQ_k [u;x]_k + rq_k^T [u;x]_k + 1/2 x_N^T Q_N x_N + q_N^T x_N,
 *   x_{k+1} = BAbt_k^T [u;x]_k + b_k  (x_0 free).
 * Vectors are strided arrays of doubles: b_k of problem p at b + sb*(p*N + k)
 * (nx entries), rq_k at rq + srq*(p*(N+1) + k) (nu + nx entries; stage N: nx),
 * ux_k = [u_k; x_k] at ux + sux*(p*(N+1) + k) (stage N: x_N), pi_k (the
 * dynamics multipliers) at pi + spi*(p*N + k).  sBAbt, sL as for
 * blasfeo_dric_trf_batch.  N >= 1, nu + nx <= 16. */
int blasfeo_dric_trs_batch(int batch, int N, int nx, int nu, struct blasfeo_dmat_batch *sBAbt,
	struct blasfeo_dmat_batch *sL, const double *b, long long sb, const double *rq, long long srq, double *ux,
	long long sux, double *pi, long long spi, void *stream);
/* Feedback gains K_k = -(R + B^T P B)^{-1} (S + B^T P A) = -Luu^{-T} Lxu^T of
 * every stage k < N from the factors L_k = [[Luu, 0], [Lxu, Lxx]] of
 * blasfeo_dric_trf_batch (u_k = K_k x_k for the homogeneous problem): sK
 * holds batch*N instances of nu x nx (problem p, stage k at p*N + k). */
int blasfeo_dric_gains_batch(int batch, int N, int nx, int nu, struct blasfeo_dmat_batch *sL,
	struct blasfeo_dmat_batch *sK, void *stream);
/* Mixed-precision LQ solve: the Riccati factorization in FP32
 * (blasfeo_sric_trf_batch on FP32 copies of BAbt_k and RSQ_k), then iterative
 * refinement in FP64 on the KKT residual
 *   RSQ_k ux_k + rq_k + BAbt_k pi_k - [0; pi_{k-1}],  Q_N x_N + q_N - pi_{N-1},
 *   BAbt_k^T ux_k + b_k - x_{k+1}
 * with corrections from the FP32 factors (the solve of blasfeo_dric_trs_batch),
 * until ||residual||_inf <= tol * ||(rq, b)||_inf or max_iter corrections.
 * Arguments as blasfeo_dric_trs_batch plus sRSQ (FP64, as for the
 * factorization); iters[p], res[p] (relative residual) and info[p] (device,
 * may be NULL): info = the factorization's pivot report, else 0, or -1 when
 * refinement did not reach tol.  work: blasfeo_dsric_sv_worksize(batch, N, nx)
 * bytes of device memory, or NULL for the library workspace. */
size_t blasfeo_dsric_sv_worksize(int batch, int N, int nx);
int blasfeo_dsric_sv_batch(int batch, int N, int nx, int nu, struct blasfeo_dmat_batch *sBAbt,
	struct blasfeo_dmat_batch *sRSQ, const double *b, long long sb, const double *rq, long long srq, double *ux,
	long long sux, double *pi, long long spi, int max_iter, double tol, int *iters, double *res, int *info,
	void *work, size_t work_bytes, void *stream);

/* Same as blasfeo_dsposv_l_vbatch, for callers whose matrices, vectors, sizes
 * and descriptors live in mapped (cudaHostAlloc / cudaHostRegister) host
 * memory: the kernels read the lower triangles straight over the host link
 * (only the lower triangle crosses it) and keep a per-CTA FP64 copy in device
 * memory for the refinement residuals; x is written back to host memory. */
int blasfeo_dsposv_l_vbatch_mapped(int batch, const int *n, int max_n, const struct blasfeo_dmat *sA,
	const struct blasfeo_dvec *sb, const struct blasfeo_dvec *sx, int max_iter, double tol,
	int *iters, double *berr, int *info, void *work, size_t work_bytes, void *stream);

/* Learned cost model kernels (no reference counterpart): an MLP
 * nin -> hidden -> hidden -> hidden -> 1 (ReLU, FP32), parameters in one flat
 * device array of blasfeo_b200_mlp_param_count(nin, hidden) floats (W1, b1,
 * W2, b2, W3, b3, W4, b4; y = x W + b).  work: device buffer of
 * blasfeo_b200_mlp_work_bytes(hidden, batch) bytes.  param_count returns -1
 * for nin <= 0 or hidden <= 0. */
int blasfeo_b200_mlp_param_count(int nin, int hidden);
size_t blasfeo_b200_mlp_work_bytes(int hidden, int batch);
int blasfeo_b200_mlp_forward(int nin, int hidden, const float *params, int batch, const float *X, float *y,
	float *work, void *stream);
int blasfeo_b200_mlp_grad(int nin, int hidden, const float *params, int batch, const float *X, const float *target,
	float *grads, float *loss, float *work, void *stream);
int blasfeo_b200_mlp_adam(int nparams, float *params, const float *grads, float *m, float *v, int step, float lr,
	void *stream);

/* Allocation-free variant of blasfeo_dsposv_l_vbatch (no counterpart in the
 * reference, which has no batched or GPU solver).  For callers that must not
 * allocate device memory while they run (embedded and real-time solvers that
 * fix their memory at start-up, or code that cannot afford the device-wide
 * synchronisation of cudaMalloc) and that do not pass a workspace: the scratch
 * is a static device array owned by the library (blasfeo_dsposv_noalloc_scratch_bytes()
 * bytes, resident on every GPU that uses the library until the process exits).
 * At most BLASFEO_B200_NOALLOC_MAX_BATCH systems per call and n <= 256, else
 * BLASFEO_B200_ENOTSUP.  All calls share the array: calls that overlap on the
 * GPU race and must be serialised by the caller.  The first call on a device
 * looks up the array's device address and caches it; make that first call
 * before any stream capture.  Under the CUDA driver's lazy module loading the
 * first launch of each kernel (so the first call of each solver engine) may
 * map memory for the kernel's code; a caller that must see no change in
 * device memory at all makes one call per engine at start-up. */
#define BLASFEO_B200_NOALLOC_MAX_BATCH 65536
size_t blasfeo_dsposv_noalloc_scratch_bytes(void);
int blasfeo_dsposv_l_vbatch_noalloc(int batch, const int *n, int max_n, const struct blasfeo_dmat *sA,
	const struct blasfeo_dvec *sb, const struct blasfeo_dvec *sx, int max_iter, double tol,
	int *iters, double *berr, int *info, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* BLASFEO_B200_H_ */
