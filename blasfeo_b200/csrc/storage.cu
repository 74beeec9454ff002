// Storage: descriptor sizing/carving (auxiliary/d_aux_lib4.c:1519-1600), host
// column-major <-> device panel-major transfers (auxiliary/d_aux_lib4.c:1607,
// 2238) and the device auxiliaries dgecp / ddiare / drowsw
// (include/blasfeo_d_aux.h:115,141,162).
//
// pack: the host block is copied with one cudaMemcpy2DAsync into a staging
// area of the library workspace (column-major, leading dimension m), then one
// kernel scatters it into the panel-major destination (any row/col offset).
// unpack is the mirror image.  Both are ordered on the current stream and, in
// synchronous mode, complete before returning.
#include "common.cuh"

namespace {

// memsize/create: pm = ceil(m/4)*4, cn = ceil(n/4)*4, dA follows pA with
// min(m,n) rounded up to 16 elements, total rounded up to 64 bytes.
template <typename T>
size_t memsize_mat(int m, int n) {
	int pm = (m + 3) / 4 * 4;
	int cn = (n + 3) / 4 * 4;
	int mn = m < n ? m : n;
	int dl = (mn + 15) / 16 * 16;
	size_t sz = ((size_t)pm * cn + dl) * sizeof(T);
	return (sz + 63) / 64 * 64;
}

template <typename T, typename S>
void create_mat(int m, int n, S *sA, void *memory) {
	int pm = (m + 3) / 4 * 4;
	int cn = (n + 3) / 4 * 4;
	sA->mem = (T *)memory;
	sA->pA = (T *)memory;
	sA->dA = (T *)memory + (size_t)pm * cn;
	sA->m = m;
	sA->n = n;
	sA->pm = pm;
	sA->cn = cn;
	sA->use_dA = 0;
	sA->memsize = (int)memsize_mat<T>(m, n);
}

template <typename T, typename S>
void create_vec(int m, S *sa, void *memory) {
	sa->mem = (T *)memory;
	sa->pa = (T *)memory;
	sa->m = m;
	sa->pm = (m + 3) / 4 * 4;
	sa->memsize = sa->pm * (int)sizeof(T);
}

template <typename T>
__global__ void k_scatter_pm(int m, int n, const T *__restrict__ src, PMat<T> dst) {
	// one thread per element, column-major source: consecutive threads read
	// consecutive source rows and write 4-element panel runs
	long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
	long long tot = (long long)m * n;
	if (idx >= tot) return;
	int i = (int)(idx % m), j = (int)(idx / m);
	dst.at(i, j) = src[idx];
}

template <typename T>
__global__ void k_gather_pm(int m, int n, PMat<T> src, T *__restrict__ dst) {
	long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
	long long tot = (long long)m * n;
	if (idx >= tot) return;
	int i = (int)(idx % m), j = (int)(idx / m);
	dst[idx] = src.at(i, j);
}

// Transposed scatter/gather (pack_tran / unpack_tran, auxiliary/d_aux_lib4.c:
// 2086, 2360): the staged host block is m x n column-major; element (i, j)
// goes to / comes from panel-major element (j, i).
template <typename T>
__global__ void k_scatter_pm_tran(int m, int n, const T *__restrict__ src, PMat<T> dst) {
	long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
	long long tot = (long long)m * n;
	if (idx >= tot) return;
	int i = (int)(idx % m), j = (int)(idx / m);
	dst.at(j, i) = src[idx];
}
template <typename T>
__global__ void k_gather_pm_tran(int m, int n, PMat<T> src, T *__restrict__ dst) {
	// dst is n x m column-major (ld n): dst[j + n*i] = src(i, j)
	long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
	long long tot = (long long)m * n;
	if (idx >= tot) return;
	int j = (int)(idx % n), i = (int)(idx / n);
	dst[idx] = src.at(i, j);
}

// Batched layout conversion between a dense column-major staging block
// (instance b at b*m*n, ld m) and the uniform-batch slab: one thread per
// element, consecutive threads on consecutive rows of one column.
template <typename T, bool TO_SLAB>
__global__ void k_convert_batch(int batch, int m, int n, T *stage, MatArg<T> slab) {
	long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
	const long long per = (long long)m * n;
	if (idx >= per * batch) return;
	const int b = (int)(idx / per);
	const long long e = idx % per;
	const int i = (int)(e % m), j = (int)(e / m);
	const PMat<T> d = slab.get(b);
	if (TO_SLAB)
		d.at(i, j) = stage[idx];
	else
		stage[idx] = d.at(i, j);
}

template <typename T>
__global__ void k_gecp(int m, int n, PMat<T> a, PMat<T> b) {
	long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
	if (idx >= (long long)m * n) return;
	int i = (int)(idx % m), j = (int)(idx / m);
	b.at(i, j) = a.at(i, j);
}

template <typename T>
__global__ void k_diare(int kmax, T alpha, PMat<T> a) {
	int l = blockIdx.x * blockDim.x + threadIdx.x;
	if (l < kmax) a.at(l, l) += alpha;
}

template <typename T>
__global__ void k_rowsw(int kmax, PMat<T> a, PMat<T> c) {
	int l = blockIdx.x * blockDim.x + threadIdx.x;
	if (l >= kmax) return;
	T t = a.at(0, l);
	a.at(0, l) = c.at(0, l);
	c.at(0, l) = t;
}

template <typename T, typename S>
PMat<T> pm_of(S *s, int ri, int cj) {
	PMat<T> p;
	p.p = s->pA;
	p.d = s->dA;
	p.cn = s->cn;
	p.ri = ri;
	p.cj = cj;
	return p;
}

template <typename T, typename S>
void pack_mat(int m, int n, const T *A, int lda, S *sA, int ai, int aj) {
	if (m <= 0 || n <= 0) return;
	if (!A || !sA || lda < m || ai < 0 || aj < 0 || ai + m > sA->m || aj + n > sA->n) {
		bf::set_error(BLASFEO_B200_EINVAL);
		return;
	}
	sA->use_dA = 0;
	cudaStream_t s = bf::cur_stream();
	size_t bytes = (size_t)m * n * sizeof(T);
	T *stage = (T *)bf::workspace(bytes, s);
	if (!stage) {
		bf::set_error(BLASFEO_B200_ENOMEM);
		return;
	}
	if (cudaMemcpy2DAsync(stage, m * sizeof(T), A, (size_t)lda * sizeof(T), m * sizeof(T), n,
	                      cudaMemcpyHostToDevice, s) != cudaSuccess) {
		bf::set_error(BLASFEO_B200_ECUDA);
		return;
	}
	long long tot = (long long)m * n;
	k_scatter_pm<T><<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(m, n, stage, pm_of<T>(sA, ai, aj));
	// the staging area is reused by the next call: always complete the copy
	if (bf::check_launch() == BLASFEO_B200_OK && cudaStreamSynchronize(s) != cudaSuccess)
		bf::set_error(BLASFEO_B200_ECUDA);
}

template <typename T, typename S>
void unpack_mat(int m, int n, S *sA, int ai, int aj, T *A, int lda) {
	if (m <= 0 || n <= 0) return;
	if (!A || !sA || lda < m || ai < 0 || aj < 0 || ai + m > sA->m || aj + n > sA->n) {
		bf::set_error(BLASFEO_B200_EINVAL);
		return;
	}
	cudaStream_t s = bf::cur_stream();
	size_t bytes = (size_t)m * n * sizeof(T);
	T *stage = (T *)bf::workspace(bytes, s);
	if (!stage) {
		bf::set_error(BLASFEO_B200_ENOMEM);
		return;
	}
	long long tot = (long long)m * n;
	k_gather_pm<T><<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(m, n, pm_of<T>(sA, ai, aj), stage);
	if (bf::check_launch() != BLASFEO_B200_OK) return;
	if (cudaMemcpy2DAsync(A, (size_t)lda * sizeof(T), stage, m * sizeof(T), m * sizeof(T), n,
	                      cudaMemcpyDeviceToHost, s) != cudaSuccess ||
	    cudaStreamSynchronize(s) != cudaSuccess)
		bf::set_error(BLASFEO_B200_ECUDA);
}

// sA(ai + i, aj + j) = A[j + lda*i] for i < n, j < m: sA's n x m block is the
// transpose of the m x n column-major A (auxiliary/d_aux_lib4.c:2086)
template <typename T, typename S>
void pack_tran_mat(int m, int n, const T *A, int lda, S *sA, int ai, int aj) {
	if (m <= 0 || n <= 0) return;
	if (!A || !sA || lda < m || ai < 0 || aj < 0 || ai + n > sA->m || aj + m > sA->n) {
		bf::set_error(BLASFEO_B200_EINVAL);
		return;
	}
	sA->use_dA = 0;
	cudaStream_t s = bf::cur_stream();
	T *stage = (T *)bf::workspace((size_t)m * n * sizeof(T), s);
	if (!stage) {
		bf::set_error(BLASFEO_B200_ENOMEM);
		return;
	}
	if (cudaMemcpy2DAsync(stage, m * sizeof(T), A, (size_t)lda * sizeof(T), m * sizeof(T), n,
	                      cudaMemcpyHostToDevice, s) != cudaSuccess) {
		bf::set_error(BLASFEO_B200_ECUDA);
		return;
	}
	long long tot = (long long)m * n;
	k_scatter_pm_tran<T><<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(m, n, stage, pm_of<T>(sA, ai, aj));
	if (bf::check_launch() == BLASFEO_B200_OK && cudaStreamSynchronize(s) != cudaSuccess)
		bf::set_error(BLASFEO_B200_ECUDA);
}

// A[j + lda*i] = sA(ai + i, aj + j) for i < m, j < n: A (n x m column-major) is
// the transpose of sA's m x n block (auxiliary/d_aux_lib4.c:2360)
template <typename T, typename S>
void unpack_tran_mat(int m, int n, S *sA, int ai, int aj, T *A, int lda) {
	if (m <= 0 || n <= 0) return;
	if (!A || !sA || lda < n || ai < 0 || aj < 0 || ai + m > sA->m || aj + n > sA->n) {
		bf::set_error(BLASFEO_B200_EINVAL);
		return;
	}
	cudaStream_t s = bf::cur_stream();
	T *stage = (T *)bf::workspace((size_t)m * n * sizeof(T), s);
	if (!stage) {
		bf::set_error(BLASFEO_B200_ENOMEM);
		return;
	}
	long long tot = (long long)m * n;
	k_gather_pm_tran<T><<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(m, n, pm_of<T>(sA, ai, aj), stage);
	if (bf::check_launch() != BLASFEO_B200_OK) return;
	if (cudaMemcpy2DAsync(A, (size_t)lda * sizeof(T), stage, n * sizeof(T), n * sizeof(T), m,
	                      cudaMemcpyDeviceToHost, s) != cudaSuccess ||
	    cudaStreamSynchronize(s) != cudaSuccess)
		bf::set_error(BLASFEO_B200_ECUDA);
}

// Batched host column-major <-> slab: instance b of the host array starts at
// A + b*strideA (column-major, ld lda).  One host<->device copy of all
// instances through the library staging buffer (a single 2-D copy when the
// instances are back to back, strideA == lda*n) and one conversion kernel;
// returns after the copies completed on `stream`.
template <typename T, typename B>
int convert_batch(int batch, int m, int n, T *A, int lda, long long strideA, B *sB, int bi, int bj, cudaStream_t s,
                  bool to_slab) {
	if (batch < 0 || m < 0 || n < 0 || !sB || (batch > 0 && m > 0 && n > 0 && !A)) return BLASFEO_B200_EINVAL;
	if (batch == 0 || m == 0 || n == 0) return BLASFEO_B200_OK;
	if (lda < m || strideA < (long long)lda * (n - 1) + m || bi < 0 || bj < 0 || bi + m > sB->m || bj + n > sB->n ||
	    batch > sB->batch)
		return BLASFEO_B200_EINVAL;
	const size_t per = (size_t)m * n;
	T *stage = (T *)bf::workspace(per * batch * sizeof(T), s);
	if (!stage) return BLASFEO_B200_ENOMEM;
	const MatArg<T> slab = batch_arg<T>(sB, bi, bj);
	const long long tot = (long long)per * batch;
	const unsigned grid = (unsigned)((tot + 255) / 256);
	const bool packed = strideA == (long long)lda * n;
	if (to_slab) {
		sB->use_dA = 0;
		if (packed) {
			if (cudaMemcpy2DAsync(stage, m * sizeof(T), A, (size_t)lda * sizeof(T), m * sizeof(T), (size_t)n * batch,
			                      cudaMemcpyHostToDevice, s) != cudaSuccess)
				return BLASFEO_B200_ECUDA;
		} else {
			for (int b = 0; b < batch; b++)
				if (cudaMemcpy2DAsync(stage + per * b, m * sizeof(T), A + strideA * b, (size_t)lda * sizeof(T),
				                      m * sizeof(T), n, cudaMemcpyHostToDevice, s) != cudaSuccess)
					return BLASFEO_B200_ECUDA;
		}
		k_convert_batch<T, true><<<grid, 256, 0, s>>>(batch, m, n, stage, slab);
		if (bf::check_launch()) return BLASFEO_B200_ECUDA;
	} else {
		k_convert_batch<T, false><<<grid, 256, 0, s>>>(batch, m, n, stage, slab);
		if (bf::check_launch()) return BLASFEO_B200_ECUDA;
		if (packed) {
			if (cudaMemcpy2DAsync(A, (size_t)lda * sizeof(T), stage, m * sizeof(T), m * sizeof(T), (size_t)n * batch,
			                      cudaMemcpyDeviceToHost, s) != cudaSuccess)
				return BLASFEO_B200_ECUDA;
		} else {
			for (int b = 0; b < batch; b++)
				if (cudaMemcpy2DAsync(A + strideA * b, (size_t)lda * sizeof(T), stage + per * b, m * sizeof(T),
				                      m * sizeof(T), n, cudaMemcpyDeviceToHost, s) != cudaSuccess)
					return BLASFEO_B200_ECUDA;
		}
	}
	// the staging buffer is reused by the next call: complete the copies
	return cudaStreamSynchronize(s) == cudaSuccess ? BLASFEO_B200_OK : BLASFEO_B200_ECUDA;
}

template <typename T, typename S>
void pack_vec(int m, const T *x, int xi, S *sa, int ai) {
	if (m <= 0) return;
	if (!x || !sa || ai < 0 || ai + m > sa->m) {
		bf::set_error(BLASFEO_B200_EINVAL);
		return;
	}
	cudaStream_t s = bf::cur_stream();
	if (cudaMemcpyAsync(sa->pa + ai, x + xi, m * sizeof(T), cudaMemcpyHostToDevice, s) != cudaSuccess ||
	    cudaStreamSynchronize(s) != cudaSuccess)
		bf::set_error(BLASFEO_B200_ECUDA);
}

template <typename T, typename S>
void unpack_vec(int m, S *sa, int ai, T *x, int xi) {
	if (m <= 0) return;
	if (!x || !sa || ai < 0 || ai + m > sa->m) {
		bf::set_error(BLASFEO_B200_EINVAL);
		return;
	}
	cudaStream_t s = bf::cur_stream();
	if (cudaMemcpyAsync(x + xi, sa->pa + ai, m * sizeof(T), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
	    cudaStreamSynchronize(s) != cudaSuccess)
		bf::set_error(BLASFEO_B200_ECUDA);
}

template <typename T, typename S>
void gecp(int m, int n, S *sA, int ai, int aj, S *sB, int bi, int bj) {
	if (m <= 0 || n <= 0) return;
	sB->use_dA = 0;
	long long tot = (long long)m * n;
	k_gecp<T><<<(unsigned)((tot + 255) / 256), 256, 0, bf::cur_stream()>>>(m, n, pm_of<T>(sA, ai, aj),
	                                                                        pm_of<T>(sB, bi, bj));
	bf::finish_single();
}

template <typename T, typename S>
void diare(int kmax, T alpha, S *sA, int ai, int aj) {
	if (kmax <= 0) return;
	sA->use_dA = 0;
	k_diare<T><<<cdiv(kmax, 256), 256, 0, bf::cur_stream()>>>(kmax, alpha, pm_of<T>(sA, ai, aj));
	bf::finish_single();
}

template <typename T, typename S>
void rowsw(int kmax, S *sA, int ai, int aj, S *sC, int ci, int cj) {
	if (kmax <= 0) return;
	sA->use_dA = 0;
	sC->use_dA = 0;
	k_rowsw<T><<<cdiv(kmax, 256), 256, 0, bf::cur_stream()>>>(kmax, pm_of<T>(sA, ai, aj), pm_of<T>(sC, ci, cj));
	bf::finish_single();
}

template <typename T, typename B>
void create_batch(int m, int n, int batch, B *sA, void *memory) {
	int pm = (m + 3) / 4 * 4;
	int cn = (n + 3) / 4 * 4;
	size_t per = memsize_mat<T>(m, n);
	sA->mem = (T *)memory;
	sA->pA = (T *)memory;
	sA->dA = (T *)memory + (size_t)pm * cn;
	sA->m = m;
	sA->n = n;
	sA->pm = pm;
	sA->cn = cn;
	sA->use_dA = 0;
	sA->batch = batch;
	sA->stride = (long long)(per / sizeof(T));
	sA->memsize = per * (size_t)batch;
}

template <typename T, typename B, typename S>
void batch_instance(B *sA, int b, S *out) {
	create_mat<T>(sA->m, sA->n, out, (void *)(sA->mem + sA->stride * b));
	out->use_dA = sA->use_dA;
}

}  // namespace

extern "C" {

size_t blasfeo_memsize_dmat(int m, int n) { return memsize_mat<double>(m, n); }
size_t blasfeo_memsize_diag_dmat(int m, int n) {
	int mn = m < n ? m : n;
	return (size_t)((mn + 15) / 16 * 16) * sizeof(double);
}
void blasfeo_create_dmat(int m, int n, struct blasfeo_dmat *sA, void *memory) { create_mat<double>(m, n, sA, memory); }
size_t blasfeo_memsize_dvec(int m) { return (size_t)((m + 3) / 4 * 4) * sizeof(double); }
void blasfeo_create_dvec(int m, struct blasfeo_dvec *sa, void *memory) { create_vec<double>(m, sa, memory); }
size_t blasfeo_memsize_smat(int m, int n) { return memsize_mat<float>(m, n); }
size_t blasfeo_memsize_diag_smat(int m, int n) {
	int mn = m < n ? m : n;
	return (size_t)((mn + 15) / 16 * 16) * sizeof(float);
}
void blasfeo_create_smat(int m, int n, struct blasfeo_smat *sA, void *memory) { create_mat<float>(m, n, sA, memory); }
size_t blasfeo_memsize_svec(int m) { return (size_t)((m + 3) / 4 * 4) * sizeof(float); }
void blasfeo_create_svec(int m, struct blasfeo_svec *sa, void *memory) { create_vec<float>(m, sa, memory); }

void blasfeo_pack_dmat(int m, int n, double *A, int lda, struct blasfeo_dmat *sA, int ai, int aj) { pack_mat<double>(m, n, A, lda, sA, ai, aj); }
void blasfeo_unpack_dmat(int m, int n, struct blasfeo_dmat *sA, int ai, int aj, double *A, int lda) { unpack_mat<double>(m, n, sA, ai, aj, A, lda); }
void blasfeo_pack_dvec(int m, double *x, int xi, struct blasfeo_dvec *sa, int ai) { pack_vec<double>(m, x, xi, sa, ai); }
void blasfeo_pack_tran_dmat(int m, int n, double *A, int lda, struct blasfeo_dmat *sA, int ai, int aj) {
	pack_tran_mat<double>(m, n, A, lda, sA, ai, aj);
}
void blasfeo_unpack_tran_dmat(int m, int n, struct blasfeo_dmat *sA, int ai, int aj, double *A, int lda) {
	unpack_tran_mat<double>(m, n, sA, ai, aj, A, lda);
}
void blasfeo_pack_tran_smat(int m, int n, float *A, int lda, struct blasfeo_smat *sA, int ai, int aj) {
	pack_tran_mat<float>(m, n, A, lda, sA, ai, aj);
}
void blasfeo_unpack_tran_smat(int m, int n, struct blasfeo_smat *sA, int ai, int aj, float *A, int lda) {
	unpack_tran_mat<float>(m, n, sA, ai, aj, A, lda);
}
int blasfeo_pack_dmat_batch(int batch, int m, int n, const double *A, int lda, long long strideA,
                            struct blasfeo_dmat_batch *sB, int bi, int bj, void *stream) {
	return convert_batch<double>(batch, m, n, (double *)A, lda, strideA, sB, bi, bj, (cudaStream_t)stream, true);
}
int blasfeo_unpack_dmat_batch(int batch, int m, int n, struct blasfeo_dmat_batch *sB, int bi, int bj, double *A,
                              int lda, long long strideA, void *stream) {
	return convert_batch<double>(batch, m, n, A, lda, strideA, sB, bi, bj, (cudaStream_t)stream, false);
}
int blasfeo_pack_smat_batch(int batch, int m, int n, const float *A, int lda, long long strideA,
                            struct blasfeo_smat_batch *sB, int bi, int bj, void *stream) {
	return convert_batch<float>(batch, m, n, (float *)A, lda, strideA, sB, bi, bj, (cudaStream_t)stream, true);
}
int blasfeo_unpack_smat_batch(int batch, int m, int n, struct blasfeo_smat_batch *sB, int bi, int bj, float *A,
                              int lda, long long strideA, void *stream) {
	return convert_batch<float>(batch, m, n, A, lda, strideA, sB, bi, bj, (cudaStream_t)stream, false);
}
void blasfeo_unpack_dvec(int m, struct blasfeo_dvec *sa, int ai, double *x, int xi) { unpack_vec<double>(m, sa, ai, x, xi); }
void blasfeo_pack_smat(int m, int n, float *A, int lda, struct blasfeo_smat *sA, int ai, int aj) { pack_mat<float>(m, n, A, lda, sA, ai, aj); }
void blasfeo_unpack_smat(int m, int n, struct blasfeo_smat *sA, int ai, int aj, float *A, int lda) { unpack_mat<float>(m, n, sA, ai, aj, A, lda); }
void blasfeo_pack_svec(int m, float *x, int xi, struct blasfeo_svec *sa, int ai) { pack_vec<float>(m, x, xi, sa, ai); }
void blasfeo_unpack_svec(int m, struct blasfeo_svec *sa, int ai, float *x, int xi) { unpack_vec<float>(m, sa, ai, x, xi); }

void blasfeo_dgecp(int m, int n, struct blasfeo_dmat *sA, int ai, int aj, struct blasfeo_dmat *sB, int bi, int bj) { gecp<double>(m, n, sA, ai, aj, sB, bi, bj); }
void blasfeo_ddiare(int kmax, double alpha, struct blasfeo_dmat *sA, int ai, int aj) { diare<double>(kmax, alpha, sA, ai, aj); }
void blasfeo_drowsw(int kmax, struct blasfeo_dmat *sA, int ai, int aj, struct blasfeo_dmat *sC, int ci, int cj) { rowsw<double>(kmax, sA, ai, aj, sC, ci, cj); }
void blasfeo_sgecp(int m, int n, struct blasfeo_smat *sA, int ai, int aj, struct blasfeo_smat *sB, int bi, int bj) { gecp<float>(m, n, sA, ai, aj, sB, bi, bj); }
void blasfeo_sdiare(int kmax, float alpha, struct blasfeo_smat *sA, int ai, int aj) { diare<float>(kmax, alpha, sA, ai, aj); }
void blasfeo_srowsw(int kmax, struct blasfeo_smat *sA, int ai, int aj, struct blasfeo_smat *sC, int ci, int cj) { rowsw<float>(kmax, sA, ai, aj, sC, ci, cj); }

size_t blasfeo_memsize_dmat_batch(int m, int n, int batch) { return memsize_mat<double>(m, n) * (size_t)batch; }
void blasfeo_create_dmat_batch(int m, int n, int batch, struct blasfeo_dmat_batch *sA, void *memory) { create_batch<double>(m, n, batch, sA, memory); }
void blasfeo_dmat_batch_instance(struct blasfeo_dmat_batch *sA, int b, struct blasfeo_dmat *out) { batch_instance<double>(sA, b, out); }
size_t blasfeo_memsize_smat_batch(int m, int n, int batch) { return memsize_mat<float>(m, n) * (size_t)batch; }
void blasfeo_create_smat_batch(int m, int n, int batch, struct blasfeo_smat_batch *sA, void *memory) { create_batch<float>(m, n, batch, sA, memory); }
void blasfeo_smat_batch_instance(struct blasfeo_smat_batch *sA, int b, struct blasfeo_smat *out) { batch_instance<float>(sA, b, out); }

}  // extern "C"
