// Batch-interleaved panel layout for uniform batches of small matrices.
//
// The instances of a batch are taken in groups of IL = 16.  Inside a group
// every element slot of the lib4 panel layout (include/blasfeo_common.h:112:
// element (i,j) at e = (i - i%4)*cn + 4j + i%4, then the inverse diagonal at
// e = pm*cn + k) holds the IL instances' values side by side:
//   value of instance b at mem[(b / IL) * gstride + e * IL + b % IL],
// gstride = IL * (pm*cn + dA slots), the slab rounded to 64 bytes per group.
// Kernels that give instance b to lanes of one warp then read one element of
// 16 instances as one contiguous 128-byte (FP64) run, whatever the element:
// every load is coalesced and vectorisable, with no staging in shared memory.
// The back-to-back slab (struct blasfeo_dmat_batch) keeps each instance
// contiguous instead, which suits kernels that give an instance to a warp and
// move it with one bulk copy.
//
// Here: layout, conversions from and to the back-to-back slab, and the
// Cholesky factorization (potrf_l, the reference's blasfeo_dpotrf_l,
// blasfeo_hp_pm/d_lapack_lib4.c:918) with a lane pair per instance for
// n <= 16: the pair holds the lower triangle in FP64 registers, even rows on
// one lane and odd rows on the other (at most 72 doubles each), pivots by the
// reference's rule (kernel/generic/kernel_dgemm_4x4_lib4.c:5700-5710: c > 0 ->
// sqrt(c) and its reciprocal, else 0 and 0), the column of each pivot passed
// to the partner by shuffles.  16 instances per warp.
#include "common.cuh"
#include "quad.cuh"

namespace {

constexpr int IL = 16;

struct IlGeom {
	int pm, cn, dl;
	long long slots, gstride;
};

__host__ __device__ inline IlGeom il_geom(int m, int n) {
	IlGeom g;
	g.pm = (m + 3) / 4 * 4;
	g.cn = (n + 3) / 4 * 4;
	const int mn = m < n ? m : n;
	g.dl = (mn + 15) / 16 * 16;
	g.slots = (long long)g.pm * g.cn + g.dl;
	g.gstride = (g.slots * IL + 7) / 8 * 8;  // 64-byte aligned groups (FP64)
	return g;
}

__device__ __forceinline__ long long pm_el(int i, int j, int cn) { return (long long)(i & ~3) * cn + 4 * j + (i & 3); }

// back-to-back slab <-> interleaved: one thread per (instance, slot), the
// interleaved side written / read in runs of IL consecutive instances
__global__ void k_to_il(long long total, int slots, const double *__restrict__ src, long long sstride,
                        double *__restrict__ dst, long long gstride) {
	for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
	     t += (long long)gridDim.x * blockDim.x) {
		const long long g = t / ((long long)slots * IL);
		const long long r = t % ((long long)slots * IL);
		const int e = (int)(r / IL), l = (int)(r % IL);
		const long long b = g * IL + l;
		dst[g * gstride + r] = src[b * sstride + e];
	}
}
__global__ void k_from_il(long long total, int slots, const double *__restrict__ src, long long gstride,
                          double *__restrict__ dst, long long dstride) {
	for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
	     t += (long long)gridDim.x * blockDim.x) {
		const long long g = t / ((long long)slots * IL);
		const long long r = t % ((long long)slots * IL);
		const int e = (int)(r / IL), l = (int)(r % IL);
		const long long b = g * IL + l;
		dst[b * dstride + e] = src[g * gstride + r];
	}
}

// Cholesky of n <= 16 per group of G lanes (quad::GCol): lane o of a group
// takes rows o + G s of instance (32 / G) * (global warp) + (lane / G); G = 2
// is a lane pair (8 rows per lane, 72 doubles of the lower triangle), G = 4 a
// quad (4 rows, 40 doubles).  Rows and columns >= n factor as an identity
// block.
#ifndef POTRF_IL_G
#define POTRF_IL_G 2
#endif
template <int G>
__global__ void __launch_bounds__(256, (G >= 4) ? 2 : 1) k_dpotrf_il(int batch, int n, const double *__restrict__ C, double *D,
                                                   long long gstride, int cn, int pmcn, int *info) {
	constexpr int P = 32 / G, R = 16 / G;
	const int lane = threadIdx.x & 31;
	const int o = lane % G, t = lane / G;
	const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	const long long b0 = gw * P;
	if (b0 >= batch) return;  // a whole warp past the batch (no block barrier follows)
	const long long b = b0 + t;
	const bool act = b < batch;
	const double *cg = C + (b0 / IL) * gstride + (b0 % IL) + t;
	double *dg = D + (b0 / IL) * gstride + (b0 % IL) + t;
	double a[R][16];
#pragma unroll
	for (int s = 0; s < R; s++)
#pragma unroll
		for (int j = 0; j < 16; j++) {
			const int i = o + G * s;
			double v = 0.0;
			if (j <= G * s + G - 1) {
				if (act && i < n && j < n && j <= i)
					v = cg[pm_el(i, j, cn) * IL];
				else if (i == j)
					v = 1.0;  // padding rows and columns factor to the identity
			}
			a[s][j] = v;
		}
	int bad = 0;
	quad::GCol<G, 0, false>::run(a, o, lane, n, nullptr, dg + (long long)pmcn * IL, act, bad);
	if (act) {
#pragma unroll
		for (int s = 0; s < R; s++)
#pragma unroll
			for (int j = 0; j < 16; j++) {
				const int i = o + G * s;
				if (j <= G * s + G - 1 && i < n && j <= i) dg[pm_el(i, j, cn) * IL] = a[s][j];
			}
		if (o == 0 && info) info[b] = bad;
	}
}

// host column-major batch (staged densely: instance b, element (i, j) at
// stage[b m n + j m + i]) <-> interleaved slab, one thread per (group, slot,
// lane) so that the slab side moves in runs of IL consecutive instances
template <bool TO_IL>
__global__ void k_cm_il(long long total, int batch, int m, int n, double *stage, double *il, long long gstride,
                        int cn) {
	const long long mn = (long long)m * n;
	for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
	     t += (long long)gridDim.x * blockDim.x) {
		const long long g = t / (mn * IL);
		const long long r = t % (mn * IL);
		const int el = (int)(r / IL), l = (int)(r % IL);
		const long long b = g * IL + l;
		if (b >= batch) continue;
		const int i = el % m, j = el / m;
		double *slot = il + g * gstride + pm_el(i, j, cn) * IL + l;
		double *dense = stage + b * mn + (long long)j * m + i;
		if (TO_IL)
			*slot = *dense;
		else
			*dense = *slot;
	}
}

inline int grid_for(long long total, int threads) {
	long long g = (total + threads - 1) / threads;
	const long long cap = (long long)bf::num_sms() * 16;
	return (int)(g < 1 ? 1 : (g > cap ? cap : g));
}

}  // namespace

extern "C" {

size_t blasfeo_memsize_dmat_batch_il(int m, int n, int batch) {
	if (m <= 0 || n <= 0 || batch <= 0) return 0;
	const IlGeom g = il_geom(m, n);
	return (size_t)((batch + IL - 1) / IL) * (size_t)g.gstride * sizeof(double);
}

void blasfeo_create_dmat_batch_il(int m, int n, int batch, struct blasfeo_dmat_batch_il *sA, void *memory) {
	const IlGeom g = il_geom(m, n);
	sA->mem = (double *)memory;
	sA->m = m;
	sA->n = n;
	sA->pm = g.pm;
	sA->cn = g.cn;
	sA->batch = batch;
	sA->il = IL;
	sA->gstride = g.gstride;
	sA->memsize = blasfeo_memsize_dmat_batch_il(m, n, batch);
}

int blasfeo_dmat_batch_to_il(const struct blasfeo_dmat_batch *src, struct blasfeo_dmat_batch_il *dst, void *stream) {
	if (!src || !dst || !src->mem || !dst->mem || src->m != dst->m || src->n != dst->n || src->batch < dst->batch)
		return BLASFEO_B200_EINVAL;
	if (dst->batch == 0) return BLASFEO_B200_OK;
	const IlGeom g = il_geom(dst->m, dst->n);
	// whole groups by the kernel, a partial last group instance by instance
	// (the slots of its missing instances are left as they are)
	const long long total = (long long)((dst->batch + IL - 1) / IL) * g.slots * IL;
	const long long full = (long long)(dst->batch / IL) * g.slots * IL;
	if (full > 0)
		k_to_il<<<grid_for(full, 256), 256, 0, (cudaStream_t)stream>>>(full, (int)g.slots, src->pA, src->stride,
		                                                               dst->mem, dst->gstride);
	if (total > full) {
		for (int b = (int)(dst->batch / IL) * IL; b < dst->batch; b++)
			cudaMemcpy2DAsync(dst->mem + (long long)(b / IL) * dst->gstride + b % IL, IL * sizeof(double),
			                  src->pA + (long long)b * src->stride, sizeof(double), sizeof(double), g.slots,
			                  cudaMemcpyDeviceToDevice, (cudaStream_t)stream);
	}
	return bf::check_launch();
}

int blasfeo_dmat_batch_from_il(const struct blasfeo_dmat_batch_il *src, struct blasfeo_dmat_batch *dst, void *stream) {
	if (!src || !dst || !src->mem || !dst->mem || src->m != dst->m || src->n != dst->n || dst->batch < src->batch)
		return BLASFEO_B200_EINVAL;
	if (src->batch == 0) return BLASFEO_B200_OK;
	const IlGeom g = il_geom(src->m, src->n);
	const long long full = (long long)(src->batch / IL) * g.slots * IL;
	if (full > 0)
		k_from_il<<<grid_for(full, 256), 256, 0, (cudaStream_t)stream>>>(full, (int)g.slots, src->mem, src->gstride,
		                                                                 dst->pA, dst->stride);
	for (int b = (int)(src->batch / IL) * IL; b < src->batch; b++)
		cudaMemcpy2DAsync(dst->pA + (long long)b * dst->stride, sizeof(double),
		                  src->mem + (long long)(b / IL) * src->gstride + b % IL, IL * sizeof(double),
		                  sizeof(double), g.slots, cudaMemcpyDeviceToDevice, (cudaStream_t)stream);
	return bf::check_launch();
}

// host column-major batch <-> interleaved slab: one host copy through a
// library-owned staging buffer and one conversion kernel; synchronous with
// `stream` on return (the staging buffer is reused by the next call)
static int cm_il(int batch, int m, int n, double *A, int lda, long long strideA, const struct blasfeo_dmat_batch_il *sB,
                 cudaStream_t s, bool to_il) {
	if (batch < 0 || m < 0 || n < 0 || !sB || !sB->mem || (batch > 0 && m > 0 && n > 0 && !A))
		return BLASFEO_B200_EINVAL;
	if (batch == 0 || m == 0 || n == 0) return BLASFEO_B200_OK;
	if (lda < m || strideA < (long long)lda * (n - 1) + m || m > sB->m || n > sB->n || batch > sB->batch)
		return BLASFEO_B200_EINVAL;
	const size_t per = (size_t)m * n;
	double *stage = (double *)bf::workspace(per * batch * sizeof(double), s);
	if (!stage) return BLASFEO_B200_ENOMEM;
	const bool packed = strideA == (long long)lda * n;
	const long long total = (long long)((batch + IL - 1) / IL) * (long long)per * IL;
	if (to_il) {
		if (packed) {
			if (cudaMemcpy2DAsync(stage, m * sizeof(double), A, (size_t)lda * sizeof(double), m * sizeof(double),
			                      (size_t)n * batch, cudaMemcpyHostToDevice, s) != cudaSuccess)
				return BLASFEO_B200_ECUDA;
		} else {
			for (int b = 0; b < batch; b++)
				if (cudaMemcpy2DAsync(stage + per * b, m * sizeof(double), A + strideA * b, (size_t)lda * sizeof(double),
				                      m * sizeof(double), n, cudaMemcpyHostToDevice, s) != cudaSuccess)
					return BLASFEO_B200_ECUDA;
		}
		k_cm_il<true><<<grid_for(total, 256), 256, 0, s>>>(total, batch, m, n, stage, sB->mem, sB->gstride, sB->cn);
		if (bf::check_launch()) return BLASFEO_B200_ECUDA;
	} else {
		k_cm_il<false><<<grid_for(total, 256), 256, 0, s>>>(total, batch, m, n, stage, sB->mem, sB->gstride, sB->cn);
		if (bf::check_launch()) return BLASFEO_B200_ECUDA;
		if (packed) {
			if (cudaMemcpy2DAsync(A, (size_t)lda * sizeof(double), stage, m * sizeof(double), m * sizeof(double),
			                      (size_t)n * batch, cudaMemcpyDeviceToHost, s) != cudaSuccess)
				return BLASFEO_B200_ECUDA;
		} else {
			for (int b = 0; b < batch; b++)
				if (cudaMemcpy2DAsync(A + strideA * b, (size_t)lda * sizeof(double), stage + per * b, m * sizeof(double),
				                      m * sizeof(double), n, cudaMemcpyDeviceToHost, s) != cudaSuccess)
					return BLASFEO_B200_ECUDA;
		}
	}
	return cudaStreamSynchronize(s) == cudaSuccess ? BLASFEO_B200_OK : BLASFEO_B200_ECUDA;
}

int blasfeo_pack_dmat_batch_il(int batch, int m, int n, const double *A, int lda, long long strideA,
                               struct blasfeo_dmat_batch_il *sB, void *stream) {
	return cm_il(batch, m, n, (double *)A, lda, strideA, sB, (cudaStream_t)stream, true);
}

int blasfeo_unpack_dmat_batch_il(int batch, int m, int n, const struct blasfeo_dmat_batch_il *sB, double *A, int lda,
                                 long long strideA, void *stream) {
	return cm_il(batch, m, n, A, lda, strideA, sB, (cudaStream_t)stream, false);
}

int blasfeo_dpotrf_l_batch_il(int batch, int m, struct blasfeo_dmat_batch_il *sC, struct blasfeo_dmat_batch_il *sD,
                              int *info, void *stream) {
	if (batch < 0 || m < 0 || !sC || !sD || !sC->mem || !sD->mem) return BLASFEO_B200_EINVAL;
	if (batch == 0 || m == 0) return BLASFEO_B200_OK;
	if (m > 16) return BLASFEO_B200_ENOTSUP;
	if (sC->m < m || sC->n < m || sD->m < m || sD->n < m || sC->batch < batch || sD->batch < batch ||
	    sC->pm != sD->pm || sC->cn != sD->cn || sC->gstride != sD->gstride)
		return BLASFEO_B200_EINVAL;
	constexpr int G = POTRF_IL_G, P = 32 / G;
	const long long warps = (batch + P - 1) / P;
	const int threads = 256;
	const long long blocks = (warps * 32 + threads - 1) / threads;
	k_dpotrf_il<G><<<(unsigned)blocks, threads, 0, (cudaStream_t)stream>>>(batch, m, sC->mem, sD->mem, sC->gstride,
	                                                                        sC->cn, sC->pm * sC->cn, info);
	return bf::check_launch();
}

}  // extern "C"
