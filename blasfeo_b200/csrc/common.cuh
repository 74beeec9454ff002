// Shared device/host helpers of libblasfeo_b200.
//
// Device layout (both precisions): panel-major with panel size 4, exactly the
// BLASFEO lib4 layout (include/blasfeo_common.h:112): element (i,j) of a matrix
// with panel stride cn lives at pA[(i - i%4)*cn + 4*j + i%4].  A 4-row panel is
// one contiguous run of 4*cn elements, so a whole matrix, a panel, or a 4x4
// tile are contiguous -- the property the kernels use for coalesced and bulk
// (TMA) copies.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stddef.h>

#include "../../include/blasfeo_b200.h"

#define BF_PS 4

// ---------------------------------------------------------------------------
// host-side library state (state.cu)
// ---------------------------------------------------------------------------
namespace bf {

void set_error(int status);
int check_launch();                       // cudaGetLastError -> status (and records it)
cudaStream_t cur_stream();
bool sync_mode();
int finish_single();                      // launch check + optional stream sync, records error
// library-owned device workspace (per device, grows; never shrinks)
void *workspace(size_t bytes, cudaStream_t s);
// a second buffer of the same kind, for the column-major routines' staging
// (they call panel-major routines that use the first one)
void *workspace_cm(size_t bytes, cudaStream_t s);
int num_sms();
size_t max_smem_optin();
int posv_engine();                        // engine of the mixed SPD solver (BLASFEO_B200_POSV_*)
unsigned int wait_limit();                // polls of a bounded mbarrier wait (blasfeo_b200_set_wait_limit)
// this host thread's second stream on the current device and its fork / join
// events (false if they cannot be made: then run on one stream)
bool side_stream(cudaStream_t *stream, cudaEvent_t *fork, cudaEvent_t *join);
// Let `kern` launch with `dyn` bytes of dynamic shared memory: the 48 KB that
// a kernel gets without opting in cover its static and dynamic shared memory
// together, so a launch whose dynamic part alone is below 48 KB can still
// need the opt-in
template <typename K>
inline void smem_optin(K *kern, size_t dyn) {
	cudaFuncAttributes a;
	const size_t st = cudaFuncGetAttributes(&a, (const void *)kern) == cudaSuccess ? a.sharedSizeBytes : 0;
	if (dyn + st > 48 * 1024)
		cudaFuncSetAttribute((const void *)kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn);
}

template <typename T> struct MatT;
template <> struct MatT<double> { typedef struct blasfeo_dmat type; typedef struct blasfeo_dmat_batch batch; typedef struct blasfeo_dvec vec; };
template <> struct MatT<float> { typedef struct blasfeo_smat type; typedef struct blasfeo_smat_batch batch; typedef struct blasfeo_svec vec; };

}  // namespace bf

// ---------------------------------------------------------------------------
// device-side views
// ---------------------------------------------------------------------------

// descriptor layout as seen from the device (same as struct blasfeo_dmat / smat)
template <typename T>
struct DevDesc {
	T *mem;
	T *pA;
	T *dA;
	int m, n, pm, cn, use_dA, memsize;
};
static_assert(sizeof(DevDesc<double>) == sizeof(struct blasfeo_dmat), "descriptor layout");
static_assert(sizeof(DevDesc<float>) == sizeof(struct blasfeo_smat), "descriptor layout");

template <typename T>
struct DevVec {
	T *mem;
	T *pa;
	int m, pm, memsize;
};
static_assert(sizeof(DevVec<double>) == sizeof(struct blasfeo_dvec), "vector layout");

// A matrix of one instance, with row/column offsets folded in.
template <typename T>
struct PMat {
	T *p;    // pA
	T *d;    // dA
	int cn;  // panel stride (columns)
	int ri, cj;
	__device__ __forceinline__ T &at(int i, int j) const {
		i += ri;
		j += cj;
		return p[(size_t)(i & ~3) * cn + j * 4 + (i & 3)];
	}
	__device__ __forceinline__ T *addr(int i, int j) const {
		i += ri;
		j += cj;
		return p + (size_t)(i & ~3) * cn + j * 4 + (i & 3);
	}
};

// How a kernel finds instance b's matrix: either a strided slab (uniform
// batch, or a single instance with stride 0) or a device array of descriptors.
template <typename T>
struct MatArg {
	T *pA;
	T *dA;
	int cn;
	int ri, cj;
	long long stride;
	const DevDesc<T> *desc;  // non-null: variable-size batch mode (offsets are zero)

	__device__ __forceinline__ PMat<T> get(int b) const {
		PMat<T> r;
		if (desc) {
			const DevDesc<T> &d = desc[b];
			r.p = d.pA;
			r.d = d.dA;
			r.cn = d.cn;
			r.ri = 0;
			r.cj = 0;
		} else {
			r.p = pA + stride * b;
			r.d = dA + stride * b;
			r.cn = cn;
			r.ri = ri;
			r.cj = cj;
		}
		return r;
	}
};

// Per-instance sizes: uniform (pm == nullptr) or device arrays.
struct SizeArg {
	int m, n, k;
	const int *pm, *pn, *pk;
	__device__ __forceinline__ int M(int b) const { return pm ? pm[b] : m; }
	__device__ __forceinline__ int N(int b) const { return pn ? pn[b] : n; }
	__device__ __forceinline__ int K(int b) const { return pk ? pk[b] : k; }
};

template <typename T>
static inline MatArg<T> single_arg(typename bf::MatT<T>::type *s, int ri, int cj) {
	MatArg<T> a;
	a.pA = s->pA;
	a.dA = s->dA;
	a.cn = s->cn;
	a.ri = ri;
	a.cj = cj;
	a.stride = 0;
	a.desc = nullptr;
	return a;
}

template <typename T>
static inline MatArg<T> batch_arg(typename bf::MatT<T>::batch *s, int ri, int cj) {
	MatArg<T> a;
	a.pA = s->pA;
	a.dA = s->dA;
	a.cn = s->cn;
	a.ri = ri;
	a.cj = cj;
	a.stride = s->stride;
	a.desc = nullptr;
	return a;
}

template <typename T>
static inline MatArg<T> vbatch_arg(const void *desc) {
	MatArg<T> a;
	a.pA = nullptr;
	a.dA = nullptr;
	a.cn = 0;
	a.ri = 0;
	a.cj = 0;
	a.stride = 0;
	a.desc = (const DevDesc<T> *)desc;
	return a;
}

static inline SizeArg uniform_sizes(int m, int n, int k) {
	SizeArg s;
	s.m = m;
	s.n = n;
	s.k = k;
	s.pm = s.pn = s.pk = nullptr;
	return s;
}

static inline SizeArg var_sizes(const int *m, const int *n, const int *k) {
	SizeArg s;
	s.m = s.n = s.k = 0;
	s.pm = m;
	s.pn = n;
	s.pk = k;
	return s;
}

// ---------------------------------------------------------------------------
// small device utilities
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ T dev_abs(T x) { return x < T(0) ? -x : x; }

// FP64 reciprocal square root pieces used by the Cholesky pivots: the pivot
// rule of the reference (kernel/generic/kernel_dgemm_4x4_lib4.c:5700-5710):
// c > 0 -> d = sqrt(c), inv = 1/d; otherwise d = 0, inv = 0.
__device__ __forceinline__ void chol_pivot(double c, double &d, double &inv) {
	if (c > 0.0) {
		d = sqrt(c);
		inv = 1.0 / d;
	} else {
		d = 0.0;
		inv = 0.0;
	}
}

__host__ __device__ __forceinline__ int cdiv(int a, int b) { return (a + b - 1) / b; }
