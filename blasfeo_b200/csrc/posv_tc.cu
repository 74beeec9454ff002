// Mixed-precision factor + solve of SPD systems (n <= 256) on the tensor
// cores: the trailing matrix of the Cholesky factorization lives in tensor
// memory (TMEM) for the whole factorization and is updated by tcgen05.mma.
//
// The chain it replaces is the reference's dpotrf_l followed by dtrsv_lnn and
// dtrsv_ltn (blasfeo_hp_pm/d_lapack_lib4.c:918, blasfeo_hp_pm/d_blas2_lib4.c),
// with FP64 iterative refinement around it.
//
// One persistent CTA per SM (per 128 rows of TMEM: NT = 128 threads for
// n <= 128, NT = 256 for n <= 256) pulls systems from the size-sorted work
// list.  Thread t owns row t of the system throughout:
//
//   load       row t of the lower triangle (FP64 global, panel-major) ->
//              FP32 -> TMEM lane t % 128 (rows >= 128 in a second column
//              range), identity in the padding up to npad = 16*ceil(n/16);
//   factor     right-looking by 16-column blocks K:
//                tcgen05.ld of block column K (thread t gets its 16 values);
//                the 16 threads of the diagonal block factor it in FP64
//                registers (FP64 rsqrt pivots and reciprocals; pivot rule of
//                kernel/generic/kernel_dgemm_4x4_lib4.c:5700-5710);
//                every row below solves its 16 entries against the diagonal
//                block (FP32, reciprocal-pivot multiply);
//                the panel goes to shared memory split into TF32 high and low
//                parts, and one thread issues the rank-16 trailing update
//                D -= P P^T as 3xTF32 (hi*hi + hi*lo + lo*hi, FP32
//                accumulation in TMEM), completion signalled on an mbarrier;
//              the factor is kept in shared memory (FP32 lower panels) with
//              FP64 reciprocal pivots and FP32 inverses of the 16x16 diagonal
//              blocks (formed in FP64);
//   refine     x = 0, r = b; repeat: d = L^-T L^-1 r (FP32, one thread per
//              row, one barrier per 16-row block), x += d (FP64), r = b - A x
//              (FP64, thread t sums row t of A from the lower triangle in
//              global memory: its row to the left of the diagonal and its
//              column below it), until ||r||_inf <= tol ||A||_inf ||x||_inf.
//
// Every mbarrier wait is bounded; on a timeout the system reports info = -3
// and the CTA stops taking work, waits (bounded) for its tensor-core work and
// frees its tensor memory before it exits.
#include <climits>

#include "chol.cuh"
#include "common.cuh"
#include "posv.cuh"
#include "tma.cuh"

namespace {

// ---------------------------------------------------------------------------
// tcgen05 wrappers (PTX ISA 8.6+, sm_100a)
// ---------------------------------------------------------------------------
__device__ __forceinline__ void tmem_alloc(uint32_t *dst, uint32_t ncols) {
	asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)), "r"(ncols)
	             : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
	asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
	asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

// 32 lanes x 16 consecutive 32-bit columns: thread l of the warp gets lane
// (taddr.lane + l), columns taddr.col .. +15
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
	uint32_t r[16];
	asm volatile(
	    "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
	    "%15}, [%16];"
	    : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
	      "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
	    : "r"(taddr)
	    : "memory");
#pragma unroll
	for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_st16(uint32_t taddr, const float (&v)[16]) {
	asm volatile(
	    "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
	    "%15, %16};" ::"r"(taddr),
	    "r"(__float_as_uint(v[0])), "r"(__float_as_uint(v[1])), "r"(__float_as_uint(v[2])), "r"(__float_as_uint(v[3])),
	    "r"(__float_as_uint(v[4])), "r"(__float_as_uint(v[5])), "r"(__float_as_uint(v[6])), "r"(__float_as_uint(v[7])),
	    "r"(__float_as_uint(v[8])), "r"(__float_as_uint(v[9])), "r"(__float_as_uint(v[10])),
	    "r"(__float_as_uint(v[11])), "r"(__float_as_uint(v[12])), "r"(__float_as_uint(v[13])),
	    "r"(__float_as_uint(v[14])), "r"(__float_as_uint(v[15]))
	    : "memory");
}

// D[tmem] (+)= A * B^T, A: M=128 rows, B: N rows, K = 8 TF32 per instruction
__device__ __forceinline__ void tc_mma_tf32(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                            uint32_t accumulate) {
	asm volatile(
	    "{\n\t.reg .pred p;\n\t"
	    "setp.ne.b32 p, %4, 0;\n\t"
	    "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
	    "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
	    : "memory");
}
// arrive on bar once all tcgen05.mma issued so far by this thread completed
__device__ __forceinline__ void tc_commit(uint64_t *bar) {
	asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
	             : "memory");
}

// Shared-memory matrix descriptor, K-major, no swizzle: the operand is a grid
// of core matrices of 8 rows x 16 bytes (each 128 contiguous bytes); lbo = byte
// distance between the two K-adjacent core matrices of one MMA (K = 8 TF32 =
// 32 bytes), sbo = byte distance between 8-row groups.  Bits: start address
// >> 4 [0,14), lbo >> 4 [16,30), sbo >> 4 [32,46), descriptor version 1
// [46,48), base offset 0, layout type 0 (no swizzle) [61,64).
__device__ __forceinline__ uint64_t smem_desc_k(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
	return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
	       ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | ((uint64_t)1 << 46);
}
// Instruction descriptor of kind::tf32: D format F32 [4,6) = 1, A and B format
// TF32 [7,10) = [10,13) = 2, negate A [13], A and B K-major [15], [16] = 0,
// N >> 3 [17,23), M >> 4 [24,29) with M = 128.
__host__ __device__ constexpr uint32_t idesc_tf32_neg_a(int N) {
	return (1u << 4) | (2u << 7) | (2u << 10) | (1u << 13) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

// round to TF32 (10 explicit mantissa bits), nearest with ties away from zero
__device__ __forceinline__ float tf32_round(float x) {
	return __uint_as_float((__float_as_uint(x) + 0x1000u) & 0xFFFFE000u);
}

// Panel operand layout (K-major, 16 K-columns per row): element (r, k) at
// float offset (r/8)*128 + (k/4)*32 + (r%8)*4 + k%4; an MMA's K-slice s
// (k = 8s..8s+7) starts 256*s bytes in; lbo = 128 B, sbo = 512 B.
__device__ __forceinline__ int pan_off(int r, int kc) { return (r >> 3) * 128 + kc * 32 + (r & 7) * 4; }

__host__ __device__ inline size_t al16(size_t x) { return (x + 15) / 16 * 16; }

// shared-memory plan for size-class upper bound U (npad <= 256)
struct TcPlan {
	uint32_t ph, pl, L, inv, lt, dinv, xs, yb, red, mbar, tmem, item, bad, err, total;
	int prow;
};
__host__ __device__ inline TcPlan tc_plan(int U) {
	TcPlan p;
	const int npad = (U + 15) / 16 * 16;
	const int NB = npad / 16;
	p.prow = npad > 128 ? 256 : 128;
	size_t o = 0;
	p.ph = (uint32_t)o;
	o += (size_t)p.prow * 64;
	p.pl = (uint32_t)o;
	o += (size_t)p.prow * 64;
	p.L = (uint32_t)o;
	o += al16((size_t)lp_size(npad) * 4);
	p.inv = (uint32_t)o;
	o += (size_t)NB * 1024;
	p.lt = (uint32_t)o;
	o += al16(16 * 17 * 4);
	p.dinv = (uint32_t)o;
	o += (size_t)npad * 8;
	p.xs = (uint32_t)o;
	o += (size_t)npad * 8;
	p.yb = (uint32_t)o;
	o += 2 * 16 * 4;
	p.red = (uint32_t)o;
	o += 8 * 4 * 8;
	p.mbar = (uint32_t)o;
	o += 8;
	p.tmem = (uint32_t)o;
	o += 4;
	p.item = (uint32_t)o;
	o += 4;
	p.bad = (uint32_t)o;
	o += 4;
	p.err = (uint32_t)o;
	o += 4;
	p.total = (uint32_t)al16(o);
	return p;
}

// ---------------------------------------------------------------------------
// the 16x16 diagonal block in FP64 registers
// ---------------------------------------------------------------------------
// Lanes hb..hb+15 of the calling warp hold rows c0..c0+15 of block column K
// (v: the trailing-matrix values after all earlier updates); all 32 lanes
// execute (full-warp shuffles), lanes outside the half-warp compute junk that
// is discarded.  Lane i keeps its diagonal entry in dg so that the next pivot
// needs no shuffle of its own row: per column the critical path is one
// shuffle of the pivot, the FP64 rsqrt, a multiply and a fused update.
// Outputs: Lt (row-major 16x17 FP32, reciprocal pivots in column 16), L_KK
// into the FP32 lower panels, FP64 reciprocal pivots dinv[c0+i], the first
// non-positive pivot (c0+j+1) into *bad.
__device__ __forceinline__ void diag16_tc(const float (&v)[16], int hb, int c0, float *Lt, float *Lsm, double *dinv,
                                          int *bad) {
	const int lane = threadIdx.x & 31;
	const int i = lane - hb;  // row in the block (valid for 0 <= i < 16)
	double r[16];
	double dg = 0.0;
#pragma unroll
	for (int l = 0; l < 16; l++) {
		r[l] = (double)v[l];
		if (l == i) dg = r[l];
	}
	double myinv = 1.0;
	int firstbad = 0;
#pragma unroll
	for (int J = 0; J < 16; J++) {
		const double cj = __shfl_sync(0xffffffffu, dg, (hb + J) & 31);
		const bool ok = cj > 0.0;
		const double inv = ok ? rsqrt(cj) : 0.0;
		const double lj = r[J] * inv;
		if (i == J) {
			r[J] = ok ? cj * inv : 0.0;
			myinv = inv;
		} else if (i > J) {
			r[J] = lj;
			dg = fma(-lj, lj, dg);
		}
		if (!ok && firstbad == 0) firstbad = c0 + J + 1;
#pragma unroll
		for (int l = J + 1; l < 16; l++) {
			const double t = __shfl_sync(0xffffffffu, r[J], (hb + l) & 31);
			if (i > l) r[l] = fma(-r[J], t, r[l]);
		}
	}
	if (i >= 0 && i < 16) {
#pragma unroll
		for (int l = 0; l < 16; l++) {
			const float x = (l <= i) ? (float)r[l] : 0.f;
			Lt[i * 17 + l] = x;
			if (l <= i) lp_at(Lsm, c0 + i, c0 + l) = x;
		}
		Lt[i * 17 + 16] = (float)myinv;
		dinv[c0 + i] = myinv;
		if (i == 0 && firstbad && *bad == 0) *bad = firstbad;
	}
}

// ---------------------------------------------------------------------------
// refinement pieces (one thread per row)
// ---------------------------------------------------------------------------
// w := L^{-1} w; thread t holds w_t in wv.  Per 16-row block K the 16 owner
// threads form y_K = inv(L_KK) w_K by half-warp shuffles and publish it; every
// row below subtracts L[t, K-block] y_K.  One barrier per block (y is double
// buffered).
__device__ __forceinline__ void trsv_fwd_rows(const float *Lsm, const float *invL, int npad, float *ybuf, float &wv) {
	const int tid = threadIdx.x, lane = tid & 31;
	const int NB = npad >> 4;
	for (int K = 0; K < NB; K++) {
		const int c0 = 16 * K;
		float *yb = ybuf + 16 * (K & 1);
		if ((tid >> 4) == K) {
			const int i = tid & 15, hb = lane & 16;
			const unsigned mask = 0xffffu << hb;
			const float *inv = invL + K * 256 + i * 16;
			float s = 0.f;
#pragma unroll
			for (int l = 0; l < 16; l++) {
				const float wl = __shfl_sync(mask, wv, hb + l);
				if (l <= i) s = fmaf(inv[l], wl, s);
			}
			yb[i] = s;
			wv = s;
		}
		__syncthreads();
		if (tid >= c0 + 16 && tid < npad) {
#pragma unroll
			for (int l = 0; l < 16; l++) wv = fmaf(-lp_at(Lsm, tid, c0 + l), yb[l], wv);
		}
	}
}

// w := L^{-T} w (same scheme from the last block up; rows above a block
// subtract the block's column slice of L).
__device__ __forceinline__ void trsv_bwd_rows(const float *Lsm, const float *invL, int npad, float *ybuf, float &wv) {
	const int tid = threadIdx.x, lane = tid & 31;
	const int NB = npad >> 4;
	for (int K = NB - 1; K >= 0; K--) {
		const int c0 = 16 * K;
		float *yb = ybuf + 16 * (K & 1);
		if ((tid >> 4) == K) {
			const int i = tid & 15, hb = lane & 16;
			const unsigned mask = 0xffffu << hb;
			const float *inv = invL + K * 256 + i;
			float s = 0.f;
#pragma unroll
			for (int l = 0; l < 16; l++) {
				const float yl = __shfl_sync(mask, wv, hb + l);
				if (l >= i) s = fmaf(inv[l * 16], yl, s);
			}
			yb[i] = s;
			wv = s;
		}
		__syncthreads();
		if (tid < c0) {
#pragma unroll
			for (int l = 0; l < 16; l++) wv = fmaf(-lp_at(Lsm, c0 + l, tid), yb[l], wv);
		}
	}
}

// Row t of b - A x for symmetric A given by its lower triangle (panel-major,
// panel stride cn, row offset 0, 16-byte aligned): sum over the row to the
// left of the diagonal (scalar loads; the 4 rows of a panel read one 32-byte
// sector together) and over the column below it (4 rows of a panel in two
// 16-byte loads).  asum: sum of |A_tj| over the whole row.
__device__ __forceinline__ void resid_row(const double *__restrict__ A, int cn, int n, int t, const double *xs,
                                          double bt, double &r, double &asum) {
	const double *rowp = A + (size_t)(t & ~3) * cn + (t & 3);
	double acc0 = 0.0, acc1 = 0.0, as0 = 0.0, as1 = 0.0;
	int j = 0;
	for (; j + 8 <= t + 1; j += 8) {
		double a[8];
#pragma unroll
		for (int u = 0; u < 8; u++) a[u] = __ldg(rowp + 4 * (j + u));
#pragma unroll
		for (int u = 0; u < 8; u += 2) {
			acc0 = fma(a[u], xs[j + u], acc0);
			acc1 = fma(a[u + 1], xs[j + u + 1], acc1);
			as0 += fabs(a[u]);
			as1 += fabs(a[u + 1]);
		}
	}
	for (; j <= t; j++) {
		const double a = __ldg(rowp + 4 * j);
		acc0 = fma(a, xs[j], acc0);
		as0 += fabs(a);
	}
	// column t below the diagonal: rest of t's own panel
	const int pe = (t | 3) < n - 1 ? (t | 3) : n - 1;
	for (j = t + 1; j <= pe; j++) {
		const double a = __ldg(A + (size_t)(t & ~3) * cn + 4 * t + (j & 3));
		acc1 = fma(a, xs[j], acc1);
		as1 += fabs(a);
	}
	// whole panels below
	int p = (t >> 2) + 1;
	for (; 4 * p + 8 <= n; p += 2) {
		const double *c0p = A + (size_t)(4 * p) * cn + 4 * t;
		const double *c1p = c0p + (size_t)4 * cn;
		const double2 a01 = __ldg((const double2 *)c0p), a23 = __ldg((const double2 *)c0p + 1);
		const double2 b01 = __ldg((const double2 *)c1p), b23 = __ldg((const double2 *)c1p + 1);
		const double *x = xs + 4 * p;
		acc0 = fma(a01.x, x[0], acc0);
		acc1 = fma(a01.y, x[1], acc1);
		acc0 = fma(a23.x, x[2], acc0);
		acc1 = fma(a23.y, x[3], acc1);
		acc0 = fma(b01.x, x[4], acc0);
		acc1 = fma(b01.y, x[5], acc1);
		acc0 = fma(b23.x, x[6], acc0);
		acc1 = fma(b23.y, x[7], acc1);
		as0 += fabs(a01.x) + fabs(a23.x) + fabs(b01.x) + fabs(b23.x);
		as1 += fabs(a01.y) + fabs(a23.y) + fabs(b01.y) + fabs(b23.y);
	}
	for (; 4 * p < n; p++) {
		const double *cp = A + (size_t)(4 * p) * cn + 4 * t;
		const double2 a01 = __ldg((const double2 *)cp), a23 = __ldg((const double2 *)cp + 1);
		const double av[4] = {a01.x, a01.y, a23.x, a23.y};
#pragma unroll
		for (int q = 0; q < 4; q++)
			if (4 * p + q < n) {
				acc0 = fma(av[q], xs[4 * p + q], acc0);
				as0 += fabs(av[q]);
			}
	}
	r = bt - (acc0 + acc1);
	asum = as0 + as1;
}

// max over the CTA of three non-negative values; every thread gets the result
__device__ __forceinline__ void block_max3(double a, double b, double c, double *red, double &ra, double &rb,
                                           double &rc) {
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
	for (int off = 16; off > 0; off >>= 1) {
		a = fmax(a, __shfl_xor_sync(0xffffffffu, a, off));
		b = fmax(b, __shfl_xor_sync(0xffffffffu, b, off));
		c = fmax(c, __shfl_xor_sync(0xffffffffu, c, off));
	}
	if (lane == 0) {
		red[4 * warp] = a;
		red[4 * warp + 1] = b;
		red[4 * warp + 2] = c;
	}
	__syncthreads();
	ra = rb = rc = 0.0;
	for (int w = 0; w < nw; w++) {
		ra = fmax(ra, red[4 * w]);
		rb = fmax(rb, red[4 * w + 1]);
		rc = fmax(rc, red[4 * w + 2]);
	}
}

// ---------------------------------------------------------------------------
// the kernel
// ---------------------------------------------------------------------------
template <int NT>
__global__ void __launch_bounds__(NT, 1)
    k_posv_tc(int cls, int U, PosvWs ws, const int *__restrict__ nvec, const DevDesc<double> *__restrict__ sA,
              const DevVec<double> *__restrict__ sb, const DevVec<double> *__restrict__ sx, int max_iter, double tol,
              int *iters, double *berr, int *info, uint32_t tmem_cols, uint32_t wait_limit) {
	extern __shared__ __align__(1024) unsigned char smem[];
	const TcPlan pl = tc_plan(U);
	float *Ph = (float *)(smem + pl.ph);
	float *Pl = (float *)(smem + pl.pl);
	float *Lsm = (float *)(smem + pl.L);
	float *invL = (float *)(smem + pl.inv);
	float *Lt = (float *)(smem + pl.lt);
	double *dinv = (double *)(smem + pl.dinv);
	double *xs = (double *)(smem + pl.xs);
	float *ybuf = (float *)(smem + pl.yb);
	double *red = (double *)(smem + pl.red);
	uint64_t *mbar = (uint64_t *)(smem + pl.mbar);
	uint32_t *s_tmem = (uint32_t *)(smem + pl.tmem);
	int *s_item = (int *)(smem + pl.item);
	int *s_bad = (int *)(smem + pl.bad);
	int *s_err = (int *)(smem + pl.err);
	const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
	const int start = ws.start[cls], count = ws.count[cls];

	for (int i = tid; i < pl.prow * 16; i += NT) {
		Ph[i] = 0.f;
		Pl[i] = 0.f;
	}
	if (warp == 0) {
		tmem_alloc(s_tmem, tmem_cols);
		tmem_relinquish();
	}
	if (tid == 0) {
		mbar_init(mbar, 1);
		mbar_fence_init();
		*s_err = 0;
	}
	tc_fence_before();
	__syncthreads();
	tc_fence_after();
	const uint32_t tbase = *s_tmem;
	const uint32_t lane_field = (uint32_t)(32 * (warp & 3)) << 16;
	const int blk = warp >> 2;  // 128-row block of this warp's rows
	uint32_t phase = 0;
	const uint32_t sm_ph = smem_u32(Ph), sm_pl = smem_u32(Pl);

	for (;;) {
		if (tid == 0) {
			int k = atomicAdd(&ws.counter[cls], 1);
			*s_item = (k < count && *s_err == 0) ? ws.list[start + k] : -1;
			*s_bad = 0;
		}
		__syncthreads();
		const int sys = *s_item;
		if (sys < 0) break;
		const int n = nvec[sys];
		if (n <= 0 || n > U) {
			if (tid == 0) {
				if (info) info[sys] = (n <= 0) ? 0 : -2;
				if (iters) iters[sys] = 0;
			}
			__syncthreads();
			continue;
		}
		const int npad = (n + 15) & ~15, NB = npad >> 4;
		const double *A = sA[sys].pA;
		const int cn = sA[sys].cn;
		const double *bg = sb[sys].pa;
		double *xg = sx[sys].pa;
		const int row = tid;
		// TMEM column of matrix column 0 for this warp's rows
		const uint32_t tcol = tbase + lane_field + (uint32_t)(blk * npad);
		const bool wact = 32 * warp < npad;
		const double bval = (row < n) ? bg[row] : 0.0;

		// ---- lower triangle -> TMEM (FP32), identity padding ----
		if (wact) {
			const int qmax = ((32 * warp + 31) >> 4) < NB - 1 ? ((32 * warp + 31) >> 4) : NB - 1;
			const double *rp = A + (size_t)(row & ~3) * cn + (row & 3);
			for (int q = 0; q <= qmax; q++) {
				float v[16];
#pragma unroll
				for (int l = 0; l < 16; l++) {
					const int j = 16 * q + l;
					float x = 0.f;
					if (j <= row && row < npad) {
						if (row < n)
							x = (float)__ldg(rp + 4 * j);
						else
							x = (j == row) ? 1.f : 0.f;
					}
					v[l] = x;
				}
				__syncwarp();
				tmem_st16(tcol + 16 * q, v);
			}
			tmem_wait_st();
		}
		if (row < npad) xs[row] = 0.0;
		tc_fence_before();
		__syncthreads();
		tc_fence_after();

		// ---- factorization ----
		bool ok_run = true;
		for (int K = 0; K < NB; K++) {
			const int c0 = 16 * K;
			if (K > 0) {
				if (!mbar_wait(mbar, phase, wait_limit)) *s_err = 1;
				phase ^= 1u;
				tc_fence_after();
			}
			float v[16];
			const bool has = wact && (32 * warp + 31 >= c0);
			if (has) {
				__syncwarp();  // tcgen05.ld is warp-collective: reconverge after the bounded wait
				tmem_ld16(tcol + c0, v);
				tmem_wait_ld();
			}
			if (warp == (c0 >> 5)) diag16_tc(v, c0 & 16, c0, Lt, Lsm, dinv, s_bad);
			__syncthreads();
			if (*s_err) {  // uniform: read after the barrier
				ok_run = false;
				break;
			}
			if (has && row >= c0 + 16 && row < npad) {
#pragma unroll
				for (int c = 0; c < 16; c++) {
					float s = v[c];
#pragma unroll
					for (int l = 0; l < c; l++) s = fmaf(-v[l], Lt[c * 17 + l], s);
					v[c] = s * Lt[c * 17 + 16];
				}
#pragma unroll
				for (int l = 0; l < 16; l++) lp_at(Lsm, row, c0 + l) = v[l];
#pragma unroll
				for (int kc = 0; kc < 4; kc++) {
					float4 h, o;
					h.x = tf32_round(v[4 * kc]);
					h.y = tf32_round(v[4 * kc + 1]);
					h.z = tf32_round(v[4 * kc + 2]);
					h.w = tf32_round(v[4 * kc + 3]);
					o.x = tf32_round(v[4 * kc] - h.x);
					o.y = tf32_round(v[4 * kc + 1] - h.y);
					o.z = tf32_round(v[4 * kc + 2] - h.z);
					o.w = tf32_round(v[4 * kc + 3] - h.w);
					*(float4 *)(Ph + pan_off(row, kc)) = h;
					*(float4 *)(Pl + pan_off(row, kc)) = o;
				}
			}
			fence_proxy_async_smem();
			tc_fence_before();
			__syncthreads();
			if (K + 1 < NB && tid == 0) {
				tc_fence_after();
				const int j0 = c0 + 16;
				const int N = npad - j0;
				const uint32_t idesc = idesc_tf32_neg_a(N);
				const uint32_t boff = (uint32_t)(j0 >> 3) * 512u;
				for (int b = 0; b < 2; b++) {
					// row block b (rows 128b..128b+127) has trailing rows?
					if (b == 1 && npad <= 128) break;
					if (b == 0 && j0 >= 128) continue;
					const uint32_t d = tbase + (uint32_t)(b * npad + j0);
					const uint32_t aoff = (uint32_t)b * 8192u;
#pragma unroll
					for (int s = 0; s < 2; s++) {
						const uint64_t ah = smem_desc_k(sm_ph + aoff + 256u * s, 128u, 512u);
						const uint64_t al = smem_desc_k(sm_pl + aoff + 256u * s, 128u, 512u);
						const uint64_t bh = smem_desc_k(sm_ph + boff + 256u * s, 128u, 512u);
						const uint64_t bl = smem_desc_k(sm_pl + boff + 256u * s, 128u, 512u);
						tc_mma_tf32(d, ah, bh, idesc, 1u);
						tc_mma_tf32(d, ah, bl, idesc, 1u);
						tc_mma_tf32(d, al, bh, idesc, 1u);
					}
				}
				tc_commit(mbar);
			}
		}
		if (!ok_run) {
			if (tid == 0 && info) info[sys] = -3;
			__syncthreads();
			break;
		}

		// ---- FP32 inverses (formed in FP64) of the diagonal blocks ----
		for (int K = warp; K < NB; K += NT / 32) chol_block_inverse<float>(Lsm, npad, K, dinv, invL + K * 256, lane);
		__syncthreads();

		// ---- refinement ----
		double rm0, xm0, am0;
		block_max3(fabs(bval), 0.0, 0.0, red, rm0, xm0, am0);
		double scale = rm0 > 0.0 ? 1.0 / rm0 : 1.0;
		float wv = (row < n) ? (float)(bval * scale) : 0.f;
		double xv = 0.0;
		double anorm = 0.0, bres = INFINITY;
		int it = 0;
		bool conv = false;
		for (;;) {
			trsv_fwd_rows(Lsm, invL, npad, ybuf, wv);
			__syncthreads();
			trsv_bwd_rows(Lsm, invL, npad, ybuf, wv);
			if (row < n) xv += (double)wv / scale;
			if (row < npad) xs[row] = xv;
			__syncthreads();
			double rv = 0.0, as = 0.0;
			if (row < n) resid_row(A, cn, n, row, xs, bval, rv, as);
			double rm, xm, am;
			block_max3(fabs(rv), fabs(xv), as, red, rm, xm, am);
			if (it == 0) anorm = am;
			it++;
			bres = (anorm > 0.0 && xm > 0.0) ? rm / (anorm * xm) : (rm == 0.0 ? 0.0 : INFINITY);
			if (bres <= tol) {
				conv = true;
				break;
			}
			if (it > max_iter) break;
			scale = rm > 0.0 ? 1.0 / rm : 1.0;
			wv = (row < n) ? (float)(rv * scale) : 0.f;
		}
		if (row < n) xg[row] = xv;
		if (tid == 0) {
			if (iters) iters[sys] = it - 1;
			if (berr) berr[sys] = bres;
			if (info) info[sys] = *s_bad ? *s_bad : (conv ? 0 : -1);
		}
		__syncthreads();
	}

	// teardown: tensor-core work finished (every commit was waited for, or a
	// last bounded wait after a timeout), then free the tensor memory
	if (*s_err) mbar_wait(mbar, phase ^ 1u, BF_DRAIN_LIMIT);
	tc_fence_before();
	__syncthreads();
	tc_fence_after();
	if (warp == 0) tmem_dealloc(tbase, tmem_cols);
}

template <int NT>
int launch_tc(int cls, int U, int batch, PosvWs ws, const int *n, const void *sA, const void *sb, const void *sx,
              int max_iter, double tol, int *iters, double *berr, int *info, cudaStream_t s) {
	const TcPlan pl = tc_plan(U);
	const int npad = (U + 15) / 16 * 16;
	uint32_t cols = npad <= 32 ? 32u : (npad <= 64 ? 64u : (npad <= 128 ? 128u : 512u));
	auto kern = k_posv_tc<NT>;
	// resident CTAs per SM may not exceed 512 / cols (each holds its tensor
	// memory for its lifetime): raise the shared-memory request until they fit
	size_t smem = pl.total;
	const size_t cap = bf::max_smem_optin();
	const int max_ctas = (int)(512u / cols);
	int per_sm = 0;
	for (;;) {
		if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
			return BLASFEO_B200_ECUDA;
		if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, NT, smem) != cudaSuccess)
			return BLASFEO_B200_ECUDA;
		if (per_sm <= max_ctas || smem >= cap) break;
		smem = smem + 8192 < cap ? smem + 8192 : cap;
	}
	if (per_sm < 1) return BLASFEO_B200_ENOTSUP;
	if (per_sm > max_ctas) per_sm = max_ctas;
	int grid = bf::num_sms() * per_sm;
	if (grid > batch) grid = batch;
	kern<<<grid, NT, smem, s>>>(cls, U, ws, n, (const DevDesc<double> *)sA, (const DevVec<double> *)sb,
	                            (const DevVec<double> *)sx, max_iter, tol, iters, berr, info, cols, bf::wait_limit());
	return bf::check_launch();
}

}  // namespace

namespace bf {

int posv_tc_launch(int cls, int upper, int batch, PosvWs ws, const int *n, const void *sA, const void *sb,
                   const void *sx, int max_iter, double tol, int *iters, double *berr, int *info, cudaStream_t s) {
	if (upper <= 0 || upper > 256) return BLASFEO_B200_ENOTSUP;
	if (upper <= 128)
		return launch_tc<128>(cls, upper, batch, ws, n, sA, sb, sx, max_iter, tol, iters, berr, info, s);
	return launch_tc<256>(cls, upper, batch, ws, n, sA, sb, sx, max_iter, tol, iters, berr, info, s);
}

}  // namespace bf
