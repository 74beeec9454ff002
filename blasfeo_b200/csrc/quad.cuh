// Building blocks of the kernels that give one instance of a batch-interleaved
// slab (interleave.cu) to a quad of lanes: lane q of the quad owns the rows
// i = q + 4s (s = 0..3) of a 16 x 16 operand, 8 instances per warp.
//
// Layout: element slot e of instance b at mem[(b / IL) * gstride + e * IL + b % IL];
// the warp's 8 instances are half of one group, so one element of all of them
// is a contiguous 64-byte run.
#pragma once

#include "common.cuh"

namespace quad {

constexpr int IL = 16;   // instances per interleaved group
constexpr int QPW = 8;   // instances per warp (a quad each)

// lib4 slot of element (i, j) with panel stride cn (include/blasfeo_common.h:112)
__device__ __forceinline__ long long pme(int i, int j, int cn) { return (long long)(i & ~3) * cn + 4 * j + (i & 3); }

// the quad's lane that owns row i
__device__ __forceinline__ int owner(int lane, int i) { return (lane & ~3) | (i & 3); }

// packed lower triangles in shared memory: strictly lower (l < j) and with the
// diagonal (l <= j)
__device__ __forceinline__ int tri(int j) { return j * (j - 1) / 2; }
__device__ __forceinline__ int tri_d(int j) { return j * (j + 1) / 2; }

// 16-byte copy HBM -> shared memory that holds no register while in flight
__device__ __forceinline__ void cpa16(void *dst, const void *src) {
	const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
	asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cpa_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cpa_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// Cholesky column J of the quad's 16 x 16 operand, J = 0..15 by recursion
// (compile-time indices only, so S stays in registers).  S[s][j] = entry
// (q + 4s, j), j <= 4s + 3.  Pivot rule of the reference
// (kernel/generic/kernel_dgemm_4x4_lib4.c:5700-5710): c > 0 -> L_jj = sqrt(c)
// (formed as c * rsqrt(c)) and 1/L_jj = rsqrt(c), else 0 and 0.  The inverse
// pivot of column J < m goes to dA[J * IL] (HBM, when act) and, when PARK, to
// ism[QPW * J] (shared memory); bad = first J < m with a non-positive pivot,
// plus one.  Columns >= m must hold an identity block (they factor to it).
template <int J, bool PARK>
struct QCol {
	static __device__ __forceinline__ void run(double (&S)[4][16], int q, int lane, int m, double *ism, double *dA,
	                                           bool act, int &bad) {
		constexpr int SJ = J >> 2;
		const double mine = (q == (J & 3)) ? S[SJ][J] : 0.0;
		const double c = __shfl_sync(0xffffffffu, mine, owner(lane, J));
		const bool ok = c > 0.0;
		const double iv = ok ? rsqrt(c) : 0.0;
		if (!ok && J < m && bad == 0) bad = J + 1;
		if (q == (J & 3)) {
			S[SJ][J] = ok ? c * iv : 0.0;
			if (PARK) ism[QPW * J] = iv;
			if (act && J < m) dA[J * IL] = iv;
		}
#pragma unroll
		for (int s = 0; s < 4; s++)
			if (J <= 4 * s + 3 && q + 4 * s > J) S[s][J] *= iv;
#pragma unroll
		for (int l = J + 1; l < 16; l++) {
			const double own = (q == (l & 3)) ? S[l >> 2][J] : 0.0;
			const double llj = __shfl_sync(0xffffffffu, own, owner(lane, l));
#pragma unroll
			for (int s = 0; s < 4; s++)
				if (l <= 4 * s + 3 && q + 4 * s >= l) S[s][l] = fma(-S[s][J], llj, S[s][l]);
		}
		QCol<J + 1, PARK>::run(S, q, lane, m, ism, dA, act, bad);
	}
};
template <bool PARK>
struct QCol<16, PARK> {
	static __device__ __forceinline__ void run(double (&)[4][16], int, int, int, double *, double *, bool, int &) {}
};

// S[s][j] += sum over the columns c < nc of W(q + 4s, c) W(j, c), W read from
// shared memory at w[16 i + c][t] (rows >= mrow read as zero): the syrk of the
// quad's rows, entries j > q + 4s computed and left for the caller to clear
__device__ __forceinline__ void syrk_rows(double (&S)[4][16], const double (*w)[QPW], int nc, int mrow, int q,
                                          int t) {
#pragma unroll 2
	for (int c = 0; c < nc; c++) {
		double col[16];
#pragma unroll
		for (int i = 0; i < 16; i++) col[i] = (i < mrow) ? w[16 * i + c][t] : 0.0;
#pragma unroll
		for (int s = 0; s < 4; s++) {
			const double ai =
			    (q == 0) ? col[4 * s] : (q == 1) ? col[4 * s + 1] : (q == 2) ? col[4 * s + 2] : col[4 * s + 3];
#pragma unroll
			for (int j = 0; j < 16; j++)
				if (j <= 4 * s + 3) S[s][j] = fma(ai, col[j], S[s][j]);
		}
	}
}

// clear the entries right of the diagonal of the quad's rows, optionally
// adding `shift` on the diagonal.  Selects, not conditional stores: a store
// under (j == q + 4s) is turned into S[s][q + 4s] and S into a local-memory
// array.
__device__ __forceinline__ void clear_upper(double (&S)[4][16], int q, double shift) {
#pragma unroll
	for (int s = 0; s < 4; s++)
#pragma unroll
		for (int j = 4 * s; j < 4 * s + 4; j++) {
			const double v = S[s][j] + ((j == q + 4 * s) ? shift : 0.0);
			S[s][j] = (j > q + 4 * s) ? 0.0 : v;
		}
}

}  // namespace quad
