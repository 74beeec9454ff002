// Building blocks of the kernels that give one instance of a batch-interleaved
// slab (interleave.cu) to a group of G lanes (G = 4: a quad): lane o of the
// group owns the rows i = o + G s of a 16 x 16 operand, 32 / G instances per
// warp.
//
// Layout: element slot e of instance b at mem[(b / IL) * gstride + e * IL + b % IL];
// the warp's 32 / G instances are consecutive inside one group, so one element
// of all of them is one contiguous run of 256 / G bytes.
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

// Cholesky column J of a 16 x 16 operand spread over a group of G lanes (G =
// 4, 8 or 16; lane o of the group owns the rows i = o + G s, s < 16 / G), J =
// 0..15 by recursion (compile-time indices only, so S stays in registers).
// S[s][j] = entry (o + G s, j), j <= G s + G - 1.  Pivot rule of the reference
// (kernel/generic/kernel_dgemm_4x4_lib4.c:5700-5710): c > 0 -> L_jj = sqrt(c)
// (formed as c * rsqrt(c)) and 1/L_jj = rsqrt(c), else 0 and 0.  The inverse
// pivot of column J < m goes to dA[J * IL] (HBM, when act) and, when PARK, to
// ism[(32 / G) * J] (shared memory); bad = first J < m with a non-positive
// pivot, plus one.  Columns >= m must hold an identity block (they factor to
// it).
template <int G>
__device__ __forceinline__ int gowner(int lane, int i) { return (lane & ~(G - 1)) | (i & (G - 1)); }

template <int G, int J, bool PARK>
struct GCol {
	static __device__ __forceinline__ void run(double (&S)[16 / G][16], int o, int lane, int m, double *ism, double *dA,
	                                           bool act, int &bad) {
		constexpr int R = 16 / G;
		constexpr int SJ = J / G;
		const double mine = (o == J % G) ? S[SJ][J] : 0.0;
		const double c = __shfl_sync(0xffffffffu, mine, gowner<G>(lane, J));
		const bool ok = c > 0.0;
		const double iv = ok ? rsqrt(c) : 0.0;
		if (!ok && J < m && bad == 0) bad = J + 1;
		if (o == J % G) {
			S[SJ][J] = ok ? c * iv : 0.0;
			if (PARK) ism[(32 / G) * J] = iv;
			if (act && J < m) dA[J * IL] = iv;
		}
#pragma unroll
		for (int s = 0; s < R; s++)
			if (J <= G * s + G - 1 && o + G * s > J) S[s][J] *= iv;
#pragma unroll
		for (int l = J + 1; l < 16; l++) {
			const double own = (o == l % G) ? S[l / G][J] : 0.0;
			const double llj = __shfl_sync(0xffffffffu, own, gowner<G>(lane, l));
#pragma unroll
			for (int s = 0; s < R; s++)
				if (l <= G * s + G - 1 && o + G * s >= l) S[s][l] = fma(-S[s][J], llj, S[s][l]);
		}
		GCol<G, J + 1, PARK>::run(S, o, lane, m, ism, dA, act, bad);
	}
};
template <int G, bool PARK>
struct GCol<G, 16, PARK> {
	static __device__ __forceinline__ void run(double (&)[16 / G][16], int, int, int, double *, double *, bool, int &) {}
};

// the quad form (G = 4) used by the n = 16 chain
template <int J, bool PARK>
using QCol = GCol<4, J, PARK>;

// S[s][j] += sum over c < nc of W(o + G s, c) W(j, c) for a group of G lanes,
// W column-major in shared memory: W(i, c) at w[16 c + i][t] (rows >= mrow
// read as zero).  Column c is read by broadcast; the lane's own entries are
// 16 consecutive slots over the group (no bank conflict).  Entries
// j > o + G s are computed and left for the caller to clear.
template <int G, int P>
__device__ __forceinline__ void syrk_rows_cm(double (&S)[16 / G][16], const double (*w)[P], int nc, int mrow, int o,
                                             int t) {
	constexpr int R = 16 / G;
#pragma unroll 2
	for (int c = 0; c < nc; c++) {
		double col[16], ai[R];
#pragma unroll
		for (int i = 0; i < 16; i++) col[i] = (i < mrow) ? w[16 * c + i][t] : 0.0;
#pragma unroll
		for (int s = 0; s < R; s++) ai[s] = (o + G * s < mrow) ? w[16 * c + o + G * s][t] : 0.0;
#pragma unroll
		for (int s = 0; s < R; s++)
#pragma unroll
			for (int j = 0; j < 16; j++)
				if (j <= G * s + G - 1) S[s][j] = fma(ai[s], col[j], S[s][j]);
	}
}

// clear the entries right of the diagonal of the group's rows, optionally
// adding `shift` on the diagonal.  Selects, not conditional stores: a store
// under (j == o + G s) is turned into S[s][o + G s] and S into a local-memory
// array.
template <int G>
__device__ __forceinline__ void clear_upper_g(double (&S)[16 / G][16], int o, double shift) {
#pragma unroll
	for (int s = 0; s < 16 / G; s++)
#pragma unroll
		for (int j = G * s; j < G * s + G; j++) {
			const double v = S[s][j] + ((j == o + G * s) ? shift : 0.0);
			S[s][j] = (j > o + G * s) ? 0.0 : v;
		}
}

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

// the quad form of clear_upper_g
__device__ __forceinline__ void clear_upper(double (&S)[4][16], int q, double shift) { clear_upper_g<4>(S, q, shift); }

}  // namespace quad
