// Level-3 (and the level-2 pieces the solve chains need) on panel-major
// device matrices: gemm_nt, syrk_ln, trsm_rltn, trmm_rlnn, gemv_n, trsv_lnn,
// trsv_ltn.  Single-instance, uniform-batch and variable-size-batch entry
// points share one kernel per routine.
//
// gemm_nt / syrk_ln (blasfeo_hp_pm/d_blas3_lib4.c:727, :5400): D = beta*C +
// alpha*A*B^T, syrk writing only the lower triangle.  One CTA computes a BMxBN
// output tile of one instance; K is walked in BK-deep slices staged in shared
// memory (coalesced loads: a 4-row panel slice is one contiguous run), each
// thread accumulates a TMxTN register tile.  C is read only when beta != 0
// (as the HP AVX2 kernels do).
#include "common.cuh"
#include "kernels.cuh"

namespace {

template <typename T, int BM, int BN, int BK, int TM, int TN, bool LOWER>
__global__ void __launch_bounds__((BM / TM) * (BN / TN))
k_gemm_nt(SizeArg sz, T alpha, MatArg<T> A, MatArg<T> B, T beta, MatArg<T> C, MatArg<T> D, int tiles_n) {
	constexpr int NT = (BM / TM) * (BN / TN);
	constexpr int PADA = 16 / sizeof(T) * 2;  // keeps 16-byte alignment, staggers banks
	__shared__ __align__(16) T sA[BK][BM + PADA];
	__shared__ __align__(16) T sB[BK][BN + PADA];

	// grid.x = instance (up to 2^31-1 instances), grid.y = output tile
	const int b = blockIdx.x;
	const int m = sz.M(b), n = sz.N(b), k = sz.K(b);
	const int tmi = blockIdx.y / tiles_n, tni = blockIdx.y % tiles_n;
	const int i0 = tmi * BM, j0 = tni * BN;
	if (i0 >= m || j0 >= n) return;
	if (LOWER && j0 > i0 + BM - 1) return;
	const PMat<T> a = A.get(b), bm = B.get(b), c = C.get(b), d = D.get(b);

	const int tid = threadIdx.x;
	const int tx = tid % (BN / TN), ty = tid / (BN / TN);
	T acc[TM][TN];
#pragma unroll
	for (int r = 0; r < TM; r++)
#pragma unroll
		for (int q = 0; q < TN; q++) acc[r][q] = T(0);

	for (int k0 = 0; k0 < k; k0 += BK) {
		// element e of the slice -> (row, col): 4 consecutive e are the 4 rows of
		// one panel column, so consecutive threads read consecutive addresses
		for (int e = tid; e < BM * BK; e += NT) {
			int p = e / (4 * BK), rem = e % (4 * BK);
			int kk = rem >> 2, r = p * 4 + (rem & 3);
			int gi = i0 + r, gk = k0 + kk;
			sA[kk][r] = (gi < m && gk < k) ? a.at(gi, gk) : T(0);
		}
		for (int e = tid; e < BN * BK; e += NT) {
			int p = e / (4 * BK), rem = e % (4 * BK);
			int kk = rem >> 2, r = p * 4 + (rem & 3);
			int gj = j0 + r, gk = k0 + kk;
			sB[kk][r] = (gj < n && gk < k) ? bm.at(gj, gk) : T(0);
		}
		__syncthreads();
#pragma unroll 4
		for (int kk = 0; kk < BK; kk++) {
			T av[TM], bv[TN];
#pragma unroll
			for (int r = 0; r < TM; r++) av[r] = sA[kk][ty * TM + r];
#pragma unroll
			for (int q = 0; q < TN; q++) bv[q] = sB[kk][tx * TN + q];
#pragma unroll
			for (int r = 0; r < TM; r++)
#pragma unroll
				for (int q = 0; q < TN; q++) acc[r][q] = fma(av[r], bv[q], acc[r][q]);
		}
		__syncthreads();
	}
#pragma unroll
	for (int r = 0; r < TM; r++) {
		int gi = i0 + ty * TM + r;
		if (gi >= m) continue;
#pragma unroll
		for (int q = 0; q < TN; q++) {
			int gj = j0 + tx * TN + q;
			if (gj >= n) continue;
			if (LOWER && gj > gi) continue;
			T v = alpha * acc[r][q];
			if (beta != T(0)) v = fma(beta, c.at(gi, gj), v);
			d.at(gi, gj) = v;
		}
	}
}

template <typename T, int BM, int BN, int BK, int TM, int TN, bool LOWER>
int launch_gemm_cfg(int batch, SizeArg sz, int max_m, int max_n, T alpha, MatArg<T> A, MatArg<T> B, T beta,
                    MatArg<T> C, MatArg<T> D, cudaStream_t s) {
	int tm = cdiv(max_m, BM), tn = cdiv(max_n, BN);
	dim3 grid(batch, tm * tn);
	k_gemm_nt<T, BM, BN, BK, TM, TN, LOWER><<<grid, (BM / TM) * (BN / TN), 0, s>>>(sz, alpha, A, B, beta, C, D, tn);
	return bf::check_launch();
}

}  // namespace

namespace bf {

template <typename T, bool LOWER>
int gemm_nt_launch(int batch, SizeArg sz, int max_m, int max_n, int max_k, T alpha, MatArg<T> A, MatArg<T> B,
                   T beta, MatArg<T> C, MatArg<T> D, cudaStream_t s, int variant) {
	if (batch <= 0 || max_m <= 0 || max_n <= 0) return BLASFEO_B200_OK;
	const int mx = max_m > max_n ? max_m : max_n;
	if (variant < 0) {
		if (sizeof(T) == 8)  // FP64 tensor cores: 64x64 tiles once the batch fills the GPU
			variant = (mx > 32 && (long long)batch * cdiv(max_m, 64) * cdiv(max_n, 64) >= 2 * num_sms()) ? 4 : 5;
		else
			variant = mx > 48 ? 2 : (mx > 16 ? 1 : 0);
	}
	(void)max_k;
	if constexpr (sizeof(T) == 8) {
		if (variant == 4 || variant == 5)
			return dgemm_nt_dmma_launch<LOWER>(batch, sz, max_m, max_n, alpha, A, B, beta, C, D, s, variant - 4);
	}
	switch (variant) {
	case 0: return launch_gemm_cfg<T, 16, 16, 16, 2, 2, LOWER>(batch, sz, max_m, max_n, alpha, A, B, beta, C, D, s);
	case 1: return launch_gemm_cfg<T, 32, 32, 16, 2, 2, LOWER>(batch, sz, max_m, max_n, alpha, A, B, beta, C, D, s);
	case 2: return launch_gemm_cfg<T, 64, 64, 16, 4, 4, LOWER>(batch, sz, max_m, max_n, alpha, A, B, beta, C, D, s);
	default: return launch_gemm_cfg<T, 32, 32, 16, 4, 4, LOWER>(batch, sz, max_m, max_n, alpha, A, B, beta, C, D, s);
	}
}
template int gemm_nt_launch<double, false>(int, SizeArg, int, int, int, double, MatArg<double>, MatArg<double>, double,
                                           MatArg<double>, MatArg<double>, cudaStream_t, int);
template int gemm_nt_launch<double, true>(int, SizeArg, int, int, int, double, MatArg<double>, MatArg<double>, double,
                                          MatArg<double>, MatArg<double>, cudaStream_t, int);
template int gemm_nt_launch<float, false>(int, SizeArg, int, int, int, float, MatArg<float>, MatArg<float>, float,
                                          MatArg<float>, MatArg<float>, cudaStream_t, int);
template int gemm_nt_launch<float, true>(int, SizeArg, int, int, int, float, MatArg<float>, MatArg<float>, float,
                                         MatArg<float>, MatArg<float>, cudaStream_t, int);

}  // namespace bf

namespace {

// dA[l] = 1 / A(l,l): the inverse diagonal trsm_rltn multiplies by
// (blasfeo_hp_pm/d_blas3_lib4.c:4162-4178)
template <typename T>
__global__ void k_invdiag(SizeArg sz, MatArg<T> A) {
	int b = blockIdx.x;
	int n = sz.N(b);
	int l = blockIdx.y * blockDim.x + threadIdx.x;
	if (l >= n) return;
	PMat<T> a = A.get(b);
	a.d[l] = T(1) / a.at(l, l);
}

// D = alpha * B * A^{-T}, A lower (trsm_rltn non-unit: each column is
// multiplied by the cached inverse diagonal, kernel/generic/
// kernel_dgemm_4x4_lib4.c:5970 kernel_dtrsm_nt_rl_inv; trsm_rltu unit: the
// diagonal of A is taken as 1 and never read, blasfeo_ref/x_blas3_ref.c:1760).
// Element (i,k) is d_ik = (alpha b_ik - sum_{l<k} d_il a_kl) * inv_k with the
// sum accumulated in increasing l.
//
// For n <= NMAX (16, 32, 64): the lower triangle of A and its
// inverse diagonal are staged in shared memory once per CTA, and each row of
// the right-hand side lives in registers, updated right-looking (after d_ij:
// c_ik -= d_ij a_kj for k > j, A's column j read by every thread at once).
// TPR threads share a row (columns interleaved, k = TPR q + h), so a row of 64
// doubles fits in registers; the thread that owns column j passes d_ij to its
// partner by a shuffle within the pair.  Element (i,k) sees alpha b_ik, then
// the FMAs over l = 0..k-1 in order; nothing is re-read from global memory
// inside the recurrence.  64 rows per CTA, blockDim.x = 64 TPR.
template <typename T, bool UNIT, int NMAX, int TPR>
__global__ void __launch_bounds__(64 * TPR) k_trsm_rltn_reg(SizeArg sz, T alpha, MatArg<T> A, MatArg<T> B,
                                                             MatArg<T> D) {
	constexpr int NQ = NMAX / TPR;
	__shared__ T sa[NMAX * NMAX];  // sa[j * NMAX + k] = a(k, j), k > j
	__shared__ T sinv[NMAX];
	const int b = blockIdx.x;
	const int m = sz.M(b), n = sz.N(b);
	const PMat<T> a = A.get(b), bb = B.get(b), d = D.get(b);
	{
		// thread t stages row t % 64 of the columns j = t / 64 (mod TPR); the
		// loop is unrolled so every load is in flight at once
		const int k = threadIdx.x & 63, j0 = threadIdx.x >> 6;
#pragma unroll
		for (int jj = 0; jj < NQ; jj++) {
			const int j = jj * TPR + j0;
			if (j < n && k < n && k > j) sa[j * NMAX + k] = a.at(k, j);
		}
		if (!UNIT && threadIdx.x < n) sinv[threadIdx.x] = a.d[threadIdx.x];
	}
	__syncthreads();
	const int h = threadIdx.x % TPR;
	const int i = blockIdx.y * 64 + threadIdx.x / TPR;
	if (i >= m) return;  // both threads of a pair leave together
	const int lane = threadIdx.x & 31;
	const unsigned pair = (TPR == 1) ? (1u << lane) : (3u << (lane & ~1));
	T c[NQ];
#pragma unroll
	for (int q = 0; q < NQ; q++) {
		const int k = q * TPR + h;
		c[q] = (k < n) ? alpha * bb.at(i, k) : T(0);
	}
#pragma unroll
	for (int j = 0; j < NMAX; j++) {
		if (j >= n) break;
		const int qj = j / TPR, hj = j % TPR;
		T dj = T(0);
		if (h == hj) dj = UNIT ? c[qj] : c[qj] * sinv[j];
		if (TPR > 1) dj = __shfl_sync(pair, dj, (lane & ~(TPR - 1)) | hj);
		if (h == hj) c[qj] = dj;
#pragma unroll
		for (int q = 0; q < NQ; q++) {
			const int k = q * TPR + h;
			if (k > j && k < n) c[q] = fma(-dj, sa[j * NMAX + k], c[q]);
		}
	}
#pragma unroll
	for (int q = 0; q < NQ; q++) {
		const int k = q * TPR + h;
		if (k < n) d.at(i, k) = c[q];
	}
}

// n > 64: the same register solve by column blocks of 64.  Block J
// (columns c0 = 64 J ..) first receives the contributions of the solved
// columns l < c0, -sum_l d_il a_kl, from chunks of 64 columns of A staged in
// shared memory (d_il re-read from D, where the row's threads wrote it), then
// runs the in-block recurrence of k_trsm_rltn_reg.  Element (i,k) again sees
// alpha b_ik followed by the FMAs over l = 0..k-1 in increasing l, as in
// k_trsm_rltn_reg.  Dynamic shared memory: two 64 x 64 blocks of
// A and 64 inverse-diagonal entries.
template <typename T, bool UNIT, int TPR>
__global__ void __launch_bounds__(64 * TPR) k_trsm_rltn_blk(SizeArg sz, T alpha, MatArg<T> A, MatArg<T> B,
                                                             MatArg<T> D) {
	constexpr int NB = 64, NQ = NB / TPR;
	extern __shared__ __align__(16) unsigned char trsm_smem[];
	T *sa = (T *)trsm_smem;      // sa[j * NB + k] = a(c0 + k, c0 + j), k > j
	T *sg = sa + NB * NB;        // sg[l * NB + k] = a(c0 + k, l0 + l)
	T *sinv = sg + NB * NB;
	const int b = blockIdx.x;
	const int m = sz.M(b), n = sz.N(b);
	const PMat<T> a = A.get(b), bb = B.get(b), d = D.get(b);
	const int tid = threadIdx.x, nt = blockDim.x;
	const int h = tid % TPR;
	const int i = blockIdx.y * 64 + tid / TPR;
	const bool row = i < m;
	const int lane = tid & 31;
	const unsigned pair = (TPR == 1) ? (1u << lane) : (3u << (lane & ~1));
	for (int c0 = 0; c0 < n; c0 += NB) {
		const int nb = n - c0 < NB ? n - c0 : NB;
		T c[NQ];
#pragma unroll
		for (int q = 0; q < NQ; q++) {
			const int k = q * TPR + h;
			c[q] = (row && k < nb) ? alpha * bb.at(i, c0 + k) : T(0);
		}
		for (int l0 = 0; l0 < c0; l0 += NB) {
			__syncthreads();
			for (int e = tid; e < NB * NB; e += nt) {
				const int k = e & (NB - 1), l = e / NB;
				sg[l * NB + k] = (k < nb) ? a.at(c0 + k, l0 + l) : T(0);
			}
			__syncthreads();
			if (row) {
#pragma unroll 4
				for (int l = 0; l < NB; l++) {
					const T dl = d.at(i, l0 + l);
#pragma unroll
					for (int q = 0; q < NQ; q++) c[q] = fma(-dl, sg[l * NB + q * TPR + h], c[q]);
				}
			}
		}
		__syncthreads();
		for (int e = tid; e < NB * NB; e += nt) {
			const int k = e & (NB - 1), j = e / NB;
			if (j < nb && k < nb && k > j) sa[j * NB + k] = a.at(c0 + k, c0 + j);
		}
		if (!UNIT && tid < nb) sinv[tid] = a.d[c0 + tid];
		__syncthreads();
#pragma unroll
		for (int j = 0; j < NB; j++) {
			if (j >= nb) break;
			const int qj = j / TPR, hj = j % TPR;
			T dj = T(0);
			if (h == hj) dj = UNIT ? c[qj] : c[qj] * sinv[j];
			if (TPR > 1) dj = __shfl_sync(pair, dj, (lane & ~(TPR - 1)) | hj);
			if (h == hj) c[qj] = dj;
#pragma unroll
			for (int q = 0; q < NQ; q++) {
				const int k = q * TPR + h;
				if (k > j && k < nb) c[q] = fma(-dj, sa[j * NB + k], c[q]);
			}
		}
		if (row) {
#pragma unroll
			for (int q = 0; q < NQ; q++) {
				const int k = q * TPR + h;
				if (k < nb) d.at(i, c0 + k) = c[q];
			}
		}
		__syncwarp();  // the row's other thread reads these columns in the next block
	}
}

// Few rows (a single instance of config-1 size): one warp per row of D, 8
// rows per CTA, so the rows' serial chains run on several SMs at once.  A's
// lower triangle and inverse diagonal are staged in shared memory per CTA;
// lane l holds the columns k = 2l, 2l + 1 of its row in registers; step j:
// the owner lane finishes d_ij, a shuffle hands it to the warp, every lane
// updates its columns k > j (same operations in the same order as
// k_trsm_rltn_reg).  n <= 64.
template <typename T, bool UNIT>
__global__ void __launch_bounds__(256) k_trsm_rltn_row(SizeArg sz, T alpha, MatArg<T> A, MatArg<T> B, MatArg<T> D) {
	__shared__ T sa[64 * 64];  // sa[j * 64 + k] = a(k, j), k > j
	__shared__ T sinv[64];
	const int b = blockIdx.x;
	const int m = sz.M(b), n = sz.N(b);
	const PMat<T> a = A.get(b), bb = B.get(b), d = D.get(b);
	for (int e = threadIdx.x; e < 64 * 64; e += blockDim.x) {
		const int k = e & 63, j = e >> 6;
		if (j < n && k < n && k > j) sa[j * 64 + k] = a.at(k, j);
	}
	if (!UNIT && threadIdx.x < n) sinv[threadIdx.x] = a.d[threadIdx.x];
	__syncthreads();
	const int lane = threadIdx.x & 31;
	const int i = blockIdx.y * 8 + (threadIdx.x >> 5);
	if (i >= m) return;  // whole warps leave
	T c0 = (2 * lane < n) ? alpha * bb.at(i, 2 * lane) : T(0);
	T c1 = (2 * lane + 1 < n) ? alpha * bb.at(i, 2 * lane + 1) : T(0);
	for (int j = 0; j < n; j++) {
		const int owner = j >> 1;
		T dj = T(0);
		if (lane == owner) {
			const T cj = (j & 1) ? c1 : c0;
			dj = UNIT ? cj : cj * sinv[j];
			if (j & 1)
				c1 = dj;
			else
				c0 = dj;
		}
		dj = __shfl_sync(0xffffffffu, dj, owner);
		const int k0 = 2 * lane, k1 = 2 * lane + 1;
		if (k0 > j && k0 < n) c0 = fma(-dj, sa[j * 64 + k0], c0);
		if (k1 > j && k1 < n) c1 = fma(-dj, sa[j * 64 + k1], c1);
	}
	if (2 * lane < n) d.at(i, 2 * lane) = c0;
	if (2 * lane + 1 < n) d.at(i, 2 * lane + 1) = c1;
}

template <typename T, bool UNIT>
void trsm_rltn_kernel(int batch, SizeArg sz, int m, int n, T alpha, MatArg<T> A, MatArg<T> B, MatArg<T> D,
                      cudaStream_t s) {
	const dim3 grid(batch, cdiv(m, 64));
	// a row of 64 doubles takes two threads (registers); everything else one
	constexpr int TPR64 = sizeof(T) == 8 ? 2 : 1;
	if (n <= 64 && (long long)batch * cdiv(m, 64) * 4 <= bf::num_sms()) {
		// too few CTAs to fill the GPU with the 64-row kernel: a warp per row
		k_trsm_rltn_row<T, UNIT><<<dim3(batch, cdiv(m, 8)), 256, 0, s>>>(sz, alpha, A, B, D);
		return;
	}
	if (n <= 16)
		k_trsm_rltn_reg<T, UNIT, 16, 1><<<grid, 64, 0, s>>>(sz, alpha, A, B, D);
	else if (n <= 32)
		k_trsm_rltn_reg<T, UNIT, 32, 1><<<grid, 64, 0, s>>>(sz, alpha, A, B, D);
	else if (n <= 64)
		k_trsm_rltn_reg<T, UNIT, 64, TPR64><<<grid, 64 * TPR64, 0, s>>>(sz, alpha, A, B, D);
	else {
		const size_t smem = (2 * 64 * 64 + 64) * sizeof(T);
		auto kern = k_trsm_rltn_blk<T, UNIT, TPR64>;
		bf::smem_optin(kern, smem);
		kern<<<grid, 64 * TPR64, smem, s>>>(sz, alpha, A, B, D);
	}
}

// D = alpha * B * A, A lower non-unit (blasfeo_hp_pm/d_blas3_lib4.c:4893).
// D must not alias B.
template <typename T>
__global__ void k_trmm_rlnn(SizeArg sz, T alpha, MatArg<T> A, MatArg<T> B, MatArg<T> D) {
	int b = blockIdx.x;
	int m = sz.M(b), n = sz.N(b);
	long long idx = (long long)blockIdx.y * blockDim.x + threadIdx.x;
	if (idx >= (long long)m * n) return;
	int i = (int)(idx % m), j = (int)(idx / m);
	PMat<T> a = A.get(b), bb = B.get(b), d = D.get(b);
	T c = T(0);
	for (int l = j; l < n; l++) c = fma(bb.at(i, l), a.at(l, j), c);
	d.at(i, j) = alpha * c;
}

template <typename T>
__global__ void k_gemv_n(int m, int n, T alpha, PMat<T> a, const T *x, T beta, const T *y, T *z) {
	int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= m) return;
	T c = T(0);
	for (int l = 0; l < n; l++) c = fma(a.at(i, l), x[l], c);
	z[i] = alpha * c + beta * y[i];
}

// triangular solves with one warp: lane r owns rows r, r+32, ...; each step
// broadcasts the freshly solved unknown.
template <typename T, bool TRANS>
__global__ void k_trsv_l(int m, PMat<T> a, const T *x, T *z) {
	extern __shared__ __align__(16) unsigned char smem_raw[];
	T *w = (T *)smem_raw;
	int lane = threadIdx.x;
	for (int i = lane; i < m; i += 32) w[i] = x[i];
	__syncwarp();
	if (!TRANS) {
		for (int j = 0; j < m; j++) {
			T zj = w[j] * (T(1) / a.at(j, j));
			__syncwarp();
			for (int i = j + 1 + lane; i < m; i += 32) w[i] = fma(-a.at(i, j), zj, w[i]);
			if (lane == 0) w[j] = zj;
			__syncwarp();
		}
	} else {
		for (int j = m - 1; j >= 0; j--) {
			T zj = w[j] * (T(1) / a.at(j, j));
			__syncwarp();
			for (int i = lane; i < j; i += 32) w[i] = fma(-a.at(j, i), zj, w[i]);
			if (lane == 0) w[j] = zj;
			__syncwarp();
		}
	}
	for (int i = lane; i < m; i += 32) z[i] = w[i];
}

template <typename T>
int trsm_core(int batch, int m, int n, T alpha, MatArg<T> A, int ai, int aj, int *use_dA, MatArg<T> B, MatArg<T> D,
              cudaStream_t s, bool unit = false) {
	SizeArg sz = uniform_sizes(m, n, 0);
	if (unit) {
		trsm_rltn_kernel<T, true>(batch, sz, m, n, alpha, A, B, D, s);
		return bf::check_launch();
	}
	// inverse diagonal of A into A's dA, reused when already valid
	bool need = !(ai == 0 && aj == 0 && *use_dA >= n);
	if (need) {
		k_invdiag<T><<<dim3(batch, cdiv(n, 128)), 128, 0, s>>>(sz, A);
		*use_dA = (ai == 0 && aj == 0) ? n : 0;
	}
	trsm_rltn_kernel<T, false>(batch, sz, m, n, alpha, A, B, D, s);
	return bf::check_launch();
}

template <typename T, typename S>
void gemm_single(int m, int n, int k, T alpha, S *sA, int ai, int aj, S *sB, int bi, int bj, T beta, S *sC, int ci,
                 int cj, S *sD, int di, int dj, bool lower) {
	if (m <= 0 || n <= 0) return;
	sD->use_dA = 0;
	SizeArg sz = uniform_sizes(m, n, k);
	MatArg<T> A = single_arg<T>(sA, ai, aj), B = single_arg<T>(sB, bi, bj), C = single_arg<T>(sC, ci, cj),
	          D = single_arg<T>(sD, di, dj);
	if (lower)
		bf::gemm_nt_launch<T, true>(1, sz, m, n, k, alpha, A, B, beta, C, D, bf::cur_stream(), -1);
	else
		bf::gemm_nt_launch<T, false>(1, sz, m, n, k, alpha, A, B, beta, C, D, bf::cur_stream(), -1);
	bf::finish_single();
}

template <typename T, typename BT>
int gemm_batch(int batch, int m, int n, int k, T alpha, BT *sA, int ai, int aj, BT *sB, int bi, int bj, T beta,
               BT *sC, int ci, int cj, BT *sD, int di, int dj, void *stream, bool lower) {
	if (batch < 0 || !sA || !sB || !sC || !sD) return BLASFEO_B200_EINVAL;
	if (m <= 0 || n <= 0 || batch == 0) return BLASFEO_B200_OK;
	sD->use_dA = 0;
	SizeArg sz = uniform_sizes(m, n, k);
	MatArg<T> A = batch_arg<T>(sA, ai, aj), B = batch_arg<T>(sB, bi, bj), C = batch_arg<T>(sC, ci, cj),
	          D = batch_arg<T>(sD, di, dj);
	if (lower) return bf::gemm_nt_launch<T, true>(batch, sz, m, n, k, alpha, A, B, beta, C, D, (cudaStream_t)stream, -1);
	return bf::gemm_nt_launch<T, false>(batch, sz, m, n, k, alpha, A, B, beta, C, D, (cudaStream_t)stream, -1);
}

template <typename T, typename S>
void trsm_single(int m, int n, T alpha, S *sA, int ai, int aj, S *sB, int bi, int bj, S *sD, int di, int dj,
                 bool unit = false) {
	if (m <= 0 || n <= 0) return;
	sD->use_dA = 0;
	trsm_core<T>(1, m, n, alpha, single_arg<T>(sA, ai, aj), ai, aj, &sA->use_dA, single_arg<T>(sB, bi, bj),
	             single_arg<T>(sD, di, dj), bf::cur_stream(), unit);
	bf::finish_single();
}

template <typename T, typename BT>
int trsm_batch(int batch, int m, int n, T alpha, BT *sA, int ai, int aj, BT *sB, int bi, int bj, BT *sD, int di,
               int dj, void *stream, bool unit = false) {
	if (batch < 0 || !sA || !sB || !sD) return BLASFEO_B200_EINVAL;
	if (m <= 0 || n <= 0 || batch == 0) return BLASFEO_B200_OK;
	sD->use_dA = 0;
	return trsm_core<T>(batch, m, n, alpha, batch_arg<T>(sA, ai, aj), ai, aj, &sA->use_dA, batch_arg<T>(sB, bi, bj),
	                    batch_arg<T>(sD, di, dj), (cudaStream_t)stream, unit);
}

template <typename T, typename S>
void trmm_single(int m, int n, T alpha, S *sA, int ai, int aj, S *sB, int bi, int bj, S *sD, int di, int dj) {
	if (m <= 0 || n <= 0) return;
	sD->use_dA = 0;
	long long tot = (long long)m * n;
	k_trmm_rlnn<T><<<dim3(1, (unsigned)((tot + 127) / 128)), 128, 0, bf::cur_stream()>>>(
	    uniform_sizes(m, n, 0), alpha, single_arg<T>(sA, ai, aj), single_arg<T>(sB, bi, bj), single_arg<T>(sD, di, dj));
	bf::finish_single();
}

PMat<double> pm1(struct blasfeo_dmat *s, int ri, int cj) {
	PMat<double> p;
	p.p = s->pA;
	p.d = s->dA;
	p.cn = s->cn;
	p.ri = ri;
	p.cj = cj;
	return p;
}

}  // namespace

extern "C" {

void blasfeo_dgemm_nt(int m, int n, int k, double alpha, struct blasfeo_dmat *sA, int ai, int aj,
                      struct blasfeo_dmat *sB, int bi, int bj, double beta, struct blasfeo_dmat *sC, int ci, int cj,
                      struct blasfeo_dmat *sD, int di, int dj) {
	gemm_single<double>(m, n, k, alpha, sA, ai, aj, sB, bi, bj, beta, sC, ci, cj, sD, di, dj, false);
}
void blasfeo_dsyrk_ln(int m, int k, double alpha, struct blasfeo_dmat *sA, int ai, int aj, struct blasfeo_dmat *sB,
                      int bi, int bj, double beta, struct blasfeo_dmat *sC, int ci, int cj, struct blasfeo_dmat *sD,
                      int di, int dj) {
	gemm_single<double>(m, m, k, alpha, sA, ai, aj, sB, bi, bj, beta, sC, ci, cj, sD, di, dj, true);
}
void blasfeo_sgemm_nt(int m, int n, int k, float alpha, struct blasfeo_smat *sA, int ai, int aj,
                      struct blasfeo_smat *sB, int bi, int bj, float beta, struct blasfeo_smat *sC, int ci, int cj,
                      struct blasfeo_smat *sD, int di, int dj) {
	gemm_single<float>(m, n, k, alpha, sA, ai, aj, sB, bi, bj, beta, sC, ci, cj, sD, di, dj, false);
}
void blasfeo_ssyrk_ln(int m, int k, float alpha, struct blasfeo_smat *sA, int ai, int aj, struct blasfeo_smat *sB,
                      int bi, int bj, float beta, struct blasfeo_smat *sC, int ci, int cj, struct blasfeo_smat *sD,
                      int di, int dj) {
	gemm_single<float>(m, m, k, alpha, sA, ai, aj, sB, bi, bj, beta, sC, ci, cj, sD, di, dj, true);
}
void blasfeo_dtrsm_rltn(int m, int n, double alpha, struct blasfeo_dmat *sA, int ai, int aj, struct blasfeo_dmat *sB,
                        int bi, int bj, struct blasfeo_dmat *sD, int di, int dj) {
	trsm_single<double>(m, n, alpha, sA, ai, aj, sB, bi, bj, sD, di, dj);
}
void blasfeo_strsm_rltn(int m, int n, float alpha, struct blasfeo_smat *sA, int ai, int aj, struct blasfeo_smat *sB,
                        int bi, int bj, struct blasfeo_smat *sD, int di, int dj) {
	trsm_single<float>(m, n, alpha, sA, ai, aj, sB, bi, bj, sD, di, dj);
}
void blasfeo_dtrsm_rltu(int m, int n, double alpha, struct blasfeo_dmat *sA, int ai, int aj, struct blasfeo_dmat *sB,
                        int bi, int bj, struct blasfeo_dmat *sD, int di, int dj) {
	trsm_single<double>(m, n, alpha, sA, ai, aj, sB, bi, bj, sD, di, dj, true);
}
void blasfeo_strsm_rltu(int m, int n, float alpha, struct blasfeo_smat *sA, int ai, int aj, struct blasfeo_smat *sB,
                        int bi, int bj, struct blasfeo_smat *sD, int di, int dj) {
	trsm_single<float>(m, n, alpha, sA, ai, aj, sB, bi, bj, sD, di, dj, true);
}
// lower trapezoid (m x n, element (i,j) for j <= i) of D = beta*C + alpha*A*B^T
void blasfeo_dsyrk_ln_mn(int m, int n, int k, double alpha, struct blasfeo_dmat *sA, int ai, int aj,
                         struct blasfeo_dmat *sB, int bi, int bj, double beta, struct blasfeo_dmat *sC, int ci, int cj,
                         struct blasfeo_dmat *sD, int di, int dj) {
	gemm_single<double>(m, n, k, alpha, sA, ai, aj, sB, bi, bj, beta, sC, ci, cj, sD, di, dj, true);
}
void blasfeo_ssyrk_ln_mn(int m, int n, int k, float alpha, struct blasfeo_smat *sA, int ai, int aj,
                         struct blasfeo_smat *sB, int bi, int bj, float beta, struct blasfeo_smat *sC, int ci, int cj,
                         struct blasfeo_smat *sD, int di, int dj) {
	gemm_single<float>(m, n, k, alpha, sA, ai, aj, sB, bi, bj, beta, sC, ci, cj, sD, di, dj, true);
}
void blasfeo_dtrmm_rlnn(int m, int n, double alpha, struct blasfeo_dmat *sA, int ai, int aj, struct blasfeo_dmat *sB,
                        int bi, int bj, struct blasfeo_dmat *sD, int di, int dj) {
	trmm_single<double>(m, n, alpha, sA, ai, aj, sB, bi, bj, sD, di, dj);
}
void blasfeo_strmm_rlnn(int m, int n, float alpha, struct blasfeo_smat *sA, int ai, int aj, struct blasfeo_smat *sB,
                        int bi, int bj, struct blasfeo_smat *sD, int di, int dj) {
	trmm_single<float>(m, n, alpha, sA, ai, aj, sB, bi, bj, sD, di, dj);
}

void blasfeo_dgemv_n(int m, int n, double alpha, struct blasfeo_dmat *sA, int ai, int aj, struct blasfeo_dvec *sx,
                     int xi, double beta, struct blasfeo_dvec *sy, int yi, struct blasfeo_dvec *sz, int zi) {
	if (m <= 0) return;
	k_gemv_n<double><<<cdiv(m, 128), 128, 0, bf::cur_stream()>>>(m, n, alpha, pm1(sA, ai, aj), sx->pa + xi, beta,
	                                                              sy->pa + yi, sz->pa + zi);
	bf::finish_single();
}
void blasfeo_dtrsv_lnn(int m, struct blasfeo_dmat *sA, int ai, int aj, struct blasfeo_dvec *sx, int xi,
                       struct blasfeo_dvec *sz, int zi) {
	if (m <= 0) return;
	k_trsv_l<double, false><<<1, 32, m * sizeof(double), bf::cur_stream()>>>(m, pm1(sA, ai, aj), sx->pa + xi, sz->pa + zi);
	bf::finish_single();
}
void blasfeo_dtrsv_ltn(int m, struct blasfeo_dmat *sA, int ai, int aj, struct blasfeo_dvec *sx, int xi,
                       struct blasfeo_dvec *sz, int zi) {
	if (m <= 0) return;
	k_trsv_l<double, true><<<1, 32, m * sizeof(double), bf::cur_stream()>>>(m, pm1(sA, ai, aj), sx->pa + xi, sz->pa + zi);
	bf::finish_single();
}

int blasfeo_dgemm_nt_batch(int batch, int m, int n, int k, double alpha, struct blasfeo_dmat_batch *sA, int ai, int aj,
                           struct blasfeo_dmat_batch *sB, int bi, int bj, double beta, struct blasfeo_dmat_batch *sC,
                           int ci, int cj, struct blasfeo_dmat_batch *sD, int di, int dj, void *stream) {
	return gemm_batch<double>(batch, m, n, k, alpha, sA, ai, aj, sB, bi, bj, beta, sC, ci, cj, sD, di, dj, stream, false);
}
int blasfeo_dsyrk_ln_batch(int batch, int m, int k, double alpha, struct blasfeo_dmat_batch *sA, int ai, int aj,
                           struct blasfeo_dmat_batch *sB, int bi, int bj, double beta, struct blasfeo_dmat_batch *sC,
                           int ci, int cj, struct blasfeo_dmat_batch *sD, int di, int dj, void *stream) {
	return gemm_batch<double>(batch, m, m, k, alpha, sA, ai, aj, sB, bi, bj, beta, sC, ci, cj, sD, di, dj, stream, true);
}
int blasfeo_sgemm_nt_batch(int batch, int m, int n, int k, float alpha, struct blasfeo_smat_batch *sA, int ai, int aj,
                           struct blasfeo_smat_batch *sB, int bi, int bj, float beta, struct blasfeo_smat_batch *sC,
                           int ci, int cj, struct blasfeo_smat_batch *sD, int di, int dj, void *stream) {
	return gemm_batch<float>(batch, m, n, k, alpha, sA, ai, aj, sB, bi, bj, beta, sC, ci, cj, sD, di, dj, stream, false);
}
int blasfeo_ssyrk_ln_batch(int batch, int m, int k, float alpha, struct blasfeo_smat_batch *sA, int ai, int aj,
                           struct blasfeo_smat_batch *sB, int bi, int bj, float beta, struct blasfeo_smat_batch *sC,
                           int ci, int cj, struct blasfeo_smat_batch *sD, int di, int dj, void *stream) {
	return gemm_batch<float>(batch, m, m, k, alpha, sA, ai, aj, sB, bi, bj, beta, sC, ci, cj, sD, di, dj, stream, true);
}
int blasfeo_dtrsm_rltn_batch(int batch, int m, int n, double alpha, struct blasfeo_dmat_batch *sA, int ai, int aj,
                             struct blasfeo_dmat_batch *sB, int bi, int bj, struct blasfeo_dmat_batch *sD, int di,
                             int dj, void *stream) {
	return trsm_batch<double>(batch, m, n, alpha, sA, ai, aj, sB, bi, bj, sD, di, dj, stream);
}
int blasfeo_strsm_rltn_batch(int batch, int m, int n, float alpha, struct blasfeo_smat_batch *sA, int ai, int aj,
                             struct blasfeo_smat_batch *sB, int bi, int bj, struct blasfeo_smat_batch *sD, int di,
                             int dj, void *stream) {
	return trsm_batch<float>(batch, m, n, alpha, sA, ai, aj, sB, bi, bj, sD, di, dj, stream);
}

int blasfeo_dtrsm_rltu_batch(int batch, int m, int n, double alpha, struct blasfeo_dmat_batch *sA, int ai, int aj,
                             struct blasfeo_dmat_batch *sB, int bi, int bj, struct blasfeo_dmat_batch *sD, int di,
                             int dj, void *stream) {
	return trsm_batch<double>(batch, m, n, alpha, sA, ai, aj, sB, bi, bj, sD, di, dj, stream, true);
}
int blasfeo_strsm_rltu_batch(int batch, int m, int n, float alpha, struct blasfeo_smat_batch *sA, int ai, int aj,
                             struct blasfeo_smat_batch *sB, int bi, int bj, struct blasfeo_smat_batch *sD, int di,
                             int dj, void *stream) {
	return trsm_batch<float>(batch, m, n, alpha, sA, ai, aj, sB, bi, bj, sD, di, dj, stream, true);
}
int blasfeo_dsyrk_ln_mn_batch(int batch, int m, int n, int k, double alpha, struct blasfeo_dmat_batch *sA, int ai,
                              int aj, struct blasfeo_dmat_batch *sB, int bi, int bj, double beta,
                              struct blasfeo_dmat_batch *sC, int ci, int cj, struct blasfeo_dmat_batch *sD, int di,
                              int dj, void *stream) {
	return gemm_batch<double>(batch, m, n, k, alpha, sA, ai, aj, sB, bi, bj, beta, sC, ci, cj, sD, di, dj, stream, true);
}
int blasfeo_ssyrk_ln_mn_batch(int batch, int m, int n, int k, float alpha, struct blasfeo_smat_batch *sA, int ai,
                              int aj, struct blasfeo_smat_batch *sB, int bi, int bj, float beta,
                              struct blasfeo_smat_batch *sC, int ci, int cj, struct blasfeo_smat_batch *sD, int di,
                              int dj, void *stream) {
	return gemm_batch<float>(batch, m, n, k, alpha, sA, ai, aj, sB, bi, bj, beta, sC, ci, cj, sD, di, dj, stream, true);
}

int blasfeo_dgemm_nt_vbatch_variant(int batch, const int *m, const int *n, const int *k, int max_m, int max_n,
                                    int max_k, double alpha, const struct blasfeo_dmat *sA, const struct blasfeo_dmat *sB,
                                    double beta, const struct blasfeo_dmat *sC, const struct blasfeo_dmat *sD,
                                    int variant, void *stream) {
	if (batch < 0 || !m || !n || !k || !sA || !sB || !sC || !sD) return BLASFEO_B200_EINVAL;
	if (variant > 5) return BLASFEO_B200_EINVAL;
	if (variant < 0 && batch > 0) variant = bf::dispatch_pick(0, batch, m, n, k, max_m, max_n, max_k, (cudaStream_t)stream);
	return bf::gemm_nt_launch<double, false>(batch, var_sizes(m, n, k), max_m, max_n, max_k, alpha,
	                                         vbatch_arg<double>(sA), vbatch_arg<double>(sB), beta,
	                                         vbatch_arg<double>(sC), vbatch_arg<double>(sD), (cudaStream_t)stream,
	                                         variant);
}
int blasfeo_dgemm_nt_vbatch(int batch, const int *m, const int *n, const int *k, int max_m, int max_n, int max_k,
                            double alpha, const struct blasfeo_dmat *sA, const struct blasfeo_dmat *sB, double beta,
                            const struct blasfeo_dmat *sC, const struct blasfeo_dmat *sD, void *stream) {
	return blasfeo_dgemm_nt_vbatch_variant(batch, m, n, k, max_m, max_n, max_k, alpha, sA, sB, beta, sC, sD, -1,
	                                       stream);
}

/* number of kernel variants of a routine: op 0 gemm_nt, 1 potrf_l, 2 getrf_rp, 3 geqrf */
int blasfeo_b200_num_variants(int op) {
	switch (op) {
	case 0: return 6;
	case 1: return 6;
	case 2: return 6;
	case 3: return 6;
	default: return 0;
	}
}

}  // extern "C"
