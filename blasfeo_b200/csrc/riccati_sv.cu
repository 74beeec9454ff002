// Batched Riccati solve (LQR forward/backward substitution), feedback gains,
// and the mixed-precision LQ solve: FP32 factorization + FP64 iterative
// refinement on the KKT residual.  One warp per problem; lane i owns entry i
// of the stage vectors (nu + nx <= 16).
//
// Problem (examples/example_d_riccati_recursion.c), stages k = 0..N-1 with
// [u;x]_k of size nu + nx, stage N with x_N only:
//   min sum_k 1/2 [u;x]_k^T RSQ_k [u;x]_k + rq_k^T [u;x]_k + 1/2 x_N^T Q_N x_N + q_N^T x_N
//   s.t. x_{k+1} = BAbt_k^T [u;x]_k + b_k
// KKT conditions (multipliers pi_k of the dynamics):
//   RSQ_k ux_k + rq_k + BAbt_k pi_k - [0; pi_{k-1}] = 0   (k < N; no pi_{-1})
//   Q_N x_N + q_N - pi_{N-1} = 0
//   BAbt_k^T ux_k + b_k - x_{k+1} = 0
//
// The solve follows d_back_ric_trs_libstr (:203-270) on the factors L_k of
// d_back_ric_trf_libstr (riccati.cu):
//   backward: Pb_k = Lxx_{k+1} Lxx_{k+1}^T b_k (dtrmv_ltn, dtrmv_lnn);
//             ux_k = rq_k + BAbt_k (Pb_k + x-part of ux_{k+1}) (dgemv_n);
//             ux_k <- L_k^{-1} ux_k over the first nu columns (dtrsv_lnn_mn;
//             the whole factor at k = 0, dtrsv_lnn);
//   forward:  pi_k = x-part of ux_{k+1}; u_k <- -u_k; ux_k <- L_k^{-T} ux_k over
//             the first nu columns (dtrsv_ltn_mn; dtrsv_ltn at k = 0);
//             x_{k+1} = BAbt_k^T ux_k + b_k (dgemv_t);
//             pi_k += Lxx_{k+1} Lxx_{k+1}^T x_{k+1}.
// The triangular solves multiply by 1/L_jj computed from L (the reference's
// dtrsv recomputes its inverse diagonal from the factor).
#include <math.h>

#include "common.cuh"

namespace {

constexpr int RV = 16;     // stage block size
constexpr int LD = 17;     // shared-memory row stride of a 16 x 16 block
constexpr int SV_WARPS = 8;
constexpr unsigned FULL = 0xffffffffu;

__device__ __forceinline__ int pmi(int i, int j, int cn) { return (i & ~3) * cn + 4 * j + (i & 3); }
__device__ __forceinline__ double shf(double v, int src) { return __shfl_sync(FULL, v, src); }

// rows 0..15, columns 0..ncol-1 of a panel-major block (panel stride cn) into
// a row-major shared block; the whole warp loads (two columns per step)
template <typename TS>
__device__ __forceinline__ void ld_block(double *M, const TS *g, int cn, int ncol, int lane) {
	const int r = lane & 15, h = lane >> 4;
	for (int l = h; l < ncol; l += 2) M[r * LD + l] = (double)g[pmi(r, l, cn)];
	__syncwarp();
}

// z_i = sum_{j<=i} M[o+i][o+j] x_{xo+j}, i < n; x in lanes xo.., z in lanes 0..n-1
__device__ __forceinline__ double trmv_lnn(const double *M, int o, int n, double x, int xo, int lane) {
	double z = 0.0;
	for (int j = 0; j < n; j++) {
		const double xj = shf(x, xo + j);
		if (lane < n && j <= lane) z = fma(M[(o + lane) * LD + o + j], xj, z);
	}
	return z;
}
// z_j = sum_{i>=j} M[o+i][o+j] x_i, j < n; x and z in lanes 0..n-1
__device__ __forceinline__ double trmv_ltn(const double *M, int o, int n, double x, int lane) {
	double z = 0.0;
	for (int i = 0; i < n; i++) {
		const double xi = shf(x, i);
		if (lane < n && i >= lane) z = fma(M[(o + i) * LD + o + lane], xi, z);
	}
	return z;
}
// forward substitution over the first n columns of the m x m lower block:
// lanes < n receive L^{-1} u, lanes n..m-1 u_i - L_i,0:n z
__device__ __forceinline__ double trsv_lnn_mn(const double *M, int m, int n, double u, int lane) {
	for (int j = 0; j < n; j++) {
		const double zj = shf(u, j) * (1.0 / M[j * LD + j]);
		if (lane == j) u = zj;
		if (lane > j && lane < m) u = fma(-M[lane * LD + j], zj, u);
	}
	return u;
}
// backward substitution with L^T over the first n columns: entries n..m-1 are
// known; lanes < n receive (u_i - sum_{l>i} L_li z_l) / L_ii
__device__ __forceinline__ double trsv_ltn_mn(const double *M, int m, int n, double u, int lane) {
	for (int l = m - 1; l >= n; l--) {
		const double zl = shf(u, l);
		if (lane < n) u = fma(-M[l * LD + lane], zl, u);
	}
	for (int i = n - 1; i >= 0; i--) {
		const double zi = shf(u, i) * (1.0 / M[i * LD + i]);
		if (lane == i) u = zi;
		if (lane < i) u = fma(-M[i * LD + lane], zi, u);
	}
	return u;
}

struct SvArgs {
	int batch, N, nx, nu;
	const double *BA;  // BAbt_k, FP64 panel-major 16 x nx, problem p stage k at BA + sba*(p*N + k)
	long long sba;
	int cnba;
	const void *L;     // factors (16 x 16 panel-major, double or float), p*(N+1) + k
	long long sl;
	const double *b;   // b_k (nx), p*N + k
	long long sb;
	const double *rq;  // rq_k (nu + nx; stage N: nx), p*(N+1) + k
	long long srq;
	double *ux;        // [u;x]_k (stage N: x_N), p*(N+1) + k
	long long sux;
	double *pi;        // pi_k (nx), p*N + k
	long long spi;
};

// per-warp shared memory: two factor blocks and one BAbt block
constexpr int SV_WARP_DBL = 3 * RV * LD;

// The Riccati solve of problem p (whole warp).
template <typename TL>
__device__ void ric_trs_one(const SvArgs &a, long long p, double *sm, int lane) {
	const int N = a.N, nx = a.nx, nu = a.nu, M = nu + nx;
	double *Lk = sm, *Lk1 = sm + RV * LD, *BAs = sm + 2 * RV * LD;
	const TL *L = (const TL *)a.L;
	// ---- backward substitution ----
	double vn = (lane < nx) ? a.rq[a.srq * (p * (N + 1) + N) + lane] : 0.0;  // ux_N
	if (lane < nx) a.ux[a.sux * (p * (N + 1) + N) + lane] = vn;
	ld_block(Lk1, L + a.sl * (p * (N + 1) + N), RV, RV, lane);
	for (int k = N - 1; k >= 0; k--) {
		const int o1 = (k + 1 == N) ? 0 : nu;
		const double bk = (lane < nx) ? a.b[a.sb * (p * N + k) + lane] : 0.0;
		const double t = trmv_ltn(Lk1, o1, nx, bk, lane);
		const double pb = trmv_lnn(Lk1, o1, nx, t, 0, lane);
		const double xn = shf(vn, (o1 + lane) & 31);
		const double w = (lane < nx) ? pb + xn : 0.0;
		ld_block(BAs, a.BA + a.sba * (p * N + k), a.cnba, nx, lane);
		double u = (lane < M) ? a.rq[a.srq * (p * (N + 1) + k) + lane] : 0.0;
		for (int j = 0; j < nx; j++) {
			const double wj = shf(w, j);
			if (lane < M) u = fma(BAs[lane * LD + j], wj, u);
		}
		ld_block(Lk, L + a.sl * (p * (N + 1) + k), RV, RV, lane);
		u = trsv_lnn_mn(Lk, M, k > 0 ? nu : M, u, lane);
		if (lane < M) a.ux[a.sux * (p * (N + 1) + k) + lane] = u;
		vn = u;
		double *tmp = Lk;
		Lk = Lk1;
		Lk1 = tmp;
		__syncwarp();
	}
	// ---- forward substitution ----
	// xk: the new x part of ux_k, in lanes nu..M-1 (k >= 1)
	double xk = 0.0;
	for (int k = 0; k < N; k++) {
		const int o1 = (k + 1 == N) ? 0 : nu;
		ld_block(Lk, L + a.sl * (p * (N + 1) + k), RV, RV, lane);
		double u = (lane < M) ? a.ux[a.sux * (p * (N + 1) + k) + lane] : 0.0;
		if (k == 0) {
			u = -u;
			u = trsv_ltn_mn(Lk, M, M, u, lane);
		} else {
			u = (lane < nu) ? -u : xk;
			u = trsv_ltn_mn(Lk, M, nu, u, lane);
		}
		if (lane < M) a.ux[a.sux * (p * (N + 1) + k) + lane] = u;
		double pk = (lane < nx) ? a.ux[a.sux * (p * (N + 1) + k + 1) + o1 + lane] : 0.0;
		ld_block(BAs, a.BA + a.sba * (p * N + k), a.cnba, nx, lane);
		double xn = (lane < nx) ? a.b[a.sb * (p * N + k) + lane] : 0.0;
		for (int i = 0; i < M; i++) {
			const double ui = shf(u, i);
			if (lane < nx) xn = fma(BAs[i * LD + lane], ui, xn);
		}
		ld_block(Lk1, L + a.sl * (p * (N + 1) + k + 1), RV, RV, lane);
		double w = trmv_ltn(Lk1, o1, nx, xn, lane);
		w = trmv_lnn(Lk1, o1, nx, w, 0, lane);
		if (lane < nx) a.pi[a.spi * (p * N + k) + lane] = pk + w;
		if (k + 1 == N) {
			if (lane < nx) a.ux[a.sux * (p * (N + 1) + N) + lane] = xn;
		}
		xk = shf(xn, (lane - nu) & 31);  // x_{k+1} moved to lanes nu..M-1
		__syncwarp();
	}
}

template <typename TL>
__global__ void __launch_bounds__(SV_WARPS * 32) k_ric_trs(SvArgs a) {
	extern __shared__ __align__(16) double sv_smem[];
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	double *sm = sv_smem + (size_t)warp * SV_WARP_DBL;
	const long long nw = (long long)gridDim.x * SV_WARPS;
	for (long long p = (long long)blockIdx.x * SV_WARPS + warp; p < a.batch; p += nw) ric_trs_one<TL>(a, p, sm, lane);
}

// K_k = -Luu^{-T} Lxu^T (nu x nx) from L_k: lane nu + j solves for column j
__global__ void __launch_bounds__(SV_WARPS * 32)
    k_ric_gains(int batch, int N, int nx, int nu, const double *pL, long long sl, double *pK, long long sk, int cnk) {
	extern __shared__ __align__(16) double sv_smem[];
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	double *Ls = sv_smem + (size_t)warp * RV * LD;
	const long long nw = (long long)gridDim.x * SV_WARPS;
	const long long total = (long long)batch * N;
	for (long long s = (long long)blockIdx.x * SV_WARPS + warp; s < total; s += nw) {
		const long long p = s / N, k = s % N;
		ld_block(Ls, pL + sl * (p * (N + 1) + k), RV, RV, lane);
		const int j = lane - nu;
		if (j >= 0 && j < nx) {
			double kc[RV];
#pragma unroll
			for (int i = RV - 1; i >= 0; i--) {
				double c = 0.0;
				if (i < nu) {
					c = -Ls[(nu + j) * LD + i];
#pragma unroll
					for (int l = i + 1; l < RV; l++)
						if (l < nu) c = fma(-Ls[l * LD + i], kc[l], c);
					c *= 1.0 / Ls[i * LD + i];
				}
				kc[i] = c;
			}
			double *g = pK + sk * s;
#pragma unroll
			for (int i = 0; i < RV; i++)
				if (i < nu) g[pmi(i, j, cnk)] = kc[i];
		}
		__syncwarp();
	}
}

// ---- mixed precision: FP32 factors, FP64 residual and correction ----

// 16 x ncol panel-major FP64 instances -> FP32 (same layout), whole slab
__global__ void k_slab_to_f32(long long n, const double *__restrict__ src, float *__restrict__ dst) {
	for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
		dst[i] = (float)src[i];
}

// KKT residual of problem p at (ux, pi) into rs (stationarity, stage k at
// rs + RV*(p*(N+1)+k)) and rd (dynamics, rd + RV*(p*N+k)); returns its max-norm
__device__ double kkt_residual(const SvArgs &a, const double *RSQ, long long srsq, const double *rq0,
                               const double *b0, double *rs, double *rd, long long p, double *sm, int lane) {
	const int N = a.N, nx = a.nx, nu = a.nu, M = nu + nx;
	double *Rs = sm, *BAs = sm + 2 * RV * LD;
	double nrm = 0.0;
	for (int k = 0; k <= N; k++) {
		const int m = (k == N) ? nx : M;
		const double u = (lane < m) ? a.ux[a.sux * (p * (N + 1) + k) + lane] : 0.0;
		ld_block(Rs, RSQ + srsq * (p * (N + 1) + k), RV, RV, lane);
		double r = (lane < m) ? rq0[a.srq * (p * (N + 1) + k) + lane] : 0.0;
		for (int j = 0; j < m; j++) {
			const double uj = shf(u, j);
			if (lane < m) r = fma((j <= lane) ? Rs[lane * LD + j] : Rs[j * LD + lane], uj, r);
		}
		if (k < N) {
			const double pk = (lane < nx) ? a.pi[a.spi * (p * N + k) + lane] : 0.0;
			ld_block(BAs, a.BA + a.sba * (p * N + k), a.cnba, nx, lane);
			for (int j = 0; j < nx; j++) {
				const double pj = shf(pk, j);
				if (lane < M) r = fma(BAs[lane * LD + j], pj, r);
			}
			// dynamics: BAbt_k^T ux_k + b_k - x_{k+1}
			const int o1 = (k + 1 == N) ? 0 : nu;
			double d = (lane < nx) ? b0[a.sb * (p * N + k) + lane] - a.ux[a.sux * (p * (N + 1) + k + 1) + o1 + lane] : 0.0;
			for (int i = 0; i < M; i++) {
				const double ui = shf(u, i);
				if (lane < nx) d = fma(BAs[i * LD + lane], ui, d);
			}
			if (lane < nx) rd[RV * (p * N + k) + lane] = d;
			nrm = fmax(nrm, fabs(d));
		}
		if (k > 0) {
			const int lo = (k == N) ? 0 : nu;  // x part of stage k
			const double pm1 = (lane < nx) ? a.pi[a.spi * (p * N + k - 1) + lane] : 0.0;
			const double sh = shf(pm1, (lane - lo) & 31);
			if (lane >= lo && lane < lo + nx) r -= sh;
		}
		if (lane < m) rs[RV * (p * (N + 1) + k) + lane] = r;
		nrm = fmax(nrm, (lane < m) ? fabs(r) : 0.0);
		__syncwarp();
	}
	for (int off = 16; off > 0; off >>= 1) nrm = fmax(nrm, __shfl_xor_sync(FULL, nrm, off));
	return nrm;
}

struct MixArgs {
	const double *RSQ;  // FP64 RSQ_k slab (16 x 16), p*(N+1) + k
	long long srsq;
	double *rs, *rd;    // residual scratch (RV doubles per stage, laid out like rq and b)
	double *dux, *dpi;  // correction scratch (RV doubles per stage, laid out like ux and pi)
	int max_iter;
	double tol;
	int *iters;
	double *res;
	int *info;
};

// z = 0; repeat: residual; stop at ||r|| <= tol ||rhs||; correction with the
// FP32 factors; z += correction
__global__ void __launch_bounds__(SV_WARPS * 32) k_ric_sv_refine(SvArgs a, MixArgs m) {
	extern __shared__ __align__(16) double sv_smem[];
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	double *sm = sv_smem + (size_t)warp * SV_WARP_DBL;
	const long long nw = (long long)gridDim.x * SV_WARPS;
	const int N = a.N, M = a.nu + a.nx;
	for (long long p = (long long)blockIdx.x * SV_WARPS + warp; p < a.batch; p += nw) {
		// ||rhs||_inf and z = 0
		double rn = 0.0;
		for (int k = 0; k <= N; k++) {
			const int mm = (k == N) ? a.nx : M;
			if (lane < mm) {
				rn = fmax(rn, fabs(a.rq[a.srq * (p * (N + 1) + k) + lane]));
				a.ux[a.sux * (p * (N + 1) + k) + lane] = 0.0;
			}
			if (k < N && lane < a.nx) {
				rn = fmax(rn, fabs(a.b[a.sb * (p * N + k) + lane]));
				a.pi[a.spi * (p * N + k) + lane] = 0.0;
			}
		}
		for (int off = 16; off > 0; off >>= 1) rn = fmax(rn, __shfl_xor_sync(FULL, rn, off));
		__syncwarp();
		int it = 0;
		double r = 0.0;
		bool conv = false;
		for (;;) {
			r = kkt_residual(a, m.RSQ, m.srsq, a.rq, a.b, m.rs, m.rd, p, sm, lane);
			if (r <= m.tol * rn) {
				conv = true;
				break;
			}
			if (it >= m.max_iter) break;
			// correction: the solve with rq <- rs, b <- rd into dux, dpi
			SvArgs c = a;
			c.rq = m.rs;
			c.srq = RV;
			c.b = m.rd;
			c.sb = RV;
			c.ux = m.dux;
			c.sux = RV;
			c.pi = m.dpi;
			c.spi = RV;
			ric_trs_one<float>(c, p, sm, lane);
			__syncwarp();
			for (int k = 0; k <= N; k++) {
				const int mm = (k == N) ? a.nx : M;
				if (lane < mm) a.ux[a.sux * (p * (N + 1) + k) + lane] += m.dux[RV * (p * (N + 1) + k) + lane];
				if (k < N && lane < a.nx) a.pi[a.spi * (p * N + k) + lane] += m.dpi[RV * (p * N + k) + lane];
			}
			__syncwarp();
			it++;
		}
		if (lane == 0) {
			if (m.iters) m.iters[p] = it;
			if (m.res) m.res[p] = rn > 0.0 ? r / rn : r;
			if (m.info && m.info[p] == 0 && !conv) m.info[p] = -1;
		}
	}
}

inline int grid_of(long long work, size_t smem, const void *kern) {
	bf::smem_optin(kern, smem);
	int per_sm = 0;
	cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, SV_WARPS * 32, smem);
	if (per_sm < 1) per_sm = 1;
	long long g = (long long)bf::num_sms() * per_sm;
	const long long need = (work + SV_WARPS - 1) / SV_WARPS;
	if (g > need) g = need;
	return (int)(g < 1 ? 1 : g);
}

template <typename BT>
bool slab_ok(const BT *s, int m, int n, long long count) {
	return s && s->pA && s->m == m && s->n == n && (long long)s->batch >= count;
}

int sv_check(int batch, int N, int nx, int nu, const struct blasfeo_dmat_batch *sBA, const double *b,
             const double *rq, const double *ux, const double *pi, long long sb, long long srq, long long sux,
             long long spi) {
	if (batch < 0 || N < 1 || nx < 1 || nu < 0) return BLASFEO_B200_EINVAL;
	if (nu + nx > RV) return BLASFEO_B200_ENOTSUP;
	if (!slab_ok(sBA, RV, nx, (long long)batch * N)) return BLASFEO_B200_EINVAL;
	if (!b || !rq || !ux || !pi || sb < nx || srq < nu + nx || sux < nu + nx || spi < nx) return BLASFEO_B200_EINVAL;
	return BLASFEO_B200_OK;
}

}  // namespace

extern "C" {

int blasfeo_dric_trs_batch(int batch, int N, int nx, int nu, struct blasfeo_dmat_batch *sBAbt,
                           struct blasfeo_dmat_batch *sL, const double *b, long long sb, const double *rq,
                           long long srq, double *ux, long long sux, double *pi, long long spi, void *stream) {
	int st = sv_check(batch, N, nx, nu, sBAbt, b, rq, ux, pi, sb, srq, sux, spi);
	if (st) return st;
	if (!slab_ok(sL, RV, RV, (long long)batch * (N + 1))) return BLASFEO_B200_EINVAL;
	if (batch == 0) return BLASFEO_B200_OK;
	SvArgs a{batch, N, nx, nu, sBAbt->pA, sBAbt->stride, sBAbt->cn, sL->pA, sL->stride, b, sb, rq, srq,
	         ux, sux, pi, spi};
	const size_t smem = (size_t)SV_WARP_DBL * SV_WARPS * sizeof(double);
	k_ric_trs<double><<<grid_of(batch, smem, (const void *)k_ric_trs<double>), SV_WARPS * 32, smem,
	                    (cudaStream_t)stream>>>(a);
	return bf::check_launch();
}

int blasfeo_dric_gains_batch(int batch, int N, int nx, int nu, struct blasfeo_dmat_batch *sL,
                             struct blasfeo_dmat_batch *sK, void *stream) {
	if (batch < 0 || N < 1 || nx < 1 || nu < 1) return BLASFEO_B200_EINVAL;
	if (nu + nx > RV) return BLASFEO_B200_ENOTSUP;
	if (!slab_ok(sL, RV, RV, (long long)batch * (N + 1)) || !slab_ok(sK, nu, nx, (long long)batch * N))
		return BLASFEO_B200_EINVAL;
	if (batch == 0) return BLASFEO_B200_OK;
	sK->use_dA = 0;
	const size_t smem = (size_t)RV * LD * SV_WARPS * sizeof(double);
	k_ric_gains<<<grid_of((long long)batch * N, smem, (const void *)k_ric_gains), SV_WARPS * 32, smem,
	              (cudaStream_t)stream>>>(batch, N, nx, nu, sL->pA, sL->stride, sK->pA, sK->stride, sK->cn);
	return bf::check_launch();
}

size_t blasfeo_dsric_sv_worksize(int batch, int N, int nx) {
	if (batch <= 0 || N < 1 || nx < 1) return 0;
	// FP32 copies of BAbt and RSQ and the FP32 factors (each slab 256-byte
	// aligned), then the residual and correction vectors
	auto r256 = [](size_t x) { return (x + 255) / 256 * 256; };
	const size_t f32 = r256(blasfeo_memsize_smat_batch(RV, nx, batch * N)) +
	                   2 * r256(blasfeo_memsize_smat_batch(RV, RV, batch * (N + 1)));
	const size_t vec = (size_t)batch * (2 * (N + 1) + 2 * N) * RV * sizeof(double);
	return f32 + vec;
}

int blasfeo_dsric_sv_batch(int batch, int N, int nx, int nu, struct blasfeo_dmat_batch *sBAbt,
                           struct blasfeo_dmat_batch *sRSQ, const double *b, long long sb, const double *rq,
                           long long srq, double *ux, long long sux, double *pi, long long spi, int max_iter,
                           double tol, int *iters, double *res, int *info, void *work, size_t work_bytes,
                           void *stream) {
	int st = sv_check(batch, N, nx, nu, sBAbt, b, rq, ux, pi, sb, srq, sux, spi);
	if (st) return st;
	if (!slab_ok(sRSQ, RV, RV, (long long)batch * (N + 1)) || max_iter < 0) return BLASFEO_B200_EINVAL;
	if (batch == 0) return BLASFEO_B200_OK;
	cudaStream_t s = (cudaStream_t)stream;
	const size_t need = blasfeo_dsric_sv_worksize(batch, N, nx);
	char *w = (char *)work;
	if (!w) {
		w = (char *)bf::workspace(need, s);
		if (!w) return BLASFEO_B200_ENOMEM;
	} else if (work_bytes < need) {
		return BLASFEO_B200_ENOMEM;
	}
	// FP32 slabs (same instance layout as the FP64 ones, FP32 elements)
	struct blasfeo_smat_batch fBA, fRSQ, fL;
	blasfeo_create_smat_batch(RV, nx, batch * N, &fBA, w);
	size_t off = (blasfeo_memsize_smat_batch(RV, nx, batch * N) + 255) / 256 * 256;
	blasfeo_create_smat_batch(RV, RV, batch * (N + 1), &fRSQ, w + off);
	off += (blasfeo_memsize_smat_batch(RV, RV, batch * (N + 1)) + 255) / 256 * 256;
	blasfeo_create_smat_batch(RV, RV, batch * (N + 1), &fL, w + off);
	off += (blasfeo_memsize_smat_batch(RV, RV, batch * (N + 1)) + 255) / 256 * 256;
	if (off > need) return BLASFEO_B200_ENOMEM;
	double *vec = (double *)(w + off);
	if (off + (size_t)batch * (2 * (N + 1) + 2 * N) * RV * sizeof(double) > need) return BLASFEO_B200_ENOMEM;
	if (fBA.stride != sBAbt->stride || fRSQ.stride != sRSQ->stride) return BLASFEO_B200_EINVAL;
	const int cg = bf::num_sms() * 8;
	k_slab_to_f32<<<cg, 256, 0, s>>>((long long)batch * N * sBAbt->stride, sBAbt->pA, fBA.pA);
	k_slab_to_f32<<<cg, 256, 0, s>>>((long long)batch * (N + 1) * sRSQ->stride, sRSQ->pA, fRSQ.pA);
	if (bf::check_launch()) return BLASFEO_B200_ECUDA;
	st = blasfeo_sric_trf_batch(batch, N, nx, nu, &fBA, &fRSQ, &fL, info, stream);
	if (st) return st;
	// info now holds the factorization's pivot report; keep it where it is non-zero
	SvArgs a{batch, N, nx, nu, sBAbt->pA, sBAbt->stride, sBAbt->cn, fL.pA, fL.stride, b, sb, rq, srq,
	         ux, sux, pi, spi};
	MixArgs m;
	m.RSQ = sRSQ->pA;
	m.srsq = sRSQ->stride;
	m.rs = vec;
	m.dux = vec + (size_t)batch * (N + 1) * RV;
	m.rd = m.dux + (size_t)batch * (N + 1) * RV;
	m.dpi = m.rd + (size_t)batch * N * RV;
	m.max_iter = max_iter;
	m.tol = tol;
	m.iters = iters;
	m.res = res;
	m.info = info;
	const size_t smem = (size_t)SV_WARP_DBL * SV_WARPS * sizeof(double);
	// the factorization's pivot report (info) is kept: refinement writes 0 / -1
	// only for problems whose factorization reported nothing
	k_ric_sv_refine<<<grid_of(batch, smem, (const void *)k_ric_sv_refine), SV_WARPS * 32, smem, s>>>(a, m);
	return bf::check_launch();
}

}  // extern "C"
