// Learned cost model: a small MLP (nin -> H -> H -> H -> 1, ReLU, FP32) that
// predicts the log run time of a batched launch for one kernel variant.  It
// is trained on the GPU by these kernels on the timings the autotuner
// collects, and only ever chooses among variants that compute identical
// results (it never touches numerics).
//
// Parameter layout (one flat FP32 array): W1 [nin x H], b1 [H], W2 [H x H],
// b2 [H], W3 [H x H], b3 [H], W4 [H x 1], b4 [1]; row-major, y = x W + b.
// Work buffer (per batch of B samples): Z1, A1, Z2, A2, Z3, A3 [B x H] each,
// y [B], plus the backward buffers dA, dZ [B x H].
#include "common.cuh"

namespace {

constexpr int TS = 32;  // tile of the small GEMM kernels

// C[M x N] = op(A) op(B) (+ bias) with op(X) = X or X^T; row-major with
// leading dimensions lda, ldb, ldc; optional ReLU output A_out = max(C, 0).
template <bool TA, bool TB>
__global__ void k_sgemm_small(int M, int N, int K, const float *__restrict__ A, int lda, const float *__restrict__ B,
                              int ldb, const float *__restrict__ bias, float *C, int ldc, float *relu_out,
                              float beta) {
	__shared__ float sA[TS][TS + 1];
	__shared__ float sB[TS][TS + 1];
	const int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8 threads, 4 rows each
	const int row0 = blockIdx.y * TS, col0 = blockIdx.x * TS;
	float acc[4] = {0.f, 0.f, 0.f, 0.f};
	for (int k0 = 0; k0 < K; k0 += TS) {
		for (int r = ty; r < TS; r += 8) {
			const int gi = row0 + r, gk = k0 + tx;
			sA[r][tx] = (gi < M && gk < K) ? (TA ? A[(size_t)gk * lda + gi] : A[(size_t)gi * lda + gk]) : 0.f;
			const int bk = k0 + r, bj = col0 + tx;
			sB[r][tx] = (bk < K && bj < N) ? (TB ? B[(size_t)bj * ldb + bk] : B[(size_t)bk * ldb + bj]) : 0.f;
		}
		__syncthreads();
#pragma unroll 8
		for (int kk = 0; kk < TS; kk++) {
			const float b = sB[kk][tx];
#pragma unroll
			for (int q = 0; q < 4; q++) acc[q] = fmaf(sA[ty + 8 * q][kk], b, acc[q]);
		}
		__syncthreads();
	}
#pragma unroll
	for (int q = 0; q < 4; q++) {
		const int gi = row0 + ty + 8 * q, gj = col0 + tx;
		if (gi < M && gj < N) {
			float v = acc[q] + (bias ? bias[gj] : 0.f);
			if (beta != 0.f) v += beta * C[(size_t)gi * ldc + gj];
			C[(size_t)gi * ldc + gj] = v;
			if (relu_out) relu_out[(size_t)gi * ldc + gj] = v > 0.f ? v : 0.f;
		}
	}
}

template <bool TA, bool TB>
void sgemm(int M, int N, int K, const float *A, int lda, const float *B, int ldb, const float *bias, float *C, int ldc,
           float *relu_out, float beta, cudaStream_t s) {
	dim3 grid(cdiv(N, TS), cdiv(M, TS)), block(32, 8);
	k_sgemm_small<TA, TB><<<grid, block, 0, s>>>(M, N, K, A, lda, B, ldb, bias, C, ldc, relu_out, beta);
}

// dy = 2 (y - t) / B; loss = mean (y - t)^2 (block reduction into *loss)
__global__ void k_mse(int B, const float *y, const float *t, float *dy, float *loss) {
	__shared__ float red[32];
	float part = 0.f;
	for (int i = threadIdx.x; i < B; i += blockDim.x) {
		const float d = y[i] - t[i];
		dy[i] = 2.f * d / (float)B;
		part += d * d;
	}
#pragma unroll
	for (int off = 16; off > 0; off >>= 1) part += __shfl_down_sync(0xffffffffu, part, off);
	if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = part;
	__syncthreads();
	if (threadIdx.x == 0) {
		float s = 0.f;
		for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += red[w];
		*loss = s / (float)B;
	}
}

// dZ = dA * (Z > 0)
__global__ void k_relu_bwd(int n, const float *dA, const float *Z, float *dZ) {
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n) dZ[i] = Z[i] > 0.f ? dA[i] : 0.f;
}

// db[j] = sum_b dZ[b][j]
__global__ void k_colsum(int B, int N, const float *dZ, float *db) {
	const int j = blockIdx.x * blockDim.x + threadIdx.x;
	if (j >= N) return;
	float s = 0.f;
	for (int b = 0; b < B; b++) s += dZ[(size_t)b * N + j];
	db[j] = s;
}

// Adam (Kingma & Ba, 2015) with bias correction
__global__ void k_adam(int n, float *p, const float *g, float *m, float *v, float lr, float b1, float b2, float eps,
                       float c1, float c2) {
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	const float gi = g[i];
	const float mi = b1 * m[i] + (1.f - b1) * gi;
	const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
	m[i] = mi;
	v[i] = vi;
	p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

struct Net {
	int nin, H;
	const float *W1, *b1, *W2, *b2, *W3, *b3, *W4, *b4;
};
struct NetGrad {
	float *W1, *b1, *W2, *b2, *W3, *b3, *W4, *b4;
};

inline int param_count(int nin, int H) { return nin * H + H + 2 * (H * H + H) + H + 1; }

template <typename P, typename F>
P carve(F *base, int nin, int H) {
	P n;
	F *q = base;
	n.W1 = q; q += nin * H;
	n.b1 = q; q += H;
	n.W2 = q; q += H * H;
	n.b2 = q; q += H;
	n.W3 = q; q += H * H;
	n.b3 = q; q += H;
	n.W4 = q; q += H;
	n.b4 = q;
	return n;
}

struct Work {
	float *Z1, *A1, *Z2, *A2, *Z3, *A3, *y, *dy, *dA, *dZ, *loss;
};

inline size_t work_floats(int B, int H) { return (size_t)8 * B * H + 2 * (size_t)B + 32; }

Work carve_work(float *w, int B, int H) {
	Work k;
	const size_t bh = (size_t)B * H;
	k.Z1 = w; k.A1 = w + bh; k.Z2 = w + 2 * bh; k.A2 = w + 3 * bh; k.Z3 = w + 4 * bh; k.A3 = w + 5 * bh;
	k.dA = w + 6 * bh; k.dZ = w + 7 * bh;
	k.y = w + 8 * bh; k.dy = k.y + B; k.loss = k.dy + B;
	return k;
}

void forward(const Net &n, int B, const float *X, const Work &w, float *y, cudaStream_t s) {
	const int H = n.H;
	sgemm<false, false>(B, H, n.nin, X, n.nin, n.W1, H, n.b1, w.Z1, H, w.A1, 0.f, s);
	sgemm<false, false>(B, H, H, w.A1, H, n.W2, H, n.b2, w.Z2, H, w.A2, 0.f, s);
	sgemm<false, false>(B, H, H, w.A2, H, n.W3, H, n.b3, w.Z3, H, w.A3, 0.f, s);
	sgemm<false, false>(B, 1, H, w.A3, H, n.W4, 1, n.b4, y, 1, nullptr, 0.f, s);
}

// gradients of the mean squared error w.r.t. all parameters
void backward(const Net &n, const NetGrad &g, int B, const float *X, const Work &w, const float *t, cudaStream_t s) {
	const int H = n.H;
	k_mse<<<1, 256, 0, s>>>(B, w.y, t, w.dy, w.loss);
	// layer 4: y = A3 W4 + b4
	sgemm<true, false>(H, 1, B, w.A3, H, w.dy, 1, nullptr, g.W4, 1, nullptr, 0.f, s);
	k_colsum<<<1, 32, 0, s>>>(B, 1, w.dy, g.b4);
	sgemm<false, true>(B, H, 1, w.dy, 1, n.W4, 1, nullptr, w.dA, H, nullptr, 0.f, s);
	// layer 3
	k_relu_bwd<<<cdiv(B * H, 256), 256, 0, s>>>(B * H, w.dA, w.Z3, w.dZ);
	sgemm<true, false>(H, H, B, w.A2, H, w.dZ, H, nullptr, g.W3, H, nullptr, 0.f, s);
	k_colsum<<<cdiv(H, 128), 128, 0, s>>>(B, H, w.dZ, g.b3);
	sgemm<false, true>(B, H, H, w.dZ, H, n.W3, H, nullptr, w.dA, H, nullptr, 0.f, s);
	// layer 2
	k_relu_bwd<<<cdiv(B * H, 256), 256, 0, s>>>(B * H, w.dA, w.Z2, w.dZ);
	sgemm<true, false>(H, H, B, w.A1, H, w.dZ, H, nullptr, g.W2, H, nullptr, 0.f, s);
	k_colsum<<<cdiv(H, 128), 128, 0, s>>>(B, H, w.dZ, g.b2);
	sgemm<false, true>(B, H, H, w.dZ, H, n.W2, H, nullptr, w.dA, H, nullptr, 0.f, s);
	// layer 1
	k_relu_bwd<<<cdiv(B * H, 256), 256, 0, s>>>(B * H, w.dA, w.Z1, w.dZ);
	sgemm<true, false>(n.nin, H, B, X, n.nin, w.dZ, H, nullptr, g.W1, H, nullptr, 0.f, s);
	k_colsum<<<cdiv(H, 128), 128, 0, s>>>(B, H, w.dZ, g.b1);
}

}  // namespace

extern "C" {

int blasfeo_b200_mlp_param_count(int nin, int hidden) {
	return (nin <= 0 || hidden <= 0) ? -1 : param_count(nin, hidden);
}

size_t blasfeo_b200_mlp_work_bytes(int hidden, int batch) { return work_floats(batch, hidden) * sizeof(float); }

/* y[b] = net(X[b, :]) for b < batch; X row-major [batch x nin] (device) */
int blasfeo_b200_mlp_forward(int nin, int hidden, const float *params, int batch, const float *X, float *y,
                             float *work, void *stream) {
	if (nin <= 0 || hidden <= 0 || batch < 0 || !params || !X || !y || !work) return BLASFEO_B200_EINVAL;
	if (batch == 0) return BLASFEO_B200_OK;
	Net n = carve<Net, const float>(params, nin, hidden);
	n.nin = nin;
	n.H = hidden;
	Work w = carve_work(work, batch, hidden);
	forward(n, batch, X, w, y, (cudaStream_t)stream);
	return bf::check_launch();
}

/* loss (device scalar) and gradients (device, same layout as params) of the
 * mean squared error between net(X) and target */
int blasfeo_b200_mlp_grad(int nin, int hidden, const float *params, int batch, const float *X, const float *target,
                          float *grads, float *loss, float *work, void *stream) {
	if (nin <= 0 || hidden <= 0 || batch <= 0 || !params || !X || !target || !grads || !work) return BLASFEO_B200_EINVAL;
	cudaStream_t s = (cudaStream_t)stream;
	Net n = carve<Net, const float>(params, nin, hidden);
	n.nin = nin;
	n.H = hidden;
	NetGrad g = carve<NetGrad, float>(grads, nin, hidden);
	Work w = carve_work(work, batch, hidden);
	forward(n, batch, X, w, w.y, s);
	backward(n, g, batch, X, w, target, s);
	if (loss) cudaMemcpyAsync(loss, w.loss, sizeof(float), cudaMemcpyDeviceToDevice, s);
	return bf::check_launch();
}

/* one Adam step (step >= 1) on params with gradients grads */
int blasfeo_b200_mlp_adam(int nparams, float *params, const float *grads, float *m, float *v, int step, float lr,
                          void *stream) {
	if (nparams <= 0 || !params || !grads || !m || !v || step < 1) return BLASFEO_B200_EINVAL;
	const float b1 = 0.9f, b2 = 0.999f;
	const float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
	k_adam<<<cdiv(nparams, 256), 256, 0, (cudaStream_t)stream>>>(nparams, params, grads, m, v, lr, b1, b2, 1e-8f, c1,
	                                                              c2);
	return bf::check_launch();
}

}  // extern "C"
