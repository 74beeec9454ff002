// Measured arithmetic peaks used as roofline denominators: a dependent-chain
// FMA kernel (8 independent chains per thread, 4 CTAs of 256 threads per SM)
// timed with CUDA events.  FP64 and FP32 FMA (SIMT) rates on this GPU.
#include "common.cuh"

namespace {

template <typename T>
__global__ void __launch_bounds__(256) k_fma_peak(T *out, int iters, T a, T b) {
	T x0 = a + threadIdx.x, x1 = x0 + T(1), x2 = x0 + T(2), x3 = x0 + T(3);
	T x4 = x0 + T(4), x5 = x0 + T(5), x6 = x0 + T(6), x7 = x0 + T(7);
	for (int i = 0; i < iters; i++) {
#pragma unroll
		for (int u = 0; u < 16; u++) {
			x0 = fma(x0, b, a); x1 = fma(x1, b, a); x2 = fma(x2, b, a); x3 = fma(x3, b, a);
			x4 = fma(x4, b, a); x5 = fma(x5, b, a); x6 = fma(x6, b, a); x7 = fma(x7, b, a);
		}
	}
	T s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
	if (s == T(-12345)) out[threadIdx.x] = s;  // keeps the chains alive
}

template <typename T>
double run(int iters) {
	int sms = bf::num_sms();
	T *out = nullptr;
	if (cudaMalloc(&out, 256 * sizeof(T)) != cudaSuccess) return -1.0;
	dim3 grid(sms * 4);
	k_fma_peak<T><<<grid, 256>>>(out, 8, T(0.5), T(0.999));
	cudaEvent_t e0, e1;
	cudaEventCreate(&e0);
	cudaEventCreate(&e1);
	cudaEventRecord(e0);
	k_fma_peak<T><<<grid, 256>>>(out, iters, T(0.5), T(0.999));
	cudaEventRecord(e1);
	cudaEventSynchronize(e1);
	float ms = 0.f;
	cudaEventElapsedTime(&ms, e0, e1);
	cudaEventDestroy(e0);
	cudaEventDestroy(e1);
	cudaFree(out);
	double flops = 2.0 * 8 * 16 * (double)iters * grid.x * 256;
	return flops / (ms * 1e-3) / 1e9;
}

}  // namespace

extern "C" {

/* FMA throughput in GFLOP/s of the current device: prec 'd' (FP64) or 's' (FP32).
 * Returns a negative value on failure. */
double blasfeo_b200_measure_fma_peak(char prec, int iters) {
	if (iters <= 0) iters = 4096;
	double r = (prec == 's') ? run<float>(iters) : run<double>(iters);
	if (cudaGetLastError() != cudaSuccess) return -1.0;
	return r;
}

}  // extern "C"

