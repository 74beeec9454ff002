// Launchers shared between translation units.
#pragma once
#include "common.cuh"

namespace bf {

// D = beta*C + alpha*A*B^T (LOWER: lower triangle only); variant < 0 picks a tile by size
template <typename T, bool LOWER>
int gemm_nt_launch(int batch, SizeArg sz, int max_m, int max_n, int max_k, T alpha, MatArg<T> A, MatArg<T> B,
                   T beta, MatArg<T> C, MatArg<T> D, cudaStream_t s, int variant);

// FP64 tensor-core (DMMA) gemm_nt / syrk_ln; tile 0 = 64x64, 1 = 32x32 (gemm_dmma.cu)
template <bool LOWER>
int dgemm_nt_dmma_launch(int batch, SizeArg sz, int max_m, int max_n, double alpha, MatArg<double> A,
                         MatArg<double> B, double beta, MatArg<double> C, MatArg<double> D, cudaStream_t s, int tile);

// FP64 potrf_l for max_m <= 64, one warp per instance on the FP64 tensor cores (potrf_dmma.cu)
int dpotrf_dmma_launch(int batch, SizeArg sz, int max_m, MatArg<double> C, MatArg<double> D, int *info,
                       cudaStream_t s);

// FP64 potrf_l for min_n < n <= max_m beyond shared memory: one CTA per
// instance, left-looking panels with FP64 tensor-core updates (potrf_ll.cu)
int dpotrf_ll_max_n();
int dpotrf_ll_launch(int batch, SizeArg sz, int min_n, int max_m, MatArg<double> C, MatArg<double> D, int *info,
                     cudaStream_t s);

// D = chol(C) lower, inverse diagonal into D's dA, info (device, may be null)
template <typename T>
int potrf_launch(int batch, SizeArg sz, int max_m, MatArg<T> C, MatArg<T> D, int *info, cudaStream_t s,
                 int variant);

// learned dispatch (dispatch.cu): the installed cost model's variant for a
// launch of op (0 gemm_nt, 1 potrf_l, 2 getrf_rp, 3 geqrf) with device size
// arrays m, n, k (k may be null: n), or -1 for the built-in rule
int dispatch_pick(int op, int batch, const int *m, const int *n, const int *k, int max_m, int max_n, int max_k,
                  cudaStream_t s);

}  // namespace bf
