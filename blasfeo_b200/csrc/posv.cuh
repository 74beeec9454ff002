// Work-list structures shared by the fused SPD solvers (posv.cu, posv_tc.cu).
#pragma once
#include "common.cuh"

constexpr int POSV_MAX_CLASSES = 12;

// bytes of the work list and class tables of one call of `batch` systems: the
// list (one int per system), then the start, count and claim-counter tables
// and a spare one, each 16-byte aligned
constexpr size_t posv_a16(size_t x) { return (x + 15) / 16 * 16; }
constexpr size_t posv_list_bytes(size_t batch) {
	return posv_a16(batch * sizeof(int)) + 4 * posv_a16(POSV_MAX_CLASSES * sizeof(int));
}

// engine of the mixed solver when the caller asks for the default: 1 = the
// tensor-core kernel (posv_tc.cu), 0 = the SIMT kernel (posv.cu)
#define POSV_TENSOR_DEFAULT 0

// size classes of one call: class c takes the systems with
// upper[c-1] < n <= upper[c] (upper ascending)
struct ClassTable {
	int nclass;
	int upper[POSV_MAX_CLASSES];
};

// workspace of one call: the size-sorted work list (batch ints) and, per
// class, the start in the list, the count and the claim counter
struct PosvWs {
	int *list;
	int *start;
	int *count;
	int *counter;
	int *hist;
};

namespace bf {

// Mixed-precision factor + solve on the tensor cores for the systems of size
// class `cls` (all n <= upper <= 256); see posv_tc.cu.
int posv_tc_launch(int cls, int upper, int batch, PosvWs ws, const int *n, const void *sA, const void *sb,
                   const void *sx, int max_iter, double tol, int *iters, double *berr, int *info, cudaStream_t s);

// The mixed solver on the caller's stream alone, with a caller-provided
// workspace (posv.cu): the path of the allocation-free entry point.
int dsposv_one_stream(int batch, const int *n, int max_n, const void *sA, const void *sb, const void *sx, int max_iter,
                      double tol, int *iters, double *berr, int *info, void *work, size_t work_bytes,
                      cudaStream_t stream);
}  // namespace bf
