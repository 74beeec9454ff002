// Allocation-free entry point of the fused mixed-precision SPD solver.
//
// blasfeo_dsposv_l_vbatch needs a little device scratch (the size-sorted work
// list and the per-class counters).  It takes that scratch from the caller or,
// when the caller passes none, from a workspace the library allocates with
// cudaMalloc.  Some callers can do neither: embedded and real-time solvers in
// the BLASFEO tradition fix their memory once at start-up and must not
// allocate (or hit the device-wide synchronisation of cudaMalloc/cudaFree)
// inside their control loop, and they may not want to size and pass a
// workspace either.  This entry point serves them: its scratch is a
// fixed-size array in device global memory that the library owns
// statically, so the call itself allocates nothing.
//
// Limits and behaviour:
//   - at most BLASFEO_B200_NOALLOC_MAX_BATCH systems per call and n <= 256
//     per system; larger requests return BLASFEO_B200_ENOTSUP before any
//     device work;
//   - the array is loaded with the library and stays resident on every GPU
//     that uses the library until the process exits;
//   - the size classes run one after the other on the caller's stream (the
//     allocating entry point spreads them over a second stream that it
//     creates on a host thread's first call, which can take device memory);
//   - all calls share the one array: calls whose executions overlap on the
//     GPU (different streams, or different host threads) race on it and must
//     be serialised by the caller; one call's kernels reset the counters they
//     use, so consecutive calls need no clearing by the caller;
//   - the first call on a device looks up the device address of the array
//     (cudaGetSymbolAddress with that device current) and caches it; make that
//     first call on each device before any stream capture.  The cached address
//     belongs to the device's primary context: after cudaDeviceReset the
//     library's module is loaded again at another address, so a process that
//     resets a device must not call this entry point on it afterwards.
#include <mutex>

#include "common.cuh"
#include "posv.cuh"

namespace {

constexpr int kMaxBatch = BLASFEO_B200_NOALLOC_MAX_BATCH;
constexpr int kMaxN = 256;
// scratch of the fused solver for kMaxBatch systems: the work list (one int
// per system) followed by four 16-byte-aligned tables of POSV_MAX_CLASSES
// ints, the layout blasfeo_dposv_worksize(kMaxBatch) sizes
constexpr size_t kScratchBytes = posv_list_bytes((size_t)kMaxBatch);
static_assert(kScratchBytes == (size_t)kMaxBatch * sizeof(int) + 4 * posv_a16(POSV_MAX_CLASSES * sizeof(int)),
              "work list followed by four class tables");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

std::mutex g_mutex;
void *g_addr[64] = {nullptr};

// device address of g_noalloc_scratch on the current device (looked up once)
int scratch_address(void **out) {
	int dev = 0;
	if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return BLASFEO_B200_ECUDA;
	std::lock_guard<std::mutex> lock(g_mutex);
	if (!g_addr[dev]) {
		void *p = nullptr;
		if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) {
			cudaGetLastError();
			return BLASFEO_B200_ECUDA;
		}
		g_addr[dev] = p;
	}
	*out = g_addr[dev];
	return BLASFEO_B200_OK;
}

}  // namespace

extern "C" {

size_t blasfeo_dsposv_noalloc_scratch_bytes(void) { return kScratchBytes; }

int blasfeo_dsposv_l_vbatch_noalloc(int batch, const int *n, int max_n, const struct blasfeo_dmat *sA,
                                    const struct blasfeo_dvec *sb, const struct blasfeo_dvec *sx, int max_iter,
                                    double tol, int *iters, double *berr, int *info, void *stream) {
	if (batch < 0 || max_n < 0) return BLASFEO_B200_EINVAL;
	if (batch > kMaxBatch || max_n > kMaxN) return BLASFEO_B200_ENOTSUP;
	if (batch == 0 || max_n == 0) return BLASFEO_B200_OK;
	if (!n || !sA || !sb || !sx) return BLASFEO_B200_EINVAL;
	void *scratch = nullptr;
	int st = scratch_address(&scratch);
	if (st != BLASFEO_B200_OK) return st;
	// on the caller's stream only: the allocating entry point's second stream
	// is created on a host thread's first call
	return bf::dsposv_one_stream(batch, n, max_n, sA, sb, sx, max_iter, tol, iters, berr, info, scratch,
	                             kScratchBytes, (cudaStream_t)stream);
}

}  // extern "C"
