// Library state: error recording, the stream of the single-instance entry
// points, the synchronous/asynchronous switch, and the library-owned device
// workspace used when a caller passes no workspace.
#include <atomic>
#include <vector>

#include "common.cuh"

namespace bf {

static thread_local int g_last_error = BLASFEO_B200_OK;
static thread_local cudaStream_t g_stream = nullptr;
static thread_local int g_sync = 1;
static thread_local int g_posv_engine = BLASFEO_B200_POSV_DEFAULT;
// polls of a bounded mbarrier wait in the kernels that use bulk copies (process-wide)
static std::atomic<unsigned int> g_wait_limit{1u << 24};

void set_error(int status) {
	if (status != BLASFEO_B200_OK) g_last_error = status;
}

int check_launch() {
	cudaError_t e = cudaGetLastError();
	if (e != cudaSuccess) {
		set_error(BLASFEO_B200_ECUDA);
		return BLASFEO_B200_ECUDA;
	}
	return BLASFEO_B200_OK;
}

cudaStream_t cur_stream() { return g_stream; }
int posv_engine() { return g_posv_engine; }
unsigned int wait_limit() { return g_wait_limit.load(std::memory_order_relaxed); }
bool sync_mode() { return g_sync != 0; }

int finish_single() {
	int st = check_launch();
	if (st == BLASFEO_B200_OK && g_sync) {
		if (cudaStreamSynchronize(g_stream) != cudaSuccess) {
			set_error(BLASFEO_B200_ECUDA);
			st = BLASFEO_B200_ECUDA;
		}
	}
	return st;
}

struct Workspace {
	void *ptr = nullptr;
	size_t bytes = 0;
	int dev = 0;
};
// One set per host thread, like the stream of the single-instance calls: two
// threads that work on their own streams never share scratch.  Per thread and
// device: [0] the general workspace, [1] the column-major staging buffer.
// Freed when the thread ends (at process exit the runtime may already be gone;
// the failed cudaFree is then harmless).
struct ThreadWorkspaces {
	std::vector<Workspace> slot[2];
	~ThreadWorkspaces() {
		int cur = 0;
		const bool have = cudaGetDevice(&cur) == cudaSuccess;
		for (auto &v : slot)
			for (auto &w : v)
				if (w.ptr) {
					cudaSetDevice(w.dev);
					cudaFree(w.ptr);
				}
		if (have) cudaSetDevice(cur);
		cudaGetLastError();
	}
};
static thread_local ThreadWorkspaces g_ws;

static void *workspace_slot(int slot, size_t bytes, cudaStream_t s) {
	int dev = 0;
	if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
	std::vector<Workspace> &v = g_ws.slot[slot];
	if ((int)v.size() <= dev) v.resize(dev + 1);
	Workspace &w = v[dev];
	w.dev = dev;
	if (w.bytes >= bytes && w.ptr) return w.ptr;
	// growing: wait for work that may still use the old buffer
	if (w.ptr) {
		cudaStreamSynchronize(s);
		cudaDeviceSynchronize();
		cudaFree(w.ptr);
		w.ptr = nullptr;
		w.bytes = 0;
	}
	size_t want = bytes < (size_t(1) << 20) ? (size_t(1) << 20) : bytes;
	want = (want + 4095) / 4096 * 4096;
	if (cudaMalloc(&w.ptr, want) != cudaSuccess) {
		cudaGetLastError();
		w.ptr = nullptr;
		return nullptr;
	}
	w.bytes = want;
	return w.ptr;
}

// A second stream and two events per host thread and device, for work a call
// forks off its stream and joins again (created on first use, released when
// the thread ends).
struct ThreadSide {
	struct Dev {
		cudaStream_t stream = nullptr;
		cudaEvent_t ev[2] = {nullptr, nullptr};
		bool failed = false;
	};
	std::vector<Dev> dev;
	~ThreadSide() {
		for (auto &d : dev) {
			for (auto &e : d.ev)
				if (e) cudaEventDestroy(e);
			if (d.stream) cudaStreamDestroy(d.stream);
		}
		cudaGetLastError();
	}
};
static thread_local ThreadSide g_side;

bool side_stream(cudaStream_t *stream, cudaEvent_t *fork, cudaEvent_t *join) {
	int dev = 0;
	if (cudaGetDevice(&dev) != cudaSuccess) return false;
	if ((int)g_side.dev.size() <= dev) g_side.dev.resize(dev + 1);
	ThreadSide::Dev &d = g_side.dev[dev];
	if (d.failed) return false;
	if (!d.stream) {
		if (cudaStreamCreateWithFlags(&d.stream, cudaStreamNonBlocking) != cudaSuccess ||
		    cudaEventCreateWithFlags(&d.ev[0], cudaEventDisableTiming) != cudaSuccess ||
		    cudaEventCreateWithFlags(&d.ev[1], cudaEventDisableTiming) != cudaSuccess) {
			cudaGetLastError();
			d.failed = true;
			return false;
		}
	}
	*stream = d.stream;
	*fork = d.ev[0];
	*join = d.ev[1];
	return true;
}

void *workspace(size_t bytes, cudaStream_t s) { return workspace_slot(0, bytes, s); }
void *workspace_cm(size_t bytes, cudaStream_t s) { return workspace_slot(1, bytes, s); }

int num_sms() {
	static int sms[64] = {0};
	int dev = 0;
	cudaGetDevice(&dev);
	if (dev < 0 || dev >= 64) return 148;
	if (!sms[dev]) {
		int v = 0;
		cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
		sms[dev] = v > 0 ? v : 148;
	}
	return sms[dev];
}

size_t max_smem_optin() {
	static int v[64] = {0};
	int dev = 0;
	cudaGetDevice(&dev);
	if (dev < 0 || dev >= 64) return 227 * 1024;
	if (!v[dev]) {
		int x = 0;
		cudaDeviceGetAttribute(&x, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
		v[dev] = x > 0 ? x : 227 * 1024;
	}
	return (size_t)v[dev];
}

}  // namespace bf

extern "C" {

int blasfeo_b200_last_error(void) {
	int e = bf::g_last_error;
	bf::g_last_error = BLASFEO_B200_OK;
	return e;
}

const char *blasfeo_b200_error_string(int status) {
	switch (status) {
	case BLASFEO_B200_OK: return "ok";
	case BLASFEO_B200_EINVAL: return "invalid argument";
	case BLASFEO_B200_ECUDA: return "CUDA error";
	case BLASFEO_B200_ENOMEM: return "workspace too small or allocation failed";
	case BLASFEO_B200_ENOTSUP: return "size not supported by this kernel";
	default: return "unknown status";
	}
}

void blasfeo_b200_set_stream(void *stream) { bf::g_stream = (cudaStream_t)stream; }
void *blasfeo_b200_get_stream(void) { return (void *)bf::g_stream; }
void blasfeo_b200_set_sync(int sync) { bf::g_sync = sync; }
int blasfeo_b200_set_posv_engine(int engine) {
	if (engine < BLASFEO_B200_POSV_DEFAULT || engine > BLASFEO_B200_POSV_TENSOR) return BLASFEO_B200_EINVAL;
	bf::g_posv_engine = engine;
	return BLASFEO_B200_OK;
}
int blasfeo_b200_get_posv_engine(void) { return bf::g_posv_engine; }
int blasfeo_b200_version(void) { return 100; }
void blasfeo_b200_set_wait_limit(unsigned int polls) { bf::g_wait_limit.store(polls ? polls : (1u << 24)); }
unsigned int blasfeo_b200_get_wait_limit(void) { return bf::wait_limit(); }

}  // extern "C"
