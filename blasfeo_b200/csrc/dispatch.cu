// Learned dispatch inside the library: when a cost model is installed, the
// variable-size batched routines called with variant -1 pick their kernel
// variant with it instead of the built-in rule.
//
// The model is the MLP of mlp.cu (nin -> hidden -> hidden -> hidden -> 1,
// ReLU, FP32) trained on the autotuner's timings to predict the (normalised)
// log run time of one launch with one variant.  Its input features are those
// of the trainer (blasfeo_b200/autotune.py features()):
//   [op one-hot (4), log2(batch)/13,
//    mean/9, max/9, std/4 of log2 m, of log2 n, of log2 k over the instances,
//    variant one-hot (6)]
// A pick computes the features of the launch on the device from the size
// arrays (one block), runs the MLP forward kernel on one row per variant,
// copies the predictions back (a synchronisation of the caller's stream) and
// takes the argmin.  Picks are cached per (device, op, batch, max sizes), so
// a launch shape that repeats -- the usual case of a solver loop -- pays for
// the model once; a stream that is being captured never runs the model (a
// cached pick is used, else the built-in rule).  The model changes the speed
// only: every variant computes the same results within the routine's
// tolerance (pivot choices identical).
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "common.cuh"

namespace {

constexpr int NOPS = 4;
constexpr int MAXVAR = 6;
constexpr int NFEAT = NOPS + 1 + 9 + MAXVAR;

struct Model {
	int nin = 0, hidden = 0;
	std::vector<float> host;  // parameters, for per-device upload
	std::map<int, float *> dev;  // device -> params | X | y | work
	std::map<std::tuple<int, int, int, int, int, int>, int> cache;
};
std::mutex g_mu;
Model *g_model = nullptr;

// features of one launch: block of 256 threads; rows r < nvar of X get the
// shared part plus the one-hot of variant r
__global__ void k_dispatch_features(int op, int batch, const int *__restrict__ m, const int *__restrict__ n,
                                    const int *__restrict__ k, int nvar, float *X) {
	__shared__ double red[3][3][8];
	double s[3] = {0, 0, 0}, q[3] = {0, 0, 0}, mx[3] = {0, 0, 0};
	const int *arr[3] = {m, n, k};
	for (int i = threadIdx.x; i < batch; i += blockDim.x)
		for (int d = 0; d < 3; d++) {
			const int v = arr[d][i];
			const double l = log2((double)(v > 1 ? v : 1));
			s[d] += l;
			q[d] += l * l;
			mx[d] = fmax(mx[d], l);
		}
	const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
	for (int d = 0; d < 3; d++) {
		for (int off = 16; off > 0; off >>= 1) {
			s[d] += __shfl_xor_sync(0xffffffffu, s[d], off);
			q[d] += __shfl_xor_sync(0xffffffffu, q[d], off);
			mx[d] = fmax(mx[d], __shfl_xor_sync(0xffffffffu, mx[d], off));
		}
		if (lane == 0) {
			red[d][0][w] = s[d];
			red[d][1][w] = q[d];
			red[d][2][w] = mx[d];
		}
	}
	__syncthreads();
	if (threadIdx.x < nvar) {
		float *row = X + (size_t)threadIdx.x * NFEAT;
		for (int c = 0; c < NFEAT; c++) row[c] = 0.f;
		row[op] = 1.f;
		row[NOPS] = (float)(log2((double)batch) / 13.0);
		const int nw = blockDim.x >> 5;
		for (int d = 0; d < 3; d++) {
			double ss = 0, qq = 0, mm = 0;
			for (int i = 0; i < nw; i++) {
				ss += red[d][0][i];
				qq += red[d][1][i];
				mm = fmax(mm, red[d][2][i]);
			}
			const double mean = ss / batch;
			const double var = fmax(qq / batch - mean * mean, 0.0);
			row[NOPS + 1 + 3 * d] = (float)(mean / 9.0);
			row[NOPS + 2 + 3 * d] = (float)(mm / 9.0);
			row[NOPS + 3 + 3 * d] = (float)(sqrt(var) / 4.0);
		}
		row[NOPS + 10 + threadIdx.x] = 1.f;
	}
}

}  // namespace

namespace bf {

// variant for a launch with variant -1: the cost model's pick, or -1 (the
// built-in rule) when no model is installed or it cannot run now
int dispatch_pick(int op, int batch, const int *m, const int *n, const int *k, int max_m, int max_n, int max_k,
                  cudaStream_t s) {
	if (op < 0 || op >= NOPS || batch <= 0) return -1;
	int dev = 0;
	if (cudaGetDevice(&dev) != cudaSuccess) return -1;
	std::lock_guard<std::mutex> lock(g_mu);
	if (!g_model) return -1;
	Model &M = *g_model;
	const auto key = std::make_tuple(dev, op, batch, max_m, max_n, max_k);
	auto it = M.cache.find(key);
	if (it != M.cache.end()) return it->second;
	cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
	if (cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) {
		cudaGetLastError();
		return -1;
	}
	const int nvar = blasfeo_b200_num_variants(op);
	const size_t np = (size_t)blasfeo_b200_mlp_param_count(M.nin, M.hidden);
	const size_t wfl = blasfeo_b200_mlp_work_bytes(M.hidden, MAXVAR) / sizeof(float);
	float *buf;
	auto d = M.dev.find(dev);
	if (d == M.dev.end()) {
		// first pick on this device: upload the parameters next to the
		// feature rows, predictions and forward scratch
		if (cudaMalloc(&buf, (np + MAXVAR * NFEAT + MAXVAR + wfl + 64) * sizeof(float)) != cudaSuccess) {
			cudaGetLastError();
			return -1;
		}
		cudaMemcpy(buf, M.host.data(), np * sizeof(float), cudaMemcpyHostToDevice);
		M.dev[dev] = buf;
	} else {
		buf = d->second;
	}
	float *X = buf + np, *y = X + MAXVAR * NFEAT, *work = y + MAXVAR;
	k_dispatch_features<<<1, 256, 0, s>>>(op, batch, m, n, k ? k : n, nvar, X);
	if (blasfeo_b200_mlp_forward(M.nin, M.hidden, buf, nvar, X, y, work, s) != BLASFEO_B200_OK) return -1;
	float h[MAXVAR];
	if (cudaMemcpyAsync(h, y, nvar * sizeof(float), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
	    cudaStreamSynchronize(s) != cudaSuccess) {
		cudaGetLastError();
		return -1;
	}
	int best = 0;
	for (int v = 1; v < nvar; v++)
		if (h[v] < h[best]) best = v;
	M.cache[key] = best;
	return best;
}

}  // namespace bf

extern "C" {

int blasfeo_b200_cost_model_nfeat(void) { return NFEAT; }

int blasfeo_b200_set_cost_model(int nin, int hidden, const float *params) {
	if (nin != NFEAT || hidden <= 0 || hidden > 1024 || !params) return BLASFEO_B200_EINVAL;
	const int np = blasfeo_b200_mlp_param_count(nin, hidden);
	if (np <= 0) return BLASFEO_B200_EINVAL;
	Model *m = new Model;
	m->nin = nin;
	m->hidden = hidden;
	m->host.assign(params, params + np);
	std::lock_guard<std::mutex> lock(g_mu);
	if (g_model)
		for (auto &d : g_model->dev) cudaFree(d.second);
	delete g_model;
	g_model = m;
	return BLASFEO_B200_OK;
}

void blasfeo_b200_clear_cost_model(void) {
	std::lock_guard<std::mutex> lock(g_mu);
	if (g_model)
		for (auto &d : g_model->dev) cudaFree(d.second);
	delete g_model;
	g_model = nullptr;
}

int blasfeo_b200_dispatch_pick(int op, int batch, const int *m, const int *n, const int *k, int max_m, int max_n,
                               int max_k, void *stream) {
	if (op < 0 || op >= NOPS || batch < 0 || (batch > 0 && (!m || !n))) return -2;
	return bf::dispatch_pick(op, batch, m, n, k, max_m, max_n, max_k, (cudaStream_t)stream);
}

}  // extern "C"
