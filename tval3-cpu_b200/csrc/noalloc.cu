// y = A^T x for a dense row-major matrix without any device allocation.
//
// Who needs this: callers that cannot allocate device memory when they call
// in - for example a host process whose device memory is reserved in full at
// start-up by another allocator (a framework's caching allocator or a serving
// runtime that claims nearly all of HBM), where a fresh cudaMalloc fails, or
// code that must not add the device-wide synchronisation a cudaMalloc /
// cudaFree can cause.  The regular path (tval3g_op_apply on a dense operator)
// allocates its partial-sum scratch; this variant takes it from a fixed array
// compiled into the library instead.
//
// The scratch: STATIC_SCRATCH_FLOATS floats (4 MiB) in a file-scope
// __device__ array.  A device holds it from the moment the library's device
// code is loaded onto it until the process exits.  Under CUDA's default lazy
// module loading that moment is the first call of this entry point on the
// device, so that first call does take 4 MiB (and the module's code) from the
// device: make it at start-up, before another allocator reserves the device's
// memory, or run the process with CUDA_MODULE_LOADING=EAGER, which loads the
// module (and places the array) when the context is created.  Later calls
// take nothing.
//
// Host code cannot pass the array's name to a kernel (on the host it is only a
// stand-in for the device symbol), so the device address is looked up with
// cudaGetSymbolAddress once per device, with that device current, during the
// first call made on that device (a failed look-up is not remembered: the next
// call tries again); make that first call before any stream capture begins.
// All calls share the one array: two calls whose work overlaps on the GPU
// (different streams, or different host threads) race on it.  Every partial
// sum a call reads is written by the same call first, so nothing has to start
// at zero.
//
// The arithmetic is that of the regular dense adjoint (k_dense_adj /
// k_dense_red in ops.cu): each row chunk's column sums accumulated in FP64 in
// row order and stored as float partials, the partials added in FP64 in a
// fixed order; with the same row chunks (a B200's 148 SMs) the two entry
// points give the same bits.
#include <algorithm>
#include <mutex>

#include "engine.cuh"

namespace tval3g {

constexpr long long STATIC_SCRATCH_FLOATS = 1 << 20;
static __device__ __align__(256) float g_static_scratch[STATIC_SCRATCH_FLOATS];

constexpr int MAX_DEVICES = 64;
struct StaticDev {
	float *scratch = nullptr;   // device address of g_static_scratch on this device
	int sms = 0;                // its multiprocessor count
};
static StaticDev g_static_dev[MAX_DEVICES];
static std::mutex g_static_mu;

// partial column sums over one chunk of rows: block (ct, kc) covers columns
// [1024 ct, 1024 ct + 1024) and rows [kc*rows_per, ...)
__global__ void __launch_bounds__(256) k_static_adj(const float *A, long long m, long long n, const float *x,
                                                    int K, float *part) {
	const long long ct = blockIdx.x / K, kc = blockIdx.x - ct * K;
	const long long rows_per = (m + K - 1) / K;
	const long long r0 = kc * rows_per, r1 = min(m, r0 + rows_per);
	const long long c0 = ct * 1024 + threadIdx.x * 4;
	double acc[4] = {0.0, 0.0, 0.0, 0.0};
	for (long long r = r0; r < r1; r++) {
		const double xv = (double)__ldg(x + r);
		const float *ar = A + r * n;
#pragma unroll
		for (int e = 0; e < 4; e++)
			if (c0 + e < n) acc[e] = fma((double)__ldg(ar + c0 + e), xv, acc[e]);
	}
	float *p = part + kc * n;
#pragma unroll
	for (int e = 0; e < 4; e++)
		if (c0 + e < n) p[c0 + e] = (float)acc[e];
}

// y = the sum of the K partials, 32 columns per block: warp w adds partials
// k = w, w + 8, ... of its lane's column, then warp 0 adds the eight warp sums
__global__ void __launch_bounds__(256) k_static_red(long long n, int K, const float *part, float *y) {
	__shared__ double ws[8][32];
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	const long long c = (long long)blockIdx.x * 32 + lane;
	double s = 0.0;
	if (c < n)
		for (int k = warp; k < K; k += 8) s += part[(long long)k * n + c];
	ws[warp][lane] = s;
	__syncthreads();
	if (warp == 0 && c < n) {
		double t = ws[0][lane];
		for (int w = 1; w < 8; w++) t += ws[w][lane];
		y[c] = (float)t;
	}
}

// the array's device address and the SM count of device `dev` (current)
static StaticDev static_dev(int dev) {
	std::lock_guard<std::mutex> lk(g_static_mu);
	StaticDev &d = g_static_dev[dev];
	if (!d.scratch) {
		void *p = nullptr;
		TG_CUDA(cudaGetSymbolAddress(&p, g_static_scratch));
		int sms = 0;
		TG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
		d.sms = std::max(1, sms);
		d.scratch = static_cast<float *>(p);   // set last: a failed look-up leaves the device unset
	}
	return d;
}

}  // namespace tval3g

using namespace tval3g;

extern "C" int tval3g_dense_adjoint_static(const float *d_A, int m, int n, const float *d_x, float *d_y,
                                           void *stream) {
	try {
		TG_ARG(d_A && d_x && d_y, "Argument error: NULL argument");
		TG_ARG(m >= 1 && n >= 1, "Argument error: m and n must be positive");
		TG_ARG((long long)n <= STATIC_SCRATCH_FLOATS,
		       "Argument error: n exceeds the static scratch of tval3g_dense_adjoint_static (1048576 columns)");
		int dev = -1;
		TG_CUDA(cudaGetDevice(&dev));
		TG_ARG(dev >= 0 && dev < MAX_DEVICES, "Argument error: device ordinal beyond 63");
		const StaticDev sd = static_dev(dev);
		// row chunks: four blocks per SM, as many chunks as the scratch holds
		const long long ct = ((long long)n + 1023) / 1024;
		long long K = (4LL * sd.sms + ct - 1) / ct;
		K = std::min(K, STATIC_SCRATCH_FLOATS / n);
		K = std::max(1LL, std::min(K, (long long)m));
		cudaStream_t s = (cudaStream_t)stream;
		k_static_adj<<<(unsigned)(ct * K), 256, 0, s>>>(d_A, m, n, d_x, (int)K, sd.scratch);
		TG_CUDA(cudaGetLastError());
		k_static_red<<<(unsigned)(((long long)n + 31) / 32), 256, 0, s>>>(n, (int)K, sd.scratch, d_y);
		TG_CUDA(cudaGetLastError());
	} catch (const Error &e) {
		set_error(e.msg);
		return e.code;
	}
	return TVAL3G_OK;
}
