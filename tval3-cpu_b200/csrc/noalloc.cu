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
// The scratch: TVAL3G_STATIC_SCRATCH_FLOATS floats (4 MiB) in a file-scope
// __device__ array.  Every device that loads the library holds it until the
// process exits.  Host code cannot pass the array's name to a kernel (on the
// host it is only a stand-in for the device symbol), so the device address is
// looked up with cudaGetSymbolAddress once per device, with that device
// current, on the first call made on that device; make that first call before
// any stream capture begins.  All calls share the one array: two calls whose
// work overlaps on the GPU (different streams, or different host threads)
// race on it.  Every partial sum a call reads is written by the same call
// first, so nothing has to start at zero.
#include <algorithm>
#include <mutex>

#include "engine.cuh"

namespace tval3g {

constexpr long long STATIC_SCRATCH_FLOATS = 1 << 20;
static __device__ __align__(256) float g_static_scratch[STATIC_SCRATCH_FLOATS];

constexpr int MAX_DEVICES = 64;
static float *g_scratch_addr[MAX_DEVICES];
static std::once_flag g_scratch_once[MAX_DEVICES];
static cudaError_t g_scratch_rc[MAX_DEVICES];

// partial column sums over one chunk of rows: block (ct, kc) covers columns
// [1024 ct, 1024 ct + 1024) and rows [kc*rows_per, ...)
__global__ void __launch_bounds__(256) k_static_adj(const float *A, long long m, long long n, const float *x,
                                                    int K, float *part) {
	const long long ct = blockIdx.x / K, kc = blockIdx.x - ct * K;
	const long long rows_per = (m + K - 1) / K;
	const long long r0 = kc * rows_per, r1 = min(m, r0 + rows_per);
	const long long c0 = ct * 1024 + threadIdx.x * 4;
	float acc[4] = {0.f, 0.f, 0.f, 0.f};
	for (long long r = r0; r < r1; r++) {
		const float xv = __ldg(x + r);
		const float *ar = A + r * n;
#pragma unroll
		for (int e = 0; e < 4; e++)
			if (c0 + e < n) acc[e] = fmaf(__ldg(ar + c0 + e), xv, acc[e]);
	}
	float *p = part + kc * n;
#pragma unroll
	for (int e = 0; e < 4; e++)
		if (c0 + e < n) p[c0 + e] = acc[e];
}

__global__ void __launch_bounds__(256) k_static_red(long long n, int K, const float *part, float *y) {
	const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
	if (c >= n) return;
	float s = 0.f;
	for (int k = 0; k < K; k++) s += part[(long long)k * n + c];
	y[c] = s;
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
		std::call_once(g_scratch_once[dev], [dev] {
			void *p = nullptr;
			g_scratch_rc[dev] = cudaGetSymbolAddress(&p, g_static_scratch);
			g_scratch_addr[dev] = static_cast<float *>(p);
		});
		if (g_scratch_rc[dev] != cudaSuccess)
			throw Error{TVAL3G_ERR_CUDA, std::string("cudaGetSymbolAddress(g_static_scratch): ") +
			                                 cudaGetErrorString(g_scratch_rc[dev])};
		float *part = g_scratch_addr[dev];
		// row chunks: enough blocks to fill the GPU, as many as the scratch holds
		const long long ct = ((long long)n + 1023) / 1024;
		long long K = (4 * 148 + ct - 1) / ct;
		K = std::min(K, STATIC_SCRATCH_FLOATS / n);
		K = std::max(1LL, std::min(K, (long long)m));
		cudaStream_t s = (cudaStream_t)stream;
		k_static_adj<<<(unsigned)(ct * K), 256, 0, s>>>(d_A, m, n, d_x, (int)K, part);
		TG_CUDA(cudaGetLastError());
		k_static_red<<<(unsigned)(((long long)n + 255) / 256), 256, 0, s>>>(n, (int)K, part, d_y);
		TG_CUDA(cudaGetLastError());
		TG_CUDA(cudaStreamSynchronize(s));
	} catch (const Error &e) {
		set_error(e.msg);
		return e.code;
	}
	return TVAL3G_OK;
}
