// Seeded Gaussian streams from a counter-based generator, the same on the
// device, on the host (C++) and in numpy (tval3g.workloads.philox_gaussian),
// so that a large synthetic operator drawn on the device can be regenerated
// elsewhere (an FP64 checker, another process) without storing it.
//
// Generator: Philox-4x32-10 (J. K. Salmon, M. A. Moraes, R. O. Dror and
// D. E. Shaw, "Parallel random numbers: as easy as 1, 2, 3", SC 2011): a
// 128-bit counter and a 64-bit key, ten rounds of two 32x32->64-bit
// multiplications with the round keys bumped by the published Weyl
// constants.  Element i of the stream (seed, offset) takes the counter block
// j = (offset + i) / 4 = (j_lo, j_hi, 0, 0) under the key (seed_lo, seed_hi),
// and word w = (offset + i) % 4 of its output.
//
// Gaussian transform (Box-Muller, in FP64): words 2p and 2p + 1 of a block
// give u1 = ((x_{2p} >> 8) + 1) 2^-24 in (0, 1] and t = (x_{2p+1} >> 8) 2^-24,
// r = sqrt(-2 ln u1), and the pair r cos(2 pi t), r sin(2 pi t); the element
// is scale times that value, rounded once to FP32.  The integer streams are
// bit-identical everywhere; the FP64 logarithm and sine/cosine of different
// math libraries can disagree in their last bit, so an element may differ
// by one FP32 unit in the last place between the device and the host in the
// rare case where the FP64 value lies that close to an FP32 rounding
// boundary.
#include <algorithm>
#include <cmath>

#include "engine.cuh"

namespace tval3g {

namespace {

constexpr unsigned PH_M0 = 0xD2511F53u, PH_M1 = 0xCD9E8D57u;   // round multipliers
constexpr unsigned PH_W0 = 0x9E3779B9u, PH_W1 = 0xBB67AE85u;   // key increments

__host__ __device__ inline void philox4x32_10(unsigned c[4], unsigned k0, unsigned k1) {
	for (int r = 0; r < 10; r++) {
		const unsigned long long p0 = (unsigned long long)PH_M0 * c[0];
		const unsigned long long p1 = (unsigned long long)PH_M1 * c[2];
		const unsigned hi0 = (unsigned)(p0 >> 32), lo0 = (unsigned)p0;
		const unsigned hi1 = (unsigned)(p1 >> 32), lo1 = (unsigned)p1;
		const unsigned n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
		c[0] = n0;
		c[1] = lo1;
		c[2] = n2;
		c[3] = lo0;
		k0 += PH_W0;
		k1 += PH_W1;
	}
}

// the four Gaussian values of counter block j
__host__ __device__ inline void gaussian_block(unsigned long long seed, unsigned long long j, double z[4]) {
	unsigned c[4] = {(unsigned)j, (unsigned)(j >> 32), 0u, 0u};
	philox4x32_10(c, (unsigned)seed, (unsigned)(seed >> 32));
	const double two_pi = 6.283185307179586476925286766559;
	const double q = 1.0 / 16777216.0;
	for (int p = 0; p < 2; p++) {
		const double u1 = (double)((c[2 * p] >> 8) + 1u) * q;
		const double t = (double)(c[2 * p + 1] >> 8) * q;
		const double r = sqrt(-2.0 * log(u1));
		z[2 * p] = r * cos(two_pi * t);
		z[2 * p + 1] = r * sin(two_pi * t);
	}
}

__global__ void __launch_bounds__(256) k_gaussian(unsigned long long seed, unsigned long long offset,
                                                  long long count, float scale, float *out) {
	const long long stride = (long long)gridDim.x * blockDim.x;
	for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += stride) {
		const unsigned long long e = offset + (unsigned long long)i;
		double z[4];
		gaussian_block(seed, e >> 2, z);
		out[i] = (float)(z[e & 3] * (double)scale);
	}
}

}  // namespace

}  // namespace tval3g

using namespace tval3g;

extern "C" int tval3g_gaussian(unsigned long long seed, unsigned long long offset, long long count, float scale,
                               float *d_out, void *stream) {
	try {
		TG_ARG(count >= 0, "Argument error: count must not be negative");
		TG_ARG(d_out || count == 0, "Argument error: NULL argument");
		if (count == 0) return TVAL3G_OK;
		int dev = 0, sms = 0;
		TG_CUDA(cudaGetDevice(&dev));
		TG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
		const long long want = (count + 255) / 256;
		const unsigned grid = (unsigned)std::min<long long>(want, 8LL * std::max(sms, 1));
		k_gaussian<<<grid, 256, 0, (cudaStream_t)stream>>>(seed, offset, count, scale, d_out);
		TG_CUDA(cudaGetLastError());
	} catch (const Error &e) {
		set_error(e.msg);
		return e.code;
	}
	return TVAL3G_OK;
}

extern "C" int tval3g_gaussian_host(unsigned long long seed, unsigned long long offset, long long count,
                                    float scale, float *out) {
	if (count < 0 || (!out && count > 0)) {
		set_error("Argument error: NULL argument or negative count");
		return TVAL3G_ERR_ARGUMENT;
	}
	for (long long i = 0; i < count; i++) {
		const unsigned long long e = offset + (unsigned long long)i;
		double z[4];
		gaussian_block(seed, e >> 2, z);
		out[i] = (float)(z[e & 3] * (double)scale);
	}
	return TVAL3G_OK;
}
