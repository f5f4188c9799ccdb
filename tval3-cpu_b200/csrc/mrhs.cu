// Multi-right-hand-side dense operator on the tcgen05 tensor cores (3xTF32).
//
// For a dense A (m x n, row-major) and N right-hand sides stored layer-major
// (x[l*K + k]), the forward y = A x and the adjoint y = A^T x are both one
// contraction D[M x N] = P[M x K] Q[N x K]^T with P = A (forward: M = m,
// K = n) or P = A^T (adjoint, M = n, K = m).  Both operands are K-major, so
// one kernel serves both directions.  P is read from a copy of A (and of A^T)
// re-laid once, at operator creation, in tile-major order: each 128 x 32 tile
// that one pipeline stage loads is 16 KB contiguous in HBM (the row-major
// layout would make every stage 128 separate 128-byte pieces 4n bytes apart,
// which held DRAM throughput near 40 %).
//
// Split precision (3xTF32): P = Ph + Pl and Q = Qh + Ql with Ph = P rounded
// to the nearest TF32 value and Pl = P - Ph (exact in FP32, |Pl| <= 2^-11 |P|);
// D = Ph Qh + Ph Ql + Pl Qh, the Pl Ql term (relative size 2^-22) dropped.
// Qh and Ql are consecutive rows of one 2N-row operand, so each K slice takes
// two MMAs: Ph [Qh; Ql] into 2N accumulator columns and Pl Qh into the first
// N.  Q is split once per product into two global arrays (a few MB,
// L2-resident); each P tile is split in shared memory by the converter warps
// right after its TMA load, so A is read from HBM exactly once per product.
//
// Accumulation: the tensor cores' FP32 accumulation is not round-to-nearest,
// and its error grows with the length of the MMA chain (2.5e-5 relative over
// 110 stages at m = 4096, n = 16384, measured), so every stage (K = 32)
// accumulates into a fresh TMEM buffer that the epilogue warps add into FP64
// registers; four buffers rotate so the MMAs of the next stages overlap the
// drain of this one.
//
// Work split (stream-K): the tiles x K-steps iterations are cut into G equal
// contiguous ranges, one per CTA, G = min(number of SMs, iterations) (one
// 448-thread CTA per SM, up to 226 KB of shared memory).  For every tile segment in its range a CTA
// writes a 128 x N FP32 partial; k_mrhs_red adds each tile's partials in CTA
// order in FP64, so the result does not depend on timing.
//
// Warp roles: warp 0 issues the TMA loads (one elected lane), warp 1 owns the
// tensor memory and issues the MMAs (one lane), warps 2-5 split P tiles (the
// high part in place, the low part into a ring of two buffers, so six TMA
// stages stay in flight), warps 6-13 drain the accumulators (warp w reads
// TMEM lanes 32 (w % 4) .. +31, half of the columns).  Every mbarrier wait is bounded: a timeout sets the
// operator's error flag and ends the CTA's loops; the producer then waits
// (bounded) for its loads in flight and the MMA lane for its MMAs before the
// tensor memory is released.
#include "mrhs.cuh"

#include <mutex>

#include "async.cuh"

TG_BEGIN

namespace {

constexpr int BM = 128;           // rows per tile (MMA M = TMEM lanes)
constexpr int BK = 32;            // K elements per stage: one 128-byte swizzle row of FP32
constexpr int STAGES = 6;          // TMA stages (P tile + both Q tiles)
constexpr int LO_BUFS = 2;         // ring of low-part P tiles
constexpr int CONV_WARPS = 4;
constexpr int EPI_WARPS = 8;       // two per TMEM lane quarter, each half of the columns
constexpr int ACC_BUFS = 4;        // TMEM accumulator buffers (one stage each)
constexpr int THREADS = (2 + CONV_WARPS + EPI_WARPS) * 32;
constexpr unsigned WAIT_LIMIT = 1u << 22;
constexpr unsigned TF32_MASK = 0xFFFFE000u;

__host__ __device__ constexpr int p_tile_bytes() { return BM * BK * 4; }
__host__ __device__ constexpr int q_tile_bytes(int N) { return N * BK * 4; }
__host__ __device__ constexpr int stage_bytes(int N) { return p_tile_bytes() + 2 * q_tile_bytes(N); }
// ACC_BUFS accumulator buffers of 2N FP32 columns each, rounded up to a power of two
__host__ __device__ constexpr int tmem_cols(int N) {
	return 2 * ACC_BUFS * N <= 128 ? 128 : 2 * ACC_BUFS * N <= 256 ? 256 : 512;
}

struct Bars {
	unsigned long long full[STAGES], conv[STAGES], empty[STAGES], lofree[LO_BUFS], accf[ACC_BUFS], acce[ACC_BUFS], done;
	unsigned tmem;
	int abort;
};

size_t smem_bytes(int N) {
	return 1024 + (size_t)STAGES * stage_bytes(N) + (size_t)LO_BUFS * p_tile_bytes() + sizeof(Bars);
}

// ---------------------------------------------------------------------------
// PTX wrappers
// ---------------------------------------------------------------------------
__device__ __forceinline__ void tma_load_2d(unsigned dst, const CUtensorMap *map, int x, int y, unsigned bar) {
	asm volatile(
	    "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
	        dst),
	    "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(y), "r"(bar)
	    : "memory");
}
__device__ __forceinline__ void tc_fence_before() {
	asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
	asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tmem_alloc(unsigned dst_smem, unsigned ncols) {
	asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst_smem), "r"(ncols)
	             : "memory");
	asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(unsigned taddr, unsigned ncols) {
	asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
// D (tmem) (+)= A (smem, desc) * B (smem, desc)^T, kind::tf32, one thread
__device__ __forceinline__ void mma_tf32(unsigned d, unsigned long long adesc, unsigned long long bdesc,
                                         unsigned idesc, unsigned accumulate) {
	asm volatile(
	    "{\n\t.reg .pred p;\n\t"
	    "setp.ne.b32 p, %4, 0;\n\t"
	    "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(d),
	    "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
	    : "memory");
}
// arrive on `bar` once every tcgen05 operation issued so far by this thread is done
__device__ __forceinline__ void mma_commit(unsigned bar) {
	asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
	             : "memory");
}
// 32 lanes x 8 consecutive FP32 columns: thread i gets lane (base + i)
__device__ __forceinline__ void tmem_ld8(unsigned taddr, float *v) {
	unsigned r[8];
	asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
	             : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
	             : "r"(taddr)
	             : "memory");
#pragma unroll
	for (int i = 0; i < 8; i++) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_wait_ld() {
	asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// nearest TF32 value (ties away from zero); exact in FP32, so P - tf32_rn(P)
// is exact too and at most half a TF32 unit in the last place
__device__ __forceinline__ float tf32_rn(float v) {
	return __uint_as_float((__float_as_uint(v) + 0x1000u) & TF32_MASK);
}

// shared-memory matrix descriptor: K-major operand in the 128-byte swizzle
// layout written by TMA (rows of 128 bytes, 8-row groups 1024 bytes apart)
__device__ __forceinline__ unsigned long long sdesc(unsigned addr) {
	return (unsigned long long)((addr & 0x3FFFFu) >> 4)   // start address / 16
	       | (1ull << 16)                                 // leading byte offset (unused when swizzled)
	       | (64ull << 32)                                // stride byte offset: 1024 / 16
	       | (1ull << 46)                                 // descriptor version of sm_100
	       | (2ull << 61);                                // 128-byte swizzle
}
// instruction descriptor: D FP32, A and B TF32, both K-major, M = 128
__host__ __device__ constexpr unsigned idesc_tf32(int N) {
	return (1u << 4)                      // D format: F32
	       | (2u << 7)                    // A format: TF32
	       | (2u << 10)                   // B format: TF32
	       | ((unsigned)(N >> 3) << 17)   // N / 8
	       | ((unsigned)(BM >> 4) << 24); // M / 16
}

// bounded waits; false on timeout (which also raises the abort flag) or abort
__device__ __forceinline__ bool wait1(unsigned bar, unsigned parity, volatile int *abort, int *err) {
	for (unsigned i = 0; i < WAIT_LIMIT; i++) {
		if (mbar_try(bar, parity)) return true;
		if ((i & 255u) == 255u && *abort) return false;
	}
	*abort = 1;
	atomicExch(err, 1);
	return false;
}
// every lane of the warp polls; the warp leaves together
__device__ __forceinline__ bool wait_warp(unsigned bar, unsigned parity, volatile int *abort, int *err) {
	for (unsigned i = 0; i < WAIT_LIMIT; i++) {
		if (__all_sync(0xffffffffu, mbar_try(bar, parity))) return true;
		if ((i & 255u) == 255u && __any_sync(0xffffffffu, *abort != 0)) return false;
	}
	if ((threadIdx.x & 31) == 0) {
		*abort = 1;
		atomicExch(err, 1);
	}
	return false;
}

struct MrhsArgs {
	const Inst *tab;
	int inst, pred;
	const int *members;   // independent right-hand sides (MrhsOp::members) or NULL
	int N;
	int M;          // rows of D
	int ks;         // K steps of BK
	int J;          // partial slots per CTA
	long long T;    // tiles x ks
	float *part;    // [G][J][N][BM]
	int *err;
	unsigned long long *launches;
};

template <int N>
__global__ void __launch_bounds__(THREADS, 1)
    k_mrhs(const __grid_constant__ CUtensorMap tmP, const __grid_constant__ CUtensorMap tmQh,
           const __grid_constant__ CUtensorMap tmQl, MrhsArgs a) {
	if (a.members) {   // independent right-hand sides: run if any of them takes part
		bool any = false;
		for (int l = 0; l < a.N && !any; l++) any = pred_ok(*a.tab[a.members[l]].ctrl, a.pred);
		if (!any) return;
	} else if (!pred_ok(*a.tab[a.inst].ctrl, a.pred)) {
		return;
	}
	if (a.launches && blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(a.launches, 1ull);
	extern __shared__ unsigned char smem_raw[];
	const unsigned raw = smem_u32(smem_raw);
	const unsigned base = (raw + 1023u) & ~1023u;   // swizzled tiles need 1024-byte alignment
	constexpr int SB = stage_bytes(N);
	constexpr unsigned TX = (unsigned)(p_tile_bytes() + 2 * q_tile_bytes(N));
	constexpr unsigned NCOLS = tmem_cols(N);
	constexpr unsigned LO0 = STAGES * SB;   // low-part ring after the stages
	Bars *bars = reinterpret_cast<Bars *>(smem_raw + (base - raw) + LO0 + LO_BUFS * p_tile_bytes());
	volatile int *abort = &bars->abort;
	auto st_p = [&](int s) { return base + s * SB; };
	auto st_qh = [&](int s) { return base + s * SB + p_tile_bytes(); };
	auto st_ql = [&](int s) { return base + s * SB + p_tile_bytes() + q_tile_bytes(N); };
	auto lo_p = [&](int l) { return base + LO0 + l * p_tile_bytes(); };
	const unsigned b_full = smem_u32(&bars->full[0]), b_conv = smem_u32(&bars->conv[0]),
	               b_empty = smem_u32(&bars->empty[0]), b_lofree = smem_u32(&bars->lofree[0]),
	               b_accf = smem_u32(&bars->accf[0]), b_acce = smem_u32(&bars->acce[0]),
	               b_done = smem_u32(&bars->done);
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

	// this CTA's range of (tile, K step) iterations
	const long long G = gridDim.x;
	const long long it0 = (long long)blockIdx.x * a.T / G, it1 = ((long long)blockIdx.x + 1) * a.T / G;
	const int tile0 = (int)(it0 / a.ks);

	if (threadIdx.x == 0) {
		for (int s = 0; s < STAGES; s++) {
			mbar_init(b_full + 8 * s, 1);
			mbar_init(b_conv + 8 * s, CONV_WARPS);
			mbar_init(b_empty + 8 * s, 1);
		}
		for (int l = 0; l < LO_BUFS; l++) mbar_init(b_lofree + 8 * l, 1);
		for (int i = 0; i < ACC_BUFS; i++) {
			mbar_init(b_accf + 8 * i, 1);
			mbar_init(b_acce + 8 * i, EPI_WARPS);
		}
		mbar_init(b_done, 1);
		bars->abort = 0;
		fence_mbar_init();
	}
	if (warp == 1) tmem_alloc(smem_u32(&bars->tmem), NCOLS);
	tc_fence_before();
	__syncthreads();
	tc_fence_after();
	const unsigned tmem = bars->tmem;

	if (warp == 0) {
		if (lane == 0) {   // TMA producer
			unsigned it = 0;
			for (long long g = it0; g < it1; g++, it++) {
				const int s = it % STAGES;
				if (!wait1(b_empty + 8 * s, ((it / STAGES) & 1) ^ 1, abort, a.err)) break;
				const int k = (int)(g % a.ks);
				mbar_expect_tx(b_full + 8 * s, TX);
				tma_load_2d(st_p(s), &tmP, 0, (int)(g * BM), b_full + 8 * s);   // tile-major copy: contiguous
				tma_load_2d(st_qh(s), &tmQh, k * BK, 0, b_full + 8 * s);
				tma_load_2d(st_ql(s), &tmQl, k * BK, 0, b_full + 8 * s);
			}
			// no load may still be writing shared memory when the CTA ends
			const unsigned issued = it;
			for (unsigned j = issued > STAGES ? issued - STAGES : 0; j < issued; j++) {
				unsigned i = 0;
				while (!mbar_try(b_full + 8 * (j % STAGES), (j / STAGES) & 1) && ++i < WAIT_LIMIT) {
				}
				if (i >= WAIT_LIMIT) atomicExch(a.err, 1);
			}
		}
	} else if (warp == 1) {
		if (lane == 0) {   // MMA issuer: one stage into one accumulator buffer
			constexpr unsigned ID2 = idesc_tf32(2 * N), ID1 = idesc_tf32(N);
			unsigned it = 0;
			for (long long g = it0; g < it1; g++, it++) {
				const int s = it % STAGES, lb = it % LO_BUFS, ab = it % ACC_BUFS;
				if (!wait1(b_acce + 8 * ab, ((it / ACC_BUFS) & 1) ^ 1, abort, a.err)) break;
				if (!wait1(b_conv + 8 * s, (it / STAGES) & 1, abort, a.err)) break;
				tc_fence_after();
				const unsigned d = tmem + (unsigned)(ab * 2 * N);
#pragma unroll
				for (int kk = 0; kk < BK / 8; kk++) {   // K = 8 per MMA: 32 bytes
					const unsigned off = kk * 32;
					// columns [0, N): Ph Qh + Pl Qh; columns [N, 2N): Ph Ql (Qh and Ql
					// are consecutive rows of one 2N-row operand)
					mma_tf32(d, sdesc(st_p(s) + off), sdesc(st_qh(s) + off), ID2, kk > 0 ? 1u : 0u);
					mma_tf32(d, sdesc(lo_p(lb) + off), sdesc(st_qh(s) + off), ID1, 1u);
				}
				mma_commit(b_empty + 8 * s);
				mma_commit(b_lofree + 8 * lb);
				mma_commit(b_accf + 8 * ab);
			}
			// every MMA issued has finished before the tensor memory is released
			mma_commit(b_done);
			unsigned i = 0;
			while (!mbar_try(b_done, 0) && ++i < WAIT_LIMIT) {
			}
			if (i >= WAIT_LIMIT) atomicExch(a.err, 1);
		}
	} else if (warp < 2 + CONV_WARPS) {   // split P tiles into high and low parts
		const int t = threadIdx.x - 64;
		unsigned it = 0;
		for (long long g = it0; g < it1; g++, it++) {
			const int s = it % STAGES, lb = it % LO_BUFS;
			if (!wait_warp(b_full + 8 * s, (it / STAGES) & 1, abort, a.err)) break;
			if (!wait_warp(b_lofree + 8 * lb, ((it / LO_BUFS) & 1) ^ 1, abort, a.err)) break;
			float4 *P = reinterpret_cast<float4 *>(smem_raw + (st_p(s) - raw));
			float4 *L = reinterpret_cast<float4 *>(smem_raw + (lo_p(lb) - raw));
#pragma unroll
			for (int i = 0; i < p_tile_bytes() / 16 / (CONV_WARPS * 32); i++) {
				const int idx = i * CONV_WARPS * 32 + t;
				const float4 v = P[idx];
				const float4 h = make_float4(tf32_rn(v.x), tf32_rn(v.y), tf32_rn(v.z), tf32_rn(v.w));
				P[idx] = h;
				L[idx] = make_float4(v.x - h.x, v.y - h.y, v.z - h.z, v.w - h.w);
			}
			fence_proxy_async_smem();   // generic-proxy writes, read next by the tensor cores
			__syncwarp();
			if (lane == 0) mbar_arrive(b_conv + 8 * s);
		}
	} else {   // epilogue: every stage's accumulator is added in FP64 (short tensor-core chains)
		constexpr int NH = N / 2;   // columns per epilogue warp
		const int ew = warp - 2 - CONV_WARPS;
		const int q = warp & 3, c0 = (ew >> 2) * NH;
		const int row = q * 32 + lane;
		const unsigned lane_base = tmem + ((unsigned)(q * 32) << 16);
		double acc[NH];
		unsigned it = 0;
		for (long long g = it0; g < it1; g++, it++) {
			const int tile = (int)(g / a.ks), k = (int)(g - (long long)tile * a.ks);
			if (g == it0 || k == 0)
#pragma unroll
				for (int c = 0; c < NH; c++) acc[c] = 0.0;
			const int ab = it % ACC_BUFS;
			if (!wait_warp(b_accf + 8 * ab, (it / ACC_BUFS) & 1, abort, a.err)) break;
			tc_fence_after();
			float lo[NH], hi[NH];   // every load of the stage in flight, one wait
#pragma unroll
			for (int c = 0; c < NH; c += 8) {
				tmem_ld8(lane_base + (unsigned)(ab * 2 * N + c0 + c), lo + c);
				tmem_ld8(lane_base + (unsigned)(ab * 2 * N + N + c0 + c), hi + c);
			}
			tmem_wait_ld();
			// Ph Ql (columns N..2N) is 2^-11 of the rest: one FP32 add, then FP64
#pragma unroll
			for (int c = 0; c < NH; c++) acc[c] += (double)(lo[c] + hi[c]);
			tc_fence_before();
			__syncwarp();
			if (lane == 0) mbar_arrive(b_acce + 8 * ab);
			if ((g == it1 - 1 || k == a.ks - 1) && (long long)tile * BM + row < a.M) {
				float *dst = a.part + ((long long)blockIdx.x * a.J + (tile - tile0)) * N * BM + (long long)c0 * BM + row;
#pragma unroll
				for (int c = 0; c < NH; c++) dst[c * BM] = (float)acc[c];
			}
		}
	}

	tc_fence_before();
	__syncthreads();
	if (warp == 1) {
		__syncwarp();
		tc_fence_after();
		tmem_dealloc(tmem, NCOLS);
	}
}

// D[r, l] = sum over the CTAs whose range meets tile r / BM of their partial
// (independent right-hand sides: row r of column l goes to element r of
// instance members[l], where its predicate holds)
__global__ void __launch_bounds__(256) k_mrhs_red(const Inst *tab, int inst, int pred, VecSel ys, const float *part,
                                                  int M, int N, int ks, long long T, int G, int J, const int *members,
                                                  unsigned long long *launches) {
	if (!members && !pred_ok(*tab[inst].ctrl, pred)) return;
	if (launches && blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(launches, 1ull);
	const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
	if (idx >= (long long)N * M) return;
	const int l = (int)(idx / M), r = (int)(idx - (long long)l * M);
	const Inst &I = tab[members ? members[l] : inst];
	if (members && !pred_ok(*I.ctrl, pred)) return;
	const int t = r / BM, row = r - t * BM;
	const long long i0 = (long long)t * ks, i1 = i0 + ks - 1;
	const int c0 = (int)(((i0 + 1) * G - 1) / T), c1 = (int)(((i1 + 1) * G - 1) / T);
	double s = 0.0;
	for (int c = c0; c <= c1; c++) {
		const long long beg = (long long)c * T / G;
		const int j = t - (int)(beg / ks);
		s += part[(((long long)c * J + j) * N + l) * BM + row];
	}
	float *y = ys.m ? I.vm[ys.idx] : I.vn[ys.idx];
	y[(members ? 0 : (long long)l * M) + r] = (float)s;
}

// right-hand sides -> high (TF32-exact) and low parts
// (independent right-hand sides: column l of length K from instance
// members[l], zero where its predicate does not hold)
__global__ void __launch_bounds__(256) k_mrhs_split(const Inst *tab, int inst, int pred, VecSel xs, long long len,
                                                    long long K, const int *members, float *hi, float *lo,
                                                    unsigned long long *launches) {
	if (!members && !pred_ok(*tab[inst].ctrl, pred)) return;
	if (launches && blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(launches, 1ull);
	for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < len; i += (long long)gridDim.x * blockDim.x) {
		float v;
		if (members) {
			const long long l = i / K;
			const Inst &J = tab[members[l]];
			v = pred_ok(*J.ctrl, pred) ? (xs.m ? J.vm[xs.idx] : J.vn[xs.idx])[i - l * K] : 0.f;
		} else {
			const Inst &I = tab[inst];
			v = (xs.m ? I.vm[xs.idx] : I.vn[xs.idx])[i];
		}
		const float h = tf32_rn(v);
		hi[i] = h;
		lo[i] = v - h;
	}
}

// tile-major copy of a row-major rows x cols matrix: 128 x 32 tiles, each
// 16 KB contiguous, tile (t, k) at ((t * ks + k) * 128 + r) * 32 + c, zero
// outside the matrix
__global__ void k_tile_major(const float *src, long long rows, long long cols, int ks, long long total, float *T) {
	for (long long o = (long long)blockIdx.x * blockDim.x + threadIdx.x; o < total;
	     o += (long long)gridDim.x * blockDim.x) {
		const int c = (int)(o & (BK - 1)), r = (int)((o >> 5) & (BM - 1));
		const long long tk = o >> 12;
		const long long t = tk / ks, k = tk - t * ks;
		const long long row = t * BM + r, col = k * BK + c;
		T[o] = (row < rows && col < cols) ? src[row * cols + col] : 0.f;
	}
}

__global__ void k_transpose(const float *A, long long m, long long n, float *At) {
	__shared__ float tile[32][33];
	const long long c0 = (long long)blockIdx.x * 32, r0 = (long long)blockIdx.y * 32;
	for (int i = threadIdx.y; i < 32; i += 8) {
		const long long r = r0 + i, c = c0 + threadIdx.x;
		if (r < m && c < n) tile[i][threadIdx.x] = A[r * n + c];
	}
	__syncthreads();
	for (int i = threadIdx.y; i < 32; i += 8) {
		const long long c = c0 + i, r = r0 + threadIdx.x;
		if (r < m && c < n) At[c * m + r] = tile[threadIdx.x][i];
	}
}

// ---------------------------------------------------------------------------
// host
// ---------------------------------------------------------------------------
typedef CUresult (*EncodeTiled)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled encoder() {
	static std::once_flag once;
	static EncodeTiled fn = nullptr;
	std::call_once(once, [] {
		void *p = nullptr;
		cudaDriverEntryPointQueryResult q;
		if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
		    q == cudaDriverEntryPointSuccess)
			fn = reinterpret_cast<EncodeTiled>(p);
	});
	if (!fn) throw Error{TVAL3G_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver"};
	return fn;
}

// row-major rows x inner FP32 matrix, box of box_rows x 32 elements, 128-byte swizzle
CUtensorMap make_map(const float *ptr, long long inner, long long rows, int box_rows) {
	CUtensorMap m;
	const cuuint64_t dims[2] = {(cuuint64_t)inner, (cuuint64_t)rows};
	const cuuint64_t strides[1] = {(cuuint64_t)inner * sizeof(float)};
	const cuuint32_t box[2] = {(cuuint32_t)BK, (cuuint32_t)box_rows};
	const cuuint32_t estr[2] = {1, 1};
	CUresult r = encoder()(&m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float *>(ptr), dims, strides, box, estr,
	                       CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
	                       CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
	if (r != CUDA_SUCCESS)
		throw Error{TVAL3G_ERR_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")"};
	return m;
}

// stream-K plan of one direction: K steps, tiles, iterations, partial slots
void plan_dir(long long M, long long K, int G, int &ks, int &tiles, long long &T, int &J) {
	ks = (int)((K + BK - 1) / BK);
	tiles = (int)((M + BM - 1) / BM);
	T = (long long)tiles * ks;
	J = 1;
	for (long long c = 0; c < G; c++) {
		const long long i0 = c * T / G, i1 = (c + 1) * T / G;
		if (i1 > i0) J = std::max(J, (int)((i1 - 1) / ks - i0 / ks + 1));
	}
}

template <int N>
void set_smem_attr() {
	static std::once_flag once;
	static cudaError_t rc = cudaSuccess;
	std::call_once(once, [] {
		rc = cudaFuncSetAttribute(k_mrhs<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes(N));
	});
	TG_CUDA(rc);
}

template <int N>
void launch_mrhs(cudaStream_t s, int G, const CUtensorMap &p, const CUtensorMap &qh, const CUtensorMap &ql,
                 const MrhsArgs &a) {
	set_smem_attr<N>();
	k_mrhs<N><<<G, THREADS, smem_bytes(N), s>>>(p, qh, ql, a);
}

}  // namespace

MrhsOp::~MrhsOp() {
	if (ta) cudaFree(ta);
	if (tat) cudaFree(tat);
	if (xh) cudaFree(xh);
	if (xl) cudaFree(xl);
	if (part) cudaFree(part);
	if (err) cudaFree(err);
	if (members) cudaFree(members);
}

void mrhs_set_members(cudaStream_t s, MrhsOp &op, const int *members) {
	if (!op.members) TG_CUDA(cudaMalloc(&op.members, sizeof(int) * (size_t)op.N));
	TG_CUDA(cudaMemcpyAsync(op.members, members, sizeof(int) * (size_t)op.N, cudaMemcpyHostToDevice, s));
	TG_CUDA(cudaStreamSynchronize(s));
}

bool mrhs_eligible(long long m, long long n, int layers) {
	return (layers == 16 || layers == 32 || layers == 48 || layers == 64) && m >= BM && n >= BM && m % 4 == 0 &&
	       n % 4 == 0 && m < (1LL << 31) / 64 && n < (1LL << 31) / 64 && (m + 31) / 32 < 65535 &&
	       ((m + BM - 1) / BM) * ((n + BK - 1) / BK) * BM < (1LL << 31) &&
	       ((n + BM - 1) / BM) * ((m + BK - 1) / BK) * BM < (1LL << 31);
}

std::shared_ptr<MrhsOp> mrhs_create(cudaStream_t s, const float *d_A, long long m, long long n, int layers) {
	TG_ARG(mrhs_eligible(m, n, layers), "Internal error: operator not eligible for the tensor-core path");
	TG_ARG((reinterpret_cast<uintptr_t>(d_A) & 15) == 0, "Argument error: A must be 16-byte aligned");
	auto op = std::make_shared<MrhsOp>();
	op->m = m;
	op->n = n;
	op->N = layers;
	int dev = 0, sms = 0;
	TG_CUDA(cudaGetDevice(&dev));
	TG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
	// one CTA per SM, fewer when there are fewer (tile, K step) iterations
	const long long tf = ((m + BM - 1) / BM) * ((n + BK - 1) / BK), ta = ((n + BM - 1) / BM) * ((m + BK - 1) / BK);
	op->grid_f = (int)std::min<long long>(sms, tf);
	op->grid_a = (int)std::min<long long>(sms, ta);
	plan_dir(m, n, op->grid_f, op->ks_f, op->tiles_f, op->t_f, op->j_f);
	plan_dir(n, m, op->grid_a, op->ks_a, op->tiles_a, op->t_a, op->j_a);
	const long long kmax = std::max(m, n);
	const long long part = std::max((long long)op->grid_f * op->j_f, (long long)op->grid_a * op->j_a) * layers * BM;
	const long long sz_f = (long long)op->tiles_f * op->ks_f * BM * BK, sz_a = (long long)op->tiles_a * op->ks_a * BM * BK;
	TG_CUDA(cudaMalloc(&op->ta, sizeof(float) * (size_t)sz_f));
	TG_CUDA(cudaMalloc(&op->tat, sizeof(float) * (size_t)sz_a));
	TG_CUDA(cudaMalloc(&op->xh, sizeof(float) * (size_t)(kmax * layers)));
	TG_CUDA(cudaMalloc(&op->xl, sizeof(float) * (size_t)(kmax * layers)));
	TG_CUDA(cudaMalloc(&op->part, sizeof(float) * (size_t)part));
	TG_CUDA(cudaMalloc(&op->err, sizeof(int)));
	TG_CUDA(cudaMemsetAsync(op->err, 0, sizeof(int), s));
	op->bytes = 4 * (sz_f + sz_a + 2 * kmax * layers + part) + 4;
	// A and A^T re-laid tile by tile (a snapshot of A, like the CSC transpose of
	// a sparse operator): every TMA stage then reads 16 KB contiguous
	float *at = nullptr;
	at = (decltype(at))dev_alloc(sizeof(float) * (size_t)(m * n), s);
	dim3 tb(32, 8), tg((unsigned)((n + 31) / 32), (unsigned)((m + 31) / 32));
	k_transpose<<<tg, tb, 0, s>>>(d_A, m, n, at);
	k_tile_major<<<4 * sms, 256, 0, s>>>(d_A, m, n, op->ks_f, sz_f, op->ta);
	k_tile_major<<<4 * sms, 256, 0, s>>>(at, n, m, op->ks_a, sz_a, op->tat);
	TG_CUDA(cudaGetLastError());
	dev_free(at, s);
	op->tm_a = make_map(op->ta, BK, sz_f / BK, BM);
	op->tm_at = make_map(op->tat, BK, sz_a / BK, BM);
	op->tm_xh_f = make_map(op->xh, n, layers, layers);
	op->tm_xl_f = make_map(op->xl, n, layers, layers);
	op->tm_xh_a = make_map(op->xh, m, layers, layers);
	op->tm_xl_a = make_map(op->xl, m, layers, layers);
	return op;
}

void mrhs_apply(cudaStream_t s, const Inst *tab, int inst, int pred, const MrhsOp &op, bool trans, VecSel x,
                VecSel y, unsigned long long *launches) {
	const long long K = trans ? op.m : op.n, M = trans ? op.n : op.m;
	const long long len = K * op.N;
	const int G = trans ? op.grid_a : op.grid_f;
	k_mrhs_split<<<(unsigned)std::min<long long>((len + 255) / 256, 4LL * G), 256, 0, s>>>(
	    tab, inst, pred, x, len, K, op.members, op.xh, op.xl, launches);
	TG_CUDA(cudaGetLastError());
	MrhsArgs a;
	a.tab = tab;
	a.inst = inst;
	a.pred = pred;
	a.members = op.members;
	a.N = op.N;
	a.M = (int)M;
	a.ks = trans ? op.ks_a : op.ks_f;
	a.J = trans ? op.j_a : op.j_f;
	a.T = trans ? op.t_a : op.t_f;
	a.part = op.part;
	a.err = op.err;
	a.launches = launches;
	const CUtensorMap &P = trans ? op.tm_at : op.tm_a;
	const CUtensorMap &QH = trans ? op.tm_xh_a : op.tm_xh_f;
	const CUtensorMap &QL = trans ? op.tm_xl_a : op.tm_xl_f;
	switch (op.N) {
	case 16: launch_mrhs<16>(s, G, P, QH, QL, a); break;
	case 32: launch_mrhs<32>(s, G, P, QH, QL, a); break;
	case 48: launch_mrhs<48>(s, G, P, QH, QL, a); break;
	case 64: launch_mrhs<64>(s, G, P, QH, QL, a); break;
	default: throw Error{TVAL3G_ERR_INTERNAL, "Internal error: unsupported right-hand-side count"};
	}
	TG_CUDA(cudaGetLastError());
	const long long outs = M * op.N;
	k_mrhs_red<<<(unsigned)((outs + 255) / 256), 256, 0, s>>>(tab, inst, pred, y, op.part, (int)M, op.N, a.ks, a.T, G,
	                                                          a.J, op.members, launches);
	TG_CUDA(cudaGetLastError());
}

int mrhs_take_error(cudaStream_t s, const MrhsOp &op) {
	int h = 0;
	TG_CUDA(cudaMemcpyAsync(&h, op.err, sizeof(int), cudaMemcpyDeviceToHost, s));
	TG_CUDA(cudaStreamSynchronize(s));
	if (h) TG_CUDA(cudaMemsetAsync(op.err, 0, sizeof(int), s));
	return h;
}

TG_END
