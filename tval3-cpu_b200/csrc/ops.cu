// Measurement operators (sm_100a); see ops.cuh.
//
//   dense     y = A x: warp per row, float4 loads (2d/mat_mult.h:18-21)
//             y = A^T x: blocks of (1024 columns x row chunk) write partial
//             column sums, a second pass adds the chunks in order
//   CSR       forward: sub-warp per row gather (mkl_csrmv, 2d/mat_mult.h:58-61);
//             adjoint: gather over the device-built CSC (mkl_cscmv, :63-66)
//   rays      forward: warp per ray, lanes take strided Bresenham steps in
//             closed form (2d/mat_mult.h:145-181, 3d/mat_mult.h:241-359);
//             adjoint: pixel-major gather over the ray->pixel index transposed
//             once on the device (deterministic, no atomics in the solve); in
//             2D per pixel tile, through shared memory
#include "ops.cuh"

#include <algorithm>
#include <vector>

#include "async.cuh"

TG_BEGIN

__device__ __forceinline__ const real *vsel(const Inst &I, VecSel s) { return s.m ? I.vm[s.idx] : I.vn[s.idx]; }
__device__ __forceinline__ real *vselw(const Inst &I, VecSel s) { return s.m ? I.vm[s.idx] : I.vn[s.idx]; }

#define OPROLOGUE()                                                                   \
	pdl_launch_next();                                                                \
	if (launches && blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(launches, 1ull);   \
	const int2 tl_ = map.tiles[blockIdx.x];                                           \
	const Inst &I = tab[tl_.x];                                                       \
	const long long local = tl_.y;                                                    \
	pdl_wait_prev();                                                                  \
	if (!pred_ok(*I.ctrl, pred)) return;

// ---------------------------------------------------------------------------
// dense
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_dense_fwd(const Inst *tab, TileMap map, int pred, VecSel xs, VecSel ys,
                                                   unsigned long long *launches) {
	OPROLOGUE();
	const OpDev &op = I.op;
	const long long m = op.m, n = op.n;
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	const long long rt = (m + WARPS - 1) / WARPS;
	const long long layer = local / rt;
	const long long row = (local - layer * rt) * WARPS + warp;
	if (row >= m) return;
	const real *a = op.A + row * n;
	const real *x = vsel(I, xs) + layer * n;
	double acc = 0.0;   // FP64 accumulation of FP32 products
	if (!FP64_BUILD && (n & 3) == 0 && ((reinterpret_cast<uintptr_t>(a) | reinterpret_cast<uintptr_t>(x)) & 15) == 0) {
		const float4 *a4 = reinterpret_cast<const float4 *>(a);
		const float4 *x4 = reinterpret_cast<const float4 *>(x);
		const long long n4 = n >> 2;
		long long j = lane;
		// four row segments in flight per lane; the FMA order is the plain loop's
		for (; j + 96 < n4; j += 128) {
			float4 av[4], xv[4];
#pragma unroll
			for (int u = 0; u < 4; u++) {
				av[u] = __ldg(a4 + j + 32 * u);
				xv[u] = __ldg(x4 + j + 32 * u);
			}
#pragma unroll
			for (int u = 0; u < 4; u++) {
				acc = fma((double)av[u].x, (double)xv[u].x, acc);
				acc = fma((double)av[u].y, (double)xv[u].y, acc);
				acc = fma((double)av[u].z, (double)xv[u].z, acc);
				acc = fma((double)av[u].w, (double)xv[u].w, acc);
			}
		}
		for (; j < n4; j += 32) {
			float4 av = __ldg(a4 + j), xv = __ldg(x4 + j);
			acc = fma((double)av.x, (double)xv.x, acc);
			acc = fma((double)av.y, (double)xv.y, acc);
			acc = fma((double)av.z, (double)xv.z, acc);
			acc = fma((double)av.w, (double)xv.w, acc);
		}
	} else {
		for (long long j = lane; j < n; j += 32) acc = fma((double)__ldg(a + j), (double)__ldg(x + j), acc);
	}
	acc = warp_sum(acc);
	if (lane == 0) vselw(I, ys)[layer * m + row] = (real)acc;
}

// partial column sums of A^T x over one row chunk
__global__ void __launch_bounds__(256) k_dense_adj(const Inst *tab, TileMap map, int pred, VecSel xs,
                                                   VecSel ys, real *part, unsigned long long *launches) {
	OPROLOGUE();
	const OpDev &op = I.op;
	const long long m = op.m, n = op.n;
	const int K = op.dense_kchunks;
	const long long ct_n = (n + 1023) / 1024;
	const long long layer = local / (ct_n * K);
	const long long rem = local - layer * ct_n * K;
	const long long ct = rem / K, kc = rem - ct * K;
	const long long rows_per = (m + K - 1) / K;
	const long long r0 = kc * rows_per, r1 = min(m, r0 + rows_per);
	const long long c0 = ct * 1024 + threadIdx.x * 4;
	const real *x = vsel(I, xs) + layer * m;
	double acc0 = 0.0, acc1 = 0.0, acc2 = 0.0, acc3 = 0.0;   // FP64 accumulation
	if (!FP64_BUILD && (n & 3) == 0 && (reinterpret_cast<uintptr_t>(op.A) & 15) == 0) {
		if (c0 < n) {
			long long r = r0;
			// four rows in flight per thread; the FMA order is the plain loop's
			for (; r + 3 < r1; r += 4) {
				real xv[4];
				float4 av[4];
#pragma unroll
				for (int u = 0; u < 4; u++) {
					xv[u] = __ldg(x + r + u);
					av[u] = __ldg(reinterpret_cast<const float4 *>(op.A + (r + u) * n + c0));
				}
#pragma unroll
				for (int u = 0; u < 4; u++) {
					acc0 = fma((double)av[u].x, (double)xv[u], acc0);
					acc1 = fma((double)av[u].y, (double)xv[u], acc1);
					acc2 = fma((double)av[u].z, (double)xv[u], acc2);
					acc3 = fma((double)av[u].w, (double)xv[u], acc3);
				}
			}
			for (; r < r1; r++) {
				real xv = __ldg(x + r);
				float4 av = __ldg(reinterpret_cast<const float4 *>(op.A + r * n + c0));
				acc0 = fma((double)av.x, (double)xv, acc0);
				acc1 = fma((double)av.y, (double)xv, acc1);
				acc2 = fma((double)av.z, (double)xv, acc2);
				acc3 = fma((double)av.w, (double)xv, acc3);
			}
		}
	} else {
		for (long long r = r0; r < r1; r++) {
			real xv = __ldg(x + r);
			const real *ar = op.A + r * n;
			if (c0 + 0 < n) acc0 = fma((double)__ldg(ar + c0 + 0), (double)xv, acc0);
			if (c0 + 1 < n) acc1 = fma((double)__ldg(ar + c0 + 1), (double)xv, acc1);
			if (c0 + 2 < n) acc2 = fma((double)__ldg(ar + c0 + 2), (double)xv, acc2);
			if (c0 + 3 < n) acc3 = fma((double)__ldg(ar + c0 + 3), (double)xv, acc3);
		}
	}
	real *p = part + op.dense_part + (layer * K + kc) * n;
	if (c0 + 0 < n) p[c0 + 0] = (real)acc0;
	if (c0 + 1 < n) p[c0 + 1] = (real)acc1;
	if (c0 + 2 < n) p[c0 + 2] = (real)acc2;
	if (c0 + 3 < n) p[c0 + 3] = (real)acc3;
}

// y = sum of the K row-chunk partials, 32 columns per block: warp w adds the
// partials k = w, w + 8, ... of its lane's column, then warp 0 adds the eight
// warp sums in a fixed order (deterministic)
__global__ void __launch_bounds__(256) k_dense_red(const Inst *tab, TileMap map, int pred, VecSel xs, VecSel ys,
                                                   const real *part, unsigned long long *launches) {
	OPROLOGUE();
	__shared__ double ws[8][32];
	const OpDev &op = I.op;
	const long long n = op.n;
	const int K = op.dense_kchunks;
	const long long ct_n = (n + 31) / 32;
	const long long layer = local / ct_n, ct = local - layer * ct_n;
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	const long long c = ct * 32 + lane;
	const real *p = part + op.dense_part + layer * K * n;
	double s = 0.0;
	if (c < n)
		for (int k = warp; k < K; k += 8) s += p[(long long)k * n + c];
	ws[warp][lane] = s;
	__syncthreads();
	if (warp == 0 && c < n) {
		double t = ws[0][lane];
		for (int w = 1; w < 8; w++) t += ws[w][lane];
		vselw(I, ys)[layer * n + c] = (real)t;
	}
}

#ifndef TVAL3G_FP64   // one-pass dense normal product: FP32 data only
// ---------------------------------------------------------------------------
// dense normal product, A read once (get_g_mult's cache-blocked dense path,
// 2d/tval3_cpu_2d.cpp:361-394): Au = A u and g = A^T Au in one pass over A.
// A is cut into bands of R = grid x rpc rows; CTA c owns rows c rpc ..
// c rpc + rpc - 1 of every band and the column slab [c S, c S + S) of g.
// Each CTA's warps take three roles that run concurrently:
//   producer (warp 0): streams the CTA's rows, chunk by chunk, with the
//     matching chunk of u, into a ring of shared-memory stages by bulk
//     asynchronous copies (full / empty barriers per stage);
//   consumers (warps 1-7): the rows' dot products from the stages; thread 0
//     of the role writes each row of Au and, after the band's rows, publishes
//     them with a release increment of flags[band];
//   reducers (warps 8-15): band after band, once all rows of the band are
//     published, the slab of A_band^T Au_band added into FP64 accumulators
//     kept for the whole launch - the band is read again from L2, where the
//     producer just brought it.
// The producer starts band b only when its CTA's reducers have finished band
// b - 2, so two bands at most are in L2.  All CTAs must be co-resident
// (cooperative launch).  Every wait is bounded: one that gives up sets *err
// and the CTA's abort flag, after which no role waits again (every named
// barrier is still passed the same number of times) and the producer lets
// its copies in flight land before the CTA exits.  Products are summed in
// FP32 over short runs (a thread's share of one chunk of a row; eight rows of
// a column) and those sums in FP64, in a fixed order: deterministic.
// ---------------------------------------------------------------------------
constexpr int FUSED_THREADS = 512;
constexpr int FUSED_ROLE = 256;                     // reducer threads
constexpr int FUSED_CONS = 224;                     // consumer threads (warps 1-7)
constexpr int FUSED_RPC_MAX = 16;                   // rows per CTA per band
constexpr int FUSED_GRID_MAX = 160;
constexpr int FUSED_NS = 4;                         // ring stages
constexpr int FUSED_CH = 4096;                      // floats per chunk (16 KB of A, 16 KB of u)
constexpr int FUSED_STAGE_BYTES = 2 * FUSED_CH * 4;
constexpr int FUSED_DYN_BYTES = FUSED_NS * FUSED_STAGE_BYTES + 2 * FUSED_NS * 8;
constexpr long long FUSED_BAND_BYTES = 24LL << 20;  // target band size
constexpr long long FUSED_L2_BYTES = 96LL << 20;    // two bands must stay in L2
constexpr unsigned FUSED_SPIN_MAX = 1u << 21;       // bounded waits (~0.2 s)

__device__ __forceinline__ int ld_acquire(const int *p) {
	int v;
	asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
	return v;
}
__device__ __forceinline__ void named_sync(int id, int threads) {   // barrier of one role's threads
	asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(threads) : "memory");
}
// one thread polls a stage barrier; false (err raised) if it gives up
__device__ __forceinline__ bool mbar_wait1(unsigned bar, unsigned parity, int *err) {
	for (unsigned i = 0; i < ASYNC_WAIT_LIMIT; i++)
		if (mbar_try(bar, parity)) return true;
	atomicExch(err, 1);
	return false;
}

__global__ void __launch_bounds__(FUSED_THREADS, 1) k_dense_normal(const Inst *tab, int inst, int pred, VecSel us,
                                                                   VecSel aus, VecSel gs, int *flags, int *err,
                                                                   unsigned long long *launches) {
	if (launches && blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(launches, 1ull);
	const Inst &I = tab[inst];
	if (!pred_ok(*I.ctrl, pred)) return;   // the same in every CTA: ctrl is not written here
	extern __shared__ __align__(128) unsigned char dsm[];
	__shared__ float sauf[FUSED_GRID_MAX * FUSED_RPC_MAX];   // the band's Au (reducers)
	__shared__ double sau[FUSED_GRID_MAX * FUSED_RPC_MAX];   // the row groups' column sums
	__shared__ double spart[2][8];                           // consumer warps' row partials
	__shared__ volatile int s_done, s_abort;                 // bands reduced; a wait gave up
	const OpDev &op = I.op;
	const int m = (int)op.m, n = (int)op.n;
	const int G = gridDim.x, c = blockIdx.x, rpc = op.fused_rpc, R = G * rpc;
	const int nb = (m + R - 1) / R, nch = (n + FUSED_CH - 1) / FUSED_CH;
	const float *A = op.A;
	const int S = op.fused_slab;   // slab width, a multiple of 4
	const int c0 = min(n, c * S), c1 = min(n, c0 + S);
	const unsigned full0 = smem_u32(dsm + FUSED_NS * FUSED_STAGE_BYTES), empty0 = full0 + 8u * FUSED_NS;
	auto stage_a = [&](int st) { return reinterpret_cast<float4 *>(dsm + st * FUSED_STAGE_BYTES); };
	auto stage_u = [&](int st) { return reinterpret_cast<float4 *>(dsm + st * FUSED_STAGE_BYTES + FUSED_CH * 4); };
	if (threadIdx.x == 0) {
		s_done = 0;
		s_abort = 0;
		for (int st = 0; st < FUSED_NS; st++) {
			mbar_init(full0 + 8u * st, 1);
			mbar_init(empty0 + 8u * st, FUSED_CONS / 32);
		}
		fence_mbar_init();
	}
	__syncthreads();
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	if (warp == 0) {
		// ---- producer ----
		if (lane == 0) {
			const float *u = vsel(I, us);
			// A's lines are read again by the reducers of other CTAs (from L2):
			// kept there until then; u is read for every row
			const unsigned long long keep = l2_policy_evict_last();
			long long it = 0;
			for (int b = 0; b < nb && !s_abort; b++) {
				for (unsigned sp = 0; s_done < b - 1 && !s_abort; sp++) {
					if (sp > FUSED_SPIN_MAX) { atomicExch(err, 1); s_abort = 1; }
					__nanosleep(32);
				}
				const int r0 = b * R + c * rpc;
				for (int j = 0; j < rpc && r0 + j < m && !s_abort; j++)
					for (int ch = 0; ch < nch && !s_abort; ch++, it++) {
						const int st = (int)(it % FUSED_NS);
						const long long ph = it / FUSED_NS;
						if (ph > 0 && !mbar_wait1(empty0 + 8u * st, (unsigned)(ph - 1) & 1u, err)) {
							s_abort = 1;
							break;
						}
						const int cnt = min(FUSED_CH, n - ch * FUSED_CH);
						mbar_expect_tx(full0 + 8u * st, 8u * cnt);
						bulk_g2s_hint(smem_u32(stage_a(st)), A + (long long)(r0 + j) * n + (long long)ch * FUSED_CH,
						              4u * cnt, full0 + 8u * st, keep);
						bulk_g2s_hint(smem_u32(stage_u(st)), u + (long long)ch * FUSED_CH, 4u * cnt, full0 + 8u * st,
						              keep);
					}
			}
			if (s_abort)   // let the copies in flight land before the CTA exits (bounded)
				for (long long k = it > FUSED_NS ? it - FUSED_NS : 0; k < it; k++)
					mbar_wait1(full0 + 8u * (int)(k % FUSED_NS), (unsigned)(k / FUSED_NS) & 1u, err);
		}
	} else if (warp < 8) {
		// ---- consumers ----
		const int ct = threadIdx.x - 32, cw = warp - 1;
		float *au = vselw(I, aus);
		long long it = 0;
		int rowc = 0;
		for (int b = 0; b < nb; b++) {
			const int r0 = b * R + c * rpc;
			for (int j = 0; j < rpc && r0 + j < m; j++, rowc++) {
				double acc = 0.0;
				for (int ch = 0; ch < nch; ch++, it++) {
					const int st = (int)(it % FUSED_NS);
					if (!s_abort && !mbar_wait_warp(full0 + 8u * st, (unsigned)(it / FUSED_NS) & 1u, err))
						if (lane == 0) s_abort = 1;
					if (!s_abort) {
						// the thread's few products of this chunk (at most 19
						// float4) summed in FP32, the chunk sums in FP64: one
						// conversion per chunk instead of two per element
						const int cnt4 = min(FUSED_CH, n - ch * FUSED_CH) >> 2;
						const float4 *sa = stage_a(st), *su = stage_u(st);
						float pf = 0.f;
						for (int k = ct; k < cnt4; k += FUSED_CONS) {
							const float4 av = sa[k], uv = su[k];
							pf = fmaf(av.x, uv.x, pf);
							pf = fmaf(av.y, uv.y, pf);
							pf = fmaf(av.z, uv.z, pf);
							pf = fmaf(av.w, uv.w, pf);
						}
						acc += (double)pf;
					}
					__syncwarp();
					if (lane == 0) mbar_arrive(empty0 + 8u * st);
				}
				acc = warp_sum(acc);
				if (lane == 0) spart[rowc & 1][cw] = acc;
				named_sync(1, FUSED_CONS);
				if (ct == 0) {
					double t = 0.0;
					for (int w = 0; w < FUSED_CONS / 32; w++) t += spart[rowc & 1][w];
					au[r0 + j] = (float)t;
				}
			}
			if (ct == 0 && r0 < m) {
				__threadfence();
				atomicAdd(&flags[b], 1);
			}
		}
	} else {
		// ---- reducers ----
		const int t = threadIdx.x - FUSED_ROLE;
		const float *au = vsel(I, aus);
		const int SV = S / 4;                                   // float4 per slab row
		const int Q = SV >= FUSED_ROLE ? 1 : FUSED_ROLE / SV;   // row groups
		const int j = t % SV, q = t / SV;
		const bool act = q < Q && c0 + 4 * j < c1;
		const unsigned long long last_use = l2_policy_evict_first();   // the second and last read of A's lines
		double acc[4] = {0.0, 0.0, 0.0, 0.0};
		for (int b = 0; b < nb; b++) {
			const int r0 = b * R, rows = min(R, m - r0);
			const int expect = min(G, (rows + rpc - 1) / rpc);
			if (t == 0 && !s_abort) {
				unsigned sp = 0;
				while (ld_acquire(flags + b) < expect) {
					if (++sp > FUSED_SPIN_MAX) { atomicExch(err, 1); s_abort = 1; break; }
					__nanosleep(32);
				}
			}
			named_sync(2, FUSED_ROLE);
			for (int k = t; k < rows; k += FUSED_ROLE) sauf[k] = __ldcg(au + r0 + k);
			named_sync(2, FUSED_ROLE);
			if (act && !s_abort) {
				// eight rows' products summed in FP32, those sums in FP64
				const float *a = A + (long long)r0 * n + c0 + 4 * j;
				int r = q;
				for (; r + 7 * Q < rows; r += 8 * Q) {
					float4 v[8];
#pragma unroll
					for (int e = 0; e < 8; e++) v[e] = ld_f4_hint(a + (long long)(r + e * Q) * n, last_use);
					float p0 = 0.f, p1 = 0.f, p2 = 0.f, p3 = 0.f;
#pragma unroll
					for (int e = 0; e < 8; e++) {
						const float w = sauf[r + e * Q];
						p0 = fmaf(v[e].x, w, p0);
						p1 = fmaf(v[e].y, w, p1);
						p2 = fmaf(v[e].z, w, p2);
						p3 = fmaf(v[e].w, w, p3);
					}
					acc[0] += (double)p0;
					acc[1] += (double)p1;
					acc[2] += (double)p2;
					acc[3] += (double)p3;
				}
				for (; r < rows; r += Q) {
					const float w = sauf[r];
					const float4 v = ld_f4_hint(a + (long long)r * n, last_use);
					acc[0] += (double)(v.x * w);
					acc[1] += (double)(v.y * w);
					acc[2] += (double)(v.z * w);
					acc[3] += (double)(v.w * w);
				}
			}
			named_sync(2, FUSED_ROLE);
			if (t == 0) {
				__threadfence_block();
				s_done = b + 1;
			}
		}
		// the row groups' sums of each column, in group order
		double *sred = sau;   // Q x S doubles (Q S <= 4 x 256)
		if (act)
#pragma unroll
			for (int e = 0; e < 4; e++) sred[q * S + 4 * j + e] = acc[e];
		named_sync(2, FUSED_ROLE);
		float *gv = vselw(I, gs);
		for (int col = t; col < c1 - c0; col += FUSED_ROLE) {
			double tot = 0.0;
			for (int qq = 0; qq < Q; qq++) tot += sred[qq * S + col];
			gv[c0 + col] = (float)tot;
		}
	}
}

int fused_grid() {
	int dev = 0, sms = 0;
	TG_CUDA(cudaGetDevice(&dev));
	TG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
	TG_CUDA(cudaFuncSetAttribute(k_dense_normal, cudaFuncAttributeMaxDynamicSharedMemorySize, FUSED_DYN_BYTES));
	return std::max(1, std::min(sms, FUSED_GRID_MAX));
}

int fused_rows_per_cta(long long m, long long n, int grid, const float *A, int *slab) {
	// rows are streamed by 16-byte bulk copies: n % 4 == 0 and A 16-byte aligned
	if (m < 1 || n < 1 || m >= (1LL << 31) || n % 4 != 0 || (reinterpret_cast<uintptr_t>(A) & 15) != 0) return 0;
	long long S = (n + grid - 1) / grid;   // slab width, a multiple of 4
	S = (S + 3) / 4 * 4;
	const long long SV = S / 4;
	if (SV > FUSED_ROLE) return 0;        // one float4 per reducer thread and slab row
	const long long Q = FUSED_ROLE / SV;  // row groups
	if (Q * S > (long long)FUSED_GRID_MAX * FUSED_RPC_MAX) return 0;   // their sums reuse the band buffer
	const long long row = 4 * n;
	long long rpc = FUSED_BAND_BYTES / (grid * row);
	rpc = std::max(1LL, std::min<long long>(rpc, FUSED_RPC_MAX));
	if (2 * grid * rpc * row > FUSED_L2_BYTES) return 0;
	*slab = (int)S;
	return (int)rpc;
}

#else   // FP64 build: no one-pass normal product (dense normal products take the gemv kernels)
int fused_grid() { return 1; }
int fused_rows_per_cta(long long, long long, int, const real *, int *) { return 0; }
#endif
// ---------------------------------------------------------------------------
// compressed gather: y[line] = w * sum_k val[k] * x[ind[k]] over a line's range
//   kind 0: CSR rows (forward), kind 1: CSC columns (adjoint of CSR),
//   kind 2: ray adjoint (implicit weight = scale, ind = measurement index)
// ---------------------------------------------------------------------------
template <int W>
__global__ void __launch_bounds__(256) k_gather(const Inst *tab, TileMap map, int pred, int kind, VecSel xs,
                                                VecSel ys, unsigned long long *launches) {
	OPROLOGUE();
	const OpDev &op = I.op;
	const int *ptr, *ind;
	const real *val;
	long long lines, xlen, ylen;
	if (kind == 0) { ptr = op.rptr; ind = op.rind; val = op.rval; lines = op.m; xlen = op.n; ylen = op.m; }
	else if (kind == 1) { ptr = op.cptr; ind = op.cind; val = op.cval; lines = op.n; xlen = op.m; ylen = op.n; }
	else { ptr = op.cptr; ind = op.cind; val = nullptr; lines = I.n; xlen = 0; ylen = 0; }
	constexpr int LPB = 256 / W;   // lines per block
	const long long lt = (lines + LPB - 1) / LPB;
	const long long layer = local / lt;
	const long long line = (local - layer * lt) * LPB + threadIdx.x / W;
	const int gl = threadIdx.x % W;
	const real *x = vsel(I, xs) + layer * xlen;
	double acc = 0.0;   // FP64 accumulation of FP32 products
	if (line < lines) {
		// four of the lane's entries per step: their indices, then the four
		// gathers, in flight together; summed in the lane's entry order
		const int k0 = ptr[line], k1 = ptr[line + 1];
		int k = k0 + gl;
		if (val) {
			for (; k + 3 * W < k1; k += 4 * W) {
				int ii[4];
				real vv[4], xx[4];
#pragma unroll
				for (int u = 0; u < 4; u++) {
					ii[u] = __ldg(ind + k + u * W);
					vv[u] = __ldg(val + k + u * W);
				}
#pragma unroll
				for (int u = 0; u < 4; u++) xx[u] = __ldg(x + ii[u]);
#pragma unroll
				for (int u = 0; u < 4; u++) acc = fma((double)vv[u], (double)xx[u], acc);
			}
			for (; k < k1; k += W) acc = fma((double)__ldg(val + k), (double)__ldg(x + __ldg(ind + k)), acc);
		} else {
			for (; k + 3 * W < k1; k += 4 * W) {
				int ii[4];
				real xx[4];
#pragma unroll
				for (int u = 0; u < 4; u++) ii[u] = __ldg(ind + k + u * W);
#pragma unroll
				for (int u = 0; u < 4; u++) xx[u] = __ldg(x + ii[u]);
#pragma unroll
				for (int u = 0; u < 4; u++) acc += xx[u];
			}
			for (; k < k1; k += W) acc += __ldg(x + __ldg(ind + k));
		}
	}
#pragma unroll
	for (int o = W / 2; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
	if (gl == 0 && line < lines) vselw(I, ys)[layer * ylen + line] = (real)(val ? acc : acc * op.scale);
}

// ---------------------------------------------------------------------------
// rays
// ---------------------------------------------------------------------------
struct RayWalk {
	int x0, y0, z0, sx, sy, sz, out;
	int drive;        // 0 x, 1 y, 2 z
	int M;            // driving length; the ray has M + 1 hits
	int a1, a2;       // |delta| of the two minor axes (in axis order, skipping drive)
	__device__ RayWalk(int4 pk) {
		int dx, dy, dz;
		unpack_ray(pk, x0, y0, z0, dx, dy, dz, out);
		sx = dx < 0 ? -1 : 1; sy = dy < 0 ? -1 : 1; sz = dz < 0 ? -1 : 1;
		int mx = abs(dx), my = abs(dy), mz = abs(dz);
		// 3d/mat_mult.h:241,280 (2D: mz = 0 gives 2d/mat_mult.h:160's le >= m)
		if (mx >= my && mx >= mz) { drive = 0; M = mx; a1 = my; a2 = mz; }
		else if (my >= mx && my >= mz) { drive = 1; M = my; a1 = mx; a2 = mz; }
		else { drive = 2; M = mz; a1 = mx; a2 = my; }
	}
	// linear index of step j given the minor offsets k1, k2
	__device__ __forceinline__ long long index(int j, int k1, int k2, int rvx, long long rvxy) const {
		int x, y, z;
		if (drive == 0) { x = x0 + sx * j; y = y0 + sy * k1; z = z0 + sz * k2; }
		else if (drive == 1) { x = x0 + sx * k1; y = y0 + sy * j; z = z0 + sz * k2; }
		else { x = x0 + sx * k1; y = y0 + sy * k2; z = z0 + sz * j; }
		return (long long)x + (long long)y * rvx + (long long)z * rvxy;
	}
};

// minor-axis offset after j driving steps: floor((2 j a + M - 1) / (2 M)),
// advanced by `stride` steps at a time with exact integer carries
struct MinorStep {
	int q, r, qa, ra, twoM;
	__device__ MinorStep(int j, int a, int M, int stride) {
		if (M == 0) { q = r = qa = ra = 0; twoM = 1; return; }
		twoM = 2 * M;
		int num = 2 * j * a + M - 1;
		q = num / twoM; r = num - q * twoM;
		int inc = 2 * stride * a;
		qa = inc / twoM; ra = inc - qa * twoM;
	}
	__device__ __forceinline__ void advance() {
		q += qa; r += ra;
		if (r >= twoM) { r -= twoM; q++; }
	}
};

// Forward projection, SUBW lanes per ray.  Lane l takes the hits j = l,
// l + SUBW, ...; the linear index advances by SUBW driving steps plus, per
// minor axis, the exact quotient / remainder increments of the closed form
// floor((2 j a + M - 1) / (2 M)) - one add and one compare-carry per axis.
// All index arithmetic is 32-bit (images and volumes are below 2^31 voxels,
// extents below 2^15).
template <int SUBW, bool D3>
__global__ void __launch_bounds__(256) k_ray_fwd(const Inst *tab, TileMap map, int pred, VecSel xs, VecSel ys,
                                                 unsigned long long *launches) {
	OPROLOGUE();
	const OpDev &op = I.op;
	constexpr int RPB = 256 / SUBW;   // rays per block
	const int gl = threadIdx.x % SUBW;
	const long long ray = local * RPB + threadIdx.x / SUBW;
	const real *x = vsel(I, xs);
	double acc = 0.0;   // FP64 accumulation along the ray (of FP32 sums of four hits)
	int out = -1;
	if (ray < op.nrays) {
		int x0, y0, z0, dx, dy, dz;
		unpack_ray(op.rays[ray], x0, y0, z0, dx, dy, dz, out);
		const int mx = abs(dx), my = abs(dy), mz = D3 ? abs(dz) : 0;
		const int sx = dx < 0 ? -1 : 1, sy = (dy < 0 ? -1 : 1) * op.rvx;
		const int sz = (dz < 0 ? -1 : 1) * op.rvx * op.rvy;
		// driving axis (3d/mat_mult.h:241,280; 2D: 2d/mat_mult.h:160)
		int M, a1, a2, sd, s1, s2;
		int idx = x0 + y0 * op.rvx + z0 * op.rvx * op.rvy;
		if (mx >= my && mx >= mz) { M = mx; sd = sx; a1 = my; s1 = sy; a2 = mz; s2 = sz; }
		else if (my >= mx && my >= mz) {
			M = my; sd = sy; a1 = mx; s1 = sx; a2 = mz; s2 = sz;
			if (!D3 && op.xT) {   // transposed image: y steps are contiguous
				x = op.xT;
				idx = y0 + x0 * op.tH;
				sd = dy < 0 ? -1 : 1;
				s1 = (dx < 0 ? -1 : 1) * op.tH;
			}
		} else { M = mz; sd = sz; a1 = mx; s1 = sx; a2 = my; s2 = sy; }
		idx += gl * sd;
		const int twoM = 2 * M > 0 ? 2 * M : 1;
		int q1 = 0, r1 = 0, qa1 = 0, ra1 = 0, q2 = 0, r2 = 0, qa2 = 0, ra2 = 0;
		if (M > 0) {
			int num = 2 * gl * a1 + M - 1;
			q1 = num / twoM; r1 = num - q1 * twoM;
			qa1 = (2 * SUBW * a1) / twoM; ra1 = 2 * SUBW * a1 - qa1 * twoM;
			idx += q1 * s1;
			if (D3) {
				num = 2 * gl * a2 + M - 1;
				q2 = num / twoM; r2 = num - q2 * twoM;
				qa2 = (2 * SUBW * a2) / twoM; ra2 = 2 * SUBW * a2 - qa2 * twoM;
				idx += q2 * s2;
			}
		}
		const int dstep = SUBW * sd + qa1 * s1 + (D3 ? qa2 * s2 : 0);
		auto step = [&]() {
			idx += dstep;
			r1 += ra1;
			if (r1 >= twoM) { r1 -= twoM; idx += s1; }
			if (D3) {
				r2 += ra2;
				if (r2 >= twoM) { r2 -= twoM; idx += s2; }
			}
		};
		// four of the lane's hits summed in FP32, those sums in FP64 (one
		// conversion per four hits)
		int j = gl;
		for (; j + 3 * SUBW <= M; j += 4 * SUBW) {
			real v[4];
#pragma unroll
			for (int u = 0; u < 4; u++) {
				v[u] = __ldg(x + idx);
				step();
			}
			acc += (double)((v[0] + v[1]) + (v[2] + v[3]));
		}
		real rest = 0.f;
		for (; j <= M; j += SUBW) {
			rest += __ldg(x + idx);
			step();
		}
		acc += (double)rest;
	}
#pragma unroll
	for (int o = SUBW / 2; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
	if (gl == 0 && out >= 0) vselw(I, ys)[out] = (real)(acc * op.scale);
}

// The adjoint by on-the-fly tracing (TVAL3G_RAY_ADJ_ATOMICS): lanes and
// steps as in k_ray_fwd (always the image's own layout), each hit adding
// scale * y[ray] to its pixel with an atomic add into the zeroed output.
// The order of the adds varies from run to run, so the sums are not
// bit-reproducible; the gather adjoints are.
__global__ void __launch_bounds__(256) k_ray_atomic_zero(const Inst *tab, TileMap map, int pred, VecSel ys,
                                                         unsigned long long *launches) {
	OPROLOGUE();
	real *out = vselw(I, ys);
	const long long i0 = local * ATOMIC_ZERO_TILE;
	for (long long i = i0 + threadIdx.x; i < min(I.n, i0 + ATOMIC_ZERO_TILE); i += blockDim.x) out[i] = 0.f;
}

template <bool D3>
__global__ void __launch_bounds__(256) k_ray_adj_atomic(const Inst *tab, TileMap map, int pred, VecSel xs,
                                                        VecSel ys, unsigned long long *launches) {
	OPROLOGUE();
	const OpDev &op = I.op;
	constexpr int SUBW = RAY_SUBW, RPB = 256 / SUBW;
	const int gl = threadIdx.x % SUBW;
	const long long ray = local * RPB + threadIdx.x / SUBW;
	if (ray >= op.nrays) return;
	real *g = vselw(I, ys);
	int x0, y0, z0, dx, dy, dz, out;
	unpack_ray(op.rays[ray], x0, y0, z0, dx, dy, dz, out);
	const real w = vsel(I, xs)[out] * op.scale;
	const int mx = abs(dx), my = abs(dy), mz = D3 ? abs(dz) : 0;
	const int sx = dx < 0 ? -1 : 1, sy = (dy < 0 ? -1 : 1) * op.rvx;
	const int sz = (dz < 0 ? -1 : 1) * op.rvx * op.rvy;
	int M, a1, a2, sd, s1, s2;
	int idx = x0 + y0 * op.rvx + z0 * op.rvx * op.rvy;
	if (mx >= my && mx >= mz) { M = mx; sd = sx; a1 = my; s1 = sy; a2 = mz; s2 = sz; }
	else if (my >= mx && my >= mz) { M = my; sd = sy; a1 = mx; s1 = sx; a2 = mz; s2 = sz; }
	else { M = mz; sd = sz; a1 = mx; s1 = sx; a2 = my; s2 = sy; }
	idx += gl * sd;
	const int twoM = 2 * M > 0 ? 2 * M : 1;
	int r1 = 0, qa1 = 0, ra1 = 0, r2 = 0, qa2 = 0, ra2 = 0;
	if (M > 0) {
		int num = 2 * gl * a1 + M - 1;
		int q = num / twoM;
		r1 = num - q * twoM;
		qa1 = (2 * SUBW * a1) / twoM; ra1 = 2 * SUBW * a1 - qa1 * twoM;
		idx += q * s1;
		if (D3) {
			num = 2 * gl * a2 + M - 1;
			q = num / twoM;
			r2 = num - q * twoM;
			qa2 = (2 * SUBW * a2) / twoM; ra2 = 2 * SUBW * a2 - qa2 * twoM;
			idx += q * s2;
		}
	}
	const int dstep = SUBW * sd + qa1 * s1 + (D3 ? qa2 * s2 : 0);
	for (int j = gl; j <= M; j += SUBW) {
		atomicAdd(g + idx, w);
		idx += dstep;
		r1 += ra1;
		if (r1 >= twoM) { r1 -= twoM; idx += s1; }
		if (D3) {
			r2 += ra2;
			if (r2 >= twoM) { r2 -= twoM; idx += s2; }
		}
	}
}

// xT[y + x*tH] = x[x + y*ld] for the 2D forward (32x32 tiles through shared
// memory; local tile = ty * ceil(ld/32) + tx)
__global__ void __launch_bounds__(256) k_transpose2d(const Inst *tab, TileMap map, int pred, VecSel xs,
                                                     unsigned long long *launches) {
	OPROLOGUE();
	__shared__ real tile[32][33];
	const OpDev &op = I.op;
	const int ld = op.rvx, H = op.tH;
	const int ntx = (ld + 31) / 32;
	const int bx = (int)local % ntx, by = (int)local / ntx;
	const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
	const real *X = vsel(I, xs);
#pragma unroll
	for (int j = 0; j < 32; j += 8) {
		const int x = bx * 32 + tx, y = by * 32 + ty + j;
		if (x < ld && y < H) tile[ty + j][tx] = X[x + y * ld];
	}
	__syncthreads();
#pragma unroll
	for (int j = 0; j < 32; j += 8) {
		const int y = by * 32 + tx, x = bx * 32 + ty + j;
		if (x < ld && y < H) op.xT[y + x * H] = tile[tx][ty + j];
	}
}

#ifndef TVAL3G_FP64   // tiled ray adjoints: FP32 data only
// ---------------------------------------------------------------------------
// tiled 2D ray adjoint
// ---------------------------------------------------------------------------
__global__ void k_to_int(const long long *in, int *out, long long n);

constexpr int RAYT_THREADS = RAYT * RAYT;   // one thread per pixel of a tile
constexpr int RAYT_WARPS = RAYT_THREADS / 32;

// Two threads per pixel: warp w and warp w + 8 of a block take the first and
// the second half of the words of pixel-warp w (its 32 pixels), and each
// warp streams its half through a ring of RAYT_STAGES shared-memory stages of
// RAYT_CW words per lane (1 KB), filled by bulk asynchronous copies that lane
// 0 issues ahead of use - two blocks per SM keep 64 KB of index in flight
// without holding it in registers.
constexpr int RAYT_ADJ_THREADS = 2 * RAYT_THREADS;      // two threads per pixel
constexpr int RAYT_ADJ_WARPS = RAYT_ADJ_THREADS / 32;
constexpr int RAYT_STAGES = 2;
constexpr int RAYT_CW = 2;                               // 16-byte words per lane per stage
constexpr int RAYT_STAGE_WORDS = RAYT_CW * 32;           // per warp
constexpr int RAYT_RING_BYTES = RAYT_ADJ_WARPS * RAYT_STAGES * RAYT_STAGE_WORDS * 16;
constexpr int RAYT_BAR_BYTES = (RAYT_ADJ_WARPS * RAYT_STAGES + 2) * 8;   // the rings' barriers, the list's
constexpr int RAYT_SACC_BYTES = RAYT_THREADS * 8;        // the second halves' sums
constexpr int RAYT_LIST_CHUNK = 8192;                    // list entries per bulk copy
constexpr int RAYT_ZERO_TILES = 64;                      // tiles without rays zeroed per block

// ring, barriers, second-half sums, then the tile's measurements: slot 0
// (the zero pad entries read) sits 12 bytes past a 16-byte boundary so that
// slots 1.. are aligned for the bulk copy of the list
int tiled_smem_bytes(int tmax) {
	return RAYT_RING_BYTES + RAYT_BAR_BYTES + RAYT_SACC_BYTES + 12 + (int)sizeof(float) * (tmax + 1);
}

// the eight entries of a 16-byte index word, summed in a fixed tree
__device__ __forceinline__ float word_sum(const float *yt, uint4 q) {
	return ((yt[q.x & 0xffff] + yt[q.x >> 16]) + (yt[q.y & 0xffff] + yt[q.y >> 16])) +
	       ((yt[q.z & 0xffff] + yt[q.z >> 16]) + (yt[q.w & 0xffff] + yt[q.w >> 16]));
}

// g[p] = scale * sum over the rays through p of y[ray] (the transposed
// projection of 2d/mat_mult.h:145-181).  Block per RAYT x RAYT tile: the
// measurements of the rays crossing the tile are gathered into shared memory
// (slot 0 holds the zero that pad entries read), then every thread sums its
// pixel's entries in ray order - eight per 16-byte word in FP32, the words in
// FP64 - from its lane's column of the warp's interleaved words, which reach
// shared memory through the warp's ring of bulk copies (issued before the
// gather, so the first stages arrive meanwhile).  Threads take the tile's
// pixels in order of decreasing hit count (OpDev::tperm), so a warp's pixels
// have lists of nearly one length and its words carry little padding.
// Deterministic, no atomics.
// g at pixel px (0 .. RAYT^2 - 1, row-major in the tile) of tile (brick) t
__device__ __forceinline__ void tiled_store(const Inst &I, const OpDev &op, VecSel ys, int t, int px, float v) {
	if (op.tile3) {   // brick of BRICK_X x BRICK_Y x BRICK_Z voxels
		const int bxy = op.ntx * op.nty;
		const int x = (t % op.ntx) * BRICK_X + px % BRICK_X;
		const int y = ((t % bxy) / op.ntx) * BRICK_Y + (px / BRICK_X) % BRICK_Y;
		const int z = (t / bxy) * BRICK_Z + px / (BRICK_X * BRICK_Y);
		if (x < op.rvx && y < op.rvy && (long long)z * op.rvx * op.rvy < I.n)
			vselw(I, ys)[x + (long long)y * op.rvx + (long long)z * op.rvx * op.rvy] = v;
		return;
	}
	const int x = (t % op.ntx) * RAYT + (px % RAYT), row = (t / op.ntx) * RAYT + (px / RAYT);
	if (x < op.rvx && row < op.tH) vselw(I, ys)[x + row * op.rvx] = v;
}

__global__ void __launch_bounds__(RAYT_ADJ_THREADS) k_ray_adj_tiled(const Inst *tab, TileMap map, int pred,
                                                                    VecSel xs, VecSel ys, int *err,
                                                                    unsigned long long *launches) {
	OPROLOGUE();
	extern __shared__ __align__(128) unsigned char smem[];
	const OpDev &op = I.op;
	if (local >= op.tfull) {
		// tiles that no ray crosses (the launch order ends with them): zeros,
		// RAYT_ZERO_TILES tiles per block, none of the list or ring machinery
		// (32-bit indices: tile counts stay below 2^24, and 64-bit ones here
		// cost the whole kernel eight registers)
		const int e0 = op.tfull + ((int)local - op.tfull) * RAYT_ZERO_TILES;
		const int e1 = min(e0 + RAYT_ZERO_TILES, op.tcount);
		const float zero = (float)(0.0 * op.scale);   // the bits a block of this tile would write
		for (int e = e0 + (int)threadIdx.x / RAYT_THREADS; e < e1; e += RAYT_ADJ_THREADS / RAYT_THREADS)
			tiled_store(I, op, ys, __ldg(op.torder + e), threadIdx.x % RAYT_THREADS, zero);
		return;
	}
	const int t = __ldg(op.torder + local);
	const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
	const int pw = wid % RAYT_WARPS, half = wid / RAYT_WARPS;   // pixel-warp, which half of its words
	uint4 *ring = reinterpret_cast<uint4 *>(smem) + wid * RAYT_STAGES * RAYT_STAGE_WORDS;
	const unsigned bar0 = smem_u32(smem + RAYT_RING_BYTES) + 8u * (wid * RAYT_STAGES);
	const unsigned bar_list = smem_u32(smem + RAYT_RING_BYTES) + 8u * (RAYT_ADJ_WARPS * RAYT_STAGES);
	double *sacc = reinterpret_cast<double *>(smem + RAYT_RING_BYTES + RAYT_BAR_BYTES);
	float *yt = reinterpret_cast<float *>(smem + RAYT_RING_BYTES + RAYT_BAR_BYTES + RAYT_SACC_BYTES + 12);
	const int wl = t * RAYT_WARPS + pw;
	const int w0 = __ldg(op.woff + wl), nvall = (__ldg(op.woff + wl + 1) - w0) >> 5;   // words per lane
	const int nfirst = (nvall + 1) / 2;
	const int v0 = half ? nfirst : 0, nv = half ? nvall - nfirst : nfirst;
	const int nch = (nv + RAYT_CW - 1) / RAYT_CW;
	const uint4 *src = op.sidx + w0 + 32LL * v0;
	auto issue = [&](int k) {   // lane 0: chunk k of this warp's words into stage k % RAYT_STAGES
		const int st = k % RAYT_STAGES, words = min(RAYT_CW, nv - k * RAYT_CW);
		const unsigned bytes = (unsigned)words * 32u * 16u;
		mbar_expect_tx(bar0 + 8u * st, bytes);
		bulk_g2s(smem_u32(ring + st * RAYT_STAGE_WORDS), src + (long long)k * RAYT_STAGE_WORDS, bytes, bar0 + 8u * st);
	};
	// the tile's list (a multiple of 4 entries from a 16-byte boundary) is
	// bulk-copied into the measurement slots 1..len, then each slot's
	// measurement index is replaced by its value
	const int k0 = __ldg(op.tptr + t), len = __ldg(op.tptr + t + 1) - k0;
	if (threadIdx.x == 0) {
		mbar_init(bar_list, 1);
		fence_mbar_init();
		mbar_expect_tx(bar_list, (unsigned)len * 4u);
		for (int c0 = 0; c0 < len; c0 += RAYT_LIST_CHUNK)
			bulk_g2s(smem_u32(yt + 1 + c0), op.tmeas + k0 + c0, (unsigned)min(RAYT_LIST_CHUNK, len - c0) * 4u, bar_list);
		yt[0] = 0.f;
	}
	if (lane == 0) {
		for (int st = 0; st < RAYT_STAGES; st++) mbar_init(bar0 + 8u * st, 1);
		fence_mbar_init();
		for (int k = 0; k < min(RAYT_STAGES, nch); k++) issue(k);
	}
	__syncthreads();   // barrier initialisation seen by every thread
	const float *y = vsel(I, xs);
	bool ok = mbar_wait_warp(bar_list, 0u, err, op.first_wait_polls ? op.first_wait_polls - 1u : ASYNC_WAIT_LIMIT);
	if (ok) {   // eight independent gathers in flight per thread
		constexpr int U8 = 8;
		int k = threadIdx.x;
		for (; k + (U8 - 1) * RAYT_ADJ_THREADS < len; k += U8 * RAYT_ADJ_THREADS) {
			float yv[U8];
#pragma unroll
			for (int u = 0; u < U8; u++) yv[u] = y[__float_as_int(yt[1 + k + u * RAYT_ADJ_THREADS])];
#pragma unroll
			for (int u = 0; u < U8; u++) yt[1 + k + u * RAYT_ADJ_THREADS] = yv[u];
		}
		for (; k < len; k += RAYT_ADJ_THREADS) yt[1 + k] = y[__float_as_int(yt[1 + k])];
	}
	__syncthreads();
	double acc = 0.0;
	int k = 0;
	for (; ok && k < nch; k++) {
		const int st = k % RAYT_STAGES;
		if (!mbar_wait_warp(bar0 + 8u * st, (unsigned)(k / RAYT_STAGES) & 1u, err)) break;
		const uint4 *buf = ring + st * RAYT_STAGE_WORDS + lane;
		const int words = min(RAYT_CW, nv - k * RAYT_CW);
		if (words == RAYT_CW) {
			uint4 q[RAYT_CW];
#pragma unroll
			for (int j = 0; j < RAYT_CW; j++) q[j] = buf[32 * j];
#pragma unroll
			for (int j = 0; j < RAYT_CW; j++) acc += (double)word_sum(yt, q[j]);
		} else {
			for (int j = 0; j < words; j++) acc += (double)word_sum(yt, buf[32 * j]);
		}
		__syncwarp();
		if (lane == 0 && k + RAYT_STAGES < nch) {
			fence_proxy_async_smem();   // the stage was read: now the bulk copy may refill it
			issue(k + RAYT_STAGES);
		}
	}
	const bool good = ok && k >= nch;
	if (!good) {   // a wait gave up: let the copies in flight land (bounded) before the block exits
		if (!ok) mbar_wait_warp(bar_list, 0u, err);
		for (int kk = k; kk < min(nch, k + RAYT_STAGES); kk++)
			mbar_wait_warp(bar0 + 8u * (kk % RAYT_STAGES), (unsigned)(kk / RAYT_STAGES) & 1u, err);
	}
	if (half) sacc[pw * 32 + lane] = acc;
	__syncthreads();
	if (half || !good) return;
	acc += sacc[pw * 32 + lane];   // first half + second half
	const int px = __ldg(op.tperm + (long long)t * RAYT_THREADS + threadIdx.x);   // this thread's pixel of the tile
	tiled_store(I, op, ys, t, px, (float)(acc * op.scale));
}

// --- index builder (once per operator) ---------------------------------------
// The rays crossing tile t, as a bitmap over traced-ray ids in shared memory,
// from the pixel-major lists of traced-ray ids (cptr, cind).
// image index of pixel px (0 .. RAYT^2 - 1, row-major) of tile t, or -1 outside the image
__device__ __forceinline__ int tile_pixel(int t, int px, int ntx, int ld, int H) {
	const int x = (t % ntx) * RAYT + px % RAYT, y = (t / ntx) * RAYT + px / RAYT;
	return (x < ld && y < H) ? x + y * ld : -1;
}

__device__ void tile_bitmap(unsigned *bm, int nwords, int p, const int *cptr, const int *cind) {
	for (int w = threadIdx.x; w < nwords; w += blockDim.x) bm[w] = 0u;
	__syncthreads();
	if (p >= 0) {
		const int k1 = cptr[p + 1];
		for (int k = cptr[p]; k < k1; k += 8) {   // eight loads in flight, then their updates
			int r[8];
#pragma unroll
			for (int j = 0; j < 8; j++) r[j] = k + j < k1 ? cind[k + j] : -1;
#pragma unroll
			for (int j = 0; j < 8; j++)
				if (r[j] >= 0) atomicOr(&bm[r[j] >> 5], 1u << (r[j] & 31));
		}
	}
	__syncthreads();
}

// rays per tile (rounded up to a multiple of 4: the pad entries stay 0, a
// valid measurement index that no position refers to); the tile's pixels in
// order of decreasing list length, ties
// by position (perm[rank] = pixel); per warp of ranks its word count: 32 x
// the longest of its pixels' lists, in 16-byte words
__global__ void __launch_bounds__(RAYT_THREADS) k_tile_count(int ld, int H, int ntx, int nrays, const int *cptr,
                                                             const int *cind, long long *tlen, long long *wlen,
                                                             unsigned char *perm, unsigned *gbm) {
	extern __shared__ unsigned bm[];
	__shared__ int ws[RAYT_WARPS];
	__shared__ int cnt[RAYT_THREADS];
	__shared__ int byrank[RAYT_THREADS];
	const int t = blockIdx.x, nwords = (nrays + 31) >> 5;
	const int p = tile_pixel(t, threadIdx.x, ntx, ld, H);
	tile_bitmap(bm, nwords, p, cptr, cind);
	int c = 0;
	for (int w = threadIdx.x; w < nwords; w += blockDim.x) {
		c += __popc(bm[w]);
		if (gbm) gbm[(long long)t * nwords + w] = bm[w];   // kept for k_tile_fill
	}
	c = __reduce_add_sync(0xffffffffu, c);
	const int mine = p >= 0 ? cptr[p + 1] - cptr[p] : 0;
	cnt[threadIdx.x] = mine;
	if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = c;
	__syncthreads();
	int rank = 0;
	for (int q = 0; q < RAYT_THREADS; q++) {
		const int o = cnt[q];
		rank += (o > mine || (o == mine && q < (int)threadIdx.x)) ? 1 : 0;
	}
	perm[(long long)t * RAYT_THREADS + rank] = (unsigned char)threadIdx.x;
	byrank[rank] = mine;
	__syncthreads();
	const int nv = __reduce_max_sync(0xffffffffu, (byrank[threadIdx.x] + 7) >> 3);
	if ((threadIdx.x & 31) == 0) wlen[(long long)t * RAYT_WARPS + (threadIdx.x >> 5)] = 32LL * nv;
	if (threadIdx.x == 0) {
		long long tot = 0;
		for (int i = 0; i < RAYT_WARPS; i++) tot += ws[i];
		tlen[t] = (tot + 3) / 4 * 4;   // lists start on 16-byte boundaries (bulk copies)
	}
}

// the tile's list (measurement indices in traced order) and its pixels'
// 1-based positions in it, padded with 0 to the warp's word count
__global__ void __launch_bounds__(RAYT_THREADS) k_tile_fill(int ld, int H, int ntx, int nrays,
                                                            const int *__restrict__ cptr,
                                                            const int *__restrict__ cind,
                                                            const int *__restrict__ live_out,
                                                            const long long *__restrict__ tptr,
                                                            const long long *__restrict__ woff,
                                                            const unsigned char *__restrict__ perm,
                                                            int *__restrict__ tmeas, uint4 *__restrict__ sidx,
                                                            const unsigned *__restrict__ gbm) {
	extern __shared__ unsigned bm[];   // nwords bits, then nwords exclusive prefix counts
	__shared__ int ws[RAYT_WARPS];
	const int t = blockIdx.x, nwords = (nrays + 31) >> 5;
	int *pre = reinterpret_cast<int *>(bm + nwords);
	// thread = rank: its pixel in the order of decreasing list length
	const int p = tile_pixel(t, perm[(long long)t * RAYT_THREADS + threadIdx.x], ntx, ld, H);
	if (gbm) {   // the bitmap k_tile_count built
		for (int w = threadIdx.x; w < nwords; w += blockDim.x) bm[w] = gbm[(long long)t * nwords + w];
		__syncthreads();
	} else {
		tile_bitmap(bm, nwords, p, cptr, cind);
	}
	// exclusive prefix of the words' popcounts: thread i scans a contiguous run
	const int per = (nwords + RAYT_THREADS - 1) / RAYT_THREADS;
	const int w0 = min(nwords, (int)threadIdx.x * per), w1 = min(nwords, w0 + per);
	int c = 0;
	for (int w = w0; w < w1; w++) c += __popc(bm[w]);
	const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
	int inc = c;
	for (int o = 1; o < 32; o <<= 1) {
		const int u = __shfl_up_sync(0xffffffffu, inc, o);
		if (lane >= o) inc += u;
	}
	if (lane == 31) ws[wid] = inc;
	__syncthreads();
	int run = inc - c;
	for (int i = 0; i < wid; i++) run += ws[i];
	for (int w = w0; w < w1; w++) {
		pre[w] = run;
		run += __popc(bm[w]);
	}
	__syncthreads();
	const long long base = tptr[t];
	for (int w = w0; w < w1; w++) {
		unsigned b = bm[w];
		int r = pre[w];
		while (b) {
			const int bit = __ffs(b) - 1;
			b &= b - 1;
			tmeas[base + r++] = live_out[w * 32 + bit];
		}
	}
	const long long wl = (long long)t * RAYT_WARPS + wid;
	const long long v0 = woff[wl];
	const int nv = (int)((woff[wl + 1] - v0) >> 5);
	int k = p >= 0 ? cptr[p] : 0;
	const int k1 = p >= 0 ? cptr[p + 1] : 0;
	for (int v = 0; v < nv; v++, k += 8) {
		int r[8];   // the word's eight loads first, then their positions
#pragma unroll
		for (int j = 0; j < 8; j++) r[j] = k + j < k1 ? cind[k + j] : -1;
		unsigned e[8];
#pragma unroll
		for (int j = 0; j < 8; j++)
			e[j] = r[j] < 0 ? 0u
			                : 1u + (unsigned)pre[r[j] >> 5] + __popc(bm[r[j] >> 5] & ((1u << (r[j] & 31)) - 1u));
		sidx[v0 + 32LL * v + lane] = make_uint4(e[0] | (e[1] << 16), e[2] | (e[3] << 16), e[4] | (e[5] << 16),
		                                        e[6] | (e[7] << 16));
	}
}

bool build_tiled_index(cudaStream_t s, int ld, int H, int nrays, const int *cptr, const int *cind,
                       const int *live_out, OpDev &d, long long *bytes, std::vector<void *> &owned) {
	if (nrays <= 0 || nrays > RAYT_MAX_RAYS) return false;
	const int ntx = (ld + RAYT - 1) / RAYT, nty = (H + RAYT - 1) / RAYT, nt = ntx * nty;
	const long long nw = (long long)nt * RAYT_WARPS;
	const int nwords = (nrays + 31) / 32;
	const int smem_count = (int)sizeof(unsigned) * nwords, smem_fill = 2 * smem_count;
	TG_CUDA(cudaFuncSetAttribute(k_tile_count, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_count));
	TG_CUDA(cudaFuncSetAttribute(k_tile_fill, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_fill));
	// Each thread walks its own pixel's list of ray ids, so a warp touches 32
	// cache lines per load and reuses each over the next 31 loads: the lines
	// must stay in L1.  With no preference the driver would size shared memory
	// for the most blocks that fit (7 of 32 KB), leaving L1 little room, while
	// there are only nt blocks (256 for a 256x256 image): ask for shared memory
	// for two blocks per SM and leave the rest to L1.
	for (auto kv : {std::make_pair((const void *)k_tile_count, smem_count),
	                std::make_pair((const void *)k_tile_fill, smem_fill)}) {
		const int pct = (int)std::min<long long>(100, (2LL * (kv.second + 2048) * 100 + 232447) / 232448);
		TG_CUDA(cudaFuncSetAttribute(kv.first, cudaFuncAttributePreferredSharedMemoryCarveout, pct));
	}
	long long *tlen = nullptr, *tptr = nullptr, *wlen = nullptr, *woff = nullptr;
	tlen = (decltype(tlen))dev_alloc(sizeof(long long) * (nt + 1), s);
	tptr = (decltype(tptr))dev_alloc(sizeof(long long) * (nt + 1), s);
	wlen = (decltype(wlen))dev_alloc(sizeof(long long) * (nw + 1), s);
	woff = (decltype(woff))dev_alloc(sizeof(long long) * (nw + 1), s);
	unsigned char *perm = (unsigned char *)dev_alloc((size_t)nt * RAYT_THREADS, s);
	// the tiles' ray bitmaps, kept from the count for the fill when they take
	// at most 512 MB (else the fill builds them again)
	const long long gbm_bytes = (long long)nt * nwords * (long long)sizeof(unsigned);
	unsigned *gbm = gbm_bytes <= (512LL << 20) ? (unsigned *)dev_alloc((size_t)gbm_bytes, s) : nullptr;
	k_tile_count<<<nt, RAYT_THREADS, smem_count, s>>>(ld, H, ntx, nrays, cptr, cind, tlen, wlen, perm, gbm);
	TG_CUDA(cudaGetLastError());
	scan_counts(s, tlen, tptr, nt);
	scan_counts(s, wlen, woff, nw);
	std::vector<long long> h_tptr(nt + 1);
	long long words = 0;
	TG_CUDA(cudaMemcpyAsync(h_tptr.data(), tptr, sizeof(long long) * (nt + 1), cudaMemcpyDeviceToHost, s));
	TG_CUDA(cudaMemcpyAsync(&words, woff + nw, sizeof(long long), cudaMemcpyDeviceToHost, s));
	TG_CUDA(cudaStreamSynchronize(s));
	long long tmax = 0;
	for (int t = 0; t < nt; t++) tmax = std::max(tmax, h_tptr[t + 1] - h_tptr[t]);
	const bool ok = tmax <= RAYT_MAX_LIST && words < (1LL << 31) && h_tptr[nt] < (1LL << 31);
	if (ok) {
		// launch order: tiles by decreasing list length (ties by index)
		std::vector<int> order(nt);
		for (int t = 0; t < nt; t++) order[t] = t;
		std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
			return h_tptr[a + 1] - h_tptr[a] > h_tptr[b + 1] - h_tptr[b];
		});
		int *torder = (int *)dev_alloc(sizeof(int) * nt, s);
		owned.push_back(torder);
		TG_CUDA(cudaMemcpyAsync(torder, order.data(), sizeof(int) * nt, cudaMemcpyHostToDevice, s));
		d.torder = torder;
		int *tmeas = (int *)dev_alloc(sizeof(int) * (size_t)std::max(h_tptr[nt], 4LL), s);
		TG_CUDA(cudaMemsetAsync(tmeas, 0, sizeof(int) * (size_t)std::max(h_tptr[nt], 4LL), s));
		uint4 *sidx = (uint4 *)dev_alloc(sizeof(uint4) * (size_t)std::max(words, 1LL), s);
		int *tptr32 = (int *)dev_alloc(sizeof(int) * (nt + 1), s);
		int *woff32 = (int *)dev_alloc(sizeof(int) * (nw + 1), s);
		owned.push_back(tmeas); owned.push_back(sidx); owned.push_back(tptr32); owned.push_back(woff32);
		k_tile_fill<<<nt, RAYT_THREADS, smem_fill, s>>>(ld, H, ntx, nrays, cptr, cind, live_out, tptr, woff, perm,
		                                                tmeas, sidx, gbm);
		TG_CUDA(cudaGetLastError());
		k_to_int<<<(unsigned)((nt + 1 + 255) / 256), 256, 0, s>>>(tptr, tptr32, nt + 1);
		k_to_int<<<(unsigned)((nw + 1 + 255) / 256), 256, 0, s>>>(woff, woff32, nw + 1);
		TG_CUDA(cudaGetLastError());
		TG_CUDA(cudaFuncSetAttribute(k_ray_adj_tiled, cudaFuncAttributeMaxDynamicSharedMemorySize,
		                             tiled_smem_bytes(RAYT_MAX_LIST)));
		d.tiled = 1;
		d.ntx = ntx;
		d.nty = nty;
		int full = 0;   // tiles with rays come first in the order
		while (full < nt && h_tptr[order[full] + 1] > h_tptr[order[full]]) full++;
		d.tfull = full;
		d.tcount = nt;
		d.ntiles = full + (nt - full + RAYT_ZERO_TILES - 1) / RAYT_ZERO_TILES;
		d.tmax = (int)tmax;
		d.tptr = tptr32; d.tmeas = tmeas; d.woff = woff32; d.sidx = sidx; d.tperm = perm;
		owned.push_back(perm);
		*bytes = (long long)sizeof(uint4) * words + (long long)sizeof(int) * (h_tptr[nt] + 2 * nt + nw + 2) +
		         (long long)nt * RAYT_THREADS;
	} else {
		dev_free(perm, s);
	}
	dev_free(gbm, s);
	dev_free(tlen, s);
	dev_free(tptr, s);
	dev_free(wlen, s);
	dev_free(woff, s);
	return ok;
}

// --- 3D brick index (once per operator) --------------------------------------
__global__ void k_entry_rows(long long rows, const int *rptr, int *row_of);
static_assert(BRICK_X * BRICK_Y * BRICK_Z == RAYT_THREADS, "a brick has as many voxels as a 2D tile has pixels");

__device__ __forceinline__ int brick_of(int v, int rvx, int rvy, int nbx, int nby) {
	const int x = v % rvx, y = (v / rvx) % rvy, z = v / (rvx * rvy);
	return x / BRICK_X + (y / BRICK_Y) * nbx + (z / BRICK_Z) * nbx * nby;
}

// run starts: hit k starts a run if it is its ray's first hit or lies in
// another brick than the hit before it (row_of: the ray of every hit)
__global__ void k_run_flags(long long total, const int *rptr, const int *row_of, const int *rind, int rvx, int rvy,
                            int nbx, int nby, long long *flag) {
	for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < total;
	     k += (long long)gridDim.x * blockDim.x) {
		const int r = row_of[k];
		const int b = brick_of(rind[k], rvx, rvy, nbx, nby);
		flag[k] = (k == rptr[r] || b != brick_of(rind[k - 1], rvx, rvy, nbx, nby)) ? 1 : 0;
	}
}

// per run (rs: exclusive scan of the flags): its brick and its ray; the
// identity row pointers of the run -> brick matrix
__global__ void k_run_info(long long total, const long long *flag, const long long *rs, const int *row_of,
                           const int *rind, int rvx, int rvy, int nbx, int nby, int *run_brick, int *run_ray,
                           int *ident, long long runs) {
	for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < total;
	     k += (long long)gridDim.x * blockDim.x)
		if (flag[k]) {
			const long long j = rs[k];
			run_brick[j] = brick_of(rind[k], rvx, rvy, nbx, nby);
			run_ray[j] = row_of[k];
		}
	for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j <= runs; j += (long long)gridDim.x * blockDim.x)
		ident[j] = (int)j;
}

// runs in brick order (bruns, brick offsets bptr): position of each run in
// its brick's list, and the list of measurement indices (padded offsets tptr)
__global__ void k_run_pos(long long runs, const int *bruns, const int *bptr, const int *run_brick, const int *run_ray,
                          const int *live_out, const int *tptr, int *pos_of_run, int *tmeas) {
	for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < runs;
	     j += (long long)gridDim.x * blockDim.x) {
		const int r = bruns[j], b = run_brick[r];
		const int pos = (int)(j - bptr[b]);
		pos_of_run[r] = pos;
		tmeas[tptr[b] + pos] = live_out[run_ray[r]];
	}
}

// per hit in traced order: its 1-based position in its brick's list
__global__ void k_hit_pos(long long total, const long long *rs, const int *pos_of_run, float *posf) {
	for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < total;
	     k += (long long)gridDim.x * blockDim.x)
		posf[k] = (float)(pos_of_run[rs[k + 1] - 1] + 1);
}

__device__ __forceinline__ int brick_voxel(int t, int px, int rvx, int rvy, int rvz, int nbx, int nby) {
	const int bxy = nbx * nby;
	const int x = (t % nbx) * BRICK_X + px % BRICK_X;
	const int y = ((t % bxy) / nbx) * BRICK_Y + (px / BRICK_X) % BRICK_Y;
	const int z = (t / bxy) * BRICK_Z + px / (BRICK_X * BRICK_Y);
	return (x < rvx && y < rvy && z < rvz) ? x + y * rvx + z * rvx * rvy : -1;
}

// per brick: its voxels by decreasing list length (perm[rank] = voxel of the
// brick), the word count of every warp of ranks (32 x its longest list in
// 16-byte words of eight positions)
__global__ void __launch_bounds__(RAYT_THREADS) k_brick_count(int rvx, int rvy, int rvz, int nbx, int nby,
                                                              const int *cptr, long long *wlen, unsigned char *perm) {
	__shared__ int cnt[RAYT_THREADS];
	__shared__ int byrank[RAYT_THREADS];
	const int t = blockIdx.x;
	const int p = brick_voxel(t, threadIdx.x, rvx, rvy, rvz, nbx, nby);
	const int mine = p >= 0 ? cptr[p + 1] - cptr[p] : 0;
	cnt[threadIdx.x] = mine;
	__syncthreads();
	int rank = 0;
	for (int q = 0; q < RAYT_THREADS; q++) {
		const int o = cnt[q];
		rank += (o > mine || (o == mine && q < (int)threadIdx.x)) ? 1 : 0;
	}
	perm[(long long)t * RAYT_THREADS + rank] = (unsigned char)threadIdx.x;
	byrank[rank] = mine;
	__syncthreads();
	const int nv = __reduce_max_sync(0xffffffffu, (byrank[threadIdx.x] + 7) >> 3);
	if ((threadIdx.x & 31) == 0) wlen[(long long)t * RAYT_WARPS + (threadIdx.x >> 5)] = 32LL * nv;
}

// per brick, thread = rank: its voxel's positions packed eight to a 16-byte
// word, the words of a warp's 32 voxels interleaved, padded with 0
__global__ void __launch_bounds__(RAYT_THREADS) k_brick_fill(int rvx, int rvy, int rvz, int nbx, int nby,
                                                             const int *__restrict__ cptr,
                                                             const float *__restrict__ cval,
                                                             const long long *__restrict__ woff,
                                                             const unsigned char *__restrict__ perm,
                                                             uint4 *__restrict__ sidx) {
	const int t = blockIdx.x, lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
	const int p = brick_voxel(t, perm[(long long)t * RAYT_THREADS + threadIdx.x], rvx, rvy, rvz, nbx, nby);
	const long long wl = (long long)t * RAYT_WARPS + wid;
	const long long v0 = woff[wl];
	const int nv = (int)((woff[wl + 1] - v0) >> 5);
	int k = p >= 0 ? cptr[p] : 0;
	const int k1 = p >= 0 ? cptr[p + 1] : 0;
	for (int v = 0; v < nv; v++, k += 8) {
		unsigned e[8];
#pragma unroll
		for (int j = 0; j < 8; j++) e[j] = k + j < k1 ? (unsigned)cval[k + j] : 0u;
		sidx[v0 + 32LL * v + lane] = make_uint4(e[0] | (e[1] << 16), e[2] | (e[3] << 16), e[4] | (e[5] << 16),
		                                        e[6] | (e[7] << 16));
	}
}

float *brick_positions(cudaStream_t s, int rvx, int rvy, int rvz, int nrays, long long total, const int *rptr,
                       const int *rind, const int *live_out, BrickLists &bl, std::vector<void *> &owned) {
	if (nrays <= 0 || total <= 0) return nullptr;
	bl.nbx = (rvx + BRICK_X - 1) / BRICK_X;
	bl.nby = (rvy + BRICK_Y - 1) / BRICK_Y;
	bl.nbz = (rvz + BRICK_Z - 1) / BRICK_Z;
	const long long nb = (long long)bl.nbx * bl.nby * bl.nbz;
	if (nb >= (1LL << 31)) return nullptr;
	bl.nb = (int)nb;
	const unsigned grid = (unsigned)std::min(8192LL, (total + 255) / 256);
	int *row_of = (int *)dev_alloc(sizeof(int) * (size_t)total, s);
	long long *flag = (long long *)dev_alloc(sizeof(long long) * (size_t)(total + 1), s);
	long long *rs = (long long *)dev_alloc(sizeof(long long) * (size_t)(total + 1), s);
	k_entry_rows<<<(unsigned)(((long long)nrays * 32 + 255) / 256), 256, 0, s>>>(nrays, rptr, row_of);
	k_run_flags<<<grid, 256, 0, s>>>(total, rptr, row_of, rind, rvx, rvy, bl.nbx, bl.nby, flag);
	TG_CUDA(cudaGetLastError());
	scan_counts(s, flag, rs, total);
	long long runs = 0;
	TG_CUDA(cudaMemcpyAsync(&runs, rs + total, sizeof(long long), cudaMemcpyDeviceToHost, s));
	TG_CUDA(cudaStreamSynchronize(s));
	float *posf = nullptr;
	int *run_brick = (int *)dev_alloc(sizeof(int) * (size_t)runs, s);
	int *run_ray = (int *)dev_alloc(sizeof(int) * (size_t)runs, s);
	int *ident = (int *)dev_alloc(sizeof(int) * (size_t)(runs + 1), s);
	int *bptr = (int *)dev_alloc(sizeof(int) * (size_t)(nb + 1), s);
	int *bruns = (int *)dev_alloc(sizeof(int) * (size_t)runs, s);
	k_run_info<<<grid, 256, 0, s>>>(total, flag, rs, row_of, rind, rvx, rvy, bl.nbx, bl.nby, run_brick, run_ray, ident,
	                                runs);
	TG_CUDA(cudaGetLastError());
	// the runs of every brick in traced (ray) order: the transpose of the
	// run -> brick matrix
	build_transpose(s, runs, nb, runs, ident, run_brick, nullptr, bptr, bruns, nullptr);
	std::vector<int> h_bptr((size_t)nb + 1);
	TG_CUDA(cudaMemcpyAsync(h_bptr.data(), bptr, sizeof(int) * (size_t)(nb + 1), cudaMemcpyDeviceToHost, s));
	TG_CUDA(cudaStreamSynchronize(s));
	bl.h_tptr.assign((size_t)nb + 1, 0);
	bl.tmax = 0;
	for (long long b = 0; b < nb; b++) {
		const long long len = h_bptr[b + 1] - h_bptr[b];
		bl.tmax = std::max(bl.tmax, len);
		bl.h_tptr[b + 1] = bl.h_tptr[b] + (len + 3) / 4 * 4;
	}
	if (bl.tmax <= RAYT_MAX_LIST && bl.h_tptr[nb] < (1LL << 31)) {
		std::vector<int> t32((size_t)nb + 1);
		for (long long b = 0; b <= nb; b++) t32[b] = (int)bl.h_tptr[b];
		bl.tptr = (int *)dev_alloc(sizeof(int) * (size_t)(nb + 1), s);
		owned.push_back(bl.tptr);
		TG_CUDA(cudaMemcpyAsync(bl.tptr, t32.data(), sizeof(int) * (size_t)(nb + 1), cudaMemcpyHostToDevice, s));
		const long long tl = std::max(bl.h_tptr[nb], 4LL);
		bl.tmeas = (int *)dev_alloc(sizeof(int) * (size_t)tl, s);
		owned.push_back(bl.tmeas);
		TG_CUDA(cudaMemsetAsync(bl.tmeas, 0, sizeof(int) * (size_t)tl, s));
		int *pos_of_run = (int *)dev_alloc(sizeof(int) * (size_t)runs, s);
		k_run_pos<<<(unsigned)std::min(8192LL, (runs + 255) / 256), 256, 0, s>>>(runs, bruns, bptr, run_brick, run_ray,
		                                                                          live_out, bl.tptr, pos_of_run, bl.tmeas);
		posf = (float *)dev_alloc(sizeof(float) * (size_t)total, s);
		k_hit_pos<<<grid, 256, 0, s>>>(total, rs, pos_of_run, posf);
		TG_CUDA(cudaGetLastError());
		dev_free(pos_of_run, s);
	}
	dev_free(row_of, s);
	dev_free(flag, s);
	dev_free(rs, s);
	dev_free(run_brick, s);
	dev_free(run_ray, s);
	dev_free(ident, s);
	dev_free(bptr, s);
	dev_free(bruns, s);
	return posf;
}

bool build_brick_words(cudaStream_t s, int rvx, int rvy, int rvz, const int *cptr, const float *cval,
                       BrickLists &bl, OpDev &d, long long *bytes, std::vector<void *> &owned) {
	const int nb = bl.nb;
	const long long nw = (long long)nb * RAYT_WARPS;
	long long *wlen = (long long *)dev_alloc(sizeof(long long) * (size_t)(nw + 1), s);
	long long *woff = (long long *)dev_alloc(sizeof(long long) * (size_t)(nw + 1), s);
	unsigned char *perm = (unsigned char *)dev_alloc((size_t)nb * RAYT_THREADS, s);
	k_brick_count<<<nb, RAYT_THREADS, 0, s>>>(rvx, rvy, rvz, bl.nbx, bl.nby, cptr, wlen, perm);
	TG_CUDA(cudaGetLastError());
	scan_counts(s, wlen, woff, nw);
	long long words = 0;
	TG_CUDA(cudaMemcpyAsync(&words, woff + nw, sizeof(long long), cudaMemcpyDeviceToHost, s));
	TG_CUDA(cudaStreamSynchronize(s));
	const bool ok = words < (1LL << 31);
	if (ok) {
		std::vector<int> order(nb);
		for (int t = 0; t < nb; t++) order[t] = t;
		std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
			return bl.h_tptr[a + 1] - bl.h_tptr[a] > bl.h_tptr[b + 1] - bl.h_tptr[b];
		});
		int *torder = (int *)dev_alloc(sizeof(int) * nb, s);
		TG_CUDA(cudaMemcpyAsync(torder, order.data(), sizeof(int) * nb, cudaMemcpyHostToDevice, s));
		uint4 *sidx = (uint4 *)dev_alloc(sizeof(uint4) * (size_t)std::max(words, 1LL), s);
		int *woff32 = (int *)dev_alloc(sizeof(int) * (size_t)(nw + 1), s);
		owned.push_back(torder); owned.push_back(sidx); owned.push_back(woff32); owned.push_back(perm);
		k_brick_fill<<<nb, RAYT_THREADS, 0, s>>>(rvx, rvy, rvz, bl.nbx, bl.nby, cptr, cval, woff, perm, sidx);
		k_to_int<<<(unsigned)((nw + 1 + 255) / 256), 256, 0, s>>>(woff, woff32, nw + 1);
		TG_CUDA(cudaGetLastError());
		TG_CUDA(cudaFuncSetAttribute(k_ray_adj_tiled, cudaFuncAttributeMaxDynamicSharedMemorySize,
		                             tiled_smem_bytes(RAYT_MAX_LIST)));
		d.tiled = 1;
		d.tile3 = 1;
		d.ntx = bl.nbx;
		d.nty = bl.nby;
		int full = 0;   // bricks with rays come first in the order
		while (full < nb && bl.h_tptr[order[full] + 1] > bl.h_tptr[order[full]]) full++;
		d.tfull = full;
		d.tcount = nb;
		d.ntiles = full + (nb - full + RAYT_ZERO_TILES - 1) / RAYT_ZERO_TILES;
		d.tmax = (int)bl.tmax;
		d.tptr = bl.tptr; d.tmeas = bl.tmeas; d.woff = woff32; d.sidx = sidx; d.tperm = perm; d.torder = torder;
		*bytes = (long long)sizeof(uint4) * words + (long long)sizeof(int) * (bl.h_tptr[nb] + 2 * (long long)nb + nw + 2) +
		         (long long)nb * RAYT_THREADS;
	} else {
		dev_free(perm, s);
	}
	dev_free(wlen, s);
	dev_free(woff, s);
	return ok;
}

#else   // FP64 build: the ray adjoints are the pixel-major gathers
bool build_tiled_index(cudaStream_t, int, int, int, const int *, const int *, const int *, OpDev &, long long *,
                       std::vector<void *> &) {
	return false;
}
int tiled_smem_bytes(int) { return 0; }
real *brick_positions(cudaStream_t, int, int, int, int, long long, const int *, const int *, const int *, BrickLists &,
                      std::vector<void *> &) {
	return nullptr;
}
bool build_brick_words(cudaStream_t, int, int, int, const int *, const real *, BrickLists &, OpDev &, long long *,
                       std::vector<void *> &) {
	return false;
}
#endif
// ---------------------------------------------------------------------------
// dispatch
// ---------------------------------------------------------------------------
template <int W>
static void gather_w(cudaStream_t s, const LaunchCtx &L, const TileMap &map, int pred, int kind, VecSel x,
                     VecSel y) {
	launch_pdl(k_gather<W>, map.count, 256, 0, s, L.inst, map, pred, kind, x, y, (unsigned long long *)L.launches);
}
static void gather(const LaunchCtx &L, const TileMap (&maps)[4], int pred, int kind, VecSel x, VecSel y) {
	if (maps[0].count > 0) gather_w<4>(L.stream, L, maps[0], pred, kind, x, y);
	if (maps[1].count > 0) gather_w<8>(L.stream, L, maps[1], pred, kind, x, y);
	if (maps[2].count > 0) gather_w<16>(L.stream, L, maps[2], pred, kind, x, y);
	if (maps[3].count > 0) gather_w<32>(L.stream, L, maps[3], pred, kind, x, y);
	TG_CUDA(cudaGetLastError());
}

void op_forward(const LaunchCtx &L, const OpBatch &B, int pred, VecSel x, VecSel y, bool unfused, bool xT_ready) {
	auto *ctr = (unsigned long long *)L.launches;
#ifndef TVAL3G_FP64
	for (const auto &e : B.mrhs) mrhs_apply(L.stream, L.inst, e.first, pred, *e.second, false, x, y, ctr);
#endif
	const TileMap &df = unfused ? B.dense_fwd_nf : B.dense_fwd;
	if (df.count > 0) {
		launch_pdl(k_dense_fwd, df.count, 256, 0, L.stream, L.inst, df, pred, x, y, ctr);
	}
	gather(L, B.csr_fwd, pred, 0, x, y);
	if (B.ray2_transpose.count > 0 && !xT_ready) {
		launch_pdl(k_transpose2d, B.ray2_transpose.count, 256, 0, L.stream, L.inst, B.ray2_transpose, pred, x, ctr);
	}
	if (B.ray2_fwd[0].count > 0)
		launch_pdl(k_ray_fwd<4, false>, B.ray2_fwd[0].count, 256, 0, L.stream, L.inst, B.ray2_fwd[0], pred, x, y, ctr);
	if (B.ray2_fwd[1].count > 0)
		launch_pdl(k_ray_fwd<8, false>, B.ray2_fwd[1].count, 256, 0, L.stream, L.inst, B.ray2_fwd[1], pred, x, y, ctr);
	if (B.ray2_fwd[2].count > 0)
		launch_pdl(k_ray_fwd<16, false>, B.ray2_fwd[2].count, 256, 0, L.stream, L.inst, B.ray2_fwd[2], pred, x, y, ctr);
	if (B.ray3_fwd[0].count > 0)
		launch_pdl(k_ray_fwd<4, true>, B.ray3_fwd[0].count, 256, 0, L.stream, L.inst, B.ray3_fwd[0], pred, x, y, ctr);
	if (B.ray3_fwd[1].count > 0)
		launch_pdl(k_ray_fwd<8, true>, B.ray3_fwd[1].count, 256, 0, L.stream, L.inst, B.ray3_fwd[1], pred, x, y, ctr);
	if (B.ray3_fwd[2].count > 0)
		launch_pdl(k_ray_fwd<16, true>, B.ray3_fwd[2].count, 256, 0, L.stream, L.inst, B.ray3_fwd[2], pred, x, y, ctr);
}

void op_adjoint(const LaunchCtx &L, const OpBatch &B, int pred, VecSel x, VecSel y, bool unfused) {
	auto *ctr = (unsigned long long *)L.launches;
#ifndef TVAL3G_FP64
	for (const auto &e : B.mrhs) mrhs_apply(L.stream, L.inst, e.first, pred, *e.second, true, x, y, ctr);
#endif
	const TileMap &da = unfused ? B.dense_adj_nf : B.dense_adj, &dr = unfused ? B.dense_red_nf : B.dense_red;
	if (da.count > 0) {
		launch_pdl(k_dense_adj, da.count, 256, 0, L.stream, L.inst, da, pred, x, y, B.dense_part, ctr);
		launch_pdl(k_dense_red, dr.count, 256, 0, L.stream, L.inst, dr, pred, x, y, (const real *)B.dense_part, ctr);
	}
	gather(L, B.csc_adj, pred, 1, x, y);
	gather(L, B.ray_adj, pred, 2, x, y);
	if (B.ray_atomic_zero.count > 0)
		launch_pdl(k_ray_atomic_zero, B.ray_atomic_zero.count, 256, 0, L.stream, L.inst, B.ray_atomic_zero, pred, y, ctr);
	if (B.ray2_adj_atomic.count > 0)
		launch_pdl(k_ray_adj_atomic<false>, B.ray2_adj_atomic.count, 256, 0, L.stream, L.inst, B.ray2_adj_atomic, pred,
		           x, y, ctr);
	if (B.ray3_adj_atomic.count > 0)
		launch_pdl(k_ray_adj_atomic<true>, B.ray3_adj_atomic.count, 256, 0, L.stream, L.inst, B.ray3_adj_atomic, pred,
		           x, y, ctr);
#ifndef TVAL3G_FP64
	if (B.ray_adj_tiled.count > 0) {
		launch_pdl(k_ray_adj_tiled, B.ray_adj_tiled.count, RAYT_ADJ_THREADS, tiled_smem_bytes(B.tiled_tmax), L.stream,
		           L.inst, B.ray_adj_tiled, pred, x, y, B.err, ctr);
	}
#endif
}

void op_fused_normal(const LaunchCtx &L, const OpBatch &B, int pred, VecSel x, VecSel y, VecSel z) {
#ifndef TVAL3G_FP64
	auto *ctr = (unsigned long long *)L.launches;
	for (const auto &f : B.fused) {
		int *flags = B.fused_flags + f.off, *err = B.err;
		TG_CUDA(cudaMemsetAsync(flags, 0, sizeof(int) * f.bands, L.stream));
		int inst = f.inst;
		const Inst *tab = L.inst;
		void *args[] = {(void *)&tab, (void *)&inst, (void *)&pred, (void *)&x, (void *)&y, (void *)&z,
		                (void *)&flags, (void *)&err, (void *)&ctr};
		TG_CUDA(cudaLaunchCooperativeKernel((const void *)k_dense_normal, dim3(B.fused_grid), dim3(FUSED_THREADS),
		                                    args, FUSED_DYN_BYTES, L.stream));
	}
#else
	(void)L; (void)B; (void)pred; (void)x; (void)y; (void)z;
#endif
}

void op_normal(const LaunchCtx &L, const OpBatch &B, int pred, VecSel x, VecSel y, VecSel z) {
	op_fused_normal(L, B, pred, x, y, z);
	op_forward(L, B, pred, x, y, true, false);
	op_adjoint(L, B, pred, y, z, true);
}

// ---------------------------------------------------------------------------
// one-time builders
// ---------------------------------------------------------------------------
constexpr int SCAN_ITEMS = 4, SCAN_T = 256, SCAN_TILE = SCAN_ITEMS * SCAN_T;

__global__ void k_scan_tiles(const long long *in, long long *out, long long n, long long *tot) {
	__shared__ long long sh[32];
	long long base = (long long)blockIdx.x * SCAN_TILE + threadIdx.x * SCAN_ITEMS;
	long long v[SCAN_ITEMS], s = 0;
	for (int k = 0; k < SCAN_ITEMS; k++) {
		v[k] = (base + k < n) ? in[base + k] : 0;
		s += v[k];
	}
	// exclusive scan of the thread sums
	int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
	long long incl = s;
	for (int o = 1; o < 32; o <<= 1) {
		long long t = __shfl_up_sync(0xffffffffu, incl, o);
		if (lane >= o) incl += t;
	}
	if (lane == 31) sh[wid] = incl;
	__syncthreads();
	if (wid == 0) {
		long long t = lane < SCAN_T / 32 ? sh[lane] : 0, ti = t;
		for (int o = 1; o < 32; o <<= 1) {
			long long u = __shfl_up_sync(0xffffffffu, ti, o);
			if (lane >= o) ti += u;
		}
		if (lane < SCAN_T / 32) sh[lane] = ti - t;
	}
	__syncthreads();
	long long run = sh[wid] + incl - s;
	for (int k = 0; k < SCAN_ITEMS; k++) {
		if (base + k < n) out[base + k] = run;
		run += v[k];
	}
	if (threadIdx.x == SCAN_T - 1) tot[blockIdx.x] = sh[wid] + incl;
}

// exclusive scan of the nb tile totals in place, by one block of 1024
// threads (each a contiguous run of totals); out[n] = the grand total
__global__ void __launch_bounds__(1024) k_scan_totals(long long *tot, int nb, long long *out, long long n) {
	__shared__ long long sh[32];
	const int t = threadIdx.x, per = (nb + 1023) / 1024;
	const int b0 = min(nb, t * per), b1 = min(nb, b0 + per);
	long long s = 0;
#pragma unroll 8
	for (int b = b0; b < b1; b++) s += tot[b];
	const int lane = t & 31, wid = t >> 5;
	long long incl = s;
	for (int o = 1; o < 32; o <<= 1) {
		const long long u = __shfl_up_sync(0xffffffffu, incl, o);
		if (lane >= o) incl += u;
	}
	if (lane == 31) sh[wid] = incl;
	__syncthreads();
	if (wid == 0) {
		const long long v = sh[lane];
		long long vi = v;
		for (int o = 1; o < 32; o <<= 1) {
			const long long u = __shfl_up_sync(0xffffffffu, vi, o);
			if (lane >= o) vi += u;
		}
		sh[lane] = vi - v;
	}
	__syncthreads();
	long long run = sh[wid] + incl - s;
	// eight loads before their stores: a load after a store to the same array
	// would wait for the store's data
	for (int b = b0; b < b1; b += 8) {
		long long v[8];
#pragma unroll
		for (int j = 0; j < 8; j++) v[j] = b + j < b1 ? tot[b + j] : 0;
#pragma unroll
		for (int j = 0; j < 8; j++)
			if (b + j < b1) {
				tot[b + j] = run;
				run += v[j];
			}
	}
	if (t == 1023) out[n] = sh[wid] + incl;
}

__global__ void k_scan_add(long long *out, long long n, const long long *tot) {
	long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n) out[i] += tot[i / SCAN_TILE];
}

void scan_counts(cudaStream_t s, const long long *cnt, long long *out, long long n) {
	long long nb = (n + SCAN_TILE - 1) / SCAN_TILE;
	if (nb < 1) nb = 1;
	long long *tot = nullptr;
	tot = (decltype(tot))dev_alloc(sizeof(long long) * nb, s);
	k_scan_tiles<<<(unsigned)nb, SCAN_T, 0, s>>>(cnt, out, n, tot);
	k_scan_totals<<<1, 1024, 0, s>>>(tot, (int)nb, out, n);
	if (n > 0) k_scan_add<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(out, n, tot);
	TG_CUDA(cudaGetLastError());
	dev_free(tot, s);
}

__global__ void k_to_int(const long long *in, int *out, long long n) {
	long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n) out[i] = (int)in[i];
}

// The transpose is a stable least-significant-digit radix sort of the CSR
// entries by column, 8 bits per pass: the entries arrive in row order, so
// each column's rows come out ascending, with no per-column sort and no
// atomics that would make the order depend on timing.
constexpr int RADIX_T = 256, RADIX_ITEMS = 16, RADIX_TILE = RADIX_T * RADIX_ITEMS;
constexpr int RADIX_WARPS = RADIX_T / 32;

// the row of every entry (warp per row)
__global__ void k_entry_rows(long long rows, const int *rptr, int *row_of) {
	long long row = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	int lane = threadIdx.x & 31;
	if (row >= rows) return;
	for (int k = rptr[row] + lane; k < rptr[row + 1]; k += 32) row_of[k] = (int)row;
}

// digit counts of one tile of entries: hist[digit * tiles + tile]
__global__ void __launch_bounds__(RADIX_T) k_radix_hist(const int *key, long long nnz, int shift,
                                                        long long *hist) {
	__shared__ int cnt[256];
	cnt[threadIdx.x] = 0;
	__syncthreads();
	const long long base = (long long)blockIdx.x * RADIX_TILE;
#pragma unroll 4
	for (int j = 0; j < RADIX_ITEMS; j++) {
		long long k = base + j * RADIX_T + threadIdx.x;
		if (k < nnz) atomicAdd(&cnt[(key[k] >> shift) & 255], 1);
	}
	__syncthreads();
	hist[(long long)threadIdx.x * gridDim.x + blockIdx.x] = cnt[threadIdx.x];
}

// stable scatter of one tile by its digit: within the tile an entry's rank
// among the entries of its digit follows the input order (round j holds
// entries j*256 + t; a warp ranks its lanes with __match_any_sync, and the
// per-digit pass over the warps orders the warps).  The tile's entries,
// loaded up front, are first placed in shared memory in digit order (digit
// d's slots start at the exclusive sum of the tile's counts below d, from
// k_radix_hist), then written out in slot order: consecutive threads write
// the consecutive entries of one digit to consecutive addresses, instead of
// one scattered 4-byte write per entry.
constexpr int RADIX_DYN_BYTES = RADIX_TILE * (8 + (int)sizeof(real));   // keys, values, entry values
__global__ void __launch_bounds__(RADIX_T) k_radix_scatter(const int *__restrict__ key, const int *__restrict__ val,
                                                           const real *__restrict__ fval, long long nnz, int shift,
                                                           const long long *__restrict__ off,
                                                           const long long *__restrict__ hist,
                                                           int *__restrict__ key_out, int *__restrict__ val_out,
                                                           real *__restrict__ fval_out) {
	extern __shared__ int stage[];   // RADIX_TILE keys, then row values, then entry values (fval only)
	int *sk = stage, *sv = stage + RADIX_TILE;
	real *sf = reinterpret_cast<real *>(stage + 2 * RADIX_TILE);
	__shared__ int wcnt[RADIX_WARPS][256];
	__shared__ int wbase[RADIX_WARPS][256];
	__shared__ long long tile_off[256];
	__shared__ int lstart[256];
	__shared__ int wsum[RADIX_WARPS];
	const int t = threadIdx.x, lane = t & 31, w = t >> 5;
	const long long tiles = gridDim.x;
	tile_off[t] = off[(long long)t * tiles + blockIdx.x];
	{   // lstart: exclusive sum of the tile's digit counts
		const int c = (int)hist[(long long)t * tiles + blockIdx.x];
		int inc = c;
#pragma unroll
		for (int o = 1; o < 32; o <<= 1) {
			const int u = __shfl_up_sync(0xffffffffu, inc, o);
			if (lane >= o) inc += u;
		}
		if (lane == 31) wsum[w] = inc;
		__syncthreads();
		int pre = 0;
		for (int q = 0; q < w; q++) pre += wsum[q];
		lstart[t] = pre + inc - c;
	}
	const long long base = (long long)blockIdx.x * RADIX_TILE;
	int kv[RADIX_ITEMS], vv[RADIX_ITEMS];
	real fv[RADIX_ITEMS];
#pragma unroll
	for (int j = 0; j < RADIX_ITEMS; j++) {   // every load up front
		const long long k = base + j * RADIX_T + t;
		const bool ok = k < nnz;
		kv[j] = ok ? key[k] : 0;
		vv[j] = ok ? val[k] : 0;
		fv[j] = ok && fval ? fval[k] : 0.f;
	}
	int running = 0;   // entries of digit t in the earlier rounds
#pragma unroll
	for (int j = 0; j < RADIX_ITEMS; j++) {
#pragma unroll
		for (int q = 0; q < RADIX_WARPS; q++) wcnt[q][t] = 0;
		__syncthreads();
		const bool ok = base + j * RADIX_T + t < nnz;
		const int d = ok ? (kv[j] >> shift) & 255 : 256;
		const unsigned peers = __match_any_sync(0xffffffffu, d);
		const int rank = __popc(peers & ((1u << lane) - 1u));
		if (ok && rank == 0) wcnt[w][d] = __popc(peers);
		__syncthreads();
		{
			int run = running;
#pragma unroll
			for (int q = 0; q < RADIX_WARPS; q++) {
				wbase[q][t] = run;
				run += wcnt[q][t];
			}
			running = run;
		}
		__syncthreads();
		if (ok) {
			const int slot = lstart[d] + wbase[w][d] + rank;
			sk[slot] = kv[j];
			sv[slot] = vv[j];
			if (fval) sf[slot] = fv[j];
		}
	}
	__syncthreads();
	const int cnt = (int)min((long long)RADIX_TILE, nnz - base);
	for (int i = t; i < cnt; i += RADIX_T) {
		const int kk = sk[i], d = (kk >> shift) & 255;
		const long long pos = tile_off[d] + (i - lstart[d]);
		if (key_out) key_out[pos] = kk;
		val_out[pos] = sv[i];
		if (fval_out) fval_out[pos] = sf[i];
	}
}

// a column's entries are contiguous in the sorted keys: its count is (its
// last entry + 1) - (its first entry), two atomic adds per column
__global__ void k_col_counts(const int *skey, long long nnz, long long *cnt) {
	for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < nnz;
	     k += (long long)gridDim.x * blockDim.x) {
		const int c = skey[k];
		if (k == nnz - 1 || skey[k + 1] != c) atomicAdd((unsigned long long *)&cnt[c], (unsigned long long)(k + 1));
		if (k == 0 || skey[k - 1] != c) atomicAdd((unsigned long long *)&cnt[c], (unsigned long long)(-k));
	}
}

void build_transpose(cudaStream_t s, long long rows, long long cols, long long nnz, const int *rptr,
                     const int *rind, const real *rval, int *cptr, int *cind, real *cval) {
	if (nnz <= 0 || rows <= 0) {
		TG_CUDA(cudaMemsetAsync(cptr, 0, sizeof(int) * (cols + 1), s));
		return;
	}
	int bits = 1;
	while (bits < 31 && (1LL << bits) < cols) bits++;
	const int passes = (bits + 7) / 8;
	const long long tiles = (nnz + RADIX_TILE - 1) / RADIX_TILE;
	int *k0 = nullptr, *k1 = nullptr, *v0 = nullptr, *v1 = nullptr;
	real *f0 = nullptr, *f1 = nullptr;
	long long *hist = nullptr, *hoff = nullptr;
	hist = (decltype(hist))dev_alloc(sizeof(long long) * (256 * tiles + 1), s);
	hoff = (decltype(hoff))dev_alloc(sizeof(long long) * (256 * tiles + 1), s);
	v0 = (decltype(v0))dev_alloc(sizeof(int) * nnz, s);
	k0 = (decltype(k0))dev_alloc(sizeof(int) * nnz, s);
	if (passes > 1) {
		k1 = (decltype(k1))dev_alloc(sizeof(int) * nnz, s);
		v1 = (decltype(v1))dev_alloc(sizeof(int) * nnz, s);
		if (rval) {
			f0 = (decltype(f0))dev_alloc(sizeof(real) * nnz, s);
			f1 = (decltype(f1))dev_alloc(sizeof(real) * nnz, s);
		}
	}
	k_entry_rows<<<(unsigned)((rows * 32 + 255) / 256), 256, 0, s>>>(rows, rptr, v0);
	TG_CUDA(cudaFuncSetAttribute(k_radix_scatter, cudaFuncAttributeMaxDynamicSharedMemorySize, RADIX_DYN_BYTES));
	// pass p reads (key, row, value) from the previous pass (the CSR itself
	// first) and writes the next triple of buffers; the last pass writes
	// cind and cval, and its keys for the column offsets
	const int *kin = rind, *vin = v0;
	const real *fin = rval;
	for (int p = 0; p < passes; p++) {
		const bool last = p == passes - 1;
		int *kout = p % 2 == 0 ? k0 : k1;
		int *vout = last ? cind : (p % 2 == 0 ? v1 : v0);
		real *fout = !rval ? nullptr : last ? cval : (p % 2 == 0 ? f0 : f1);
		k_radix_hist<<<(unsigned)tiles, RADIX_T, 0, s>>>(kin, nnz, 8 * p, hist);
		scan_counts(s, hist, hoff, 256 * tiles);
		const int dyn = RADIX_TILE * 8 + (fin ? RADIX_TILE * (int)sizeof(real) : 0);   // values staged only when there are some
		k_radix_scatter<<<(unsigned)tiles, RADIX_T, dyn, s>>>(kin, vin, fin, nnz, 8 * p, hoff, hist, kout, vout, fout);
		kin = kout;
		vin = vout;
		fin = fout;
	}
	long long *cnt = (long long *)dev_alloc(sizeof(long long) * (cols + 1), s);
	long long *off = (long long *)dev_alloc(sizeof(long long) * (cols + 1), s);
	TG_CUDA(cudaMemsetAsync(cnt, 0, sizeof(long long) * (cols + 1), s));
	k_col_counts<<<(unsigned)std::min(8192LL, (nnz + 255) / 256), 256, 0, s>>>(kin, nnz, cnt);
	scan_counts(s, cnt, off, cols);
	k_to_int<<<(unsigned)((cols + 1 + 255) / 256), 256, 0, s>>>(off, cptr, cols + 1);
	TG_CUDA(cudaGetLastError());
	for (void *ptr : {(void *)hist, (void *)hoff, (void *)v0, (void *)v1, (void *)k0, (void *)k1, (void *)f0,
	                  (void *)f1, (void *)cnt, (void *)off})
		if (ptr) dev_free(ptr, s);
}

__global__ void k_ray_flags(long long cand, const int *up, long long ER, long long *flag) {
	for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < cand;
	     i += (long long)gridDim.x * blockDim.x)
		flag[i] = up[i % ER] != 0 ? 1 : 0;
}

// err[0] / err[1]: the first candidate (loop order) with an endpoint outside
// the image / a use_path index beyond numPaths
__global__ void k_ray_pack(RayGeo g, long long cand, const long long *flag, const long long *slot, int4 *rays,
                           int *out, unsigned long long *err) {
	const long long ER = (long long)g.E * g.R;
	for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < cand;
	     i += (long long)gridDim.x * blockDim.x) {
		if (!flag[i]) continue;
		const long long mp = i / ER, er = i - mp * ER;
		const int e = (int)(er / g.R), r = (int)(er - (long long)e * g.R);
		const int u = g.up[er];
		const long long ie = mp * g.E + e, ir = mp * g.R + r;
		const int x0 = g.xe[ie], y0 = g.ye[ie], x1 = g.xr[ir], y1 = g.yr[ir];
		const int z0 = g.is3 ? g.ze[ie] : 0, z1 = g.is3 ? g.zr[ir] : 0;
		const bool inside = x0 >= 0 && x0 < g.nx && x1 >= 0 && x1 < g.nx && y0 >= 0 && y0 < g.ny && y1 >= 0 &&
		                    y1 < g.ny && z0 >= 0 && z0 < g.nz && z1 >= 0 && z1 < g.nz;
		const long long o = g.is3 ? mp * g.numPaths + u - 1 : er;
		const bool path_ok = !g.is3 || (u >= 1 && o < g.mtot);
		if (!inside) atomicMin(err, (unsigned long long)i);
		else if (!path_ok) atomicMin(err + 1, (unsigned long long)i);
		else {
			rays[slot[i]] = pack_ray(x0, y0, z0, x1 - x0, y1 - y0, z1 - z0, (int)o);
			out[slot[i]] = (int)o;
		}
	}
}

void pack_rays(cudaStream_t s, const RayGeo &g, long long cand, long long *nrays, int4 **rays, int **out) {
	long long *flag = (long long *)dev_alloc(sizeof(long long) * (size_t)(cand + 1), s);
	long long *slot = (long long *)dev_alloc(sizeof(long long) * (size_t)(cand + 1), s);
	unsigned long long *err = (unsigned long long *)dev_alloc(2 * sizeof(unsigned long long), s);
	const unsigned grid = (unsigned)std::max(1LL, std::min(8192LL, (cand + 255) / 256));
	if (cand > 0) k_ray_flags<<<grid, 256, 0, s>>>(cand, g.up, (long long)g.E * g.R, flag);
	scan_counts(s, flag, slot, cand);
	TG_CUDA(cudaMemsetAsync(err, 0xff, 2 * sizeof(unsigned long long), s));
	long long nr = 0;
	TG_CUDA(cudaMemcpyAsync(&nr, slot + cand, sizeof(long long), cudaMemcpyDeviceToHost, s));
	TG_CUDA(cudaStreamSynchronize(s));
	int4 *r = (int4 *)dev_alloc(sizeof(int4) * (size_t)std::max(nr, 1LL), s);
	int *o = (int *)dev_alloc(sizeof(int) * (size_t)std::max(nr, 1LL), s);
	if (cand > 0) k_ray_pack<<<grid, 256, 0, s>>>(g, cand, flag, slot, r, o, err);
	TG_CUDA(cudaGetLastError());
	unsigned long long h_err[2];
	TG_CUDA(cudaMemcpyAsync(h_err, err, sizeof(h_err), cudaMemcpyDeviceToHost, s));
	TG_CUDA(cudaStreamSynchronize(s));
	dev_free(flag, s);
	dev_free(slot, s);
	dev_free(err, s);
	if (h_err[0] != ~0ull || h_err[1] != ~0ull) {
		dev_free(r, s);
		dev_free(o, s);
		if (h_err[0] <= h_err[1])
			throw Error{TVAL3G_ERR_ARGUMENT, g.is3 ? "Argument error: a ray endpoint lies outside the volume"
			                                       : "Argument error: a ray endpoint lies outside the image"};
		throw Error{TVAL3G_ERR_ARGUMENT, "Argument error: use_path index exceeds numPaths"};
	}
	*nrays = nr;
	*rays = r;
	*out = o;
}

__global__ void k_ray_len(int nrays, const int4 *rays, long long *len) {
	int r = blockIdx.x * blockDim.x + threadIdx.x;
	if (r >= nrays) return;
	RayWalk w(rays[r]);
	len[r] = (long long)w.M + 1;
}

__global__ void k_ray_trace(int nrays, const int4 *rays, int rvx, int rvy, const int *rptr, int *rind) {
	long long ray = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	int lane = threadIdx.x & 31;
	if (ray >= nrays) return;
	RayWalk w(rays[ray]);
	const long long rvxy = (long long)rvx * rvy;
	MinorStep s1(lane, w.a1, w.M, 32), s2(lane, w.a2, w.M, 32);
	const int base = rptr[ray];
	for (int j = lane; j <= w.M; j += 32) {
		rind[base + j] = (int)w.index(j, s1.q, s2.q, rvx, rvxy);
		s1.advance();
		s2.advance();
	}
}

int *trace_rays(cudaStream_t s, int nrays, const int4 *rays, int rvx, int rvy, int *rptr, long long *total_out) {
	long long *len = nullptr, *off = nullptr;
	len = (decltype(len))dev_alloc(sizeof(long long) * (nrays + 1), s);
	off = (decltype(off))dev_alloc(sizeof(long long) * (nrays + 1), s);
	if (nrays > 0) k_ray_len<<<(nrays + 255) / 256, 256, 0, s>>>(nrays, rays, len);
	scan_counts(s, len, off, nrays);
	long long total = 0;
	TG_CUDA(cudaMemcpyAsync(&total, off + nrays, sizeof(long long), cudaMemcpyDeviceToHost, s));
	TG_CUDA(cudaStreamSynchronize(s));
	*total_out = total;
	if (total >= (1LL << 31) - 1) {
		dev_free(len, s);
		dev_free(off, s);
		throw Error{TVAL3G_ERR_ARGUMENT, "Argument error: the ray operator has more than 2^31-1 hits"};
	}
	k_to_int<<<(unsigned)((nrays + 1 + 255) / 256), 256, 0, s>>>(off, rptr, nrays + 1);
	int *rind = (int *)dev_alloc(sizeof(int) * (size_t)std::max(total, 1LL), s);
	if (nrays > 0) k_ray_trace<<<(unsigned)(((long long)nrays * 32 + 255) / 256), 256, 0, s>>>(nrays, rays, rvx, rvy, rptr, rind);
	TG_CUDA(cudaGetLastError());
	dev_free(len, s);
	dev_free(off, s);
	return rind;
}

TG_END
