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
//             once on the device (deterministic, no atomics in the solve)
#include "ops.cuh"

namespace tval3g {

__device__ __forceinline__ const float *vsel(const Inst &I, VecSel s) { return s.m ? I.vm[s.idx] : I.vn[s.idx]; }
__device__ __forceinline__ float *vselw(const Inst &I, VecSel s) { return s.m ? I.vm[s.idx] : I.vn[s.idx]; }

#define OPROLOGUE()                                                                   \
	if (launches && blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(launches, 1ull);   \
	const int2 tl_ = map.tiles[blockIdx.x];                                           \
	const Inst &I = tab[tl_.x];                                                       \
	const long long local = tl_.y;                                                    \
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
	const float *a = op.A + row * n;
	const float *x = vsel(I, xs) + layer * n;
	double acc = 0.0;   // FP64 accumulation of FP32 products
	if ((n & 3) == 0 && ((reinterpret_cast<uintptr_t>(a) | reinterpret_cast<uintptr_t>(x)) & 15) == 0) {
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
	if (lane == 0) vselw(I, ys)[layer * m + row] = (float)acc;
}

// partial column sums of A^T x over one row chunk
__global__ void __launch_bounds__(256) k_dense_adj(const Inst *tab, TileMap map, int pred, VecSel xs,
                                                   VecSel ys, float *part, unsigned long long *launches) {
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
	const float *x = vsel(I, xs) + layer * m;
	double acc0 = 0.0, acc1 = 0.0, acc2 = 0.0, acc3 = 0.0;   // FP64 accumulation
	if ((n & 3) == 0 && (reinterpret_cast<uintptr_t>(op.A) & 15) == 0) {
		if (c0 < n) {
			long long r = r0;
			// four rows in flight per thread; the FMA order is the plain loop's
			for (; r + 3 < r1; r += 4) {
				float xv[4];
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
				float xv = __ldg(x + r);
				float4 av = __ldg(reinterpret_cast<const float4 *>(op.A + r * n + c0));
				acc0 = fma((double)av.x, (double)xv, acc0);
				acc1 = fma((double)av.y, (double)xv, acc1);
				acc2 = fma((double)av.z, (double)xv, acc2);
				acc3 = fma((double)av.w, (double)xv, acc3);
			}
		}
	} else {
		for (long long r = r0; r < r1; r++) {
			float xv = __ldg(x + r);
			const float *ar = op.A + r * n;
			if (c0 + 0 < n) acc0 = fma((double)__ldg(ar + c0 + 0), (double)xv, acc0);
			if (c0 + 1 < n) acc1 = fma((double)__ldg(ar + c0 + 1), (double)xv, acc1);
			if (c0 + 2 < n) acc2 = fma((double)__ldg(ar + c0 + 2), (double)xv, acc2);
			if (c0 + 3 < n) acc3 = fma((double)__ldg(ar + c0 + 3), (double)xv, acc3);
		}
	}
	float *p = part + op.dense_part + (layer * K + kc) * n;
	if (c0 + 0 < n) p[c0 + 0] = (float)acc0;
	if (c0 + 1 < n) p[c0 + 1] = (float)acc1;
	if (c0 + 2 < n) p[c0 + 2] = (float)acc2;
	if (c0 + 3 < n) p[c0 + 3] = (float)acc3;
}

// y = sum of the K row-chunk partials, 32 columns per block: warp w adds the
// partials k = w, w + 8, ... of its lane's column, then warp 0 adds the eight
// warp sums in a fixed order (deterministic)
__global__ void __launch_bounds__(256) k_dense_red(const Inst *tab, TileMap map, int pred, VecSel xs, VecSel ys,
                                                   const float *part, unsigned long long *launches) {
	OPROLOGUE();
	__shared__ double ws[8][32];
	const OpDev &op = I.op;
	const long long n = op.n;
	const int K = op.dense_kchunks;
	const long long ct_n = (n + 31) / 32;
	const long long layer = local / ct_n, ct = local - layer * ct_n;
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	const long long c = ct * 32 + lane;
	const float *p = part + op.dense_part + layer * K * n;
	double s = 0.0;
	if (c < n)
		for (int k = warp; k < K; k += 8) s += p[(long long)k * n + c];
	ws[warp][lane] = s;
	__syncthreads();
	if (warp == 0 && c < n) {
		double t = ws[0][lane];
		for (int w = 1; w < 8; w++) t += ws[w][lane];
		vselw(I, ys)[layer * n + c] = (float)t;
	}
}

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
	const float *val;
	long long lines, xlen, ylen;
	if (kind == 0) { ptr = op.rptr; ind = op.rind; val = op.rval; lines = op.m; xlen = op.n; ylen = op.m; }
	else if (kind == 1) { ptr = op.cptr; ind = op.cind; val = op.cval; lines = op.n; xlen = op.m; ylen = op.n; }
	else { ptr = op.cptr; ind = op.cind; val = nullptr; lines = I.n; xlen = 0; ylen = 0; }
	constexpr int LPB = 256 / W;   // lines per block
	const long long lt = (lines + LPB - 1) / LPB;
	const long long layer = local / lt;
	const long long line = (local - layer * lt) * LPB + threadIdx.x / W;
	const int gl = threadIdx.x % W;
	const float *x = vsel(I, xs) + layer * xlen;
	double acc = 0.0;   // FP64 accumulation of FP32 products
	if (line < lines) {
		const int k0 = ptr[line], k1 = ptr[line + 1];
		if (val)
			for (int k = k0 + gl; k < k1; k += W)
				acc = fma((double)__ldg(val + k), (double)__ldg(x + __ldg(ind + k)), acc);
		else
			for (int k = k0 + gl; k < k1; k += W) acc += __ldg(x + __ldg(ind + k));
	}
#pragma unroll
	for (int o = W / 2; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
	if (gl == 0 && line < lines) vselw(I, ys)[layer * ylen + line] = (float)(val ? acc : acc * op.scale);
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
	const float *x = vsel(I, xs);
	double acc = 0.0;   // FP64 accumulation along the ray
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
#pragma unroll 4
		for (int j = gl; j <= M; j += SUBW) {
			acc += __ldg(x + idx);
			idx += dstep;
			r1 += ra1;
			if (r1 >= twoM) { r1 -= twoM; idx += s1; }
			if (D3) {
				r2 += ra2;
				if (r2 >= twoM) { r2 -= twoM; idx += s2; }
			}
		}
	}
#pragma unroll
	for (int o = SUBW / 2; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
	if (gl == 0 && out >= 0) vselw(I, ys)[out] = (float)(acc * op.scale);
}

// xT[y + x*tH] = x[x + y*ld] for the 2D forward (32x32 tiles through shared
// memory; local tile = ty * ceil(ld/32) + tx)
__global__ void __launch_bounds__(256) k_transpose2d(const Inst *tab, TileMap map, int pred, VecSel xs,
                                                     unsigned long long *launches) {
	OPROLOGUE();
	__shared__ float tile[32][33];
	const OpDev &op = I.op;
	const int ld = op.rvx, H = op.tH;
	const int ntx = (ld + 31) / 32;
	const int bx = (int)local % ntx, by = (int)local / ntx;
	const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
	const float *X = vsel(I, xs);
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

// ---------------------------------------------------------------------------
// staged 2D ray adjoint
// ---------------------------------------------------------------------------
// ylive[k] = y[measurement index of traced ray k]
__global__ void __launch_bounds__(256) k_ray_compact(const Inst *tab, TileMap map, int pred, VecSel xs,
                                                     unsigned long long *launches) {
	OPROLOGUE();
	const OpDev &op = I.op;
	const int k = (int)local * 256 + threadIdx.x;
	if (k < op.nrays) op.ylive[k] = vsel(I, xs)[op.live_out[k]];
}

constexpr int STAGED_THREADS = 512;   // one pixel per thread: ppb <= 512
constexpr int STAGED_PAD = 8;         // per-chunk segments padded to 8 entries (16 bytes)
constexpr unsigned short STAGED_SENTINEL = RAY_CHUNK;   // pad entry: reads the zero slot

int staged_smem_bytes(int) { return (int)sizeof(float) * (RAY_CHUNK + STAGED_PAD); }

// g[p] = scale * sum over the rays through p of ylive[ray]: chunk by chunk,
// the chunk of ylive is copied to shared memory (slot RAY_CHUNK holds 0 for
// the pad entries) and each thread sums its pixel's entries of the chunk in
// ray order, reading them eight at a time with 16-byte loads
__global__ void __launch_bounds__(STAGED_THREADS) k_ray_adj_staged(const Inst *tab, TileMap map, int pred,
                                                                   VecSel ys, unsigned long long *launches) {
	OPROLOGUE();
	extern __shared__ float smem[];
	float *chunk = smem;
	const OpDev &op = I.op;
	const int n = (int)I.n, NC = op.nchunks;
	const int p = (int)local * op.ppb + threadIdx.x;
	const bool own = threadIdx.x < op.ppb && p < n;
	constexpr int V4 = RAY_CHUNK / 4 / STAGED_THREADS;   // float4 per thread per chunk
	if (threadIdx.x < STAGED_PAD) chunk[RAY_CHUNK + threadIdx.x] = 0.f;
	const int *so = op.soff + (long long)(own ? p : 0) * (NC + 1);
	// eight interleaved FP64 partial sums (one per index slot), added by a
	// fixed tree at the end: deterministic
	double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
	for (int c = 0; c < NC; c++) {
		const int c0 = c * RAY_CHUNK, cl = min(RAY_CHUNK, op.nrays - c0);
		__syncthreads();
		// all loads of the chunk in flight at once (ylive holds whole chunks)
		const float4 *src = reinterpret_cast<const float4 *>(op.ylive + c0);
		float4 r[V4];
#pragma unroll
		for (int u = 0; u < V4; u++) {
			const int t4 = threadIdx.x + u * STAGED_THREADS;
			r[u] = (4 * t4 < cl) ? __ldcg(src + t4) : make_float4(0.f, 0.f, 0.f, 0.f);
		}
#pragma unroll
		for (int u = 0; u < V4; u++) reinterpret_cast<float4 *>(chunk)[threadIdx.x + u * STAGED_THREADS] = r[u];
		__syncthreads();
		if (own) {
			const int k0 = __ldg(so + c), k1 = __ldg(so + c + 1);
			const uint4 *ix = reinterpret_cast<const uint4 *>(op.sidx + k0);
			const int nv = (k1 - k0) / STAGED_PAD;
#pragma unroll 4
			for (int v = 0; v < nv; v++) {
				const uint4 w = __ldg(ix + v);
				acc[0] += chunk[w.x & 0xffff]; acc[1] += chunk[w.x >> 16];
				acc[2] += chunk[w.y & 0xffff]; acc[3] += chunk[w.y >> 16];
				acc[4] += chunk[w.z & 0xffff]; acc[5] += chunk[w.z >> 16];
				acc[6] += chunk[w.w & 0xffff]; acc[7] += chunk[w.w >> 16];
			}
		}
	}
	const double sum = ((acc[0] + acc[1]) + (acc[2] + acc[3])) + ((acc[4] + acc[5]) + (acc[6] + acc[7]));
	if (own) vselw(I, ys)[p] = (float)(sum * op.scale);
}

// padded length of every pixel's list (each chunk segment rounded up to 8)
__global__ void k_stage_count(long long n, int nchunks, const int *cptr, const int *cind, long long *plen) {
	const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
	if (p >= n) return;
	long long len = 0;
	int k = cptr[p];
	const int k1 = cptr[p + 1];
	for (int c = 0; c < nchunks; c++) {
		int cnt = 0;
		while (k < k1 && cind[k] < (c + 1) * RAY_CHUNK) { k++; cnt++; }
		len += (cnt + STAGED_PAD - 1) / STAGED_PAD * STAGED_PAD;
	}
	plen[p] = len;
}

// write the padded 16-bit lists and the per-pixel chunk boundaries
__global__ void k_stage_fill(long long n, int nchunks, const int *cptr, const int *cind, const long long *pbase,
                             unsigned short *sidx, int *soff) {
	const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
	if (p >= n) return;
	int k = cptr[p];
	const int k1 = cptr[p + 1];
	int *so = soff + p * (nchunks + 1);
	long long w = pbase[p];
	for (int c = 0; c < nchunks; c++) {
		so[c] = (int)w;
		int cnt = 0;
		while (k < k1 && cind[k] < (c + 1) * RAY_CHUNK) {
			sidx[w++] = (unsigned short)(cind[k] - c * RAY_CHUNK);
			k++; cnt++;
		}
		while (cnt % STAGED_PAD) { sidx[w++] = STAGED_SENTINEL; cnt++; }
	}
	so[nchunks] = (int)w;
}

long long build_staged_index(cudaStream_t s, long long n, int nrays, const int *cptr, const int *cind,
                             unsigned short **sidx_out, int *soff, std::vector<void *> &owned) {
	const int nchunks = (nrays + RAY_CHUNK - 1) / RAY_CHUNK;
	long long *plen = nullptr, *pbase = nullptr;
	TG_CUDA(cudaMallocAsync(&plen, sizeof(long long) * (n + 1), s));
	TG_CUDA(cudaMallocAsync(&pbase, sizeof(long long) * (n + 1), s));
	k_stage_count<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(n, nchunks, cptr, cind, plen);
	scan_counts(s, plen, pbase, n);
	long long total = 0;
	TG_CUDA(cudaMemcpyAsync(&total, pbase + n, sizeof(long long), cudaMemcpyDeviceToHost, s));
	TG_CUDA(cudaStreamSynchronize(s));
	unsigned short *sidx = nullptr;
	TG_CUDA(cudaMalloc(&sidx, sizeof(unsigned short) * (size_t)std::max(total, 8LL)));
	owned.push_back(sidx);
	k_stage_fill<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(n, nchunks, cptr, cind, pbase, sidx, soff);
	TG_CUDA(cudaGetLastError());
	TG_CUDA(cudaFreeAsync(plen, s));
	TG_CUDA(cudaFreeAsync(pbase, s));
	TG_CUDA(cudaFuncSetAttribute(k_ray_adj_staged, cudaFuncAttributeMaxDynamicSharedMemorySize,
	                             staged_smem_bytes(0)));
	*sidx_out = sidx;
	return total;
}

// ---------------------------------------------------------------------------
// dispatch
// ---------------------------------------------------------------------------
template <int W>
static void gather_w(cudaStream_t s, const LaunchCtx &L, const TileMap &map, int pred, int kind, VecSel x,
                     VecSel y) {
	k_gather<W><<<map.count, 256, 0, s>>>(L.inst, map, pred, kind, x, y, (unsigned long long *)L.launches);
}
static void gather(const LaunchCtx &L, const TileMap (&maps)[4], int pred, int kind, VecSel x, VecSel y) {
	if (maps[0].count > 0) gather_w<4>(L.stream, L, maps[0], pred, kind, x, y);
	if (maps[1].count > 0) gather_w<8>(L.stream, L, maps[1], pred, kind, x, y);
	if (maps[2].count > 0) gather_w<16>(L.stream, L, maps[2], pred, kind, x, y);
	if (maps[3].count > 0) gather_w<32>(L.stream, L, maps[3], pred, kind, x, y);
	TG_CUDA(cudaGetLastError());
}

void op_forward(const LaunchCtx &L, const OpBatch &B, int pred, VecSel x, VecSel y) {
	auto *ctr = (unsigned long long *)L.launches;
	for (const auto &e : B.mrhs) mrhs_apply(L.stream, L.inst, e.first, pred, *e.second, false, x, y, ctr);
	if (B.dense_fwd.count > 0) {
		k_dense_fwd<<<B.dense_fwd.count, 256, 0, L.stream>>>(L.inst, B.dense_fwd, pred, x, y, ctr);
		TG_CUDA(cudaGetLastError());
	}
	gather(L, B.csr_fwd, pred, 0, x, y);
	if (B.ray2_transpose.count > 0) {
		k_transpose2d<<<B.ray2_transpose.count, 256, 0, L.stream>>>(L.inst, B.ray2_transpose, pred, x, ctr);
		TG_CUDA(cudaGetLastError());
	}
	if (B.ray2_fwd.count > 0) {
		k_ray_fwd<32, false><<<B.ray2_fwd.count, 256, 0, L.stream>>>(L.inst, B.ray2_fwd, pred, x, y, ctr);
		TG_CUDA(cudaGetLastError());
	}
	if (B.ray3_fwd.count > 0) {
		k_ray_fwd<16, true><<<B.ray3_fwd.count, 256, 0, L.stream>>>(L.inst, B.ray3_fwd, pred, x, y, ctr);
		TG_CUDA(cudaGetLastError());
	}
}

void op_adjoint(const LaunchCtx &L, const OpBatch &B, int pred, VecSel x, VecSel y) {
	auto *ctr = (unsigned long long *)L.launches;
	for (const auto &e : B.mrhs) mrhs_apply(L.stream, L.inst, e.first, pred, *e.second, true, x, y, ctr);
	if (B.dense_adj.count > 0) {
		k_dense_adj<<<B.dense_adj.count, 256, 0, L.stream>>>(L.inst, B.dense_adj, pred, x, y, B.dense_part, ctr);
		TG_CUDA(cudaGetLastError());
		k_dense_red<<<B.dense_red.count, 256, 0, L.stream>>>(L.inst, B.dense_red, pred, x, y, B.dense_part, ctr);
		TG_CUDA(cudaGetLastError());
	}
	gather(L, B.csc_adj, pred, 1, x, y);
	gather(L, B.ray_adj, pred, 2, x, y);
	if (B.ray_adj_staged.count > 0) {
		k_ray_compact<<<B.ray_compact.count, 256, 0, L.stream>>>(L.inst, B.ray_compact, pred, x, ctr);
		TG_CUDA(cudaGetLastError());
		k_ray_adj_staged<<<B.ray_adj_staged.count, STAGED_THREADS, staged_smem_bytes(B.staged_ppb_max),
		                   L.stream>>>(L.inst, B.ray_adj_staged, pred, y, ctr);
		TG_CUDA(cudaGetLastError());
	}
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

__global__ void k_scan_totals(long long *tot, int nb, long long *out, long long n) {
	// one thread: nb is small (n / 1024)
	if (threadIdx.x != 0 || blockIdx.x != 0) return;
	long long run = 0;
	for (int b = 0; b < nb; b++) {
		long long t = tot[b];
		tot[b] = run;
		run += t;
	}
	out[n] = run;
}

__global__ void k_scan_add(long long *out, long long n, const long long *tot) {
	long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n) out[i] += tot[i / SCAN_TILE];
}

void scan_counts(cudaStream_t s, const long long *cnt, long long *out, long long n) {
	long long nb = (n + SCAN_TILE - 1) / SCAN_TILE;
	if (nb < 1) nb = 1;
	long long *tot = nullptr;
	TG_CUDA(cudaMallocAsync(&tot, sizeof(long long) * nb, s));
	k_scan_tiles<<<(unsigned)nb, SCAN_T, 0, s>>>(cnt, out, n, tot);
	k_scan_totals<<<1, 32, 0, s>>>(tot, (int)nb, out, n);
	if (n > 0) k_scan_add<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(out, n, tot);
	TG_CUDA(cudaGetLastError());
	TG_CUDA(cudaFreeAsync(tot, s));
}

__global__ void k_to_int(const long long *in, int *out, long long n) {
	long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n) out[i] = (int)in[i];
}

__global__ void k_count_cols(const int *rind, long long nnz, long long *cnt) {
	for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < nnz; k += (long long)gridDim.x * blockDim.x)
		atomicAdd((unsigned long long *)&cnt[rind[k]], 1ull);
}

// warp per row: place every entry at the next free slot of its column
__global__ void k_scatter_cols(long long rows, const int *rptr, const int *rind, const float *rval, int *cursor,
                               int *cind, float *cval) {
	long long row = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	int lane = threadIdx.x & 31;
	if (row >= rows) return;
	for (int k = rptr[row] + lane; k < rptr[row + 1]; k += 32) {
		int pos = atomicAdd(&cursor[rind[k]], 1);
		cind[pos] = (int)row;
		if (cval) cval[pos] = rval[k];
	}
}

// block per column: sort its (row, value) entries by row (bitonic in shared
// memory; long columns fall back to an insertion sort in global memory)
constexpr int SEG_CAP = 4096;
__global__ void k_sort_cols(long long cols, const int *cptr, int *cind, float *cval) {
	__shared__ int key[SEG_CAP];
	__shared__ float val[SEG_CAP];
	for (long long col = blockIdx.x; col < cols; col += gridDim.x) {
		const int k0 = cptr[col], len = cptr[col + 1] - k0;
		if (len <= 1) continue;
		if (len > SEG_CAP) {
			if (threadIdx.x == 0)
				for (int a = 1; a < len; a++) {
					int kk = cind[k0 + a];
					float vv = cval ? cval[k0 + a] : 0.f;
					int b = a - 1;
					while (b >= 0 && cind[k0 + b] > kk) {
						cind[k0 + b + 1] = cind[k0 + b];
						if (cval) cval[k0 + b + 1] = cval[k0 + b];
						b--;
					}
					cind[k0 + b + 1] = kk;
					if (cval) cval[k0 + b + 1] = vv;
				}
			__syncthreads();
			continue;
		}
		int P = 1;
		while (P < len) P <<= 1;
		for (int t = threadIdx.x; t < P; t += blockDim.x) {
			key[t] = t < len ? cind[k0 + t] : INT_MAX;
			val[t] = (t < len && cval) ? cval[k0 + t] : 0.f;
		}
		__syncthreads();
		for (int size = 2; size <= P; size <<= 1)
			for (int stride = size >> 1; stride > 0; stride >>= 1) {
				for (int t = threadIdx.x; t < P; t += blockDim.x) {
					int o = t ^ stride;
					if (o > t) {
						bool up = (t & size) == 0;
						if ((key[t] > key[o]) == up) {
							int tk = key[t]; key[t] = key[o]; key[o] = tk;
							float tv = val[t]; val[t] = val[o]; val[o] = tv;
						}
					}
				}
				__syncthreads();
			}
		for (int t = threadIdx.x; t < len; t += blockDim.x) {
			cind[k0 + t] = key[t];
			if (cval) cval[k0 + t] = val[t];
		}
		__syncthreads();
	}
}

void build_transpose(cudaStream_t s, long long rows, long long cols, long long nnz, const int *rptr,
                     const int *rind, const float *rval, int *cptr, int *cind, float *cval) {
	long long *cnt = nullptr, *off = nullptr;
	int *cursor = nullptr;
	TG_CUDA(cudaMallocAsync(&cnt, sizeof(long long) * (cols + 1), s));
	TG_CUDA(cudaMallocAsync(&off, sizeof(long long) * (cols + 1), s));
	TG_CUDA(cudaMemsetAsync(cnt, 0, sizeof(long long) * (cols + 1), s));
	if (nnz > 0) k_count_cols<<<(unsigned)min(4096LL, (nnz + 255) / 256), 256, 0, s>>>(rind, nnz, cnt);
	scan_counts(s, cnt, off, cols);
	k_to_int<<<(unsigned)((cols + 1 + 255) / 256), 256, 0, s>>>(off, cptr, cols + 1);
	TG_CUDA(cudaMallocAsync(&cursor, sizeof(int) * (cols + 1), s));
	TG_CUDA(cudaMemcpyAsync(cursor, cptr, sizeof(int) * (cols + 1), cudaMemcpyDeviceToDevice, s));
	if (rows > 0) k_scatter_cols<<<(unsigned)((rows * 32 + 255) / 256), 256, 0, s>>>(rows, rptr, rind, rval, cursor, cind, cval);
	if (cols > 0) k_sort_cols<<<(unsigned)min(cols, 148LL * 64), 256, 0, s>>>(cols, cptr, cind, cval);
	TG_CUDA(cudaGetLastError());
	TG_CUDA(cudaFreeAsync(cnt, s));
	TG_CUDA(cudaFreeAsync(off, s));
	TG_CUDA(cudaFreeAsync(cursor, s));
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

void trace_rays(cudaStream_t s, int nrays, const int4 *rays, int rvx, int rvy, int *rptr, int *rind,
                long long *total_out) {
	long long *len = nullptr, *off = nullptr;
	TG_CUDA(cudaMallocAsync(&len, sizeof(long long) * (nrays + 1), s));
	TG_CUDA(cudaMallocAsync(&off, sizeof(long long) * (nrays + 1), s));
	if (nrays > 0) k_ray_len<<<(nrays + 255) / 256, 256, 0, s>>>(nrays, rays, len);
	scan_counts(s, len, off, nrays);
	long long total = 0;
	TG_CUDA(cudaMemcpyAsync(&total, off + nrays, sizeof(long long), cudaMemcpyDeviceToHost, s));
	TG_CUDA(cudaStreamSynchronize(s));
	*total_out = total;
	if (total >= (1LL << 31) - 1) {
		cudaFreeAsync(len, s);
		cudaFreeAsync(off, s);
		throw Error{TVAL3G_ERR_ARGUMENT, "Argument error: the ray operator has more than 2^31-1 hits"};
	}
	k_to_int<<<(unsigned)((nrays + 1 + 255) / 256), 256, 0, s>>>(off, rptr, nrays + 1);
	if (rind && nrays > 0) k_ray_trace<<<(unsigned)(((long long)nrays * 32 + 255) / 256), 256, 0, s>>>(nrays, rays, rvx, rvy, rptr, rind);
	TG_CUDA(cudaGetLastError());
	TG_CUDA(cudaFreeAsync(len, s));
	TG_CUDA(cudaFreeAsync(off, s));
}

}  // namespace tval3g
