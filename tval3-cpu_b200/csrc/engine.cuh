// Internal declarations of the tval3g engine (sm_100a).
//
// Layout in HBM.  A plan holds `count` instances (independent reconstructions).
// Each instance owns NVN image-sized vectors and NVM measurement-sized
// vectors (of `real`: float, or double in the FP64 build) carved from one
// arena, a Ctrl block of FP64 scalars and flags,
// and a slice of the FP64 partial-sum buffer.  Kernels are launched over tile
// maps: a tile map is a device array of (instance, local tile) pairs, so one
// launch covers every instance of a batch; per-instance predicates (Ctrl flags)
// let instances that are done or on another branch skip a launch.
//
// Reductions are deterministic: every tile writes its FP64 partial sums, and
// the last tile of an instance to finish (atomic ticket) sums them in tile
// order and runs that instance's scalar control step (the reference's host
// code: step length, Armijo test, stopping tests, continuation).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <climits>

#include <string>
#include <vector>

#include "../../include/tval3g.h"

// Storage precision of the engine.  The engine's sources are compiled twice:
// once with FP32 storage (the solver behind tval3g_solve and the float
// overloads) and once, with TVAL3G_FP64 defined, with FP64 storage (behind
// tval3g_solve_f64 and the double overloads).  Each build puts its types,
// kernels and host code in its own inline namespace (tval3g::f32,
// tval3g::f64); the error reporting and the device-memory pool below are
// shared.  FP32-only parts (the tcgen05 multi-RHS product, the one-pass dense
// normal product, the tiled ray adjoints, the autotuner, the unrolled solve)
// exist only in the FP32 build.
#ifdef TVAL3G_FP64
#define TG_PREC f64
#else
#define TG_PREC f32
#endif
#define TG_BEGIN           \
	namespace tval3g {     \
	inline namespace TG_PREC {
#define TG_END \
	}          \
	}

namespace tval3g {

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------
void set_error(const std::string &msg);
struct Error {
	int code;
	std::string msg;
};
#define TG_CUDA(call)                                                                               \
	do {                                                                                            \
		cudaError_t e_ = (call);                                                                    \
		if (e_ != cudaSuccess)                                                                      \
			throw ::tval3g::Error{TVAL3G_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)}; \
	} while (0)
// Device memory of plans, operators and host-buffer solves: stream-ordered
// allocations from a per-device pool of this library that keeps freed blocks
// for reuse (unlimited release threshold), so repeated solves do not go back
// to the driver for their buffers and no free synchronises the device.  A
// block may be freed only when no queued work still uses it.
void *dev_alloc(size_t bytes, cudaStream_t s);
void dev_free(void *p, cudaStream_t s);
cudaMemPool_t library_pool();   // the current device's pool

#define TG_ARG(cond, msg)                                                                           \
	do {                                                                                            \
		if (!(cond)) throw ::tval3g::Error{TVAL3G_ERR_ARGUMENT, (msg)};                             \
	} while (0)

}  // namespace tval3g

TG_BEGIN

// element type of the image and measurement vectors and of dense / CSR
// operator values
#ifdef TVAL3G_FP64
typedef double real;
#else
typedef float real;
#endif
constexpr bool FP64_BUILD = sizeof(real) == 8;
// math on `real` (the float forms in the FP32 build, the double forms in the
// FP64 build)
__device__ __forceinline__ float tsqrt(float x) { return sqrtf(x); }
__device__ __forceinline__ double tsqrt(double x) { return sqrt(x); }
__device__ __forceinline__ float tfabs(float x) { return fabsf(x); }
__device__ __forceinline__ double tfabs(double x) { return fabs(x); }
__device__ __forceinline__ float tfma(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ double tfma(double a, double b, double c) { return fma(a, b, c); }
__device__ __forceinline__ float thypot(float a, float b) { return hypotf(a, b); }
__device__ __forceinline__ double thypot(double a, double b) { return hypot(a, b); }
// a problem's dense A and CSR values as the build's element type
// (tval3g_solve_f64 passes its double arrays in these fields)
inline const real *prob_A(const tval3g_problem &p) { return reinterpret_cast<const real *>(p.A); }
inline const real *prob_val(const tval3g_problem &p) { return reinterpret_cast<const real *>(p.csr_val); }

// ---------------------------------------------------------------------------
// per-instance vectors
// ---------------------------------------------------------------------------
enum VecN {
	vU, vUp, vUUP, vUx, vUy, vUz, vUxp, vUyp, vUzp, vWx, vWy, vWz,
	vSx, vSy, vSz, vAtb, vD, vG, vGp, vG2, vG2p, vDts, vRcd, NVN
};
enum VecM { vB, vAu, vAup, vDelta, vLastAu, vAd, NVM };

// scalar state of one instance (the reference's tval3_data scalars and the
// locals of its driver, 2d/tval3_cpu_2d.cpp:99-196,752-853)
struct Ctrl {
	double mu, beta, muDbeta, gam, Q, C, f;
	double lam1, lam2, lam3, lam4, lam5;
	double tau, alpha, c_armij, scl, nrmup, relchg, relchg_out, beta0;
	double dd, dDd;
	double currSkip;
	double rel_error;
	double relerr_ut;            // last |U/scl - Ut| / |Ut| (target mode)
	double step;                 // step of the last descent: U = Up - step * d
	double sched_ratio;          // schedule mode: beta of the last iteration / beta of this one
	int currInit;
	int count_outer, count_total;
	int fst, active, need_bt, bt_cnt, restart, inner_break, need_mlp, need_Ad, skip_adj;
	int status;
	unsigned ticket;
	int pad;
};

// predicates: which instances take part in a launch
enum Pred {
	P_ALL = 0,      // every instance (initialisation)
	P_ACTIVE,       // not yet converged
	P_NEED_AD,      // first-iteration step length needs A*d
	P_NEED_BT,      // Armijo test failed: backtracking (not restarting)
	P_RESTART,      // five backtracking steps failed: restart from Up
	P_INNER_BREAK,  // inner loop ended: outer step
	P_NEED_MLP,     // multiplier update and continuation
	P_ACTIVE_MUL,   // active and the A^T multiplication is not skipped
	P_RESTART_MUL,  // restarting (the restart always multiplies)
	P_FIRST,        // active and the step length needs the first-iteration form (or a restart)
};

__device__ __forceinline__ bool pred_ok(const Ctrl &c, int p) {
	switch (p) {
	case P_ALL: return true;
	case P_ACTIVE: return c.active != 0;
	case P_NEED_AD: return c.need_Ad != 0;
	case P_NEED_BT: return c.active != 0 && c.need_bt != 0 && c.restart == 0;
	case P_RESTART: return c.restart != 0;
	case P_INNER_BREAK: return c.inner_break != 0;
	case P_NEED_MLP: return c.need_mlp != 0;
	case P_ACTIVE_MUL: return c.active != 0 && c.skip_adj == 0;
	case P_RESTART_MUL: return c.restart != 0;
	case P_FIRST: return c.active != 0 && (c.fst != 0 || c.restart != 0);
	}
	return false;
}

// measurement operator of one instance (device side)
struct OpDev {
	int kind;
	int layers;
	long long m;      // rows of one layer
	long long n;      // columns of one layer
	// dense
	const real *A;
	int mrhs;              // layers on the tcgen05 3xTF32 path (mrhs.cu) instead of the gemv kernels
	int dense_kchunks;     // row chunks of the transposed product
	int fused_rpc;         // rows per CTA per band of the one-pass normal product (0: not used)
	int fused_slab;        // its column slab per CTA
	long long dense_part;  // offset of this instance in the dense partial buffer (floats)
	// compressed gather operators: forward rows (CSR) and transpose (CSC)
	const int *rptr, *rind;
	const real *rval;       // NULL = implicit unit weights
	const int *cptr, *cind;
	const real *cval;       // NULL = implicit unit weights
	float scale;            // multiplies every implicit weight
	// rays: packed (x0, y0, z0, dx, dy, dz, out) per traced ray (ops.cuh pack_ray)
	int nrays;
	const int4 *rays;
	int rvx, rvy;           // index = x + y*rvx + z*rvx*rvy (2D: rvx = ld)
	// 2D ray adjoint over pixel tiles (tiled != 0): the image is cut into
	// RAYT x RAYT tiles, ntx per row; tile t lists the measurement indices of
	// the rays that cross it, tmeas[tptr[t] .. tptr[t+1]), in traced order,
	// and each pixel lists its hits as 16-bit 1-based positions in its tile's
	// list (0: a pad entry), eight to a 16-byte word.  Thread r of tile t's
	// block takes pixel tperm[RAYT^2 t + r] (row-major in the tile; pixels by
	// decreasing list length); the words of warp w's 32 pixels (tile t's
	// warps are RAYT^2/32 t + 0, 1, ...) are interleaved: word v of lane l is
	// sidx[woff[w] + 32 v + l].  Block b of a launch takes tile torder[b]:
	// tiles by decreasing list length, so the longest start first and the
	// short ones fill the SMs that finish early.
	int tiled;
	int tile3;              // 3D: tiles are bricks of 8 x 8 x 4 voxels (x, y, z), ntx x nty per z layer
	int ntiles;             // blocks of the tiled adjoint's launch
	int tfull;              // tiles crossed by rays: torder[0 .. tfull) one block each; the rest,
	int tcount;             // up to torder[tcount), no ray crosses (zeros, RAYT_ZERO_TILES a block)
	int nty;
	int ntx;
	int tmax;               // longest tile list
	const int *tptr, *tmeas, *woff;
	const uint4 *sidx;
	const unsigned char *tperm;
	const int *torder;
	// 2D forward: y-driven rays read a transposed copy of the image (rows of
	// length tH = n / ld), in which their steps are contiguous; NULL = off
	real *xT;
	int tH;
	// launch shapes chosen by the autotuner (tune.cu); 0 = the built-in
	// choice: lanes per ray of the ray forward (4, 8 or 16), and 1 + the
	// width class (4, 8, 16, 32 lanes per line) of the compressed gathers of
	// the forward (CSR rows) and of the adjoint (CSC columns, 3D ray index)
	int fwd_lanes;
	int gcls_fwd, gcls_adj;
	// polls of the tiled 2D adjoint's first wait (its ray list), plus one;
	// 0 = the normal limit.  Set only by the failure-path test hook
	// TVAL3G_TEST_FIRST_WAIT_POLLS, read when the operator is prepared: with
	// it the wait gives up and the error path (copies in flight drained at
	// the normal limit, error word raised, TVAL3G_ERR_CUDA) runs without a
	// fault or an unbounded wait.
	unsigned first_wait_polls;
	// ray adjoint by on-the-fly tracing and atomic adds (TVAL3G_RAY_ADJ_ATOMICS)
	int adj_atomic;
};

#ifndef TVAL3G_RAYT
#define TVAL3G_RAYT 16
#endif
constexpr int RAYT = TVAL3G_RAYT;       // tile side of the tiled 2D ray adjoint
constexpr int RAYT_MAX_RAYS = 1 << 18;  // its index builder keeps a bitmap of the traced rays in shared memory
constexpr int RAYT_MAX_LIST = 40960;    // rays per tile (16-bit positions; 160 KB of shared memory beside the index rings)

// Unsigned 32-bit division by a run-time constant with one multiply-high
// (Granlund & Montgomery, "Division by invariant integers using
// multiplication", PLDI 1994): sh = ceil(log2 d), mul = 2^32 (2^sh - d) / d + 1,
// n / d = (umulhi(n, mul) + n) >> sh for every 32-bit n.
struct FastDiv {
	unsigned d, mul, sh;
	void init(unsigned div) {
		d = div;
		sh = 0;
		while ((1ull << sh) < div) sh++;
		mul = (unsigned)(((1ull << 32) * ((1ull << sh) - div)) / div + 1);
	}
	__device__ __forceinline__ unsigned div(unsigned n) const {
		return (unsigned)(((unsigned long long)__umulhi(n, mul) + n) >> sh);
	}
};

// one instance as the kernels see it
struct Inst {
	int dims, p, q, r;           // image: dim_y, dim_x, dim_z (r = 1 in 2D)
	FastDiv fq, fp;              // division by q and by p
	long long n, m;              // vector lengths (n and m include layers)
	real *vn[NVN];
	real *vm[NVM];
	const real *b_user;          // caller's b (device)
	const real *ut_user;         // caller's Ut (device) or NULL
	real *u_user;                // caller's U (device)
	Ctrl *ctrl;
	double *trace;               // maxit records of 5 doubles, or NULL
	double *part;                // this instance's partial sums
	int ntn, ntm;                // tiles over n and m
	int ept;                     // image elements per thread of an n tile (a tile is BLOCK x ept elements)
	// options (2d/tval3_cpu_2d.cpp:769-772)
	double muf, betaf, mu0, beta0, tol, tol_inn, c, gamma, gam0, rate_gam, rate_cnt;
	double skipRatio, maxRelChange;
	double target;               // > 0: also stop once |U/scl - Ut| <= target |Ut|
	const double *sched;         // schedule mode: mu_1..mu_maxit, beta_1..beta_maxit (device), or NULL
	int maxit, maxcnt, nonneg, tv_norm, numInit, skip_enabled;
	// complex data (2D): the image vectors hold the real plane (z = 0) and
	// the imaginary plane (z = 1) of the complex image, the measurement
	// vectors Re b then Im b, and the operator is the real form
	// [[Re A, -Im A], [Im A, Re A]]; the caller's b, Ut and U stay
	// interleaved (re, im) pairs (cplx_index)
	int cplx;
	int isreal;                  // complex data: keep the real part of the final U (2d:855-859)
	OpDev op;
};

// position in the caller's interleaved complex array of element i of a
// planar vector of length len (two planes of len / 2); i itself for real data
__device__ __forceinline__ long long cplx_index(const Inst &I, long long i, long long len) {
	if (!I.cplx) return i;
	const long long h = len >> 1;
	return i < h ? 2 * i : 2 * (i - h) + 1;
}

// Tiles: image vectors BLOCK x Inst::ept elements - one element per thread
// for images of up to about 0.3M elements (a 256^2 image is 256 blocks), up
// to eight for large ones, so that a block's fixed costs (descriptor loads,
// its tile sums, the ticket) are spread over more elements while the grid
// still fills the GPU once (ept_for); measurement vectors four elements per
// thread (their kernels do little per element, and fewer tiles contend less
// for the instance's reduction ticket)
constexpr int TILE = 256;   // n tile of ept 1
constexpr int TILE_M = 1024;
constexpr int BLOCK = 256;
// elements per thread of the n tiles of an image of n elements: the largest
// power of two up to 8 that leaves at least one wave of 4 blocks per SM on
// 148 SMs.  Measured on the 128^3 hemisphere solve (the 20-launch stencil
// timings, µs, and the solve, ms) for 1 / 2 / 4 / 8 / 16 / 32 elements per
// thread: k_shrink_grad 142 / 101 / 83 / 74 / 72 / 120, k_getg 113 / 66 /
// 55 / 54 / 55 / 88, solve 150.8 / 135.4 / 129.9 / 127.6 / 127.2 / 136.3:
// the blocks' fixed costs outweigh the last wave's idle SMs up to 8
inline int ept_for(long long n) {
	int e = 1;
	while (e < 8 && n >= (148LL * 4) * BLOCK * (2 * e)) e *= 2;
	return e;
}
constexpr int EPT_M = TILE_M / BLOCK;
constexpr int NSUM = 10;         // partial sums per tile
constexpr int TRACE_DOUBLES = (int)(sizeof(tval3g_trace_record) / sizeof(double));

// tile maps
enum MapKind { MAP_N = 0, MAP_M, MAP_NM, NMAPS };

struct TileMap {
	const int2 *tiles = nullptr;  // (instance, local tile); local >= ntn means an m tile (MAP_NM)
	int count = 0;
};

// ---------------------------------------------------------------------------
// programmatic dependent launch.  The solve's kernels are launched with
// programmatic stream serialisation (launch_pdl): each lets the next kernel
// of its stream launch as soon as all of its blocks are running
// (pdl_launch_next, first thing), and the next kernel's blocks load their
// tile and instance descriptors meanwhile, then wait in pdl_wait_prev - in
// every block, before the first read of anything an earlier kernel wrote and
// before any early return - for the previous kernel to finish and its writes
// to be visible.  Without the launch attribute both are no-ops.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void pdl_launch_next() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait_prev() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

template <typename... KParams, typename... Args>
inline void launch_pdl(void (*kern)(KParams...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                       Args... args) {
	cudaLaunchConfig_t cfg = {};
	cfg.gridDim = grid;
	cfg.blockDim = block;
	cfg.dynamicSmemBytes = smem;
	cfg.stream = s;
	cudaLaunchAttribute at[1];
	at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
	at[0].val.programmaticStreamSerializationAllowed = 1;
	cfg.attrs = at;
	cfg.numAttrs = 1;
	TG_CUDA(cudaLaunchKernelEx(&cfg, kern, static_cast<KParams>(args)...));
}

// ---------------------------------------------------------------------------
// device helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
	for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
	return v;
}
__device__ __forceinline__ float warp_sumf(float v) {
#pragma unroll
	for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
	return v;
}

// Reduce NS per-thread values over the block; thread 0 gets the totals.
template <int NS>
__device__ __forceinline__ void block_sums(double (&v)[NS], double *sh /* [NS * 32] */) {
	const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
	for (int s = 0; s < NS; s++) v[s] = warp_sum(v[s]);
	if (lane == 0)
#pragma unroll
		for (int s = 0; s < NS; s++) sh[s * 32 + wid] = v[s];
	__syncthreads();
	if (wid == 0) {
#pragma unroll
		for (int s = 0; s < NS; s++) {
			double t = lane < nw ? sh[s * 32 + lane] : 0.0;
			v[s] = warp_sum(t);
		}
	}
	__syncthreads();
}

// Write this tile's NS sums; return true (in every thread) in the block that
// is the last of its instance, with tot[] = the instance totals (summed in
// tile order).  `ntiles` = tiles of this instance in the launch.
template <int NS>
__device__ __forceinline__ bool tile_reduce(const Inst &I, int local, int ntiles, double (&v)[NS],
                                            double (&tot)[NS]) {
	__shared__ double sh[NSUM * 32];
	__shared__ int last;
	block_sums<NS>(v, sh);
	if (threadIdx.x == 0) {
#pragma unroll
		for (int s = 0; s < NS; s++) I.part[(long long)local * NSUM + s] = v[s];
		__threadfence();
		unsigned t = atomicAdd(&I.ctrl->ticket, 1u);
		last = (t == (unsigned)ntiles - 1);
	}
	__syncthreads();
	if (!last) return false;
	__threadfence();
	double acc[NS];
#pragma unroll
	for (int s = 0; s < NS; s++) acc[s] = 0.0;
	// fixed assignment of tiles to threads (thread t adds tiles t, t + B,
	// t + 2B, ... in that order), then a fixed-shape block tree.  This block
	// runs alone at the end of the launch, so the loads of U tiles are issued
	// before their adds (U x NS of them in flight): a 128^3 image has 10240
	// tiles, 40 per thread.
	constexpr int U = NS <= 2 ? 8 : (16 / NS > 1 ? 16 / NS : 1);
	const int B = blockDim.x;
	for (int t0 = threadIdx.x; t0 < ntiles; t0 += U * B) {
		double x[U][NS];
#pragma unroll
		for (int u = 0; u < U; u++)
#pragma unroll
			for (int s = 0; s < NS; s++)
				x[u][s] = t0 + u * B < ntiles ? __ldcg(&I.part[(long long)(t0 + u * B) * NSUM + s]) : 0.0;
#pragma unroll
		for (int u = 0; u < U; u++)
			if (t0 + u * B < ntiles)
#pragma unroll
				for (int s = 0; s < NS; s++) acc[s] += x[u][s];
	}
	block_sums<NS>(acc, sh);
	if (threadIdx.x == 0) {
#pragma unroll
		for (int s = 0; s < NS; s++) tot[s] = acc[s];
		I.ctrl->ticket = 0;
	}
	return true;
}

// ---------------------------------------------------------------------------
// host-side launch interfaces (implemented in the .cu files)
// ---------------------------------------------------------------------------
struct LaunchCtx {
	cudaStream_t stream;
	const Inst *inst;       // device table
	long long *launches;    // host counter of kernel launches issued
};

// operators (op_*.cu): y = A x over every instance of the batch whose Pred
// holds; x, y select vectors of the instance (is_m tells which bank).
struct VecSel {
	bool m;   // false: vn[idx], true: vm[idx]
	int idx;
};

struct OpBatch;   // per-kind launch data, built by the plan
// unfused: leave out the dense instances of the one-pass normal product;
// xT_ready: the 2D ray operators' transposed image already holds x (k_descend
// wrote it), so the forward skips its transpose
void op_forward(const LaunchCtx &L, const OpBatch &B, int pred, VecSel x, VecSel y, bool unfused = false,
                bool xT_ready = false);
void op_adjoint(const LaunchCtx &L, const OpBatch &B, int pred, VecSel x, VecSel y, bool unfused = false);

TG_END
