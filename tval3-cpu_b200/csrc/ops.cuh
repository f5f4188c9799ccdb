// Measurement operators of the TVAL3 solve (modk/tval3-cpu 2d/mat_mult.h,
// 3d/mat_mult.h), batched over the instances of a plan.
#pragma once
#include <vector>
#include <memory>
#include <utility>

#include "engine.cuh"
#include "mrhs.cuh"

TG_BEGIN

constexpr int WARPS = 8;   // warps per block in the operator kernels
// lanes per ray of the on-the-fly forward projectors: a warp traces
// 32 / RAY_SUBW rays at once, which spreads the per-ray set-up (unpacking,
// the closed-form start of every lane, the final shuffle sum) over several
// rays; 2D rays of 100-400 hits and 3D rays of ~60 hits keep 8 lanes busy
constexpr int RAY_SUBW = 8;
constexpr int RAYS_PER_BLOCK = 256 / RAY_SUBW;
constexpr int RAY_LANES[3] = {4, 8, 16};   // lanes-per-ray classes of the forward

struct OpBatch {
	// dense (2d/mat_mult.h:15-36): forward warp-per-row gemv; adjoint over
	// (column tile, row chunk) blocks into partials, then a column reduction
	TileMap dense_fwd, dense_adj, dense_red;
	real *dense_part = nullptr;
	// dense operators whose normal product A^T (A u) reads A once
	// (k_dense_normal, one cooperative launch per instance); the gemv maps
	// without them serve the rest of a normal product
	struct Fused {
		int inst;
		int bands;
		long long off;   // of its band flags in fused_flags
	};
	std::vector<Fused> fused;
	TileMap dense_fwd_nf, dense_adj_nf, dense_red_nf;
	int fused_grid = 0;
	long long fused_words = 0;   // band flags of all fused instances
	int *fused_flags = nullptr;
	// set (to nonzero) by a kernel whose bounded wait gave up: its results
	// are invalid; the owner checks and clears it after each solve or product
	int *err = nullptr;
	// dense operators with 16-64 layers: one launch sequence per instance on
	// the tensor cores (mrhs.cu)
	std::vector<std::pair<int, std::shared_ptr<MrhsOp>>> mrhs;
	// compressed gathers: CSR rows (forward), CSC columns (adjoint of CSR and
	// of the ray operators).  Each instance gets the sub-warp width that suits
	// its mean line length (4, 8, 16 or 32 lanes per line: class 0..3), so its
	// summation order does not depend on the other instances of a batch.
	TileMap csr_fwd[4], csc_adj[4], ray_adj[4];
	// rays: on-the-fly Bresenham, 4, 8 or 16 lanes per ray (class 0..2;
	// RAY_SUBW = 8 unless the autotuner chose otherwise), 2D and 3D
	TileMap ray2_fwd[3], ray3_fwd[3];
	TileMap ray2_transpose;   // 32x32 tiles of the image, for 2D ray operators with xT
	// tiled 2D ray adjoint: one block per RAYT x RAYT pixel tile; dynamic
	// shared memory for the longest tile list of the batch
	TileMap ray_adj_tiled;
	int tiled_tmax = 0;
	// ray adjoints by on-the-fly tracing with atomic adds (OpDev::adj_atomic):
	// the output zeroed (ATOMIC_ZERO_TILE elements per block), then
	// RAYS_PER_BLOCK rays per block, 2D and 3D
	TileMap ray_atomic_zero, ray2_adj_atomic, ray3_adj_atomic;
};
constexpr int ATOMIC_ZERO_TILE = 1024;

// the tiled 2D ray adjoint's index (OpDev::tiled) for an ld x H image, from
// the pixel-major lists of traced-ray ids (cptr, cind; sorted by ray) and the
// measurement index of every traced ray.  Fills d's tiled fields, allocates
// the index (recorded in `owned`, its size stored in *bytes) and returns true;
// returns false, allocating nothing, when there are more than RAYT_MAX_RAYS
// traced rays or a tile list would exceed RAYT_MAX_LIST.
bool build_tiled_index(cudaStream_t s, int ld, int H, int nrays, const int *cptr, const int *cind,
                       const int *live_out, OpDev &d, long long *bytes, std::vector<void *> &owned);
int tiled_smem_bytes(int tmax);

// The same tiled adjoint for 3D rays, over bricks of BRICK_X x BRICK_Y x
// BRICK_Z voxels (as many as the 2D tile's pixels).  Built in two steps
// around the voxel-major transpose of the traced hits:
//  brick_positions (before it): splits every traced ray into its runs of
//    consecutive hits in one brick (a Bresenham ray enters a brick once: its
//    coordinates are monotone), lists each brick's rays in traced order
//    (tmeas, padded to multiples of 4 from 16-byte boundaries) and returns,
//    per hit in traced order, its 1-based position in its brick's list as a
//    float (exact), for the transpose to carry; NULL when a list would exceed
//    RAYT_MAX_LIST (the plain gather then stays).
//  build_brick_words (after it, with the voxel-major positions cval): the
//    per-brick voxel order, the interleaved 16-bit position words and the
//    launch order; fills d's tiled fields.
constexpr int BRICK_X = 8, BRICK_Y = 8, BRICK_Z = 4;
struct BrickLists {
	int nbx = 0, nby = 0, nbz = 0, nb = 0;
	std::vector<long long> h_tptr;   // padded list offsets (host copy), nb + 1
	int *tptr = nullptr, *tmeas = nullptr;
	long long tmax = 0;
};
real *brick_positions(cudaStream_t s, int rvx, int rvy, int rvz, int nrays, long long total, const int *rptr,
                       const int *rind, const int *live_out, BrickLists &bl, std::vector<void *> &owned);
bool build_brick_words(cudaStream_t s, int rvx, int rvy, int rvz, const int *cptr, const real *cval,
                       BrickLists &bl, OpDev &d, long long *bytes, std::vector<void *> &owned);
// the dense normal product's launch: CTAs (one per SM), and rows per CTA per
// band for an m x n operator A (0: the operator does not suit it - n not a
// multiple of 4, A not 16-byte aligned, its slab or two bands do not fit),
// with the slab width
int fused_grid();
int fused_rows_per_cta(long long m, long long n, int grid, const real *A, int *slab);
// Au = A u and g = A^T Au for the fused dense instances (A read once)
void op_fused_normal(const LaunchCtx &L, const OpBatch &B, int pred, VecSel u, VecSel au, VecSel g);
// the normal product of every instance: fused dense instances in one pass,
// the others as op_forward then op_adjoint
void op_normal(const LaunchCtx &L, const OpBatch &B, int pred, VecSel u, VecSel au, VecSel g);

// one-time builders (ops.cu)
// exclusive scan of n int64 counts into out[0..n] (out[n] = total)
void scan_counts(cudaStream_t s, const long long *cnt, long long *out, long long n);
// CSR (rows x cols, rptr int32) -> CSC sorted by row within a column; cval may be NULL
void build_transpose(cudaStream_t s, long long rows, long long cols, long long nnz, const int *rptr,
                     const int *rind, const real *rval, int *cptr, int *cind, real *cval);
// The traced rays of a ray geometry, packed on the device in the reference's
// loop order (measurement plane, emitter, receiver; a ray for every nonzero
// use_path entry): 2D: out = e R + r; 3D: out = mp numPaths + use_path - 1.
// All arrays are device copies of the geometry's.  pack_rays allocates the
// packed rays and their measurement indices (stream-ordered, the caller's)
// and throws the reference's argument error for the first offending ray in
// loop order (an endpoint outside the image or volume; a use_path index
// beyond numPaths).
struct RayGeo {
	int E, R, is3, numPaths;
	long long mtot;
	int nx, ny, nz;   // endpoint bounds (2D: ld and min(height, 32767))
	const int *up, *xe, *ye, *ze, *xr, *yr, *zr;
};
void pack_rays(cudaStream_t s, const RayGeo &g, long long cand, long long *nrays, int4 **rays, int **out);
// rasterise nrays packed rays into CSR over rays (offsets int32 into rptr,
// nrays + 1 of them; the indices, int32, in a new stream-ordered allocation
// that the caller owns: dev_free)
int *trace_rays(cudaStream_t s, int nrays, const int4 *rays, int rvx, int rvy, int *rptr, long long *total_out);
// apply one instance's operator outside a plan (C ABI)
void apply_single(cudaStream_t s, const Inst *dtab, const OpDev &op, int trans, long long rows,
                  long long cols, const OpBatch &B);

// pack (x0, y0, z0, out, dx, dy, dz) into 16 bytes; coordinates in [-32768, 32767]
__host__ __device__ inline int4 pack_ray(int x0, int y0, int z0, int dx, int dy, int dz, int out) {
	int4 r;
	r.x = (x0 & 0xffff) | (y0 << 16);
	r.y = (z0 & 0xffff) | (dx << 16);
	r.z = (dy & 0xffff) | (dz << 16);
	r.w = out;
	return r;
}
__host__ __device__ inline void unpack_ray(int4 r, int &x0, int &y0, int &z0, int &dx, int &dy, int &dz,
                                           int &out) {
	x0 = (int)(short)(r.x & 0xffff); y0 = r.x >> 16;
	z0 = (int)(short)(r.y & 0xffff); dx = r.y >> 16;
	dy = (int)(short)(r.z & 0xffff); dz = r.z >> 16;
	out = r.w;
}

TG_END
