// Measurement operators of the TVAL3 solve (modk/tval3-cpu 2d/mat_mult.h,
// 3d/mat_mult.h), batched over the instances of a plan.
#pragma once
#include <memory>
#include <utility>

#include "engine.cuh"
#include "mrhs.cuh"

namespace tval3g {

constexpr int WARPS = 8;   // warps per block in the operator kernels

struct OpBatch {
	// dense (2d/mat_mult.h:15-36): forward warp-per-row gemv; adjoint over
	// (column tile, row chunk) blocks into partials, then a column reduction
	TileMap dense_fwd, dense_adj, dense_red;
	float *dense_part = nullptr;
	// dense operators with 16-64 layers: one launch sequence per instance on
	// the tensor cores (mrhs.cu)
	std::vector<std::pair<int, std::shared_ptr<MrhsOp>>> mrhs;
	// compressed gathers: CSR rows (forward), CSC columns (adjoint of CSR and
	// of the ray operators).  Each instance gets the sub-warp width that suits
	// its mean line length (4, 8, 16 or 32 lanes per line: class 0..3), so its
	// summation order does not depend on the other instances of a batch.
	TileMap csr_fwd[4], csc_adj[4], ray_adj[4];
	// rays: on-the-fly Bresenham, 32 lanes per 2D ray (8 rays per block),
	// 16 lanes per 3D ray (16 rays per block)
	TileMap ray2_fwd, ray3_fwd;
	TileMap ray2_transpose;   // 32x32 tiles of the image, for 2D ray operators with xT
	// staged 2D ray adjoint: compaction of the input to traced rays, then one
	// block per ppb pixels
	TileMap ray_compact, ray_adj_staged;
	int staged_ppb_max = 0;
};

// the staged 2D ray adjoint's index: 16-bit in-chunk ray offsets, every
// pixel's segment of every chunk padded to 8 entries, and the per-pixel chunk
// boundaries, from a pixel-major index of traced-ray ids.  Allocates the
// index (recorded in `owned`) and returns its length.
long long build_staged_index(cudaStream_t s, long long n, int nrays, const int *cptr, const int *cind,
                             unsigned short **sidx, int *soff, std::vector<void *> &owned);
int staged_smem_bytes(int ppb);

// one-time builders (ops.cu)
// exclusive scan of n int64 counts into out[0..n] (out[n] = total)
void scan_counts(cudaStream_t s, const long long *cnt, long long *out, long long n);
// CSR (rows x cols, rptr int32) -> CSC sorted by row within a column; cval may be NULL
void build_transpose(cudaStream_t s, long long rows, long long cols, long long nnz, const int *rptr,
                     const int *rind, const float *rval, int *cptr, int *cind, float *cval);
// rasterise nrays packed rays into CSR over rays (offsets int32, indices int32)
void trace_rays(cudaStream_t s, int nrays, const int4 *rays, int rvx, int rvy, int *rptr, int *rind,
                long long *total_out);
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

}  // namespace tval3g
