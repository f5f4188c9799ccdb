// Multi-right-hand-side dense operator on the tcgen05 tensor cores (3xTF32):
// the reference's multi-layer dense gemv (2d/mat_mult.h:15-36, a cblas_gemm
// over `layers` right-hand sides) for layers in {16, 32, 48, 64}.
#pragma once
#include <cuda.h>

#include <memory>

#include "engine.cuh"

TG_BEGIN

struct MrhsOp {
	// forward: D[m x N] = A[m x n] X[N x n]^T; adjoint: D[n x N] = At[n x m] R[N x m]^T
	// (tm_a, tm_at: the tile-major copies as 2D arrays of 32 columns, one box per tile)
	CUtensorMap tm_a, tm_at, tm_xh_f, tm_xl_f, tm_xh_a, tm_xl_a;
	long long m = 0, n = 0;
	int N = 0;                  // layers (right-hand sides)
	int grid_f = 0, grid_a = 0; // CTAs per direction (one per SM at most)
	int ks_f = 0, ks_a = 0;     // K steps of 32 (forward: n, adjoint: m)
	int tiles_f = 0, tiles_a = 0;
	int j_f = 0, j_a = 0;       // tile segments per CTA (partial slots)
	long long t_f = 0, t_a = 0; // tiles x K steps
	float *ta = nullptr, *tat = nullptr;   // A and A^T in tile-major order (128 x 32 tiles), owned
	float *xh = nullptr, *xl = nullptr;   // split right-hand sides, N x max(m, n) each
	float *part = nullptr;      // grid x J x N x 128 partial tiles
	int *err = nullptr;         // device flag: a bounded wait timed out
	// independent right-hand sides: column l of X (and of D) belongs to
	// instance members[l] of the table (one layer each, its own scalar
	// control), taken only where that instance's predicate holds; NULL: the
	// N layers of one instance (the reference's joint multi-layer solve)
	int *members = nullptr;
	long long bytes = 0;
	~MrhsOp();
};

// the tensor-core path applies to a dense operator with `layers` right-hand
// sides when layers is 16, 32, 48 or 64 and both dimensions are at least 128
// and multiples of 4 (16-byte row pitch for TMA)
bool mrhs_eligible(long long m, long long n, int layers);
// build A^T and the descriptors for a device-resident row-major A
std::shared_ptr<MrhsOp> mrhs_create(cudaStream_t s, const float *d_A, long long m, long long n, int layers);
// y = A x (trans = 0) or A^T x over the N layers of instance `inst` of the
// table, when its predicate holds
void mrhs_apply(cudaStream_t s, const Inst *tab, int inst, int pred, const MrhsOp &op, bool trans, VecSel x,
                VecSel y, unsigned long long *launches);
// independent right-hand sides: the N instances (device table indices,
// host array) share this operator's products (MrhsOp::members)
void mrhs_set_members(cudaStream_t s, MrhsOp &op, const int *members);
// nonzero if a kernel of this operator gave up a bounded wait (resets it)
int mrhs_take_error(cudaStream_t s, const MrhsOp &op);

TG_END
