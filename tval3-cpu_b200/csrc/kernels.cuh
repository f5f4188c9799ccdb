// Fused TVAL3 iteration kernels (sm_100a).  Each kernel runs over a tile map
// (every instance of a batch in one launch), skips instances whose predicate
// is false, and - where the reference computes inner products - reduces FP64
// partial sums deterministically and runs the instance's scalar control step
// in its last tile.  Reference lines: 2d = modk/tval3-cpu 2d/tval3_cpu_2d.cpp,
// 3d = 3d/tval3_cpu_3d.cpp.
#pragma once
#include "engine.cuh"

TG_BEGIN

enum Stage { ST_INIT = 0, ST_LOOP, ST_DESCEND, ST_RESTART, ST_OUTER };
enum TauMode { TAU_ACTIVE = 0, TAU_RESTART };

// Graph conditionals that the kernel itself sets (single-instance graph
// plans): after its scalar step, handle h[k] (nonzero) gets pred_ok(ctrl,
// p[k]) - in place of a separate condition kernel before the node
struct CondSet {
	unsigned long long h[2] = {0ull, 0ull};
	int p[2] = {0, 0};
	CondSet &add(unsigned long long hh, int pp) {   // hh = 0: none (plans that evaluate conditions apart)
		if (!hh) return *this;
		const int k = h[0] ? 1 : 0;
		h[k] = hh;
		p[k] = pp;
		return *this;
	}
};

struct KArgs {
	const Inst *tab;
	TileMap map;
	int pred;
	int stage;
	int multi;   // some instance has n tiles of more than one element per thread (Inst::ept)
	unsigned long long *launches;
	CondSet cs;
	KArgs &cond(unsigned long long h, int p) {
		cs.add(h, p);
		return *this;
	}
};

void launch_scaleb(cudaStream_t s, const KArgs &a);
void launch_init(cudaStream_t s, const KArgs &a);
void launch_init_u(cudaStream_t s, const KArgs &a);
void launch_D(cudaStream_t s, const KArgs &a);
void launch_shrink(cudaStream_t s, const KArgs &a);
void launch_getg(cudaStream_t s, const KArgs &a);
void launch_grad(cudaStream_t s, const KArgs &a);
void launch_shrink_grad(cudaStream_t s, const KArgs &a);
void launch_tau_prep(cudaStream_t s, const KArgs &a);
void launch_tau_bb_cplx(cudaStream_t s, const KArgs &a);
void launch_tau_first(cudaStream_t s, const KArgs &a);
void launch_descend(cudaStream_t s, const KArgs &a);
void launch_bt_search(cudaStream_t s, const KArgs &a);
void launch_lerp(cudaStream_t s, const KArgs &a);
void launch_outer(cudaStream_t s, const KArgs &a);
void launch_mlp(cudaStream_t s, const KArgs &a);
void launch_final(cudaStream_t s, const KArgs &a);
void launch_skip_norms(cudaStream_t s, const KArgs &a);
void launch_copy_lastau(cudaStream_t s, const KArgs &a);
// schedule mode: set (mu_k, beta_k) of the coming iteration (instances with a schedule)
void launch_sched(cudaStream_t s, const Inst *tab, int count, unsigned long long *launches);
// any instance with pred true -> *flag (device) and the graph conditional
void launch_cond(cudaStream_t s, const Inst *tab, int count, int pred, int *flag,
                 unsigned long long handle, unsigned long long *launches);

// standalone stencils (C ABI helpers)
void launch_D_plain(cudaStream_t s, int dims, int p, int q, int r, const real *U, real *Ux, real *Uy,
                    real *Uz);
void launch_Dt_plain(cudaStream_t s, int dims, int p, int q, int r, const real *X, const real *Y,
                     const real *Z, real *res);
void launch_shrink_plain(cudaStream_t s, int dims, long long n, int tv_norm, double beta, const real *Ux,
                         const real *Uy, const real *Uz, const real *sx, const real *sy,
                         const real *sz, real *Wx, real *Wy, real *Wz, double *lam1_dev);

TG_END
