// Fused TVAL3 iteration kernels; see kernels.cuh.
//
// Every kernel copies its instance descriptor into registers (a by-value
// Inst: stores to the vectors cannot alias it, so its pointers are
// loaded once), indexes with 32-bit integers (image and measurement lengths
// are below 2^31) and computes image coordinates with multiply-high division.
#include <math.h>

#include "kernels.cuh"

TG_BEGIN

// ---------------------------------------------------------------------------
// prologue / image geometry
// ---------------------------------------------------------------------------
// the graph conditionals this launch sets (single-instance plans only), from
// the instance's state
__device__ __forceinline__ void set_conds(const CondSet &cs, const Ctrl &c) {
#pragma unroll
	for (int k = 0; k < 2; k++)
		if (cs.h[k]) cudaGraphSetConditional((cudaGraphConditionalHandle)cs.h[k], pred_ok(c, cs.p[k]) ? 1u : 0u);
}

// A launch whose instance is excluded by its predicate still sets its
// conditionals (block 0), from the state it leaves unchanged.
#define KPROLOGUE(a)                                                                        \
	pdl_launch_next();                                                                      \
	if ((a).launches && blockIdx.x == 0 && threadIdx.x == 0) atomicAdd((a).launches, 1ull); \
	const int2 tl_ = (a).map.tiles[blockIdx.x];                                             \
	const Inst I = (a).tab[tl_.x];                                                          \
	const int local = tl_.y;                                                                \
	pdl_wait_prev();                                                                        \
	if (!pred_ok(*I.ctrl, (a).pred)) {                                                      \
		if (blockIdx.x == 0 && threadIdx.x == 0) set_conds((a).cs, *I.ctrl);                \
		return;                                                                             \
	}

// element k of this thread in the instance's n tile `local` (BLOCK x I.ept
// elements; each element's loads precede its stores, so the elements run one
// after the other).  Every kernel comes in two forms: MULTI = false for
// launches whose instances all have ept 1 (one element per thread, the small
// images, compiled as straight-line code), MULTI = true for the others (the
// element loop, with launch bounds that give the large images' grids more
// resident warps).
#define FOR_TILE(local, len, i)                                                      \
	_Pragma("unroll 1") for (int k_ = 0; k_ < (MULTI ? I.ept : 1); k_++)             \
		if (const int i = (int)(local) * (BLOCK * (MULTI ? I.ept : 1)) + (int)threadIdx.x + k_ * BLOCK; \
		    i < (len))
// the same over a tile of measurement elements (TILE_M = BLOCK x EPT_M)
#define FOR_TILE_M(i0, len, i)                                \
	_Pragma("unroll") for (int k_ = 0; k_ < EPT_M; k_++)      \
		if (const int i = (i0) + (int)threadIdx.x + k_ * BLOCK; i < (len))
// The loads of all EPT_M elements first, then the stores: the compiler cannot
// tell that two vectors do not alias, so a load that follows a store in
// program order would wait for the store's data.
#define LOAD_TILE_M(i0, len, reg, expr)              \
	real reg[EPT_M];                                \
	FOR_TILE_M(i0, len, i) reg[k_] = (expr);

// resident blocks per SM asked of the register allocator: the FP64 build's
// elements take twice the registers, so it asks for half as many blocks
#define MINB(x) (FP64_BUILD ? ((x) + 1) / 2 : (x))

struct Geo {
	int dims, p, q, r, S, n;
	FastDiv fq, fp;
	__device__ Geo(const Inst &I)
		: dims(I.dims), p(I.p), q(I.q), r(I.r), S(I.p * I.q), n((int)I.n), fq(I.fq), fp(I.fp) {}
	__device__ __forceinline__ void coords(int i, int &x, int &y, int &z) const {
		const unsigned row = fq.div((unsigned)i);
		x = i - (int)row * q;
		const unsigned zz = fp.div(row);
		z = (int)zz;
		y = (int)row - (int)zz * p;
		if (z >= r) z -= r;   // complex data: the imaginary plane repeats the real plane's z
	}
};

// periodic forward differences at i (2d:268-278, 3d:365-389)
__device__ __forceinline__ real dxf(const real *__restrict__ U, const Geo &g, int i, int x) {
	return (x < g.q - 1) ? U[i + 1] - U[i] : U[i - (g.q - 1)] - U[i];
}
__device__ __forceinline__ real dyf(const real *__restrict__ U, const Geo &g, int i, int y) {
	return (y < g.p - 1) ? U[i + g.q] - U[i] : U[i - (g.p - 1) * g.q] - U[i];
}
__device__ __forceinline__ real dzf(const real *__restrict__ U, const Geo &g, int i, int z) {
	return (z < g.r - 1) ? U[i + g.S] - U[i] : U[i - (g.r - 1) * g.S] - U[i];
}

// Dt at i with component accessors vx(j), vy(j), vz(j); the additions (in the element type)
// are made in the reference's order (2d:280-293, 3d:394-425), including the
// 3D y term the reference adds on the first row of slices z >= 1.
template <class FX, class FY, class FZ>
__device__ __forceinline__ real dt_at(const Geo &g, int i, int x, int y, int z, FX vx, FY vy, FZ vz) {
	real res = (x > 0) ? vx(i - 1) - vx(i) : vx(i + g.q - 1) - vx(i);
	if (g.dims == 2) {
		if (y > 0) { res = res + vy(i - g.q); res = res + (-vy(i)); }
		else { res = res + vy(i + (g.p - 1) * g.q); res = res + (-vy(i)); }
	} else {
		if (!(z == 0 && y == 0)) { res = res + vy(i - g.q); res = res + (-vy(i)); }
		if (y == 0) { res = res + vy(i + (g.p - 1) * g.q); res = res + (-vy(i)); }
		if (z > 0) { res = res + vz(i - g.S); res = res + (-vz(i)); }
		else { res = res + vz(i + (g.r - 1) * g.S); res = res + (-vz(i)); }
	}
	return res;
}

// shrinkage of one pixel: anisotropic 2d:588-611 / 3d:834-871; isotropic:
// W = max(|Ubar|_2 - 1/beta, 0) * Ubar / |Ubar|_2 (no reference counterpart)
//
// sigma / beta is formed as sigma * (1 / beta): identical to the reference's
// division whenever beta is a power of two (beta0 = 2^k and rate_cnt = 2
// keep it one), within one rounding otherwise.
struct Shrink {
	real rbeta, thr;
	int iso, dims;
	__device__ Shrink(const Inst &I, double beta_d)
		: rbeta((real)(1.0 / beta_d)), thr((real)(1.0 / beta_d)), iso(I.tv_norm), dims(I.dims) {}
	__device__ __forceinline__ real apply(const real (&u)[3], const real (&s)[3], real (&w)[3]) const {
		real ub[3];
#pragma unroll
		for (int c = 0; c < 3; c++) ub[c] = (c < dims) ? u[c] - s[c] * rbeta : 0.f;
		if (iso) {
			real nrm = tsqrt(ub[0] * ub[0] + ub[1] * ub[1] + ub[2] * ub[2]);
			real t = nrm - thr;
			t = t >= 0.f ? t : 0.f;
			const real sc = nrm > 0.f ? t / nrm : 0.f;
#pragma unroll
			for (int c = 0; c < 3; c++) w[c] = sc * ub[c];
			return t;
		}
		real lam = 0.f;
#pragma unroll
		for (int c = 0; c < 3; c++) {
			real t = tfabs(ub[c]) - thr;
			t = t >= 0.f ? t : 0.f;
			if (c < dims) lam += t;
			w[c] = ub[c] >= 0.f ? t : -t;
		}
		return lam;
	}
	// one component of the anisotropic shrinkage (apply's per-component
	// arithmetic): W_c depends on U_c and sigma_c alone
	__device__ __forceinline__ real apply1(real u, real s) const {
		const real ub = u - s * rbeta;
		real t = tfabs(ub) - thr;
		t = t >= 0.f ? t : 0.f;
		return ub >= 0.f ? t : -t;
	}
	// complex data: (u, s) of this plane and (up, sp) of the other plane at
	// the same pixel; anisotropic: each component's Ubar = (re, im) shrinks
	// by its modulus, W = max(|Ubar| - 1/beta, 0) Ubar / |Ubar| (2d:614-649);
	// isotropic: by the modulus over all components.  Returns this plane's
	// share of lambda1 (the real plane carries it, the imaginary plane 0).
	__device__ __forceinline__ real apply_c(const real (&u)[3], const real (&s)[3], const real (&up)[3],
	                                         const real (&sp)[3], bool imag, real (&w)[3]) const {
		real re[3], im[3];
#pragma unroll
		for (int c = 0; c < 3; c++) {
			const real a = (c < dims) ? u[c] - s[c] * rbeta : 0.f;
			const real b = (c < dims) ? up[c] - sp[c] * rbeta : 0.f;
			re[c] = imag ? b : a;
			im[c] = imag ? a : b;
		}
		if (iso) {
			real nrm2 = 0.f;
#pragma unroll
			for (int c = 0; c < 3; c++) nrm2 += re[c] * re[c] + im[c] * im[c];
			const real nrm = tsqrt(nrm2);
			real t = nrm - thr;
			t = t >= 0.f ? t : 0.f;
			const real sc = nrm > 0.f ? t / nrm : 0.f;
#pragma unroll
			for (int c = 0; c < 3; c++) w[c] = sc * (imag ? im[c] : re[c]);
			return imag ? 0.f : t;
		}
		real lam = 0.f;
#pragma unroll
		for (int c = 0; c < 3; c++) {
			const real ab = tsqrt(re[c] * re[c] + im[c] * im[c]);
			real t = ab - thr;
			t = t >= 0.f ? t : 0.f;
			if (c < dims) lam += t;
			// the reference's 3D complex shrinkage scales the z component's
			// modulus by the y component's direction (3d/tval3_cpu_3d.cpp:934-937);
			// kept, as its 3D Dt quirk is
			const int dc = (dims == 3 && c == 2) ? 1 : c;
			w[c] = ab > 0.f ? t * (imag ? im[dc] : re[dc]) / ab : 0.f;
		}
		return imag ? 0.f : lam;
	}
};

// shrinkage at image element j: loads its gradient components u and
// multipliers s (and, for complex data, the other plane's) and returns the
// lambda1 share
__device__ __forceinline__ real shrink_at(const Inst &I, const Shrink &sh, int j, const real *const (&Uc)[3],
                                           const real *const (&Sc)[3], real (&u)[3], real (&s)[3],
                                           real (&w)[3]) {
	const int dims = I.dims;
#pragma unroll
	for (int c = 0; c < 3; c++) {
		u[c] = c < dims ? Uc[c][j] : 0.f;
		s[c] = c < dims ? Sc[c][j] : 0.f;
	}
	if (!I.cplx) return sh.apply(u, s, w);
	const int h = (int)(I.n >> 1);
	const bool imag = j >= h;
	const int jp = imag ? j - h : j + h;
	real up[3], sp[3];
#pragma unroll
	for (int c = 0; c < 3; c++) {
		up[c] = c < dims ? Uc[c][jp] : 0.f;
		sp[c] = c < dims ? Sc[c][jp] : 0.f;
	}
	return sh.apply_c(u, s, up, sp, imag, w);
}

__device__ __forceinline__ bool bad(double v) { return !isfinite(v); }

// ---------------------------------------------------------------------------
// scaleb (2d:229-266): first min |b| and first max |b|, scale into [0.5, 1.5]
// ---------------------------------------------------------------------------
__device__ __forceinline__ void better_min(real &a, int &ia, real b, int ib) {
	if (b < a || (b == a && ib < ia)) { a = b; ia = ib; }
}
__device__ __forceinline__ void better_max(real &a, int &ia, real b, int ib) {
	if (b > a || (b == a && ib < ia)) { a = b; ia = ib; }
}

template <bool MULTI>
__global__ void __launch_bounds__(BLOCK) k_scaleb(KArgs a) {
	KPROLOGUE(a);
	// complex data: over the m / 2 complex entries, |b| their modulus
	const int m = I.cplx ? (int)(I.m >> 1) : (int)I.m, i0 = local * TILE_M;
	real mn = INFINITY, mx = -INFINITY;
	int imn = INT_MAX, imx = INT_MAX;
	FOR_TILE_M(i0, m, i) {
		real v = I.cplx ? thypot(I.b_user[2 * i], I.b_user[2 * i + 1]) : tfabs(I.b_user[i]);
		better_min(mn, imn, v, i);
		better_max(mx, imx, v, i);
	}
	for (int o = 16; o > 0; o >>= 1) {
		real v = __shfl_xor_sync(0xffffffffu, mn, o);
		int iv = __shfl_xor_sync(0xffffffffu, imn, o);
		better_min(mn, imn, v, iv);
		v = __shfl_xor_sync(0xffffffffu, mx, o);
		iv = __shfl_xor_sync(0xffffffffu, imx, o);
		better_max(mx, imx, v, iv);
	}
	__shared__ real smn[32], smx[32];
	__shared__ int simn[32], simx[32];
	__shared__ int last;
	int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
	if (lane == 0) { smn[wid] = mn; simn[wid] = imn; smx[wid] = mx; simx[wid] = imx; }
	__syncthreads();
	if (threadIdx.x == 0) {
		for (int w = 1; w < BLOCK / 32; w++) {
			better_min(mn, imn, smn[w], simn[w]);
			better_max(mx, imx, smx[w], simx[w]);
		}
		double *P = I.part + (long long)local * NSUM;
		P[0] = mn; P[1] = (double)imn; P[2] = mx; P[3] = (double)imx;
		__threadfence();
		unsigned t = atomicAdd(&I.ctrl->ticket, 1u);
		last = (t == (unsigned)I.ntm - 1);
	}
	__syncthreads();
	if (!last || threadIdx.x != 0) return;
	__threadfence();
	real gmn = INFINITY, gmx = -INFINITY;
	int gimn = INT_MAX, gimx = INT_MAX;
	for (int t = 0; t < I.ntm; t++) {   // tiles in index order: first occurrence wins
		const double *P = I.part + (long long)t * NSUM;
		better_min(gmn, gimn, (real)__ldcg(P + 0), (int)__ldcg(P + 1));
		better_max(gmx, gimx, (real)__ldcg(P + 2), (int)__ldcg(P + 3));
	}
	Ctrl &c = *I.ctrl;
	double scl = 1.0;
	if (gimn < m && gimx < m) {   // (all-NaN data leaves no index: no scaling)
		// |bmax - bmin|; complex: the modulus of the difference (element type)
		double dif = I.cplx ? (double)thypot(I.b_user[2 * gimx] - I.b_user[2 * gimn],
		                                     I.b_user[2 * gimx + 1] - I.b_user[2 * gimn + 1])
		                    : fabs((double)I.b_user[gimx] - (double)I.b_user[gimn]);
		if (dif < 0.5) scl = 0.5 / dif;
		else if (dif > 1.5) scl = 1.5 / dif;
	}
	c.scl = scl;
	c.ticket = 0;
}

// ---------------------------------------------------------------------------
// initial state (2d:767-779): zero the vectors, bs = b*scl, scalar defaults
// ---------------------------------------------------------------------------
template <bool MULTI>
__global__ void __launch_bounds__(BLOCK) k_init(KArgs a) {
	KPROLOGUE(a);
	Ctrl &c = *I.ctrl;
	if (local < I.ntn) {
		FOR_TILE(local, (int)I.n, i) {
#pragma unroll
			for (int v = 0; v < NVN; v++) I.vn[v][i] = 0.f;
		}
		if (local == 0 && threadIdx.x == 0) {
			c.mu = I.mu0; c.beta = I.beta0;
			if (c.mu > I.muf) c.mu = I.muf;
			if (c.beta > I.betaf) c.beta = I.betaf;
			if (I.sched) { c.mu = I.sched[0]; c.beta = I.sched[I.maxit]; }   // (mu_1, beta_1)
			c.step = 0; c.sched_ratio = 1;
			c.muDbeta = c.mu / c.beta;
			c.gam = I.gam0; c.Q = 1; c.C = 0; c.f = 0;
			c.lam1 = c.lam2 = c.lam3 = c.lam4 = c.lam5 = 0;
			c.tau = c.alpha = c.c_armij = c.nrmup = c.relchg = c.relchg_out = c.beta0 = 0;
			c.dd = c.dDd = 0; c.currSkip = 0; c.currInit = 0; c.rel_error = 0;
			c.count_outer = c.count_total = 0;
			c.fst = 1; c.active = 1; c.need_bt = c.bt_cnt = c.restart = c.inner_break = 0;
			c.need_mlp = c.need_Ad = c.skip_adj = 0; c.status = 0;
		}
	} else {
		const real scl = (real)c.scl;
		FOR_TILE_M((local - I.ntn) * TILE_M, (int)I.m, i) {
#pragma unroll
			for (int v = 0; v < NVM; v++) I.vm[v][i] = 0.f;
			const real bu = I.b_user[cplx_index(I, i, I.m)];
			I.vm[vB][i] = scl != 1.f ? bu * scl : bu;
		}
	}
}

// U = Atb, rcdU = U (2d:775,779)
template <bool MULTI>
__global__ void __launch_bounds__(BLOCK) k_init_u(KArgs a) {
	KPROLOGUE(a);
	FOR_TILE(local, (int)I.n, i) {
		real u = I.vn[vAtb][i];
		I.vn[vU][i] = u;
		I.vn[vRcd][i] = u;
	}
}

// (Ux, Uy[, Uz]) = D U
template <bool MULTI>
__global__ void __launch_bounds__(BLOCK) k_D(KArgs a) {
	KPROLOGUE(a);
	Geo g(I);
	const real *__restrict__ U = I.vn[vU];
	real *__restrict__ ux = I.vn[vUx], *__restrict__ uy = I.vn[vUy], *__restrict__ uz = I.vn[vUz];
	FOR_TILE(local, g.n, i) {
		int x, y, z;
		g.coords(i, x, y, z);
		ux[i] = dxf(U, g, i, x);
		uy[i] = dyf(U, g, i, y);
		if (g.dims == 3) uz[i] = dzf(U, g, i, z);
	}
}

// ---------------------------------------------------------------------------
// update_W (2d:651-671) at initialisation: shrinkage W, lambda1, lambda2,
// lambda4 (g2 follows in k_getg).  In the inner loop update_W runs inside
// k_shrink_grad.
// ---------------------------------------------------------------------------
template <bool MULTI>
__global__ void __launch_bounds__(BLOCK) k_shrink(KArgs a) {
	KPROLOGUE(a);
	Ctrl &c = *I.ctrl;
	Shrink sh(I, c.beta);
	const int n = (int)I.n, dims = I.dims;
	const real *const Uc[3] = {I.vn[vUx], I.vn[vUy], I.vn[vUz]};
	const real *const Sc[3] = {I.vn[vSx], I.vn[vSy], I.vn[vSz]};
	double v[3] = {0, 0, 0};   // lam1, lam2, lam4
	FOR_TILE(local, n, i) {
		real u[3], s[3], w[3];
		v[0] += shrink_at(I, sh, i, Uc, Sc, u, s, w);
#pragma unroll
		for (int cc = 0; cc < 3; cc++)
			if (cc < dims) {
				I.vn[vWx + cc][i] = w[cc];
				real vv = u[cc] - w[cc];
				v[1] += (double)vv * vv;
				v[2] += (double)s[cc] * vv;
			}
	}
	double tot[3];
	if (!tile_reduce<3>(I, local, I.ntn, v, tot)) return;
	if (threadIdx.x != 0) return;
	c.lam1 = tot[0]; c.lam2 = tot[1]; c.lam4 = tot[2];
	set_conds(a.cs, c);
}

// component cc of D U at j, from U (2d:268-278, 3d:365-389)
__device__ __forceinline__ real du_at(const real *__restrict__ U, const Geo &g, int j, int cc) {
	int x, y, z;
	g.coords(j, x, y, z);
	return cc == 0 ? dxf(U, g, j, x) : cc == 1 ? dyf(U, g, j, y) : dzf(U, g, j, z);
}

// g2 at i: Dt(DU - W) with D U formed from U here (2d:280-293)
__device__ __forceinline__ real g2_at_u(const Inst &I, const Geo &g, int i, int x, int y, int z) {
	const real *__restrict__ U = I.vn[vU];
	const real *const Wc[3] = {I.vn[vWx], I.vn[vWy], I.vn[vWz]};
	auto V = [&](int cc) { return [&, cc](int j) { return du_at(U, g, j, cc) - Wc[cc][j]; }; };
	return dt_at(g, i, x, y, z, V(0), V(1), V(2));
}

// ---------------------------------------------------------------------------
// get_g epilogue (2d:396-423): g -= Atb; V = DU - W; g2 = Dt V; lam2, lam4;
// Aub = Au - b; lam3, lam5; f.  Descent stage also runs the Armijo test
// (2d:543-548).  The gradient components (Ux, Uy[, Uz]) = D U of the new U
// (the end of descend, 2d:481-493) are formed here and stored.
// ---------------------------------------------------------------------------
template <bool MULTI>
__global__ void __launch_bounds__(BLOCK, MULTI ? MINB(6) : 1) k_getg(KArgs a) {
	KPROLOGUE(a);
	Ctrl &c = *I.ctrl;
	double v[4] = {0, 0, 0, 0};   // lam2, lam4, lam3, lam5
	if (local < I.ntn) {
		Geo g(I);
		const real *__restrict__ U = I.vn[vU];
		real *const Uc[3] = {I.vn[vUx], I.vn[vUy], I.vn[vUz]};
		const real *const Wc[3] = {I.vn[vWx], I.vn[vWy], I.vn[vWz]};
		const real *const Sc[3] = {I.vn[vSx], I.vn[vSy], I.vn[vSz]};
		real *__restrict__ gv = I.vn[vG];
		real *__restrict__ g2 = I.vn[vG2];
		const real *__restrict__ atb = I.vn[vAtb];
		FOR_TILE(local, g.n, i) {
			int x, y, z;
			g.coords(i, x, y, z);
			// every load before the first store (the vectors do not alias)
			const real gi = gv[i] - atb[i];
			// in the inner loop k_shrink_grad forms g2 again from the new W
			// before anything reads it, so only the initialisation needs it
			const real g2i = a.stage == ST_INIT ? g2_at_u(I, g, i, x, y, z) : 0.f;
			real du[3] = {dxf(U, g, i, x), dyf(U, g, i, y), g.dims == 3 ? dzf(U, g, i, z) : 0.f};
			real wc[3], sc[3];
#pragma unroll
			for (int cc = 0; cc < 3; cc++) {
				wc[cc] = cc < g.dims ? Wc[cc][i] : 0.f;
				sc[cc] = cc < g.dims ? Sc[cc][i] : 0.f;
			}
			gv[i] = gi;
			if (a.stage == ST_INIT) g2[i] = g2i;
#pragma unroll
			for (int cc = 0; cc < 3; cc++)
				if (cc < g.dims) {
					Uc[cc][i] = du[cc];
					real vv = du[cc] - wc[cc];
					v[0] += (double)vv * vv;
					v[1] += (double)sc[cc] * vv;
				}
		}
	} else {
		const real *__restrict__ au = I.vm[vAu], *__restrict__ bb = I.vm[vB], *__restrict__ dl = I.vm[vDelta];
		FOR_TILE_M((local - I.ntn) * TILE_M, (int)I.m, i) {
			real r = au[i] - bb[i];
			v[2] += (double)r * r;
			v[3] += (double)dl[i] * r;
		}
	}
	double tot[4];
	if (!tile_reduce<4>(I, local, I.ntn + I.ntm, v, tot)) return;
	if (threadIdx.x != 0) return;
	c.lam2 = tot[0]; c.lam4 = tot[1]; c.lam3 = tot[2]; c.lam5 = tot[3];
	c.f = (c.lam1 + c.beta / 2 * c.lam2 + c.mu / 2 * c.lam3) - c.lam4 - c.lam5;
	if (a.stage == ST_DESCEND || a.stage == ST_RESTART) c.step = c.tau;
	if (a.stage == ST_DESCEND) {
		c.alpha = 1;
		c.c_armij = c.dd * c.tau * I.c * c.beta;
		c.need_bt = fabs(c.f) > fabs(c.C - c.alpha * c.c_armij);
		c.bt_cnt = 0;
		if (bad(c.f)) { c.status = TVAL3G_ERR_NONFINITE; c.active = 0; c.need_bt = 0; }
	} else if (a.stage == ST_RESTART) {
		c.restart = 0;
		c.need_bt = 0;
		c.bt_cnt = 6;   // marks the restart in the trace
		if (I.skip_enabled) c.currSkip = 0;
	} else if (a.stage == ST_INIT) {
		if (I.skip_enabled) c.currSkip = 0;
	}
	set_conds(a.cs, c);
}

// ---------------------------------------------------------------------------
// get_gradient (2d:578-585) outside the inner loop:
//   ST_INIT:  d = DtsAtd + g2 + muDbeta*g (DtsAtd = 0); Q = 1, C = f
//   ST_OUTER: DtsAtd = (beta0/beta) d; d = ... (2d:844-852)
// ---------------------------------------------------------------------------
template <bool MULTI>
__global__ void __launch_bounds__(BLOCK) k_grad(KArgs a) {
	KPROLOGUE(a);
	Ctrl &c = *I.ctrl;
	const real mdb = (real)c.muDbeta;
	const real bscale = a.stage == ST_OUTER ? (real)(c.beta0 / c.beta) : 1.f;
	real *__restrict__ dts = I.vn[vDts], *__restrict__ d = I.vn[vD];
	const real *__restrict__ g2 = I.vn[vG2], *__restrict__ gv = I.vn[vG];
	double v[1] = {0};   // |d|^2
	FOR_TILE(local, (int)I.n, i) {
		// every load before the first store
		real t = a.stage == ST_OUTER ? d[i] * bscale : dts[i];
		const real g2i = g2[i], gvi = gv[i];
		if (a.stage == ST_OUTER) dts[i] = t;
		real dv = t + g2i;
		dv = tfma(mdb, gvi, dv);
		d[i] = dv;
		v[0] += (double)dv * dv;
	}
	double tot[1];
	if (!tile_reduce<1>(I, local, I.ntn, v, tot)) return;
	if (threadIdx.x != 0) return;
	c.dd = tot[0];
	if (a.stage == ST_INIT) {
		c.Q = 1; c.C = c.f;
		c.count_outer = 0; c.count_total = 0; c.fst = 1;
		c.active = (I.maxcnt > 0 && I.maxit > 0);
		if (bad(c.f) || bad(c.dd)) { c.status = TVAL3G_ERR_NONFINITE; c.active = 0; }
	} else {   // ST_OUTER
		c.need_mlp = 0; c.fst = 1; c.inner_break = 0;
		c.gam = I.gam0; c.Q = 1; c.C = c.f;
	}
	set_conds(a.cs, c);
}

// ---------------------------------------------------------------------------
// The inner loop's update_W (2d:651-671) and get_gradient with the inner
// stopping test (2d:578-585, 803-817) in one pass over the image:
//   W = shrink(U_c - sigma_c / beta) at the pixel, stored, and recomputed
//   from their U_c and sigma_c at the pixels Dt reads; g2 = Dt(DU - W);
//   d = DtsAtd + g2 + muDbeta*g; uup = U - Up; the sums of both steps.
// The last tile runs update_W's scalar step (f, the nonmonotone reference
// values Q and C, 2d:802) and then the inner loop's (RelChg, stopping test,
// trace, time-to-solution target).
// ---------------------------------------------------------------------------
template <bool MULTI>
__global__ void __launch_bounds__(BLOCK, MULTI ? MINB(4) : MINB(3)) k_shrink_grad(KArgs a) {
	KPROLOGUE(a);
	Ctrl &c = *I.ctrl;
	Geo g(I);
	Shrink sh(I, c.beta);
	const int dims = I.dims;
	const real *const Uc[3] = {I.vn[vUx], I.vn[vUy], I.vn[vUz]};
	const real *const Sc[3] = {I.vn[vSx], I.vn[vSy], I.vn[vSz]};
	const real mdb = (real)c.muDbeta;
	real *__restrict__ d = I.vn[vD], *__restrict__ uup = I.vn[vUUP];
	const real *__restrict__ dts = I.vn[vDts], *__restrict__ gv = I.vn[vG];
	const real *__restrict__ U = I.vn[vU], *__restrict__ Up = I.vn[vUp];
	// distance to Ut after the iteration (trace / time-to-solution target)
	const bool ut = I.ut_user && (I.trace || I.target > 0);
	const real rscl = (real)(1.0 / c.scl);
	// the next iteration's Barzilai-Borwein step (get_tau, 2d:444-451) from
	// this iteration's uup, g - gp, g2 - g2p (schedule mode: k_tau_prep, as
	// mu and beta change before that step)
	// (complex data: k_tau_bb_cplx, which needs the other plane's g2)
	const bool bb = !I.sched && !I.cplx;
	const real *__restrict__ gp = I.vn[vGp], *__restrict__ g2p = I.vn[vG2p];
	// lam1, lam2, lam4, |d|^2, |Up|^2, |uup|^2, |U/scl - Ut|^2, |Ut|^2, <uup, dg2 + muDbeta dg>
	double v[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
	FOR_TILE(local, g.n, i) {
		int x, y, z;
		g.coords(i, x, y, z);
		real u[3], s[3], w[3];
		v[0] += shrink_at(I, sh, i, Uc, Sc, u, s, w);
#pragma unroll
		for (int cc = 0; cc < 3; cc++)
			if (cc < dims) {
				const real vv = u[cc] - w[cc];
				v[1] += (double)vv * vv;
				v[2] += (double)s[cc] * vv;
			}
		// component cc of DU - W at j (the neighbours' W recomputed)
		// (anisotropic real data: only component cc of U and sigma at j)
		const bool one = !sh.iso && !I.cplx;
		auto V = [&](int cc) {
			return [&, cc](int j) -> real {
				if (j == i) return u[cc] - w[cc];
				if (one) {
					const real uj = Uc[cc][j];
					return uj - sh.apply1(uj, Sc[cc][j]);
				}
				real uj[3], sj[3], wj[3];
				shrink_at(I, sh, j, Uc, Sc, uj, sj, wj);
				return uj[cc] - wj[cc];
			};
		};
		// every load before the first store (the vectors do not alias: a load
		// the compiler kept behind a store would wait for the store's data)
		const real g2i = dt_at(g, i, x, y, z, V(0), V(1), V(2));
		const real dtsi = dts[i], gvi = gv[i], up = Up[i], Ui = U[i];
		const real gpi = bb ? gp[i] : 0.f, g2pi = bb ? g2p[i] : 0.f;
		const real uti = ut ? I.ut_user[cplx_index(I, i, I.n)] : 0.f;
#pragma unroll
		for (int cc = 0; cc < 3; cc++)
			if (cc < dims) I.vn[vWx + cc][i] = w[cc];
		I.vn[vG2][i] = g2i;
		real dv = dtsi + g2i;
		dv = tfma(mdb, gvi, dv);
		d[i] = dv;
		v[3] += (double)dv * dv;
		const real uu = Ui - up;
		uup[i] = uu;
		v[4] += (double)up * up;
		v[5] += (double)uu * uu;
		if (bb) {
			const real tmp = tfma(mdb, gvi - gpi, g2i - g2pi);
			v[8] += (double)uu * tmp;
		}
		if (ut) {
			const real e = Ui * rscl - uti;
			v[6] += (double)e * e;
			v[7] += (double)uti * uti;
		}
	}
	double tot[9];
	if (!tile_reduce<9>(I, local, I.ntn, v, tot)) return;
	if (threadIdx.x != 0) return;
	// update_W: objective and nonmonotone reference values
	c.f -= (c.lam1 + c.beta / 2 * c.lam2 - c.lam4);
	c.lam1 = tot[0]; c.lam2 = tot[1]; c.lam4 = tot[2];
	c.f += (c.lam1 + c.beta / 2 * c.lam2 - c.lam4);
	const double Qp = c.Q;
	c.Q = c.gam * Qp + 1;
	c.C = (c.gam * Qp * c.C + c.f) / c.Q;
	// get_gradient and the inner stopping test
	c.dd = tot[3];
	c.count_total++;
	c.nrmup = sqrt(tot[4]);
	c.relchg = sqrt(tot[5]) / c.nrmup;
	c.relerr_ut = ut ? sqrt(tot[6]) / sqrt(tot[7]) : 0.0;
	if (I.trace && c.count_total <= I.maxit) {
		double *t = I.trace + (long long)(c.count_total - 1) * TRACE_DOUBLES;
		t[0] = c.tau; t[1] = c.f; t[2] = c.relchg; t[3] = c.bt_cnt; t[4] = c.skip_adj; t[5] = c.relerr_ut;
		t[6] = c.step; t[7] = 0;
	}
	c.bt_cnt = 0;
	c.need_bt = 0;   // an accepted backtracking step leaves it set for k_lerp
	const bool brk = (c.relchg < I.tol_inn) && !c.fst;
	c.inner_break = brk || c.count_total >= I.maxit;
	if (!brk) c.fst = 0;
	if (ut && I.target > 0 && c.relerr_ut <= I.target) {   // time-to-solution target reached
		c.active = 0;
		c.inner_break = 0;
	}
	if (bad(c.dd)) { c.status = TVAL3G_ERR_NONFINITE; c.active = 0; c.inner_break = 0; }
	// the next iteration's step length when it takes the Barzilai-Borwein form
	if (bb && c.active && !c.inner_break && !c.fst) {
		c.tau = fabs(tot[5] / tot[8]);
		if (bad(c.tau)) { c.status = TVAL3G_ERR_NONFINITE; c.active = 0; }
	}
	set_conds(a.cs, c);
}

// ---------------------------------------------------------------------------
// The Barzilai-Borwein step of complex data (2d:444-451, 3d:605-616):
// tau = |ss / sy| with ss = <uup, uup> and sy = <uup, dg2 + muDbeta dg> the
// complex inner product; on the planar vectors (real plane, imaginary plane
// of h elements each) Re sy = sum over both planes of uup tmp and
// Im sy = sum_i uup_i tmp_{i+h} - uup_{i+h} tmp_i.  It runs after
// k_shrink_grad (which writes the imaginary plane's g2 too); real instances
// take the step from k_shrink_grad.
// ---------------------------------------------------------------------------
template <bool MULTI>
__global__ void __launch_bounds__(BLOCK) k_tau_bb_cplx(KArgs a) {
	KPROLOGUE(a);
	if (!I.cplx) return;
	Ctrl &c = *I.ctrl;
	const real mdb = (real)c.muDbeta;
	const int h = (int)(I.n >> 1);
	const real *__restrict__ gv = I.vn[vG], *__restrict__ gp = I.vn[vGp];
	const real *__restrict__ g2 = I.vn[vG2], *__restrict__ g2p = I.vn[vG2p], *__restrict__ uup = I.vn[vUUP];
	double v[3] = {0, 0, 0};   // ss, Re sy, Im sy
	FOR_TILE(local, h, i) {
		const real ur = uup[i], ui = uup[i + h];
		const real tr = tfma(mdb, gv[i] - gp[i], g2[i] - g2p[i]);
		const real ti = tfma(mdb, gv[i + h] - gp[i + h], g2[i + h] - g2p[i + h]);
		v[0] += (double)ur * ur + (double)ui * ui;
		v[1] += (double)ur * tr + (double)ui * ti;
		v[2] += (double)ur * ti - (double)ui * tr;
	}
	double tot[3];
	if (!tile_reduce<3>(I, local, I.ntn, v, tot)) return;
	if (threadIdx.x != 0) return;
	if (c.active && !c.inner_break && !c.fst) {
		c.tau = fabs(tot[0]) / sqrt(tot[1] * tot[1] + tot[2] * tot[2]);
		if (bad(c.tau)) { c.status = TVAL3G_ERR_NONFINITE; c.active = 0; }
	}
}

// ---------------------------------------------------------------------------
// get_tau (2d:425-453), first part.  First iteration (or restart): dDd =
// |D d|^2 and request A d.  Otherwise Barzilai-Borwein from uup, dg, dg2.
// ---------------------------------------------------------------------------
template <bool MULTI>
__global__ void __launch_bounds__(BLOCK) k_tau_prep(KArgs a) {
	KPROLOGUE(a);
	Ctrl &c = *I.ctrl;
	const bool first = c.restart || c.fst;
	const real mdb = (real)c.muDbeta;
	Geo g(I);
	double v[3] = {0, 0, 0};
	const real *__restrict__ d = I.vn[vD];
	if (first) {
		FOR_TILE(local, g.n, i) {
			int x, y, z;
			g.coords(i, x, y, z);
			real t = dxf(d, g, i, x);
			v[0] += (double)t * t;
			t = dyf(d, g, i, y);
			v[0] += (double)t * t;
			if (g.dims == 3) { t = dzf(d, g, i, z); v[0] += (double)t * t; }
		}
	} else {
		const real *__restrict__ gv = I.vn[vG], *__restrict__ gp = I.vn[vGp];
		const real *__restrict__ g2 = I.vn[vG2], *__restrict__ g2p = I.vn[vG2p], *__restrict__ uup = I.vn[vUUP];
		FOR_TILE(local, g.n, i) {
			real dg = gv[i] - gp[i];
			real dg2 = g2[i] - g2p[i];
			real uu = uup[i];
			real tmp = tfma(mdb, dg, dg2);
			v[0] += (double)uu * uu;
			v[1] += (double)uu * tmp;
			if (I.cplx && i < g.n / 2) {   // Im sy (complex data, as k_tau_bb_cplx)
				const int j = i + g.n / 2;
				const real tj = tfma(mdb, gv[j] - gp[j], g2[j] - g2p[j]);
				v[2] += (double)uu * tj - (double)uup[j] * tmp;
			}
		}
	}
	double tot[3];
	if (!tile_reduce<3>(I, local, I.ntn, v, tot)) return;
	if (threadIdx.x != 0) return;
	if (first) {
		c.dDd = tot[0];
		c.need_Ad = 1;
	} else {
		c.tau = fabs(tot[0]) / sqrt(tot[1] * tot[1] + tot[2] * tot[2]);
		if (bad(c.tau)) { c.status = TVAL3G_ERR_NONFINITE; c.active = 0; }
	}
	set_conds(a.cs, c);
}

// first-iteration step: tau = |dd / (dDd + muDbeta * |A d|^2)| (2d:430-442)
template <bool MULTI>
__global__ void __launch_bounds__(BLOCK) k_tau_first(KArgs a) {
	KPROLOGUE(a);
	Ctrl &c = *I.ctrl;
	double v[1] = {0};
	const real *__restrict__ ad = I.vm[vAd];
	FOR_TILE_M(local * TILE_M, (int)I.m, i) {
		real t = ad[i];
		v[0] += (double)t * t;
	}
	double tot[1];
	if (!tile_reduce<1>(I, local, I.ntm, v, tot)) return;
	if (threadIdx.x != 0) return;
	c.tau = fabs(c.dd / (c.dDd + c.muDbeta * tot[0]));
	c.need_Ad = 0;
	if (bad(c.tau)) { c.status = TVAL3G_ERR_NONFINITE; c.active = 0; c.restart = 0; c.need_bt = 0; }
	set_conds(a.cs, c);
}

// ---------------------------------------------------------------------------
// descend (2d:481-493) with the snapshot of min_u (2d:536-537); for a 2D ray
// operator it also writes the new U transposed (OpDev::xT), which the
// forward projection that follows reads for its y-driven rays:
//   ST_DESCEND: Up=U, gp=g, g2p=g2, U[xyz]p=U[xyz], Aup=Au; U = U - tau d
//   ST_RESTART: U = Up - tau d (2d:565-566)
// then nonneg (2d:455-465)
// ---------------------------------------------------------------------------
template <bool MULTI>
__global__ void __launch_bounds__(BLOCK, MULTI ? MINB(6) : 1) k_descend(KArgs a) {
	KPROLOGUE(a);
	Ctrl &c = *I.ctrl;
	const real ntau = (real)(-1 * c.tau);
	const bool snap = a.stage == ST_DESCEND;
	const real sratio = (real)c.sched_ratio;
	if (local < I.ntn) {
		real *__restrict__ U = I.vn[vU], *__restrict__ Up = I.vn[vUp];
		const real *__restrict__ d = I.vn[vD];
		real *__restrict__ xT = I.op.xT;   // 2D ray operators: the new U transposed for the forward
		const int ld = I.op.rvx, tH = I.op.tH;   // the geometry's row length (its ld)
		FOR_TILE(local, (int)I.n, i) {
			real u;
			const real dv = d[i];
			if (snap) {
				// every load before the first store: the compiler cannot tell that
				// the vectors do not alias, and a load after a store would wait
				// for the store's data
				u = U[i];
				const real gi = I.vn[vG][i], g2i = I.vn[vG2][i];
				real uc[3];
#pragma unroll
				for (int cc = 0; cc < 3; cc++) uc[cc] = cc < I.dims ? I.vn[vUx + cc][i] : 0.f;
				const real dts = I.sched ? I.vn[vDts][i] : 0.f;
				Up[i] = u;
				I.vn[vGp][i] = gi;
				I.vn[vG2p][i] = g2i;
#pragma unroll
				for (int cc = 0; cc < 3; cc++)
					if (cc < I.dims) I.vn[vUxp + cc][i] = uc[cc];
				// schedule mode: DtsAtd = -(Dt sigma + At delta) / beta for this iteration's beta
				if (I.sched) I.vn[vDts][i] = dts * sratio;
			} else {
				u = Up[i];
			}
			u = tfma(ntau, dv, u);
			if (I.nonneg) u = (I.cplx && i >= (int)(I.n >> 1)) ? 0.f : (u < 0.f ? 0.f : u);   // complex: Re >= 0, Im = 0 (2d:467-479)
			U[i] = u;
			if (xT) {
				const int row = i / ld;
				xT[row + (i - row * ld) * tH] = u;
			}
		}
	} else if (snap) {
		const int i0 = (local - I.ntn) * TILE_M;
		LOAD_TILE_M(i0, (int)I.m, au, I.vm[vAu][i])
		FOR_TILE_M(i0, (int)I.m, i) I.vm[vAup][i] = au[k_];
	}
}

// Nonmonotone Armijo backtracking (2d:544-574) in one pass over the vectors.
// The reference's loop sets alpha *= gamma and evaluates f at
//   U(alpha) = Up + alpha (U - Up),  likewise g, g2, Ux, Uy (, Uz), Au
// (update_g, 2d:495-524), up to five times, then restarts.  Every term of
// f is a polynomial in alpha over these interpolants:
//   lam2(a) = |E0 + a dU'|^2,  lam4(a) = <S, E0> + a <S, dU'>      (E0 = U'p - W, dU' = U' - U'p)
//   lam3(a) = |R0 + a dAu|^2,  lam5(a) = <delta, R0> + a <delta, dAu>   (R0 = Aup - b)
// so k_bt_search forms their coefficients once (lam4(1), lam5(1) come from
// k_getg) and its last block runs the loop on them; k_lerp then moves the
// vectors to the accepted alpha once, with the reference's arithmetic in the element type
// (fma(alpha, U - Up, Up)).  When all five steps fail the vectors are not
// moved: the restart (2d:561-567) recomputes every one of them from Up.
template <bool MULTI>
__global__ void __launch_bounds__(BLOCK) k_bt_search(KArgs a) {
	KPROLOGUE(a);
	Ctrl &c = *I.ctrl;
	// |E0|^2, <E0, dU'>, |dU'|^2, <S, E0>; |R0|^2, <R0, dAu>, |dAu|^2, <delta, R0>
	double v[8] = {0, 0, 0, 0, 0, 0, 0, 0};
	if (local < I.ntn) {
		FOR_TILE(local, (int)I.n, i) {
#pragma unroll
			for (int cc = 0; cc < 3; cc++)
				if (cc < I.dims) {
					const real up = I.vn[vUxp + cc][i];
					const real du = I.vn[vUx + cc][i] - up;
					const real e0 = up - I.vn[vWx + cc][i];
					v[0] += (double)e0 * e0;
					v[1] += (double)e0 * du;
					v[2] += (double)du * du;
					v[3] += (double)I.vn[vSx + cc][i] * e0;
				}
		}
	} else {
		FOR_TILE_M((local - I.ntn) * TILE_M, (int)I.m, i) {
			const real ap = I.vm[vAup][i];
			const real da = I.vm[vAu][i] - ap;
			const real r0 = ap - I.vm[vB][i];
			v[4] += (double)r0 * r0;
			v[5] += (double)r0 * da;
			v[6] += (double)da * da;
			v[7] += (double)I.vm[vDelta][i] * r0;
		}
	}
	double t[8];
	if (!tile_reduce<8>(I, local, I.ntn + I.ntm, v, t)) return;
	if (threadIdx.x != 0) return;
	const double s4 = c.lam4 - t[3], s5 = c.lam5 - t[7];   // slopes of the linear terms
	double al = c.alpha;
	int cnt = c.bt_cnt;
	for (;;) {
		if (cnt == 5) {   // backtracking not successful: restart
			c.gam *= I.rate_gam;
			c.restart = 1;
			break;
		}
		al *= I.gamma;
		cnt++;
		c.lam2 = t[0] + al * (2 * t[1] + al * t[2]);
		c.lam4 = t[3] + al * s4;
		c.lam3 = t[4] + al * (2 * t[5] + al * t[6]);
		c.lam5 = t[7] + al * s5;
		c.f = c.lam1 + c.beta / 2 * c.lam2 + c.mu / 2 * c.lam3 - c.lam4 - c.lam5;
		if (bad(c.f)) { c.status = TVAL3G_ERR_NONFINITE; c.active = 0; c.need_bt = 0; c.restart = 0; break; }
		if (!(fabs(c.f) > fabs(c.C - al * c.c_armij))) break;   // accepted: need_bt stays set for k_lerp
	}
	c.alpha = al;
	c.step = c.tau * al;
	c.bt_cnt = cnt;
	set_conds(a.cs, c);
}

// the accepted backtracking step: U' = U'p + alpha (U' - U'p) for U, g, Ux,
// Uy (, Uz) and Au (g2 is formed again by k_shrink_grad, which follows)
template <bool MULTI>
__global__ void __launch_bounds__(BLOCK) k_lerp(KArgs a) {
	KPROLOGUE(a);
	const real al = (real)I.ctrl->alpha;
	if (local < I.ntn) {
		FOR_TILE(local, (int)I.n, i) {
			// every load before the first store
			const real gi = I.vn[vG][i], gpi = I.vn[vGp][i], ui = I.vn[vU][i], upi = I.vn[vUp][i];
			real uc[3], ucp[3];
#pragma unroll
			for (int cc = 0; cc < 3; cc++) {
				uc[cc] = cc < I.dims ? I.vn[vUx + cc][i] : 0.f;
				ucp[cc] = cc < I.dims ? I.vn[vUxp + cc][i] : 0.f;
			}
			I.vn[vG][i] = tfma(al, gi - gpi, gpi);
			I.vn[vU][i] = tfma(al, ui - upi, upi);
#pragma unroll
			for (int cc = 0; cc < 3; cc++)
				if (cc < I.dims) I.vn[vUx + cc][i] = tfma(al, uc[cc] - ucp[cc], ucp[cc]);
		}
	} else {
		const int i0 = (local - I.ntn) * TILE_M;
		LOAD_TILE_M(i0, (int)I.m, au, I.vm[vAu][i])
		LOAD_TILE_M(i0, (int)I.m, aup, I.vm[vAup][i])
		FOR_TILE_M(i0, (int)I.m, i) I.vm[vAu][i] = tfma(al, au[k_] - aup[k_], aup[k_]);
	}
}

// outer stopping test (2d:820-828): RelChgOut = |U - rcdU| / nrmup; rcdU = U
template <bool MULTI>
__global__ void __launch_bounds__(BLOCK) k_outer(KArgs a) {
	KPROLOGUE(a);
	Ctrl &c = *I.ctrl;
	double v[1] = {0};
	real *__restrict__ rcd = I.vn[vRcd];
	const real *__restrict__ U = I.vn[vU];
	FOR_TILE(local, (int)I.n, i) {
		real u = U[i];
		real dlt = u - rcd[i];
		v[0] += (double)dlt * dlt;
		rcd[i] = u;
	}
	double tot[1];
	if (!tile_reduce<1>(I, local, I.ntn, v, tot)) return;
	if (threadIdx.x != 0) return;
	c.count_outer++;
	c.relchg_out = sqrt(tot[0]) / c.nrmup;
	c.inner_break = 0;
	// after the last outer step the reference still updates the multipliers,
	// which no longer changes U; that step is skipped here
	if (c.relchg_out < I.tol || c.count_outer >= I.maxcnt || c.count_total >= I.maxit) c.active = 0;
	else c.need_mlp = 1;
	if (I.trace && c.count_total >= 1 && c.count_total <= I.maxit)
		I.trace[(long long)(c.count_total - 1) * TRACE_DOUBLES + 7] = c.need_mlp;
}

// update_mlp (2d:673-694) and the continuation step (2d:834-842)
template <bool MULTI>
__global__ void __launch_bounds__(BLOCK) k_mlp(KArgs a) {
	KPROLOGUE(a);
	Ctrl &c = *I.ctrl;
	const real nbeta = (real)(-1 * c.beta), nmu = (real)(-1 * c.mu);
	double v[2] = {0, 0};   // lam4, lam5
	if (local < I.ntn) {
		FOR_TILE(local, (int)I.n, i) {
			real vv[3], sv[3];   // every load before the first store
#pragma unroll
			for (int cc = 0; cc < 3; cc++) {
				vv[cc] = cc < I.dims ? I.vn[vUx + cc][i] - I.vn[vWx + cc][i] : 0.f;
				sv[cc] = cc < I.dims ? I.vn[vSx + cc][i] : 0.f;
			}
#pragma unroll
			for (int cc = 0; cc < 3; cc++)
				if (cc < I.dims) {
					real s = tfma(nbeta, vv[cc], sv[cc]);
					I.vn[vSx + cc][i] = s;
					v[0] += (double)s * vv[cc];
				}
		}
	} else {
		const int i0 = (local - I.ntn) * TILE_M;
		LOAD_TILE_M(i0, (int)I.m, r, I.vm[vAu][i] - I.vm[vB][i])
		LOAD_TILE_M(i0, (int)I.m, dl0, I.vm[vDelta][i])
		FOR_TILE_M(i0, (int)I.m, i) {
			const real dl = tfma(nmu, r[k_], dl0[k_]);
			I.vm[vDelta][i] = dl;
			v[1] += (double)dl * r[k_];
		}
	}
	double tot[2];
	if (!tile_reduce<2>(I, local, I.ntn + I.ntm, v, tot)) return;
	if (threadIdx.x != 0) return;
	c.f += (c.lam4 + c.lam5);
	c.lam4 = tot[0]; c.lam5 = tot[1];
	c.f -= (c.lam4 + c.lam5);
	c.beta0 = c.beta;
	if (!I.sched) {   // schedule mode: mu and beta come from the schedule
		c.beta *= I.rate_cnt;
		c.mu *= I.rate_cnt;
		if (c.beta > I.betaf) c.beta = I.betaf;
		if (c.mu > I.muf) c.mu = I.muf;
	}
	c.muDbeta = c.mu / c.beta;
	c.f = c.lam1 + c.beta / 2 * c.lam2 + c.mu / 2 * c.lam3 - c.lam4 - c.lam5;
}

// final scaling and rel_error (2d:855-877)
template <bool MULTI>
__global__ void __launch_bounds__(BLOCK) k_final(KArgs a) {
	KPROLOGUE(a);
	Ctrl &c = *I.ctrl;
	const real scl = (real)c.scl;
	double v[2] = {0, 0};
	FOR_TILE(local, (int)I.n, i) {
		real u = I.vn[vU][i];
		if (I.cplx && I.isreal && i >= (int)(I.n >> 1)) u = 0.f;   // isreal: U = real(U) before scaling
		u = u / scl;
		const long long ui = cplx_index(I, i, I.n);
		I.u_user[ui] = u;
		if (I.ut_user) {
			real t = I.ut_user[ui];
			real dlt = t - u;
			v[0] += (double)dlt * dlt;
			v[1] += (double)t * t;
		}
	}
	double tot[2];
	if (!tile_reduce<2>(I, local, I.ntn, v, tot)) return;
	if (threadIdx.x != 0) return;
	c.rel_error = I.ut_user ? sqrt(tot[0]) / sqrt(tot[1]) : 0.0;
}

// A^T-skip heuristic (2d:306-355), decision part (not forced)
template <bool MULTI>
__global__ void __launch_bounds__(BLOCK) k_skip_norms(KArgs a) {
	KPROLOGUE(a);
	if (!I.skip_enabled) return;
	Ctrl &c = *I.ctrl;
	double v[2] = {0, 0};
	FOR_TILE_M(local * TILE_M, (int)I.m, i) {
		real au = I.vm[vAu][i];
		real dl = au - I.vm[vLastAu][i];
		v[0] += (double)dl * dl;
		v[1] += (double)au * au;
	}
	double tot[2];
	if (!tile_reduce<2>(I, local, I.ntm, v, tot)) return;
	if (threadIdx.x != 0) return;
	double rel = sqrt(tot[0]) / sqrt(tot[1]);
	bool mul = true;
	if (c.currInit < I.numInit) { c.currInit++; c.currSkip = 0; }
	else if (c.currSkip < 1) { c.currSkip += I.skipRatio; }
	else if (rel > I.maxRelChange) { }
	else { mul = false; c.currSkip -= 1; }
	c.skip_adj = !mul;
}

template <bool MULTI>
__global__ void __launch_bounds__(BLOCK) k_copy_lastau(KArgs a) {
	KPROLOGUE(a);
	if (!I.skip_enabled) return;
	LOAD_TILE_M(local * TILE_M, (int)I.m, au, I.vm[vAu][i])
	FOR_TILE_M(local * TILE_M, (int)I.m, i) I.vm[vLastAu][i] = au[k_];
}

__global__ void k_cond(const Inst *tab, int count, int pred, int *flag, unsigned long long handle,
                       unsigned long long *launches) {
	pdl_launch_next();
	if (launches && threadIdx.x == 0) atomicAdd(launches, 1ull);
	pdl_wait_prev();
	int any = 0;
	for (int i = threadIdx.x; i < count; i += blockDim.x) any |= pred_ok(*tab[i].ctrl, pred) ? 1 : 0;
	any = __syncthreads_or(any);
	if (threadIdx.x == 0) {
		*flag = any;
		if (handle) cudaGraphSetConditional((cudaGraphConditionalHandle)handle, any ? 1u : 0u);
	}
}

// schedule mode: the coming iteration's (mu_k, beta_k) from the schedule, and
// the ratio by which DtsAtd = -(Dt sigma + At delta) / beta must be rescaled
__global__ void k_sched(const Inst *tab, int count, unsigned long long *launches) {
	pdl_launch_next();
	if (launches && blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(launches, 1ull);
	pdl_wait_prev();
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= count) return;
	const Inst &I = tab[i];
	Ctrl &c = *I.ctrl;
	if (!I.sched || !c.active) return;
	const int k = c.count_total;   // iterations done: the coming one is k + 1
	if (k >= I.maxit) return;
	const double mu = I.sched[k], beta = I.sched[I.maxit + k];
	c.sched_ratio = c.beta / beta;
	c.mu = mu;
	c.beta = beta;
	c.muDbeta = mu / beta;
}

// ---------------------------------------------------------------------------
// standalone stencils
// ---------------------------------------------------------------------------
struct PlainGeo {
	int dims, p, q, r;
	FastDiv fq, fp;
};

__device__ __forceinline__ Geo plain_geo(const PlainGeo &pg) {
	Inst I{};
	I.dims = pg.dims; I.p = pg.p; I.q = pg.q; I.r = pg.r;
	I.n = (long long)pg.p * pg.q * pg.r;
	I.fq = pg.fq; I.fp = pg.fp;
	return Geo(I);
}

__global__ void k_D_plain(PlainGeo pg, const real *U, real *Ux, real *Uy, real *Uz) {
	Geo g = plain_geo(pg);
	for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < g.n; i += gridDim.x * blockDim.x) {
		int x, y, z;
		g.coords(i, x, y, z);
		Ux[i] = dxf(U, g, i, x);
		Uy[i] = dyf(U, g, i, y);
		if (g.dims == 3) Uz[i] = dzf(U, g, i, z);
	}
}

__global__ void k_Dt_plain(PlainGeo pg, const real *X, const real *Y, const real *Z, real *res) {
	Geo g = plain_geo(pg);
	for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < g.n; i += gridDim.x * blockDim.x) {
		int x, y, z;
		g.coords(i, x, y, z);
		res[i] = dt_at(g, i, x, y, z, [&](int j) { return X[j]; }, [&](int j) { return Y[j]; },
		               [&](int j) { return Z ? Z[j] : 0.f; });
	}
}

__global__ void k_shrink_plain(int dims, long long n, int iso, double beta, const real *Ux, const real *Uy,
                               const real *Uz, const real *sx, const real *sy, const real *sz, real *Wx,
                               real *Wy, real *Wz, double *lam1) {
	Inst I{};
	I.dims = dims; I.tv_norm = iso;
	Shrink sh(I, beta);
	double acc[1] = {0};
	for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
	     i += (long long)gridDim.x * blockDim.x) {
		real u[3] = {Ux[i], Uy[i], dims == 3 ? Uz[i] : 0.f};
		real s[3] = {sx[i], sy[i], dims == 3 ? sz[i] : 0.f};
		real w[3];
		acc[0] += sh.apply(u, s, w);
		Wx[i] = w[0]; Wy[i] = w[1];
		if (dims == 3) Wz[i] = w[2];
	}
	__shared__ double sm[NSUM * 32];
	block_sums<1>(acc, sm);
	if (threadIdx.x == 0) atomicAdd(lam1, acc[0]);
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
#define LAUNCHER(name, kern)                                                  \
	void name(cudaStream_t s, const KArgs &a) {                               \
		if (a.map.count <= 0) return;                                         \
		if (a.multi) launch_pdl(kern<true>, a.map.count, BLOCK, 0, s, a);     \
		else launch_pdl(kern<false>, a.map.count, BLOCK, 0, s, a);            \
	}
LAUNCHER(launch_scaleb, k_scaleb)
LAUNCHER(launch_init, k_init)
LAUNCHER(launch_init_u, k_init_u)
LAUNCHER(launch_D, k_D)
LAUNCHER(launch_shrink, k_shrink)
LAUNCHER(launch_getg, k_getg)
LAUNCHER(launch_grad, k_grad)
LAUNCHER(launch_shrink_grad, k_shrink_grad)
LAUNCHER(launch_tau_prep, k_tau_prep)
LAUNCHER(launch_tau_bb_cplx, k_tau_bb_cplx)
LAUNCHER(launch_tau_first, k_tau_first)
LAUNCHER(launch_descend, k_descend)
LAUNCHER(launch_bt_search, k_bt_search)
LAUNCHER(launch_lerp, k_lerp)
LAUNCHER(launch_outer, k_outer)
LAUNCHER(launch_mlp, k_mlp)
LAUNCHER(launch_final, k_final)
LAUNCHER(launch_skip_norms, k_skip_norms)
LAUNCHER(launch_copy_lastau, k_copy_lastau)

void launch_sched(cudaStream_t s, const Inst *tab, int count, unsigned long long *launches) {
	launch_pdl(k_sched, (count + 127) / 128, 128, 0, s, tab, count, launches);
}

void launch_cond(cudaStream_t s, const Inst *tab, int count, int pred, int *flag, unsigned long long handle,
                 unsigned long long *launches) {
	launch_pdl(k_cond, 1, 128, 0, s, tab, count, pred, flag, handle, launches);
}

static int grid_for(long long n) {
	long long g = (n + 255) / 256;
	if (g > 148 * 16) g = 148 * 16;
	return (int)(g < 1 ? 1 : g);
}

static PlainGeo plain(int dims, int p, int q, int r) {
	PlainGeo g{dims, p, q, dims == 3 ? r : 1, {}, {}};
	g.fq.init((unsigned)q);
	g.fp.init((unsigned)p);
	return g;
}

void launch_D_plain(cudaStream_t s, int dims, int p, int q, int r, const real *U, real *Ux, real *Uy,
                    real *Uz) {
	PlainGeo g = plain(dims, p, q, r);
	k_D_plain<<<grid_for((long long)p * q * g.r), 256, 0, s>>>(g, U, Ux, Uy, Uz);
	TG_CUDA(cudaGetLastError());
}

void launch_Dt_plain(cudaStream_t s, int dims, int p, int q, int r, const real *X, const real *Y,
                     const real *Z, real *res) {
	PlainGeo g = plain(dims, p, q, r);
	k_Dt_plain<<<grid_for((long long)p * q * g.r), 256, 0, s>>>(g, X, Y, Z, res);
	TG_CUDA(cudaGetLastError());
}

void launch_shrink_plain(cudaStream_t s, int dims, long long n, int tv_norm, double beta, const real *Ux,
                         const real *Uy, const real *Uz, const real *sx, const real *sy, const real *sz,
                         real *Wx, real *Wy, real *Wz, double *lam1_dev) {
	k_shrink_plain<<<grid_for(n), 256, 0, s>>>(dims, n, tv_norm, beta, Ux, Uy, Uz, sx, sy, sz, Wx, Wy, Wz,
	                                           lam1_dev);
	TG_CUDA(cudaGetLastError());
}

TG_END
