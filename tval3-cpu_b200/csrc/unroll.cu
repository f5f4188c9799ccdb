// Differentiable unrolled TVAL3 (2D): K inner iterations of the solve with
// per-iteration (mu_k, beta_k), gradients of <gU, U_K / scl> with respect to
// b, mu_k and beta_k by a hand-written adjoint.
//
// Forward.  A plan in schedule mode runs the real solve for exactly K inner
// iterations (tol = 0, no A^T skipping) and records, per instance and
// iteration, the step actually taken (tau times the Armijo backtracking
// factor, or the restart's tau; 2d/tval3_cpu_2d.cpp:425-453,526-576) and
// whether the multipliers were updated after it (2d:673-694,820-842).  These
// decisions are then held fixed: the differentiated function F is the
// iteration map with them as constants (with bs = scl b; iteration 0 uses
// (mu_1, beta_1)):
//
//   U_0 = A^T bs;  sigma_0 = 0;  delta_0 = 0
//   iteration k >= 1:  U_k = U_{k-1} - step_k d_{k-1}
//   state(k): V = D U_k, Z = V - sigma_{k-1} / beta_k, W = S(Z, 1/beta_k),
//             E = V - W, r = A U_k - bs,
//             if outer_k: sigma_k = sigma_{k-1} - beta_k E, delta_k = delta_{k-1} - mu_k r
//             d_k = D^T (E - sigma_k / beta_k) + A^T ((mu_k r - delta_k) / beta_k)
//
// F is replayed on the device in FP32 (the projector, stencil and shrinkage
// kernels), with a checkpoint of (U, sigma, delta, d) every `ckpt`
// iterations; its U_K / scl is the forward output.
//
// Backward.  Segment by segment from the last, the states of the segment are
// recomputed from its checkpoint and the adjoint runs back through them:
// per iteration one forward and one adjoint projector application, D and D^T,
// the shrinkage's Jacobian-transpose, and FP64 inner products (block partials
// summed in a fixed order) for the mu_k and beta_k gradients.
#include <algorithm>
#include <cstring>
#include <vector>

#include "plan.cuh"

namespace tval3g {
namespace {

constexpr int EW_BLOCKS = 296;   // grid-stride elementwise kernels: 2 blocks per SM
constexpr int EW_THREADS = 256;
constexpr int NPIX = 4, NMEAS = 3;   // inner products per reverse step

__device__ __forceinline__ void shrink2(float zx, float zy, float t, bool iso, float &wx, float &wy) {
	if (iso) {
		const float nrm = sqrtf(zx * zx + zy * zy);
		const float s = nrm > t ? (nrm - t) / nrm : 0.f;
		wx = s * zx;
		wy = s * zy;
	} else {
		const float ax = fabsf(zx) - t, ay = fabsf(zy) - t;
		wx = ax > 0.f ? (zx >= 0.f ? ax : -ax) : 0.f;
		wy = ay > 0.f ? (zy >= 0.f ? ay : -ay) : 0.f;
	}
}

// Z-cotangent and the t-derivative term of W = S(Z, t) for the W-cotangent (wbx, wby)
__device__ __forceinline__ void shrink2_vjp(float zx, float zy, float t, bool iso, float wbx, float wby,
                                            float &zbx, float &zby, double &tbar) {
	if (iso) {
		const float nrm = sqrtf(zx * zx + zy * zy);
		if (nrm > t) {
			const float zw = (zx * wbx + zy * wby) / nrm;
			const float a = 1.f - t / nrm, c = t / (nrm * nrm);
			zbx = a * wbx + c * zx * zw;
			zby = a * wby + c * zy * zw;
			tbar += -(double)zw;
		} else {
			zbx = zby = 0.f;
		}
	} else {
		const bool onx = fabsf(zx) > t, ony = fabsf(zy) > t;
		zbx = onx ? wbx : 0.f;
		zby = ony ? wby : 0.f;
		if (onx) tbar += (zx >= 0.f ? -1.0 : 1.0) * wbx;
		if (ony) tbar += (zy >= 0.f ? -1.0 : 1.0) * wby;
	}
}

template <int NS>
__device__ __forceinline__ void block_partials(double (&v)[NS], double *part) {
	__shared__ double sh[NS][EW_THREADS / 32];
	const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
	for (int s = 0; s < NS; s++) {
		double t = warp_sum(v[s]);
		if (lane == 0) sh[s][w] = t;
	}
	__syncthreads();
	if (threadIdx.x < NS) {
		double t = 0;
		for (int k = 0; k < EW_THREADS / 32; k++) t += sh[threadIdx.x][k];
		part[blockIdx.x * NS + threadIdx.x] = t;
	}
}

// y += a x
__global__ void k_axpy(long long n, float a, const float *x, float *y) {
	for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
		y[i] = fmaf(a, x[i], y[i]);
}
// y = a x
__global__ void k_scale(long long n, float a, const float *x, float *y) {
	for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
		y[i] = a * x[i];
}
// out = x + y
__global__ void k_add(long long n, const float *x, const float *y, float *out) {
	for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
		out[i] = x[i] + y[i];
}

// forward state, pixels: shrinkage, multiplier update of sigma, G = E - sigma_k / beta
__global__ void k_state_pix(long long n, const float *vx, const float *vy, float *sx, float *sy, float beta,
                            int outer, int iso, float *gx, float *gy) {
	const float t = 1.f / beta;
	for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
		const float Vx = vx[i], Vy = vy[i];
		float s_x = sx[i], s_y = sy[i];
		float wx, wy;
		shrink2(Vx - s_x / beta, Vy - s_y / beta, t, iso, wx, wy);
		const float ex = Vx - wx, ey = Vy - wy;
		if (outer) {
			s_x = fmaf(-beta, ex, s_x);
			s_y = fmaf(-beta, ey, s_y);
			sx[i] = s_x;
			sy[i] = s_y;
		}
		gx[i] = ex - s_x / beta;
		gy[i] = ey - s_y / beta;
	}
}

// forward state, measurements: r = Au - bs, multiplier update of delta, q = (mu r - delta) / beta
__global__ void k_state_meas(long long m, const float *au, const float *bs, float *r, float *dl, float mu,
                             float beta, int outer, float *q) {
	for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < m; i += (long long)gridDim.x * blockDim.x) {
		const float rr = au[i] - bs[i];
		float d = dl[i];
		if (outer) {
			d = fmaf(-mu, rr, d);
			dl[i] = d;
		}
		r[i] = rr;
		q[i] = (mu * rr - d) / beta;
	}
}

// reverse step, pixels (see the file comment); partials: <Dd, sigma_k>,
// <sigma_k-bar, E>, sum of the shrinkage's t-derivative term, <Zbar, sigma_{k-1}>
__global__ void __launch_bounds__(EW_THREADS) k_rev_pix(long long n, const float *ddx, const float *ddy,
                                                        const float *vx, const float *vy, const float *s0x,
                                                        const float *s0y, const float *s1x, const float *s1y,
                                                        float *sbx, float *sby, float beta, int outer, int iso,
                                                        float *vbx, float *vby, double *part) {
	const float t = 1.f / beta;
	double acc[NPIX] = {0, 0, 0, 0};
	for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
		const float zx = vx[i] - s0x[i] / beta, zy = vy[i] - s0y[i] / beta;
		float wx, wy;
		shrink2(zx, zy, t, iso, wx, wy);
		const float ex = vx[i] - wx, ey = vy[i] - wy;
		const float dx = ddx ? ddx[i] : 0.f, dy = ddy ? ddy[i] : 0.f;
		float sx = sbx[i] - dx / beta, sy = sby[i] - dy / beta;   // cotangent of sigma_k
		float ebx = dx, eby = dy;
		acc[0] += (double)dx * s1x[i] + (double)dy * s1y[i];
		if (outer) {
			ebx = fmaf(-beta, sx, ebx);
			eby = fmaf(-beta, sy, eby);
			acc[1] += (double)sx * ex + (double)sy * ey;
		}
		float zbx, zby;
		shrink2_vjp(zx, zy, t, iso, -ebx, -eby, zbx, zby, acc[2]);
		acc[3] += (double)zbx * s0x[i] + (double)zby * s0y[i];
		vbx[i] = ebx + zbx;
		vby[i] = eby + zby;
		sbx[i] = sx - zbx / beta;   // cotangent of sigma_{k-1}
		sby[i] = sy - zby / beta;
	}
	block_partials<NPIX>(acc, part);
}

// reverse step, measurements; partials: <Ad, r>, <Ad, delta - mu r>, <delta_k-bar, r>
__global__ void __launch_bounds__(EW_THREADS) k_rev_meas(long long m, const float *ad, const float *r, const float *dl,
                                                         float *dlb, float *bsb, float mu, float beta, int outer,
                                                         float *rb, double *part) {
	double acc[NMEAS] = {0, 0, 0};
	for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < m; i += (long long)gridDim.x * blockDim.x) {
		const float a = ad ? ad[i] : 0.f, rr = r[i];
		const float db = dlb[i] - a / beta;   // cotangent of delta_k
		float rbv = (mu / beta) * a;
		acc[0] += (double)a * rr;
		acc[1] += (double)a * (dl[i] - mu * rr);
		if (outer) {
			rbv = fmaf(-mu, db, rbv);
			acc[2] += (double)db * rr;
		}
		dlb[i] = db;
		rb[i] = rbv;
		bsb[i] -= rbv;
	}
	block_partials<NMEAS>(acc, part);
}

// Ubar += t1 + t2; dd = -step Ubar
__global__ void k_rev_u(long long n, const float *t1, const float *t2, float *ub, float nstep, float *dd) {
	for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
		const float u = ub[i] + t1[i] + t2[i];
		ub[i] = u;
		if (dd) dd[i] = nstep * u;
	}
}

// the mu_j and beta_j gradient terms of one reverse step, summed in block order
__global__ void k_rev_scalars(const double *pp, const double *pm, int nb, double mu, double beta, double *gmu,
                              double *gbeta) {
	if (threadIdx.x != 0 || blockIdx.x != 0) return;
	double P[NPIX] = {0, 0, 0, 0}, M[NMEAS] = {0, 0, 0};
	for (int b = 0; b < nb; b++) {
		for (int s = 0; s < NPIX; s++) P[s] += pp[b * NPIX + s];
		for (int s = 0; s < NMEAS; s++) M[s] += pm[b * NMEAS + s];
	}
	const double b2 = beta * beta;
	*gmu += M[0] / beta - M[2];
	*gbeta += P[0] / b2 + M[1] / b2 - P[1] - P[2] / b2 + P[3] / b2;
}

}  // namespace

// one instance's device buffers for the replay and the adjoint
struct UnrolledInst {
	std::vector<double> steps;
	std::vector<int> outer;
	double scl = 1;
	float *bs = nullptr;   // scl * b
};

class Unrolled {
public:
	Unrolled(const tval3g_problem &p, int count, const tval3g_options &o, int K, int ckpt);
	~Unrolled();
	void forward(const float *const *d_b, const double *mu, const double *beta, float *const *d_U, cudaStream_t s);
	void backward(const float *const *d_gU, float *const *d_gb, double *g_mu, double *g_beta, cudaStream_t s);
	const UnrolledInst &inst(int i) const { return in_[i]; }
	int count() const { return count_; }
	int K() const { return K_; }

private:
	int count_, K_, C_, p_, q_, iso_;
	long long n_, m_;
	Plan *plan_ = nullptr;
	tval3g_operator *op_ = nullptr;
	// used when the caller passes the legacy default stream: blocking, so it
	// is ordered with that stream's work on both sides, and every launch
	// here (and the operator's) goes to one stream
	cudaStream_t own_ = nullptr;
	std::vector<UnrolledInst> in_;
	std::vector<double> mu_, beta_;
	std::vector<float *> eng_u_;       // the engine's U (decisions only)
	std::vector<void *> allocs_;
	// checkpoints: [instance][c] -> U, sx, sy, delta, d
	std::vector<std::vector<float *>> ck_;
	// segment states, j = 0..C: U, sx, sy, delta, r
	std::vector<float *> segU_, segSx_, segSy_, segDl_, segR_;
	// scratch
	float *vx_, *vy_, *gx_, *gy_, *t1_, *t2_, *d_, *U_, *sx_, *sy_, *au_, *qv_, *dl_, *r_;
	float *ub_, *sbx_, *sby_, *dlb_, *bsb_, *dd_, *ddx_, *ddy_, *ad_, *rb_, *vbx_, *vby_;
	double *pp_, *pm_, *gsc_;   // partials, gradient scalars (2K)
	float *fa(long long count);
	void release();
	void apply(bool trans, const float *x, float *y, cudaStream_t s);
	void state(int k, const float *bs, float *U, float *sx, float *sy, float *dl, float *r, float *d, int o,
	           cudaStream_t s);
	void replay_from(int i, int k0, int k1, cudaStream_t s, bool store_seg, bool ckpt);
};

float *Unrolled::fa(long long count) {
	void *p = nullptr;
	TG_CUDA(cudaMalloc(&p, sizeof(float) * (size_t)std::max(count, 1LL)));
	allocs_.push_back(p);
	return static_cast<float *>(p);
}

Unrolled::Unrolled(const tval3g_problem &p, int count, const tval3g_options &o, int K, int ckpt)
	: count_(count), K_(K), C_(ckpt) {
	TG_ARG(count >= 1 && K >= 1 && ckpt >= 1, "Argument error: count, K and the checkpoint interval must be >= 1");
	TG_ARG(p.dims == 2 && (p.op_kind == TVAL3G_OP_RAY2D || p.op_kind == TVAL3G_OP_CSR ||
	                       (p.op_kind == TVAL3G_OP_DENSE && p.layers <= 1)),
	       "Argument error: the unrolled solve is 2D with one layer");
	TG_ARG(!o.nonneg, "Argument error: the unrolled solve has no nonnegativity projection");
	p_ = p.dim_y;
	q_ = p.dim_x;
	iso_ = o.tv_norm != 0;
	tval3g_options oo = o;
	oo.maxit = K;
	oo.tol = 0;                 // exactly K inner iterations
	oo.maxcnt = 1 << 30;
	oo.skipMulRatio = 0;        // g = A^T (A U - b) every iteration
	std::vector<tval3g_problem> probs(count, p);
	std::vector<tval3g_options> opts(count, oo);
	try {
		TG_CUDA(cudaStreamCreate(&own_));
		plan_ = new Plan(count, probs.data(), opts.data(), TVAL3G_GRAPH | TVAL3G_TRACE | PLAN_SCHEDULE);
		int rc = tval3g_op_create(&op_, &p, 0);
		if (rc != TVAL3G_OK) throw Error{rc, tval3g_last_error()};
		long long rows = 0, cols = 0, nnz = 0;
		tval3g_op_shape(op_, &rows, &cols, &nnz);
		m_ = rows;
		n_ = cols;
		in_.resize(count);
		for (int i = 0; i < count; i++) {
			in_[i].bs = fa(m_);
			eng_u_.push_back(fa(n_));
		}
		const int nck = K / C_ + 1;
		ck_.resize(count);
		for (int i = 0; i < count; i++)
			for (int c = 0; c < nck; c++)
				for (int v = 0; v < 5; v++) ck_[i].push_back(fa(v == 3 ? m_ : n_));
		for (int j = 0; j <= C_; j++) {
			segU_.push_back(fa(n_));
			segSx_.push_back(fa(n_));
			segSy_.push_back(fa(n_));
			segDl_.push_back(fa(m_));
			segR_.push_back(fa(m_));
		}
		for (float **v : {&vx_, &vy_, &gx_, &gy_, &t1_, &t2_, &d_, &U_, &sx_, &sy_, &ub_, &sbx_, &sby_, &dd_, &ddx_,
		                  &ddy_, &vbx_, &vby_})
			*v = fa(n_);
		for (float **v : {&au_, &qv_, &dl_, &r_, &dlb_, &bsb_, &ad_, &rb_}) *v = fa(m_);
		void *pp = nullptr;
		TG_CUDA(cudaMalloc(&pp, sizeof(double) * (size_t)(EW_BLOCKS * (NPIX + NMEAS) + 2 * K)));
		allocs_.push_back(pp);
		pp_ = static_cast<double *>(pp);
		pm_ = pp_ + EW_BLOCKS * NPIX;
		gsc_ = pm_ + EW_BLOCKS * NMEAS;
	} catch (...) {
		release();
		throw;
	}
}

Unrolled::~Unrolled() { release(); }

void Unrolled::release() {
	cudaDeviceSynchronize();
	for (void *p : allocs_) cudaFree(p);
	allocs_.clear();
	if (op_) tval3g_op_destroy(op_);
	op_ = nullptr;
	delete plan_;
	plan_ = nullptr;
	if (own_) cudaStreamDestroy(own_);
	own_ = nullptr;
}

void Unrolled::apply(bool trans, const float *x, float *y, cudaStream_t s) {
	int rc = tval3g_op_apply_n(op_, trans ? 1 : 0, x, y, 1, s);
	if (rc != TVAL3G_OK) throw Error{rc, tval3g_last_error()};
}

#define EW(kern, ...)                                                     \
	do {                                                                  \
		kern<<<EW_BLOCKS, EW_THREADS, 0, s>>>(__VA_ARGS__);               \
		TG_CUDA(cudaGetLastError());                                      \
	} while (0)

// state(k) from U (in place: sigma, delta updated when o); d written
void Unrolled::state(int k, const float *bs, float *U, float *sx, float *sy, float *dl, float *r, float *d, int o,
                     cudaStream_t s) {
	const int j = std::max(k, 1) - 1;
	const float mu = (float)mu_[j], beta = (float)beta_[j];
	launch_D_plain(s, 2, p_, q_, 1, U, vx_, vy_, nullptr);
	EW(k_state_pix, n_, vx_, vy_, sx, sy, beta, o, iso_, gx_, gy_);
	apply(false, U, au_, s);
	EW(k_state_meas, m_, au_, bs, r, dl, mu, beta, o, qv_);
	apply(true, qv_, t1_, s);
	launch_Dt_plain(s, 2, p_, q_, 1, gx_, gy_, nullptr, t2_);
	EW(k_add, n_, t1_, t2_, d);
}

// replay iterations k0 + 1 .. k1 of instance i from the working state (U_,
// sx_, sy_, dl_, d_ = iteration k0); store_seg: keep every state (j = k - k0)
void Unrolled::replay_from(int i, int k0, int k1, cudaStream_t s, bool store_seg, bool ckpt) {
	const UnrolledInst &I = in_[i];
	const size_t nb = sizeof(float) * (size_t)n_, mb = sizeof(float) * (size_t)m_;
	auto save_seg = [&](int j) {
		TG_CUDA(cudaMemcpyAsync(segU_[j], U_, nb, cudaMemcpyDeviceToDevice, s));
		TG_CUDA(cudaMemcpyAsync(segSx_[j], sx_, nb, cudaMemcpyDeviceToDevice, s));
		TG_CUDA(cudaMemcpyAsync(segSy_[j], sy_, nb, cudaMemcpyDeviceToDevice, s));
		TG_CUDA(cudaMemcpyAsync(segDl_[j], dl_, mb, cudaMemcpyDeviceToDevice, s));
		TG_CUDA(cudaMemcpyAsync(segR_[j], r_, mb, cudaMemcpyDeviceToDevice, s));
	};
	auto save_ck = [&](int k) {
		float *const *c = &ck_[i][(size_t)(k / C_) * 5];
		TG_CUDA(cudaMemcpyAsync(c[0], U_, nb, cudaMemcpyDeviceToDevice, s));
		TG_CUDA(cudaMemcpyAsync(c[1], sx_, nb, cudaMemcpyDeviceToDevice, s));
		TG_CUDA(cudaMemcpyAsync(c[2], sy_, nb, cudaMemcpyDeviceToDevice, s));
		TG_CUDA(cudaMemcpyAsync(c[3], dl_, mb, cudaMemcpyDeviceToDevice, s));
		TG_CUDA(cudaMemcpyAsync(c[4], d_, nb, cudaMemcpyDeviceToDevice, s));
	};
	if (store_seg) save_seg(0);
	if (ckpt && k0 % C_ == 0) save_ck(k0);
	for (int k = k0 + 1; k <= k1; k++) {
		EW(k_axpy, n_, (float)(-I.steps[k - 1]), d_, U_);
		state(k, I.bs, U_, sx_, sy_, dl_, r_, d_, I.outer[k - 1], s);
		if (store_seg) save_seg(k - k0);
		if (ckpt && k % C_ == 0) save_ck(k);
	}
}

void Unrolled::forward(const float *const *d_b, const double *mu, const double *beta, float *const *d_U,
                       cudaStream_t s) {
	if (!s) s = own_;
	mu_.assign(mu, mu + K_);
	beta_.assign(beta, beta + K_);
	// the solve that records the decisions
	plan_->set_schedule(mu, beta);
	std::vector<tval3g_info> info(count_);
	plan_->solve(d_b, nullptr, eng_u_.data(), info.data(), s);
	const std::vector<Ctrl> c = plan_->ctrl();
	std::vector<tval3g_trace_record> tr(K_);
	for (int i = 0; i < count_; i++) {
		TG_ARG(info[i].status == TVAL3G_OK, "Argument error: the forward solve stopped on a non-finite value");
		const int got = plan_->trace(i, tr.data(), K_);
		TG_ARG(got == K_, "Internal error: the forward solve did not run K iterations");
		UnrolledInst &I = in_[i];
		I.steps.resize(K_);
		I.outer.resize(K_);
		for (int k = 0; k < K_; k++) {
			I.steps[k] = tr[k].step;
			I.outer[k] = tr[k].outer != 0;
		}
		I.scl = c[i].scl;
	}
	// replay F with checkpoints
	for (int i = 0; i < count_; i++) {
		UnrolledInst &I = in_[i];
		EW(k_scale, m_, (float)I.scl, d_b[i], I.bs);
		apply(true, I.bs, U_, s);
		TG_CUDA(cudaMemsetAsync(sx_, 0, sizeof(float) * (size_t)n_, s));
		TG_CUDA(cudaMemsetAsync(sy_, 0, sizeof(float) * (size_t)n_, s));
		TG_CUDA(cudaMemsetAsync(dl_, 0, sizeof(float) * (size_t)m_, s));
		state(0, I.bs, U_, sx_, sy_, dl_, r_, d_, 0, s);
		replay_from(i, 0, K_, s, false, true);
		EW(k_scale, n_, (float)(1.0 / I.scl), U_, d_U[i]);
	}
	TG_CUDA(cudaStreamSynchronize(s));
}

void Unrolled::backward(const float *const *d_gU, float *const *d_gb, double *g_mu, double *g_beta, cudaStream_t s) {
	TG_ARG(!mu_.empty(), "Argument error: backward before forward");
	if (!s) s = own_;
	TG_CUDA(cudaMemsetAsync(gsc_, 0, sizeof(double) * 2 * (size_t)K_, s));
	const size_t nb = sizeof(float) * (size_t)n_, mb = sizeof(float) * (size_t)m_;
	for (int i = 0; i < count_; i++) {
		const UnrolledInst &I = in_[i];
		EW(k_scale, n_, (float)(1.0 / I.scl), d_gU[i], ub_);
		for (float *v : {sbx_, sby_}) TG_CUDA(cudaMemsetAsync(v, 0, nb, s));
		for (float *v : {dlb_, bsb_}) TG_CUDA(cudaMemsetAsync(v, 0, mb, s));
		bool has_d = false;
		for (int c = K_ / C_; c >= 0; c--) {
			const int k0 = c * C_, k1 = std::min(k0 + C_, K_);
			if (k0 > K_ || (k0 == K_ && K_ > 0 && c > 0 && k1 == k0)) continue;
			// the checkpoint state of iteration k0, r of iteration k0, then the segment
			float *const *ck = &ck_[i][(size_t)c * 5];
			TG_CUDA(cudaMemcpyAsync(U_, ck[0], nb, cudaMemcpyDeviceToDevice, s));
			TG_CUDA(cudaMemcpyAsync(sx_, ck[1], nb, cudaMemcpyDeviceToDevice, s));
			TG_CUDA(cudaMemcpyAsync(sy_, ck[2], nb, cudaMemcpyDeviceToDevice, s));
			TG_CUDA(cudaMemcpyAsync(dl_, ck[3], mb, cudaMemcpyDeviceToDevice, s));
			TG_CUDA(cudaMemcpyAsync(d_, ck[4], nb, cudaMemcpyDeviceToDevice, s));
			apply(false, U_, au_, s);
			EW(k_state_meas, m_, au_, I.bs, r_, dl_, 1.f, 1.f, 0, qv_);   // r only (q unused)
			replay_from(i, k0, k1, s, true, false);
			const int klo = c == 0 ? 0 : k0 + 1;
			for (int k = k1; k >= klo; k--) {
				const int jj = k - k0, j = std::max(k, 1) - 1;
				const float mu = (float)mu_[j], beta = (float)beta_[j];
				const int o = k >= 1 ? I.outer[k - 1] : 0;
				const float *s0x = k >= 1 ? segSx_[jj - 1] : nullptr, *s0y = k >= 1 ? segSy_[jj - 1] : nullptr;
				if (k == 0) {   // sigma_{-1} = 0
					TG_CUDA(cudaMemsetAsync(gx_, 0, nb, s));
					TG_CUDA(cudaMemsetAsync(gy_, 0, nb, s));
					s0x = gx_;
					s0y = gy_;
				}
				if (has_d) {
					launch_D_plain(s, 2, p_, q_, 1, dd_, ddx_, ddy_, nullptr);
					apply(false, dd_, ad_, s);
				}
				launch_D_plain(s, 2, p_, q_, 1, segU_[jj], vx_, vy_, nullptr);
				EW(k_rev_pix, n_, has_d ? ddx_ : nullptr, has_d ? ddy_ : nullptr, vx_, vy_, s0x, s0y, segSx_[jj],
				   segSy_[jj], sbx_, sby_, beta, o, iso_, vbx_, vby_, pp_);
				EW(k_rev_meas, m_, has_d ? ad_ : nullptr, segR_[jj], segDl_[jj], dlb_, bsb_, mu, beta, o, rb_, pm_);
				k_rev_scalars<<<1, 32, 0, s>>>(pp_, pm_, EW_BLOCKS, mu_[j], beta_[j], gsc_ + j, gsc_ + K_ + j);
				TG_CUDA(cudaGetLastError());
				apply(true, rb_, t1_, s);
				launch_Dt_plain(s, 2, p_, q_, 1, vbx_, vby_, nullptr, t2_);
				EW(k_rev_u, n_, t1_, t2_, ub_, k >= 1 ? (float)(-I.steps[k - 1]) : 0.f, k >= 1 ? dd_ : nullptr);
				has_d = k >= 1;
			}
		}
		// U_0 = A^T bs: bsbar += A Ubar; gb = scl bsbar
		apply(false, ub_, au_, s);
		EW(k_add, m_, bsb_, au_, bsb_);
		EW(k_scale, m_, (float)I.scl, bsb_, d_gb[i]);
	}
	std::vector<double> h(2 * (size_t)K_);
	TG_CUDA(cudaMemcpyAsync(h.data(), gsc_, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, s));
	TG_CUDA(cudaStreamSynchronize(s));
	for (int k = 0; k < K_; k++) {
		g_mu[k] = h[k];
		g_beta[k] = h[K_ + k];
	}
}

}  // namespace tval3g

using namespace tval3g;

struct tval3g_unrolled {
	Unrolled *u;
};

#define UNR_BEGIN try {
#define UNR_END                                                      \
	}                                                                \
	catch (const Error &e) {                                         \
		set_error(e.msg);                                            \
		return e.code;                                               \
	}                                                                \
	catch (const std::exception &e) {                                \
		set_error(std::string("Internal error: ") + e.what());       \
		return TVAL3G_ERR_INTERNAL;                                  \
	}                                                                \
	return TVAL3G_OK;

extern "C" int tval3g_unrolled_create(tval3g_unrolled **h, const tval3g_problem *prob, int count,
                                      const tval3g_options *opts, int K, int ckpt) {
	UNR_BEGIN
	TG_ARG(h && prob && opts, "Argument error: NULL argument");
	*h = nullptr;
	auto *u = new tval3g_unrolled{nullptr};
	try {
		u->u = new Unrolled(*prob, count, *opts, K, ckpt);
	} catch (...) {
		delete u;
		throw;
	}
	*h = u;
	UNR_END
}

extern "C" int tval3g_unrolled_forward(tval3g_unrolled *h, const float *const *d_b, const double *mu,
                                       const double *beta, float *const *d_U, void *stream) {
	UNR_BEGIN
	TG_ARG(h && h->u && d_b && mu && beta && d_U, "Argument error: NULL argument");
	h->u->forward(d_b, mu, beta, d_U, (cudaStream_t)stream);
	UNR_END
}

extern "C" int tval3g_unrolled_backward(tval3g_unrolled *h, const float *const *d_gU, float *const *d_gb,
                                        double *g_mu, double *g_beta, void *stream) {
	UNR_BEGIN
	TG_ARG(h && h->u && d_gU && d_gb && g_mu && g_beta, "Argument error: NULL argument");
	h->u->backward(d_gU, d_gb, g_mu, g_beta, (cudaStream_t)stream);
	UNR_END
}

extern "C" int tval3g_unrolled_decisions(const tval3g_unrolled *h, int index, double *steps, int *outer,
                                         double *scl) {
	UNR_BEGIN
	TG_ARG(h && h->u && steps && outer && scl, "Argument error: NULL argument");
	TG_ARG(index >= 0 && index < h->u->count(), "Argument error: index out of range");
	const UnrolledInst &I = h->u->inst(index);
	TG_ARG(!I.steps.empty(), "Argument error: decisions before forward");
	for (int k = 0; k < h->u->K(); k++) {
		steps[k] = I.steps[k];
		outer[k] = I.outer[k];
	}
	*scl = I.scl;
	UNR_END
}

extern "C" int tval3g_unrolled_destroy(tval3g_unrolled *h) {
	UNR_BEGIN
	if (h) {
		delete h->u;
		delete h;
	}
	UNR_END
}
