// Differentiable unrolled TVAL3 (2D): K inner iterations of the solve with
// per-iteration (mu_k, beta_k), gradients of <gU, U_K / scl> with respect to
// b, mu_k and beta_k by a hand-written adjoint.
//
// Forward.  A plan in schedule mode runs the real FP32 solve for exactly K
// inner iterations (tol = 0, no A^T skipping) and records, per instance and
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
// F is replayed on the device in FP64, with a checkpoint of (U, sigma,
// delta, d) every `ckpt` iterations; its U_K / scl is the forward output.
// FP64, because F is only piecewise smooth (the shrinkage switches pixels on
// and off at |Z| = 1/beta): rounding the trajectory's states to FP32 moves
// the exact gradient by up to 8e-4 relative at 128x128 with K = 50 (measured
// on the FP64 restatement), far above the FP32 forward's 2e-6.
//
// Backward.  Segment by segment from the last, the states of the segment are
// recomputed from its checkpoint and the adjoint runs back through them:
// per iteration one forward and one adjoint projector application (FP64
// gathers over the operator's CSR and its device-built CSC; for ray
// operators the traced Bresenham lists), D and D^T, the shrinkage's
// Jacobian-transpose, and FP64 inner products (block partials summed in a
// fixed order) for the mu_k and beta_k gradients.
#include <algorithm>
#include <cstring>
#include <vector>

#include "plan.cuh"

TG_BEGIN
namespace {

constexpr int EW_BLOCKS = 296;   // grid-stride elementwise kernels: 2 blocks per SM
constexpr int EW_THREADS = 256;
constexpr int NPIX = 4, NMEAS = 3;   // inner products per reverse step

#define GRID_STRIDE(i, n) \
	for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < (n); i += (long long)gridDim.x * blockDim.x)

__device__ __forceinline__ void shrink2(double zx, double zy, double t, bool iso, double &wx, double &wy) {
	if (iso) {
		const double nrm = sqrt(zx * zx + zy * zy);
		const double s = nrm > t ? (nrm - t) / nrm : 0.0;
		wx = s * zx;
		wy = s * zy;
	} else {
		const double ax = fabs(zx) - t, ay = fabs(zy) - t;
		wx = ax > 0.0 ? (zx >= 0.0 ? ax : -ax) : 0.0;
		wy = ay > 0.0 ? (zy >= 0.0 ? ay : -ay) : 0.0;
	}
}

// Z-cotangent and the t-derivative term of W = S(Z, t) for the W-cotangent (wbx, wby)
__device__ __forceinline__ void shrink2_vjp(double zx, double zy, double t, bool iso, double wbx, double wby,
                                            double &zbx, double &zby, double &tbar) {
	if (iso) {
		const double nrm = sqrt(zx * zx + zy * zy);
		if (nrm > t) {
			const double zw = (zx * wbx + zy * wby) / nrm;
			const double a = 1.0 - t / nrm, c = t / (nrm * nrm);
			zbx = a * wbx + c * zx * zw;
			zby = a * wby + c * zy * zw;
			tbar += -zw;
		} else {
			zbx = zby = 0.0;
		}
	} else {
		const bool onx = fabs(zx) > t, ony = fabs(zy) > t;
		zbx = onx ? wbx : 0.0;
		zby = ony ? wby : 0.0;
		if (onx) tbar += (zx >= 0.0 ? -1.0 : 1.0) * wbx;
		if (ony) tbar += (zy >= 0.0 ? -1.0 : 1.0) * wby;
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

// y = A x over a CSR (rows of `ptr`), warp per row, FP64; val NULL = every
// weight w (ray operators: the scale factor)
__global__ void __launch_bounds__(256) k_spmv64(long long rows, const int *ptr, const int *ind, const float *val,
                                                double w, const double *x, double *y) {
	const long long row = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	const int lane = threadIdx.x & 31;
	if (row >= rows) return;
	double acc = 0.0;
	for (int k = ptr[row] + lane; k < ptr[row + 1]; k += 32) acc += (val ? (double)val[k] : w) * x[ind[k]];
	acc = warp_sum(acc);
	if (lane == 0) y[row] = acc;
}

// periodic forward differences / their adjoint on a p x q image (2d:268-293)
__global__ void k_D64(int p, int q, const double *U, double *ux, double *uy) {
	GRID_STRIDE(i, (long long)p * q) {
		const int y = (int)(i / q), x = (int)(i - (long long)y * q);
		ux[i] = (x < q - 1 ? U[i + 1] : U[i - (q - 1)]) - U[i];
		uy[i] = (y < p - 1 ? U[i + q] : U[i - (long long)(p - 1) * q]) - U[i];
	}
}
__global__ void k_Dt64(int p, int q, const double *X, const double *Y, double *res) {
	GRID_STRIDE(i, (long long)p * q) {
		const int y = (int)(i / q), x = (int)(i - (long long)y * q);
		res[i] = ((x > 0 ? X[i - 1] : X[i + q - 1]) - X[i]) +
		         ((y > 0 ? Y[i - q] : Y[i + (long long)(p - 1) * q]) - Y[i]);
	}
}

__global__ void k_axpy(long long n, double a, const double *x, double *y) {
	GRID_STRIDE(i, n) y[i] = fma(a, x[i], y[i]);
}
__global__ void k_add(long long n, const double *x, const double *y, double *out) {
	GRID_STRIDE(i, n) out[i] = x[i] + y[i];
}
__global__ void k_to64(long long n, double a, const float *x, double *y) {
	GRID_STRIDE(i, n) y[i] = a * (double)x[i];
}
__global__ void k_to32(long long n, double a, const double *x, float *y) {
	GRID_STRIDE(i, n) y[i] = (float)(a * x[i]);
}

// forward state, pixels: shrinkage, multiplier update of sigma, G = E - sigma_k / beta
__global__ void k_state_pix(long long n, const double *vx, const double *vy, double *sx, double *sy, double beta,
                            int outer, int iso, double *gx, double *gy) {
	const double t = 1.0 / beta;
	GRID_STRIDE(i, n) {
		const double Vx = vx[i], Vy = vy[i];
		double s_x = sx[i], s_y = sy[i], wx, wy;
		shrink2(Vx - s_x / beta, Vy - s_y / beta, t, iso, wx, wy);
		const double ex = Vx - wx, ey = Vy - wy;
		if (outer) {
			s_x -= beta * ex;
			s_y -= beta * ey;
			sx[i] = s_x;
			sy[i] = s_y;
		}
		gx[i] = ex - s_x / beta;
		gy[i] = ey - s_y / beta;
	}
}

// forward state, measurements: r = Au - bs, multiplier update of delta, q = (mu r - delta) / beta
__global__ void k_state_meas(long long m, const double *au, const double *bs, double *r, double *dl, double mu,
                             double beta, int outer, double *q) {
	GRID_STRIDE(i, m) {
		const double rr = au[i] - bs[i];
		double d = dl[i];
		if (outer) {
			d -= mu * rr;
			dl[i] = d;
		}
		r[i] = rr;
		q[i] = (mu * rr - d) / beta;
	}
}

// reverse step, pixels; partials: <Dd, sigma_k>, <sigma_k-bar, E>, the
// shrinkage's t-derivative term, <Zbar, sigma_{k-1}>
__global__ void __launch_bounds__(EW_THREADS) k_rev_pix(long long n, const double *ddx, const double *ddy,
                                                        const double *vx, const double *vy, const double *s0x,
                                                        const double *s0y, const double *s1x, const double *s1y,
                                                        double *sbx, double *sby, double beta, int outer, int iso,
                                                        double *vbx, double *vby, double *part) {
	const double t = 1.0 / beta;
	double acc[NPIX] = {0, 0, 0, 0};
	GRID_STRIDE(i, n) {
		const double zx = vx[i] - s0x[i] / beta, zy = vy[i] - s0y[i] / beta;
		double wx, wy;
		shrink2(zx, zy, t, iso, wx, wy);
		const double ex = vx[i] - wx, ey = vy[i] - wy;
		const double dx = ddx ? ddx[i] : 0.0, dy = ddy ? ddy[i] : 0.0;
		const double sx = sbx[i] - dx / beta, sy = sby[i] - dy / beta;   // cotangent of sigma_k
		double ebx = dx, eby = dy;
		acc[0] += dx * s1x[i] + dy * s1y[i];
		if (outer) {
			ebx -= beta * sx;
			eby -= beta * sy;
			acc[1] += sx * ex + sy * ey;
		}
		double zbx, zby;
		shrink2_vjp(zx, zy, t, iso, -ebx, -eby, zbx, zby, acc[2]);
		acc[3] += zbx * s0x[i] + zby * s0y[i];
		vbx[i] = ebx + zbx;
		vby[i] = eby + zby;
		sbx[i] = sx - zbx / beta;   // cotangent of sigma_{k-1}
		sby[i] = sy - zby / beta;
	}
	block_partials<NPIX>(acc, part);
}

// reverse step, measurements; partials: <Ad, r>, <Ad, delta - mu r>, <delta_k-bar, r>
__global__ void __launch_bounds__(EW_THREADS) k_rev_meas(long long m, const double *ad, const double *r,
                                                         const double *dl, double *dlb, double *bsb, double mu,
                                                         double beta, int outer, double *rb, double *part) {
	double acc[NMEAS] = {0, 0, 0};
	GRID_STRIDE(i, m) {
		const double a = ad ? ad[i] : 0.0, rr = r[i];
		const double db = dlb[i] - a / beta;   // cotangent of delta_k
		double rbv = (mu / beta) * a;
		acc[0] += a * rr;
		acc[1] += a * (dl[i] - mu * rr);
		if (outer) {
			rbv -= mu * db;
			acc[2] += db * rr;
		}
		dlb[i] = db;
		rb[i] = rbv;
		bsb[i] -= rbv;
	}
	block_partials<NMEAS>(acc, part);
}

// Ubar += t1 + t2; dd = -step Ubar
__global__ void k_rev_u(long long n, const double *t1, const double *t2, double *ub, double nstep, double *dd) {
	GRID_STRIDE(i, n) {
		const double u = ub[i] + t1[i] + t2[i];
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

struct UnrolledInst {
	std::vector<double> steps;
	std::vector<int> outer;
	double scl = 1;
	double *bs = nullptr;   // scl * b (FP64)
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
	long long n_, m_, nnz_ = 0;
	Plan *plan_ = nullptr;
	// used when the caller passes the legacy default stream: blocking, so it
	// is ordered with that stream's work on both sides
	cudaStream_t own_ = nullptr;
	// the operator as a CSR over measurements and its CSC over pixels
	int *rptr_ = nullptr, *rind_ = nullptr, *cptr_ = nullptr, *cind_ = nullptr;
	float *rval_ = nullptr, *cval_ = nullptr;
	double w_ = 1.0;
	std::vector<UnrolledInst> in_;
	std::vector<double> mu_, beta_;
	std::vector<float *> eng_u_;       // the FP32 solve's U (decisions only)
	std::vector<void *> allocs_;
	// checkpoints: [instance][c] -> U, sx, sy, delta, d
	std::vector<std::vector<double *>> ck_;
	// segment states, j = 0..C: U, sx, sy, delta, r
	std::vector<double *> segU_, segSx_, segSy_, segDl_, segR_;
	// scratch
	double *vx_, *vy_, *gx_, *gy_, *t1_, *t2_, *d_, *U_, *sx_, *sy_, *au_, *qv_, *dl_, *r_;
	double *ub_, *sbx_, *sby_, *dlb_, *bsb_, *dd_, *ddx_, *ddy_, *ad_, *rb_, *vbx_, *vby_, *zero_;
	double *pp_, *pm_, *gsc_;   // partials, gradient scalars (2K)
	void *dmalloc(size_t bytes);
	double *da(long long count) { return static_cast<double *>(dmalloc(sizeof(double) * (size_t)std::max(count, 1LL))); }
	void release();
	void apply(bool trans, const double *x, double *y, cudaStream_t s);
	void state(int k, const double *bs, double *U, double *sx, double *sy, double *dl, double *r, double *d, int o,
	           cudaStream_t s);
	void replay_from(int i, int k0, int k1, cudaStream_t s, bool store_seg, bool ckpt);
};

void *Unrolled::dmalloc(size_t bytes) {
	void *p = nullptr;
	TG_CUDA(cudaMalloc(&p, std::max(bytes, (size_t)8)));
	allocs_.push_back(p);
	return p;
}

Unrolled::Unrolled(const tval3g_problem &p, int count, const tval3g_options &o, int K, int ckpt)
	: count_(count), K_(K), C_(ckpt) {
	TG_ARG(count >= 1 && K >= 1 && ckpt >= 1, "Argument error: count, K and the checkpoint interval must be >= 1");
	TG_ARG(p.dims == 2 && (p.op_kind == TVAL3G_OP_RAY2D || p.op_kind == TVAL3G_OP_CSR ||
	                       (p.op_kind == TVAL3G_OP_DENSE && p.layers <= 1)) && p.layers <= 1,
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
	tval3g_operator *op = nullptr;
	try {
		TG_CUDA(cudaStreamCreate(&own_));
		plan_ = new Plan(count, probs.data(), opts.data(), TVAL3G_GRAPH | TVAL3G_TRACE | PLAN_SCHEDULE);
		// the operator's CSR on the host: the traced rays, the caller's CSR, or the dense rows
		std::vector<long long> hp;
		std::vector<int> hi;
		std::vector<float> hv;
		if (p.op_kind == TVAL3G_OP_RAY2D) {
			int rc = tval3g_op_create(&op, &p, 0);
			if (rc != TVAL3G_OK) throw Error{rc, tval3g_last_error()};
			long long rows = 0, cols = 0, nnz = 0;
			tval3g_op_shape(op, &rows, &cols, &nnz);
			m_ = rows;
			n_ = cols;
			hp.resize(m_ + 1);
			hi.resize(std::max(nnz, 1LL));
			rc = tval3g_op_ray_csr(op, hp.data(), hi.data());
			if (rc != TVAL3G_OK) throw Error{rc, tval3g_last_error()};
			tval3g_op_destroy(op);
			op = nullptr;
			w_ = p.scale_factor;
		} else if (p.op_kind == TVAL3G_OP_CSR) {
			m_ = p.m;
			n_ = p.n_cols;
			hp.assign(p.csr_ptr, p.csr_ptr + m_ + 1);
			hi.assign(p.csr_ind, p.csr_ind + p.nnz);
			hv.assign(p.csr_val, p.csr_val + p.nnz);
		} else {
			m_ = p.m;
			n_ = p.n_cols;
			hp.resize(m_ + 1);
			for (long long r = 0; r <= m_; r++) hp[r] = r * n_;
			hi.resize(m_ * n_);
			for (long long k = 0; k < m_ * n_; k++) hi[k] = (int)(k % n_);
			hv.assign(p.A, p.A + m_ * n_);
		}
		TG_ARG(n_ == (long long)p_ * q_, "Argument error: the operator does not match the image");
		nnz_ = hp[m_];
		TG_ARG(nnz_ < (1LL << 31), "Argument error: too many operator entries");
		std::vector<int> hp32(hp.begin(), hp.end());
		rptr_ = static_cast<int *>(dmalloc(sizeof(int) * (m_ + 1)));
		rind_ = static_cast<int *>(dmalloc(sizeof(int) * (size_t)nnz_));
		cptr_ = static_cast<int *>(dmalloc(sizeof(int) * (n_ + 1)));
		cind_ = static_cast<int *>(dmalloc(sizeof(int) * (size_t)nnz_));
		TG_CUDA(cudaMemcpy(rptr_, hp32.data(), sizeof(int) * (m_ + 1), cudaMemcpyHostToDevice));
		TG_CUDA(cudaMemcpy(rind_, hi.data(), sizeof(int) * (size_t)nnz_, cudaMemcpyHostToDevice));
		if (!hv.empty()) {
			rval_ = static_cast<float *>(dmalloc(sizeof(float) * (size_t)nnz_));
			cval_ = static_cast<float *>(dmalloc(sizeof(float) * (size_t)nnz_));
			TG_CUDA(cudaMemcpy(rval_, hv.data(), sizeof(float) * (size_t)nnz_, cudaMemcpyHostToDevice));
		}
		build_transpose(own_, m_, n_, nnz_, rptr_, rind_, rval_, cptr_, cind_, cval_);
		TG_CUDA(cudaStreamSynchronize(own_));
		in_.resize(count);
		for (int i = 0; i < count; i++) {
			in_[i].bs = da(m_);
			eng_u_.push_back(static_cast<float *>(dmalloc(sizeof(float) * (size_t)n_)));
		}
		const int nck = K / C_ + 1;
		ck_.resize(count);
		for (int i = 0; i < count; i++)
			for (int c = 0; c < nck; c++)
				for (int v = 0; v < 5; v++) ck_[i].push_back(da(v == 3 ? m_ : n_));
		for (int j = 0; j <= C_; j++) {
			segU_.push_back(da(n_));
			segSx_.push_back(da(n_));
			segSy_.push_back(da(n_));
			segDl_.push_back(da(m_));
			segR_.push_back(da(m_));
		}
		for (double **v : {&vx_, &vy_, &gx_, &gy_, &t1_, &t2_, &d_, &U_, &sx_, &sy_, &ub_, &sbx_, &sby_, &dd_, &ddx_,
		                   &ddy_, &vbx_, &vby_, &zero_})
			*v = da(n_);
		for (double **v : {&au_, &qv_, &dl_, &r_, &dlb_, &bsb_, &ad_, &rb_}) *v = da(m_);
		TG_CUDA(cudaMemset(zero_, 0, sizeof(double) * (size_t)n_));
		pp_ = da(EW_BLOCKS * (NPIX + NMEAS) + 2 * (long long)K);
		pm_ = pp_ + EW_BLOCKS * NPIX;
		gsc_ = pm_ + EW_BLOCKS * NMEAS;
	} catch (...) {
		if (op) tval3g_op_destroy(op);
		release();
		throw;
	}
}

Unrolled::~Unrolled() { release(); }

void Unrolled::release() {
	cudaDeviceSynchronize();
	for (void *p : allocs_) cudaFree(p);
	allocs_.clear();
	delete plan_;
	plan_ = nullptr;
	if (own_) cudaStreamDestroy(own_);
	own_ = nullptr;
}

#define EW(kern, ...)                                                     \
	do {                                                                  \
		kern<<<EW_BLOCKS, EW_THREADS, 0, s>>>(__VA_ARGS__);               \
		TG_CUDA(cudaGetLastError());                                      \
	} while (0)

// y = A x (trans = false) or A^T x, FP64
void Unrolled::apply(bool trans, const double *x, double *y, cudaStream_t s) {
	const long long rows = trans ? n_ : m_;
	k_spmv64<<<(unsigned)((rows * 32 + 255) / 256), 256, 0, s>>>(rows, trans ? cptr_ : rptr_, trans ? cind_ : rind_,
	                                                            trans ? cval_ : rval_, w_, x, y);
	TG_CUDA(cudaGetLastError());
}

// state(k) from U (in place: sigma, delta updated when o); d written
void Unrolled::state(int k, const double *bs, double *U, double *sx, double *sy, double *dl, double *r, double *d,
                     int o, cudaStream_t s) {
	const int j = std::max(k, 1) - 1;
	const double mu = mu_[j], beta = beta_[j];
	EW(k_D64, p_, q_, U, vx_, vy_);
	EW(k_state_pix, n_, vx_, vy_, sx, sy, beta, o, iso_, gx_, gy_);
	apply(false, U, au_, s);
	EW(k_state_meas, m_, au_, bs, r, dl, mu, beta, o, qv_);
	apply(true, qv_, t1_, s);
	EW(k_Dt64, p_, q_, gx_, gy_, t2_);
	EW(k_add, n_, t1_, t2_, d);
}

// replay iterations k0 + 1 .. k1 of instance i from the working state (U_,
// sx_, sy_, dl_, d_ = iteration k0); store_seg: keep every state (j = k - k0)
void Unrolled::replay_from(int i, int k0, int k1, cudaStream_t s, bool store_seg, bool ckpt) {
	const UnrolledInst &I = in_[i];
	const size_t nb = sizeof(double) * (size_t)n_, mb = sizeof(double) * (size_t)m_;
	auto save_seg = [&](int j) {
		TG_CUDA(cudaMemcpyAsync(segU_[j], U_, nb, cudaMemcpyDeviceToDevice, s));
		TG_CUDA(cudaMemcpyAsync(segSx_[j], sx_, nb, cudaMemcpyDeviceToDevice, s));
		TG_CUDA(cudaMemcpyAsync(segSy_[j], sy_, nb, cudaMemcpyDeviceToDevice, s));
		TG_CUDA(cudaMemcpyAsync(segDl_[j], dl_, mb, cudaMemcpyDeviceToDevice, s));
		TG_CUDA(cudaMemcpyAsync(segR_[j], r_, mb, cudaMemcpyDeviceToDevice, s));
	};
	auto save_ck = [&](int k) {
		double *const *c = &ck_[i][(size_t)(k / C_) * 5];
		TG_CUDA(cudaMemcpyAsync(c[0], U_, nb, cudaMemcpyDeviceToDevice, s));
		TG_CUDA(cudaMemcpyAsync(c[1], sx_, nb, cudaMemcpyDeviceToDevice, s));
		TG_CUDA(cudaMemcpyAsync(c[2], sy_, nb, cudaMemcpyDeviceToDevice, s));
		TG_CUDA(cudaMemcpyAsync(c[3], dl_, mb, cudaMemcpyDeviceToDevice, s));
		TG_CUDA(cudaMemcpyAsync(c[4], d_, nb, cudaMemcpyDeviceToDevice, s));
	};
	if (store_seg) save_seg(0);
	if (ckpt && k0 % C_ == 0) save_ck(k0);
	for (int k = k0 + 1; k <= k1; k++) {
		EW(k_axpy, n_, -I.steps[k - 1], d_, U_);
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
	// the FP32 solve that records the decisions
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
	// replay F in FP64 with checkpoints
	const size_t nb = sizeof(double) * (size_t)n_, mb = sizeof(double) * (size_t)m_;
	for (int i = 0; i < count_; i++) {
		UnrolledInst &I = in_[i];
		EW(k_to64, m_, I.scl, d_b[i], I.bs);
		apply(true, I.bs, U_, s);
		TG_CUDA(cudaMemsetAsync(sx_, 0, nb, s));
		TG_CUDA(cudaMemsetAsync(sy_, 0, nb, s));
		TG_CUDA(cudaMemsetAsync(dl_, 0, mb, s));
		state(0, I.bs, U_, sx_, sy_, dl_, r_, d_, 0, s);
		replay_from(i, 0, K_, s, false, true);
		EW(k_to32, n_, 1.0 / I.scl, U_, d_U[i]);
	}
	TG_CUDA(cudaStreamSynchronize(s));
}

void Unrolled::backward(const float *const *d_gU, float *const *d_gb, double *g_mu, double *g_beta, cudaStream_t s) {
	TG_ARG(!mu_.empty(), "Argument error: backward before forward");
	if (!s) s = own_;
	TG_CUDA(cudaMemsetAsync(gsc_, 0, sizeof(double) * 2 * (size_t)K_, s));
	const size_t nb = sizeof(double) * (size_t)n_, mb = sizeof(double) * (size_t)m_;
	for (int i = 0; i < count_; i++) {
		const UnrolledInst &I = in_[i];
		EW(k_to64, n_, 1.0 / I.scl, d_gU[i], ub_);
		for (double *v : {sbx_, sby_}) TG_CUDA(cudaMemsetAsync(v, 0, nb, s));
		for (double *v : {dlb_, bsb_}) TG_CUDA(cudaMemsetAsync(v, 0, mb, s));
		bool has_d = false;
		for (int c = K_ / C_; c >= 0; c--) {
			const int k0 = c * C_, k1 = std::min(k0 + C_, K_);
			if (c > 0 && k0 >= K_) continue;   // a segment without iterations
			// the checkpoint state of iteration k0, r of iteration k0, then the segment
			double *const *ck = &ck_[i][(size_t)c * 5];
			TG_CUDA(cudaMemcpyAsync(U_, ck[0], nb, cudaMemcpyDeviceToDevice, s));
			TG_CUDA(cudaMemcpyAsync(sx_, ck[1], nb, cudaMemcpyDeviceToDevice, s));
			TG_CUDA(cudaMemcpyAsync(sy_, ck[2], nb, cudaMemcpyDeviceToDevice, s));
			TG_CUDA(cudaMemcpyAsync(dl_, ck[3], mb, cudaMemcpyDeviceToDevice, s));
			TG_CUDA(cudaMemcpyAsync(d_, ck[4], nb, cudaMemcpyDeviceToDevice, s));
			apply(false, U_, au_, s);
			EW(k_state_meas, m_, au_, I.bs, r_, dl_, 1.0, 1.0, 0, qv_);   // r only (q unused)
			replay_from(i, k0, k1, s, true, false);
			const int klo = c == 0 ? 0 : k0 + 1;
			for (int k = k1; k >= klo; k--) {
				const int jj = k - k0, j = std::max(k, 1) - 1;
				const double mu = mu_[j], beta = beta_[j];
				const int o = k >= 1 ? I.outer[k - 1] : 0;
				const double *s0x = k >= 1 ? segSx_[jj - 1] : zero_, *s0y = k >= 1 ? segSy_[jj - 1] : zero_;
				if (has_d) {
					EW(k_D64, p_, q_, dd_, ddx_, ddy_);
					apply(false, dd_, ad_, s);
				}
				EW(k_D64, p_, q_, segU_[jj], vx_, vy_);
				EW(k_rev_pix, n_, has_d ? ddx_ : nullptr, has_d ? ddy_ : nullptr, vx_, vy_, s0x, s0y, segSx_[jj],
				   segSy_[jj], sbx_, sby_, beta, o, iso_, vbx_, vby_, pp_);
				EW(k_rev_meas, m_, has_d ? ad_ : nullptr, segR_[jj], segDl_[jj], dlb_, bsb_, mu, beta, o, rb_, pm_);
				k_rev_scalars<<<1, 32, 0, s>>>(pp_, pm_, EW_BLOCKS, mu, beta, gsc_ + j, gsc_ + K_ + j);
				TG_CUDA(cudaGetLastError());
				apply(true, rb_, t1_, s);
				EW(k_Dt64, p_, q_, vbx_, vby_, t2_);
				EW(k_rev_u, n_, t1_, t2_, ub_, k >= 1 ? -I.steps[k - 1] : 0.0, k >= 1 ? dd_ : nullptr);
				has_d = k >= 1;
			}
		}
		// U_0 = A^T bs: bsbar += A Ubar; gb = scl bsbar
		apply(false, ub_, au_, s);
		EW(k_add, m_, bsb_, au_, bsb_);
		EW(k_to32, m_, I.scl, bsb_, d_gb[i]);
	}
	std::vector<double> h(2 * (size_t)K_);
	TG_CUDA(cudaMemcpyAsync(h.data(), gsc_, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, s));
	TG_CUDA(cudaStreamSynchronize(s));
	for (int k = 0; k < K_; k++) {
		g_mu[k] = h[k];
		g_beta[k] = h[K_ + k];
	}
}

TG_END

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
	TG_ARG(!prob->complex_data, "Argument error: the unrolled solve takes real data");
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
