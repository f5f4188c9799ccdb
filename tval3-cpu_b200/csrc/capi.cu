// C ABI of libtval3g.so (include/tval3g.h).
#include <chrono>
#include <cstdlib>
#include <cstring>

#include "plan.cuh"

using namespace tval3g;

namespace tval3g {
static thread_local std::string g_err;
void set_error(const std::string &msg) { g_err = msg; }
}  // namespace tval3g

struct tval3g_plan {
	Plan *p;
};

// operator objects: one instance, its OpStore and the launch maps
struct tval3g_operator {
	OpStore st;
	OpBatch ob;
	Inst h{};
	Inst *d_inst = nullptr;
	Ctrl *d_ctrl = nullptr;
	int2 *d_tiles = nullptr;
	float *d_part = nullptr;
	int *d_fused = nullptr;   // band flags of the one-pass dense normal product
	int *d_err = nullptr;     // set by a kernel whose bounded wait gave up
	float *d_au = nullptr;    // A x of a normal product (trans = 2)
	cudaStream_t s = nullptr;
	long long rows = 0, cols = 0;
};

#define CAPI_BEGIN try {
#define CAPI_END                                                     \
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

static void need_device() {
	int n = 0;
	if (cudaGetDeviceCount(&n) != cudaSuccess || n < 1) {
		cudaGetLastError();
		throw Error{TVAL3G_ERR_NO_DEVICE, "no CUDA device is available"};
	}
}

static long long b_len_of(const tval3g_problem &p) {
	switch (p.op_kind) {
	case TVAL3G_OP_RAY2D: return (long long)p.num_emitters * p.num_receivers;
	case TVAL3G_OP_RAY3D: return (long long)p.numPaths * p.numMPs;
	default: return (long long)p.m * (p.dims == 3 ? 1 : p.layers);
	}
}

extern "C" {

const char *tval3g_last_error(void) { return g_err.c_str(); }
int tval3g_version(void) { return 1; }

int tval3g_solve_batch(int count, const tval3g_problem *probs, const float *const *b, const tval3g_options *opts,
                       const float *const *Ut, float *const *U, tval3g_info *info, int flags) {
	CAPI_BEGIN
	TG_ARG(count >= 1 && probs && b && opts && U, "Argument error: NULL argument");
	auto t0 = std::chrono::steady_clock::now();
	for (int i = 0; i < count; i++) validate(probs[i], b_len_of(probs[i]), 0);
	need_device();
	Plan plan(count, probs, opts, flags & (TVAL3G_GRAPH | TVAL3G_TUNE));
	std::vector<float *> db(count), du(count), dut(count, nullptr);
	std::vector<long long> ns(count);
	cudaStream_t s;
	TG_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
	struct Guard {
		std::vector<float *> *a, *b, *c;
		cudaStream_t s;
		~Guard() {
			cudaStreamSynchronize(s);
			for (auto *v : {a, b, c})
				for (float *p : *v) dev_free(p, s);
			cudaStreamDestroy(s);
		}
	} guard{&db, &du, &dut, s};
	for (int i = 0; i < count; i++) {
		const tval3g_problem &p = probs[i];
		const int planes = p.complex_data ? 2 : 1;   // complex data: interleaved (re, im) floats
		long long n = (long long)p.dim_x * p.dim_y * (p.dims == 3 ? p.dim_z : 1) * planes, bl = b_len_of(p) * planes;
		ns[i] = n;
		db[i] = (float *)dev_alloc(sizeof(float) * bl, s);
		du[i] = (float *)dev_alloc(sizeof(float) * n, s);
		TG_CUDA(cudaMemcpyAsync(db[i], b[i], sizeof(float) * bl, cudaMemcpyHostToDevice, s));
		if (Ut && Ut[i]) {
			dut[i] = (float *)dev_alloc(sizeof(float) * n, s);
			TG_CUDA(cudaMemcpyAsync(dut[i], Ut[i], sizeof(float) * n, cudaMemcpyHostToDevice, s));
		}
	}
	plan.solve(db.data(), dut.data(), du.data(), info, s);
	for (int i = 0; i < count; i++)
		TG_CUDA(cudaMemcpyAsync(U[i], du[i], sizeof(float) * ns[i], cudaMemcpyDeviceToHost, s));
	TG_CUDA(cudaStreamSynchronize(s));
	double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
	if (info)
		for (int i = 0; i < count; i++) info[i].secs = secs;
	int worst = TVAL3G_OK;
	if (info)
		for (int i = 0; i < count; i++)
			if (info[i].status != TVAL3G_OK) worst = info[i].status;
	if (worst != TVAL3G_OK) {
		set_error("a non-finite step length or objective stopped the solve");
		return worst;
	}
	CAPI_END
}

int tval3g_solve(const tval3g_problem *prob, const float *b, int b_len, const tval3g_options *opts,
                 const float *Ut, int ut_len, float *U, tval3g_info *info) {
	CAPI_BEGIN
	TG_ARG(prob && b && opts && U, "Argument error: NULL argument");
	validate(*prob, b_len, Ut ? ut_len : 0, false);   // tval3g_solve_batch checks the rays
	const float *bb[1] = {b};
	const float *uu[1] = {Ut && ut_len > 0 ? Ut : nullptr};
	float *out[1] = {U};
	// the drop-in path takes no flags: TVAL3G_TUNE=1 in the environment turns
	// the autotuner on for it
	const char *tune = std::getenv("TVAL3G_TUNE");
	const int flags = TVAL3G_GRAPH | (tune && std::atoi(tune) != 0 ? TVAL3G_TUNE : 0);
	int rc = tval3g_solve_batch(1, prob, bb, opts, uu, out, info, flags);
	return rc;
	CAPI_END
}

int tval3g_tune_stats(long long *measured, long long *cached) {
	CAPI_BEGIN
	autotune_stats(measured, cached);
	CAPI_END
}

int tval3g_op_launch_shape(const tval3g_operator *op, int *fwd_lanes, int *gather_fwd, int *gather_adj) {
	CAPI_BEGIN
	TG_ARG(op, "Argument error: NULL operator");
	if (fwd_lanes) *fwd_lanes = op->st.dev.fwd_lanes;
	if (gather_fwd) *gather_fwd = op->st.dev.gcls_fwd;
	if (gather_adj) *gather_adj = op->st.dev.gcls_adj;
	CAPI_END
}

int tval3g_trim_memory(long long keep_bytes) {
	CAPI_BEGIN
	TG_ARG(keep_bytes >= 0, "Argument error: keep_bytes must not be negative");
	need_device();
	TG_CUDA(cudaDeviceSynchronize());
	TG_CUDA(cudaMemPoolTrimTo(library_pool(), (size_t)keep_bytes));
	CAPI_END
}

int tval3g_plan_create(tval3g_plan **plan, int count, const tval3g_problem *probs, const tval3g_options *opts,
                       int flags) {
	CAPI_BEGIN
	TG_ARG(plan && probs && opts && count >= 1, "Argument error: NULL argument");
	*plan = nullptr;
	for (int i = 0; i < count; i++) validate(probs[i], b_len_of(probs[i]), 0);
	need_device();
	auto *p = new tval3g_plan{nullptr};
	try {
		p->p = new Plan(count, probs, opts, flags);
	} catch (...) {
		delete p;
		throw;
	}
	*plan = p;
	CAPI_END
}

int tval3g_plan_solve(tval3g_plan *plan, const float *const *d_b, const float *const *d_Ut, float *const *d_U,
                      tval3g_info *info, void *stream) {
	CAPI_BEGIN
	TG_ARG(plan && plan->p, "Argument error: NULL plan");
	plan->p->solve(d_b, d_Ut, d_U, info, (cudaStream_t)stream);
	CAPI_END
}

int tval3g_plan_stats(const tval3g_plan *plan, long long *kernel_launches, long long *device_bytes) {
	CAPI_BEGIN
	TG_ARG(plan && plan->p, "Argument error: NULL plan");
	if (kernel_launches) *kernel_launches = plan->p->launches();
	if (device_bytes) *device_bytes = plan->p->device_bytes();
	CAPI_END
}

int tval3g_plan_time_stencils(tval3g_plan *plan, int reps, double *ms) {
	CAPI_BEGIN
	TG_ARG(plan && plan->p && ms && reps >= 1, "Argument error: NULL plan or output, or reps < 1");
	plan->p->time_stencils(reps, ms);
	CAPI_END
}

int tval3g_plan_set_target(tval3g_plan *plan, double target) {
	CAPI_BEGIN
	TG_ARG(plan && plan->p && target >= 0, "Argument error: NULL plan or negative target");
	plan->p->set_target(target);
	CAPI_END
}

int tval3g_plan_trace(const tval3g_plan *plan, int index, tval3g_trace_record *out, int cap, int *count) {
	CAPI_BEGIN
	TG_ARG(plan && plan->p && out && count, "Argument error: NULL argument");
	*count = plan->p->trace(index, out, cap);
	CAPI_END
}

int tval3g_plan_destroy(tval3g_plan *plan) {
	CAPI_BEGIN
	if (plan) {
		delete plan->p;
		delete plan;
	}
	CAPI_END
}

// --- operators ---------------------------------------------------------------
int tval3g_op_create(tval3g_operator **out, const tval3g_problem *prob, int flags) {
	CAPI_BEGIN
	TG_ARG(out && prob, "Argument error: NULL argument");
	*out = nullptr;
	validate(*prob, b_len_of(*prob), 0);
	need_device();
	auto *op = new tval3g_operator();
	try {
		TG_CUDA(cudaStreamCreateWithFlags(&op->s, cudaStreamNonBlocking));
		prepare_op(op->s, *prob, flags, op->st, true);
		const tval3g_problem &p = *prob;
		Inst &I = op->h;
		const int planes = p.complex_data ? 2 : 1;   // complex: the real form on planar vectors
		I.dims = p.dims; I.p = p.dim_y; I.q = p.dim_x; I.r = p.dims == 3 ? p.dim_z : planes;
		I.n = (long long)p.dim_x * p.dim_y * (p.dims == 3 ? p.dim_z : 1) * planes;
		I.m = op->st.b_len;
		I.cplx = p.complex_data != 0;
		if (flags & TVAL3G_TUNE) autotune_operator(op->s, op->st, I);
		I.op = op->st.dev;
		op->rows = I.m;
		op->cols = I.n;
		TG_CUDA(cudaMalloc(&op->d_ctrl, sizeof(Ctrl)));
		TG_CUDA(cudaMemsetAsync(op->d_ctrl, 0, sizeof(Ctrl), op->s));
		I.ctrl = op->d_ctrl;
		// tile maps (same builder as plans)
		std::vector<Inst> v(1, I);
		std::vector<OpStore> ops(1);
		ops[0].nnz = op->st.nnz;
		ops[0].dev = op->st.dev;
		ops[0].mrhs = op->st.mrhs;
		long long dense_part = build_op_maps_upload(v, ops, op->ob, &op->d_tiles, op->s);
		op->h = v[0];
		if (dense_part > 0) {
			TG_CUDA(cudaMalloc(&op->d_part, sizeof(float) * dense_part));
			op->ob.dense_part = op->d_part;
		}
		if (op->ob.fused_words > 0) {
			TG_CUDA(cudaMalloc(&op->d_fused, sizeof(int) * op->ob.fused_words));
			TG_CUDA(cudaMemsetAsync(op->d_fused, 0, sizeof(int) * op->ob.fused_words, op->s));
			op->ob.fused_flags = op->d_fused;
		}
		TG_CUDA(cudaMalloc(&op->d_err, sizeof(int)));
		TG_CUDA(cudaMemsetAsync(op->d_err, 0, sizeof(int), op->s));
		op->ob.err = op->d_err;
		TG_CUDA(cudaMalloc(&op->d_au, sizeof(float) * std::max<long long>(op->rows, 1)));
		TG_CUDA(cudaMalloc(&op->d_inst, sizeof(Inst)));
		TG_CUDA(cudaStreamSynchronize(op->s));
	} catch (...) {
		free_op(op->st, op->s);
		delete op;
		throw;
	}
	*out = op;
	CAPI_END
}

int tval3g_op_shape(const tval3g_operator *op, long long *rows, long long *cols, long long *nnz) {
	CAPI_BEGIN
	TG_ARG(op, "Argument error: NULL operator");
	if (rows) *rows = op->rows;
	if (cols) *cols = op->cols;
	if (nnz) *nnz = op->st.nnz;
	CAPI_END
}

int tval3g_op_adjoint_index_bytes(const tval3g_operator *op, long long *bytes) {
	CAPI_BEGIN
	TG_ARG(op && bytes, "Argument error: NULL argument");
	*bytes = op->st.adj_index_bytes;
	CAPI_END
}

int tval3g_op_apply(tval3g_operator *op, int trans, const float *d_x, float *d_y, void *stream) {
	int rc = tval3g_op_apply_n(op, trans, d_x, d_y, 1, stream);
	if (rc != TVAL3G_OK) return rc;
	CAPI_BEGIN
	cudaStream_t s = stream ? (cudaStream_t)stream : op->s;
	int e = 0;
	TG_CUDA(cudaMemcpyAsync(&e, op->d_err, sizeof(int), cudaMemcpyDeviceToHost, s));
	TG_CUDA(cudaStreamSynchronize(s));
	if (op->st.mrhs && mrhs_take_error(s, *op->st.mrhs))
		throw Error{TVAL3G_ERR_CUDA, "tensor-core operator: a bounded wait timed out (results invalid)"};
	if (e) {
		TG_CUDA(cudaMemsetAsync(op->d_err, 0, sizeof(int), s));
		TG_CUDA(cudaStreamSynchronize(s));
		throw Error{TVAL3G_ERR_CUDA, "operator: a bounded wait timed out (results invalid)"};
	}
	CAPI_END
}

int tval3g_op_apply_n(tval3g_operator *op, int trans, const float *d_x, float *d_y, int reps, void *stream) {
	CAPI_BEGIN
	TG_ARG(op && d_x && d_y && reps >= 1, "Argument error: NULL argument or reps < 1");
	cudaStream_t s = stream ? (cudaStream_t)stream : op->s;
	Inst I = op->h;
	TG_ARG(trans >= 0 && trans <= 2, "Argument error: trans must be 0, 1 or 2");
	// x lives in the bank of its length: image vectors vn, measurement vectors vm
	VecSel xs, ys;
	if (trans == 2) {   // y = A^T (A x): vn[0] = x, vm[0] = A x, vn[1] = y
		I.vn[0] = const_cast<float *>(d_x); I.vm[0] = op->d_au; I.vn[1] = d_y;
		if (op->st.dev.kind == TVAL3G_OP_RAY2D || op->st.dev.kind == TVAL3G_OP_RAY3D)
			TG_CUDA(cudaMemsetAsync(op->d_au, 0, sizeof(float) * op->rows, s));
		TG_CUDA(cudaMemcpyAsync(op->d_inst, &I, sizeof(Inst), cudaMemcpyHostToDevice, s));
		LaunchCtx L{s, op->d_inst, nullptr};
		// the one-pass dense kernel reads x as float4: a misaligned x takes the two products
		const bool aligned = (reinterpret_cast<uintptr_t>(d_x) & 15) == 0;
		for (int r = 0; r < reps; r++) {
			if (aligned) {
				op_normal(L, op->ob, P_ALL, VecSel{false, 0}, VecSel{true, 0}, VecSel{false, 1});
			} else {
				op_forward(L, op->ob, P_ALL, VecSel{false, 0}, VecSel{true, 0});
				op_adjoint(L, op->ob, P_ALL, VecSel{true, 0}, VecSel{false, 1});
			}
		}
		return TVAL3G_OK;
	}
	if (!trans) {
		I.vn[0] = const_cast<float *>(d_x); I.vm[0] = d_y;
		xs = VecSel{false, 0}; ys = VecSel{true, 0};
		if (op->st.dev.kind == TVAL3G_OP_RAY2D || op->st.dev.kind == TVAL3G_OP_RAY3D)
			TG_CUDA(cudaMemsetAsync(d_y, 0, sizeof(float) * op->rows, s));
	} else {
		I.vm[0] = const_cast<float *>(d_x); I.vn[0] = d_y;
		xs = VecSel{true, 0}; ys = VecSel{false, 0};
	}
	TG_CUDA(cudaMemcpyAsync(op->d_inst, &I, sizeof(Inst), cudaMemcpyHostToDevice, s));
	LaunchCtx L{s, op->d_inst, nullptr};
	for (int r = 0; r < reps; r++) {
		if (!trans) op_forward(L, op->ob, P_ALL, xs, ys);
		else op_adjoint(L, op->ob, P_ALL, xs, ys);
	}
	CAPI_END
}

int tval3g_op_ray_csr(const tval3g_operator *op, long long *rowptr, int *colind) {
	CAPI_BEGIN
	TG_ARG(op && rowptr, "Argument error: NULL argument");
	TG_ARG(op->st.ray_rptr != nullptr, "Argument error: not a ray operator");
	const int nr = op->st.dev.nrays;
	std::vector<int> rp(nr + 1);
	TG_CUDA(cudaMemcpy(rp.data(), op->st.ray_rptr, sizeof(int) * (nr + 1), cudaMemcpyDeviceToHost));
	std::vector<long long> len(op->rows, 0);
	for (int k = 0; k < nr; k++) len[op->st.ray_out[k]] = rp[k + 1] - rp[k];
	rowptr[0] = 0;
	for (long long r = 0; r < op->rows; r++) rowptr[r + 1] = rowptr[r] + len[r];
	if (colind) {
		std::vector<int> ind(op->st.nnz);
		if (op->st.nnz > 0)
			TG_CUDA(cudaMemcpy(ind.data(), op->st.ray_rind, sizeof(int) * op->st.nnz, cudaMemcpyDeviceToHost));
		for (int k = 0; k < nr; k++)
			std::memcpy(colind + rowptr[op->st.ray_out[k]], ind.data() + rp[k], sizeof(int) * (rp[k + 1] - rp[k]));
	}
	CAPI_END
}

int tval3g_op_destroy(tval3g_operator *op) {
	CAPI_BEGIN
	if (op) {
		if (op->s) cudaStreamSynchronize(op->s);
		free_op(op->st, op->s);
		cudaFree(op->d_inst);
		cudaFree(op->d_ctrl);
		cudaFree(op->d_tiles);
		cudaFree(op->d_part);
		cudaFree(op->d_fused);
		cudaFree(op->d_err);
		cudaFree(op->d_au);
		if (op->s) cudaStreamDestroy(op->s);
		delete op;
	}
	CAPI_END
}

// --- stencils ------------------------------------------------------------------
int tval3g_D(int dims, int dim_y, int dim_x, int dim_z, const float *U, float *Ux, float *Uy, float *Uz,
             void *stream) {
	CAPI_BEGIN
	TG_ARG((dims == 2 || dims == 3) && dim_y >= 1 && dim_x >= 1 && (dims == 2 || dim_z >= 1) && U && Ux && Uy &&
	           (dims == 2 || Uz),
	       "Argument error: bad stencil arguments");
	launch_D_plain((cudaStream_t)stream, dims, dim_y, dim_x, dim_z, U, Ux, Uy, Uz);
	TG_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
	CAPI_END
}

int tval3g_Dt(int dims, int dim_y, int dim_x, int dim_z, const float *X, const float *Y, const float *Z,
              float *res, void *stream) {
	CAPI_BEGIN
	TG_ARG((dims == 2 || dims == 3) && dim_y >= 1 && dim_x >= 1 && (dims == 2 || dim_z >= 1) && X && Y && res &&
	           (dims == 2 || Z),
	       "Argument error: bad stencil arguments");
	launch_Dt_plain((cudaStream_t)stream, dims, dim_y, dim_x, dim_z, X, Y, Z, res);
	TG_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
	CAPI_END
}

int tval3g_shrink(int dims, long long n, int tv_norm, double beta, const float *Ux, const float *Uy,
                  const float *Uz, const float *sx, const float *sy, const float *sz, float *Wx, float *Wy,
                  float *Wz, double *lam1, void *stream) {
	CAPI_BEGIN
	TG_ARG((dims == 2 || dims == 3) && n >= 1 && beta > 0 && Ux && Uy && sx && sy && Wx && Wy &&
	           (dims == 2 || (Uz && sz && Wz)),
	       "Argument error: bad shrinkage arguments");
	double *d = nullptr;
	cudaStream_t s = (cudaStream_t)stream;
	d = (decltype(d))dev_alloc(sizeof(double), s);
	TG_CUDA(cudaMemsetAsync(d, 0, sizeof(double), s));
	launch_shrink_plain(s, dims, n, tv_norm, beta, Ux, Uy, Uz, sx, sy, sz, Wx, Wy, Wz, d);
	double h = 0;
	TG_CUDA(cudaMemcpyAsync(&h, d, sizeof(double), cudaMemcpyDeviceToHost, s));
	dev_free(d, s);
	TG_CUDA(cudaStreamSynchronize(s));
	if (lam1) *lam1 = h;
	CAPI_END
}

}  // extern "C"
