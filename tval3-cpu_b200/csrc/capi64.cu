// C ABI of the FP64 engine (include/tval3g.h: tval3g_solve_f64).  This file
// is compiled with TVAL3G_FP64: its Plan, operators and kernels are the FP64
// build of the engine (tval3g::f64), whose vectors, operator values and
// stencil arithmetic are double.
#include <chrono>
#include <cstring>

#include "plan.cuh"

using namespace tval3g;

namespace {

void need_device64() {
	int n = 0;
	if (cudaGetDeviceCount(&n) != cudaSuccess || n < 1) {
		cudaGetLastError();
		throw Error{TVAL3G_ERR_NO_DEVICE, "no CUDA device is available"};
	}
}

}  // namespace

extern "C" int tval3g_solve_f64(const tval3g_problem *prob, const double *A64, const double *b, int b_len,
                                const tval3g_options *opts, const double *Ut, int ut_len, double *U,
                                tval3g_info *info) {
	try {
		TG_ARG(prob && b && opts && U, "Argument error: NULL argument");
		auto t0 = std::chrono::steady_clock::now();
		// the double operator values travel in the problem's A / csr_val
		// fields, which the FP64 build reads as double (prob_A, prob_val)
		tval3g_problem p = *prob;
		p.A = nullptr;
		p.csr_val = nullptr;
		if (p.op_kind == TVAL3G_OP_DENSE) p.A = reinterpret_cast<const float *>(A64);
		else if (p.op_kind == TVAL3G_OP_CSR) p.csr_val = reinterpret_cast<const float *>(A64);
		validate(p, b_len, Ut ? ut_len : 0);
		need_device64();
		Plan plan(1, &p, opts, TVAL3G_GRAPH);
		const int planes = p.complex_data ? 2 : 1;   // complex data: interleaved (re, im) doubles
		const long long n = (long long)p.dim_x * p.dim_y * (p.dims == 3 ? p.dim_z : 1) * planes;
		const long long bl = (long long)b_len * planes;
		cudaStream_t s;
		TG_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
		double *db = nullptr, *du = nullptr, *dut = nullptr;
		struct Guard {
			double **a, **b, **c;
			cudaStream_t s;
			~Guard() {
				cudaStreamSynchronize(s);
				for (double **v : {a, b, c})
					if (*v) dev_free(*v, s);
				cudaStreamDestroy(s);
			}
		} guard{&db, &du, &dut, s};
		db = (double *)dev_alloc(sizeof(double) * (size_t)bl, s);
		du = (double *)dev_alloc(sizeof(double) * (size_t)n, s);
		TG_CUDA(cudaMemcpyAsync(db, b, sizeof(double) * (size_t)bl, cudaMemcpyHostToDevice, s));
		if (Ut && ut_len > 0) {
			dut = (double *)dev_alloc(sizeof(double) * (size_t)n, s);
			TG_CUDA(cudaMemcpyAsync(dut, Ut, sizeof(double) * (size_t)n, cudaMemcpyHostToDevice, s));
		}
		const double *bb[1] = {db};
		const double *uu[1] = {dut};
		double *out[1] = {du};
		tval3g_info inf;
		std::memset(&inf, 0, sizeof(inf));
		plan.solve(bb, uu, out, &inf, s);
		TG_CUDA(cudaMemcpyAsync(U, du, sizeof(double) * (size_t)n, cudaMemcpyDeviceToHost, s));
		TG_CUDA(cudaStreamSynchronize(s));
		inf.secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
		if (info) *info = inf;
		if (inf.status != TVAL3G_OK) {
			set_error("a non-finite step length or objective stopped the solve");
			return inf.status;
		}
	} catch (const Error &e) {
		set_error(e.msg);
		return e.code;
	} catch (const std::exception &e) {
		set_error(std::string("Internal error: ") + e.what());
		return TVAL3G_ERR_INTERNAL;
	}
	return TVAL3G_OK;
}
