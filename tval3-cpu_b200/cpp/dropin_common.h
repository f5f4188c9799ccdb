// Shared pieces of the C++ drop-in libraries (libtval3_gpu_2d.so,
// libtval3_gpu_3d.so): conversions between the reference's C++ types and the
// C ABI, and the exception contract of the reference's driver
// (2d/tval3_cpu_2d.cpp:878-884: tval3_exception passes through, any other
// std::exception becomes "Internal error: ...").
#ifndef TVAL3_DROPIN_COMMON_H_
#define TVAL3_DROPIN_COMMON_H_

#include <complex>
#include <cstring>
#include <string>

#include "tval3/container.h"
#include "tval3/tval3_types.h"
#include "tval3g.h"

namespace tval3g_dropin {

template <class S>
inline tval3g_options to_c(const tval3_options<S> &o) {
	tval3g_options c;
	std::memset(&c, 0, sizeof(c));
	c.mu = o.mu; c.beta = o.beta; c.mu0 = o.mu0; c.beta0 = o.beta0; c.tol = o.tol; c.tol_inn = o.tol_inn;
	c.c = o.c; c.gamma = o.gamma; c.gam = o.gam; c.rate_gam = o.rate_gam; c.rate_cnt = o.rate_cnt;
	c.skipMulRatio = o.skipMulRatio; c.maxRelativeChange = o.maxRelativeChange;
	c.maxit = o.maxit; c.maxcnt = o.maxcnt; c.nonneg = o.nonneg ? 1 : 0; c.isreal = o.isreal ? 1 : 0;
	c.numInitIterations = (int)o.numInitIterations; c.tv_norm = o.tv_norm;
	return c;
}

template <class S>
inline tval3_info<S> from_c(const tval3g_info &i) {
	tval3_info<S> r;
	r.secs = i.secs;
	r.outer_iters = i.outer_iters;
	r.total_iters = i.total_iters;
	r.rel_chg = (S)i.rel_chg;
	r.rel_error = (S)i.rel_error;
	return r;
}

inline tval3g_problem empty_problem() {
	tval3g_problem p;
	std::memset(&p, 0, sizeof(p));
	p.layers = 1;
	p.numMPs = 1;
	return p;
}

// image shape of U: dim_z is used only by 3D problems
template <class T>
inline void set_image(tval3g_problem &p, int dims, const mat<T> &U) {
	p.dims = dims;
	p.dim_y = U.dim_y;
	p.dim_x = U.dim_x;
	p.dim_z = dims == 3 ? U.dim_z : 1;
}

// element type of real or complex data (complex: interleaved re, im)
template <class T> struct elem { typedef T type; };
template <class T> struct elem<std::complex<T> > { typedef T type; };
template <class T>
inline const typename elem<T>::type *edata(const mat<T> &a) {
	return reinterpret_cast<const typename elem<T>::type *>(a.data());
}
template <class T>
inline typename elem<T>::type *edata(mat<T> &a) {
	return reinterpret_cast<typename elem<T>::type *>(a.data());
}
// the operator values of a dense or sparse matrix as the problem's A /
// csr_val fields hold them: float data as it is; double data still in
// double, which c_solve passes on to tval3g_solve_f64 as its A64 argument
template <class T>
inline const float *raw_values(const T *v) {
	return reinterpret_cast<const float *>(v);
}

// float and complex<float> data: the FP32 engine
inline int c_solve(const tval3g_problem &p, const float *b, int b_len, const tval3g_options *o, const float *Ut,
                   int ut_len, float *U, tval3g_info *info) {
	return tval3g_solve(&p, b, b_len, o, Ut, ut_len, U, info);
}
// double and complex<double> data: the FP64 engine (the reference's double
// instantiations, 2d/tval3_cpu_2d.cpp:905,948,991 and 3d/tval3_cpu_3d.cpp:
// 1408,1475,1542, compute in double)
inline int c_solve(const tval3g_problem &p, const double *b, int b_len, const tval3g_options *o,
                   const double *Ut, int ut_len, double *U, tval3g_info *info) {
	const double *A64 = p.op_kind == TVAL3G_OP_DENSE ? reinterpret_cast<const double *>(p.A)
	                    : p.op_kind == TVAL3G_OP_CSR ? reinterpret_cast<const double *>(p.csr_val)
	                                                 : 0;
	tval3g_problem q = p;
	q.A = 0;
	q.csr_val = 0;
	return tval3g_solve_f64(&q, A64, b, b_len, o, Ut, ut_len, U, info);
}

// run a solve (T = float or double, or their complex forms with
// p.complex_data = 1); throws tval3_exception with the C ABI's message on
// failure
template <class S, class T>
inline tval3_info<S> solve(const tval3g_problem &p, mat<T> &U, const mat<T> &b, const tval3_options<S> &opts,
                           const mat<T> &Ut) {
	tval3g_options o = to_c(opts);
	tval3g_info info;
	std::memset(&info, 0, sizeof(info));
	int rc = c_solve(p, edata(b), b.len, &o, Ut.len > 0 ? edata(Ut) : 0, Ut.len, edata(U), &info);
	if (rc != TVAL3G_OK) {
		std::string msg = tval3g_last_error();
		if (rc == TVAL3G_ERR_ARGUMENT) throw tval3_exception(msg);
		throw tval3_exception("Internal error: " + msg);
	}
	return from_c<S>(info);
}

}  // namespace tval3g_dropin

#endif
