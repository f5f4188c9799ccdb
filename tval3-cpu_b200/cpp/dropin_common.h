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

// the float view of float or complex<float> data (interleaved re, im)
inline const float *fdata(const mat<float> &a) { return a.data(); }
inline float *fdata(mat<float> &a) { return a.data(); }
inline const float *fdata(const mat<std::complex<float> > &a) { return reinterpret_cast<const float *>(a.data()); }
inline float *fdata(mat<std::complex<float> > &a) { return reinterpret_cast<float *>(a.data()); }

// run a solve (T = float, or complex<float> with p.complex_data = 1); throws
// tval3_exception with the C ABI's message on failure
template <class S, class T>
inline tval3_info<S> solve(const tval3g_problem &p, mat<T> &U, const mat<T> &b, const tval3_options<S> &opts,
                           const mat<T> &Ut) {
	tval3g_options o = to_c(opts);
	tval3g_info info;
	std::memset(&info, 0, sizeof(info));
	int rc = tval3g_solve(&p, fdata(b), b.len, &o, Ut.len > 0 ? fdata(Ut) : 0, Ut.len, fdata(U), &info);
	if (rc != TVAL3G_OK) {
		std::string msg = tval3g_last_error();
		if (rc == TVAL3G_ERR_ARGUMENT) throw tval3_exception(msg);
		throw tval3_exception("Internal error: " + msg);
	}
	return from_c<S>(info);
}

// Double data (the reference's double overloads, 2d/tval3_cpu_2d.cpp:905,
// 948,991 and 3d/tval3_cpu_3d.cpp:1408,1475,1542) runs through the FP32
// engine: FP32 copies of the arrays (shape and format kept), the FP32 solve
// with its FP64 reductions, the solution widened into the caller's U.  The
// result therefore carries FP32 storage error, not double precision.
inline mat<float> narrow(const mat<double> &a) {
	mat<float> f(a.dim_y, a.dim_x, a.dim_z, a.format);
	for (int i = 0; i < a.len; i++) f[i] = (float)a[i];
	return f;
}
inline void narrow(const sparse_mat<double> &a, sparse_mat<float> &f) {   // f: sized as a
	std::memcpy(f.csr_ptr(), a.csr_ptr(), sizeof(int) * ((size_t)a.dim_y + 1));
	std::memcpy(f.csc_ptr(), a.csc_ptr(), sizeof(int) * ((size_t)a.dim_x + 1));
	if (a.nnz > 0) {
		std::memcpy(f.csr_ind(), a.csr_ind(), sizeof(int) * (size_t)a.nnz);
		std::memcpy(f.csc_ind(), a.csc_ind(), sizeof(int) * (size_t)a.nnz);
	}
	for (int k = 0; k < a.nnz; k++) {
		f.csr_val()[k] = (float)a.csr_val()[k];
		f.csc_val()[k] = (float)a.csc_val()[k];
	}
}
inline void widen(const mat<float> &f, mat<double> &a) {
	for (int i = 0; i < a.len && i < f.len; i++) a[i] = (double)f[i];
}
// complex<double> data (the reference's complex<double> overloads) likewise
// through complex<float>
inline mat<std::complex<float> > narrow(const mat<std::complex<double> > &a) {
	mat<std::complex<float> > f(a.dim_y, a.dim_x, a.dim_z, a.format);
	for (int i = 0; i < a.len; i++) f[i] = std::complex<float>((float)a[i].real(), (float)a[i].imag());
	return f;
}
inline void narrow(const sparse_mat<std::complex<double> > &a, sparse_mat<std::complex<float> > &f) {
	std::memcpy(f.csr_ptr(), a.csr_ptr(), sizeof(int) * ((size_t)a.dim_y + 1));
	std::memcpy(f.csc_ptr(), a.csc_ptr(), sizeof(int) * ((size_t)a.dim_x + 1));
	if (a.nnz > 0) {
		std::memcpy(f.csr_ind(), a.csr_ind(), sizeof(int) * (size_t)a.nnz);
		std::memcpy(f.csc_ind(), a.csc_ind(), sizeof(int) * (size_t)a.nnz);
	}
	for (int k = 0; k < a.nnz; k++) {
		f.csr_val()[k] = std::complex<float>((float)a.csr_val()[k].real(), (float)a.csr_val()[k].imag());
		f.csc_val()[k] = std::complex<float>((float)a.csc_val()[k].real(), (float)a.csc_val()[k].imag());
	}
}
inline void widen(const mat<std::complex<float> > &f, mat<std::complex<double> > &a) {
	for (int i = 0; i < a.len && i < f.len; i++) a[i] = std::complex<double>(f[i].real(), f[i].imag());
}


}  // namespace tval3g_dropin

#endif
