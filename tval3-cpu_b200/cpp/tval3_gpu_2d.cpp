// libtval3_gpu_2d.so: the reference's 2D C++ entry points on the GPU
// (include/tval3_gpu_2d.h).  Argument checks follow check_params
// (2d/tval3_cpu_2d.cpp:696-750) in order and wording; the size checks that
// follow the format checks are made by tval3g_solve with the same messages.
#include "../../include/tval3_gpu_2d.h"

#include "dropin_common.h"

using namespace tval3g_dropin;

namespace {

template <class T> struct is_cplx { static const int value = 0; };
template <class T> struct is_cplx<std::complex<T> > { static const int value = 1; };

template <class S, class T>
tval3_info<S> dense2d(mat<T> &U, const mat<T> &A, const mat<T> &b, const tval3_options<S> &opts, const mat<T> &Ut) {
	if (U.format != mat_col_major || Ut.format != mat_col_major || A.format != mat_row_major)
		throw tval3_exception(std::string("Argument error: Matrices must be in row major format!"));
	tval3g_problem p = empty_problem();
	set_image(p, 2, U);
	p.op_kind = TVAL3G_OP_DENSE;
	p.m = A.dim_y;
	p.n_cols = A.dim_x;
	p.layers = A.dim_y > 0 ? b.len / A.dim_y : 0;   // 2d/tval3_cpu_2d.cpp:894
	p.A = raw_values(A.data());
	p.complex_data = is_cplx<T>::value;
	return solve<S>(p, U, b, opts, Ut);
}

template <class S, class T>
tval3_info<S> sparse2d(mat<T> &U, const sparse_mat<T> &A, const mat<T> &b, const tval3_options<S> &opts,
                       const mat<T> &Ut) {
	if (U.format != mat_col_major || Ut.format != mat_col_major)
		throw tval3_exception(std::string("Argument error: Matrices must be in row major format!"));
	if (A.format != sparse_mat_both)
		throw tval3_exception(std::string("Argument error: A must be available in CSR and CSC format!"));
	tval3g_problem p = empty_problem();
	set_image(p, 2, U);
	p.op_kind = TVAL3G_OP_CSR;
	p.m = A.dim_y;
	p.n_cols = A.dim_x;
	p.layers = A.dim_y > 0 ? b.len / A.dim_y : 0;
	p.nnz = A.nnz;
	p.csr_ptr = A.csr_ptr();
	p.csr_ind = A.csr_ind();
	p.csr_val = raw_values(A.csr_val());
	p.complex_data = is_cplx<T>::value;
	return solve<S>(p, U, b, opts, Ut);
}

template <class S, class T>
tval3_info<S> ray2d(mat<T> &U, const geometry &A, const mat<T> &b, const tval3_options<S> &opts, const mat<T> &Ut) {
	if (U.format != mat_row_major || Ut.format != mat_row_major)
		throw tval3_exception(std::string("Argument error: Matrices must be in row major format!"));
	tval3g_problem p = empty_problem();
	set_image(p, 2, U);
	p.op_kind = TVAL3G_OP_RAY2D;
	p.num_emitters = A.num_emitters;
	p.num_receivers = A.num_receivers;
	p.use_path = A.use_path;
	p.x_emitters = A.x_emitters;
	p.y_emitters = A.y_emitters;
	p.x_receivers = A.x_receivers;
	p.y_receivers = A.y_receivers;
	p.ld = A.ld;
	p.scale_factor = A.scale_factor;
	p.complex_data = is_cplx<T>::value;
	return solve<S>(p, U, b, opts, Ut);
}

}  // namespace

// ---- dense -----------------------------------------------------------------
const tval3_info<float> tval3_cpu_2d(mat<float> &U, const mat<float> &A, const mat<float> &b,
                                     const tval3_options<float> &opts, const mat<float> &Ut, int, int) {
	return dense2d<float>(U, A, b, opts, Ut);
}
const tval3_info<double> tval3_cpu_2d(mat<float> &U, const mat<float> &A, const mat<float> &b,
                                      const tval3_options<double> &opts, const mat<float> &Ut, int, int) {
	return dense2d<double>(U, A, b, opts, Ut);
}
const tval3_info<double> tval3_cpu_2d(mat<double> &U, const mat<double> &A, const mat<double> &b,
                                      const tval3_options<double> &opts, const mat<double> &Ut, int, int) {
	return dense2d<double>(U, A, b, opts, Ut);
}
const tval3_info<float> tval3_cpu_2d(mat<std::complex<float> > &U, const mat<std::complex<float> > &A,
                                     const mat<std::complex<float> > &b, const tval3_options<float> &opts,
                                     const mat<std::complex<float> > &Ut, int, int) {
	return dense2d<float>(U, A, b, opts, Ut);
}
const tval3_info<double> tval3_cpu_2d(mat<std::complex<double> > &U, const mat<std::complex<double> > &A,
                                      const mat<std::complex<double> > &b, const tval3_options<double> &opts,
                                      const mat<std::complex<double> > &Ut, int, int) {
	return dense2d<double>(U, A, b, opts, Ut);
}

// ---- sparse ----------------------------------------------------------------
const tval3_info<float> tval3_cpu_2d(mat<float> &U, const sparse_mat<float> &A, const mat<float> &b,
                                     const tval3_options<float> &opts, const mat<float> &Ut, int, int) {
	return sparse2d<float>(U, A, b, opts, Ut);
}
const tval3_info<double> tval3_cpu_2d(mat<float> &U, const sparse_mat<float> &A, const mat<float> &b,
                                      const tval3_options<double> &opts, const mat<float> &Ut, int, int) {
	return sparse2d<double>(U, A, b, opts, Ut);
}
const tval3_info<double> tval3_cpu_2d(mat<double> &U, const sparse_mat<double> &A, const mat<double> &b,
                                      const tval3_options<double> &opts, const mat<double> &Ut, int, int) {
	return sparse2d<double>(U, A, b, opts, Ut);
}
const tval3_info<float> tval3_cpu_2d(mat<std::complex<float> > &U, const sparse_mat<std::complex<float> > &A,
                                     const mat<std::complex<float> > &b, const tval3_options<float> &opts,
                                     const mat<std::complex<float> > &Ut, int, int) {
	return sparse2d<float>(U, A, b, opts, Ut);
}
const tval3_info<double> tval3_cpu_2d(mat<std::complex<double> > &U, const sparse_mat<std::complex<double> > &A,
                                      const mat<std::complex<double> > &b, const tval3_options<double> &opts,
                                      const mat<std::complex<double> > &Ut, int, int) {
	return sparse2d<double>(U, A, b, opts, Ut);
}

// ---- geometry --------------------------------------------------------------
const tval3_info<float> tval3_cpu_2d(mat<float> &U, const geometry &A, const mat<float> &b,
                                     const tval3_options<float> &opts, const mat<float> &Ut, int, int) {
	return ray2d<float>(U, A, b, opts, Ut);
}
const tval3_info<double> tval3_cpu_2d(mat<float> &U, const geometry &A, const mat<float> &b,
                                      const tval3_options<double> &opts, const mat<float> &Ut, int, int) {
	return ray2d<double>(U, A, b, opts, Ut);
}
const tval3_info<double> tval3_cpu_2d(mat<double> &U, const geometry &A, const mat<double> &b,
                                      const tval3_options<double> &opts, const mat<double> &Ut, int, int) {
	return ray2d<double>(U, A, b, opts, Ut);
}
const tval3_info<float> tval3_cpu_2d(mat<std::complex<float> > &U, const geometry &A,
                                     const mat<std::complex<float> > &b, const tval3_options<float> &opts,
                                     const mat<std::complex<float> > &Ut, int, int) {
	return ray2d<float>(U, A, b, opts, Ut);
}
const tval3_info<double> tval3_cpu_2d(mat<std::complex<double> > &U, const geometry &A,
                                      const mat<std::complex<double> > &b, const tval3_options<double> &opts,
                                      const mat<std::complex<double> > &Ut, int, int) {
	return ray2d<double>(U, A, b, opts, Ut);
}
