// libtval3_gpu_3d.so: the reference's 3D C++ entry points on the GPU
// (include/tval3_gpu_3d.h).  Argument checks follow check_params
// (3d/tval3_cpu_3d.cpp:1028-1165) in order and wording; the size checks that
// follow the format checks are made by tval3g_solve with the same messages.
#include <vector>

#include "../../include/tval3_gpu_3d.h"

#include "dropin_common.h"

using namespace tval3g_dropin;

namespace {

template <class T> struct is_cplx { static const int value = 0; };
template <class T> struct is_cplx<std::complex<T> > { static const int value = 1; };

template <class S, class T>
tval3_info<S> dense3d(mat<T> &U, const mat<T> &A, const mat<T> &b, const tval3_options<S> &opts, const mat<T> &Ut) {
	if (U.format != mat_row_major || Ut.format != mat_row_major || A.format != mat_row_major)
		throw tval3_exception(std::string("Argument error: Matrices must be in row major format!"));
	tval3g_problem p = empty_problem();
	set_image(p, 3, U);
	p.op_kind = TVAL3G_OP_DENSE;
	p.m = A.dim_y;
	p.n_cols = A.dim_x;
	p.A = raw_values(A.data());
	p.complex_data = is_cplx<T>::value;
	return solve<S>(p, U, b, opts, Ut);
}

template <class S, class T>
tval3_info<S> sparse3d(mat<T> &U, const sparse_mat<T> &A, const mat<T> &b, const tval3_options<S> &opts,
                       const mat<T> &Ut) {
	if (U.format != mat_col_major || Ut.format != mat_col_major)
		throw tval3_exception(std::string("Argument error: Matrices must be in row major format!"));
	if (A.format != sparse_mat_both)
		throw tval3_exception(std::string("Argument error: A must be available in csr and csc format!"));
	tval3g_problem p = empty_problem();
	set_image(p, 3, U);
	p.op_kind = TVAL3G_OP_CSR;
	p.m = A.dim_y;
	p.n_cols = A.dim_x;
	p.nnz = A.nnz;
	p.csr_ptr = A.csr_ptr();
	p.csr_ind = A.csr_ind();
	p.csr_val = raw_values(A.csr_val());
	p.complex_data = is_cplx<T>::value;
	return solve<S>(p, U, b, opts, Ut);
}

template <class S, class T>
tval3_info<S> ray3d(mat<T> &U, const geometry &A, const mat<T> &b, const tval3_options<S> &opts, const mat<T> &Ut) {
	if (U.format != mat_row_major || Ut.format != mat_row_major)
		throw tval3_exception(std::string("Argument error: Matrices must be in row major format!"));
	// per-measurement-position coordinate arrays, flattened [mp*E + e]
	const int nmp = A.numMPs > 0 ? A.numMPs : 0, E = A.num_emitters, R = A.num_receivers;
	std::vector<int> xe((size_t)nmp * E), ye(xe.size()), ze(xe.size()), xr((size_t)nmp * R), yr(xr.size()),
		zr(xr.size());
	for (int mp = 0; mp < nmp; mp++) {
		for (int e = 0; e < E; e++) {
			xe[(size_t)mp * E + e] = A.x_emitters[mp][e];
			ye[(size_t)mp * E + e] = A.y_emitters[mp][e];
			ze[(size_t)mp * E + e] = A.z_emitters[mp][e];
		}
		for (int r = 0; r < R; r++) {
			xr[(size_t)mp * R + r] = A.x_receivers[mp][r];
			yr[(size_t)mp * R + r] = A.y_receivers[mp][r];
			zr[(size_t)mp * R + r] = A.z_receivers[mp][r];
		}
	}
	tval3g_problem p = empty_problem();
	set_image(p, 3, U);
	p.op_kind = TVAL3G_OP_RAY3D;
	p.numMPs = A.numMPs;
	p.numPaths = A.numPaths;
	p.num_emitters = E;
	p.num_receivers = R;
	p.use_path = A.use_path;
	p.x_emitters = xe.data(); p.y_emitters = ye.data(); p.z_emitters = ze.data();
	p.x_receivers = xr.data(); p.y_receivers = yr.data(); p.z_receivers = zr.data();
	p.rv_x = A.rv_x; p.rv_y = A.rv_y; p.rv_z = A.rv_z;
	p.scale_factor = A.scale_factor;
	p.complex_data = is_cplx<T>::value;
	return solve<S>(p, U, b, opts, Ut);
}

}  // namespace

typedef std::complex<float> cf;
typedef std::complex<double> cd;

const tval3_info<float> tval3_cpu_3d(mat<float> &U, const mat<float> &A, const mat<float> &b,
                                     const tval3_options<float> &opts, const mat<float> &Ut, int, int) {
	return dense3d<float>(U, A, b, opts, Ut);
}
const tval3_info<double> tval3_cpu_3d(mat<float> &U, const mat<float> &A, const mat<float> &b,
                                      const tval3_options<double> &opts, const mat<float> &Ut, int, int) {
	return dense3d<double>(U, A, b, opts, Ut);
}
const tval3_info<double> tval3_cpu_3d(mat<double> &U, const mat<double> &A, const mat<double> &b,
                                      const tval3_options<double> &opts, const mat<double> &Ut, int, int) {
	return dense3d<double>(U, A, b, opts, Ut);
}
const tval3_info<float> tval3_cpu_3d(mat<cf> &U, const mat<cf> &A, const mat<cf> &b,
                                     const tval3_options<float> &opts, const mat<cf> &Ut, int, int) {
	return dense3d<float>(U, A, b, opts, Ut);
}
const tval3_info<double> tval3_cpu_3d(mat<cd> &U, const mat<cd> &A, const mat<cd> &b,
                                      const tval3_options<double> &opts, const mat<cd> &Ut, int, int) {
	return dense3d<double>(U, A, b, opts, Ut);
}

const tval3_info<float> tval3_cpu_3d(mat<float> &U, const sparse_mat<float> &A, const mat<float> &b,
                                     const tval3_options<float> &opts, const mat<float> &Ut, int, int) {
	return sparse3d<float>(U, A, b, opts, Ut);
}
const tval3_info<double> tval3_cpu_3d(mat<float> &U, const sparse_mat<float> &A, const mat<float> &b,
                                      const tval3_options<double> &opts, const mat<float> &Ut, int, int) {
	return sparse3d<double>(U, A, b, opts, Ut);
}
const tval3_info<double> tval3_cpu_3d(mat<double> &U, const sparse_mat<double> &A, const mat<double> &b,
                                      const tval3_options<double> &opts, const mat<double> &Ut, int, int) {
	return sparse3d<double>(U, A, b, opts, Ut);
}
const tval3_info<float> tval3_cpu_3d(mat<cf> &U, const sparse_mat<cf> &A, const mat<cf> &b,
                                     const tval3_options<float> &opts, const mat<cf> &Ut, int, int) {
	return sparse3d<float>(U, A, b, opts, Ut);
}
const tval3_info<double> tval3_cpu_3d(mat<cd> &U, const sparse_mat<cd> &A, const mat<cd> &b,
                                      const tval3_options<double> &opts, const mat<cd> &Ut, int, int) {
	return sparse3d<double>(U, A, b, opts, Ut);
}

const tval3_info<float> tval3_cpu_3d(mat<float> &U, const geometry &A, const mat<float> &b,
                                     const tval3_options<float> &opts, const mat<float> &Ut, int, int) {
	return ray3d<float>(U, A, b, opts, Ut);
}
const tval3_info<double> tval3_cpu_3d(mat<float> &U, const geometry &A, const mat<float> &b,
                                      const tval3_options<double> &opts, const mat<float> &Ut, int, int) {
	return ray3d<double>(U, A, b, opts, Ut);
}
const tval3_info<double> tval3_cpu_3d(mat<double> &U, const geometry &A, const mat<double> &b,
                                      const tval3_options<double> &opts, const mat<double> &Ut, int, int) {
	return ray3d<double>(U, A, b, opts, Ut);
}
const tval3_info<float> tval3_cpu_3d(mat<cf> &U, const geometry &A, const mat<cf> &b,
                                     const tval3_options<float> &opts, const mat<cf> &Ut, int, int) {
	return ray3d<float>(U, A, b, opts, Ut);
}
const tval3_info<double> tval3_cpu_3d(mat<cd> &U, const geometry &A, const mat<cd> &b,
                                      const tval3_options<double> &opts, const mat<cd> &Ut, int, int) {
	return ray3d<double>(U, A, b, opts, Ut);
}
