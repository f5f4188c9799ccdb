/*
 * Oracle (test infrastructure only): C entry points around the reference's
 * 3D overloads tval3_cpu_3d (3d/tval3_cpu_3d.cpp:32-146,1384-1581), re-declared
 * as the reference declares them and linked against its own object file.
 * The reference prints "count_outer = ..." to stdout and writes profile.txt to
 * the current directory on every call (3d/tval3_cpu_3d.cpp:1228,1328-1349).
 */
#include <complex>
#include <cstring>
#include <string>
#include <vector>
#include "container.h"
#include "tval3_types.h"
#include "ref_capi.h"

#define DECL(T, S, OP) \
	extern const tval3_info<S> tval3_cpu_3d(mat<T> &U, const OP &A, const mat<T> &b, \
		const tval3_options<S> &opts, const mat<T> &Ut, int submat_mb, int vppc) throw(tval3_exception);
DECL(float, float, mat<float>)
DECL(float, double, mat<float>)
DECL(double, double, mat<double>)
DECL(float, float, sparse_mat<float>)
DECL(float, double, sparse_mat<float>)
DECL(double, double, sparse_mat<double>)
DECL(float, float, geometry)
DECL(float, double, geometry)
DECL(double, double, geometry)
typedef std::complex<float> cf;
typedef std::complex<double> cd;
DECL(cf, float, mat<cf>)
DECL(cd, double, mat<cd>)
DECL(cf, float, sparse_mat<cf>)
DECL(cd, double, sparse_mat<cd>)
DECL(cf, float, geometry)
DECL(cd, double, geometry)
#undef DECL

template <class T, class S, class OP>
static int run(void *U_, int dim_y, int dim_x, int dim_z, int ufmt, const OP &A, const void *b_, int blen,
               const ref_opts *o, const void *Ut_, int utlen, int utfmt, int submat_mb, int vppc,
               ref_info *info, char *err, int errlen) {
	try {
		mat<T> U(dim_y, dim_x, dim_z, (mat_format)ufmt);
		fill(U, U_);
		mat<T> b(blen);
		fill(b, b_);
		bool same = (utlen == U.len);
		mat<T> Ut(same ? dim_y : utlen, same ? dim_x : 1, same ? dim_z : 1, (mat_format)utfmt);
		fill(Ut, Ut_);
		tval3_options<S> opts = to_opts<S>(o);
		tval3_info<S> r = tval3_cpu_3d(U, A, b, opts, Ut, submat_mb, vppc);
		from_info(r, info);
		std::memcpy(U_, U.data(), sizeof(T) * (size_t)U.len);
		return 0;
	} catch (const tval3_exception &e) {
		set_err(err, errlen, e.what());
		return 1;
	}
}

template <class T>
static void fill_sparse(sparse_mat<T> &A, const int *rptr, const int *rind, const void *rval,
                        const int *cptr, const int *cind, const void *cval) {
	std::memcpy(A.csr_ptr(), rptr, sizeof(int) * (A.dim_y + 1));
	std::memcpy(A.csr_ind(), rind, sizeof(int) * (size_t)A.nnz);
	std::memcpy(A.csr_val(), rval, sizeof(T) * (size_t)A.nnz);
	std::memcpy(A.csc_ptr(), cptr, sizeof(int) * (A.dim_x + 1));
	std::memcpy(A.csc_ind(), cind, sizeof(int) * (size_t)A.nnz);
	std::memcpy(A.csc_val(), cval, sizeof(T) * (size_t)A.nnz);
}

extern "C" {

int ref3d_dense(int dtype, void *U, int dim_y, int dim_x, int dim_z, int ufmt, const void *A_, int m, int n,
                int afmt, const void *b, int blen, const ref_opts *o, const void *Ut, int utlen, int utfmt,
                int submat_mb, int vppc, ref_info *info, char *err, int errlen) {
	if (dtype == 3 || dtype == 4) {   // complex<float> / complex<double> data
		if (dtype == 3) {
			mat<cf> A(m, n, (mat_format)afmt);
			fill(A, A_);
			return run<cf, float>(U, dim_y, dim_x, dim_z, ufmt, A, b, blen, o, Ut, utlen, utfmt, submat_mb, vppc, info, err, errlen);
		}
		mat<cd> A(m, n, (mat_format)afmt);
		fill(A, A_);
		return run<cd, double>(U, dim_y, dim_x, dim_z, ufmt, A, b, blen, o, Ut, utlen, utfmt, submat_mb, vppc, info, err, errlen);
	}
	if (dtype == 2) {
		mat<double> A(m, n, (mat_format)afmt);
		fill(A, A_);
		return run<double, double>(U, dim_y, dim_x, dim_z, ufmt, A, b, blen, o, Ut, utlen, utfmt, submat_mb, vppc, info, err, errlen);
	}
	mat<float> A(m, n, (mat_format)afmt);
	fill(A, A_);
	if (dtype == 0)
		return run<float, float>(U, dim_y, dim_x, dim_z, ufmt, A, b, blen, o, Ut, utlen, utfmt, submat_mb, vppc, info, err, errlen);
	return run<float, double>(U, dim_y, dim_x, dim_z, ufmt, A, b, blen, o, Ut, utlen, utfmt, submat_mb, vppc, info, err, errlen);
}

int ref3d_csr(int dtype, void *U, int dim_y, int dim_x, int dim_z, int ufmt, int m, int n, int nnz, int afmt,
              const int *rptr, const int *rind, const void *rval, const int *cptr, const int *cind,
              const void *cval, const void *b, int blen, const ref_opts *o, const void *Ut, int utlen,
              int utfmt, int submat_mb, int vppc, ref_info *info, char *err, int errlen) {
	if (dtype == 3) {
		sparse_mat<cf> A(m, n, nnz, (sparse_mat_format)afmt);
		fill_sparse(A, rptr, rind, rval, cptr, cind, cval);
		return run<cf, float>(U, dim_y, dim_x, dim_z, ufmt, A, b, blen, o, Ut, utlen, utfmt, submat_mb, vppc, info, err, errlen);
	}
	if (dtype == 4) {
		sparse_mat<cd> A(m, n, nnz, (sparse_mat_format)afmt);
		fill_sparse(A, rptr, rind, rval, cptr, cind, cval);
		return run<cd, double>(U, dim_y, dim_x, dim_z, ufmt, A, b, blen, o, Ut, utlen, utfmt, submat_mb, vppc, info, err, errlen);
	}
	if (dtype == 2) {
		sparse_mat<double> A(m, n, nnz, (sparse_mat_format)afmt);
		fill_sparse(A, rptr, rind, rval, cptr, cind, cval);
		return run<double, double>(U, dim_y, dim_x, dim_z, ufmt, A, b, blen, o, Ut, utlen, utfmt, submat_mb, vppc, info, err, errlen);
	}
	sparse_mat<float> A(m, n, nnz, (sparse_mat_format)afmt);
	fill_sparse(A, rptr, rind, rval, cptr, cind, cval);
	if (dtype == 0)
		return run<float, float>(U, dim_y, dim_x, dim_z, ufmt, A, b, blen, o, Ut, utlen, utfmt, submat_mb, vppc, info, err, errlen);
	return run<float, double>(U, dim_y, dim_x, dim_z, ufmt, A, b, blen, o, Ut, utlen, utfmt, submat_mb, vppc, info, err, errlen);
}

/* Coordinates are passed flattened: xe[mp*E + e], xr[mp*R + r]. */
int ref3d_ray(int dtype, void *U, int dim_y, int dim_x, int dim_z, int ufmt, int numMPs, int numPaths,
              int E, int R, const int *use_path, int *xe, int *ye, int *ze, int *xr, int *yr, int *zr,
              int rv_x, int rv_y, int rv_z, float scale, const void *b, int blen, const ref_opts *o,
              const void *Ut, int utlen, int utfmt, int submat_mb, int vppc, ref_info *info, char *err,
              int errlen) {
	std::vector<int *> pxe(numMPs), pye(numMPs), pze(numMPs), pxr(numMPs), pyr(numMPs), pzr(numMPs);
	for (int i = 0; i < numMPs; i++) {
		pxe[i] = xe + (size_t)i * E; pye[i] = ye + (size_t)i * E; pze[i] = ze + (size_t)i * E;
		pxr[i] = xr + (size_t)i * R; pyr[i] = yr + (size_t)i * R; pzr[i] = zr + (size_t)i * R;
	}
	geometry g;
	g.numMPs = numMPs; g.numPaths = numPaths; g.num_emitters = E; g.num_receivers = R;
	g.use_path = use_path;
	g.x_emitters = &pxe[0]; g.y_emitters = &pye[0]; g.z_emitters = &pze[0];
	g.x_receivers = &pxr[0]; g.y_receivers = &pyr[0]; g.z_receivers = &pzr[0];
	g.rv_x = rv_x; g.rv_y = rv_y; g.rv_z = rv_z; g.scale_factor = scale;
	if (dtype == 0)
		return run<float, float>(U, dim_y, dim_x, dim_z, ufmt, g, b, blen, o, Ut, utlen, utfmt, submat_mb, vppc, info, err, errlen);
	if (dtype == 1)
		return run<float, double>(U, dim_y, dim_x, dim_z, ufmt, g, b, blen, o, Ut, utlen, utfmt, submat_mb, vppc, info, err, errlen);
	if (dtype == 3)
		return run<cf, float>(U, dim_y, dim_x, dim_z, ufmt, g, b, blen, o, Ut, utlen, utfmt, submat_mb, vppc, info, err, errlen);
	if (dtype == 4)
		return run<cd, double>(U, dim_y, dim_x, dim_z, ufmt, g, b, blen, o, Ut, utlen, utfmt, submat_mb, vppc, info, err, errlen);
	return run<double, double>(U, dim_y, dim_x, dim_z, ufmt, g, b, blen, o, Ut, utlen, utfmt, submat_mb, vppc, info, err, errlen);
}

}
