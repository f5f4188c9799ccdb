/*
 * Oracle (test infrastructure only): C entry points around the reference's
 * 2D overloads tval3_cpu_2d (2d/tval3_cpu_2d.cpp:16-95,889-1016).  The
 * overloads are re-declared here exactly as the reference declares them and
 * resolved at link time against the reference's own object file.
 */
#include <complex>
#include <cstring>
#include <string>
#include "container.h"
#include "tval3_types.h"
#include "ref_capi.h"

extern const tval3_info<float> tval3_cpu_2d(mat<float> &U, const mat<float> &A, const mat<float> &b,
		const tval3_options<float> &opts, const mat<float> &Ut, int submat_mb, int vppc) throw(tval3_exception);
extern const tval3_info<double> tval3_cpu_2d(mat<float> &U, const mat<float> &A, const mat<float> &b,
		const tval3_options<double> &opts, const mat<float> &Ut, int submat_mb, int vppc) throw(tval3_exception);
extern const tval3_info<double> tval3_cpu_2d(mat<double> &U, const mat<double> &A, const mat<double> &b,
		const tval3_options<double> &opts, const mat<double> &Ut, int submat_mb, int vppc) throw(tval3_exception);
extern const tval3_info<float> tval3_cpu_2d(mat<float> &U, const sparse_mat<float> &A, const mat<float> &b,
		const tval3_options<float> &opts, const mat<float> &Ut, int submat_mb, int vppc) throw(tval3_exception);
extern const tval3_info<double> tval3_cpu_2d(mat<float> &U, const sparse_mat<float> &A, const mat<float> &b,
		const tval3_options<double> &opts, const mat<float> &Ut, int submat_mb, int vppc) throw(tval3_exception);
extern const tval3_info<double> tval3_cpu_2d(mat<double> &U, const sparse_mat<double> &A, const mat<double> &b,
		const tval3_options<double> &opts, const mat<double> &Ut, int submat_mb, int vppc) throw(tval3_exception);
typedef std::complex<float> cf;
typedef std::complex<double> cd;
extern const tval3_info<float> tval3_cpu_2d(mat<cf> &U, const mat<cf> &A, const mat<cf> &b,
		const tval3_options<float> &opts, const mat<cf> &Ut, int submat_mb, int vppc) throw(tval3_exception);
extern const tval3_info<double> tval3_cpu_2d(mat<cd> &U, const mat<cd> &A, const mat<cd> &b,
		const tval3_options<double> &opts, const mat<cd> &Ut, int submat_mb, int vppc) throw(tval3_exception);
extern const tval3_info<float> tval3_cpu_2d(mat<cf> &U, const sparse_mat<cf> &A, const mat<cf> &b,
		const tval3_options<float> &opts, const mat<cf> &Ut, int submat_mb, int vppc) throw(tval3_exception);
extern const tval3_info<double> tval3_cpu_2d(mat<cd> &U, const sparse_mat<cd> &A, const mat<cd> &b,
		const tval3_options<double> &opts, const mat<cd> &Ut, int submat_mb, int vppc) throw(tval3_exception);

template <class T, class S, class OP>
static int run(void *U_, int dim_y, int dim_x, int ufmt, const OP &A, const void *b_, int blen,
               const ref_opts *o, const void *Ut_, int utlen, int utfmt, int submat_mb, int vppc,
               ref_info *info, char *err, int errlen) {
	try {
		mat<T> U(dim_y, dim_x, (mat_format)ufmt);
		fill(U, U_);
		mat<T> b(blen);
		fill(b, b_);
		mat<T> Ut(utlen == U.len ? dim_y : utlen, utlen == U.len ? dim_x : 1, (mat_format)utfmt);
		fill(Ut, Ut_);
		tval3_options<S> opts = to_opts<S>(o);
		tval3_info<S> r = tval3_cpu_2d(U, A, b, opts, Ut, submat_mb, vppc);
		from_info(r, info);
		std::memcpy(U_, U.data(), sizeof(T) * (size_t)U.len);
		return 0;
	} catch (const tval3_exception &e) {
		set_err(err, errlen, e.what());
		return 1;
	}
}

template <class T, class S>
static int dense(void *U, int dim_y, int dim_x, int ufmt, const void *A_, int m, int n, int afmt,
                 const void *b, int blen, const ref_opts *o, const void *Ut, int utlen, int utfmt,
                 int submat_mb, int vppc, ref_info *info, char *err, int errlen) {
	mat<T> A(m, n, (mat_format)afmt);
	fill(A, A_);
	return run<T, S>(U, dim_y, dim_x, ufmt, A, b, blen, o, Ut, utlen, utfmt, submat_mb, vppc, info, err, errlen);
}

template <class T, class S>
static int sparse(void *U, int dim_y, int dim_x, int ufmt, int m, int n, int nnz, int afmt,
                  const int *rptr, const int *rind, const void *rval, const int *cptr, const int *cind,
                  const void *cval, const void *b, int blen, const ref_opts *o, const void *Ut, int utlen,
                  int utfmt, int submat_mb, int vppc, ref_info *info, char *err, int errlen) {
	sparse_mat<T> A(m, n, nnz, (sparse_mat_format)afmt);
	std::memcpy(A.csr_ptr(), rptr, sizeof(int) * (m + 1));
	std::memcpy(A.csr_ind(), rind, sizeof(int) * (size_t)nnz);
	std::memcpy(A.csr_val(), rval, sizeof(T) * (size_t)nnz);
	std::memcpy(A.csc_ptr(), cptr, sizeof(int) * (n + 1));
	std::memcpy(A.csc_ind(), cind, sizeof(int) * (size_t)nnz);
	std::memcpy(A.csc_val(), cval, sizeof(T) * (size_t)nnz);
	return run<T, S>(U, dim_y, dim_x, ufmt, A, b, blen, o, Ut, utlen, utfmt, submat_mb, vppc, info, err, errlen);
}

extern "C" {

int ref2d_dense(int dtype, void *U, int dim_y, int dim_x, int ufmt, const void *A, int m, int n, int afmt,
                const void *b, int blen, const ref_opts *o, const void *Ut, int utlen, int utfmt, int submat_mb,
                int vppc, ref_info *info, char *err, int errlen) {
	if (dtype == 0) return dense<float, float>(U, dim_y, dim_x, ufmt, A, m, n, afmt, b, blen, o, Ut, utlen, utfmt, submat_mb, vppc, info, err, errlen);
	if (dtype == 1) return dense<float, double>(U, dim_y, dim_x, ufmt, A, m, n, afmt, b, blen, o, Ut, utlen, utfmt, submat_mb, vppc, info, err, errlen);
	if (dtype == 3) return dense<cf, float>(U, dim_y, dim_x, ufmt, A, m, n, afmt, b, blen, o, Ut, utlen, utfmt, submat_mb, vppc, info, err, errlen);
	if (dtype == 4) return dense<cd, double>(U, dim_y, dim_x, ufmt, A, m, n, afmt, b, blen, o, Ut, utlen, utfmt, submat_mb, vppc, info, err, errlen);
	return dense<double, double>(U, dim_y, dim_x, ufmt, A, m, n, afmt, b, blen, o, Ut, utlen, utfmt, submat_mb, vppc, info, err, errlen);
}

int ref2d_csr(int dtype, void *U, int dim_y, int dim_x, int ufmt, int m, int n, int nnz, int afmt,
              const int *rptr, const int *rind, const void *rval, const int *cptr, const int *cind,
              const void *cval, const void *b, int blen, const ref_opts *o, const void *Ut, int utlen,
              int utfmt, int submat_mb, int vppc, ref_info *info, char *err, int errlen) {
	if (dtype == 0) return sparse<float, float>(U, dim_y, dim_x, ufmt, m, n, nnz, afmt, rptr, rind, rval, cptr, cind, cval, b, blen, o, Ut, utlen, utfmt, submat_mb, vppc, info, err, errlen);
	if (dtype == 1) return sparse<float, double>(U, dim_y, dim_x, ufmt, m, n, nnz, afmt, rptr, rind, rval, cptr, cind, cval, b, blen, o, Ut, utlen, utfmt, submat_mb, vppc, info, err, errlen);
	if (dtype == 3) return sparse<cf, float>(U, dim_y, dim_x, ufmt, m, n, nnz, afmt, rptr, rind, rval, cptr, cind, cval, b, blen, o, Ut, utlen, utfmt, submat_mb, vppc, info, err, errlen);
	if (dtype == 4) return sparse<cd, double>(U, dim_y, dim_x, ufmt, m, n, nnz, afmt, rptr, rind, rval, cptr, cind, cval, b, blen, o, Ut, utlen, utfmt, submat_mb, vppc, info, err, errlen);
	return sparse<double, double>(U, dim_y, dim_x, ufmt, m, n, nnz, afmt, rptr, rind, rval, cptr, cind, cval, b, blen, o, Ut, utlen, utfmt, submat_mb, vppc, info, err, errlen);
}

}
