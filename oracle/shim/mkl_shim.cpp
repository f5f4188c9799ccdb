/*
 * Oracle shim (test infrastructure only): stand-in for the Intel MKL routines
 * the reference calls.  MKL is not in this image and the reference pins no
 * version, so these are plain loops that follow the documented BLAS / NIST
 * sparse BLAS semantics.  They are parallelised with OpenMP over the thread
 * count set by mkl_set_num_threads (the reference sets it to
 * omp_get_num_procs()/virtual_procs_per_core, 2d/tval3_cpu_2d.cpp:765), so a
 * timed reference run uses the host's cores as MKL would.
 *
 * Rounding choices (MKL's exact summation order is unknown):
 *   ?dot / ?dotc accumulate in the data type, 8 interleaved lanes per thread
 *   (like a SIMD BLAS kernel); ?nrm2 accumulates the sum of squares in double.
 */
#include <omp.h>
#include <cmath>
#include <complex>
#include <cstring>
#include <vector>

#include "mkl.h"

namespace {

int g_threads = 0;

int nthreads() { return g_threads > 0 ? g_threads : omp_get_max_threads(); }

/* minimum length before a level-1 loop is split across threads */
const long PAR_MIN = 1 << 15;

template <class T> T conj_(const T &v) { return v; }
template <class T> std::complex<T> conj_(const std::complex<T> &v) { return std::conj(v); }
template <class T> double abs2(const T &v) { return (double)v * (double)v; }
template <class T> double abs2(const std::complex<T> &v) {
	return (double)v.real() * v.real() + (double)v.imag() * v.imag();
}

template <class T> void scal(long n, T a, T *x, long inc) {
#pragma omp parallel for num_threads(nthreads()) if (n > PAR_MIN)
	for (long i = 0; i < n; i++) x[i * inc] *= a;
}
template <class S, class T> void scal_real(long n, S a, T *x, long inc) {
#pragma omp parallel for num_threads(nthreads()) if (n > PAR_MIN)
	for (long i = 0; i < n; i++) x[i * inc] *= a;
}
template <class T> void axpy(long n, T a, const T *x, long incx, T *y, long incy) {
#pragma omp parallel for num_threads(nthreads()) if (n > PAR_MIN)
	for (long i = 0; i < n; i++) y[i * incy] += a * x[i * incx];
}
template <class T> void copy(long n, const T *x, long incx, T *y, long incy) {
#pragma omp parallel for num_threads(nthreads()) if (n > PAR_MIN)
	for (long i = 0; i < n; i++) y[i * incy] = x[i * incx];
}

/* sum_i conj(x_i) * y_i, accumulated in T with 8 lanes per thread */
template <class T> T dotc(long n, const T *x, long incx, const T *y, long incy) {
	int nt = n > PAR_MIN ? nthreads() : 1;
	std::vector<T> part(nt, T(0));
#pragma omp parallel num_threads(nt)
	{
		int t = omp_get_thread_num();
		long lo = n * t / nt, hi = n * (t + 1) / nt;
		T lane[8];
		for (int l = 0; l < 8; l++) lane[l] = T(0);
		for (long i = lo; i < hi; i++) lane[(i - lo) & 7] += conj_(x[i * incx]) * y[i * incy];
		T s = T(0);
		for (int l = 0; l < 8; l++) s += lane[l];
		part[t] = s;
	}
	T s = T(0);
	for (int t = 0; t < nt; t++) s += part[t];
	return s;
}

template <class T> double nrm2(long n, const T *x, long inc) {
	double s = 0;
#pragma omp parallel for reduction(+ : s) num_threads(nthreads()) if (n > PAR_MIN)
	for (long i = 0; i < n; i++) s += abs2(x[i * inc]);
	return std::sqrt(s);
}

/* y = alpha*op(A)*x + beta*y for a row- or column-major A of M x N */
template <class T>
void gemv(CBLAS_ORDER order, CBLAS_TRANSPOSE ta, long M, long N, T alpha, const T *A, long lda,
          const T *x, long incx, T beta, T *y, long incy) {
	/* reduce to row-major: a column-major A is the row-major transpose */
	bool trans = (ta != CblasNoTrans);
	bool conj = (ta == CblasConjTrans);
	if (order == CblasColMajor) {
		std::swap(M, N);
		trans = !trans;
	}
	/* now A is row-major M x N; op(A) = A or A^T (conjugated if conj) */
	if (!trans) {
#pragma omp parallel for num_threads(nthreads()) if (M * N > PAR_MIN)
		for (long i = 0; i < M; i++) {
			T s = T(0);
			const T *row = A + i * lda;
			for (long j = 0; j < N; j++) s += (conj ? conj_(row[j]) : row[j]) * x[j * incx];
			y[i * incy] = alpha * s + (beta == T(0) ? T(0) : beta * y[i * incy]);
		}
	} else {
		int nt = (M * N > PAR_MIN) ? nthreads() : 1;
		std::vector<T> acc((size_t)nt * N, T(0));
#pragma omp parallel num_threads(nt)
		{
			int t = omp_get_thread_num();
			long lo = M * t / nt, hi = M * (t + 1) / nt;
			T *a = &acc[(size_t)t * N];
			for (long i = lo; i < hi; i++) {
				const T *row = A + i * lda;
				T xi = x[i * incx];
				for (long j = 0; j < N; j++) a[j] += (conj ? conj_(row[j]) : row[j]) * xi;
			}
		}
#pragma omp parallel for num_threads(nthreads()) if (N > PAR_MIN)
		for (long j = 0; j < N; j++) {
			T s = T(0);
			for (int t = 0; t < nt; t++) s += acc[(size_t)t * N + j];
			y[j * incy] = alpha * s + (beta == T(0) ? T(0) : beta * y[j * incy]);
		}
	}
}

/* C = alpha*op(A)*op(B) + beta*C, all row-major (column-major is mapped onto
 * the row-major transpose problem C^T = op(B)^T op(A)^T). */
template <class T>
void gemm(CBLAS_ORDER order, CBLAS_TRANSPOSE ta, CBLAS_TRANSPOSE tb, long M, long N, long K, T alpha,
          const T *A, long lda, const T *B, long ldb, T beta, T *C, long ldc) {
	if (order == CblasColMajor) {
		gemm<T>(CblasRowMajor, tb, ta, N, M, K, alpha, B, ldb, A, lda, beta, C, ldc);
		return;
	}
#pragma omp parallel for num_threads(nthreads()) if (M * N * K > PAR_MIN)
	for (long i = 0; i < M; i++)
		for (long j = 0; j < N; j++) {
			T s = T(0);
			for (long k = 0; k < K; k++) {
				T a = (ta == CblasNoTrans) ? A[i * lda + k] : A[k * lda + i];
				if (ta == CblasConjTrans) a = conj_(a);
				T b = (tb == CblasNoTrans) ? B[k * ldb + j] : B[j * ldb + k];
				if (tb == CblasConjTrans) b = conj_(b);
				s += a * b;
			}
			C[i * ldc + j] = alpha * s + (beta == T(0) ? T(0) : beta * C[i * ldc + j]);
		}
}

int base_of(const char *descr) { return (descr[3] == 'F' || descr[3] == 'f') ? 1 : 0; }
bool is_trans(const char *t) { return *t != 'n' && *t != 'N'; }
bool is_conj(const char *t) { return *t == 'c' || *t == 'C'; }

/* Compressed-storage product.  "Row-compressed" storage of an R x Cc matrix
 * (rows rlen = R, stored lines over R): op == direct computes
 * y[line] = sum val*x[ind]; op == scatter computes y[ind] += val*x[line].
 * CSR is row-compressed; CSC is the row-compressed storage of A^T. */
template <class T>
void compressed_mv(bool gather, long lines, long outlen, const T *val, const int *ind,
                   const int *pb, const int *pe, int base, const T *x, T alpha, T beta, T *y,
                   bool conj) {
	if (gather) {
#pragma omp parallel for schedule(dynamic, 64) num_threads(nthreads()) if (lines > 1024)
		for (long i = 0; i < lines; i++) {
			T s = T(0);
			for (int p = pb[i] - base; p < pe[i] - base; p++)
				s += (conj ? conj_(val[p]) : val[p]) * x[ind[p] - base];
			y[i] = alpha * s + (beta == T(0) ? T(0) : beta * y[i]);
		}
	} else {
		int nt = lines > 1024 ? nthreads() : 1;
		std::vector<T> acc((size_t)nt * outlen, T(0));
#pragma omp parallel num_threads(nt)
		{
			int t = omp_get_thread_num();
			long lo = lines * t / nt, hi = lines * (t + 1) / nt;
			T *a = &acc[(size_t)t * outlen];
			for (long i = lo; i < hi; i++)
				for (int p = pb[i] - base; p < pe[i] - base; p++)
					a[ind[p] - base] += (conj ? conj_(val[p]) : val[p]) * x[i];
		}
#pragma omp parallel for num_threads(nthreads()) if (outlen > PAR_MIN)
		for (long j = 0; j < outlen; j++) {
			T s = T(0);
			for (int t = 0; t < nt; t++) s += acc[(size_t)t * outlen + j];
			y[j] = alpha * s + (beta == T(0) ? T(0) : beta * y[j]);
		}
	}
}

template <class T>
void csrmv(const char *ta, const int *m, const int *k, const T *alpha, const char *descr, const T *val,
           const int *ind, const int *pb, const int *pe, const T *x, const T *beta, T *y) {
	/* A: m x k in CSR (m compressed rows) */
	if (!is_trans(ta))
		compressed_mv<T>(true, *m, *m, val, ind, pb, pe, base_of(descr), x, *alpha, *beta, y, false);
	else
		compressed_mv<T>(false, *m, *k, val, ind, pb, pe, base_of(descr), x, *alpha, *beta, y, is_conj(ta));
}

template <class T>
void cscmv(const char *ta, const int *m, const int *k, const T *alpha, const char *descr, const T *val,
           const int *ind, const int *pb, const int *pe, const T *x, const T *beta, T *y) {
	/* A: m x k in CSC (k compressed columns) */
	if (!is_trans(ta))
		compressed_mv<T>(false, *k, *m, val, ind, pb, pe, base_of(descr), x, *alpha, *beta, y, false);
	else
		compressed_mv<T>(true, *k, *k, val, ind, pb, pe, base_of(descr), x, *alpha, *beta, y, is_conj(ta));
}

template <class T>
void cscmm(const char *ta, const int *m, const int *n, const int *k, const T *alpha, const char *descr,
           const T *val, const int *ind, const int *pb, const int *pe, const T *b, const int *ldb,
           const T *beta, T *c, const int *ldc) {
	/* A: m x k in CSC; B, C row-major with n columns (zero-based layout). */
	int base = base_of(descr);
	bool trans = is_trans(ta), conj = is_conj(ta);
	long outrows = trans ? *k : *m;
	for (long r = 0; r < outrows; r++)
		for (long j = 0; j < *n; j++)
			c[r * *ldc + j] = (*beta == T(0)) ? T(0) : *beta * c[r * *ldc + j];
	if (trans) {
#pragma omp parallel for num_threads(nthreads())
		for (long col = 0; col < *k; col++)
			for (int p = pb[col] - base; p < pe[col] - base; p++) {
				T a = conj ? conj_(val[p]) : val[p];
				long row = ind[p] - base;
				for (long j = 0; j < *n; j++) c[col * *ldc + j] += *alpha * a * b[row * *ldb + j];
			}
	} else {
		for (long col = 0; col < *k; col++)
			for (int p = pb[col] - base; p < pe[col] - base; p++) {
				long row = ind[p] - base;
				for (long j = 0; j < *n; j++) c[row * *ldc + j] += *alpha * val[p] * b[col * *ldb + j];
			}
	}
}

typedef std::complex<float> c8;
typedef std::complex<double> c16;

} // namespace

extern "C" {

void mkl_set_num_threads(int nt) { g_threads = nt > 0 ? nt : 1; }
int mkl_get_max_threads(void) { return nthreads(); }

void cblas_sscal(MKL_INT N, float a, float *X, MKL_INT inc) { scal<float>(N, a, X, inc); }
void cblas_dscal(MKL_INT N, double a, double *X, MKL_INT inc) { scal<double>(N, a, X, inc); }
void cblas_cscal(MKL_INT N, const void *a, void *X, MKL_INT inc) { scal<c8>(N, *(const c8 *)a, (c8 *)X, inc); }
void cblas_zscal(MKL_INT N, const void *a, void *X, MKL_INT inc) { scal<c16>(N, *(const c16 *)a, (c16 *)X, inc); }
void cblas_csscal(MKL_INT N, float a, void *X, MKL_INT inc) { scal_real<float, c8>(N, a, (c8 *)X, inc); }
void cblas_zdscal(MKL_INT N, double a, void *X, MKL_INT inc) { scal_real<double, c16>(N, a, (c16 *)X, inc); }

void cblas_saxpy(MKL_INT N, float a, const float *X, MKL_INT ix, float *Y, MKL_INT iy) { axpy<float>(N, a, X, ix, Y, iy); }
void cblas_daxpy(MKL_INT N, double a, const double *X, MKL_INT ix, double *Y, MKL_INT iy) { axpy<double>(N, a, X, ix, Y, iy); }
void cblas_caxpy(MKL_INT N, const void *a, const void *X, MKL_INT ix, void *Y, MKL_INT iy) {
	axpy<c8>(N, *(const c8 *)a, (const c8 *)X, ix, (c8 *)Y, iy);
}
void cblas_zaxpy(MKL_INT N, const void *a, const void *X, MKL_INT ix, void *Y, MKL_INT iy) {
	axpy<c16>(N, *(const c16 *)a, (const c16 *)X, ix, (c16 *)Y, iy);
}

void cblas_scopy(MKL_INT N, const float *X, MKL_INT ix, float *Y, MKL_INT iy) { copy<float>(N, X, ix, Y, iy); }
void cblas_dcopy(MKL_INT N, const double *X, MKL_INT ix, double *Y, MKL_INT iy) { copy<double>(N, X, ix, Y, iy); }
void cblas_ccopy(MKL_INT N, const void *X, MKL_INT ix, void *Y, MKL_INT iy) { copy<c8>(N, (const c8 *)X, ix, (c8 *)Y, iy); }
void cblas_zcopy(MKL_INT N, const void *X, MKL_INT ix, void *Y, MKL_INT iy) { copy<c16>(N, (const c16 *)X, ix, (c16 *)Y, iy); }

float cblas_sdot(MKL_INT N, const float *X, MKL_INT ix, const float *Y, MKL_INT iy) { return dotc<float>(N, X, ix, Y, iy); }
double cblas_ddot(MKL_INT N, const double *X, MKL_INT ix, const double *Y, MKL_INT iy) { return dotc<double>(N, X, ix, Y, iy); }
void cblas_cdotc_sub(MKL_INT N, const void *X, MKL_INT ix, const void *Y, MKL_INT iy, void *r) {
	*(c8 *)r = dotc<c8>(N, (const c8 *)X, ix, (const c8 *)Y, iy);
}
void cblas_zdotc_sub(MKL_INT N, const void *X, MKL_INT ix, const void *Y, MKL_INT iy, void *r) {
	*(c16 *)r = dotc<c16>(N, (const c16 *)X, ix, (const c16 *)Y, iy);
}

float cblas_snrm2(MKL_INT N, const float *X, MKL_INT inc) { return (float)nrm2<float>(N, X, inc); }
double cblas_dnrm2(MKL_INT N, const double *X, MKL_INT inc) { return nrm2<double>(N, X, inc); }
float cblas_scnrm2(MKL_INT N, const void *X, MKL_INT inc) { return (float)nrm2<c8>(N, (const c8 *)X, inc); }
double cblas_dznrm2(MKL_INT N, const void *X, MKL_INT inc) { return nrm2<c16>(N, (const c16 *)X, inc); }

void cblas_sgemv(CBLAS_ORDER o, CBLAS_TRANSPOSE t, MKL_INT M, MKL_INT N, float a, const float *A, MKL_INT lda,
                 const float *X, MKL_INT ix, float b, float *Y, MKL_INT iy) {
	gemv<float>(o, t, M, N, a, A, lda, X, ix, b, Y, iy);
}
void cblas_dgemv(CBLAS_ORDER o, CBLAS_TRANSPOSE t, MKL_INT M, MKL_INT N, double a, const double *A, MKL_INT lda,
                 const double *X, MKL_INT ix, double b, double *Y, MKL_INT iy) {
	gemv<double>(o, t, M, N, a, A, lda, X, ix, b, Y, iy);
}
void cblas_cgemv(CBLAS_ORDER o, CBLAS_TRANSPOSE t, MKL_INT M, MKL_INT N, const void *a, const void *A, MKL_INT lda,
                 const void *X, MKL_INT ix, const void *b, void *Y, MKL_INT iy) {
	gemv<c8>(o, t, M, N, *(const c8 *)a, (const c8 *)A, lda, (const c8 *)X, ix, *(const c8 *)b, (c8 *)Y, iy);
}
void cblas_zgemv(CBLAS_ORDER o, CBLAS_TRANSPOSE t, MKL_INT M, MKL_INT N, const void *a, const void *A, MKL_INT lda,
                 const void *X, MKL_INT ix, const void *b, void *Y, MKL_INT iy) {
	gemv<c16>(o, t, M, N, *(const c16 *)a, (const c16 *)A, lda, (const c16 *)X, ix, *(const c16 *)b, (c16 *)Y, iy);
}

void cblas_sgemm(CBLAS_ORDER o, CBLAS_TRANSPOSE ta, CBLAS_TRANSPOSE tb, MKL_INT M, MKL_INT N, MKL_INT K, float a,
                 const float *A, MKL_INT lda, const float *B, MKL_INT ldb, float b, float *C, MKL_INT ldc) {
	gemm<float>(o, ta, tb, M, N, K, a, A, lda, B, ldb, b, C, ldc);
}
void cblas_dgemm(CBLAS_ORDER o, CBLAS_TRANSPOSE ta, CBLAS_TRANSPOSE tb, MKL_INT M, MKL_INT N, MKL_INT K, double a,
                 const double *A, MKL_INT lda, const double *B, MKL_INT ldb, double b, double *C, MKL_INT ldc) {
	gemm<double>(o, ta, tb, M, N, K, a, A, lda, B, ldb, b, C, ldc);
}
void cblas_cgemm(CBLAS_ORDER o, CBLAS_TRANSPOSE ta, CBLAS_TRANSPOSE tb, MKL_INT M, MKL_INT N, MKL_INT K,
                 const void *a, const void *A, MKL_INT lda, const void *B, MKL_INT ldb, const void *b, void *C,
                 MKL_INT ldc) {
	gemm<c8>(o, ta, tb, M, N, K, *(const c8 *)a, (const c8 *)A, lda, (const c8 *)B, ldb, *(const c8 *)b, (c8 *)C, ldc);
}
void cblas_zgemm(CBLAS_ORDER o, CBLAS_TRANSPOSE ta, CBLAS_TRANSPOSE tb, MKL_INT M, MKL_INT N, MKL_INT K,
                 const void *a, const void *A, MKL_INT lda, const void *B, MKL_INT ldb, const void *b, void *C,
                 MKL_INT ldc) {
	gemm<c16>(o, ta, tb, M, N, K, *(const c16 *)a, (const c16 *)A, lda, (const c16 *)B, ldb, *(const c16 *)b,
	          (c16 *)C, ldc);
}

#define ORACLE_SPBLAS_DEF(P, T, CT)                                                                         \
	void mkl_##P##csrmv(const char *ta, const MKL_INT *m, const MKL_INT *k, const T *alpha, const char *d,  \
	                    const T *val, const MKL_INT *ind, const MKL_INT *pb, const MKL_INT *pe, const T *x, \
	                    const T *beta, T *y) {                                                              \
		csrmv<CT>(ta, m, k, (const CT *)alpha, d, (const CT *)val, ind, pb, pe, (const CT *)x,              \
		          (const CT *)beta, (CT *)y);                                                               \
	}                                                                                                       \
	void mkl_##P##cscmv(const char *ta, const MKL_INT *m, const MKL_INT *k, const T *alpha, const char *d,  \
	                    const T *val, const MKL_INT *ind, const MKL_INT *pb, const MKL_INT *pe, const T *x, \
	                    const T *beta, T *y) {                                                              \
		cscmv<CT>(ta, m, k, (const CT *)alpha, d, (const CT *)val, ind, pb, pe, (const CT *)x,              \
		          (const CT *)beta, (CT *)y);                                                               \
	}                                                                                                       \
	void mkl_##P##cscmm(const char *ta, const MKL_INT *m, const MKL_INT *n, const MKL_INT *k,              \
	                    const T *alpha, const char *d, const T *val, const MKL_INT *ind, const MKL_INT *pb, \
	                    const MKL_INT *pe, const T *b, const MKL_INT *ldb, const T *beta, T *c,             \
	                    const MKL_INT *ldc) {                                                               \
		cscmm<CT>(ta, m, n, k, (const CT *)alpha, d, (const CT *)val, ind, pb, pe, (const CT *)b, ldb,      \
		          (const CT *)beta, (CT *)c, ldc);                                                          \
	}
ORACLE_SPBLAS_DEF(s, float, float)
ORACLE_SPBLAS_DEF(d, double, double)
ORACLE_SPBLAS_DEF(c, MKL_Complex8, c8)
ORACLE_SPBLAS_DEF(z, MKL_Complex16, c16)

} // extern "C"
