/* Oracle shim (test infrastructure only): the subset of Intel MKL's CBLAS
 * interface that the reference calls (2d/blas_wrap.h, 3d/blas_wrap.h).
 * MKL itself is absent from this image and its version is not pinned by the
 * reference; oracle/shim/mkl_shim.cpp implements these entry points with
 * plain loops that follow the documented BLAS semantics. */
#ifndef ORACLE_SHIM_MKL_CBLAS_H_
#define ORACLE_SHIM_MKL_CBLAS_H_
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif
typedef int MKL_INT;
typedef struct { float real, imag; } MKL_Complex8;
typedef struct { double real, imag; } MKL_Complex16;
typedef enum { CblasRowMajor = 101, CblasColMajor = 102 } CBLAS_ORDER;
typedef CBLAS_ORDER CBLAS_LAYOUT;
typedef enum { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 } CBLAS_TRANSPOSE;

void cblas_sscal(MKL_INT N, float alpha, float *X, MKL_INT incX);
void cblas_dscal(MKL_INT N, double alpha, double *X, MKL_INT incX);
void cblas_cscal(MKL_INT N, const void *alpha, void *X, MKL_INT incX);
void cblas_zscal(MKL_INT N, const void *alpha, void *X, MKL_INT incX);
void cblas_csscal(MKL_INT N, float alpha, void *X, MKL_INT incX);
void cblas_zdscal(MKL_INT N, double alpha, void *X, MKL_INT incX);

void cblas_saxpy(MKL_INT N, float alpha, const float *X, MKL_INT incX, float *Y, MKL_INT incY);
void cblas_daxpy(MKL_INT N, double alpha, const double *X, MKL_INT incX, double *Y, MKL_INT incY);
void cblas_caxpy(MKL_INT N, const void *alpha, const void *X, MKL_INT incX, void *Y, MKL_INT incY);
void cblas_zaxpy(MKL_INT N, const void *alpha, const void *X, MKL_INT incX, void *Y, MKL_INT incY);

void cblas_scopy(MKL_INT N, const float *X, MKL_INT incX, float *Y, MKL_INT incY);
void cblas_dcopy(MKL_INT N, const double *X, MKL_INT incX, double *Y, MKL_INT incY);
void cblas_ccopy(MKL_INT N, const void *X, MKL_INT incX, void *Y, MKL_INT incY);
void cblas_zcopy(MKL_INT N, const void *X, MKL_INT incX, void *Y, MKL_INT incY);

float cblas_sdot(MKL_INT N, const float *X, MKL_INT incX, const float *Y, MKL_INT incY);
double cblas_ddot(MKL_INT N, const double *X, MKL_INT incX, const double *Y, MKL_INT incY);
void cblas_cdotc_sub(MKL_INT N, const void *X, MKL_INT incX, const void *Y, MKL_INT incY, void *dotc);
void cblas_zdotc_sub(MKL_INT N, const void *X, MKL_INT incX, const void *Y, MKL_INT incY, void *dotc);

float cblas_snrm2(MKL_INT N, const float *X, MKL_INT incX);
double cblas_dnrm2(MKL_INT N, const double *X, MKL_INT incX);
float cblas_scnrm2(MKL_INT N, const void *X, MKL_INT incX);
double cblas_dznrm2(MKL_INT N, const void *X, MKL_INT incX);

void cblas_sgemv(CBLAS_ORDER order, CBLAS_TRANSPOSE TransA, MKL_INT M, MKL_INT N, float alpha,
                 const float *A, MKL_INT lda, const float *X, MKL_INT incX, float beta, float *Y, MKL_INT incY);
void cblas_dgemv(CBLAS_ORDER order, CBLAS_TRANSPOSE TransA, MKL_INT M, MKL_INT N, double alpha,
                 const double *A, MKL_INT lda, const double *X, MKL_INT incX, double beta, double *Y, MKL_INT incY);
void cblas_cgemv(CBLAS_ORDER order, CBLAS_TRANSPOSE TransA, MKL_INT M, MKL_INT N, const void *alpha,
                 const void *A, MKL_INT lda, const void *X, MKL_INT incX, const void *beta, void *Y, MKL_INT incY);
void cblas_zgemv(CBLAS_ORDER order, CBLAS_TRANSPOSE TransA, MKL_INT M, MKL_INT N, const void *alpha,
                 const void *A, MKL_INT lda, const void *X, MKL_INT incX, const void *beta, void *Y, MKL_INT incY);

void cblas_sgemm(CBLAS_ORDER Order, CBLAS_TRANSPOSE TransA, CBLAS_TRANSPOSE TransB, MKL_INT M, MKL_INT N, MKL_INT K,
                 float alpha, const float *A, MKL_INT lda, const float *B, MKL_INT ldb, float beta, float *C, MKL_INT ldc);
void cblas_dgemm(CBLAS_ORDER Order, CBLAS_TRANSPOSE TransA, CBLAS_TRANSPOSE TransB, MKL_INT M, MKL_INT N, MKL_INT K,
                 double alpha, const double *A, MKL_INT lda, const double *B, MKL_INT ldb, double beta, double *C, MKL_INT ldc);
void cblas_cgemm(CBLAS_ORDER Order, CBLAS_TRANSPOSE TransA, CBLAS_TRANSPOSE TransB, MKL_INT M, MKL_INT N, MKL_INT K,
                 const void *alpha, const void *A, MKL_INT lda, const void *B, MKL_INT ldb, const void *beta, void *C, MKL_INT ldc);
void cblas_zgemm(CBLAS_ORDER Order, CBLAS_TRANSPOSE TransA, CBLAS_TRANSPOSE TransB, MKL_INT M, MKL_INT N, MKL_INT K,
                 const void *alpha, const void *A, MKL_INT lda, const void *B, MKL_INT ldb, const void *beta, void *C, MKL_INT ldc);
#ifdef __cplusplus
}
#endif
#endif
