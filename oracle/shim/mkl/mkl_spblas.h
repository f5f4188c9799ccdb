/* Oracle shim (test infrastructure only): the NIST-style sparse BLAS entry
 * points of Intel MKL that the reference calls (2d/blas_wrap.h:182-281,
 * 3d/blas_wrap.h:542-791).  Semantics implemented in oracle/shim/mkl_shim.cpp:
 *   ?csrmv / ?cscmv: y = alpha*op(A)*x + beta*y, A is m x k (rows x columns)
 *   in CSR / CSC with pointerB/pointerE arrays;
 *   ?cscmm: C = alpha*op(A)*B + beta*C with B, C row-major (zero-based);
 *   matdescra[0] must be 'G' (general), matdescra[3] 'C' (zero-based) or
 *   'F' (one-based); transa 'n'/'N', 't'/'T' or 'c'/'C'. */
#ifndef ORACLE_SHIM_MKL_SPBLAS_H_
#define ORACLE_SHIM_MKL_SPBLAS_H_
#include "mkl_cblas.h"
#ifdef __cplusplus
extern "C" {
#endif
#define ORACLE_SPBLAS_DECL(P, T)                                                              \
	void mkl_##P##csrmv(const char *transa, const MKL_INT *m, const MKL_INT *k, const T *alpha,  \
	                    const char *matdescra, const T *val, const MKL_INT *indx,                 \
	                    const MKL_INT *pntrb, const MKL_INT *pntre, const T *x, const T *beta,    \
	                    T *y);                                                                    \
	void mkl_##P##cscmv(const char *transa, const MKL_INT *m, const MKL_INT *k, const T *alpha,  \
	                    const char *matdescra, const T *val, const MKL_INT *indx,                 \
	                    const MKL_INT *pntrb, const MKL_INT *pntre, const T *x, const T *beta,    \
	                    T *y);                                                                    \
	void mkl_##P##cscmm(const char *transa, const MKL_INT *m, const MKL_INT *n, const MKL_INT *k, \
	                    const T *alpha, const char *matdescra, const T *val, const MKL_INT *indx, \
	                    const MKL_INT *pntrb, const MKL_INT *pntre, const T *b, const MKL_INT *ldb,\
	                    const T *beta, T *c, const MKL_INT *ldc);
ORACLE_SPBLAS_DECL(s, float)
ORACLE_SPBLAS_DECL(d, double)
ORACLE_SPBLAS_DECL(c, MKL_Complex8)
ORACLE_SPBLAS_DECL(z, MKL_Complex16)
#undef ORACLE_SPBLAS_DECL
#ifdef __cplusplus
}
#endif
#endif
