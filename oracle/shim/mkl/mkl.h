/* Oracle shim (test infrastructure only): MKL's umbrella header, reduced to
 * what the reference uses: the CBLAS / sparse BLAS subsets and
 * mkl_set_num_threads (2d/tval3_cpu_2d.cpp:765). */
#ifndef ORACLE_SHIM_MKL_H_
#define ORACLE_SHIM_MKL_H_
#include "mkl_cblas.h"
#include "mkl_spblas.h"
#ifdef __cplusplus
extern "C" {
#endif
void mkl_set_num_threads(int nt);
int mkl_get_max_threads(void);
#ifdef __cplusplus
}
#endif
#endif
