/*
 * Drop-in replacement of modk/tval3-cpu's 3D entry points on a B200.
 *
 * The 15 overloads below are those the reference declares and exports
 * (3d/tval3_cpu_3d.cpp:32-146, defined at :1384-1581), with the same names,
 * argument types and defaults, so existing callers relink against
 * libtval3_gpu_3d.so (which exports the same C++ symbols) without source
 * changes.  Each forwards to tval3g_solve or, for double data,
 * tval3g_solve_f64 (include/tval3g.h).
 *
 * Differences from the reference:
 *   - float and complex<float> data run on the FP32 engine (FP32 storage,
 *     FP64 reductions: closer to the reference's double build than the
 *     reference's own float build is); double and complex<double> data run
 *     on the FP64 engine (tval3g_solve_f64: double storage and arithmetic,
 *     as the reference's double instantiations compute), held to the
 *     reference's double builds in tests/test_gpu_f64.py;
 *   - submat_mb and virtual_procs_per_core are accepted and ignored (they
 *     tune the reference's CPU cache blocking and thread count);
 *   - ray endpoints outside the volume are rejected with an argument error
 *     instead of being read out of bounds; nothing is printed and no
 *     profile.txt is written (the reference does both on every call,
 *     3d/tval3_cpu_3d.cpp:1228,1328-1349);
 *   - tval3_options::tv_norm selects isotropic TV (the reference computes
 *     anisotropic TV only).
 * Argument errors are thrown as tval3_exception with the reference's messages.
 */
#ifndef TVAL3_GPU_3D_H_
#define TVAL3_GPU_3D_H_

#include <complex>

#include "tval3/container.h"
#include "tval3/geometry_3d.h"
#include "tval3/tval3_types.h"

const tval3_info<float> tval3_cpu_3d(mat<float> &U, const mat<float> &A, const mat<float> &b,
                                     const tval3_options<float> &opts, const mat<float> &Ut,
                                     int submat_mb = 5, int virtual_procs_per_core = 2);
const tval3_info<double> tval3_cpu_3d(mat<float> &U, const mat<float> &A, const mat<float> &b,
                                      const tval3_options<double> &opts, const mat<float> &Ut,
                                      int submat_mb = 5, int virtual_procs_per_core = 2);
const tval3_info<double> tval3_cpu_3d(mat<double> &U, const mat<double> &A, const mat<double> &b,
                                      const tval3_options<double> &opts, const mat<double> &Ut,
                                      int submat_mb = 5, int virtual_procs_per_core = 2);
const tval3_info<float> tval3_cpu_3d(mat<std::complex<float> > &U, const mat<std::complex<float> > &A,
                                     const mat<std::complex<float> > &b, const tval3_options<float> &opts,
                                     const mat<std::complex<float> > &Ut, int submat_mb = 5,
                                     int virtual_procs_per_core = 2);
const tval3_info<double> tval3_cpu_3d(mat<std::complex<double> > &U, const mat<std::complex<double> > &A,
                                      const mat<std::complex<double> > &b, const tval3_options<double> &opts,
                                      const mat<std::complex<double> > &Ut, int submat_mb = 5,
                                      int virtual_procs_per_core = 2);

const tval3_info<float> tval3_cpu_3d(mat<float> &U, const sparse_mat<float> &A, const mat<float> &b,
                                     const tval3_options<float> &opts, const mat<float> &Ut,
                                     int submat_mb = 5, int virtual_procs_per_core = 2);
const tval3_info<double> tval3_cpu_3d(mat<float> &U, const sparse_mat<float> &A, const mat<float> &b,
                                      const tval3_options<double> &opts, const mat<float> &Ut,
                                      int submat_mb = 5, int virtual_procs_per_core = 2);
const tval3_info<double> tval3_cpu_3d(mat<double> &U, const sparse_mat<double> &A, const mat<double> &b,
                                      const tval3_options<double> &opts, const mat<double> &Ut,
                                      int submat_mb = 5, int virtual_procs_per_core = 2);
const tval3_info<float> tval3_cpu_3d(mat<std::complex<float> > &U, const sparse_mat<std::complex<float> > &A,
                                     const mat<std::complex<float> > &b, const tval3_options<float> &opts,
                                     const mat<std::complex<float> > &Ut, int submat_mb = 5,
                                     int virtual_procs_per_core = 2);
const tval3_info<double> tval3_cpu_3d(mat<std::complex<double> > &U, const sparse_mat<std::complex<double> > &A,
                                      const mat<std::complex<double> > &b, const tval3_options<double> &opts,
                                      const mat<std::complex<double> > &Ut, int submat_mb = 5,
                                      int virtual_procs_per_core = 2);

const tval3_info<float> tval3_cpu_3d(mat<float> &U, const geometry &A, const mat<float> &b,
                                     const tval3_options<float> &opts, const mat<float> &Ut,
                                     int submat_mb = 5, int virtual_procs_per_core = 2);
const tval3_info<double> tval3_cpu_3d(mat<float> &U, const geometry &A, const mat<float> &b,
                                      const tval3_options<double> &opts, const mat<float> &Ut,
                                      int submat_mb = 5, int virtual_procs_per_core = 2);
const tval3_info<double> tval3_cpu_3d(mat<double> &U, const geometry &A, const mat<double> &b,
                                      const tval3_options<double> &opts, const mat<double> &Ut,
                                      int submat_mb = 5, int virtual_procs_per_core = 2);
const tval3_info<float> tval3_cpu_3d(mat<std::complex<float> > &U, const geometry &A,
                                     const mat<std::complex<float> > &b, const tval3_options<float> &opts,
                                     const mat<std::complex<float> > &Ut, int submat_mb = 5,
                                     int virtual_procs_per_core = 2);
const tval3_info<double> tval3_cpu_3d(mat<std::complex<double> > &U, const geometry &A,
                                      const mat<std::complex<double> > &b, const tval3_options<double> &opts,
                                      const mat<std::complex<double> > &Ut, int submat_mb = 5,
                                      int virtual_procs_per_core = 2);

#endif /* TVAL3_GPU_3D_H_ */
