/*
 * tval3g — TVAL3 total-variation reconstruction on one NVIDIA B200 (sm_100a).
 *
 * C ABI of the solver core (libtval3g.so).  Plain C types only; every pointer
 * is a host pointer unless the function or flag says "device".  All entry
 * points return TVAL3G_OK (0) or a negative status; tval3g_last_error()
 * returns the calling thread's last message.
 *
 * The C++ drop-in overloads tval3_cpu_2d / tval3_cpu_3d (include/tval3_gpu_2d.h,
 * include/tval3_gpu_3d.h) forward to tval3g_solve.  What each entry point
 * replaces in modk/tval3-cpu:
 *
 *   tval3g_solve        the 15 + 15 overloads tval3_cpu_2d (2d/tval3_cpu_2d.cpp:16-95,
 *                       889-1016) and tval3_cpu_3d (3d/tval3_cpu_3d.cpp:32-146,
 *                       1384-1581) for float data, through the templated driver
 *                       (2d/tval3_cpu_2d.cpp:752-886, 3d/tval3_cpu_3d.cpp:1172-1378)
 *   tval3g_solve_f64    the same overloads for double and complex<double> data
 *                       (the driver's double instantiations), solved in double
 *   tval3g_solve_batch  no reference counterpart: many independent solves in one
 *                       batched launch sequence (each one as tval3g_solve)
 *   tval3g_plan_*       no reference counterpart: the same solves with device-
 *                       resident operators, data and state, reusable
 *   tval3g_op_*         the measurement operator gemv(TransA, A, x, y) overloads
 *                       (2d/mat_mult.h:15-194, 3d/mat_mult.h:17-595)
 *   tval3g_D / _Dt      D / Dt (2d/tval3_cpu_2d.cpp:268-293, 3d/tval3_cpu_3d.cpp:365-425)
 *   tval3g_shrink       shrinkage (2d/tval3_cpu_2d.cpp:588-611, 3d/tval3_cpu_3d.cpp:834-871)
 *   tval3g_unrolled_*   no reference counterpart: gradients of an unrolled K-iteration
 *                       solve (2d/tval3_cpu_2d.cpp:752-853 with decisions held fixed)
 */
#ifndef TVAL3G_H_
#define TVAL3G_H_

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define TVAL3G_OK 0
#define TVAL3G_ERR_ARGUMENT -1   /* the reference would throw "Argument error: ..." */
#define TVAL3G_ERR_CUDA -2       /* a CUDA call failed (message says which) */
#define TVAL3G_ERR_NO_DEVICE -3  /* no usable CUDA device / extension */
#define TVAL3G_ERR_NONFINITE -4  /* a non-finite step length or objective stopped a solve */
#define TVAL3G_ERR_INTERNAL -5

/* measurement operator kinds (2d/mat_mult.h, 3d/mat_mult.h) */
#define TVAL3G_OP_DENSE 0  /* mat<T>: row-major m x n */
#define TVAL3G_OP_CSR 1    /* sparse_mat<T>: CSR, 0-based int32; the transpose is built on the device */
#define TVAL3G_OP_RAY2D 2  /* 2D geometry: on-the-fly Bresenham rays */
#define TVAL3G_OP_RAY3D 3  /* 3D geometry: on-the-fly Bresenham rays */

/* total-variation norm */
#define TVAL3G_TV_ANISO 0  /* the reference's (only) norm */
#define TVAL3G_TV_ISO 1

/* flags of tval3g_plan_create / tval3g_solve_batch */
#define TVAL3G_DEVICE_INPUTS 1  /* A / CSR arrays of the problems are device pointers */
#define TVAL3G_GRAPH 2          /* run the iteration loop as one CUDA graph with
                                   conditional nodes (no host round trips) */
#define TVAL3G_TRACE 4          /* record one tval3g_trace_record per inner
                                   iteration on the device (tval3g_plan_trace) */
#define TVAL3G_NO_TENSOR 8      /* dense operators with 16, 32, 48 or 64 layers
                                   use the FP64-accumulating gemv kernels instead
                                   of the tcgen05 3xTF32 tensor-core path */
#define TVAL3G_TUNE 16          /* time each operator's launch-shape candidates
                                   once (lanes per ray of the ray forward,
                                   sub-warp width of the compressed gathers)
                                   and keep the fastest; cached per operator
                                   signature in memory and, if the environment
                                   variable TVAL3G_TUNE_CACHE names a file, on
                                   disk.  Results then equal the untuned ones
                                   within rounding (other summation order). */
#define TVAL3G_RAY_ADJ_PLAIN 64    /* ray operators: the plain pixel-major gather
                                   adjoint (4-byte traced-ray ids per hit,
                                   measurements gathered from L2) instead of
                                   the tiled one (2D: 16 x 16 pixel tiles; 3D:
                                   8 x 8 x 4 voxel bricks; each tile's rays'
                                   measurements staged in shared memory and
                                   16-bit positions per hit).  A comparison
                                   form; results equal within rounding. */
#define TVAL3G_RAY_ADJ_ATOMICS 32  /* ray operators: the adjoint traces the rays
                                   on the fly and accumulates into the image
                                   with atomic adds (no pixel-major index),
                                   instead of the pixel-major gather; sums are
                                   then not bit-reproducible (the order of the
                                   atomic adds varies).  A comparison form:
                                   the gather is the default because it
                                   measured faster (and is deterministic). */

/* Per inner iteration: step length, objective after update_W, relative
 * change, backtracking steps taken (6 = restart after five failures), whether
 * the A^T multiplication was skipped (skipMulRatio heuristic), when the
 * solve was given Ut, ||U/scl - Ut|| / ||Ut|| after the iteration (else 0),
 * the step actually taken (U = U_prev - step * d: tau times the backtracking
 * factor, or the restart's tau) and whether the multipliers were updated
 * after the iteration (1) or not (0). */
typedef struct tval3g_trace_record {
	double tau, f, relchg, backtracks, skipped, relerr_ut, step, outer;
} tval3g_trace_record;

/* Options; field meaning as tval3_options<T> (include/tval3/tval3_types.h). */
typedef struct tval3g_options {
	double mu, beta, mu0, beta0, tol, tol_inn, c, gamma, gam, rate_gam, rate_cnt;
	double skipMulRatio, maxRelativeChange;
	int maxit, maxcnt, nonneg, isreal, numInitIterations, tv_norm;
} tval3g_options;

/* Result of one solve; fields as tval3_info<T> plus a per-solve status. */
typedef struct tval3g_info {
	double secs;      /* wall seconds of the call (batch: of the whole batch) */
	double rel_chg;   /* last outer relative change */
	double rel_error; /* ||Ut - U|| / ||Ut|| when Ut was given, else 0 */
	int outer_iters;
	int total_iters;
	int status;       /* TVAL3G_OK or TVAL3G_ERR_NONFINITE */
	int reserved;
} tval3g_info;

/* One reconstruction problem.
 * Image: dims = 2 (dim_z = 1) or 3; element i = x + y*dim_x + z*dim_x*dim_y.
 * n = dim_y*dim_x*dim_z.
 * DENSE / CSR: m = rows of A (A.dim_y), n_cols = columns (A.dim_x), layers =
 *   the reference's "layers" (2d/tval3_cpu_2d.cpp:894: b.len / A.dim_y; 3D
 *   always 1); valid when n == n_cols*layers and b_len == m*layers.
 * RAY2D: b_len = num_emitters*num_receivers (uncompacted; 2d/tval3_cpu_2d.cpp:748).
 * RAY3D: b_len = numPaths*numMPs (3d/tval3_cpu_3d.cpp:1153).
 * Ray coordinate arrays are host pointers; emitters [numMPs*E], receivers
 * [numMPs*R] (2D: numMPs = 1, z arrays unused). */
typedef struct tval3g_problem {
	int dims;
	int dim_y, dim_x, dim_z;
	int op_kind;
	int m;                          /* DENSE / CSR: rows of A (A.dim_y) */
	int n_cols;                     /* DENSE / CSR: columns of A (A.dim_x) */
	int layers;
	const float *A;                 /* DENSE */
	long long nnz;                  /* CSR */
	const int *csr_ptr;             /* [m+1] */
	const int *csr_ind;             /* [nnz] column (pixel) indices */
	const float *csr_val;           /* [nnz] */
	int num_emitters, num_receivers;/* RAY2D / RAY3D */
	int numMPs, numPaths;           /* RAY3D */
	const int *use_path;            /* [E*R] */
	const int *x_emitters, *y_emitters, *z_emitters;
	const int *x_receivers, *y_receivers, *z_receivers;
	int ld;                         /* RAY2D row stride of the image */
	int rv_x, rv_y, rv_z;           /* RAY3D volume extent */
	float scale_factor;             /* RAY2D / RAY3D weight of one hit */
	/* 1: complex data (the reference's complex<float> overloads,
	 * 2d/tval3_cpu_2d.cpp:913-929 and the sparse / geometry ones): b, Ut and
	 * U hold interleaved (re, im) float pairs (b_len, ut_len and n count
	 * complex elements), as do DENSE A and CSR csr_val; the adjoint is the
	 * conjugate transpose.  2D (layers too) and 3D; host operator arrays. */
	int complex_data;
} tval3g_problem;

const char *tval3g_last_error(void);
int tval3g_version(void);

/* One solve with host buffers (the drop-in path): U (n floats, output),
 * b (b_len floats), Ut (ut_len floats: 0 or n; may be NULL).  With the
 * environment variable TVAL3G_TUNE=1 its operator is built with the
 * autotuner (TVAL3G_TUNE). */
int tval3g_solve(const tval3g_problem *prob, const float *b, int b_len, const tval3g_options *opts,
                 const float *Ut, int ut_len, float *U, tval3g_info *info);

/* One solve in double precision with host buffers: the FP64 build of the
 * engine (double vectors, double operator values and products, double
 * stencils and shrinkage; the same kernels' algorithm as tval3g_solve, with
 * the pixel-major gather adjoint for ray operators and the gemv kernels for
 * dense ones; the autotuner, TVAL3G_TUNE, does not apply).  prob describes the problem as for tval3g_solve except that
 * its float arrays A and csr_val are not read: A64 holds the dense matrix
 * (DENSE: m x n_cols row-major) or the CSR values (CSR: nnz of them), and is
 * NULL for ray geometries; b (b_len), Ut (ut_len: 0 or n; may be NULL) and U
 * (n, output) are doubles.  With complex_data = 1 every one of these arrays
 * holds interleaved (re, im) double pairs, and the lengths count complex
 * elements.  Replaces the double and complex<double> instantiations of the
 * drivers (2d/tval3_cpu_2d.cpp:905-1016, 3d/tval3_cpu_3d.cpp:1408-1581),
 * which compute in double. */
int tval3g_solve_f64(const tval3g_problem *prob, const double *A64, const double *b, int b_len,
                     const tval3g_options *opts, const double *Ut, int ut_len, double *U, tval3g_info *info);

/* count independent solves with host buffers, run as one batch (flags:
 * TVAL3G_GRAPH, TVAL3G_TUNE).  Arrays are indexed by problem; Ut may be NULL. */
int tval3g_solve_batch(int count, const tval3g_problem *probs, const float *const *b,
                       const tval3g_options *opts, const float *const *Ut, float *const *U,
                       tval3g_info *info, int flags);

/* Plans: operators prepared once on the device (dense A copied or borrowed,
 * CSR transpose built, ray index built), solver state allocated once.
 * tval3g_plan_solve takes DEVICE pointers for b, Ut (may be NULL) and U and
 * runs on `stream` (a cudaStream_t, or NULL for the plan's own stream); it
 * returns after the solve finished and info was filled. */
typedef struct tval3g_plan tval3g_plan;
int tval3g_plan_create(tval3g_plan **plan, int count, const tval3g_problem *probs,
                       const tval3g_options *opts, int flags);
int tval3g_plan_solve(tval3g_plan *plan, const float *const *d_b, const float *const *d_Ut,
                      float *const *d_U, tval3g_info *info, void *stream);
/* Kernel launches issued by the last tval3g_plan_solve (graph mode: kernel
 * nodes executed, counted on the device), and the plan's device bytes. */
int tval3g_plan_stats(const tval3g_plan *plan, long long *kernel_launches, long long *device_bytes);
/* Measurement: the mean device time in ms of one launch of each of the
 * iteration's image-sized vector kernels over all instances - ms[0] the
 * gradient epilogue (g -= Atb, D U, the objective's sums), ms[1] the descent
 * (U = U - tau d with the snapshot of the previous iterate), ms[2] the
 * shrinkage with Dt(DU - W), d and the step-length sums - each launched reps
 * times back to back on the plan's stream after a solve.  It overwrites the
 * plan's state (the next solve starts afresh).  No counterpart in the
 * reference. */
int tval3g_plan_time_stencils(tval3g_plan *plan, int reps, double *ms);
/* Time-to-solution mode: with target > 0, every instance solved with a Ut
 * also stops after the first inner iteration at which
 * ||U/scl - Ut|| <= target * ||Ut|| (checked on the device each iteration);
 * info.rel_error then reports that value.  target = 0 restores the
 * reference's stopping rules only.  No counterpart in the reference. */
int tval3g_plan_set_target(tval3g_plan *plan, double target);
/* Trace of instance `index` of the last solve of a plan created with
 * TVAL3G_TRACE: copies up to `cap` records to out, *count = records written. */
int tval3g_plan_trace(const tval3g_plan *plan, int index, tval3g_trace_record *out, int cap, int *count);
int tval3g_plan_destroy(tval3g_plan *plan);

/* Device memory of plans, operators and their one-time builders comes from a
 * stream-ordered pool of the library (one per device), which keeps freed
 * blocks for the next solve.  tval3g_trim_memory returns the current device's
 * cached blocks beyond keep_bytes to the driver.  No counterpart in the
 * reference (it allocates host memory per call). */
int tval3g_trim_memory(long long keep_bytes);

/* Autotuner (TVAL3G_TUNE): operators timed, and choices taken from the cache,
 * in this process so far.  No counterpart in the reference. */
int tval3g_tune_stats(long long *measured, long long *cached);

/* Operators alone.  tval3g_op_apply: y = A x (trans = 0), y = A^T x
 * (trans = 1) or the normal product y = A^T (A x) of the solve's get_g_mult
 * (trans = 2; a one-layer dense operator reads A once, as the reference's
 * cache-blocked dense path, 2d/tval3_cpu_2d.cpp:361-394) with DEVICE x, y
 * (lengths rows/cols as reported; both cols for trans = 2). */
typedef struct tval3g_operator tval3g_operator;
int tval3g_op_create(tval3g_operator **op, const tval3g_problem *prob, int flags);
int tval3g_op_shape(const tval3g_operator *op, long long *rows, long long *cols, long long *nnz);
int tval3g_op_apply(tval3g_operator *op, int trans, const float *d_x, float *d_y, void *stream);
/* The same product `reps` times, enqueued back to back on `stream` (the
 * result is that of one application); returns without waiting, so events
 * recorded around it on the stream time the kernels alone. */
int tval3g_op_apply_n(tval3g_operator *op, int trans, const float *d_x, float *d_y, int reps, void *stream);
/* Ray operators: the device-built CSR (rows = b_len, untraced rows empty) of
 * the Bresenham rasterisation, copied to HOST arrays rowptr [rows+1] and
 * colind [nnz]; with colind == NULL only rowptr is written. */
int tval3g_op_ray_csr(const tval3g_operator *op, long long *rowptr, int *colind);
/* Bytes of the index that one adjoint application (y = A^T x) reads besides
 * x and y: the device-built CSC of a sparse operator, the pixel-major ray
 * index of a ray operator (for 2D rays: the tile lists, the per-pixel 16-bit
 * positions and their offsets), 0 for a dense operator.  No counterpart in
 * the reference (its operators keep no derived index). */
int tval3g_op_adjoint_index_bytes(const tval3g_operator *op, long long *bytes);
/* The operator's launch shapes (tval3g_op_create with TVAL3G_TUNE): lanes per
 * ray of the ray forward and 1 + the width class (4, 8, 16, 32 lanes per
 * line) of the forward and adjoint gathers; 0 = the built-in choice.  No
 * counterpart in the reference. */
int tval3g_op_launch_shape(const tval3g_operator *op, int *fwd_lanes, int *gather_fwd, int *gather_adj);
int tval3g_op_destroy(tval3g_operator *op);

/* Stencils on DEVICE arrays of an image dim_y x dim_x (x dim_z for dims 3).
 * Dt reproduces the reference's 3D adjoint exactly (including the extra y term
 * on the first row of every slice z >= 1, 3d/tval3_cpu_3d.cpp:402-413). */
int tval3g_D(int dims, int dim_y, int dim_x, int dim_z, const float *U, float *Ux, float *Uy,
             float *Uz, void *stream);
int tval3g_Dt(int dims, int dim_y, int dim_x, int dim_z, const float *X, const float *Y,
              const float *Z, float *res, void *stream);
/* W = shrink(U_c - sigma_c/beta); returns lambda1 in *lam1 (host). */
int tval3g_shrink(int dims, long long n, int tv_norm, double beta, const float *Ux, const float *Uy,
                  const float *Uz, const float *sx, const float *sy, const float *sz, float *Wx,
                  float *Wy, float *Wz, double *lam1, void *stream);

/* Differentiable unrolled solve (2D, one layer, no nonnegativity).  No
 * counterpart in the reference.  `count` instances share the operator of
 * `prob` and the options; the solve runs exactly K inner iterations with
 * per-iteration (mu_k, beta_k) instead of the continuation.  The forward
 * records, per instance and iteration, the step taken (BB step length times
 * the Armijo backtracking factor) and whether the multipliers were updated,
 * then replays the iteration map with those decisions held fixed, keeping a
 * checkpoint every `ckpt` iterations; U = U_K / scl (DEVICE, count x n).
 * The backward gives, for DEVICE cotangents gU (count x n), the gradients of
 * sum_i <gU_i, U_i>: gb (DEVICE, count x m) and g_mu, g_beta (HOST, K each,
 * summed over the instances), recomputing each segment from its checkpoint.
 * d_b / d_U / d_gU / d_gb are arrays of `count` device pointers. */
typedef struct tval3g_unrolled tval3g_unrolled;
int tval3g_unrolled_create(tval3g_unrolled **h, const tval3g_problem *prob, int count,
                           const tval3g_options *opts, int K, int ckpt);
int tval3g_unrolled_forward(tval3g_unrolled *h, const float *const *d_b, const double *mu,
                            const double *beta, float *const *d_U, void *stream);
int tval3g_unrolled_backward(tval3g_unrolled *h, const float *const *d_gU, float *const *d_gb,
                             double *g_mu, double *g_beta, void *stream);
/* the recorded decisions of instance `index`: steps[K], outer[K], scl */
int tval3g_unrolled_decisions(const tval3g_unrolled *h, int index, double *steps, int *outer, double *scl);
int tval3g_unrolled_destroy(tval3g_unrolled *h);

/* Seeded Gaussian streams (no counterpart in the reference; its callers
 * bring their own data): out[i] = scale * z(seed, offset + i) for i < count,
 * z a standard normal value from the counter-based Philox-4x32-10 generator
 * with a Box-Muller transform in FP64, rounded to FP32.  tval3g_gaussian
 * writes DEVICE memory on `stream` (stream-ordered); tval3g_gaussian_host
 * computes the same stream on the host.  The integer streams are identical;
 * an element may differ by one FP32 unit in the last place between the two
 * when the math libraries' FP64 log / sin / cos round differently. */
int tval3g_gaussian(unsigned long long seed, unsigned long long offset, long long count, float scale,
                    float *d_out, void *stream);
int tval3g_gaussian_host(unsigned long long seed, unsigned long long offset, long long count, float scale,
                         float *out);

/* y = A^T x for a dense row-major m x n float matrix, with DEVICE pointers,
 * for callers that cannot allocate device memory at call time (for example
 * when another allocator has reserved the device's memory, or when a
 * cudaMalloc's synchronisation is not acceptable).  It allocates nothing: its
 * partial-sum scratch is a fixed 4 MiB array compiled into the library, so n
 * may be at most 1048576 (larger n is rejected with TVAL3G_ERR_ARGUMENT).
 * A device holds that array once the library's device code is loaded onto
 * it: under CUDA's default lazy module loading that is this entry point's
 * first call on the device, which therefore takes the 4 MiB (and the code)
 * from the device - make that first call at start-up, before another
 * allocator reserves the memory, or set CUDA_MODULE_LOADING=EAGER.  The first
 * call on each device also looks up the array's device address; make it
 * before any stream capture begins.  All calls share the array: calls whose
 * work overlaps on the GPU race.  Stream-ordered: the call returns once the
 * work is enqueued on `stream` (NULL: the legacy default stream), and y is
 * complete when the stream reaches that point.  Same arithmetic as
 * tval3g_op_apply's dense adjoint (FP64 accumulation).
 * No counterpart in the reference (it has no device code). */
int tval3g_dense_adjoint_static(const float *d_A, int m, int n, const float *d_x, float *d_y, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* TVAL3G_H_ */
