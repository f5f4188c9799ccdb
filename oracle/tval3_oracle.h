/*
 * TVAL3 oracle: a plain-C FP64 restatement of the reference solver, used ONLY
 * as a checker by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
 * leg.  Nothing in the product path links or calls it.
 *
 * It follows modk/tval3-cpu's 2d/tval3_cpu_2d.cpp and 3d/tval3_cpu_3d.cpp line
 * by line (each function cites the lines it restates) and adds what the
 * reference cannot run:
 *   - the 2D Bresenham projector, whose reference body is commented out
 *     (2d/mat_mult.h:109-194); restated from that commented code;
 *   - isotropic shrinkage, which the reference does not have (restated from
 *     the TVAL3 mathematics, selected by tv_norm = 1).
 * Its aniso results are pinned against the reference itself, built from its
 * own sources in oracle/_ref (tests/test_oracle_vs_reference.py).
 */
#ifndef TVAL3_ORACLE_H_
#define TVAL3_ORACLE_H_

#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_DENSE = 0, ORC_CSR = 1, ORC_RAY2D = 2, ORC_RAY3D = 3 };

typedef struct orc_op orc_op;

typedef struct {
	double mu, beta, mu0, beta0, tol, tol_inn, c, gamma, gam, rate_gam, rate_cnt;
	double skipMulRatio, maxRelativeChange;
	int maxit, maxcnt, nonneg, isreal, numInitIterations, tv_norm;
	/* 1: complex data as two planes (the reference's complex<T> overloads,
	 * 2d/tval3_cpu_2d.cpp:913-929): U, b and every vector hold the real
	 * plane then the imaginary plane, the operator is the caller's real form
	 * [[Re A, -Im A], [Im A, Re A]] (its transpose is A^H), D and Dt act per
	 * plane, the shrinkage takes each gradient component's complex modulus
	 * (2d:614-649; 3D with the reference's z quirk, 3d/tval3_cpu_3d.cpp:934-937),
	 * scaleb complex moduli (2d:229-266), nonneg Re >= 0 and Im = 0
	 * (2d:467-479), isreal keeps the real plane (2d:855-859).  Anisotropic
	 * TV only (the reference has no other). */
	int cplx;
	/* > 0: a model of FP32 storage for the checker's noise floor - after each
	 * inner iteration's descent, every element of U, its differences, Au, g
	 * and g2 is multiplied by 1 + noise * xi, xi uniform in [-1, 1] from a
	 * xorshift64 stream seeded by noise_seed.  0 (the default): none. */
	double noise;
	unsigned long long noise_seed;
} orc_opts;

typedef struct {
	double secs, rel_chg, rel_error;
	int outer_iters, total_iters;
} orc_info;

/* Per inner iteration record (optional): tau, f after update_W, RelChg, the
 * number of backtracking steps (6 = restart after 5 failures), whether the
 * descent step skipped the A^T multiplication and whether the inner loop
 * ended after the iteration. */
typedef struct {
	double tau, f, relchg;
	int backtracks;
	int skipped;
	int inner_end;
	int pad;
} orc_iter;

/* Operators (all arrays are copied). */
orc_op *orc_op_dense(int m, int n, int layers, const double *A);
orc_op *orc_op_csr(int m, int n, int layers, int nnz, const int *rowptr, const int *colind,
                   const double *val);
orc_op *orc_op_ray2d(int E, int R, const int *use_path, const int *xe, const int *ye,
                     const int *xr, const int *yr, int ld, double scale, int n_pixels);
orc_op *orc_op_ray3d(int numMPs, int numPaths, int E, int R, const int *use_path,
                     const int *xe, const int *ye, const int *ze, const int *xr, const int *yr,
                     const int *zr, int rv_x, int rv_y, int rv_z, double scale);
void orc_op_free(orc_op *op);
int orc_op_rows(const orc_op *op);   /* y length of A*x */
int orc_op_cols(const orc_op *op);   /* x length of A*x */

/* y = A x (trans = 0) or y = A^T x (trans = 1), y overwritten. */
void orc_apply(const orc_op *op, int trans, const double *x, double *y);

/* Bresenham pixel / voxel lists of a ray operator, following the sequential
 * recurrence of 2d/mat_mult.h:145-181 and 3d/mat_mult.h:205-359.  For every
 * traced ray in the reference's loop order, writes its measurement index to
 * ray_index[k], the start of its list to offsets[k] (offsets[count] = total)
 * and the linear indices to pix[].  With pix == NULL only counts.
 * Returns the number of traced rays; *total receives the number of hits. */
int orc_ray_lists(const orc_op *op, int *ray_index, long *offsets, int *pix, long *total);

/* Finite differences (periodic) and their reference adjoints on an image of
 * dim_y x dim_x (x dim_z, 3D when dim_z > 0 is passed with dims = 3). */
void orc_D(int dims, int p, int q, int r, const double *U, double *Ux, double *Uy, double *Uz);
void orc_Dt(int dims, int p, int q, int r, const double *X, const double *Y, const double *Z,
            double *res);

/* Shrinkage of (Ux,Uy[,Uz]) - sigma/beta; returns lambda1. */
double orc_shrink(int dims, int n, int tv_norm, double beta, const double *Ux, const double *Uy,
                  const double *Uz, const double *sx, const double *sy, const double *sz, double *Wx,
                  double *Wy, double *Wz);

/* The solve.  dims = 2 or 3; U is dim_y*dim_x(*dim_z) and is overwritten.
 * Ut may be NULL.  iters may be NULL, else it holds room for opts->maxit
 * records.  Returns 0, or a negative code for argument errors. */
int orc_solve(int dims, int dim_y, int dim_x, int dim_z, const orc_op *op, const double *b, int blen,
              const orc_opts *opts, const double *Ut, double *U, orc_info *info, orc_iter *iters);

/* Decisions recorded by another solver (for example the GPU's per-iteration
 * trace), replayed by orc_solve_replay so that the FP64 solve takes the same
 * discrete path: per iteration k < count, the backtracking steps (0-5, or 6 =
 * five and the restart), whether the descent skipped the A^T multiplication
 * (-1: the heuristic decides) and whether the inner loop ended after it
 * (inner_end[k] = 1: multipliers and continuation updated next).  The solve
 * stops after `count` iterations; it then also updates the multipliers if
 * inner_end[count - 1] says so.  This replaces the Armijo test, the skip
 * heuristic and the inner / outer stopping tests of 2d:790-853; everything
 * continuous (step lengths, objective, vectors) is computed in FP64 as in
 * orc_solve.  A test-only device: it lets an FP32 solve be compared with the
 * FP64 one at the same iteration count and decisions. */
typedef struct {
	int count;
	const int *backtracks;
	const int *skipped;
	const int *inner_end;
} orc_replay;

int orc_solve_replay(int dims, int dim_y, int dim_x, int dim_z, const orc_op *op, const double *b, int blen,
                     const orc_opts *opts, const double *Ut, double *U, orc_info *info, orc_iter *iters,
                     const orc_replay *replay);

#ifdef __cplusplus
}
#endif
#endif
