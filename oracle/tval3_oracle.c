/*
 * TVAL3 oracle (test infrastructure only; see tval3_oracle.h).
 *
 * FP64 restatement of modk/tval3-cpu.  Reference lines are cited per function
 * as 2d:<line> = 2d/tval3_cpu_2d.cpp, 3d:<line> = 3d/tval3_cpu_3d.cpp,
 * 2d/mat_mult.h:<line>, 3d/mat_mult.h:<line>.
 */
#include "tval3_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <sys/time.h>

struct orc_op {
	int kind;
	int m, n, layers;
	/* dense */
	double *A;
	/* csr (and its transpose, built here) */
	int nnz;
	int *rowptr, *colind;
	double *val;
	int *colptr, *rowind;
	double *cval;
	/* rays */
	int nmp, npaths, E, R;
	int *use_path;
	int *xe, *ye, *ze, *xr, *yr, *zr;
	int ld, rvx, rvy, rvz;
	double scale;
};

static void *dup(const void *src, size_t bytes) {
	void *p = malloc(bytes ? bytes : 1);
	if (src && bytes) memcpy(p, src, bytes);
	return p;
}

static double *zeros(long n) { return (double *)calloc(n > 0 ? n : 1, sizeof(double)); }
static void materialize_rays(orc_op *op);

orc_op *orc_op_dense(int m, int n, int layers, const double *A) {
	orc_op *op = (orc_op *)calloc(1, sizeof(orc_op));
	op->kind = ORC_DENSE; op->m = m; op->n = n; op->layers = layers < 1 ? 1 : layers;
	op->A = (double *)dup(A, sizeof(double) * (size_t)m * n);
	return op;
}

orc_op *orc_op_csr(int m, int n, int layers, int nnz, const int *rowptr, const int *colind,
                   const double *val) {
	orc_op *op = (orc_op *)calloc(1, sizeof(orc_op));
	op->kind = ORC_CSR; op->m = m; op->n = n; op->layers = layers < 1 ? 1 : layers; op->nnz = nnz;
	op->rowptr = (int *)dup(rowptr, sizeof(int) * (m + 1));
	op->colind = (int *)dup(colind, sizeof(int) * (size_t)nnz);
	op->val = (double *)dup(val, sizeof(double) * (size_t)nnz);
	/* column-compressed copy, rows ascending within a column */
	op->colptr = (int *)calloc(n + 1, sizeof(int));
	op->rowind = (int *)malloc(sizeof(int) * (nnz ? nnz : 1));
	op->cval = (double *)malloc(sizeof(double) * (nnz ? nnz : 1));
	for (int k = 0; k < nnz; k++) op->colptr[colind[k] + 1]++;
	for (int j = 0; j < n; j++) op->colptr[j + 1] += op->colptr[j];
	int *next = (int *)dup(op->colptr, sizeof(int) * (n + 1));
	for (int i = 0; i < m; i++)
		for (int k = rowptr[i]; k < rowptr[i + 1]; k++) {
			int p = next[colind[k]]++;
			op->rowind[p] = i;
			op->cval[p] = val[k];
		}
	free(next);
	return op;
}

orc_op *orc_op_ray2d(int E, int R, const int *use_path, const int *xe, const int *ye,
                     const int *xr, const int *yr, int ld, double scale, int n_pixels) {
	orc_op *op = (orc_op *)calloc(1, sizeof(orc_op));
	op->kind = ORC_RAY2D; op->E = E; op->R = R; op->nmp = 1; op->layers = 1;
	op->use_path = (int *)dup(use_path, sizeof(int) * (size_t)E * R);
	op->xe = (int *)dup(xe, sizeof(int) * E); op->ye = (int *)dup(ye, sizeof(int) * E);
	op->xr = (int *)dup(xr, sizeof(int) * R); op->yr = (int *)dup(yr, sizeof(int) * R);
	op->ld = ld; op->scale = scale;
	op->m = E * R;       /* uncompacted, 2d:748 */
	op->n = n_pixels;    /* the image is the caller's: 2d/mat_mult.h has no size */
	materialize_rays(op);
	return op;
}

orc_op *orc_op_ray3d(int numMPs, int numPaths, int E, int R, const int *use_path,
                     const int *xe, const int *ye, const int *ze, const int *xr, const int *yr,
                     const int *zr, int rv_x, int rv_y, int rv_z, double scale) {
	orc_op *op = (orc_op *)calloc(1, sizeof(orc_op));
	op->kind = ORC_RAY3D; op->nmp = numMPs; op->npaths = numPaths; op->E = E; op->R = R; op->layers = 1;
	op->use_path = (int *)dup(use_path, sizeof(int) * (size_t)E * R);
	op->xe = (int *)dup(xe, sizeof(int) * (size_t)numMPs * E);
	op->ye = (int *)dup(ye, sizeof(int) * (size_t)numMPs * E);
	op->ze = (int *)dup(ze, sizeof(int) * (size_t)numMPs * E);
	op->xr = (int *)dup(xr, sizeof(int) * (size_t)numMPs * R);
	op->yr = (int *)dup(yr, sizeof(int) * (size_t)numMPs * R);
	op->zr = (int *)dup(zr, sizeof(int) * (size_t)numMPs * R);
	op->rvx = rv_x; op->rvy = rv_y; op->rvz = rv_z; op->scale = scale;
	op->m = numPaths * numMPs;           /* 3d:1153 */
	op->n = rv_x * rv_y * rv_z;
	materialize_rays(op);
	return op;
}

/* Rasterise every traced ray once with the sequential recurrence and keep the
 * result as row- and column-compressed index lists (rows = measurements), so
 * that applications are parallel loops.  Rays that share a measurement index
 * are concatenated in loop order, as the reference accumulates them. */
static void materialize_rays(orc_op *op) {
	long total = 0;
	int cnt = orc_ray_lists(op, NULL, NULL, NULL, &total);
	int *ray = (int *)malloc(sizeof(int) * (cnt ? cnt : 1));
	long *off = (long *)malloc(sizeof(long) * (cnt + 1));
	int *pix = (int *)malloc(sizeof(int) * (total ? total : 1));
	orc_ray_lists(op, ray, off, pix, &total);
	op->nnz = (int)total;
	op->rowptr = (int *)calloc(op->m + 1, sizeof(int));
	for (int k = 0; k < cnt; k++) op->rowptr[ray[k] + 1] += (int)(off[k + 1] - off[k]);
	for (int i = 0; i < op->m; i++) op->rowptr[i + 1] += op->rowptr[i];
	op->colind = (int *)malloc(sizeof(int) * (total ? total : 1));
	int *next = (int *)dup(op->rowptr, sizeof(int) * (op->m + 1));
	for (int k = 0; k < cnt; k++)
		for (long t = off[k]; t < off[k + 1]; t++) op->colind[next[ray[k]]++] = pix[t];
	free(next);
	op->colptr = (int *)calloc(op->n + 1, sizeof(int));
	op->rowind = (int *)malloc(sizeof(int) * (total ? total : 1));
	for (long k = 0; k < total; k++) op->colptr[op->colind[k] + 1]++;
	for (int j = 0; j < op->n; j++) op->colptr[j + 1] += op->colptr[j];
	next = (int *)dup(op->colptr, sizeof(int) * (op->n + 1));
	for (int i = 0; i < op->m; i++)
		for (int k = op->rowptr[i]; k < op->rowptr[i + 1]; k++) op->rowind[next[op->colind[k]]++] = i;
	free(next);
	free(ray); free(off); free(pix);
}

void orc_op_free(orc_op *op) {
	if (!op) return;
	free(op->A); free(op->rowptr); free(op->colind); free(op->val);
	free(op->colptr); free(op->rowind); free(op->cval);
	free(op->use_path); free(op->xe); free(op->ye); free(op->ze);
	free(op->xr); free(op->yr); free(op->zr);
	free(op);
}

int orc_op_rows(const orc_op *op) { return op->m * op->layers; }
int orc_op_cols(const orc_op *op) { return op->n * op->layers; }

/* ---------------------------------------------------------------------------
 * Bresenham tracing.  2D: 2d/mat_mult.h:145-181 (driving axis x when
 * |dx| >= |dy|; error term err = 2m - le; both endpoints included).  3D:
 * 3d/mat_mult.h:205-359 (driving axis x if mx >= my && mx >= mz, else y if
 * my >= mx && my >= mz, else z; two independent error terms).
 * The visitor gets (ray, linear pixel index).
 * ------------------------------------------------------------------------- */
typedef void (*visit_fn)(void *ctx, int ray, long pix);

static void trace2d(int x, int y, int dx, int dy, int ld, int ray, visit_fn fn, void *ctx) {
	int x_inc = dx < 0 ? -1 : 1, le = abs(dx);
	int y_inc = dy < 0 ? -1 : 1, m = abs(dy);
	fn(ctx, ray, (long)x + (long)y * ld);
	if (le >= m) {
		int err = 2 * m - le;
		for (int j = 1; j < le + 1; j++) {
			if (err > 0) { y += y_inc; err -= 2 * le; }
			err += 2 * m;
			x += x_inc;
			fn(ctx, ray, (long)x + (long)y * ld);
		}
	} else {
		int err = 2 * le - m;
		for (int j = 1; j < m + 1; j++) {
			if (err > 0) { x += x_inc; err -= 2 * m; }
			err += 2 * le;
			y += y_inc;
			fn(ctx, ray, (long)x + (long)y * ld);
		}
	}
}

static void trace3d(int x, int y, int z, int dx, int dy, int dz, int rvx, int rvy, int ray,
                    visit_fn fn, void *ctx) {
	int x_inc = dx < 0 ? -1 : 1, mx = abs(dx);
	int y_inc = dy < 0 ? -1 : 1, my = abs(dy);
	int z_inc = dz < 0 ? -1 : 1, mz = abs(dz);
	long sxy = (long)rvx * rvy;
#define VOX() fn(ctx, ray, (long)x + (long)y * rvx + (long)z * sxy)
	VOX();
	if (mx >= my && mx >= mz) {
		int e1 = 2 * my - mx, e2 = 2 * mz - mx;
		for (int j = 1; j < mx + 1; j++) {
			if (e1 > 0) { y += y_inc; e1 -= 2 * mx; }
			if (e2 > 0) { z += z_inc; e2 -= 2 * mx; }
			e1 += 2 * my; e2 += 2 * mz; x += x_inc;
			VOX();
		}
	} else if (my >= mx && my >= mz) {
		int e1 = 2 * mx - my, e2 = 2 * mz - my;
		for (int j = 1; j < my + 1; j++) {
			if (e1 > 0) { x += x_inc; e1 -= 2 * my; }
			if (e2 > 0) { z += z_inc; e2 -= 2 * my; }
			e1 += 2 * mx; e2 += 2 * mz; y += y_inc;
			VOX();
		}
	} else {
		int e1 = 2 * mx - mz, e2 = 2 * my - mz;
		for (int j = 1; j < mz + 1; j++) {
			if (e1 > 0) { x += x_inc; e1 -= 2 * mz; }
			if (e2 > 0) { y += y_inc; e2 -= 2 * mz; }
			e1 += 2 * mx; e2 += 2 * my; z += z_inc;
			VOX();
		}
	}
#undef VOX
}

/* Walk every traced ray in the reference's loop order (mp, emitter, receiver). */
static void walk_rays(const orc_op *op, visit_fn fn, void *ctx, void (*begin)(void *, int)) {
	for (int mp = 0; mp < op->nmp; mp++)
		for (int e = 0; e < op->E; e++)
			for (int r = 0; r < op->R; r++) {
				int pr = e * op->R + r;
				if (op->use_path[pr] == 0) continue;
				if (op->kind == ORC_RAY2D) {
					if (begin) begin(ctx, pr);
					trace2d(op->xe[e], op->ye[e], op->xr[r] - op->xe[e], op->yr[r] - op->ye[e], op->ld,
					        pr, fn, ctx);
				} else {
					int ray = mp * op->npaths + op->use_path[pr] - 1;   /* 3d/mat_mult.h:201-202 */
					long ie = (long)mp * op->E + e, ir = (long)mp * op->R + r;
					if (begin) begin(ctx, ray);
					trace3d(op->xe[ie], op->ye[ie], op->ze[ie], op->xr[ir] - op->xe[ie],
					        op->yr[ir] - op->ye[ie], op->zr[ir] - op->ze[ie], op->rvx, op->rvy, ray, fn,
					        ctx);
				}
			}
}

typedef struct { int *ray_index; long *offsets; int *pix; long total; int count; } list_ctx;
static void list_begin(void *c, int ray) {
	list_ctx *l = (list_ctx *)c;
	if (l->ray_index) l->ray_index[l->count] = ray;
	if (l->offsets) l->offsets[l->count] = l->total;
	l->count++;
}
static void list_visit(void *c, int ray, long pix) {
	list_ctx *l = (list_ctx *)c;
	(void)ray;
	if (l->pix) l->pix[l->total] = (int)pix;
	l->total++;
}

int orc_ray_lists(const orc_op *op, int *ray_index, long *offsets, int *pix, long *total) {
	list_ctx l = {ray_index, offsets, pix, 0, 0};
	walk_rays(op, list_visit, &l, list_begin);
	if (offsets) offsets[l.count] = l.total;
	if (total) *total = l.total;
	return l.count;
}

/* y = op(A) x for one layer; y has the output length and is overwritten. */
static void apply_layer(const orc_op *op, int trans, const double *x, double *y, long ylen) {
	memset(y, 0, sizeof(double) * ylen);
	switch (op->kind) {
	case ORC_DENSE:          /* cblas_gemv row-major, 2d/mat_mult.h:18-21 */
		if (!trans) {
#pragma omp parallel for if (op->m > 256)
			for (int i = 0; i < op->m; i++) {
				double s = 0;
				const double *row = op->A + (size_t)i * op->n;
				for (int j = 0; j < op->n; j++) s += row[j] * x[j];
				y[i] = s;
			}
		} else {
#pragma omp parallel for if (op->n > 256)
			for (int j = 0; j < op->n; j++) {
				double s = 0;
				for (int i = 0; i < op->m; i++) s += op->A[(size_t)i * op->n + j] * x[i];
				y[j] = s;
			}
		}
		break;
	case ORC_CSR:            /* mkl_csrmv / mkl_cscmv, 2d/mat_mult.h:58-66 */
		if (!trans) {
#pragma omp parallel for schedule(dynamic, 256)
			for (int i = 0; i < op->m; i++) {
				double s = 0;
				for (int k = op->rowptr[i]; k < op->rowptr[i + 1]; k++) s += op->val[k] * x[op->colind[k]];
				y[i] = s;
			}
		} else {
#pragma omp parallel for schedule(dynamic, 256)
			for (int j = 0; j < op->n; j++) {
				double s = 0;
				for (int k = op->colptr[j]; k < op->colptr[j + 1]; k++) s += op->cval[k] * x[op->rowind[k]];
				y[j] = s;
			}
		}
		break;
	default:                 /* rays: y[ray] += x[pix]*scale per hit, 2d/mat_mult.h:95-105 */
		if (!trans) {
#pragma omp parallel for schedule(dynamic, 256)
			for (int i = 0; i < op->m; i++) {
				double s = 0;
				for (int k = op->rowptr[i]; k < op->rowptr[i + 1]; k++) s += x[op->colind[k]] * op->scale;
				y[i] = s;
			}
		} else {
#pragma omp parallel for schedule(dynamic, 256)
			for (int j = 0; j < op->n; j++) {
				double s = 0;
				for (int k = op->colptr[j]; k < op->colptr[j + 1]; k++) s += x[op->rowind[k]] * op->scale;
				y[j] = s;
			}
		}
	}
}

void orc_apply(const orc_op *op, int trans, const double *x, double *y) {
	long min_ = op->m, nin = op->n;
	/* layers: block-diagonal, 2d/mat_mult.h:22-35,68-90 */
	for (int l = 0; l < op->layers; l++) {
		if (!trans) apply_layer(op, 0, x + l * nin, y + l * min_, min_);
		else apply_layer(op, 1, x + l * min_, y + l * nin, nin);
	}
}

/* ---------------------------------------------------------------------------
 * Finite differences.  D, Dt: 2d:268-293 (2D), 3d:365-425 (3D).  The 3D Dt is
 * restated exactly as the reference computes it: its y part adds, on the first
 * row of every slice z >= 1, the extra term X[last row of slice z-1] - X[first
 * row of slice z] (the axpys at 3d:402-405 run across slice boundaries), so it
 * is not the exact adjoint of D there.
 * ------------------------------------------------------------------------- */
void orc_D(int dims, int p, int q, int r, const double *U, double *Ux, double *Uy, double *Uz) {
	long n = (long)p * q * (dims == 3 ? r : 1);
	long S = (long)p * q;
	int nz = dims == 3 ? r : 1;
	for (long i = 0; i < n - 1; i++) Ux[i] = U[i + 1] - U[i];
	for (long row = 0; row < (long)p * nz; row++) Ux[row * q + q - 1] = U[row * q] - U[row * q + q - 1];
	for (long i = 0; i < ((long)p * nz - 1) * q; i++) Uy[i] = U[i + q] - U[i];
	for (int z = 0; z < nz; z++)
		for (int x = 0; x < q; x++)
			Uy[z * S + (long)(p - 1) * q + x] = U[z * S + x] - U[z * S + (long)(p - 1) * q + x];
	if (dims == 3) {
		for (long i = 0; i < S * (r - 1); i++) Uz[i] = U[i + S] - U[i];
		for (long i = 0; i < S; i++) Uz[(r - 1) * S + i] = U[i] - U[(r - 1) * S + i];
	}
}

void orc_Dt(int dims, int p, int q, int r, const double *X, const double *Y, const double *Z,
            double *res) {
	int nz = dims == 3 ? r : 1;
	long S = (long)p * q;
	long n = S * nz;
	for (long j = 1; j < n; j++) res[j] = X[j - 1] - X[j];
	for (long row = 0; row < (long)p * nz; row++) res[row * q] = X[row * q + q - 1] - X[row * q];
	long cnt = ((long)p * nz - 1) * q;      /* 2D: (p-1)q; 3D: (p*r-1)q */
	for (long i = 0; i < cnt; i++) res[q + i] += Y[i];
	for (long i = 0; i < cnt; i++) res[q + i] += -Y[q + i];
	for (int z = 0; z < nz; z++) {
		for (int x = 0; x < q; x++) res[z * S + x] += Y[(long)(p - 1) * q + z * S + x];
		for (int x = 0; x < q; x++) res[z * S + x] += -Y[z * S + x];
	}
	if (dims == 3) {
		for (long i = 0; i < S * (r - 1); i++) res[S + i] += Z[i];
		for (long i = 0; i < S * (r - 1); i++) res[S + i] += -Z[S + i];
		for (long i = 0; i < S; i++) res[i] += Z[(r - 1) * S + i];
		for (long i = 0; i < S; i++) res[i] += -Z[i];
	}
}

/* Shrinkage: anisotropic 2d:588-611 / 3d:834-871; isotropic (no reference
 * counterpart): W = max(|Ubar|_2 - 1/beta, 0) * Ubar / |Ubar|_2. */
double orc_shrink(int dims, int n, int tv_norm, double beta, const double *Ux, const double *Uy,
                  const double *Uz, const double *sx, const double *sy, const double *sz, double *Wx,
                  double *Wy, double *Wz) {
	double sum = 0;
	for (int i = 0; i < n; i++) {
		double bx = Ux[i] - sx[i] / beta;
		double by = Uy[i] - sy[i] / beta;
		double bz = dims == 3 ? Uz[i] - sz[i] / beta : 0;
		if (tv_norm == 1) {
			double nrm = sqrt(bx * bx + by * by + bz * bz);
			double t = nrm - 1 / beta;
			t = t >= 0 ? t : 0;
			sum += t;
			double s = nrm > 0 ? t / nrm : 0;
			Wx[i] = s * bx; Wy[i] = s * by;
			if (dims == 3) Wz[i] = s * bz;
		} else {
			double tx = fabs(bx) - 1 / beta, ty = fabs(by) - 1 / beta, tz = fabs(bz) - 1 / beta;
			tx = tx >= 0 ? tx : 0; ty = ty >= 0 ? ty : 0; tz = tz >= 0 ? tz : 0;
			if (dims != 3) tz = 0;
			sum += tx + ty + tz;
			Wx[i] = bx >= 0 ? tx : -tx;
			Wy[i] = by >= 0 ? ty : -ty;
			if (dims == 3) Wz[i] = bz >= 0 ? tz : -tz;
		}
	}
	return sum;
}

/* ---------------------------------------------------------------------------
 * Solver state: tval3_data, 2d:99-196 / 3d:155-245.
 * ------------------------------------------------------------------------- */
typedef struct {
	int dims, p, q, r;
	long n, m;
	int planes;     /* 2: complex data (real plane, imaginary plane) */
	long np, mp;    /* elements per plane */
	double mu, beta, muDbeta;
	double *delta, *sx, *sy, *sz;
	double f, lam1, lam2, lam3, lam4, lam5;
	double *Up, *dU, *uup, *Ux, *Uxp, *dUx, *Uy, *Uyp, *dUy, *Uz, *Uzp, *dUz, *Wx, *Wy, *Wz;
	double *Atb, *Au, *Aup, *dAu, *d, *g, *gp, *dg, *g2, *g2p, *dg2;
	unsigned numInit, currInit;
	double skipRatio, maxRelChange, currSkip;
	double *last_Au;
	double *V[3];   /* scratch for Ux - Wx etc. */
	int last_skip;  /* the last get_g_mult skipped A^T (trace only) */
	int force_skip; /* replay: -1 own decision, 0 multiply, 1 skip (next get_g_mult only) */
	double *tmp_n, *tmp_m;
	const orc_op *op;
	int tv_norm;
} st_t;

static double dot(long n, const double *a, const double *b) {
	double s = 0;
	for (long i = 0; i < n; i++) s += a[i] * b[i];
	return s;
}
static double nrm2(long n, const double *a) { return sqrt(dot(n, a, a)); }
static void axpy(long n, double a, const double *x, double *y) { for (long i = 0; i < n; i++) y[i] += a * x[i]; }
static void vadd(long n, const double *x, double a, const double *y, double *z) {
	for (long i = 0; i < n; i++) z[i] = x[i] + a * y[i];
}
static void cpy(long n, const double *x, double *y) { memcpy(y, x, sizeof(double) * n); }

static void Dst(st_t *s, const double *U, double *Ux, double *Uy, double *Uz) {
	for (int k = 0; k < s->planes; k++) {
		const long o = k * s->np;
		orc_D(s->dims, s->p, s->q, s->r, U + o, Ux + o, Uy + o, Uz ? Uz + o : NULL);
	}
}
static void Dts(st_t *s, const double *X, const double *Y, const double *Z, double *res) {
	for (int k = 0; k < s->planes; k++) {
		const long o = k * s->np;
		orc_Dt(s->dims, s->p, s->q, s->r, X + o, Y + o, Z ? Z + o : NULL, res + o);
	}
}

/* get_g_mult: generic with the A^T-skip heuristic 2d:300-357 / 3d:433-493;
 * dense always multiplies (2d:361-394 / 3d:498-529). */
static void get_g_mult(st_t *s, const double *U, int force) {
	int want = s->force_skip;
	s->force_skip = -1;
	s->last_skip = 0;
	orc_apply(s->op, 0, U, s->Au);
	if (s->op->kind == ORC_DENSE || s->skipRatio == 0) {
		orc_apply(s->op, 1, s->Au, s->g);
		return;
	}
	vadd(s->m, s->Au, -1, s->last_Au, s->tmp_m);
	double rel = nrm2(s->m, s->tmp_m) / nrm2(s->m, s->Au);
	if (force) {
		cpy(s->m, s->Au, s->last_Au); orc_apply(s->op, 1, s->Au, s->g); s->currSkip = 0;
	} else if (want == 1) {   /* replayed skip */
		s->currSkip -= 1;
		s->last_skip = 1;
	} else if (s->currInit < s->numInit) {
		cpy(s->m, s->Au, s->last_Au); orc_apply(s->op, 1, s->Au, s->g); s->currInit++; s->currSkip = 0;
	} else if (s->currSkip < 1) {
		cpy(s->m, s->Au, s->last_Au); orc_apply(s->op, 1, s->Au, s->g); s->currSkip += s->skipRatio;
	} else if (rel > s->maxRelChange || want == 0) {
		cpy(s->m, s->Au, s->last_Au); orc_apply(s->op, 1, s->Au, s->g);
	} else {
		s->currSkip -= 1;
		s->last_skip = 1;
	}
}

/* V = DU - W; lam2 = |V|^2; lam4 = <sigma, V> (shared by get_g, update_g,
 * update_W, update_mlp). */
static void form_V(st_t *s) {
	vadd(s->n, s->Ux, -1, s->Wx, s->V[0]);
	vadd(s->n, s->Uy, -1, s->Wy, s->V[1]);
	if (s->dims == 3) vadd(s->n, s->Uz, -1, s->Wz, s->V[2]);
}
static void lam24(st_t *s) {
	s->lam2 = dot(s->n, s->V[0], s->V[0]) + dot(s->n, s->V[1], s->V[1]);
	s->lam4 = dot(s->n, s->sx, s->V[0]) + dot(s->n, s->sy, s->V[1]);
	if (s->dims == 3) {
		s->lam2 += dot(s->n, s->V[2], s->V[2]);
		s->lam4 += dot(s->n, s->sz, s->V[2]);
	}
}
static void lam35(st_t *s, const double *b) {
	vadd(s->m, s->Au, -1, b, s->tmp_m);
	s->lam3 = dot(s->m, s->tmp_m, s->tmp_m);
	s->lam5 = dot(s->m, s->delta, s->tmp_m);
}
static double fval(st_t *s) {
	return (s->lam1 + s->beta / 2 * s->lam2 + s->mu / 2 * s->lam3) - s->lam4 - s->lam5;
}

/* get_g 2d:396-423 / 3d:535-576 */
static void get_g(st_t *s, const double *U, const double *b, int force) {
	get_g_mult(s, U, force);
	axpy(s->n, -1, s->Atb, s->g);
	form_V(s);
	Dts(s, s->V[0], s->V[1], s->V[2], s->g2);
	lam24(s);
	lam35(s, b);
	s->f = fval(s);
}

/* get_tau 2d:425-453 / 3d:581-619 */
static double get_tau(st_t *s, int fst) {
	if (fst) {
		double *dx = zeros(s->n), *dy = zeros(s->n), *dz = zeros(s->n);
		Dst(s, s->d, dx, dy, dz);
		double dDd = dot(s->n, dx, dx) + dot(s->n, dy, dy) + (s->dims == 3 ? dot(s->n, dz, dz) : 0);
		double dd = dot(s->n, s->d, s->d);
		orc_apply(s->op, 0, s->d, s->tmp_m);
		double Add = dot(s->m, s->tmp_m, s->tmp_m);
		free(dx); free(dy); free(dz);
		return fabs(dd / (dDd + s->muDbeta * Add));
	}
	vadd(s->n, s->g, -1, s->gp, s->dg);
	vadd(s->n, s->g2, -1, s->g2p, s->dg2);
	double ss = dot(s->n, s->uup, s->uup);
	cpy(s->n, s->dg2, s->tmp_n);
	axpy(s->n, s->muDbeta, s->dg, s->tmp_n);
	double sy = dot(s->n, s->uup, s->tmp_n);
	if (s->planes == 2) {   /* complex: |ss / sy| with sy = <uup, tmp> complex (2d:446-451) */
		const long h = s->np;
		double syi = 0;
		for (long i = 0; i < h; i++) syi += s->uup[i] * s->tmp_n[i + h] - s->uup[i + h] * s->tmp_n[i];
		return fabs(ss) / sqrt(sy * sy + syi * syi);
	}
	return fabs(ss / sy);
}

/* descend 2d:481-493 (nonneg 2d:455-465) */
static void descend(st_t *s, double *U, const double *b, double tau, int nonneg, int force) {
	axpy(s->n, -tau, s->d, U);
	if (nonneg) {
		for (long i = 0; i < s->np; i++) U[i] = U[i] < 0 ? 0 : U[i];
		for (long i = s->np; i < s->n; i++) U[i] = 0;   /* complex: Im = 0 (2d:467-479) */
	}
	Dst(s, U, s->Ux, s->Uy, s->Uz);
	get_g(s, U, b, force);
}

/* update_g 2d:495-524 / 3d:696-745 */
static void update_g(st_t *s, double alpha, double *U, const double *b) {
	vadd(s->n, s->gp, alpha, s->dg, s->g);
	vadd(s->n, s->g2p, alpha, s->dg2, s->g2);
	vadd(s->n, s->Up, alpha, s->dU, U);
	vadd(s->m, s->Aup, alpha, s->dAu, s->Au);
	vadd(s->n, s->Uxp, alpha, s->dUx, s->Ux);
	vadd(s->n, s->Uyp, alpha, s->dUy, s->Uy);
	if (s->dims == 3) vadd(s->n, s->Uzp, alpha, s->dUz, s->Uz);
	form_V(s);
	lam24(s);
	lam35(s, b);
	s->f = s->lam1 + s->beta / 2 * s->lam2 + s->mu / 2 * s->lam3 - s->lam4 - s->lam5;
}

/* min_u 2d:526-576 / 3d:750-814; returns the backtracking count (6 = restart).
 * force_bt >= 0 (replay): take exactly that many backtracking steps (6: five,
 * then the restart) instead of testing the Armijo condition. */
static int min_u(st_t *s, double *U, double *gam, const double *b, const orc_opts *o, double C,
                 int fst, double *tau_out, int force_bt) {
	double tau = get_tau(s, fst);
	cpy(s->n, U, s->Up); cpy(s->n, s->g, s->gp); cpy(s->n, s->g2, s->g2p);
	cpy(s->m, s->Au, s->Aup); cpy(s->n, s->Ux, s->Uxp); cpy(s->n, s->Uy, s->Uyp);
	if (s->dims == 3) cpy(s->n, s->Uz, s->Uzp);
	descend(s, U, b, tau, o->nonneg, 0);
	double alpha = 1;
	vadd(s->n, U, -1, s->Up, s->dU);
	double c_armij = dot(s->n, s->d, s->d) * tau * o->c * s->beta;
	int cnt = 0;
	if (force_bt >= 0 ? force_bt > 0 : fabs(s->f) > fabs(C - alpha * c_armij)) {
		vadd(s->n, s->g, -1, s->gp, s->dg);
		vadd(s->n, s->g2, -1, s->g2p, s->dg2);
		vadd(s->m, s->Au, -1, s->Aup, s->dAu);
		vadd(s->n, s->Ux, -1, s->Uxp, s->dUx);
		vadd(s->n, s->Uy, -1, s->Uyp, s->dUy);
		if (s->dims == 3) vadd(s->n, s->Uz, -1, s->Uzp, s->dUz);
		while (force_bt >= 0 ? cnt < force_bt : fabs(s->f) > fabs(C - alpha * c_armij)) {
			if (cnt == 5) {
				*gam *= o->rate_gam;
				tau = get_tau(s, 1);
				cpy(s->n, s->Up, U);
				descend(s, U, b, tau, o->nonneg, 1);
				cnt = 6;
				break;
			}
			alpha *= o->gamma;
			update_g(s, alpha, U, b);
			cnt++;
		}
	}
	*tau_out = tau;
	return cnt;
}

/* get_gradient 2d:578-585 */
static void get_gradient(st_t *s, const double *DtsAtd) {
	cpy(s->n, DtsAtd, s->d);
	axpy(s->n, 1, s->g2, s->d);
	axpy(s->n, s->muDbeta, s->g, s->d);
}

/* complex shrinkage 2d:614-649 / 3d:876-947 (each component's complex
 * modulus; the reference's 3D z component takes the y component's direction) */
static double shrink_complex(st_t *s) {
	const long h = s->np;
	const int nc = s->dims == 3 ? 3 : 2;
	double *const U[3] = {s->Ux, s->Uy, s->Uz}, *const S[3] = {s->sx, s->sy, s->sz}, *const W[3] = {s->Wx, s->Wy, s->Wz};
	double sum = 0;
	for (long i = 0; i < h; i++) {
		double re[3], im[3], ab[3], t[3];
		for (int c = 0; c < nc; c++) {
			re[c] = U[c][i] - S[c][i] / s->beta;
			im[c] = U[c][i + h] - S[c][i + h] / s->beta;
			ab[c] = sqrt(re[c] * re[c] + im[c] * im[c]);
			t[c] = ab[c] - 1 / s->beta;
			t[c] = t[c] >= 0 ? t[c] : 0;
			sum += t[c];
		}
		for (int c = 0; c < nc; c++) {
			const int dir = c == 2 ? 1 : c;   /* 3d/tval3_cpu_3d.cpp:934-937 */
			W[c][i] = ab[c] > 0 ? t[c] * re[dir] / ab[c] : 0;
			W[c][i + h] = ab[c] > 0 ? t[c] * im[dir] / ab[c] : 0;
		}
	}
	return sum;
}

static void shrinkage(st_t *s) {
	if (s->planes == 2) {
		s->lam1 = shrink_complex(s);
		return;
	}
	s->lam1 = orc_shrink(s->dims, (int)s->n, s->tv_norm, s->beta, s->Ux, s->Uy, s->Uz, s->sx, s->sy,
	                     s->sz, s->Wx, s->Wy, s->Wz);
}

/* update_W 2d:651-671 / 3d:952-983 */
static void update_W(st_t *s) {
	s->f -= (s->lam1 + s->beta / 2 * s->lam2 - s->lam4);
	shrinkage(s);
	form_V(s);
	Dts(s, s->V[0], s->V[1], s->V[2], s->g2);
	lam24(s);
	s->f += (s->lam1 + s->beta / 2 * s->lam2 - s->lam4);
}

/* update_mlp 2d:673-694 / 3d:988-1022 */
static void update_mlp(st_t *s, const double *b) {
	s->f += (s->lam4 + s->lam5);
	form_V(s);
	axpy(s->n, -s->beta, s->V[0], s->sx);
	axpy(s->n, -s->beta, s->V[1], s->sy);
	if (s->dims == 3) axpy(s->n, -s->beta, s->V[2], s->sz);
	s->lam4 = dot(s->n, s->sx, s->V[0]) + dot(s->n, s->sy, s->V[1]);
	if (s->dims == 3) s->lam4 += dot(s->n, s->sz, s->V[2]);
	vadd(s->m, s->Au, -1, b, s->tmp_m);
	axpy(s->m, -s->mu, s->tmp_m, s->delta);
	s->lam5 = dot(s->m, s->delta, s->tmp_m);
	s->f -= (s->lam4 + s->lam5);
}

/* scaleb 2d:229-266 */
/* complex data (planes of length h): the entries of least and largest
 * modulus, scl from the modulus of their difference */
static double scaleb_complex(double *b, long h) {
	double scl = 1;
	if (h > 0) {
		long imin = 0, imax = 0;
		double amin = sqrt(b[0] * b[0] + b[h] * b[h]), amax = amin;
		for (long i = 0; i < h; i++) {
			double a = sqrt(b[i] * b[i] + b[i + h] * b[i + h]);
			if (a < amin) { imin = i; amin = a; }
			if (a > amax) { imax = i; amax = a; }
		}
		double dr = b[imax] - b[imin], di = b[imax + h] - b[imin + h];
		double dif = sqrt(dr * dr + di * di);
		if (dif < 0.5) scl = 0.5 / dif;
		else if (dif > 1.5) scl = 1.5 / dif;
		if (dif < 0.5 || dif > 1.5)
			for (long i = 0; i < 2 * h; i++) b[i] *= scl;
	}
	return scl;
}

static double scaleb(double *b, long len) {
	double scl = 1;
	if (len > 0) {
		double bmin = b[0], bmax = b[0], amin = fabs(b[0]), amax = amin;
		for (long i = 0; i < len; i++) {
			double a = fabs(b[i]);
			if (a < amin) { bmin = b[i]; amin = a; }
			if (a > amax) { bmax = b[i]; amax = a; }
		}
		double dif = fabs(bmax - bmin);
		if (dif < 0.5) { scl = 0.5 / dif; for (long i = 0; i < len; i++) b[i] *= scl; }
		else if (dif > 1.5) { scl = 1.5 / dif; for (long i = 0; i < len; i++) b[i] *= scl; }
	}
	return scl;
}

static double now(void) {
	struct timeval tv;
	gettimeofday(&tv, NULL);
	return tv.tv_sec + tv.tv_usec / 1e6;
}

/* FP32-storage noise model (orc_opts.noise): x *= 1 + eps * xi */
static void perturb(double *x, long n, double eps, unsigned long long *state) {
	for (long i = 0; i < n; i++) {
		unsigned long long z = *state;
		z ^= z << 13; z ^= z >> 7; z ^= z << 17;
		*state = z;
		const double xi = (double)(z >> 11) * (2.0 / 9007199254740992.0) - 1.0;
		x[i] *= 1.0 + eps * xi;
	}
}

/* the driver, 2d:752-886 / 3d:1172-1378; rp != NULL replays recorded decisions */
static int solve_impl(int dims, int dim_y, int dim_x, int dim_z, const orc_op *op, const double *b_in, int blen,
                      const orc_opts *o, const double *Ut, double *U, orc_info *info, orc_iter *iters,
                      const orc_replay *rp) {
	double t0 = now();
	st_t S, *s = &S;
	memset(s, 0, sizeof(S));
	s->dims = dims; s->p = dim_y; s->q = dim_x; s->r = dims == 3 ? dim_z : 1;
	s->planes = o->cplx ? 2 : 1;
	if (o->cplx && o->tv_norm != 0) return -4;
	if (o->cplx && blen % 2) return -1;
	s->np = (long)dim_y * dim_x * s->r;
	s->n = s->np * s->planes;
	s->m = blen;
	s->mp = blen / s->planes;
	s->op = op; s->tv_norm = o->tv_norm;
	if (op->m * op->layers != blen) return -1;
	if (op->n * op->layers != s->n) return -2;
	long n = s->n, m = s->m;
	double **nv[] = {&s->sx, &s->sy, &s->sz, &s->Up, &s->dU, &s->uup, &s->Ux, &s->Uxp, &s->dUx, &s->Uy,
	                 &s->Uyp, &s->dUy, &s->Uz, &s->Uzp, &s->dUz, &s->Wx, &s->Wy, &s->Wz, &s->Atb, &s->d,
	                 &s->g, &s->gp, &s->dg, &s->g2, &s->g2p, &s->dg2, &s->V[0], &s->V[1], &s->V[2],
	                 &s->tmp_n};
	double **mv[] = {&s->delta, &s->Au, &s->Aup, &s->dAu, &s->last_Au, &s->tmp_m};
	for (size_t i = 0; i < sizeof(nv) / sizeof(nv[0]); i++) *nv[i] = zeros(n);
	for (size_t i = 0; i < sizeof(mv) / sizeof(mv[0]); i++) *mv[i] = zeros(m);
	s->mu = o->mu0; s->beta = o->beta0;
	s->numInit = (unsigned)o->numInitIterations; s->skipRatio = o->skipMulRatio;
	s->maxRelChange = o->maxRelativeChange;
	s->force_skip = -1;

	double *bs = zeros(m);
	cpy(m, b_in, bs);
	double muf = o->mu, betaf = o->beta, beta0 = 0;
	double *DtsAtd = zeros(n), *rcdU = zeros(n), *UrcdU = zeros(n);
	double gam = o->gam;
	double scl = s->planes == 2 ? scaleb_complex(bs, s->mp) : scaleb(bs, m);
	orc_apply(op, 1, bs, s->Atb);
	cpy(n, s->Atb, U);
	if (s->mu > muf) s->mu = muf;
	if (s->beta > betaf) s->beta = betaf;
	s->muDbeta = s->mu / s->beta;
	cpy(n, U, rcdU);
	Dst(s, U, s->Ux, s->Uy, s->Uz);
	shrinkage(s);
	get_g(s, U, bs, 1);
	get_gradient(s, DtsAtd);
	unsigned long long noise_state = o->noise_seed * 0x9E3779B97F4A7C15ull + 1;
	double Q = 1, Qp, C = s->f;
	int count_outer = 0, count_total = 0, fst;
	double RelChg, RelChgOut = 0, nrmup = 0;

	while (count_outer < o->maxcnt && count_total < o->maxit) {
		if (rp && count_total >= rp->count) break;
		fst = 1;
		while (count_total < o->maxit) {
			double tau;
			if (rp) s->force_skip = rp->skipped[count_total];
			int bt = min_u(s, U, &gam, bs, o, C, fst, &tau, rp ? rp->backtracks[count_total] : -1);
			if (o->noise > 0) {
				double *vs[] = {U, s->Ux, s->Uy, s->Uz, s->g, s->g2};
				for (int v = 0; v < 6; v++)
					if (v != 3 || s->dims == 3) perturb(vs[v], n, o->noise, &noise_state);
				perturb(s->Au, m, o->noise, &noise_state);
			}
			update_W(s);
			Qp = Q; Q = gam * Qp + 1; C = (gam * Qp * C + s->f) / Q;
			vadd(n, U, -1, s->Up, s->uup);
			get_gradient(s, DtsAtd);
			nrmup = nrm2(n, s->Up);
			RelChg = nrm2(n, s->uup) / nrmup;
			if (iters) {
				iters[count_total].tau = tau; iters[count_total].f = s->f;
				iters[count_total].relchg = RelChg; iters[count_total].backtracks = bt;
				iters[count_total].skipped = s->last_skip;
				iters[count_total].inner_end = 0;
			}
			count_total++;
			int end = rp ? rp->inner_end[count_total - 1] || count_total >= rp->count : RelChg < o->tol_inn && !fst;
			if (iters) iters[count_total - 1].inner_end = end || count_total >= o->maxit;
			if (end) break;
			fst = 0;
		}
		count_outer++;
		vadd(n, U, -1, rcdU, UrcdU);
		RelChgOut = nrm2(n, UrcdU) / nrmup;
		cpy(n, U, rcdU);
		if (rp ? count_total >= rp->count && !rp->inner_end[count_total - 1] : RelChgOut < o->tol) break;
		update_mlp(s, bs);
		beta0 = s->beta;
		s->beta *= o->rate_cnt;
		s->mu *= o->rate_cnt;
		if (s->beta > betaf) s->beta = betaf;
		if (s->mu > muf) s->mu = muf;
		s->muDbeta = s->mu / s->beta;
		s->f = s->lam1 + s->beta / 2 * s->lam2 + s->mu / 2 * s->lam3 - s->lam4 - s->lam5;
		cpy(n, s->d, DtsAtd);
		for (long i = 0; i < n; i++) DtsAtd[i] *= beta0 / s->beta;
		get_gradient(s, DtsAtd);
		gam = o->gam; Q = 1; C = s->f;
	}
	if (s->planes == 2 && o->isreal)   /* keep the real part (2d:855-859) */
		for (long i = s->np; i < n; i++) U[i] = 0;
	for (long i = 0; i < n; i++) U[i] = U[i] / scl;

	info->secs = now() - t0;
	info->outer_iters = count_outer;
	info->total_iters = count_total;
	info->rel_chg = RelChgOut;
	info->rel_error = 0;
	if (Ut) {
		double dn = 0, tn = 0;
		for (long i = 0; i < n; i++) { dn += (Ut[i] - U[i]) * (Ut[i] - U[i]); tn += Ut[i] * Ut[i]; }
		info->rel_error = sqrt(dn) / sqrt(tn);
	}
	for (size_t i = 0; i < sizeof(nv) / sizeof(nv[0]); i++) free(*nv[i]);
	for (size_t i = 0; i < sizeof(mv) / sizeof(mv[0]); i++) free(*mv[i]);
	free(bs); free(DtsAtd); free(rcdU); free(UrcdU);
	return 0;
}

int orc_solve(int dims, int dim_y, int dim_x, int dim_z, const orc_op *op, const double *b, int blen,
              const orc_opts *opts, const double *Ut, double *U, orc_info *info, orc_iter *iters) {
	return solve_impl(dims, dim_y, dim_x, dim_z, op, b, blen, opts, Ut, U, info, iters, NULL);
}

int orc_solve_replay(int dims, int dim_y, int dim_x, int dim_z, const orc_op *op, const double *b, int blen,
                     const orc_opts *opts, const double *Ut, double *U, orc_info *info, orc_iter *iters,
                     const orc_replay *replay) {
	if (!replay || replay->count < 1 || !replay->backtracks || !replay->skipped || !replay->inner_end) return -3;
	return solve_impl(dims, dim_y, dim_x, dim_z, op, b, blen, opts, Ut, U, info, iters, replay);
}
