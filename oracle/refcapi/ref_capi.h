/*
 * Oracle (test infrastructure only): C entry points around the reference's
 * own C++ solver overloads, built from the reference sources by
 * oracle/Makefile into oracle/_ref/.  Only tests, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg load these libraries.
 *
 * dtype: 0 = float data + tval3_options<float>, 1 = float data +
 *        tval3_options<double>, 2 = double data + tval3_options<double>,
 *        3 = complex<float> data + tval3_options<float>, 4 = complex<double>
 *        data + tval3_options<double> (2D dense and CSR; 3D dense, CSR
 *        and geometry).
 * Returns 0, or 1 with the exception's message in err (the reference throws
 * tval3_exception, 2d/tval3_cpu_2d.cpp:878-884).
 */
#ifndef ORACLE_REF_CAPI_H_
#define ORACLE_REF_CAPI_H_
#ifdef __cplusplus
extern "C" {
#endif
typedef struct {
	double mu, beta, mu0, beta0, tol, tol_inn, c, gamma, gam, rate_gam, rate_cnt;
	double skipMulRatio, maxRelativeChange;
	int maxit, maxcnt, nonneg, isreal, numInitIterations;
} ref_opts;

typedef struct {
	double secs, rel_chg, rel_error;
	int outer_iters, total_iters;
} ref_info;
#ifdef __cplusplus
}

template <class S>
static tval3_options<S> to_opts(const ref_opts *o) {
	tval3_options<S> t;
	t.mu = (S)o->mu; t.beta = (S)o->beta; t.mu0 = (S)o->mu0; t.beta0 = (S)o->beta0;
	t.tol = (S)o->tol; t.tol_inn = (S)o->tol_inn; t.c = (S)o->c; t.gamma = (S)o->gamma;
	t.gam = (S)o->gam; t.rate_gam = (S)o->rate_gam; t.rate_cnt = (S)o->rate_cnt;
	t.skipMulRatio = (S)o->skipMulRatio; t.maxRelativeChange = (S)o->maxRelativeChange;
	t.maxit = o->maxit; t.maxcnt = o->maxcnt; t.nonneg = o->nonneg != 0; t.isreal = o->isreal != 0;
	t.numInitIterations = (unsigned)o->numInitIterations;
	return t;
}

template <class S>
static void from_info(const tval3_info<S> &i, ref_info *o) {
	o->secs = i.secs; o->rel_chg = (double)i.rel_chg; o->rel_error = (double)i.rel_error;
	o->outer_iters = i.outer_iters; o->total_iters = i.total_iters;
}

static void set_err(char *err, int errlen, const char *msg) {
	if (err && errlen > 0) {
		std::strncpy(err, msg, errlen - 1);
		err[errlen - 1] = 0;
	}
}

template <class T>
static void fill(mat<T> &m, const void *src) {
	if (src && m.len > 0) std::memcpy(m.data(), src, sizeof(T) * (size_t)m.len);
}
#endif
#endif
