/*
 * Option, result and exception types of the TVAL3 C++ interface.
 *
 * The reference includes "tval3_types.h" but does not ship it
 * (2d/tval3_cpu_2d.cpp:6, 3d/tval3_cpu_3d.cpp:18).  Field names follow every use
 * in the reference:
 *   mu, beta, mu0, beta0          2d/tval3_cpu_2d.cpp:163-164,769-770
 *   tol, tol_inn, maxit, maxcnt   2d/tval3_cpu_2d.cpp:790,793,814,827
 *   c, gamma, gam, rate_gam       2d/tval3_cpu_2d.cpp:546,563,569,772
 *   rate_cnt                      2d/tval3_cpu_2d.cpp:835-836
 *   nonneg, isreal                2d/tval3_cpu_2d.cpp:487,857
 *   numInitIterations, skipMulRatio, maxRelativeChange
 *                                 2d/tval3_cpu_2d.cpp:190-192
 *   info.secs, outer_iters, total_iters, rel_chg, rel_error
 *                                 2d/tval3_cpu_2d.cpp:865-877
 *   tval3_exception(std::string)  2d/tval3_cpu_2d.cpp:702,878-884
 *
 * One field is appended that the reference does not have: tv_norm selects
 * anisotropic (the only norm the reference computes, 2d/tval3_cpu_2d.cpp:588-611)
 * or isotropic total variation.  It defaults to anisotropic, so a caller that
 * never sets it gets the reference's behaviour.
 *
 * The reference's default values live in the missing header.  The defaults here
 * are the published TVAL3 option set (mu 2^8, beta 2^5, mu0 = mu, beta0 = beta,
 * tol 1e-6, tol_inn 1e-3, maxcnt 10, maxit 1025, c 1e-5, gamma 0.6,
 * gam 0.9995, rate_cnt 2, rate_gam 0.9); callers that need a particular run
 * should set every field.
 *
 * C++98 compatible (the reference sources are built against it).
 */
#ifndef TVAL3_TYPES_H_
#define TVAL3_TYPES_H_

#include <exception>
#include <string>

#if __cplusplus >= 201103L
#define TVAL3_NOTHROW noexcept
#else
#define TVAL3_NOTHROW throw()
#endif

enum tval3_tv_norm { tval3_tv_aniso = 0, tval3_tv_iso = 1 };

template <class T>
struct tval3_options {
	T mu;        /* final weight of the data term */
	T beta;      /* final weight of the gradient splitting term */
	T mu0;       /* initial mu of the continuation scheme */
	T beta0;     /* initial beta of the continuation scheme */
	T tol;       /* outer stopping tolerance on ||U - U_outer_prev|| / ||Up|| */
	T tol_inn;   /* inner stopping tolerance on ||U - Up|| / ||Up|| */
	int maxit;   /* maximum total inner iterations */
	int maxcnt;  /* maximum outer iterations */
	T c;         /* Armijo constant */
	T gamma;     /* backtracking step factor */
	T gam;       /* nonmonotone averaging weight */
	T rate_gam;  /* shrink factor of gam after a failed backtracking */
	T rate_cnt;  /* continuation growth factor of mu and beta */
	bool nonneg; /* project U onto U >= 0 after each descent step */
	bool isreal; /* return the real part only (complex data) */
	unsigned int numInitIterations; /* Aᵀ-skip heuristic, see get_g_mult */
	T skipMulRatio;                 /* 0 disables the Aᵀ-skip heuristic */
	T maxRelativeChange;
	int tv_norm; /* tval3_tv_aniso (reference behaviour) or tval3_tv_iso */

	tval3_options()
		: mu(256), beta(32), mu0(256), beta0(32), tol(1e-6), tol_inn(1e-3),
		  maxit(1025), maxcnt(10), c(1e-5), gamma(0.6), gam(0.9995),
		  rate_gam(0.9), rate_cnt(2), nonneg(false), isreal(false),
		  numInitIterations(0), skipMulRatio(0), maxRelativeChange(0),
		  tv_norm(tval3_tv_aniso) {}
};

template <class T>
struct tval3_info {
	double secs;      /* wall-clock seconds of the whole call */
	int outer_iters;  /* outer (continuation) iterations run */
	int total_iters;  /* inner iterations run */
	T rel_chg;        /* last outer relative change */
	T rel_error;      /* ||Ut - U|| / ||Ut|| when Ut is given, else 0 */
	tval3_info() : secs(0), outer_iters(0), total_iters(0), rel_chg(0), rel_error(0) {}
};

class tval3_exception : public std::exception {
public:
	tval3_exception(const std::string &msg) : message(msg) {}
	virtual ~tval3_exception() TVAL3_NOTHROW {}
	virtual const char *what() const TVAL3_NOTHROW { return message.c_str(); }
private:
	std::string message;
};

#endif /* TVAL3_TYPES_H_ */
