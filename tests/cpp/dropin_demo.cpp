// A caller of the reference's C++ interface, built against the drop-in
// headers and linked to libtval3_gpu_2d.so (tests/test_dropin.py).
//
//   dropin_demo errors   argument errors only (no GPU needed): prints one
//                        exception message per line
//   dropin_demo solve    a small dense, CSR and 2D-ray solve through
//                        tval3_cpu_2d, each compared with tval3g_solve (float
//                        and complex<float> data) or tval3g_solve_f64 (double
//                        data) on the same inputs; prints
//                        "<case> <rc> <max |diff|> <iters> <C ABI iters>"
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "tval3_gpu_2d.h"
#include "tval3g.h"

static unsigned lcg = 12345u;
static float frand() {
	lcg = lcg * 1664525u + 1013904223u;
	return ((lcg >> 8) & 0xffffff) / float(1 << 24) - 0.5f;
}

static tval3_options<float> opts() {
	tval3_options<float> o;
	o.mu = 256; o.beta = 32; o.mu0 = 256; o.beta0 = 32; o.tol = 1e-4f; o.tol_inn = 1e-3f;
	o.maxit = 30; o.maxcnt = 10;
	return o;
}

static void err(const char *tag, void (*f)()) {
	try {
		f();
		std::printf("%s: no exception\n", tag);
	} catch (const tval3_exception &e) {
		std::printf("%s: %s\n", tag, e.what());
	}
}

static void e_format() {
	mat<float> U(8, 8, mat_row_major), A(20, 64, mat_row_major), b(20), Ut(0, mat_col_major);
	tval3_cpu_2d(U, A, b, opts(), Ut);
}
static void e_ut() {
	mat<float> U(8, 8, mat_col_major), A(20, 64, mat_row_major), b(20), Ut(7, mat_col_major);
	tval3_cpu_2d(U, A, b, opts(), Ut);
}
static void e_ulen() {
	mat<float> U(8, 9, mat_col_major), A(20, 64, mat_row_major), b(20), Ut(0, mat_col_major);
	tval3_cpu_2d(U, A, b, opts(), Ut);
}
static void e_blen() {
	mat<float> U(8, 8, mat_col_major), A(20, 64, mat_row_major), b(21), Ut(0, mat_col_major);
	tval3_cpu_2d(U, A, b, opts(), Ut);
}
static void e_csc() {
	mat<float> U(8, 8, mat_col_major), b(20), Ut(0, mat_col_major);
	sparse_mat<float> A(20, 64, 0, sparse_mat_csr);
	tval3_cpu_2d(U, A, b, opts(), Ut);
}
static void e_geom_layers() {
	mat<float> U(8, 8, mat_row_major), b(10), Ut(0, mat_row_major);
	int use[4] = {1, 1, 1, 1}, xe[2] = {0, 7}, ye[2] = {0, 7}, xr[2] = {7, 0}, yr[2] = {0, 7};
	geometry g = {2, 2, use, xe, ye, xr, yr, 8, 1.0f};
	tval3_cpu_2d(U, g, b, opts(), Ut);
}
static void e_double() {   // double data: the same argument checks
	mat<double> U(8, 8, mat_row_major), A(20, 64, mat_row_major), b(20), Ut(0, mat_col_major);
	tval3_options<double> o;
	tval3_cpu_2d(U, A, b, o, Ut);
}
static void e_complex() {   // complex data: the layered size check
	mat<std::complex<float> > U(8, 16, mat_col_major), A(20, 64, mat_row_major), b(41), Ut(0, mat_col_major);
	tval3_cpu_2d(U, A, b, opts(), Ut);
}
static void e_complex_format() {   // complex data: the same argument checks
	mat<std::complex<double> > U(8, 8, mat_row_major), A(20, 64, mat_row_major), b(20), Ut(0, mat_col_major);
	tval3_options<double> o;
	tval3_cpu_2d(U, A, b, o, Ut);
}

static double maxdiff(const float *a, const float *b, int n) {
	double d = 0;
	for (int i = 0; i < n; i++) d = std::fmax(d, std::fabs((double)a[i] - b[i]));
	return d;
}

static void solve_cases() {
	const int p = 16, q = 16, n = p * q, m = 77;
	// dense
	mat<float> A(m, n, mat_row_major), U(p, q, mat_col_major), b(m), Ut(0, mat_col_major);
	for (int i = 0; i < m * n; i++) A[i] = frand() / std::sqrt((float)m);
	std::vector<float> u0(n);
	for (int i = 0; i < n; i++) u0[i] = ((i % q) > 4 && (i % q) < 11 && (i / q) > 3 && (i / q) < 12) ? 1.f : 0.f;
	for (int r = 0; r < m; r++) {
		double s = 0;
		for (int c = 0; c < n; c++) s += (double)A[r * n + c] * u0[c];
		b[r] = (float)s;
	}
	tval3_info<float> info = tval3_cpu_2d(U, A, b, opts(), Ut);
	tval3g_problem pr;
	std::memset(&pr, 0, sizeof(pr));
	pr.dims = 2; pr.dim_y = p; pr.dim_x = q; pr.dim_z = 1; pr.op_kind = TVAL3G_OP_DENSE;
	pr.m = m; pr.n_cols = n; pr.layers = 1; pr.A = A.data();
	tval3_options<float> o = opts();
	tval3g_options co;
	std::memset(&co, 0, sizeof(co));
	co.mu = o.mu; co.beta = o.beta; co.mu0 = o.mu0; co.beta0 = o.beta0; co.tol = o.tol; co.tol_inn = o.tol_inn;
	co.c = o.c; co.gamma = o.gamma; co.gam = o.gam; co.rate_gam = o.rate_gam; co.rate_cnt = o.rate_cnt;
	co.maxit = o.maxit; co.maxcnt = o.maxcnt;
	std::vector<float> U2(n);
	tval3g_info ci;
	int rc = tval3g_solve(&pr, b.data(), m, &co, 0, 0, U2.data(), &ci);
	std::printf("dense %d %.3e %d %d\n", rc, maxdiff(U.data(), U2.data(), n), info.total_iters, ci.total_iters);
	tval3_options<double> od;
	od.mu = o.mu; od.beta = o.beta; od.mu0 = o.mu0; od.beta0 = o.beta0; od.tol = o.tol; od.tol_inn = o.tol_inn;
	od.maxit = o.maxit; od.maxcnt = o.maxcnt;
	od.c = o.c; od.gamma = o.gamma; od.gam = o.gam; od.rate_gam = o.rate_gam; od.rate_cnt = o.rate_cnt;
	{   // double data through the double overload and through tval3g_solve_f64 (the FP64 engine)
		mat<double> Ad(m, n, mat_row_major), Ud(p, q, mat_col_major), bd(m), Utd(0, mat_col_major);
		for (int i = 0; i < m * n; i++) Ad[i] = A[i];
		for (int r = 0; r < m; r++) bd[r] = b[r];
		tval3_info<double> infod = tval3_cpu_2d(Ud, Ad, bd, od, Utd);
		tval3g_problem pd = pr;
		pd.A = 0;
		std::vector<double> Ud2(n);
		tval3g_info cid;
		int rcd = tval3g_solve_f64(&pd, Ad.data(), bd.data(), m, &co, 0, 0, Ud2.data(), &cid);
		double d = 0, df = 0;
		for (int i = 0; i < n; i++) {
			d = std::fmax(d, std::fabs(Ud[i] - Ud2[i]));
			df = std::fmax(df, std::fabs(Ud[i] - (double)U2[i]));
		}
		std::printf("dense_f64 %d %.3e %d %d %.3e\n", rcd, d, infod.total_iters, cid.total_iters, df);
	}
	// CSR twin of A restricted to |a| > 0.2
	std::vector<int> ptr(1, 0), ind;
	std::vector<float> val;
	for (int r = 0; r < m; r++) {
		for (int c = 0; c < n; c++)
			if (std::fabs(A[r * n + c]) * std::sqrt((float)m) > 0.2f) { ind.push_back(c); val.push_back(A[r * n + c]); }
		ptr.push_back((int)ind.size());
	}
	sparse_mat<float> S(m, n, (int)ind.size(), sparse_mat_both);
	std::memcpy(S.csr_ptr(), ptr.data(), sizeof(int) * ptr.size());
	std::memcpy(S.csr_ind(), ind.data(), sizeof(int) * ind.size());
	std::memcpy(S.csr_val(), val.data(), sizeof(float) * val.size());
	S.build_csc_from_csr();
	mat<float> Us(p, q, mat_col_major);
	info = tval3_cpu_2d(Us, S, b, opts(), Ut);
	pr.op_kind = TVAL3G_OP_CSR; pr.A = 0; pr.nnz = (long long)ind.size();
	pr.csr_ptr = ptr.data(); pr.csr_ind = ind.data(); pr.csr_val = val.data();
	rc = tval3g_solve(&pr, b.data(), m, &co, 0, 0, U2.data(), &ci);
	std::printf("csr %d %.3e %d %d\n", rc, maxdiff(Us.data(), U2.data(), n), info.total_iters, ci.total_iters);
	// 2D rays: 8 transducers on the border of the 16x16 image, all pairs
	const int T = 8;
	int xs[T] = {0, 7, 15, 15, 15, 8, 0, 0}, ys[T] = {0, 0, 0, 7, 15, 15, 15, 8};
	std::vector<int> use(T * T);
	for (int e = 0; e < T; e++)
		for (int r = 0; r < T; r++) use[e * T + r] = (e != r);
	geometry g = {T, T, use.data(), xs, ys, xs, ys, q, 1.0f};
	mat<float> Ur(p, q, mat_row_major), br(T * T), Utr(0, mat_row_major);
	for (int i = 0; i < T * T; i++) br[i] = use[i] ? 1.f + 0.1f * frand() : 0.f;
	info = tval3_cpu_2d(Ur, g, br, opts(), Utr);
	pr.op_kind = TVAL3G_OP_RAY2D; pr.nnz = 0; pr.csr_ptr = 0; pr.csr_ind = 0; pr.csr_val = 0; pr.m = 0; pr.n_cols = 0;
	pr.num_emitters = T; pr.num_receivers = T; pr.numMPs = 1; pr.use_path = use.data();
	pr.x_emitters = xs; pr.y_emitters = ys; pr.x_receivers = xs; pr.y_receivers = ys; pr.ld = q; pr.scale_factor = 1.f;
	rc = tval3g_solve(&pr, br.data(), T * T, &co, 0, 0, U2.data(), &ci);
	std::printf("ray2d %d %.3e %d %d\n", rc, maxdiff(Ur.data(), U2.data(), n), info.total_iters, ci.total_iters);
	{   // the same rays with double data: the double overload and tval3g_solve_f64
		mat<double> Urd(p, q, mat_row_major), brd(T * T), Utrd(0, mat_row_major);
		for (int i = 0; i < T * T; i++) brd[i] = br[i];
		tval3_info<double> infod = tval3_cpu_2d(Urd, g, brd, od, Utrd);
		std::vector<double> Ud2(n);
		tval3g_info cid;
		int rcd = tval3g_solve_f64(&pr, 0, brd.data(), T * T, &co, 0, 0, Ud2.data(), &cid);
		double d = 0;
		for (int i = 0; i < n; i++) d = std::fmax(d, std::fabs(Urd[i] - Ud2[i]));
		std::printf("ray2d_f64 %d %.3e %d %d\n", rcd, d, infod.total_iters, cid.total_iters);
	}
	{   // complex data through the complex<float> overload and through the C ABI
		mat<std::complex<float> > Ac(m, n, mat_row_major), Uc(p, q, mat_col_major), bc(m), Utc(0, mat_col_major);
		for (int i = 0; i < m * n; i++) Ac[i] = std::complex<float>(A[i], frand() / std::sqrt((float)m));
		for (int r = 0; r < m; r++) {
			std::complex<double> s = 0;
			for (int c = 0; c < n; c++) s += std::complex<double>(Ac[r * n + c]) * (double)u0[c];
			bc[r] = std::complex<float>(s);
		}
		info = tval3_cpu_2d(Uc, Ac, bc, opts(), Utc);
		tval3g_problem pc;
		std::memset(&pc, 0, sizeof(pc));
		pc.dims = 2; pc.dim_y = p; pc.dim_x = q; pc.dim_z = 1; pc.op_kind = TVAL3G_OP_DENSE;
		pc.m = m; pc.n_cols = n; pc.layers = 1; pc.A = reinterpret_cast<const float *>(Ac.data());
		pc.complex_data = 1;
		std::vector<std::complex<float> > Uc2(n);
		rc = tval3g_solve(&pc, reinterpret_cast<const float *>(bc.data()), m, &co, 0, 0,
		                  reinterpret_cast<float *>(Uc2.data()), &ci);
		std::printf("cdense %d %.3e %d %d\n", rc,
		            maxdiff(reinterpret_cast<const float *>(Uc.data()), reinterpret_cast<const float *>(Uc2.data()),
		                    2 * n),
		            info.total_iters, ci.total_iters);
	}
}

int main(int argc, char **argv) {
	std::string mode = argc > 1 ? argv[1] : "errors";
	if (mode == "errors") {
		err("format", e_format);
		err("ut", e_ut);
		err("ulen", e_ulen);
		err("blen", e_blen);
		err("csc", e_csc);
		err("geom_layers_or_blen", e_geom_layers);
		err("double", e_double);
		err("complex", e_complex);
		err("complex_format", e_complex_format);
		return 0;
	}
	try {
		solve_cases();
	} catch (const tval3_exception &e) {
		std::printf("exception: %s\n", e.what());
		return 1;
	}
	return 0;
}
