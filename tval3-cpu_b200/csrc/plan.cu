// Plans: validation, operator preparation, state layout and the solve program.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>

#include "plan.cuh"

#include <map>
#include <tuple>
#include <mutex>

namespace tval3g {
// the device-memory pool is shared by both precision builds (defined once)
#ifndef TVAL3G_FP64
cudaMemPool_t library_pool() {
	static std::mutex mu;
	static std::map<int, cudaMemPool_t> pools;
	int dev = 0;
	TG_CUDA(cudaGetDevice(&dev));
	std::lock_guard<std::mutex> lock(mu);
	auto it = pools.find(dev);
	if (it != pools.end()) return it->second;
	cudaMemPoolProps props;
	std::memset(&props, 0, sizeof(props));
	props.allocType = cudaMemAllocationTypePinned;
	props.location.type = cudaMemLocationTypeDevice;
	props.location.id = dev;
	cudaMemPool_t pool;
	TG_CUDA(cudaMemPoolCreate(&pool, &props));
	unsigned long long keep = ~0ull;
	TG_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
	pools[dev] = pool;
	return pool;
}

void *dev_alloc(size_t bytes, cudaStream_t s) {
	void *p = nullptr;
	TG_CUDA(cudaMallocFromPoolAsync(&p, std::max<size_t>(bytes, 16), library_pool(), s));
	return p;
}

void dev_free(void *p, cudaStream_t s) {
	if (p) cudaFreeAsync(p, s);
}
#endif
}  // namespace tval3g

TG_BEGIN


// ---------------------------------------------------------------------------
// validation (2d/tval3_cpu_2d.cpp:696-750, 3d/tval3_cpu_3d.cpp:1028-1165)
// ---------------------------------------------------------------------------
long long validate(const tval3g_problem &p, long long b_len, long long ut_len, bool rays) {
	TG_ARG(p.dims == 2 || p.dims == 3, "Argument error: dims must be 2 or 3");
	TG_ARG(p.dim_x >= 1 && p.dim_y >= 1 && (p.dims == 2 || p.dim_z >= 1),
	       "Argument error: image dimensions must be positive");
	const long long n = (long long)p.dim_x * p.dim_y * (p.dims == 3 ? p.dim_z : 1);
	TG_ARG(n < (1LL << 31), "Argument error: the image has more than 2^31-1 elements");
	TG_ARG(ut_len == 0 || ut_len == n, "Argument error: U and Ut must have the same size!");
	TG_ARG(b_len >= 1, "Argument error: b must not be empty");
	TG_ARG(b_len < (1LL << 31), "Argument error: b has more than 2^31-1 elements");
	switch (p.op_kind) {
	case TVAL3G_OP_DENSE:
	case TVAL3G_OP_CSR: {
		const int layers = p.dims == 3 ? 1 : p.layers;
		TG_ARG(p.m >= 1 && p.n_cols >= 1, "Argument error: A must not be empty");
		if (p.dims == 2) {
			TG_ARG(n == (long long)p.n_cols * layers,
			       "Argument error: the length of U must be equal to A.dim_x * layers!");
			TG_ARG(b_len == (long long)p.m * layers, "Argument error: b.len must be equal to A.dim_y * layers!");
		} else {
			TG_ARG(n == p.n_cols, "Argument error: the length of U must be equal to A.dim_x!");
			TG_ARG(b_len == p.m, "Argument error: b.len must be equal to A.dim_y!");
		}
		if (p.op_kind == TVAL3G_OP_DENSE) TG_ARG(p.A != nullptr, "Argument error: A is NULL");
		else
			TG_ARG(p.csr_ptr && (p.nnz == 0 || (p.csr_ind && p.csr_val)) && p.nnz >= 0 && p.nnz < (1LL << 31),
			       "Argument error: A must be available in CSR and CSC format!");
		break;
	}
	case TVAL3G_OP_RAY2D:
		TG_ARG(p.dims == 2, "Argument error: 2D ray geometry needs a 2D image");
		TG_ARG(p.layers <= 1,
		       "Argument error: multilayer reconstruction with dynamic calculation is not supported!");
		TG_ARG(b_len == (long long)p.num_emitters * p.num_receivers,
		       "Argument error: b.len must be equal to A.num_emitters * A.num_receivers!");
		TG_ARG(p.use_path && p.x_emitters && p.y_emitters && p.x_receivers && p.y_receivers,
		       "Argument error: incomplete ray geometry");
		TG_ARG(p.ld >= 1 && p.ld < 32768, "Argument error: geometry ld must be in [1, 32767]");
		break;
	case TVAL3G_OP_RAY3D:
		TG_ARG(p.dims == 3, "Argument error: 3D ray geometry needs a 3D image");
		TG_ARG(b_len == (long long)p.numPaths * p.numMPs,
		       "Argument error: b.len must be equal to A.num_emitters * A.num_receivers!");
		TG_ARG(p.use_path && p.x_emitters && p.y_emitters && p.z_emitters && p.x_receivers && p.y_receivers &&
		           p.z_receivers && p.numMPs >= 1,
		       "Argument error: incomplete ray geometry");
		TG_ARG(p.rv_x >= 1 && p.rv_y >= 1 && p.rv_z >= 1 && p.rv_x < 32768 && p.rv_y < 32768 && p.rv_z < 32768,
		       "Argument error: geometry rv_x, rv_y, rv_z must be in [1, 32767]");
		TG_ARG((long long)p.rv_x * p.rv_y * p.rv_z <= n, "Argument error: the geometry volume exceeds U");
		break;
	default:
		throw Error{TVAL3G_ERR_ARGUMENT, "Argument error: unknown operator kind"};
	}
	if (rays && (p.op_kind == TVAL3G_OP_RAY2D || p.op_kind == TVAL3G_OP_RAY3D)) {
		// every traced ray must stay inside the image (Bresenham stays inside
		// the bounding box of its endpoints); the reference does not check
		const bool is3 = p.op_kind == TVAL3G_OP_RAY3D;
		const int E = p.num_emitters, R = p.num_receivers, nmp = is3 ? p.numMPs : 1;
		const long long ny = is3 ? 0 : n / p.ld;
		for (int mp = 0; mp < nmp; mp++)
			for (int e = 0; e < E; e++)
				for (int r = 0; r < R; r++) {
					const int up = p.use_path[(long long)e * R + r];
					if (up == 0) continue;
					if (!is3) {
						const int x0 = p.x_emitters[e], y0 = p.y_emitters[e], x1 = p.x_receivers[r], y1 = p.y_receivers[r];
						TG_ARG(x0 >= 0 && x0 < p.ld && x1 >= 0 && x1 < p.ld && y0 >= 0 && y0 < ny && y1 >= 0 && y1 < ny,
						       "Argument error: a ray endpoint lies outside the image");
					} else {
						const long long ie = (long long)mp * E + e, ir = (long long)mp * R + r;
						const int x0 = p.x_emitters[ie], y0 = p.y_emitters[ie], z0 = p.z_emitters[ie];
						const int x1 = p.x_receivers[ir], y1 = p.y_receivers[ir], z1 = p.z_receivers[ir];
						TG_ARG(x0 >= 0 && x0 < p.rv_x && x1 >= 0 && x1 < p.rv_x && y0 >= 0 && y0 < p.rv_y && y1 >= 0 &&
						           y1 < p.rv_y && z0 >= 0 && z0 < p.rv_z && z1 >= 0 && z1 < p.rv_z,
						       "Argument error: a ray endpoint lies outside the volume");
						TG_ARG(up >= 1 && up <= p.numPaths, "Argument error: use_path index exceeds numPaths");
					}
				}
	}
	return n;
}

void check_options(const tval3g_options &o) {
	TG_ARG(o.beta > 0 && o.beta0 > 0 && o.mu > 0 && o.mu0 > 0, "Argument error: mu, beta, mu0, beta0 must be positive");
	TG_ARG(o.tv_norm == TVAL3G_TV_ANISO || o.tv_norm == TVAL3G_TV_ISO, "Argument error: tv_norm must be 0 or 1");
	TG_ARG(o.maxit >= 0 && o.maxcnt >= 0, "Argument error: maxit and maxcnt must be >= 0");
}

// ---------------------------------------------------------------------------
// operators
// ---------------------------------------------------------------------------
template <class T>
static T *dcopy(cudaStream_t s, OpStore &st, const T *src, long long count, bool borrow) {
	if (borrow) return const_cast<T *>(src);
	size_t bytes = sizeof(T) * (size_t)std::max(count, 1LL);
	T *d = (T *)dev_alloc(bytes, s);
	st.owned.push_back(d);
	st.bytes += (long long)bytes;
	if (count > 0) TG_CUDA(cudaMemcpyAsync(d, src, sizeof(T) * (size_t)count, cudaMemcpyHostToDevice, s));
	return d;
}
template <class T>
static T *dalloc_op(cudaStream_t s, OpStore &st, long long count) {
	T *d = (T *)dev_alloc(sizeof(T) * (size_t)std::max(count, 1LL), s);
	st.owned.push_back(d);
	st.bytes += (long long)(sizeof(T) * (size_t)std::max(count, 1LL));
	return d;
}

__global__ void k_map_out(long long nnz, const int4 *rays, int *cind) {
	long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
	if (k < nnz) cind[k] = rays[cind[k]].w;
}

// Complex data (2D): the operator becomes its real form on planar vectors
// [Re x; Im x] -> [Re A x; Im A x], i.e. [[Re A, -Im A], [Im A, Re A]], whose
// transpose gives [Re A^H y; Im A^H y] - the reference's conjugate-transposed
// products (2d/mat_mult.h:15-91, CblasConjTrans / 'c').  Dense A and CSR
// values arrive as interleaved (re, im) pairs; a ray geometry (real
// weights, 2D or 3D) becomes the CSR form of diag(A, A) over its traced rays.
static void prepare_complex_op(cudaStream_t s, const tval3g_problem &p, int flags, OpStore &st,
                               bool keep_ray_csr) {
	TG_ARG(!(flags & TVAL3G_DEVICE_INPUTS), "Argument error: complex operators must be given in host memory");
	tval3g_problem q = p;
	q.complex_data = 0;
	q.layers = 1;
	const long long L = p.dims == 2 && p.op_kind != TVAL3G_OP_RAY2D ? std::max(p.layers, 1) : 1;
	if (p.op_kind == TVAL3G_OP_DENSE && L == 1) {
		const long long m = p.m, nc = p.n_cols;
		const real *pa = prob_A(p);
		std::vector<real> R((size_t)(4 * m * nc));
		for (long long r = 0; r < m; r++)
			for (long long c = 0; c < nc; c++) {
				const real ar = pa[2 * (r * nc + c)], ai = pa[2 * (r * nc + c) + 1];
				R[(size_t)(r * 2 * nc + c)] = ar;
				R[(size_t)(r * 2 * nc + nc + c)] = -ai;
				R[(size_t)((m + r) * 2 * nc + c)] = ai;
				R[(size_t)((m + r) * 2 * nc + nc + c)] = ar;
			}
		q.m = (int)(2 * m);
		q.n_cols = (int)(2 * nc);
		q.A = reinterpret_cast<const float *>(R.data());   // read back as real (prob_A)
		prepare_op(s, q, flags, st, keep_ray_csr);   // copies R before it returns
		return;
	}
	// CSR rows of the real form from (row pointers, columns, complex values).
	// With L layers (2D, the reference's stacked layers) the planar vectors
	// hold all layers' real parts, then all imaginary parts, so layer l's
	// block maps columns l nc (+ L nc for Im x) to rows l m (+ L m for Im y).
	auto expand = [&](long long m, long long nc, const std::vector<int> &ptr, const std::vector<int> &ind,
	                  const real *re, const real *im, int re_stride) {
		const long long nnz = ptr[m], P = L * nc;
		TG_ARG(4 * nnz * L < (1LL << 31), "Argument error: the complex operator has too many entries");
		std::vector<int> rp((size_t)(2 * m * L + 1)), ri((size_t)(4 * nnz * L));
		std::vector<real> rv((size_t)(4 * nnz * L));
		long long o = 0;
		for (int half = 0; half < 2; half++)
			for (long long l = 0; l < L; l++)
				for (long long r = 0; r < m; r++) {
					rp[(size_t)(half * m * L + l * m + r)] = (int)o;
					for (int part = 0; part < 2; part++)   // columns of Re x, then of Im x
						for (long long k = ptr[r]; k < ptr[r + 1]; k++) {
							const real vr = re[k * re_stride], vi = im ? im[k * re_stride] : 0.f;
							ri[(size_t)o] = (int)(ind[(size_t)k] + l * nc + (part ? P : 0));
							// [[Re A, -Im A], [Im A, Re A]]
							rv[(size_t)o++] = half == 0 ? (part == 0 ? vr : -vi) : (part == 0 ? vi : vr);
						}
				}
		rp[(size_t)(2 * m * L)] = (int)o;
		tval3g_problem c = p;
		c.complex_data = 0;
		c.layers = 1;
		c.op_kind = TVAL3G_OP_CSR;
		c.m = (int)(2 * m * L);
		c.n_cols = (int)(2 * nc * L);
		c.nnz = o;
		c.csr_ptr = rp.data();
		c.csr_ind = ri.data();
		c.csr_val = reinterpret_cast<const float *>(rv.data());   // read back as real (prob_val)
		prepare_op(s, c, flags, st, keep_ray_csr);
		TG_CUDA(cudaStreamSynchronize(s));
	};
	if (p.op_kind == TVAL3G_OP_CSR) {
		std::vector<int> ptr(p.csr_ptr, p.csr_ptr + p.m + 1), ind(p.csr_ind, p.csr_ind + p.nnz);
		expand(p.m, p.n_cols, ptr, ind, prob_val(p), prob_val(p) + 1, 2);
		return;
	}
	if (p.op_kind == TVAL3G_OP_DENSE) {   // layered: every entry of A as a CSR entry
		std::vector<int> ptr((size_t)p.m + 1), ind((size_t)p.m * p.n_cols);
		for (long long r = 0; r <= p.m; r++) ptr[(size_t)r] = (int)(r * p.n_cols);
		for (long long k = 0; k < (long long)p.m * p.n_cols; k++) ind[(size_t)k] = (int)(k % p.n_cols);
		expand(p.m, p.n_cols, ptr, ind, prob_A(p), prob_A(p) + 1, 2);
		return;
	}
	// rays: trace on the device, then the CSR over all measurements (2D: E x
	// R; 3D: numPaths x numMPs, the compact index)
	OpStore tmp;
	q.complex_data = 0;
	prepare_op(s, q, flags, tmp, true);
	const bool is3 = p.op_kind == TVAL3G_OP_RAY3D;
	const long long m = is3 ? (long long)p.numPaths * p.numMPs : (long long)p.num_emitters * p.num_receivers;
	const long long n = (long long)p.dim_x * p.dim_y * (is3 ? p.dim_z : 1);
	const int nr = tmp.dev.nrays;
	std::vector<int> trp((size_t)nr + 1), tri((size_t)std::max(tmp.nnz, 1LL));
	TG_CUDA(cudaMemcpyAsync(trp.data(), tmp.ray_rptr, sizeof(int) * ((size_t)nr + 1), cudaMemcpyDeviceToHost, s));
	if (tmp.nnz > 0)
		TG_CUDA(cudaMemcpyAsync(tri.data(), tmp.ray_rind, sizeof(int) * (size_t)tmp.nnz, cudaMemcpyDeviceToHost, s));
	TG_CUDA(cudaStreamSynchronize(s));
	const float scale = tmp.dev.scale;
	free_op(tmp, s);
	std::vector<int> ptr((size_t)m + 1, 0), ind((size_t)std::max(tmp.nnz, 1LL));
	for (int k = 0; k < nr; k++) ptr[(size_t)tmp.ray_out[k] + 1] = trp[(size_t)k + 1] - trp[(size_t)k];
	for (long long r = 0; r < m; r++) ptr[(size_t)r + 1] += ptr[(size_t)r];
	for (int k = 0; k < nr; k++)
		std::copy(tri.begin() + trp[(size_t)k], tri.begin() + trp[(size_t)k + 1],
		          ind.begin() + ptr[(size_t)tmp.ray_out[k]]);
	std::vector<real> val((size_t)std::max(tmp.nnz, 1LL), (real)scale);
	expand(m, n, ptr, ind, val.data(), nullptr, 1);
}

void prepare_op(cudaStream_t s, const tval3g_problem &p, int flags, OpStore &st, bool keep_ray_csr) {
	if (p.complex_data) {
		prepare_complex_op(s, p, flags, st, keep_ray_csr);
		return;
	}
	OpDev &d = st.dev;
	d = OpDev{};
	d.kind = p.op_kind;
	d.layers = (p.dims == 2 && (p.op_kind == TVAL3G_OP_DENSE || p.op_kind == TVAL3G_OP_CSR)) ? p.layers : 1;
	const long long n = (long long)p.dim_x * p.dim_y * (p.dims == 3 ? p.dim_z : 1);
	const bool borrow = (flags & TVAL3G_DEVICE_INPUTS) != 0;
	d.scale = 1.f;
	if (p.op_kind == TVAL3G_OP_DENSE) {
		d.m = p.m; d.n = p.n_cols;
		d.A = dcopy(s, st, prob_A(p), (long long)p.m * p.n_cols, borrow);
		st.b_len = (long long)p.m * d.layers;
#ifndef TVAL3G_FP64   // the tensor-core path takes FP32 data
		if (!(flags & TVAL3G_NO_TENSOR) && mrhs_eligible(d.m, d.n, d.layers)) {
			st.mrhs = mrhs_create(s, d.A, d.m, d.n, d.layers);
			st.bytes += st.mrhs->bytes;
			d.mrhs = 1;
		}
#endif
	} else if (p.op_kind == TVAL3G_OP_CSR) {
		d.m = p.m; d.n = p.n_cols;
		st.nnz = p.nnz;
		if (!borrow) {   // host arrays can be checked here (the reference trusts them)
			TG_ARG(p.csr_ptr[0] == 0 && p.csr_ptr[p.m] == p.nnz, "Argument error: CSR row pointers are inconsistent");
			for (int i = 0; i < p.m; i++)
				TG_ARG(p.csr_ptr[i + 1] >= p.csr_ptr[i], "Argument error: CSR row pointers are not monotone");
			for (long long k = 0; k < p.nnz; k++)
				TG_ARG(p.csr_ind[k] >= 0 && p.csr_ind[k] < p.n_cols, "Argument error: CSR column index out of range");
		}
		d.rptr = dcopy(s, st, p.csr_ptr, (long long)p.m + 1, borrow);
		d.rind = dcopy(s, st, p.csr_ind, p.nnz, borrow);
		d.rval = dcopy(s, st, prob_val(p), p.nnz, borrow);
		int *cptr = dalloc_op<int>(s, st, d.n + 1);
		int *cind = dalloc_op<int>(s, st, p.nnz);
		real *cval = dalloc_op<real>(s, st, p.nnz);
		build_transpose(s, d.m, d.n, p.nnz, d.rptr, d.rind, d.rval, cptr, cind, cval);
		d.cptr = cptr; d.cind = cind; d.cval = cval;
		st.adj_index_bytes = (long long)sizeof(int) * (d.n + 1) + 8LL * p.nnz;
		st.b_len = (long long)p.m * d.layers;
	} else {
		// traced rays in the reference's loop order (mp, emitter, receiver),
		// packed on the device from the geometry (use_path and endpoints)
		const bool is3 = p.op_kind == TVAL3G_OP_RAY3D;
		const int E = p.num_emitters, R = p.num_receivers, nmp = is3 ? p.numMPs : 1;
		const long long mtot = is3 ? (long long)p.numPaths * p.numMPs : (long long)E * R;
		RayGeo g{};
		g.E = E; g.R = R; g.is3 = is3; g.numPaths = is3 ? p.numPaths : 0; g.mtot = mtot;
		g.nx = is3 ? p.rv_x : (int)p.ld;
		g.ny = is3 ? p.rv_y : (int)std::min<long long>(n / p.ld, 32767);
		g.nz = is3 ? p.rv_z : 1;
		const long long ER = (long long)E * R, cand = (long long)nmp * ER;
		std::vector<void *> tmp;
		auto up = [&](const int *h, long long cnt) {   // a temporary device copy of a geometry array
			int *dp = (int *)dev_alloc(sizeof(int) * (size_t)std::max(cnt, 1LL), s);
			tmp.push_back(dp);
			if (cnt > 0) TG_CUDA(cudaMemcpyAsync(dp, h, sizeof(int) * (size_t)cnt, cudaMemcpyHostToDevice, s));
			return (const int *)dp;
		};
		g.up = up(p.use_path, ER);
		g.xe = up(p.x_emitters, (long long)nmp * E); g.ye = up(p.y_emitters, (long long)nmp * E);
		g.xr = up(p.x_receivers, (long long)nmp * R); g.yr = up(p.y_receivers, (long long)nmp * R);
		g.ze = is3 ? up(p.z_emitters, (long long)nmp * E) : nullptr;
		g.zr = is3 ? up(p.z_receivers, (long long)nmp * R) : nullptr;
		long long nr = 0;
		int4 *drays = nullptr;
		int *dout = nullptr;
		try {
			pack_rays(s, g, cand, &nr, &drays, &dout);   // throws the reference's argument errors
		} catch (...) {
			for (void *q : tmp) dev_free(q, s);
			throw;
		}
		for (void *q : tmp) dev_free(q, s);
		TG_ARG(nr < (1LL << 31), "Argument error: too many rays");
		st.owned.push_back(drays); st.owned.push_back(dout);
		st.bytes += (long long)(sizeof(int4) + sizeof(int)) * std::max(nr, 1LL);
		d.nrays = (int)nr;
		d.m = mtot; d.n = n;
		d.rvx = is3 ? p.rv_x : p.ld;
		d.rvy = is3 ? p.rv_y : 1;
		d.scale = p.scale_factor;
		d.rays = drays;
		st.ray_out.clear();
		if (keep_ray_csr && nr > 0) {   // the host copy the CSR export and the complex form read
			st.ray_out.resize((size_t)nr);
			TG_CUDA(cudaMemcpyAsync(st.ray_out.data(), dout, sizeof(int) * (size_t)nr, cudaMemcpyDeviceToHost, s));
		}
		// forward CSR over traced rays, then its transpose: the pixel-major
		// index of the adjoint, entries = measurement indices sorted by ray
		int *rptr = dalloc_op<int>(s, st, (long long)d.nrays + 1);
		long long total = 0;
		int *rind = trace_rays(s, d.nrays, drays, d.rvx, d.rvy, rptr, &total);
		st.owned.push_back(rind);
		st.bytes += (long long)sizeof(int) * std::max(total, 1LL);
		st.nnz = total;
		d.adj_atomic = (flags & TVAL3G_RAY_ADJ_ATOMICS) != 0;
		const bool tile_ok = !d.adj_atomic && !(flags & TVAL3G_RAY_ADJ_PLAIN);
		// 3D: each hit's position in its brick's ray list, carried through the
		// transpose (the brick-tiled adjoint)
		BrickLists bl;
		real *posf = nullptr, *cposf = nullptr;
		if (is3 && tile_ok) {
			const int *lo = dout;
			posf = brick_positions(s, p.rv_x, p.rv_y, p.rv_z, d.nrays, total, rptr, rind, lo, bl, st.owned);
			if (posf) cposf = (real *)dev_alloc(sizeof(real) * (size_t)std::max(total, 1LL), s);
		}
		int *cptr = dalloc_op<int>(s, st, n + 1);
		int *cind = dalloc_op<int>(s, st, total);
		build_transpose(s, d.nrays, n, total, rptr, rind, posf, cptr, cind, cposf);
		if (posf) {
			long long ib = 0;
			if (build_brick_words(s, p.rv_x, p.rv_y, p.rv_z, cptr, cposf, bl, d, &ib, st.owned)) {
				st.bytes += ib;
				st.adj_index_bytes = ib;
			}
			dev_free(posf, s);
			dev_free(cposf, s);
		}
		if (!is3 && n % p.ld == 0) {   // transposed image for the y-driven rays
			d.xT = dalloc_op<real>(s, st, n);
			d.tH = (int)(n / p.ld);
		}
		if (!is3 && n % p.ld == 0 && d.nrays > 0 && d.nrays <= RAYT_MAX_RAYS && tile_ok) {
			// tiled adjoint (cind still holds traced-ray ids)
			const int *lo = dout;
			long long ib = 0;
			if (build_tiled_index(s, (int)p.ld, (int)(n / p.ld), d.nrays, cptr, cind, lo, d, &ib, st.owned)) {
				st.bytes += ib;
				st.adj_index_bytes = ib;
				if (const char *e = std::getenv("TVAL3G_TEST_FIRST_WAIT_POLLS"))   // failure-path test hook
					d.first_wait_polls = 1u + (unsigned)std::strtoul(e, nullptr, 10);
			}
		}
		if (!d.tiled) {   // pixel-major gather over measurement indices
			st.adj_index_bytes = (long long)sizeof(int) * (n + 1 + total);
			if (total > 0) k_map_out<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(total, drays, cind);
			TG_CUDA(cudaGetLastError());
			d.cptr = cptr; d.cind = cind;
		} else {          // the tiled index replaces the pixel-major one
			for (void *&q : st.owned)
				if (q == cptr || q == cind) {
					st.bytes -= q == cptr ? (long long)sizeof(int) * (n + 1) : (long long)sizeof(int) * std::max(total, 1LL);
					dev_free(q, s);
					q = nullptr;
				}
			d.cptr = nullptr; d.cind = nullptr;
		}
		d.cval = nullptr;
		st.ray_rptr = rptr; st.ray_rind = rind;
		st.b_len = mtot;
		if (!keep_ray_csr) {   // (stream-ordered frees: the kernels queued before them still read them)
			for (void *&q : st.owned)
				if (q == rptr || q == rind) { dev_free(q, s); q = nullptr; }
			st.ray_rptr = st.ray_rind = nullptr;
		}
	}
}

void free_op(OpStore &st, cudaStream_t s) {
	for (void *q : st.owned) dev_free(q, s);
	st.owned.clear();
	st.mrhs.reset();
}

// ---------------------------------------------------------------------------
// tile maps
// ---------------------------------------------------------------------------
struct TileBuilder {
	std::vector<int2> all;
	struct Pending { TileMap *map; size_t off; size_t cnt; };
	std::vector<Pending> pend;
	std::vector<int2> cur;
	void add(int inst, long long tiles) {
		for (long long t = 0; t < tiles; t++) cur.push_back(make_int2(inst, (int)t));
	}
	void close(TileMap *m) {
		pend.push_back({m, all.size(), cur.size()});
		all.insert(all.end(), cur.begin(), cur.end());
		cur.clear();
	}
	int2 *upload(cudaStream_t s) {
		int2 *d = (int2 *)dev_alloc(sizeof(int2) * std::max<size_t>(all.size(), 1), s);
		if (!all.empty())
			TG_CUDA(cudaMemcpyAsync(d, all.data(), sizeof(int2) * all.size(), cudaMemcpyHostToDevice, s));
		for (auto &p : pend) {
			p.map->tiles = d + p.off;
			p.map->count = (int)p.cnt;
		}
		return d;
	}
};

// lanes per line of the compressed gathers: about eight entries per lane, so
// that the gather's four-deep unrolled steps run (a 3D voxel's ~60 hits: 8
// lanes; a CSR row of ~200: 16)
static int subwarp_for(double avg) {
	if (avg >= 256) return 32;
	if (avg >= 128) return 16;
	if (avg >= 32) return 8;
	return 4;
}

// operator tile maps of a batch; returns the dense partial buffer size (elements)
static long long build_op_maps(std::vector<Inst> &inst, const std::vector<OpStore> &ops, TileBuilder &tb,
                               OpBatch &ob) {
	const int cnt = (int)inst.size();
	long long dense_part = 0;
	// dense operators of one layer: the normal product reads A once
	ob.fused.clear();
	ob.fused_grid = fused_grid();
	ob.fused_words = 0;
	for (int i = 0; i < cnt; i++) {
		OpDev &d = inst[i].op;
		d.fused_rpc = 0;
		if (d.kind != TVAL3G_OP_DENSE || d.mrhs || d.layers != 1) continue;
		d.fused_rpc = fused_rows_per_cta(d.m, d.n, ob.fused_grid, d.A, &d.fused_slab);
		if (d.fused_rpc <= 0) continue;
		const long long R = (long long)ob.fused_grid * d.fused_rpc;
		const int bands = (int)((d.m + R - 1) / R);
		ob.fused.push_back({i, bands, ob.fused_words});
		ob.fused_words += bands;
	}
	// dense gemv maps: all dense instances, then those outside the fused set
	for (int nf = 0; nf < 2; nf++) {
		for (int i = 0; i < cnt; i++) {
			OpDev &d = inst[i].op;
			if (d.kind != TVAL3G_OP_DENSE || d.mrhs || (nf && d.fused_rpc)) continue;
			tb.add(i, d.layers * ((d.m + WARPS - 1) / WARPS));
		}
		tb.close(nf ? &ob.dense_fwd_nf : &ob.dense_fwd);
	}
	for (int i = 0; i < cnt; i++) {
		OpDev &d = inst[i].op;
		if (d.kind != TVAL3G_OP_DENSE) continue;
		if (d.mrhs) {   // independent right-hand sides: the group's first instance holds the operator
			if (ops[i].mrhs) ob.mrhs.emplace_back(i, ops[i].mrhs);
			continue;
		}
		long long ct = (d.n + 1023) / 1024;
		long long K = (4 * 148 + d.layers * ct - 1) / (d.layers * ct);
		K = std::max(1LL, std::min(K, d.m));
		d.dense_kchunks = (int)K;
		d.dense_part = dense_part;
		dense_part += d.layers * K * d.n;
	}
	for (int nf = 0; nf < 2; nf++) {
		for (int i = 0; i < cnt; i++) {
			const OpDev &d = inst[i].op;
			if (d.kind != TVAL3G_OP_DENSE || d.mrhs || (nf && d.fused_rpc)) continue;
			tb.add(i, d.layers * ((d.n + 1023) / 1024) * d.dense_kchunks);
		}
		tb.close(nf ? &ob.dense_adj_nf : &ob.dense_adj);
		for (int i = 0; i < cnt; i++) {
			const OpDev &d = inst[i].op;
			if (d.kind != TVAL3G_OP_DENSE || d.mrhs || (nf && d.fused_rpc)) continue;
			tb.add(i, d.layers * ((d.n + 31) / 32));
		}
		tb.close(nf ? &ob.dense_red_nf : &ob.dense_red);
	}
	// compressed gathers: each instance in the width class of its own mean
	// line length (lines per block = 256 / width)
	// (or in the class the autotuner measured fastest, OpDev::gcls_*)
	static const int widths[4] = {4, 8, 16, 32};
	auto cls = [](double avg, int tuned) {
		if (tuned > 0) return tuned - 1;
		int w = subwarp_for(avg);
		return w == 4 ? 0 : w == 8 ? 1 : w == 16 ? 2 : 3;
	};
	for (int c = 0; c < 4; c++) {
		for (int i = 0; i < cnt; i++) {
			const OpDev &d = inst[i].op;
			if (d.kind != TVAL3G_OP_CSR || cls((double)ops[i].nnz / d.m, d.gcls_fwd) != c) continue;
			long long lpb = 256 / widths[c];
			tb.add(i, d.layers * ((d.m + lpb - 1) / lpb));
		}
		tb.close(&ob.csr_fwd[c]);
		for (int i = 0; i < cnt; i++) {
			const OpDev &d = inst[i].op;
			if (d.kind != TVAL3G_OP_CSR || cls((double)ops[i].nnz / d.n, d.gcls_adj) != c) continue;
			long long lpb = 256 / widths[c];
			tb.add(i, d.layers * ((d.n + lpb - 1) / lpb));
		}
		tb.close(&ob.csc_adj[c]);
		for (int i = 0; i < cnt; i++) {
			const OpDev &d = inst[i].op;
			if ((d.kind != TVAL3G_OP_RAY2D && d.kind != TVAL3G_OP_RAY3D) || d.tiled || d.adj_atomic ||
			    cls((double)ops[i].nnz / inst[i].n, d.gcls_adj) != c)
				continue;
			long long lpb = 256 / widths[c];
			tb.add(i, (inst[i].n + lpb - 1) / lpb);
		}
		tb.close(&ob.ray_adj[c]);
	}
	// ray forwards by lanes per ray (RAY_SUBW unless tuned)
	for (int dim3 = 0; dim3 < 2; dim3++)
		for (int c = 0; c < 3; c++) {
			for (int i = 0; i < cnt; i++) {
				const OpDev &d = inst[i].op;
				if (d.kind != (dim3 ? TVAL3G_OP_RAY3D : TVAL3G_OP_RAY2D)) continue;
				const int lanes = d.fwd_lanes > 0 ? d.fwd_lanes : RAY_SUBW;
				if (lanes != RAY_LANES[c]) continue;
				const int rpb = 256 / lanes;
				tb.add(i, (d.nrays + rpb - 1) / rpb);
			}
			tb.close(dim3 ? &ob.ray3_fwd[c] : &ob.ray2_fwd[c]);
		}
	for (int i = 0; i < cnt; i++) {
		const OpDev &d = inst[i].op;
		if (d.kind != TVAL3G_OP_RAY2D || !d.xT) continue;
		tb.add(i, (long long)((d.rvx + 31) / 32) * ((d.tH + 31) / 32));
	}
	tb.close(&ob.ray2_transpose);
	// adjoints by on-the-fly tracing with atomic adds
	for (int i = 0; i < cnt; i++)
		if (inst[i].op.adj_atomic) tb.add(i, (inst[i].n + ATOMIC_ZERO_TILE - 1) / ATOMIC_ZERO_TILE);
	tb.close(&ob.ray_atomic_zero);
	for (int dim3 = 0; dim3 < 2; dim3++) {
		for (int i = 0; i < cnt; i++) {
			const OpDev &d = inst[i].op;
			if (!d.adj_atomic || d.kind != (dim3 ? TVAL3G_OP_RAY3D : TVAL3G_OP_RAY2D)) continue;
			tb.add(i, (d.nrays + RAYS_PER_BLOCK - 1) / RAYS_PER_BLOCK);
		}
		tb.close(dim3 ? &ob.ray3_adj_atomic : &ob.ray2_adj_atomic);
	}
	ob.tiled_tmax = 0;
	for (int i = 0; i < cnt; i++) {
		const OpDev &d = inst[i].op;
		if (!d.tiled || d.adj_atomic) continue;
		tb.add(i, d.ntiles);
		ob.tiled_tmax = std::max(ob.tiled_tmax, d.tmax);
	}
	tb.close(&ob.ray_adj_tiled);
	return dense_part;
}

long long build_op_maps_upload(std::vector<Inst> &inst, const std::vector<OpStore> &ops, OpBatch &ob,
                               int2 **d_tiles, cudaStream_t s) {
	TileBuilder tb;
	long long dense_part = build_op_maps(inst, ops, tb, ob);
	*d_tiles = tb.upload(s);
	return dense_part;
}

// ---------------------------------------------------------------------------
// Plan
// ---------------------------------------------------------------------------
void *Plan::dalloc(size_t bytes) {
	void *p = dev_alloc(bytes, stream_);
	allocs_.push_back(p);
	device_bytes_ += (long long)bytes;
	return p;
}

// Independent right-hand sides: dense instances of one layer whose A is the
// same device matrix (TVAL3G_DEVICE_INPUTS: the same pointer and shape) are
// cut into groups of 64, 48, 32 or 16 (largest first, in instance order),
// and each group shares one tensor-core operator (mrhs.cu): every product of
// the group is one 3xTF32 contraction over its members' vectors, each member
// keeping its own scalar control (step lengths, line search, stopping).
// Members left over (fewer than 16) keep their own gemv products.
void Plan::group_shared_dense(const tval3g_problem *probs, int flags) {
#ifdef TVAL3G_FP64   // the tensor-core path takes FP32 data
	(void)probs;
	(void)flags;
	return;
#else
	if (!(flags & TVAL3G_DEVICE_INPUTS) || (flags & TVAL3G_NO_TENSOR)) return;
	std::map<std::tuple<const float *, int, int, int>, std::vector<int>> by_a;
	for (int i = 0; i < count_; i++) {
		const tval3g_problem &p = probs[i];
		if (p.op_kind == TVAL3G_OP_DENSE && ops_[i].dev.layers == 1 && !p.complex_data && p.A && !ops_[i].dev.mrhs)
			by_a[std::make_tuple(p.A, p.m, p.n_cols, p.dims)].push_back(i);
	}
	for (const auto &kv : by_a) {
		const std::vector<int> &v = kv.second;
		const long long m = std::get<1>(kv.first), n = std::get<2>(kv.first);
		size_t k = 0;
		while (v.size() - k >= 16) {
			int sz = 0;
			for (int c : {64, 48, 32, 16})
				if ((size_t)c <= v.size() - k && mrhs_eligible(m, n, c)) { sz = c; break; }
			if (!sz) break;
			std::vector<int> mem(v.begin() + k, v.begin() + k + sz);
			auto op = mrhs_create(stream_, ops_[mem[0]].dev.A, m, n, sz);
			mrhs_set_members(stream_, *op, mem.data());
			ops_[mem[0]].mrhs = op;
			ops_[mem[0]].bytes += op->bytes;
			for (int i : mem) {
				ops_[i].dev.mrhs = 1;
				h_inst_[i].op.mrhs = 1;
			}
			k += sz;
		}
	}
#endif
}

Plan::Plan(int count, const tval3g_problem *probs, const tval3g_options *opts, int flags)
	: count_(count), flags_(flags), graph_mode_((flags & TVAL3G_GRAPH) != 0) {
	TG_ARG(count >= 1, "Argument error: count must be >= 1");
	int dev = 0;
	if (cudaGetDevice(&dev) != cudaSuccess) throw Error{TVAL3G_ERR_NO_DEVICE, "no CUDA device"};
	for (int i = 0; i < count; i++) check_options(opts[i]);
	TG_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
	ops_.resize(count);
	h_inst_.assign(count, Inst{});
	try {
		// operators and sizes
		for (int i = 0; i < count; i++) {
			const tval3g_problem &p = probs[i];
			long long b_len = (p.op_kind == TVAL3G_OP_RAY2D) ? (long long)p.num_emitters * p.num_receivers
			                  : (p.op_kind == TVAL3G_OP_RAY3D) ? (long long)p.numPaths * p.numMPs
			                  : (long long)p.m * (p.dims == 3 ? 1 : p.layers);
			long long n = validate(p, b_len, 0, false);   // the callers validated p
			prepare_op(stream_, p, flags, ops_[i], false);
			Inst &I = h_inst_[i];
			const int planes = p.complex_data ? 2 : 1;   // complex: real and imaginary planes
			I.dims = p.dims; I.p = p.dim_y; I.q = p.dim_x; I.r = p.dims == 3 ? p.dim_z : planes;
			I.fq.init((unsigned)I.q);
			I.fp.init((unsigned)I.p);
			I.n = n * planes; I.m = b_len * planes;
			I.cplx = p.complex_data != 0;
			n = I.n;
			b_len = I.m;
			I.ept = ept_for(n);
			I.ntn = (int)((n + (long long)BLOCK * I.ept - 1) / ((long long)BLOCK * I.ept));
			I.ntm = (int)((b_len + TILE_M - 1) / TILE_M);
			const tval3g_options &o = opts[i];
			I.muf = o.mu; I.betaf = o.beta; I.mu0 = o.mu0; I.beta0 = o.beta0; I.tol = o.tol; I.tol_inn = o.tol_inn;
			I.c = o.c; I.gamma = o.gamma; I.gam0 = o.gam; I.rate_gam = o.rate_gam; I.rate_cnt = o.rate_cnt;
			I.skipRatio = o.skipMulRatio; I.maxRelChange = o.maxRelativeChange;
			I.maxit = o.maxit; I.maxcnt = o.maxcnt; I.nonneg = o.nonneg != 0; I.tv_norm = o.tv_norm;
			I.isreal = o.isreal != 0;
			I.numInit = o.numInitIterations;
			I.skip_enabled = (o.skipMulRatio != 0 && p.op_kind != TVAL3G_OP_DENSE);
			any_skip_ |= I.skip_enabled != 0;
			any_cplx_ |= I.cplx != 0;
#ifndef TVAL3G_FP64   // the autotuner measures the FP32 kernels
			if (flags & TVAL3G_TUNE) autotune_operator(stream_, ops_[i], I);
#endif
			I.op = ops_[i].dev;
		}
		group_shared_dense(probs, flags);
		// vectors: one arena, every vector 256-byte aligned
		long long total = 0;
		std::vector<long long> base(count);
		for (int i = 0; i < count; i++) {
			long long np = (h_inst_[i].n + 63) / 64 * 64, mp = (h_inst_[i].m + 63) / 64 * 64;
			base[i] = total;
			total += NVN * np + NVM * mp;
		}
		d_arena_ = (real *)dalloc(sizeof(real) * (size_t)total);
		long long parts = 0;
		for (int i = 0; i < count; i++) parts += (long long)(h_inst_[i].ntn + h_inst_[i].ntm) * NSUM;
		d_part_ = (double *)dalloc(sizeof(double) * (size_t)parts);
		d_ctrl_ = (Ctrl *)dalloc(sizeof(Ctrl) * count);
		TG_CUDA(cudaMemsetAsync(d_ctrl_, 0, sizeof(Ctrl) * count, stream_));
		if (flags & PLAN_SCHEDULE) {
			const int K = h_inst_[0].maxit;
			for (int i = 0; i < count; i++)
				TG_ARG(h_inst_[i].maxit == K && K >= 1, "Argument error: a schedule needs one maxit >= 1");
			sched_mode_ = true;
			d_sched_ = (double *)dalloc(sizeof(double) * 2 * (size_t)K);
			std::vector<double> def(2 * (size_t)K);
			for (int k = 0; k < K; k++) { def[k] = h_inst_[0].mu0; def[K + k] = h_inst_[0].beta0; }
			TG_CUDA(cudaMemcpyAsync(d_sched_, def.data(), sizeof(double) * def.size(), cudaMemcpyHostToDevice, stream_));
			TG_CUDA(cudaStreamSynchronize(stream_));
			for (int i = 0; i < count; i++) h_inst_[i].sched = d_sched_;
		}
		if (flags & TVAL3G_TRACE) {
			long long recs = 0;
			for (int i = 0; i < count; i++) {
				trace_off_.push_back(recs);
				recs += std::max(h_inst_[i].maxit, 1);
			}
			d_trace_ = (double *)dalloc(sizeof(tval3g_trace_record) * (size_t)recs);
			TG_CUDA(cudaMemsetAsync(d_trace_, 0, sizeof(tval3g_trace_record) * (size_t)recs, stream_));
			for (int i = 0; i < count; i++) h_inst_[i].trace = d_trace_ + TRACE_DOUBLES * trace_off_[i];
		}
		long long poff = 0;
		for (int i = 0; i < count; i++) {
			Inst &I = h_inst_[i];
			long long np = (I.n + 63) / 64 * 64, mp = (I.m + 63) / 64 * 64;
			real *b0 = d_arena_ + base[i];
			for (int v = 0; v < NVN; v++) I.vn[v] = b0 + v * np;
			for (int v = 0; v < NVM; v++) I.vm[v] = b0 + NVN * np + v * mp;
			I.ctrl = d_ctrl_ + i;
			I.part = d_part_ + poff;
			poff += (long long)(I.ntn + I.ntm) * NSUM;
		}
		// tile maps
		TileBuilder tb;
		for (int i = 0; i < count; i++) tb.add(i, h_inst_[i].ntn);
		tb.close(&maps_[MAP_N]);
		for (int i = 0; i < count; i++) tb.add(i, h_inst_[i].ntm);
		tb.close(&maps_[MAP_M]);
		for (int i = 0; i < count; i++) tb.add(i, h_inst_[i].ntn + h_inst_[i].ntm);
		tb.close(&maps_[MAP_NM]);
		long long dense_part = build_op_maps(h_inst_, ops_, tb, ob_);
		d_tiles_ = tb.upload(stream_);
		allocs_.push_back(d_tiles_);
		if (dense_part > 0) ob_.dense_part = (real *)dalloc(sizeof(real) * (size_t)dense_part);
		if (ob_.fused_words > 0) {
			ob_.fused_flags = (int *)dalloc(sizeof(int) * (size_t)ob_.fused_words);
			TG_CUDA(cudaMemsetAsync(ob_.fused_flags, 0, sizeof(int) * (size_t)ob_.fused_words, stream_));
		}
		ob_.err = (int *)dalloc(sizeof(int));
		TG_CUDA(cudaMemsetAsync(ob_.err, 0, sizeof(int), stream_));
		d_inst_ = (Inst *)dalloc(sizeof(Inst) * count);
		TG_CUDA(cudaMemcpyAsync(d_inst_, h_inst_.data(), sizeof(Inst) * count, cudaMemcpyHostToDevice, stream_));
		d_flag_ = (int *)dalloc(sizeof(int));
		d_launches_ = (unsigned long long *)dalloc(sizeof(unsigned long long));
		for (auto &o : ops_) device_bytes_ += o.bytes;
		// the graph is captured and instantiated while the operator
		// preparation still runs on the device, and uploaded behind it
		if (graph_mode_) {
			build_graph();
			TG_CUDA(cudaGraphUpload(exec_, stream_));
		}
		TG_CUDA(cudaStreamSynchronize(stream_));
	} catch (...) {
		release();
		throw;
	}
}

Plan::~Plan() { release(); }

void Plan::time_stencils(int reps, double ms[3]) {
	cur_ = stream_;
	const bool gm = graph_mode_;
	graph_mode_ = false;   // es() is the launch stream
	cudaEvent_t e0 = nullptr, e1 = nullptr;
	try {
		TG_CUDA(cudaEventCreate(&e0));
		TG_CUDA(cudaEventCreate(&e1));
		for (int k = 0; k < 3; k++) {
			auto launch = [&] {
				if (k == 0) launch_getg(stream_, kargs(MAP_NM, P_ALL, ST_DESCEND));
				else if (k == 1) launch_descend(stream_, kargs(MAP_NM, P_ALL, ST_DESCEND));
				else launch_shrink_grad(stream_, kargs(MAP_N, P_ALL, ST_LOOP));
			};
			launch();   // warm
			TG_CUDA(cudaEventRecord(e0, stream_));
			for (int r = 0; r < reps; r++) launch();
			TG_CUDA(cudaEventRecord(e1, stream_));
			TG_CUDA(cudaEventSynchronize(e1));
			float t = 0.f;
			TG_CUDA(cudaEventElapsedTime(&t, e0, e1));
			ms[k] = (double)t / std::max(reps, 1);
		}
	} catch (...) {
		graph_mode_ = gm;
		if (e0) cudaEventDestroy(e0);
		if (e1) cudaEventDestroy(e1);
		throw;
	}
	graph_mode_ = gm;
	cudaEventDestroy(e0);
	cudaEventDestroy(e1);
}

int Plan::trace(int index, tval3g_trace_record *out, int cap) const {
	TG_ARG(d_trace_ != nullptr, "Argument error: the plan was created without TVAL3G_TRACE");
	TG_ARG(index >= 0 && index < count_, "Argument error: instance index out of range");
	int n = index < (int)last_iters_.size() ? std::min(last_iters_[index], h_inst_[index].maxit) : 0;
	n = std::min(n, cap);
	if (n > 0)
		TG_CUDA(cudaMemcpy(out, d_trace_ + TRACE_DOUBLES * trace_off_[index], sizeof(tval3g_trace_record) * n,
		                   cudaMemcpyDeviceToHost));
	return n;
}

void Plan::release() {
	if (exec_) cudaGraphExecDestroy(exec_);
	if (graph_) cudaGraphDestroy(graph_);
	exec_ = nullptr; graph_ = nullptr;
	if (cap_) cudaStreamDestroy(cap_);
	cap_ = nullptr;
	if (stream_) cudaStreamSynchronize(stream_);
	for (void *p : allocs_) dev_free(p, stream_);
	allocs_.clear();
	ob_.mrhs.clear();
	for (auto &o : ops_) free_op(o, stream_);
	ops_.clear();
	if (stream_) cudaStreamDestroy(stream_);
	stream_ = nullptr;
}

KArgs Plan::kargs(MapKind mk, int pred, int stage) const {
	KArgs a;
	a.tab = d_inst_;
	a.map = maps_[mk];
	a.pred = pred;
	a.stage = stage;
	a.multi = 0;
	for (const Inst &I : h_inst_) a.multi |= I.ept > 1 ? 1 : 0;
	a.launches = d_launches_;
	return a;
}

LaunchCtx Plan::lctx() const {
	LaunchCtx L;
	L.stream = es();
	L.inst = d_inst_;
	L.launches = (long long *)d_launches_;
	return L;
}

// --- control flow -----------------------------------------------------------
void Plan::seg_begin() {
	Frame &f = frames_.back();
	TG_CUDA(cudaStreamBeginCaptureToGraph(cap_, f.g, f.deps.empty() ? nullptr : f.deps.data(), nullptr,
	                                      f.deps.size(), cudaStreamCaptureModeRelaxed));
	capturing_ = true;
}

void Plan::seg_end() {
	Frame &f = frames_.back();
	cudaStreamCaptureStatus st;
	const cudaGraphNode_t *deps = nullptr;
	size_t nd = 0;
	TG_CUDA(cudaStreamGetCaptureInfo(cap_, &st, nullptr, nullptr, &deps, &nd));
	std::vector<cudaGraphNode_t> d(deps, deps + nd);
	cudaGraph_t g;
	TG_CUDA(cudaStreamEndCapture(cap_, &g));
	f.deps = d;
	capturing_ = false;
}

unsigned long long Plan::cond_handle() {
	// single-instance graph plans: the deciding kernel sets the condition
	if (!graph_mode_ || count_ != 1) return 0ull;
	cudaGraphConditionalHandle h;
	TG_CUDA(cudaGraphConditionalHandleCreate(&h, frames_.back().g, 0, cudaGraphCondAssignDefault));
	return (unsigned long long)h;
}

void Plan::if_(int pred, const std::function<void()> &body, unsigned long long hset) {
	if (!graph_mode_) {
		launch_cond(cur_, d_inst_, count_, pred, d_flag_, 0, d_launches_);
		TG_CUDA(cudaMemcpyAsync(&h_flag_, d_flag_, sizeof(int), cudaMemcpyDeviceToHost, cur_));
		TG_CUDA(cudaStreamSynchronize(cur_));
		if (h_flag_) body();
		return;
	}
	cudaGraphConditionalHandle h = (cudaGraphConditionalHandle)hset;
	if (!hset) {
		TG_CUDA(cudaGraphConditionalHandleCreate(&h, frames_.back().g, 0, cudaGraphCondAssignDefault));
		launch_cond(cap_, d_inst_, count_, pred, d_flag_, (unsigned long long)h, d_launches_);
	}
	seg_end();
	alignas(cudaGraphNodeParams) unsigned char np_raw[sizeof(cudaGraphNodeParams)] = {};
	cudaGraphNodeParams &np = *reinterpret_cast<cudaGraphNodeParams *>(np_raw);
	np.type = cudaGraphNodeTypeConditional;
	np.conditional.handle = h;
	np.conditional.type = cudaGraphCondTypeIf;
	np.conditional.size = 1;
	cudaGraphNode_t node;
	{
		Frame &f = frames_.back();
		TG_CUDA(cudaGraphAddNode(&node, f.g, f.deps.empty() ? nullptr : f.deps.data(), f.deps.size(), &np));
	}
	frames_.push_back(Frame{np.conditional.phGraph_out[0], {}});
	seg_begin();
	body();
	seg_end();
	frames_.pop_back();
	frames_.back().deps.assign(1, node);
	seg_begin();
}

void Plan::while_(int pred, const std::function<void()> &body, unsigned long long hset) {
	if (!graph_mode_) {
		for (;;) {
			launch_cond(cur_, d_inst_, count_, pred, d_flag_, 0, d_launches_);
			TG_CUDA(cudaMemcpyAsync(&h_flag_, d_flag_, sizeof(int), cudaMemcpyDeviceToHost, cur_));
			TG_CUDA(cudaStreamSynchronize(cur_));
			if (!h_flag_) break;
			body();
		}
		return;
	}
	cudaGraphConditionalHandle h = (cudaGraphConditionalHandle)hset;
	if (!hset) {
		TG_CUDA(cudaGraphConditionalHandleCreate(&h, frames_.back().g, 0, cudaGraphCondAssignDefault));
		launch_cond(cap_, d_inst_, count_, pred, d_flag_, (unsigned long long)h, d_launches_);
	}
	seg_end();
	alignas(cudaGraphNodeParams) unsigned char np_raw[sizeof(cudaGraphNodeParams)] = {};
	cudaGraphNodeParams &np = *reinterpret_cast<cudaGraphNodeParams *>(np_raw);
	np.type = cudaGraphNodeTypeConditional;
	np.conditional.handle = h;
	np.conditional.type = cudaGraphCondTypeWhile;
	np.conditional.size = 1;
	cudaGraphNode_t node;
	{
		Frame &f = frames_.back();
		TG_CUDA(cudaGraphAddNode(&node, f.g, f.deps.empty() ? nullptr : f.deps.data(), f.deps.size(), &np));
	}
	frames_.push_back(Frame{np.conditional.phGraph_out[0], {}});
	seg_begin();
	body();
	if (!hset) launch_cond(cap_, d_inst_, count_, pred, d_flag_, (unsigned long long)h, d_launches_);
	seg_end();
	frames_.pop_back();
	frames_.back().deps.assign(1, node);
	seg_begin();
}

// --- the program (2d/tval3_cpu_2d.cpp:752-886) ---------------------------------
void Plan::emit_program() {
	cudaStream_t s = es();
	const LaunchCtx L = lctx();
	const VecSel U{false, vU}, Atb{false, vAtb}, G{false, vG}, D{false, vD};
	const VecSel B{true, vB}, Au{true, vAu}, Ad{true, vAd};
	// initialisation: scaleb, Atb = A'b, U = Atb, D, shrinkage, get_g, gradient
	launch_scaleb(s, kargs(MAP_M, P_ALL));
	launch_init(s, kargs(MAP_NM, P_ALL));
	op_adjoint(L, ob_, P_ALL, B, Atb);
	launch_init_u(s, kargs(MAP_N, P_ALL));
	launch_D(s, kargs(MAP_N, P_ALL));
	launch_shrink(s, kargs(MAP_N, P_ALL, ST_INIT));
	op_fused_normal(L, ob_, P_ALL, U, Au, G);
	op_forward(L, ob_, P_ALL, U, Au, true);
	if (any_skip_) launch_copy_lastau(s, kargs(MAP_M, P_ALL));
	op_adjoint(L, ob_, P_ALL, Au, G, true);
	launch_getg(s, kargs(MAP_NM, P_ALL, ST_INIT));
	const unsigned long long h_act = cond_handle();
	launch_grad(s, kargs(MAP_N, P_ALL, ST_INIT).cond(h_act, P_ACTIVE));
	if (!sched_mode_) emit_first_tau(h_act);
	(void)D; (void)Ad;
	while_(P_ACTIVE, [&] { emit_iteration(h_act); }, h_act);
	launch_final(es(), kargs(MAP_N, P_ALL));
}

std::vector<Ctrl> Plan::ctrl() const {
	std::vector<Ctrl> h(count_);
	TG_CUDA(cudaMemcpy(h.data(), d_ctrl_, sizeof(Ctrl) * count_, cudaMemcpyDeviceToHost));
	return h;
}

void Plan::set_schedule(const double *mu, const double *beta) {
	TG_ARG(sched_mode_, "Internal error: the plan has no schedule");
	const int K = h_inst_[0].maxit;
	std::vector<double> h(2 * (size_t)K);
	for (int k = 0; k < K; k++) {
		TG_ARG(mu[k] > 0 && beta[k] > 0, "Argument error: mu_k and beta_k must be positive");
		h[k] = mu[k];
		h[K + k] = beta[k];
	}
	TG_CUDA(cudaMemcpy(d_sched_, h.data(), sizeof(double) * h.size(), cudaMemcpyHostToDevice));
}

// The first-iteration step length (get_tau, 2d:430-442) of an inner loop:
// |D d|^2, then A d and tau.  Outside schedule mode it runs where an inner
// loop begins - after the initialisation and after each outer step - and the
// Barzilai-Borwein form of the other iterations comes from k_shrink_grad.
// Its kernels also set the loop's condition (h_active).
void Plan::emit_first_tau(unsigned long long h_active) {
	const VecSel D{false, vD}, Ad{true, vAd};
	const unsigned long long h_ad = cond_handle();
	launch_tau_prep(es(), kargs(MAP_N, P_FIRST).cond(h_ad, P_NEED_AD).cond(h_active, P_ACTIVE));
	if_(P_NEED_AD, [&] {
		op_forward(lctx(), ob_, P_NEED_AD, D, Ad);
		launch_tau_first(es(), kargs(MAP_M, P_NEED_AD).cond(h_active, P_ACTIVE));
	}, h_ad);
}

// h_active: the loop's condition handle when the iteration's last kernel sets
// it (0: a condition kernel evaluates it)
void Plan::emit_iteration(unsigned long long h_active) {
	const LaunchCtx L = lctx();
	cudaStream_t s = es();
	if (sched_mode_) launch_sched(s, d_inst_, count_, d_launches_);
	const VecSel U{false, vU}, G{false, vG}, D{false, vD};
	const VecSel Au{true, vAu}, Ad{true, vAd};
	// min_u (2d:526-576): step length
	// (outside schedule mode, where mu and beta change at the iteration's
	// start, tau is ready: emit_first_tau or the previous k_shrink_grad)
	if (sched_mode_) {
		const unsigned long long h_ad = cond_handle();
		launch_tau_prep(s, kargs(MAP_N, P_ACTIVE).cond(h_ad, P_NEED_AD));
		if_(P_NEED_AD, [&] {
			op_forward(lctx(), ob_, P_NEED_AD, D, Ad);
			launch_tau_first(es(), kargs(MAP_M, P_NEED_AD));
		}, h_ad);
	}
	// descent step and get_g
	launch_descend(es(), kargs(MAP_NM, P_ACTIVE, ST_DESCEND));   // D U: in k_getg
	// get_g_mult: dense instances in one pass over A (they never skip)
	op_fused_normal(lctx(), ob_, P_ACTIVE, U, Au, G);
	op_forward(lctx(), ob_, P_ACTIVE, U, Au, true, true);
	if (any_skip_) {
		launch_skip_norms(es(), kargs(MAP_M, P_ACTIVE));
		launch_copy_lastau(es(), kargs(MAP_M, P_ACTIVE_MUL));
	}
	op_adjoint(lctx(), ob_, P_ACTIVE_MUL, Au, G, true);
	const unsigned long long h_bt = cond_handle();
	launch_getg(es(), kargs(MAP_NM, P_ACTIVE, ST_DESCEND).cond(h_bt, P_NEED_BT));
	// nonmonotone Armijo backtracking, restart after five failures
	if_(P_NEED_BT, [&] {
		const unsigned long long h_lerp = cond_handle(), h_restart = cond_handle();
		launch_bt_search(es(), kargs(MAP_NM, P_NEED_BT).cond(h_lerp, P_NEED_BT).cond(h_restart, P_RESTART));
		if_(P_NEED_BT, [&] { launch_lerp(es(), kargs(MAP_NM, P_NEED_BT)); }, h_lerp);
		if_(P_RESTART, [&] {
			launch_tau_prep(es(), kargs(MAP_N, P_RESTART));
			op_forward(lctx(), ob_, P_NEED_AD, D, Ad);
			launch_tau_first(es(), kargs(MAP_M, P_NEED_AD));
			launch_descend(es(), kargs(MAP_NM, P_RESTART, ST_RESTART));
			op_fused_normal(lctx(), ob_, P_RESTART, U, Au, G);
			op_forward(lctx(), ob_, P_RESTART, U, Au, true, true);
			if (any_skip_) launch_copy_lastau(es(), kargs(MAP_M, P_RESTART));
			op_adjoint(lctx(), ob_, P_RESTART, Au, G, true);
			launch_getg(es(), kargs(MAP_NM, P_RESTART, ST_RESTART));
		}, h_restart);
	}, h_bt);
	// update_W, reference values, gradient, inner stopping test
	const unsigned long long h_brk = cond_handle();
	launch_shrink_grad(es(), kargs(MAP_N, P_ACTIVE, ST_LOOP).cond(h_brk, P_INNER_BREAK).cond(h_active, P_ACTIVE));
	if (any_cplx_ && !sched_mode_) launch_tau_bb_cplx(es(), kargs(MAP_N, P_ACTIVE));
	// outer step: stopping test, multipliers, continuation
	if_(P_INNER_BREAK, [&] {
		launch_outer(es(), kargs(MAP_N, P_INNER_BREAK));
		launch_mlp(es(), kargs(MAP_NM, P_NEED_MLP));
		launch_grad(es(), kargs(MAP_N, P_NEED_MLP, ST_OUTER).cond(h_active, P_ACTIVE));
		if (!sched_mode_) emit_first_tau(h_active);
	}, h_brk);
	(void)L; (void)s;
}

void Plan::build_graph() {
	TG_CUDA(cudaStreamCreateWithFlags(&cap_, cudaStreamNonBlocking));
	TG_CUDA(cudaGraphCreate(&graph_, 0));
	frames_.clear();
	frames_.push_back(Frame{graph_, {}});
	seg_begin();
	emit_program();
	seg_end();
	frames_.clear();
	TG_CUDA(cudaGraphInstantiate(&exec_, graph_, 0));
}

void Plan::solve(const real *const *d_b, const real *const *d_Ut, real *const *d_U, tval3g_info *info,
                 cudaStream_t stream) {
	auto t0 = std::chrono::steady_clock::now();
	cur_ = stream ? stream : stream_;
	for (int i = 0; i < count_; i++) {
		TG_ARG(d_b && d_b[i] && d_U && d_U[i], "Argument error: b and U must not be NULL");
		h_inst_[i].b_user = d_b[i];
		h_inst_[i].ut_user = d_Ut ? d_Ut[i] : nullptr;
		h_inst_[i].u_user = d_U[i];
	}
	TG_CUDA(cudaMemcpyAsync(d_inst_, h_inst_.data(), sizeof(Inst) * count_, cudaMemcpyHostToDevice, cur_));
	TG_CUDA(cudaMemsetAsync(d_launches_, 0, sizeof(unsigned long long), cur_));
	if (graph_mode_) {
		if (!exec_) build_graph();
		TG_CUDA(cudaGraphLaunch(exec_, cur_));
	} else {
		emit_program();
	}
	std::vector<Ctrl> hc(count_);
	unsigned long long nl = 0;
	TG_CUDA(cudaMemcpyAsync(hc.data(), d_ctrl_, sizeof(Ctrl) * count_, cudaMemcpyDeviceToHost, cur_));
	TG_CUDA(cudaMemcpyAsync(&nl, d_launches_, sizeof(nl), cudaMemcpyDeviceToHost, cur_));
	int op_err = 0;
	TG_CUDA(cudaMemcpyAsync(&op_err, ob_.err, sizeof(int), cudaMemcpyDeviceToHost, cur_));
	TG_CUDA(cudaStreamSynchronize(cur_));
#ifndef TVAL3G_FP64
	for (const auto &e : ob_.mrhs)
		if (mrhs_take_error(cur_, *e.second))
			throw Error{TVAL3G_ERR_CUDA, "tensor-core operator: a bounded wait timed out (results invalid)"};
#endif
	if (op_err) {
		TG_CUDA(cudaMemsetAsync(ob_.err, 0, sizeof(int), cur_));
		throw Error{TVAL3G_ERR_CUDA, "operator: a bounded wait timed out (results invalid)"};
	}
	last_launches_ = (long long)nl;
	last_iters_.resize(count_);
	for (int i = 0; i < count_; i++) last_iters_[i] = hc[i].count_total;
	double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
	if (info)
		for (int i = 0; i < count_; i++) {
			info[i].secs = secs;
			info[i].outer_iters = hc[i].count_outer;
			info[i].total_iters = hc[i].count_total;
			info[i].rel_chg = hc[i].relchg_out;
			info[i].rel_error = hc[i].rel_error;
			info[i].status = hc[i].status;
			info[i].reserved = 0;
		}
}

TG_END
