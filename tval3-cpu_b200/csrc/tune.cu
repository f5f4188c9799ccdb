// Autotuner of the operators' launch shapes (TVAL3G_TUNE).
//
// The measurement operators have shapes whose best value depends on the
// geometry and the GPU rather than on the algorithm: the lanes per ray of the
// on-the-fly Bresenham forward (4, 8 or 16) and the sub-warp width of the
// compressed gathers (4, 8, 16 or 32 lanes per CSR row, CSC column or 3D
// pixel list).  Without tuning they follow built-in rules (8 lanes per ray,
// width by mean line length).  With TVAL3G_TUNE an operator is timed under
// every candidate on its own data once, right after it is built, and keeps
// the fastest; the choice is cached per operator signature (kind, sizes,
// entries, device) in memory and, when TVAL3G_TUNE_CACHE names a file, on
// disk, one line per signature, so later processes skip the timing.  A
// candidate must beat the built-in choice by 2 % to replace it, which keeps
// timing noise from flipping the choice.  The shapes change the order of the
// FP32/FP64 sums only, so a tuned solve is equal to the untuned one within
// rounding, not bitwise.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <functional>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>
#include <string>

#include "ops.cuh"
#include "plan.cuh"

TG_BEGIN
namespace {

struct Choice {
	int fwd_lanes = 0, gcls_fwd = 0, gcls_adj = 0;
};

std::mutex g_mu;
std::map<std::string, Choice> g_cache;
bool g_loaded = false;
long long g_measured = 0, g_cached = 0;

std::string cache_file() {
	const char *e = std::getenv("TVAL3G_TUNE_CACHE");
	return e ? std::string(e) : std::string();
}

// lines "<signature>\t<fwd_lanes> <gcls_fwd> <gcls_adj>"
void load_cache() {
	if (g_loaded) return;
	g_loaded = true;
	const std::string path = cache_file();
	if (path.empty()) return;
	std::ifstream f(path);
	std::string line;
	while (std::getline(f, line)) {
		const size_t tab = line.find('\t');
		if (tab == std::string::npos) continue;
		std::istringstream v(line.substr(tab + 1));
		Choice c;
		if (v >> c.fwd_lanes >> c.gcls_fwd >> c.gcls_adj) g_cache[line.substr(0, tab)] = c;
	}
}

void store_cache(const std::string &key, const Choice &c) {
	const std::string path = cache_file();
	if (path.empty()) return;
	std::ofstream f(path, std::ios::app);
	if (f) f << key << '\t' << c.fwd_lanes << ' ' << c.gcls_fwd << ' ' << c.gcls_adj << '\n';
}

// the device part of a signature, looked up once per device
std::string device_tag() {
	static std::mutex mu;
	static std::map<int, std::string> tags;
	int dev = 0;
	TG_CUDA(cudaGetDevice(&dev));
	std::lock_guard<std::mutex> lock(mu);
	auto it = tags.find(dev);
	if (it != tags.end()) return it->second;
	cudaDeviceProp prop;
	TG_CUDA(cudaGetDeviceProperties(&prop, dev));
	std::ostringstream k;
	k << "sm=" << prop.multiProcessorCount << " dev=" << prop.name;
	return tags[dev] = k.str();
}

std::string signature(const OpStore &st, long long rows, long long cols) {
	const OpDev &d = st.dev;
	std::ostringstream k;
	k << "v1 kind=" << d.kind << " rows=" << rows << " cols=" << cols << " layers=" << d.layers
	  << " nnz=" << st.nnz << " rays=" << d.nrays << " tiled=" << d.tiled << " " << device_tag();
	std::string s = k.str();
	for (char &ch : s)
		if (ch == '\t' || ch == '\n') ch = ' ';
	return s;
}

// Median-free timing: the best of a few back-to-back applications (after a
// warm-up), in ms per application, of the forward (trans 0) or the adjoint
// (trans 1) under choice c.
float time_choice(cudaStream_t s, const OpStore &st, const Inst &base, int trans, const Choice &c, float *dx,
                  float *dy, Inst *dinst, int *derr) {
	Inst I = base;
	I.op.fwd_lanes = c.fwd_lanes;
	I.op.gcls_fwd = c.gcls_fwd;
	I.op.gcls_adj = c.gcls_adj;
	std::vector<Inst> v(1, I);
	std::vector<OpStore> ops(1);
	ops[0].nnz = st.nnz;
	ops[0].dev = I.op;
	OpBatch ob;
	int2 *tiles = nullptr;
	build_op_maps_upload(v, ops, ob, &tiles, s);
	I = v[0];
	ob.err = derr;
	VecSel xs, ys;
	if (!trans) {
		I.vn[0] = dx; I.vm[0] = dy;
		xs = VecSel{false, 0}; ys = VecSel{true, 0};
	} else {
		I.vm[0] = dy; I.vn[0] = dx;
		xs = VecSel{true, 0}; ys = VecSel{false, 0};
	}
	TG_CUDA(cudaMemcpyAsync(dinst, &I, sizeof(Inst), cudaMemcpyHostToDevice, s));
	LaunchCtx L{s, dinst, nullptr};
	auto apply = [&] {
		if (!trans) op_forward(L, ob, P_ALL, xs, ys);
		else op_adjoint(L, ob, P_ALL, xs, ys);
	};
	cudaEvent_t e0, e1;
	TG_CUDA(cudaEventCreate(&e0));
	TG_CUDA(cudaEventCreate(&e1));
	float best = 1e30f;
	try {
		apply();
		apply();
		for (int r = 0; r < 5; r++) {
			TG_CUDA(cudaEventRecord(e0, s));
			apply();
			TG_CUDA(cudaEventRecord(e1, s));
			TG_CUDA(cudaEventSynchronize(e1));
			float ms = 0.f;
			TG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
			best = std::min(best, ms);
		}
	} catch (...) {
		cudaEventDestroy(e0);
		cudaEventDestroy(e1);
		dev_free(tiles, s);
		throw;
	}
	cudaEventDestroy(e0);
	cudaEventDestroy(e1);
	dev_free(tiles, s);
	return best;
}

// the fastest of the candidates for one field, the built-in choice (0)
// first; another candidate must be 2 % faster to win
template <class Set>
int pick(const Choice &start, int Choice::*field, const Set &cands, const std::function<float(const Choice &)> &t) {
	Choice c = start;
	c.*field = 0;
	float best = t(c);
	int arg = 0;
	for (int v : cands) {
		c.*field = v;
		const float ms = t(c);
		if (ms < 0.98f * best) {
			best = ms;
			arg = v;
		}
	}
	return arg;
}

}  // namespace

void autotune_operator(cudaStream_t s, OpStore &st, const Inst &shape) {
	OpDev &d = st.dev;
	const bool rays = d.kind == TVAL3G_OP_RAY2D || d.kind == TVAL3G_OP_RAY3D;
	const bool tune_fwd = rays || d.kind == TVAL3G_OP_CSR;
	const bool tune_adj = d.kind == TVAL3G_OP_CSR || (rays && !d.tiled);
	if (!tune_fwd && !tune_adj) return;   // dense: no launch shape to choose
	const std::string key = signature(st, shape.m, shape.n);
	{
		std::lock_guard<std::mutex> lock(g_mu);
		load_cache();
		auto it = g_cache.find(key);
		if (it != g_cache.end()) {
			d.fwd_lanes = it->second.fwd_lanes;
			d.gcls_fwd = it->second.gcls_fwd;
			d.gcls_adj = it->second.gcls_adj;
			g_cached++;
			return;
		}
	}
	Inst base = shape;
	base.op = d;
	float *dx = (float *)dev_alloc(sizeof(float) * (size_t)std::max(shape.n, 1LL), s);
	float *dy = (float *)dev_alloc(sizeof(float) * (size_t)std::max(shape.m, 1LL), s);
	Ctrl *dctrl = (Ctrl *)dev_alloc(sizeof(Ctrl), s);
	Inst *dinst = (Inst *)dev_alloc(sizeof(Inst), s);
	int *derr = (int *)dev_alloc(sizeof(int), s);
	Choice best;
	try {
		TG_CUDA(cudaMemsetAsync(dx, 0, sizeof(float) * (size_t)std::max(shape.n, 1LL), s));
		TG_CUDA(cudaMemsetAsync(dy, 0, sizeof(float) * (size_t)std::max(shape.m, 1LL), s));
		TG_CUDA(cudaMemsetAsync(dctrl, 0, sizeof(Ctrl), s));
		TG_CUDA(cudaMemsetAsync(derr, 0, sizeof(int), s));
		base.ctrl = dctrl;
		auto t_fwd = [&](const Choice &c) { return time_choice(s, st, base, 0, c, dx, dy, dinst, derr); };
		auto t_adj = [&](const Choice &c) { return time_choice(s, st, base, 1, c, dx, dy, dinst, derr); };
		static const int lanes[] = {4, 16};   // besides the built-in 8
		static const int widths[] = {1, 2, 3, 4};
		if (rays) best.fwd_lanes = pick(best, &Choice::fwd_lanes, lanes, t_fwd);
		else if (tune_fwd) best.gcls_fwd = pick(best, &Choice::gcls_fwd, widths, t_fwd);
		if (tune_adj) best.gcls_adj = pick(best, &Choice::gcls_adj, widths, t_adj);
		int e = 0;
		TG_CUDA(cudaMemcpyAsync(&e, derr, sizeof(int), cudaMemcpyDeviceToHost, s));
		TG_CUDA(cudaStreamSynchronize(s));
		TG_ARG(e == 0, "Internal error: a bounded wait timed out while the operator was tuned");
	} catch (...) {
		for (void *q : {(void *)dx, (void *)dy, (void *)dctrl, (void *)dinst, (void *)derr}) dev_free(q, s);
		throw;
	}
	for (void *q : {(void *)dx, (void *)dy, (void *)dctrl, (void *)dinst, (void *)derr}) dev_free(q, s);
	d.fwd_lanes = best.fwd_lanes;
	d.gcls_fwd = best.gcls_fwd;
	d.gcls_adj = best.gcls_adj;
	std::lock_guard<std::mutex> lock(g_mu);
	g_measured++;
	g_cache[key] = best;
	store_cache(key, best);
}

void autotune_stats(long long *measured, long long *cached) {
	std::lock_guard<std::mutex> lock(g_mu);
	if (measured) *measured = g_measured;
	if (cached) *cached = g_cached;
}

TG_END
