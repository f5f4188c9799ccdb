// Plans: device-resident operators, state and the emitted solve program.
#pragma once
#include <functional>
#include <memory>

#include "kernels.cuh"
#include "mrhs.cuh"
#include "ops.cuh"

TG_BEGIN

// device operator storage owned by a plan / operator object
struct OpStore {
	OpDev dev{};
	std::vector<void *> owned;   // device allocations to free
	std::shared_ptr<MrhsOp> mrhs;   // multi-RHS dense operator on the tensor cores, or null
	long long bytes = 0;         // device bytes allocated for the operator
	long long adj_index_bytes = 0;   // index read by one adjoint application (besides x and y)
	long long nnz = 0;           // CSR nnz, or Bresenham hits of a ray operator
	long long b_len = 0;
	// ray operators: forward CSR over traced rays (kept on request) and the
	// host copy of each traced ray's measurement index
	int *ray_rptr = nullptr, *ray_rind = nullptr;
	std::vector<int> ray_out;
};

// validate a problem against (b_len, ut_len) with the reference's messages;
// returns n (image length).  rays = false leaves out the per-ray endpoint
// check, for callers that validated the same problem already (the operator
// builder checks every endpoint again while it packs the rays)
long long validate(const tval3g_problem &p, long long b_len, long long ut_len, bool rays = true);
// prepare the device operator of a problem (flags: TVAL3G_DEVICE_INPUTS)
void prepare_op(cudaStream_t s, const tval3g_problem &p, int flags, OpStore &st, bool keep_ray_csr);
void free_op(OpStore &st, cudaStream_t s);
void check_options(const tval3g_options &o);
// TVAL3G_TUNE: time the operator's launch-shape candidates on its own data
// (or take the cached choice of its signature) and store the fastest in
// st.dev; shape gives the instance's image and vector sizes (tune.cu)
void autotune_operator(cudaStream_t s, OpStore &st, const Inst &shape);
void autotune_stats(long long *measured, long long *cached);
// operator tile maps of a batch, uploaded to *d_tiles; returns the dense
// partial-buffer size in floats
long long build_op_maps_upload(std::vector<Inst> &inst, const std::vector<OpStore> &ops, OpBatch &ob,
                               int2 **d_tiles, cudaStream_t s);

// internal plan flag: per-iteration (mu_k, beta_k) from set_schedule instead of
// the continuation (every instance must have the same maxit)
constexpr int PLAN_SCHEDULE = 1 << 16;

class Plan {
public:
	Plan(int count, const tval3g_problem *probs, const tval3g_options *opts, int flags);
	~Plan();
	void solve(const real *const *d_b, const real *const *d_Ut, real *const *d_U, tval3g_info *info,
	           cudaStream_t stream);
	long long launches() const { return last_launches_; }
	int trace(int index, tval3g_trace_record *out, int cap) const;
	void set_target(double target) {
		for (auto &I : h_inst_) I.target = target;
	}
	long long device_bytes() const { return device_bytes_; }
	// schedule mode: mu[0..maxit), beta[0..maxit) (host) for the next solves
	void set_schedule(const double *mu, const double *beta);
	int maxit() const { return h_inst_.empty() ? 0 : h_inst_[0].maxit; }
	// the instances' scalar state after the last solve
	std::vector<Ctrl> ctrl() const;
	// mean device time (ms) of one launch of k_getg (descent stage), k_descend
	// (descent stage) and k_shrink_grad over every instance, each launched reps
	// times back to back after the last solve (whose state they overwrite)
	void time_stencils(int reps, double ms[3]);

private:
	struct Frame {
		cudaGraph_t g;
		std::vector<cudaGraphNode_t> deps;
	};
	int count_;
	int flags_;
	bool graph_mode_;
	bool any_skip_ = false;
	bool any_cplx_ = false;   // complex instances: their Barzilai-Borwein step in k_tau_bb_cplx
	bool sched_mode_ = false;
	double *d_sched_ = nullptr;
	cudaStream_t stream_ = nullptr;   // the plan's own stream
	cudaStream_t cur_ = nullptr;      // stream of the solve in progress
	std::vector<OpStore> ops_;
	std::vector<Inst> h_inst_;
	Inst *d_inst_ = nullptr;
	Ctrl *d_ctrl_ = nullptr;
	double *d_part_ = nullptr;
	real *d_arena_ = nullptr;
	int2 *d_tiles_ = nullptr;
	int *d_flag_ = nullptr;
	int h_flag_ = 0;                  // host copy of d_flag_ (host-driven plans)
	unsigned long long *d_launches_ = nullptr;
	TileMap maps_[NMAPS];
	OpBatch ob_;
	long long last_launches_ = 0;
	double *d_trace_ = nullptr;
	std::vector<long long> trace_off_;
	std::vector<int> last_iters_;
	long long device_bytes_ = 0;
	std::vector<void *> allocs_;
	// graph
	cudaGraph_t graph_ = nullptr;
	cudaGraphExec_t exec_ = nullptr;
	cudaStream_t cap_ = nullptr;      // stream used for capture
	std::vector<Frame> frames_;
	bool capturing_ = false;

	void *dalloc(size_t bytes);
	void release();
	void group_shared_dense(const tval3g_problem *probs, int flags);
	KArgs kargs(MapKind mk, int pred, int stage = 0) const;
	LaunchCtx lctx() const;
	void emit_program();
	void emit_iteration(unsigned long long h_active);
	void emit_first_tau(unsigned long long h_active);
	// control flow: direct execution or graph construction
	// Conditional regions.  With a handle from cond_handle() the kernel launched
	// just before (and, for while_, the body's last kernel) sets the condition;
	// with h = 0 a condition kernel evaluates it (batches, host-driven plans).
	unsigned long long cond_handle();
	void if_(int pred, const std::function<void()> &body, unsigned long long h = 0);
	void while_(int pred, const std::function<void()> &body, unsigned long long h = 0);
	void seg_begin();
	void seg_end();
	cudaStream_t es() const { return graph_mode_ ? cap_ : cur_; }
	void build_graph();
};

TG_END
