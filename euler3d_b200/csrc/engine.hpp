// Device-resident solver over one case (all blocks on one GPU).
#pragma once
#include <cuda_runtime.h>

#include <array>
#include <memory>
#include <string>
#include <vector>

#include "launch.hpp"
#include "mesh.hpp"

namespace e3d {

enum Precision : int { PREC_FP64 = 0, PREC_FP32 = 1 };

struct EngineOptions {
	int precision = PREC_FP64;
	int carry_w0 = -1;   // -1: default (off for FP64, on for FP32): keep W in FP64 across iterations
	int use_graph = 1;   // capture one outer iteration in a CUDA graph
	int device = -1;     // -1: current device
	cudaStream_t stream = nullptr;  // nullptr: the engine creates its own stream
	size_t hist_capacity = 4096;    // iterations of per-block norm/force history kept on device
	int renumber = 16;   // RENUMBER_*: device order of each block's real cells (file order, boundary cells last)
};

// Device order of the real cells inside each block (renumber.cpp).  Slots keep
// each cell's ascending face order, so every per-cell sum runs in the
// reference's order whatever the cell order.
enum Renumber : int {
	RENUMBER_NONE = 0,
	RENUMBER_RCM = 1,
	RENUMBER_MORTON = 2,
	RENUMBER_SHUFFLE = 3,
	RENUMBER_BOUNDARY_LAST = 16  // added to a base order: cells with a ghost neighbour last
};
// order[i] = block-local real cell placed i-th on the device
std::vector<int> cell_order(const HostBlock& b, int mode);

// Block sharding (shard.cpp): rank r of n holds the case blocks
// [first_block[r], first_block[r+1]).  Halo entries that cross ranks are
// listed in transport order: by peer rank, then topology order, then cell pair.
struct ShardPlan {
	int rank = 0, n_ranks = 1, b0 = 0, b1 = 0;
	std::vector<int> first_block;                   // n_ranks + 1
	std::vector<long long> send_count, recv_count;  // halo entries per peer rank
	std::vector<int> send_block, send_cell;         // origin (case block, block-local cell) of each sent entry
	std::vector<int> recv_block, recv_cell;         // destination (case block, block-local ghost) of each received one
	std::vector<Connexion> local;                   // connexions with both blocks on this rank (case block ids)
};
// the reference's distribution: n_blocks / n_ranks blocks each, one more for
// the first n_blocks % n_ranks ranks (BlockCommunicator.cpp:29-38)
std::vector<int> shard_first_blocks(int n_blocks, int n_ranks);
ShardPlan shard_plan(const HostCase& hc, const std::vector<int>& first_block, int rank);

// Host copy of one outer iteration's results (reference PostProcessing fields).
struct IterRecord {
	int iter;
	double rms[5];          // mesh residual norms (sum of per-block norms)
	double conv[5];         // log10(rms) - log10(rms at iteration 0)
	double cl, cd, cmx, cmy, cmz;
};

inline void cuda_ok(cudaError_t e, const char* what) {
	if (e != cudaSuccess) throw Error(E3D_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

template <class T>
struct DevBuf {
	T* p = nullptr;
	size_t n = 0;
	void alloc(size_t count);
	void upload(const std::vector<T>& h);
	void free();
	~DevBuf() { free(); }
};

class Engine {
public:
	Engine(const HostCase& hc, const EngineOptions& opt);
	// several cases advanced together in one device arena (a batch); they must
	// share gamma, CFL, RK stages and the strategy choices, and may differ in
	// mesh, Mach number, angle of attack and reference chord
	Engine(const std::vector<const HostCase*>& cases, const EngineOptions& opt);
	// one rank's blocks of a block-sharded case (plan from shard_plan); block
	// indices of the engine's methods are local to the rank's range
	Engine(const HostCase& hc, const EngineOptions& opt, const ShardPlan& plan);
	~Engine();
	Engine(const Engine&) = delete;
	Engine& operator=(const Engine&) = delete;

	// --- strategy-level operations (FP64 engine); block = -1 means every block
	void save_w0(int block);
	void spectral_radius(int block);
	void timestep(int block);
	void gradients(int block, int kind);
	void limiters(int block, int kind, double omega, double k);
	void flux_conv(int block, int scheme);
	void flux_diss(int block, int scheme, double beta);
	void update_internal(int block, double alpha);
	void update_boundary(int block);
	void smooth_residual(int block);  // CentralIrsSmoother::smoothResidual
	void halo();
	// per-block norms and forces of the current state (PostProcessing::computeFlowData)
	void flow_data(std::vector<double>& per_block10);

	// --- whole outer iterations (fused kernels); appends to history()
	void iterate(int n_iter);
	// iterate with CUDA events recorded on the engine stream around the launches;
	// returns the device time of the n iterations in milliseconds
	double iterate_timed(int n_iter);
	// checkpoint: the complete solver state (current primitives in device
	// precision, FP64 W0, iteration count, iteration-0 norms) to / from a host buffer
	size_t state_bytes() const;
	void export_state(void* host, size_t bytes);
	void import_state(const void* host, size_t bytes);
	// run until the reference stop test (max_iter or criterion) fires
	int solve(int max_iter, double criterion, int check_every);

	// --- block sharding: the halo entries that cross ranks.  After every
	// iteration (and before the first) each rank packs what its peers need,
	// the caller moves the buffers (an all-to-all with per-peer counts), and
	// each rank unpacks what it received; a shard refuses to iterate until it
	// has.  Buffers are device memory of 5 values per entry in the engine's
	// precision, entry-major, in ShardPlan order; work is queued on stream().
	bool is_shard() const { return shard_; }
	const ShardPlan& shard() const { return plan_; }
	void shard_pack(void* send);
	void shard_unpack(const void* recv);
	// raw per-block norms and forces ([n][local blocks][10]) of the iterations
	// run since the last call; the caller gathers every rank's, in block
	// order, and pushes them back with shard_push (the history then holds
	// whole-case records, summed in block order as one GPU sums them)
	int shard_pending();  // brings the device records over; iterations waiting to be taken
	std::vector<double> shard_take_flow_data(int& n_iters);
	void shard_push(const double* all_blocks, int n_iters);

	// --- batches: every active case advanced by the persistent cooperative
	// kernel (FP32); a case stops (its tiles leave the work list) once its
	// density drop reaches `criterion` or it has run max_iter iterations.
	// iters_done[c] = iterations case c ran.  Returns the device time in ms.
	double solve_batch(int max_iter, double criterion, int iters_per_launch, int stall_window,
	                   std::vector<int>& iters_done);
	struct Tuning {
		int tile_cells = 0, grid = 0;
		double ms_per_iter = 0.0;
		bool from_cache = false, graph = false, tiled = false;
	};
	const Tuning& tuning() const { return tuning_; }

	const std::vector<IterRecord>& history() const { return hist_case_[0]; }
	const std::vector<IterRecord>& history(int c) const { return hist_case_.at(c); }
	int n_cases() const { return ncases_; }

	// --- warm start and precision switch (batched / learned forms)
	// raw surrogate inputs of every real cell, [NR][8] floats on the device:
	// centroid x y z, distance to the nearest wall-face centre of the cell's case, Mach, alpha (deg), 0, 0
	void cell_features(float* dev_out);
	// conservative state of every real cell, [NR][8] floats on the device (5 used)
	void conservative_rows(float* dev_out);
	// writes a conservative state ([NR][ld] floats on the device) into every real cell; cells whose
	// prediction is not physical keep the freestream state of their case; returns how many did
	int apply_conservative(const float* dev_w, int ld);
	// FP32 solver -> FP64 solver in place: FP64 geometry and state (real cells from the carried FP64
	// conservative state), histories and reference norms kept, FP32 buffers released
	void widen_to_fp64();
	// FP64 batch solves with the kernels built with fused multiply-add (same discrete equations, last-bit
	// differences from the bit-identical FP64 path); affects e3d_batch_solve only
	void set_fp64_contracted(bool on);
	bool fp64_contracted() const { return fast64_; }
	// FP32 solver -> FP32 iterations in difference form (delta.cu) for batch
	// solves: first-order AUSM on all-tetrahedron meshes.  The state is an FP64
	// base (rebased before every batch launch, with its residual evaluated in
	// FP64) plus FP32 differences, so the residual falls below the FP32 floor.
	// widen_to_fp64 leaves the form; get("prim") returns the full state.
	void enter_delta();
	bool delta() const { return delta_; }
	long long n_real_case(int c) const;
	void sync();  // waits for queued work; throws on a CUDA error or a non-finite norm

	// --- state transfer (block-local cell order, FP64 on the host side)
	void get(const std::string& name, int block, std::vector<double>& out);
	void set(const std::string& name, int block, const std::vector<double>& in);

	int n_blocks() const { return nb_; }
	int n_real(int b) const { return roff_[b + 1] - roff_[b]; }
	long long n_real_total() const { return NR_; }
	int precision() const { return opt_.precision; }
	cudaStream_t stream() const { return st_; }
	size_t device_bytes() const { return dev_bytes_; }
	// number of kernel launches one outer iteration issues
	int launches_per_iteration() const;
	const Deck& deck() const { return deck_; }
	// algorithmic bytes (distinct elements touched) of one launch of each fused kernel
	double bytes_recon(bool first) const;
	double bytes_start() const;
	double bytes_flux(bool order1, bool diss, bool last) const;
	// times each fused kernel of `n` eager (un-captured) iterations with CUDA events on
	// the engine stream; returns {name, launches, total_ms}
	struct KernelTime {
		std::string name;
		int launches;
		double total_ms;
		double bytes_per_launch;
	};
	std::vector<KernelTime> time_kernels(int n);

private:
	template <class T>
	struct Fused {
		DevBuf<T> P0, P1, FS, Rc, Rd, dt, sgeo, sS, srv, lsw, vol;
		FusedView<T> view(bool flip) const;
	};
	Engine(const std::vector<const HostCase*>& cases, const EngineOptions& opt, const ShardPlan* plan);
	void setup(const std::vector<const HostCase*>& cases, const ShardPlan* plan);
	int device_cell(int b, int local) const;
	IterRecord make_record(int cs, const double* x, int nblocks, const int* n_real);
	void require_exchanged(int n_iter) const;
	void build_blocks(const std::vector<const HostBlock*>& blocks, const std::vector<Connexion>& conns);
	void to_local(int b, std::vector<double>& a, int rows, int ld) const;
	void to_device(int b, std::vector<double>& a, int rows, int ld) const;
	void init_state();
	void count_device_bytes();
	void check(const char* what);
	template <class T>
	void iteration_body(Fused<T>& f, int parity, std::vector<cudaEvent_t>* marks);
	template <class T>
	void run_iterations(Fused<T>& f, int n);
	void collect_history(int first_iter, int n);
	void smoothed_iteration_body();
	void block_range(int block, int& r0, int& r1, int& g0, int& g1) const;
	void require_fp64(const char* what) const;
	StateView state64();
	const double* cur_prim64() const;

	Deck deck_;
	EngineOptions opt_;
	cudaStream_t st_ = nullptr;
	bool own_stream_ = false;
	int nb_ = 0, NR_ = 0, NG_ = 0, NA_ = 0, NF_ = 0, NS_ = 0, tet4_ = 0;
	std::vector<int> roff_, goff_, foff_, soff_;  // per block offsets (nb_+1)
	std::vector<int> n_real_b_, n_all_b_;
	std::vector<std::vector<int>> pos_;  // per block: device position (0..n_real-1) of each local real cell
	Physics ph_{};
	double denom_ = 1.0, aoa_rad_ = 0.0;
	int ncases_ = 1;
	std::vector<int> case_boff_;      // ncases+1 block offsets of each case
	std::vector<int> block_case_;     // case of each block
	std::vector<double> case_free_h_, case_denom_, case_aoa_;
	DevBuf<double> case_free_d_, wall_denom_d_;
	std::vector<float> case_ma_h_;        // Mach, alpha (deg) of each case
	DevBuf<float> cen_d_, case_ma_d_;     // real-cell centroids [NR][3]; per-case Mach/alpha
	DevBuf<int> block_case_d_, case_wall_off_d_, fallback_d_;
	DevBuf<int> gcase_d_;
	int carry_ = 0;
	int grad_kind_ = GRAD_LEAST_SQUARES, lim_kind_ = LIM_VENKATAKRISHNAN, scheme_ = FLUX_ROE, order_ = 1;
	std::vector<double> alpha_, beta_;
	// geometry / topology
	DevBuf<int> slot_ptr_, slot_face_, slot_nbr_, slot_mate_, face_lr_, halo_dst_, halo_src_, wall_off_, wall_face_,
	    roff_d_;
	DevBuf<signed char> gkind_, grefl_;
	DevBuf<double> S_, nhat_, area_, rl_, rr_, fc_, vol64_, lsw64_;
	// FP64 strategy-level state
	DevBuf<double> W0_, srad_, grad_, lim_;
	Fused<double> f64_;
	Fused<float> f32_;
	int cur_ = 0;  // which of P0/P1 holds the current state
	// reductions
	DevBuf<double> partial_, hist_d_, fd_hist_, wall_terms_;
	DevBuf<int> iter_d_, bad_d_, zero_d_;
	bool started_ = false;
	int chunk_ = 0, max_chunks_ = 0;
	int dev_iter_ = 0;  // iterations recorded on the device since the last collect
	int total_iter_ = 0;
	std::vector<char> have_rms0_;
	std::vector<std::array<double, 5>> rms0_;
	std::vector<std::vector<IterRecord>> hist_case_;
	// block sharding
	bool shard_ = false, need_exchange_ = false;
	ShardPlan plan_;
	std::vector<int> all_n_real_;   // real cells of every block of the case
	DevBuf<int> xsend_, xrecv_;     // device cells of the sent / received halo entries
	std::vector<double> raw_pending_;
	int raw_iters_ = 0;
	cudaGraphExec_t graph_[2] = {nullptr, nullptr};
	// batch (persistent kernel) state
	std::vector<char> case_active_, case_failed_;  // failed: residual turned non-finite in a batch solve
	bool tolerate_nonfinite_ = false;
	DevBuf<int> work_d_, block_work_d_;
	DevBuf<double> wpart_d_;
	int n_work_ = 0, tile_mult_ = 1, grid_ = 0;
	Tuning tuning_;
	cudaGraphExec_t pgraph_ = nullptr;
	int pgraph_iters_ = 0, pgraph_parity_ = -1, pgraph_grid_ = 0;
	bool tiled_ = false, pgraph_tiled_ = false, fast64_ = false;
	void build_work();
	double run_persistent(int iters);
	template <class T>
	double run_persistent_t(int iters);
	template <class T>
	Fused<T>& fused();
	void autotune(int iters);
	void snapshot(bool save);
	DevBuf<unsigned char> snap_;
	DevBuf<double> irs_;  // residual-smoothing Jacobi start values, 10 x NR
	// difference form: base primitives (FP32 copy and FP64), carried conserved
	// differences, base residual; W0_ holds the FP64 base conserved state
	bool delta_ = false;
	DevBuf<float> Pb32_, dW_, Rb_;
	DevBuf<double> Pb64_;
	FusedView<float> delta_view(bool flip) const;
	void rebase();
	void leave_delta();
	void require_not_delta(const char* what) const;
	size_t dev_bytes_ = 0;
};

template <>
inline Engine::Fused<float>& Engine::fused<float>() {
	return f32_;
}
template <>
inline Engine::Fused<double>& Engine::fused<double>() {
	return f64_;
}

}  // namespace e3d
