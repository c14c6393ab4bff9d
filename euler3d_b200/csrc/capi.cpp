// extern "C" boundary: status codes, thread-local error text, no exceptions
// crossing the ABI.
#include "../../include/e3d.h"

#include <cstring>
#include <string>

#include "engine.hpp"
#include "surrogate.hpp"
#include "mesh.hpp"

struct e3d_case {
	e3d::HostCase hc;
};
struct e3d_solver {
	std::unique_ptr<e3d::Engine> eng;
};
struct e3d_surrogate {
	std::unique_ptr<e3d::Surrogate> net;
};

namespace {
thread_local std::string g_err;

int fail(int code, const std::string& msg) {
	g_err = msg;
	return code;
}

template <class F>
int guard(F&& f) {
	try {
		f();
		g_err.clear();
		return E3D_OK;
	} catch (const e3d::Error& e) {
		return fail(e.code, e.what());
	} catch (const std::bad_alloc&) {
		return fail(E3D_ERR_LIMIT, "host allocation failed");
	} catch (const std::exception& e) {
		return fail(E3D_ERR_STATE, e.what());
	}
}

const e3d::HostBlock& block_of(const e3d_case* c, int b) {
	if (!c) throw e3d::Error(E3D_ERR_ARG, "null case");
	if (b < 0 || b >= (int)c->hc.blocks.size()) throw e3d::Error(E3D_ERR_ARG, "block index out of range");
	return c->hc.blocks[b];
}

e3d::Engine& eng(e3d_solver* s) {
	if (!s || !s->eng) throw e3d::Error(E3D_ERR_ARG, "null solver");
	return *s->eng;
}
}  // namespace

namespace e3d {
void set_last_error(const std::string& msg) { g_err = msg; }
}  // namespace e3d

extern "C" {

const char* e3d_last_error(void) { return g_err.c_str(); }
const char* e3d_version(void) { return "euler3d_b200 0.1 (sm_100a)"; }

void e3d_default_options(e3d_options* o) {
	if (!o) return;
	o->precision = E3D_FP64;
	o->carry_w0 = -1;
	o->use_graph = 1;
	o->device = -1;
	o->stream = nullptr;
	o->hist_capacity = 4096;
	o->renumber = E3D_RENUMBER_NONE | E3D_RENUMBER_BOUNDARY_LAST;
}

int e3d_case_load(const char* deck_path, const char* workdir, e3d_case** out) {
	if (!deck_path || !out) return fail(E3D_ERR_ARG, "null argument");
	*out = nullptr;
	return guard([&] {
		auto* c = new e3d_case;
		try {
			c->hc = e3d::load_case(deck_path, workdir ? workdir : "");
		} catch (...) {
			delete c;
			throw;
		}
		*out = c;
	});
}

int e3d_case_free(e3d_case* c) {
	delete c;
	return E3D_OK;
}

int e3d_case_deck(const e3d_case* c, e3d_deck_info* o) {
	if (!c || !o) return fail(E3D_ERR_ARG, "null argument");
	const e3d::Deck& d = c->hc.deck;
	o->cfl = d.cfl;
	o->gamma = d.gamma;
	o->aoa_deg = d.aoa_deg;
	o->mach = d.mach;
	o->cmac = d.cmac;
	o->criterion = d.criterion;
	o->omega = d.omega;
	o->k = d.k;
	o->stages = d.stages;
	o->max_iter = d.max_iter;
	o->smoothing = d.smoothing ? 1 : 0;
	o->order = d.order;
	o->flux = d.flux == "roe" ? E3D_FLUX_ROE : d.flux == "ausm" ? E3D_FLUX_AUSM : -1;
	o->gradient = d.gradient == "leastsquares" ? E3D_GRAD_LEAST_SQUARES : E3D_GRAD_GREEN_GAUSS;
	o->limiter = d.limiter == "venkatakrishnan" ? E3D_LIM_VENKATAKRISHNAN : E3D_LIM_BARTH_JESPERSEN;
	return E3D_OK;
}

int e3d_case_n_blocks(const e3d_case* c, int* n) {
	if (!c || !n) return fail(E3D_ERR_ARG, "null argument");
	*n = (int)c->hc.blocks.size();
	return E3D_OK;
}

int e3d_case_block_info(const e3d_case* c, int block, e3d_block_info* o) {
	if (!o) return fail(E3D_ERR_ARG, "null argument");
	return guard([&] {
		const e3d::HostBlock& B = block_of(c, block);
		o->n_real = B.n_real;
		o->n_all = B.n_all;
		o->n_faces = B.n_faces;
		o->n_nodes = B.n_nodes;
		o->n_markers = (int)B.markers.size();
		o->n_real_boundaries = B.n_real_boundaries;
		o->n_wall_faces = (int)B.wall_faces.size();
	});
}

int e3d_case_get_f64(const e3d_case* c, int block, const char* name, double* dst, int64_t* count) {
	if (!name || !count) return fail(E3D_ERR_ARG, "null argument");
	return guard([&] {
		const e3d::HostBlock& B = block_of(c, block);
		const std::vector<double>* v = nullptr;
		const std::string n(name);
		if (n == "face_normal") v = &B.face_normal;
		else if (n == "face_area") v = &B.face_area;
		else if (n == "face_center") v = &B.face_center;
		else if (n == "r_left") v = &B.r_left;
		else if (n == "r_right") v = &B.r_right;
		else if (n == "cell_volume") v = &B.cell_volume;
		else if (n == "cell_center") v = &B.cell_center;
		else if (n == "ls_weights") v = &B.ls_weights;
		else if (n == "node_xyz") v = &B.node_xyz;
		else throw e3d::Error(E3D_ERR_ARG, "unknown float array '" + n + "'");
		if (!dst) {
			*count = (int64_t)v->size();
			return;
		}
		if (*count != (int64_t)v->size()) throw e3d::Error(E3D_ERR_ARG, n + ": wrong count");
		std::memcpy(dst, v->data(), v->size() * sizeof(double));
	});
}

int e3d_case_cell_order(const e3d_case* c, int block, int mode, int32_t* order, int64_t n_real) {
	if (!order) return fail(E3D_ERR_ARG, "null argument");
	return guard([&] {
		const e3d::HostBlock& B = block_of(c, block);
		if (n_real != B.n_real) throw e3d::Error(E3D_ERR_ARG, "order: wrong count");
		const std::vector<int> o = e3d::cell_order(B, mode);
		std::copy(o.begin(), o.end(), order);
	});
}

int e3d_case_get_i32(const e3d_case* c, int block, const char* name, int32_t* dst, int64_t* count) {
	if (!name || !count) return fail(E3D_ERR_ARG, "null argument");
	return guard([&] {
		const e3d::HostBlock& B = block_of(c, block);
		std::vector<int> tmp;
		const std::vector<int>* v = &tmp;
		const std::string n(name);
		if (n == "face_cells") v = &B.face_cells;
		else if (n == "cell_face_ptr") v = &B.cell_face_ptr;
		else if (n == "cell_faces") v = &B.cell_faces;
		else if (n == "cell_cells") v = &B.cell_cells;
		else if (n == "wall_faces") v = &B.wall_faces;
		else if (n == "face_nodes") v = &B.face_nodes;
		else if (n == "marker_kind") {
			for (const auto& m : B.markers) tmp.push_back(m.kind);
		} else if (n == "marker_size") {
			for (const auto& m : B.markers) tmp.push_back((int)m.ghosts.size());
		} else if (n == "marker_cells") {
			for (const auto& m : B.markers) tmp.insert(tmp.end(), m.ghosts.begin(), m.ghosts.end());
		} else
			throw e3d::Error(E3D_ERR_ARG, "unknown int array '" + n + "'");
		if (!dst) {
			*count = (int64_t)v->size();
			return;
		}
		if (*count != (int64_t)v->size()) throw e3d::Error(E3D_ERR_ARG, n + ": wrong count");
		std::memcpy(dst, v->data(), v->size() * sizeof(int));
	});
}

static e3d::EngineOptions engine_options(const e3d_options* opt) {
	e3d_options o;
	e3d_default_options(&o);
	if (opt) o = *opt;
	e3d::EngineOptions eo;
	eo.precision = o.precision;
	eo.carry_w0 = o.carry_w0;
	eo.use_graph = o.use_graph;
	eo.device = o.device;
	eo.stream = static_cast<cudaStream_t>(o.stream);
	eo.hist_capacity = o.hist_capacity > 0 ? (size_t)o.hist_capacity : 4096;
	eo.renumber = o.renumber;
	return eo;
}

int e3d_solver_create(const e3d_case* c, const e3d_options* opt, e3d_solver** out) {
	if (!c || !out) return fail(E3D_ERR_ARG, "null argument");
	*out = nullptr;
	return guard([&] {
		const e3d::EngineOptions eo = engine_options(opt);
		auto s = std::make_unique<e3d_solver>();
		s->eng.reset(new e3d::Engine(c->hc, eo));
		*out = s.release();
	});
}

// ---- block sharding
static std::vector<int> first_blocks(const e3d_case* c, const int32_t* first_block, int n_ranks) {
	if (!c || !first_block) throw e3d::Error(E3D_ERR_ARG, "null argument");
	if (n_ranks < 1) throw e3d::Error(E3D_ERR_ARG, "sharding: at least one rank");
	return std::vector<int>(first_block, first_block + n_ranks + 1);
}

int e3d_shard_first_blocks(int n_blocks, int n_ranks, int32_t* first_block) {
	if (!first_block) return fail(E3D_ERR_ARG, "null argument");
	return guard([&] {
		const std::vector<int> f = e3d::shard_first_blocks(n_blocks, n_ranks);
		std::copy(f.begin(), f.end(), first_block);
	});
}

int e3d_case_shard_plan(const e3d_case* c, const int32_t* first_block, int n_ranks, int rank, int64_t* send_counts,
                        int64_t* recv_counts, int32_t* send_cells, int32_t* recv_cells) {
	if (!send_counts || !recv_counts) return fail(E3D_ERR_ARG, "null argument");
	return guard([&] {
		const e3d::ShardPlan p = e3d::shard_plan(c->hc, first_blocks(c, first_block, n_ranks), rank);
		for (int r = 0; r < n_ranks; r++) {
			send_counts[r] = p.send_count[r];
			recv_counts[r] = p.recv_count[r];
		}
		if (send_cells)
			for (size_t i = 0; i < p.send_cell.size(); i++) {
				send_cells[2 * i] = p.send_block[i];
				send_cells[2 * i + 1] = p.send_cell[i];
			}
		if (recv_cells)
			for (size_t i = 0; i < p.recv_cell.size(); i++) {
				recv_cells[2 * i] = p.recv_block[i];
				recv_cells[2 * i + 1] = p.recv_cell[i];
			}
	});
}

int e3d_shard_create(const e3d_case* c, const int32_t* first_block, int n_ranks, int rank, const e3d_options* opt,
                     e3d_solver** out) {
	if (!c || !out) return fail(E3D_ERR_ARG, "null argument");
	*out = nullptr;
	return guard([&] {
		const e3d::ShardPlan p = e3d::shard_plan(c->hc, first_blocks(c, first_block, n_ranks), rank);
		const e3d::EngineOptions eo = engine_options(opt);
		auto s = std::make_unique<e3d_solver>();
		s->eng.reset(new e3d::Engine(c->hc, eo, p));
		*out = s.release();
	});
}

static e3d::Engine& shard(e3d_solver* s) {
	e3d::Engine& e = eng(s);
	if (!e.is_shard()) throw e3d::Error(E3D_ERR_STATE, "not a shard solver (e3d_shard_create)");
	return e;
}

int e3d_shard_halo_counts(const e3d_solver* s, int64_t* send_counts, int64_t* recv_counts) {
	if (!send_counts || !recv_counts) return fail(E3D_ERR_ARG, "null argument");
	return guard([&] {
		const e3d::ShardPlan& p = shard(const_cast<e3d_solver*>(s)).shard();
		for (int r = 0; r < p.n_ranks; r++) {
			send_counts[r] = p.send_count[r];
			recv_counts[r] = p.recv_count[r];
		}
	});
}

int e3d_shard_pack(e3d_solver* s, void* send) { return guard([&] { shard(s).shard_pack(send); }); }

int e3d_shard_unpack(e3d_solver* s, const void* recv) { return guard([&] { shard(s).shard_unpack(recv); }); }

int e3d_shard_flow_data(e3d_solver* s, double* out, int64_t capacity, int* n_iters) {
	if (!n_iters) return fail(E3D_ERR_ARG, "null argument");
	return guard([&] {
		e3d::Engine& e = shard(s);
		const int n = e.shard_pending();
		*n_iters = n;
		if (!out) return;
		if (capacity < (int64_t)n * e.n_blocks() * 10) throw e3d::Error(E3D_ERR_ARG, "flow data: buffer too small");
		int m = 0;
		const std::vector<double> v = e.shard_take_flow_data(m);
		std::copy(v.begin(), v.end(), out);
	});
}

int e3d_shard_push_flow_data(e3d_solver* s, const double* all_blocks, int n_iters) {
	return guard([&] { shard(s).shard_push(all_blocks, n_iters); });
}

int e3d_batch_create(const e3d_case* const* cases, int n_cases, const e3d_options* opt, e3d_solver** out) {
	if (!cases || n_cases <= 0 || !out) return fail(E3D_ERR_ARG, "null argument or no case");
	*out = nullptr;
	return guard([&] {
		std::vector<const e3d::HostCase*> list;
		for (int i = 0; i < n_cases; i++) {
			if (!cases[i]) throw e3d::Error(E3D_ERR_ARG, "null case in batch");
			list.push_back(&cases[i]->hc);
		}
		e3d_options o;
		e3d_default_options(&o);
		if (opt) o = *opt;
		e3d::EngineOptions eo;
		eo.precision = o.precision;
		eo.carry_w0 = o.carry_w0;
		eo.use_graph = o.use_graph;
		eo.device = o.device;
		eo.stream = static_cast<cudaStream_t>(o.stream);
		eo.hist_capacity = o.hist_capacity > 0 ? (size_t)o.hist_capacity : 4096;
		eo.renumber = o.renumber;
		auto* s = new e3d_solver;
		try {
			s->eng.reset(new e3d::Engine(list, eo));
		} catch (...) {
			delete s;
			throw;
		}
		*out = s;
	});
}

int e3d_batch_solve(e3d_solver* s, int max_iter, double criterion, int iters_per_launch, int stall_window,
                    int* iters_done, double* device_ms) {
	return guard([&] {
		std::vector<int> done;
		const double ms = eng(s).solve_batch(max_iter, criterion, iters_per_launch, stall_window, done);
		if (iters_done)
			for (size_t i = 0; i < done.size(); i++) iters_done[i] = done[i];
		if (device_ms) *device_ms = ms;
	});
}

int e3d_case_count(const e3d_solver* s, int* n) {
	if (!s || !s->eng || !n) return fail(E3D_ERR_ARG, "null argument");
	*n = s->eng->n_cases();
	return E3D_OK;
}

int e3d_case_history_length(const e3d_solver* s, int case_index, int* n) {
	if (!s || !s->eng || !n) return fail(E3D_ERR_ARG, "null argument");
	if (case_index < 0 || case_index >= s->eng->n_cases()) return fail(E3D_ERR_ARG, "case index out of range");
	*n = (int)s->eng->history(case_index).size();
	return E3D_OK;
}

int e3d_case_history(const e3d_solver* s, int case_index, int first, int count, e3d_iter_record* out) {
	if (!s || !s->eng || !out) return fail(E3D_ERR_ARG, "null argument");
	if (case_index < 0 || case_index >= s->eng->n_cases()) return fail(E3D_ERR_ARG, "case index out of range");
	const auto& h = s->eng->history(case_index);
	if (first < 0 || count < 0 || (size_t)first + (size_t)count > h.size()) return fail(E3D_ERR_ARG, "history range");
	for (int i = 0; i < count; i++) {
		const e3d::IterRecord& r = h[(size_t)first + i];
		e3d_iter_record& o = out[i];
		o.iter = r.iter;
		for (int q = 0; q < 5; q++) {
			o.rms[q] = r.rms[q];
			o.conv[q] = r.conv[q];
		}
		o.cl = r.cl;
		o.cd = r.cd;
		o.cmx = r.cmx;
		o.cmy = r.cmy;
		o.cmz = r.cmz;
	}
	return E3D_OK;
}

int e3d_batch_tuning(const e3d_solver* s, int* tile_cells, int* grid, double* ms_per_iter, int* from_cache) {
	if (!s || !s->eng) return fail(E3D_ERR_ARG, "null argument");
	const auto& t = s->eng->tuning();
	if (tile_cells) *tile_cells = t.tile_cells;
	if (grid) *grid = t.grid;
	if (ms_per_iter) *ms_per_iter = t.ms_per_iter;
	if (from_cache) *from_cache = t.from_cache ? 1 : 0;
	return E3D_OK;
}

int e3d_solver_set_precision(e3d_solver* s, int precision) {
	return guard([&] {
		if (precision == E3D_FP64 || precision == E3D_FP64_FMA) {
			eng(s).widen_to_fp64();
			eng(s).set_fp64_contracted(precision == E3D_FP64_FMA);
		} else if (precision == E3D_FP32_DELTA) {
			eng(s).enter_delta();
		} else if (precision != E3D_FP32 || eng(s).precision() != e3d::PREC_FP32) {
			throw e3d::Error(E3D_ERR_ARG, "a solver switches from FP32 to FP64 or to the FP32 difference form only");
		}
	});
}

int e3d_cell_features(e3d_solver* s, float* out, int64_t n_floats) {
	return guard([&] {
		e3d::Engine& e = eng(s);
		const long long nr = e.n_real_total();
		if (!out || n_floats < 8 * nr) throw e3d::Error(E3D_ERR_ARG, "feature buffer too small");
		e3d::DevBuf<float> d;
		d.alloc((size_t)nr * 8);
		e.cell_features(d.p);
		e3d::cuda_ok(cudaMemcpyAsync(out, d.p, (size_t)nr * 8 * sizeof(float), cudaMemcpyDeviceToHost, e.stream()),
		             "features");
		e3d::cuda_ok(cudaStreamSynchronize(e.stream()), "sync");
	});
}

static e3d::Surrogate& net(e3d_surrogate* m) {
	if (!m || !m->net) throw e3d::Error(E3D_ERR_ARG, "null surrogate");
	return *m->net;
}

int e3d_surrogate_create(int device, uint64_t seed, double gamma, e3d_surrogate** out) {
	if (!out) return fail(E3D_ERR_ARG, "null argument");
	*out = nullptr;
	return guard([&] {
		static_assert(e3d::SurrogateShape::N_PARAM == E3D_SURROGATE_PARAMS, "parameter count");
		static_assert(e3d::SurrogateShape::N_NORM == E3D_SURROGATE_NORM, "normalisation count");
		if (!(gamma > 1.0)) throw e3d::Error(E3D_ERR_ARG, "gamma must exceed 1");
		auto* m = new e3d_surrogate;
		try {
			m->net.reset(new e3d::Surrogate(device, seed, gamma));
		} catch (...) {
			delete m;
			throw;
		}
		*out = m;
	});
}

int e3d_surrogate_free(e3d_surrogate* m) {
	return guard([&] { delete m; });
}

int e3d_surrogate_add_solution(e3d_surrogate* m, e3d_solver* s) {
	return guard([&] { net(m).add_solution(eng(s)); });
}

int e3d_surrogate_add_samples(e3d_surrogate* m, const float* features6, const float* states5, int64_t n) {
	return guard([&] {
		if (n < 0 || (n > 0 && (!features6 || !states5))) throw e3d::Error(E3D_ERR_ARG, "bad sample arrays");
		net(m).add_samples_host(features6, states5, n);
	});
}

int e3d_surrogate_sample_count(const e3d_surrogate* m, int64_t* n) {
	if (!m || !m->net || !n) return fail(E3D_ERR_ARG, "null argument");
	*n = m->net->n_samples();
	return E3D_OK;
}

int e3d_surrogate_clear(e3d_surrogate* m) {
	return guard([&] { net(m).clear_samples(); });
}

int e3d_surrogate_train(e3d_surrogate* m, int steps, int batch, double lr, float* loss_per_step, double* final_loss) {
	return guard([&] {
		if (steps < 0 || !(lr > 0.0)) throw e3d::Error(E3D_ERR_ARG, "steps must be >= 0 and lr > 0");
		std::vector<float> h;
		const double l = net(m).train(steps, batch, lr, loss_per_step ? &h : nullptr);
		if (loss_per_step) std::copy(h.begin(), h.end(), loss_per_step);
		if (final_loss) *final_loss = l;
	});
}

int e3d_surrogate_gradient(e3d_surrogate* m, const float* features6, const float* states5, int n, float* grad,
                           double* loss) {
	return guard([&] {
		if (!features6 || !states5 || !grad) throw e3d::Error(E3D_ERR_ARG, "null argument");
		std::vector<float> g;
		const double l = net(m).gradient(features6, states5, n, g);
		std::copy(g.begin(), g.end(), grad);
		if (loss) *loss = l;
	});
}

int e3d_surrogate_predict(e3d_surrogate* m, const float* features6, int64_t n, float* states5) {
	return guard([&] {
		if (n < 0 || (n > 0 && (!features6 || !states5))) throw e3d::Error(E3D_ERR_ARG, "bad arrays");
		net(m).predict_host(features6, n, states5);
	});
}

int e3d_surrogate_get_params(const e3d_surrogate* m, float* params, float* norm) {
	return guard([&] {
		if (!m || !m->net) throw e3d::Error(E3D_ERR_ARG, "null surrogate");
		if (params) m->net->get_params(params);
		if (norm) m->net->get_normalisation(norm);
	});
}

int e3d_surrogate_set_params(e3d_surrogate* m, const float* params, const float* norm) {
	return guard([&] {
		if (params) net(m).set_params(params);
		if (norm) net(m).set_normalisation(norm);
	});
}

int e3d_warm_start(e3d_solver* s, e3d_surrogate* m, int* n_fallback) {
	return guard([&] {
		const int n = net(m).warm_start(eng(s));
		if (n_fallback) *n_fallback = n;
	});
}

int e3d_solver_free(e3d_solver* s) {
	delete s;
	return E3D_OK;
}

int e3d_solver_sync(e3d_solver* s) { return guard([&] { eng(s).sync(); }); }

int e3d_solver_device_bytes(const e3d_solver* s, int64_t* bytes) {
	if (!s || !s->eng || !bytes) return fail(E3D_ERR_ARG, "null argument");
	*bytes = (int64_t)s->eng->device_bytes();
	return E3D_OK;
}

int e3d_save_w0(e3d_solver* s, int block) { return guard([&] { eng(s).save_w0(block); }); }
int e3d_spectral_radius(e3d_solver* s, int block) { return guard([&] { eng(s).spectral_radius(block); }); }
int e3d_timestep(e3d_solver* s, int block) { return guard([&] { eng(s).timestep(block); }); }
int e3d_gradients(e3d_solver* s, int block, int kind) {
	if (kind != E3D_GRAD_GREEN_GAUSS && kind != E3D_GRAD_LEAST_SQUARES) return fail(E3D_ERR_ARG, "unknown gradient kind");
	return guard([&] { eng(s).gradients(block, kind); });
}
int e3d_limiters(e3d_solver* s, int block, int kind, double omega, double k) {
	if (kind != E3D_LIM_BARTH_JESPERSEN && kind != E3D_LIM_VENKATAKRISHNAN) return fail(E3D_ERR_ARG, "unknown limiter kind");
	return guard([&] { eng(s).limiters(block, kind, omega, k); });
}
int e3d_flux_conv(e3d_solver* s, int block, int scheme) {
	if (scheme != E3D_FLUX_ROE && scheme != E3D_FLUX_AUSM) return fail(E3D_ERR_ARG, "unknown flux scheme");
	return guard([&] { eng(s).flux_conv(block, scheme); });
}
int e3d_flux_diss(e3d_solver* s, int block, int scheme, double beta) {
	if (scheme != E3D_FLUX_ROE && scheme != E3D_FLUX_AUSM) return fail(E3D_ERR_ARG, "unknown flux scheme");
	return guard([&] { eng(s).flux_diss(block, scheme, beta); });
}
int e3d_update_internal(e3d_solver* s, int block, double alpha) {
	return guard([&] { eng(s).update_internal(block, alpha); });
}
int e3d_update_boundary(e3d_solver* s, int block) { return guard([&] { eng(s).update_boundary(block); }); }
int e3d_smooth_residual(e3d_solver* s, int block) { return guard([&] { eng(s).smooth_residual(block); }); }
int e3d_halo(e3d_solver* s) { return guard([&] { eng(s).halo(); }); }

int e3d_flow_data(e3d_solver* s, double* out, int64_t count) {
	if (!out) return fail(E3D_ERR_ARG, "null argument");
	return guard([&] {
		std::vector<double> v;
		eng(s).flow_data(v);
		if (count != (int64_t)v.size()) throw e3d::Error(E3D_ERR_ARG, "flow_data: count must be 10 * n_blocks");
		std::memcpy(out, v.data(), v.size() * sizeof(double));
	});
}

int e3d_iterate(e3d_solver* s, int n_iter) { return guard([&] { eng(s).iterate(n_iter); }); }

int e3d_solve(e3d_solver* s, int max_iter, double criterion, int check_every, int* iters_done) {
	return guard([&] {
		const int n = eng(s).solve(max_iter, criterion, check_every);
		if (iters_done) *iters_done = n;
	});
}

int e3d_iterate_timed(e3d_solver* s, int n_iter, double* device_ms) {
	return guard([&] {
		const double ms = eng(s).iterate_timed(n_iter);
		if (device_ms) *device_ms = ms;
	});
}

int e3d_state_bytes(const e3d_solver* s, int64_t* bytes) {
	if (!s || !s->eng || !bytes) return fail(E3D_ERR_ARG, "null argument");
	*bytes = (int64_t)s->eng->state_bytes();
	return E3D_OK;
}

int e3d_state_export(e3d_solver* s, void* host, int64_t bytes) {
	if (bytes < 0) return fail(E3D_ERR_ARG, "negative size");
	return guard([&] { eng(s).export_state(host, (size_t)bytes); });
}

int e3d_state_import(e3d_solver* s, const void* host, int64_t bytes) {
	if (bytes < 0) return fail(E3D_ERR_ARG, "negative size");
	return guard([&] { eng(s).import_state(host, (size_t)bytes); });
}

int e3d_history_length(const e3d_solver* s, int* n) {
	if (!s || !s->eng || !n) return fail(E3D_ERR_ARG, "null argument");
	*n = (int)s->eng->history().size();
	return E3D_OK;
}

int e3d_history(const e3d_solver* s, int first, int count, e3d_iter_record* out) {
	if (!s || !s->eng || !out) return fail(E3D_ERR_ARG, "null argument");
	const auto& h = s->eng->history();
	if (first < 0 || count < 0 || (size_t)first + (size_t)count > h.size()) return fail(E3D_ERR_ARG, "history range");
	for (int i = 0; i < count; i++) {
		const e3d::IterRecord& r = h[(size_t)first + i];
		e3d_iter_record& o = out[i];
		o.iter = r.iter;
		for (int q = 0; q < 5; q++) {
			o.rms[q] = r.rms[q];
			o.conv[q] = r.conv[q];
		}
		o.cl = r.cl;
		o.cd = r.cd;
		o.cmx = r.cmx;
		o.cmy = r.cmy;
		o.cmz = r.cmz;
	}
	return E3D_OK;
}

int e3d_state_get(e3d_solver* s, int block, const char* name, double* dst, int64_t count) {
	if (!name || !dst) return fail(E3D_ERR_ARG, "null argument");
	return guard([&] {
		std::vector<double> v;
		eng(s).get(name, block, v);
		if (count != (int64_t)v.size())
			throw e3d::Error(E3D_ERR_ARG, std::string(name) + ": count " + std::to_string(count) + " != " +
			                                  std::to_string(v.size()));
		std::memcpy(dst, v.data(), v.size() * sizeof(double));
	});
}

int e3d_state_set(e3d_solver* s, int block, const char* name, const double* src, int64_t count) {
	if (!name || !src || count < 0) return fail(E3D_ERR_ARG, "null argument");
	return guard([&] { eng(s).set(name, block, std::vector<double>(src, src + count)); });
}

int e3d_time_kernels(e3d_solver* s, int n_iter, char* names, int names_len, int* launches, double* total_ms,
                     double* bytes_per_launch, int max_rows, int* rows) {
	if (!names || !launches || !total_ms || !bytes_per_launch || !rows) return fail(E3D_ERR_ARG, "null argument");
	return guard([&] {
		auto t = eng(s).time_kernels(n_iter);
		std::string joined;
		int r = 0;
		for (const auto& k : t) {
			if (r >= max_rows) break;
			if (r) joined += ",";
			joined += k.name;
			launches[r] = k.launches;
			total_ms[r] = k.total_ms;
			bytes_per_launch[r] = k.bytes_per_launch;
			r++;
		}
		if ((int)joined.size() + 1 > names_len) throw e3d::Error(E3D_ERR_ARG, "names buffer too small");
		std::memcpy(names, joined.c_str(), joined.size() + 1);
		*rows = r;
	});
}

int e3d_launches_per_iteration(const e3d_solver* s, int* n) {
	if (!s || !s->eng || !n) return fail(E3D_ERR_ARG, "null argument");
	*n = s->eng->launches_per_iteration();
	return E3D_OK;
}

}  // extern "C"
