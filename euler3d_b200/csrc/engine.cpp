// Device-resident solver: global numbering, uploads, stage sequencing and the
// captured outer iteration.
#include "engine.hpp"
#include "warm.hpp"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <mutex>
#include <tuple>
#include <type_traits>

namespace e3d {

template <class T>
void DevBuf<T>::alloc(size_t count) {
	free();
	n = count;
	if (count) cuda_ok(cudaMalloc(&p, count * sizeof(T)), "cudaMalloc");
}
template <class T>
void DevBuf<T>::upload(const std::vector<T>& h) {
	alloc(h.size());
	if (!h.empty()) cuda_ok(cudaMemcpy(p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice), "upload");
}
template <class T>
void DevBuf<T>::free() {
	if (p) cudaFree(p);
	p = nullptr;
	n = 0;
}
template struct DevBuf<int>;
template struct DevBuf<signed char>;
template struct DevBuf<double>;
template struct DevBuf<float>;
template struct DevBuf<unsigned char>;
template struct DevBuf<unsigned short>;

template <class T>
FusedView<T> Engine::Fused<T>::view(bool flip) const {
	FusedView<T> v{};
	v.Pin = flip ? P1.p : P0.p;
	v.Pout = flip ? P0.p : P1.p;
	v.FS = FS.p;
	v.Rc = Rc.p;
	v.Rd = Rd.p;
	v.dt = dt.p;
	v.sgeo = sgeo.p;
	v.sS = sS.p;
	v.srv = srv.p;
	v.lsw = lsw.p;
	v.vol = vol.p;
	return v;
}

// RK stage tables (Solver/src/RungeKutta.cpp:23-68).
static void rk_tables(int stages, std::vector<double>& a, std::vector<double>& b) {
	switch (stages) {
	case 1: a = {1.0}; b = {1.0}; break;
	case 2: a = {0.6, 1.0}; b = {1.0, 0.0}; break;
	case 3: a = {0.6, 0.6, 1.0}; b = {1.0, 0.0, 0.0}; break;
	case 4: a = {0.25, 1.0 / 3.0, 0.5, 1.0}; b = {1.0, 0.5, 0.0, 0.0}; break;
	case 5: a = {0.2742, 0.2067, 0.5020, 0.5142, 1.0}; b = {1.0, 0.0, 0.56, 0.0, 0.44}; break;
	default: throw Error(E3D_ERR_ARG, "Invalid number of RK stages: " + std::to_string(stages));
	}
}

Engine::Engine(const HostCase& hc, const EngineOptions& opt) : Engine(std::vector<const HostCase*>{&hc}, opt) {}

Engine::Engine(const HostCase& hc, const EngineOptions& opt, const ShardPlan& plan)
    : Engine(std::vector<const HostCase*>{&hc}, opt, &plan) {}

Engine::Engine(const std::vector<const HostCase*>& cases, const EngineOptions& opt) : Engine(cases, opt, nullptr) {}

Engine::Engine(const std::vector<const HostCase*>& cases, const EngineOptions& opt, const ShardPlan* plan)
    : deck_(cases.empty() ? Deck() : cases[0]->deck), opt_(opt) {
	if (cases.empty()) throw Error(E3D_ERR_ARG, "no case");
	for (const HostCase* c : cases) {
		const Deck& d = c->deck;
		if (d.gamma != deck_.gamma || d.cfl != deck_.cfl || d.stages != deck_.stages || d.flux != deck_.flux ||
		    d.order != deck_.order || d.gradient != deck_.gradient || d.limiter != deck_.limiter ||
		    d.omega != deck_.omega || d.k != deck_.k || d.smoothing != deck_.smoothing)
			throw Error(E3D_ERR_ARG, "cases of a batch must share gamma, CFL, RK stages, flux, order, gradient, "
			                         "limiter, omega and k");
	}
	if (opt_.precision != PREC_FP64 && opt_.precision != PREC_FP32) throw Error(E3D_ERR_ARG, "unknown precision");
	if (opt_.device >= 0) cuda_ok(cudaSetDevice(opt_.device), "cudaSetDevice");
	carry_ = opt_.carry_w0 >= 0 ? opt_.carry_w0 : (opt_.precision == PREC_FP32 ? 1 : 0);
	// strategy selection (ResidualCalculator.cpp:72-95, SecondOrder.cpp:50-61)
	if (deck_.flux == "roe") scheme_ = FLUX_ROE;
	else if (deck_.flux == "ausm") scheme_ = FLUX_AUSM;
	else throw Error(E3D_ERR_ARG, "unknown flux scheme '" + deck_.flux + "' (roe|ausm)");
	order_ = deck_.order == 2 ? 2 : 1;
	grad_kind_ = deck_.gradient == "leastsquares" ? GRAD_LEAST_SQUARES : GRAD_GREEN_GAUSS;
	lim_kind_ = deck_.limiter == "venkatakrishnan" ? LIM_VENKATAKRISHNAN : LIM_BARTH_JESPERSEN;
	if (deck_.smoothing && opt_.precision != PREC_FP64)
		throw Error(E3D_ERR_ARG, "residual smoothing (deck smoothing = 1) runs on the FP64 path");
	rk_tables(deck_.stages, alpha_, beta_);
	// physics constants, computed with the reference's expressions on the host
	ph_.gamma = deck_.gamma;
	ph_.gm1 = deck_.gamma - 1.0;
	ph_.gr = deck_.gamma / (deck_.gamma - 1.0);
	ph_.cfl = deck_.cfl;
	ph_.omega = deck_.omega;
	ph_.k3 = deck_.k * deck_.k * deck_.k;
	{  // PrimitiveVariables::calculateFreeVariables (PrimitiveVariables.cpp:41-56)
		const double pi = std::atan(1.0) * 4.0;
		const double a = deck_.aoa_deg * pi / 180.0;
		const double c = std::cos(a), s = std::sin(a);
		ph_.free[0] = 1.0;
		ph_.free[1] = deck_.mach * std::sqrt(deck_.gamma) * c;
		ph_.free[2] = deck_.mach * std::sqrt(deck_.gamma) * s;
		ph_.free[3] = 0.0;
		ph_.free[4] = 1.0;
	}
	// AerodynamicParameters (AerodynamicParameters.cpp:22, :167, :212)
	aoa_rad_ = deck_.aoa_deg * 4. * std::atan(1.) / 180;
	denom_ = (0.5 * deck_.gamma * deck_.mach * deck_.mach) * deck_.cmac;
	ncases_ = (int)cases.size();
	for (const HostCase* c : cases) {
		const Deck& d = c->deck;
		const double pi = std::atan(1.0) * 4.0;
		const double a = d.aoa_deg * pi / 180.0;
		const double cs = std::cos(a), sn = std::sin(a);
		const double f[5] = {1.0, d.mach * std::sqrt(d.gamma) * cs, d.mach * std::sqrt(d.gamma) * sn, 0.0, 1.0};
		case_free_h_.insert(case_free_h_.end(), f, f + 5);
		case_denom_.push_back((0.5 * d.gamma * d.mach * d.mach) * d.cmac);
		case_aoa_.push_back(d.aoa_deg * 4. * std::atan(1.) / 180);
		case_ma_h_.push_back((float)d.mach);
		case_ma_h_.push_back((float)d.aoa_deg);
	}
	have_rms0_.assign(ncases_, 0);
	rms0_.assign(ncases_, {0, 0, 0, 0, 0});
	hist_case_.assign(ncases_, {});
	case_active_.assign(ncases_, 1);
	case_failed_.assign(ncases_, 0);

	if (opt_.stream) {
		st_ = opt_.stream;
	} else {
		cuda_ok(cudaStreamCreateWithFlags(&st_, cudaStreamNonBlocking), "cudaStreamCreate");
		own_stream_ = true;
	}
	setup(cases, plan);
	init_state();
}

void Engine::setup(const std::vector<const HostCase*>& cases, const ShardPlan* plan) {
	case_boff_.assign(1, 0);
	std::vector<const HostBlock*> blocks;
	std::vector<Connexion> conns;
	if (plan) {
		// one rank's range of a single case: its blocks renumbered from 0, the
		// connexions inside the range kept as device copies
		if (cases.size() != 1) throw Error(E3D_ERR_ARG, "a shard holds blocks of one case");
		const HostCase& hc = *cases[0];
		if (plan->b1 > (int)hc.blocks.size() || plan->b0 < 0 || plan->b0 >= plan->b1)
			throw Error(E3D_ERR_ARG, "sharding: block range outside the case");
		for (int b = plan->b0; b < plan->b1; b++) blocks.push_back(&hc.blocks[b]);
		for (Connexion k : plan->local) {
			k.dest_block -= plan->b0;
			k.origin_block -= plan->b0;
			conns.push_back(std::move(k));
		}
		case_boff_.push_back((int)blocks.size());
		build_blocks(blocks, conns);
		shard_ = true;
		need_exchange_ = true;  // Solver.cpp:48: the halo runs before the first iteration
		plan_ = *plan;
		for (const HostBlock& B : hc.blocks) all_n_real_.push_back(B.n_real);
		std::vector<int> xs(plan->send_cell.size()), xr(plan->recv_cell.size());
		for (size_t i = 0; i < xs.size(); i++) {
			const int b = plan->send_block[i] - plan->b0;
			if (b < 0 || b >= nb_ || plan->send_cell[i] < 0 || plan->send_cell[i] >= n_all_b_[b])
				throw Error(E3D_ERR_MESH, "sharding: sent halo cell outside its block");
			xs[i] = device_cell(b, plan->send_cell[i]);
		}
		for (size_t i = 0; i < xr.size(); i++) {
			const int b = plan->recv_block[i] - plan->b0;
			if (b < 0 || b >= nb_ || plan->recv_cell[i] < n_real_b_[b] || plan->recv_cell[i] >= n_all_b_[b])
				throw Error(E3D_ERR_MESH, "sharding: received halo entry is not a ghost cell of its block");
			xr[i] = device_cell(b, plan->recv_cell[i]);
		}
		xsend_.upload(xs);
		xrecv_.upload(xr);
		return;
	}
	for (const HostCase* c : cases) {
		const int off = (int)blocks.size();
		for (const HostBlock& b : c->blocks) blocks.push_back(&b);
		for (Connexion k : c->topo.connexions) {
			k.dest_block += off;
			k.origin_block += off;
			conns.push_back(std::move(k));
		}
		case_boff_.push_back((int)blocks.size());
	}
	build_blocks(blocks, conns);
}

int Engine::device_cell(int b, int local) const {
	return local < n_real_b_[b] ? roff_[b] + pos_[b][local] : NR_ + goff_[b] + (local - n_real_b_[b]);
}

long long Engine::n_real_case(int c) const {
	return (long long)roff_[case_boff_.at(c + 1)] - roff_[case_boff_.at(c)];
}

Engine::~Engine() {
	for (auto& g : graph_)
		if (g) cudaGraphExecDestroy(g);
	if (pgraph_) cudaGraphExecDestroy(pgraph_);
	if (own_stream_ && st_) cudaStreamDestroy(st_);
}

void Engine::check(const char* what) { cuda_ok(cudaGetLastError(), what); }

void Engine::build_blocks(const std::vector<const HostBlock*>& blocks, const std::vector<Connexion>& conns) {
	struct View {
		const std::vector<const HostBlock*>& b;
		size_t size() const { return b.size(); }
		const HostBlock& operator[](size_t i) const { return *b[i]; }
	};
	struct {
		View blocks;
		struct {
			const std::vector<Connexion>& connexions;
		} topo;
	} hc{View{blocks}, {conns}};
	nb_ = (int)hc.blocks.size();
	roff_.assign(nb_ + 1, 0);
	goff_.assign(nb_ + 1, 0);
	foff_.assign(nb_ + 1, 0);
	for (int b = 0; b < nb_; b++) {
		const HostBlock& B = hc.blocks[b];
		roff_[b + 1] = roff_[b] + B.n_real;
		goff_[b + 1] = goff_[b] + (B.n_all - B.n_real);
		foff_[b + 1] = foff_[b] + B.n_faces;
		n_real_b_.push_back(B.n_real);
		n_all_b_.push_back(B.n_all);
	}
	NR_ = roff_[nb_];
	NG_ = goff_[nb_];
	NA_ = NR_ + NG_;
	NF_ = foff_[nb_];
	// device order of each block's real cells (identity unless renumbered)
	pos_.assign(nb_, {});
	for (int b = 0; b < nb_; b++) {
		const HostBlock& B = hc.blocks[b];
		pos_[b].resize(B.n_real);
		const std::vector<int> order = cell_order(B, opt_.renumber);
		for (int i = 0; i < B.n_real; i++) pos_[b][order[i]] = i;
	}
	auto gid = [&](int b, int local) {
		const HostBlock& B = hc.blocks[b];
		return local < B.n_real ? roff_[b] + pos_[b][local] : NR_ + goff_[b] + (local - B.n_real);
	};
	// slots, in global cell order
	std::vector<int> slot_ptr(NA_ + 1, 0);
	for (int b = 0; b < nb_; b++) {
		const HostBlock& B = hc.blocks[b];
		for (int c = 0; c < B.n_all; c++) slot_ptr[gid(b, c) + 1] = B.cell_face_ptr[c + 1] - B.cell_face_ptr[c];
	}
	for (int c = 0; c < NA_; c++) slot_ptr[c + 1] += slot_ptr[c];
	NS_ = slot_ptr[NA_];
	tet4_ = 1;
	for (int c = 0; c < NR_ && tet4_; c++)
		if (slot_ptr[c] != 4 * c || slot_ptr[c + 1] != 4 * c + 4) tet4_ = 0;
	std::vector<int> slot_face(NS_), slot_nbr(NS_), slot_mate(NS_);
	std::vector<double> lsw(3 * (size_t)NS_, 0.0);
	std::vector<int> face_lr(2 * (size_t)NF_);
	std::vector<double> S(3 * (size_t)NF_), nhat(3 * (size_t)NF_), area(NF_), rl(3 * (size_t)NF_), rr(3 * (size_t)NF_),
	    fc(3 * (size_t)NF_), vol(NA_);
	std::vector<int> face_slot_l(NF_, -1), face_slot_r(NF_, -1);
	std::vector<signed char> gkind(NG_, GK_NONE), grefl(NG_, 0);
	std::vector<int> gcase(NG_, 0);
	std::vector<double> wall_denom;
	block_case_.assign(nb_, 0);
	for (int c = 0; c < ncases_; c++)
		for (int b = case_boff_[c]; b < case_boff_[c + 1]; b++) block_case_[b] = c;
	std::vector<int> wall_off(nb_ + 1, 0), wall_face;
	for (int b = 0; b < nb_; b++) {
		const HostBlock& B = hc.blocks[b];
		for (int f = 0; f < B.n_faces; f++) {
			const int F = foff_[b] + f;
			face_lr[2 * (size_t)F] = gid(b, B.face_cells[2 * (size_t)f]);
			face_lr[2 * (size_t)F + 1] = gid(b, B.face_cells[2 * (size_t)f + 1]);
			const double a = B.face_area[f];
			area[F] = a;
			for (int k = 0; k < 3; k++) {
				S[3 * (size_t)F + k] = B.face_normal[3 * (size_t)f + k];
				// the reference normalises by the recomputed norm, which equals face_area_
				nhat[3 * (size_t)F + k] = B.face_normal[3 * (size_t)f + k] / a;
				rl[3 * (size_t)F + k] = B.r_left[3 * (size_t)f + k];
				rr[3 * (size_t)F + k] = B.r_right[3 * (size_t)f + k];
				fc[3 * (size_t)F + k] = B.face_center[3 * (size_t)f + k];
			}
		}
		for (int c = 0; c < B.n_all; c++) {
			const int g = gid(b, c);
			vol[g] = B.cell_volume[c];
			for (int j = B.cell_face_ptr[c]; j < B.cell_face_ptr[c + 1]; j++) {
				const int k = slot_ptr[g] + (j - B.cell_face_ptr[c]);
				const int F = foff_[b] + B.cell_faces[j];
				slot_face[k] = F;
				slot_nbr[k] = gid(b, B.cell_cells[j]);
				if (c < B.n_real)
					for (int d = 0; d < 3; d++) lsw[3 * (size_t)k + d] = B.ls_weights[3 * (size_t)j + d];
				if (face_lr[2 * (size_t)F] == g) face_slot_l[F] = k;
				else face_slot_r[F] = k;
			}
		}
		for (size_t m = 0; m < B.markers.size(); m++) {
			const Marker& mk = B.markers[m];
			const bool real_bnd = (int)m < B.n_real_boundaries;
			for (int gl : mk.ghosts) {
				const int gi = gid(b, gl) - NR_;
				grefl[gi] = real_bnd ? 1 : 0;
				gkind[gi] = (!real_bnd || mk.kind == MK_CONNEXION) ? GK_NONE
				            : mk.kind == MK_WALL                  ? GK_WALL
				            : mk.kind == MK_FARFIELD              ? GK_FARFIELD
				                                                  : GK_SYMMETRY;
			}
		}
		for (int f : B.wall_faces) {
			wall_face.push_back(foff_[b] + f);
			wall_denom.push_back(case_denom_[block_case_[b]]);
		}
		wall_off[b + 1] = (int)wall_face.size();
		for (int g = B.n_real; g < B.n_all; g++) gcase[gid(b, g) - NR_] = block_case_[b];
	}
	for (int F = 0; F < NF_; F++)
		if (face_slot_l[F] < 0 || face_slot_r[F] < 0) throw Error(E3D_ERR_MESH, "internal: face without two slots");
	for (int k = 0; k < NS_; k++) {
		const int F = slot_face[k];
		slot_mate[k] = (face_slot_l[F] == k) ? face_slot_r[F] : ~face_slot_l[F];
	}
	std::vector<int> hdst, hsrc;
	for (const Connexion& c : hc.topo.connexions)
		for (size_t q = 0; q < c.dest_cells.size(); q++) {
			hdst.push_back(gid(c.dest_block, c.dest_cells[q]));
			hsrc.push_back(gid(c.origin_block, c.origin_cells[q]));
		}

	slot_ptr_.upload(slot_ptr);
	slot_face_.upload(slot_face);
	slot_nbr_.upload(slot_nbr);
	slot_mate_.upload(slot_mate);
	face_lr_.upload(face_lr);
	halo_dst_.upload(hdst);
	halo_src_.upload(hsrc);
	wall_off_.upload(wall_off);
	wall_face_.upload(wall_face);
	roff_d_.upload(roff_);
	if (ncases_ > 1) {
		gcase_d_.upload(gcase);
		wall_denom_d_.upload(wall_denom);
	}
	case_free_d_.upload(case_free_h_);
	{  // per-cell and per-case data of the warm-start features
		std::vector<float> cen(3 * (size_t)NR_);
		for (int b = 0; b < nb_; b++) {
			const HostBlock& B = hc.blocks[b];
			for (int c = 0; c < B.n_real; c++)
				for (int d = 0; d < 3; d++) cen[3 * (size_t)gid(b, c) + d] = (float)B.cell_center[3 * (size_t)c + d];
		}
		cen_d_.upload(cen);
		block_case_d_.upload(block_case_);
		std::vector<int> cwo(ncases_ + 1);
		for (int c = 0; c <= ncases_; c++) cwo[c] = wall_off[case_boff_[c]];
		case_wall_off_d_.upload(cwo);
		case_ma_d_.upload(case_ma_h_);
		fallback_d_.alloc(1);
	}
	gkind_.upload(gkind);
	grefl_.upload(grefl);
	S_.upload(S);
	nhat_.upload(nhat);
	area_.upload(area);
	rl_.upload(rl);
	rr_.upload(rr);
	fc_.upload(fc);
	vol64_.upload(vol);
	lsw64_.upload(lsw);

	// fused per-slot geometry, face orientation for fluxes, owner sign for GG
	std::vector<double> sgeo(4 * (size_t)NS_), sS(3 * (size_t)NS_), srv(3 * (size_t)NS_);
	for (int k = 0; k < NS_; k++) {
		const int F = slot_face[k];
		const bool left = face_slot_l[F] == k;
		for (int d = 0; d < 3; d++) {
			sgeo[4 * (size_t)k + d] = nhat[3 * (size_t)F + d];
			double sv = S[3 * (size_t)F + d];
			if (!left) sv *= -1.0;
			sS[3 * (size_t)k + d] = sv;
			srv[3 * (size_t)k + d] = left ? rl[3 * (size_t)F + d] : rr[3 * (size_t)F + d];
		}
		sgeo[4 * (size_t)k + 3] = area[F];
	}
	const bool need_gg = order_ == 2 && grad_kind_ == GRAD_GREEN_GAUSS;
	const bool need_ls = order_ == 2 && grad_kind_ == GRAD_LEAST_SQUARES;
	if (opt_.precision == PREC_FP64) {
		f64_.sgeo.upload(sgeo);
		if (need_gg) f64_.sS.upload(sS);
		f64_.srv.upload(srv);
		if (need_ls) f64_.lsw.upload(lsw);
		f64_.vol.upload(vol);
	} else {
		auto tof = [](const std::vector<double>& a) { return std::vector<float>(a.begin(), a.end()); };
		f32_.sgeo.upload(tof(sgeo));
		if (need_gg) f32_.sS.upload(tof(sS));
		f32_.srv.upload(tof(srv));
		if (need_ls) f32_.lsw.upload(tof(lsw));
		f32_.vol.upload(tof(vol));
	}
	// reductions: chunks of 4096 cells, never straddling a block
	chunk_ = 4096;
	max_chunks_ = 1;
	for (int b = 0; b < nb_; b++) max_chunks_ = std::max(max_chunks_, (roff_[b + 1] - roff_[b] + chunk_ - 1) / chunk_);
	partial_.alloc((size_t)nb_ * max_chunks_ * 5);
	hist_d_.alloc(opt_.hist_capacity * (size_t)nb_ * 10);
	fd_hist_.alloc((size_t)nb_ * 10);
	wall_terms_.alloc(5 * std::max<size_t>(1, wall_face_.n));
	iter_d_.alloc(1);
	bad_d_.alloc(1);
	zero_d_.alloc(1);
	cuda_ok(cudaMemset(iter_d_.p, 0, sizeof(int)), "memset");
	cuda_ok(cudaMemset(bad_d_.p, 0, sizeof(int)), "memset");
	cuda_ok(cudaMemset(zero_d_.p, 0, sizeof(int)), "memset");
}

void Engine::init_state() {
	// all cells, ghosts included, start at freestream
	// (PrimitiveVariables::initializeFlowField, PrimitiveVariables.cpp:58-69);
	// residuals, W0, gradients and limiters start at zero (value-initialised arrays)
	std::vector<double> P(5 * (size_t)NA_);  // packed: [NA] x (rho,u,v,w), then [NA] p
	auto fill_cell = [&](int cell, const double* f) {
		for (int q = 0; q < 4; q++) P[4 * (size_t)cell + q] = f[q];
		P[4 * (size_t)NA_ + cell] = f[4];
	};
	for (int b = 0; b < nb_; b++) {
		const double* f = &case_free_h_[5 * (size_t)block_case_[b]];
		for (int c = roff_[b]; c < roff_[b + 1]; c++) fill_cell(c, f);
		for (int g = NR_ + goff_[b]; g < NR_ + goff_[b + 1]; g++) fill_cell(g, f);
	}
	std::vector<double> zR(5 * (size_t)NR_, 0.0);
	if (opt_.precision == PREC_FP64) {
		f64_.P0.upload(P);
		f64_.P1.upload(P);
		f64_.Rc.upload(zR);
		f64_.Rd.upload(zR);
		f64_.dt.upload(std::vector<double>(NR_, 0.0));
		f64_.FS.alloc(order_ == 2 ? 5 * (size_t)NS_ : 0);
		srad_.upload(std::vector<double>(NR_, 0.0));
		grad_.upload(std::vector<double>(15 * (size_t)NA_, 0.0));
		lim_.upload(std::vector<double>(5 * (size_t)NA_, 0.0));
	} else {
		std::vector<float> Pf(P.begin(), P.end());
		f32_.P0.upload(Pf);
		f32_.P1.upload(Pf);
		f32_.Rc.upload(std::vector<float>(5 * (size_t)NR_, 0.f));
		f32_.Rd.upload(std::vector<float>(5 * (size_t)NR_, 0.f));
		f32_.dt.upload(std::vector<float>(NR_, 0.f));
		f32_.FS.alloc(order_ == 2 ? 5 * (size_t)NS_ : 0);
	}
	W0_.upload(zR);
	if (deck_.smoothing) irs_.alloc(10 * (size_t)NR_);  // before any graph capture
	if (carry_) {
		// W carried in FP64 from the freestream conservative state
		std::vector<double> W(5 * (size_t)NR_);
		for (int c = 0; c < NR_; c++) {
			const int b = (int)(std::upper_bound(roff_.begin(), roff_.end(), c) - roff_.begin()) - 1;
			const double* f = &case_free_h_[5 * (size_t)block_case_[b]];
			W[c] = f[0];
			W[(size_t)NR_ + c] = f[0] * f[1];
			W[2 * (size_t)NR_ + c] = f[0] * f[2];
			W[3 * (size_t)NR_ + c] = f[0] * f[3];
			W[4 * (size_t)NR_ + c] = 0.5 * f[0] * (f[1] * f[1] + f[2] * f[2] + f[3] * f[3]) + 1. / (ph_.gamma - 1.0) * f[4];
		}
		W0_.upload(W);
	}
	cur_ = 0;
	count_device_bytes();
}

void Engine::count_device_bytes() {
	size_t bytes = 0;
	for (auto* b : {&slot_ptr_, &slot_face_, &slot_nbr_, &slot_mate_, &face_lr_, &halo_dst_, &halo_src_, &wall_off_,
	                &wall_face_, &roff_d_, &xsend_, &xrecv_})
		bytes += b->n * sizeof(int);
	for (auto* b : {&S_, &nhat_, &area_, &rl_, &rr_, &fc_, &vol64_, &lsw64_, &W0_, &srad_, &grad_, &lim_, &partial_,
	                &hist_d_})
		bytes += b->n * sizeof(double);
	for (auto* b : {&f64_.P0, &f64_.P1, &f64_.FS, &f64_.Rc, &f64_.Rd, &f64_.dt, &f64_.sgeo, &f64_.sS, &f64_.srv,
	                &f64_.lsw, &f64_.vol})
		bytes += b->n * sizeof(double);
	for (auto* b : {&f32_.P0, &f32_.P1, &f32_.FS, &f32_.Rc, &f32_.Rd, &f32_.dt, &f32_.sgeo, &f32_.sS, &f32_.srv,
	                &f32_.lsw, &f32_.vol, &Pb32_, &dW_, &Rb_})
		bytes += b->n * sizeof(float);
	bytes += Pb64_.n * sizeof(double);
	dev_bytes_ = bytes;
}

void Engine::require_fp64(const char* what) const {
	if (opt_.precision != PREC_FP64)
		throw Error(E3D_ERR_STATE, std::string(what) + " needs an FP64 solver (strategy-level calls keep the "
		                                               "reference's FP64 arrays)");
}

StateView Engine::state64() {
	StateView s{};
	s.prim = cur_ ? f64_.P1.p : f64_.P0.p;
	s.rc = f64_.Rc.p;
	s.rd = f64_.Rd.p;
	s.w0 = W0_.p;
	s.grad = grad_.p;
	s.lim = lim_.p;
	s.dt = f64_.dt.p;
	s.srad = srad_.p;
	return s;
}

static GeoView make_geo(int NR, int NG, int NA, int NF, int NS, const int* sp, const int* sf, const int* sn,
                        const int* flr, const double* S, const double* nh, const double* ar, const double* rl,
                        const double* rr, const double* vol, const double* lsw, const signed char* gk,
                        const signed char* gr) {
	GeoView g{};
	g.NR = NR;
	g.NG = NG;
	g.NA = NA;
	g.NF = NF;
	g.NS = NS;
	g.slot_ptr = sp;
	g.slot_face = sf;
	g.slot_nbr = sn;
	g.face_lr = flr;
	g.S = S;
	g.nhat = nh;
	g.area = ar;
	g.rl = rl;
	g.rr = rr;
	g.vol = vol;
	g.lsw = lsw;
	g.gkind = gk;
	g.grefl = gr;
	return g;
}

void Engine::block_range(int block, int& r0, int& r1, int& g0, int& g1) const {
	if (block < -1 || block >= nb_) throw Error(E3D_ERR_ARG, "block index out of range");
	if (block < 0) {
		r0 = 0;
		r1 = NR_;
		g0 = 0;
		g1 = NG_;
	} else {
		r0 = roff_[block];
		r1 = roff_[block + 1];
		g0 = goff_[block];
		g1 = goff_[block + 1];
	}
}

#define E3D_GEO                                                                                                     \
	make_geo(NR_, NG_, NA_, NF_, NS_, slot_ptr_.p, slot_face_.p, slot_nbr_.p, face_lr_.p, S_.p, nhat_.p, area_.p, rl_.p, \
	         rr_.p, vol64_.p, lsw64_.p, gkind_.p, grefl_.p)

void Engine::save_w0(int block) {
	require_fp64("save_w0");
	int r0, r1, g0, g1;
	block_range(block, r0, r1, g0, g1);
	launch_save_w0(E3D_GEO, state64(), ph_, r0, r1, st_);
	check("save_w0");
}
void Engine::spectral_radius(int block) {
	require_fp64("spectral_radius");
	int r0, r1, g0, g1;
	block_range(block, r0, r1, g0, g1);
	launch_spectral_radius(E3D_GEO, state64(), ph_, r0, r1, st_);
	check("spectral_radius");
}
void Engine::timestep(int block) {
	require_fp64("timestep");
	int r0, r1, g0, g1;
	block_range(block, r0, r1, g0, g1);
	launch_timestep(E3D_GEO, state64(), ph_, r0, r1, st_);
	check("timestep");
}
void Engine::gradients(int block, int kind) {
	require_fp64("gradients");
	int r0, r1, g0, g1;
	block_range(block, r0, r1, g0, g1);
	launch_gradients(E3D_GEO, state64(), kind, r0, r1, st_);
	check("gradients");
}
void Engine::limiters(int block, int kind, double omega, double k) {
	require_fp64("limiters");
	int r0, r1, g0, g1;
	block_range(block, r0, r1, g0, g1);
	Physics ph = ph_;
	ph.omega = omega;
	ph.k3 = k * k * k;
	launch_limiters(E3D_GEO, state64(), ph, kind, r0, r1, g0, g1, st_);
	check("limiters");
}
void Engine::flux_conv(int block, int scheme) {
	require_fp64("flux_conv");
	int r0, r1, g0, g1;
	block_range(block, r0, r1, g0, g1);
	launch_flux_conv(E3D_GEO, state64(), ph_, scheme, r0, r1, st_);
	check("flux_conv");
}
void Engine::flux_diss(int block, int scheme, double beta) {
	require_fp64("flux_diss");
	int r0, r1, g0, g1;
	block_range(block, r0, r1, g0, g1);
	launch_flux_diss(E3D_GEO, state64(), ph_, scheme, beta, r0, r1, st_);
	check("flux_diss");
}
void Engine::update_internal(int block, double alpha) {
	require_fp64("update_internal");
	int r0, r1, g0, g1;
	block_range(block, r0, r1, g0, g1);
	launch_update(E3D_GEO, state64(), ph_, alpha, r0, r1, st_);
	check("update_internal");
}
void Engine::smooth_residual(int block) {
	require_fp64("smooth_residual");
	int r0, r1, g0, g1;
	block_range(block, r0, r1, g0, g1);
	if (irs_.n < 10 * (size_t)NR_) irs_.alloc(10 * (size_t)NR_);
	launch_smooth(E3D_GEO, state64(), irs_.p, r0, r1, st_);
	check("smooth_residual");
}
void Engine::update_boundary(int block) {
	require_fp64("update_boundary");
	int r0, r1, g0, g1;
	block_range(block, r0, r1, g0, g1);
	launch_bc(E3D_GEO, state64(), ph_, g0, g1, st_);
	check("update_boundary");
}
void Engine::halo() {
	if (opt_.precision == PREC_FP64)
		launch_halo<double>((int)halo_dst_.n, halo_dst_.p, halo_src_.p, NA_, cur_ ? f64_.P1.p : f64_.P0.p,
		                    cur_ ? f64_.P0.p : f64_.P1.p, st_);
	else
		launch_halo<float>((int)halo_dst_.n, halo_dst_.p, halo_src_.p, NA_, cur_ ? f32_.P1.p : f32_.P0.p,
		                   cur_ ? f32_.P0.p : f32_.P1.p, st_);
	check("halo");
	started_ = true;
}

static ReduceArgs make_reduce(int NR, int NA, int nb, const int* roff, int chunk, int max_chunks, double* partial,
                              const int* woff, const int* wface, int n_wall, double* wall_terms, const int* flr,
                              const double* S, const double* fc, double denom, double* hist, const int* d_iter,
                              int* d_bad) {
	ReduceArgs a{};
	a.NR = NR;
	a.NA = NA;
	a.nblocks = nb;
	a.roff = roff;
	a.chunk = chunk;
	a.max_chunks = max_chunks;
	a.partial = partial;
	a.wall_off = woff;
	a.wall_face = wface;
	a.n_wall = n_wall;
	a.wall_terms = wall_terms;
	a.face_lr = flr;
	a.S = S;
	a.fc = fc;
	a.denom = denom;
	a.wall_denom = nullptr;
	a.hist = hist;
	a.stride = nb * 10;
	a.d_iter = d_iter;
	a.d_bad = d_bad;
	return a;
}

void Engine::flow_data(std::vector<double>& out) {
	require_not_delta("flow_data");
	ReduceArgs a = make_reduce(NR_, NA_, nb_, roff_d_.p, chunk_, max_chunks_, partial_.p, wall_off_.p, wall_face_.p,
	                           (int)wall_face_.n, wall_terms_.p, face_lr_.p, S_.p, fc_.p, denom_, fd_hist_.p, zero_d_.p,
	                           bad_d_.p);
	a.wall_denom = wall_denom_d_.p;
	if (opt_.precision == PREC_FP64)
		launch_reduce<double>(a, f64_.Rc.p, f64_.Rd.p, cur_ ? f64_.P1.p : f64_.P0.p, st_);
	else
		launch_reduce<float>(a, f32_.Rc.p, f32_.Rd.p, cur_ ? f32_.P1.p : f32_.P0.p, st_);
	check("flow_data");
	out.resize((size_t)nb_ * 10);
	cuda_ok(cudaMemcpyAsync(out.data(), fd_hist_.p, out.size() * sizeof(double), cudaMemcpyDeviceToHost, st_), "d2h");
	cuda_ok(cudaStreamSynchronize(st_), "sync");
}

// One outer iteration (Solver::solve body, Solver.cpp:83-96, all blocks at
// once): W0 + time step, the RK stages (RungeKutta.cpp:85-92), norms and forces
// (PostProcessing::computeFlowData), then the inter-block halo.
// One outer iteration with residual smoothing (deck smoothing = 1): the
// reference's call sequence on the FP64 strategy-level kernels
// (RungeKutta.cpp:85-92, ResidualCalculator.cpp:24-41 with the smoother between
// the dissipative flux and the update), primitives updated in place.
void Engine::smoothed_iteration_body() {
	save_w0(-1);
	spectral_radius(-1);
	timestep(-1);
	for (size_t s = 0; s < alpha_.size(); s++) {
		if (order_ == 2) {
			gradients(-1, grad_kind_);
			limiters(-1, lim_kind_, deck_.omega, deck_.k);
		}
		flux_conv(-1, scheme_);
		flux_diss(-1, scheme_, beta_[s]);
		smooth_residual(-1);
		update_internal(-1, alpha_[s]);
		update_boundary(-1);
	}
	double* prim = cur_ ? f64_.P1.p : f64_.P0.p;
	double* other = cur_ ? f64_.P0.p : f64_.P1.p;
	ReduceArgs a = make_reduce(NR_, NA_, nb_, roff_d_.p, chunk_, max_chunks_, partial_.p, wall_off_.p, wall_face_.p,
	                           (int)wall_face_.n, wall_terms_.p, face_lr_.p, S_.p, fc_.p, denom_, hist_d_.p, iter_d_.p,
	                           bad_d_.p);
	a.wall_denom = wall_denom_d_.p;
	launch_reduce<double>(a, f64_.Rc.p, f64_.Rd.p, prim, st_);
	launch_halo<double>((int)halo_dst_.n, halo_dst_.p, halo_src_.p, NA_, prim, other, st_);
	launch_iter_advance(iter_d_.p, st_);
}

template <class T>
void Engine::iteration_body(Fused<T>& f, int parity, std::vector<cudaEvent_t>* marks) {
	if (deck_.smoothing) {
		smoothed_iteration_body();
		return;
	}
	const int stages = (int)alpha_.size();
	auto mark = [&]() {
		if (marks) {
			cudaEvent_t e;
			cuda_ok(cudaEventCreate(&e), "event");
			cuda_ok(cudaEventRecord(e, st_), "event");
			marks->push_back(e);
		}
	};
	int p = parity;
	for (int s = 0; s < stages; s++) {
		FusedView<T> v = f.view(p != 0);
		v.NR = NR_;
		v.NG = NG_;
		v.NA = NA_;
		v.NS = NS_;
		v.tet4 = tet4_;
		v.slot_ptr = slot_ptr_.p;
		v.slot_nbr = slot_nbr_.p;
		v.slot_mate = slot_mate_.p;
		v.gkind = gkind_.p;
		v.grefl = grefl_.p;
		v.W0 = W0_.p;
		v.case_free = ncases_ > 1 ? case_free_d_.p : nullptr;  // single case: Physics::free
		v.gcase = gcase_d_.p;
		if (order_ == 2) {
			launch_recon<T>(v, ph_, grad_kind_, lim_kind_, s == 0, carry_, st_);
			mark();
		} else if (s == 0) {
			launch_start<T>(v, ph_, carry_, st_);
			mark();
		}
		// the reference always evaluates the dissipative flux: its guard
		// `beta > (10^-16)` is an XOR (== -6) and is always true
		// (ResidualCalculator.cpp:33)
		launch_flux_update<T>(v, ph_, scheme_, order_ == 1, alpha_[s], beta_[s], s == stages - 1, carry_, st_);
		mark();
		p ^= 1;
	}
	ReduceArgs a = make_reduce(NR_, NA_, nb_, roff_d_.p, chunk_, max_chunks_, partial_.p, wall_off_.p, wall_face_.p,
	                           (int)wall_face_.n, wall_terms_.p, face_lr_.p, S_.p, fc_.p, denom_, hist_d_.p, iter_d_.p,
	                           bad_d_.p);
	a.wall_denom = wall_denom_d_.p;
	launch_reduce<T>(a, f.Rc.p, f.Rd.p, p ? f.P1.p : f.P0.p, st_);
	launch_halo<T>((int)halo_dst_.n, halo_dst_.p, halo_src_.p, NA_, p ? f.P1.p : f.P0.p, p ? f.P0.p : f.P1.p, st_);
	launch_iter_advance(iter_d_.p, st_);
	mark();
}

int Engine::launches_per_iteration() const {
	const int stages = (int)alpha_.size();
	if (deck_.smoothing)  // W0, spectral radius, time step; per stage (grad, lim,) conv, diss, 2 smoothing, update, BC
		return 3 + stages * ((order_ == 2 ? 2 : 0) + 6) + 3 + (halo_dst_.n ? 1 : 0) + 1;
	return (order_ == 2 ? 2 * stages : stages + 1) + 3 /*reduce*/ + (halo_dst_.n ? 1 : 0) + 1 /*advance*/;
}

template <class T>
void Engine::run_iterations(Fused<T>& f, int n) {
	const int stages = (int)alpha_.size();
	while (n > 0) {
		if (dev_iter_ == (int)opt_.hist_capacity) collect_history(total_iter_, dev_iter_);
		const int room = (int)opt_.hist_capacity - dev_iter_;
		const int m = std::min(n, room);
		for (int i = 0; i < m; i++) {
			if (opt_.use_graph) {
				if (!graph_[cur_]) {
					cudaGraph_t g;
					cuda_ok(cudaStreamBeginCapture(st_, cudaStreamCaptureModeThreadLocal), "capture");
					iteration_body<T>(f, cur_, nullptr);
					cuda_ok(cudaStreamEndCapture(st_, &g), "capture");
					cuda_ok(cudaGraphInstantiate(&graph_[cur_], g, 0), "graph instantiate");
					cudaGraphDestroy(g);
				}
				cuda_ok(cudaGraphLaunch(graph_[cur_], st_), "graph launch");
			} else {
				iteration_body<T>(f, cur_, nullptr);
				check("iteration");
			}
			cur_ ^= deck_.smoothing ? 0 : (stages & 1);
		}
		dev_iter_ += m;
		n -= m;
		// a shard's records need every rank's norms: kept on the device until taken
		if (!shard_) collect_history(total_iter_, dev_iter_);
	}
	if (shard_) need_exchange_ = !plan_.recv_cell.empty() || !plan_.send_cell.empty();
}

void Engine::require_exchanged(int n_iter) const {
	if (!shard_ || (plan_.recv_cell.empty() && plan_.send_cell.empty())) return;
	if (n_iter > 1)
		throw Error(E3D_ERR_ARG, "a shard advances one iteration at a time: its halo crosses ranks after each one");
	if (n_iter == 1 && need_exchange_)
		throw Error(E3D_ERR_STATE, "shard halo not exchanged: pack, move the buffers and unpack before iterating");
}

void Engine::iterate(int n) {
	require_not_delta("iterate");
	if (n < 0) throw Error(E3D_ERR_ARG, "negative iteration count");
	require_exchanged(n);
	if (!started_) halo();  // Solver.cpp:48, before the first iteration
	if (opt_.precision == PREC_FP64) run_iterations(f64_, n);
	else run_iterations(f32_, n);
}

double Engine::iterate_timed(int n) {
	require_not_delta("iterate_timed");
	if (n < 0) throw Error(E3D_ERR_ARG, "negative iteration count");
	require_exchanged(n);
	if (!started_) halo();
	if ((int)opt_.hist_capacity - dev_iter_ < n) collect_history(total_iter_, dev_iter_);
	if ((int)opt_.hist_capacity < n) throw Error(E3D_ERR_LIMIT, "timed run longer than the history capacity");
	cudaEvent_t e0, e1;
	cuda_ok(cudaEventCreate(&e0), "event");
	cuda_ok(cudaEventCreate(&e1), "event");
	cuda_ok(cudaEventRecord(e0, st_), "event");
	const int stages = (int)alpha_.size();
	for (int i = 0; i < n; i++) {
		if (opt_.use_graph) {
			if (!graph_[cur_]) {
				cudaGraph_t g;
				cuda_ok(cudaStreamBeginCapture(st_, cudaStreamCaptureModeThreadLocal), "capture");
				if (opt_.precision == PREC_FP64) iteration_body<double>(f64_, cur_, nullptr);
				else iteration_body<float>(f32_, cur_, nullptr);
				cuda_ok(cudaStreamEndCapture(st_, &g), "capture");
				cuda_ok(cudaGraphInstantiate(&graph_[cur_], g, 0), "graph instantiate");
				cudaGraphDestroy(g);
			}
			cuda_ok(cudaGraphLaunch(graph_[cur_], st_), "graph launch");
		} else {
			if (opt_.precision == PREC_FP64) iteration_body<double>(f64_, cur_, nullptr);
			else iteration_body<float>(f32_, cur_, nullptr);
			check("iteration");
		}
		cur_ ^= deck_.smoothing ? 0 : (stages & 1);
	}
	cuda_ok(cudaEventRecord(e1, st_), "event");
	cuda_ok(cudaEventSynchronize(e1), "event sync");
	float ms = 0.f;
	cuda_ok(cudaEventElapsedTime(&ms, e0, e1), "elapsed");
	cudaEventDestroy(e0);
	cudaEventDestroy(e1);
	dev_iter_ += n;
	if (shard_) need_exchange_ = !plan_.recv_cell.empty() || !plan_.send_cell.empty();
	else collect_history(total_iter_, dev_iter_);
	return (double)ms;
}

namespace {
struct StateHeader {
	char magic[8];
	int32_t precision, n_blocks;
	int64_t NA, NR, iters;
	int32_t have_rms0, carry;
	double rms0[5];
};
}  // namespace

size_t Engine::state_bytes() const {
	const size_t b = opt_.precision == PREC_FP64 ? 8 : 4;
	return sizeof(StateHeader) + 5 * (size_t)NA_ * b + 5 * (size_t)NR_ * 8;
}

// Layout: header, then primitives [5][NA] in device order (real cells of every
// block, then ghost cells of every block) and precision, then FP64 W0 [5][NR].
void Engine::export_state(void* host, size_t bytes) {
	require_not_delta("export_state");
	if (!host || bytes < state_bytes()) throw Error(E3D_ERR_ARG, "state buffer too small");
	StateHeader h{};
	std::memcpy(h.magic, "E3DSTAT1", 8);
	h.precision = opt_.precision;
	h.n_blocks = nb_;
	h.NA = NA_;
	h.NR = NR_;
	h.iters = total_iter_ + dev_iter_;
	if (ncases_ != 1) throw Error(E3D_ERR_STATE, "state export covers single-case solvers");
	h.have_rms0 = have_rms0_[0] ? 1 : 0;
	h.carry = carry_;
	for (int q = 0; q < 5; q++) h.rms0[q] = rms0_[0][q];
	std::memcpy(host, &h, sizeof(h));
	char* p = static_cast<char*>(host) + sizeof(h);
	const size_t pb = (opt_.precision == PREC_FP64 ? 8 : 4) * 5 * (size_t)NA_;
	const void* P = opt_.precision == PREC_FP64 ? (const void*)(cur_ ? f64_.P1.p : f64_.P0.p)
	                                            : (const void*)(cur_ ? f32_.P1.p : f32_.P0.p);
	cuda_ok(cudaMemcpyAsync(p, P, pb, cudaMemcpyDeviceToHost, st_), "export");
	cuda_ok(cudaMemcpyAsync(p + pb, W0_.p, 5 * (size_t)NR_ * 8, cudaMemcpyDeviceToHost, st_), "export");
	cuda_ok(cudaStreamSynchronize(st_), "sync");
}

void Engine::import_state(const void* host, size_t bytes) {
	require_not_delta("import_state");
	if (!host || bytes < sizeof(StateHeader)) throw Error(E3D_ERR_ARG, "state buffer too small");
	StateHeader h;
	std::memcpy(&h, host, sizeof(h));
	if (std::memcmp(h.magic, "E3DSTAT1", 8) != 0) throw Error(E3D_ERR_FORMAT, "not an e3d state buffer");
	if (h.precision != opt_.precision || h.NA != NA_ || h.NR != NR_ || h.n_blocks != nb_)
		throw Error(E3D_ERR_ARG, "state buffer is for another case or precision");
	if (bytes < state_bytes()) throw Error(E3D_ERR_ARG, "state buffer truncated");
	const char* p = static_cast<const char*>(host) + sizeof(h);
	const size_t pb = (opt_.precision == PREC_FP64 ? 8 : 4) * 5 * (size_t)NA_;
	void* P = opt_.precision == PREC_FP64 ? (void*)(cur_ ? f64_.P1.p : f64_.P0.p) : (void*)(cur_ ? f32_.P1.p : f32_.P0.p);
	void* Q = opt_.precision == PREC_FP64 ? (void*)(cur_ ? f64_.P0.p : f64_.P1.p) : (void*)(cur_ ? f32_.P0.p : f32_.P1.p);
	cuda_ok(cudaMemcpyAsync(P, p, pb, cudaMemcpyHostToDevice, st_), "import");
	// the other buffer too: ghost cells that no stage rewrites must agree in both
	cuda_ok(cudaMemcpyAsync(Q, P, pb, cudaMemcpyDeviceToDevice, st_), "import");
	cuda_ok(cudaMemcpyAsync(W0_.p, p + pb, 5 * (size_t)NR_ * 8, cudaMemcpyHostToDevice, st_), "import");
	cuda_ok(cudaStreamSynchronize(st_), "sync");
	if (dev_iter_) collect_history(total_iter_, dev_iter_);
	total_iter_ = (int)h.iters;
	if (ncases_ != 1) throw Error(E3D_ERR_STATE, "state import covers single-case solvers");
	have_rms0_[0] = h.have_rms0 != 0;
	for (int q = 0; q < 5; q++) rms0_[0][q] = h.rms0[q];
	started_ = true;
}

// One whole-case record from the per-block norms and forces x[nblocks][10].
IterRecord Engine::make_record(int cs, const double* x, int nblocks, const int* n_real) {
	IterRecord r{};
	r.iter = (int)hist_case_[cs].size();
	const double aoa = case_aoa_[cs];
	for (int b = 0; b < nblocks; b++, x += 10) {
		const double N = (double)n_real[b];
		// Convergence::calculate*Rms (Convergence.cpp:27-48) then the block sum
		// (BlockCommunicator.cpp:342-369)
		for (int q = 0; q < 5; q++) r.rms[q] += (1. / N) * std::pow(x[q], 0.5);
		// AerodynamicParameters::calculateGlobalCl/Cd (AerodynamicParameters.cpp:114-138)
		const double cl_ = x[5], cd_ = x[6];
		r.cl += cl_ * std::cos(aoa) - cd_ * std::sin(aoa);
		r.cd += cl_ * std::sin(aoa) + cd_ * std::cos(aoa);
		r.cmx += x[7];
		r.cmy += x[8];
		r.cmz += x[9];
	}
	if (!have_rms0_[cs]) {
		for (int q = 0; q < 5; q++) rms0_[cs][q] = r.rms[q];
		have_rms0_[cs] = 1;
	}
	for (int q = 0; q < 5; q++) r.conv[q] = std::log10(r.rms[q]) - std::log10(rms0_[cs][q]);
	return r;
}

void Engine::shard_pack(void* send) {
	if (!shard_) throw Error(E3D_ERR_STATE, "not a shard");
	const int n = (int)xsend_.n;
	if (n && !send) throw Error(E3D_ERR_ARG, "null send buffer");
	if (opt_.precision == PREC_FP64)
		launch_halo_pack<double>(n, xsend_.p, NA_, cur_ ? f64_.P1.p : f64_.P0.p, static_cast<double*>(send), st_);
	else
		launch_halo_pack<float>(n, xsend_.p, NA_, cur_ ? f32_.P1.p : f32_.P0.p, static_cast<float*>(send), st_);
	check("halo pack");
}

void Engine::shard_unpack(const void* recv) {
	if (!shard_) throw Error(E3D_ERR_STATE, "not a shard");
	const int n = (int)xrecv_.n;
	if (n && !recv) throw Error(E3D_ERR_ARG, "null receive buffer");
	if (opt_.precision == PREC_FP64)
		launch_halo_unpack<double>(n, xrecv_.p, NA_, static_cast<const double*>(recv), cur_ ? f64_.P1.p : f64_.P0.p,
		                           cur_ ? f64_.P0.p : f64_.P1.p, st_);
	else
		launch_halo_unpack<float>(n, xrecv_.p, NA_, static_cast<const float*>(recv), cur_ ? f32_.P1.p : f32_.P0.p,
		                          cur_ ? f32_.P0.p : f32_.P1.p, st_);
	check("halo unpack");
	need_exchange_ = false;
}

int Engine::shard_pending() {
	if (!shard_) throw Error(E3D_ERR_STATE, "not a shard");
	collect_history(total_iter_, dev_iter_);
	return raw_iters_;
}

std::vector<double> Engine::shard_take_flow_data(int& n_iters) {
	shard_pending();
	std::vector<double> out;
	out.swap(raw_pending_);
	n_iters = raw_iters_;
	raw_iters_ = 0;
	return out;
}

void Engine::shard_push(const double* all_blocks, int n_iters) {
	if (!shard_) throw Error(E3D_ERR_STATE, "not a shard");
	if (n_iters < 0 || (n_iters && !all_blocks)) throw Error(E3D_ERR_ARG, "flow data: bad arguments");
	const int nb = (int)all_n_real_.size();
	for (int i = 0; i < n_iters; i++)
		hist_case_[0].push_back(make_record(0, all_blocks + (size_t)i * nb * 10, nb, all_n_real_.data()));
}

// Pulls the device history records, converts them to the reference's mesh-level
// quantities (a shard keeps them raw until the caller has every rank's), and
// resets the device counter.
void Engine::collect_history(int first_iter, int n) {
	if (n <= 0) return;
	std::vector<double> h((size_t)n * nb_ * 10);
	cuda_ok(cudaMemcpyAsync(h.data(), hist_d_.p, h.size() * sizeof(double), cudaMemcpyDeviceToHost, st_), "d2h");
	cuda_ok(cudaMemsetAsync(iter_d_.p, 0, sizeof(int), st_), "memset");
	int bad = 0;
	cuda_ok(cudaMemcpyAsync(&bad, bad_d_.p, sizeof(int), cudaMemcpyDeviceToHost, st_), "d2h");
	cuda_ok(cudaStreamSynchronize(st_), "sync");
	dev_iter_ = 0;
	if (shard_) {
		raw_pending_.insert(raw_pending_.end(), h.begin(), h.end());
		raw_iters_ += n;
		total_iter_ += n;
		if (bad) throw Error(E3D_ERR_NONFINITE, "non-finite residual norm by iteration " + std::to_string(total_iter_ - 1));
		return;
	}
	for (int i = 0; i < n; i++)
		for (int cs = 0; cs < ncases_; cs++) {
			if (!case_active_[cs]) continue;
			const int b0 = case_boff_[cs];
			hist_case_[cs].push_back(make_record(cs, &h[((size_t)i * nb_ + b0) * 10], case_boff_[cs + 1] - b0,
			                                     &n_real_b_[b0]));
		}
	total_iter_ += n;
	if (bad && tolerate_nonfinite_) {
		// a batch solve drops the cases whose residual turned non-finite and goes on
		int failed = 0, alive = 0;
		for (int cs = 0; cs < ncases_; cs++) {
			if (!case_active_[cs]) continue;
			const auto& hc = hist_case_[cs];
			bool ok = true;
			for (int i = std::max(0, (int)hc.size() - n); i < (int)hc.size(); i++)
				for (int q = 0; q < 5; q++) ok = ok && std::isfinite(hc[i].rms[q]);
			if (!ok) {
				case_failed_[cs] = 1;
				case_active_[cs] = 0;
				failed++;
			} else {
				alive++;
			}
		}
		if (failed > 0 && alive > 0) {
			cuda_ok(cudaMemsetAsync(bad_d_.p, 0, sizeof(int), st_), "memset");
			bad = 0;
		}
	}
	if (bad) throw Error(E3D_ERR_NONFINITE, "non-finite residual norm by iteration " + std::to_string(total_iter_ - 1));
}

int Engine::solve(int max_iter, double criterion, int check_every) {
	require_not_delta("solve");
	if (shard_)
		throw Error(E3D_ERR_STATE, "a shard's stop test needs the norms of every rank: iterate, exchange and push "
		                           "the gathered flow data instead");
	if (check_every < 1) check_every = 1;
	int done = 0;
	while (true) {
		const std::vector<IterRecord>& hist_ = hist_case_[0];
		const size_t before = hist_.size();
		iterate(std::min(check_every, std::max(1, max_iter - total_iter_)));
		for (size_t i = before; i < hist_.size(); i++) {
			// PostProcessing::checkStopSolver (PostProcessing.cpp:77)
			if (hist_[i].iter + 1 == max_iter || hist_[i].conv[0] <= criterion) return hist_[i].iter + 1;
		}
		done = total_iter_;
		if (done >= max_iter) return done;
	}
}

void Engine::sync() {
	cuda_ok(cudaStreamSynchronize(st_), "sync");
	int bad = 0;
	cuda_ok(cudaMemcpy(&bad, bad_d_.p, sizeof(int), cudaMemcpyDeviceToHost), "d2h");
	if (bad) throw Error(E3D_ERR_NONFINITE, "non-finite residual norm");
}

// ---------------------------------------------------------------- state transfer
namespace {
template <class T>
void d2h_rows(const T* dev, int ld, int rows, int begin, int count, std::vector<double>& out, size_t out_off,
              int out_ld, cudaStream_t st) {
	std::vector<T> tmp((size_t)count);
	for (int q = 0; q < rows; q++) {
		if (count == 0) continue;
		cuda_ok(cudaMemcpyAsync(tmp.data(), dev + (size_t)q * ld + begin, count * sizeof(T), cudaMemcpyDeviceToHost, st),
		        "d2h");
		cuda_ok(cudaStreamSynchronize(st), "sync");
		for (int i = 0; i < count; i++) out[out_off + (size_t)q * out_ld + i] = (double)tmp[i];
	}
}
// Packed five-variable arrays (kernels.cuh ld5/st5): [n] x (rho,u,v,w) then [n] p.
template <class T>
void d2h_packed(const T* dev, int n, int begin, int count, std::vector<double>& out, size_t out_off, int out_ld,
                cudaStream_t st) {
	if (count == 0) return;
	std::vector<T> v4(4 * (size_t)count), p((size_t)count);
	cuda_ok(cudaMemcpyAsync(v4.data(), dev + 4 * (size_t)begin, 4 * (size_t)count * sizeof(T), cudaMemcpyDeviceToHost,
	                        st),
	        "d2h");
	cuda_ok(cudaMemcpyAsync(p.data(), dev + 4 * (size_t)n + begin, count * sizeof(T), cudaMemcpyDeviceToHost, st), "d2h");
	cuda_ok(cudaStreamSynchronize(st), "sync");
	for (int i = 0; i < count; i++) {
		for (int q = 0; q < 4; q++) out[out_off + (size_t)q * out_ld + i] = (double)v4[4 * (size_t)i + q];
		out[out_off + 4 * (size_t)out_ld + i] = (double)p[i];
	}
}
template <class T>
void h2d_packed(T* dev, int n, int begin, int count, const std::vector<double>& in, size_t in_off, int in_ld,
                cudaStream_t st) {
	if (count == 0) return;
	std::vector<T> v4(4 * (size_t)count), p((size_t)count);
	for (int i = 0; i < count; i++) {
		for (int q = 0; q < 4; q++) v4[4 * (size_t)i + q] = (T)in[in_off + (size_t)q * in_ld + i];
		p[i] = (T)in[in_off + 4 * (size_t)in_ld + i];
	}
	cuda_ok(cudaMemcpyAsync(dev + 4 * (size_t)begin, v4.data(), 4 * (size_t)count * sizeof(T), cudaMemcpyHostToDevice,
	                        st),
	        "h2d");
	cuda_ok(cudaMemcpyAsync(dev + 4 * (size_t)n + begin, p.data(), count * sizeof(T), cudaMemcpyHostToDevice, st), "h2d");
	cuda_ok(cudaStreamSynchronize(st), "sync");
}
template <class T>
void h2d_rows(T* dev, int ld, int rows, int begin, int count, const std::vector<double>& in, size_t in_off, int in_ld,
              cudaStream_t st) {
	std::vector<T> tmp((size_t)count);
	for (int q = 0; q < rows; q++) {
		if (count == 0) continue;
		for (int i = 0; i < count; i++) tmp[i] = (T)in[in_off + (size_t)q * in_ld + i];
		cuda_ok(cudaMemcpyAsync(dev + (size_t)q * ld + begin, tmp.data(), count * sizeof(T), cudaMemcpyHostToDevice, st),
		        "h2d");
		cuda_ok(cudaStreamSynchronize(st), "sync");
	}
}
}  // namespace

// Names and layouts match the reference's arrays for block `block`:
//   prim [5][n_all], limiter [5][n_all], grad [5][n_all][3],
//   conv_res/diss_res/w0 [5][n_real], dt/spectral_radius [n_real]
// Real cells of block b sit on the device in the order pos_[b]; these move
// the first nr entries of each of `rows` rows of length ld between device
// order and the block's local (file) order.
void Engine::to_local(int b, std::vector<double>& a, int rows, int ld) const {
	const std::vector<int>& pos = pos_[b];
	std::vector<double> t(pos.size());
	for (int q = 0; q < rows; q++) {
		double* r = a.data() + (size_t)q * ld;
		for (size_t c = 0; c < pos.size(); c++) t[c] = r[pos[c]];
		std::copy(t.begin(), t.end(), r);
	}
}
void Engine::to_device(int b, std::vector<double>& a, int rows, int ld) const {
	const std::vector<int>& pos = pos_[b];
	std::vector<double> t(pos.size());
	for (int q = 0; q < rows; q++) {
		double* r = a.data() + (size_t)q * ld;
		for (size_t c = 0; c < pos.size(); c++) t[pos[c]] = r[c];
		std::copy(t.begin(), t.end(), r);
	}
}

void Engine::get(const std::string& name, int b, std::vector<double>& out) {
	if (b < 0 || b >= nb_) throw Error(E3D_ERR_ARG, "block index out of range");
	cuda_ok(cudaStreamSynchronize(st_), "sync");
	const int nr = n_real_b_[b], na = n_all_b_[b], ng = na - nr, r0 = roff_[b], g0 = NR_ + goff_[b];
	const bool f64 = opt_.precision == PREC_FP64;
	auto rows_all = [&](int rows, auto* dev) {
		out.assign((size_t)rows * na, 0.0);
		d2h_rows(dev, NA_, rows, r0, nr, out, 0, na, st_);
		d2h_rows(dev, NA_, rows, g0, ng, out, nr, na, st_);
		to_local(b, out, rows, na);
	};
	auto rows_real = [&](int rows, auto* dev) {
		out.assign((size_t)rows * nr, 0.0);
		d2h_rows(dev, NR_, rows, r0, nr, out, 0, nr, st_);
		to_local(b, out, rows, nr);
	};
	auto packed_all = [&](auto* dev) {
		out.assign((size_t)5 * na, 0.0);
		d2h_packed(dev, NA_, r0, nr, out, 0, na, st_);
		d2h_packed(dev, NA_, g0, ng, out, nr, na, st_);
		to_local(b, out, 5, na);
	};
	if (delta_ && name != "prim" && name != "w0") throw Error(E3D_ERR_STATE, "only prim and w0 are readable in difference form");
	if (delta_) {
		rebase();  // differences folded into the base: base = full state
		cuda_ok(cudaStreamSynchronize(st_), "sync");
	}
	if (name == "prim") {
		if (delta_) packed_all(Pb64_.p);
		else if (f64) packed_all(cur_ ? f64_.P1.p : f64_.P0.p);
		else packed_all(cur_ ? f32_.P1.p : f32_.P0.p);
	} else if (name == "conv_res") {
		if (f64) rows_real(5, f64_.Rc.p);
		else rows_real(5, f32_.Rc.p);
	} else if (name == "diss_res") {
		if (f64) rows_real(5, f64_.Rd.p);
		else rows_real(5, f32_.Rd.p);
	} else if (name == "w0") {
		rows_real(5, W0_.p);
	} else if (name == "dt") {
		if (f64) rows_real(1, f64_.dt.p);
		else rows_real(1, f32_.dt.p);
	} else if (name == "spectral_radius") {
		require_fp64("spectral_radius download");
		rows_real(1, srad_.p);
	} else if (name == "limiter") {
		require_fp64("limiter download");
		rows_all(5, lim_.p);
	} else if (name == "grad") {
		require_fp64("grad download");
		std::vector<double> t;
		out.swap(t);
		rows_all(15, grad_.p);  // [var*3+dim][cell]
		std::vector<double> o((size_t)15 * na);
		for (int q = 0; q < 5; q++)
			for (int c = 0; c < na; c++)
				for (int d = 0; d < 3; d++) o[((size_t)q * na + c) * 3 + d] = out[(size_t)(q * 3 + d) * na + c];
		out.swap(o);
	} else {
		throw Error(E3D_ERR_ARG, "unknown state array '" + name + "'");
	}
}

void Engine::set(const std::string& name, int b, const std::vector<double>& in_local) {
	require_not_delta("set");
	if (b < 0 || b >= nb_) throw Error(E3D_ERR_ARG, "block index out of range");
	cuda_ok(cudaStreamSynchronize(st_), "sync");
	const int nr = n_real_b_[b], na = n_all_b_[b], ng = na - nr, r0 = roff_[b], g0 = NR_ + goff_[b];
	const bool f64 = opt_.precision == PREC_FP64;
	std::vector<double> in(in_local);  // real cells moved to device order below
	auto put_all = [&](int rows, auto* dev) {
		if (in.size() != (size_t)rows * na) throw Error(E3D_ERR_ARG, name + ": wrong length");
		to_device(b, in, rows, na);
		h2d_rows(dev, NA_, rows, r0, nr, in, 0, na, st_);
		h2d_rows(dev, NA_, rows, g0, ng, in, nr, na, st_);
		in = in_local;
	};
	auto put_real = [&](int rows, auto* dev) {
		if (in.size() != (size_t)rows * nr) throw Error(E3D_ERR_ARG, name + ": wrong length");
		to_device(b, in, rows, nr);
		h2d_rows(dev, NR_, rows, r0, nr, in, 0, nr, st_);
		in = in_local;
	};
	auto put_packed = [&](auto* dev) {
		if (in.size() != (size_t)5 * na) throw Error(E3D_ERR_ARG, name + ": wrong length");
		to_device(b, in, 5, na);
		h2d_packed(dev, NA_, r0, nr, in, 0, na, st_);
		h2d_packed(dev, NA_, g0, ng, in, nr, na, st_);
		in = in_local;
	};
	if (name == "prim") {
		// both ping-pong buffers, so ghost cells that no stage rewrites stay consistent
		if (f64) {
			put_packed(f64_.P0.p);
			put_packed(f64_.P1.p);
		} else {
			put_packed(f32_.P0.p);
			put_packed(f32_.P1.p);
		}
	} else if (name == "conv_res") {
		if (f64) put_real(5, f64_.Rc.p);
		else put_real(5, f32_.Rc.p);
	} else if (name == "diss_res") {
		if (f64) put_real(5, f64_.Rd.p);
		else put_real(5, f32_.Rd.p);
	} else if (name == "w0") {
		put_real(5, W0_.p);
	} else if (name == "dt") {
		if (f64) put_real(1, f64_.dt.p);
		else put_real(1, f32_.dt.p);
	} else if (name == "limiter") {
		require_fp64("limiter upload");
		put_all(5, lim_.p);
	} else if (name == "grad") {
		require_fp64("grad upload");
		if (in.size() != (size_t)15 * na) throw Error(E3D_ERR_ARG, "grad: wrong length");
		std::vector<double> t((size_t)15 * na);
		for (int q = 0; q < 5; q++)
			for (int c = 0; c < na; c++)
				for (int d = 0; d < 3; d++) t[(size_t)(q * 3 + d) * na + c] = in[((size_t)q * na + c) * 3 + d];
		to_device(b, t, 15, na);
		h2d_rows(grad_.p, NA_, 15, r0, nr, t, 0, na, st_);
		h2d_rows(grad_.p, NA_, 15, g0, ng, t, nr, na, st_);
	} else {
		throw Error(E3D_ERR_ARG, "unknown or read-only state array '" + name + "'");
	}
}

// ---------------------------------------------------------------- measurement
double Engine::bytes_recon(bool first) const {
	const double b = opt_.precision == PREC_FP64 ? 8.0 : 4.0;
	const double NSR = tet4_ ? 4.0 * NR_ : (double)NS_ - NG_;
	double x = 5 * b * NA_                                  // cell states, every cell read once
	           + 4.0 * NSR + 4.0 * NG_                      // neighbour ids (+ ghost mates)
	           + 3 * b * NSR                                // LS weights or signed area vectors
	           + 3 * b * NS_                                // r-vectors, ghost slots included
	           + b * NA_                                    // volumes
	           + 4 * b * NG_ + 2.0 * NG_                    // ghost face normals, ghost flags
	           + 5 * b * NS_;                               // face states written
	if (first) x += 5 * 8.0 * (carry_ ? 0 : NR_) + b * NR_ + 4 * b * NSR;  // W0, dt written; face normals
	return x;
}
double Engine::bytes_start() const {
	const double b = opt_.precision == PREC_FP64 ? 8.0 : 4.0;
	const double NSR = tet4_ ? 4.0 * NR_ : (double)NS_ - NG_;
	return 5 * b * NR_ + 4 * b * NSR + b * NR_ + 5 * 8.0 * (carry_ ? 0 : NR_) + b * NR_;
}
double Engine::bytes_flux(bool order1, bool diss, bool last) const {
	const double b = opt_.precision == PREC_FP64 ? 8.0 : 4.0;
	const double NSR = tet4_ ? 4.0 * NR_ : (double)NS_ - NG_;
	double x = 4.0 * NSR + 4.0 * NSR       // mate and neighbour ids
	           + 4 * b * NSR               // face normal and area
	           + 5 * b * NR_               // Rd read
	           + 5 * 8.0 * NR_             // W0 read
	           + 2 * b * NR_               // dt, volume
	           + 5 * b * NA_               // new cell and ghost states written
	           + 1.0 * NG_;                // ghost kinds
	x += order1 ? 5 * b * NA_ : 5 * b * NS_;  // cell states or face states read
	if (diss) x += 5 * b * NR_;               // Rd written
	if (last) x += 5 * b * NR_ + (carry_ ? 5 * 8.0 * NR_ : 0.0);  // Rc (and carried W) written
	return x;
}

std::vector<Engine::KernelTime> Engine::time_kernels(int n) {
	require_not_delta("time_kernels");
	if (deck_.smoothing) throw Error(E3D_ERR_STATE, "per-kernel timing covers the fused path (no residual smoothing)");
	std::vector<KernelTime> out;
	if (!started_) halo();
	const int stages = (int)alpha_.size();
	std::vector<std::string> names;
	std::vector<double> bytes;
	for (int s = 0; s < stages; s++) {
		if (order_ == 2) {
			names.push_back(s == 0 ? "recon_first" : "recon");
			bytes.push_back(bytes_recon(s == 0));
		} else if (s == 0) {
			names.push_back("start");
			bytes.push_back(bytes_start());
		}
		const bool diss = beta_[s] != 0.0, last = s == stages - 1;
		names.push_back(last ? "flux_update_last" : diss ? "flux_update" : "flux_update_nodiss");
		bytes.push_back(bytes_flux(order_ == 1, diss, last));
	}
	names.push_back("reduce_halo");
	bytes.push_back(0.0);
	std::vector<double> acc(names.size(), 0.0);
	for (int it = 0; it < n; it++) {
		std::vector<cudaEvent_t> marks;
		cudaEvent_t e0;
		cuda_ok(cudaEventCreate(&e0), "event");
		cuda_ok(cudaEventRecord(e0, st_), "event");
		marks.push_back(e0);
		if (opt_.precision == PREC_FP64) iteration_body<double>(f64_, cur_, &marks);
		else iteration_body<float>(f32_, cur_, &marks);
		cur_ ^= (stages & 1);
		cuda_ok(cudaEventSynchronize(marks.back()), "event sync");
		for (size_t i = 1; i < marks.size() && i - 1 < acc.size(); i++) {
			float ms = 0.f;
			cuda_ok(cudaEventElapsedTime(&ms, marks[i - 1], marks[i]), "elapsed");
			acc[i - 1] += ms;
		}
		for (auto e : marks) cudaEventDestroy(e);
		dev_iter_ += 1;
		if (dev_iter_ >= (int)opt_.hist_capacity) collect_history(total_iter_, dev_iter_);
	}
	collect_history(total_iter_, dev_iter_);
	// merge repeated names
	for (size_t i = 0; i < names.size(); i++) {
		auto it = std::find_if(out.begin(), out.end(), [&](const KernelTime& k) { return k.name == names[i]; });
		if (it == out.end()) out.push_back({names[i], n, acc[i], bytes[i]});
		else {
			it->launches += n;
			it->total_ms += acc[i];
		}
	}
	return out;
}

}  // namespace e3d

// ---------------------------------------------------------------- batches
namespace e3d {

namespace {
// autotuning results per problem-size bucket (total cells rounded to a power
// of two) and strategy; kept for the process and in $E3D_AUTOTUNE_CACHE if set
struct TuneKey {
	int bucket, scheme, grad, lim, order;
	bool operator<(const TuneKey& o) const {
		return std::tie(bucket, scheme, grad, lim, order) < std::tie(o.bucket, o.scheme, o.grad, o.lim, o.order);
	}
};
std::map<TuneKey, std::pair<int, int>> g_tune;  // -> (tile_mult, blocks per SM)
std::mutex g_tune_mu;

void tune_cache_load() {
	static bool loaded = false;
	if (loaded) return;
	loaded = true;
	const char* path = std::getenv("E3D_AUTOTUNE_CACHE");
	if (!path) return;
	std::ifstream in(path);
	TuneKey k;
	int tm, bps;
	while (in >> k.bucket >> k.scheme >> k.grad >> k.lim >> k.order >> tm >> bps) g_tune[k] = {tm, bps};
}
void tune_cache_store() {
	const char* path = std::getenv("E3D_AUTOTUNE_CACHE");
	if (!path) return;
	std::ofstream out(path);
	for (const auto& e : g_tune)
		out << e.first.bucket << " " << e.first.scheme << " " << e.first.grad << " " << e.first.lim << " "
		    << e.first.order << " " << e.second.first << " " << e.second.second << "\n";
}
}  // namespace

// Work list: tiles of tile_mult * 128 consecutive real cells, never straddling
// a block, for the blocks of active cases; block_work gives each block's range.
void Engine::build_work() {
	const int tile = tile_mult_ * kPersistThreads;
	std::vector<int> work;
	std::vector<int> bw(nb_ + 1, 0);
	for (int b = 0; b < nb_; b++) {
		if (case_active_[block_case_[b]])
			for (int c = roff_[b]; c < roff_[b + 1]; c += tile) {
				work.push_back(c);
				work.push_back(std::min(c + tile, roff_[b + 1]));
				work.push_back(b);
				work.push_back(0);
			}
		bw[b + 1] = (int)work.size() / 4;
	}
	n_work_ = (int)work.size() / 4;
	const size_t cap = 4 * ((size_t)NR_ / kPersistThreads + (size_t)nb_ + 1);
	if (work_d_.n < cap) work_d_.alloc(cap);
	if (wpart_d_.n < cap / 4 * 5) wpart_d_.alloc(cap / 4 * 5);
	if (!work.empty())
		cuda_ok(cudaMemcpyAsync(work_d_.p, work.data(), work.size() * sizeof(int), cudaMemcpyHostToDevice, st_), "work");
	block_work_d_.upload(bw);
	if (pgraph_) {
		cudaGraphExecDestroy(pgraph_);
		pgraph_ = nullptr;
	}
}

// One cooperative launch of `iters` outer iterations over the work list,
// through a captured CUDA graph when the capture succeeds.  Returns device ms.
double Engine::run_persistent(int iters) {
	return opt_.precision == PREC_FP32 ? run_persistent_t<float>(iters) : run_persistent_t<double>(iters);
}

template <class T>
double Engine::run_persistent_t(int iters) {
	if (n_work_ == 0 || iters <= 0) return 0.0;
	if (!tet4_) throw Error(E3D_ERR_STATE, "the persistent batch kernel covers all-tetrahedron meshes");
	if ((int)opt_.hist_capacity - dev_iter_ < iters) collect_history(total_iter_, dev_iter_);
	if ((int)opt_.hist_capacity < iters) throw Error(E3D_ERR_LIMIT, "launch longer than the history capacity");
	PersistArgs a{};
	a.n_work = n_work_;
	a.work = reinterpret_cast<const int4*>(work_d_.p);
	a.block_work = block_work_d_.p;
	a.nblocks = nb_;
	a.stages = (int)alpha_.size();
	for (int s = 0; s < a.stages; s++) {
		a.alpha[s] = alpha_[s];
		a.beta[s] = beta_[s];
	}
	a.carry = carry_;
	a.iters = iters;
	a.start_parity = cur_;
	a.tile_mult = tile_mult_;
	a.wpart = wpart_d_.p;
	a.wall_off = wall_off_.p;
	a.wall_face = wall_face_.p;
	a.n_wall = (int)wall_face_.n;
	a.wall_terms = wall_terms_.p;
	a.wall_denom = wall_denom_d_.p;
	a.denom = denom_;
	a.face_lr = face_lr_.p;
	a.S = S_.p;
	a.fc = fc_.p;
	a.hist = hist_d_.p;
	a.stride = nb_ * 10;
	a.d_iter = iter_d_.p;
	a.hist_capacity = (int)opt_.hist_capacity;
	a.d_bad = bad_d_.p;
	a.n_halo = (int)halo_dst_.n;
	a.halo_dst = halo_dst_.p;
	a.halo_src = halo_src_.p;
	Fused<T>& fb = fused<T>();
	auto view = [&](bool flip) {
		FusedView<T> v = fb.view(flip);
		v.NR = NR_;
		v.NG = NG_;
		v.NA = NA_;
		v.NS = NS_;
		v.tet4 = tet4_;
		v.slot_ptr = slot_ptr_.p;
		v.slot_nbr = slot_nbr_.p;
		v.slot_mate = slot_mate_.p;
		v.gkind = gkind_.p;
		v.grefl = grefl_.p;
		v.W0 = W0_.p;
		v.case_free = ncases_ > 1 ? case_free_d_.p : nullptr;  // single case: Physics::free
		v.gcase = gcase_d_.p;
		if (delta_) {
			v.Pb = Pb32_.p;
			v.Pb64 = Pb64_.p;
			v.dW = dW_.p;
			v.Rb = Rb_.p;
			v.slot_face = slot_face_.p;
			v.nhat64 = nhat_.p;
		}
		return v;
	};
	a.Pb64 = delta_ ? Pb64_.p : nullptr;
	const FusedView<T> v0 = view(false), v1 = view(true);
	const int grid = tiled_ ? n_work_ : std::max(1, std::min(grid_, n_work_));
	const bool fast = std::is_same<T, double>::value && fast64_;
	auto launch = [&]() {
		const bool o2 = order_ == 2;
		if constexpr (std::is_same<T, float>::value)
			if (delta_) return delta::launch_iterations(v0, v1, ph_, a, st_);
		if (fast)
			return tiled_ ? batch_fast::launch_tiled_iterations<T>(v0, v1, ph_, a, grad_kind_, lim_kind_, scheme_, o2, st_)
			              : batch_fast::launch_persistent<T>(v0, v1, ph_, a, grad_kind_, lim_kind_, scheme_, o2, grid, st_);
		return tiled_ ? batch::launch_tiled_iterations<T>(v0, v1, ph_, a, grad_kind_, lim_kind_, scheme_, o2, st_)
		              : batch::launch_persistent<T>(v0, v1, ph_, a, grad_kind_, lim_kind_, scheme_, o2, grid, st_);
	};
	cudaEvent_t e0, e1;
	cuda_ok(cudaEventCreate(&e0), "event");
	cuda_ok(cudaEventCreate(&e1), "event");
	cuda_ok(cudaEventRecord(e0, st_), "event");
	bool launched = false;
	if (opt_.use_graph) {
		if (pgraph_ && (pgraph_iters_ != iters || pgraph_parity_ != cur_ || pgraph_grid_ != grid ||
		                pgraph_tiled_ != tiled_)) {
			cudaGraphExecDestroy(pgraph_);
			pgraph_ = nullptr;
		}
		if (!pgraph_) {
			cudaGraph_t g;
			if (cudaStreamBeginCapture(st_, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
				const cudaError_t le = launch();
				const cudaError_t ce = cudaStreamEndCapture(st_, &g);
				if (le == cudaSuccess && ce == cudaSuccess) {
					if (cudaGraphInstantiate(&pgraph_, g, 0) != cudaSuccess) pgraph_ = nullptr;
					cudaGraphDestroy(g);
				} else if (ce == cudaSuccess) {
					cudaGraphDestroy(g);
				}
				cudaGetLastError();
			}
			pgraph_iters_ = iters;
			pgraph_parity_ = cur_;
			pgraph_grid_ = grid;
			pgraph_tiled_ = tiled_;
		}
		if (pgraph_) {
			cuda_ok(cudaGraphLaunch(pgraph_, st_), "graph launch");
			launched = true;
			tuning_.graph = true;
		}
	}
	if (!launched) cuda_ok(launch(), tiled_ ? "tiled launch" : "cooperative launch");
	cuda_ok(cudaEventRecord(e1, st_), "event");
	cuda_ok(cudaEventSynchronize(e1), "event sync");
	float ms = 0.f;
	cuda_ok(cudaEventElapsedTime(&ms, e0, e1), "elapsed");
	cudaEventDestroy(e0);
	cudaEventDestroy(e1);
	if (alpha_.size() & 1) cur_ ^= (iters & 1);
	dev_iter_ += iters;
	started_ = true;
	return (double)ms;
}

template double Engine::run_persistent_t<float>(int);
template double Engine::run_persistent_t<double>(int);

// Saves (save=true) or restores the state an iteration changes: both primitive
// buffers, the FP64 W0 / carried state and the device iteration counter.
void Engine::snapshot(bool save) {
	const size_t ep = opt_.precision == PREC_FP32 ? sizeof(float) : sizeof(double);
	const size_t np = (opt_.precision == PREC_FP32 ? f32_.P0.n : f64_.P0.n) * ep;
	const size_t nw = W0_.n * sizeof(double);
	if (snap_.n < 2 * np + nw + 16) snap_.alloc(2 * np + nw + 16);
	void* p0 = opt_.precision == PREC_FP32 ? (void*)f32_.P0.p : (void*)f64_.P0.p;
	void* p1 = opt_.precision == PREC_FP32 ? (void*)f32_.P1.p : (void*)f64_.P1.p;
	unsigned char* b = snap_.p;
	struct Part {
		void* dev;
		unsigned char* bak;
		size_t n;
	} parts[4] = {{p0, b, np}, {p1, b + np, np}, {W0_.p, b + 2 * np, nw}, {iter_d_.p, b + 2 * np + nw, sizeof(int)}};
	for (const Part& q : parts)
		if (q.n)
			cuda_ok(cudaMemcpyAsync(save ? (void*)q.bak : q.dev, save ? q.dev : (void*)q.bak, q.n,
			                        cudaMemcpyDeviceToDevice, st_),
			        "snapshot");
	// a trial that met a non-finite state leaves no flag behind: the restored state is the one before
	if (!save) cuda_ok(cudaMemsetAsync(bad_d_.p, 0, sizeof(int), st_), "memset");
}

// Picks the tile size (cells per work item) and the grid (resident blocks per
// SM) by timing short launches on the live state, which is saved before and
// restored after, so tuning never changes the solution; the choice is cached
// per problem-size bucket (and in $E3D_AUTOTUNE_CACHE when set).
void Engine::autotune(int iters) {
	std::lock_guard<std::mutex> lk(g_tune_mu);
	tune_cache_load();
	int dev = 0, sms = 0;
	cudaGetDevice(&dev);
	cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
	const bool o2 = order_ == 2;
	const int maxb = opt_.precision == PREC_FP32 ? batch::persistent_blocks_per_sm<float>(grad_kind_, lim_kind_, scheme_, o2)
	                 : fast64_ ? batch_fast::persistent_blocks_per_sm<double>(grad_kind_, lim_kind_, scheme_, o2)
	                           : batch::persistent_blocks_per_sm<double>(grad_kind_, lim_kind_, scheme_, o2);
	if (maxb <= 0) throw Error(E3D_ERR_CUDA, "persistent kernel cannot be resident");
	int bucket = 0;
	while ((1LL << bucket) < (long long)NR_) bucket++;
	const TuneKey key{bucket, scheme_, grad_kind_, lim_kind_, order_ + 4 * (int)opt_.precision + 8 * (int)fast64_};
	// E3D_BATCH_FORM=persistent or per-pass restricts the search (and bypasses the cache)
	const char* form_env = std::getenv("E3D_BATCH_FORM");
	const std::string form = form_env ? form_env : "";
	const bool only_tiled = form == "per-pass", only_persistent = form == "persistent";
	auto it = (only_tiled || only_persistent) ? g_tune.end() : g_tune.find(key);
	if (it != g_tune.end()) {  // blocks per SM 0: the tiled per-pass form
		tile_mult_ = it->second.first;
		tiled_ = it->second.second == 0;
		grid_ = tiled_ ? sms : std::min(maxb, it->second.second) * sms;
		build_work();
		tuning_.tile_cells = tile_mult_ * kPersistThreads;
		tuning_.grid = tiled_ ? 0 : grid_;
		tuning_.tiled = tiled_;
		tuning_.from_cache = true;
		return;
	}
	if ((int)opt_.hist_capacity - dev_iter_ < iters + 1) collect_history(total_iter_, dev_iter_);
	const int dev_iter0 = dev_iter_, cur0 = cur_;
	snapshot(true);
	double best = 1e300;
	int best_tm = 1, best_b = maxb;
	for (int tm : {1, 2, 4}) {
		tile_mult_ = tm;
		build_work();
		// b = 0: the tiled per-pass form (one 128-cell tile per block); b > 0: the persistent kernel
		// with b blocks per SM
		for (int b = maxb; b >= (tm == 1 ? 0 : 1); b = b > 2 ? b - 2 : b - 1) {
			if ((only_tiled && b > 0) || (only_persistent && b == 0)) continue;
			tiled_ = b == 0;
			grid_ = tiled_ ? sms : b * sms;
			run_persistent(1);  // warm (and capture)
			const double ms = run_persistent(iters) / iters;
			if (ms < best) {
				best = ms;
				best_tm = tm;
				best_b = b;
			}
			snapshot(false);
			dev_iter_ = dev_iter0;
			cur_ = cur0;
		}
	}
	tile_mult_ = best_tm;
	tiled_ = best_b == 0;
	grid_ = tiled_ ? sms : best_b * sms;
	build_work();
	if (!only_tiled && !only_persistent) {
		g_tune[key] = {best_tm, best_b};
		tune_cache_store();
	}
	tuning_.tile_cells = best_tm * kPersistThreads;
	tuning_.grid = tiled_ ? 0 : grid_;
	tuning_.tiled = tiled_;
	tuning_.ms_per_iter = best;
	tuning_.from_cache = false;
}

double Engine::solve_batch(int max_iter, double criterion, int iters_per_launch, int stall_window,
                           std::vector<int>& iters_done) {
	if (shard_) throw Error(E3D_ERR_STATE, "batch solves run on a whole case, not on a shard");
	if (iters_per_launch < 1) iters_per_launch = 1;
	if (!started_) halo();
	collect_history(total_iter_, dev_iter_);
	struct Tolerate {
		bool& flag;
		explicit Tolerate(bool& f) : flag(f) { flag = true; }
		~Tolerate() { flag = false; }
	} tolerate(tolerate_nonfinite_);
	for (int c = 0; c < ncases_; c++) case_active_[c] = case_failed_[c] ? 0 : 1;
	double ms_total = 0.0;
	auto update_active = [&]() {
		bool changed = false;
		for (int c = 0; c < ncases_; c++) {
			if (!case_active_[c]) continue;
			const auto& h = hist_case_[c];
			bool stop = (int)h.size() >= max_iter;
			for (const IterRecord& r : h) stop = stop || r.conv[0] <= criterion;
			if (!stop && stall_window > 0 && (int)h.size() >= 2 * stall_window) {
				// stalled: the last window brought no new minimum deeper by 0.05 decades
				const size_t split = h.size() - (size_t)stall_window;
				double before = 1e300, recent = 1e300;
				for (size_t i = 0; i < split; i++) before = std::min(before, h[i].conv[0]);
				for (size_t i = split; i < h.size(); i++) recent = std::min(recent, h[i].conv[0]);
				stop = recent > before - 0.05;
			}
			if (stop) {
				case_active_[c] = 0;
				changed = true;
			}
		}
		return changed;
	};
	if (grid_ == 0) {
		cudaEvent_t e0, e1;
		cuda_ok(cudaEventCreate(&e0), "event");
		cuda_ok(cudaEventCreate(&e1), "event");
		cuda_ok(cudaEventRecord(e0, st_), "event");
		autotune(3);
		cuda_ok(cudaEventRecord(e1, st_), "event");
		cuda_ok(cudaEventSynchronize(e1), "event sync");
		float ms = 0.f;
		cudaEventElapsedTime(&ms, e0, e1);
		ms_total += ms;
		cudaEventDestroy(e0);
		cudaEventDestroy(e1);
		update_active();
	}
	build_work();
	while (true) {
		int room = max_iter;
		bool any = false;
		for (int c = 0; c < ncases_; c++)
			if (case_active_[c]) {
				any = true;
				room = std::min(room, max_iter - (int)hist_case_[c].size());
			}
		if (!any || room <= 0) break;
		if (delta_) rebase();  // device work on the stream, counted in the launch's time below
		ms_total += run_persistent(std::min(iters_per_launch, room));
		const auto n_failed = [&]() { return std::count(case_failed_.begin(), case_failed_.end(), 1); };
		const auto failed_before = n_failed();
		collect_history(total_iter_, dev_iter_);
		// a case dropped for a non-finite residual leaves the work list too, else its
		// tiles run on and raise the flag again with no active case to claim it
		const bool dropped = n_failed() != failed_before;
		if (update_active() || dropped) build_work();
	}
	iters_done.assign(ncases_, 0);
	for (int c = 0; c < ncases_; c++) {
		if (case_failed_[c]) {
			iters_done[c] = -1;
			continue;
		}
		const auto& h = hist_case_[c];
		int n = (int)h.size();
		for (int i = 0; i < (int)h.size(); i++)
			if (h[i].conv[0] <= criterion) {
				n = i + 1;
				break;
			}
		iters_done[c] = n;
	}
	for (int c = 0; c < ncases_; c++) case_active_[c] = case_failed_[c] ? 0 : 1;
	return ms_total;
}

// ---------------------------------------------------------------- warm start / precision
void Engine::cell_features(float* dev_out) {
	launch_cell_features(NR_, nb_, roff_d_.p, block_case_d_.p, cen_d_.p, case_wall_off_d_.p, wall_face_.p, fc_.p,
	                     case_ma_d_.p, dev_out, st_);
	check("cell_features");
}

void Engine::conservative_rows(float* dev_out) {
	require_not_delta("conservative_rows");
	if (opt_.precision == PREC_FP32)
		launch_prims_to_conservative<float>(NR_, NA_, cur_ ? f32_.P1.p : f32_.P0.p, ph_.gamma, dev_out, st_);
	else
		launch_prims_to_conservative<double>(NR_, NA_, cur_ ? f64_.P1.p : f64_.P0.p, ph_.gamma, dev_out, st_);
	check("conservative_rows");
}

int Engine::apply_conservative(const float* dev_w, int ld) {
	require_not_delta("apply_conservative");
	if (ld < 5) throw Error(E3D_ERR_ARG, "conservative rows need at least 5 columns");
	cuda_ok(cudaMemsetAsync(fallback_d_.p, 0, sizeof(int), st_), "memset");
	if (opt_.precision == PREC_FP32)
		launch_apply_conservative<float>(NR_, NA_, nb_, roff_d_.p, block_case_d_.p, dev_w, ld, case_free_d_.p,
		                                 ph_.gamma, f32_.P0.p, f32_.P1.p, carry_ ? W0_.p : nullptr, fallback_d_.p,
		                                 st_);
	else
		launch_apply_conservative<double>(NR_, NA_, nb_, roff_d_.p, block_case_d_.p, dev_w, ld, case_free_d_.p,
		                                  ph_.gamma, f64_.P0.p, f64_.P1.p, carry_ ? W0_.p : nullptr, fallback_d_.p,
		                                  st_);
	check("apply_conservative");
	int n = 0;
	cuda_ok(cudaMemcpyAsync(&n, fallback_d_.p, sizeof(int), cudaMemcpyDeviceToHost, st_), "fallback count");
	cuda_ok(cudaStreamSynchronize(st_), "sync");
	return n;
}

void Engine::set_fp64_contracted(bool on) {
	if (opt_.precision != PREC_FP64) throw Error(E3D_ERR_STATE, "contracted FP64 batch kernels need an FP64 solver");
	if (fast64_ == on) return;
	fast64_ = on;
	if (pgraph_) {
		cudaGraphExecDestroy(pgraph_);
		pgraph_ = nullptr;
	}
	grid_ = 0;
	tuning_ = Tuning{};
}

void Engine::widen_to_fp64() {
	if (opt_.precision == PREC_FP64) return;
	if (delta_) leave_delta();
	cuda_ok(cudaStreamSynchronize(st_), "sync");
	const bool need_gg = order_ == 2 && grad_kind_ == GRAD_GREEN_GAUSS;
	const bool need_ls = order_ == 2 && grad_kind_ == GRAD_LEAST_SQUARES;
	f64_.sgeo.alloc(4 * (size_t)NS_);
	f64_.srv.alloc(3 * (size_t)NS_);
	if (need_gg) f64_.sS.alloc(3 * (size_t)NS_);
	launch_slot_geometry64(NS_, slot_face_.p, slot_mate_.p, S_.p, nhat_.p, area_.p, rl_.p, rr_.p, f64_.sgeo.p,
	                       need_gg ? f64_.sS.p : nullptr, f64_.srv.p, st_);
	if (need_ls) {
		f64_.lsw.alloc(lsw64_.n);
		cuda_ok(cudaMemcpyAsync(f64_.lsw.p, lsw64_.p, lsw64_.n * sizeof(double), cudaMemcpyDeviceToDevice, st_), "lsw");
	}
	f64_.vol.alloc(vol64_.n);
	cuda_ok(cudaMemcpyAsync(f64_.vol.p, vol64_.p, vol64_.n * sizeof(double), cudaMemcpyDeviceToDevice, st_), "vol");
	f64_.P0.alloc(5 * (size_t)NA_);
	f64_.P1.alloc(5 * (size_t)NA_);
	launch_widen_state(NA_, NR_, cur_ ? f32_.P1.p : f32_.P0.p, carry_ ? W0_.p : nullptr, ph_.gm1, f64_.P0.p,
	                   f64_.P1.p, st_);
	check("widen");
	f64_.Rc.alloc(5 * (size_t)NR_);
	f64_.Rd.alloc(5 * (size_t)NR_);
	f64_.dt.alloc(NR_);
	cuda_ok(cudaMemsetAsync(f64_.Rc.p, 0, f64_.Rc.n * sizeof(double), st_), "memset");
	cuda_ok(cudaMemsetAsync(f64_.Rd.p, 0, f64_.Rd.n * sizeof(double), st_), "memset");
	cuda_ok(cudaMemsetAsync(f64_.dt.p, 0, f64_.dt.n * sizeof(double), st_), "memset");
	f64_.FS.alloc(order_ == 2 ? 5 * (size_t)NS_ : 0);
	srad_.alloc(NR_);
	grad_.alloc(15 * (size_t)NA_);
	lim_.alloc(5 * (size_t)NA_);
	cuda_ok(cudaMemsetAsync(srad_.p, 0, srad_.n * sizeof(double), st_), "memset");
	cuda_ok(cudaMemsetAsync(grad_.p, 0, grad_.n * sizeof(double), st_), "memset");
	cuda_ok(cudaMemsetAsync(lim_.p, 0, lim_.n * sizeof(double), st_), "memset");
	cuda_ok(cudaStreamSynchronize(st_), "sync");
	for (auto* b : {&f32_.P0, &f32_.P1, &f32_.FS, &f32_.Rc, &f32_.Rd, &f32_.dt, &f32_.sgeo, &f32_.sS, &f32_.srv,
	                &f32_.lsw, &f32_.vol})
		b->free();
	cur_ = 0;
	opt_.precision = PREC_FP64;
	for (auto& g : graph_)
		if (g) {
			cudaGraphExecDestroy(g);
			g = nullptr;
		}
	if (pgraph_) {
		cudaGraphExecDestroy(pgraph_);
		pgraph_ = nullptr;
	}
	grid_ = 0;
	tuning_ = Tuning{};
	snap_.free();
	count_device_bytes();
}

// ---------------------------------------------------------------- difference form
void Engine::require_not_delta(const char* what) const {
	if (delta_)
		throw Error(E3D_ERR_STATE, std::string(what) + ": the solver runs batch solves in difference form");
}

FusedView<float> Engine::delta_view(bool flip) const {
	FusedView<float> v = f32_.view(flip);
	v.NR = NR_;
	v.NG = NG_;
	v.NA = NA_;
	v.NS = NS_;
	v.tet4 = tet4_;
	v.slot_ptr = slot_ptr_.p;
	v.slot_nbr = slot_nbr_.p;
	v.slot_mate = slot_mate_.p;
	v.gkind = gkind_.p;
	v.grefl = grefl_.p;
	v.W0 = W0_.p;
	v.case_free = ncases_ > 1 ? case_free_d_.p : nullptr;
	v.gcase = gcase_d_.p;
	v.Pb = Pb32_.p;
	v.Pb64 = Pb64_.p;
	v.dW = dW_.p;
	v.Rb = Rb_.p;
	v.slot_face = slot_face_.p;
	v.nhat64 = nhat_.p;
	return v;
}

// W_b <- W_b + dW, base primitives and ghosts from it, base residual in FP64,
// differences cleared (both primitive buffers)
void Engine::rebase() {
	delta::launch_rebase(delta_view(false), ph_, W0_.p, area_.p, (int)halo_dst_.n, halo_dst_.p, halo_src_.p, f32_.P0.p,
	                     f32_.P1.p, st_);
	check("rebase");
}

void Engine::enter_delta() {
	if (delta_) return;
	if (opt_.precision != PREC_FP32) throw Error(E3D_ERR_STATE, "the difference form starts from an FP32 solver");
	if (order_ != 1 || scheme_ != FLUX_AUSM)
		throw Error(E3D_ERR_ARG, "the difference form covers first-order AUSM");
	if (!tet4_) throw Error(E3D_ERR_ARG, "the difference form covers all-tetrahedron meshes");
	if (!carry_) throw Error(E3D_ERR_STATE, "the difference form needs the carried FP64 state");
	if (shard_) throw Error(E3D_ERR_STATE, "the difference form runs on a whole case, not on a shard");
	cuda_ok(cudaStreamSynchronize(st_), "sync");
	Pb32_.alloc(5 * (size_t)NA_);
	Pb64_.alloc(5 * (size_t)NA_);
	dW_.alloc(5 * (size_t)NR_);
	Rb_.alloc(5 * (size_t)NR_);
	// every cell's base from the current state (real cells from the carried W,
	// others from the FP32 primitives: ghosts that no condition or halo rewrites)
	launch_widen_state(NA_, NR_, cur_ ? f32_.P1.p : f32_.P0.p, W0_.p, ph_.gm1, Pb64_.p, nullptr, st_);
	launch_narrow_state(NA_, Pb64_.p, Pb32_.p, st_);
	cuda_ok(cudaMemsetAsync(dW_.p, 0, dW_.n * sizeof(float), st_), "memset");
	cuda_ok(cudaMemsetAsync(f32_.P0.p, 0, f32_.P0.n * sizeof(float), st_), "memset");
	cuda_ok(cudaMemsetAsync(f32_.P1.p, 0, f32_.P1.n * sizeof(float), st_), "memset");
	check("enter difference form");
	delta_ = true;
	rebase();
	cuda_ok(cudaStreamSynchronize(st_), "sync");
	if (pgraph_) {
		cudaGraphExecDestroy(pgraph_);
		pgraph_ = nullptr;
	}
	for (auto& g : graph_)
		if (g) {
			cudaGraphExecDestroy(g);
			g = nullptr;
		}
	// one form: tiles of 128 cells, per-pass launches in a graph (no autotuning)
	tiled_ = true;
	tile_mult_ = 1;
	grid_ = 1;
	tuning_ = Tuning{};
	tuning_.tile_cells = kPersistThreads;
	tuning_.tiled = true;
	snap_.free();
	count_device_bytes();
}

// back to the plain FP32 form: fold the differences into the base and write the
// base primitives (FP32) into both buffers; W0_ holds the full FP64 state
void Engine::leave_delta() {
	rebase();
	cuda_ok(cudaMemcpyAsync(f32_.P0.p, Pb32_.p, Pb32_.n * sizeof(float), cudaMemcpyDeviceToDevice, st_), "d2d");
	cuda_ok(cudaMemcpyAsync(f32_.P1.p, Pb32_.p, Pb32_.n * sizeof(float), cudaMemcpyDeviceToDevice, st_), "d2d");
	cuda_ok(cudaStreamSynchronize(st_), "sync");
	for (auto* b : {&Pb32_, &dW_, &Rb_}) b->free();
	Pb64_.free();
	delta_ = false;
	if (pgraph_) {
		cudaGraphExecDestroy(pgraph_);
		pgraph_ = nullptr;
	}
	grid_ = 0;
	tuning_ = Tuning{};
	count_device_bytes();
}

}  // namespace e3d
