// Oracle driver around the reference CPU solver (test infrastructure only).
//
// It builds the case with the reference's own Interface / BlockCommunicator /
// CompleteMesh / Initializer objects (main.cpp:61-87) and runs the reference's
// outer iteration (Solver::solve, Solver/src/Solver.cpp:48-97) step by step with
// the reference's own strategy objects, so that arrays can be dumped between
// stages.  The arithmetic is entirely the reference's: this file only sequences
// the same calls in the same order and copies arrays out.
//
//   e3d_refdriver DECK [--iters N] [--dump-dir DIR] [--dump-init] [--dump-stages]
//                      [--dump-every K] [--history FILE] [--blocks A:B] [--warmup W] [--quiet]
//
// --warmup W runs W outer iterations before the timer starts (the reported
// iterations and rate cover the remaining --iters minus W).
// --blocks A:B owns only blocks [A,B) (the reference's per-rank block range,
// BlockCommunicator.cpp:284-294); connexions touching other blocks are then not
// exchanged.  That mode exists to time bounded samples on several host cores.
#include "Interface.h"
#include "Initializer.h"
#include "Solver.h"
#include "Timestep.h"
#include "RungeKutta.h"
#include "ResidualCalculator.h"
#include "Updater.h"
#include "PostProcessing.h"
#include "BlockCommunicator.h"
#include "CompleteMesh.h"
#include "Block.h"
#include "WallCellIds.h"
#include "FarfieldCellIds.h"
#include "SymmetryCellIds.h"
#include "ConnexionBlockCellIds.h"
#include "ConnexionCellIds.h"
#include "refdump.h"

#include <chrono>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <limits>
#include <string>
#include <vector>

namespace {

struct Options {
	std::string deck;
	int iters = -1;
	std::string dump_dir;
	bool dump_init = false;
	bool dump_stages = false;
	int dump_every = 0;
	int warmup = 0;
	std::string history;
	int block_lo = -1, block_hi = -1;
	bool quiet = false;
};

void dump_geometry(RefDump& d, Block* b) {
	const std::string p = "b" + std::to_string(b->block_id_) + ".";
	const int nr = b->n_real_cells_in_block_, na = b->n_all_cells_in_block_, nf = b->n_faces_in_block_;
	std::vector<int> counts = {nr, na, nf, b->n_real_boundaries_in_block_, b->n_all_boundaries_in_block_, b->n_wall_faces_};
	d.put(p + "counts", counts);
	std::vector<int> f2c(2 * nf), fnn(nf);
	std::vector<double> fn(3 * nf), fa(nf), fc(3 * nf), rl(3 * nf), rr(3 * nf);
	std::vector<int> fnodes;
	for (int f = 0; f < nf; f++) {
		Face* F = b->block_faces_[f];
		f2c[2 * f] = F->face_2_cells_connectivity_[0];
		f2c[2 * f + 1] = F->face_2_cells_connectivity_[1];
		fnn[f] = F->n_nodes_per_face_;
		for (int k = 0; k < F->n_nodes_per_face_; k++) fnodes.push_back(F->face_2_nodes_connectivity_[k]);
		fa[f] = F->face_area_;
		for (int k = 0; k < 3; k++) {
			fn[3 * f + k] = F->face_normals_[k];
			fc[3 * f + k] = F->face_center_[k];
			rl[3 * f + k] = F->left_cell_r_vector_[k];
			rr[3 * f + k] = F->right_cell_r_vector_[k];
		}
	}
	d.put(p + "face_cells", f2c);
	d.put(p + "face_nnodes", fnn);
	d.put(p + "face_nodes", fnodes);
	d.put(p + "face_normal", fn);
	d.put(p + "face_area", fa);
	d.put(p + "face_center", fc);
	d.put(p + "r_left", rl);
	d.put(p + "r_right", rr);
	std::vector<int> cnf(na), c2f, c2c;
	std::vector<double> vol(na), cc(3 * na), wls;
	for (int c = 0; c < na; c++) {
		Cell* C = b->block_cells_[c];
		cnf[c] = C->n_faces_per_cell_;
		vol[c] = C->cell_volume_;
		for (int k = 0; k < 3; k++) cc[3 * c + k] = C->cell_coordinates_[k];
		for (int k = 0; k < C->n_faces_per_cell_; k++) {
			c2f.push_back(C->cell_2_faces_connectivity_[k]);
			c2c.push_back(C->cell_2_cells_connectivity_[k]);
			if (c < nr)
				for (int q = 0; q < 3; q++) wls.push_back(C->cell_weights_[k][q]);
		}
	}
	d.put(p + "cell_nfaces", cnf);
	d.put(p + "cell_faces", c2f);
	d.put(p + "cell_cells", c2c);
	d.put(p + "cell_volume", vol);
	d.put(p + "cell_center", cc);
	d.put(p + "ls_weights", wls);
	// boundary markers: kind code (1 wall, 2 farfield, 3 symmetry, 4 connexion) and ghost ids
	std::vector<int> kinds, sizes, ids;
	for (int j = 0; j < b->n_all_boundaries_in_block_; j++) {
		BoundaryCellIds* bc = b->block_boundary_cell_ids_[j];
		int kind = 0;
		if (dynamic_cast<WallCellIds*>(bc)) kind = 1;
		else if (dynamic_cast<FarfieldCellIds*>(bc)) kind = 2;
		else if (dynamic_cast<SymmetryCellIds*>(bc)) kind = 3;
		else if (dynamic_cast<ConnexionBlockCellIds*>(bc)) kind = 4;
		kinds.push_back(kind);
		sizes.push_back(bc->n_cell_in_boundary_);
		for (int i = 0; i < bc->n_cell_in_boundary_; i++) ids.push_back(bc->cell_ids_in_boundary_[i]);
	}
	d.put(p + "marker_kind", kinds);
	d.put(p + "marker_size", sizes);
	d.put(p + "marker_cells", ids);
	std::vector<int> wall(b->block_wall_face_ids_, b->block_wall_face_ids_ + b->n_wall_faces_);
	d.put(p + "wall_faces", wall);
}

void dump_state(RefDump& d, Block* b) {
	const std::string p = "b" + std::to_string(b->block_id_) + ".";
	const int nr = b->n_real_cells_in_block_, na = b->n_all_cells_in_block_;
	PrimitiveVariables* pv = b->block_primitive_variables_;
	InterpolationVariables* iv = b->block_interpolation_variables_;
	auto put5 = [&](const char* name, double* a0, double* a1, double* a2, double* a3, double* a4, int n) {
		std::vector<double> v(5 * (size_t)n);
		double* a[5] = {a0, a1, a2, a3, a4};
		for (int q = 0; q < 5; q++)
			for (int c = 0; c < n; c++) v[(size_t)q * n + c] = a[q][c];
		d.put(p + name, v);
	};
	put5("prim", pv->ro_, pv->uu_, pv->vv_, pv->ww_, pv->pp_, na);
	put5("conv_res", pv->conv_res_ro_, pv->conv_res_uu_, pv->conv_res_vv_, pv->conv_res_ww_, pv->conv_res_pp_, na);
	put5("diss_res", pv->diss_res_ro_, pv->diss_res_uu_, pv->diss_res_vv_, pv->diss_res_ww_, pv->diss_res_pp_, na);
	put5("w0", pv->ro_0_, pv->ru_0_, pv->rv_0_, pv->rw_0_, pv->re_0_, na);
	put5("limiter", iv->limiter_ro_, iv->limiter_uu_, iv->limiter_vv_, iv->limiter_ww_, iv->limiter_pp_, na);
	std::vector<double> g(15 * (size_t)na);
	double** gr[5] = {iv->grad_ro_, iv->grad_uu_, iv->grad_vv_, iv->grad_ww_, iv->grad_pp_};
	for (int q = 0; q < 5; q++)
		for (int c = 0; c < na; c++)
			for (int k = 0; k < 3; k++) g[((size_t)q * na + c) * 3 + k] = gr[q][c][k];
	d.put(p + "grad", g);
	d.put(p + "dt", b->block_time_variables_->dt_, nr);
	d.put(p + "spectral_radius", b->block_time_variables_->spectral_radius_, nr);
}

void dump_all(const Options& o, const std::string& tag, CompleteMesh* mesh, PostProcessing* pp, bool geometry) {
	RefDump d(o.dump_dir + "/" + tag + ".bin");
	if (!d.ok()) {
		std::cerr << "cannot write dump " << tag << std::endl;
		std::exit(3);
	}
	for (int i = 0; i < mesh->n_blocks_in_process_; i++) {
		Block* b = mesh->all_blocks_[mesh->my_blocks_[i]];
		if (geometry) dump_geometry(d, b);
		dump_state(d, b);
	}
	if (pp) {
		int nb = mesh->n_blocks_;
		d.put("rms_blocks.ro", pp->ro_rms_blocks_, nb);
		d.put("rms_blocks.uu", pp->uu_rms_blocks_, nb);
		d.put("rms_blocks.vv", pp->vv_rms_blocks_, nb);
		d.put("rms_blocks.ww", pp->ww_rms_blocks_, nb);
		d.put("rms_blocks.pp", pp->pp_rms_blocks_, nb);
		d.put("cl_blocks", pp->cl_geometry_blocks_, nb);
		d.put("cd_blocks", pp->cd_geometry_blocks_, nb);
		double g[15] = {pp->ro_rms_mesh_, pp->uu_rms_mesh_, pp->vv_rms_mesh_, pp->ww_rms_mesh_, pp->pp_rms_mesh_,
		                pp->cl_geometry_mesh_, pp->cd_geometry_mesh_, pp->cmx_geometry_mesh_, pp->cmy_geometry_mesh_,
		                pp->cmz_geometry_mesh_, pp->ro_convergence_, pp->uu_convergence_, pp->vv_convergence_,
		                pp->ww_convergence_, pp->pp_convergence_};
		d.put("global", g, 15);
	}
}

void dump_block(const Options& o, const std::string& tag, Block* b) {
	RefDump d(o.dump_dir + "/" + tag + ".bin");
	if (!d.ok()) {
		std::cerr << "cannot write dump " << tag << std::endl;
		std::exit(3);
	}
	dump_state(d, b);
}

// Serial halo of the reference (BlockCommunicator.cpp:212-268) restricted to
// connexions whose two blocks are both owned; used only with --blocks.
void partial_halo(BlockCommunicator* comm, CompleteMesh* mesh, const std::vector<char>& owned) {
	for (int i = 0; i < comm->n_inter_block_boundaries_; i++) {
		ConnexionCellIds* bd = comm->inter_block_boundaries_[i];
		if (!owned[bd->block_origin_] || !owned[bd->block_destination_]) continue;
		Block* src = mesh->all_blocks_[bd->block_origin_];
		Block* dst = mesh->all_blocks_[bd->block_destination_];
		PrimitiveVariables* s = src->block_primitive_variables_;
		PrimitiveVariables* t = dst->block_primitive_variables_;
		for (int j = 0; j < bd->n_cell_in_boundary_; j++) {
			int a = bd->cell_ids_in_boundary_other_block_[j], c = bd->cell_ids_in_boundary_[j];
			t->ro_[c] = s->ro_[a];
			t->uu_[c] = s->uu_[a];
			t->vv_[c] = s->vv_[a];
			t->ww_[c] = s->ww_[a];
			t->pp_[c] = s->pp_[a];
		}
	}
}

}  // namespace

int main(int argc, char** argv) {
	Options o;
	if (argc < 2) {
		std::cerr << "usage: e3d_refdriver DECK [--iters N] [--dump-dir DIR] [--dump-init] [--dump-stages] "
		             "[--dump-every K] [--history FILE] [--blocks A:B] [--warmup W] [--quiet]" << std::endl;
		return 2;
	}
	o.deck = argv[1];
	for (int i = 2; i < argc; i++) {
		std::string a = argv[i];
		auto next = [&]() -> std::string {
			if (i + 1 >= argc) { std::cerr << "missing value for " << a << std::endl; std::exit(2); }
			return argv[++i];
		};
		if (a == "--iters") o.iters = std::atoi(next().c_str());
		else if (a == "--dump-dir") o.dump_dir = next();
		else if (a == "--dump-init") o.dump_init = true;
		else if (a == "--dump-stages") o.dump_stages = true;
		else if (a == "--dump-every") o.dump_every = std::atoi(next().c_str());
		else if (a == "--warmup") o.warmup = std::atoi(next().c_str());
		else if (a == "--history") o.history = next();
		else if (a == "--blocks") {
			std::string v = next();
			size_t c = v.find(':');
			o.block_lo = std::atoi(v.substr(0, c).c_str());
			o.block_hi = std::atoi(v.substr(c + 1).c_str());
		} else if (a == "--quiet") o.quiet = true;
		else { std::cerr << "unknown option " << a << std::endl; return 2; }
	}
	if ((o.dump_init || o.dump_stages || o.dump_every) && o.dump_dir.empty()) {
		std::cerr << "dumps need --dump-dir" << std::endl;
		return 2;
	}

	std::streambuf* saved = nullptr;
	if (o.quiet) saved = std::cout.rdbuf(nullptr);

	Interface* interface = new Interface(argv[1], false);
	Initializer* initializer = new Initializer();
	const int n_blocks = interface->n_blocks_interface_;
	BlockCommunicator* comm = new BlockCommunicator(n_blocks);
	int n_mine;
	int* mine;
	comm->getMyBlocks(n_mine, mine);
	std::vector<char> owned(n_blocks, 1);
	if (o.block_lo >= 0) {
		if (o.block_hi > n_blocks || o.block_lo >= o.block_hi) { std::cerr << "bad --blocks" << std::endl; return 2; }
		n_mine = o.block_hi - o.block_lo;
		mine = new int[n_mine];
		for (int i = 0; i < n_mine; i++) mine[i] = o.block_lo + i;
		for (int b = 0; b < n_blocks; b++) owned[b] = (b >= o.block_lo && b < o.block_hi);
	}
	const bool all_owned = (o.block_lo < 0);

	auto t_pre0 = std::chrono::high_resolution_clock::now();
	CompleteMesh* mesh = new CompleteMesh(n_blocks, n_mine, mine, interface->topology_file_name_interface_);
	mesh->InitializeMyBlocks(interface, comm);
	comm->initializeBuffers();
	Solver* solver = initializer->initializeSolver(interface);
	auto t_pre1 = std::chrono::high_resolution_clock::now();

	PostProcessing* pp = solver->post_processing_;
	const int iters = o.iters > 0 ? o.iters : interface->max_iter_interface_;
	// The driver decides when to stop; the reference stop test must not fire
	// (it would also write Tecplot files), so push its limits out of reach.
	pp->max_iter_ = INT_MAX;
	pp->convergence_criterion_ = -std::numeric_limits<double>::infinity();

	FILE* hist = nullptr;
	if (!o.history.empty()) {
		hist = std::fopen(o.history.c_str(), "w");
		std::fprintf(hist, "iter,ro_conv,uu_conv,vv_conv,ww_conv,pp_conv,cl,cd,cmx,cmy,cmz,rms_ro,rms_uu,rms_vv,rms_ww,rms_pp\n");
	}

	if (all_owned) comm->updateBoundaries(mesh); else partial_halo(comm, mesh, owned);  // Solver.cpp:48
	if (o.dump_init) dump_all(o, "init", mesh, nullptr, true);

	RungeKutta* rk = solver->runge_kutta_;
	auto t0 = std::chrono::high_resolution_clock::now();
	for (int it = 0; it < iters; it++) {
		if (it == o.warmup) t0 = std::chrono::high_resolution_clock::now();
		for (int i = 0; i < mesh->n_blocks_in_process_; i++) {  // Solver.cpp:83-91
			Block* b = mesh->all_blocks_[mesh->my_blocks_[i]];
			solver->saveW0(b);
			solver->timestep_->computeSpectralRadius(b);
			solver->timestep_->computeTimestep(b);
			for (int s = 0; s < rk->stage_number_; s++) {  // RungeKutta.cpp:85-92
				rk->residual_calculator_->current_stage_ = s;
				rk->residual_calculator_->computeResidual(b);
				const std::string st = "it0_b" + std::to_string(b->block_id_) + "_s" + std::to_string(s);
				if (o.dump_stages && it == 0) dump_block(o, st + "_res", b);
				rk->updater_->current_stage_ = s;
				rk->updater_->updateInternalBlock(b);
				rk->updater_->updateBoundary(b);
				if (o.dump_stages && it == 0) dump_block(o, st + "_upd", b);
			}
			pp->computeFlowData(b);
		}
		if (all_owned) comm->updateBoundaries(mesh); else partial_halo(comm, mesh, owned);  // Solver.cpp:94
		pp->process(mesh, comm);                             // Solver.cpp:96
		if (hist) {
			std::fprintf(hist, "%d,%.17g,%.17g,%.17g,%.17g,%.17g,%.17g,%.17g,%.17g,%.17g,%.17g,%.17g,%.17g,%.17g,%.17g,%.17g\n",
			             it, pp->ro_convergence_, pp->uu_convergence_, pp->vv_convergence_, pp->ww_convergence_,
			             pp->pp_convergence_, pp->cl_geometry_mesh_, pp->cd_geometry_mesh_, pp->cmx_geometry_mesh_,
			             pp->cmy_geometry_mesh_, pp->cmz_geometry_mesh_, pp->ro_rms_mesh_, pp->uu_rms_mesh_,
			             pp->vv_rms_mesh_, pp->ww_rms_mesh_, pp->pp_rms_mesh_);
		}
		if (o.dump_every > 0 && ((it + 1) % o.dump_every == 0 || it + 1 == iters))
			dump_all(o, "iter" + std::to_string(it + 1), mesh, pp, false);
	}
	auto t1 = std::chrono::high_resolution_clock::now();
	if (hist) std::fclose(hist);
	if (saved) std::cout.rdbuf(saved);

	long long cells = 0;
	for (int i = 0; i < mesh->n_blocks_in_process_; i++) cells += mesh->all_blocks_[mesh->my_blocks_[i]]->n_real_cells_in_block_;
	const double solve_s = std::chrono::duration<double>(t1 - t0).count();
	const int timed = iters > o.warmup ? iters - o.warmup : 0;
	std::printf("{\"cells\": %lld, \"iters\": %d, \"solve_s\": %.6f, \"preprocess_s\": %.6f, \"cell_iters_per_s\": %.6g}\n",
	            cells, timed, solve_s, std::chrono::duration<double>(t_pre1 - t_pre0).count(),
	            solve_s > 0 ? (double)cells * timed / solve_s : 0.0);
	return 0;
}
