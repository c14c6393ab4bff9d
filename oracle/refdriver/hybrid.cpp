// The reference program's outer loop with the B200 strategies plugged in
// (test infrastructure: proves the C++ adapters of include/e3d_reference_adapters.hpp
// are a drop-in for the reference's strategy objects).
//
//   e3d_hybrid DECK [--iters N] [--history FILE]
//
// Setup, post-processing (norms, Cl/Cd, convergence test, Convergence.dat) and
// the host block arrays are the reference's own objects (main.cpp:61-87,
// Solver.cpp:76-97).  Fluxes, gradients, limiters, time step, W0, update,
// boundary conditions and halo run on the GPU through the adapters; each block
// is copied back to the reference's host arrays before the reference's
// PostProcessing::computeFlowData reads it.
#include <climits>
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <limits>
#include <string>
#include <vector>

#include "Block.h"
#include "BlockCommunicator.h"
#include "CompleteMesh.h"
#include "Initializer.h"
#include "Interface.h"
#include "PostProcessing.h"
#include "Solver.h"
#include "e3d_reference_adapters.hpp"

using namespace e3d_adapters;

int main(int argc, char** argv) {
	if (argc < 2) {
		std::cerr << "usage: e3d_hybrid DECK [--iters N] [--history FILE]" << std::endl;
		return 2;
	}
	int iters = -1;
	std::string history;
	for (int i = 2; i < argc; i++) {
		std::string a = argv[i];
		if (a == "--iters" && i + 1 < argc) iters = std::atoi(argv[++i]);
		else if (a == "--history" && i + 1 < argc) history = argv[++i];
		else {
			std::cerr << "unknown option " << a << std::endl;
			return 2;
		}
	}
	std::streambuf* saved = std::cout.rdbuf(nullptr);
	Interface* interface = new Interface(argv[1], false);
	Initializer* initializer = new Initializer();
	BlockCommunicator* comm = new BlockCommunicator(interface->n_blocks_interface_);
	int n_mine;
	int* mine;
	comm->getMyBlocks(n_mine, mine);
	CompleteMesh* mesh = new CompleteMesh(interface->n_blocks_interface_, n_mine, mine,
	                                      interface->topology_file_name_interface_);
	mesh->InitializeMyBlocks(interface, comm);
	comm->initializeBuffers();
	Solver* solver = initializer->initializeSolver(interface);
	PostProcessing* pp = solver->post_processing_;
	if (iters <= 0) iters = interface->max_iter_interface_;
	pp->max_iter_ = INT_MAX;
	pp->convergence_criterion_ = -std::numeric_limits<double>::infinity();

	// the device side of the same case
	e3d_case* ec = nullptr;
	check(e3d_case_load(argv[1], nullptr, &ec), "case_load");
	e3d_solver* es = nullptr;
	e3d_options opt;
	e3d_default_options(&opt);
	check(e3d_solver_create(ec, &opt, &es), "solver_create");

	// strategy objects selected by the reference's strings (ResidualCalculator.cpp:72-95,
	// SecondOrder.cpp:50-61) and the smoother (ResidualCalculator.cpp:90-93), RK tables of
	// RungeKutta.cpp:23-68 taken from its objects
	const double gamma = interface->gamma_interface_;
	FluxScheme* flux = interface->flux_scheme_choice_interface_ == "ausm"
	                       ? static_cast<FluxScheme*>(new GpuAusmScheme(es, gamma))
	                       : static_cast<FluxScheme*>(new GpuRoeScheme(es, gamma));
	Gradient* grad = nullptr;
	Limiter* lim = nullptr;
	const bool second = interface->interpolation_choice_interface_ == 2;
	if (second) {
		if (interface->gradient_choice_interface_ == "leastsquares") grad = new GpuLeastSquares(es);
		else grad = new GpuGreenGauss(es);
		if (interface->limiter_choice_interface_ == "venkatakrishnan") lim = new GpuVenkatakrishnan(es, interface->k_interface_);
		else lim = new GpuBarthJespersen(es, interface->omega_interface_);
	}
	ResidualSmoother* smoother = nullptr;
	if (interface->residual_smoother_choice_interface_) smoother = new GpuCentralIrsSmoother(es);
	GpuTimestep ts(es, gamma, interface->cfl_interface_);
	const std::vector<double> beta = solver->runge_kutta_->residual_calculator_->beta_rk_;
	GpuUpdater up(es, gamma, solver->runge_kutta_->updater_->alpha_rk_);
	const int stages = solver->runge_kutta_->stage_number_;

	FILE* hist = history.empty() ? nullptr : std::fopen(history.c_str(), "w");
	if (hist) std::fprintf(hist, "iter,ro_conv,cl,cd,cmx,cmy,cmz,rms_ro\n");
	comm->updateBoundaries(mesh);  // Solver.cpp:48
	halo(es);
	for (int it = 0; it < iters; it++) {
		for (int i = 0; i < mesh->n_blocks_in_process_; i++) {
			Block* b = mesh->all_blocks_[mesh->my_blocks_[i]];
			save_w0(es, b);
			ts.computeSpectralRadius(b);
			ts.computeTimestep(b);
			for (int s = 0; s < stages; s++) {
				if (second) {
					grad->computeGradients(b);
					lim->computeLimiters(b);
				}
				flux->computeFluxConv(b);
				flux->current_beta_ = beta[s];
				flux->computeFluxDiss(b);
				if (smoother) smoother->smoothResidual(b);
				up.current_stage_ = s;
				up.updateInternalBlock(b);
				up.updateBoundary(b);
			}
			sync_to_host(es, b, second);
			pp->computeFlowData(b);  // the reference's norms and forces on the GPU's results
		}
		halo(es);
		comm->updateBoundaries(mesh);
		pp->process(mesh, comm);
		if (hist)
			std::fprintf(hist, "%d,%.17g,%.17g,%.17g,%.17g,%.17g,%.17g,%.17g\n", it, pp->ro_convergence_,
			             pp->cl_geometry_mesh_, pp->cd_geometry_mesh_, pp->cmx_geometry_mesh_, pp->cmy_geometry_mesh_,
			             pp->cmz_geometry_mesh_, pp->ro_rms_mesh_);
	}
	if (hist) std::fclose(hist);
	std::cout.rdbuf(saved);
	std::printf("{\"iters\": %d}\n", iters);
	e3d_solver_free(es);
	e3d_case_free(ec);
	return 0;
}
