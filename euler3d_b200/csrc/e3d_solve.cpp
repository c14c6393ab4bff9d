// e3d_solve DECK [--fp32] [--check-every N] [--no-graph]
//
// Command-line counterpart of the reference program (main.cpp:17-101) for the
// residual/update path: reads the same deck, topology and SU2 blocks, runs the
// outer iterations on the GPU until the reference stop test fires
// (PostProcessing::checkStopSolver, PostProcessing.cpp:59-83: max_iter, the
// density-convergence criterion, or a file named STOP in the working
// directory), prints the reference's per-iteration line and writes
// ./bin/Convergence.dat and ./bin/AerodynamicCoefficients.dat in the
// reference's layout (OutputTecplot.cpp:413-470).  Tecplot flow files are not
// written.
#include <sys/stat.h>

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include "../../include/e3d.h"

static int die(const char* what) {
	std::cerr << "ERROR: " << what << ": " << e3d_last_error() << std::endl;
	return 42;
}

int main(int argc, char** argv) {
	if (argc < 2) {
		std::cout << "ERROR: No input file" << std::endl;
		return 255;
	}
	e3d_options opt;
	e3d_default_options(&opt);
	int check_every = 1;
	for (int i = 2; i < argc; i++) {
		if (!std::strcmp(argv[i], "--fp32")) opt.precision = E3D_FP32;
		else if (!std::strcmp(argv[i], "--no-graph")) opt.use_graph = 0;
		else if (!std::strcmp(argv[i], "--check-every") && i + 1 < argc) {
			// each pass of the loop below must advance, or the stop test never runs
			check_every = std::atoi(argv[++i]);
			if (check_every < 1) {
				std::cerr << "--check-every needs a positive iteration count" << std::endl;
				return 2;
			}
		} else {
			std::cerr << "unknown option " << argv[i] << std::endl;
			return 2;
		}
	}
	std::cout << "Input file is : " << argv[1] << std::endl;
	e3d_case* c = nullptr;
	if (e3d_case_load(argv[1], nullptr, &c)) return die("reading the case");
	e3d_deck_info d;
	e3d_case_deck(c, &d);
	e3d_solver* s = nullptr;
	if (e3d_solver_create(c, &opt, &s)) return die("creating the solver");

	auto t0 = std::chrono::high_resolution_clock::now();
	int done = 0;
	bool stop = false;
	int printed = 0;
	std::ofstream conv;
	while (!stop) {
		const int chunk = check_every;
		if (e3d_iterate(s, chunk)) return die("iterating");
		int n = 0;
		e3d_history_length(s, &n);
		std::vector<e3d_iter_record> h((size_t)(n - printed));
		e3d_history(s, printed, n - printed, h.data());
		struct stat sb;
		const bool stop_file = stat("STOP", &sb) == 0;
		for (const auto& r : h) {
			const bool last = (r.iter + 1 == d.max_iter) || (r.conv[0] <= d.criterion) || stop_file;
			std::cout << "Iter: " << r.iter << " Convergence Ro: " << r.conv[0] << " cl: " << r.cl << " cd: " << r.cd
			          << std::endl;
			if (r.iter == 0) {
				conv.open("./bin/Convergence.dat");
				conv << "Iteration Cl Cd Cmx Cmy Cmz Density_Convergence Uu_Convergence Vv_Convergence "
				        "Ww_Convergence Pressure_Convergence \n";
			}
			if (conv.is_open())
				conv << r.iter << " " << r.cl << " " << r.cd << " " << r.cmx << " " << r.cmy << " " << r.cmz << " "
				     << r.conv[0] << " " << r.conv[1] << " " << r.conv[2] << " " << r.conv[3] << " " << r.conv[4]
				     << std::endl;
			done = r.iter + 1;
			if (last) {
				stop = true;
				if (stop_file) std::remove("STOP");
				std::ofstream ac("./bin/AerodynamicCoefficients.dat");
				ac << "Angle of attack Cl Cd Cmx Cmy Cmz\n"
				   << d.aoa_deg << " " << r.cl << " " << r.cd << " " << r.cmx << " " << r.cmy << " " << r.cmz << "\n";
				break;
			}
		}
		printed = n;
	}
	auto t1 = std::chrono::high_resolution_clock::now();
	std::cout << "Time elapsed solving: " << std::chrono::duration<double, std::milli>(t1 - t0).count() / 1000.0
	          << "s." << std::endl;
	std::cout << "Iterations: " << done << std::endl;
	e3d_solver_free(s);
	e3d_case_free(c);
	return 0;
}
