// e3d_reference_adapters.hpp -- the reference's strategy interfaces backed by
// the B200 path.
//
// Header-only C++ for maintainers of the reference code: compile it inside the
// reference tree (it includes the reference's own headers FluxScheme.h,
// Gradient.h, Limiter.h, ResidualSmoother.h, Block.h, PrimitiveVariables.h, InterpolationVariables.h,
// TimeVariables.h) and link libe3d.so.  Each class derives from, or has the same
// methods as, the reference class it replaces and forwards to one entry point of
// include/e3d.h on the device-resident copy of the same block (the reference's
// block_id_ is the block index).  State stays on the device; sync_to_host()
// copies a block back into the reference's host arrays at observation points
// (post-processing, output), never per call.
#pragma once

#include <stdexcept>
#include <string>
#include <vector>

#include "Block.h"
#include "FluxScheme.h"
#include "Gradient.h"
#include "InterpolationVariables.h"
#include "Limiter.h"
#include "PrimitiveVariables.h"
#include "ResidualSmoother.h"
#include "TimeVariables.h"
#include "e3d.h"

namespace e3d_adapters {

inline void check(int rc, const char* what) {
	if (rc != E3D_OK) throw std::runtime_error(std::string(what) + ": " + e3d_last_error());
}

// FluxScheme (Solver/head/FluxScheme.h:9-23) -> RoeScheme / AusmScheme
class GpuFluxScheme : public FluxScheme {
public:
	GpuFluxScheme(e3d_solver* s, double gamma, int scheme) : s_(s), scheme_(scheme) {
		gamma_ = gamma;
		current_beta_ = 1.0;
	}
	void computeFluxConv(Block* b) override { check(e3d_flux_conv(s_, b->block_id_, scheme_), "flux_conv"); }
	void computeFluxDiss(Block* b) override {
		check(e3d_flux_diss(s_, b->block_id_, scheme_, current_beta_), "flux_diss");
	}

private:
	e3d_solver* s_;
	int scheme_;
};
class GpuRoeScheme : public GpuFluxScheme {
public:
	GpuRoeScheme(e3d_solver* s, double gamma) : GpuFluxScheme(s, gamma, E3D_FLUX_ROE) {}
};
class GpuAusmScheme : public GpuFluxScheme {
public:
	GpuAusmScheme(e3d_solver* s, double gamma) : GpuFluxScheme(s, gamma, E3D_FLUX_AUSM) {}
};

// Gradient (Solver/head/Gradient.h:8-18) -> GreenGauss / LeastSquares
class GpuGradient : public Gradient {
public:
	GpuGradient(e3d_solver* s, int kind) : s_(s), kind_(kind) {}
	void computeGradients(Block* b) override { check(e3d_gradients(s_, b->block_id_, kind_), "gradients"); }

private:
	e3d_solver* s_;
	int kind_;
};
class GpuGreenGauss : public GpuGradient {
public:
	explicit GpuGreenGauss(e3d_solver* s) : GpuGradient(s, E3D_GRAD_GREEN_GAUSS) {}
};
class GpuLeastSquares : public GpuGradient {
public:
	explicit GpuLeastSquares(e3d_solver* s) : GpuGradient(s, E3D_GRAD_LEAST_SQUARES) {}
};

// Limiter (Solver/head/Limiter.h:8-18) -> BarthJespersen(omega) / Venkatakrishnan(k)
class GpuLimiter : public Limiter {
public:
	GpuLimiter(e3d_solver* s, int kind, double omega, double k) : s_(s), kind_(kind), omega_(omega), k_(k) {}
	void computeLimiters(Block* b) override { check(e3d_limiters(s_, b->block_id_, kind_, omega_, k_), "limiters"); }

private:
	e3d_solver* s_;
	int kind_;
	double omega_, k_;
};
class GpuBarthJespersen : public GpuLimiter {
public:
	GpuBarthJespersen(e3d_solver* s, double omega) : GpuLimiter(s, E3D_LIM_BARTH_JESPERSEN, omega, 0.0) {}
};
class GpuVenkatakrishnan : public GpuLimiter {
public:
	GpuVenkatakrishnan(e3d_solver* s, double k) : GpuLimiter(s, E3D_LIM_VENKATAKRISHNAN, 0.0, k) {}
};

// ResidualSmoother (Solver/head/ResidualSmoother.h:8-18) -> CentralIrsSmoother
class GpuCentralIrsSmoother : public ResidualSmoother {
public:
	explicit GpuCentralIrsSmoother(e3d_solver* s) : s_(s) {}
	void smoothResidual(Block* b) override { check(e3d_smooth_residual(s_, b->block_id_), "smooth_residual"); }

private:
	e3d_solver* s_;
};

// Timestep (Solver/head/Timestep.h:10-27): same methods, device arrays
class GpuTimestep {
public:
	GpuTimestep(e3d_solver* s, double gamma, double cfl) : gamma_(gamma), cfl_(cfl), s_(s) {}
	void computeSpectralRadius(Block* b) { check(e3d_spectral_radius(s_, b->block_id_), "spectral_radius"); }
	void computeTimestep(Block* b) { check(e3d_timestep(s_, b->block_id_), "timestep"); }
	double gamma_, cfl_;

private:
	e3d_solver* s_;
};

// Updater (Solver/head/Updater.h:10-27): same fields and methods
class GpuUpdater {
public:
	GpuUpdater(e3d_solver* s, double gamma, std::vector<double> alpha_rk)
	    : gamma_(gamma), current_stage_(0), alpha_rk_(alpha_rk), s_(s) {}
	void updateInternalBlock(Block* b) {
		check(e3d_update_internal(s_, b->block_id_, alpha_rk_[current_stage_]), "update_internal");
	}
	void updateBoundary(Block* b) { check(e3d_update_boundary(s_, b->block_id_), "update_boundary"); }
	double gamma_;
	int current_stage_;
	std::vector<double> alpha_rk_;

private:
	e3d_solver* s_;
};

// Solver::saveW0 (Solver/src/Solver.cpp:161-210) and the inter-block halo
// (BlockCommunicator::updateBoundaries) on the device
inline void save_w0(e3d_solver* s, Block* b) { check(e3d_save_w0(s, b->block_id_), "save_w0"); }
inline void halo(e3d_solver* s) { check(e3d_halo(s), "halo"); }

// Copies the device state of block b into the reference's host arrays:
// primitives of every cell, convective/dissipative residuals and W0 of the real
// cells, time steps, and (second order) gradients and limiters.
inline void sync_to_host(e3d_solver* s, Block* b, bool interpolation = true) {
	const int nr = b->n_real_cells_in_block_, na = b->n_all_cells_in_block_;
	std::vector<double> v;
	PrimitiveVariables* pv = b->block_primitive_variables_;
	auto get = [&](const char* name, size_t n) {
		v.resize(n);
		check(e3d_state_get(s, b->block_id_, name, v.data(), (int64_t)n), name);
	};
	auto scatter5 = [&](int n, double* a0, double* a1, double* a2, double* a3, double* a4) {
		double* a[5] = {a0, a1, a2, a3, a4};
		for (int q = 0; q < 5; q++)
			for (int c = 0; c < n; c++) a[q][c] = v[(size_t)q * n + c];
	};
	get("prim", 5 * (size_t)na);
	scatter5(na, pv->ro_, pv->uu_, pv->vv_, pv->ww_, pv->pp_);
	get("conv_res", 5 * (size_t)nr);
	scatter5(nr, pv->conv_res_ro_, pv->conv_res_uu_, pv->conv_res_vv_, pv->conv_res_ww_, pv->conv_res_pp_);
	get("diss_res", 5 * (size_t)nr);
	scatter5(nr, pv->diss_res_ro_, pv->diss_res_uu_, pv->diss_res_vv_, pv->diss_res_ww_, pv->diss_res_pp_);
	get("w0", 5 * (size_t)nr);
	scatter5(nr, pv->ro_0_, pv->ru_0_, pv->rv_0_, pv->rw_0_, pv->re_0_);
	get("dt", (size_t)nr);
	for (int c = 0; c < nr; c++) b->block_time_variables_->dt_[c] = v[c];
	if (interpolation) {
		InterpolationVariables* iv = b->block_interpolation_variables_;
		get("limiter", 5 * (size_t)na);
		scatter5(na, iv->limiter_ro_, iv->limiter_uu_, iv->limiter_vv_, iv->limiter_ww_, iv->limiter_pp_);
		get("grad", 15 * (size_t)na);
		double** g[5] = {iv->grad_ro_, iv->grad_uu_, iv->grad_vv_, iv->grad_ww_, iv->grad_pp_};
		for (int q = 0; q < 5; q++)
			for (int c = 0; c < na; c++)
				for (int d = 0; d < 3; d++) g[q][c][d] = v[((size_t)q * na + c) * 3 + d];
	}
}

}  // namespace e3d_adapters
