// Kernels of the residual/update path.
//
// Granular kernels (FP64) mirror one reference strategy method each and keep
// the reference's array meanings, so the drop-in adapters can call them one by
// one.  Fused kernels (templated on T) do the same arithmetic per RK stage in
// two passes: k_recon (gradient + limiter + MUSCL face states, ghost cells
// included) and k_flux_update (both fluxes, residual gather, conservative
// update, boundary conditions).  Every per-cell sum runs over the cell's slots
// in ascending face id, the reference's accumulation order, and no kernel uses
// atomics: each cell (or ghost) is written by exactly one thread.
#pragma once
#include "physics.cuh"
#include "views.hpp"

namespace e3d {
// Internal linkage: k64.cu and k32.cu each compile their own copy.
namespace {

template <class T>
__device__ __forceinline__ Q5<T> ld5(const T* __restrict__ P, int n, int c) {
	Q5<T> q;
	q.r = P[c];
	q.u = P[n + c];
	q.v = P[2 * n + c];
	q.w = P[3 * n + c];
	q.p = P[4 * n + c];
	return q;
}
template <class T>
__device__ __forceinline__ void st5(T* __restrict__ P, int n, int c, const Q5<T>& q) {
	P[c] = q.r;
	P[n + c] = q.u;
	P[2 * n + c] = q.v;
	P[3 * n + c] = q.w;
	P[4 * n + c] = q.p;
}
template <class T>
__device__ __forceinline__ T& qv(Q5<T>& q, int v) { return (&q.r)[v]; }
template <class T>
__device__ __forceinline__ T qv(const Q5<T>& q, int v) { return (&q.r)[v]; }

// Thread index -> cell of a per-block range: real cells [r0, r1) then ghost
// cells [NR+g0, NR+g1).
__device__ __forceinline__ int range_cell(int t, int r0, int r1, int NR, int g0, int g1) {
	const int nr = r1 - r0;
	if (t < nr) return r0 + t;
	t -= nr;
	if (t < g1 - g0) return NR + g0 + t;
	return -1;
}

// ===================================================================== granular
// Solver::saveW0 (Solver/src/Solver.cpp:161-210).
__global__ void k_save_w0(GeoView g, StateView s, Physics ph, int r0, int r1) {
	const int c = r0 + blockIdx.x * blockDim.x + threadIdx.x;
	if (c >= r1) return;
	const Q5<double> q = ld5(s.prim, g.NA, c);
	const int n = g.NR;
	s.w0[c] = q.r;
	s.w0[n + c] = q.r * q.u;
	s.w0[2 * n + c] = q.r * q.v;
	s.w0[3 * n + c] = q.r * q.w;
	s.w0[4 * n + c] = 0.5 * q.r * (q.u * q.u + q.v * q.v + q.w * q.w) + 1. / (ph.gamma - 1.0) * q.p;
}

// Timestep::computeSpectralRadius (Solver/src/Timestep.cpp:26-121): the cell's
// own state on every face.
__global__ void k_spectral_radius(GeoView g, StateView s, Physics ph, int r0, int r1) {
	const int c = r0 + blockIdx.x * blockDim.x + threadIdx.x;
	if (c >= r1) return;
	const Q5<double> q = ld5(s.prim, g.NA, c);
	const double cc = sqrt(ph.gamma * q.p / q.r);
	double sr = 0.0;
	for (int k = g.slot_ptr[c]; k < g.slot_ptr[c + 1]; k++) {
		const int f = g.slot_face[k];
		const double nx = g.nhat[3 * f], ny = g.nhat[3 * f + 1], nz = g.nhat[3 * f + 2], ds = g.area[f];
		sr += (fabs((q.u) * nx + (q.v) * ny + (q.w) * nz) + (cc)) * ds;
	}
	s.srad[c] = sr;
}

// Timestep::computeTimestep (Timestep.cpp:123-148).
__global__ void k_timestep(GeoView g, StateView s, Physics ph, int r0, int r1) {
	const int c = r0 + blockIdx.x * blockDim.x + threadIdx.x;
	if (c >= r1) return;
	s.dt[c] = ph.cfl * g.vol[c] / s.srad[c];
}

// Writes the ghost gradients owned by real cell c: reflected for ghosts of the
// first n_real_boundaries markers, zero for the others (GreenGauss.cpp:68-81,
// 175-232; LeastSquares.cpp:62-75, 127-184).
__device__ __forceinline__ void write_ghost_grads(const GeoView& g, const StateView& s, int c, const double gr[5][3]) {
	for (int k = g.slot_ptr[c]; k < g.slot_ptr[c + 1]; k++) {
		const int nb = g.slot_nbr[k];
		if (nb < g.NR) continue;
		const int f = g.slot_face[k];
		for (int v = 0; v < 5; v++) {
			double go[3] = {0.0, 0.0, 0.0};
			if (g.grefl[nb - g.NR]) reflect_grad(gr[v], g.nhat[3 * f], g.nhat[3 * f + 1], g.nhat[3 * f + 2], go);
			for (int d = 0; d < 3; d++) s.grad[(v * 3 + d) * g.NA + nb] = go[d];
		}
	}
}

// GreenGauss::computeGradients (Solver/src/GreenGauss.cpp:86-166).
__global__ void k_grad_gg(GeoView g, StateView s, int r0, int r1) {
	const int c = r0 + blockIdx.x * blockDim.x + threadIdx.x;
	if (c >= r1) return;
	double gr[5][3];
	for (int v = 0; v < 5; v++) gr[v][0] = gr[v][1] = gr[v][2] = 0.0;
	for (int k = g.slot_ptr[c]; k < g.slot_ptr[c + 1]; k++) {
		const int f = g.slot_face[k];
		double n[3] = {g.S[3 * f], g.S[3 * f + 1], g.S[3 * f + 2]};
		if (c != g.face_lr[2 * f])
			for (int d = 0; d < 3; d++) n[d] *= -1.0;
		const Q5<double> L = ld5(s.prim, g.NA, g.face_lr[2 * f]);
		const Q5<double> R = ld5(s.prim, g.NA, g.face_lr[2 * f + 1]);
		for (int d = 0; d < 3; d++)
			for (int v = 0; v < 5; v++) gr[v][d] += 0.5 * (qv(L, v) + qv(R, v)) * n[d];
	}
	const double V = g.vol[c];
	for (int d = 0; d < 3; d++)
		for (int v = 0; v < 5; v++) gr[v][d] /= V;
	for (int v = 0; v < 5; v++)
		for (int d = 0; d < 3; d++) s.grad[(v * 3 + d) * g.NA + c] = gr[v][d];
	write_ghost_grads(g, s, c, gr);
}

// LeastSquares::computeGradients (Solver/src/LeastSquares.cpp:80-119).
__global__ void k_grad_ls(GeoView g, StateView s, int r0, int r1) {
	const int c = r0 + blockIdx.x * blockDim.x + threadIdx.x;
	if (c >= r1) return;
	double gr[5][3];
	for (int v = 0; v < 5; v++) gr[v][0] = gr[v][1] = gr[v][2] = 0.0;
	const Q5<double> q0 = ld5(s.prim, g.NA, c);
	for (int k = g.slot_ptr[c]; k < g.slot_ptr[c + 1]; k++) {
		const Q5<double> qi = ld5(s.prim, g.NA, g.slot_nbr[k]);
		for (int d = 0; d < 3; d++) {
			const double w = g.lsw[3 * k + d];
			for (int v = 0; v < 5; v++) gr[v][d] += w * (qv(qi, v) - qv(q0, v));
		}
	}
	for (int v = 0; v < 5; v++)
		for (int d = 0; d < 3; d++) s.grad[(v * 3 + d) * g.NA + c] = gr[v][d];
	write_ghost_grads(g, s, c, gr);
}

// BarthJespersen::computeLimiters / Venkatakrishnan::computeLimiters
// (Solver/src/BarthJespersen.cpp:88-331, Venkatakrishnan.cpp:87-324), all cells.
template <int LIM>
__global__ void k_limiter(GeoView g, StateView s, Physics ph, int r0, int r1, int g0, int g1) {
	const int c = range_cell(blockIdx.x * blockDim.x + threadIdx.x, r0, r1, g.NR, g0, g1);
	if (c < 0) return;
	const Q5<double> q0 = ld5(s.prim, g.NA, c);
	Q5<double> mx = q0, mn = q0;
	for (int k = g.slot_ptr[c]; k < g.slot_ptr[c + 1]; k++) {
		const Q5<double> qn = ld5(s.prim, g.NA, g.slot_nbr[k]);
		for (int v = 0; v < 5; v++) {
			if (qv(qn, v) > qv(mx, v)) qv(mx, v) = qv(qn, v);
			if (qv(qn, v) < qv(mn, v)) qv(mn, v) = qv(qn, v);
		}
	}
	double dmax[5], dmin[5], phi[5], gr[5][3];
	for (int v = 0; v < 5; v++) {
		dmax[v] = qv(mx, v) - qv(q0, v);
		dmin[v] = qv(mn, v) - qv(q0, v);
		phi[v] = INFINITY;
		for (int d = 0; d < 3; d++) gr[v][d] = s.grad[(v * 3 + d) * g.NA + c];
	}
	const double eps2 = ph.k3 * g.vol[c];
	for (int k = g.slot_ptr[c]; k < g.slot_ptr[c + 1]; k++) {
		const int f = g.slot_face[k];
		const double* r = (c == g.face_lr[2 * f]) ? &g.rl[3 * f] : &g.rr[3 * f];
		for (int v = 0; v < 5; v++) {
			double d2 = 0.0;
			for (int d = 0; d < 3; d++) d2 += gr[v][d] * r[d];
			const double lf = (LIM == LIM_BARTH_JESPERSEN) ? limiter_bj_face(d2, dmax[v], dmin[v], ph.omega)
			                                               : limiter_venkat_face(d2, dmax[v], dmin[v], eps2);
			if (lf < phi[v]) phi[v] = lf;
		}
	}
	for (int v = 0; v < 5; v++) s.lim[v * g.NA + c] = phi[v];
}

// Left/right states of face f reconstructed from gradients and limiters.
__device__ __forceinline__ void face_states(const GeoView& g, const StateView& s, int f, Q5<double>& L, Q5<double>& R) {
	const int l = g.face_lr[2 * f], r = g.face_lr[2 * f + 1];
	L = ld5(s.prim, g.NA, l);
	R = ld5(s.prim, g.NA, r);
	for (int v = 0; v < 5; v++) {
		const double* gl = &s.grad[0];
		qv(L, v) = recon(qv(L, v), s.lim[v * g.NA + l], gl[(v * 3 + 0) * g.NA + l], gl[(v * 3 + 1) * g.NA + l],
		                 gl[(v * 3 + 2) * g.NA + l], g.rl[3 * f], g.rl[3 * f + 1], g.rl[3 * f + 2]);
		qv(R, v) = recon(qv(R, v), s.lim[v * g.NA + r], gl[(v * 3 + 0) * g.NA + r], gl[(v * 3 + 1) * g.NA + r],
		                 gl[(v * 3 + 2) * g.NA + r], g.rr[3 * f], g.rr[3 * f + 1], g.rr[3 * f + 2]);
	}
}

// FluxScheme::computeFluxConv / AusmScheme::computeFluxConv gathered per cell
// (FluxScheme.cpp:83-207, AusmScheme.cpp:716-871).
template <int SCHEME>
__global__ void k_flux_conv(GeoView g, StateView s, Physics ph, int r0, int r1) {
	const int c = r0 + blockIdx.x * blockDim.x + threadIdx.x;
	if (c >= r1) return;
	double acc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
	for (int k = g.slot_ptr[c]; k < g.slot_ptr[c + 1]; k++) {
		const int f = g.slot_face[k];
		Q5<double> L, R;
		face_states(g, s, f, L, R);
		double fl[5];
		const double nx = g.nhat[3 * f], ny = g.nhat[3 * f + 1], nz = g.nhat[3 * f + 2], nn = g.area[f];
		if (SCHEME == FLUX_ROE) flux_central(L, R, nx, ny, nz, nn, ph.gr, fl);
		else flux_ausm_conv(L, R, nx, ny, nz, nn, ph.gamma, ph.gr, fl);
		if (c == g.face_lr[2 * f])
			for (int v = 0; v < 5; v++) acc[v] += fl[v];
		else
			for (int v = 0; v < 5; v++) acc[v] -= fl[v];
	}
	for (int v = 0; v < 5; v++) s.rc[v * g.NR + c] = acc[v];
}

// RoeScheme::computeFluxDiss / AusmScheme::computeFluxDiss gathered per cell
// (RoeScheme.cpp:87-291, AusmScheme.cpp:84-243): Rd <- (1-beta) Rd + beta * D.
template <int SCHEME>
__global__ void k_flux_diss(GeoView g, StateView s, Physics ph, double beta, int r0, int r1) {
	const int c = r0 + blockIdx.x * blockDim.x + threadIdx.x;
	if (c >= r1) return;
	double acc[5];
	for (int v = 0; v < 5; v++) acc[v] = s.rd[v * g.NR + c] * (1.0 - beta);
	for (int k = g.slot_ptr[c]; k < g.slot_ptr[c + 1]; k++) {
		const int f = g.slot_face[k];
		Q5<double> L, R;
		face_states(g, s, f, L, R);
		double fl[5];
		const double nx = g.nhat[3 * f], ny = g.nhat[3 * f + 1], nz = g.nhat[3 * f + 2], nn = g.area[f];
		if (SCHEME == FLUX_ROE) flux_roe_diss(L, R, nx, ny, nz, nn, ph.gr, ph.gm1, fl);
		else flux_ausm_diss(L, R, nx, ny, nz, nn, ph.gamma, ph.gr, fl);
		if (c == g.face_lr[2 * f])
			for (int v = 0; v < 5; v++) acc[v] += fl[v] * beta;
		else
			for (int v = 0; v < 5; v++) acc[v] -= fl[v] * beta;
	}
	for (int v = 0; v < 5; v++) s.rd[v * g.NR + c] = acc[v];
}

// Conservative update and primitive recovery, W0 - alpha*dt/V*(Rc-Rd)
// (Updater::updateInternalBlock, Solver/src/Updater.cpp:31-76).
template <class T>
__device__ __forceinline__ Q5<T> conservative_update(const double w0[5], T coef, const T rc[5], const T rd[5], T gm1,
                                                     double wn[5]) {
	for (int v = 0; v < 5; v++) wn[v] = w0[v] - (double)(coef) * (double)(rc[v] - rd[v]);
	Q5<T> q;
	q.r = (T)wn[0];
	q.u = (T)(wn[1] / wn[0]);
	q.v = (T)(wn[2] / wn[0]);
	q.w = (T)(wn[3] / wn[0]);
	q.p = (T)((double)gm1 * (wn[4] - 0.5 * (wn[1] * wn[1] + wn[2] * wn[2] + wn[3] * wn[3]) / wn[0]));
	return q;
}

__global__ void k_update(GeoView g, StateView s, Physics ph, double alpha, int r0, int r1) {
	const int c = r0 + blockIdx.x * blockDim.x + threadIdx.x;
	if (c >= r1) return;
	const int n = g.NR;
	double w0[5], rc[5], rd[5], wn[5];
	for (int v = 0; v < 5; v++) {
		w0[v] = s.w0[v * n + c];
		rc[v] = s.rc[v * n + c];
		rd[v] = s.rd[v * n + c];
	}
	const double coef = alpha * s.dt[c] / g.vol[c];
	const Q5<double> q = conservative_update<double>(w0, coef, rc, rd, ph.gamma - 1.0, wn);
	st5(s.prim, g.NA, c, q);
}

// Ghost states of the first n_real_boundaries markers (Updater::updateBoundary,
// Updater.cpp:84-87, and the *CellIds::updateBoundary implementations).
template <class T>
__device__ __forceinline__ Q5<T> ghost_state(int kind, const Q5<T>& qi, const Q5<T>& fr, T nx, T ny, T nz, T gamma) {
	if (kind == GK_FARFIELD) return bc_farfield(qi, fr, nx, ny, nz, gamma);
	return bc_slip(qi, nx, ny, nz);
}

__global__ void k_bc(GeoView g, StateView s, Physics ph, int g0, int g1) {
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= g1 - g0) return;
	const int gi = g0 + t, c = g.NR + gi;
	const int kind = g.gkind[gi];
	if (kind == GK_NONE) return;
	const int k = g.slot_ptr[c];
	const int f = g.slot_face[k], in = g.slot_nbr[k];
	Q5<double> fr;
	fr.r = ph.free[0];
	fr.u = ph.free[1];
	fr.v = ph.free[2];
	fr.w = ph.free[3];
	fr.p = ph.free[4];
	const Q5<double> q = ghost_state(kind, ld5(s.prim, g.NA, in), fr, g.nhat[3 * f], g.nhat[3 * f + 1],
	                                 g.nhat[3 * f + 2], ph.gamma);
	st5(s.prim, g.NA, c, q);
}

// Inter-block halo: connexion ghost primitives <- origin cell primitives, once
// per outer iteration (BlockCommunicator::updateBoundaries, serial path
// MPI/src/BlockCommunicator.cpp:212-268; the other 35 copied values are
// rewritten before any read).  Writes every buffer in `bufs`.
template <class T>
__global__ void k_halo(int n, const int* __restrict__ dst, const int* __restrict__ src, int NA, T* b0, T* b1) {
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= n) return;
	const int d = dst[t], o = src[t];
	for (int v = 0; v < 5; v++) {
		const T x = b0[v * NA + o];
		b0[v * NA + d] = x;
		if (b1) b1[v * NA + d] = x;
	}
}

// ===================================================================== fused
// Pass 1 of a stage, one thread per real cell: gradient, limiter and MUSCL
// face states of the cell and of its ghost cells.  FIRST additionally computes
// W0 (unless carried) and the local time step from the stage-0 state.
template <class T, int GRAD, int LIM, bool FIRST>
__global__ void __launch_bounds__(128) k_recon(FusedView<T> v, Physics ph, int carry_w0) {
	const int c = blockIdx.x * blockDim.x + threadIdx.x;
	if (c >= v.NR) return;
	const int s0 = v.tet4 ? 4 * c : v.slot_ptr[c];
	const int s1 = v.tet4 ? s0 + 4 : v.slot_ptr[c + 1];
	const Q5<T> q0 = ld5(v.Pin, v.NA, c);
	T gr[5][3];
	for (int q = 0; q < 5; q++) gr[q][0] = gr[q][1] = gr[q][2] = T(0.0);
	Q5<T> mx = q0, mn = q0;
	for (int k = s0; k < s1; k++) {
		const Q5<T> qn = ld5(v.Pin, v.NA, v.slot_nbr[k]);
		if (GRAD == GRAD_GREEN_GAUSS) {
			const T n0 = v.sS[3 * k], n1 = v.sS[3 * k + 1], n2 = v.sS[3 * k + 2];
			for (int q = 0; q < 5; q++) {
				const T a = T(0.5) * (qv(q0, q) + qv(qn, q));
				gr[q][0] += a * n0;
				gr[q][1] += a * n1;
				gr[q][2] += a * n2;
			}
		} else {
			const T w0 = v.lsw[3 * k], w1 = v.lsw[3 * k + 1], w2 = v.lsw[3 * k + 2];
			for (int q = 0; q < 5; q++) {
				const T dq = qv(qn, q) - qv(q0, q);
				gr[q][0] += w0 * dq;
				gr[q][1] += w1 * dq;
				gr[q][2] += w2 * dq;
			}
		}
		for (int q = 0; q < 5; q++) {
			if (qv(qn, q) > qv(mx, q)) qv(mx, q) = qv(qn, q);
			if (qv(qn, q) < qv(mn, q)) qv(mn, q) = qv(qn, q);
		}
	}
	const T V = v.vol[c];
	if (GRAD == GRAD_GREEN_GAUSS)
		for (int d = 0; d < 3; d++)
			for (int q = 0; q < 5; q++) gr[q][d] /= V;
	T phi[5], dmax[5], dmin[5];
	for (int q = 0; q < 5; q++) {
		dmax[q] = qv(mx, q) - qv(q0, q);
		dmin[q] = qv(mn, q) - qv(q0, q);
		phi[q] = T(INFINITY);
	}
	const T eps2 = T(ph.k3) * V;
	for (int k = s0; k < s1; k++) {
		const T r0 = v.srv[3 * k], r1 = v.srv[3 * k + 1], r2 = v.srv[3 * k + 2];
		for (int q = 0; q < 5; q++) {
			T d2 = T(0.0);
			d2 += gr[q][0] * r0;
			d2 += gr[q][1] * r1;
			d2 += gr[q][2] * r2;
			const T lf = (LIM == LIM_BARTH_JESPERSEN) ? limiter_bj_face(d2, dmax[q], dmin[q], T(ph.omega))
			                                          : limiter_venkat_face(d2, dmax[q], dmin[q], eps2);
			if (lf < phi[q]) phi[q] = lf;
		}
	}
	for (int k = s0; k < s1; k++) {
		const T r0 = v.srv[3 * k], r1 = v.srv[3 * k + 1], r2 = v.srv[3 * k + 2];
		for (int q = 0; q < 5; q++) v.FS[q * v.NS + k] = recon(qv(q0, q), phi[q], gr[q][0], gr[q][1], gr[q][2], r0, r1, r2);
		const int nb = v.slot_nbr[k];
		if (nb < v.NR) continue;
		// ghost cell of this face: its gradient, limiter (its only neighbour is c)
		// and face state
		int ms = v.slot_mate[k];
		ms = ms >= 0 ? ms : ~ms;
		const Q5<T> qg = ld5(v.Pin, v.NA, nb);
		const T nx = v.sgeo[4 * k], ny = v.sgeo[4 * k + 1], nz = v.sgeo[4 * k + 2];
		const T g0 = v.srv[3 * ms], g1 = v.srv[3 * ms + 1], g2 = v.srv[3 * ms + 2];
		const bool refl = v.grefl[nb - v.NR] != 0;
		const T eps2g = T(ph.k3) * v.vol[nb];
		for (int q = 0; q < 5; q++) {
			T gg[3] = {T(0.0), T(0.0), T(0.0)};
			if (refl) reflect_grad(gr[q], nx, ny, nz, gg);
			T gmx = qv(qg, q), gmn = qv(qg, q);
			if (qv(q0, q) > gmx) gmx = qv(q0, q);
			if (qv(q0, q) < gmn) gmn = qv(q0, q);
			T d2 = T(0.0);
			d2 += gg[0] * g0;
			d2 += gg[1] * g1;
			d2 += gg[2] * g2;
			const T dmx = gmx - qv(qg, q), dmn = gmn - qv(qg, q);
			const T lf = (LIM == LIM_BARTH_JESPERSEN) ? limiter_bj_face(d2, dmx, dmn, T(ph.omega))
			                                          : limiter_venkat_face(d2, dmx, dmn, eps2g);
			T pg = T(INFINITY);
			if (lf < pg) pg = lf;
			v.FS[q * v.NS + ms] = recon(qv(qg, q), pg, gg[0], gg[1], gg[2], g0, g1, g2);
		}
	}
	if (FIRST) {
		if (!carry_w0) {
			const int n = v.NR;
			v.W0[c] = (double)q0.r;
			v.W0[n + c] = (double)(q0.r * q0.u);
			v.W0[2 * n + c] = (double)(q0.r * q0.v);
			v.W0[3 * n + c] = (double)(q0.r * q0.w);
			v.W0[4 * n + c] = (double)(T(0.5) * q0.r * (q0.u * q0.u + q0.v * q0.v + q0.w * q0.w) +
			                           T(1.) / (T(ph.gamma) - T(1.0)) * q0.p);
		}
		const T cc = tsqrt(T(ph.gamma) * q0.p / q0.r);
		T sr = T(0.0);
		for (int k = s0; k < s1; k++) {
			const T nx = v.sgeo[4 * k], ny = v.sgeo[4 * k + 1], nz = v.sgeo[4 * k + 2], ds = v.sgeo[4 * k + 3];
			sr += (tabs((q0.u) * nx + (q0.v) * ny + (q0.w) * nz) + (cc)) * ds;
		}
		v.dt[c] = T(ph.cfl) * V / sr;
	}
}

// W0 and the local time step without a reconstruction pass (first order).
template <class T>
__global__ void __launch_bounds__(128) k_start(FusedView<T> v, Physics ph, int carry_w0) {
	const int c = blockIdx.x * blockDim.x + threadIdx.x;
	if (c >= v.NR) return;
	const int s0 = v.tet4 ? 4 * c : v.slot_ptr[c];
	const int s1 = v.tet4 ? s0 + 4 : v.slot_ptr[c + 1];
	const Q5<T> q0 = ld5(v.Pin, v.NA, c);
	if (!carry_w0) {
		const int n = v.NR;
		v.W0[c] = (double)q0.r;
		v.W0[n + c] = (double)(q0.r * q0.u);
		v.W0[2 * n + c] = (double)(q0.r * q0.v);
		v.W0[3 * n + c] = (double)(q0.r * q0.w);
		v.W0[4 * n + c] = (double)(T(0.5) * q0.r * (q0.u * q0.u + q0.v * q0.v + q0.w * q0.w) +
		                           T(1.) / (T(ph.gamma) - T(1.0)) * q0.p);
	}
	const T cc = tsqrt(T(ph.gamma) * q0.p / q0.r);
	T sr = T(0.0);
	for (int k = s0; k < s1; k++) {
		const T nx = v.sgeo[4 * k], ny = v.sgeo[4 * k + 1], nz = v.sgeo[4 * k + 2], ds = v.sgeo[4 * k + 3];
		sr += (tabs((q0.u) * nx + (q0.v) * ny + (q0.w) * nz) + (cc)) * ds;
	}
	v.dt[c] = T(ph.cfl) * v.vol[c] / sr;
}

// Pass 2 of a stage, one thread per real cell: convective and dissipative
// fluxes of each face (computed identically from both sides), residual gather,
// conservative update into Pout and the ghost states of the cell's boundary
// faces.  ORDER1 reads cell states directly (first order).  LAST stores the
// final conservative state as the next W0 when carry_w0 is set.
template <class T, int SCHEME, bool ORDER1>
__global__ void __launch_bounds__(128) k_flux_update(FusedView<T> v, Physics ph, T alpha, T beta, int last, int carry_w0) {
	const int c = blockIdx.x * blockDim.x + threadIdx.x;
	if (c >= v.NR) return;
	const int s0 = v.tet4 ? 4 * c : v.slot_ptr[c];
	const int s1 = v.tet4 ? s0 + 4 : v.slot_ptr[c + 1];
	const T g = T(ph.gamma), gr = T(ph.gr), gm1 = T(ph.gm1);
	T ac[5], ad[5];
	for (int q = 0; q < 5; q++) {
		ac[q] = T(0.0);
		ad[q] = v.Rd[q * v.NR + c] * (T(1.0) - beta);
	}
	Q5<T> qc;
	if (ORDER1) qc = ld5(v.Pin, v.NA, c);
	for (int k = s0; k < s1; k++) {
		int m = v.slot_mate[k];
		const bool left = m >= 0;
		if (!left) m = ~m;
		Q5<T> qo, qn;
		if (ORDER1) {
			qo = qc;
			qn = ld5(v.Pin, v.NA, v.slot_nbr[k]);
		} else {
			qo = ld5(v.FS, v.NS, k);
			qn = ld5(v.FS, v.NS, m);
		}
		const Q5<T>& L = left ? qo : qn;
		const Q5<T>& R = left ? qn : qo;
		const T nx = v.sgeo[4 * k], ny = v.sgeo[4 * k + 1], nz = v.sgeo[4 * k + 2], nn = v.sgeo[4 * k + 3];
		T fc[5], fd[5];
		if (SCHEME == FLUX_ROE) {
			flux_central(L, R, nx, ny, nz, nn, gr, fc);
			flux_roe_diss(L, R, nx, ny, nz, nn, gr, gm1, fd);
		} else {
			flux_ausm_conv(L, R, nx, ny, nz, nn, g, gr, fc);
			flux_ausm_diss(L, R, nx, ny, nz, nn, g, gr, fd);
		}
		if (left) {
			for (int q = 0; q < 5; q++) {
				ac[q] += fc[q];
				ad[q] += fd[q] * beta;
			}
		} else {
			for (int q = 0; q < 5; q++) {
				ac[q] -= fc[q];
				ad[q] -= fd[q] * beta;
			}
		}
	}
	double w0[5], wn[5];
	for (int q = 0; q < 5; q++) {
		v.Rc[q * v.NR + c] = ac[q];
		v.Rd[q * v.NR + c] = ad[q];
		w0[q] = v.W0[q * v.NR + c];
	}
	const T coef = alpha * v.dt[c] / v.vol[c];
	const Q5<T> qnew = conservative_update<T>(w0, coef, ac, ad, gm1, wn);
	st5(v.Pout, v.NA, c, qnew);
	if (last && carry_w0)
		for (int q = 0; q < 5; q++) v.W0[q * v.NR + c] = wn[q];
	Q5<T> fr;
	fr.r = T(ph.free[0]);
	fr.u = T(ph.free[1]);
	fr.v = T(ph.free[2]);
	fr.w = T(ph.free[3]);
	fr.p = T(ph.free[4]);
	for (int k = s0; k < s1; k++) {
		const int nb = v.slot_nbr[k];
		if (nb < v.NR) continue;
		const int kind = v.gkind[nb - v.NR];
		if (kind == GK_NONE) continue;
		const Q5<T> qg = ghost_state(kind, qnew, fr, v.sgeo[4 * k], v.sgeo[4 * k + 1], v.sgeo[4 * k + 2], g);
		st5(v.Pout, v.NA, nb, qg);
	}
}

// ===================================================================== reductions
// Per-block partial sums of (Rc-Rd)^2 (Convergence::calculate*Rms,
// PostProcessing/src/Convergence.cpp:27-143).  grid = (chunks, blocks); a
// chunk never straddles two blocks; the final sum runs in fixed chunk order.
template <class T, int THREADS>
__global__ void __launch_bounds__(THREADS) k_norm_partial(const T* __restrict__ Rc, const T* __restrict__ Rd, int NR,
                                                          const int* __restrict__ roff, int chunk, int max_chunks,
                                                          double* __restrict__ partial) {
	const int b = blockIdx.y;
	const int beg = roff[b] + blockIdx.x * chunk;
	const int end = min(roff[b + 1], beg + chunk);
	double acc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
	for (int c = beg + threadIdx.x; c < end; c += THREADS)
		for (int q = 0; q < 5; q++) {
			const double r = (double)Rc[q * NR + c] - (double)Rd[q * NR + c];
			acc[q] += r * r;
		}
	__shared__ double sm[5][THREADS];
	for (int q = 0; q < 5; q++) sm[q][threadIdx.x] = acc[q];
	__syncthreads();
	for (int w = THREADS / 2; w > 0; w >>= 1) {
		if (threadIdx.x < w)
			for (int q = 0; q < 5; q++) sm[q][threadIdx.x] += sm[q][threadIdx.x + w];
		__syncthreads();
	}
	if (threadIdx.x < 5) partial[((size_t)b * max_chunks + blockIdx.x) * 5 + threadIdx.x] = sm[threadIdx.x][0];
}

// hist[iter*stride + b*10 + q] = sum over chunks in fixed order; sets *bad
// when a sum is not finite (NaN propagates silently in the reference).
__global__ void k_norm_final(const double* __restrict__ partial, int nblocks, int max_chunks, double* __restrict__ hist,
                             int stride, const int* __restrict__ d_iter, int* __restrict__ bad) {
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= nblocks * 5) return;
	const int b = t / 5, q = t % 5;
	double s = 0.0;
	for (int i = 0; i < max_chunks; i++) s += partial[((size_t)b * max_chunks + i) * 5 + q];
	hist[(size_t)(*d_iter) * stride + b * 10 + q] = s;
	if (!isfinite(s)) *bad = 1;
}

// Wall pressure force sums per block, sequential in wall-face order like
// AerodynamicParameters::computeAerodynamic (AerodynamicParameters.cpp:189-232).
// hist[iter*stride + b*10 + 5 + {0..4}] = sum fy, sum fx, cmx, cmy, cmz.
template <class T>
__global__ void k_forces(const T* __restrict__ P, int NA, const int* __restrict__ wall_off,
                         const int* __restrict__ wall_face, const int* __restrict__ face_lr,
                         const double* __restrict__ S, const double* __restrict__ fc, double denom, int nblocks,
                         double* __restrict__ hist, int stride, const int* __restrict__ d_iter) {
	const int b = blockIdx.x * blockDim.x + threadIdx.x;
	if (b >= nblocks) return;
	double cl = 0., cd = 0., cmx = 0., cmy = 0., cmz = 0.;
	for (int i = wall_off[b]; i < wall_off[b + 1]; i++) {
		const int f = wall_face[i];
		const double p0 = (double)P[4 * NA + face_lr[2 * f]], p1 = (double)P[4 * NA + face_lr[2 * f + 1]];
		const double pbc = 0.5 * (p0 + p1);
		const double cp = (pbc - 1.) / denom;
		const double fx = cp * S[3 * f], fy = cp * S[3 * f + 1], fz = cp * S[3 * f + 2];
		const double x = fc[3 * f], y = fc[3 * f + 1], z = fc[3 * f + 2];
		cl += fy;
		cd += fx;
		cmx += y * fz - z * fy;
		cmy += z * fx - x * fz;
		cmz += x * fy - y * fx;
	}
	double* out = hist + (size_t)(*d_iter) * stride + b * 10 + 5;
	out[0] = cl;
	out[1] = cd;
	out[2] = cmx;
	out[3] = cmy;
	out[4] = cmz;
}

__global__ void k_iter_advance(int* d_iter) { *d_iter += 1; }

}  // namespace
}  // namespace e3d
