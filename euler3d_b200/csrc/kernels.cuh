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
#include <cooperative_groups.h>

#include "physics.cuh"
#include "views.hpp"

namespace e3d {
// Internal linkage: k64.cu and k32.cu each compile their own copy.
namespace {

// Five-variable arrays use a packed layout: [n] vectors of (rho, u, v, w)
// followed by [n] p.  A gather of one cell's state touches two memory sectors
// (one 16/32-byte vector + one scalar) instead of five.
template <class T>
struct Vec4;
template <>
struct Vec4<float> {
	using type = float4;
};
template <>
struct Vec4<double> {
	using type = double4;
};

template <class T>
__device__ __forceinline__ Q5<T> ld5(const T* __restrict__ P, int n, int c) {
	const typename Vec4<T>::type a = reinterpret_cast<const typename Vec4<T>::type*>(P)[c];
	Q5<T> q;
	q.r = a.x;
	q.u = a.y;
	q.v = a.z;
	q.w = a.w;
	q.p = P[4 * (size_t)n + c];
	return q;
}
template <class T>
__device__ __forceinline__ void st5(T* __restrict__ P, int n, int c, const Q5<T>& q) {
	typename Vec4<T>::type a;
	a.x = q.r;
	a.y = q.u;
	a.z = q.v;
	a.w = q.w;
	reinterpret_cast<typename Vec4<T>::type*>(P)[c] = a;
	P[4 * (size_t)n + c] = q.p;
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
#ifdef E3D_SHARED_SIDES
	if constexpr (sizeof(T) == 8) {  // contracted FP64 batch kernels: one reciprocal of rho
		const double ir = 1.0 / wn[0];
		q.r = wn[0];
		q.u = wn[1] * ir;
		q.v = wn[2] * ir;
		q.w = wn[3] * ir;
		q.p = gm1 * (wn[4] - 0.5 * (wn[1] * wn[1] + wn[2] * wn[2] + wn[3] * wn[3]) * ir);
		return q;
	}
#endif
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
// CentralIrsSmoother::smoothResidual (Solver/src/CentralIrsSmoother.cpp:12-166):
// one Jacobi step of central implicit residual smoothing, eps = 0.8, applied to
// the convective and the dissipative residuals of the real cells.  Pass 1: the
// start value J1 = R / (1 + eps N) (N = the cell's face count) of all ten arrays.
// The reference fills J1 of the dissipative v-momentum from the w-momentum and
// never fills J1 of the dissipative w-momentum (:90); these two follow the
// formula of the other eight here.
constexpr double IRS_EPS = 0.8;
__global__ void k_irs_start(GeoView g, StateView s, double* __restrict__ j1, int r0, int r1) {
	const int c = r0 + blockIdx.x * blockDim.x + threadIdx.x;
	if (c >= r1) return;
	const int na = g.slot_ptr[c + 1] - g.slot_ptr[c];
	for (int q = 0; q < 5; q++) {
		j1[q * (size_t)g.NR + c] = (s.rc[q * (size_t)g.NR + c] + 0.) / (1. + IRS_EPS * na);
		j1[(5 + q) * (size_t)g.NR + c] = (s.rd[q * (size_t)g.NR + c] + 0.) / (1. + IRS_EPS * na);
	}
}

// Pass 2: R = (R + eps * sum of J1 over the real neighbours in slot order) / (1 + eps N),
// in place (each thread reads only its own R and the neighbours' J1).
__global__ void k_irs_smooth(GeoView g, StateView s, const double* __restrict__ j1, int r0, int r1) {
	const int c = r0 + blockIdx.x * blockDim.x + threadIdx.x;
	if (c >= r1) return;
	double sc[5] = {0., 0., 0., 0., 0.}, sd[5] = {0., 0., 0., 0., 0.};
	for (int k = g.slot_ptr[c]; k < g.slot_ptr[c + 1]; k++) {
		const int nb = g.slot_nbr[k];
		if (nb < g.NR)
			for (int q = 0; q < 5; q++) {
				sc[q] += j1[q * (size_t)g.NR + nb];
				sd[q] += j1[(5 + q) * (size_t)g.NR + nb];
			}
	}
	const int na = g.slot_ptr[c + 1] - g.slot_ptr[c];
	for (int q = 0; q < 5; q++) {
		double& rc = s.rc[q * (size_t)g.NR + c];
		double& rd = s.rd[q * (size_t)g.NR + c];
		rc = (rc + IRS_EPS * sc[q]) / (1. + IRS_EPS * na);
		rd = (rd + IRS_EPS * sd[q]) / (1. + IRS_EPS * na);
	}
}

template <class T>
__global__ void k_halo(int n, const int* __restrict__ dst, const int* __restrict__ src, int NA, T* b0, T* b1) {
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= n) return;
	const int d = dst[t], o = src[t];
	const Q5<T> q = ld5(b0, NA, o);
	st5(b0, NA, d, q);
	if (b1) st5(b1, NA, d, q);
}

// The halo of a block-sharded case, split at the transport: pack gathers the
// primitives of the origin cells another process needs into an entry-major
// buffer (buf[5*i + q], q = rho u v w p), unpack writes received entries into
// the connexion ghosts of both state buffers, as k_halo does for local ones.
template <class T>
__global__ void k_halo_pack(int n, const int* __restrict__ src, int NA, const T* __restrict__ P,
                            T* __restrict__ buf) {
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= n) return;
	const Q5<T> q = ld5(P, NA, src[t]);
	T* o = buf + 5 * (size_t)t;
	o[0] = q.r;
	o[1] = q.u;
	o[2] = q.v;
	o[3] = q.w;
	o[4] = q.p;
}

template <class T>
__global__ void k_halo_unpack(int n, const int* __restrict__ dst, int NA, const T* __restrict__ buf, T* b0, T* b1) {
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= n) return;
	const T* i = buf + 5 * (size_t)t;
	const Q5<T> q{i[0], i[1], i[2], i[3], i[4]};
	st5(b0, NA, dst[t], q);
	if (b1) st5(b1, NA, dst[t], q);
}

// ===================================================================== fused
// Slot data of one real cell.  NSL = 4 is the all-tetrahedron fast path:
// slots of cell c are 4c..4c+3, so per-slot arrays load as vectors.  NSL = 0
// reads the slot range from slot_ptr (any cell type).
template <class T, int NSL>
struct SlotRange {
	int s0, n;
	__device__ __forceinline__ SlotRange(const FusedView<T>& v, int c) {
		if (NSL == 4) {
			s0 = 4 * c;
			n = 4;
		} else {
			s0 = v.slot_ptr[c];
			n = v.slot_ptr[c + 1] - s0;
		}
	}
};
constexpr int MAXSL = 6;  // hexahedra

// 3 consecutive values per slot (r-vectors, LS weights, signed area vectors)
template <class T, int NSL>
__device__ __forceinline__ void load3(const T* __restrict__ a, const SlotRange<T, NSL>& r, T o[MAXSL][3]) {
	if (NSL == 4 && sizeof(T) == 4) {
		const float4* p = reinterpret_cast<const float4*>(a + 3 * (size_t)r.s0);
		const float4 x = __ldg(p), y = __ldg(p + 1), z = __ldg(p + 2);
		const float f[12] = {x.x, x.y, x.z, x.w, y.x, y.y, y.z, y.w, z.x, z.y, z.z, z.w};
#pragma unroll
		for (int k = 0; k < 4; k++)
			for (int d = 0; d < 3; d++) o[k][d] = (T)f[3 * k + d];
	} else if (NSL == 4) {
		const double2* p = reinterpret_cast<const double2*>(a + 3 * (size_t)r.s0);
		double f[12];
#pragma unroll
		for (int i = 0; i < 6; i++) {
			const double2 t = __ldg(p + i);
			f[2 * i] = t.x;
			f[2 * i + 1] = t.y;
		}
#pragma unroll
		for (int k = 0; k < 4; k++)
			for (int d = 0; d < 3; d++) o[k][d] = (T)f[3 * k + d];
	} else {
		for (int k = 0; k < r.n; k++)
			for (int d = 0; d < 3; d++) o[k][d] = a[3 * (size_t)(r.s0 + k) + d];
	}
}
template <class T, int NSL>
__device__ __forceinline__ void load_int(const int* __restrict__ a, const SlotRange<T, NSL>& r, int o[MAXSL]) {
	if (NSL == 4) {
		const int4 x = __ldg(reinterpret_cast<const int4*>(a + r.s0));
		o[0] = x.x;
		o[1] = x.y;
		o[2] = x.z;
		o[3] = x.w;
	} else {
		for (int k = 0; k < r.n; k++) o[k] = a[r.s0 + k];
	}
}
// face normal + area of each slot (face orientation)
template <class T, int NSL>
__device__ __forceinline__ void load_geo(const T* __restrict__ a, const SlotRange<T, NSL>& r, T o[MAXSL][4]) {
	const typename Vec4<T>::type* p = reinterpret_cast<const typename Vec4<T>::type*>(a) + r.s0;
#pragma unroll
	for (int k = 0; k < (NSL == 4 ? 4 : MAXSL); k++) {
		if (NSL != 4 && k >= r.n) break;
		const typename Vec4<T>::type t = p[k];
		o[k][0] = t.x;
		o[k][1] = t.y;
		o[k][2] = t.z;
		o[k][3] = t.w;
	}
}

#define E3D_SLOTS(k, r) for (int k = 0; k < (NSL == 4 ? 4 : MAXSL); k++) if (NSL == 4 || k < r.n)

// First-order AUSM with each cell's side quantities formed once (built only
// where E3D_SHARED_SIDES is defined: the FP64 batch kernels with contraction,
// which are not held to the reference's operation order).  The reference forms
// a side's p/rho, speed of sound, enthalpy and c-scaled flux vector again in
// every face flux, convective and dissipative alike (AusmScheme.cpp:716-871,
// 102-243); a cell's own side is the same at all its faces, so here it is
// formed once per cell and the neighbour's once per face, the normal Mach
// number is V times 1/c, and c and 1/c come from one reciprocal square root.
// Same formulas otherwise, including the branch tests.
template <class T>
struct AusmSide {
	T u, v, w, p, ic;  // velocity, pressure, 1/c
	T F[5];            // rho c (1, u, v, w, H)
};
template <class T>
__device__ __forceinline__ AusmSide<T> ausm_side(const Q5<T>& q, T g, T gr) {
	AusmSide<T> s;
	const T pr = q.p / q.r;
	const T x = g * pr;
	s.ic = rsqrt(x);  // 1/c, and c = x/c: one reciprocal square root for both
	const T c = x * s.ic;
	const T H = T(0.5) * (q.u * q.u + q.v * q.v + q.w * q.w) + gr * pr;
	s.u = q.u;
	s.v = q.v;
	s.w = q.w;
	s.p = q.p;
	s.F[0] = q.r * c;
	s.F[1] = s.F[0] * q.u;
	s.F[2] = s.F[0] * q.v;
	s.F[3] = s.F[0] * q.w;
	s.F[4] = s.F[0] * H;
	return s;
}
template <class T, bool DISS>
__device__ __forceinline__ void ausm_face_sides(const AusmSide<T>& L, const AusmSide<T>& R, T nx, T ny, T nz, T nn,
                                                T fc[5], T fd[5]) {
	const T ML = (L.u * nx + L.v * ny + L.w * nz) * L.ic;
	const T MR = (R.u * nx + R.v * ny + R.w * nz) * R.ic;
	T pLp, MLp, pRm, MRm;
	if (ML <= T(-1.0)) {
		pLp = T(0);
		MLp = T(0);
	} else if (ML < T(1.0)) {
		MLp = T(0.25) * (ML + T(1.0)) * (ML + T(1.0));
		pLp = L.p * MLp * (T(2.0) - ML);
	} else {
		MLp = ML;
		pLp = L.p;
	}
	if (MR <= T(-1.0)) {
		pRm = R.p;
		MRm = MR;
	} else if (MR < T(1.0)) {
		MRm = T(-0.25) * (MR - T(1.0)) * (MR - T(1.0));
		pRm = -R.p * MRm * (T(2.0) + MR);
	} else {
		pRm = T(0);
		MRm = T(0);
	}
	const T M = MLp + MRm;
	const T hM = T(0.5) * M * nn, ps = (pLp + pRm) * nn;
	for (int k = 0; k < 5; k++) fc[k] = hM * (L.F[k] + R.F[k]);
	fc[1] += nx * ps;
	fc[2] += ny * ps;
	fc[3] += nz * ps;
	if (DISS) {
		const T delta = T(0.25);
		T Mf = M;
		if (!(tabs(Mf) > delta)) Mf = (Mf * Mf + delta * delta) / (T(2.0) * delta);
		const T ha = T(0.5) * tabs(Mf) * nn;
		for (int k = 0; k < 5; k++) fd[k] = ha * (R.F[k] - L.F[k]);
	}
}

// Pass 1 of a stage, one thread per real cell: gradient, limiter and MUSCL
// face states of the cell and of its ghost cells.  FIRST additionally computes
// W0 (unless carried) and the local time step from the stage-0 state.
// first stage only: W0 (unless carried) and the local time step (Timestep.cpp:26-148)
template <class T, int NSL>
__device__ __forceinline__ void first_stage_extras(const FusedView<T>& v, const Physics& ph, int carry_w0, int c) {
	const SlotRange<T, NSL> sr(v, c);
	const Q5<T> q0 = ld5(v.Pin, v.NA, c);
	const T V = v.vol[c];
	if (!carry_w0) {
		const int n = v.NR;
		v.W0[c] = (double)q0.r;
		v.W0[n + c] = (double)(q0.r * q0.u);
		v.W0[2 * n + c] = (double)(q0.r * q0.v);
		v.W0[3 * n + c] = (double)(q0.r * q0.w);
		v.W0[4 * n + c] = (double)(T(0.5) * q0.r * (q0.u * q0.u + q0.v * q0.v + q0.w * q0.w) +
		                           T(1.) / (T(ph.gamma) - T(1.0)) * q0.p);
	}
	T geo[MAXSL][4];
	load_geo<T, NSL>(v.sgeo, sr, geo);
	const T cc = tsqrt(T(ph.gamma) * q0.p / q0.r);
	T srad = T(0.0);
#pragma unroll
	E3D_SLOTS(k, sr) srad += (tabs((q0.u) * geo[k][0] + (q0.v) * geo[k][1] + (q0.w) * geo[k][2]) + (cc)) * geo[k][3];
	v.dt[c] = T(ph.cfl) * V / srad;
}

template <class T, int GRAD, int LIM, bool FIRST, int NSL>
__device__ __forceinline__ void recon_cell(const FusedView<T>& v, const Physics& ph, int carry_w0, int c) {
	const SlotRange<T, NSL> sr(v, c);
	const Q5<T> q0 = ld5(v.Pin, v.NA, c);
	int nb[MAXSL];
	load_int<T, NSL>(v.slot_nbr, sr, nb);
	T w[MAXSL][3];
	if (GRAD == GRAD_GREEN_GAUSS) load3<T, NSL>(v.sS, sr, w);
	else load3<T, NSL>(v.lsw, sr, w);
	T gr[5][3];
	for (int q = 0; q < 5; q++) gr[q][0] = gr[q][1] = gr[q][2] = T(0.0);
	Q5<T> mx = q0, mn = q0;
#pragma unroll
	E3D_SLOTS(k, sr) {
		const Q5<T> qn = ld5(v.Pin, v.NA, nb[k]);
		for (int q = 0; q < 5; q++) {
			if (GRAD == GRAD_GREEN_GAUSS) {
				// 0.5*(q_L+q_R)*(+-S): addition commutes, so owner/neighbour order is exact
				const T a = T(0.5) * (qv(q0, q) + qv(qn, q));
				gr[q][0] += a * w[k][0];
				gr[q][1] += a * w[k][1];
				gr[q][2] += a * w[k][2];
			} else {
				const T dq = qv(qn, q) - qv(q0, q);
				gr[q][0] += w[k][0] * dq;
				gr[q][1] += w[k][1] * dq;
				gr[q][2] += w[k][2] * dq;
			}
			if (qv(qn, q) > qv(mx, q)) qv(mx, q) = qv(qn, q);
			if (qv(qn, q) < qv(mn, q)) qv(mn, q) = qv(qn, q);
		}
	}
	const T V = v.vol[c];
	if (GRAD == GRAD_GREEN_GAUSS)
		for (int d = 0; d < 3; d++)
			for (int q = 0; q < 5; q++) gr[q][d] /= V;
	T rv[MAXSL][3];
	load3<T, NSL>(v.srv, sr, rv);
	const T eps2 = T(ph.k3) * V;
	if constexpr (sizeof(T) == 4 && NSL == 4) {
		// FP32: the face value q + phi (g.r) reuses the limiter's d2 = g.r
		Q5<T> fs[4];
		for (int q = 0; q < 5; q++) {
			const T dmax = qv(mx, q) - qv(q0, q), dmin = qv(mn, q) - qv(q0, q);
			T d2[4], phi = T(INFINITY);
#pragma unroll
			for (int k = 0; k < 4; k++) {
				d2[k] = gr[q][0] * rv[k][0];
				d2[k] += gr[q][1] * rv[k][1];
				d2[k] += gr[q][2] * rv[k][2];
				const T lf = (LIM == LIM_BARTH_JESPERSEN) ? limiter_bj_face(d2[k], dmax, dmin, T(ph.omega))
				                                          : limiter_venkat_face(d2[k], dmax, dmin, eps2);
				if (lf < phi) phi = lf;
			}
#pragma unroll
			for (int k = 0; k < 4; k++) qv(fs[k], q) = qv(q0, q) + phi * d2[k];
		}
#pragma unroll
		for (int k = 0; k < 4; k++) st5(v.FS, v.NS, sr.s0 + k, fs[k]);
	} else {
		// FP64 (and the generic slot path): the reference's accumulation order
		T phi[5];
		for (int q = 0; q < 5; q++) {
			const T dmax = qv(mx, q) - qv(q0, q), dmin = qv(mn, q) - qv(q0, q);
			phi[q] = T(INFINITY);
#pragma unroll
			E3D_SLOTS(k, sr) {
				T d2 = T(0.0);
				d2 += gr[q][0] * rv[k][0];
				d2 += gr[q][1] * rv[k][1];
				d2 += gr[q][2] * rv[k][2];
				const T lf = (LIM == LIM_BARTH_JESPERSEN) ? limiter_bj_face(d2, dmax, dmin, T(ph.omega))
				                                          : limiter_venkat_face(d2, dmax, dmin, eps2);
				if (lf < phi[q]) phi[q] = lf;
			}
		}
#pragma unroll
		E3D_SLOTS(k, sr) {
			Q5<T> fs;
			for (int q = 0; q < 5; q++)
				qv(fs, q) = recon(qv(q0, q), phi[q], gr[q][0], gr[q][1], gr[q][2], rv[k][0], rv[k][1], rv[k][2]);
			st5(v.FS, v.NS, sr.s0 + k, fs);
		}
	}
	// ghost cells of this cell's boundary faces: gradient (reflected or zero),
	// limiter (the ghost's only neighbour is c) and face state.  Later stages read
	// the slot neighbours again (a cache hit) rather than hold them through the
	// pass, which takes the FP32 pass from 32-68 bytes of spills to none; the
	// first stage spills less keeping them.
	if (!FIRST) load_int<T, NSL>(v.slot_nbr, sr, nb);
#pragma unroll
	E3D_SLOTS(k, sr) {
		if (nb[k] >= v.NR) {
			const int g = nb[k];
			int ms = v.slot_mate[sr.s0 + k];
			ms = ms >= 0 ? ms : ~ms;
			const Q5<T> qg = ld5(v.Pin, v.NA, g);
			const T nx = v.sgeo[4 * (size_t)(sr.s0 + k)], ny = v.sgeo[4 * (size_t)(sr.s0 + k) + 1],
			        nz = v.sgeo[4 * (size_t)(sr.s0 + k) + 2];
			const T g0 = v.srv[3 * (size_t)ms], g1 = v.srv[3 * (size_t)ms + 1], g2 = v.srv[3 * (size_t)ms + 2];
			const bool refl = v.grefl[g - v.NR] != 0;
			const T eps2g = T(ph.k3) * v.vol[g];
			Q5<T> fs;
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
				qv(fs, q) = recon(qv(qg, q), pg, gg[0], gg[1], gg[2], g0, g1, g2);
			}
			st5(v.FS, v.NS, ms, fs);
		}
	}
	if (FIRST) first_stage_extras<T, NSL>(v, ph, carry_w0, c);
}

// resident blocks per SM the FP32 reconstruction pass is compiled for (8: 64
// registers) and the FP64 stage passes (4: 128 registers)
#ifndef E3D_RECON_MIN_BLOCKS
#define E3D_RECON_MIN_BLOCKS 8
#endif
#ifndef E3D_FP64_MIN_BLOCKS
#define E3D_FP64_MIN_BLOCKS 4
#endif
template <class T, int GRAD, int LIM, bool FIRST, int NSL>
__global__ void __launch_bounds__(128, sizeof(T) == 4 ? E3D_RECON_MIN_BLOCKS : E3D_FP64_MIN_BLOCKS) k_recon(FusedView<T> v, Physics ph, int carry_w0) {
	const int c = blockIdx.x * blockDim.x + threadIdx.x;
	if (c < v.NR) recon_cell<T, GRAD, LIM, FIRST, NSL>(v, ph, carry_w0, c);
}

// FP64 reconstruction of the later stages with one lane per (cell, variable),
// all-tetrahedron meshes.  Gradient, limiter and face states of one variable
// depend on that variable alone, so five lanes per cell run the same
// per-variable arithmetic as recon_cell's FP64 branch, in the same order (bit
// for bit), with a fifth of its gradient/limiter state and the slot weights
// read per slot: 64 registers instead of 128, 30 resident warps per SM instead
// of 16.  A block covers RV_CELLS cells (5 * RV_CELLS threads, cell-major: the
// four lanes of a cell's (rho, u, v, w) read and write one 32-byte vector
// together).  Measured on B200 (3.07M tets, second order): 2.61 TB/s against
// 2.44 for the one-thread-per-cell pass.  The first stage keeps recon_cell: its
// time step and W0 need the whole cell, and one lane of five doing them made
// that pass slower (2.82 against 2.89 TB/s).
constexpr int RV_CELLS = 32;
#ifndef E3D_RV_MIN_BLOCKS
#define E3D_RV_MIN_BLOCKS 6
#endif

__device__ __forceinline__ double ldq(const double* __restrict__ P, int n, int c, int q) {
	return q < 4 ? P[4 * (size_t)c + q] : P[4 * (size_t)n + c];
}
__device__ __forceinline__ void stq(double* __restrict__ P, int n, int c, int q, double x) {
	if (q < 4) P[4 * (size_t)c + q] = x;
	else P[4 * (size_t)n + c] = x;
}

template <int GRAD, int LIM>
__global__ void __launch_bounds__(5 * RV_CELLS, E3D_RV_MIN_BLOCKS) k_recon_var(FusedView<double> v, Physics ph) {
	const int c = blockIdx.x * RV_CELLS + threadIdx.x / 5, q = threadIdx.x % 5;
	if (c >= v.NR) return;
	const SlotRange<double, 4> sr(v, c);
	const double q0 = ldq(v.Pin, v.NA, c, q);
	int nb[4];
	load_int<double, 4>(v.slot_nbr, sr, nb);
	double gr[3] = {0.0, 0.0, 0.0};
	double mx = q0, mn = q0;
	{
		const double* __restrict__ wa = (GRAD == GRAD_GREEN_GAUSS ? v.sS : v.lsw) + 3 * (size_t)sr.s0;
#pragma unroll
		for (int k = 0; k < 4; k++) {
			const double w[1][3] = {{__ldg(wa + 3 * k), __ldg(wa + 3 * k + 1), __ldg(wa + 3 * k + 2)}};
			const double qn = ldq(v.Pin, v.NA, nb[k], q);
			if (GRAD == GRAD_GREEN_GAUSS) {
				const double a = 0.5 * (q0 + qn);
				gr[0] += a * w[0][0];
				gr[1] += a * w[0][1];
				gr[2] += a * w[0][2];
			} else {
				const double dq = qn - q0;
				gr[0] += w[0][0] * dq;
				gr[1] += w[0][1] * dq;
				gr[2] += w[0][2] * dq;
			}
			if (qn > mx) mx = qn;
			if (qn < mn) mn = qn;
		}
	}
	const double V = v.vol[c];
	if (GRAD == GRAD_GREEN_GAUSS)
		for (int d = 0; d < 3; d++) gr[d] /= V;
	const double* __restrict__ ra = v.srv + 3 * (size_t)sr.s0;
	const double eps2 = ph.k3 * V;
	const double dmax = mx - q0, dmin = mn - q0;
	double phi = INFINITY;
#pragma unroll
	for (int k = 0; k < 4; k++) {
		double d2 = 0.0;
		d2 += gr[0] * __ldg(ra + 3 * k);
		d2 += gr[1] * __ldg(ra + 3 * k + 1);
		d2 += gr[2] * __ldg(ra + 3 * k + 2);
		const double lf = (LIM == LIM_BARTH_JESPERSEN) ? limiter_bj_face(d2, dmax, dmin, ph.omega)
		                                               : limiter_venkat_face(d2, dmax, dmin, eps2);
		if (lf < phi) phi = lf;
	}
#pragma unroll
	for (int k = 0; k < 4; k++)
		stq(v.FS, v.NS, sr.s0 + k, q,
		    recon(q0, phi, gr[0], gr[1], gr[2], __ldg(ra + 3 * k), __ldg(ra + 3 * k + 1), __ldg(ra + 3 * k + 2)));
	// ghost cells of this cell's boundary faces (recon_cell's tail, one variable)
#pragma unroll
	for (int k = 0; k < 4; k++) {
		if (nb[k] < v.NR) continue;
		const int g = nb[k];
		int ms = v.slot_mate[sr.s0 + k];
		ms = ms >= 0 ? ms : ~ms;
		const double qg = ldq(v.Pin, v.NA, g, q);
		const double* n = v.sgeo + 4 * (size_t)(sr.s0 + k);
		const double g0 = v.srv[3 * (size_t)ms], g1 = v.srv[3 * (size_t)ms + 1], g2 = v.srv[3 * (size_t)ms + 2];
		double gg[3] = {0.0, 0.0, 0.0};
		if (v.grefl[g - v.NR] != 0) reflect_grad(gr, n[0], n[1], n[2], gg);
		double gmx = qg, gmn = qg;
		if (q0 > gmx) gmx = q0;
		if (q0 < gmn) gmn = q0;
		double d2 = 0.0;
		d2 += gg[0] * g0;
		d2 += gg[1] * g1;
		d2 += gg[2] * g2;
		const double dmx = gmx - qg, dmn = gmn - qg;
		const double lf = (LIM == LIM_BARTH_JESPERSEN) ? limiter_bj_face(d2, dmx, dmn, ph.omega)
		                                               : limiter_venkat_face(d2, dmx, dmn, ph.k3 * v.vol[g]);
		double pg = INFINITY;
		if (lf < pg) pg = lf;
		stq(v.FS, v.NS, ms, q, recon(qg, pg, gg[0], gg[1], gg[2], g0, g1, g2));
	}
}

// W0 and the local time step without a reconstruction pass (first order).
template <class T, int NSL>
__device__ __forceinline__ void start_cell(const FusedView<T>& v, const Physics& ph, int carry_w0, int c) {
	const SlotRange<T, NSL> sr(v, c);
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
	T geo[MAXSL][4];
	load_geo<T, NSL>(v.sgeo, sr, geo);
	const T cc = tsqrt(T(ph.gamma) * q0.p / q0.r);
	T srad = T(0.0);
#pragma unroll
	E3D_SLOTS(k, sr) srad += (tabs((q0.u) * geo[k][0] + (q0.v) * geo[k][1] + (q0.w) * geo[k][2]) + (cc)) * geo[k][3];
	v.dt[c] = T(ph.cfl) * v.vol[c] / srad;
}

template <class T, int NSL>
__global__ void __launch_bounds__(128) k_start(FusedView<T> v, Physics ph, int carry_w0) {
	const int c = blockIdx.x * blockDim.x + threadIdx.x;
	if (c < v.NR) start_cell<T, NSL>(v, ph, carry_w0, c);
}

// Pass 2 of a stage, one thread per real cell: convective and dissipative
// fluxes of each face (computed identically from both sides), residual gather,
// conservative update into Pout and the ghost states of the cell's boundary
// faces.  ORDER1 reads cell states directly (first order).  LAST stores the
// final conservative state as the next W0 when carry_w0 is set.
//
// DISS = false is used for stages with beta = 0: the reference still evaluates
// the dissipative flux (its guard is always true) but Rd*(1-0) + sum(D*0) equals
// Rd for finite fluxes, so the flux and the Rd store are skipped.  Rc is stored
// only at the last stage, the one the norms (and callers) read.
template <class T, int SCHEME, bool ORDER1, int NSL, bool DISS>
__device__ __forceinline__ void flux_update_cell(const FusedView<T>& v, const Physics& ph, T alpha, T beta, int last,
                                                 int carry_w0, int c) {
	const SlotRange<T, NSL> sr(v, c);
	const T g = T(ph.gamma), gr = T(ph.gr), gm1 = T(ph.gm1);
	int mate[MAXSL];
	load_int<T, NSL>(v.slot_mate, sr, mate);
	T ac[5], ad[5];
	for (int q = 0; q < 5; q++) {
		ac[q] = T(0.0);
		ad[q] = DISS ? v.Rd[q * v.NR + c] * (T(1.0) - beta) : v.Rd[q * v.NR + c];
	}
	Q5<T> qc;
	int nb[MAXSL];
	if (ORDER1) {
		qc = ld5(v.Pin, v.NA, c);
		load_int<T, NSL>(v.slot_nbr, sr, nb);
	}
#ifdef E3D_SHARED_SIDES
	constexpr bool shared_sides = ORDER1 && SCHEME == FLUX_AUSM;
	AusmSide<T> own;
	if constexpr (shared_sides) own = ausm_side(qc, g, gr);
#endif
	T geo[MAXSL][4];
	load_geo<T, NSL>(v.sgeo, sr, geo);
#pragma unroll
	E3D_SLOTS(k, sr) {
		const bool left = mate[k] >= 0;
		const int m = left ? mate[k] : ~mate[k];
		Q5<T> qo, qn;
		if (ORDER1) {
			qo = qc;
			qn = ld5(v.Pin, v.NA, nb[k]);
		} else {
			qo = ld5(v.FS, v.NS, sr.s0 + k);
			qn = ld5(v.FS, v.NS, m);
		}
		Q5<T> L, R;
		for (int q = 0; q < 5; q++) {
			qv(L, q) = left ? qv(qo, q) : qv(qn, q);
			qv(R, q) = left ? qv(qn, q) : qv(qo, q);
		}
		T fc[5], fd[5];
#ifdef E3D_SHARED_SIDES
		if constexpr (shared_sides) {
			const AusmSide<T> nbr = ausm_side(qn, g, gr);
			// sides selected by value: a branch on the orientation would run the
			// face arithmetic twice in warps whose cells differ
			ausm_face_sides<T, DISS>(left ? own : nbr, left ? nbr : own, geo[k][0], geo[k][1], geo[k][2], geo[k][3],
			                         fc, fd);
		} else
#endif
		if (SCHEME == FLUX_ROE) {
			flux_central(L, R, geo[k][0], geo[k][1], geo[k][2], geo[k][3], gr, fc);
			if (DISS) flux_roe_diss(L, R, geo[k][0], geo[k][1], geo[k][2], geo[k][3], gr, gm1, fd);
		} else {
			flux_ausm_conv(L, R, geo[k][0], geo[k][1], geo[k][2], geo[k][3], g, gr, fc);
			if (DISS) flux_ausm_diss(L, R, geo[k][0], geo[k][1], geo[k][2], geo[k][3], g, gr, fd);
		}
		if (left) {
			for (int q = 0; q < 5; q++) {
				ac[q] += fc[q];
				if (DISS) ad[q] += fd[q] * beta;
			}
		} else {
			for (int q = 0; q < 5; q++) {
				ac[q] -= fc[q];
				if (DISS) ad[q] -= fd[q] * beta;
			}
		}
	}
	double w0[5], wn[5];
	for (int q = 0; q < 5; q++) {
		if (last) v.Rc[q * v.NR + c] = ac[q];
		if (DISS) v.Rd[q * v.NR + c] = ad[q];
		w0[q] = v.W0[q * v.NR + c];
	}
	const T coef = alpha * v.dt[c] / v.vol[c];
	const Q5<T> qnew = conservative_update<T>(w0, coef, ac, ad, gm1, wn);
	st5(v.Pout, v.NA, c, qnew);
	if (last && carry_w0)
		for (int q = 0; q < 5; q++) v.W0[q * v.NR + c] = wn[q];
	if (!ORDER1) load_int<T, NSL>(v.slot_nbr, sr, nb);
#pragma unroll
	E3D_SLOTS(k, sr) {
		if (nb[k] >= v.NR) {
			const int gi = nb[k] - v.NR;
			const int kind = v.gkind[gi];
			if (kind != GK_NONE) {
				// freestream of the ghost's case (batched cases differ in Mach and alpha)
				const double* f = v.case_free ? v.case_free + 5 * v.gcase[gi] : ph.free;
				Q5<T> fr;
				fr.r = T(f[0]);
				fr.u = T(f[1]);
				fr.v = T(f[2]);
				fr.w = T(f[3]);
				fr.p = T(f[4]);
				// the face normal is read again here (boundary slots only) so that the
				// slots' geometry need not stay live through the update
				const T* n = v.sgeo + 4 * (size_t)(sr.s0 + k);
				st5(v.Pout, v.NA, nb[k], ghost_state(kind, qnew, fr, n[0], n[1], n[2], g));
			}
		}
	}
}

template <class T, int SCHEME, bool ORDER1, int NSL, bool DISS>
__global__ void __launch_bounds__(128, sizeof(T) == 4 ? 8 : E3D_FP64_MIN_BLOCKS) k_flux_update(FusedView<T> v, Physics ph, T alpha, T beta, int last, int carry_w0) {
	const int c = blockIdx.x * blockDim.x + threadIdx.x;
	if (c < v.NR) flux_update_cell<T, SCHEME, ORDER1, NSL, DISS>(v, ph, alpha, beta, last, carry_w0, c);
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

// Wall pressure forces (AerodynamicParameters::computeAerodynamic,
// AerodynamicParameters.cpp:189-232) in two passes that keep the reference's
// sequential wall-face order: per-face terms in parallel, then one ordered sum
// per block and component from shared memory.
// terms[q*nwall + i], q = fy, fx, cmx, cmy, cmz of wall face i.
template <class T>
__global__ void k_wall_terms(const T* __restrict__ P, int NA, int nwall, const int* __restrict__ wall_face,
                             const int* __restrict__ face_lr, const double* __restrict__ S,
                             const double* __restrict__ fc, double denom, const double* __restrict__ wall_denom,
                             double* __restrict__ terms) {
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= nwall) return;
	const int f = wall_face[i];
	const double p0 = (double)P[4 * (size_t)NA + face_lr[2 * f]], p1 = (double)P[4 * (size_t)NA + face_lr[2 * f + 1]];
	const double pbc = 0.5 * (p0 + p1);
	const double cp = (pbc - 1.) / (wall_denom ? wall_denom[i] : denom);
	const double fx = cp * S[3 * f], fy = cp * S[3 * f + 1], fz = cp * S[3 * f + 2];
	const double x = fc[3 * f], y = fc[3 * f + 1], z = fc[3 * f + 2];
	terms[i] = fy;
	terms[(size_t)nwall + i] = fx;
	terms[2 * (size_t)nwall + i] = y * fz - z * fy;
	terms[3 * (size_t)nwall + i] = z * fx - x * fz;
	terms[4 * (size_t)nwall + i] = x * fy - y * fx;
}

// hist[iter*stride + b*10 + 5 + q] = sum of terms q over block b's wall faces, in order.
constexpr int WALL_CHUNK = 1024;
__global__ void __launch_bounds__(128) k_wall_sums(const double* __restrict__ terms, int nwall,
                                                   const int* __restrict__ wall_off, double* __restrict__ hist,
                                                   int stride, const int* __restrict__ d_iter) {
	__shared__ double buf[5][WALL_CHUNK];
	const int b = blockIdx.x;
	const int beg = wall_off[b], end = wall_off[b + 1];
	double acc = 0.;
	for (int base = beg; base < end; base += WALL_CHUNK) {
		const int n = min(WALL_CHUNK, end - base);
		for (int j = threadIdx.x; j < 5 * n; j += blockDim.x) {
			const int q = j / n, i = j - q * n;
			buf[q][i] = terms[(size_t)q * nwall + base + i];
		}
		__syncthreads();
		if (threadIdx.x < 5)
			for (int i = 0; i < n; i++) acc += buf[threadIdx.x][i];
		__syncthreads();
	}
	if (threadIdx.x < 5) hist[(size_t)(*d_iter) * stride + b * 10 + 5 + threadIdx.x] = acc;
}

__global__ void k_iter_advance(int* d_iter) { *d_iter += 1; }


// ===================================================================== batches
// Phases of one outer iteration over a work list (tiles of real cells of the
// active cases), shared by the persistent kernel and the tiled per-pass
// kernels.  TPB threads cooperate on one tile.

// Sum of (Rc-Rd)^2 over the cells of tile w, fixed tree order (red: [5][TPB]).
template <class T, int TPB>
__device__ __forceinline__ void tile_norms(const FusedView<T>& vf, const PersistArgs& a, int w, double (*red)[TPB]) {
	const int4 t = a.work[w];
	double acc[5] = {0., 0., 0., 0., 0.};
	for (int c = t.x + threadIdx.x; c < t.y; c += TPB)
		for (int q = 0; q < 5; q++) {
			const double r = (double)vf.Rc[q * vf.NR + c] - (double)vf.Rd[q * vf.NR + c];
			acc[q] += r * r;
		}
	for (int q = 0; q < 5; q++) red[q][threadIdx.x] = acc[q];
	__syncthreads();
	for (int h = TPB / 2; h > 0; h >>= 1) {
		if (threadIdx.x < h)
			for (int q = 0; q < 5; q++) red[q][threadIdx.x] += red[q][threadIdx.x + h];
		__syncthreads();
	}
	if (threadIdx.x < 5) a.wpart[(size_t)w * 5 + threadIdx.x] = red[threadIdx.x][0];
	__syncthreads();
}

// Force terms of wall faces i0, i0+stride, ... (frozen cases included: cheap, ignored by the host).
template <class T>
__device__ __forceinline__ void wall_terms_range(const FusedView<T>& vf, const PersistArgs& a, int i0, int stride) {
	for (int i = i0; i < a.n_wall; i += stride) {
		const int f = a.wall_face[i];
		const size_t i0 = 4 * (size_t)vf.NA + a.face_lr[2 * f], i1 = 4 * (size_t)vf.NA + a.face_lr[2 * f + 1];
		double p0 = (double)vf.Pin[i0], p1 = (double)vf.Pin[i1];
		if (a.Pb64) {  // difference form: base + difference
			p0 += a.Pb64[i0];
			p1 += a.Pb64[i1];
		}
		const double cp = (0.5 * (p0 + p1) - 1.) / (a.wall_denom ? a.wall_denom[i] : a.denom);
		const double fx = cp * a.S[3 * f], fy = cp * a.S[3 * f + 1], fz = cp * a.S[3 * f + 2];
		const double x = a.fc[3 * f], y = a.fc[3 * f + 1], z = a.fc[3 * f + 2];
		a.wall_terms[i] = fy;
		a.wall_terms[(size_t)a.n_wall + i] = fx;
		a.wall_terms[2 * (size_t)a.n_wall + i] = y * fz - z * fy;
		a.wall_terms[3 * (size_t)a.n_wall + i] = z * fx - x * fz;
		a.wall_terms[4 * (size_t)a.n_wall + i] = x * fy - y * fx;
	}
}

// Inter-block halo copies i0, i0+stride, ... into both primitive buffers.
template <class T>
__device__ __forceinline__ void halo_range(const FusedView<T>& vf, const PersistArgs& a, int i0, int stride) {
	for (int i = i0; i < a.n_halo; i += stride) {
		const Q5<T> q = ld5(vf.Pin, vf.NA, a.halo_src[i]);
		st5(const_cast<T*>(vf.Pin), vf.NA, a.halo_dst[i], q);
		st5(vf.Pout, vf.NA, a.halo_dst[i], q);
	}
}

// Per-block sums of block b into history slot `slot`: tiles in a fixed tree
// order, wall faces sequentially in the reference's order.
template <int TPB>
__device__ __forceinline__ void block_sums(const PersistArgs& a, int b, int slot, double (*red)[TPB],
                                           double (*wbuf)[WALL_CHUNK / 4]) {
	const int w0 = a.block_work[b], w1 = a.block_work[b + 1];
	double acc[5] = {0., 0., 0., 0., 0.};
	for (int w = w0 + threadIdx.x; w < w1; w += TPB)
		for (int q = 0; q < 5; q++) acc[q] += a.wpart[(size_t)w * 5 + q];
	for (int q = 0; q < 5; q++) red[q][threadIdx.x] = acc[q];
	__syncthreads();
	for (int h = TPB / 2; h > 0; h >>= 1) {
		if (threadIdx.x < h)
			for (int q = 0; q < 5; q++) red[q][threadIdx.x] += red[q][threadIdx.x + h];
		__syncthreads();
	}
	double* out = a.hist + (size_t)slot * a.stride + b * 10;
	if (threadIdx.x < 5) {
		out[threadIdx.x] = red[threadIdx.x][0];
		if (!isfinite(red[threadIdx.x][0]) && w1 > w0) *a.d_bad = 1;
	}
	const int beg = a.wall_off[b], end = a.wall_off[b + 1];
	double fs = 0.;
	constexpr int CH = WALL_CHUNK / 4;
	for (int base_i = beg; base_i < end; base_i += CH) {
		const int n = min(CH, end - base_i);
		__syncthreads();
		for (int j = threadIdx.x; j < 5 * n; j += TPB) {
			const int q = j / n, i = j - q * n;
			wbuf[q][i] = a.wall_terms[(size_t)q * a.n_wall + base_i + i];
		}
		__syncthreads();
		if (threadIdx.x < 5)
			for (int i = 0; i < n; i++) fs += wbuf[threadIdx.x][i];
	}
	if (threadIdx.x < 5) out[5 + threadIdx.x] = fs;
	__syncthreads();
}

// Persistent form: one cooperative launch runs `iters` outer iterations;
// phases are separated by grid-wide barriers.  Tiles of converged cases are
// absent from the work list.
template <class T, int GRAD, int LIM, int SCHEME, bool ORDER2, int TPB>
__global__ void __launch_bounds__(TPB, 512 / TPB) k_persistent(FusedView<T> v0, FusedView<T> v1, Physics ph,
                                                               PersistArgs a) {
	namespace cg = cooperative_groups;
	cg::grid_group grid = cg::this_grid();
	__shared__ double red[5][TPB];
	__shared__ double wbuf[5][WALL_CHUNK / 4];
	const int base = *a.d_iter;
	int parity = a.start_parity;  // which primitive buffer holds the current state
	for (int it = 0; it < a.iters; it++) {
		for (int s = 0; s < a.stages; s++) {
			const FusedView<T>& v = parity ? v1 : v0;
			if (ORDER2 || s == 0) {
				for (int w = blockIdx.x; w < a.n_work; w += gridDim.x) {
					const int4 t = a.work[w];
					for (int c = t.x + threadIdx.x; c < t.y; c += TPB) {
						if (ORDER2) {
							if (s == 0) recon_cell<T, GRAD, LIM, true, 4>(v, ph, a.carry, c);
							else recon_cell<T, GRAD, LIM, false, 4>(v, ph, a.carry, c);
						} else {
							start_cell<T, 4>(v, ph, a.carry, c);
						}
					}
				}
				grid.sync();
			}
			const T al = T(a.alpha[s]), be = T(a.beta[s]);
			const int last = s == a.stages - 1;
			for (int w = blockIdx.x; w < a.n_work; w += gridDim.x) {
				const int4 t = a.work[w];
				for (int c = t.x + threadIdx.x; c < t.y; c += TPB) {
					if (a.beta[s] != 0.0) flux_update_cell<T, SCHEME, !ORDER2, 4, true>(v, ph, al, be, last, a.carry, c);
					else flux_update_cell<T, SCHEME, !ORDER2, 4, false>(v, ph, al, be, last, a.carry, c);
				}
			}
			grid.sync();
			parity ^= 1;
		}
		const FusedView<T>& vf = parity ? v1 : v0;  // Pin of the next stage = current state
		for (int w = blockIdx.x; w < a.n_work; w += gridDim.x) tile_norms<T, TPB>(vf, a, w, red);
		wall_terms_range(vf, a, blockIdx.x * TPB + threadIdx.x, gridDim.x * TPB);
		halo_range(vf, a, blockIdx.x * TPB + threadIdx.x, gridDim.x * TPB);
		grid.sync();
		const int slot = min(base + it, a.hist_capacity - 1);
		for (int b = blockIdx.x; b < a.nblocks; b += gridDim.x) block_sums<TPB>(a, b, slot, red, wbuf);
		grid.sync();
	}
	if (blockIdx.x == 0 && threadIdx.x == 0) *a.d_iter = base + a.iters;
}

// Tiled per-pass form: the same phases as separate launches over the work
// list (one block of 128 threads per tile of at most 128 cells), captured in a
// CUDA graph by the host.  Each pass keeps only its own registers and shared
// memory, so more warps stay resident than in the persistent kernel.
template <class T, int GRAD, int LIM, bool FIRST>
__global__ void __launch_bounds__(128, sizeof(T) == 4 ? 8 : 4) k_recon_tiles(FusedView<T> v, Physics ph, int carry_w0,
                                                                             const int4* __restrict__ work) {
	const int4 t = work[blockIdx.x];
	const int c = t.x + threadIdx.x;
	if (c < t.y) recon_cell<T, GRAD, LIM, FIRST, 4>(v, ph, carry_w0, c);
}

template <class T>
__global__ void __launch_bounds__(128) k_start_tiles(FusedView<T> v, Physics ph, int carry_w0,
                                                     const int4* __restrict__ work) {
	const int4 t = work[blockIdx.x];
	const int c = t.x + threadIdx.x;
	if (c < t.y) start_cell<T, 4>(v, ph, carry_w0, c);
}

template <class T, int SCHEME, bool ORDER1, bool DISS>
__global__ void __launch_bounds__(128, sizeof(T) == 4 ? 8 : 4) k_flux_update_tiles(FusedView<T> v, Physics ph, T alpha,
                                                                                   T beta, int last, int carry_w0,
                                                                                   const int4* __restrict__ work) {
	const int4 t = work[blockIdx.x];
	const int c = t.x + threadIdx.x;
	if (c < t.y) flux_update_cell<T, SCHEME, ORDER1, 4, DISS>(v, ph, alpha, beta, last, carry_w0, c);
}

// end of an iteration, part 1 (grid = n_work): tile norms, wall terms, halo
template <class T>
__global__ void __launch_bounds__(128) k_iter_tail(FusedView<T> vf, PersistArgs a) {
	__shared__ double red[5][128];
	tile_norms<T, 128>(vf, a, blockIdx.x, red);
	wall_terms_range(vf, a, blockIdx.x * 128 + threadIdx.x, gridDim.x * 128);
	halo_range(vf, a, blockIdx.x * 128 + threadIdx.x, gridDim.x * 128);
}

// end of an iteration, part 2 (grid = nblocks): per-block sums into history slot *d_iter + it
__global__ void __launch_bounds__(128) k_iter_sums(PersistArgs a, int it) {
	__shared__ double red[5][128];
	__shared__ double wbuf[5][WALL_CHUNK / 4];
	const int slot = min(*a.d_iter + it, a.hist_capacity - 1);
	block_sums<128>(a, blockIdx.x, slot, red, wbuf);
}

__global__ void k_iter_add(int* d_iter, int n) { *d_iter += n; }

}  // namespace
}  // namespace e3d
