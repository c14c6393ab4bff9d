// FP32 iterations in difference form (defect correction) for the FP64
// finishing phase of batched first-order AUSM solves.
//
// The FP32 variant's residual stops dropping near 5 orders: each face flux
// F(q) is O(1) and carries FP32 rounding of that size, and a converged cell's
// residual is the near-cancelling sum of such fluxes.  Here the state is split
// into a base state q_b, fixed between rebases and held in FP64, and an FP32
// difference d = q - q_b.  The residual is
//
//     R(q) = R64(q_b) + [R(q_b + d) - R(q_b)],
//
// where R64(q_b) is evaluated once per rebase in FP64 (k_base_residual) and the
// bracket is evaluated per stage in FP32 by algebra in which every term carries
// a factor of the difference (ausm_delta_face): (a+da)(b+db) - ab = da(b+db) +
// a db, sqrt(x+dx) - sqrt(x) = dx / (sqrt(x+dx) + sqrt(x)), and so on.  The
// rounding of the bracket is then FP32 rounding of the *change* of each face
// flux since the base, not of the flux itself, so the residual keeps falling
// below the FP32 floor; rebasing every few dozen iterations keeps the
// differences, and hence their rounding, small against the residual.
//
// The reference's AUSM (AusmScheme.cpp:12-243, 716-871) has branches: the
// Mach and pressure splits at |M| = 1 and the |M| <= 0.25 fix of the
// dissipation.  All are continuous functions of M, so a difference across a
// branch point is summed piece by piece through the branch point
// (piecewise_delta), each piece again a small difference.
//
// Conserved differences dW = W - W_b are carried in FP32 across iterations (the
// base W_b is FP64, in the engine's W0 array); primitives follow from them in
// difference form too.  Boundary ghost states are evaluated in FP64 from the
// cell's full FP64 state (base + difference) with the FP64 face normals, the
// same arithmetic that gives the ghost's base state, so their difference is
// exact to FP32 rounding of the difference.
//
// The discrete equations are the reference's; the converged state is the
// FP64 path's converged state to the accuracy of the FP64 base residual.  The
// iterates are not bit-identical to the reference's.
#include "launch_common.cuh"

namespace e3d {
namespace {

// ------------------------------------------------------------ face flux in difference form

// One cell's state as base primitives + differences, with the quantities of
// the AUSM flux that do not depend on the face: enthalpy, speed of sound and
// rho c as base value + difference (the normal Mach number is formed per face).
struct DCell {
	float u, v, w, p;
	float du, dv, dw, dp;
	float H, dH;
	float dc, ic, ic1;  // c' - c, 1/c, 1/c'
	float F1, dF1;      // rho c
};

__device__ __forceinline__ DCell dcell(const Q5<float>& b, const Q5<float>& d, float g, float gr) {
	DCell s;
	s.u = b.u;
	s.v = b.v;
	s.w = b.w;
	s.p = b.p;
	s.du = d.u;
	s.dv = d.v;
	s.dw = d.w;
	s.dp = d.p;
	const float qq = b.u * b.u + b.v * b.v + b.w * b.w;
	const float dqq = d.u * (2.f * b.u + d.u) + d.v * (2.f * b.v + d.v) + d.w * (2.f * b.w + d.w);
	const float ir = 1.f / b.r;
	const float pr = b.p * ir;
	const float dpr = (d.p - pr * d.r) / (b.r + d.r);  // p'/r' - p/r
	s.H = 0.5f * qq + gr * pr;
	s.dH = 0.5f * dqq + gr * dpr;
	const float x = g * pr, x1 = g * (pr + dpr);
	s.ic = rsqrtf(x);  // 1/c, and c = x/c: one reciprocal square root for both
	s.ic1 = rsqrtf(x1);
	const float c = x * s.ic, c1 = x1 * s.ic1;
	s.dc = g * dpr / (c + c1);
	s.F1 = b.r * c;
	s.dF1 = d.r * c1 + b.r * s.dc;
	return s;
}

// normal Mach number of a cell at a face: M = V/c and M' - M = (dV - M dc)/c'
__device__ __forceinline__ void dmach(const DCell& s, float nx, float ny, float nz, float& M, float& dM) {
	const float V = s.u * nx + s.v * ny + s.w * nz;
	const float dV = s.du * nx + s.dv * ny + s.dw * nz;
	M = V * s.ic;
	dM = (dV - M * s.dc) * s.ic1;
}

// F = (rho c, rho u c, rho v c, rho w c, rho H c) of one side and its difference
__device__ __forceinline__ void side_flux(const DCell& s, float F[5], float dF[5]) {
	F[0] = s.F1;
	dF[0] = s.dF1;
	F[1] = s.F1 * s.u;
	dF[1] = s.dF1 * (s.u + s.du) + s.F1 * s.du;
	F[2] = s.F1 * s.v;
	dF[2] = s.dF1 * (s.v + s.dv) + s.F1 * s.dv;
	F[3] = s.F1 * s.w;
	dF[3] = s.dF1 * (s.w + s.dw) + s.F1 * s.dw;
	F[4] = s.F1 * s.H;
	dF[4] = s.dF1 * (s.H + s.dH) + s.F1 * s.dH;
}

// f(x + d) - f(x) for a continuous function of three pieces split at lo < hi;
// i0, i1 are the pieces of x and x + d (by the reference's branch tests) and
// piece(i, x0, e) = f_i(x0 + e) - f_i(x0) on piece i.  Across branch points
// the difference is summed through them, so every term stays a difference.
template <class P>
__device__ __forceinline__ float piecewise_delta(float x, float d, float lo, float hi, int i0, int i1, P piece) {
	if (i0 == i1) return piece(i0, x, d);
	float acc = 0.f, x0 = x, rest = d;
	if (i1 > i0) {
		for (int i = i0; i < i1; i++) {
			const float bp = i == 0 ? lo : hi;
			const float e = bp - x0;
			acc += piece(i, x0, e);
			rest -= e;
			x0 = bp;
		}
	} else {
		for (int i = i0; i > i1; i--) {
			const float bp = i == 2 ? hi : lo;
			const float e = bp - x0;
			acc += piece(i, x0, e);
			rest -= e;
			x0 = bp;
		}
	}
	return acc + piece(i1, x0, rest);
}

// branch of the Mach / pressure splits (AusmScheme.cpp:777-833): M <= -1, -1 < M < 1, M >= 1
__device__ __forceinline__ int split_piece(float M) { return M <= -1.f ? 0 : (M < 1.f ? 1 : 2); }
// branch of the dissipation's |M| with the |M| <= 0.25 fix (AusmScheme.cpp:201-209)
__device__ __forceinline__ int fix_piece(float M) { return M < -0.25f ? 0 : (M <= 0.25f ? 1 : 2); }

// Difference of the AUSM convective (fc) and dissipative (fd, when DISS) face
// fluxes between the states (bL+dL, bR+dR) and (bL, bR).
template <bool DISS>
__device__ __forceinline__ void ausm_delta_face(const DCell& L, const DCell& R, float nx, float ny, float nz, float nn,
                                                float fc[5], float fd[5]) {
	float LM, LdM, RM, RdM;
	dmach(L, nx, ny, nz, LM, LdM);
	dmach(R, nx, ny, nz, RM, RdM);
	// plus splits of the left state
	const int iL0 = split_piece(LM), iL1 = split_piece(LM + LdM);
	const float MLp = iL0 == 0 ? 0.f : (iL0 == 1 ? 0.25f * (LM + 1.f) * (LM + 1.f) : LM);
	const float PLp = iL0 == 0 ? 0.f : (iL0 == 1 ? 0.25f * (LM + 1.f) * (LM + 1.f) * (2.f - LM) : 1.f);
	const float dMLp = piecewise_delta(LM, LdM, -1.f, 1.f, iL0, iL1, [](int i, float x, float e) {
		return i == 0 ? 0.f : (i == 1 ? 0.25f * e * (2.f * (x + 1.f) + e) : e);
	});
	const float dPLp = piecewise_delta(LM, LdM, -1.f, 1.f, iL0, iL1, [](int i, float x, float e) {
		return i == 1 ? 0.25f * e * (3.f - 3.f * x * x - 3.f * x * e - e * e) : 0.f;
	});
	// minus splits of the right state
	const int iR0 = split_piece(RM), iR1 = split_piece(RM + RdM);
	const float MRm = iR0 == 0 ? RM : (iR0 == 1 ? -0.25f * (RM - 1.f) * (RM - 1.f) : 0.f);
	const float PRm = iR0 == 0 ? 1.f : (iR0 == 1 ? 0.25f * (1.f - RM) * (1.f - RM) * (2.f + RM) : 0.f);
	const float dMRm = piecewise_delta(RM, RdM, -1.f, 1.f, iR0, iR1, [](int i, float x, float e) {
		return i == 0 ? e : (i == 1 ? -0.25f * e * (2.f * (x - 1.f) + e) : 0.f);
	});
	const float dPRm = piecewise_delta(RM, RdM, -1.f, 1.f, iR0, iR1, [](int i, float x, float e) {
		return i == 1 ? 0.25f * e * (-3.f + 3.f * x * x + 3.f * x * e + e * e) : 0.f;
	});
	const float M = MLp + MRm, dM = dMLp + dMRm;
	const float dpLp = L.dp * (PLp + dPLp) + L.p * dPLp;  // (p P)' - p P
	const float dpRm = R.dp * (PRm + dPRm) + R.p * dPRm;
	float FL[5], dFL[5], FR[5], dFR[5];
	side_flux(L, FL, dFL);
	side_flux(R, FR, dFR);
	const float h = 0.5f * nn;
#pragma unroll
	for (int k = 0; k < 5; k++) {
		const float S = FL[k] + FR[k], dS = dFL[k] + dFR[k];
		fc[k] = h * (dM * (S + dS) + M * dS);  // 0.5 M (FL+FR) |S|
	}
	const float dps = (dpLp + dpRm) * nn;
	fc[1] += nx * dps;
	fc[2] += ny * dps;
	fc[3] += nz * dps;
	if (DISS) {
		const int j0 = fix_piece(M), j1 = fix_piece(M + dM);
		const float aM = j0 == 0 ? -M : (j0 == 1 ? (M * M + 0.0625f) * 2.f : M);
		const float daM = piecewise_delta(M, dM, -0.25f, 0.25f, j0, j1, [](int i, float x, float e) {
			return i == 0 ? -e : (i == 1 ? 2.f * e * (2.f * x + e) : e);
		});
#pragma unroll
		for (int k = 0; k < 5; k++) {
			const float D = FR[k] - FL[k], dD = dFR[k] - dFL[k];
			fd[k] = h * (daM * (D + dD) + aM * dD);  // 0.5 |M| (FR-FL) |S|
		}
	}
}

// Primitive differences from conserved differences dw = W - W_b, with b the
// base primitives of W_b: u = m/rho, p = (gamma-1)(rhoE - rho q^2/2).
__device__ __forceinline__ Q5<float> prim_delta(const Q5<float>& b, const float dw[5], float gm1) {
	Q5<float> d;
	const float r1 = b.r + dw[0];
	d.r = dw[0];
	d.u = (dw[1] - b.u * dw[0]) / r1;
	d.v = (dw[2] - b.v * dw[0]) / r1;
	d.w = (dw[3] - b.w * dw[0]) / r1;
	const float u1 = b.u + d.u, v1 = b.v + d.v, w1 = b.w + d.w;
	const float dqq = d.u * (b.u + u1) + d.v * (b.v + v1) + d.w * (b.w + w1);
	d.p = gm1 * (dw[4] - 0.5f * (dw[0] * (u1 * u1 + v1 * v1 + w1 * w1) + b.r * dqq));
	return d;
}

__device__ __forceinline__ Q5<double> freestream64(const FusedView<float>& v, const Physics& ph, int gi) {
	const double* f = v.case_free ? v.case_free + 5 * v.gcase[gi] : ph.free;
	return Q5<double>{f[0], f[1], f[2], f[3], f[4]};
}

// ------------------------------------------------------------ stage kernels (tiles of real cells)

// stage 0: local time step from the full state (W is carried, no W0 pass)
__global__ void __launch_bounds__(128) k_delta_start_tiles(FusedView<float> v, Physics ph,
                                                           const int4* __restrict__ work) {
	const int4 t = work[blockIdx.x];
	const int c = t.x + threadIdx.x;
	if (c >= t.y) return;
	const Q5<float> b = ld5(v.Pb, v.NA, c), d = ld5(v.Pin, v.NA, c);
	const Q5<float> q{b.r + d.r, b.u + d.u, b.v + d.v, b.w + d.w, b.p + d.p};
	const float4* geo = reinterpret_cast<const float4*>(v.sgeo) + 4 * (size_t)c;
	const float cc = sqrtf(float(ph.gamma) * q.p / q.r);
	float srad = 0.f;
#pragma unroll
	for (int k = 0; k < 4; k++) {
		const float4 n = geo[k];
		srad += (fabsf(q.u * n.x + q.v * n.y + q.w * n.z) + cc) * n.w;
	}
	v.dt[c] = float(ph.cfl) * v.vol[c] / srad;
}

// one RK stage: flux differences, residual, conserved-difference update,
// primitive differences and the boundary ghosts' differences
#ifndef E3D_DELTA_MIN_BLOCKS
#define E3D_DELTA_MIN_BLOCKS 5
#endif
template <bool DISS>
__global__ void __launch_bounds__(128, E3D_DELTA_MIN_BLOCKS) k_delta_flux_tiles(FusedView<float> v, Physics ph, float alpha, float beta,
                                                             int last, const int4* __restrict__ work) {
	const int4 t = work[blockIdx.x];
	const int c = t.x + threadIdx.x;
	if (c >= t.y) return;
	const float g = float(ph.gamma), gr = float(ph.gr), gm1 = float(ph.gm1);
	const int4 mate4 = __ldg(reinterpret_cast<const int4*>(v.slot_mate) + c);
	const int4 nb4 = __ldg(reinterpret_cast<const int4*>(v.slot_nbr) + c);
	const int mate[4] = {mate4.x, mate4.y, mate4.z, mate4.w};
	const int nb[4] = {nb4.x, nb4.y, nb4.z, nb4.w};
	const int NR = v.NR;
	float ac[5], ad[5];
#pragma unroll
	for (int q = 0; q < 5; q++) {
		ac[q] = 0.f;
		ad[q] = DISS ? v.Rd[q * NR + c] * (1.f - beta) : v.Rd[q * NR + c];
	}
	const Q5<float> bc = ld5(v.Pb, v.NA, c);
	const DCell own = dcell(bc, ld5(v.Pin, v.NA, c), g, gr);
	const float4* geo = reinterpret_cast<const float4*>(v.sgeo) + 4 * (size_t)c;
#pragma unroll
	for (int k = 0; k < 4; k++) {
		const bool left = mate[k] >= 0;
		const DCell nbr = dcell(ld5(v.Pb, v.NA, nb[k]), ld5(v.Pin, v.NA, nb[k]), g, gr);
		const float4 n = geo[k];
		float fc[5], fd[5];
		// one call with the sides selected by value: a branch on the orientation
		// would run the face arithmetic twice in warps whose cells differ
		ausm_delta_face<DISS>(left ? own : nbr, left ? nbr : own, n.x, n.y, n.z, n.w, fc, fd);
		if (left) {
#pragma unroll
			for (int q = 0; q < 5; q++) {
				ac[q] += fc[q];
				if (DISS) ad[q] += fd[q] * beta;
			}
		} else {
#pragma unroll
			for (int q = 0; q < 5; q++) {
				ac[q] -= fc[q];
				if (DISS) ad[q] -= fd[q] * beta;
			}
		}
	}
	const float coef = alpha * v.dt[c] / v.vol[c];
	float dw[5];
#pragma unroll
	for (int q = 0; q < 5; q++) {
		const float rc = v.Rb[q * NR + c] + ac[q];  // R64(q_b) - D64(q_b) + change of the convective sum
		dw[q] = v.dW[q * NR + c] - coef * (rc - ad[q]);
		if (last) v.Rc[q * NR + c] = rc;  // Rc - Rd is the full residual (norms)
		if (DISS) v.Rd[q * NR + c] = ad[q];
		if (last) v.dW[q * NR + c] = dw[q];  // next iteration's W0 - W_b
	}
	const Q5<float> dq = prim_delta(bc, dw, gm1);
	st5(v.Pout, v.NA, c, dq);
	// boundary ghosts in FP64: full state of the cell, FP64 face normal
#pragma unroll
	for (int k = 0; k < 4; k++) {
		if (nb[k] < NR) continue;
		const int gi = nb[k] - NR;
		const int kind = v.gkind[gi];
		if (kind == GK_NONE) continue;
		const Q5<double> b64 = ld5(v.Pb64, v.NA, c);
		const Q5<double> q64{b64.r + (double)dq.r, b64.u + (double)dq.u, b64.v + (double)dq.v, b64.w + (double)dq.w,
		                     b64.p + (double)dq.p};
		const int f = v.slot_face[4 * c + k];
		const double* n = v.nhat64 + 3 * (size_t)f;
		const Q5<double> g64 = ghost_state<double>(kind, q64, freestream64(v, ph, gi), n[0], n[1], n[2], ph.gamma);
		const Q5<double> gb = ld5(v.Pb64, v.NA, nb[k]);
		const Q5<float> dg{(float)(g64.r - gb.r), (float)(g64.u - gb.u), (float)(g64.v - gb.v), (float)(g64.w - gb.w),
		                   (float)(g64.p - gb.p)};
		st5(v.Pout, v.NA, nb[k], dg);
	}
}

// ------------------------------------------------------------ rebase

__device__ __forceinline__ void zero_cell(float* d0, float* d1, int NA, int c) {
	const Q5<float> z{0.f, 0.f, 0.f, 0.f, 0.f};
	st5(d0, NA, c, z);
	st5(d1, NA, c, z);
}

// real cells: W_b += dW, base primitives from W_b (FP64 and FP32 copies), differences cleared
__global__ void k_rebase_cells(int NR, int NA, double* __restrict__ Wb, float* __restrict__ dW, double gm1,
                               double* __restrict__ Pb64, float* __restrict__ Pb32, float* d0, float* d1) {
	const int c = blockIdx.x * blockDim.x + threadIdx.x;
	if (c >= NR) return;
	double w[5];
	for (int q = 0; q < 5; q++) {
		w[q] = Wb[(size_t)q * NR + c] + (double)dW[(size_t)q * NR + c];
		Wb[(size_t)q * NR + c] = w[q];
		dW[(size_t)q * NR + c] = 0.f;
	}
	Q5<double> p;
	p.r = w[0];
	p.u = w[1] / w[0];
	p.v = w[2] / w[0];
	p.w = w[3] / w[0];
	p.p = gm1 * (w[4] - 0.5 * (w[1] * w[1] + w[2] * w[2] + w[3] * w[3]) / w[0]);
	st5(Pb64, NA, c, p);
	st5(Pb32, NA, c, Q5<float>{(float)p.r, (float)p.u, (float)p.v, (float)p.w, (float)p.p});
	zero_cell(d0, d1, NA, c);
}

// boundary ghosts: base state from the owner cell's base state (FP64 normals)
__global__ void k_rebase_ghosts(FusedView<float> v, Physics ph, double* __restrict__ Pb64, float* __restrict__ Pb32,
                                float* d0, float* d1) {
	const int c = blockIdx.x * blockDim.x + threadIdx.x;
	if (c >= v.NR) return;
	for (int k = 0; k < 4; k++) {
		const int g = v.slot_nbr[4 * c + k];
		if (g < v.NR) continue;
		const int kind = v.gkind[g - v.NR];
		if (kind == GK_NONE) continue;
		const int f = v.slot_face[4 * c + k];
		const double* n = v.nhat64 + 3 * (size_t)f;
		const Q5<double> q =
		    ghost_state<double>(kind, ld5(Pb64, v.NA, c), freestream64(v, ph, g - v.NR), n[0], n[1], n[2], ph.gamma);
		st5(Pb64, v.NA, g, q);
		st5(Pb32, v.NA, g, Q5<float>{(float)q.r, (float)q.u, (float)q.v, (float)q.w, (float)q.p});
		zero_cell(d0, d1, v.NA, g);
	}
}

// connexion ghosts: copies of their origin cells
__global__ void k_rebase_halo(int n, const int* __restrict__ dst, const int* __restrict__ src, int NA,
                              double* __restrict__ Pb64, float* __restrict__ Pb32, float* d0, float* d1) {
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= n) return;
	const Q5<double> q = ld5(Pb64, NA, src[t]);
	st5(Pb64, NA, dst[t], q);
	st5(Pb32, NA, dst[t], Q5<float>{(float)q.r, (float)q.u, (float)q.v, (float)q.w, (float)q.p});
	zero_cell(d0, d1, NA, dst[t]);
}

// base residual in FP64: Rb = sum(+-Fc) - sum(+-Fd) of the base state (first-order AUSM,
// FP64 face normals and areas); the carried dissipation difference restarts at zero
__global__ void __launch_bounds__(128) k_base_residual(FusedView<float> v, Physics ph, const double* __restrict__ area64,
                                                       float* __restrict__ Rb, float* __restrict__ Rd) {
	const int c = blockIdx.x * blockDim.x + threadIdx.x;
	if (c >= v.NR) return;
	double ac[5] = {0., 0., 0., 0., 0.}, ad[5] = {0., 0., 0., 0., 0.};
	const Q5<double> qc = ld5(v.Pb64, v.NA, c);
	for (int k = 0; k < 4; k++) {
		const int s = 4 * c + k;
		const bool left = v.slot_mate[s] >= 0;
		const Q5<double> qn = ld5(v.Pb64, v.NA, v.slot_nbr[s]);
		const int f = v.slot_face[s];
		const double* n = v.nhat64 + 3 * (size_t)f;
		const Q5<double>& L = left ? qc : qn;
		const Q5<double>& R = left ? qn : qc;
		double fc[5], fd[5];
		flux_ausm_conv<double>(L, R, n[0], n[1], n[2], area64[f], ph.gamma, ph.gr, fc);
		flux_ausm_diss<double>(L, R, n[0], n[1], n[2], area64[f], ph.gamma, ph.gr, fd);
		for (int q = 0; q < 5; q++) {
			ac[q] += left ? fc[q] : -fc[q];
			ad[q] += left ? fd[q] : -fd[q];
		}
	}
	for (int q = 0; q < 5; q++) {
		Rb[(size_t)q * v.NR + c] = (float)(ac[q] - ad[q]);
		Rd[(size_t)q * v.NR + c] = 0.f;
	}
}

inline int grid_of(long long n, int tpb) { return (int)((n + tpb - 1) / tpb); }

}  // namespace

namespace delta {

cudaError_t launch_iterations(const FusedView<float>& v0, const FusedView<float>& v1, const Physics& ph,
                              const PersistArgs& a, cudaStream_t st) {
	if (a.n_work <= 0) return cudaSuccess;
	int parity = a.start_parity;
	for (int it = 0; it < a.iters; it++) {
		for (int s = 0; s < a.stages; s++) {
			const FusedView<float>& v = parity ? v1 : v0;
			if (s == 0) k_delta_start_tiles<<<a.n_work, 128, 0, st>>>(v, ph, a.work);
			const float al = float(a.alpha[s]), be = float(a.beta[s]);
			const int last = s == a.stages - 1;
			if (a.beta[s] != 0.0) k_delta_flux_tiles<true><<<a.n_work, 128, 0, st>>>(v, ph, al, be, last, a.work);
			else k_delta_flux_tiles<false><<<a.n_work, 128, 0, st>>>(v, ph, al, be, last, a.work);
			parity ^= 1;
		}
		const FusedView<float>& vf = parity ? v1 : v0;
		k_iter_tail<float><<<a.n_work, 128, 0, st>>>(vf, a);
		k_iter_sums<<<a.nblocks, 128, 0, st>>>(a, it);
	}
	k_iter_add<<<1, 1, 0, st>>>(a.d_iter, a.iters);
	return cudaGetLastError();
}

void launch_rebase(const FusedView<float>& v, const Physics& ph, double* Wb, const double* area64, int n_halo,
                   const int* halo_dst, const int* halo_src, float* d0, float* d1, cudaStream_t st) {
	double* Pb64 = const_cast<double*>(v.Pb64);
	float* Pb32 = const_cast<float*>(v.Pb);
	if (v.NR > 0) {
		k_rebase_cells<<<grid_of(v.NR, 256), 256, 0, st>>>(v.NR, v.NA, Wb, v.dW, ph.gm1, Pb64, Pb32, d0, d1);
		k_rebase_ghosts<<<grid_of(v.NR, 256), 256, 0, st>>>(v, ph, Pb64, Pb32, d0, d1);
	}
	if (n_halo > 0) k_rebase_halo<<<grid_of(n_halo, 256), 256, 0, st>>>(n_halo, halo_dst, halo_src, v.NA, Pb64, Pb32, d0, d1);
	if (v.NR > 0) k_base_residual<<<grid_of(v.NR, 128), 128, 0, st>>>(v, ph, area64, v.Rb, v.Rd);
}

}  // namespace delta
}  // namespace e3d
