/*
 * e3d_oracle.c -- CPU restatement of the euler3D residual/update path (FP64).
 *
 * TEST INFRASTRUCTURE ONLY (see e3d_oracle.h).  Compiled with
 * -O2 -ffp-contract=off; every expression keeps the reference's operand order
 * (file:line cited per function) so results are bit-identical to the
 * reference's x86-64 build.
 */
#include <stdlib.h>
#include "e3d_oracle.h"

#include <math.h>
#include <string.h>

#define V5(a, n, q, c) ((a)[(size_t)(q) * (size_t)(n) + (size_t)(c)])
#define G3(a, n, q, c, d) ((a)[((size_t)(q) * (size_t)(n) + (size_t)(c)) * 3 + (d)])

/* PrimitiveVariables::calculateFreeVariables (DataStructure/src/PrimitiveVariables.cpp:41-56) */
void e3d_oracle_freestream(const e3d_oracle_params* p, double q[5]) {
	const double pi = atan(1.0) * 4.0;
	const double a = p->aoa_deg * pi / 180.0;
	const double c = cos(a), s = sin(a);
	q[0] = 1.0;
	q[1] = p->mach * sqrt(p->gamma) * c;
	q[2] = p->mach * sqrt(p->gamma) * s;
	q[3] = 0.0;
	q[4] = 1.0;
}

/* initializeFlowField (PrimitiveVariables.cpp:58-69) plus the zero-initialised
 * residual, W0, gradient and limiter arrays (PrimitiveVariables.cpp:7-33,
 * InterpolationVariables.cpp:6-33, TimeVariables.cpp:6-14) */
void e3d_oracle_init_state(e3d_oracle_block* b, const e3d_oracle_params* p) {
	double f[5];
	e3d_oracle_freestream(p, f);
	for (int q = 0; q < 5; q++)
		for (int c = 0; c < b->n_all; c++) V5(b->prim, b->n_all, q, c) = f[q];
	memset(b->conv_res, 0, sizeof(double) * 5 * (size_t)b->n_all);
	memset(b->diss_res, 0, sizeof(double) * 5 * (size_t)b->n_all);
	memset(b->w0, 0, sizeof(double) * 5 * (size_t)b->n_all);
	memset(b->grad, 0, sizeof(double) * 15 * (size_t)b->n_all);
	memset(b->limiter, 0, sizeof(double) * 5 * (size_t)b->n_all);
	memset(b->dt, 0, sizeof(double) * (size_t)b->n_real);
	memset(b->spectral_radius, 0, sizeof(double) * (size_t)b->n_real);
}

/* Solver::saveW0 (Solver/src/Solver.cpp:161-210) */
void e3d_oracle_save_w0(e3d_oracle_block* b, const e3d_oracle_params* p) {
	const int n = b->n_all;
	for (int c = 0; c < b->n_real; c++) {
		const double ro = V5(b->prim, n, 0, c), uu = V5(b->prim, n, 1, c), vv = V5(b->prim, n, 2, c),
		             ww = V5(b->prim, n, 3, c), pp = V5(b->prim, n, 4, c);
		V5(b->w0, n, 0, c) = ro;
		V5(b->w0, n, 1, c) = ro * uu;
		V5(b->w0, n, 2, c) = ro * vv;
		V5(b->w0, n, 3, c) = ro * ww;
		V5(b->w0, n, 4, c) = 0.5 * ro * (uu * uu + vv * vv + ww * ww) + 1. / (p->gamma - 1.0) * pp;
	}
}

/* Timestep::computeSpectralRadius (Solver/src/Timestep.cpp:26-121) */
void e3d_oracle_spectral_radius(e3d_oracle_block* b, const e3d_oracle_params* p) {
	const int n = b->n_all;
	for (int c = 0; c < b->n_real; c++) {
		const double cc = sqrt(p->gamma * V5(b->prim, n, 4, c) / V5(b->prim, n, 0, c));
		b->spectral_radius[c] = 0.0;
		for (int k = b->cell_face_ptr[c]; k < b->cell_face_ptr[c + 1]; k++) {
			const int f = b->cell_faces[k];
			double nx = b->face_normal[3 * f], ny = b->face_normal[3 * f + 1], nz = b->face_normal[3 * f + 2];
			const double ds = sqrt(nx * nx + ny * ny + nz * nz);
			nx /= ds;
			ny /= ds;
			nz /= ds;
			b->spectral_radius[c] +=
			    (fabs((V5(b->prim, n, 1, c)) * nx + (V5(b->prim, n, 2, c)) * ny + (V5(b->prim, n, 3, c)) * nz) + (cc)) * ds;
		}
	}
}

/* Timestep::computeTimestep (Timestep.cpp:123-148) */
void e3d_oracle_timestep(e3d_oracle_block* b, const e3d_oracle_params* p) {
	for (int c = 0; c < b->n_real; c++) b->dt[c] = p->cfl * b->cell_volume[c] / b->spectral_radius[c];
}

/* Ghost-gradient reflection about the face plane for the ghosts of the first
 * n_real_boundaries markers (GreenGauss.cpp:175-232, LeastSquares.cpp:127-184) */
static void reflect_ghost_gradients(e3d_oracle_block* b) {
	const int n = b->n_all;
	int off = 0;
	for (int j = 0; j < b->n_markers; j++) {
		if (j < b->n_real_boundaries) {
			for (int i = 0; i < b->marker_size[j]; i++) {
				const int ext = b->marker_cells[off + i];
				const int f = b->cell_faces[b->cell_face_ptr[ext]];
				const int in = b->face_cells[2 * f];
				const double area = b->face_area[f];
				double nn[3];
				for (int d = 0; d < 3; d++) {
					nn[d] = b->face_normal[3 * f + d];
					nn[d] /= area;
				}
				for (int q = 0; q < 5; q++) {
					double dot = 0.0;
					for (int d = 0; d < 3; d++) dot += G3(b->grad, n, q, in, d) * nn[d];
					for (int d = 0; d < 3; d++) G3(b->grad, n, q, ext, d) = G3(b->grad, n, q, in, d) - 2.0 * dot * nn[d];
				}
			}
		}
		off += b->marker_size[j];
	}
}

/* GreenGauss::computeGradients (Solver/src/GreenGauss.cpp:12-234) and
 * LeastSquares::computeGradients (Solver/src/LeastSquares.cpp:12-186) */
void e3d_oracle_gradients(e3d_oracle_block* b, int kind) {
	const int n = b->n_all;
	memset(b->grad, 0, sizeof(double) * 15 * (size_t)n);
	for (int c = 0; c < b->n_real; c++) {
		for (int k = b->cell_face_ptr[c]; k < b->cell_face_ptr[c + 1]; k++) {
			if (kind == 0) {
				const int f = b->cell_faces[k];
				double nn[3] = {b->face_normal[3 * f], b->face_normal[3 * f + 1], b->face_normal[3 * f + 2]};
				if (c != b->face_cells[2 * f])
					for (int d = 0; d < 3; d++) nn[d] *= -1.0;
				const int l = b->face_cells[2 * f], r = b->face_cells[2 * f + 1];
				for (int d = 0; d < 3; d++)
					for (int q = 0; q < 5; q++)
						G3(b->grad, n, q, c, d) += 0.5 * (V5(b->prim, n, q, l) + V5(b->prim, n, q, r)) * nn[d];
			} else {
				const int nb = b->cell_cells[k];
				const double* w = &b->ls_weights[3 * (size_t)k];
				for (int d = 0; d < 3; d++)
					for (int q = 0; q < 5; q++)
						G3(b->grad, n, q, c, d) += w[d] * (V5(b->prim, n, q, nb) - V5(b->prim, n, q, c));
			}
		}
		if (kind == 0)
			for (int d = 0; d < 3; d++)
				for (int q = 0; q < 5; q++) G3(b->grad, n, q, c, d) /= b->cell_volume[c];
	}
	reflect_ghost_gradients(b);
}

/* BarthJespersen::computeLimiters (Solver/src/BarthJespersen.cpp:14-333) and
 * Venkatakrishnan::computeLimiters (Solver/src/Venkatakrishnan.cpp:12-326), all cells */
void e3d_oracle_limiters(e3d_oracle_block* b, int kind, double omega, double k) {
	const int n = b->n_all;
	for (int c = 0; c < n; c++) {
		const double eps2 = k * k * k * (b->cell_volume[c]);
		double mx[5], mn[5], dmax[5], dmin[5];
		for (int q = 0; q < 5; q++) mx[q] = mn[q] = V5(b->prim, n, q, c);
		for (int s = b->cell_face_ptr[c]; s < b->cell_face_ptr[c + 1]; s++) {
			const int nb = b->cell_cells[s];
			for (int q = 0; q < 5; q++) {
				const double v = V5(b->prim, n, q, nb);
				if (v > mx[q]) mx[q] = v;
				if (v < mn[q]) mn[q] = v;
			}
		}
		for (int q = 0; q < 5; q++) {
			dmax[q] = mx[q] - V5(b->prim, n, q, c);
			dmin[q] = mn[q] - V5(b->prim, n, q, c);
			V5(b->limiter, n, q, c) = INFINITY;
		}
		for (int s = b->cell_face_ptr[c]; s < b->cell_face_ptr[c + 1]; s++) {
			const int f = b->cell_faces[s];
			const double* r = (c == b->face_cells[2 * f]) ? &b->r_left[3 * f] : &b->r_right[3 * f];
			for (int q = 0; q < 5; q++) {
				double d2 = 0.0, lf;
				for (int d = 0; d < 3; d++) d2 += G3(b->grad, n, q, c, d) * r[d];
				if (kind == 0) {
					d2 = (copysign(1.0, d2)) * (fabs(d2) + omega);
					if (d2 > 0.0) lf = fmin(1.0, dmax[q] / d2);
					else if (d2 < 0.0) lf = fmin(1.0, dmin[q] / d2);
					else lf = 1.0;
				} else {
					if (d2 > 0.0)
						lf = (1.0 / d2) * ((dmax[q] * dmax[q] + eps2) * d2 + 2.0 * d2 * d2 * dmax[q]) /
						     (dmax[q] * dmax[q] + 2.0 * d2 * d2 + dmax[q] * d2 + eps2);
					else if (d2 < 0.0)
						lf = (1.0 / d2) * ((dmin[q] * dmin[q] + eps2) * d2 + 2.0 * d2 * d2 * dmin[q]) /
						     (dmin[q] * dmin[q] + 2.0 * d2 * d2 + dmin[q] * d2 + eps2);
					else lf = 1.0;
				}
				if (lf < V5(b->limiter, n, q, c)) V5(b->limiter, n, q, c) = lf;
			}
		}
	}
}

/* MUSCL face values of one side (FluxScheme.cpp:127-159) */
static void side_state(const e3d_oracle_block* b, int c, const double* r, double q[5]) {
	const int n = b->n_all;
	for (int v = 0; v < 5; v++) {
		q[v] = V5(b->prim, n, v, c);
		for (int d = 0; d < 3; d++) q[v] += V5(b->limiter, n, v, c) * G3(b->grad, n, v, c, d) * r[d];
	}
}

static void face_geometry(const e3d_oracle_block* b, int f, double* nx, double* ny, double* nz, double* nn) {
	*nx = b->face_normal[3 * f];
	*ny = b->face_normal[3 * f + 1];
	*nz = b->face_normal[3 * f + 2];
	*nn = sqrt(*nx * *nx + *ny * *ny + *nz * *nz);
	*nx /= *nn;
	*ny /= *nn;
	*nz /= *nn;
}

/* FluxScheme::computeFluxConv (Solver/src/FluxScheme.cpp:16-211) for Roe and
 * AusmScheme::computeFluxConv (Solver/src/AusmScheme.cpp:647-871) for AUSM */
void e3d_oracle_flux_conv(e3d_oracle_block* b, const e3d_oracle_params* p) {
	const int n = b->n_all;
	const double g = p->gamma;
	for (int c = 0; c < b->n_real; c++)
		for (int q = 0; q < 5; q++) V5(b->conv_res, n, q, c) = 0.0;
	for (int f = 0; f < b->n_faces; f++) {
		double nx, ny, nz, nn, L[5], R[5], fl[5];
		face_geometry(b, f, &nx, &ny, &nz, &nn);
		const int l = b->face_cells[2 * f], r = b->face_cells[2 * f + 1];
		side_state(b, l, &b->r_left[3 * f], L);
		side_state(b, r, &b->r_right[3 * f], R);
		const double qqL = L[1] * L[1] + L[2] * L[2] + L[3] * L[3];
		const double HL = (0.5 * qqL + g / (g - 1.0) * L[4] / L[0]);
		const double VL = L[1] * nx + L[2] * ny + L[3] * nz;
		const double qqR = R[1] * R[1] + R[2] * R[2] + R[3] * R[3];
		const double HR = (0.5 * qqR + g / (g - 1.0) * R[4] / R[0]);
		const double VR = R[1] * nx + R[2] * ny + R[3] * nz;
		if (p->flux == 0) {
			const double FL[5] = {L[0] * VL, L[0] * L[1] * VL + nx * L[4], L[0] * L[2] * VL + ny * L[4],
			                      L[0] * L[3] * VL + nz * L[4], L[0] * HL * VL};
			const double FR[5] = {R[0] * VR, R[0] * R[1] * VR + nx * R[4], R[0] * R[2] * VR + ny * R[4],
			                      R[0] * R[3] * VR + nz * R[4], R[0] * HR * VR};
			for (int q = 0; q < 5; q++) fl[q] = 0.5 * (FL[q] + FR[q]) * nn;
		} else {
			const double cL = sqrt(g * L[4] / L[0]), ML = VL / cL;
			double pLp, MLp, pRm, MRm;
			if (ML <= -1.0) { pLp = 0; MLp = 0; }
			else if (ML < 1.0) { pLp = L[4] * 0.25 * (ML + 1.0) * (ML + 1.0) * (2.0 - ML); MLp = 0.25 * (ML + 1.0) * (ML + 1.0); }
			else { MLp = ML; pLp = L[4]; }
			const double cR = sqrt(g * R[4] / R[0]), MR = VR / cR;
			if (MR <= -1.0) { pRm = R[4]; MRm = MR; }
			else if (MR < 1.0) { pRm = R[4] * 0.25 * (1.0 - MR) * (1.0 - MR) * (2.0 + MR); MRm = -0.25 * (MR - 1.0) * (MR - 1.0); }
			else { pRm = 0; MRm = 0; }
			const double M = MLp + MRm;
			const double FL[5] = {L[0] * cL, L[0] * L[1] * cL, L[0] * L[2] * cL, L[0] * L[3] * cL, L[0] * HL * cL};
			const double FR[5] = {R[0] * cR, R[0] * R[1] * cR, R[0] * R[2] * cR, R[0] * R[3] * cR, R[0] * HR * cR};
			fl[0] = 0.5 * M * (FL[0] + FR[0]) * nn;
			fl[1] = 0.5 * M * (FL[1] + FR[1]) * nn + nx * (pLp + pRm) * nn;
			fl[2] = 0.5 * M * (FL[2] + FR[2]) * nn + ny * (pLp + pRm) * nn;
			fl[3] = 0.5 * M * (FL[3] + FR[3]) * nn + nz * (pLp + pRm) * nn;
			fl[4] = 0.5 * M * (FL[4] + FR[4]) * nn;
		}
		for (int q = 0; q < 5; q++) V5(b->conv_res, n, q, l) += fl[q];
		for (int q = 0; q < 5; q++) V5(b->conv_res, n, q, r) -= fl[q];
	}
}

/* RoeScheme::computeFluxDiss (Solver/src/RoeScheme.cpp:12-311) and
 * AusmScheme::computeFluxDiss (Solver/src/AusmScheme.cpp:12-243) */
void e3d_oracle_flux_diss(e3d_oracle_block* b, const e3d_oracle_params* p, double beta) {
	const int n = b->n_all;
	const double g = p->gamma;
	for (int c = 0; c < b->n_real; c++)
		for (int q = 0; q < 5; q++) V5(b->diss_res, n, q, c) *= (1.0 - beta);
	for (int f = 0; f < b->n_faces; f++) {
		double nx, ny, nz, nn, L[5], R[5], fl[5];
		face_geometry(b, f, &nx, &ny, &nz, &nn);
		const int l = b->face_cells[2 * f], r = b->face_cells[2 * f + 1];
		side_state(b, l, &b->r_left[3 * f], L);
		side_state(b, r, &b->r_right[3 * f], R);
		const double qqL = L[1] * L[1] + L[2] * L[2] + L[3] * L[3];
		const double HL = (0.5 * qqL + g / (g - 1.0) * L[4] / L[0]);
		const double VL = L[1] * nx + L[2] * ny + L[3] * nz;
		const double qqR = R[1] * R[1] + R[2] * R[2] + R[3] * R[3];
		const double HR = (0.5 * qqR + g / (g - 1.0) * R[4] / R[0]);
		const double VR = R[1] * nx + R[2] * ny + R[3] * nz;
		if (p->flux == 0) {
			const double dp = (R[4] - L[4]), dV = (VR - VL), drho = (R[0] - L[0]);
			const double du = (R[1] - L[1]), dv = (R[2] - L[2]), dw = (R[3] - L[3]);
			const double rw = sqrt(L[0] * R[0]);
			const double uw = (L[1] * sqrt(L[0]) + R[1] * sqrt(R[0])) / (sqrt(L[0]) + sqrt(R[0]));
			const double vw = (L[2] * sqrt(L[0]) + R[2] * sqrt(R[0])) / (sqrt(L[0]) + sqrt(R[0]));
			const double ww = (L[3] * sqrt(L[0]) + R[3] * sqrt(R[0])) / (sqrt(L[0]) + sqrt(R[0]));
			const double Hw = (HL * sqrt(L[0]) + HR * sqrt(R[0])) / (sqrt(L[0]) + sqrt(R[0]));
			const double q2 = uw * uw + vw * vw + ww * ww;
			const double cw = sqrt((g - 1.) * (Hw - q2 / 2.));
			const double Vw = uw * nx + vw * ny + ww * nz;
			const double delta = 1. / 10. * cw;
			double L1, L234, L5;
			if (fabs(Vw - cw) <= delta) L1 = (fabs(Vw - cw) * fabs(Vw - cw) + delta * delta) / (2. * delta);
			else L1 = fabs(Vw - cw);
			if (fabs(Vw) <= delta) L234 = (fabs(Vw) * fabs(Vw) + delta * delta) / (2. * delta);
			else L234 = fabs(Vw);
			if (fabs(Vw + cw) <= delta) L5 = (fabs(Vw + cw) * fabs(Vw + cw) + delta * delta) / (2. * delta);
			else L5 = fabs(Vw + cw);
			const double F1 = L1 * (dp - rw * cw * dV) / (2. * cw * cw);
			const double F234 = (drho - dp / (cw * cw));
			const double F5 = L5 * (dp + rw * cw * dV) / (2. * cw * cw);
			const double A0 = F1 * 1. + L234 * (F234 * 1. + rw * 0.) + F5 * 1.;
			const double A1 = F1 * (uw - cw * nx) + L234 * ((F234 * uw) + rw * (du - dV * nx)) + F5 * (uw + cw * nx);
			const double A2 = F1 * (vw - cw * ny) + L234 * ((F234 * vw) + rw * (dv - dV * ny)) + F5 * (vw + cw * ny);
			const double A3 = F1 * (ww - cw * nz) + L234 * ((F234 * ww) + rw * (dw - dV * nz)) + F5 * (ww + cw * nz);
			const double A4 = F1 * (Hw - cw * Vw) +
			                  L234 * ((F234 * q2 / 2.) + rw * (uw * du + vw * dv + ww * dw - Vw * dV)) +
			                  F5 * (Hw + cw * Vw);
			fl[0] = 0.5 * (A0)*nn;
			fl[1] = 0.5 * (A1)*nn;
			fl[2] = 0.5 * (A2)*nn;
			fl[3] = 0.5 * (A3)*nn;
			fl[4] = 0.5 * (A4)*nn;
		} else {
			const double delta = 0.25;
			const double cL = sqrt(g * L[4] / L[0]), ML = VL / cL;
			double MLp, MRm;
			if (ML <= -1.0) MLp = 0;
			else if (ML < 1.0) MLp = 0.25 * (ML + 1.0) * (ML + 1.0);
			else MLp = ML;
			const double cR = sqrt(g * R[4] / R[0]), MR = VR / cR;
			if (MR <= -1.0) MRm = MR;
			else if (MR < 1.0) MRm = -0.25 * (MR - 1.0) * (MR - 1.0);
			else MRm = 0;
			double M = MLp + MRm;
			if (fabs(M) > delta) {
			} else {
				M = (M * M + delta * delta) / (2.0 * delta);
			}
			const double FL[5] = {L[0] * cL, L[0] * L[1] * cL, L[0] * L[2] * cL, L[0] * L[3] * cL, L[0] * HL * cL};
			const double FR[5] = {R[0] * cR, R[0] * R[1] * cR, R[0] * R[2] * cR, R[0] * R[3] * cR, R[0] * HR * cR};
			for (int q = 0; q < 5; q++) fl[q] = 0.5 * fabs(M) * (-FL[q] + FR[q]) * nn;
		}
		for (int q = 0; q < 5; q++) V5(b->diss_res, n, q, l) += fl[q] * beta;
		for (int q = 0; q < 5; q++) V5(b->diss_res, n, q, r) -= fl[q] * beta;
	}
}

/* Updater::updateInternalBlock (Solver/src/Updater.cpp:12-78) */
void e3d_oracle_update_internal(e3d_oracle_block* b, const e3d_oracle_params* p, double alpha) {
	const int n = b->n_all;
	for (int c = 0; c < b->n_real; c++) {
		double w[5];
		for (int q = 0; q < 5; q++)
			w[q] = V5(b->w0, n, q, c) -
			       (alpha * b->dt[c] / b->cell_volume[c]) * (V5(b->conv_res, n, q, c) - V5(b->diss_res, n, q, c));
		V5(b->prim, n, 0, c) = w[0];
		V5(b->prim, n, 1, c) = w[1] / w[0];
		V5(b->prim, n, 2, c) = w[2] / w[0];
		V5(b->prim, n, 3, c) = w[3] / w[0];
		V5(b->prim, n, 4, c) = (p->gamma - 1.0) * (w[4] - 0.5 * (w[1] * w[1] + w[2] * w[2] + w[3] * w[3]) / w[0]);
	}
}

/* Updater::updateBoundary (Updater.cpp:80-88): WallCellIds / SymmetryCellIds
 * (slip, DataStructure/src/WallCellIds.cpp:9-95, SymmetryCellIds.cpp:9-96),
 * FarfieldCellIds (characteristic, FarfieldCellIds.cpp:10-205); CONNEXION no-op */
/* CentralIrsSmoother::smoothResidual (Solver/src/CentralIrsSmoother.cpp:12-166):
 * J1 = R / (1 + eps Na) for every real cell (:78-91), then
 * R = (R + eps * sum of J1 over the real neighbours in cell_2_cells order) / (1 + eps Na)
 * (:92-142), eps = 0.8, Na = the cell's face count.  The reference sets the
 * dissipative v start value from w and leaves w unset (:90); here both follow
 * the formula of the other eight arrays. */
void e3d_oracle_smooth(e3d_oracle_block* b) {
	const int nr = b->n_real, na = b->n_all;
	const double epsilon = 0.8;
	double* j1 = (double*)malloc(sizeof(double) * 10 * (size_t)nr);
	double* out = (double*)malloc(sizeof(double) * 10 * (size_t)nr);
	for (int c = 0; c < nr; c++) {
		const int Na = b->cell_face_ptr[c + 1] - b->cell_face_ptr[c];
		for (int q = 0; q < 5; q++) {
			j1[q * (size_t)nr + c] = (b->conv_res[q * (size_t)na + c] + 0.) / (1. + epsilon * Na);
			j1[(5 + q) * (size_t)nr + c] = (b->diss_res[q * (size_t)na + c] + 0.) / (1. + epsilon * Na);
		}
	}
	for (int c = 0; c < nr; c++) {
		double sum[10] = {0., 0., 0., 0., 0., 0., 0., 0., 0., 0.};
		for (int k = b->cell_face_ptr[c]; k < b->cell_face_ptr[c + 1]; k++) {
			const int j = b->cell_cells[k];
			if (j < nr)
				for (int q = 0; q < 10; q++) sum[q] += j1[q * (size_t)nr + j];
		}
		const int Na = b->cell_face_ptr[c + 1] - b->cell_face_ptr[c];
		for (int q = 0; q < 5; q++) {
			out[q * (size_t)nr + c] = (b->conv_res[q * (size_t)na + c] + epsilon * sum[q]) / (1. + epsilon * Na);
			out[(5 + q) * (size_t)nr + c] = (b->diss_res[q * (size_t)na + c] + epsilon * sum[5 + q]) / (1. + epsilon * Na);
		}
	}
	for (int c = 0; c < nr; c++)
		for (int q = 0; q < 5; q++) {
			b->conv_res[q * (size_t)na + c] = out[q * (size_t)nr + c];
			b->diss_res[q * (size_t)na + c] = out[(5 + q) * (size_t)nr + c];
		}
	free(j1);
	free(out);
}

void e3d_oracle_update_boundary(e3d_oracle_block* b, const e3d_oracle_params* p) {
	const int n = b->n_all;
	double fr[5];
	e3d_oracle_freestream(p, fr);
	int off = 0;
	for (int j = 0; j < b->n_markers; j++) {
		const int kind = b->marker_kind[j];
		if (j < b->n_real_boundaries && kind != 4) {
			for (int i = 0; i < b->marker_size[j]; i++) {
				const int ext = b->marker_cells[off + i];
				const int f = b->cell_faces[b->cell_face_ptr[ext]];
				const int in = b->cell_cells[b->cell_face_ptr[ext]];
				const double area = b->face_area[f];
				double nx = b->face_normal[3 * f], ny = b->face_normal[3 * f + 1], nz = b->face_normal[3 * f + 2];
				nx /= area;
				ny /= area;
				nz /= area;
				const double ro = V5(b->prim, n, 0, in), uu = V5(b->prim, n, 1, in), vv = V5(b->prim, n, 2, in),
				             ww = V5(b->prim, n, 3, in), pp = V5(b->prim, n, 4, in);
				double o[5];
				if (kind == 1 || kind == 3) {
					const double un = uu * nx + vv * ny + ww * nz;
					const double ub = uu - un * nx, vb = vv - un * ny, wb = ww - un * nz;
					o[0] = ro;
					o[1] = 2.0 * ub - uu;
					o[2] = 2.0 * vb - vv;
					o[3] = 2.0 * wb - ww;
					o[4] = pp;
				} else {
					const double c = sqrt(p->gamma * pp / ro);
					const double un = uu * nx + vv * ny + ww * nz;
					if (fabs(un / c) > 1.0) {
						if (un < 0.0) {
							o[0] = 2.0 * fr[0] - ro;
							o[1] = 2.0 * fr[1] - uu;
							o[2] = 2.0 * fr[2] - vv;
							o[3] = 2.0 * fr[3] - ww;
							o[4] = 2.0 * fr[4] - pp;
						} else {
							o[0] = ro;
							o[1] = uu;
							o[2] = vv;
							o[3] = ww;
							o[4] = pp;
						}
					} else if (un < 0.0) {
						const double pb = 0.5 * (fr[4] + pp - ro * c * (nx * (fr[1] - uu) + ny * (fr[2] - vv) + nz * (fr[3] - ww)));
						const double rb = fr[0] + (pb - fr[4]) / (c * c);
						const double ub = fr[1] - nx * (fr[4] - pb) / (ro * c);
						const double vb = fr[2] - ny * (fr[4] - pb) / (ro * c);
						const double wb = fr[3] - nz * (fr[4] - pb) / (ro * c);
						o[0] = 2.0 * rb - ro;
						o[1] = 2.0 * ub - uu;
						o[2] = 2.0 * vb - vv;
						o[3] = 2.0 * wb - ww;
						o[4] = 2.0 * pb - pp;
					} else {
						const double pb = fr[4];
						const double rb = ro + (pb - pp) / (c * c);
						const double ub = uu + nx * (pp - pb) / (ro * c);
						const double vb = vv + ny * (pp - pb) / (ro * c);
						const double wb = ww + nz * (pp - pb) / (ro * c);
						o[0] = 2.0 * rb - ro;
						o[1] = 2.0 * ub - uu;
						o[2] = 2.0 * vb - vv;
						o[3] = 2.0 * wb - ww;
						o[4] = 2.0 * pb - pp;
					}
				}
				for (int q = 0; q < 5; q++) V5(b->prim, n, q, ext) = o[q];
			}
		}
		off += b->marker_size[j];
	}
}

/* BlockCommunicator::updateBoundaries, serial path (MPI/src/BlockCommunicator.cpp:212-268);
 * only the five primitives matter (the other copied arrays are rewritten before use) */
void e3d_oracle_halo(e3d_oracle_block* blocks, const e3d_oracle_connexion* c, int n_connexions) {
	for (int i = 0; i < n_connexions; i++) {
		e3d_oracle_block* d = &blocks[c[i].dest_block];
		const e3d_oracle_block* o = &blocks[c[i].origin_block];
		for (int j = 0; j < c[i].n; j++)
			for (int q = 0; q < 5; q++)
				V5(d->prim, d->n_all, q, c[i].dest_cells[j]) = V5(o->prim, o->n_all, q, c[i].origin_cells[j]);
	}
}

/* Convergence::calculate*Rms sums (PostProcessing/src/Convergence.cpp:27-143) and
 * AerodynamicParameters::computeAerodynamic sums (AerodynamicParameters.cpp:163-239) */
void e3d_oracle_flow_data(const e3d_oracle_block* b, const e3d_oracle_params* p, double out[10]) {
	const int n = b->n_all;
	for (int q = 0; q < 5; q++) {
		double s = 0.0;
		for (int c = 0; c < b->n_real; c++) {
			const double r = V5(b->conv_res, n, q, c) - V5(b->diss_res, n, q, c);
			s += r * r;
		}
		out[q] = s;
	}
	const double dyn = 0.5 * p->gamma * p->mach * p->mach;
	double cl = 0., cd = 0., cmx = 0., cmy = 0., cmz = 0.;
	for (int i = 0; i < b->n_wall_faces; i++) {
		const int f = b->wall_faces[i];
		const double pbc = 0.5 * (V5(b->prim, n, 4, b->face_cells[2 * f]) + V5(b->prim, n, 4, b->face_cells[2 * f + 1]));
		const double cp = (pbc - 1.) / (dyn * p->cmac);
		const double fx = cp * b->face_normal[3 * f], fy = cp * b->face_normal[3 * f + 1], fz = cp * b->face_normal[3 * f + 2];
		const double x = b->face_center[3 * f], y = b->face_center[3 * f + 1], z = b->face_center[3 * f + 2];
		cl += fy;
		cd += fx;
		cmx += y * fz - z * fy;
		cmy += z * fx - x * fz;
		cmz += x * fy - y * fx;
	}
	out[5] = cl;
	out[6] = cd;
	out[7] = cmx;
	out[8] = cmy;
	out[9] = cmz;
}

static const double* rk_alpha(int stages) {
	static const double a1[] = {1.0}, a2[] = {0.6, 1.0}, a3[] = {0.6, 0.6, 1.0}, a4[] = {0.25, 1.0 / 3.0, 0.5, 1.0},
	                    a5[] = {0.2742, 0.2067, 0.5020, 0.5142, 1.0};
	switch (stages) {
	case 1: return a1;
	case 2: return a2;
	case 3: return a3;
	case 4: return a4;
	case 5: return a5;
	default: return 0;
	}
}
static const double* rk_beta(int stages) {
	static const double b1[] = {1.0}, b2[] = {1.0, 0.0}, b3[] = {1.0, 0.0, 0.0}, b4[] = {1.0, 0.5, 0.0, 0.0},
	                    b5[] = {1.0, 0.0, 0.56, 0.0, 0.44};
	switch (stages) {
	case 1: return b1;
	case 2: return b2;
	case 3: return b3;
	case 4: return b4;
	case 5: return b5;
	default: return 0;
	}
}

/* Solver::solve body (Solver/src/Solver.cpp:76-97) with RungeKutta::computeRungeKutta
 * (RungeKutta.cpp:80-94) and ResidualCalculator::computeResidual (ResidualCalculator.cpp:24-41) */
int e3d_oracle_iterate(e3d_oracle_block* blocks, int n_blocks, const e3d_oracle_connexion* c, int n_connexions,
                       const e3d_oracle_params* p, int n_iter, int first_iter, double* rms0, int* have_rms0,
                       double* hist) {
	const double* alpha = rk_alpha(p->stages);
	const double* beta = rk_beta(p->stages);
	if (!alpha) return -1;
	const double aoa = p->aoa_deg * 4. * atan(1.) / 180;
	if (first_iter == 0) e3d_oracle_halo(blocks, c, n_connexions);
	for (int it = 0; it < n_iter; it++) {
		double rms[5] = {0, 0, 0, 0, 0}, cl = 0, cd = 0, cmx = 0, cmy = 0, cmz = 0;
		for (int bi = 0; bi < n_blocks; bi++) {
			e3d_oracle_block* b = &blocks[bi];
			e3d_oracle_save_w0(b, p);
			e3d_oracle_spectral_radius(b, p);
			e3d_oracle_timestep(b, p);
			for (int s = 0; s < p->stages; s++) {
				if (p->order == 2) {
					e3d_oracle_gradients(b, p->gradient);
					e3d_oracle_limiters(b, p->limiter, p->omega, p->k);
				}
				e3d_oracle_flux_conv(b, p);
				e3d_oracle_flux_diss(b, p, beta[s]);
				if (p->smoothing) e3d_oracle_smooth(b);
				e3d_oracle_update_internal(b, p, alpha[s]);
				e3d_oracle_update_boundary(b, p);
			}
			double fd[10];
			e3d_oracle_flow_data(b, p, fd);
			for (int q = 0; q < 5; q++) rms[q] += (1. / b->n_real) * pow(fd[q], 0.5);
			cl += fd[5] * cos(aoa) - fd[6] * sin(aoa);
			cd += fd[5] * sin(aoa) + fd[6] * cos(aoa);
			cmx += fd[7];
			cmy += fd[8];
			cmz += fd[9];
		}
		e3d_oracle_halo(blocks, c, n_connexions);
		if (!*have_rms0) {
			for (int q = 0; q < 5; q++) rms0[q] = rms[q];
			*have_rms0 = 1;
		}
		double* h = &hist[(size_t)it * 15];
		for (int q = 0; q < 5; q++) {
			h[q] = rms[q];
			h[10 + q] = log10(rms[q]) - log10(rms0[q]);
		}
		h[5] = cl;
		h[6] = cd;
		h[7] = cmx;
		h[8] = cmy;
		h[9] = cmz;
	}
	return 0;
}
