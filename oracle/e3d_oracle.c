/*
 * e3d_oracle.c -- CPU restatement of the euler3D residual/update path.
 *
 * TEST INFRASTRUCTURE ONLY (see e3d_oracle.h).  Compiled with
 * -O2 -ffp-contract=off; every expression keeps the reference's operand order
 * (file:line cited per function) so results are bit-identical to the
 * reference's x86-64 build.
 *
 * The same source builds a second library, libe3d_oracle32.so
 * (-DE3D_ORACLE_FP32): a model of the B200 FP32 variant used to derive that
 * variant's error bounds.  There `real` is float and values are rounded where
 * the FP32 kernels round them: geometry (unit normals, areas, r-vectors,
 * least-squares weights, volumes) and primitives are held in FP32; gradient,
 * limiter, flux, time-step and boundary arithmetic runs in FP32; the residual
 * accumulators are FP32; the conservative update is FP64 from FP32 residuals,
 * and the FP64 conservative state W is carried from stage to stage across
 * iterations (W0 of the next iteration = W of the last stage, starting from
 * the FP64 freestream state); norms and forces are FP64 sums.  The FP32
 * Venkatakrishnan limiter uses the kernels' one-division form and the face
 * value of a tetrahedron's own side is q + phi (g.r).  e3d_oracle_set_noise
 * moves each face flux by one FP32 unit up or down, or leaves it, by a seeded
 * hash (what another FP32 evaluation order, contraction or approximate
 * division gives): independent rounding realisations for the error
 * distribution.
 * In the FP64 build (real = double) every macro below is the identity and
 * the arithmetic is the reference's.
 */
#include <stdint.h>
#include <stdlib.h>
#include "e3d_oracle.h"

#include <math.h>
#include <string.h>

#ifdef E3D_ORACLE_FP32
typedef float real;
#define r_sqrt sqrtf
#define r_fabs fabsf
#define r_fmin fminf
#define r_copysign copysignf
#define FP32_MODEL 1
#else
typedef double real;
#define r_sqrt sqrt
#define r_fabs fabs
#define r_fmin fmin
#define r_copysign copysign
#define FP32_MODEL 0
#endif
#define K(x) ((real)(x))            /* a constant or a double parameter in working precision */
#define LD(x) ((real)(x))           /* an array value read in working precision */
#define ST(x) ((double)(real)(x))   /* a value stored in working precision */

static uint64_t g_noise_seed = 0, g_noise_calls = 0;

void e3d_oracle_set_noise(unsigned long long seed) {
	g_noise_seed = seed;
	g_noise_calls = 0;
}

#if FP32_MODEL
/* splitmix64 finaliser: fixed pseudo-random bits per (seed, call, face, variable) */
static uint64_t mix64(uint64_t x) {
	x += 0x9e3779b97f4a7c15ULL;
	x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ULL;
	x = (x ^ (x >> 27)) * 0x94d049bb133111ebULL;
	return x ^ (x >> 31);
}
/* A face flux as another FP32 evaluation order could give it: unchanged, one
 * FP32 unit up or one down (seeded hash: 1/2, 1/4, 1/4).  The identity while
 * no seed is set. */
static float perturb_flux(float v, int f, int q) {
	if (!g_noise_seed) return v;
	const uint64_t h = mix64(g_noise_seed ^ mix64(g_noise_calls * 0x100000001b3ULL + (uint64_t)f * 8u + (uint64_t)q));
	if (!(h & 1)) return v;
	return nextafterf(v, (h & 2) ? INFINITY : -INFINITY);
}
#define FLUX_OUT(v, f, q) perturb_flux((v), (f), (q))
#else
#define FLUX_OUT(v, f, q) (v)
#endif

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
		for (int c = 0; c < b->n_all; c++) V5(b->prim, b->n_all, q, c) = ST(f[q]);
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
		const real cc = r_sqrt(K(p->gamma) * LD(V5(b->prim, n, 4, c)) / LD(V5(b->prim, n, 0, c)));
		real sr = K(0.0);
		for (int k = b->cell_face_ptr[c]; k < b->cell_face_ptr[c + 1]; k++) {
			const int f = b->cell_faces[k];
			double nx = b->face_normal[3 * f], ny = b->face_normal[3 * f + 1], nz = b->face_normal[3 * f + 2];
			const double ds = sqrt(nx * nx + ny * ny + nz * nz);
			nx /= ds;
			ny /= ds;
			nz /= ds;
			sr += (r_fabs((LD(V5(b->prim, n, 1, c))) * K(nx) + (LD(V5(b->prim, n, 2, c))) * K(ny) +
			              (LD(V5(b->prim, n, 3, c))) * K(nz)) +
			       (cc)) *
			      K(ds);
		}
		b->spectral_radius[c] = ST(sr);
	}
}

/* Timestep::computeTimestep (Timestep.cpp:123-148) */
void e3d_oracle_timestep(e3d_oracle_block* b, const e3d_oracle_params* p) {
	for (int c = 0; c < b->n_real; c++)
		b->dt[c] = ST(K(p->cfl) * LD(b->cell_volume[c]) / LD(b->spectral_radius[c]));
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
				real nn[3];
				for (int d = 0; d < 3; d++) {
					double t = b->face_normal[3 * f + d];
					t /= area;
					nn[d] = K(t);
				}
				for (int q = 0; q < 5; q++) {
					real dot = K(0.0);
					for (int d = 0; d < 3; d++) dot += LD(G3(b->grad, n, q, in, d)) * nn[d];
					for (int d = 0; d < 3; d++)
						G3(b->grad, n, q, ext, d) = ST(LD(G3(b->grad, n, q, in, d)) - K(2.0) * dot * nn[d]);
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
		real acc[5][3];
		for (int q = 0; q < 5; q++) acc[q][0] = acc[q][1] = acc[q][2] = K(0.0);
		for (int k = b->cell_face_ptr[c]; k < b->cell_face_ptr[c + 1]; k++) {
			if (kind == 0) {
				const int f = b->cell_faces[k];
				double nn[3] = {b->face_normal[3 * f], b->face_normal[3 * f + 1], b->face_normal[3 * f + 2]};
				if (c != b->face_cells[2 * f])
					for (int d = 0; d < 3; d++) nn[d] *= -1.0;
				const int l = b->face_cells[2 * f], r = b->face_cells[2 * f + 1];
				for (int d = 0; d < 3; d++)
					for (int q = 0; q < 5; q++)
						acc[q][d] += K(0.5) * (LD(V5(b->prim, n, q, l)) + LD(V5(b->prim, n, q, r))) * K(nn[d]);
			} else {
				const int nb = b->cell_cells[k];
				const double* w = &b->ls_weights[3 * (size_t)k];
				for (int d = 0; d < 3; d++)
					for (int q = 0; q < 5; q++)
						acc[q][d] += LD(w[d]) * (LD(V5(b->prim, n, q, nb)) - LD(V5(b->prim, n, q, c)));
			}
		}
		if (kind == 0)
			for (int d = 0; d < 3; d++)
				for (int q = 0; q < 5; q++) acc[q][d] /= LD(b->cell_volume[c]);
		for (int q = 0; q < 5; q++)
			for (int d = 0; d < 3; d++) G3(b->grad, n, q, c, d) = ST(acc[q][d]);
	}
	reflect_ghost_gradients(b);
}

/* BarthJespersen::computeLimiters (Solver/src/BarthJespersen.cpp:14-333) and
 * Venkatakrishnan::computeLimiters (Solver/src/Venkatakrishnan.cpp:12-326), all cells */
void e3d_oracle_limiters(e3d_oracle_block* b, int kind, double omega, double k) {
	const int n = b->n_all;
	for (int c = 0; c < n; c++) {
		const real eps2 = K(k * k * k) * LD(b->cell_volume[c]);
		real mx[5], mn[5], dmax[5], dmin[5], phi[5];
		for (int q = 0; q < 5; q++) mx[q] = mn[q] = LD(V5(b->prim, n, q, c));
		for (int s = b->cell_face_ptr[c]; s < b->cell_face_ptr[c + 1]; s++) {
			const int nb = b->cell_cells[s];
			for (int q = 0; q < 5; q++) {
				const real v = LD(V5(b->prim, n, q, nb));
				if (v > mx[q]) mx[q] = v;
				if (v < mn[q]) mn[q] = v;
			}
		}
		for (int q = 0; q < 5; q++) {
			dmax[q] = mx[q] - LD(V5(b->prim, n, q, c));
			dmin[q] = mn[q] - LD(V5(b->prim, n, q, c));
			phi[q] = (real)INFINITY;
		}
		for (int s = b->cell_face_ptr[c]; s < b->cell_face_ptr[c + 1]; s++) {
			const int f = b->cell_faces[s];
			const double* r = (c == b->face_cells[2 * f]) ? &b->r_left[3 * f] : &b->r_right[3 * f];
			for (int q = 0; q < 5; q++) {
				real d2 = K(0.0), lf;
				for (int d = 0; d < 3; d++) d2 += LD(G3(b->grad, n, q, c, d)) * LD(r[d]);
				if (kind == 0) {
					d2 = (r_copysign(K(1.0), d2)) * (r_fabs(d2) + K(omega));
					if (d2 > K(0.0)) lf = r_fmin(K(1.0), dmax[q] / d2);
					else if (d2 < K(0.0)) lf = r_fmin(K(1.0), dmin[q] / d2);
					else lf = K(1.0);
				} else {
#if FP32_MODEL
					/* the FP32 kernels' form: d2 cancelled, one division */
					if (!(d2 > 0.0f) && !(d2 < 0.0f)) lf = 1.0f;
					else {
						const float D = d2 > 0.0f ? dmax[q] : dmin[q];
						const float A = fmaf(D, D, eps2);
						lf = fmaf(2.0f * d2, D, A) / fmaf(d2, fmaf(2.0f, d2, D), A);
					}
#else
					if (d2 > 0.0)
						lf = (1.0 / d2) * ((dmax[q] * dmax[q] + eps2) * d2 + 2.0 * d2 * d2 * dmax[q]) /
						     (dmax[q] * dmax[q] + 2.0 * d2 * d2 + dmax[q] * d2 + eps2);
					else if (d2 < 0.0)
						lf = (1.0 / d2) * ((dmin[q] * dmin[q] + eps2) * d2 + 2.0 * d2 * d2 * dmin[q]) /
						     (dmin[q] * dmin[q] + 2.0 * d2 * d2 + dmin[q] * d2 + eps2);
					else lf = 1.0;
#endif
				}
				if (lf < phi[q]) phi[q] = lf;
			}
		}
		for (int q = 0; q < 5; q++) V5(b->limiter, n, q, c) = ST(phi[q]);
	}
}

/* 1 when every real cell of the block is a tetrahedron (the FP32 kernels' 4-slot path) */
static int all_tets(const e3d_oracle_block* b) {
	for (int c = 0; c < b->n_real; c++)
		if (b->cell_face_ptr[c + 1] - b->cell_face_ptr[c] != 4) return 0;
	return 1;
}

/* MUSCL face values of one side (FluxScheme.cpp:127-159).  FP32 model: a real
 * tetrahedron's own side is q + phi (g.r), the FP32 kernels' form. */
static void side_state(const e3d_oracle_block* b, int c, const double* r, real q[5], int tet) {
	const int n = b->n_all;
	(void)tet;
	for (int v = 0; v < 5; v++) {
		q[v] = LD(V5(b->prim, n, v, c));
#if FP32_MODEL
		if (tet && c < b->n_real) {
			real d2 = LD(G3(b->grad, n, v, c, 0)) * LD(r[0]);
			d2 += LD(G3(b->grad, n, v, c, 1)) * LD(r[1]);
			d2 += LD(G3(b->grad, n, v, c, 2)) * LD(r[2]);
			q[v] = q[v] + LD(V5(b->limiter, n, v, c)) * d2;
			continue;
		}
#endif
		for (int d = 0; d < 3; d++) q[v] += LD(V5(b->limiter, n, v, c)) * LD(G3(b->grad, n, v, c, d)) * LD(r[d]);
	}
}

/* unit normal and area: the reference's per-face normalisation in FP64 (the
 * FP32 kernels read these values precomputed and rounded) */
static void face_geometry(const e3d_oracle_block* b, int f, real* rx, real* ry, real* rz, real* rn) {
	double nx = b->face_normal[3 * f];
	double ny = b->face_normal[3 * f + 1];
	double nz = b->face_normal[3 * f + 2];
	const double nn = sqrt(nx * nx + ny * ny + nz * nz);
	nx /= nn;
	ny /= nn;
	nz /= nn;
	*rx = K(nx);
	*ry = K(ny);
	*rz = K(nz);
	*rn = K(nn);
}

/* FluxScheme::computeFluxConv (Solver/src/FluxScheme.cpp:16-211) for Roe and
 * AusmScheme::computeFluxConv (Solver/src/AusmScheme.cpp:647-871) for AUSM */
void e3d_oracle_flux_conv(e3d_oracle_block* b, const e3d_oracle_params* p) {
	const int n = b->n_all;
	const real g = K(p->gamma);
	const real gr = K(p->gamma / (p->gamma - 1.0)); /* g / (g - 1.0), formed in FP64 */
	const int tet = all_tets(b);
	for (int c = 0; c < b->n_real; c++)
		for (int q = 0; q < 5; q++) V5(b->conv_res, n, q, c) = 0.0;
	for (int f = 0; f < b->n_faces; f++) {
		real nx, ny, nz, nn, L[5], R[5], fl[5];
		face_geometry(b, f, &nx, &ny, &nz, &nn);
		const int l = b->face_cells[2 * f], r = b->face_cells[2 * f + 1];
		side_state(b, l, &b->r_left[3 * f], L, tet);
		side_state(b, r, &b->r_right[3 * f], R, tet);
		const real qqL = L[1] * L[1] + L[2] * L[2] + L[3] * L[3];
		const real HL = (K(0.5) * qqL + gr * L[4] / L[0]);
		const real VL = L[1] * nx + L[2] * ny + L[3] * nz;
		const real qqR = R[1] * R[1] + R[2] * R[2] + R[3] * R[3];
		const real HR = (K(0.5) * qqR + gr * R[4] / R[0]);
		const real VR = R[1] * nx + R[2] * ny + R[3] * nz;
		if (p->flux == 0) {
			const real FL[5] = {L[0] * VL, L[0] * L[1] * VL + nx * L[4], L[0] * L[2] * VL + ny * L[4],
			                    L[0] * L[3] * VL + nz * L[4], L[0] * HL * VL};
			const real FR[5] = {R[0] * VR, R[0] * R[1] * VR + nx * R[4], R[0] * R[2] * VR + ny * R[4],
			                    R[0] * R[3] * VR + nz * R[4], R[0] * HR * VR};
			for (int q = 0; q < 5; q++) fl[q] = K(0.5) * (FL[q] + FR[q]) * nn;
		} else {
			const real cL = r_sqrt(g * L[4] / L[0]), ML = VL / cL;
			real pLp, MLp, pRm, MRm;
			if (ML <= K(-1.0)) { pLp = 0; MLp = 0; }
			else if (ML < K(1.0)) { pLp = L[4] * K(0.25) * (ML + K(1.0)) * (ML + K(1.0)) * (K(2.0) - ML); MLp = K(0.25) * (ML + K(1.0)) * (ML + K(1.0)); }
			else { MLp = ML; pLp = L[4]; }
			const real cR = r_sqrt(g * R[4] / R[0]), MR = VR / cR;
			if (MR <= K(-1.0)) { pRm = R[4]; MRm = MR; }
			else if (MR < K(1.0)) { pRm = R[4] * K(0.25) * (K(1.0) - MR) * (K(1.0) - MR) * (K(2.0) + MR); MRm = K(-0.25) * (MR - K(1.0)) * (MR - K(1.0)); }
			else { pRm = 0; MRm = 0; }
			const real M = MLp + MRm;
			const real FL[5] = {L[0] * cL, L[0] * L[1] * cL, L[0] * L[2] * cL, L[0] * L[3] * cL, L[0] * HL * cL};
			const real FR[5] = {R[0] * cR, R[0] * R[1] * cR, R[0] * R[2] * cR, R[0] * R[3] * cR, R[0] * HR * cR};
			fl[0] = K(0.5) * M * (FL[0] + FR[0]) * nn;
			fl[1] = K(0.5) * M * (FL[1] + FR[1]) * nn + nx * (pLp + pRm) * nn;
			fl[2] = K(0.5) * M * (FL[2] + FR[2]) * nn + ny * (pLp + pRm) * nn;
			fl[3] = K(0.5) * M * (FL[3] + FR[3]) * nn + nz * (pLp + pRm) * nn;
			fl[4] = K(0.5) * M * (FL[4] + FR[4]) * nn;
		}
		for (int q = 0; q < 5; q++) fl[q] = FLUX_OUT(fl[q], f, q);
		for (int q = 0; q < 5; q++) V5(b->conv_res, n, q, l) = ST(LD(V5(b->conv_res, n, q, l)) + fl[q]);
		for (int q = 0; q < 5; q++) V5(b->conv_res, n, q, r) = ST(LD(V5(b->conv_res, n, q, r)) - fl[q]);
	}
	g_noise_calls++;
}

/* RoeScheme::computeFluxDiss (Solver/src/RoeScheme.cpp:12-311) and
 * AusmScheme::computeFluxDiss (Solver/src/AusmScheme.cpp:12-243) */
void e3d_oracle_flux_diss(e3d_oracle_block* b, const e3d_oracle_params* p, double beta) {
	const int n = b->n_all;
	const real g = K(p->gamma);
	const real gr = K(p->gamma / (p->gamma - 1.0)); /* g / (g - 1.0), formed in FP64 */
	const real gm1 = K(p->gamma - 1.);
	const real rb = K(beta);
	const int tet = all_tets(b);
	for (int c = 0; c < b->n_real; c++)
		for (int q = 0; q < 5; q++) V5(b->diss_res, n, q, c) = ST(LD(V5(b->diss_res, n, q, c)) * (K(1.0) - rb));
	for (int f = 0; f < b->n_faces; f++) {
		real nx, ny, nz, nn, L[5], R[5], fl[5];
		face_geometry(b, f, &nx, &ny, &nz, &nn);
		const int l = b->face_cells[2 * f], r = b->face_cells[2 * f + 1];
		side_state(b, l, &b->r_left[3 * f], L, tet);
		side_state(b, r, &b->r_right[3 * f], R, tet);
		const real qqL = L[1] * L[1] + L[2] * L[2] + L[3] * L[3];
		const real HL = (K(0.5) * qqL + gr * L[4] / L[0]);
		const real VL = L[1] * nx + L[2] * ny + L[3] * nz;
		const real qqR = R[1] * R[1] + R[2] * R[2] + R[3] * R[3];
		const real HR = (K(0.5) * qqR + gr * R[4] / R[0]);
		const real VR = R[1] * nx + R[2] * ny + R[3] * nz;
		if (p->flux == 0) {
			const real dp = (R[4] - L[4]), dV = (VR - VL), drho = (R[0] - L[0]);
			const real du = (R[1] - L[1]), dv = (R[2] - L[2]), dw = (R[3] - L[3]);
			const real rw = r_sqrt(L[0] * R[0]);
			const real uw = (L[1] * r_sqrt(L[0]) + R[1] * r_sqrt(R[0])) / (r_sqrt(L[0]) + r_sqrt(R[0]));
			const real vw = (L[2] * r_sqrt(L[0]) + R[2] * r_sqrt(R[0])) / (r_sqrt(L[0]) + r_sqrt(R[0]));
			const real ww = (L[3] * r_sqrt(L[0]) + R[3] * r_sqrt(R[0])) / (r_sqrt(L[0]) + r_sqrt(R[0]));
			const real Hw = (HL * r_sqrt(L[0]) + HR * r_sqrt(R[0])) / (r_sqrt(L[0]) + r_sqrt(R[0]));
			const real q2 = uw * uw + vw * vw + ww * ww;
			const real cw = r_sqrt(gm1 * (Hw - q2 / K(2.)));
			const real Vw = uw * nx + vw * ny + ww * nz;
			const real delta = K(1. / 10.) * cw;
			real L1, L234, L5;
			if (r_fabs(Vw - cw) <= delta) L1 = (r_fabs(Vw - cw) * r_fabs(Vw - cw) + delta * delta) / (K(2.) * delta);
			else L1 = r_fabs(Vw - cw);
			if (r_fabs(Vw) <= delta) L234 = (r_fabs(Vw) * r_fabs(Vw) + delta * delta) / (K(2.) * delta);
			else L234 = r_fabs(Vw);
			if (r_fabs(Vw + cw) <= delta) L5 = (r_fabs(Vw + cw) * r_fabs(Vw + cw) + delta * delta) / (K(2.) * delta);
			else L5 = r_fabs(Vw + cw);
			const real F1 = L1 * (dp - rw * cw * dV) / (K(2.) * cw * cw);
			const real F234 = (drho - dp / (cw * cw));
			const real F5 = L5 * (dp + rw * cw * dV) / (K(2.) * cw * cw);
			const real A0 = F1 * K(1.) + L234 * (F234 * K(1.) + rw * K(0.)) + F5 * K(1.);
			const real A1 = F1 * (uw - cw * nx) + L234 * ((F234 * uw) + rw * (du - dV * nx)) + F5 * (uw + cw * nx);
			const real A2 = F1 * (vw - cw * ny) + L234 * ((F234 * vw) + rw * (dv - dV * ny)) + F5 * (vw + cw * ny);
			const real A3 = F1 * (ww - cw * nz) + L234 * ((F234 * ww) + rw * (dw - dV * nz)) + F5 * (ww + cw * nz);
			const real A4 = F1 * (Hw - cw * Vw) +
			                L234 * ((F234 * q2 / K(2.)) + rw * (uw * du + vw * dv + ww * dw - Vw * dV)) +
			                F5 * (Hw + cw * Vw);
			fl[0] = K(0.5) * (A0)*nn;
			fl[1] = K(0.5) * (A1)*nn;
			fl[2] = K(0.5) * (A2)*nn;
			fl[3] = K(0.5) * (A3)*nn;
			fl[4] = K(0.5) * (A4)*nn;
		} else {
			const real delta = K(0.25);
			const real cL = r_sqrt(g * L[4] / L[0]), ML = VL / cL;
			real MLp, MRm;
			if (ML <= K(-1.0)) MLp = 0;
			else if (ML < K(1.0)) MLp = K(0.25) * (ML + K(1.0)) * (ML + K(1.0));
			else MLp = ML;
			const real cR = r_sqrt(g * R[4] / R[0]), MR = VR / cR;
			if (MR <= K(-1.0)) MRm = MR;
			else if (MR < K(1.0)) MRm = K(-0.25) * (MR - K(1.0)) * (MR - K(1.0));
			else MRm = 0;
			real M = MLp + MRm;
			if (r_fabs(M) > delta) {
			} else {
				M = (M * M + delta * delta) / (K(2.0) * delta);
			}
			const real FL[5] = {L[0] * cL, L[0] * L[1] * cL, L[0] * L[2] * cL, L[0] * L[3] * cL, L[0] * HL * cL};
			const real FR[5] = {R[0] * cR, R[0] * R[1] * cR, R[0] * R[2] * cR, R[0] * R[3] * cR, R[0] * HR * cR};
			for (int q = 0; q < 5; q++) fl[q] = K(0.5) * r_fabs(M) * (-FL[q] + FR[q]) * nn;
		}
		for (int q = 0; q < 5; q++) fl[q] = FLUX_OUT(fl[q], f, q);
		for (int q = 0; q < 5; q++) V5(b->diss_res, n, q, l) = ST(LD(V5(b->diss_res, n, q, l)) + fl[q] * rb);
		for (int q = 0; q < 5; q++) V5(b->diss_res, n, q, r) = ST(LD(V5(b->diss_res, n, q, r)) - fl[q] * rb);
	}
	g_noise_calls++;
}

/* Updater::updateInternalBlock (Solver/src/Updater.cpp:12-78).  FP32 model:
 * the coefficient alpha dt / V and the residual difference in FP32, the update
 * and the primitive recovery in FP64, primitives stored in FP32; wout (when
 * set) receives the FP64 conservative state. */
static void update_internal(e3d_oracle_block* b, const e3d_oracle_params* p, double alpha, double* wout) {
	const int n = b->n_all;
	const double gm1 = (double)K(p->gamma - 1.0);
	for (int c = 0; c < b->n_real; c++) {
		double w[5];
		for (int q = 0; q < 5; q++)
			w[q] = V5(b->w0, n, q, c) - (double)(K(alpha) * LD(b->dt[c]) / LD(b->cell_volume[c])) *
			                                (double)(LD(V5(b->conv_res, n, q, c)) - LD(V5(b->diss_res, n, q, c)));
		V5(b->prim, n, 0, c) = ST(w[0]);
		V5(b->prim, n, 1, c) = ST(w[1] / w[0]);
		V5(b->prim, n, 2, c) = ST(w[2] / w[0]);
		V5(b->prim, n, 3, c) = ST(w[3] / w[0]);
		V5(b->prim, n, 4, c) = ST(gm1 * (w[4] - 0.5 * (w[1] * w[1] + w[2] * w[2] + w[3] * w[3]) / w[0]));
		if (wout)
			for (int q = 0; q < 5; q++) wout[(size_t)q * n + c] = w[q];
	}
}

void e3d_oracle_update_internal(e3d_oracle_block* b, const e3d_oracle_params* p, double alpha) {
	update_internal(b, p, alpha, 0);
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
	double frd[5];
	real fr[5];
	e3d_oracle_freestream(p, frd);
	for (int q = 0; q < 5; q++) fr[q] = K(frd[q]);
	int off = 0;
	for (int j = 0; j < b->n_markers; j++) {
		const int kind = b->marker_kind[j];
		if (j < b->n_real_boundaries && kind != 4) {
			for (int i = 0; i < b->marker_size[j]; i++) {
				const int ext = b->marker_cells[off + i];
				const int f = b->cell_faces[b->cell_face_ptr[ext]];
				const int in = b->cell_cells[b->cell_face_ptr[ext]];
				const double area = b->face_area[f];
				double dx = b->face_normal[3 * f], dy = b->face_normal[3 * f + 1], dz = b->face_normal[3 * f + 2];
				dx /= area;
				dy /= area;
				dz /= area;
				const real nx = K(dx), ny = K(dy), nz = K(dz);
				const real ro = LD(V5(b->prim, n, 0, in)), uu = LD(V5(b->prim, n, 1, in)), vv = LD(V5(b->prim, n, 2, in)),
				           ww = LD(V5(b->prim, n, 3, in)), pp = LD(V5(b->prim, n, 4, in));
				real o[5];
				if (kind == 1 || kind == 3) {
					const real un = uu * nx + vv * ny + ww * nz;
					const real ub = uu - un * nx, vb = vv - un * ny, wb = ww - un * nz;
					o[0] = ro;
					o[1] = K(2.0) * ub - uu;
					o[2] = K(2.0) * vb - vv;
					o[3] = K(2.0) * wb - ww;
					o[4] = pp;
				} else {
					const real c = r_sqrt(K(p->gamma) * pp / ro);
					const real un = uu * nx + vv * ny + ww * nz;
					if (r_fabs(un / c) > K(1.0)) {
						if (un < K(0.0)) {
							o[0] = K(2.0) * fr[0] - ro;
							o[1] = K(2.0) * fr[1] - uu;
							o[2] = K(2.0) * fr[2] - vv;
							o[3] = K(2.0) * fr[3] - ww;
							o[4] = K(2.0) * fr[4] - pp;
						} else {
							o[0] = ro;
							o[1] = uu;
							o[2] = vv;
							o[3] = ww;
							o[4] = pp;
						}
					} else if (un < K(0.0)) {
						const real pb = K(0.5) * (fr[4] + pp - ro * c * (nx * (fr[1] - uu) + ny * (fr[2] - vv) + nz * (fr[3] - ww)));
						const real rb = fr[0] + (pb - fr[4]) / (c * c);
						const real ub = fr[1] - nx * (fr[4] - pb) / (ro * c);
						const real vb = fr[2] - ny * (fr[4] - pb) / (ro * c);
						const real wb = fr[3] - nz * (fr[4] - pb) / (ro * c);
						o[0] = K(2.0) * rb - ro;
						o[1] = K(2.0) * ub - uu;
						o[2] = K(2.0) * vb - vv;
						o[3] = K(2.0) * wb - ww;
						o[4] = K(2.0) * pb - pp;
					} else {
						const real pb = fr[4];
						const real rb = ro + (pb - pp) / (c * c);
						const real ub = uu + nx * (pp - pb) / (ro * c);
						const real vb = vv + ny * (pp - pb) / (ro * c);
						const real wb = ww + nz * (pp - pb) / (ro * c);
						o[0] = K(2.0) * rb - ro;
						o[1] = K(2.0) * ub - uu;
						o[2] = K(2.0) * vb - vv;
						o[3] = K(2.0) * wb - ww;
						o[4] = K(2.0) * pb - pp;
					}
				}
				for (int q = 0; q < 5; q++) V5(b->prim, n, q, ext) = ST(o[q]);
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
	if (first_iter == 0) {
		e3d_oracle_halo(blocks, c, n_connexions);
#if FP32_MODEL
		/* the carried FP64 conservative state starts from the FP64 freestream */
		double f[5];
		e3d_oracle_freestream(p, f);
		for (int bi = 0; bi < n_blocks; bi++) {
			e3d_oracle_block* b = &blocks[bi];
			for (int cc = 0; cc < b->n_real; cc++) {
				V5(b->w0, b->n_all, 0, cc) = f[0];
				V5(b->w0, b->n_all, 1, cc) = f[0] * f[1];
				V5(b->w0, b->n_all, 2, cc) = f[0] * f[2];
				V5(b->w0, b->n_all, 3, cc) = f[0] * f[3];
				V5(b->w0, b->n_all, 4, cc) = 0.5 * f[0] * (f[1] * f[1] + f[2] * f[2] + f[3] * f[3]) + 1. / (p->gamma - 1.0) * f[4];
			}
		}
#endif
	}
	for (int it = 0; it < n_iter; it++) {
		double rms[5] = {0, 0, 0, 0, 0}, cl = 0, cd = 0, cmx = 0, cmy = 0, cmz = 0;
		for (int bi = 0; bi < n_blocks; bi++) {
			e3d_oracle_block* b = &blocks[bi];
			if (!FP32_MODEL) e3d_oracle_save_w0(b, p);
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
				update_internal(b, p, alpha[s], (FP32_MODEL && s == p->stages - 1) ? b->w0 : 0);
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
