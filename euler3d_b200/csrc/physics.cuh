// Per-face and per-cell arithmetic of the residual/update path, templated on
// the working precision T (double: drop-in path; float: FP32 variant).
//
// Every expression keeps the reference's operand order and parenthesisation so
// that, built with -fmad=false, the double instantiation reproduces the
// reference's FP64 results bit for bit (IEEE division and square root are
// correctly rounded on both the CPU and the GPU).
#pragma once
#include <cuda_runtime.h>
#include <math.h>

namespace e3d {

template <class T>
struct Q5 {
	T r, u, v, w, p;
};

__host__ __device__ __forceinline__ double tabs(double x) { return fabs(x); }
__host__ __device__ __forceinline__ float tabs(float x) { return fabsf(x); }
__host__ __device__ __forceinline__ double tsqrt(double x) { return sqrt(x); }
__host__ __device__ __forceinline__ float tsqrt(float x) { return sqrtf(x); }
__host__ __device__ __forceinline__ double tmin(double a, double b) { return fmin(a, b); }
__host__ __device__ __forceinline__ float tmin(float a, float b) { return fminf(a, b); }
__host__ __device__ __forceinline__ double tcopysign(double a, double b) { return copysign(a, b); }
__host__ __device__ __forceinline__ float tcopysign(float a, float b) { return copysignf(a, b); }

// MUSCL value at a face: q + phi*g0*r0 + phi*g1*r1 + phi*g2*r2, accumulated in
// that order (FluxScheme.cpp:127-134).
template <class T>
__device__ __forceinline__ T recon(T q, T phi, T g0, T g1, T g2, T r0, T r1, T r2) {
	q += phi * g0 * r0;
	q += phi * g1 * r1;
	q += phi * g2 * r2;
	return q;
}

// Central convective flux 0.5*(F_L+F_R)*|S| (FluxScheme.cpp:161-192).
// gr = gamma/(gamma-1).
template <class T>
__device__ __forceinline__ void flux_central(const Q5<T>& L, const Q5<T>& R, T nx, T ny, T nz, T nn, T gr, T f[5]) {
	const T qqL = L.u * L.u + L.v * L.v + L.w * L.w;
	const T HL = (T(0.5) * qqL + gr * L.p / L.r);
	const T VL = L.u * nx + L.v * ny + L.w * nz;
	const T qqR = R.u * R.u + R.v * R.v + R.w * R.w;
	const T HR = (T(0.5) * qqR + gr * R.p / R.r);
	const T VR = R.u * nx + R.v * ny + R.w * nz;
	const T FL1 = L.r * VL, FR1 = R.r * VR;
	const T FL2 = L.r * L.u * VL + nx * L.p, FR2 = R.r * R.u * VR + nx * R.p;
	const T FL3 = L.r * L.v * VL + ny * L.p, FR3 = R.r * R.v * VR + ny * R.p;
	const T FL4 = L.r * L.w * VL + nz * L.p, FR4 = R.r * R.w * VR + nz * R.p;
	const T FL5 = L.r * HL * VL, FR5 = R.r * HR * VR;
	f[0] = T(0.5) * (FL1 + FR1) * nn;
	f[1] = T(0.5) * (FL2 + FR2) * nn;
	f[2] = T(0.5) * (FL3 + FR3) * nn;
	f[3] = T(0.5) * (FL4 + FR4) * nn;
	f[4] = T(0.5) * (FL5 + FR5) * nn;
}

// Roe dissipative flux 0.5*|A_roe|(U_R-U_L)*|S| with Harten's entropy fix
// delta = c/10 (RoeScheme.cpp:159-270).  gm1 = gamma-1.
template <class T>
__device__ __forceinline__ void flux_roe_diss(const Q5<T>& L, const Q5<T>& R, T nx, T ny, T nz, T nn, T gr, T gm1,
                                              T f[5]) {
	const T qqL = L.u * L.u + L.v * L.v + L.w * L.w;
	const T HL = (T(0.5) * qqL + gr * L.p / L.r);
	const T VL = L.u * nx + L.v * ny + L.w * nz;
	const T qqR = R.u * R.u + R.v * R.v + R.w * R.w;
	const T HR = (T(0.5) * qqR + gr * R.p / R.r);
	const T VR = R.u * nx + R.v * ny + R.w * nz;
	const T dp = (R.p - L.p), dV = (VR - VL), drho = (R.r - L.r);
	const T du = (R.u - L.u), dv = (R.v - L.v), dw = (R.w - L.w);
	const T sL = tsqrt(L.r), sR = tsqrt(R.r);
	const T rw = tsqrt(L.r * R.r);
	const T uw = (L.u * sL + R.u * sR) / (sL + sR);
	const T vw = (L.v * sL + R.v * sR) / (sL + sR);
	const T ww = (L.w * sL + R.w * sR) / (sL + sR);
	const T Hw = (HL * sL + HR * sR) / (sL + sR);
	const T q2w = uw * uw + vw * vw + ww * ww;
	const T cw = tsqrt(gm1 * (Hw - q2w / T(2.)));
	const T Vw = uw * nx + vw * ny + ww * nz;
	const T delta = T(0.1) * cw;
	const T a1 = tabs(Vw - cw), a234 = tabs(Vw), a5 = tabs(Vw + cw);
	const T L1 = (a1 <= delta) ? (a1 * a1 + delta * delta) / (T(2.) * delta) : a1;
	const T L234 = (a234 <= delta) ? (a234 * a234 + delta * delta) / (T(2.) * delta) : a234;
	const T L5 = (a5 <= delta) ? (a5 * a5 + delta * delta) / (T(2.) * delta) : a5;
	const T F1c = L1 * (dp - rw * cw * dV) / (T(2.) * cw * cw);
	const T F1m = F1c * T(1.);
	const T F1u = F1c * (uw - cw * nx);
	const T F1v = F1c * (vw - cw * ny);
	const T F1w = F1c * (ww - cw * nz);
	const T F1e = F1c * (Hw - cw * Vw);
	const T F234c = (drho - dp / (cw * cw));
	const T F234m = L234 * (F234c * T(1.) + rw * T(0.));
	const T F234u = L234 * ((F234c * uw) + rw * (du - dV * nx));
	const T F234v = L234 * ((F234c * vw) + rw * (dv - dV * ny));
	const T F234w = L234 * ((F234c * ww) + rw * (dw - dV * nz));
	const T F234e = L234 * ((F234c * q2w / T(2.)) + rw * (uw * du + vw * dv + ww * dw - Vw * dV));
	const T F5c = L5 * (dp + rw * cw * dV) / (T(2.) * cw * cw);
	const T F5m = F5c * T(1.);
	const T F5u = F5c * (uw + cw * nx);
	const T F5v = F5c * (vw + cw * ny);
	const T F5w = F5c * (ww + cw * nz);
	const T F5e = F5c * (Hw + cw * Vw);
	f[0] = T(0.5) * (F1m + F234m + F5m) * nn;
	f[1] = T(0.5) * (F1u + F234u + F5u) * nn;
	f[2] = T(0.5) * (F1v + F234v + F5v) * nn;
	f[3] = T(0.5) * (F1w + F234w + F5w) * nn;
	f[4] = T(0.5) * (F1e + F234e + F5e) * nn;
}

// Liou-Steffen AUSM convective flux (AusmScheme.cpp:716-871).  g = gamma.
template <class T>
__device__ __forceinline__ void flux_ausm_conv(const Q5<T>& L, const Q5<T>& R, T nx, T ny, T nz, T nn, T g, T gr,
                                               T f[5]) {
	const T qqL = L.u * L.u + L.v * L.v + L.w * L.w;
	const T HL = (T(0.5) * qqL + gr * L.p / L.r);
	const T VL = L.u * nx + L.v * ny + L.w * nz;
	const T cL = tsqrt(g * L.p / L.r);
	const T ML = VL / cL;
	T pLp, MLp;
	if (ML <= T(-1.0)) {
		pLp = T(0);
		MLp = T(0);
	} else if (ML < T(1.0)) {
		pLp = L.p * T(0.25) * (ML + T(1.0)) * (ML + T(1.0)) * (T(2.0) - ML);
		MLp = T(0.25) * (ML + T(1.0)) * (ML + T(1.0));
	} else {
		MLp = ML;
		pLp = L.p;
	}
	const T qqR = R.u * R.u + R.v * R.v + R.w * R.w;
	const T HR = (T(0.5) * qqR + gr * R.p / R.r);
	const T VR = R.u * nx + R.v * ny + R.w * nz;
	const T cR = tsqrt(g * R.p / R.r);
	const T MR = VR / cR;
	T pRm, MRm;
	if (MR <= T(-1.0)) {
		pRm = R.p;
		MRm = MR;
	} else if (MR < T(1.0)) {
		pRm = R.p * T(0.25) * (T(1.0) - MR) * (T(1.0) - MR) * (T(2.0) + MR);
		MRm = T(-0.25) * (MR - T(1.0)) * (MR - T(1.0));
	} else {
		pRm = T(0);
		MRm = T(0);
	}
	const T M = MLp + MRm;
	const T FL1 = L.r * cL, FR1 = R.r * cR;
	const T FL2 = L.r * L.u * cL, FR2 = R.r * R.u * cR;
	const T FL3 = L.r * L.v * cL, FR3 = R.r * R.v * cR;
	const T FL4 = L.r * L.w * cL, FR4 = R.r * R.w * cR;
	const T FL5 = L.r * HL * cL, FR5 = R.r * HR * cR;
	f[0] = T(0.5) * M * (FL1 + FR1) * nn;
	f[1] = T(0.5) * M * (FL2 + FR2) * nn + nx * (pLp + pRm) * nn;
	f[2] = T(0.5) * M * (FL3 + FR3) * nn + ny * (pLp + pRm) * nn;
	f[3] = T(0.5) * M * (FL4 + FR4) * nn + nz * (pLp + pRm) * nn;
	f[4] = T(0.5) * M * (FL5 + FR5) * nn;
}

// AUSM dissipative flux 0.5*|M_LR|(F_R-F_L)*|S| with the |M|<=0.25 fix
// (AusmScheme.cpp:102-243).
template <class T>
__device__ __forceinline__ void flux_ausm_diss(const Q5<T>& L, const Q5<T>& R, T nx, T ny, T nz, T nn, T g, T gr,
                                               T f[5]) {
	const T delta = T(0.25);
	const T qqL = L.u * L.u + L.v * L.v + L.w * L.w;
	const T HL = (T(0.5) * qqL + gr * L.p / L.r);
	const T VL = L.u * nx + L.v * ny + L.w * nz;
	const T cL = tsqrt(g * L.p / L.r);
	const T ML = VL / cL;
	T MLp;
	if (ML <= T(-1.0)) MLp = T(0);
	else if (ML < T(1.0)) MLp = T(0.25) * (ML + T(1.0)) * (ML + T(1.0));
	else MLp = ML;
	const T qqR = R.u * R.u + R.v * R.v + R.w * R.w;
	const T HR = (T(0.5) * qqR + gr * R.p / R.r);
	const T VR = R.u * nx + R.v * ny + R.w * nz;
	const T cR = tsqrt(g * R.p / R.r);
	const T MR = VR / cR;
	T MRm;
	if (MR <= T(-1.0)) MRm = MR;
	else if (MR < T(1.0)) MRm = T(-0.25) * (MR - T(1.0)) * (MR - T(1.0));
	else MRm = T(0);
	T M = MLp + MRm;
	if (!(tabs(M) > delta)) M = (M * M + delta * delta) / (T(2.0) * delta);
	const T FL1 = L.r * cL, FR1 = R.r * cR;
	const T FL2 = L.r * L.u * cL, FR2 = R.r * R.u * cR;
	const T FL3 = L.r * L.v * cL, FR3 = R.r * R.v * cR;
	const T FL4 = L.r * L.w * cL, FR4 = R.r * R.w * cR;
	const T FL5 = L.r * HL * cL, FR5 = R.r * HR * cR;
	const T aM = tabs(M);
	f[0] = T(0.5) * aM * (-FL1 + FR1) * nn;
	f[1] = T(0.5) * aM * (-FL2 + FR2) * nn;
	f[2] = T(0.5) * aM * (-FL3 + FR3) * nn;
	f[3] = T(0.5) * aM * (-FL4 + FR4) * nn;
	f[4] = T(0.5) * aM * (-FL5 + FR5) * nn;
}

// Barth-Jespersen face limiter with the omega shift (BarthJespersen.cpp:226-245).
template <class T>
__device__ __forceinline__ T limiter_bj_face(T d2, T dmax, T dmin, T omega) {
	d2 = (tcopysign(T(1.0), d2)) * (tabs(d2) + omega);
	if (d2 > T(0.0)) return tmin(T(1.0), dmax / d2);
	if (d2 < T(0.0)) return tmin(T(1.0), dmin / d2);
	return T(1.0);
}

// Venkatakrishnan face limiter, eps2 = K^3 * V (Venkatakrishnan.cpp:92,227-238).
// The double version keeps the reference's expression (two divisions); the
// float version uses the same function with d2 cancelled from numerator and
// denominator, (D^2+eps2+2 d2 D) / (D^2+eps2 + d2 (2 d2 + D)), one division.
template <class T>
__device__ __forceinline__ T limiter_venkat_face(T d2, T dmax, T dmin, T eps2);
template <>
__device__ __forceinline__ float limiter_venkat_face<float>(float d2, float dmax, float dmin, float eps2) {
	if (!(d2 > 0.0f) && !(d2 < 0.0f)) return 1.0f;  // zero or NaN, as the reference's branches
	const float D = d2 > 0.0f ? dmax : dmin;
	const float A = fmaf(D, D, eps2);
	return fmaf(2.0f * d2, D, A) / fmaf(d2, fmaf(2.0f, d2, D), A);
}
template <>
__device__ __forceinline__ double limiter_venkat_face<double>(double d2, double dmax, double dmin, double eps2) {
	if (d2 > double(0.0))
		return (double(1.0) / d2) * ((dmax * dmax + eps2) * d2 + double(2.0) * d2 * d2 * dmax) /
		       (dmax * dmax + double(2.0) * d2 * d2 + dmax * d2 + eps2);
	if (d2 < double(0.0))
		return (double(1.0) / d2) * ((dmin * dmin + eps2) * d2 + double(2.0) * d2 * d2 * dmin) /
		       (dmin * dmin + double(2.0) * d2 * d2 + dmin * d2 + eps2);
	return double(1.0);
}

// Slip wall / symmetry ghost state (WallCellIds.cpp:40-62, SymmetryCellIds.cpp:41-63).
template <class T>
__device__ __forceinline__ Q5<T> bc_slip(const Q5<T>& q, T nx, T ny, T nz) {
	const T un = q.u * nx + q.v * ny + q.w * nz;
	const T ub = q.u - un * nx, vb = q.v - un * ny, wb = q.w - un * nz;
	Q5<T> o;
	o.r = q.r;
	o.u = T(2.0) * ub - q.u;
	o.v = T(2.0) * vb - q.v;
	o.w = T(2.0) * wb - q.w;
	o.p = q.p;
	return o;
}

// Characteristic farfield ghost state (FarfieldCellIds.cpp:53-113).
template <class T>
__device__ __forceinline__ Q5<T> bc_farfield(const Q5<T>& q, const Q5<T>& fr, T nx, T ny, T nz, T g) {
	const T c = tsqrt(g * q.p / q.r);
	const T un = q.u * nx + q.v * ny + q.w * nz;
	Q5<T> o;
	if (tabs(un / c) > T(1.0)) {
		if (un < T(0.0)) {
			o.r = T(2.0) * fr.r - q.r;
			o.u = T(2.0) * fr.u - q.u;
			o.v = T(2.0) * fr.v - q.v;
			o.w = T(2.0) * fr.w - q.w;
			o.p = T(2.0) * fr.p - q.p;
		} else {
			o = q;
		}
	} else if (un < T(0.0)) {
		const T pb = T(0.5) * (fr.p + q.p - q.r * c * (nx * (fr.u - q.u) + ny * (fr.v - q.v) + nz * (fr.w - q.w)));
		const T rb = fr.r + (pb - fr.p) / (c * c);
		const T ub = fr.u - nx * (fr.p - pb) / (q.r * c);
		const T vb = fr.v - ny * (fr.p - pb) / (q.r * c);
		const T wb = fr.w - nz * (fr.p - pb) / (q.r * c);
		o.r = T(2.0) * rb - q.r;
		o.u = T(2.0) * ub - q.u;
		o.v = T(2.0) * vb - q.v;
		o.w = T(2.0) * wb - q.w;
		o.p = T(2.0) * pb - q.p;
	} else {
		const T pb = fr.p;
		const T rb = q.r + (pb - q.p) / (c * c);
		const T ub = q.u + nx * (q.p - pb) / (q.r * c);
		const T vb = q.v + ny * (q.p - pb) / (q.r * c);
		const T wb = q.w + nz * (q.p - pb) / (q.r * c);
		o.r = T(2.0) * rb - q.r;
		o.u = T(2.0) * ub - q.u;
		o.v = T(2.0) * vb - q.v;
		o.w = T(2.0) * wb - q.w;
		o.p = T(2.0) * pb - q.p;
	}
	return o;
}

// Ghost gradient: interior gradient reflected about the face plane
// (GreenGauss.cpp:199-230, LeastSquares.cpp:151-182).
template <class T>
__device__ __forceinline__ void reflect_grad(const T gi[3], T nx, T ny, T nz, T go[3]) {
	T dot = T(0.0);
	dot += gi[0] * nx;
	dot += gi[1] * ny;
	dot += gi[2] * nz;
	go[0] = gi[0] - T(2.0) * dot * nx;
	go[1] = gi[1] - T(2.0) * dot * ny;
	go[2] = gi[2] - T(2.0) * dot * nz;
}

}  // namespace e3d
