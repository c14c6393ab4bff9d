// Surrogate inputs, warm-start state writes and FP32 -> FP64 widening.
#include <cmath>

#include "warm.hpp"

namespace e3d {
namespace {

constexpr int TPB = 256;
inline int grid_for(long long n) { return (int)((n + TPB - 1) / TPB); }

__device__ __forceinline__ int block_of(const int* __restrict__ roff, int nb, int c) {
	int lo = 0, hi = nb;  // roff[lo] <= c < roff[hi]
	while (hi - lo > 1) {
		const int mid = (lo + hi) >> 1;
		if (roff[mid] <= c) lo = mid;
		else hi = mid;
	}
	return lo;
}

__global__ void k_slot_geometry64(int NS, const int* __restrict__ slot_face, const int* __restrict__ slot_mate,
                                  const double* __restrict__ S, const double* __restrict__ nhat,
                                  const double* __restrict__ area, const double* __restrict__ rl,
                                  const double* __restrict__ rr, double* __restrict__ sgeo, double* __restrict__ sS,
                                  double* __restrict__ srv) {
	const int k = blockIdx.x * blockDim.x + threadIdx.x;
	if (k >= NS) return;
	const int F = slot_face[k];
	const bool left = slot_mate[k] >= 0;
	for (int d = 0; d < 3; d++) {
		sgeo[4 * (size_t)k + d] = nhat[3 * (size_t)F + d];
		if (sS) sS[3 * (size_t)k + d] = left ? S[3 * (size_t)F + d] : -S[3 * (size_t)F + d];
		srv[3 * (size_t)k + d] = left ? rl[3 * (size_t)F + d] : rr[3 * (size_t)F + d];
	}
	sgeo[4 * (size_t)k + 3] = area[F];
}

__global__ void k_widen_state(int NA, int NR, const float* __restrict__ P32, const double* __restrict__ W, double gm1,
                              double* __restrict__ P0, double* __restrict__ P1) {
	const int c = blockIdx.x * blockDim.x + threadIdx.x;
	if (c >= NA) return;
	double q[5];
	if (W && c < NR) {
		const double r = W[c];
		q[0] = r;
		q[1] = W[(size_t)NR + c] / r;
		q[2] = W[2 * (size_t)NR + c] / r;
		q[3] = W[3 * (size_t)NR + c] / r;
		q[4] = gm1 * (W[4 * (size_t)NR + c] - 0.5 * r * (q[1] * q[1] + q[2] * q[2] + q[3] * q[3]));
	} else {
		for (int v = 0; v < 4; v++) q[v] = (double)P32[4 * (size_t)c + v];
		q[4] = (double)P32[4 * (size_t)NA + c];
	}
	for (int v = 0; v < 4; v++) P0[4 * (size_t)c + v] = q[v];
	P0[4 * (size_t)NA + c] = q[4];
	if (P1) {
		for (int v = 0; v < 4; v++) P1[4 * (size_t)c + v] = q[v];
		P1[4 * (size_t)NA + c] = q[4];
	}
}

__global__ void k_narrow_state(size_t n, const double* __restrict__ P64, float* __restrict__ P32) {
	const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
	if (i < n) P32[i] = (float)P64[i];
}

__global__ void k_cell_features(int NR, int nb, const int* __restrict__ roff, const int* __restrict__ block_case,
                                const float* __restrict__ cen, const int* __restrict__ case_wall_off,
                                const int* __restrict__ wall_face, const double* __restrict__ fc,
                                const float* __restrict__ case_ma, float* __restrict__ out) {
	const int c = blockIdx.x * blockDim.x + threadIdx.x;
	if (c >= NR) return;
	const int cs = block_case[block_of(roff, nb, c)];
	const float x = cen[3 * (size_t)c], y = cen[3 * (size_t)c + 1], z = cen[3 * (size_t)c + 2];
	float d2 = 3.4e38f;
	const int w0 = case_wall_off[cs], w1 = case_wall_off[cs + 1];
	for (int i = w0; i < w1; i++) {
		const int f = wall_face[i];
		const float dx = x - (float)fc[3 * (size_t)f], dy = y - (float)fc[3 * (size_t)f + 1],
		            dz = z - (float)fc[3 * (size_t)f + 2];
		d2 = fminf(d2, dx * dx + dy * dy + dz * dz);
	}
	float* o = out + 8 * (size_t)c;
	o[0] = x;
	o[1] = y;
	o[2] = z;
	o[3] = w1 > w0 ? sqrtf(d2) : 1.f;
	o[4] = case_ma[2 * cs];
	o[5] = case_ma[2 * cs + 1];
	o[6] = 0.f;
	o[7] = 0.f;
}

template <class T>
__global__ void k_apply_conservative(int NR, int NA, int nb, const int* __restrict__ roff,
                                     const int* __restrict__ block_case, const float* __restrict__ Wp, int ld,
                                     const double* __restrict__ case_free, double gamma, T* __restrict__ P0,
                                     T* __restrict__ P1, double* __restrict__ W, int* __restrict__ n_fallback) {
	const int c = blockIdx.x * blockDim.x + threadIdx.x;
	if (c >= NR) return;
	const int cs = block_case[block_of(roff, nb, c)];
	const double* f = case_free + 5 * (size_t)cs;
	const double gm1 = gamma - 1.0;
	double w[5];
	for (int v = 0; v < 5; v++) w[v] = (double)Wp[(size_t)ld * c + v];
	double q[5];
	q[0] = w[0];
	q[1] = w[1] / w[0];
	q[2] = w[2] / w[0];
	q[3] = w[3] / w[0];
	q[4] = gm1 * (w[4] - 0.5 * w[0] * (q[1] * q[1] + q[2] * q[2] + q[3] * q[3]));
	bool ok = true;
	for (int v = 0; v < 5; v++) ok = ok && isfinite(q[v]);
	ok = ok && q[0] > 1e-3 * f[0] && q[4] > 1e-3 * f[4];
	if (!ok) {
		for (int v = 0; v < 5; v++) q[v] = f[v];
		w[0] = f[0];
		w[1] = f[0] * f[1];
		w[2] = f[0] * f[2];
		w[3] = f[0] * f[3];
		w[4] = 0.5 * f[0] * (f[1] * f[1] + f[2] * f[2] + f[3] * f[3]) + 1. / gm1 * f[4];
		atomicAdd(n_fallback, 1);
	}
	for (int v = 0; v < 4; v++) {
		P0[4 * (size_t)c + v] = (T)q[v];
		P1[4 * (size_t)c + v] = (T)q[v];
	}
	P0[4 * (size_t)NA + c] = (T)q[4];
	P1[4 * (size_t)NA + c] = (T)q[4];
	if (W)
		for (int v = 0; v < 5; v++) W[(size_t)v * NR + c] = w[v];
}

template <class T>
__global__ void k_prims_to_conservative(int NR, int NA, const T* __restrict__ P, double gamma, float* __restrict__ out) {
	const int c = blockIdx.x * blockDim.x + threadIdx.x;
	if (c >= NR) return;
	const double r = (double)P[4 * (size_t)c], u = (double)P[4 * (size_t)c + 1], v = (double)P[4 * (size_t)c + 2],
	             w = (double)P[4 * (size_t)c + 3], p = (double)P[4 * (size_t)NA + c];
	float* o = out + 8 * (size_t)c;
	o[0] = (float)r;
	o[1] = (float)(r * u);
	o[2] = (float)(r * v);
	o[3] = (float)(r * w);
	o[4] = (float)(0.5 * r * (u * u + v * v + w * w) + p / (gamma - 1.0));
	o[5] = o[6] = o[7] = 0.f;
}

}  // namespace

template <class T>
void launch_prims_to_conservative(int NR, int NA, const T* P, double gamma, float* out, cudaStream_t st) {
	if (NR > 0) k_prims_to_conservative<T><<<grid_for(NR), TPB, 0, st>>>(NR, NA, P, gamma, out);
}
template void launch_prims_to_conservative<float>(int, int, const float*, double, float*, cudaStream_t);
template void launch_prims_to_conservative<double>(int, int, const double*, double, float*, cudaStream_t);

void launch_slot_geometry64(int NS, const int* slot_face, const int* slot_mate, const double* S, const double* nhat,
                            const double* area, const double* rl, const double* rr, double* sgeo, double* sS,
                            double* srv, cudaStream_t st) {
	if (NS > 0)
		k_slot_geometry64<<<grid_for(NS), TPB, 0, st>>>(NS, slot_face, slot_mate, S, nhat, area, rl, rr, sgeo, sS, srv);
}

void launch_widen_state(int NA, int NR, const float* P32, const double* W, double gm1, double* P0, double* P1,
                        cudaStream_t st) {
	if (NA > 0) k_widen_state<<<grid_for(NA), TPB, 0, st>>>(NA, NR, P32, W, gm1, P0, P1);
}

void launch_narrow_state(int NA, const double* P64, float* P32, cudaStream_t st) {
	if (NA > 0) k_narrow_state<<<grid_for(5LL * NA), TPB, 0, st>>>(5 * (size_t)NA, P64, P32);
}

void launch_cell_features(int NR, int nb, const int* roff, const int* block_case, const float* centroid,
                          const int* case_wall_off, const int* wall_face, const double* fc, const float* case_mach_aoa,
                          float* out, cudaStream_t st) {
	if (NR > 0)
		k_cell_features<<<grid_for(NR), TPB, 0, st>>>(NR, nb, roff, block_case, centroid, case_wall_off, wall_face, fc,
		                                                case_mach_aoa, out);
}

template <class T>
void launch_apply_conservative(int NR, int NA, int nb, const int* roff, const int* block_case, const float* Wpred,
                               int ld, const double* case_free, double gamma, T* P0, T* P1, double* W,
                               int* n_fallback, cudaStream_t st) {
	if (NR > 0)
		k_apply_conservative<T><<<grid_for(NR), TPB, 0, st>>>(NR, NA, nb, roff, block_case, Wpred, ld, case_free,
		                                                      gamma, P0, P1, W, n_fallback);
}

template void launch_apply_conservative<float>(int, int, int, const int*, const int*, const float*, int,
                                               const double*, double, float*, float*, double*, int*, cudaStream_t);
template void launch_apply_conservative<double>(int, int, int, const int*, const int*, const float*, int,
                                                const double*, double, double*, double*, double*, int*, cudaStream_t);

}  // namespace e3d
