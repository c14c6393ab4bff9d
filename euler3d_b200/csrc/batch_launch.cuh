// Batch launchers (persistent cooperative kernel and tiled per-pass form).
// Included by k32.cu and k64.cu with E3D_BATCH_NS = batch, and by k64f.cu
// with E3D_BATCH_NS = batch_fast: the same kernels compiled with FMA
// contraction for the FP64 finishing phase of batched solves.
#pragma once
#include "kernels.cuh"
#include "launch.hpp"

#ifndef E3D_BATCH_NS
#define E3D_BATCH_NS batch
#endif

namespace e3d {
namespace E3D_BATCH_NS {

// ---- persistent batch kernel (cooperative launch)
constexpr int PERSIST_TPB = 128;

template <class T, int GRAD, int LIM, int SCHEME, bool ORDER2>
void* persistent_fn() {
	return reinterpret_cast<void*>(&k_persistent<T, GRAD, LIM, SCHEME, ORDER2, PERSIST_TPB>);
}

template <class T>
void* persistent_select(int grad, int lim, int scheme, bool order2) {
#define E3D_P(G, L, S)                                                                      \
	if (grad == G && lim == L && scheme == S)                                               \
		return order2 ? persistent_fn<T, G, L, S, true>() : persistent_fn<T, G, L, S, false>();
	E3D_P(GRAD_GREEN_GAUSS, LIM_BARTH_JESPERSEN, FLUX_ROE)
	E3D_P(GRAD_GREEN_GAUSS, LIM_BARTH_JESPERSEN, FLUX_AUSM)
	E3D_P(GRAD_GREEN_GAUSS, LIM_VENKATAKRISHNAN, FLUX_ROE)
	E3D_P(GRAD_GREEN_GAUSS, LIM_VENKATAKRISHNAN, FLUX_AUSM)
	E3D_P(GRAD_LEAST_SQUARES, LIM_BARTH_JESPERSEN, FLUX_ROE)
	E3D_P(GRAD_LEAST_SQUARES, LIM_BARTH_JESPERSEN, FLUX_AUSM)
	E3D_P(GRAD_LEAST_SQUARES, LIM_VENKATAKRISHNAN, FLUX_ROE)
	E3D_P(GRAD_LEAST_SQUARES, LIM_VENKATAKRISHNAN, FLUX_AUSM)
#undef E3D_P
	return nullptr;
}

template <class T>
int persistent_blocks_per_sm(int grad, int lim, int scheme, bool order2) {
	int n = 0;
	void* fn = persistent_select<T>(grad, lim, scheme, order2);
	if (!fn || cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, PERSIST_TPB, 0) != cudaSuccess) return 0;
	return n;
}

template <class T>
cudaError_t launch_persistent(const FusedView<T>& v0, const FusedView<T>& v1, const Physics& ph, const PersistArgs& a,
                              int grad, int lim, int scheme, bool order2, int grid, cudaStream_t st) {
	void* fn = persistent_select<T>(grad, lim, scheme, order2);
	if (!fn) return cudaErrorInvalidValue;
	FusedView<T> x0 = v0, x1 = v1;
	Physics p = ph;
	PersistArgs q = a;
	void* args[] = {&x0, &x1, &p, &q};
	return cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(PERSIST_TPB), args, 0, st);
}

// ---- tiled per-pass batch iterations (enqueued on `st`, captured by the caller)
template <class T, int GRAD, int LIM>
void recon_tiles(const FusedView<T>& v, const Physics& ph, int carry, bool first, int n_work, const int4* work,
                 cudaStream_t st) {
	if (first) k_recon_tiles<T, GRAD, LIM, true><<<n_work, 128, 0, st>>>(v, ph, carry, work);
	else k_recon_tiles<T, GRAD, LIM, false><<<n_work, 128, 0, st>>>(v, ph, carry, work);
}

template <class T, int SCHEME>
void flux_tiles(const FusedView<T>& v, const Physics& ph, bool order1, bool diss, T al, T be, int last, int carry,
                int n_work, const int4* work, cudaStream_t st) {
	if (order1) {
		if (diss) k_flux_update_tiles<T, SCHEME, true, true><<<n_work, 128, 0, st>>>(v, ph, al, be, last, carry, work);
		else k_flux_update_tiles<T, SCHEME, true, false><<<n_work, 128, 0, st>>>(v, ph, al, be, last, carry, work);
	} else {
		if (diss) k_flux_update_tiles<T, SCHEME, false, true><<<n_work, 128, 0, st>>>(v, ph, al, be, last, carry, work);
		else k_flux_update_tiles<T, SCHEME, false, false><<<n_work, 128, 0, st>>>(v, ph, al, be, last, carry, work);
	}
}

template <class T>
cudaError_t launch_tiled_iterations(const FusedView<T>& v0, const FusedView<T>& v1, const Physics& ph,
                                    const PersistArgs& a, int grad, int lim, int scheme, bool order2, cudaStream_t st) {
	if (a.n_work <= 0) return cudaSuccess;
	int parity = a.start_parity;
	for (int it = 0; it < a.iters; it++) {
		for (int s = 0; s < a.stages; s++) {
			const FusedView<T>& v = parity ? v1 : v0;
			if (order2) {
				const bool first = s == 0;
				if (grad == GRAD_LEAST_SQUARES) {
					if (lim == LIM_VENKATAKRISHNAN)
						recon_tiles<T, GRAD_LEAST_SQUARES, LIM_VENKATAKRISHNAN>(v, ph, a.carry, first, a.n_work, a.work, st);
					else
						recon_tiles<T, GRAD_LEAST_SQUARES, LIM_BARTH_JESPERSEN>(v, ph, a.carry, first, a.n_work, a.work, st);
				} else {
					if (lim == LIM_VENKATAKRISHNAN)
						recon_tiles<T, GRAD_GREEN_GAUSS, LIM_VENKATAKRISHNAN>(v, ph, a.carry, first, a.n_work, a.work, st);
					else
						recon_tiles<T, GRAD_GREEN_GAUSS, LIM_BARTH_JESPERSEN>(v, ph, a.carry, first, a.n_work, a.work, st);
				}
			} else if (s == 0) {
				k_start_tiles<T><<<a.n_work, 128, 0, st>>>(v, ph, a.carry, a.work);
			}
			const T al = T(a.alpha[s]), be = T(a.beta[s]);
			const int last = s == a.stages - 1;
			const bool diss = a.beta[s] != 0.0;
			if (scheme == FLUX_AUSM) flux_tiles<T, FLUX_AUSM>(v, ph, !order2, diss, al, be, last, a.carry, a.n_work, a.work, st);
			else flux_tiles<T, FLUX_ROE>(v, ph, !order2, diss, al, be, last, a.carry, a.n_work, a.work, st);
			parity ^= 1;
		}
		const FusedView<T>& vf = parity ? v1 : v0;
		k_iter_tail<T><<<a.n_work, 128, 0, st>>>(vf, a);
		k_iter_sums<<<a.nblocks, 128, 0, st>>>(a, it);
	}
	k_iter_add<<<1, 1, 0, st>>>(a.d_iter, a.iters);
	return cudaGetLastError();
}

}  // namespace E3D_BATCH_NS
}  // namespace e3d
