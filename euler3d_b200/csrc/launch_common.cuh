// Launcher templates shared by k64.cu and k32.cu (each instantiates its T).
#pragma once
#include "kernels.cuh"
#include "launch.hpp"

namespace e3d {

template <class T>
void launch_halo(int n, const int* dst, const int* src, int NA, T* b0, T* b1, cudaStream_t st) {
	if (n > 0) k_halo<T><<<(n + 127) / 128, 128, 0, st>>>(n, dst, src, NA, b0, b1);
}

template <class T>
void launch_halo_pack(int n, const int* src, int NA, const T* P, T* buf, cudaStream_t st) {
	if (n > 0) k_halo_pack<T><<<(n + 127) / 128, 128, 0, st>>>(n, src, NA, P, buf);
}

template <class T>
void launch_halo_unpack(int n, const int* dst, int NA, const T* buf, T* b0, T* b1, cudaStream_t st) {
	if (n > 0) k_halo_unpack<T><<<(n + 127) / 128, 128, 0, st>>>(n, dst, NA, buf, b0, b1);
}

template <class T>
void launch_reduce(const ReduceArgs& a, const T* Rc, const T* Rd, const T* P, cudaStream_t st) {
	constexpr int THREADS = 256;
	dim3 grid(a.max_chunks, a.nblocks);
	k_norm_partial<T, THREADS><<<grid, THREADS, 0, st>>>(Rc, Rd, a.NR, a.roff, a.chunk, a.max_chunks, a.partial);
	k_norm_final<<<(a.nblocks * 5 + 127) / 128, 128, 0, st>>>(a.partial, a.nblocks, a.max_chunks, a.hist, a.stride,
	                                                         a.d_iter, a.d_bad);
	if (a.n_wall > 0)
		k_wall_terms<T><<<(a.n_wall + 127) / 128, 128, 0, st>>>(P, a.NA, a.n_wall, a.wall_face, a.face_lr, a.S, a.fc,
		                                                     a.denom, a.wall_denom, a.wall_terms);
	k_wall_sums<<<a.nblocks, 128, 0, st>>>(a.wall_terms, a.n_wall, a.wall_off, a.hist, a.stride, a.d_iter);
}

// FP64 later stages on tetrahedra: one lane per (cell, variable)
// (k_recon_var); build with -DE3D_FP64_RECON_VAR=0 for the one-thread-per-cell pass
#ifndef E3D_FP64_RECON_VAR
#define E3D_FP64_RECON_VAR 1
#endif
template <class T, int GRAD, int LIM>
void recon_dispatch_first(const FusedView<T>& v, const Physics& ph, bool first, int carry, cudaStream_t st) {
	const int grid = (v.NR + 127) / 128;
	if constexpr (sizeof(T) == 8 && E3D_FP64_RECON_VAR) {
		if (v.tet4 && !first) {
			k_recon_var<GRAD, LIM><<<(v.NR + RV_CELLS - 1) / RV_CELLS, 5 * RV_CELLS, 0, st>>>(v, ph);
			return;
		}
	}
	if (v.tet4) {
		if (first) k_recon<T, GRAD, LIM, true, 4><<<grid, 128, 0, st>>>(v, ph, carry);
		else k_recon<T, GRAD, LIM, false, 4><<<grid, 128, 0, st>>>(v, ph, carry);
	} else {
		if (first) k_recon<T, GRAD, LIM, true, 0><<<grid, 128, 0, st>>>(v, ph, carry);
		else k_recon<T, GRAD, LIM, false, 0><<<grid, 128, 0, st>>>(v, ph, carry);
	}
}

template <class T>
void launch_recon(const FusedView<T>& v, const Physics& ph, int grad, int lim, bool first, int carry, cudaStream_t st) {
	if (v.NR <= 0) return;
	if (grad == GRAD_LEAST_SQUARES) {
		if (lim == LIM_VENKATAKRISHNAN)
			recon_dispatch_first<T, GRAD_LEAST_SQUARES, LIM_VENKATAKRISHNAN>(v, ph, first, carry, st);
		else
			recon_dispatch_first<T, GRAD_LEAST_SQUARES, LIM_BARTH_JESPERSEN>(v, ph, first, carry, st);
	} else {
		if (lim == LIM_VENKATAKRISHNAN)
			recon_dispatch_first<T, GRAD_GREEN_GAUSS, LIM_VENKATAKRISHNAN>(v, ph, first, carry, st);
		else
			recon_dispatch_first<T, GRAD_GREEN_GAUSS, LIM_BARTH_JESPERSEN>(v, ph, first, carry, st);
	}
}

template <class T>
void launch_start(const FusedView<T>& v, const Physics& ph, int carry, cudaStream_t st) {
	if (v.NR <= 0) return;
	if (v.tet4) k_start<T, 4><<<(v.NR + 127) / 128, 128, 0, st>>>(v, ph, carry);
	else k_start<T, 0><<<(v.NR + 127) / 128, 128, 0, st>>>(v, ph, carry);
}

template <class T>
void launch_flux_update(const FusedView<T>& v, const Physics& ph, int scheme, bool order1, double alpha, double beta,
                        int last, int carry, cudaStream_t st) {
	if (v.NR <= 0) return;
	const int grid = (v.NR + 127) / 128;
	const T a = T(alpha), b = T(beta);
#define E3D_FLUX(S, O)                                                                                  \
	do {                                                                                                \
		if (beta != 0.0) {                                                                              \
			if (v.tet4) k_flux_update<T, S, O, 4, true><<<grid, 128, 0, st>>>(v, ph, a, b, last, carry);  \
			else k_flux_update<T, S, O, 0, true><<<grid, 128, 0, st>>>(v, ph, a, b, last, carry);         \
		} else {                                                                                        \
			if (v.tet4) k_flux_update<T, S, O, 4, false><<<grid, 128, 0, st>>>(v, ph, a, b, last, carry); \
			else k_flux_update<T, S, O, 0, false><<<grid, 128, 0, st>>>(v, ph, a, b, last, carry);        \
		}                                                                                               \
	} while (0)
	if (scheme == FLUX_AUSM) {
		if (order1) E3D_FLUX(FLUX_AUSM, true);
		else E3D_FLUX(FLUX_AUSM, false);
	} else {
		if (order1) E3D_FLUX(FLUX_ROE, true);
		else E3D_FLUX(FLUX_ROE, false);
	}
#undef E3D_FLUX
}

}  // namespace e3d
