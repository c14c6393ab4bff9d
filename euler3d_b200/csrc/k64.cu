// FP64 kernels.  This translation unit is built with -fmad=false: no multiply-
// add contraction, so every double expression rounds exactly as the
// reference's x86-64 build does.
#include "kernels.cuh"
#include "launch.hpp"
#include "launch_common.cuh"
#include "batch_launch.cuh"

namespace e3d {

namespace {
inline int blocks_for(int n, int t) { return (n + t - 1) / t; }
constexpr int TPB = 128;
}  // namespace

void launch_save_w0(const GeoView& g, const StateView& s, const Physics& ph, int r0, int r1, cudaStream_t st) {
	if (r1 > r0) k_save_w0<<<blocks_for(r1 - r0, TPB), TPB, 0, st>>>(g, s, ph, r0, r1);
}
void launch_spectral_radius(const GeoView& g, const StateView& s, const Physics& ph, int r0, int r1, cudaStream_t st) {
	if (r1 > r0) k_spectral_radius<<<blocks_for(r1 - r0, TPB), TPB, 0, st>>>(g, s, ph, r0, r1);
}
void launch_timestep(const GeoView& g, const StateView& s, const Physics& ph, int r0, int r1, cudaStream_t st) {
	if (r1 > r0) k_timestep<<<blocks_for(r1 - r0, TPB), TPB, 0, st>>>(g, s, ph, r0, r1);
}
void launch_gradients(const GeoView& g, const StateView& s, int kind, int r0, int r1, cudaStream_t st) {
	if (r1 <= r0) return;
	if (kind == GRAD_LEAST_SQUARES) k_grad_ls<<<blocks_for(r1 - r0, TPB), TPB, 0, st>>>(g, s, r0, r1);
	else k_grad_gg<<<blocks_for(r1 - r0, TPB), TPB, 0, st>>>(g, s, r0, r1);
}
void launch_limiters(const GeoView& g, const StateView& s, const Physics& ph, int kind, int r0, int r1, int g0, int g1,
                     cudaStream_t st) {
	const int n = (r1 - r0) + (g1 - g0);
	if (n <= 0) return;
	if (kind == LIM_VENKATAKRISHNAN)
		k_limiter<LIM_VENKATAKRISHNAN><<<blocks_for(n, TPB), TPB, 0, st>>>(g, s, ph, r0, r1, g0, g1);
	else
		k_limiter<LIM_BARTH_JESPERSEN><<<blocks_for(n, TPB), TPB, 0, st>>>(g, s, ph, r0, r1, g0, g1);
}
void launch_flux_conv(const GeoView& g, const StateView& s, const Physics& ph, int scheme, int r0, int r1,
                      cudaStream_t st) {
	if (r1 <= r0) return;
	if (scheme == FLUX_AUSM) k_flux_conv<FLUX_AUSM><<<blocks_for(r1 - r0, TPB), TPB, 0, st>>>(g, s, ph, r0, r1);
	else k_flux_conv<FLUX_ROE><<<blocks_for(r1 - r0, TPB), TPB, 0, st>>>(g, s, ph, r0, r1);
}
void launch_flux_diss(const GeoView& g, const StateView& s, const Physics& ph, int scheme, double beta, int r0, int r1,
                      cudaStream_t st) {
	if (r1 <= r0) return;
	if (scheme == FLUX_AUSM)
		k_flux_diss<FLUX_AUSM><<<blocks_for(r1 - r0, TPB), TPB, 0, st>>>(g, s, ph, beta, r0, r1);
	else
		k_flux_diss<FLUX_ROE><<<blocks_for(r1 - r0, TPB), TPB, 0, st>>>(g, s, ph, beta, r0, r1);
}
void launch_update(const GeoView& g, const StateView& s, const Physics& ph, double alpha, int r0, int r1,
                   cudaStream_t st) {
	if (r1 > r0) k_update<<<blocks_for(r1 - r0, TPB), TPB, 0, st>>>(g, s, ph, alpha, r0, r1);
}
void launch_bc(const GeoView& g, const StateView& s, const Physics& ph, int g0, int g1, cudaStream_t st) {
	if (g1 > g0) k_bc<<<blocks_for(g1 - g0, TPB), TPB, 0, st>>>(g, s, ph, g0, g1);
}
void launch_iter_advance(int* d_iter, cudaStream_t st) { k_iter_advance<<<1, 1, 0, st>>>(d_iter); }
void launch_smooth(const GeoView& g, const StateView& s, double* j1, int r0, int r1, cudaStream_t st) {
	if (r1 <= r0) return;
	k_irs_start<<<blocks_for(r1 - r0, TPB), TPB, 0, st>>>(g, s, j1, r0, r1);
	k_irs_smooth<<<blocks_for(r1 - r0, TPB), TPB, 0, st>>>(g, s, j1, r0, r1);
}

template void launch_halo<double>(int, const int*, const int*, int, double*, double*, cudaStream_t);
template void launch_halo_pack<double>(int, const int*, int, const double*, double*, cudaStream_t);
template void launch_halo_unpack<double>(int, const int*, int, const double*, double*, double*, cudaStream_t);
template void launch_reduce<double>(const ReduceArgs&, const double*, const double*, const double*, cudaStream_t);
template void launch_recon<double>(const FusedView<double>&, const Physics&, int, int, bool, int, cudaStream_t);
template void launch_start<double>(const FusedView<double>&, const Physics&, int, cudaStream_t);
template void launch_flux_update<double>(const FusedView<double>&, const Physics&, int, bool, double, double, int, int,
                                         cudaStream_t);
template int batch::persistent_blocks_per_sm<double>(int, int, int, bool);
template cudaError_t batch::launch_persistent<double>(const FusedView<double>&, const FusedView<double>&, const Physics&,
                                               const PersistArgs&, int, int, int, bool, int, cudaStream_t);

template cudaError_t batch::launch_tiled_iterations<double>(const FusedView<double>&, const FusedView<double>&, const Physics&,
                                                    const PersistArgs&, int, int, int, bool, cudaStream_t);

}  // namespace e3d
