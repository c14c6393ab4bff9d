// Host-callable kernel launchers.  k64.cu (built with -fmad=false, so double
// arithmetic keeps the reference's rounding) defines the FP64 granular kernels
// and the double instantiations; k32.cu defines the float instantiations.
#pragma once
#include <cuda_runtime.h>

#include "views.hpp"

namespace e3d {

// ---- granular FP64 drop-in kernels (one per reference strategy method) ----
void launch_save_w0(const GeoView&, const StateView&, const Physics&, int r0, int r1, cudaStream_t);
void launch_spectral_radius(const GeoView&, const StateView&, const Physics&, int r0, int r1, cudaStream_t);
void launch_timestep(const GeoView&, const StateView&, const Physics&, int r0, int r1, cudaStream_t);
void launch_gradients(const GeoView&, const StateView&, int kind, int r0, int r1, cudaStream_t);
void launch_limiters(const GeoView&, const StateView&, const Physics&, int kind, int r0, int r1, int g0, int g1,
                     cudaStream_t);
void launch_flux_conv(const GeoView&, const StateView&, const Physics&, int scheme, int r0, int r1, cudaStream_t);
void launch_flux_diss(const GeoView&, const StateView&, const Physics&, int scheme, double beta, int r0, int r1,
                      cudaStream_t);
void launch_update(const GeoView&, const StateView&, const Physics&, double alpha, int r0, int r1, cudaStream_t);
void launch_bc(const GeoView&, const StateView&, const Physics&, int g0, int g1, cudaStream_t);
// central implicit residual smoothing of Rc and Rd (j1: 10 x NR FP64 scratch)
void launch_smooth(const GeoView&, const StateView&, double* j1, int r0, int r1, cudaStream_t);

// ---- shared by both paths, per precision ----
template <class T>
void launch_halo(int n, const int* dst, const int* src, int NA, T* b0, T* b1, cudaStream_t);
// halo entries of a block-sharded case: gather into / scatter from an
// entry-major buffer of 5 values per entry (k_halo_pack, k_halo_unpack)
template <class T>
void launch_halo_pack(int n, const int* src, int NA, const T* P, T* buf, cudaStream_t);
template <class T>
void launch_halo_unpack(int n, const int* dst, int NA, const T* buf, T* b0, T* b1, cudaStream_t);

// Per-block reductions written into hist[iter*stride + b*10 + (0..4 norms, 5..9 forces)],
// iter read from *d_iter (the device iteration counter).
struct ReduceArgs {
	int NR, NA, nblocks;
	const int* roff;       // nblocks+1 real-cell offsets
	int chunk, max_chunks;
	double* partial;       // nblocks*max_chunks*5
	const int* wall_off;   // nblocks+1
	const int* wall_face;
	int n_wall;
	double* wall_terms;    // 5*n_wall
	const int* face_lr;
	const double* S;
	const double* fc;
	double denom;          // 0.5*gamma*M*M*cmac
	const double* wall_denom;  // per wall face (cases of a batch differ in Mach), or null
	double* hist;
	int stride;
	const int* d_iter;
	int* d_bad;
};
template <class T>
void launch_reduce(const ReduceArgs&, const T* Rc, const T* Rd, const T* P, cudaStream_t);
void launch_iter_advance(int* d_iter, cudaStream_t);

// ---- fused stage kernels ----
template <class T>
void launch_recon(const FusedView<T>&, const Physics&, int grad, int lim, bool first, int carry, cudaStream_t);
template <class T>
void launch_start(const FusedView<T>&, const Physics&, int carry, cudaStream_t);

// batch launchers: threads per block; per namespace: resident blocks per SM of
// the persistent kernel, its cooperative launch, and the tiled per-pass form.
// `batch` is built with the working precision's flags (FP64: no contraction,
// the same arithmetic as the single-case path); `batch_fast` holds FP64
// kernels built with FMA contraction (k64f.cu).
constexpr int kPersistThreads = 128;
namespace batch {
template <class T>
int persistent_blocks_per_sm(int grad, int lim, int scheme, bool order2);
template <class T>
cudaError_t launch_persistent(const FusedView<T>& v0, const FusedView<T>& v1, const Physics& ph, const PersistArgs& a,
                              int grad, int lim, int scheme, bool order2, int grid, cudaStream_t st);
// the same iterations as separate per-pass launches over the work list
template <class T>
cudaError_t launch_tiled_iterations(const FusedView<T>& v0, const FusedView<T>& v1, const Physics& ph,
                                    const PersistArgs& a, int grad, int lim, int scheme, bool order2, cudaStream_t st);
}  // namespace batch
namespace batch_fast {
template <class T>
int persistent_blocks_per_sm(int grad, int lim, int scheme, bool order2);
template <class T>
cudaError_t launch_persistent(const FusedView<T>& v0, const FusedView<T>& v1, const Physics& ph, const PersistArgs& a,
                              int grad, int lim, int scheme, bool order2, int grid, cudaStream_t st);
// the same iterations as separate per-pass launches over the work list
template <class T>
cudaError_t launch_tiled_iterations(const FusedView<T>& v0, const FusedView<T>& v1, const Physics& ph,
                                    const PersistArgs& a, int grad, int lim, int scheme, bool order2, cudaStream_t st);
}  // namespace batch_fast

// FP32 iterations in difference form (delta.cu): first-order AUSM, all-tetrahedron
// meshes, tiled per-pass form.  v0/v1 carry the base and difference arrays.
namespace delta {
cudaError_t launch_iterations(const FusedView<float>& v0, const FusedView<float>& v1, const Physics& ph,
                              const PersistArgs& a, cudaStream_t st);
// new base state from W_b + dW (Wb: the FP64 base conserved state, updated in
// place), base ghosts, base residual in FP64; differences d0, d1 cleared
void launch_rebase(const FusedView<float>& v, const Physics& ph, double* Wb, const double* area64, int n_halo,
                   const int* halo_dst, const int* halo_src, float* d0, float* d1, cudaStream_t st);
}  // namespace delta

template <class T>
void launch_flux_update(const FusedView<T>&, const Physics&, int scheme, bool order1, double alpha, double beta,
                        int last, int carry, cudaStream_t);

}  // namespace e3d
