// Residual norms without device allocation.
//
// Some callers cannot allocate device memory at the point where they need the
// convergence norms: a host application that owns every device byte through its
// own pool and forbids cudaMalloc inside plugins, or a caller that must not
// trigger an allocation (and the implicit synchronisation that cudaMalloc /
// cudaFree can bring) in the middle of its time-stepping loop.  For them this
// file provides the per-block sums of (Rc - Rd)^2 with the reduction's
// scratch in a fixed-size static device array instead of memory from cudaMalloc.
//
// The scratch holds E3D_NOALLOC_MAX_PARTIALS partial sums per equation
// (8192 x 5 doubles = 320 KiB).  Every GPU that loads libe3d.so keeps this
// array until the process exits.  Its device address is looked up once per
// device, on that device's first call, with cudaGetSymbolAddress; make that
// first call before any stream capture.  All calls share the one array and it
// keeps the last call's contents, so calls that overlap on the GPU (different
// streams, or several host threads) race and must be ordered by the caller.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/e3d.h"
#include "mesh.hpp"

namespace e3d {
void set_last_error(const std::string& msg);  // capi.cpp
}

namespace {

constexpr int kThreads = 256;
constexpr int kChunk = 4096;  // cells per partial sum
constexpr int kMaxDevices = 64;

__device__ __align__(256) double g_norm_scratch[E3D_NOALLOC_MAX_PARTIALS * 5];

// partial[(b*max_chunks + chunk)*5 + q] = sum over the chunk's cells of (rc-rd)^2;
// every slot of the grid is written, so nothing needs clearing between calls.
// The grid covers max_chunks * kChunk cells per block.  A block whose offsets
// span more cells than that (max_block_cells understated by the caller) would
// lose its tail silently; instead its last chunk writes NaN, so all five of
// that block's outputs come back NaN.
__global__ void __launch_bounds__(kThreads) k_partial_static(const double* __restrict__ rc, const double* __restrict__ rd,
                                                             long long n, const int* __restrict__ off, int max_chunks,
                                                             double* __restrict__ partial) {
	const int b = blockIdx.y;
	// offsets are clamped to [0, n]: a bad offset array cannot index outside rc/rd
	const long long o0 = max(0LL, min((long long)off[b], n)), o1 = max(o0, min((long long)off[b + 1], n));
	const long long beg = o0 + (long long)blockIdx.x * kChunk;
	const long long end = min(o1, beg + kChunk);
	const bool uncovered = blockIdx.x == max_chunks - 1 && o1 - o0 > (long long)max_chunks * kChunk;
	double acc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
	for (long long c = beg + threadIdx.x; c < end; c += kThreads)
		for (int q = 0; q < 5; q++) {
			const double r = rc[q * n + c] - rd[q * n + c];
			acc[q] += r * r;
		}
	__shared__ double sm[5][kThreads];
	for (int q = 0; q < 5; q++) sm[q][threadIdx.x] = acc[q];
	__syncthreads();
	for (int w = kThreads / 2; w > 0; w >>= 1) {
		if (threadIdx.x < w)
			for (int q = 0; q < 5; q++) sm[q][threadIdx.x] += sm[q][threadIdx.x + w];
		__syncthreads();
	}
	if (threadIdx.x < 5)
		partial[((size_t)b * max_chunks + blockIdx.x) * 5 + threadIdx.x] = uncovered ? __longlong_as_double(0x7ff8000000000000LL)
		                                                                             : sm[threadIdx.x][0];
}

__global__ void k_final_static(const double* __restrict__ partial, int n_blocks, int max_chunks, double* __restrict__ out) {
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= n_blocks * 5) return;
	const int b = t / 5, q = t % 5;
	double s = 0.0;
	for (int i = 0; i < max_chunks; i++) s += partial[((size_t)b * max_chunks + i) * 5 + q];
	out[t] = s;
}

std::mutex g_mu;
double* g_scratch_ptr[kMaxDevices] = {};

// Device address of the scratch array on the current device (looked up once).
int scratch_for_current_device(double** out) {
	int dev = -1;
	cudaError_t e = cudaGetDevice(&dev);
	if (e != cudaSuccess) {
		e3d::set_last_error(std::string("cudaGetDevice: ") + cudaGetErrorString(e));
		return E3D_ERR_CUDA;
	}
	if (dev < 0 || dev >= kMaxDevices) {
		e3d::set_last_error("device index above the supported maximum");
		return E3D_ERR_LIMIT;
	}
	std::lock_guard<std::mutex> lk(g_mu);
	if (!g_scratch_ptr[dev]) {
		void* p = nullptr;
		e = cudaGetSymbolAddress(&p, g_norm_scratch);
		if (e != cudaSuccess || !p) {
			e3d::set_last_error(std::string("cudaGetSymbolAddress(norm scratch): ") + cudaGetErrorString(e));
			return E3D_ERR_CUDA;
		}
		g_scratch_ptr[dev] = static_cast<double*>(p);
	}
	*out = g_scratch_ptr[dev];
	return E3D_OK;
}

}  // namespace

extern "C" int e3d_residual_norms_noalloc(const double* rc, const double* rd, int64_t n_cells, int n_blocks,
                                          const int32_t* block_offsets, int max_block_cells, double* out,
                                          void* stream) {
	if (!rc || !rd || !block_offsets || !out || n_cells < 0 || n_blocks <= 0 || max_block_cells < 0) {
		e3d::set_last_error("e3d_residual_norms_noalloc: null pointer or negative size");
		return E3D_ERR_ARG;
	}
	// chunk count in 64 bits: a max_block_cells near INT_MAX must not wrap
	const long long chunks64 = max_block_cells > 0 ? ((long long)max_block_cells + kChunk - 1) / kChunk : 1;
	if ((long long)n_blocks * chunks64 > E3D_NOALLOC_MAX_PARTIALS) {
		e3d::set_last_error("e3d_residual_norms_noalloc: " + std::to_string(n_blocks) + " blocks x " +
		                    std::to_string(chunks64) + " chunks of " + std::to_string(kChunk) +
		                    " cells exceed the static scratch of " + std::to_string(E3D_NOALLOC_MAX_PARTIALS) +
		                    " partial sums");
		return E3D_ERR_LIMIT;
	}
	const int max_chunks = static_cast<int>(chunks64);  // <= E3D_NOALLOC_MAX_PARTIALS here
	double* scratch = nullptr;
	const int rcode = scratch_for_current_device(&scratch);
	if (rcode != E3D_OK) return rcode;
	cudaStream_t st = static_cast<cudaStream_t>(stream);
	k_partial_static<<<dim3(max_chunks, n_blocks), kThreads, 0, st>>>(rc, rd, n_cells, block_offsets, max_chunks, scratch);
	k_final_static<<<(n_blocks * 5 + 127) / 128, 128, 0, st>>>(scratch, n_blocks, max_chunks, out);
	const cudaError_t e = cudaGetLastError();
	if (e != cudaSuccess) {
		e3d::set_last_error(std::string("e3d_residual_norms_noalloc: ") + cudaGetErrorString(e));
		return E3D_ERR_CUDA;
	}
	return E3D_OK;
}
