// Warm-start surrogate: training and inference kernels (see surrogate.hpp).
//
// The 128-wide layers run as one templated tensor-core GEMM, C = A * B^T
// with BF16 operands staged in shared memory and FP32 accumulators
// (mma.sync m16n8k16), and a per-use epilogue: bias + GELU (forward), times
// GELU'(z) (backward data), or an FP32 partial of a split-K slice (weight
// gradients, summed over slices in a fixed order).  The 5-wide output layer
// runs on the CUDA cores.  No floating-point atomics anywhere: every sum is
// a fixed-order loop or tree, so a training run is reproducible bit for bit.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>

#include "surrogate.hpp"
#include "warm.hpp"

namespace e3d {
namespace {

using S = SurrogateShape;
constexpr int H = S::H;

// ------------------------------------------------------------------ helpers
__device__ __forceinline__ uint16_t f2bf(float x) {
	const __nv_bfloat16 b = __float2bfloat16_rn(x);
	return *reinterpret_cast<const uint16_t*>(&b);
}
__device__ __forceinline__ float bf2f(uint16_t u) { return __uint_as_float(((uint32_t)u) << 16); }

__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.f + erff(z * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_d(float z) {
	return 0.5f * (1.f + erff(z * 0.70710678118654752f)) + z * 0.39894228040143268f * expf(-0.5f * z * z);
}

__host__ __device__ __forceinline__ uint64_t mix64(uint64_t x) {
	// splitmix64 finaliser
	x += 0x9E3779B97F4A7C15ull;
	x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
	x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
	return x ^ (x >> 31);
}

// freestream conservative state of (Mach, alpha in degrees), the reference's
// nondimensionalisation (rho = 1, p = 1, |u| = M sqrt(gamma))
__device__ __forceinline__ void wfree(float mach, float aoa_deg, float gamma, float w[5]) {
	const float a = aoa_deg * 0.017453292519943295f;
	const float q = mach * sqrtf(gamma);
	const float u = q * cosf(a), v = q * sinf(a);
	w[0] = 1.f;
	w[1] = u;
	w[2] = v;
	w[3] = 0.f;
	w[4] = 0.5f * (u * u + v * v) + 1.f / (gamma - 1.f);
}

// ------------------------------------------------------------------ GEMM
enum { L_ROW = 0, L_COL = 1 };
enum { EPI_FWD_GELU = 0, EPI_BWD_GELU = 1, EPI_PARTIAL = 2 };

struct Epi {
	const float* bias;  // EPI_FWD_GELU
	float* zout;        // EPI_FWD_GELU: pre-activation [M][ldo]
	uint16_t* hout;     // EPI_FWD_GELU: GELU(z) BF16; EPI_BWD_GELU: g BF16 [M][ldo]
	const float* zin;   // EPI_BWD_GELU: pre-activation of the layer below [M][ldo]
	float* part;        // EPI_PARTIAL: [slices][M][N]
	int ldo;
};

constexpr int BM = 64, BN = 64, BK = 32, SPAD = 8;

__device__ __forceinline__ uint32_t ld32(const uint16_t* p) { return *reinterpret_cast<const uint32_t*>(p); }

__device__ __forceinline__ void mma_bf16(float c[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3, uint32_t b0,
                                         uint32_t b1) {
	asm volatile(
	    "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
	    "{%0,%1,%2,%3};\n"
	    : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
	    : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// C[m][n] = sum_k A(m,k) B(n,k);  A(m,k) = A[m*lda+k] (L_ROW) or A[k*lda+m] (L_COL),
// B(n,k) = B[n*ldb+k] (L_ROW) or B[k*ldb+n] (L_COL).  blockIdx.z = split-K slice.
template <int AL, int BL, int EPI>
__global__ void __launch_bounds__(128) k_gemm(int M, int N, int K, const uint16_t* __restrict__ A, int lda,
                                              const uint16_t* __restrict__ B, int ldb, int k_slice, Epi ep) {
	__shared__ __align__(16) uint16_t As[BM][BK + SPAD];
	__shared__ __align__(16) uint16_t Bs[BN][BK + SPAD];
	const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
	const int g = lane >> 2, t = lane & 3;
	const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
	const int kb = blockIdx.z * k_slice, ke = min(K, kb + k_slice);
	const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
	float acc[2][4][4];
#pragma unroll
	for (int i = 0; i < 2; i++)
#pragma unroll
		for (int j = 0; j < 4; j++)
#pragma unroll
			for (int r = 0; r < 4; r++) acc[i][j][r] = 0.f;

	for (int k0 = kb; k0 < ke; k0 += BK) {
#pragma unroll 4
		for (int e = 0; e < (BM * BK) / 128; e++) {
			const int idx = e * 128 + tid;
			int m, k;
			if (AL == L_ROW) {
				m = idx / BK;
				k = idx % BK;
			} else {
				m = idx % BM;
				k = idx / BM;
			}
			const int gm = m0 + m, gk = k0 + k;
			uint16_t v = 0;
			if (gm < M && gk < ke) v = AL == L_ROW ? A[(size_t)gm * lda + gk] : A[(size_t)gk * lda + gm];
			As[m][k] = v;
		}
#pragma unroll 4
		for (int e = 0; e < (BN * BK) / 128; e++) {
			const int idx = e * 128 + tid;
			int n, k;
			if (BL == L_ROW) {
				n = idx / BK;
				k = idx % BK;
			} else {
				n = idx % BN;
				k = idx / BN;
			}
			const int gn = n0 + n, gk = k0 + k;
			uint16_t v = 0;
			if (gn < N && gk < ke) v = BL == L_ROW ? B[(size_t)gn * ldb + gk] : B[(size_t)gk * ldb + gn];
			Bs[n][k] = v;
		}
		__syncthreads();
#pragma unroll
		for (int ks = 0; ks < BK; ks += 16) {
			uint32_t a[2][4], b[4][2];
#pragma unroll
			for (int i = 0; i < 2; i++) {
				const int r = wm + 16 * i + g;
				a[i][0] = ld32(&As[r][ks + 2 * t]);
				a[i][1] = ld32(&As[r + 8][ks + 2 * t]);
				a[i][2] = ld32(&As[r][ks + 2 * t + 8]);
				a[i][3] = ld32(&As[r + 8][ks + 2 * t + 8]);
			}
#pragma unroll
			for (int j = 0; j < 4; j++) {
				const int c = wn + 8 * j + g;
				b[j][0] = ld32(&Bs[c][ks + 2 * t]);
				b[j][1] = ld32(&Bs[c][ks + 2 * t + 8]);
			}
#pragma unroll
			for (int i = 0; i < 2; i++)
#pragma unroll
				for (int j = 0; j < 4; j++) mma_bf16(acc[i][j], a[i][0], a[i][1], a[i][2], a[i][3], b[j][0], b[j][1]);
		}
		__syncthreads();
	}
	// epilogue: acc[i][j] = rows (g, g+8) x cols (2t, 2t+1) of the 16x8 tile
#pragma unroll
	for (int i = 0; i < 2; i++)
#pragma unroll
		for (int j = 0; j < 4; j++)
#pragma unroll
			for (int r = 0; r < 4; r++) {
				const int m = m0 + wm + 16 * i + g + (r >= 2 ? 8 : 0);
				const int n = n0 + wn + 8 * j + 2 * t + (r & 1);
				if (m >= M || n >= N) continue;
				const float v = acc[i][j][r];
				if (EPI == EPI_FWD_GELU) {
					const float z = v + ep.bias[n];
					ep.zout[(size_t)m * ep.ldo + n] = z;
					ep.hout[(size_t)m * ep.ldo + n] = f2bf(gelu(z));
				} else if (EPI == EPI_BWD_GELU) {
					ep.hout[(size_t)m * ep.ldo + n] = f2bf(v * gelu_d(ep.zin[(size_t)m * ep.ldo + n]));
				} else {
					ep.part[((size_t)blockIdx.z * M + m) * N + n] = v;
				}
			}
}

template <int AL, int BL, int EPI>
void gemm(int M, int N, int K, const uint16_t* A, int lda, const uint16_t* B, int ldb, int slices, const Epi& ep,
          cudaStream_t st) {
	const int ks = ((K + slices - 1) / slices + BK - 1) / BK * BK;
	const int sl = (K + ks - 1) / ks;
	dim3 grid((N + BN - 1) / BN, (M + BM - 1) / BM, sl);
	k_gemm<AL, BL, EPI><<<grid, 128, 0, st>>>(M, N, K, A, lda, B, ldb, ks, ep);
}

// ------------------------------------------------------------------ small kernels
// minibatch rows: standardised features (BF16, [n][IN]) and scaled targets ([n][OUT])
__global__ void k_prepare(int n, const float* __restrict__ feat, int ldf, const float* __restrict__ state, int lds,
                          long long n_store, uint64_t seed, long long step, const float* __restrict__ norm, float gamma,
                          uint16_t* __restrict__ x, float* __restrict__ tgt) {
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	long long src = i;
	if (n_store > 0) src = (long long)(mix64(seed ^ mix64((uint64_t)step * 0x100000001B3ull + (uint64_t)i)) %
	                                   (uint64_t)n_store);
	const float* f = feat + (size_t)src * ldf;
	for (int j = 0; j < S::IN; j++)
		x[(size_t)i * S::IN + j] = j < S::N_IN ? f2bf((f[j] - norm[j]) / norm[8 + j]) : (uint16_t)0;
	if (tgt) {
		float wf[5];
		wfree(f[4], f[5], gamma, wf);
		const float* s = state + (size_t)src * lds;
		for (int q = 0; q < S::OUT; q++) tgt[(size_t)i * S::OUT + q] = q < S::N_OUT ? (s[q] - wf[q]) / norm[16 + q] : 0.f;
	}
}

// output layer on the CUDA cores: y[b][q] = b4[q] + sum_j W4[q][j] a3[b][j]
__global__ void k_out_layer(int n, const uint16_t* __restrict__ a3, const uint16_t* __restrict__ w4,
                            const float* __restrict__ b4, float* __restrict__ y) {
	__shared__ float w[S::N_OUT][H];
	for (int i = threadIdx.x; i < S::N_OUT * H; i += blockDim.x) w[i / H][i % H] = bf2f(w4[i]);
	__syncthreads();
	const int b = blockIdx.x * blockDim.x + threadIdx.x;
	if (b >= n) return;
	float acc[S::N_OUT];
	for (int q = 0; q < S::N_OUT; q++) acc[q] = 0.f;
	const uint16_t* a = a3 + (size_t)b * H;
	for (int j = 0; j < H; j += 2) {
		const uint32_t p = *reinterpret_cast<const uint32_t*>(a + j);
		const float x0 = bf2f((uint16_t)(p & 0xFFFFu)), x1 = bf2f((uint16_t)(p >> 16));
		for (int q = 0; q < S::N_OUT; q++) acc[q] += w[q][j] * x0 + w[q][j + 1] * x1;
	}
	for (int q = 0; q < S::OUT; q++) y[(size_t)b * S::OUT + q] = q < S::N_OUT ? acc[q] + b4[q] : 0.f;
}

// d4 = dL/dy for L = mean over rows and the 5 outputs of (y - t)^2; per-block squared-error sums
__global__ void k_loss(int n, const float* __restrict__ y, const float* __restrict__ t, float* __restrict__ d4,
                       float* __restrict__ lossp) {
	__shared__ float red[256];
	const int b = blockIdx.x * blockDim.x + threadIdx.x;
	float se = 0.f;
	if (b < n)
		for (int q = 0; q < S::OUT; q++) {
			const float e = q < S::N_OUT ? y[(size_t)b * S::OUT + q] - t[(size_t)b * S::OUT + q] : 0.f;
			d4[(size_t)b * S::OUT + q] = 2.f * e / (float)(n * S::N_OUT);
			se += e * e;
		}
	red[threadIdx.x] = se;
	__syncthreads();
	for (int h = blockDim.x / 2; h > 0; h >>= 1) {
		if (threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
		__syncthreads();
	}
	if (threadIdx.x == 0) lossp[blockIdx.x] = red[0];
}

__global__ void k_loss_final(int nparts, const float* __restrict__ lossp, int n, double* __restrict__ out) {
	if (threadIdx.x != 0 || blockIdx.x != 0) return;
	double s = 0.0;
	for (int i = 0; i < nparts; i++) s += (double)lossp[i];
	*out = s / ((double)n * S::N_OUT);
}

// g3[b][j] = gelu'(z3[b][j]) * sum_q d4[b][q] W4[q][j]  (BF16 out)
__global__ void k_out_back(int n, const float* __restrict__ d4, const uint16_t* __restrict__ w4,
                           const float* __restrict__ z3, uint16_t* __restrict__ g3) {
	const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= (long long)n * H) return;
	const int b = (int)(i / H), j = (int)(i % H);
	float s = 0.f;
	for (int q = 0; q < S::N_OUT; q++) s += d4[(size_t)b * S::OUT + q] * bf2f(w4[q * H + j]);
	g3[i] = f2bf(s * gelu_d(z3[i]));
}

// per-slice partial sums over rows: dW4[q][j] = sum_b d4[b][q] a3[b][j] and db4[q] = sum_b d4[b][q]
// part layout [slice][OUT*H + OUT]
__global__ void k_out_wgrad(int n, int rows, const float* __restrict__ d4, const uint16_t* __restrict__ a3,
                            float* __restrict__ part) {
	const int j = threadIdx.x;  // H threads
	const int r0 = blockIdx.x * rows, r1 = min(n, r0 + rows);
	float acc[S::N_OUT], bacc[S::N_OUT];
	for (int q = 0; q < S::N_OUT; q++) acc[q] = bacc[q] = 0.f;
	for (int b = r0; b < r1; b++) {
		const float a = bf2f(a3[(size_t)b * H + j]);
		for (int q = 0; q < S::N_OUT; q++) {
			const float d = d4[(size_t)b * S::OUT + q];
			acc[q] += d * a;
			bacc[q] += d;
		}
	}
	float* p = part + (size_t)blockIdx.x * (S::OUT * H + S::OUT);
	for (int q = 0; q < S::OUT; q++) p[q * H + j] = q < S::N_OUT ? acc[q] : 0.f;
	if (j < S::OUT) p[S::OUT * H + j] = j < S::N_OUT ? bacc[j] : 0.f;
}

// per-slice column sums of a BF16 [n][H] matrix (bias gradients); part [slice][H]
__global__ void k_colsum(int n, int rows, const uint16_t* __restrict__ g, float* __restrict__ part) {
	const int j = threadIdx.x;
	const int r0 = blockIdx.x * rows, r1 = min(n, r0 + rows);
	float s = 0.f;
	for (int b = r0; b < r1; b++) s += bf2f(g[(size_t)b * H + j]);
	part[(size_t)blockIdx.x * H + j] = s;
}

// out[i] = sum over slices s (in order) of part[s*len + i]
__global__ void k_reduce_slices(int slices, int len, const float* __restrict__ part, float* __restrict__ out) {
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= len) return;
	float s = 0.f;
	for (int k = 0; k < slices; k++) s += part[(size_t)k * len + i];
	out[i] = s;
}

__global__ void k_adam(int n, float* __restrict__ w, float* __restrict__ m, float* __restrict__ v,
                       const float* __restrict__ g, uint16_t* __restrict__ wb, float lr, float b1, float b2, float eps,
                       float c1, float c2) {
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	const float gi = g[i];
	const float mi = b1 * m[i] + (1.f - b1) * gi;
	const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
	m[i] = mi;
	v[i] = vi;
	const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
	w[i] = wi;
	wb[i] = f2bf(wi);
}

__global__ void k_to_bf16(int n, const float* __restrict__ w, uint16_t* __restrict__ wb) {
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n) wb[i] = f2bf(w[i]);
}

// conservative state from the network output
__global__ void k_denormalise(int n, const float* __restrict__ y, const float* __restrict__ feat, int ldf,
                              const float* __restrict__ norm, float gamma, float* __restrict__ out, int ldo) {
	const int b = blockIdx.x * blockDim.x + threadIdx.x;
	if (b >= n) return;
	const float* f = feat + (size_t)b * ldf;
	float wf[5];
	wfree(f[4], f[5], gamma, wf);
	for (int q = 0; q < S::N_OUT; q++) out[(size_t)b * ldo + q] = wf[q] + norm[16 + q] * y[(size_t)b * S::OUT + q];
	for (int q = S::N_OUT; q < ldo; q++) out[(size_t)b * ldo + q] = 0.f;
}

// feature statistics: per-block partial sums of x and x^2 (double), fixed order
__global__ void k_feat_stats(long long n, const float* __restrict__ feat, const float* __restrict__ state, float gamma,
                             long long rows, double* __restrict__ part) {
	const int j = threadIdx.x;  // 16 threads: 0..5 features, 8..12 target deviations
	const long long r0 = (long long)blockIdx.x * rows, r1 = min(n, r0 + rows);
	double s = 0.0, s2 = 0.0;
	for (long long b = r0; b < r1; b++) {
		double x;
		if (j < 8) {
			x = j < S::N_IN ? (double)feat[b * 8 + j] : 0.0;
		} else {
			float wf[5];
			wfree(feat[b * 8 + 4], feat[b * 8 + 5], gamma, wf);
			const int q = j - 8;
			x = q < S::N_OUT ? (double)state[b * 8 + q] - (double)wf[q] : 0.0;
		}
		s += x;
		s2 += x * x;
	}
	part[(size_t)blockIdx.x * 32 + j] = s;
	part[(size_t)blockIdx.x * 32 + 16 + j] = s2;
}

inline void ok(cudaError_t e, const char* what) {
	if (e != cudaSuccess) throw Error(E3D_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}
inline int blocks(long long n, int t) { return (int)((n + t - 1) / t); }

}  // namespace

// ------------------------------------------------------------------ Surrogate
Surrogate::Surrogate(int device, uint64_t seed, double gamma) : device_(device), gamma_(gamma), seed_(seed) {
	if (device_ >= 0) ok(cudaSetDevice(device_), "cudaSetDevice");
	ok(cudaStreamCreateWithFlags(&st_, cudaStreamNonBlocking), "cudaStreamCreate");
	// Kaiming-uniform initialisation from a seeded generator (host), padding entries zero
	std::vector<float> w(S::N_PARAM, 0.f);
	std::mt19937_64 rng(seed);
	auto fill = [&](int off, int rows, int cols, int used_rows, int used_cols) {
		const float bound = std::sqrt(6.f / (float)used_cols);
		std::uniform_real_distribution<float> u(-bound, bound);
		for (int r = 0; r < rows; r++)
			for (int c = 0; c < cols; c++) w[off + r * cols + c] = (r < used_rows && c < used_cols) ? u(rng) : 0.f;
	};
	fill(S::OFF_W1, H, S::IN, H, S::N_IN);
	fill(S::OFF_W2, H, H, H, H);
	fill(S::OFF_W3, H, H, H, H);
	fill(S::OFF_W4, S::OUT, H, S::N_OUT, H);
	for (int i = 0; i < S::OUT * H; i++) w[S::OFF_W4 + i] *= 0.1f;  // small initial output: start near freestream
	master_.upload(w);
	std::vector<float> z(S::N_PARAM, 0.f);
	m1_.upload(z);
	m2_.upload(z);
	grad_.upload(z);
	wb_.alloc(S::N_PARAM);
	norm_h_.assign(S::N_NORM, 0.f);
	for (int j = 0; j < 8; j++) norm_h_[8 + j] = 1.f;
	for (int q = 0; q < 8; q++) norm_h_[16 + q] = 1.f;
	norm_.upload(norm_h_);
	loss_d_.alloc(1);
	upload_params();
}

Surrogate::~Surrogate() {
	if (st_) cudaStreamDestroy(st_);
}

void Surrogate::upload_params() {
	k_to_bf16<<<blocks(S::N_PARAM, 256), 256, 0, st_>>>(S::N_PARAM, master_.p, wb_.p);
	ok(cudaGetLastError(), "to_bf16");
}

void Surrogate::add_samples_device(const float* feat, const float* state, long long n, cudaStream_t producer) {
	if (n <= 0) return;
	if (producer) ok(cudaStreamSynchronize(producer), "sync");
	if (n_samples_ + n > cap_samples_) {
		const long long cap = std::max(n_samples_ + n, cap_samples_ * 3 / 2 + 1024);
		DevBuf<float> f2, s2;
		f2.alloc((size_t)cap * 8);
		s2.alloc((size_t)cap * 8);
		if (n_samples_) {
			ok(cudaMemcpyAsync(f2.p, feat_.p, (size_t)n_samples_ * 8 * sizeof(float), cudaMemcpyDeviceToDevice, st_),
			   "grow");
			ok(cudaMemcpyAsync(s2.p, state_.p, (size_t)n_samples_ * 8 * sizeof(float), cudaMemcpyDeviceToDevice, st_),
			   "grow");
		}
		ok(cudaStreamSynchronize(st_), "sync");
		std::swap(feat_.p, f2.p);
		std::swap(feat_.n, f2.n);
		std::swap(state_.p, s2.p);
		std::swap(state_.n, s2.n);
		cap_samples_ = cap;
	}
	ok(cudaMemcpyAsync(feat_.p + (size_t)n_samples_ * 8, feat, (size_t)n * 8 * sizeof(float), cudaMemcpyDeviceToDevice,
	                   st_),
	   "samples");
	ok(cudaMemcpyAsync(state_.p + (size_t)n_samples_ * 8, state, (size_t)n * 8 * sizeof(float),
	                   cudaMemcpyDeviceToDevice, st_),
	   "samples");
	ok(cudaStreamSynchronize(st_), "sync");
	n_samples_ += n;
}

void Surrogate::add_samples_host(const float* feat6, const float* state5, long long n) {
	if (n <= 0) return;
	std::vector<float> f((size_t)n * 8, 0.f), s((size_t)n * 8, 0.f);
	for (long long i = 0; i < n; i++) {
		for (int j = 0; j < 6; j++) f[i * 8 + j] = feat6[i * 6 + j];
		for (int q = 0; q < 5; q++) s[i * 8 + q] = state5[i * 5 + q];
	}
	DevBuf<float> fd, sd;
	fd.upload(f);
	sd.upload(s);
	add_samples_device(fd.p, sd.p, n, nullptr);
}

void Surrogate::add_solution(Engine& e) {
	const int nr = e.n_real_total();
	DevBuf<float> f, s;
	f.alloc((size_t)nr * 8);
	s.alloc((size_t)nr * 8);
	e.cell_features(f.p);
	e.conservative_rows(s.p);
	add_samples_device(f.p, s.p, nr, e.stream());
}

void Surrogate::clear_samples() {
	n_samples_ = 0;
	normalised_ = false;
}

void Surrogate::fit_normalisation() {
	if (n_samples_ < 2) throw Error(E3D_ERR_STATE, "surrogate: no training samples");
	const long long rows = 65536;
	const int nb = (int)((n_samples_ + rows - 1) / rows);
	DevBuf<double> part;
	part.alloc((size_t)nb * 32);
	k_feat_stats<<<nb, 16, 0, st_>>>(n_samples_, feat_.p, state_.p, (float)gamma_, rows, part.p);
	ok(cudaGetLastError(), "feat_stats");
	std::vector<double> h((size_t)nb * 32);
	ok(cudaMemcpyAsync(h.data(), part.p, h.size() * sizeof(double), cudaMemcpyDeviceToHost, st_), "stats");
	ok(cudaStreamSynchronize(st_), "sync");
	double s[16] = {0}, s2[16] = {0};
	for (int b = 0; b < nb; b++)
		for (int j = 0; j < 16; j++) {
			s[j] += h[(size_t)b * 32 + j];
			s2[j] += h[(size_t)b * 32 + 16 + j];
		}
	const double n = (double)n_samples_;
	for (int j = 0; j < 8; j++) {
		const double mu = s[j] / n, var = std::max(0.0, s2[j] / n - mu * mu);
		norm_h_[j] = (float)mu;
		norm_h_[8 + j] = (float)std::max(std::sqrt(var), 1e-6);
		const double t2 = s2[8 + j] / n;  // target scale: RMS deviation from freestream
		norm_h_[16 + j] = (float)std::max(std::sqrt(t2), 1e-6);
	}
	norm_.upload(norm_h_);
	normalised_ = true;
}

void Surrogate::ensure_work(int n) {
	if (n <= work_n_) return;
	work_n_ = n;
	x_.alloc((size_t)n * S::IN);
	for (auto* b : {&a1_, &a2_, &a3_, &g1_, &g2_, &g3_}) b->alloc((size_t)n * H);
	for (auto* b : {&z1_, &z2_, &z3_}) b->alloc((size_t)n * H);
	y_.alloc((size_t)n * S::OUT);
	t_.alloc((size_t)n * S::OUT);
	lossp_.alloc((size_t)blocks(n, 256));
	// split-K partials: up to 64 slices of the largest weight block (+ output layer)
	part_.alloc((size_t)64 * (H * H + S::OUT * H + S::OUT));
}

// forward of n prepared rows (x_ filled): z1..z3, a1..a3, y
void Surrogate::forward(int n) {
	Epi e{};
	e.ldo = H;
	e.bias = master_.p + S::OFF_B1;
	e.zout = z1_.p;
	e.hout = a1_.p;
	gemm<L_ROW, L_ROW, EPI_FWD_GELU>(n, H, S::IN, x_.p, S::IN, wb_.p + S::OFF_W1, S::IN, 1, e, st_);
	e.bias = master_.p + S::OFF_B2;
	e.zout = z2_.p;
	e.hout = a2_.p;
	gemm<L_ROW, L_ROW, EPI_FWD_GELU>(n, H, H, a1_.p, H, wb_.p + S::OFF_W2, H, 1, e, st_);
	e.bias = master_.p + S::OFF_B3;
	e.zout = z3_.p;
	e.hout = a3_.p;
	gemm<L_ROW, L_ROW, EPI_FWD_GELU>(n, H, H, a2_.p, H, wb_.p + S::OFF_W3, H, 1, e, st_);
	k_out_layer<<<blocks(n, 128), 128, 0, st_>>>(n, a3_.p, wb_.p + S::OFF_W4, master_.p + S::OFF_B4, y_.p);
	ok(cudaGetLastError(), "forward");
}

// backward of the rows of the last forward against the targets in t_: loss and grad_ (all parameters)
void Surrogate::backward(int n, double* loss_out) {
	float* d4 = reinterpret_cast<float*>(g1_.p);  // reuse: d4 [n][OUT] floats fit in g1 ([n][H] BF16)
	const int lb = blocks(n, 256);
	k_loss<<<lb, 256, 0, st_>>>(n, y_.p, t_.p, d4, lossp_.p);
	k_loss_final<<<1, 1, 0, st_>>>(lb, lossp_.p, n, loss_d_.p);
	// output layer gradients
	const int rows = std::max(64, (n + 63) / 64);
	const int sl = (n + rows - 1) / rows;
	const int lo = S::OUT * H + S::OUT;
	k_out_wgrad<<<sl, H, 0, st_>>>(n, rows, d4, a3_.p, part_.p);
	k_reduce_slices<<<blocks(lo, 256), 256, 0, st_>>>(sl, lo, part_.p, grad_.p + S::OFF_W4);  // W4 then b4
	k_out_back<<<blocks((long long)n * H, 256), 256, 0, st_>>>(n, d4, wb_.p + S::OFF_W4, z3_.p, g3_.p);
	ok(cudaGetLastError(), "backward out");
	const int slices = std::min(64, std::max(1, n / 256));
	auto wgrad = [&](const uint16_t* g, const uint16_t* a, int in, int off_w, int off_b) {
		Epi e{};
		e.part = part_.p;
		gemm<L_COL, L_COL, EPI_PARTIAL>(H, in, n, g, H, a, in, slices, e, st_);
		const int ks = ((n + slices - 1) / slices + BK - 1) / BK * BK;
		const int s_used = (n + ks - 1) / ks;
		k_reduce_slices<<<blocks(H * in, 256), 256, 0, st_>>>(s_used, H * in, part_.p, grad_.p + off_w);
		k_colsum<<<sl, H, 0, st_>>>(n, rows, g, part_.p);
		k_reduce_slices<<<1, H, 0, st_>>>(sl, H, part_.p, grad_.p + off_b);
	};
	wgrad(g3_.p, a2_.p, H, S::OFF_W3, S::OFF_B3);
	Epi e{};
	e.ldo = H;
	e.zin = z2_.p;
	e.hout = g2_.p;
	gemm<L_ROW, L_COL, EPI_BWD_GELU>(n, H, H, g3_.p, H, wb_.p + S::OFF_W3, H, 1, e, st_);
	wgrad(g2_.p, a1_.p, H, S::OFF_W2, S::OFF_B2);
	e.zin = z1_.p;
	e.hout = g1_.p;  // d4 is dead by now
	gemm<L_ROW, L_COL, EPI_BWD_GELU>(n, H, H, g2_.p, H, wb_.p + S::OFF_W2, H, 1, e, st_);
	wgrad(g1_.p, x_.p, S::IN, S::OFF_W1, S::OFF_B1);
	ok(cudaGetLastError(), "backward");
	if (loss_out) {
		ok(cudaMemcpyAsync(loss_out, loss_d_.p, sizeof(double), cudaMemcpyDeviceToHost, st_), "loss");
		ok(cudaStreamSynchronize(st_), "sync");
	}
}

double Surrogate::train(int steps, int batch, double lr, std::vector<float>* loss_per_step) {
	if (steps <= 0) return 0.0;
	if (batch < 64 || batch > (1 << 20)) throw Error(E3D_ERR_ARG, "surrogate: batch must be in [64, 2^20]");
	if (n_samples_ < 2) throw Error(E3D_ERR_STATE, "surrogate: no training samples");
	if (!normalised_) fit_normalisation();
	ensure_work(batch);
	DevBuf<double> hist;
	hist.alloc((size_t)steps);
	const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
	for (int s = 0; s < steps; s++) {
		k_prepare<<<blocks(batch, 256), 256, 0, st_>>>(batch, feat_.p, 8, state_.p, 8, n_samples_, seed_, step_,
		                                               norm_.p, (float)gamma_, x_.p, t_.p);
		forward(batch);
		backward(batch, nullptr);
		ok(cudaMemcpyAsync(hist.p + s, loss_d_.p, sizeof(double), cudaMemcpyDeviceToDevice, st_), "loss");
		step_++;
		// cosine decay to 5% of lr over this call
		const double frac = steps > 1 ? (double)s / (steps - 1) : 1.0;
		const float lr_s = (float)(lr * (0.05 + 0.95 * 0.5 * (1.0 + std::cos(3.14159265358979 * frac))));
		const float c1 = 1.f - std::pow(b1, (float)step_), c2 = 1.f - std::pow(b2, (float)step_);
		k_adam<<<blocks(S::N_PARAM, 256), 256, 0, st_>>>(S::N_PARAM, master_.p, m1_.p, m2_.p, grad_.p, wb_.p, lr_s,
		                                                 b1, b2, eps, c1, c2);
	}
	ok(cudaGetLastError(), "train");
	std::vector<double> h(steps);
	ok(cudaMemcpyAsync(h.data(), hist.p, steps * sizeof(double), cudaMemcpyDeviceToHost, st_), "loss history");
	ok(cudaStreamSynchronize(st_), "sync");
	if (loss_per_step) loss_per_step->assign(h.begin(), h.end());
	const int k = std::min(steps, 50);
	double m = 0.0;
	for (int i = steps - k; i < steps; i++) m += h[i];
	return m / k;
}

double Surrogate::gradient(const float* feat6, const float* state5, int n, std::vector<float>& grad) {
	if (n < 1 || n > (1 << 20)) throw Error(E3D_ERR_ARG, "surrogate: sample count out of range");
	std::vector<float> f((size_t)n * 8, 0.f), s((size_t)n * 8, 0.f);
	for (int i = 0; i < n; i++) {
		for (int j = 0; j < 6; j++) f[(size_t)i * 8 + j] = feat6[(size_t)i * 6 + j];
		for (int q = 0; q < 5; q++) s[(size_t)i * 8 + q] = state5[(size_t)i * 5 + q];
	}
	DevBuf<float> fd, sd;
	fd.upload(f);
	sd.upload(s);
	ensure_work(n);
	k_prepare<<<blocks(n, 256), 256, 0, st_>>>(n, fd.p, 8, sd.p, 8, 0, 0, 0, norm_.p, (float)gamma_, x_.p, t_.p);
	forward(n);
	double loss = 0.0;
	backward(n, &loss);
	grad.resize(S::N_PARAM);
	ok(cudaMemcpyAsync(grad.data(), grad_.p, S::N_PARAM * sizeof(float), cudaMemcpyDeviceToHost, st_), "grad");
	ok(cudaStreamSynchronize(st_), "sync");
	return loss;
}

void Surrogate::predict_device(const float* feat, long long n, float* state, cudaStream_t consumer) {
	if (consumer) ok(cudaStreamSynchronize(consumer), "sync");
	const int chunk = 1 << 20;
	ensure_work((int)std::min<long long>(n, chunk));
	for (long long b0 = 0; b0 < n; b0 += chunk) {
		const int m = (int)std::min<long long>(chunk, n - b0);
		k_prepare<<<blocks(m, 256), 256, 0, st_>>>(m, feat + b0 * 8, 8, nullptr, 0, 0, 0, 0, norm_.p, (float)gamma_,
		                                           x_.p, nullptr);
		forward(m);
		k_denormalise<<<blocks(m, 256), 256, 0, st_>>>(m, y_.p, feat + b0 * 8, 8, norm_.p, (float)gamma_,
		                                               state + b0 * 8, 8);
	}
	ok(cudaGetLastError(), "predict");
	ok(cudaStreamSynchronize(st_), "sync");
}

void Surrogate::predict_host(const float* feat6, long long n, float* state5) {
	if (n <= 0) return;
	std::vector<float> f((size_t)n * 8, 0.f);
	for (long long i = 0; i < n; i++)
		for (int j = 0; j < 6; j++) f[i * 8 + j] = feat6[i * 6 + j];
	DevBuf<float> fd, sd;
	fd.upload(f);
	sd.alloc((size_t)n * 8);
	predict_device(fd.p, n, sd.p, nullptr);
	std::vector<float> s((size_t)n * 8);
	ok(cudaMemcpy(s.data(), sd.p, s.size() * sizeof(float), cudaMemcpyDeviceToHost), "predict");
	for (long long i = 0; i < n; i++)
		for (int q = 0; q < 5; q++) state5[i * 5 + q] = s[i * 8 + q];
}

int Surrogate::warm_start(Engine& e) {
	const int nr = e.n_real_total();
	DevBuf<float> f, w;
	f.alloc((size_t)nr * 8);
	w.alloc((size_t)nr * 8);
	e.cell_features(f.p);
	predict_device(f.p, nr, w.p, e.stream());
	return e.apply_conservative(w.p, 8);
}

void Surrogate::get_params(float* out) const {
	ok(cudaMemcpy(out, master_.p, S::N_PARAM * sizeof(float), cudaMemcpyDeviceToHost), "params");
}
void Surrogate::set_params(const float* in) {
	ok(cudaMemcpy(master_.p, in, S::N_PARAM * sizeof(float), cudaMemcpyHostToDevice), "params");
	upload_params();
	ok(cudaStreamSynchronize(st_), "sync");
}
void Surrogate::get_normalisation(float* out) const { std::memcpy(out, norm_h_.data(), S::N_NORM * sizeof(float)); }
void Surrogate::set_normalisation(const float* in) {
	norm_h_.assign(in, in + S::N_NORM);
	norm_.upload(norm_h_);
	normalised_ = true;
}

}  // namespace e3d
