// Per-cell warm-start surrogate: a 4-layer MLP 6 -> 128 -> 128 -> 128 -> 5
// with exact-erf GELU after the three hidden layers, BF16 weights and FP32
// accumulation on the tensor cores (mma.sync m16n8k16), trained by its own
// forward/backward kernels and Adam on FP32 master weights.
//
// Inputs (raw): centroid x, y, z, wall distance, Mach, alpha in degrees; they
// are standardised with the mean and standard deviation of the training set.
// Output: the conservative state (rho, rho u, rho v, rho w, rho E) as
// W = W_free(Mach, alpha) + scale * y, where y is the network output and scale
// the per-component RMS of W - W_free over the training set.
// No part of this has a counterpart in the reference solver.
#pragma once
#include <cstdint>
#include <vector>

#include <cuda_runtime.h>

#include "engine.hpp"

namespace e3d {

struct SurrogateShape {
	static constexpr int IN = 16;     // padded input width (6 used)
	static constexpr int H = 128;     // hidden width
	static constexpr int OUT = 8;     // padded output width (5 used)
	static constexpr int N_IN = 6, N_OUT = 5;
	// flat FP32 parameter vector: W1 [H][IN], b1 [H], W2 [H][H], b2 [H], W3 [H][H], b3 [H], W4 [OUT][H], b4 [OUT]
	static constexpr int OFF_W1 = 0, OFF_B1 = OFF_W1 + H * IN, OFF_W2 = OFF_B1 + H, OFF_B2 = OFF_W2 + H * H,
	                     OFF_W3 = OFF_B2 + H, OFF_B3 = OFF_W3 + H * H, OFF_W4 = OFF_B3 + H, OFF_B4 = OFF_W4 + OUT * H,
	                     N_PARAM = OFF_B4 + OUT;
	static constexpr int N_NORM = 24;  // feature mean [8], feature std [8], target scale [8]
};

class Surrogate {
public:
	Surrogate(int device, uint64_t seed, double gamma);
	~Surrogate();
	Surrogate(const Surrogate&) = delete;
	Surrogate& operator=(const Surrogate&) = delete;

	// training set: raw features [n][8] (6 used) and conservative states [n][8] (5 used), device pointers
	void add_samples_device(const float* feat, const float* state, long long n, cudaStream_t producer);
	void add_samples_host(const float* feat6, const float* state5, long long n);
	void add_solution(Engine& e);
	void clear_samples();
	long long n_samples() const { return n_samples_; }

	// fits the normalisation on the first call (or when refit), then runs `steps` Adam steps on minibatches
	// of `batch` samples drawn with a counter-based hash; returns the mean loss of the last min(steps, 50) steps
	double train(int steps, int batch, double lr, std::vector<float>* loss_per_step);
	// full-batch loss and gradient of the FP32 master parameters for the given host samples (no update)
	double gradient(const float* feat6, const float* state5, int n, std::vector<float>& grad);
	// inference: raw features [n][8] device -> conservative states [n][8] device
	void predict_device(const float* feat, long long n, float* state, cudaStream_t consumer);
	void predict_host(const float* feat6, long long n, float* state5);
	// predicted state into every real cell of every case of the solver; returns the fallback count
	int warm_start(Engine& e);

	void get_params(float* out) const;
	void set_params(const float* in);
	void get_normalisation(float* out) const;
	void set_normalisation(const float* in);

private:
	void fit_normalisation();
	void upload_params();
	void forward(int n);                         // rows prepared in x_ (n <= work_n_)
	void backward(int n, double* loss_out);      // against the targets in t_
	void ensure_work(int n);

	int device_;
	double gamma_;
	uint64_t seed_;
	cudaStream_t st_ = nullptr;
	long long n_samples_ = 0, cap_samples_ = 0;
	DevBuf<float> feat_, state_;             // sample store
	DevBuf<float> master_, m1_, m2_, grad_;  // FP32 params, Adam moments, reduced gradient
	DevBuf<uint16_t> wb_;                    // BF16 copies of W1..W4 (same offsets, biases unused)
	DevBuf<float> norm_;                     // N_NORM floats
	std::vector<float> norm_h_;
	bool normalised_ = false;
	long long step_ = 0;
	// per-minibatch work buffers
	int work_n_ = 0;
	DevBuf<uint16_t> x_, a1_, a2_, a3_, g1_, g2_, g3_;
	DevBuf<float> z1_, z2_, z3_, y_, t_, part_, lossp_;
	DevBuf<double> loss_d_;
};

}  // namespace e3d
