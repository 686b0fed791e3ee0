// Learned (nw, ns) policy: sizes of the 64-128-128-2 FP32 MLP, the flat
// parameter layout and the launchers of its kernels (policy.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace qz {

constexpr int kPolicyBins = 62;  // log-spaced distance-from-bottom bins
constexpr int kPolicyIn = 64;    // bins + log2(nh)/14 + last AED deflation fraction
constexpr int kPolicyHidden = 128;
constexpr int kPolicyOut = 2;    // (nw - 16) / 64 and ns / nw, both in [0, 1]
constexpr int kPolicyW1 = 0;
constexpr int kPolicyB1 = kPolicyW1 + kPolicyHidden * kPolicyIn;
constexpr int kPolicyW2 = kPolicyB1 + kPolicyHidden;
constexpr int kPolicyB2 = kPolicyW2 + kPolicyHidden * kPolicyHidden;
constexpr int kPolicyW3 = kPolicyB2 + kPolicyHidden;
constexpr int kPolicyB3 = kPolicyW3 + kPolicyOut * kPolicyHidden;
constexpr int kPolicyParams = kPolicyB3 + kPolicyOut;

// decoding of the two outputs (clamped to [0, 1] first)
constexpr int kPolicyNwMin = 16;
constexpr int kPolicyNwSpan = 64;  // nw = 16 + y0 * 64, at most the AED window limit

void launch_policy_features(cudaStream_t st, const double* H, int64_t ld, int ktop, int kbot, float lastfrac,
                            float* out);
void launch_mlp_forward(cudaStream_t st, const float* P, const float* X, int B, float* A1, float* A2, float* Y);
void launch_mlp_backward(cudaStream_t st, const float* P, const float* X, const float* Tg, int B, const float* A1,
                         const float* A2, const float* Y, float* DY, float* D2, float* D1, float* G);
void launch_adam(cudaStream_t st, float* P, const float* G, float* M, float* V, float lr, int step);
void launch_mse(cudaStream_t st, const float* Y, const float* Tg, int count, float* out);

}  // namespace qz
