// Learned tuning of the multishift QZ iteration: a 64-128-128-2 FP32 MLP
// that picks the AED window size nw and the shift count ns at every AED
// decision from a profile of the active block's subdiagonal.  It takes the
// place of the fixed PIPARMQ/PILAENVX table (piparmq.f:438-535), which stays
// the fallback: the solver uses the table whenever no weights are loaded or
// a prediction is not finite.  A bad prediction can only change how fast
// the iteration converges: the transformations stay orthogonal.
//
// Kernels (all hand-written, FP32):
//   k_features   one CTA: 64 features of the active block [ktop, kbot]
//   k_mlp_fwd    one CTA per sample: the two hidden layers and the output
//   k_mlp_delta  one CTA per sample: back-propagated deltas of the MSE loss
//   k_mlp_grad   one thread per parameter: weight gradients summed over the
//                batch in a fixed order (deterministic)
//   k_adam       Adam update of the flat parameter vector
//
// Parameter layout (flat, row-major out x in):
//   W1[128x64] b1[128] W2[128x128] b2[128] W3[2x128] b3[2]
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "policy.h"

namespace qz {

namespace {

constexpr int kThreadsF = 256;

// x_k in [0, 1]: -log10 of the relative subdiagonal |h(k+1,k)| /
// (|h(k,k)| + |h(k+1,k+1)|) (the deflation test's ratio), clipped to 16
// decades; 1 means negligible.
__device__ __forceinline__ float subdiag_level(double hs, double d0, double d1) {
  double den = fabs(d0) + fabs(d1);
  double a = fabs(hs);
  if (a == 0.0) return 1.0f;
  if (den == 0.0) return 0.0f;
  double r = -log10(a / den);
  r = r < 0.0 ? 0.0 : (r > 16.0 ? 16.0 : r);
  return (float)(r / 16.0);
}

__global__ void __launch_bounds__(kThreadsF) k_features(const double* __restrict__ H, int64_t ld, int ktop, int kbot,
                                                        float lastfrac, float* __restrict__ out) {
  __shared__ float sum[kPolicyBins];
  __shared__ int cnt[kPolicyBins];
  for (int b = threadIdx.x; b < kPolicyBins; b += blockDim.x) { sum[b] = 0.f; cnt[b] = 0; }
  __syncthreads();
  const int nh = kbot - ktop + 1;
  const double lg = log((double)(nh > 2 ? nh : 2));
  // subdiagonal k (rows k+1, k), distance from the bottom d = kbot-1-k
  for (int k = ktop + threadIdx.x; k < kbot; k += blockDim.x) {
    const double hs = H[(k + 1) + (int64_t)k * ld];
    const double d0 = H[k + (int64_t)k * ld];
    const double d1 = H[(k + 1) + (int64_t)(k + 1) * ld];
    const float x = subdiag_level(hs, d0, d1);
    const int d = kbot - 1 - k;
    int b = (int)((double)kPolicyBins * log(1.0 + (double)d) / lg);
    b = b < 0 ? 0 : (b >= kPolicyBins ? kPolicyBins - 1 : b);
    atomicAdd(&sum[b], x);
    atomicAdd(&cnt[b], 1);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    float prev = 0.f;
    for (int b = 0; b < kPolicyBins; ++b) {
      float v = cnt[b] > 0 ? sum[b] / (float)cnt[b] : prev;
      out[b] = v;
      prev = v;
    }
    out[kPolicyBins] = log2f((float)nh) / 14.0f;
    out[kPolicyBins + 1] = lastfrac;
  }
}

__global__ void __launch_bounds__(kPolicyHidden) k_mlp_fwd(const float* __restrict__ P, const float* __restrict__ X,
                                                           float* __restrict__ A1, float* __restrict__ A2,
                                                           float* __restrict__ Y) {
  __shared__ float x[kPolicyIn];
  __shared__ float a1[kPolicyHidden];
  __shared__ float a2[kPolicyHidden];
  const int b = blockIdx.x, j = threadIdx.x;
  if (j < kPolicyIn) x[j] = X[(int64_t)b * kPolicyIn + j];
  __syncthreads();
  float acc = P[kPolicyB1 + j];
  const float* w1 = P + kPolicyW1 + j * kPolicyIn;
  for (int i = 0; i < kPolicyIn; ++i) acc = fmaf(w1[i], x[i], acc);
  acc = acc > 0.f ? acc : 0.f;
  a1[j] = acc;
  A1[(int64_t)b * kPolicyHidden + j] = acc;
  __syncthreads();
  acc = P[kPolicyB2 + j];
  const float* w2 = P + kPolicyW2 + j * kPolicyHidden;
  for (int i = 0; i < kPolicyHidden; ++i) acc = fmaf(w2[i], a1[i], acc);
  acc = acc > 0.f ? acc : 0.f;
  a2[j] = acc;
  A2[(int64_t)b * kPolicyHidden + j] = acc;
  __syncthreads();
  if (j < kPolicyOut) {
    float y = P[kPolicyB3 + j];
    const float* w3 = P + kPolicyW3 + j * kPolicyHidden;
    for (int i = 0; i < kPolicyHidden; ++i) y = fmaf(w3[i], a2[i], y);
    Y[(int64_t)b * kPolicyOut + j] = y;
  }
}

// Deltas of L = (1 / (B * 2)) * sum (Y - T)^2 for one sample.
__global__ void __launch_bounds__(kPolicyHidden) k_mlp_delta(const float* __restrict__ P, const float* __restrict__ Tg,
                                                             const float* __restrict__ A1,
                                                             const float* __restrict__ A2,
                                                             const float* __restrict__ Y, int B,
                                                             float* __restrict__ DY, float* __restrict__ D2,
                                                             float* __restrict__ D1) {
  __shared__ float dy[kPolicyOut];
  __shared__ float d2[kPolicyHidden];
  const int b = blockIdx.x, j = threadIdx.x;
  if (j < kPolicyOut) {
    float v = 2.f * (Y[(int64_t)b * kPolicyOut + j] - Tg[(int64_t)b * kPolicyOut + j]) / (float)(B * kPolicyOut);
    dy[j] = v;
    DY[(int64_t)b * kPolicyOut + j] = v;
  }
  __syncthreads();
  float acc = 0.f;
  for (int o = 0; o < kPolicyOut; ++o) acc = fmaf(P[kPolicyW3 + o * kPolicyHidden + j], dy[o], acc);
  acc = A2[(int64_t)b * kPolicyHidden + j] > 0.f ? acc : 0.f;
  d2[j] = acc;
  D2[(int64_t)b * kPolicyHidden + j] = acc;
  __syncthreads();
  acc = 0.f;
  for (int k = 0; k < kPolicyHidden; ++k) acc = fmaf(P[kPolicyW2 + k * kPolicyHidden + j], d2[k], acc);
  acc = A1[(int64_t)b * kPolicyHidden + j] > 0.f ? acc : 0.f;
  D1[(int64_t)b * kPolicyHidden + j] = acc;
}

// One thread per parameter: the gradient summed over the batch in sample
// order.
__global__ void k_mlp_grad(const float* __restrict__ X, const float* __restrict__ A1, const float* __restrict__ A2,
                           const float* __restrict__ DY, const float* __restrict__ D2, const float* __restrict__ D1,
                           int B, float* __restrict__ G) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= kPolicyParams) return;
  const float* d;
  const float* a;
  int dstride, astride, row, col;
  bool bias = false;
  if (p < kPolicyB1) {
    row = (p - kPolicyW1) / kPolicyIn; col = (p - kPolicyW1) % kPolicyIn;
    d = D1; dstride = kPolicyHidden; a = X; astride = kPolicyIn;
  } else if (p < kPolicyW2) {
    row = p - kPolicyB1; col = 0; bias = true; d = D1; dstride = kPolicyHidden; a = nullptr; astride = 0;
  } else if (p < kPolicyB2) {
    row = (p - kPolicyW2) / kPolicyHidden; col = (p - kPolicyW2) % kPolicyHidden;
    d = D2; dstride = kPolicyHidden; a = A1; astride = kPolicyHidden;
  } else if (p < kPolicyW3) {
    row = p - kPolicyB2; col = 0; bias = true; d = D2; dstride = kPolicyHidden; a = nullptr; astride = 0;
  } else if (p < kPolicyB3) {
    row = (p - kPolicyW3) / kPolicyHidden; col = (p - kPolicyW3) % kPolicyHidden;
    d = DY; dstride = kPolicyOut; a = A2; astride = kPolicyHidden;
  } else {
    row = p - kPolicyB3; col = 0; bias = true; d = DY; dstride = kPolicyOut; a = nullptr; astride = 0;
  }
  float acc = 0.f;
  for (int b = 0; b < B; ++b) {
    const float dv = d[(int64_t)b * dstride + row];
    acc = bias ? acc + dv : fmaf(dv, a[(int64_t)b * astride + col], acc);
  }
  G[p] = acc;
}

__global__ void k_adam(float* __restrict__ P, const float* __restrict__ G, float* __restrict__ M,
                       float* __restrict__ V, float lr, float b1, float b2, float eps, float c1, float c2) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= kPolicyParams) return;
  const float g = G[p];
  const float m = b1 * M[p] + (1.f - b1) * g;
  const float v = b2 * V[p] + (1.f - b2) * g * g;
  M[p] = m;
  V[p] = v;
  P[p] -= lr * (m / c1) / (sqrtf(v / c2) + eps);
}

__global__ void k_mse(const float* __restrict__ Y, const float* __restrict__ Tg, int count, float* __restrict__ out) {
  __shared__ float red[256];
  float acc = 0.f;
  for (int i = threadIdx.x; i < count; i += blockDim.x) {
    float e = Y[i] - Tg[i];
    acc += e * e;
  }
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[0] = red[0] / (float)count;
}

}  // namespace

void launch_policy_features(cudaStream_t st, const double* H, int64_t ld, int ktop, int kbot, float lastfrac,
                            float* out) {
  k_features<<<1, kThreadsF, 0, st>>>(H, ld, ktop, kbot, lastfrac, out);
}

void launch_mlp_forward(cudaStream_t st, const float* P, const float* X, int B, float* A1, float* A2, float* Y) {
  if (B > 0) k_mlp_fwd<<<B, kPolicyHidden, 0, st>>>(P, X, A1, A2, Y);
}

void launch_mlp_backward(cudaStream_t st, const float* P, const float* X, const float* Tg, int B, const float* A1,
                         const float* A2, const float* Y, float* DY, float* D2, float* D1, float* G) {
  if (B <= 0) return;
  k_mlp_delta<<<B, kPolicyHidden, 0, st>>>(P, Tg, A1, A2, Y, B, DY, D2, D1);
  k_mlp_grad<<<(kPolicyParams + 255) / 256, 256, 0, st>>>(X, A1, A2, DY, D2, D1, B, G);
}

void launch_adam(cudaStream_t st, float* P, const float* G, float* M, float* V, float lr, int step) {
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
  k_adam<<<(kPolicyParams + 255) / 256, 256, 0, st>>>(P, G, M, V, lr, b1, b2, 1e-8f, c1, c2);
}

void launch_mse(cudaStream_t st, const float* Y, const float* Tg, int count, float* out) {
  k_mse<<<1, 256, 0, st>>>(Y, Tg, count, out);
}

}  // namespace qz
