// Per-front precision selector: a 12-64-64-1 perceptron (ReLU hidden layers,
// sigmoid output) that predicts from cheap front features whether the mixed
// form's tensor-core Schur updates keep a front's pivots within bound.  One
// warp evaluates one sample; lane l owns hidden units l and l + 32.  The
// parameter vector is float32: the trained part (W1, b1, W2, b2, W3, b3, row
// major, W[u][c] = weight of input c into unit u) followed by the input
// normalisation (mean and standard deviation per feature, not trained).
#pragma once
#include <cstdint>

namespace rvg {

constexpr int MLP_IN = 12, MLP_H = 64;
constexpr int MLP_W1 = 0, MLP_B1 = MLP_W1 + MLP_H * MLP_IN, MLP_W2 = MLP_B1 + MLP_H,
              MLP_B2 = MLP_W2 + MLP_H * MLP_H, MLP_W3 = MLP_B2 + MLP_H, MLP_B3 = MLP_W3 + MLP_H;
constexpr int MLP_NTRAIN = MLP_B3 + 1;  // 5057 trained parameters
constexpr int MLP_MU = MLP_NTRAIN, MLP_SD = MLP_MU + MLP_IN;
constexpr int MLP_NPARAM = MLP_SD + MLP_IN;  // 5081 with the normalisation

// Activations of one sample in a warp's shared scratch.
struct MlpAct {
  float x[MLP_IN];  // normalised input
  float h1[MLP_H];
  float h2[MLP_H];
  float d2[MLP_H];  // dL/dz2 (backward)
};

__device__ __forceinline__ float mlp_warp_sum(float v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;  // the same butterfly on every lane: identical, order-fixed result
}

// Forward pass of the sample whose raw features lanes 0..MLP_IN-1 hold in
// `xin`; returns the output logit on every lane and leaves the activations in
// `a`.  Sums run in a fixed order with explicit fused multiply-adds.
__device__ __forceinline__ float mlp_forward_warp(const float* __restrict__ P, float xin, MlpAct& a) {
  const int lane = threadIdx.x & 31;
  if (lane < MLP_IN) a.x[lane] = (xin - P[MLP_MU + lane]) / P[MLP_SD + lane];
  __syncwarp();
#pragma unroll
  for (int r = 0; r < 2; ++r) {
    const int u = lane + 32 * r;
    float z = P[MLP_B1 + u];
    for (int c = 0; c < MLP_IN; ++c) z = __fmaf_rn(P[MLP_W1 + u * MLP_IN + c], a.x[c], z);
    a.h1[u] = z > 0.f ? z : 0.f;
  }
  __syncwarp();
#pragma unroll
  for (int r = 0; r < 2; ++r) {
    const int u = lane + 32 * r;
    float z = P[MLP_B2 + u];
    for (int c = 0; c < MLP_H; ++c) z = __fmaf_rn(P[MLP_W2 + u * MLP_H + c], a.h1[c], z);
    a.h2[u] = z > 0.f ? z : 0.f;
  }
  __syncwarp();
  float part = __fmaf_rn(P[MLP_W3 + lane + 32], a.h2[lane + 32], __fmul_rn(P[MLP_W3 + lane], a.h2[lane]));
  return __fadd_rn(mlp_warp_sum(part), P[MLP_B3]);
}

__device__ __forceinline__ float mlp_sigmoid(float z) {
  return z >= 0.f ? 1.f / (1.f + expf(-z)) : expf(z) / (1.f + expf(z));
}

}  // namespace rvg
