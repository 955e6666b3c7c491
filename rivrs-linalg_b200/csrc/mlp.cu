// Training and inference kernels of the per-front precision selector (the
// perceptron of mlp.cuh): forward pass, the gradient of the weighted binary
// cross-entropy over a sample set, and an Adam step.  The selector has no
// counterpart in the reference; its labels come from factoring fronts both
// ways (FP64 and the mixed form), see selector.py.
//
// The gradient is deterministic: each CTA owns a fixed slice of the samples,
// each of its 8 warps accumulates its samples' gradients in a private
// shared-memory copy, the CTA adds the 8 copies in warp order into its own
// partial, and a second kernel adds the partials in CTA order.  The caller
// passes that partial buffer (rvg_mlp_work_floats), so nothing is allocated.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>

#include "mlp.cuh"
#include "rvg_internal.h"

namespace rvg {

constexpr int MLP_WARPS = 8;
constexpr int MLP_MAX_BLOCKS = 296;
constexpr size_t MLP_GRAD_SMEM = (size_t)MLP_WARPS * (MLP_NTRAIN * sizeof(float) + sizeof(MlpAct)) + 64;

int64_t mlp_blocks(int64_t n) { return std::max<int64_t>(1, std::min<int64_t>((n + 31) / 32, MLP_MAX_BLOCKS)); }

__global__ void k_mlp_forward(const float* __restrict__ P, const float* __restrict__ X, int64_t n,
                              float* __restrict__ prob) {
  __shared__ MlpAct act[MLP_WARPS];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int64_t i = (int64_t)blockIdx.x * MLP_WARPS + warp; i < n; i += (int64_t)gridDim.x * MLP_WARPS) {
    const float xin = lane < MLP_IN ? X[i * MLP_IN + lane] : 0.f;
    const float z = mlp_forward_warp(P, xin, act[warp]);
    if (lane == 0) prob[i] = mlp_sigmoid(z);
    __syncwarp();
  }
}

__global__ void __launch_bounds__(MLP_WARPS * 32) k_mlp_grad(const float* __restrict__ P,
                                                             const float* __restrict__ X,
                                                             const float* __restrict__ Y,
                                                             const float* __restrict__ Wt, int64_t n,
                                                             float inv_norm, float* __restrict__ partial) {
  extern __shared__ float smem[];
  float* G = smem;  // MLP_WARPS private gradient copies
  MlpAct* act = (MlpAct*)(smem + (size_t)MLP_WARPS * MLP_NTRAIN);
  __shared__ float wloss[MLP_WARPS];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int p = threadIdx.x; p < MLP_WARPS * MLP_NTRAIN; p += blockDim.x) G[p] = 0.f;
  __syncthreads();
  float* g = G + (size_t)warp * MLP_NTRAIN;
  MlpAct& a = act[warp];
  const int64_t chunk = (n + gridDim.x - 1) / gridDim.x;
  const int64_t i0 = (int64_t)blockIdx.x * chunk, i1 = min(n, i0 + chunk);
  float lsum = 0.f;
  for (int64_t i = i0 + warp; i < i1; i += MLP_WARPS) {
    const float xin = lane < MLP_IN ? X[i * MLP_IN + lane] : 0.f;
    const float z = mlp_forward_warp(P, xin, a);
    const float y = Y[i], w = Wt ? Wt[i] : 1.f;
    const float pr = mlp_sigmoid(z);
    // loss = w (softplus(z) - y z), in the form that never overflows
    const float sp = __fadd_rn(z > 0.f ? z : 0.f, log1pf(expf(-fabsf(z))));
    lsum = __fadd_rn(lsum, __fmul_rn(__fmul_rn(w, __fsub_rn(sp, __fmul_rn(y, z))), inv_norm));
    const float dz = __fmul_rn(__fmul_rn(w, __fsub_rn(pr, y)), inv_norm);
    if (lane == 0) g[MLP_B3] = __fadd_rn(g[MLP_B3], dz);
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      const int u = lane + 32 * r;
      g[MLP_W3 + u] = __fmaf_rn(dz, a.h2[u], g[MLP_W3 + u]);
      const float d2 = a.h2[u] > 0.f ? __fmul_rn(dz, P[MLP_W3 + u]) : 0.f;
      a.d2[u] = d2;
      g[MLP_B2 + u] = __fadd_rn(g[MLP_B2 + u], d2);
    }
    __syncwarp();
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      const int c = lane + 32 * r;  // this lane's column of W2 and unit of layer 1
      const float hc = a.h1[c];
      float dh = 0.f;
      for (int u = 0; u < MLP_H; ++u) {
        const float d2 = a.d2[u];
        g[MLP_W2 + u * MLP_H + c] = __fmaf_rn(d2, hc, g[MLP_W2 + u * MLP_H + c]);
        dh = __fmaf_rn(P[MLP_W2 + u * MLP_H + c], d2, dh);
      }
      const float d1 = hc > 0.f ? dh : 0.f;
      g[MLP_B1 + c] = __fadd_rn(g[MLP_B1 + c], d1);
      for (int j = 0; j < MLP_IN; ++j) g[MLP_W1 + c * MLP_IN + j] = __fmaf_rn(d1, a.x[j], g[MLP_W1 + c * MLP_IN + j]);
    }
    __syncwarp();
  }
  if (lane == 0) wloss[warp] = lsum;
  __syncthreads();
  float* out = partial + (size_t)blockIdx.x * (MLP_NTRAIN + 1);
  for (int p = threadIdx.x; p < MLP_NTRAIN; p += blockDim.x) {
    float s = 0.f;
    for (int w = 0; w < MLP_WARPS; ++w) s = __fadd_rn(s, G[(size_t)w * MLP_NTRAIN + p]);
    out[p] = s;
  }
  if (threadIdx.x == 0) {
    float s = 0.f;
    for (int w = 0; w < MLP_WARPS; ++w) s = __fadd_rn(s, wloss[w]);
    out[MLP_NTRAIN] = s;
  }
}

__global__ void k_mlp_reduce(const float* __restrict__ partial, int nb, float* __restrict__ grad,
                             float* __restrict__ loss) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p > MLP_NTRAIN) return;
  float s = 0.f;
  for (int b = 0; b < nb; ++b) s = __fadd_rn(s, partial[(size_t)b * (MLP_NTRAIN + 1) + p]);
  if (p < MLP_NTRAIN) grad[p] = s;
  else if (loss) *loss = s;
}

// Adam (Kingma & Ba, 2015) with decoupled weight decay; bc1 = 1 - beta1^t,
// bc2 = 1 - beta2^t.
__global__ void k_mlp_adam(float* __restrict__ P, const float* __restrict__ G, float* __restrict__ M,
                           float* __restrict__ V, float lr, float b1, float b2, float eps, float wd, float bc1,
                           float bc2) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= MLP_NTRAIN) return;
  const float g = G[p];
  const float m = __fadd_rn(__fmul_rn(b1, M[p]), __fmul_rn(__fsub_rn(1.f, b1), g));
  const float v = __fadd_rn(__fmul_rn(b2, V[p]), __fmul_rn(__fsub_rn(1.f, b2), __fmul_rn(g, g)));
  M[p] = m;
  V[p] = v;
  const float mh = m / bc1, vh = v / bc2;
  const float step = __fadd_rn(mh / __fadd_rn(sqrtf(vh), eps), __fmul_rn(wd, P[p]));
  P[p] = __fsub_rn(P[p], __fmul_rn(lr, step));
}

}  // namespace rvg

using namespace rvg;

#define MLP_CK(call)                                                                            \
  do {                                                                                          \
    cudaError_t e_ = (call);                                                                    \
    if (e_ != cudaSuccess) {                                                                    \
      set_error(std::string("CUDA error: ") + cudaGetErrorString(e_) + " at " #call);           \
      return RVG_ERR_DEVICE;                                                                    \
    }                                                                                           \
  } while (0)

extern "C" {

int64_t rvg_mlp_param_count(void) { return MLP_NPARAM; }
int64_t rvg_mlp_trained_count(void) { return MLP_NTRAIN; }
int64_t rvg_mlp_work_floats(int64_t n) { return n < 0 ? 0 : mlp_blocks(n) * (MLP_NTRAIN + 1); }

rvg_status rvg_mlp_forward(const float* d_params, const float* d_x, int64_t n, float* d_prob, void* stream) {
  if (n < 0 || (n > 0 && (!d_params || !d_x || !d_prob))) { set_error("mlp_forward: null argument"); return RVG_ERR_INVALID_INPUT; }
  if (n == 0) return RVG_OK;
  const int64_t blocks = std::min<int64_t>((n + MLP_WARPS - 1) / MLP_WARPS, 148 * 8);
  k_mlp_forward<<<(unsigned)blocks, MLP_WARPS * 32, 0, (cudaStream_t)stream>>>(d_params, d_x, n, d_prob);
  MLP_CK(cudaGetLastError());
  return RVG_OK;
}

rvg_status rvg_mlp_grad(const float* d_params, const float* d_x, const float* d_y, const float* d_weight, int64_t n,
                        double norm, float* d_grad, float* d_loss, float* d_work, int64_t work_floats, void* stream) {
  if (n <= 0 || !d_params || !d_x || !d_y || !d_grad || !d_work) { set_error("mlp_grad: null argument or no samples"); return RVG_ERR_INVALID_INPUT; }
  if (!(norm > 0)) { set_error("mlp_grad: norm must be positive"); return RVG_ERR_INVALID_INPUT; }
  const int64_t nb = mlp_blocks(n);
  if (work_floats < nb * (MLP_NTRAIN + 1)) { set_error("mlp_grad: work buffer smaller than rvg_mlp_work_floats(n)"); return RVG_ERR_INVALID_INPUT; }
  int dev = 0;
  MLP_CK(cudaGetDevice(&dev));
  static bool attr[256] = {};
  if (dev < 0 || dev >= 256) { set_error("mlp_grad: device ordinal beyond the supported range"); return RVG_ERR_INVALID_INPUT; }
  if (!attr[dev]) {  // the kernel's shared-memory limit, once per device
    MLP_CK(cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)MLP_GRAD_SMEM));
    attr[dev] = true;
  }
  cudaStream_t st = (cudaStream_t)stream;
  k_mlp_grad<<<(unsigned)nb, MLP_WARPS * 32, MLP_GRAD_SMEM, st>>>(d_params, d_x, d_y, d_weight, n,
                                                                 (float)(1.0 / norm), d_work);
  MLP_CK(cudaGetLastError());
  k_mlp_reduce<<<(MLP_NTRAIN + 1 + 255) / 256, 256, 0, st>>>(d_work, (int)nb, d_grad, d_loss);
  MLP_CK(cudaGetLastError());
  return RVG_OK;
}

rvg_status rvg_mlp_adam(float* d_params, const float* d_grad, float* d_m, float* d_v, int64_t step, float lr,
                        float beta1, float beta2, float eps, float weight_decay, void* stream) {
  if (!d_params || !d_grad || !d_m || !d_v || step < 1) { set_error("mlp_adam: null argument or step < 1"); return RVG_ERR_INVALID_INPUT; }
  const float bc1 = (float)(1.0 - std::pow((double)beta1, (double)step));
  const float bc2 = (float)(1.0 - std::pow((double)beta2, (double)step));
  k_mlp_adam<<<(MLP_NTRAIN + 255) / 256, 256, 0, (cudaStream_t)stream>>>(d_params, d_grad, d_m, d_v, lr, beta1, beta2,
                                                                       eps, weight_decay, bc1, bc2);
  MLP_CK(cudaGetLastError());
  return RVG_OK;
}

}  // extern "C"
