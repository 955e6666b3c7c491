// FP64 lower-triangular rank-K update, the Schur-complement contraction of
// the numeric phase:
//
//     C[i, j] = fma(-W[i, c], L[j, c], C[i, j])   for c = 0 .. K-1 in order,
//     over rows i in [r0, r1), columns j in [c0, c1), only where i >= j.
//
// W = L * D (the pivot block applied); both W and L are column-major.  Used
// for the deferred trailing update of a two-level outer block
// (update_trailing, sparse/src/symmetric/factor.rs:1418-1526, applied once per
// 256-column outer block) and the NFS x NFS contribution block
// (compute_contribution_gemm, factor.rs:1590-1652).
//
// sm_100a has no FP64 tcgen05 kind, so this is a register-blocked SIMT DFMA
// kernel: 128 x 128 CTA tile, 256 threads, 8 x 8 outputs per thread (rows
// tx + 16a, columns ty + 16b so C loads and stores coalesce along columns),
// K staged through shared memory in chunks of 16 with a register-prefetched
// double buffer.  Each output keeps one fma chain in K order, so the result is
// bit-identical to the oracle's per-entry loop.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace rvg {

constexpr int G_BM = 128, G_BN = 128, G_BK = 16, G_T = 256;

struct SyrkArgs {
  double* C;
  int64_t ldc;
  const double* W;  // W[i, c] = W[(i - r0) + c * ldw]
  int64_t ldw;
  const double* L;  // L[j, c] = L[j + c * ldl]   (j in C's column coordinates)
  int64_t ldl;
  int64_t r0, r1, c0, c1;
  int64_t K;
  const int32_t* Kdev;  // when set, K is read from device memory
};

constexpr size_t G_SMEM = 2 * 2 * G_BK * G_BM * sizeof(double);  // 64 KB, dynamic

__global__ void __launch_bounds__(G_T, 2) k_syrk_lower(SyrkArgs a) {
  const int64_t i0 = a.r0 + (int64_t)blockIdx.y * G_BM;
  const int64_t j0 = a.c0 + (int64_t)blockIdx.x * G_BN;
  if (i0 >= a.r1 || j0 >= a.c1) return;
  if (i0 + G_BM - 1 < j0) return;  // tile entirely above the diagonal
  if (a.Kdev) a.K = *a.Kdev;
  extern __shared__ double gsm[];
  double(*sW)[G_BK][G_BM] = reinterpret_cast<double(*)[G_BK][G_BM]>(gsm);
  double(*sL)[G_BK][G_BN] = reinterpret_cast<double(*)[G_BK][G_BN]>(gsm + 2 * G_BK * G_BM);
  const int tid = threadIdx.x;
  const int tx = tid & 15, ty = tid >> 4;
  double acc[8][8];
#pragma unroll
  for (int x = 0; x < 8; ++x)
#pragma unroll
    for (int y = 0; y < 8; ++y) {
      int64_t i = i0 + tx + 16 * x, j = j0 + ty + 16 * y;
      acc[x][y] = (i < a.r1 && j < a.c1 && i >= j) ? a.C[i + j * a.ldc] : 0.0;
    }
  // loader: element e (0..2047) of a 128 x 16 chunk -> row e % 128, k e / 128
  double pw[8], pl[8];
  auto load = [&](int64_t k0) {
#pragma unroll
    for (int e = 0; e < 8; ++e) {
      int idx = tid + G_T * e;
      int r = idx & (G_BM - 1), k = idx >> 7;
      int64_t kk = k0 + k;
      int64_t i = i0 + r, j = j0 + r;
      pw[e] = (i < a.r1 && kk < a.K) ? a.W[(i - a.r0) + kk * a.ldw] : 0.0;
      pl[e] = (j < a.c1 && kk < a.K) ? a.L[j + kk * a.ldl] : 0.0;
    }
  };
  auto store = [&](int buf) {
#pragma unroll
    for (int e = 0; e < 8; ++e) {
      int idx = tid + G_T * e;
      int r = idx & (G_BM - 1), k = idx >> 7;
      sW[buf][k][r] = pw[e];
      sL[buf][k][r] = pl[e];
    }
  };
  const int64_t nchunk = (a.K + G_BK - 1) / G_BK;
  if (nchunk > 0) {
    load(0);
    store(0);
  }
  __syncthreads();
  for (int64_t ch = 0; ch < nchunk; ++ch) {
    const int buf = (int)(ch & 1);
    if (ch + 1 < nchunk) load((ch + 1) * G_BK);
    const int kc = (int)((a.K - ch * G_BK) < G_BK ? (a.K - ch * G_BK) : G_BK);
#pragma unroll 4
    for (int k = 0; k < kc; ++k) {
      double wv[8], lv[8];
#pragma unroll
      for (int x = 0; x < 8; ++x) wv[x] = -sW[buf][k][tx + 16 * x];
#pragma unroll
      for (int y = 0; y < 8; ++y) lv[y] = sL[buf][k][ty + 16 * y];
#pragma unroll
      for (int x = 0; x < 8; ++x)
#pragma unroll
        for (int y = 0; y < 8; ++y) acc[x][y] = __fma_rn(wv[x], lv[y], acc[x][y]);
    }
    if (ch + 1 < nchunk) store(buf ^ 1);
    __syncthreads();
  }
#pragma unroll
  for (int x = 0; x < 8; ++x)
#pragma unroll
    for (int y = 0; y < 8; ++y) {
      int64_t i = i0 + tx + 16 * x, j = j0 + ty + 16 * y;
      if (i < a.r1 && j < a.c1 && i >= j) a.C[i + j * a.ldc] = acc[x][y];
    }
}

inline dim3 syrk_grid(const SyrkArgs& a) {
  int64_t nr = (a.r1 - a.r0 + G_BM - 1) / G_BM, nc = (a.c1 - a.c0 + G_BN - 1) / G_BN;
  return dim3((unsigned)(nc > 0 ? nc : 0), (unsigned)(nr > 0 ? nr : 0));
}

}  // namespace rvg
