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
// sm_100a has no FP64 tcgen05 kind.  The library uses the FP64 tensor-core
// mma.sync (DMMA) kernel below; the register-blocked SIMT DFMA kernel
// k_syrk_lower_t is kept as the reference formulation.  SIMT design:
// kernel: 128 x 128 CTA tile, 256 threads (one CTA per SM: the 64 FP64
// accumulators of a thread take 128 registers), 8 x 8 outputs per thread
// (rows tx + 16a, columns ty + 16b so C loads and stores coalesce along
// columns), K staged through shared memory in chunks of 16 by cp.async in a
// three-stage pipeline (8-byte copies: panel leading dimensions are odd in
// general; out-of-range elements are zero-filled by the copy itself).  Each output keeps one fma chain in K order, so the result is
// bit-identical to the oracle's per-entry loop.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace rvg {

constexpr int G_BK = 16, G_STAGES = 3;

struct SyrkArgs {
  double* C;
  int64_t ldc;
  const double* W;  // W[i, c] = W[(i - r0) + c * ldw]
  int64_t ldw;
  const double* L;  // L[j, c] = L[j + c * ldl]   (j in C's column coordinates)
  int64_t ldl;
  int64_t r0, r1, c0, c1;
  int64_t K;
  const int32_t* Kdev;  // when set, *Kdev is added to K (columns counted on the device)
  // k_syrk_inner only: the region starts on the device: rows and
  // columns at ts = *dk + *dbs (r0 = c0 = 0 on the host), L's columns at
  // *dk, and W is indexed by absolute row
  const int32_t* dk;
  const int32_t* dbs;
  // when set, the update runs only if *cond < cond_lt (decided on the device)
  const int32_t* cond;
  int32_t cond_lt;
  const int32_t* skip;  // when set and nonzero, the launch does nothing
};

__device__ __forceinline__ void cp_async8(double* dst, const double* src, bool valid) {
  unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  int n = valid ? 8 : 0;  // 0 source bytes: the 8 destination bytes are zero-filled
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src), "r"(n));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

// NT threads; thread (tx = tid % 16, ty = tid / 16) owns rows tx + 16x
// (x < TM) and columns ty + (NT/16) y (y < TN) of a (16 TM) x ((NT/16) TN)
// tile.
template <int NT, int TM, int TN>
struct SyrkCfg {
  static constexpr int BM = 16 * TM, BN = (NT / 16) * TN, CSTR = NT / 16;
  static constexpr size_t SMEM = (size_t)G_STAGES * G_BK * (BM + BN) * sizeof(double);
};

template <int NT, int TM, int TN, int MINB>
__global__ void __launch_bounds__(NT, MINB) k_syrk_lower_t(SyrkArgs a) {
  using Cfg = SyrkCfg<NT, TM, TN>;
  constexpr int BM = Cfg::BM, BN = Cfg::BN, CS = Cfg::CSTR;
  const int64_t i0 = a.r0 + (int64_t)blockIdx.y * BM;
  const int64_t j0 = a.c0 + (int64_t)blockIdx.x * BN;
  if (i0 >= a.r1 || j0 >= a.c1) return;
  if (i0 + BM - 1 < j0) return;  // tile entirely above the diagonal
  if ((a.cond && *a.cond >= a.cond_lt) || (a.skip && *a.skip)) return;
  const int64_t K = (a.Kdev ? (int64_t)*a.Kdev : 0) + a.K;
  extern __shared__ double gsm[];
  // stage s: W chunk [k][BM] then L chunk [k][BN]
  const int tid = threadIdx.x;
  const int tx = tid & 15, ty = tid >> 4;
  const int64_t nchunk = (K + G_BK - 1) / G_BK;
  auto issue = [&](int64_t ch) {
    double* sw = gsm + (ch % G_STAGES) * G_BK * (BM + BN);
    double* sl = sw + G_BK * BM;
    const int64_t k0 = ch * G_BK;
#pragma unroll
    for (int e = 0; e < (G_BK * BM) / NT; ++e) {
      const int idx = tid + NT * e;
      const int r = idx % BM, k = idx / BM;
      const int64_t kk = k0 + k, i = i0 + r;
      const bool v = kk < K && i < a.r1;
      cp_async8(sw + k * BM + r, v ? a.W + (i - a.r0) + kk * a.ldw : a.W, v);
    }
#pragma unroll
    for (int e = 0; e < (G_BK * BN) / NT; ++e) {
      const int idx = tid + NT * e;
      const int r = idx % BN, k = idx / BN;
      const int64_t kk = k0 + k, j = j0 + r;
      const bool v = kk < K && j < a.c1;
      cp_async8(sl + k * BN + r, v ? a.L + j + kk * a.ldl : a.L, v);
    }
  };
#pragma unroll
  for (int s = 0; s < G_STAGES - 1; ++s) {
    if (s < nchunk) issue(s);
    cp_async_commit();
  }
  double acc[TM][TN];
#pragma unroll
  for (int x = 0; x < TM; ++x)
#pragma unroll
    for (int y = 0; y < TN; ++y) {
      const int64_t i = i0 + tx + 16 * x, j = j0 + ty + CS * y;
      acc[x][y] = (i < a.r1 && j < a.c1 && i >= j) ? a.C[i + j * a.ldc] : 0.0;
    }
  for (int64_t ch = 0; ch < nchunk; ++ch) {
    cp_async_wait<G_STAGES - 2>();  // chunk ch has landed
    __syncthreads();                // ... for every thread, and chunk ch-1's buffer is free
    if (ch + G_STAGES - 1 < nchunk) issue(ch + G_STAGES - 1);
    cp_async_commit();
    const double* sw = gsm + (ch % G_STAGES) * G_BK * (BM + BN);
    const double* sl = sw + G_BK * BM;
    const int kc = (int)((K - ch * G_BK) < G_BK ? (K - ch * G_BK) : G_BK);
    if (kc == G_BK) {
#pragma unroll
      for (int k = 0; k < G_BK; ++k) {
        double wv[TM], lv[TN];
#pragma unroll
        for (int x = 0; x < TM; ++x) wv[x] = -sw[k * BM + tx + 16 * x];
#pragma unroll
        for (int y = 0; y < TN; ++y) lv[y] = sl[k * BN + ty + CS * y];
#pragma unroll
        for (int x = 0; x < TM; ++x)
#pragma unroll
          for (int y = 0; y < TN; ++y) acc[x][y] = __fma_rn(wv[x], lv[y], acc[x][y]);
      }
    } else {
      for (int k = 0; k < kc; ++k) {
        double wv[TM], lv[TN];
#pragma unroll
        for (int x = 0; x < TM; ++x) wv[x] = -sw[k * BM + tx + 16 * x];
#pragma unroll
        for (int y = 0; y < TN; ++y) lv[y] = sl[k * BN + ty + CS * y];
#pragma unroll
        for (int x = 0; x < TM; ++x)
#pragma unroll
          for (int y = 0; y < TN; ++y) acc[x][y] = __fma_rn(wv[x], lv[y], acc[x][y]);
      }
    }
  }
  cp_async_wait<0>();
#pragma unroll
  for (int x = 0; x < TM; ++x)
#pragma unroll
    for (int y = 0; y < TN; ++y) {
      const int64_t i = i0 + tx + 16 * x, j = j0 + ty + CS * y;
      if (i < a.r1 && j < a.c1 && i >= j) a.C[i + j * a.ldc] = acc[x][y];
    }
}

// ---------------------------------------------------------------------------
// FP64 tensor-core variant: mma.sync m8n8k4 (DMMA).  Each 8x8x4 step adds a
// chain of four products to the accumulator in k order, the same
// per-output fma sequence as the SIMT kernel and the oracle (checked bit for
// bit on the device).  WR x WC warps of 32 x 32 outputs (4 x 4 fragments of
// 8 x 8); W is negated when its fragments are read.
// ---------------------------------------------------------------------------
template <int WR, int WC>
struct DmmaCfg {
  static constexpr int NT = 32 * WR * WC, BM = 32 * WR, BN = 32 * WC;
  static constexpr int LDW = BM + 8, LDL = BN + 8;  // k rows shifted 64 B apart: conflict-free fragment reads
  static constexpr size_t SMEM = (size_t)G_STAGES * G_BK * (LDW + LDL) * sizeof(double);
};

template <int WR, int WC, int MINB, bool DEV = false>
__global__ void __launch_bounds__(32 * WR * WC, MINB) k_syrk_dmma(SyrkArgs a) {
  using Cfg = DmmaCfg<WR, WC>;
  constexpr int NT = Cfg::NT, BM = Cfg::BM, BN = Cfg::BN, LDW = Cfg::LDW, LDL = Cfg::LDL;
  if (DEV) chain_enter();  // the inner update runs in the large-front chain
  if (DEV) {
    const int64_t k = *a.dk, ts = k + *a.dbs;
    a.L += k * a.ldl;
    a.W += ts;
    a.r0 = ts;
    a.c0 = ts;
  }
  const int64_t i0 = a.r0 + (int64_t)blockIdx.y * BM;
  const int64_t j0 = a.c0 + (int64_t)blockIdx.x * BN;
  if (i0 >= a.r1 || j0 >= a.c1) return;
  if (i0 + BM - 1 < j0) return;
  if ((a.cond && *a.cond >= a.cond_lt) || (a.skip && *a.skip)) return;
  const int64_t K = (a.Kdev ? (int64_t)*a.Kdev : 0) + a.K;
  if (K <= 0) return;  // nothing eliminated: C unchanged
  extern __shared__ double gsm[];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wr = (warp % WR) * 32, wc = (warp / WR) * 32;
  const int64_t nchunk = (K + G_BK - 1) / G_BK;
  auto issue = [&](int64_t ch) {
    double* sw = gsm + (ch % G_STAGES) * G_BK * (LDW + LDL);
    double* sl = sw + G_BK * LDW;
    const int64_t k0 = ch * G_BK;
#pragma unroll
    for (int e = 0; e < (G_BK * BM) / NT; ++e) {
      const int idx = tid + NT * e;
      const int r = idx % BM, k = idx / BM;
      const int64_t kk = k0 + k, i = i0 + r;
      const bool v = kk < K && i < a.r1;
      cp_async8(sw + k * LDW + r, v ? a.W + (i - a.r0) + kk * a.ldw : a.W, v);
    }
#pragma unroll
    for (int e = 0; e < (G_BK * BN) / NT; ++e) {
      const int idx = tid + NT * e;
      const int r = idx % BN, k = idx / BN;
      const int64_t kk = k0 + k, j = j0 + r;
      const bool v = kk < K && j < a.c1;
      cp_async8(sl + k * LDL + r, v ? a.L + j + kk * a.ldl : a.L, v);
    }
  };
#pragma unroll
  for (int s = 0; s < G_STAGES - 1; ++s) {
    if (s < nchunk) issue(s);
    cp_async_commit();
  }
  double acc[4][4][2];
  const int fr = lane >> 2, fc = (lane & 3) * 2;
#pragma unroll
  for (int mi = 0; mi < 4; ++mi)
#pragma unroll
    for (int ni = 0; ni < 4; ++ni)
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const int64_t i = i0 + wr + mi * 8 + fr, j = j0 + wc + ni * 8 + fc + q;
        acc[mi][ni][q] = (i < a.r1 && j < a.c1 && i >= j) ? a.C[i + j * a.ldc] : 0.0;
      }
  for (int64_t ch = 0; ch < nchunk; ++ch) {
    cp_async_wait<G_STAGES - 2>();
    __syncthreads();
    if (ch + G_STAGES - 1 < nchunk) issue(ch + G_STAGES - 1);
    cp_async_commit();
    const double* sw = gsm + (ch % G_STAGES) * G_BK * (LDW + LDL);
    const double* sl = sw + G_BK * LDW;
    // k beyond K is zero-filled in both operands: those steps add exact zeros
#pragma unroll
    for (int k4 = 0; k4 < G_BK; k4 += 4) {
      double af[4], bf[4];
      const int kk = k4 + (lane & 3);
#pragma unroll
      for (int mi = 0; mi < 4; ++mi) af[mi] = -sw[kk * LDW + wr + mi * 8 + fr];
#pragma unroll
      for (int ni = 0; ni < 4; ++ni) bf[ni] = sl[kk * LDL + wc + ni * 8 + fr];
#pragma unroll
      for (int mi = 0; mi < 4; ++mi)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni)
          asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                       : "+d"(acc[mi][ni][0]), "+d"(acc[mi][ni][1])
                       : "d"(af[mi]), "d"(bf[ni]));
    }
  }
  cp_async_wait<0>();
#pragma unroll
  for (int mi = 0; mi < 4; ++mi)
#pragma unroll
    for (int ni = 0; ni < 4; ++ni)
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const int64_t i = i0 + wr + mi * 8 + fr, j = j0 + wc + ni * 8 + fc + q;
        if (i < a.r1 && j < a.c1 && i >= j) a.C[i + j * a.ldc] = acc[mi][ni][q];
      }
}


// the configuration used by the library: DMMA, 2 x 2 warps (64 x 64 tile),
// four CTAs per SM (the fastest of the measured shapes: 25-28 TFLOP/s on a
// 16384^2 rank-256 / rank-1024 update)
#ifndef RVG_SYRK_WR
#define RVG_SYRK_WR 2
#define RVG_SYRK_WC 2
#define RVG_SYRK_MINB 4
#endif
using SyrkMain = DmmaCfg<RVG_SYRK_WR, RVG_SYRK_WC>;
constexpr int G_T = SyrkMain::NT;
constexpr size_t G_SMEM = SyrkMain::SMEM;
#define k_syrk_lower k_syrk_dmma<RVG_SYRK_WR, RVG_SYRK_WC, RVG_SYRK_MINB>
// the same kernel with the region start read from the device (SyrkArgs::dk)
#define k_syrk_inner k_syrk_dmma<RVG_SYRK_WR, RVG_SYRK_WC, 3, true>

template <class Cfg>
inline dim3 syrk_grid_cfg(const SyrkArgs& a) {
  int64_t nr = (a.r1 - a.r0 + Cfg::BM - 1) / Cfg::BM, nc = (a.c1 - a.c0 + Cfg::BN - 1) / Cfg::BN;
  return dim3((unsigned)(nc > 0 ? nc : 0), (unsigned)(nr > 0 ? nr : 0));
}
inline dim3 syrk_grid(const SyrkArgs& a) { return syrk_grid_cfg<SyrkMain>(a); }

}  // namespace rvg
