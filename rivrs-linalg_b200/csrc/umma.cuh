// Mixed-form Schur-complement update on the 5th-generation tensor cores.
//
//   C[i, j] -= sum_c W[i, c] L[j, c]      for the lower entries i >= j of
//   rows [r0, r1) x columns [c0, c1) of C (FP64, column-major)
//
// which is the deferred trailing update of a two-level APTP outer block and
// the NFS x NFS contribution GEMM (update_trailing and
// compute_contribution_gemm, sparse/src/aptp/factor.rs:1418-1652, the
// tri-matmul call at factor.rs:1639-1651), computed as three TF32 products
// per term (each FP64 operand split once into v = hi + lo, both parts exact
// TF32 values; lo*hi + hi*lo + hi*hi, the dropped lo*lo is below 2^-22 of
// the term) on the tensor cores, FP32 partial sums in tensor memory added
// into FP64, and subtracted from C in FP64.  The mixed factorization that
// uses it is followed by FP64 iterative refinement.
//
// Operand packing (k_pack_tf32x3).  Each operand X (R rows x K, FP64,
// column-major) is rewritten once per update as 128-row tiles x 32-deep K
// chunks; a (tile, chunk) block is 32 KB: the hi parts (16 KB) then the lo
// parts (16 KB), each in the tensor core's K-major "no swizzle" canonical
// layout: core matrices of 8 rows x 16 bytes (4 TF32 values), the 16 row
// groups of a K column of core matrices at a 128-byte stride (SBO) and the 8
// core-matrix columns of the chunk at a 2048-byte stride (LBO).  Rows >= R and
// k >= K are zeros, so partial tiles and chunks add exact zeros.
//
// The GEMM (k_syrk_tc) is persistent: one CTA per SM walks the lower tiles
// (128 x 128) in column order, with three warp roles:
//   warp 0, one thread  producer: per K chunk two cp.async.bulk copies (the
//                       W block and the L block, 32 KB each) into a 3-stage
//                       shared-memory ring, completion counted in bytes on
//                       the stage's mbarrier;
//   warp 1, one thread  MMA issuer: per chunk 4 k-steps x 3 products of
//                       tcgen05.mma.cta_group::1.kind::tf32, M = N = 128,
//                       K = 8, into one of two tensor-memory partial-sum
//                       buffers (128 FP32 columns each); tcgen05.commit frees
//                       the stage, and after G chunks hands the buffer to
//                       the epilogue;
//   warps 2..9          epilogue: warp e reads its 32-lane quarter (rows) x
//                       64-column half of a partial sum with tcgen05.ld,
//                       adds it into 64 FP64 registers and frees the buffer;
//                       after the tile's last partial sum it does C -= acc in
//                       FP64 (coalesced 256-byte column segments), while the
//                       MMAs of the next tile already run.
// The tensor cores accumulate FP32 with truncation, so the error of one
// partial sum grows about linearly with its length: G (32-deep chunks per
// partial sum) trades accuracy for epilogue work.
// Every mbarrier wait is bounded by the global timer; a wait that runs out
// sets *err, raises a CTA-wide abort flag that ends the other roles' loops,
// and the CTA still waits (bounded) for its copies and MMAs in flight and
// frees its tensor memory before it returns.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "gemm64.cuh"

namespace rvg {

constexpr int TC_BM = 128, TC_BN = 128, TC_BK = 32;
constexpr int TC_STAGES = 3;
constexpr int TC_PART = TC_BM * TC_BK;              // floats in one TF32 part of a block (4096)
constexpr int TC_BLOCK = 2 * TC_PART;               // floats in a packed (tile, chunk) block: hi + lo
constexpr uint32_t TC_BLOCK_BYTES = TC_BLOCK * 4;   // 32 KB
constexpr uint32_t TC_STAGE_BYTES = 2 * TC_BLOCK_BYTES;  // W block + L block
constexpr int TC_EPI_WARPS = 8;
constexpr int TC_THREADS = 32 * (2 + TC_EPI_WARPS);
constexpr uint32_t TC_TMEM_COLS = 2 * TC_BN;        // two accumulators
constexpr size_t TC_SMEM = (size_t)TC_STAGES * TC_STAGE_BYTES + 1024 + 32768;  // + alignment slack and a guard
constexpr uint64_t TC_TIMEOUT_NS = 2000000000ull;   // 2 s per wait
constexpr uint32_t TC_LBO = 2048, TC_SBO = 128;     // core-matrix strides of the packed layout
constexpr int TC_NO_FLUSH = 1 << 24;               // chunks per partial sum when it spans all of K

// Operand formats: each FP64 operand is split once into hi + lo parts of
// TF32 (kind::tf32, 4-byte elements, 11 significant bits per part) or of BF16
// (kind::f16 with both operands BF16, 2-byte elements, 8 significant bits per
// part: half the operand bytes, half the products' accuracy).  A packed
// (tile, chunk) block always starts TC_BLOCK floats after the previous one;
// the BF16 parts fill its first half.  A chunk is 32 deep in both formats;
// core matrices are 8 rows x 16 bytes (4 TF32 or 8 BF16 values), so one MMA
// (32 bytes of K) spans two core-matrix columns in both.
constexpr int TC_TF32 = 0, TC_BF16 = 1;
template <int FMT>
struct TcFmt {
  static constexpr int EB = FMT == TC_BF16 ? 2 : 4;              // bytes per element
  static constexpr uint32_t PART_BYTES = TC_BM * TC_BK * EB;    // hi (or lo) part of a block
  static constexpr uint32_t BLOCK_BYTES = 2 * PART_BYTES;       // bytes of a block that are read
  static constexpr int KSTEPS = TC_BK * EB / 32;                // MMAs per chunk and product
  static constexpr uint32_t AB = FMT == TC_BF16 ? 1u : 2u;      // A / B format field (BF16 in kind::f16, TF32)
  static constexpr uint32_t IDESC = (1u << 4) | (AB << 7) | (AB << 10) | ((uint32_t)(TC_BN >> 3) << 17) |
                                    ((uint32_t)(TC_BM >> 4) << 24);
};

struct TcArgs {
  double* C;
  int64_t ldc;
  int64_t r0, r1, c0, c1;
  const float* Ap;  // packed W: tile t (C rows r0 + 128 t ...), chunk q at Ap + (t * Q + q) * TC_BLOCK
  const float* Bp;  // packed L: tile u (C columns c0 + 128 u ...)
  int64_t Q;        // chunks per packed tile
  const int32_t* Kdev;  // K = *Kdev (when set) + K
  int64_t K;
  int64_t nr, nc, ntiles;
  int32_t* err;
  const int32_t* cond;  // when set, the update runs only if *cond < cond_lt
  int32_t cond_lt;
  int32_t stall;        // self-test of the bounded waits: the producer issues no copies
  const int32_t* skip;  // when set and nonzero, the launch does nothing
};

struct PackArgs {
  const double* X;  // row r, column c at X[r + c * ldx]
  int64_t ldx, R, Q;
  const int32_t* Kdev;  // K = *Kdev (when set) + K: columns >= K are zeros
  int64_t K;
  float* P;         // block (t0 + t, q) at P + ((t0 + t) * Q + q) * TC_BLOCK
  int64_t q0, t0;   // first chunk packed (blockIdx.x = q - q0), first tile
  const int32_t* cond;  // when set, packs only if *cond < cond_lt
  int32_t cond_lt;
  const int32_t* skip;  // when set and nonzero, the launch does nothing
};

// ---------------------------------------------------------------- PTX helpers
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t gtimer() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
// bounded wait for the phase with the given parity; false on abort or timeout
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, volatile int* abort_flag, int32_t* err) {
  if (mbar_try(bar, parity)) return true;
  const uint64_t t0 = gtimer();
  while (true) {
    if (mbar_try(bar, parity)) return true;
    if (*abort_flag) return false;
    if (gtimer() - t0 > TC_TIMEOUT_NS) {
      *abort_flag = 1;
      atomicExch(err, 1);
      return false;
    }
  }
}

__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ uint64_t tc_desc(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)(TC_LBO >> 4) << 16) | ((uint64_t)(TC_SBO >> 4) << 32) |
         (1ull << 46);  // descriptor version 1, no swizzle, base offset 0
}

template <int FMT>
__device__ __forceinline__ void tc_mma(uint32_t d, uint64_t a, uint64_t b, uint32_t accumulate) {
  if constexpr (FMT == TC_BF16) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d),
        "l"(a), "l"(b), "r"(TcFmt<FMT>::IDESC), "r"(accumulate)
        : "memory");
  } else {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(d),
        "l"(a), "l"(b), "r"(TcFmt<FMT>::IDESC), "r"(accumulate)
        : "memory");
  }
}
__device__ __forceinline__ void tc_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

// 32 lanes x 32 consecutive FP32 columns: thread t gets its lane's row
__device__ __forceinline__ void tc_ld32(uint32_t taddr, uint32_t* v) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
      "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
        "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
        "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
        "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tc_ld16(uint32_t taddr, uint32_t* v) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
        "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// ---------------------------------------------------------------- packing
__device__ __forceinline__ void split_tf32_exact(double x, float& hi, float& lo) {
  uint32_t h, l;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(h) : "f"((float)x));
  hi = __uint_as_float(h);
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(l) : "f"((float)(x - (double)hi)));
  lo = __uint_as_float(l);
}

// grid (Q chunks, tiles), 256 threads; thread item = one row x 4 consecutive k
__global__ void __launch_bounds__(256) k_pack_tf32x3(PackArgs a) {
  if ((a.cond && *a.cond >= a.cond_lt) || (a.skip && *a.skip)) return;
  int64_t K = (a.Kdev ? (int64_t)*a.Kdev : 0) + a.K;
  if (K > a.Q * TC_BK) K = a.Q * TC_BK;  // never beyond the chunks the buffer holds
  const int64_t q = a.q0 + blockIdx.x, t = blockIdx.y;
  if (q * TC_BK >= K) return;  // the GEMM reads chunks < ceil(K / 32) only
  float* hi = a.P + ((a.t0 + t) * a.Q + q) * TC_BLOCK;
  float* lo = hi + TC_PART;
#pragma unroll
  for (int e = 0; e < (TC_BM * TC_BK / 4) / 256; ++e) {
    const int idx = threadIdx.x + 256 * e;
    const int r = idx % TC_BM, kq = idx / TC_BM;
    const int64_t row = t * TC_BM + r;
    float hv[4], lv[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const int64_t k = q * TC_BK + kq * 4 + c;
      const double x = (row < a.R && k < K) ? a.X[row + k * a.ldx] : 0.0;
      split_tf32_exact(x, hv[c], lv[c]);
    }
    const int off = (kq * (TC_BM / 8) + (r >> 3)) * 32 + (r & 7) * 4;
    *reinterpret_cast<float4*>(hi + off) = make_float4(hv[0], hv[1], hv[2], hv[3]);
    *reinterpret_cast<float4*>(lo + off) = make_float4(lv[0], lv[1], lv[2], lv[3]);
  }
}

__device__ __forceinline__ uint16_t bf16_rn(float x) {
  uint16_t h;
  asm("cvt.rn.bf16.f32 %0, %1;" : "=h"(h) : "f"(x));
  return h;
}
__device__ __forceinline__ float bf16_to_f32(uint16_t h) { return __uint_as_float((uint32_t)h << 16); }

// BF16 parts: hi = bf16(x), lo = bf16(x - hi); grid (Q chunks, tiles), 256
// threads; thread item = one row x 8 consecutive k (one 16-byte core-matrix row)
__global__ void __launch_bounds__(256) k_pack_bf16x3(PackArgs a) {
  if ((a.cond && *a.cond >= a.cond_lt) || (a.skip && *a.skip)) return;
  int64_t K = (a.Kdev ? (int64_t)*a.Kdev : 0) + a.K;
  if (K > a.Q * TC_BK) K = a.Q * TC_BK;
  const int64_t q = a.q0 + blockIdx.x, t = blockIdx.y;
  if (q * TC_BK >= K) return;
  uint16_t* hi = reinterpret_cast<uint16_t*>(a.P + ((a.t0 + t) * a.Q + q) * TC_BLOCK);
  uint16_t* lo = hi + TcFmt<TC_BF16>::PART_BYTES / 2;
#pragma unroll
  for (int e = 0; e < (TC_BM * TC_BK / 8) / 256; ++e) {
    const int idx = threadIdx.x + 256 * e;
    const int r = idx % TC_BM, kq = idx / TC_BM;
    const int64_t row = t * TC_BM + r;
    uint32_t hw[4], lw[4];
#pragma unroll
    for (int c = 0; c < 8; c += 2) {
      uint16_t h2[2], l2[2];
#pragma unroll
      for (int u = 0; u < 2; ++u) {
        const int64_t k = q * TC_BK + kq * 8 + c + u;
        const double x = (row < a.R && k < K) ? a.X[row + k * a.ldx] : 0.0;
        h2[u] = bf16_rn((float)x);
        l2[u] = bf16_rn((float)(x - (double)bf16_to_f32(h2[u])));
      }
      hw[c / 2] = (uint32_t)h2[0] | ((uint32_t)h2[1] << 16);
      lw[c / 2] = (uint32_t)l2[0] | ((uint32_t)l2[1] << 16);
    }
    const int off = (kq * (TC_BM / 8) + (r >> 3)) * 64 + (r & 7) * 8;
    *reinterpret_cast<uint4*>(hi + off) = make_uint4(hw[0], hw[1], hw[2], hw[3]);
    *reinterpret_cast<uint4*>(lo + off) = make_uint4(lw[0], lw[1], lw[2], lw[3]);
  }
}

// ---------------------------------------------------------------- tiles
// Lower tiles in column order: column tile bx holds row tiles by >= first_row_tile(bx).
__host__ __device__ inline int64_t tc_first_row_tile(int64_t bx, int64_t r0, int64_t c0) {
  const int64_t d = c0 + TC_BN * bx - r0 - (TC_BM - 1);
  return d <= 0 ? 0 : (d + TC_BM - 1) / TC_BM;
}
__host__ __device__ inline int64_t tc_count_tiles(int64_t nr, int64_t nc, int64_t r0, int64_t c0) {
  int64_t n = 0;
  for (int64_t bx = 0; bx < nc; ++bx) {
    const int64_t f = tc_first_row_tile(bx, r0, c0);
    if (f < nr) n += nr - f;
  }
  return n;
}
__device__ inline void tc_tile(const TcArgs& a, int64_t t, int64_t& bx, int64_t& by) {
  for (bx = 0; bx < a.nc; ++bx) {
    const int64_t f = tc_first_row_tile(bx, a.r0, a.c0);
    const int64_t cnt = f < a.nr ? a.nr - f : 0;
    if (t < cnt) {
      by = f + t;
      return;
    }
    t -= cnt;
  }
  by = 0;  // not reached for t < ntiles
}

// ---------------------------------------------------------------- GEMM
// G: K chunks (of 32) per FP32 partial sum.  The tensor core accumulates in
// FP32 with truncation, so an accumulation run over K terms carries an error
// that grows about linearly with K; each run of G chunks starts from zero in
// tensor memory and is then added into FP64 accumulators held in registers
// by the epilogue warps (warp e owns 32 rows x 64 columns of the tile).
template <int G, int FMT>
__global__ void __launch_bounds__(TC_THREADS, 1) k_syrk_tc(TcArgs a) {
  using F = TcFmt<FMT>;
  constexpr int STAGES = TC_STAGES * (4 / F::EB);       // the same shared memory either way
  constexpr uint32_t STAGE_BYTES = 2 * F::BLOCK_BYTES;     // W block + L block
  extern __shared__ __align__(1024) uint8_t tc_smem[];
  __shared__ __align__(8) uint64_t bars[2 * STAGES + 5];
  __shared__ uint32_t tslot;
  __shared__ volatile int abort_flag;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if ((a.cond && *a.cond >= a.cond_lt) || (a.skip && *a.skip)) return;  // uniform over the CTA
  int64_t K = (a.Kdev ? (int64_t)*a.Kdev : 0) + a.K;
  if (K > a.Q * TC_BK) K = a.Q * TC_BK;  // never beyond the packed chunks
  if (K <= 0) return;  // nothing eliminated: C unchanged (uniform over the CTA)
  const int64_t nq = (K + TC_BK - 1) / TC_BK;
  const int64_t ngrp = (nq + G - 1) / G;  // partial sums per tile
  const uint32_t stage0 = (smem_u32(tc_smem) + 1023u) & ~1023u;
  auto full = [&](int s) { return smem_u32(&bars[s]); };
  auto empty = [&](int s) { return smem_u32(&bars[STAGES + s]); };
  auto pfull = [&](int b) { return smem_u32(&bars[2 * STAGES + b]); };
  auto pempty = [&](int b) { return smem_u32(&bars[2 * STAGES + 2 + b]); };
  const uint32_t fin = smem_u32(&bars[2 * STAGES + 4]);  // completion of every MMA issued

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tslot)),
                 "r"(TC_TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (threadIdx.x == 32) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(full(s), 1);
      mbar_init(empty(s), 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(pfull(b), 1);
      mbar_init(pempty(b), TC_EPI_WARPS);
    }
    mbar_init(fin, 1);
    abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tbase = tslot;

  if (warp == 0) {
    // ---------------- producer
    if (lane == 0) {
      int64_t g = 0, last_round[STAGES];
      for (int s = 0; s < STAGES; ++s) last_round[s] = -1;
      for (int64_t t = blockIdx.x; t < a.ntiles && !abort_flag && !a.stall; t += gridDim.x) {
        int64_t bx, by;
        tc_tile(a, t, bx, by);
        const float* A = a.Ap + by * a.Q * TC_BLOCK;
        const float* B = a.Bp + bx * a.Q * TC_BLOCK;
        for (int64_t q = 0; q < nq; ++q, ++g) {
          const int s = (int)(g % STAGES);
          const int64_t r = g / STAGES;
          if (r > 0 && !mbar_wait(empty(s), (uint32_t)((r - 1) & 1), &abort_flag, a.err)) break;
          const uint32_t dst = stage0 + (uint32_t)s * STAGE_BYTES;
          mbar_expect_tx(full(s), STAGE_BYTES);
          bulk_g2s(dst, A + q * TC_BLOCK, F::BLOCK_BYTES, full(s));
          bulk_g2s(dst + F::BLOCK_BYTES, B + q * TC_BLOCK, F::BLOCK_BYTES, full(s));
          last_round[s] = r;
        }
      }
      // the copies issued last land before the CTA's shared memory goes away
      for (int s = 0; s < STAGES; ++s) {
        if (last_round[s] < 0) continue;
        const uint64_t t0 = gtimer();
        while (!mbar_try(full(s), (uint32_t)(last_round[s] & 1)) && gtimer() - t0 < TC_TIMEOUT_NS) {
        }
      }
    }
    __syncwarp();
  } else if (warp == 1) {
    // ---------------- MMA issuer
    if (lane == 0) {
      int64_t g = 0, grp = 0;
      bool ok = true;
      for (int64_t t = blockIdx.x; t < a.ntiles && ok; t += gridDim.x) {
        for (int64_t q = 0; q < nq && ok; ++q, ++g) {
          const int b = (int)(grp & 1);
          if (q % G == 0) {
            const int64_t rb = grp >> 1;
            if (rb > 0 && !mbar_wait(pempty(b), (uint32_t)((rb - 1) & 1), &abort_flag, a.err)) {
              ok = false;
              break;
            }
            tc_fence_after();
          }
          const int s = (int)(g % STAGES);
          if (!mbar_wait(full(s), (uint32_t)((g / STAGES) & 1), &abort_flag, a.err)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t d = tbase + (uint32_t)(b * TC_BN);
          const uint32_t base = stage0 + (uint32_t)s * STAGE_BYTES;
#pragma unroll
          for (int ks = 0; ks < F::KSTEPS; ++ks) {
            const uint32_t ko = (uint32_t)ks * 2 * TC_LBO;
            const uint64_t ah = tc_desc(base + ko), al = tc_desc(base + F::PART_BYTES + ko);
            const uint64_t bh = tc_desc(base + F::BLOCK_BYTES + ko), bl = tc_desc(base + F::BLOCK_BYTES + F::PART_BYTES + ko);
            tc_mma<FMT>(d, al, bh, (q % G > 0 || ks > 0) ? 1u : 0u);
            tc_mma<FMT>(d, ah, bl, 1u);
            tc_mma<FMT>(d, ah, bh, 1u);
          }
          tc_commit(empty(s));  // the stage is free once these MMAs have read it
          if (q % G == G - 1 || q == nq - 1) {
            tc_commit(pfull(b));  // the partial sum is complete
            ++grp;
          }
        }
      }
      // every MMA issued has completed before tensor memory is freed
      tc_commit(fin);
      const uint64_t t0 = gtimer();
      while (!mbar_try(fin, 0) && gtimer() - t0 < TC_TIMEOUT_NS) {
      }
    }
    __syncwarp();
  } else {
    // ---------------- epilogue
    const int e = warp - 2;
    const int qd = warp & 3, ch = e >> 2;  // lane quarter, column half
    const int64_t rl = 32 * qd + lane;
    int64_t grp = 0;
    bool ok = true;
    for (int64_t t = blockIdx.x; t < a.ntiles && ok; t += gridDim.x) {
      double acc[64];
#pragma unroll
      for (int c = 0; c < 64; ++c) acc[c] = 0.0;
      for (int64_t gi = 0; gi < ngrp; ++gi, ++grp) {
        const int b = (int)(grp & 1);
        int w = 1;
        if (lane == 0) w = mbar_wait(pfull(b), (uint32_t)((grp >> 1) & 1), &abort_flag, a.err) ? 1 : 0;
        ok = __shfl_sync(0xffffffffu, w, 0) != 0;
        if (!ok) break;
        tc_fence_after();
#pragma unroll
        for (int h = 0; h < 4; ++h) {
          uint32_t v[16];
          tc_ld16(tbase + ((uint32_t)(32 * qd) << 16) + (uint32_t)(b * TC_BN + ch * 64 + h * 16), v);
#pragma unroll
          for (int c = 0; c < 16; ++c) acc[h * 16 + c] += (double)__uint_as_float(v[c]);
        }
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(pempty(b));
      }
      if (!ok) break;
      int64_t bx, by;
      tc_tile(a, t, bx, by);
      const int64_t i = a.r0 + by * TC_BM + rl;
      const int64_t jb = a.c0 + bx * TC_BN + ch * 64;
      if (i < a.r1) {
        double* col = a.C + i + jb * a.ldc;
#pragma unroll
        for (int c0 = 0; c0 < 64; c0 += 16) {
          double cv[16];
#pragma unroll
          for (int c = 0; c < 16; ++c) {
            const int64_t j = jb + c0 + c;
            cv[c] = (j < a.c1 && i >= j) ? col[(c0 + c) * a.ldc] : 0.0;
          }
#pragma unroll
          for (int c = 0; c < 16; ++c) {
            const int64_t j = jb + c0 + c;
            if (j < a.c1 && i >= j) col[(c0 + c) * a.ldc] = cv[c] - acc[c0 + c];
          }
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase), "r"(TC_TMEM_COLS) : "memory");
}

// ---------------------------------------------------------------- GEMM, column-tile pairs
// The one-partial-sum form (no flush) with two 128-column output tiles per CTA
// tile: both read the same 128-row W tile from shared memory, so a CTA brings
// in 3 operand tiles per 2 output tiles instead of 4 (the update is bound by
// the operand stream out of L2).  A stage holds 8 KB of each part of the W
// tile and of both L tiles (16 deep in TF32, a whole 32-deep chunk in BF16:
// 48 KB, six cp.async.bulk copies), four stages; tensor memory holds two 256-column
// accumulators (tile 0 at columns [0, 128), tile 1 at [128, 256) of each).
// Each output tile gets the same MMA sequence as in k_syrk_tc (per k-step
// lo*hi, hi*lo, hi*hi, k-steps in order), and the epilogue does
// C - (0 + partial) in FP64 like k_syrk_tc's one-group case, so the two
// kernels give bit-identical results.  Epilogue warp e takes tile e / 4 of the
// pair and its 32-row lane quarter, 16 columns at a time (tensor memory read,
// then the C read-modify-write), and frees the accumulator after the tile.
constexpr int TP_STAGES = 4;
constexpr uint32_t TP_HALF_BYTES = 8192;                  // a stage's slice of one part
constexpr uint32_t TP_OPND_BYTES = 2 * TP_HALF_BYTES;    // hi + lo halves of one operand tile
constexpr uint32_t TP_STAGE_BYTES = 3 * TP_OPND_BYTES;   // W tile + two L tiles: 48 KB
constexpr size_t TP_SMEM = (size_t)TP_STAGES * TP_STAGE_BYTES + 1024 + 32768;
constexpr uint32_t TP_TMEM_COLS = 512;

// lower column-tile pairs (px: column tiles 2 px and 2 px + 1) in column order
__host__ __device__ inline int64_t tp_count_tiles(int64_t nr, int64_t nc, int64_t r0, int64_t c0) {
  int64_t n = 0;
  for (int64_t px = 0; 2 * px < nc; ++px) {
    const int64_t f = tc_first_row_tile(2 * px, r0, c0);
    if (f < nr) n += nr - f;
  }
  return n;
}
// Tile t of the pair kernel.  The column pairs go TP_GROUP at a time; inside a
// group the row tiles go in order and, for each row tile, the group's pairs
// whose lower part reaches it.  The CTAs working at the same time then share
// a few row tiles of W and the group's L tiles (a few MB, resident in L2),
// where walking one column pair at a time streamed every row tile of W once
// per pair (~240 MB per pair on a 59k-row front, more than the L2 holds).
// Every tile is computed the same way in any order.
constexpr int TP_GROUP = 8;
__host__ __device__ inline void tp_tile_at(int64_t nr, int64_t nc, int64_t r0, int64_t c0, int64_t t, int64_t& px,
                                           int64_t& by) {
  const int64_t np = (nc + 1) / 2;
  for (int64_t p0 = 0; p0 < np; p0 += TP_GROUP) {
    const int g = (int)(np - p0 < TP_GROUP ? np - p0 : TP_GROUP);
    int64_t f[TP_GROUP];  // first row tile of each pair of the group, at most nr (non-decreasing)
    int64_t cnt = 0;
    for (int j = 0; j < g; ++j) {
      const int64_t fj = tc_first_row_tile(2 * (p0 + j), r0, c0);
      f[j] = fj < nr ? fj : nr;
      cnt += nr - f[j];
    }
    if (t >= cnt) {
      t -= cnt;
      continue;
    }
    // rows [f[0], f[g-1]): the pairs j with f[j] <= row, in order of j
    int v = 0;
    for (int64_t b = f[0]; b < f[g - 1]; ++b) {
      while (v < g && f[v] <= b) ++v;  // pairs 0 .. v - 1 reach row b
      if (t < v) {
        px = p0 + t;
        by = b;
        return;
      }
      t -= v;
    }
    // rows from f[g-1]: all g pairs
    by = f[g - 1] + t / g;
    px = p0 + t % g;
    return;
  }
  px = 0;  // not reached for t < ntiles
  by = 0;
}
__device__ inline void tp_tile(const TcArgs& a, int64_t t, int64_t& px, int64_t& by) {
  tp_tile_at(a.nr, a.nc, a.r0, a.c0, t, px, by);
}

template <int FMT>
__global__ void __launch_bounds__(TC_THREADS, 1) k_syrk_tc_pair(TcArgs a) {
  using F = TcFmt<FMT>;
  constexpr int SK = 64 / F::EB;                 // K per stage: 16 (TF32) or 32 (BF16), 8 KB per part either way
  constexpr int SPC = TC_BK / SK;                // stages per packed chunk
  static_assert(TC_BM * SK * F::EB == (int)TP_HALF_BYTES, "a stage part is 8 KB");
  extern __shared__ __align__(1024) uint8_t tc_smem[];
  __shared__ __align__(8) uint64_t bars[2 * TP_STAGES + 5];
  __shared__ uint32_t tslot;
  __shared__ volatile int abort_flag;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if ((a.cond && *a.cond >= a.cond_lt) || (a.skip && *a.skip)) return;  // uniform over the CTA
  int64_t K = (a.Kdev ? (int64_t)*a.Kdev : 0) + a.K;
  if (K > a.Q * TC_BK) K = a.Q * TC_BK;  // never beyond the packed chunks
  if (K <= 0) return;
  const int64_t nh = (K + SK - 1) / SK;  // stages of SK
  const uint32_t stage0 = (smem_u32(tc_smem) + 1023u) & ~1023u;
  auto full = [&](int s) { return smem_u32(&bars[s]); };
  auto empty = [&](int s) { return smem_u32(&bars[TP_STAGES + s]); };
  auto pfull = [&](int b) { return smem_u32(&bars[2 * TP_STAGES + b]); };
  auto pempty = [&](int b) { return smem_u32(&bars[2 * TP_STAGES + 2 + b]); };
  const uint32_t fin = smem_u32(&bars[2 * TP_STAGES + 4]);

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tslot)),
                 "r"(TP_TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (threadIdx.x == 32) {
    for (int s = 0; s < TP_STAGES; ++s) {
      mbar_init(full(s), 1);
      mbar_init(empty(s), 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(pfull(b), 1);
      mbar_init(pempty(b), TC_EPI_WARPS);
    }
    mbar_init(fin, 1);
    abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tbase = tslot;

  if (warp == 0) {
    // ---------------- producer
    if (lane == 0) {
      int64_t g = 0, last_round[TP_STAGES];
      for (int s = 0; s < TP_STAGES; ++s) last_round[s] = -1;
      for (int64_t t = blockIdx.x; t < a.ntiles && !abort_flag && !a.stall; t += gridDim.x) {
        int64_t px, by;
        tp_tile(a, t, px, by);
        const bool two = 2 * px + 1 < a.nc;
        const float* A = a.Ap + by * a.Q * TC_BLOCK;
        const float* B0 = a.Bp + 2 * px * a.Q * TC_BLOCK;
        const float* B1 = B0 + a.Q * TC_BLOCK;
        for (int64_t h = 0; h < nh; ++h, ++g) {
          const int s = (int)(g % TP_STAGES);
          const int64_t r = g / TP_STAGES;
          if (r > 0 && !mbar_wait(empty(s), (uint32_t)((r - 1) & 1), &abort_flag, a.err)) break;
          const uint32_t dst = stage0 + (uint32_t)s * TP_STAGE_BYTES;
          // the stage's slice of the hi part (at +0) and of the lo part (at +PART_BYTES) of the block
          constexpr int64_t PF = F::PART_BYTES / 4;  // a part, in floats
          const int64_t off = (h / SPC) * TC_BLOCK + (h % SPC) * (TP_HALF_BYTES / 4);
          mbar_expect_tx(full(s), (two ? 3u : 2u) * TP_OPND_BYTES);
          bulk_g2s(dst, A + off, TP_HALF_BYTES, full(s));
          bulk_g2s(dst + TP_HALF_BYTES, A + off + PF, TP_HALF_BYTES, full(s));
          bulk_g2s(dst + TP_OPND_BYTES, B0 + off, TP_HALF_BYTES, full(s));
          bulk_g2s(dst + TP_OPND_BYTES + TP_HALF_BYTES, B0 + off + PF, TP_HALF_BYTES, full(s));
          if (two) {
            bulk_g2s(dst + 2 * TP_OPND_BYTES, B1 + off, TP_HALF_BYTES, full(s));
            bulk_g2s(dst + 2 * TP_OPND_BYTES + TP_HALF_BYTES, B1 + off + PF, TP_HALF_BYTES, full(s));
          }
          last_round[s] = r;
        }
      }
      for (int s = 0; s < TP_STAGES; ++s) {
        if (last_round[s] < 0) continue;
        const uint64_t t0 = gtimer();
        while (!mbar_try(full(s), (uint32_t)(last_round[s] & 1)) && gtimer() - t0 < TC_TIMEOUT_NS) {
        }
      }
    }
    __syncwarp();
  } else if (warp == 1) {
    // ---------------- MMA issuer
    if (lane == 0) {
      int64_t g = 0, grp = 0;
      bool ok = true;
      for (int64_t t = blockIdx.x; t < a.ntiles && ok; t += gridDim.x, ++grp) {
        int64_t px, by;
        tp_tile(a, t, px, by);
        const bool two = 2 * px + 1 < a.nc;
        const int b = (int)(grp & 1);
        const int64_t rb = grp >> 1;
        if (rb > 0 && !mbar_wait(pempty(b), (uint32_t)((rb - 1) & 1), &abort_flag, a.err)) break;
        tc_fence_after();
        const uint32_t d0 = tbase + (uint32_t)(b * 2 * TC_BN), d1 = d0 + TC_BN;
        for (int64_t h = 0; h < nh; ++h, ++g) {
          const int s = (int)(g % TP_STAGES);
          if (!mbar_wait(full(s), (uint32_t)((g / TP_STAGES) & 1), &abort_flag, a.err)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t base = stage0 + (uint32_t)s * TP_STAGE_BYTES;
#pragma unroll
          for (int ks = 0; ks < 2; ++ks) {  // 32 bytes of K per MMA, 64 per stage
            const uint32_t ko = (uint32_t)ks * 2 * TC_LBO;
            const uint64_t ah = tc_desc(base + ko), al = tc_desc(base + TP_HALF_BYTES + ko);
            const uint32_t b0 = base + TP_OPND_BYTES, b1 = base + 2 * TP_OPND_BYTES;
            const uint32_t acc = (h > 0 || ks > 0) ? 1u : 0u;
            tc_mma<FMT>(d0, al, tc_desc(b0 + ko), acc);
            tc_mma<FMT>(d0, ah, tc_desc(b0 + TP_HALF_BYTES + ko), 1u);
            tc_mma<FMT>(d0, ah, tc_desc(b0 + ko), 1u);
            if (two) {
              tc_mma<FMT>(d1, al, tc_desc(b1 + ko), acc);
              tc_mma<FMT>(d1, ah, tc_desc(b1 + TP_HALF_BYTES + ko), 1u);
              tc_mma<FMT>(d1, ah, tc_desc(b1 + ko), 1u);
            }
          }
          tc_commit(empty(s));
        }
        if (!ok) break;
        tc_commit(pfull(b));
      }
      tc_commit(fin);
      const uint64_t t0 = gtimer();
      while (!mbar_try(fin, 0) && gtimer() - t0 < TC_TIMEOUT_NS) {
      }
    }
    __syncwarp();
  } else {
    // ---------------- epilogue
    const int e = warp - 2;
    const int qd = warp & 3, ch = e >> 2;  // lane quarter, tile of the pair
    const int64_t rl = 32 * qd + lane;
    int64_t grp = 0;
    for (int64_t t = blockIdx.x; t < a.ntiles; t += gridDim.x, ++grp) {
      const int b = (int)(grp & 1);
      int w = 1;
      if (lane == 0) w = mbar_wait(pfull(b), (uint32_t)((grp >> 1) & 1), &abort_flag, a.err) ? 1 : 0;
      if (__shfl_sync(0xffffffffu, w, 0) == 0) break;
      tc_fence_after();
      int64_t px, by;
      tp_tile(a, t, px, by);
      const int64_t i = a.r0 + by * TC_BM + rl;
      const int64_t jb = a.c0 + (2 * px + ch) * TC_BN;
      if (2 * px + ch < a.nc) {
        double* col = a.C + i + jb * a.ldc;
        for (int c0 = 0; c0 < TC_BN; c0 += 16) {
          uint32_t v[16];
          tc_ld16(tbase + ((uint32_t)(32 * qd) << 16) + (uint32_t)(b * 2 * TC_BN + ch * TC_BN + c0), v);
          if (i < a.r1) {
            double cv[16];
#pragma unroll
            for (int c = 0; c < 16; ++c) {
              const int64_t j = jb + c0 + c;
              cv[c] = (j < a.c1 && i >= j) ? col[(int64_t)(c0 + c) * a.ldc] : 0.0;
            }
#pragma unroll
            for (int c = 0; c < 16; ++c) {
              const int64_t j = jb + c0 + c;
              if (j < a.c1 && i >= j) col[(int64_t)(c0 + c) * a.ldc] = cv[c] - (0.0 + (double)__uint_as_float(v[c]));
            }
          }
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(pempty(b));
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase), "r"(TP_TMEM_COLS) : "memory");
}

}  // namespace rvg
