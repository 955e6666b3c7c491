// Supernodal solve (aptp_solve, sparse/src/symmetric/solve.rs:57-326) as one
// launch per wave and direction: forward_solve_supernode (solve.rs:161-230)
// with the diagonal solve (solve.rs:232-252) folded into the backward pass,
// and backward_solve_supernode (solve.rs:254-326).
//
// Every front of the wave is cut into 64-row blocks; CTAs take blocks in
// ticket order from one atomic counter (front by front, and inside a front in
// dependency order), so a block only ever waits for blocks with a smaller
// ticket, which are held by CTAs that are already running: no deadlock, and
// no co-residency assumption beyond that.  Waits are bounded by the global
// timer; one that runs out sets *err and the solve goes on (the caller gets
// RVG_ERR_DEVICE_TIMEOUT).
//
// forward, per front (y kept in the front's work vector v, rows < ne):
//   diagonal block r (rows [64r, 64r + 64) of L11): y = x[col] - sum over the
//     finished column blocks b < r of L[rows, b] y_b (each as soon as its flag
//     is up), then the unit lower solve of the 64 x 64 diagonal block by one
//     warp; publish y_r, raise flag r;
//   L21 block (rows >= ne): -sum over all column blocks of L[rows, b] y_b,
//     added atomically into x at the parent's rows (siblings share rows).
// backward, per front, in ticket order:
//   gather tickets: the parent's final values at 64 rows of L21 into v + m
//     (rows >= ne);
//   partial-sum tickets: for a column block and a group of up to 8 L21 row
//     blocks, the sums L[rows, cols]^T x[rows] over the group, into a slot of
//     the wave's partial-sum buffer (the L21 reduction of one column block is
//     spread over CTAs, as the forward pass spreads its rows);
//   column blocks, descending (x_final in v + m): z = D^-1 y on the block's
//     columns (2x2 pairs may straddle blocks: y is still intact in v), minus
//     the block's partial sums in group order, minus L[rows of later blocks,
//     cols]^T x_final of those blocks (each once its flag is up), then the
//     unit upper solve (L11^T) of the diagonal block by one warp;
//     x[col] = x_final; raise the flag.
// Per row (forward) and per column (backward) the sums run in ascending
// column / row order inside each 64-block.  Up to 8 right-hand sides go
// through one launch (template R), each L value read once for all of them.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "front.cuh"

namespace rvg {

constexpr int SF_B = 64;                            // block rows / columns
constexpr uint64_t SF_TIMEOUT_NS = 1000000000ull;   // 1 s per wait

// one front of a wave: its first ticket and its block counts
constexpr int SF_PG = 8;  // backward: L21 row blocks per partial-sum ticket (512 rows)
constexpr int SF_BWD_DYN = SF_B * (SF_B + 1) * 8;  // k_sf_bwd's dynamic shared memory

struct SfFront {
  int32_t s;      // supernode
  int32_t blk0;   // first ticket of the front
  int32_t nbd;    // diagonal blocks (ceil(ne / 64))
  int32_t nbr;    // L21 blocks (ceil((m - ne) / 64)): forward row blocks, backward gather tickets
  int32_t ngrp;   // backward: partial-sum tickets per column block (ceil(nbr / SF_PG))
  int32_t pslot;  // backward: the front's first partial-sum slot (R x 64 values each)
};

struct SfWave {
  const SfFront* fr;
  double* part;     // backward partial sums: slot q at part + q R 64
  int32_t nfr, nblk;
  int32_t* ticket;  // zeroed before the launch
  int32_t* flags;   // nblk entries, zeroed before the launch
  double* x;        // solution vectors, permuted order: right-hand side r at x + r ldx
  int64_t ldx;
  double* work;     // per-front work at DFront::scratch: y (R x m) then x_final (R x m)
  int32_t* err;
};

__device__ __forceinline__ int32_t sf_ld_acquire(const int32_t* p) {
  int32_t v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void sf_st_release(int32_t* p, int32_t v) {
  asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ uint64_t sf_timer() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// bounded wait for a published block (thread 0 of the CTA)
__device__ __forceinline__ void sf_wait(const int32_t* flag, int32_t* err) {
  if (sf_ld_acquire(flag)) return;
  const uint64_t t0 = sf_timer();
  while (!sf_ld_acquire(flag)) {
    if (sf_timer() - t0 > SF_TIMEOUT_NS) {
      atomicExch(err, 2);
      return;
    }
  }
}

// the wave's front holding ticket blk (last front with blk0 <= blk)
__device__ __forceinline__ int sf_front(const SfWave& w, int blk) {
  int lo = 0, hi = w.nfr - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (w.fr[mid].blk0 <= blk) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

__device__ __forceinline__ int32_t sf_col(const int32_t* rows, const int32_t* perm, int64_t i) { return rows[perm[i]]; }
__device__ __forceinline__ int32_t sf_row(const int32_t* rows, const int32_t* perm, int64_t ne, int64_t k,
                                          int64_t t) {
  const int64_t q = ne + t;
  return q < k ? rows[perm[q]] : rows[q];
}

// One row of a 64-column strip (columns at stride m) into dst[0, nc), 16
// loads in flight per thread (the loads are independent; issuing them before
// the first use keeps the row's memory latency from serialising).
__device__ __forceinline__ void sf_load_strip(const double* src, int64_t m, int nc, double* dst) {
#pragma unroll
  for (int c0 = 0; c0 < SF_B; c0 += 16) {
    double r[16];
#pragma unroll
    for (int u = 0; u < 16; ++u) r[u] = c0 + u < nc ? __ldg(src + (int64_t)(c0 + u) * m) : 0.0;
#pragma unroll
    for (int u = 0; u < 16; ++u) dst[c0 + u] = r[u];
  }
}

// R right-hand sides at once: every L value read is used R times.
template <int R>
__global__ void __launch_bounds__(SF_B) k_sf_fwd(SfWave w, const DFront* F, Arenas A) {
  __shared__ int s_blk;
  __shared__ double yb[R][SF_B];
  __shared__ double Ls[SF_B][SF_B + 1];
  const int t = threadIdx.x;
  for (;;) {
    if (t == 0) s_blk = atomicAdd(w.ticket, 1);
    __syncthreads();
    const int blk = s_blk;
    __syncthreads();
    if (blk >= w.nblk) break;
    const SfFront sf = w.fr[sf_front(w, blk)];
    const DFront fr = F[sf.s];
    const int64_t m = fr.m, ne = fr.ne;
    const double* L = A.panel + fr.panel;
    const int32_t* rows = A.idx + fr.idx;
    const int32_t* perm = rows + m;
    double* v = w.work + fr.scratch;  // y of right-hand side r at v + r m
    int32_t* flags = w.flags + sf.blk0;
    const int b = blk - sf.blk0;
    const bool diag = b < sf.nbd;
    const int64_t r0 = diag ? (int64_t)b * SF_B : ne + (int64_t)(b - sf.nbd) * SF_B;
    const int64_t r1 = diag ? (r0 + SF_B < ne ? r0 + SF_B : ne) : (r0 + SF_B < m ? r0 + SF_B : m);
    const int64_t i = r0 + t;
    const bool row = i < r1;
    double acc[R];
    if (diag && row) {
      const int32_t g = sf_col(rows, perm, i);
#pragma unroll
      for (int r = 0; r < R; ++r) acc[r] = w.x[r * w.ldx + g];
    } else {
#pragma unroll
      for (int r = 0; r < R; ++r) acc[r] = 0.0;
    }
    // The factor is final: the L strips are read before the waits on the
    // blocks they multiply, so only the y values are on the chain.
    const int nr = (int)(r1 - r0);
    if (diag && row) sf_load_strip(L + i + r0 * m, m, nr, &Ls[t][0]);  // the diagonal block, staged early
    const int ncb = diag ? b : sf.nbd;
    for (int cb = 0; cb < ncb; ++cb) {
      const int64_t c0 = (int64_t)cb * SF_B;
      const int nc = (int)((c0 + SF_B < ne ? c0 + SF_B : ne) - c0);
      double lr[SF_B];
      if (row) sf_load_strip(L + i + c0 * m, m, nc, lr);
      if (t == 0) sf_wait(&flags[cb], w.err);
      __syncthreads();
      if (t < nc) {
#pragma unroll
        for (int r = 0; r < R; ++r) yb[r][t] = __ldcg(&v[r * m + c0 + t]);
      }
      __syncthreads();
      if (row) {
#pragma unroll
        for (int c = 0; c < SF_B; ++c)
          if (c < nc) {
#pragma unroll
            for (int r = 0; r < R; ++r) acc[r] = __fma_rn(-lr[c], yb[r][c], acc[r]);
          }
      }
      __syncthreads();
    }
    if (diag) {
      // unit lower solve of rows [r0, r1) by warp 0 (lane: rows r0 + lane, r0 + 32 + lane),
      // on the diagonal block staged in shared memory above
#pragma unroll
      for (int r = 0; r < R; ++r) yb[r][t] = acc[r];
      __syncthreads();
      if (t < 32) {
#pragma unroll
        for (int r = 0; r < R; ++r) {
          double a0 = yb[r][t], a1 = yb[r][t + 32];
          for (int j = 0; j < nr; ++j) {
            const double yj = __shfl_sync(0xffffffffu, j < 32 ? a0 : a1, j & 31);
            if (t > j && t < nr) a0 = __fma_rn(-Ls[t][j], yj, a0);
            if (t + 32 > j && t + 32 < nr) a1 = __fma_rn(-Ls[t + 32][j], yj, a1);
          }
          if (t < nr) v[r * m + r0 + t] = a0;
          if (t + 32 < nr) v[r * m + r0 + t + 32] = a1;
        }
      }
      __threadfence();
      __syncthreads();
      if (t == 0) sf_st_release(&flags[b], 1);
    } else if (row) {
      const int32_t g = sf_row(rows, perm, ne, fr.k, i - ne);
#pragma unroll
      for (int r = 0; r < R; ++r) atomicAdd(&w.x[r * w.ldx + g], acc[r]);
    }
  }
}

// z = D^-1 y for column c of a front (MixedDiagonal::solve_in_place,
// diagonal.rs:312-360: zero pivots give 0, 2x2 blocks by Cramer's rule)
__device__ __forceinline__ double sf_dinv(const DFront& fr, const Arenas& A, const double* y, int64_t c) {
  const int8_t* dt = A.dtype + fr.dpos;
  const double* dd = A.ddiag + fr.dpos;
  const double* dof = A.doff + fr.dpos;
  if (dt[c] == PT_1X1) {
    const double d = dd[c];
    return d == 0.0 ? 0.0 : __ddiv_rn(y[c], d);
  }
  const int64_t c0 = dt[c] == PT_2X2 ? c : c - 1;
  const double a = dd[c0], b = dof[c0], cc = dd[c0 + 1];
  const double det = __dsub_rn(__dmul_rn(a, cc), __dmul_rn(b, b));
  const double r1 = y[c0], r2 = y[c0 + 1];
  if (det == 0.0) return 0.0;
  return c == c0 ? __ddiv_rn(__dsub_rn(__dmul_rn(cc, r1), __dmul_rn(b, r2)), det)
                 : __ddiv_rn(__dsub_rn(__dmul_rn(a, r2), __dmul_rn(b, r1)), det);
}

template <int R>
__global__ void __launch_bounds__(SF_B) k_sf_bwd(SfWave w, const DFront* F, Arenas A) {
  __shared__ int s_blk;
  __shared__ double Ls[SF_B][SF_B + 1];
  // a column block's diagonal block, staged before its waits (dynamic shared memory: SF_BWD_DYN bytes)
  extern __shared__ double sf_dyn[];
  double(*Ld)[SF_B + 1] = reinterpret_cast<double(*)[SF_B + 1]>(sf_dyn);
  __shared__ double xs[R][SF_B];
  const int t = threadIdx.x;
  for (;;) {
    if (t == 0) s_blk = atomicAdd(w.ticket, 1);
    __syncthreads();
    const int blk = s_blk;
    __syncthreads();
    if (blk >= w.nblk) break;
    const SfFront sf = w.fr[sf_front(w, blk)];
    const DFront fr = F[sf.s];
    const int64_t m = fr.m, ne = fr.ne;
    const double* L = A.panel + fr.panel;
    const int32_t* rows = A.idx + fr.idx;
    const int32_t* perm = rows + m;
    const double* y = w.work + fr.scratch;      // forward results of right-hand side r at y + r m
    double* xf = w.work + fr.scratch + R * m;   // final values of this front's columns, at xf + r m
    int32_t* flags = w.flags + sf.blk0;
    const int nbr = sf.nbr, ngrp = sf.ngrp;
    const int lt = blk - sf.blk0;  // ticket within the front
    const int npart = sf.nbd * ngrp;
    if (lt < nbr) {
      // gather ticket: the parent's final values at 64 rows of L21 into xf
      const int64_t i = ne + (int64_t)lt * SF_B + t;
      if (i < m) {
        const int32_t g = sf_row(rows, perm, ne, fr.k, i - ne);
#pragma unroll
        for (int r = 0; r < R; ++r) xf[r * m + i] = w.x[r * w.ldx + g];
      }
      __threadfence();
      __syncthreads();
      if (t == 0) sf_st_release(&flags[lt], 1);
      continue;
    }
    if (lt < nbr + npart) {
      // partial-sum ticket (column blocks descending, groups ascending)
      const int pq = lt - nbr;
      const int b = sf.nbd - 1 - pq / ngrp, gi = pq % ngrp;
      const int64_t c0 = (int64_t)b * SF_B;
      const int nc = (int)((c0 + SF_B < ne ? c0 + SF_B : ne) - c0);
      double ps[R];
#pragma unroll
      for (int r = 0; r < R; ++r) ps[r] = 0.0;
      const int rb1 = (gi + 1) * SF_PG < nbr ? (gi + 1) * SF_PG : nbr;
      for (int rb = gi * SF_PG; rb < rb1; ++rb) {
        if (t == 0) sf_wait(&flags[rb], w.err);
        const int64_t i0 = ne + (int64_t)rb * SF_B;
        const int nr = (int)((i0 + SF_B < m ? i0 + SF_B : m) - i0);
        __syncthreads();
        if (t < nr) {
#pragma unroll
          for (int r = 0; r < R; ++r) xs[r][t] = __ldcg(&xf[r * m + i0 + t]);
          sf_load_strip(L + i0 + t + c0 * m, m, nc, &Ls[t][0]);
        }
        __syncthreads();
        if (t < nc)
          for (int rr = 0; rr < nr; ++rr) {
            const double l = Ls[rr][t];
#pragma unroll
            for (int r = 0; r < R; ++r) ps[r] = __fma_rn(l, xs[r][rr], ps[r]);
          }
      }
      double* slot = w.part + ((int64_t)sf.pslot + pq) * R * SF_B;
#pragma unroll
      for (int r = 0; r < R; ++r) slot[r * SF_B + t] = ps[r];
      __threadfence();
      __syncthreads();
      if (t == 0) sf_st_release(&flags[lt], 1);
      continue;
    }
    const int q = lt - nbr - npart;  // column blocks, descending
    const int b = sf.nbd - 1 - q;
    const int64_t c0 = (int64_t)b * SF_B;
    const int nc = (int)((c0 + SF_B < ne ? c0 + SF_B : ne) - c0);
    const bool col = t < nc;
    if (col) sf_load_strip(L + (c0 + t) + c0 * m, m, nc, &Ld[t][0]);  // Ld[row][col]; the factor is final
    double acc[R];
#pragma unroll
    for (int r = 0; r < R; ++r) acc[r] = col ? sf_dinv(fr, A, y + r * m, c0 + t) : 0.0;
    // the block's L21 partial sums, in group order
    for (int gi = 0; gi < ngrp; ++gi) {
      const int pq = q * ngrp + gi;
      if (t == 0) sf_wait(&flags[nbr + pq], w.err);
      __syncthreads();
      const double* slot = w.part + ((int64_t)sf.pslot + pq) * R * SF_B;
#pragma unroll
      for (int r = 0; r < R; ++r) acc[r] = __dsub_rn(acc[r], __ldcg(&slot[r * SF_B + t]));
    }
    // rows of later diagonal blocks, from the last one down, as they finish
    const int cb0 = nbr + npart;  // flag of column block q' at flags[cb0 + q']
    for (int rblk = sf.nbd - 1; rblk > b; --rblk) {
      const int64_t i0 = (int64_t)rblk * SF_B;
      const int nr = (int)((i0 + SF_B < ne ? i0 + SF_B : ne) - i0);
      double lr[SF_B];  // the strip, read before the wait on its block
      if (t < nr) sf_load_strip(L + i0 + t + c0 * m, m, nc, lr);
      if (t == 0) sf_wait(&flags[cb0 + (sf.nbd - 1 - rblk)], w.err);
      __syncthreads();
      if (t < nr) {
#pragma unroll
        for (int r = 0; r < R; ++r) xs[r][t] = __ldcg(&xf[r * m + i0 + t]);
#pragma unroll
        for (int c = 0; c < SF_B; ++c) Ls[t][c] = lr[c];
      }
      __syncthreads();
      if (col)
        for (int rr = 0; rr < nr; ++rr) {
          const double l = Ls[rr][t];
#pragma unroll
          for (int r = 0; r < R; ++r) acc[r] = __fma_rn(-l, xs[r][rr], acc[r]);
        }
    }
    // the diagonal block: x_c = acc_c - sum_{c < i < c0 + nc} L(i, c) x_i, from the bottom
    __syncthreads();
#pragma unroll
    for (int r = 0; r < R; ++r) xs[r][t] = acc[r];
    __syncthreads();
    if (t < 32) {
#pragma unroll
      for (int r = 0; r < R; ++r) {
        double a0 = xs[r][t], a1 = xs[r][t + 32];
        for (int j = nc - 1; j >= 0; --j) {
          const double xj = __shfl_sync(0xffffffffu, j < 32 ? a0 : a1, j & 31);
          if (t < j) a0 = __fma_rn(-Ld[j][t], xj, a0);
          if (t + 32 < j) a1 = __fma_rn(-Ld[j][t + 32], xj, a1);
        }
        if (t < nc) {
          xf[r * m + c0 + t] = a0;
          w.x[r * w.ldx + sf_col(rows, perm, c0 + t)] = a0;
        }
        if (t + 32 < nc) {
          xf[r * m + c0 + t + 32] = a1;
          w.x[r * w.ldx + sf_col(rows, perm, c0 + t + 32)] = a1;
        }
      }
    }
    __threadfence();
    __syncthreads();
    if (t == 0) sf_st_release(&flags[blk - sf.blk0], 1);
  }
}

}  // namespace rvg
