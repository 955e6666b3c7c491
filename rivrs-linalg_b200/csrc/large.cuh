// Multi-kernel APTP for one large front (front order >= the large-front
// threshold): the same algorithm as the CTA kernel (factor_inner,
// factor.rs:1811-2095; two_level_factor, factor.rs:2108-2252) with every
// row-parallel step spread over the whole GPU and the pivot state kept on the
// device, so the host issues a fixed launch sequence:
//
//   per 32-column inner block (view-local position k):
//     lf_block   1 CTA    the previous inner block's delayed columns to the
//                         end of the outer block (lf_delay_cta), complete
//                         pivoting on the diagonal block, row permutation of
//                         the outer block's earlier columns
//     lf_panel   grid     backup, column permutation, TRSM, D^-1 scaling and
//                         the a-posteriori threshold scan of every panel row
//     lf_wi      grid     CTA 0 first (lf_post_cta): 2x2 boundary adjustment,
//                         restore of the failed part of the diagonal block,
//                         failed x failed cross term, D entries; then every
//                         CTA: restore of the failed panel columns, W = L D,
//                         the trailing x failed cross term
//     k_syrk_dmma         rank-nelim update of the outer block's trailing
//                         columns (region start read from the device)
//   after the last inner block:
//     lf_delay   1 CTA    its delayed columns to the end of the outer block
//   per 256-column outer block:
//     lf_prop    grid     row permutation of the front's earlier columns
//     lf_w       grid     W = L D for the rows below the outer block, into
//                         the window of pending columns
//     Schur GEMM          the deferred update (update_trailing), split in
//                         two: the next outer block's columns take every
//                         pending column at once (near field); the columns
//                         after it (far field) only when the window is full
//                         (LF_WINDOW outer blocks, mixed_window in the mixed
//                         form) or when this block delayed
//                         a column (decided on the device), so each far-field
//                         entry is read and written once per window instead
//                         of once per block.  Each entry still takes one fma
//                         chain over the eliminated columns in order, so the
//                         result is bit-identical to the per-block update.
//     lf_outer   1 CTA    column order, delays to the end of the remaining
//                         fully-summed columns
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "dense.cuh"

namespace rvg {

struct LFState {
  int32_t k, end_pos, bs, bnelim, eff, nelim;
  int32_t gne, n1, n2, bne;
  // set when an outer block was launched for another start column than the
  // device reached (the host issues blocks ahead assuming no delays): every
  // later launch of the front returns at once until the host clears it
  int32_t spec_bad;
  int32_t bperm[32];
  int8_t bdt[32];
  double bdd[32], bdo[32];
  double T[32][33];   // factored block, 2x2 off-diagonals zeroed (the L11 of the TRSM)
  double Tb[32][33];  // the block before factorization
};

struct LFArgs {
  double* a;        // front panel (m x p), ld m
  int64_t m, p;
  int32_t* perm;    // front pivot order (p)
  DRec D;           // front D (p)
  LFState* st;
  int32_t* lp;      // outer-block local column order (nb)
  double* pb;       // panel backup, rows x 32 (ld = bm)
  double* w;        // inner W, rows x 32 (column-major, ld = rows of the view)
  double* wo;       // pending W (column-major, ld wld): row i, pending column c at wo[(i - wrow0) + c * wld]
  int64_t wld, wrow0, wcol0;  // leading dimension, first row, this block's first pending column
  int64_t cs, bcols, nfsb;  // outer block start, width, NFS boundary (global p)
  DevOpts o;
};

__global__ void k_lf_init(LFState* st, int32_t* perm, int64_t p) {
  if (blockIdx.x == 0 && threadIdx.x == 0) { st->gne = 0; st->n1 = 0; st->n2 = 0; st->spec_bad = 0; }
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < p; i += (int64_t)gridDim.x * blockDim.x)
    perm[i] = (int32_t)i;
}

__global__ void k_lf_begin_outer(LFArgs A) {
  chain_enter();
  LFState* st = A.st;
  if (st->spec_bad) return;
  if (st->gne != (int32_t)A.cs) {  // issued for a start column the factorization did not reach
    __syncthreads();               // every thread has read gne before it is flagged
    if (threadIdx.x == 0) st->spec_bad = 1;
    return;
  }
  if (threadIdx.x == 0) { st->k = 0; st->end_pos = (int32_t)A.bcols; st->bne = 0; }
  for (int i = threadIdx.x; i < A.bcols; i += blockDim.x) A.lp[i] = i;
}

__device__ void lf_delay_cta(const LFArgs& A);

// complete pivoting on the diagonal block (1 CTA); with after_delay set it
// first moves the previous inner block's delayed columns to the end of the
// outer block (lf_delay_cta, that block's last step)
__global__ void __launch_bounds__(NT) k_lf_block(LFArgs A, int after_delay) {
  chain_enter();
  if (A.st->spec_bad) return;  // a block issued past a mispredicted start column
  if (after_delay) {
    lf_delay_cta(A);
    __syncthreads();
  }
  __shared__ CtaShared sh;
  LFState* st = A.st;
  const int tid = threadIdx.x;
  const int64_t cs = A.cs;
  PanelView V{A.a + cs + cs * A.m, A.m};
  const int k = st->k, end_pos = st->end_pos;
  const int bs = min(end_pos - k, A.o.ib);
  if (k >= end_pos) {  // no columns left in this outer block
    if (tid == 0) { st->bs = 0; st->bnelim = 0; st->eff = 0; st->nelim = 0; }
    return;
  }
  {
    // the block's loads before any global store (4 per thread)
    constexpr int PER = IBMAX * IBMAX / NT;
    double v[PER];
#pragma unroll
    for (int u = 0; u < PER; ++u) {
      const int t = tid + u * NT, i = t % IBMAX, j = t / IBMAX;
      v[u] = (i < bs && j < bs && i >= j) ? V(k + i, k + j) : 0.0;
    }
#pragma unroll
    for (int u = 0; u < PER; ++u) {
      const int t = tid + u * NT, i = t % IBMAX, j = t / IBMAX;
      if (i < bs && j < bs && i >= j) { sh.T[i][j] = v[u]; st->Tb[i][j] = v[u]; }
    }
  }
  __syncthreads();
  cta_block_factor(sh, bs, A.o.small);
  const int bnelim = sh.bnelim;
  if (bnelim > 0) {
    for (int t = tid; t < bs * bs; t += NT) {
      int i = t % bs, j = t / bs;
      if (i >= j) V(k + i, k + j) = sh.T[i][j];
    }
    __syncthreads();
    if (tid == 0) {
      int bc = 0;
      while (bc < bnelim) {
        if (sh.bdt[bc] == PT_2X2) { V(k + bc + 1, k + bc) = 0.0; sh.T[bc + 1][bc] = 0.0; bc += 2; }
        else bc += 1;
      }
    }
    // (the row permutation of the view columns 0..k, step 5, is done by k_lf_panel's threads c < k)
    if (tid < 32) {  // column order (step 6): lane i takes the entry of lane bperm[i]
      const int32_t ob = tid < bs ? A.lp[k + tid] : 0;
      const int32_t nbv = __shfl_sync(0xffffffffu, ob, sh.bperm[tid] & 31);
      if (tid < bs) A.lp[k + tid] = nbv;
    }
    __syncthreads();
  }
  for (int t = tid; t < bs * bs; t += NT) {
    int i = t % bs, j = t / bs;
    if (i >= j) st->T[i][j] = sh.T[i][j];
  }
  if (tid < 32) {
    st->bperm[tid] = sh.bperm[tid];
    st->bdt[tid] = sh.bdt[tid];
    st->bdd[tid] = sh.bdd[tid];
    st->bdo[tid] = sh.bdo[tid];
  }
  if (tid == 0) { st->bs = bs; st->bnelim = bnelim; st->eff = bnelim; }
}

// One row of W = L D over pivots [0, n) (l(c) = l[c * ld]; D given by type,
// diagonal and off-diagonal; the second column of a 2x2 is written with its
// first), 16 columns at a time: the chunk's L and D values are loaded before
// any W store, so the row's memory latency is not paid per column.
__device__ __forceinline__ void lf_w_row(const double* l, int64_t ld, int n, const int8_t* dt, const double* dd,
                                         const double* dof, double* w, int64_t wld) {
  for (int c0 = 0; c0 < n; c0 += 16) {
    double lv[17], dv[17], ov[16];
    int8_t tv[16];
#pragma unroll
    for (int u = 0; u < 17; ++u) {
      const bool in = c0 + u < n;
      lv[u] = in ? l[(int64_t)(c0 + u) * ld] : 0.0;
      dv[u] = in ? dd[c0 + u] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < 16; ++u) {
      const bool in = c0 + u < n;
      ov[u] = in ? dof[c0 + u] : 0.0;
      tv[u] = in ? dt[c0 + u] : (int8_t)PT_DELAYED;
    }
#pragma unroll
    for (int u = 0; u < 16; ++u) {
      const int64_t c = c0 + u;
      if (tv[u] == PT_1X1) {
        w[c * wld] = __dmul_rn(lv[u], dv[u]);
      } else if (tv[u] == PT_2X2) {
        w[c * wld] = __dadd_rn(__dmul_rn(lv[u], dv[u]), __dmul_rn(lv[u + 1], ov[u]));
        w[(c + 1) * wld] = __dadd_rn(__dmul_rn(lv[u], ov[u]), __dmul_rn(lv[u + 1], dv[u + 1]));
      }
    }
  }
}

// panel rows: backup, permute, TRSM, D^-1, threshold scan (grid over rows,
// one row per thread, the row's 32 values in registers: every index into
// them is a compile-time constant)
constexpr int LF_PANEL_T = 64;
__global__ void __launch_bounds__(LF_PANEL_T) k_lf_panel(LFArgs A) {
  chain_enter();
  if (A.st->spec_bad) return;  // a block issued past a mispredicted start column
  LFState* st = A.st;
  const int bnelim = st->bnelim;
  if (bnelim == 0) return;
  __shared__ double T[IBMAX][IBMAX + 1];
  __shared__ int bperm[IBMAX];
  __shared__ int8_t bdt[IBMAX];
  __shared__ double bdd[IBMAX], bdo[IBMAX], dinv[IBMAX];
  __shared__ int s_fail;
  const int bs = st->bs, k = st->k;
  {
    // the factored block: thread t takes column t / 2 (rows of one half), all loads before the stores
    const int j = threadIdx.x >> 1, h = threadIdx.x & 1;
    double v[16];
#pragma unroll
    for (int u = 0; u < 16; ++u) {
      const int i = h * 16 + u;
      v[u] = (j < bs && i < bs && i >= j) ? st->T[i][j] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < 16; ++u) T[h * 16 + u][j] = v[u];
  }
  if (threadIdx.x < IBMAX) {
    const int c = threadIdx.x;
    bperm[c] = st->bperm[c];
    const int8_t t = st->bdt[c];
    const double d = st->bdd[c], o = st->bdo[c];
    bdt[c] = t;
    bdd[c] = d;
    bdo[c] = o;
    // the reciprocal each row's D^-1 step uses: 1 / d (1x1) or 1 / det (2x2 first column)
    double r = 0.0;
    if (c < bnelim && t == PT_1X1) r = 1.0 / d;
    else if (c < bnelim && t == PT_2X2 && c + 1 < IBMAX) r = 1.0 / __dsub_rn(__dmul_rn(d, st->bdd[c + 1]), __dmul_rn(o, o));
    dinv[c] = r;
  }
  if (threadIdx.x == 0) s_fail = bnelim;
  __syncthreads();
  const int64_t bm = A.m - A.cs;
  PanelView V{A.a + A.cs + A.cs * A.m, A.m};
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t be = k + bs;
  const double bound = 1.0 / A.o.threshold;
  if (r < k) {
    // the block's row permutation applied to the view's earlier column r (step 5 of the block, left to
    // the threads that have no panel row: they touch rows k .. be of columns before k, which no other
    // thread of this launch reads); all loads of the column before its stores
    double buf[IBMAX];
#pragma unroll
    for (int i = 0; i < IBMAX; ++i) buf[i] = i < bs ? V(k + bperm[i], r) : 0.0;
#pragma unroll
    for (int i = 0; i < IBMAX; ++i)
      if (i < bs) V(k + i, r) = buf[i];
  }
  if (r >= be && r < bm) {
    // every load of the row before the first store: the backup may alias the
    // panel as far as the compiler knows, so a load placed after a store
    // would wait for it (one memory round trip per column)
    double raw[IBMAX], x[IBMAX];
#pragma unroll
    for (int i = 0; i < IBMAX; ++i) raw[i] = i < bs ? V(r, k + i) : 0.0;
#pragma unroll
    for (int i = 0; i < IBMAX; ++i) x[i] = i < bs ? V(r, k + bperm[i]) : 0.0;
#pragma unroll
    for (int i = 0; i < IBMAX; ++i)
      if (i < bs) A.pb[r + (int64_t)i * bm] = raw[i];
#pragma unroll
    for (int j = 1; j < IBMAX; ++j)
      if (j < bnelim) {
#pragma unroll
        for (int l = 0; l < j; ++l) x[j] = __fma_rn(-x[l], T[j][l], x[j]);
      }
    // D^-1 over the pivots (the second column of a 2x2 is handled with its first)
#pragma unroll
    for (int c = 0; c < IBMAX; ++c) {
      if (c >= bnelim) continue;
      if (bdt[c] == PT_1X1) {
        x[c] = __dmul_rn(x[c], dinv[c]);
      } else if (bdt[c] == PT_2X2 && c + 1 < IBMAX) {
        const double A_ = bdd[c], B_ = bdo[c], C_ = bdd[c + 1];
        const double inv_det = dinv[c];
        const double x1 = x[c], x2 = x[c + 1];
        x[c] = __dmul_rn(__dsub_rn(__dmul_rn(x1, C_), __dmul_rn(x2, B_)), inv_det);
        x[c + 1] = __dmul_rn(__dsub_rn(__dmul_rn(x2, A_), __dmul_rn(x1, B_)), inv_det);
      }
    }
#pragma unroll
    for (int i = 0; i < IBMAX; ++i)
      if (i < bs) V(r, k + i) = x[i];
    // first pivot (1x1 or 2x2 start) with an entry at or above 1/u
    int fail = bnelim;
#pragma unroll
    for (int c = IBMAX - 1; c >= 0; --c) {
      if (c >= bnelim || bdt[c] == PT_2X2B) continue;
      const bool two = bdt[c] == PT_2X2;
      const double x2 = c + 1 < IBMAX ? x[c + 1 < IBMAX ? c + 1 : c] : 0.0;
      if (fabs(x[c]) >= bound || (two && fabs(x2) >= bound)) fail = c;
    }
    if (fail < bnelim) atomicMin(&s_fail, fail);
  }
  __syncthreads();
  if (threadIdx.x == 0 && s_fail < bnelim) atomicMin(&st->eff, s_fail);
}

// 2x2 boundary, restore of the failed diagonal part, failed x failed term,
// D entries: one CTA of 256 threads (CTA 0 of k_lf_wi, before its rows).  It
// writes only the block's own rows, the D entries and the counters; the
// adjusted eliminated count it stores in st->eff / st->nelim is the one every
// CTA of k_lf_wi derives from st->eff itself (the adjustment is idempotent).
__device__ __forceinline__ void lf_post_cta(const LFArgs& A) {
  LFState* st = A.st;
  const int bnelim = st->bnelim, bs = st->bs, k = st->k;
  const int tid = threadIdx.x;
  if (bnelim == 0) {
    if (tid == 0) st->nelim = 0;
    return;
  }
  int eff = st->eff;
  if (eff > 0 && st->bdt[eff - 1] == PT_2X2) eff -= 1;
  PanelView V{A.a + A.cs + A.cs * A.m, A.m};
  if (eff < bnelim) {
    for (int t = tid; t < bs * bs; t += blockDim.x) {
      int i = t % bs, j = t / bs;
      if (i < eff || j < eff) continue;
      int c = st->bperm[j], r = st->bperm[i];
      V(k + i, k + j) = r >= c ? st->Tb[r][c] : st->Tb[c][r];
    }
  }
  __syncthreads();
  const int nelim = eff;
  if (nelim > 0 && nelim < bs) {
    const int nf = bs - nelim;
    for (int t = tid; t < nf * nf; t += blockDim.x) {
      int i = t % nf, j = t / nf;
      if (i < j) continue;
      // sum over the eliminated columns c of (L D)(row i, c) * L(row j, c), each W entry formed as it is
      // added (no local array), in column order
      const double* l = &V(k + nelim + i, k);
      const double* lj = &V(k + nelim + j, k);
      double s = 0.0;
      int c = 0;
      while (c < nelim) {
        if (st->bdt[c] == PT_1X1) {
          s = __dadd_rn(s, __dmul_rn(__dmul_rn(l[c * A.m], st->bdd[c]), lj[c * A.m]));
          c += 1;
        } else {
          const double A_ = st->bdd[c], B_ = st->bdo[c], C_ = st->bdd[c + 1];
          const double l1 = l[c * A.m], l2 = l[(c + 1) * A.m];
          const double w0 = __dadd_rn(__dmul_rn(l1, A_), __dmul_rn(l2, B_));
          const double w1 = __dadd_rn(__dmul_rn(l1, B_), __dmul_rn(l2, C_));
          s = __dadd_rn(s, __dmul_rn(w0, lj[c * A.m]));
          s = __dadd_rn(s, __dmul_rn(w1, lj[(c + 1) * A.m]));
          c += 2;
        }
      }
      V(k + nelim + i, k + nelim + j) = __dsub_rn(V(k + nelim + i, k + nelim + j), s);
    }
  }
  if (tid < 32) {
    // D entries, one pivot column per lane (the adjusted nelim never splits a 2x2)
    DRec VD{A.D.type + A.cs, A.D.diag + A.cs, A.D.off + A.cs};
    const int c = tid;
    const int8_t t = c < nelim ? st->bdt[c] : (int8_t)PT_DELAYED;
    const bool one = t == PT_1X1;
    const bool first = t == PT_2X2 && c + 1 < nelim;
    const bool second = t == PT_2X2B;
    if (one || first || second) {
      VD.type[k + c] = one ? PT_1X1 : (first ? PT_2X2 : PT_2X2B);
      VD.diag[k + c] = st->bdd[c];
      VD.off[k + c] = first ? st->bdo[c] : 0.0;
    }
    const int n1 = __popc(__ballot_sync(0xffffffffu, one));
    const int n2 = __popc(__ballot_sync(0xffffffffu, first));
    if (tid == 0) {
      st->n1 += n1; st->n2 += n2;
      st->nelim = nelim;
      st->eff = eff;
    }
  }
}

// Rows below the inner block (one thread per row): restore of the failed
// panel columns from the backup, W = L D over the eliminated columns
// (column-major, ld = rows of the view, indexed by absolute row) and the
// trailing x failed cross term.  The rank-nelim update of the outer block's
// trailing columns that follows is the DMMA GEMM (k_syrk_dmma with the
// region start read from the device), the same fma chain per entry.
__global__ void __launch_bounds__(256) k_lf_wi(LFArgs A) {
  chain_enter();
  if (A.st->spec_bad) return;  // a block issued past a mispredicted start column
  LFState* st = A.st;
  const int bnelim = st->bnelim;
  if (bnelim > 0) {
    const int bs = st->bs, k = st->k;
    // the eliminated count: the panel's first failing column, one less where it would split a 2x2 (the
    // value CTA 0 stores below)
    int eff = st->eff;
    if (eff > 0 && st->bdt[eff - 1] == PT_2X2) eff -= 1;
    const int nelim = eff;
    const int64_t bm = A.m - A.cs;
    const int64_t ts = k + bs;
    const int nf = bs - nelim;
    __shared__ double Ls[IBMAX][IBMAX + 1];
    __shared__ int bperm[IBMAX];
    __shared__ int8_t bdt[IBMAX];
    __shared__ double bdd[IBMAX], bdo[IBMAX];
    PanelView V{A.a + A.cs + A.cs * A.m, A.m};
    if (threadIdx.x < IBMAX) {
      bperm[threadIdx.x] = st->bperm[threadIdx.x];
      bdt[threadIdx.x] = st->bdt[threadIdx.x];
      bdd[threadIdx.x] = st->bdd[threadIdx.x];
      bdo[threadIdx.x] = st->bdo[threadIdx.x];
    }
    if (nelim > 0 && nf > 0)
      for (int t = threadIdx.x; t < nf * nelim; t += blockDim.x) {
        int jj = t % nf, c = t / nf;
        Ls[jj][c] = V(k + nelim + jj, k + c);
      }
    __syncthreads();
    const int64_t i = ts + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < bm) {
      if (eff < bnelim)
        for (int j = eff; j < bs; ++j) V(i, k + j) = A.pb[i + (int64_t)bperm[j] * bm];
      if (nelim > 0) {
        double* W = A.w + i;
        lf_w_row(&V(i, k), A.m, nelim, bdt, bdd, bdo, W, bm);
        for (int jj = 0; jj < nf; ++jj) {
          double s = 0.0;
          for (int c2 = 0; c2 < nelim; ++c2) s = __dadd_rn(s, __dmul_rn(W[(int64_t)c2 * bm], Ls[jj][c2]));
          V(i, k + nelim + jj) = __dsub_rn(V(i, k + nelim + jj), s);
        }
      }
    }
  }
  // the block's own rows, its D entries and counts (CTA 0, after its rows: the two touch different rows)
  if (blockIdx.x == 0) lf_post_cta(A);  // uniform over the CTA
}

// delayed columns of the inner block to the end of the outer block (1 CTA)
__device__ void lf_delay_cta(const LFArgs& A) {
  LFState* st = A.st;
  const int tid = threadIdx.x;
  const int k = st->k, bs = st->bs, bnelim = st->bnelim, nelim = st->nelim;
  int end_pos = st->end_pos;
  if (bs == 0) return;
  const int64_t bm = A.m - A.cs;
  PanelView V{A.a + A.cs + A.cs * A.m, A.m};
  __syncthreads();
  if (bnelim == 0) {
    for (int off = 0; off < bs; ++off) {
      end_pos -= 1;
      if (k + off < end_pos) {
        cta_swap(V, bm, k + off, end_pos);
        if (tid == 0) { int32_t t = A.lp[k + off]; A.lp[k + off] = A.lp[end_pos]; A.lp[end_pos] = t; }
      }
    }
  } else if (nelim < bs) {
    int nd = bs - nelim;
    for (int i = nd - 1; i >= 0; --i) {
      int dp = k + nelim + i;
      end_pos -= 1;
      if (dp < end_pos) {
        cta_swap(V, bm, dp, end_pos);
        if (tid == 0) { int32_t t = A.lp[dp]; A.lp[dp] = A.lp[end_pos]; A.lp[end_pos] = t; }
      }
    }
  }
  __syncthreads();
  if (tid == 0) { st->k = k + nelim; st->end_pos = end_pos; st->bne = k + nelim; }
}
// the last inner block's delays (the others run at the start of the next k_lf_block)
__global__ void __launch_bounds__(NT) k_lf_delay(LFArgs A) {
  chain_enter();
  if (A.st->spec_bad) return;  // a block issued past a mispredicted start column
  lf_delay_cta(A);
}

// row permutation of the outer block applied to the front's earlier columns
// 0..cs (two_level_factor, factor.rs:2165-2181): 16 columns per CTA
constexpr int LF_PROP_COLS = 16;
__global__ void __launch_bounds__(256) k_lf_prop(LFArgs A) {
  chain_enter();
  if (A.st->spec_bad) return;  // a block issued past a mispredicted start column
  extern __shared__ double buf[];  // bcols x LF_PROP_COLS
  const int64_t c0 = (int64_t)blockIdx.x * LF_PROP_COLS;
  const int nc = (int)((A.cs - c0) < LF_PROP_COLS ? (A.cs - c0) : LF_PROP_COLS);
  if (nc <= 0) return;
  const int bc = (int)A.bcols;
  for (int t = threadIdx.x; t < nc * bc; t += blockDim.x) {
    int i = t % bc, c = t / bc;
    buf[t] = A.a[(A.cs + A.lp[i]) + (c0 + c) * A.m];
  }
  __syncthreads();
  for (int t = threadIdx.x; t < nc * bc; t += blockDim.x) {
    int i = t % bc, c = t / bc;
    A.a[(A.cs + i) + (c0 + c) * A.m] = buf[t];
  }
}

// W = L D for the rows below the outer block, over its bne eliminated
// columns, appended to the pending window
__global__ void __launch_bounds__(128) k_lf_w(LFArgs A) {
  chain_enter();
  if (A.st->spec_bad) return;  // a block issued past a mispredicted start column
  const int bne = A.st->bne;
  const int64_t oe = A.cs + A.bcols;
  const int64_t i = oe + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= A.m) return;
  const int8_t* dt = A.D.type + A.cs;
  const double* dd = A.D.diag + A.cs;
  const double* dof = A.D.off + A.cs;
  const double* l = A.a + i + A.cs * A.m;
  double* w = A.wo + (i - A.wrow0) + A.wcol0 * A.wld;
  lf_w_row(l, A.m, bne, dt, dd, dof, w, A.wld);
}

// end of an outer block: column order, delays to the end of the remaining
// fully-summed columns (two_level), eliminated total (1 CTA)
// The delayed columns of the outer block [cs, cs + bcols) (its last
// bcols - bne) swap places with the last columns of the remaining range
// [cs, cs + rem), so the next block starts on columns that were not tried
// (two_level_factor's swap, factor.rs:2108-2252).  One CTA.
__device__ __forceinline__ void lf_swap_delayed(const LFArgs& A, int64_t cs, int64_t bcols, int64_t rem, int bne) {
  const int tid = threadIdx.x;
  PanelView F{A.a, A.m};
  const int nf = (int)(bcols - bne);
  for (int i = 0; i < nf; ++i) {
    int64_t fp = cs + bne + i, e = cs + rem - 1 - i;
    if (fp < e) {
      cta_swap(F, A.m, fp, e);
      if (tid == 0) { int32_t t = A.perm[fp]; A.perm[fp] = A.perm[e]; A.perm[e] = t; }
    }
  }
}

// End of an outer block: its column order into the front's pivot order, the
// delay swap (unless `swap` is 0: a far-field update may still be running on
// another stream, and the host issues the swap itself, k_lf_swap, once it has
// seen the delay), the eliminated total.
__global__ void __launch_bounds__(NT) k_lf_outer(LFArgs A, int64_t rem, int two_level, int swap) {
  chain_enter();
  if (A.st->spec_bad) return;  // a block issued past a mispredicted start column
  LFState* st = A.st;
  const int tid = threadIdx.x;
  const int bne = st->bne;
  const int64_t cs = A.cs, bcols = A.bcols;
  // perm[cs + i] = orig[lp[i]], via the inner W scratch as the copy buffer
  int32_t* orig = (int32_t*)A.w;
  for (int i = tid; i < bcols; i += NT) orig[i] = A.perm[cs + i];
  __syncthreads();
  for (int i = tid; i < bcols; i += NT) A.perm[cs + i] = orig[A.lp[i]];
  __syncthreads();
  if (swap && two_level && bne < bcols) lf_swap_delayed(A, cs, bcols, rem, bne);
  __syncthreads();
  if (tid == 0) st->gne += bne;
}

// The delay swap of an outer block issued without it (k_lf_outer with swap =
// 0), with the block's start column, width, remaining range and eliminated
// count as the host read them.  One CTA.
__global__ void __launch_bounds__(NT) k_lf_swap(LFArgs A, int64_t cs, int64_t bcols, int64_t rem, int bne) {
  lf_swap_delayed(A, cs, bcols, rem, bne);
}

// TPP fallback on the leftover columns, then the front's results
__global__ void k_lf_finish(LFArgs A, DFront* F, int s) {
  LFState* st = A.st;
  __shared__ int cnt[2];
  const int lane = threadIdx.x;
  int gne = st->gne;
  if (lane == 0) { cnt[0] = 0; cnt[1] = 0; }
  __syncwarp();
  if (gne < A.p && A.o.failed_pivot_tpp) {
    WarpTpp T{PanelView{A.a, A.m}, A.m, A.p, lane};
    gne += (int)T.run(gne, A.p, A.perm, A.D, &cnt[0], &cnt[1], A.o);
  }
  __syncwarp();
  if (lane == 0) {
    F[s].ne = gne;
    F[s].n1 = st->n1 + cnt[0];
    F[s].n2 = st->n2 + cnt[1];
  }
}

}  // namespace rvg
