// B200 numeric phase: level-set multifrontal APTP factorization and the
// supernodal solve, behind the C ABI of include/rivrs_b200.h.
//
// Reference path (rivrs-linalg, sparse/src/symmetric/):
//   AptpNumeric::factor            numeric.rs:844-1023
//   factor_tree_levelset           numeric.rs:1957-2163
//   factor_single_supernode        numeric.rs:1226-1533
//   factor_small_leaf_subtree      numeric.rs:1562-1938
//   aptp_factor_in_place & kernels factor.rs:301-404, 891-3181
//   aptp_solve                     solve.rs:57-326
//   SparseLDLT::solve_in_place     solver.rs:370-428
//
// Layout in HBM (one handle):
//   panel arena   m x k column-major panel per front (the FS columns of the
//                 frontal matrix); after factorization it IS the factor:
//                 L11 in rows [0,ne), L21 in rows [ne,m), columns [0,ne).
//   index arena   per front: row list (m global indices: owned ++ delayed
//                 ++ pattern) followed by the local pivot order (k).
//   D arrays      per front k entries (type, diag, off).
//   contribution  the NFS x NFS Schur block of each non-root front, one
//                 stream-ordered allocation per wave, released once every
//                 parent that reads it has been assembled.
// Each wave (all fronts whose children are done) runs: row lists -> scatter
// of original entries -> extend-add, one pass per child ordinal so every
// destination receives its terms in the reference's order without atomics
// -> dense factorization (warp TPP or CTA APTP) -> contribution GEMM.  One
// small device->host copy per wave returns the eliminated counts that size
// the next wave (delays change front sizes at run time).
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <string>
#include <thread>
#include <type_traits>
#include <vector>

#include <thread>

#include "dense.cuh"
#include "front.cuh"
#include "mlp.cuh"
#include "rvg_internal.h"

namespace rvg {

// ---------------------------------------------------------------------------
// error plumbing
// ---------------------------------------------------------------------------
thread_local std::string g_err;
void set_error(const std::string& s) { g_err = s; }

#define CK(call)                                                                                \
  do {                                                                                          \
    cudaError_t e_ = (call);                                                                    \
    if (e_ != cudaSuccess) {                                                                    \
      set_error(std::string("CUDA error: ") + cudaGetErrorString(e_) + " at " #call);           \
      return e_ == cudaErrorMemoryAllocation ? RVG_ERR_OUT_OF_MEMORY : RVG_ERR_DEVICE;          \
    }                                                                                           \
  } while (0)

// ---------------------------------------------------------------------------
// assembly kernels
// ---------------------------------------------------------------------------

// Row list of each front: owned ++ delayed-from-children ++ pattern
// (numeric.rs:1239-1262), and the identity pivot order.
__global__ void k_front_rows(const int32_t* ids, int n, DFront* F, Statics S, Arenas A) {
  int f = blockIdx.x;
  if (f >= n) return;
  int s = ids[f];
  const DFront fr = F[s];
  int32_t* rows = A.idx + fr.idx;
  int32_t* perm = rows + fr.m;
  int64_t o0 = S.own_ptr[s];
  for (int i = threadIdx.x; i < fr.nown; i += blockDim.x) rows[i] = S.own_idx[o0 + i];
  int64_t p0 = S.pat_ptr[s];
  for (int i = threadIdx.x; i < fr.nfs; i += blockDim.x) rows[fr.k + i] = S.pat_idx[p0 + i];
  for (int i = threadIdx.x; i < fr.k; i += blockDim.x) perm[i] = i;
  for (int64_t q = S.ch_ptr[s]; q < S.ch_ptr[s + 1]; ++q) {
    const DFront c = F[S.ch_idx[q]];
    int nd = c.k - c.ne;
    const int32_t* crow = A.idx + c.idx;
    const int32_t* cperm = crow + c.m;
    for (int i = threadIdx.x; i < nd; i += blockDim.x) rows[fr.nown + c.dly_off + i] = crow[cperm[c.ne + i]];
  }
}

struct ScatterItem { int32_t front; int32_t pad; int64_t e0; };

// Original entries (numeric.rs:1306-1344 amap path, 2376-2435 per-entry
// path); each destination receives at most one original entry.
__global__ void k_scatter(const ScatterItem* items, const DFront* F, Statics S, Arenas A, const double* vals,
                          const double* scal) {
  ScatterItem it = items[blockIdx.x];
  const DFront fr = F[it.front];
  int64_t e = it.e0 + threadIdx.x;
  if (e >= S.amap_ptr[it.front + 1]) return;
  const int32_t* q = S.amap + 5 * e;
  int32_t r = q[1], c = q[2];
  if (r >= fr.nown) r += fr.ndin;
  if (c >= fr.nown) c += fr.ndin;
  double v = vals[q[0]];
  if (scal) {
    if (fr.ndin == 0) v = __dmul_rn(__dmul_rn(v, scal[q[3]]), scal[q[4]]);
    else v = __dmul_rn(v, __dmul_rn(scal[q[3]], scal[q[4]]));
  }
  if (c < fr.k) {
    double* a = A.panel + fr.panel;
    a[r + (int64_t)c * fr.m] += v;
  } else if ((fr.flags & FF_HAS_CB) && r >= fr.k) {
    A.cbase[fr.cb + (r - fr.k) + (int64_t)(c - fr.k) * fr.nfs] += v;
  }
}

// Extend-add of one child's contribution into its parent
// (numeric.rs:2445-2559).  The child block is [delayed; NFS] x [delayed;
// NFS]: its delayed columns live in the child's panel (rows ne..k and k..m
// of columns ne..k), its NFS x NFS part in the child's contribution buffer.
// An item is a 32-column group [j0, j0+32) of one child's block and a
// segment of its rows [i0, i0 + EA_ROWS), i >= j only.  Each CTA stages the group's 32 destination
// columns in shared memory, then walks its rows in tiles of 256, one row per
// thread: the thread maps its row once, then handles the 32 columns in
// batches of 8 with all eight source loads, then all eight destination
// loads, in flight together (the one-entry-at-a-time loop kept too few bytes
// in flight per SM to reach HBM bandwidth).  Source reads are coalesced (a
// column of the child block is contiguous); each destination entry still
// receives exactly one term from this child, so the per-ordinal launches
// keep the reference's order of terms.
constexpr int EA_ROWS = 4096;  // rows per item
struct EaTile { int32_t parent; int32_t child; int32_t j0; int32_t i0; };

__global__ void __launch_bounds__(256, 3) k_extend_add_tiled(const EaTile* items, const DFront* F, Statics S, Arenas A) {
  const EaTile it = items[blockIdx.x];
  const DFront P = F[it.parent];
  const DFront C = F[it.child];
  const int nd = C.k - C.ne;
  const int sz = C.m - C.ne;
  const int32_t* __restrict__ ea = S.ea_map + S.ea_ptr[it.child];
  const double* __restrict__ cp = A.panel + C.panel;
  const double* __restrict__ cb = A.cbase + (C.cb < 0 ? 0 : C.cb);
  double* pp = A.panel + P.panel;
  double* pc = A.cbase + (P.cb < 0 ? 0 : P.cb);
  const bool pcb = (P.flags & FF_HAS_CB) != 0;
  auto map = [&](int i) -> int {
    if (i < nd) return P.nown + C.dly_off + i;
    int l = __ldg(ea + (i - nd));
    return l < P.nown ? l : l + P.ndin;
  };
  __shared__ int s_lj[32];
  const int jn = min(32, sz - it.j0);
  if (threadIdx.x < 32) s_lj[threadIdx.x] = threadIdx.x < jn ? map(it.j0 + threadIdx.x) : 0;
  __syncthreads();
  const int i1 = min(sz, it.i0 + EA_ROWS);
  for (int ib = it.i0; ib < i1; ib += 256) {
    const int i = ib + threadIdx.x;
    if (i >= i1) break;
    const int li = map(i);
    // rows of the child block: delayed rows live in the child's panel rows ne.., NFS rows at k..
    const int64_t prow = i < nd ? (int64_t)(C.ne + i) : (int64_t)(C.k + (i - nd));
#pragma unroll 1
    for (int jb = 0; jb < 32; jb += 8) {
      double v[8];
      double* dst[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const int jj = jb + q, j = it.j0 + jj;
        v[q] = 0.0;
        if (jj < jn && i >= j) {
          v[q] = j < nd ? cp[prow + (int64_t)(C.ne + j) * C.m] : cb[(i - nd) + (int64_t)(j - nd) * C.nfs];
        }
      }
      double old[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        dst[q] = nullptr;
        if (v[q] != 0.0) {
          const int lj = s_lj[jb + q];
          const int r = li >= lj ? li : lj, c = li >= lj ? lj : li;
          if (c < P.k) dst[q] = pp + r + (int64_t)c * P.m;
          else if (pcb && r >= P.k) dst[q] = pc + (r - P.k) + (int64_t)(c - P.k) * P.nfs;
        }
        old[q] = dst[q] ? *dst[q] : 0.0;
      }
#pragma unroll
      for (int q = 0; q < 8; ++q)
        if (dst[q]) *dst[q] = old[q] + v[q];
    }
  }
}

// Zeros the lower triangle (rows j..nfs of column j) of the contribution
// blocks of a wave: item = (front, first of 32 columns).  The upper
// triangle is never read.
struct CbZeroItem { int32_t front; int32_t j0; };
__global__ void __launch_bounds__(256) k_zero_cb_lower(const CbZeroItem* items, const DFront* F, Arenas A) {
  const CbZeroItem it = items[blockIdx.x];
  const DFront f = F[it.front];
  double* c = A.cbase + f.cb;
  const int jend = min(f.nfs, it.j0 + 32);
  for (int j = it.j0; j < jend; ++j) {
    double* col = c + (int64_t)j * f.nfs;
    for (int i = j + threadIdx.x; i < f.nfs; i += blockDim.x) col[i] = 0.0;
  }
}

// ---------------------------------------------------------------------------
// dense factorization kernels
// ---------------------------------------------------------------------------

// One warp per front: TPP on all k columns (small-leaf fronts, numeric.rs:
// 1805; fronts with k < ib, factor.rs:360-362).
// TPP on all k columns of front s by one warp; cnt: the warp's two shared counters.
__device__ void warp_tpp_front(int s, DFront* F, const Arenas& A, const DevOpts& o, int* cnt) {
  const int lane = threadIdx.x & 31;
  const DFront fr = F[s];
  if (lane == 0) { cnt[0] = 0; cnt[1] = 0; }
  __syncwarp();
  WarpTpp T{PanelView{A.panel + fr.panel, fr.m}, fr.m, fr.k, lane};
  int32_t* perm = A.idx + fr.idx + fr.m;
  DRec d{A.dtype + fr.dpos, A.ddiag + fr.dpos, A.doff + fr.dpos};
  int64_t ne = T.run(0, fr.k, perm, d, &cnt[0], &cnt[1], o);
  __syncwarp();
  if (lane == 0) { F[s].ne = (int32_t)ne; F[s].n1 = cnt[0]; F[s].n2 = cnt[1]; }
}

__global__ void k_tpp(const int32_t* ids, int n, DFront* F, Arenas A, DevOpts o) {
  int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (w >= n) return;
  __shared__ int cnt[8][2];
  warp_tpp_front(ids[w], F, A, o, cnt[threadIdx.x >> 5]);
}

constexpr int NT = APTP_THREADS;  // threads of the CTA APTP kernel
constexpr int IBMAX = 32; // inner block size supported by the kernels

struct CtaShared {
  double T[IBMAX][IBMAX + 1];
  double Lj[IBMAX];
  int bperm[IBMAX];
  int8_t bdt[IBMAX];
  double bdd[IBMAX];
  double bdo[IBMAX];
  int bnelim, eff, n1, n2, end_pos, k;
  int tmpi[NT];
  double tmpd[NT];
};

// Complete pivoting on the bs x bs diagonal block held in shared memory
// (factor_block_diagonal, factor.rs:891-1153).  Per pivot step, warp 0 finds
// the pivot (lane = column, its rows in registers; the reduction keeps the
// largest magnitude and, among equal ones, the smallest (column, row) key: the
// reference's column-then-row scan with a strict >), performs the symmetric
// swaps, the reciprocal and the scaling of the pivot column(s); then every
// warp takes part in the rank-1 / rank-2 update (warps take columns, lanes
// rows).  Two CTA barriers per step; every entry gets the same operations as
// in the reference's loops.
__device__ void cta_block_factor(CtaShared& sh, int bs, double small) {
  static_assert(NT == 256 && IBMAX == 32, "the update's column split assumes 8 warps and 32-column blocks");
  double(*T)[IBMAX + 1] = sh.T;
  __shared__ int s_kind;
  __shared__ double s_d[3];
  // column maxima of the trailing triangle after each update (bits of |v| and the (column, row) key of the
  // first maximum in row order), left by the updating warps for the next step's pivot search
  __shared__ unsigned s_chi[IBMAX], s_clo[IBMAX], s_ckey[IBMAX];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid < IBMAX) { sh.bperm[tid] = tid; sh.bdt[tid] = PT_DELAYED; sh.bdd[tid] = 0; sh.bdo[tid] = 0; }
  __syncthreads();
  // swap_symmetric_block limited to the block (warp 0)
  auto swp = [&](int i, int j) {
    if (i == j) return;
    if (i > j) { int t = i; i = j; j = t; }
    if (lane == 0) {
      double t = T[i][i]; T[i][i] = T[j][j]; T[j][j] = t;
      int p = sh.bperm[i]; sh.bperm[i] = sh.bperm[j]; sh.bperm[j] = p;
    }
    if (lane < i) { double t = T[i][lane]; T[i][lane] = T[j][lane]; T[j][lane] = t; }
    if (lane > i && lane < j) { double t = T[lane][i]; T[lane][i] = T[j][lane]; T[j][lane] = t; }
    if (lane > j && lane < bs) { double t = T[lane][i]; T[lane][i] = T[lane][j]; T[lane][j] = t; }
    __syncwarp();
  };
  // each updated column j0 + 8q of this warp: the maximum of |T[i][j]| over rows j <= i < bs (the lanes'
  // new values) and the smallest row holding it, as the scan in row order finds them (entries that are not
  // > 0, NaN included, never count)
  auto col_maxima = [&](int j0, int i, const double* nvq) {
#pragma unroll
    for (int q = 0; q < IBMAX / 8; ++q) {
      const int j = j0 + 8 * q;
      if (j < bs) {  // uniform over the warp
        const double a = (i >= j && i < bs) ? fabs(nvq[q]) : 0.0;
        const bool pos = a > 0.0;
        const unsigned long long bits = pos ? (unsigned long long)__double_as_longlong(a) : 0ull;
        const unsigned h1 = (unsigned)(bits >> 32), l1 = (unsigned)bits;
        const unsigned mh = __reduce_max_sync(0xffffffffu, h1);
        const unsigned ml = __reduce_max_sync(0xffffffffu, h1 == mh ? l1 : 0u);
        const unsigned kk = __reduce_min_sync(0xffffffffu, (pos && h1 == mh && l1 == ml) ? (unsigned)(j * 64 + i)
                                                                                          : 0xffffffffu);
        if (lane == 0) { s_chi[j] = mh; s_clo[j] = ml; s_ckey[j] = kk; }
      }
    }
  };
  int k = 0;
  for (;;) {
    const int cur = k;
    if (warp == 0) {
      int kind = 0;  // 0 stop, 1 1x1 (+ rank-1 update), 2 2x2 (+ rank-2 update)
      if (cur < bs) {
        // arg-max over the lower triangle of [cur, bs)^2: lane = column, its first maximum in row order
        unsigned hi = 0, lo = 0, key = 0xffffffffu;
        if (lane >= cur && lane < bs) {
          if (cur == 0) {  // the first step scans the block
            double col[IBMAX];
#pragma unroll
            for (int i = 0; i < IBMAX; ++i) col[i] = T[i][lane];
            // four interleaved scans (rows i mod 4), each keeping its first maximum,
            // merged to the first maximum in row order
            double b4[4] = {0.0, 0.0, 0.0, 0.0};
            unsigned k4[4] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0xffffffffu};
#pragma unroll
            for (int i = 0; i < IBMAX; ++i)
              if (i >= lane && i < bs) {
                const double v = fabs(col[i]);
                if (v > b4[i & 3]) { b4[i & 3] = v; k4[i & 3] = (unsigned)(lane * 64 + i); }
              }
            double bv = 0.0;
#pragma unroll
            for (int q = 0; q < 4; ++q)
              if (b4[q] > bv || (b4[q] == bv && k4[q] < key)) { bv = b4[q]; key = k4[q]; }
            const unsigned long long bits = (unsigned long long)__double_as_longlong(bv);  // bv >= 0
            hi = (unsigned)(bits >> 32);
            lo = (unsigned)bits;
          } else {  // left by the previous step's update
            hi = s_chi[lane];
            lo = s_clo[lane];
            key = s_ckey[lane];
          }
        }
        const unsigned mhi = __reduce_max_sync(0xffffffffu, hi);
        const unsigned mlo = __reduce_max_sync(0xffffffffu, hi == mhi ? lo : 0u);
        key = __reduce_min_sync(0xffffffffu, (hi == mhi && lo == mlo) ? key : 0xffffffffu);
        const double maxv = __longlong_as_double((long long)(((unsigned long long)mhi << 32) | mlo));
        int mr = cur, mc = cur;
        if (key != 0xffffffffu) { mc = (int)(key / 64); mr = (int)(key % 64); }
        if (maxv >= small) {
          if (mr == mc) {
            // the pivot's reciprocal from its value before the swap (the same number), so
            // the division overlaps the swap
            const double dkk = T[mr][mr], inv = 1.0 / dkk;
            swp(cur, mr);
            if (lane > cur && lane < bs) T[lane][cur] = __dmul_rn(T[lane][cur], inv);
            if (lane == 0) { sh.bdt[cur] = PT_1X1; sh.bdd[cur] = dkk; s_d[0] = dkk; }
            kind = 1;
          } else {
            const int t = mr, mi = mc;
            const double amm = T[mi][mi], att = T[t][t], atm = T[t][mi];
            const double delta = __dsub_rn(__dmul_rn(amm, att), __dmul_rn(atm, atm));
            const int remaining = bs - cur;
            if (remaining < 2) {
              const int pp = fabs(amm) >= fabs(att) ? mi : t;
              const double dkk = T[pp][pp], inv = 1.0 / dkk;
              swp(cur, pp);
              if (!(fabs(dkk) < small)) {
                if (lane > cur && lane < bs) T[lane][cur] = __dmul_rn(T[lane][cur], inv);
                if (lane == 0) { sh.bdt[cur] = PT_1X1; sh.bdd[cur] = dkk; s_d[0] = dkk; }
                kind = 1;  // the rank-1 update is empty here
              }
            } else if (fabs(delta) >= __dmul_rn(__dmul_rn(0.5, atm), atm)) {
              // the swaps bring (mi, t) to (cur, cur + 1): a11 = amm, a22 = att, a21 = atm, and the
              // determinant a11 a22 - a21 a21 is delta; its reciprocal overlaps the swaps
              const double inv_det = 1.0 / delta;
              swp(cur, mi);
              const int nt = (t == cur) ? mi : t;
              swp(cur + 1, nt);
              const double a11 = T[cur][cur], a22 = T[cur + 1][cur + 1], a21 = T[cur + 1][cur];
              if (lane >= cur + 2 && lane < bs) {
                const double ai1 = T[lane][cur], ai2 = T[lane][cur + 1];
                T[lane][cur] = __dmul_rn(__dsub_rn(__dmul_rn(ai1, a22), __dmul_rn(ai2, a21)), inv_det);
                T[lane][cur + 1] = __dmul_rn(__dsub_rn(__dmul_rn(ai2, a11), __dmul_rn(ai1, a21)), inv_det);
              }
              if (lane == 0) {
                sh.bdt[cur] = PT_2X2; sh.bdt[cur + 1] = PT_2X2B;
                sh.bdd[cur] = a11; sh.bdd[cur + 1] = a22; sh.bdo[cur] = a21;
                s_d[0] = a11; s_d[1] = a21; s_d[2] = a22;
              }
              kind = 2;
            } else {
              const int pp = fabs(amm) >= fabs(att) ? mi : t;
              const double dkk = T[pp][pp], inv = 1.0 / dkk;
              swp(cur, pp);
              if (lane > cur && lane < bs) T[lane][cur] = __dmul_rn(T[lane][cur], inv);
              if (lane == 0) { sh.bdt[cur] = PT_1X1; sh.bdd[cur] = dkk; s_d[0] = dkk; }
              kind = 1;
            }
          }
        }
      }
      if (lane == 0) s_kind = kind;
    }
    __syncthreads();
    const int kind = s_kind;
    if (kind == 0) break;
    const int i = lane;
    double nv[IBMAX / 8] = {};  // the lane's (row's) new entries in the warp's columns
    if (kind == 1) {  // T[i][j] -= T[i][cur] (T[j][cur] d), cur < j <= i
      const double dkk = s_d[0];
      if (i > cur && i < bs) {
        const double lc = T[i][cur];
        double lj[IBMAX / 8], tij[IBMAX / 8];
#pragma unroll
        for (int q = 0; q < IBMAX / 8; ++q) {
          const int j = cur + 1 + warp + 8 * q;
          const bool in = j <= i;
          lj[q] = in ? T[j][cur] : 0.0;
          tij[q] = in ? T[i][j] : 0.0;
        }
#pragma unroll
        for (int q = 0; q < IBMAX / 8; ++q) {
          const int j = cur + 1 + warp + 8 * q;
          if (j <= i) {
            nv[q] = __dsub_rn(tij[q], __dmul_rn(lc, __dmul_rn(lj[q], dkk)));
            T[i][j] = nv[q];
          }
        }
      }
      col_maxima(cur + 1 + warp, i, nv);
      k += 1;
    } else {  // rank-2 over cur + 2 <= j <= i
      const double a11 = s_d[0], a21 = s_d[1], a22 = s_d[2];
      if (i >= cur + 2 && i < bs) {
        const double c1 = T[i][cur], c2 = T[i][cur + 1];
        double l1[IBMAX / 8], l2[IBMAX / 8], tij[IBMAX / 8];
#pragma unroll
        for (int q = 0; q < IBMAX / 8; ++q) {
          const int j = cur + 2 + warp + 8 * q;
          const bool in = j <= i;
          l1[q] = in ? T[j][cur] : 0.0;
          l2[q] = in ? T[j][cur + 1] : 0.0;
          tij[q] = in ? T[i][j] : 0.0;
        }
#pragma unroll
        for (int q = 0; q < IBMAX / 8; ++q) {
          const int j = cur + 2 + warp + 8 * q;
          if (j <= i) {
            const double w1 = __dadd_rn(__dmul_rn(l1[q], a11), __dmul_rn(l2[q], a21));
            const double w2 = __dadd_rn(__dmul_rn(l1[q], a21), __dmul_rn(l2[q], a22));
            nv[q] = __dsub_rn(tij[q], __dadd_rn(__dmul_rn(c1, w1), __dmul_rn(c2, w2)));
            T[i][j] = nv[q];
          }
        }
      }
      col_maxima(cur + 2 + warp, i, nv);
      k += 2;
    }
    __syncthreads();
  }
  if (tid == 0) sh.bnelim = k;
  __syncthreads();
}

// Full symmetric swap of positions i, j inside a view of `rows` rows
// (swap_symmetric, factor.rs:458-461), all threads of the CTA.
__device__ void cta_swap(PanelView V, int64_t rows, int64_t i, int64_t j) {
  if (i == j) return;
  if (i > j) { int64_t t = i; i = j; j = t; }
  __syncthreads();
  int tid = threadIdx.x;
  if (tid == 0) { double t = V(i, i); V(i, i) = V(j, j); V(j, j) = t; }
  for (int64_t k = tid; k < i; k += NT) { double t = V(i, k); V(i, k) = V(j, k); V(j, k) = t; }
  for (int64_t k = i + 1 + tid; k < j; k += NT) { double t = V(k, i); V(k, i) = V(j, k); V(j, k) = t; }
  for (int64_t k = j + 1 + tid; k < rows; k += NT) { double t = V(k, i); V(k, i) = V(k, j); V(k, j) = t; }
  __syncthreads();
}

// W = L * D for one row of the panel (compute_ld_into, factor.rs:1536-1563)
__device__ __forceinline__ void row_ld(const double* l, int64_t lstride, const CtaShared& sh, int nelim, double* w) {
  int c = 0;
  while (c < nelim) {
    if (sh.bdt[c] == PT_1X1) { w[c] = __dmul_rn(l[c * lstride], sh.bdd[c]); c += 1; }
    else {
      double A_ = sh.bdd[c], B_ = sh.bdo[c], C_ = sh.bdd[c + 1];
      double l1 = l[c * lstride], l2 = l[(c + 1) * lstride];
      w[c] = __dadd_rn(__dmul_rn(l1, A_), __dmul_rn(l2, B_));
      w[c + 1] = __dadd_rn(__dmul_rn(l1, B_), __dmul_rn(l2, C_));
      c += 2;
    }
  }
}

// factor_inner (factor.rs:1811-2095) on the view V (rows `bm`, `pl` FS
// columns, NFS boundary `nfsb`), executed by the whole CTA.  D entries go to
// VD (view-relative), the view-local column order to lp.  Returns the number
// of eliminated columns.
__device__ int cta_factor_inner(CtaShared& sh, PanelView V, int64_t bm, int pl, int64_t nfsb, DRec VD, int32_t* lp,
                                double* bk, int64_t ldb, double* W, const DevOpts& o) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int ib = o.ib;
  for (int i = tid; i < pl; i += NT) lp[i] = i;
  if (tid == 0) { sh.k = 0; sh.end_pos = pl; sh.n1 = 0; sh.n2 = 0; }
  __syncthreads();
  while (true) {
    int k = sh.k, end_pos = sh.end_pos;
    if (k >= end_pos) break;
    int bs = min(end_pos - k, ib), be = k + bs;
    int64_t rows = bm - k;
    // 1. backup a[k..bm, k..k+bs]
    for (int j = 0; j < bs; ++j)
      for (int64_t i = tid; i < rows; i += NT) bk[i + j * ldb] = V(k + i, k + j);
    // 2. load the diagonal block, factor it with the whole CTA
    for (int t = tid; t < bs * bs; t += NT) {
      int i = t % bs, j = t / bs;
      if (i >= j) sh.T[i][j] = V(k + i, k + j);
    }
    __syncthreads();
    cta_block_factor(sh, bs, o.small);
    int bnelim = sh.bnelim;
    if (bnelim == 0) {
      for (int j = 0; j < bs; ++j)
        for (int64_t i = tid; i < rows; i += NT) V(k + i, k + j) = bk[i + j * ldb];
      __syncthreads();
      for (int off = 0; off < bs; ++off) {
        end_pos -= 1;
        if (k + off < end_pos) {
          cta_swap(V, bm, k + off, end_pos);
          if (tid == 0) { int32_t t = lp[k + off]; lp[k + off] = lp[end_pos]; lp[end_pos] = t; }
        }
      }
      __syncthreads();
      if (tid == 0) sh.end_pos = end_pos;
      __syncthreads();
      continue;
    }
    // write the factored block back (lower triangle) and zero the D
    // off-diagonals of 2x2 pivots (step 4) both there and in the L11 copy
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
      sh.eff = bnelim;
    }
    // 5. row permutation of view columns 0..k
    for (int64_t c = tid; c < k; c += NT) {
      double buf[IBMAX];
      for (int i = 0; i < bs; ++i) buf[i] = V(k + sh.bperm[i], c);
      for (int i = 0; i < bs; ++i) V(k + i, c) = buf[i];
    }
    // 6. column order
    if (tid == 0) {
      int32_t ob[IBMAX];
      for (int i = 0; i < bs; ++i) ob[i] = lp[k + i];
      for (int i = 0; i < bs; ++i) lp[k + i] = ob[sh.bperm[i]];
    }
    __syncthreads();
    // 3 + 7. permute each panel row, TRSM with L11, D^-1 scaling and the
    // threshold scan (apply_and_check, factor.rs:1295-1408)
    const double bound = 1.0 / o.threshold;
    for (int64_t r = be + tid; r < bm; r += NT) {
      double x[IBMAX];
      for (int i = 0; i < bs; ++i) x[i] = V(r, k + sh.bperm[i]);
      for (int j = 0; j < bnelim; ++j)
        for (int l = 0; l < j; ++l) x[j] = __fma_rn(-x[l], sh.T[j][l], x[j]);
      int c = 0;
      while (c < bnelim) {
        if (sh.bdt[c] == PT_1X1) { x[c] = __dmul_rn(x[c], 1.0 / sh.bdd[c]); c += 1; }
        else {
          double A_ = sh.bdd[c], B_ = sh.bdo[c], C_ = sh.bdd[c + 1];
          double inv_det = 1.0 / __dsub_rn(__dmul_rn(A_, C_), __dmul_rn(B_, B_));
          double x1 = x[c], x2 = x[c + 1];
          x[c] = __dmul_rn(__dsub_rn(__dmul_rn(x1, C_), __dmul_rn(x2, B_)), inv_det);
          x[c + 1] = __dmul_rn(__dsub_rn(__dmul_rn(x2, A_), __dmul_rn(x1, B_)), inv_det);
          c += 2;
        }
      }
      for (int i = 0; i < bs; ++i) V(r, k + i) = x[i];
      int fail = bnelim;
      c = 0;
      while (c < bnelim) {
        int w = sh.bdt[c] == PT_2X2 ? 2 : 1;
        bool bad = fabs(x[c]) >= bound || (w == 2 && fabs(x[c + 1]) >= bound);
        if (bad) { fail = c; break; }
        c += w;
      }
      if (fail < bnelim) atomicMin(&sh.eff, fail);
    }
    __syncthreads();
    int eff = sh.eff;
    // 8. adjust_for_2x2_boundary (factor.rs:1161-1174)
    if (eff > 0 && sh.bdt[eff - 1] == PT_2X2) eff -= 1;
    // 9. partial restore of the failed columns
    if (eff < bnelim) {
      for (int t = tid; t < bs * bs; t += NT) {
        int i = t % bs, j = t / bs;
        if (i < eff || j < eff) continue;
        int c = sh.bperm[j], r = sh.bperm[i];
        V(k + i, k + j) = (r >= c) ? bk[r + (int64_t)c * ldb] : bk[c + (int64_t)r * ldb];
      }
      for (int j = eff; j < bs; ++j) {
        int c = sh.bperm[j];
        for (int64_t i = bs + tid; i < rows; i += NT) V(k + i, k + j) = bk[i + (int64_t)c * ldb];
      }
    }
    __syncthreads();
    const int nelim = eff;
    const int64_t ts = be, tsz = bm - be;
    // 10. Schur updates (update_trailing factor.rs:1418-1526, update_cross_terms 1669-1766)
    if (nelim > 0) {
      for (int64_t i = tid; i < tsz; i += NT) row_ld(&V(ts + i, k), V.ld, sh, nelim, W + i * IBMAX);
      __syncthreads();
      // columns are independent: no barrier between them; L[j, :] is a
      // warp-uniform (broadcast) read
      for (int64_t j = ts; j < nfsb; ++j) {
        const double* lj = &V(j, k);
        for (int64_t i = j + tid; i < bm; i += NT) {
          const double* w = W + (i - ts) * IBMAX;
          double acc = V(i, j);
          for (int c = 0; c < nelim; ++c) acc = __fma_rn(-w[c], lj[c * V.ld], acc);
          V(i, j) = acc;
        }
      }
      __syncthreads();
      if (nelim < bs) {
        const int nf = bs - nelim;
        // failed x failed, and trailing x failed; W_blk from the failed rows
        for (int t = tid; t < nf * nf; t += NT) {
          int i = t % nf, j = t / nf;
          if (i < j) continue;
          double wb[IBMAX];
          row_ld(&V(k + nelim + i, k), V.ld, sh, nelim, wb);
          double s = 0.0;
          for (int c = 0; c < nelim; ++c) s = __dadd_rn(s, __dmul_rn(wb[c], V(k + nelim + j, k + c)));
          V(k + nelim + i, k + nelim + j) = __dsub_rn(V(k + nelim + i, k + nelim + j), s);
        }
        for (int j = 0; j < nf; ++j) {
          const double* lj = &V(k + nelim + j, k);
          for (int64_t i = tid; i < tsz; i += NT) {
            const double* w = W + i * IBMAX;
            double s = 0.0;
            for (int c = 0; c < nelim; ++c) s = __dadd_rn(s, __dmul_rn(w[c], lj[c * V.ld]));
            V(ts + i, k + nelim + j) = __dsub_rn(V(ts + i, k + nelim + j), s);
          }
        }
        __syncthreads();
      }
    }
    // 11. D entries and counts for the passed columns
    if (tid == 0) {
      int c = 0;
      while (c < nelim) {
        if (sh.bdt[c] == PT_1X1) {
          VD.type[k + c] = PT_1X1; VD.diag[k + c] = sh.bdd[c]; VD.off[k + c] = 0.0; sh.n1++; c += 1;
        } else if (c + 1 < nelim) {
          VD.type[k + c] = PT_2X2; VD.type[k + c + 1] = PT_2X2B;
          VD.diag[k + c] = sh.bdd[c]; VD.diag[k + c + 1] = sh.bdd[c + 1];
          VD.off[k + c] = sh.bdo[c]; VD.off[k + c + 1] = 0.0; sh.n2++; c += 2;
        } else c += 1;
      }
    }
    __syncthreads();
    // 12. delay the failed columns to end_pos
    if (nelim < bs) {
      int nd = bs - nelim;
      for (int i = nd - 1; i >= 0; --i) {
        int dp = k + nelim + i;
        end_pos -= 1;
        if (dp < end_pos) {
          cta_swap(V, bm, dp, end_pos);
          if (tid == 0) { int32_t t = lp[dp]; lp[dp] = lp[end_pos]; lp[end_pos] = t; }
        }
      }
    }
    __syncthreads();
    if (tid == 0) { sh.k = k + nelim; sh.end_pos = end_pos; }
    __syncthreads();
  }
  return sh.k;
}

// One CTA per front: aptp_factor_in_place (factor.rs:301-404) for fronts with
// k >= ib outside small-leaf subtrees: factor_inner (k <= nb) or
// two_level_factor (k > nb), then the TPP fallback on the leftover columns.
// One front by the whole CTA (aptp_factor_in_place, factor.rs:301-404).
// Every thread reaches every barrier; the CTA's shared state is free again
// when it returns.
__device__ __forceinline__ void cta_aptp_front(CtaShared& sh, int* tpp_cnt, int s, DFront* F, const Arenas& A,
                                               const DevOpts& o) {
  const int tid = threadIdx.x;
  const DFront fr = F[s];
  const int64_t m = fr.m;
  const int p = fr.k;
  PanelView Av{A.panel + fr.panel, m};
  int32_t* perm = A.idx + fr.idx + m;
  DRec D{A.dtype + fr.dpos, A.ddiag + fr.dpos, A.doff + fr.dpos};
  double* bk = A.scratch + fr.scratch;            // m x ib
  double* W = bk + m * IBMAX;                     // m x IBMAX (row-major)
  int32_t* lp = (int32_t*)(W + m * IBMAX);        // nb ints
  int n1 = 0, n2 = 0;
  int gne = 0;
  if (p <= o.nb) {
    gne = cta_factor_inner(sh, Av, m, p, p, D, lp, bk, m, W, o);
    n1 = sh.n1; n2 = sh.n2;
    for (int i = tid; i < p; i += NT) perm[i] = lp[i];
    __syncthreads();
  } else {
    // two_level_factor (factor.rs:2108-2252)
    int rem = p;
    while (rem > 0) {
      int cs = gne, bcols = min(rem, o.nb);
      PanelView V{&Av(cs, cs), m};
      DRec VD{D.type + cs, D.diag + cs, D.off + cs};
      int bne = cta_factor_inner(sh, V, m - cs, bcols, (int64_t)p - cs, VD, lp, bk, m, W, o);
      n1 += sh.n1; n2 += sh.n2;
      // propagate the row permutation to columns 0..cs
      if (cs > 0) {
        // two-pass propagation through the backup buffer: gather, then write
        for (int64_t c0 = 0; c0 < cs; c0 += IBMAX) {
          int nc = (int)(cs - c0 < IBMAX ? cs - c0 : IBMAX);
          for (int t = tid; t < nc * bcols; t += NT) {
            int i = t % bcols, cc = t / bcols;
            bk[i + (int64_t)cc * m] = Av(cs + lp[i], c0 + cc);
          }
          __syncthreads();
          for (int t = tid; t < nc * bcols; t += NT) {
            int i = t % bcols, cc = t / bcols;
            Av(cs + i, c0 + cc) = bk[i + (int64_t)cc * m];
          }
          __syncthreads();
        }
      }
      // column order of the outer block
      if (tid == 0) {
        for (int i = 0; i < bcols; ++i) ((int32_t*)W)[i] = perm[cs + i];
        for (int i = 0; i < bcols; ++i) perm[cs + i] = ((int32_t*)W)[lp[i]];
      }
      __syncthreads();
      // delayed columns to the end of the unprocessed region
      if (bne < bcols) {
        int nf = bcols - bne;
        for (int i = 0; i < nf; ++i) {
          int fp = cs + bne + i, e = cs + rem - 1 - i;
          if (fp < e) {
            cta_swap(Av, m, fp, e);
            if (tid == 0) { int32_t t = perm[fp]; perm[fp] = perm[e]; perm[e] = t; }
          }
        }
      }
      __syncthreads();
      gne += bne;
      rem -= bcols;
    }
  }
  // TPP fallback on columns gne..p (factor.rs:376-401)
  if (gne < p && o.failed_pivot_tpp) {
    if (tid < 32) {
      if (tid == 0) { tpp_cnt[0] = 0; tpp_cnt[1] = 0; }
      __syncwarp();
      WarpTpp T{Av, m, p, tid};
      int64_t add = T.run(gne, p, perm, D, &tpp_cnt[0], &tpp_cnt[1], o);
      if (tid == 0) sh.tmpi[0] = (int)add;
    }
    __syncthreads();
    gne += sh.tmpi[0];
    n1 += tpp_cnt[0];
    n2 += tpp_cnt[1];
  }
  if (tid == 0) { F[s].ne = gne; F[s].n1 = n1; F[s].n2 = n2; }
  __syncthreads();
}

__global__ void __launch_bounds__(NT) k_aptp(const int32_t* ids, int n, DFront* F, Arenas A, DevOpts o) {
  if ((int)blockIdx.x >= n) return;
  __shared__ CtaShared sh;
  __shared__ int tpp_cnt[2];
  cta_aptp_front(sh, tpp_cnt, ids[blockIdx.x], F, A, o);
}

// The medium fronts of a wave (across every system of a union) as one
// persistent launch: a grid of at most the resident CTAs, each taking the
// next front from a work queue (*next, zero at launch) until the list is
// done.  The host lists the fronts largest first, so the long ones start
// early and the short ones fill in behind them.  Which CTA factors a front
// changes nothing in its result.
// One persistent launch for a wave's small and medium fronts: items
// [0, na) are medium fronts (one CTA each, listed largest first), items
// [na, na + ceil(nt / 8)) groups of 8 small fronts (TPP, one warp each),
// taken in order from one atomic counter, so the small fronts fill the
// multiprocessors the long medium fronts leave.  Which CTA or warp takes a
// front changes nothing in its arithmetic.
__global__ void __launch_bounds__(NT) k_front_queue(const int32_t* ids, int na, const int32_t* tids, int nt,
                                                    int32_t* next, DFront* F, Arenas A, DevOpts o) {
  static_assert(NT == 256, "a group of small fronts is one per warp of the CTA");
  __shared__ CtaShared sh;
  __shared__ int tpp_cnt[2];
  __shared__ int wcnt[NT / 32][2];
  __shared__ int s_i;
  const int ng = (nt + 7) / 8;
  for (;;) {
    if (threadIdx.x == 0) s_i = atomicAdd(next, 1);
    __syncthreads();
    const int i = s_i;
    __syncthreads();  // every thread has read s_i before thread 0 takes the next item
    if (i >= na + ng) break;
    if (i < na) {
      cta_aptp_front(sh, tpp_cnt, ids[i], F, A, o);
    } else {
      const int wl = threadIdx.x >> 5, f = (i - na) * 8 + wl;
      if (f < nt) warp_tpp_front(tids[f], F, A, o, wcnt[wl]);
    }
  }
}

}  // namespace rvg

#include "gemm64.cuh"
#include "umma.cuh"
#include "large.cuh"
#include "solve_sf.cuh"

namespace rvg {

// ---------------------------------------------------------------------------
// contribution GEMM: CB -= (L21_NFS D) L21_NFS^T, lower triangle
// (compute_contribution_gemm, factor.rs:1590-1652)
// ---------------------------------------------------------------------------
struct TileItem { int32_t front; int32_t ti; int32_t tj; int32_t pad; };

// W = L21_NFS * D into scratch (nfs x ne, column-major)
__global__ void k_cb_w(const TileItem* items, const DFront* F, Arenas A) {
  TileItem it = items[blockIdx.x];
  const DFront fr = F[it.front];
  const double* L = A.panel + fr.panel;
  double* W = A.scratch + fr.scratch;
  const int8_t* dt = A.dtype + fr.dpos;
  const double* dd = A.ddiag + fr.dpos;
  const double* dof = A.doff + fr.dpos;
  int64_t i = (int64_t)it.ti * 256 + threadIdx.x;
  if (i >= fr.nfs) return;
  const double* l = L + fr.k + i;
  int c = 0;
  while (c < fr.ne) {
    if (dt[c] == PT_1X1) { W[i + (int64_t)c * fr.nfs] = __dmul_rn(l[(int64_t)c * fr.m], dd[c]); c += 1; }
    else {
      double l1 = l[(int64_t)c * fr.m], l2 = l[(int64_t)(c + 1) * fr.m];
      W[i + (int64_t)c * fr.nfs] = __dadd_rn(__dmul_rn(l1, dd[c]), __dmul_rn(l2, dof[c]));
      W[i + (int64_t)(c + 1) * fr.nfs] = __dadd_rn(__dmul_rn(l1, dof[c]), __dmul_rn(l2, dd[c + 1]));
      c += 2;
    }
  }
}

constexpr int GT = 64;  // output tile
constexpr int GK = 16;  // reduction chunk

// C[i,j] = fma(-W[i,c], L[j,c], C[i,j]) for c ascending (each output entry an
// fma chain in the oracle's order); 256 threads, 4x4 outputs per thread.
__global__ void __launch_bounds__(256) k_cb_gemm(const TileItem* items, const DFront* F, Arenas A) {
  TileItem it = items[blockIdx.x];
  const DFront fr = F[it.front];
  const int64_t nfs = fr.nfs, ne = fr.ne, ldl = fr.m;
  const double* L = A.panel + fr.panel + fr.k;  // L21_NFS(j, c) = L[j + c*ldl]
  const double* W = A.scratch + fr.scratch;     // W(i, c) = W[i + c*nfs]
  double* C = A.cbase + fr.cb;
  __shared__ double sW[GK][GT + 1];
  __shared__ double sL[GK][GT + 1];
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  const int64_t i0 = (int64_t)it.ti * GT, j0 = (int64_t)it.tj * GT;
  double acc[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      int64_t i = i0 + ty + 16 * a, j = j0 + tx + 16 * b;
      acc[a][b] = (i < nfs && j < nfs && i >= j) ? C[i + j * nfs] : 0.0;
    }
  for (int64_t c0 = 0; c0 < ne; c0 += GK) {
    for (int t = threadIdx.x; t < GK * GT; t += 256) {
      int r = t % GT, c = t / GT;
      int64_t cc = c0 + c;
      sW[c][r] = (i0 + r < nfs && cc < ne) ? W[i0 + r + cc * nfs] : 0.0;
      sL[c][r] = (j0 + r < nfs && cc < ne) ? L[j0 + r + cc * ldl] : 0.0;
    }
    __syncthreads();
    int kc = (int)(ne - c0 < GK ? ne - c0 : GK);
    for (int c = 0; c < kc; ++c) {
      double wv[4], lv[4];
#pragma unroll
      for (int a = 0; a < 4; ++a) wv[a] = sW[c][ty + 16 * a];
#pragma unroll
      for (int b = 0; b < 4; ++b) lv[b] = sL[c][tx + 16 * b];
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b] = __fma_rn(-wv[a], lv[b], acc[a][b]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      int64_t i = i0 + ty + 16 * a, j = j0 + tx + 16 * b;
      if (i < nfs && j < nfs && i >= j) C[i + j * nfs] = acc[a][b];
    }
}

// ---------------------------------------------------------------------------
// solve kernels (aptp_solve, solve.rs:57-326; SparseLDLT::solve_in_place,
// solver.rs:396-425)
// ---------------------------------------------------------------------------
__global__ void k_perm_scale_in(const double* rhs, int64_t ldb, int64_t nrhs, double* x, int64_t n,
                                const int64_t* pfwd, const double* scal) {
  int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n * nrhs) return;
  int64_t i = t % n, r = t / n;
  double v = rhs[pfwd[i] + r * ldb];
  if (scal) v = __dmul_rn(v, scal[i]);
  x[i + r * n] = v;
}
__global__ void k_perm_scale_out(double* rhs, int64_t ldb, int64_t nrhs, const double* x, int64_t n,
                                 const int64_t* pfwd, const double* scal) {
  int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n * nrhs) return;
  int64_t i = t % n, r = t / n;
  double v = x[i + r * n];
  if (scal) v = __dmul_rn(v, scal[i]);
  rhs[pfwd[i] + r * ldb] = v;
}

// ---------------------------------------------------------------------------
// FP64 iterative refinement (residual of the unfactored matrix)
// ---------------------------------------------------------------------------
// r = b - A x; A full symmetric CSC, so column i is also row i
// right-hand side j = blockIdx.y of columns at stride ldx (x, b) and ldr (r)
__global__ void k_residual(const int64_t* colptr, const int32_t* rowidx, const double* val, const double* x,
                           const double* b, double* r, int64_t n, int64_t ldx, int64_t ldr) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  x += blockIdx.y * ldx;
  b += blockIdx.y * ldx;
  r += blockIdx.y * ldr;
  double s = 0.0;
  for (int64_t p = colptr[i]; p < colptr[i + 1]; ++p) s = __fma_rn(val[p], x[rowidx[p]], s);
  r[i] = b[i] - s;
}
// out[3j] += ||r_j||^2, out[3j + 1] += ||x_j||^2, out[3j + 2] += ||b_j||^2 for j = blockIdx.y
__global__ void k_norms3(const double* r, const double* x, const double* b, int64_t n, double* out, int64_t ldx,
                         int64_t ldr) {
  x += blockIdx.y * ldx;
  b += blockIdx.y * ldx;
  r += blockIdx.y * ldr;
  out += 3 * blockIdx.y;
  double s0 = 0, s1 = 0, s2 = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    s0 += r[i] * r[i]; s1 += x[i] * x[i]; s2 += b[i] * b[i];
  }
  for (int o = 16; o > 0; o >>= 1) {
    s0 += __shfl_xor_sync(0xffffffffu, s0, o);
    s1 += __shfl_xor_sync(0xffffffffu, s1, o);
    s2 += __shfl_xor_sync(0xffffffffu, s2, o);
  }
  if ((threadIdx.x & 31) == 0) { atomicAdd(out, s0); atomicAdd(out + 1, s1); atomicAdd(out + 2, s2); }
}
// Raises *flag when any of the n values is NaN or infinite.
__global__ void k_nonfinite(const double* v, int64_t n, int32_t* flag) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    if (!isfinite(v[i])) { atomicExch(flag, 1); return; }
}

__global__ void k_sumsq(const double* v, int64_t n, double* out) {
  double s = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) s += v[i] * v[i];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(out, s);
}
// GMRES building blocks (one right-hand side): y = A x over the full symmetric CSC
__global__ void k_spmv(const int64_t* colptr, const int32_t* rowidx, const double* val, const double* x, double* y,
                       int64_t n) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double s = 0.0;
  for (int64_t p = colptr[i]; p < colptr[i + 1]; ++p) s = __fma_rn(val[p], x[rowidx[p]], s);
  y[i] = s;
}
// out[i] += V_i . w for the basis vectors i = blockIdx.y (columns of V at stride n)
__global__ void k_dots(const double* V, const double* w, int64_t n, double* out) {
  const double* v = V + blockIdx.y * n;
  double s = 0.0;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
    s = __fma_rn(v[k], w[k], s);
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(out + blockIdx.y, s);
}
// w -= sum_{i < cnt} c_i V_i   (c on the device)
__global__ void k_sub_comb(double* w, const double* V, const double* c, int cnt, int64_t n) {
  int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  double s = w[k];
  for (int i = 0; i < cnt; ++i) s = __fma_rn(-c[i], V[(int64_t)i * n + k], s);
  w[k] = s;
}
// x += sum_{i < cnt} c_i Z_i
__global__ void k_add_comb(double* x, const double* Z, const double* c, int cnt, int64_t n) {
  int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  double s = x[k];
  for (int i = 0; i < cnt; ++i) s = __fma_rn(c[i], Z[(int64_t)i * n + k], s);
  x[k] = s;
}
__global__ void k_scale_to(double* v, const double* w, double a, int64_t n) {
  int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) v[k] = w[k] * a;
}

__global__ void k_axpy1(double* x, const double* d, int64_t n, int64_t ldx, int64_t ldd) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) x[blockIdx.y * ldx + i] += d[blockIdx.y * ldd + i];
}

}  // namespace rvg

// ===========================================================================
// host driver
// ===========================================================================
namespace rvg {

// publish a wave's descriptors / pick up the children's delay offsets
__global__ void k_put_fronts(const DFront* staged, const int32_t* ids, int n, DFront* F) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) F[ids[i]] = staged[i];
}
__global__ void k_put_dly(const int32_t* ids, const int32_t* vals, int n, DFront* F) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) F[ids[i]].dly_off = vals[i];
}
__global__ void k_get_counts(const int32_t* ids, int n, const DFront* F, int32_t* out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) { const DFront& f = F[ids[i]]; out[3 * i] = f.ne; out[3 * i + 1] = f.n1; out[3 * i + 2] = f.n2; }
}
// Refactorization replay checks: the counts (and a large front's progress)
// the captured schedule assumed.  On a difference the flag is raised and the
// recorded value put in place of the computed one, so that every later launch
// of the graph indexes the fronts exactly as the recorded factorization did
// (the parents' sizes and delayed-row offsets were laid out from the record);
// the factor is then discarded and recomputed dynamically.
__global__ void k_check_counts(const int32_t* ids, int n, DFront* F, const int32_t* rec, int32_t* mismatch) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int s = ids[i];
  DFront& f = F[s];
  const int32_t* r = rec + 3 * (int64_t)s;
  if (f.ne != r[0] || f.n1 != r[1] || f.n2 != r[2]) {
    atomicExch(mismatch, 1);
    f.ne = r[0]; f.n1 = r[1]; f.n2 = r[2];
  }
}
__global__ void k_check_gne(LFState* st, int32_t expect, int32_t* mismatch) {
  if (threadIdx.x == 0 && st->gne != expect) {
    atomicExch(mismatch, 1);
    st->gne = expect;
  }
}

// ---------------------------------------------------------------------------
// learned precision (precision = 2): per large front, features of the
// assembled front, the selector's decision, and the observed pivot growth.
// Row of a front in the feature table (FEAT_STRIDE 32-bit words):
//   0 max |a| over the fully-summed columns (lower part), 1 max |a_jj|,
//   2 min |a_jj|, 3 min over columns of |a_jj| / max_{i>j} |a_ij|, 4 columns
//   with that ratio < u, 5 negative diagonals, 6 zero diagonals (as counts),
//   7 max |D| after the factorization; 8..19 the 12 features; 20 the
//   selector's probability that the mixed form is safe; 21 the route (1 =
//   mixed).  Maxima, minima and counts combine by atomics whose result does
//   not depend on their order, so features and routes are reproducible.
// ---------------------------------------------------------------------------
constexpr int FEAT_STRIDE = 32;
constexpr unsigned F_POS_INF = 0x7f800000u;

__global__ void k_feat_init(const int32_t* ids, int n, unsigned* feat) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    unsigned* r = feat + (size_t)ids[i] * FEAT_STRIDE;
    r[0] = 0u; r[1] = 0u; r[2] = F_POS_INF; r[3] = F_POS_INF; r[4] = 0u; r[5] = 0u; r[6] = 0u; r[7] = 0u;
  }
}

__device__ __forceinline__ unsigned fbits(double v) { return __float_as_uint((float)v); }

// grid (column chunks of 8, fronts): warp w of chunk x reads column 8x + w
// of the front's fully-summed block from its diagonal down.
__global__ void __launch_bounds__(256) k_front_features(const int32_t* ids, const DFront* F, Arenas A, double u,
                                                        unsigned* feat) {
  const int s = ids[blockIdx.y];
  const DFront f = F[s];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t j = (int64_t)blockIdx.x * 8 + warp;
  __shared__ unsigned sv[8][7];
  unsigned v[7] = {0u, 0u, F_POS_INF, F_POS_INF, 0u, 0u, 0u};
  if (j < f.k) {
    const double* col = A.panel + f.panel + j * (int64_t)f.m;
    double cm = 0.0;
    for (int64_t i = j + 1 + lane; i < f.m; i += 32) cm = fmax(cm, fabs(col[i]));
    for (int o = 16; o > 0; o >>= 1) cm = fmax(cm, __shfl_xor_sync(0xffffffffu, cm, o));
    const double d = col[j], ad = fabs(d);
    v[0] = fbits(fmax(cm, ad));
    v[1] = fbits(ad);
    v[2] = fbits(ad);
    const double ratio = cm > 0.0 ? ad / cm : INFINITY;
    v[3] = fbits(ratio);
    v[4] = ratio < u ? 1u : 0u;
    v[5] = d < 0.0 ? 1u : 0u;
    v[6] = d == 0.0 ? 1u : 0u;
  }
  if (lane == 0)
    for (int q = 0; q < 7; ++q) sv[warp][q] = v[q];
  __syncthreads();
  if (threadIdx.x == 0) {
    if ((int64_t)blockIdx.x * 8 >= f.k) return;
    unsigned r[7] = {0u, 0u, F_POS_INF, F_POS_INF, 0u, 0u, 0u};
    for (int w = 0; w < 8; ++w) {
      r[0] = max(r[0], sv[w][0]); r[1] = max(r[1], sv[w][1]);
      r[2] = min(r[2], sv[w][2]); r[3] = min(r[3], sv[w][3]);
      r[4] += sv[w][4]; r[5] += sv[w][5]; r[6] += sv[w][6];
    }
    unsigned* row = feat + (size_t)s * FEAT_STRIDE;
    atomicMax(row + 0, r[0]); atomicMax(row + 1, r[1]);
    atomicMin(row + 2, r[2]); atomicMin(row + 3, r[3]);
    if (r[4]) atomicAdd(row + 4, r[4]);
    if (r[5]) atomicAdd(row + 5, r[5]);
    if (r[6]) atomicAdd(row + 6, r[6]);
  }
}

// One warp per front: the 12 features, the network, the route.
__global__ void k_mlp_route(const int32_t* ids, int n, const DFront* F, const float* P, float thresh, int force_fp64,
                            unsigned* feat, int32_t* route_out) {
  __shared__ MlpAct act;
  __shared__ float fx[MLP_IN];
  const int i = blockIdx.x, lane = threadIdx.x;
  if (i >= n) return;
  const int s = ids[i];
  const DFront f = F[s];
  unsigned* row = feat + (size_t)s * FEAT_STRIDE;
  if (lane == 0) {
    const float lo = 1e-30f;
    const float mx = fmaxf(__uint_as_float(row[0]), lo);
    const float k = (float)max(f.k, 1), m = (float)max(f.m, 1);
    fx[0] = log2f(m);
    fx[1] = log2f(k);
    fx[2] = k / m;
    fx[3] = log2f(1.f + (float)f.ndin);
    fx[4] = (float)f.ndin / k;
    fx[5] = log10f(mx);
    fx[6] = log10f(fmaxf(__uint_as_float(row[1]) / mx, lo));
    fx[7] = log10f(fmaxf(__uint_as_float(row[2]) / mx, lo));
    fx[8] = log10f(fminf(fmaxf(__uint_as_float(row[3]), lo), 1e10f));
    fx[9] = (float)row[4] / k;
    fx[10] = (float)row[5] / k;
    fx[11] = (float)row[6] / k;
  }
  __syncwarp();
  const float xin = lane < MLP_IN ? fx[lane] : 0.f;
  const float z = mlp_forward_warp(P, xin, act);
  if (lane < MLP_IN) row[8 + lane] = __float_as_uint(fx[lane]);
  if (lane == 0) {
    const float pr = mlp_sigmoid(z);
    const int r = (!force_fp64 && pr >= thresh) ? 1 : 0;
    row[20] = __float_as_uint(pr);
    row[21] = __float_as_uint((float)r);
    route_out[i] = r;
  }
}

// After the wave's factorization: max |D| of each large front; a front that
// took the mixed form and whose max |D| exceeds bound * max |a| raises flag.
__global__ void k_front_growth(const int32_t* ids, const DFront* F, Arenas A, double bound, unsigned* feat,
                               int32_t* flag, int32_t* route) {
  const int s = ids[blockIdx.x];
  const DFront f = F[s];
  __shared__ double sm[8];
  double mx = 0.0;
  for (int c = threadIdx.x; c < f.ne; c += blockDim.x) {
    const int64_t q = f.dpos + c;
    mx = fmax(mx, A.dtype[q] == PT_2X2 ? fmax(fabs(A.ddiag[q]), fabs(A.doff[q])) : fabs(A.ddiag[q]));
  }
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = mx;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) mx = fmax(mx, sm[w]);
    unsigned* row = feat + (size_t)s * FEAT_STRIDE;
    row[7] = fbits(mx);
    const double amax = (double)__uint_as_float(row[0]);
    if (__uint_as_float(row[21]) == 1.f && mx > bound * amax) {
      atomicAdd(flag, 1);
      route[blockIdx.x] = 2;  // refactored in FP64 once the wave is done
    }
  }
}

}  // namespace rvg

using namespace rvg;

// One large front in flight: the stream its launches go to, its pivot state
// on the device and the packed window of its mixed-form updates.  Context 0
// is the handle's own stream; the others let the large fronts of one wave run
// side by side (one host thread each).
constexpr int LF_AHEAD = 8;  // outer blocks of a large front issued ahead of the host's check of their start
struct LfCtx {
  cudaStream_t st = nullptr;
  LFState* lf = nullptr;
  float* wpack = nullptr; size_t wpack_cap = 0;
  bool own = false;        // stream and state created for this context
  bool marks = false;      // profiling marks (only one front in flight, on the handle's stream)
  int64_t launches = 0;
  double sync_ms = 0, syrk_flops = 0;
  // issue-ahead of outer blocks: the device's eliminated total after each
  // issued block lands in a pinned slot, with an event behind it
  int32_t* h_gne = nullptr;
  cudaEvent_t ring_ev[LF_AHEAD] = {};
  double wait_ms = 0;     // host waits on blocks issued ahead (the stream still holds later blocks)
  int64_t misses = 0;     // blocks issued for a start column the factorization did not reach
  // far-field part of a full window's update, beside the next outer blocks (mixed form)
  cudaStream_t far_st = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_far = nullptr;
  int64_t far_launches = 0;
  int id = 0;  // position in the handle's contexts (its window buffer's address-stable arena)
};
// A full window's far field (the columns after the next window's blocks but
// its last) is updated on a second stream while those blocks are factored;
// the GEMM leaves LF_FAR_SMS multiprocessors to their latency-bound kernels.
constexpr int LF_FAR_SMS = 24;  // the default of rvg_options::far_field_sms
constexpr int LF_CONCURRENT = 8;  // large fronts of a wave in flight at once

struct VmArenas;

struct rvg_handle {
  Plan P;
  rvg_options opt;
  VmArenas* vm = nullptr;  // address-stable arenas (graph_refactor = 2), else nullptr
  int device = 0;
  cudaStream_t st = nullptr;
  cudaEvent_t ev[8] = {};
  int64_t nnz = 0;
  // static device data
  int64_t *d_own_ptr = nullptr, *d_pat_ptr = nullptr, *d_amap_ptr = nullptr, *d_ea_ptr = nullptr, *d_ch_ptr = nullptr;
  int32_t *d_own_idx = nullptr, *d_pat_idx = nullptr, *d_amap = nullptr, *d_ea_map = nullptr, *d_ch_idx = nullptr;
  int64_t* d_pfwd = nullptr;
  // per-factor device data
  DFront* d_fronts = nullptr;
  std::vector<DFront> h_fronts;
  double* panel = nullptr; size_t panel_cap = 0;
  int32_t* idx = nullptr; size_t idx_cap = 0;
  int8_t* dtype = nullptr; double* ddiag = nullptr; double* doff = nullptr; size_t d_cap = 0;
  double* d_vals = nullptr; double* d_scal = nullptr; bool has_scaling = false;
  double* d_x = nullptr; size_t x_cap = 0;
  double* solve_work = nullptr; size_t solve_work_cap = 0;
  char* d_stage = nullptr; size_t stage_cap = 0;   // per-wave packed launch data
  char* h_stage = nullptr; size_t h_stage_cap = 0; // pinned host mirror
  int32_t* h_counts = nullptr; size_t h_counts_cap = 0;
  LFState* d_lf = nullptr;                          // state of the large-front path
  std::vector<LfCtx> lfx;                            // concurrent large-front contexts 1.. (0 = the handle's)
  int64_t* d_colptr = nullptr;                      // matrix pattern (full symmetric CSC = its own CSR)
  int32_t* d_rowidx = nullptr;
  double a_fro = 0;                                 // ||A||_F of the last factored values
  double* d_ref = nullptr; size_t ref_cap = 0;      // refinement vectors r, d, b (3n) and norms
  double* d_gm = nullptr; size_t gm_cap = 0;        // GMRES-IR: Krylov basis, preconditioned basis, work
  double* h_norms = nullptr;
  char* h_norms_m = nullptr; size_t h_norms_m_cap = 0;  // pinned per-column norms of the refinement
  double* scratch = nullptr; size_t scratch_cap = 0; // per-wave scratch, persistent across factors
  double* cb_arena = nullptr; size_t cb_cap = 0;     // contribution blocks, first-fit by wave
  float* pack = nullptr; size_t pack_cap = 0;        // TF32 hi/lo operand tiles of the mixed-form updates
  float* wpack = nullptr; size_t wpack_cap = 0;      // the same for a large front's window of pending columns
  int32_t* d_err = nullptr;                          // set by a device wait that timed out
  int32_t* sf_sync = nullptr; size_t sf_sync_cap = 0; // solve: ticket counter and block flags of one wave
  double* sf_part = nullptr; size_t sf_part_cap = 0;   // backward solve: partial sums of one wave
  int nsm = 0;                                       // SMs of the device (persistent grids)
  bool chain_pdl = true;                             // large-front chain kernels by programmatic dependent launch
  std::map<int64_t, int64_t> cb_free;                // offset -> length of the free ranges
  bool factored = false;
  bool need_presize = false;                         // arenas released by rvg_trim
  // refactorization replay (graph_refactor): the host's decisions in the last dynamic factorization
  bool rec_ok = false;                               // a complete record is available
  std::vector<int32_t> rec_cnt;                      // per front: eliminated, 1x1 and 2x2 counts
  std::vector<std::vector<int32_t>> rec_g;           // per large front: eliminated count after each outer block
  std::vector<size_t> rec_stage;                     // per wave: bytes of the packed launch data
  int64_t rec_d_used = 0;                            // D entries used
  bool replay = false;                               // run_factor is being captured into the graph
  int32_t* d_rec = nullptr; size_t d_rec_cap = 0;    // rec_cnt on the device (for the checks)
  int32_t* d_mismatch = nullptr;                     // set by a check that sees another decision
  char* h_stage_all = nullptr; size_t h_stage_all_cap = 0;  // pinned launch data of every wave (replay)
  std::vector<size_t> stage_off;                     // per wave: its offset in h_stage_all
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
  const double* graph_ds = nullptr;                  // the scaling pointer the graph reads
  // learned precision (precision = 2)
  float* d_sel = nullptr;                            // selector parameters (MLP_NPARAM floats)
  float sel_thresh = 0.5f;                           // probability at or above which a front takes the mixed form
  double sel_bound = 1e6;                            // growth bound: max |D| <= bound * max |a| for a mixed front
  unsigned* d_feat = nullptr; size_t d_feat_cap = 0; // feature table, FEAT_STRIDE words per front
  int32_t* d_sel_flag = nullptr;                     // mixed fronts over the growth bound in the last run
  std::vector<int8_t> route;                         // per front: 1 = mixed form (decided on the device)
  std::vector<int32_t> sel_large;                    // the large fronts of the last factorization
  bool sel_force_fp64 = false;                       // the FP64 refactorization after a growth flag
  int aptp_ctas = 0;                                 // resident CTAs of the medium fronts' queue kernel
  int32_t* d_nonfinite = nullptr;                    // set when the values or the scaling hold NaN or Inf
  int64_t sel_routed = 0, sel_flagged = 0, sel_fallback = 0;
  // measurement
  bool profiling = false;
  std::vector<cudaEvent_t> ev_pool;
  size_t ev_used = 0;
  double syrk_flops = 0, syrk_ms = 0;
  std::vector<cudaEvent_t> mk_pool;                  // per-kind marks (profiling): event, kind
  std::vector<int> mk_kind;
  size_t mk_used = 0;
  double part_ms[RVG_PARTS] = {};
  int64_t syrk_launches = 0, launches = 0, factor_launches = 0, solve_launches = 0;
  int64_t arena_bytes = 0, peak_bytes = 0;
  double host_alloc_ms = 0, host_sync_ms = 0, host_total_ms = 0;
  double host_wait_ms = 0;  // waits on large-front blocks issued ahead (later blocks still queued)
  double host_gap_ms = 0;   // host time between a wave's synchronisation and the next wave's first launch
  bool sf_attr = false;     // the backward solve kernels' shared-memory limit raised
  char* d_stage2 = nullptr; size_t stage2_cap = 0;  // launch data of FP64 refactorizations of single fronts
  char* h_stage2 = nullptr; size_t h_stage2_cap = 0;
  int64_t sel_refactored = 0;                       // fronts refactored in FP64 after their growth check
  int64_t lf_misses = 0;    // large-front blocks issued past a delay (returned at once, issued again)
  int64_t lf_far = 0;       // far-field window updates run on a large front's second stream
  // results
  int64_t tot1 = 0, tot2 = 0, totdel = 0, zero_piv = 0, max_front = 0;
  double t_assembly = 0, t_kernel = 0, t_gemm = 0, t_factor = 0, t_solve = 0, t_dom = 0, n_dom = 0;
};

namespace {

double now_ms() {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// Profiling marks: the time between a mark and the one before it is charged
// to the later mark's kind (a kind < 0 starts a new segment).  Read back
// after each stream synchronisation.
void mark(rvg_handle* h, int kind) {
  if (!h->profiling || h->replay) return;
  if (h->mk_used == h->mk_pool.size()) {
    cudaEvent_t e;
    if (cudaEventCreate(&e) != cudaSuccess) return;
    h->mk_pool.push_back(e);
    h->mk_kind.push_back(-1);
  }
  cudaEventRecord(h->mk_pool[h->mk_used], h->st);
  h->mk_kind[h->mk_used++] = kind;
}
void mark_flush(rvg_handle* h) {
  for (size_t i = 1; i < h->mk_used; ++i) {
    float ms = 0;
    if (h->mk_kind[i] >= 0 && cudaEventElapsedTime(&ms, h->mk_pool[i - 1], h->mk_pool[i]) == cudaSuccess)
      h->part_ms[h->mk_kind[i]] += ms;
  }
  h->mk_used = 0;
}

// Set while a refactorization graph is captured: every buffer must already be
// large enough (the capture replays the sizes of the last factorization), so a
// growth request aborts the capture and the factorization runs dynamically.
thread_local bool tl_no_alloc = false;
static int no_alloc_fail() {
  set_error("refactorization replay would allocate");
  return RVG_ERR_DEVICE;
}

template <class T>
int ensure(T*& p, size_t& cap, size_t need, cudaStream_t st) {
  if (need <= cap && p) return RVG_OK;
  if (tl_no_alloc) return no_alloc_fail();
  size_t nc = std::max(need, cap + cap / 2);
  if (nc == 0) nc = 1;
  T* np = nullptr;
  CK(cudaMallocAsync((void**)&np, nc * sizeof(T), st));
  if (p) {
    if (cap) CK(cudaMemcpyAsync(np, p, cap * sizeof(T), cudaMemcpyDeviceToDevice, st));
    CK(cudaFreeAsync(p, st));
  }
  p = np;
  cap = nc;
  return RVG_OK;
}

int ensure_host(char*& p, size_t& cap, size_t need) {
  if (need <= cap && p) return RVG_OK;
  if (tl_no_alloc) return no_alloc_fail();
  size_t nc = std::max(need, cap + cap / 2);
  if (p) CK(cudaFreeHost(p));
  p = nullptr;
  CK(cudaMallocHost((void**)&p, nc));
  cap = nc;
  return RVG_OK;
}

int vm_d_arrays(rvg_handle* h, size_t need);
int ensure_d_arrays(rvg_handle* h, size_t need) {  // type / diag / off share one capacity
  if (h->vm) return vm_d_arrays(h, need);
  if (need <= h->d_cap && h->dtype) return RVG_OK;
  if (tl_no_alloc) return no_alloc_fail();
  size_t nc = std::max(need, h->d_cap + h->d_cap / 2);
  int8_t* t; double *a, *b;
  CK(cudaMallocAsync((void**)&t, nc, h->st));
  CK(cudaMallocAsync((void**)&a, nc * 8, h->st));
  CK(cudaMallocAsync((void**)&b, nc * 8, h->st));
  if (h->dtype) {
    CK(cudaMemcpyAsync(t, h->dtype, h->d_cap, cudaMemcpyDeviceToDevice, h->st));
    CK(cudaMemcpyAsync(a, h->ddiag, h->d_cap * 8, cudaMemcpyDeviceToDevice, h->st));
    CK(cudaMemcpyAsync(b, h->doff, h->d_cap * 8, cudaMemcpyDeviceToDevice, h->st));
    CK(cudaFreeAsync(h->dtype, h->st)); CK(cudaFreeAsync(h->ddiag, h->st)); CK(cudaFreeAsync(h->doff, h->st));
  }
  h->dtype = t; h->ddiag = a; h->doff = b; h->d_cap = nc;
  return RVG_OK;
}

template <class T>
int ensure_nocopy(T*& p, size_t& cap, size_t need, cudaStream_t st) {
  if (need <= cap && p) return RVG_OK;
  if (tl_no_alloc) return no_alloc_fail();
  size_t nc = std::max(need, cap + cap / 4);
  if (nc == 0) nc = 1;
  if (p) CK(cudaFreeAsync(p, st));
  p = nullptr;
  CK(cudaMallocAsync((void**)&p, nc * sizeof(T), st));
  cap = nc;
  return RVG_OK;
}

// ---------------------------------------------------------------------------
// Address-stable arenas (graph_refactor = 2).  A captured refactorization
// graph holds the addresses of the factorization's arenas, and rvg_trim
// releases their memory so that many handles can take turns on one device.
// In this mode each arena is a range of virtual addresses reserved once for
// the handle's life (as large as the device's memory); physical memory is
// mapped into it in chunks as the arena grows (contents and address kept),
// unmapped by rvg_trim, and mapped again by the next factorization up to the
// largest size the arena reached, so the graph's addresses stay valid.
enum VmSlotId {
  VM_PANEL = 0, VM_IDX, VM_DTYPE, VM_DDIAG, VM_DOFF, VM_SCRATCH, VM_CB, VM_PACK, VM_STAGE,
  VM_WPACK0,  // + context id
  VM_NSLOTS = VM_WPACK0 + LF_CONCURRENT
};
}  // namespace (the arenas' types complete the handle's forward declaration, at file scope)
struct VmSlot {
  CUdeviceptr va = 0;
  size_t reserved = 0, mapped = 0, high = 0;
  std::vector<std::pair<size_t, CUmemGenericAllocationHandle>> chunks;  // (bytes, physical memory) from va on
};
struct VmArenas {
  size_t gran = 0, reserve = 0;  // reserve: the device's memory, the most any range grows to
  CUmemAllocationProp prop = {};
  CUmemAccessDesc access = {};
  VmSlot slot[VM_NSLOTS];
};
namespace {

// The driver's virtual-memory calls, looked up through the runtime
// (cudaGetDriverEntryPoint) so that the library does not link the driver
// library itself and still loads on a machine without one.
struct VmApi {
  decltype(&cuGetErrorString) err = nullptr;
  decltype(&cuMemGetAllocationGranularity) gran = nullptr;
  decltype(&cuMemAddressReserve) reserve = nullptr;
  decltype(&cuMemAddressFree) free = nullptr;
  decltype(&cuMemCreate) create = nullptr;
  decltype(&cuMemRelease) release = nullptr;
  decltype(&cuMemMap) map = nullptr;
  decltype(&cuMemUnmap) unmap = nullptr;
  decltype(&cuMemSetAccess) access = nullptr;
};
VmApi g_vm;

int vm_api() {
  if (g_vm.access) return RVG_OK;
  VmApi a;
  bool ok = true;
  auto get = [&](const char* name, auto& fp) {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint(name, &f, cudaEnableDefault, &q) != cudaSuccess || q != cudaDriverEntryPointSuccess ||
        !f)
      ok = false;
    fp = reinterpret_cast<std::remove_reference_t<decltype(fp)>>(f);
  };
  get("cuGetErrorString", a.err);
  get("cuMemGetAllocationGranularity", a.gran);
  get("cuMemAddressReserve", a.reserve);
  get("cuMemAddressFree", a.free);
  get("cuMemCreate", a.create);
  get("cuMemRelease", a.release);
  get("cuMemMap", a.map);
  get("cuMemUnmap", a.unmap);
  get("cuMemSetAccess", a.access);
  if (!ok) {
    cudaGetLastError();
    set_error("the driver's virtual-memory calls are not available (graph_refactor = 2)");
    return RVG_ERR_DEVICE;
  }
  g_vm = a;
  return RVG_OK;
}

int cu_fail(CUresult r, const char* what) {
  const char* msg = nullptr;
  if (g_vm.err) g_vm.err(r, &msg);
  set_error(std::string("CUDA driver error: ") + (msg ? msg : "unknown") + " at " + what);
  return r == CUDA_ERROR_OUT_OF_MEMORY ? RVG_ERR_OUT_OF_MEMORY : RVG_ERR_DEVICE;
}
#define CU(x)                                  \
  do {                                         \
    const CUresult cu_r_ = (x);                \
    if (cu_r_ != CUDA_SUCCESS) return cu_fail(cu_r_, #x); \
  } while (0)

int vm_create(rvg_handle* h) {
  if (int rc = vm_api()) return rc;
  std::unique_ptr<VmArenas> v(new VmArenas);
  v->prop.type = CU_MEM_ALLOCATION_TYPE_PINNED;
  v->prop.location.type = CU_MEM_LOCATION_TYPE_DEVICE;
  v->prop.location.id = h->device;
  CU(g_vm.gran(&v->gran, &v->prop, CU_MEM_ALLOC_GRANULARITY_RECOMMENDED));
  size_t fr = 0, tot = 0;
  CK(cudaMemGetInfo(&fr, &tot));
  v->reserve = (tot + v->gran - 1) / v->gran * v->gran;
  v->access.location = v->prop.location;
  v->access.flags = CU_MEM_ACCESS_FLAGS_PROT_READWRITE;
  h->vm = v.release();
  return RVG_OK;
}

void vm_unmap(VmSlot& s);

// backs at least `bytes` of slot `id` (at least its largest earlier size).
// A range is reserved at four times its first size (256 MB at least); one that
// must grow past its reservation moves to a larger one (contents copied, the
// replay graph dropped: it held the old addresses).
int vm_map(rvg_handle* h, int id, size_t bytes) {
  VmArenas* v = h->vm;
  VmSlot& s = v->slot[id];
  const size_t want = std::max((bytes + v->gran - 1) / v->gran * v->gran, s.high);
  if (want <= s.mapped) return RVG_OK;
  if (want > v->reserve) {
    set_error("an arena would exceed the device's memory");
    return RVG_ERR_OUT_OF_MEMORY;
  }
  if (!s.va || want > s.reserved) {
    const size_t r = std::min(v->reserve, std::max<size_t>(4 * want, (size_t)256 << 20) / v->gran * v->gran);
    CUdeviceptr nva = 0;
    CU(g_vm.reserve(&nva, r, v->gran, 0, 0));
    if (s.va) {  // move: map the new range, copy what the old one held, release the old one
      VmSlot old = s;
      s = VmSlot();
      s.va = nva;
      s.reserved = r;
      int rc = vm_map(h, id, old.mapped);
      if (rc) {  // the old range stays the arena; the new one goes
        vm_unmap(s);
        g_vm.free(nva, r);
        s = old;
        return rc;
      }
      CK(cudaDeviceSynchronize());
      CK(cudaMemcpy((void*)s.va, (const void*)old.va, old.mapped, cudaMemcpyDeviceToDevice));
      vm_unmap(old);
      g_vm.free(old.va, old.reserved);
      s.high = std::max(s.high, old.high);
      if (h->gexec) cudaGraphExecDestroy(h->gexec);  // the replay graph held the old addresses
      if (h->graph) cudaGraphDestroy(h->graph);
      h->gexec = nullptr;
      h->graph = nullptr;
    } else {
      s.va = nva;
      s.reserved = r;
    }
  }
  size_t add = std::max(want - s.mapped, (s.mapped / 4 + v->gran - 1) / v->gran * v->gran);  // fewer, larger chunks
  add = std::min(add, s.reserved - s.mapped);
  CUmemGenericAllocationHandle m = 0;
  CUresult r = g_vm.create(&m, add, &v->prop, 0);
  if (r == CUDA_ERROR_OUT_OF_MEMORY) {  // memory kept by the stream-ordered pool: hand it back, try again
    cudaDeviceSynchronize();
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, h->device) == cudaSuccess) cudaMemPoolTrimTo(pool, 0);
    r = g_vm.create(&m, add, &v->prop, 0);
  }
  if (r != CUDA_SUCCESS) return cu_fail(r, "cuMemCreate");
  r = g_vm.map(s.va + s.mapped, add, 0, m, 0);
  if (r != CUDA_SUCCESS) {
    g_vm.release(m);
    return cu_fail(r, "cuMemMap");
  }
  r = g_vm.access(s.va + s.mapped, add, &v->access, 1);
  if (r != CUDA_SUCCESS) {
    g_vm.unmap(s.va + s.mapped, add);
    g_vm.release(m);
    return cu_fail(r, "cuMemSetAccess");
  }
  s.chunks.emplace_back(add, m);
  s.mapped += add;
  s.high = std::max(s.high, s.mapped);
  return RVG_OK;
}

// releases a slot's physical memory, keeping its addresses (the device must
// be done with it: the callers synchronise the device first)
void vm_unmap(VmSlot& s) {
  size_t off = 0;
  for (auto& c : s.chunks) {
    g_vm.unmap(s.va + off, c.first);
    g_vm.release(c.second);
    off += c.first;
  }
  s.chunks.clear();
  s.mapped = 0;
}

void vm_destroy(rvg_handle* h) {
  if (!h->vm) return;
  cudaDeviceSynchronize();
  for (VmSlot& s : h->vm->slot) {
    vm_unmap(s);
    if (s.va) g_vm.free(s.va, s.reserved);
  }
  delete h->vm;
  h->vm = nullptr;
}

// The arena of slot `id` with room for `need` elements: address-stable in the
// graph_refactor = 2 mode (growth maps more memory behind the contents), else
// ensure()'s stream-ordered reallocation (`copy`: the contents move along).
template <class T>
int arena_ensure(rvg_handle* h, int id, T*& p, size_t& cap, size_t need, cudaStream_t st, bool copy) {
  if (!h->vm) return copy ? ensure(p, cap, need, st) : ensure_nocopy(p, cap, need, st);
  if (need <= cap && p) return RVG_OK;
  if (tl_no_alloc) return no_alloc_fail();
  int rc = vm_map(h, id, std::max<size_t>(need, 1) * sizeof(T));
  if (rc) return rc;
  p = reinterpret_cast<T*>(h->vm->slot[id].va);
  cap = h->vm->slot[id].mapped / sizeof(T);
  return RVG_OK;
}

// Every arena mapped again up to its largest size and bound to its pointer:
// a replayed graph touches them all without the host's ensure calls.
int vm_restore(rvg_handle* h) {
  for (int id = 0; id < VM_NSLOTS; ++id) {
    VmSlot& sl = h->vm->slot[id];
    if (sl.high > sl.mapped) {
      int rc = vm_map(h, id, sl.high);
      if (rc) return rc;
    }
  }
  auto bind = [&](int id, auto*& p, size_t& cap) {
    const VmSlot& sl = h->vm->slot[id];
    if (sl.mapped && !p) {
      p = reinterpret_cast<std::remove_reference_t<decltype(p)>>(sl.va);
      cap = sl.mapped / sizeof(*p);
    }
  };
  bind(VM_PANEL, h->panel, h->panel_cap);
  bind(VM_IDX, h->idx, h->idx_cap);
  bind(VM_SCRATCH, h->scratch, h->scratch_cap);
  bind(VM_CB, h->cb_arena, h->cb_cap);
  bind(VM_PACK, h->pack, h->pack_cap);
  bind(VM_STAGE, h->d_stage, h->stage_cap);
  bind(VM_WPACK0, h->wpack, h->wpack_cap);
  for (size_t t = 1; t < h->lfx.size(); ++t) bind(VM_WPACK0 + (int)t, h->lfx[t].wpack, h->lfx[t].wpack_cap);
  if (!h->dtype && h->vm->slot[VM_DTYPE].mapped) {
    size_t ct = 0, ca = 0, cb = 0;
    bind(VM_DTYPE, h->dtype, ct);
    bind(VM_DDIAG, h->ddiag, ca);
    bind(VM_DOFF, h->doff, cb);
    h->d_cap = std::min(ct, std::min(ca, cb));
  }
  return RVG_OK;
}

int vm_d_arrays(rvg_handle* h, size_t need) {
  if (need <= h->d_cap && h->dtype) return RVG_OK;
  if (tl_no_alloc) return no_alloc_fail();
  size_t ct = 0, ca = 0, cb = 0;
  int rc;
  if ((rc = arena_ensure(h, VM_DTYPE, h->dtype, ct, need, h->st, true)) ||
      (rc = arena_ensure(h, VM_DDIAG, h->ddiag, ca, need, h->st, true)) ||
      (rc = arena_ensure(h, VM_DOFF, h->doff, cb, need, h->st, true)))
    return rc;
  h->d_cap = std::min(ct, std::min(ca, cb));
  return RVG_OK;
}

// first-fit allocation of `len` doubles in the CB arena; grows (with a copy of
// the live contents) when no free range fits
int cb_alloc(rvg_handle* h, int64_t len, int64_t* off) {
  for (auto it = h->cb_free.begin(); it != h->cb_free.end(); ++it) {
    if (it->second >= len) {
      *off = it->first;
      int64_t rest = it->second - len, start = it->first + len;
      h->cb_free.erase(it);
      if (rest > 0) h->cb_free[start] = rest;
      return RVG_OK;
    }
  }
  if (tl_no_alloc) return no_alloc_fail();
  // grow: new capacity covers the old one plus the request
  size_t old = h->cb_cap;
  size_t nc = std::max(old + (size_t)len, old + old / 4);
  if (h->vm) {  // more memory behind the same addresses
    size_t cap = old;
    int rc = arena_ensure(h, VM_CB, h->cb_arena, cap, nc, h->st, true);
    if (rc) return rc;
    nc = cap;
  } else {
    double* np = nullptr;
    CK(cudaMallocAsync((void**)&np, nc * sizeof(double), h->st));
    if (h->cb_arena) {
      if (old) CK(cudaMemcpyAsync(np, h->cb_arena, old * sizeof(double), cudaMemcpyDeviceToDevice, h->st));
      CK(cudaFreeAsync(h->cb_arena, h->st));
    }
    h->cb_arena = np;
  }
  h->cb_cap = nc;
  // the tail [old, nc) is free; merge with a free range ending at `old`
  int64_t start = (int64_t)old, length = (int64_t)(nc - old);
  auto it = h->cb_free.lower_bound(start);
  if (it != h->cb_free.begin()) {
    auto pv = std::prev(it);
    if (pv->first + pv->second == start) { start = pv->first; length += pv->second; h->cb_free.erase(pv); }
  }
  h->cb_free[start] = length;
  return cb_alloc(h, len, off);
}

void cb_release(rvg_handle* h, int64_t off, int64_t len) {
  if (len <= 0) return;
  auto it = h->cb_free.emplace(off, len).first;
  auto nx = std::next(it);
  if (nx != h->cb_free.end() && it->first + it->second == nx->first) { it->second += nx->second; h->cb_free.erase(nx); }
  if (it != h->cb_free.begin()) {
    auto pv = std::prev(it);
    if (pv->first + pv->second == it->first) { pv->second += it->second; h->cb_free.erase(it); }
  }
}

template <class T>
int upload(T*& d, const std::vector<T>& h, cudaStream_t st) {
  size_t n = std::max<size_t>(h.size(), 1);
  CK(cudaMallocAsync((void**)&d, n * sizeof(T), st));
  if (!h.empty()) CK(cudaMemcpyAsync(d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, st));
  return RVG_OK;
}

// Packs the typed arrays of one wave into one buffer (16-byte aligned
// sections) so the whole wave is a single host->device copy.
struct Packer {
  std::vector<char> buf;
  template <class T>
  size_t add(const std::vector<T>& v) {
    size_t off = (buf.size() + 15) & ~size_t(15);
    buf.resize(off + v.size() * sizeof(T));
    if (!v.empty()) std::memcpy(buf.data() + off, v.data(), v.size() * sizeof(T));
    return off;
  }
};

Statics statics(rvg_handle* h) {
  return Statics{h->d_own_ptr, h->d_own_idx, h->d_pat_ptr, h->d_pat_idx, h->d_amap_ptr,
                 h->d_amap, h->d_ea_ptr, h->d_ea_map, h->d_ch_ptr, h->d_ch_idx};
}

DevOpts devopts(const rvg_options& o) {
  return DevOpts{o.threshold, o.small, (int)o.outer_block_size, (int)o.inner_block_size, o.failed_pivot_tpp};
}

unsigned blocks_for(size_t n, unsigned t) { return (unsigned)((n + t - 1) / t); }

// Columns of the pending window of a large front's deferred updates: LF_WINDOW
// outer blocks, or rvg_options::mixed_window of them in the mixed form (a full
// window's update reads and writes every trailing entry once in FP64 for K =
// window columns of BF16 or TF32 products: at K = 1024 that C stream already
// asks for most of the HBM bandwidth at the tensor cores' rate, so a deeper
// window is faster, and less accurate), except in the mixed form when the
// outer block is not a whole number of 128-row tiles (its packed operands are
// appended tile- and chunk-aligned): then one block (every block's update
// applied at once).
constexpr int64_t LF_WINDOW = 4;
constexpr int64_t LF_WINDOW_MAX = 8;
int64_t lf_mixed_window(const rvg_handle* h) { return h->opt.mixed_window > 0 ? h->opt.mixed_window : LF_WINDOW; }
int64_t lf_window_cols(const rvg_handle* h, int64_t nb, bool mixed) {
  return !mixed ? LF_WINDOW * nb : (nb % 128 == 0 ? lf_mixed_window(h) * nb : nb);
}
// outer blocks of window storage a large front's scratch holds (any front of the handle may take the mixed
// form unless the precision is plain FP64)
int64_t lf_window_blocks(const rvg_handle* h) {
  return h->opt.precision == 0 ? LF_WINDOW : std::max(LF_WINDOW, lf_mixed_window(h));
}

// Which fronts of a wave take the multi-kernel path (the whole GPU, one front
// after another) instead of one CTA each: every front of order >= T, and
// those of order >= T / 2 when the wave holds at most LF_FEW of them (a few
// such fronts leave most SMs idle on the CTA path; many keep them busy).
// Results do not depend on the choice: both paths perform the same
// arithmetic.  mid = the wave's count of non-TPP fronts with T/2 <= m < T.
constexpr int64_t LF_FEW = 16;
inline bool front_is_large(int64_t m, bool tpp, int64_t T, int64_t mid) {
  return !tpp && (m >= T || (m >= T / 2 && mid <= LF_FEW));
}

// Arena sizes of the delay-free schedule, computed from the pattern alone
// (delays can only add to them; the arenas grow in that case).
int presize_arenas(rvg_handle* h) {
  Plan& P = h->P;
  const int64_t nb = h->opt.outer_block_size, ib = h->opt.inner_block_size;
  int64_t panel = 0, idx = 0, dsz = 0, scratch = 0;
  std::vector<int64_t> cbw(P.waves.size(), 0), rel(P.waves.size(), -1);
  const int64_t T = h->opt.large_front_threshold;
  for (size_t w = 0; w < P.waves.size(); ++w) {
    int64_t sc_w = 0, mid = 0;
    for (int64_t s : P.waves[w]) {
      const Snode& x = P.sn[s];
      const int64_t k = x.n_owned(), m = k + (int64_t)x.pattern.size();
      if (!(x.in_small_leaf || k < ib) && m >= T / 2 && m < T) ++mid;
    }
    for (int64_t s : P.waves[w]) {
      const Snode& x = P.sn[s];
      int64_t k = x.n_owned(), nfs = (int64_t)x.pattern.size(), m = k + nfs;
      panel += m * k;
      idx += m + k;
      dsz += k;
      bool has_cb = x.parent >= 0 && nfs > 0;
      if (has_cb) cbw[w] += nfs * nfs;
      bool tpp = x.in_small_leaf || k < ib;
      bool large = front_is_large(m, tpp, T, mid);
      int64_t sc = tpp ? 0 : (2 * IBMAX * m + nb);
      if (large) sc = m * (2 * IBMAX + lf_window_blocks(h) * nb) + nb;
      if (has_cb) sc = std::max<int64_t>(sc, nfs * k);
      sc_w += sc;
      if (x.parent >= 0) rel[w] = std::max<int64_t>(rel[w], P.height[x.parent]);
    }
    scratch = std::max(scratch, sc_w);
  }
  // first-fit simulation of the contribution arena
  std::map<int64_t, int64_t> fr;
  int64_t hw = 0;
  std::vector<int64_t> off(P.waves.size(), -1);
  auto sim_free = [&](int64_t o, int64_t l) {
    auto it = fr.emplace(o, l).first;
    auto nx = std::next(it);
    if (nx != fr.end() && it->first + it->second == nx->first) { it->second += nx->second; fr.erase(nx); }
    if (it != fr.begin()) {
      auto pv = std::prev(it);
      if (pv->first + pv->second == it->first) { pv->second += it->second; fr.erase(it); }
    }
  };
  for (size_t w = 0; w < P.waves.size(); ++w) {
    // same order as run_factor: this wave's block is allocated before the
    // blocks its assembly consumed are released
    if (w > 0)
      for (size_t w2 = 0; w2 + 1 < w; ++w2)
        if (off[w2] >= 0 && rel[w2] == (int64_t)(w - 1)) { sim_free(off[w2], cbw[w2]); off[w2] = -1; }
    if (!cbw[w]) continue;
    bool placed = false;
    for (auto it = fr.begin(); it != fr.end(); ++it)
      if (it->second >= cbw[w]) {
        off[w] = it->first;
        int64_t rest = it->second - cbw[w], st = it->first + cbw[w];
        fr.erase(it);
        if (rest > 0) fr[st] = rest;
        placed = true;
        break;
      }
    if (!placed) {
      // extend at the end (merging a free tail)
      int64_t start = hw;
      auto it = fr.end();
      if (!fr.empty()) {
        auto last = std::prev(it);
        if (last->first + last->second == hw) { start = last->first; fr.erase(last); }
      }
      off[w] = start;
      hw = start + cbw[w];
    }
  }
  int rc;
  cudaStream_t st = h->st;
  if ((rc = arena_ensure(h, VM_PANEL, h->panel, h->panel_cap, (size_t)(panel + panel / 16 + 1024), st, true)))
    return rc;
  if ((rc = arena_ensure(h, VM_IDX, h->idx, h->idx_cap, (size_t)(idx + idx / 16 + 1024), st, true))) return rc;
  if ((rc = ensure_d_arrays(h, (size_t)(dsz + dsz / 8 + 1024)))) return rc;
  if ((rc = arena_ensure(h, VM_SCRATCH, h->scratch, h->scratch_cap, (size_t)(scratch + 1024), st, false)))
    return rc;
  if (hw > 0 && !h->cb_arena) {
    const size_t want = (size_t)(hw + hw / 16 + 1024);
    if (h->vm) {
      size_t cap = 0;
      if ((rc = arena_ensure(h, VM_CB, h->cb_arena, cap, want, st, false))) return rc;
      h->cb_cap = cap;
    } else {
      h->cb_cap = want;
      CK(cudaMallocAsync((void**)&h->cb_arena, h->cb_cap * sizeof(double), st));
    }
  }
  return RVG_OK;
}

double lower_entries(int64_t r0, int64_t r1, int64_t c0, int64_t c1) {
  double e = 0;
  for (int64_t j = c0; j < c1; ++j) {
    int64_t lo = j > r0 ? j : r0;
    if (r1 > lo) e += (double)(r1 - lo);
  }
  return e;
}

// CUDA events around each Schur GEMM launch (profiling): their sum is the
// GEMM time the measured rate is based on.
int syrk_ev(rvg_handle* h, bool on = true) {
  if (!h->profiling || !on || h->replay) return RVG_OK;
  if (h->ev_used + 1 > h->ev_pool.size()) {
    for (int i = 0; i < 64; ++i) {
      cudaEvent_t e;
      CK(cudaEventCreate(&e));
      h->ev_pool.push_back(e);
    }
  }
  CK(cudaEventRecord(h->ev_pool[h->ev_used++], h->st));
  return RVG_OK;
}

// The tensor-core Schur GEMM over a.ntiles 128 x 128 lower tiles: the flush
// depth picks the k_syrk_tc instance; without flushing, 256-column CTA tiles
// (k_syrk_tc_pair, over column-tile pairs) unless 128 is asked for.
template <int FMT>
static void launch_tc_fmt(rvg_handle* h, cudaStream_t st, TcArgs ta, int max_ctas) {
  const int64_t cap = max_ctas > 0 ? std::min<int64_t>(max_ctas, h->nsm) : h->nsm;
  if (h->opt.mixed_flush == 0 && h->opt.mixed_tile_cols == 256) {
    ta.ntiles = tp_count_tiles(ta.nr, ta.nc, ta.r0, ta.c0);
    const unsigned grid = (unsigned)std::min<int64_t>(ta.ntiles, cap);
    k_syrk_tc_pair<FMT><<<grid, TC_THREADS, TP_SMEM, st>>>(ta);
    return;
  }
  const unsigned grid = (unsigned)std::min<int64_t>(ta.ntiles, cap);
  switch (h->opt.mixed_flush) {
    case 1: k_syrk_tc<1, FMT><<<grid, TC_THREADS, TC_SMEM, st>>>(ta); break;
    case 2: k_syrk_tc<2, FMT><<<grid, TC_THREADS, TC_SMEM, st>>>(ta); break;
    case 4: k_syrk_tc<4, FMT><<<grid, TC_THREADS, TC_SMEM, st>>>(ta); break;
    case 8: k_syrk_tc<8, FMT><<<grid, TC_THREADS, TC_SMEM, st>>>(ta); break;
    default: k_syrk_tc<TC_NO_FLUSH, FMT><<<grid, TC_THREADS, TC_SMEM, st>>>(ta); break;
  }
}
static void launch_tc(rvg_handle* h, cudaStream_t st, TcArgs ta, int max_ctas = 0) {
  if (h->opt.mixed_operands == 1) launch_tc_fmt<TC_BF16>(h, st, ta, max_ctas);
  else launch_tc_fmt<TC_TF32>(h, st, ta, max_ctas);
}
// the operand split of the mixed form (TF32 or BF16 parts)
static void launch_pack(rvg_handle* h, cudaStream_t st, dim3 grid, const PackArgs& pa) {
  if (h->opt.mixed_operands == 1) k_pack_bf16x3<<<grid, 256, 0, st>>>(pa);
  else k_pack_tf32x3<<<grid, 256, 0, st>>>(pa);
}

// The Schur update C -= W L^T (lower) of one contribution block.  kmax bounds
// the device-side K (columns eliminated).
// Whether front s takes the mixed form's tensor-core updates: every large
// front with precision = 1, the selector's choice with precision = 2.
bool front_mixed(const rvg_handle* h, int64_t s) {
  if (h->opt.precision == 1) return true;
  if (h->opt.precision != 2 || h->sel_force_fp64) return false;
  return s >= 0 && s < (int64_t)h->route.size() && h->route[s] != 0;
}

// A kernel of the large-front chain: with programmatic stream serialization
// it may start while the previous kernel of the stream still runs (each chain
// kernel waits for its predecessor in chain_enter() before any memory access),
// which hides the launch gap between the chain's short dependent kernels.
template <typename... KP, typename... AP>
static void launch_chain(const rvg_handle* h, void (*kern)(KP...), dim3 grid, dim3 block, size_t smem,
                         cudaStream_t st, AP... args) {
  if (!h->chain_pdl) {
    kern<<<grid, block, smem, st>>>(args...);
    return;
  }
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  (void)cudaLaunchKernelEx(&cfg, kern, args...);  // a failure stays the thread's last error, checked as for <<<>>>
}

int launch_syrk(rvg_handle* h, const SyrkArgs& ga, int64_t kmax, bool mixed) {
  cudaStream_t st = h->st;
  if (mixed) {
    const int64_t nr = (ga.r1 - ga.r0 + TC_BM - 1) / TC_BM, nc = (ga.c1 - ga.c0 + TC_BN - 1) / TC_BN;
    const int64_t Q = (kmax + TC_BK - 1) / TC_BK;
    const int64_t ntiles = (nr > 0 && nc > 0) ? tc_count_tiles(nr, nc, ga.r0, ga.c0) : 0;
    if (ntiles > 0 && Q > 0) {
      int rc = arena_ensure(h, VM_PACK, h->pack, h->pack_cap, (size_t)(nr + nc) * Q * TC_BLOCK, st, false);
      if (rc) return rc;
      float* pl = h->pack + (size_t)nr * Q * TC_BLOCK;
      PackArgs aw{ga.W, ga.ldw, ga.r1 - ga.r0, Q, ga.Kdev, ga.K, h->pack};
      PackArgs al{ga.L + ga.c0, ga.ldl, ga.c1 - ga.c0, Q, ga.Kdev, ga.K, pl};
      launch_pack(h, st, dim3((unsigned)Q, (unsigned)nr), aw);
      launch_pack(h, st, dim3((unsigned)Q, (unsigned)nc), al);
      TcArgs ta{ga.C, ga.ldc, ga.r0, ga.r1, ga.c0, ga.c1, h->pack, pl, Q, ga.Kdev, ga.K, nr, nc, ntiles, h->d_err};
      if ((rc = syrk_ev(h))) return rc;
      launch_tc(h, st, ta);
      if ((rc = syrk_ev(h))) return rc;
      h->launches += 3;
      h->syrk_launches++;
    }
  } else {
    int rc = syrk_ev(h);
    if (rc) return rc;
    k_syrk_lower<<<syrk_grid(ga), G_T, G_SMEM, st>>>(ga);
    if ((rc = syrk_ev(h))) return rc;
    h->launches++;
    h->syrk_launches++;
  }
  return RVG_OK;
}

// Deferred update of a large front's columns [c0, c1) (rows [c0, m)) by the
// window of pending columns [wd, wd + kadd + *kdev): W rows start at wrow
// (ld m - wrow), L is the panel itself; the mixed form reads the packed
// window (tile 0 = rows [wrow, wrow + 128), F / 32 chunks per tile).  With
// cond set the launch only acts if *cond < cond_lt.
int launch_window_gemm(rvg_handle* h, LfCtx& cx, const LFArgs& a, int64_t m, int64_t c0, int64_t c1, int64_t wd,
                       int64_t wrow, int64_t F, const float* pk_w, const float* pk_l, int64_t kadd,
                       const int32_t* kdev, const int32_t* cond, int32_t cond_lt, bool mixed,
                       const int32_t* skip = nullptr, cudaStream_t on = nullptr, int max_ctas = 0) {
  cudaStream_t st = on ? on : cx.st;
  if (c1 <= c0) return RVG_OK;
  int rc = syrk_ev(h, cx.marks);
  if (rc) return rc;
  if (mixed) {
    const int64_t Fq = F / TC_BK;
    const int64_t nr = (m - c0 + TC_BM - 1) / TC_BM, nc = (c1 - c0 + TC_BN - 1) / TC_BN;
    const int64_t ntiles = tc_count_tiles(nr, nc, c0, c0);
    const int64_t t0 = (c0 - wrow) / TC_BM;
    TcArgs ta{a.a, m, c0, m, c0, c1, pk_w + (size_t)t0 * Fq * TC_BLOCK, pk_l + (size_t)t0 * Fq * TC_BLOCK, Fq, kdev,
              kadd, nr, nc, ntiles, h->d_err, cond, cond_lt, 0, skip};
    launch_tc(h, st, ta, max_ctas);
  } else {
    SyrkArgs ga{};
    ga.C = a.a;
    ga.ldc = m;
    ga.W = a.wo + (c0 - wrow);
    ga.ldw = m - wrow;
    ga.L = a.a + wd * m;
    ga.ldl = m;
    ga.r0 = c0;
    ga.r1 = m;
    ga.c0 = c0;
    ga.c1 = c1;
    ga.K = kadd;
    ga.Kdev = kdev;
    ga.cond = cond;
    ga.cond_lt = cond_lt;
    ga.skip = skip;
    k_syrk_lower<<<syrk_grid(ga), G_T, G_SMEM, st>>>(ga);
  }
  if ((rc = syrk_ev(h, cx.marks))) return rc;
  cx.launches++;
  if (cx.marks) h->syrk_launches++;
  return RVG_OK;
}

// One large front on the whole GPU: the launch sequence of large.cuh, with
// one host synchronisation per 256-column outer block (its start column
// depends on the delays of the previous block).
int factor_large_front(rvg_handle* h, LfCtx& cx, int32_t s, const Arenas& Ar, const DevOpts& dop) {
  cudaStream_t st = cx.st;
  auto mk = [&](int kind) { if (cx.marks) mark(h, kind); };
  const DFront& f = h->h_fronts[s];
  const int64_t m = f.m, p = f.k, nb = h->opt.outer_block_size, ib = h->opt.inner_block_size;
  LFArgs a{};
  a.a = Ar.panel + f.panel;
  a.m = m;
  a.p = p;
  a.perm = Ar.idx + f.idx + m;
  a.D = DRec{Ar.dtype + f.dpos, Ar.ddiag + f.dpos, Ar.doff + f.dpos};
  a.st = cx.lf;
  double* sc = Ar.scratch + f.scratch;
  a.pb = sc;
  a.w = sc + m * IBMAX;
  a.wo = sc + 2 * m * IBMAX;
  const bool mixed = front_mixed(h, s);
  const int64_t F = lf_window_cols(h, nb, mixed);
  a.lp = (int32_t*)(sc + m * (2 * IBMAX + lf_window_blocks(h) * nb));
  a.nfsb = p;
  a.o = dop;
  const int two_level = p > nb;
  const int64_t Fq = F / TC_BK;
  // the packed window (W and L parts), twice: a full window's far-field update may still read one
  // buffer on the far stream while the next blocks pack into the other
  float* pk_wb[2] = {nullptr, nullptr};
  float* pk_lb[2] = {nullptr, nullptr};
  if (mixed && two_level) {
    const int64_t tiles = (m + TC_BM - 1) / TC_BM;
    const size_t one = (size_t)tiles * Fq * TC_BLOCK;
    int rc = arena_ensure(h, VM_WPACK0 + cx.id, cx.wpack, cx.wpack_cap, 4 * one, st, false);
    if (rc) return rc;
    pk_wb[0] = cx.wpack; pk_lb[0] = cx.wpack + one;
    pk_wb[1] = cx.wpack + 2 * one; pk_lb[1] = cx.wpack + 3 * one;
  }
  // far-field updates beside the next blocks: the mixed form in the dynamic schedule (not while
  // recording profiling marks, not inside a captured graph)
  const bool profiling_marks = cx.marks && h->profiling;  // this front's launches carry the profiling events
  // (the far part starts far_ahead blocks after the window's first W row: a whole number of the packed
  // window's 128-row tiles only when the block width is a multiple of 128).  The far part of a flush
  // runs beside every block of the next window but its last, whose near-field update writes the first
  // far-field columns and so waits for it.
  const int64_t far_ahead = std::max<int64_t>(1, F / nb - 1);
  const int far_sms = h->opt.far_field_sms < 0 ? LF_FAR_SMS : h->opt.far_field_sms;
  const bool async_far = mixed && two_level && !profiling_marks && !h->replay && nb % TC_BM == 0 && far_sms > 0 &&
                         far_sms < h->nsm;
  if (async_far && !cx.far_st) {
    if (tl_no_alloc) return no_alloc_fail();
    CK(cudaStreamCreateWithFlags(&cx.far_st, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&cx.ev_fork, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&cx.ev_far, cudaEventDisableTiming));
  }
  mk(-1);
  k_lf_init<<<blocks_for(p, 256), 256, 0, st>>>(a.st, a.perm, p);
  cx.launches++;
  if (!h->replay) h->rec_g[s].clear();
  const int32_t* skip = &a.st->spec_bad;
  int irc = RVG_OK;  // first error of a launch helper inside issue()
  // Host view of the loop before an outer block: start column (eliminated so far), remaining
  // columns, the window of pending columns [wd, gne) whose W rows start at wrow, the block's index,
  // the packed-window buffer in use, and the block at which a far-field update running on the far
  // stream must be waited for (-1: none running).
  struct HostLF { int64_t gne, rem, wd, wrow; size_t outer; int par; int64_t far_due; };
  // what the host decided when it issued a block
  struct Issued { HostLF before; int64_t cs, bcols, oe, kadd, ncol; bool flush, window, far, waited; int slot; };
  // a CUDA call inside issue(): its failure becomes issue()'s error
  auto ck = [&](cudaError_t e, const char* what) {
    if (e != cudaSuccess && !irc) {
      set_error(std::string("CUDA error: ") + cudaGetErrorString(e) + " at " + what);
      irc = RVG_ERR_DEVICE;
    }
  };
  auto far_wait = [&]() {  // the stream takes up after the running far-field update
    ck(cudaStreamWaitEvent(st, cx.ev_far, 0), "cudaStreamWaitEvent (far-field update)");
    return irc;
  };
  // Launches one outer block for start column S.gne (2 + 6 per inner block + the outer-block steps).
  auto issue = [&](const HostLF& S, int slot) -> Issued {
    Issued I{};
    I.before = S;
    I.slot = slot;
    const int64_t rem = S.rem, cs = S.gne, wd = S.wd, wrow = S.wrow;
    const int64_t bcols = std::min(rem, nb), bm = m - cs, oe = cs + bcols;
    float* pk_w = pk_wb[S.par];
    float* pk_l = pk_lb[S.par];
    I.cs = cs; I.bcols = bcols; I.oe = oe;
    a.cs = cs;
    a.bcols = bcols;
    launch_chain(h, k_lf_begin_outer, 1, 256, 0, st, a);
    mk(RVG_PART_LF_SETUP);
    const int64_t ninner = (bcols + ib - 1) / ib;
    // the inner block's trailing update: rows and columns from ts = k + bs
    // (device values) within the outer block's view
    SyrkArgs gi{};
    gi.C = a.a + cs + cs * m;
    gi.ldc = m;
    gi.W = a.w;
    gi.ldw = bm;
    gi.L = a.a + cs + cs * m;
    gi.ldl = m;
    gi.r1 = bm;
    gi.c1 = bcols;
    gi.Kdev = &a.st->nelim;
    gi.dk = &a.st->k;
    gi.dbs = &a.st->bs;
    gi.skip = skip;
    // per inner block: the diagonal block (after the previous inner block's delays), the panel rows, the
    // post-processing with W = L D (k_lf_wi, its CTA 0 doing the block's own rows and D entries), the
    // rank-nelim update; the last inner block's delays on their own
    for (int64_t it = 0; it < ninner; ++it) {
      launch_chain(h, k_lf_block, 1, NT, 0, st, a, it > 0 ? 1 : 0);
      mk(RVG_PART_LF_BLOCK);
      launch_chain(h, k_lf_panel, blocks_for(bm, LF_PANEL_T), LF_PANEL_T, 0, st, a);
      mk(RVG_PART_LF_PANEL);
      launch_chain(h, k_lf_wi, blocks_for(bm, 256), 256, 0, st, a);
      launch_chain(h, k_syrk_inner, syrk_grid(gi), G_T, G_SMEM, st, gi);
      mk(RVG_PART_LF_UPDATE);
    }
    launch_chain(h, k_lf_delay, 1, NT, 0, st, a);
    mk(RVG_PART_LF_DELAY);
    cx.launches += 2 + 4 * ninner;
    if (two_level) {
      if (cs > 0) {
        launch_chain(h, k_lf_prop, (unsigned)((cs + LF_PROP_COLS - 1) / LF_PROP_COLS), 256,
                     (size_t)bcols * LF_PROP_COLS * 8, st, a);
        cx.launches++;
        mk(RVG_PART_LF_PROP);
      }
      if (oe < p) {
        I.window = true;
        // this block's W joins the window [wd, gne + bne)
        const int64_t kadd = cs - wd;
        I.kadd = kadd;
        a.wld = m - wrow;
        a.wrow0 = wrow;
        a.wcol0 = kadd;
        launch_chain(h, k_lf_w, blocks_for(m - oe, 128), 128, 0, st, a);
        cx.launches++;
        mk(RVG_PART_LF_W);
        // The next outer block is [g, g + min(rem - bcols, nb)); columns past
        // rem (delayed ones parked at the end) belong to no later block.  The
        // window is applied everywhere when it is full, or when the next block
        // is the last one (so no column is left pending for the end of the front).
        I.flush = kadd + bcols >= F || rem - bcols < nb;
        I.ncol = nb;
        const int32_t* bne_dev = &a.st->bne;
        if (mixed) {
          // append this block's chunks of W (rows [oe, m)) and L (rows [oe, p))
          const int64_t q0 = kadd / TC_BK, nqb = (bcols + TC_BK - 1) / TC_BK, t0 = (oe - wrow) / TC_BM;
          PackArgs pw{a.wo + (oe - wrow), a.wld, m - oe, Fq, bne_dev, kadd, pk_w, q0, t0, nullptr, 0, skip};
          PackArgs pl{a.a + wd * m + oe, m, p - oe, Fq, bne_dev, kadd, pk_l, q0, t0, nullptr, 0, skip};
          launch_pack(h, st, dim3((unsigned)nqb, blocks_for(m - oe, TC_BM)), pw);
          launch_pack(h, st, dim3((unsigned)nqb, blocks_for(p - oe, TC_BM)), pl);
          cx.launches += 2;
        }
        // columns of a far-field update still running: the next block's (the near field) from the
        // block it was launched for on, every trailing column at a flush
        if (S.far_due >= 0 && ((int64_t)S.outer >= S.far_due || I.flush)) {
          irc = irc ? irc : far_wait();
          I.waited = true;
        }
        if (I.flush) {
          const int64_t split = oe + far_ahead * nb;
          if (async_far && p - split >= 2 * nb) {
            // the next far_ahead blocks' columns now, the rest on the far stream beside them (both
            // after the packs; they touch different columns)
            ck(cudaEventRecord(cx.ev_fork, st), "cudaEventRecord (far-field fork)");
            ck(cudaStreamWaitEvent(cx.far_st, cx.ev_fork, 0), "cudaStreamWaitEvent (far-field fork)");
            irc = irc ? irc : launch_window_gemm(h, cx, a, m, oe, split, wd, wrow, F, pk_w, pk_l, kadd, bne_dev,
                                                 nullptr, 0, mixed, skip);
            irc = irc ? irc : launch_window_gemm(h, cx, a, m, split, p, wd, wrow, F, pk_w, pk_l, kadd, bne_dev,
                                                 nullptr, 0, mixed, skip, cx.far_st, h->nsm - far_sms);
            ck(cudaEventRecord(cx.ev_far, cx.far_st), "cudaEventRecord (far-field join)");
            cx.far_launches++;
            I.far = true;
          } else {
            // the window is full: every trailing column takes it (one GEMM)
            irc = irc ? irc : launch_window_gemm(h, cx, a, m, oe, p, wd, wrow, F, pk_w, pk_l, kadd, bne_dev,
                                                 nullptr, 0, mixed, skip);
          }
        } else {
          // near field: the next outer block's columns (oe + nb <= p here) take the whole window
          irc = irc ? irc : launch_window_gemm(h, cx, a, m, oe, oe + I.ncol, wd, wrow, F, pk_w, pk_l, kadd, bne_dev,
                                               nullptr, 0, mixed, skip);
          // far field: only if this block delayed columns (decided on the device); with far-field
          // updates on the far stream the host issues it once it has seen the delay
          if (oe + nb < p && !async_far)
            irc = irc ? irc : launch_window_gemm(h, cx, a, m, oe + nb, p, wd, wrow, F, pk_w, pk_l, kadd, bne_dev,
                                                 bne_dev, (int32_t)bcols, mixed, skip);
        }
        mk(RVG_PART_LF_SYRK);
      }
    }
    launch_chain(h, k_lf_outer, 1, NT, 0, st, a, rem, (int)two_level, async_far ? 0 : 1);
    cx.launches++;
    mk(RVG_PART_LF_OUTER);
    return I;
  };
  // The state after block I if it eliminated up to column g (no side effects).
  auto next_state = [&](const Issued& I, int32_t g) -> HostLF {
    HostLF S = I.before;
    const int64_t bne = g - I.cs;
    if (two_level && I.window && (I.flush || bne < I.bcols)) {  // every column is up to date: a new, empty window
      S.wd = g;
      S.wrow = g + std::min(S.rem - I.bcols, nb);
    }
    if (I.flush) S.par ^= 1;
    S.far_due = I.far ? (int64_t)I.before.outer + far_ahead : (I.waited ? -1 : I.before.far_due);
    S.gne = g;
    S.rem -= I.bcols;
    S.outer += 1;
    return S;
  };
  // The Schur-GEMM flops of block I (where the GEMM's events are recorded: the front carrying the marks).
  auto account = [&](const Issued& I, int32_t g) {
    if (!(two_level && I.window) || !cx.marks) return;
    const int64_t bne = g - I.cs;
    const double K = (double)(I.kadd + bne);
    if (I.flush) {
      cx.syrk_flops += 2.0 * K * lower_entries(I.oe, m, I.oe, p);
    } else {
      cx.syrk_flops += 2.0 * K * lower_entries(I.oe, m, I.oe, I.oe + I.ncol);
      if (I.oe + nb < p && bne < I.bcols) cx.syrk_flops += 2.0 * K * lower_entries(I.oe + nb, m, I.oe + nb, p);
    }
  };
  HostLF S{0, p, 0, std::min(p, nb), 0, 0, -1};
  if (h->replay) {
    // the progress of the recorded factorization, checked on the device
    const std::vector<int32_t>& rg = h->rec_g[s];
    while (S.rem > 0) {
      Issued I = issue(S, 0);
      if (irc) return irc;
      if (S.outer >= rg.size()) { set_error("refactorization replay: record too short"); return RVG_ERR_DEVICE; }
      const int32_t g = rg[S.outer];
      k_check_gne<<<1, 32, 0, st>>>(a.st, g, h->d_mismatch);
      CK(cudaGetLastError());
      account(I, g);
      S = next_state(I, g);
    }
  } else {
    // Blocks go out ahead on the guess that none delays a column (the next
    // start column is then this one plus its width); the device checks each
    // guess when the block begins (k_lf_begin_outer), and a wrong one turns
    // every later launch of the front into a no-op.  The host reads the
    // device's eliminated total after each block in issue order, at most
    // LF_AHEAD blocks behind; at the first one that differs it waits for the
    // streams, issues what that block's delay asks for (with far-field
    // updates on the far stream: the far field's update by the window and the
    // delay swap), clears the flag and issues again from the true start column.
    if (!cx.h_gne) {
      if (tl_no_alloc) return no_alloc_fail();
      CK(cudaHostAlloc((void**)&cx.h_gne, LF_AHEAD * sizeof(int32_t), cudaHostAllocDefault));
      for (int i = 0; i < LF_AHEAD; ++i) CK(cudaEventCreateWithFlags(&cx.ring_ev[i], cudaEventDisableTiming));
    }
    std::deque<Issued> q;
    int next_slot = 0;
    // with the profiling marks on, one block at a time: the marks are read back after each block
    const int ahead = profiling_marks ? 1 : LF_AHEAD;
    while (S.rem > 0 || !q.empty()) {
      if (S.rem > 0 && (int)q.size() < ahead) {
        const int slot = next_slot;
        next_slot = (next_slot + 1) % LF_AHEAD;
        Issued I = issue(S, slot);
        if (irc) return irc;
        CK(cudaMemcpyAsync(cx.h_gne + slot, &a.st->gne, 4, cudaMemcpyDeviceToHost, st));
        CK(cudaEventRecord(cx.ring_ev[slot], st));
        CK(cudaGetLastError());
        q.push_back(I);
        S = next_state(I, (int32_t)(I.cs + I.bcols));  // the guess: no delayed column in this block
        continue;
      }
      const Issued I = q.front();
      q.pop_front();
      const double t0 = now_ms();
      CK(cudaEventSynchronize(cx.ring_ev[I.slot]));
      const double waited = now_ms() - t0;
      const int32_t g = cx.h_gne[I.slot];
      h->rec_g[s].push_back(g);
      if (profiling_marks) {
        mark_flush(h);
        mk(-1);
      }
      account(I, g);
      // the device worked on this and the queued blocks meanwhile
      cx.wait_ms += waited;
      if (g == I.cs + I.bcols) continue;  // as guessed
      // a block delayed columns: the blocks issued after it did nothing; the
      // streams run dry while the host issues them again
      const double t1 = now_ms();
      CK(cudaStreamSynchronize(st));
      if (cx.far_st) CK(cudaStreamSynchronize(cx.far_st));
      cx.sync_ms += now_ms() - t1;
      cx.misses += (int64_t)q.size();
      q.clear();
      HostLF T = next_state(I, g);
      T.far_due = -1;  // nothing runs on the far stream any more
      if (async_far) {
        const int64_t bne = g - I.cs;
        a.cs = I.cs;
        a.bcols = I.bcols;
        if (two_level && I.window && !I.flush && I.oe + nb < p) {
          // the far field takes the window, this block's eliminated columns included
          irc = launch_window_gemm(h, cx, a, m, I.oe + nb, p, I.before.wd, I.before.wrow, F, pk_wb[I.before.par],
                                   pk_lb[I.before.par], I.kadd + bne, nullptr, nullptr, 0, mixed);
          if (irc) return irc;
        }
        if (two_level && bne < I.bcols)
          k_lf_swap<<<1, NT, 0, st>>>(a, I.cs, I.bcols, I.before.rem, (int)bne);
        cx.launches += 2;
      }
      CK(cudaMemsetAsync(&a.st->spec_bad, 0, sizeof(int32_t), st));
      CK(cudaGetLastError());
      S = T;
    }
  }
  if (S.far_due >= 0) CK(cudaStreamWaitEvent(st, cx.ev_far, 0));  // a far-field update still running
  k_lf_finish<<<1, 32, 0, st>>>(a, h->d_fronts, s);
  cx.launches++;
  mk(RVG_PART_LF_SETUP);
  CK(cudaGetLastError());
  return RVG_OK;
}

// The large fronts of one wave: one after another on the handle's stream when
// there is one (profiling marks on), otherwise up to LF_CONCURRENT at a time,
// each context's fronts in turn on its own host thread and stream, ordered
// after the wave's assembly and before what follows by events.
int factor_large_fronts(rvg_handle* h, const std::vector<int32_t>& ids, const Arenas& A, const DevOpts& dop) {
  if (ids.empty()) return RVG_OK;
  if (h->lfx.empty()) {
    h->lfx.resize(1);
    h->lfx[0].st = h->st;
    h->lfx[0].lf = h->d_lf;
  }
  auto fold = [&](LfCtx& c) {
    h->launches += c.launches;
    h->host_sync_ms += c.sync_ms;
    h->host_wait_ms += c.wait_ms;
    h->lf_misses += c.misses;
    h->lf_far += c.far_launches;
    h->syrk_flops += c.syrk_flops;
    c.launches = 0; c.sync_ms = 0; c.syrk_flops = 0; c.wait_ms = 0; c.misses = 0; c.far_launches = 0;
  };
  // (a capture forks into the same contexts with the fronts dealt the same way:
  // the replayed graph runs them concurrently on the buffers the dynamic run sized)
  const int nc = (int)std::min<size_t>(ids.size(), LF_CONCURRENT);
  while ((int)h->lfx.size() < nc) {  // grown before any reference into lfx is taken
    if (tl_no_alloc) return no_alloc_fail();
    LfCtx c;
    c.own = true;
    c.id = (int)h->lfx.size();
    CK(cudaStreamCreateWithFlags(&c.st, cudaStreamNonBlocking));
    CK(cudaMalloc((void**)&c.lf, sizeof(LFState)));
    h->lfx.push_back(c);
  }
  LfCtx& c0 = h->lfx[0];
  c0.wpack = h->wpack; c0.wpack_cap = h->wpack_cap;
  int rc = RVG_OK;
  if (nc == 1) {
    c0.marks = true;
    for (int32_t s : ids)
      if ((rc = factor_large_front(h, c0, s, A, dop))) break;
    h->wpack = c0.wpack; h->wpack_cap = c0.wpack_cap;
    fold(c0);
    return rc;
  }
  mark(h, -1);
  cudaEvent_t ready;
  CK(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming));
  CK(cudaEventRecord(ready, h->st));
  for (int t = 1; t < nc; ++t) CK(cudaStreamWaitEvent(h->lfx[t].st, ready, 0));
  std::vector<int> rcs(nc, RVG_OK);
  std::vector<std::string> errs(nc);
  const bool no_alloc = tl_no_alloc;
  auto work = [&](int t) {
    cudaSetDevice(h->device);
    const bool was = tl_no_alloc;
    tl_no_alloc = no_alloc;
    LfCtx& c = h->lfx[t];
    c.marks = false;
    for (size_t i = t; i < ids.size(); i += nc)
      if ((rcs[t] = factor_large_front(h, c, ids[i], A, dop))) { errs[t] = g_err; break; }
    tl_no_alloc = was;
  };
  std::vector<std::thread> th;
  for (int t = 1; t < nc; ++t) th.emplace_back(work, t);
  work(0);
  for (auto& x : th) x.join();
  h->wpack = c0.wpack; h->wpack_cap = c0.wpack_cap;
  for (int t = 1; t < nc; ++t) {
    CK(cudaEventRecord(ready, h->lfx[t].st));
    CK(cudaStreamWaitEvent(h->st, ready, 0));
  }
  CK(cudaEventDestroy(ready));
  mark(h, RVG_PART_OTHER);
  for (int t = 0; t < nc; ++t) {
    fold(h->lfx[t]);
    if (rcs[t] && !rc) { rc = rcs[t]; set_error(errs[t]); }
  }
  return rc;
}

int finish_factor(rvg_handle* h, int64_t d_used);

// Learned precision: large fronts of the wave just factored whose mixed-form
// D grew past the bound (k_front_growth) are factored again in FP64, alone.
// Each is assembled again from scratch -- original entries and its children's
// contribution blocks, which the wave released to the allocator but which no
// allocation overwrites before the next wave -- then factored on the
// large-front path with FP64 updates, and its contribution block is formed
// again with the FP64 GEMM.  The results are those a plain FP64 factorization
// gives the front from the same children.
int refactor_fp64(rvg_handle* h, const std::vector<int32_t>& redo, const Arenas& A, const DevOpts& dop,
                  const double* d_vals, const double* d_scal) {
  cudaStream_t st = h->st;
  const Plan& P = h->P;
  int rc;
  for (int32_t s : redo) h->route[s] = 0;
  h->sel_refactored += (int64_t)redo.size();
  for (int32_t s : redo) {
    const DFront& f = h->h_fronts[s];
    CK(cudaMemsetAsync(A.panel + f.panel, 0, (size_t)f.m * f.k * 8, st));
    if (f.flags & FF_HAS_CB) CK(cudaMemsetAsync(A.cbase + f.cb, 0, (size_t)f.nfs * f.nfs * 8, st));
  }
  const int n = (int)redo.size();
  std::vector<ScatterItem> sitems;
  for (int32_t s : redo)
    for (int64_t e = P.amap_ptr[s]; e < P.amap_ptr[s + 1]; e += 256) sitems.push_back(ScatterItem{s, 0, e});
  size_t maxch = 0;
  for (int32_t s : redo) maxch = std::max(maxch, P.children[s].size());
  std::vector<std::vector<EaTile>> eitems(maxch);
  for (size_t q = 0; q < maxch; ++q)
    for (int32_t s : redo) {
      if (q >= P.children[s].size()) continue;
      const int64_t c = P.children[s][q];
      const DFront& cf = h->h_fronts[c];
      if (!(cf.flags & FF_HAS_PARENT) || cf.ne >= cf.m) continue;
      const int sz = cf.m - cf.ne;
      for (int j0 = 0; j0 < sz; j0 += 32)
        for (int i0 = j0; i0 < sz; i0 += EA_ROWS) eitems[q].push_back(EaTile{s, (int32_t)c, j0, i0});
    }
  std::vector<TileItem> witems, gitems;
  std::vector<int32_t> big_cb;
  for (int32_t s : redo) {
    const DFront& f = h->h_fronts[s];
    if (!(f.flags & FF_HAS_CB) || f.k == 0) continue;
    for (int ti = 0; ti * 256 < f.nfs; ++ti) witems.push_back(TileItem{s, ti, 0, 0});
    if (f.nfs >= 256) { big_cb.push_back(s); continue; }  // GEMM by launch_syrk
    const int nt = (f.nfs + GT - 1) / GT;
    for (int tj = 0; tj < nt; ++tj)
      for (int ti = tj; ti < nt; ++ti) gitems.push_back(TileItem{s, ti, tj, 0});
  }
  Packer pk;
  const size_t o_ids = pk.add(redo), o_s = pk.add(sitems), o_w = pk.add(witems), o_g = pk.add(gitems);
  std::vector<size_t> o_e(maxch);
  for (size_t q = 0; q < maxch; ++q) o_e[q] = pk.add(eitems[q]);
  const size_t o_cnt = pk.add(std::vector<int32_t>(3 * (size_t)n, 0));
  if ((rc = ensure(h->d_stage2, h->stage2_cap, pk.buf.size(), st))) return rc;
  if ((rc = ensure_host(h->h_stage2, h->h_stage2_cap, std::max(pk.buf.size(), (size_t)3 * n * 4)))) return rc;
  std::memcpy(h->h_stage2, pk.buf.data(), pk.buf.size());
  CK(cudaMemcpyAsync(h->d_stage2, h->h_stage2, pk.buf.size(), cudaMemcpyHostToDevice, st));
  char* D = h->d_stage2;
  const int32_t* d_ids = (const int32_t*)(D + o_ids);
  k_front_rows<<<n, 128, 0, st>>>(d_ids, n, h->d_fronts, statics(h), A);
  if (!sitems.empty())
    k_scatter<<<(unsigned)sitems.size(), 256, 0, st>>>((const ScatterItem*)(D + o_s), h->d_fronts, statics(h), A,
                                                       d_vals, d_scal);
  for (size_t q = 0; q < maxch; ++q)
    if (!eitems[q].empty())
      k_extend_add_tiled<<<(unsigned)eitems[q].size(), 256, 0, st>>>((const EaTile*)(D + o_e[q]), h->d_fronts,
                                                                      statics(h), A);
  CK(cudaGetLastError());
  if ((rc = factor_large_fronts(h, redo, A, dop))) return rc;
  if (!witems.empty())
    k_cb_w<<<(unsigned)witems.size(), 256, 0, st>>>((const TileItem*)(D + o_w), h->d_fronts, A);
  if (!gitems.empty())
    k_cb_gemm<<<(unsigned)gitems.size(), 256, 0, st>>>((const TileItem*)(D + o_g), h->d_fronts, A);
  for (int32_t s : big_cb) {
    const DFront& f = h->h_fronts[s];
    SyrkArgs ga{A.cbase + f.cb, f.nfs, A.scratch + f.scratch, f.nfs, A.panel + f.panel + f.k, f.m,
                0, f.nfs, 0, f.nfs, 0, &h->d_fronts[s].ne};
    if ((rc = launch_syrk(h, ga, f.k, false))) return rc;
  }
  k_get_counts<<<blocks_for(n, 128), 128, 0, st>>>(d_ids, n, h->d_fronts, (int32_t*)(D + o_cnt));
  int32_t* hc = (int32_t*)h->h_stage2;
  CK(cudaMemcpyAsync(hc, D + o_cnt, (size_t)3 * n * 4, cudaMemcpyDeviceToHost, st));
  const double ts0 = now_ms();
  CK(cudaStreamSynchronize(st));
  h->host_sync_ms += now_ms() - ts0;
  for (int i = 0; i < n; ++i) {
    DFront& f = h->h_fronts[redo[i]];
    f.ne = hc[3 * i]; f.n1 = hc[3 * i + 1]; f.n2 = hc[3 * i + 2];
  }
  h->launches += 4 + (int64_t)maxch + (sitems.empty() ? 0 : 1);
  return RVG_OK;
}

// The numeric factorization proper: the level-set schedule of
// factor_tree_levelset (numeric.rs:1957-2163) with every front of a wave
// processed by the same launches.
int run_factor(rvg_handle* h, const double* d_vals, const double* d_scal) {
  Plan& P = h->P;
  cudaStream_t st = h->st;
  const int64_t ns = (int64_t)P.sn.size();
  h->factored = false;
  h->h_fronts.assign(ns, DFront());
  int64_t panel_used = 0, idx_used = 0, d_used = 0;
  std::vector<int64_t> cb_block(P.waves.size(), -1), cb_len(P.waves.size(), 0);
  std::vector<int64_t> cb_release_at(P.waves.size(), -1);
  h->cb_free.clear();
  if (h->cb_cap) h->cb_free[0] = (int64_t)h->cb_cap;
  const DevOpts dop = devopts(h->opt);
  const int ib = (int)h->opt.inner_block_size;
  double t_asm = 0, t_ker = 0, t_gem = 0;
  int rc;
  const double t_start = now_ms();
  h->host_alloc_ms = 0;
  h->host_sync_ms = 0;
  h->host_wait_ms = 0;
  h->host_gap_ms = 0;
  h->lf_misses = 0;
  h->lf_far = 0;
  h->ev_used = 0;
  h->mk_used = 0;
  for (double& v : h->part_ms) v = 0;
  h->syrk_flops = 0;
  h->syrk_ms = 0;
  h->syrk_launches = 0;
  h->launches = 0;
  h->peak_bytes = 0;
  if (h->opt.precision == 2) {
    if (!h->d_sel) { set_error("precision = 2 (learned) needs a selector: call rvg_set_selector first"); return RVG_ERR_INVALID_INPUT; }
    if ((rc = ensure(h->d_feat, h->d_feat_cap, (size_t)std::max<int64_t>(ns, 1) * FEAT_STRIDE, st))) return rc;
    if (!h->d_sel_flag) CK(cudaMalloc((void**)&h->d_sel_flag, sizeof(int32_t)));
    CK(cudaMemsetAsync(h->d_sel_flag, 0, sizeof(int32_t), st));
    h->route.assign(ns, 0);
    h->sel_large.clear();
    h->sel_routed = 0;
    h->sel_refactored = 0;
  }
  if (!h->replay) {
    h->rec_ok = false;
    h->rec_g.assign(ns, {});
    h->rec_stage.assign(P.waves.size(), 0);
  }
  CK(cudaEventRecord(h->ev[0], st));
  double t_ret = -1;  // host time the last wave synchronisation returned, until the next wave's first launch
  for (size_t w = 0; w < P.waves.size(); ++w) {
    const std::vector<int64_t>& wave = P.waves[w];
    const int nw = (int)wave.size();
    // ---- sizes from the children's eliminated counts (numeric.rs:1239-1262)
    int64_t panel_need = 0, idx_need = 0, d_need = 0, cb_need = 0, scratch_need = 0;
    std::vector<int32_t> dly_ids, dly_vals;
    for (int64_t s : wave) {
      DFront& f = h->h_fronts[s];
      int64_t nown = P.sn[s].n_owned(), ndin = 0;
      for (int64_t c : P.children[s]) {
        DFront& cf = h->h_fronts[c];
        cf.dly_off = (int32_t)ndin;
        dly_ids.push_back((int32_t)c);
        dly_vals.push_back((int32_t)ndin);
        ndin += cf.k - cf.ne;
      }
      int64_t k = nown + ndin, nfs = (int64_t)P.sn[s].pattern.size(), m = k + nfs;
      f.m = (int32_t)m; f.k = (int32_t)k; f.nown = (int32_t)nown; f.ndin = (int32_t)ndin; f.nfs = (int32_t)nfs;
      f.ne = 0; f.n1 = 0; f.n2 = 0;
      f.parent = (int32_t)P.sn[s].parent;
      f.flags = (P.sn[s].in_small_leaf ? FF_SMALL_LEAF : 0) | (f.parent >= 0 ? FF_HAS_PARENT : 0) |
                ((f.parent >= 0 && nfs > 0) ? FF_HAS_CB : 0);
      f.panel = panel_used + panel_need; panel_need += m * k;
      f.idx = idx_used + idx_need; idx_need += m + k;
      f.dpos = d_used + d_need; d_need += k;
      if (f.flags & FF_HAS_CB) cb_need += nfs * nfs;
    }
    {
      const int64_t T = h->opt.large_front_threshold;
      int64_t mid = 0;
      for (int64_t s : wave) {
        const DFront& f = h->h_fronts[s];
        if (!((f.flags & FF_SMALL_LEAF) || f.k < ib) && f.m >= T / 2 && f.m < T) ++mid;
      }
      for (int64_t s : wave) {
        DFront& f = h->h_fronts[s];
        const int64_t m = f.m, k = f.k, nfs = f.nfs;
        const bool tpp = (f.flags & FF_SMALL_LEAF) || k < ib;
        const bool large = front_is_large(m, tpp, T, mid);
        if (large) f.flags |= FF_LARGE;
        int64_t sc = tpp ? 0 : (2 * IBMAX * m + h->opt.outer_block_size);
        if (large) sc = m * (2 * IBMAX + lf_window_blocks(h) * h->opt.outer_block_size) + h->opt.outer_block_size;
        if (f.flags & FF_HAS_CB) sc = std::max<int64_t>(sc, nfs * k);
        f.scratch = scratch_need; scratch_need += sc;
      }
    }
    double ta = now_ms();
    if (t_ret >= 0) {  // the stream has been empty since the last wave's synchronisation returned
      h->host_gap_ms += ta - t_ret;
      t_ret = -1;
    }
    if ((rc = arena_ensure(h, VM_PANEL, h->panel, h->panel_cap, (size_t)(panel_used + panel_need), st, true)))
      return rc;
    if ((rc = arena_ensure(h, VM_IDX, h->idx, h->idx_cap, (size_t)(idx_used + idx_need), st, true))) return rc;
    if ((rc = ensure_d_arrays(h, (size_t)(d_used + d_need)))) return rc;
    if ((rc = arena_ensure(h, VM_SCRATCH, h->scratch, h->scratch_cap, (size_t)std::max<int64_t>(scratch_need, 1), st,
                           false)))
      return rc;
    double* scratch = h->scratch;
    if (cb_need) {
      if ((rc = cb_alloc(h, cb_need, &cb_block[w]))) return rc;
      cb_len[w] = cb_need;
    }
    h->host_alloc_ms += now_ms() - ta;
    {
      int64_t off = cb_block[w];
      for (int64_t s : wave) {
        DFront& f = h->h_fronts[s];
        if (f.flags & FF_HAS_CB) { f.cb = off; off += (int64_t)f.nfs * f.nfs; }
        else f.cb = -1;
      }
    }
    if (panel_need) CK(cudaMemsetAsync(h->panel + panel_used, 0, (size_t)panel_need * 8, st));
    const Arenas A{h->panel, h->idx, h->dtype, h->ddiag, h->doff, scratch, h->cb_arena};
    // ---- launch data of the whole wave, packed into one upload
    std::vector<int32_t> ids(wave.begin(), wave.end()), tpp_ids, aptp_ids, large_ids;
    std::vector<DFront> staged;
    staged.reserve(nw);
    for (int64_t s : wave) {
      staged.push_back(h->h_fronts[s]);
      const DFront& f = h->h_fronts[s];
      if ((f.flags & FF_SMALL_LEAF) || f.k < ib) tpp_ids.push_back((int32_t)s);
      else if (f.flags & FF_LARGE) large_ids.push_back((int32_t)s);
      else aptp_ids.push_back((int32_t)s);
    }
    // medium fronts largest first (dense work ~ k m^2): the persistent launch starts the long ones early
    std::stable_sort(aptp_ids.begin(), aptp_ids.end(), [&](int32_t a, int32_t b) {
      const DFront &fa = h->h_fronts[a], &fb = h->h_fronts[b];
      return (double)fa.k * fa.m * fa.m > (double)fb.k * fb.m * fb.m;
    });
    std::vector<ScatterItem> sitems;
    for (int64_t s : wave)
      for (int64_t e = P.amap_ptr[s]; e < P.amap_ptr[s + 1]; e += 256) sitems.push_back(ScatterItem{(int32_t)s, 0, e});
    size_t maxch = 0;
    for (int64_t s : wave) maxch = std::max(maxch, P.children[s].size());
    std::vector<std::vector<EaTile>> eitems(maxch);
    for (size_t q = 0; q < maxch; ++q)
      for (int64_t s : wave) {
        if (q >= P.children[s].size()) continue;
        int64_t c = P.children[s][q];
        const DFront& cf = h->h_fronts[c];
        if (!(cf.flags & FF_HAS_PARENT) || cf.ne >= cf.m) continue;
        int sz = cf.m - cf.ne;
        for (int j0 = 0; j0 < sz; j0 += 32)
          for (int i0 = j0; i0 < sz; i0 += EA_ROWS) eitems[q].push_back(EaTile{(int32_t)s, (int32_t)c, j0, i0});
      }
    std::vector<CbZeroItem> zitems;
    for (int64_t s : wave) {
      const DFront& f = h->h_fronts[s];
      if (f.flags & FF_HAS_CB)
        for (int j0 = 0; j0 < f.nfs; j0 += 32) zitems.push_back(CbZeroItem{(int32_t)s, j0});
    }
    std::vector<TileItem> witems, gitems;
    std::vector<int64_t> cb_syrk_fronts;
    for (int64_t s : wave) {
      const DFront& f = h->h_fronts[s];
      if (!(f.flags & FF_HAS_CB) || f.k == 0) continue;
      for (int ti = 0; ti * 256 < f.nfs; ++ti) witems.push_back(TileItem{(int32_t)s, ti, 0, 0});
      if ((f.flags & FF_LARGE) && f.nfs >= 256) continue;  // GEMM by launch_syrk
      int nt = (f.nfs + GT - 1) / GT;
      for (int tj = 0; tj < nt; ++tj)
        for (int ti = tj; ti < nt; ++ti) gitems.push_back(TileItem{(int32_t)s, ti, tj, 0});
    }
    Packer pk;
    size_t o_staged = pk.add(staged), o_ids = pk.add(ids), o_dly_ids = pk.add(dly_ids), o_dly_vals = pk.add(dly_vals);
    size_t o_tpp = pk.add(tpp_ids), o_aptp = pk.add(aptp_ids), o_s = pk.add(sitems);
    std::vector<size_t> o_e(maxch);
    for (size_t q = 0; q < maxch; ++q) o_e[q] = pk.add(eitems[q]);
    size_t o_w = pk.add(witems), o_g = pk.add(gitems), o_z = pk.add(zitems);
    size_t o_cnt = pk.add(std::vector<int32_t>(3 * (size_t)nw + 4, 0));
    size_t o_q = pk.add(std::vector<int32_t>(4, 0));  // work-queue counter of the medium fronts' launch
    const bool learned = h->opt.precision == 2 && !large_ids.empty();
    size_t o_lg = 0, o_rt = 0;
    if (learned) {
      o_lg = pk.add(large_ids);
      o_rt = pk.add(std::vector<int32_t>(large_ids.size(), 0));
    }
    if ((rc = arena_ensure(h, VM_STAGE, h->d_stage, h->stage_cap, pk.buf.size(), st, true))) return rc;
    char* hs;
    if (h->replay) {  // a slice of its own: the graph copies from it at every replay
      if (pk.buf.size() != h->rec_stage[w]) { set_error("refactorization replay: launch data differ"); return RVG_ERR_DEVICE; }
      hs = h->h_stage_all + h->stage_off[w];
    } else {
      if ((rc = ensure_host(h->h_stage, h->h_stage_cap, pk.buf.size()))) return rc;
      hs = h->h_stage;
      h->rec_stage[w] = pk.buf.size();
    }
    std::memcpy(hs, pk.buf.data(), pk.buf.size());
    CK(cudaMemcpyAsync(h->d_stage, hs, pk.buf.size(), cudaMemcpyHostToDevice, st));
    char* D = h->d_stage;
    const int32_t* d_ids = (const int32_t*)(D + o_ids);
    // ---- descriptors
    k_put_fronts<<<blocks_for(nw, 128), 128, 0, st>>>((const DFront*)(D + o_staged), d_ids, nw, h->d_fronts);
    if (!dly_ids.empty())
      k_put_dly<<<blocks_for(dly_ids.size(), 128), 128, 0, st>>>((const int32_t*)(D + o_dly_ids),
                                                                 (const int32_t*)(D + o_dly_vals), (int)dly_ids.size(),
                                                                 h->d_fronts);
    // contribution blocks of this wave: zero lower triangles (the extend-add adds into them)
    if (!zitems.empty())
      k_zero_cb_lower<<<(unsigned)zitems.size(), 256, 0, st>>>((const CbZeroItem*)(D + o_z), h->d_fronts, A);
    CK(cudaEventRecord(h->ev[1], st));
    // ---- assembly
    k_front_rows<<<nw, 128, 0, st>>>(d_ids, nw, h->d_fronts, statics(h), A);
    if (!sitems.empty())
      k_scatter<<<(unsigned)sitems.size(), 256, 0, st>>>((const ScatterItem*)(D + o_s), h->d_fronts, statics(h), A,
                                                         d_vals, d_scal);
    for (size_t q = 0; q < maxch; ++q)
      if (!eitems[q].empty())
        k_extend_add_tiled<<<(unsigned)eitems[q].size(), 256, 0, st>>>((const EaTile*)(D + o_e[q]), h->d_fronts,
                                                                        statics(h), A);
    CK(cudaEventRecord(h->ev[2], st));
    // contribution blocks whose parents are now all assembled
    for (size_t w2 = 0; w2 < w; ++w2)
      if (cb_block[w2] >= 0 && cb_release_at[w2] == (int64_t)w) { cb_release(h, cb_block[w2], cb_len[w2]); cb_block[w2] = -1; }
    // ---- learned precision: features of the assembled large fronts, the
    // selector's route for each (read back: it picks the launches below)
    if (learned) {
      const int nl = (int)large_ids.size();
      const int32_t* d_lg = (const int32_t*)(D + o_lg);
      int32_t* d_rt = (int32_t*)(D + o_rt);
      int64_t kmax = 0;
      for (int32_t s : large_ids) kmax = std::max<int64_t>(kmax, h->h_fronts[s].k);
      k_feat_init<<<1, 256, 0, st>>>(d_lg, nl, h->d_feat);
      k_front_features<<<dim3((unsigned)((kmax + 7) / 8), (unsigned)nl), 256, 0, st>>>(d_lg, h->d_fronts, A,
                                                                                     h->opt.threshold, h->d_feat);
      k_mlp_route<<<nl, 32, 0, st>>>(d_lg, nl, h->d_fronts, h->d_sel, h->sel_thresh, h->sel_force_fp64 ? 1 : 0,
                                    h->d_feat, d_rt);
      CK(cudaGetLastError());
      if ((rc = ensure_host((char*&)h->h_counts, h->h_counts_cap, (size_t)(std::max(3 * nw + 4, nl)) * 4))) return rc;
      CK(cudaMemcpyAsync(h->h_counts, d_rt, (size_t)nl * 4, cudaMemcpyDeviceToHost, st));
      CK(cudaEventRecord(h->ev[6], st));  // read below, once the wave's small and medium fronts are queued
      h->launches += 3;
    }
    // ---- dense factorization
    mark(h, -1);
    if (!tpp_ids.empty() || !aptp_ids.empty()) {
      // the wave's small and medium fronts in one persistent launch (profiling: part "aptp")
      if (!h->aptp_ctas) {  // resident CTAs of the queue kernel on this device
        int occ = 0, sms = 0;
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_front_queue, NT, 0));
        CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device));
        h->aptp_ctas = std::max(1, occ) * std::max(1, sms);
      }
      const int na = (int)aptp_ids.size(), nt = (int)tpp_ids.size(), items = na + (nt + 7) / 8;
      k_front_queue<<<(unsigned)std::min(items, h->aptp_ctas), NT, 0, st>>>(
          (const int32_t*)(D + o_aptp), na, (const int32_t*)(D + o_tpp), nt, (int32_t*)(D + o_q), h->d_fronts, A,
          dop);
    }
    mark(h, RVG_PART_APTP);
    if (learned) {  // the routes of the large fronts (the device is busy with the fronts queued above)
      const int nl = (int)large_ids.size();
      const double ts0 = now_ms();
      CK(cudaEventSynchronize(h->ev[6]));
      h->host_wait_ms += now_ms() - ts0;
      for (int i = 0; i < nl; ++i) {
        h->route[large_ids[i]] = (int8_t)(h->h_counts[i] != 0);
        h->sel_routed += h->h_counts[i] != 0;
      }
      h->sel_large.insert(h->sel_large.end(), large_ids.begin(), large_ids.end());
    }
    if ((rc = factor_large_fronts(h, large_ids, A, dop))) return rc;
    CK(cudaEventRecord(h->ev[3], st));
    // ---- contribution GEMM (fronts with nothing eliminated skip inside)
    mark(h, -1);
    if (!witems.empty())
      k_cb_w<<<(unsigned)witems.size(), 256, 0, st>>>((const TileItem*)(D + o_w), h->d_fronts, A);
    mark(h, RVG_PART_CB_W);
    if (!gitems.empty())
      k_cb_gemm<<<(unsigned)gitems.size(), 256, 0, st>>>((const TileItem*)(D + o_g), h->d_fronts, A);
    mark(h, RVG_PART_CB_GEMM);
    for (int64_t s : wave) {
      const DFront& f = h->h_fronts[s];
      if (!(f.flags & FF_HAS_CB) || f.k == 0 || !((f.flags & FF_LARGE) && f.nfs >= 256)) continue;
      SyrkArgs ga{A.cbase + f.cb, f.nfs, A.scratch + f.scratch, f.nfs, A.panel + f.panel + f.k, f.m,
                  0, f.nfs, 0, f.nfs, 0, &h->d_fronts[s].ne};
      if ((rc = launch_syrk(h, ga, f.k, front_mixed(h, s)))) return rc;
      mark(h, RVG_PART_CB_SYRK);
      cb_syrk_fronts.push_back(s);
    }
    if (learned) {
      k_front_growth<<<(unsigned)large_ids.size(), 256, 0, st>>>((const int32_t*)(D + o_lg), h->d_fronts, A,
                                                                 h->sel_bound, h->d_feat, h->d_sel_flag,
                                                                 (int32_t*)(D + o_rt));
      h->launches++;
    }
    CK(cudaEventRecord(h->ev[4], st));
    CK(cudaGetLastError());
    // ---- eliminated counts back to the host (replay: the recorded ones, checked on the device)
    if (h->replay) {
      k_check_counts<<<blocks_for(nw, 128), 128, 0, st>>>(d_ids, nw, h->d_fronts, h->d_rec, h->d_mismatch);
      CK(cudaGetLastError());
      for (int i = 0; i < nw; ++i) {
        DFront& f = h->h_fronts[wave[i]];
        const int32_t* r = &h->rec_cnt[3 * (size_t)wave[i]];
        f.ne = r[0]; f.n1 = r[1]; f.n2 = r[2];
      }
      for (int64_t s : cb_syrk_fronts) {
        const DFront& f = h->h_fronts[s];
        h->syrk_flops += 2.0 * (double)f.ne * (double)f.nfs * (double)(f.nfs + 1) / 2.0;
      }
      int64_t last = -1;
      for (int64_t s : wave) if (P.sn[s].parent >= 0) last = std::max(last, P.height[P.sn[s].parent]);
      cb_release_at[w] = last;
      panel_used += panel_need; idx_used += idx_need; d_used += d_need;
      continue;
    }
    k_get_counts<<<blocks_for(nw, 128), 128, 0, st>>>(d_ids, nw, h->d_fronts, (int32_t*)(D + o_cnt));
    const size_t nlr = learned ? large_ids.size() : 0;  // the large fronts' routes after the growth check
    if ((rc = ensure_host((char*&)h->h_counts, h->h_counts_cap, (size_t)(3 * nw + 4 + nlr) * 4))) return rc;
    CK(cudaMemcpyAsync(h->h_counts, D + o_cnt, (size_t)3 * nw * 4, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(h->h_counts + 3 * nw, h->d_err, 4, cudaMemcpyDeviceToHost, st));
    if (nlr) CK(cudaMemcpyAsync(h->h_counts + 3 * nw + 4, D + o_rt, nlr * 4, cudaMemcpyDeviceToHost, st));
    {
      double ts0 = now_ms();
      CK(cudaStreamSynchronize(st));
      t_ret = now_ms();
      h->host_sync_ms += t_ret - ts0;
    }
    mark_flush(h);
    if (h->h_counts[3 * nw]) {
      CK(cudaMemsetAsync(h->d_err, 0, sizeof(int32_t), st));
      set_error("a tensor-core Schur update gave up waiting on its pipeline (device timeout)");
      return RVG_ERR_DEVICE_TIMEOUT;
    }
    for (int i = 0; i < nw; ++i) {
      DFront& f = h->h_fronts[wave[i]];
      f.ne = h->h_counts[3 * i]; f.n1 = h->h_counts[3 * i + 1]; f.n2 = h->h_counts[3 * i + 2];
    }
    if (nlr) {
      std::vector<int32_t> redo;
      for (size_t i = 0; i < nlr; ++i)
        if (h->h_counts[3 * nw + 4 + i] == 2) redo.push_back(large_ids[i]);
      if (!redo.empty() && (rc = refactor_fp64(h, redo, A, dop, d_vals, d_scal))) return rc;
    }
    for (int64_t s : cb_syrk_fronts) {
      const DFront& f = h->h_fronts[s];
      h->syrk_flops += 2.0 * (double)f.ne * (double)f.nfs * (double)(f.nfs + 1) / 2.0;
    }
    h->launches += 1 + (int64_t)eitems.size() * 0 + (sitems.empty() ? 0 : 1) +
                   ((tpp_ids.empty() && aptp_ids.empty()) ? 0 : 1) + (witems.empty() ? 0 : 1) + (gitems.empty() ? 0 : 1) + 2 +
                   (dly_ids.empty() ? 0 : 1) + (zitems.empty() ? 0 : 1);
    for (size_t q = 0; q < maxch; ++q) h->launches += eitems[q].empty() ? 0 : 1;
    if (h->profiling) {  // the device memory in use (profiling runs only: the query costs host time)
      size_t fb = 0, tb = 0;
      cudaMemGetInfo(&fb, &tb);
      h->peak_bytes = std::max<int64_t>(h->peak_bytes, (int64_t)(tb - fb));
    }
    int64_t last = -1;
    for (int64_t s : wave) if (P.sn[s].parent >= 0) last = std::max(last, P.height[P.sn[s].parent]);
    cb_release_at[w] = last;
    float a1 = 0, a2 = 0, a3 = 0;
    cudaEventElapsedTime(&a1, h->ev[1], h->ev[2]);
    cudaEventElapsedTime(&a2, h->ev[2], h->ev[3]);
    cudaEventElapsedTime(&a3, h->ev[3], h->ev[4]);
    t_asm += a1; t_ker += a2; t_gem += a3;
    panel_used += panel_need; idx_used += idx_need; d_used += d_need;
  }
  for (size_t w = 0; w < cb_block.size(); ++w)
    if (cb_block[w] >= 0) { cb_release(h, cb_block[w], cb_len[w]); cb_block[w] = -1; }
  CK(cudaEventRecord(h->ev[5], st));
  if (h->replay) {
    if (d_used != h->rec_d_used) { set_error("refactorization replay: sizes differ"); return RVG_ERR_DEVICE; }
    return RVG_OK;  // captured; the statistics follow each replay (finish_factor)
  }
  h->factor_launches = h->launches;
  h->host_total_ms = now_ms() - t_start;
  h->rec_cnt.assign(3 * ns, 0);
  for (int64_t s = 0; s < ns; ++s) {
    const DFront& f = h->h_fronts[s];
    h->rec_cnt[3 * s] = f.ne; h->rec_cnt[3 * s + 1] = f.n1; h->rec_cnt[3 * s + 2] = f.n2;
  }
  h->rec_d_used = d_used;
  h->t_assembly = t_asm; h->t_kernel = t_ker; h->t_gemm = t_gem;
  rc = finish_factor(h, d_used);
  if (rc) return rc;
  h->rec_ok = true;
  return RVG_OK;
}

// Host side of the end of a factorization (dynamic or replayed): the total
// time, the Schur GEMM time of the profiling events, the aggregate statistics.
int finish_factor(rvg_handle* h, int64_t d_used) {
  cudaStream_t st = h->st;
  const int64_t ns = (int64_t)h->P.sn.size();
  CK(cudaStreamSynchronize(st));
  float tot = 0;
  cudaEventElapsedTime(&tot, h->ev[0], h->ev[5]);
  h->t_factor = tot;
  if (h->profiling)
    for (size_t e = 0; e + 1 < h->ev_used; e += 2) {
      float ms = 0;
      cudaEventElapsedTime(&ms, h->ev_pool[e], h->ev_pool[e + 1]);
      h->syrk_ms += ms;
    }
  // aggregate stats (numeric.rs:929-1009)
  h->tot1 = h->tot2 = h->totdel = h->zero_piv = h->max_front = 0;
  std::vector<int8_t> dt(d_used);
  std::vector<double> dd(d_used);
  if (d_used) {
    CK(cudaMemcpy(dt.data(), h->dtype, d_used, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(dd.data(), h->ddiag, d_used * 8, cudaMemcpyDeviceToHost));
  }
  for (int64_t s = 0; s < ns; ++s) {
    const DFront& f = h->h_fronts[s];
    h->tot1 += f.n1; h->tot2 += f.n2; h->totdel += f.k - f.ne;
    h->max_front = std::max<int64_t>(h->max_front, f.m);
    for (int c = 0; c < f.ne; ++c)
      if (dt[f.dpos + c] == PT_1X1 && dd[f.dpos + c] == 0.0) h->zero_piv++;
    if (f.parent < 0 && f.ne < f.m) h->zero_piv += f.k - f.ne;
  }
  h->factored = true;
  return RVG_OK;
}

}  // namespace

// ===========================================================================
// C ABI (numeric part)
// ===========================================================================
extern "C" {

const char* rvg_last_error(void) { return g_err.c_str(); }

void rvg_default_options(rvg_options* o) {
  o->threshold = 0.01;
  o->small = 1e-20;
  o->outer_block_size = 256;
  o->inner_block_size = 32;
  o->nemin = 32;
  o->small_leaf_threshold = 256;
  o->failed_pivot_tpp = 1;
  o->fallback_bk = 1;
  o->large_front_threshold = 2048;
  o->precision = 0;
  o->mixed_flush = 4;
  o->mixed_tile_cols = 256;
  o->mixed_operands = 0;
  o->graph_refactor = 0;
  o->far_field_sms = -1;
  o->mixed_window = 0;
}

static int check_opts(const rvg_options& o) {  // factor.rs:307-347 (precision and below: no counterpart)
  if (!(o.threshold > 0.0 && o.threshold <= 1.0)) { set_error("threshold must be in (0, 1]"); return RVG_ERR_INVALID_INPUT; }
  if (!(o.small >= 0.0)) { set_error("small must be >= 0.0"); return RVG_ERR_INVALID_INPUT; }
  if (o.outer_block_size <= 0) { set_error("outer_block_size must be > 0"); return RVG_ERR_INVALID_INPUT; }
  if (o.inner_block_size <= 0) { set_error("inner_block_size must be > 0"); return RVG_ERR_INVALID_INPUT; }
  if (o.inner_block_size > o.outer_block_size) {
    set_error("inner_block_size must be <= outer_block_size");
    return RVG_ERR_INVALID_INPUT;
  }
  if (o.inner_block_size > IBMAX) { set_error("inner_block_size above 32 is not supported by the B200 kernels"); return RVG_ERR_INVALID_INPUT; }
  if (o.nemin < 1) { set_error("nemin must be >= 1"); return RVG_ERR_INVALID_INPUT; }
  if (o.large_front_threshold < 1) { set_error("large_front_threshold must be >= 1"); return RVG_ERR_INVALID_INPUT; }
  if (o.precision < 0 || o.precision > 2) { set_error("precision must be 0 (FP64), 1 (mixed) or 2 (learned)"); return RVG_ERR_INVALID_INPUT; }
  if (o.mixed_flush != 0 && o.mixed_flush != 1 && o.mixed_flush != 2 && o.mixed_flush != 4 && o.mixed_flush != 8) {
    set_error("mixed_flush must be 0, 1, 2, 4 or 8");
    return RVG_ERR_INVALID_INPUT;
  }
  if (o.mixed_operands != 0 && o.mixed_operands != 1) {
    set_error("mixed_operands must be 0 (TF32) or 1 (BF16)");
    return RVG_ERR_INVALID_INPUT;
  }
  if (o.mixed_tile_cols != 128 && o.mixed_tile_cols != 256) {
    set_error("mixed_tile_cols must be 128 or 256");
    return RVG_ERR_INVALID_INPUT;
  }
  if (o.far_field_sms < -1) { set_error("far_field_sms must be -1 (default), 0 (no split) or a count"); return RVG_ERR_INVALID_INPUT; }
  if (o.mixed_window < 0 || o.mixed_window > LF_WINDOW_MAX) {
    set_error("mixed_window must be 0 (default) or 1 to 8 outer blocks");
    return RVG_ERR_INVALID_INPUT;
  }
  if (o.graph_refactor < 0 || o.graph_refactor > 2) {
    set_error("graph_refactor must be 0 (off), 1 (replay) or 2 (replay, arenas kept at their addresses across rvg_trim)");
    return RVG_ERR_INVALID_INPUT;
  }
  return RVG_OK;
}

rvg_status rvg_create(int64_t n, int64_t nsup, const int64_t* sup_begin, const int64_t* sup_end, const int64_t* pat_ptr,
                      const int64_t* pat_idx, const int64_t* sup_parent, const int64_t* perm_fwd, const int64_t* colptr,
                      const int64_t* rowidx, const rvg_options* opt, rvg_handle** out) {
  if (!out) { set_error("null output handle"); return RVG_ERR_INVALID_INPUT; }
  *out = nullptr;
  rvg_options o;
  rvg_default_options(&o);
  if (opt) o = *opt;
  int rc = check_opts(o);
  if (rc) return (rvg_status)rc;
  if (n < 0 || nsup < 0) { set_error("negative size"); return RVG_ERR_INVALID_INPUT; }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    set_error("no CUDA device available (the numeric phase has no CPU fallback)");
    return RVG_ERR_DEVICE;
  }
  std::unique_ptr<rvg_handle> h(new rvg_handle());
  h->opt = o;
  h->nnz = n ? colptr[n] : 0;
  std::string err;
  rc = build_plan(nullptr, n, nsup, sup_begin, sup_end, pat_ptr, pat_idx, sup_parent, perm_fwd, colptr, rowidx, o, h->P, &err);
  if (rc) { set_error(err); return (rvg_status)rc; }
  CK(cudaGetDevice(&h->device));
  CK(cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking));
  for (auto& e : h->ev) CK(cudaEventCreate(&e));
  {
    cudaMemPool_t pool;
    CK(cudaDeviceGetDefaultMemPool(&pool, h->device));
    uint64_t thr = UINT64_MAX;
    CK(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr));
  }
  Plan& P = h->P;
  const int64_t ns = (int64_t)P.sn.size();
  std::vector<int64_t> chp(ns + 1, 0);
  std::vector<int32_t> chi;
  for (int64_t s = 0; s < ns; ++s) {
    chp[s + 1] = chp[s] + (int64_t)P.children[s].size();
    for (int64_t c : P.children[s]) chi.push_back((int32_t)c);
  }
  cudaStream_t st = h->st;
  if ((rc = upload(h->d_own_ptr, P.own_ptr, st)) || (rc = upload(h->d_own_idx, P.own_idx, st)) ||
      (rc = upload(h->d_pat_ptr, P.pat_ptr, st)) || (rc = upload(h->d_pat_idx, P.pat_idx, st)) ||
      (rc = upload(h->d_amap_ptr, P.amap_ptr, st)) || (rc = upload(h->d_amap, P.amap, st)) ||
      (rc = upload(h->d_ea_ptr, P.ea_ptr, st)) || (rc = upload(h->d_ea_map, P.ea_map, st)) ||
      (rc = upload(h->d_ch_ptr, chp, st)) || (rc = upload(h->d_ch_idx, chi, st)) ||
      (rc = upload(h->d_pfwd, P.perm_fwd, st)))
    return (rvg_status)rc;
  CK(cudaMallocAsync((void**)&h->d_fronts, std::max<int64_t>(ns, 1) * sizeof(DFront), st));
  CK(cudaMallocAsync((void**)&h->d_lf, sizeof(LFState), st));
  {
    std::vector<int64_t> cp(colptr, colptr + n + 1);
    std::vector<int32_t> ri(rowidx, rowidx + h->nnz);
    if ((rc = upload(h->d_colptr, cp, st)) || (rc = upload(h->d_rowidx, ri, st))) return (rvg_status)rc;
  }
  CK(cudaMallocHost((void**)&h->h_norms, 4 * sizeof(double)));
  if (o.graph_refactor == 2 && (rc = vm_create(h.get()))) return (rvg_status)rc;  // address-stable arenas
  if ((rc = presize_arenas(h.get()))) return (rvg_status)rc;
  CK(cudaFuncSetAttribute(k_syrk_lower, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)G_SMEM));
  CK(cudaFuncSetAttribute(k_syrk_inner, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)G_SMEM));
  CK(cudaFuncSetAttribute(k_syrk_tc<1, TC_TF32>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TC_SMEM));
  CK(cudaFuncSetAttribute(k_syrk_tc<2, TC_TF32>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TC_SMEM));
  CK(cudaFuncSetAttribute(k_syrk_tc<4, TC_TF32>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TC_SMEM));
  CK(cudaFuncSetAttribute(k_syrk_tc<8, TC_TF32>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TC_SMEM));
  CK(cudaFuncSetAttribute(k_syrk_tc<TC_NO_FLUSH, TC_TF32>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TC_SMEM));
  CK(cudaFuncSetAttribute(k_syrk_tc_pair<TC_TF32>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TP_SMEM));
  CK(cudaFuncSetAttribute(k_syrk_tc<1, TC_BF16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TC_SMEM));
  CK(cudaFuncSetAttribute(k_syrk_tc<2, TC_BF16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TC_SMEM));
  CK(cudaFuncSetAttribute(k_syrk_tc<4, TC_BF16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TC_SMEM));
  CK(cudaFuncSetAttribute(k_syrk_tc<8, TC_BF16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TC_SMEM));
  CK(cudaFuncSetAttribute(k_syrk_tc<TC_NO_FLUSH, TC_BF16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TC_SMEM));
  CK(cudaFuncSetAttribute(k_syrk_tc_pair<TC_BF16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TP_SMEM));
  CK(cudaDeviceGetAttribute(&h->nsm, cudaDevAttrMultiProcessorCount, h->device));
  {  // RVG_CHAIN_PDL=0 launches the large-front chain kernels plainly (same results; for timing comparisons)
    const char* e = std::getenv("RVG_CHAIN_PDL");
    h->chain_pdl = !(e && e[0] == '0');
  }

  CK(cudaMallocAsync((void**)&h->d_err, sizeof(int32_t), st));
  CK(cudaMemsetAsync(h->d_err, 0, sizeof(int32_t), st));
  CK(cudaMallocAsync((void**)&h->d_vals, std::max<int64_t>(h->nnz, 1) * 8, st));
  CK(cudaMallocAsync((void**)&h->d_scal, std::max<int64_t>(n, 1) * 8, st));
  CK(cudaStreamSynchronize(st));
  *out = h.release();
  return RVG_OK;
}

static int device_wait_status(rvg_handle* h);

static void drop_graph(rvg_handle* h) {
  if (h->gexec) cudaGraphExecDestroy(h->gexec);
  if (h->graph) cudaGraphDestroy(h->graph);
  h->gexec = nullptr;
  h->graph = nullptr;
}

// Refactorization as one CUDA graph launch.  The first call after a dynamic
// factorization captures run_factor with every host decision taken from that
// factorization's record (front sizes, eliminated counts, the large fronts'
// progress per outer block) and the launch data of each wave in a pinned slice
// of its own; device checks compare what the replayed factorization actually
// eliminated with the record.  Later calls launch the graph.  *done = false
// (and the graph dropped) when the checks saw another decision, when a buffer
// would have to grow, or when capture fails: the caller then factors
// dynamically, which records again.  The results are the dynamic path's.
static int replay_factor(rvg_handle* h, const double* ds, bool* done) {
  *done = false;
  cudaStream_t st = h->st;
  if (h->gexec && h->graph_ds != ds) drop_graph(h);
  if (!h->gexec) {
    // device copy of the recorded counts, the mismatch word, the pinned launch data
    const size_t nc = h->rec_cnt.size();
    int rc;
    if ((rc = ensure(h->d_rec, h->d_rec_cap, std::max<size_t>(nc, 1), st))) return rc;
    if (!h->d_mismatch) CK(cudaMalloc((void**)&h->d_mismatch, sizeof(int32_t)));
    if (nc) CK(cudaMemcpyAsync(h->d_rec, h->rec_cnt.data(), nc * 4, cudaMemcpyHostToDevice, st));
    h->stage_off.assign(h->rec_stage.size(), 0);
    size_t tot = 0;
    for (size_t w = 0; w < h->rec_stage.size(); ++w) { h->stage_off[w] = tot; tot += (h->rec_stage[w] + 255) & ~size_t(255); }
    if ((rc = ensure_host(h->h_stage_all, h->h_stage_all_cap, std::max<size_t>(tot, 1)))) return rc;
    CK(cudaStreamSynchronize(st));
    cudaGraph_t g = nullptr;
    CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    h->replay = true;
    tl_no_alloc = true;
    rc = run_factor(h, h->d_vals, ds);
    tl_no_alloc = false;
    h->replay = false;
    const cudaError_t ec = cudaStreamEndCapture(st, &g);
    if (rc || ec != cudaSuccess || !g) {
      if (g) cudaGraphDestroy(g);
      cudaGetLastError();
      h->rec_ok = false;
      return RVG_OK;  // not replayable: factor dynamically
    }
    if (cudaGraphInstantiate(&h->gexec, g, 0) != cudaSuccess) {
      cudaGraphDestroy(g);
      cudaGetLastError();
      h->gexec = nullptr;
      h->rec_ok = false;
      return RVG_OK;
    }
    h->graph = g;
    h->graph_ds = ds;
  }
  CK(cudaMemsetAsync(h->d_mismatch, 0, sizeof(int32_t), st));
  const double t0 = now_ms();
  h->ev_used = 0;  // no per-launch events inside the graph
  CK(cudaEventRecord(h->ev[0], st));  // (the records inside the capture only ordered the capture)
  CK(cudaGraphLaunch(h->gexec, st));
  CK(cudaEventRecord(h->ev[5], st));
  int32_t mis = 0;
  CK(cudaMemcpyAsync(&mis, h->d_mismatch, 4, cudaMemcpyDeviceToHost, st));
  int rc = finish_factor(h, h->rec_d_used);  // synchronises
  if (rc) return rc;
  if ((rc = device_wait_status(h))) return rc;
  h->host_total_ms = now_ms() - t0;
  for (double& v : h->part_ms) v = 0;
  if (mis) {  // another decision than the recorded one: this factor is not valid
    h->factored = false;
    drop_graph(h);
    h->rec_ok = false;
    return RVG_OK;
  }
  h->factor_launches = 1;
  h->host_sync_ms = 0;
  h->host_wait_ms = 0;
  h->host_gap_ms = 0;
  h->lf_misses = 0;
  h->lf_far = 0;
  *done = true;
  return RVG_OK;
}

static int factor_common(rvg_handle* h, const double* dv, const double* ds) {
  int rc;
  if (h->need_presize) {  // after rvg_trim: the arenas at their delay-free size again
    if ((rc = presize_arenas(h))) return rc;
    if (h->vm && (rc = vm_restore(h))) return rc;  // (address-stable: up to their largest size, all of them)
    h->need_presize = false;
  }
  // the refinement needs the unfactored values and ||A||_F
  if (dv != h->d_vals && h->nnz) CK(cudaMemcpyAsync(h->d_vals, dv, h->nnz * 8, cudaMemcpyDeviceToDevice, h->st));
  // NaN or Inf in the values or the scaling: a clean InvalidInput before any factor kernel runs (the
  // reference rejects them in its MC64 scaling, ordering/matching.rs:143-157)
  if (h->nnz || (ds && h->P.n)) {
    if (!h->d_nonfinite) CK(cudaMalloc((void**)&h->d_nonfinite, sizeof(int32_t)));
    CK(cudaMemsetAsync(h->d_nonfinite, 0, sizeof(int32_t), h->st));
    if (h->nnz) k_nonfinite<<<296, 256, 0, h->st>>>(h->d_vals, h->nnz, h->d_nonfinite);
    if (ds && h->P.n) k_nonfinite<<<296, 256, 0, h->st>>>(ds, h->P.n, h->d_nonfinite);
    CK(cudaGetLastError());
    int32_t bad = 0;
    CK(cudaMemcpyAsync(&bad, h->d_nonfinite, 4, cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    if (bad) {
      h->factored = false;
      set_error("the matrix values or the scaling contain NaN or Inf");
      return RVG_ERR_INVALID_INPUT;
    }
  }
  bool done = false;
  if (h->opt.graph_refactor && h->rec_ok && h->opt.precision != 2) {
    if ((rc = replay_factor(h, ds, &done))) return rc;
  }
  if (!done) {
    drop_graph(h);  // a dynamic run may move buffers: the next refactorization captures anew
    rc = run_factor(h, h->d_vals, ds);
    if (rc) return rc;
  }
  if (h->opt.precision == 2) {
    // fronts that took the mixed form and grew past the bound were factored
    // again in FP64 at the end of their wave (refactor_fp64)
    int32_t flagged = 0;
    CK(cudaMemcpyAsync(&flagged, h->d_sel_flag, 4, cudaMemcpyDeviceToHost, h->st));
    CK(cudaStreamSynchronize(h->st));
    h->sel_flagged = flagged;
    h->sel_fallback = h->sel_refactored;
  }
  double* d_acc = nullptr;
  CK(cudaMallocAsync((void**)&d_acc, 8, h->st));
  CK(cudaMemsetAsync(d_acc, 0, 8, h->st));
  if (h->nnz) k_sumsq<<<296, 256, 0, h->st>>>(h->d_vals, h->nnz, d_acc);
  CK(cudaMemcpyAsync(h->h_norms, d_acc, 8, cudaMemcpyDeviceToHost, h->st));
  CK(cudaFreeAsync(d_acc, h->st));
  CK(cudaStreamSynchronize(h->st));
  h->a_fro = std::sqrt(h->h_norms[0]);
  return RVG_OK;
}

rvg_status rvg_factor(rvg_handle* h, const double* values, const double* scaling) {
  if (!h) { set_error("null handle"); return RVG_ERR_INVALID_INPUT; }
  if (h->P.n > 0 && !values) { set_error("null values"); return RVG_ERR_INVALID_INPUT; }
  CK(cudaSetDevice(h->device));
  if (h->nnz) CK(cudaMemcpyAsync(h->d_vals, values, h->nnz * 8, cudaMemcpyHostToDevice, h->st));
  h->has_scaling = scaling != nullptr;
  if (scaling && h->P.n) CK(cudaMemcpyAsync(h->d_scal, scaling, h->P.n * 8, cudaMemcpyHostToDevice, h->st));
  return (rvg_status)factor_common(h, h->d_vals, h->has_scaling ? h->d_scal : nullptr);
}

rvg_status rvg_factor_device(rvg_handle* h, const double* d_values, const double* d_scaling) {
  if (!h) { set_error("null handle"); return RVG_ERR_INVALID_INPUT; }
  CK(cudaSetDevice(h->device));
  h->has_scaling = d_scaling != nullptr;
  if (d_scaling && h->P.n) CK(cudaMemcpyAsync(h->d_scal, d_scaling, h->P.n * 8, cudaMemcpyDeviceToDevice, h->st));
  return (rvg_status)factor_common(h, d_values, h->has_scaling ? h->d_scal : nullptr);
}

// Status of the bounded device waits (mixed-form GEMM pipeline, solve
// dependencies) since the last check; resets the word.  Synchronises.
static int device_wait_status(rvg_handle* h) {
  int32_t e = 0;
  CK(cudaMemcpyAsync(&e, h->d_err, 4, cudaMemcpyDeviceToHost, h->st));
  CK(cudaStreamSynchronize(h->st));
  if (e) {
    CK(cudaMemsetAsync(h->d_err, 0, 4, h->st));
    set_error(e == 2 ? "a solve block gave up waiting for the blocks it depends on (device timeout)"
                     : "a tensor-core Schur update gave up waiting on its pipeline (device timeout)");
    return RVG_ERR_DEVICE_TIMEOUT;
  }
  return RVG_OK;
}

// aptp_solve (solve.rs:57-326) with the permutation and scaling of
// SparseLDLT::solve_in_place (solver.rs:396-425): per wave one forward launch
// (leaves first) and, in reverse, one backward launch of solve_sf.cuh.
static int solve_common(rvg_handle* h, double* d_rhs, int64_t nrhs, int64_t ldb) {
  Plan& P = h->P;
  const int64_t n = P.n;
  cudaStream_t st = h->st;
  if (n == 0 || nrhs == 0) return RVG_OK;
  int rc = ensure(h->d_x, h->x_cap, (size_t)(n * nrhs), st);
  if (rc) return rc;
  // right-hand sides per launch (a power of two up to 8) and the per-front
  // solve workspace: forward results, then final values (R x m each)
  const int rmax = nrhs >= 8 ? 8 : nrhs >= 4 ? 4 : nrhs >= 2 ? 2 : 1;
  int64_t wneed = 0;
  std::vector<DFront> fr = h->h_fronts;
  for (auto& f : fr) { f.scratch = wneed; wneed += 2 * (int64_t)rmax * f.m; }
  if ((rc = ensure(h->solve_work, h->solve_work_cap, (size_t)std::max<int64_t>(wneed, 1), st))) return rc;
  CK(cudaMemcpyAsync(h->d_fronts, fr.data(), fr.size() * sizeof(DFront), cudaMemcpyHostToDevice, st));
  Arenas A{h->panel, h->idx, h->dtype, h->ddiag, h->doff, nullptr, h->cb_arena};
  CK(cudaEventRecord(h->ev[6], st));
  int64_t launches = 0;
  int64_t tot = n * nrhs;
  k_perm_scale_in<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(d_rhs, ldb, nrhs, h->d_x, n, h->d_pfwd,
                                                                 h->has_scaling ? h->d_scal : nullptr);
  launches++;
  // block layout of every wave: forward (diagonal then L21 blocks per front) and backward (diagonal blocks)
  const size_t nw = P.waves.size();
  Packer pk;
  std::vector<size_t> offf(nw), offb(nw);
  std::vector<int32_t> nfr(nw, 0), nbf(nw, 0), nbb(nw, 0);
  int32_t maxblk = 1;
  int64_t maxslots = 1;
  for (size_t w = 0; w < nw; ++w) {
    std::vector<SfFront> vf, vb;
    int32_t slots = 0;
    for (int64_t s : P.waves[w]) {
      const DFront& f = fr[s];
      if (f.ne == 0) continue;
      const int32_t nbd = (f.ne + SF_B - 1) / SF_B, nbr = (f.m - f.ne + SF_B - 1) / SF_B;
      const int32_t ngrp = (nbr + SF_PG - 1) / SF_PG;
      vf.push_back(SfFront{(int32_t)s, nbf[w], nbd, nbr, 0, 0});
      vb.push_back(SfFront{(int32_t)s, nbb[w], nbd, nbr, ngrp, slots});
      nbf[w] += nbd + nbr;
      nbb[w] += nbr + nbd * ngrp + nbd;  // gathers, partial sums, column blocks
      slots += nbd * ngrp;
    }
    maxslots = std::max<int64_t>(maxslots, slots);
    nfr[w] = (int32_t)vf.size();
    offf[w] = pk.add(vf);
    offb[w] = pk.add(vb);
    maxblk = std::max(maxblk, std::max(nbf[w], nbb[w]));
  }
  if ((rc = arena_ensure(h, VM_STAGE, h->d_stage, h->stage_cap, pk.buf.size() + 16, st, true))) return rc;
  if ((rc = ensure_host(h->h_stage, h->h_stage_cap, pk.buf.size() + 16))) return rc;
  std::memcpy(h->h_stage, pk.buf.data(), pk.buf.size());
  CK(cudaMemcpyAsync(h->d_stage, h->h_stage, pk.buf.size(), cudaMemcpyHostToDevice, st));
  if ((rc = ensure(h->sf_sync, h->sf_sync_cap, (size_t)maxblk + 1, st))) return rc;
  if ((rc = ensure_nocopy(h->sf_part, h->sf_part_cap, (size_t)maxslots * 8 * SF_B, st))) return rc;
  auto wave = [&](size_t w, bool fwd, int64_t rh) {
    SfWave sw;
    sw.part = h->sf_part;
    sw.fr = (const SfFront*)(h->d_stage + (fwd ? offf[w] : offb[w]));
    sw.nfr = nfr[w];
    sw.nblk = fwd ? nbf[w] : nbb[w];
    sw.ticket = h->sf_sync;
    sw.flags = h->sf_sync + 1;
    sw.x = h->d_x + rh * n;
    sw.ldx = n;
    sw.work = h->solve_work;
    sw.err = h->d_err;
    return sw;
  };
  auto fwd = [&](int r, size_t w, const SfWave& sw) {
    const unsigned g = (unsigned)std::min<int64_t>(nbf[w], 16LL * h->nsm);
    switch (r) {
      case 8: k_sf_fwd<8><<<g, SF_B, 0, st>>>(sw, h->d_fronts, A); break;
      case 4: k_sf_fwd<4><<<g, SF_B, 0, st>>>(sw, h->d_fronts, A); break;
      case 2: k_sf_fwd<2><<<g, SF_B, 0, st>>>(sw, h->d_fronts, A); break;
      default: k_sf_fwd<1><<<g, SF_B, 0, st>>>(sw, h->d_fronts, A); break;
    }
  };
  if (!h->sf_attr) {  // the backward kernels' static + dynamic shared memory exceeds the default 48 KB
    CK(cudaFuncSetAttribute(k_sf_bwd<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, SF_BWD_DYN));
    CK(cudaFuncSetAttribute(k_sf_bwd<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, SF_BWD_DYN));
    CK(cudaFuncSetAttribute(k_sf_bwd<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, SF_BWD_DYN));
    CK(cudaFuncSetAttribute(k_sf_bwd<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, SF_BWD_DYN));
    h->sf_attr = true;
  }
  auto bwd = [&](int r, size_t w, const SfWave& sw) {
    const unsigned g = (unsigned)std::min<int64_t>(nbb[w], 6LL * h->nsm);
    switch (r) {
      case 8: k_sf_bwd<8><<<g, SF_B, SF_BWD_DYN, st>>>(sw, h->d_fronts, A); break;
      case 4: k_sf_bwd<4><<<g, SF_B, SF_BWD_DYN, st>>>(sw, h->d_fronts, A); break;
      case 2: k_sf_bwd<2><<<g, SF_B, SF_BWD_DYN, st>>>(sw, h->d_fronts, A); break;
      default: k_sf_bwd<1><<<g, SF_B, SF_BWD_DYN, st>>>(sw, h->d_fronts, A); break;
    }
  };
  for (int64_t rh = 0; rh < nrhs;) {
    const int64_t left = nrhs - rh;
    const int r = left >= 8 ? 8 : left >= 4 ? 4 : left >= 2 ? 2 : 1;
    for (size_t w = 0; w < nw; ++w) {
      if (!nbf[w]) continue;
      CK(cudaMemsetAsync(h->sf_sync, 0, (size_t)(nbf[w] + 1) * 4, st));
      fwd(r, w, wave(w, true, rh));
      launches++;
    }
    for (size_t w = nw; w-- > 0;) {
      if (!nbb[w]) continue;
      CK(cudaMemsetAsync(h->sf_sync, 0, (size_t)(nbb[w] + 1) * 4, st));
      bwd(r, w, wave(w, false, rh));
      launches++;
    }
    rh += r;
  }
  k_perm_scale_out<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(d_rhs, ldb, nrhs, h->d_x, n, h->d_pfwd,
                                                                  h->has_scaling ? h->d_scal : nullptr);
  launches++;
  h->solve_launches = launches;
  CK(cudaEventRecord(h->ev[7], st));
  CK(cudaGetLastError());
  return RVG_OK;
}

rvg_status rvg_solve_device(rvg_handle* h, double* d_rhs, int64_t nrhs, int64_t ldb) {
  if (!h) { set_error("null handle"); return RVG_ERR_INVALID_INPUT; }
  if (!h->factored) { set_error("factor() must be called before solve()"); return RVG_ERR_SOLVE_BEFORE_FACTOR; }
  if (nrhs < 0 || (nrhs > 0 && ldb < h->P.n)) { set_error("RHS length must match matrix dimension"); return RVG_ERR_DIMENSION_MISMATCH; }
  CK(cudaSetDevice(h->device));
  int rc = solve_common(h, d_rhs, nrhs, ldb);
  if (rc) return (rvg_status)rc;
  CK(cudaStreamSynchronize(h->st));
  float ms = 0;
  cudaEventElapsedTime(&ms, h->ev[6], h->ev[7]);
  h->t_solve = ms;
  return RVG_OK;
}

rvg_status rvg_solve(rvg_handle* h, double* rhs, int64_t nrhs, int64_t ldb) {
  if (!h) { set_error("null handle"); return RVG_ERR_INVALID_INPUT; }
  if (!h->factored) { set_error("factor() must be called before solve()"); return RVG_ERR_SOLVE_BEFORE_FACTOR; }
  if (nrhs < 0 || (nrhs > 0 && ldb < h->P.n)) { set_error("RHS length must match matrix dimension"); return RVG_ERR_DIMENSION_MISMATCH; }
  if (h->P.n == 0 || nrhs == 0) return RVG_OK;
  CK(cudaSetDevice(h->device));
  double* d = nullptr;
  size_t bytes = (size_t)ldb * (size_t)(nrhs - 1) * 8 + (size_t)h->P.n * 8;
  CK(cudaMallocAsync((void**)&d, bytes, h->st));
  CK(cudaMemcpyAsync(d, rhs, bytes, cudaMemcpyHostToDevice, h->st));
  int rc = solve_common(h, d, nrhs, ldb);
  if (rc) return (rvg_status)rc;
  CK(cudaMemcpyAsync(rhs, d, bytes, cudaMemcpyDeviceToHost, h->st));
  CK(cudaFreeAsync(d, h->st));
  if ((rc = device_wait_status(h))) return (rvg_status)rc;
  float ms = 0;
  cudaEventElapsedTime(&ms, h->ev[6], h->ev[7]);
  h->t_solve = ms;
  return RVG_OK;
}

// nrhs right-hand sides at once (columns at stride ld of b and x): the blocked
// solve, then residuals, norms and corrections of every column until each
// column's scaled backward error is <= tol (or max_iter corrections); bwd[j]
// is column j's final error.
static int refine_common(rvg_handle* h, const double* d_b, double* d_x, int64_t nrhs, int64_t ld, double tol,
                         int32_t max_iter, int32_t* iters, double* bwd, bool* stalled = nullptr) {
  const int64_t n = h->P.n;
  cudaStream_t st = h->st;
  int rc = ensure(h->d_ref, h->ref_cap, (size_t)((nrhs + 1) * n + 3 * nrhs + 8), st);
  if (rc) return rc;
  double* r = h->d_ref;                  // n x nrhs, ld n
  double* nrm = h->d_ref + nrhs * n;     // 3 per column
  if ((rc = ensure_host((char*&)h->h_norms_m, h->h_norms_m_cap, (size_t)(3 * nrhs + 1) * 8))) return rc;
  double* hn = (double*)h->h_norms_m;
  if (ld == n) CK(cudaMemcpyAsync(d_x, d_b, (size_t)(n * nrhs) * 8, cudaMemcpyDeviceToDevice, st));
  else CK(cudaMemcpy2DAsync(d_x, ld * 8, d_b, ld * 8, n * 8, nrhs, cudaMemcpyDeviceToDevice, st));
  if ((rc = solve_common(h, d_x, nrhs, ld))) return rc;
  int it = 0;
  double prev_worst = 0;
  if (stalled) *stalled = false;
  const dim3 g((unsigned)blocks_for(n, 256), (unsigned)nrhs), gn(64, (unsigned)nrhs);
  for (;;) {
    k_residual<<<g, 256, 0, st>>>(h->d_colptr, h->d_rowidx, h->d_vals, d_x, d_b, r, n, ld, n);
    CK(cudaMemsetAsync(nrm, 0, (size_t)(3 * nrhs) * 8, st));
    k_norms3<<<gn, 256, 0, st>>>(r, d_x, d_b, n, nrm, ld, n);
    CK(cudaMemcpyAsync(hn, nrm, (size_t)(3 * nrhs) * 8, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    bool done = true;
    double worst = 0;
    for (int64_t j = 0; j < nrhs; ++j) {
      const double denom = h->a_fro * std::sqrt(hn[3 * j + 1]) + std::sqrt(hn[3 * j + 2]);
      const double e = denom == 0 ? 0.0 : std::sqrt(hn[3 * j]) / denom;
      if (bwd) bwd[j] = e;
      if (!(e <= tol)) done = false;
      worst = std::max(worst, e);
    }
    if (done || it >= max_iter) break;
    // with `stalled` given: stop once a correction no longer halves the error
    if (stalled && it > 0 && !(worst <= 0.5 * prev_worst)) { *stalled = true; break; }
    prev_worst = worst;
    if ((rc = solve_common(h, r, nrhs, n))) return rc;
    k_axpy1<<<g, 256, 0, st>>>(d_x, r, n, ld, n);
    ++it;
  }
  CK(cudaGetLastError());
  if ((rc = device_wait_status(h))) return rc;
  if (iters) *iters = it;
  return RVG_OK;
}

// GMRES-IR: restarted flexible GMRES in FP64 on A x = b with the factor as
// right preconditioner (z_j = solve(v_j), w = A z_j, Gram-Schmidt applied
// twice, Givens rotations on the host, x += Z y at every restart).  It stops
// when the scaled backward error of the true residual, checked at every
// restart and when the rotated residual estimate reaches tol, is <= tol, or
// after max_iter preconditioned products; *iters counts them (one solve each).
static int gmres_common(rvg_handle* h, const double* d_b, double* d_x, double tol, int32_t max_iter, int32_t restart,
                        int32_t* iters, double* bwd, bool x_given = false) {
  const int64_t n = h->P.n;
  cudaStream_t st = h->st;
  const int m = restart;
  // V (m + 1 basis vectors), Z (m preconditioned ones), r / w, coefficients
  int rc = ensure(h->d_gm, h->gm_cap, (size_t)((2 * m + 2) * n + 4 * (m + 2) + 8), st);
  if (rc) return rc;
  double* V = h->d_gm;
  double* Z = V + (int64_t)(m + 1) * n;
  double* w = Z + (int64_t)m * n;
  double* dc = w + n;          // m + 1 coefficients
  double* dn = dc + (m + 2);   // norms
  if ((rc = ensure_host((char*&)h->h_norms_m, h->h_norms_m_cap, (size_t)(4 * (m + 2) + 8) * 8))) return rc;
  double* hn = (double*)h->h_norms_m;
  const unsigned nb = blocks_for(n, 256);
  const dim3 gd(64, 1);
  auto sync_read = [&](const double* src, int cnt) -> int {
    CK(cudaMemcpyAsync(hn, src, (size_t)cnt * 8, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return RVG_OK;
  };
  // true residual r = b - A x into w; its backward error and ||r||
  auto residual = [&](double& e, double& rn) -> int {
    k_residual<<<dim3(nb, 1), 256, 0, st>>>(h->d_colptr, h->d_rowidx, h->d_vals, d_x, d_b, w, n, n, n);
    CK(cudaMemsetAsync(dn, 0, 3 * 8, st));
    k_norms3<<<dim3(64, 1), 256, 0, st>>>(w, d_x, d_b, n, dn, n, n);
    int r2 = sync_read(dn, 3);
    if (r2) return r2;
    const double denom = h->a_fro * std::sqrt(hn[1]) + std::sqrt(hn[2]);
    rn = std::sqrt(hn[0]);
    e = denom == 0 ? 0.0 : rn / denom;
    return RVG_OK;
  };
  if (!x_given) {
    CK(cudaMemcpyAsync(d_x, d_b, n * 8, cudaMemcpyDeviceToDevice, st));
    if ((rc = solve_common(h, d_x, 1, n))) return rc;  // x0 = M^-1 b
  }
  int it = 0;
  double e = 0, beta = 0;
  std::vector<double> H((size_t)(m + 1) * m), cs(m), sn(m), g(m + 1), y(m);
  for (;;) {
    if ((rc = residual(e, beta))) return rc;
    if (e <= tol || it >= max_iter || beta == 0) break;
    // target for the residual estimate: the backward error with the current ||x||
    const double xnorm = std::sqrt(hn[1]), bnorm = std::sqrt(hn[2]);
    const double target = 0.5 * tol * (h->a_fro * xnorm + bnorm);
    k_scale_to<<<nb, 256, 0, st>>>(V, w, 1.0 / beta, n);
    std::fill(g.begin(), g.end(), 0.0);
    g[0] = beta;
    int j = 0;
    for (; j < m && it < max_iter; ++j) {
      double* z = Z + (int64_t)j * n;
      CK(cudaMemcpyAsync(z, V + (int64_t)j * n, n * 8, cudaMemcpyDeviceToDevice, st));
      if ((rc = solve_common(h, z, 1, n))) return rc;
      ++it;
      k_spmv<<<nb, 256, 0, st>>>(h->d_colptr, h->d_rowidx, h->d_vals, z, w, n);
      // Gram-Schmidt twice against v_0..v_j
      for (int pass = 0; pass < 2; ++pass) {
        CK(cudaMemsetAsync(dc, 0, (size_t)(j + 1) * 8, st));
        k_dots<<<dim3(64, (unsigned)(j + 1)), 256, 0, st>>>(V, w, n, dc);
        k_sub_comb<<<nb, 256, 0, st>>>(w, V, dc, j + 1, n);
        if ((rc = sync_read(dc, j + 1))) return rc;
        for (int i = 0; i <= j; ++i) H[(size_t)i * m + j] = (pass ? H[(size_t)i * m + j] : 0.0) + hn[i];
      }
      CK(cudaMemsetAsync(dn, 0, 8, st));
      k_sumsq<<<64, 256, 0, st>>>(w, n, dn);
      if ((rc = sync_read(dn, 1))) return rc;
      const double hn1 = std::sqrt(hn[0]);
      H[(size_t)(j + 1) * m + j] = hn1;
      if (hn1 > 0) k_scale_to<<<nb, 256, 0, st>>>(V + (int64_t)(j + 1) * n, w, 1.0 / hn1, n);
      // Givens rotations
      for (int i = 0; i < j; ++i) {
        const double a = H[(size_t)i * m + j], b2 = H[(size_t)(i + 1) * m + j];
        H[(size_t)i * m + j] = cs[i] * a + sn[i] * b2;
        H[(size_t)(i + 1) * m + j] = -sn[i] * a + cs[i] * b2;
      }
      const double a = H[(size_t)j * m + j], b2 = H[(size_t)(j + 1) * m + j];
      const double rr = std::hypot(a, b2);
      cs[j] = rr == 0 ? 1.0 : a / rr;
      sn[j] = rr == 0 ? 0.0 : b2 / rr;
      H[(size_t)j * m + j] = rr;
      H[(size_t)(j + 1) * m + j] = 0.0;
      g[j + 1] = -sn[j] * g[j];
      g[j] = cs[j] * g[j];
      if (std::fabs(g[j + 1]) <= target || hn1 == 0) { ++j; break; }
    }
    // y = H^-1 g on the leading j x j triangle, x += Z y
    for (int i = j - 1; i >= 0; --i) {
      double s2 = g[i];
      for (int k = i + 1; k < j; ++k) s2 -= H[(size_t)i * m + k] * y[k];
      y[i] = H[(size_t)i * m + i] == 0 ? 0.0 : s2 / H[(size_t)i * m + i];
    }
    if (j > 0) {
      CK(cudaMemcpyAsync(dc, y.data(), (size_t)j * 8, cudaMemcpyHostToDevice, st));
      k_add_comb<<<nb, 256, 0, st>>>(d_x, Z, dc, j, n);
    }
  }
  CK(cudaGetLastError());
  if ((rc = device_wait_status(h))) return rc;
  if (iters) *iters = it;
  if (bwd) *bwd = e;
  return RVG_OK;
}

// Iterative refinement while every correction at least halves the backward
// error, then GMRES-IR from the refined x: the cheap method when it converges,
// the robust one when the factor's error times the condition number is too
// large for it.  *method: 0 refinement alone, 1 escalated to GMRES-IR;
// *iters: the solves after the first one (corrections + GMRES products).
static int auto_common(rvg_handle* h, const double* d_b, double* d_x, double tol, int32_t max_iter, int32_t* iters,
                       double* bwd, int32_t* method) {
  bool stalled = false;
  int32_t it1 = 0, it2 = 0;
  double e = 0;
  int rc = refine_common(h, d_b, d_x, 1, h->P.n, tol, std::min<int32_t>(max_iter, 10), &it1, &e, &stalled);
  if (rc) return rc;
  if (method) *method = 0;
  if (!(e <= tol) && it1 < max_iter) {
    if ((rc = gmres_common(h, d_b, d_x, tol, max_iter - it1, 30, &it2, &e, true))) return rc;
    if (method) *method = 1;
  }
  if (iters) *iters = it1 + it2;
  if (bwd) *bwd = e;
  return RVG_OK;
}

rvg_status rvg_solve_auto_device(rvg_handle* h, const double* d_rhs, double* d_x, double tol, int32_t max_iter,
                                 int32_t* iters, double* bwd_err, int32_t* method) {
  if (!h) { set_error("null handle"); return RVG_ERR_INVALID_INPUT; }
  if (!h->factored) { set_error("factor() must be called before solve()"); return RVG_ERR_SOLVE_BEFORE_FACTOR; }
  if (h->P.n == 0) { if (iters) *iters = 0; if (bwd_err) *bwd_err = 0; if (method) *method = 0; return RVG_OK; }
  CK(cudaSetDevice(h->device));
  double t0 = now_ms();
  int rc = auto_common(h, d_rhs, d_x, tol, max_iter, iters, bwd_err, method);
  h->t_solve = now_ms() - t0;
  return (rvg_status)rc;
}

rvg_status rvg_solve_auto(rvg_handle* h, const double* rhs, double* x, double tol, int32_t max_iter, int32_t* iters,
                          double* bwd_err, int32_t* method) {
  if (!h) { set_error("null handle"); return RVG_ERR_INVALID_INPUT; }
  if (!h->factored) { set_error("factor() must be called before solve()"); return RVG_ERR_SOLVE_BEFORE_FACTOR; }
  const int64_t n = h->P.n;
  if (n == 0) { if (iters) *iters = 0; if (bwd_err) *bwd_err = 0; if (method) *method = 0; return RVG_OK; }
  CK(cudaSetDevice(h->device));
  double t0 = now_ms();
  double* d = nullptr;
  CK(cudaMallocAsync((void**)&d, 2 * n * 8, h->st));
  CK(cudaMemcpyAsync(d, rhs, n * 8, cudaMemcpyHostToDevice, h->st));
  int rc = auto_common(h, d, d + n, tol, max_iter, iters, bwd_err, method);
  if (rc) return (rvg_status)rc;
  CK(cudaMemcpyAsync(x, d + n, n * 8, cudaMemcpyDeviceToHost, h->st));
  CK(cudaFreeAsync(d, h->st));
  CK(cudaStreamSynchronize(h->st));
  h->t_solve = now_ms() - t0;
  return RVG_OK;
}

rvg_status rvg_solve_gmres_device(rvg_handle* h, const double* d_rhs, double* d_x, double tol, int32_t max_iter,
                                  int32_t restart, int32_t* iters, double* bwd_err) {
  if (!h) { set_error("null handle"); return RVG_ERR_INVALID_INPUT; }
  if (!h->factored) { set_error("factor() must be called before solve()"); return RVG_ERR_SOLVE_BEFORE_FACTOR; }
  if (restart < 1 || restart > 200) { set_error("restart must be in [1, 200]"); return RVG_ERR_INVALID_INPUT; }
  if (h->P.n == 0) { if (iters) *iters = 0; if (bwd_err) *bwd_err = 0; return RVG_OK; }
  CK(cudaSetDevice(h->device));
  double t0 = now_ms();
  int rc = gmres_common(h, d_rhs, d_x, tol, max_iter, restart, iters, bwd_err);
  h->t_solve = now_ms() - t0;
  return (rvg_status)rc;
}

rvg_status rvg_solve_gmres(rvg_handle* h, const double* rhs, double* x, double tol, int32_t max_iter, int32_t restart,
                           int32_t* iters, double* bwd_err) {
  if (!h) { set_error("null handle"); return RVG_ERR_INVALID_INPUT; }
  if (!h->factored) { set_error("factor() must be called before solve()"); return RVG_ERR_SOLVE_BEFORE_FACTOR; }
  if (restart < 1 || restart > 200) { set_error("restart must be in [1, 200]"); return RVG_ERR_INVALID_INPUT; }
  const int64_t n = h->P.n;
  if (n == 0) { if (iters) *iters = 0; if (bwd_err) *bwd_err = 0; return RVG_OK; }
  CK(cudaSetDevice(h->device));
  double t0 = now_ms();
  double* d = nullptr;
  CK(cudaMallocAsync((void**)&d, 2 * n * 8, h->st));
  CK(cudaMemcpyAsync(d, rhs, n * 8, cudaMemcpyHostToDevice, h->st));
  int rc = gmres_common(h, d, d + n, tol, max_iter, restart, iters, bwd_err);
  if (rc) return (rvg_status)rc;
  CK(cudaMemcpyAsync(x, d + n, n * 8, cudaMemcpyDeviceToHost, h->st));
  CK(cudaFreeAsync(d, h->st));
  CK(cudaStreamSynchronize(h->st));
  h->t_solve = now_ms() - t0;
  return RVG_OK;
}

rvg_status rvg_solve_refine_device(rvg_handle* h, const double* d_rhs, double* d_x, double tol, int32_t max_iter,
                                   int32_t* iters, double* bwd_err) {
  if (!h) { set_error("null handle"); return RVG_ERR_INVALID_INPUT; }
  if (!h->factored) { set_error("factor() must be called before solve()"); return RVG_ERR_SOLVE_BEFORE_FACTOR; }
  if (h->P.n == 0) { if (iters) *iters = 0; if (bwd_err) *bwd_err = 0; return RVG_OK; }
  CK(cudaSetDevice(h->device));
  double t0 = now_ms();
  int rc = refine_common(h, d_rhs, d_x, 1, h->P.n, tol, max_iter, iters, bwd_err);
  h->t_solve = now_ms() - t0;
  return (rvg_status)rc;
}

rvg_status rvg_solve_refine(rvg_handle* h, const double* rhs, double* x, double tol, int32_t max_iter, int32_t* iters,
                            double* bwd_err) {
  if (!h) { set_error("null handle"); return RVG_ERR_INVALID_INPUT; }
  if (!h->factored) { set_error("factor() must be called before solve()"); return RVG_ERR_SOLVE_BEFORE_FACTOR; }
  const int64_t n = h->P.n;
  if (n == 0) { if (iters) *iters = 0; if (bwd_err) *bwd_err = 0; return RVG_OK; }
  CK(cudaSetDevice(h->device));
  double t0 = now_ms();
  double* d = nullptr;
  CK(cudaMallocAsync((void**)&d, 2 * n * 8, h->st));
  CK(cudaMemcpyAsync(d, rhs, n * 8, cudaMemcpyHostToDevice, h->st));
  int rc = refine_common(h, d, d + n, 1, n, tol, max_iter, iters, bwd_err);
  if (rc) return (rvg_status)rc;
  CK(cudaMemcpyAsync(x, d + n, n * 8, cudaMemcpyDeviceToHost, h->st));
  CK(cudaFreeAsync(d, h->st));
  CK(cudaStreamSynchronize(h->st));
  h->t_solve = now_ms() - t0;
  return RVG_OK;
}

rvg_status rvg_solve_refine_nrhs_device(rvg_handle* h, const double* d_rhs, double* d_x, int64_t nrhs, int64_t ldb,
                                        double tol, int32_t max_iter, int32_t* iters, double* bwd_err) {
  if (!h) { set_error("null handle"); return RVG_ERR_INVALID_INPUT; }
  if (!h->factored) { set_error("factor() must be called before solve()"); return RVG_ERR_SOLVE_BEFORE_FACTOR; }
  const int64_t n = h->P.n;
  if (nrhs < 1 || ldb < n || (n > 0 && (!d_rhs || !d_x))) { set_error("need nrhs >= 1, ldb >= n and both vectors"); return RVG_ERR_INVALID_INPUT; }
  if (n == 0) { if (iters) *iters = 0; if (bwd_err) for (int64_t j = 0; j < nrhs; ++j) bwd_err[j] = 0; return RVG_OK; }
  CK(cudaSetDevice(h->device));
  double t0 = now_ms();
  int rc = refine_common(h, d_rhs, d_x, nrhs, ldb, tol, max_iter, iters, bwd_err);
  h->t_solve = now_ms() - t0;
  return (rvg_status)rc;
}

rvg_status rvg_solve_refine_nrhs(rvg_handle* h, const double* rhs, double* x, int64_t nrhs, int64_t ldb, double tol,
                                 int32_t max_iter, int32_t* iters, double* bwd_err) {
  if (!h) { set_error("null handle"); return RVG_ERR_INVALID_INPUT; }
  if (!h->factored) { set_error("factor() must be called before solve()"); return RVG_ERR_SOLVE_BEFORE_FACTOR; }
  const int64_t n = h->P.n;
  if (nrhs < 1 || ldb < n || (n > 0 && (!rhs || !x))) { set_error("need nrhs >= 1, ldb >= n and both arrays"); return RVG_ERR_INVALID_INPUT; }
  if (n == 0) { if (iters) *iters = 0; if (bwd_err) for (int64_t j = 0; j < nrhs; ++j) bwd_err[j] = 0; return RVG_OK; }
  CK(cudaSetDevice(h->device));
  double t0 = now_ms();
  double* d = nullptr;
  CK(cudaMallocAsync((void**)&d, 2 * (size_t)(n * nrhs) * 8, h->st));
  CK(cudaMemcpy2DAsync(d, n * 8, rhs, ldb * 8, n * 8, nrhs, cudaMemcpyHostToDevice, h->st));
  int rc = refine_common(h, d, d + n * nrhs, nrhs, n, tol, max_iter, iters, bwd_err);
  if (rc) return (rvg_status)rc;
  CK(cudaMemcpy2DAsync(x, ldb * 8, d + n * nrhs, n * 8, n * 8, nrhs, cudaMemcpyDeviceToHost, h->st));
  CK(cudaFreeAsync(d, h->st));
  CK(cudaStreamSynchronize(h->st));
  h->t_solve = now_ms() - t0;
  return RVG_OK;
}

rvg_status rvg_inertia(rvg_handle* h, int64_t out3[3]) {
  if (!h) { set_error("null handle"); return RVG_ERR_INVALID_INPUT; }
  if (!h->factored) { set_error("factor() must be called first"); return RVG_ERR_SOLVE_BEFORE_FACTOR; }
  int64_t pos = 0, neg = 0, zer = 0;
  int64_t tot = 0;
  for (auto& f : h->h_fronts) tot = std::max<int64_t>(tot, f.dpos + f.k);
  std::vector<int8_t> dt(tot);
  std::vector<double> dd(tot), dof(tot);
  if (tot) {
    CK(cudaMemcpy(dt.data(), h->dtype, tot, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(dd.data(), h->ddiag, tot * 8, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(dof.data(), h->doff, tot * 8, cudaMemcpyDeviceToHost));
  }
  // MixedDiagonal::compute_inertia (diagonal.rs:391-461) per front
  for (auto& f : h->h_fronts) {
    int c = 0;
    while (c < f.ne) {
      int64_t q = f.dpos + c;
      if (dt[q] == PT_1X1) {
        double d = dd[q];
        if (d > 0) pos++; else if (d < 0) neg++; else zer++;
        c += 1;
      } else {
        double a = dd[q], b = dof[q], cc = dd[q + 1];
        double det = a * cc - b * b, tr = a + cc;
        if (det > 0) { if (tr > 0) pos += 2; else neg += 2; }
        else if (det < 0) { pos++; neg++; }
        else { if (tr > 0) { pos++; zer++; } else if (tr < 0) { neg++; zer++; } else zer += 2; }
        c += 2;
      }
    }
  }
  out3[0] = pos; out3[1] = neg; out3[2] = zer;
  return RVG_OK;
}

rvg_status rvg_get_stats(rvg_handle* h, rvg_stats* o) {
  if (!h || !o) { set_error("null argument"); return RVG_ERR_INVALID_INPUT; }
  if (!h->factored) { set_error("factor() must be called first"); return RVG_ERR_SOLVE_BEFORE_FACTOR; }
  o->total_1x1_pivots = h->tot1;
  o->total_2x2_pivots = h->tot2;
  o->total_delayed = h->totdel;
  o->zero_pivots = h->zero_piv;
  o->max_front_size = h->max_front;
  o->supernodes_before_amalgamation = h->P.nsup_before;
  o->supernodes_after_amalgamation = (int64_t)h->P.sn.size();
  o->merges_performed = h->P.merges;
  o->small_leaf_subtrees = h->P.sl_subtrees;
  o->small_leaf_nodes = h->P.sl_nodes;
  return RVG_OK;
}

rvg_status rvg_pivot_record(rvg_handle* h, int64_t* col, int8_t* code, double* d_diag, double* d_off, int64_t* count) {
  if (!h || !count) { set_error("null argument"); return RVG_ERR_INVALID_INPUT; }
  if (!h->factored) { set_error("factor() must be called first"); return RVG_ERR_SOLVE_BEFORE_FACTOR; }
  int64_t tot = 0, isz = 0;
  for (auto& f : h->h_fronts) { tot = std::max<int64_t>(tot, f.dpos + f.k); isz = std::max<int64_t>(isz, f.idx + f.m + f.k); }
  std::vector<int8_t> dt(tot);
  std::vector<double> dd(tot), dof(tot);
  std::vector<int32_t> ix(isz);
  if (tot) {
    CK(cudaMemcpy(dt.data(), h->dtype, tot, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(dd.data(), h->ddiag, tot * 8, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(dof.data(), h->doff, tot * 8, cudaMemcpyDeviceToHost));
  }
  if (isz) CK(cudaMemcpy(ix.data(), h->idx, isz * 4, cudaMemcpyDeviceToHost));
  int64_t t = 0;
  for (auto& f : h->h_fronts) {
    const int32_t* rows = ix.data() + f.idx;
    const int32_t* perm = rows + f.m;
    for (int c = 0; c < f.ne; ++c) {
      int64_t q = f.dpos + c;
      if (col) col[t] = rows[perm[c]];
      int8_t cd = dt[q];
      if (code) code[t] = cd;
      if (d_diag) d_diag[t] = dd[q];
      if (d_off) d_off[t] = cd == 2 ? dof[q] : 0.0;
      ++t;
    }
  }
  *count = t;
  return RVG_OK;
}

rvg_status rvg_front_info(rvg_handle* h, int64_t* out9, int64_t* nsup) {
  if (!h || !nsup) { set_error("null argument"); return RVG_ERR_INVALID_INPUT; }
  *nsup = (int64_t)h->P.sn.size();
  if (!out9) return RVG_OK;
  for (size_t s = 0; s < h->P.sn.size(); ++s) {
    const DFront& f = h->factored ? h->h_fronts[s] : DFront();
    int64_t* o = out9 + 9 * s;
    o[0] = f.m; o[1] = f.k; o[2] = f.ne; o[3] = f.n1; o[4] = f.n2; o[5] = h->P.sn[s].parent;
    o[6] = h->P.sn[s].n_owned(); o[7] = h->P.sn[s].in_small_leaf ? 1 : 0; o[8] = h->P.height[s];
  }
  return RVG_OK;
}

rvg_status rvg_work(rvg_handle* h, double out6[6]) {
  if (!h) { set_error("null handle"); return RVG_ERR_INVALID_INPUT; }
  Plan& P = h->P;
  double solve_bytes = 0;
  for (auto& s : P.sn) {
    double k = (double)s.n_owned(), r = (double)s.pattern.size();
    double stored = k * (k + 1) / 2 + r * k;
    solve_bytes += 2 * 8 * stored + 8 * k + 2 * 4 * (k + r) + 2 * 2 * 8 * (k + r);
  }
  out6[0] = P.flops_factor; out6[1] = P.flops_schur; out6[2] = P.bytes_assembly; out6[3] = solve_bytes;
  out6[4] = (double)P.nnz_l; out6[5] = (double)P.max_front;
  return RVG_OK;
}

rvg_status rvg_timings(rvg_handle* h, double out7[7]) {
  if (!h) { set_error("null handle"); return RVG_ERR_INVALID_INPUT; }
  out7[0] = h->t_assembly; out7[1] = h->t_kernel; out7[2] = h->t_gemm; out7[3] = h->t_factor; out7[4] = h->t_solve;
  out7[5] = h->t_dom; out7[6] = h->n_dom;
  return RVG_OK;
}

rvg_status rvg_set_profiling(rvg_handle* h, int32_t enable) {
  if (!h) { set_error("null handle"); return RVG_ERR_INVALID_INPUT; }
  h->profiling = enable != 0;
  return RVG_OK;
}

// A one-thread wait on a flag that nothing raises (the solve's flag wait).
__global__ void k_wait_probe(const int32_t* flag, int32_t* err) { sf_wait(flag, err); }

rvg_status rvg_selftest_waits(rvg_handle* h, int32_t which) {
  if (!h) { set_error("null handle"); return RVG_ERR_INVALID_INPUT; }
  if (which != 0 && which != 1) { set_error("which must be 0 (solve flag) or 1 (tensor-core pipeline)"); return RVG_ERR_INVALID_INPUT; }
  CK(cudaSetDevice(h->device));
  cudaStream_t st = h->st;
  int rc = device_wait_status(h);  // start from a clean error word
  if (rc) return (rvg_status)rc;
  if ((rc = ensure(h->sf_sync, h->sf_sync_cap, 2, st))) return (rvg_status)rc;
  CK(cudaMemsetAsync(h->sf_sync, 0, 2 * sizeof(int32_t), st));
  if (which == 0) {
    k_wait_probe<<<1, 1, 0, st>>>(h->sf_sync, h->d_err);
  } else {
    // one 128 x 128 tile, K = 32, operands never copied in: the MMA warp's wait runs out
    double* c = nullptr;
    float* p = nullptr;
    CK(cudaMallocAsync((void**)&c, 128 * 128 * sizeof(double), st));
    CK(cudaMallocAsync((void**)&p, 2 * (size_t)TC_BLOCK * sizeof(float), st));
    TcArgs ta{c, 128, 0, 128, 0, 128, p, p + TC_BLOCK, 1, nullptr, 32, 1, 1, 1, h->d_err, nullptr, 0, 1};
    k_syrk_tc<4, TC_TF32><<<1, TC_THREADS, TC_SMEM, st>>>(ta);
    CK(cudaFreeAsync(c, st));
    CK(cudaFreeAsync(p, st));
  }
  CK(cudaGetLastError());
  return (rvg_status)device_wait_status(h);
}

rvg_status rvg_get_profile(rvg_handle* h, rvg_profile* o) {
  if (!h || !o) { set_error("null argument"); return RVG_ERR_INVALID_INPUT; }
  o->factor_ms = h->t_factor;
  o->solve_ms = h->t_solve;
  o->assembly_ms = h->t_assembly;
  o->dense_ms = h->t_kernel;
  o->cbgemm_ms = h->t_gemm;
  o->syrk_ms = h->syrk_ms;
  o->syrk_flops = h->syrk_flops;
  o->syrk_launches = h->syrk_launches;
  o->factor_launches = h->factor_launches;
  o->solve_launches = h->solve_launches;
  o->peak_bytes = h->peak_bytes;
  o->host_total_ms = h->host_total_ms;
  o->host_alloc_ms = h->host_alloc_ms;
  o->host_sync_ms = h->host_sync_ms;
  for (int i = 0; i < RVG_PARTS; ++i) o->part_ms[i] = h->part_ms[i];
  o->host_wait_ms = h->host_wait_ms;
  o->lf_misses = h->lf_misses;
  o->host_gap_ms = h->host_gap_ms;
  o->lf_far_updates = h->lf_far;
  return RVG_OK;
}

static int trim_buf(void* p, cudaStream_t st) {
  if (p) CK(cudaFreeAsync(p, st));
  return RVG_OK;
}

static float ubits(unsigned u) {
  float f;
  std::memcpy(&f, &u, 4);
  return f;
}

rvg_status rvg_set_selector(rvg_handle* h, const float* params, int64_t nparams, float threshold,
                            double growth_bound) {
  if (!h || !params) { set_error("null argument"); return RVG_ERR_INVALID_INPUT; }
  if (nparams != MLP_NPARAM) { set_error("selector parameters: expected rvg_mlp_param_count() floats"); return RVG_ERR_DIMENSION_MISMATCH; }
  for (int c = 0; c < MLP_IN; ++c)
    if (!(params[MLP_SD + c] > 0.f)) { set_error("selector normalisation: standard deviations must be positive"); return RVG_ERR_INVALID_INPUT; }
  if (!(growth_bound > 0)) { set_error("growth bound must be positive"); return RVG_ERR_INVALID_INPUT; }
  CK(cudaSetDevice(h->device));
  if (!h->d_sel) CK(cudaMalloc((void**)&h->d_sel, MLP_NPARAM * sizeof(float)));
  CK(cudaMemcpyAsync(h->d_sel, params, MLP_NPARAM * sizeof(float), cudaMemcpyHostToDevice, h->st));
  CK(cudaStreamSynchronize(h->st));
  h->sel_thresh = threshold;
  h->sel_bound = growth_bound;
  return RVG_OK;
}

rvg_status rvg_front_features(rvg_handle* h, double* out, int64_t cap_rows, int64_t* nrows) {
  if (!h || !nrows) { set_error("null argument"); return RVG_ERR_INVALID_INPUT; }
  if (!h->factored || h->opt.precision != 2) { set_error("no learned-precision factorization to report"); return RVG_ERR_SOLVE_BEFORE_FACTOR; }
  *nrows = (int64_t)h->sel_large.size();
  if (!out) return RVG_OK;
  if (cap_rows < *nrows) { set_error("feature table: too few rows"); return RVG_ERR_DIMENSION_MISMATCH; }
  std::vector<unsigned> rows((size_t)h->P.sn.size() * FEAT_STRIDE);
  if (!rows.empty()) CK(cudaMemcpy(rows.data(), h->d_feat, rows.size() * 4, cudaMemcpyDeviceToHost));
  for (size_t i = 0; i < h->sel_large.size(); ++i) {
    const int32_t s = h->sel_large[i];
    const DFront& f = h->h_fronts[s];
    const unsigned* r = rows.data() + (size_t)s * FEAT_STRIDE;
    double* o = out + i * RVG_FRONT_FEATURE_COLS;
    o[0] = s; o[1] = f.m; o[2] = f.k; o[3] = f.ne; o[4] = f.n1; o[5] = f.n2;
    o[6] = ubits(r[21]);  // route
    o[7] = ubits(r[20]);  // probability
    o[8] = ubits(r[0]);   // max |a|
    o[9] = ubits(r[7]);   // max |D|
    for (int c = 0; c < MLP_IN; ++c) o[10 + c] = ubits(r[8 + c]);
  }
  return RVG_OK;
}

rvg_status rvg_selector_stats(rvg_handle* h, int64_t out4[4]) {
  if (!h || !out4) { set_error("null argument"); return RVG_ERR_INVALID_INPUT; }
  out4[0] = (int64_t)h->sel_large.size();
  out4[1] = h->sel_routed;
  out4[2] = h->sel_flagged;
  out4[3] = h->sel_fallback;
  return RVG_OK;
}

rvg_status rvg_trim(rvg_handle* h, int32_t what) {
  if (!h) { set_error("null handle"); return RVG_ERR_INVALID_INPUT; }
  if (what & ~3) { set_error("what: bit 0 = workspace, bit 1 = factor"); return RVG_ERR_INVALID_INPUT; }
  CK(cudaSetDevice(h->device));
  cudaStream_t st = h->st;
  int rc;
#define RVG_TRIM(p, cap)                              \
  do {                                                \
    if ((rc = trim_buf(p, st))) return (rvg_status)rc; \
    p = nullptr;                                      \
    cap = 0;                                          \
  } while (0)
  if (h->vm && what) CK(cudaDeviceSynchronize());  // nothing may use an arena whose memory goes
  auto vm_trim = [&](int id, auto*& p, size_t& cap) {  // address-stable arenas: the memory goes, the addresses stay
    vm_unmap(h->vm->slot[id]);
    p = nullptr;
    cap = 0;
  };
  if ((what & 1) && h->vm) {
    vm_trim(VM_SCRATCH, h->scratch, h->scratch_cap);
    vm_trim(VM_CB, h->cb_arena, h->cb_cap);
    vm_trim(VM_PACK, h->pack, h->pack_cap);
    vm_trim(VM_WPACK0, h->wpack, h->wpack_cap);
    for (size_t t = 1; t < h->lfx.size(); ++t) vm_trim(VM_WPACK0 + (int)t, h->lfx[t].wpack, h->lfx[t].wpack_cap);
    if (!h->lfx.empty()) { h->lfx[0].wpack = nullptr; h->lfx[0].wpack_cap = 0; }
    vm_trim(VM_STAGE, h->d_stage, h->stage_cap);
  } else if (what & 1) {
    RVG_TRIM(h->scratch, h->scratch_cap);
    RVG_TRIM(h->cb_arena, h->cb_cap);
    RVG_TRIM(h->pack, h->pack_cap);
    RVG_TRIM(h->wpack, h->wpack_cap);
    for (size_t t = 1; t < h->lfx.size(); ++t) RVG_TRIM(h->lfx[t].wpack, h->lfx[t].wpack_cap);
    if (!h->lfx.empty()) { h->lfx[0].wpack = nullptr; h->lfx[0].wpack_cap = 0; }
    RVG_TRIM(h->d_stage, h->stage_cap);
  }
  if (what & 1) {
    RVG_TRIM(h->solve_work, h->solve_work_cap);
    RVG_TRIM(h->sf_part, h->sf_part_cap);
    RVG_TRIM(h->d_x, h->x_cap);
    RVG_TRIM(h->d_ref, h->ref_cap);
    RVG_TRIM(h->d_gm, h->gm_cap);
    RVG_TRIM(h->d_stage2, h->stage2_cap);
    h->cb_free.clear();
  }
  if ((what & 2) && h->vm) {
    vm_trim(VM_PANEL, h->panel, h->panel_cap);
    vm_trim(VM_IDX, h->idx, h->idx_cap);
    size_t c1 = 0, c2 = 0;
    vm_trim(VM_DTYPE, h->dtype, h->d_cap);
    vm_trim(VM_DDIAG, h->ddiag, c1);
    vm_trim(VM_DOFF, h->doff, c2);
    h->factored = false;
  } else if (what & 2) {
    RVG_TRIM(h->panel, h->panel_cap);
    RVG_TRIM(h->idx, h->idx_cap);
    if ((rc = trim_buf(h->dtype, st)) || (rc = trim_buf(h->ddiag, st)) || (rc = trim_buf(h->doff, st)))
      return (rvg_status)rc;
    h->dtype = nullptr; h->ddiag = nullptr; h->doff = nullptr; h->d_cap = 0;
    h->factored = false;
  }
#undef RVG_TRIM
  if (what) {
    h->need_presize = true;
    if (!h->vm) drop_graph(h);  // it holds the addresses of the released buffers (kept in the vm mode)
  }
  CK(cudaStreamSynchronize(st));  // the memory is back in the pool when this returns
  return RVG_OK;
}

rvg_status rvg_mem_info(int64_t out2[2]) {
  if (!out2) { set_error("null argument"); return RVG_ERR_INVALID_INPUT; }
  size_t f = 0, t = 0;
  CK(cudaMemGetInfo(&f, &t));
  out2[0] = (int64_t)f;
  out2[1] = (int64_t)t;
  return RVG_OK;
}

rvg_status rvg_stream(rvg_handle* h, void** s) {
  if (!h || !s) { set_error("null argument"); return RVG_ERR_INVALID_INPUT; }
  *s = (void*)h->st;
  return RVG_OK;
}

void rvg_destroy(rvg_handle* h) {
  if (!h) return;
  cudaSetDevice(h->device);
  cudaStream_t st = h->st;
  auto fr = [&](void* p) { if (p) cudaFreeAsync(p, st); };
  fr(h->d_own_ptr); fr(h->d_own_idx); fr(h->d_pat_ptr); fr(h->d_pat_idx); fr(h->d_amap_ptr); fr(h->d_amap);
  fr(h->d_ea_ptr); fr(h->d_ea_map); fr(h->d_ch_ptr); fr(h->d_ch_idx); fr(h->d_pfwd); fr(h->d_fronts);
  if (!h->vm) {  // (address-stable arenas are released by vm_destroy below)
    fr(h->panel); fr(h->idx); fr(h->dtype); fr(h->ddiag); fr(h->doff);
    fr(h->d_stage); fr(h->scratch); fr(h->cb_arena); fr(h->pack); fr(h->wpack);
  }
  fr(h->d_vals); fr(h->d_scal);
  fr(h->d_x); fr(h->solve_work); fr(h->d_stage2); fr(h->d_lf); fr(h->sf_sync); fr(h->sf_part); fr(h->d_gm);
  drop_graph(h);
  fr(h->d_rec);
  if (h->d_sel) cudaFree(h->d_sel);
  fr(h->d_feat);
  if (h->d_sel_flag) cudaFree(h->d_sel_flag);
  if (h->d_nonfinite) cudaFree(h->d_nonfinite);
  if (h->d_mismatch) cudaFree(h->d_mismatch);
  if (h->h_stage_all) cudaFreeHost(h->h_stage_all);
  for (size_t t = 0; t < h->lfx.size(); ++t) {
    LfCtx& c = h->lfx[t];
    if (c.h_gne) cudaFreeHost(c.h_gne);
    for (auto& e : c.ring_ev) if (e) cudaEventDestroy(e);
    if (c.far_st) { cudaStreamSynchronize(c.far_st); cudaStreamDestroy(c.far_st); }
    if (c.ev_fork) cudaEventDestroy(c.ev_fork);
    if (c.ev_far) cudaEventDestroy(c.ev_far);
    if (t == 0) continue;  // the handle's own stream, state and window buffer
    if (!h->vm) fr(c.wpack);
    if (c.lf) cudaFree(c.lf);
    if (c.own && c.st) { cudaStreamSynchronize(c.st); cudaStreamDestroy(c.st); }
  }
  fr(h->d_err);
  fr(h->d_colptr); fr(h->d_rowidx); fr(h->d_ref);
  if (st) { cudaStreamSynchronize(st); cudaStreamDestroy(st); }
  vm_destroy(h);
  if (h->h_stage) cudaFreeHost(h->h_stage);
  if (h->h_stage2) cudaFreeHost(h->h_stage2);
  if (h->h_counts) cudaFreeHost(h->h_counts);
  if (h->h_norms) cudaFreeHost(h->h_norms);
  if (h->h_norms_m) cudaFreeHost(h->h_norms_m);
  for (auto e : h->ev_pool) cudaEventDestroy(e);
  for (auto e : h->mk_pool) cudaEventDestroy(e);
  for (auto& e : h->ev) if (e) cudaEventDestroy(e);
  delete h;
  cudaGetLastError();  // nothing of this handle's teardown is left for the caller's next call to report
}

}  // extern "C"
