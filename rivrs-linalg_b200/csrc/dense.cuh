// Dense APTP building blocks for one front, on sm_100a.
//
// A front is stored as an m x k column-major panel (leading dimension m): the
// k fully-summed columns of the reference's m x m frontal matrix.  The APTP
// kernel never reads or writes columns >= k (swaps stay inside the FS
// columns, updates stop at the NFS boundary: sparse/src/symmetric/factor.rs:
// 1418-1526, 2616-2683), so the NFS x NFS block lives in a separate
// contribution buffer.
//
// Two executors:
//   * warp_tpp_*  : one warp runs threshold partial pivoting
//                   (factor.rs:2335-2506, 2761-2947); used for small-leaf
//                   fronts, fronts with k < ib, and the TPP fallback.
//   * cta_aptp_*  : one CTA runs the blocked APTP (factor_inner,
//                   factor.rs:1811-2095, and two_level_factor,
//                   factor.rs:2108-2252), with the 32x32 complete-pivoting
//                   block (factor.rs:891-1153) done by one warp in shared
//                   memory with warp-shuffle arg-max reductions.
// Per-entry arithmetic follows the oracle's operation order, so the values a
// front produces match the oracle's bit for bit wherever no cross-thread
// reduction order is involved.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace rvg {

// pivot codes: 1x1, first and second column of a 2x2 pair
enum : int8_t { PT_DELAYED = 0, PT_1X1 = 1, PT_2X2 = 2, PT_2X2B = 3 };

// Programmatic dependent launch.  A kernel launched with programmatic stream
// serialization may start while the kernel before it on the stream still
// runs; chain_enter() is its first statement: it waits until that kernel has
// completed and its stores are visible (a no-op for a plain launch), then lets
// the next kernel of the stream be launched early in turn.  Every kernel that
// may be launched this way calls it unconditionally, so completion is
// transitive along the chain.
__device__ __forceinline__ void chain_enter() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

struct DevOpts {
  double threshold;
  double small;
  int nb;
  int ib;
  int failed_pivot_tpp;
};

struct PanelView {
  double* a;
  int64_t ld;
  __device__ __forceinline__ double& operator()(int64_t i, int64_t j) const { return a[i + j * ld]; }
};

// ---------------------------------------------------------------------------
// warp reductions
// ---------------------------------------------------------------------------
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
// arg-max keeping the smallest key among equal values (first occurrence in
// the serial scan order encoded by `key`).
__device__ __forceinline__ void warp_argmax(double& v, int64_t& key) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    double ov = __shfl_xor_sync(0xffffffffu, v, o);
    int64_t ok = __shfl_xor_sync(0xffffffffu, key, o);
    if (ov > v || (ov == v && ok < key)) { v = ov; key = ok; }
  }
}

// ---------------------------------------------------------------------------
// Pivot record of a front: type / diag / off per eliminated position.
// ---------------------------------------------------------------------------
struct DRec {
  int8_t* type;    // PT_*
  double* diag;
  double* off;     // off-diagonal stored on the first column of a 2x2
};

// ---------------------------------------------------------------------------
// Warp TPP (factor.rs:2268-2947).  `nc` is the stored width (k); all column
// indices used are < n <= nc.  perm has n entries (the FS part of col_order).
// ---------------------------------------------------------------------------
struct WarpTpp {
  PanelView a;
  int64_t m, nc;
  int lane;

  __device__ double sym(int64_t row, int64_t col) const {  // factor.rs:2597-2606
    return (col < nc && row >= col) ? a(row, col) : a(col, row);
  }
  __device__ bool col_small(int64_t idx, int64_t from, int64_t to, double small) const {  // 2674-2690
    bool big = false;
    int64_t ce = idx < nc ? idx : nc;
    for (int64_t c = from + lane; c < ce; c += 32) big |= fabs(a(idx, c)) >= small;
    if (idx < nc)
      for (int64_t r = idx + lane; r < to; r += 32) big |= fabs(a(r, idx)) >= small;
    return !__any_sync(0xffffffffu, big);
  }
  __device__ int64_t row_abs_max(int64_t p, int64_t from, int64_t to) const {  // 2695-2710
    if (from >= to) return from;
    double bv = -1.0;
    int64_t bk = INT64_MAX;
    for (int64_t c = from + lane; c < to; c += 32) {
      double v = fabs(sym(p, c));
      if (v > bv) { bv = v; bk = c; }
    }
    warp_argmax(bv, bk);
    return bk;
  }
  __device__ double rc_abs_max_excl(int64_t col, int64_t nelim, int64_t excl) const {  // 2715-2737
    double best = 0.0;
    int64_t ce = col < nc ? col : nc;
    for (int64_t c = nelim + lane; c < ce; c += 32) if (c != excl) best = fmax(best, fabs(a(col, c)));
    if (col < nc)
      for (int64_t r = col + 1 + lane; r < m; r += 32) if (r != excl) best = fmax(best, fabs(a(r, col)));
    return warp_max(best);
  }
  __device__ bool test_2x2(int64_t t, int64_t p, double maxt, double maxp, double u, double small) const {
    double a11 = a(t, t), a21 = a(p, t), a22 = a(p, p);  // factor.rs:2268-2315
    double maxpiv = fmax(fmax(fabs(a11), fabs(a21)), fabs(a22));
    if (maxpiv < small) return false;
    double ds = 1.0 / maxpiv;
    double dp0 = (a11 * ds) * a22, dp1 = (a21 * ds) * a21, dp = dp0 - dp1;
    if (fabs(dp) < fmax(fmax(small, fabs(dp0 / 2.0)), fabs(dp1 / 2.0))) return false;
    double di11 = (a22 * ds) / dp, di12 = (-a21 * ds) / dp, di22 = (a11 * ds) / dp;
    if (fmax(maxt, maxp) < small) return true;
    double x1 = fabs(di11) * maxt + fabs(di12) * maxp;
    double x2 = fabs(di12) * maxt + fabs(di22) * maxp;
    return u * fmax(x1, x2) < 1.0;
  }
  __device__ void swap(int64_t i, int64_t j) const {  // swap_rect (2528-2580), i,j < nc
    if (i == j) return;
    if (i > j) { int64_t t = i; i = j; j = t; }
    __syncwarp();
    if (lane == 0) { double t = a(i, i); a(i, i) = a(j, j); a(j, j) = t; }
    for (int64_t k = lane; k < i; k += 32) { double t = a(i, k); a(i, k) = a(j, k); a(j, k) = t; }
    for (int64_t k = i + 1 + lane; k < j; k += 32) { double t = a(k, i); a(k, i) = a(j, k); a(j, k) = t; }
    for (int64_t k = j + 1 + lane; k < m; k += 32) { double t = a(k, i); a(k, i) = a(k, j); a(k, j) = t; }
    __syncwarp();
  }
  __device__ void apply_1x1(int64_t ne, int64_t p) const {  // 2616-2641
    double d = a(ne, ne), inv = 1.0 / d;
    for (int64_t i = ne + 1 + lane; i < m; i += 32) a(i, ne) = a(i, ne) * inv;
    __syncwarp();
    int64_t ce = p < nc ? p : nc;
    for (int64_t j = ne + 1; j < ce; ++j) {
      double ldlj = a(j, ne) * d;
      for (int64_t i = j + lane; i < m; i += 32) a(i, j) -= a(i, ne) * ldlj;
    }
    __syncwarp();
  }
  __device__ void apply_2x2(int64_t ne, int64_t p) const {  // 2649-2683
    double a11 = a(ne, ne), a21 = a(ne + 1, ne), a22 = a(ne + 1, ne + 1);
    double det = a11 * a22 - a21 * a21, inv_det = 1.0 / det;
    for (int64_t i = ne + 2 + lane; i < m; i += 32) {
      double ai1 = a(i, ne), ai2 = a(i, ne + 1);
      a(i, ne) = (ai1 * a22 - ai2 * a21) * inv_det;
      a(i, ne + 1) = (ai2 * a11 - ai1 * a21) * inv_det;
    }
    __syncwarp();
    int64_t ce = p < nc ? p : nc;
    for (int64_t j = ne + 2; j < ce; ++j) {
      double w1 = a(j, ne) * a11 + a(j, ne + 1) * a21, w2 = a(j, ne) * a21 + a(j, ne + 1) * a22;
      for (int64_t i = j + lane; i < m; i += 32) a(i, j) -= a(i, ne) * w1 + a(i, ne + 1) * w2;
    }
    __syncwarp();
    if (lane == 0) a(ne + 1, ne) = 0.0;
    __syncwarp();
  }
  __device__ void zero_col(int64_t ne) const {
    if (ne < nc)
      for (int64_t r = ne + 1 + lane; r < m; r += 32) a(r, ne) = 0.0;
    __syncwarp();
  }

  // The TPP loop (shared body of tpp_factor / tpp_factor_rect).  Returns the
  // number of columns eliminated from `start`; counters are updated by lane 0.
  __device__ int64_t run(int64_t start, int64_t n, int32_t* perm, DRec d, int* n1, int* n2,
                         const DevOpts& o) const {
    const double u = o.threshold, small = o.small;
    int64_t ne = start;
    while (ne < n) {
      if (col_small(ne, ne, m, small)) {
        if (lane == 0) { d.type[ne] = PT_1X1; d.diag[ne] = 0.0; d.off[ne] = 0.0; (*n1)++; }
        zero_col(ne);
        ne += 1;
        continue;
      }
      bool found = false;
      for (int64_t p = ne + 1; p < n; ++p) {
        if (col_small(p, ne, m, small)) {
          if (p != ne) {
            swap(p, ne);
            if (lane == 0) { int32_t t = perm[p]; perm[p] = perm[ne]; perm[ne] = t; }
          }
          if (lane == 0) { d.type[ne] = PT_1X1; d.diag[ne] = 0.0; d.off[ne] = 0.0; (*n1)++; }
          for (int64_t r = ne + 1 + lane; r < m; r += 32) a(r, ne) = 0.0;
          __syncwarp();
          ne += 1;
          found = true;
          break;
        }
        int64_t t = row_abs_max(p, ne, p);
        double maxt = rc_abs_max_excl(t, ne, p);
        double maxp = rc_abs_max_excl(p, ne, t);
        if (test_2x2(t, p, maxt, maxp, u, small)) {
          if (t != ne) {
            swap(t, ne);
            if (lane == 0) { int32_t q = perm[t]; perm[t] = perm[ne]; perm[ne] = q; }
          }
          int64_t np = (p == ne) ? t : p;
          if (np != ne + 1) {
            swap(np, ne + 1);
            if (lane == 0) { int32_t q = perm[np]; perm[np] = perm[ne + 1]; perm[ne + 1] = q; }
          }
          double d11 = a(ne, ne), d21 = a(ne + 1, ne), d22 = a(ne + 1, ne + 1);
          apply_2x2(ne, n);
          if (lane == 0) {
            d.type[ne] = PT_2X2; d.type[ne + 1] = PT_2X2B;
            d.diag[ne] = d11; d.diag[ne + 1] = d22; d.off[ne] = d21; d.off[ne + 1] = 0.0;
            (*n2)++;
          }
          ne += 2;
          found = true;
          break;
        }
        double maxp_t = fmax(maxp, fabs(sym(p, t)));
        if (fabs(a(p, p)) >= u * maxp_t) {
          if (p != ne) {
            swap(p, ne);
            if (lane == 0) { int32_t q = perm[p]; perm[p] = perm[ne]; perm[ne] = q; }
          }
          apply_1x1(ne, n);
          if (lane == 0) { d.type[ne] = PT_1X1; d.diag[ne] = a(ne, ne); d.off[ne] = 0.0; (*n1)++; }
          ne += 1;
          found = true;
          break;
        }
      }
      if (!found) {
        double maxp = rc_abs_max_excl(ne, ne, INT64_MAX);
        if (fabs(a(ne, ne)) >= u * maxp) {
          apply_1x1(ne, n);
          if (lane == 0) { d.type[ne] = PT_1X1; d.diag[ne] = a(ne, ne); d.off[ne] = 0.0; (*n1)++; }
          ne += 1;
        } else {
          break;
        }
      }
      __syncwarp();
    }
    __syncwarp();
    return ne - start;
  }
};

}  // namespace rvg
