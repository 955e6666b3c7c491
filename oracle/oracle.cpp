// ORACLE — test infrastructure only, never the product path.
//
// A single-threaded (optionally OpenMP level-parallel) C++ restatement of the
// rivrs-sparse numeric phase: multifrontal assembly, the dense APTP kernel
// (complete-pivoting 32x32 blocks, TRSM + a-posteriori threshold check,
// two-level 256-column outer loop, TPP fallback), the deferred contribution
// GEMM, and the supernodal forward/diagonal/backward solve.
//
// Every routine cites the reference function (file:line within the
// rivrs-linalg project) whose control flow and comparisons it follows.  The
// dense BLAS calls of the reference (faer 0.24, a semver range with no lock
// file, source absent) are replaced by loops with a fixed arithmetic
// contract:
//   * where the reference calls faer (TRSM, GEMM, triangular GEMM), each
//     output entry is an fma chain over the reduction index in ascending
//     order: c = fma(-a_k, b_k, c);
//   * where the reference has its own scalar Rust loops, the arithmetic is
//     unfused, expression for expression (build with -ffp-contract=off).
// The GPU kernels follow the same contract, which makes the two bit-identical
// on the same inputs; results agree with the reference to rounding, while
// every pivot decision follows the same comparisons in the same order.
//
// Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load
// this library, and only as the checker / the timed CPU baseline.
//
// Parity pinning: checked by tests/test_oracle.py against the reference's own
// hand-constructed fixtures (exact inertia, sparse/test-data/hand-constructed),
// its dense-kernel known-answer tests (sparse/src/symmetric/factor.rs tests)
// and the backward-error gates of sparse/tests/solve.rs.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <numeric>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif
#if defined(__x86_64__) && defined(__GNUC__)
#include <immintrin.h>
#endif
#include <stdlib.h>
#include <sys/mman.h>

#include <condition_variable>
#include <map>
#include <mutex>
#include <thread>

namespace {

typedef int64_t i64;

// ---------------------------------------------------------------------------
// Options (sparse/src/symmetric/factor.rs:86-130 AptpOptions, solver.rs:72-116)
// ---------------------------------------------------------------------------
struct Opts {
  double threshold = 0.01;
  double small = 1e-20;
  int fallback_bk = 1;        // AptpFallback::BunchKaufman (unused by the blocked path)
  int failed_pivot_tpp = 1;   // FailedPivotMethod::Tpp
  i64 nb = 256;               // outer_block_size
  i64 ib = 32;                // inner_block_size
  i64 nemin = 32;
  i64 small_leaf_threshold = 256;
};

const double BUNCH_KAUFMAN_ALPHA = 0.5;  // factor.rs:50

// near-tie reporting: a comparison a >= b (or a > b) is a near tie when
// |a - b| <= TIE_REL * max(|a|, |b|).
const double TIE_REL = 1e-12;
thread_local i64 g_ties = 0;
inline void note_tie(double a, double b) {
  double s = std::max(std::fabs(a), std::fabs(b));
  if (std::fabs(a - b) <= TIE_REL * s && s > 0) g_ties++;
}

// ---------------------------------------------------------------------------
// MixedDiagonal (sparse/src/symmetric/diagonal.rs:49-465)
// ---------------------------------------------------------------------------
enum : int8_t { PT_DELAYED = 0, PT_1X1 = 1, PT_2X2 = 2 };

struct MixedD {
  std::vector<int8_t> type;
  std::vector<i64> partner;
  std::vector<double> diag, off;
  i64 n = 0;
  void init(i64 n_) {
    n = n_;
    type.assign(n, PT_DELAYED);
    partner.assign(n, -1);
    diag.assign(n, 0.0);
    off.assign(n, 0.0);
  }
  void set1(i64 c, double v) { type[c] = PT_1X1; diag[c] = v; }
  void set2(i64 c, double a, double b, double cc) {
    type[c] = PT_2X2; partner[c] = c + 1;
    type[c + 1] = PT_2X2; partner[c + 1] = c;
    diag[c] = a; diag[c + 1] = cc; off[c] = b;
  }
  bool is2first(i64 c) const { return type[c] == PT_2X2 && partner[c] > c; }
  // diagonal.rs:185-198
  void grow(i64 nn) {
    if (nn > n) {
      type.resize(nn, PT_DELAYED); partner.resize(nn, -1);
      diag.resize(nn, 0.0); off.resize(nn, 0.0); n = nn;
    }
  }
  void truncate(i64 nn) {
    type.resize(nn); partner.resize(nn); diag.resize(nn); off.resize(nn); n = nn;
  }
  // diagonal.rs:216-259 copy_from_offset
  void copy_from_offset(const MixedD& s, i64 off0, i64 count) {
    i64 c = 0;
    while (c < count) {
      if (s.type[c] == PT_1X1) {
        type[off0 + c] = PT_1X1; partner[off0 + c] = -1; diag[off0 + c] = s.diag[c]; c += 1;
      } else if (s.type[c] == PT_2X2 && c + 1 < count) {
        i64 d = off0 + c;
        type[d] = PT_2X2; partner[d] = d + 1; type[d + 1] = PT_2X2; partner[d + 1] = d;
        diag[d] = s.diag[c]; diag[d + 1] = s.diag[c + 1]; off[d] = s.off[c];
        c += 2;
      } else {
        c += 1;
      }
    }
  }
  // diagonal.rs:312-365 solve_in_place (zero pivot -> 0)
  void solve(double* x) const {
    i64 c = 0;
    while (c < n) {
      if (type[c] == PT_1X1) {
        double d = diag[c];
        if (d == 0.0) x[c] = 0.0; else x[c] /= d;
        c += 1;
      } else {
        i64 p = partner[c];
        if (p > c) {
          double a = diag[c], b = off[c], cc = diag[p];
          double det = a * cc - b * b;
          if (det == 0.0) { x[c] = 0.0; x[p] = 0.0; }
          else { double r1 = x[c], r2 = x[p]; x[c] = (cc * r1 - b * r2) / det; x[p] = (a * r2 - b * r1) / det; }
        }
        c += 1;
      }
    }
  }
  // diagonal.rs:391-461 compute_inertia
  void inertia(i64* pos, i64* neg, i64* zer) const {
    i64 c = 0;
    while (c < n) {
      if (type[c] == PT_1X1) {
        double d = diag[c];
        if (d > 0) (*pos)++; else if (d < 0) (*neg)++; else (*zer)++;
        c += 1;
      } else {
        i64 p = partner[c];
        if (p > c) {
          double a = diag[c], b = off[c], cc = diag[p];
          double det = a * cc - b * b, tr = a + cc;
          if (det > 0) { if (tr > 0) *pos += 2; else *neg += 2; }
          else if (det < 0) { (*pos)++; (*neg)++; }
          else { if (tr > 0) { (*pos)++; (*zer)++; } else if (tr < 0) { (*neg)++; (*zer)++; } else *zer += 2; }
        }
        c += 1;
      }
    }
  }
};

struct Stats { i64 n1 = 0, n2 = 0, ndel = 0; double maxl = 0; };

struct FactorResult {
  MixedD d;
  std::vector<i64> perm;
  i64 ne = 0;
  Stats st;
};

// A vector whose elements are not value-initialised on growth: large
// front and factor buffers are filled in parallel instead (first touch by
// the threads that use them).
// Buffers of 32 MB and more (fronts, contribution blocks, factors) come
// from a cache of released buffers when one of at most twice the size is
// free (best fit), so the front-by-front allocation pattern of the
// multifrontal method reuses memory that is already mapped instead of
// faulting in fresh pages; new ones are 2 MB aligned and marked for
// transparent huge pages.  The cache holds at most 48 GB and is emptied by
// orc_release_cache().
const size_t BIG = (size_t)32 << 20;
struct BigCache {
  std::mutex mu;
  std::multimap<size_t, void*> free_;  // capacity -> block
  std::map<void*, size_t> cap_;        // every live or cached block -> capacity
  size_t cached = 0;
  void* get(size_t bytes) {
    const size_t HP = (size_t)2 << 20;
    const size_t want = (bytes + HP - 1) / HP * HP;
    {
      std::lock_guard<std::mutex> lk(mu);
      auto it = free_.lower_bound(want);
      if (it != free_.end() && it->first <= 2 * want) {
        void* p = it->second;
        cached -= it->first;
        free_.erase(it);
        return p;
      }
    }
    void* p = nullptr;
    if (posix_memalign(&p, HP, want) != 0) throw std::bad_alloc();
#ifdef MADV_HUGEPAGE
    madvise(p, want, MADV_HUGEPAGE);
#endif
    std::lock_guard<std::mutex> lk(mu);
    cap_[p] = want;
    return p;
  }
  void put(void* p) {
    std::lock_guard<std::mutex> lk(mu);
    const size_t c = cap_.at(p);
    const size_t LIMIT = (size_t)48 << 30;
    while (cached + c > LIMIT && !free_.empty()) {  // drop the largest cached blocks first
      auto it = std::prev(free_.end());
      cached -= it->first;
      cap_.erase(it->second);
      free(it->second);
      free_.erase(it);
    }
    if (cached + c > LIMIT) { cap_.erase(p); free(p); return; }
    free_.emplace(c, p);
    cached += c;
  }
  void release() {
    std::lock_guard<std::mutex> lk(mu);
    for (auto& kv : free_) { cap_.erase(kv.second); free(kv.second); }
    free_.clear();
    cached = 0;
  }
};
BigCache& big_cache() {
  static BigCache* c = new BigCache();  // never destroyed: buffers may be released at exit
  return *c;
}

template <class T>
struct NoInitAlloc : std::allocator<T> {
  template <class U> struct rebind { using other = NoInitAlloc<U>; };
  NoInitAlloc() = default;
  template <class U> NoInitAlloc(const NoInitAlloc<U>&) {}
  T* allocate(size_t n) {
    if (n * sizeof(T) < BIG) return std::allocator<T>::allocate(n);
    return static_cast<T*>(big_cache().get(n * sizeof(T)));
  }
  void deallocate(T* p, size_t n) {
    if (n * sizeof(T) < BIG) std::allocator<T>::deallocate(p, n);
    else big_cache().put(p);
  }
  template <class U> void construct(U* p) noexcept { ::new (static_cast<void*>(p)) U; }
  template <class U, class... A> void construct(U* p, A&&... a) { ::new (static_cast<void*>(p)) U(std::forward<A>(a)...); }
};
typedef std::vector<double, NoInitAlloc<double>> dvec;

void fill_zero(double* p, size_t n) {
  const size_t CH = (size_t)1 << 20;
  const i64 nch = (i64)((n + CH - 1) / CH);
  bool par = n > (size_t)4 << 20;
#ifdef _OPENMP
  par = par && !omp_in_parallel();
#pragma omp parallel for schedule(static) if (par)
#endif
  for (i64 c = 0; c < nch; ++c) {
    size_t b = (size_t)c * CH, e = std::min(n, b + CH);
    std::memset(p + b, 0, (e - b) * sizeof(double));
  }
  (void)par;
}

// column-major dense view
struct MV {
  double* a; i64 ld;
  double& operator()(i64 i, i64 j) const { return a[i + j * ld]; }
  MV sub(i64 r0, i64 c0) const { return MV{a + r0 + c0 * ld, ld}; }
};

// ---------------------------------------------------------------------------
// Symmetric swaps (factor.rs:466-517 swap_symmetric_block, 458-461 swap_symmetric)
// ---------------------------------------------------------------------------
void swap_sym_block(MV a, i64 i, i64 j, i64 col_start, i64 row_limit) {
  if (i == j) return;
  if (i > j) std::swap(i, j);
  std::swap(a(i, i), a(j, j));
  for (i64 k = col_start; k < i; ++k) std::swap(a(i, k), a(j, k));
  for (i64 k = i + 1; k < j; ++k) std::swap(a(k, i), a(j, k));
  for (i64 k = j + 1; k < row_limit; ++k) std::swap(a(k, i), a(k, j));
}
inline void swap_sym(MV a, i64 m, i64 i, i64 j) { swap_sym_block(a, i, j, 0, m); }

// ---------------------------------------------------------------------------
// factor_block_diagonal (factor.rs:891-1153): complete pivoting on an ib x ib block
// ---------------------------------------------------------------------------
void factor_block_diagonal(MV a, i64 col_start, i64 bs, double small, i64 row_limit,
                           MixedD& d, std::vector<i64>& lperm, i64& nelim_out, Stats& st) {
  i64 block_end = col_start + bs;
  lperm.resize(bs);
  for (i64 i = 0; i < bs; ++i) lperm[i] = i;
  d.init(bs);
  i64 k = 0;
  while (k < bs) {
    i64 cur = col_start + k;
    i64 remaining = bs - k;
    double maxv = 0.0; i64 mr = cur, mc = cur;
    for (i64 j = cur; j < block_end; ++j)
      for (i64 i = j; i < block_end; ++i) {
        double v = std::fabs(a(i, j));
        note_tie(v, maxv);
        if (v > maxv) { maxv = v; mr = i; mc = j; }
      }
    if (maxv < small) { st.ndel += remaining; break; }
    if (mr == mc) {
      if (mr != cur) { swap_sym_block(a, cur, mr, col_start, row_limit); std::swap(lperm[k], lperm[mr - col_start]); }
      double dkk = a(cur, cur), inv = 1.0 / dkk, maxl = 0.0;
      for (i64 i = cur + 1; i < block_end; ++i) { double l = a(i, cur) * inv; a(i, cur) = l; maxl = std::max(maxl, std::fabs(l)); }
      for (i64 j = cur + 1; j < block_end; ++j) {
        double ldl = a(j, cur) * dkk;
        for (i64 i = j; i < block_end; ++i) a(i, j) -= a(i, cur) * ldl;
      }
      d.set1(k, dkk); st.n1++; st.maxl = std::max(st.maxl, maxl);
      k += 1;
    } else {
      i64 t = mr, mi = mc;
      double amm = a(mi, mi), att = a(t, t), atm = a(t, mi);
      double delta = amm * att - atm * atm;
      if (remaining < 2) {
        i64 pp = std::fabs(amm) >= std::fabs(att) ? mi : t;
        if (pp != cur) { swap_sym_block(a, cur, pp, col_start, row_limit); std::swap(lperm[k], lperm[pp - col_start]); }
        double dkk = a(cur, cur);
        if (std::fabs(dkk) < small) { st.ndel += 1; break; }
        double inv = 1.0 / dkk;
        for (i64 i = cur + 1; i < block_end; ++i) a(i, cur) *= inv;
        d.set1(k, dkk); st.n1++;
        k += 1;
        continue;
      }
      note_tie(std::fabs(delta), BUNCH_KAUFMAN_ALPHA * atm * atm);
      if (std::fabs(delta) >= BUNCH_KAUFMAN_ALPHA * atm * atm) {
        if (mi != cur) { swap_sym_block(a, cur, mi, col_start, row_limit); std::swap(lperm[k], lperm[mi - col_start]); }
        i64 nt = (t == cur) ? mi : t;
        if (nt != cur + 1) { swap_sym_block(a, cur + 1, nt, col_start, row_limit); std::swap(lperm[k + 1], lperm[nt - col_start]); }
        double a11 = a(cur, cur), a22 = a(cur + 1, cur + 1), a21 = a(cur + 1, cur);
        double det = a11 * a22 - a21 * a21, inv_det = 1.0 / det, maxl = 0.0;
        for (i64 i = cur + 2; i < block_end; ++i) {
          double ai1 = a(i, cur), ai2 = a(i, cur + 1);
          double l1 = (ai1 * a22 - ai2 * a21) * inv_det, l2 = (ai2 * a11 - ai1 * a21) * inv_det;
          a(i, cur) = l1; a(i, cur + 1) = l2;
          maxl = std::max(maxl, std::max(std::fabs(l1), std::fabs(l2)));
        }
        for (i64 j = cur + 2; j < block_end; ++j) {
          double l1j = a(j, cur), l2j = a(j, cur + 1);
          double w1 = l1j * a11 + l2j * a21, w2 = l1j * a21 + l2j * a22;
          for (i64 i = j; i < block_end; ++i) a(i, j) -= a(i, cur) * w1 + a(i, cur + 1) * w2;
        }
        d.set2(k, a11, a21, a22); st.n2++; st.maxl = std::max(st.maxl, maxl);
        k += 2;
      } else {
        note_tie(std::fabs(amm), std::fabs(att));
        i64 pp = std::fabs(amm) >= std::fabs(att) ? mi : t;
        if (pp != cur) { swap_sym_block(a, cur, pp, col_start, row_limit); std::swap(lperm[k], lperm[pp - col_start]); }
        double dkk = a(cur, cur), inv = 1.0 / dkk, maxl = 0.0;
        for (i64 i = cur + 1; i < block_end; ++i) { double l = a(i, cur) * inv; a(i, cur) = l; maxl = std::max(maxl, std::fabs(l)); }
        for (i64 j = cur + 1; j < block_end; ++j) {
          double ldl = a(j, cur) * dkk;
          for (i64 i = j; i < block_end; ++i) a(i, j) -= a(i, cur) * ldl;
        }
        d.set1(k, dkk); st.n1++; st.maxl = std::max(st.maxl, maxl);
        k += 1;
      }
    }
  }
  nelim_out = k;
}

// adjust_for_2x2_boundary (factor.rs:1161-1174)
i64 adjust_2x2(i64 e, const MixedD& d) {
  if (e == 0) return 0;
  i64 last = e - 1;
  if (d.type[last] == PT_2X2 && d.partner[last] > last) return e - 1;
  return e;
}

// apply_and_check (factor.rs:1295-1408): TRSM, D^-1 scaling, first failing column.
// Rows are independent in all three steps, so blocks of rows go to threads;
// each block records, per column, its first row at or over the bound and the
// near ties up to it, and the blocks are then read in row order, which gives
// the serial scan's result and tie count exactly.
i64 apply_and_check(MV a, i64 col_start, i64 nelim, i64 bcols, i64 m, const MixedD& d, double thr) {
  if (nelim == 0) return 0;
  i64 prows = m - col_start - bcols;
  if (prows == 0) return nelim;
  i64 ps = col_start + bcols;
  const double bound = 1.0 / thr;
  const i64 RB = 256;
  const i64 nrb = (prows + RB - 1) / RB;
  std::vector<i64> first_fail((size_t)nrb * nelim), ties((size_t)nrb * nelim);
  bool par = prows * nelim > 200000;
#ifdef _OPENMP
  par = par && !omp_in_parallel();
#pragma omp parallel for schedule(static) if (par)
#endif
  for (i64 rb = 0; rb < nrb; ++rb) {
    i64 r0 = rb * RB, r1 = std::min(prows, r0 + RB);
    // panel * L11^T = A21  (L11 unit lower, from a[col_start.., col_start..])
    // faer TRSM (factor.rs:1338); per entry an fma chain over l ascending
    for (i64 j = 0; j < nelim; ++j)
      for (i64 l = 0; l < j; ++l) {
        double lij = a(col_start + j, col_start + l);
        for (i64 r = r0; r < r1; ++r)
          a(ps + r, col_start + j) = std::fma(-a(ps + r, col_start + l), lij, a(ps + r, col_start + j));
      }
    i64 c = 0;
    while (c < nelim) {
      if (d.type[c] == PT_1X1) {
        double inv = 1.0 / d.diag[c];
        for (i64 r = r0; r < r1; ++r) a(ps + r, col_start + c) *= inv;
        c += 1;
      } else if (d.is2first(c)) {
        double A = d.diag[c], B = d.off[c], C = d.diag[c + 1];
        double inv_det = 1.0 / (A * C - B * B);
        for (i64 r = r0; r < r1; ++r) {
          double x1 = a(ps + r, col_start + c), x2 = a(ps + r, col_start + c + 1);
          a(ps + r, col_start + c) = (x1 * C - x2 * B) * inv_det;
          a(ps + r, col_start + c + 1) = (x2 * A - x1 * B) * inv_det;
        }
        c += 2;
      } else c += 1;
    }
    for (i64 cc = 0; cc < nelim; ++cc) {
      i64 ff = -1, t = 0;
      for (i64 r = r0; r < r1; ++r) {
        double v = std::fabs(a(ps + r, col_start + cc));
        double sc = std::max(v, bound);
        if (std::fabs(v - bound) <= TIE_REL * sc && sc > 0) t++;
        if (v >= bound) { ff = r; break; }
      }
      first_fail[rb * nelim + cc] = ff;
      ties[rb * nelim + cc] = t;
    }
  }
  (void)par;
  i64 eff = nelim, sc = 0;
  while (sc < nelim) {
    i64 w = d.is2first(sc) ? 2 : 1;
    bool ok = true;
    for (i64 cc = sc; cc < sc + w && ok; ++cc) {
      if (cc >= nelim) break;
      for (i64 rb = 0; rb < nrb; ++rb) {
        g_ties += ties[rb * nelim + cc];
        if (first_fail[rb * nelim + cc] >= 0) { ok = false; break; }
      }
    }
    if (!ok) { eff = sc; break; }
    sc += w;
  }
  return eff;
}

// compute_ld_into (factor.rs:1536-1563): W = L * D.  Rows are independent;
// large blocks are split over threads by rows (the arithmetic per entry is
// unchanged).
void compute_ld(const double* l, i64 ldl, i64 nrows, const MixedD& d, i64 nelim, double* w, i64 ldw) {
  const i64 RB = 2048;
  const i64 nrb = (nrows + RB - 1) / RB;
  bool par = nrows * nelim > 100000;
#ifdef _OPENMP
  par = par && !omp_in_parallel();
#pragma omp parallel for schedule(static) if (par)
#endif
  for (i64 rb = 0; rb < nrb; ++rb) {
    const i64 r0 = rb * RB, r1 = std::min(nrows, r0 + RB);
    i64 c = 0;
    while (c < nelim) {
      if (d.type[c] == PT_1X1) {
        double dv = d.diag[c];
        for (i64 i = r0; i < r1; ++i) w[i + c * ldw] = l[i + c * ldl] * dv;
        c += 1;
      } else if (d.is2first(c)) {
        double A = d.diag[c], B = d.off[c], C = d.diag[c + 1];
        for (i64 i = r0; i < r1; ++i) {
          double l1 = l[i + c * ldl], l2 = l[i + (c + 1) * ldl];
          w[i + c * ldw] = l1 * A + l2 * B;
          w[i + (c + 1) * ldw] = l1 * B + l2 * C;
        }
        c += 2;
      } else c += 1;
    }
  }
  (void)par;
}

// Copy of the column block src[0..nrows, 0..ncols] (leading dimension lds)
// into dst (leading dimension ldd), split over threads by rows when large.
void copy_block(double* dst, i64 ldd, const double* src, i64 lds, i64 nrows, i64 ncols) {
  const i64 RB = 4096;
  const i64 nrb = (nrows + RB - 1) / RB;
  bool par = nrows * ncols > 200000;
#ifdef _OPENMP
  par = par && !omp_in_parallel();
#pragma omp parallel for schedule(static) if (par)
#endif
  for (i64 rb = 0; rb < nrb; ++rb) {
    const i64 r0 = rb * RB, r1 = std::min(nrows, r0 + RB);
    for (i64 j = 0; j < ncols; ++j) std::memcpy(dst + r0 + j * ldd, src + r0 + j * lds, (size_t)(r1 - r0) * 8);
  }
  (void)par;
}

// Per-thread scratch that grows and is never zeroed (every entry used is written first).
double* scratch(int slot, size_t n) {
  static thread_local std::vector<double, NoInitAlloc<double>> buf[8];
  if (buf[slot].size() < n) buf[slot].resize(n);
  return buf[slot].data();
}

// ---------------------------------------------------------------------------
// Rank-K update used by every faer GEMM call site:
//   C[i, j] = fma(-W[i, c], L[j, c], C[i, j]) for c = 0..K-1 in order,
// over i in [0, nr), j in [0, nc), where i + row_shift >= j (lower part of
// the output relative to the diagonal).
//
// Each entry's fma chain keeps its order whatever the blocking: K is cut into
// chunks taken one after another (an entry's running value is stored as a
// double between chunks, exactly what the chain holds); per chunk W and L are
// packed into tile-contiguous panels (24 rows x chunk for W, 8 columns x chunk
// for L), and the output is cut into 64-column panels (OpenMP, dynamic),
// 384-row blocks and 24 x 8 register tiles: 24 accumulator vectors of 8
// doubles, each step c loading three vectors of W and broadcasting 8 entries
// of L.  The tile arithmetic is vfnmadd (-(w * l) + acc, one rounding), equal
// to fma(-w, l, acc).  Tiles that straddle the diagonal, columns past the last
// full 8-column group and builds without AVX-512 take the scalar path, which
// runs the same chain entry by entry on the unpacked operands.
// ---------------------------------------------------------------------------
void syrk_scalar(double* C, i64 ldc, const double* W, i64 ldw, const double* L, i64 ldl, i64 r0, i64 r1, i64 j0,
                 i64 j1, i64 K, i64 row_shift) {
  for (i64 j = j0; j < j1; ++j) {
    double* col = C + j * ldc;
    const i64 is = std::max(r0, j - row_shift);
    for (i64 i = is; i < r1; ++i) {
      double acc = col[i];
      for (i64 c = 0; c < K; ++c) acc = std::fma(-W[i + c * ldw], L[j + c * ldl], acc);
      col[i] = acc;
    }
  }
}

#if defined(__x86_64__) && defined(__GNUC__)
#define ORC_HAVE_TILE 1
// One tile: rows [0, mr) (mr <= 24) of C, columns [0, 8); Wp holds 24
// doubles per step c, Lp 8.
__attribute__((target("avx512f,fma"))) void syrk_tile24x8(double* C, i64 ldc, const double* Wp, const double* Lp,
                                                           i64 K, int mr) {
  const __mmask8 m0 = (__mmask8)(mr >= 8 ? 0xFF : ((1u << mr) - 1));
  const __mmask8 m1 = (__mmask8)(mr >= 16 ? 0xFF : (mr <= 8 ? 0 : ((1u << (mr - 8)) - 1)));
  const __mmask8 m2 = (__mmask8)(mr >= 24 ? 0xFF : (mr <= 16 ? 0 : ((1u << (mr - 16)) - 1)));
  __m512d a0[8], a1[8], a2[8];
  for (int j = 0; j < 8; ++j) {
    a0[j] = _mm512_maskz_loadu_pd(m0, C + j * ldc);
    a1[j] = _mm512_maskz_loadu_pd(m1, C + j * ldc + 8);
    a2[j] = _mm512_maskz_loadu_pd(m2, C + j * ldc + 16);
  }
  for (i64 c = 0; c < K; ++c) {
    const double* w = Wp + c * 24;
    const __m512d w0 = _mm512_loadu_pd(w);
    const __m512d w1 = _mm512_loadu_pd(w + 8);
    const __m512d w2 = _mm512_loadu_pd(w + 16);
    const double* l = Lp + c * 8;
#pragma GCC unroll 8
    for (int j = 0; j < 8; ++j) {
      const __m512d lj = _mm512_set1_pd(l[j]);
      a0[j] = _mm512_fnmadd_pd(w0, lj, a0[j]);
      a1[j] = _mm512_fnmadd_pd(w1, lj, a1[j]);
      a2[j] = _mm512_fnmadd_pd(w2, lj, a2[j]);
    }
  }
  for (int j = 0; j < 8; ++j) {
    _mm512_mask_storeu_pd(C + j * ldc, m0, a0[j]);
    _mm512_mask_storeu_pd(C + j * ldc + 8, m1, a1[j]);
    _mm512_mask_storeu_pd(C + j * ldc + 16, m2, a2[j]);
  }
}
bool tile_ok() {
  static const bool ok = __builtin_cpu_supports("avx512f") && __builtin_cpu_supports("fma");
  return ok;
}
#else
#define ORC_HAVE_TILE 0
#endif

void syrk_fma(double* C, i64 ldc, const double* W, i64 ldw, const double* L, i64 ldl, i64 nr, i64 nc, i64 K,
              i64 row_shift) {
  if (nr <= 0 || nc <= 0 || K <= 0) return;
  const i64 JB = 64, IB = 384, KB = 256;
#if ORC_HAVE_TILE
  const bool tiles = tile_ok() && nr >= 24 && nc >= 8;
#else
  const bool tiles = false;
#endif
  const i64 njb = (nc + JB - 1) / JB;
  bool par = (double)nr * (double)nc * (double)K > 4e6;
#ifdef _OPENMP
  par = par && !omp_in_parallel();
#endif
  if (!tiles) {
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 1) if (par)
#endif
    for (i64 jb = 0; jb < njb; ++jb)
      syrk_scalar(C, ldc, W, ldw, L, ldl, 0, nr, jb * JB, std::min(nc, jb * JB + JB), K, row_shift);
    return;
  }
  const i64 nt = (nr + 23) / 24, ng = nc / 8;  // 24-row tiles, full 8-column groups
  for (i64 k0 = 0; k0 < K; k0 += KB) {
    const i64 kn = std::min(KB, K - k0);
    double* Wp = scratch(4, (size_t)nt * 24 * kn);
    double* Lp = scratch(5, (size_t)std::max<i64>(ng, 1) * 8 * kn);
#ifdef _OPENMP
#pragma omp parallel if (par)
#endif
    {
#ifdef _OPENMP
#pragma omp for schedule(static)
#endif
      for (i64 t = 0; t < nt; ++t) {
        double* dst = Wp + t * 24 * kn;
        const i64 i0 = t * 24, mr = std::min<i64>(24, nr - i0);
        for (i64 c = 0; c < kn; ++c) {
          const double* src = W + i0 + (k0 + c) * ldw;
          for (i64 r = 0; r < mr; ++r) dst[c * 24 + r] = src[r];
          for (i64 r = mr; r < 24; ++r) dst[c * 24 + r] = 0.0;
        }
      }
#ifdef _OPENMP
#pragma omp for schedule(static)
#endif
      for (i64 g = 0; g < ng; ++g) {
        double* dst = Lp + g * 8 * kn;
        for (i64 c = 0; c < kn; ++c)
          for (i64 q = 0; q < 8; ++q) dst[c * 8 + q] = L[g * 8 + q + (k0 + c) * ldl];
      }
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 1)
#endif
      for (i64 jb = 0; jb < njb; ++jb) {
        const i64 j0 = jb * JB, j1 = std::min(nc, j0 + JB);
        const double* Wk = W + k0 * ldw;
        const double* Lk = L + k0 * ldl;
        i64 tstart[JB / 8];
        i64 t_all = nt;
        const i64 ngp = (j1 - j0 + 7) / 8;
        for (i64 q = 0; q < ngp; ++q) {
          const i64 jm = j0 + 8 * q, nj = std::min<i64>(8, j1 - jm);
          if (nj < 8) {  // the last, partial group: scalar
            syrk_scalar(C, ldc, Wk, ldw, Lk, ldl, 0, nr, jm, jm + nj, kn, row_shift);
            tstart[q] = nt;
            continue;
          }
          // first tile whose rows are all in the lower part for the group's 8 columns
          const i64 need = jm + 7 - row_shift;  // row index from which every column qualifies
          const i64 tf = need <= 0 ? 0 : std::min(nt, (need + 23) / 24);
          const i64 first = std::max<i64>(0, jm - row_shift);
          const i64 rfull = std::min(nr, tf * 24);
          if (rfull > first) syrk_scalar(C, ldc, Wk, ldw, Lk, ldl, first, rfull, jm, jm + 8, kn, row_shift);
          tstart[q] = tf;
          t_all = std::min(t_all, tf);
        }
#if ORC_HAVE_TILE
        const i64 TB = IB / 24;
        for (i64 tb0 = t_all; tb0 < nt; tb0 += TB) {
          const i64 tb1 = std::min(nt, tb0 + TB);
          for (i64 q = 0; q < ngp; ++q) {
            const i64 jm = j0 + 8 * q;
            if (j1 - jm < 8) continue;
            const double* lp = Lp + (jm / 8) * 8 * kn;
            for (i64 t = std::max(tb0, tstart[q]); t < tb1; ++t)
              syrk_tile24x8(C + t * 24 + jm * ldc, ldc, Wp + t * 24 * kn, lp, kn,
                            (int)std::min<i64>(24, nr - t * 24));
          }
        }
#endif
      }
    }
  }
  (void)par;
}

// update_trailing (factor.rs:1418-1526): FS x FS lower and NFS x FS rectangle
void update_trailing(MV a, i64 col_start, i64 nelim, i64 bcols, i64 m, i64 p, const MixedD& d) {
  if (nelim == 0) return;
  i64 ts = col_start + bcols, tsz = m - ts;
  if (tsz <= 0) return;
  i64 fs = std::max<i64>(p - ts, 0);
  if (fs <= 0) return;
  double* L = scratch(0, (size_t)tsz * nelim);
  double* W = scratch(1, (size_t)tsz * nelim);
  copy_block(L, tsz, &a(ts, col_start), a.ld, tsz, nelim);
  compute_ld(L, tsz, tsz, d, nelim, W, tsz);
  // faer triangular / rectangular GEMM (factor.rs:1491, 1513); per entry an
  // fma chain over c ascending.  Region 1 is the lower triangle of
  // A[ts..p, ts..p], region 2 the rectangle A[p..m, ts..p]: together the
  // rows i >= j of the trailing columns ts..p.
  syrk_fma(&a(ts, ts), a.ld, W, tsz, L, tsz, tsz, fs, nelim, 0);
}

// update_cross_terms (factor.rs:1669-1766)
void update_cross_terms(MV a, i64 col_start, i64 nelim, i64 bcols, i64 m, const MixedD& d) {
  if (nelim == 0 || nelim >= bcols) return;
  i64 nf = bcols - nelim, ts = col_start + bcols, tsz = m - ts;
  std::vector<double> Lb((size_t)nf * nelim), Wb((size_t)nf * nelim, 0.0);
  for (i64 c = 0; c < nelim; ++c)
    for (i64 i = 0; i < nf; ++i) Lb[i + c * nf] = a(col_start + nelim + i, col_start + c);
  compute_ld(Lb.data(), nf, nf, d, nelim, Wb.data(), nf);
  for (i64 j = 0; j < nf; ++j)
    for (i64 i = j; i < nf; ++i) {
      double s = 0.0;
      for (i64 c = 0; c < nelim; ++c) s += Wb[i + c * nf] * Lb[j + c * nf];
      a(col_start + nelim + i, col_start + nelim + j) -= s;
    }
  if (tsz > 0) {
    double* Lp = scratch(0, (size_t)tsz * nelim);
    double* Wp = scratch(1, (size_t)tsz * nelim);
    copy_block(Lp, tsz, &a(ts, col_start), a.ld, tsz, nelim);
    compute_ld(Lp, tsz, tsz, d, nelim, Wp, tsz);
    const i64 RB = 1024, nrb = (tsz + RB - 1) / RB;
    bool par = tsz * nf * nelim > 400000;
#ifdef _OPENMP
    par = par && !omp_in_parallel();
#pragma omp parallel for schedule(static) if (par)
#endif
    for (i64 rb = 0; rb < nrb; ++rb) {
      const i64 r0 = rb * RB, r1 = std::min(tsz, r0 + RB);
      for (i64 j = 0; j < nf; ++j)
        for (i64 i = r0; i < r1; ++i) {
          double s = 0.0;
          for (i64 c = 0; c < nelim; ++c) s += Wp[i + c * tsz] * Lb[j + c * nf];
          a(ts + i, col_start + nelim + j) -= s;
        }
    }
    (void)par;
  }
}

// factor_inner (factor.rs:1811-2095): 32-column Factor / Apply / Update loop
FactorResult factor_inner(MV a, i64 m, i64 p, i64 nfs_boundary, const Opts& o) {
  i64 ib = o.ib;
  FactorResult R;
  R.perm.resize(m);
  std::iota(R.perm.begin(), R.perm.end(), 0);
  R.d.init(p);
  i64 k = 0, end_pos = p;
  std::vector<double> buf(ib);
  std::vector<i64> obuf(ib);
  while (k < end_pos) {
    i64 bs = std::min(end_pos - k, ib), be = k + bs;
    // 1. backup a[k..m, k..k+bs]   (BlockBackup::create, factor.rs:1191-1206)
    i64 rows = m - k;
    double* backup = scratch(2, (size_t)rows * bs);
    copy_block(backup, rows, &a(k, k), a.ld, rows, bs);
    // 2. factor diagonal block
    MixedD bd; std::vector<i64> bperm; i64 bnelim; Stats bst;
    factor_block_diagonal(a, k, bs, o.small, be, bd, bperm, bnelim, bst);
    if (bnelim == 0) {
      copy_block(&a(k, k), a.ld, backup, rows, rows, bs);
      for (i64 off = 0; off < bs; ++off) {
        end_pos -= 1;
        if (k + off < end_pos) { swap_sym(a, m, k + off, end_pos); std::swap(R.perm[k + off], R.perm[end_pos]); }
        R.st.ndel += 1;
      }
      continue;
    }
    // 3. permute panel columns (rows are independent: blocks of rows to threads)
    {
      const i64 nrow = m - be, RB = 4096, nrb = (nrow + RB - 1) / RB;
      bool par = nrow * bs > 200000;
#ifdef _OPENMP
      par = par && !omp_in_parallel();
#pragma omp parallel for schedule(static) if (par)
#endif
      for (i64 rb = 0; rb < nrb; ++rb) {
        double tb[64];
        for (i64 r = be + rb * RB; r < std::min(m, be + (rb + 1) * RB); ++r) {
          for (i64 i = 0; i < bs; ++i) tb[i] = a(r, k + bperm[i]);
          for (i64 i = 0; i < bs; ++i) a(r, k + i) = tb[i];
        }
      }
      (void)par;
    }
    // 4. zero D off-diagonals of 2x2 pivots
    {
      i64 bc = 0;
      while (bc < bnelim) {
        if (bd.is2first(bc)) { a(k + bc + 1, k + bc) = 0.0; bc += 2; } else bc += 1;
      }
    }
    // 5. row permutation of columns 0..k
    for (i64 c = 0; c < k; ++c) {
      for (i64 i = 0; i < bs; ++i) buf[i] = a(k + bperm[i], c);
      for (i64 i = 0; i < bs; ++i) a(k + i, c) = buf[i];
    }
    // 6. col_order
    for (i64 i = 0; i < bs; ++i) obuf[i] = R.perm[k + i];
    for (i64 i = 0; i < bs; ++i) R.perm[k + i] = obuf[bperm[i]];
    // 7. apply + check
    i64 eff = apply_and_check(a, k, bnelim, bs, m, bd, o.threshold);
    // 8. adjust
    eff = adjust_2x2(eff, bd);
    // 9. partial restore with permutation (restore_diagonal_with_perm, factor.rs:1244-1275)
    if (eff < bnelim) {
      for (i64 j = eff; j < bs; ++j) {
        i64 c = bperm[j];
        for (i64 i = eff; i < bs; ++i) {
          i64 r = bperm[i];
          a(k + i, k + j) = (r >= c) ? backup[r + c * rows] : backup[c + r * rows];
        }
      }
      for (i64 j = eff; j < bs; ++j) {
        i64 c = bperm[j];
        std::memcpy(&a(k + bs, k + j), backup + bs + c * rows, (size_t)(rows - bs) * 8);
      }
    }
    i64 nelim = eff;
    // 10. Schur updates
    if (nelim > 0) {
      update_trailing(a, k, nelim, bs, m, nfs_boundary, bd);
      update_cross_terms(a, k, nelim, bs, m, bd);
    }
    // 11. accumulate D and stats
    R.d.copy_from_offset(bd, k, nelim);
    {
      i64 sc = 0;
      while (sc < nelim) {
        if (bd.type[sc] == PT_1X1) { R.st.n1++; sc += 1; }
        else if (bd.is2first(sc)) { R.st.n2++; sc += 2; }
        else sc += 1;
      }
    }
    R.st.maxl = std::max(R.st.maxl, bst.maxl);
    {
      double ml = R.st.maxl;
      const i64 nrow = m - be;
      bool par = nrow * nelim > 200000;
#ifdef _OPENMP
      par = par && !omp_in_parallel();
#pragma omp parallel for schedule(static) reduction(max : ml) if (par)
#endif
      for (i64 c = 0; c < nelim; ++c)
        for (i64 i = be; i < m; ++i) ml = std::max(ml, std::fabs(a(i, k + c)));
      R.st.maxl = ml;
      (void)par;
    }
    // 12. delay failed columns to end_pos
    if (nelim < bs) {
      i64 nd = bs - nelim;
      for (i64 i = nd - 1; i >= 0; --i) {
        i64 dp = k + nelim + i;
        end_pos -= 1;
        if (dp < end_pos) { swap_sym(a, m, dp, end_pos); std::swap(R.perm[dp], R.perm[end_pos]); }
        R.st.ndel += 1;
      }
    }
    k += nelim;
  }
  R.ne = k;
  R.d.truncate(k);
  return R;
}

// Progress hook of a factorization run in slices (orc_session_*): the thread
// that runs the factorization reports the delay-free flops done so far at
// safe points, and waits there while its slice is used up.  Not called from
// inside parallel regions.
struct Run;
thread_local Run* tl_run = nullptr;
thread_local double tl_front_base = 0.0;  // flops of the fronts finished before the one in progress
void checkpoint(double done_now);

// Delay-free flops of the first `cols` eliminated columns of an m-row front:
// sum_{j < cols} [(m - j - 1) + (m - j - 1)(m - j)].
double front_flops(double m, double cols) {
  double s = 0.0;
  for (double j = 0; j < cols; j += 1.0) s += (m - j - 1.0) * (m - j + 1.0);
  return s;
}

// two_level_factor (factor.rs:2108-2252)
FactorResult two_level_factor(MV a, i64 m, i64 p, const Opts& o) {
  FactorResult R;
  R.perm.resize(m);
  std::iota(R.perm.begin(), R.perm.end(), 0);
  R.d.init(p);
  i64 gne = 0, rem = p;
  while (rem > 0) {
    i64 cs = gne, bcols = std::min(rem, o.nb);
    i64 bm = m - cs;
    FactorResult B = factor_inner(a.sub(cs, cs), bm, bcols, p - cs, o);
    i64 bne = B.ne;
    if (cs > 0) {
      bool par = cs * bcols > 200000;
#ifdef _OPENMP
      par = par && !omp_in_parallel();
#pragma omp parallel if (par)
#endif
      {
        std::vector<double> tmp(bcols);
#ifdef _OPENMP
#pragma omp for schedule(static)
#endif
        for (i64 c = 0; c < cs; ++c) {
          for (i64 i = 0; i < bcols; ++i) tmp[i] = a(cs + B.perm[i], c);
          for (i64 i = 0; i < bcols; ++i) a(cs + i, c) = tmp[i];
        }
      }
      (void)par;
    }
    {
      std::vector<i64> orig(R.perm.begin() + cs, R.perm.begin() + cs + bcols);
      for (i64 i = 0; i < bcols; ++i)
        if (B.perm[i] < bcols) R.perm[cs + i] = orig[B.perm[i]];
    }
    if (bne < bcols) {
      i64 nf = bcols - bne;
      for (i64 i = 0; i < nf; ++i) {
        i64 fp = cs + bne + i, e = cs + rem - 1 - i;
        if (fp < e) { swap_sym(a, m, fp, e); std::swap(R.perm[fp], R.perm[e]); }
      }
      R.st.ndel += nf;
    }
    R.d.copy_from_offset(B.d, gne, bne);
    R.st.n1 += B.st.n1; R.st.n2 += B.st.n2; R.st.maxl = std::max(R.st.maxl, B.st.maxl);
    gne += bne;
    rem -= bcols;
    if (tl_run) checkpoint(tl_front_base + front_flops((double)m, (double)(p - rem)));
  }
  R.ne = gne;
  R.d.truncate(gne);
  return R;
}

// ---------------------------------------------------------------------------
// TPP (factor.rs:2268-2947)
// ---------------------------------------------------------------------------
// `nc` = number of stored columns (a.ncols()): m for square fronts, k for the
// rectangular small-leaf storage.
struct TppCtx { MV a; i64 m; i64 nc; };

inline double sym_entry(const TppCtx& t, i64 row, i64 col) {  // factor.rs:2597-2606
  if (col < t.nc && row >= col) return t.a(row, col);
  return t.a(col, row);
}
bool is_col_small(const TppCtx& t, i64 idx, i64 from, i64 to, double small) {  // factor.rs:2674-2690
  for (i64 c = from; c < std::min(idx, t.nc); ++c) if (std::fabs(t.a(idx, c)) >= small) return false;
  if (idx < t.nc) for (i64 r = idx; r < to; ++r) if (std::fabs(t.a(r, idx)) >= small) return false;
  return true;
}
i64 find_row_abs_max(const TppCtx& t, i64 p, i64 from, i64 to) {  // factor.rs:2695-2710
  if (from >= to) return from;
  i64 bi = from; double bv = std::fabs(sym_entry(t, p, from));
  for (i64 c = from + 1; c < to; ++c) {
    double v = std::fabs(sym_entry(t, p, c));
    note_tie(v, bv);
    if (v > bv) { bi = c; bv = v; }
  }
  return bi;
}
double find_rc_abs_max_exclude(const TppCtx& t, i64 col, i64 nelim, i64 m, i64 exclude) {  // 2715-2737
  double best = 0.0;
  for (i64 c = nelim; c < std::min(col, t.nc); ++c) { if (c == exclude) continue; best = std::max(best, std::fabs(t.a(col, c))); }
  if (col < t.nc) for (i64 r = col + 1; r < m; ++r) { if (r == exclude) continue; best = std::max(best, std::fabs(t.a(r, col))); }
  return best;
}
bool test_2x2(const TppCtx& t, i64 ti, i64 p, double maxt, double maxp, double u, double small) {  // 2268-2315
  double a11 = t.a(ti, ti), a21 = t.a(p, ti), a22 = t.a(p, p);
  double maxpiv = std::max(std::max(std::fabs(a11), std::fabs(a21)), std::fabs(a22));
  if (maxpiv < small) return false;
  double ds = 1.0 / maxpiv;
  double dp0 = (a11 * ds) * a22, dp1 = (a21 * ds) * a21, dp = dp0 - dp1;
  double lim = std::max(std::max(small, std::fabs(dp0 / 2.0)), std::fabs(dp1 / 2.0));
  note_tie(std::fabs(dp), lim);
  if (std::fabs(dp) < lim) return false;
  double di11 = (a22 * ds) / dp, di12 = (-a21 * ds) / dp, di22 = (a11 * ds) / dp;
  if (std::max(maxt, maxp) < small) return true;
  double x1 = std::fabs(di11) * maxt + std::fabs(di12) * maxp;
  double x2 = std::fabs(di12) * maxt + std::fabs(di22) * maxp;
  note_tie(u * std::max(x1, x2), 1.0);
  return u * std::max(x1, x2) < 1.0;
}
// swap_rect (factor.rs:2528-2580); with nc == m it equals swap_symmetric
void swap_rect(const TppCtx& t, i64 i, i64 j) {
  if (i == j) return;
  if (i > j) std::swap(i, j);
  MV a = t.a; i64 n = t.nc;
  if (i < n && j < n) std::swap(a(i, i), a(j, j));
  for (i64 k = 0; k < std::min(i, n); ++k) std::swap(a(i, k), a(j, k));
  for (i64 k = i + 1; k < j; ++k) {
    if (k < n) std::swap(a(k, i), a(j, k));
    else if (i < n) break;
  }
  if (i < n && j < n) for (i64 k = j + 1; k < t.m; ++k) std::swap(a(k, i), a(k, j));
}
double tpp_apply_1x1(const TppCtx& t, i64 ne, i64 p) {  // 2616-2641
  MV a = t.a; i64 m = t.m;
  double d = a(ne, ne), inv = 1.0 / d, maxl = 0.0;
  for (i64 i = ne + 1; i < m; ++i) { double l = a(i, ne) * inv; a(i, ne) = l; maxl = std::max(maxl, std::fabs(l)); }
  i64 ce = std::min(p, t.nc);
  for (i64 j = ne + 1; j < ce; ++j) {
    double ldlj = a(j, ne) * d;
    for (i64 i = j; i < m; ++i) a(i, j) -= a(i, ne) * ldlj;
  }
  return maxl;
}
double tpp_apply_2x2(const TppCtx& t, i64 ne, i64 p) {  // 2649-2683
  MV a = t.a; i64 m = t.m;
  double a11 = a(ne, ne), a21 = a(ne + 1, ne), a22 = a(ne + 1, ne + 1);
  double det = a11 * a22 - a21 * a21, inv_det = 1.0 / det, maxl = 0.0;
  for (i64 i = ne + 2; i < m; ++i) {
    double ai1 = a(i, ne), ai2 = a(i, ne + 1);
    double l1 = (ai1 * a22 - ai2 * a21) * inv_det, l2 = (ai2 * a11 - ai1 * a21) * inv_det;
    a(i, ne) = l1; a(i, ne + 1) = l2;
    maxl = std::max(maxl, std::max(std::fabs(l1), std::fabs(l2)));
  }
  i64 ce = std::min(p, t.nc);
  for (i64 j = ne + 2; j < ce; ++j) {
    double w1 = a(j, ne) * a11 + a(j, ne + 1) * a21, w2 = a(j, ne) * a21 + a(j, ne + 1) * a22;
    for (i64 i = j; i < m; ++i) a(i, j) -= a(i, ne) * w1 + a(i, ne + 1) * w2;
  }
  a(ne + 1, ne) = 0.0;
  return maxl;
}

// Shared body of tpp_factor (factor.rs:2335-2506) and tpp_factor_rect
// (factor.rs:2761-2947): the two loops are identical apart from the storage
// width, which TppCtx carries.
i64 tpp_loop(const TppCtx& t, i64 start, i64 n, std::vector<i64>& perm, MixedD& d, Stats& st, const Opts& o) {
  double u = o.threshold, small = o.small;
  MV a = t.a; i64 m = t.m;
  i64 ne = start;
  while (ne < n) {
    if (is_col_small(t, ne, ne, m, small)) {
      d.set1(ne, 0.0); st.n1++;
      if (ne < t.nc) for (i64 r = ne + 1; r < m; ++r) a(r, ne) = 0.0;
      ne += 1;
      continue;
    }
    bool found = false;
    for (i64 p = ne + 1; p < n; ++p) {
      if (is_col_small(t, p, ne, m, small)) {
        if (p != ne) { swap_rect(t, p, ne); std::swap(perm[p], perm[ne]); }
        d.set1(ne, 0.0); st.n1++;
        for (i64 r = ne + 1; r < m; ++r) a(r, ne) = 0.0;
        ne += 1; found = true; break;
      }
      i64 ti = find_row_abs_max(t, p, ne, p);
      double maxt = find_rc_abs_max_exclude(t, ti, ne, m, p);
      double maxp = find_rc_abs_max_exclude(t, p, ne, m, ti);
      if (test_2x2(t, ti, p, maxt, maxp, u, small)) {
        if (ti != ne) { swap_rect(t, ti, ne); std::swap(perm[ti], perm[ne]); }
        i64 np = (p == ne) ? ti : p;
        if (np != ne + 1) { swap_rect(t, np, ne + 1); std::swap(perm[np], perm[ne + 1]); }
        double d11 = a(ne, ne), d21 = a(ne + 1, ne), d22 = a(ne + 1, ne + 1);
        double ml = tpp_apply_2x2(t, ne, n);
        d.set2(ne, d11, d21, d22); st.n2++; st.maxl = std::max(st.maxl, ml);
        ne += 2; found = true; break;
      }
      double maxp_t = std::max(maxp, std::fabs(sym_entry(t, p, ti)));
      note_tie(std::fabs(a(p, p)), u * maxp_t);
      if (std::fabs(a(p, p)) >= u * maxp_t) {
        if (p != ne) { swap_rect(t, p, ne); std::swap(perm[p], perm[ne]); }
        double ml = tpp_apply_1x1(t, ne, n);
        d.set1(ne, a(ne, ne)); st.n1++; st.maxl = std::max(st.maxl, ml);
        ne += 1; found = true; break;
      }
    }
    if (!found) {
      double maxp = find_rc_abs_max_exclude(t, ne, ne, m, INT64_MAX);
      note_tie(std::fabs(a(ne, ne)), u * maxp);
      if (std::fabs(a(ne, ne)) >= u * maxp) {
        double ml = tpp_apply_1x1(t, ne, n);
        d.set1(ne, a(ne, ne)); st.n1++; st.maxl = std::max(st.maxl, ml);
        ne += 1;
      } else break;
    }
  }
  return ne - start;
}

FactorResult tpp_factor_rect(MV a, i64 m, i64 nc, i64 n, const Opts& o) {  // factor.rs:2761-2947
  FactorResult R;
  R.perm.resize(m);
  std::iota(R.perm.begin(), R.perm.end(), 0);
  R.d.init(n);
  TppCtx t{a, m, nc};
  i64 ne = tpp_loop(t, 0, n, R.perm, R.d, R.st, o);
  R.ne = ne;
  R.d.truncate(ne);
  R.st.ndel = n - ne;
  return R;
}

// aptp_factor_in_place (factor.rs:301-404)
FactorResult aptp_factor_in_place(MV a, i64 m, i64 p, const Opts& o) {
  FactorResult R;
  if (p < o.ib) R = tpp_factor_rect(a, m, m, p, o);
  else if (p > o.nb) R = two_level_factor(a, m, p, o);
  else R = factor_inner(a, m, p, p, o);
  if (R.ne < p && o.failed_pivot_tpp) {
    i64 q = R.ne;
    R.d.grow(p);
    TppCtx t{a, m, m};
    i64 add = tpp_loop(t, q, p, R.perm, R.d, R.st, o);
    R.ne = q + add;
    R.d.truncate(R.ne);
    R.st.ndel = p - R.ne;
  }
  return R;
}

// compute_contribution_gemm (factor.rs:1590-1652) with the NFS x NFS block
// already assembled in `cb` (nfs x nfs, lower); L21_NFS = l[p..m, 0..ne].
void contribution_gemm(const double* l, i64 ldl, i64 p, i64 ne, i64 m, const MixedD& d, double* cb, i64 ldc) {
  i64 nfs = m - p;
  if (nfs == 0 || ne == 0) return;
  double* W = scratch(3, (size_t)nfs * ne);
  compute_ld(l + p, ldl, nfs, d, ne, W, nfs);
  // faer triangular GEMM (factor.rs:1639); per entry an fma chain over c ascending
  syrk_fma(cb, ldc, W, nfs, l + p, ldl, nfs, nfs, ne, 0);
}

// ---------------------------------------------------------------------------
// Supernodes, amalgamation, small-leaf classification
// ---------------------------------------------------------------------------
struct SN {
  i64 col_begin, col_end;
  std::vector<i64> pattern;
  i64 parent;  // -1 = root
  std::vector<std::pair<i64, i64>> owned;  // [begin, end) ranges
  bool in_small_leaf = false;
  i64 n_owned() const { i64 s = 0; for (auto& r : owned) s += r.second - r.first; return s; }
};

// do_merge (amalgamation.rs:38-54)
bool do_merge(i64 pn, i64 pcc, i64 cn, i64 ccc, i64 nemin) {
  if (pn == 1 && pcc == std::max<i64>(ccc - 1, 0)) return true;
  if (pn < nemin && cn < nemin) return true;
  return false;
}
// sorted_union_excluding (amalgamation.rs:57-95)
std::vector<i64> union_excl(const std::vector<i64>& a, const std::vector<i64>& b, i64 eb, i64 ee) {
  std::vector<i64> r; r.reserve(a.size() + b.size());
  size_t ia = 0, ib = 0;
  auto push = [&](i64 v) { if (!(v >= eb && v < ee)) r.push_back(v); };
  while (ia < a.size() && ib < b.size()) {
    i64 va = a[ia], vb = b[ib], nx;
    if (va < vb) { ia++; nx = va; } else if (vb < va) { ib++; nx = vb; } else { ia++; ib++; nx = va; }
    push(nx);
  }
  for (; ia < a.size(); ++ia) push(a[ia]);
  for (; ib < b.size(); ++ib) push(b[ib]);
  return r;
}
// amalgamate (amalgamation.rs:115-231)
std::vector<SN> amalgamate(std::vector<SN> sn, i64 nemin, i64* merges) {
  i64 n = (i64)sn.size();
  *merges = 0;
  if (n <= 1) return sn;
  std::vector<bool> del(n, false);
  std::vector<i64> nel(n);
  for (i64 s = 0; s < n; ++s) nel[s] = sn[s].col_end - sn[s].col_begin;
  std::vector<std::vector<i64>> ch(n);
  for (i64 s = 0; s < n; ++s) if (sn[s].parent >= 0) ch[sn[s].parent].push_back(s);
  for (i64 p = 0; p < n; ++p) {
    if (del[p]) continue;
    std::vector<i64> pch; pch.swap(ch[p]);
    for (i64 c : pch) {
      if (del[c]) continue;
      i64 pn = nel[p], pcc = nel[p] + (i64)sn[p].pattern.size();
      i64 cn = nel[c], ccc = nel[c] + (i64)sn[c].pattern.size();
      if (do_merge(pn, pcc, cn, ccc, nemin)) {
        i64 nb = std::min(sn[p].col_begin, sn[c].col_begin), ne_ = std::max(sn[p].col_end, sn[c].col_end);
        std::vector<i64> cp; cp.swap(sn[c].pattern);
        std::vector<i64> pp; pp.swap(sn[p].pattern);
        sn[p].pattern = union_excl(pp, cp, nb, ne_);
        for (auto& r : sn[c].owned) sn[p].owned.push_back(r);
        sn[c].owned.clear();
        sn[p].col_begin = nb; sn[p].col_end = ne_;
        nel[p] += nel[c];
        std::vector<i64> cc; cc.swap(ch[c]);
        for (i64 g : cc) if (!del[g]) sn[g].parent = p;
        for (i64 g : cc) ch[p].push_back(g);
        del[c] = true;
      }
    }
    for (i64 c : pch) if (!del[c]) ch[p].push_back(c);
  }
  std::vector<i64> o2n(n, 0);
  i64 ni = 0;
  for (i64 s = 0; s < n; ++s) if (!del[s]) o2n[s] = ni++;
  std::vector<SN> out; out.reserve(ni);
  for (i64 s = 0; s < n; ++s)
    if (!del[s]) {
      SN x = std::move(sn[s]);
      if (x.parent >= 0) x.parent = o2n[x.parent];
      out.push_back(std::move(x));
    }
  *merges = n - ni;
  return out;
}

struct Subtree { i64 root; std::vector<i64> nodes; i64 max_front; i64 parent_of_root; };

// classify_small_leaf_subtrees (numeric.rs:2278-2369)
std::vector<Subtree> classify_small_leaf(std::vector<SN>& sn, const std::vector<std::vector<i64>>& ch, i64 thr) {
  std::vector<Subtree> out;
  if (thr == 0) return out;
  i64 n = (i64)sn.size();
  for (i64 s = 0; s < n; ++s) {
    i64 fs = sn[s].n_owned() + (i64)sn[s].pattern.size();
    if (fs >= thr) { sn[s].in_small_leaf = false; continue; }
    if (ch[s].empty()) sn[s].in_small_leaf = true;
    else {
      bool all = true;
      for (i64 c : ch[s]) if (!sn[c].in_small_leaf) { all = false; break; }
      sn[s].in_small_leaf = all;
    }
  }
  for (i64 s = 0; s < n; ++s) {
    if (!sn[s].in_small_leaf) continue;
    bool is_root = sn[s].parent < 0 || !sn[sn[s].parent].in_small_leaf;
    if (!is_root) continue;
    std::vector<i64> nodes, stack{s}, visit;
    while (!stack.empty()) {
      i64 x = stack.back(); stack.pop_back();
      visit.push_back(x);
      for (i64 c : ch[x]) if (sn[c].in_small_leaf) stack.push_back(c);
    }
    while (!visit.empty()) { nodes.push_back(visit.back()); visit.pop_back(); }
    if (nodes.size() < 2) { sn[s].in_small_leaf = false; continue; }
    i64 mf = 0;
    for (i64 x : nodes) mf = std::max(mf, sn[x].n_owned() + (i64)sn[x].pattern.size());
    out.push_back(Subtree{s, nodes, mf, sn[s].parent});
  }
  return out;
}

// ---------------------------------------------------------------------------
// Multifrontal driver (numeric.rs:844-1023, 1226-1533, 1562-1938, 1957-2163)
// ---------------------------------------------------------------------------
struct Front {      // FrontFactors (numeric.rs:543-596) plus per-supernode stats
  i64 m = 0, k = 0, ne = 0;
  dvec l11, l21;                  // ne x ne, r x ne (column-major)
  MixedD d11;
  std::vector<i64> col_idx, row_idx, local_perm;
  i64 n1 = 0, n2 = 0;
  double maxl = 0;
  i64 ties = 0;
};

struct CB { dvec data; i64 size = 0; std::vector<i64> rows; i64 ndel = 0; };

struct Problem {
  i64 n;
  const i64 *colptr, *rowidx;
  const double* val;
  const double* scaling;  // elimination order or null
  std::vector<i64> pfwd, pinv;
};

struct Oracle {
  i64 n = 0;
  Opts o;
  std::vector<SN> sn;
  std::vector<std::vector<i64>> ch;
  std::vector<Front> fr;
  std::vector<i64> pfwd;
  std::vector<double> scaling;
  bool has_scaling = false;
  i64 sn_before = 0, merges = 0, n_sl_sub = 0, n_sl_nodes = 0;
  i64 tot1 = 0, tot2 = 0, totdel = 0, zero_piv = 0, max_front = 0;
  i64 ties = 0;
  std::string err;
};

// extract_front_factors (numeric.rs:2579-2713) from a front stored as m x nc
void extract_factors(Front& F, const double* a, i64 lda, i64 m, i64 k, const std::vector<i64>& rows, const FactorResult& R) {
  i64 ne = R.ne;
  F.m = m; F.k = k; F.ne = ne;
  F.l11.resize((size_t)ne * ne);
  {
    // column by column: zeros above the diagonal, 1 on it, L below (the
    // second column of a 2x2 pivot keeps a zero at its first sub-diagonal)
    bool par = ne * ne > (1 << 20);
#ifdef _OPENMP
    par = par && !omp_in_parallel();
#pragma omp parallel for schedule(dynamic, 16) if (par)
#endif
    for (i64 c = 0; c < ne; ++c) {
      double* col = F.l11.data() + c * ne;
      std::memset(col, 0, (size_t)c * sizeof(double));
      col[c] = 1.0;
      const bool second = R.d.type[c] == PT_2X2 && R.d.partner[c] < c;
      const bool first = R.d.is2first(c);
      const bool known = R.d.type[c] == PT_1X1 || first || second;
      i64 i0 = c + 1;
      if (first && c + 1 < ne) { col[c + 1] = 0.0; i0 = c + 2; }
      if (known) std::memcpy(col + i0, a + i0 + c * lda, (size_t)std::max<i64>(0, ne - i0) * sizeof(double));
      else std::memset(col + i0, 0, (size_t)std::max<i64>(0, ne - i0) * sizeof(double));
    }
    (void)par;
  }
  F.d11.init(ne);
  i64 c = 0;
  while (c < ne) {
    if (R.d.type[c] == PT_1X1) { F.d11.set1(c, R.d.diag[c]); c += 1; }
    else { F.d11.set2(c, R.d.diag[c], R.d.off[c], R.d.diag[c + 1]); c += 2; }
  }
  i64 r = m - ne;
  F.l21.resize((size_t)r * ne);
  copy_block(F.l21.data(), r, a + ne, lda, r, ne);
  F.local_perm.assign(R.perm.begin(), R.perm.begin() + k);
  F.col_idx.resize(ne);
  for (i64 i = 0; i < ne; ++i) F.col_idx[i] = rows[R.perm[i]];
  F.row_idx.clear();
  for (i64 i = ne; i < k; ++i) F.row_idx.push_back(rows[R.perm[i]]);
  for (i64 i = k; i < m; ++i) F.row_idx.push_back(rows[i]);
  F.n1 = R.st.n1; F.n2 = R.st.n2; F.maxl = R.st.maxl;
}

// extract_contribution (numeric.rs:2739-2809): delayed block from the front,
// NFS x NFS from `nfsblk` (nfs x nfs).
CB extract_contrib(const double* a, i64 lda, i64 m, i64 k, const std::vector<i64>& rows, const FactorResult& R, dvec&& nfsblk) {
  CB cb;
  i64 ne = R.ne, size = m - ne, nd = k - ne, nfs = m - k;
  cb.size = size; cb.ndel = nd;
  if (nd > 0) {
    cb.data.resize((size_t)size * size);
    fill_zero(cb.data.data(), cb.data.size());
    for (i64 j = 0; j < nd; ++j)
      for (i64 i = j; i < nd; ++i) cb.data[i + j * size] = a[ne + i + (ne + j) * lda];
    for (i64 j = 0; j < nd; ++j)
      for (i64 i = 0; i < nfs; ++i) cb.data[nd + i + j * size] = a[k + i + (ne + j) * lda];
    for (i64 j = 0; j < nfs; ++j)
      for (i64 i = j; i < nfs; ++i) cb.data[nd + i + (nd + j) * size] = nfsblk[i + j * nfs];
  } else {
    cb.data = std::move(nfsblk);
  }
  for (i64 i = ne; i < k; ++i) cb.rows.push_back(rows[R.perm[i]]);
  for (i64 i = k; i < m; ++i) cb.rows.push_back(rows[i]);
  return cb;
}

// Assembly shared by both node kinds: scatter original entries of owned columns
// (scatter_original_entries_multi numeric.rs:2376-2435 and the amap fast path
// numeric.rs:1306-1332, which produce the same sums) and extend-add of children
// (extend_add numeric.rs:2445-2485). FS columns go to `fs` (m x k), NFS x NFS
// entries to `nfsb` (nfs x nfs).
void assemble(const Oracle& O, const Problem& P, const SN& s, i64 m, i64 k, std::vector<i64>& g2l,
              double* fs, double* nfsb, bool has_nfs, std::vector<CB*>& cbs) {
  i64 tot_owned = s.n_owned();
  i64 nfs = m - k;
  auto put = [&](i64 r, i64 c, double v) {
    if (c < k) fs[r + c * m] += v;
    else if (has_nfs && r >= k) nfsb[(r - k) + (c - k) * nfs] += v;
  };
  for (auto& rg : s.owned)
    for (i64 pj = rg.first; pj < rg.second; ++pj) {
      i64 oc = P.pfwd[pj];
      i64 lc = g2l[pj];
      for (i64 idx = P.colptr[oc]; idx < P.colptr[oc + 1]; ++idx) {
        i64 orow = P.rowidx[idx];
        if (orow < oc) {
          i64 lp = g2l[P.pinv[orow]];
          if (lp >= 0 && lp < tot_owned) continue;
        }
        i64 gr = P.pinv[orow];
        i64 lr = g2l[gr];
        if (lr < 0) continue;
        if (lr >= tot_owned && lr < k) continue;
        double v = P.val[idx];
        // amap fast path (no delays): val * s[row] * s[col] (numeric.rs:1317);
        // per-entry path: val *= s[row] * s[col] (numeric.rs:2421)
        if (P.scaling) {
          if (k == tot_owned) v = v * P.scaling[gr] * P.scaling[pj];
          else v *= P.scaling[gr] * P.scaling[pj];
        }
        if (lr >= lc) put(lr, lc, v); else put(lc, lr, v);
      }
    }
  std::vector<i64> loc;
  for (CB* cb : cbs) {
    // When the child's rows map to increasing front rows (no delayed rows
    // out of order), column j of the child's block lands in front column lj
    // only, so columns go to threads; each destination still receives its
    // terms in the same order (children in turn, one term per child).
    const i64 sz = cb->size;
    loc.resize(sz);
    bool mono = true;
    for (i64 i = 0; i < sz; ++i) {
      loc[i] = g2l[cb->rows[i]];
      if (i > 0 && loc[i] <= loc[i - 1]) mono = false;
    }
    bool par = mono && sz > 512;
#ifdef _OPENMP
    par = par && !omp_in_parallel();
#pragma omp parallel for schedule(dynamic, 8) if (par)
#endif
    for (i64 j = 0; j < sz; ++j) {
      i64 lj = loc[j];
      const double* col = cb->data.data() + j * sz;
      for (i64 i = j; i < sz; ++i) {
        double v = col[i];
        if (v != 0.0) {
          i64 li = loc[i];
          if (li >= lj) put(li, lj, v); else put(lj, li, v);
        }
      }
    }
    (void)par;
  }
  (void)O;
}

// One supernode: factor_single_supernode (numeric.rs:1226-1533) when
// small_leaf is false, the per-node body of factor_small_leaf_subtree
// (numeric.rs:1597-1935) when true.  Both keep the FS columns as m x k and the
// NFS x NFS block separately; the square path's NFS x NFS region is only ever
// copied into the contribution buffer (factor.rs:1615-1619) so the split is
// value-identical.
void factor_node(Oracle& O, const Problem& P, i64 s, std::vector<CB>& contrib, std::vector<i64>& g2l) {
  SN& S = O.sn[s];
  std::vector<i64> delayed;
  std::vector<CB*> cbs;
  for (i64 c : O.ch[s]) {
    CB& cb = contrib[c];
    if (cb.size > 0 || !cb.rows.empty()) {
      for (i64 i = 0; i < cb.ndel; ++i) delayed.push_back(cb.rows[i]);
      cbs.push_back(&cb);
    }
  }
  i64 nown = S.n_owned();
  i64 k = nown + (i64)delayed.size();
  std::vector<i64> rows;
  rows.reserve(k + S.pattern.size());
  for (auto& rg : S.owned) for (i64 c = rg.first; c < rg.second; ++c) rows.push_back(c);
  for (i64 c : delayed) rows.push_back(c);
  for (i64 c : S.pattern) rows.push_back(c);
  i64 m = (i64)rows.size();
  for (i64 i = 0; i < m; ++i) g2l[rows[i]] = i;
  i64 nfs = m - k;
  bool has_nfs = nfs > 0 && S.parent >= 0;
  dvec fs((size_t)m * k);
  fill_zero(fs.data(), fs.size());
  dvec nfsb(has_nfs ? (size_t)nfs * nfs : 0);
  fill_zero(nfsb.data(), nfsb.size());
  assemble(O, P, S, m, k, g2l, fs.data(), nfsb.data(), has_nfs, cbs);
  for (CB* cb : cbs) { cb->data.clear(); cb->data.shrink_to_fit(); cb->rows.clear(); cb->size = 0; }
  i64 t0 = g_ties;
  FactorResult R;
  MV a{fs.data(), m};
  if (S.in_small_leaf) {
    R = tpp_factor_rect(a, m, k, k, O.o);
  } else {
    // aptp_factor_in_place on the m x m front: it never reads or writes
    // columns >= k (swaps stay within FS, updates stop at the NFS boundary),
    // so the m x k storage is sufficient.
    FactorResult RR;
    if (k < O.o.ib) {
      RR = tpp_factor_rect(a, m, k, k, O.o);
    } else if (k > O.o.nb) RR = two_level_factor(a, m, k, O.o);
    else RR = factor_inner(a, m, k, k, O.o);
    if (RR.ne < k && O.o.failed_pivot_tpp) {
      i64 q = RR.ne;
      RR.d.grow(k);
      TppCtx t{a, m, k};
      i64 add = tpp_loop(t, q, k, RR.perm, RR.d, RR.st, O.o);
      RR.ne = q + add;
      RR.d.truncate(RR.ne);
      RR.st.ndel = k - RR.ne;
    }
    R = std::move(RR);
  }
  i64 ne = R.ne;
  Front& F = O.fr[s];
  F.ties = g_ties - t0;
  if (S.parent >= 0 && ne < m) {
    if (has_nfs && ne > 0) contribution_gemm(fs.data(), m, k, ne, m, R.d, nfsb.data(), nfs);
    contrib[s] = extract_contrib(fs.data(), m, m, k, rows, R, std::move(nfsb));
  }
  extract_factors(F, fs.data(), m, m, k, rows, R);
  for (i64 i = 0; i < m; ++i) g2l[rows[i]] = -1;
}

}  // namespace

// ---------------------------------------------------------------------------
// C API (test / baseline use only)
// ---------------------------------------------------------------------------
extern "C" {

struct orc_options {
  double threshold;
  double small;
  int64_t outer_block_size;
  int64_t inner_block_size;
  int64_t nemin;
  int64_t small_leaf_threshold;
  int32_t failed_pivot_tpp;
  int32_t fallback_bk;
};

}  // extern "C"

namespace {

// One factorization: the pattern-only set-up (amalgamation, children,
// small-leaf classification), then the numeric phase, which runs either in
// one go or in slices (a worker thread that stops at checkpoints).
struct Run {
  Oracle* O = nullptr;
  Problem P;
  std::vector<CB> contrib;
  std::vector<Subtree> subs;
  int nthreads = 0;
  std::vector<double> fflops;  // delay-free flops per (amalgamated) front
  double total = 0.0;
  std::mutex mu;
  std::condition_variable cv;
  double target = 0.0, done = 0.0;
  bool running = false, finished = false, abort = false;
  std::thread th;
};

struct Aborted {};

void checkpoint(double done_now) {
  Run* r = tl_run;
  if (!r || omp_in_parallel()) return;
  std::unique_lock<std::mutex> lk(r->mu);
  r->done = done_now;
  if (r->done >= r->target) {
    r->running = false;
    r->cv.notify_all();
    r->cv.wait(lk, [&] { return r->running; });
  }
  if (r->abort) throw Aborted();  // unwinds the worker's stack (never inside a parallel region)
}

Run* run_setup(int64_t n, int64_t nsup, const int64_t* sup_begin, const int64_t* sup_end, const int64_t* pat_ptr,
               const int64_t* pat_idx, const int64_t* sup_parent, const int64_t* perm_fwd, const int64_t* colptr,
               const int64_t* rowidx, const double* values, const double* scaling, const orc_options* opt,
               int32_t nthreads) {
  Run* r = new Run();
  Oracle* O = r->O = new Oracle();
  O->n = n;
  if (opt) {
    O->o.threshold = opt->threshold; O->o.small = opt->small; O->o.nb = opt->outer_block_size;
    O->o.ib = opt->inner_block_size; O->o.nemin = opt->nemin; O->o.small_leaf_threshold = opt->small_leaf_threshold;
    O->o.failed_pivot_tpp = opt->failed_pivot_tpp; O->o.fallback_bk = opt->fallback_bk;
  }
  std::vector<SN> sn(nsup);
  for (i64 s = 0; s < nsup; ++s) {
    sn[s].col_begin = sup_begin[s]; sn[s].col_end = sup_end[s];
    sn[s].pattern.assign(pat_idx + pat_ptr[s], pat_idx + pat_ptr[s + 1]);
    sn[s].parent = sup_parent[s];
    sn[s].owned = {{sup_begin[s], sup_end[s]}};
  }
  O->sn_before = nsup;
  O->sn = amalgamate(std::move(sn), O->o.nemin, &O->merges);
  i64 ns = (i64)O->sn.size();
  O->ch.assign(ns, {});
  for (i64 s = 0; s < ns; ++s) if (O->sn[s].parent >= 0) O->ch[O->sn[s].parent].push_back(s);
  r->subs = classify_small_leaf(O->sn, O->ch, O->o.small_leaf_threshold);
  O->n_sl_sub = (i64)r->subs.size();
  for (auto& st : r->subs) O->n_sl_nodes += (i64)st.nodes.size();
  Problem& P = r->P;
  P.n = n; P.colptr = colptr; P.rowidx = rowidx; P.val = values; P.scaling = scaling;
  P.pfwd.assign(perm_fwd, perm_fwd + n);
  P.pinv.assign(n, 0);
  for (i64 i = 0; i < n; ++i) P.pinv[P.pfwd[i]] = i;
  O->pfwd = P.pfwd;
  if (scaling) { O->has_scaling = true; O->scaling.assign(scaling, scaling + n); }
  O->fr.assign(ns, Front());
  r->contrib.resize(ns);
  r->nthreads = nthreads;
  r->fflops.resize(ns);
  for (i64 s = 0; s < ns; ++s) {
    const double k = (double)O->sn[s].n_owned();
    r->fflops[s] = front_flops(k + (double)O->sn[s].pattern.size(), k);
    r->total += r->fflops[s];
  }
  return r;
}

// The numeric phase: small-leaf pre-pass (numeric.rs:1984-2010), then
// level-set waves (2038-2160), then the aggregate statistics (929-1009).
void run_body(Run* r) {
  Oracle* O = r->O;
  Problem& P = r->P;
  std::vector<CB>& contrib = r->contrib;
  const i64 n = O->n, ns = (i64)O->sn.size();
#ifdef _OPENMP
  if (r->nthreads > 0) omp_set_num_threads(r->nthreads);
#endif
  g_ties = 0;
  double done = 0.0;
  std::vector<i64> remaining(ns);
  for (i64 s = 0; s < ns; ++s) remaining[s] = (i64)O->ch[s].size();
  {
    // the subtrees are independent (numeric.rs factors them in parallel);
    // each one's fronts in order on one thread
    const i64 nsub = (i64)r->subs.size();
#ifdef _OPENMP
#pragma omp parallel if (nsub > 1)
#endif
    {
      std::vector<i64> g2l(n, -1);
      i64 ties0 = g_ties; g_ties = 0;
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 1)
#endif
      for (i64 t = 0; t < nsub; ++t)
        for (i64 x : r->subs[t].nodes) factor_node(*O, P, x, contrib, g2l);
      g_ties = ties0;
    }
    for (auto& st : r->subs) {
      if (st.parent_of_root >= 0) remaining[st.parent_of_root] -= 1;
      for (i64 x : st.nodes) done += r->fflops[x];
    }
    checkpoint(done);
  }
  std::vector<i64> ready;
  for (i64 s = 0; s < ns; ++s) if (remaining[s] == 0 && !O->sn[s].in_small_leaf) ready.push_back(s);
  while (!ready.empty()) {
    i64 nr = (i64)ready.size();
#ifdef _OPENMP
    // The fronts of a wave are independent.  Fronts whose dense work would
    // hold up the wave if one thread took them (more than the wave's average
    // per thread, or large in absolute terms) run one at a time with the
    // dense loops inside in parallel; the rest one front per thread.  Which
    // thread takes a front changes nothing in its arithmetic.
    {
      const i64 nth = omp_get_max_threads();
      std::vector<double> work(nr);
      double tot = 0;
      for (i64 i = 0; i < nr; ++i) {
        const SN& S = O->sn[ready[i]];
        double k = (double)S.n_owned(), m = k + (double)S.pattern.size();
        work[i] = k * m * m;
        tot += work[i];
      }
      std::vector<i64> big, small;
      for (i64 i = 0; i < nr; ++i) {
        const bool b = nth > 1 && (work[i] > 2e9 || (nr > 1 && work[i] > tot / (double)nth) || nr == 1);
        (b ? big : small).push_back(ready[i]);
      }
      {
        std::vector<i64> g2l(n, -1);
        for (i64 s : big) {
          tl_front_base = done;
          factor_node(*O, P, s, contrib, g2l);
          done += r->fflops[s];
          checkpoint(done);
        }
      }
      const i64 ns_ = (i64)small.size();
#pragma omp parallel if (ns_ > 1)
      {
        std::vector<i64> g2l(n, -1);
        i64 ties0 = g_ties; g_ties = 0;
#pragma omp for schedule(dynamic, 1)
        for (i64 i = 0; i < ns_; ++i) factor_node(*O, P, small[i], contrib, g2l);
        g_ties = ties0;
      }
      for (i64 s : small) done += r->fflops[s];
      checkpoint(done);
    }
#else
    {
      std::vector<i64> g2l(n, -1);
      for (i64 i = 0; i < nr; ++i) factor_node(*O, P, ready[i], contrib, g2l);
    }
#endif
    std::vector<i64> next;
    for (i64 s : ready) {
      i64 p = O->sn[s].parent;
      if (p >= 0) { remaining[p] -= 1; if (remaining[p] == 0) next.push_back(p); }
    }
    ready.swap(next);
  }
  // aggregate stats (numeric.rs:929-1009)
  for (i64 s = 0; s < ns; ++s) {
    Front& F = O->fr[s];
    O->tot1 += F.n1; O->tot2 += F.n2; O->totdel += F.k - F.ne;
    O->max_front = std::max(O->max_front, F.m);
    O->ties += F.ties;
    for (i64 c = 0; c < F.ne; ++c) if (F.d11.type[c] == PT_1X1 && F.d11.diag[c] == 0.0) O->zero_piv++;
    if (O->sn[s].parent < 0 && F.ne < F.m) O->zero_piv += F.k - F.ne;
  }
  contrib.clear();
}

}  // namespace

extern "C" {

// Factor: the symbolic input is the pre-amalgamation supernode partition
// (what AptpSymbolic exposes), the permutation perm_fwd[new] = old, the full
// symmetric CSC and the MC64 scaling in elimination order (or NULL).
void* orc_factor(int64_t n, int64_t nsup, const int64_t* sup_begin, const int64_t* sup_end,
                 const int64_t* pat_ptr, const int64_t* pat_idx, const int64_t* sup_parent,
                 const int64_t* perm_fwd, const int64_t* colptr, const int64_t* rowidx,
                 const double* values, const double* scaling, const orc_options* opt, int32_t nthreads) {
  Run* r = run_setup(n, nsup, sup_begin, sup_end, pat_ptr, pat_idx, sup_parent, perm_fwd, colptr, rowidx, values,
                     scaling, opt, nthreads);
  run_body(r);
  Oracle* O = r->O;
  delete r;
  return O;
}

// The same factorization in slices, for timing a long run step by step: the
// set-up happens here; the numeric phase runs on a worker thread that stops
// at checkpoints (after every front of a wave that is taken alone, after
// every wave, after every 256-column outer block of such a front) once its
// delay-free flops reach the target of the last orc_session_advance.
// Every input array must stay alive until orc_session_finish.
void* orc_session_begin(int64_t n, int64_t nsup, const int64_t* sup_begin, const int64_t* sup_end,
                        const int64_t* pat_ptr, const int64_t* pat_idx, const int64_t* sup_parent,
                        const int64_t* perm_fwd, const int64_t* colptr, const int64_t* rowidx,
                        const double* values, const double* scaling, const orc_options* opt, int32_t nthreads) {
  Run* r = run_setup(n, nsup, sup_begin, sup_end, pat_ptr, pat_idx, sup_parent, perm_fwd, colptr, rowidx, values,
                     scaling, opt, nthreads);
  r->th = std::thread([r] {
    tl_run = r;
    {
      std::unique_lock<std::mutex> lk(r->mu);
      r->cv.wait(lk, [&] { return r->running; });
    }
    try {
      if (!r->abort) run_body(r);
    } catch (const Aborted&) {
    }
    std::lock_guard<std::mutex> lk(r->mu);
    r->finished = true;
    r->running = false;
    r->cv.notify_all();
  });
  return r;
}

// Delay-free flops of the whole factorization (the unit of the targets).
double orc_session_total(void* h) { return ((Run*)h)->total; }

// Flops done at the last checkpoint.
double orc_session_done(void* h) { return ((Run*)h)->done; }

// Runs the factorization until its flops reach `target` at a checkpoint or
// it ends; returns 1 when it has ended.
int32_t orc_session_advance(void* h, double target) {
  Run* r = (Run*)h;
  std::unique_lock<std::mutex> lk(r->mu);
  if (r->finished) return 1;
  r->target = target;
  r->running = true;
  r->cv.notify_all();
  r->cv.wait(lk, [&] { return !r->running || r->finished; });
  return r->finished ? 1 : 0;
}

// Stops a sliced factorization at its current checkpoint and frees it.
void orc_session_abort(void* h) {
  Run* r = (Run*)h;
  {
    std::lock_guard<std::mutex> lk(r->mu);
    r->abort = true;
    r->running = true;
    r->cv.notify_all();
  }
  r->th.join();
  delete r->O;
  delete r;
}

// Runs the rest, ends the worker and returns the factorization handle (as
// orc_factor does).
void* orc_session_finish(void* h) {
  Run* r = (Run*)h;
  orc_session_advance(h, 1e300);
  r->th.join();
  Oracle* O = r->O;
  delete r;
  return O;
}

void orc_free(void* h) { delete (Oracle*)h; }

// Return the cached front buffers to the system.
void orc_release_cache() { big_cache().release(); }

// counts: [n1x1, n2x2, delayed, zero_pivots, max_front, sn_before, sn_after, merges, sl_subtrees, sl_nodes, ties]
void orc_stats(void* h, int64_t* out) {
  Oracle* O = (Oracle*)h;
  out[0] = O->tot1; out[1] = O->tot2; out[2] = O->totdel; out[3] = O->zero_piv; out[4] = O->max_front;
  out[5] = O->sn_before; out[6] = (i64)O->sn.size(); out[7] = O->merges; out[8] = O->n_sl_sub; out[9] = O->n_sl_nodes;
  out[10] = O->ties;
}

// SparseLDLT::inertia (solver.rs:504-519)
void orc_inertia(void* h, int64_t* out) {
  Oracle* O = (Oracle*)h;
  i64 p = 0, n = 0, z = 0;
  for (auto& F : O->fr) F.d11.inertia(&p, &n, &z);
  out[0] = p; out[1] = n; out[2] = z;
}

int64_t orc_nsup(void* h) { return (i64)((Oracle*)h)->sn.size(); }

// per supernode (post-amalgamation): m, k, ne, n1, n2, parent, n_owned, in_small_leaf, ties
void orc_front_info(void* h, int64_t* out9) {
  Oracle* O = (Oracle*)h;
  for (size_t s = 0; s < O->fr.size(); ++s) {
    Front& F = O->fr[s];
    i64* o = out9 + 9 * s;
    o[0] = F.m; o[1] = F.k; o[2] = F.ne; o[3] = F.n1; o[4] = F.n2; o[5] = O->sn[s].parent;
    o[6] = O->sn[s].n_owned(); o[7] = O->sn[s].in_small_leaf ? 1 : 0; o[8] = F.ties;
  }
}

// Elimination record, fronts in supernode order: eliminated global (permuted)
// column, pivot code (1 = 1x1, 2 = first of 2x2, 3 = second of 2x2), D diag and
// D off-diagonal (for the first of a 2x2).  Returns the number of entries.
int64_t orc_elim(void* h, int64_t* col, int8_t* code, double* dd, double* doff) {
  Oracle* O = (Oracle*)h;
  i64 t = 0;
  for (auto& F : O->fr)
    for (i64 c = 0; c < F.ne; ++c) {
      col[t] = F.col_idx[c];
      code[t] = F.d11.type[c] == PT_1X1 ? 1 : (F.d11.partner[c] > c ? 2 : 3);
      dd[t] = F.d11.diag[c];
      doff[t] = (code[t] == 2) ? F.d11.off[c] : 0.0;
      ++t;
    }
  return t;
}

// SparseLDLT::solve_in_place (solver.rs:370-428) + aptp_solve (solve.rs:57-144)
//
// Large fronts split their triangular solves and products over threads
// without changing what any thread computes for a given front size: the
// forward L11 and L21 updates go by blocks of rows (each entry still takes
// its terms in column order, as in the serial loop), the backward L21 and
// L11 dot products by columns.  The backward L11 solve takes blocks of SB
// columns from the bottom: the dot products against the rows below the block
// run in parallel, then the block itself serially, so for fronts larger than
// SB the order of the subtractions differs from the serial loop (rounding
// only; the factor is not affected), and the result is the same for any
// thread count.
namespace {
const i64 SOLVE_PAR = 2048;  // fronts at least this wide use the blocked, threaded loops
const i64 SB = 256;

void fwd_front(const Front& F, std::vector<double>& x, std::vector<double>& w, std::vector<double>& w2) {
  i64 ne = F.ne;
  i64 r = (i64)F.row_idx.size();
  w.assign(ne, 0.0);
  for (i64 i = 0; i < ne; ++i) w[i] = x[F.col_idx[i]];
  const bool par = ne >= SOLVE_PAR && !omp_in_parallel();
  if (!par) {
    for (i64 j = 0; j < ne; ++j) { double xj = w[j]; for (i64 i = j + 1; i < ne; ++i) w[i] -= F.l11[i + j * ne] * xj; }
  } else {
    // column blocks: finish the block's own rows serially, then the rows below in parallel
    for (i64 j0 = 0; j0 < ne; j0 += SB) {
      const i64 j1 = std::min(ne, j0 + SB);
      for (i64 j = j0; j < j1; ++j) { double xj = w[j]; for (i64 i = j + 1; i < j1; ++i) w[i] -= F.l11[i + j * ne] * xj; }
      const i64 nrow = ne - j1, RB = 1024, nrb = (nrow + RB - 1) / RB;
#pragma omp parallel for schedule(static)
      for (i64 rb = 0; rb < nrb; ++rb) {
        const i64 r0 = j1 + rb * RB, r1 = std::min(ne, r0 + RB);
        for (i64 j = j0; j < j1; ++j) {
          const double xj = w[j];
          const double* l = F.l11.data() + j * ne;
          for (i64 i = r0; i < r1; ++i) w[i] -= l[i] * xj;
        }
      }
    }
  }
  for (i64 i = 0; i < ne; ++i) x[F.col_idx[i]] = w[i];
  if (r > 0) {
    w2.assign(r, 0.0);
    if (!(par || (r * ne >= SOLVE_PAR * SOLVE_PAR && !omp_in_parallel()))) {
      for (i64 j = 0; j < ne; ++j) { double xj = w[j]; const double* l = F.l21.data() + j * r; for (i64 i = 0; i < r; ++i) w2[i] += l[i] * xj; }
    } else {
      const i64 RB = 1024, nrb = (r + RB - 1) / RB;
#pragma omp parallel for schedule(static)
      for (i64 rb = 0; rb < nrb; ++rb) {
        const i64 r0 = rb * RB, r1 = std::min(r, r0 + RB);
        for (i64 j = 0; j < ne; ++j) {
          const double xj = w[j];
          const double* l = F.l21.data() + j * r;
          for (i64 i = r0; i < r1; ++i) w2[i] += l[i] * xj;
        }
      }
    }
    for (i64 i = 0; i < r; ++i) x[F.row_idx[i]] -= w2[i];
  }
}

void bwd_front(const Front& F, std::vector<double>& x, std::vector<double>& w, std::vector<double>& w2) {
  i64 ne = F.ne;
  i64 r = (i64)F.row_idx.size();
  w.assign(ne, 0.0);
  for (i64 i = 0; i < ne; ++i) w[i] = x[F.col_idx[i]];
  const bool big = (ne >= SOLVE_PAR || r * ne >= SOLVE_PAR * SOLVE_PAR) && !omp_in_parallel();
  if (r > 0) {
    w2.assign(r, 0.0);
    for (i64 i = 0; i < r; ++i) w2[i] = x[F.row_idx[i]];
#pragma omp parallel for schedule(static) if (big)
    for (i64 j = 0; j < ne; ++j) {
      const double* l = F.l21.data() + j * r;
      double s2 = 0.0;
      for (i64 i = 0; i < r; ++i) s2 += l[i] * w2[i];
      w[j] -= s2;
    }
  }
  if (ne < SOLVE_PAR || omp_in_parallel()) {
    for (i64 j = ne - 1; j >= 0; --j) { double s2 = w[j]; for (i64 i = j + 1; i < ne; ++i) s2 -= F.l11[i + j * ne] * w[i]; w[j] = s2; }
  } else {
    std::vector<double> t(SB);
    for (i64 j1 = ne; j1 > 0; j1 -= SB) {
      const i64 j0 = std::max<i64>(0, j1 - SB);
#pragma omp parallel for schedule(static)
      for (i64 j = j0; j < j1; ++j) {
        const double* l = F.l11.data() + j * ne;
        double s2 = 0.0;
        for (i64 i = j1; i < ne; ++i) s2 += l[i] * w[i];
        t[j - j0] = s2;
      }
      for (i64 j = j1 - 1; j >= j0; --j) {
        double s2 = w[j] - t[j - j0];
        for (i64 i = j + 1; i < j1; ++i) s2 -= F.l11[i + j * ne] * w[i];
        w[j] = s2;
      }
    }
  }
  for (i64 i = 0; i < ne; ++i) x[F.col_idx[i]] = w[i];
}
}  // namespace

void orc_solve(void* h, double* rhs) {
  Oracle* O = (Oracle*)h;
  i64 n = O->n;
  if (n == 0) return;
  std::vector<double> x(n);
  for (i64 i = 0; i < n; ++i) x[i] = rhs[O->pfwd[i]];
  if (O->has_scaling) for (i64 i = 0; i < n; ++i) x[i] *= O->scaling[i];
  std::vector<double> w, w2;
  // forward (solve.rs:161-225)
  for (auto& F : O->fr) {
    if (F.ne == 0) continue;
    fwd_front(F, x, w, w2);
  }
  // diagonal (solve.rs:232-252)
  for (auto& F : O->fr) {
    i64 ne = F.ne; if (ne == 0) continue;
    w.assign(ne, 0.0);
    for (i64 i = 0; i < ne; ++i) w[i] = x[F.col_idx[i]];
    F.d11.solve(w.data());
    for (i64 i = 0; i < ne; ++i) x[F.col_idx[i]] = w[i];
  }
  // backward (solve.rs:261-326)
  for (i64 s = (i64)O->fr.size() - 1; s >= 0; --s) {
    Front& F = O->fr[s];
    if (F.ne == 0) continue;
    bwd_front(F, x, w, w2);
  }
  if (O->has_scaling) for (i64 i = 0; i < n; ++i) x[i] *= O->scaling[i];
  for (i64 i = 0; i < n; ++i) rhs[O->pfwd[i]] = x[i];
}

// Dense entry: aptp_factor_in_place (factor.rs:301-404) on an m x m
// column-major matrix with p fully summed columns.  Outputs the column
// permutation (m), the D entries (type/diag/off, length p) and
// [ne, n1x1, n2x2, ndelayed]; `maxl` receives stats.max_l_entry.
void orc_dense_aptp(int64_t m, int64_t p, double* a, const orc_options* opt, int64_t* perm,
                    int8_t* dtype, double* ddiag, double* doff, int64_t* st4, double* maxl) {
  Opts o;
  if (opt) {
    o.threshold = opt->threshold; o.small = opt->small; o.nb = opt->outer_block_size; o.ib = opt->inner_block_size;
    o.failed_pivot_tpp = opt->failed_pivot_tpp;
  }
  MV A{a, m};
  FactorResult R = aptp_factor_in_place(A, m, p, o);
  for (i64 i = 0; i < m; ++i) perm[i] = R.perm[i];
  for (i64 c = 0; c < p; ++c) {
    if (c < R.ne) {
      dtype[c] = R.d.type[c] == PT_1X1 ? 1 : (R.d.partner[c] > c ? 2 : 3);
      ddiag[c] = R.d.diag[c];
      doff[c] = R.d.is2first(c) ? R.d.off[c] : 0.0;
    } else { dtype[c] = 0; ddiag[c] = 0; doff[c] = 0; }
  }
  st4[0] = R.ne; st4[1] = R.st.n1; st4[2] = R.st.n2; st4[3] = R.st.ndel;
  *maxl = R.st.maxl;
}

}  // extern "C"
