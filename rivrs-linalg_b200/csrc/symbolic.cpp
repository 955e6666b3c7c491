// Host symbolic analysis: the stand-in for the AptpSymbolic the numeric phase
// consumes (sparse/src/symmetric/symbolic.rs:248-310, which wraps faer's
// symbolic Cholesky; faer's source is not part of the reference, so the
// partition rules below are this project's own).
//
// Given the full symmetric CSC pattern and a fill-reducing order
// (order[new] = old, the UserSupplied semantics of solver.rs:51-52), it
// computes
//   * the elimination tree of P A P^T (Liu's algorithm with path compression),
//   * a postorder of that tree, composed into the returned permutation,
//   * column counts of L (Gilbert-Ng-Peyton row-subtree / LCA method),
//   * fundamental supernodes (parent(j) == j+1, j the only child of j+1 and
//     cc(j) == cc(j+1) + 1), then relaxed: a supernode is merged into its
//     parent when it ends where the parent begins and the explicit zeros of
//     the merged block stay under 100% / 80% / 10% / 5% of its storage for
//     merged widths <= 4 / 16 / 48 / above,
//   * each supernode's row pattern (rows of L below its last column) and its
//     parent in the assembly tree (supernode_parent, symbolic.rs:576-598).
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "rvg_internal.h"

namespace rvg {

static int sym_fail(std::string* err, const std::string& m) {
  if (err) *err = m;
  return RVG_ERR_INVALID_INPUT;
}

int symbolic_analyze(int64_t n, const int64_t* colptr, const int64_t* rowidx, const int64_t* order,
                     Symbolic& S, std::string* err) {
  S = Symbolic();
  S.n = n;
  if (n < 0) return sym_fail(err, "negative dimension");
  if (n == 0) { S.pat_ptr.assign(1, 0); return RVG_OK; }
  if (n >= (int64_t)INT32_MAX) return sym_fail(err, "dimension too large for 32-bit front indices");
  for (int64_t j = 0; j < n; ++j)
    if (colptr[j + 1] < colptr[j]) return sym_fail(err, "column pointers are not monotone");
  for (int64_t p = 0; p < colptr[n]; ++p)
    if (rowidx[p] < 0 || rowidx[p] >= n) return sym_fail(err, "row index out of range");
  // initial order and its inverse
  std::vector<int64_t> ord(n), inv(n, -1);
  for (int64_t k = 0; k < n; ++k) {
    int64_t o = order ? order[k] : k;
    if (o < 0 || o >= n || inv[o] != -1) return sym_fail(err, "ordering is not a permutation");
    ord[k] = o;
    inv[o] = k;
  }
  // 1. elimination tree of P A P^T
  std::vector<int64_t> parent(n, -1), anc(n, -1);
  for (int64_t k = 0; k < n; ++k) {
    int64_t oc = ord[k];
    for (int64_t p = colptr[oc]; p < colptr[oc + 1]; ++p) {
      int64_t i = inv[rowidx[p]];
      while (i != -1 && i < k) {
        int64_t nx = anc[i];
        anc[i] = k;
        if (nx == -1) { parent[i] = k; break; }
        i = nx;
      }
    }
  }
  // 2. postorder (roots and children in ascending order)
  std::vector<int64_t> head(n, -1), next(n, -1);
  for (int64_t j = n - 1; j >= 0; --j)
    if (parent[j] != -1) { next[j] = head[parent[j]]; head[parent[j]] = j; }
  std::vector<int64_t> post; post.reserve(n);
  std::vector<int64_t> stack; stack.reserve(n);
  for (int64_t r = 0; r < n; ++r) {
    if (parent[r] != -1) continue;
    stack.push_back(r);
    while (!stack.empty()) {
      int64_t x = stack.back();
      int64_t c = head[x];
      if (c == -1) { post.push_back(x); stack.pop_back(); }
      else { head[x] = next[c]; stack.push_back(c); }
    }
  }
  if ((int64_t)post.size() != n) return sym_fail(err, "elimination tree is not a forest");
  std::vector<int64_t> where(n);
  for (int64_t k = 0; k < n; ++k) where[post[k]] = k;
  S.perm_fwd.resize(n);
  S.perm_inv.resize(n);
  std::vector<int64_t> et(n);
  for (int64_t k = 0; k < n; ++k) {
    S.perm_fwd[k] = ord[post[k]];
    int64_t p = parent[post[k]];
    et[k] = p == -1 ? -1 : where[p];
  }
  for (int64_t k = 0; k < n; ++k) S.perm_inv[S.perm_fwd[k]] = k;
  // 3. column counts by row subtrees: delta(+1 at each leaf of a row subtree,
  //    -1 at the LCA of consecutive leaves and at parent(row)), summed over
  //    each subtree.
  std::vector<int64_t> first(n, -1);
  for (int64_t k = 0; k < n; ++k)
    for (int64_t j = k; j != -1 && first[j] == -1; j = et[j]) first[j] = k;
  std::vector<int64_t> delta(n, 0), lastcol(n, -1), prevleaf(n, -1), uf(n);
  for (int64_t k = 0; k < n; ++k) uf[k] = k;
  auto find = [&](int64_t x) {
    int64_t r = x;
    while (uf[r] != r) r = uf[r];
    while (uf[x] != r) { int64_t nx = uf[x]; uf[x] = r; x = nx; }
    return r;
  };
  for (int64_t j = 0; j < n; ++j) {
    int64_t oc = S.perm_fwd[j];
    for (int64_t p = colptr[oc]; p < colptr[oc + 1]; ++p) {
      int64_t i = S.perm_inv[rowidx[p]];
      if (i <= j) continue;
      if (first[j] > lastcol[i]) {
        delta[j] += 1;
        if (prevleaf[i] != -1) delta[find(prevleaf[i])] -= 1;
        prevleaf[i] = j;
      }
      lastcol[i] = j;
    }
    if (et[j] != -1) uf[j] = et[j];
  }
  for (int64_t i = 0; i < n; ++i) {
    if (prevleaf[i] == -1) delta[i] += 1;  // row without off-diagonal entries: {i}
    if (et[i] != -1) delta[et[i]] -= 1;    // every row subtree ends at i
  }
  std::vector<int64_t> cc(delta);
  for (int64_t j = 0; j < n; ++j)
    if (et[j] != -1) cc[et[j]] += cc[j];
  // 4. fundamental supernodes
  std::vector<int64_t> nchild(n, 0);
  for (int64_t j = 0; j < n; ++j) if (et[j] != -1) nchild[et[j]]++;
  std::vector<int64_t> snode_of(n);
  S.sup_begin.clear(); S.sup_end.clear();
  for (int64_t j = 0; j < n; ++j) {
    bool join = j > 0 && et[j - 1] == j && nchild[j] == 1 && cc[j - 1] == cc[j] + 1;
    if (!join) S.sup_begin.push_back(j);
    snode_of[j] = (int64_t)S.sup_begin.size() - 1;
  }
  int64_t ns = (int64_t)S.sup_begin.size();
  S.sup_end.resize(ns);
  for (int64_t s = 0; s < ns; ++s) S.sup_end[s] = (s + 1 < ns) ? S.sup_begin[s + 1] : n;
  S.sup_parent.assign(ns, -1);
  for (int64_t s = 0; s < ns; ++s) {
    int64_t p = et[S.sup_end[s] - 1];
    S.sup_parent[s] = p == -1 ? -1 : snode_of[p];
  }
  // 5. relaxed supernodes: merge a supernode into its parent when it ends
  //    where the parent begins and the merged block keeps its explicit-zero
  //    fraction under a size-dependent bound.  Only column counts are needed:
  //    a fundamental supernode's pattern has cc(begin) - width rows, and
  //    merging s into p keeps p's pattern (pattern(s) lies inside
  //    cols(p) + pattern(p)), so each column of s gains
  //    (k_p + |pat p| - |pat s|) stored entries.
  std::vector<int64_t> gbeg(ns), gk(ns), gpat(ns);
  std::vector<double> gzero(ns, 0.0), gstore(ns, 0.0);
  for (int64_t s = 0; s < ns; ++s) {
    gbeg[s] = S.sup_begin[s];
    gk[s] = S.sup_end[s] - S.sup_begin[s];
    gpat[s] = cc[S.sup_begin[s]] - gk[s];
    double k = (double)gk[s];
    gstore[s] = k * (k + 1) / 2 + k * (double)gpat[s];
    double nz = 0;
    for (int64_t j = S.sup_begin[s]; j < S.sup_end[s]; ++j) nz += (double)cc[j];
    gzero[s] = gstore[s] - nz;
  }
  std::vector<char> absorbed(ns, 0);
  for (int64_t s = 0; s < ns; ++s) {
    int64_t p = S.sup_parent[s];
    if (p < 0 || S.sup_end[s] != S.sup_begin[p]) continue;
    double ks = (double)gk[s], kp = (double)gk[p];
    double extra = ks * (kp + (double)gpat[p] - (double)gpat[s]);
    double km = ks + kp;
    double store = ks * (ks + 1) / 2 + ks * (kp + (double)gpat[p]) + gstore[p];
    double zero = gzero[s] + gzero[p] + extra;
    double lim = km <= 4 ? 1.0 : km <= 16 ? 0.8 : km <= 48 ? 0.1 : 0.05;
    if (zero > lim * store) continue;
    absorbed[s] = 1;
    gbeg[p] = gbeg[s];
    gk[p] += gk[s];
    gstore[p] = store;
    gzero[p] = zero;
  }
  {
    int64_t nn = 0;
    std::vector<int64_t> newid(ns, -1);
    for (int64_t s = 0; s < ns; ++s) if (!absorbed[s]) newid[s] = nn++;
    std::vector<int64_t> nb(nn), ne_(nn), np(nn, -1), npp(nn + 1, 0);
    std::vector<int64_t> col_group(n, -1);
    for (int64_t s = 0; s < ns; ++s)
      if (!absorbed[s]) {
        int64_t g = newid[s];
        nb[g] = gbeg[s];
        ne_[g] = S.sup_end[s];
        for (int64_t j = nb[g]; j < ne_[g]; ++j) col_group[j] = g;
        npp[g + 1] = npp[g] + gpat[s];
      }
    for (int64_t g = 0; g < nn; ++g) {
      int64_t pc = et[ne_[g] - 1];
      np[g] = pc < 0 ? -1 : col_group[pc];
    }
    S.sup_begin.swap(nb);
    S.sup_end.swap(ne_);
    S.sup_parent.swap(np);
    S.pat_ptr.swap(npp);
    ns = nn;
  }
  // 6. patterns of the relaxed supernodes: rows >= end of A's columns in s
  //    plus the children's patterns (children precede their parent); the
  //    sizes are known from the column counts.
  std::vector<std::vector<int64_t>> ch(ns);
  for (int64_t s = 0; s < ns; ++s) if (S.sup_parent[s] >= 0) ch[S.sup_parent[s]].push_back(s);
  S.pat_idx.resize(S.pat_ptr[ns]);
  std::vector<int64_t> mark(n, -1), P;
  for (int64_t s = 0; s < ns; ++s) {
    int64_t b = S.sup_begin[s], e = S.sup_end[s];
    P.clear();
    for (int64_t j = b; j < e; ++j) {
      int64_t oc = S.perm_fwd[j];
      for (int64_t p = colptr[oc]; p < colptr[oc + 1]; ++p) {
        int64_t i = S.perm_inv[rowidx[p]];
        if (i >= e && mark[i] != s) { mark[i] = s; P.push_back(i); }
      }
    }
    for (int64_t c : ch[s])
      for (int64_t q = S.pat_ptr[c]; q < S.pat_ptr[c + 1]; ++q) {
        int64_t i = S.pat_idx[q];
        if (i >= e && mark[i] != s) { mark[i] = s; P.push_back(i); }
      }
    if ((int64_t)P.size() != S.pat_ptr[s + 1] - S.pat_ptr[s])
      return sym_fail(err, "internal: supernode pattern disagrees with column count");
    std::sort(P.begin(), P.end());
    std::copy(P.begin(), P.end(), S.pat_idx.begin() + S.pat_ptr[s]);
  }
  S.colcount = std::move(cc);
  S.etree = std::move(et);
  return RVG_OK;
}

}  // namespace rvg
