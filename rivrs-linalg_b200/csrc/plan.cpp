// Pattern-only preparation of the numeric phase, done once per sparsity
// pattern on the host: the first half of AptpNumeric::factor
// (sparse/src/symmetric/numeric.rs:844-905).
//   * supernode descriptors from the symbolic partition (build_supernode_info,
//     numeric.rs:2179-2236),
//   * amalgamation with the nemin / structural-match rule
//     (amalgamation.rs:38-54 do_merge, 115-231 amalgamate),
//   * the children map (numeric.rs:2239-2248),
//   * small-leaf subtree classification (numeric.rs:2278-2369),
//   * the delay-free assembly maps (numeric.rs:264-408),
//   * the wave (height) of every front for the level-set schedule, and the
//     algorithmic work of the delay-free structure.
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "rvg_internal.h"

namespace rvg {

namespace {

// Merge predicate (amalgamation.rs:38-54).
bool merge_rule(int64_t pn, int64_t pcc, int64_t cn, int64_t ccc, int64_t nemin) {
  if (pn == 1 && pcc == (ccc > 0 ? ccc - 1 : 0)) return true;
  return pn < nemin && cn < nemin;
}

// Sorted union of two ascending lists, dropping values inside [lo, hi)
// (amalgamation.rs:57-95).
std::vector<int64_t> merge_patterns(const std::vector<int64_t>& a, const std::vector<int64_t>& b, int64_t lo,
                                    int64_t hi) {
  std::vector<int64_t> out;
  out.reserve(a.size() + b.size());
  size_t i = 0, j = 0;
  while (i < a.size() || j < b.size()) {
    int64_t v;
    if (j == b.size() || (i < a.size() && a[i] < b[j])) v = a[i++];
    else if (i == a.size() || b[j] < a[i]) v = b[j++];
    else { v = a[i]; ++i; ++j; }
    if (v < lo || v >= hi) out.push_back(v);
  }
  return out;
}

// amalgamation.rs:115-231.  Parents are visited in ascending (postorder)
// index; each parent tests its original children in order and absorbs the
// ones the rule accepts, inheriting their owned column ranges and children.
void amalgamate(std::vector<Snode>& sn, int64_t nemin, int64_t* merges) {
  const int64_t n = (int64_t)sn.size();
  *merges = 0;
  if (n <= 1) return;
  std::vector<char> gone(n, 0);
  std::vector<int64_t> nel(n);
  std::vector<std::vector<int64_t>> kids(n);
  for (int64_t s = 0; s < n; ++s) {
    nel[s] = sn[s].col_end - sn[s].col_begin;
    if (sn[s].parent >= 0) kids[sn[s].parent].push_back(s);
  }
  for (int64_t p = 0; p < n; ++p) {
    if (gone[p]) continue;
    std::vector<int64_t> orig = std::move(kids[p]);
    kids[p].clear();
    for (int64_t c : orig) {
      if (gone[c]) continue;
      if (!merge_rule(nel[p], nel[p] + (int64_t)sn[p].pattern.size(), nel[c],
                      nel[c] + (int64_t)sn[c].pattern.size(), nemin))
        continue;
      int64_t lo = std::min(sn[p].col_begin, sn[c].col_begin);
      int64_t hi = std::max(sn[p].col_end, sn[c].col_end);
      sn[p].pattern = merge_patterns(sn[p].pattern, sn[c].pattern, lo, hi);
      sn[c].pattern.clear();
      sn[p].owned.insert(sn[p].owned.end(), sn[c].owned.begin(), sn[c].owned.end());
      sn[c].owned.clear();
      sn[p].col_begin = lo;
      sn[p].col_end = hi;
      nel[p] += nel[c];
      for (int64_t g : kids[c]) if (!gone[g]) sn[g].parent = p;
      kids[p].insert(kids[p].end(), kids[c].begin(), kids[c].end());
      kids[c].clear();
      gone[c] = 1;
    }
    for (int64_t c : orig) if (!gone[c]) kids[p].push_back(c);
  }
  std::vector<int64_t> renum(n, -1);
  int64_t m = 0;
  for (int64_t s = 0; s < n; ++s) if (!gone[s]) renum[s] = m++;
  std::vector<Snode> out;
  out.reserve(m);
  for (int64_t s = 0; s < n; ++s) {
    if (gone[s]) continue;
    Snode x = std::move(sn[s]);
    if (x.parent >= 0) x.parent = renum[x.parent];
    out.push_back(std::move(x));
  }
  *merges = n - m;
  sn.swap(out);
}

// numeric.rs:2278-2369: mark fronts below the threshold whose children are
// all marked; keep only subtrees of two or more nodes.
void classify_small_leaf(std::vector<Snode>& sn, const std::vector<std::vector<int64_t>>& ch, int64_t thr,
                         int64_t* nsub, int64_t* nnodes) {
  *nsub = 0;
  *nnodes = 0;
  if (thr == 0) return;
  const int64_t n = (int64_t)sn.size();
  for (int64_t s = 0; s < n; ++s) {
    int64_t front = sn[s].n_owned() + (int64_t)sn[s].pattern.size();
    bool mark = front < thr;
    if (mark) for (int64_t c : ch[s]) mark = mark && sn[c].in_small_leaf;
    sn[s].in_small_leaf = mark;
  }
  for (int64_t s = 0; s < n; ++s) {
    if (!sn[s].in_small_leaf) continue;
    if (sn[s].parent >= 0 && sn[sn[s].parent].in_small_leaf) continue;
    // count the subtree below s restricted to marked nodes
    int64_t cnt = 0;
    std::vector<int64_t> st{s};
    while (!st.empty()) {
      int64_t x = st.back();
      st.pop_back();
      ++cnt;
      for (int64_t c : ch[x]) if (sn[c].in_small_leaf) st.push_back(c);
    }
    if (cnt < 2) { sn[s].in_small_leaf = false; continue; }
    *nsub += 1;
    *nnodes += cnt;
  }
}

}  // namespace

int build_plan(const Symbolic* S, int64_t n, int64_t nsup, const int64_t* sup_begin, const int64_t* sup_end,
               const int64_t* pat_ptr, const int64_t* pat_idx, const int64_t* sup_parent,
               const int64_t* perm_fwd, const int64_t* colptr, const int64_t* rowidx,
               const rvg_options& opt, Plan& P, std::string* err) {
  (void)S;
  P = Plan();
  P.n = n;
  P.perm_fwd.assign(perm_fwd, perm_fwd + n);
  std::vector<int64_t> pinv(n, -1);
  for (int64_t i = 0; i < n; ++i) {
    if (perm_fwd[i] < 0 || perm_fwd[i] >= n || pinv[perm_fwd[i]] != -1) {
      if (err) *err = "perm_fwd is not a permutation";
      return RVG_ERR_INVALID_INPUT;
    }
    pinv[perm_fwd[i]] = i;
  }
  // supernode descriptors
  P.sn.resize(nsup);
  for (int64_t s = 0; s < nsup; ++s) {
    Snode& x = P.sn[s];
    x.col_begin = sup_begin[s];
    x.col_end = sup_end[s];
    if (x.col_end <= x.col_begin || x.col_end > n) {
      if (err) *err = "empty or out-of-range supernode";
      return RVG_ERR_INVALID_INPUT;
    }
    x.pattern.assign(pat_idx + pat_ptr[s], pat_idx + pat_ptr[s + 1]);
    x.parent = sup_parent[s];
    if (x.parent >= nsup || (x.parent >= 0 && x.parent <= s)) {
      if (err) *err = "supernode parents must follow their children (postorder)";
      return RVG_ERR_INVALID_INPUT;
    }
    x.owned.assign(1, {x.col_begin, x.col_end});
  }
  P.nsup_before = nsup;
  amalgamate(P.sn, opt.nemin, &P.merges);
  const int64_t ns = (int64_t)P.sn.size();
  P.children.assign(ns, {});
  for (int64_t s = 0; s < ns; ++s) if (P.sn[s].parent >= 0) P.children[P.sn[s].parent].push_back(s);
  classify_small_leaf(P.sn, P.children, opt.small_leaf_threshold, &P.sl_subtrees, &P.sl_nodes);
  // waves: height above the leaves
  P.height.assign(ns, 0);
  int64_t hmax = 0;
  for (int64_t s = 0; s < ns; ++s) {
    for (int64_t c : P.children[s]) P.height[s] = std::max(P.height[s], P.height[c] + 1);
    hmax = std::max(hmax, P.height[s]);
  }
  P.waves.assign(ns ? hmax + 1 : 0, {});
  for (int64_t s = 0; s < ns; ++s) P.waves[P.height[s]].push_back(s);
  // owned columns and patterns, front-local numbering
  P.own_ptr.assign(ns + 1, 0);
  P.pat_ptr.assign(ns + 1, 0);
  for (int64_t s = 0; s < ns; ++s) {
    P.own_ptr[s + 1] = P.own_ptr[s] + P.sn[s].n_owned();
    P.pat_ptr[s + 1] = P.pat_ptr[s] + (int64_t)P.sn[s].pattern.size();
  }
  P.own_idx.resize(P.own_ptr[ns]);
  P.pat_idx.resize(P.pat_ptr[ns]);
  for (int64_t s = 0; s < ns; ++s) {
    int64_t t = P.own_ptr[s];
    for (auto& r : P.sn[s].owned) for (int64_t c = r.first; c < r.second; ++c) P.own_idx[t++] = (int32_t)c;
    for (size_t q = 0; q < P.sn[s].pattern.size(); ++q) P.pat_idx[P.pat_ptr[s] + q] = (int32_t)P.sn[s].pattern[q];
  }
  // assembly maps (numeric.rs:264-408)
  std::vector<int64_t> g2l(n, -1);
  P.amap_ptr.assign(ns + 1, 0);
  P.amap.clear();
  for (int64_t s = 0; s < ns; ++s) {
    const Snode& x = P.sn[s];
    int64_t no = x.n_owned();
    int64_t loc = 0;
    for (int64_t q = P.own_ptr[s]; q < P.own_ptr[s + 1]; ++q) g2l[P.own_idx[q]] = loc++;
    for (int64_t c : x.pattern) g2l[c] = loc++;
    int64_t m = loc;
    for (int64_t q = P.own_ptr[s]; q < P.own_ptr[s + 1]; ++q) {
      int64_t pj = P.own_idx[q];
      int64_t oc = perm_fwd[pj];
      int64_t lc = g2l[pj];
      for (int64_t idx = colptr[oc]; idx < colptr[oc + 1]; ++idx) {
        int64_t orow = rowidx[idx];
        if (orow < oc) {
          int64_t lp = g2l[pinv[orow]];
          if (lp >= 0 && lp < no) continue;  // both owned: keep the lower copy only
        }
        int64_t gr = pinv[orow];
        int64_t lr = g2l[gr];
        if (lr < 0) continue;
        int64_t dr = lr >= lc ? lr : lc, dc = lr >= lc ? lc : lr;
        if (idx > INT32_MAX) {
          if (err) *err = "more than 2^31 stored entries";
          return RVG_ERR_INVALID_INPUT;
        }
        P.amap.push_back((int32_t)idx);
        P.amap.push_back((int32_t)dr);
        P.amap.push_back((int32_t)dc);
        P.amap.push_back((int32_t)gr);
        P.amap.push_back((int32_t)pj);
      }
    }
    for (int64_t q = P.own_ptr[s]; q < P.own_ptr[s + 1]; ++q) g2l[P.own_idx[q]] = -1;
    for (int64_t c : x.pattern) g2l[c] = -1;
    P.amap_ptr[s + 1] = (int64_t)P.amap.size() / 5;
    (void)m;
  }
  P.ea_ptr.assign(ns + 1, 0);
  P.ea_map.clear();
  for (int64_t s = 0; s < ns; ++s) {
    // ea_map is stored per CHILD s: its pattern rows located in the parent
    P.ea_ptr[s + 1] = P.ea_ptr[s] + (int64_t)P.sn[s].pattern.size();
  }
  P.ea_map.resize(P.ea_ptr[ns]);
  for (int64_t p = 0; p < ns; ++p) {
    int64_t loc = 0;
    for (int64_t q = P.own_ptr[p]; q < P.own_ptr[p + 1]; ++q) g2l[P.own_idx[q]] = loc++;
    for (int64_t c : P.sn[p].pattern) g2l[c] = loc++;
    for (int64_t c : P.children[p]) {
      for (size_t q = 0; q < P.sn[c].pattern.size(); ++q) {
        int64_t l = g2l[P.sn[c].pattern[q]];
        if (l < 0) {
          if (err) *err = "child pattern row not in parent front";
          return RVG_ERR_INVALID_INPUT;
        }
        P.ea_map[P.ea_ptr[c] + q] = (int32_t)l;
      }
    }
    for (int64_t q = P.own_ptr[p]; q < P.own_ptr[p + 1]; ++q) g2l[P.own_idx[q]] = -1;
    for (int64_t c : P.sn[p].pattern) g2l[c] = -1;
  }
  // algorithmic work of the delay-free structure
  P.flops_factor = 0; P.flops_schur = 0; P.bytes_assembly = 0; P.nnz_l = 0; P.max_front = 0;
  for (int64_t s = 0; s < ns; ++s) {
    double k = (double)P.sn[s].n_owned(), m = k + (double)P.sn[s].pattern.size();
    double nfs = m - k;
    for (int64_t j = 0; j < (int64_t)k; ++j) {
      double r = m - j - 1;
      P.flops_factor += r + r * (m - j);
    }
    P.flops_schur += nfs * (nfs + 1) * k;
    P.nnz_l += (int64_t)(k * (k + 1) / 2 + nfs * k);
    P.max_front = std::max<int64_t>(P.max_front, (int64_t)m);
    if (P.sn[s].parent >= 0) {
      double cb = nfs * (nfs + 1) / 2;
      P.bytes_assembly += cb * 24 + 4 * nfs;
    }
  }
  P.bytes_assembly += (double)(P.amap.size() / 5) * (8 + 16 + 16);
  return RVG_OK;
}

}  // namespace rvg
