// MC64 maximum-product matching and symmetric scaling (mc64_matching,
// sparse/src/ordering/matching.rs:121-248), restated from the published
// method: Duff & Koster, "On algorithms for permuting large entries to the
// diagonal of a sparse matrix" (SIMAX 2001), algorithm MPD, and the symmetric
// scaling of Duff & Pralet (SIMAX 2005).
//
// Maximise prod |a_{i,sigma(i)}| <=> minimise sum c_{i,sigma(i)} with
// c_ij = log(max_k |a_kj|) - log|a_ij| >= 0 (columns normalised to a maximum
// of 1).  Row duals u and column duals v are kept dual feasible
// (c_ij - u_i - v_j >= 0) and tight on matched edges.  Start: u_i = row
// minimum, v_j = column minimum of the reduced costs, a greedy matching on
// tight edges; then every unmatched column is matched along a shortest
// augmenting path (Dijkstra on reduced costs from the column, through matched
// edges of zero reduced cost), after which the duals of the nodes settled
// before the path's end are shifted by their distance gap, which keeps every
// reduced cost non-negative and makes the new matched edges tight.
//
// Scaling: s_i = exp((u_i + v_i - log colmax_i) / 2).  With optimal duals,
// |s_i a_ij s_j| = exp(-(rc_ij + rc_ji) / 2) <= 1, and because the transposed
// matching of a symmetric matrix is optimal too, complementary slackness makes
// both rc_{i,sigma(i)} and rc_{sigma(i),i} zero: every nonzero row reaches 1.
// For structurally singular matrices (rows left unmatched) the duals of the
// unmatched rows are set to zero and those of unmatched columns too, the
// convention of matching.rs:214-226; unmatched rows take the free columns in
// order (build_singular_permutation, matching.rs:326-357).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <limits>
#include <queue>
#include <string>
#include <vector>

#include "../../include/rivrs_b200.h"

namespace rvg {
void set_error(const std::string& s);
}

namespace {

constexpr double kLogScaleClamp = 500.0;  // exp() stays finite (matching.rs:99)
constexpr int64_t kNone = -1;

struct CostGraph {
  int64_t n = 0;
  std::vector<int64_t> ptr, row;
  std::vector<double> cost, colmax_log;
};

// Full symmetric pattern (an entry stored once or twice becomes both (i, j)
// and (j, i)), explicit zeros dropped, rows sorted per column.
CostGraph build_graph(int64_t n, const int64_t* colptr, const int64_t* rowidx, const double* val) {
  using Entry = std::pair<int64_t, double>;  // (row, |a|)
  // one array for every column's entries, both orientations: count, place, then sort each column
  std::vector<int64_t> start(n + 1, 0);
  for (int64_t j = 0; j < n; ++j)
    for (int64_t k = colptr[j]; k < colptr[j + 1]; ++k) {
      if (val[k] == 0.0) continue;
      const int64_t i = rowidx[k];
      ++start[j + 1];
      if (i != j) ++start[i + 1];
    }
  for (int64_t j = 0; j < n; ++j) start[j + 1] += start[j];
  std::vector<Entry> ent(start[n]);
  {
    std::vector<int64_t> fill(start.begin(), start.end() - 1);
    for (int64_t j = 0; j < n; ++j)
      for (int64_t k = colptr[j]; k < colptr[j + 1]; ++k) {
        const double a = std::fabs(val[k]);
        if (a == 0.0) continue;
        const int64_t i = rowidx[k];
        ent[fill[j]++] = {i, a};
        if (i != j) ent[fill[i]++] = {j, a};
      }
  }
  CostGraph g;
  g.n = n;
  g.ptr.assign(n + 1, 0);
  g.colmax_log.assign(n, -std::numeric_limits<double>::infinity());
  g.row.resize(start[n]);
  g.cost.resize(start[n]);
  int64_t p = 0;
  for (int64_t j = 0; j < n; ++j) {
    // rows in increasing order; an entry stored in both triangles appears twice: keep one (the smaller |a|)
    auto b = ent.begin() + start[j], e = ent.begin() + start[j + 1];
    std::sort(b, e, [](const Entry& x, const Entry& y) { return x.first < y.first || (x.first == y.first && x.second < y.second); });
    e = std::unique(b, e, [](const Entry& x, const Entry& y) { return x.first == y.first; });
    const int64_t p0 = p;
    for (auto it = b; it != e; ++it, ++p) {
      g.row[p] = it->first;
      g.cost[p] = std::log(it->second);  // log |a| for now
      g.colmax_log[j] = std::max(g.colmax_log[j], g.cost[p]);
    }
    for (int64_t q = p0; q < p; ++q) g.cost[q] = g.colmax_log[j] - g.cost[q];
    g.ptr[j + 1] = p;
  }
  g.row.resize(p);
  g.cost.resize(p);
  return g;
}

struct Matcher {
  const CostGraph& g;
  std::vector<double> u, v;
  std::vector<int64_t> row_match, col_match;
  // Dijkstra state, reset through the touched lists
  std::vector<double> dist;      // per row
  std::vector<int64_t> pred;     // per row: column it was reached from
  std::vector<char> done;        // per row: settled
  std::vector<int64_t> touched;  // rows with a finite distance

  explicit Matcher(const CostGraph& gr)
      : g(gr), u(gr.n, 0.0), v(gr.n, 0.0), row_match(gr.n, kNone), col_match(gr.n, kNone),
        dist(gr.n, std::numeric_limits<double>::infinity()), pred(gr.n, kNone), done(gr.n, 0) {}

  double rc(int64_t k, int64_t j) const { return g.cost[k] - u[g.row[k]] - v[j]; }

  void initial() {
    const int64_t n = g.n;
    std::vector<double> umin(n, std::numeric_limits<double>::infinity());
    for (int64_t j = 0; j < n; ++j)
      for (int64_t k = g.ptr[j]; k < g.ptr[j + 1]; ++k) umin[g.row[k]] = std::min(umin[g.row[k]], g.cost[k]);
    for (int64_t i = 0; i < n; ++i) u[i] = std::isinf(umin[i]) ? 0.0 : umin[i];
    for (int64_t j = 0; j < n; ++j) {
      double best = std::numeric_limits<double>::infinity();
      int64_t bk = kNone;
      for (int64_t k = g.ptr[j]; k < g.ptr[j + 1]; ++k) {
        const double r = g.cost[k] - u[g.row[k]];
        // the smallest reduced cost; among equal ones an unmatched row
        if (r < best || (r == best && bk != kNone && row_match[g.row[bk]] != kNone && row_match[g.row[k]] == kNone)) {
          best = r;
          bk = k;
        }
      }
      if (bk == kNone) continue;  // empty column
      v[j] = best;
      const int64_t i = g.row[bk];
      if (row_match[i] == kNone) {  // rc = 0 on this edge: a tight match
        row_match[i] = j;
        col_match[j] = i;
      }
    }
  }

  // shortest augmenting path from the unmatched column root
  bool augment(int64_t root) {
    using Item = std::pair<double, int64_t>;
    std::priority_queue<Item, std::vector<Item>, std::greater<Item>> heap;
    auto relax = [&](int64_t j, double dj) {
      for (int64_t k = g.ptr[j]; k < g.ptr[j + 1]; ++k) {
        const int64_t i = g.row[k];
        if (done[i]) continue;
        const double d = dj + std::max(0.0, rc(k, j));
        if (d < dist[i]) {
          if (std::isinf(dist[i])) touched.push_back(i);
          dist[i] = d;
          pred[i] = j;
          heap.push({d, i});
        }
      }
    };
    relax(root, 0.0);
    std::vector<int64_t> settled;
    int64_t end = kNone;
    double delta = 0.0;
    while (!heap.empty()) {
      const auto [d, i] = heap.top();
      heap.pop();
      if (done[i] || d > dist[i]) continue;
      done[i] = 1;
      if (row_match[i] == kNone) {
        end = i;
        delta = d;
        break;
      }
      settled.push_back(i);
      relax(row_match[i], d);  // through the matched edge (reduced cost 0)
    }
    if (end != kNone) {
      // dual shift of the nodes settled before the end: rows by -(delta - d),
      // their matched columns and the root by +(delta - d)
      v[root] += delta;
      for (int64_t i : settled) {
        const double gap = delta - dist[i];
        u[i] -= gap;
        v[row_match[i]] += gap;
      }
      // flip the path
      int64_t i = end;
      for (;;) {
        const int64_t j = pred[i];
        const int64_t prev = col_match[j];
        col_match[j] = i;
        row_match[i] = j;
        if (j == root) break;
        i = prev;
      }
    }
    for (int64_t i : touched) {
      dist[i] = std::numeric_limits<double>::infinity();
      pred[i] = kNone;
      done[i] = 0;
    }
    touched.clear();
    return end != kNone;
  }
};

}  // namespace

extern "C" rvg_status rvg_mc64(int64_t n, const int64_t* colptr, const int64_t* rowidx, const double* values,
                               int64_t* matching, double* scaling, int64_t* matched) {
  if (n <= 0) { rvg::set_error("MC64 requires a non-empty matrix"); return RVG_ERR_INVALID_INPUT; }
  if (!colptr || !rowidx || !values || !matching || !scaling) { rvg::set_error("null argument"); return RVG_ERR_INVALID_INPUT; }
  for (int64_t k = 0; k < colptr[n]; ++k) {
    if (!std::isfinite(values[k])) { rvg::set_error("MC64 requires finite matrix entries"); return RVG_ERR_INVALID_INPUT; }
    if (rowidx[k] < 0 || rowidx[k] >= n) { rvg::set_error("row index out of range"); return RVG_ERR_INVALID_INPUT; }
  }
  const CostGraph g = build_graph(n, colptr, rowidx, values);
  Matcher M(g);
  M.initial();
  for (int64_t j = 0; j < n; ++j)
    if (M.col_match[j] == kNone && g.ptr[j + 1] > g.ptr[j]) M.augment(j);
  int64_t cnt = 0;
  for (int64_t j = 0; j < n; ++j) cnt += M.col_match[j] != kNone;
  // duals of the scaling: unmatched rows and columns at zero; matched columns
  // from complementary slackness on their matched edge
  for (int64_t i = 0; i < n; ++i)
    if (M.row_match[i] == kNone) M.u[i] = 0.0;
  for (int64_t j = 0; j < n; ++j) {
    const int64_t i = M.col_match[j];
    if (i == kNone) { M.v[j] = 0.0; continue; }
    for (int64_t k = g.ptr[j]; k < g.ptr[j + 1]; ++k)
      if (g.row[k] == i) { M.v[j] = g.cost[k] - M.u[i]; break; }
  }
  for (int64_t i = 0; i < n; ++i) {
    double ls = (M.u[i] + M.v[i] - g.colmax_log[i]) / 2.0;
    ls = std::min(std::max(ls, -kLogScaleClamp), kLogScaleClamp);
    scaling[i] = std::exp(ls);
  }
  // the matching as a permutation: matched rows keep their column, unmatched
  // rows take the free columns in increasing order
  std::vector<char> used(n, 0);
  for (int64_t i = 0; i < n; ++i)
    if (M.row_match[i] != kNone) used[M.row_match[i]] = 1;
  int64_t free_col = 0;
  for (int64_t i = 0; i < n; ++i) {
    if (M.row_match[i] != kNone) { matching[i] = M.row_match[i]; continue; }
    while (used[free_col]) ++free_col;
    matching[i] = free_col;
    used[free_col] = 1;
  }
  if (matched) *matched = cnt;
  return RVG_OK;
}
