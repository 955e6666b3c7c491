// Internal declarations shared by the host planner, the CUDA driver and the
// C ABI.  Nothing here crosses the library boundary.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/rivrs_b200.h"

namespace rvg {

// Host symbolic result (the AptpSymbolic stand-in).
struct Symbolic {
  int64_t n = 0;
  std::vector<int64_t> perm_fwd, perm_inv;  // perm_fwd[new] = old
  std::vector<int64_t> etree, colcount;     // permuted numbering
  std::vector<int64_t> sup_begin, sup_end, sup_parent;
  std::vector<int64_t> pat_ptr, pat_idx;
};

int symbolic_analyze(int64_t n, const int64_t* colptr, const int64_t* rowidx, const int64_t* order,
                     Symbolic& S, std::string* err);

// Post-amalgamation supernode (numeric.rs:431-448 SupernodeInfo).
struct Snode {
  int64_t col_begin = 0, col_end = 0;
  std::vector<int64_t> pattern;
  int64_t parent = -1;
  std::vector<std::pair<int64_t, int64_t>> owned;
  bool in_small_leaf = false;
  int64_t n_owned() const {
    int64_t s = 0;
    for (auto& r : owned) s += r.second - r.first;
    return s;
  }
};

// The factor plan: everything that depends on the sparsity pattern only.
struct Plan {
  int64_t n = 0;
  int64_t nsup_before = 0, merges = 0;
  int64_t sl_subtrees = 0, sl_nodes = 0;
  std::vector<Snode> sn;
  std::vector<std::vector<int64_t>> children;
  std::vector<int64_t> height;                 // wave index (0 = leaves)
  std::vector<std::vector<int64_t>> waves;     // fronts per wave
  std::vector<int64_t> perm_fwd;               // new -> old
  // assembly maps (numeric.rs:264-408), delay-free local coordinates
  std::vector<int64_t> amap_ptr;               // per supernode
  std::vector<int32_t> amap;                   // 5 x int32 per entry: src, row, col, srow, scol
  std::vector<int64_t> ea_ptr;                 // per supernode: child pattern -> parent local
  std::vector<int32_t> ea_map;
  std::vector<int64_t> own_ptr, pat_ptr;       // owned columns / pattern per supernode
  std::vector<int32_t> own_idx, pat_idx;
  // algorithmic work from the delay-free structure
  double flops_factor = 0, flops_schur = 0, bytes_assembly = 0;
  int64_t nnz_l = 0, max_front = 0;
};

void set_error(const std::string& s);

int build_plan(const Symbolic* S, int64_t n, int64_t nsup, const int64_t* sup_begin, const int64_t* sup_end,
               const int64_t* pat_ptr, const int64_t* pat_idx, const int64_t* sup_parent,
               const int64_t* perm_fwd, const int64_t* colptr, const int64_t* rowidx,
               const rvg_options& opt, Plan& P, std::string* err);

}  // namespace rvg
