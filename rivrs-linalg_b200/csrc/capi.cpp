// C ABI of the host symbolic analysis (the AptpSymbolic stand-in).
#include <cstring>
#include <string>

#include "rvg_internal.h"

namespace rvg {
void set_error(const std::string& s);
}

struct rvg_symbolic {
  rvg::Symbolic S;
};

extern "C" {

rvg_status rvg_analyze(int64_t n, const int64_t* colptr, const int64_t* rowidx, const int64_t* order,
                       rvg_symbolic** out) {
  if (!out || (n > 0 && (!colptr || !rowidx))) {
    rvg::set_error("null argument");
    return RVG_ERR_INVALID_INPUT;
  }
  *out = nullptr;
  rvg_symbolic* s = new rvg_symbolic();
  std::string err;
  int rc = rvg::symbolic_analyze(n, colptr, rowidx, order, s->S, &err);
  if (rc) {
    delete s;
    rvg::set_error(err);
    return (rvg_status)rc;
  }
  *out = s;
  return RVG_OK;
}

rvg_status rvg_symbolic_sizes(const rvg_symbolic* s, int64_t out4[4]) {
  if (!s || !out4) { rvg::set_error("null argument"); return RVG_ERR_INVALID_INPUT; }
  out4[0] = s->S.n;
  out4[1] = (int64_t)s->S.sup_begin.size();
  out4[2] = (int64_t)s->S.pat_idx.size();
  int64_t nnz = 0;
  for (int64_t c : s->S.colcount) nnz += c;
  out4[3] = nnz;
  return RVG_OK;
}

rvg_status rvg_symbolic_export(const rvg_symbolic* s, int64_t* perm_fwd, int64_t* sup_begin, int64_t* sup_end,
                               int64_t* sup_parent, int64_t* pat_ptr, int64_t* pat_idx) {
  if (!s) { rvg::set_error("null argument"); return RVG_ERR_INVALID_INPUT; }
  const rvg::Symbolic& S = s->S;
  auto cp = [](int64_t* dst, const std::vector<int64_t>& v) {
    if (dst && !v.empty()) std::memcpy(dst, v.data(), v.size() * sizeof(int64_t));
  };
  cp(perm_fwd, S.perm_fwd);
  cp(sup_begin, S.sup_begin);
  cp(sup_end, S.sup_end);
  cp(sup_parent, S.sup_parent);
  cp(pat_ptr, S.pat_ptr);
  cp(pat_idx, S.pat_idx);
  return RVG_OK;
}

void rvg_symbolic_free(rvg_symbolic* s) { delete s; }

}  // extern "C"
