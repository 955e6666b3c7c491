// Host analysis for CPU-only runs (test infrastructure: the bench's CPU arms
// and tests).  oracle/build.py links this file with the library's own host
// analysis sources -- symbolic analysis (rivrs-linalg_b200/csrc/symbolic.cpp,
// capi.cpp) and MC64 matching and scaling (mc64.cpp) -- into
// oracle/_build/libanalysis.so, without the CUDA numeric phase, so a process
// that times the CPU restatement analyses its input exactly as the GPU path
// does and loads no GPU library.  This file supplies the error channel those
// sources report through (in the full library it lives beside the CUDA driver).
#include <string>

namespace rvg {
thread_local std::string g_analysis_err;
void set_error(const std::string& s) { g_analysis_err = s; }
}  // namespace rvg

extern "C" const char* rvg_last_error(void) { return rvg::g_analysis_err.c_str(); }
