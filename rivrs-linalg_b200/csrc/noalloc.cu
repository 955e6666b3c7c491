// Dense APTP factorization of one front with no device allocation.
//
// Some callers cannot allocate device memory while they run: code that runs
// inside another runtime's memory budget (a solver embedded in a simulation
// or an optimizer that owns the whole device and forbids allocation after
// start-up), callers in the middle of stream-ordered work that an allocation
// would synchronise or fragment, and hosts that must not call cudaMalloc at
// all (real-time loops, callbacks).  For them this file offers one entry
// point, rvg_dense_factor_noalloc, which runs the same front kernels as the
// sparse factorization (k_aptp, k_tpp of numeric.cu) with their scratch
// memory taken from a fixed, file-scope device array instead of an
// allocation.  The caller passes the matrix and every output buffer.
//
// Limits and sharing:
//   * front order m <= RVG_NOALLOC_MAX_ORDER (4096) and outer block size
//     <= RVG_NOALLOC_MAX_NB (4096): the array holds 16 + 64*4096 + 4096
//     doubles (about 2.1 MB), resident on every GPU that loads the library;
//   * the array is shared by all calls on a device and keeps the last call's
//     contents; nothing in it has to start at zero (every word is written
//     before it is read), but two calls that overlap on the GPU (different
//     streams, no ordering between them) race on it;
//   * the first call on a device looks up the array's device address
//     (cudaGetSymbolAddress); make that first call before any stream capture.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <string>

#include "../../include/rivrs_b200.h"
#include "front.cuh"

namespace rvg {

void set_error(const std::string& s);

constexpr int64_t NOALLOC_HDR = 16;  // doubles: the front descriptor and its id
constexpr int64_t NOALLOC_DOUBLES = NOALLOC_HDR + 64 * RVG_NOALLOC_MAX_ORDER + RVG_NOALLOC_MAX_NB;
static_assert(sizeof(DFront) + sizeof(int32_t) <= NOALLOC_HDR * sizeof(double), "descriptor does not fit");

// scratch of the allocation-free entry point: descriptor, TRSM backup
// (m x 32), W = L*D (m x 32), outer-block column order (nb)
static __device__ __align__(256) double g_noalloc_scratch[NOALLOC_DOUBLES];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_mu;
double* g_ptr[kMaxDevices] = {};

// The array's device address on the current device (host code may not use
// the symbol itself: in host code it names a host-side stand-in).
int scratch_address(double** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    set_error(std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    return RVG_ERR_DEVICE;
  }
  if (dev < 0 || dev >= kMaxDevices) {
    set_error("device ordinal beyond the supported range");
    return RVG_ERR_DEVICE;
  }
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_ptr[dev]) {
    double* p = nullptr;
    e = cudaGetSymbolAddress((void**)&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      set_error(std::string("cudaGetSymbolAddress of the no-allocation scratch: ") + cudaGetErrorString(e));
      return RVG_ERR_DEVICE;
    }
    g_ptr[dev] = p;
  }
  *out = g_ptr[dev];
  return RVG_OK;
}

// descriptor of the single front, its id, and the identity pivot order
__global__ void k_noalloc_setup(double* scratch, int64_t m, int64_t p, int32_t* perm) {
  DFront* F = reinterpret_cast<DFront*>(scratch);
  int32_t* ids = reinterpret_cast<int32_t*>(F + 1);
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    DFront f{};
    f.panel = 0;
    f.idx = -m;  // the kernels read the pivot order at idx + m: the caller's buffer
    f.dpos = 0;
    f.scratch = NOALLOC_HDR;
    f.cb = -1;
    f.m = (int32_t)m;
    f.k = (int32_t)p;
    f.nown = (int32_t)p;
    f.ndin = 0;
    f.nfs = (int32_t)(m - p);
    f.parent = -1;
    f.flags = 0;
    *F = f;
    ids[0] = 0;
  }
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < p; i += (int64_t)gridDim.x * blockDim.x)
    perm[i] = (int32_t)i;
}

__global__ void k_noalloc_counts(const double* scratch, int32_t* counts) {
  const DFront* F = reinterpret_cast<const DFront*>(scratch);
  if (threadIdx.x == 0) { counts[0] = F->ne; counts[1] = F->n1; counts[2] = F->n2; }
}

}  // namespace
}  // namespace rvg

using namespace rvg;

extern "C" rvg_status rvg_dense_factor_noalloc(double* d_a, int64_t m, int64_t p, const rvg_options* opt,
                                               int32_t* d_perm, int8_t* d_dtype, double* d_ddiag, double* d_doff,
                                               int32_t* d_counts, void* stream) {
  rvg_options o;
  rvg_default_options(&o);
  if (opt) o = *opt;
  if (m < 0 || p < 0 || p > m) { set_error("need 0 <= p <= m"); return RVG_ERR_INVALID_INPUT; }
  if (m > RVG_NOALLOC_MAX_ORDER) {
    set_error("front order " + std::to_string(m) + " exceeds the no-allocation limit of " +
              std::to_string(RVG_NOALLOC_MAX_ORDER));
    return RVG_ERR_INVALID_INPUT;
  }
  if (!(o.threshold > 0.0 && o.threshold <= 1.0)) { set_error("threshold must be in (0, 1]"); return RVG_ERR_INVALID_INPUT; }
  if (!(o.small >= 0.0)) { set_error("small must be >= 0.0"); return RVG_ERR_INVALID_INPUT; }
  if (o.inner_block_size <= 0 || o.inner_block_size > 32 || o.outer_block_size < o.inner_block_size) {
    set_error("need 0 < inner_block_size <= 32 and inner_block_size <= outer_block_size");
    return RVG_ERR_INVALID_INPUT;
  }
  if (o.outer_block_size > RVG_NOALLOC_MAX_NB) {
    set_error("outer_block_size exceeds the no-allocation limit of " + std::to_string(RVG_NOALLOC_MAX_NB));
    return RVG_ERR_INVALID_INPUT;
  }
  if (m == 0 || p == 0) {
    if (d_counts && cudaMemsetAsync(d_counts, 0, 3 * sizeof(int32_t), (cudaStream_t)stream) != cudaSuccess) {
      set_error("cudaMemsetAsync of the counts failed");
      return RVG_ERR_DEVICE;
    }
    return RVG_OK;
  }
  if (!d_a || !d_perm || !d_dtype || !d_ddiag || !d_doff || !d_counts) {
    set_error("null buffer");
    return RVG_ERR_INVALID_INPUT;
  }
  double* scratch = nullptr;
  int rc = scratch_address(&scratch);
  if (rc) return (rvg_status)rc;
  cudaStream_t st = (cudaStream_t)stream;
  DevOpts dop{o.threshold, o.small, (int)o.outer_block_size, (int)o.inner_block_size, o.failed_pivot_tpp};
  DFront* F = reinterpret_cast<DFront*>(scratch);
  const int32_t* ids = reinterpret_cast<const int32_t*>(F + 1);
  Arenas A{d_a, d_perm, d_dtype, d_ddiag, d_doff, scratch, nullptr};
  k_noalloc_setup<<<(unsigned)((p + 255) / 256), 256, 0, st>>>(scratch, m, p, d_perm);
  if (p < o.inner_block_size) k_tpp<<<1, 32, 0, st>>>(ids, 1, F, A, dop);
  else k_aptp<<<1, APTP_THREADS, 0, st>>>(ids, 1, F, A, dop);
  k_noalloc_counts<<<1, 32, 0, st>>>(scratch, d_counts);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error(std::string("CUDA error: ") + cudaGetErrorString(e));
    return RVG_ERR_DEVICE;
  }
  return RVG_OK;
}
