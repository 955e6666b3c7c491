// Device descriptors of the numeric phase, shared by its translation units.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "dense.cuh"

namespace rvg {

enum : int32_t { FF_SMALL_LEAF = 1, FF_HAS_CB = 2, FF_HAS_PARENT = 4, FF_LARGE = 8 };

struct DFront {
  int64_t panel;    // offset (doubles) in the panel arena, ld = m
  int64_t idx;      // offset (int32) in the index arena: rows[m], perm[k]
  int64_t dpos;     // offset in the D arrays (k entries)
  int64_t scratch;  // offset (doubles) in the wave scratch
  int64_t cb;       // offset (doubles) of the NFS x NFS contribution block (ld nfs) in the CB arena, -1 if none
  int32_t m, k, nown, ndin, nfs;
  int32_t ne, n1, n2;
  int32_t parent;
  int32_t dly_off;  // position of this front's delayed columns among the parent's delayed block
  int32_t flags;
  int32_t pad;
};

struct Statics {
  const int64_t* own_ptr;
  const int32_t* own_idx;
  const int64_t* pat_ptr;
  const int32_t* pat_idx;
  const int64_t* amap_ptr;
  const int32_t* amap;
  const int64_t* ea_ptr;
  const int32_t* ea_map;
  const int64_t* ch_ptr;
  const int32_t* ch_idx;
};

struct Arenas {
  double* panel;
  int32_t* idx;
  int8_t* dtype;
  double* ddiag;
  double* doff;
  double* scratch;
  double* cbase;  // contribution-block arena
};

// dense factorization kernels of numeric.cu (one warp / one CTA per front)
constexpr int APTP_THREADS = 256;
__global__ void k_tpp(const int32_t* ids, int n, DFront* F, Arenas A, DevOpts o);
__global__ void __launch_bounds__(APTP_THREADS) k_aptp(const int32_t* ids, int n, DFront* F, Arenas A, DevOpts o);

}  // namespace rvg
