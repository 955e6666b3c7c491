// Supernodal solve of one large front on the whole GPU (forward_solve_supernode
// and backward_solve_supernode, sparse/src/symmetric/solve.rs:161-326, with
// the diagonal solve of solve.rs:232-252 fused into the forward pass).
//
// The front's factor is its m x k panel: L11 in rows [0, ne), L21 in rows
// [ne, m) of columns [0, ne).  A work vector v of length m holds the
// gathered right-hand side (rows < ne) and the L21 products (rows >= ne).
//   forward : per 64-column block, one warp solves the unit lower diagonal
//             block (lsf_diag), then every row below it takes the block's
//             update (lsf_update, one row per thread, fma chain in column
//             order); finally the L21 part is scattered and D^-1 applied.
//   backward: per 64-column block from the bottom, each column's dot product
//             with the solved rows below the block is split over 8 row
//             ranges (lsb_dot), summed in a fixed order by one warp, which
//             then solves the unit upper (L11^T) diagonal block (lsb_diag).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "dense.cuh"

namespace rvg {

constexpr int LS_B = 64;   // diagonal block width
constexpr int LS_RS = 8;   // row splits of the backward dot products

struct LSArgs {
  const double* L;   // panel, ld m
  int64_t m, k, ne;
  const int32_t* rows;
  const int32_t* perm;
  const int8_t* dt;
  const double* dd;
  const double* dof;
  double* v;         // m
  double* part;      // LS_RS x LS_B partial sums
  double* x;         // solution vector (permuted order), one RHS
};

__device__ __forceinline__ int32_t ls_col(const LSArgs& a, int64_t i) { return a.rows[a.perm[i]]; }
__device__ __forceinline__ int32_t ls_row(const LSArgs& a, int64_t t) {  // t-th row below ne
  int64_t q = a.ne + t;
  return q < a.k ? a.rows[a.perm[q]] : a.rows[q];
}

__global__ void k_lsf_gather(LSArgs a) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < a.ne) a.v[i] = a.x[ls_col(a, i)];
  else if (i < a.m) a.v[i] = 0.0;
}

// one warp: unit lower solve of v[b0, b1) by L[b0..b1, b0..b1)
__global__ void k_lsf_diag(LSArgs a, int64_t b0) {
  const int lane = threadIdx.x;
  const int64_t b1 = b0 + LS_B < a.ne ? b0 + LS_B : a.ne;
  const int64_t r0 = b0 + lane, r1 = b0 + 32 + lane;
  double v0 = r0 < b1 ? a.v[r0] : 0.0, v1 = r1 < b1 ? a.v[r1] : 0.0;
  for (int64_t j = b0; j < b1; ++j) {
    const int src = (int)(j - b0);
    double vj = __shfl_sync(0xffffffffu, src < 32 ? v0 : v1, src & 31);
    if (r0 > j && r0 < b1) v0 = __fma_rn(-a.L[r0 + j * a.m], vj, v0);
    if (r1 > j && r1 < b1) v1 = __fma_rn(-a.L[r1 + j * a.m], vj, v1);
  }
  if (r0 < b1) a.v[r0] = v0;
  if (r1 < b1) a.v[r1] = v1;
}

// rows i >= b1 take the update of the block's columns
__global__ void k_lsf_update(LSArgs a, int64_t b0) {
  const int64_t b1 = b0 + LS_B < a.ne ? b0 + LS_B : a.ne;
  __shared__ double vb[LS_B];
  if (threadIdx.x < b1 - b0) vb[threadIdx.x] = a.v[b0 + threadIdx.x];
  __syncthreads();
  const int64_t i = b1 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.m) return;
  double acc = a.v[i];
  for (int64_t c = b0; c < b1; ++c) acc = __fma_rn(-a.L[i + c * a.m], vb[c - b0], acc);
  a.v[i] = acc;
}

// L21 products to the parent rows; D^-1 on the eliminated columns
__global__ void k_lsf_finish(LSArgs a) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.m) return;
  if (i >= a.ne) {
    atomicAdd(&a.x[ls_row(a, i - a.ne)], a.v[i]);
    return;
  }
  const int32_t g = ls_col(a, i);
  if (a.dt[i] == PT_1X1) {
    const double d = a.dd[i];
    a.x[g] = d == 0.0 ? 0.0 : __ddiv_rn(a.v[i], d);
  } else {
    const int64_t c0 = a.dt[i] == PT_2X2 ? i : i - 1;
    const double A = a.dd[c0], B = a.dof[c0], C = a.dd[c0 + 1];
    const double det = __dsub_rn(__dmul_rn(A, C), __dmul_rn(B, B));
    const double r1 = a.v[c0], r2 = a.v[c0 + 1];
    if (det == 0.0) a.x[g] = 0.0;
    else a.x[g] = (i == c0) ? __ddiv_rn(__dsub_rn(__dmul_rn(C, r1), __dmul_rn(B, r2)), det)
                            : __ddiv_rn(__dsub_rn(__dmul_rn(A, r2), __dmul_rn(B, r1)), det);
  }
}

__global__ void k_lsb_gather(LSArgs a) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < a.ne) a.v[i] = a.x[ls_col(a, i)];
  else if (i < a.m) a.v[i] = a.x[ls_row(a, i - a.ne)];
}

// partial dot products of the block's columns with v over rows (b1, m):
// grid (LS_B columns, LS_RS splits)
__global__ void k_lsb_dot(LSArgs a, int64_t b0) {
  const int64_t b1 = b0 + LS_B < a.ne ? b0 + LS_B : a.ne;
  const int64_t c = b0 + blockIdx.x;
  __shared__ double red[8];
  double s = 0.0;
  if (c < b1) {
    const int64_t len = a.m - b1;
    const int64_t per = (len + LS_RS - 1) / LS_RS;
    const int64_t lo = b1 + (int64_t)blockIdx.y * per;
    const int64_t hi = lo + per < a.m ? lo + per : a.m;
    for (int64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) s = __fma_rn(a.L[i + c * a.m], a.v[i], s);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int q = 0; q < (int)(blockDim.x >> 5); ++q) t += red[q];
    a.part[blockIdx.y * LS_B + blockIdx.x] = t;
  }
}

// one warp: subtract the partial sums, then unit upper solve of the block
__global__ void k_lsb_diag(LSArgs a, int64_t b0) {
  const int lane = threadIdx.x;
  const int64_t b1 = b0 + LS_B < a.ne ? b0 + LS_B : a.ne;
  const int64_t r0 = b0 + lane, r1 = b0 + 32 + lane;
  double v0 = 0.0, v1 = 0.0;
  if (r0 < b1) {
    double t = 0.0;
    for (int q = 0; q < LS_RS; ++q) t += a.part[q * LS_B + lane];
    v0 = a.v[r0] - t;
  }
  if (r1 < b1) {
    double t = 0.0;
    for (int q = 0; q < LS_RS; ++q) t += a.part[q * LS_B + 32 + lane];
    v1 = a.v[r1] - t;
  }
  for (int64_t j = b1 - 1; j >= b0; --j) {
    // v_j -= sum_{i in (j, b1)} L[i, j] v_i
    double p = 0.0;
    if (r0 > j && r0 < b1) p = __fma_rn(a.L[r0 + j * a.m], v0, p);
    if (r1 > j && r1 < b1) p = __fma_rn(a.L[r1 + j * a.m], v1, p);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) p += __shfl_xor_sync(0xffffffffu, p, o);
    if (r0 == j) v0 -= p;
    if (r1 == j) v1 -= p;
  }
  if (r0 < b1) a.v[r0] = v0;
  if (r1 < b1) a.v[r1] = v1;
}

__global__ void k_lsb_scatter(LSArgs a) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < a.ne) a.x[ls_col(a, i)] = a.v[i];
}

}  // namespace rvg
