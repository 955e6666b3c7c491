/* rivrs_b200.h — C ABI of the B200 numeric phase for sparse symmetric
 * indefinite LDL^T with a-posteriori threshold pivoting (APTP).
 *
 * The entry points replace the numeric half of rivrs-sparse behind its
 * analyze -> factor -> solve API.  Each declaration cites the reference
 * interface it stands in for (paths inside the rivrs-linalg project).
 *
 * Conventions
 *   - Indices are int64_t (the reference's usize), matrices are FULL symmetric
 *     CSC (both triangles stored, sparse/src/lib.rs:121-125).
 *   - Permutations are "forward": perm_fwd[new] = old.
 *   - Every call returns an rvg_status; rvg_last_error() gives the message of
 *     the last failing call on the calling thread.
 *   - A handle is single-threaded and owns one CUDA stream on the current
 *     device.  There is no CPU fallback: without a usable GPU the calls that
 *     need one return RVG_ERR_DEVICE.
 */
#ifndef RIVRS_B200_H
#define RIVRS_B200_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes, one per SparseError variant that the numeric path can raise
 * (sparse/src/error.rs:20-100) plus the device-side failures. */
typedef enum {
  RVG_OK = 0,
  RVG_ERR_DIMENSION_MISMATCH = 1, /* SparseError::DimensionMismatch */
  RVG_ERR_INVALID_INPUT = 2,      /* SparseError::InvalidInput / NotSquare */
  RVG_ERR_SOLVE_BEFORE_FACTOR = 3,/* SparseError::SolveBeforeFactor */
  RVG_ERR_ANALYSIS = 4,           /* SparseError::AnalysisFailure */
  RVG_ERR_DEVICE = 5,             /* CUDA error or no device */
  RVG_ERR_DEVICE_TIMEOUT = 6,     /* a bounded device-side wait gave up */
  RVG_ERR_OUT_OF_MEMORY = 7
} rvg_status;

/* FactorOptions / AptpOptions (sparse/src/symmetric/solver.rs:72-116,
 * sparse/src/symmetric/factor.rs:86-130).  rvg_default_options() fills the
 * reference defaults: threshold 0.01, small 1e-20, nb 256, ib 32, nemin 32,
 * small_leaf_threshold 256, failed_pivot_method Tpp (and
 * large_front_threshold 2048). */
typedef struct {
  double threshold;
  double small;
  int64_t outer_block_size;
  int64_t inner_block_size;
  int64_t nemin;
  int64_t small_leaf_threshold;
  int32_t failed_pivot_tpp; /* 1 = FailedPivotMethod::Tpp, 0 = Pass */
  int32_t fallback_bk;      /* 1 = AptpFallback::BunchKaufman, 0 = Delay */
  /* B200 scheduling, no reference counterpart: fronts of order >= this use
   * the multi-kernel path (whole GPU per front), and so do fronts of at least
   * half this order in a wave that holds at most 16 of them; the others are
   * batched one CTA or warp per front.  Results do not depend on it.
   * Default 2048. */
  int64_t large_front_threshold;
  /* Arithmetic of the large Schur-complement updates, no reference
   * counterpart: 0 = plain FP64 (tensor-core DMMA, bit-identical to the CPU
   * restatement), 1 = mixed: the updates on the TF32 tensor cores (tcgen05)
   * with each FP64 operand split once into two TF32 parts (three products per
   * term, FP32-level products), FP32 partial sums added into FP64; pivot
   * tests, 2x2 inversions, TRSM and storage stay FP64.  Pair the mixed form
   * with rvg_solve_refine.  2 = learned: each large front takes the mixed
   * form or plain FP64 as the per-front selector (rvg_set_selector) predicts
   * from the features of the assembled front; a mixed front whose pivots grow
   * past the selector's bound is assembled again and factored in FP64 at the
   * end of its wave, before any parent reads it (rvg_selector_stats). */
  int32_t precision;
  /* Mixed form only: 32-deep K chunks per FP32 partial sum before it is
   * added in FP64 (1, 2, 4 or 8; 0 = one partial sum over the whole K range).
   * Smaller is more accurate (the tensor cores accumulate FP32 with
   * truncation) and slower.  Default 4. */
  int32_t mixed_flush;
  /* Mixed form with mixed_flush = 0 only: output columns per CTA tile of the
   * tensor-core Schur GEMM, 128 or 256 (two 128-column tiles sharing one
   * W tile in shared memory: a quarter fewer operand bytes per flop).  Results
   * do not depend on it.  Default 256. */
  int32_t mixed_tile_cols;
  /* Mixed form: the parts each FP64 operand is split into, 0 = two TF32 parts
   * (kind::tf32, about 22 significant bits per product), 1 = two BF16 parts
   * (kind::f16, about 16 bits: half the operand bytes and twice the tensor
   * rate, so more refinement steps).  Default 0. */
  int32_t mixed_operands;
  /* Refactorization as one CUDA graph launch, no reference counterpart
   * (the reference's refactor, solver.rs:335-341, reruns the numeric phase).
   * 1 = a factorization of the same handle after a dynamic one captures the
   * whole numeric phase, with the host decisions (front sizes, eliminated
   * counts, large fronts' progress per outer block) taken from the dynamic
   * one, into a CUDA graph, and later factorizations launch that graph.  Checks
   * on the device compare the pivoting the new values give with the recorded
   * one; when they differ (other delays or 2x2 pivots) the factorization is
   * redone dynamically, which records anew.  Results are the dynamic path's,
   * bit for bit.  2 = the same, and the factorization's arenas are kept at
   * fixed virtual addresses (the driver's virtual-memory calls): rvg_trim
   * gives their memory back without dropping the graph, so handles that take
   * turns on one device each keep replaying theirs.  Default 0. */
  int32_t graph_refactor;
  /* Mixed form, large fronts: multiprocessors a full window's far-field
   * update leaves to the next outer blocks while it runs on a second stream
   * (no reference counterpart; scheduling only, results do not depend on
   * it).  0 = no split (the whole window update before the next block),
   * -1 = the default (24). */
  int32_t far_field_sms;
  /* Mixed form, large fronts: outer blocks per window of deferred Schur
   * updates (no reference counterpart), 1 to 8; 0 = the default, 4.  A deeper
   * window reads and writes each trailing entry fewer times (faster where the
   * update is bound by that traffic) but sums longer runs of products in
   * FP32 before they reach FP64, so the mixed factor is less accurate; the
   * autotuner (autotune.py) takes 8 only where a full factor + solve is faster
   * and the inertia is unchanged. */
  int32_t mixed_window;
} rvg_options;

/* FactorizationStats (sparse/src/symmetric/numeric.rs:661-719). */
typedef struct {
  int64_t total_1x1_pivots;
  int64_t total_2x2_pivots;
  int64_t total_delayed;
  int64_t zero_pivots;
  int64_t max_front_size;
  int64_t supernodes_before_amalgamation;
  int64_t supernodes_after_amalgamation;
  int64_t merges_performed;
  int64_t small_leaf_subtrees;
  int64_t small_leaf_nodes;
} rvg_stats;

typedef struct rvg_symbolic rvg_symbolic;
typedef struct rvg_handle rvg_handle;

void rvg_default_options(rvg_options* opt);
const char* rvg_last_error(void);

/* ---- host symbolic analysis -------------------------------------------
 * Stand-in for AptpSymbolic::analyze(matrix, SymmetricOrdering::Custom(perm))
 * (sparse/src/symmetric/symbolic.rs:248-310): elimination tree, postorder,
 * column counts and the supernode partition of P A P^T.  `order` is the
 * fill-reducing order (order[new] = old, UserSupplied semantics of
 * solver.rs:51-52) or NULL for the identity; the returned permutation
 * composes it with the elimination-tree postorder. */
rvg_status rvg_analyze(int64_t n, const int64_t* colptr, const int64_t* rowidx, const int64_t* order,
                       rvg_symbolic** out);
/* Sizes: [n, n_supernodes, total pattern length, predicted nnz(L)]. */
rvg_status rvg_symbolic_sizes(const rvg_symbolic* s, int64_t out4[4]);
/* Copies out perm_fwd (n), supernode_begin/end/parent (nsup), pattern_ptr
 * (nsup+1) and pattern_idx (total pattern length); mirrors symbolic.perm_vecs()
 * (symbolic.rs:420-440) and the SymbolicSupernodalCholesky accessors. */
rvg_status rvg_symbolic_export(const rvg_symbolic* s, int64_t* perm_fwd, int64_t* sup_begin,
                               int64_t* sup_end, int64_t* sup_parent, int64_t* pat_ptr, int64_t* pat_idx);
void rvg_symbolic_free(rvg_symbolic* s);

/* ---- numeric phase -----------------------------------------------------
 * rvg_create replaces the pattern-only work at the start of
 * AptpNumeric::factor (numeric.rs:844-905: build_supernode_info, amalgamate,
 * classify_small_leaf_subtrees, build_assembly_maps) and uploads the
 * structure to the device once.  The supernode arrays are the
 * PRE-amalgamation partition (as AptpSymbolic exposes it).  `opt` may be
 * NULL for the defaults. */
rvg_status rvg_create(int64_t n, int64_t nsup, const int64_t* sup_begin, const int64_t* sup_end,
                      const int64_t* pat_ptr, const int64_t* pat_idx, const int64_t* sup_parent,
                      const int64_t* perm_fwd, const int64_t* colptr, const int64_t* rowidx,
                      const rvg_options* opt, rvg_handle** out);

/* AptpNumeric::factor (numeric.rs:844-1023) / SparseLDLT::factor and
 * ::refactor (solver.rs:296-341).  `values` are the CSC values (host memory),
 * `scaling` the MC64 scaling in elimination order (solver.rs:276-280) or
 * NULL.  Replaces any previous factorization held by the handle. */
rvg_status rvg_factor(rvg_handle* h, const double* values, const double* scaling);
/* Same with values and scaling already in device memory (nnz and n doubles). */
rvg_status rvg_factor_device(rvg_handle* h, const double* d_values, const double* d_scaling);

/* SparseLDLT::solve_in_place (solver.rs:370-428): permute, scale,
 * aptp_solve (solve.rs:57-144), scale, unpermute, in place, for nrhs
 * right-hand sides stored column-major with leading dimension ldb (host). */
rvg_status rvg_solve(rvg_handle* h, double* rhs, int64_t nrhs, int64_t ldb);
/* Same on device memory. */
rvg_status rvg_solve_device(rvg_handle* h, double* d_rhs, int64_t nrhs, int64_t ldb);

/* Solve with iterative refinement in FP64 (no reference counterpart; the
 * mixed form's way back to full accuracy): x = solve(b), then while the
 * scaled backward error ||Ax-b|| / (||A||_F ||x|| + ||b||)
 * (sparse/src/validate.rs:209-258) is above `tol`, r = b - A x in FP64 and
 * x += solve(r), at most `max_iter` corrections.  One right-hand side; `rhs`
 * and `x` are host (rvg_solve_refine) or device (_device) vectors of length
 * n.  Reports the corrections made and the final backward error. */
rvg_status rvg_solve_refine(rvg_handle* h, const double* rhs, double* x, double tol, int32_t max_iter,
                            int32_t* iters, double* bwd_err);
rvg_status rvg_solve_refine_device(rvg_handle* h, const double* d_rhs, double* d_x, double tol, int32_t max_iter,
                                   int32_t* iters, double* bwd_err);
/* The same for nrhs right-hand sides (columns at stride ldb >= n), host
 * (rvg_solve_refine_nrhs) or device (_device) arrays: every solve is blocked
 * over the columns, corrections continue until every column's scaled
 * backward error is <= tol; bwd_err receives nrhs values, *iters the
 * corrections made (the same for all columns). */
/* GMRES-IR (no reference counterpart; the mixed form's way back to full
 * accuracy where plain refinement stalls, e.g. BF16 operand parts on an
 * ill-conditioned matrix): restarted flexible GMRES in FP64 on A x = b with
 * the factor as right preconditioner, `restart` basis vectors (1..200), until
 * the scaled backward error (as rvg_solve_refine) is <= tol or after
 * `max_iter` preconditioned products (one solve each, reported in *iters). */
rvg_status rvg_solve_gmres(rvg_handle* h, const double* rhs, double* x, double tol, int32_t max_iter,
                           int32_t restart, int32_t* iters, double* bwd_err);
rvg_status rvg_solve_gmres_device(rvg_handle* h, const double* d_rhs, double* d_x, double tol, int32_t max_iter,
                                  int32_t restart, int32_t* iters, double* bwd_err);
/* Refinement that escalates (no reference counterpart): FP64 iterative
 * refinement while every correction at least halves the backward error, then
 * GMRES-IR (restart 30) from the refined x until tol or max_iter solves after
 * the first.  *method = 0 if refinement alone reached the result, 1 if it
 * escalated to GMRES-IR. */
rvg_status rvg_solve_auto(rvg_handle* h, const double* rhs, double* x, double tol, int32_t max_iter, int32_t* iters,
                          double* bwd_err, int32_t* method);
rvg_status rvg_solve_auto_device(rvg_handle* h, const double* d_rhs, double* d_x, double tol, int32_t max_iter,
                                 int32_t* iters, double* bwd_err, int32_t* method);
rvg_status rvg_solve_refine_nrhs(rvg_handle* h, const double* rhs, double* x, int64_t nrhs, int64_t ldb, double tol,
                                 int32_t max_iter, int32_t* iters, double* bwd_err);
rvg_status rvg_solve_refine_nrhs_device(rvg_handle* h, const double* d_rhs, double* d_x, int64_t nrhs, int64_t ldb,
                                        double tol, int32_t max_iter, int32_t* iters, double* bwd_err);

/* SparseLDLT::inertia (solver.rs:504-519): [positive, negative, zero]. */
rvg_status rvg_inertia(rvg_handle* h, int64_t out3[3]);
/* SparseLDLT::stats (solver.rs:530-532). */
rvg_status rvg_get_stats(rvg_handle* h, rvg_stats* out);

/* Pivot record, fronts in supernode (postorder) order, the eliminated columns
 * of each front in elimination order (FrontFactors::col_indices, numeric.rs:
 * 543-596): global permuted column, code (1 = 1x1, 2 = first of a 2x2,
 * 3 = second of a 2x2) and the D entries (diag, and the off-diagonal on the
 * first column of a 2x2).  Returns the count through *count. */
rvg_status rvg_pivot_record(rvg_handle* h, int64_t* col, int8_t* code, double* d_diag, double* d_off,
                            int64_t* count);
/* Per supernode (post-amalgamation): m, k, ne, n1x1, n2x2, parent, n_owned,
 * in_small_leaf, wave (PerSupernodeStats, numeric.rs:604-655). */
rvg_status rvg_front_info(rvg_handle* h, int64_t* out9, int64_t* nsup);
/* Algorithmic work of the delay-free structure: [factor flops, Schur GEMM
 * flops, assembly bytes, solve bytes per RHS, nnz(L), max front]. */
rvg_status rvg_work(rvg_handle* h, double out6[6]);
/* Device time of the last factor / solve phases in milliseconds:
 * [assembly, dense kernel, contribution GEMM, total factor, last solve,
 *  dominant-kernel time, dominant-kernel launches]. */
rvg_status rvg_timings(rvg_handle* h, double out7[7]);
/* Measurement counters of the last factor and solve.  With profiling on,
 * every launch of the FP64 Schur-complement GEMM is bracketed by CUDA events
 * on the handle's stream, so syrk_ms is its device time; flops count the
 * executed work of those launches (2 per multiply-add, lower triangle only). */
typedef struct {
  double factor_ms, solve_ms;
  double assembly_ms, dense_ms, cbgemm_ms;
  double syrk_ms, syrk_flops;
  int64_t syrk_launches;
  int64_t factor_launches, solve_launches;
  int64_t peak_bytes;
  /* host wall time of the last factor: total, in allocation calls, waiting
   * at wave boundaries and after a large-front block issued past a delay */
  double host_total_ms, host_alloc_ms, host_sync_ms;
  /* device time of the last factor by kind of work (CUDA events between
   * consecutive launches, profiling mode only), indexed by rvg_part */
  double part_ms[16];
  /* large fronts issue their 256-column outer blocks ahead, on the guess
   * that no column is delayed: host time spent waiting for the first of
   * several queued blocks (the device stays busy with the rest), and the
   * blocks issued past a delay (they return at once and are issued again) */
  double host_wait_ms;
  int64_t lf_misses;
  /* host time from a wave's synchronisation (the eliminated counts size the
   * next wave's fronts) to the next wave's first launch: the device has
   * nothing of this factorization queued meanwhile */
  double host_gap_ms;
  /* full-window updates of a large front whose far field (the columns after
   * the next three outer blocks) ran on a second stream beside those blocks */
  int64_t lf_far_updates;
} rvg_profile;

/* Indices of rvg_profile.part_ms.  Large fronts (whole GPU per front): */
enum {
  RVG_PART_LF_SETUP = 0,   /* per-front and per-outer-block bookkeeping */
  RVG_PART_LF_BLOCK = 1,   /* 32x32 diagonal block, complete pivoting */
  RVG_PART_LF_PANEL = 2,   /* TRSM + D^-1 of the rows below, threshold test */
  RVG_PART_LF_POST = 3,    /* (unused: the first failing column is handled inside LF_UPDATE) */
  RVG_PART_LF_UPDATE = 4,  /* rank-32 update inside the outer block */
  RVG_PART_LF_DELAY = 5,   /* delayed columns to the end */
  RVG_PART_LF_PROP = 6,    /* row order propagated to earlier columns */
  RVG_PART_LF_W = 7,       /* W = L D of the outer block */
  RVG_PART_LF_SYRK = 8,    /* deferred trailing Schur update */
  RVG_PART_LF_OUTER = 9,   /* end of outer block */
  /* batched fronts and contribution blocks: */
  RVG_PART_TPP = 10,       /* warp-per-front TPP fronts */
  RVG_PART_APTP = 11,      /* CTA-per-front APTP fronts */
  RVG_PART_CB_W = 12,      /* W = L21 D of contribution blocks */
  RVG_PART_CB_GEMM = 13,   /* small contribution GEMMs (batched) */
  RVG_PART_CB_SYRK = 14,   /* large contribution GEMMs */
  RVG_PART_OTHER = 15,
  RVG_PARTS = 16
};
rvg_status rvg_set_profiling(rvg_handle* h, int32_t enable);
rvg_status rvg_get_profile(rvg_handle* h, rvg_profile* out);

/* MC64 maximum-product matching and symmetric scaling (mc64_matching,
 * sparse/src/ordering/matching.rs:121-248; Duff & Koster 2001, Duff & Pralet
 * 2005), host code.  Input: a square symmetric matrix in CSC (either triangle
 * or both; explicit zeros ignored), n > 0, finite values.  Output:
 * matching[i] = column matched to row i (a permutation; unmatched rows take
 * the free columns in increasing order), scaling[i] > 0 with
 * |scaling[i] a_ij scaling[j]| <= 1 on every entry touching a matched index
 * and a scaled entry of 1 in every nonzero matched row, *matched = number of
 * matched rows (< n: structurally singular).  RVG_ERR_INVALID_INPUT for n == 0
 * or non-finite entries (SparseError::InvalidInput). */
rvg_status rvg_mc64(int64_t n, const int64_t* colptr, const int64_t* rowidx, const double* values,
                    int64_t* matching, double* scaling, int64_t* matched);

/* Self-test of the bounded device waits (no reference counterpart): runs one
 * wait that nothing releases, on the handle's stream, and returns the status
 * the host then reads: RVG_ERR_DEVICE_TIMEOUT when the wait ran out and was
 * reported (the handle stays usable).  which = 0: a solve block's flag wait
 * (1 s); which = 1: the mixed-form GEMM's pipeline wait (2 s). */
rvg_status rvg_selftest_waits(rvg_handle* h, int32_t which);
/* Device memory release (no reference counterpart; the Rust numeric object
 * is dropped whole, solver.rs:312-315).  what: bit 0 = the workspace of
 * factor and solve (contribution and scratch arenas, packed operands, solve
 * vectors), bit 1 = the factor itself (the handle is then unfactored:
 * RVG_ERR_SOLVE_BEFORE_FACTOR until the next rvg_factor).  The analysis, the
 * assembly maps and the other pattern data stay on the device; the next
 * rvg_factor allocates the arenas again at their delay-free size.  Lets many
 * handles take turns on one device. */
rvg_status rvg_trim(rvg_handle* h, int32_t what);
/* Free and total bytes of the current device (cudaMemGetInfo). */
rvg_status rvg_mem_info(int64_t out2[2]);

/* ---- learned per-front precision (no reference counterpart) ------------
 * The selector is a 12-64-64-1 perceptron (ReLU, sigmoid output) on float32
 * parameters: W1 (64 x 12, row major), b1, W2 (64 x 64), b2, W3 (64), b3
 * (rvg_mlp_trained_count() values), then the per-feature mean and standard
 * deviation the inputs are normalised with (rvg_mlp_param_count() in all).
 * Its output is the probability that a front's tensor-core Schur updates keep
 * its pivots within bound. */
#define RVG_MLP_FEATURES 12
#define RVG_FRONT_FEATURE_COLS 22
int64_t rvg_mlp_param_count(void);
int64_t rvg_mlp_trained_count(void);
/* Floats of the work buffer rvg_mlp_grad needs for n samples. */
int64_t rvg_mlp_work_floats(int64_t n);
/* Probabilities of n samples (features n x 12, row major); device pointers,
 * enqueued on `stream` (a cudaStream_t or NULL). */
rvg_status rvg_mlp_forward(const float* d_params, const float* d_x, int64_t n, float* d_prob, void* stream);
/* Loss sum_i w_i (softplus(z_i) - y_i z_i) / norm and its gradient with
 * respect to the trained parameters (d_grad: rvg_mlp_trained_count() floats,
 * d_loss: one float, may be NULL); d_weight may be NULL (all 1).  The result
 * is deterministic (fixed summation order).  Allocates nothing: d_work holds
 * rvg_mlp_work_floats(n) floats. */
rvg_status rvg_mlp_grad(const float* d_params, const float* d_x, const float* d_y, const float* d_weight, int64_t n,
                        double norm, float* d_grad, float* d_loss, float* d_work, int64_t work_floats, void* stream);
/* One Adam step (t = step >= 1) with decoupled weight decay on the trained
 * parameters; d_m and d_v are the moment estimates (same length, start 0). */
rvg_status rvg_mlp_adam(float* d_params, const float* d_grad, float* d_m, float* d_v, int64_t step, float lr,
                        float beta1, float beta2, float eps, float weight_decay, void* stream);
/* Installs a selector on a handle (host parameters, copied): fronts whose
 * probability is >= threshold take the mixed form; a mixed front whose
 * largest |D| entry exceeds growth_bound times its largest assembled |a|
 * is refactored in FP64 (that front alone). */
rvg_status rvg_set_selector(rvg_handle* h, const float* params, int64_t nparams, float threshold,
                            double growth_bound);
/* The large fronts of the last learned-precision factorization, one row of
 * RVG_FRONT_FEATURE_COLS doubles each: supernode, m, k, eliminated, 1x1 and
 * 2x2 pivots, route (1 = mixed), probability, max |a| of the assembled
 * fully-summed columns, max |D|, then the 12 features: log2 m, log2 k, k/m,
 * log2(1 + delayed rows in), delayed rows in / k, log10 max |a|, log10 of
 * max |a_jj| / max |a|, log10 of min |a_jj| / max |a|, log10 of the smallest
 * column ratio |a_jj| / max_{i>j} |a_ij|, the fractions of columns with that
 * ratio below the pivot threshold, with a negative and with a zero diagonal.
 * out == NULL: *nrows only. */
rvg_status rvg_front_features(rvg_handle* h, double* out, int64_t cap_rows, int64_t* nrows);
/* [large fronts, fronts the selector sent to the mixed form, mixed fronts
 * over the growth bound, fronts factored again in FP64 at the end of their
 * wave because they were over it]. */
rvg_status rvg_selector_stats(rvg_handle* h, int64_t out4[4]);
/* The CUDA stream the handle launches on (cudaStream_t as void*). */
rvg_status rvg_stream(rvg_handle* h, void** stream);
void rvg_destroy(rvg_handle* h);

/* ---- allocation-free dense front factorization -------------------------
 * No counterpart in the reference: an extra entry point for callers that
 * cannot allocate device memory while they run -- a solver embedded in a
 * host application that owns the device's memory budget and forbids
 * allocation after start-up, code inside stream-ordered work that an
 * allocation would synchronise or fragment, real-time loops and callbacks.
 * It factors one dense symmetric front in place with the same kernels and
 * the same pivoting as rvg_factor uses for a front: d_a is m x m
 * column-major (lower triangle read, the first p columns factored, the
 * factored columns' rows below p updated as well),
 * d_perm receives the pivot order (p), d_dtype / d_ddiag / d_doff the D
 * entries (p; codes as in rvg_pivot_record), d_counts [ne, n1x1, n2x2].
 * All buffers are the caller's device memory; the call allocates nothing.
 * Its scratch is one fixed device array inside the library (about 2.1 MB per
 * GPU, held until exit), which limits m to RVG_NOALLOC_MAX_ORDER and the outer
 * block size to RVG_NOALLOC_MAX_NB; larger sizes return RVG_ERR_INVALID_INPUT.
 * Every call on a device shares that array: calls that overlap on the GPU
 * (different streams without ordering) race.  The first call on a device
 * looks up the array's address; make it before any stream capture.  Work is
 * enqueued on `stream` (a cudaStream_t, NULL for the default stream); the
 * call does not synchronise.  `opt` may be NULL for the defaults. */
#define RVG_NOALLOC_MAX_ORDER 4096
#define RVG_NOALLOC_MAX_NB 4096
rvg_status rvg_dense_factor_noalloc(double* d_a, int64_t m, int64_t p, const rvg_options* opt, int32_t* d_perm,
                                    int8_t* d_dtype, double* d_ddiag, double* d_doff, int32_t* d_counts,
                                    void* stream);

#ifdef __cplusplus
}
#endif
#endif
