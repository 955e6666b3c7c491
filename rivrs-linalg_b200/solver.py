"""Host-side mirror of rivrs-sparse's user API for the numeric path
(SparseLDLT, sparse/src/symmetric/solver.rs:178-549): the same three phases,
option names, defaults and error behaviour, with the numeric phase running
on the B200 through the C ABI of include/rivrs_b200.h.

    solver = SparseLDLT.analyze_with_matrix(system, AnalyzeOptions())
    solver.factor(system.values, FactorOptions())
    x = solver.solve(b)
    solver.inertia(), solver.stats()

Differences forced by the environment (no Rust, no METIS): the ordering is a
project-provided permutation (`OrderingStrategy.USER_SUPPLIED` semantics for
every strategy), and MC64 scaling is taken from `scaling=` when given.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import enum

import numpy as np

from . import _native as N
from . import ordering as orderings


class OrderingStrategy(enum.Enum):
    """solver.rs:42-53; METIS is replaced by project orderings (see ordering.py)."""
    AMD = "amd"
    METIS = "metis"
    MATCH_ORDER_METIS = "match_order_metis"
    USER_SUPPLIED = "user_supplied"


@dataclasses.dataclass
class AnalyzeOptions:
    ordering: OrderingStrategy = OrderingStrategy.METIS
    perm: np.ndarray | None = None  # for USER_SUPPLIED: order[new] = old


@dataclasses.dataclass
class FactorOptions:
    """FactorOptions (solver.rs:72-116) with the AptpOptions extras."""
    threshold: float = 0.01
    small: float = 1e-20
    outer_block_size: int = 256
    inner_block_size: int = 32
    nemin: int = 32
    small_leaf_threshold: int = 256
    failed_pivot_tpp: bool = True
    fallback_bunch_kaufman: bool = True
    large_front_threshold: int = 2048  # B200 scheduling only; results do not depend on it
    precision: str = "fp64"  # "fp64" (plain), "mixed" (tensor-core Schur updates; pair with solve_refine/solve_auto)
    # or "learned" (per front, as the selector installed with set_selector predicts)
    mixed_flush: int = 4  # mixed form: 32-deep K chunks per FP32 partial sum (1, 2, 4, 8; 0 = all of K)
    mixed_tile_cols: int = 256  # mixed form, mixed_flush 0: Schur GEMM output columns per CTA tile (128, 256)
    mixed_operands: str = "tf32"  # mixed form: FP64 operands split into two "tf32" or two "bf16" parts
    graph_refactor: int = 0  # 1: refactorizations replayed as one CUDA graph (same pivoting); 2: the same, with
    #                          the arenas kept at their addresses while SparseLDLT.trim gives their memory back
    far_field_sms: int = -1  # mixed form: SMs a window's far-field update leaves to the next blocks (0 = no split)
    mixed_window: int = 0  # mixed form: outer blocks per window of deferred updates, 1-8 (0 = default 4)

    def native(self) -> N.Options:
        return N.default_options(threshold=self.threshold, small=self.small,
                                 outer_block_size=self.outer_block_size, inner_block_size=self.inner_block_size,
                                 nemin=self.nemin, small_leaf_threshold=self.small_leaf_threshold,
                                 failed_pivot_tpp=int(self.failed_pivot_tpp),
                                 fallback_bk=int(self.fallback_bunch_kaufman),
                                 large_front_threshold=self.large_front_threshold,
                                 precision={"fp64": 0, "mixed": 1, "learned": 2}[self.precision],
                                 mixed_flush=self.mixed_flush, mixed_tile_cols=self.mixed_tile_cols,
                                 mixed_operands={"tf32": 0, "bf16": 1}[self.mixed_operands],
                                 graph_refactor=int(self.graph_refactor), far_field_sms=int(self.far_field_sms),
                                 mixed_window=int(self.mixed_window))


class SparseError(RuntimeError):
    """SparseError (sparse/src/error.rs:20-100)."""


class DimensionMismatch(SparseError):
    pass


class InvalidInput(SparseError):
    pass


class SolveBeforeFactor(SparseError):
    pass


class IoError(SparseError):
    """SparseError::IoError (error.rs:64-71): a file that cannot be read."""

    def __init__(self, path, source):
        super().__init__(f"IO error for '{path}': {source}")
        self.path, self.source = path, source


class ParseError(SparseError):
    """SparseError::ParseError (error.rs:72-80): malformed input."""

    def __init__(self, path, reason, line=None):
        where = f"'{path}' at line {line}" if line is not None else f"'{path}'"
        super().__init__(f"Parse error in {where}: {reason}")
        self.path, self.reason, self.line = path, reason, line


_ERRMAP = {1: DimensionMismatch, 2: InvalidInput, 3: SolveBeforeFactor}


def _check(status):
    if status != 0:
        cls = _ERRMAP.get(status, SparseError)
        raise cls(f"{N.STATUS.get(status, status)}: {N.lib().rvg_last_error().decode()}")


@dataclasses.dataclass
class SymbolicStructure:
    """What AptpSymbolic exposes to the numeric phase."""
    n: int
    perm_fwd: np.ndarray
    sup_begin: np.ndarray
    sup_end: np.ndarray
    sup_parent: np.ndarray
    pat_ptr: np.ndarray
    pat_idx: np.ndarray
    predicted_nnz: int


def symbolic_analyze(n, colptr, rowidx, order=None) -> SymbolicStructure:
    """AptpSymbolic::analyze with a custom ordering (symbolic.rs:248-310)."""
    L = N.lib()
    colptr = N.as_i64(colptr)
    rowidx = N.as_i64(rowidx)
    order = None if order is None else N.as_i64(order)
    h = C.c_void_p()
    _check(L.rvg_analyze(n, N.ptr(colptr, N.i64p), N.ptr(rowidx, N.i64p), N.ptr(order, N.i64p), C.byref(h)))
    try:
        sz = np.zeros(4, np.int64)
        _check(L.rvg_symbolic_sizes(h, N.ptr(sz, N.i64p)))
        nn, ns, npat, nnz = (int(x) for x in sz)
        perm = np.zeros(nn, np.int64)
        b = np.zeros(ns, np.int64)
        e = np.zeros(ns, np.int64)
        par = np.zeros(ns, np.int64)
        pp = np.zeros(ns + 1, np.int64)
        pi = np.zeros(max(npat, 1), np.int64)
        _check(L.rvg_symbolic_export(h, N.ptr(perm, N.i64p), N.ptr(b, N.i64p), N.ptr(e, N.i64p),
                                     N.ptr(par, N.i64p), N.ptr(pp, N.i64p), N.ptr(pi, N.i64p)))
    finally:
        L.rvg_symbolic_free(h)
    return SymbolicStructure(nn, perm, b, e, par, pp, pi[:npat], nnz)


class SparseLDLT:
    """Three-phase solver: analyze -> factor -> solve (solver.rs:178-549)."""

    def __init__(self, system, symbolic: SymbolicStructure, scaling_elim: np.ndarray | None):
        self.system = system
        self.symbolic = symbolic
        self._scaling = scaling_elim
        self._handle = None
        self._factored = False
        self._opts = None
        self._selector = None

    # -- analyze -----------------------------------------------------------
    @classmethod
    def analyze(cls, system, options: AnalyzeOptions | None = None):
        options = options or AnalyzeOptions()
        if options.ordering == OrderingStrategy.USER_SUPPLIED:
            if options.perm is None:
                raise InvalidInput("USER_SUPPLIED ordering needs a permutation")
            order = N.as_i64(options.perm)
        else:
            order = orderings.default_order(system)
        sym = symbolic_analyze(system.n, system.colptr, system.rowidx, order)
        return cls(system, sym, None)

    @classmethod
    def analyze_with_matrix(cls, system, options: AnalyzeOptions | None = None, scaling: np.ndarray | None = None):
        """analyze plus scaling in ORIGINAL order, transformed to elimination order
        (solver.rs:261-285).  With MATCH_ORDER_METIS the scaling is MC64's
        (matching.rs:121-248); the fill-reducing order is the project's ordering
        (METIS is not available)."""
        options = options or AnalyzeOptions()
        if scaling is None and options.ordering == OrderingStrategy.MATCH_ORDER_METIS:
            try:
                _, scaling, _ = orderings.mc64(system)
            except N.RvgError as e:
                raise InvalidInput(str(e)) from None
        s = cls.analyze(system, options)
        if scaling is not None:
            s._scaling = N.as_f64(np.asarray(scaling)[s.symbolic.perm_fwd])
        return s

    # -- factor --------------------------------------------------------------
    def _ensure_handle(self, options: FactorOptions):
        if self._handle is not None and self._opts == options:
            return
        self.close()
        sym = self.symbolic
        h = C.c_void_p()
        o = options.native()
        _check(N.lib().rvg_create(sym.n, sym.sup_begin.size, N.ptr(sym.sup_begin, N.i64p), N.ptr(sym.sup_end, N.i64p),
                                  N.ptr(sym.pat_ptr, N.i64p), N.ptr(sym.pat_idx, N.i64p),
                                  N.ptr(sym.sup_parent, N.i64p), N.ptr(sym.perm_fwd, N.i64p),
                                  N.ptr(self.system.colptr, N.i64p), N.ptr(self.system.rowidx, N.i64p),
                                  C.byref(o), C.byref(h)))
        self._handle = h
        self._opts = options
        if self._selector is not None:
            self._install_selector()

    def factor(self, values=None, options: FactorOptions | None = None):
        """SparseLDLT::factor (solver.rs:296-324); `values` default to the
        analyzed system's values."""
        options = options or FactorOptions()
        vals = N.as_f64(self.system.values if values is None else values)
        if vals.size != self.system.rowidx.size:
            raise DimensionMismatch("values do not match the analyzed pattern")
        self._ensure_handle(options)
        self._factored = False
        _check(N.lib().rvg_factor(self._handle, N.ptr(vals, N.dp), N.ptr(self._scaling, N.dp)))
        self._factored = True

    refactor = factor  # solver.rs:335-341

    def factor_device(self, d_values_ptr: int, d_scaling_ptr: int | None, options: FactorOptions | None = None):
        options = options or FactorOptions()
        self._ensure_handle(options)
        self._factored = False
        _check(N.lib().rvg_factor_device(self._handle, C.c_void_p(d_values_ptr),
                                         C.c_void_p(d_scaling_ptr) if d_scaling_ptr else None))
        self._factored = True

    # -- solve ---------------------------------------------------------------
    def solve(self, rhs: np.ndarray) -> np.ndarray:
        """SparseLDLT::solve (allocating, solver.rs:351-362)."""
        x = np.array(rhs, dtype=np.float64, order="F", copy=True)
        self.solve_in_place(x)
        return x

    def solve_in_place(self, rhs: np.ndarray):
        if not self._factored:
            raise SolveBeforeFactor("factor() must be called before solve()")
        if rhs.dtype != np.float64 or not (rhs.flags.f_contiguous or rhs.ndim == 1):
            raise InvalidInput("rhs must be a float64 Fortran-ordered array")
        n = self.system.n
        if rhs.shape[0] != n:
            raise DimensionMismatch(f"RHS length must match matrix dimension: expected {n}, got {rhs.shape[0]}")
        nrhs = 1 if rhs.ndim == 1 else rhs.shape[1]
        _check(N.lib().rvg_solve(self._handle, rhs.ctypes.data_as(N.dp), nrhs, n))

    def solve_refine(self, rhs: np.ndarray, tol: float = 1e-14, max_iter: int = 10):
        """x with FP64 iterative refinement until the scaled backward error is <= tol.
        Returns (x, corrections, backward error)."""
        if not self._factored:
            raise SolveBeforeFactor("factor() must be called before solve()")
        if np.ndim(rhs) == 2:  # several right-hand sides: blocked solves, per-column errors
            b = np.asfortranarray(np.asarray(rhs, dtype=np.float64))
            if b.shape[0] != self.system.n:
                raise DimensionMismatch("RHS length must match matrix dimension")
            x = np.empty_like(b, order="F")
            it = C.c_int32()
            errs = np.zeros(b.shape[1])
            _check(N.lib().rvg_solve_refine_nrhs(self._handle, b.ctypes.data_as(N.dp), x.ctypes.data_as(N.dp),
                                                 b.shape[1], b.shape[0], tol, max_iter, C.byref(it),
                                                 errs.ctypes.data_as(N.dp)))
            return x, it.value, errs
        b = N.as_f64(rhs)
        if b.ndim != 1 or b.size != self.system.n:
            raise DimensionMismatch("RHS length must match matrix dimension")
        x = np.empty_like(b)
        it = C.c_int32()
        err = C.c_double()
        _check(N.lib().rvg_solve_refine(self._handle, N.ptr(b, N.dp), N.ptr(x, N.dp), tol, max_iter, C.byref(it),
                                        C.byref(err)))
        return x, it.value, err.value

    def solve_refine_device(self, d_rhs_ptr: int, d_x_ptr: int, tol: float = 1e-14, max_iter: int = 10):
        if not self._factored:
            raise SolveBeforeFactor("factor() must be called before solve()")
        it = C.c_int32()
        err = C.c_double()
        _check(N.lib().rvg_solve_refine_device(self._handle, C.c_void_p(d_rhs_ptr), C.c_void_p(d_x_ptr), tol, max_iter,
                                               C.byref(it), C.byref(err)))
        return it.value, err.value

    def solve_gmres(self, rhs: np.ndarray, tol: float = 1e-14, max_iter: int = 100, restart: int = 30):
        """x by GMRES-IR: FP64 flexible GMRES preconditioned by the factor.
        Returns (x, preconditioned products, backward error)."""
        if not self._factored:
            raise SolveBeforeFactor("factor() must be called before solve()")
        b = N.as_f64(rhs)
        if b.ndim != 1 or b.size != self.system.n:
            raise DimensionMismatch("RHS length must match matrix dimension")
        x = np.empty_like(b)
        it = C.c_int32()
        err = C.c_double()
        _check(N.lib().rvg_solve_gmres(self._handle, N.ptr(b, N.dp), N.ptr(x, N.dp), tol, max_iter, restart,
                                       C.byref(it), C.byref(err)))
        return x, it.value, err.value

    def solve_auto(self, rhs: np.ndarray, tol: float = 1e-14, max_iter: int = 100):
        """x by iterative refinement, escalating to GMRES-IR when it stalls.
        Returns (x, solves after the first, backward error, "ir" or "gmres")."""
        if not self._factored:
            raise SolveBeforeFactor("factor() must be called before solve()")
        b = N.as_f64(rhs)
        if b.ndim != 1 or b.size != self.system.n:
            raise DimensionMismatch("RHS length must match matrix dimension")
        x = np.empty_like(b)
        it, err, meth = C.c_int32(), C.c_double(), C.c_int32()
        _check(N.lib().rvg_solve_auto(self._handle, N.ptr(b, N.dp), N.ptr(x, N.dp), tol, max_iter, C.byref(it),
                                      C.byref(err), C.byref(meth)))
        return x, it.value, err.value, ("gmres" if meth.value else "ir")

    def solve_auto_device(self, d_rhs_ptr: int, d_x_ptr: int, tol: float = 1e-14, max_iter: int = 100):
        if not self._factored:
            raise SolveBeforeFactor("factor() must be called before solve()")
        it, err, meth = C.c_int32(), C.c_double(), C.c_int32()
        _check(N.lib().rvg_solve_auto_device(self._handle, C.c_void_p(d_rhs_ptr), C.c_void_p(d_x_ptr), tol, max_iter,
                                             C.byref(it), C.byref(err), C.byref(meth)))
        return it.value, err.value, ("gmres" if meth.value else "ir")

    def solve_gmres_device(self, d_rhs_ptr: int, d_x_ptr: int, tol: float = 1e-14, max_iter: int = 100,
                           restart: int = 30):
        if not self._factored:
            raise SolveBeforeFactor("factor() must be called before solve()")
        it = C.c_int32()
        err = C.c_double()
        _check(N.lib().rvg_solve_gmres_device(self._handle, C.c_void_p(d_rhs_ptr), C.c_void_p(d_x_ptr), tol,
                                              max_iter, restart, C.byref(it), C.byref(err)))
        return it.value, err.value

    def solve_refine_nrhs_device(self, d_rhs_ptr: int, d_x_ptr: int, nrhs: int, ldb: int | None = None,
                                 tol: float = 1e-14, max_iter: int = 10):
        """Refined solve of nrhs device-resident columns; returns (corrections, errors per column)."""
        if not self._factored:
            raise SolveBeforeFactor("factor() must be called before solve()")
        it = C.c_int32()
        errs = np.zeros(nrhs)
        _check(N.lib().rvg_solve_refine_nrhs_device(self._handle, C.c_void_p(d_rhs_ptr), C.c_void_p(d_x_ptr), nrhs,
                                                    ldb or self.system.n, tol, max_iter, C.byref(it),
                                                    errs.ctypes.data_as(N.dp)))
        return it.value, errs

    def solve_device(self, d_rhs_ptr: int, nrhs: int = 1, ldb: int | None = None):
        if not self._factored:
            raise SolveBeforeFactor("factor() must be called before solve()")
        _check(N.lib().rvg_solve_device(self._handle, C.c_void_p(d_rhs_ptr), nrhs, ldb or self.system.n))

    # -- results -------------------------------------------------------------
    def inertia(self):
        """(positive, negative, zero) -- solver.rs:504-519; None before factor."""
        if not self._factored:
            return None
        out = np.zeros(3, np.int64)
        _check(N.lib().rvg_inertia(self._handle, N.ptr(out, N.i64p)))
        return tuple(int(x) for x in out)

    def stats(self):
        if not self._factored:
            return None
        st = N.Stats()
        _check(N.lib().rvg_get_stats(self._handle, C.byref(st)))
        return st.as_dict()

    def pivot_record(self):
        """(col, code, d_diag, d_off) per eliminated column, fronts in order."""
        n = self.system.n
        cap = max(n, 1)
        col = np.zeros(cap, np.int64)
        code = np.zeros(cap, np.int8)
        dd = np.zeros(cap)
        do = np.zeros(cap)
        cnt = C.c_int64()
        _check(N.lib().rvg_pivot_record(self._handle, N.ptr(col, N.i64p), N.ptr(code, N.i8p), N.ptr(dd, N.dp),
                                        N.ptr(do, N.dp), C.byref(cnt)))
        t = cnt.value
        return col[:t], code[:t], dd[:t], do[:t]

    def front_info(self):
        ns = C.c_int64()
        _check(N.lib().rvg_front_info(self._handle, None, C.byref(ns)))
        out = np.zeros(9 * max(ns.value, 1), np.int64)
        _check(N.lib().rvg_front_info(self._handle, N.ptr(out, N.i64p), C.byref(ns)))
        return out[:9 * ns.value].reshape(ns.value, 9)

    def per_supernode_stats(self):
        """SparseLDLT::per_supernode_stats (solver.rs:533-543, PerSupernodeStats
        numeric.rs:604-650): one dict per supernode of the last factorization,
        or None before factor().  `max_l_entry` is not computed by this library
        (None); the diagnostic timings of the reference's `diagnostic` feature
        are not kept per supernode (see profile())."""
        if not self._factored:
            return None
        fi = self.front_info()
        return [dict(snode_id=s, front_size=int(r[0]), num_fully_summed=int(r[1]), num_eliminated=int(r[2]),
                     num_delayed=int(r[1] - r[2]), num_1x1=int(r[3]), num_2x2=int(r[4]), max_l_entry=None)
                for s, r in enumerate(fi)]

    # -- learned per-front precision ----------------------------------------
    def set_selector(self, selector, threshold: float | None = None, growth_bound: float | None = None):
        """Installs a trained selector (selector.PrecisionSelector) for
        factorizations with precision="learned"."""
        self._selector = (selector, selector.threshold if threshold is None else threshold,
                          selector.growth_bound if growth_bound is None else growth_bound)
        if self._handle is not None:
            self._install_selector()

    def _install_selector(self):
        sel, thr, bound = self._selector
        p = np.ascontiguousarray(sel.params, dtype=np.float32)
        _check(N.lib().rvg_set_selector(self._handle, p.ctypes.data_as(C.POINTER(C.c_float)), p.size,
                                        float(thr), float(bound)))

    def front_features(self) -> np.ndarray:
        """Rows (RVG_FRONT_FEATURE_COLS) of the large fronts of the last
        learned-precision factorization: supernode, m, k, eliminated, 1x1, 2x2,
        route, probability, max|a|, max|D|, then the 12 features."""
        nr = C.c_int64()
        _check(N.lib().rvg_front_features(self._handle, None, 0, C.byref(nr)))
        out = np.zeros((max(nr.value, 1), 22))
        _check(N.lib().rvg_front_features(self._handle, N.ptr(out, N.dp), nr.value, C.byref(nr)))
        return out[:nr.value]

    def selector_stats(self) -> dict:
        out = np.zeros(4, np.int64)
        _check(N.lib().rvg_selector_stats(self._handle, N.ptr(out, N.i64p)))
        return dict(large_fronts=int(out[0]), routed_mixed=int(out[1]), over_bound=int(out[2]),
                    fp64_refactored=int(out[3]), fp64_rerun=bool(out[3]))

    def work(self):
        out = np.zeros(6)
        _check(N.lib().rvg_work(self._handle, N.ptr(out, N.dp)))
        return dict(flops_factor=out[0], flops_schur=out[1], bytes_assembly=out[2], bytes_solve_per_rhs=out[3],
                    nnz_l=int(out[4]), max_front=int(out[5]))

    def timings(self):
        out = np.zeros(7)
        _check(N.lib().rvg_timings(self._handle, N.ptr(out, N.dp)))
        return dict(assembly_ms=out[0], kernel_ms=out[1], gemm_ms=out[2], factor_ms=out[3], solve_ms=out[4])

    def trim(self, workspace: bool = True, factor: bool = False):
        """Release device memory: the factor/solve workspace and, with
        factor=True, the factor too (solve then needs a new factor())."""
        if self._handle is None:
            return
        _check(N.lib().rvg_trim(self._handle, (1 if workspace else 0) | (2 if factor else 0)))
        if factor:
            self._factored = False

    def set_profiling(self, enable: bool = True):
        if self._handle is None:
            self._ensure_handle(self._opts or FactorOptions())
        _check(N.lib().rvg_set_profiling(self._handle, int(enable)))

    def profile(self):
        p = N.Profile()
        _check(N.lib().rvg_get_profile(self._handle, C.byref(p)))
        return p.as_dict()

    def stream(self) -> int:
        s = C.c_void_p()
        _check(N.lib().rvg_stream(self._handle, C.byref(s)))
        return s.value or 0

    def close(self):
        if self._handle is not None:
            N.lib().rvg_destroy(self._handle)
            self._handle = None
            self._factored = False

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def n(self):
        return self.system.n


def solve_full(system, b, analyze=None, factor=None, scaling=None):
    """SparseLDLT::solve_full (solver.rs:470-494)."""
    s = SparseLDLT.analyze_with_matrix(system, analyze, scaling)
    s.factor(None, factor)
    x = s.solve(b)
    s.close()
    return x
