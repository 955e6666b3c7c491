"""ctypes binding of the oracle (oracle.cpp): the CPU restatement of the
rivrs-sparse numeric phase.  Test infrastructure: only tests/, the smoke
check and the CPU-baseline leg of bench.py use it, as the checker.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liboracle.so")

i64 = C.c_int64
i64p = C.POINTER(C.c_int64)
dp = C.POINTER(C.c_double)
i8p = C.POINTER(C.c_int8)


class OrcOptions(C.Structure):
    _fields_ = [("threshold", C.c_double), ("small", C.c_double), ("outer_block_size", i64),
                ("inner_block_size", i64), ("nemin", i64), ("small_leaf_threshold", i64),
                ("failed_pivot_tpp", C.c_int32), ("fallback_bk", C.c_int32)]


def options(threshold=0.01, small=1e-20, outer_block_size=256, inner_block_size=32, nemin=32,
            small_leaf_threshold=256, failed_pivot_tpp=True, fallback_bunch_kaufman=True, **device_only):
    # device_only: scheduling options of the GPU path (e.g. large_front_threshold)
    # that do not change results and have no meaning for the oracle
    return OrcOptions(threshold, small, outer_block_size, inner_block_size, nemin, small_leaf_threshold,
                      int(failed_pivot_tpp), int(fallback_bunch_kaufman))


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            import importlib.util
            spec = importlib.util.spec_from_file_location("_oracle_build", os.path.join(HERE, "build.py"))
            mod = importlib.util.module_from_spec(spec)
            spec.loader.exec_module(mod)
            mod.build()
        L = C.CDLL(LIB)
        L.orc_factor.restype = C.c_void_p
        L.orc_factor.argtypes = [i64, i64, i64p, i64p, i64p, i64p, i64p, i64p, i64p, i64p, dp, dp,
                                 C.POINTER(OrcOptions), C.c_int32]
        L.orc_free.argtypes = [C.c_void_p]
        L.orc_stats.argtypes = [C.c_void_p, i64p]
        L.orc_inertia.argtypes = [C.c_void_p, i64p]
        L.orc_nsup.restype = i64
        L.orc_nsup.argtypes = [C.c_void_p]
        L.orc_front_info.argtypes = [C.c_void_p, i64p]
        L.orc_elim.restype = i64
        L.orc_elim.argtypes = [C.c_void_p, i64p, i8p, dp, dp]
        L.orc_solve.argtypes = [C.c_void_p, dp]
        L.orc_dense_aptp.argtypes = [i64, i64, dp, C.POINTER(OrcOptions), i64p, i8p, dp, dp, i64p, dp]
        L.orc_session_begin.restype = C.c_void_p
        L.orc_session_begin.argtypes = L.orc_factor.argtypes
        L.orc_session_total.restype = C.c_double
        L.orc_session_total.argtypes = [C.c_void_p]
        L.orc_session_done.restype = C.c_double
        L.orc_session_done.argtypes = [C.c_void_p]
        L.orc_session_advance.restype = C.c_int32
        L.orc_session_advance.argtypes = [C.c_void_p, C.c_double]
        L.orc_session_finish.restype = C.c_void_p
        L.orc_session_finish.argtypes = [C.c_void_p]
        L.orc_release_cache.argtypes = []
        L.orc_session_abort.argtypes = [C.c_void_p]
        _lib = L
    return _lib


def _p(a, t):
    return None if a is None else a.ctypes.data_as(t)


class OracleFactor:
    """AptpNumeric::factor + aptp_solve restated on the CPU."""

    STAT_KEYS = ["total_1x1_pivots", "total_2x2_pivots", "total_delayed", "zero_pivots", "max_front_size",
                 "supernodes_before_amalgamation", "supernodes_after_amalgamation", "merges_performed",
                 "small_leaf_subtrees", "small_leaf_nodes", "near_ties"]

    def __init__(self, system, symbolic, scaling_elim=None, opts=None, nthreads=1, sliced=False):
        L = lib()
        self.n = system.n
        self._keep = [np.ascontiguousarray(x) for x in (symbolic.sup_begin, symbolic.sup_end, symbolic.pat_ptr,
                                                         symbolic.pat_idx, symbolic.sup_parent, symbolic.perm_fwd,
                                                         system.colptr, system.rowidx)]
        vals = np.ascontiguousarray(system.values, dtype=np.float64)
        sc = None if scaling_elim is None else np.ascontiguousarray(scaling_elim, dtype=np.float64)
        o = opts or options()
        k = self._keep
        self._keep += [vals, sc, o]
        args = (system.n, symbolic.sup_begin.size, _p(k[0], i64p), _p(k[1], i64p), _p(k[2], i64p),
                _p(k[3], i64p), _p(k[4], i64p), _p(k[5], i64p), _p(k[6], i64p), _p(k[7], i64p),
                _p(vals, dp), _p(sc, dp), C.byref(o), nthreads)
        self.h = None
        self.session = None
        if sliced:
            # the numeric phase runs in slices: advance() / finish()
            self.session = L.orc_session_begin(*args)
        else:
            self.h = L.orc_factor(*args)

    def total_flops(self):
        """Delay-free flops of the factorization (sliced runs)."""
        return lib().orc_session_total(self.session)

    def advance(self, target_flops):
        """Run the factorization until target_flops are done (at the next
        checkpoint) or it ends; True when it has ended."""
        return bool(lib().orc_session_advance(self.session, float(target_flops)))

    def finish(self):
        if self.session is not None:
            self.h = lib().orc_session_finish(self.session)
            self.session = None

    def stats(self):
        out = np.zeros(11, np.int64)
        lib().orc_stats(self.h, _p(out, i64p))
        return dict(zip(self.STAT_KEYS, (int(x) for x in out)))

    def inertia(self):
        out = np.zeros(3, np.int64)
        lib().orc_inertia(self.h, _p(out, i64p))
        return tuple(int(x) for x in out)

    def front_info(self):
        ns = lib().orc_nsup(self.h)
        out = np.zeros(9 * max(ns, 1), np.int64)
        lib().orc_front_info(self.h, _p(out, i64p))
        return out[:9 * ns].reshape(ns, 9)

    def pivot_record(self):
        cap = max(self.n, 1)
        col = np.zeros(cap, np.int64)
        code = np.zeros(cap, np.int8)
        dd = np.zeros(cap)
        do = np.zeros(cap)
        t = lib().orc_elim(self.h, _p(col, i64p), _p(code, i8p), _p(dd, dp), _p(do, dp))
        return col[:t], code[:t], dd[:t], do[:t]

    def solve(self, b):
        b = np.asarray(b, dtype=np.float64)
        if b.ndim == 1:
            x = b.copy()
            lib().orc_solve(self.h, _p(x, dp))
            return x
        x = np.array(b, order="F", copy=True)
        for j in range(x.shape[1]):
            col = np.ascontiguousarray(x[:, j])
            lib().orc_solve(self.h, _p(col, dp))
            x[:, j] = col
        return x

    def abort(self):
        """Stop a sliced factorization where it is and free it."""
        if self.session is not None:
            lib().orc_session_abort(self.session)
            self.session = None

    def close(self):
        self.abort()
        if self.h:
            lib().orc_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---- host analysis for CPU-only runs (libanalysis.so) ----------------------
ALIB = os.path.join(HERE, "_build", "libanalysis.so")
_alib = None


def alib():
    global _alib
    if _alib is None:
        if not os.path.exists(ALIB):
            lib()  # builds both libraries
            import importlib.util
            spec = importlib.util.spec_from_file_location("_oracle_build", os.path.join(HERE, "build.py"))
            mod = importlib.util.module_from_spec(spec)
            spec.loader.exec_module(mod)
            mod.build()
        L = C.CDLL(ALIB)
        L.rvg_last_error.restype = C.c_char_p
        L.rvg_analyze.restype = C.c_int
        L.rvg_analyze.argtypes = [i64, i64p, i64p, i64p, C.POINTER(C.c_void_p)]
        L.rvg_symbolic_sizes.argtypes = [C.c_void_p, i64p]
        L.rvg_symbolic_export.argtypes = [C.c_void_p, i64p, i64p, i64p, i64p, i64p, i64p]
        L.rvg_symbolic_free.argtypes = [C.c_void_p]
        L.rvg_mc64.restype = C.c_int
        L.rvg_mc64.argtypes = [i64, i64p, i64p, dp, i64p, dp, i64p]
        _alib = L
    return _alib


class Symbolic:
    """The symbolic structure the numeric phase takes (what AptpSymbolic
    exposes): perm_fwd[new] = old, supernode column ranges, parents and row
    patterns."""

    def __init__(self, n, perm_fwd, sup_begin, sup_end, sup_parent, pat_ptr, pat_idx):
        self.n, self.perm_fwd, self.sup_begin, self.sup_end = n, perm_fwd, sup_begin, sup_end
        self.sup_parent, self.pat_ptr, self.pat_idx = sup_parent, pat_ptr, pat_idx


def _acheck(st):
    if st != 0:
        raise RuntimeError(f"analysis failed ({st}): {alib().rvg_last_error().decode()}")


def analyze(system, order, mc64=True):
    """Symbolic analysis for a fill-reducing `order` and, with mc64, the MC64
    symmetric scaling in elimination order -- the library's host analysis
    (the same code the GPU path uses), loaded without the GPU library.
    Returns (Symbolic, scaling or None)."""
    L = alib()
    n = int(system.n)
    colptr = np.ascontiguousarray(system.colptr, dtype=np.int64)
    rowidx = np.ascontiguousarray(system.rowidx, dtype=np.int64)
    order = np.ascontiguousarray(order, dtype=np.int64)
    h = C.c_void_p()
    _acheck(L.rvg_analyze(n, _p(colptr, i64p), _p(rowidx, i64p), _p(order, i64p), C.byref(h)))
    try:
        sz = np.zeros(4, np.int64)
        _acheck(L.rvg_symbolic_sizes(h, _p(sz, i64p)))
        nn, ns, npat, _ = (int(x) for x in sz)
        perm = np.zeros(nn, np.int64)
        b, e, par = np.zeros(ns, np.int64), np.zeros(ns, np.int64), np.zeros(ns, np.int64)
        pp, pi = np.zeros(ns + 1, np.int64), np.zeros(max(npat, 1), np.int64)
        _acheck(L.rvg_symbolic_export(h, _p(perm, i64p), _p(b, i64p), _p(e, i64p), _p(par, i64p), _p(pp, i64p),
                                      _p(pi, i64p)))
    finally:
        L.rvg_symbolic_free(h)
    sym = Symbolic(nn, perm, b, e, par, pp, pi[:npat])
    scaling = None
    if mc64 and n > 0:
        vals = np.ascontiguousarray(system.values, dtype=np.float64)
        matching = np.zeros(n, np.int64)
        sc = np.zeros(n, np.float64)
        matched = C.c_int64(0)
        _acheck(L.rvg_mc64(n, _p(colptr, i64p), _p(rowidx, i64p), _p(vals, dp), _p(matching, i64p), _p(sc, dp),
                           C.byref(matched)))
        scaling = np.ascontiguousarray(sc[perm])
    return sym, scaling


def release_cache():
    """Give the oracle's cached front buffers back to the system."""
    lib().orc_release_cache()


def dense_aptp(a, p=None, opts=None):
    """aptp_factor_in_place on a dense matrix (lower triangle read).  Returns
    (factored matrix, perm, dtype, ddiag, doff, [ne, n1x1, n2x2, ndelayed], max_l)."""
    a = np.array(a, dtype=np.float64, order="F", copy=True)
    m = a.shape[0]
    p = m if p is None else p
    perm = np.zeros(m, np.int64)
    dt = np.zeros(max(p, 1), np.int8)
    dd = np.zeros(max(p, 1))
    do = np.zeros(max(p, 1))
    st = np.zeros(4, np.int64)
    ml = C.c_double()
    o = opts or options()
    lib().orc_dense_aptp(m, p, _p(a, dp), C.byref(o), _p(perm, i64p), _p(dt, i8p), _p(dd, dp), _p(do, dp),
                         _p(st, i64p), C.byref(ml))
    return a, perm, dt[:p], dd[:p], do[:p], st, ml.value
