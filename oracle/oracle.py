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
        _lib = L
    return _lib


def _p(a, t):
    return None if a is None else a.ctypes.data_as(t)


class OracleFactor:
    """AptpNumeric::factor + aptp_solve restated on the CPU."""

    STAT_KEYS = ["total_1x1_pivots", "total_2x2_pivots", "total_delayed", "zero_pivots", "max_front_size",
                 "supernodes_before_amalgamation", "supernodes_after_amalgamation", "merges_performed",
                 "small_leaf_subtrees", "small_leaf_nodes", "near_ties"]

    def __init__(self, system, symbolic, scaling_elim=None, opts=None, nthreads=1):
        L = lib()
        self.n = system.n
        self._keep = [np.ascontiguousarray(x) for x in (symbolic.sup_begin, symbolic.sup_end, symbolic.pat_ptr,
                                                         symbolic.pat_idx, symbolic.sup_parent, symbolic.perm_fwd,
                                                         system.colptr, system.rowidx)]
        vals = np.ascontiguousarray(system.values, dtype=np.float64)
        sc = None if scaling_elim is None else np.ascontiguousarray(scaling_elim, dtype=np.float64)
        o = opts or options()
        k = self._keep
        self.h = L.orc_factor(system.n, symbolic.sup_begin.size, _p(k[0], i64p), _p(k[1], i64p), _p(k[2], i64p),
                              _p(k[3], i64p), _p(k[4], i64p), _p(k[5], i64p), _p(k[6], i64p), _p(k[7], i64p),
                              _p(vals, dp), _p(sc, dp), C.byref(o), nthreads)

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

    def close(self):
        if self.h:
            lib().orc_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


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
