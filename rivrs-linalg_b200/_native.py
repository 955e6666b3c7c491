"""ctypes binding of the in-tree library librivrs_b200.so (include/rivrs_b200.h).

The library is the product: there is no Python or CPU fallback for the
numeric phase.  Loading fails loudly when the shared object is missing.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "librivrs_b200.so")

i64 = C.c_int64
i64p = C.POINTER(C.c_int64)
dp = C.POINTER(C.c_double)
i8p = C.POINTER(C.c_int8)
vp = C.c_void_p

STATUS = {
    0: "OK", 1: "DimensionMismatch", 2: "InvalidInput", 3: "SolveBeforeFactor", 4: "AnalysisFailure",
    5: "DeviceError", 6: "DeviceTimeout", 7: "OutOfMemory",
}


class Options(C.Structure):
    _fields_ = [("threshold", C.c_double), ("small", C.c_double), ("outer_block_size", i64),
                ("inner_block_size", i64), ("nemin", i64), ("small_leaf_threshold", i64),
                ("failed_pivot_tpp", C.c_int32), ("fallback_bk", C.c_int32), ("large_front_threshold", i64),
                ("precision", C.c_int32), ("mixed_flush", C.c_int32),
                ("mixed_tile_cols", C.c_int32), ("mixed_operands", C.c_int32),
                ("graph_refactor", C.c_int32), ("far_field_sms", C.c_int32),
                ("mixed_window", C.c_int32)]


class Stats(C.Structure):
    _fields_ = [("total_1x1_pivots", i64), ("total_2x2_pivots", i64), ("total_delayed", i64),
                ("zero_pivots", i64), ("max_front_size", i64), ("supernodes_before_amalgamation", i64),
                ("supernodes_after_amalgamation", i64), ("merges_performed", i64),
                ("small_leaf_subtrees", i64), ("small_leaf_nodes", i64)]

    def as_dict(self):
        return {k: int(getattr(self, k)) for k, _ in self._fields_}


class Profile(C.Structure):
    _fields_ = [("factor_ms", C.c_double), ("solve_ms", C.c_double), ("assembly_ms", C.c_double),
                ("dense_ms", C.c_double), ("cbgemm_ms", C.c_double), ("syrk_ms", C.c_double),
                ("syrk_flops", C.c_double), ("syrk_launches", i64), ("factor_launches", i64),
                ("solve_launches", i64), ("peak_bytes", i64), ("host_total_ms", C.c_double),
                ("host_alloc_ms", C.c_double), ("host_sync_ms", C.c_double), ("part_ms", C.c_double * 16),
                ("host_wait_ms", C.c_double), ("lf_misses", i64), ("host_gap_ms", C.c_double),
                ("lf_far_updates", i64)]

    PARTS = ("lf_setup", "lf_block", "lf_panel", "lf_post", "lf_update", "lf_delay", "lf_prop", "lf_w", "lf_syrk",
             "lf_outer", "tpp", "aptp", "cb_w", "cb_gemm", "cb_syrk", "other")

    def as_dict(self):
        d = {}
        for k, t in self._fields_:
            if k == "part_ms":
                d[k] = {n: float(v) for n, v in zip(self.PARTS, self.part_ms)}
            else:
                d[k] = float(getattr(self, k)) if t is C.c_double else int(getattr(self, k))
        return d


class RvgError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


_lib = None

SIGNATURES = {
    "rvg_default_options": (None, [C.POINTER(Options)]),
    "rvg_last_error": (C.c_char_p, []),
    "rvg_analyze": (C.c_int, [i64, i64p, i64p, i64p, C.POINTER(vp)]),
    "rvg_symbolic_sizes": (C.c_int, [vp, i64p]),
    "rvg_symbolic_export": (C.c_int, [vp, i64p, i64p, i64p, i64p, i64p, i64p]),
    "rvg_symbolic_free": (None, [vp]),
    "rvg_create": (C.c_int, [i64, i64, i64p, i64p, i64p, i64p, i64p, i64p, i64p, i64p, C.POINTER(Options),
                             C.POINTER(vp)]),
    "rvg_factor": (C.c_int, [vp, dp, dp]),
    "rvg_factor_device": (C.c_int, [vp, vp, vp]),
    "rvg_solve": (C.c_int, [vp, dp, i64, i64]),
    "rvg_solve_device": (C.c_int, [vp, vp, i64, i64]),
    "rvg_solve_refine": (C.c_int, [vp, dp, dp, C.c_double, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_double)]),
    "rvg_solve_gmres": (C.c_int, [vp, dp, dp, C.c_double, C.c_int32, C.c_int32, C.POINTER(C.c_int32),
                                  C.POINTER(C.c_double)]),
    "rvg_solve_gmres_device": (C.c_int, [vp, vp, vp, C.c_double, C.c_int32, C.c_int32, C.POINTER(C.c_int32),
                                         C.POINTER(C.c_double)]),
    "rvg_solve_auto": (C.c_int, [vp, dp, dp, C.c_double, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_double),
                                 C.POINTER(C.c_int32)]),
    "rvg_solve_auto_device": (C.c_int, [vp, vp, vp, C.c_double, C.c_int32, C.POINTER(C.c_int32),
                                        C.POINTER(C.c_double), C.POINTER(C.c_int32)]),
    "rvg_solve_refine_nrhs": (C.c_int, [vp, dp, dp, i64, i64, C.c_double, C.c_int32, C.POINTER(C.c_int32), dp]),
    "rvg_solve_refine_nrhs_device": (C.c_int, [vp, vp, vp, i64, i64, C.c_double, C.c_int32, C.POINTER(C.c_int32),
                                               dp]),
    "rvg_solve_refine_device": (C.c_int, [vp, vp, vp, C.c_double, C.c_int32, C.POINTER(C.c_int32),
                                          C.POINTER(C.c_double)]),
    "rvg_inertia": (C.c_int, [vp, i64p]),
    "rvg_get_stats": (C.c_int, [vp, C.POINTER(Stats)]),
    "rvg_pivot_record": (C.c_int, [vp, i64p, i8p, dp, dp, i64p]),
    "rvg_front_info": (C.c_int, [vp, i64p, i64p]),
    "rvg_work": (C.c_int, [vp, dp]),
    "rvg_timings": (C.c_int, [vp, dp]),
    "rvg_stream": (C.c_int, [vp, C.POINTER(vp)]),
    "rvg_set_profiling": (C.c_int, [vp, C.c_int32]),
    "rvg_get_profile": (C.c_int, [vp, C.POINTER(Profile)]),
    "rvg_selftest_waits": (C.c_int, [vp, C.c_int32]),
    "rvg_trim": (C.c_int, [vp, C.c_int32]),
    "rvg_mem_info": (C.c_int, [i64p]),
    "rvg_mc64": (C.c_int, [i64, i64p, i64p, dp, i64p, dp, i64p]),
    "rvg_dense_factor_noalloc": (C.c_int, [vp, i64, i64, C.POINTER(Options), vp, vp, vp, vp, vp, vp]),
    "rvg_mlp_param_count": (i64, []),
    "rvg_mlp_trained_count": (i64, []),
    "rvg_mlp_work_floats": (i64, [i64]),
    "rvg_mlp_forward": (C.c_int, [vp, vp, i64, vp, vp]),
    "rvg_mlp_grad": (C.c_int, [vp, vp, vp, vp, i64, C.c_double, vp, vp, vp, i64, vp]),
    "rvg_mlp_adam": (C.c_int, [vp, vp, vp, vp, i64, C.c_float, C.c_float, C.c_float, C.c_float, C.c_float, vp]),
    "rvg_set_selector": (C.c_int, [vp, C.POINTER(C.c_float), i64, C.c_float, C.c_double]),
    "rvg_front_features": (C.c_int, [vp, dp, i64, i64p]),
    "rvg_selector_stats": (C.c_int, [vp, i64p]),
    "rvg_destroy": (None, [vp]),
}


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python rivrs-linalg_b200/build.py` "
                              "(the numeric phase has no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(status):
    if status != 0:
        raise RvgError(status, lib().rvg_last_error().decode())


def ptr(a, ctype):
    return a.ctypes.data_as(ctype) if a is not None else None


def as_i64(a):
    return np.ascontiguousarray(a, dtype=np.int64)


def as_f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def default_options(**kw) -> Options:
    o = Options()
    lib().rvg_default_options(C.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o
