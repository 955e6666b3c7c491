"""The C-ABI library: builds, loads and exports every symbol that
include/rivrs_b200.h declares; option validation maps onto InvalidInput
(factor.rs:307-347) before any device work."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from conftest import HAS_GPU, ROOT


def declared_symbols():
    txt = open(os.path.join(ROOT, "include", "rivrs_b200.h")).read()
    return sorted(set(re.findall(r"\b(rvg_[a-z_0-9]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol(rv):
    L = C.CDLL(rv.LIB_PATH)
    names = declared_symbols()
    assert len(names) >= 19
    for n in names:
        assert hasattr(L, n), n


def test_default_options_match_reference(rv):
    o = rv._native.default_options()
    assert (o.threshold, o.small, o.outer_block_size, o.inner_block_size, o.nemin, o.small_leaf_threshold,
            o.failed_pivot_tpp, o.fallback_bk) == (0.01, 1e-20, 256, 32, 32, 256, 1, 1)
    assert (o.far_field_sms, o.mixed_window) == (-1, 0)  # scheduling options: their defaults


@pytest.mark.parametrize("bad", [dict(threshold=0.0), dict(threshold=1.5), dict(small=-1.0),
                                 dict(outer_block_size=0), dict(inner_block_size=0),
                                 dict(inner_block_size=64, outer_block_size=32), dict(far_field_sms=-2),
                                 dict(mixed_window=-1), dict(mixed_window=9), dict(graph_refactor=-1),
                                 dict(graph_refactor=3)])
def test_invalid_options_rejected(rv, bad):
    s = rv.problems.shifted_laplacian(3, 0.1)
    solver = rv.SparseLDLT.analyze(s)
    kw = dict(rv.FactorOptions().__dict__)
    kw.update(bad)
    with pytest.raises(rv.InvalidInput):
        solver.factor(None, rv.FactorOptions(**kw))


def test_solve_before_factor(rv):
    s = rv.problems.shifted_laplacian(3, 0.1)
    solver = rv.SparseLDLT.analyze(s)
    with pytest.raises(rv.SolveBeforeFactor):
        solver.solve(np.ones(s.n))
    assert solver.inertia() is None and solver.stats() is None


@pytest.mark.skipif(HAS_GPU, reason="checks the no-device error path")
def test_no_device_fails_loudly(rv):
    s = rv.problems.shifted_laplacian(3, 0.1)
    solver = rv.SparseLDLT.analyze(s)
    with pytest.raises(rv.SparseError, match="DeviceError"):
        solver.factor()


def test_binding_table_covers_every_symbol(rv):
    """The Python host mirror gives every entry point the header declares a
    ctypes signature (argument and result types), so no call goes through
    ctypes' default int conversion of 64-bit arguments."""
    table = rv._native.SIGNATURES
    missing = [n for n in declared_symbols() if n not in table]
    assert not missing, missing
    extra = [n for n in table if n not in declared_symbols()]
    assert not extra, extra
