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


@pytest.mark.parametrize("bad", [dict(threshold=0.0), dict(threshold=1.5), dict(small=-1.0),
                                 dict(outer_block_size=0), dict(inner_block_size=0),
                                 dict(inner_block_size=64, outer_block_size=32)])
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


def test_integration_guide_binds_every_symbol():
    """Every entry point the header declares has its binding in INTEGRATION.md."""
    guide = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    missing = [n for n in declared_symbols() if f"fn {n}(" not in guide]
    assert not missing, missing
