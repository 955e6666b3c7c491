"""Bounded device waits: a wait that nothing releases runs out, the host reads
RVG_ERR_DEVICE_TIMEOUT, and the handle (and its CUDA context) stays usable.

The waits are made to run out on purpose without faulting anything: a flag
that is never raised (the solve's block dependencies) and a tensor-core GEMM
whose producer issues no copies (the mixed-form pipeline)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RVG_ERR_DEVICE_TIMEOUT = 6


@pytest.mark.parametrize("which", [0, 1])
def test_wait_runs_out_and_is_reported(rv, which):
    s = rv.problems.shifted_laplacian(8, 0.1)
    solver = rv.SparseLDLT.analyze(s)
    solver.factor(None, rv.FactorOptions(precision="mixed"))
    st = rv._native.lib().rvg_selftest_waits(solver._handle, which)
    assert st == RVG_ERR_DEVICE_TIMEOUT
    # the status was consumed: the next calls succeed and are correct
    solver.factor(None, rv.FactorOptions(precision="mixed"))
    b = rv.problems.rhs_normal(s.n, 1)
    x, iters, err = solver.solve_refine(b, tol=1e-14, max_iter=10)
    assert err <= 1e-14
    assert solver.inertia() == s.inertia
    solver.close()


def test_selftest_rejects_bad_argument(rv):
    s = rv.problems.shifted_laplacian(4, 0.1)
    solver = rv.SparseLDLT.analyze(s)
    solver.factor()
    assert rv._native.lib().rvg_selftest_waits(solver._handle, 7) == 2  # RVG_ERR_INVALID_INPUT
    solver.close()
