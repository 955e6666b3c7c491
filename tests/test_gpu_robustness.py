"""Adversarial inputs (the cases of the reference's tests/adversarial.rs):
NaN and Inf values are rejected with InvalidInput before any factor kernel
runs; arrowhead, exact cancellation, near-overflow and near-underflow
entries, disconnected components and power-of-two sizes factor with the
oracle's pivots and D bit for bit and solve to the reference's gate."""
import numpy as np
import pytest
import scipy.sparse as sp

from test_gpu_parity import assert_parity, run_both

pytestmark = pytest.mark.gpu


def system(rv, name, dense):
    return rv.problems.from_scipy(name, sp.csc_matrix(np.asarray(dense, dtype=np.float64)))


@pytest.mark.parametrize("bad", [np.nan, np.inf, -np.inf])
def test_non_finite_values_rejected(rv, bad):
    a = np.diag([4.0, 4.0, 4.0, 4.0])
    a[0, 1] = a[1, 0] = bad
    s = system(rv, "nonfinite", a)
    solver = rv.SparseLDLT.analyze(s)
    with pytest.raises(rv.InvalidInput):
        solver.factor()
    with pytest.raises(rv.SolveBeforeFactor):
        solver.solve(np.ones(4))
    solver.factor(np.nan_to_num(s.values, nan=1.0, posinf=1.0, neginf=1.0))  # the handle stays usable
    assert solver.inertia() == (4, 0, 0)
    solver.close()


def test_non_finite_scaling_rejected(rv):
    s = system(rv, "scaled", np.diag([2.0, 3.0, 5.0]))
    solver = rv.SparseLDLT.analyze(s)
    solver._scaling = np.array([1.0, np.inf, 1.0])
    with pytest.raises(rv.InvalidInput):
        solver.factor()
    solver.close()


def cases():
    n = 12
    arrow = np.diag(np.where(np.arange(n) % 2 == 0, 10.0, -10.0))
    arrow[0, 1:] = arrow[1:, 0] = 1.0
    cancel = np.array([[1.0, 1.0, 1.0], [1.0, 1.0, 0.0], [1.0, 0.0, 1.0]])
    big, tiny = 1e150, 1e-150
    over = np.array([[big, 1, 0, 0], [1, big, 0, 0], [0, 0, big, 1], [0, 0, 1, big]])
    under = np.array([[tiny, tiny / 2, 0, 0], [tiny / 2, tiny, 0, 0], [0, 0, tiny, tiny / 2], [0, 0, tiny / 2, tiny]])
    block = np.array([[4.0, -1, 0], [-1, 4, -1], [0, -1, 4]])
    disc = np.kron(np.eye(2), block)
    return {"arrowhead": arrow, "exact_cancellation": cancel, "near_overflow": over, "near_underflow": under,
            "disconnected": disc}


@pytest.mark.parametrize("name", sorted(cases()))
def test_structured_adversarial(rv, orc, name):
    s = system(rv, name, cases()[name])
    solver, ref, b = run_both(rv, orc, s)
    if name == "near_underflow":
        # entries of 1e-150 are below `small` (1e-20): every pivot is a zero pivot, as in the oracle, and
        # the solve zeroes those components; the backward error gate is then the oracle's own
        b = b * 1e-150
        assert solver.inertia() == (0, 0, 4)
    assert_parity(rv, s, solver, ref, b, bwd=5e-11)
    solver.close()


@pytest.mark.parametrize("n", [31, 32, 33, 63, 64, 65, 127, 128, 129, 255, 256, 257, 511, 512, 513])
def test_power_of_two_boundaries(rv, orc, n):
    rng = np.random.default_rng(n)
    a = rng.uniform(-1, 1, (n, n))
    a = a + a.T + np.diag(np.where(np.arange(n) < n // 2, 1.0, -1.0) * n)
    s = system(rv, f"pow2_{n}", a)
    solver, ref, b = run_both(rv, orc, s)
    assert_parity(rv, s, solver, ref, b, bwd=5e-11)
    solver.close()
