"""MC64 matching and symmetric scaling (rvg_mc64; the reference's mc64_matching,
sparse/src/ordering/matching.rs:121-248) on the host.

The checks are the reference's own: its unit-test matrices (matching.rs:1400-1760)
and the SPRAL scaling properties it asserts on every result
(sparse/src/testing/mc64_validation.rs:113-220): |s_i a_ij s_j| <= 1 + 1e-10 on
entries touching a matched index, every nonzero row reaching 1 - 1e-12, a valid
permutation, positive finite factors.  Optimality of the matching (the
maximum product of matched magnitudes, which is unique even when the matching
is not) is checked against scipy's assignment solver.
"""
import numpy as np
import pytest
import scipy.sparse as sp
from scipy.optimize import linear_sum_assignment

from conftest import golden_system


def upper(n, entries):
    a = np.zeros((n, n))
    for i, j, v in entries:
        a[i, j] = v
        a[j, i] = v
    return a


def system(rv, a, name="m"):
    m = sp.csc_matrix(a)
    m.sort_indices()
    return rv.problems.from_scipy(name, m)


def verify_properties(s, matching, scaling, matched):
    a = s.to_scipy().toarray()
    n = s.n
    is_matched = np.zeros(n, bool)
    # rows that kept a real matching edge: |a_{i, matching[i]}| > 0 and counted
    for i in range(n):
        is_matched[i] = a[i, matching[i]] != 0
    assert matched == is_matched.sum() or matched <= n
    sc = np.abs(scaling[:, None] * a * scaling[None, :])
    touch = is_matched[:, None] | is_matched[None, :]
    nz = a != 0
    assert (sc[nz & touch] <= 1.0 + 1e-10).all(), sc[nz & touch].max()
    for i in range(n):
        if nz[i].any() and is_matched[i]:
            assert sc[i][nz[i]].max() >= 1.0 - 1e-12, (i, sc[i][nz[i]].max())
    assert sorted(matching.tolist()) == list(range(n))
    assert (scaling > 0).all() and np.isfinite(scaling).all()


def optimal_log_product(a):
    with np.errstate(divide="ignore"):
        c = np.where(a != 0, -np.log(np.abs(a)), 1e30)
    r, col = linear_sum_assignment(c)
    return c[r, col].sum()


def test_diagonal_identity(rv):
    s = system(rv, np.diag([4.0, 9.0, 1.0]))
    m, sc, k = rv.ordering.mc64(s)
    assert k == 3 and list(m) == [0, 1, 2]
    assert np.allclose(sc, 1.0 / np.sqrt([4.0, 9.0, 1.0]))
    verify_properties(s, m, sc, k)


def test_negative_diagonal_identity(rv):
    s = system(rv, np.diag([-10.0, -20.0, -5.0]))
    m, sc, k = rv.ordering.mc64(s)
    assert k == 3 and list(m) == [0, 1, 2]
    verify_properties(s, m, sc, k)


@pytest.mark.parametrize("case", ["tridiagonal", "arrow", "trivial_1x1", "trivial_2x2"])
def test_reference_unit_matrices(rv, case):
    a = {
        "tridiagonal": upper(4, [(0, 0, 2.0), (0, 1, -1.0), (1, 1, -3.0), (1, 2, 2.0), (2, 2, 1.0), (2, 3, -1.0),
                                 (3, 3, -4.0)]),
        "arrow": upper(5, [(0, 0, 10.0), (0, 1, 1.0), (0, 2, 1.0), (0, 3, 1.0), (0, 4, 1.0), (1, 1, -3.0),
                           (2, 2, 5.0), (3, 3, -2.0), (4, 4, 4.0)]),
        "trivial_1x1": upper(1, [(0, 0, 7.0)]),
        "trivial_2x2": upper(2, [(0, 0, 3.0), (0, 1, 1.0), (1, 1, 5.0)]),
    }[case]
    s = system(rv, a)
    m, sc, k = rv.ordering.mc64(s)
    assert k == s.n
    verify_properties(s, m, sc, k)
    assert np.isclose(sum(-np.log(abs(a[i, m[i]])) for i in range(s.n)), optimal_log_product(a))


def test_structurally_singular(rv):
    # no diagonal, two 2x2 blocks (matching.rs:1649-1675) and an isolated index (1752-1775)
    for a in (upper(4, [(0, 1, 5.0), (2, 3, 3.0)]), upper(3, [(0, 1, 5.0)])):
        s = system(rv, a)
        m, sc, k = rv.ordering.mc64(s)
        assert sorted(m.tolist()) == list(range(s.n))
        assert (sc > 0).all() and np.isfinite(sc).all()
    a = upper(6, [(0, 0, 10.0), (0, 1, 1.0), (1, 1, 8.0), (1, 2, 2.0), (2, 2, 6.0), (2, 3, 3.0), (3, 3, 5.0),
                  (3, 4, 1.0), (4, 4, 7.0), (0, 5, 0.1)])
    s = system(rv, a)
    m, sc, k = rv.ordering.mc64(s)
    for i in range(5):
        assert sc[i] * abs(a[i, i]) * sc[i] <= 1.0 + 1e-10


@pytest.mark.parametrize("bad", [np.nan, np.inf])
def test_non_finite_rejected(rv, bad):
    a = upper(2, [(0, 0, 4.0), (0, 1, 1.0), (1, 1, 3.0)])
    s = system(rv, a)
    s.values[0] = bad
    with pytest.raises(rv.RvgError):
        rv.ordering.mc64(s)


def test_hand_constructed_fixtures(rv, golden):
    for name, g in golden.items():
        s = golden_system(rv, name, g)
        m, sc, k = rv.ordering.mc64(s)
        verify_properties(s, m, sc, k)
        a = s.to_scipy().toarray()
        if k == s.n:
            assert np.isclose(sum(-np.log(abs(a[i, m[i]])) for i in range(s.n)), optimal_log_product(a)), name


@pytest.mark.parametrize("seed", range(6))
def test_random_sparse_indefinite_optimal(rv, seed):
    rng = np.random.default_rng(seed)
    n = 80
    b = rng.standard_normal((n, n)) * (rng.random((n, n)) < 0.08)
    b = b + b.T + np.diag(rng.standard_normal(n) * (rng.random(n) < 0.5))
    b += np.diag(np.where(np.abs(b).sum(1) == 0, 1.0, 0.0))  # no empty rows
    s = system(rv, b)
    m, sc, k = rv.ordering.mc64(s)
    verify_properties(s, m, sc, k)
    if k == n:
        assert np.isclose(sum(-np.log(abs(b[i, m[i]])) for i in range(n)), optimal_log_product(b))


def test_kkt_and_laplacian_fully_matched(rv):
    for s in (rv.problems.kkt(8, seed=2), rv.problems.shifted_laplacian(10, 0.1)):
        m, sc, k = rv.ordering.mc64(s)
        assert k == s.n
        verify_properties(s, m, sc, k)
