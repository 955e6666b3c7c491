"""Mixed form: the large Schur-complement updates on the TF32 tensor cores
(tcgen05, operands split hi + lo), everything else FP64, then FP64 iterative
refinement (rvg_solve_refine).

The mixed factor is not bit-identical to the oracle (its products are rounded
differently), so the gates are the ones the solution must meet: exact
inertia where it is known, and a scaled backward error <= 1e-14 after at most
10 corrections; the plain form must reach it with at most one correction.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# force the multi-kernel large-front path (and with it the Schur GEMM) onto small fronts
SMALL_LARGE = dict(large_front_threshold=64)


def factor_refine(rv, s, b, **opts):
    solver = rv.SparseLDLT.analyze(s)
    solver.factor(None, rv.FactorOptions(**opts))
    x, iters, err = solver.solve_refine(b, tol=1e-14, max_iter=10)
    inertia = solver.inertia()
    solver.close()
    return x, iters, err, inertia


@pytest.mark.parametrize("name", ["lap", "kkt", "dense"])
def test_mixed_reaches_fp64_accuracy(rv, name):
    if name == "lap":
        s = rv.problems.shifted_laplacian(16, 0.1)
    elif name == "kkt":
        s = rv.problems.kkt(12, seed=2)
    else:
        rng = np.random.default_rng(5)
        a = rng.standard_normal((700, 700))
        a = a + a.T + np.diag(np.full(700, 60.0))
        import scipy.sparse as sp
        s = rv.problems.from_scipy("dense700", sp.csc_matrix(a))
    b = rv.problems.rhs_normal(s.n, 3)
    for precision, flush in (("fp64", 2), ("mixed", 1), ("mixed", 2), ("mixed", 8), ("mixed", 0)):
        x, iters, err, inertia = factor_refine(rv, s, b, precision=precision, mixed_flush=flush, **SMALL_LARGE)
        assert err <= 1e-14, (precision, flush, err, iters)
        assert rv.problems.backward_error(s, x, b) <= 1e-14
        if s.inertia is not None:
            assert inertia == s.inertia
        if precision == "fp64":
            assert iters <= 1


@pytest.mark.parametrize("n,nb,kind", [(1400, 256, "plain"), (1400, 256, "delay"), (900, 128, "plain"),
                                       (700, 64, "delay")])
def test_mixed_window(rv, n, nb, kind):
    # the mixed form's packed window of pending columns (flushed every four outer
    # blocks, or at once after a delay; one block when nb is not a multiple of 128)
    import scipy.sparse as sp
    rng = np.random.default_rng(n + nb)
    a = rng.standard_normal((n, n))
    a = a + a.T
    if kind == "delay":
        a[np.arange(n), np.arange(n)] *= 1e-6
    s = rv.problems.from_scipy(f"dense{n}", sp.csc_matrix(a))
    b = rv.problems.rhs_normal(s.n, 4)
    for flush in (4, 0):
        x, iters, err, inertia = factor_refine(rv, s, b, precision="mixed", mixed_flush=flush,
                                               large_front_threshold=33, outer_block_size=nb)
        assert err <= 1e-14, (flush, err, iters)
        assert rv.problems.backward_error(s, x, b) <= 1e-14
    xp, _, _, inertia_p = factor_refine(rv, s, b, precision="fp64", large_front_threshold=33, outer_block_size=nb)
    assert inertia == inertia_p


def test_refine_errors(rv):
    s = rv.problems.shifted_laplacian(4, 0.1)
    solver = rv.SparseLDLT.analyze(s)
    with pytest.raises(rv.SolveBeforeFactor):
        solver.solve_refine(np.ones(s.n))
    solver.factor()
    with pytest.raises(rv.DimensionMismatch):
        solver.solve_refine(np.ones(s.n + 2))
    with pytest.raises(rv.InvalidInput):
        solver.factor(None, rv.FactorOptions(precision="fp64", threshold=2.0))
    with pytest.raises(rv.InvalidInput):
        solver.factor(None, rv.FactorOptions(precision="mixed", mixed_flush=3))


@pytest.mark.parametrize("case", ["kkt", "dense_plain", "dense_delay", "dense_nb64"])
def test_pair_tiles_bit_identical(rv, case):
    # the no-flush Schur GEMM over 256-column CTA tiles (two 128-column tiles
    # sharing the W tile) gives the same factor, bit for bit, as 128-column tiles
    import scipy.sparse as sp
    opts = dict(precision="mixed", mixed_flush=0)
    if case == "kkt":
        s = rv.problems.kkt(14, seed=4)
        opts.update(large_front_threshold=64)
    else:
        n = 1500 if case != "dense_nb64" else 900
        rng = np.random.default_rng(len(case))
        a = rng.standard_normal((n, n))
        a = a + a.T
        if case == "dense_delay":
            a[np.arange(n), np.arange(n)] *= 1e-6
        s = rv.problems.from_scipy(case, sp.csc_matrix(a))
        opts.update(large_front_threshold=33, outer_block_size=64 if case == "dense_nb64" else 256)
    b = rv.problems.rhs_normal(s.n, 6)
    out = []
    for cols in (128, 256):
        solver = rv.SparseLDLT.analyze(s)
        solver.factor(None, rv.FactorOptions(mixed_tile_cols=cols, **opts))
        out.append((solver.pivot_record(), solver.inertia(), solver.solve(b)))
        solver.close()
    (c0, k0, d0, o0), i0, x0 = out[0]
    (c1, k1, d1, o1), i1, x1 = out[1]
    assert i0 == i1
    assert np.array_equal(c0, c1) and np.array_equal(k0, k1)
    assert np.array_equal(d0, d1) and np.array_equal(o0, o1), "D differs"
    # the solve adds sibling contributions with atomics: equal to rounding
    assert np.linalg.norm(x0 - x1) <= 1e-13 * np.linalg.norm(x0)


def test_pair_tiles_option_checked(rv):
    s = rv.problems.shifted_laplacian(4, 0.1)
    solver = rv.SparseLDLT.analyze(s)
    with pytest.raises(rv.InvalidInput):
        solver.factor(None, rv.FactorOptions(precision="mixed", mixed_tile_cols=192))
