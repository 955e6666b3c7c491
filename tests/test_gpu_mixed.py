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
    for precision, flush, ops in (("fp64", 2, "tf32"), ("mixed", 1, "tf32"), ("mixed", 2, "tf32"), ("mixed", 8, "tf32"),
                                  ("mixed", 0, "tf32"), ("mixed", 4, "bf16"), ("mixed", 0, "bf16")):
        x, iters, err, inertia = factor_refine(rv, s, b, precision=precision, mixed_flush=flush, mixed_operands=ops,
                                               **SMALL_LARGE)
        assert err <= 1e-14, (precision, flush, ops, err, iters)
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
    # (TF32 parts only: these random dense matrices are too ill-conditioned for plain refinement
    # of a BF16-split factor)
    for flush, ops in ((4, "tf32"), (0, "tf32")):
        x, iters, err, inertia = factor_refine(rv, s, b, precision="mixed", mixed_flush=flush, mixed_operands=ops,
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


@pytest.mark.parametrize("ops", ["tf32", "bf16"])
@pytest.mark.parametrize("case", ["kkt", "dense_plain", "dense_delay", "dense_nb64"])
def test_pair_tiles_bit_identical(rv, case, ops):
    # the no-flush Schur GEMM over 256-column CTA tiles (two 128-column tiles
    # sharing the W tile) gives the same factor, bit for bit, as 128-column tiles
    import scipy.sparse as sp
    opts = dict(precision="mixed", mixed_flush=0, mixed_operands=ops)
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


def test_bf16_parts_are_less_accurate_but_refine(rv):
    # the BF16 split keeps about 16 bits per product against 22 for TF32: a larger
    # first residual, and the refinement still ends at the FP64 target
    import scipy.sparse as sp
    rng = np.random.default_rng(11)
    n = 1200
    a = rng.standard_normal((n, n))
    a = a + a.T + np.diag(np.full(n, 4.0 * np.sqrt(n)))
    s = rv.problems.from_scipy("dense1200", sp.csc_matrix(a))
    b = rv.problems.rhs_normal(n, 2)
    first = {}
    for ops in ("tf32", "bf16"):
        solver = rv.SparseLDLT.analyze(s)
        solver.factor(None, rv.FactorOptions(precision="mixed", mixed_flush=4, mixed_operands=ops,
                                             large_front_threshold=33))
        x0 = solver.solve(b)
        first[ops] = rv.problems.backward_error(s, x0, b)
        x, iters, err = solver.solve_refine(b, tol=1e-14, max_iter=10)
        assert err <= 1e-14, (ops, err, iters)
        solver.close()
    assert first["bf16"] > first["tf32"]
    assert first["bf16"] < 1e-3


@pytest.mark.parametrize("ops", ["tf32", "bf16"])
def test_refine_several_rhs(rv, ops):
    # blocked refinement of 5 right-hand sides: every column reaches the target, and each
    # agrees with the one-column refinement of the same factor (to the forward error a
    # backward error of 1e-14 allows on this matrix)
    s = rv.problems.kkt(12, seed=3)
    b = rv.problems.rhs_normal(s.n, 9, 5)
    solver = rv.SparseLDLT.analyze(s)
    solver.factor(None, rv.FactorOptions(precision="mixed", mixed_flush=0, mixed_operands=ops,
                                         large_front_threshold=64))
    x, iters, errs = solver.solve_refine(b, tol=1e-14, max_iter=10)
    assert x.shape == b.shape and errs.shape == (5,)
    assert (errs <= 1e-14).all(), errs
    for j in range(5):
        assert rv.problems.backward_error(s, x[:, j], b[:, j]) <= 1e-14
        x1, _, _ = solver.solve_refine(b[:, j].copy(), tol=1e-14, max_iter=10)
        assert np.linalg.norm(x[:, j] - x1) <= 1e-8 * np.linalg.norm(x1)
    solver.close()


@pytest.mark.parametrize("ops,flush", [("tf32", 0), ("bf16", 0), ("bf16", 4)])
def test_gmres_ir_where_refinement_stalls(rv, ops, flush):
    # a random dense indefinite matrix (ill-conditioned): GMRES-IR with the mixed factor as
    # preconditioner reaches the FP64 target for both operand splits
    import scipy.sparse as sp
    n = 900
    rng = np.random.default_rng(n + 128)
    a = rng.standard_normal((n, n))
    a = a + a.T
    s = rv.problems.from_scipy("dense900", sp.csc_matrix(a))
    b = rv.problems.rhs_normal(n, 4)
    solver = rv.SparseLDLT.analyze(s)
    solver.factor(None, rv.FactorOptions(precision="mixed", mixed_flush=flush, mixed_operands=ops,
                                         large_front_threshold=33, outer_block_size=128))
    x, its, err = solver.solve_gmres(b, tol=1e-14, max_iter=200, restart=30)
    assert err <= 1e-14, (ops, flush, err, its)
    assert rv.problems.backward_error(s, x, b) <= 1e-14
    solver.close()


def test_gmres_ir_on_kkt_and_errors(rv):
    s = rv.problems.kkt(10, seed=5)
    b = rv.problems.rhs_normal(s.n, 7)
    solver = rv.SparseLDLT.analyze(s)
    with pytest.raises(rv.SolveBeforeFactor):
        solver.solve_gmres(b)
    solver.factor(None, rv.FactorOptions(precision="mixed", mixed_flush=0, mixed_operands="bf16",
                                         large_front_threshold=64))
    x, its, err = solver.solve_gmres(b, tol=1e-14, restart=5)
    assert err <= 1e-14 and its >= 1
    assert rv.problems.backward_error(s, x, b) <= 1e-14
    with pytest.raises(rv.InvalidInput):
        solver.solve_gmres(b, restart=0)
    solver.close()


def test_auto_refinement_escalates_only_when_needed(rv):
    import scipy.sparse as sp
    # well conditioned: refinement alone
    s = rv.problems.kkt(10, seed=6)
    b = rv.problems.rhs_normal(s.n, 3)
    solver = rv.SparseLDLT.analyze(s)
    solver.factor(None, rv.FactorOptions(precision="mixed", mixed_flush=4, large_front_threshold=64))
    x, its, err, how = solver.solve_auto(b)
    assert err <= 1e-14 and how == "ir"
    solver.close()
    # ill conditioned with a BF16-split factor: refinement stalls, GMRES-IR finishes
    n = 900
    rng = np.random.default_rng(n + 128)
    a = rng.standard_normal((n, n))
    a = a + a.T
    s = rv.problems.from_scipy("dense900", sp.csc_matrix(a))
    b = rv.problems.rhs_normal(n, 4)
    solver = rv.SparseLDLT.analyze(s)
    solver.factor(None, rv.FactorOptions(precision="mixed", mixed_flush=0, mixed_operands="bf16",
                                         large_front_threshold=33, outer_block_size=128))
    x, its, err, how = solver.solve_auto(b, max_iter=200)
    assert err <= 1e-14 and how == "gmres", (err, its, how)
    assert rv.problems.backward_error(s, x, b) <= 1e-14
    solver.close()


@pytest.mark.parametrize("case,window", [("dense_delay", 0), ("kkt26", 0), ("dense_delay", 8), ("kkt26", 8)])
def test_far_field_overlap_is_bit_identical(rv, case, window):
    """A full window's far-field update runs on a second stream beside the next window's outer blocks but
    its last (three at the default depth, seven at eight), and a delayed block's far-field update and swap
    wait until the host has seen the delay; the factor equals the one-block-at-a-time schedule of the
    profiling mode (no second stream) bit for bit."""
    import numpy as np
    if case == "dense_delay":
        # order 4000 at the default depth; at eight blocks the far part of the first full window (from column
        # 2048 + 7 * 256) needs more trailing columns
        n = 4000 if window == 0 else 6000
        rng = np.random.default_rng(4000)
        a = rng.standard_normal((n, n))
        a = a + a.T
        weak = np.arange(2050, 2114)  # rows and columns scaled down: their block's pivots fail the threshold test
        a[weak, :] *= 1e-3
        a[:, weak] *= 1e-3
        s = rv.problems.from_scipy(f"dense{n}_delay", a)
        opts = rv.FactorOptions(precision="mixed", mixed_flush=0, mixed_operands="bf16", large_front_threshold=33,
                                mixed_window=window)
        solver = rv.SparseLDLT.analyze(s)
    else:
        s = rv.problems.kkt(26, seed=26)
        opts = rv.FactorOptions(precision="mixed", mixed_flush=0, mixed_operands="bf16", mixed_window=window)
        solver = rv.SparseLDLT.analyze_with_matrix(s, rv.AnalyzeOptions(rv.OrderingStrategy.MATCH_ORDER_METIS))
    solver.factor(None, opts)
    far = solver.profile()["lf_far_updates"]
    got = [x.copy() for x in solver.pivot_record()]
    st = solver.stats()
    assert far > 0
    if case == "dense_delay":  # outer blocks delayed columns after full windows had gone to the far stream
        assert solver.profile()["lf_misses"] > 0
    solver.set_profiling(True)
    solver.factor(None, opts)
    assert solver.profile()["lf_far_updates"] == 0
    ref = solver.pivot_record()
    assert all(np.array_equal(x, y) for x, y in zip(got, ref))
    assert solver.stats() == st
    solver.set_profiling(False)
    if case == "kkt26":
        b = rv.problems.rhs_normal(s.n, 3)
        x, its, err, how = solver.solve_auto(b)
        assert err <= 1e-14 and solver.inertia() == s.inertia
    solver.close()


@pytest.mark.parametrize("window", [1, 2, 8])
def test_window_depth_option(rv, window):
    """mixed_window changes how many outer blocks of updates are deferred (and
    so the FP32 partial sums' length): every depth reaches 1e-14 after
    refinement with the exact inertia, with and without the far-field split,
    on a KKT whose large fronts span several full windows."""
    s = rv.problems.kkt(26, seed=4)
    b = rv.problems.rhs_normal(s.n, 6)
    solver = rv.SparseLDLT.analyze_with_matrix(s, rv.AnalyzeOptions(rv.OrderingStrategy.MATCH_ORDER_METIS))
    for far in (-1, 0):
        solver.factor(None, rv.FactorOptions(precision="mixed", mixed_flush=0, mixed_operands="bf16",
                                             large_front_threshold=512, mixed_window=window, far_field_sms=far))
        assert tuple(solver.inertia()) == tuple(s.inertia)
        x, its, err, how = solver.solve_auto(b)
        assert err <= 1e-14 and rv.problems.backward_error(s, x, b) <= 1e-14, (window, far, its, how)
    solver.close()
