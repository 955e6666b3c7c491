"""GPU numeric phase vs the oracle, through the C ABI.

The kernels and the oracle follow one arithmetic contract (fma chains where
the reference calls faer, unfused arithmetic elsewhere), so on the same
inputs the pivot record -- eliminated column order, 1x1/2x2 codes and the D
values -- must agree bit for bit, the inertia exactly, and the solution to
rounding (the GPU solve reassociates sibling updates; tolerance 1e-10
relative).  Backward error gates follow tests/solve.rs (<= 1e-14 on the
synthetic systems, < 1e-10 on the hand-constructed ones).
"""
import numpy as np
import pytest

from conftest import golden_system

pytestmark = pytest.mark.gpu

SOL_RTOL = 1e-10


LARGE = dict(large_front_threshold=33)  # forces the multi-kernel large-front path onto small fronts


def run_both(rv, orc, s, order=None, nrhs=1, seed=0, scaling=None, **opts):
    order = rv.ordering.default_order(s) if order is None else order
    solver = rv.SparseLDLT.analyze(s, rv.AnalyzeOptions(rv.OrderingStrategy.USER_SUPPLIED, order))
    if scaling is not None:
        solver._scaling = np.ascontiguousarray(scaling[solver.symbolic.perm_fwd])
    solver.factor(None, rv.FactorOptions(**opts))
    ref = orc.OracleFactor(s, solver.symbolic, solver._scaling, orc.options(**opts))
    b = rv.problems.rhs_uniform(s.n, seed, nrhs)
    return solver, ref, b


def assert_parity(rv, s, solver, ref, b, bwd=1e-14):
    assert solver.inertia() == ref.inertia()
    gs, os_ = solver.stats(), ref.stats()
    for k in ["total_1x1_pivots", "total_2x2_pivots", "total_delayed", "zero_pivots", "max_front_size",
              "supernodes_before_amalgamation", "supernodes_after_amalgamation", "merges_performed",
              "small_leaf_subtrees", "small_leaf_nodes"]:
        assert gs[k] == os_[k], (k, gs[k], os_[k])
    gf, of = solver.front_info(), ref.front_info()
    assert np.array_equal(gf[:, :8], of[:, :8])
    gc, gcode, gd, go = solver.pivot_record()
    oc, ocode, od, oo = ref.pivot_record()
    assert np.array_equal(gc, oc), "elimination order differs"
    assert np.array_equal(gcode, ocode), "pivot pattern differs"
    assert np.array_equal(gd, od) and np.array_equal(go, oo), "D differs"
    x = solver.solve(b)
    xr = ref.solve(b)
    assert np.linalg.norm(x - xr) <= SOL_RTOL * max(np.linalg.norm(xr), 1e-300)
    # the backward error gate, or (ill-conditioned cases) within 4x of the oracle's on the same factor:
    # the solve's sums run in another order than the oracle's, and the forward pass adds sibling
    # contributions atomically
    xs, xrs, bs = (x, xr, b) if b.ndim == 2 else (x[:, None], xr[:, None], b[:, None])
    for j in range(bs.shape[1]):
        e = rv.problems.backward_error(s, xs[:, j], bs[:, j])
        er = rv.problems.backward_error(s, xrs[:, j], bs[:, j])
        assert e <= max(bwd, 4 * er), (e, er)


@pytest.mark.parametrize("g,frac", [(4, 0.1), (8, 0.1), (12, 0.05), (16, 0.1), (20, 0.1)])
def test_shifted_laplacian(rv, orc, g, frac):
    s = rv.problems.shifted_laplacian(g, frac)
    solver, ref, b = run_both(rv, orc, s)
    assert solver.inertia() == s.inertia
    assert_parity(rv, s, solver, ref, b)


def test_hand_constructed(rv, orc, golden):
    for name, gd in golden.items():
        s = golden_system(rv, name, gd)
        solver, ref, b = run_both(rv, orc, s)
        assert solver.inertia() == tuple(gd["inertia"]), name
        xt = np.arange(1, s.n + 1, dtype=float)
        assert_parity(rv, s, solver, ref, s.to_scipy() @ xt, bwd=1e-10)


@pytest.mark.parametrize("g", [4, 6, 8])
def test_kkt(rv, orc, g):
    s = rv.problems.kkt(g, seed=g)
    solver, ref, b = run_both(rv, orc, s)
    assert solver.inertia() == s.inertia
    assert_parity(rv, s, solver, ref, b)


@pytest.mark.parametrize("opts", [dict(nemin=1), dict(small_leaf_threshold=0), dict(small_leaf_threshold=0, nemin=4),
                                  dict(threshold=0.5), dict(outer_block_size=64),
                                  dict(outer_block_size=32, small_leaf_threshold=0),
                                  dict(failed_pivot_tpp=False)])
def test_option_variants(rv, orc, opts):
    s = rv.problems.shifted_laplacian(12, 0.1)
    solver, ref, b = run_both(rv, orc, s, **opts)
    assert solver.inertia() == s.inertia
    assert_parity(rv, s, solver, ref, b, bwd=1e-12 if not opts.get("failed_pivot_tpp", True) else 1e-14)


def dense_system(rv, n, seed, kind):
    """Dense symmetric indefinite inputs in the spirit of the reference's torture
    mix (testing/perturbations.rs:22-51): delay-prone, singular and plain."""
    rng = np.random.default_rng(seed)
    a = rng.standard_normal((n, n))
    a = a + a.T
    if kind == "delay":
        a[np.arange(n), np.arange(n)] *= 1e-6
    elif kind == "singular":
        q = rng.standard_normal((n, n - 2))
        a = q @ np.diag(rng.choice([-1.0, 1.0], n - 2)) @ q.T
    return rv.problems.from_scipy(f"dense{n}_{kind}", a)


@pytest.mark.parametrize("n", [20, 32, 48, 64, 100, 128, 257, 300, 520])
@pytest.mark.parametrize("kind", ["plain", "delay", "singular"])
def test_dense_fronts(rv, orc, n, kind):
    s = dense_system(rv, n, n, kind)
    solver, ref, b = run_both(rv, orc, s)
    assert_parity(rv, s, solver, ref, b, bwd=1e-8 if kind == "singular" else 1e-13)


def test_multiple_rhs_and_refactor(rv, orc):
    s = rv.problems.shifted_laplacian(10, 0.1)
    solver, ref, b = run_both(rv, orc, s, nrhs=4)
    assert_parity(rv, s, solver, ref, b)
    # refactor with perturbed values, same pattern (solver.rs:335-341)
    rng = np.random.default_rng(3)
    s2 = rv.problems.System(s.name, s.n, s.colptr, s.rowidx, s.values * (1 + 0.01 * rng.standard_normal(s.values.size)))
    sv = s2.values.copy()
    # keep symmetry: average with the transpose pattern
    a = s2.to_scipy()
    a = (a + a.T) * 0.5
    s2 = rv.problems.from_scipy("perturbed", a)
    solver.refactor(s2.values)
    ref2 = orc.OracleFactor(s2, solver.symbolic)
    b1 = rv.problems.rhs_uniform(s.n, 1)
    assert_parity(rv, s2, solver, ref2, b1)
    del sv


@pytest.mark.parametrize("nrhs", [2, 3, 8, 13])
@pytest.mark.parametrize("large", [False, True])
def test_blocked_multi_rhs(rv, orc, nrhs, large):
    # right-hand sides go through the solve 8, 4, 2 or 1 at a time; each column must
    # match the oracle's solve and the single-RHS solve of the same factor
    s = rv.problems.kkt(8, seed=4)
    solver, ref, b = run_both(rv, orc, s, nrhs=nrhs, **(LARGE if large else {}))
    assert_parity(rv, s, solver, ref, b)
    x = solver.solve(b)
    for r in range(nrhs):
        xr = solver.solve(np.ascontiguousarray(b[:, r]))
        assert np.linalg.norm(x[:, r] - xr) <= SOL_RTOL * np.linalg.norm(xr)


@pytest.mark.parametrize("large", [False, True])
def test_mc64_scaled_factorization(rv, orc, large):
    # MatchOrderMetis: MC64 scaling in elimination order, applied inside the factorization
    for s in (rv.problems.shifted_laplacian(12, 0.1), rv.problems.kkt(8, seed=5)):
        solver = rv.SparseLDLT.analyze_with_matrix(s, rv.AnalyzeOptions(rv.OrderingStrategy.MATCH_ORDER_METIS))
        assert solver._scaling is not None
        solver.factor(None, rv.FactorOptions(**(LARGE if large else {})))
        ref = orc.OracleFactor(s, solver.symbolic, solver._scaling, orc.options())
        assert solver.inertia() == s.inertia
        assert_parity(rv, s, solver, ref, rv.problems.rhs_uniform(s.n, 0))


def test_scaling(rv, orc):
    s = rv.problems.shifted_laplacian(8, 0.1)
    sc = np.random.default_rng(7).uniform(0.5, 2.0, s.n)
    solver, ref, b = run_both(rv, orc, s, scaling=sc)
    assert solver.inertia() == s.inertia
    assert_parity(rv, s, solver, ref, b)


def test_errors(rv):
    s = rv.problems.shifted_laplacian(4, 0.1)
    solver = rv.SparseLDLT.analyze(s)
    solver.factor()
    with pytest.raises(rv.DimensionMismatch):
        solver.solve(np.ones(s.n + 1))
    with pytest.raises(rv.DimensionMismatch):
        solver.factor(np.ones(3))


# ---- the multi-kernel large-front path, forced onto small fronts ----------


@pytest.mark.parametrize("n", [48, 100, 257, 300, 520, 700])
@pytest.mark.parametrize("kind", ["plain", "delay", "singular"])
def test_large_front_path_dense(rv, orc, n, kind):
    s = dense_system(rv, n, n + 1, kind)
    solver, ref, b = run_both(rv, orc, s, **LARGE)
    assert_parity(rv, s, solver, ref, b, bwd=1e-8 if kind == "singular" else 1e-13)


@pytest.mark.parametrize("opts", [dict(), dict(outer_block_size=64), dict(outer_block_size=32),
                                  dict(small_leaf_threshold=0, nemin=8)])
def test_large_front_path_sparse(rv, orc, opts):
    o = dict(LARGE)
    o.update(opts)
    for s in (rv.problems.shifted_laplacian(14, 0.1), rv.problems.kkt(7, seed=3)):
        solver, ref, b = run_both(rv, orc, s, **o)
        assert solver.inertia() == s.inertia
        assert_parity(rv, s, solver, ref, b)


@pytest.mark.parametrize("n,nb", [(1400, 256), (700, 64), (600, 96), (520, 128)])
@pytest.mark.parametrize("kind", ["plain", "delay"])
def test_large_front_window(rv, orc, n, nb, kind):
    # deferred far-field updates: windows of four outer blocks, applied when
    # full or as soon as a block delays columns; bit-identical to per-block updates
    s = dense_system(rv, n, n + 2, kind)
    solver, ref, b = run_both(rv, orc, s, large_front_threshold=33, outer_block_size=nb)
    assert_parity(rv, s, solver, ref, b)


def test_large_front_path_nfs_gemm(rv, orc):
    # fronts with >= 256 NFS rows take the syrk contribution GEMM
    s = rv.problems.kkt(10, seed=1)
    solver, ref, b = run_both(rv, orc, s, large_front_threshold=300)
    assert solver.inertia() == s.inertia
    assert_parity(rv, s, solver, ref, b)


@pytest.mark.parametrize("case", ["one_pos", "one_neg", "zero2", "zero40", "diag100", "offdiag_only"])
def test_edge_cases(rv, orc, case):
    # tiny, zero and structurally trivial matrices: the same pivots, D and inertia as the oracle
    import scipy.sparse as sp
    if case == "one_pos":
        a = sp.csc_matrix(np.array([[4.0]]))
    elif case == "one_neg":
        a = sp.csc_matrix(np.array([[-2.5]]))
    elif case == "zero2":
        a = sp.csc_matrix((np.zeros(4), (np.array([0, 1, 0, 1]), np.array([0, 0, 1, 1]))), shape=(2, 2))
    elif case == "zero40":
        i = np.arange(40)
        a = sp.csc_matrix((np.zeros(40), (i, i)), shape=(40, 40)) + sp.csc_matrix(
            (np.zeros(39), (i[1:], i[:-1])), shape=(40, 40))
        a = a + a.T
    elif case == "diag100":
        d = np.random.default_rng(1).standard_normal(100)
        a = sp.diags(d).tocsc()
    else:
        # pure 2x2 coupling, zero diagonal: every pivot a 2x2 block
        n = 30
        r = np.arange(0, n, 2)
        a = sp.csc_matrix((np.ones(n // 2), (r, r + 1)), shape=(n, n))
        a = a + a.T
    s = rv.problems.from_scipy(case, a)
    solver, ref, b = run_both(rv, orc, s)
    assert_parity(rv, s, solver, ref, b)
    solver.close()


def test_empty_system(rv):
    import scipy.sparse as sp
    s = rv.problems.from_scipy("empty", sp.csc_matrix((0, 0)))
    solver = rv.SparseLDLT.analyze(s)
    solver.factor()
    x = solver.solve(np.zeros(0))
    assert x.shape == (0,)
    assert solver.inertia() == (0, 0, 0)
    solver.close()
