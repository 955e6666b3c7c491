"""The oracle (CPU restatement of the reference numeric phase) pinned against
the reference's own fixtures and known answers:

* exact inertia of the 15 hand-constructed matrices
  (sparse/test-data/hand-constructed/*.json; tests/solve.rs:210-246),
* backward error < 1e-10 with x = 1..n (tests/solve.rs:159-206),
* dense-kernel known answers (sparse/src/symmetric/factor.rs tests),
* closed-form inertia of shifted Laplacians and KKT systems,
* nemin 1 vs 32 backward error < 1e-14 (tests/solve.rs:1517-1560).
"""
import numpy as np
import pytest

from conftest import golden_system

SOLVE_FULL_CASES = ["arrow-5-pd", "tridiag-5-pd", "trivial-1x1", "trivial-2x2", "block-diag-15",
                    "stress-delayed-pivots", "arrow-10-indef", "tridiag-10-indef", "zero-diagonal-3", "singular-3",
                    "bordered-block-20"]


def oracle_factor(rv, orc, sysm, order=None, **opts):
    order = rv.ordering.default_order(sysm) if order is None else order
    sym = rv.symbolic_analyze(sysm.n, sysm.colptr, sysm.rowidx, order)
    return orc.OracleFactor(sysm, sym, None, orc.options(**opts)), sym


def test_hand_constructed_inertia(rv, orc, golden):
    for name, g in golden.items():
        s = golden_system(rv, name, g)
        f, _ = oracle_factor(rv, orc, s)
        assert f.inertia() == tuple(g["inertia"]), name


@pytest.mark.parametrize("name", SOLVE_FULL_CASES)
def test_hand_constructed_backward_error(rv, orc, golden, name):
    s = golden_system(rv, name, golden[name])
    f, _ = oracle_factor(rv, orc, s)
    xt = np.arange(1, s.n + 1, dtype=float)
    b = s.to_scipy() @ xt
    x = f.solve(b)
    assert rv.problems.backward_error(s, x, b) < 1e-10


def test_reference_inertia_cases(rv, orc, golden):
    for name, pos, neg in [("arrow-5-pd", 5, 0), ("tridiag-5-pd", 5, 0), ("trivial-1x1", 1, 0),
                           ("trivial-2x2", 1, 1)]:
        f, _ = oracle_factor(rv, orc, golden_system(rv, name, golden[name]))
        assert f.inertia()[:2] == (pos, neg)


def test_pd_cases_have_no_2x2_or_delays(rv, orc):
    # multifrontal.rs asserts 0 2x2 and 0 delays on PD inputs (tests/multifrontal.rs:204-205)
    import scipy.sparse as sp
    for g in (4, 7):
        a = rv.problems.laplacian_7pt(g)
        s = rv.problems.from_scipy("pd", a)
        f, _ = oracle_factor(rv, orc, s, small_leaf_threshold=0)
        st = f.stats()
        assert st["total_delayed"] == 0
        assert f.inertia() == (s.n, 0, 0)


# ---- dense kernel known answers (factor.rs tests) -------------------------
def sym(n, f):
    return np.array([[f(max(i, j), min(i, j)) for j in range(n)] for i in range(n)], dtype=float)


def reconstruct(a_fact, perm, dt, dd, do, ne):
    n = a_fact.shape[0]
    L = np.eye(n)
    D = np.zeros((n, n))
    c = 0
    while c < ne:
        if dt[c] == 1:
            L[c + 1:, c] = a_fact[c + 1:, c]
            D[c, c] = dd[c]
            c += 1
        else:
            L[c + 2:, c] = a_fact[c + 2:, c]
            L[c + 2:, c + 1] = a_fact[c + 2:, c + 1]
            D[c, c], D[c + 1, c + 1], D[c, c + 1], D[c + 1, c] = dd[c], dd[c + 1], do[c], do[c]
            c += 2
    M = L[:, :ne] @ D[:ne, :ne] @ L[:, :ne].T
    out = np.zeros((n, n))
    out[np.ix_(perm, perm)] = M
    return out


@pytest.mark.parametrize("n", [1, 2, 3, 5, 8, 16, 32, 33, 64, 100, 128, 300])
def test_dense_reconstruction(orc, n):
    rng = np.random.default_rng(n)
    a = rng.standard_normal((n, n))
    a = a + a.T
    af, perm, dt, dd, do, st, _ = orc.dense_aptp(a)
    ne = st[0]
    assert st[1] + 2 * st[2] + st[3] == n
    if ne == n:
        r = reconstruct(af, perm, dt, dd, do, ne)
        assert np.linalg.norm(r - a) / np.linalg.norm(a) < 5e-11


def test_dense_known_counts(orc):
    # test_1x1_trivial_diagonal / test_1x1_positive_definite_3x3 / test_1x1_matrix / statistics invariant
    _, _, _, _, _, st, _ = orc.dense_aptp(np.diag([4.0, 9.0]))
    assert st[3] == 0 and st[1] + 2 * st[2] == 2
    _, _, _, _, _, st, _ = orc.dense_aptp(np.array([[4, 2, 1], [2, 5, 3], [1, 3, 6.0]]))
    assert st[3] == 0 and st[1] + 2 * st[2] == 3
    _, _, _, _, _, st, _ = orc.dense_aptp(np.array([[5.0]]))
    assert st[1] == 1 and st[3] == 0
    a = sym(5, lambda i, j: [[10, 1, 0, 0, 0], [1, 20, 2, 0, 0], [0, 2, 30, 3, 0], [0, 0, 3, 40, 4],
                             [0, 0, 0, 4, 50]][i][j])
    _, _, _, _, _, st, _ = orc.dense_aptp(a)
    assert st[1] + 2 * st[2] + st[3] == 5
    # zero matrix: TPP records zero pivots (test_all_delayed_zero_matrix)
    _, _, dt, dd, _, st, _ = orc.dense_aptp(np.zeros((4, 4)), opts=orc.options(failed_pivot_tpp=False))
    assert st[1] + 2 * st[2] + st[3] == 4
    # 2x2 complete-pivoting case with a 40x40 embedding so the blocked path runs
    b = np.eye(40) * 3.0
    b[0, 0] = b[1, 1] = 0.1
    b[0, 1] = b[1, 0] = 10.0
    _, _, dt, _, _, st, ml = orc.dense_aptp(b)
    assert st[2] >= 1 and ml <= 4 + 1e-10


@pytest.mark.parametrize("m,p", [(64, 32), (128, 48), (100, 50), (300, 280), (520, 300)])
def test_dense_partial_factorization(orc, m, p):
    # factor.rs:5377-5727: partial factorization; FS columns eliminated with
    # the Schur complement left in the trailing block
    rng = np.random.default_rng(m * 7 + p)
    a = rng.standard_normal((m, m))
    a = a + a.T + np.diag(rng.uniform(-4, 4, m))
    af, perm, dt, dd, do, st, _ = orc.dense_aptp(a, p=p)
    assert st[1] + 2 * st[2] + st[3] == p


# ---- closed-form inertia ---------------------------------------------------
@pytest.mark.parametrize("g,frac", [(4, 0.1), (8, 0.1), (10, 0.05), (16, 0.1)])
def test_shifted_laplacian_inertia(rv, orc, g, frac):
    s = rv.problems.shifted_laplacian(g, frac)
    f, _ = oracle_factor(rv, orc, s)
    assert f.inertia() == s.inertia
    b = rv.problems.rhs_uniform(s.n, 0)
    assert rv.problems.backward_error(s, f.solve(b), b) <= 1e-14


@pytest.mark.parametrize("g", [4, 6])
def test_kkt_inertia(rv, orc, g):
    s = rv.problems.kkt(g, seed=g)
    f, _ = oracle_factor(rv, orc, s)
    assert f.inertia() == s.inertia
    b = rv.problems.rhs_normal(s.n, 0)
    assert rv.problems.backward_error(s, f.solve(b), b) <= 1e-14


def test_nemin_and_small_leaf_equivalence(rv, orc):
    s = rv.problems.shifted_laplacian(10, 0.1)
    b = rv.problems.rhs_uniform(s.n, 0)
    for opts in [dict(nemin=1), dict(nemin=32), dict(small_leaf_threshold=0), dict(small_leaf_threshold=256)]:
        f, _ = oracle_factor(rv, orc, s, **opts)
        assert f.inertia() == s.inertia
        assert rv.problems.backward_error(s, f.solve(b), b) < 1e-14


# ---- torture mix for the dense kernel (factor.rs:6862-6960; generators of testing/perturbations.rs) ----
def _indefinite_dominant(m, rng):
    """Random symmetric entries in [-1, 1) with a diagonal that dominates its
    row, positive in the first half of the rows and negative in the rest."""
    a = rng.uniform(-1.0, 1.0, (m, m))
    a = np.tril(a) + np.tril(a, -1).T
    off = np.abs(a).sum(1) - np.abs(np.diag(a))
    margin = 1.0 + rng.uniform(0.0, 1.0, m)
    sign = np.where(np.arange(m) < m // 2, 1.0, -1.0)
    a[np.arange(m), np.arange(m)] = sign * (off + margin)
    return a


def _cause_delays(a, ib, rng):
    """n/8 rows (with their columns) and n/8 single symmetric entries scaled by
    1000; the first scaled row lies past the first inner block."""
    m = a.shape[0]
    if m < 8:
        return
    for t in range(m // 8):
        r = ib + int(rng.integers(0, m - ib)) if (t == 0 and m > ib) else int(rng.integers(0, m))
        a[r, :] *= 1000.0
        a[:, r] *= 1000.0
        a[r, r] /= 1000.0
    for _ in range(m // 8):
        i, j = int(rng.integers(0, m)), int(rng.integers(0, m))
        a[i, j] *= 1000.0
        if i != j:
            a[j, i] *= 1000.0


def _make_singular(a, c1, c2, scale=2.0):
    """Column (and row) c2 becomes scale times column c1: rank drops by one."""
    d1 = a[c1, c1]
    col = a[:, c1].copy()
    a[:, c2] = scale * col
    a[c2, :] = scale * col
    a[c2, c1] = a[c1, c2] = scale * d1
    a[c2, c2] = scale * scale * d1


@pytest.mark.parametrize("m,n", [(32, 32), (64, 64), (128, 128), (128, 48)])
def test_dense_torture_mix(orc, m, n):
    """70% delay-inducing, 20% singular, 10% singular-diagonal-block instances
    (SPRAL's mix, as the reference's torture tests use it): every instance
    accounts for all n fully-summed columns, and square non-singular ones that
    are fully eliminated reconstruct to 5e-11."""
    rng = np.random.default_rng(12345 + m + n)
    ib = min(32, n)
    opts = orc.options(inner_block_size=ib)
    failures = []
    for inst in range(150):
        a = _indefinite_dominant(m, rng)
        roll = rng.uniform()
        singular = True
        if roll < 0.70:
            _cause_delays(a, ib, rng)
            singular = False
        elif roll < 0.90:
            c1 = int(rng.integers(0, m))
            c2 = int(rng.integers(0, m - 1))
            c2 += c2 >= c1
            _make_singular(a, c1, c2)
        else:
            b = int(rng.integers(0, m - ib + 1))
            _make_singular(a, b, b + ib - 1)
        af, perm, dt, dd, do, st, _ = orc.dense_aptp(a.copy(), p=n, opts=opts)
        if st[1] + 2 * st[2] + st[3] != n:
            failures.append((inst, "count", tuple(st)))
            continue
        if m == n and not singular and st[0] == n:
            err = np.linalg.norm(reconstruct(af, perm, dt, dd, do, st[0]) - a) / np.linalg.norm(a)
            if err > 5e-11:
                failures.append((inst, "recon", err))
    assert not failures, failures[:5]


@pytest.mark.parametrize("kind", ["lap", "kkt", "dense"])
def test_thread_count_invariance(rv, orc, kind):
    """The oracle's OpenMP blocking reorders only independent output entries:
    its pivot record, D and statistics are the same for any thread count."""
    if kind == "lap":
        s = rv.problems.shifted_laplacian(20, 0.1)
    elif kind == "kkt":
        s = rv.problems.kkt(14, seed=2)
    else:
        rng = np.random.default_rng(9)
        a = rng.standard_normal((700, 700))
        a = a + a.T
        a[np.arange(700), np.arange(700)] *= 1e-3
        s = rv.problems.from_scipy("dense700", a)
    sym = rv.symbolic_analyze(s.n, s.colptr, s.rowidx, rv.ordering.default_order(s))
    recs = []
    for nt in (1, 3, 8):
        f = orc.OracleFactor(s, sym, None, orc.options(), nthreads=nt)
        recs.append((f.pivot_record(), f.stats(), f.inertia()))
        f.close()
    for (p, st, ine) in recs[1:]:
        for x, y in zip(p, recs[0][0]):
            assert np.array_equal(x, y)
        assert st == recs[0][1] and ine == recs[0][2]


def test_cpu_only_analysis_matches_library(rv, orc):
    """The oracle's analysis library (the library's host analysis sources
    without the CUDA numeric phase) gives the same symbolic structure and
    MC64 scaling as the library itself, so a CPU-only run factors the same
    fronts as the GPU path."""
    for s in (rv.problems.kkt(10, seed=3), rv.problems.shifted_laplacian(12, 0.1)):
        solver = rv.SparseLDLT.analyze_with_matrix(s, rv.AnalyzeOptions(rv.OrderingStrategy.MATCH_ORDER_METIS))
        sym, sc = orc.analyze(s, rv.ordering.default_order(s), mc64=True)
        a = solver.symbolic
        for f in ("perm_fwd", "sup_begin", "sup_end", "sup_parent", "pat_ptr", "pat_idx"):
            assert np.array_equal(getattr(a, f), getattr(sym, f)), f
        assert np.array_equal(solver._scaling, sc)


def test_sliced_factorization_is_the_same(rv, orc):
    """The factorization run in slices (the timed CPU reference: a worker that
    stops at checkpoints between fronts and outer blocks) gives the same
    pivot record and statistics as one uninterrupted run."""
    s = rv.problems.kkt(16, seed=5)
    sym, sc = orc.analyze(s, rv.ordering.default_order(s), mc64=True)
    ref = orc.OracleFactor(s, sym, sc, orc.options(), nthreads=4)
    ses = orc.OracleFactor(s, sym, sc, orc.options(), nthreads=4, sliced=True)
    tot = ses.total_flops()
    ends = [ses.advance(tot * (i + 1) / 5) for i in range(4)]
    assert not any(ends)
    ses.finish()
    for x, y in zip(ref.pivot_record(), ses.pivot_record()):
        assert np.array_equal(x, y)
    assert ref.stats() == ses.stats()
    b = rv.problems.rhs_normal(s.n, 0)
    assert np.array_equal(ref.solve(b), ses.solve(b))


def test_sliced_factorization_abort(rv, orc):
    """A sliced run closed before its end stops at its checkpoint instead of
    running the rest."""
    import time
    s = rv.problems.kkt(16, seed=5)
    sym, sc = orc.analyze(s, rv.ordering.default_order(s), mc64=True)
    ses = orc.OracleFactor(s, sym, sc, orc.options(), nthreads=2, sliced=True)
    ses.advance(ses.total_flops() * 0.01)
    t0 = time.perf_counter()
    ses.close()
    assert ses.session is None and ses.h is None
    full = orc.OracleFactor(s, sym, sc, orc.options(), nthreads=2)
    assert full.inertia() == s.inertia
    assert time.perf_counter() - t0 < 60
