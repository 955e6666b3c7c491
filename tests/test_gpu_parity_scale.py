"""GPU numeric phase vs the oracle at the sizes where the production path runs,
with default options.

The parity tests in test_gpu_parity.py force the multi-kernel large-front path
onto small fronts.  Here nothing is forced: fronts of order >= 2048 (and of at
least 1024 in waves that hold few of them) take the large-front path on their
own, several large fronts of a wave run concurrently on their own streams,
outer blocks fill the 1024-column window of deferred far-field updates, and
the medium fronts of every wave go through the persistent work-queue launch.
The gates are those of the reference's own seq/par comparison
(tests/solve.rs:1105-1185): the same elimination order, 1x1/2x2 codes, D,
delayed count, inertia and statistics bit for bit, the solution to 1e-10
relative and the scaled backward error <= 1e-14.

The oracle runs with several threads here: its blocking reorders only
independent entries, so its results do not depend on the thread count
(tests/test_oracle.py::test_thread_count_invariance).
"""
import os

import numpy as np
import pytest
import scipy.sparse as sp

from test_gpu_parity import assert_parity

pytestmark = pytest.mark.gpu

THREADS = max(1, min(16, os.cpu_count() or 1))


def analyze_mc64(rv, s):
    # MatchOrderMetis, the reference's default strategy (solver.rs:57-67)
    return rv.SparseLDLT.analyze_with_matrix(s, rv.AnalyzeOptions(rv.OrderingStrategy.MATCH_ORDER_METIS))


def factor_both(rv, orc, s, solver):
    solver.factor(None, rv.FactorOptions())
    ref = orc.OracleFactor(s, solver.symbolic, solver._scaling, orc.options(), nthreads=THREADS)
    return ref


def large_path_ran(rv, solver, s):
    """Refactor once with the per-launch profiling marks and report the time
    spent in the large-front kernels and in the work-queue launch."""
    solver.set_profiling(True)
    solver.factor(None, rv.FactorOptions())
    p = solver.profile()["part_ms"]
    solver.set_profiling(False)
    return p.get("lf_block", 0.0), p.get("aptp", 0.0)


def random_stencil(rv, g, seed, diag_scale):
    """The 7-point pattern of a g^3 grid with N(0,1) off-diagonal values and a
    diagonal of diag_scale * N(0,1): strongly indefinite, so threshold tests
    fail and columns are delayed, on fronts of the sizes a Laplacian gives."""
    base = rv.problems.shifted_laplacian(g, 0.1).to_scipy().tocoo()
    rng = np.random.default_rng(seed)
    lo = base.row > base.col
    r, c = base.row[lo], base.col[lo]
    v = rng.standard_normal(r.size)
    n = base.shape[0]
    i = np.arange(n)
    d = diag_scale * rng.standard_normal(n)
    a = sp.csc_matrix((np.concatenate([v, v, d]), (np.concatenate([r, c, i]), np.concatenate([c, r, i]))),
                      shape=(n, n))
    return rv.problems.from_scipy(f"random_stencil{g}", a)


def test_c1_as_configured(rv, orc):
    # 7-point Laplacian 16^3 shifted to 10% negative, MC64 scaling, APTP u = 0.01,
    # one RHS b ~ U[-1, 1] from seed 0
    s = rv.problems.shifted_laplacian(16, 0.10)
    solver = analyze_mc64(rv, s)
    assert solver._scaling is not None
    ref = factor_both(rv, orc, s, solver)
    assert solver.inertia() == s.inertia == ref.inertia()
    assert_parity(rv, s, solver, ref, rv.problems.rhs_uniform(s.n, 0))
    solver.close()
    ref.close()


@pytest.mark.parametrize("g", [24, 26])
def test_kkt_default_options(rv, orc, g):
    # KKT of the C2 family (27-point H + diag U[0,1e-2], J with 4 N(0,1) per row),
    # MC64; the root front (order 4296 / 5382) takes the large-front path natively,
    # 2x2 pivots throughout
    s = rv.problems.kkt(g, seed=g)
    solver = analyze_mc64(rv, s)
    ref = factor_both(rv, orc, s, solver)
    assert solver.inertia() == s.inertia
    assert ref.stats()["total_2x2_pivots"] > 0
    assert_parity(rv, s, solver, ref, rv.problems.rhs_normal(s.n, 0))
    lf, _ = large_path_ran(rv, solver, s)
    assert lf > 0.0, "no front took the large-front path"
    assert_parity(rv, s, solver, ref, rv.problems.rhs_normal(s.n, 1))
    solver.close()
    ref.close()


def test_laplacian48_default_options(rv, orc):
    # 3456-order fronts in sibling pairs: concurrent large fronts on their own streams
    s = rv.problems.shifted_laplacian(48, 0.10)
    solver = analyze_mc64(rv, s)
    ref = factor_both(rv, orc, s, solver)
    fi = ref.front_info()
    big = fi[fi[:, 0] >= 2048]
    parents, counts = np.unique(big[:, 5], return_counts=True)
    assert counts.max() >= 2, "expected sibling large fronts"
    assert solver.inertia() == s.inertia
    assert_parity(rv, s, solver, ref, rv.problems.rhs_uniform(s.n, 0))
    lf, aq = large_path_ran(rv, solver, s)
    assert lf > 0.0 and aq > 0.0
    assert_parity(rv, s, solver, ref, rv.problems.rhs_uniform(s.n, 2))
    solver.close()
    ref.close()


def test_random_stencil_delays(rv, orc):
    # delayed columns at scale: ~5,000 delays, ~300 fronts of order >= 1024, the top
    # waves on the large-front path and the rest in the work-queue launch
    s = random_stencil(rv, 40, 40, 0.1)
    solver = analyze_mc64(rv, s)
    ref = factor_both(rv, orc, s, solver)
    st = ref.stats()
    assert st["total_delayed"] > 1000 and st["total_2x2_pivots"] > 0
    assert_parity(rv, s, solver, ref, rv.problems.rhs_uniform(s.n, 0), bwd=1e-13)
    lf, aq = large_path_ran(rv, solver, s)
    assert lf > 0.0 and aq > 0.0
    solver.close()
    ref.close()
