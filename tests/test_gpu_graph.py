"""Refactorization replayed as one CUDA graph (graph_refactor): a replayed
factorization gives bit for bit the factor of a dynamic one with the same
values, and when the new values change the pivoting decisions (other delays),
the graph's device checks catch it and the factorization runs dynamically."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def record(solver):
    col, code, dd, do = solver.pivot_record()
    return col.copy(), code.copy(), dd.copy(), do.copy(), solver.inertia()


def same(r1, r2):
    return all(np.array_equal(a, b) for a, b in zip(r1[:4], r2[:4])) and r1[4] == r2[4]


def dynamic(rv, s, values, **opts):
    solver = rv.SparseLDLT.analyze(s)
    solver.factor(values, rv.FactorOptions(**opts))
    r = record(solver)
    x = solver.solve(rv.problems.rhs_normal(s.n, 2))
    solver.close()
    return r, x


def dense_system(rv, name, n, seed, diag):
    import scipy.sparse as sp
    rng = np.random.default_rng(seed)
    a = rng.standard_normal((n, n))
    a = a + a.T
    a[np.arange(n), np.arange(n)] = diag(a.diagonal(), n)
    return rv.problems.from_scipy(name, sp.csc_matrix(a))


@pytest.mark.parametrize("case", ["lap", "kkt_large", "mixed_large", "delays"])
def test_replay_matches_dynamic(rv, case):
    opts = {}
    if case == "lap":
        s = rv.problems.shifted_laplacian(14, 0.1)
    elif case == "kkt_large":  # several whole-GPU fronts per wave (concurrent contexts in the graph)
        s = rv.problems.kkt(12, seed=3)
        opts = dict(large_front_threshold=64)
    elif case == "mixed_large":
        s = rv.problems.kkt(12, seed=3)
        opts = dict(large_front_threshold=64, precision="mixed", mixed_flush=0, mixed_operands="bf16")
    else:  # delays in every factorization, the same ones for the scaled values
        s = dense_system(rv, "delays", 600, 9, lambda d, n: d * 1e-6)
        opts = dict(large_front_threshold=33, outer_block_size=128)
    solver = rv.SparseLDLT.analyze(s)
    fo = rv.FactorOptions(graph_refactor=True, **opts)
    b = rv.problems.rhs_normal(s.n, 2)
    launches = []
    for rnd in range(4):
        # factorization 0: dynamic (records); 1: captured and replayed; 2-3: replayed
        vals = s.values * (1.0 + 0.25 * rnd) if case != "lap" else rv.problems.perturb_symmetric(s, 1e-9, rnd)
        solver.factor(vals, fo)
        launches.append(solver.profile()["factor_launches"])
        r = record(solver)
        ref, xref = dynamic(rv, s, vals, **opts)
        assert same(r, ref), (case, rnd)
        x = solver.solve(b)
        assert np.linalg.norm(x - xref) <= 1e-12 * np.linalg.norm(xref)
    assert launches[0] > 1 and launches[2] == launches[3] == 1, launches
    solver.close()


def test_replay_falls_back_when_delays_change(rv):
    import scipy.sparse as sp
    s = dense_system(rv, "fallback", 500, 4, lambda d, n: d + 3.0 * np.sqrt(n))  # dominant: no delays
    opts = dict(large_front_threshold=33, outer_block_size=128)
    solver = rv.SparseLDLT.analyze(s)
    fo = rv.FactorOptions(graph_refactor=True, **opts)
    solver.factor(None, fo)
    solver.factor(None, fo)  # captured and replayed
    assert solver.profile()["factor_launches"] == 1
    # same pattern, diagonal almost gone: the pivoting (delays, 2x2 pivots) changes
    c = s.to_scipy().tolil()
    c.setdiag(np.asarray(c.diagonal()) * 1e-8)
    vals = sp.csc_matrix(c)
    vals.sort_indices()
    v2 = np.asarray(vals.data)
    assert v2.size == s.values.size
    solver.factor(v2, fo)
    assert solver.profile()["factor_launches"] > 1  # the checks caught it: factored dynamically
    ref, _ = dynamic(rv, s, v2, **opts)
    assert same(record(solver), ref)
    assert solver.stats()["total_2x2_pivots"] > 0
    # the next refactorization with these values replays a new capture of the new record
    solver.factor(v2, fo)
    assert solver.profile()["factor_launches"] == 1
    assert same(record(solver), ref)
    solver.close()


def test_replay_scaling_pointer_change(rv):
    """factor_device with another scaling buffer: the graph (which reads the
    scaling through its captured address) is captured anew, results stay equal."""
    import torch
    s = rv.problems.kkt(8, seed=1)
    solver = rv.SparseLDLT.analyze_with_matrix(s, rv.AnalyzeOptions(rv.OrderingStrategy.MATCH_ORDER_METIS))
    fo = rv.FactorOptions(graph_refactor=True, large_front_threshold=64)
    d_vals = torch.from_numpy(s.values).to("cuda")
    sc = [torch.from_numpy(solver._scaling).to("cuda"), torch.from_numpy(solver._scaling.copy()).to("cuda")]
    recs = []
    for i in range(5):
        solver.factor_device(d_vals.data_ptr(), sc[i // 3].data_ptr(), fo)
        torch.cuda.synchronize()
        recs.append(record(solver))
    assert all(same(recs[0], r) for r in recs[1:])
    solver.close()
