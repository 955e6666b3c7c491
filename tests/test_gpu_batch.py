"""Many systems factored as one block-diagonal union on the GPU: every
system's pivots and D are bit-identical to a separate factorization with the
same ordering and scaling, refactorization with new values matches too, and
every system's solution meets the backward-error gate."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def family(rv, count=6, seed=3):
    fam = rv.problems.batch_family(count=count, seed=seed, n_lo=300, n_hi=6000, max_rhs=9)
    return [s for s, _ in fam], [r for _, r in fam]


def separate(rv, bl, i, values, opts):
    s = bl.systems[i]
    g = next(g for g in bl.groups if g.first <= i < g.first + g.count)
    sc = np.empty(g.union.n)
    sc[g.solver.symbolic.perm_fwd] = g.solver._scaling
    lo = bl.offsets[i] - bl.offsets[g.first]
    solver = rv.SparseLDLT.analyze_with_matrix(s, scaling=sc[lo:lo + s.n])
    solver.factor(values, opts)
    return solver


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_union_matches_separate_factorizations(rv, precision):
    systems, nrhs = family(rv)
    opts = rv.FactorOptions(precision=precision, mixed_flush=0, large_front_threshold=256)
    bl = rv.BatchLDLT(systems, device_budget=0)
    for rnd in range(2):  # factor, then a refactorization with perturbed values
        vals = [None if rnd == 0 else rv.problems.perturb_symmetric(s, 0.01, seed=10 + i)
                for i, s in enumerate(systems)]
        bl.factor(None if rnd == 0 else vals, opts)
        inert = bl.inertias()
        rhs = [rv.problems.rhs_normal(s.n, i, r) for i, (s, r) in enumerate(zip(systems, nrhs))]
        xs = bl.solve(rhs)
        for i, s in enumerate(systems):
            if rnd == 0:
                assert inert[i] == s.inertia
            one = separate(rv, bl, i, vals[i], opts)
            c0, k0, d0, o0 = bl.system_record(i)
            c1, k1, d1, o1 = one.pivot_record()
            assert np.array_equal(c0, c1 - c1.min()) and np.array_equal(k0, k1)
            assert np.array_equal(d0, d1) and np.array_equal(o0, o1), ("D differs", i)
            assert inert[i] == one.inertia()
            x1 = one.solve(rhs[i])
            assert np.linalg.norm(xs[i] - x1) <= 1e-12 * np.linalg.norm(x1)
            if precision == "fp64":
                a = s.to_scipy()
                if vals[i] is not None:
                    a = a.copy()
                    a.data = vals[i]
                sv = rv.problems.from_scipy("v", a)
                b = rhs[i] if rhs[i].ndim == 2 else rhs[i][:, None]
                x = xs[i] if xs[i].ndim == 2 else xs[i][:, None]
                for j in range(b.shape[1]):
                    assert rv.problems.backward_error(sv, x[:, j], b[:, j]) <= 1e-14
            one.close()
    bl.close()


def test_union_refined_solve(rv):
    systems, _ = family(rv, count=4, seed=5)
    bl = rv.BatchLDLT(systems, device_budget=0)
    bl.factor(None, rv.FactorOptions(precision="mixed", mixed_flush=0, large_front_threshold=256))
    g = bl.groups[0]
    b = rv.problems.rhs_normal(bl.n, 1)
    x, iters, err = g.solver.solve_refine(b, tol=1e-14, max_iter=10)
    assert err <= 1e-14
    assert g.solver.inertia() == g.union.inertia
    bl.close()


def test_groups_and_trim_match_one_union(rv):
    # a budget that forces several groups: factor_solve (each group factored,
    # solved and released in turn) gives every system the same D and solution
    # as one union holding all of them; a second round reuses the trimmed handles
    systems, nrhs = family(rv, count=6, seed=7)
    opts = rv.FactorOptions(precision="fp64", large_front_threshold=256)
    one = rv.BatchLDLT(systems, device_budget=0)
    est = [sum(rv.batch.memory_estimate(rv.SparseLDLT.analyze(s).symbolic)) for s in systems]
    many = rv.BatchLDLT(systems, device_budget=int(1.1 * 2 * max(est)) + 1)
    assert len(many.groups) > 1
    rhs = [rv.problems.rhs_normal(s.n, i, r) for i, (s, r) in enumerate(zip(systems, nrhs))]
    one.factor(None, opts)
    x1 = one.solve(rhs)
    for rnd in range(2):
        xs = many.factor_solve(None, rhs, opts)
        assert many.inertias() == one.inertias() == [s.inertia for s in systems]
        for a, b in zip(xs, x1):
            assert np.linalg.norm(a - b) <= 1e-12 * np.linalg.norm(b)
    # factor + solve with every group's factor kept (workspace trimmed between groups)
    many.factor(None, opts)
    for i in range(len(systems)):
        c0, k0, d0, o0 = one.system_record(i)
        c1, k1, d1, o1 = many.system_record(i)
        assert np.array_equal(c0, c1) and np.array_equal(k0, k1)
        assert np.array_equal(d0, d1) and np.array_equal(o0, o1)
    xs = many.solve(rhs)
    for a, b in zip(xs, x1):
        assert np.linalg.norm(a - b) <= 1e-12 * np.linalg.norm(b)
    # the trimmed handle refuses to solve until it is factored again
    g = many.groups[0]
    g.solver.trim(workspace=True, factor=True)
    with pytest.raises(rv.SolveBeforeFactor):
        g.solver.solve(np.zeros(g.union.n))
    one.close()
    many.close()


def test_autotuned_groups_give_the_same_factors(rv):
    # each union's scheduling options tuned on its own pattern; in the plain form the choice changes no
    # result, so every system's pivots and D equal those of the untuned factorization
    import torch
    systems, nrhs = family(rv, count=5, seed=7)
    bl = rv.BatchLDLT(systems, device_budget=0)
    bl.factor(None, rv.FactorOptions())
    ref = [bl.system_record(i) for i in range(len(systems))]
    d_vals = torch.from_numpy(bl.values()).to("cuda")
    scals = [torch.from_numpy(g.solver._scaling).to("cuda") for g in bl.groups]
    tables = bl.autotune_groups(d_vals.data_ptr(), [t.data_ptr() for t in scals],
                                rv.FactorOptions(large_front_threshold=2048), reps=1)
    assert len(tables) == len(bl.groups) and all(len(t) >= 2 for t in tables)
    assert all(g.options is not None for g in bl.groups)
    rhs = [rv.problems.rhs_normal(s.n, i, r) for i, (s, r) in enumerate(zip(systems, nrhs))]
    bl.factor(None)  # each union with its tuned options
    xs = bl.solve(rhs)
    for i, s in enumerate(systems):
        got = bl.system_record(i)
        assert all(np.array_equal(a, b) for a, b in zip(got, ref[i])), i
        bb = rhs[i] if rhs[i].ndim == 2 else rhs[i][:, None]
        xx = xs[i] if xs[i].ndim == 2 else xs[i][:, None]
        assert max(rv.problems.backward_error(s, xx[:, j], bb[:, j]) for j in range(bb.shape[1])) <= 1e-14
    bl.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_refactorizations_replay_as_graphs_across_turns(rv, precision):
    """graph_refactor = 2: each union's arenas keep their addresses while rvg_trim gives their memory back,
    so the unions take turns on the device and each still replays its captured refactorization graph (one
    launch per factorization from the third on). Every system's pivot order, codes and D equal those of a
    batch that factors dynamically, round after round of new values; the solutions meet the gate."""
    import dataclasses
    fam = rv.problems.batch_family(count=6, seed=5, n_lo=300, n_hi=6000, max_rhs=9)
    systems, nrhs = [s for s, _ in fam], [r for _, r in fam]
    base = rv.FactorOptions(precision=precision, mixed_flush=0, large_front_threshold=256)
    budget = 14 * 2 ** 20  # several unions of these systems' estimated memory
    dyn = rv.BatchLDLT(systems, device_budget=budget)
    rep = rv.BatchLDLT(systems, device_budget=budget)
    assert len(rep.groups) >= 2
    opts = dataclasses.replace(base, graph_refactor=2)
    rhs = [rv.problems.rhs_normal(s.n, i, r) for i, (s, r) in enumerate(zip(systems, nrhs))]
    for rnd in range(4):
        # factorization 0: dynamic (records); 1: captured and replayed; 2-3: replayed.  The values change by
        # a factor per round, which keeps every pivot decision (a replay whose checks see another decision
        # falls back to a dynamic factorization, tested for one handle in test_gpu_graph.py)
        vals = None if rnd == 0 else [s.values * (1.0 + 0.25 * rnd) for s in systems]
        dyn.factor(vals, base)
        rep.factor(vals, opts)
        launches = [g.solver.profile()["factor_launches"] for g in rep.groups]
        if rnd >= 2:
            assert all(n == 1 for n in launches), launches  # replayed
        for i in range(len(systems)):
            a, b = dyn.system_record(i), rep.system_record(i)
            assert all(np.array_equal(x, y) for x, y in zip(a, b)), ("record differs", rnd, i)
        assert rep.inertias() == dyn.inertias()
        xs = rep.solve(rhs)
        if precision == "fp64":
            for i, s in enumerate(systems):
                a = s.to_scipy()
                if vals is not None:
                    a = a.copy()
                    a.data = vals[i]
                sv = rv.problems.from_scipy("v", a)
                bb = rhs[i] if rhs[i].ndim == 2 else rhs[i][:, None]
                x = xs[i] if xs[i].ndim == 2 else xs[i][:, None]
                for j in range(bb.shape[1]):
                    assert rv.problems.backward_error(sv, x[:, j], bb[:, j]) <= 1e-14
    dyn.close()
    rep.close()
