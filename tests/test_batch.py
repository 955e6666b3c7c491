"""Many systems as one block-diagonal union (BatchLDLT): host-side checks.

The union keeps each system's values contiguous, its elimination order keeps
each system's indices contiguous, and its symbolic structure is the systems'
structures side by side (supernode counts add up), so each system's fronts in
the union are the ones of its own analysis.
"""
import numpy as np

import pytest


def small_family(rv):
    fam = rv.problems.batch_family(count=6, seed=3, n_lo=200, n_hi=3000, max_rhs=5)
    return [s for s, _ in fam], [r for _, r in fam]


def test_family_is_seeded_and_in_range(rv):
    a = rv.problems.batch_family(count=8, seed=1, n_lo=5e3, n_hi=2e5)
    b = rv.problems.batch_family(count=8, seed=1, n_lo=5e3, n_hi=2e5)
    assert [(s.n, r) for s, r in a] == [(s.n, r) for s, r in b]
    for i, (s, r) in enumerate(a):
        assert 1 <= r <= 32
        assert (s.n_h > 0) == (i % 2 == 1)
        assert 0.4 * 5e3 <= s.n <= 1.3 * 2e5


def test_block_diagonal_union(rv):
    systems, _ = small_family(rv)
    u = rv.problems.block_diagonal(systems)
    assert u.n == sum(s.n for s in systems)
    assert u.inertia == tuple(sum(s.inertia[k] for s in systems) for k in range(3))
    dense = u.to_scipy().toarray()
    for i, s in enumerate(systems):
        lo, hi = u.meta["offsets"][i], u.meta["offsets"][i + 1]
        assert np.array_equal(dense[lo:hi, lo:hi], s.to_scipy().toarray())


def test_union_analysis_is_the_systems_side_by_side(rv):
    systems, _ = small_family(rv)
    bl = rv.BatchLDLT(systems, scaling=False, device_budget=0)
    assert len(bl.groups) == 1
    offs = bl.offsets
    perm = bl.groups[0].solver.symbolic.perm_fwd
    # each system's indices stay contiguous in elimination order
    sysid = np.searchsorted(offs, perm, side="right") - 1
    assert np.all(np.diff(sysid) >= 0)
    nsup = 0
    for s in systems:
        nsup += rv.SparseLDLT.analyze(s).symbolic.sup_begin.size
    assert bl.groups[0].solver.symbolic.sup_begin.size == nsup


def test_union_scaling_is_per_system_mc64(rv):
    systems, _ = small_family(rv)
    bl = rv.BatchLDLT(systems, device_budget=0)
    g = bl.groups[0]
    sc = np.empty(bl.n)
    sc[g.solver.symbolic.perm_fwd] = g.solver._scaling
    for i, s in enumerate(systems):
        _, si, _ = rv.ordering.mc64(s)
        assert np.allclose(sc[bl.offsets[i]:bl.offsets[i + 1]], si, rtol=1e-12, atol=0)


def test_rhs_packing(rv):
    systems, nrhs = small_family(rv)
    bl = rv.BatchLDLT(systems, scaling=False, device_budget=0)
    rhs = [rv.problems.rhs_normal(s.n, i, r) for i, (s, r) in enumerate(zip(systems, nrhs))]
    big = bl.rhs_matrix(rhs)
    assert big.shape == (bl.n, max(nrhs))
    back = bl.split(big, rhs)
    for a, b in zip(back, rhs):
        assert np.array_equal(a, b)


def test_perturbation_keeps_symmetry(rv):
    s = rv.problems.kkt(6, seed=1)
    v = rv.problems.perturb_symmetric(s, 0.01, seed=2)
    a = s.to_scipy().copy()
    a.data = v
    d = (a - a.T).toarray()
    assert np.max(np.abs(d)) == 0.0
    assert not np.array_equal(v, s.values)
    with pytest.raises(rv.InvalidInput):
        rv.BatchLDLT(systems=[], scaling=False, device_budget=0)


def test_groups_follow_the_memory_budget(rv):
    systems, nrhs = small_family(rv)
    est = [sum(rv.batch.memory_estimate(rv.SparseLDLT.analyze(s).symbolic)) for s in systems]
    budget = int(1.1 * (max(est) + sorted(est)[-2]) + 1)
    bl = rv.BatchLDLT(systems, scaling=False, device_budget=budget)
    assert len(bl.groups) > 1
    assert sum(g.count for g in bl.groups) == len(systems)
    nxt = 0
    for g in bl.groups:
        assert g.first == nxt
        nxt += g.count
        assert 1.1 * sum(est[g.first:g.first + g.count]) <= budget or g.count == 1
        assert g.union.n == sum(s.n for s in systems[g.first:g.first + g.count])
    # a group's right-hand sides and values are its systems' slices
    rhs = [rv.problems.rhs_normal(s.n, i, r) for i, (s, r) in enumerate(zip(systems, nrhs))]
    vals = bl.values()
    for g in bl.groups:
        assert np.array_equal(bl.group_values(g, vals), g.union.values)
        big = bl.rhs_matrix(rhs, g.first, g.count)
        back = bl.split(big, rhs, g.first, g.count)
        for a, b in zip(back, rhs[g.first:g.first + g.count]):
            assert np.array_equal(a, b)


def test_memory_estimate_bounds_the_factor(rv):
    s = rv.problems.kkt(10, seed=1)
    sym = rv.SparseLDLT.analyze(s).symbolic
    f, w = rv.batch.memory_estimate(sym)
    assert f >= 8 * sym.predicted_nnz
    assert w > 0
