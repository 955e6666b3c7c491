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


def per_system_record(bl, i):
    col, code, dd, do = bl.solver.pivot_record()
    sel = bl._sys_of_pos[col] == i
    return col[sel] - col[sel].min(), code[sel], dd[sel], do[sel]


def separate(rv, bl, i, values, opts):
    s = bl.systems[i]
    sc = np.empty(bl.n)
    sc[bl.solver.symbolic.perm_fwd] = bl.solver._scaling
    solver = rv.SparseLDLT.analyze_with_matrix(s, scaling=sc[bl.offsets[i]:bl.offsets[i + 1]])
    solver.factor(values, opts)
    return solver


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_union_matches_separate_factorizations(rv, precision):
    systems, nrhs = family(rv)
    opts = rv.FactorOptions(precision=precision, mixed_flush=0, large_front_threshold=256)
    bl = rv.BatchLDLT(systems)
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
            c0, k0, d0, o0 = per_system_record(bl, i)
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
    bl = rv.BatchLDLT(systems)
    bl.factor(None, rv.FactorOptions(precision="mixed", mixed_flush=0, large_front_threshold=256))
    b = rv.problems.rhs_normal(bl.n, 1)
    x, iters, err = bl.solver.solve_refine(b, tol=1e-14, max_iter=10)
    assert err <= 1e-14
    assert bl.solver.inertia() == bl.union.inertia
    bl.close()
