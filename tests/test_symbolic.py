"""Host symbolic analysis (the AptpSymbolic stand-in) against brute force."""
import numpy as np
import pytest
import scipy.sparse as sp


def brute_force_structure(a, order):
    """Column structure of L for P A P^T by symbolic elimination (small n)."""
    n = a.shape[0]
    b = a[order][:, order].tocsc()
    cols = [set(b.indices[b.indptr[j]:b.indptr[j + 1]][b.indices[b.indptr[j]:b.indptr[j + 1]] > j]) for j in range(n)]
    parent = [-1] * n
    for j in range(n):
        if cols[j]:
            p = min(cols[j])
            parent[j] = p
            cols[p] |= {i for i in cols[j] if i > p}
    return cols, parent


def random_sym(n, density, seed):
    rng = np.random.default_rng(seed)
    m = sp.random(n, n, density=density, random_state=seed, format="csc")
    m = m + m.T + sp.identity(n)
    m.data = rng.standard_normal(m.data.size)
    m = (m + m.T).tocsc()
    return m


@pytest.mark.parametrize("n,density,seed", [(1, 0.0, 0), (2, 0.5, 1), (10, 0.2, 2), (40, 0.05, 3), (60, 0.1, 4),
                                            (120, 0.02, 5)])
def test_supernodes_match_brute_force(rv, n, density, seed):
    a = random_sym(n, density, seed)
    s = rv.problems.from_scipy("r", a)
    order = np.random.default_rng(seed).permutation(n).astype(np.int64)
    sym = rv.symbolic_analyze(n, s.colptr, s.rowidx, order)
    assert sorted(sym.perm_fwd.tolist()) == list(range(n))
    cols, parent = brute_force_structure(s.to_scipy(), sym.perm_fwd)
    # relaxed supernodes: every column's structure lies inside its supernode's
    # columns below it plus the pattern, and the pattern is exactly the
    # structure of the last column
    for sidx in range(sym.sup_begin.size):
        b, e = sym.sup_begin[sidx], sym.sup_end[sidx]
        pat = set(sym.pat_idx[sym.pat_ptr[sidx]:sym.pat_ptr[sidx + 1]].tolist())
        for j in range(b, e):
            assert cols[j] <= set(range(j + 1, e)) | pat, (sidx, j)
        assert cols[e - 1] == pat
        # parent supernode holds etree parent of the last column
        p = parent[e - 1]
        if p == -1:
            assert sym.sup_parent[sidx] == -1
        else:
            ps = sym.sup_parent[sidx]
            assert sym.sup_begin[ps] <= p < sym.sup_end[ps]
    # postorder: parents after children
    for sidx, p in enumerate(sym.sup_parent):
        assert p == -1 or p > sidx
    assert sym.predicted_nnz == sum(len(c) + 1 for c in cols)


def test_grid_nested_dissection_is_a_permutation(rv):
    for dims in [(1, 1, 1), (3, 4, 5), (16, 16, 16), (7, 1, 9)]:
        o = rv.ordering.nested_dissection_grid(dims)
        assert np.array_equal(np.sort(o), np.arange(np.prod(dims)))


def test_laplacian_structure_against_brute_force(rv):
    s = rv.problems.shifted_laplacian(6, 0.1)
    order = rv.ordering.default_order(s)
    sym = rv.symbolic_analyze(s.n, s.colptr, s.rowidx, order)
    cols, _ = brute_force_structure(s.to_scipy(), sym.perm_fwd)
    assert sym.predicted_nnz == sum(len(c) + 1 for c in cols)


def test_analyze_rejects_bad_permutation(rv):
    s = rv.problems.shifted_laplacian(3, 0.1)
    with pytest.raises(rv.InvalidInput):
        rv.symbolic_analyze(s.n, s.colptr, s.rowidx, np.zeros(s.n, np.int64))
