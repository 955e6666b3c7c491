"""The allocation-free entry point rvg_dense_factor_noalloc.

It serves callers that cannot allocate device memory while they run (a
solver inside an application that owns the device's memory, work inside
stream-ordered pipelines, real-time loops): its scratch is a fixed array in
the library, and the caller passes every buffer.  This test calls it through
the C ABI on dense symmetric fronts -- two calls in a row, on different
matrices and both kernel paths (TPP for fewer than 32 columns, blocked APTP
with the two-level outer loop above 256) -- and checks each result against
the existing entry point (rvg_create / rvg_factor on the same matrix as a
sparse system of one front): the pivot order, the 1x1/2x2 codes and the D
entries must agree exactly, as in the other parity tests, and so must the
counts.  Buffers come from torch, i.e. from the test, never from the call.

Fronts with fewer fully-summed columns than rows (p < m) are checked against
the oracle's dense APTP kernel on the same front: pivot order, D, counts and
the factored columns, including their non-fully-summed rows, bit for bit.

The file sorts last so that a run stopping at its first failure has run every
other test before this one; it shares no state with them and passes alone.
"""
import ctypes as C

import numpy as np
import pytest
import scipy.sparse as sp

pytestmark = pytest.mark.gpu


def dense_matrix(n, seed, kind):
    rng = np.random.default_rng(seed)
    a = rng.standard_normal((n, n))
    a = a + a.T
    if kind == "delay":
        a[np.arange(n), np.arange(n)] *= 1e-6
    return a


def existing_entry_point(rv, a):
    n = a.shape[0]
    s = rv.problems.from_scipy("dense", sp.csc_matrix(a))
    solver = rv.SparseLDLT.analyze(s, rv.AnalyzeOptions(rv.OrderingStrategy.USER_SUPPLIED, np.arange(n)))
    assert solver.symbolic.sup_begin.size == 1  # one front holding every column
    solver.factor()
    col, code, dd, do = solver.pivot_record()
    st = solver.stats()
    solver.close()
    return col, code, dd, do, st


def no_alloc_call(rv, torch, a, p=None, with_matrix=False):
    n = a.shape[0]
    p = n if p is None else p
    d_a = torch.tensor(np.asfortranarray(a).ravel(order="F"), dtype=torch.float64, device="cuda")
    d_perm = torch.empty(max(p, 1), dtype=torch.int32, device="cuda")
    d_dt = torch.empty(max(p, 1), dtype=torch.int8, device="cuda")
    d_dd = torch.empty(max(p, 1), dtype=torch.float64, device="cuda")
    d_do = torch.empty(max(p, 1), dtype=torch.float64, device="cuda")
    d_cnt = torch.empty(3, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    st = rv._native.lib().rvg_dense_factor_noalloc(
        C.c_void_p(d_a.data_ptr()), n, p, None, C.c_void_p(d_perm.data_ptr()), C.c_void_p(d_dt.data_ptr()),
        C.c_void_p(d_dd.data_ptr()), C.c_void_p(d_do.data_ptr()), C.c_void_p(d_cnt.data_ptr()),
        C.c_void_p(stream))
    assert st == 0, rv._native.lib().rvg_last_error().decode()
    torch.cuda.synchronize()
    out = (d_perm.cpu().numpy().astype(np.int64)[:p], d_dt.cpu().numpy()[:p], d_dd.cpu().numpy()[:p],
           d_do.cpu().numpy()[:p], d_cnt.cpu().numpy())
    if with_matrix:
        out = out + (d_a.cpu().numpy().reshape(n, n).T.copy(),)  # back to row-major (i, j)
    return out


def check(ref, got):
    col, code, dd, do, st = ref
    perm, dt, ddg, dog, cnt = got
    ne = int(cnt[0])
    assert ne == col.size
    assert int(cnt[1]) == st["total_1x1_pivots"] and int(cnt[2]) == st["total_2x2_pivots"]
    assert np.array_equal(perm[:ne], col), "pivot order differs"
    assert np.array_equal(dt[:ne], code), "pivot codes differ"
    assert np.array_equal(ddg[:ne], dd) and np.array_equal(dog[:ne], do), "D differs"


@pytest.mark.parametrize("sizes", [(20, 300), (200, 120)])
def test_no_alloc_matches_existing_entry_point(rv, sizes):
    torch = pytest.importorskip("torch")
    cases = [dense_matrix(sizes[0], 11, "plain"), dense_matrix(sizes[1], 12, "delay")]
    refs = [existing_entry_point(rv, a) for a in cases]
    outs = [no_alloc_call(rv, torch, a) for a in cases]  # two calls in a row
    for ref, got in zip(refs, outs):
        check(ref, got)


@pytest.mark.parametrize("m,p,kind", [(300, 120, "delay"), (300, 120, "plain"), (100, 20, "delay")])
def test_no_alloc_partial_front_matches_oracle(rv, orc, m, p, kind):
    # p < m: the last m - p rows are not fully summed; the kernels update them too
    # (the L21 rows of every eliminated column), TPP below 32 columns, blocked APTP above
    torch = pytest.importorskip("torch")
    a = dense_matrix(m, 100 + m + p, kind)
    af, perm, dt, dd, do, st, _ = orc.dense_aptp(a.copy(), p=p)
    ne = int(st[0])
    for _ in range(2):  # two calls in a row share the scratch array
        gperm, gdt, gdd, gdo, cnt, ga = no_alloc_call(rv, torch, a, p, with_matrix=True)
        assert (int(cnt[0]), int(cnt[1]), int(cnt[2])) == (ne, int(st[1]), int(st[2]))
        assert np.array_equal(gperm[:ne], perm[:ne]), "pivot order differs"
        assert np.array_equal(gdt[:ne], dt[:ne]) and np.array_equal(gdd[:ne], dd[:ne]) and np.array_equal(gdo[:ne], do[:ne])
        low = np.tril(np.ones((m, ne), dtype=bool), -1)  # strictly below the diagonal, eliminated columns
        assert np.array_equal(ga[:, :ne][low], af[:, :ne][low]), "factored columns differ"


def test_no_alloc_rejects_oversized_fronts(rv):
    st = rv._native.lib().rvg_dense_factor_noalloc(None, 4097, 4097, None, None, None, None, None, None, None)
    assert st == 2
    assert "no-allocation limit" in rv._native.lib().rvg_last_error().decode()
