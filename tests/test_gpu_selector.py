"""Learned per-front precision: the selector's CUDA kernels against the
float64 oracle (forward, gradient, Adam), training on the GPU, and the
precision = learned factorization path (routes honoured bit for bit, the FP64
rerun after a growth flag, accuracy after refinement)."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def random_params(mo, seed=0):
    rng = np.random.default_rng(seed)
    p = rng.normal(0, 0.3, mo.NPARAM)
    p[mo.MU:mo.SD] = rng.normal(0, 1, mo.IN)
    p[mo.SD:] = rng.uniform(0.5, 2.0, mo.IN)
    return p.astype(np.float32)


def vp(t):
    return C.c_void_p(t.data_ptr())


def gpu_grad(rv, p, x, y, w, norm):
    import torch
    L = rv._native.lib()
    n = y.size
    dP, dX, dY = (torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda() for a in (p, x, y))
    dW = torch.from_numpy(np.ascontiguousarray(w, np.float32)).cuda() if w is not None else None
    dG = torch.zeros(L.rvg_mlp_trained_count(), dtype=torch.float32, device="cuda")
    dL = torch.zeros(1, dtype=torch.float32, device="cuda")
    work = torch.empty(L.rvg_mlp_work_floats(n), dtype=torch.float32, device="cuda")
    st = rv._native.lib().rvg_mlp_grad(vp(dP), vp(dX), vp(dY), vp(dW) if dW is not None else None, n, float(norm),
                                       vp(dG), vp(dL), vp(work), work.numel(), None)
    rv._native.check(st)
    torch.cuda.synchronize()
    return float(dL.item()), dG.cpu().numpy()


def test_forward_matches_oracle(rv, mlp_oracle):
    mo = mlp_oracle
    p = random_params(mo, 1)
    x = np.random.default_rng(2).normal(0, 2, (3001, mo.IN)).astype(np.float32)
    sel = rv.PrecisionSelector(p)
    got = sel.predict_proba(x)
    ref = mo.sigmoid(mo.forward(p.astype(np.float64), x.astype(np.float64))[0])
    assert np.max(np.abs(got - ref)) <= 2e-6


@pytest.mark.parametrize("n,weighted", [(1, False), (37, True), (5000, True), (40000, False)])
def test_gradient_matches_oracle(rv, mlp_oracle, n, weighted):
    mo = mlp_oracle
    rng = np.random.default_rng(n)
    p = random_params(mo, 3)
    x = rng.normal(0, 1.5, (n, mo.IN)).astype(np.float32)
    y = (rng.uniform(size=n) < 0.3).astype(np.float32)
    w = rng.uniform(0.5, 2.0, n).astype(np.float32) if weighted else None
    norm = float(w.sum()) if weighted else float(n)
    loss, g = gpu_grad(rv, p, x, y, w, norm)
    lref, gref = mo.loss_grad(p.astype(np.float64), x.astype(np.float64), y, w, norm)
    assert abs(loss - lref) <= 1e-5 * max(1.0, abs(lref))
    # float32 sums over n samples against float64: normwise and entrywise tolerances
    assert np.linalg.norm(g - gref) <= 1e-4 * np.linalg.norm(gref)
    assert np.max(np.abs(g - gref)) <= 1e-4 * np.max(np.abs(gref))


def test_gradient_is_deterministic(rv, mlp_oracle):
    mo = mlp_oracle
    rng = np.random.default_rng(5)
    p = random_params(mo, 4)
    x = rng.normal(0, 1, (20000, mo.IN)).astype(np.float32)
    y = (rng.uniform(size=20000) < 0.5).astype(np.float32)
    l1, g1 = gpu_grad(rv, p, x, y, None, 20000.0)
    l2, g2 = gpu_grad(rv, p, x, y, None, 20000.0)
    assert l1 == l2 and np.array_equal(g1, g2)


def test_adam_matches_oracle(rv, mlp_oracle):
    import torch
    mo = mlp_oracle
    L = rv._native.lib()
    p = random_params(mo, 6)
    rng = np.random.default_rng(7)
    g = rng.normal(0, 1, mo.NTRAIN).astype(np.float32)
    m = rng.normal(0, 0.1, mo.NTRAIN).astype(np.float32)
    v = rng.uniform(0, 0.1, mo.NTRAIN).astype(np.float32)
    dP, dG, dM, dV = (torch.from_numpy(a.copy()).cuda() for a in (p, g, m, v))
    rv._native.check(L.rvg_mlp_adam(vp(dP), vp(dG), vp(dM), vp(dV), 5, 1e-3, 0.9, 0.999, 1e-8, 1e-4, None))
    torch.cuda.synchronize()
    # the kernel's constants are float32: give the oracle the same values
    b1, b2, wd = (float(np.float32(c)) for c in (0.9, 0.999, 1e-4))
    pr, mr, vr = mo.adam(p.astype(np.float64), g.astype(np.float64), m, v, 5, float(np.float32(1e-3)), b1, b2,
                         float(np.float32(1e-8)), wd)
    assert np.allclose(dM.cpu().numpy(), mr, rtol=1e-5, atol=1e-7)
    assert np.allclose(dV.cpu().numpy(), vr, rtol=1e-5, atol=1e-9)
    assert np.allclose(dP.cpu().numpy(), pr, rtol=1e-5, atol=1e-7)


def test_training_learns_a_separable_rule(rv):
    rng = np.random.default_rng(8)
    x = rng.normal(0, 1, (4000, 12))
    y = ((x[:, 0] - 0.5 * x[:, 7] + 0.2 * x[:, 3] ** 2) > 0.1).astype(float)
    sel = rv.PrecisionSelector(seed=1)
    sel.fit_normalisation(x)
    hist = sel.train(x, y, steps=400, lr=1e-2)
    assert hist[-1][1] < 0.5 * hist[0][1]
    xt = rng.normal(0, 1, (2000, 12))
    yt = ((xt[:, 0] - 0.5 * xt[:, 7] + 0.2 * xt[:, 3] ** 2) > 0.1)
    acc = np.mean((sel.predict_proba(xt) >= 0.5) == yt)
    assert acc >= 0.95, acc


def record(solver):
    col, code, dd, do = solver.pivot_record()
    return col.copy(), code.copy(), dd.copy(), do.copy()


def same(a, b):
    return all(np.array_equal(x, y) for x, y in zip(a, b))


def forced(rv, mixed, bound=1e300):
    sel = rv.PrecisionSelector()
    sel.threshold = -1.0 if mixed else 2.0
    sel.growth_bound = bound
    return sel


BASE = dict(large_front_threshold=128, mixed_flush=0, mixed_operands="bf16")


@pytest.mark.parametrize("mixed", [False, True])
def test_forced_routes_reproduce_the_uniform_forms(rv, mixed):
    s = rv.problems.kkt(10, seed=2)
    solver = rv.SparseLDLT.analyze(s)
    solver.factor(None, rv.FactorOptions(precision="mixed" if mixed else "fp64", **BASE))
    ref = record(solver)
    solver.set_selector(forced(rv, mixed))
    solver.factor(None, rv.FactorOptions(precision="learned", **BASE))
    assert same(record(solver), ref)
    st = solver.selector_stats()
    assert st["large_fronts"] > 0 and st["routed_mixed"] == (st["large_fronts"] if mixed else 0)
    assert not st["fp64_rerun"]
    t = solver.front_features()
    assert t.shape == (st["large_fronts"], 22)
    assert np.all(t[:, 6] == (1.0 if mixed else 0.0)) and np.all(np.isfinite(t[:, 10:]))
    assert np.all(t[:, 8] > 0) and np.all(t[:, 9] > 0)  # max |a| and max |D|
    solver.close()


def test_growth_flag_refactors_the_front_in_fp64(rv):
    # every mixed front is over the bound: each is assembled again and factored in FP64 at the end of its
    # wave, so the whole factor is the plain FP64 one, bit for bit
    s = rv.problems.kkt(10, seed=2)
    solver = rv.SparseLDLT.analyze(s)
    solver.factor(None, rv.FactorOptions(precision="fp64", **BASE))
    ref = record(solver)
    solver.set_selector(forced(rv, True, bound=1e-300))
    solver.factor(None, rv.FactorOptions(precision="learned", **BASE))
    st = solver.selector_stats()
    assert st["over_bound"] > 0 and st["fp64_refactored"] == st["over_bound"] == st["large_fronts"]
    assert same(record(solver), ref)
    b = rv.problems.rhs_normal(s.n, 4)
    x = solver.solve(b)
    assert rv.problems.backward_error(s, x, b) <= 1e-14
    solver.close()


def test_learned_routes_mixed_and_fp64_fronts_and_refines(rv):
    s = rv.problems.kkt(12, seed=3)
    solver = rv.SparseLDLT.analyze(s)
    solver.set_selector(forced(rv, False))
    solver.factor(None, rv.FactorOptions(precision="learned", **BASE))
    feats = solver.front_features()
    # a selector that sends the larger half of the fronts to the mixed form
    sel = rv.PrecisionSelector(seed=0)
    sel.fit_normalisation(feats[:, 10:])
    y = (feats[:, 1] >= np.median(feats[:, 1])).astype(float)
    sel.train(feats[:, 10:], y, steps=300, lr=1e-2)
    solver.set_selector(sel)
    solver.factor(None, rv.FactorOptions(precision="learned", **BASE))
    st = solver.selector_stats()
    assert 0 < st["routed_mixed"] < st["large_fronts"]
    t = solver.front_features()
    assert np.array_equal(t[:, 6] == 1.0, t[:, 7] >= sel.threshold)
    assert solver.inertia() == s.inertia
    b = rv.problems.rhs_normal(s.n, 4)
    x, its, err, how = solver.solve_auto(b)
    assert err <= 1e-14 and rv.problems.backward_error(s, x, b) <= 1e-14
    solver.close()


def test_learned_needs_a_selector(rv):
    s = rv.problems.kkt(6, seed=1)
    solver = rv.SparseLDLT.analyze(s)
    with pytest.raises(rv.InvalidInput):
        solver.factor(None, rv.FactorOptions(precision="learned", **BASE))
    solver.close()


def test_label_fronts(rv):
    s = rv.problems.kkt(10, seed=4)
    X, y, err, m = rv.selector.label_fronts(s, tau=1e-3, opts=rv.FactorOptions(**BASE))
    assert X.shape == (y.size, 12) and err.size == y.size and y.size > 0
    assert np.all((y == 1) == (err <= 1e-3))
    assert np.all(m >= 64)  # whole-GPU fronts: order >= the threshold, or half of it in a wave with few


def test_shipped_selector_gains_over_uniform_forms(rv):
    """The committed selector (trained by rivrs-linalg_b200/train_selector.py on
    generated matrices) on held-out ones, factor + solve to 1e-14 timed after a
    warm-up: on a KKT, where the mixed form is accurate, it sends most fronts to
    the mixed form and takes less time than plain FP64; on an indefinite
    Laplacian, where the all-mixed factor needs many more solves than FP64, it
    keeps the large separators in FP64 and needs fewer solves than all-mixed.
    Time is asserted on the KKT only: on this 64k-unknown Laplacian the three
    forms take 36, 47 and 50 ms (plain, all-mixed, learned; B200), within the
    run-to-run spread of one another.  Each form's time is the best of three
    runs."""
    import os
    sel = rv.PrecisionSelector.load(os.path.join(os.path.dirname(rv.__file__), "data", "selector_bf16.npz"))
    S = rv.selector
    base = dict(large_front_threshold=256, mixed_flush=0, mixed_operands="bf16")
    for s, kind in ((rv.problems.shifted_laplacian(40, 0.05), "lap"), (rv.problems.kkt(48, seed=777, reg_hi=1e-4), "kkt")):
        solver = rv.SparseLDLT.analyze_with_matrix(s, rv.AnalyzeOptions(rv.OrderingStrategy.MATCH_ORDER_METIS))
        solver.set_selector(sel)
        b = rv.problems.rhs_normal(s.n, 9)
        res = {}
        for f in ("fp64", "mixed", "learned"):
            runs = [S.timed_solve(solver, s, rv.FactorOptions(precision=f, **base), b, warmup=1 if r == 0 else 0)
                    for r in range(3)]
            res[f] = min(runs, key=lambda r: r["s"])
        solver.close()
        for f, r in res.items():
            assert r["bwd"] <= 1e-14, (kind, f, r)
        lr = res["learned"]
        frac = lr["routed_mixed"] / max(lr["large_fronts"], 1)
        if kind == "lap":
            assert res["mixed"]["solves_after_first"] > res["fp64"]["solves_after_first"], res
            assert lr["solves_after_first"] < res["mixed"]["solves_after_first"], res
            assert lr["routed_mixed"] < lr["large_fronts"], lr  # the large separators stay FP64
        else:
            assert frac >= 0.5, lr
            assert lr["solves_after_first"] <= res["mixed"]["solves_after_first"] + 1, res
            assert lr["s"] <= 0.8 * res["fp64"]["s"], res


def test_autotune_picks_a_candidate_and_caches(rv, tmp_path):
    import torch
    s = rv.problems.kkt(14, seed=5)
    solver = rv.SparseLDLT.analyze(s)
    d_vals = torch.from_numpy(s.values).cuda()
    base = rv.FactorOptions(precision="mixed", mixed_flush=0, mixed_operands="bf16")
    cache = str(tmp_path / "tune.json")
    best, table = rv.autotune.autotune(solver, d_vals.data_ptr(), None, base, reps=1, thresholds=(64, 512),
                                       cache=cache)
    assert len(table) == 4 and min(t for _, t in table) == [t for c, t in table if
                                                            c["large_front_threshold"] == best.large_front_threshold
                                                            and c["mixed_tile_cols"] == best.mixed_tile_cols][0]
    best2, table2 = rv.autotune.autotune(solver, d_vals.data_ptr(), None, base, reps=1, thresholds=(64, 512),
                                         cache=cache)
    assert best2 == best and [c for c, _ in table2] == [c for c, _ in table]
    # in the plain form the scheduling options change no result
    plain = rv.FactorOptions()
    best_p, _ = rv.autotune.autotune(solver, d_vals.data_ptr(), None, plain, reps=1, thresholds=(64, 512))
    solver.factor(None, best_p)
    r1 = record(solver)
    solver.factor(None, rv.FactorOptions(large_front_threshold=64 if best_p.large_front_threshold == 512 else 512))
    assert same(record(solver), r1)
    solver.close()
