"""Autotuner host logic: candidate sets and pattern fingerprints (no GPU)."""
import pytest


def test_candidates(rv):
    A = rv.autotune
    mixed = rv.FactorOptions(precision="mixed", mixed_flush=0, mixed_operands="bf16")
    c = A.candidates(mixed)
    assert len(c) == 6 and {(o.large_front_threshold, o.mixed_tile_cols) for o in c} == {
        (t, w) for t in (1024, 2048, 4096) for w in (128, 256)}
    assert all(o.precision == "mixed" and o.mixed_operands == "bf16" for o in c)
    plain = rv.FactorOptions()
    assert [o.large_front_threshold for o in A.candidates(plain)] == [1024, 2048, 4096]
    flushed = rv.FactorOptions(precision="mixed", mixed_flush=4)
    assert len(A.candidates(flushed)) == 3  # the tile width only applies without flushing


def test_fingerprint(rv):
    A = rv.autotune
    s1 = rv.SparseLDLT.analyze(rv.problems.shifted_laplacian(6, 0.1))
    s2 = rv.SparseLDLT.analyze(rv.problems.shifted_laplacian(6, 0.2))  # same pattern, other values
    s3 = rv.SparseLDLT.analyze(rv.problems.shifted_laplacian(7, 0.1))
    assert A.fingerprint(s1) == A.fingerprint(s2) != A.fingerprint(s3)


def test_autotune_choice_and_cache_with_a_host_timer(rv, tmp_path):
    A = rv.autotune
    s = rv.SparseLDLT.analyze(rv.problems.shifted_laplacian(6, 0.1))
    base = rv.FactorOptions(precision="mixed", mixed_flush=0, mixed_operands="bf16")
    cost = {(1024, 128): 3.0, (1024, 256): 2.0, (2048, 128): 2.5, (2048, 256): 1.5, (4096, 128): 4.0,
            (4096, 256): 1.75}
    calls = []

    def timer(o):
        calls.append(o)
        return cost[(o.large_front_threshold, o.mixed_tile_cols)]
    cache = str(tmp_path / "tune.json")
    best, table = A.autotune(s, None, None, base, cache=cache, timer=timer, device_name="test-gpu")
    assert (best.large_front_threshold, best.mixed_tile_cols) == (2048, 256)
    assert best.precision == "mixed" and best.mixed_operands == "bf16"
    assert len(calls) == 6 and len(table) == 6
    # the second call reads the cache: no timing
    best2, table2 = A.autotune(s, None, None, base, cache=cache, timer=timer, device_name="test-gpu")
    assert best2 == best and len(calls) == 6 and table2 == table
    # another device or another precision is another key
    A.autotune(s, None, None, base, cache=cache, timer=timer, device_name="other-gpu")
    assert len(calls) == 12


def _window_step(cost, inertia):
    calls = []

    def step(o):
        calls.append(o.mixed_window)
        return cost[o.mixed_window], inertia[o.mixed_window]
    return step, calls


def test_window_stage_takes_a_faster_deeper_window_with_the_same_inertia(rv, tmp_path):
    A = rv.autotune
    s = rv.SparseLDLT.analyze(rv.problems.shifted_laplacian(6, 0.1))
    base = rv.FactorOptions(precision="mixed", mixed_flush=0, mixed_operands="bf16")
    step, calls = _window_step({4: 1.0, 8: 0.9}, {4: (10, 5, 0), 8: (10, 5, 0)})
    best, table = A.autotune(s, None, None, base, timer=lambda o: 1.0, device_name="g", step=step,
                             expect_inertia=(10, 5, 0), cache=str(tmp_path / "t.json"))
    assert best.mixed_window == 8 and calls == [4, 8]
    assert [r[0].get("accepted") for r in table[-2:]] == [True, True]
    # cached with the window
    best2, _ = A.autotune(s, None, None, base, timer=lambda o: 1.0, device_name="g", step=step,
                          expect_inertia=(10, 5, 0), cache=str(tmp_path / "t.json"))
    assert best2.mixed_window == 8 and calls == [4, 8]


@pytest.mark.parametrize("cost,inertia,expect,want", [
    ({4: 1.0, 8: 0.9}, {4: (10, 5, 0), 8: (11, 4, 0)}, (10, 5, 0), 4),   # the deeper window flips a pivot's sign
    ({4: 1.0, 8: 0.9}, {4: (10, 5, 0), 8: (11, 4, 0)}, None, 4),         # against the default window's inertia
    ({4: 1.0, 8: 1.2}, {4: (10, 5, 0), 8: (10, 5, 0)}, (10, 5, 0), 4),   # slower once the solves are counted
])
def test_window_stage_keeps_the_default_window(rv, cost, inertia, expect, want):
    best, rows = rv.autotune.tune_window(rv.FactorOptions(precision="mixed", mixed_flush=0), _window_step(cost, inertia)[0],
                                         expect)
    assert best.mixed_window == want and len(rows) == 2


def test_window_stage_only_for_the_unflushed_mixed_form(rv):
    A = rv.autotune
    s = rv.SparseLDLT.analyze(rv.problems.shifted_laplacian(6, 0.1))
    step, calls = _window_step({4: 1.0, 8: 0.5}, {4: (1, 1, 0), 8: (1, 1, 0)})
    for base in (rv.FactorOptions(precision="fp64"), rv.FactorOptions(precision="mixed", mixed_flush=4)):
        best, _ = A.autotune(s, None, None, base, timer=lambda o: 1.0, device_name="g", step=step)
        assert best.mixed_window == 0
    assert calls == []
