"""Autotuner host logic: candidate sets and pattern fingerprints (no GPU)."""


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
