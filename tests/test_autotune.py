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
