"""The known-factorization fixtures (the reference's JSON layout,
sparse/src/io/reference.rs) read back with the same checks and errors, and
each published factorization reconstructing its matrix."""
import json

import numpy as np
import pytest


def dense(entry):
    n = entry["n"]
    A = np.zeros((n, n))
    for r, c, v in entry["entries"]:
        A[r, c] = v
        A[c, r] = v
    return A


def test_every_fixture_reconstructs_its_matrix(rv, golden):
    io = rv.reference_io
    assert len(golden) == 15
    for name, e in golden.items():
        ref = io.parse_reference(e["reference"], name)
        assert ref.matrix_name == name and ref.n == e["n"]
        A = dense(e)
        err = np.abs(ref.reconstruct() - A).max()
        assert err <= 1e-13 * max(np.abs(A).max(), 1.0), (name, err)
        assert [1 if np.ndim(b) == 0 else 2 for b in ref.d_blocks] == e["d_block_sizes"]
        assert ref.inertia == tuple(e["inertia"])
        assert ref.block_inertia() == tuple(e["inertia"]), name


def test_oracle_inertia_matches_the_published_factorizations(rv, orc, golden):
    io = rv.reference_io
    for name, e in golden.items():
        ref = io.parse_reference(e["reference"], name)
        s = rv.problems.from_scipy(name, __import__("scipy.sparse", fromlist=["csc_matrix"]).csc_matrix(dense(e)))
        solver = rv.SparseLDLT.analyze(s)
        f = orc.OracleFactor(s, solver.symbolic)
        assert f.inertia() == ref.inertia, name
        f.close()


def test_load_from_file_and_errors(rv, golden, tmp_path):
    io = rv.reference_io
    good = golden["arrow-5-pd"]["reference"]
    p = tmp_path / "arrow.json"
    p.write_text(json.dumps(good))
    ref = io.load_reference(p)
    assert ref.inertia == (5, 0, 0) and ref.l_rows.size == 10 and ref.n == 5
    assert all(np.ndim(b) == 0 for b in ref.d_blocks)
    with pytest.raises(rv.solver.IoError):
        io.load_reference(tmp_path / "missing.json")
    bad = tmp_path / "bad.json"
    bad.write_text("{ not valid json }")
    with pytest.raises(rv.solver.ParseError):
        io.load_reference(bad)

    def broken(**change):
        obj = json.loads(json.dumps(good))
        for k, v in change.items():
            obj[k] = v
        return obj
    cases = [
        broken(l_entries=[{"row": 1, "col": 1, "value": 1.0}]),           # not strictly lower
        broken(l_entries=[{"row": 0, "col": 3, "value": 1.0}]),
        broken(permutation=[0, 1, 1, 3, 4]),                              # repeated index
        broken(permutation=[0, 1, 2, 3, 9]),                              # out of range
        broken(d_blocks=[{"size": 3, "values": [1, 2, 3]}]),              # bad block size
        broken(d_blocks=[{"size": 1, "values": [1.0, 2.0]}]),
        broken(d_blocks=[{"size": 2, "values": [[1.0, 2.0]]}]),
        broken(d_blocks=[{"size": 2, "values": [[1.0, 2.0], [3.0]]}]),
        broken(d_blocks=[{"values": [1.0]}]),
        {k: v for k, v in good.items() if k != "permutation"},
    ]
    for obj in cases:
        with pytest.raises(rv.solver.ParseError):
            io.parse_reference(obj)


def write_mtx(path, e, header="%%MatrixMarket matrix coordinate real symmetric"):
    with open(path, "w") as f:
        f.write(header + "\n% a comment\n")
        f.write(f"{e['n']} {e['n']} {len(e['entries'])}\n")
        for r, c, v in e["entries"]:
            f.write(f"{r + 1} {c + 1} {v!r}\n")


def test_load_mtx_round_trip(rv, golden, tmp_path):
    io = rv.reference_io
    for name, e in golden.items():
        p = tmp_path / f"{name}.mtx"
        write_mtx(p, e)
        s = io.load_mtx(p)
        assert s.name == name and s.n == e["n"]
        A = dense(e)
        A[A == 0.0] = 0.0
        assert np.array_equal(s.to_scipy().toarray(), A), name


def test_load_mtx_errors(rv, tmp_path):
    io = rv.reference_io
    ok_head = "%%MatrixMarket matrix coordinate real symmetric\n"

    def load(text):
        p = tmp_path / "m.mtx"
        p.write_text(text)
        return io.load_mtx(p)
    s = load(ok_head + "3 3 4\n1 1 2.0\n2 1 0.0\n3 2 -1.5\n3 3 4.0\n")  # the explicit zero is dropped
    assert s.to_scipy().nnz == 4 and s.to_scipy()[1, 2] == -1.5 and s.to_scipy()[0, 1] == 0
    with pytest.raises(rv.solver.IoError):
        io.load_mtx(tmp_path / "none.mtx")
    bad = [("", 1), ("%%MatrixMarket matrix coordinate real general\n2 2 1\n1 1 1.0\n", 1),
           ("%%MatrixMarket matrix array real symmetric\n2 2\n1\n", 1),
           (ok_head + "% only comments\n", None),
           (ok_head + "2 2\n", 2), (ok_head + "2 x 1\n", 2),
           (ok_head + "2 2 1\n1 1\n", 3), (ok_head + "2 2 1\n0 1 1.0\n", 3),
           (ok_head + "2 2 1\n3 1 1.0\n", 3), (ok_head + "2 2 1\na 1 1.0\n", 3),
           (ok_head + "2 2 1\n1 1 nan?\n", 3)]
    for text, line in bad:
        with pytest.raises(rv.solver.ParseError) as ei:
            load(text)
        assert ei.value.line == line, (text, ei.value)
