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
