"""Per-supernode statistics (SparseLDLT::per_supernode_stats) agree with the
aggregate FactorizationStats and with the oracle's fronts."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_per_supernode_stats_sum_to_the_totals(rv, orc):
    s = rv.problems.kkt(8, seed=2)
    solver = rv.SparseLDLT.analyze(s)
    assert solver.per_supernode_stats() is None
    solver.factor()
    ps = solver.per_supernode_stats()
    st = solver.stats()
    assert len(ps) == st["supernodes_after_amalgamation"]
    assert sum(p["num_1x1"] for p in ps) == st["total_1x1_pivots"]
    assert sum(p["num_2x2"] for p in ps) == st["total_2x2_pivots"]
    assert sum(p["num_delayed"] for p in ps) == st["total_delayed"]
    assert max(p["front_size"] for p in ps) == st["max_front_size"]
    assert all(p["num_eliminated"] + p["num_delayed"] == p["num_fully_summed"] for p in ps)
    ref = orc.OracleFactor(s, solver.symbolic)
    assert np.array_equal(solver.front_info()[:, :5], ref.front_info()[:, :5])
    ref.close()
    solver.close()
