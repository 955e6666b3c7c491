"""Host logic of the learned precision selector (no GPU): the generated
training family, the sample weights and the misprediction counts."""
import numpy as np


def test_c5_family_alternates_and_respects_ranges(rv):
    fam = rv.selector.c5_family(6, seed=3, grid_lo=6, grid_hi=9)
    assert len(fam) == 6
    for i, s in enumerate(fam):
        if i % 2 == 0:
            assert s.name.startswith("laplace7_")
            g = round(s.n ** (1 / 3))
            assert 6 <= g <= 9 and g ** 3 == s.n
            frac = float(s.name.split("shift")[1])
            assert 0.01 <= frac <= 0.20
            neg = s.inertia[1] / s.n
            assert 0.0 < neg <= 0.25
        else:
            assert s.name.startswith("kkt27_")
            assert s.inertia[2] == 0 and s.inertia[0] + s.inertia[1] == s.n
    again = rv.selector.c5_family(6, seed=3, grid_lo=6, grid_hi=9)
    assert [s.name for s in again] == [s.name for s in fam]
    assert all(np.array_equal(a.values, b.values) for a, b in zip(again, fam))


def test_sample_weights(rv):
    S = rv.selector
    X = np.zeros((4, S.NFEAT))
    X[:, 1] = [4, 4, 6, 6]  # log2 k
    d = S.Labelled(X, np.array([1.0, 1.0, 1.0, 0.0]), np.zeros(4), np.array([32.0, 32.0, 128.0, 128.0]))
    w0 = S.sample_weights(d, 0.0)
    # classes balanced: each class carries half the total weight
    assert np.isclose(w0[:3].sum(), w0[3]) and np.isclose(w0.sum(), 4.0)
    w1 = S.sample_weights(d, 0.5)
    cost = d.m * 2.0 ** X[:, 1]
    assert np.allclose(w1 / w0, (cost / cost.mean()) ** 0.5)


def test_misprediction_counts(rv):
    p = np.array([0.9, 0.2, 0.7, 0.4, 0.55])
    y = np.array([1.0, 1.0, 0.0, 0.0, 1.0])
    r = rv.selector.misprediction_of(p, 0.5, y)
    assert r == dict(fronts=5, safe=3, routed_mixed=3, unsafe_sent_mixed=1, safe_kept_fp64=1, rate=0.4)
    assert rv.selector.misprediction_of(np.zeros(0), 0.5, np.zeros(0))["fronts"] == 0
