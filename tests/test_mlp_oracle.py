"""The selector network's CPU oracle (oracle/mlp_oracle.py) pinned by
finite differences, and its layout against the library's."""
import numpy as np


def random_params(mo, seed=0):
    rng = np.random.default_rng(seed)
    p = rng.normal(0, 0.3, mo.NPARAM)
    p[mo.MU:mo.SD] = rng.normal(0, 1, mo.IN)
    p[mo.SD:] = rng.uniform(0.5, 2.0, mo.IN)
    return p


def test_layout_matches_library(rv, mlp_oracle):
    L = rv._native.lib()
    assert L.rvg_mlp_param_count() == mlp_oracle.NPARAM == 5081
    assert L.rvg_mlp_trained_count() == mlp_oracle.NTRAIN == 5057
    assert L.rvg_mlp_work_floats(10 ** 6) == 296 * (mlp_oracle.NTRAIN + 1)
    assert L.rvg_mlp_work_floats(1) == mlp_oracle.NTRAIN + 1


def test_gradient_matches_finite_differences(mlp_oracle):
    mo = mlp_oracle
    rng = np.random.default_rng(1)
    p = random_params(mo, 2)
    x = rng.normal(0, 1.5, (40, mo.IN))
    y = (rng.uniform(size=40) < 0.4).astype(float)
    w = rng.uniform(0.5, 2.0, 40)
    loss, g = mo.loss_grad(p, x, y, w, norm=w.sum())
    assert np.isclose(loss, mo.loss(p, x, y, w, norm=w.sum()))
    idx = np.concatenate([rng.choice(mo.NTRAIN, 60, replace=False), [mo.B3, mo.W3, mo.B1, mo.W1]])
    h = 1e-6
    for i in idx:
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (mo.loss(pp, x, y, w, norm=w.sum()) - mo.loss(pm, x, y, w, norm=w.sum())) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(g[i])), (i, fd, g[i])


def test_adam_step(mlp_oracle):
    mo = mlp_oracle
    p = random_params(mo, 3)
    g = np.linspace(-1, 1, mo.NTRAIN)
    p1, m1, v1 = mo.adam(p, g, np.zeros(mo.NTRAIN), np.zeros(mo.NTRAIN), 1, 0.01)
    # first step of Adam moves every parameter by lr * sign(g) (up to eps)
    d = p[:mo.NTRAIN] - p1[:mo.NTRAIN]
    nz = np.abs(g) > 1e-3
    assert np.allclose(d[nz], 0.01 * np.sign(g[nz]), rtol=1e-4)
    assert np.array_equal(p1[mo.NTRAIN:], p[mo.NTRAIN:])  # normalisation untouched
