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


def test_gradient_matches_torch_autograd(mlp_oracle):
    """The oracle's hand-written backward pass against torch autograd (float64, CPU)."""
    import torch
    mo = mlp_oracle
    rng = np.random.default_rng(11)
    p = random_params(mo, 12)
    x = rng.normal(0, 1.5, (300, mo.IN))
    y = (rng.uniform(size=300) < 0.4).astype(float)
    w = rng.uniform(0.5, 2.0, 300)
    loss, g = mo.loss_grad(p, x, y, w, norm=w.sum())
    P = torch.tensor(p, dtype=torch.float64, requires_grad=True)
    W1 = P[mo.W1:mo.B1].reshape(mo.H, mo.IN)
    W2 = P[mo.W2:mo.B2].reshape(mo.H, mo.H)
    xn = (torch.tensor(x) - P[mo.MU:mo.SD].detach()) / P[mo.SD:].detach()
    h1 = torch.relu(xn @ W1.T + P[mo.B1:mo.W2])
    h2 = torch.relu(h1 @ W2.T + P[mo.B2:mo.W3])
    z = h2 @ P[mo.W3:mo.B3] + P[mo.B3]
    lt = torch.sum(torch.tensor(w) * torch.nn.functional.binary_cross_entropy_with_logits(
        z, torch.tensor(y), reduction="none")) / float(w.sum())
    lt.backward()
    assert np.isclose(lt.item(), loss, rtol=1e-12)
    assert np.allclose(P.grad.numpy()[:mo.NTRAIN], g, rtol=1e-10, atol=1e-13)
    assert np.all(P.grad.numpy()[mo.NTRAIN:] == 0)  # the normalisation is not trained
