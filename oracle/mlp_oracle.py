"""CPU oracle of the per-front precision selector's network (test
infrastructure only: tests and the bench's checks import it, the product
path never does).

The selector has no counterpart in the reference crate, so there is no
reference file to cite: this is the textbook computation of a 12-64-64-1
perceptron (ReLU hidden layers, sigmoid output) and of the gradient of the
weighted binary cross-entropy by backpropagation, in float64, on the same
flat parameter layout as the CUDA kernels (`rivrs-linalg_b200/csrc/mlp.cuh`):
W1 (64 x 12, row major), b1 (64), W2 (64 x 64), b2 (64), W3 (64), b3 (1),
then the input normalisation (mean and standard deviation per feature).
It is pinned by finite differences (`tests/test_mlp_oracle.py`); the GPU
kernels are checked against it within float32 tolerances.
"""
import numpy as np

IN, H = 12, 64
W1, B1 = 0, H * IN
W2 = B1 + H
B2 = W2 + H * H
W3 = B2 + H
B3 = W3 + H
NTRAIN = B3 + 1
MU = NTRAIN
SD = MU + IN
NPARAM = SD + IN


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    return (p[W1:B1].reshape(H, IN), p[B1:W2], p[W2:B2].reshape(H, H), p[B2:W3], p[W3:B3], p[B3],
            p[MU:SD], p[SD:NPARAM])


def forward(p, x):
    """Logits z (n,) and the activations, for raw features x (n, 12)."""
    w1, b1, w2, b2, w3, b3, mu, sd = unpack(p)
    xn = (np.asarray(x, np.float64) - mu) / sd
    z1 = xn @ w1.T + b1
    h1 = np.maximum(z1, 0.0)
    z2 = h1 @ w2.T + b2
    h2 = np.maximum(z2, 0.0)
    z = h2 @ w3 + b3
    return z, (xn, z1, h1, z2, h2)


def sigmoid(z):
    z = np.asarray(z, np.float64)
    out = np.empty_like(z)
    pos = z >= 0
    out[pos] = 1.0 / (1.0 + np.exp(-z[pos]))
    e = np.exp(z[~pos])
    out[~pos] = e / (1.0 + e)
    return out


def loss(p, x, y, w=None, norm=None):
    z, _ = forward(p, x)
    y = np.asarray(y, np.float64)
    w = np.ones_like(y) if w is None else np.asarray(w, np.float64)
    norm = float(y.size) if norm is None else float(norm)
    sp = np.maximum(z, 0.0) + np.log1p(np.exp(-np.abs(z)))
    return float(np.sum(w * (sp - y * z)) / norm)


def loss_grad(p, x, y, w=None, norm=None):
    """(loss, gradient of the trained parameters (NTRAIN,)) of
    sum_i w_i (softplus(z_i) - y_i z_i) / norm."""
    z, (xn, z1, h1, z2, h2) = forward(p, x)
    w1, b1, w2, b2, w3, b3, mu, sd = unpack(p)
    y = np.asarray(y, np.float64)
    w = np.ones_like(y) if w is None else np.asarray(w, np.float64)
    norm = float(y.size) if norm is None else float(norm)
    dz = w * (sigmoid(z) - y) / norm
    g = np.zeros(NTRAIN)
    g[B3] = dz.sum()
    g[W3:B3] = h2.T @ dz
    d2 = np.outer(dz, w3) * (z2 > 0)
    g[B2:W3] = d2.sum(0)
    g[W2:B2] = (d2.T @ h1).ravel()
    d1 = (d2 @ w2) * (z1 > 0)
    g[B1:W2] = d1.sum(0)
    g[W1:B1] = (d1.T @ xn).ravel()
    sp = np.maximum(z, 0.0) + np.log1p(np.exp(-np.abs(z)))
    return float(np.sum(w * (sp - y * z)) / norm), g


def adam(p, g, m, v, step, lr, b1=0.9, b2=0.999, eps=1e-8, wd=0.0):
    """One Adam step with decoupled weight decay on the trained part; returns (p, m, v)."""
    p = np.array(p, np.float64)
    m = b1 * np.asarray(m, np.float64) + (1 - b1) * g
    v = b2 * np.asarray(v, np.float64) + (1 - b2) * g * g
    mh, vh = m / (1 - b1 ** step), v / (1 - b2 ** step)
    p[:NTRAIN] -= lr * (mh / (np.sqrt(vh) + eps) + wd * p[:NTRAIN])
    return p, m, v
