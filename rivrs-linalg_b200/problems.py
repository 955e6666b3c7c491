"""Synthetic systems with exactly known inertia, and Matrix Market input.

The build has no network, so the workloads are generated, seeded:

* ``shifted_laplacian(g, frac)`` -- the 7-point Dirichlet Laplacian on a g^3
  grid (h = 1/(g+1)), A = L_h - sigma*I.  L_h's spectrum is closed form,
  ``(4/h^2) * (sin^2(i pi h/2) + sin^2(j pi h/2) + sin^2(k pi h/2))``, so the
  inertia is exact without an eigensolver.  sigma sits at the midpoint between
  the eigenvalue at the requested percentile and the next distinct one (grid
  eigenvalues repeat; a shift equal to one would make A singular).
* ``kkt(g, ...)`` -- [[H, J^T], [J, 0]] with H the 27-point Laplacian (26 on
  the diagonal, -1 to each of the 26 neighbours, Dirichlet) plus
  diag(U[0, 1e-2]), and J of m = n_H/4 rows with 4 N(0,1) entries at distinct
  seeded random columns.  H is SPD and J has full row rank (checked
  structurally by a bipartite matching), so the inertia is exactly
  (n_H, m, 0).

Matrices are returned as full symmetric CSC (both triangles), the input
convention of rivrs-sparse (sparse/src/lib.rs:121-125).
"""
from __future__ import annotations

import dataclasses

import numpy as np
import scipy.sparse as sp


@dataclasses.dataclass
class System:
    name: str
    n: int
    colptr: np.ndarray  # int64, n+1
    rowidx: np.ndarray  # int64
    values: np.ndarray  # float64
    inertia: tuple | None = None  # (positive, negative, zero) when known exactly
    grid: tuple | None = None  # grid dimensions for geometric orderings
    n_h: int = 0  # KKT: number of H rows (constraints follow)
    meta: dict = dataclasses.field(default_factory=dict)

    def to_scipy(self) -> sp.csc_matrix:
        return sp.csc_matrix((self.values, self.rowidx, self.colptr), shape=(self.n, self.n))


def from_scipy(name, a, **kw) -> System:
    a = sp.csc_matrix(a)
    a.sum_duplicates()
    a.sort_indices()
    return System(name=name, n=a.shape[0], colptr=a.indptr.astype(np.int64), rowidx=a.indices.astype(np.int64),
                  values=a.data.astype(np.float64), **kw)


def laplacian_eigenvalues(g: int) -> np.ndarray:
    h = 1.0 / (g + 1)
    s = (4.0 / h ** 2) * np.sin(np.arange(1, g + 1) * np.pi * h / 2) ** 2
    return (s[:, None, None] + s[None, :, None] + s[None, None, :]).ravel()


def laplacian_7pt(g: int) -> sp.csc_matrix:
    h = 1.0 / (g + 1)
    e = np.ones(g)
    t = sp.diags([-e[:-1], 2 * e, -e[:-1]], [-1, 0, 1])
    i = sp.identity(g)
    lap = sp.kron(sp.kron(t, i), i) + sp.kron(sp.kron(i, t), i) + sp.kron(sp.kron(i, i), t)
    return (lap / h ** 2).tocsc()


def shifted_laplacian(g: int, frac: float = 0.10) -> System:
    """A = L_h - sigma*I with about `frac` of the eigenvalues negative."""
    lam = np.sort(laplacian_eigenvalues(g))
    n = lam.size
    q = max(int(np.floor(frac * n)) - 1, 0)
    lo = lam[q]
    above = lam[lam > lo * (1 + 1e-12) + 1e-300]
    hi = above[0] if above.size else lo * 2
    sigma = 0.5 * (lo + hi)
    neg = int(np.count_nonzero(lam < sigma))
    a = laplacian_7pt(g) - sigma * sp.identity(n)
    sysm = from_scipy(f"laplace7_{g}^3_shift{frac:g}", a, inertia=(n - neg, neg, 0), grid=(g, g, g))
    sysm.meta.update(sigma=float(sigma), frac=frac)
    return sysm


def laplacian_27pt(g: int) -> sp.csc_matrix:
    idx = np.arange(g ** 3).reshape(g, g, g)
    rows, cols = [], []
    for dx in (-1, 0, 1):
        for dy in (-1, 0, 1):
            for dz in (-1, 0, 1):
                if dx == dy == dz == 0:
                    continue
                sx = slice(max(dx, 0), g + min(dx, 0))
                sy = slice(max(dy, 0), g + min(dy, 0))
                sz = slice(max(dz, 0), g + min(dz, 0))
                tx = slice(max(-dx, 0), g + min(-dx, 0))
                ty = slice(max(-dy, 0), g + min(-dy, 0))
                tz = slice(max(-dz, 0), g + min(-dz, 0))
                rows.append(idx[sx, sy, sz].ravel())
                cols.append(idx[tx, ty, tz].ravel())
    r = np.concatenate(rows)
    c = np.concatenate(cols)
    n = g ** 3
    off = sp.csc_matrix((-np.ones(r.size), (r, c)), shape=(n, n))
    return (off + 26.0 * sp.identity(n)).tocsc()


def kkt(g: int, rows_per_h: float = 0.25, nnz_per_row: int = 4, seed: int = 0, reg_hi: float = 1e-2) -> System:
    """Saddle-point [[H, J^T], [J, 0]] with exactly known inertia (n_H, m, 0)."""
    rng = np.random.default_rng(seed)
    nh = g ** 3
    m = int(round(rows_per_h * nh))
    h = laplacian_27pt(g) + sp.diags(rng.uniform(0.0, reg_hi, nh))
    cols = np.empty((m, nnz_per_row), dtype=np.int64)
    for i in range(m):
        cols[i] = rng.choice(nh, size=nnz_per_row, replace=False)
    vals = rng.standard_normal((m, nnz_per_row))
    j = sp.csr_matrix((vals.ravel(), cols.ravel(), np.arange(0, m * nnz_per_row + 1, nnz_per_row)), shape=(m, nh))
    from scipy.sparse.csgraph import maximum_bipartite_matching
    match = maximum_bipartite_matching(j.tocsr(), perm_type="column")
    if np.count_nonzero(match >= 0) != m:
        raise RuntimeError("constraint block is structurally rank deficient; change the seed")
    a = sp.bmat([[h, j.T], [j, None]], format="csc")
    return from_scipy(f"kkt27_{g}^3_m{m}", a, inertia=(nh, m, 0), grid=(g, g, g), n_h=nh,
                      meta=dict(m=m, seed=seed))


def read_mtx(path: str) -> System:
    """Matrix Market coordinate reader; symmetric files are mirrored."""
    with open(path) as f:
        header = f.readline().lower().split()
        symmetric = "symmetric" in header
        pattern = "pattern" in header
        line = f.readline()
        while line.startswith("%"):
            line = f.readline()
        nr, nc, nz = (int(x) for x in line.split())
        data = np.loadtxt(f, ndmin=2) if nz else np.zeros((0, 3))
    r = data[:, 0].astype(np.int64) - 1
    c = data[:, 1].astype(np.int64) - 1
    v = np.ones(r.size) if pattern else data[:, 2].astype(np.float64)
    if symmetric:
        off = r != c
        r, c, v = np.concatenate([r, c[off]]), np.concatenate([c, r[off]]), np.concatenate([v, v[off]])
    a = sp.csc_matrix((v, (r, c)), shape=(nr, nc))
    return from_scipy(path.rsplit("/", 1)[-1].replace(".mtx", ""), a)


def batch_family(count: int = 64, seed: int = 1, n_lo: float = 5e3, n_hi: float = 2e5,
                 max_rhs: int = 32) -> list:
    """The many-systems workload: `count` systems with sizes drawn
    log-uniform in [n_lo, n_hi] from `seed`; even slots are shifted 7-point
    Laplacians (10% negative eigenvalues, g^3 nearest the drawn size), odd
    slots KKT systems as kkt() (1.25 g^3 nearest the drawn size, seeded per
    slot); each slot also draws its number of right-hand sides in
    [1, max_rhs].  Returns [(System, nrhs)]."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = float(np.exp(rng.uniform(np.log(n_lo), np.log(n_hi))))
        nrhs = int(rng.integers(1, max_rhs + 1))
        if i % 2 == 0:
            s = shifted_laplacian(max(2, int(round(n ** (1.0 / 3.0)))), 0.10)
        else:
            s = kkt(max(4, int(round((n / 1.25) ** (1.0 / 3.0)))), seed=seed * 1000 + i)
        out.append((s, nrhs))
    return out


def block_diagonal(systems, name: str = "batch") -> System:
    """One system holding `systems` as its diagonal blocks, in order.  Its
    values are the blocks' values concatenated (column-major CSC keeps each
    block's columns, and their entries, contiguous); meta['offsets'] holds the
    first index of each block (and n), meta['parts'] the systems."""
    a = sp.block_diag([s.to_scipy() for s in systems], format="csc")
    inert = None
    if all(s.inertia is not None for s in systems):
        inert = tuple(int(sum(s.inertia[k] for s in systems)) for k in range(3))
    out = from_scipy(name, a, inertia=inert)
    if not np.array_equal(out.values, np.concatenate([s.values for s in systems])):
        raise RuntimeError("block values are not contiguous")
    out.meta.update(offsets=np.cumsum([0] + [s.n for s in systems]).astype(np.int64), parts=list(systems))
    return out


def perturb_symmetric(sysm: System, rel: float = 0.01, seed: int = 0) -> np.ndarray:
    """Values of sysm scaled entrywise by 1 + rel * N(0,1), the two stored
    copies (i, j) and (j, i) of an off-diagonal entry by the same factor, so
    the matrix stays symmetric."""
    rng = np.random.default_rng(seed)
    col = np.repeat(np.arange(sysm.n, dtype=np.int64), np.diff(sysm.colptr))
    row = sysm.rowidx
    key = np.minimum(row, col) * np.int64(sysm.n) + np.maximum(row, col)
    uniq, inv = np.unique(key, return_inverse=True)
    f = 1.0 + rel * rng.standard_normal(uniq.size)
    return sysm.values * f[inv]


def rhs_uniform(n: int, seed: int = 0, nrhs: int = 1) -> np.ndarray:
    rng = np.random.default_rng(seed)
    b = rng.uniform(-1.0, 1.0, (nrhs, n))
    return b[0].copy() if nrhs == 1 else np.asfortranarray(b.T)


def rhs_normal(n: int, seed: int = 0, nrhs: int = 1) -> np.ndarray:
    rng = np.random.default_rng(seed)
    b = rng.standard_normal((nrhs, n))
    return b[0].copy() if nrhs == 1 else np.asfortranarray(b.T)


def backward_error(sysm: System, x: np.ndarray, b: np.ndarray) -> float:
    """||Ax - b||_2 / (||A||_F ||x||_2 + ||b||_2)  (sparse/src/validate.rs:209-258)."""
    a = sysm.to_scipy()
    r = a @ x - b
    anorm = np.sqrt(np.sum(sysm.values ** 2))
    denom = anorm * np.linalg.norm(x) + np.linalg.norm(b)
    return 0.0 if denom == 0 else float(np.linalg.norm(r) / denom)
